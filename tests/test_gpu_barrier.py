"""The failure path of the grid transforms' barriers, exercised without a GPU fault: a block waits at a barrier
that expects one block more than the launch has, so nothing ever ends its wait.  The wait gives up after its
bounded number of polls (about a second), sets the error flag the host reads, and returns; the context stays
usable and the next evaluation is correct."""

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu


def test_grid_barrier_wait_gives_up_and_reports():
    S = PKG.systems.water216()
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-8,
                                  precision=PKG.FP64))
    eng.set_system(S)
    before = eng.compute(S.pos, S.box).energy
    gave_up, seconds = eng.probe_barrier_timeout()
    assert gave_up
    assert 1e-3 < seconds < 10.0
    after = eng.compute(S.pos, S.box).energy
    assert np.isfinite(after) and abs(after - before) <= 1e-12 * abs(before)
