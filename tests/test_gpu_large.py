"""Full-size checks on the 98304-atom water box (104^3 grid) through size-independent properties: the pair set
bit-exact against the oracle's exact test (candidates from a cell grid), the mixed path against the FP64 path,
and invariance of the direct-space energy and the pair set under a rigid translation."""

import numpy as np
import pytest

from conftest import PKG
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    return PKG.systems.water98304(tol=1e-6)


def engine(S, precision):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-6, max_iter=300, peek=0.0,
                                predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    e.set_system(S)
    return e


def test_large_pair_set_bit_exact(big):
    e = engine(big, PKG.FP64)
    r = e.compute(big.pos, big.box)
    gi, gj = e.pairs()
    oi, oj = O.pair_set_cells(big.pos, big.box, big.cutoff)
    assert np.array_equal(gi, oi) and np.array_equal(gj, oj)
    # rigid translation: the same pair set; energies change only through PME's grid aliasing (which moves the
    # induced dipoles slightly, and with them the direct term)
    shift = np.array([0.1234, 0.4567, 0.7891])
    r2 = e.compute(big.pos + shift, big.box)
    ti, tj = e.pairs()
    assert np.array_equal(ti, gi) and np.array_equal(tj, gj)
    assert abs(r2.terms.direct - r.terms.direct) <= 1e-7 * abs(r.terms.direct)
    assert abs(r2.energy - r.energy) <= 1e-6 * abs(r.energy)


def test_large_mixed_vs_fp64(big):
    a = engine(big, PKG.FP64).compute(big.pos, big.box)
    b = engine(big, PKG.MIXED).compute(big.pos, big.box)
    assert abs(a.energy - b.energy) <= 1e-6 * abs(a.energy)
    assert np.linalg.norm(a.forces - b.forces) <= 1e-5 * np.linalg.norm(a.forces)
    assert np.abs(a.strain - b.strain).max() <= 1e-5 * np.abs(a.strain).max()
