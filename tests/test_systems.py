"""The seeded synthetic workloads: sizes, units and determinism."""

import numpy as np

from conftest import PKG


def test_water216():
    S = PKG.systems.water216()
    assert S.n == 648 and len(S.cov_atom) == 432
    assert np.allclose(S.box, np.eye(3) * 1.864)
    assert S.grid == (20, 20, 20) and abs(S.beta - 3.5) < 1e-12 and abs(S.cutoff - 0.9) < 1e-12
    d = np.linalg.norm(S.pos[1::3] - S.pos[0::3], axis=1)
    assert np.allclose(d, 0.09572)
    assert abs(S.q.sum()) < 1e-12


def test_dimethylphenol8550():
    S = PKG.systems.dimethylphenol8550()
    assert S.n == 8550 and len(S.cov_atom) == 8550
    assert S.grid == (48, 48, 48)
    mol = S.q.reshape(450, 19).sum(axis=1)
    assert np.abs(mol).max() < 1e-12
    R = S.radius[:19] * 10
    assert R.min() >= 0.7 and R.max() <= 1.1
    S2 = PKG.systems.dimethylphenol8550()
    assert np.array_equal(S.pos, S2.pos)


def test_water_batch():
    B = PKG.systems.water_batch(nsys=16, seed=3)
    assert len(B) == 16
    for S in B:
        L = S.box[0, 0]
        assert abs(S.cutoff - min(0.9, L / 2)) < 1e-12
        assert S.grid[0] >= 6 and S.n % 3 == 0
