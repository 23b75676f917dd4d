import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

PKG = __graft_entry__.load_package()
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built engine library")


@pytest.fixture(scope="session")
def pkg():
    return PKG


def oracle_settings(S, tol=1e-10, predictor=0, peek=0.0, ke=None, polarizable=True):
    from oracle import pgm_oracle as O
    return O.Settings(cutoff=float(S.cutoff), beta=float(S.beta), grid=tuple(int(g) for g in S.grid), order=int(S.order),
                      tol=tol, max_iter=1000, peek=peek, predictor=predictor,
                      ke=PKG.systems.KE_DEFAULT if ke is None else ke, polarizable=polarizable)


def oracle_topology(S):
    from oracle import pgm_oracle as O
    return O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)


def load_golden_system(name):
    d = np.load(GOLDEN / f"ref_{name}.npz")
    S = PKG.systems.System(name=name, pos=d["pos"], box=d["box"], q=d["q"], radius=d["radius"], alpha=d["alpha"],
                           cov_atom=d["cov_atom"], cov_partner=d["cov_partner"], cov_strength=d["cov_strength"],
                           cutoff=float(d["cutoff"]), beta=float(d["beta"]), grid=tuple(int(g) for g in d["grid"]),
                           order=int(d["order"]))
    return S, d


def load_dmp_real():
    """The reference's real 8550-atom dimethylphenol liquid with pgm_core's outputs (tests/golden/dmp8550_real.npz):
    (System, fixture).  The molecule's parameters are tiled by the generator's own function."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("pgm_b200_make_golden", GOLDEN / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = np.load(GOLDEN / "dmp8550_real.npz")
    mol = {k[4:]: d[k] for k in d.files if k.startswith("mol_")}
    return mg.dmp_system(mol, d["pos"], d["box"], PKG.systems), d
