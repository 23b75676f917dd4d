"""CUDA engine against the FP64 oracle, through the C ABI, on cuda:0.

Tolerances (stated per test): the FP64 path within 1e-7 relative in every energy term and 1e-6 relative
RMS in forces (the reference's bar for pgm_core parity); the mixed path within 1e-5 relative RMS in forces
against the FP64 oracle at tol 1e-10, the pair set bit-exact in both.
"""

import numpy as np
import pytest

from conftest import GOLDEN, PKG, load_dmp_real, load_golden_system, oracle_settings, oracle_topology
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu

TERMS = ("direct", "reciprocal", "self", "background", "polarization")


def make_engine(S, precision, tol=1e-10, predictor=0, peek=0.0, ke=None, **kw):
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=tol, max_iter=1000,
                                  peek=peek, predictor=predictor, ke=PKG.systems.KE_DEFAULT if ke is None else ke,
                                  precision=precision, **kw))
    eng.set_system(S)
    return eng


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", ["tiny_triclinic", "water216"])
def test_fp64_matches_reference_outputs(name):
    S, d = load_golden_system(name)
    eng = make_engine(S, PKG.FP64)
    r = eng.compute(S.pos, S.box)
    t = r.terms.as_dict()
    for k, nm in enumerate(TERMS):
        assert abs(t[nm] - d["terms"][k]) <= 1e-7 * max(abs(d["terms"][k]), 1e-3), nm
    assert abs(r.energy - float(d["energy"])) <= 1e-9 * abs(float(d["energy"]))
    assert rel_rms(r.forces, d["forces"]) <= 1e-6
    assert np.abs(r.strain - d["strain"]).max() <= 1e-6 * np.abs(d["strain"]).max()
    assert np.abs(eng.induced_dipoles() - d["mu"]).max() <= 1e-6 * np.abs(d["mu"]).max()
    assert np.abs(eng.permanent_dipoles() - d["perm"]).max() <= 1e-12


@pytest.mark.parametrize("name", ["tiny_triclinic", "water216"])
def test_mixed_matches_reference_outputs(name):
    S, d = load_golden_system(name)
    eng = make_engine(S, PKG.MIXED)
    r = eng.compute(S.pos, S.box)
    assert abs(r.energy - float(d["energy"])) <= 1e-6 * abs(float(d["energy"]))
    assert rel_rms(r.forces, d["forces"]) <= 1e-5
    assert np.abs(r.strain - d["strain"]).max() <= 1e-5 * np.abs(d["strain"]).max()


@pytest.mark.parametrize("name", ["tiny_triclinic", "water216"])
@pytest.mark.parametrize("precision", [0, 1])
def test_pair_set_bit_exact(name, precision):
    S, _ = load_golden_system(name)
    eng = make_engine(S, precision)
    eng.compute(S.pos, S.box)
    gi, gj = eng.pairs()
    oi, oj, _ = O.pair_set(S.pos, S.box, S.cutoff)
    assert np.array_equal(gi, oi) and np.array_equal(gj, oj)
    assert eng.num_candidates() == 2 * len(oi)


def test_pair_set_knife_edge_and_far_images():
    """Pairs at r == rc exactly are out, one ulp inside in; positions many boxes away from the primary cell
    and a triclinic box give the reference's minimum image."""
    rng = np.random.default_rng(1)
    S = PKG.systems.tiny_triclinic(nmol=10, seed=4)
    rc = S.cutoff
    pos = S.pos.copy()
    pos[1] = pos[0] + np.array([rc, 0.0, 0.0])
    pos[2] = pos[0] + np.array([0.0, np.nextafter(rc, 0), 0.0])
    pos[5:] += np.round(rng.uniform(-3, 3, (len(pos) - 5, 1))) * S.box[2]   # far images along c
    for prec in (0, 1):
        eng = make_engine(S, prec)
        eng.compute(pos, S.box)
        gi, gj = eng.pairs()
        oi, oj, _ = O.pair_set(pos, S.box, rc)
        assert np.array_equal(gi, oi) and np.array_equal(gj, oj)


@pytest.mark.parametrize("level", ["q", "qp", "qi", "qpi"])
def test_fp64_matches_pgmjax_goldens(level):
    g = np.load(GOLDEN / "w512_pgmjax.npz")
    cs = g["cov_strength"] if "p" in level else 0 * g["cov_strength"]
    eng = PKG.Engine(PKG.Settings(cutoff=float(g["cutoff"]), beta=float(g["beta"]), grid=tuple(g["grid"]),
                                  order=int(g["order"]), tol=float(g["tol"]), max_iter=1000, peek=0.0, predictor=0,
                                  ke=float(g["ke"]), precision=PKG.FP64, polarizable="i" in level))
    eng.set_atoms(g["q"], g["radius"], g["alpha"])
    eng.set_covalent(g["cov_atom"], g["cov_partner"], cs)
    r = eng.compute(g["pos"], g["H"])
    e = float(g[f"{level}_energy"])
    assert abs(r.energy - e) <= 1e-7 * abs(e)
    assert rel_rms(r.forces, g[f"{level}_forces"]) <= 1e-6
    if "i" in level:
        assert np.abs(eng.induced_dipoles() - g[f"{level}_mu"]).max() <= 1e-6 * np.abs(g[f"{level}_mu"]).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_real_dmp_liquid_matches_reference(precision):
    """The reference's real 8550-atom dimethylphenol liquid (amber/test/dmp) with the benchmark's settings against
    pgm_core at tol 1e-10 (tests/golden/dmp8550_real.npz): FP64 within 1e-7 relative in energy and 1e-6 relative
    RMS in forces, mixed within 1e-6 and 1e-5; induced dipoles alike."""
    S, d = load_dmp_real()
    eng = make_engine(S, precision)
    r = eng.compute(S.pos, S.box)
    e = float(d["energy"])
    lim_e, lim_f = (1e-7, 1e-6) if precision == 0 else (1e-6, 1e-5)
    assert abs(r.energy - e) <= lim_e * abs(e)
    assert rel_rms(r.forces, d["forces"].astype(np.float64)) <= lim_f
    mu = d["mu"].astype(np.float64)
    assert np.abs(eng.induced_dipoles() - mu).max() <= 10 * lim_f * np.abs(mu).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_field_matches_oracle(precision):
    S = PKG.systems.tiny_triclinic(nmol=20, seed=9)
    rng = np.random.default_rng(2)
    q = rng.normal(0, 0.5, S.n)
    d = rng.normal(0, 0.01, (S.n, 3))
    eng = make_engine(S, precision)
    E = eng.field(S.pos, S.box, q, d)
    ora = O.Engine(oracle_topology(S), oracle_settings(S))
    ora.set_geometry(S.pos, S.box)
    Eo = ora.field(q, d)
    assert rel_rms(E, Eo) <= (1e-12 if precision == 0 else 2e-6)


@pytest.mark.parametrize("precision", [0, 1])
def test_predictor_history_over_steps(precision):
    """mu4 predictor over moved steps (the reference harness core/cuda/tests/test_cuda.cpp:300-341): energies
    track the oracle at tol 1e-10 within 1e-6 relative; a repeated evaluation (new_step False) reuses the guess."""
    S = PKG.systems.tiny_triclinic(nmol=20, seed=13)
    eng = make_engine(S, precision, predictor=2)
    rng = np.random.default_rng(11)
    phase = rng.uniform(0, 2 * np.pi, S.pos.shape)
    its = []
    for step in range(8):   # smooth motion, as in MD (amplitude 0.01 nm, period 100 steps)
        pos = S.pos + 0.01 * np.sin(2 * np.pi * step / 100 + phase)
        r = eng.compute(pos, S.box, new_step=True)
        ora = O.Engine(oracle_topology(S), oracle_settings(S))
        e = ora.compute(pos, S.box)
        assert abs(r.energy - e) <= 1e-6 * abs(e)
        its.append(r.iterations)
    assert its[-1] < its[0]   # the extrapolation saves iterations
    # a repeated evaluation of the same step starts from that step's solution (FP64: already converged; the
    # mixed path's FP32 matvec cannot hold a residual of 1e-10, so it only starts far ahead)
    limit = 1 if precision == 0 else its[0] // 2
    again = eng.compute(pos, S.box, new_step=False)
    assert again.iterations <= limit
    blob = eng.get_history()
    eng.reset_history()
    eng.set_history(blob)
    assert eng.compute(pos, S.box, new_step=False).iterations <= limit


def test_compute_f_and_device_paths():
    """computeF (float positions) and launchDevice into a 64-bit fixed-point force buffer (OpenMM's layout,
    x at i, y at i + stride, z at i + 2 stride, scale 2^32) give the forces of compute()."""
    import torch
    S = PKG.systems.tiny_triclinic(nmol=20, seed=17)
    pf = S.pos.astype(np.float32)
    eng = make_engine(S, PKG.FP64)
    r = eng.compute(pf.astype(np.float64), S.box)
    rf = eng.compute_f(pf, S.box)
    assert abs(rf.energy - r.energy) <= 1e-12 * abs(r.energy)
    assert rel_rms(rf.forces, r.forces) <= 1e-12
    dev = torch.device("cuda:0")
    posq = torch.zeros((S.n, 4), dtype=torch.float32, device=dev)
    posq[:, :3] = torch.from_numpy(pf).to(dev)
    stride = ((S.n + 31) // 32) * 32
    fixed = torch.zeros(3 * stride, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    eng.launch_device(posq.data_ptr(), S.box, True, fixed.data_ptr(), stride, 2.0 ** 32, stream.cuda_stream)
    valid, t = eng.finish_device()
    assert valid
    torch.cuda.synchronize()
    f = fixed.cpu().numpy().astype(np.float64) / 2.0 ** 32
    F = np.stack([f[:S.n], f[stride:stride + S.n], f[2 * stride:2 * stride + S.n]], axis=1)
    assert abs(t.total() - r.energy) <= 1e-12 * abs(r.energy)
    assert rel_rms(F, r.forces) <= 1e-8   # 2^-32 resolution of the fixed-point buffer
    # device-resident double path
    pd = torch.from_numpy(pf.astype(np.float64)).to(dev).contiguous()
    fo = torch.zeros((S.n, 3), dtype=torch.float64, device=dev)
    eng.launch_resident(pd.data_ptr(), S.box, True, fo.data_ptr(), stream.cuda_stream)
    valid, t2 = eng.finish_device()
    torch.cuda.synchronize()
    assert abs(t2.total() - r.energy) <= 1e-12 * abs(r.energy)
    assert rel_rms(fo.cpu().numpy(), r.forces) <= 1e-12


def test_repeatable_bits():
    """The same evaluation twice gives the same bits (deterministic reductions, fixed list order)."""
    S = PKG.systems.water216()
    eng = make_engine(S, PKG.FP64)
    a = eng.compute(S.pos, S.box)
    b = eng.compute(S.pos, S.box)
    assert a.energy == b.energy
    assert np.array_equal(a.forces, b.forces) or rel_rms(a.forces, b.forces) < 1e-14


@pytest.mark.parametrize("mode", [0, 3, 4])
def test_mixed_repeatable_bits(mode):
    """Mixed precision repeats bit for bit: the spread adds 64-bit fixed-point contributions (integer sums do not
    depend on the atomics' order) and every other sum has a fixed order.  The real 8550-atom liquid, cuFFT
    (transforms 0, a conversion kernel before the transforms), the grid kernel (3, the conversion on its load) and
    the persistent CG kernel (4, its own spread and gather phases), three evaluations each, and a new engine on
    the same input."""
    S, _ = load_dmp_real()
    runs = []
    for _ in range(2):
        eng = make_engine(S, PKG.MIXED, tol=1e-5, peek=0.65)
        eng.set_transforms(mode)
        assert eng.transforms() == mode
        for _ in range(3):
            r = eng.compute(S.pos, S.box)
            runs.append((r.energy, r.forces.copy(), eng.induced_dipoles().copy(), r.iterations))
        eng.close()
    e0, f0, mu0, it0 = runs[0]
    for e, f, mu, it in runs[1:]:
        assert e == e0 and it == it0
        assert np.array_equal(f, f0)
        assert np.array_equal(mu, mu0)


def test_errors_are_status_codes():
    S = PKG.systems.tiny_triclinic(nmol=4, seed=1)
    eng = make_engine(S, PKG.FP64)
    bad = S.pos.copy()
    bad[0, 0] = np.nan
    with pytest.raises(PKG.PgmArgumentError, match="non-finite"):
        eng.compute(bad, S.box)
    with pytest.raises(PKG.PgmArgumentError, match="reduced"):
        eng.compute(S.pos, np.array([[2.0, 0.1, 0], [0, 2, 0], [0, 0, 2]]))
    with pytest.raises(PKG.PgmArgumentError):
        eng.set_covalent([0], [0], [0.1])
    r = eng.compute(S.pos, S.box)   # still usable
    assert np.isfinite(r.energy)


def test_mixed_fp64_refinement():
    """The mixed path with FP64 iterative refinement: the induced dipoles reach the FP64 oracle's (tol 1e-10)
    to 1e-8 relative, where the plain mixed path stops near its FP32 operator's accuracy; forces stay within the
    mixed bar (their final pass is FP32)."""
    S, d = load_golden_system("water216")
    plain = make_engine(S, PKG.MIXED)
    rp = plain.compute(S.pos, S.box)
    err_plain = np.abs(plain.induced_dipoles() - d["mu"]).max() / np.abs(d["mu"]).max()
    ref = make_engine(S, PKG.MIXED, refine=True)
    rr = ref.compute(S.pos, S.box)
    err_ref = np.abs(ref.induced_dipoles() - d["mu"]).max() / np.abs(d["mu"]).max()
    assert err_ref <= 1e-8 and err_ref < err_plain / 10, (err_plain, err_ref)
    assert abs(rr.energy - float(d["energy"])) <= 1e-7 * abs(float(d["energy"]))
    assert rel_rms(rr.forces, d["forces"]) <= 1e-5


@pytest.mark.parametrize("order", [4, 5, 7, 8])
def test_other_spline_orders(order):
    """Spline orders other than 6: the kernels with the order as a compile-time constant (4, 5, 8) and with the
    order at run time (7) against the oracle (FP64: 1e-7 energy, 1e-6 forces)."""
    S = PKG.systems.tiny_triclinic(nmol=16, seed=21)
    S.order = order
    eng = make_engine(S, PKG.FP64)
    r = eng.compute(S.pos, S.box)
    ora = O.Engine(oracle_topology(S), oracle_settings(S))
    e = ora.compute(S.pos, S.box)
    assert abs(r.energy - e) <= 1e-7 * abs(e)
    assert rel_rms(r.forces, ora.forces) <= 1e-6

