"""Python surface of the pgm_b200 engine over its C ABI.

``Engine`` mirrors the reference GPU engine ``pgmcuda::Engine`` (core/cuda/pgm_cuda.h:47-127 of
larryhuang98/pGM-MD): same settings, same call sequence (set_atoms, set_covalent, compute), same semantics
of ``new_step`` and of the predictor history, same getters; errors raise ``PgmError`` (``PgmArgumentError``
for what the reference rejects with std::invalid_argument).  Units: nm, e, e nm, nm^3, kJ/mol.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

FP64, MIXED = 0, 1


class PgmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class PgmArgumentError(PgmError, ValueError):
    pass


def _check(rc):
    if rc != 0:
        msg = _lib.load().pgm_last_error().decode()
        raise (PgmArgumentError if rc == -1 else PgmError)(rc, msg)


def _d(a):
    return a.ctypes.data_as(_lib.P_D) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_lib.P_I) if a is not None else None


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


@dataclass
class Settings:
    """pgmcuda::Settings (core/cuda/pgm_cuda.h:25-39) with the precision and initial-guess choices."""
    cutoff: float = 0.9
    beta: float = 3.5
    grid: tuple = (36, 36, 36)
    order: int = 6
    tol: float = 1e-5
    max_iter: int = 100
    peek: float = 0.65
    predictor: int = 2
    ke: float = 138.935458
    device: int = 0
    skin: float = 0.15
    precision: int = MIXED
    zero_guess: bool = False
    polarizable: bool = True
    refine: bool = False

    def to_c(self):
        s = _lib.PgmSettings()
        s.cutoff, s.beta = self.cutoff, self.beta
        for a in range(3):
            s.grid[a] = int(self.grid[a])
        s.order, s.tol, s.max_iter, s.peek = int(self.order), self.tol, int(self.max_iter), self.peek
        s.predictor, s.ke, s.device, s.skin = int(self.predictor), self.ke, int(self.device), self.skin
        s.precision, s.zero_guess, s.polarizable = int(self.precision), int(self.zero_guess), int(self.polarizable)
        s.refine = int(self.refine)
        return s


@dataclass
class Terms:
    """pgmcuda::Terms (core/cuda/pgm_cuda.h:41-45), kJ/mol."""
    direct: float = 0.0
    reciprocal: float = 0.0
    self: float = 0.0
    background: float = 0.0
    polarization: float = 0.0
    gvdw: float = 0.0

    @staticmethod
    def from_c(t):
        return Terms(t.direct, t.reciprocal, t.self, t.background, t.polarization, t.gvdw)

    def total(self):
        return self.direct + self.reciprocal + self.self + self.background + self.polarization + self.gvdw

    def as_dict(self):
        return dict(direct=self.direct, reciprocal=self.reciprocal, self=self.self, background=self.background,
                    polarization=self.polarization)


@dataclass
class Result:
    terms: Terms
    forces: np.ndarray = None
    strain: np.ndarray = None
    iterations: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def energy(self):
        return self.terms.total()


class Engine:
    """One engine on one GPU (pgmcuda::Engine).  Not thread safe: one thread at a time."""

    def __init__(self, settings: Settings | None = None, **kw):
        self.settings = settings or Settings(**kw)
        self._L = _lib.load()
        h = ctypes.c_void_p()
        _check(self._L.pgm_engine_create(ctypes.byref(self.settings.to_c()), ctypes.byref(h)))
        self._h = h
        self.n = 0
        self.ncov = 0
        self.nsys = 0

    def close(self):
        if getattr(self, "_h", None):
            self._L.pgm_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- topology
    def set_atoms(self, q, radius, alpha, global_index=None, num_global=None):
        """pgmcuda::Engine::setAtoms (core/cuda/pgm_cuda.h:55-56)."""
        q, radius, alpha = _f64(q), _f64(radius), _f64(alpha)
        n = len(q)
        gi = _i32(global_index) if global_index is not None else None
        ng = int(num_global) if num_global is not None else n
        _check(self._L.pgm_engine_set_atoms(self._h, n, _d(q), _d(radius), _d(alpha), _i(gi), ng))
        self.n = n
        self.nsys = 1
        self.ncov = 0

    def set_covalent(self, atom, partner, strength):
        """pgmcuda::Engine::setCovalent (core/cuda/pgm_cuda.h:67)."""
        atom, partner, strength = _i32(atom), _i32(partner), _f64(strength)
        _check(self._L.pgm_engine_set_covalent(self._h, len(atom), _i(atom), _i(partner), _d(strength)))
        self.ncov = len(atom)

    def set_candidates(self, seg_i, seg_shift, seg_begin, cand_j):
        """pgmcuda::Engine::setCandidates (core/cuda/pgm_cuda.h:68-73): the caller's pair candidates in place of the
        own pair search, until the next set_atoms.  Segment s: pairs (seg_i[s], cand_j[k]) for k in
        [seg_begin[s], seg_begin[s + 1]), x = r_i + t.box - r_j with t = seg_shift[s] (integer box vectors)."""
        seg_i, seg_begin, cand_j = _i32(seg_i), _i32(seg_begin), _i32(cand_j)
        seg_shift = np.ascontiguousarray(np.asarray(seg_shift, dtype=np.int32).reshape(-1, 3))
        if len(seg_begin) != len(seg_i) + 1 or len(seg_shift) != len(seg_i):
            raise ValueError("set_candidates: seg_begin needs len(seg_i) + 1 entries and seg_shift len(seg_i) rows")
        _check(self._L.pgm_engine_set_candidates(self._h, len(seg_i), _i(seg_i), _i(seg_shift), _i(seg_begin),
                                                 _i(cand_j)))

    def set_gvdw(self, repulsion, rvdw, sqrt_a, sqrt_c6, b, skip_i=(), skip_j=()):
        """pgmcuda::Engine::setGvdw (core/cuda/pgm_cuda.h:57-65): the combination-rule GVDW van der Waals
        (repulsion 0 Gaussian, 1 Slater) for the pairs within rvdw (<= cutoff) except the skipped ones; per atom
        sqrt(A), sqrt(C6), b.  Its energy is Terms.gvdw; until the next set_atoms."""
        sa, sc, bb = _f64(sqrt_a), _f64(sqrt_c6), _f64(b)
        si, sj = _i32(skip_i), _i32(skip_j)
        if not (len(sa) == len(sc) == len(bb) == self.n) or len(si) != len(sj):
            raise ValueError("set_gvdw: per-atom arrays of n entries and skipped pairs of equal length")
        _check(self._L.pgm_engine_set_gvdw(self._h, int(repulsion), float(rvdw), _d(sa), _d(sc), _d(bb), len(si),
                                           _i(si), _i(sj)))

    def probe_barrier_timeout(self):
        """Self-test of the grid transforms' bounded barrier: (gave_up, seconds); gave_up is True when the wait
        ran out and reported it, as designed."""
        flag = np.zeros(1, np.int32)
        sec = np.zeros(1)
        _check(self._L.pgm_engine_probe_barrier_timeout(self._h, _i(flag), _d(sec)))
        return bool(flag[0]), float(sec[0])

    def set_system(self, system):
        """set_atoms + set_covalent from a ``systems.System``."""
        self.set_atoms(system.q, system.radius, system.alpha)
        self.set_covalent(system.cov_atom, system.cov_partner, system.cov_strength)

    # ---------------------------------------------------------------- evaluation
    def compute(self, pos, box, new_step=True, forces=True, strain=True) -> Result:
        """pgmcuda::Engine::compute (core/cuda/pgm_cuda.h:79): host positions (n, 3), box rows (3, 3)."""
        pos = _f64(pos)
        box = _f64(box)
        f = np.zeros((self.n, 3)) if forces else None
        s = np.zeros(9) if strain else None
        t = _lib.PgmTerms()
        _check(self._L.pgm_engine_compute(self._h, _d(pos), _d(box), int(bool(new_step)), _d(f), _d(s),
                                          ctypes.byref(t)))
        return Result(Terms.from_c(t), f, s, self.iterations())

    def compute_f(self, pos, box, new_step=True):
        """pgmcuda::Engine::computeF (core/cuda/pgm_cuda.h:82): float positions; forces from forces()."""
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        box = _f64(box)
        s = np.zeros(9)
        t = _lib.PgmTerms()
        _check(self._L.pgm_engine_compute_f(self._h, pos.ctypes.data_as(_lib.P_F), _d(box), int(bool(new_step)),
                                            _d(s), ctypes.byref(t)))
        p = self._L.pgm_engine_forces(self._h)
        f = np.ctypeslib.as_array(p, shape=(self.n * 3,)).copy().reshape(self.n, 3)
        return Result(Terms.from_c(t), f, s, self.iterations())

    def launch_device(self, posq4_ptr, box, new_step, force_fixed_ptr, stride, fixed_scale, stream_ptr):
        """pgmcuda::Engine::launchDevice (core/cuda/pgm_cuda.h:102-103): device float4 positions, device
        64-bit fixed-point force buffer, caller stream (raw pointers/handles as ints)."""
        box = _f64(box)
        _check(self._L.pgm_engine_launch_device(self._h, ctypes.c_void_p(posq4_ptr), _d(box), int(bool(new_step)),
                                                ctypes.c_void_p(force_fixed_ptr), int(stride), float(fixed_scale),
                                                ctypes.c_void_p(stream_ptr)))

    def finish_device(self):
        """pgmcuda::Engine::finishDevice (core/cuda/pgm_cuda.h:104): (valid, terms)."""
        t = _lib.PgmTerms()
        v = ctypes.c_int()
        _check(self._L.pgm_engine_finish_device(self._h, ctypes.byref(t), ctypes.byref(v)))
        return bool(v.value), Terms.from_c(t)

    def wait_device(self, stream_ptr):
        _check(self._L.pgm_engine_wait_device(self._h, ctypes.c_void_p(stream_ptr)))

    def launch_resident(self, pos_dev_ptr, box, new_step, forces_dev_ptr, stream_ptr=0):
        """Device-resident evaluation: device double positions (n*3), device double forces written."""
        box = _f64(box)
        _check(self._L.pgm_engine_launch_resident(self._h, ctypes.c_void_p(pos_dev_ptr), _d(box), int(bool(new_step)),
                                                  ctypes.c_void_p(forces_dev_ptr), ctypes.c_void_p(stream_ptr)))

    # ---------------------------------------------------------------- getters
    def iterations(self):
        return int(self._L.pgm_engine_iterations(self._h))

    def residual(self):
        return float(self._L.pgm_engine_residual(self._h))

    def induced_dipoles(self):
        m = np.zeros((self.n, 3))
        _check(self._L.pgm_engine_induced_dipoles(self._h, _d(m)))
        return m

    def permanent_dipoles(self):
        m = np.zeros((self.n, 3))
        _check(self._L.pgm_engine_permanent_dipoles(self._h, _d(m)))
        return m

    def reset_history(self):
        _check(self._L.pgm_engine_reset_history(self._h))

    def list_builds(self):
        return int(self._L.pgm_engine_list_builds(self._h))

    def late_list_checks(self):
        return int(self._L.pgm_engine_late_list_checks(self._h))

    def num_candidates(self):
        return int(self._L.pgm_engine_num_candidates(self._h))

    def strain_derivative(self):
        s = np.zeros(9)
        _check(self._L.pgm_engine_strain(self._h, _d(s)))
        return s

    def field(self, pos, box, q, d):
        """pgmcore::Engine::field (core/pgm_core.h:76-77): direct + reciprocal + self field [e/nm^2]."""
        pos, box, q, d = _f64(pos), _f64(box), _f64(q), _f64(d)
        E = np.zeros((self.n, 3))
        _check(self._L.pgm_engine_field(self._h, _d(pos), _d(box), _d(q), _d(d), _d(E)))
        return E

    def pairs(self):
        """The pair set of the last evaluation as (i, j) arrays with i < j, sorted."""
        cnt = ctypes.c_longlong()
        _check(self._L.pgm_engine_pairs(self._h, None, None, 0, ctypes.byref(cnt)))
        pi = np.zeros(cnt.value, np.int32)
        pj = np.zeros(cnt.value, np.int32)
        _check(self._L.pgm_engine_pairs(self._h, _i(pi), _i(pj), cnt.value, ctypes.byref(cnt)))
        order = np.lexsort((pj, pi))
        return pi[order].astype(np.int64), pj[order].astype(np.int64)

    def get_history(self):
        size = int(self._L.pgm_engine_history_size(self._h))
        blob = (ctypes.c_char * size)()
        _check(self._L.pgm_engine_get_history(self._h, blob))
        return bytes(blob)

    def set_history(self, blob: bytes):
        buf = ctypes.create_string_buffer(blob, len(blob))
        _check(self._L.pgm_engine_set_history(self._h, buf))

    def param_grad(self):
        """dE/d(q, radius, alpha) per atom and dE/d(strength) per covalent dipole at the last solution."""
        dq, dR, da = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        dc = np.zeros(max(self.ncov, 1))
        _check(self._L.pgm_engine_param_grad(self._h, _d(dq), _d(dR), _d(da), _d(dc)))
        return dict(q=dq, radius=dR, alpha=da, cov_strength=dc[: self.ncov])

    def force_matching_grad(self, F_target, tol=1e-10):
        """Gradient of the force-matching loss L = sum |F - F_target|^2 of the last evaluation (peek 0) with
        respect to the per-atom q, radius, alpha and the per-dipole strengths: one adjoint solve to ``tol`` and
        analytic tangent passes on the GPU (pgm_engine_force_matching_grad).  Batched engines: F_target holds
        every system's target forces, concatenated.  Returns (L, gradients dict, adjoint CG iterations)."""
        ft = _f64(F_target, (self.n, 3))
        dq, dR, da = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        dc = np.zeros(max(self.ncov, 1))
        L = ctypes.c_double(0)
        it = ctypes.c_int(0)
        _check(self._L.pgm_engine_force_matching_grad(self._h, _d(ft), float(tol), _d(dq), _d(dR), _d(da), _d(dc),
                                                       ctypes.byref(L), ctypes.byref(it)))
        return L.value, dict(q=dq, radius=dR, alpha=da, cov_strength=dc[: self.ncov]), it.value

    def evaluate_fixed(self, pos, box, mu, keep_list=False):
        """Energy, forces and total field [e/nm^2] at given induced dipoles, no solve (adjoint probes); with
        keep_list the previous evaluation's pair list and box are reused.  param_grad() then gives dE/dtheta at
        these dipoles."""
        pos, box, mu = _f64(pos), _f64(box), _f64(mu)
        f = np.zeros((self.n, 3))
        E = np.zeros((self.n, 3))
        t = _lib.PgmTerms()
        _check(self._L.pgm_engine_evaluate_fixed(self._h, _d(pos), _d(box), _d(mu), int(bool(keep_list)), _d(f), _d(E),
                                                 ctypes.byref(t)))
        return Result(Terms.from_c(t), f, None, 0, {"field": E})

    def solve(self, rhs, tol=1e-10):
        """x with (alpha^-1 - T) x = rhs on the geometry of the last evaluation (rows of non-polarizable atoms
        are 0): the adjoint solve, the same symmetric operator as the induced dipoles'."""
        rhs = _f64(rhs)
        x = np.zeros((self.n, 3))
        it = ctypes.c_int()
        _check(self._L.pgm_engine_solve(self._h, _d(rhs), _d(x), float(tol), ctypes.byref(it)))
        return x, it.value

    def kernel_launches(self):
        return int(self._L.pgm_engine_kernel_launches(self._h))

    KERNELS = ("pair_list", "pair_field", "spread", "gather", "pair_final", "fft_chain", "cg_update")

    def active_systems(self):
        """Batched engines: systems still iterating before each CG iteration of the last evaluation."""
        counts = np.zeros(1024, np.int32)
        m = int(self._L.pgm_engine_active_systems(self._h, _i(counts), len(counts)))
        if m < 0:
            raise PgmError(m, self._L.pgm_last_error().decode())
        return counts[:m].tolist()

    def kernel_times(self, reps=20, flush_ptr=None, flush_bytes=0):
        """Average device durations [ms] of the main kernels relaunched alone (CUDA events on the engine's
        stream) after an evaluation: warm (back to back), or cold when a device buffer larger than L2 is given
        (flush_ptr, flush_bytes; overwritten before every launch, only the launch timed)."""
        ms = np.zeros(7)
        if flush_ptr is None:
            _check(self._L.pgm_engine_kernel_times(self._h, int(reps), _d(ms)))
        else:
            _check(self._L.pgm_engine_kernel_times_cold(self._h, int(reps), ctypes.c_void_p(flush_ptr),
                                                        int(flush_bytes), _d(ms)))
        return dict(zip(self.KERNELS, ms.tolist()))

    def time_evaluations(self, reps=20):
        """Median device time [ms] of ``reps`` whole new-step evaluations at the last evaluation's positions
        (already on the device); the predictor history is left as it was."""
        ms = ctypes.c_double(0)
        _check(self._L.pgm_engine_time_evaluations(self._h, int(reps), ctypes.byref(ms)))
        return ms.value

    def set_pme_kernels(self, kind):
        """PME spread / gather of the field passes: 0 a warp per atom, 1 plane-owner tiles in shared memory
        (mixed precision, one system, order 6), 2 float4 lines (mixed precision, orders 4, 5, 6, 8, batches
        too), 3 cell-group tiles in shared memory (mixed precision, one system, orders 4, 5, 6, 8);
        pme_kernels() tells which runs."""
        _check(self._L.pgm_engine_set_pme_kernels(self._h, int(kind)))

    def pme_kernels(self):
        return int(self._L.pgm_engine_pme_kernels(self._h))

    def set_pair_lanes(self, lanes):
        _check(self._L.pgm_engine_set_pair_lanes(self._h, int(lanes)))

    def pair_lanes(self):
        return int(self._L.pgm_engine_pair_lanes(self._h))

    def set_transforms(self, mode):
        """Field-pass transforms: 0 cuFFT 3D plans + influence product, 1 one cluster kernel per pass, 2 cuFFT 2D
        plans over the x-planes + one x-line kernel with the influence product, 3 one cooperative kernel with a
        block per x-plane, 4 that kernel for the field passes around the CG loop and the whole CG loop as one
        persistent cooperative kernel (mixed precision, one system, order 6); transforms() tells which runs."""
        _check(self._L.pgm_engine_set_transforms(self._h, int(mode)))

    def transforms(self):
        return int(self._L.pgm_engine_transforms(self._h))

    def autotune(self, pos, box, reps=20, candidates=(4, 8, 16, 32), reproducible=True):
        """Picks the lanes per atom of the pair passes, the kind of field-pass transforms and the PME kernels by
        timing whole evaluations of this system (batched engines: pass the batch's positions and boxes): every
        (lanes, transforms, PME kernels) the grids allow, each the median of ``reps`` new-step evaluations on the
        device (inputs resident, no host copies).  Every candidate's time is in ``self.autotune_report`` [ms].
        Keeps the fastest of those whose results repeat bit for bit (reproducible=True: in mixed precision the
        warp-per-atom spread into the 64-bit fixed-point grid, PME kernels 0; the others add float atomics), or
        of all (reproducible=False).  Returns the lanes."""
        batched = getattr(self, "nsys", 1) > 1
        if batched:
            self.compute_batch(pos, box)
        else:
            self.compute(pos, box)
        report = {}
        for mode in (0, 1, 2, 3, 4):
            self.set_transforms(mode)
            if self.transforms() != mode:
                continue
            for pme in (0, 1, 2, 3):
                self.set_pme_kernels(pme)
                if self.pme_kernels() != pme:
                    continue
                for lanes in candidates:
                    self.set_pair_lanes(lanes)
                    self.time_evaluations(2)   # (captures the graph of this choice)
                    report[(lanes, mode, pme)] = self.time_evaluations(reps)
        pool = {k: v for k, v in report.items() if k[2] == 0} if reproducible else report
        lanes, mode, pme = min(pool or report, key=(pool or report).get)
        self.set_pair_lanes(lanes)
        self.set_transforms(mode)
        self.set_pme_kernels(pme)
        self.autotune_report = {f"lanes{k[0]}_transforms{k[1]}_pme{k[2]}": v for k, v in report.items()}
        return lanes

    # ---------------------------------------------------------------- batched
    def set_systems(self, systems):
        """Many independent systems (``systems.System`` list) evaluated together by compute_batch."""
        counts = _i32([s.n for s in systems])
        cut = _f64([s.cutoff for s in systems])
        bet = _f64([s.beta for s in systems])
        grid = _i32(np.array([s.grid for s in systems]).reshape(-1))
        q = _f64(np.concatenate([s.q for s in systems]))
        R = _f64(np.concatenate([s.radius for s in systems]))
        al = _f64(np.concatenate([s.alpha for s in systems]))
        cc = _i32([len(s.cov_atom) for s in systems])
        ca = _i32(np.concatenate([s.cov_atom for s in systems]))
        cp = _i32(np.concatenate([s.cov_partner for s in systems]))
        cs = _f64(np.concatenate([s.cov_strength for s in systems]))
        _check(self._L.pgm_engine_set_systems(self._h, len(systems), _i(counts), _d(cut), _d(bet), _i(grid), _d(q),
                                              _d(R), _d(al), _i(cc), _i(ca), _i(cp), _d(cs)))
        self.nsys = len(systems)
        self.n = int(counts.sum())
        self.ncov = int(cc.sum())
        self._counts = counts

    def compute_batch(self, pos, boxes, forces=True):
        pos = _f64(pos)
        boxes = _f64(boxes)
        E = np.zeros((self.nsys, 6))
        S = np.zeros((self.nsys, 9))
        it = np.zeros(self.nsys, np.int32)
        f = np.zeros((self.n, 3)) if forces else None
        _check(self._L.pgm_engine_compute_batch(self._h, _d(pos), _d(boxes), _d(E), _d(f), _d(S), _i(it)))
        return dict(energies=E, forces=f, strain=S, iterations=it)


def pair_list_noalloc(n, pos_dev_ptr, box, cutoff, cap, slot_atom_ptr, counts_ptr, neighbors_ptr, stream_ptr=0):
    """The directed pair list of one periodic system into caller-owned device buffers, allocating nothing
    (pgm_pair_list_noalloc of include/pgm_b200.h): for callers that cannot allocate device memory, such as
    MD engines whose memory pool owns the whole GPU, or hosts that reserve their device memory up front.
    Buffers are raw device pointers: positions double n*3; slot_atom int n, counts int n, neighbors int n*cap.
    Returns the longest row; raises PgmError (status -4, with .max_count the longest row) when n exceeds 16384
    or a row exceeds cap.  The call waits for its own work on the stream before it returns."""
    L = _lib.load()
    box = _f64(box)
    mx = ctypes.c_int(0)
    rc = L.pgm_pair_list_noalloc(int(n), ctypes.c_void_p(pos_dev_ptr), _d(box), float(cutoff), int(cap),
                                 ctypes.c_void_p(slot_atom_ptr), ctypes.c_void_p(counts_ptr),
                                 ctypes.c_void_p(neighbors_ptr), ctypes.c_void_p(stream_ptr), ctypes.byref(mx))
    if rc != 0:
        err = PgmError(rc, L.pgm_last_error().decode())
        err.max_count = mx.value
        raise err
    return mx.value
