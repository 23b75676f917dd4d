#!/usr/bin/env python
"""Benchmark: pGM energy + force + virial evaluations per second of the 8550-atom periodic liquid
(450 rigid C8H10O molecules, 44.5 A box, beta 0.35/A, cutoff 9 A, 48^3 grid, order 6, tol 1e-5) on one
B200, mixed precision, beside this engine's FP64 path on the same input.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pgm_b200|reference]

A step is one full evaluation (cell and pair list, permanent field, CG induced-dipole solve from the
alpha E_perm guess, final energies, forces and strain derivative).  N > 1 runs N independent replicas, one
process per GPU (the single-system evaluation does not shard; weak scaling).  Inputs are resident in HBM
for ``value``; ``e2e`` goes through the C ABI's host call with host positions and host forces.  L2 is
flushed (a 256 MiB write) before every timed step.  ``--impl reference`` times the reference's own FP64
CPU engine (core/pgm_core.cpp built from its sources into oracle/_ref) on every host core.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "pGM E+F evals/s, 8550-atom PME, mixed vs FP64 GPU at force relRMS≤1e-5"
WORKLOAD = "dimethylphenol8550"
TOL = 1e-5
TRANSFORMS = {0: "cuFFT + influence product", 1: "cluster kernel", 2: "cuFFT 2D + x-line kernel",
              3: "grid kernel (block per x-plane)",
              4: "grid kernel + persistent CG kernel (whole solve in one cooperative launch)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="pgm_b200", choices=["pgm_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--ref-steps-cap", type=int, default=0, help="reference arm: cap on timed steps (0: --steps)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: only warmup + steps evaluations of one precision, no other legs")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"], help="with --profile")
    ap.add_argument("--profile-workload", default=WORKLOAD, choices=[WORKLOAD, "water98304", "water_batch1024"],
                    help="with --profile: the system evaluated")
    ap.add_argument("--profile-transforms", type=int, default=-1,
                    help="with --profile: the field-pass transforms (0..4; -1: the engine's default)")
    ap.add_argument("--profile-pme", type=int, default=0, help="with --profile: PME kernels (0 warp per atom, 1 plane tiles, 2 float4 lines, 3 cell tiles)")
    ap.add_argument("--profile-lanes", type=int, default=16, help="with --profile: pair lanes")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 1024-system leg")
    ap.add_argument("--no-large", action="store_true", help="skip the 98304-atom leg")
    ap.add_argument("--no-grad", action="store_true", help="skip the parameter-gradient leg")
    ap.add_argument("--ref-large", action="store_true",
                    help="reference arm: also one evaluation of the 98304-atom box on one core (about a minute)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip the reference GPU engine timed on this GPU")
    return ap.parse_args()


def system():
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    return pkg, pkg.systems.dimethylphenol8550(tol=TOL)


def config(S, extra=None):
    c = {"workload": WORKLOAD, "atoms": S.n, "molecules": 450, "box_nm": float(S.box[0, 0]), "cutoff_nm": S.cutoff,
         "beta_per_nm": S.beta, "grid": list(S.grid), "order": S.order, "tol": TOL, "predictor": "none",
         "peek": 0.65, "l2": "flushed (256 MiB write) before every timed step"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every 2 ms during the timed region
    (read-only queries)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = None
        self._thread = None

    def _sample(self):
        import pynvml
        self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(self._h, pynvml.NVML_CLOCK_SM)))
        try:
            self.reasons |= int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(self._h))
        except Exception:
            self.reasons |= int(pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(self._h))

    def _run(self):
        try:
            while not self._stop.wait(0.002):
                self._sample()
        except Exception:
            pass

    def __enter__(self):
        # NVML is set up before the timed region starts (it can take longer than a short region lasts); one
        # sample as the region opens, the thread's every 2 ms, one as it closes
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
            self._sample()
        except Exception:
            self._h = None
        self._stop = threading.Event()
        if self._h is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *a):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self._h is not None:
            try:
                import pynvml
                self._sample()
                pynvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(v for k, v in self.REASONS.items() if self.reasons & k), "samples": len(self.samples),
                "source": "NVML, every 2 ms during the timed region"}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_of(kernel):
    """DRAM bytes per launch of a kernel from the committed ncu summary (profiles/traffic.json), or None."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        v = d.get(WORKLOAD, {}).get(kernel)
        return v
    return None


def algorithmic_bytes(kernel, S, precision, it):
    """Algorithmic bytes per launch of the main kernels, the minimum each must move (per unit: atom, directed
    pair, grid point): s = real size, g = grid real size (= s), P = directed pairs within the cutoff,
    p = order, G = K1 K2 K3, G_c = K1 K2 (K3/2 + 1):
      spread      N (7 s + p^3 g)          q, d, base, fraction in; p^3 grid updates
      gather      N (7 s + 3 s + p^3 g)    the same in, p^3 grid reads, the field out
      pair field  P 4 + N 10 s             a list index per pair, own position, charge and dipole, field out
      FFT chain   2 (G g + 2 G_c g) + 4 G_c g   r2c and c2r, the convolution (read F and G, write F)
      CG update   3 N 8 10                 ten FP64 vector streams of 3N
      pair list   N 24 + P 4               positions in, list entries out
      final pass  P 4 + N (10 s + 128)     a list index per pair, the sources, 16 doubles out per atom"""
    s = 4 if precision else 8
    g = s
    n, p = S.n, S.order
    P = S.meta.get("pairs", 0)
    K1, K2, K3 = S.grid
    G = K1 * K2 * K3
    Gc = K1 * K2 * (K3 // 2 + 1)
    return {"spread": n * (7 * s + p ** 3 * g), "gather": n * (7 * s + 3 * s + p ** 3 * g),
            "pair_field": P * 4 + n * 10 * s, "fft_chain": 2 * (G * g + 2 * Gc * g) + 4 * Gc * g,
            "cg_update": 3 * n * 8 * 10, "pair_list": n * 24 + P * 4,
            "pair_final": P * 4 + n * (10 * s + 128)}.get(kernel)


def design_bytes(kernel, S, precision):
    """The bytes the engine's own data layout moves per launch, where it differs from the algorithmic figure:
    the pair passes stream a record per directed pair (mixed: x, G1 | G2, slot of j, 24 B; FP64: the 4 B entry
    and (G1, G2)) instead of recomputing the radial kernels."""
    s = 4 if precision else 8
    n, P = S.n, S.meta.get("pairs", 0)
    if kernel == "pair_field":
        return P * 24 + n * (4 * s + 24) if precision else P * (4 + 2 * s) + n * (32 + 4 * s + 24)
    if kernel == "pair_list":
        rec = 24 if precision else 2 * s
        return n * (32 + 32 + 16 + 8) + P * (4 + 4 + 4 + rec)
    return algorithmic_bytes(kernel, S, precision, 0)


def roofline_table(S, kt, it, precision, kt_cold=None):
    """Per-kernel algorithmic bandwidth against the measured HBM copy bandwidth.  Each kernel is relaunched
    alone on the engine's stream: warm (back to back, as inside an evaluation: inputs that fit the 126 MB L2
    stay there) and cold (L2 overwritten before each launch).  The dominant kernel is the engine's own kernel
    with the largest share of an evaluation (the FFT chain, cuFFT's or the grid kernel, is listed beside it)."""
    peak, peak_kind = peaks()
    share = {k: v * launches_per_eval(k, it) for k, v in kt.items()}
    total = sum(share.values())
    per = {}
    for k, ms in kt.items():
        alg = algorithmic_bytes(k, S, precision, it)
        ach = alg / (ms * 1e-3) / 1e9 if alg else None
        row = {"ms_per_launch": ms, "launches_per_eval": launches_per_eval(k, it), "share": share[k] / total,
               "bytes_per_launch": alg, "achieved_gbs": ach, "frac": ach / peak if ach else None,
               "design_bytes": design_bytes(k, S, precision)}
        if kt_cold:
            mc = kt_cold[k]
            row.update({"ms_per_launch_cold": mc, "achieved_gbs_cold": alg / (mc * 1e-3) / 1e9,
                        "frac_cold": alg / (mc * 1e-3) / 1e9 / peak})
        per[k] = row
    own = {k: v for k, v in share.items() if k != "fft_chain"}
    dom = max(own, key=own.get)
    out = {"kernel": dom, "bound": "hbm", "achieved": per[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
           "frac": per[dom]["frac"], "peak_source": peak_kind, "traffic": traffic_of(dom),
           "bytes_per_launch": per[dom]["bytes_per_launch"], "design_bytes": per[dom]["design_bytes"],
           "ms_per_launch": kt[dom], "fft_chain_share": per["fft_chain"]["share"], "per_kernel": per,
           "bytes_convention": "algorithmic bytes per launch (pair field P*4 + N*10s, spread N(7s + p^3 g), "
                               "gather N(10s + p^3 g), ...); design_bytes: what the engine's layout moves",
           "note": "frac: warm relaunches (back to back, inputs that fit the 126 MB L2 stay there, as inside an "
                   "evaluation); frac_cold: L2 overwritten before each launch; traffic: DRAM bytes of one cold "
                   "launch from the committed ncu summary"}
    if kt_cold:
        out["frac_cold"] = per[dom]["frac_cold"]
        out["ms_per_launch_cold"] = kt_cold[dom]
    return out


def md_positions(S, phase, count):
    """The moving positions of steps 0 .. count - 1: amplitude 0.01 nm, period 100 steps, per-coordinate phases
    (the reference harness's moving timing, core/cuda/tests/test_cuda.cpp:351-372).  Generated before a timed loop:
    in numpy each step's positions take about 0.4 ms of host time, as much as an engine call."""
    return [S.pos + 0.01 * np.sin(2 * np.pi * st / 100 + phase) for st in range(count)]


def md_leg(pkg, S, make, lanes, dev, steps=60):
    """MD-like use: positions move smoothly every step (amplitude 0.01 nm, period 100 steps, random phases,
    as the reference harness's moving timing, core/cuda/tests/test_cuda.cpp:351-372), new step every call,
    mu4 predictor, the Verlet list kept with the default 0.15 nm skin (as the reference engine's); host call with
    host positions and forces.  Both precisions; mixed again with the predicted steps' dual first pass
    (PGM_B200_DUAL=1) for its gain."""
    import torch
    rng = np.random.default_rng(7)
    phase = rng.uniform(0, 2 * np.pi, S.pos.shape)
    out = {}
    for name, prec in (("mixed", pkg.MIXED), ("fp64", pkg.FP64), ("mixed_dual_first_pass", pkg.MIXED)):
        if name == "mixed_dual_first_pass":
            os.environ["PGM_B200_DUAL"] = "1"
        eng = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=TOL, max_iter=200,
                                      peek=0.65, predictor=2, ke=pkg.systems.KE_DEFAULT, precision=prec,
                                      device=dev.index or 0))
        eng.set_system(S)
        eng.set_pair_lanes(lanes)
        its = []
        traj = md_positions(S, phase, 10 + steps)
        for st in range(10):
            eng.compute(traj[st], S.box)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for st in range(10, 10 + steps):
            r = eng.compute(traj[st], S.box)
            its.append(r.iterations)
        dt = (time.perf_counter() - t0) / steps
        out[name] = {"evals_per_s": 1.0 / dt, "mean_cg_iterations": float(np.mean(its)),
                     "list_builds": eng.list_builds()}
        eng.close()
        os.environ.pop("PGM_B200_DUAL", None)
    out["mixed_over_fp64"] = out["mixed"]["evals_per_s"] / out["fp64"]["evals_per_s"]
    out["dual_first_pass_gain"] = out["mixed_dual_first_pass"]["evals_per_s"] / out["mixed"]["evals_per_s"]
    out["note"] = ("host call with host positions and forces (positions generated before the timed loop); "
                   "predictor mu4; Verlet list, skin 0.15 nm; predicted steps take two first passes "
                   "(mixed_dual_first_pass: the same with the dual first pass, PGM_B200_DUAL=1)")
    return out


def launches_per_eval(kernel, it):
    return {"pair_list": 1, "pair_field": it + 2, "spread": it + 3, "gather": it + 3, "pair_final": 1,
            "fft_chain": it + 3, "cg_update": it}.get(kernel, 1)


def reference_arm(args):
    """The reference's own CPU implementation (pgm_core, FP64) on all host cores: one process per core, each
    step one evaluation per process."""
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import ref as R
    pkg, S = system()
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpgmcore_ref.so not built "
                          "(make -C oracle where the reference sources are present)"}))
        return 0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    ctx = mp.get_context("spawn")
    steps = args.steps if not args.ref_steps_cap else min(args.steps, args.ref_steps_cap)
    with ctx.Pool(cores, initializer=_ref_worker_init) as pool:
        pool.map(_ref_worker_eval, range(cores))          # untimed: every worker builds its engine
        for _ in range(args.warmup):
            pool.map(_ref_worker_eval, range(cores))
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            pool.map(_ref_worker_eval, range(cores))
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = cores * steps / total
    line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": config(S, {"parallelism": "1 GPU"}),
            "reference_impl": {"implementation": "reference pgm_core (core/pgm_core.cpp) FP64, one process per core",
                               "step": f"{cores} evaluations in parallel, one per process"},
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "reference",
                             "sample": f"{steps} steps x {cores} full evaluations of {WORKLOAD}",
                             "cpu": cpu_model()},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["cpu_other_configs"] = cpu_other_configs(pkg, cores, ctx, args.ref_large)
    if not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_leg(pkg, S, steps, max(args.warmup, 3))
    print(json.dumps(line))
    return 0


BATCH_SAMPLE = 64


def _ref_engine(pkg, S, tol):
    from oracle import pgm_oracle as O
    from oracle import ref as R
    top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
    st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=tol, max_iter=500, peek=0.65,
                    predictor=0, ke=pkg.systems.KE_DEFAULT)
    return R.RefEngine(top, st)


def _batch_worker_init():
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    pkg, _ = system()
    systems = pkg.systems.water_batch(nsys=1024, seed=1024, tol=TOL)[:BATCH_SAMPLE]
    _REF["batch"] = [(S, _ref_engine(pkg, S, TOL)) for S in systems]


def _batch_worker_eval(k):
    S, e = _REF["batch"][k]
    return e.compute(S.pos, S.box)


def cpu_other_configs(pkg, cores, ctx, large):
    """The reference pgm_core on the other configurations (bounded samples, FP64): the 216-water box on one
    core; the first 64 boxes of the 1024-box water batch sequentially on one core and spread over all cores (one
    process per core); with ``large`` one evaluation of the 98304-atom water box on one core (about a minute
    and more: pgm_core's pair search tests all N^2 pairs)."""
    out = {}
    S = pkg.systems.water216()
    e = _ref_engine(pkg, S, S.tol)
    e.compute(S.pos, S.box)
    t0 = time.perf_counter()
    for _ in range(5):
        e.compute(S.pos, S.box)
    out["water216"] = {"evals_per_s": 5 / (time.perf_counter() - t0), "cores": 1, "tol": S.tol}
    systems = pkg.systems.water_batch(nsys=1024, seed=1024, tol=TOL)[:BATCH_SAMPLE]
    engines = [_ref_engine(pkg, B, TOL) for B in systems]
    t0 = time.perf_counter()
    for B, eb in zip(systems, engines):
        eb.compute(B.pos, B.box)
    seq = time.perf_counter() - t0
    with ctx.Pool(cores, initializer=_batch_worker_init) as pool:
        pool.map(_batch_worker_eval, range(BATCH_SAMPLE))   # untimed: every worker's engines warm
        t0 = time.perf_counter()
        pool.map(_batch_worker_eval, range(BATCH_SAMPLE))
        par = time.perf_counter() - t0
    out["water_batch1024"] = {"sample": f"the first {BATCH_SAMPLE} of the 1024 boxes",
                              "atoms": int(sum(B.n for B in systems)),
                              "systems_per_s_1_core": BATCH_SAMPLE / seq,
                              "systems_per_s_all_cores": BATCH_SAMPLE / par, "cores": cores}
    if large:
        S = pkg.systems.water98304(tol=TOL)
        e = _ref_engine(pkg, S, TOL)
        t0 = time.perf_counter()
        e.compute(S.pos, S.box)
        out["water98304"] = {"evals_per_s": 1.0 / (time.perf_counter() - t0), "cores": 1, "tol": TOL}
    return out


def reference_gpu_leg(pkg, S, steps, warmup):
    """The reference's own GPU engine (core/cuda/pgm_cuda.cu, unchanged, built into oracle/_ref) on this GPU,
    with its defaults (mixed precision, CUDA graph, own pair list with a 0.15 nm skin):
      step: the benchmark step (predictor none, tol 1e-5, peek 0.65, the same positions every call) through its
        OpenMM path (float4 device positions in, 64-bit fixed-point device forces out, launchDevice + waitDevice
        on the caller's stream), CUDA events on that stream, L2 flushed before every step.  Its pair list is
        built at the first call and reused, since the positions do not move (pgm_b200 builds its list in every
        step);
      md_moving: as md_leg (host call, mu4 predictor, smooth motions, same phases and steps);
      accuracy: forces and energy against the FP64 oracle at tol 1e-10."""
    try:
        import torch
        from oracle import ref_cuda as RC
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
        if not RC.available():
            return {"unavailable": "oracle/_ref/libpgmcuda_ref.so not built (make -C oracle cuda)"}
        dev = torch.device("cuda:0")
        torch.cuda.set_device(dev)
        stream = torch.cuda.current_stream(dev)
        ke = pkg.systems.KE_DEFAULT
        out = {"engine": "reference pgm_cuda (core/cuda/pgm_cuda.cu) built for sm_100a, its default settings"}
        eng = RC.RefCudaEngine(S, TOL, predictor=0, peek=0.65, ke=ke)
        posq = torch.zeros((S.n, 4), dtype=torch.float32, device=dev)
        posq[:, :3] = torch.from_numpy(S.pos).to(dev, torch.float32)
        ffix = torch.zeros(3 * S.n, dtype=torch.int64, device=dev)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

        def one():
            while True:
                eng.launch_device(posq.data_ptr(), S.box, True, ffix.data_ptr(), S.n, 2.0 ** 32, stream.cuda_stream)
                eng.wait_device(stream.cuda_stream)
                if eng.finish_device():
                    return
        for _ in range(warmup):
            one()
        torch.cuda.synchronize()
        ms, its = 0.0, []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one()
            b.record(stream)
            torch.cuda.synchronize()
            ms += a.elapsed_time(b)
            its.append(eng.iterations())
        out["step"] = {"evals_per_s": steps / (ms / 1e3), "ms_per_eval": ms / steps,
                       "cg_iterations": int(np.median(its)), "list_builds": eng.list_builds(), "steps": steps}
        E, F = eng.compute(S.pos, S.box)
        ref = _oracle_reference(pkg, S, 1e-10)
        E0, F0, kind = ref["energy"], ref["forces"], ref["kind"]
        out["accuracy"] = {"oracle": kind, "force_rel_rms": float(np.linalg.norm(F - F0) / np.linalg.norm(F0)),
                           "energy_rel": float(abs(E - E0) / abs(E0))}
        eng.close()
        rng = np.random.default_rng(7)
        phase = rng.uniform(0, 2 * np.pi, S.pos.shape)
        eng = RC.RefCudaEngine(S, TOL, predictor=2, peek=0.65, ke=ke)
        md_steps, its = 30, []
        traj = md_positions(S, phase, 10 + md_steps)
        for st in range(10):
            eng.compute(traj[st], S.box)
        t0 = time.perf_counter()
        for st in range(10, 10 + md_steps):
            eng.compute(traj[st], S.box)
            its.append(eng.iterations())
        dt = (time.perf_counter() - t0) / md_steps
        out["md_moving"] = {"evals_per_s": 1.0 / dt, "mean_cg_iterations": float(np.mean(its)),
                            "list_builds": eng.list_builds(),
                            "note": "host call with host positions and forces (positions generated before the "
                                    "timed loop); predictor mu4"}
        eng.close()
        return out
    except Exception as e:   # the comparison is reported, never fatal to the reference arm
        return {"unavailable": f"{type(e).__name__}: {e}"}


_REF = {}


def _ref_worker_init():
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    from oracle import pgm_oracle as O
    from oracle import ref as R
    pkg, S = system()
    top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
    st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=TOL, max_iter=500, peek=0.65,
                    predictor=0, ke=pkg.systems.KE_DEFAULT)
    _REF["eng"] = R.RefEngine(top, st)
    _REF["S"] = S


def _ref_worker_eval(_):
    from oracle import ref as R
    e = _REF["eng"]
    S = _REF["S"]
    R.lib().ref_reset_history(e.h)   # an independent evaluation (no reuse of the previous solution)
    return e.compute(S.pos, S.box)


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device(f"cuda:{local}"))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    pkg, S = system()

    def make(precision):
        # skin 0: the pair list is built in every step (a full, independent evaluation)
        eng = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=TOL,
                                      max_iter=200, peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT,
                                      precision=precision, device=local, skin=0.0))
        eng.set_system(S)
        return eng

    stream = torch.cuda.current_stream(dev)
    if args.profile:
        if args.profile_workload == "water_batch1024":
            systems = pkg.systems.water_batch(nsys=1024, seed=1024, tol=1e-5)
            eng = pkg.Engine(pkg.Settings(cutoff=0.9, beta=3.5, grid=(24, 24, 24), order=6, tol=1e-5, max_iter=200,
                                          peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT,
                                          precision=pkg.MIXED if args.precision == "mixed" else pkg.FP64,
                                          device=local, skin=0.0))
            eng.set_systems(systems)
            pos = np.concatenate([s.pos for s in systems])
            boxes = np.stack([s.box for s in systems])
            eng.set_pair_lanes(16)
            for _ in range(args.warmup + args.steps):
                r = eng.compute_batch(pos, boxes)
            print(json.dumps({"profile": args.precision, "workload": "water_batch1024",
                              "evaluations": args.warmup + args.steps, "max_iterations": int(r["iterations"].max()),
                              "launches_per_eval": eng.kernel_launches()}))
            eng.close()
            return 0
        if args.profile_workload == "water98304":
            S = pkg.systems.water98304(tol=TOL)
        eng = make(pkg.MIXED if args.precision == "mixed" else pkg.FP64)
        eng.set_pair_lanes(args.profile_lanes)
        if args.profile_transforms >= 0:
            eng.set_transforms(args.profile_transforms)
        eng.set_pme_kernels(args.profile_pme)
        pos_p = torch.from_numpy(S.pos).to(dev).contiguous()
        f_p = torch.zeros((S.n, 3), dtype=torch.float64, device=dev)
        for _ in range(args.warmup + args.steps):
            eng.launch_resident(pos_p.data_ptr(), S.box, True, f_p.data_ptr(), stream.cuda_stream)
            eng.wait_device(stream.cuda_stream)
            eng.finish_device()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.precision, "evaluations": args.warmup + args.steps,
                          "iterations": eng.iterations(), "launches_per_eval": eng.kernel_launches(),
                          "transforms": eng.transforms(), "pme_kernels": eng.pme_kernels()}))
        eng.close()
        return 0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    pos_d = torch.from_numpy(S.pos).to(dev).contiguous()
    f_d = torch.zeros((S.n, 3), dtype=torch.float64, device=dev)

    def timed_resident(eng, steps, warmup, sampler=None):
        for _ in range(warmup):
            eng.launch_resident(pos_d.data_ptr(), S.box, True, f_d.data_ptr(), stream.cuda_stream)
            eng.wait_device(stream.cuda_stream)
            eng.finish_device()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        its = []
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            for k in range(steps):
                flush.zero_()
                evs[k][0].record(stream)
                eng.launch_resident(pos_d.data_ptr(), S.box, True, f_d.data_ptr(), stream.cuda_stream)
                eng.wait_device(stream.cuda_stream)
                evs[k][1].record(stream)
                eng.finish_device()
                its.append(eng.iterations())
            torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        return ms, its

    # mixed: autotune, time
    mixed = make(pkg.MIXED)
    r0 = mixed.compute(S.pos, S.box)
    lanes = mixed.autotune(S.pos, S.box)
    S.meta["pairs"] = mixed.num_candidates()
    sampler = ClockSampler(local)
    ms_mixed, its_mixed = timed_resident(mixed, args.steps, max(args.warmup, 3), sampler)
    clocks = sampler.summary()
    t = torch.tensor([ms_mixed], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_mixed = float(t.item())
    value = world * args.steps / (ms_mixed / 1e3)
    # FP64 path on the same input (the metric's denominator)
    fp64 = make(pkg.FP64)
    fp64.compute(S.pos, S.box)
    lanes64 = fp64.autotune(S.pos, S.box)
    fsteps = max(3, min(args.steps, 20))
    ms_fp64, its_fp64 = timed_resident(fp64, fsteps, 3)
    t = torch.tensor([ms_fp64], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    fp64_value = world * fsteps / (float(t.item()) / 1e3)
    # the same step with the Verlet list kept (default 0.15 nm skin; the positions do not move, so it is built
    # once), the protocol of the reference GPU engine's step in the reference arm
    kept = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=TOL, max_iter=200,
                                   peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT, precision=pkg.MIXED,
                                   device=local))
    kept.set_system(S)
    kept.compute(S.pos, S.box)
    kept.set_pair_lanes(lanes)
    kept.set_transforms(mixed.transforms())
    ms_kept, _ = timed_resident(kept, fsteps, 3)
    t = torch.tensor([ms_kept], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    kept_value = world * fsteps / (float(t.item()) / 1e3)
    kept_builds = kept.list_builds()
    kept.close()
    # end to end through the C ABI host call (host positions in, host forces out)
    for _ in range(2):
        mixed.compute(S.pos, S.box)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps = args.steps
    for _ in range(e2e_steps):
        res = mixed.compute(S.pos, S.box)
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * e2e_steps / float(t.item())
    # roofline of the dominant kernel (relaunched alone, CUDA events on the engine's stream): warm, and cold with
    # the L2 overwritten before every launch
    mixed.compute(S.pos, S.box)
    it = mixed.iterations()
    kt = mixed.kernel_times(reps=20)
    kt_cold = mixed.kernel_times(reps=10, flush_ptr=flush.data_ptr(), flush_bytes=flush.numel() * 4)
    roof = roofline_table(S, kt, it, 1, kt_cold)
    fp64.compute(S.pos, S.box)
    kt64 = fp64.kernel_times(reps=10)
    kt64_cold = fp64.kernel_times(reps=5, flush_ptr=flush.data_ptr(), flush_bytes=flush.numel() * 4)
    roof64 = roofline_table(S, kt64, fp64.iterations(), 0, kt64_cold)
    md = md_leg(pkg, S, make, lanes, dev)
    line = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
            "config": config(S, {"parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                                 "pair_lanes": lanes, "transforms": TRANSFORMS[mixed.transforms()],
                                 "pme_kernels": mixed.pme_kernels(),
                                 "bitwise_reproducible": mixed.pme_kernels() == 0,
                                 "cg_iterations": int(np.median(its_mixed)),
                                 "fp64_evals_per_s": fp64_value, "mixed_over_fp64": value / fp64_value}),
            "fp64": {"value": fp64_value, "unit": "evals/s", "steps": fsteps, "pair_lanes": lanes64,
                     "transforms": TRANSFORMS[fp64.transforms()],
                     "cg_iterations": int(np.median(its_fp64)), "kernel_ms": kt64,
                     "roofline_per_kernel": roof64["per_kernel"],
                     "autotune_ms": getattr(fp64, "autotune_report", None)},
            "autotune_ms": getattr(mixed, "autotune_report", None),
            "mixed_over_fp64": value / fp64_value,
            "kept_list": {"value": kept_value, "unit": "evals/s", "steps": fsteps, "list_builds": kept_builds,
                          "note": "mixed, Verlet list kept (skin 0.15 nm, positions unchanged): the reference "
                                  "GPU engine's step protocol"},
            "ns_per_day_2fs": value / world * 86400 * 2e-6,
            "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": S.n * 3 * 8,
                    "d2h_bytes_per_step": S.n * 3 * 8 + 16 * 8},
            "gpu_launches": mixed.kernel_launches() * args.steps,
            "roofline": roof, "clocks": clocks, "md_moving": md}
    if rank == 0 and not args.no_accuracy:
        def make_refined():
            e = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=TOL,
                                        max_iter=200, peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT,
                                        precision=pkg.MIXED, device=local, refine=True, skin=0.0))
            e.set_system(S)
            e.set_pair_lanes(lanes)
            return e
        line["accuracy"] = accuracy(pkg, S, mixed, fp64, make_refined)
    mixed.close()
    fp64.close()
    if not args.no_large:
        line["water98304"] = large_leg(pkg, local, world, dist if world > 1 else None)
    if not args.no_batch:
        line["water_batch1024"] = batch_leg(pkg, local, rank, world, dist if world > 1 else None)
    if not args.no_grad and rank == 0:
        line["gradients"] = grad_leg(pkg, local)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(pkg, S)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def _timed(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / steps


def large_leg(pkg, local, world, dist):
    """32768 waters (98304 atoms), 99.4 A box, 104^3 grid, order 6, mixed precision, tol 1e-4 and 1e-5: evals/s
    and ns/day at 2 fs (host call, positions and forces through host memory); replicas on N > 1."""
    import torch
    out = {"workload": "water98304", "atoms": 98304, "grid": [104, 104, 104]}
    S = pkg.systems.water98304()
    for tol in (1e-4, 1e-5):
        eng = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=tol, max_iter=200,
                                      peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT, precision=pkg.MIXED,
                                      device=local, skin=0.0))
        eng.set_system(S)
        eng.compute(S.pos, S.box)
        out["pair_lanes"] = eng.autotune(S.pos, S.box, reps=3)
        res = {}
        dt = _timed(lambda: res.__setitem__("r", eng.compute(S.pos, S.box)), 5, 2)
        t = torch.tensor([dt], dtype=torch.float64, device=f"cuda:{local}")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        v = world / float(t.item())
        out[f"tol{tol:g}"] = {"evals_per_s": v, "ms_per_eval": 1e3 * float(t.item()),
                              "ns_per_day_2fs": v / world * 86400 * 2e-6, "cg_iterations": res["r"].iterations}
        if tol == 1e-5:
            kt = eng.kernel_times(reps=5)
            flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
            kt_cold = eng.kernel_times(reps=5, flush_ptr=flush.data_ptr(), flush_bytes=flush.numel() * 4)
            del flush
            S.meta["pairs"] = eng.num_candidates()
            out["kernel_ms"] = kt
            out["roofline_per_kernel"] = roofline_table(S, kt, res["r"].iterations, 1, kt_cold)["per_kernel"]
        eng.close()
    return out


def batch_leg(pkg, local, rank, world, dist):
    """1024 independent water boxes of 8..512 molecules (0.0334 / A^3, grids <= 1 A spacing with 2-3-5 sizes,
    cutoff min(9 A, L/2), tol 1e-5, mixed) in one launch per rank (systems partitioned by atom count across
    ranks), against the same systems evaluated one after the other by single-system engines (a sample of 64, on
    rank 0); with the main kernels' times and the field pair pass against the HBM roofline."""
    import torch
    import pgm_md_b200.shard as sh
    systems = pkg.systems.water_batch(nsys=1024, seed=1024, tol=1e-5)
    parts = sh.partition([s.n for s in systems], world)
    mine = [systems[k] for k in parts[rank]]
    eng = pkg.Engine(pkg.Settings(cutoff=0.9, beta=3.5, grid=(24, 24, 24), order=6, tol=1e-5, max_iter=200,
                                  peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT, precision=pkg.MIXED,
                                  device=local, skin=0.0))
    eng.set_systems(mine)
    pos = np.concatenate([s.pos for s in mine])
    boxes = np.stack([s.box for s in mine])
    lanes = eng.autotune(pos, boxes, reps=3)
    chosen = eng.transforms()
    res = {}
    per_mode = {}
    for mode in (0, 1, 2, 3, 4):   # every kind of transforms timed (every rank the same steps); the autotuned one reported
        eng.set_transforms(mode)
        if eng.transforms() != mode:
            continue
        dt = _timed(lambda: res.__setitem__("r", eng.compute_batch(pos, boxes)), 5, 2)
        t = torch.tensor([dt], dtype=torch.float64, device=f"cuda:{local}")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        per_mode[mode] = float(t.item())
    eng.set_transforms(chosen)
    res["r"] = eng.compute_batch(pos, boxes)
    active = eng.active_systems()
    dt = per_mode[chosen]
    # main kernels relaunched alone; the field pair pass streams P x 24-byte pair records (mixed) from HBM here
    kt = eng.kernel_times(reps=3)
    npairs = eng.num_candidates()
    peak, peak_kind = peaks()
    pf_bytes = npairs * 4 + eng.n * 40          # the algorithmic bytes: a list index per pair, 10 reals per atom
    pf_design = npairs * 24 + eng.n * 40        # the engine's 24 B pair records
    pf_gbs = pf_bytes / (kt["pair_field"] * 1e-3) / 1e9
    energies = sh.gather_energies(parts[rank], res["r"]["energies"], len(systems))
    out = {"workload": "water_batch1024", "systems": len(systems), "atoms": int(sum(s.n for s in systems)),
           "systems_per_s": len(systems) / dt, "ms_per_batch": 1e3 * dt,
           "max_cg_iterations": int(res["r"]["iterations"].max()), "partition": "atom-balanced, one launch per rank",
           "active_systems_per_iteration": active,
           "pair_lanes": lanes, "transforms": TRANSFORMS[chosen],
           "ms_per_batch_by_transforms": {TRANSFORMS[m]: 1e3 * v for m, v in per_mode.items()},
           "directed_pairs": npairs, "kernel_ms": kt,
           "pair_field_roofline": {"bound": "hbm", "bytes_per_launch": pf_bytes, "achieved": pf_gbs, "peak": peak,
                                   "unit": "GB/s", "frac": pf_gbs / peak, "peak_source": peak_kind,
                                   "design_bytes": pf_design,
                                   "design_frac": pf_design / (kt["pair_field"] * 1e-3) / 1e9 / peak},
           "energies_finite": bool(np.isfinite(energies).all())}
    eng.close()
    if rank == 0:
        sample = systems[:: len(systems) // 64][:64]
        engines = []
        for S in sample:
            e = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-5, max_iter=200,
                                        peek=0.65, predictor=0, ke=pkg.systems.KE_DEFAULT, precision=pkg.MIXED,
                                        device=local, skin=0.0))
            e.set_system(S)
            e.compute(S.pos, S.box)
            engines.append((e, S))
        ts = _timed(lambda: [e.compute(S.pos, S.box) for e, S in engines], 2, 1)
        per = ts / len(engines)
        out["sequential_systems_per_s"] = 1.0 / per
        out["sequential_sample"] = f"{len(engines)} systems, one engine each, evaluated one after the other"
        out["batched_over_sequential"] = out["systems_per_s"] / world / out["sequential_systems_per_s"]
        for e, _ in engines:
            e.close()
    return out


def grad_leg(pkg, local):
    """Parameter gradients of the differentiation workload: dE/d(per-atom q, R, alpha; per-dipole strength) (the
    stationary energy's partial derivatives) and the force-matching gradient dL/d(same) of L = sum |F - F_t|^2
    (one adjoint solve with analytic tangent passes), for (a) the 256 boxes of 64 waters in one batched
    evaluation and (b) the 8550-atom liquid, both precisions, tol 1e-8, peek 0.  F_t: the forces at parameters
    scaled by (1 + N(0, 0.05))."""
    import pgm_md_b200.autograd as ag
    out = {}
    boxes = pkg.systems.water64_boxes(nsys=256)
    _, S = system()
    for name, prec in (("mixed", pkg.MIXED), ("fp64", pkg.FP64)):
        eng = pkg.Engine(pkg.Settings(cutoff=boxes[0].cutoff, beta=boxes[0].beta, grid=boxes[0].grid, order=6,
                                      tol=1e-8, max_iter=300, peek=0.0, predictor=0, ke=pkg.systems.KE_DEFAULT,
                                      precision=prec, device=local))
        eng.set_systems([pkg.systems.perturbed(b, rel=0.05, seed=1 + k) for k, b in enumerate(boxes)])
        pos = np.concatenate([b.pos for b in boxes])
        bx = np.stack([b.box for b in boxes])
        Ft = eng.compute_batch(pos, bx)["forces"]
        eng.set_systems(boxes)

        def batch_energy_grad():
            eng.compute_batch(pos, bx)
            eng.param_grad()

        dt = _timed(batch_energy_grad, 5, 2)
        out[f"water64x256_energy_grad_{name}"] = {"systems_per_s": 256 / dt, "ms_per_batch": 1e3 * dt}
        dt = _timed(lambda: ag.force_matching_atom_grads(eng, boxes, Ft, tol=1e-8), 3, 1)
        out[f"water64x256_force_matching_grad_{name}"] = {"systems_per_s": 256 / dt, "ms_per_batch": 1e3 * dt}
        eng.close()
        eng = pkg.Engine(pkg.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-8, max_iter=300,
                                      peek=0.0, predictor=0, ke=pkg.systems.KE_DEFAULT, precision=prec,
                                      device=local))
        eng.set_system(pkg.systems.perturbed(S, rel=0.05, seed=4))
        Ft1 = eng.compute(S.pos, S.box).forces
        eng.set_system(S)

        def single_energy_grad():
            eng.compute(S.pos, S.box)
            eng.param_grad()

        dt = _timed(single_energy_grad, 5, 2)
        out[f"dimethylphenol8550_energy_grad_{name}"] = {"evals_per_s": 1.0 / dt, "ms": 1e3 * dt}
        dt = _timed(lambda: ag.force_matching_atom_grads(eng, S, Ft1, tol=1e-8), 3, 1)
        out[f"dimethylphenol8550_force_matching_grad_{name}"] = {"evals_per_s": 1.0 / dt, "ms": 1e3 * dt}
        eng.close()
    return out


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def _oracle_reference(pkg, S, tol):
    from oracle import pgm_oracle as O
    from oracle import ref as R
    top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
    st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=tol, max_iter=1000, peek=0.0,
                    predictor=0, ke=pkg.systems.KE_DEFAULT)
    names = ("direct", "reciprocal", "self", "background", "polarization")
    if R.available():
        e = R.RefEngine(top, st)
        E = e.compute(S.pos, S.box)
        t = e.terms()
        return dict(energy=E, forces=e.forces, terms=[t[k] for k in names], mu=e.induced(), strain=e.strain(),
                    kind="reference pgm_core (oracle/_ref), tol 1e-10")
    e = O.Engine(top, st)
    E = e.compute(S.pos, S.box)
    return dict(energy=E, forces=e.forces, terms=[e.terms[k] for k in names], mu=e.mu, strain=e.strain,
                kind="numpy oracle, tol 1e-10")


def accuracy(pkg, S, mixed, fp64, make_refined=None):
    """Errors of the GPU paths (at the benchmark tolerance) against the FP64 oracle at tol 1e-10: the total
    energy, every energy term (relative to the term, and to the total), the forces (relative RMS), the strain
    derivative and the induced dipoles (relative RMS and largest component error relative to the largest
    dipole); the mixed path with FP64 refinement also timed (host call, direct launches)."""
    ref = _oracle_reference(pkg, S, 1e-10)
    E0, F0, mu0 = ref["energy"], ref["forces"], ref["mu"]
    out = {"oracle": ref["kind"]}
    engines = [("mixed", mixed), ("fp64", fp64)]
    if make_refined is not None:
        engines.append(("mixed_fp64_refined", make_refined()))
    names = ("direct", "reciprocal", "self", "background", "polarization")
    for name, eng in engines:
        r = eng.compute(S.pos, S.box)
        mu = eng.induced_dipoles()
        td = r.terms.as_dict()
        out[name] = {"force_rel_rms": float(np.linalg.norm(r.forces - F0) / np.linalg.norm(F0)),
                     "energy_rel": float(abs(r.energy - E0) / abs(E0)), "iterations": r.iterations,
                     "term_rel": {k: (float(abs(td[k] - ref["terms"][j]) / abs(ref["terms"][j]))
                                      if abs(ref["terms"][j]) > 1e-12 * abs(E0) else None)
                                  for j, k in enumerate(names)},
                     "term_err_over_total": {k: float(abs(td[k] - ref["terms"][j]) / abs(E0))
                                             for j, k in enumerate(names)},
                     "strain_rel_max": float(np.abs(r.strain - ref["strain"]).max() / np.abs(ref["strain"]).max()),
                     "dipole_rel_rms": float(np.linalg.norm(mu - mu0) / np.linalg.norm(mu0)),
                     "dipole_max_err_rel": float(np.abs(mu - mu0).max() / np.abs(mu0).max())}
        if name == "mixed_fp64_refined":
            dt = _timed(lambda: eng.compute(S.pos, S.box), 5, 1)
            out[name]["evals_per_s_host_call"] = 1.0 / dt
            eng.close()
    return out


def cpu_baseline(pkg, S):
    """The reference pgm_core on one host core: two full evaluations of the same workload."""
    from oracle import pgm_oracle as O
    from oracle import ref as R
    if not R.available():
        return None
    top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
    st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=TOL, max_iter=500, peek=0.65,
                    predictor=0, ke=pkg.systems.KE_DEFAULT)
    e = R.RefEngine(top, st)
    e.compute(S.pos, S.box)
    n = 2
    t0 = time.perf_counter()
    for _ in range(n):
        R.lib().ref_reset_history(e.h)
        e.compute(S.pos, S.box)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "evals/s", "cores": 1, "kind": "reference",
            "sample": f"{n} full evaluations of {WORKLOAD} (pgm_core, single-threaded)", "cpu": cpu_model()}


def cpu_model():
    """The host CPU's model name and logical core count (from /proc/cpuinfo)."""
    name, count = None, 0
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                count += 1
                name = name or ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return {"model": name, "logical_cores": count or os.cpu_count()}


if __name__ == "__main__":
    sys.exit(main())
