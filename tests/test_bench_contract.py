"""The bench line's roofline arithmetic, without a GPU: algorithmic bytes per launch follow the per-unit figures
of the hot path's byte convention (a pair-field launch moves a 4 B list index per directed pair plus 10 reals
per atom; the engine's own 24 B pair records are reported apart as design bytes), achieved = bytes / launch
time, frac = achieved / the peak, warm and cold, and the dominant kernel is the engine's own kernel with the
largest share of an evaluation (the FFT chain listed beside it, never chosen)."""

import importlib.util

import numpy as np
import pytest

from conftest import PKG, ROOT


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("pgm_b200_bench", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_algorithmic_bytes_per_unit(bench):
    S = PKG.systems.water216()
    S.meta["pairs"] = 1000
    n, p = S.n, S.order
    assert bench.algorithmic_bytes("pair_field", S, 1, 9) == 1000 * 4 + n * 10 * 4
    assert bench.algorithmic_bytes("pair_field", S, 0, 9) == 1000 * 4 + n * 10 * 8
    assert bench.design_bytes("pair_field", S, 1) == 1000 * 24 + n * (4 * 4 + 24)
    assert bench.design_bytes("pair_field", S, 0) == 1000 * (4 + 16) + n * (32 + 32 + 24)
    assert bench.algorithmic_bytes("spread", S, 1, 9) == n * (7 * 4 + p ** 3 * 4)
    assert bench.algorithmic_bytes("spread", S, 0, 9) == n * (7 * 8 + p ** 3 * 8)
    assert bench.algorithmic_bytes("gather", S, 1, 9) == n * (10 * 4 + p ** 3 * 4)
    G = int(np.prod(S.grid))
    Gc = S.grid[0] * S.grid[1] * (S.grid[2] // 2 + 1)
    assert bench.algorithmic_bytes("fft_chain", S, 1, 9) == 2 * (G * 4 + Gc * 8) + Gc * 16
    assert bench.algorithmic_bytes("cg_update", S, 1, 9) == 3 * n * 8 * 10
    assert bench.algorithmic_bytes("no_such_kernel", S, 1, 9) is None


def test_roofline_table_arithmetic(bench):
    S = PKG.systems.water216()
    S.meta["pairs"] = 200000
    it = 9
    kt = {"pair_list": 0.05, "pair_field": 0.010, "spread": 0.008, "gather": 0.009, "pair_final": 0.02,
          "fft_chain": 0.5, "cg_update": 0.004}
    kt_cold = {k: 1.5 * v for k, v in kt.items()}
    roof = bench.roofline_table(S, kt, it, 1, kt_cold)
    peak, _ = bench.peaks()
    for k, ms in kt.items():
        row = roof["per_kernel"][k]
        assert row["launches_per_eval"] == bench.launches_per_eval(k, it)
        b = bench.algorithmic_bytes(k, S, 1, it)
        assert row["bytes_per_launch"] == b
        assert row["achieved_gbs"] == pytest.approx(b / (ms * 1e-3) / 1e9)
        assert row["frac"] == pytest.approx(row["achieved_gbs"] / peak)
        assert row["frac_cold"] == pytest.approx(b / (1.5 * ms * 1e-3) / 1e9 / peak)
        assert row["design_bytes"] == bench.design_bytes(k, S, 1)
    shares = {k: ms * bench.launches_per_eval(k, it) for k, ms in kt.items() if k != "fft_chain"}
    assert roof["kernel"] == max(shares, key=shares.get) != "fft_chain"
    assert roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"])
    assert roof["frac_cold"] == pytest.approx(roof["frac"] / 1.5)
    assert roof["bound"] == "hbm" and roof["unit"] == "GB/s" and "note" in roof
    assert sum(r["share"] for r in roof["per_kernel"].values()) == pytest.approx(1.0)
