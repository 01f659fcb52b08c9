"""Host-side figures of bench.py that need no GPU: which tiling the committed
ncu summary describes, the state-update HBM roofline arithmetic, and the
workload name both arms of the bench report."""
import json
import os

import pytest

import bench
from pawan_b200 import geometry as g


def test_profile_figures_apply_only_to_the_profiled_tiling():
    prof = bench.profile_summary()
    if not prof.get("tile"):
        pytest.skip("no committed ncu summary")
    tile = dict(prof["tile"], items_per_slot=64)
    assert bench.profiled_tiling_matches(tile)
    # the chunking does not change the DRAM bytes (chunk sums stay in L2)
    assert bench.profiled_tiling_matches(dict(tile, items_per_slot=128))
    assert bench.traffic_from_profiles(tile) == prof["dram_bytes_per_launch_full_size"]
    ex = bench.executed_from_profiles(tile)
    assert ex["same_tiling"] and ex["profiled_kernel"] == prof["kernel"]
    other = dict(tile, packed=2 if tile["packed"] != 2 else 1)
    assert not bench.profiled_tiling_matches(other)
    assert bench.traffic_from_profiles(other) is None
    assert bench.executed_from_profiles(other)["same_tiling"] is False


def test_state_update_roofline_arithmetic():
    peak, src = bench.hbm_peak()
    r = bench.state_update_roofline({"stage_ms": 2.0, "stage_launches": 4, "stage_bytes": 4 * 1.0e8})
    assert r["ms_per_launch"] == pytest.approx(0.5)
    assert r["bytes_per_launch"] == pytest.approx(1.0e8)
    assert r["achieved"] == pytest.approx(1.0e8 / 0.5e-3 / 1e9)  # 200 GB/s
    assert r["frac"] == pytest.approx(r["achieved"] / peak)
    assert r["peak_source"] == src and r["unit"] == "GB/s" and r["bound"] == "hbm"


def test_hbm_peak_reads_the_measured_file(tmp_path, monkeypatch):
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6000.5}))
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    peak, src = bench.hbm_peak()
    assert peak == 6000.5 and src.startswith("measured")
    os.remove(tmp_path / "MEASURED_PEAKS.json")
    peak, src = bench.hbm_peak()
    assert peak == 6650.0 and src.startswith("fallback")


def test_both_arms_name_the_same_workload():
    sc = g.ring_pair(steps=1)
    name = bench.workload_name(sc)
    assert name == "leapfrogging coaxial ring pair, N=131072, nu=0.0001, dt=0.005, RK4 step"
