"""The roofline arithmetic of bench.py's bench line (advance_roofline): the
algorithmic work per unit of k_advance, FP32 node tests counted at 40 B and
16 FP32 FLOP with the undecided ones re-tested in FP64 (48 B, 12 FLOP), or
FP64 node tests at 64 B and 12 FLOP; the tail's share left out; the bound
named by the largest fraction of its peak."""
import bench


def _stats():
    return {"node_tests": 11_000_000, "tail_node_tests": 1_000_000, "cell_tests": 52_000_000,
            "tail_cell_tests": 2_000_000, "tri_tests": 5_500_000, "tail_tri_tests": 500_000,
            "node_tests_fp64": 4_000, "advance_ms": 5.0, "rounds": 4}


def test_fp32_node_model(monkeypatch):
    monkeypatch.setattr(bench, "NODE_F32", True)
    r = bench.advance_roofline(_stats(), fp64_peak=30.0, fp32_peak=60.0, l2_peak=16000.0)
    secs = 5e-3
    nbytes = 40 * 10_000_000 + 48 * 4_000 + 24 * 50_000_000 + 104 * 5_000_000
    assert abs(r["pipes"]["hbm"]["achieved"] - nbytes / secs / 1e9) < 1e-6
    assert abs(r["pipes"]["fp32"]["achieved"] - (16 * 10_000_000 + 18 * 50_000_000) / secs / 1e12) < 1e-9
    assert abs(r["pipes"]["fp64"]["achieved"] - (12 * 4_000 + 46 * 5_000_000) / secs / 1e12) < 1e-9
    assert r["bound"] == max(r["pipes"], key=lambda k: r["pipes"][k]["frac"])
    assert r["frac"] == r["pipes"][r["bound"]]["frac"] and r["kernel"] == "k_advance"


def test_fp64_node_model(monkeypatch):
    monkeypatch.setattr(bench, "NODE_F32", False)
    r = bench.advance_roofline(_stats(), fp64_peak=30.0, fp32_peak=60.0, l2_peak=16000.0)
    secs = 5e-3
    nbytes = 64 * 10_000_000 + 24 * 50_000_000 + 104 * 5_000_000
    assert abs(r["pipes"]["l2"]["achieved"] - nbytes / secs / 1e9) < 1e-6
    assert abs(r["pipes"]["fp64"]["achieved"] - (12 * 10_000_000 + 46 * 5_000_000) / secs / 1e12) < 1e-9


def test_no_time_no_roofline():
    s = _stats()
    s["advance_ms"] = 0.0
    assert bench.advance_roofline(s, 30.0, 60.0, 16000.0) is None
