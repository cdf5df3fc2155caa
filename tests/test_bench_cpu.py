"""bench.py's roofline fields from the committed ncu record (no GPU): frac
is measured DRAM traffic per launch over the kernel time against the peak,
the algorithmic bytes are reported beside it, and the issue fraction is the
captured warp instructions against 4 per SM per cycle."""
import json
import os

import bench


def test_roofline_from_the_committed_record():
    rec = bench.profile_record("learned")
    assert rec is not None, "profiles/triangle_kernel_rmat22_learned_dram.json is missing"
    for k in ("dram_bytes_read", "dram_bytes_write", "warp_instructions", "candidates", "command"):
        assert k in rec, k
    assert "--clock-control none" in rec["command"]
    kernel_ms, alg, wedges, peak = 8.0, 173602877880, int(rec["candidates"]), 6545.0
    r = bench.roofline(kernel_ms, alg, wedges, "learned", peak, "measured (hbm_gbs)", 1965.0)
    traffic = int(rec["dram_bytes_read"]) + int(rec["dram_bytes_write"])
    assert r["traffic"] == traffic
    assert abs(r["achieved"] - traffic / 8e-3 / 1e9) < 1e-6
    assert abs(r["frac"] - traffic / 8e-3 / 1e9 / peak) < 1e-9
    assert abs(r["alg_over_peak"] - alg / 8e-3 / 1e9 / peak) < 1e-9
    issue = r["issue"]
    assert abs(issue["issue_frac"] - int(rec["warp_instructions"]) / (4 * 148 * 1965e6 * 8e-3)) < 1e-9
    assert abs(issue["per_candidate"] - int(rec["warp_instructions"]) / wedges) < 1e-12
    assert r["bound"] == "hbm" and 0 < r["frac"] < 1.2


def test_roofline_without_a_record_reports_no_fraction():
    r = bench.roofline(8.0, 1, 1, "no-such-layout", 6545.0, "measured", None)
    assert r["frac"] is None and r["traffic"] is None and r["achieved"] is None


def test_measured_peaks_committed():
    p = os.path.join(bench.ROOT, "MEASURED_PEAKS.json")
    d = json.load(open(p))
    assert d["hbm_gbs"] > 1000
