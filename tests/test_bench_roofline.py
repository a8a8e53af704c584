"""bench.py's SGD roofline arithmetic, on the CPU: the contract's HBM view
(algorithmic bytes 4 nnz + 56 F + 8 N_neg per epoch over the stage time,
against the measured HBM peak) with the L2 random-access view beside it,
checked on the counts and times of a measured 1M-point run (the figures its
line reported: 906.6 GB/s, 0.1405 of HBM, 0.2827 of the L2 ceiling)."""
import json

import bench


def test_sgd_roofline_reproduces_a_measured_line():
    peaks = {"hbm_gbs": 6454.3, "source": "measured"}
    l2 = {"gather_per_s": 289.5e9, "atomic_add_per_s": 195.3e9}
    r = bench.sgd_roofline(25_953_500, 200, 1_449_480_438, 7_226_298_288, 176.199, peaks, l2, 610_600_000.0, "capture")
    json.dumps(r)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] == 6454.3
    assert abs(r["achieved"] - 906.6) <= 0.2
    assert abs(r["frac"] - 0.1405) <= 1e-4 and abs(r["frac"] - r["achieved"] / r["peak"]) <= 1e-4
    assert abs(r["frac_l2"] - 0.2827) <= 2e-4
    assert abs(r["frac_l2"] - r["achieved_l2"] / r["peak_l2"]) <= 1e-3
    assert r["traffic"] == 610_600_000.0
    expect = (4 * 25_953_500 * 200 + 56 * 1_449_480_438 + 8 * 7_226_298_288) / 200
    assert abs(r["algorithmic_bytes_per_launch"] - expect) <= 1


def test_stage_rooflines_bytes_and_fractions():
    peaks = {"hbm_gbs": 6454.3, "source": "measured"}
    r = bench.stage_rooflines(1_000_000, 15, 25_953_500, {"similarities": 2.108, "union": 2.523}, peaks)
    json.dumps(r)
    sim, uni = r["similarities"], r["union"]
    assert sim["algorithmic_bytes"] == 1_000_000 * 15 * 8 + 16 * 1_000_000
    assert uni["algorithmic_bytes"] == 1_000_000 * 15 * 8 + 25_953_500 * 8 + 1_000_001 * 8
    for x in (sim, uni):
        assert x["bound"] == "hbm" and x["unit"] == "GB/s"
        assert abs(x["achieved"] - x["algorithmic_bytes"] / (x["time_ms"] * 1e-3) / 1e9) <= 0.1
        assert abs(x["frac"] - x["achieved"] / 6454.3) <= 1e-4
    # a stage that did not run reports zero, not a division error
    assert bench.stage_rooflines(10, 3, 20, {}, peaks)["union"]["achieved"] == 0.0
