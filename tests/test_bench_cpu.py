"""The roofline arithmetic of bench.py on a synthetic kernel-family profile:
the dominant family by time, achieved = algorithmic bytes per launch over
the average launch duration, the fraction of the peak, the DRAM traffic
scaled from the ncu ratio, and the family shares summing to one."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, str(ROOT))
    import bench as b
    return b


def test_roofline_of_the_dominant_family(bench):
    prof = {
        "sgs": {"ms": 20.0, "launches": 100, "bytes": 100 * 0.5e9},   # 0.2 ms and 0.5 GB per launch
        "spmv": {"ms": 10.0, "launches": 20, "bytes": 20 * 1.0e9},
        "lu": {"ms": 0.0, "launches": 0, "bytes": 0.0},               # not launched: left out
        "krylov": {"ms": 2.0, "launches": 40, "bytes": 40 * 4.0e7},
    }
    r = bench._roofline(prof, 6500.0, "measured")
    assert r["kernel"] == "sgs" and r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["achieved"] == pytest.approx(0.5e9 / 0.2e-3 / 1e9, rel=1e-9)  # 2500 GB/s
    assert r["frac"] == pytest.approx(2500.0 / 6500.0, abs=1e-4)
    assert r["traffic"] == round(0.5e9 * bench.TRAFFIC_PER_ALG_BYTE["sgs"])
    assert set(r["families"]) == {"sgs", "spmv", "krylov"}
    assert sum(f["ms_per_step_share"] for f in r["families"].values()) == pytest.approx(1.0, abs=1e-3)
    assert list(r["families"])[0] == "sgs"  # ordered by time


def test_roofline_without_an_ncu_ratio_reports_no_traffic(bench):
    prof = {"jacobian": {"ms": 5.0, "launches": 1, "bytes": 1.0e9}}
    r = bench._roofline(prof, 6650.0, "fallback")
    assert r["kernel"] == "jacobian" and r["traffic"] is None and r["peak_source"] == "fallback"


def test_replica_throughput_is_whole_job(bench):
    # 2 replicas of 1M cells, 10 iterations each in 50 ms (slowest rank)
    assert bench.replica_throughput(2, 1_000_000, 10, 50.0) == pytest.approx(400.0)
