"""bench.py's host-side pieces, on the CPU: the per-class DRAM traffic read
from the committed ncu summaries (roofline.traffic) and the workload table."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_default_workload_traffic_parses(bench):
    """Both kernel classes of the default workload carry a per-step byte
    count; the table pass writes at least the 34.4 GB of int32 level and
    parent tables (1024 sources x 2^22 vertices x 8 bytes)."""
    tr = bench.traffic_from_profile("rmat22_k1024")
    assert set(tr) == {"0", "1"}
    assert tr["0"] > 1e9
    assert tr["1"] >= 1024 * (1 << 22) * 8


def test_missing_traffic_profile_reads_as_none(bench):
    assert bench.traffic_from_profile("no_such_workload") is None


def test_every_traffic_profile_names_a_workload(bench):
    """Each committed traffic_<workload>.txt belongs to a workload bench.py
    can run, so no summary is orphaned."""
    prof = os.path.join(ROOT, "profiles")
    for f in os.listdir(prof):
        if f.startswith("traffic_") and f.endswith(".txt"):
            assert f[len("traffic_"):-len(".txt")] in bench.WORKLOADS, f
