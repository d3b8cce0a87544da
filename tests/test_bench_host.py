"""CPU: the benchmark's host-side pieces -- the seeded `hubs` workload, the
tuning option, and the reference arm's lines for the configurations the
reference has no mode for (no GPU needed)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_hub_edges_seeded_and_in_range():
    kw = dict(hubs_n=4096, hubs=40, hub_deg=(64, 400), seed=3)
    n, s, d = bench.hub_edges(**kw)
    n2, s2, d2 = bench.hub_edges(**kw)
    assert n == n2 == 4096
    assert np.array_equal(s, s2) and np.array_equal(d, d2)
    assert s.dtype == np.int32 and d.dtype == np.int32
    assert s.min() >= 0 and d.min() >= 0 and s.max() < n and d.max() < n
    out_deg = np.bincount(s, minlength=n)
    in_deg = np.bincount(d, minlength=n)
    # every vertex keeps out-degree 2; 40 hubs add 64..399 out- and in-edges
    assert (out_deg >= 2).all()
    assert (out_deg >= 2 + 64).sum() == 40
    assert in_deg.max() >= 64


def test_workload_edges_dispatch():
    n, s, d = bench.workload_edges(bench.CPU_SAMPLES["hubs"])
    assert n == bench.CPU_SAMPLES["hubs"]["hubs_n"] and s.size == d.size > 2 * n
    from dynamicgraphs_scc_b200 import generate_edges_host
    n1, s1, d1 = bench.workload_edges(bench.WORKLOADS["c1"])
    n2, s2, d2 = generate_edges_host(**bench.WORKLOADS["c1"])
    assert n1 == n2 and np.array_equal(s1, s2) and np.array_equal(d1, d2)


def test_parse_tuning():
    assert bench.parse_tuning("") == {}
    assert bench.parse_tuning("bu_alpha=1,cta_deg=256") == {"bu_alpha": 1, "cta_deg": 256}
    assert bench.parse_tuning(" tail_live=-1 ") == {"tail_live": -1}
    with pytest.raises(ValueError):
        bench.parse_tuning("bu_alpha")


@pytest.mark.parametrize("workload", ["c4", "c5"])
def test_reference_arm_unavailable_lines(workload):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", workload],
                       capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
