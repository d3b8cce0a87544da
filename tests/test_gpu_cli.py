"""GPU: the drop-in `scc` driver against the reference's own CLI (compiled from
its sources into oracle/_ref/scc) on the same text edge list: the stdout lines
scripts parse, the SCC count, and a byte-identical scc_list.txt."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import random_graph, seeded_graph

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUR_CLI = os.path.join(ROOT, "dynamicgraphs_scc_b200", "lib", "scc")


def write_edges(path, s, d):
    with open(path, "w") as f:
        for a, b in zip(s.tolist(), d.tolist()):
            f.write(f"{a + 1} {b + 1}\n")


def parse(out):
    info = {}
    for line in out.splitlines():
        if line.startswith("data="):
            info["data"] = line.split("=", 1)[1].split(" ")
        m = re.match(r"\[(\d+)\]running_time\(ms\)=([0-9.]+)", line)
        if m:
            info["threads"] = int(m.group(1)); info["ms"] = float(m.group(2))
        if "Total # SCCs" in line:
            info["sccs"] = int(line.split("=")[1])
    return info


def graphs():
    n, s, d, _ = seeded_graph(rmat_scale=12, edge_factor=8, grid_side=48, seed=6)
    # make vertex n-1 an endpoint so the loader's N = max id equals n
    s = np.append(s, n - 1).astype(np.int32); d = np.append(d, 0).astype(np.int32)
    yield "rmat_grid", s, d
    s2, d2 = random_graph(3000, 5000, 4)
    s2 = np.append(s2, 2999).astype(np.int32); d2 = np.append(d2, 2999).astype(np.int32)
    yield "random_loops_dups", s2, d2


@pytest.mark.parametrize("case", [0, 1])
def test_cli_matches_reference_cli(gpu, tmp_path, case):
    name, s, d = list(graphs())[case]
    g = tmp_path / f"{name}.txt"
    write_edges(g, s, d)
    ours_dir = tmp_path / "ours"; ours_dir.mkdir()
    r = subprocess.run([OUR_CLI, str(g), "4", "2", "-p"], cwd=ours_dir, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    mine = parse(r.stdout)
    assert mine["data"] == [str(g), "2", "4"] and mine["threads"] == 4
    n = int(max(s.max(), d.max())) + 1
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    assert mine["sccs"] == len(np.unique(exp))
    ours_list = (ours_dir / "scc_list.txt").read_text()
    if os.path.exists(O.REF_CLI):
        ref_dir = tmp_path / "ref"; ref_dir.mkdir()
        rr = subprocess.run([O.REF_CLI, str(g), "4", "2", "-p"], cwd=ref_dir, capture_output=True, text=True,
                            timeout=300)
        assert rr.returncode == 0
        ref = parse(rr.stdout)
        assert ref["sccs"] == mine["sccs"]
        assert (ref_dir / "scc_list.txt").read_text() == ours_list
    else:
        first = {}
        lines = []
        for i, r_ in enumerate(exp.tolist()):
            first.setdefault(r_, len(first))
            lines.append(f"{i} {first[r_]}")
        assert ours_list == "\n".join(lines) + "\n"


def test_cli_methods_and_flags(gpu, tmp_path):
    _, s, d = list(graphs())[0]
    g = tmp_path / "g.txt"
    write_edges(g, s, d)
    counts = set()
    for method in ("0", "1", "2"):
        r = subprocess.run([OUR_CLI, str(g), "1", method, "-d"], cwd=tmp_path, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        assert "[TRIM1 phase:" in r.stdout and "[FB phase:" in r.stdout
        counts.add(parse(r.stdout)["sccs"])
    assert len(counts) == 1
    r = subprocess.run([OUR_CLI, str(g), "1", "2", "-a"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "1 => " in r.stdout
    r = subprocess.run([OUR_CLI, str(g), "1", "3"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 1 and "unsupported" in r.stderr
    r = subprocess.run([OUR_CLI, str(tmp_path / "missing.txt"), "1", "2"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 1


def _line(out, prefix):
    for line in out.splitlines():
        if line.startswith(prefix):
            return line[len(prefix):].strip()
    return None


def test_cli_update_methods(gpu, tmp_path):
    """Methods 5-11 as the reference driver runs them: the batch file, the
    original graph in refined_edges.txt beside it, the previous decomposition
    in scc_list.txt (written by a method-2 "-p" run)."""
    rng = np.random.default_rng(21)
    n = 6000
    s, d = random_graph(n, 9000, 8)
    s = np.append(s, n - 1).astype(np.int32); d = np.append(d, 0).astype(np.int32)
    write_edges(tmp_path / "refined_edges.txt", s, d)
    r = subprocess.run([OUR_CLI, str(tmp_path / "refined_edges.txt"), "1", "2", "-p"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    labels = O.tarjan_canonical(*O.build_csr(n, s, d)[:2])
    ids, k = O.scc_ids(labels)
    isrc = rng.integers(0, n, 12).astype(np.int32); idst = rng.integers(0, n, 12).astype(np.int32)
    isrc[-1] = n - 1                                # the batch's N must not exceed the graph's
    write_edges(tmp_path / "ins.txt", isrc, idst)
    upd = O.tarjan_canonical(*O.build_csr(n, np.concatenate([s, isrc]), np.concatenate([d, idst]))[:2])
    b, a = O.condensation_csr(ids, k, s, d)
    lev, ml = O.topo_levels(b, a)
    _, unaffected = O.affected_levels(ids, lev, ml, isrc, idst)
    for method in ("5", "6", "7", "11"):
        r = subprocess.run([OUR_CLI, str(tmp_path / "ins.txt"), "2", method, "-d"], cwd=tmp_path,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (method, r.stderr)
        info = parse(r.stdout)
        assert info["data"] == [str(tmp_path / "ins.txt"), method, "2"]
        assert info["sccs"] == len(np.unique(upd)), method
        if method == "7":
            assert int(_line(r.stdout, "max_level:")) == ml
            assert int(_line(r.stdout, "size of unaffected_levels:")) == unaffected
            assert _line(r.stdout, "Trimmed nodes=") == "0"
    # deletions: one edge inside a non-trivial SCC, one across SCCs
    big = np.flatnonzero((labels[s] == labels[d]) & (s != d))
    cross = np.flatnonzero(labels[s] != labels[d])
    pick = np.array([big[0], cross[0]])
    dsrc, ddst = s[pick].astype(np.int32), d[pick].astype(np.int32)
    write_edges(tmp_path / "del.txt", dsrc, ddst)
    gone = np.zeros(s.size, bool)
    for x, y in zip(dsrc.tolist(), ddst.tolist()):
        gone |= (s == x) & (d == y)
    after = O.tarjan_canonical(*O.build_csr(n, s[~gone], d[~gone])[:2])
    for method in ("8", "9", "10"):
        r = subprocess.run([OUR_CLI, str(tmp_path / "del.txt"), "1", method], cwd=tmp_path,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (method, r.stderr)
        assert parse(r.stdout)["sccs"] == len(np.unique(after)), method
        if method == "9":
            assert _line(r.stdout, "affect_sccs:") == f"1 unaffect_sccs:{k - 1}"
    # a batch naming a vertex beyond the original graph is an error
    write_edges(tmp_path / "bad.txt", np.array([0], np.int32), np.array([n + 5], np.int32))
    r = subprocess.run([OUR_CLI, str(tmp_path / "bad.txt"), "1", "6"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 1
