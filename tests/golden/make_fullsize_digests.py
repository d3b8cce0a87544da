"""Record the reference's own labels on the full-size configurations as digests.

For the large mixed-structure graph (R-MAT s24 ef16 U 4096x4096 oriented grid)
and the planted-cycles graph (R-MAT s24 ef16 + 1,000 directed cycles), this
script builds the seeded edge list on the host, removes self-loops and
duplicates, builds gm_graph's sorted CSR, and runs the reference's own code
paths on it, compiled from its sources by oracle/Makefile into
oracle/_ref/libscc_ref.so:

  * do_tarjan_all (src/scc_tarjan.cc:137-149), on one large-stack thread;
  * method 2, do_baseline_global_wcc_fb (src/scc_main.cc:272-351 via
    my_main::run, src/scc_main.cc:120-145), on all host cores;
  * method 1, do_baseline_global_fb (src/scc_main.cc:222-270), on all host
    cores, where method 2 cannot run.

Each reference call runs in a child process, so a crash of the reference is
recorded (with its signal) instead of ending the script.  On the mixed graph
method 2 reads past its pool of 65,536 node sets (init_node_set_pool(65536),
src/scc_weak.cc:35; get_node_set_from_pool takes one per weak component with
no bound check, :24-29): the oriented grid leaves more weak components than
that after trimming.

Every label array that was produced is relabelled canonically (component id =
smallest member vertex) and must equal Tarjan's.  The arrays themselves
(64-134 MB each) are not stored: tests/golden/fullsize_digests.json keeps the
SHA-256 of the canonical labels as little-endian int32, the SCC count, the
size of the largest SCC, a SHA-256 of the CSR (so a test can tell that it
decomposed the same graph) and the reference's timings on this host.

    python tests/golden/make_fullsize_digests.py [name ...]
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "fullsize_digests.json")

FULL = {
    "c2": dict(rmat_scale=24, edge_factor=16, grid_side=4096, seed=2024),
    "c3": dict(rmat_scale=24, edge_factor=16, num_cycles=1000, cycle_min=3, cycle_max=100000, seed=2024),
}

# one reference call in a child process: reads the CSR, writes canonical labels
_CHILD = r"""
import sys, json, numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import oracle as O
b = np.load(sys.argv[2]); a = np.load(sys.argv[3])
what = sys.argv[4]
if what == "tarjan":
    lab, ms = O.ref_tarjan((b, a))
else:
    lab, ms = O.ref_method(int(what[1:]), (b, a), threads=int(sys.argv[6]))
np.save(sys.argv[5], lab)
print(json.dumps({"ms": ms}))
"""


def sha256_i32(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


def csr_digest(begin, adj) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(begin, dtype="<i4").tobytes())
    h.update(np.ascontiguousarray(adj, dtype="<i4").tobytes())
    return h.hexdigest()


def label_summary(lab):
    lab = np.asarray(lab, np.int32)
    roots = lab == np.arange(lab.size, dtype=np.int32)
    sizes = np.bincount(lab)
    return {"labels_sha256": sha256_i32(lab), "num_sccs": int(np.count_nonzero(roots)),
            "largest_scc": int(sizes.max()) if sizes.size else 0}


def run_child(tmp, what, threads):
    out = os.path.join(tmp, f"{what}.npy")
    t0 = time.perf_counter()
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, os.path.join(tmp, "b.npy"), os.path.join(tmp, "a.npy"),
                        what, out, str(threads)], capture_output=True, text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        sig = -r.returncode if r.returncode < 0 else None
        return None, {"status": f"crashed (signal {sig})" if sig else f"failed (exit {r.returncode})",
                      "wall_s": round(wall, 1)}
    ms = json.loads(r.stdout.strip().splitlines()[-1])["ms"]
    return np.load(out), {"status": "ok", "ms": round(ms, 1), "wall_s": round(wall, 1)}


def record(name: str) -> dict:
    from oracle import oracle as O
    from dynamicgraphs_scc_b200 import generate_edges_host
    kw = FULL[name]
    t0 = time.perf_counter()
    n, s, d = generate_edges_host(**kw)
    s, d = O.dedup_edges(s, d, n=n)
    b, a, _, _ = O.build_csr(n, s, d)
    del s, d
    threads = os.cpu_count() or 1
    ref = {"host_build_s": round(time.perf_counter() - t0, 1), "threads": threads}
    with tempfile.TemporaryDirectory() as tmp:
        np.save(os.path.join(tmp, "b.npy"), b)
        np.save(os.path.join(tmp, "a.npy"), a)
        tar, ref["tarjan"] = run_child(tmp, "tarjan", 1)
        if tar is None:
            raise SystemExit(f"{name}: the reference's Tarjan did not finish: {ref['tarjan']}")
        for what in ("m2", "m1"):
            lab, ref[f"method{what[1:]}"] = run_child(tmp, what, threads)
            if lab is not None:
                eq = bool(np.array_equal(lab, tar))
                ref[f"method{what[1:]}"]["equals_tarjan"] = eq
                if not eq:
                    raise SystemExit(f"{name}: the reference's method {what[1:]} disagrees with its Tarjan on "
                                     f"{int(np.count_nonzero(lab != tar))} of {n} labels")
            if what == "m2" and lab is not None:
                break                          # method 1 only where method 2 cannot run
    out = {"params": kw, "n": int(n), "m": int(a.size), "csr_sha256": csr_digest(b, a), **label_summary(tar),
           "reference": ref}
    print(name, json.dumps(out), flush=True)
    return out


def main(names):
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for name in names or sorted(FULL):
        data[name] = record(name)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:])
