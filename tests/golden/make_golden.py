"""Regenerate tests/golden/golden.npz from the reference itself.

Runs the reference's own OpenMP method-2 pipeline and its do_tarjan_all
(compiled from its sources by oracle/Makefile into oracle/_ref/libscc_ref.so)
on seeded synthetic graphs and hand-made known-answer graphs, and stores the
canonical labels (component id = smallest member).  The reference ships no
golden vectors of its own; these pin the oracle and the engine to its
behaviour.  Needs the reference sources to have been built (make -C oracle).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from dynamicgraphs_scc_b200 import generate_edges_host  # noqa: E402

# seeded synthetic cases: (name, generator params)
GEN_CASES = [
    ("rmat16_ef8_seed42", dict(rmat_scale=16, edge_factor=8, seed=42)),          # the small plain config
    ("rmat12_grid64_seed3", dict(rmat_scale=12, edge_factor=8, grid_side=64, seed=3)),
    ("rmat14_cycles20_seed5", dict(rmat_scale=14, edge_factor=4, num_cycles=20, cycle_min=3, cycle_max=2000, seed=5)),
    ("grid128_seed11", dict(grid_side=128, seed=11)),
]


def kat_cases():
    """Hand-made known-answer graphs: (name, n, src, dst), kept with duplicates/self-loops as given."""
    c = []
    c.append(("cycle8", 8, list(range(8)), [(i + 1) % 8 for i in range(8)]))
    c.append(("dag_chain6", 6, [0, 1, 2, 3, 4], [1, 2, 3, 4, 5]))
    c.append(("two_cycles_2", 6, [0, 1, 2, 3, 4], [1, 0, 3, 2, 5]))
    c.append(("selfloops_dups", 5, [0, 0, 1, 1, 2, 2, 3, 4, 4], [0, 1, 0, 0, 2, 3, 4, 3, 4]))
    # bowtie: two 3-cycles sharing vertex 2, plus tails in and out
    c.append(("bowtie", 8, [0, 1, 2, 2, 3, 4, 5, 6], [1, 2, 0, 3, 4, 2, 2, 7]))
    c.append(("isolated_tail", 10, [0, 1, 2], [1, 2, 0]))
    c.append(("single_vertex", 1, [], []))
    c.append(("two_vertices_no_edge", 2, [], []))
    # nested: big cycle with chords and a hanging 2-cycle
    src = list(range(20)) + [0, 5, 10, 15, 20, 21]
    dst = [(i + 1) % 20 for i in range(20)] + [10, 15, 0, 5, 21, 20]
    c.append(("cycle_chords_pair", 22, src, dst))
    # ladder of 2-cycles connected one way (trim2 + DAG)
    s, d = [], []
    for k in range(10):
        a, b = 2 * k, 2 * k + 1
        s += [a, b]; d += [b, a]
        if k < 9:
            s.append(b); d.append(a + 2)
    c.append(("ladder_2cycles", 20, s, d))
    return c


def edge_digest(src, dst) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(src, np.int32).tobytes())
    h.update(np.ascontiguousarray(dst, np.int32).tobytes())
    return h.hexdigest()[:16]


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libscc_ref.so missing: run make -C oracle first")
    arrays = {}
    meta = []
    for name, kw in GEN_CASES:
        n, s, d = generate_edges_host(**kw)
        s, d = O.dedup_edges(s, d, n=n)
        csr = O.build_csr(n, s, d)
        m2, _ = O.ref_method2(csr)
        tj, _ = O.ref_tarjan(csr)
        arrays[f"{name}__m2"] = m2
        arrays[f"{name}__tarjan"] = tj
        meta.append(dict(name=name, kind="gen", params=kw, n=int(n), m=int(s.size), digest=edge_digest(s, d)))
    for name, n, s, d in kat_cases():
        s = np.asarray(s, np.int32); d = np.asarray(d, np.int32)
        csr = O.build_csr(n, s, d)
        m2, _ = O.ref_method2(csr)
        tj, _ = O.ref_tarjan(csr)
        arrays[f"{name}__src"] = s
        arrays[f"{name}__dst"] = d
        arrays[f"{name}__m2"] = m2
        arrays[f"{name}__tarjan"] = tj
        meta.append(dict(name=name, kind="kat", n=int(n), m=int(s.size)))
    arrays["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    print(f"wrote {len(meta)} cases")


if __name__ == "__main__":
    main()
