"""Shared test helpers: golden fixtures and seeded graphs."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from oracle import oracle as O
from dynamicgraphs_scc_b200 import generate_edges_host

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def edge_digest(src, dst) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(src, np.int32).tobytes())
    h.update(np.ascontiguousarray(dst, np.int32).tobytes())
    return h.hexdigest()[:16]


def golden_cases():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["__meta__"]).decode())
    out = []
    for c in meta:
        name = c["name"]
        if c["kind"] == "gen":
            n, s, d = generate_edges_host(**c["params"])
            s, d = O.dedup_edges(s, d, n=n)
        else:
            n, s, d = c["n"], z[f"{name}__src"], z[f"{name}__dst"]
        out.append(dict(name=name, n=n, src=np.asarray(s, np.int32), dst=np.asarray(d, np.int32),
                        m2=z[f"{name}__m2"], tarjan=z[f"{name}__tarjan"], meta=c))
    return out


def seeded_graph(**kw):
    """Deduplicated seeded edge list and its oracle CSR."""
    n, s, d = generate_edges_host(**kw)
    s, d = O.dedup_edges(s, d, n=n)
    return n, s, d, O.build_csr(n, s, d)


def random_graph(n, m, seed, self_loops=True, dups=True):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m).astype(np.int32)
    d = rng.integers(0, n, m).astype(np.int32)
    if not self_loops:
        keep = s != d
        s, d = s[keep], d[keep]
    if not dups:
        s, d = O.dedup_edges(s, d, drop_self_loops=False)
    return s, d
