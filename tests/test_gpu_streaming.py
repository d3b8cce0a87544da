"""GPU: the adjacency streaming paths of the level kernels, compared with the
oracle's Tarjan.

* Block-wide expansion: top-down items of degree in (cta_deg, huge_deg] are
  expanded by a whole block, their adjacency lists copied into shared memory
  by 1-D bulk copies, chunk by chunk, two buffers deep.  The cases force it on
  (low cta_deg, bottom-up off so every level is top-down) for mid-degree hubs,
  a list of several chunks that starts off a 16-byte boundary, and lists of
  every length modulo 4 (the unstaged tail).  A level of fewer blocks than
  SMs sends the same items edge-parallel over the whole GPU instead, so the
  small cases cover that route and a wide level covers the block bucket.
* Bottom-up probes: both directions at once, an aligned int4 chunk of each
  list per probe; rounds over one class and over many classes, lists that
  start at every offset modulo 4, and a list that ends at the last entry of
  the adjacency array (the per-entry fallback near the end).
"""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State
from tests.helpers import seeded_graph

pytestmark = pytest.mark.gpu

TOP_DOWN = dict(bu_alpha=1)          # bottom-up never pays: every level is top-down


def _check(n, s, d, methods=(0, 1, 2), **tuning):
    s = np.asarray(s, np.int32); d = np.asarray(d, np.int32)
    s, d = O.dedup_edges(s, d, n=n)
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.set_tuning(**tuning)
    for method in methods:
        st.reset()
        r = st.run(method)
        got = st.canonical_labels()
        assert np.array_equal(got, exp), (method, tuning, int((got != exp).sum()))
        assert r["num_sccs"] == len(np.unique(exp)), method
    st.free(); g.free()


def _mid_hubs(seed, n=40000, hubs=300):
    # a sparse random digraph (out-degree 2) plus hubs of out- and in-degree
    # 40..4000, so top-down levels hold many items between one warp's and the
    # edge-parallel path's degrees
    rng = np.random.default_rng(seed)
    s = [np.repeat(np.arange(n), 2)]
    d = [rng.integers(0, n, 2 * n)]
    for h in rng.choice(n, hubs, replace=False):
        k_out, k_in = rng.integers(40, 4000, 2)
        s += [np.full(k_out, h), rng.integers(0, n, k_in)]
        d += [rng.integers(0, n, k_out), np.full(k_in, h)]
    return n, np.concatenate(s), np.concatenate(d)


@pytest.mark.parametrize("cta_deg", [33, 256, 1024, -1])
def test_block_expansion_mid_degree_hubs(gpu, cta_deg):
    n, s, d = _mid_hubs(5)
    _check(n, s, d, cta_deg=cta_deg, **TOP_DOWN)


def test_block_expansion_wide_level(gpu):
    # levels of more than 148 blocks' worth of items (37,888): the block
    # bucket proper, beside the edge-parallel route of the first levels
    n, s, d = _mid_hubs(7, n=300000, hubs=2000)
    _check(n, s, d, methods=(2,), cta_deg=256, **TOP_DOWN)


def test_block_expansion_default_traversal(gpu):
    # the same hubs under the default direction choice
    n, s, d = _mid_hubs(6)
    _check(n, s, d, cta_deg=64)


@pytest.mark.parametrize("lead", [0, 1, 2, 3, 5])
def test_block_expansion_multi_chunk_unaligned(gpu, lead):
    # a star of 5,000 leaves (one class, hub <-> leaf) whose lists span five
    # 1,024-entry chunks; `lead` edges before the hub's lists move their start
    # off the 16-byte boundary, and the leaf count leaves an unstaged tail
    n = 5003 + 8
    hub = 7
    leaves = np.arange(8, n)
    s = [np.arange(lead) % 7, np.full(leaves.size, hub), leaves]
    d = [(np.arange(lead) + 1) % 7, leaves, np.full(leaves.size, hub)]
    _check(n, np.concatenate(s), np.concatenate(d), cta_deg=64, huge_deg=8192, **TOP_DOWN)


def test_block_expansion_every_tail_length(gpu):
    # hubs whose degrees cover every residue mod 4 and mod the chunk size
    rng = np.random.default_rng(17)
    n = 12000
    s = [np.arange(n - 1), np.arange(1, n)]          # a bidirectional path: one class
    d = [np.arange(1, n), np.arange(n - 1)]
    for i, k in enumerate([65, 66, 67, 68, 1023, 1024, 1025, 1026, 2047, 2049, 3071]):
        h = 100 + 37 * i
        s += [np.full(k, h), rng.integers(0, n, k)]
        d += [rng.integers(0, n, k), np.full(k, h)]
    _check(n, np.concatenate(s), np.concatenate(d), cta_deg=64, **TOP_DOWN)


def test_bottom_up_probes_rmat_and_grid(gpu):
    # R-MAT (bottom-up sweeps from the hub pivot) beside a grid (many classes
    # in later rounds: the probes then check the parent's colour too)
    n, s, d, _ = seeded_graph(rmat_scale=15, edge_factor=16, grid_side=200, seed=31)
    _check(n, s, d, bu_alpha=40, bu_div=48)


def test_bottom_up_probes_list_at_array_end(gpu):
    # the last vertex's lists end at the last entries of both adjacency
    # arrays, where a probe's aligned chunk reaches past the end and the
    # probe falls back to one load per entry
    n = 3001
    rng = np.random.default_rng(4)
    ring = np.arange(n)
    s = [ring, np.full(999, n - 1), rng.integers(0, n - 1, 998)]
    d = [(ring + 1) % n, rng.integers(0, n - 1, 999), np.full(998, n - 1)]
    _check(n, np.concatenate(s), np.concatenate(d), bu_alpha=40, bu_div=48)
