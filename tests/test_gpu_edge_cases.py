"""GPU: structural edge cases, each compared with the oracle's Tarjan for the
three methods.  Each case exercises one path: the deepest peel cascades
(a long path), the asynchronous drain on a long chain of hops (a long cycle),
edge-parallel hub expansion (a bidirectional star above the hub threshold),
warp-cooperative lists (a clique), self-loops that must not keep a vertex
alive, many tiny classes (thousands of disjoint 3-cycles), and one giant SCC
of long diameter (a fully bidirectional grid)."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State

pytestmark = pytest.mark.gpu


def _check(n, s, d):
    s = np.asarray(s, np.int32); d = np.asarray(d, np.int32)
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, s, d)
    st = State(g)
    for method in (0, 1, 2):
        st.reset()
        r = st.run(method)
        assert np.array_equal(st.canonical_labels(), exp), method
        assert r["num_sccs"] == len(np.unique(exp)), method
    st.free(); g.free()


def test_weak_split_on_a_million_live_vertices(gpu):
    # after the global step more than 2^20 vertices stay live: an oriented
    # 1024 x 1024 grid (one giant weak component of many SCCs) beside 120,000
    # disjoint 3-cycles, all split by one union-find pass over the live list
    from tests.helpers import seeded_graph
    n0, s, d, _ = seeded_graph(rmat_scale=10, edge_factor=8, grid_side=1024, seed=5)
    k = 120000
    base = n0 + 3 * np.arange(k, dtype=np.int32)
    ts = np.concatenate([base, base + 1, base + 2]); td = np.concatenate([base + 1, base + 2, base])
    n = n0 + 3 * k
    s = np.concatenate([s, ts]).astype(np.int32); d = np.concatenate([d, td]).astype(np.int32)
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, s, d)
    st = State(g)
    r = st.run(2)
    assert n - r["trimmed_first"] - r["first_scc_size"] - r["trimmed_second"] >= 1 << 20   # live at the split
    assert r["num_wcc_classes"] > k
    assert np.array_equal(st.canonical_labels(), exp)
    st.free(); g.free()


def test_long_path_all_trimmed(gpu):
    n = 300000
    s = np.arange(n - 1); _check(n, s, s + 1)


def test_long_cycle(gpu):
    n = 200000
    s = np.arange(n); _check(n, s, (s + 1) % n)


def test_bidirectional_star_with_huge_hub(gpu):
    leaves = 20000                                   # hub degree far above the 4,096 hub threshold
    l = np.arange(1, leaves + 1)
    _check(leaves + 1, np.concatenate([np.zeros(leaves, int), l]), np.concatenate([l, np.zeros(leaves, int)]))


def test_clique(gpu):
    k = 300
    a, b = np.meshgrid(np.arange(k), np.arange(k), indexing="ij")
    keep = a != b
    _check(k, a[keep], b[keep])


def test_self_loops_only(gpu):
    n = 10000
    s = np.arange(n); _check(n, s, s)


def test_many_disjoint_triangles(gpu):
    t = 5000
    base = np.arange(t) * 3
    s = np.concatenate([base, base + 1, base + 2]); d = np.concatenate([base + 1, base + 2, base])
    _check(3 * t, s, d)


def test_fully_bidirectional_grid(gpu):
    side = 300
    idx = np.arange(side * side).reshape(side, side)
    h = (idx[:, :-1].ravel(), idx[:, 1:].ravel()); v = (idx[:-1, :].ravel(), idx[1:, :].ravel())
    s = np.concatenate([h[0], h[1], v[0], v[1]]); d = np.concatenate([h[1], h[0], v[1], v[0]])
    _check(side * side, s, d)


def test_single_vertex_cases(gpu):
    _check(1, [0], [0])                              # one vertex with a self-loop
    _check(2, [0, 1], [1, 0])                        # a 2-cycle
    _check(3, [0, 0, 0], [1, 1, 1])                  # duplicates only


def test_very_long_cycle_completes(gpu):
    # one SCC crossed by a single chain of 2,000,000 hops: the asynchronous
    # drain runs for seconds with one item outstanding, and idle warps must
    # keep waiting (their bound counts stalls, not traversal length)
    n = 2000000
    s = np.arange(n, dtype=np.int32)
    g = Graph.from_edges(n, s, ((s + 1) % n).astype(np.int32))
    st = State(g)
    r = st.run(2)
    assert r["num_sccs"] == 1 and r["first_scc_size"] == n
    assert not st.canonical_labels().any()
    st.free(); g.free()


def test_several_long_chains_at_once(gpu):
    # four disjoint cycles of 0.6-1.2 M vertices: the global step walks one
    # (its FW and BW chains in two warps), then one round walks the other
    # three at once, six single-hop chains of different lengths in different
    # warps while idle warps run out their wait bound; every chain must still
    # reach its end, and the chains that end first must not end the drain
    lens = [1200000, 1000000, 800000, 600000]
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
    s = np.concatenate([st + np.arange(L) for st, L in zip(starts, lens)]).astype(np.int32)
    d = np.concatenate([st + (np.arange(L) + 1) % L for st, L in zip(starts, lens)]).astype(np.int32)
    n = int(sum(lens))
    g = Graph.from_edges(n, s, d)
    st = State(g)
    r = st.run(2)
    assert r["num_sccs"] == 4
    exp = np.repeat(starts, lens).astype(np.int32)
    assert np.array_equal(st.canonical_labels(), exp)
    st.free(); g.free()


def _hub_graph():
    rng = np.random.default_rng(51)
    leaves = 200000
    base = 10000
    s_r, d_r = rng.integers(0, base, 30000), rng.integers(0, base, 30000)
    h1 = base
    l1 = np.arange(base + 1, base + 1 + leaves)
    src = base + 1 + leaves
    h2 = src + 1
    l2 = np.arange(h2 + 1, h2 + 1 + leaves)
    h3 = h2 + 1 + leaves
    n = h3 + 1
    s = np.concatenate([s_r, np.full(leaves, h1), [src], np.full(leaves, h2), l2, rng.integers(0, base, 50)])
    d = np.concatenate([d_r, l1, [h2], l2, np.full(leaves, h3), np.full(50, h1)])
    return n, s, d


def test_scanning_peel_hubs_edge_parallel(gpu):
    # the same hubs through the peel of a state that is not fresh (colours
    # given explicitly), whose overflowed vertices are re-checked over the grid
    n, s, d = _hub_graph()
    csr = O.build_csr(n, np.asarray(s, np.int32), np.asarray(d, np.int32))
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, np.asarray(s, np.int32), np.asarray(d, np.int32))
    st = State(g)
    for method in (0, 2):
        st.reset()
        st.set_color(np.full(n, -1, np.int32))
        st.run(method)
        assert np.array_equal(st.canonical_labels(), exp), method
    st.free(); g.free()


def test_peel_hubs_expanded_edge_parallel(gpu):
    # a source hub with 200,000 out-edges (trimmed as a seed), a hub reached
    # from a source by one edge (trimmed by a cascade), a sink hub with
    # 200,000 in-edges, and a random graph with real SCCs beside them: hubs
    # above 4,096 edges are expanded over the whole grid, not by one warp
    rng = np.random.default_rng(51)
    leaves = 200000
    base = 10000
    s_r, d_r = rng.integers(0, base, 30000), rng.integers(0, base, 30000)
    h1 = base
    l1 = np.arange(base + 1, base + 1 + leaves)
    src = base + 1 + leaves
    h2 = src + 1
    l2 = np.arange(h2 + 1, h2 + 1 + leaves)
    h3 = h2 + 1 + leaves
    n = h3 + 1
    s = np.concatenate([s_r, np.full(leaves, h1), [src], np.full(leaves, h2), l2, rng.integers(0, base, 50)])
    d = np.concatenate([d_r, l1, [h2], l2, np.full(leaves, h3), np.full(50, h1)])
    _check(n, s, d)
