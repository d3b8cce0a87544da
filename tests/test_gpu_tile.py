"""GPU: the tile drain (one id range per SM, marks in shared memory) on the
shapes it is built for and on the ones that stress its protocol, compared with
the oracle's Tarjan.  The tunables force it on for small graphs: every round
with a live vertex may use it, and tiles may be as small as 16 ids, so waves
cross tiles constantly.  Cases: an oriented grid (many classes, deep waves), a
long cycle (one chain of single hops through every tile), a fully
bidirectional grid (one giant class of long diameter), R-MAT beside a grid
(hubs' neighbours spread over all tiles), thousands of 3-cycles beside a grid
(many classes per round), and a frontier that starts narrow and grows past
the drain's hand-back bound (the bail: every item goes back to the level
kernels)."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State
from tests.helpers import seeded_graph

pytestmark = pytest.mark.gpu

TILE_ON = dict(tile_min_live=1, tile_min_span=16)


def _check(n, s, d, methods=(0, 1, 2), **tuning):
    s = np.asarray(s, np.int32); d = np.asarray(d, np.int32)
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.set_tuning(**{**TILE_ON, **tuning})
    for method in methods:
        st.reset()
        r = st.run(method)
        got = st.canonical_labels()
        assert np.array_equal(got, exp), (method, int((got != exp).sum()))
        assert r["num_sccs"] == len(np.unique(exp)), method
    st.free(); g.free()


def test_tile_drain_oriented_grid(gpu):
    n, s, d, _ = seeded_graph(grid_side=512, seed=21)
    _check(n, s, d)


def test_tile_drain_long_cycle(gpu):
    n = 150000
    s = np.arange(n)
    _check(n, s, (s + 1) % n, methods=(2,))


def test_tile_drain_bidirectional_grid(gpu):
    k = 400
    idx = np.arange(k * k).reshape(k, k)
    h = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()])
    v = np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()])
    e = np.concatenate([h, v], axis=1)
    s = np.concatenate([e[0], e[1]]); d = np.concatenate([e[1], e[0]])
    _check(k * k, s, d, methods=(2,))


def test_tile_drain_rmat_beside_grid(gpu):
    n, s, d, _ = seeded_graph(rmat_scale=14, edge_factor=8, grid_side=256, seed=9)
    _check(n, s, d)


def test_tile_drain_large_tiles(gpu):
    # few tiles of many ids each: most hops stay inside a tile
    n, s, d, _ = seeded_graph(rmat_scale=12, edge_factor=8, grid_side=384, seed=4)
    _check(n, s, d, methods=(2,), tile_min_span=1 << 16)


def test_tile_drain_many_classes(gpu):
    n0, s, d, _ = seeded_graph(grid_side=256, seed=8)
    k = 20000
    base = n0 + 3 * np.arange(k, dtype=np.int32)
    s = np.concatenate([s, base, base + 1, base + 2]); d = np.concatenate([d, base + 1, base + 2, base])
    _check(n0 + 3 * k, s, d)


def test_tile_drain_hands_back_a_wide_frontier(gpu):
    # a random digraph of out-degree 3 (one giant class) whose best pivot has
    # 20 in- and 20 out-edges: the frontier starts at 40 items, so the drain
    # takes it after one level, then it grows past 65,536 outstanding items
    # and the drain hands every item back to the level kernels
    rng = np.random.default_rng(12)
    n = 300000
    s = np.repeat(np.arange(n), 3); d = rng.integers(0, n, 3 * n)
    hub = 7
    nb_out = rng.integers(0, n, 20); nb_in = rng.integers(0, n, 20)
    s = np.concatenate([s, np.full(20, hub), nb_in]); d = np.concatenate([d, nb_out, np.full(20, hub)])
    s, d = O.dedup_edges(s, d, n=n)
    _check(n, s, d, methods=(2,), async_max=64, async_after=1)


@pytest.mark.parametrize("tail", [dict(tail_live=-1), dict(tail_live=1 << 30, tail_class=16),
                                  dict(tail_live=1 << 30, tail_class=1 << 20)])
def test_recursion_tail_in_one_launch(gpu, tail):
    # the recursion's last rounds finished by one launch with a block per
    # class (on from the second round, off, or deferred until every class has
    # at most 16 vertices): the labels never change
    n, s, d, _ = seeded_graph(rmat_scale=13, edge_factor=6, grid_side=200, seed=12)
    _check(n, s, d, methods=(0, 1, 2), tile_min_live=-1, **tail)
