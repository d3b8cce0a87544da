"""GPU: batched uneven graphs (many independent graphs decomposed together),
the batch generator (device == host), subgraph extraction, the autotuner."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State, generate_batch_edges_host

pytestmark = pytest.mark.gpu

KW = dict(num_graphs=24, n_min=64, n_max=3000, mean_degree=3.0, rmat_fraction=0.3, seed=77)


def host_batch():
    n, offs, s, d = generate_batch_edges_host(**KW)
    s, d = O.dedup_edges(s, d, n=n)
    return n, offs, s, d


def test_batch_generator_device_matches_host(gpu):
    n, offs, s, d = host_batch()
    g, goffs = Graph.generate_batch(**KW)
    assert np.array_equal(goffs, offs) and g.num_nodes() == n and g.num_edges() == s.size
    for x, y in zip(g.csr(), O.build_csr(n, s, d)):
        assert np.array_equal(x, y)
    # no edge leaves its graph
    assert np.all(np.searchsorted(offs, s, side="right") == np.searchsorted(offs, d, side="right"))


def test_batched_labels_equal_per_graph_labels(gpu):
    n, offs, s, d = host_batch()
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g, _ = Graph.generate_batch(**KW)
    st = State(g)
    st.run(2)
    union = st.canonical_labels()
    assert np.array_equal(union, exp)
    for i in range(0, len(offs) - 1, 5):
        sub = g.subgraph(int(offs[i]), int(offs[i + 1]))
        ss = State(sub)
        ss.run(2)
        assert np.array_equal(ss.canonical_labels() + offs[i], union[offs[i]:offs[i + 1]])


def test_subgraph_rejects_open_range(gpu):
    g = Graph.from_edges(4, [0, 1, 2], [1, 2, 3])
    with pytest.raises(Exception):
        g.subgraph(0, 2)


def test_autotune_keeps_labels(gpu):
    n, s, d = 3000, *np.random.default_rng(5).integers(0, 3000, (2, 5000)).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    best, ms = st.autotune(max_trials=6)
    assert ms > 0 and st.get_tuning() == best
    st.run(2)
    csr = O.build_csr(n, s, d)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))


def test_persistent_batch_plan_equals_tarjan_twice(gpu):
    """The one-launch batched run (each block decomposes whole graphs; the run
    replayed from a captured CUDA graph) gives Tarjan's labels, twice in a row
    on the same plan, with one host submission and one kernel per run."""
    from dynamicgraphs_scc_b200 import BatchPlan
    n, offs, s, d = host_batch()
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g, goffs = Graph.generate_batch(**KW)
    st = State(g)
    plan = BatchPlan(g, st, goffs)
    for _ in range(2):
        r = plan.run()
        assert r["host_submissions"] == 1 and r["kernels"] == 1 and r["graphs"] == len(goffs) - 1
        assert np.array_equal(st.canonical_labels(), exp)
    plan.free()


@pytest.mark.parametrize("tuning", [dict(threads=256, blocks_per_sm=1, warp_deg=8),
                                    dict(threads=1024, blocks_per_sm=2, warp_deg=64)])
def test_batch_plan_tunings_and_structures(gpu, tuning):
    """Launch shapes and warp cut-offs change speed only: graphs of long
    cycles, long paths, a bidirectional star (one list far above the warp
    cut-off) and 3-cycles, batched with random graphs, all equal Tarjan."""
    from dynamicgraphs_scc_b200 import BatchPlan
    parts, src, dst, offs = [], [], [], [0]
    rng = np.random.default_rng(4)
    specs = [("cycle", 5000), ("path", 4000), ("star", 3000), ("tri", 900), ("rand", 2000), ("rand", 64)]
    for kind, k in specs:
        base = offs[-1]
        if kind == "cycle":
            a = np.arange(k); b = (a + 1) % k
        elif kind == "path":
            a = np.arange(k - 1); b = a + 1
        elif kind == "star":
            leaves = np.arange(1, k)
            a = np.concatenate([np.zeros(k - 1, int), leaves]); b = np.concatenate([leaves, np.zeros(k - 1, int)])
        elif kind == "tri":
            t = 3 * np.arange(k // 3)
            a = np.concatenate([t, t + 1, t + 2]); b = np.concatenate([t + 1, t + 2, t])
        else:
            a, b = rng.integers(0, k, (2, 3 * k))
        src.append(a + base); dst.append(b + base)
        offs.append(base + k)
    n = offs[-1]
    s = np.concatenate(src).astype(np.int32); d = np.concatenate(dst).astype(np.int32)
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, s, d)
    st = State(g)
    plan = BatchPlan(g, st, np.asarray(offs, np.int32), tuning=tuning)
    plan.run()
    assert np.array_equal(st.canonical_labels(), exp)
    plan.free()


def test_batch_autotune_successive_halving(gpu):
    from dynamicgraphs_scc_b200 import BatchPlan, batch_autotune
    n, offs, s, d = host_batch()
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g, goffs = Graph.generate_batch(**KW)
    st = State(g)
    best, ms = batch_autotune(g, st, goffs)
    assert ms > 0 and best["threads"] in (256, 512, 1024)
    plan = BatchPlan(g, st, goffs, tuning=best)
    plan.run()
    assert np.array_equal(st.canonical_labels(), exp)
    plan.free()
