"""GPU: edge-batch updates (incremental / decremental) against a full oracle
recomputation of the updated graph: labels bit-exact after every batch, and the
merged CSR equal to gm_graph's CSR of the updated edge list."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State, condensation_graph
from tests.helpers import random_graph, seeded_graph

pytestmark = pytest.mark.gpu


def apply_batch(s, d, ins_s, ins_d, del_s, del_d):
    """Reference semantics: every copy of a deleted pair goes, inserted pairs are appended."""
    s = np.asarray(s, np.int64); d = np.asarray(d, np.int64)
    if len(del_s):
        dk = set((np.asarray(del_s, np.int64) << 32 | np.asarray(del_d, np.int64)).tolist())
        keep = np.array([(a << 32 | b) not in dk for a, b in zip(s.tolist(), d.tolist())], bool)
        s, d = s[keep], d[keep]
    s = np.concatenate([s, np.asarray(ins_s, np.int64)]); d = np.concatenate([d, np.asarray(ins_d, np.int64)])
    return s.astype(np.int32), d.astype(np.int32)


def check(g, st, n, s, d):
    csr = O.build_csr(n, s, d)
    b, a, rb, ra = g.csr()
    assert np.array_equal(b, csr[0]) and np.array_equal(a, csr[1])
    assert np.array_equal(rb, csr[2]) and np.array_equal(ra, csr[3])
    exp = O.tarjan_canonical(csr[0], csr[1])
    assert np.array_equal(st.canonical_labels(), exp)
    assert np.all(st.color() == -2)
    return exp


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_batches(gpu, seed):
    n = 2000
    s, d = random_graph(n, 3200, seed)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    check(g, st, n, s, d)
    rng = np.random.default_rng(100 + seed)
    for _ in range(6):
        k_ins, k_del = int(rng.integers(0, 80)), int(rng.integers(0, 60))
        ins_s = rng.integers(0, n, k_ins).astype(np.int32); ins_d = rng.integers(0, n, k_ins).astype(np.int32)
        pick = rng.integers(0, len(s), k_del)
        del_s = np.concatenate([s[pick], rng.integers(0, n, 5)]).astype(np.int32)   # plus pairs that may not exist
        del_d = np.concatenate([d[pick], rng.integers(0, n, 5)]).astype(np.int32)
        stats = st.update_batch(ins_s, ins_d, del_s, del_d)
        s, d = apply_batch(s, d, ins_s, ins_d, del_s, del_d)
        exp = check(g, st, n, s, d)
        assert stats["num_sccs"] == len(np.unique(exp)) and stats["m_after"] == len(s)


def test_insert_closes_cycle_and_delete_splits(gpu):
    n = 50
    s = np.arange(n - 1, dtype=np.int32); d = np.arange(1, n, dtype=np.int32)   # a path: 50 singletons
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    st.incremental_insert([n - 1], [0])                       # closes the cycle: one SCC
    assert np.all(st.canonical_labels() == 0)
    st.decremental_delete([20], [21])                         # breaks it: singletons again
    assert np.array_equal(st.canonical_labels(), np.arange(n, dtype=np.int32))
    st.update_batch([10], [0], [], [])                        # 0..10 merge
    lab = st.canonical_labels()
    assert np.all(lab[:11] == 0) and np.array_equal(lab[11:], np.arange(11, n, dtype=np.int32))


def test_empty_and_idempotent_batches(gpu):
    n = 300
    s, d = random_graph(n, 600, 9)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    before = st.canonical_labels()
    st.update_batch([], [], [], [])
    assert np.array_equal(st.canonical_labels(), before)
    # deleting a pair that is not an edge, then inserting and deleting the same self-loop
    present = set(zip(s.tolist(), d.tolist()))
    missing = next((u, v) for u in range(n) for v in range(n) if (u, v) not in present)
    st.decremental_delete([missing[0]], [missing[1]])
    assert np.array_equal(st.canonical_labels(), before)
    st.incremental_insert([5], [5])
    st.decremental_delete([5], [5])
    check(g, st, n, *apply_batch(s, d, [], [], [5], [5]))


def test_mixed_structure_batches(gpu):
    n, s, d, _ = seeded_graph(rmat_scale=13, edge_factor=6, grid_side=48, seed=12)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    rng = np.random.default_rng(7)
    for _ in range(3):
        ins_s = rng.integers(0, n, 1500).astype(np.int32); ins_d = rng.integers(0, n, 1500).astype(np.int32)
        pick = rng.integers(0, len(s), 700)
        del_s, del_d = s[pick], d[pick]
        st.update_batch(ins_s, ins_d, del_s, del_d)
        s, d = apply_batch(s, d, ins_s, ins_d, del_s, del_d)
        check(g, st, n, s, d)


def test_insert_idea1_recomputes(gpu):
    n = 1000
    s, d = random_graph(n, 1400, 21)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    rng = np.random.default_rng(1)
    ins_s = rng.integers(0, n, 200).astype(np.int32); ins_d = rng.integers(0, n, 200).astype(np.int32)
    st.insert_idea1(ins_s, ins_d)
    check(g, st, n, *apply_batch(s, d, ins_s, ins_d, [], []))


def test_condensation_graph_chunk_layout(gpu):
    # the cross-pair kernel works in 2,048-edge chunks: a hub spanning many
    # chunks, isolated runs wider than a chunk's vertex tile (in the middle
    # and at the end), and an edge count off every chunk boundary
    rng = np.random.default_rng(11)
    n = 60000
    parts = [(np.full(50001, 5), rng.integers(0, n, 50001)),
             (rng.integers(0, 20000, 30000), rng.integers(0, n, 30000)),
             (rng.integers(40000, 55000, 7777), rng.integers(0, n, 7777)),
             (np.arange(20000, 20003), np.arange(40000, 40003))]
    s = np.concatenate([p[0] for p in parts]).astype(np.int32)
    d = np.concatenate([p[1] for p in parts]).astype(np.int32)
    k = 3000
    ids = rng.integers(0, k, n).astype(np.int32)   # any grouping, not only SCCs
    ins_s = rng.integers(0, n, 64).astype(np.int32); ins_d = rng.integers(0, n, 64).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    for bs, bd in (((), ()), (ins_s, ins_d)):
        c = condensation_graph(g, ids, k, bs, bd)
        ms = np.concatenate([ids[s], ids[np.asarray(bs, np.int32)]])
        md = np.concatenate([ids[d], ids[np.asarray(bd, np.int32)]])
        keep = ms != md
        exp_s, exp_d = O.dedup_edges(ms[keep], md[keep], n=k)
        cb, ca, rb, ra = c.csr()
        assert np.array_equal(np.repeat(np.arange(k, dtype=np.int32), np.diff(cb)), exp_s)
        assert np.array_equal(ca, exp_d)
        order = np.lexsort((exp_s, exp_d))
        assert np.array_equal(np.repeat(np.arange(k, dtype=np.int32), np.diff(rb)), exp_d[order])
        assert np.array_equal(ra, exp_s[order])
        c.free()
    g.free()


def test_condensation_graph(gpu):
    n = 800
    s, d = random_graph(n, 1500, 5)
    csr = O.build_csr(n, s, d)
    lab = O.tarjan_canonical(csr[0], csr[1])
    ids = np.unique(lab, return_inverse=True)[1].astype(np.int32)
    k = int(ids.max()) + 1
    rng = np.random.default_rng(3)
    ins_s = rng.integers(0, n, 40).astype(np.int32); ins_d = rng.integers(0, n, 40).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    c = condensation_graph(g, ids, k, ins_s, ins_d)
    assert c.num_nodes() == k
    ms = np.concatenate([ids[s], ids[ins_s]]); md = np.concatenate([ids[d], ids[ins_d]])
    keep = ms != md
    exp_s, exp_d = O.dedup_edges(ms[keep], md[keep], n=k)
    cb, ca, _, _ = c.csr()
    got_s = np.repeat(np.arange(k, dtype=np.int32), np.diff(cb))
    assert np.array_equal(got_s, exp_s) and np.array_equal(ca, exp_d)
    # decomposing the condensation merges exactly what the inserted edges close
    st = State(c)
    st.run(2)
    merged = st.canonical_labels()[ids]
    exp = O.tarjan_canonical(*O.build_csr(n, *apply_batch(s, d, ins_s, ins_d, [], []))[:2])
    assert len(np.unique(merged)) == len(np.unique(exp))
