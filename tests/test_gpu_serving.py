"""GPU: the serving loop.  Each session's results must be the same when its
requests run alone and when they run mixed with other sessions' requests on
several slots (continuous batching), and equal to the oracle; admission
rejects what can never fit the HBM budget."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, Server
from tests.test_gpu_update import apply_batch
from tests.helpers import random_graph, seeded_graph

pytestmark = pytest.mark.gpu


def sessions_and_batches():
    graphs = []
    for seed in (1, 2):
        n, s, d, _ = seeded_graph(rmat_scale=12, edge_factor=6, seed=seed)
        graphs.append((n, s, d))
    n, s, d, _ = seeded_graph(grid_side=48, seed=3)
    graphs.append((n, s, d))
    s4, d4 = random_graph(2500, 4000, 4)
    graphs.append((2500, s4, d4))
    batches = []
    rng = np.random.default_rng(11)
    for n, s, d in graphs:
        bl = []
        for _ in range(5):
            ki, kd = int(rng.integers(10, 400)), int(rng.integers(10, 200))
            pick = rng.integers(0, len(s), kd)
            bl.append((rng.integers(0, n, ki).astype(np.int32), rng.integers(0, n, ki).astype(np.int32),
                       s[pick].astype(np.int32), d[pick].astype(np.int32)))
        batches.append(bl)
    return graphs, batches


def run_server(graphs, batches, slots, mixed):
    sv = Server(num_slots=slots, hbm_budget_bytes=8 << 30)
    sids = [sv.add_graph(Graph.from_edges(n, s, d)) for n, s, d in graphs]
    counts = {}
    if mixed:
        rids = []
        for j in range(len(batches[0])):
            for k, sid in enumerate(sids):
                rids.append((k, j, sv.submit(sid, *batches[k][j])))
        for k, j, rid in rids:
            r = sv.wait(rid)
            assert r["status"] == 0
            counts[(k, j)] = r["num_sccs"]
    else:
        for k, sid in enumerate(sids):
            for j, b in enumerate(batches[k]):
                r = sv.wait(sv.submit(sid, *b))
                assert r["status"] == 0
                counts[(k, j)] = r["num_sccs"]
    sv.drain()
    labels = [sv.labels(sid) for sid in sids]
    stats = sv.stats()
    sv.free()
    return counts, labels, stats


def test_alone_equals_mixed_equals_oracle(gpu):
    graphs, batches = sessions_and_batches()
    c_alone, l_alone, st_alone = run_server(graphs, batches, slots=1, mixed=False)
    c_mix, l_mix, st_mix = run_server(graphs, batches, slots=4, mixed=True)
    assert c_alone == c_mix
    for a, b in zip(l_alone, l_mix):
        assert np.array_equal(a, b)
    for (n, s, d), bl, lab in zip(graphs, batches, l_mix):
        for b in bl:
            s, d = apply_batch(s, d, *b)
        csr = O.build_csr(n, s, d)
        assert np.array_equal(lab, O.tarjan_canonical(csr[0], csr[1]))
    assert st_mix["completed"] == sum(len(b) for b in batches) and st_mix["rejected"] == 0
    assert st_mix["max_inflight"] >= 2            # requests of different sessions overlapped
    assert 0 < st_mix["p50_ms"] <= st_mix["p99_ms"]


def test_admission_by_hbm_budget(gpu):
    n, s, d, _ = seeded_graph(rmat_scale=10, edge_factor=4, seed=5)
    sv = Server(num_slots=2, hbm_budget_bytes=8 << 20)     # 8 MiB
    sid = sv.add_graph(Graph.from_edges(n, s, d))
    rng = np.random.default_rng(0)
    small = sv.wait(sv.submit(sid, rng.integers(0, n, 50), rng.integers(0, n, 50)))
    assert small["status"] == 0
    big = sv.wait(sv.submit(sid, rng.integers(0, n, 200000), rng.integers(0, n, 200000)))
    assert big["status"] == 3                               # SCC_ERR_OOM: never fits
    st = sv.stats()
    assert st["rejected"] == 1 and st["completed"] == 2
    with pytest.raises(Exception):
        sv.add_graph(Graph.generate(rmat_scale=16, edge_factor=8, seed=1))   # larger than the budget left
    sv.free()


def test_coalesced_requests_equal_sequential(gpu):
    """With coalescing on, a session's queued batches are applied as one composed
    batch; the final labels equal the sequential run's and Tarjan's, and the last
    request of each session reports the same SCC count.  The batches insert and
    later delete the same pairs, so the composition rule is exercised."""
    n, s, d, _ = seeded_graph(rmat_scale=11, edge_factor=6, seed=9)
    rng = np.random.default_rng(5)
    batches = []
    prev = None
    for j in range(12):
        ki, kd = int(rng.integers(20, 300)), int(rng.integers(10, 150))
        pick = rng.integers(0, len(s), kd)
        ins = (rng.integers(0, n, ki).astype(np.int32), rng.integers(0, n, ki).astype(np.int32))
        dels = [s[pick].astype(np.int32), d[pick].astype(np.int32)]
        if prev is not None:           # delete some pairs the previous batch inserted
            dels[0] = np.concatenate([dels[0], prev[0][:10]]); dels[1] = np.concatenate([dels[1], prev[1][:10]])
        batches.append((ins[0], ins[1], dels[0], dels[1]))
        prev = ins

    def serve(coalesce):
        sv = Server(num_slots=2, hbm_budget_bytes=8 << 30)
        if coalesce:
            sv.set_coalesce(8)
        sid = sv.add_graph(Graph.from_edges(n, s, d))
        # hold the session busy with a first request so the rest queue up together
        rids = [sv.submit(sid, *b) for b in batches]
        res = [sv.wait(r) for r in rids]
        sv.drain()
        lab = sv.labels(sid)
        st = sv.stats()
        sv.free()
        return res, lab, st

    r_seq, l_seq, st_seq = serve(False)
    r_co, l_co, st_co = serve(True)
    assert all(r["status"] == 0 for r in r_seq + r_co)
    assert np.array_equal(l_seq, l_co)
    assert r_seq[-1]["num_sccs"] == r_co[-1]["num_sccs"]
    assert st_seq["groups"] == len(batches)
    assert st_co["groups"] < len(batches)          # some requests were composed
    assert st_co["completed"] == len(batches)
    ss, dd = s, d
    for b in batches:
        ss, dd = apply_batch(ss, dd, *b)
    csr = O.build_csr(n, ss, dd)
    assert np.array_equal(l_co, O.tarjan_canonical(csr[0], csr[1]))


def test_backpressure_sheds_and_expires(gpu):
    """Admission by backlog and age: with one slot and a backlog limit of three
    batches, a burst of twenty batches is partly refused at submit (request id
    -1); with a short age limit, queued requests may also be dropped when a
    slot reaches them (status SCC_ERR_BUSY).  Whatever was refused or dropped
    changed nothing: the labels equal Tarjan of the graph with only the
    applied batches, in order, and the counts add up."""
    n, s, d, _ = seeded_graph(rmat_scale=12, edge_factor=6, seed=21)
    rng = np.random.default_rng(8)
    batches = []
    for _ in range(20):
        pick = rng.integers(0, len(s), 300)
        batches.append((rng.integers(0, n, 700).astype(np.int32), rng.integers(0, n, 700).astype(np.int32),
                        s[pick].astype(np.int32), d[pick].astype(np.int32)))
    sv = Server(num_slots=1, hbm_budget_bytes=8 << 30)
    sid = sv.add_graph(Graph.from_edges(n, s, d))
    sv.set_admission(max_queued_edges=3000, max_queue_ms=2.0)
    rids = [sv.submit(sid, *b) for b in batches]
    res = [sv.wait(r) if r >= 0 else None for r in rids]
    sv.drain()
    lab = sv.labels(sid)
    st = sv.stats()
    sv.free()
    shed = sum(r is None for r in res)
    applied = [b for b, r in zip(batches, res) if r is not None and r["status"] == 0]
    expired = sum(r is not None and r["status"] == 9 for r in res)
    assert shed >= 1 and st["shed"] == shed and st["expired"] == expired
    assert st["offered_edges"] == 20 * 1000 and st["shed_edges"] == 1000 * shed
    assert st["completed"] == 20 - shed
    assert len(applied) >= 1 and st["max_queued_edges"] <= 3000
    ss, dd = s, d
    for b in applied:
        ss, dd = apply_batch(ss, dd, *b)
    csr = O.build_csr(n, ss, dd)
    assert np.array_equal(lab, O.tarjan_canonical(csr[0], csr[1]))
