"""GPU parity: the CUDA path, called through the C ABI, against the oracle and
the reference's own outputs (golden fixtures).  Integer work: bit-exact."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State, capi, decompose_csr
from tests.helpers import golden_cases, random_graph, seeded_graph

pytestmark = pytest.mark.gpu

KEEP = capi.SCC_BUILD_KEEP_ALL
CLEAN = capi.SCC_BUILD_DEDUP | capi.SCC_BUILD_NO_SELF_LOOPS


@pytest.fixture(scope="module")
def cases():
    return golden_cases()


def run_labels(n, s, d, method=2, flags=KEEP):
    g = Graph.from_edges(n, s, d, flags=flags)
    st = State(g)
    stats = st.run(method)
    lab = st.canonical_labels()
    cnt = st.count_sccs()
    return lab, cnt, stats


@pytest.mark.parametrize("method", [0, 1, 2])
def test_golden_labels_all_methods(gpu, cases, method):
    for c in cases:
        lab, cnt, _ = run_labels(c["n"], c["src"], c["dst"], method)
        assert np.array_equal(lab, c["tarjan"]), (c["name"], method)
        assert np.array_equal(lab, c["m2"]), (c["name"], method)
        assert cnt == len(np.unique(c["tarjan"])), c["name"]


def test_device_csr_build_matches_gm_graph(gpu):
    s, d = random_graph(500, 3000, 3)
    g = Graph.from_edges(500, s, d, flags=KEEP)
    b, a, rb, ra = g.csr()
    ob, oa, orb, ora = O.build_csr(500, s, d)
    assert np.array_equal(b, ob) and np.array_equal(a, oa)
    assert np.array_equal(rb, orb) and np.array_equal(ra, ora)


def test_csr_upload_builds_transpose(gpu):
    s, d = random_graph(300, 2000, 5)
    ob, oa, orb, ora = O.build_csr(300, s, d)
    g = Graph.from_csr(ob, oa)
    b, a, rb, ra = g.csr()
    assert np.array_equal(rb, orb) and np.array_equal(ra, ora)


@pytest.mark.parametrize("kw", [
    dict(rmat_scale=12, edge_factor=8, seed=7),
    dict(rmat_scale=10, edge_factor=4, grid_side=48, seed=2),
    dict(rmat_scale=12, edge_factor=4, num_cycles=15, cycle_min=3, cycle_max=900, seed=8),
])
def test_device_generator_matches_host(gpu, kw):
    n, s, d, csr = seeded_graph(**kw)
    g = Graph.generate(**kw)
    assert g.num_nodes() == n and g.num_edges() == s.size
    for x, y in zip(g.csr(), csr):
        assert np.array_equal(x, y)


def test_trim1_fixpoint_exact(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=14, edge_factor=6, grid_side=64, seed=31)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    t = st.repeat_global_trim1(100)
    color = np.full(n, -1, np.int32); scc = np.full(n, -1, np.int32)
    ot = O.trim1_fixpoint(csr, color, scc)
    assert t == ot
    assert np.array_equal(st.color(), color)
    assert np.array_equal(st.scc(), scc)


def test_trim1_respects_colours(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=12, edge_factor=8, seed=13)
    rng = np.random.default_rng(0)
    color = rng.integers(-1, 3, n).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.set_color(color)
    t = st.do_global_trim1()
    oc = color.copy(); os_ = np.full(n, -1, np.int32)
    ot = O.trim1_fixpoint(csr, oc, os_)
    assert t == ot and np.array_equal(st.color(), oc)


@pytest.mark.parametrize("seed", [3, 4])
def test_trim1_on_live_list_within_colours(gpu, seed):
    # a long live list (>= 32,768 vertices) is peeled by counting neighbours
    # inside colours once and expanding trims from warp queues: the same
    # fixpoint as the oracle's scanning peel, with finished vertices, several
    # colours, duplicate and self-loop edges, and a 10,000-edge hub that is a
    # seed (no in-edges) and is expanded edge-parallel
    n0, s, d, _ = seeded_graph(rmat_scale=16, edge_factor=4, grid_side=256, seed=seed)
    rng = np.random.default_rng(seed)
    hub = n0
    n = n0 + 1
    s = np.concatenate([s, np.full(10000, hub, np.int32), rng.integers(0, n0, 3000).astype(np.int32)])
    d = np.concatenate([d, rng.integers(0, n0, 10000).astype(np.int32), rng.integers(0, n0, 3000).astype(np.int32)])
    s = np.concatenate([s, s[:500]]); d = np.concatenate([d, d[:500]])          # duplicates
    s = np.concatenate([s, np.arange(0, 200, dtype=np.int32)]); d = np.concatenate([d, np.arange(0, 200, dtype=np.int32)])
    csr = O.build_csr(n, s, d)
    color = rng.integers(-2, 3, n).astype(np.int32)
    color[hub] = 0
    scc = np.where(color == -2, np.arange(n, dtype=np.int32), -1).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.set_color(color); st.set_scc(scc)
    assert st.create_trim1_compact() >= 32768
    t = st.repeat_global_trim1_compact()
    oc = color.copy(); os_ = scc.copy()
    ot = O.trim1_fixpoint(csr, oc, os_)
    assert t == ot and t > 0
    assert np.array_equal(st.color(), oc)
    assert np.array_equal(st.scc(), os_)


def test_global_fw_bw_exact(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=14, edge_factor=8, seed=17)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.repeat_global_trim1()
    st.create_trim1_compact()
    color = st.color(); scc = st.scc()
    p = O.choose_pivot(csr, color, -1)
    assert st.choose_pivot_from_color(-1) == p
    size = st.do_fw_bw_global_main(-1, 0, True)
    osize, ofw, obw = O.fw_bw(csr, color, scc, -1, p, 0, 1)
    assert size == osize
    assert np.array_equal(st.color(), color)
    assert np.array_equal(st.scc(), scc)
    cols, cnts = st.work_q_items()
    expect = [(c, k) for c, k in ((0, ofw), (1, obw), (-1, int((color == -1).sum()))) if k > 0]
    assert list(zip(cols.tolist(), cnts.tolist())) == expect


def test_trim2_exact(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=12, edge_factor=3, grid_side=64, seed=23)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.repeat_global_trim1()
    st.create_trim1_compact()
    color = st.color(); scc = st.scc()
    t = st.do_global_trim2_new()
    ot = O.trim2(csr, color, scc)
    assert t == ot and t > 0
    assert np.array_equal(st.color(), color)
    assert np.array_equal(st.scc(), scc)


def test_wcc_minreach_exact(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=13, edge_factor=6, grid_side=40, seed=29)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.repeat_global_trim1()
    st.create_trim1_compact()
    st.do_fw_bw_global_main(-1)
    st.repeat_global_trim1_compact()
    color = st.color()
    st.do_global_wcc()
    w = st.wcc()
    ow = O.wcc_minreach(csr, color)
    live = color != -2
    assert np.array_equal(w[live], ow[live])
    # colouring: same root <=> same colour
    newc = st.color()
    roots = ow[live] & 0x1FFFFFFF
    _, inv_r = np.unique(roots, return_inverse=True)
    _, inv_c = np.unique(newc[live], return_inverse=True)
    assert np.array_equal(inv_r, inv_c)
    k = st.create_work_items_from_wcc()
    assert k == len(np.unique(roots))
    st.start_workers_fw_bw_dfs(40)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))


@pytest.mark.parametrize("seed", range(6))
def test_random_graphs_with_loops_and_duplicates(gpu, seed):
    n = [1, 2, 17, 300, 2000, 5000][seed]
    s, d = random_graph(n, int(n * 1.6) + 1, seed)
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    for method in (0, 1, 2):
        lab, _, _ = run_labels(n, s, d, method)
        assert np.array_equal(lab, exp), method


def test_no_edges(gpu):
    lab, cnt, st = run_labels(5, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert lab.tolist() == [0, 1, 2, 3, 4] and cnt == 5


def test_mixed_structure_medium(gpu):
    """C2-shaped union (R-MAT + oriented grid) at a size the oracle finishes quickly."""
    kw = dict(rmat_scale=17, edge_factor=16, grid_side=256, seed=99)
    n, s, d, csr = seeded_graph(**kw)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.generate(**kw)
    st = State(g)
    stats = st.run(2)
    assert np.array_equal(st.canonical_labels(), exp)
    assert stats["num_sccs"] == len(np.unique(exp))


def test_planted_cycles_medium(gpu):
    kw = dict(rmat_scale=16, edge_factor=8, num_cycles=50, cycle_min=3, cycle_max=5000, seed=77)
    n, s, d, csr = seeded_graph(**kw)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.generate(**kw)
    st = State(g)
    st.run(2)
    assert np.array_equal(st.canonical_labels(), exp)


def test_output_scc_list_format(gpu, tmp_path, cases):
    c = [x for x in cases if x["name"] == "bowtie"][0]
    g = Graph.from_edges(c["n"], c["src"], c["dst"])
    st = State(g)
    st.run(2)
    p = tmp_path / "scc_list.txt"
    st.output_scc_list(str(p))
    lines = p.read_text().split("\n")[:-1]
    # reference numbering: ids by first appearance over i (scc_post_analyze.cc:31-53)
    first = {}
    exp = []
    for i, r in enumerate(c["tarjan"].tolist()):
        first.setdefault(r, len(first))
        exp.append(f"{i} {first[r]}")
    assert lines == exp


def test_edge_list_loader_semantics(gpu, tmp_path):
    # 1-based ids, N = max id; duplicates and self-loops are kept
    p = tmp_path / "g.txt"
    p.write_text("1 2\n2 3\n3 1\n3 3\n3 1\n4 5\n")
    g = Graph.load_edge_list(str(p))
    assert g.num_nodes() == 5 and g.num_edges() == 6
    st = State(g)
    st.run(2)
    assert st.canonical_labels().tolist() == [0, 0, 0, 3, 4]


def test_binary_snapshot_roundtrip(gpu, tmp_path):
    n, s, d, csr = seeded_graph(rmat_scale=10, edge_factor=4, seed=3)
    g = Graph.from_edges(n, s, d)
    p = str(tmp_path / "g.bin")
    g.save_binary(p)
    h = Graph.load_binary(p)
    for x, y in zip(g.csr(), h.csr()):
        assert np.array_equal(x, y)


def test_decompose_csr_one_call(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=13, edge_factor=8, seed=41)
    lab, k, st = decompose_csr(csr[0], csr[1], csr[2], csr[3])
    exp = O.tarjan_canonical(csr[0], csr[1])
    assert np.array_equal(lab, exp) and k == len(np.unique(exp))


def test_histogram_and_counts(gpu, cases):
    c = [x for x in cases if x["name"] == "rmat16_ef8_seed42"][0]
    g = Graph.from_edges(c["n"], c["src"], c["dst"])
    st = State(g)
    st.run(2)
    h = st.histogram()
    sizes = np.bincount(np.unique(c["tarjan"], return_counts=True)[1])
    exp = {i: int(v) for i, v in enumerate(sizes) if v}
    assert h == exp


def test_state_reset_and_rerun(gpu):
    n, s, d, csr = seeded_graph(rmat_scale=12, edge_factor=8, seed=5)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    a = st.canonical_labels()
    st.reset()
    assert np.all(st.color() == -1) and np.all(st.scc() == -1)
    st.run(0)
    assert np.array_equal(st.canonical_labels(), a)


def test_colour_allocator(gpu):
    g = Graph.from_edges(3, [0, 1], [1, 2])
    st = State(g)
    assert st.get_curr_color() == -1
    assert [st.get_new_color() for _ in range(3)] == [0, 1, 2]
    assert st.get_curr_color() == 2


def test_generate_compact_set_and_pivot(gpu):
    s, d = random_graph(200, 600, 9)
    g = Graph.from_edges(200, s, d)
    st = State(g)
    col = np.full(200, -1, np.int32)
    col[::3] = 5
    st.set_color(col)
    assert np.array_equal(st.generate_compact_set(5), np.arange(0, 200, 3, dtype=np.int32))
    csr = O.build_csr(200, s, d)
    assert st.choose_pivot_from_color(5) == O.choose_pivot(csr, col, 5)
    assert st.choose_pivot_from_color(77) == -1


def test_pivot_tie_break_salt_changes_speed_not_labels(gpu):
    # other tie-breaks of the degree rule pick other equally good pivots; the
    # decomposition must not change
    n, s, d, csr = seeded_graph(rmat_scale=12, edge_factor=6, grid_side=96, seed=41)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g = Graph.from_edges(n, s, d)
    st = State(g)
    for salt in (7, 123456, -1):
        st.set_tuning(pivot_salt=salt)
        st.reset()
        st.run(2)
        assert np.array_equal(st.canonical_labels(), exp), salt
    assert st.get_tuning()["pivot_salt"] == 0
    st.free(); g.free()
