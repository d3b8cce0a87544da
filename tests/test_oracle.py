"""CPU: pin the oracle against the reference's own outputs (golden fixtures and,
where it was built, the reference library itself), and check the phase
restatements against their defining properties."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import edge_digest, golden_cases, random_graph, seeded_graph


@pytest.fixture(scope="module")
def cases():
    return golden_cases()


def test_golden_inputs_unchanged(cases):
    for c in cases:
        if c["meta"]["kind"] == "gen":
            assert edge_digest(c["src"], c["dst"]) == c["meta"]["digest"], c["name"]
            assert c["src"].size == c["meta"]["m"]


def test_oracle_tarjan_matches_reference_fixtures(cases):
    for c in cases:
        csr = O.build_csr(c["n"], c["src"], c["dst"])
        lab = O.tarjan_canonical(csr[0], csr[1])
        assert np.array_equal(lab, c["tarjan"]), c["name"]
        assert np.array_equal(lab, c["m2"]), c["name"]


def test_known_answers(cases):
    by = {c["name"]: c for c in cases}
    assert np.array_equal(by["cycle8"]["tarjan"], np.zeros(8, np.int32))
    assert np.array_equal(by["dag_chain6"]["tarjan"], np.arange(6, dtype=np.int32))
    assert np.array_equal(by["two_cycles_2"]["tarjan"], np.array([0, 0, 2, 2, 4, 5], np.int32))
    assert np.array_equal(by["bowtie"]["tarjan"], np.array([0, 0, 0, 0, 0, 5, 6, 7], np.int32))
    assert np.array_equal(by["isolated_tail"]["tarjan"], np.array([0, 0, 0, 3, 4, 5, 6, 7, 8, 9], np.int32))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_vs_reference_library_random(seed):
    s, d = random_graph(3000, 4500, seed)
    csr = O.build_csr(3000, s, d)
    lab = O.tarjan_canonical(csr[0], csr[1])
    m2, _ = O.ref_method2(csr, threads=4)
    tj, _ = O.ref_tarjan(csr)
    assert np.array_equal(lab, m2)
    assert np.array_equal(lab, tj)


def _nbr_sets(csr):
    b, a, rb, ra = csr
    return b, a, rb, ra


def test_trim1_fixpoint_properties():
    n, s, d, csr = seeded_graph(rmat_scale=12, edge_factor=4, seed=9)
    b, a, rb, ra = csr
    color = np.full(n, -1, np.int32)
    scc = np.full(n, -1, np.int32)
    cnt = O.trim1_fixpoint(csr, color, scc)
    assert cnt == int((color == -2).sum())
    lab = O.tarjan_canonical(b, a)
    sizes = np.bincount(lab, minlength=n)
    # every trimmed vertex is a singleton SCC
    trimmed = np.where(color == -2)[0]
    assert np.all(sizes[lab[trimmed]] == 1)
    assert np.all(scc[trimmed] == trimmed)
    # fixpoint: every survivor has a live out- and in-neighbour other than itself
    live = color != -2
    for v in np.where(live)[0][:2000]:
        outs = a[b[v]:b[v + 1]]
        ins = ra[rb[v]:rb[v + 1]]
        assert np.any(live[outs] & (outs != v))
        assert np.any(live[ins] & (ins != v))


def test_trim2_pairs_are_sccs():
    n, s, d, csr = seeded_graph(rmat_scale=11, edge_factor=3, grid_side=40, seed=4)
    color = np.full(n, -1, np.int32)
    scc = np.full(n, -1, np.int32)
    O.trim1_fixpoint(csr, color, scc)
    before = color.copy()
    cnt = O.trim2(csr, color, scc)
    newly = np.where((before != -2) & (color == -2))[0]
    assert cnt == newly.size and cnt % 2 == 0
    lab = O.tarjan_canonical(csr[0], csr[1])
    sizes = np.bincount(lab, minlength=n)
    assert np.all(sizes[lab[newly]] == 2)
    # the pair representative is the smaller id of the pair
    for v in newly:
        assert scc[v] == lab[v]


def test_wcc_minreach_is_reachability_min():
    s, d = random_graph(400, 700, 12)
    csr = O.build_csr(400, s, d)
    b, a, rb, ra = csr
    color = np.full(400, -1, np.int32)
    w = O.wcc_minreach(csr, color)
    deg = np.diff(b)
    raw = np.where(deg >= 50, np.arange(400) | 0x20000000, np.arange(400)).astype(np.int64)
    for v in range(0, 400, 7):
        r = np.zeros(400, np.uint8)
        O.lib().orc_reach(400, O._p(b), O._p(a), O._p(color), -1, v, r.ctypes.data_as(O._U8P))
        assert w[v] == raw[r.astype(bool)].min()


def test_fw_bw_restatement_finds_pivot_scc():
    n, s, d, csr = seeded_graph(rmat_scale=12, edge_factor=8, seed=21)
    color = np.full(n, -1, np.int32)
    scc = np.full(n, -1, np.int32)
    O.trim1_fixpoint(csr, color, scc)
    p = O.choose_pivot(csr, color, -1)
    size, fw, bw = O.fw_bw(csr, color, scc, -1, p, 0, 1)
    lab = O.tarjan_canonical(csr[0], csr[1])
    assert size == int((lab == lab[p]).sum())
    assert np.all(scc[lab == lab[p]] == p)
    assert fw == int((color == 0).sum()) and bw == int((color == 1).sum())
