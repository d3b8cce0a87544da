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


# ---------------------------------------------------------------- learned pivot network
def _mlp_case(seed, n=48):
    rng = np.random.default_rng(seed)
    p = O.bf16((rng.standard_normal(O.MLP_PARAMS) * 0.3).astype(np.float32))
    x = O.bf16(rng.uniform(0, 6, (n, 8)).astype(np.float32))
    t = rng.uniform(0, 1, n).astype(np.float32)
    return p, x, t


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(4000).astype(np.float32) * 50,
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.0029296875, 65504.0, 3.4e38], np.float32)])
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(O.bf16(x), ref)
    assert all(O.bf16_scalar(float(v)) == r for v, r in zip(x[:200], ref[:200]))


def test_mlp_oracle_gradient_matches_finite_differences():
    """Pins the oracle's backward pass: central differences of the loss (double
    parameters, step 1e-6) against the analytic gradient, on the BF16 grid."""
    p, x, t = _mlp_case(7)
    loss, g = O.mlp_loss_grad(p, x, t)
    w = p.astype(np.float64)
    assert abs(O.mlp_loss(w, x, t) - loss) < 1e-12
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(512, 24, replace=False),                 # W1
                          512 + rng.choice(64, 8, replace=False),             # b1
                          576 + rng.choice(4096, 40, replace=False),          # W2
                          4672 + rng.choice(64, 8, replace=False),            # b2
                          4736 + rng.choice(64, 8, replace=False), [4800]])   # w3, b3
    h = 1e-6
    for i in idx:
        wp = w.copy(); wp[i] += h
        wm = w.copy(); wm[i] -= h
        fd = (O.mlp_loss(wp, x, t) - O.mlp_loss(wm, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (int(i), fd, g[i])


def test_mlp_oracle_forward_consistent_with_loss():
    p, x, t = _mlp_case(11)
    y = O.mlp_forward(p, x)
    assert abs(np.mean((y - t.astype(np.float64)) ** 2) - O.mlp_loss_grad(p, x, t)[0]) < 1e-12
    yb = O.mlp_forward(p, x, bf16_acts=True)          # activation rounding moves y only slightly
    assert np.max(np.abs(yb - y)) < 0.05 * (1 + np.max(np.abs(y)))


def test_pivot_features_oracle_known_answer():
    # 0 -> 1, 0 -> 2, 1 -> 0, 2 -> 0, 3 -> 0: vertex 0 has out-degree 2, in-degree 3
    n = 4
    s = np.array([0, 0, 1, 2, 3], np.int32); d = np.array([1, 2, 0, 0, 0], np.int32)
    csr = O.build_csr(n, s, d)
    f = O.pivot_features(csr, 0, class_size=3)
    exp = np.log1p(np.array([2, 3, 6, 2, 3, 3, 0, 0], np.float32))
    exp[6] = np.float32(np.log1p(1.0))               # out-neighbours 1, 2 have out-degree 1
    exp[7] = np.float32(np.log1p(1.0))               # in-neighbours 1, 2, 3: in-degrees 1, 1, 0
    np.testing.assert_allclose(f, O.bf16(exp), rtol=0, atol=0)
    cnt_out, cnt_in = O.trim_residue(csr, np.array([-1, -1, -1, 3], np.int32))   # vertex 3 trimmed
    assert list(cnt_out) == [2, 1, 1, 1] and list(cnt_in) == [2, 1, 1, 0]
    f2 = O.pivot_features(csr, 0, class_size=3, cnt_out=cnt_out, cnt_in=cnt_in)
    assert f2[4] == O.bf16(np.float32(np.log1p(2.0)))


# ---------------------------------------------------------------- method 7 levels
def _levels_by_max(begin, adj):
    """Longest path from the sources; nodes never released keep the largest
    level + 1 of their released predecessors (the order-free form)."""
    n = begin.size - 1
    indeg = np.bincount(adj, minlength=n).astype(np.int64)
    level = np.zeros(n, np.int64)
    stack = [v for v in range(n) if indeg[v] == 0]
    while stack:
        v = stack.pop()
        for c in adj[begin[v]:begin[v + 1]]:
            level[c] = max(level[c], level[v] + 1)
            indeg[c] -= 1
            if indeg[c] == 0:
                stack.append(int(c))
    return level


def test_topo_levels_known_answers():
    # chain 0->1->2->3 plus 0->3: longest path gives 3 its level 3
    b, a = O.condensation_csr(np.arange(4), 4, [0, 1, 2, 0], [1, 2, 3, 3])
    lev, ml = O.topo_levels(b, a)
    assert lev.tolist() == [0, 1, 2, 3] and ml == 3
    # diamond with a duplicate edge: 0->1, 0->2, 1->3, 2->3, 2->3
    b, a = O.condensation_csr(np.arange(4), 4, [0, 0, 1, 2, 2], [1, 2, 3, 3, 3])
    lev, ml = O.topo_levels(b, a)
    assert lev.tolist() == [0, 1, 1, 2] and ml == 2
    # labels that are not SCCs: 1<->2 is a cycle fed by 0, 3 hangs off it.
    # 1 and 2 are never released; 1 keeps 0's level + 1, 2 and 3 stay 0.
    b, a = O.condensation_csr(np.arange(4), 4, [0, 1, 2, 2], [1, 2, 1, 3])
    lev, ml = O.topo_levels(b, a)
    assert lev.tolist() == [0, 1, 0, 0] and ml == 1
    # affected: edge 3->0 covers levels [0, 2] of the diamond
    aff, z = O.affected_levels(np.arange(4), np.array([0, 1, 1, 2]), 2, [3], [0])
    assert aff.tolist() == [1, 1, 1] and z == 0
    aff, z = O.affected_levels(np.arange(4), np.array([0, 1, 1, 2]), 2, [1, 2], [2, 1])
    assert aff.tolist() == [0, 2, 0] and z == 2


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_topo_levels_fifo_equals_longest_path(seed):
    rng = np.random.default_rng(seed)
    n = 2000
    s = rng.integers(0, n, 3 * n).astype(np.int32)
    d = rng.integers(0, n, 3 * n).astype(np.int32)
    for ids, k in [O.scc_ids(O.tarjan_canonical(*O.build_csr(n, s, d)[:2])), (np.arange(n, dtype=np.int32), n)]:
        b, a = O.condensation_csr(ids, k, s, d)
        lev, ml = O.topo_levels(b, a)
        assert np.array_equal(lev, _levels_by_max(b, a))
        assert ml == int(lev.max(initial=0))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", [4, 5, 6, 7])
def test_method7_levels_match_reference(seed):
    """Levels and the prefix-summed affect_level against the reference's own
    create_scc_edges (met_algo 7) on seeded graphs and batches."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(500, 4000))
    m = int(n * rng.uniform(1.2, 2.5))
    s = rng.integers(0, n, m).astype(np.int32)
    d = rng.integers(0, n, m).astype(np.int32)
    ids, k = O.scc_ids(O.tarjan_canonical(*O.build_csr(n, s, d)[:2]))
    b, a = O.condensation_csr(ids, k, s, d)
    lev, ml = O.topo_levels(b, a)
    for nb in (1, 3, 10):
        isrc = rng.integers(0, n, nb).astype(np.int32)
        idst = rng.integers(0, n, nb).astype(np.int32)
        aff, z = O.affected_levels(ids, lev, ml, isrc, idst)
        if z == 0:
            continue                  # the reference's closing loop needs an unaffected level
        rl, ra = O.ref_method7_levels(n, s, d, isrc, idst, ids, k)
        assert np.array_equal(rl, lev)
        assert np.array_equal(ra[:ml + 1], aff)
