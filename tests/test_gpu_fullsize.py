"""GPU: the benchmark configurations at their full sizes (hundreds of millions
of edges), pinned to the reference itself.  tests/golden/fullsize_digests.json
holds, per configuration, the SHA-256 of the CSR and of the canonical labels
(component id = smallest member vertex) that the reference's own
do_tarjan_all produced on that CSR, together with its method 2 where that
runs (tests/golden/make_fullsize_digests.py made the file).  The device must
build the same CSR and give labels with the same digest.  Two
size-independent properties are checked beside: a graph and its transpose
have the same SCCs, and the SCC count is the number of vertices that label
themselves."""
import hashlib
import json
import os

import numpy as np
import pytest

from dynamicgraphs_scc_b200 import Graph, State

pytestmark = pytest.mark.gpu

DIGESTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fullsize_digests.json")
with open(DIGESTS) as _f:
    FULL = json.load(_f)


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype="<i4").tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_size_equals_reference_digest_and_transpose(gpu, name):
    ref = FULL[name]
    g = Graph.generate(**ref["params"])
    assert g.num_nodes() == ref["n"] and g.num_edges() == ref["m"]
    b, a, rb, ra = g.csr()
    assert _sha(b, a) == ref["csr_sha256"], name
    st = State(g)
    stats = st.run(2)
    lab = st.canonical_labels()
    st.free()
    g.free()
    assert _sha(lab) == ref["labels_sha256"], name
    assert stats["num_sccs"] == ref["num_sccs"]
    assert int(np.count_nonzero(lab == np.arange(lab.size, dtype=np.int32))) == ref["num_sccs"]
    assert int(np.bincount(lab).max()) == ref["largest_scc"]
    gt = Graph.from_csr(rb, ra, b, a)          # the transpose: same strongly connected components
    del b, a, rb, ra
    stt = State(gt)
    stt.run(2)
    assert np.array_equal(stt.canonical_labels(), lab), name
    stt.free(); gt.free()
