"""CPU: the C-ABI library loads, exports every symbol the public headers
declare, and rejects bad arguments with status codes (no GPU work)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from dynamicgraphs_scc_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(scc_\w+)\s*\(", text, flags=re.M):
            syms.append(m.group(1))
    return sorted(set(syms))


def test_library_loads():
    L = capi.lib()
    assert L.scc_version() >= 100


def test_every_declared_symbol_is_exported():
    L = capi.lib()
    syms = header_symbols()
    assert len(syms) >= 60
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    declared = set(capi.declared_symbols())
    missing = [s for s in header_symbols() if s not in declared]
    assert not missing, missing


def test_status_strings():
    L = capi.lib()
    for code in range(0, 9):
        assert L.scc_status_string(code)


def test_null_arguments_are_rejected():
    L = capi.lib()
    assert L.scc_graph_num_nodes(None, None) == 1
    assert L.scc_state_create(None, None) == 1
    assert L.scc_run(None, None, 2, 0, None) == 1
    assert b"NULL" in L.scc_last_error()


def test_bad_sizes_rejected_before_device_work():
    L = capi.lib()
    h = C.c_void_p()
    s = np.zeros(1, np.int32)
    assert L.scc_graph_create_edges(-1, 1, capi.i32p(s), capi.i32p(s), 0, 0, C.byref(h)) == 1
    assert L.scc_graph_create_csr(-5, 0, capi.i32p(s), None, None, None, 0, C.byref(h)) == 1


def test_missing_file_is_io_error(tmp_path):
    L = capi.lib()
    h = C.c_void_p()
    assert L.scc_graph_load_edge_list(str(tmp_path / "nope.txt").encode(), 0, C.byref(h)) == 6
    assert L.scc_graph_load_binary(str(tmp_path / "nope.bin").encode(), 0, C.byref(h)) == 6


def test_scc_list_reader(tmp_path):
    p = tmp_path / "scc_list.txt"
    p.write_text("0 0\n1 0\n2 1\n3 2\n")
    from dynamicgraphs_scc_b200 import read_scc_list
    lab, k = read_scc_list(str(p), 4)
    assert k == 3 and lab.tolist() == [0, 0, 1, 2]


def test_host_generator_is_deterministic():
    from dynamicgraphs_scc_b200 import generate_edges_host
    a = generate_edges_host(rmat_scale=10, edge_factor=4, grid_side=16, seed=5)
    b = generate_edges_host(rmat_scale=10, edge_factor=4, grid_side=16, seed=5)
    c = generate_edges_host(rmat_scale=10, edge_factor=4, grid_side=16, seed=6)
    assert a[0] == b[0] == 1024 + 256
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert not np.array_equal(a[1], c[1])
    assert a[1].max() < a[0] and a[2].max() < a[0] and a[1].min() >= 0


def test_generator_rejects_bad_params():
    from dynamicgraphs_scc_b200 import generate_edges_host
    from dynamicgraphs_scc_b200.capi import SccError
    with pytest.raises(SccError):
        generate_edges_host(rmat_scale=40, edge_factor=1)


def test_read_edge_list_host_parser(tmp_path):
    """read_file's format on the host (no device work): 1-based ids, comment
    lines skipped, N = the largest id, malformed lines rejected."""
    from dynamicgraphs_scc_b200 import SccError, read_edge_list
    p = tmp_path / "e.txt"
    p.write_text("% header\n1 2\n2 3\n# note\n3 1\n7 7\n")
    s, d, n = read_edge_list(str(p))
    assert s.tolist() == [0, 1, 2, 6] and d.tolist() == [1, 2, 0, 6] and n == 7
    p.write_text("")
    s, d, n = read_edge_list(str(p))
    assert s.size == 0 and n == 0
    p.write_text("1 x\n")
    with pytest.raises(SccError):
        read_edge_list(str(p))
