"""CPU: every struct the C ABI passes by pointer is laid out the same in the
headers (include/*.h) and in the Python binding: same fields, same order, same
C types.  A field added on one side only (a new tunable, a new statistic)
would shift every later field for ctypes callers and for reference-side
bindings generated from the header."""
import os
import re

import pytest

from dynamicgraphs_scc_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in ("scc_capi.h", "scc_gen_api.h")]

C_TYPES = {"double": "double", "int32_t": "int32", "int": "int32", "int64_t": "int64", "uint64_t": "uint64"}
CT_TYPES = {capi.C.c_double: "double", capi.C.c_int32: "int32", capi.C.c_int: "int32", capi.C.c_int64: "int64",
            capi.C.c_uint64: "uint64"}

PAIRS = {"scc_run_stats": capi.RunStats, "scc_update_stats": capi.UpdateStats,
         "scc_request_result": capi.RequestResult, "scc_server_stats": capi.ServerStats,
         "scc_tuning": capi.Tuning, "scc_batch_tuning": capi.BatchTuning, "scc_batch_stats": capi.BatchStats,
         "scc_gen_params": capi.GenParams, "scc_batch_params": capi.BatchParams}


def header_structs():
    text = ""
    for h in HEADERS:
        with open(h) as f:
            text += f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name, body, tail in re.findall(r"typedef struct (\w+) \{(.*?)\} (\w+);", text, flags=re.S):
        assert name == tail
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ctype, names = decl.split(None, 1)
            for n in names.split(","):
                fields.append((n.strip(), C_TYPES.get(ctype, ctype)))
        out[name] = fields
    return out


def binding_fields(cls):
    return [(n, CT_TYPES.get(t, getattr(t, "__name__", str(t)))) for n, t in cls._fields_]


NESTED = {capi.UpdateStats.__name__: "scc_update_stats"}


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_struct_matches_header(name):
    structs = header_structs()
    assert name in structs, f"{name} not declared in include/"
    got = [(n, NESTED.get(t, t)) for n, t in binding_fields(PAIRS[name])]
    assert got == structs[name]


def test_every_header_struct_is_bound():
    assert set(header_structs()) == set(PAIRS)
