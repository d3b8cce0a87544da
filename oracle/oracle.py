"""CPU oracle for the SCC engine -- TEST INFRASTRUCTURE ONLY.

Loads two native libraries built by oracle/Makefile:
  build/liboracle.so  -- the C restatement of the reference algorithms (scc_oracle.c) and of
                         the learned pivot network, its gradient and features (mlp_oracle.c);
  _ref/libscc_ref.so  -- the reference's own OpenMP engine compiled from its sources
                         plus ref_harness.cc (optional: absent if never built).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libscc_ref.so")
REF_CLI = os.path.join(HERE, "_ref", "scc")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libscc_ref_cuda.so")

_I32P = C.POINTER(C.c_int32)
_U8P = C.POINTER(C.c_uint8)
_I64P = C.POINTER(C.c_int64)
_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_lib = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data_as(_I32P)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(ORACLE_SO)
        L.orc_build_csr.argtypes = [C.c_int32, C.c_int64, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P]
        L.orc_build_csr.restype = None
        L.orc_dedup_edges.argtypes = [C.c_int32, C.c_int64, _I32P, _I32P]
        L.orc_dedup_edges.restype = C.c_int64
        L.orc_tarjan.argtypes = [C.c_int32, _I32P, _I32P, _I32P]
        L.orc_tarjan.restype = None
        L.orc_canonical.argtypes = [C.c_int32, _I32P, _I32P]
        L.orc_canonical.restype = None
        L.orc_scc_canonical.argtypes = [C.c_int32, _I32P, _I32P, _I32P]
        L.orc_scc_canonical.restype = None
        L.orc_trim1_fixpoint.argtypes = [C.c_int32, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P]
        L.orc_trim1_fixpoint.restype = C.c_int64
        L.orc_trim2.argtypes = [C.c_int32, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P]
        L.orc_trim2.restype = C.c_int64
        L.orc_wcc_minreach.argtypes = [C.c_int32, _I32P, _I32P, _I32P, _I32P, _I32P]
        L.orc_wcc_minreach.restype = None
        L.orc_reach.argtypes = [C.c_int32, _I32P, _I32P, _I32P, C.c_int32, C.c_int32, _U8P]
        L.orc_reach.restype = C.c_int64
        L.orc_fw_bw.argtypes = [C.c_int32, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P, C.c_int32, C.c_int32,
                                C.c_int32, C.c_int32, _I64P, _I64P]
        L.orc_fw_bw.restype = C.c_int64
        L.orc_choose_pivot.argtypes = [C.c_int32, _I32P, _I32P, _I32P, C.c_int32]
        L.orc_topo_levels.argtypes = [C.c_int32, _I32P, _I32P, _I32P]
        L.orc_topo_levels.restype = C.c_int32
        L.orc_affected_levels.argtypes = [_I32P, _I32P, C.c_int32, C.c_int64, _I32P, _I32P, _I32P]
        L.orc_affected_levels.restype = C.c_int32
        L.orc_choose_pivot.restype = C.c_int32
        L.orc_bf16.argtypes = [C.c_float]
        L.orc_bf16.restype = C.c_float
        L.orc_mlp_forward.argtypes = [_F32P, _F32P, C.c_int64, C.c_int, _F64P]
        L.orc_mlp_forward.restype = None
        L.orc_mlp_loss_grad.argtypes = [_F32P, _F32P, _F32P, C.c_int64, _F64P]
        L.orc_mlp_loss_grad.restype = C.c_double
        L.orc_mlp_loss.argtypes = [_F64P, _F32P, _F32P, C.c_int64]
        L.orc_mlp_loss.restype = C.c_double
        L.orc_pivot_features.argtypes = [_I32P, _I32P, _I32P, _I32P, _I32P, _I32P, C.c_int32, C.c_int32, _F32P]
        L.orc_pivot_features.restype = None
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        L.ref_method2.argtypes = [C.c_int32, C.c_int64, _I32P, _I32P, C.c_int, C.c_int, _I32P,
                                  C.POINTER(C.c_double)]
        L.ref_method2.restype = C.c_int
        L.ref_method.argtypes = [C.c_int, C.c_int32, C.c_int64, _I32P, _I32P, C.c_int, C.c_int, _I32P,
                                 C.POINTER(C.c_double)]
        L.ref_method.restype = C.c_int
        L.ref_tarjan.argtypes = [C.c_int32, C.c_int64, _I32P, _I32P, _I32P, C.POINTER(C.c_double)]
        L.ref_tarjan.restype = C.c_int
        L.ref_method7_levels.argtypes = [C.c_int32, C.c_int64, _I32P, _I32P, C.c_int64, _I32P, _I32P, _I32P,
                                         C.c_int32, _I32P, _I32P]
        L.ref_method7_levels.restype = C.c_int
        _ref = L
    return _ref


# ------------------------------------------------------------------------ graph helpers
def dedup_edges(src, dst, drop_self_loops=True, n=None):
    """Remove self-loops and duplicate (src, dst) pairs (the generators' post-processing),
    returned sorted by (src, dst)."""
    if drop_self_loops and n is not None:
        s = np.array(src, np.int32, copy=True)
        d = np.array(dst, np.int32, copy=True)
        k = lib().orc_dedup_edges(n, s.size, _p(s), _p(d))
        return s[:k].copy(), d[:k].copy()
    s = np.asarray(src, np.int64)
    d = np.asarray(dst, np.int64)
    if drop_self_loops:
        keep = s != d
        s, d = s[keep], d[keep]
    key = np.unique((s << 32) | d)
    return (key >> 32).astype(np.int32), (key & 0xFFFFFFFF).astype(np.int32)


def build_csr(n, src, dst):
    """gm_graph CSR + transpose, adjacency sorted (freeze + semi-sort + make_reverse_edges)."""
    s = np.ascontiguousarray(src, np.int32)
    d = np.ascontiguousarray(dst, np.int32)
    m = s.size
    b = np.empty(n + 1, np.int32); a = np.empty(max(m, 1), np.int32)
    rb = np.empty(n + 1, np.int32); ra = np.empty(max(m, 1), np.int32)
    lib().orc_build_csr(n, m, _p(s), _p(d), _p(b), _p(a), _p(rb), _p(ra))
    return b, a[:m].copy(), rb, ra[:m].copy()


def canonical(scc):
    scc = np.ascontiguousarray(scc, np.int32)
    out = np.empty_like(scc)
    lib().orc_canonical(scc.size, _p(scc), _p(out))
    return out


def tarjan_canonical(begin, node_idx):
    n = begin.size - 1
    out = np.empty(max(n, 1), np.int32)
    lib().orc_scc_canonical(n, _p(begin), _p(node_idx), _p(out))
    return out[:n]


def trim1_fixpoint(csr, color, scc):
    b, a, rb, ra = csr
    return int(lib().orc_trim1_fixpoint(b.size - 1, _p(b), _p(a), _p(rb), _p(ra), _p(color), _p(scc)))


def trim2(csr, color, scc):
    b, a, rb, ra = csr
    return int(lib().orc_trim2(b.size - 1, _p(b), _p(a), _p(rb), _p(ra), _p(color), _p(scc)))


def wcc_minreach(csr, color):
    b, a, rb, ra = csr
    n = b.size - 1
    out = np.empty(max(n, 1), np.int32)
    lib().orc_wcc_minreach(n, _p(b), _p(rb), _p(ra), _p(color), _p(out))
    return out[:n]


def choose_pivot(csr, color, c):
    b, a, rb, ra = csr
    return int(lib().orc_choose_pivot(b.size - 1, _p(b), _p(rb), _p(color), c))


def fw_bw(csr, color, scc, base, pivot, fw_color, bw_color):
    b, a, rb, ra = csr
    f = C.c_int64(); w = C.c_int64()
    s = lib().orc_fw_bw(b.size - 1, _p(b), _p(a), _p(rb), _p(ra), _p(color), _p(scc), base, pivot, fw_color,
                        bw_color, C.byref(f), C.byref(w))
    return int(s), f.value, w.value


class _QuietStdout:
    """Send the reference's own printf output (it announces each method on stdout)
    to /dev/null, flushing C stdio before the descriptor is restored."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def ref_method(method, csr, threads=None, pin=False, quiet=True):
    """The reference's own method-0/1/2 pipeline (my_main::run): (canonical labels, run ms)."""
    b, a = csr[0], csr[1]
    n = b.size - 1
    out = np.empty(max(n, 1), np.int32)
    ms = C.c_double()
    th = threads or os.cpu_count() or 1
    if quiet:
        with _QuietStdout():
            rc = ref().ref_method(method, n, a.size, _p(b), _p(a), th, int(pin), _p(out), C.byref(ms))
    else:
        rc = ref().ref_method(method, n, a.size, _p(b), _p(a), th, int(pin), _p(out), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference method {method} failed")
    return canonical(out[:n]), ms.value


def ref_method2(csr, threads=None, pin=False, quiet=True):
    """The reference's own method-2 pipeline: (canonical labels, run ms)."""
    return ref_method(2, csr, threads=threads, pin=pin, quiet=quiet)


_ref_cuda = None


def ref_cuda_available() -> bool:
    return os.path.exists(REF_CUDA_SO)


def ref_cuda_method2(csr, threads=None, quiet=True):
    """The reference's own CUDA method 2 (src_CUDA, built for sm_100a) on the
    current GPU, from a CSR and its transpose: (canonical labels, run ms)."""
    global _ref_cuda
    if _ref_cuda is None:
        L = C.CDLL(REF_CUDA_SO)
        L.refcuda_method2.argtypes = [C.c_int32, C.c_int64, _I32P, _I32P, _I32P, _I32P, C.c_int, _I32P,
                                      C.POINTER(C.c_double)]
        L.refcuda_method2.restype = C.c_int
        _ref_cuda = L
    b, a, rb, ra = csr
    n = b.size - 1
    out = np.empty(max(n, 1), np.int32)
    ms = C.c_double()
    th = threads or os.cpu_count() or 1
    if quiet:
        with _QuietStdout():
            rc = _ref_cuda.refcuda_method2(n, a.size, _p(b), _p(a), _p(rb), _p(ra), th, _p(out), C.byref(ms))
    else:
        rc = _ref_cuda.refcuda_method2(n, a.size, _p(b), _p(a), _p(rb), _p(ra), th, _p(out), C.byref(ms))
    if rc != 0:
        raise RuntimeError("reference CUDA method 2 failed")
    return out[:n].copy(), ms.value


def ref_tarjan(csr):
    """The reference's own do_tarjan_all: (canonical labels, run ms)."""
    b, a = csr[0], csr[1]
    n = b.size - 1
    out = np.empty(max(n, 1), np.int32)
    ms = C.c_double()
    rc = ref().ref_tarjan(n, a.size, _p(b), _p(a), _p(out), C.byref(ms))
    if rc != 0:
        raise RuntimeError("reference Tarjan failed")
    return canonical(out[:n]), ms.value


# ---------------------------------------------------------------- method 7 levels (scc_oracle.c)
def scc_ids(labels):
    """scc_list.txt ids of canonical labels: numbered by first appearance over
    the vertices (output_scc_list, src/scc_post_analyze.cc:31-53)."""
    labels = np.asarray(labels)
    first = {}
    out = np.empty(labels.size, np.int32)
    for i, r in enumerate(labels.tolist()):
        out[i] = first.setdefault(r, len(first))
    return out, len(first)


def condensation_csr(ids, num_sccs, src, dst):
    """The original edges' condensation as create_scc_edges builds adj_list:
    one entry per edge joining two SCCs, duplicates kept, in edge order."""
    ids = np.asarray(ids, np.int64)
    a = ids[np.asarray(src, np.int64)]
    b = ids[np.asarray(dst, np.int64)]
    keep = a != b
    a, b = a[keep], b[keep]
    order = np.argsort(a, kind="stable")
    begin = np.zeros(num_sccs + 1, np.int32)
    np.add.at(begin, a + 1, 1)
    return np.cumsum(begin).astype(np.int32), b[order].astype(np.int32)


def topo_levels(begin, adj):
    """(levels, max_level) by the reference's FIFO level BFS."""
    n = begin.size - 1
    lev = np.empty(max(n, 1), np.int32)
    m = lib().orc_topo_levels(n, _p(np.ascontiguousarray(begin, np.int32)),
                              _p(np.ascontiguousarray(adj, np.int32) if adj.size else np.zeros(1, np.int32)), _p(lev))
    return lev[:n], int(m)


def affected_levels(ids, levels, max_level, src, dst):
    """(affected[0..max_level], number of unaffected levels)."""
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    out = np.empty(max_level + 1, np.int32)
    z = lib().orc_affected_levels(_p(np.ascontiguousarray(ids, np.int32)), _p(np.ascontiguousarray(levels, np.int32)),
                                  max_level, src.size, _p(src if src.size else np.zeros(1, np.int32)),
                                  _p(dst if dst.size else np.zeros(1, np.int32)), _p(out))
    return out, int(z)


def ref_method7_levels(nv, src, dst, ins_src, ins_dst, ids, num_sccs):
    """The reference's own create_scc_edges with met_algo 7: (level_ver,
    prefix-summed affect_level).  Only for batches that leave a level
    unaffected (its closing loop misbehaves otherwise)."""
    src, dst = np.ascontiguousarray(src, np.int32), np.ascontiguousarray(dst, np.int32)
    isrc, idst = np.ascontiguousarray(ins_src, np.int32), np.ascontiguousarray(ins_dst, np.int32)
    lev = np.empty(max(num_sccs, 1), np.int32)
    aff = np.empty(num_sccs + 5, np.int32)
    one = np.zeros(1, np.int32)
    with _QuietStdout():
        rc = ref().ref_method7_levels(nv, src.size, _p(src if src.size else one), _p(dst if dst.size else one),
                                      isrc.size, _p(isrc if isrc.size else one), _p(idst if idst.size else one),
                                      _p(np.ascontiguousarray(ids, np.int32)), num_sccs, _p(lev), _p(aff))
    if rc != 0:
        raise RuntimeError("reference create_scc_edges failed")
    return lev[:num_sccs], aff


# ---------------------------------------------------------------- learned pivot network (mlp_oracle.c)
MLP_PARAMS = 4801


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even), numpy restatement."""
    x = _f32(x)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    out = u.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), x, out)


def bf16_scalar(v: float) -> float:
    return float(lib().orc_bf16(v))


def mlp_forward(params, x, bf16_acts=False):
    p = _f32(params); xx = _f32(x).reshape(-1, 8)
    y = np.empty(xx.shape[0], np.float64)
    lib().orc_mlp_forward(p.ctypes.data_as(_F32P), xx.ctypes.data_as(_F32P), xx.shape[0], int(bf16_acts),
                          y.ctypes.data_as(_F64P))
    return y


def mlp_loss_grad(params, x, t):
    p = _f32(params); xx = _f32(x).reshape(-1, 8); tt = _f32(t)
    g = np.empty(MLP_PARAMS, np.float64)
    loss = lib().orc_mlp_loss_grad(p.ctypes.data_as(_F32P), xx.ctypes.data_as(_F32P), tt.ctypes.data_as(_F32P),
                                   xx.shape[0], g.ctypes.data_as(_F64P))
    return float(loss), g


def mlp_loss(params64, x, t):
    """Loss at double parameters taken as given (no BF16 rounding)."""
    p = np.ascontiguousarray(np.asarray(params64, np.float64)); xx = _f32(x).reshape(-1, 8); tt = _f32(t)
    return float(lib().orc_mlp_loss(p.ctypes.data_as(_F64P), xx.ctypes.data_as(_F32P), tt.ctypes.data_as(_F32P),
                                    xx.shape[0]))


def pivot_features(csr, v, class_size, cnt_out=None, cnt_in=None):
    b, a, rb, ra = csr
    f = np.empty(8, np.float32)
    lib().orc_pivot_features(_p(b), _p(a), _p(rb), _p(ra), _p(cnt_out), _p(cnt_in), int(v), int(class_size),
                             f.ctypes.data_as(_F32P))
    return f


def trim_residue(csr, scc_after_trim):
    """Live out/in neighbours (self-loops excluded) of every vertex after the
    first Trim1 fixpoint: the engine's trim-residue features."""
    b, a, rb, ra = csr
    n = b.size - 1
    live = scc_after_trim < 0
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(b))
    ok = live[a] & (a != src)
    cnt_out = np.bincount(src[ok], minlength=n).astype(np.int32)
    rsrc = np.repeat(np.arange(n, dtype=np.int64), np.diff(rb))
    ok = live[ra] & (ra != rsrc)
    cnt_in = np.bincount(rsrc[ok], minlength=n).astype(np.int32)
    return cnt_out, cnt_in
