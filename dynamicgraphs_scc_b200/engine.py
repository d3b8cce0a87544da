"""Python mirror of the reference's SCC phase API over the C ABI.

Names and argument meanings follow the reference's phase functions
(ShashwaTTrigunayaT/DynamicGraphs_SCC src/scc.h:18-92): a ``Graph`` stands for
gm_graph (int32 CSR + transpose, here resident on the GPU) and a ``State`` for
the G_Color / G_SCC globals plus the work queue.  Errors raise ``SccError``
instead of the reference's assert()/exit(1).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import SccError, call, f32p, i32p

METHOD_BASELINE = 0
METHOD_GLOBAL_FB = 1
METHOD_GLOBAL_WCC_FB = 2
PIVOT_DEGREE = 0
PIVOT_LEARNED = 1


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class Graph:
    """Device-resident CSR + transpose (gm_graph / GPUGraph)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    # -- construction -------------------------------------------------------------------------
    @classmethod
    def from_edges(cls, n: int, src, dst, flags: int = capi.SCC_BUILD_KEEP_ALL, device: int = 0) -> "Graph":
        s, d = _i32(src), _i32(dst)
        if s.shape != d.shape:
            raise ValueError("src and dst differ in length")
        h = C.c_void_p()
        call("scc_graph_create_edges", n, int(s.size), i32p(s), i32p(d), flags, device, C.byref(h))
        return cls(h)

    @classmethod
    def from_csr(cls, begin, node_idx, r_begin=None, r_node_idx=None, device: int = 0) -> "Graph":
        b, a = _i32(begin), _i32(node_idx)
        rb = _i32(r_begin) if r_begin is not None else None
        ra = _i32(r_node_idx) if r_node_idx is not None else None
        h = C.c_void_p()
        call("scc_graph_create_csr", int(b.size - 1), int(a.size), i32p(b), i32p(a), i32p(rb), i32p(ra), device,
             C.byref(h))
        return cls(h)

    @classmethod
    def load_edge_list(cls, path: str, device: int = 0) -> "Graph":
        h = C.c_void_p()
        call("scc_graph_load_edge_list", path.encode(), device, C.byref(h))
        return cls(h)

    @classmethod
    def load_binary(cls, path: str, device: int = 0) -> "Graph":
        h = C.c_void_p()
        call("scc_graph_load_binary", path.encode(), device, C.byref(h))
        return cls(h)

    @classmethod
    def generate(cls, rmat_scale=0, edge_factor=0, grid_side=0, num_cycles=0, cycle_min=3, cycle_max=100000,
                 seed=1, flags=capi.SCC_BUILD_DEDUP | capi.SCC_BUILD_NO_SELF_LOOPS, device=0) -> "Graph":
        p = gen_params(rmat_scale, edge_factor, grid_side, num_cycles, cycle_min, cycle_max, seed)
        h = C.c_void_p()
        call("scc_gen_graph", C.byref(p), flags, device, C.byref(h))
        return cls(h)

    @classmethod
    def generate_batch(cls, num_graphs=4096, n_min=1024, n_max=65536, mean_degree=6.0, rmat_fraction=0.3, seed=1,
                       flags=capi.SCC_BUILD_DEDUP | capi.SCC_BUILD_NO_SELF_LOOPS, device=0):
        """Disjoint union of many seeded uneven graphs; returns (graph, per-graph vertex offsets)."""
        p = capi.BatchParams(num_graphs, n_min, n_max, mean_degree, rmat_fraction, seed)
        offs = np.empty(num_graphs + 1, np.int32)
        call("scc_gen_batch_layout", C.byref(p), i32p(offs), None, None)
        h = C.c_void_p()
        call("scc_gen_batch_graph", C.byref(p), flags, device, C.byref(h))
        return cls(h), offs

    def subgraph(self, v_begin: int, v_end: int) -> "Graph":
        """Induced subgraph on a closed id range (one graph of a batch), rebased to 0."""
        h = C.c_void_p()
        call("scc_graph_subgraph", self.handle, v_begin, v_end, C.byref(h))
        return Graph(h)

    # -- properties ---------------------------------------------------------------------------
    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise SccError(5, "Graph", "graph was freed")
        return self._h

    def num_nodes(self) -> int:
        n = C.c_int32()
        call("scc_graph_num_nodes", self.handle, C.byref(n))
        return n.value

    def num_edges(self) -> int:
        m = C.c_int64()
        call("scc_graph_num_edges", self.handle, C.byref(m))
        return m.value

    def csr(self):
        n, m = self.num_nodes(), self.num_edges()
        b = np.empty(n + 1, np.int32); a = np.empty(m, np.int32)
        rb = np.empty(n + 1, np.int32); ra = np.empty(m, np.int32)
        call("scc_graph_copy_csr", self.handle, i32p(b), i32p(a), i32p(rb), i32p(ra))
        return b, a, rb, ra

    def upload_csr(self, begin, node_idx, r_begin=None, r_node_idx=None, stream: int = 0) -> None:
        """Replace the graph's contents with host CSR arrays of the same n and m; without a
        transpose, only the forward CSR crosses the bus and the transpose is rebuilt on the device."""
        b, a = _i32(begin), _i32(node_idx)
        if r_begin is None:
            call("scc_graph_upload_csr_out", self.handle, b.ctypes.data, a.ctypes.data, stream or None)
        else:
            rb, ra = _i32(r_begin), _i32(r_node_idx)
            call("scc_graph_upload_csr", self.handle, b.ctypes.data, a.ctypes.data, rb.ctypes.data, ra.ctypes.data,
                 stream or None)

    def save_binary(self, path: str) -> None:
        call("scc_graph_save_binary", self.handle, path.encode())

    def free(self) -> None:
        if self._h is not None:
            capi.lib().scc_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def gen_params(rmat_scale=0, edge_factor=0, grid_side=0, num_cycles=0, cycle_min=3, cycle_max=100000, seed=1):
    return capi.GenParams(rmat_scale, edge_factor, grid_side, num_cycles, cycle_min, cycle_max, seed)


def generate_edges_host(**kw):
    """Raw seeded edge list on the host (the same multiset Graph.generate builds)."""
    p = gen_params(**kw)
    n = C.c_int32(); cap = C.c_int64()
    call("scc_gen_sizes", C.byref(p), C.byref(n), C.byref(cap))
    src = np.empty(max(cap.value, 1), np.int32)
    dst = np.empty(max(cap.value, 1), np.int32)
    m = C.c_int64()
    call("scc_gen_edges_host", C.byref(p), i32p(src), i32p(dst), cap.value, C.byref(m))
    return n.value, src[:m.value], dst[:m.value]


def generate_batch_edges_host(num_graphs=8, n_min=1024, n_max=65536, mean_degree=6.0, rmat_fraction=0.3, seed=1):
    """Raw edges of a seeded batch on the host: (n, offsets, src, dst)."""
    p = capi.BatchParams(num_graphs, n_min, n_max, mean_degree, rmat_fraction, seed)
    offs = np.empty(num_graphs + 1, np.int32)
    n = C.c_int32(); cap = C.c_int64()
    call("scc_gen_batch_layout", C.byref(p), i32p(offs), C.byref(n), C.byref(cap))
    src = np.empty(max(cap.value, 1), np.int32); dst = np.empty(max(cap.value, 1), np.int32)
    m = C.c_int64()
    call("scc_gen_batch_edges_host", C.byref(p), i32p(src), i32p(dst), cap.value, C.byref(m))
    return n.value, offs, src[:m.value], dst[:m.value]


class State:
    """G_Color / G_SCC / work queue (GPUState); one per graph run."""

    def __init__(self, graph: Graph):
        self.graph = graph
        h = C.c_void_p()
        call("scc_state_create", graph.handle, C.byref(h))
        self._h = h
        self.n = graph.num_nodes()

    @property
    def handle(self):
        if self._h is None:
            raise SccError(5, "State", "state was freed")
        return self._h

    def _g(self):
        return self.graph.handle

    def _out(self):
        return C.c_int32(0)

    # -- arrays ----------------------------------------------------------------------------------
    def reset(self):
        call("scc_state_reset", self.handle)

    def color(self) -> np.ndarray:
        a = np.empty(self.n, np.int32)
        call("scc_state_get_color", self.handle, i32p(a))
        return a

    def scc(self) -> np.ndarray:
        a = np.empty(self.n, np.int32)
        call("scc_state_get_scc", self.handle, i32p(a))
        return a

    def wcc(self) -> np.ndarray:
        a = np.empty(self.n, np.int32)
        call("scc_state_get_wcc", self.handle, i32p(a))
        return a

    def set_color(self, a) -> None:
        call("scc_state_set_color", self.handle, i32p(_i32(a)))

    def set_scc(self, a) -> None:
        call("scc_state_set_scc", self.handle, i32p(_i32(a)))

    def finish_unaffected(self, levels, affected, max_level: int) -> int:
        """Method 7's trim shortcut: finish every node of an unaffected level as its own SCC."""
        k = C.c_int32()
        call("scc_state_finish_unaffected", self.handle, i32p(_i32(levels)), i32p(_i32(affected)), max_level,
             C.byref(k))
        return k.value

    def trim_targets(self) -> np.ndarray:
        c = C.c_int32()
        call("scc_state_get_trim_targets", self.handle, None, 0, C.byref(c))
        a = np.empty(c.value, np.int32)
        call("scc_state_get_trim_targets", self.handle, i32p(a), c.value, C.byref(c))
        return a

    def stream(self) -> int:
        p = C.c_void_p()
        call("scc_state_stream", self.handle, C.byref(p))
        return p.value or 0

    def synchronize(self) -> None:
        call("scc_state_synchronize", self.handle)

    def get_tuning(self) -> dict:
        t = capi.Tuning()
        call("scc_state_get_tuning", self.handle, C.byref(t))
        return t.as_dict()

    def autotune(self, method: int = METHOD_GLOBAL_WCC_FB, max_trials: int = 32):
        """Grid-search the tunables on this state's graph; keeps and returns the fastest."""
        t = capi.Tuning()
        ms = C.c_double()
        call("scc_autotune", self._g(), self.handle, method, max_trials, C.byref(t), C.byref(ms))
        return t.as_dict(), ms.value

    def set_tuning(self, **kw) -> None:
        """Change traversal tunables (keys of scc_tuning); unspecified keys keep their value."""
        t = capi.Tuning(*([0] * len(capi.Tuning._fields_)))
        for k, v in kw.items():
            if not hasattr(t, k):
                raise KeyError(k)
            setattr(t, k, int(v))
        call("scc_state_set_tuning", self.handle, C.byref(t))

    # -- colour ----------------------------------------------------------------------------------
    def get_new_color(self) -> int:
        o = self._out(); call("scc_get_new_color", self.handle, C.byref(o)); return o.value

    def get_curr_color(self) -> int:
        o = self._out(); call("scc_get_curr_color", self.handle, C.byref(o)); return o.value

    def choose_pivot_from_color(self, color: int) -> int:
        o = self._out()
        rc = capi.lib().scc_choose_pivot_from_color(self._g(), self.handle, color, C.byref(o))
        if rc == 7:
            return capi.SCC_NIL_NODE
        if rc != 0:
            raise SccError(rc, "scc_choose_pivot_from_color", capi.lib().scc_last_error().decode())
        return o.value

    def generate_compact_set(self, color: int) -> np.ndarray:
        c = C.c_int32()
        call("scc_generate_compact_set", self._g(), self.handle, color, None, 0, C.byref(c))
        a = np.empty(c.value, np.int32)
        call("scc_generate_compact_set", self._g(), self.handle, color, i32p(a), c.value, C.byref(c))
        return a

    # -- trim ------------------------------------------------------------------------------------
    def do_global_trim1(self) -> int:
        o = self._out(); call("scc_do_global_trim1", self._g(), self.handle, C.byref(o)); return o.value

    def do_global_trim1_compact(self) -> int:
        o = self._out(); call("scc_do_global_trim1_compact", self._g(), self.handle, C.byref(o)); return o.value

    def repeat_global_trim1(self, trim_stop: int = 100) -> int:
        o = self._out(); call("scc_repeat_global_trim1", self._g(), self.handle, trim_stop, C.byref(o)); return o.value

    def repeat_global_trim1_compact(self, trim_stop: int = 100) -> int:
        o = self._out()
        call("scc_repeat_global_trim1_compact", self._g(), self.handle, trim_stop, C.byref(o))
        return o.value

    def create_trim1_compact(self) -> int:
        o = self._out(); call("scc_create_trim1_compact", self._g(), self.handle, C.byref(o)); return o.value

    def do_global_trim2_new(self) -> int:
        o = self._out(); call("scc_do_global_trim2_new", self._g(), self.handle, C.byref(o)); return o.value

    def do_global_trim2(self) -> int:
        o = self._out(); call("scc_do_global_trim2", self._g(), self.handle, C.byref(o)); return o.value

    def repeat_global_trim2_new(self, exit_count: int = 100) -> int:
        o = self._out()
        call("scc_repeat_global_trim2_new", self._g(), self.handle, exit_count, C.byref(o))
        return o.value

    # -- FW-BW / WCC ---------------------------------------------------------------------------
    def do_fw_bw_global_main(self, curr_color: int = -1, count: int = 0, create_work_items: bool = False) -> int:
        o = self._out()
        call("scc_do_fw_bw_global_main", self._g(), self.handle, curr_color, count, int(create_work_items), C.byref(o))
        return o.value

    def do_fw_bw_global_pivot(self, curr_color: int, pivot: int, create_work_items: bool = False) -> int:
        o = self._out()
        call("scc_do_fw_bw_global_pivot", self._g(), self.handle, curr_color, pivot, int(create_work_items), C.byref(o))
        return o.value

    def create_works_after_bfs_trim(self) -> int:
        o = self._out(); call("scc_create_works_after_bfs_trim", self._g(), self.handle, C.byref(o)); return o.value

    def start_workers_fw_bw(self, local_items: int = 1) -> None:
        call("scc_start_workers_fw_bw", self._g(), self.handle, local_items)

    def start_workers_fw_bw_dfs(self, local_items: int = 40) -> None:
        call("scc_start_workers_fw_bw_dfs", self._g(), self.handle, local_items)

    def work_q_size(self) -> int:
        o = self._out(); call("scc_work_q_size", self.handle, C.byref(o)); return o.value

    def work_q_items(self):
        k = C.c_int32()
        call("scc_work_q_items", self.handle, None, None, 0, C.byref(k))
        cols = np.empty(k.value, np.int32); cnts = np.empty(k.value, np.int32)
        call("scc_work_q_items", self.handle, i32p(cols), i32p(cnts), k.value, C.byref(k))
        return cols, cnts

    def do_global_wcc(self) -> None:
        call("scc_do_global_wcc", self._g(), self.handle)

    def create_work_items_from_wcc(self) -> int:
        o = self._out(); call("scc_create_work_items_from_wcc", self._g(), self.handle, C.byref(o)); return o.value

    # -- driver ----------------------------------------------------------------------------------
    def run(self, method: int = METHOD_GLOBAL_WCC_FB, pivot_mode: int = PIVOT_DEGREE) -> dict:
        st = capi.RunStats()
        call("scc_run", self._g(), self.handle, method, pivot_mode, C.byref(st))
        return st.as_dict()

    def count_sccs(self) -> int:
        o = self._out(); call("scc_count_sccs", self.handle, C.byref(o)); return o.value

    def canonical_labels(self) -> np.ndarray:
        a = np.empty(self.n, np.int32)
        call("scc_canonical_labels", self.handle, i32p(a))
        return a

    def output_scc_list(self, path: str = "scc_list.txt") -> None:
        call("scc_output_scc_list", self.handle, path.encode())

    def histogram(self):
        k = C.c_int32()
        call("scc_histogram", self.handle, None, None, 0, C.byref(k))
        sz = np.empty(k.value, np.int32); ct = np.empty(k.value, np.int32)
        call("scc_histogram", self.handle, i32p(sz), i32p(ct), k.value, C.byref(k))
        return dict(zip(sz.tolist(), ct.tolist()))

    # -- updates (methods 5-11 of the reference) ------------------------------------------------
    def update_batch(self, ins_src=(), ins_dst=(), del_src=(), del_dst=()) -> dict:
        """Apply deletions then insertions to the graph and update the labels in place."""
        a, b = _i32(ins_src), _i32(ins_dst)
        c, d = _i32(del_src), _i32(del_dst)
        if a.shape != b.shape or c.shape != d.shape:
            raise ValueError("edge arrays differ in length")
        st = capi.UpdateStats()
        P = lambda x: x.ctypes.data_as(C.c_void_p) if x.size else None  # noqa: E731
        call("scc_update_batch", self._g(), self.handle, int(a.size), P(a), P(b), int(c.size), P(c), P(d), 0,
             C.byref(st))
        return st.as_dict()

    def incremental_insert(self, src, dst) -> dict:
        return self.update_batch(ins_src=src, ins_dst=dst)

    def decremental_delete(self, src, dst) -> dict:
        return self.update_batch(del_src=src, del_dst=dst)

    def insert_idea1(self, src, dst) -> dict:
        s, d = _i32(src), _i32(dst)
        st = capi.RunStats()
        call("scc_insert_idea1", self._g(), self.handle, int(s.size), i32p(s), i32p(d), C.byref(st))
        return st.as_dict()

    # -- learned pivot ---------------------------------------------------------------------------
    def set_pivot_model(self, model: "PivotModel | None") -> None:
        call("scc_state_set_pivot_model", self.handle, model.handle if model is not None else None)
        self._model = model            # keep the model alive while attached

    def pivot_log(self, capacity: int, per_round: int = 4096) -> None:
        """Record training samples in the following runs (capacity 0 stops and drops them)."""
        call("scc_state_pivot_log", self.handle, int(capacity), int(per_round))

    def pivot_records(self):
        """(x [k, 8] float32, t [k] float32, v [k] int32, class_size [k] int32) after a run."""
        k = C.c_int64()
        call("scc_state_pivot_records", self.handle, None, None, None, None, 0, C.byref(k))
        n = k.value
        x = np.empty((n, 8), np.float32); t = np.empty(n, np.float32)
        v = np.empty(n, np.int32); cs = np.empty(n, np.int32)
        if n:
            call("scc_state_pivot_records", self.handle, f32p(x), f32p(t), i32p(v), i32p(cs), n, C.byref(k))
        return x[:k.value], t[:k.value], v[:k.value], cs[:k.value]

    def free(self) -> None:
        if self._h is not None:
            capi.lib().scc_state_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


MLP_FEATURES = 8
MLP_PARAMS = 4801


class PivotModel:
    """The learned pivot proposer: 8 -> 64 -> 64 -> 1 ReLU network on the device
    (BF16 weights, FP32 accumulation), trained by the engine's own kernels."""

    def __init__(self, seed: int = 0, device: int = 0, handle=None):
        if handle is None:
            handle = C.c_void_p()
            call("scc_pivot_model_create", device, int(seed), C.byref(handle))
        self._h = handle

    @classmethod
    def load(cls, path: str, device: int = 0) -> "PivotModel":
        h = C.c_void_p()
        call("scc_pivot_model_load", device, path.encode(), C.byref(h))
        return cls(handle=h)

    @property
    def handle(self):
        if self._h is None:
            raise SccError(capi.SCC_ERR_STATE, "PivotModel", "model was freed")
        return self._h

    def save(self, path: str) -> None:
        call("scc_pivot_model_save", self.handle, path.encode())

    def params(self) -> np.ndarray:
        p = np.empty(MLP_PARAMS, np.float32)
        call("scc_pivot_model_get_params", self.handle, f32p(p))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(np.asarray(p, np.float32))
        assert p.size == MLP_PARAMS
        call("scc_pivot_model_set_params", self.handle, f32p(p))

    def forward(self, x, tensor_cores: bool = True) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1, MLP_FEATURES))
        y = np.empty(x.shape[0], np.float32)
        call("scc_pivot_model_forward", self.handle, f32p(x), x.shape[0], int(bool(tensor_cores)), f32p(y))
        return y

    def bench_inference(self, count: int, iters: int = 10) -> float:
        """Device ms of one tensor-core inference launch over `count` resident rows."""
        ms = C.c_double()
        call("scc_pivot_model_bench", self.handle, int(count), int(iters), C.byref(ms))
        return ms.value

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1, MLP_FEATURES))
        t = np.ascontiguousarray(np.asarray(t, np.float32))
        g = np.empty(MLP_PARAMS, np.float32)
        loss = C.c_float()
        call("scc_pivot_model_loss_grad", self.handle, f32p(x), f32p(t), x.shape[0], f32p(g), C.byref(loss))
        return float(loss.value), g

    def train(self, x, t, epochs: int = 20, batch: int = 1024, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1, MLP_FEATURES))
        t = np.ascontiguousarray(np.asarray(t, np.float32))
        losses = np.empty(max(epochs, 1), np.float32)
        call("scc_pivot_model_train", self.handle, f32p(x), f32p(t), x.shape[0], int(epochs), int(batch),
             float(lr), int(seed), f32p(losses))
        return losses[:epochs]

    def free(self) -> None:
        if self._h is not None:
            capi.lib().scc_pivot_model_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def collect_pivot_records(graph: Graph, capacity: int = 1 << 20, per_round: int = 4096,
                          method: int = METHOD_GLOBAL_WCC_FB):
    """One plain (degree-pivot) run of `graph` with logging on; returns its records (x, t)."""
    st = State(graph)
    try:
        st.pivot_log(capacity, per_round)
        st.reset()
        st.run(method, PIVOT_DEGREE)
        x, t, _, _ = st.pivot_records()
        return x, t
    finally:
        st.free()


class BatchPlan:
    """One persistent launch over a disjoint union of independent graphs (offsets
    give each graph's vertex range), captured once into a CUDA graph; run()
    replays it.  Results land in the state (canonical_labels etc.)."""

    def __init__(self, graph: Graph, state: "State", offsets, tuning: dict | None = None):
        self.graph, self.state = graph, state
        self.offsets = np.ascontiguousarray(offsets, np.int32)
        t = None
        if tuning is not None:
            t = capi.BatchTuning()
            call("scc_batch_default_tuning", C.byref(t))
            for k, v in tuning.items():
                setattr(t, k, int(v))
        h = C.c_void_p()
        call("scc_batch_plan_create", graph.handle, state.handle, i32p(self.offsets), int(self.offsets.size - 1),
             C.byref(t) if t is not None else None, C.byref(h))
        self._h = h

    def run(self) -> dict:
        st = capi.BatchStats()
        call("scc_batch_plan_run", self._h, C.byref(st))
        return st.as_dict()

    def free(self) -> None:
        if self._h is not None:
            call("scc_batch_plan_free", self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def batch_autotune(graph: Graph, state: "State", offsets):
    """Successive-halving search of the batched run's launch shape; (tuning dict, ms on the whole batch)."""
    offs = np.ascontiguousarray(offsets, np.int32)
    t = capi.BatchTuning()
    ms = C.c_double()
    call("scc_batch_autotune", graph.handle, state.handle, i32p(offs), int(offs.size - 1), C.byref(t), C.byref(ms))
    return t.as_dict(), ms.value


class Server:
    """Serving loop: device-resident graphs updated by streamed edge batches
    (continuous batching over worker slots, HBM-budget admission)."""

    def __init__(self, num_slots: int = 4, hbm_budget_bytes: int = 64 << 30, device: int = 0):
        h = C.c_void_p()
        call("scc_server_create", device, num_slots, hbm_budget_bytes, C.byref(h))
        self._h = h
        self.sizes = {}

    def add_graph(self, graph: Graph) -> int:
        """Takes ownership of the graph (the Python object is emptied) and decomposes it."""
        sid = C.c_int32()
        n = graph.num_nodes()
        call("scc_server_add_graph", self._h, graph.handle, C.byref(sid))
        graph._h = None
        self.sizes[sid.value] = n
        return sid.value

    def submit(self, session: int, ins_src=(), ins_dst=(), del_src=(), del_dst=()) -> int:
        """Queues a batch; returns its request id, or -1 when backpressure refused it
        (the queue is over its admission limit)."""
        a, b, c, d = _i32(ins_src), _i32(ins_dst), _i32(del_src), _i32(del_dst)
        rid = C.c_int64()
        rc = capi.lib().scc_server_submit(self._h, session, int(a.size), i32p(a), i32p(b), int(c.size), i32p(c),
                                          i32p(d), C.byref(rid))
        if rc == capi.SCC_ERR_BUSY:
            return -1
        if rc != 0:
            raise capi.SccError(rc, "scc_server_submit", capi.lib().scc_last_error().decode(errors="replace"))
        return rid.value

    def set_admission(self, max_queued_edges: int = 0, max_queue_ms: float = 0.0) -> None:
        """Backpressure: refuse submissions beyond a backlog of queued edges, drop
        requests older than max_queue_ms when a slot reaches them (0 = no limit)."""
        call("scc_server_set_admission", self._h, int(max_queued_edges), float(max_queue_ms))

    def wait(self, request_id: int) -> dict:
        r = capi.RequestResult()
        call("scc_server_wait", self._h, request_id, C.byref(r))
        out = {"status": r.status, "session": r.session, "latency_ms": r.latency_ms, "queue_ms": r.queue_ms}
        out.update(r.update.as_dict())
        return out

    def drain(self) -> None:
        call("scc_server_drain", self._h)

    def set_coalesce(self, max_requests: int, max_edges: int = 1 << 24) -> None:
        """Compose up to max_requests queued batches of a session into one update (1 = off)."""
        call("scc_server_set_coalesce", self._h, int(max_requests), int(max_edges))

    def stats(self) -> dict:
        s = capi.ServerStats()
        call("scc_server_get_stats", self._h, C.byref(s))
        return s.as_dict()

    def labels(self, session: int) -> np.ndarray:
        a = np.empty(self.sizes[session], np.int32)
        call("scc_server_labels", self._h, session, i32p(a))
        return a

    def session_csr(self, session: int):
        h = C.c_void_p()
        call("scc_server_session_graph", self._h, session, C.byref(h))
        g = Graph(h)
        try:
            return g.csr()
        finally:
            g._h = None       # borrowed

    def free(self) -> None:
        if self._h is not None:
            capi.lib().scc_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def condensation_graph(graph: Graph, labels, num_sccs: int, ins_src=(), ins_dst=()) -> Graph:
    """create_scc_edges + insert_idea2: the condensation over SCC ids plus inserted cross edges."""
    lab = _i32(labels)
    s, d = _i32(ins_src), _i32(ins_dst)
    h = C.c_void_p()
    call("scc_condensation_graph", graph.handle, i32p(lab), num_sccs, int(s.size), i32p(s) if s.size else None,
         i32p(d) if d.size else None, C.byref(h))
    return Graph(h)


def topological_levels(dag: Graph):
    """Method 7's BFS levels of a condensation DAG: (levels, max_level)."""
    n = dag.num_nodes()
    lev = np.empty(max(n, 1), np.int32)
    ml = C.c_int32()
    call("scc_topological_levels", dag.handle, i32p(lev), C.byref(ml))
    return lev[:n], ml.value


def affected_levels(dag: Graph, levels, max_level: int, labels, ins_src=(), ins_dst=()):
    """Method 7's affect_level: (coverage per level 0..max_level, unaffected level count)."""
    lev, lab = _i32(levels), _i32(labels)
    s, d = _i32(ins_src), _i32(ins_dst)
    out = np.empty(max_level + 1, np.int32)
    z = C.c_int32()
    call("scc_affected_levels", dag.handle, i32p(lev), max_level, int(lab.size), i32p(lab), int(s.size),
         i32p(s) if s.size else None, i32p(d) if d.size else None, i32p(out), C.byref(z))
    return out, z.value


def read_edge_list(path: str):
    """read_file: (src, dst) 0-based and N, the largest 1-based id."""
    m = C.c_int64()
    mx = C.c_int32()
    call("scc_read_edge_list", path.encode(), 0, None, None, C.byref(m), C.byref(mx))
    src = np.empty(max(m.value, 1), np.int32)
    dst = np.empty(max(m.value, 1), np.int32)
    if m.value:
        call("scc_read_edge_list", path.encode(), m.value, i32p(src), i32p(dst), C.byref(m), C.byref(mx))
    return src[:m.value], dst[:m.value], mx.value


def read_scc_list(path: str, n: int):
    a = np.empty(n, np.int32)
    k = C.c_int32()
    call("scc_read_scc_list", path.encode(), n, i32p(a), C.byref(k))
    return a, k.value


def decompose_csr(begin, node_idx, r_begin=None, r_node_idx=None, method: int = METHOD_GLOBAL_WCC_FB, device=0):
    """Host CSR in, canonical labels out (H2D + run + D2H in one call)."""
    b, a = _i32(begin), _i32(node_idx)
    rb = _i32(r_begin) if r_begin is not None else None
    ra = _i32(r_node_idx) if r_node_idx is not None else None
    n = b.size - 1
    labels = np.empty(n, np.int32)
    k = C.c_int32()
    st = capi.RunStats()
    call("scc_decompose_csr", n, int(a.size), i32p(b), i32p(a), i32p(rb), i32p(ra), method, device, i32p(labels),
         C.byref(k), C.byref(st))
    return labels, k.value, st.as_dict()


def device_count() -> int:
    c = C.c_int()
    call("scc_device_count", C.byref(c))
    return c.value
