"""B200-native strongly-connected-components engine.

A drop-in for the SCC path of ShashwaTTrigunayaT/DynamicGraphs_SCC: the
reference's phase API (trim1 / trim2 / FW-BW / WCC / colour / work queue /
driver) over device-resident int32 CSR, computed by hand-written sm_100a
kernels behind a C ABI (include/scc_capi.h).
"""
from .capi import SccError, lib  # noqa: F401
from .engine import (  # noqa: F401
    METHOD_BASELINE, METHOD_GLOBAL_FB, METHOD_GLOBAL_WCC_FB, PIVOT_DEGREE, PIVOT_LEARNED,
    BatchPlan, Graph, PivotModel, Server, State, batch_autotune, collect_pivot_records, condensation_graph, decompose_csr, device_count, gen_params, generate_batch_edges_host, generate_edges_host,
    read_edge_list, read_scc_list, topological_levels, affected_levels,
)

__version__ = "0.1.0"
