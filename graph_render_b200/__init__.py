"""graph_render_b200: a B200 (sm_100a) ForceAtlas2 / Barnes-Hut layout engine.

A drop-in for graph-core's ``layout.forceatlas2.barnes_hut`` registry row,
registered as ``layout.forceatlas2.barnes_hut.cuda``. The compute path is the
CUDA library ``libgraph_cuda.so`` behind the C ABI in ``include/graph_cuda.h``;
this package is its host-side face (registry mirror, parameter schema,
per-tick handle) and the workload generators.
"""

from .registry import (D3_ID, FA2_ID, PM_ID, Capability, Geometry, ParamSpec, ParamsError, ParamsView, StageError,
                       Topology, find, layouts)
from .fa2 import Fa2, layout, params_bytes, run_values
from .d3force import ForceParams, ForceSession

__all__ = [
    "D3_ID", "FA2_ID", "PM_ID", "ForceParams", "ForceSession", "Capability", "Geometry", "ParamSpec", "ParamsError", "ParamsView", "StageError",
    "Topology", "find", "layouts", "Fa2", "layout", "params_bytes", "run_values",
]
