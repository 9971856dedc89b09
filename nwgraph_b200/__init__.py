"""nwgraph_b200 -- a B200-native (sm_100a) PageRank engine behind the call
surface of NWGraph's ``nw::graph::page_rank``.

* ``page_rank`` / ``Graph``     -- the drop-in solve (pagerank.py)
* ``graphs``                    -- seeded RMAT / grid inputs (adjacency<1> CSR)
* ``build``                     -- in-tree build of libnwgpu.so / libnwgen.so

The CUDA library (``libnwgpu.so``, C ABI in ``include/nwgpu.h``) is loaded on
first use; there is no CPU fallback.
"""
from ._native import NwgpuError
from .pagerank import Graph, GraphBatch, PageRankStats, PprBatchStats, RaggedStats, page_rank

__all__ = ["Graph", "GraphBatch", "PageRankStats", "PprBatchStats", "RaggedStats", "NwgpuError", "page_rank"]
