"""networkit_b200: NetworKit's PageRank path on NVIDIA B200 (sm_100a).

Drop-in for ``networkit.centrality.PageRank`` (plus the Graph container it
reads): ``from networkit_b200 import Graph, centrality`` then
``centrality.PageRank(G, 0.85, 1e-8).run().scores()``. The CUDA library
(``_lib/libnkgpu.so``, C ABI in include/nkgpu.h) does all the work.
"""
from . import centrality, graph
from .graph import Graph, InCSR, in_csr_from_edges

__version__ = "0.1.0"

__all__ = ["Graph", "InCSR", "in_csr_from_edges", "centrality", "graph"]
