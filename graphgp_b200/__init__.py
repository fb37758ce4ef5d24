"""graphgp_b200: GraphGP's graph build and Vecchia refinement on B200 GPUs.

The names below are the reference's public API (graphgp/__init__.py), on CUDA torch tensors; the C ABI is
declared in include/graphgp_b200.h and bound by ``graphgp_b200.graphgp_cuda``.
"""
from . import autograd, extras
from .api import (
    Graph,
    build_graph,
    build_tree,
    check_graph,
    compute_cov_matrix,
    compute_depths,
    generate,
    generate_and_logdet,
    generate_dense,
    generate_dense_inv,
    generate_dense_logdet,
    generate_inv,
    generate_logdet,
    generate_vjp,
    load_graph,
    order_by_depth,
    query_neighbors,
    query_preceding_neighbors,
    refine,
    refine_inv,
    refine_logdet,
    save_graph,
)

__all__ = [
    "build_tree", "query_preceding_neighbors", "query_neighbors", "Graph", "check_graph", "build_graph",
    "compute_depths", "order_by_depth", "generate", "generate_and_logdet", "generate_inv", "generate_logdet", "generate_dense",
    "generate_dense_inv", "generate_dense_logdet", "refine", "refine_inv", "refine_logdet", "compute_cov_matrix",
    "generate_vjp", "save_graph", "load_graph", "extras", "autograd",
]
