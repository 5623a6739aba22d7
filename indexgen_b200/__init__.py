"""indexgen_b200 -- B200-native conflict-graph + greedy codebook path of IndexGen.

The compute lives in libindexgen_cuda.so (hand-written CUDA for sm_100a behind
the C ABI of include/indexgen_cuda.h); this package is the Python host mirror
of the reference's GPU path (src/cuda_edit_distance.py, src/gpu_graph_generator.py,
SolveIndependentSet / VerifyDist of src/SparseMat.cpp, src/Utils.cpp, and the
nearest-centre assignment of src/gpu_cluster.py).
"""
from .graph import (  # noqa: F401
    ConflictGraph,
    Context,
    FAULT_DEVICE_ALLOC,
    FAULT_NONE,
    FAULT_TILE_COPY,
    IndexGenError,
    LANES_BYTE,
    LANES_FULL,
    LANES_NIBBLE,
    LISTS_AUTO,
    LISTS_PACKED,
    LISTS_PLAIN,
    Server,
    apply_filters,
    assign_centers,
    build_batch,
    build_conflict_graph,
    cluster_centres,
    cluster_solve,
    codebook_from_adjacency,
    codebook_from_upper_csr,
    count_conflicts,
    default_context,
    fill_adj_list_gpu,
    greedy_stats,
    lane_form,
    pack_sequences,
    random_cluster_fit,
    read_adj_list,
    set_greedy_threads,
    solve,
    solve_batch,
    solve_assignments_cuda,
    solve_edit_distance_cuda,
    solve_independent_set,
    verify_dist,
)

__version__ = "0.1.0"
