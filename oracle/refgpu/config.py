"""The dataset the reference's own GPU programs run on (TEST INFRASTRUCTURE ONLY).

Their per-dataset sizes are compile-time macros (gpu_cuda/<DS>/dataset_config.cuh), so the
programs under oracle/_ref/ are built for exactly this seeded synthetic graph: 6,000 vertices,
120,000 temporal edges, reference chains of depth 3, generated in the reference-safe layout
(vertex 0 and the largest id receive no edge, the smallest timestamp is 0), which keeps clear of
the reference decoder's hazards with a first residual equal to 0, a successor equal to MAX_LABEL
and a timestamp base other than the minTimestamp macro; in that layout the encoder also never
writes a copy mask whose first copy block is empty (the reference's GPU decoder reads those lists
differently).
"""

NAME = "refgpu"
PARAMS = dict(n=6000, m=120_000, deg_exponent=2.1, repeat_frac=0.3, local_frac=0.6, local_radius=32, copy_frac=0.3,
              ts_kind=0, ts_span=1_000_000, seed=41, ref_safe=True)
N = 6000
# The BFS source compiled in (BFS_START_VERTEX): the vertex with the largest out-list of this graph.
BFS_SOURCE = 65
# The reference defaults kept for the other macros (gpu_cuda/shared/dataset_config_base.cuh):
# PAGERANK_ITERATIONS 10, HITS_ITERATIONS 10, CONNECTED_COMPONENTS_VERTEX_BEGIN 1,
# ACTIVE_VERTEX_BEGIN 0, MIN_GRAPH_VERTEX 0.
PR_ITERS = 10
HITS_ITERS = 10
CC_BEGIN = 1

# Programs built, and for each the device buffers whose contents are compared (found in the source
# by their allocation statement, `cudaMalloc((void**)&<name>, ...)`).
PROGRAMS = {
    "bfs": ["d_timeAndP"],
    "pagerank": ["Rank"],
    "hits": ["hub", "authority"],
    "connected_components": ["component"],
    "graph_coloring": ["d_vpl", "d_rand"],
    "neighbor_access": ["dv2"],
}
