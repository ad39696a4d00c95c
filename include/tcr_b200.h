/*
 * tcr_b200.h -- C ABI of the B200 (sm_100a) compact-hashing neighbour search.
 *
 * Plain pointers and sizes only: every array argument is a device pointer unless stated
 * otherwise, every `stream` is a cudaStream_t passed as void*, and every function returns
 * TCR_OK (0) or a negative TCR_ERR_* code with a message in tcr_last_error().  Nothing here
 * allocates device memory: callers pass buffers of the sizes tcr_search_sizes() reports.
 *
 * The reference (wi-re/torchCompactRadius) exposes this path as torch operators registered in
 * src/torchCompactRadius/cppSrc/cppWrapper.cpp:38-59 and driven from Python by
 * compactHashing/cppSearch.py:12-98 (searchNeighbors_cpp) and :179-244 (neighborSearch_cpp).
 * Each entry point below names the reference interface it replaces.
 */
#ifndef TCR_B200_H
#define TCR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCR_ABI_VERSION 10

#define TCR_OK 0
#define TCR_ERR_INVALID (-1) /* bad argument or workspace too small */
#define TCR_ERR_CUDA (-2)    /* a CUDA call failed */

/* Support modes (reference cppSrc/common.h:68-70 enum supportMode; thresholds
 * neighborhoodDynamic.h:63-69): gather h_i, scatter h_j, symmetric (h_i+h_j)/2,
 * superSymmetric max(h_i, h_j). */
#define TCR_GATHER 0
#define TCR_SCATTER 1
#define TCR_SYMMETRIC 2
#define TCR_SUPERSYMMETRIC 3

/* One search.  Positions are row-major float32 [n, dim]; supports float32 [n].  The domain
 * (DomainDescription, reference util.py:280-292) is given by value on the host. */
typedef struct tcr_search_desc {
    int32_t dim;             /* 1, 2 or 3 */
    int32_t mode;            /* TCR_GATHER .. TCR_SUPERSYMMETRIC */
    int32_t periodic_mask;   /* bit d set: dimension d is periodic */
    int32_t self_search;     /* 1: the query cloud is the reference cloud (same positions) */
    float domain_min[3];
    float domain_max[3];
    int64_t hash_map_length; /* the reference's hashMapLength; selects hash buckets exactly as
                                cppSrc/neighborhood.h:73-96 does */
    int64_t n_query;
    int64_t n_ref;
    const float* query_pos;  /* device [n_query*dim] */
    const float* query_sup;  /* device [n_query]; may be NULL for TCR_SCATTER */
    const float* ref_pos;    /* device [n_ref*dim] */
    const float* ref_sup;    /* device [n_ref]; may be NULL for TCR_GATHER */
    /* Optional extensions (all zero / NULL: the reference's compact search). */
    const int32_t* query_ids; /* device [n_query]: row index written for local query q (subset searches) */
    const int32_t* ref_ids;   /* device [n_ref]: column index written for local reference j */
    float hcell[3];           /* > 0: per-dimension cell sizes to use instead of the reference's compute_h */
    int32_t clamped_grid;     /* 1: exact grid semantics for caller-chosen cells (multi-level search):
                                 cell coordinates clamped into [0, count), stencil cells outside the grid
                                 skipped, wrapped stencil cells on periodic dims with < 3 cells visited
                                 once (the reference visits them twice and reports those pairs twice) */
    /* Tuning of this search (no reference counterpart; 0 keeps the default; no setting changes a
     * result): queries per work unit of the walks -- 32, 16 or 8 -- and resident walk blocks per
     * SM (1..64).  tcr_count and tcr_emit of one search must be given the same unit_queries. */
    int32_t unit_queries;
    int32_t walk_blocks_per_sm;
    int32_t reserved;
} tcr_search_desc;

/* One cloud of a batch: an independent search with its own domain, periodicity, supports and
 * hashMapLength (the fields mean what they mean in tcr_search_desc). */
typedef struct tcr_cloud_desc {
    int32_t dim;             /* 1, 2 or 3 */
    int32_t periodic_mask;   /* bit d set: dimension d is periodic */
    float domain_min[3];
    float domain_max[3];
    int64_t hash_map_length;
    int64_t n_query;
    int64_t n_ref;
    const float* query_pos;  /* device [n_query*dim] */
    const float* query_sup;  /* device [n_query] or NULL (TCR_SCATTER) */
    const float* ref_pos;    /* device [n_ref*dim] */
    const float* ref_sup;    /* device [n_ref] or NULL (TCR_GATHER) */
    float hcell[3];          /* > 0: caller-chosen cell sizes (as tcr_search_desc.hcell) */
    int32_t clamped_grid;    /* 1: exact grid semantics for caller-chosen cells (as tcr_search_desc) */
    int32_t reserved;
} tcr_cloud_desc;

/* A batch of independent searches run by one set of launches (the many scenes or timesteps of a
 * simulation sweep; the reference runs them one call at a time, or through its batched
 * radius(), neighborhood.py:313-363, which searches each batch id on its own).  Clouds never see
 * each other.  Points are numbered globally in table order: query q of cloud k has the global
 * index (n_query of clouds 0..k-1) + q, and likewise for reference points.  Offsets, counts and
 * indptr span all clouds' queries in global order; with local_index = 0 the written rows and
 * columns are global indices, with local_index = 1 they are indices within the cloud (query_ids /
 * ref_ids, when given, map global indices and take precedence). */
typedef struct tcr_batch_desc {
    int32_t n_clouds;        /* >= 1 */
    int32_t mode;            /* TCR_GATHER .. TCR_SUPERSYMMETRIC, for every cloud */
    int32_t self_search;     /* 1: every cloud's query set is its reference set */
    int32_t local_index;     /* 1: rows and columns numbered within each cloud */
    const tcr_cloud_desc* clouds;  /* HOST array [n_clouds] */
    const int32_t* query_ids;      /* device [total queries] or NULL */
    const int32_t* ref_ids;        /* device [total references] or NULL */
    /* Incremental re-sort (optional).  ref_lin_hint (device int32 [total references]): the
     * reference points are given in the cell order of an earlier build of the same grid, and
     * ref_lin_hint[i] is the linear cell point i had there; the build then sorts only the points
     * that changed cell and merges them into the rest.  The result is the one of a full build for
     * any hint (a hint that does not hold makes the build fall back to the full sort on the device).
     * ref_lin_out (device int32 [total references]): receives the linear cell of every point in
     * the new cell order (reference slot k of cloud c is the cloud's k-th point in cell order), the
     * hint of the next build once the caller has put its points in that order. */
    const int32_t* ref_lin_hint;
    int32_t* ref_lin_out;
    /* Optional (device int32 [total references]): the global input index of every reference point
     * in the new cell order -- the permutation that puts a cloud's points in that order. */
    int32_t* ref_order_out;
    /* Tuning of this batch, as in tcr_search_desc (0: the defaults). */
    int32_t unit_queries;
    int32_t walk_blocks_per_sm;
} tcr_batch_desc;

/* Message of the last failing call on this thread. */
const char* tcr_last_error(void);

/* TCR_ABI_VERSION of the loaded library. */
int tcr_version(void);

/* sizeof(tcr_search_desc), sizeof(tcr_cloud_desc) and sizeof(tcr_batch_desc) as compiled into
 * the library, for FFI layout checks. */
int64_t tcr_desc_bytes(void);
int64_t tcr_cloud_desc_bytes(void);
int64_t tcr_batch_desc_bytes(void);

/* Total number of CUDA kernels this library has launched in this process (launch accounting
 * for benchmarks; no reference counterpart). */
int64_t tcr_kernel_launches(void);

/* Per-launch timing of the heaviest kernels, for benchmarks (no reference counterpart).  While
 * enabled, tcr_count / tcr_batch_count record a pair of CUDA events around the count walk launch
 * and tcr_emit / tcr_batch_emit around the record expansion, on the launching stream, for calls
 * on the device that was current at tcr_profile_kernels(1).  tcr_profile_kernel_ms waits for the
 * last such launch and returns its duration in milliseconds. */
#define TCR_PROFILE_COUNT_WALK 0
#define TCR_PROFILE_EXPAND 1
int tcr_profile_kernels(int32_t enable);
int tcr_profile_kernel_ms(int32_t kernel, float* ms);

/* Byte sizes of the persistent structure (reference-side cell table and hash map, kept for
 * reuse like the reference's CompactHashMap, compactHashing/datastructure.py:8-31) and of the
 * per-search scratch.  Host-only; no device work. */
int tcr_search_sizes(int64_t n_query, int64_t n_ref, int32_t dim, int64_t* structure_bytes,
                     int64_t* scratch_bytes);

/* Layout of the structure buffer, so a caller can view its parts (the fields of the reference's
 * CompactHashMap, datastructure.py:8-31, are derived from them).  Host-only.  offsets[k] is the
 * byte offset of field k (TCR_STRUCT_*), except offsets[TCR_STRUCT_MAP_CAPACITY], which is the
 * number of 64-bit slots of the linear-index map.  Field contents:
 *   GRID          float hmax, float hCell, float hcell_d[3], int32 cellCount[3], int32 exact_only, ...
 *   NUM_CELLS     int32 number of occupied cells C
 *   SORTED_POINTS float4 [n_ref] wrapped reference positions in cell order, .w = support
 *   SORT_INDEX    int32 [n_ref] original index of each sorted point
 *   CELL_START    int32 [C+1] first sorted point of each cell (cells in linear-index order)
 *   CELL_LIN      int32 [C] linear cell index (cellTable.py:31)
 *   CELL_COORDS   int32 [3*C] integer cell coordinates
 *   CELL_BUCKET   int32 [C] reference hash of the coordinates mod hashMapLength
 *   MAP           uint64 [cap] open-addressing map (lin << 32 | cell), empty = ~0 */
#define TCR_STRUCT_GRID 0
#define TCR_STRUCT_NUM_CELLS 1
#define TCR_STRUCT_SORTED_POINTS 2
#define TCR_STRUCT_SORT_INDEX 3
#define TCR_STRUCT_CELL_START 4
#define TCR_STRUCT_CELL_LIN 5
#define TCR_STRUCT_CELL_COORDS 6
#define TCR_STRUCT_CELL_BUCKET 7
#define TCR_STRUCT_MAP 8
#define TCR_STRUCT_MAP_CAPACITY 9
#define TCR_STRUCT_NFIELDS 10
int tcr_structure_offsets(int64_t n_ref, int64_t* offsets, int32_t n);

/* Builds the search structure over the reference cloud: grid support (cellTable.py:40-81),
 * cell size (util.py:28-79 compute_h), periodic wraps, sort by linear cell index, cell table
 * and hash map.  Replaces buildCompactHashMap_compat (compactHashing/hashTable.py:159-234)
 * together with the computeHashIndices operator (cppSrc/hashing.h:37-39, cppWrapper.cpp:45).
 * The query supports of `d` enter the grid support for gather/symmetric modes, as in the
 * reference. */
int tcr_build_structure(const tcr_search_desc* d, void* structure, int64_t structure_bytes, void* scratch,
                        int64_t scratch_bytes, void* stream);

/* Counts the neighbours of every query and scans them.  Replaces the countNeighbors operator
 * (cppSrc/neighborhood.h:140-146, cppWrapper.cpp:39) plus the cumsum of cppSearch.py:81-84.
 * Every (query, candidate) pair is tested once here: each work unit (<= 32 queries of one cell)
 * writes a record of its candidate runs and of one 32-bit hit mask per (query, 32 candidates) to
 * `stage` (device int32, stage_capacity words) for tcr_emit to expand into place.  Units that do
 * not fit (or every unit when stage is NULL / capacity 0) are tested again by tcr_emit.
 * offsets: device int64 [n_query+1] (exclusive scan, offsets[n_query] = total pairs).
 * indptr_out (device int32 [n_query+1]) and row_entries_out (device int64 [n_query]) are the
 * SparseCSR fields of util.py:321-358 and may be NULL.  info_out (host, 8 x int64, may be NULL)
 * receives, asynchronously on `stream`: {total pairs, clouds without a valid grid, queries walked serially,
 * exact-only mode, staging words the units asked for, units left for tcr_emit to re-test, chunks
 * (32 candidates of a unit) tested again with exact decisions because a pair lay within the fast
 * test's rounding band, and
 * for a batch built with a linear-cell hint the points its incremental re-sort sorted (-1: it fell
 * back to the full sort; -2: no hint)};
 * a caller sizes the next search's staging list from entry 4. */
int tcr_count(const tcr_search_desc* d, const void* structure, void* scratch, int64_t scratch_bytes, int32_t* stage,
              int64_t stage_capacity, int64_t* offsets, int32_t* indptr_out, int64_t* row_entries_out,
              int64_t* info_out, void* stream);

/* Writes the neighbour pairs at the offsets of tcr_count (same scratch, stage and descriptor).
 * Replaces the buildNeighborList operator (cppSrc/neighborhood.h:155-162, cppWrapper.cpp:40)
 * and the j = sortIndex[j] unsort of cppSearch.py:97: col_out receives original reference
 * indices, row_out (NULL for CSR) original query indices, int64 [out_capacity] each.  It may be
 * enqueued right after tcr_count without waiting for the total: pairs at positions >=
 * out_capacity are dropped, so a caller that guessed too small a buffer reads the total from
 * tcr_count's info and calls tcr_emit again with a large enough one. */
int tcr_emit(const tcr_search_desc* d, const void* structure, void* scratch, int64_t scratch_bytes,
             const int32_t* stage, const int64_t* offsets, int64_t* row_out, int64_t* col_out, int64_t out_capacity,
             void* stream);

/* The batched counterparts of tcr_search_sizes / tcr_build_structure / tcr_count / tcr_emit:
 * the same phases over every cloud of `b` at once, with the same buffer contracts (offsets,
 * indptr and row entries over all clouds' queries, pairs of all clouds in one output).  All four
 * calls of one search take descriptors with the same clouds in the same order.  A cloud with
 * points on both sides and no valid cell grid finds no pairs; info entry 1 counts such clouds and
 * entry 3 the clouds decided by the exact test alone.  No reference counterpart beyond the
 * per-cloud operators named above. */
int tcr_batch_sizes(const tcr_batch_desc* b, int64_t* structure_bytes, int64_t* scratch_bytes);
int tcr_batch_build_structure(const tcr_batch_desc* b, void* structure, int64_t structure_bytes, void* scratch,
                              int64_t scratch_bytes, void* stream);
int tcr_batch_count(const tcr_batch_desc* b, const void* structure, void* scratch, int64_t scratch_bytes,
                    int32_t* stage, int64_t stage_capacity, int64_t* offsets, int32_t* indptr_out,
                    int64_t* row_entries_out, int64_t* info_out, void* stream);
int tcr_batch_emit(const tcr_batch_desc* b, const void* structure, void* scratch, int64_t scratch_bytes,
                   const int32_t* stage, const int64_t* offsets, int64_t* row_out, int64_t* col_out,
                   int64_t out_capacity, void* stream);

/* One whole search -- tcr_build_structure, tcr_count and tcr_emit -- that allocates nothing.
 * No counterpart in the reference: it exists for callers that cannot allocate device memory at
 * search time (a host that gives the search a fixed arena at start-up and forbids cudaMalloc
 * afterwards, e.g. because cudaMalloc can synchronise the device inside a real-time loop, or a
 * plugin host whose allocator the search cannot reach).  The structure and scratch live in a
 * 32 MiB file-scope device array that every GPU loading this library holds until exit.  A search
 * fits when its structure plus scratch bytes (tcr_search_sizes) do not exceed the array; larger
 * searches are rejected with TCR_ERR_INVALID before any device work, naming the bytes they need.
 * What is left of the array after structure and scratch is the staging list of tcr_count (units
 * whose records do not fit it are tested again by the emit).
 * The caller passes its inputs in `d` and its outputs: offsets (device int64 [n_query+1]),
 * optional indptr_out / row_entries_out as in tcr_count, row_out (NULL for CSR) and col_out of
 * pair_capacity entries.  The call synchronises `stream` once to learn the pair count
 * (*total_out); if it exceeds pair_capacity nothing is emitted and TCR_ERR_INVALID is returned,
 * so the caller can retry with a larger output.
 * The call synchronises `stream` (between the count and the emit), so it can never run inside a
 * stream capture or a CUDA graph; callers that need graphs use tcr_build_structure / tcr_count /
 * tcr_emit with their own buffers.  All calls share the one array: calls whose work overlaps on
 * the GPU (other streams, other host threads) race and must be serialised by the caller. */
int tcr_search_noalloc(const tcr_search_desc* d, int64_t* offsets, int32_t* indptr_out, int64_t* row_entries_out,
                       int64_t* row_out, int64_t* col_out, int64_t pair_capacity, int64_t* total_out, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Float64 inputs.  The reference's operators dispatch on float and double
 * (cppSrc/neighborhoodDynamic_cpu.cpp:504,531); for double positions it computes cell indices,
 * moduloOp, the squared sum, sqrt and the threshold in double.  These two calls replace tcr_count /
 * tcr_emit for such inputs.  The structure is built by tcr_build_structure from float32 copies of
 * the wrapped positions and supports, with hcell set to a cell size no smaller than the reference's
 * double hCell (so every pair within the double support lies in a query's 3^d stencil); the walks
 * test candidates on the float32 copies and decide every pair whose float32 test lies within the
 * copies' rounding of the threshold on the double arrays below, by the reference's double
 * expression.
 * ------------------------------------------------------------------------------------------- */
typedef struct tcr_f64_inputs {
    const double* query_pos;  /* device [n_query*dim], wrapped as the reference wraps queries
                                 (util.py:375-387) */
    const double* query_sup;  /* device [n_query]; may be NULL for TCR_SCATTER */
    const double* ref_pos;    /* device [n_ref*dim], wrapped as the reference wraps references
                                 (util.py:375-387, then compactHashing/cppSearch.py:221) */
    const double* ref_sup;    /* device [n_ref]; may be NULL for TCR_GATHER */
    double* ref_sorted;       /* device workspace [n_ref*4] (32-byte aligned): tcr_count_f64 writes the
                                 references in cell order there, tcr_emit_f64 reads them */
    double domain_min[3];     /* the domain in double: periodic differences use max - min */
    double domain_max[3];
} tcr_f64_inputs;

/* countNeighbors at scalar_t = double (neighborhoodDynamic.h:37-74) + the offsets scan; d describes
 * the float32 copies the structure was built from (hcell > 0, clamped_grid 0).  stage and the other
 * arguments as in tcr_count. */
int tcr_count_f64(const tcr_search_desc* d, const tcr_f64_inputs* in, const void* structure, void* scratch,
                  int64_t scratch_bytes, int32_t* stage, int64_t stage_capacity, int64_t* offsets,
                  int32_t* indptr_out, int64_t* row_entries_out, int64_t* info_out, void* stream);

/* buildNeighborList at scalar_t = double (neighborhoodDynamic.h:76-115): writes each query's pairs
 * from offsets[q] in stencil order (same stage as tcr_count_f64; the other arguments as in
 * tcr_emit). */
int tcr_emit_f64(const tcr_search_desc* d, const tcr_f64_inputs* in, const void* structure, void* scratch,
                 int64_t scratch_bytes, const int32_t* stage, const int64_t* offsets, int64_t* row_out,
                 int64_t* col_out, int64_t out_capacity, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Reductions of values onto an index: the reference's scatter operators scatter_sum, scatter_mul,
 * scatter_mean, scatter_min and scatter_max (src/torchCompactRadius/cppSrc/sparseOperations/
 * scatter.h:10-36, registered in cppSrc/cppWrapper.cpp:54-58; forward scatter_cpu.cpp:7-85 and
 * scatter_cuda.cu:52-128).  src is viewed as [B][E][K] (E along the scattered dimension), out and
 * arg_out as [B][N][K].  Every output element is reduced in increasing e, one element after the
 * other in the element type's own arithmetic, exactly as the reference's CPU loop does: the sums
 * and products are bit-identical to it (its CUDA kernel adds with atomics in an arbitrary order),
 * and min/max keep the first of equal values as the reference's CPU loop does.
 * ------------------------------------------------------------------------------------------- */
#define TCR_REDUCE_SUM 0
#define TCR_REDUCE_MEAN 1
#define TCR_REDUCE_MUL 2
#define TCR_REDUCE_MIN 3
#define TCR_REDUCE_MAX 4

/* Element types of src and out (AT_DISPATCH_ALL_TYPES_AND2(Half, BFloat16) in the reference). */
#define TCR_DTYPE_U8 0
#define TCR_DTYPE_I8 1
#define TCR_DTYPE_I16 2
#define TCR_DTYPE_I32 3
#define TCR_DTYPE_I64 4
#define TCR_DTYPE_F16 5
#define TCR_DTYPE_BF16 6
#define TCR_DTYPE_F32 7
#define TCR_DTYPE_F64 8

typedef struct tcr_scatter_desc {
    int32_t reduce;        /* TCR_REDUCE_* */
    int32_t dtype;         /* TCR_DTYPE_* of src and out */
    int32_t index_full;    /* 0: index[E], the same for every b and k (an index broadcast along the
                              scattered dimension); 1: index[B][E][K] */
    int32_t index_sorted;  /* index_full == 0: 1 when index is non-decreasing (stats[2] == 0 from
                              tcr_index_stats); such an index needs no sort */
    int32_t accumulate;    /* 1: out holds the starting values (the reference's optional_out);
                              0: out is overwritten (0 where no element lands) */
    int32_t reserved;
    int64_t B, E, K, N;
    const void* src;       /* device [B*E*K], contiguous */
    const int64_t* index;  /* device [E] or [B*E*K] */
    void* out;             /* device [B*N*K] */
    int64_t* arg_out;      /* TCR_REDUCE_MIN / MAX: device [B*N*K], the e of the kept value or E when
                              none (the reference's arg_out); otherwise NULL */
} tcr_scatter_desc;

/* sizeof(tcr_scatter_desc) as compiled into the library, for FFI layout checks. */
int64_t tcr_scatter_desc_bytes(void);

/* stats[0] = min, stats[1] = max (INT64_MAX / INT64_MIN for n == 0) and stats[2] = the number of
 * positions i > 0 with index[i] < index[i - 1], over the n values of index.  stats is 3 int64 of
 * device memory; when stats_host is not NULL (pinned host memory) they are also copied there, in
 * stream order.  Replaces the host side of the reference's sizing (`index.max()`,
 * scatter_cpu.cpp:29-35) and tells whether the index needs sorting. */
int tcr_index_stats(const int64_t* index, int64_t n, int64_t* stats, int64_t* stats_host, void* stream);

/* Scratch bytes tcr_scatter needs for this description. */
int tcr_scatter_sizes(const tcr_scatter_desc* d, int64_t* scratch_bytes);

/* One reduction (the reference's scatter_fw, scatterWrapper.cpp:29-42, with the reduce of
 * Reducer<>::update, reducer.h:44-66).  TCR_REDUCE_MEAN divides by the count of elements that
 * landed, counted in the element type, below 1 taken as 1 (true division for floating types,
 * floor division for integers), as the reference's scatter_mean does (scatterWrapper.cpp:121-146).
 * Without accumulate, MIN / MAX outputs still at the type's max / lowest become 0.  With E == 0
 * (no elements) and no accumulate, out becomes 0 and arg_out E, for every reduce.
 * The index is checked on the device while it is read: when some value lies outside [0, N), or
 * index_sorted is 1 and the index descends somewhere, nothing is written (out and arg_out keep
 * their contents).  stats_host (pinned host memory, 3 int64, may be NULL) receives the index's
 * min, max and (with index_sorted = 1) number of descents, in stream order, so that a caller who
 * guessed "sorted" learns whether the call ran and otherwise calls again with index_sorted = 0
 * (the reference writes outside out for such indices). */
int tcr_scatter(const tcr_scatter_desc* d, void* scratch, int64_t scratch_bytes, int64_t* stats_host, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TCR_B200_H */
