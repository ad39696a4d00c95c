// tcr_search.cu -- compact-hashing fixed-radius neighbour search for sm_100a, with a C ABI.
//
// One engine serves a single search and a batch of independent clouds (the scenes or timesteps
// of a simulation sweep, of uneven sizes, each with its own domain, periodicity, supports and
// hashMapLength); a single search is a batch of one cloud.  Every phase is one set of launches
// over all clouds, on one CUDA stream, with no host synchronisation inside a phase:
//   build:  per-cloud support max-reductions -> per-cloud grid parameters (compute_h) -> wrap and
//           pack reference points into float4 (x, y, z, h) with (cloud, linear cell) sort keys ->
//           stable radix sort -> run-length cell table (begin, coords, bucket, cloud) and one
//           open-addressing lin -> cell map region per cloud.
//   count:  query packing (a self search reuses the reference order) -> query groups (cells) ->
//           work units of <= 32 queries of one group -> warp-per-unit candidate walk that tests
//           every (query, candidate) pair once, counts, and stages per-unit hit records -> scan.
//   emit:   expansion of the staged records into CSR/COO slots; units that were not staged are
//           walked again.
// The candidate set of every query is the reference's (cppSrc/neighborhood.h:73-132): the
// stencil cells of its own cell, found by linear index inside the bucket of the stencil cell's
// hash; the pair test is the reference's float test (tcr_common.cuh).  Clouds never see each
// other: keys, cells, map regions and work units all carry the cloud.
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <cstddef>
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <vector>

#include "tcr_common.cuh"
#include "tcr_scan.cuh"
#include "tcr_sort.cuh"
#include "../../include/tcr_b200.h"

namespace tcr {

// ------------------------------------------------------------------------------------------
// error reporting (set_error / g_err: tcr_common.cuh)
#define TCR_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return set_error(TCR_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------------------------------
// workspace layout
static inline int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }
static inline int64_t next_pow2(int64_t x) {
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
// Map slots of a cloud with n reference points: a power of two >= 2n (load factor <= 1/2).
static inline int64_t hash_capacity(int64_t n_ref, int64_t min_cap) {
    return std::max<int64_t>(min_cap, next_pow2(2 * std::max<int64_t>(n_ref, 1)));
}
constexpr int64_t kSingleMapMin = 1024;  // one search
constexpr int64_t kBatchMapMin = 64;     // per cloud of a batch
// Work counters: [0] count walk, [1] emit walk, [2 + cls] / [8 + cls] the count / emit walk of
// one cloud class (cls = dim * 2 + periodic, 2..7) in a batch that mixes classes, [16 + the same]
// for the count walk of the units recorded window by window.
constexpr int kWorkCounters = 32;

// Default tuning of a search (tcr_search_desc / tcr_batch_desc unit_queries and walk_blocks_per_sm):
// queries per work unit and resident walk blocks per SM.  Neither changes a result: a query's
// candidates and their order do not depend on how queries are grouped into units.
constexpr int kDefaultUnitQueries = 32;
constexpr int kDefaultWalkBlocksPerSM = 12;

struct Carve {
    char* base;
    int64_t off;
    template <typename T>
    T* take(int64_t count) {
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += align256(count * (int64_t)sizeof(T));
        return p;
    }
};

// Persistent structure (reference side); kept alive for reuse.
struct Structure {
    GridParams* grid;         // [C] per cloud
    int32_t* num_cells;       // [1]
    int32_t* bad_grids;       // [1] clouds with points on both sides and no valid grid
    float4* rsorted;          // [nr] wrapped reference points in (cloud, cell) order, .w = support
    int32_t* rsidx;           // [nr] global index of each sorted point
    int32_t* cell_start;      // [nr+1]
    int32_t* cell_lin;        // [nr]
    int32_t* cell_coords;     // [3*nr]
    int32_t* cell_bucket;     // [nr] reference hash of the cell's coordinates mod hashMapLength
    int32_t* cell_cloud;      // [nr]
    unsigned long long* map;  // [map_total] per-cloud regions of (lin << 32 | cell), empty = ~0
    int64_t map_total;
};

static Structure carve_structure(void* buf, int64_t nr, int64_t C, int64_t map_total, int64_t* bytes) {
    Carve c{(char*)buf, 0};
    Structure s;
    s.grid = c.take<GridParams>(C);
    s.num_cells = c.take<int32_t>(1);
    s.bad_grids = c.take<int32_t>(1);
    s.rsorted = c.take<float4>(nr);
    s.rsidx = c.take<int32_t>(nr);
    s.cell_start = c.take<int32_t>(nr + 1);
    s.cell_lin = c.take<int32_t>(nr);
    s.cell_coords = c.take<int32_t>(3 * nr);
    s.cell_bucket = c.take<int32_t>(nr);
    s.cell_cloud = c.take<int32_t>(nr);
    s.map_total = map_total;
    s.map = c.take<unsigned long long>(map_total);
    if (bytes) *bytes = c.off;
    return s;
}

// Per-search scratch.
struct Scratch {
    CloudParams* table;     // [C] this search's cloud table
    int32_t* query_prefix;  // [C+1] global index of each cloud's first query (last: total)
    int32_t* ref_prefix;    // [C+1] the same for reference points
    QueryParams* qparams;   // [C]
    void* sort_state;       // SortState32 or SortState64
    int32_t* num_qgroups;   // [1]
    int32_t* num_units;     // [1]
    int32_t* num_stray;     // [1]
    int32_t* work;          // [kWorkCounters] work distribution counters
    int64_t* total;         // [1]
    int64_t* info;          // [8] see tcr_count
    int32_t* num_flagged;   // [1]
    int32_t* exact_clouds;  // [1] clouds whose every pair takes the exact test
    int32_t* num_exact;     // [1] units the count walk re-tested with exact decisions
    int32_t* unit_cap;      // [1] queries per work unit of this search (set by the count phase)
    unsigned long long* cursor;  // [1] staging fill
    float4* pack;           // [max(nq,nr)] packed input points before sorting
    void* keys[2];          // [max(nq,nr)] 64-bit slots (32-bit keys use the first half)
    int32_t* vals[2];
    int32_t* hist;
    int32_t* tile_sums;
    int64_t* scan_tiles64;  // [scan_tiles(max)]
    int32_t* scan_tiles32;  // [scan_tiles(max)]
    float4* qsorted;        // [nq]
    int32_t* qsidx;         // [nq] global query index of each sorted query
    int32_t* qgroup_start;  // [nq+1]
    int32_t* qgroup_coords; // [3*nq]
    int32_t* qgroup_cloud;  // [nq]
    int32_t* unit_group;    // [nq]
    int32_t* unit_t0;       // [nq]
    int32_t* counts;        // [nq] global query order
    int32_t* stray;         // [nq]
    int32_t* rec;           // [nq] per unit: offset of its record in the staging list (-1: not staged)
    int32_t* flagged;       // [nq] units re-walked by the emit pass
    // incremental re-sort (builds given the previous cell of every reference point), else null
    int32_t* stay;          // [nr] 1: the point is still in its previous cell
    void* stay_keys;        // [nr] keys of the unmoved points, input order (sorted when the hint holds)
    int32_t* stay_idx;      // [nr]
    void* moved_keys[2];    // [nr] keys of the moved points (sorted in place)
    int32_t* moved_vals[2]; // [nr]
    void* moved_state;      // SortState of the moved points' sort
    int32_t* inc_count;     // [2] unmoved points, hint broken (1: fall back to the full sort)
};

static Scratch carve_scratch(void* buf, int64_t nq, int64_t nr, int64_t C, bool incremental, int64_t* bytes) {
    Carve c{(char*)buf, 0};
    Scratch s;
    const int64_t nmax = std::max<int64_t>(std::max<int64_t>(nq, nr), 1);
    s.table = c.take<CloudParams>(C);
    s.query_prefix = c.take<int32_t>(C + 1);
    s.ref_prefix = c.take<int32_t>(C + 1);
    s.qparams = c.take<QueryParams>(C);
    s.sort_state = c.take<SortState64>(1);
    s.num_qgroups = c.take<int32_t>(1);
    s.num_units = c.take<int32_t>(1);
    s.num_stray = c.take<int32_t>(1);
    s.work = c.take<int32_t>(kWorkCounters);
    s.total = c.take<int64_t>(1);
    s.info = c.take<int64_t>(8);
    s.num_flagged = c.take<int32_t>(1);
    s.exact_clouds = c.take<int32_t>(1);
    s.num_exact = c.take<int32_t>(1);
    s.unit_cap = c.take<int32_t>(1);
    s.cursor = c.take<unsigned long long>(1);
    s.pack = c.take<float4>(nmax);
    s.keys[0] = c.take<unsigned long long>(nmax);
    s.keys[1] = c.take<unsigned long long>(nmax);
    s.vals[0] = c.take<int32_t>(nmax);
    s.vals[1] = c.take<int32_t>(nmax);
    s.hist = c.take<int32_t>(sort_hist_elems(nmax));
    s.tile_sums = c.take<int32_t>(kBins);  // the sort's digit totals
    s.scan_tiles64 = c.take<int64_t>(scan_tiles(nmax + 1));
    s.scan_tiles32 = c.take<int32_t>(scan_tiles(nmax + 1));
    const int64_t q = std::max<int64_t>(nq, 1);
    s.qsorted = c.take<float4>(q);
    s.qsidx = c.take<int32_t>(q);
    s.qgroup_start = c.take<int32_t>(q + 1);
    s.qgroup_coords = c.take<int32_t>(3 * q);
    s.qgroup_cloud = c.take<int32_t>(q);
    s.unit_group = c.take<int32_t>(q);
    s.unit_t0 = c.take<int32_t>(q);
    s.counts = c.take<int32_t>(q);
    s.stray = c.take<int32_t>(q);
    s.rec = c.take<int32_t>(q);
    s.flagged = c.take<int32_t>(q);
    const int64_t ni = incremental ? std::max<int64_t>(nr, 1) : 0;
    s.stay = incremental ? c.take<int32_t>(ni) : nullptr;
    s.stay_keys = incremental ? c.take<unsigned long long>(ni) : nullptr;
    s.stay_idx = incremental ? c.take<int32_t>(ni) : nullptr;
    for (int k = 0; k < 2; ++k) {
        s.moved_keys[k] = incremental ? c.take<unsigned long long>(ni) : nullptr;
        s.moved_vals[k] = incremental ? c.take<int32_t>(ni) : nullptr;
    }
    s.moved_state = incremental ? c.take<SortState64>(1) : nullptr;
    s.inc_count = incremental ? c.take<int32_t>(2) : nullptr;
    if (bytes) *bytes = c.off;
    return s;
}

template <typename K>
static SortWorkspaceT<K> sort_workspace(const Scratch& W) {
    SortWorkspaceT<K> s;
    s.keys[0] = reinterpret_cast<K*>(W.keys[0]);
    s.keys[1] = reinterpret_cast<K*>(W.keys[1]);
    s.vals[0] = W.vals[0];
    s.vals[1] = W.vals[1];
    s.hist = W.hist;
    s.tile_sums = W.tile_sums;
    s.state = reinterpret_cast<SortStateT<K>*>(W.sort_state);
    return s;
}

// ------------------------------------------------------------------------------------------
// the cloud table

// Host -> device copy of the table as kernel parameters (no pageable copy, so it also records
// into a CUDA graph): chunks of kUploadChunk clouds per launch.
constexpr int kUploadChunk = 24;
struct CloudChunk {
    int32_t first, count, n_clouds, query_total, ref_total, pad;
    CloudParams p[kUploadChunk];
};
static_assert(sizeof(CloudChunk) <= 4000, "kernel parameter block too large");

__global__ void upload_clouds_kernel(CloudChunk ch, CloudParams* table, int32_t* query_prefix, int32_t* ref_prefix) {
    const int i = threadIdx.x;
    if (i < ch.count) {
        const int c = ch.first + i;
        table[c] = ch.p[i];
        query_prefix[c] = ch.p[i].query_base;
        ref_prefix[c] = ch.p[i].ref_base;
    }
    if (i == 0 && ch.first + ch.count == ch.n_clouds) {
        query_prefix[ch.n_clouds] = ch.query_total;
        ref_prefix[ch.n_clouds] = ch.ref_total;
    }
}

// Cloud of global point index i: the last c with prefix[c] <= i (empty clouds are skipped).
__device__ __forceinline__ int cloud_of(const int32_t* __restrict__ prefix, int C, int64_t i) {
    if (C == 1) return 0;
    int lo = 0, hi = C;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------------------------------------
// build kernels

// Block reduction of max / or; one atomic per block and field.
__device__ __forceinline__ void block_reduce_stats(uint32_t kmax, int bad, SupportStats* out) {
    __shared__ uint32_t s_max[32];
    __shared__ int s_bad[32];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { s_max[w] = kmax; s_bad[w] = bad; }
    __syncthreads();
    if (w == 0) {
        kmax = lane < nw ? s_max[lane] : 0u;
        bad = lane < nw ? s_bad[lane] : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        }
        if (lane == 0) {
            atomicMax(&out->max_key, kmax);
            if (bad) atomicOr(&out->bad, 1);
        }
    }
}

__device__ __forceinline__ SupportStats* stats_at(char* base, int64_t stride, int c) {
    return reinterpret_cast<SupportStats*>(base + stride * c);
}
__device__ __forceinline__ void stats_atomic(SupportStats* s, uint32_t kmax, int bad) {
    if (kmax) atomicMax(&s->max_key, kmax);
    if (bad) atomicOr(&s->bad, 1);
}

// Per-cloud maximum support (computeGridSupport, cellTable.py:40-81, needs it) and whether every
// support lies in [1e-18, 1e18] (else the exact test decides every pair).  Each block reduces a
// contiguous range, so a thread changes cloud only at cloud boundaries; a block that stayed in one
// cloud issues one atomic per field.  The record of cloud c is at out + c * stride.
__global__ void support_stats_kernel(const CloudParams* __restrict__ table, const int32_t* __restrict__ prefix, int C,
                                     int64_t n, int query_side, char* out, int64_t stride) {
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * per;
    const int64_t hi = min(n, lo + per);
    int cur = -1;
    int64_t cbase = 0, cend = 0;
    const float* h = nullptr;
    uint32_t kmax = 0;
    int bad = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        if (cur < 0 || i >= cend) {
            if (cur >= 0) stats_atomic(stats_at(out, stride, cur), kmax, bad);
            cur = cloud_of(prefix, C, i);
            cbase = prefix[cur];
            cend = prefix[cur + 1];
            h = query_side ? table[cur].query_sup : table[cur].ref_sup;
            kmax = 0;
            bad = 0;
        }
        if (h) {
            const float v = h[i - cbase];
            kmax = max(kmax, float_key(v));
            bad |= !(v >= 1e-18f && v <= 1e18f);
        }
    }
    __shared__ int s_cloud;
    if (threadIdx.x == 0) s_cloud = cur;  // thread 0 holds the block's first point, if it has any
    __syncthreads();
    if (__syncthreads_and(cur < 0 || cur == s_cloud)) {
        if (s_cloud >= 0) block_reduce_stats(kmax, bad, stats_at(out, stride, s_cloud));
    } else if (cur >= 0) {
        stats_atomic(stats_at(out, stride, cur), kmax, bad);
    }
}

// Start of a build: per-cloud statistics and flags, counters, the sort state.
template <typename K>
__global__ void grid_init_kernel(GridParams* g, int C, Structure S, Scratch W) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        g[c].ref_stats.max_key = 0;
        g[c].ref_stats.bad = 0;
        g[c].build_query_stats.max_key = 0;
        g[c].build_query_stats.bad = 0;
        g[c].error = 0;
        g[c].out_of_grid = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *S.bad_grids = 0;
        *S.num_cells = 0;
        sort_state_reset(reinterpret_cast<SortStateT<K>*>(W.sort_state));
    }
}

template <typename K>
__global__ void sort_state_init_kernel(SortStateT<K>* st) { sort_state_reset(st); }

// End of the last cell (or query group): cell_start[C] = n.
__global__ void finish_cells_kernel(int32_t* cell_start, const int32_t* num_cells, int64_t n) {
    cell_start[*num_cells] = (int32_t)n;
}

// Per cloud: util.py:28-79 compute_h and cellTable.py:27-29, float32 throughout.
// same_sup: the query supports are the reference support array (statistics reduced once).
__global__ void grid_params_kernel(const CloudParams* __restrict__ table, GridParams* grid, int C,
                                   int32_t* bad_grids, int same_sup) {
    const float grow = 1.00010001659393310546875f;  // fl32(1e-4 + 1)
    for (int cl = blockIdx.x * blockDim.x + threadIdx.x; cl < C; cl += gridDim.x * blockDim.x) {
        const CloudParams& sp = table[cl];
        GridParams* g = &grid[cl];
        if (same_sup) g->build_query_stats = g->ref_stats;
        // computeGridSupport: scatter reads the reference supports, gather the query supports,
        // (super)symmetric both (torch.max propagates NaN, as the key maximum does).
        uint32_t key = 0;
        if (sp.mode != kGather) key = max(key, g->ref_stats.max_key);
        if (sp.mode != kScatter) key = max(key, g->build_query_stats.max_key);
        const float hmax = key_float(key);
        float ext[3], nc[3], h[3];
        bool any = false;
        for (int d = 0; d < sp.dim; ++d) {
            ext[d] = __fsub_rn(sp.dmax[d], sp.dmin[d]);
            nc[d] = floorf(__fdiv_rn(ext[d], hmax));
            h[d] = __fdiv_rn(ext[d], nc[d]);
        }
        for (int d = 0; d < sp.dim; ++d) any |= __fsub_rn(__fdiv_rn(ext[d], h[d]), nc[d]) > 0.0f;
        if (any)
            for (int d = 0; d < sp.dim; ++d) {
                nc[d] = __fsub_rn(nc[d], 1.0f);
                h[d] = __fdiv_rn(ext[d], nc[d]);
            }
        any = false;
        for (int d = 0; d < sp.dim; ++d) {
            const float r = __fdiv_rn(ext[d], h[d]);
            any |= ceilf(r) > r;
        }
        if (any)
            for (int d = 0; d < sp.dim; ++d) h[d] = __fmul_rn(h[d], grow);
        float hc = h[0];
        for (int d = 1; d < sp.dim; ++d) {
            const float v = h[d];
            if (hc != hc) break;
            if (v != v || v > hc) hc = v;  // torch.max propagates NaN
        }
        g->hmax = hmax;
        g->hcell = hc;
        if (sp.hcell_override[0] > 0.0f) {  // caller-chosen grid (multi-level search)
            hc = sp.hcell_override[0];
            for (int d = 0; d < 3; ++d) {
                g->hcell_d[d] = d < sp.dim ? sp.hcell_override[d] : 1.0f;
                hc = fminf(hc, g->hcell_d[d]);
            }
            for (int d = 0; d < 3; ++d) {
                if (d >= sp.dim) { g->count[d] = 1; continue; }
                const float r = __fdiv_rn(ext[d], g->hcell_d[d]);
                // periodic dims of a clamped grid hold a whole number of cells (ext / n each);
                // rounding must not add a sliver cell at the seam
                g->count[d] = (sp.dedupe && ((sp.periodic_mask >> d) & 1)) ? max(1, (int32_t)rintf(r))
                                                                             : (int32_t)ceilf(r);
            }
        } else {
            for (int d = 0; d < 3; ++d) {
                g->hcell_d[d] = hc;
                g->count[d] = d < sp.dim ? (int32_t)ceilf(__fdiv_rn(ext[d], hc)) : 1;
            }
        }
        g->always_exact = ((sp.mode != kGather && g->ref_stats.bad) || (sp.mode != kScatter && g->build_query_stats.bad))
                              ? 1 : 0;
        int err = 0;
        if (!(hc > 0.0f) || !isfinite(hc)) err = 1;  // no valid grid (support larger than the domain, NaN, ...)
        if (sp.dedupe) {  // clamped grid: linear indices must not wrap
            double cells = 1.0;
            for (int d = 0; d < sp.dim; ++d) cells *= (double)max(g->count[d], 1);
            if (cells >= 2147483647.0) err = 1;
        }
        for (int d = 0; d < sp.dim; ++d)
            if (((sp.periodic_mask >> d) & 1) && g->count[d] <= 0) err = 1;
        g->error = err;
        if (err && sp.n_query > 0 && sp.n_ref > 0) atomicAdd(bad_grids, 1);
    }
}

// Per cloud: the query-side parameters of the lean test.
// same_sup: the queries are the reference points with the same support array, whose statistics the
// build reduced already.
__global__ void query_params_kernel(const CloudParams* __restrict__ table, const GridParams* __restrict__ grid, int C,
                                    QueryParams* qp, int32_t* exact_clouds, int same_sup) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        const CloudParams& cp = table[c];
        QueryParams& q = qp[c];
        if (same_sup) q.stats = grid[c].ref_stats;
        const bool has_q = cp.query_sup != nullptr;
        const float qmax = has_q ? key_float(q.stats.max_key) : 0.0f;
        q.qmax = (cp.mode == kScatter) ? 0.0f : qmax;
        const bool qbad = (cp.mode != kScatter) && has_q && q.stats.bad;
        const bool rbad = (cp.mode != kGather) && grid[c].ref_stats.bad;
        q.exact_all = (qbad || rbad || !(fabsf(q.qmax) <= 1e18f)) ? 1 : 0;
        if (q.exact_all && cp.n_query > 0) atomicAdd(exact_clouds, 1);
    }
}

// Zeroes the per-search counters, the per-cloud query statistics and the per-query counts.
__global__ void count_init_kernel(Scratch W, int C, int unit_cap, int64_t nq) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        W.qparams[c].stats.max_key = 0;
        W.qparams[c].stats.bad = 0;
        W.qparams[c].coord_key = 0;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x)
        W.counts[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int k = 0; k < kWorkCounters; ++k) W.work[k] = 0;
        *W.num_stray = 0;
        *W.num_units = 0;
        *W.num_flagged = 0;
        *W.exact_clouds = 0;
        *W.num_exact = 0;
        *W.unit_cap = unit_cap;
        *W.cursor = 0ull;
    }
}

__device__ __forceinline__ float4 load_point(const float* x, const float* h, int64_t i, int dim) {
    float4 v = make_float4(0.f, 0.f, 0.f, h ? h[i] : 0.0f);
    const float* p = x + i * dim;
    v.x = p[0];
    if (dim > 1) v.y = p[1];
    if (dim > 2) v.z = p[2];
    return v;
}

__device__ __forceinline__ float4 wrap_point(int dim, int mask, const float* dmin, const float* ext, float4 v,
                                             int times) {
    for (int d = 0; d < dim; ++d)
        if ((mask >> d) & 1) {
            float c = comp(v, d);
            for (int t = 0; t < times; ++t) c = wrap_coord(c, dmin[d], ext[d]);
            if (d == 0) v.x = c; else if (d == 1) v.y = c; else v.z = c;
        }
    return v;
}

// Integer cell of a point; a clamped grid (dedupe) puts every point in a cell of [0, count):
// no aliasing, no short seam cell.
__device__ __forceinline__ void cell_of(int dim, int dedupe, const float* dmin, const float* hcell,
                                        const int32_t* count, const float4& v, int32_t* c) {
    c[0] = cell_coord(v.x, dmin[0], hcell[0]);
    c[1] = dim > 1 ? cell_coord(v.y, dmin[1], hcell[1]) : 0;
    c[2] = dim > 2 ? cell_coord(v.z, dmin[2], hcell[2]) : 0;
    if (dedupe)
        for (int d = 0; d < dim; ++d) c[d] = min(max(c[d], 0), count[d] - 1);
}

// (cloud, signed-order linear index) sort keys; one cloud needs no cloud bits.
__device__ __forceinline__ void make_key(uint32_t& k, int, uint32_t lin_key) { k = lin_key; }
__device__ __forceinline__ void make_key(unsigned long long& k, int cloud, uint32_t lin_key) {
    k = ((unsigned long long)(uint32_t)cloud << 32) | lin_key;
}
__device__ __forceinline__ int key_cloud(uint32_t) { return 0; }
__device__ __forceinline__ int key_cloud(unsigned long long k) { return (int)(k >> 32); }
__device__ __forceinline__ uint32_t key_low(uint32_t k) { return k; }
__device__ __forceinline__ uint32_t key_low(unsigned long long k) { return (uint32_t)k; }
template <typename K>
__device__ __forceinline__ K kmin2(K a, K b) { return a < b ? a : b; }
template <typename K>
__device__ __forceinline__ K kmax2(K a, K b) { return a < b ? b : a; }

// What a point-parallel kernel needs of the point's cloud, reloaded when a thread crosses into
// another cloud.
struct PointCtx {
    int32_t cloud, dim, periodic_mask, dedupe, error;
    int64_t base, end;
    float dmin[3], ext[3], hcell[3];
    int32_t count[3];
    const float* pos;
    const float* sup;
};
__device__ __forceinline__ void load_point_ctx(PointCtx& p, const CloudParams* __restrict__ table,
                                               const GridParams* grid, const int32_t* __restrict__ prefix, int c,
                                               bool query_side) {
    const CloudParams& cp = table[c];
    const GridParams& g = grid[c];
    p.cloud = c;
    p.dim = cp.dim;
    p.periodic_mask = cp.periodic_mask;
    p.dedupe = cp.dedupe;
    p.error = g.error;
    p.base = prefix[c];
    p.end = prefix[c + 1];
    for (int d = 0; d < 3; ++d) {
        p.dmin[d] = cp.dmin[d];
        p.ext[d] = cp.ext[d];
        p.hcell[d] = g.hcell_d[d];
        p.count[d] = g.count[d];
    }
    p.pos = query_side ? cp.query_pos : cp.ref_pos;
    p.sup = query_side ? cp.query_sup : cp.ref_sup;
}

// Wrap (twice for the reference cloud, cppSearch.py:221 after neighborhood.py:203; once for a
// query cloud), pack to float4 and emit the (cloud, linear cell) key.  A cloud without a valid
// grid gets one constant key (its points form one cell that no walk visits).
// hint (incremental build): the point's previous linear cell; stay[i] = it is still there.
template <typename K>
__global__ void pack_points_kernel(const CloudParams* __restrict__ table, GridParams* grid,
                                   const int32_t* __restrict__ prefix, int C, int64_t n, int query_side, int wraps,
                                   int track_grid, float4* __restrict__ pack, K* __restrict__ keys,
                                   int32_t* __restrict__ vals, SortStateT<K>* st,
                                   const int32_t* __restrict__ hint = nullptr, int32_t* __restrict__ stay = nullptr) {
    K kmin = ~(K)0, kmax = 0;
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * per;
    const int64_t hi = min(n, lo + per);
    PointCtx p;
    p.cloud = -1;
    p.end = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        if (p.cloud < 0 || i >= p.end) load_point_ctx(p, table, grid, prefix, cloud_of(prefix, C, i), query_side != 0);
        float4 v = load_point(p.pos, p.sup, i - p.base, p.dim);
        uint32_t lin = 0;
        if (!p.error) {
            v = wrap_point(p.dim, p.periodic_mask, p.dmin, p.ext, v, wraps);
            int32_t c[3];
            cell_of(p.dim, p.dedupe, p.dmin, p.hcell, p.count, v, c);
            if (track_grid) {
                bool out = false;
                for (int d = 0; d < p.dim; ++d) out |= c[d] < 0 || c[d] >= p.count[d];
                if (out && !*(volatile int32_t*)&grid[p.cloud].out_of_grid) atomicOr(&grid[p.cloud].out_of_grid, 1);
            }
            lin = (uint32_t)linear_index(p.dim, c, p.count);
        }
        K key;
        make_key(key, p.cloud, lin ^ 0x80000000u);
        if (stay) stay[i] = (!p.error && hint[i] == (int32_t)lin) ? 1 : 0;
        pack[i] = v;
        keys[i] = key;
        vals[i] = (int32_t)i;
        kmin = kmin2(kmin, key);
        kmax = kmax2(kmax, key);
    }
    __shared__ K s_min[32], s_max[32];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        kmin = kmin2(kmin, (K)__shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = kmax2(kmax, (K)__shfl_xor_sync(0xffffffffu, kmax, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { s_min[w] = kmin; s_max[w] = kmax; }
    __syncthreads();
    if (w == 0) {
        kmin = lane < nw ? s_min[lane] : ~(K)0;
        kmax = lane < nw ? s_max[lane] : (K)0;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            kmin = kmin2(kmin, (K)__shfl_xor_sync(0xffffffffu, kmin, o));
            kmax = kmax2(kmax, (K)__shfl_xor_sync(0xffffffffu, kmax, o));
        }
        if (lane == 0) {
            atomicMin(&st->key_min, kmin);
            atomicMax(&st->key_max, kmax);
        }
    }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ void map_insert(unsigned long long* map, int64_t cap, int32_t lin, int32_t cell) {
    const unsigned long long entry = ((unsigned long long)(uint32_t)lin << 32) | (uint32_t)cell;
    uint64_t slot = mix32((uint32_t)lin) & (cap - 1);
    for (int64_t probe = 0; probe < cap; ++probe) {
        unsigned long long prev = atomicCAS(&map[slot], ~0ull, entry);
        if (prev == ~0ull || (uint32_t)(prev >> 32) == (uint32_t)lin) return;
        slot = (slot + 1) & (cap - 1);
    }
}

__device__ __forceinline__ int32_t map_find(const unsigned long long* __restrict__ map, int64_t cap, int32_t lin) {
    uint64_t slot = mix32((uint32_t)lin) & (cap - 1);
    for (int64_t probe = 0; probe < cap; ++probe) {
        unsigned long long e = __ldg(&map[slot]);
        if (e == ~0ull) return -1;
        if ((uint32_t)(e >> 32) == (uint32_t)lin) return (int32_t)(uint32_t)e;
        slot = (slot + 1) & (cap - 1);
    }
    return -1;
}

// Run starts of the sorted keys (unique_consecutive, hashTable.py:193).
template <typename K>
struct RunFlagIn {
    const K* keys0;
    const K* keys1;
    const SortStateT<K>* st;
    __device__ int32_t operator()(int64_t i) const {
        const K* k = st->sel[key_passes<K>()] ? keys1 : keys0;
        return (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
    }
};

// Writes one cell record per run start: begin, lin, cloud, coords of the run's first point,
// bucket, and the cell's entry in its cloud's map region.
template <typename K>
struct CellOut {
    const CloudParams* table;
    const GridParams* grid;
    const K* keys0;
    const K* keys1;
    const SortStateT<K>* st;
    const float4* rsorted;
    int32_t* cell_start;
    int32_t* cell_lin;
    int32_t* cell_coords;
    int32_t* cell_bucket;
    int32_t* cell_cloud;
    unsigned long long* map;
    int32_t n_points;
    __device__ void write(int64_t i, int32_t ex) const {
        const K* k = st->sel[key_passes<K>()] ? keys1 : keys0;
        const K key = k[i];
        const int cloud = key_cloud(key);
        const int32_t lin = (int32_t)(key_low(key) ^ 0x80000000u);
        const CloudParams& cp = table[cloud];
        const GridParams& g = grid[cloud];
        int32_t c[3] = {0, 0, 0};
        uint32_t bucket = 0;
        if (!g.error) {
            cell_of(cp.dim, cp.dedupe, cp.dmin, g.hcell_d, g.count, rsorted[i], c);
            bucket = ref_hash(cp.dim, c, cp.hash_len);
            map_insert(map + cp.map_base, cp.map_cap, lin, ex);
        }
        cell_start[ex] = (int32_t)i;
        cell_lin[ex] = lin;
        cell_cloud[ex] = cloud;
        cell_coords[3 * ex + 0] = c[0];
        cell_coords[3 * ex + 1] = c[1];
        cell_coords[3 * ex + 2] = c[2];
        cell_bucket[ex] = (int32_t)bucket;
    }
};

// The run-start scan writes only where each cell begins; the cell records are then written by one
// thread per cell (a run start is one element in 16 here, so doing that work inside the scan left
// most lanes of every warp idle behind a long chain of dependent loads and the map insert).
struct CellStartOut {
    int32_t* cell_start;
    int32_t n_points;
    __device__ void operator()(int64_t i, int32_t ex, int32_t flag) const {
        if (flag && TCR_IN(ex, n_points)) cell_start[ex] = (int32_t)i;
    }
};
template <typename K>
__global__ void cell_records_kernel(CellOut<K> co, const int32_t* __restrict__ num_cells, int64_t n) {
    const int32_t nc = *num_cells;
    if (blockIdx.x == 0 && threadIdx.x == 0) co.cell_start[nc] = (int32_t)n;  // end of the last cell
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int32_t i = co.cell_start[c];
        if (TCR_GUARD(i, n)) co.write(i, c);
    }
}

// lin_out (optional): the linear cell of each sorted point, the hint of the next incremental build;
// order_out (optional): a copy of the sort index.
// The build's consumer of its sort: the sorted points, their input indices and (for the serving
// loop) each point's linear cell and input index, written as the sort's last pass places them.
template <typename K>
struct SortedPointsOut {
    static constexpr bool kActive = true;
    const float4* __restrict__ pack;
    float4* __restrict__ sorted;
    int32_t* __restrict__ sidx;
    int32_t* __restrict__ lin_out;
    int32_t* __restrict__ order_out;
    int64_t n;
    __device__ __forceinline__ void operator()(int64_t i, K key, int32_t p) const {
        if (!TCR_IN(p, n)) return;
        sorted[i] = pack[p];
        sidx[i] = p;
        if (lin_out) lin_out[i] = (int32_t)(key_low(key) ^ 0x80000000u);
        if (order_out) order_out[i] = p;
    }
};

// The same placement when the sort's last pass did not do it (no pass moved the points, or an
// incremental build's merge ordered them).
template <typename K>
__global__ void gather_sorted_kernel(const float4* __restrict__ pack, const int32_t* vals0, const int32_t* vals1,
                                     const SortStateT<K>* st, int64_t n, float4* __restrict__ sorted,
                                     int32_t* __restrict__ sidx, const K* keys0 = nullptr, const K* keys1 = nullptr,
                                     int32_t* __restrict__ lin_out = nullptr,
                                     int32_t* __restrict__ order_out = nullptr) {
    if (st->consumed) return;
    const int32_t* v = st->sel[key_passes<K>()] ? vals1 : vals0;
    const K* k = st->sel[key_passes<K>()] ? keys1 : keys0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int32_t p = v[i];
        if (!TCR_IN(p, n)) continue;
        sorted[i] = pack[p];
        sidx[i] = p;
        if (lin_out) lin_out[i] = (int32_t)(key_low(k[i]) ^ 0x80000000u);
        if (order_out) order_out[i] = p;
    }
}

// ------------------------------------------------------------------------------------------
// incremental re-sort
//
// A build may be given the reference points in the cell order of a previous build, with each
// point's previous linear cell (the hint).  The points still in their cell ("unmoved") then form
// a subsequence already sorted by (key, input index); only the moved points are radix-sorted, and
// the two sorted lists are merged by (key, input index) -- exactly the stable sort of the input.
// The unmoved subsequence is verified on the device; if it is not sorted (a wrong hint), or too
// many points moved, the full radix sort runs instead.  Every kernel reads the decision from the
// device, so the build enqueues without a host round trip.

struct StayIn {
    const int32_t* stay;
    __device__ int32_t operator()(int64_t i) const { return stay[i]; }
};
template <typename K>
struct StayOut {
    const K* keys;        // the pack output, input order
    K* stay_keys;
    int32_t* stay_idx;
    K* moved_keys;
    int32_t* moved_vals;
    __device__ void operator()(int64_t i, int32_t ex, int32_t flag) const {
        if (flag) {
            stay_keys[ex] = keys[i];
            stay_idx[ex] = (int32_t)i;
        } else {
            moved_keys[i - ex] = keys[i];
            moved_vals[i - ex] = (int32_t)i;
        }
    }
};

template <typename K>
__global__ void inc_check_kernel(const K* __restrict__ stay_keys, const int32_t* n_stay, int32_t* bad) {
    const int64_t n = *n_stay;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    bool ok = true;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k + 1 < n; k += stride)
        ok &= stay_keys[k] <= stay_keys[k + 1];
    if (!__all_sync(0xffffffffu, ok) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
}

// Chooses the path: the moved points' sort and the merge, or the full sort (one thread).
template <typename K>
__global__ void inc_decide_kernel(SortStateT<K>* full, SortStateT<K>* moved, const int32_t* counts, int64_t n) {
    const int64_t n_stay = counts[0];
    const bool fallback = counts[1] != 0 || 2 * n_stay < n;  // wrong hint, or most points moved
    sort_state_reset(moved);
    if (fallback) {
        moved->key_min = moved->key_max = 0;  // no moved sort
        return;
    }
    moved->key_min = full->key_min;  // a superset of the moved keys' range
    moved->key_max = full->key_max;
    moved->n_dev = n - n_stay;
    full->key_min = full->key_max = 0;  // no full sort: the merge writes the sorted keys in place
}

// Number of list entries ordered before (key, idx); the list is sorted by (key, idx).
template <typename K>
__device__ __forceinline__ int64_t count_before(const K* keys, const int32_t* idx, int64_t n, K key, int32_t i) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const K km = keys[mid];
        if (km < key || (km == key && idx[mid] < i)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Merges the unmoved and the sorted moved points into keys/vals (input buffer 0 of the full sort,
// whose passes are all skipped on this path).
template <typename K>
__global__ void inc_merge_kernel(const K* __restrict__ stay_keys, const int32_t* __restrict__ stay_idx,
                                 const K* moved_k0, const K* moved_k1, const int32_t* moved_v0,
                                 const int32_t* moved_v1, const SortStateT<K>* moved, const int32_t* counts,
                                 int64_t n, K* __restrict__ keys, int32_t* __restrict__ vals) {
    if (counts[1] != 0 || 2 * (int64_t)counts[0] < n) return;  // the full sort runs instead
    const int64_t n_stay = counts[0], n_moved = n - n_stay;
    const int s = moved->sel[key_passes<K>()];
    const K* mk = s ? moved_k1 : moved_k0;
    const int32_t* mv = s ? moved_v1 : moved_v0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        K key;
        int32_t i;
        int64_t pos;
        if (t < n_stay) {
            key = stay_keys[t];
            i = stay_idx[t];
            pos = t + count_before(mk, mv, n_moved, key, i);
        } else {
            key = mk[t - n_stay];
            i = mv[t - n_stay];
            pos = (t - n_stay) + count_before(stay_keys, stay_idx, n_stay, key, i);
        }
        keys[pos] = key;
        vals[pos] = i;
    }
}

// ------------------------------------------------------------------------------------------
// query side

// Self search: query i is reference i, so the reference order and cells group the queries.
// Positions are the once-wrapped query coordinates (only periodic dims differ from rsorted).
__global__ void pack_self_queries_kernel(const CloudParams* __restrict__ table, const GridParams* grid,
                                         const int32_t* __restrict__ prefix, int C, const int32_t* __restrict__ rsidx,
                                         int64_t n, float4* __restrict__ qsorted, int32_t* __restrict__ qsidx) {
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * per;
    const int64_t hi = min(n, lo + per);
    PointCtx p;
    p.cloud = -1;
    p.base = p.end = 0;
    for (int64_t t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        const int32_t i = rsidx[t];
        if (p.cloud < 0 || i < p.base || i >= p.end) load_point_ctx(p, table, grid, prefix, cloud_of(prefix, C, i), true);
        qsorted[t] = wrap_point(p.dim, p.periodic_mask, p.dmin, p.ext, load_point(p.pos, p.sup, i - p.base, p.dim), 1);
        qsidx[t] = i;
    }
}

template <typename K>
struct QueryGroupOut {
    const CloudParams* table;
    const GridParams* grid;
    const K* keys0;
    const K* keys1;
    const SortStateT<K>* st;
    const float4* qsorted;
    int32_t* group_start;
    int32_t* group_coords;
    int32_t* group_cloud;
    int32_t n_points;
    __device__ void operator()(int64_t i, int32_t ex, int32_t flag) const {
        if (!flag) return;
        const K* k = st->sel[key_passes<K>()] ? keys1 : keys0;
        const int cloud = key_cloud(k[i]);
        const CloudParams& cp = table[cloud];
        const GridParams& g = grid[cloud];
        int32_t c[3] = {0, 0, 0};
        if (!g.error) cell_of(cp.dim, cp.dedupe, cp.dmin, g.hcell_d, g.count, qsorted[i], c);
        group_start[ex] = (int32_t)i;
        group_cloud[ex] = cloud;
        group_coords[3 * ex + 0] = c[0];
        group_coords[3 * ex + 1] = c[1];
        group_coords[3 * ex + 2] = c[2];
    }
};

// Group count comes from a device scalar; the scan kernels are launched over the upper bound
// and read the true count through the functor.  A unit holds at most `cap` (<= 32) queries.
struct BoundedUnitCountIn {
    const int32_t* group_start;
    const int32_t* num_groups;
    int32_t cap;
    __device__ int32_t operator()(int64_t g) const {
        if (g >= *num_groups) return 0;
        int32_t n = group_start[g + 1] - group_start[g];
        return (n + cap - 1) / cap;
    }
};
struct BoundedUnitOut {
    const int32_t* group_start;
    const int32_t* num_groups;
    int32_t* unit_group;
    int32_t* unit_t0;
    int32_t cap;
    int64_t bound = 1ll << 62;  // entries of unit_group / unit_t0 (checked build)
    __device__ void operator()(int64_t g, int32_t ex, int32_t nunits) const {
        if (g >= *num_groups) return;
        const int32_t s = group_start[g];
        for (int32_t u = 0; u < nunits; ++u) {
            if (!TCR_IN(ex + u, bound)) break;
            unit_group[ex + u] = (int32_t)g;
            unit_t0[ex + u] = s + u * cap;
        }
    }
};

// ------------------------------------------------------------------------------------------
// the candidate walk
//
// Work unit: <= 32 queries of one query group (cell).  One warp takes a unit, looks up its
// cloud (one copy of the cloud's parameters in shared memory, refreshed when the warp moves to
// another cloud), finds the unit's 3^d stencil cells and walks their candidates in chunks of 32.
// The count walk tests every (query, candidate) pair once and writes the unit's record -- its
// candidate runs and the 32-bit hit mask of every (query, chunk) -- to a staging list; the emit
// pass expands the records into CSR/COO slots.  A unit that finds the staging list full is only
// counted and is walked again by the emit walk, which writes its pairs directly.

// Float64 inputs (tcr_count_f64 / tcr_emit_f64): the walks find and test candidates on the float32
// copies and decide every pair inside the widened rounding band on these double arrays with the
// reference's double expression.  qpos == null: a float32 search.
struct F64Walk {
    const double* qpos;      // [nq * dim] queries, wrapped as the reference wraps them
    const double* qsup;      // [nq] or null
    const double4* rsorted;  // [nr] the references in the structure's cell order, .w = support
    double ext[3];           // max - min of the domain, in double
};

// common.h:106-129 and neighborhoodDynamic.h:59-70 at scalar_t = double: per dimension
// diff = moduloOp(x_i, x_j, max - min) = ((x_i - x_j + h/2) - floor((x_i - x_j + h/2) / h) * h) - h/2
// on periodic dimensions, x_i - x_j otherwise; sum += diff * diff; sqrt(sum) < the mode's
// threshold.  Explicit intrinsics keep every operation rounded on its own (no FMA).
__device__ __noinline__ bool f64_pair_test(int dim, int mask, int mode, const double* ext, const double* xi,
                                           double hi, const double* xj, double hj) {
    double sum = 0.0;
    for (int d = 0; d < dim; ++d) {
        double diff;
        if ((mask >> d) & 1) {
            const double h = ext[d];
            const double half = __ddiv_rn(h, 2.0);
            const double t = __dadd_rn(__dsub_rn(xi[d], xj[d]), half);
            diff = __dsub_rn(__dsub_rn(t, __dmul_rn(floor(__ddiv_rn(t, h)), h)), half);
        } else {
            diff = __dsub_rn(xi[d], xj[d]);
        }
        sum = __dadd_rn(sum, __dmul_rn(diff, diff));
    }
    const double dist = __dsqrt_rn(sum);
    double thr;
    switch (mode) {
        case kGather: thr = hi; break;
        case kScatter: thr = hj; break;
        case kSymmetric: thr = __ddiv_rn(__dadd_rn(hi, hj), 2.0); break;
        default: thr = hi < hj ? hj : hi; break;  // std::max
    }
    return dist < thr;
}

// Pair (cloud-local query qi, sorted reference j) of a float64 search decided on the double arrays.
__device__ __noinline__ bool f64_pair_decide(F64Walk f, int dim, int mask, int mode, int64_t qi, int32_t j) {
    double xi[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < dim; ++d) xi[d] = f.qpos[qi * dim + d];
    const double4 c = f.rsorted[j];
    const double xj[3] = {c.x, c.y, c.z};
    return f64_pair_test(dim, mask, mode, f.ext, xi, f.qsup ? f.qsup[qi] : 0.0, xj, c.w);
}

// The unit's cloud, as the walk kernels read it (shared memory, warp-uniform).
struct UnitCtx {
    int32_t cloud, dim, periodic_mask, dedupe;
    uint32_t hash_len;
    int32_t error, out_of_grid, exact_all;
    int32_t count[3];
    int32_t qshift, rshift;  // subtracted from global query / reference indices (cloud-local numbering)
    float dmin[3], hcell[3], ext[3];
    float rmax, qmax;        // largest reference / query support (band of the fast test)
    float f64_err;           // float64 inputs: bound on the error of a float32 coordinate difference
    int32_t shift_ok;        // periodic dims all hold >= 6 cells: candidates across a seam are shifted
    float shift_delta;       // bound on the error a shift adds to a difference
    int64_t map_base, map_cap;
};

struct WalkArgs {
    const CloudParams* __restrict__ table;
    const GridParams* grid;
    const QueryParams* __restrict__ qparams;
    const int32_t* __restrict__ query_prefix;
    int32_t num_clouds;
    int32_t local_index;          // 1: rows and columns numbered within each cloud
    int32_t mode;
    int32_t no_stray_check;       // self search, no periodic dims, same positions: a query's cell is its
                                  // group's unless its cloud has points outside the grid (out_of_grid)
    int32_t class_filter;         // >= 0: walk only units of clouds of this class (dim * 2 + periodic)
    int32_t pad0;
    const float4* __restrict__ rsorted;
    const int32_t* __restrict__ rsidx;
    const int32_t* __restrict__ cell_start;
    const int32_t* __restrict__ cell_bucket;
    const unsigned long long* __restrict__ map;
    const float4* __restrict__ qsorted;
    const int32_t* __restrict__ qsidx;
    const int32_t* __restrict__ group_start;
    const int32_t* __restrict__ group_coords;
    const int32_t* __restrict__ group_cloud;
    const int32_t* __restrict__ unit_group;
    const int32_t* __restrict__ unit_t0;
    const int32_t* __restrict__ num_units;
    const int32_t* __restrict__ unit_cap;   // queries per unit
    const int32_t* __restrict__ unit_list;  // emit re-walk: the units to walk
    const int32_t* __restrict__ num_list;
    int32_t* work;
    int32_t* stray;
    int32_t* num_stray;
    int32_t* counts;              // [nq] count output, global query order
    int32_t* rec;                 // [units] offset of each unit's record in the staging list, -1 if not staged
    int32_t* flagged;             // [units] units to re-walk in the emit pass
    int32_t* num_flagged;
    int32_t* num_exact;           // units re-tested with exact decisions
    unsigned long long* cursor;   // staging list fill
    int32_t* stage;               // staging list
    int64_t stage_cap;
    const int32_t* __restrict__ query_ids;  // optional: row written for global query q is query_ids[q]
    const int32_t* __restrict__ ref_ids;    // optional: column written for global reference j is ref_ids[j]
    const int64_t* offsets;       // emit input [nq+1]
    int64_t* row_out;             // emit: COO rows or null
    int64_t* col_out;             // emit: columns
    int64_t out_cap;              // emit: entries of row_out/col_out; writes beyond are dropped
    F64Walk f64;                  // float64 inputs, or qpos == null
    int64_t nq_total, nr_total;   // point counts (bounds of the checked build)
};

__device__ __forceinline__ void load_unit_ctx(UnitCtx& u, const WalkArgs& a, int cloud) {
    const CloudParams& cp = a.table[cloud];
    const GridParams& g = a.grid[cloud];
    const QueryParams& q = a.qparams[cloud];
    u.cloud = cloud;
    u.dim = cp.dim;
    u.periodic_mask = cp.periodic_mask;
    u.dedupe = cp.dedupe;
    u.hash_len = cp.hash_len;
    u.error = g.error;
    u.out_of_grid = g.out_of_grid;
    u.exact_all = q.exact_all;
    for (int d = 0; d < 3; ++d) {
        u.count[d] = g.count[d];
        u.dmin[d] = cp.dmin[d];
        u.hcell[d] = g.hcell_d[d];
        u.ext[d] = cp.ext[d];
    }
    u.qshift = a.local_index ? cp.query_base : 0;
    u.rshift = a.local_index ? cp.ref_base : 0;
    u.rmax = key_float(g.ref_stats.max_key);
    u.qmax = q.qmax;
    // Points of a stencil cell across the periodic seam can be moved by +-ext while staged, so
    // the fast test needs no wrap: with >= 6 cells on every periodic dimension no candidate is near
    // half the extent away, so the reference's moduloOp wraps exactly the shifted cells.  A shift
    // changes a difference by at most one rounding of the shifted coordinate plus the reference's
    // own rounding of q - c before its exact wrap: shift_delta bounds both.
    bool ok = cp.periodic_mask != 0;
    float delta = 0.0f;
    for (int d = 0; d < cp.dim; ++d)
        if ((cp.periodic_mask >> d) & 1) {
            ok = ok && g.count[d] >= 6;
            // two roundings of magnitude <= half an ulp of (|coordinate| + ext) each: <= 2^-23 of it
            delta = fmaxf(delta, (fmaxf(fabsf(cp.dmin[d]), fabsf(cp.dmax[d])) + cp.ext[d]) * 1.1920928955078125e-7f);
        }
    u.shift_ok = ok && isfinite(delta);
    u.shift_delta = delta;
    u.map_base = cp.map_base;
    u.map_cap = cp.map_cap;
    // a float32 copy of a double coordinate x is off by <= |x| 2^-24, the float difference adds one
    // rounding: 2^-21 of the largest |coordinate| bounds a difference's error with room to spare
    u.f64_err = a.f64.qpos ? key_float(q.coord_key) * 4.76837158203125e-7f : 0.0f;
}

__device__ __forceinline__ ExactCtx unit_exact_ctx(const UnitCtx& u, int mode) {
    ExactCtx c;
    c.dim = u.dim;
    c.mode = mode;
    c.periodic_mask = u.periodic_mask;
    c.ext[0] = u.ext[0];
    c.ext[1] = u.ext[1];
    c.ext[2] = u.ext[2];
    return c;
}

// Looks up stencil cell `o` (getOffsets order, last coordinate fastest) around cell gc with the
// reference's semantics; returns the sorted range or an empty one.
__device__ __forceinline__ void stencil_lookup(const WalkArgs& a, const UnitCtx& u, const int32_t* gc, int o,
                                               int32_t& beg, int32_t& cnt) {
    int32_t c[3] = {0, 0, 0};
    int rem = o;
    bool dup = false;
    for (int d = u.dim - 1; d >= 0; --d) {
        const int32_t off = rem % 3 - 1;
        rem /= 3;
        int32_t v = gc[d] + off;
        if ((u.periodic_mask >> d) & 1) {
            const int32_t n = u.count[d];
            v = pymod(v, n);
            // with fewer than 3 cells the wrapped offsets repeat a cell; the clamped grid visits it once
            if (u.dedupe && ((n == 1 && off != 0) || (n == 2 && off == 1))) dup = true;
        } else if (u.dedupe && (v < 0 || v >= u.count[d])) {
            dup = true;  // clamped grid: nothing lies outside it
        }
        c[d] = v;
    }
    beg = 0;
    cnt = 0;
    if (dup) return;
    const int32_t lin = linear_index(u.dim, c, u.count);
    const int32_t cell = map_find(a.map + u.map_base, u.map_cap, lin);
    if (cell < 0 || !TCR_GUARD(cell, a.nr_total)) return;
    // queryHashMap matches the linear index inside bucket hash(c) only.
    if ((uint32_t)__ldg(&a.cell_bucket[cell]) != ref_hash(u.dim, c, u.hash_len)) return;
    beg = __ldg(&a.cell_start[cell]);
    cnt = __ldg(&a.cell_start[cell + 1]) - beg;
}

template <int DIM>
__device__ __forceinline__ bool same_cell(const int32_t* a, const int32_t* b) {
    bool s = a[0] == b[0];
    if (DIM > 1) s &= a[1] == b[1];
    if (DIM > 2) s &= a[2] == b[2];
    return s;
}

// Per-candidate pieces of the lean test: the candidate's share of the threshold and the half
// width of the band (conservative over every query: qmax is the largest query support).
template <int MODE>
__device__ __forceinline__ float cand_share(float hc) {
    return MODE == kSymmetric ? 0.5f * hc : hc;
}
template <int MODE>
__device__ __forceinline__ float cand_band(float cw, float qmax) {
    float t;
    if (MODE == kGather) t = qmax;
    else if (MODE == kScatter) t = cw;
    else if (MODE == kSymmetric) t = fmaf(qmax, 0.5f, cw);
    else t = fmaxf(qmax, cw);
    return kBandEps * t * t;
}
// thr for (query support hq, candidate share cw), float-exact as the reference evaluates it.
template <int MODE>
__device__ __forceinline__ float pair_thr(float hq, float cw) {
    if (MODE == kGather) return hq;
    if (MODE == kScatter) return cw;
    if (MODE == kSymmetric) return fmaf(hq, 0.5f, cw);  // fl(hq/2 + hc/2) == fl(hq + hc) / 2
    return fmaxf(hq, cw);
}

// Per-dimension constants of the fast periodic difference: the extent h, the half extent at which
// a difference wraps (+inf on a non-periodic dimension, which never wraps) and the band around it
// inside which the wrap decision is left to the exact test.
struct WrapCtx {
    float h[3], half[3], epsh[3];
};
__device__ __forceinline__ WrapCtx wrap_ctx(int periodic_mask, const float* ext) {
    WrapCtx w;
    for (int d = 0; d < 3; ++d) {
        const bool p = (periodic_mask >> d) & 1;
        w.h[d] = ext[d];
        w.half[d] = p ? 0.5f * ext[d] : __int_as_float(0x7f800000);
        w.epsh[d] = p ? kBandEps * ext[d] : 0.0f;
    }
    return w;
}

// Float difference q - c along dimension d, wrapped once into [-h/2, h/2] on a periodic dimension
// (the reference's moduloOp decides exactly; a difference within the band of +-h/2 sets wrap_unc).
template <bool PERIODIC>
__device__ __forceinline__ float fast_diff(const WrapCtx& wc, int d, float q, float c, bool& wrap_unc) {
    float diff = q - c;
    if (PERIODIC) {
        const float ad = fabsf(diff);
        wrap_unc |= fabsf(ad - wc.half[d]) <= wc.epsh[d];
        if (ad >= wc.half[d]) diff -= copysignf(wc.h[d], diff);
    }
    return diff;
}

// One (query, candidate) test.  in: decided; unc: needs the exact reference test.
template <int DIM, bool PERIODIC, int MODE>
__device__ __forceinline__ void lean_test(const WrapCtx& wc, const float4& q, const float4& c, float cw, float band,
                                          bool& in, bool& unc) {
    bool wrap_unc = false;
    float dd[3];
#pragma unroll
    for (int d = 0; d < DIM; ++d) dd[d] = fast_diff<PERIODIC>(wc, d, comp(q, d), comp(c, d), wrap_unc);
    float d2 = dd[0] * dd[0];
    if (DIM > 1) d2 = fmaf(dd[1], dd[1], d2);
    if (DIM > 2) d2 = fmaf(dd[2], dd[2], d2);
    const float thr = pair_thr<MODE>(q.w, cw);
    const float r = fmaf(-thr, thr, d2);  // d2 - thr^2, one rounding; sign exact
    in = r < 0.0f;
    unc = (fabsf(r) <= band) || wrap_unc;
}

constexpr int kWalkWarps = 4;
// Resident blocks per SM the count walk is compiled for (registers <= 65536 / (128 * blocks)):
// eight (64 registers) on non-periodic clouds and seven (72) on periodic ones.  More resident
// warps beat the spills they cost: on the 1M workload 8/7/6/5/4 blocks measured
// 0.348/0.355/0.363/0.372/0.385 ms non-periodic, 8/7/6/5/4 blocks 0.414/0.403/0.426/0.436/0.467 ms
// periodic.
#ifndef TCR_WALK_MIN_BLOCKS
#define TCR_WALK_MIN_BLOCKS 8
#endif
#ifndef TCR_WALK_MIN_BLOCKS_PERIODIC
#define TCR_WALK_MIN_BLOCKS_PERIODIC 7
#endif
constexpr int kWalkMinBlocks = TCR_WALK_MIN_BLOCKS;
constexpr int kWalkMinBlocksPeriodic = TCR_WALK_MIN_BLOCKS_PERIODIC;

// Record of a staged unit in the staging list (int32 words):
//   [0] chunks of 32 candidates   [1] R, candidate runs   [2] nb, queries   [3] 0
//   [4, 4 + R)          first sorted index of each run
//   [4 + R, 5 + 2R)     candidate prefix of each run; entry R is the unit's candidate count M
//   [5 + 2R, ...)       hit masks, chunk-major: word c * nb + q, bit j set when query q meets
//                       candidate 32 c + j
// A run is a stretch of consecutive sorted points: stencil cells whose ranges continue each other
// (the row neighbours of a linear-order grid) merge into one.
constexpr int kRecHeader = 4;
__host__ __device__ __forceinline__ int64_t record_words(int32_t runs, int32_t nchunks, int32_t nb) {
    return kRecHeader + 2 * (int64_t)runs + 1 + (int64_t)nchunks * nb;
}

struct WalkSmem {
    float4 q[kWalkWarps][32];        // the unit's queries: x, y, z and the query's share of the test
    float4 qp[kWalkWarps][32];       // the same as 16 query pairs for the packed test (store_query_pair)
    float qh[kWalkWarps][32];        // the queries' supports (for the exact re-test)
    int32_t qid[kWalkWarps][32];     // the queries' cloud-local indices (float64 re-test)
    int32_t run_beg[kWalkWarps][32];
    int32_t run_pre[kWalkWarps][33];
    float shift[kWalkWarps][3][32];  // per run: +-ext on the dimensions its cells lie across a seam
    float4 ring[kWalkWarps][4][32];  // candidate chunks in flight (cp.async), one slot per lane
    UnitCtx u[kWalkWarps];
};

// cp.async of 16 bytes from global to shared memory, its commit and wait (the copies of one
// thread land in program order of their groups; a thread reads back only what it copied itself).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Candidate k of the unit (prefix pre[0..S]): returns its sorted index.
__device__ __forceinline__ int32_t cand_index(const int32_t* pre, const int32_t* beg, int S, int32_t k) {
    int lo = 0, hi = S;  // pre[lo] <= k < pre[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (pre[mid] <= k) lo = mid; else hi = mid;
    }
    return beg[lo] + (k - pre[lo]);
}

// The query's share of the test, kept in the .w of its shared-memory copy: gather hq^2 (the test is
// d2 - hq^2), symmetric hq / 2 (thr = hq / 2 + hc / 2 == fl(hq + hc) / 2), superSymmetric hq.
template <int MODE>
__device__ __forceinline__ float query_share(float hq) {
    return MODE == kSymmetric ? 0.5f * hq : (MODE == kGather ? hq * hq : hq);
}

// The largest threshold candidate c (share cw) can meet over every query (qmax: the largest query
// support); the band of the fast test is kBandEps times its square.
template <int MODE>
__device__ __forceinline__ float cand_tmax(float cw, float qmax) {
    if (MODE == kGather) return qmax;
    if (MODE == kScatter) return cw;
    if (MODE == kSymmetric) return fmaf(qmax, 0.5f, cw);
    return fmaxf(qmax, cw);
}

// Float test of query q (share in q.w) against candidate c (share cw): r < 0 means inside.
template <int DIM, bool PERIODIC, int MODE>
__device__ __forceinline__ float pair_residual(const WrapCtx& wc, const float4& q, const float4& c, float cw,
                                               bool& wrap_unc) {
    float dd[3];
#pragma unroll
    for (int d = 0; d < DIM; ++d) dd[d] = fast_diff<PERIODIC>(wc, d, comp(q, d), comp(c, d), wrap_unc);
    float d2 = dd[0] * dd[0];
    if (DIM > 1) d2 = fmaf(dd[1], dd[1], d2);
    if (DIM > 2) d2 = fmaf(dd[2], dd[2], d2);
    if (MODE == kGather) return d2 - q.w;  // same sign as d2 - hq * hq up to the band
    if (MODE == kScatter) return fmaf(-c.w, c.w, d2);
    const float thr = MODE == kSymmetric ? q.w + cw : fmaxf(q.w, c.w);
    return fmaf(-thr, thr, d2);
}

// Warp-wide 32 x 32 bit transpose: lane j holds row j (bit k = entry (j, k)); lane k receives
// column k (bit j = entry (j, k)).  Five butterfly stages swap ever smaller off-diagonal blocks
// with the partner lane (lane ^ s): the 16- and 8-bit stages are one byte permutation of the own
// and the partner's row each; in the 4-, 2- and 1-bit stages a lane keeps its own bits under a
// lane-dependent mask and takes the partner's row rotated into place (right by s in the upper
// lane of a pair, left by s in the lower one) under the complement.  The per-lane selectors,
// masks and rotations depend on the lane only, so a loop over chunks computes them once.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
    const uint32_t sel16 = (lane & 16) ? 0x3276u : 0x5410u;
    const uint32_t sel8 = (lane & 8) ? 0x3715u : 0x6240u;
    const uint32_t keep4 = (lane & 4) ? 0xf0f0f0f0u : 0x0f0f0f0fu, rot4 = (lane & 4) ? 4u : 28u;
    const uint32_t keep2 = (lane & 2) ? 0xccccccccu : 0x33333333u, rot2 = (lane & 2) ? 2u : 30u;
    const uint32_t keep1 = (lane & 1) ? 0xaaaaaaaau : 0x55555555u, rot1 = (lane & 1) ? 1u : 31u;
    x = __byte_perm(x, __shfl_xor_sync(0xffffffffu, x, 16), sel16);
    x = __byte_perm(x, __shfl_xor_sync(0xffffffffu, x, 8), sel8);
    uint32_t y = __shfl_xor_sync(0xffffffffu, x, 4);
    x = (x & keep4) | (__funnelshift_r(y, y, rot4) & ~keep4);
    y = __shfl_xor_sync(0xffffffffu, x, 2);
    x = (x & keep2) | (__funnelshift_r(y, y, rot2) & ~keep2);
    y = __shfl_xor_sync(0xffffffffu, x, 1);
    x = (x & keep1) | (__funnelshift_r(y, y, rot1) & ~keep1);
    return x;
}

// The lane's candidate against queries K4-1 .. 0 of the unit (K4 a multiple of 4; rows past the
// unit's queries are NaN and never hit): bit k of the result is query k's hit, taken from the sign
// of the residual (an arithmetic NaN is positive).  `unc` collects pairs inside the band.
template <int DIM, bool P, int MODE>
__device__ __forceinline__ uint32_t chunk_hits(const WrapCtx& wc, const float4* __restrict__ qsm, int K4,
                                               const float4& cv, float cw, float band, bool& unc) {
    uint32_t hit = 0;
    for (int k = K4 - 4; k >= 0; k -= 4) {
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            const float4 q = qsm[k + i];
            bool wu = false;
            const float r = pair_residual<DIM, P, MODE>(wc, q, cv, cw, wu);
            hit = __funnelshift_l(__float_as_uint(r), hit, 1);
            unc |= (fabsf(r) <= band) || wu;
        }
    }
    return hit;
}

// Query pairs for the packed test: pair p holds queries 2p and 2p + 1 as two float4,
// {x0, x1, y0, y1} and {z0, z1, s0, s1}, where s is the pair-share of packed_share.
template <int MODE>
__device__ __forceinline__ float packed_share(float hq) {
    return MODE == kGather ? -(hq * hq) : (MODE == kSymmetric ? 0.5f * hq : hq);
}
__device__ __forceinline__ void store_query_pair(float4* qp, int lane, float x, float y, float z, float s) {
    float* f = reinterpret_cast<float*>(qp + 2 * (lane >> 1));
    const int hi = lane & 1;
    f[hi] = x;
    f[2 + hi] = y;
    f[4 + hi] = z;
    f[6 + hi] = s;
}

// chunk_hits for non-wrapping differences (non-periodic clouds and pre-shifted seam candidates) in
// gather, scatter and symmetric mode, two queries per instruction: the differences and the squared
// distance run as packed float32x2 operations (each element rounded exactly as the scalar operation),
// so the residuals and hit bits equal chunk_hits's bit for bit.  umin collects the smallest |r|
// (NaN rows are ignored by fminf); the caller compares it with the candidate's band once per chunk.
template <int DIM, int MODE>
__device__ __forceinline__ uint32_t chunk_hits_x2(const float4* __restrict__ qp, int K4, const float4& cv, float cw,
                                                  float& umin) {
    const float2 ncx = make_float2(-cv.x, -cv.x), ncy = make_float2(-cv.y, -cv.y), ncz = make_float2(-cv.z, -cv.z);
    const float2 ncw = make_float2(-cv.w, -cv.w), pcw = make_float2(cv.w, cv.w);
    uint32_t hit = 0;
    for (int p = (K4 >> 1) - 2; p >= 0; p -= 2) {  // two query pairs per iteration (K4 a multiple of 4)
#pragma unroll
        for (int i = 1; i >= 0; --i) {
            const float4 a = qp[2 * (p + i)];
            const float4 b = qp[2 * (p + i) + 1];
            const float2 dx = __fadd2_rn(make_float2(a.x, a.y), ncx);
            float2 d2 = __fmul2_rn(dx, dx);
            if (DIM > 1) {
                const float2 dy = __fadd2_rn(make_float2(a.z, a.w), ncy);
                d2 = __ffma2_rn(dy, dy, d2);
            }
            if (DIM > 2) {
                const float2 dz = __fadd2_rn(make_float2(b.x, b.y), ncz);
                d2 = __ffma2_rn(dz, dz, d2);
            }
            float r0, r1;
            if (MODE == kGather) {  // d2 - hq^2, the share holding -hq^2
                const float2 r = __fadd2_rn(d2, make_float2(b.z, b.w));
                r0 = r.x;
                r1 = r.y;
            } else if (MODE == kScatter) {  // d2 - hc^2
                const float2 r = __ffma2_rn(ncw, pcw, d2);
                r0 = r.x;
                r1 = r.y;
            } else {  // symmetric: thr = hq / 2 + hc / 2, d2 - thr^2
                const float t0 = b.z + cw, t1 = b.w + cw;
                r0 = fmaf(-t0, t0, d2.x);
                r1 = fmaf(-t1, t1, d2.y);
            }
            hit = __funnelshift_l(__float_as_uint(r1), hit, 1);
            hit = __funnelshift_l(__float_as_uint(r0), hit, 1);
            umin = fminf(umin, fminf(fabsf(r0), fabsf(r1)));
        }
    }
    return hit;
}

// chunk_hits_x2 for the lane's candidates of two chunks at once: each query pair is read once for
// both, and the two candidates' chains of operations are independent, so they overlap.
template <int DIM, int MODE>
__device__ __forceinline__ void chunk_hits_x2_two(const float4* __restrict__ qp, int K4, const float4& cv0,
                                                  float cw0, const float4& cv1, float cw1, float& umin0,
                                                  float& umin1, uint32_t& hit0, uint32_t& hit1) {
    const float2 ax = make_float2(-cv0.x, -cv0.x), ay = make_float2(-cv0.y, -cv0.y), az = make_float2(-cv0.z, -cv0.z);
    const float2 bx = make_float2(-cv1.x, -cv1.x), by = make_float2(-cv1.y, -cv1.y), bz = make_float2(-cv1.z, -cv1.z);
    const float2 an = make_float2(-cv0.w, -cv0.w), ap = make_float2(cv0.w, cv0.w);
    const float2 bn = make_float2(-cv1.w, -cv1.w), bp = make_float2(cv1.w, cv1.w);
    uint32_t h0 = 0, h1 = 0;
    for (int p = (K4 >> 1) - 1; p >= 0; --p) {
        const float4 a = qp[2 * p];
        const float4 b = qp[2 * p + 1];
        const float2 qx = make_float2(a.x, a.y), qy = make_float2(a.z, a.w), qz = make_float2(b.x, b.y);
        const float2 dx0 = __fadd2_rn(qx, ax), dx1 = __fadd2_rn(qx, bx);
        float2 e0 = __fmul2_rn(dx0, dx0), e1 = __fmul2_rn(dx1, dx1);
        if (DIM > 1) {
            const float2 dy0 = __fadd2_rn(qy, ay), dy1 = __fadd2_rn(qy, by);
            e0 = __ffma2_rn(dy0, dy0, e0);
            e1 = __ffma2_rn(dy1, dy1, e1);
        }
        if (DIM > 2) {
            const float2 dz0 = __fadd2_rn(qz, az), dz1 = __fadd2_rn(qz, bz);
            e0 = __ffma2_rn(dz0, dz0, e0);
            e1 = __ffma2_rn(dz1, dz1, e1);
        }
        float2 r0, r1;  // residuals of the query pair against each candidate
        if (MODE == kGather) {
            const float2 s = make_float2(b.z, b.w);
            r0 = __fadd2_rn(e0, s);
            r1 = __fadd2_rn(e1, s);
        } else if (MODE == kScatter) {
            r0 = __ffma2_rn(an, ap, e0);
            r1 = __ffma2_rn(bn, bp, e1);
        } else {
            const float t00 = b.z + cw0, t01 = b.w + cw0, t10 = b.z + cw1, t11 = b.w + cw1;
            r0 = make_float2(fmaf(-t00, t00, e0.x), fmaf(-t01, t01, e0.y));
            r1 = make_float2(fmaf(-t10, t10, e1.x), fmaf(-t11, t11, e1.y));
        }
        h0 = __funnelshift_l(__float_as_uint(r0.y), h0, 1);
        h0 = __funnelshift_l(__float_as_uint(r0.x), h0, 1);
        h1 = __funnelshift_l(__float_as_uint(r1.y), h1, 1);
        h1 = __funnelshift_l(__float_as_uint(r1.x), h1, 1);
        umin0 = fminf(umin0, fminf(fabsf(r0.x), fabsf(r0.y)));
        umin1 = fminf(umin1, fminf(fabsf(r1.x), fabsf(r1.y)));
    }
    hit0 = h0;
    hit1 = h1;
}

// The same with every pair inside the band decided by the reference's exact test, on the original
// (unshifted) candidate of sorted index j -- in double on the double arrays for float64 inputs;
// rare units only, so out of line.
template <int DIM, int MODE>
__device__ __noinline__ uint32_t chunk_hits_exact(ExactCtx xc, const float4* qsm, const float* qh, const int32_t* qid,
                                                  int K4, float4 cv, int32_t j, float band, F64Walk f64) {
    const WrapCtx wc = wrap_ctx(xc.periodic_mask, xc.ext);
    const float cw = cand_share<MODE>(cv.w);
    uint32_t hit = 0;
    for (int k = K4 - 1; k >= 0; --k) {
        const float4 q = qsm[k];
        bool wu = false;
        const float r = pair_residual<DIM, true, MODE>(wc, q, cv, cw, wu);
        bool in = r < 0.0f;
        if ((fabsf(r) <= band) || wu)
            in = f64.qpos ? f64_pair_decide(f64, DIM, xc.periodic_mask, MODE, qid[k], j)
                          : exact_pair_test(xc, q, qh[k], cv, cv.w);
        hit = (hit << 1) | (in ? 1u : 0u);
    }
    return hit;
}

// Count walk of one unit: test every (query, candidate) once, count, and stage the unit's record.
//
// The unit's candidates stream in chunks of 32, one per lane (a coalesced load of consecutive
// sorted points); the unit's queries sit in shared memory and are broadcast to every lane, so each
// lane tests its candidate against every query with no lane left idle but the last chunk's.  A
// lane's hit bits over the queries are transposed across the warp into the (query, chunk) masks.
template <int DIM, bool PERIODIC, int MODE>
__device__ __forceinline__ void count_unit(const WalkArgs& a, WalkSmem& sm, int32_t unit, int32_t grp, int lane,
                                           int w) {
    constexpr int S = DIM == 1 ? 3 : (DIM == 2 ? 9 : 27);
    const UnitCtx& u = sm.u[w];
    const float inf = __int_as_float(0x7f800000);
    const float4 nan4 = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
    const int32_t t0 = a.unit_t0[unit];
    const int32_t nb = min(*a.unit_cap, a.group_start[grp + 1] - t0);
    const int32_t gc[3] = {a.group_coords[3 * grp], a.group_coords[3 * grp + 1], a.group_coords[3 * grp + 2]};
    // the unit's queries, loaded before the stencil look-ups so that both latencies overlap
    const bool qlane = lane < nb && TCR_IN(t0 + lane, a.nq_total);
    float4 qv = nan4;
    int32_t qorig = 0;
    if (qlane) {
        qv = a.qsorted[t0 + lane];
        qorig = a.qsidx[t0 + lane];
    }
    int32_t beg = 0, cnt = 0;
    if (lane < S) stencil_lookup(a, u, gc, lane, beg, cnt);
    const bool shift_mode = PERIODIC && u.shift_ok;
    float sh[3] = {0.f, 0.f, 0.f};  // the stencil cell's seam shift, in stencil_lookup's offset order
    if (shift_mode) {
        int rem = lane;
#pragma unroll
        for (int d = DIM - 1; d >= 0; --d) {
            const int32_t v = gc[d] + rem % 3 - 1;
            rem /= 3;
            if (lane < S && ((u.periodic_mask >> d) & 1))
                sh[d] = v < 0 ? -u.ext[d] : (v >= u.count[d] ? u.ext[d] : 0.f);
        }
    }
    const bool seam = shift_mode && __any_sync(0xffffffffu, sh[0] != 0.f || sh[1] != 0.f || sh[2] != 0.f);
    // runs: a stencil cell whose range continues the previous cell's (same shift) extends its run
    const int32_t inc = warp_inclusive_scan(cnt);
    const int32_t M = __shfl_sync(0xffffffffu, inc, 31);
    const int32_t pbeg = __shfl_up_sync(0xffffffffu, beg, 1);
    const int32_t pcnt = __shfl_up_sync(0xffffffffu, cnt, 1);
    bool cont = lane > 0 && pcnt > 0 && pbeg + pcnt == beg;
    if (shift_mode) {  // every lane takes part in the shuffles (no short-circuit around them)
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const float psh = __shfl_up_sync(0xffffffffu, sh[d], 1);
            cont = cont && psh == sh[d];
        }
    }
    const bool starts = cnt > 0 && !cont;
    const uint32_t smask = __ballot_sync(0xffffffffu, starts);
    const int32_t R = __popc(smask);
    const int rid = __popc(smask & ((1u << lane) - 1u));
    if (starts) {
        sm.run_beg[w][rid] = beg;
        sm.run_pre[w][rid] = inc - cnt;
        sm.shift[w][0][rid] = sh[0];
        sm.shift[w][1][rid] = sh[1];
        sm.shift[w][2][rid] = sh[2];
    }
    if (lane == 0) sm.run_pre[w][R] = M;
    // the unit's queries: a query whose own cell differs from the group's leaves for the serial path
    bool active = false;
    if (qlane) {
        const int32_t t = t0 + lane;
        active = TCR_IN(qorig, a.nq_total);
        if (active && (!a.no_stray_check || u.out_of_grid)) {
            int32_t qc[3];
            cell_of(DIM, u.dedupe, u.dmin, u.hcell, u.count, qv, qc);
            active = same_cell<DIM>(qc, gc);
        }
        if (!active) {  // own cell differs from the group's (aliasing or wrap rounding): serial path
            const int32_t k = atomicAdd(a.num_stray, 1);
            if (TCR_IN(k, a.nq_total)) a.stray[k] = t;
            qv = nan4;
        }
    }
    sm.qh[w][lane] = qv.w;
    sm.qid[w][lane] = qorig - u.qshift;
    sm.q[w][lane] = make_float4(qv.x, qv.y, qv.z, query_share<MODE>(qv.w));  // rows >= nb: NaN, never hit
    store_query_pair(sm.qp[w], lane, qv.x, qv.y, qv.z, packed_share<MODE>(qv.w));
    // the unit's record, reserved up front
    const int32_t nchunks = (M + 31) >> 5;
    bool stage = false;
    uint32_t* msk = nullptr;
    if (a.stage_cap > 0 && nchunks > 0) {
        const int64_t words = record_words(R, nchunks, nb);
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.cursor, (unsigned long long)words);
        base = __shfl_sync(0xffffffffu, base, 0);
        stage = base + (unsigned long long)words <= (unsigned long long)a.stage_cap;
        if (stage) {
            int32_t* rec = a.stage + base;
            if (lane == 0) {
                rec[0] = nchunks;
                rec[1] = R;
                rec[2] = nb;
                rec[3] = 0;
                rec[kRecHeader + 2 * R] = M;
                a.rec[unit] = (int32_t)base;
            }
            if (starts) {
                rec[kRecHeader + rid] = beg;
                rec[kRecHeader + R + rid] = inc - cnt;
            }
            msk = reinterpret_cast<uint32_t*>(rec + kRecHeader + 2 * R + 1);
        }
    }
    __syncwarp();
    // lane k of chunk c holds candidate 32c + k; its run only moves forward from chunk to chunk
    const int32_t* rpre = sm.run_pre[w];
    const int32_t* rbeg = sm.run_beg[w];
    const float4* __restrict__ rs = a.rsorted;
    int32_t cr = 0;
    const WrapCtx wc = wrap_ctx(u.periodic_mask, u.ext);
    const float qmax = u.qmax;
    const bool exact_all = u.exact_all != 0;
    const float dl = u.shift_delta;
    const float fe = u.f64_err;
    const int K4 = (nb + 3) & ~3;
    const float4* qsm = sm.q[w];
    uint32_t count = 0;
    // The fast pass takes the chunks two at a time (each lane tests its candidate of both against
    // every query, reading each query pair once) and streams them into a four-slot ring in shared
    // memory by cp.async, a pair of chunks ahead of its use, so the loads' latency hides behind the
    // tests without holding registers.  Lanes past the unit's candidates get NaN (never a hit).
    float4* ring = &sm.ring[w][0][0];
    auto issue = [&](int32_t c) {
        const int32_t k = (c << 5) + lane;
        float4* dst = ring + (c & 3) * 32 + lane;
        bool copied = false;
        if (k < M) {
            while (rpre[cr + 1] <= k) ++cr;
            const int32_t j = rbeg[cr] + (k - rpre[cr]);
            if (TCR_GUARD(j, a.nr_total)) {
                cp_async16(dst, &rs[j]);
                copied = true;
            }
        }
        if (!copied) *dst = nan4;
        cp_async_commit();
        return cr;
    };
    // one landed chunk: the candidate (shifted across a seam for the fast test) and its bands
    auto take = [&](int32_t c, int32_t crn, float4& cv, float& cw, float& band, float& band_exact) {
        cv = ring[(c & 3) * 32 + lane];
        if (PERIODIC && shift_mode) {
            cv.x += sm.shift[w][0][crn];
            if (DIM > 1) cv.y += sm.shift[w][1][crn];
            if (DIM > 2) cv.z += sm.shift[w][2][crn];
        }
        cw = cand_share<MODE>(cv.w);
        const float t = cand_tmax<MODE>(cw, qmax);
        band = exact_all ? inf : kBandEps * t * t;
        // float64 inputs: the band also covers the rounding of the coordinates to float32
        if (fe > 0.0f) band += fmaf(2.0f * 1.7320508f * t, fe, 3.0f * fe * fe);
        band_exact = band;
        // shifted candidates: the band also covers the shift's rounding (|d2 error| <= 2 T delta + delta^2)
        if (seam) band += fmaf(2.0f * t, dl, dl * dl);
    };
    // some pair of a chunk lies within the band: the chunk again, every pair in the band decided by
    // the reference's exact test on the original (unshifted) candidates
    auto exact = [&](int32_t c, int32_t crn, float band_exact) {
        if (lane == 0) atomicAdd(a.num_exact, 1);
        const int32_t k = (c << 5) + lane;
        float4 v0 = nan4;
        int32_t j = 0;
        if (k < M) {
            j = rbeg[crn] + (k - rpre[crn]);
            if (TCR_GUARD(j, a.nr_total)) v0 = __ldg(&rs[j]);
        }
        return chunk_hits_exact<DIM, MODE>(unit_exact_ctx(u, MODE), qsm, sm.qh[w], sm.qid[w], K4, v0, j, band_exact,
                                           a.f64);
    };
    auto store = [&](int32_t c, uint32_t m) {
        if (lane < nb) {
            count += __popc(m);
            if (stage && TCR_IN((int64_t)(msk - reinterpret_cast<uint32_t*>(a.stage)) + c * nb + lane, a.stage_cap))
                msk[c * nb + lane] = m;
        }
    };
    int32_t cr0 = issue(0);  // runs of the candidates of chunks c and c + 1 (seam shifts)
    int32_t cr1 = issue(1);
    for (int32_t c = 0; c < nchunks; c += 2) {
        const int32_t cr2 = issue(c + 2), cr3 = issue(c + 3);
        cp_async_wait<2>();  // chunks c and c + 1 have landed
        const bool two = c + 1 < nchunks;  // (past the last chunk the ring holds NaN: no hits)
        float4 cv0, cv1;
        float cw0, cw1, band0, band1, bx0, bx1;
        take(c, cr0, cv0, cw0, band0, bx0);
        take(c + 1, cr1, cv1, cw1, band1, bx1);
        uint32_t hit0, hit1 = 0;
        bool in0 = false, in1 = false;  // some pair of this lane's candidate lies within the band
        if (MODE != kSuperSymmetric && (!PERIODIC || shift_mode)) {
            float umin0 = inf, umin1 = inf;
            chunk_hits_x2_two<DIM, MODE>(sm.qp[w], K4, cv0, cw0, cv1, cw1, umin0, umin1, hit0, hit1);
            in0 = umin0 <= band0;
            in1 = umin1 <= band1;
        } else if (shift_mode) {
            hit0 = chunk_hits<DIM, false, MODE>(wc, qsm, K4, cv0, cw0, band0, in0);
            if (two) hit1 = chunk_hits<DIM, false, MODE>(wc, qsm, K4, cv1, cw1, band1, in1);
        } else {
            hit0 = chunk_hits<DIM, PERIODIC, MODE>(wc, qsm, K4, cv0, cw0, band0, in0);
            if (two) hit1 = chunk_hits<DIM, PERIODIC, MODE>(wc, qsm, K4, cv1, cw1, band1, in1);
        }
        if (__any_sync(0xffffffffu, in0)) hit0 = exact(c, cr0, bx0);
        if (two && __any_sync(0xffffffffu, in1)) hit1 = exact(c + 1, cr1, bx1);
        // the two transposes are independent, so their shuffle chains overlap
        const uint32_t m0 = warp_transpose32(hit0, lane);
        const uint32_t m1 = warp_transpose32(hit1, lane);
        store(c, m0);
        if (two) store(c + 1, m1);
        cr0 = cr2;
        cr1 = cr3;
    }
    if (active) a.counts[qorig] = (int32_t)count;
    if (lane == 0 && !stage && TCR_IN(unit, a.nq_total)) {
        a.rec[unit] = -1;
        if (nchunks > 0) {  // not staged: the emit walk tests the unit again
            const int32_t f = atomicAdd(a.num_flagged, 1);
            if (TCR_IN(f, a.nq_total)) a.flagged[f] = unit;
        }
    }
    __syncwarp();
}

// Class (dim * 2 + any periodic dim) of a cloud, the key of the walk kernels' template.
__device__ __forceinline__ int cloud_class(const CloudParams& cp) { return cp.dim * 2 + (cp.periodic_mask ? 1 : 0); }

// Next units of a warp.  Without a class filter one unit per atomic; with one (a batch that mixes
// classes runs one launch per class) a chunk of 32 consecutive units, of which the units of other
// classes are dropped by one ballot -- units of a cloud are consecutive, so chunks rarely mix.
__device__ __forceinline__ uint32_t next_units(const WalkArgs& a, int32_t* counter, const int32_t* list,
                                               int32_t nlist, int lane, int32_t& base) {
    const bool filter = a.class_filter >= 0;
    int32_t b = 0;
    if (lane == 0) b = atomicAdd(counter, filter ? 32 : 1);
    base = __shfl_sync(0xffffffffu, b, 0);
    if (base >= nlist) return 0u;
    if (!filter) return 1u;
    bool mine = false;
    if (base + lane < nlist) {
        const int32_t unit = list ? list[base + lane] : base + lane;
        const int32_t grp = a.unit_group[unit];
        mine = cloud_class(a.table[a.group_cloud[grp]]) == a.class_filter;
    }
    return __ballot_sync(0xffffffffu, mine);  // bit k: unit base + k belongs to this launch
}

template <int DIM, bool PERIODIC, int MODE>
__global__ void __launch_bounds__(kWalkWarps * 32, PERIODIC ? kWalkMinBlocksPeriodic : kWalkMinBlocks)
    walk_count_kernel(WalkArgs a) {
    __shared__ WalkSmem sm;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int32_t nunits = *a.num_units;
    int32_t* counter = &a.work[a.class_filter >= 0 ? 2 + a.class_filter : 0];
    int cur = -1;
    const bool filter = a.class_filter >= 0;
    int32_t claim = 0;
    if (lane == 0) claim = atomicAdd(counter, filter ? 32 : 1);
    for (;;) {
        const int32_t base = __shfl_sync(0xffffffffu, claim, 0);
        if (base >= nunits) break;
        uint32_t todo = 1u;
        if (filter) {  // a chunk of 32 consecutive units; the units of other classes are dropped
            bool mine = false;
            if (base + lane < nunits) mine = cloud_class(a.table[a.group_cloud[a.unit_group[base + lane]]]) ==
                                             a.class_filter;
            todo = __ballot_sync(0xffffffffu, mine);
        }
        // the next claim is issued before this one's units run and read after them, so the
        // atomic's latency overlaps their work
        if (lane == 0) claim = atomicAdd(counter, filter ? 32 : 1);
        while (todo) {
            const int32_t unit = base + (__ffs(todo) - 1);
            todo &= todo - 1;
            const int32_t grp = a.unit_group[unit];
            const int cloud = a.num_clouds == 1 ? 0 : a.group_cloud[grp];
            if (cloud != cur) {
                __syncwarp();
                if (lane == 0) load_unit_ctx(sm.u[w], a, cloud);
                cur = cloud;
                __syncwarp();
            }
            if (sm.u[w].error) {  // no grid: nothing found, nothing staged
                if (lane == 0) a.rec[unit] = -1;
                continue;
            }
            count_unit<DIM, PERIODIC, MODE>(a, sm, unit, grp, lane, w);
        }
    }
}

struct EmitSmem {
    int32_t pre[kWalkWarps][33];
    int32_t beg[kWalkWarps][32];
    float4 q[kWalkWarps][32];
    UnitCtx u[kWalkWarps];
};

// Emit walk of one unit that was not staged: walk again and write the pairs straight to their slots.
template <int DIM, bool PERIODIC, int MODE>
__device__ __forceinline__ void emit_unit(const WalkArgs& a, EmitSmem& sm, int32_t unit, int32_t grp, int lane,
                                          int w) {
    constexpr int S = DIM == 1 ? 3 : (DIM == 2 ? 9 : 27);
    const UnitCtx& u = sm.u[w];
    const WrapCtx wc = wrap_ctx(u.periodic_mask, u.ext);
    const float qmax = u.qmax;
    const bool exact_all = u.exact_all != 0;
    const unsigned lt = (1u << lane) - 1u;
    const float4 nan4 = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
    const int32_t t0 = a.unit_t0[unit];
    const int32_t nb = min(*a.unit_cap, a.group_start[grp + 1] - t0);
    const int32_t gc[3] = {a.group_coords[3 * grp], a.group_coords[3 * grp + 1], a.group_coords[3 * grp + 2]};
    int32_t beg = 0, cnt = 0;
    if (lane < S) stencil_lookup(a, u, gc, lane, beg, cnt);
    const int32_t inc = warp_inclusive_scan(cnt);
    sm.pre[w][lane + 1] = inc;
    if (lane == 0) sm.pre[w][0] = 0;
    sm.beg[w][lane] = beg;
    const int32_t M = __shfl_sync(0xffffffffu, inc, 31);
    int32_t qorig = 0;
    float4 qv = nan4;
    int64_t obase = 0;
    if (lane < nb) {
        const int32_t t = t0 + lane;
        qv = a.qsorted[t];
        qorig = a.qsidx[t];
        int32_t qc[3];
        cell_of(DIM, u.dedupe, u.dmin, u.hcell, u.count, qv, qc);
        if (same_cell<DIM>(qc, gc)) obase = a.offsets[qorig];
        else qv = nan4;  // stray: written by the serial kernel
    }
    sm.q[w][lane] = qv;
    __syncwarp();
    for (int32_t base = 0; base < M; base += 32) {
        const int32_t k = base + lane;
        float4 cv = nan4;
        int32_t j = 0;
        if (k < M) {
            j = cand_index(sm.pre[w], sm.beg[w], S, k);
            if (TCR_GUARD(j, a.nr_total)) cv = __ldg(&a.rsorted[j]);
            else j = 0;
        }
        int32_t jl = __ldg(&a.rsidx[j]);
        jl = a.ref_ids ? __ldg(&a.ref_ids[jl]) : jl - u.rshift;
        const int64_t jorig = (int64_t)jl;
        const float cw = cand_share<MODE>(cv.w);
        float band = exact_all ? __int_as_float(0x7f800000) : cand_band<MODE>(cw, qmax);
        if (u.f64_err > 0.0f) {  // float64 inputs: the coordinates' rounding to float32 widens the band
            const float t = cand_tmax<MODE>(cw, qmax), fe = u.f64_err;
            band += fmaf(2.0f * 1.7320508f * t, fe, 3.0f * fe * fe);
        }
        for (int qi = 0; qi < nb; ++qi) {
            const float4 q = sm.q[w][qi];
            bool in, unc;
            lean_test<DIM, PERIODIC, MODE>(wc, q, cv, cw, band, in, unc);
            const uint32_t ub = __ballot_sync(0xffffffffu, unc);
            int32_t qrow = __shfl_sync(0xffffffffu, qorig, qi);
            if (ub && unc)
                in = a.f64.qpos ? f64_pair_decide(a.f64, DIM, u.periodic_mask, MODE, qrow - u.qshift, j)
                                : exact_pair_test(unit_exact_ctx(u, MODE), q, q.w, cv, cv.w);
            const uint32_t b = __ballot_sync(0xffffffffu, in);
            const int64_t qb = __shfl_sync(0xffffffffu, obase, qi);
            qrow = a.query_ids ? __ldg(&a.query_ids[qrow]) : qrow - u.qshift;
            if (in) {
                const int64_t pos = qb + __popc(b & lt);
                if (pos < a.out_cap) {
                    a.col_out[pos] = jorig;
                    if (a.row_out) a.row_out[pos] = (int64_t)qrow;
                }
            }
            if (lane == qi) obase += __popc(b);
        }
    }
    __syncwarp();
}

template <int DIM, bool PERIODIC, int MODE>
__global__ void __launch_bounds__(kWalkWarps * 32) walk_emit_kernel(WalkArgs a) {
    __shared__ EmitSmem sm;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int32_t nlist = *a.num_list;
    if (nlist == 0) return;  // every unit was staged: no claim atomics at all
    int32_t* counter = a.class_filter >= 0 ? &a.work[8 + a.class_filter] : &a.work[1];
    int cur = -1;
    for (;;) {
        int32_t base;
        uint32_t todo = next_units(a, counter, a.unit_list, nlist, lane, base);
        if (base >= nlist) break;
        while (todo) {
            const int32_t unit = a.unit_list[base + (__ffs(todo) - 1)];
            todo &= todo - 1;
            const int32_t grp = a.unit_group[unit];
            const int cloud = a.num_clouds == 1 ? 0 : a.group_cloud[grp];
            if (cloud != cur) {
                __syncwarp();
                if (lane == 0) load_unit_ctx(sm.u[w], a, cloud);
                cur = cloud;
                __syncwarp();
            }
            if (sm.u[w].error) continue;
            emit_unit<DIM, PERIODIC, MODE>(a, sm, unit, grp, lane, w);
        }
    }
}

// Position of the highest set bit of a non-zero word (one bfind).
__device__ __forceinline__ uint32_t top_set_bit(uint32_t m) {
    uint32_t b;
    asm("bfind.u32 %0, %1;" : "=r"(b) : "r"(m));
    return b;
}

// Emit pass for staged units: expand each unit's record into its queries' CSR/COO slots, one warp
// per unit, window by window of kExpandWin chunks.  The window's candidate columns are gathered
// into shared memory once (consecutive sorted indices: coalesced reads of the sort index; each
// lane finds its candidate's run by a rank in the window's run-start bitmap).  Lanes over
// (query, chunk) pairs -- lane = query + nbp * g takes chunk g of each group of 32 / nbp chunks,
// nbp the unit's query count rounded up to a power of two -- expand their hit bits into a shared
// output table (query, chunk and bit of every output, in output order), and lanes over output
// positions write consecutive slots.  A window of more than kExpandTab outputs is written query by
// query instead.
constexpr int kExpandWarps = 8;
constexpr int kExpandWin = 16;    // chunks per window: 512 candidates
constexpr int kExpandTab = 1920;  // outputs one table holds (four blocks of eight warps fit an SM)
constexpr int kExpandBatch = 8;   // global loads a lane issues before it waits for the first
struct ExpandSmem {
    int32_t col[kExpandWarps][kExpandWin * 32];    // output column of each candidate of the window
    uint16_t tab[kExpandWarps][kExpandTab];        // (query << 9) | (chunk << 5) | bit, in output order
    uint32_t rstart[kExpandWarps][kExpandWin];     // bit k of word c: a run starts at candidate 32 c + k
    int32_t rrank[kExpandWarps][kExpandWin];       // runs starting before word c, minus one
    int32_t run_beg[kExpandWarps][32];
    int32_t run_pre[kExpandWarps][33];
    long long* qcol[kExpandWarps][32];             // column output of table entry 0 of each query (this window)
    int64_t qoff[kExpandWarps][32];                // output position of each query's next hit
    int32_t qrow[kExpandWarps][32];
};

struct ExpandArgs {
    const int32_t* __restrict__ stage;
    const int32_t* __restrict__ rec;
    const int32_t* __restrict__ num_units;
    const int32_t* __restrict__ unit_t0;
    const int32_t* __restrict__ unit_group;
    const int32_t* __restrict__ group_cloud;
    const int32_t* __restrict__ qsidx;
    const int32_t* __restrict__ rsidx;
    const int64_t* __restrict__ offsets;
    const int32_t* __restrict__ query_ids;
    const int32_t* __restrict__ ref_ids;
    const CloudParams* __restrict__ table;
    int32_t num_clouds;
    int32_t local_index;
    int64_t* __restrict__ row_out;
    int64_t* __restrict__ col_out;
    int64_t out_cap;
    int64_t stage_cap, nq, nr;  // bounds of the checked build
};

__global__ void __launch_bounds__(kExpandWarps * 32, 4) expand_records_kernel(ExpandArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ExpandSmem& sm = *reinterpret_cast<ExpandSmem*>(smem_raw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int32_t nu = *a.num_units;
    const int64_t warps = (int64_t)gridDim.x * kExpandWarps;
    int32_t* __restrict__ rbeg = sm.run_beg[w];
    int32_t* __restrict__ rpre = sm.run_pre[w];
    int32_t* __restrict__ cols = sm.col[w];
    uint16_t* __restrict__ tab = sm.tab[w];
    int64_t u = (int64_t)blockIdx.x * kExpandWarps + w;
    // A unit's record offset and first query are read two iterations before it runs, its record
    // header (lanes 0..2) and query rows (lane < 32 covers every unit size) one iteration before,
    // so a unit starts with its header at hand instead of two dependent round trips.
    auto header = [&](int32_t r0) -> int32_t {
        return (r0 >= 0 && lane < 3 && TCR_GUARD(r0 + 3, a.stage_cap)) ? a.stage[r0 + lane] : 0;
    };
    auto qrows = [&](int64_t v, int32_t t0) -> int32_t {
        return (v < nu && TCR_GUARD(t0 + lane, a.nq)) ? a.qsidx[t0 + lane] : -1;
    };
    int32_t r0a = u < nu ? a.rec[u] : -1, t0a = u < nu ? a.unit_t0[u] : 0;
    int32_t r0b = u + warps < nu ? a.rec[u + warps] : -1, t0b = u + warps < nu ? a.unit_t0[u + warps] : 0;
    int32_t ha = header(r0a), qa = qrows(u, t0a);
    for (; u < nu; u += warps) {
        const int32_t r0 = r0a, hw = ha, qrow_l = qa;
        ha = header(r0b);
        qa = qrows(u + warps, t0b);
        r0a = r0b;
        t0a = t0b;
        r0b = -1;
        if (u + 2 * warps < nu) {
            r0b = a.rec[u + 2 * warps];
            t0b = a.unit_t0[u + 2 * warps];
        }
        if (r0 < 0) continue;  // no candidates, or re-tested by the emit walk
        if (!TCR_GUARD(r0 + 3, a.stage_cap)) continue;
        const int32_t* rec = a.stage + r0;
        const int32_t nchunks = __shfl_sync(0xffffffffu, hw, 0), R = __shfl_sync(0xffffffffu, hw, 1),
                      nb = __shfl_sync(0xffffffffu, hw, 2);
        if (!TCR_GUARD(R, 28) || !TCR_GUARD(nb - 1, 32) || !TCR_GUARD(r0 + record_words(R, nchunks, nb) - 1, a.stage_cap))
            continue;
        const uint32_t* masks = reinterpret_cast<const uint32_t*>(rec + kRecHeader + 2 * R + 1);
        int32_t rshift = 0, qshift = 0;
        if (a.local_index) {
            const CloudParams& cp = a.table[a.num_clouds == 1 ? 0 : a.group_cloud[a.unit_group[u]]];
            rshift = cp.ref_base;
            qshift = cp.query_base;
        }
        if (lane < R) rbeg[lane] = rec[kRecHeader + lane];
        if (lane <= R) rpre[lane] = rec[kRecHeader + R + lane];
        if (lane < nb && TCR_GUARD(qrow_l, a.nq)) {
            sm.qrow[w][lane] = a.query_ids ? a.query_ids[qrow_l] : qrow_l - qshift;
            sm.qoff[w][lane] = a.offsets[qrow_l];
        }
        __syncwarp();
        const int32_t M = rpre[R];
        // lane = q + nbp * g: query q, chunk g of each group of G chunks
        const int lg = nb > 1 ? 32 - __clz(nb - 1) : 0;
        const int nbp = 1 << lg, G = 32 >> lg;
        const int q = lane & (nbp - 1), g = lane >> lg;
        const bool qlane = q < nb;
        for (int32_t c0 = 0; c0 < nchunks; c0 += kExpandWin) {
            const int32_t nc = min(kExpandWin, nchunks - c0);
            const int32_t wbase = c0 << 5;
            // the window's masks, in registers: lane (q, g) holds the masks of chunks g, g + G, ...
            // (G = 1 when the unit has more than 16 queries), all loaded at the window's start;
            // consecutive lanes read consecutive words
            const uint32_t* src = masks + (int64_t)c0 * nb;
            uint32_t mv[kExpandWin];
#pragma unroll
            for (int t = 0; t < kExpandWin; ++t) {
                const int32_t c = g + G * t;
                mv[t] = (qlane && c < nc) ? __ldcs(&src[c * nb + q]) : 0u;
            }
            // run of candidate wbase + k: the runs starting at or before it, minus one
            if (lane < kExpandWin) sm.rstart[w][lane] = 0u;
            __syncwarp();
            const bool rl = lane < R;
            const int32_t rs = rl ? rpre[lane] - wbase : -1;
            const int32_t nbefore = __popc(__ballot_sync(0xffffffffu, rl && rs < 0));
            if (rl && rs >= 0 && rs < (nc << 5)) atomicOr(&sm.rstart[w][rs >> 5], 1u << (rs & 31));
            __syncwarp();
            const int32_t wp = lane < kExpandWin ? __popc(sm.rstart[w][lane]) : 0;
            const int32_t wpi = warp_inclusive_scan(wp);
            if (lane < kExpandWin) sm.rrank[w][lane] = nbefore + wpi - wp - 1;
            __syncwarp();
            // the window's candidate columns, the loads of each batch issued together so that their
            // latencies overlap (one load waited for at a time left the warps idle)
            const uint32_t le = (2u << lane) - 1u;  // bits 0 .. lane
            for (int32_t cc0 = 0; cc0 < nc; cc0 += kExpandBatch) {
                int32_t jl[kExpandBatch];
                bool ok[kExpandBatch];
#pragma unroll
                for (int i = 0; i < kExpandBatch; ++i) {
                    const int32_t cc = cc0 + i;
                    const int32_t k = wbase + (cc << 5) + lane;
                    jl[i] = 0;
                    ok[i] = false;
                    if (cc < nc && k < M) {
                        const int32_t cr = sm.rrank[w][cc] + __popc(sm.rstart[w][cc] & le);
                        if (TCR_GUARD(cr, R)) {
                            const int32_t j = rbeg[cr] + (k - rpre[cr]);
                            ok[i] = true;
                            if (TCR_GUARD(j, a.nr)) jl[i] = __ldg(&a.rsidx[j]);
                        }
                    }
                }
                int32_t col[kExpandBatch];
#pragma unroll
                for (int i = 0; i < kExpandBatch; ++i)
                    col[i] = !ok[i] ? 0 : (a.ref_ids ? __ldg(&a.ref_ids[jl[i]]) : jl[i] - rshift);
#pragma unroll
                for (int i = 0; i < kExpandBatch; ++i)
                    if (cc0 + i < nc) cols[((cc0 + i) << 5) + lane] = col[i];
            }
            __syncwarp();
            // the window's outputs of each query, and their exclusive prefix over the queries
            int32_t tot = 0;
#pragma unroll
            for (int t = 0; t < kExpandWin; ++t) tot += __popc(mv[t]);
            for (int sft = nbp; sft < 32; sft <<= 1) tot += __shfl_xor_sync(0xffffffffu, tot, sft);
            const int32_t tv = (g == 0 && qlane) ? tot : 0;
            const int32_t tinc = warp_inclusive_scan(tv);
            const int32_t n = __shfl_sync(0xffffffffu, tinc, 31);
            const int32_t qpre = __shfl_sync(0xffffffffu, tinc - tv, q);
            if (n <= kExpandTab) {
                // each lane expands its (query, chunk) mask into the table, highest bit at the end
                int32_t run = qpre;  // table slot of the query's next output
#pragma unroll
                for (int t = 0; t < kExpandWin; ++t) {
                    if (G * t >= nc) break;
                    const int32_t c = G * t + g;
                    uint32_t m = mv[t];
                    int32_t inc = __popc(m);
                    for (int sft = nbp; sft < 32; sft <<= 1) {  // inclusive scan over g, per query
                        const int32_t t = __shfl_up_sync(0xffffffffu, inc, sft);
                        if (lane >= sft) inc += t;
                    }
                    const int32_t tq = __shfl_sync(0xffffffffu, inc, q + 32 - nbp);
                    int32_t pos = run + inc;
                    const uint32_t tag = ((uint32_t)q << 9) | ((uint32_t)c << 5);
                    while (m) {
                        const uint32_t bit = top_set_bit(m);
                        m ^= 1u << bit;
                        tab[--pos] = (uint16_t)(tag | bit);
                    }
                    run += tq;
                }
                // per query: the output slot of its table entry 0, and whether all of the window's
                // outputs fit the output buffer (then the column-only loop writes without checks)
                bool fits = true;
                if (g == 0 && qlane) {
                    sm.qcol[w][q] = reinterpret_cast<long long*>(a.col_out) + (sm.qoff[w][q] - qpre);
                    fits = sm.qoff[w][q] + tot <= a.out_cap;
                }
                fits = __all_sync(0xffffffffu, fits);
                __syncwarp();
                const bool rows = a.row_out != nullptr;
                if (fits && !rows) {
#pragma unroll 4
                    for (int32_t o = lane; o < n; o += 32) {
                        const uint32_t v = tab[o];
                        __stcs(sm.qcol[w][v >> 9] + o, (long long)cols[v & 0x1ffu]);
                    }
                } else if (fits) {  // COO: the row of an output sits at the same slot of row_out
                    const int64_t rd = ((intptr_t)a.row_out - (intptr_t)a.col_out) / 8;  // both int64-aligned
#pragma unroll 4
                    for (int32_t o = lane; o < n; o += 32) {
                        const uint32_t v = tab[o];
                        const uint32_t vq = v >> 9;
                        long long* p = sm.qcol[w][vq] + o;
                        __stcs(p, (long long)cols[v & 0x1ffu]);
                        __stcs(p + rd, (long long)sm.qrow[w][vq]);
                    }
                } else {
#pragma unroll 4
                    for (int32_t o = lane; o < n; o += 32) {
                        const uint32_t v = tab[o];
                        const uint32_t vq = v >> 9;
                        const int64_t pos = (sm.qcol[w][vq] - reinterpret_cast<long long*>(a.col_out)) + o;
                        if (TCR_GUARD(pos, a.out_cap)) {
                            __stcs(reinterpret_cast<long long*>(&a.col_out[pos]), (long long)cols[v & 0x1ffu]);
                            if (rows) __stcs(reinterpret_cast<long long*>(&a.row_out[pos]), (long long)sm.qrow[w][vq]);
                        }
                    }
                }
            } else {
                // many outputs: query by query, lanes over the window's chunks
                for (int32_t qq = 0; qq < nb; ++qq) {
                    uint32_t m = lane < nc ? __ldcs(&src[lane * nb + qq]) : 0u;
                    const int32_t cnt = __popc(m);
                    const int32_t inc = warp_inclusive_scan(cnt);
                    int64_t pos = sm.qoff[w][qq] + (inc - cnt);
                    const long long row = sm.qrow[w][qq];
                    while (m) {
                        const int bit = __ffs(m) - 1;
                        m &= m - 1;
                        if (TCR_GUARD(pos, a.out_cap)) {
                            a.col_out[pos] = (int64_t)cols[(lane << 5) + bit];
                            if (a.row_out) a.row_out[pos] = row;
                        }
                        ++pos;
                    }
                }
            }
            __syncwarp();
            if (g == 0 && qlane) sm.qoff[w][q] += tot;
            __syncwarp();
        }
    }
}

// Serial walk for queries whose own cell differs from their group's (one thread per query).
template <bool EMIT>
__global__ void stray_kernel(WalkArgs a) {
    const int32_t ns = *a.num_stray;
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
        const int32_t t = a.stray[s];
        const float4 q = a.qsorted[t];
        const int32_t qorig = a.qsidx[t];
        UnitCtx u;
        load_unit_ctx(u, a, cloud_of(a.query_prefix, a.num_clouds, qorig));
        if (u.error) continue;
        const int S = u.dim == 1 ? 3 : (u.dim == 2 ? 9 : 27);
        const ExactCtx xc = unit_exact_ctx(u, a.mode);
        int32_t qc[3];
        cell_of(u.dim, u.dedupe, u.dmin, u.hcell, u.count, q, qc);
        int64_t pos = EMIT ? a.offsets[qorig] : 0;
        int32_t n = 0;
        for (int o = 0; o < S; ++o) {
            int32_t beg, cnt;
            stencil_lookup(a, u, qc, o, beg, cnt);
            for (int32_t j = beg; j < beg + cnt; ++j) {
                const float4 cv = a.rsorted[j];
                const bool in = a.f64.qpos ? f64_pair_decide(a.f64, u.dim, u.periodic_mask, a.mode, qorig - u.qshift, j)
                                           : exact_pair_test(xc, q, q.w, cv, cv.w);
                if (in) {
                    if (EMIT) {
                        if (pos < a.out_cap) {
                            const int32_t jl = a.rsidx[j];
                            a.col_out[pos] = (int64_t)(a.ref_ids ? a.ref_ids[jl] : jl - u.rshift);
                            if (a.row_out) a.row_out[pos] = a.query_ids ? a.query_ids[qorig] : qorig - u.qshift;
                        }
                        ++pos;
                    } else {
                        ++n;
                    }
                }
            }
        }
        if (!EMIT) a.counts[qorig] = n;
    }
}

// ------------------------------------------------------------------------------------------
// float64 inputs (the reference dispatches its operators on float and double,
// neighborhoodDynamic_cpu.cpp:504,531).  The structure is built from float32 copies with a cell
// size no smaller than the reference's double one, so every pair within the double support lies
// in the query's 3^d stencil; the walks then test candidates on the float32 copies with a band
// widened by the copies' rounding, and every pair inside the band is decided on the caller's double
// positions and supports by the reference's double expression.
struct F64Args {
    const double* qpos;  // [nq * dim], wrapped as the reference wraps queries
    const double* qsup;  // [nq] or null
    const double* rpos;  // [nr * dim], reference j at row j, wrapped as the reference wraps references
    const double* rsup;  // [nr] or null
    double4* rsorted;    // [nr] the references in the structure's cell order, .w = support
    double ext[3];       // max - min of the domain, in double
    int64_t nq, nr;
};

static F64Walk f64_walk(const F64Args& f) {
    F64Walk w;
    w.qpos = f.qpos;
    w.qsup = f.qsup;
    w.rsorted = f.rsorted;
    for (int d = 0; d < 3; ++d) w.ext[d] = f.ext[d];
    return w;
}

// The double references in cell order (a stencil cell's candidates are one contiguous run), and the
// largest |coordinate| of the double positions (NaN ignored, rounded up) for the band of the float
// test.
__global__ void f64_prep_kernel(const int32_t* __restrict__ rsidx, F64Args f, int dim, QueryParams* qp) {
    float m = 0.0f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < f.nr; j += stride) {
        const int64_t jl = rsidx[j];
        double4 v = make_double4(0.0, 0.0, 0.0, f.rsup ? f.rsup[jl] : 0.0);
        v.x = f.rpos[jl * dim];
        if (dim > 1) v.y = f.rpos[jl * dim + 1];
        if (dim > 2) v.z = f.rpos[jl * dim + 2];
        f.rsorted[j] = v;
        m = fmaxf(m, __double2float_ru(fmax(fabs(v.x), fmax(fabs(v.y), fabs(v.z)))));
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < f.nq * dim; i += stride)
        m = fmaxf(m, __double2float_ru(fabs(f.qpos[i])));
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(&qp->coord_key, float_key(m));
}

// counts -> offsets (int64, nq+1), optional CSR indptr (int32) and rowEntries (int64).
struct CountIn {
    const int32_t* counts;
    int64_t n;
    __device__ int64_t operator()(int64_t i) const { return i < n ? (int64_t)counts[i] : 0; }
};
struct OffsetOut {
    int64_t n;
    int64_t* offsets;
    int32_t* indptr;
    int64_t* entries;
    __device__ void operator()(int64_t i, int64_t ex, int64_t v) const {
        offsets[i] = ex;
        if (indptr) indptr[i] = (int32_t)ex;
        if (entries && i < n) entries[i] = v;
    }
};

__global__ void info_kernel(const int32_t* bad_grids, const int64_t* total, const int32_t* num_stray,
                            const int32_t* exact_clouds, const unsigned long long* cursor, const int32_t* num_flagged,
                            const int32_t* num_exact, const int32_t* inc_count, int64_t n_ref, int64_t* info) {
    info[0] = *total;
    info[1] = *bad_grids;
    info[2] = *num_stray;
    info[3] = *exact_clouds;
    info[4] = (int64_t)*cursor;
    info[5] = *num_flagged;
    info[6] = *num_exact;
    // incremental build: points sorted by the small sort (-1: the full sort ran); -2: no hint
    info[7] = inc_count ? ((inc_count[1] != 0 || 2 * (int64_t)inc_count[0] < n_ref) ? -1 : n_ref - inc_count[0]) : -2;
}

// ------------------------------------------------------------------------------------------
// host orchestration

// One search as the kernels see it: the cloud table plus what holds for all clouds.
struct HostBatch {
    int32_t C = 0, mode = 0, self = 0, local_index = 0;
    std::vector<CloudParams> clouds;
    int64_t nq = 0, nr = 0, map_total = 0;
    const int32_t* query_ids = nullptr;
    const int32_t* ref_ids = nullptr;
    bool any_query_sup = false, any_ref_sup = false;
    bool same_sorted = false;     // self search, no periodic dims, queries are the references (same arrays)
    bool same_positions = false;  // self search, no periodic dims, same position arrays
    int walk_class = 0;           // dim * 2 + (any periodic dim) when every cloud shares it, else 0
    uint32_t class_mask = 0;      // bit cls: some cloud with queries has class cls
    bool wide = false;            // 64-bit (cloud, cell) sort keys
    const int32_t* lin_hint = nullptr;  // incremental build: previous linear cell of every reference point
    int32_t* lin_out = nullptr;         // receives the linear cell of every sorted reference point
    int32_t* order_out = nullptr;       // receives the input index of every sorted reference point
    int unit_cap = kDefaultUnitQueries;           // queries per work unit
    int walk_bps = kDefaultWalkBlocksPerSM;       // resident walk blocks per SM
};

// The descriptors' tuning fields (0: default).
static int take_tuning(HostBatch& b, int32_t unit_queries, int32_t walk_blocks_per_sm) {
    if (unit_queries != 0 && unit_queries != 8 && unit_queries != 16 && unit_queries != 32)
        return set_error(TCR_ERR_INVALID, "unit_queries must be 8, 16 or 32 (0: default 32)");
    if (walk_blocks_per_sm < 0 || walk_blocks_per_sm > 64)
        return set_error(TCR_ERR_INVALID, "walk_blocks_per_sm must be in [1, 64] (0: default 12)");
    b.unit_cap = unit_queries ? unit_queries : kDefaultUnitQueries;
    b.walk_bps = walk_blocks_per_sm ? walk_blocks_per_sm : kDefaultWalkBlocksPerSM;
    return TCR_OK;
}

// Validation shared by both descriptors.  level 0: sizes only; 1: query phases (the reference
// supports come from the structure); 2: structure build.
static int check_cloud(const char* who, int dim, int mode, int64_t L, int64_t nq, int64_t nr, const void* qpos,
                       const void* qsup, const void* rpos, const void* rsup, int self, int level) {
    if (dim < 1 || dim > 3) return set_error(TCR_ERR_INVALID, "%sdim must be 1, 2 or 3 (got %d)", who, dim);
    if (mode < 0 || mode > 3) return set_error(TCR_ERR_INVALID, "%sinvalid mode %d", who, mode);
    if (nq < 0 || nr < 0 || nq > 0x7fffffffLL || nr > 0x7ffffff0LL)
        return set_error(TCR_ERR_INVALID, "%spoint counts must be in [0, 2^31)", who);
    if (self && nq != nr) return set_error(TCR_ERR_INVALID, "%sself search needs one cloud", who);
    if (level == 0) return TCR_OK;
    if (L <= 0 || L > 0xffffffffLL) return set_error(TCR_ERR_INVALID, "%shashMapLength must be in [1, 2^32)", who);
    if ((nq && !qpos) || (nr && !rpos)) return set_error(TCR_ERR_INVALID, "%smissing positions", who);
    if ((mode == kGather || mode == kSymmetric || mode == kSuperSymmetric) && nq && !qsup)
        return set_error(TCR_ERR_INVALID, "%sthis mode needs query supports", who);
    if (level >= 2 && (mode == kScatter || mode == kSymmetric || mode == kSuperSymmetric) && nr && !rsup)
        return set_error(TCR_ERR_INVALID, "%sthis mode needs reference supports", who);
    return TCR_OK;
}

static int finish_batch(HostBatch& b, int64_t map_min) {
    int64_t qb = 0, rb = 0, mb = 0;
    bool same_pos = b.self != 0, same_sorted = b.self != 0;
    int cls = -1;
    bool mixed = false;
    b.any_query_sup = b.any_ref_sup = false;
    b.class_mask = 0;
    for (CloudParams& cp : b.clouds) {
        cp.query_base = (int32_t)qb;
        cp.ref_base = (int32_t)rb;
        qb += cp.n_query;
        rb += cp.n_ref;
        if (qb > 0x7ffffff0LL || rb > 0x7ffffff0LL)
            return set_error(TCR_ERR_INVALID, "the clouds hold more than 2^31 query or reference points");
        cp.map_cap = hash_capacity(cp.n_ref, map_min);
        cp.map_base = mb;
        mb += cp.map_cap;
        same_pos = same_pos && cp.periodic_mask == 0 && cp.query_pos == cp.ref_pos;
        same_sorted = same_sorted && cp.periodic_mask == 0 && cp.query_pos == cp.ref_pos && cp.query_sup == cp.ref_sup;
        b.any_query_sup = b.any_query_sup || cp.query_sup != nullptr;
        b.any_ref_sup = b.any_ref_sup || cp.ref_sup != nullptr;
        const int c = cp.dim * 2 + (cp.periodic_mask != 0 ? 1 : 0);
        if (cls < 0) cls = c;
        else if (c != cls) mixed = true;
        if (cp.n_query > 0) b.class_mask |= 1u << c;
    }
    b.nq = qb;
    b.nr = rb;
    b.map_total = mb;
    b.same_positions = same_pos;
    b.same_sorted = same_sorted;
    b.walk_class = mixed ? 0 : cls;
    b.wide = b.C > 1;
    return TCR_OK;
}

static void fill_domain(CloudParams& cp, int dim, const float* lo, const float* hi) {
    for (int k = 0; k < 3; ++k) {
        cp.dmin[k] = k < dim ? lo[k] : 0.f;
        cp.dmax[k] = k < dim ? hi[k] : 1.f;
        cp.ext[k] = cp.dmax[k] - cp.dmin[k];
    }
}

static int batch_of_desc(const tcr_search_desc* d, int level, HostBatch& b) {
    if (!d) return set_error(TCR_ERR_INVALID, "null descriptor");
    int rc = check_cloud("", d->dim, d->mode, d->hash_map_length, d->n_query, d->n_ref, d->query_pos, d->query_sup,
                         d->ref_pos, d->ref_sup, d->self_search, level);
    if (rc) return rc;
    if (d->hcell[0] > 0.0f)
        for (int k = 0; k < d->dim; ++k)
            if (!(d->hcell[k] > 0.0f) || !(d->hcell[k] < 3.0e38f))
                return set_error(TCR_ERR_INVALID, "cell size override must be positive and finite in every dimension");
    CloudParams cp;
    memset(&cp, 0, sizeof(cp));
    cp.dim = d->dim;
    cp.mode = d->mode;
    cp.periodic_mask = d->periodic_mask;
    cp.hash_len = (uint32_t)d->hash_map_length;
    fill_domain(cp, d->dim, d->domain_min, d->domain_max);
    for (int k = 0; k < 3; ++k) cp.hcell_override[k] = d->hcell[0] > 0.0f ? (k < d->dim ? d->hcell[k] : 1.0f) : 0.0f;
    cp.dedupe = d->clamped_grid ? 1 : 0;
    cp.n_query = (int32_t)d->n_query;
    cp.n_ref = (int32_t)d->n_ref;
    cp.query_pos = d->query_pos;
    cp.query_sup = d->query_sup;
    cp.ref_pos = d->ref_pos;
    cp.ref_sup = d->ref_sup;
    b = HostBatch();
    b.C = 1;
    b.mode = d->mode;
    b.self = d->self_search ? 1 : 0;
    b.query_ids = d->query_ids;
    b.ref_ids = d->ref_ids;
    b.clouds.push_back(cp);
    if ((rc = take_tuning(b, d->unit_queries, d->walk_blocks_per_sm))) return rc;
    return finish_batch(b, kSingleMapMin);
}

static int batch_of(const tcr_batch_desc* bd, int level, HostBatch& b) {
    if (!bd) return set_error(TCR_ERR_INVALID, "null batch descriptor");
    if (bd->n_clouds < 1 || bd->n_clouds > (1 << 22))
        return set_error(TCR_ERR_INVALID, "n_clouds must be in [1, 2^22] (got %d)", bd->n_clouds);
    if (!bd->clouds) return set_error(TCR_ERR_INVALID, "missing cloud table");
    b = HostBatch();
    b.C = bd->n_clouds;
    b.mode = bd->mode;
    b.self = bd->self_search ? 1 : 0;
    b.local_index = bd->local_index ? 1 : 0;
    b.query_ids = bd->query_ids;
    b.ref_ids = bd->ref_ids;
    b.lin_hint = bd->ref_lin_hint;
    b.lin_out = bd->ref_lin_out;
    b.order_out = bd->ref_order_out;
    b.clouds.resize(bd->n_clouds);
    if (int rc = take_tuning(b, bd->unit_queries, bd->walk_blocks_per_sm)) return rc;
    char who[48];
    for (int k = 0; k < bd->n_clouds; ++k) {
        const tcr_cloud_desc& c = bd->clouds[k];
        snprintf(who, sizeof(who), "cloud %d: ", k);
        int rc = check_cloud(who, c.dim, bd->mode, c.hash_map_length, c.n_query, c.n_ref, c.query_pos, c.query_sup,
                             c.ref_pos, c.ref_sup, bd->self_search, level);
        if (rc) return rc;
        if (level >= 1 && c.hcell[0] > 0.0f)
            for (int d = 0; d < c.dim; ++d)
                if (!(c.hcell[d] > 0.0f) || !(c.hcell[d] < 3.0e38f))
                    return set_error(TCR_ERR_INVALID, "%scell size override must be positive and finite", who);
        CloudParams& cp = b.clouds[k];
        memset(&cp, 0, sizeof(cp));
        cp.dim = c.dim;
        cp.mode = bd->mode;
        cp.periodic_mask = c.periodic_mask & ((1 << c.dim) - 1);
        for (int d = 0; d < 3; ++d) cp.hcell_override[d] = c.hcell[0] > 0.0f ? (d < c.dim ? c.hcell[d] : 1.0f) : 0.0f;
        cp.dedupe = c.clamped_grid ? 1 : 0;
        cp.hash_len = (uint32_t)c.hash_map_length;
        fill_domain(cp, c.dim, c.domain_min, c.domain_max);
        cp.n_query = (int32_t)c.n_query;
        cp.n_ref = (int32_t)c.n_ref;
        cp.query_pos = c.query_pos;
        cp.query_sup = c.query_sup;
        cp.ref_pos = c.ref_pos;
        cp.ref_sup = c.ref_sup;
    }
    return finish_batch(b, kBatchMapMin);
}

static void batch_sizes(const HostBatch& b, int64_t* s, int64_t* w) {
    if (s) carve_structure(nullptr, b.nr, b.C, b.map_total, s);
    if (w) carve_scratch(nullptr, b.nq, b.nr, b.C, b.lin_hint != nullptr, w);
}

static inline unsigned grid_for(int64_t n, int threads, int max_blocks = 148 * 16) {
    int64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, max_blocks));
}

static int num_sms() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

// Optional per-launch timing of the two heaviest kernels (count walk, record expansion): events
// recorded around the launch on its own stream; read back with tcr_profile_kernel_ms.
static std::mutex g_prof_mu;
static int g_prof_on = 0;
static int g_prof_dev = -1;
static cudaEvent_t g_prof_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
static int g_prof_recorded[2] = {0, 0};

static void prof_mark(int kernel, int end, cudaStream_t st) {
    if (!g_prof_on) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != g_prof_dev) return;
    // External: under stream capture the record becomes an event node of the graph, so replays
    // of a recorded search time the kernel too
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return;
    const unsigned flags = cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
    if (cudaEventRecordWithFlags(g_prof_ev[kernel][end], st, flags) == cudaSuccess && end) g_prof_recorded[kernel] = 1;
}

static int upload_table(const HostBatch& b, const Scratch& W, cudaStream_t st) {
    for (int first = 0; first < b.C; first += kUploadChunk) {
        CloudChunk ch;
        memset(&ch, 0, sizeof(ch));
        ch.first = first;
        ch.count = std::min(kUploadChunk, b.C - first);
        ch.n_clouds = b.C;
        ch.query_total = (int32_t)b.nq;
        ch.ref_total = (int32_t)b.nr;
        memcpy(ch.p, &b.clouds[first], sizeof(CloudParams) * ch.count);
        upload_clouds_kernel<<<1, 32, 0, st>>>(ch, W.table, W.query_prefix, W.ref_prefix);
        note_launches(1);
    }
    TCR_CUDA(cudaGetLastError());
    return TCR_OK;
}

static WalkArgs make_walk(const HostBatch& b, const Structure& S, const Scratch& W) {
    WalkArgs a;
    memset(&a, 0, sizeof(a));
    a.table = W.table;
    a.grid = S.grid;
    a.qparams = W.qparams;
    a.query_prefix = W.query_prefix;
    a.num_clouds = b.C;
    a.local_index = b.local_index;
    a.mode = b.mode;
    a.no_stray_check = b.same_positions ? 1 : 0;
    a.rsorted = S.rsorted;
    a.rsidx = S.rsidx;
    a.cell_start = S.cell_start;
    a.cell_bucket = S.cell_bucket;
    a.map = S.map;
    a.qsorted = b.same_sorted ? S.rsorted : W.qsorted;
    a.qsidx = b.same_sorted ? S.rsidx : W.qsidx;
    a.group_start = b.self ? S.cell_start : W.qgroup_start;
    a.group_coords = b.self ? S.cell_coords : W.qgroup_coords;
    a.group_cloud = b.self ? S.cell_cloud : W.qgroup_cloud;
    a.unit_group = W.unit_group;
    a.unit_t0 = W.unit_t0;
    a.num_units = W.num_units;
    a.unit_cap = W.unit_cap;
    a.unit_list = W.flagged;
    a.num_list = W.num_flagged;
    a.work = W.work;
    a.stray = W.stray;
    a.num_stray = W.num_stray;
    a.counts = W.counts;
    a.rec = W.rec;
    a.flagged = W.flagged;
    a.num_flagged = W.num_flagged;
    a.num_exact = W.num_exact;
    a.cursor = W.cursor;
    a.query_ids = b.query_ids;
    a.ref_ids = b.ref_ids;
    a.nq_total = b.nq;
    a.nr_total = b.nr;
    return a;
}

// Dispatches a walk kernel template on a cloud class (dim * 2 + any periodic dim) and the mode.
template <template <int, bool, int> class L>
static cudaError_t dispatch_walk(const WalkArgs& a, int cls, int mode, dim3 grid, dim3 block, size_t smem,
                                 cudaStream_t st) {
#define TCR_M(D, P)                                                                    \
    switch (mode) {                                                                    \
        case kGather: return L<D, P, kGather>::launch(a, grid, block, smem, st);       \
        case kScatter: return L<D, P, kScatter>::launch(a, grid, block, smem, st);     \
        case kSymmetric: return L<D, P, kSymmetric>::launch(a, grid, block, smem, st); \
        default: return L<D, P, kSuperSymmetric>::launch(a, grid, block, smem, st);    \
    }
    switch (cls) {
        case 2: TCR_M(1, false)
        case 3: TCR_M(1, true)
        case 4: TCR_M(2, false)
        case 5: TCR_M(2, true)
        case 6: TCR_M(3, false)
        default: TCR_M(3, true)
    }
#undef TCR_M
}

// Raises a kernel's dynamic shared memory limit once per device (not a stream operation, so a
// search can be recorded into a CUDA graph after its first eager run).
template <typename F>
static cudaError_t ensure_smem(F* kernel, int bytes, uint64_t* done_mask) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if (__atomic_load_n(done_mask, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) __atomic_fetch_or(done_mask, bit, __ATOMIC_ACQ_REL);
    return e;
}

template <int D, bool P, int M>
struct CountLaunch {
    static cudaError_t launch(const WalkArgs& a, dim3 g, dim3 b, size_t, cudaStream_t st) {
        walk_count_kernel<D, P, M><<<g, b, 0, st>>>(a);
        return cudaGetLastError();
    }
};
template <int D, bool P, int M>
struct EmitLaunch {
    static cudaError_t launch(const WalkArgs& a, dim3 g, dim3 b, size_t, cudaStream_t st) {
        walk_emit_kernel<D, P, M><<<g, b, 0, st>>>(a);
        return cudaGetLastError();
    }
};

// One walk launch for a batch of one class; one per class present (each filtering its units)
// when the clouds mix classes.
template <template <int, bool, int> class L>
static cudaError_t launch_walks(const HostBatch& b, WalkArgs a, dim3 grid, dim3 block, size_t smem,
                                cudaStream_t st) {
    if (b.walk_class != 0) {
        a.class_filter = -1;
        note_launches(1);
        return dispatch_walk<L>(a, b.walk_class, b.mode, grid, block, smem, st);
    }
    for (int cls = 2; cls <= 7; ++cls) {
        if (!((b.class_mask >> cls) & 1)) continue;
        a.class_filter = cls;
        note_launches(1);
        cudaError_t e = dispatch_walk<L>(a, cls, b.mode, grid, block, smem, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Persistent walk grid: the blocks loop over units through an atomic counter, so the size only
// sets the parallelism -- about two units per query group's worth of full units per warp.
static unsigned walk_blocks(const HostBatch& b, int64_t nq) {
    const int64_t max_units = 2 * nq / b.unit_cap + 1;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)num_sms() * b.walk_bps,
                                                            (max_units + kWalkWarps - 1) / kWalkWarps));
}

template <typename K>
static int build_impl(const HostBatch& b, const Structure& S, const Scratch& W, cudaStream_t st) {
    const SortWorkspaceT<K> sw = sort_workspace<K>(W);
    const int C = b.C;
    const int64_t nr = b.nr, nq = b.nq;
    int rc = upload_table(b, W, st);
    if (rc) return rc;
    grid_init_kernel<K><<<grid_for(C, 128), 128, 0, st>>>(S.grid, C, S, W);
    note_launches(1);
    // computeGridSupport: which supports set hMax depends on the mode
    if (b.any_ref_sup && nr > 0) {
        support_stats_kernel<<<grid_for(nr, 256, num_sms() * 4), 256, 0, st>>>(
            W.table, W.ref_prefix, C, nr, 0, reinterpret_cast<char*>(S.grid) + offsetof(GridParams, ref_stats),
            (int64_t)sizeof(GridParams));
        note_launches(1);
    }
    if (b.any_query_sup && nq > 0 && !b.same_sorted) {
        support_stats_kernel<<<grid_for(nq, 256, num_sms() * 4), 256, 0, st>>>(
            W.table, W.query_prefix, C, nq, 1,
            reinterpret_cast<char*>(S.grid) + offsetof(GridParams, build_query_stats), (int64_t)sizeof(GridParams));
        note_launches(1);
    }
    grid_params_kernel<<<grid_for(C, 128), 128, 0, st>>>(W.table, S.grid, C, S.bad_grids, b.same_sorted ? 1 : 0);
    note_launches(1);
    TCR_CUDA(cudaMemsetAsync(S.map, 0xff, sizeof(unsigned long long) * S.map_total, st));
    if (nr > 0) {
        const bool inc = b.lin_hint != nullptr;
        // few blocks: each ends with one atomic on the key range, so thousands of them would queue
        pack_points_kernel<K><<<grid_for(nr, 256, num_sms() * 4), 256, 0, st>>>(
            W.table, S.grid, W.ref_prefix, C, nr, 0, 2, 1, W.pack, sw.keys[0], sw.vals[0], sw.state,
            inc ? b.lin_hint : nullptr, inc ? W.stay : nullptr);
        note_launches(1);
        if (inc) {
            SortWorkspaceT<K> mw = sw;
            mw.keys[0] = reinterpret_cast<K*>(W.moved_keys[0]);
            mw.keys[1] = reinterpret_cast<K*>(W.moved_keys[1]);
            mw.vals[0] = W.moved_vals[0];
            mw.vals[1] = W.moved_vals[1];
            mw.state = reinterpret_cast<SortStateT<K>*>(W.moved_state);
            TCR_CUDA(cudaMemsetAsync(W.inc_count, 0, 2 * sizeof(int32_t), st));
            StayOut<K> so{sw.keys[0], reinterpret_cast<K*>(W.stay_keys), W.stay_idx, mw.keys[0], mw.vals[0]};
            TCR_CUDA(device_exclusive_scan<int32_t>(StayIn{W.stay}, so, nr, W.scan_tiles32, W.inc_count, st));
            inc_check_kernel<K><<<grid_for(nr, 256), 256, 0, st>>>(reinterpret_cast<const K*>(W.stay_keys),
                                                                   W.inc_count, W.inc_count + 1);
            inc_decide_kernel<K><<<1, 1, 0, st>>>(sw.state, mw.state, W.inc_count, nr);
            note_launches(2);
            TCR_CUDA(radix_sort_pairs<K>(mw, nr, st));
            inc_merge_kernel<K><<<grid_for(nr, 256), 256, 0, st>>>(
                reinterpret_cast<const K*>(W.stay_keys), W.stay_idx, mw.keys[0], mw.keys[1], mw.vals[0], mw.vals[1],
                mw.state, W.inc_count, nr, sw.keys[0], sw.vals[0]);
            note_launches(1);
        }
        TCR_CUDA(radix_sort_pairs<K>(sw, nr, st, SortedPointsOut<K>{W.pack, S.rsorted, S.rsidx, b.lin_out, b.order_out, nr}));
        gather_sorted_kernel<K><<<grid_for(nr, 256), 256, 0, st>>>(W.pack, sw.vals[0], sw.vals[1], sw.state, nr,
                                                                   S.rsorted, S.rsidx, sw.keys[0], sw.keys[1],
                                                                   b.lin_out, b.order_out);
        note_launches(1);
        RunFlagIn<K> fi{sw.keys[0], sw.keys[1], sw.state};
        TCR_CUDA(device_exclusive_scan<int32_t>(fi, CellStartOut{S.cell_start, (int32_t)nr}, nr, W.scan_tiles32,
                                                S.num_cells, st));
        CellOut<K> co{W.table, S.grid, sw.keys[0], sw.keys[1], sw.state, S.rsorted, S.cell_start, S.cell_lin,
                      S.cell_coords, S.cell_bucket, S.cell_cloud, S.map, (int32_t)nr};
        cell_records_kernel<K><<<grid_for(nr, 256, num_sms() * 8), 256, 0, st>>>(co, S.num_cells, nr);
    } else {
        finish_cells_kernel<<<1, 1, 0, st>>>(S.cell_start, S.num_cells, nr);
    }
    note_launches(1);
    TCR_CUDA(cudaGetLastError());
    return TCR_OK;
}

template <typename K>
static int count_impl(const HostBatch& b, const Structure& S, const Scratch& W, int32_t* stage, int64_t stage_cap,
                      int64_t* offsets, int32_t* indptr_out, int64_t* row_entries_out, int64_t* info_out,
                      cudaStream_t st, const F64Args* f64) {
    const int C = b.C;
    const int64_t nq = b.nq;
    int rc = upload_table(b, W, st);
    if (rc) return rc;
    const int unit_cap = b.unit_cap;
    count_init_kernel<<<grid_for(std::max<int64_t>(C, nq), 256), 256, 0, st>>>(W, C, unit_cap, nq);
    note_launches(1);
    if (b.any_query_sup && nq > 0 && !b.same_sorted) {
        support_stats_kernel<<<grid_for(nq, 256, num_sms() * 4), 256, 0, st>>>(
            W.table, W.query_prefix, C, nq, 1, reinterpret_cast<char*>(W.qparams) + offsetof(QueryParams, stats),
            (int64_t)sizeof(QueryParams));
        note_launches(1);
    }
    query_params_kernel<<<grid_for(C, 128), 128, 0, st>>>(W.table, S.grid, C, W.qparams, W.exact_clouds,
                                                          b.same_sorted ? 1 : 0);
    note_launches(1);
    if (f64 && (b.nr > 0 || nq > 0)) {
        f64_prep_kernel<<<grid_for(std::max<int64_t>(b.nr, nq * b.clouds[0].dim), 256), 256, 0, st>>>(
            S.rsidx, *f64, b.clouds[0].dim, W.qparams);
        note_launches(1);
    }
    if (nq > 0) {
        const int32_t* gstart;
        const int32_t* ngroups;
        if (b.self) {
            if (!b.same_sorted) {
                pack_self_queries_kernel<<<grid_for(nq, 256), 256, 0, st>>>(W.table, S.grid, W.query_prefix, C, S.rsidx,
                                                                            nq, W.qsorted, W.qsidx);
                note_launches(1);
            }
            gstart = S.cell_start;
            ngroups = S.num_cells;
        } else {
            // sort the queries by their own (cloud, cell)
            const SortWorkspaceT<K> sw = sort_workspace<K>(W);
            sort_state_init_kernel<K><<<1, 1, 0, st>>>(sw.state);
            note_launches(1);
            pack_points_kernel<K><<<grid_for(nq, 256, num_sms() * 4), 256, 0, st>>>(
                W.table, S.grid, W.query_prefix, C, nq, 1, 1, 0, W.pack, sw.keys[0], sw.vals[0], sw.state);
            note_launches(1);
            TCR_CUDA(radix_sort_pairs<K>(sw, nq, st));
            gather_sorted_kernel<K><<<grid_for(nq, 256), 256, 0, st>>>(W.pack, sw.vals[0], sw.vals[1], sw.state, nq,
                                                                       W.qsorted, W.qsidx);
            note_launches(1);
            QueryGroupOut<K> qo{W.table, S.grid, sw.keys[0], sw.keys[1], sw.state, W.qsorted,
                                W.qgroup_start, W.qgroup_coords, W.qgroup_cloud, (int32_t)nq};
            RunFlagIn<K> fi{sw.keys[0], sw.keys[1], sw.state};
            TCR_CUDA(device_exclusive_scan<int32_t>(fi, qo, nq, W.scan_tiles32, W.num_qgroups, st));
            finish_cells_kernel<<<1, 1, 0, st>>>(W.qgroup_start, W.num_qgroups, nq);
            note_launches(1);
            gstart = W.qgroup_start;
            ngroups = W.num_qgroups;
        }
        BoundedUnitCountIn ui{gstart, ngroups, unit_cap};
        BoundedUnitOut uo{gstart, ngroups, W.unit_group, W.unit_t0, unit_cap, nq};
        TCR_CUDA(device_exclusive_scan<int32_t>(ui, uo, nq, W.scan_tiles32, W.num_units, st));
        WalkArgs a = make_walk(b, S, W);
        if (f64) a.f64 = f64_walk(*f64);
        a.stage = stage;
        a.stage_cap = stage_cap;
        prof_mark(TCR_PROFILE_COUNT_WALK, 0, st);
        TCR_CUDA(launch_walks<CountLaunch>(b, a, dim3(walk_blocks(b, nq)), dim3(kWalkWarps * 32), 0, st));
        prof_mark(TCR_PROFILE_COUNT_WALK, 1, st);
        stray_kernel<false><<<grid_for(nq, 128, num_sms() * 4), 128, 0, st>>>(a);
        note_launches(1);
    }
    CountIn ci{W.counts, nq};
    OffsetOut oo{nq, offsets, indptr_out, row_entries_out};
    TCR_CUDA(device_exclusive_scan<int64_t>(ci, oo, nq + 1, W.scan_tiles64, W.total, st));
    info_kernel<<<1, 1, 0, st>>>(S.bad_grids, W.total, W.num_stray, W.exact_clouds, W.cursor, W.num_flagged,
                                 W.num_exact, b.lin_hint && b.nr > 0 ? W.inc_count : nullptr, b.nr, W.info);
    note_launches(1);
    if (info_out) TCR_CUDA(cudaMemcpyAsync(info_out, W.info, 8 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    return TCR_OK;
}

static int emit_impl(const HostBatch& b, const Structure& S, const Scratch& W, const int32_t* stage,
                     const int64_t* offsets, int64_t* row_out, int64_t* col_out, int64_t out_capacity,
                     cudaStream_t st, const F64Args* f64) {
    const int64_t nq = b.nq;
    if (out_capacity < 0 || (out_capacity > 0 && !col_out)) return set_error(TCR_ERR_INVALID, "bad output buffer");
    if (nq <= 0) return TCR_OK;
    WalkArgs a = make_walk(b, S, W);
    if (f64) a.f64 = f64_walk(*f64);
    a.offsets = offsets;
    a.row_out = row_out;
    a.col_out = col_out;
    a.out_cap = out_capacity;
    if (stage) {
        const int nsm = num_sms();
        const unsigned blocks = (unsigned)std::max<int64_t>(
            1, std::min<int64_t>((int64_t)nsm * 16, (nq / 16 + kExpandWarps) / kExpandWarps));
        ExpandArgs e;
        e.stage = stage;
        e.rec = W.rec;
        e.num_units = W.num_units;
        e.unit_t0 = W.unit_t0;
        e.unit_group = W.unit_group;
        e.group_cloud = a.group_cloud;
        e.qsidx = a.qsidx;
        e.rsidx = S.rsidx;
        e.offsets = offsets;
        e.query_ids = b.query_ids;
        e.ref_ids = b.ref_ids;
        e.table = W.table;
        e.num_clouds = b.C;
        e.local_index = b.local_index;
        e.row_out = row_out;
        e.col_out = col_out;
        e.out_cap = out_capacity;
        e.stage_cap = 0x7fffffffLL;  // the records lie below the staging capacity of tcr_count (< 2^31 words)
        e.nq = nq;
        e.nr = b.nr;
        static uint64_t expand_attr_done = 0;
        TCR_CUDA(ensure_smem(expand_records_kernel, (int)sizeof(ExpandSmem), &expand_attr_done));
        prof_mark(TCR_PROFILE_EXPAND, 0, st);
        expand_records_kernel<<<blocks, kExpandWarps * 32, sizeof(ExpandSmem), st>>>(e);
        prof_mark(TCR_PROFILE_EXPAND, 1, st);
        note_launches(1);
    }
    TCR_CUDA(cudaMemsetAsync(W.work, 0, sizeof(int32_t) * kWorkCounters, st));
    TCR_CUDA(launch_walks<EmitLaunch>(b, a, dim3(walk_blocks(b, nq)), dim3(kWalkWarps * 32), 0, st));
    stray_kernel<true><<<grid_for(nq, 128, num_sms() * 4), 128, 0, st>>>(a);
    note_launches(1);
    return TCR_OK;
}

static int run_build(const HostBatch& b, void* structure, int64_t structure_bytes, void* scratch,
                     int64_t scratch_bytes, void* stream) {
    int64_t need_s = 0, need_w = 0;
    batch_sizes(b, &need_s, &need_w);
    if (!structure || !scratch || structure_bytes < need_s || scratch_bytes < need_w)
        return set_error(TCR_ERR_INVALID, "workspace too small (structure %lld/%lld, scratch %lld/%lld)",
                         (long long)structure_bytes, (long long)need_s, (long long)scratch_bytes, (long long)need_w);
    const Structure S = carve_structure(structure, b.nr, b.C, b.map_total, nullptr);
    const Scratch W = carve_scratch(scratch, b.nq, b.nr, b.C, b.lin_hint != nullptr, nullptr);
    cudaStream_t st = (cudaStream_t)stream;
    return b.wide ? build_impl<unsigned long long>(b, S, W, st) : build_impl<uint32_t>(b, S, W, st);
}

static int run_count(const HostBatch& b, const void* structure, void* scratch, int64_t scratch_bytes, int32_t* stage,
                     int64_t stage_capacity, int64_t* offsets, int32_t* indptr_out, int64_t* row_entries_out,
                     int64_t* info_out, void* stream, const F64Args* f64 = nullptr) {
    int64_t need_w = 0;
    batch_sizes(b, nullptr, &need_w);
    if (!structure || !scratch || scratch_bytes < need_w || !offsets)
        return set_error(TCR_ERR_INVALID, "workspace too small or offsets missing");
    if (stage_capacity < 0 || stage_capacity > 0x7fffffffLL || (stage_capacity > 0 && !stage))
        return set_error(TCR_ERR_INVALID, "stage capacity must be in [0, 2^31) with a buffer");
    const Structure S = carve_structure(const_cast<void*>(structure), b.nr, b.C, b.map_total, nullptr);
    const Scratch W = carve_scratch(scratch, b.nq, b.nr, b.C, b.lin_hint != nullptr, nullptr);
    cudaStream_t st = (cudaStream_t)stream;
    return b.wide ? count_impl<unsigned long long>(b, S, W, stage, stage_capacity, offsets, indptr_out,
                                                   row_entries_out, info_out, st, f64)
                  : count_impl<uint32_t>(b, S, W, stage, stage_capacity, offsets, indptr_out, row_entries_out,
                                         info_out, st, f64);
}

static int run_emit(const HostBatch& b, const void* structure, void* scratch, int64_t scratch_bytes,
                    const int32_t* stage, const int64_t* offsets, int64_t* row_out, int64_t* col_out,
                    int64_t out_capacity, void* stream, const F64Args* f64 = nullptr) {
    int64_t need_w = 0;
    batch_sizes(b, nullptr, &need_w);
    if (!structure || !scratch || scratch_bytes < need_w || !offsets)
        return set_error(TCR_ERR_INVALID, "workspace too small or offsets missing");
    const Structure S = carve_structure(const_cast<void*>(structure), b.nr, b.C, b.map_total, nullptr);
    const Scratch W = carve_scratch(scratch, b.nq, b.nr, b.C, b.lin_hint != nullptr, nullptr);
    return emit_impl(b, S, W, stage, offsets, row_out, col_out, out_capacity, (cudaStream_t)stream, f64);
}

}  // namespace tcr

using namespace tcr;

extern "C" {

const char* tcr_last_error(void) { return g_err; }

int tcr_version(void) { return TCR_ABI_VERSION; }

int64_t tcr_desc_bytes(void) { return (int64_t)sizeof(tcr_search_desc); }

int64_t tcr_cloud_desc_bytes(void) { return (int64_t)sizeof(tcr_cloud_desc); }

int64_t tcr_batch_desc_bytes(void) { return (int64_t)sizeof(tcr_batch_desc); }

int64_t tcr_kernel_launches(void) { return (int64_t)__atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int tcr_profile_kernels(int32_t enable) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!enable) {
        g_prof_on = 0;
        return TCR_OK;
    }
    int dev = 0;
    TCR_CUDA(cudaGetDevice(&dev));
    if (dev != g_prof_dev) {
        for (auto& pair : g_prof_ev)
            for (auto& e : pair) {
                if (e) cudaEventDestroy(e);
                e = nullptr;
            }
        for (auto& pair : g_prof_ev)
            for (auto& e : pair) TCR_CUDA(cudaEventCreate(&e));
        g_prof_dev = dev;
    }
    g_prof_recorded[0] = g_prof_recorded[1] = 0;
    g_prof_on = 1;
    return TCR_OK;
}

int tcr_profile_kernel_ms(int32_t kernel, float* ms) {
    if (kernel < 0 || kernel > 1 || !ms) return set_error(TCR_ERR_INVALID, "invalid kernel id or output");
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_recorded[kernel]) return set_error(TCR_ERR_INVALID, "no profiled launch of kernel %d", kernel);
    TCR_CUDA(cudaEventSynchronize(g_prof_ev[kernel][1]));
    TCR_CUDA(cudaEventElapsedTime(ms, g_prof_ev[kernel][0], g_prof_ev[kernel][1]));
    return TCR_OK;
}

#ifdef TCR_CHECKED
// Checked build only: the first failed bounds check (source line, index, bound), then cleared.
int tcr_debug_checks(int64_t* out3) {
    unsigned long long h[3] = {0, 0, 0};
    TCR_CUDA(cudaMemcpyFromSymbol(h, g_check, sizeof(h)));
    const unsigned long long z[3] = {0, 0, 0};
    TCR_CUDA(cudaMemcpyToSymbol(g_check, z, sizeof(z)));
    for (int k = 0; k < 3; ++k) out3[k] = (int64_t)h[k];
    return TCR_OK;
}
#endif

int tcr_search_sizes(int64_t n_query, int64_t n_ref, int32_t dim, int64_t* structure_bytes, int64_t* scratch_bytes) {
    if (dim < 1 || dim > 3 || n_query < 0 || n_ref < 0) return set_error(TCR_ERR_INVALID, "invalid sizes");
    if (structure_bytes) carve_structure(nullptr, n_ref, 1, hash_capacity(n_ref, kSingleMapMin), structure_bytes);
    if (scratch_bytes) carve_scratch(nullptr, n_query, n_ref, 1, false, scratch_bytes);
    return TCR_OK;
}

int tcr_structure_offsets(int64_t n_ref, int64_t* offsets, int32_t n) {
    if (n_ref < 0 || !offsets || n < TCR_STRUCT_NFIELDS) return set_error(TCR_ERR_INVALID, "invalid arguments");
    char* const base = reinterpret_cast<char*>(256);  // any non-null base; offsets are relative
    const Structure s = carve_structure(base, n_ref, 1, hash_capacity(n_ref, kSingleMapMin), nullptr);
    auto off = [&](const void* p) { return (int64_t)((const char*)p - base); };
    offsets[TCR_STRUCT_GRID] = off(s.grid);
    offsets[TCR_STRUCT_NUM_CELLS] = off(s.num_cells);
    offsets[TCR_STRUCT_SORTED_POINTS] = off(s.rsorted);
    offsets[TCR_STRUCT_SORT_INDEX] = off(s.rsidx);
    offsets[TCR_STRUCT_CELL_START] = off(s.cell_start);
    offsets[TCR_STRUCT_CELL_LIN] = off(s.cell_lin);
    offsets[TCR_STRUCT_CELL_COORDS] = off(s.cell_coords);
    offsets[TCR_STRUCT_CELL_BUCKET] = off(s.cell_bucket);
    offsets[TCR_STRUCT_MAP] = off(s.map);
    offsets[TCR_STRUCT_MAP_CAPACITY] = s.map_total;
    return TCR_OK;
}

int tcr_build_structure(const tcr_search_desc* d, void* structure, int64_t structure_bytes, void* scratch,
                        int64_t scratch_bytes, void* stream) {
    NvtxRange nvtx_("tcr_build_structure");
    HostBatch b;
    int rc = batch_of_desc(d, 2, b);
    if (rc) return rc;
    return run_build(b, structure, structure_bytes, scratch, scratch_bytes, stream);
}

int tcr_count(const tcr_search_desc* d, const void* structure, void* scratch, int64_t scratch_bytes, int32_t* stage,
              int64_t stage_capacity, int64_t* offsets, int32_t* indptr_out, int64_t* row_entries_out, int64_t* info_out,
              void* stream) {
    NvtxRange nvtx_("tcr_count");
    HostBatch b;
    int rc = batch_of_desc(d, 1, b);
    if (rc) return rc;
    return run_count(b, structure, scratch, scratch_bytes, stage, stage_capacity, offsets, indptr_out, row_entries_out,
                     info_out, stream);
}

int tcr_emit(const tcr_search_desc* d, const void* structure, void* scratch, int64_t scratch_bytes,
             const int32_t* stage, const int64_t* offsets, int64_t* row_out, int64_t* col_out, int64_t out_capacity,
             void* stream) {
    NvtxRange nvtx_("tcr_emit");
    HostBatch b;
    int rc = batch_of_desc(d, 1, b);
    if (rc) return rc;
    return run_emit(b, structure, scratch, scratch_bytes, stage, offsets, row_out, col_out, out_capacity, stream);
}

static int f64_args(const tcr_search_desc* d, const tcr_f64_inputs* in, F64Args& f) {
    if (!in) return set_error(TCR_ERR_INVALID, "missing float64 inputs");
    if ((d->n_query > 0 && !in->query_pos) || (d->n_ref > 0 && (!in->ref_pos || !in->ref_sorted)))
        return set_error(TCR_ERR_INVALID, "missing float64 positions or the sorted-reference workspace");
    if (d->mode != TCR_SCATTER && d->n_query > 0 && !in->query_sup)
        return set_error(TCR_ERR_INVALID, "this mode needs float64 query supports");
    if (d->mode != TCR_GATHER && d->n_ref > 0 && !in->ref_sup)
        return set_error(TCR_ERR_INVALID, "this mode needs float64 reference supports");
    if (d->hcell[0] <= 0.0f) return set_error(TCR_ERR_INVALID, "float64 searches need the cell size in hcell");
    if (d->clamped_grid) return set_error(TCR_ERR_INVALID, "float64 searches use the reference's unclamped grid");
    f.qpos = in->query_pos;
    f.qsup = in->query_sup;
    f.rpos = in->ref_pos;
    f.rsup = in->ref_sup;
    f.rsorted = reinterpret_cast<double4*>(in->ref_sorted);
    for (int k = 0; k < 3; ++k) f.ext[k] = in->domain_max[k] - in->domain_min[k];
    f.nq = d->n_query;
    f.nr = d->n_ref;
    return TCR_OK;
}

int tcr_count_f64(const tcr_search_desc* d, const tcr_f64_inputs* in, const void* structure, void* scratch,
                  int64_t scratch_bytes, int32_t* stage, int64_t stage_capacity, int64_t* offsets,
                  int32_t* indptr_out, int64_t* row_entries_out, int64_t* info_out, void* stream) {
    NvtxRange nvtx_("tcr_count_f64");
    HostBatch b;
    int rc = batch_of_desc(d, 1, b);
    if (rc) return rc;
    F64Args f;
    rc = f64_args(d, in, f);
    if (rc) return rc;
    return run_count(b, structure, scratch, scratch_bytes, stage, stage_capacity, offsets, indptr_out, row_entries_out,
                     info_out, stream, &f);
}

int tcr_emit_f64(const tcr_search_desc* d, const tcr_f64_inputs* in, const void* structure, void* scratch,
                 int64_t scratch_bytes, const int32_t* stage, const int64_t* offsets, int64_t* row_out,
                 int64_t* col_out, int64_t out_capacity, void* stream) {
    NvtxRange nvtx_("tcr_emit_f64");
    HostBatch b;
    int rc = batch_of_desc(d, 1, b);
    if (rc) return rc;
    F64Args f;
    rc = f64_args(d, in, f);
    if (rc) return rc;
    return run_emit(b, structure, scratch, scratch_bytes, stage, offsets, row_out, col_out, out_capacity, stream, &f);
}

int tcr_batch_sizes(const tcr_batch_desc* bd, int64_t* structure_bytes, int64_t* scratch_bytes) {
    HostBatch b;
    int rc = batch_of(bd, 0, b);
    if (rc) return rc;
    batch_sizes(b, structure_bytes, scratch_bytes);
    return TCR_OK;
}

int tcr_batch_build_structure(const tcr_batch_desc* bd, void* structure, int64_t structure_bytes, void* scratch,
                              int64_t scratch_bytes, void* stream) {
    NvtxRange nvtx_("tcr_batch_build_structure");
    HostBatch b;
    int rc = batch_of(bd, 2, b);
    if (rc) return rc;
    return run_build(b, structure, structure_bytes, scratch, scratch_bytes, stream);
}

int tcr_batch_count(const tcr_batch_desc* bd, const void* structure, void* scratch, int64_t scratch_bytes,
                    int32_t* stage, int64_t stage_capacity, int64_t* offsets, int32_t* indptr_out,
                    int64_t* row_entries_out, int64_t* info_out, void* stream) {
    NvtxRange nvtx_("tcr_batch_count");
    HostBatch b;
    int rc = batch_of(bd, 1, b);
    if (rc) return rc;
    return run_count(b, structure, scratch, scratch_bytes, stage, stage_capacity, offsets, indptr_out, row_entries_out,
                     info_out, stream);
}

int tcr_batch_emit(const tcr_batch_desc* bd, const void* structure, void* scratch, int64_t scratch_bytes,
                   const int32_t* stage, const int64_t* offsets, int64_t* row_out, int64_t* col_out,
                   int64_t out_capacity, void* stream) {
    NvtxRange nvtx_("tcr_batch_emit");
    HostBatch b;
    int rc = batch_of(bd, 1, b);
    if (rc) return rc;
    return run_emit(b, structure, scratch, scratch_bytes, stage, offsets, row_out, col_out, out_capacity, stream);
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Search without any device allocation.
//
// Some callers cannot allocate device memory at search time: a host application that hands the
// search a fixed memory arena at start-up and forbids cudaMalloc afterwards (cudaMalloc can
// synchronise the device and stall a real-time loop), or a plugin host whose allocator the
// search cannot reach.  tcr_search_noalloc serves them: the structure and the scratch of one
// whole search live in the file-scope device array below, so the caller passes only its inputs
// and its output buffers.  The array is kTcrStaticScratchBytes (32 MiB) on every GPU that loads
// this library, held until the process exits.
namespace tcr {
constexpr int64_t kTcrStaticScratchBytes = 32ll << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kTcrStaticScratchBytes];

constexpr int kMaxDevices = 64;
static void* g_static_ptr[kMaxDevices] = {nullptr};
static int g_static_err[kMaxDevices] = {0};
static std::once_flag g_static_once[kMaxDevices];

// Device address of g_static_scratch on the current device.  In host code the symbol's name is
// only a host-side stand-in, so the address is asked from the runtime, once per device, with that
// device current.
static int static_scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(TCR_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(TCR_ERR_INVALID, "device ordinal %d out of range", dev);
    std::call_once(g_static_once[dev], [dev]() {
        void* p = nullptr;
        cudaError_t r = cudaGetSymbolAddress(&p, g_static_scratch);
        if (r == cudaSuccess) g_static_ptr[dev] = p;
        else g_static_err[dev] = (int)r;
    });
    if (!g_static_ptr[dev])
        return set_error(TCR_ERR_CUDA, "cudaGetSymbolAddress(static scratch) failed on device %d: %s", dev,
                         cudaGetErrorString((cudaError_t)g_static_err[dev]));
    *out = g_static_ptr[dev];
    return TCR_OK;
}
}  // namespace tcr

extern "C" int tcr_search_noalloc(const tcr_search_desc* d, int64_t* offsets, int32_t* indptr_out,
                                  int64_t* row_entries_out, int64_t* row_out, int64_t* col_out,
                                  int64_t pair_capacity, int64_t* total_out, void* stream) {
    using namespace tcr;
    NvtxRange nvtx_("tcr_search_noalloc");
    HostBatch b;
    int rc = batch_of_desc(d, 2, b);
    if (rc) return rc;
    if (!offsets || (pair_capacity > 0 && !col_out) || pair_capacity < 0)
        return set_error(TCR_ERR_INVALID, "offsets and a column buffer of pair_capacity entries are required");
    int64_t s_bytes = 0, w_bytes = 0;
    batch_sizes(b, &s_bytes, &w_bytes);
    if (s_bytes + w_bytes > kTcrStaticScratchBytes)
        return set_error(TCR_ERR_INVALID,
                         "tcr_search_noalloc: %lld query and %lld reference points need %lld bytes of structure "
                         "and scratch, more than the static %lld bytes; use tcr_build_structure/tcr_count/tcr_emit "
                         "with caller-allocated buffers",
                         (long long)d->n_query, (long long)d->n_ref, (long long)(s_bytes + w_bytes),
                         (long long)kTcrStaticScratchBytes);
    void* base = nullptr;
    rc = static_scratch_address(&base);
    if (rc) return rc;
    void* structure = base;
    void* scratch = static_cast<char*>(base) + s_bytes;
    // The rest of the array is the staging list: units whose records fit are expanded by the emit
    // without being tested again.
    const int64_t stage_off = align256(s_bytes + w_bytes);
    const int64_t stage_words = std::min<int64_t>((kTcrStaticScratchBytes - stage_off) / 4, 0x7fffffff);
    int32_t* stage = stage_words > 0 ? reinterpret_cast<int32_t*>(static_cast<char*>(base) + stage_off) : nullptr;
    // Every kernel below initialises what it reads (counters, map, sort state), so the contents a
    // previous call left in the array do not matter.
    rc = tcr_build_structure(d, structure, s_bytes, scratch, w_bytes, stream);
    if (rc) return rc;
    int64_t info[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    rc = tcr_count(d, structure, scratch, w_bytes, stage, stage ? stage_words : 0, offsets, indptr_out,
                   row_entries_out, info, stream);
    if (rc) return rc;
    TCR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (total_out) *total_out = info[0];
    if (info[1]) return set_error(TCR_ERR_INVALID, "no valid cell grid for this domain and support");
    if (info[0] > pair_capacity)
        return set_error(TCR_ERR_INVALID, "tcr_search_noalloc: %lld pairs do not fit the %lld-entry output",
                         (long long)info[0], (long long)pair_capacity);
    if (info[0] == 0) return TCR_OK;
    return tcr_emit(d, structure, scratch, w_bytes, stage, offsets, row_out, col_out, pair_capacity, stream);
}
