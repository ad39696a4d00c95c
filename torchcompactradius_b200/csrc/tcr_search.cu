// tcr_search.cu -- compact-hashing fixed-radius neighbour search for sm_100a, with a C ABI.
//
// Pipeline (one CUDA stream, no host synchronisation inside a phase):
//   build:  support max-reduction -> grid parameters (compute_h) -> wrap + pack reference points
//           into float4 (x, y, z, h) and int32 linear cell keys -> stable radix sort ->
//           run-length cell table (begin, coords, bucket) + open-addressing lin -> cell map.
//   count:  query packing (self search reuses the reference order) -> query groups (cells) ->
//           work units of <= 32 queries -> warp-per-unit candidate walk over the 3^d stencil with
//           broadcast query positions and ballot counting -> device scan -> offsets.
//   emit:   the same walk writing int64 (row, col) pairs at the scanned offsets.
// The candidate set of every query is the reference's (cppSrc/neighborhood.h:73-132): the
// stencil cells of its own cell, found by linear index inside the bucket of the stencil cell's
// hash; the pair test is the reference's float test (tcr_common.cuh).
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <algorithm>
#include <mutex>

#include "tcr_common.cuh"
#include "tcr_scan.cuh"
#include "tcr_sort.cuh"
#include "../../include/tcr_b200.h"

namespace tcr {

// ------------------------------------------------------------------------------------------
// error reporting
static thread_local char g_err[512];
static int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}
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
static inline int64_t hash_capacity(int64_t n_ref) { return std::max<int64_t>(1024, next_pow2(2 * std::max<int64_t>(n_ref, 1))); }

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
    GridParams* grid;       // [1]
    float4* rsorted;        // [nr] wrapped reference points in cell order, .w = support
    int32_t* rsidx;         // [nr] original index of each sorted point
    int32_t* cell_start;    // [nr+1]
    int32_t* cell_lin;      // [nr]
    int32_t* cell_coords;   // [3*nr]
    int32_t* cell_bucket;   // [nr] ref hash of the cell's coordinates mod hashMapLength
    int32_t* num_cells;     // [1]
    unsigned long long* map;  // [H] (lin << 32 | cell), empty = ~0
    int64_t map_cap;
};

static Structure carve_structure(void* buf, int64_t nr, int64_t* bytes) {
    Carve c{(char*)buf, 0};
    Structure s;
    s.grid = c.take<GridParams>(1);
    s.num_cells = c.take<int32_t>(1);
    s.rsorted = c.take<float4>(nr);
    s.rsidx = c.take<int32_t>(nr);
    s.cell_start = c.take<int32_t>(nr + 1);
    s.cell_lin = c.take<int32_t>(nr);
    s.cell_coords = c.take<int32_t>(3 * nr);
    s.cell_bucket = c.take<int32_t>(nr);
    s.map_cap = hash_capacity(nr);
    s.map = c.take<unsigned long long>(s.map_cap);
    if (bytes) *bytes = c.off;
    return s;
}

// Per-search scratch.
struct Scratch {
    float4* pack;           // [max(nq,nr)] packed input points before sorting
    SortWorkspace sort;
    int64_t* scan_tiles64;  // [scan_tiles(max)]
    int32_t* scan_tiles32;  // [scan_tiles(max)]
    float4* qsorted;        // [nq]
    int32_t* qsidx;         // [nq]
    int32_t* qgroup_start;  // [nq+1]
    int32_t* qgroup_coords; // [3*nq]
    int32_t* num_qgroups;   // [1]
    int32_t* unit_group;    // [nq]
    int32_t* unit_t0;       // [nq]
    int32_t* num_units;     // [1]
    int32_t* counts;        // [nq]
    int32_t* stray;         // [nq]
    int32_t* num_stray;     // [1]
    int32_t* work;          // [4] work counters
    int64_t* total;         // [1]
    int64_t* info;          // [8] total pairs, grid error, stray queries, exact-only mode, staging words
                            //     requested, units re-walked by tcr_emit, 0, 0
    QueryParams* qparams;   // [1]
    int32_t* rec;           // [nq] per unit: offset of its record in the staging list (-1: not staged)
    int32_t* query_unit;    // [nq] unit of each sorted query
    int32_t* flagged;       // [nq] units re-walked by the emit pass
    int32_t* num_flagged;   // [1]
    unsigned long long* cursor;  // [1] staging fill
};

static Scratch carve_scratch(void* buf, int64_t nq, int64_t nr, int64_t* bytes) {
    Carve c{(char*)buf, 0};
    Scratch s;
    int64_t nmax = std::max<int64_t>(std::max<int64_t>(nq, nr), 1);
    s.sort.state = c.take<SortState>(1);
    s.num_qgroups = c.take<int32_t>(1);
    s.num_units = c.take<int32_t>(1);
    s.num_stray = c.take<int32_t>(1);
    s.work = c.take<int32_t>(4);
    s.total = c.take<int64_t>(1);
    s.info = c.take<int64_t>(8);
    s.qparams = c.take<QueryParams>(1);
    s.num_flagged = c.take<int32_t>(1);
    s.cursor = c.take<unsigned long long>(1);
    s.pack = c.take<float4>(nmax);
    s.sort.keys[0] = c.take<uint32_t>(nmax);
    s.sort.keys[1] = c.take<uint32_t>(nmax);
    s.sort.vals[0] = c.take<int32_t>(nmax);
    s.sort.vals[1] = c.take<int32_t>(nmax);
    s.sort.hist = c.take<int32_t>(sort_hist_elems(nmax));
    s.sort.tile_sums = c.take<int32_t>(scan_tiles(sort_hist_elems(nmax)));
    s.scan_tiles64 = c.take<int64_t>(scan_tiles(nmax + 1));
    s.scan_tiles32 = c.take<int32_t>(scan_tiles(nmax + 1));
    int64_t q = std::max<int64_t>(nq, 1);
    s.qsorted = c.take<float4>(q);
    s.qsidx = c.take<int32_t>(q);
    s.qgroup_start = c.take<int32_t>(q + 1);
    s.qgroup_coords = c.take<int32_t>(3 * q);
    s.unit_group = c.take<int32_t>(q);
    s.unit_t0 = c.take<int32_t>(q);
    s.counts = c.take<int32_t>(q);
    s.stray = c.take<int32_t>(q);
    s.rec = c.take<int32_t>(q);
    s.query_unit = c.take<int32_t>(q);
    s.flagged = c.take<int32_t>(q);
    if (bytes) *bytes = c.off;
    return s;
}

// ------------------------------------------------------------------------------------------
// build kernels


// Block reduction of max / or over a strided array; one atomic per block and field.
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

// computeGridSupport (cellTable.py:40-81) needs the largest support; the lean test needs to know
// whether every support lies in [1e-18, 1e18] (else the exact test decides every pair).
__global__ void support_stats_kernel(const float* __restrict__ h, int64_t n, SupportStats* out) {
    uint32_t kmax = 0;
    int bad = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float v = h[i];
        kmax = max(kmax, float_key(v));
        bad |= !(v >= 1e-18f && v <= 1e18f);
    }
    block_reduce_stats(kmax, bad, out);
}

__global__ void stats_init_kernel(SupportStats* a, SupportStats* b) {
    a->max_key = 0; a->bad = 0;
    if (b) { b->max_key = 0; b->bad = 0; }
}

// Query-side parameters of one search.
__global__ void query_params_kernel(const GridParams* g, int mode, int has_query_sup, QueryParams* qp) {
    const float qmax = has_query_sup ? key_float(qp->stats.max_key) : 0.0f;
    qp->qmax = (mode == kScatter) ? 0.0f : qmax;
    const bool qbad = (mode != kScatter) && has_query_sup && qp->stats.bad;
    const bool rbad = (mode != kGather) && g->ref_stats.bad;
    qp->exact_all = (qbad || rbad || !(fabsf(qp->qmax) <= 1e18f)) ? 1 : 0;
}

__global__ void sort_state_init_kernel(SortState* st) {
    st->key_min = 0xffffffffu;
    st->key_max = 0;
    st->sel[0] = 0;
}

__global__ void grid_init_kernel(GridParams* g, SortState* st) {
    g->ref_stats.max_key = 0;
    g->ref_stats.bad = 0;
    g->build_query_stats.max_key = 0;
    g->build_query_stats.bad = 0;
    g->error = 0;
    g->out_of_grid = 0;
    st->key_min = 0xffffffffu;
    st->key_max = 0;
    st->sel[0] = 0;
}

// util.py:28-79 compute_h and cellTable.py:27-29, float32 throughout.
__global__ void grid_params_kernel(SearchParams sp, GridParams* g, SortState* st) {
    const float grow = 1.00010001659393310546875f;  // fl32(1e-4 + 1)
    // computeGridSupport: scatter reads the reference supports, gather the query supports,
    // (super)symmetric both (torch.max propagates NaN, as the key maximum does).
    uint32_t key = 0;
    if (sp.mode != kGather) key = max(key, g->ref_stats.max_key);
    if (sp.mode != kScatter) key = max(key, g->build_query_stats.max_key);
    float hmax = key_float(key);
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
        float r = __fdiv_rn(ext[d], h[d]);
        any |= ceilf(r) > r;
    }
    if (any)
        for (int d = 0; d < sp.dim; ++d) h[d] = __fmul_rn(h[d], grow);
    float hc = h[0];
    for (int d = 1; d < sp.dim; ++d) {
        float v = h[d];
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
            // periodic dims of a clamped grid hold a whole number of cells (ext / n each); rounding
            // must not add a sliver cell at the seam
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
    if (err) st->key_min = st->key_max = 0;  // no radix pass runs on keys that were never written
}

__device__ __forceinline__ float4 load_point(const float* x, const float* h, int64_t i, int dim) {
    float4 v = make_float4(0.f, 0.f, 0.f, h ? h[i] : 0.0f);
    const float* p = x + i * dim;
    v.x = p[0];
    if (dim > 1) v.y = p[1];
    if (dim > 2) v.z = p[2];
    return v;
}

__device__ __forceinline__ float4 wrap_point(const SearchParams& sp, float4 v, int times) {
    for (int d = 0; d < sp.dim; ++d)
        if ((sp.periodic_mask >> d) & 1) {
            float c = comp(v, d);
            for (int t = 0; t < times; ++t) c = wrap_coord(c, sp.dmin[d], sp.ext[d]);
            if (d == 0) v.x = c; else if (d == 1) v.y = c; else v.z = c;
        }
    return v;
}

__device__ __forceinline__ void point_cell(const SearchParams& sp, const GridParams* g, const float4& v, int32_t* c) {
    c[0] = cell_coord(v.x, sp.dmin[0], g->hcell_d[0]);
    c[1] = sp.dim > 1 ? cell_coord(v.y, sp.dmin[1], g->hcell_d[1]) : 0;
    c[2] = sp.dim > 2 ? cell_coord(v.z, sp.dmin[2], g->hcell_d[2]) : 0;
    if (sp.dedupe)  // clamped grid: every point in a cell of [0, count) -- no aliasing, no short seam cell
        for (int d = 0; d < sp.dim; ++d) c[d] = min(max(c[d], 0), g->count[d] - 1);
}

// Wrap (twice for the reference cloud, cppSearch.py:221 after neighborhood.py:203; once for a
// query cloud), pack to float4 and emit the signed-order linear key.
__global__ void pack_points_kernel(SearchParams sp, GridParams* g, const float* x, const float* h, int64_t n,
                                   int wraps, float4* pack, uint32_t* keys, int32_t* vals, SortState* st,
                                   int track_grid) {
    uint32_t kmin = 0xffffffffu, kmax = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n && !g->error; i += stride) {
        float4 v = wrap_point(sp, load_point(x, h, i, sp.dim), wraps);
        int32_t c[3];
        point_cell(sp, g, v, c);
        if (track_grid) {
            bool out = false;
            for (int d = 0; d < sp.dim; ++d) out |= c[d] < 0 || c[d] >= g->count[d];
            if (out && !g->out_of_grid) atomicOr(&g->out_of_grid, 1);
        }
        uint32_t key = (uint32_t)linear_index(sp.dim, c, g->count) ^ 0x80000000u;
        pack[i] = v;
        keys[i] = key;
        vals[i] = (int32_t)i;
        kmin = min(kmin, key);
        kmax = max(kmax, key);
    }
    __shared__ uint32_t s_min[32], s_max[32];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { s_min[w] = kmin; s_max[w] = kmax; }
    __syncthreads();
    if (w == 0) {
        kmin = lane < nw ? s_min[lane] : 0xffffffffu;
        kmax = lane < nw ? s_max[lane] : 0u;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
            kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
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

// Gathers sorted points and flags run starts (unique_consecutive, hashTable.py:193).
struct RunFlagIn {
    const GridParams* g;
    const uint32_t* keys0;
    const uint32_t* keys1;
    const SortState* st;
    __device__ int32_t operator()(int64_t i) const {
        if (g->error) return 0;
        const uint32_t* k = st->sel[4] ? keys1 : keys0;
        return (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
    }
};

// Writes one cell record per run start: begin, lin, coords of the run's first point, bucket.
struct CellOut {
    SearchParams sp;
    const GridParams* g;
    const uint32_t* keys0;
    const uint32_t* keys1;
    const SortState* st;
    const float4* rsorted;
    int32_t* cell_start;
    int32_t* cell_lin;
    int32_t* cell_coords;
    int32_t* cell_bucket;
    unsigned long long* map;
    int64_t map_cap;
    __device__ void operator()(int64_t i, int32_t ex, int32_t flag) const {
        if (!flag) return;
        const uint32_t* k = st->sel[4] ? keys1 : keys0;
        const int32_t cell = ex;
        const int32_t lin = (int32_t)(k[i] ^ 0x80000000u);
        int32_t c[3];
        point_cell(sp, g, rsorted[i], c);
        cell_start[cell] = (int32_t)i;
        cell_lin[cell] = lin;
        cell_coords[3 * cell + 0] = c[0];
        cell_coords[3 * cell + 1] = c[1];
        cell_coords[3 * cell + 2] = c[2];
        cell_bucket[cell] = (int32_t)ref_hash(sp.dim, c, sp.hash_len);
        map_insert(map, map_cap, lin, cell);
    }
};

__global__ void gather_sorted_kernel(const GridParams* g, const float4* pack, const int32_t* vals0,
                                     const int32_t* vals1, const SortState* st, int64_t n, float4* sorted,
                                     int32_t* sidx) {
    if (g->error) return;
    const int32_t* v = st->sel[4] ? vals1 : vals0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int32_t p = v[i];
        sorted[i] = pack[p];
        sidx[i] = p;
    }
}

__global__ void finish_cells_kernel(int32_t* cell_start, const int32_t* num_cells, int64_t n) {
    cell_start[*num_cells] = (int32_t)n;
}

// ------------------------------------------------------------------------------------------
// query side

// Self search: query i is reference i, so the reference order and cells group the queries.
// Positions are the once-wrapped query coordinates (only periodic dims differ from rsorted).
__global__ void pack_self_queries_kernel(SearchParams sp, const GridParams* g, const float* x, const float* h,
                                         const int32_t* rsidx, int64_t n, float4* qsorted, int32_t* qsidx) {
    if (g->error) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        int32_t i = rsidx[t];
        qsorted[t] = wrap_point(sp, load_point(x, h, i, sp.dim), 1);
        qsidx[t] = i;
    }
}

struct QueryGroupOut {
    SearchParams sp;
    const GridParams* g;
    const float4* qsorted;
    int32_t* group_start;
    int32_t* group_coords;
    __device__ void operator()(int64_t i, int32_t ex, int32_t flag) const {
        if (!flag) return;
        int32_t c[3];
        point_cell(sp, g, qsorted[i], c);
        group_start[ex] = (int32_t)i;
        group_coords[3 * ex + 0] = c[0];
        group_coords[3 * ex + 1] = c[1];
        group_coords[3 * ex + 2] = c[2];
    }
};

constexpr int kUnit = 32;  // queries per work unit (one warp)

// Group count comes from a device scalar; the scan kernels are launched over the upper bound
// and read the true count through the functor.
struct BoundedUnitCountIn {
    const int32_t* group_start;
    const int32_t* num_groups;
    __device__ int32_t operator()(int64_t g) const {
        if (g >= *num_groups) return 0;
        int32_t n = group_start[g + 1] - group_start[g];
        return (n + kUnit - 1) / kUnit;
    }
};
struct BoundedUnitOut {
    const int32_t* group_start;
    const int32_t* num_groups;
    int32_t* unit_group;
    int32_t* unit_t0;
    int32_t* query_unit;
    __device__ void operator()(int64_t g, int32_t ex, int32_t nunits) const {
        if (g >= *num_groups) return;
        const int32_t s = group_start[g], e = group_start[g + 1];
        for (int32_t u = 0; u < nunits; ++u) {
            unit_group[ex + u] = (int32_t)g;
            unit_t0[ex + u] = s + u * kUnit;
        }
        for (int32_t t = s; t < e; ++t) query_unit[t] = ex + (t - s) / kUnit;
    }
};

// ------------------------------------------------------------------------------------------
// the candidate walk
//
// Work unit: <= 32 queries of one query group (cell).  One warp walks the unit's stencil
// candidates in chunks of 32 (lane = candidate) and tests every query of the unit against the
// chunk (query positions broadcast from shared memory); __ballot_sync gives, per query and chunk,
// the 32-bit hit mask.  Pass 1 keeps the masks of a unit with <= kSegChunks chunks in shared
// memory, reserves room for the unit's hits in a staging list with one atomic and writes them
// there query by query; pass 2 moves each query's staged hits to its CSR/COO slot (a memory-bound
// copy).  A unit with more chunks, or one that finds the staging list full, is only counted in
// pass 1 and is walked again (with the test) in pass 2 to write its pairs directly.

struct WalkArgs {
    SearchParams sp;
    const GridParams* g;
    const QueryParams* qp;
    const float4* __restrict__ rsorted;
    const int32_t* __restrict__ rsidx;
    const int32_t* __restrict__ cell_start;
    const int32_t* __restrict__ cell_coords;
    const int32_t* __restrict__ cell_bucket;
    const unsigned long long* __restrict__ map;
    int64_t map_cap;
    const float4* __restrict__ qsorted;
    const int32_t* __restrict__ qsidx;
    const int32_t* __restrict__ group_start;
    const int32_t* __restrict__ group_coords;
    const int32_t* __restrict__ unit_group;
    const int32_t* __restrict__ unit_t0;
    const int32_t* __restrict__ num_units;
    const int32_t* __restrict__ unit_list;  // emit re-walk: the units to walk (null: all units)
    const int32_t* __restrict__ num_list;
    int32_t* work;
    int32_t* stray;
    int32_t* num_stray;
    int32_t* counts;              // [nq] pass-1 output, original query order
    int32_t* rec;                 // [units] offset of each unit's record in the staging list, -1 if not staged
    int32_t no_stray_check;       // self search, no periodic dims, every point in the grid: a query's cell is
                                  // its group's (the device flag out_of_grid withdraws this)
    int32_t* query_unit;          // [nq] unit of each sorted query
    int32_t* flagged;             // [units] units to re-walk in pass 2
    int32_t* num_flagged;
    unsigned long long* cursor;   // staging list fill
    int32_t* stage;               // staging list (original reference indices)
    int64_t stage_cap;
    const int32_t* __restrict__ query_ids;  // optional: row written for local query q is query_ids[q]
    const int32_t* __restrict__ ref_ids;    // optional: column written for local reference j is ref_ids[j]
    const int64_t* offsets;       // pass-2 input [nq+1]
    int64_t* row_out;             // pass 2: COO rows or null
    int64_t* col_out;             // pass 2: columns
    int64_t out_cap;              // pass 2: entries of row_out/col_out; writes beyond are dropped
};

// Looks up stencil cell `o` (getOffsets order, last coordinate fastest) around cell gc with the
// reference's semantics; returns the sorted range or an empty one.
__device__ __forceinline__ void stencil_lookup(const WalkArgs& a, const int32_t* gc, int o, int32_t& beg,
                                               int32_t& cnt) {
    const SearchParams& sp = a.sp;
    int32_t c[3] = {0, 0, 0};
    int rem = o;
    bool dup = false;
    for (int d = sp.dim - 1; d >= 0; --d) {
        int32_t off = rem % 3 - 1;
        rem /= 3;
        int32_t v = gc[d] + off;
        if ((sp.periodic_mask >> d) & 1) {
            const int32_t n = a.g->count[d];
            v = pymod(v, n);
            // with fewer than 3 cells the wrapped offsets repeat a cell; the clamped grid visits it once
            if (sp.dedupe && ((n == 1 && off != 0) || (n == 2 && off == 1))) dup = true;
        } else if (sp.dedupe && (v < 0 || v >= a.g->count[d])) {
            dup = true;  // clamped grid: nothing lies outside it
        }
        c[d] = v;
    }
    beg = 0;
    cnt = 0;
    if (dup) return;
    int32_t lin = linear_index(sp.dim, c, a.g->count);
    int32_t cell = map_find(a.map, a.map_cap, lin);
    if (cell < 0) return;
    // queryHashMap matches the linear index inside bucket hash(c) only.
    if ((uint32_t)__ldg(&a.cell_bucket[cell]) != ref_hash(sp.dim, c, sp.hash_len)) return;
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

// One (query, candidate) test.  in: decided; unc: needs the exact reference test.
template <int DIM, bool PERIODIC, int MODE>
__device__ __forceinline__ void lean_test(const SearchParams& sp, const float4& q, const float4& c, float cw,
                                          float band, bool& in, bool& unc) {
    float d2;
    bool wrap_unc = false;
    {
        float dd[3];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            float diff = comp(q, d) - comp(c, d);
            if (PERIODIC && ((sp.periodic_mask >> d) & 1)) {
                const float h = sp.ext[d];
                const float half = 0.5f * h;
                wrap_unc |= fabsf(fabsf(diff) - half) <= kBandEps * h;
                if (diff >= half) diff -= h;
                else if (diff < -half) diff += h;
            }
            dd[d] = diff;
        }
        d2 = dd[0] * dd[0];
        if (DIM > 1) d2 = fmaf(dd[1], dd[1], d2);
        if (DIM > 2) d2 = fmaf(dd[2], dd[2], d2);
    }
    const float thr = pair_thr<MODE>(q.w, cw);
    const float r = fmaf(-thr, thr, d2);  // d2 - thr^2, one rounding; sign exact
    in = r < 0.0f;
    unc = (fabsf(r) <= band) || wrap_unc;
}

constexpr int kWalkWarps = 4;
constexpr int kSegChunks = 24;  // staged units: at most 24 chunks (768 candidates)
constexpr int kMaskStride = kSegChunks + 1;  // padded rows: conflict-free per-lane reads

struct WalkSmem {
    int32_t pre[kWalkWarps][33];
    int32_t beg[kWalkWarps][32];
    float4 q[kWalkWarps][32];
    float4 cand[kWalkWarps][36];                  // the chunk's candidates, stream-major, rows padded
    uint32_t mask[kWalkWarps][32 * kMaskStride];  // [query][chunk] hit masks
    int32_t sj[kWalkWarps][kSegChunks][32];       // original index of candidate (chunk, lane)
};

// Candidate k of the unit (prefix pre[0..S]): returns its sorted index.
__device__ __forceinline__ int32_t cand_index(const int32_t* pre, const int32_t* beg, int S, int32_t k) {
    int lo = 0, hi = S;  // pre[lo] <= k < pre[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (pre[mid] <= k) lo = mid; else hi = mid;
    }
    return beg[lo] + (k - pre[lo]);
}

// Lane-side constants of the lean test for query q (support hq): the query's share of the
// threshold and the half width of the band, conservative over every candidate (rmax is the
// largest reference support).
template <int MODE>
__device__ __forceinline__ float query_share(float hq) {
    return MODE == kSymmetric ? 0.5f * hq : (MODE == kGather ? hq * hq : hq);
}
template <int MODE>
__device__ __forceinline__ float query_band(float hq, float rmax) {
    float t;
    if (MODE == kGather) t = hq;
    else if (MODE == kScatter) t = rmax;
    else if (MODE == kSymmetric) t = fmaf(hq, 0.5f, 0.5f * rmax);
    else t = fmaxf(hq, rmax);
    return kBandEps * t * t;
}

// Float test of query q (lane) against candidate c; r < 0 means inside.
template <int DIM, bool PERIODIC, int MODE>
__device__ __forceinline__ float lane_residual(const ExactCtx& sp, const float4& q, float qs, const float4& c,
                                               bool& wrap_unc) {
    float dd[3];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        float diff = comp(q, d) - comp(c, d);
        if (PERIODIC && ((sp.periodic_mask >> d) & 1)) {
            const float h = sp.ext[d];
            const float half = 0.5f * h;
            wrap_unc |= fabsf(fabsf(diff) - half) <= kBandEps * h;
            if (diff >= half) diff -= h;
            else if (diff < -half) diff += h;
        }
        dd[d] = diff;
    }
    float d2 = dd[0] * dd[0];
    if (DIM > 1) d2 = fmaf(dd[1], dd[1], d2);
    if (DIM > 2) d2 = fmaf(dd[2], dd[2], d2);
    if (MODE == kGather) return d2 - qs;                 // qs = hq^2 (same sign as d2 - hq*hq)
    if (MODE == kScatter) return fmaf(-c.w, c.w, d2);
    const float thr = (MODE == kSymmetric) ? fmaf(c.w, 0.5f, qs) : fmaxf(q.w, c.w);
    return fmaf(-thr, thr, d2);
}

// Tests the lane's query against the Q candidates of its stream; returns the Q-bit hit mask and
// ORs into `unc` whether any pair lies in the band (those units are redone with exact decisions).
template <int DIM, bool PERIODIC, int MODE, int Q>
__device__ __forceinline__ uint32_t stream_mask(const ExactCtx& sp, const float4* cand, const float4& q, float qs,
                                                float band, bool& unc) {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const float4 c = cand[k];
        bool wrap_unc = false;
        const float r = lane_residual<DIM, PERIODIC, MODE>(sp, q, qs, c, wrap_unc);
        if (r < 0.0f) m |= 1u << k;
        unc |= (fabsf(r) <= band) || wrap_unc;
    }
    return m;
}

// The same with every in-band pair decided by the exact reference test (rare units only).
template <int DIM, bool PERIODIC, int MODE>
__device__ __noinline__ uint32_t stream_mask_exact(ExactCtx xc, const float4* cand, int n, float4 q, float qs,
                                                   float band) {
    const ExactCtx& sp = xc;
    uint32_t m = 0;
    for (int k = 0; k < n; ++k) {
        const float4 c = cand[k];
        bool wrap_unc = false;
        const float r = lane_residual<DIM, PERIODIC, MODE>(sp, q, qs, c, wrap_unc);
        bool in = r < 0.0f;
        if ((fabsf(r) <= band) || wrap_unc) in = exact_pair_test(xc, q, q.w, c, c.w);
        if (in) m |= 1u << k;
    }
    return m;
}

// Pass 1: test every (query, candidate) once; count, stage the hits of small units.
//
// Each chunk's 32 candidates are staged in shared memory; lane (q, s) holds query q and tests it
// against the Q candidates of stream s (Q = 8, 16 or 32 as the unit has <= 8, <= 16 or <= 32
// queries, so 32/Q streams keep every lane busy).  Hits become bits of a per-lane mask, merged
// across streams with shuffles into the 32-bit (query, chunk) mask.
template <int DIM, bool PERIODIC, int MODE>
__global__ void __launch_bounds__(kWalkWarps * 32) walk_count_kernel(WalkArgs a) {
    if (a.g->error) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WalkSmem& sm = *reinterpret_cast<WalkSmem*>(smem_raw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int S = DIM == 1 ? 3 : (DIM == 2 ? 9 : 27);
    const ExactCtx xc = exact_ctx(a.sp);
    const float rmax = key_float(a.g->ref_stats.max_key);
    const bool exact_all = a.qp->exact_all != 0;
    const int32_t nunits = *a.num_units;
    const float4 nan4 = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
    for (;;) {
        int32_t unit = 0;
        if (lane == 0) unit = atomicAdd(&a.work[0], 1);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= nunits) break;
        const int32_t grp = a.unit_group[unit];
        const int32_t t0 = a.unit_t0[unit];
        const int32_t nb = min(32, a.group_start[grp + 1] - t0);
        const int32_t gc[3] = {a.group_coords[3 * grp], a.group_coords[3 * grp + 1], a.group_coords[3 * grp + 2]};
        int32_t beg = 0, cnt = 0;
        if (lane < S) stencil_lookup(a, gc, lane, beg, cnt);
        const int32_t inc = warp_inclusive_scan(cnt);
        sm.pre[w][lane + 1] = inc;
        if (lane == 0) sm.pre[w][0] = 0;
        sm.beg[w][lane] = beg;
        const int32_t M = __shfl_sync(0xffffffffu, inc, 31);
        bool active = false;
        int32_t qorig = 0;
        float4 qv = nan4;
        if (lane < nb) {
            const int32_t t = t0 + lane;
            qv = a.qsorted[t];
            qorig = a.qsidx[t];
            active = true;
            if (!a.no_stray_check || a.g->out_of_grid) {
                int32_t qc[3];
                point_cell(a.sp, a.g, qv, qc);
                active = same_cell<DIM>(qc, gc);
            }
            if (!active) {  // own cell differs from the group's (aliasing or wrap rounding): serial path
                int32_t k = atomicAdd(a.num_stray, 1);
                a.stray[k] = t;
                qv = nan4;
            }
        }
        sm.q[w][lane] = qv;  // rows >= nb hold NaN queries and never hit
        const int32_t nchunks = (M + 31) >> 5;
        const bool stage = a.stage_cap > 0 && nchunks <= kSegChunks;
        const int Q = nb <= 8 ? 8 : (nb <= 16 ? 16 : 32);
        const int lq = lane & (Q - 1);      // this lane's query
        const int ls = lane / Q;            // this lane's stream
        __syncwarp();
        const float4 myq = sm.q[w][lq];
        const float qs = query_share<MODE>(myq.w);
        const float band = exact_all ? __int_as_float(0x7f800000) : query_band<MODE>(myq.w, rmax);
        const float4* my_cand = &sm.cand[w][ls * (Q + 1)];
        // Lane k of chunk c holds candidate 32c + k.  Its stencil cell r only moves forward from
        // chunk to chunk, so it is tracked incrementally instead of searched.
        int32_t cr = 0;
        const int32_t* pre = sm.pre[w];
        const int32_t* begs = sm.beg[w];
        const float4* __restrict__ rs = a.rsorted;
        const int32_t* __restrict__ ri = a.rsidx;
        const int32_t* __restrict__ rid = a.ref_ids;
        auto fetch = [&cr, pre, begs, rs, ri, rid, M, nan4](int32_t k, float4& v, int32_t& jo) {
            v = nan4;
            jo = 0;
            if (k < M) {
                while (pre[cr + 1] <= k) ++cr;
                const int32_t j = begs[cr] + (k - pre[cr]);
                v = __ldg(&rs[j]);
                jo = __ldg(&ri[j]);
                if (rid) jo = __ldg(&rid[jo]);
            }
        };
        // the unit's chunk loop; `exact` redoes it deciding in-band pairs with the reference test
        int32_t qcount = 0;
        bool unc = false;
        for (int pass = 0; pass < 2; ++pass) {
            const bool exact = pass == 1;
            cr = 0;
            qcount = 0;
            float4 nxt;
            int32_t nxt_j;
            fetch(lane, nxt, nxt_j);
            for (int32_t c = 0; c < nchunks; ++c) {
                // stage candidate `lane` of this chunk: stream lane / Q, slot lane % Q
                sm.cand[w][(lane / Q) * (Q + 1) + (lane & (Q - 1))] = nxt;
                if (stage) sm.sj[w][c][lane] = nxt_j;
                fetch(((c + 1) << 5) + lane, nxt, nxt_j);  // prefetch the next chunk's candidate
                __syncwarp();
                uint32_t m;
                if (exact) {
                    m = stream_mask_exact<DIM, PERIODIC, MODE>(xc, my_cand, Q, myq, qs, band) << (Q == 32 ? 0 : Q * ls);
                } else if (Q == 32) {
                    m = stream_mask<DIM, PERIODIC, MODE, 32>(xc, my_cand, myq, qs, band, unc);
                } else if (Q == 16) {
                    m = stream_mask<DIM, PERIODIC, MODE, 16>(xc, my_cand, myq, qs, band, unc) << (16 * ls);
                } else {
                    m = stream_mask<DIM, PERIODIC, MODE, 8>(xc, my_cand, myq, qs, band, unc) << (8 * ls);
                }
                if (Q <= 16) m |= __shfl_xor_sync(0xffffffffu, m, 16);
                if (Q == 8) m |= __shfl_xor_sync(0xffffffffu, m, 8);
                if (lane < nb) {
                    qcount += __popc(m);
                    if (stage) sm.mask[w][lane * kMaskStride + c] = m;
                }
                __syncwarp();
            }
            if (exact || !__any_sync(0xffffffffu, unc)) break;
        }
        if (active) a.counts[qorig] = qcount;
        bool staged = false;
        if (stage) {
            // record: [nchunks] [masks: nb x nchunks, query-major] [candidates: nchunks x 32]
            const int64_t words = 1 + (int64_t)nb * nchunks + 32 * (int64_t)nchunks;
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(a.cursor, (unsigned long long)words);
            base = __shfl_sync(0xffffffffu, base, 0);
            staged = base + (unsigned long long)words <= (unsigned long long)a.stage_cap;
            if (staged) {
                int32_t* r = a.stage + base;
                if (lane == 0) {
                    r[0] = nchunks;
                    a.rec[unit] = (int32_t)base;
                }
                __syncwarp();
                for (int q = 0; q < nb; ++q)
                    if (lane < nchunks) r[1 + q * nchunks + lane] = sm.mask[w][q * kMaskStride + lane];
                int32_t* rj = r + 1 + nb * nchunks;
                for (int32_t c = 0; c < nchunks; ++c) rj[c * 32 + lane] = sm.sj[w][c][lane];
            }
        }
        if (!staged && lane == 0) {
            int32_t f = atomicAdd(a.num_flagged, 1);
            a.flagged[f] = unit;
        }
        __syncwarp();
    }
}

// Pass 2 for flagged units: walk again and write the pairs straight to their slots.
template <int DIM, bool PERIODIC, int MODE>
__global__ void __launch_bounds__(kWalkWarps * 32) walk_emit_kernel(WalkArgs a) {
    if (a.g->error) return;
    __shared__ int32_t s_pre[kWalkWarps][33];
    __shared__ int32_t s_beg[kWalkWarps][32];
    __shared__ float4 s_q[kWalkWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    constexpr int S = DIM == 1 ? 3 : (DIM == 2 ? 9 : 27);
    const ExactCtx xc = exact_ctx(a.sp);
    const float qmax = a.qp->qmax;
    const bool exact_all = a.qp->exact_all != 0;
    const int32_t nlist = *a.num_list;
    const float4 nan4 = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
    for (;;) {
        int32_t li = 0;
        if (lane == 0) li = atomicAdd(&a.work[1], 1);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= nlist) break;
        const int32_t unit = a.unit_list[li];
        const int32_t grp = a.unit_group[unit];
        const int32_t t0 = a.unit_t0[unit];
        const int32_t nb = min(32, a.group_start[grp + 1] - t0);
        const int32_t gc[3] = {a.group_coords[3 * grp], a.group_coords[3 * grp + 1], a.group_coords[3 * grp + 2]};
        int32_t beg = 0, cnt = 0;
        if (lane < S) stencil_lookup(a, gc, lane, beg, cnt);
        const int32_t inc = warp_inclusive_scan(cnt);
        s_pre[w][lane + 1] = inc;
        if (lane == 0) s_pre[w][0] = 0;
        s_beg[w][lane] = beg;
        const int32_t M = __shfl_sync(0xffffffffu, inc, 31);
        int32_t qorig = 0;
        float4 qv = nan4;
        int64_t obase = 0;
        if (lane < nb) {
            const int32_t t = t0 + lane;
            qv = a.qsorted[t];
            qorig = a.qsidx[t];
            int32_t qc[3];
            point_cell(a.sp, a.g, qv, qc);
            if (same_cell<DIM>(qc, gc)) obase = a.offsets[qorig];
            else qv = nan4;  // stray: written by the serial kernel
        }
        s_q[w][lane] = qv;
        __syncwarp();
        for (int32_t base = 0; base < M; base += 32) {
            const int32_t k = base + lane;
            float4 cv = nan4;
            int32_t j = 0;
            if (k < M) {
                j = cand_index(s_pre[w], s_beg[w], S, k);
                cv = __ldg(&a.rsorted[j]);
            }
            int32_t jl = __ldg(&a.rsidx[j]);
            if (a.ref_ids) jl = __ldg(&a.ref_ids[jl]);
            const int64_t jorig = (int64_t)jl;
            const float cw = cand_share<MODE>(cv.w);
            const float band = exact_all ? __int_as_float(0x7f800000) : cand_band<MODE>(cw, qmax);
            for (int qi = 0; qi < nb; ++qi) {
                const float4 q = s_q[w][qi];
                bool in, unc;
                lean_test<DIM, PERIODIC, MODE>(a.sp, q, cv, cw, band, in, unc);
                const uint32_t ub = __ballot_sync(0xffffffffu, unc);
                if (ub) in = unc ? exact_pair_test(xc, q, q.w, cv, cv.w) : in;
                const uint32_t b = __ballot_sync(0xffffffffu, in);
                const int64_t qb = __shfl_sync(0xffffffffu, obase, qi);
                int32_t qrow = __shfl_sync(0xffffffffu, qorig, qi);
                if (a.query_ids) qrow = __ldg(&a.query_ids[qrow]);
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
}

// Pass 2 for staged units: expand each unit's record into its queries' CSR/COO slots, one warp
// per unit.  The warp stages the unit's mask block in shared memory; lane q expands query q's hit
// bits into a shared output table (source chunk and bit of each of the unit's outputs, in output
// order); then lanes = output positions read the table and write consecutive slots.  A unit with
// more than kExpandTab outputs locates each output by binary searches over the prefixes instead.
constexpr int kExpandWarps = 8;
constexpr int kExpandTab = 2048;
struct ExpandSmem {
    uint16_t tab[kExpandWarps][kExpandTab];        // (query << 10) | (chunk << 5) | bit, in output order
    int32_t qpre[kExpandWarps][33];                // exclusive output prefix over queries
    int64_t qoff[kExpandWarps][32];
    int32_t qrow[kExpandWarps][32];
};

__global__ void __launch_bounds__(kExpandWarps * 32) expand_records_kernel(
    const int32_t* __restrict__ stage, const int32_t* __restrict__ rec, const int32_t* __restrict__ num_units,
    const int32_t* __restrict__ unit_t0, const int32_t* __restrict__ unit_group,
    const int32_t* __restrict__ group_start, const int32_t* __restrict__ qsidx, const int64_t* __restrict__ offsets,
    const int32_t* __restrict__ query_ids, int64_t* __restrict__ row_out, int64_t* __restrict__ col_out,
    int64_t out_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ExpandSmem& sm = *reinterpret_cast<ExpandSmem*>(smem_raw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int32_t nu = *num_units;
    const int64_t warps = (int64_t)gridDim.x * kExpandWarps;
    uint16_t* tab = sm.tab[w];
    int64_t u = (int64_t)blockIdx.x * kExpandWarps + w;
    int32_t r0n = u < nu ? rec[u] : -1;
    int32_t t0n = u < nu ? unit_t0[u] : 0;
    int32_t gn = u < nu ? unit_group[u] : 0;
    for (; u < nu; u += warps) {
        const int32_t r0 = r0n, t0 = t0n, grp = gn;
        if (u + warps < nu) {  // the next unit's header, ahead of its use
            r0n = rec[u + warps];
            t0n = unit_t0[u + warps];
            gn = unit_group[u + warps];
        }
        if (r0 < 0) continue;  // re-tested by the emit walk
        const int32_t* r = stage + r0;
        const int32_t nchunks = r[0];
        if (nchunks <= 0) continue;  // no candidates, no outputs
        const int32_t nb = min(32, group_start[grp + 1] - t0);
        const int32_t nm = nb * nchunks;
        const uint32_t* mk = reinterpret_cast<const uint32_t*>(r + 1);  // [query][chunk]
        const int32_t* cands = r + 1 + nm;                               // [chunk][32]
        int32_t total = 0;
        if (lane < nb) {
            const int32_t row = qsidx[t0 + lane];
            sm.qrow[w][lane] = query_ids ? query_ids[row] : row;
            sm.qoff[w][lane] = offsets[row];
            for (int c = 0; c < nchunks; ++c) total += __popc(mk[lane * nchunks + c]);
        }
        const int32_t qinc = warp_inclusive_scan(total);
        sm.qpre[w][lane + 1] = qinc;
        if (lane == 0) sm.qpre[w][0] = 0;
        const int32_t n = __shfl_sync(0xffffffffu, qinc, 31);
        if (n <= kExpandTab) {
            // lanes over (query, chunk) pairs in output order; each expands its few hit bits
            int32_t carry = 0;
            int pq = 0, pc = lane;  // pair (query, chunk) of p = base + lane, advanced without division
            while (pc >= nchunks) { pc -= nchunks; ++pq; }
            for (int32_t base = 0; base < nm; base += 32) {
                const int32_t p = base + lane;
                uint32_t m = p < nm ? mk[p] : 0u;
                const int32_t cnt = __popc(m);
                const int32_t inc = warp_inclusive_scan(cnt);
                int32_t k = carry + inc - cnt;
                carry += __shfl_sync(0xffffffffu, inc, 31);
                const int32_t tag = (pq << 10) | (pc << 5);
                while (m) {
                    const int bit = __ffs(m) - 1;
                    m &= m - 1;
                    tab[k++] = (uint16_t)(tag | bit);
                }
                pc += 32;
                while (pc >= nchunks) { pc -= nchunks; ++pq; }
            }
            __syncwarp();
#pragma unroll 4
            for (int32_t o = lane; o < n; o += 32) {
                const int32_t v = tab[o];
                const int q = v >> 10;
                const int64_t pos = sm.qoff[w][q] + (o - sm.qpre[w][q]);
                if (pos < out_cap) {
                    col_out[pos] = (int64_t)cands[v & 0x3ff];
                    if (row_out) row_out[pos] = (int64_t)sm.qrow[w][q];
                }
            }
        } else {
            __syncwarp();
            for (int32_t o = lane; o < n; o += 32) {
                int lo = 0, hi = nb;  // query: qpre[lo] <= o < qpre[hi]
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (sm.qpre[w][mid] <= o) lo = mid; else hi = mid;
                }
                const int q = lo;
                int32_t tq = o - sm.qpre[w][q];
                int c = 0;  // chunk holding the query's tq-th hit (tq < hits of q, so c < nchunks)
                for (; c < nchunks; ++c) {
                    const int32_t pcnt = __popc(mk[q * nchunks + c]);
                    if (tq < pcnt) break;
                    tq -= pcnt;
                }
                if (c >= nchunks) continue;
                const int bit = __fns(mk[q * nchunks + c], 0, tq + 1);
                const int64_t pos = sm.qoff[w][q] + (o - sm.qpre[w][q]);
                if (pos < out_cap) {
                    col_out[pos] = (int64_t)cands[c * 32 + bit];
                    if (row_out) row_out[pos] = (int64_t)sm.qrow[w][q];
                }
            }
        }
        __syncwarp();
    }
}

// Serial walk for queries whose own cell differs from their group's (one thread per query).
template <bool EMIT>
__global__ void stray_kernel(WalkArgs a) {
    if (a.g->error) return;
    const int32_t ns = *a.num_stray;
    const int S = a.sp.dim == 1 ? 3 : (a.sp.dim == 2 ? 9 : 27);
    const ExactCtx xc = exact_ctx(a.sp);
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
        const int32_t t = a.stray[s];
        const float4 q = a.qsorted[t];
        const int32_t qorig = a.qsidx[t];
        int32_t qc[3];
        point_cell(a.sp, a.g, q, qc);
        int64_t pos = EMIT ? a.offsets[qorig] : 0;
        int32_t n = 0;
        for (int o = 0; o < S; ++o) {
            int32_t beg, cnt;
            stencil_lookup(a, qc, o, beg, cnt);
            for (int32_t j = beg; j < beg + cnt; ++j) {
                const float4 cv = a.rsorted[j];
                if (exact_pair_test(xc, q, q.w, cv, cv.w)) {
                    if (EMIT) {
                        if (pos < a.out_cap) {
                            const int32_t jl = a.rsidx[j];
                            a.col_out[pos] = (int64_t)(a.ref_ids ? a.ref_ids[jl] : jl);
                            if (a.row_out) a.row_out[pos] = a.query_ids ? a.query_ids[qorig] : qorig;
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

__global__ void info_kernel(const GridParams* g, const int64_t* total, const int32_t* num_stray,
                            const QueryParams* qp, const unsigned long long* cursor, const int32_t* num_flagged,
                            int64_t* info) {
    info[0] = *total;
    info[1] = g->error;
    info[2] = *num_stray;
    info[3] = qp->exact_all;
    info[4] = (int64_t)*cursor;
    info[5] = *num_flagged;
    info[6] = 0;
    info[7] = 0;
}

// ------------------------------------------------------------------------------------------
// host orchestration

static SearchParams make_params(const tcr_search_desc* d) {
    SearchParams sp;
    memset(&sp, 0, sizeof(sp));
    sp.dim = d->dim;
    sp.mode = d->mode;
    sp.periodic_mask = d->periodic_mask;
    sp.hash_len = (uint32_t)d->hash_map_length;
    for (int k = 0; k < 3; ++k) {
        sp.dmin[k] = k < d->dim ? d->domain_min[k] : 0.f;
        sp.dmax[k] = k < d->dim ? d->domain_max[k] : 1.f;
        sp.ext[k] = sp.dmax[k] - sp.dmin[k];
    }
    sp.n_query = d->n_query;
    sp.n_ref = d->n_ref;
    for (int k = 0; k < 3; ++k) sp.hcell_override[k] = d->hcell[0] > 0.0f ? (k < d->dim ? d->hcell[k] : 1.0f) : 0.0f;
    sp.dedupe = d->clamped_grid ? 1 : 0;
    return sp;
}

// need_ref_sup: the structure build reads reference supports; the query phases take them from
// the structure and only need the query supports.
static int validate(const tcr_search_desc* d, bool need_ref_sup = true) {
    if (!d) return set_error(TCR_ERR_INVALID, "null descriptor");
    if (d->dim < 1 || d->dim > 3) return set_error(TCR_ERR_INVALID, "dim must be 1, 2 or 3 (got %d)", d->dim);
    if (d->mode < 0 || d->mode > 3) return set_error(TCR_ERR_INVALID, "invalid mode %d", d->mode);
    if (d->hash_map_length <= 0 || d->hash_map_length > 0xffffffffLL)
        return set_error(TCR_ERR_INVALID, "hashMapLength must be in [1, 2^32)");
    if (d->n_query < 0 || d->n_ref < 0 || d->n_query > 0x7fffffffLL || d->n_ref > 0x7ffffff0LL)
        return set_error(TCR_ERR_INVALID, "point counts must be in [0, 2^31)");
    if ((d->n_query && !d->query_pos) || (d->n_ref && !d->ref_pos))
        return set_error(TCR_ERR_INVALID, "missing positions");
    if ((d->mode == kGather || d->mode == kSymmetric || d->mode == kSuperSymmetric) && d->n_query && !d->query_sup)
        return set_error(TCR_ERR_INVALID, "this mode needs query supports");
    if (need_ref_sup && (d->mode == kScatter || d->mode == kSymmetric || d->mode == kSuperSymmetric) && d->n_ref &&
        !d->ref_sup)
        return set_error(TCR_ERR_INVALID, "this mode needs reference supports");
    if (d->self_search && d->n_query != d->n_ref)
        return set_error(TCR_ERR_INVALID, "self search needs one cloud");
    if (d->hcell[0] > 0.0f)
        for (int k = 0; k < d->dim; ++k)
            if (!(d->hcell[k] > 0.0f) || !(d->hcell[k] < 3.0e38f))
                return set_error(TCR_ERR_INVALID, "cell size override must be positive and finite in every dimension");
    return TCR_OK;
}

// Self search on one cloud with no periodic dimension: the queries, wrapped once, are the
// references, wrapped twice, so the sorted query array is the sorted reference array.
static inline bool same_sorted_points(const tcr_search_desc* d) {
    return d->self_search && d->periodic_mask == 0 && d->query_pos == d->ref_pos && d->query_sup == d->ref_sup;
}

static inline unsigned grid_for(int64_t n, int threads, int max_blocks = 148 * 16) {
    int64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, max_blocks));
}

static WalkArgs make_walk(const SearchParams& sp, const Structure& S, const Scratch& W, bool self) {
    WalkArgs a;
    memset(&a, 0, sizeof(a));
    a.sp = sp;
    a.g = S.grid;
    a.qp = W.qparams;
    a.rsorted = S.rsorted;
    a.rsidx = S.rsidx;
    a.cell_start = S.cell_start;
    a.cell_coords = S.cell_coords;
    a.cell_bucket = S.cell_bucket;
    a.map = S.map;
    a.map_cap = S.map_cap;
    a.qsorted = W.qsorted;
    a.qsidx = W.qsidx;
    a.group_start = self ? S.cell_start : W.qgroup_start;
    a.group_coords = self ? S.cell_coords : W.qgroup_coords;
    a.unit_group = W.unit_group;
    a.unit_t0 = W.unit_t0;
    a.num_units = W.num_units;
    a.unit_list = W.flagged;
    a.num_list = W.num_flagged;
    a.work = W.work;
    a.stray = W.stray;
    a.num_stray = W.num_stray;
    a.counts = W.counts;
    a.rec = W.rec;
    a.flagged = W.flagged;
    a.num_flagged = W.num_flagged;
    a.cursor = W.cursor;
    return a;
}

static int num_sms() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

// Dispatches a walk kernel template on (dim, any periodic dim, mode).
template <template <int, bool, int> class K>
static cudaError_t dispatch_walk(const WalkArgs& a, int dim, bool periodic, int mode, dim3 grid, dim3 block,
                                 size_t smem, cudaStream_t st) {
#define TCR_M(D, P)                                                                 \
    switch (mode) {                                                                 \
        case kGather: return K<D, P, kGather>::launch(a, grid, block, smem, st);    \
        case kScatter: return K<D, P, kScatter>::launch(a, grid, block, smem, st);  \
        case kSymmetric: return K<D, P, kSymmetric>::launch(a, grid, block, smem, st); \
        default: return K<D, P, kSuperSymmetric>::launch(a, grid, block, smem, st); \
    }
    if (dim == 1) { if (periodic) { TCR_M(1, true) } else { TCR_M(1, false) } }
    if (dim == 2) { if (periodic) { TCR_M(2, true) } else { TCR_M(2, false) } }
    if (periodic) { TCR_M(3, true) } else { TCR_M(3, false) }
#undef TCR_M
}

template <int D, bool P, int M>
struct CountLaunch {
    static cudaError_t launch(const WalkArgs& a, dim3 g, dim3 b, size_t smem, cudaStream_t st) {
        cudaError_t e = cudaFuncSetAttribute(walk_count_kernel<D, P, M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        walk_count_kernel<D, P, M><<<g, b, smem, st>>>(a);
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

static unsigned walk_blocks(int64_t nq) {
    const int64_t max_units = (nq + kUnit - 1) / kUnit + 1;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)num_sms() * 12, (max_units + kWalkWarps - 1) /
                                                                                             kWalkWarps));
}

}  // namespace tcr

using namespace tcr;

extern "C" {

const char* tcr_last_error(void) { return g_err; }

int tcr_version(void) { return TCR_ABI_VERSION; }

int64_t tcr_desc_bytes(void) { return (int64_t)sizeof(tcr_search_desc); }

int64_t tcr_kernel_launches(void) { return (int64_t)__atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int tcr_search_sizes(int64_t n_query, int64_t n_ref, int32_t dim, int64_t* structure_bytes, int64_t* scratch_bytes) {
    if (dim < 1 || dim > 3 || n_query < 0 || n_ref < 0) return set_error(TCR_ERR_INVALID, "invalid sizes");
    if (structure_bytes) carve_structure(nullptr, n_ref, structure_bytes);
    if (scratch_bytes) carve_scratch(nullptr, n_query, n_ref, scratch_bytes);
    return TCR_OK;
}

int tcr_structure_offsets(int64_t n_ref, int64_t* offsets, int32_t n) {
    if (n_ref < 0 || !offsets || n < TCR_STRUCT_NFIELDS) return set_error(TCR_ERR_INVALID, "invalid arguments");
    char* const base = reinterpret_cast<char*>(256);  // any non-null base; offsets are relative
    Structure s = carve_structure(base, n_ref, nullptr);
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
    offsets[TCR_STRUCT_MAP_CAPACITY] = s.map_cap;
    return TCR_OK;
}

int tcr_build_structure(const tcr_search_desc* d, void* structure, int64_t structure_bytes, void* scratch,
                        int64_t scratch_bytes, void* stream) {
    int rc = validate(d);
    if (rc) return rc;
    int64_t need_s = 0, need_w = 0;
    carve_structure(nullptr, d->n_ref, &need_s);
    carve_scratch(nullptr, d->n_query, d->n_ref, &need_w);
    if (!structure || !scratch || structure_bytes < need_s || scratch_bytes < need_w)
        return set_error(TCR_ERR_INVALID, "workspace too small (structure %lld/%lld, scratch %lld/%lld)",
                         (long long)structure_bytes, (long long)need_s, (long long)scratch_bytes, (long long)need_w);
    cudaStream_t st = (cudaStream_t)stream;
    const SearchParams sp = make_params(d);
    Structure S = carve_structure(structure, d->n_ref, nullptr);
    Scratch W = carve_scratch(scratch, d->n_query, d->n_ref, nullptr);
    const int64_t nr = d->n_ref, nq = d->n_query;
    grid_init_kernel<<<1, 1, 0, st>>>(S.grid, W.sort.state);
    note_launches(1);
    // computeGridSupport: which supports set hMax depends on the mode
    if (d->ref_sup && nr > 0) {
        support_stats_kernel<<<grid_for(nr, 256, num_sms() * 8), 256, 0, st>>>(d->ref_sup, nr, &S.grid->ref_stats);
        note_launches(1);
    }
    if (d->query_sup && nq > 0) {
        support_stats_kernel<<<grid_for(nq, 256, num_sms() * 8), 256, 0, st>>>(d->query_sup, nq,
                                                                                &S.grid->build_query_stats);
        note_launches(1);
    }
    grid_params_kernel<<<1, 1, 0, st>>>(sp, S.grid, W.sort.state);
    note_launches(1);
    TCR_CUDA(cudaMemsetAsync(S.map, 0xff, sizeof(unsigned long long) * S.map_cap, st));
    TCR_CUDA(cudaMemsetAsync(S.num_cells, 0, sizeof(int32_t), st));
    if (nr > 0) {
        pack_points_kernel<<<grid_for(nr, 256), 256, 0, st>>>(sp, S.grid, d->ref_pos, d->ref_sup, nr, 2, W.pack,
                                                              W.sort.keys[0], W.sort.vals[0], W.sort.state, 1);
        note_launches(1);
        TCR_CUDA(radix_sort_pairs(W.sort, nr, st));
        gather_sorted_kernel<<<grid_for(nr, 256), 256, 0, st>>>(S.grid, W.pack, W.sort.vals[0], W.sort.vals[1], W.sort.state,
                                                                nr, S.rsorted, S.rsidx);
        note_launches(1);
        CellOut co{sp, S.grid, W.sort.keys[0], W.sort.keys[1], W.sort.state, S.rsorted, S.cell_start, S.cell_lin,
                   S.cell_coords, S.cell_bucket, S.map, S.map_cap};
        RunFlagIn fi{S.grid, W.sort.keys[0], W.sort.keys[1], W.sort.state};
        TCR_CUDA(device_exclusive_scan<int32_t>(fi, co, nr, W.scan_tiles32, S.num_cells, st));
    }
    finish_cells_kernel<<<1, 1, 0, st>>>(S.cell_start, S.num_cells, nr);
    note_launches(1);
    TCR_CUDA(cudaGetLastError());
    return TCR_OK;
}

int tcr_count(const tcr_search_desc* d, const void* structure, void* scratch, int64_t scratch_bytes, int32_t* stage,
              int64_t stage_capacity, int64_t* offsets, int32_t* indptr_out, int64_t* row_entries_out, int64_t* info_out,
              void* stream) {
    int rc = validate(d, false);
    if (rc) return rc;
    int64_t need_w = 0;
    carve_scratch(nullptr, d->n_query, d->n_ref, &need_w);
    if (!structure || !scratch || scratch_bytes < need_w || !offsets)
        return set_error(TCR_ERR_INVALID, "workspace too small or offsets missing");
    if (stage_capacity < 0 || stage_capacity > 0x7fffffffLL || (stage_capacity > 0 && !stage))
        return set_error(TCR_ERR_INVALID, "stage capacity must be in [0, 2^31) with a buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const SearchParams sp = make_params(d);
    Structure S = carve_structure(const_cast<void*>(structure), d->n_ref, nullptr);
    Scratch W = carve_scratch(scratch, d->n_query, d->n_ref, nullptr);
    const int64_t nq = d->n_query;
    const bool self = d->self_search != 0;
    TCR_CUDA(cudaMemsetAsync(W.work, 0, sizeof(int32_t) * 4, st));
    TCR_CUDA(cudaMemsetAsync(W.num_stray, 0, sizeof(int32_t), st));
    TCR_CUDA(cudaMemsetAsync(W.num_units, 0, sizeof(int32_t), st));
    TCR_CUDA(cudaMemsetAsync(W.num_flagged, 0, sizeof(int32_t), st));
    TCR_CUDA(cudaMemsetAsync(W.cursor, 0, sizeof(unsigned long long), st));
    TCR_CUDA(cudaMemsetAsync(&W.qparams->stats, 0, sizeof(SupportStats), st));
    if (d->query_sup && nq > 0) {
        support_stats_kernel<<<grid_for(nq, 256, num_sms() * 8), 256, 0, st>>>(d->query_sup, nq, &W.qparams->stats);
        note_launches(1);
    }
    query_params_kernel<<<1, 1, 0, st>>>(S.grid, d->mode, d->query_sup != nullptr, W.qparams);
    note_launches(1);
    if (nq > 0) {
        TCR_CUDA(cudaMemsetAsync(W.counts, 0, sizeof(int32_t) * nq, st));
        TCR_CUDA(cudaMemsetAsync(W.rec, 0xff, sizeof(int32_t) * nq, st));
        const int32_t* gstart;
        const int32_t* ngroups;
        if (self) {
            if (!same_sorted_points(d)) {
                pack_self_queries_kernel<<<grid_for(nq, 256), 256, 0, st>>>(sp, S.grid, d->query_pos, d->query_sup,
                                                                            S.rsidx, nq, W.qsorted, W.qsidx);
                note_launches(1);
            }
            gstart = S.cell_start;
            ngroups = S.num_cells;
        } else {
            // sort the queries by their own cells
            sort_state_init_kernel<<<1, 1, 0, st>>>(W.sort.state);
            note_launches(1);
            pack_points_kernel<<<grid_for(nq, 256), 256, 0, st>>>(sp, S.grid, d->query_pos, d->query_sup, nq, 1,
                                                                  W.pack, W.sort.keys[0], W.sort.vals[0],
                                                                  W.sort.state, 0);
            note_launches(1);
            TCR_CUDA(radix_sort_pairs(W.sort, nq, st));
            gather_sorted_kernel<<<grid_for(nq, 256), 256, 0, st>>>(S.grid, W.pack, W.sort.vals[0], W.sort.vals[1],
                                                                    W.sort.state, nq, W.qsorted, W.qsidx);
            note_launches(1);
            QueryGroupOut qo{sp, S.grid, W.qsorted, W.qgroup_start, W.qgroup_coords};
            RunFlagIn fi{S.grid, W.sort.keys[0], W.sort.keys[1], W.sort.state};
            TCR_CUDA(device_exclusive_scan<int32_t>(fi, qo, nq, W.scan_tiles32, W.num_qgroups, st));
            finish_cells_kernel<<<1, 1, 0, st>>>(W.qgroup_start, W.num_qgroups, nq);
            note_launches(1);
            gstart = W.qgroup_start;
            ngroups = W.num_qgroups;
        }
        BoundedUnitCountIn ui{gstart, ngroups};
        BoundedUnitOut uo{gstart, ngroups, W.unit_group, W.unit_t0, W.query_unit};
        TCR_CUDA(device_exclusive_scan<int32_t>(ui, uo, nq, W.scan_tiles32, W.num_units, st));
        WalkArgs a = make_walk(sp, S, W, self);
        if (same_sorted_points(d)) {  // the sorted queries are the sorted references
            a.qsorted = S.rsorted;
            a.qsidx = S.rsidx;
        }
        a.query_ids = d->query_ids;
        a.ref_ids = d->ref_ids;
        a.stage = stage;
        a.stage_cap = stage_capacity;
        // identical positions: every query sits in its group's cell
        a.no_stray_check = self && d->periodic_mask == 0 && d->query_pos == d->ref_pos;
        TCR_CUDA(dispatch_walk<CountLaunch>(a, d->dim, d->periodic_mask != 0, d->mode, dim3(walk_blocks(nq)),
                                            dim3(kWalkWarps * 32), sizeof(WalkSmem), st));
        note_launches(1);
        stray_kernel<false><<<grid_for(nq, 128, num_sms() * 4), 128, 0, st>>>(a);
        note_launches(1);
    }
    CountIn ci{W.counts, nq};
    OffsetOut oo{nq, offsets, indptr_out, row_entries_out};
    TCR_CUDA(device_exclusive_scan<int64_t>(ci, oo, nq + 1, W.scan_tiles64, W.total, st));
    info_kernel<<<1, 1, 0, st>>>(S.grid, W.total, W.num_stray, W.qparams, W.cursor, W.num_flagged, W.info);
    note_launches(1);
    if (info_out) TCR_CUDA(cudaMemcpyAsync(info_out, W.info, 8 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    return TCR_OK;
}

int tcr_emit(const tcr_search_desc* d, const void* structure, void* scratch, int64_t scratch_bytes,
             const int32_t* stage, const int64_t* offsets, int64_t* row_out, int64_t* col_out, int64_t out_capacity,
             void* stream) {
    int rc = validate(d, false);
    if (rc) return rc;
    int64_t need_w = 0;
    carve_scratch(nullptr, d->n_query, d->n_ref, &need_w);
    if (!structure || !scratch || scratch_bytes < need_w || !offsets)
        return set_error(TCR_ERR_INVALID, "workspace too small or offsets missing");
    cudaStream_t st = (cudaStream_t)stream;
    const SearchParams sp = make_params(d);
    Structure S = carve_structure(const_cast<void*>(structure), d->n_ref, nullptr);
    Scratch W = carve_scratch(scratch, d->n_query, d->n_ref, nullptr);
    const int64_t nq = d->n_query;
    if (nq <= 0) return TCR_OK;
    WalkArgs a = make_walk(sp, S, W, d->self_search != 0);
    if (same_sorted_points(d)) {
        a.qsorted = S.rsorted;
        a.qsidx = S.rsidx;
    }
    a.query_ids = d->query_ids;
    a.ref_ids = d->ref_ids;
    a.offsets = offsets;
    a.row_out = row_out;
    a.col_out = col_out;
    a.out_cap = out_capacity;
    if (out_capacity < 0 || (out_capacity > 0 && !col_out)) return set_error(TCR_ERR_INVALID, "bad output buffer");
    if (stage) {
        const int nsm = num_sms();
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)nsm * 16, (nq / 16 + kExpandWarps) / kExpandWarps));
        const int32_t* group_start = d->self_search ? S.cell_start : W.qgroup_start;
        TCR_CUDA(cudaFuncSetAttribute(expand_records_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(ExpandSmem)));
        expand_records_kernel<<<blocks, kExpandWarps * 32, sizeof(ExpandSmem), st>>>(
            stage, W.rec, W.num_units, W.unit_t0, W.unit_group, group_start, a.qsidx, offsets, d->query_ids, row_out,
            col_out, out_capacity);
        note_launches(1);
    }
    TCR_CUDA(cudaMemsetAsync(W.work + 1, 0, sizeof(int32_t), st));
    TCR_CUDA(dispatch_walk<EmitLaunch>(a, d->dim, d->periodic_mask != 0, d->mode, dim3(walk_blocks(nq)),
                                       dim3(kWalkWarps * 32), 0, st));
    note_launches(1);
    stray_kernel<true><<<grid_for(nq, 128, num_sms() * 4), 128, 0, st>>>(a);
    note_launches(1);
    return TCR_OK;
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
    int rc = validate(d);
    if (rc) return rc;
    if (!offsets || (pair_capacity > 0 && !col_out) || pair_capacity < 0)
        return set_error(TCR_ERR_INVALID, "offsets and a column buffer of pair_capacity entries are required");
    int64_t s_bytes = 0, w_bytes = 0;
    carve_structure(nullptr, d->n_ref, &s_bytes);
    carve_scratch(nullptr, d->n_query, d->n_ref, &w_bytes);
    if (s_bytes + w_bytes > kTcrStaticScratchBytes)
        return set_error(TCR_ERR_INVALID,
                         "tcr_search_noalloc: %lld query and %lld reference points need %lld bytes of scratch, "
                         "more than the static %lld bytes (about 180K points); use tcr_build_structure/"
                         "tcr_count/tcr_emit with caller-allocated buffers",
                         (long long)d->n_query, (long long)d->n_ref, (long long)(s_bytes + w_bytes),
                         (long long)kTcrStaticScratchBytes);
    void* base = nullptr;
    rc = static_scratch_address(&base);
    if (rc) return rc;
    void* structure = base;
    void* scratch = static_cast<char*>(base) + s_bytes;
    // Every kernel below initialises what it reads (counters, map, sort state), so the contents a
    // previous call left in the array do not matter.
    rc = tcr_build_structure(d, structure, s_bytes, scratch, w_bytes, stream);
    if (rc) return rc;
    int64_t info[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    rc = tcr_count(d, structure, scratch, w_bytes, nullptr, 0, offsets, indptr_out, row_entries_out, info, stream);
    if (rc) return rc;
    TCR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (total_out) *total_out = info[0];
    if (info[1]) return set_error(TCR_ERR_INVALID, "no valid cell grid for this domain and support");
    if (info[0] > pair_capacity)
        return set_error(TCR_ERR_INVALID, "tcr_search_noalloc: %lld pairs do not fit the %lld-entry output",
                         (long long)info[0], (long long)pair_capacity);
    if (info[0] == 0) return TCR_OK;
    return tcr_emit(d, structure, scratch, w_bytes, nullptr, offsets, row_out, col_out, pair_capacity, stream);
}
