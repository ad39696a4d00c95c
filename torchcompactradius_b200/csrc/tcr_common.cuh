// tcr_common.cuh -- shared device definitions for the compact-hashing neighbour search.
//
// Parity-critical arithmetic follows the reference's float path exactly
// (src/torchCompactRadius/cppSrc/common.h:95-129, neighborhoodDynamic.h:37-115):
//   * per dimension the difference is a double: moduloOp (float subtraction, the rest in double)
//     on periodic dimensions, the widened float subtraction otherwise;
//   * the running sum is float: sum = (float)((double)sum + diff*diff);
//   * dist = sqrtf(sum) and the test is a strict '<' against the mode's float threshold.
// Every double operation is written with an explicit __d*_rn intrinsic so that nvcc cannot
// contract it into an FMA; the float fast test below is decided exactly by this path whenever
// its result lies inside a narrow band around the threshold.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace tcr {

// Number of kernels this library has launched (all threads, every source file), for launch
// accounting.
inline unsigned long long g_launches = 0;
static inline void note_launches(int k) { __atomic_fetch_add(&g_launches, (unsigned long long)k, __ATOMIC_RELAXED); }

// A named NVTX range around one C-ABI call (the host-side enqueue of a build, count, emit or scatter
// stage), for timeline profilers; without a profiler attached a push or pop is one pointer check.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// The calling thread's last error message (tcr_last_error), shared by every source file.
inline thread_local char g_err[512];
static inline int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

// Checked build (-DTCR_CHECKED, debugging only): TCR_IN(i, n) verifies 0 <= i < n before an
// access; a failing check records its source line, the index and the bound (the first failure
// wins) and the access is skipped.  tcr_debug_checks() reads the record.  In a normal build the
// check is the constant true and costs nothing.
#ifdef TCR_CHECKED
static __device__ unsigned long long g_check[3];
__device__ __forceinline__ bool tcr_in_range(long long i, long long n, int line) {
    if (i >= 0 && i < n) return true;
    if (atomicCAS(&g_check[0], 0ull, (unsigned long long)line) == 0ull) {
        g_check[1] = (unsigned long long)i;
        g_check[2] = (unsigned long long)n;
    }
    return false;
}
#define TCR_IN(i, n) ::tcr::tcr_in_range((long long)(i), (long long)(n), __LINE__)
#define TCR_GUARD(i, n) TCR_IN(i, n)
#else
#define TCR_IN(i, n) true
// An index taken from device data (sort indices, cell ranges, staged records) is range-checked in
// every build before it addresses memory; an out-of-range index skips the access.
#define TCR_GUARD(i, n) ((unsigned long long)(long long)(i) < (unsigned long long)(long long)(n))
#endif

enum Mode : int { kGather = 0, kScatter = 1, kSymmetric = 2, kSuperSymmetric = 3 };

constexpr int kMaxDim = 3;
constexpr int kWarp = 32;
// Relative half-width of the band around thr^2 inside which the float fast test defers to the
// exact reference arithmetic.  The fast squared distance and the reference's rounded sum differ
// by at most ~10 float ulps and sqrtf's rounding moves the decision by < 2^-22 relative, so
// 4e-6 (~67 ulps) is a safe margin.
constexpr float kBandEps = 4e-6f;

// Host-filled description of one cloud's search: one entry per cloud in a device table (a single
// search is a table of one).  Global point indices count the clouds' points in table order.
struct CloudParams {
    int32_t dim;
    int32_t mode;
    int32_t periodic_mask;   // bit d: dimension d is periodic
    uint32_t hash_len;       // the reference's hashMapLength (bucket semantics)
    float dmin[3];
    float dmax[3];
    float ext[3];            // fl(dmax - dmin), as the reference computes it
    float hcell_override[3]; // > 0: use these per-dimension cell sizes instead of compute_h
    int32_t dedupe;          // clamped grid (multi-level): clamp cells, skip outside cells, no repeats
    int32_t n_query, n_ref;  // the cloud's points
    int32_t query_base, ref_base;  // global index of the cloud's first query / reference point
    int32_t pad;
    int64_t map_base, map_cap;     // the cloud's region of the lin -> cell map (capacity a power of two)
    const float* query_pos;  // [n_query * dim]
    const float* query_sup;  // [n_query] or null
    const float* ref_pos;    // [n_ref * dim]
    const float* ref_sup;    // [n_ref] or null
};

// Reduction record over one set of supports.
struct SupportStats {
    uint32_t max_key;        // float_key of the largest support (NaN propagates)
    int32_t bad;             // some support is not in [1e-18, 1e18] (negative, zero, tiny, huge, NaN)
};

// Device-computed grid description (one record in device memory).
struct GridParams {
    float hmax;              // computeGridSupport result
    float hcell;             // compute_h result (the reference's single cell size)
    float hcell_d[3];        // per-dimension cell size actually used (all hcell unless overridden)
    int32_t count[3];        // ceil(ext / hcell_d) as int32
    int32_t always_exact;    // 1: some support outside [1e-18, 1e18] or non-finite: exact test always
    int32_t error;           // nonzero: invalid grid (e.g. zero cells on a periodic dim)
    int32_t out_of_grid;     // some reference point's cell lies outside [0, count) (linear indices may alias)
    SupportStats ref_stats;  // over the reference supports (the candidates' thresholds)
    SupportStats build_query_stats;  // over the query supports seen at build time
};

// Per-search query-side parameters of the lean test (scratch).
struct QueryParams {
    SupportStats stats;      // over this search's query supports
    float qmax;              // largest query support (band of the fast test)
    int32_t exact_all;       // decide every pair with the exact reference test
    uint32_t coord_key;      // float64 inputs: float_key of the largest |coordinate| of the double positions
    int32_t pad;
};

// Ordered uint32 encoding of floats: a < b  <=>  key(a) < key(b); NaN maps above +inf.
__device__ __forceinline__ uint32_t float_key(float f) {
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7fffffffu) > 0x7f800000u) return 0xffffffffu;  // NaN: propagates through max
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
    if (k == 0xffffffffu) return __uint_as_float(0x7fc00000u);
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// hashing.h:20-34 -- uint32 wrap-around with the reference's primes; 1-D is c mod L.
__device__ __forceinline__ uint32_t ref_hash(int dim, const int32_t* c, uint32_t L) {
    if (dim == 1) return ((uint32_t)c[0]) % L;
    uint32_t h = (uint32_t)c[0] * 73856093u;
    h += (uint32_t)c[1] * 19349663u;
    if (dim == 3) h += (uint32_t)c[2] * 83492791u;
    return h % L;
}

// neighborhood.h:51-61 -- int32 wrap-around linear index.
__device__ __forceinline__ int32_t linear_index(int dim, const int32_t* c, const int32_t* cnt) {
    uint32_t lin = (uint32_t)c[0];
    uint32_t prod = (uint32_t)cnt[0];
    if (dim > 1) { lin += (uint32_t)c[1] * prod; prod *= (uint32_t)cnt[1]; }
    if (dim > 2) { lin += (uint32_t)c[2] * prod; }
    return (int32_t)lin;
}

// common.h:95-97 -- Python modulo.
__device__ __forceinline__ int32_t pymod(int32_t n, int32_t m) { return n >= 0 ? n % m : ((n % m) + m) % m; }

// cellTable.py:30 / neighborhoodDynamic.h:52 -- floor((x - min) / hCell) in float, to int32.
__device__ __forceinline__ int32_t cell_coord(float x, float lo, float hcell) {
    return (int32_t)floorf(__fdiv_rn(__fsub_rn(x, lo), hcell));
}

// util.py:387 torch.remainder(x - min, max - min) + min for float32 (fmod, +b if signs differ).
__device__ __forceinline__ float wrap_coord(float x, float lo, float ext) {
    float t = __fsub_rn(x, lo);
    float m = fmodf(t, ext);
    if (m != 0.0f && ((ext < 0.0f) != (m < 0.0f))) m = __fadd_rn(m, ext);
    return __fadd_rn(m, lo);
}

__device__ __forceinline__ float comp(const float4& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }

// Mode threshold in float, exactly as the reference evaluates it.
__device__ __forceinline__ float mode_threshold(int mode, float hi, float hj) {
    switch (mode) {
        case kGather: return hi;
        case kScatter: return hj;
        case kSymmetric: return __fdiv_rn(__fadd_rn(hi, hj), 2.0f);
        default: return (hi < hj) ? hj : hi;  // std::max(hi, hj)
    }
}

// What the exact test needs, small enough to pass by value into a non-inlined call.
struct ExactCtx {
    int32_t dim, mode, periodic_mask;
    float ext[3];
};
// The reference's exact distance test (common.h:106-129 at scalar_t=float).
static __device__ __noinline__ bool exact_pair_test(ExactCtx sp, float4 xi, float hi, float4 xj, float hj) {
    float sum = 0.0f;
    for (int d = 0; d < sp.dim; ++d) {
        float a = comp(xi, d), b = comp(xj, d);
        float pq = __fsub_rn(a, b);
        double diff;
        if ((sp.periodic_mask >> d) & 1) {
            double h = (double)(d == 0 ? sp.ext[0] : (d == 1 ? sp.ext[1] : sp.ext[2]));
            double half = __dmul_rn(h, 0.5);           // h / 2.0, exact
            double t = __dadd_rn((double)pq, half);
            double k = floor(__ddiv_rn(t, h));
            diff = __dsub_rn(__dsub_rn(t, __dmul_rn(k, h)), half);
        } else {
            diff = (double)pq;
        }
        sum = __double2float_rn(__dadd_rn((double)sum, __dmul_rn(diff, diff)));
    }
    float dist = __fsqrt_rn(sum);
    return dist < mode_threshold(sp.mode, hi, hj);
}

}  // namespace tcr
