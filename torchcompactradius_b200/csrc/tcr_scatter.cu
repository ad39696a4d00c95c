// tcr_scatter.cu -- deterministic reductions of values onto an index for sm_100a: the reference's
// scatter_sum / scatter_mul / scatter_mean / scatter_min / scatter_max operators
// (src/torchCompactRadius/cppSrc/sparseOperations/scatter.h:10-36), the consumers of a neighbour
// list in SPH and GNN codes (sums over each particle's neighbours).
//
// The reference's CPU loop (sparseOperations/scatter_cpu.cpp:56-77) walks src in row-major order
// and folds each element into out[b][index][k] with Reducer<>::update (reducer.h:44-66), one
// element after the other in the element type's own arithmetic; its CUDA kernel
// (scatter_cuda.cu:13-31) does the same folds with atomics in the order threads arrive.  Here each
// output element is owned by one thread that folds its elements in increasing e:
//   1. an index that is non-decreasing along e (the rows of a neighbour list) is used as it is;
//      any other index is sorted once by a stable radix sort of (slot, position) pairs;
//   2. the start of every output slot's run of elements is marked in an offsets array;
//   3. one thread per output element folds its run in order and writes the result once.
// No atomics touch the data and nothing is reassociated, so the results equal the reference's CPU
// operators bit for bit and repeat from run to run; min / max keep the first of equal values, as
// the CPU loop does (its strict comparisons).
#include <cfloat>
#include <climits>
#include <cstdint>
#include <mutex>
#include <type_traits>
#include <unordered_map>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tcr_common.cuh"
#include "tcr_scan.cuh"
#include "tcr_sort.cuh"
#include "../../include/tcr_b200.h"

namespace tcr {
namespace {

#define TCR_SCATTER_CUDA(call)                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return set_error(TCR_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

constexpr int kThreads = 256;
// Runs of empty slots longer than this are filled by a whole block instead of the marking thread.
constexpr int64_t kInlineGap = 16;

inline int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

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

inline int sm_count() {
    static int sms[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    int& s = sms[dev & 63];
    if (s == 0) {
        if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || s <= 0) s = 148;
    }
    return s;
}

// Grid of a grid-stride kernel over n items: enough blocks to fill every SM, no more than needed.
inline unsigned grid_for(int64_t n) {
    const int64_t want = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)sm_count() * 8;
    return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

// The same for a streaming kernel whose blocks all carry equal shares of the work: exactly the
// blocks that are resident at once (one wave), so no SM idles through a partial second wave.
template <typename Kern>
unsigned grid_resident(Kern kernel, int64_t n) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> per_sm;
    int nb = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = per_sm.find(reinterpret_cast<const void*>(kernel));
        if (it != per_sm.end()) {
            nb = it->second;
        } else {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kThreads, 0) != cudaSuccess || nb <= 0)
                nb = 4;
            per_sm[reinterpret_cast<const void*>(kernel)] = nb;
        }
    }
    const int64_t want = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)sm_count() * nb;
    return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

// ------------------------------------------------------------------------------------------
// element arithmetic, rounded the way the reference's CPU element types round: float and double
// operations are single IEEE operations (written as __*_rn intrinsics so nothing is contracted),
// Half / BFloat16 compute in float and round to nearest even after every operation (c10::Half
// and c10::BFloat16 arithmetic), integers wrap in two's complement.
template <typename T>
struct Num;

template <>
struct Num<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ bool lt(float a, float b) { return a < b; }
    static __device__ __forceinline__ bool eq(float a, float b) { return a == b; }
    static __device__ __forceinline__ float zero() { return 0.0f; }
    static __device__ __forceinline__ float one() { return 1.0f; }
    static __device__ __forceinline__ float maxv() { return FLT_MAX; }
    static __device__ __forceinline__ float lowest() { return -FLT_MAX; }
};

template <>
struct Num<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ bool lt(double a, double b) { return a < b; }
    static __device__ __forceinline__ bool eq(double a, double b) { return a == b; }
    static __device__ __forceinline__ double zero() { return 0.0; }
    static __device__ __forceinline__ double one() { return 1.0; }
    static __device__ __forceinline__ double maxv() { return DBL_MAX; }
    static __device__ __forceinline__ double lowest() { return -DBL_MAX; }
};

template <>
struct Num<__half> {
    static __device__ __forceinline__ float f(__half a) { return __half2float(a); }
    static __device__ __forceinline__ __half h(float a) { return __float2half_rn(a); }
    static __device__ __forceinline__ __half add(__half a, __half b) { return h(__fadd_rn(f(a), f(b))); }
    static __device__ __forceinline__ __half mul(__half a, __half b) { return h(__fmul_rn(f(a), f(b))); }
    static __device__ __forceinline__ __half div(__half a, __half b) { return h(__fdiv_rn(f(a), f(b))); }
    static __device__ __forceinline__ bool lt(__half a, __half b) { return f(a) < f(b); }
    static __device__ __forceinline__ bool eq(__half a, __half b) { return f(a) == f(b); }
    static __device__ __forceinline__ __half zero() { return __ushort_as_half((unsigned short)0x0000u); }
    static __device__ __forceinline__ __half one() { return __ushort_as_half((unsigned short)0x3C00u); }
    static __device__ __forceinline__ __half maxv() { return __ushort_as_half((unsigned short)0x7BFFu); }    // 65504
    static __device__ __forceinline__ __half lowest() { return __ushort_as_half((unsigned short)0xFBFFu); }  // -65504
};

template <>
struct Num<__nv_bfloat16> {
    using B = __nv_bfloat16;
    static __device__ __forceinline__ float f(B a) { return __bfloat162float(a); }
    static __device__ __forceinline__ B h(float a) { return __float2bfloat16_rn(a); }
    static __device__ __forceinline__ B add(B a, B b) { return h(__fadd_rn(f(a), f(b))); }
    static __device__ __forceinline__ B mul(B a, B b) { return h(__fmul_rn(f(a), f(b))); }
    static __device__ __forceinline__ B div(B a, B b) { return h(__fdiv_rn(f(a), f(b))); }
    static __device__ __forceinline__ bool lt(B a, B b) { return f(a) < f(b); }
    static __device__ __forceinline__ bool eq(B a, B b) { return f(a) == f(b); }
    static __device__ __forceinline__ B zero() { return __ushort_as_bfloat16((unsigned short)0x0000u); }
    static __device__ __forceinline__ B one() { return __ushort_as_bfloat16((unsigned short)0x3F80u); }
    static __device__ __forceinline__ B maxv() { return __ushort_as_bfloat16((unsigned short)0x7F7Fu); }
    static __device__ __forceinline__ B lowest() { return __ushort_as_bfloat16((unsigned short)0xFF7Fu); }
};

// Integers: the reference's `*val + new_val` / `*val * new_val` promote to int (or stay 64-bit)
// and are stored back with truncation; unsigned arithmetic gives the same low bits without
// signed overflow.  Division is the floor division of `div_(count, "floor")` by a count >= 1.
template <typename T, typename U, T MAXV, T LOWV>
struct NumInt {
    static __device__ __forceinline__ T add(T a, T b) { return (T)((U)a + (U)b); }
    static __device__ __forceinline__ T mul(T a, T b) { return (T)((U)a * (U)b); }
    static __device__ __forceinline__ T div(T a, T b) {  // b >= 1 (a clamped count)
        T q = (T)(a / b);
        if constexpr (std::is_signed<T>::value) {
            if ((T)(a % b) != 0 && a < 0) q = (T)(q - 1);
        }
        return q;
    }
    static __device__ __forceinline__ bool lt(T a, T b) { return a < b; }
    static __device__ __forceinline__ bool eq(T a, T b) { return a == b; }
    static __device__ __forceinline__ T zero() { return (T)0; }
    static __device__ __forceinline__ T one() { return (T)1; }
    static __device__ __forceinline__ T maxv() { return MAXV; }
    static __device__ __forceinline__ T lowest() { return LOWV; }
};
template <>
struct Num<uint8_t> : NumInt<uint8_t, uint32_t, (uint8_t)255, (uint8_t)0> {};
template <>
struct Num<int8_t> : NumInt<int8_t, uint32_t, (int8_t)127, (int8_t)-128> {};
template <>
struct Num<int16_t> : NumInt<int16_t, uint32_t, (int16_t)32767, (int16_t)-32768> {};
template <>
struct Num<int32_t> : NumInt<int32_t, uint32_t, INT_MAX, INT_MIN> {};
template <>
struct Num<int64_t> : NumInt<int64_t, unsigned long long, LLONG_MAX, LLONG_MIN> {};

template <typename T, int R>
__device__ __forceinline__ T reduce_init() {
    using N = Num<T>;
    if (R == TCR_REDUCE_MUL) return N::one();
    if (R == TCR_REDUCE_MIN) return N::maxv();
    if (R == TCR_REDUCE_MAX) return N::lowest();
    return N::zero();
}

// ------------------------------------------------------------------------------------------
// index statistics: min, max and the number of descents
__global__ void stats_init_kernel(int64_t* stats) {
    stats[0] = LLONG_MAX;
    stats[1] = LLONG_MIN;
    stats[2] = 0;
}

// One warp's contribution to stats (min, max, descents); every lane of the warp calls it.
__device__ __forceinline__ void stats_add(int64_t* stats, long long lo, long long hi, unsigned long long desc) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long l2 = __shfl_down_sync(0xffffffffu, lo, o);
        const long long h2 = __shfl_down_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
        desc += __shfl_down_sync(0xffffffffu, desc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (lo != LLONG_MAX) atomicMin(reinterpret_cast<long long*>(&stats[0]), lo);
        if (hi != LLONG_MIN) atomicMax(reinterpret_cast<long long*>(&stats[1]), hi);
        if (desc) atomicAdd(reinterpret_cast<unsigned long long*>(&stats[2]), desc);
    }
}

__global__ void __launch_bounds__(kThreads) index_stats_kernel(const int64_t* __restrict__ idx, int64_t n,
                                                               int64_t* stats) {
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    unsigned long long desc = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long v = idx[i];
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
        if (i > 0 && v < idx[i - 1]) ++desc;
    }
    stats_add(stats, lo, hi, desc);
}

// The fold may run: every index value lies in [0, N) and, when the index is used in its own
// order, it never descends.  Otherwise the folds write nothing and the caller, who reads the
// statistics back, reports the index or sorts it.
__device__ __forceinline__ bool stats_allow(const int64_t* stats, int64_t N, bool need_sorted) {
    return stats[0] >= 0 && stats[1] < N && (!need_sorted || stats[2] == 0);
}

// ------------------------------------------------------------------------------------------
// sort keys: the output slot of every element (slot = index for an index over e, (b*K + k)*N +
// index for a full index), with all ones for an index outside [0, N) so that it sorts past every
// slot; the values are the element's e (index over e) or flat src position (full index).
template <typename K>
__global__ void sort_init_kernel(SortStateT<K>* st) { sort_state_reset(st); }

template <typename K, bool FULL>
__global__ void __launch_bounds__(kThreads) pack_keys_kernel(const int64_t* __restrict__ idx, int64_t M, int64_t E,
                                                             int64_t Kdim, int64_t N, K* keys, int32_t* vals,
                                                             SortStateT<K>* st, int64_t* stats) {
    K kmin = ~(K)0, kmax = 0;
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        const int64_t v = idx[i];
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
        K key = ~(K)0;
        if (v >= 0 && v < N) {
            if (FULL) {
                const int64_t k = i % Kdim;
                const int64_t b = i / (E * Kdim);
                key = (K)((b * Kdim + k) * N + v);
            } else {
                key = (K)v;
            }
        }
        keys[i] = key;
        vals[i] = (int32_t)i;
        kmin = key < kmin ? key : kmin;
        kmax = key > kmax ? key : kmax;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const K a = __shfl_down_sync(0xffffffffu, kmin, o);
        const K b = __shfl_down_sync(0xffffffffu, kmax, o);
        kmin = a < kmin ? a : kmin;
        kmax = b > kmax ? b : kmax;
    }
    if ((threadIdx.x & 31) == 0) {
        if (kmin != ~(K)0) atomicMin(&st->key_min, kmin);
        if (kmax != 0) atomicMax(&st->key_max, kmax);
    }
    stats_add(stats, lo, hi, 0ull);
}

// ------------------------------------------------------------------------------------------
// run starts: off[s] = the first position (in sorted order) whose slot is >= s, for s in
// [0, nslots]; off[nslots] also excludes every element outside [0, N).  Position j writes the
// slots after its predecessor's up to its own; runs of empty slots longer than kInlineGap go to a
// list that fill_gaps_kernel writes with whole blocks.
__device__ __forceinline__ int64_t key_slot(int64_t k, int64_t nslots) {
    return k < 0 ? -1 : (k > nslots ? nslots : k);
}
__device__ __forceinline__ int64_t key_slot(uint32_t k, int64_t nslots) {
    return (int64_t)k > nslots ? nslots : (int64_t)k;
}
__device__ __forceinline__ int64_t key_slot(unsigned long long k, int64_t nslots) {
    return k > (unsigned long long)nslots ? nslots : (int64_t)k;
}

__device__ __forceinline__ void mark_range(int64_t lo, int64_t hi, int64_t value, int64_t* off, int64_t* gaps,
                                           unsigned long long* ngaps, int64_t gap_cap, unsigned long long* descents) {
    if (hi < lo) return;
    if (hi - lo + 1 > kInlineGap) {
        // The runs of a non-decreasing index are disjoint, so at most gap_cap of them are longer
        // than kInlineGap; more means the index descends (its fold will not run): count a descent
        // and drop the run, so that an unsorted index costs bounded work here.
        const unsigned long long g = atomicAdd(ngaps, 1ull);
        if (g < (unsigned long long)gap_cap) {
            gaps[3 * g] = lo;
            gaps[3 * g + 1] = hi;
            gaps[3 * g + 2] = value;
        } else {
            atomicAdd(descents, 1ull);
        }
        return;
    }
    for (int64_t s = lo; s <= hi; ++s) off[s] = value;
}

// Eight consecutive keys from base (fewer at the end of the array): loaded before any of them is
// used, with 16-byte vector loads when the keys are 16-byte aligned, so each thread keeps eight
// loads in flight.
constexpr int kMarkKeys = 8;

template <typename KT>
__device__ __forceinline__ void load_keys(const KT* keys, int64_t base, int64_t M, bool aligned, KT (&v)[kMarkKeys]) {
    if (base + kMarkKeys <= M) {
        if constexpr (sizeof(KT) == 8) {
            if (aligned) {
                const longlong2* p = reinterpret_cast<const longlong2*>(keys + base);
#pragma unroll
                for (int k = 0; k < kMarkKeys / 2; ++k) {
                    const longlong2 q = p[k];
                    v[2 * k] = (KT)q.x;
                    v[2 * k + 1] = (KT)q.y;
                }
                return;
            }
        } else {
            if (aligned) {
                const uint4* p = reinterpret_cast<const uint4*>(keys + base);
#pragma unroll
                for (int k = 0; k < kMarkKeys / 4; ++k) {
                    const uint4 q = p[k];
                    v[4 * k] = (KT)q.x;
                    v[4 * k + 1] = (KT)q.y;
                    v[4 * k + 2] = (KT)q.z;
                    v[4 * k + 3] = (KT)q.w;
                }
                return;
            }
        }
#pragma unroll
        for (int k = 0; k < kMarkKeys; ++k) v[k] = keys[base + k];
    } else {
#pragma unroll
        for (int k = 0; k < kMarkKeys; ++k) v[k] = base + k < M ? keys[base + k] : (KT)0;
    }
}

// RAW: the keys are the caller's index in its own order (min, max and descents go to stats).
// Each thread takes kMarkKeys consecutive positions.  Most such chunks lie inside one run (a run
// of a neighbour list's rows is ~50 long): a chunk that never descends and ends on the key before
// it marks nothing, so it costs a few compares; only chunks where the key changes mark run starts.
template <typename KT, bool RAW>
__global__ void __launch_bounds__(kThreads) mark_runs_kernel(const KT* k0, const KT* k1, const int32_t* sel, int64_t M,
                                                             int64_t nslots, int64_t* off, int64_t* gaps,
                                                             unsigned long long* ngaps, int64_t gap_cap,
                                                             int64_t* stats) {
    const KT* keys = (sel && *sel) ? k1 : k0;
    const bool aligned = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
    unsigned long long* dsc = reinterpret_cast<unsigned long long*>(&stats[2]);
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    unsigned long long desc = 0;
    const int64_t nchunks = (M + kMarkKeys - 1) / kMarkKeys;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += stride) {
        const int64_t base = c * kMarkKeys;
        const int nk = M - base < kMarkKeys ? (int)(M - base) : kMarkKeys;
        KT v[kMarkKeys];
        load_keys(keys, base, M, aligned, v);
        const KT pk = base == 0 ? v[0] : keys[base - 1];
        bool mono = true;
        KT last = v[0];
#pragma unroll
        for (int k = 0; k < kMarkKeys; ++k) {
            if (k < nk) {
                const KT before = k == 0 ? pk : v[k - 1];
                if (v[k] < before) {
                    mono = false;
                    if (RAW) ++desc;
                }
                last = v[k];
            }
        }
        if (RAW) {
            if (mono) {
                const long long a = (long long)v[0], b = (long long)last;
                lo = a < lo ? a : lo;
                hi = b > hi ? b : hi;
            } else {
#pragma unroll
                for (int k = 0; k < kMarkKeys; ++k) {
                    if (k < nk) {
                        const long long x = (long long)v[k];
                        lo = x < lo ? x : lo;
                        hi = x > hi ? x : hi;
                    }
                }
            }
        }
        if (!(mono && base > 0 && last == pk)) {  // some run starts in this chunk
            int64_t prev = base == 0 ? -1 : key_slot(pk, nslots);
#pragma unroll
            for (int k = 0; k < kMarkKeys; ++k) {
                // a key equal to the one before it starts no run (same slot): one compare
                if (k < nk && (v[k] != (k == 0 ? pk : v[k - 1]) || (k == 0 && base == 0))) {
                    const int64_t cur = key_slot(v[k], nslots);
                    mark_range(prev + 1 < 0 ? 0 : prev + 1, cur, base + k, off, gaps, ngaps, gap_cap, dsc);
                    prev = cur;
                }
            }
        }
        if (base + nk == M) {  // after the last key: the remaining slots start at M
            const int64_t cur = key_slot(last, nslots);
            mark_range(cur + 1 < 0 ? 0 : cur + 1, nslots, M, off, gaps, ngaps, gap_cap, dsc);
        }
    }
    if (RAW) stats_add(stats, lo, hi, desc);
}

// need_sorted: the runs come from the caller's index in its own order, which holds only when it
// never descends (otherwise the runs may overlap and the fold will not run: nothing to fill).
__global__ void __launch_bounds__(kThreads) fill_gaps_kernel(const int64_t* gaps, const unsigned long long* ngaps,
                                                             int64_t gap_cap, int64_t* off, const int64_t* stats,
                                                             int need_sorted) {
    if (need_sorted && stats[2] != 0) return;
    unsigned long long n = *ngaps;
    if (n > (unsigned long long)gap_cap) n = (unsigned long long)gap_cap;
    for (unsigned long long g = blockIdx.x; g < n; g += gridDim.x) {
        const int64_t lo = gaps[3 * g], hi = gaps[3 * g + 1], v = gaps[3 * g + 2];
        for (int64_t s = lo + threadIdx.x; s <= hi; s += blockDim.x) off[s] = v;
    }
}

// ------------------------------------------------------------------------------------------
// the fold: one thread per output element [b][n][k], its run in increasing e.
// P = 0: index over e, non-decreasing (run positions are e); P = 1: index over e, sorted order in
// perm (perm[j] = e); P = 2: full index (perm[j] = flat src position).
struct FoldArgs {
    const void* src;
    void* out;
    int64_t* arg;
    const int64_t* off;
    const int32_t* perm0;
    const int32_t* perm1;
    const int32_t* sel;   // which perm buffer holds the sorted order (null: perm0)
    const int64_t* stats; // index statistics of this call (stats_allow)
    int64_t B, E, K, N;
    int32_t accumulate;
};

template <typename T, int R>
struct Fold {
    T acc, cnt;
    int64_t arg;
    __device__ __forceinline__ void take(T v, int64_t e) {
        using Nm = Num<T>;
        if (R == TCR_REDUCE_SUM) {
            acc = Nm::add(acc, v);
        } else if (R == TCR_REDUCE_MEAN) {
            acc = Nm::add(acc, v);
            cnt = Nm::add(cnt, Nm::one());
        } else if (R == TCR_REDUCE_MUL) {
            acc = Nm::mul(acc, v);
        } else if (R == TCR_REDUCE_MIN) {
            if (Nm::lt(v, acc)) { acc = v; arg = e; }
        } else {
            if (Nm::lt(acc, v)) { acc = v; arg = e; }
        }
    }
};

template <typename T, int R>
__device__ __forceinline__ void fold_write(const FoldArgs& a, T* out, int64_t t, const Fold<T, R>& f) {
    using Nm = Num<T>;
    if (R == TCR_REDUCE_MEAN) {
        T c = f.cnt;
        if (Nm::lt(c, Nm::one())) c = Nm::one();
        out[t] = Nm::div(f.acc, c);
    } else if (R == TCR_REDUCE_MIN || R == TCR_REDUCE_MAX) {
        T v = f.acc;
        if (!a.accumulate && Nm::eq(v, reduce_init<T, R>())) v = Nm::zero();
        out[t] = v;
        a.arg[t] = f.arg;
    } else {
        out[t] = f.acc;
    }
}

// Index over e, non-decreasing, one value per (b, e) (K == 1): a block owns kThreads consecutive
// rows of one b, whose elements are one contiguous range of src.  The range streams through
// shared memory in tiles with coalesced loads; each thread folds its own row from the tile in
// order.
constexpr int kFoldTileBytes = 16384;

template <typename T, int R>
__global__ void __launch_bounds__(kThreads) fold_rows_kernel(FoldArgs a) {
    using Nm = Num<T>;
    constexpr int TILE = kFoldTileBytes / (int)sizeof(T);
    __shared__ __align__(16) unsigned char tile_raw[kFoldTileBytes];
    T* tile = reinterpret_cast<T*>(tile_raw);
    if (!stats_allow(a.stats, a.N, true)) return;
    const T* __restrict__ src = static_cast<const T*>(a.src);
    T* __restrict__ out = static_cast<T*>(a.out);
    const int64_t M = a.E;
    const int64_t rb = (a.N + kThreads - 1) / kThreads;
    for (int64_t blk = blockIdx.x; blk < a.B * rb; blk += gridDim.x) {
        const int64_t b = blk / rb, n0 = (blk % rb) * kThreads;
        const int64_t n = n0 + threadIdx.x;
        const int64_t nend = n0 + kThreads < a.N ? n0 + kThreads : a.N;
        int64_t E0 = a.off[n0], E1 = a.off[nend];
        E0 = E0 < 0 ? 0 : (E0 > M ? M : E0);
        E1 = E1 < E0 ? E0 : (E1 > M ? M : E1);
        int64_t lo = E1, hi = E1;
        if (n < a.N) {
            lo = a.off[n];
            hi = a.off[n + 1];
            lo = lo < E0 ? E0 : (lo > E1 ? E1 : lo);
            hi = hi < lo ? lo : (hi > E1 ? E1 : hi);
        }
        Fold<T, R> f;
        f.acc = (a.accumulate && n < a.N) ? out[b * a.N + n] : reduce_init<T, R>();
        f.cnt = Nm::zero();
        f.arg = a.E;
        const T* s = src + b * a.E;
        for (int64_t t0 = E0; t0 < E1; t0 += TILE) {
            const int len = (int)(E1 - t0 < TILE ? E1 - t0 : TILE);
            __syncthreads();  // the previous tile is consumed
#pragma unroll 8
            for (int i = threadIdx.x; i < len; i += kThreads) tile[i] = s[t0 + i];
            __syncthreads();
            const int64_t j0 = lo > t0 ? lo : t0;
            const int64_t j1 = hi < t0 + len ? hi : t0 + len;
            for (int64_t j = j0; j < j1; ++j) f.take(tile[j - t0], j);
        }
        if (n < a.N) fold_write<T, R>(a, out, b * a.N + n, f);
    }
}

template <typename T, int R, int P>
__global__ void __launch_bounds__(kThreads) fold_kernel(FoldArgs a) {
    using Nm = Num<T>;
    if (!stats_allow(a.stats, a.N, P == 0)) return;
    const T* __restrict__ src = static_cast<const T*>(a.src);
    T* __restrict__ out = static_cast<T*>(a.out);
    const int32_t* __restrict__ perm = (a.sel && *a.sel) ? a.perm1 : a.perm0;
    const int64_t total = a.B * a.N * a.K;
    const int64_t M = P == 2 ? a.B * a.E * a.K : a.E;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int64_t k = 0, n, b;
        if (a.K == 1) {
            n = t % a.N;
            b = t / a.N;
        } else {
            k = t % a.K;
            const int64_t bn = t / a.K;
            n = bn % a.N;
            b = bn / a.N;
        }
        const int64_t slot = P == 2 ? (b * a.K + k) * a.N + n : n;
        int64_t lo = a.off[slot], hi = a.off[slot + 1];
        lo = lo < 0 ? 0 : (lo > M ? M : lo);
        hi = hi < lo ? lo : (hi > M ? M : hi);
        Fold<T, R> f;
        f.acc = a.accumulate ? out[t] : reduce_init<T, R>();
        f.cnt = Nm::zero();
        f.arg = a.E;
        if (P == 0) {
            const T* s = src + b * a.E * a.K + k;
            int64_t j = lo;
            for (; j + 4 <= hi; j += 4) {  // four loads in flight, folded in order
                const T v0 = s[j * a.K], v1 = s[(j + 1) * a.K], v2 = s[(j + 2) * a.K], v3 = s[(j + 3) * a.K];
                f.take(v0, j);
                f.take(v1, j + 1);
                f.take(v2, j + 2);
                f.take(v3, j + 3);
            }
            for (; j < hi; ++j) f.take(s[j * a.K], j);
        } else if (P == 1) {
            const T* s = src + b * a.E * a.K + k;
            for (int64_t j = lo; j < hi; ++j) {
                const int64_t e = perm[j];
                f.take(s[e * a.K], e);
            }
        } else {
            for (int64_t j = lo; j < hi; ++j) {
                const int64_t pos = perm[j];
                f.take(src[pos], (pos / a.K) % a.E);
            }
        }
        fold_write<T, R>(a, out, t, f);
    }
}

template <typename T, int R, int P>
void launch_one(const FoldArgs& fa, unsigned grid, cudaStream_t st) {
    if constexpr (P == 3)
        fold_rows_kernel<T, R><<<grid, kThreads, 0, st>>>(fa);
    else
        fold_kernel<T, R, P><<<grid, kThreads, 0, st>>>(fa);
}

// P = 0, 1, 2: fold_kernel paths; P = 3: fold_rows_kernel (index over e, non-decreasing, K == 1).
template <typename T, int P>
cudaError_t launch_fold_r(int reduce, const FoldArgs& fa, unsigned grid, cudaStream_t st) {
    switch (reduce) {
        case TCR_REDUCE_SUM: launch_one<T, TCR_REDUCE_SUM, P>(fa, grid, st); break;
        case TCR_REDUCE_MEAN: launch_one<T, TCR_REDUCE_MEAN, P>(fa, grid, st); break;
        case TCR_REDUCE_MUL: launch_one<T, TCR_REDUCE_MUL, P>(fa, grid, st); break;
        case TCR_REDUCE_MIN: launch_one<T, TCR_REDUCE_MIN, P>(fa, grid, st); break;
        default: launch_one<T, TCR_REDUCE_MAX, P>(fa, grid, st); break;
    }
    return cudaGetLastError();
}

template <int P>
cudaError_t launch_fold(int dtype, int reduce, const FoldArgs& fa, unsigned grid, cudaStream_t st) {
    switch (dtype) {
        case TCR_DTYPE_U8: return launch_fold_r<uint8_t, P>(reduce, fa, grid, st);
        case TCR_DTYPE_I8: return launch_fold_r<int8_t, P>(reduce, fa, grid, st);
        case TCR_DTYPE_I16: return launch_fold_r<int16_t, P>(reduce, fa, grid, st);
        case TCR_DTYPE_I32: return launch_fold_r<int32_t, P>(reduce, fa, grid, st);
        case TCR_DTYPE_I64: return launch_fold_r<int64_t, P>(reduce, fa, grid, st);
        case TCR_DTYPE_F16: return launch_fold_r<__half, P>(reduce, fa, grid, st);
        case TCR_DTYPE_BF16: return launch_fold_r<__nv_bfloat16, P>(reduce, fa, grid, st);
        case TCR_DTYPE_F32: return launch_fold_r<float, P>(reduce, fa, grid, st);
        default: return launch_fold_r<double, P>(reduce, fa, grid, st);
    }
}

int elem_bytes(int dtype) {
    switch (dtype) {
        case TCR_DTYPE_U8:
        case TCR_DTYPE_I8: return 1;
        case TCR_DTYPE_I16:
        case TCR_DTYPE_F16:
        case TCR_DTYPE_BF16: return 2;
        case TCR_DTYPE_I32:
        case TCR_DTYPE_F32: return 4;
        default: return 8;
    }
}

// ------------------------------------------------------------------------------------------
// workspace
struct Plan {
    int path;             // P of fold_kernel
    bool wide;            // 64-bit sort keys
    int64_t M;            // elements (sort keys)
    int64_t nslots;       // output slots (run starts)
    int64_t gap_cap;      // capacity of the long-gap list
};

struct Work {
    int64_t* stats;
    int64_t* off;
    int64_t* gaps;
    unsigned long long* ngaps;
    void* state;
    void* keys[2];
    int32_t* vals[2];
    int32_t* hist;
    int32_t* tile_sums;
};

int64_t carve_work(const Plan& p, char* base, Work& w) {
    Carve c{base, 0};
    w.stats = c.take<int64_t>(4);
    w.off = c.take<int64_t>(p.nslots + 1);
    w.gaps = c.take<int64_t>(3 * p.gap_cap);
    w.ngaps = c.take<unsigned long long>(1);
    w.state = w.keys[0] = w.keys[1] = nullptr;
    w.vals[0] = w.vals[1] = nullptr;
    w.hist = w.tile_sums = nullptr;
    if (p.path != 0) {
        const int64_t kb = p.wide ? 8 : 4;
        w.state = p.wide ? (void*)c.take<SortState64>(1) : (void*)c.take<SortState32>(1);
        w.keys[0] = c.take<char>(p.M * kb);
        w.keys[1] = c.take<char>(p.M * kb);
        w.vals[0] = c.take<int32_t>(p.M);
        w.vals[1] = c.take<int32_t>(p.M);
        const int64_t nh = sort_hist_elems(p.M);
        w.hist = c.take<int32_t>(nh);
        w.tile_sums = c.take<int32_t>(kBins);  // the sort's digit totals
    }
    return c.off;
}

// Checks the description (and, for a call that runs, its pointers) and plans the path.
int check_desc(const tcr_scatter_desc* d, Plan& p, bool pointers) {
    if (!d) return set_error(TCR_ERR_INVALID, "tcr_scatter: null description");
    if (d->reduce < TCR_REDUCE_SUM || d->reduce > TCR_REDUCE_MAX)
        return set_error(TCR_ERR_INVALID, "tcr_scatter: invalid reduce %d", d->reduce);
    if (d->dtype < TCR_DTYPE_U8 || d->dtype > TCR_DTYPE_F64)
        return set_error(TCR_ERR_INVALID, "tcr_scatter: invalid dtype %d", d->dtype);
    if (d->B < 0 || d->E < 0 || d->K < 0 || d->N < 0)
        return set_error(TCR_ERR_INVALID, "tcr_scatter: negative size");
    const double outs = (double)d->B * (double)d->N * (double)d->K;
    const double elems = (double)d->B * (double)d->E * (double)d->K;
    if (outs > 9.0e18 || elems > 9.0e18) return set_error(TCR_ERR_INVALID, "tcr_scatter: sizes overflow int64");
    const bool minmax = d->reduce == TCR_REDUCE_MIN || d->reduce == TCR_REDUCE_MAX;
    const int64_t nout = d->B * d->N * d->K, nel = d->B * d->E * d->K;
    if (pointers && nout > 0 && !d->out) return set_error(TCR_ERR_INVALID, "tcr_scatter: missing out");
    if (pointers && nout > 0 && minmax && !d->arg_out)
        return set_error(TCR_ERR_INVALID, "tcr_scatter: min / max need arg_out");
    if (pointers && nel > 0 && (!d->src || !d->index))
        return set_error(TCR_ERR_INVALID, "tcr_scatter: missing src or index");
    p.path = d->index_full ? 2 : (d->index_sorted ? 0 : 1);
    p.M = d->index_full ? nel : d->E;
    p.nslots = d->index_full ? nout : d->N;
    if (p.path != 0 && p.M >= 0x7fffffffLL)
        return set_error(TCR_ERR_INVALID, "tcr_scatter: an index that needs sorting must have < 2^31 entries (got %lld)",
                         (long long)p.M);
    p.wide = p.nslots >= 0xffffffffLL;
    p.gap_cap = (p.nslots + 1) / (kInlineGap + 1) + 2;
    return TCR_OK;
}

template <typename K>
cudaError_t sort_path(const tcr_scatter_desc* d, const Plan& p, const Work& w, cudaStream_t st) {
    SortStateT<K>* state = static_cast<SortStateT<K>*>(w.state);
    K* k0 = static_cast<K*>(w.keys[0]);
    K* k1 = static_cast<K*>(w.keys[1]);
    sort_init_kernel<K><<<1, 1, 0, st>>>(state);
    if (p.path == 2)
        pack_keys_kernel<K, true><<<grid_for(p.M), kThreads, 0, st>>>(d->index, p.M, d->E, d->K, d->N, k0, w.vals[0],
                                                                       state, w.stats);
    else
        pack_keys_kernel<K, false><<<grid_for(p.M), kThreads, 0, st>>>(d->index, p.M, d->E, d->K, d->N, k0, w.vals[0],
                                                                        state, w.stats);
    note_launches(2);
    SortWorkspaceT<K> ws;
    ws.keys[0] = k0;
    ws.keys[1] = k1;
    ws.vals[0] = w.vals[0];
    ws.vals[1] = w.vals[1];
    ws.hist = w.hist;
    ws.tile_sums = w.tile_sums;
    ws.state = state;
    cudaError_t e = radix_sort_pairs<K>(ws, p.M, st);
    if (e != cudaSuccess) return e;
    const int32_t* sel = &state->sel[key_passes<K>()];
    const unsigned mgrid = grid_resident(mark_runs_kernel<K, false>, (p.M + kMarkKeys - 1) / kMarkKeys);
    mark_runs_kernel<K, false><<<mgrid, kThreads, 0, st>>>(k0, k1, sel, p.M, p.nslots, w.off, w.gaps, w.ngaps, p.gap_cap,
                                                           w.stats);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace
}  // namespace tcr

using namespace tcr;

extern "C" {

int64_t tcr_scatter_desc_bytes(void) { return (int64_t)sizeof(tcr_scatter_desc); }

int tcr_index_stats(const int64_t* index, int64_t n, int64_t* stats, int64_t* stats_host, void* stream) {
    NvtxRange nvtx_("tcr_index_stats");
    if (n < 0 || !stats || (n > 0 && !index)) return set_error(TCR_ERR_INVALID, "tcr_index_stats: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    stats_init_kernel<<<1, 1, 0, st>>>(stats);
    note_launches(1);
    if (n > 0) {
        index_stats_kernel<<<grid_for(n), kThreads, 0, st>>>(index, n, stats);
        note_launches(1);
    }
    TCR_SCATTER_CUDA(cudaGetLastError());
    if (stats_host) TCR_SCATTER_CUDA(cudaMemcpyAsync(stats_host, stats, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    return TCR_OK;
}

int tcr_scatter_sizes(const tcr_scatter_desc* d, int64_t* scratch_bytes) {
    Plan p;
    int rc = check_desc(d, p, false);
    if (rc) return rc;
    Work w;
    const int64_t bytes = carve_work(p, nullptr, w);
    if (scratch_bytes) *scratch_bytes = bytes;
    return TCR_OK;
}

int tcr_scatter(const tcr_scatter_desc* d, void* scratch, int64_t scratch_bytes, int64_t* stats_host, void* stream) {
    NvtxRange nvtx_("tcr_scatter");
    Plan p;
    int rc = check_desc(d, p, true);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nout = d->B * d->N * d->K;
    if (nout == 0) return TCR_OK;
    const bool minmax = d->reduce == TCR_REDUCE_MIN || d->reduce == TCR_REDUCE_MAX;
    if (d->E == 0) {  // no elements: the reference returns out filled with 0 (scatter_cpu.cpp:45-49)
        if (!d->accumulate) TCR_SCATTER_CUDA(cudaMemsetAsync(d->out, 0, (size_t)nout * elem_bytes(d->dtype), st));
        if (minmax) TCR_SCATTER_CUDA(cudaMemsetAsync(d->arg_out, 0, (size_t)nout * sizeof(int64_t), st));
        return TCR_OK;
    }
    Work w;
    const int64_t need = carve_work(p, nullptr, w);
    if (!scratch || scratch_bytes < need)
        return set_error(TCR_ERR_INVALID, "tcr_scatter: scratch of %lld bytes, %lld needed", (long long)scratch_bytes,
                         (long long)need);
    carve_work(p, static_cast<char*>(scratch), w);
    stats_init_kernel<<<1, 1, 0, st>>>(w.stats);
    note_launches(1);
    TCR_SCATTER_CUDA(cudaMemsetAsync(w.ngaps, 0, sizeof(unsigned long long), st));
    if (p.path == 0) {
        const unsigned mgrid = grid_resident(mark_runs_kernel<int64_t, true>, (p.M + kMarkKeys - 1) / kMarkKeys);
        mark_runs_kernel<int64_t, true><<<mgrid, kThreads, 0, st>>>(d->index, nullptr, nullptr, p.M, p.nslots, w.off,
                                                                    w.gaps, w.ngaps, p.gap_cap, w.stats);
        note_launches(1);
        TCR_SCATTER_CUDA(cudaGetLastError());
    } else if (p.wide) {
        TCR_SCATTER_CUDA(sort_path<unsigned long long>(d, p, w, st));
    } else {
        TCR_SCATTER_CUDA(sort_path<uint32_t>(d, p, w, st));
    }
    fill_gaps_kernel<<<grid_for((p.nslots + 1) / 4), kThreads, 0, st>>>(w.gaps, w.ngaps, p.gap_cap, w.off, w.stats,
                                                                         p.path == 0 ? 1 : 0);
    note_launches(1);
    TCR_SCATTER_CUDA(cudaGetLastError());

    FoldArgs fa;
    fa.src = d->src;
    fa.out = d->out;
    fa.arg = d->arg_out;
    fa.off = w.off;
    fa.perm0 = w.vals[0];
    fa.perm1 = w.vals[1];
    fa.sel = nullptr;
    if (p.path != 0)
        fa.sel = p.wide ? &static_cast<SortState64*>(w.state)->sel[key_passes<unsigned long long>()]
                        : &static_cast<SortState32*>(w.state)->sel[key_passes<uint32_t>()];
    fa.stats = w.stats;
    fa.B = d->B;
    fa.E = d->E;
    fa.K = d->K;
    fa.N = d->N;
    fa.accumulate = d->accumulate;
    cudaError_t e;
    if (p.path == 0 && d->K == 1) {
        const int64_t rows = d->B * ((d->N + kThreads - 1) / kThreads);
        e = launch_fold<3>(d->dtype, d->reduce, fa, grid_for(rows * kThreads), st);
    } else {
        const unsigned grid = grid_for(nout);
        e = p.path == 0   ? launch_fold<0>(d->dtype, d->reduce, fa, grid, st)
            : p.path == 1 ? launch_fold<1>(d->dtype, d->reduce, fa, grid, st)
                          : launch_fold<2>(d->dtype, d->reduce, fa, grid, st);
    }
    note_launches(1);
    TCR_SCATTER_CUDA(e);
    if (stats_host)
        TCR_SCATTER_CUDA(cudaMemcpyAsync(stats_host, w.stats, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    return TCR_OK;
}

}  // extern "C"
