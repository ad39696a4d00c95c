// tcr_scan.cuh -- device-wide exclusive prefix sums in one pass (decoupled look-back).
//
// Each block takes the next tile from a ticket counter, scans it, publishes the tile's total and
// then its inclusive prefix in a status word, and finds its own exclusive prefix by reading the
// status words of the tiles before it (stopping at the first inclusive prefix).  A tile only ever
// waits for tiles with smaller tickets, which belong to blocks already running, so every wait
// ends; each wait is bounded all the same, and a wait that gives up sets a fault word instead of
// spinning on.  Input and output are functors so that producers (flags, counts) and consumers
// (cell tables, offsets) fuse into the scan instead of round-tripping through HBM.  The status
// words and the ticket of a scan must be zero when it starts.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "tcr_common.cuh"

namespace tcr {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Status word of a tile: 2 flag bits over a 62-bit non-negative value.
constexpr unsigned long long kStatusAggregate = 1ull << 62;  // the tile's own total
constexpr unsigned long long kStatusInclusive = 2ull << 62;  // the inclusive prefix up to the tile
constexpr unsigned long long kStatusValue = (1ull << 62) - 1;
// Iterations a look-back waits for one status word before it gives up and reports a fault.
constexpr int kLookbackSpins = 1 << 22;

__device__ __forceinline__ void store_release(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long load_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Waits (bounded) for a published status word; on giving up, records a fault and returns an
// inclusive zero so that the caller finishes.
__device__ __forceinline__ unsigned long long wait_status(const unsigned long long* p, int32_t* fault) {
    unsigned long long v = load_acquire(p);
    for (int spin = 0; (v >> 62) == 0; ++spin) {
        if (spin >= kLookbackSpins) {
            atomicOr(fault, 1);
            return kStatusInclusive;
        }
        __nanosleep(32);
        v = load_acquire(p);
    }
    return v;
}

// Where one scan keeps its look-back state: tile statuses, the tile ticket and the fault word.
struct LookbackSlot {
    unsigned long long* status;  // [scan_tiles(n)]
    int32_t* ticket;             // [1]
    int32_t* fault;              // [1] set when a wait gave up
};

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (unsigned)o) v += n;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive prefix and writes
// the block total.  smem must hold NWARPS + 1 entries.
template <typename T, int NTHREADS>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T& total) {
    constexpr int NW = NTHREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T s = lane < NW ? smem[lane] : T(0);
        T si = warp_inclusive_scan(s);
        if (lane < NW) smem[lane] = si - s;
        if (lane == NW - 1) smem[NW] = si;
    }
    __syncthreads();
    T excl = inc - v + smem[warp];
    total = smem[NW];
    __syncthreads();
    return excl;
}

// Exclusive prefix of tile `tile` (whose own total is `total`) over the tiles before it, computed
// by one whole warp: publishes the aggregate, looks back 32 tiles at a time, publishes the
// inclusive prefix.  Every lane returns the prefix.
__device__ __forceinline__ unsigned long long lookback_prefix(unsigned long long* status, int64_t tile,
                                                              unsigned long long total, int32_t* fault) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) store_release(&status[0], kStatusInclusive | total);
        return 0;
    }
    if (lane == 0) store_release(&status[tile], kStatusAggregate | total);
    unsigned long long excl = 0;
    int64_t p = tile - 1;
    for (;;) {
        const int64_t i = p - lane;
        const unsigned long long v = i >= 0 ? wait_status(&status[i], fault) : kStatusInclusive;
        const uint32_t incl = __ballot_sync(0xffffffffu, (v >> 62) == 2);
        const int stop = incl ? __ffs(incl) - 1 : 31;  // lanes 0..stop contribute
        unsigned long long mine = lane <= stop ? (v & kStatusValue) : 0ull;
#pragma unroll
        for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        excl += mine;
        if (incl) break;
        p -= 32;
    }
    if (lane == 0) store_release(&status[tile], kStatusInclusive | (excl + total));
    return excl;
}

// One-pass exclusive scan.  In(i) returns the value of element i (non-negative; 0 for i >= n);
// Out(i, exclusive_prefix, value) consumes each element in blocked order (thread t owns
// kScanItems consecutive elements of its tile); the tile holding the last element writes the
// grand total and calls out.finish(total) (a no-op for most consumers).
template <typename T, typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_lookback_kernel(In in, Out out, int64_t n, LookbackSlot slot,
                                                                     T* grand_total) {
    __shared__ int64_t s_tile;
    __shared__ T sm[kScanThreads / 32 + 1];
    __shared__ T s_excl;
    if (threadIdx.x == 0) s_tile = atomicAdd(slot.ticket, 1);
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t base = tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        v[k] = i < n ? in(i) : T(0);
        s += v[k];
    }
    T total;
    T ex = block_exclusive_scan<T, kScanThreads>(s, sm, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_prefix(slot.status, tile, (unsigned long long)total, slot.fault);
        if (threadIdx.x == 0) s_excl = (T)e;
    }
    __syncthreads();
    ex += s_excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (i < n) out(i, ex, v[k]);
        ex += v[k];
    }
    if (threadIdx.x == 0 && (tile + 1) * kScanTile >= n) {  // the last tile
        const T g = s_excl + total;
        if (grand_total) *grand_total = g;
        out.finish(g);
    }
}

inline int64_t scan_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

// Host launcher: one kernel.  The slot's statuses (scan_tiles(n) of them) and ticket must be zero;
// grand_total may be null.
template <typename T, typename In, typename Out>
cudaError_t device_exclusive_scan(In in, Out out, int64_t n, LookbackSlot slot, T* grand_total, cudaStream_t st) {
    const int64_t nt = scan_tiles(n);
    if (nt == 0) {
        if (grand_total) return cudaMemsetAsync(grand_total, 0, sizeof(T), st);
        return cudaSuccess;
    }
    scan_lookback_kernel<T><<<(unsigned)nt, kScanThreads, 0, st>>>(in, out, n, slot, grand_total);
    note_launches(1);
    return cudaGetLastError();
}

// Zeroes `words` 64-bit words with a grid-stride loop (look-back statuses and tickets).
__device__ __forceinline__ void zero_words(unsigned long long* p, int64_t words) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) p[i] = 0ull;
}

}  // namespace tcr
