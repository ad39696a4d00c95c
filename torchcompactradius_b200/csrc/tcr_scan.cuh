// tcr_scan.cuh -- device-wide exclusive prefix sums built from a block scan.
//
// A per-tile reduction, then a per-tile scan that adds the tile's prefix.  Up to kScanDirectTiles
// tiles, each tile sums the totals of the tiles before it itself (at most 16 KB of reads, from L2);
// above that a single-CTA scan of the tile totals runs in between.  No block waits for another.
// Input and output are functors so that producers (flags, counts) and consumers (cell tables,
// offsets) fuse into the scan instead of round-tripping through HBM.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "tcr_common.cuh"

namespace tcr {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int64_t kScanDirectTiles = 2048;  // 4M elements

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
// the block total.  smem must hold NWARPS entries.
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

// Pass 1: tile totals.  In(i) returns the value of element i (0 for i >= n).
template <typename T, typename In>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(In in, int64_t n, T* tile_sums) {
    __shared__ T sm[kScanThreads / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += in(i);
    }
    T total;
    block_exclusive_scan<T, kScanThreads>(s, sm, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Pass 2: one CTA scans the tile totals in place (exclusive) and stores the grand total.
template <typename T>
__global__ void __launch_bounds__(1024) scan_tiles_kernel(T* tile_sums, int64_t ntiles, T* grand_total) {
    __shared__ T sm[1024 / 32 + 1];
    T carry = 0;
    for (int64_t b = 0; b < ntiles; b += 1024) {
        int64_t i = b + threadIdx.x;
        T v = i < ntiles ? tile_sums[i] : T(0);
        T total;
        T ex = block_exclusive_scan<T, 1024>(v, sm, total);
        if (i < ntiles) tile_sums[i] = ex + carry;
        carry += total;
    }
    if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}

// Pass 3: per-tile exclusive scan; Out(i, exclusive_prefix, value) consumes each element.  The
// tile's values are read and its results consumed in striped order (element base + k * threads +
// thread), so that the producer's loads and the consumer's stores coalesce; in between they pass
// through shared memory to the blocked order (kScanItems consecutive elements per thread) the
// scan works in.  A padded index keeps the blocked reads free of bank conflicts.
__device__ __forceinline__ int scan_pad(int i) { return i + (i >> 5); }

// DIRECT: tile_sums holds the tiles' own totals; the tile's prefix is their sum over the tiles
// before it, and the last tile stores the grand total.  Otherwise tile_sums holds the prefixes.
template <typename T, bool DIRECT, typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(In in, Out out, int64_t n, const T* tile_sums,
                                                                  T* grand_total) {
    __shared__ T sm[kScanThreads / 32 + 1];
    __shared__ T sval[kScanTile + kScanTile / 32];
    __shared__ T sex[kScanTile + kScanTile / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const int64_t i = base + j;
        sval[scan_pad(j)] = i < n ? in(i) : T(0);
    }
    T prefix;
    if (DIRECT) {
        T acc = 0;
        for (int64_t t = threadIdx.x; t < (int64_t)blockIdx.x; t += kScanThreads) acc += tile_sums[t];
        block_exclusive_scan<T, kScanThreads>(acc, sm, prefix);  // (its barriers also publish sval)
    } else {
        prefix = tile_sums[blockIdx.x];
        __syncthreads();
    }
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = sval[scan_pad(threadIdx.x * kScanItems + k)];
        s += v[k];
    }
    T total;
    T ex = block_exclusive_scan<T, kScanThreads>(s, sm, total) + prefix;
    if (DIRECT && grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *grand_total = prefix + total;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        sex[scan_pad(threadIdx.x * kScanItems + k)] = ex;
        ex += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const int64_t i = base + j;
        if (i < n) out(i, sex[scan_pad(j)], sval[scan_pad(j)]);
    }
}

inline int64_t scan_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

// Host launcher.  tile_sums must hold scan_tiles(n) elements; grand_total may be null.
template <typename T, typename In, typename Out>
cudaError_t device_exclusive_scan(In in, Out out, int64_t n, T* tile_sums, T* grand_total, cudaStream_t st) {
    int64_t nt = scan_tiles(n);
    if (nt == 0) {
        if (grand_total) return cudaMemsetAsync(grand_total, 0, sizeof(T), st);
        return cudaSuccess;
    }
    scan_reduce_kernel<T><<<(unsigned)nt, kScanThreads, 0, st>>>(in, n, tile_sums);
    if (nt <= kScanDirectTiles) {
        scan_apply_kernel<T, true><<<(unsigned)nt, kScanThreads, 0, st>>>(in, out, n, tile_sums, grand_total);
        note_launches(2);
        return cudaGetLastError();
    }
    scan_tiles_kernel<T><<<1, 1024, 0, st>>>(tile_sums, nt, grand_total);
    scan_apply_kernel<T, false><<<(unsigned)nt, kScanThreads, 0, st>>>(in, out, n, tile_sums, nullptr);
    note_launches(3);
    return cudaGetLastError();
}

}  // namespace tcr
