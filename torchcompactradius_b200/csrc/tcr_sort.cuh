// tcr_sort.cuh -- stable LSD radix sort of (uint32 key, int32 value) pairs.
//
// Per 8-bit digit: a tile histogram kernel, a device scan of the digit-major histogram and a
// stable scatter.  Inside a tile the scatter ranks keys with warp match/ballot so equal digits
// keep their input order; tiles are concatenated in order, so the whole sort is stable.  A
// digit that is the same for every key (known from the key range the producer reduced) is
// skipped on the device without a host round trip: the kernels of that pass return at once
// and the per-pass buffer selector stays put.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "tcr_scan.cuh"

namespace tcr {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
constexpr int kBins = 256;

struct SortState {
    uint32_t key_min, key_max;  // reduced by the producer of the keys
    int32_t sel[5];             // sel[p]: which buffer (0/1) holds the input of pass p
    int32_t pad;
};

// A pass is needed iff some key differs from another in bits [shift, shift+8): equivalently the
// keys' common prefix ends inside or below this digit.
__device__ __forceinline__ bool pass_needed(const SortState* st, int shift) {
    uint32_t x = st->key_min ^ st->key_max;
    if (x == 0) return false;
    int top = 31 - __clz(x);  // highest differing bit
    return top >= shift;
}

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint32_t* keys0, const uint32_t* keys1,
                                                                  int64_t n, int shift, int pass, int64_t ntiles,
                                                                  SortState* st, int32_t* hist) {
    if (!pass_needed(st, shift)) return;
    const uint32_t* keys = st->sel[pass] ? keys1 : keys0;
    __shared__ int32_t sh[kBins];
    for (int i = threadIdx.x; i < kBins; i += kSortThreads) sh[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        int64_t i = base + (int64_t)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&sh[(keys[i] >> shift) & 0xff], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kBins; d += kSortThreads) hist[(int64_t)d * ntiles + blockIdx.x] = sh[d];
}

// Stable scatter of one tile.  Warp w owns keys [w*256, w*256+256) of the tile, processed in 8
// rounds of 32 consecutive keys, so (warp, round, lane) order is the input order.
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(uint32_t* keys0, uint32_t* keys1, int32_t* vals0,
                                                                     int32_t* vals1, int64_t n, int shift, int pass,
                                                                     int64_t ntiles, SortState* st,
                                                                     const int32_t* hist_scanned) {
    const bool need = pass_needed(st, shift);
    const int s = st->sel[pass];
    if (!need) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->sel[pass + 1] = s;
        return;
    }
    const uint32_t* kin = s ? keys1 : keys0;
    const int32_t* vin = s ? vals1 : vals0;
    uint32_t* kout = s ? keys0 : keys1;
    int32_t* vout = s ? vals0 : vals1;
    constexpr int NW = kSortThreads / 32;
    __shared__ int32_t warp_hist[NW][kBins];
    __shared__ int32_t tile_base[kBins];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < NW * kBins; i += kSortThreads) (&warp_hist[0][0])[i] = 0;
    for (int d = threadIdx.x; d < kBins; d += kSortThreads) tile_base[d] = hist_scanned[(int64_t)d * ntiles + blockIdx.x];
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * (kSortItems * 32);
    const unsigned lt = (1u << lane) - 1u;
    uint32_t key[kSortItems];
    int32_t val[kSortItems];
    int32_t rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        int64_t i = base + r * 32 + lane;
        bool valid = i < n;
        key[r] = valid ? kin[i] : 0xffffffffu;
        val[r] = valid ? vin[i] : 0;
        uint32_t dig = valid ? ((key[r] >> shift) & 0xff) : 0x100u;  // invalid lanes form their own group
        unsigned peers = __match_any_sync(0xffffffffu, dig);
        int before = __popc(peers & lt);
        int run = valid ? warp_hist[warp][dig] : 0;
        __syncwarp();
        if (valid && before == 0) warp_hist[warp][dig] = run + __popc(peers);
        __syncwarp();
        rank[r] = run + before;
    }
    __syncthreads();
    // exclusive scan over warps for each digit
    for (int d = threadIdx.x; d < kBins; d += kSortThreads) {
        int acc = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            int c = warp_hist[w][d];
            warp_hist[w][d] = acc;
            acc += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        int64_t i = base + r * 32 + lane;
        if (i < n) {
            int dig = (key[r] >> shift) & 0xff;
            int64_t pos = (int64_t)tile_base[dig] + warp_hist[warp][dig] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->sel[pass + 1] = s ^ 1;
}

// Scan kernels for the histogram, gated on the pass being needed.
__global__ void __launch_bounds__(kScanThreads) hist_scan_reduce(const int32_t* h, int64_t n, int32_t* tile_sums,
                                                                 const SortState* st, int shift) {
    if (!pass_needed(st, shift)) return;
    __shared__ int32_t sm[kScanThreads / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += h[i];
    }
    int32_t total;
    block_exclusive_scan<int32_t, kScanThreads>(s, sm, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}
__global__ void __launch_bounds__(1024) hist_scan_tiles(int32_t* tile_sums, int64_t ntiles, const SortState* st,
                                                        int shift) {
    if (!pass_needed(st, shift)) return;
    __shared__ int32_t sm[1024 / 32 + 1];
    int32_t carry = 0;
    for (int64_t b = 0; b < ntiles; b += 1024) {
        int64_t i = b + threadIdx.x;
        int32_t v = i < ntiles ? tile_sums[i] : 0;
        int32_t total;
        int32_t ex = block_exclusive_scan<int32_t, 1024>(v, sm, total);
        if (i < ntiles) tile_sums[i] = ex + carry;
        carry += total;
    }
}
__global__ void __launch_bounds__(kScanThreads) hist_scan_apply(int32_t* h, int64_t n, const int32_t* tile_sums,
                                                                const SortState* st, int shift) {
    if (!pass_needed(st, shift)) return;
    __shared__ int32_t sm[kScanThreads / 32 + 1];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        v[k] = i < n ? h[i] : 0;
        s += v[k];
    }
    int32_t total;
    int32_t ex = block_exclusive_scan<int32_t, kScanThreads>(s, sm, total) + tile_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        if (i < n) h[i] = ex;
        ex += v[k];
    }
}

struct SortWorkspace {
    uint32_t* keys[2];
    int32_t* vals[2];
    int32_t* hist;       // kBins * ntiles
    int32_t* tile_sums;  // scan_tiles(kBins * ntiles)
    SortState* state;    // device
};

inline int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }
inline int64_t sort_hist_elems(int64_t n) { return (int64_t)kBins * sort_tiles(n); }

// Sorts keys[sel0]/vals[sel0] (sel0 = state->sel[0], set by the producer).  The result lives in
// buffer state->sel[4] after the call; consumers read the selector on the device.
inline cudaError_t radix_sort_pairs(const SortWorkspace& w, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t nt = sort_tiles(n);
    const int64_t nh = (int64_t)kBins * nt;
    const int64_t nht = scan_tiles(nh);
    for (int p = 0; p < 4; ++p) {
        int shift = 8 * p;
        radix_hist_kernel<<<(unsigned)nt, kSortThreads, 0, st>>>(w.keys[0], w.keys[1], n, shift, p, nt, w.state, w.hist);
        hist_scan_reduce<<<(unsigned)nht, kScanThreads, 0, st>>>(w.hist, nh, w.tile_sums, w.state, shift);
        hist_scan_tiles<<<1, 1024, 0, st>>>(w.tile_sums, nht, w.state, shift);
        hist_scan_apply<<<(unsigned)nht, kScanThreads, 0, st>>>(w.hist, nh, w.tile_sums, w.state, shift);
        radix_scatter_kernel<<<(unsigned)nt, kSortThreads, 0, st>>>(w.keys[0], w.keys[1], w.vals[0], w.vals[1], n, shift,
                                                                   p, nt, w.state, w.hist);
        note_launches(5);
    }
    return cudaGetLastError();
}

}  // namespace tcr
