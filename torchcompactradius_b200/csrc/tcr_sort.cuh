// tcr_sort.cuh -- stable LSD radix sort of (key, int32 value) pairs, 32- or 64-bit keys.
//
// Per 8-bit digit: a tile histogram kernel, a per-digit scan of the tiles' counts and a stable
// scatter.  Inside a tile the scatter ranks keys with warp match/ballot so equal digits
// keep their input order; tiles are concatenated in order, so the whole sort is stable.  A pass
// whose digit is the same for every key is skipped on the device without a host round trip:
// digits above the highest bit in which two keys differ (from the key range the producer
// reduced) are not even counted, and a digit whose histogram met a single value is neither
// scanned nor scattered.  The per-pass buffer selector then stays put.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "tcr_scan.cuh"

namespace tcr {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile (1024 measured slower)
constexpr int kBins = 256;
static_assert(kSortThreads == kBins, "the scatter scans one digit per thread");

template <typename K>
struct SortStateT {
    K key_min, key_max;   // reduced by the producer of the keys
    int32_t sel[9];       // sel[p]: which buffer (0/1) holds the input of pass p
    int32_t pad;
    int64_t n_dev;        // >= 0: sort only the first n_dev keys (a count known on the device only)
    uint32_t seen[8][8];  // per pass: bitmap of the digit values the histogram met
    int32_t consumed;     // the last pass handed the sorted pairs to the caller's consumer
};
using SortState32 = SortStateT<uint32_t>;
using SortState64 = SortStateT<unsigned long long>;

template <typename K>
__host__ __device__ constexpr int key_passes() { return (int)sizeof(K); }

__device__ __forceinline__ int top_bit(uint32_t x) { return 31 - __clz(x); }
__device__ __forceinline__ int top_bit(unsigned long long x) { return 63 - __clzll(x); }

// Producer-side reset (one thread): empty key range, input in buffer 0, no digits seen.
template <typename K>
__device__ __forceinline__ void sort_state_reset(SortStateT<K>* st) {
    st->key_min = ~(K)0;
    st->key_max = 0;
    st->sel[0] = 0;
    st->n_dev = -1;
    st->consumed = 0;
    for (int p = 0; p < 8; ++p)
        for (int i = 0; i < 8; ++i) st->seen[p][i] = 0u;
}

// Some key differs from another at or above bit `shift`.
template <typename K>
__device__ __forceinline__ bool pass_needed(const SortStateT<K>* st, int shift) {
    const K x = st->key_min ^ st->key_max;
    if (x == 0) return false;
    return top_bit(x) >= shift;
}

// The histogram of this pass met more than one digit value.
template <typename K>
__device__ __forceinline__ bool pass_varies(const SortStateT<K>* st, int pass) {
    int n = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) n += __popc(st->seen[pass][i]);
    return n > 1;
}

template <typename K>
__device__ __forceinline__ bool pass_runs(const SortStateT<K>* st, int shift, int pass) {
    return pass_needed(st, shift) && pass_varies(st, pass);
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const K* keys0, const K* keys1, int64_t n, int shift,
                                                                  int pass, int64_t ntiles, SortStateT<K>* st,
                                                                  int32_t* hist) {
    if (!pass_needed(st, shift)) return;
    if (st->n_dev >= 0 && st->n_dev < n) n = st->n_dev;
    const K* keys = st->sel[pass] ? keys1 : keys0;
    __shared__ int32_t sh[kBins];
    for (int i = threadIdx.x; i < kBins; i += kSortThreads) sh[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        int64_t i = base + (int64_t)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&sh[(int)((keys[i] >> shift) & 0xff)], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kBins; d += kSortThreads) hist[(int64_t)d * ntiles + blockIdx.x] = sh[d];
    if (threadIdx.x < kBins / 32) {  // the digit values this tile met
        uint32_t bits = 0;
        for (int b = 0; b < 32; ++b) bits |= (sh[threadIdx.x * 32 + b] != 0 ? 1u : 0u) << b;
        if (bits && (bits & ~st->seen[pass][threadIdx.x])) atomicOr(&st->seen[pass][threadIdx.x], bits);
    }
}

// A consumer of the sorted pairs that takes nothing: every pass writes keys and values.
struct NoSortConsumer {
    static constexpr bool kActive = false;
    template <typename K>
    __device__ void operator()(int64_t, K, int32_t) const {}
};

// Stable scatter of one tile.  Warp w owns keys [w*R*32, (w+1)*R*32) of the tile (R = kSortItems),
// processed in R rounds of 32 consecutive keys, so (warp, round, lane) order is the input order.  The tile is
// first ordered by digit in shared memory (stable), then written out by consecutive threads over
// that order: the keys of one digit land in consecutive output slots, so the stores coalesce into
// runs instead of one sector per key.
// With an active consumer, a pass above which no digit differs (the last one that can move keys)
// hands the consumer each (slot, key, value) instead of writing the value -- the keys are still
// written -- and sets st->consumed.
template <typename K, typename Consumer>
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(K* keys0, K* keys1, int32_t* vals0,
                                                                     int32_t* vals1, int64_t n, int shift, int pass,
                                                                     int64_t ntiles, SortStateT<K>* st,
                                                                     const int32_t* hist_scanned,
                                                                     const int32_t* digit_total, Consumer consume) {
    const int s = st->sel[pass];
    if (!pass_runs(st, shift, pass)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->sel[pass + 1] = s;
        return;
    }
    if (st->n_dev >= 0 && st->n_dev < n) n = st->n_dev;
    const K* kin = s ? keys1 : keys0;
    const int32_t* vin = s ? vals1 : vals0;
    K* kout = s ? keys0 : keys1;
    int32_t* vout = s ? vals0 : vals1;
    constexpr int NW = kSortThreads / 32;
    __shared__ int32_t warp_hist[NW][kBins];
    __shared__ int32_t tile_base[kBins];   // first output slot of each digit of this tile
    __shared__ int32_t digit_start[kBins + 1];  // first slot of each digit in the tile's digit order
    __shared__ K sk[kSortTile];
    __shared__ int32_t sv[kSortTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < NW * kBins; i += kSortThreads) (&warp_hist[0][0])[i] = 0;
    {
        // first slot of digit d in the output: the keys of smaller digits, then this digit's keys in
        // earlier tiles (one digit per thread)
        __shared__ int32_t base_sm[kSortThreads / 32 + 1];
        int32_t total;
        const int d = threadIdx.x;
        const int32_t db = block_exclusive_scan<int32_t, kSortThreads>(digit_total[d], base_sm, total);
        tile_base[d] = db + hist_scanned[(int64_t)d * ntiles + blockIdx.x];
    }
    __syncthreads();
    const int64_t tile0 = (int64_t)blockIdx.x * kSortTile;
    const int64_t base = tile0 + (int64_t)warp * (kSortItems * 32);
    const unsigned lt = (1u << lane) - 1u;
    K key[kSortItems];
    int32_t val[kSortItems];
    int32_t rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        int64_t i = base + r * 32 + lane;
        bool valid = i < n;
        key[r] = valid ? kin[i] : (K)0;
        val[r] = valid ? vin[i] : 0;
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        int64_t i = base + r * 32 + lane;
        bool valid = i < n;
        uint32_t dig = valid ? (uint32_t)((key[r] >> shift) & 0xff) : 0x100u;  // invalid lanes: own group
        unsigned peers = __match_any_sync(0xffffffffu, dig);
        int before = __popc(peers & lt);
        int run = valid ? warp_hist[warp][dig] : 0;
        __syncwarp();
        if (valid && before == 0) warp_hist[warp][dig] = run + __popc(peers);
        __syncwarp();
        rank[r] = run + before;
    }
    __syncthreads();
    // per digit: exclusive scan over warps; the digit's total, scanned over digits, is its start
    // in the tile's digit order
    int32_t dtot = 0;
    const int d0 = threadIdx.x;  // kSortThreads == kBins: one digit per thread
    {
        int acc = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            int c = warp_hist[w][d0];
            warp_hist[w][d0] = acc;
            acc += c;
        }
        dtot = acc;
    }
    {
        __shared__ int32_t scan_sm[kSortThreads / 32 + 1];
        int32_t total;
        const int32_t ex = block_exclusive_scan<int32_t, kSortThreads>(dtot, scan_sm, total);
        digit_start[d0] = ex;
        if (d0 == 0) digit_start[kBins] = total;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        int64_t i = base + r * 32 + lane;
        if (i < n) {
            int dig = (int)((key[r] >> shift) & 0xff);
            const int loc = digit_start[dig] + warp_hist[warp][dig] + rank[r];
            sk[loc] = key[r];
            sv[loc] = val[r];
        }
    }
    __syncthreads();
    const int tn = digit_start[kBins];
    const bool last = Consumer::kActive && !pass_needed(st, shift + 8);
    for (int i = threadIdx.x; i < tn; i += kSortThreads) {
        const K k = sk[i];
        const int dig = (int)((k >> shift) & 0xff);
        const int64_t pos = (int64_t)tile_base[dig] + (i - digit_start[dig]);
        kout[pos] = k;
        if (last)
            consume(pos, k, sv[i]);
        else
            vout[pos] = sv[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->sel[pass + 1] = s ^ 1;
        if (last) st->consumed = 1;
    }
}

// Per digit (one block each): exclusive scan of the digit's tile counts in place, and the
// digit's total; the scatter adds the totals of the smaller digits.  Gated on the pass running.
template <typename K>
__global__ void __launch_bounds__(kScanThreads) hist_scan_digits(int32_t* hist, int64_t ntiles, int32_t* digit_total,
                                                                 const SortStateT<K>* st, int shift, int pass) {
    if (!pass_runs(st, shift, pass)) return;
    __shared__ int32_t sm[kScanThreads / 32 + 1];
    int32_t* row = hist + (int64_t)blockIdx.x * ntiles;
    int32_t carry = 0;
    for (int64_t b = 0; b < ntiles; b += kScanTile) {
        const int64_t i0 = b + (int64_t)threadIdx.x * kScanItems;
        int32_t v[kScanItems];
        int32_t sum = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            v[k] = i0 + k < ntiles ? row[i0 + k] : 0;
            sum += v[k];
        }
        int32_t total;
        int32_t ex = block_exclusive_scan<int32_t, kScanThreads>(sum, sm, total) + carry;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (i0 + k < ntiles) row[i0 + k] = ex;
            ex += v[k];
        }
        carry += total;
    }
    if (threadIdx.x == 0) digit_total[blockIdx.x] = carry;
}

template <typename K>
struct SortWorkspaceT {
    K* keys[2];
    int32_t* vals[2];
    int32_t* hist;          // kBins * ntiles
    int32_t* tile_sums;     // kBins digit totals of the running pass
    SortStateT<K>* state;   // device
};

inline int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }
inline int64_t sort_hist_elems(int64_t n) { return (int64_t)kBins * sort_tiles(n); }

// Sorts keys[sel0]/vals[sel0] (sel0 = state->sel[0], set by the producer, which also reduced the
// key range and cleared the digit bitmaps), n keys or state->n_dev when that is set and smaller.  The result lives in buffer state->sel[key_passes<K>()]
// after the call; consumers read the selector on the device.  An active `consume` takes the pairs
// from the last pass that moves keys instead of the value buffer (st->consumed then reads 1).
template <typename K, typename Consumer = NoSortConsumer>
inline cudaError_t radix_sort_pairs(const SortWorkspaceT<K>& w, int64_t n, cudaStream_t st,
                                    Consumer consume = Consumer()) {
    if (n <= 0) return cudaSuccess;
    const int64_t nt = sort_tiles(n);
    for (int p = 0; p < key_passes<K>(); ++p) {
        const int shift = 8 * p;
        radix_hist_kernel<K><<<(unsigned)nt, kSortThreads, 0, st>>>(w.keys[0], w.keys[1], n, shift, p, nt, w.state,
                                                                    w.hist);
        hist_scan_digits<K><<<kBins, kScanThreads, 0, st>>>(w.hist, nt, w.tile_sums, w.state, shift, p);
        radix_scatter_kernel<K, Consumer><<<(unsigned)nt, kSortThreads, 0, st>>>(
            w.keys[0], w.keys[1], w.vals[0], w.vals[1], n, shift, p, nt, w.state, w.hist, w.tile_sums, consume);
        note_launches(3);
    }
    return cudaGetLastError();
}

}  // namespace tcr
