// tcr_sort.cuh -- stable LSD radix sort of (key, int32 value) pairs, 32- or 64-bit keys.
//
// One histogram kernel counts the 8-bit digits of every pass in a single read of the keys; then
// one kernel per digit pass ranks and scatters a tile of keys: inside the tile keys are ranked
// with warp match/ballot so equal digits keep their input order, and the tile's global position
// for each digit is the digit's global offset plus a decoupled look-back over the tiles before it
// (tiles are taken in ticket order, so a tile only waits for blocks already running; each wait is
// bounded and reports a fault instead of spinning on).  Tiles are concatenated in order, so the
// whole sort is stable.  A pass whose digit is the same for every key (its histogram met one
// value, or the key range's top differing bit lies below it) is skipped on the device without a
// host round trip; the per-pass buffer selector then stays put.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "tcr_scan.cuh"

namespace tcr {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
constexpr int kBins = 256;
static_assert(kSortThreads == kBins, "one thread per digit value");

template <typename K>
struct SortStateT {
    K key_min, key_max;       // reduced by the producer of the keys
    int32_t sel[9];           // sel[p]: which buffer (0/1) holds the input of pass p
    int32_t pad;
    int64_t n_dev;            // >= 0: sort only the first n_dev keys (a count known on the device only)
    int32_t ticket[8];        // per pass: tile tickets
    uint32_t hist[8][kBins];  // per pass: global count of every digit value
};
using SortState32 = SortStateT<uint32_t>;
using SortState64 = SortStateT<unsigned long long>;

template <typename K>
__host__ __device__ constexpr int key_passes() { return (int)sizeof(K); }

__device__ __forceinline__ int top_bit(uint32_t x) { return 31 - __clz(x); }
__device__ __forceinline__ int top_bit(unsigned long long x) { return 63 - __clzll(x); }

// Producer-side reset, by every thread of one block: empty key range, input in buffer 0, no
// digits counted, tickets at zero.
template <typename K>
__device__ __forceinline__ void sort_state_reset(SortStateT<K>* st) {
    if (threadIdx.x == 0) {
        st->key_min = ~(K)0;
        st->key_max = 0;
        st->sel[0] = 0;
        st->n_dev = -1;
    }
    if (threadIdx.x < 8) st->ticket[threadIdx.x] = 0;
    for (int i = threadIdx.x; i < 8 * kBins; i += blockDim.x) (&st->hist[0][0])[i] = 0u;
}

// Some key differs from another at or above bit `shift`.
template <typename K>
__device__ __forceinline__ bool pass_needed(const SortStateT<K>* st, int shift) {
    const K x = st->key_min ^ st->key_max;
    if (x == 0) return false;
    return top_bit(x) >= shift;
}

// Every pass's digit histogram in one read of the keys (shared-memory counts, then one atomic per
// block and non-zero bin); passes above the key range's top differing bit are not counted.  Also
// zeroes the passes' look-back statuses.
template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const K* keys0, const K* keys1, int64_t n,
                                                                  SortStateT<K>* st, unsigned long long* status,
                                                                  int64_t status_words) {
    zero_words(status, status_words);
    if (!pass_needed(st, 0)) return;
    if (st->n_dev >= 0 && st->n_dev < n) n = st->n_dev;
    const K* keys = st->sel[0] ? keys1 : keys0;
    constexpr int P = key_passes<K>();
    __shared__ uint32_t sh[P][kBins];
    for (int i = threadIdx.x; i < P * kBins; i += kSortThreads) (&sh[0][0])[i] = 0u;
    __syncthreads();
    const int top = top_bit(st->key_min ^ st->key_max) >> 3;
    const int64_t stride = (int64_t)gridDim.x * kSortThreads;
    for (int64_t i = (int64_t)blockIdx.x * kSortThreads + threadIdx.x; i < n; i += stride) {
        const K k = keys[i];
#pragma unroll
        for (int p = 0; p < P; ++p)
            if (p <= top) atomicAdd(&sh[p][(int)((k >> (8 * p)) & 0xff)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P * kBins; i += kSortThreads) {
        const uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&(&st->hist[0][0])[i], c);
    }
}

// One digit pass over the tiles.  Warp w of a tile owns keys [w*256, w*256+256) of it, in 8
// rounds of 32 consecutive keys, so (warp, round, lane) order is the input order.  status: this
// pass's look-back words [tiles][kBins] (zero on entry); status_next: the next pass's, zeroed here.
template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_onesweep_kernel(K* keys0, K* keys1, int32_t* vals0,
                                                                      int32_t* vals1, int64_t n, int pass,
                                                                      SortStateT<K>* st,
                                                                      unsigned long long* status,
                                                                      unsigned long long* status_next,
                                                                      int32_t* fault) {
    const int t = threadIdx.x;
    const int shift = 8 * pass;
    if (pass + 1 < key_passes<K>()) status_next[(int64_t)blockIdx.x * kBins + t] = 0ull;
    const uint32_t gcount = st->hist[pass][t];
    const int distinct = __syncthreads_count(gcount != 0);
    const int s = st->sel[pass];
    if (distinct <= 1 || !pass_needed(st, shift)) {  // every key has the same digit: nothing moves
        if (blockIdx.x == 0 && t == 0) st->sel[pass + 1] = s;
        return;
    }
    if (st->n_dev >= 0 && st->n_dev < n) n = st->n_dev;
    const K* kin = s ? keys1 : keys0;
    const int32_t* vin = s ? vals1 : vals0;
    K* kout = s ? keys0 : keys1;
    int32_t* vout = s ? vals0 : vals1;
    constexpr int NW = kSortThreads / 32;
    __shared__ int32_t warp_hist[NW][kBins];
    __shared__ int64_t tile_base[kBins];
    __shared__ int64_t s_tile;
    __shared__ uint32_t s_scan[NW + 1];
    const int lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = atomicAdd(&st->ticket[pass], 1);
    for (int i = t; i < NW * kBins; i += kSortThreads) (&warp_hist[0][0])[i] = 0;
    // global offset of digit t: exclusive scan of the pass histogram (its barriers publish the above)
    uint32_t gtotal;
    const uint32_t gexcl = block_exclusive_scan<uint32_t, kSortThreads>(gcount, s_scan, gtotal);
    const int64_t tile = s_tile;
    const int64_t base = tile * kSortTile + (int64_t)warp * (kSortItems * 32);
    const unsigned lt = (1u << lane) - 1u;
    K key[kSortItems];
    int32_t val[kSortItems];
    int32_t rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t i = base + r * 32 + lane;
        const bool valid = i < n;
        key[r] = valid ? kin[i] : (K)0;
        val[r] = valid ? vin[i] : 0;
        const uint32_t dig = valid ? (uint32_t)((key[r] >> shift) & 0xff) : 0x100u;  // invalid lanes: own group
        const unsigned peers = __match_any_sync(0xffffffffu, dig);
        const int before = __popc(peers & lt);
        const int run = valid ? warp_hist[warp][dig] : 0;
        __syncwarp();
        if (valid && before == 0) warp_hist[warp][dig] = run + __popc(peers);
        __syncwarp();
        rank[r] = run + before;
    }
    __syncthreads();
    // digit t: exclusive prefix over the tile's warps, the tile's count, its place among the tiles
    int32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const int32_t c = warp_hist[w][t];
        warp_hist[w][t] = cnt;
        cnt += c;
    }
    unsigned long long* st_d = status + t;  // digit t's words, kBins apart from tile to tile
    unsigned long long excl = 0;
    if (tile == 0) {
        store_release(&st_d[0], kStatusInclusive | (unsigned long long)cnt);
    } else {
        store_release(&st_d[tile * kBins], kStatusAggregate | (unsigned long long)cnt);
        for (int64_t p = tile - 1; p >= 0; --p) {
            const unsigned long long v = wait_status(&st_d[p * kBins], fault);
            excl += v & kStatusValue;
            if ((v >> 62) == 2) break;
        }
        store_release(&st_d[tile * kBins], kStatusInclusive | (excl + (unsigned long long)cnt));
    }
    tile_base[t] = (int64_t)gexcl + (int64_t)excl;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t i = base + r * 32 + lane;
        if (i < n) {
            const int dig = (int)((key[r] >> shift) & 0xff);
            const int64_t pos = tile_base[dig] + warp_hist[warp][dig] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
    if (blockIdx.x == 0 && t == 0) st->sel[pass + 1] = s ^ 1;
}

template <typename K>
struct SortWorkspaceT {
    K* keys[2];
    int32_t* vals[2];
    unsigned long long* status;  // sort_status_words(n) look-back words (the sort zeroes them itself)
    SortStateT<K>* state;        // device; reset by the producer of the keys (sort_state_reset)
    int32_t* fault;              // device word set when a look-back wait gave up (the result is not valid)
};

inline int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }
// Two buffers of per-(tile, digit) status words: pass p uses buffer p & 1 and clears the other.
inline int64_t sort_status_words(int64_t n) { return 2 * (int64_t)kBins * std::max<int64_t>(sort_tiles(n), 1); }

// Sorts keys[sel0]/vals[sel0] (sel0 = state->sel[0], set by the producer, which also reduced the
// key range and reset the state), n keys or state->n_dev when that is set and smaller.  The result
// lives in buffer state->sel[key_passes<K>()] after the call; consumers read the selector on the
// device.  *w.fault is set if a look-back wait gave up.
template <typename K>
inline cudaError_t radix_sort_pairs(const SortWorkspaceT<K>& w, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t nt = sort_tiles(n);
    const int64_t half = (int64_t)kBins * nt;
    const unsigned hblocks = (unsigned)std::min<int64_t>(nt, 148 * 4);
    radix_hist_kernel<K><<<hblocks, kSortThreads, 0, st>>>(w.keys[0], w.keys[1], n, w.state, w.status, 2 * half);
    for (int p = 0; p < key_passes<K>(); ++p)
        radix_onesweep_kernel<K><<<(unsigned)nt, kSortThreads, 0, st>>>(
            w.keys[0], w.keys[1], w.vals[0], w.vals[1], n, p, w.state, w.status + (p & 1) * half,
            w.status + ((p + 1) & 1) * half, w.fault);
    note_launches(1 + key_passes<K>());
    return cudaGetLastError();
}

}  // namespace tcr
