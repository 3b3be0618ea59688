// Stable LSD radix sort of (key, value) pairs and single-pass prefix scans.
//
// Replaces RadixSort::sort (radix_sort/RadixSort.cpp:181-238), which runs
// three kernels per 5-bit digit (upsweep / spine scan / downsweep,
// radix_sort/RadixSortKernels.cu:204,249,812) with a host synchronisation
// after each launch. Here every 8-bit digit is one kernel:
//   * all digit histograms are counted in one read of the keys up front
//     (or by the kernel that produced the keys);
//   * each pass counts a tile's digits and publishes the counts first, finds
//     the tile's global digit offsets by decoupled look-back over earlier tiles
//     (tiles are taken in launch order from an atomic ticket, so a tile only
//     waits on tiles that are already running; every wait is bounded), ranks
//     keys within each warp with ballots, and writes keys and values out of a
//     shared-memory staging buffer so that runs of equal digits leave as
//     contiguous stores.
// The result equals a stable sort by key: ties keep their input order, so
// with values 0..n-1 ties are ordered by original index, as in the reference.
#include <algorithm>
#include <mutex>
#include <string>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {

constexpr uint32_t ST_FLAG_A = 1u << 30;   // tile aggregate available
constexpr uint32_t ST_FLAG_P = 2u << 30;   // inclusive prefix available
constexpr uint32_t ST_MASK = (1u << 30) - 1u;
constexpr uint32_t LOOKBACK_SPIN_LIMIT = HP_SORT_SPIN_LIMIT_DEFAULT;

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift, uint32_t mask) {
    return (uint32_t)(k >> shift) & mask;
}

// Digit histograms of every pass in one read of the keys.
template <typename K>
__global__ void k_sort_hist(const K* __restrict__ keys, int64_t n, int passes, int bits,
                            uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t sh[];
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        K k = keys[i];
        for (int p = 0; p < passes; ++p) {
            int shift = 8 * p;
            int w = min(8, bits - shift);
            atomicAdd(&sh[p * 256 + digit_of(k, shift, (1u << w) - 1u)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive scan of two values over the first 256 threads of the block
// (BLOCK >= 256). Returns exclusive prefixes; uses s_w[2][8].
__device__ __forceinline__ void scan256x2(uint32_t a, uint32_t b, uint32_t& ea, uint32_t& eb,
                                          uint32_t (*s_w)[8]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t ia = a, ib = b;
    if (tid < 256) {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t ya = __shfl_up_sync(HP_FULL_MASK, ia, o);
            uint32_t yb = __shfl_up_sync(HP_FULL_MASK, ib, o);
            if (lane >= o) { ia += ya; ib += yb; }
        }
        if (lane == 31) { s_w[0][warp] = ia; s_w[1][warp] = ib; }
    }
    __syncthreads();
    if (tid < 256) {
        uint32_t oa = 0, ob = 0;
        for (int w = 0; w < warp; ++w) { oa += s_w[0][w]; ob += s_w[1][w]; }
        ea = oa + ia - a;
        eb = ob + ib - b;
    }
}

// Digit-offset look-back for digit `tid` of this tile: the sum of the digit's
// counts over all earlier tiles, walking back over LB status words per round
// until a tile whose inclusive prefix is published. Every wait is bounded.
template <int LB>
__device__ __forceinline__ uint32_t lookback(const uint32_t* status, uint32_t tile, int tid, int* err,
                                             uint32_t spin_limit) {
    uint32_t prefix = 0, spins = 0;
    int64_t t = (int64_t)tile - 1;
    bool done = tile == 0;
    while (!done) {
        uint32_t sw[LB];
#pragma unroll
        for (int k = 0; k < LB; ++k)
            sw[k] = (t - k >= 0) ? ld_relaxed_u32(&status[(size_t)(t - k) * 256 + tid]) : 0u;
#pragma unroll
        for (int k = 0; k < LB; ++k) {
            if (done) break;
            if (t - k < 0) { done = true; break; }
            uint32_t s = sw[k];
            while ((s & ~ST_MASK) == 0u) {
                if (++spins > spin_limit) {
                    hp_report(err, HP_DEV_SPIN_LIMIT, (int)tile);
                    s = ST_FLAG_P;
                    break;
                }
                s = ld_relaxed_u32(&status[(size_t)(t - k) * 256 + tid]);
            }
            prefix += s & ST_MASK;
            if ((s & ~ST_MASK) == ST_FLAG_P || t - k == 0) done = true;
        }
        t -= LB;
    }
    return prefix;
}

// One LSD pass over a tile of TILE keys:
//   1. load the keys (and values) of the tile;
//   2. count the tile's digits with shared-memory atomics and publish the
//      counts at once, so that later tiles' look-backs see them early;
//   3. look back for the digit offsets of all earlier tiles (256 threads, one
//      per digit) while the other warps go on to rank;
//   4. rank within each warp in index order (round i, then lane): the lanes
//      of equal digit are found with 8 ballots, and per-warp counters carry
//      the counts from round to round;
//   5. stage the keys in shared memory in digit order and write them out, so
//      that runs of equal digits leave as contiguous stores.
template <typename K, int BLOCK, int ITEMS, int LB = 4>
__global__ void __launch_bounds__(BLOCK) k_onesweep(
    const K* __restrict__ keys_in, const int32_t* __restrict__ vals_in,
    K* __restrict__ keys_out, int32_t* __restrict__ vals_out, int64_t n, int shift,
    uint32_t dmask, const uint32_t* __restrict__ hist, uint32_t* status,
    uint32_t* tile_counter, int* err, uint32_t spin_limit) {
    constexpr int NW = BLOCK / 32;
    constexpr int TILE = BLOCK * ITEMS;
    static_assert(BLOCK >= 256, "one thread per digit");
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* cnt = reinterpret_cast<uint32_t*>(smem);          // [NW][256] while ranking
    K* skeys = reinterpret_cast<K*>(smem);                        // [TILE] while scattering
    int32_t* svals = reinterpret_cast<int32_t*>(smem + (size_t)TILE * sizeof(K));
    __shared__ uint32_t s_count[256];
    __shared__ uint32_t s_block_start[256];
    __shared__ uint32_t s_global[256];
    __shared__ uint32_t s_w[2][8];
    __shared__ uint32_t s_tile;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int i = tid; i < NW * 256; i += BLOCK) cnt[i] = 0;
    if (tid < 256) s_count[tid] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * TILE;
    const int64_t wbase = base + (int64_t)warp * 32 * ITEMS;
    const uint32_t lt_mask = (1u << lane) - 1u;

    K key[ITEMS];
    int32_t val[ITEMS];
    uint32_t rnk[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        int64_t idx = wbase + i * 32 + lane;
        bool valid = idx < n;
        key[i] = valid ? keys_in[idx] : K(0);
        val[i] = valid ? (vals_in ? vals_in[idx] : (int32_t)idx) : 0;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
        if (wbase + i * 32 + lane < n) atomicAdd(&s_count[digit_of(key[i], shift, dmask)], 1u);
    __syncthreads();

    uint32_t total = 0, hval = 0;
    if (tid < 256) {
        total = s_count[tid];
        st_relaxed_u32(&status[(size_t)tile * 256 + tid], (tile == 0 ? ST_FLAG_P : ST_FLAG_A) | total);
        hval = hist[tid];
    }
    uint32_t block_start = 0, hist_excl = 0;
    scan256x2(total, hval, block_start, hist_excl, s_w);
    if (tid < 256) {
        s_block_start[tid] = block_start;
        const uint32_t prefix = lookback<LB>(status, tile, tid, err, spin_limit);
        if (tile > 0) st_relaxed_u32(&status[(size_t)tile * 256 + tid], ST_FLAG_P | (prefix + total));
        s_global[tid] = hist_excl + prefix - block_start;
    }

    // Rank within the warp: items are visited in index order (round i, then lane).
    uint32_t* wcnt = cnt + warp * 256;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int64_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? digit_of(key[i], shift, dmask) : 0u;
        uint32_t peers = __ballot_sync(HP_FULL_MASK, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t bal = __ballot_sync(HP_FULL_MASK, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bal : ~bal;
        }
        const uint32_t below = __popc(peers & lt_mask);
        const uint32_t c = valid ? wcnt[d] : 0u;
        __syncwarp();
        if (valid && below == 0) wcnt[d] = c + __popc(peers);
        __syncwarp();
        rnk[i] = c + below;
    }
    __syncthreads();
    // Per digit: exclusive offsets of the warps within the tile.
    if (tid < 256) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const uint32_t c = cnt[w * 256 + tid];
            cnt[w * 256 + tid] = run;
            run += c;
        }
    }
    __syncthreads();
    uint32_t pos[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t d = digit_of(key[i], shift, dmask);
        pos[i] = s_block_start[d] + cnt[warp * 256 + d] + rnk[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        int64_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            skeys[pos[i]] = key[i];
            svals[pos[i]] = val[i];
        }
    }
    __syncthreads();
    // Output positions are in range whenever every look-back completed. After
    // a wait gave up (reported above), this pass's prefixes are too small and
    // the next pass reads keys whose digit counts no longer match the
    // histograms, so positions are checked before every store.
    const int count = (int)min((int64_t)TILE, n - base);
    for (int j = tid; j < count; j += BLOCK) {
        K k = skeys[j];
        uint32_t g = s_global[digit_of(k, shift, dmask)] + (uint32_t)j;
        if ((int64_t)g < n) {
            keys_out[g] = k;
            vals_out[g] = svals[j];
        } else {
            hp_report(err, HP_DEV_BAD_INDEX, (int)tile);
        }
    }
}

// Keys per thread of a pass; the CTA size (512 by default, 256 as a tuning
// choice) is chosen at run time.
template <typename K> struct sort_cfg;
template <> struct sort_cfg<uint32_t> { static constexpr int BLOCK = 512, ITEMS = 12; };
template <> struct sort_cfg<uint64_t> { static constexpr int BLOCK = 512, ITEMS = 10; };

template <typename K, int BLOCK>
constexpr size_t onesweep_smem() {
    constexpr int TILE = BLOCK * sort_cfg<K>::ITEMS;
    constexpr size_t a = (size_t)(BLOCK / 32) * 256 * 4;
    constexpr size_t b = (size_t)TILE * (sizeof(K) + 4);
    return a > b ? a : b;
}

// ---- wide keys: top 24 bits by three LSD passes, then a sort of every segment ----
// For keys of more than 48 bits, the full LSD sort is ceil(bits/8) passes over
// global memory (8 for 60-bit Morton codes). Instead: three of those passes
// order the keys stably by their top 24 sorted bits; the array is then a
// sequence of segments of equal 24-bit prefix, each in input order, and most
// segments are short (a 24-bit prefix of a Morton code is a cell of 1/256 of
// the scene per axis). k_seg_sort gives every CTA the segments that start in
// its window of SEG_WINDOW positions: one-key segments are copied, segments of
// up to 32 keys are sorted by one warp each (a bitonic network over
// (low bits, position), so equal keys keep their order), longer ones by the
// whole CTA with stable 8-bit passes in shared memory. Every key is read and
// written once more instead of five more times; the result equals the stable
// sort by key. Segments larger than SEG_CAP (very uneven key distributions)
// are listed and sorted by k_seg_big, one CTA per segment, with stable passes
// through global memory.
constexpr int SEG_BLOCK = 256, SEG_ITEMS = 8, SEG_CAP = SEG_BLOCK * SEG_ITEMS, SEG_WINDOW = 1536;
constexpr int SEG_NW = SEG_BLOCK / 32;
constexpr int SEG_RANK_MAX = 512;  // segments ranked element by element
constexpr int SEG_MED_CAP = SEG_CAP / (SEG_RANK_MAX + 1) + 1;  // longer segments in one chunk
constexpr int64_t HYBRID_MIN_N = int64_t(1) << 20;

__host__ __device__ constexpr bool hybrid_sort(int64_t n, int key_bytes, int bits) {
    return key_bytes == 8 && bits > 48 && n >= HYBRID_MIN_N;
}

constexpr int SEG_TOP = 3;  // 8-bit digits ordered by global passes
constexpr int SEG_WALK = 6;  // steps of the linear search for a segment's bounds

// Histograms of the SEG_TOP 8-bit digits at shifts s0, s0 + 8, ...
__global__ void k_hist_top(const uint64_t* __restrict__ keys, int64_t n, int s0, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[256 * SEG_TOP];
    for (int i = threadIdx.x; i < 256 * SEG_TOP; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
#pragma unroll
        for (int d = 0; d < SEG_TOP; ++d) atomicAdd(&sh[256 * d + ((uint32_t)(k >> (s0 + 8 * d)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256 * SEG_TOP; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// The prefix of a key: its bits [L, L + 8 * SEG_TOP) (bits above the sorted
// width are not part of the order).
__device__ __forceinline__ uint32_t seg_prefix(uint64_t k, int L) {
    return (uint32_t)(k >> L) & ((1u << (8 * SEG_TOP)) - 1u);
}

// First position after the segment (run of equal prefix) holding `pos`; keys
// are sorted by prefix.
__device__ __forceinline__ int64_t seg_end(const uint64_t* __restrict__ keys, int64_t n, int64_t pos, int L) {
    const uint32_t pre = seg_prefix(keys[pos], L);
    int64_t lo = pos + 1, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (seg_prefix(keys[mid], L) > pre) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Stable rank of a block's SEG_CAP-element tile by the 8-bit digit at `shift`:
// element e = warp * 32 * ITEMS + i * 32 + lane is key[i] of that lane. On
// return pos[i] is its position in the tile sorted by digit (ties in element
// order) and tot[d] the tile's count of digit d. cnt [SEG_NW][256] and
// dstart [256] are shared scratch. Ends with a barrier.
__device__ __forceinline__ void seg_block_rank(const uint64_t (&key)[SEG_ITEMS], int m, int shift,
                                               uint16_t* cnt, uint32_t* dstart, uint32_t* tot,
                                               uint32_t (&pos)[SEG_ITEMS]) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (int i = tid; i < SEG_NW * 256; i += SEG_BLOCK) cnt[i] = 0;
    __syncthreads();
    uint16_t* wc = cnt + warp * 256;
    uint32_t dg[SEG_ITEMS], rk[SEG_ITEMS];
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i) {
        const int e = warp * 32 * SEG_ITEMS + i * 32 + lane;
        const bool valid = e < m;
        const uint32_t d = valid ? ((uint32_t)(key[i] >> shift) & 255u) : 0u;
        uint32_t peers = __ballot_sync(HP_FULL_MASK, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t bal = __ballot_sync(HP_FULL_MASK, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bal : ~bal;
        }
        const uint32_t below = __popc(peers & lt);
        const uint32_t c = valid ? wc[d] : 0u;
        __syncwarp();
        if (valid && below == 0) wc[d] = (uint16_t)(c + __popc(peers));
        __syncwarp();
        dg[i] = d;
        rk[i] = c + below;
    }
    __syncthreads();
    if (tid < 256) {  // per digit: exclusive offsets of the warps, and the digit's total
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < SEG_NW; ++w) {
            const uint32_t c = cnt[w * 256 + tid];
            cnt[w * 256 + tid] = (uint16_t)run;
            run += c;
        }
        tot[tid] = run;
        // exclusive scan of the totals over the 256 digits (8 warps)
        uint32_t x = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(HP_FULL_MASK, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) dstart[256 + warp] = x;  // warp totals in dstart[256..263]
        dstart[tid] = x - run;
    }
    __syncthreads();
    if (tid < 256) {
        uint32_t add = 0;
        for (int w = 0; w < warp; ++w) add += dstart[256 + w];
        dstart[tid] += add;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i) pos[i] = dstart[dg[i]] + cnt[warp * 256 + dg[i]] + rk[i];
    __syncthreads();
}

struct seg_smem {
    uint64_t key[2][SEG_CAP];
    int32_t val[2][SEG_CAP];
    uint16_t cnt[SEG_NW * 256];
    uint32_t dstart[256 + 8];
    uint32_t tot[256];
    uint32_t part[SEG_BLOCK];
    int2 med[SEG_MED_CAP];  // segments longer than SEG_RANK_MAX keys
    int64_t range[4];
    int nseg, nmed;
};

// Sorts the low L bits of one segment held in S.key[0][0, m) (positions in
// S.val[0]) with stable 8-bit passes in shared memory; returns the buffer
// holding the result.
__device__ int seg_block_sort(seg_smem& S, int m, int L) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int passes = (L + 7) / 8;
    int src = 0;
    for (int p = 0; p < passes; ++p) {
        uint64_t key[SEG_ITEMS];
        int32_t val[SEG_ITEMS];
#pragma unroll
        for (int i = 0; i < SEG_ITEMS; ++i) {
            const int e = warp * 32 * SEG_ITEMS + i * 32 + lane;
            key[i] = e < m ? S.key[src][e] : 0ull;
            val[i] = e < m ? S.val[src][e] : 0;
        }
        uint32_t pos[SEG_ITEMS];
        seg_block_rank(key, m, 8 * p, S.cnt, S.dstart, S.tot, pos);
#pragma unroll
        for (int i = 0; i < SEG_ITEMS; ++i) {
            const int e = warp * 32 * SEG_ITEMS + i * 32 + lane;
            if (e < m) {
                S.key[1 - src][pos[i]] = key[i];
                S.val[1 - src][pos[i]] = val[i];
            }
        }
        __syncthreads();
        src = 1 - src;
    }
    return src;
}

// Sorts in[cs, cs + m) (m <= SEG_CAP, whole segments of equal prefix) by the
// low L bits within each segment and writes the result to out[cs, cs + m).
// The chunk's keys and values are ck[0, m) and cv[0, m) in shared memory.
// Segments of up to SEG_RANK_MAX keys (almost all of them) need no
// coordination: every element finds its segment's bounds (the warp's ballots
// of segment starts and ends tell them for the segments inside its 32
// elements; a short walk, then a binary search, for the others), counts the
// smaller (low bits, position) pairs in its segment and stores itself at
// start + count. Longer segments are listed and sorted by the CTA with stable
// 8-bit passes, which reuse all of the shared buffers (ck and cv included:
// those segments are read again from in).
// Every index is checked against the chunk: inputs whose prefixes are not in
// order (only after an earlier pass gave up a bounded wait, which is reported)
// must not make it read or write outside the chunk.
__device__ void seg_sort_chunk(seg_smem& S, const uint64_t* ck, const int32_t* cv,
                               const uint64_t* __restrict__ kin, const int32_t* __restrict__ vin,
                               uint64_t* __restrict__ kout, int32_t* __restrict__ vout, int64_t cs, int m,
                               int L, int* err) {
    const int tid = threadIdx.x, lane = tid & 31;
    const uint64_t low = (uint64_t(1) << L) - 1u;
    if (tid == 0) S.nmed = 0;
    __syncthreads();
    // warp-contiguous groups of 32 elements; the loop bound is uniform over the
    // block, so every lane takes part in the ballots
    for (int c0 = tid - lane; c0 < m; c0 += SEG_BLOCK) {
        const int c = c0 + lane;
        const bool valid = c < m;
        const uint64_t kc = valid ? ck[c] : 0ull;
        const uint32_t pc = seg_prefix(kc, L);
        const bool head = valid && (c == 0 || seg_prefix(ck[c - 1], L) != pc);
        const bool tail = valid && (c + 1 == m || seg_prefix(ck[c + 1], L) != pc);
        const unsigned H = __ballot_sync(HP_FULL_MASK, head), T = __ballot_sync(HP_FULL_MASK, tail);
        if (!valid) continue;
        if (head && tail) {  // a one-key segment is in place
            kout[cs + c] = kc;
            vout[cs + c] = cv[c];
            continue;
        }
        // the segment's bounds (the chunk is sorted by prefix)
        const unsigned hb = H & (lane == 31 ? HP_FULL_MASK : ((2u << lane) - 1u));  // starts at or below
        const unsigned tb = T & (HP_FULL_MASK << lane);                             // ends at or above
        int a, b;
        if (hb) {
            a = c0 + 31 - __clz(hb);
        } else {  // the segment starts before this group
            a = c0;
            for (int w = 0; w < SEG_WALK && a > 0 && seg_prefix(ck[a - 1], L) == pc; ++w) --a;
            if (a > 0 && seg_prefix(ck[a - 1], L) == pc) {
                int e = a - 1;
                a = 0;
                while (a < e) {
                    const int mid = (a + e) >> 1;
                    if (seg_prefix(ck[mid], L) < pc) a = mid + 1;
                    else e = mid;
                }
            }
        }
        if (tb) {
            b = c0 + __ffs(tb);
        } else {  // the segment ends after this group
            b = min(c0 + 32, m);
            for (int w = 0; w < SEG_WALK && b < m && seg_prefix(ck[b], L) == pc; ++w) ++b;
            if (b < m && seg_prefix(ck[b], L) == pc) {
                int f = m;
                ++b;
                while (b < f) {
                    const int mid = (b + f) >> 1;
                    if (seg_prefix(ck[mid], L) > pc) f = mid;
                    else b = mid + 1;
                }
            }
        }
        a = max(a, 0);
        b = min(max(b, c + 1), m);
        if (a > c) a = c;
        if (b - a <= SEG_RANK_MAX) {
            const uint64_t lc = kc & low;
            int rank = 0;
            for (int k = a; k < b; ++k) {
                const uint64_t lk = ck[k] & low;
                rank += (lk < lc) || (lk == lc && k < c);
            }
            kout[cs + a + rank] = kc;
            vout[cs + a + rank] = cv[c];
        } else if (a == c) {  // the first element of a longer segment lists it
            const int q = atomicAdd(&S.nmed, 1);
            if (q < SEG_MED_CAP) S.med[q] = make_int2(a, b);
            else hp_report(err, HP_DEV_BAD_INDEX, (int)(cs + c));
        }
    }
    __syncthreads();
    const int nmed = min(S.nmed, SEG_MED_CAP);
    for (int q = 0; q < nmed; ++q) {  // longer segments, one at a time by the CTA
        const int a = S.med[q].x, sz = S.med[q].y - a;
        __syncthreads();
        if (a < 0 || sz <= 0 || a + sz > m) continue;  // uniform: every thread reads the same entry
        for (int j = tid; j < sz; j += SEG_BLOCK) {
            S.key[0][j] = kin[cs + a + j];
            S.val[0][j] = j;
        }
        __syncthreads();
        const int src = seg_block_sort(S, sz, L);
        for (int j = tid; j < sz; j += SEG_BLOCK) {
            const int from = a + S.val[src][j];
            kout[cs + a + j] = kin[cs + from];
            vout[cs + a + j] = vin ? vin[cs + from] : (int32_t)(cs + from);
        }
    }
    __syncthreads();
}

// A chunk read from global memory into the first key and value buffers.
__device__ void seg_sort_chunk_global(seg_smem& S, const uint64_t* __restrict__ kin,
                                      const int32_t* __restrict__ vin, uint64_t* __restrict__ kout,
                                      int32_t* __restrict__ vout, int64_t cs, int m, int L, int* err) {
    for (int j = threadIdx.x; j < m; j += SEG_BLOCK) {
        S.key[0][j] = kin[cs + j];
        S.val[0][j] = vin ? vin[cs + j] : (int32_t)(cs + j);
    }
    seg_sort_chunk(S, S.key[0], S.val[0], kin, vin, kout, vout, cs, m, L, err);
}

// One CTA per window of SEG_WINDOW positions: the segments that start in it.
// The window and the SEG_EXT positions after it are loaded once (coalesced);
// the first segment start in the window and the first one after it are found
// there. Only a segment running past the extension needs a binary search.
constexpr int SEG_EXT = 256;
constexpr int SEG_NONE = 0x7fffffff;

__global__ void __launch_bounds__(SEG_BLOCK, 4) k_seg_sort(const uint64_t* __restrict__ kin,
                                                        const int32_t* __restrict__ vin,
                                                        uint64_t* __restrict__ kout, int32_t* __restrict__ vout,
                                                        int64_t n, int L, int2* big, uint32_t* big_count,
                                                        int64_t big_cap, int* err) {
    extern __shared__ __align__(16) unsigned char seg_raw[];
    seg_smem& S = *reinterpret_cast<seg_smem*>(seg_raw);
    const int tid = threadIdx.x;
    const int64_t wb = (int64_t)blockIdx.x * SEG_WINDOW;
    const int64_t we = min(wb + SEG_WINDOW, n);
    const int64_t lo = wb > 0 ? wb - 1 : 0, hi = min(we + SEG_EXT, n);
    int* first = reinterpret_cast<int*>(&S.range[2]);  // [0] first start in the window, [1] first after it
    if (tid == 0) { first[0] = SEG_NONE; first[1] = SEG_NONE; }
    for (int64_t j = lo + tid; j < hi; j += SEG_BLOCK) {
        S.key[1][j - lo] = kin[j];
        S.val[1][j - lo] = vin ? vin[j] : (int32_t)j;
    }
    __syncthreads();
    // one shared atomic per warp and step: the warp's lowest starting lane
    // (the loop bound is uniform over the block, so every lane takes part)
    for (int64_t j0 = wb; j0 < hi; j0 += SEG_BLOCK) {
        const int64_t j = j0 + tid;
        const bool start = j < hi &&
                           (j == 0 || seg_prefix(S.key[1][j - lo], L) != seg_prefix(S.key[1][j - 1 - lo], L));
        const unsigned in_win = __ballot_sync(HP_FULL_MASK, start && j < we);
        const unsigned after = __ballot_sync(HP_FULL_MASK, start && j >= we);
        const int lane = tid & 31;
        if (in_win && lane == __ffs(in_win) - 1) atomicMin(&first[0], (int)(j - wb));
        if (after && lane == __ffs(after) - 1) atomicMin(&first[1], (int)(j - we));
    }
    __syncthreads();
    if (first[0] == SEG_NONE) return;  // a segment that started earlier covers the window
    if (tid == 0) {
        const int64_t cs = wb + first[0];
        int64_t ce;
        if (we == n) ce = n;
        else if (first[1] != SEG_NONE) ce = we + first[1];
        else if (hi == n) ce = n;
        else ce = seg_end(kin, n, we - 1, L);  // the last segment runs past the extension
        S.range[0] = cs;
        S.range[1] = ce;
    }
    __syncthreads();
    const int64_t cs = S.range[0], ce = S.range[1];
    if (ce - cs <= SEG_CAP) {
        if (ce <= hi)  // the chunk was loaded with the window
            seg_sort_chunk(S, S.key[1] + (cs - lo), S.val[1] + (cs - lo), kin, vin, kout, vout, cs,
                           (int)(ce - cs), L, err);
        else
            seg_sort_chunk_global(S, kin, vin, kout, vout, cs, (int)(ce - cs), L, err);
        return;
    }
    // A large run: batches of whole segments up to SEG_CAP keys; a segment
    // larger than that goes to the list k_seg_big sorts.
    int64_t cur = cs;
    while (cur < ce) {
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t e1 = seg_end(kin, n, cur, L);
            if (e1 - cur > SEG_CAP) {
                const uint32_t slot = atomicAdd(big_count, 1u);
                if ((int64_t)slot < big_cap) big[slot] = make_int2((int)cur, (int)e1);
                else hp_report(err, HP_DEV_BAD_INDEX, (int)cur);
                S.range[2] = e1;
                S.range[3] = e1;  // nothing to sort here
            } else {
                int64_t be = e1;
                while (be < ce) {
                    const int64_t e2 = seg_end(kin, n, be, L);
                    if (e2 - cur > SEG_CAP) break;
                    be = e2;
                }
                S.range[2] = cur;
                S.range[3] = be;
            }
        }
        __syncthreads();
        const int64_t b0 = S.range[2], b1 = S.range[3];
        if (b1 > b0) seg_sort_chunk_global(S, kin, vin, kout, vout, b0, (int)(b1 - b0), L, err);
        cur = b1;
    }
}

// Segments larger than SEG_CAP: one CTA each, stable 8-bit passes over the
// low L bits through global memory, tiles in order with running digit
// offsets; the input and output ranges serve as the two buffers.
__global__ void __launch_bounds__(SEG_BLOCK, 4) k_seg_big(uint64_t* kin, int32_t* vin_buf, const int32_t* vin,
                                                       uint64_t* kout, int32_t* vout, int L, const int2* big,
                                                       const uint32_t* big_count, int64_t big_cap, int64_t n,
                                                       int* err) {
    extern __shared__ __align__(16) unsigned char seg_raw[];
    seg_smem& S = *reinterpret_cast<seg_smem*>(seg_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t count = min((int64_t)*big_count, big_cap);
    const int passes = (L + 7) / 8;
    for (int64_t g = blockIdx.x; g < count; g += gridDim.x) {
        const int64_t s0 = big[g].x, s1 = big[g].y;
        if (s0 < 0 || s1 > n || s0 >= s1) {
            if (threadIdx.x == 0) hp_report(err, HP_DEV_BAD_INDEX, (int)g);
            continue;
        }
        // the first pass reads the input buffers, then output and input
        // ranges alternate; an even pass count ends with a copy to the output
        for (int p = 0; p < passes; ++p) {
            const bool to_out = (p & 1) == 0;
            const uint64_t* ks = to_out ? kin : kout;
            uint64_t* kd = to_out ? kout : kin;
            const int32_t* vs = p == 0 ? vin : (to_out ? vin_buf : vout);
            int32_t* vd = to_out ? vout : vin_buf;
            const int shift = 8 * p;
            // digit histogram of the segment, exclusive offsets
            if (tid < 256) S.tot[tid] = 0;
            __syncthreads();
            for (int64_t j = s0 + tid; j < s1; j += SEG_BLOCK) atomicAdd(&S.tot[(uint32_t)(ks[j] >> shift) & 255u], 1u);
            __syncthreads();
            if (tid == 0) {
                uint32_t run = 0;
                for (int d = 0; d < 256; ++d) { const uint32_t c = S.tot[d]; S.part[d] = run; run += c; }
            }
            __syncthreads();
            for (int64_t t0 = s0; t0 < s1; t0 += SEG_CAP) {
                const int m = (int)min((int64_t)SEG_CAP, s1 - t0);
                uint64_t key[SEG_ITEMS];
                int32_t val[SEG_ITEMS];
#pragma unroll
                for (int i = 0; i < SEG_ITEMS; ++i) {
                    const int e = warp * 32 * SEG_ITEMS + i * 32 + lane;
                    key[i] = e < m ? ks[t0 + e] : 0ull;
                    val[i] = e < m ? (vs ? vs[t0 + e] : (int32_t)(t0 + e)) : 0;
                }
                uint32_t pos[SEG_ITEMS];
                seg_block_rank(key, m, shift, S.cnt, S.dstart, S.tot, pos);
#pragma unroll
                for (int i = 0; i < SEG_ITEMS; ++i) {
                    const int e = warp * 32 * SEG_ITEMS + i * 32 + lane;
                    if (e < m) {
                        const uint32_t d = (uint32_t)(key[i] >> shift) & 255u;
                        const int64_t o = s0 + S.part[d] + (pos[i] - S.dstart[d]);
                        if (o >= s0 && o < s1) {  // always, unless ranges listed twice overlap
                            kd[o] = key[i];
                            vd[o] = val[i];
                        } else {
                            hp_report(err, HP_DEV_BAD_INDEX, (int)g);
                        }
                    }
                }
                __syncthreads();
                if (tid < 256) S.part[tid] += S.tot[tid];
                __syncthreads();
            }
        }
        if ((passes & 1) == 0) {  // the last pass wrote the input range
            for (int64_t j = s0 + tid; j < s1; j += SEG_BLOCK) {
                kout[j] = kin[j];
                vout[j] = vin_buf[j];
            }
        }
        __syncthreads();
    }
}

template <typename K, int BLOCK>
hp_status sort_run_t(const hp_sort_plan& plan, const hp_sort_args& a, cudaStream_t stream) {
    constexpr int ITEMS = sort_cfg<K>::ITEMS;
    const int64_t n = plan.n;
    hp_carve cv(reinterpret_cast<char*>(a.scratch));
    K* kA = cv.take<K>(n);
    int32_t* vA = cv.take<int32_t>(n);
    K* kB = cv.take<K>(n);
    int32_t* vB = cv.take<int32_t>(n);
    uint32_t* status = cv.take<uint32_t>((size_t)plan.passes * plan.tiles * 256 + 64);
    uint32_t* counters = status + (size_t)plan.passes * plan.tiles * 256;
    HP_CUDA(cudaMemsetAsync(status, 0, ((size_t)plan.passes * plan.tiles * 256 + 64) * 4, stream));
    if (!a.hist_ready && !(sizeof(K) == 8 && hybrid_sort(n, 8, plan.bits))) {
        HP_CUDA(cudaMemsetAsync(a.hist, 0, hp_sort_hist_bytes(plan.passes), stream));
        int grid = (int)std::min<int64_t>(hp_div_up(n, 1024), 148 * 8);
        k_sort_hist<K><<<std::max(grid, 1), 1024, plan.passes * 256 * 4, stream>>>(
            reinterpret_cast<const K*>(a.keys_in), n, plan.passes, plan.bits, a.hist);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(a.ctx, stream, "sort_hist");
    }
    constexpr size_t smem = onesweep_smem<K, BLOCK>();
    HP_CUDA(cudaFuncSetAttribute(k_onesweep<K, BLOCK, ITEMS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const K* kin = reinterpret_cast<const K*>(a.keys_in);
    const int32_t* vin = a.vals_in;
    if constexpr (sizeof(K) == 8) {
        if (hybrid_sort(n, 8, plan.bits)) {
            // top 24 bits by three LSD passes, then every segment of equal prefix
            const int s0 = plan.bits - 8 * SEG_TOP;
            if (!a.hist_ready) {
                HP_CUDA(cudaMemsetAsync(a.hist, 0, 256 * SEG_TOP * sizeof(uint32_t), stream));
                k_hist_top<<<std::max(1, (int)std::min<int64_t>(hp_div_up(n, 1024), 148 * 8)), 1024, 0,
                             stream>>>(kin, n, s0, a.hist);
                HP_CUDA(cudaGetLastError());
                hp_count_launch();
            }
            const uint32_t sl = a.ctx ? a.ctx->sort_spin_limit : LOOKBACK_SPIN_LIMIT;
            const K* src_k = kin;
            const int32_t* src_v = vin;
            for (int d = 0; d < SEG_TOP; ++d) {  // in -> A -> B -> A
                K* dk = (d & 1) ? kB : kA;
                int32_t* dv = (d & 1) ? vB : vA;
                k_onesweep<K, BLOCK, ITEMS><<<(unsigned)plan.tiles, BLOCK, smem, stream>>>(
                    src_k, src_v, dk, dv, n, s0 + 8 * d, 0xffu, a.hist + 256 * d,
                    status + (size_t)d * plan.tiles * 256, counters + d, a.status, sl);
                HP_CUDA(cudaGetLastError());
                hp_count_launch();
                hp_mark(a.ctx, stream, "sort_pass");
                src_k = dk;
                src_v = dv;
            }
            uint64_t* sk = const_cast<uint64_t*>(reinterpret_cast<const uint64_t*>(src_k));
            int32_t* sv = const_cast<int32_t*>(src_v);
            uint32_t* big_count = counters + 32;  // zeroed with the status words
            const int64_t big_cap = n / (SEG_CAP + 1) + 1;
            int2* big = reinterpret_cast<int2*>(cv.take<int2>((size_t)big_cap));
            const size_t seg_bytes = sizeof(seg_smem);
            HP_CUDA(cudaFuncSetAttribute(k_seg_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)seg_bytes));
            HP_CUDA(cudaFuncSetAttribute(k_seg_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)seg_bytes));
            k_seg_sort<<<(unsigned)hp_div_up(n, SEG_WINDOW), SEG_BLOCK, seg_bytes, stream>>>(
                sk, sv, reinterpret_cast<uint64_t*>(a.keys_out), a.vals_out, n, s0, big, big_count, big_cap,
                a.status);
            HP_CUDA(cudaGetLastError());
            k_seg_big<<<(unsigned)std::min<int64_t>(big_cap, 296), SEG_BLOCK, seg_bytes, stream>>>(
                sk, sv, sv, reinterpret_cast<uint64_t*>(a.keys_out), a.vals_out, s0, big, big_count, big_cap, n,
                a.status);
            HP_CUDA(cudaGetLastError());
            hp_count_launch(2);
            hp_mark(a.ctx, stream, "sort_segments");
            return HP_OK;
        }
    }
    for (int p = 0; p < plan.passes; ++p) {
        K* kout;
        int32_t* vout;
        if (p == plan.passes - 1) {
            kout = reinterpret_cast<K*>(a.keys_out);
            vout = a.vals_out;
        } else if ((p & 1) == 0) {
            kout = kA;
            vout = vA;
        } else {
            kout = kB;
            vout = vB;
        }
        int shift = 8 * p;
        int w = std::min(8, plan.bits - shift);
        k_onesweep<K, BLOCK, ITEMS><<<(unsigned)plan.tiles, BLOCK, smem, stream>>>(
            kin, vin, kout, vout, n, shift, (1u << w) - 1u, a.hist + 256 * p,
            status + (size_t)p * plan.tiles * 256, counters + p, a.status,
            a.ctx ? a.ctx->sort_spin_limit : LOOKBACK_SPIN_LIMIT);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
        hp_mark(a.ctx, stream, "sort_pass");
        kin = kout;
        vin = vout;
    }
    return HP_OK;
}

// ---- single-pass scans with decoupled look-back ---------------------------------
// Status word: [63:62] flag, [61:31] value a, [30:0] value b (values < 2^31).
constexpr uint64_t SC_FLAG_A = 1ull << 62, SC_FLAG_P = 2ull << 62, SC_FLAGS = 3ull << 62;
constexpr int SCAN_BLOCK = 256, SCAN_ITEMS = 16, SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ uint64_t sc_pack(uint64_t flag, uint32_t a, uint32_t b) {
    return flag | ((uint64_t)(a & 0x7fffffffu) << 31) | (uint64_t)(b & 0x7fffffffu);
}

// MAX = false: exclusive sums of a and b. MAX = true: exclusive max of a
// (identity -1; stored shifted by +1), b unused.
template <bool MAX>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_lb(
    const int32_t* __restrict__ a, int64_t na, const int32_t* __restrict__ b, int64_t nb,
    int32_t* __restrict__ a_out, int32_t* __restrict__ b_out, int32_t* totals,
    uint64_t* status, uint32_t* tile_counter, int64_t num_tiles, int* err) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_wa[SCAN_BLOCK / 32], s_wb[SCAN_BLOCK / 32];
    __shared__ uint32_t s_pa, s_pb;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * SCAN_TILE + (int64_t)tid * SCAN_ITEMS;
    uint32_t va[SCAN_ITEMS], vb[SCAN_ITEMS];
    uint32_t ta = 0, tb = 0;  // thread aggregate (a stored shifted by +1 for MAX)
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + i;
        if (MAX) {
            va[i] = (idx < na) ? (uint32_t)(a[idx] + 1) : 0u;
            ta = max(ta, va[i]);
        } else {
            va[i] = (idx < na) ? (uint32_t)a[idx] : 0u;
            vb[i] = (b && idx < nb) ? (uint32_t)b[idx] : 0u;
            ta += va[i];
            tb += vb[i];
        }
    }
    // block-level inclusive scan of thread aggregates
    uint32_t ia = ta, ib = tb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t ya = __shfl_up_sync(HP_FULL_MASK, ia, o);
        uint32_t yb = __shfl_up_sync(HP_FULL_MASK, ib, o);
        if (lane >= o) {
            if (MAX) ia = max(ia, ya);
            else { ia += ya; ib += yb; }
        }
    }
    if (lane == 31) { s_wa[warp] = ia; s_wb[warp] = ib; }
    __syncthreads();
    uint32_t wa = 0, wb = 0, blk_a = 0, blk_b = 0;
#pragma unroll
    for (int w = 0; w < SCAN_BLOCK / 32; ++w) {
        if (w < warp) {
            if (MAX) wa = max(wa, s_wa[w]);
            else { wa += s_wa[w]; wb += s_wb[w]; }
        }
        if (MAX) blk_a = max(blk_a, s_wa[w]);
        else { blk_a += s_wa[w]; blk_b += s_wb[w]; }
    }
    if (tid == 0) {
        st_relaxed_u64(&status[tile], sc_pack(tile == 0 ? SC_FLAG_P : SC_FLAG_A, blk_a, blk_b));
        uint32_t pa = 0, pb = 0;
        if (tile > 0) {
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (true) {
                uint64_t s = ld_relaxed_u64(&status[t]);
                uint64_t f = s & SC_FLAGS;
                if (f == 0) {
                    if (++spins > LOOKBACK_SPIN_LIMIT) {
                        hp_report(err, HP_DEV_SPIN_LIMIT, (int)tile);
                        break;
                    }
                    continue;
                }
                uint32_t xa = (uint32_t)((s >> 31) & 0x7fffffffu), xb = (uint32_t)(s & 0x7fffffffu);
                if (MAX) pa = max(pa, xa);
                else { pa += xa; pb += xb; }
                if (f == SC_FLAG_P || t == 0) break;
                --t;
            }
            uint32_t ia2 = MAX ? max(pa, blk_a) : pa + blk_a;
            st_relaxed_u64(&status[tile], sc_pack(SC_FLAG_P, ia2, pb + blk_b));
        }
        s_pa = pa;
        s_pb = pb;
        if (tile == num_tiles - 1 && totals) {
            if (MAX) totals[0] = (int32_t)max(pa, blk_a) - 1;
            else { totals[0] = (int32_t)(pa + blk_a); totals[1] = (int32_t)(pb + blk_b); }
        }
    }
    __syncthreads();
    uint32_t ra, rb;
    // running exclusive value for this thread's first item
    if (MAX) {
        // exclusive prefix of the thread = max(tile prefix, warps before, lanes before)
        uint32_t lanes_before = __shfl_up_sync(HP_FULL_MASK, ia, 1);
        if (lane == 0) lanes_before = 0;
        ra = max(max(s_pa, wa), lanes_before);
        rb = 0;
    } else {
        ra = s_pa + wa + ia - ta;
        rb = s_pb + wb + ib - tb;
    }
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + i;
        if (MAX) {
            if (idx < na) a_out[idx] = (int32_t)ra - 1;
            ra = max(ra, va[i]);
        } else {
            if (idx < na) a_out[idx] = (int32_t)ra;
            if (b && idx < nb) b_out[idx] = (int32_t)rb;
            ra += va[i];
            rb += vb[i];
        }
    }
}

// Checked mode: every adjacent pair of the output in order by its low `bits`
// bits; the first pair found out of order is reported with its position.
template <typename K>
__global__ void k_sort_check(const K* __restrict__ keys, int64_t n, int bits, int* status) {
    const K mask = bits >= (int)(8 * sizeof(K)) ? ~K(0) : ((K(1) << bits) - 1);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x + 1; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if ((__ldg(keys + i - 1) & mask) > (__ldg(keys + i) & mask))
            hp_report(status, HP_DEV_CHECK_FAILED, (int)i);
}

}  // namespace

hp_status hp_sort_check_launch(hp_ctx* ctx, const void* keys_out, int64_t n, int key_bytes, int bits,
                               cudaStream_t s) {
    if (n < 2) return HP_OK;
    const unsigned grid = (unsigned)std::min<int64_t>(hp_div_up(n, 256), 8 * (int64_t)ctx->sm_count);
    if (key_bytes == 4)
        k_sort_check<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(keys_out), n, bits, ctx->d_status);
    else
        k_sort_check<uint64_t><<<grid, 256, 0, s>>>(static_cast<const uint64_t*>(keys_out), n, bits, ctx->d_status);
    HP_CUDA(cudaGetLastError());
    hp_count_launch();
    return HP_OK;
}

hp_sort_plan hp_sort_make_plan(int64_t n, int key_bytes, int bits, int block) {
    hp_sort_plan p;
    p.n = n;
    p.key_bytes = key_bytes;
    p.bits = bits;
    p.passes = (bits + 7) / 8;
    p.block = block == 256 ? 256 : 512;
    p.tile = p.block * (key_bytes == 4 ? sort_cfg<uint32_t>::ITEMS : sort_cfg<uint64_t>::ITEMS);
    p.tiles = std::max<int64_t>(1, (n + p.tile - 1) / p.tile);
    size_t kv = hp_carve::pad((size_t)n * key_bytes) + hp_carve::pad((size_t)n * 4);
    p.scratch_bytes = 2 * kv + hp_carve::pad(((size_t)p.passes * p.tiles * 256 + 64) * 4);
    if (hybrid_sort(n, key_bytes, bits))  // the list of segments too large for one CTA's shared memory
        p.scratch_bytes += hp_carve::pad((size_t)(n / (SEG_CAP + 1) + 1) * 8);
    return p;
}

size_t hp_sort_hist_bytes(int passes) { return (size_t)passes * 256 * 4; }

void hp_sort_hist_digits(const hp_sort_plan& plan, int* shift0, int* count) {
    if (hybrid_sort(plan.n, plan.key_bytes, plan.bits)) {
        *shift0 = plan.bits - 8 * SEG_TOP;
        *count = SEG_TOP;
    } else {
        *shift0 = 0;
        *count = plan.passes;
    }
}

hp_status hp_sort_run(const hp_sort_plan& plan, const hp_sort_args& a, cudaStream_t stream) {
    if (plan.n <= 0) return HP_OK;
    if (plan.n >= (int64_t(1) << 30))
        return hp_fail(HP_ERR_ARG, "radix sort: n must be below 2^30");
    if (plan.block == 256) {
        if (plan.key_bytes == 4) return sort_run_t<uint32_t, 256>(plan, a, stream);
        return sort_run_t<uint64_t, 256>(plan, a, stream);
    }
    if (plan.key_bytes == 4) return sort_run_t<uint32_t, 512>(plan, a, stream);
    return sort_run_t<uint64_t, 512>(plan, a, stream);
}

size_t hp_scan2_scratch_bytes(int64_t n) {
    int64_t tiles = std::max<int64_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    return hp_carve::pad((size_t)tiles * 8 + 256);
}

void hp_scan2_sum(const int32_t* a, int64_t na, const int32_t* b, int64_t nb, int32_t* a_out,
                  int32_t* b_out, int32_t* totals, void* scratch, int* status, cudaStream_t stream) {
    int64_t n = std::max(na, nb);
    int64_t tiles = std::max<int64_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    uint64_t* st = reinterpret_cast<uint64_t*>(scratch);
    uint32_t* counter = reinterpret_cast<uint32_t*>(st + tiles);
    cudaMemsetAsync(scratch, 0, (size_t)tiles * 8 + 256, stream);
    k_scan_lb<false><<<(unsigned)tiles, SCAN_BLOCK, 0, stream>>>(a, na, b, nb, a_out, b_out, totals,
                                                                 st, counter, tiles, status);
    hp_count_launch();
}

void hp_scan_max_excl(const int32_t* in, int64_t n, int32_t* out, void* scratch, int* status,
                      cudaStream_t stream) {
    int64_t tiles = std::max<int64_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    uint64_t* st = reinterpret_cast<uint64_t*>(scratch);
    uint32_t* counter = reinterpret_cast<uint32_t*>(st + tiles);
    cudaMemsetAsync(scratch, 0, (size_t)tiles * 8 + 256, stream);
    k_scan_lb<true><<<(unsigned)tiles, SCAN_BLOCK, 0, stream>>>(in, n, nullptr, 0, out, nullptr,
                                                                nullptr, st, counter, tiles, status);
    hp_count_launch();
}

// ---- sort without allocation --------------------------------------------------------------
// Callers that may not allocate device memory (a plugin whose host application
// owns the GPU memory budget, or a loop where cudaMalloc's implicit device
// synchronisation is not acceptable) get the same sort with its scratch in
// this file-scope device array. Host code never names the array as a pointer:
// the symbol is a host-side stand-in, so its device address is looked up once
// per device with cudaGetSymbolAddress and then passed to the kernels.
namespace {

constexpr size_t noalloc_pad(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t noalloc_sort_scratch(int64_t n, size_t key_bytes, int tile, int passes) {
    return 2 * (noalloc_pad((size_t)n * key_bytes) + noalloc_pad((size_t)n * 4)) +
           noalloc_pad(((size_t)passes * (size_t)((n + tile - 1) / tile) * 256 + 64) * 4);
}
constexpr size_t noalloc_max(size_t a, size_t b) { return a > b ? a : b; }
// Largest sort scratch over both key widths, plus the digit histograms and an error word.
constexpr size_t NOALLOC_BYTES =
    noalloc_max(noalloc_sort_scratch(HP_NOALLOC_SORT_MAX_KEYS, 8,
                                     sort_cfg<uint64_t>::BLOCK * sort_cfg<uint64_t>::ITEMS, 8),
                noalloc_sort_scratch(HP_NOALLOC_SORT_MAX_KEYS, 4,
                                     sort_cfg<uint32_t>::BLOCK * sort_cfg<uint32_t>::ITEMS, 4)) +
    noalloc_pad(8 * 256 * 4) + 256;

__device__ __align__(256) unsigned char g_noalloc_sort_scratch[NOALLOC_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_base[NOALLOC_MAX_DEVICES] = {};

// The sort's kernels report into a (code, info) pair inside the fixed array;
// the caller's status is one int32 and receives only the code.
__global__ void k_noalloc_status_out(const int* own, int32_t* out) { *out = own[0]; }

}  // namespace

extern "C" hp_status hp_radix_sort_noalloc(const void* keys_in, const int32_t* vals_in, void* keys_out,
                                           int32_t* vals_out, int64_t n, int32_t key_bytes, int32_t bits,
                                           int32_t* device_status, void* stream) {
    if (key_bytes != 4 && key_bytes != 8)
        return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: key_bytes must be 4 or 8");
    if (bits < 1 || bits > 8 * key_bytes) return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: bits out of range");
    if (n < 0) return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: negative n");
    if (n > HP_NOALLOC_SORT_MAX_KEYS)
        return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: n = " + std::to_string(n) +
                                       " exceeds the fixed scratch capacity of " +
                                       std::to_string(HP_NOALLOC_SORT_MAX_KEYS) + " keys");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (device_status) HP_CUDA(cudaMemsetAsync(device_status, 0, sizeof(int32_t), s));
        return HP_OK;
    }
    if (!keys_in || !keys_out || !vals_out) return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: null buffer");
    int dev = 0;
    HP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: device id too large");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_base[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
            if (e != cudaSuccess) return hp_cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_sort_scratch)");
            g_noalloc_base[dev] = p;
        }
        base = g_noalloc_base[dev];
    }
    const hp_sort_plan plan = hp_sort_make_plan(n, key_bytes, bits);
    hp_carve cv(reinterpret_cast<char*>(base));
    void* scratch = cv.take<char>(plan.scratch_bytes);
    uint32_t* hist = cv.take<uint32_t>(plan.passes * 256);
    int* own_status = cv.take<int>(64);
    if (cv.off > NOALLOC_BYTES) return hp_fail(HP_ERR_ARG, "hp_radix_sort_noalloc: scratch plan exceeds the fixed array");
    // The array keeps the previous call's contents: the status pair starts at
    // zero every call (the sort clears its own look-back words and histograms).
    HP_CUDA(cudaMemsetAsync(own_status, 0, 2 * sizeof(int), s));
    hp_sort_args a{keys_in, vals_in, keys_out, vals_out, scratch, hist, false, own_status, nullptr};
    HP_TRY(hp_sort_run(plan, a, s));
    if (device_status) {
        k_noalloc_status_out<<<1, 1, 0, s>>>(own_status, device_status);
        HP_CUDA(cudaGetLastError());
        hp_count_launch();
    }
    return HP_OK;
}
