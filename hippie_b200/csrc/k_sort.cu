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
    if (!a.hist_ready) {
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

}  // namespace

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
    return p;
}

size_t hp_sort_hist_bytes(int passes) { return (size_t)passes * 256 * 4; }

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
