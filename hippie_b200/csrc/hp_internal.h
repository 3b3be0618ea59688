// Host-side internal declarations shared by the library's translation units.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include "../../include/hippie_b200.h"

struct hp_node_bin;

// ---- error handling ------------------------------------------------------
void hp_set_error(const std::string& msg);
hp_status hp_fail(hp_status code, const std::string& msg);
hp_status hp_cuda_fail(cudaError_t e, const char* what);
#define HP_CUDA(call)                                                \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return hp_cuda_fail(e_, #call);       \
    } while (0)
#define HP_TRY(call)                                                 \
    do {                                                             \
        hp_status s_ = (call);                                       \
        if (s_ != HP_OK) return s_;                                  \
    } while (0)

// ---- device-side BVH summary -------------------------------------------------
struct hp_bvh_info {
    int32_t num_interior;
    int32_t num_leaf;
    uint32_t box_ord[6];    // scene box as order-preserving uints (min xyz, max xyz)
    float scale[3];         // Morton scale actually used
    int32_t pad;
};

struct hp_bvh_impl {
    hp_node_bin* nodes = nullptr;
    float4* woop = nullptr;
    int32_t* tri_idx = nullptr;
    int32_t* counters = nullptr;   // refit termination counters [capacity]
    hp_bvh_info* info = nullptr;   // device
    int64_t capacity = 0;          // references
    size_t node_capacity = 0;      // bytes of the node buffer
    int layout = 2;                // children per node: 2, 4 or 8
    bool view = false;             // storage owned by a batch (hp_batch_bvh)
};

// ---- context: scratch arena, error words, phase events ------------------------
struct hp_prof_mark {
    cudaEvent_t ev;
    char name[32];
};

struct hp_ctx {
    int device = 0;
    int sm_count = 148;
    size_t l2_bytes = 0;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    int* d_status = nullptr;       // [64] device words: 0-1 error code and info, 16-17 trace ray counter, 20-23 hp_trace_host counters, 32 LBVH climb leaf ticket
    int* h_status = nullptr;       // pinned mirror
    bool profiling = false;
    hp_prof_mark* marks = nullptr; // event pool
    int num_marks = 0;
    int cap_marks = 0;
    hp_tune tune{512, 0, 16, 0, 0, 0, 0, 0.0f, 0.0f, {0}};  // launch choices (hp_ctx_set_tune)
    int ray_key_method = HP_RAY_KEYS_AILA;  // hp_ctx_set_ray_keys
    float ray_length = 0.25f;
    // Spins of one look-back wait of the radix sort before it gives up and
    // reports HP_DEV_SPIN_LIMIT (hp_ctx_set_sort_spin_limit).
    uint32_t sort_spin_limit = HP_SORT_SPIN_LIMIT_DEFAULT;
    int arith = HP_ARITH_IEEE;  // hp_ctx_set_arithmetic
    // Checked mode (hp_ctx_set_checked, or HP_CHECKED=1 in the environment at
    // hp_ctx_create): every entry point synchronises and verifies its output.
    bool checked = false;
    // hp_trace_host: copy streams, one trace stream per staging slot, events
    // and two device staging slots
    cudaStream_t io_h2d = nullptr, io_d2h = nullptr, io_trace[2] = {nullptr, nullptr};
    cudaEvent_t io_start = nullptr;
    cudaEvent_t io_up[2] = {nullptr, nullptr}, io_traced[2] = {nullptr, nullptr}, io_free[2] = {nullptr, nullptr};
    char* io_slot[2] = {nullptr, nullptr};
    size_t io_slot_bytes = 0;
};

// An NVTX range around a public entry point (header-only NVTX 3: a no-op
// unless a profiler such as Nsight Systems injects its handler).
struct hp_nvtx_range {
    explicit hp_nvtx_range(const char* name) { nvtxRangePushA(name); }
    ~hp_nvtx_range() { nvtxRangePop(); }
    hp_nvtx_range(const hp_nvtx_range&) = delete;
    hp_nvtx_range& operator=(const hp_nvtx_range&) = delete;
};

// Checked mode: true when the context verifies outputs and the stream can be
// synchronised (a stream under capture is not: the checks are skipped there).
bool hp_checking(const hp_ctx* ctx, cudaStream_t s);
// Checked mode's verification of a sort output: keys_out ordered by their low
// `bits` bits, else HP_DEV_CHECK_FAILED in the context's status word.
hp_status hp_sort_check_launch(hp_ctx* ctx, const void* keys_out, int64_t n, int key_bytes, int bits,
                               cudaStream_t s);

// Record a phase boundary on the stream when profiling is enabled.
void hp_mark(hp_ctx* ctx, cudaStream_t s, const char* name);
// Count kernel launches made by the library on this thread.
void hp_count_launch(int k = 1);

hp_status hp_ctx_reserve(hp_ctx* ctx, size_t bytes, cudaStream_t stream);

// Reference arithmetic (k_refarith.cu): Woop rows of every reference of a
// built BVH rewritten with the fast-math reciprocal, and the binary tracer
// with the fast-math reciprocals (same arguments as hp_trace_launch).
hp_status hp_woop_ref_launch(hp_ctx* ctx, hp_bvh_impl* b, int64_t n_refs, const hp_mesh* m, cudaStream_t s);
hp_status hp_trace_ref_launch(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                              int64_t num_rays, int32_t* results, int32_t* stats, uint32_t flags,
                              unsigned long long* counter, const int32_t* order, cudaStream_t s);

// Bump allocator over the context arena (256-byte aligned pieces).
struct hp_carve {
    char* base;
    size_t off = 0;
    explicit hp_carve(char* b) : base(b) {}
    template <typename T> T* take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += bytes;
        return p;
    }
    static size_t pad(size_t bytes) { return (bytes + 255) & ~size_t(255); }
};

// ---- N-wide layouts (k_wide.cu, k_trace_wide.cu) -------------------------------
// The final binary tree of a build (root 0, leaf n-1+p holding sorted position p).
struct hp_wide_in {
    int n = 0;
    int width = 4;
    const int* parent = nullptr;     // [2n-1]
    const int* left = nullptr;       // interior nodes
    const int* right = nullptr;
    const float4* nbmin = nullptr;   // [2n-1], xyz used
    const float4* nbmax = nullptr;
    const int32_t* sorted_tri = nullptr;  // sorted position -> triangle
    bool reorder = true;             // write references (and Woop) in depth-first order
    float ct = 3.0f, ci = 2.0f;
    int max_leaf = 0x7fffffff;       // INT_MAX: adaptive leaves
    const float* verts = nullptr;
    int64_t nv = 0;
    const int32_t* tris = nullptr;
};
size_t hp_wide_scratch_bytes(int64_t n, int width);
hp_status hp_wide_collapse(hp_ctx* ctx, const hp_wide_in& in, hp_bvh_impl* out, void* scratch, cudaStream_t s);
hp_status hp_wide_single(hp_ctx* ctx, const hp_mesh* m, int width, hp_bvh_impl* out, cudaStream_t s);
hp_status hp_trace_wide_launch(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                               int64_t num_rays, int32_t* results, int32_t* stats, uint32_t flags,
                               unsigned long long* counter, const int32_t* order, cudaStream_t s);
inline int hp_layout_of(const hp_build_params* p) { return p->layout == 0 ? 2 : p->layout; }

// ---- BVH statistics and validation (k_stats.cu) ------------------------------
hp_status hp_bvh_stats_run(hp_ctx* ctx, const hp_bvh* bvh, hp_bvh_stats* out, cudaStream_t s);
hp_status hp_bvh_validate_run(hp_ctx* ctx, const hp_bvh* bvh, const hp_mesh* m, int32_t* valid, cudaStream_t s);

// ---- radix sort ------------------------------------------------------------
struct hp_sort_plan {
    int64_t n = 0;
    int key_bytes = 4;
    int bits = 32;
    int passes = 0;
    int tile = 0;
    int64_t tiles = 0;
    size_t scratch_bytes = 0;      // keys/vals ping-pong + histograms + status
    int block = 512;               // threads per pass CTA: 512 or 256
};
hp_sort_plan hp_sort_make_plan(int64_t n, int key_bytes, int bits, int block = 512);
// The digit histograms a sort starts from: `count` 8-bit digits at shifts
// shift0, shift0 + 8, ... (digit width min(8, bits - shift)), laid out
// [count][256] (uint32). An LSD sort counts every pass's digit from shift 0;
// the wide-key sort only the three digits below its top bit.
void hp_sort_hist_digits(const hp_sort_plan& plan, int* shift0, int* count);
// The histograms must be zero before the first key is counted; hp_sort_run
// zeroes and fills them itself unless hist_ready is set, in which case the
// caller has already filled them as hp_sort_hist_digits says (the Morton
// kernels do).
struct hp_sort_args {
    const void* keys_in;
    const int32_t* vals_in;        // nullptr: values are 0..n-1
    void* keys_out;
    int32_t* vals_out;
    void* scratch;                 // plan.scratch_bytes
    uint32_t* hist;                // [passes*256]; inside or outside scratch
    bool hist_ready;
    int* status;                   // device error word
    hp_ctx* ctx;                   // for phase marks (may be null)
};
hp_status hp_sort_run(const hp_sort_plan& plan, const hp_sort_args& a, cudaStream_t stream);

// Ray order of a sorted trace: the context's ray keys of `bits` bits
// (32-bit keys with the digit histograms made in the key kernel when bits <=
// 32), stably sorted; order[k] is the k-th ray. Scratch of
// hp_ray_order_scratch_bytes(n, bits, ctx->tune.sort_block) bytes.
size_t hp_ray_order_scratch_bytes(int64_t n, int bits, int block);
hp_status hp_ray_order(hp_ctx* ctx, const float* rays, int64_t n, int bits, int32_t* order, void* scratch,
                       cudaStream_t s);
size_t hp_sort_hist_bytes(int passes);

// ---- single-pass scans --------------------------------------------------------
// Exclusive prefix sums of two int arrays at once (a: na items, b: nb items),
// written to a_out / b_out; totals written to totals[0], totals[1].
size_t hp_scan2_scratch_bytes(int64_t n);
void hp_scan2_sum(const int32_t* a, int64_t na, const int32_t* b, int64_t nb,
                  int32_t* a_out, int32_t* b_out, int32_t* totals, void* scratch,
                  int* status, cudaStream_t stream);
// Exclusive max-scan of in[0..n) with identity -1 into out.
void hp_scan_max_excl(const int32_t* in, int64_t n, int32_t* out, void* scratch,
                      int* status, cudaStream_t stream);

// ---- LBVH / collapse --------------------------------------------------------------
size_t hp_lbvh_scratch_bytes(int64_t n, int key_bytes, int bits);
hp_status hp_lbvh_build(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p,
                        hp_bvh_impl* out, const hp_build_taps* taps, cudaStream_t stream);
// PLOC clustering and depth-first collapse after the references are sorted.
size_t hp_ploc_scratch_bytes(int64_t n);
// woop_src (or null): Woop rows per scene triangle, gathered by the collapse.
hp_status hp_ploc_stage(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out,
                        const int32_t* sorted_tri, const float4* tbmin, const float4* tbmax,
                        void* scratch, void* wide_scratch, cudaStream_t stream, const float4* woop_src = nullptr);
// Depth-first collapse of a binary tree (interior nodes 0..n-2, leaves n-1..2n-2,
// sorted reference p at leaf n-1+p) into 64-byte nodes, the triangle order and
// Woop triangles. nbmax.w holds each node's size; counts the surviving interior
// nodes and collapsed leaves of each subtree. order (2n-1) lists the nodes with
// every parent before its children; null means parents have lower indices.
struct hp_topdown_in {
    int n;
    const int* left;
    const int* right;
    const int* parent;
    const int2* counts;
    const uint8_t* state;
    const float4* nbmin;
    const float4* nbmax;
    const int* order;
    const int32_t* sorted_tri;
};
size_t hp_topdown_scratch_bytes(int64_t n);
hp_status hp_topdown_collapse(hp_ctx* ctx, const hp_mesh* m, const hp_topdown_in& in, hp_bvh_impl* out,
                              void* scratch, cudaStream_t stream);
// ATR restructuring of a Karras tree and its collapse (method HP_METHOD_ATR).
size_t hp_atr_scratch_bytes(int64_t n);
hp_status hp_atr_stage(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh_impl* out, int n,
                       const int32_t* sorted_tri, int* parent, int* left, int* right, float4* nbmin,
                       float4* nbmax, int* counters, const float4* tbmin, const float4* tbmax, void* scratch,
                       void* wide_scratch, cudaStream_t stream);
// HLBVH top-level rebuild of a Karras tree over its sorted keys (method
// HP_METHOD_HLBVH): refits the LBVH boxes, finds the clusters below the top
// hlbvh_sah_bits of the key and rebuilds the tree above them by binned SAH.
// The tree is then refitted and collapsed by hp_atr_stage with no iterations.
size_t hp_hlbvh_scratch_bytes(int64_t n, int sah_bits);
hp_status hp_hlbvh_stage(hp_ctx* ctx, const hp_build_params* p, int n, const void* skeys, int key_bytes,
                         const int32_t* sorted_tri, const float4* tbmin, const float4* tbmax, int* parent, int* left,
                         int* right, const int2* range, float4* nbmin, float4* nbmax, int* counters, void* scratch,
                         cudaStream_t stream);
hp_status hp_refit_launch(hp_ctx* ctx, hp_bvh_impl* b, int64_t n_refs, const hp_mesh* m,
                          cudaStream_t stream);

// ---- batches of meshes -------------------------------------------------------------
// One entry per mesh of a batch (device table). The mesh's sorted positions,
// woop rows and triangle-index slots start at tri_off, its node slots at
// node_off (max(2n-1, 3) of them) and its rays at ray_off.
struct hp_batch_seg {
    const float* verts;
    const int32_t* tris;
    int64_t nv;
    int32_t n;
    int32_t tri_off;
    int64_t node_off;
    int64_t ray_off;
};
struct hp_batch_trace_args {
    const float* rays;
    int64_t num_rays;
    int32_t* results;
    int32_t* stats;
    const hp_node_bin* nodes;
    const float4* woop;
    const int32_t* tri_idx;
    const hp_batch_seg* segs;
    const int64_t* ray_off;   // [num_segs + 1]
    int num_segs;
};
hp_status hp_trace_batch_launch(hp_ctx* ctx, const hp_batch_trace_args& t, uint32_t flags, cudaStream_t stream);

// ---- trace / adjoint ---------------------------------------------------------------
// order (or null): slot k of the launch traces ray order[k]. counter (or null
// for the context's own): the launch's 8-byte work counter; launches that may
// run at the same time need counters of their own.
hp_status hp_trace_launch(hp_ctx* ctx, const hp_bvh_impl* b, int64_t n_refs, const float* rays,
                          int64_t num_rays, int32_t* results, int32_t* stats, uint32_t flags,
                          cudaStream_t stream, const int32_t* order = nullptr,
                          unsigned long long* counter = nullptr);
hp_status hp_adjoint_launch(hp_ctx* ctx, const hp_mesh* m, const float* rays,
                            const int32_t* results, const float* dl_dtuv, int64_t num_rays,
                            float* dl_dvertices, cudaStream_t stream);

inline int hp_div_up(int64_t a, int64_t b) { return int((a + b - 1) / b); }
