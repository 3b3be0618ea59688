// C ABI entry points: context and scratch arena, BVH objects, build / refit /
// trace / adjoint dispatch, host-side cost and validation.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "hp_device.cuh"
#include "hp_internal.h"

namespace {
thread_local std::string g_last_error;
thread_local int64_t g_launches = 0;
}

void hp_count_launch(int k) { g_launches += k; }

void hp_mark(hp_ctx* ctx, cudaStream_t s, const char* name) {
    if (!ctx || !ctx->profiling) return;
    if (ctx->num_marks == ctx->cap_marks) {
        int cap = ctx->cap_marks ? 2 * ctx->cap_marks : 64;
        hp_prof_mark* m = new hp_prof_mark[cap];
        for (int i = 0; i < ctx->num_marks; ++i) m[i] = ctx->marks[i];
        for (int i = ctx->num_marks; i < cap; ++i) cudaEventCreate(&m[i].ev);
        delete[] ctx->marks;
        ctx->marks = m;
        ctx->cap_marks = cap;
    }
    hp_prof_mark& mk = ctx->marks[ctx->num_marks++];
    std::snprintf(mk.name, sizeof(mk.name), "%s", name);
    cudaEventRecord(mk.ev, s);
}

void hp_set_error(const std::string& msg) { g_last_error = msg; }

hp_status hp_fail(hp_status code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

hp_status hp_cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return HP_ERR_OOM;
    }
    return HP_ERR_CUDA;
}

hp_status hp_ctx_reserve(hp_ctx* ctx, size_t bytes, cudaStream_t stream) {
    if (bytes <= ctx->arena_bytes) return HP_OK;
    // Growing the arena: wait for work that may still use the old one.
    HP_CUDA(cudaDeviceSynchronize());
    if (ctx->arena) HP_CUDA(cudaFree(ctx->arena));
    ctx->arena = nullptr;
    ctx->arena_bytes = 0;
    size_t grow = std::max(bytes, bytes + bytes / 8);
    cudaError_t e = cudaMalloc(&ctx->arena, grow);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&ctx->arena, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return hp_fail(HP_ERR_OOM, "scratch arena: cannot allocate " + std::to_string(bytes) + " bytes");
        }
        grow = bytes;
    }
    ctx->arena_bytes = grow;
    (void)stream;
    return HP_OK;
}

namespace {

hp_status check_mesh(const hp_mesh* m) {
    if (!m) return hp_fail(HP_ERR_ARG, "mesh is null");
    if (m->num_triangles < 0 || m->num_vertices < 0) return hp_fail(HP_ERR_ARG, "negative mesh size");
    if (m->num_triangles > 0 && (!m->vertices || !m->triangles))
        return hp_fail(HP_ERR_ARG, "mesh pointers are null");
    if (m->num_triangles >= (int64_t(1) << 29))
        return hp_fail(HP_ERR_ARG, "mesh too large: at most 2^29 - 1 triangles per BVH");
    return HP_OK;
}

hp_status check_params(const hp_build_params* p) {
    if (!p) return hp_fail(HP_ERR_ARG, "build params are null");
    if (p->morton_bits < 6 || p->morton_bits > 60) return hp_fail(HP_ERR_ARG, "morton_bits must be in [6,60]");
    if (p->ct <= 0.0f || p->ci <= 0.0f) return hp_fail(HP_ERR_ARG, "ct and ci must be positive");
    if (p->max_leaf_size <= 0 || p->max_leaf_size > 1024) return hp_fail(HP_ERR_ARG, "max_leaf_size must be in (0,1024]");
    if (p->method == HP_METHOD_PLOC) {
        if (p->ploc_max_radius < 1) return hp_fail(HP_ERR_ARG, "ploc_max_radius must be positive");
        if (p->ploc_radius < 1 || p->ploc_radius > p->ploc_max_radius)
            return hp_fail(HP_ERR_ARG, "ploc_radius must be in [1, ploc_max_radius]");
    } else if (p->method == HP_METHOD_ATR) {
        if (p->atr_iterations < 0 || p->atr_iterations > 25) return hp_fail(HP_ERR_ARG, "atr_iterations must be in [0,25]");
        if (p->atr_treelet < 4 || p->atr_treelet > 30) return hp_fail(HP_ERR_ARG, "atr_treelet must be in [4,30]");
    } else if (p->method == HP_METHOD_TR) {
        if (p->atr_iterations < 0 || p->atr_iterations > 25) return hp_fail(HP_ERR_ARG, "iterations must be in [0,25]");
    } else if (p->method == HP_METHOD_HLBVH) {
        // HLBVHBuilder::setMortonCodeSAHBits (rt/bvh/HLBVHBuilder.cpp:431-435) takes [6,15] up to the Morton
        // bits; only multiples of 3 give every axis whole bins, so the others are not supported.
        if (p->hlbvh_sah_bits < 6 || p->hlbvh_sah_bits > 15 || p->hlbvh_sah_bits > p->morton_bits)
            return hp_fail(HP_ERR_ARG, "hlbvh_sah_bits must be in [6,15] and at most morton_bits");
        if (p->hlbvh_sah_bits % 3 != 0)
            return hp_fail(HP_ERR_UNSUPPORTED, "hlbvh_sah_bits must be a multiple of 3 (6, 9, 12 or 15)");
    } else if (p->method != HP_METHOD_LBVH) {
        return hp_fail(HP_ERR_ARG, "unknown build method");
    }
    if (p->layout != 0 && p->layout != HP_LAYOUT_BIN && p->layout != HP_LAYOUT_QUAD && p->layout != HP_LAYOUT_OCT)
        return hp_fail(HP_ERR_ARG, "layout must be 2 (bin), 4 (quad) or 8 (oct)");
    return HP_OK;
}

// Nodes of a tree over n references: at most 2n - 1 (3 for a single reference).
hp_status bvh_alloc(hp_bvh* out, int64_t n, int layout) {
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(out->impl);
    const size_t node_bytes = 32 * (size_t)layout;
    const size_t need_nodes = (size_t)std::max<int64_t>(2 * std::max<int64_t>(n, 2) - 1, 3) * node_bytes;
    if (b && b->capacity >= n && b->nodes && b->node_capacity >= need_nodes) return HP_OK;
    if (b) {
        cudaFree(b->nodes);
        cudaFree(b->woop);
        cudaFree(b->tri_idx);
        cudaFree(b->counters);
        cudaFree(b->info);
    } else {
        b = new hp_bvh_impl();
        out->impl = b;
    }
    *b = hp_bvh_impl();
    const int64_t cap = std::max<int64_t>(n, 2);
    const int64_t max_nodes = std::max<int64_t>(2 * cap - 1, 3);
    const size_t node_cap = (size_t)max_nodes * std::max<size_t>(node_bytes, sizeof(hp_node_bin));
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&b->nodes, node_cap);
    if (e == cudaSuccess) e = cudaMalloc(&b->woop, 3 * cap * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&b->tri_idx, cap * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->counters, cap * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->info, sizeof(hp_bvh_info));
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(b->nodes); cudaFree(b->woop); cudaFree(b->tri_idx); cudaFree(b->counters); cudaFree(b->info);
        *b = hp_bvh_impl();
        return hp_fail(HP_ERR_OOM, "BVH allocation failed for " + std::to_string(n) + " references");
    }
    HP_CUDA(cudaMemset(b->info, 0, sizeof(hp_bvh_info)));
    b->capacity = cap;
    b->node_capacity = node_cap;
    out->nodes = b->nodes;
    out->woop = b->woop;
    out->tri_indices = b->tri_idx;
    out->capacity_refs = cap;
    return HP_OK;
}

float ord2f_host(uint32_t u) {
    uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    std::memcpy(&f, &v, 4);
    return f;
}

uint32_t f2ord_host(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

}  // namespace

bool hp_checking(const hp_ctx* ctx, cudaStream_t s) {
    if (!ctx->checked) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return false;
    return cs == cudaStreamCaptureStatusNone;
}

namespace {

// Checked mode after a build or refit: the device error words, the node counts
// against the reference count, and the HipBVH::validate invariants
// (rt/bvh/HipBVH.cpp:157-307) over the whole tree.
hp_status checked_bvh(hp_ctx* ctx, hp_bvh* bvh, const hp_mesh* m, cudaStream_t s, const char* who) {
    HP_TRY(hp_bvh_sync(ctx, bvh, s));
    const int64_t n = bvh->num_refs;
    const int64_t ni = bvh->num_interior, nl = bvh->num_leaf;
    if (ni < 0 || nl < 1 || nl > std::max<int64_t>(n, 2) || ni + nl > 2 * n + 1)
        return hp_fail(HP_ERR_DEVICE_STATUS, std::string("checked mode: ") + who + " produced " +
                                                 std::to_string(ni) + " interior nodes and " + std::to_string(nl) +
                                                 " leaves for " + std::to_string(n) + " references");
    int32_t valid = 0;
    HP_TRY(hp_bvh_validate(ctx, bvh, m, &valid, s));
    if (!valid)
        return hp_fail(HP_ERR_DEVICE_STATUS, std::string("checked mode: ") + who +
                                                 " produced a BVH that fails validation");
    return HP_OK;
}

}  // namespace

extern "C" {

const char* hp_last_error(void) { return g_last_error.c_str(); }
int32_t hp_abi_version(void) { return HP_ABI_VERSION; }
int64_t hp_launch_count(void) { return g_launches; }

hp_status hp_profile_enable(hp_ctx* ctx, int32_t on) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_profile_enable: null context");
    ctx->profiling = on != 0;
    return HP_OK;
}

hp_status hp_profile_reset(hp_ctx* ctx) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_profile_reset: null context");
    ctx->num_marks = 0;
    return HP_OK;
}

int32_t hp_profile_count(hp_ctx* ctx) { return ctx ? ctx->num_marks : 0; }

// Phase i (>= 1) is the interval from mark i-1 to mark i, named after mark i.
hp_status hp_profile_get(hp_ctx* ctx, int32_t i, char* name, int64_t name_size, float* ms) {
    if (!ctx || i < 1 || i >= ctx->num_marks) return hp_fail(HP_ERR_ARG, "hp_profile_get: bad index");
    HP_CUDA(cudaEventSynchronize(ctx->marks[i].ev));
    float t = 0.0f;
    HP_CUDA(cudaEventElapsedTime(&t, ctx->marks[i - 1].ev, ctx->marks[i].ev));
    if (ms) *ms = t;
    if (name && name_size > 0) std::snprintf(name, (size_t)name_size, "%s", ctx->marks[i].name);
    return HP_OK;
}

hp_status hp_ctx_set_checked(hp_ctx* ctx, int32_t on) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_ctx_set_checked: null context");
    ctx->checked = on != 0;
    return HP_OK;
}

int32_t hp_ctx_get_checked(const hp_ctx* ctx) { return ctx && ctx->checked ? 1 : 0; }

hp_status hp_ctx_create(hp_ctx** out, int32_t device) {
    if (!out) return hp_fail(HP_ERR_ARG, "hp_ctx_create: null output");
    *out = nullptr;
    int count = 0;
    HP_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return hp_fail(HP_ERR_ARG, "hp_ctx_create: no such device");
    HP_CUDA(cudaSetDevice(device));
    hp_ctx* c = new hp_ctx();
    c->device = device;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) { delete c; return hp_cuda_fail(e, "cudaGetDeviceProperties"); }
    c->sm_count = prop.multiProcessorCount;
    c->l2_bytes = prop.l2CacheSize;
    if (const char* chk = std::getenv("HP_CHECKED")) c->checked = chk[0] != '\0' && chk[0] != '0';
    e = cudaMalloc(&c->d_status, 64 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->d_status, 0, 64 * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_status, 64 * sizeof(int));
    if (e != cudaSuccess) {
        cudaFree(c->d_status);
        delete c;
        return hp_cuda_fail(e, "hp_ctx_create");
    }
    *out = c;
    return HP_OK;
}

hp_status hp_ctx_destroy(hp_ctx* ctx) {
    if (!ctx) return HP_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    cudaFree(ctx->arena);
    cudaFree(ctx->d_status);
    cudaFreeHost(ctx->h_status);
    for (int i = 0; i < ctx->cap_marks; ++i) cudaEventDestroy(ctx->marks[i].ev);
    delete[] ctx->marks;
    for (int i = 0; i < 2; ++i) {
        cudaFree(ctx->io_slot[i]);
        if (ctx->io_up[i]) cudaEventDestroy(ctx->io_up[i]);
        if (ctx->io_traced[i]) cudaEventDestroy(ctx->io_traced[i]);
        if (ctx->io_free[i]) cudaEventDestroy(ctx->io_free[i]);
    }
    if (ctx->io_h2d) cudaStreamDestroy(ctx->io_h2d);
    if (ctx->io_d2h) cudaStreamDestroy(ctx->io_d2h);
    for (int i = 0; i < 2; ++i)
        if (ctx->io_trace[i]) cudaStreamDestroy(ctx->io_trace[i]);
    if (ctx->io_start) cudaEventDestroy(ctx->io_start);
    delete ctx;
    return HP_OK;
}

hp_status hp_ctx_check(hp_ctx* ctx, void* stream) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_ctx_check: null context");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    HP_CUDA(cudaMemcpyAsync(ctx->h_status, ctx->d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    if (ctx->h_status[0] != 0) {
        int code = ctx->h_status[0], info = ctx->h_status[1];
        HP_CUDA(cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(int), s));
        HP_CUDA(cudaStreamSynchronize(s));
        const char* what = code == HP_DEV_SPIN_LIMIT ? "bounded wait gave up"
                         : code == HP_DEV_BAD_INDEX ? "index out of range"
                         : code == HP_DEV_STACK_OVERFLOW ? "traversal stack overflow"
                         : code == HP_DEV_BAD_INPUT ? "invalid input (vertex index out of range)"
                         : code == HP_DEV_CHECK_FAILED ? "checked mode: output failed its verification"
                                                    : "device error";
        return hp_fail(HP_ERR_DEVICE_STATUS, std::string("kernel reported: ") + what + " (info " +
                                                 std::to_string(info) + ")");
    }
    return HP_OK;
}

void hp_build_params_default(hp_build_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->method = HP_METHOD_LBVH;
    p->morton_bits = 60;
    p->ploc_radius = 1;
    p->ploc_max_radius = 512;
    p->ploc_adaptive = 0;
    p->atr_iterations = 2;
    p->atr_treelet = 20;
    p->ct = 3.0f;
    p->ci = 2.0f;
    p->max_leaf_size = 8;
    p->adaptive_leaf = 1;
    p->layout = HP_LAYOUT_BIN;
    p->hlbvh_sah_bits = 15;
}

hp_status hp_build(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, hp_bvh* out,
                   const hp_build_taps* taps, void* stream) {
    hp_nvtx_range nvtx_("hp_build");
    if (!ctx || !out) return hp_fail(HP_ERR_ARG, "hp_build: null argument");
    HP_TRY(check_mesh(m));
    HP_TRY(check_params(p));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t n = m->num_triangles;
    if (out->impl && reinterpret_cast<hp_bvh_impl*>(out->impl)->view)
        return hp_fail(HP_ERR_ARG, "hp_build: the output is a view into a batch");
    const int layout = hp_layout_of(p);
    HP_TRY(bvh_alloc(out, n, layout));
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(out->impl);
    b->layout = layout;
    out->layout = layout;
    out->node_bytes = 32 * layout;
    out->num_refs = n;
    out->method = p->method;
    out->ct = p->ct;
    out->ci = p->ci;
    out->num_interior = out->num_leaf = -1;
    if (n == 0) {
        HP_CUDA(cudaMemsetAsync(b->info, 0, sizeof(hp_bvh_info), s));
        return HP_OK;
    }
    hp_mark(ctx, s, "begin");
    HP_TRY(hp_lbvh_build(ctx, m, p, b, taps, s));
    if (ctx->arith == HP_ARITH_REFERENCE) HP_TRY(hp_woop_ref_launch(ctx, b, n, m, s));
    if (hp_checking(ctx, s)) HP_TRY(checked_bvh(ctx, out, m, s, "hp_build"));
    return HP_OK;
}

hp_status hp_bvh_reserve(hp_ctx* ctx, hp_bvh* out, int64_t num_refs, int32_t layout) {
    if (!ctx || !out) return hp_fail(HP_ERR_ARG, "hp_bvh_reserve: null argument");
    if (num_refs < 0 || num_refs >= (int64_t(1) << 30)) return hp_fail(HP_ERR_ARG, "hp_bvh_reserve: num_refs out of range");
    if (layout == 0) layout = HP_LAYOUT_BIN;
    if (layout != HP_LAYOUT_BIN && layout != HP_LAYOUT_QUAD && layout != HP_LAYOUT_OCT)
        return hp_fail(HP_ERR_ARG, "hp_bvh_reserve: layout must be 2, 4 or 8");
    if (out->impl && reinterpret_cast<hp_bvh_impl*>(out->impl)->view)
        return hp_fail(HP_ERR_ARG, "hp_bvh_reserve: the output is a view into a batch");
    HP_TRY(bvh_alloc(out, num_refs, layout));
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(out->impl);
    b->layout = layout;
    out->layout = layout;
    out->node_bytes = 32 * layout;
    out->num_refs = num_refs;
    out->num_interior = out->num_leaf = -1;
    return HP_OK;
}

hp_status hp_bvh_set_info(hp_ctx* ctx, hp_bvh* bvh, int32_t num_interior, int32_t num_leaf,
                          const float* scene_box6, const float* morton_scale3, void* stream) {
    if (!ctx || !bvh || !bvh->impl || !scene_box6 || !morton_scale3)
        return hp_fail(HP_ERR_ARG, "hp_bvh_set_info: null argument");
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(bvh->impl);
    const int64_t max_nodes = std::max<int64_t>(2 * std::max<int64_t>(bvh->num_refs, 2) - 1, 3);
    if (num_interior < 0 || num_leaf < 0 || (int64_t)num_interior + num_leaf > max_nodes)
        return hp_fail(HP_ERR_ARG, "hp_bvh_set_info: node counts do not fit the BVH");
    hp_bvh_info info{};
    info.num_interior = num_interior;
    info.num_leaf = num_leaf;
    for (int k = 0; k < 6; ++k) info.box_ord[k] = f2ord_host(scene_box6[k]);
    for (int k = 0; k < 3; ++k) info.scale[k] = morton_scale3[k];
    // pageable source: the call returns once the 48 bytes are staged
    HP_CUDA(cudaMemcpyAsync(b->info, &info, sizeof(info), cudaMemcpyHostToDevice,
                            reinterpret_cast<cudaStream_t>(stream)));
    bvh->num_interior = num_interior;
    bvh->num_leaf = num_leaf;
    for (int k = 0; k < 6; ++k) bvh->scene_box[k] = scene_box6[k];
    for (int k = 0; k < 3; ++k) bvh->morton_scale[k] = morton_scale3[k];
    return HP_OK;
}

hp_status hp_bvh_sync(hp_ctx* ctx, hp_bvh* bvh, void* stream) {
    if (!ctx || !bvh || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_bvh_sync: null argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(bvh->impl);
    hp_bvh_info info;
    HP_CUDA(cudaMemcpyAsync(&info, b->info, sizeof(info), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    HP_TRY(hp_ctx_check(ctx, stream));
    bvh->num_interior = info.num_interior;
    bvh->num_leaf = info.num_leaf;
    for (int k = 0; k < 6; ++k) bvh->scene_box[k] = ord2f_host(info.box_ord[k]);
    for (int k = 0; k < 3; ++k) bvh->morton_scale[k] = info.scale[k];
    return HP_OK;
}

hp_status hp_bvh_download(hp_ctx* ctx, hp_bvh* bvh, void* nodes_host, void* woop_host, int32_t* tri_host,
                          void* stream) {
    HP_TRY(hp_bvh_sync(ctx, bvh, stream));
    const int64_t count = (int64_t)bvh->num_interior + bvh->num_leaf;
    const int64_t n = bvh->num_refs;
    if (nodes_host && count > 0)
        HP_CUDA(cudaMemcpy(nodes_host, bvh->nodes, count * (size_t)(bvh->node_bytes > 0 ? bvh->node_bytes : 64),
                           cudaMemcpyDeviceToHost));
    if (woop_host && n > 0)
        HP_CUDA(cudaMemcpy(woop_host, bvh->woop, n * 3 * sizeof(float4), cudaMemcpyDeviceToHost));
    if (tri_host && n > 0)
        HP_CUDA(cudaMemcpy(tri_host, bvh->tri_indices, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return HP_OK;
}

hp_status hp_bvh_free(hp_ctx* ctx, hp_bvh* bvh) {
    (void)ctx;
    if (!bvh) return HP_OK;
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(bvh->impl);
    if (b && b->view) {  // a view into a batch: the batch owns the storage
        std::memset(bvh, 0, sizeof(*bvh));
        return HP_OK;
    }
    if (b) {
        cudaFree(b->nodes);
        cudaFree(b->woop);
        cudaFree(b->tri_idx);
        cudaFree(b->counters);
        cudaFree(b->info);
        delete b;
    }
    std::memset(bvh, 0, sizeof(*bvh));
    return HP_OK;
}

// HipBVH::getCost (rt/bvh/HipBVH.cpp:346-370) on the device (k_stats.cu).
hp_status hp_bvh_cost(hp_ctx* ctx, const hp_bvh* bvh, double* cost, void* stream) {
    if (!ctx || !bvh || !cost || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_bvh_cost: null argument");
    hp_bvh_stats st;
    HP_TRY(hp_bvh_stats_run(ctx, bvh, &st, reinterpret_cast<cudaStream_t>(stream)));
    *cost = st.sah_cost;
    return HP_OK;
}

// getCost, getAvgLeafSize and getLeafSizeHistogram (rt/bvh/HipBVH.cpp:346-442).
hp_status hp_bvh_stats_get(hp_ctx* ctx, const hp_bvh* bvh, hp_bvh_stats* out, void* stream) {
    if (!ctx || !bvh || !out || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_bvh_stats_get: null argument");
    return hp_bvh_stats_run(ctx, bvh, out, reinterpret_cast<cudaStream_t>(stream));
}

// HipBVH::validate (rt/bvh/HipBVH.cpp:157-307) on the device (k_stats.cu).
hp_status hp_bvh_validate(hp_ctx* ctx, const hp_bvh* bvh, const hp_mesh* m, int32_t* valid, void* stream) {
    hp_nvtx_range nvtx_("hp_bvh_validate");
    if (!ctx || !bvh || !valid || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_bvh_validate: null argument");
    HP_TRY(check_mesh(m));
    *valid = 0;
    if (bvh->num_refs != m->num_triangles) return hp_fail(HP_ERR_ARG, "hp_bvh_validate: mesh does not match the BVH");
    if (bvh->num_refs == 0) {
        hp_bvh tmp = *bvh;
        HP_TRY(hp_bvh_sync(ctx, &tmp, stream));
        *valid = (tmp.num_interior + tmp.num_leaf) == 0;
        return HP_OK;
    }
    return hp_bvh_validate_run(ctx, bvh, m, valid, reinterpret_cast<cudaStream_t>(stream));
}

hp_status hp_refit(hp_ctx* ctx, hp_bvh* bvh, const hp_mesh* m, void* stream) {
    hp_nvtx_range nvtx_("hp_refit");
    if (!ctx || !bvh || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_refit: null argument");
    HP_TRY(check_mesh(m));
    if (m->num_triangles != bvh->num_refs) return hp_fail(HP_ERR_ARG, "hp_refit: mesh does not match the BVH");
    if (reinterpret_cast<hp_bvh_impl*>(bvh->impl)->view)
        return hp_fail(HP_ERR_UNSUPPORTED, "hp_refit: a BVH of a batch is rebuilt with hp_batch_build");
    if (reinterpret_cast<hp_bvh_impl*>(bvh->impl)->layout != HP_LAYOUT_BIN)
        return hp_fail(HP_ERR_UNSUPPORTED, "hp_refit: only the binary layout is refitted in place (rebuild wide BVHs)");
    hp_bvh_impl* b = reinterpret_cast<hp_bvh_impl*>(bvh->impl);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    HP_TRY(hp_refit_launch(ctx, b, bvh->num_refs, m, s));
    if (ctx->arith == HP_ARITH_REFERENCE) HP_TRY(hp_woop_ref_launch(ctx, b, bvh->num_refs, m, s));
    if (hp_checking(ctx, s)) HP_TRY(checked_bvh(ctx, bvh, m, s, "hp_refit"));
    return HP_OK;
}

hp_status hp_trace(hp_ctx* ctx, const hp_bvh* bvh, const float* rays, int64_t num_rays, int32_t* results,
                   int32_t* stats, uint32_t flags, void* stream) {
    if (!ctx || !bvh || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_trace: null argument");
    if (num_rays < 0) return hp_fail(HP_ERR_ARG, "hp_trace: negative ray count");
    if (num_rays > 0 && (!rays || !results)) return hp_fail(HP_ERR_ARG, "hp_trace: null ray or result buffer");
    hp_nvtx_range nvtx_("hp_trace");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // A context tuned for it traces large batches in ray Morton order (same results).
    if (ctx->tune.trace_sorted && num_rays >= 65536 && num_rays < (int64_t(1) << 30))
        HP_TRY(hp_trace_sorted(ctx, bvh, rays, num_rays, results, stats, flags, 30, nullptr, stream));
    else
        HP_TRY(hp_trace_launch(ctx, reinterpret_cast<const hp_bvh_impl*>(bvh->impl), bvh->num_refs, rays,
                               num_rays, results, stats, flags, s));
    // checked mode: a traversal stack overflow or an out-of-range node index
    // reported by the tracer comes back from this call
    if (hp_checking(ctx, s)) HP_TRY(hp_ctx_check(ctx, stream));
    return HP_OK;
}

hp_status hp_trace_host(hp_ctx* ctx, const hp_bvh* bvh, const float* rays_host, int64_t num_rays,
                        int32_t* results_host, int32_t* stats_host, uint32_t flags, int64_t chunk_rays,
                        void* stream) {
    if (!ctx || !bvh || !bvh->impl) return hp_fail(HP_ERR_ARG, "hp_trace_host: null argument");
    if (num_rays < 0 || chunk_rays < 0) return hp_fail(HP_ERR_ARG, "hp_trace_host: negative count");
    if (num_rays == 0) return HP_OK;
    if (!rays_host || !results_host) return hp_fail(HP_ERR_ARG, "hp_trace_host: null ray or result buffer");
    hp_nvtx_range nvtx_("hp_trace_host");
    const int64_t C = std::min<int64_t>(chunk_rays > 0 ? chunk_rays : (int64_t(1) << 22), num_rays);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // A context tuned for sorted tracing sorts each chunk by 30-bit ray keys, as
    // hp_trace does for a batch of that size.
    const int sort_bits = 30;
    const bool sorted = ctx->tune.trace_sorted && C >= 65536 && C < (int64_t(1) << 30);
    // slot layout: rays (32 B per ray), results (16 B), stats (8 B), then, when
    // sorting, the order and the ray sort's keys and scratch
    const size_t ray_b = hp_carve::pad((size_t)C * 32), res_b = hp_carve::pad((size_t)C * 16);
    const size_t st_b = hp_carve::pad((size_t)C * 8);
    const size_t sort_b = sorted ? hp_carve::pad((size_t)C * 4) + hp_ray_order_scratch_bytes(C, sort_bits,
                                                                                              ctx->tune.sort_block)
                                 : 0;
    const size_t need = ray_b + res_b + st_b + sort_b;
    if (!ctx->io_h2d) {
        HP_CUDA(cudaStreamCreateWithFlags(&ctx->io_h2d, cudaStreamNonBlocking));
        HP_CUDA(cudaStreamCreateWithFlags(&ctx->io_d2h, cudaStreamNonBlocking));
        HP_CUDA(cudaEventCreateWithFlags(&ctx->io_start, cudaEventDisableTiming));
        for (int i = 0; i < 2; ++i) {
            HP_CUDA(cudaStreamCreateWithFlags(&ctx->io_trace[i], cudaStreamNonBlocking));
            HP_CUDA(cudaEventCreateWithFlags(&ctx->io_up[i], cudaEventDisableTiming));
            HP_CUDA(cudaEventCreateWithFlags(&ctx->io_traced[i], cudaEventDisableTiming));
            HP_CUDA(cudaEventCreateWithFlags(&ctx->io_free[i], cudaEventDisableTiming));
        }
    }
    if (ctx->io_slot_bytes < need) {
        // earlier calls may still use the slots (their traces end before their downloads)
        HP_CUDA(cudaStreamSynchronize(ctx->io_d2h));
        for (int i = 0; i < 2; ++i) {
            HP_CUDA(cudaFree(ctx->io_slot[i]));
            ctx->io_slot[i] = nullptr;
        }
        ctx->io_slot_bytes = 0;
        for (int i = 0; i < 2; ++i) HP_CUDA(cudaMalloc(&ctx->io_slot[i], need));
        ctx->io_slot_bytes = need;
    }
    // Work queued on the caller's stream (the build of this BVH) comes first.
    HP_CUDA(cudaEventRecord(ctx->io_start, s));
    for (int k = 0; k < 2; ++k) HP_CUDA(cudaStreamWaitEvent(ctx->io_trace[k], ctx->io_start, 0));
    const hp_bvh_impl* bi = reinterpret_cast<const hp_bvh_impl*>(bvh->impl);
    // Chunk sizes: chunk_rays each, or by default doubling from 262,144 rays up
    // to 4,194,304 and halving again at the end, so that the first upload and
    // the last download, which nothing overlaps, stay short.
    std::vector<int64_t> sizes;
    if (chunk_rays > 0) {
        for (int64_t off = 0; off < num_rays; off += C) sizes.push_back(std::min(C, num_rays - off));
    } else {
        const int64_t lo = std::min<int64_t>(C, 262144);
        int64_t left = num_rays;
        std::vector<int64_t> tail;
        for (int64_t a = lo; a < C && left > 4 * a; a *= 2) {
            sizes.push_back(a);
            tail.push_back(a);
            left -= 2 * a;
        }
        const int64_t mid = (left + C - 1) / C;
        for (int64_t j = 0; j < mid; ++j) sizes.push_back(left / mid + (j < left % mid ? 1 : 0));
        sizes.insert(sizes.end(), tail.rbegin(), tail.rend());
    }
    int64_t off = 0;
    for (size_t i = 0; i < sizes.size(); off += sizes[i], ++i) {
        // Chunks alternate between two slots, each traced on a stream of its own,
        // so that a chunk's trace starts on the SMs that the previous chunk's
        // trace leaves idle as it drains.
        const int k = (int)(i & 1);
        const int64_t m = sizes[i];
        cudaStream_t t = ctx->io_trace[k];
        hp_carve cv(ctx->io_slot[k]);
        float* d_rays = cv.take<float>((size_t)C * 8);
        int32_t* d_res = cv.take<int32_t>((size_t)C * 4);
        int32_t* d_stats = cv.take<int32_t>((size_t)C * 2);
        if (!stats_host) d_stats = nullptr;
        unsigned long long* counter = reinterpret_cast<unsigned long long*>(ctx->d_status + 20 + 2 * k);
        // up: once the slot's previous results are home
        HP_CUDA(cudaStreamWaitEvent(ctx->io_h2d, ctx->io_free[k], 0));
        HP_CUDA(cudaMemcpyAsync(d_rays, rays_host + 8 * off, (size_t)m * 32, cudaMemcpyHostToDevice, ctx->io_h2d));
        HP_CUDA(cudaEventRecord(ctx->io_up[k], ctx->io_h2d));
        // trace
        HP_CUDA(cudaStreamWaitEvent(t, ctx->io_up[k], 0));
        HP_CUDA(cudaMemsetAsync(d_res, 0, (size_t)m * 16, t));
        const int32_t* order = nullptr;
        if (sorted && m >= 65536) {
            int32_t* ord = cv.take<int32_t>((size_t)C);
            void* scratch = cv.take<char>(hp_ray_order_scratch_bytes(C, sort_bits, ctx->tune.sort_block));
            HP_TRY(hp_ray_order(ctx, d_rays, m, sort_bits, ord, scratch, t));
            order = ord;
        }
        HP_TRY(hp_trace_launch(ctx, bi, bvh->num_refs, d_rays, m, d_res, d_stats, flags, t, order, counter));
        HP_CUDA(cudaEventRecord(ctx->io_traced[k], t));
        // down
        HP_CUDA(cudaStreamWaitEvent(ctx->io_d2h, ctx->io_traced[k], 0));
        HP_CUDA(cudaMemcpyAsync(results_host + 4 * off, d_res, (size_t)m * 16, cudaMemcpyDeviceToHost, ctx->io_d2h));
        if (stats_host)
            HP_CUDA(cudaMemcpyAsync(stats_host + 2 * off, d_stats, (size_t)m * 8, cudaMemcpyDeviceToHost,
                                    ctx->io_d2h));
        HP_CUDA(cudaEventRecord(ctx->io_free[k], ctx->io_d2h));
    }
    // the caller's stream completes once every result is home
    for (int k = 0; k < 2; ++k) HP_CUDA(cudaStreamWaitEvent(s, ctx->io_free[k], 0));
    if (hp_checking(ctx, s)) HP_TRY(hp_ctx_check(ctx, stream));
    return HP_OK;
}

hp_status hp_trace_adjoint(hp_ctx* ctx, const hp_mesh* m, const float* rays, const int32_t* results,
                           const float* dl_dtuv, int64_t num_rays, float* dl_dvertices, void* stream) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_trace_adjoint: null context");
    HP_TRY(check_mesh(m));
    if (num_rays < 0) return hp_fail(HP_ERR_ARG, "hp_trace_adjoint: negative ray count");
    if (num_rays > 0 && (!rays || !results || !dl_dtuv || !dl_dvertices))
        return hp_fail(HP_ERR_ARG, "hp_trace_adjoint: null buffer");
    hp_nvtx_range nvtx_("hp_trace_adjoint");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    HP_TRY(hp_adjoint_launch(ctx, m, rays, results, dl_dtuv, num_rays, dl_dvertices, s));
    if (hp_checking(ctx, s)) HP_TRY(hp_ctx_check(ctx, stream));
    return HP_OK;
}

hp_status hp_radix_sort(hp_ctx* ctx, const void* keys_in, const int32_t* vals_in, void* keys_out,
                        int32_t* vals_out, int64_t n, int32_t key_bytes, int32_t bits, void* stream) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_radix_sort: null context");
    if (key_bytes != 4 && key_bytes != 8) return hp_fail(HP_ERR_ARG, "hp_radix_sort: key_bytes must be 4 or 8");
    if (bits < 1 || bits > 8 * key_bytes) return hp_fail(HP_ERR_ARG, "hp_radix_sort: bits out of range");
    if (n < 0 || n >= (int64_t(1) << 30)) return hp_fail(HP_ERR_ARG, "hp_radix_sort: n out of range");
    if (n == 0) return HP_OK;
    if (!keys_in || !keys_out || !vals_out) return hp_fail(HP_ERR_ARG, "hp_radix_sort: null buffer");
    hp_nvtx_range nvtx_("hp_radix_sort");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    hp_sort_plan plan = hp_sort_make_plan(n, key_bytes, bits, ctx->tune.sort_block);
    const size_t hist_bytes = hp_carve::pad(hp_sort_hist_bytes(plan.passes));
    HP_TRY(hp_ctx_reserve(ctx, hp_carve::pad(plan.scratch_bytes) + hist_bytes, s));
    hp_carve cv(ctx->arena);
    void* scratch = cv.take<char>(plan.scratch_bytes);
    uint32_t* hist = cv.take<uint32_t>(plan.passes * 256);
    hp_sort_args a{keys_in, vals_in, keys_out, vals_out, scratch, hist, false, ctx->d_status, ctx};
    HP_TRY(hp_sort_run(plan, a, s));
    if (hp_checking(ctx, s)) {
        HP_TRY(hp_sort_check_launch(ctx, keys_out, n, key_bytes, bits, s));
        HP_TRY(hp_ctx_check(ctx, stream));
    }
    return HP_OK;
}

hp_status hp_ctx_set_arithmetic(hp_ctx* ctx, int32_t mode) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_ctx_set_arithmetic: null context");
    if (mode != HP_ARITH_IEEE && mode != HP_ARITH_REFERENCE)
        return hp_fail(HP_ERR_ARG, "hp_ctx_set_arithmetic: mode must be HP_ARITH_IEEE or HP_ARITH_REFERENCE");
    ctx->arith = mode;
    return HP_OK;
}

hp_status hp_ctx_set_sort_spin_limit(hp_ctx* ctx, uint32_t spins) {
    if (!ctx) return hp_fail(HP_ERR_ARG, "hp_ctx_set_sort_spin_limit: null context");
    ctx->sort_spin_limit = spins ? spins : HP_SORT_SPIN_LIMIT_DEFAULT;
    return HP_OK;
}

}  // extern "C"
