// Launch-choice tuning of a context (hp_tune / hp_autotune).
//
// The result-neutral choices (sort CTA size, tracer CTAs per SM, shared-memory
// stack depth, Morton-ordered tracing) are timed with CUDA events on the
// caller's own mesh and rays and applied to the context; the PLOC radius
// schedule, which changes the tree, is compared by build time plus the trace
// time it buys and only reported.
#include <algorithm>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "hp_internal.h"

namespace {

bool tune_valid(const hp_tune& t) {
    return (t.sort_block == 256 || t.sort_block == 512) && t.trace_ctas_per_sm >= 0 && t.trace_ctas_per_sm <= 64 &&
           (t.trace_stack == 8 || t.trace_stack == 16 || t.trace_stack == 32) &&
           (t.trace_sorted == 0 || t.trace_sorted == 1);
}

// Median of three timed runs of f (after one untimed run), in milliseconds.
template <typename F>
hp_status time_ms(cudaStream_t s, F f, float* ms) {
    cudaEvent_t a, b;
    HP_CUDA(cudaEventCreate(&a));
    HP_CUDA(cudaEventCreate(&b));
    hp_status st = f();
    float t[3] = {0, 0, 0};
    for (int k = 0; k < 3 && st == HP_OK; ++k) {
        cudaEventRecord(a, s);
        st = f();
        cudaEventRecord(b, s);
        if (cudaEventSynchronize(b) != cudaSuccess) st = hp_fail(HP_ERR_CUDA, "hp_autotune: timing failed");
        else cudaEventElapsedTime(&t[k], a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::sort(t, t + 3);
    *ms = t[1];
    return st;
}

}  // namespace

extern "C" void hp_tune_default(hp_tune* t) {
    if (!t) return;
    std::memset(t, 0, sizeof(*t));
    t->sort_block = 512;
    t->trace_ctas_per_sm = 0;
    t->trace_stack = 16;
    t->trace_sorted = 0;
}

extern "C" hp_status hp_ctx_set_tune(hp_ctx* ctx, const hp_tune* t) {
    if (!ctx || !t) return hp_fail(HP_ERR_ARG, "hp_ctx_set_tune: null argument");
    if (!tune_valid(*t)) return hp_fail(HP_ERR_ARG, "hp_ctx_set_tune: a setting is out of range");
    ctx->tune = *t;
    return HP_OK;
}

extern "C" hp_status hp_ctx_get_tune(hp_ctx* ctx, hp_tune* t) {
    if (!ctx || !t) return hp_fail(HP_ERR_ARG, "hp_ctx_get_tune: null argument");
    *t = ctx->tune;
    return HP_OK;
}

extern "C" hp_status hp_autotune(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, const float* rays,
                                 int64_t num_rays, uint32_t flags, hp_tune* out, void* stream) {
    if (!ctx || !m || !p || !out || num_rays < 0 || (num_rays > 0 && !rays))
        return hp_fail(HP_ERR_ARG, "hp_autotune: bad argument");
    if (m->num_triangles < 2) return hp_fail(HP_ERR_ARG, "hp_autotune: needs a mesh of at least two triangles");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const hp_tune saved = ctx->tune;
    hp_tune best;
    hp_tune_default(&best);
    best.trace_ctas_per_sm = saved.trace_ctas_per_sm;
    const int64_t sample = std::min<int64_t>(num_rays, int64_t(1) << 21);
    hp_bvh bvh;
    std::memset(&bvh, 0, sizeof(bvh));
    int32_t* results = nullptr;
    if (sample > 0 && cudaMalloc(&results, sample * 16) != cudaSuccess) {
        cudaGetLastError();
        return hp_fail(HP_ERR_OOM, "hp_autotune: cannot allocate the result buffer");
    }
    hp_status st = HP_OK;
    auto build = [&]() { return hp_build(ctx, m, p, &bvh, nullptr, stream); };
    auto trace = [&]() { return hp_trace(ctx, &bvh, rays, sample, results, nullptr, 0, stream); };
    // 1. sort CTA size, on the build
    float bms = 0.0f, b_best = 1e30f;
    for (int blk : {512, 256}) {
        if (st != HP_OK) break;
        ctx->tune = best;
        ctx->tune.sort_block = blk;
        st = time_ms(s, build, &bms);
        if (st == HP_OK && bms < b_best) { b_best = bms; best.sort_block = blk; }
    }
    // 2. trace launch choices, on the ray sample
    float t_best = 0.0f;
    if (st == HP_OK && sample > 0) {
        ctx->tune = best;
        st = build();
        t_best = 1e30f;
        int per_sm_max = 12;
        hp_tune base = best;
        for (int sorted : {0, 1})
            for (int stack : {8, 16, 32})
                for (int ctas : {0, per_sm_max / 2, per_sm_max / 3}) {
                    if (st != HP_OK) break;
                    hp_tune c = base;
                    c.trace_sorted = sorted;
                    c.trace_stack = stack;
                    c.trace_ctas_per_sm = ctas;
                    ctx->tune = c;
                    float tms = 0.0f;
                    st = time_ms(s, trace, &tms);
                    if (st == HP_OK && tms < t_best) {
                        t_best = tms;
                        best.trace_sorted = sorted;
                        best.trace_stack = stack;
                        best.trace_ctas_per_sm = ctas;
                    }
                }
    }
    best.build_ms = b_best;
    best.trace_ms = sample > 0 ? t_best : 0.0f;
    // 3. PLOC radius schedule (reported, not applied)
    if (st == HP_OK && (flags & HP_TUNE_PLOC_RADIUS) && p->method == HP_METHOD_PLOC) {
        struct sched { int r, adaptive, rmax; };
        const sched cand[] = {{8, 0, 8}, {16, 0, 16}, {32, 0, 32}, {4, 1, 64}};
        float total_best = 1e30f;
        for (const sched& c : cand) {
            if (st != HP_OK) break;
            hp_build_params q = *p;
            q.ploc_radius = c.r;
            q.ploc_adaptive = c.adaptive;
            q.ploc_max_radius = c.rmax;
            ctx->tune = best;
            float b_ms = 0.0f, tr_ms = 0.0f;
            auto bq = [&]() { return hp_build(ctx, m, &q, &bvh, nullptr, stream); };
            st = time_ms(s, bq, &b_ms);
            if (st == HP_OK && sample > 0) st = time_ms(s, trace, &tr_ms);
            const float total = b_ms + (sample > 0 ? tr_ms * (float)((double)num_rays / (double)sample) : 0.0f);
            if (st == HP_OK && total < total_best) {
                total_best = total;
                best.ploc_radius = c.r;
                best.ploc_adaptive = c.adaptive;
                best.ploc_max_radius = c.rmax;
            }
        }
    }
    if (st == HP_OK) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = hp_cuda_fail(e, "hp_autotune");
    }
    hp_bvh_free(ctx, &bvh);
    cudaFree(results);
    if (st != HP_OK) {
        ctx->tune = saved;
        return st;
    }
    ctx->tune = best;
    *out = best;
    return HP_OK;
}
