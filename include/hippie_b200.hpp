/*
 * hippie_b200.hpp — C++ facade over the C ABI of include/hippie_b200.h.
 *
 * The classes keep the reference's names and semantics so that C++ host code
 * written against hippie's builder / BVH / tracer / environment reads the same
 * (meistdan/hippie, paths relative to src/hippie/):
 *   Environment   Environment / AppEnvironment     environment/Environment.cpp:290-466
 *   BVH           HipBVH (getCost, validate, update) rt/bvh/HipBVH.h:19-106
 *   Builder       BVHBuilder (build, rebuild, clear) rt/bvh/BVHBuilder.h:16-68
 *   Tracer        HipTracer (setBVH, trace, traceStats, traceSort)
 *                                                   rt/tracer/HipTracer.h:16-42
 * Scenes are device meshes (hp_mesh) instead of Scene objects. Times are
 * seconds of summed phase time on the GPU, as the reference's
 * HipKernel::launchTimed sums reported them. Errors throw hippie_b200::Error
 * (the reference logs and exits). Header only; link libhippie_b200.so.
 */
#ifndef HIPPIE_B200_HPP_
#define HIPPIE_B200_HPP_

#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "hippie_b200.h"

namespace hippie_b200 {

struct Error : std::runtime_error {
    hp_status status;
    Error(hp_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(hp_status s, const char* what) {
    if (s != HP_OK) throw Error(s, std::string(what) + ": " + hp_last_error());
}

class Context {
public:
    explicit Context(int device = 0) { check(hp_ctx_create(&h_, device), "hp_ctx_create"); }
    ~Context() { hp_ctx_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    hp_ctx* get() const { return h_; }
    /* Wait for the device; throws if a kernel reported an error. */
    void synchronize(void* stream = nullptr) const { check(hp_ctx_check(h_, stream), "hp_ctx_check"); }

    /* Seconds of GPU time between the first and last phase mark of f(). */
    template <typename F>
    float timed(F f, void* stream = nullptr) const {
        check(hp_profile_reset(h_), "hp_profile_reset");
        check(hp_profile_enable(h_, 1), "hp_profile_enable");
        f();
        float total = 0.0f, ms = 0.0f;
        const int n = hp_profile_count(h_);
        for (int i = 1; i < n; ++i) {
            check(hp_profile_get(h_, i, nullptr, 0, &ms), "hp_profile_get");
            total += ms;
        }
        hp_profile_enable(h_, 0);
        hp_profile_reset(h_);
        synchronize(stream);
        return total * 1.0e-3f;
    }

private:
    hp_ctx* h_ = nullptr;
};

/* Environment file with the reference's keys, parse rules and defaults. */
class Environment {
public:
    Environment() { check(hp_env_create(&h_), "hp_env_create"); }
    ~Environment() { hp_env_destroy(h_); }
    Environment(const Environment&) = delete;
    Environment& operator=(const Environment&) = delete;
    void readFile(const std::string& path) { check(hp_env_read_file(h_, path.c_str()), "hp_env_read_file"); }
    void readString(const std::string& text) { check(hp_env_read_string(h_, text.c_str()), "hp_env_read_string"); }
    int getInt(const char* name) const {
        int32_t v = 0;
        check(hp_env_get_int(h_, name, &v), name);
        return v;
    }
    float getFloat(const char* name) const {
        float v = 0.0f;
        check(hp_env_get_float(h_, name, &v), name);
        return v;
    }
    bool getBool(const char* name) const {
        int32_t v = 0;
        check(hp_env_get_bool(h_, name, &v), name);
        return v != 0;
    }
    std::string getString(const char* name) const {
        char buf[4096];
        check(hp_env_get_string(h_, name, buf, sizeof(buf)), name);
        return buf;
    }
    /* A three-component option ("x y z"). */
    void getVector(const char* name, float out[3]) const {
        std::istringstream is(getString(name));
        if (!(is >> out[0] >> out[1] >> out[2])) throw Error(HP_ERR_PARSE, std::string("not a vector: ") + name);
    }
    hp_build_params buildParams() const {
        hp_build_params p;
        check(hp_env_build_params(h_, &p), "hp_env_build_params");
        return p;
    }
    const hp_env* get() const { return h_; }

private:
    hp_env* h_ = nullptr;
};

class BVH {
public:
    explicit BVH(Context& c) : ctx_(c) { std::memset(&b_, 0, sizeof(b_)); }
    ~BVH() { hp_bvh_free(ctx_.get(), &b_); }
    BVH(const BVH&) = delete;
    BVH& operator=(const BVH&) = delete;
    hp_bvh* get() { return &b_; }
    const hp_bvh* get() const { return &b_; }
    /* Node counts and scene box (synchronises). */
    void sync(void* stream = nullptr) { check(hp_bvh_sync(ctx_.get(), &b_, stream), "hp_bvh_sync"); }
    int getNumberOfNodes() {
        sync();
        return b_.num_interior + b_.num_leaf;
    }
    /* HipBVH::getCost: SAH cost of the collapsed tree. */
    double getCost(void* stream = nullptr) const {
        double c = 0.0;
        check(hp_bvh_cost(ctx_.get(), &b_, &c, stream), "hp_bvh_cost");
        return c;
    }
    /* HipBVH::getAvgLeafSize. */
    float getAvgLeafSize(void* stream = nullptr) const { return (float)stats(stream).avg_leaf_size; }
    /* HipBVH::getLeafSizeHistogram: fraction of leaves of each size 0..32. */
    std::vector<float> getLeafSizeHistogram(void* stream = nullptr) const {
        const hp_bvh_stats st = stats(stream);
        return std::vector<float>(st.leaf_size_histogram, st.leaf_size_histogram + HP_MAX_LEAF_SIZE_HIST + 1);
    }
    /* All of the above in one device pass. */
    hp_bvh_stats stats(void* stream = nullptr) const {
        hp_bvh_stats st;
        check(hp_bvh_stats_get(ctx_.get(), &b_, &st, stream), "hp_bvh_stats_get");
        return st;
    }
    /* HipBVH::validate. */
    bool validate(const hp_mesh& m, void* stream = nullptr) const {
        int32_t ok = 0;
        check(hp_bvh_validate(ctx_.get(), &b_, &m, &ok, stream), "hp_bvh_validate");
        return ok != 0;
    }
    /* HipBVH::update: refit after vertex moves (same topology). */
    void update(const hp_mesh& m, void* stream = nullptr) { check(hp_refit(ctx_.get(), &b_, &m, stream), "hp_refit"); }

private:
    Context& ctx_;
    hp_bvh b_;
};

/* BVHBuilder: LBVH, PLOC or ATR according to the build parameters. */
class Builder {
public:
    Builder(Context& c, const hp_build_params& p) : ctx_(c), p_(p) {}
    static Builder fromEnvironment(Context& c, const Environment& env) { return Builder(c, env.buildParams()); }
    BVH* build(const hp_mesh& m) {
        float t = 0.0f;
        return build(m, t);
    }
    BVH* build(const hp_mesh& m, float& seconds) {
        BVH* b = new BVH(ctx_);
        try {
            seconds = rebuild(*b, m);
        } catch (...) {
            delete b;
            throw;
        }
        return b;
    }
    /* Build into an existing BVH; returns seconds of build time on the GPU. */
    float rebuild(BVH& bvh, const hp_mesh& m, void* stream = nullptr) {
        return ctx_.timed([&] { check(hp_build(ctx_.get(), &m, &p_, bvh.get(), nullptr, stream), "hp_build"); },
                          stream);
    }
    void clear() {}  // scratch belongs to the context and is reused
    hp_build_params& params() { return p_; }

private:
    Context& ctx_;
    hp_build_params p_;
};

/* HipTracer: rays are 8 floats ({origin, tmin, direction, tmax}), results 4
 * int32 ({triangle, t, u, v}), stats 2 int32; all device pointers. */
class Tracer {
public:
    explicit Tracer(Context& c) : ctx_(c) {}
    void setBVH(BVH* b) { bvh_ = b; }
    BVH* getBVH() { return bvh_; }
    float trace(const float* rays, int64_t n, int32_t* results, bool anyHit = false, void* stream = nullptr) {
        return run(rays, n, results, nullptr, anyHit ? HP_TRACE_ANY_HIT : 0u, false, stream);
    }
    float traceStats(const float* rays, int64_t n, int32_t* results, int32_t* stats, void* stream = nullptr) {
        return run(rays, n, results, stats, HP_TRACE_STATS, false, stream);
    }
    float traceSort(const float* rays, int64_t n, int32_t* results, void* stream = nullptr) {
        return run(rays, n, results, nullptr, 0u, true, stream);
    }
    /* A RayBuffer in host memory: rays and results on the host (pinned for
     * overlap), uploaded, traced and downloaded in overlapping chunks. */
    float traceHost(const float* rays_host, int64_t n, int32_t* results_host, bool anyHit = false,
                    void* stream = nullptr) {
        if (!bvh_) throw Error(HP_ERR_ARG, "Tracer: no BVH set");
        return ctx_.timed(
            [&] {
                check(hp_trace_host(ctx_.get(), bvh_->get(), rays_host, n, results_host, nullptr,
                                    anyHit ? HP_TRACE_ANY_HIT : 0u, 0, stream),
                      "hp_trace_host");
            },
            stream);
    }
    /* RayBuffer::setMortonCodeMethod / setRayLength for traceSort, by the
     * renderer's method names ("aila", "paraboloid", ..., "reise"). */
    void setMortonCodeMethod(const char* name, float rayLength = 0.25f) {
        check(hp_ctx_set_ray_keys(ctx_.get(), hp_ray_keys_method(name), rayLength), "hp_ctx_set_ray_keys");
    }

private:
    float run(const float* rays, int64_t n, int32_t* results, int32_t* stats, uint32_t flags, bool sorted,
              void* stream) {
        if (!bvh_) throw Error(HP_ERR_ARG, "Tracer: no BVH set");
        return ctx_.timed(
            [&] {
                if (sorted)
                    check(hp_trace_sorted(ctx_.get(), bvh_->get(), rays, n, results, stats, flags, 30, nullptr,
                                          stream),
                          "hp_trace_sorted");
                else
                    check(hp_trace(ctx_.get(), bvh_->get(), rays, n, results, stats, flags, stream), "hp_trace");
            },
            stream);
    }
    Context& ctx_;
    BVH* bvh_ = nullptr;
};

}  // namespace hippie_b200

#endif /* HIPPIE_B200_HPP_ */
