// hippie_b200_bench — the benchmark caller of the build-and-trace path in C++,
// driven by the reference's environment files (Benchmark::testStatic,
// src/hippie/benchmark/Benchmark.cpp:44-220, with its Bvh.*, Scene.filename,
// Resolution.*, Camera.* and Renderer.numberOfPrimarySamples options).
//
// For the scene it builds the BVH with the method of the env file (timed over
// --steps builds), then renders primary rays of the env file's camera, one
// Halton-jittered sample per Renderer.numberOfPrimarySamples, in pixel-table
// order, and traces them (closest hit). It prints one JSON line.
//
// Scene.filename: a scene file loaded as SceneLoader::loadStaticScene does
// (the binary cache "<file>.bin" if present, else a Wavefront OBJ file whose
// geometry is then cached; vertices normalised to the unit box), or a
// synthetic scene, used as generated: "synthetic:uniform:<n>",
// "synthetic:clustered:<n>" or "synthetic:heightfield:<nx>x<ny>".
//
// Besides build and trace rates, the line carries the BVH statistics that
// Benchmark::testStatic prints (Benchmark.cpp:80-90): SAH cost, average leaf
// size and the leaf-size histogram.
//
// Usage: hippie_b200_bench <file.env> [--steps K] [--dry-run]
//   --dry-run  parse the env file, load the scene and print the resolved
//              settings and the scene's size; no GPU use.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hippie_b200.hpp"

namespace {

using hippie_b200::check;
using hippie_b200::Error;

struct HostMesh {
    std::vector<float> v;    // xyz per vertex
    std::vector<int32_t> t;  // three vertex indices per triangle
};

// A scene file as SceneLoader::loadStaticScene reads it: the binary cache
// beside it (name + ".bin") or the OBJ file itself (then cached), normalised.
HostMesh load_file(const std::string& path) {
    hp_host_scene sc;
    check(hp_scene_load(path.c_str(), 1, &sc), "hp_scene_load");
    HostMesh m;
    m.v.assign(sc.vertices, sc.vertices + 3 * sc.num_vertices);
    m.t.assign(sc.triangles, sc.triangles + 3 * sc.num_triangles);
    hp_scene_free(&sc);
    return m;
}

HostMesh make_scene(const std::string& name) {
    HostMesh m;
    auto num = [&](const std::string& s) { return std::strtoll(s.c_str(), nullptr, 10); };
    const std::string pre = "synthetic:";
    if (name.compare(0, pre.size(), pre) != 0) return load_file(name);
    const std::string rest = name.substr(pre.size());
    const size_t colon = rest.find(':');
    const std::string kind = rest.substr(0, colon), arg = colon == std::string::npos ? "" : rest.substr(colon + 1);
    if (kind == "uniform" || kind == "clustered") {
        const int64_t n = num(arg);
        if (n <= 0) throw Error(HP_ERR_ARG, "synthetic scene needs a triangle count: " + name);
        m.v.resize(9 * n);
        m.t.resize(3 * n);
        if (kind == "uniform") check(hp_gen_uniform_mesh(0xC0FFEE, n, 0.01f, m.v.data(), m.t.data()), "hp_gen");
        else check(hp_gen_clustered_mesh(0xC0FFEE, n, 1024, 0.02f, 0.005f, m.v.data(), m.t.data()), "hp_gen");
    } else if (kind == "heightfield") {
        const size_t x = arg.find('x');
        const int nx = (int)num(arg.substr(0, x)), ny = x == std::string::npos ? 0 : (int)num(arg.substr(x + 1));
        if (nx < 2 || ny < 2) throw Error(HP_ERR_ARG, "heightfield needs <nx>x<ny>: " + name);
        m.v.resize(3 * (size_t)nx * ny);
        m.t.resize(6 * (size_t)(nx - 1) * (ny - 1));
        check(hp_gen_heightfield(0xC0FFEE, nx, ny, 1.0f, 2.0f, 16, m.v.data(), m.t.data()), "hp_gen");
    } else {
        throw Error(HP_ERR_ARG, "unknown synthetic scene: " + name);
    }
    return m;
}

template <typename T>
T* to_device(const std::vector<T>& h) {
    T* d = nullptr;
    if (cudaMalloc(&d, std::max<size_t>(h.size(), 1) * sizeof(T)) != cudaSuccess)
        throw Error(HP_ERR_OOM, "cudaMalloc failed");
    if (!h.empty() && cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        throw Error(HP_ERR_CUDA, "cudaMemcpy failed");
    return d;
}

const char* method_name(int m) {
    switch (m) {
    case HP_METHOD_PLOC: return "ploc";
    case HP_METHOD_ATR: return "atr";
    case HP_METHOD_TR: return "tr";
    case HP_METHOD_HLBVH: return "hlbvh";
    default: return "lbvh";
    }
}

int run(int argc, char** argv) {
    if (argc < 2 || !std::strcmp(argv[1], "--help")) {
        std::printf("usage: hippie_b200_bench <file.env> [--steps K] [--dry-run]\n");
        return argc < 2 ? 2 : 0;
    }
    int steps = 5;
    bool dry = false;
    for (int i = 2; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--steps") && i + 1 < argc) steps = std::max(1, std::atoi(argv[++i]));
        else if (!std::strcmp(argv[i], "--dry-run")) dry = true;
        else throw Error(HP_ERR_ARG, std::string("unknown argument ") + argv[i]);
    }
    hippie_b200::Environment env;
    env.readFile(argv[1]);
    const hp_build_params p = env.buildParams();
    const std::string scene = env.getString("Scene.filename");
    const int w = env.getInt("Resolution.width"), h = env.getInt("Resolution.height");
    const int samples = env.getInt("Renderer.numberOfPrimarySamples");
    float pos[3], dir[3];
    env.getVector("Camera.position", pos);
    env.getVector("Camera.direction", dir);
    const float fov = env.getFloat("Camera.fieldOfView"), znear = env.getFloat("Camera.nearPlane"),
                zfar = env.getFloat("Camera.farPlane");
    if (env.getFloat("Camera.wheelAngle") != 0.0f) throw Error(HP_ERR_UNSUPPORTED, "Camera.wheelAngle must be 0");
    if (dry) {
        const HostMesh dm = make_scene(scene);
        std::printf("{\"scene\": \"%s\", \"triangles\": %lld, \"vertices\": %lld, \"method\": \"%s\", \"morton_bits\": %d, \"ploc_radius\": %d, "
                    "\"atr_iterations\": %d, \"atr_treelet\": %d, \"ct\": %g, \"ci\": %g, \"max_leaf_size\": %d, "
                    "\"adaptive_leaf\": %d, \"width\": %d, \"height\": %d, \"samples\": %d, "
                    "\"camera\": [%g, %g, %g, %g, %g, %g], \"fov\": %g, \"near\": %g, \"far\": %g}\n",
                    scene.c_str(), (long long)(dm.t.size() / 3), (long long)(dm.v.size() / 3), method_name(p.method),
                    p.morton_bits, p.ploc_radius, p.atr_iterations,
                    p.atr_treelet, p.ct, p.ci, p.max_leaf_size, p.adaptive_leaf, w, h, samples, pos[0], pos[1],
                    pos[2], dir[0], dir[1], dir[2], fov, znear, zfar);
        return 0;
    }
    const HostMesh hm = make_scene(scene);
    hippie_b200::Context ctx(0);
    float* dv = to_device(hm.v);
    int32_t* dt = to_device(hm.t);
    const hp_mesh mesh{dv, dt, (int64_t)(hm.v.size() / 3), (int64_t)(hm.t.size() / 3)};
    hippie_b200::Builder builder(ctx, p);
    hippie_b200::BVH bvh(ctx);
    builder.rebuild(bvh, mesh);  // warm-up
    double build_s = 0.0;
    for (int k = 0; k < steps; ++k) build_s += builder.rebuild(bvh, mesh);
    build_s /= steps;
    const int nodes = bvh.getNumberOfNodes();
    const hp_bvh_stats st = bvh.stats();
    const double cost = st.sah_cost;
    const bool valid = bvh.validate(mesh);
    std::string hist;
    for (int k = 0; k <= HP_MAX_LEAF_SIZE_HIST; ++k) {
        char buf[32];
        std::snprintf(buf, sizeof(buf), "%s%.9g", k ? ", " : "", st.leaf_size_histogram[k]);
        hist += buf;
    }

    std::vector<int32_t> table((size_t)w * h);
    check(hp_pixel_table(w, h, table.data()), "hp_pixel_table");
    int32_t* dtable = to_device(table);
    float m[16];
    check(hp_camera_screen_to_world(pos, dir, fov, w, h, znear, zfar, m), "hp_camera_screen_to_world");
    float* drays = nullptr;
    int32_t* dres = nullptr;
    const int64_t nrays = (int64_t)w * h;
    if (cudaMalloc(&drays, nrays * 32) != cudaSuccess || cudaMalloc(&dres, nrays * 16) != cudaSuccess)
        throw Error(HP_ERR_OOM, "cudaMalloc failed");
    hippie_b200::Tracer tracer(ctx);
    tracer.setBVH(&bvh);
    double trace_s = 0.0;
    int64_t hits = 0;
    std::vector<int32_t> res((size_t)nrays * 4);
    for (int s = 0; s < samples; ++s) {
        check(hp_gen_primary_rays(ctx.get(), pos, m, w, h, zfar, s, dtable, drays, nullptr), "hp_gen_primary_rays");
        trace_s += tracer.trace(drays, nrays, dres);
        if (cudaMemcpy(res.data(), dres, res.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw Error(HP_ERR_CUDA, "cudaMemcpy failed");
        for (int64_t i = 0; i < nrays; ++i) hits += res[4 * i] >= 0;
    }
    ctx.synchronize();
    const int64_t tris = mesh.num_triangles;
    std::printf("{\"scene\": \"%s\", \"triangles\": %lld, \"method\": \"%s\", \"nodes\": %d, \"valid\": %s, "
                "\"sah_cost\": %.17g, \"build_ms\": %.4f, \"build_mtris_s\": %.2f, \"rays\": %lld, "
                "\"trace_ms\": %.4f, \"trace_mrays_s\": %.2f, \"hits\": %lld, \"hit_fraction\": %.17g, "
                "\"avg_leaf_size\": %.17g, \"leaf_size_histogram\": [%s]}\n",
                scene.c_str(), (long long)tris, method_name(p.method), nodes, valid ? "true" : "false", cost,
                build_s * 1e3, tris / build_s / 1e6, (long long)(nrays * samples), trace_s * 1e3,
                nrays * samples / trace_s / 1e6, (long long)hits,
                samples ? (double)hits / (double)(nrays * samples) : 0.0, st.avg_leaf_size, hist.c_str());
    cudaFree(dv);
    cudaFree(dt);
    cudaFree(dtable);
    cudaFree(drays);
    cudaFree(dres);
    return valid ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "hippie_b200_bench: %s\n", e.what());
        return 1;
    }
}
