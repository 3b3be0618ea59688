// Scene files on the host: the reference's binary cache format, a Wavefront
// OBJ reader, and SceneLoader's normalisation.
//
// Reference (paths relative to src/hippie/):
//   BinImporter::importScene   util/BinImporter.cpp:16-84
//   BinExporter::exportScene   util/BinExporter.cpp:14-70
//   SceneLoader::loadScene     rt/scene/SceneLoader.cpp:14-101 (BINARY_CACHE 1: the
//                              ".bin" file beside the scene first, else the importer,
//                              whose result is then written to the ".bin" file)
//   SceneLoader::loadStaticScene  rt/scene/SceneLoader.cpp:103-160 (vertices moved to
//                              the box's minimum corner and scaled by 1 / longest side)
//   AssimpImporter::importScene   util/AssimpImporter.cpp:20-200 (REMOVE_DEGENERATES 1:
//                              triangles whose box has zero area are dropped; the box
//                              is the bound of all vertices)
//
// The binary format: int32 {vertices, triangles, materials, textures}, the box
// as 6 float32 (min xyz, max xyz), then vertices (3 float32 each), normals (3
// float32 each), texture coordinates (2 float32 each), triangles (3 int32
// each), material indices (int32 each), materials and texture names. Only the
// first five parts are read: the build and trace path needs no materials.
#include <sys/types.h>
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "hippie_b200.h"
#include "hp_internal.h"

namespace {

struct file_closer {
    std::FILE* f;
    ~file_closer() {
        if (f) std::fclose(f);
    }
};

void box_of(const float* v, int64_t nv, float* box) {
    const float big = std::numeric_limits<float>::max();
    box[0] = box[1] = box[2] = big;
    box[3] = box[4] = box[5] = -big;
    for (int64_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) {
            box[a] = std::min(box[a], v[3 * i + a]);
            box[3 + a] = std::max(box[3 + a], v[3 * i + a]);
        }
}

// AABB::area (util/AABB.h:36): zero for an invalid box.
float box_area(const float* mn, const float* mx) {
    if (!(mn[0] <= mx[0] && mn[1] <= mx[1] && mn[2] <= mx[2])) return 0.0f;
    const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

hp_status fill(hp_host_scene* out, std::vector<float>& v, std::vector<int32_t>& t, const float* box) {
    out->num_vertices = (int64_t)(v.size() / 3);
    out->num_triangles = (int64_t)(t.size() / 3);
    out->vertices = static_cast<float*>(std::malloc(std::max<size_t>(v.size(), 1) * sizeof(float)));
    out->triangles = static_cast<int32_t*>(std::malloc(std::max<size_t>(t.size(), 1) * sizeof(int32_t)));
    if (!out->vertices || !out->triangles) {
        std::free(out->vertices);
        std::free(out->triangles);
        out->vertices = nullptr;
        out->triangles = nullptr;
        return hp_fail(HP_ERR_OOM, "scene: out of host memory");
    }
    if (!v.empty()) std::memcpy(out->vertices, v.data(), v.size() * sizeof(float));
    if (!t.empty()) std::memcpy(out->triangles, t.data(), t.size() * sizeof(int32_t));
    std::memcpy(out->box, box, 6 * sizeof(float));
    return HP_OK;
}

bool ends_with(const std::string& s, const char* suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

}  // namespace

extern "C" {

hp_status hp_scene_read_bin(const char* path, hp_host_scene* out) {
    if (!path || !out) return hp_fail(HP_ERR_ARG, "hp_scene_read_bin: null argument");
    std::memset(out, 0, sizeof(*out));
    file_closer fc{std::fopen(path, "rb")};
    if (!fc.f) return hp_fail(HP_ERR_ARG, std::string("hp_scene_read_bin: cannot open ") + path);
    int32_t header[4];
    float box[6];
    if (std::fread(header, sizeof(int32_t), 4, fc.f) != 4 || std::fread(box, sizeof(float), 6, fc.f) != 6)
        return hp_fail(HP_ERR_PARSE, std::string("hp_scene_read_bin: truncated header in ") + path);
    const int64_t nv = header[0], nt = header[1];
    if (nv < 0 || nt < 0 || header[2] < 0 || header[3] < 0)
        return hp_fail(HP_ERR_PARSE, std::string("hp_scene_read_bin: negative count in ") + path);
    std::vector<float> v(3 * (size_t)nv);
    std::vector<int32_t> t(3 * (size_t)nt);
    // vertices, then skip normals (3 floats) and texture coordinates (2 floats) per vertex
    if (std::fread(v.data(), sizeof(float), v.size(), fc.f) != v.size() ||
        fseeko(fc.f, (off_t)(5 * sizeof(float)) * (off_t)nv, SEEK_CUR) != 0 ||
        std::fread(t.data(), sizeof(int32_t), t.size(), fc.f) != t.size())
        return hp_fail(HP_ERR_PARSE, std::string("hp_scene_read_bin: truncated data in ") + path);
    for (size_t i = 0; i < t.size(); ++i)
        if (t[i] < 0 || t[i] >= nv)
            return hp_fail(HP_ERR_PARSE, std::string("hp_scene_read_bin: vertex index out of range in ") + path);
    return fill(out, v, t, box);
}

hp_status hp_scene_write_bin(const char* path, const hp_host_scene* s) {
    if (!path || !s || (s->num_vertices && !s->vertices) || (s->num_triangles && !s->triangles))
        return hp_fail(HP_ERR_ARG, "hp_scene_write_bin: null argument");
    if (s->num_vertices > INT32_MAX || s->num_triangles > INT32_MAX)
        return hp_fail(HP_ERR_ARG, "hp_scene_write_bin: counts exceed the format's int32 header");
    file_closer fc{std::fopen(path, "wb")};
    if (!fc.f) return hp_fail(HP_ERR_ARG, std::string("hp_scene_write_bin: cannot create ") + path);
    const int32_t header[4] = {(int32_t)s->num_vertices, (int32_t)s->num_triangles, 0, 0};
    const std::vector<float> zeros(5 * (size_t)s->num_vertices, 0.0f);    // normals, texture coordinates
    const std::vector<int32_t> mat((size_t)s->num_triangles, 0);          // material indices
    bool ok = std::fwrite(header, sizeof(int32_t), 4, fc.f) == 4 && std::fwrite(s->box, sizeof(float), 6, fc.f) == 6;
    ok = ok && std::fwrite(s->vertices, sizeof(float), 3 * s->num_vertices, fc.f) == (size_t)(3 * s->num_vertices);
    ok = ok && std::fwrite(zeros.data(), sizeof(float), zeros.size(), fc.f) == zeros.size();
    ok = ok && std::fwrite(s->triangles, sizeof(int32_t), 3 * s->num_triangles, fc.f) ==
                   (size_t)(3 * s->num_triangles);
    ok = ok && std::fwrite(mat.data(), sizeof(int32_t), mat.size(), fc.f) == mat.size();
    if (!ok) return hp_fail(HP_ERR_ARG, std::string("hp_scene_write_bin: write failed for ") + path);
    return HP_OK;
}

hp_status hp_scene_read_obj(const char* path, hp_host_scene* out) {
    if (!path || !out) return hp_fail(HP_ERR_ARG, "hp_scene_read_obj: null argument");
    std::memset(out, 0, sizeof(*out));
    std::ifstream in(path);
    if (!in) return hp_fail(HP_ERR_ARG, std::string("hp_scene_read_obj: cannot open ") + path);
    std::vector<float> v;
    std::vector<int32_t> t;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream is(line);
        std::string tag;
        if (!(is >> tag)) continue;
        if (tag == "v") {
            float x, y, z;
            if (!(is >> x >> y >> z)) return hp_fail(HP_ERR_PARSE, "hp_scene_read_obj: bad vertex line: " + line);
            v.insert(v.end(), {x, y, z});
        } else if (tag == "f") {
            std::vector<int32_t> idx;
            std::string tok;
            const long nv = (long)(v.size() / 3);
            while (is >> tok) {
                errno = 0;
                const long k = std::strtol(tok.c_str(), nullptr, 10);
                const long i = k > 0 ? k - 1 : nv + k;
                if (errno || k == 0 || i < 0 || i >= nv)
                    return hp_fail(HP_ERR_PARSE, "hp_scene_read_obj: bad face index in: " + line);
                idx.push_back((int32_t)i);
            }
            for (size_t j = 1; j + 1 < idx.size(); ++j) {  // polygons as triangle fans
                const int32_t tri[3] = {idx[0], idx[j], idx[j + 1]};
                float mn[3], mx[3];
                for (int a = 0; a < 3; ++a) {
                    mn[a] = std::min({v[3 * tri[0] + a], v[3 * tri[1] + a], v[3 * tri[2] + a]});
                    mx[a] = std::max({v[3 * tri[0] + a], v[3 * tri[1] + a], v[3 * tri[2] + a]});
                }
                if (box_area(mn, mx) > 0.0f) t.insert(t.end(), tri, tri + 3);  // REMOVE_DEGENERATES
            }
        }
    }
    if (t.empty()) return hp_fail(HP_ERR_PARSE, std::string("hp_scene_read_obj: no triangles in ") + path);
    float box[6];
    box_of(v.data(), (int64_t)(v.size() / 3), box);
    return fill(out, v, t, box);
}

hp_status hp_scene_normalize(hp_host_scene* s) {
    if (!s || (s->num_vertices && !s->vertices)) return hp_fail(HP_ERR_ARG, "hp_scene_normalize: null argument");
    const float dx = s->box[3] - s->box[0], dy = s->box[4] - s->box[1], dz = s->box[5] - s->box[2];
    const float scale = 1.0f / std::max(std::max(dx, dy), dz);
    for (int64_t i = 0; i < s->num_vertices; ++i)
        for (int a = 0; a < 3; ++a) {
            float x = s->vertices[3 * i + a];
            x -= s->box[a];
            x *= scale;
            s->vertices[3 * i + a] = x;
        }
    return HP_OK;
}

hp_status hp_scene_load(const char* path, int32_t write_cache, hp_host_scene* out) {
    if (!path || !out) return hp_fail(HP_ERR_ARG, "hp_scene_load: null argument");
    std::memset(out, 0, sizeof(*out));
    const std::string p(path);
    const std::string cache = ends_with(p, ".bin") ? p : p + ".bin";
    if (std::FILE* f = std::fopen(cache.c_str(), "rb")) {
        std::fclose(f);
        HP_TRY(hp_scene_read_bin(cache.c_str(), out));
    } else {
        HP_TRY(hp_scene_read_obj(path, out));
        if (write_cache) hp_scene_write_bin(cache.c_str(), out);  // a cache that cannot be written is skipped
    }
    return hp_scene_normalize(out);
}

void hp_scene_free(hp_host_scene* s) {
    if (!s) return;
    std::free(s->vertices);
    std::free(s->triangles);
    std::memset(s, 0, sizeof(*s));
}

}  // extern "C"
