// Block-structured environment files with the reference's option set and
// semantics (environment/Environment.cpp:17-466, environment/AppEnvironment.cpp:10-91):
//   * `Block { key value ... }`, `#` starts a comment, words split on space / tab;
//   * every option is registered with a type and a default; an unknown key or a
//     value that does not parse as the option's type fails the whole file;
//   * int values are normalised through an integer, float values through the
//     6-significant-digit text form QString::number(float) produces, bools
//     accept true/yes/on/1 and false/no/off/0 (lower or upper case), vectors
//     take three floats;
//   * repeated keys append values and getters return the first one.
// One option is added: Bvh.atrTreeletSize (default 20, the ATRBuilder default,
// rt/bvh/ATRBuilder.h:13), so that the treelet size can be configured.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include "hp_internal.h"

namespace {

enum opt_type { OPT_INT, OPT_FLOAT, OPT_BOOL, OPT_VECTOR, OPT_STRING };

struct option {
    std::string name;
    opt_type type;
    std::string def;
    std::vector<std::string> values;
};

bool parse_int(const std::string& s, long& out) {
    if (s.empty()) return false;
    char* end = nullptr;
    errno = 0;
    long v = std::strtol(s.c_str(), &end, 10);
    if (errno != 0 || *end != '\0' || v < INT32_MIN || v > INT32_MAX) return false;
    out = v;
    return true;
}

bool parse_float(const std::string& s, float& out) {
    if (s.empty()) return false;
    char* end = nullptr;
    errno = 0;
    float v = std::strtof(s.c_str(), &end);
    if (*end != '\0' || errno == ERANGE) return false;
    out = v;
    return true;
}

std::string fmt_float(float v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%g", (double)v);
    return buf;
}

bool filter_value(const std::string& value, std::string& filtered, opt_type type) {
    switch (type) {
    case OPT_INT: {
        long v;
        if (!parse_int(value, v)) return false;
        filtered = std::to_string(v);
        return true;
    }
    case OPT_FLOAT: {
        float v;
        if (!parse_float(value, v)) return false;
        filtered = fmt_float(v);
        return true;
    }
    case OPT_BOOL:
        if (value == "true" || value == "yes" || value == "on" || value == "1" || value == "TRUE" ||
            value == "YES" || value == "ON") {
            filtered = "1";
            return true;
        }
        if (value == "false" || value == "no" || value == "off" || value == "0" || value == "FALSE" ||
            value == "NO" || value == "OFF") {
            filtered = "0";
            return true;
        }
        return false;
    case OPT_VECTOR: {
        std::istringstream is(value);
        std::string a, b, c, extra;
        if (!(is >> a >> b >> c) || (is >> extra)) return false;
        float x, y, z;
        if (!parse_float(a, x) || !parse_float(b, y) || !parse_float(c, z)) return false;
        filtered = fmt_float(x) + " " + fmt_float(y) + " " + fmt_float(z);
        return true;
    }
    case OPT_STRING:
        filtered = value;
        return !value.empty();
    }
    return false;
}

void warn(const std::string& msg) {
    if (!std::getenv("HP_QUIET")) std::fprintf(stderr, "WARN <Environment> %s\n", msg.c_str());
}

}  // namespace

struct hp_env {
    std::vector<option> options;

    void reg(const char* name, const char* def, opt_type t) {
        option o;
        o.name = name;
        o.type = t;
        if (def && !filter_value(def, o.def, t)) o.def.clear();
        options.push_back(o);
    }
    option* find(const std::string& name) {
        for (auto& o : options)
            if (o.name == name) return &o;
        return nullptr;
    }
    const option* find(const std::string& name) const {
        for (auto& o : options)
            if (o.name == name) return &o;
        return nullptr;
    }
    const std::string* first(const std::string& name) const {
        const option* o = find(name);
        if (!o) return nullptr;
        if (!o->values.empty() && !o->values.front().empty()) return &o->values.front();
        if (!o->def.empty()) return &o->def;
        return nullptr;
    }

    hp_env() {
        reg("Application.mode", "interactive", OPT_STRING);
        reg("Application.stats", "1", OPT_BOOL);
        reg("Benchmark.output", "default", OPT_STRING);
        reg("Benchmark.images", "0", OPT_BOOL);
        reg("Resolution.width", "1024", OPT_INT);
        reg("Resolution.height", "768", OPT_INT);
        reg("Scene.filename", nullptr, OPT_STRING);
        reg("Scene.filefilter", nullptr, OPT_STRING);
        reg("Scene.environment", nullptr, OPT_STRING);
        reg("Scene.light", "5.0 -2.0 1.0", OPT_VECTOR);
        reg("Renderer.numberOfPrimarySamples", "1", OPT_INT);
        reg("Renderer.numberOfAOSamples", "8", OPT_INT);
        reg("Renderer.numberOfShadowSamples", "2", OPT_INT);
        reg("Renderer.aoRadius", "0.01", OPT_FLOAT);
        reg("Renderer.shadowRadius", "0.001", OPT_FLOAT);
        reg("Renderer.rayType", "primary", OPT_STRING);
        reg("Renderer.nodeSizeThreshold", "5000", OPT_INT);
        reg("Renderer.thermalThreshold", "250", OPT_INT);
        reg("Renderer.recursionDepth", "1", OPT_INT);
        reg("Renderer.keyValue", "0.6", OPT_FLOAT);
        reg("Renderer.whitePoint", "2.0", OPT_FLOAT);
        reg("Renderer.russianRoulette", "0", OPT_BOOL);
        reg("Renderer.sortShadowRays", "0", OPT_BOOL);
        reg("Renderer.sortAORays", "0", OPT_BOOL);
        reg("Renderer.sortPathRays", "0", OPT_BOOL);
        reg("Renderer.shadowRayLength", "0.0", OPT_FLOAT);
        reg("Renderer.aoRayLength", "0.25", OPT_FLOAT);
        reg("Renderer.pathRayLength", "0.25", OPT_FLOAT);
        reg("Renderer.shadowMortonCodeBits", "32", OPT_INT);
        reg("Renderer.aoMortonCodeBits", "32", OPT_INT);
        reg("Renderer.pathMortonCodeBits", "32", OPT_INT);
        reg("Renderer.shadowMortonCodeMethod", "aila", OPT_STRING);
        reg("Renderer.aoMortonCodeMethod", "aila", OPT_STRING);
        reg("Renderer.pathMortonCodeMethod", "aila", OPT_STRING);
        reg("Bvh.layout", "bin", OPT_STRING);
        reg("Bvh.ct", "3.0", OPT_FLOAT);
        reg("Bvh.ci", "2.0", OPT_FLOAT);
        reg("Bvh.maxLeafSize", "8", OPT_INT);
        reg("Bvh.adaptiveLeafSize", "1", OPT_BOOL);
        reg("Bvh.presplitting", "0", OPT_BOOL);
        reg("Bvh.lbvhMortonCodeBits", "60", OPT_INT);
        reg("Bvh.hlbvhMortonCodeBits", "60", OPT_INT);
        reg("Bvh.hlbvhMortonCodeSAHBits", "15", OPT_INT);
        reg("Bvh.trIterations", "2", OPT_INT);
        reg("Bvh.trMortonCodeBits", "60", OPT_INT);
        reg("Bvh.atrIterations", "2", OPT_INT);
        reg("Bvh.atrMortonCodeBits", "60", OPT_INT);
        reg("Bvh.atrTreeletSize", "20", OPT_INT);
        reg("Bvh.insertionMortonCodeBits", "60", OPT_INT);
        reg("Bvh.insertionMod", "1", OPT_INT);
        reg("Bvh.insertionSbvh", "0", OPT_BOOL);
        reg("Bvh.plocRadius", "1", OPT_INT);
        reg("Bvh.plocMaxRadius", "512", OPT_INT);
        reg("Bvh.plocMortonCodeBits", "60", OPT_INT);
        reg("Bvh.plocAdaptive", "0", OPT_BOOL);
        reg("Bvh.sbvhAlpha", "0.00001", OPT_FLOAT);
        reg("Bvh.presplitterBeta", "0.1", OPT_FLOAT);
        reg("Bvh.method", "lbvh", OPT_STRING);
        reg("Bvh.update", "refit", OPT_STRING);
        reg("Camera.position", "0.0 0.0 0.0", OPT_VECTOR);
        reg("Camera.direction", "0.0 0.0 -1.0", OPT_VECTOR);
        reg("Camera.wheelAngle", "0.0", OPT_FLOAT);
        reg("Camera.nearPlane", "0.001", OPT_FLOAT);
        reg("Camera.farPlane", "3.0", OPT_FLOAT);
        reg("Camera.fieldOfView", "45.0", OPT_FLOAT);
        reg("Camera.step", "0.025", OPT_FLOAT);
        reg("Animation.frameRate", "30.0", OPT_FLOAT);
        reg("Animation.loop", "1", OPT_BOOL);
        reg("Animation.pause", "0", OPT_BOOL);
        reg("Screenshots.directory", "screenshots", OPT_STRING);
    }

    // Environment::readEnvFile (Environment.cpp:309-466) over text.
    hp_status read(const std::string& text, const std::string& source) {
        std::istringstream in(text);
        std::string line, block_name, last;
        bool block = false;
        int line_no = 0;
        while (std::getline(in, line)) {
            ++line_no;
            if (!line.empty() && line.back() == '\r') line.pop_back();
            size_t hash = line.find('#');
            if (hash != std::string::npos) line = line.substr(0, hash);
            std::vector<std::string> words;
            {
                std::string w;
                for (char ch : line) {
                    if (ch == ' ' || ch == '\t' || ch == '\n') {
                        if (!w.empty()) words.push_back(w);
                        w.clear();
                    } else {
                        w.push_back(ch);
                    }
                }
                if (!w.empty()) words.push_back(w);
            }
            for (size_t i = 0; i < words.size(); ++i) {
                const std::string& word = words[i];
                if (word == "{") {
                    block_name = last;
                    block = true;
                } else if (word == "}") {
                    if (block_name.empty())
                        return hp_fail(HP_ERR_PARSE, "unpaired } in '" + source + "' (line " +
                                                         std::to_string(line_no) + ")");
                    block = false;
                    block_name.clear();
                } else if (block) {
                    const std::string name = block_name + "." + word;
                    option* o = find(name);
                    if (!o)
                        return hp_fail(HP_ERR_PARSE, "unknown option '" + name + "' in '" + source +
                                                         "' (line " + std::to_string(line_no) + ")");
                    std::string value;
                    if (o->type == OPT_VECTOR) {
                        if (i + 3 >= words.size())
                            return hp_fail(HP_ERR_PARSE, "mismatch in vector variable " + name +
                                                             " (line " + std::to_string(line_no) + ")");
                        if (!filter_value(words[i + 1] + " " + words[i + 2] + " " + words[i + 3], value,
                                          OPT_VECTOR))
                            return hp_fail(HP_ERR_PARSE, "mismatch in vector variable " + name +
                                                             " (line " + std::to_string(line_no) + ")");
                        o->values.push_back(value);
                        i += 3;
                    } else {
                        if (i + 1 >= words.size() || !filter_value(words[i + 1], value, o->type))
                            return hp_fail(HP_ERR_PARSE, "mismatch in variable " + name + " (line " +
                                                             std::to_string(line_no) + ")");
                        ++i;
                        o->values.push_back(value);
                    }
                }
                last = words[i];
            }
        }
        return HP_OK;
    }
};

extern "C" {

hp_status hp_env_create(hp_env** out) {
    if (!out) return hp_fail(HP_ERR_ARG, "hp_env_create: null output");
    *out = new hp_env();
    return HP_OK;
}

hp_status hp_env_destroy(hp_env* env) {
    delete env;
    return HP_OK;
}

hp_status hp_env_read_string(hp_env* env, const char* text) {
    if (!env || !text) return hp_fail(HP_ERR_ARG, "hp_env_read_string: null argument");
    return env->read(text, "<string>");
}

hp_status hp_env_read_file(hp_env* env, const char* path) {
    if (!env || !path) return hp_fail(HP_ERR_ARG, "hp_env_read_file: null argument");
    std::ifstream f(path);
    if (!f) return hp_fail(HP_ERR_PARSE, std::string("cannot open environment file '") + path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    return env->read(ss.str(), path);
}

hp_status hp_env_get_int(const hp_env* env, const char* name, int32_t* value) {
    if (!env || !name || !value) return hp_fail(HP_ERR_ARG, "hp_env_get_int: null argument");
    const std::string* s = env->first(name);
    if (!s) return hp_fail(HP_ERR_ARG, std::string("option has no value: ") + name);
    *value = (int32_t)std::strtol(s->c_str(), nullptr, 10);
    return HP_OK;
}

hp_status hp_env_get_float(const hp_env* env, const char* name, float* value) {
    if (!env || !name || !value) return hp_fail(HP_ERR_ARG, "hp_env_get_float: null argument");
    const std::string* s = env->first(name);
    if (!s) return hp_fail(HP_ERR_ARG, std::string("option has no value: ") + name);
    *value = std::strtof(s->c_str(), nullptr);
    return HP_OK;
}

hp_status hp_env_get_bool(const hp_env* env, const char* name, int32_t* value) {
    if (!env || !name || !value) return hp_fail(HP_ERR_ARG, "hp_env_get_bool: null argument");
    const std::string* s = env->first(name);
    if (!s) return hp_fail(HP_ERR_ARG, std::string("option has no value: ") + name);
    *value = std::strtol(s->c_str(), nullptr, 10) != 0;
    return HP_OK;
}

hp_status hp_env_get_string(const hp_env* env, const char* name, char* buf, int64_t buf_size) {
    if (!env || !name || !buf || buf_size <= 0)
        return hp_fail(HP_ERR_ARG, "hp_env_get_string: bad argument");
    const std::string* s = env->first(name);
    if (!s) return hp_fail(HP_ERR_ARG, std::string("option has no value: ") + name);
    if ((int64_t)s->size() + 1 > buf_size) return hp_fail(HP_ERR_ARG, "hp_env_get_string: buffer too small");
    std::memcpy(buf, s->c_str(), s->size() + 1);
    return HP_OK;
}

// The builders' option handling: BVHBuilder (rt/bvh/BVHBuilder.h:26-32,60-63),
// LBVHBuilder::setMortonCodeBits (LBVHBuilder.cpp:269-272), PLOCBuilder
// constructor and setters (PLOCBuilder.cpp:210-275), ATRBuilder setters
// (ATRBuilder.cpp:277-289) and HipBVH's ct / ci (HipBVH.cpp:331-335). A value
// outside its range keeps the previous value and logs a warning.
hp_status hp_env_build_params(const hp_env* env, hp_build_params* p) {
    if (!env || !p) return hp_fail(HP_ERR_ARG, "hp_env_build_params: null argument");
    hp_build_params_default(p);
    int32_t iv;
    float fv;
    char method[64] = {0};
    char layout[64] = {0};
    HP_TRY(hp_env_get_string(env, "Bvh.method", method, sizeof(method)));
    HP_TRY(hp_env_get_string(env, "Bvh.layout", layout, sizeof(layout)));
    // HipBVH::HipBVH (rt/bvh/HipBVH.cpp:317-325): "bin", "quad", anything else Oct
    if (!std::strcmp(layout, "bin")) p->layout = HP_LAYOUT_BIN;
    else if (!std::strcmp(layout, "quad")) p->layout = HP_LAYOUT_QUAD;
    else p->layout = HP_LAYOUT_OCT;
    const char* bits_key;
    if (!std::strcmp(method, "lbvh")) { p->method = HP_METHOD_LBVH; bits_key = "Bvh.lbvhMortonCodeBits"; }
    else if (!std::strcmp(method, "ploc")) { p->method = HP_METHOD_PLOC; bits_key = "Bvh.plocMortonCodeBits"; }
    else if (!std::strcmp(method, "atr")) { p->method = HP_METHOD_ATR; bits_key = "Bvh.atrMortonCodeBits"; }
    else if (!std::strcmp(method, "tr")) { p->method = HP_METHOD_TR; bits_key = "Bvh.trMortonCodeBits"; }
    else if (!std::strcmp(method, "hlbvh")) { p->method = HP_METHOD_HLBVH; bits_key = "Bvh.hlbvhMortonCodeBits"; }
    else return hp_fail(HP_ERR_UNSUPPORTED, std::string("Bvh.method ") + method + " is not supported");
    if (hp_env_get_int(env, "Bvh.maxLeafSize", &iv) == HP_OK) {
        if (iv > 0 && iv <= 1024) p->max_leaf_size = iv;
        else warn("Maximum leaf size must be in range (0,1024].");
    }
    if (hp_env_get_bool(env, "Bvh.adaptiveLeafSize", &iv) == HP_OK) p->adaptive_leaf = iv;
    if (hp_env_get_bool(env, "Bvh.presplitting", &iv) == HP_OK && iv)
        return hp_fail(HP_ERR_UNSUPPORTED, "Bvh.presplitting is not supported");
    if (hp_env_get_int(env, bits_key, &iv) == HP_OK) {
        if (iv < 6 || iv > 60) warn("Morton code bits must be in range [6,60].");
        else p->morton_bits = iv;
    }
    // HLBVHBuilder::setMortonCodeSAHBits (rt/bvh/HLBVHBuilder.cpp:431-435)
    if (hp_env_get_int(env, "Bvh.hlbvhMortonCodeSAHBits", &iv) == HP_OK) {
        if (iv < 6 || iv > 15) warn("Morton code SAH bits must be in range [6,15].");
        else if (p->morton_bits < iv) warn("Morton code SAH bits must be less than Morton bits.");
        else p->hlbvh_sah_bits = iv;
    }
    if (hp_env_get_int(env, "Bvh.plocMaxRadius", &iv) == HP_OK) {
        if (iv < 1) warn("Max. radius must be positive.");
        else p->ploc_max_radius = iv;
    }
    if (hp_env_get_int(env, "Bvh.plocRadius", &iv) == HP_OK) {
        if (iv < 1 || iv > p->ploc_max_radius) warn("Radius must be in range [1,maxRadius].");
        else p->ploc_radius = iv;
    }
    if (hp_env_get_bool(env, "Bvh.plocAdaptive", &iv) == HP_OK) p->ploc_adaptive = iv;
    // TRBuilder::setIterations (rt/bvh/TRBuilder.cpp:331-334) / ATRBuilder's: [0,25]
    if (hp_env_get_int(env, p->method == HP_METHOD_TR ? "Bvh.trIterations" : "Bvh.atrIterations", &iv) == HP_OK) {
        if (iv < 0 || iv > 25) warn("Number of iterations must be in range [0,25].");
        else p->atr_iterations = iv;
    }
    if (hp_env_get_int(env, "Bvh.atrTreeletSize", &iv) == HP_OK) {
        if (iv < 4 || iv > 30) warn("Treelet size must be in range [4,30].");
        else p->atr_treelet = iv;
    }
    if (hp_env_get_float(env, "Bvh.ct", &fv) == HP_OK && fv > 0.0f) p->ct = fv;
    if (hp_env_get_float(env, "Bvh.ci", &fv) == HP_OK && fv > 0.0f) p->ci = fv;
    return HP_OK;
}

}  // extern "C"
