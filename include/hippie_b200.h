/*
 * hippie_b200.h — C ABI of the B200-native build-and-trace hot path.
 *
 * This is the boundary a host program binds to (cgo / ctypes / JNI style):
 * plain pointers, 64-bit sizes and status codes, no CUDA or C++ types.
 * Streams are passed as `void*` (a cudaStream_t; NULL = legacy default stream).
 *
 * The entry points replace these reference interfaces (meistdan/hippie,
 * paths relative to src/hippie/):
 *   hp_build            BVHBuilder::build / rebuild           rt/bvh/BVHBuilder.h:16-68,
 *                       LBVHBuilder::build                    rt/bvh/LBVHBuilder.cpp:183-241,
 *                       PLOCBuilder::build                    rt/bvh/PLOCBuilder.cpp:161-208,
 *                       ATRBuilder::build                     rt/bvh/ATRBuilder.cpp:180-236
 *   hp_bvh_*            HipBVH (nodes, woop, triangle idx)    rt/bvh/HipBVH.h:19-106
 *   hp_bvh_cost         HipBVH::getCost                       rt/bvh/HipBVH.cpp:346-370
 *   hp_bvh_validate     HipBVH::validate                      rt/bvh/HipBVH.cpp:157-307
 *   hp_bvh_stats_get    HipBVH::getAvgLeafSize, getLeafSizeHistogram
 *                                                             rt/bvh/HipBVH.cpp:372-442
 *   hp_refit            HipBVH::update (woopify + refit)      rt/bvh/HipBVH.cpp:472-477
 *   hp_trace            HipTracer::trace / traceStats         rt/tracer/HipTracer.cpp:13-52
 *   hp_trace_sorted     HipTracer::traceSort                  rt/tracer/HipTracer.cpp:109-125
 *   hp_gen_primary_rays RayGen::primary                       rt/ray/RayGen.cpp:35-62
 *   hp_pixel_table      PixelTable::recalculate               rt/ray/PixelTable.cpp:10-80
 *   hp_ray_keys         RayBuffer::computeMortonCodes         rt/ray/RayBuffer.cpp:31-80
 *   hp_radix_sort       RadixSort::sort                       radix_sort/RadixSort.cpp:181-238
 *   hp_env_*            Environment / AppEnvironment          environment/Environment.cpp:290-466,
 *                                                             environment/AppEnvironment.cpp:10-91
 * and add the batched and adjoint entry points the reference does not have.
 *
 * Every function returns hp_status and never exits the process; the text of
 * the last error on the calling thread is available from hp_last_error().
 * All device work is stream-ordered and asynchronous unless stated.
 */
#ifndef HIPPIE_B200_H_
#define HIPPIE_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HP_ABI_VERSION 2

typedef enum hp_status {
    HP_OK = 0,
    HP_ERR_CUDA = 1,          /* a CUDA runtime call failed */
    HP_ERR_ARG = 2,           /* invalid argument (null pointer, size out of range, ...) */
    HP_ERR_OOM = 3,           /* device or host allocation failed */
    HP_ERR_TIMEOUT = 4,       /* a host-side wait exceeded its limit */
    HP_ERR_DEVICE_STATUS = 5, /* a kernel reported an error word (bounded spin gave up, bad index) */
    HP_ERR_UNSUPPORTED = 6,   /* option not supported by the library */
    HP_ERR_PARSE = 7          /* environment file could not be parsed */
} hp_status;

typedef enum hp_method {
    HP_METHOD_LBVH = 0,       /* Bvh.method lbvh */
    HP_METHOD_PLOC = 1,       /* Bvh.method ploc */
    HP_METHOD_ATR = 2,        /* Bvh.method atr  (LBVH + agglomerative treelet restructuring) */
    HP_METHOD_TR = 3,         /* Bvh.method tr   (LBVH + treelet restructuring by dynamic programming,
                                 treelet 7: TRBuilder) */
    HP_METHOD_HLBVH = 4       /* Bvh.method hlbvh (LBVH clusters below the top Morton bits, binned SAH
                                 above them: HLBVHBuilder) */
} hp_method;

/* Node layouts: children per node (HipBVH::Layout, rt/bvh/HipBVH.h:23-27). A
 * node of layout L is 32*L bytes (HipBVHNodeN<L>, rt/bvh/HipBVHNode.h:14-218). */
typedef enum hp_layout {
    HP_LAYOUT_BIN = 2,
    HP_LAYOUT_QUAD = 4,
    HP_LAYOUT_OCT = 8
} hp_layout;

/* Trace flags (HipTracer: `anyHit` kernel argument and the traceStats variant). */
#define HP_TRACE_ANY_HIT 1u
#define HP_TRACE_STATS   2u

/* Triangle mesh in device memory: vertices are 3 floats each, triangles are
 * 3 int vertex indices each (the Scene vertex / vertIndices buffers). */
typedef struct hp_mesh {
    const float* vertices;
    const int32_t* triangles;
    int64_t num_vertices;
    int64_t num_triangles;
} hp_mesh;

/* Build options: the Bvh.* environment keys of the reference
 * (environment/AppEnvironment.cpp:52-75) plus Bvh.atrTreeletSize. */
typedef struct hp_build_params {
    int32_t method;           /* hp_method                     Bvh.method          */
    int32_t morton_bits;      /* [6,60]                        Bvh.{lbvh,ploc,atr,tr,hlbvh}MortonCodeBits */
    int32_t ploc_radius;      /* [1,ploc_max_radius]           Bvh.plocRadius      */
    int32_t ploc_max_radius;  /* >= 1                          Bvh.plocMaxRadius   */
    int32_t ploc_adaptive;    /* 0/1                           Bvh.plocAdaptive    */
    int32_t atr_iterations;   /* [0,25]                        Bvh.atrIterations (tr: Bvh.trIterations) */
    int32_t atr_treelet;      /* [4,30]                        Bvh.atrTreeletSize  */
    float ct;                 /* > 0                           Bvh.ct              */
    float ci;                 /* > 0                           Bvh.ci              */
    int32_t max_leaf_size;    /* (0,1024]                      Bvh.maxLeafSize     */
    int32_t adaptive_leaf;    /* 0/1                           Bvh.adaptiveLeafSize */
    int32_t layout;           /* hp_layout; 0 means Bin        Bvh.layout          */
    int32_t hlbvh_sah_bits;   /* 6, 9, 12 or 15, <= morton_bits Bvh.hlbvhMortonCodeSAHBits */
    int32_t reserved[3];
} hp_build_params;

/* A built BVH. Device pointers are owned by the library; release with
 * hp_bvh_free. The node buffer uses the reference's 64-byte binary node
 * layout (rt/bvh/HipBVHNode.h:116-218):
 *   int[16]: [0..3] child0 {lo.x, hi.x, lo.y, hi.y}, [4..7] child1 same,
 *            [8..11] {c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z},
 *            [12],[13] child indices (a leaf child is ~nodeIndex) or, in a leaf
 *            node, the triangle range [begin, end), [14] size (~size in a
 *            leaf), [15] parent index (-1 at the root).
 * Interior nodes occupy [0, num_interior) with the root at 0; leaf nodes
 * occupy [num_interior, num_interior + num_leaf).
 * With layout Quad (N = 4) or Oct (N = 8) a node is HipBVHNodeN<N>
 * (rt/bvh/HipBVHNode.h:14-114), int[8N]: [4i..4i+3] child i {lo.x, hi.x, lo.y,
 * hi.y}; [4(N+i)], [4(N+i)+1] child i lo.z, hi.z; [4(N+i)+2] child i's index
 * (~index for a leaf); [8N-9] child count, [8N-5] size (~size in a leaf),
 * [8N-1] parent; a leaf holds its box in every child slot and its range
 * [begin, end) at [4N+2], [4N+3]. Nodes are numbered breadth first, interior
 * nodes from 0 and leaves after them (BVHConverter::convert). Unused child
 * slots hold child 0's minimum corner as an empty box and child 0's index.
 * woop holds 3 float4 per leaf-ordered reference (rt/bvh/HipBVHKernels.cu:35-65),
 * tri_indices maps a leaf-ordered reference to its scene triangle. */
typedef struct hp_bvh {
    void* nodes;
    void* woop;
    int32_t* tri_indices;
    int64_t num_refs;         /* number of references (= triangles)           */
    int64_t capacity_refs;    /* allocation size in references                */
    int32_t num_interior;     /* filled by hp_bvh_sync                        */
    int32_t num_leaf;         /* filled by hp_bvh_sync                        */
    float scene_box[6];       /* filled by hp_bvh_sync: min xyz, max xyz      */
    float morton_scale[3];    /* filled by hp_bvh_sync: scale used for keys   */
    int32_t method;
    float ct, ci;
    void* impl;               /* library private                              */
    int32_t layout;           /* hp_layout of the nodes                       */
    int32_t node_bytes;       /* 32 * layout                                  */
} hp_bvh;

/* Optional device buffers that receive intermediate results of an LBVH build
 * (for parity tests). Any pointer may be NULL. Sizes: n = num_triangles. */
typedef struct hp_build_taps {
    uint64_t* morton_keys;    /* [n] keys before sorting (always 64-bit)            */
    uint64_t* sorted_keys;    /* [n] keys after sorting                             */
    int32_t* sorted_refs;     /* [n] reference index per sorted position            */
    int32_t* node_parent;     /* [2n-1] binary radix tree before collapse           */
    int32_t* node_left;       /* [2n-1] left child (leaf node j: j-(n-1))           */
    int32_t* node_right;      /* [2n-1] right child (leaf node j: j-(n-1)+1)        */
    float* node_box_min;      /* [2n-1][4] refitted boxes before collapse (w = 0)   */
    float* node_box_max;      /* [2n-1][4]                                           */
    float* scene_box;         /* [6]                                                 */
} hp_build_taps;

typedef struct hp_ctx hp_ctx;

/* ---- context ---------------------------------------------------------- */
hp_status hp_ctx_create(hp_ctx** out, int32_t device);
hp_status hp_ctx_destroy(hp_ctx* ctx);
/* Wait for all work of the context's device; returns HP_ERR_DEVICE_STATUS if a
 * kernel reported an error word since the last check (and clears it). */
hp_status hp_ctx_check(hp_ctx* ctx, void* stream);
const char* hp_last_error(void);
int32_t hp_abi_version(void);
/* Phase timing, the counterpart of HipKernel::launchTimed's per-kernel event
 * times (gpu/HipKernel.cpp:296-325) without host synchronisation: when enabled,
 * build and trace record a CUDA event after every phase on the stream.
 * hp_profile_count / hp_profile_get read the phases of the last enabled call
 * sequence (they synchronise); hp_profile_reset clears them. */
hp_status hp_profile_enable(hp_ctx* ctx, int32_t on);
hp_status hp_profile_reset(hp_ctx* ctx);
int32_t hp_profile_count(hp_ctx* ctx);
hp_status hp_profile_get(hp_ctx* ctx, int32_t i, char* name, int64_t name_size, float* ms);
/* Number of kernels this library has launched from the calling thread. */
int64_t hp_launch_count(void);

/* ---- scene files (host) ------------------------------------------------------
 * A triangle mesh in host memory, allocated by the library (hp_scene_free).
 *   hp_scene_read_bin   BinImporter::importScene   util/BinImporter.cpp:16-84
 *   hp_scene_write_bin  BinExporter::exportScene   util/BinExporter.cpp:14-70
 *                       (zero normals, texture coordinates and material
 *                       indices; no materials or textures)
 *   hp_scene_read_obj   the geometry AssimpImporter::importScene returns for
 *                       an OBJ file (util/AssimpImporter.cpp:20-200): polygons
 *                       as triangle fans, triangles whose box has zero area
 *                       dropped, box = bound of all vertices
 *   hp_scene_normalize  SceneLoader::loadStaticScene (rt/scene/SceneLoader.cpp:
 *                       125-134): v = (v - box.min) * (1 / longest box side)
 *   hp_scene_load       SceneLoader::loadScene + loadStaticScene: path + ".bin"
 *                       if it exists (or path itself if it ends in ".bin"),
 *                       else the OBJ file, whose geometry is then written to
 *                       path + ".bin" when write_cache is set; then normalised. */
typedef struct hp_host_scene {
    float* vertices;          /* [num_vertices][3] */
    int32_t* triangles;       /* [num_triangles][3] */
    int64_t num_vertices;
    int64_t num_triangles;
    float box[6];             /* as stored / computed, before normalisation */
} hp_host_scene;
hp_status hp_scene_read_bin(const char* path, hp_host_scene* out);
hp_status hp_scene_write_bin(const char* path, const hp_host_scene* scene);
hp_status hp_scene_read_obj(const char* path, hp_host_scene* out);
hp_status hp_scene_normalize(hp_host_scene* scene);
hp_status hp_scene_load(const char* path, int32_t write_cache, hp_host_scene* out);
void hp_scene_free(hp_host_scene* scene);

/* ---- build (BVHBuilder) --------------------------------------------------- */
void hp_build_params_default(hp_build_params* p);
/* Build a BVH over mesh m into *out (allocates on first use; reuses the
 * allocation on later builds of the same or smaller size, like
 * BVHBuilder::rebuild). No host synchronisation; capturable in a CUDA graph
 * once out has capacity for the mesh. taps may be NULL. */
hp_status hp_build(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p,
                   hp_bvh* out, const hp_build_taps* taps, void* stream);
/* Synchronise the stream and fill num_interior, num_leaf, scene_box, morton_scale. */
hp_status hp_bvh_sync(hp_ctx* ctx, hp_bvh* bvh, void* stream);
/* Copy the BVH to host memory (any pointer may be NULL): nodes_host receives
 * (num_interior + num_leaf) * 64 bytes, woop_host num_refs * 48 bytes,
 * tri_host num_refs int32. Synchronous; calls hp_bvh_sync first. */
hp_status hp_bvh_download(hp_ctx* ctx, hp_bvh* bvh, void* nodes_host, void* woop_host,
                          int32_t* tri_host, void* stream);
hp_status hp_bvh_free(hp_ctx* ctx, hp_bvh* bvh);
/* Replicating a built BVH into another device's memory (one mesh, its rays
 * split across GPUs): the receiver reserves storage for num_refs references
 * in a layout, the sender's nodes, woop and tri_indices arrays are copied or
 * broadcast into it (for example ncclBroadcast of the three device buffers),
 * and the receiver then records the sender's node counts, scene box and
 * Morton scale (from the sender's hp_bvh after hp_bvh_sync). The reference
 * has no counterpart (HipBVH lives on one device, gpu/HipModule.cpp:19-50).
 * hp_bvh_reserve allocates (or keeps storage of sufficient capacity) and
 * leaves the contents undefined; hp_bvh_set_info is stream-ordered. */
hp_status hp_bvh_reserve(hp_ctx* ctx, hp_bvh* out, int64_t num_refs, int32_t layout);
hp_status hp_bvh_set_info(hp_ctx* ctx, hp_bvh* bvh, int32_t num_interior, int32_t num_leaf,
                          const float* scene_box6, const float* morton_scale3, void* stream);
/* SAH cost as HipBVH::getCost (sum over nodes of ct|ci*size times node area
 * over scene area), computed on the device and summed in a fixed order in
 * double precision, so repeated calls agree bit for bit. Synchronous. */
hp_status hp_bvh_cost(hp_ctx* ctx, const hp_bvh* bvh, double* cost, void* stream);

/* Quality statistics of a built BVH (rt/bvh/HipBVH.cpp:346-442):
 *   sah_cost              HipBVH::getCost
 *   avg_leaf_size         HipBVH::getAvgLeafSize = sum_of_leaf_sizes / num_leaf
 *   leaf_size_histogram   HipBVH::getLeafSizeHistogram: fraction of leaves
 *                         holding s references, s = 0..HP_MAX_LEAF_SIZE_HIST
 *                         (MAX_LEAF_SIZE, rt/bvh/HipBVHKernels.h:13); larger
 *                         leaves are counted in num_leaf only. */
#define HP_MAX_LEAF_SIZE_HIST 32
typedef struct hp_bvh_stats {
    double sah_cost;
    double avg_leaf_size;
    int64_t sum_of_leaf_sizes;
    int32_t num_interior;
    int32_t num_leaf;
    float leaf_size_histogram[HP_MAX_LEAF_SIZE_HIST + 1];
    int32_t pad;
} hp_bvh_stats;
/* One pass over the nodes on the device; synchronous. */
hp_status hp_bvh_stats_get(hp_ctx* ctx, const hp_bvh* bvh, hp_bvh_stats* out, void* stream);

/* Structural validation as HipBVH::validate (rt/bvh/HipBVH.cpp:157-307);
 * *valid = 1 if consistent, else 0 and hp_last_error names the first failed
 * check. Runs on the device with every index bounds-checked; synchronous. */
hp_status hp_bvh_validate(hp_ctx* ctx, const hp_bvh* bvh, const hp_mesh* m,
                          int32_t* valid, void* stream);
/* Refit-only update after vertex moves (HipBVH::update): re-woopify and
 * recompute every node box bottom-up from the mesh's current vertices. */
hp_status hp_refit(hp_ctx* ctx, hp_bvh* bvh, const hp_mesh* m, void* stream);

/* ---- trace (HipTracer) ---------------------------------------------------- */
/* rays: 8 floats per ray {ox, oy, oz, tmin, dx, dy, dz, tmax} (Ray, rt/ray/Ray.h:16-27);
 * results: 4 int32 per ray {triangle id, t bits, u bits, v bits} (RayResult);
 * on a miss only {-1, tmax bits} are written. stats (or NULL): 2 int32 per ray
 * {traversed nodes, tested triangles}. Closest hits break ties in t by the
 * lower triangle id. */
hp_status hp_trace(hp_ctx* ctx, const hp_bvh* bvh, const float* rays, int64_t num_rays,
                   int32_t* results, int32_t* stats, uint32_t flags, void* stream);

/* hp_trace over HOST buffers (HipTracer::trace on a RayBuffer whose rays live
 * in host memory, which the reference's Buffer migrates to the device on use,
 * gpu/Buffer.cpp:437-498): rays_host, results_host and stats_host (or NULL)
 * are host memory, pinned for overlap. The rays go up in chunks of
 * chunk_rays (0: sizes doubling from 262,144 rays to at most 4,194,304 and
 * halving again at the end, so that the first upload and the last download,
 * which nothing overlaps, stay short) on a copy stream while the previous chunk is
 * traced and the one before comes back on another copy stream, through two
 * device staging slots the context keeps; each slot's chunks trace on a
 * stream of their own (after the work already queued on `stream`), so that
 * one chunk's trace fills the SMs that its predecessor's leaves as it drains.
 * A context tuned for sorted tracing sorts each chunk of at least 65,536 rays
 * by 30-bit ray keys, in scratch of its slot. Results are identical
 * to hp_trace's, except that every result record is written in full (a miss
 * reads {-1, tmax bits, 0, 0}). The call is asynchronous on `stream`: the
 * host buffers may be read / are complete once `stream` has synchronised. */
hp_status hp_trace_host(hp_ctx* ctx, const hp_bvh* bvh, const float* rays_host, int64_t num_rays,
                        int32_t* results_host, int32_t* stats_host, uint32_t flags, int64_t chunk_rays,
                        void* stream);

/* Trace in ray Morton order (HipTracer::traceSort, rt/tracer/HipTracer.cpp:109-125;
 * RayBuffer::mortonSort, rt/ray/RayBuffer.cpp:112-131): keys as hp_ray_keys
 * with the reference's [0,1]^3 ray box and `bits` key bits (the reference's
 * default is 30), a stable radix sort, then a traversal whose slot k takes
 * ray order[k]. Results land at each ray's own index, as with hp_trace.
 * order_out (device, num_rays int32, or NULL) receives the ray order. */
hp_status hp_trace_sorted(hp_ctx* ctx, const hp_bvh* bvh, const float* rays, int64_t num_rays,
                          int32_t* results, int32_t* stats, uint32_t flags, int32_t bits,
                          int32_t* order_out, void* stream);

/* ---- ray generation (RayGen, PixelTable) ---------------------------------- */
/* Pixel order of PixelTable::recalculate (rt/ray/PixelTable.cpp:10-80): 8x8
 * blocks in Morton order, pixels swizzled within a block, then the stripes
 * below and to the right. Host memory, width*height entries. */
hp_status hp_pixel_table(int32_t width, int32_t height, int32_t* index_to_pixel);
/* inverse(projection * view) of the reference's Camera (rt/scene/Camera.cpp:95-109)
 * for a camera at `position` looking along `direction` (no roll), vertical
 * field of view fov_deg, aspect width/height; row-major 4x4 into out16. */
hp_status hp_camera_screen_to_world(const float* position, const float* direction, float fov_deg,
                                    int32_t width, int32_t height, float near_plane, float far_plane,
                                    float* out16);
/* Primary rays (RayGen::primary, rt/ray/RayGen.cpp:35-62; generatePrimaryRays,
 * rt/ray/RayGenKernels.cu:106-153): ray k goes through pixel index_to_pixel[k]
 * (device array, or NULL for row-major order) jittered by the Halton point of
 * sample_index, from `position` (host, 3 floats), tmin 0, tmax max_dist.
 * rays: device, width*height rays of 8 floats. */
hp_status hp_gen_primary_rays(hp_ctx* ctx, const float* position, const float* screen_to_world16,
                              int32_t width, int32_t height, float max_dist, int32_t sample_index,
                              const int32_t* index_to_pixel, float* rays, void* stream);
/* Ray Morton key methods (RayBuffer::MortonCodeMethod, rt/ray/RayBuffer.h:20-28;
 * the 64-bit kernels computeMortonCodes*64, rt/ray/RayBufferKernels.cu:492-921,
 * which RayBuffer::computeMortonCodes always uses, RayBuffer.cpp:31-80). */
typedef enum hp_ray_keys_method_e {
    HP_RAY_KEYS_TWO_POINT = 0,   /* origin and a point rayLength along the ray, 13 bits per axis */
    HP_RAY_KEYS_AILA = 1,        /* origin and direction, 13 bits per axis (the default) */
    HP_RAY_KEYS_PARABOLOID = 2,  /* origin 15 bits, direction by dual-paraboloid map */
    HP_RAY_KEYS_OCTAHEDRON = 3,  /* origin 15 bits, direction by octahedral map */
    HP_RAY_KEYS_ORIGIN = 4,      /* origin only, 23 bits per axis */
    HP_RAY_KEYS_COSTA = 5,       /* spherical direction (atan2, acos) first, then origin */
    HP_RAY_KEYS_REIS = 6         /* origin 21 bits, then spherical direction */
} hp_ray_keys_method_e;
/* The context's key method and two-point ray length (RayBuffer::
 * setMortonCodeMethod / setRayLength; defaults Aila and 0.25), used by
 * hp_ray_keys, hp_trace_sorted and a context tuned for sorted tracing. */
hp_status hp_ctx_set_ray_keys(hp_ctx* ctx, int32_t method, float ray_length);
/* Renderer::stringToMortonCodeMethod (rt/renderer/Renderer.cpp:37-52): "aila",
 * "paraboloid", "octahedron", "origin", "costa", "reise"; anything else is the
 * two-point method. */
int32_t hp_ray_keys_method(const char* name);
/* Ray Morton keys by the context's method: the origin normalised to ray_box6
 * (host {min xyz, max xyz}; NULL = [0,1]^3 as the reference), the direction
 * mapped by the method, quantised and interleaved as the reference's 64-bit
 * kernel; the top `bits` of the 64-bit code. keys: device, num_rays uint64. */
hp_status hp_ray_keys(hp_ctx* ctx, const float* rays, int64_t num_rays, const float* ray_box6,
                      int32_t bits, uint64_t* keys, void* stream);

/* ---- adjoint ------------------------------------------------------------ */
/* Scatter dL/d(t,u,v) (3 floats per ray) of closest hits into dL/dvertices
 * (3 floats per vertex, accumulated: the caller zeroes it). results must come
 * from hp_trace on the same bvh, rays and mesh. Misses contribute nothing. */
hp_status hp_trace_adjoint(hp_ctx* ctx, const hp_mesh* m, const float* rays,
                           const int32_t* results, const float* dl_dtuv, int64_t num_rays,
                           float* dl_dvertices, void* stream);

/* ---- tuning ---------------------------------------------------------------- */
/* Launch choices of a context. The first four never change a result: they are
 * the sort's CTA size (its tile), the tracer's persistent CTAs per SM (warps
 * per SM = 4 x that) and shared-memory stack depth, and tracing in ray Morton
 * order. The PLOC radius fields report the schedule hp_autotune measured best;
 * it changes the tree, so it is applied only by the caller (hp_build_params).
 * New: the reference has no tuner. */
typedef struct hp_tune {
    int32_t sort_block;        /* threads per radix-sort CTA: 512 (default) or 256 */
    int32_t trace_ctas_per_sm; /* persistent tracer CTAs of 128 threads per SM; 0 = as many as fit */
    int32_t trace_stack;       /* traversal stack entries per ray kept in shared memory: 8, 16 (default), 32 */
    int32_t trace_sorted;      /* 1: hp_trace traces in ray Morton order (30-bit keys, as hp_trace_sorted) */
    int32_t ploc_radius;       /* hp_autotune: best PLOC radius found (0 = not tuned) */
    int32_t ploc_adaptive;     /* hp_autotune: 1 if the adaptive schedule was best */
    int32_t ploc_max_radius;   /* hp_autotune: the schedule's maximum radius */
    float build_ms;            /* hp_autotune: build time with the chosen settings */
    float trace_ms;            /* hp_autotune: trace time of the ray sample with the chosen settings */
    int32_t reserved[7];
} hp_tune;
#define HP_TUNE_PLOC_RADIUS 1u     /* hp_autotune flag: also compare PLOC radius schedules */
void hp_tune_default(hp_tune* t);
/* Set / read the context's launch choices (validated; HP_ERR_ARG if out of range). */
hp_status hp_ctx_set_tune(hp_ctx* ctx, const hp_tune* t);
hp_status hp_ctx_get_tune(hp_ctx* ctx, hp_tune* t);
/* Time the launch choices on the caller's mesh and rays (a sample of at most
 * 2^21 rays): sort CTA size on the build, then stack depth x CTAs per SM x
 * Morton order on the trace, each by CUDA events (median of three runs). The
 * fastest result-neutral choices are applied to the context and written to
 * *out; with HP_TUNE_PLOC_RADIUS and a PLOC method, the radius schedules
 * {8, 16, 32 fixed; adaptive from 4 up to 64} are also compared by build time
 * plus the sample's trace time scaled to num_rays, and the best is reported
 * in *out (not applied). Synchronous; allocates a temporary BVH and buffers. */
hp_status hp_autotune(hp_ctx* ctx, const hp_mesh* m, const hp_build_params* p, const float* rays,
                      int64_t num_rays, uint32_t flags, hp_tune* out, void* stream);

/* ---- batches of meshes ---------------------------------------------------- */
/* Many independent meshes of uneven size built (LBVH) and traced in a fixed
 * number of launches, replayed from a CUDA graph. New entry points with no
 * counterpart in the reference; each mesh gets exactly the BVH hp_build makes
 * for it. The meshes' device buffers stay owned by the caller and must live
 * as long as the batch. Rays of mesh m occupy rays [offset(m), offset(m+1))
 * of the ray array (hp_batch_ray_offset), in mesh order, 8 floats each;
 * results and stats follow the same order and layout as hp_trace's, with
 * mesh-local triangle ids. Morton bits + ceil(log2(num_meshes)) must be <= 64. */
typedef struct hp_batch hp_batch;
#define HP_BATCH_NO_GRAPH 0x100u   /* flags: launch directly instead of from a CUDA graph */
hp_status hp_batch_create(hp_ctx* ctx, const hp_mesh* meshes, int32_t num_meshes,
                          const int64_t* rays_per_mesh, const hp_build_params* p, hp_batch** out);
hp_status hp_batch_destroy(hp_batch* b);
hp_status hp_batch_info(const hp_batch* b, int32_t* num_meshes, int64_t* num_triangles, int64_t* num_rays);
hp_status hp_batch_ray_offset(const hp_batch* b, int32_t mesh, int64_t* offset);
/* Build every mesh's BVH, trace every ray against its mesh, or both. A CUDA
 * graph needs a non-default stream; it is captured on the first call and again
 * whenever the buffers, flags or the context's scratch arena change. */
hp_status hp_batch_build(hp_ctx* ctx, hp_batch* b, uint32_t flags, void* stream);
hp_status hp_batch_trace(hp_ctx* ctx, hp_batch* b, const float* rays, int32_t* results, int32_t* stats,
                         uint32_t flags, void* stream);
hp_status hp_batch_build_trace(hp_ctx* ctx, hp_batch* b, const float* rays, int32_t* results,
                               int32_t* stats, uint32_t flags, void* stream);
/* A non-owning hp_bvh for mesh m of the batch (for hp_bvh_sync / download /
 * cost / validate / hp_trace); hp_bvh_free on it releases nothing. */
hp_status hp_batch_bvh(hp_batch* b, int32_t mesh, hp_bvh* out);

/* ---- arithmetic ---------------------------------------------------------- */
/* The reference compiles its kernels with -use_fast_math
 * (gpu/HipCompiler.cpp:127-129): its `1.0f / x` in the tracer's ray setup and
 * triangle test (rt/tracer/HipTracerBinKernels.cu:87-89, 219-220) and in the
 * Woop inverse (rcp, util/Math.h:20,368; rt/bvh/HipBVHKernels.cu:12-33) is the
 * approximate quotient, and denormals are flushed to zero. By default this
 * library computes those reciprocals with IEEE round-to-nearest
 * (HP_ARITH_IEEE). HP_ARITH_REFERENCE computes them as the reference's build
 * does, with denormals flushed, so that Woop rows and closest hits match the
 * reference's bit for bit (ties in t still go to the lower triangle id). It
 * applies to hp_build and hp_refit (the Woop rows of every layout) and to the
 * binary-layout tracer (hp_trace, hp_trace_sorted, hp_trace_host); batches
 * and the Quad / Oct tracer keep IEEE arithmetic. Builds are otherwise
 * unchanged (the Morton scale always uses the reference's quotient). */
#define HP_ARITH_IEEE 0
#define HP_ARITH_REFERENCE 1
hp_status hp_ctx_set_arithmetic(hp_ctx* ctx, int32_t mode);

/* ---- primitives ------------------------------------------------------------ */
/* Stable LSD radix sort of (key, value) pairs by key bits [0, bits). key_bytes
 * is 4 or 8. vals_in may be NULL (values are then 0..n-1). Output in keys_out /
 * vals_out (may not alias the inputs). Uses the context's scratch arena. */
hp_status hp_radix_sort(hp_ctx* ctx, const void* keys_in, const int32_t* vals_in,
                        void* keys_out, int32_t* vals_out, int64_t n,
                        int32_t key_bytes, int32_t bits, void* stream);

/* Spins one look-back wait of the context's radix sort passes (hp_radix_sort
 * and every build) makes before it gives up: the wait then records
 * HP_ERR_DEVICE_STATUS for the next hp_ctx_check and the sort goes on with the
 * prefix it has, so its output is not sorted but every write stays inside the
 * output. 0 restores the default, HP_SORT_SPIN_LIMIT_DEFAULT. The reference
 * has no such bound (its sort synchronises the host after every kernel). */
#define HP_SORT_SPIN_LIMIT_DEFAULT 4194304u
hp_status hp_ctx_set_sort_spin_limit(hp_ctx* ctx, uint32_t spins);

/* Checked mode: every entry point verifies what it produced before it
 * returns, at the cost of a host synchronisation per call. hp_build and
 * hp_refit sync the BVH, check its node counts against the reference count
 * and run hp_bvh_validate; hp_radix_sort checks that its output is ordered;
 * hp_trace, hp_trace_host, hp_trace_adjoint and the batch calls return the
 * device error words (traversal stack overflow, index out of range, a bounded
 * wait that gave up) as HP_ERR_DEVICE_STATUS from the call itself instead of
 * from a later hp_ctx_check. On a stream that is being captured into a CUDA
 * graph the checks, which synchronise, are skipped. Off by default; a
 * context created while the environment variable HP_CHECKED is set to a
 * value other than "0" starts with it on. The bounds checks that report into
 * the error words are always compiled in. The reference has no counterpart
 * (it stops the process on the first HIP error, gpu/HipModule.cpp:216-222). */
hp_status hp_ctx_set_checked(hp_ctx* ctx, int32_t on);
int32_t hp_ctx_get_checked(const hp_ctx* ctx);

/* The same sort for callers that must not allocate GPU memory: no context, no
 * cudaMalloc / cudaFree / allocating library call. This entry point has no
 * counterpart in the reference. It serves code that runs where the device
 * memory budget is owned by someone else (a plugin inside a host
 * application that hands it only fixed buffers) or where an allocation's
 * implicit device synchronisation is not allowed (a latency-critical frame
 * loop). Its scratch is a fixed array in the library's device memory, loaded
 * once on every GPU that uses the library and kept until the process exits:
 * at most HP_NOALLOC_SORT_MAX_KEYS keys per call, larger n returns HP_ERR_ARG.
 * The first call on a device looks up that array's device address, so make
 * the first call on each device before any stream capture. That address is
 * cached for the life of the process: it assumes the device's primary
 * context lives as long (after cudaDeviceReset the cached address is stale
 * and this entry point must not be called again). All calls share the one
 * array: calls whose GPU work overlaps (different streams, or several host
 * threads) race; serialise them on one stream. Every call clears the scratch
 * state it needs. device_status (optional, device memory, ONE int32, need
 * not be zeroed) is written by every call, in stream order: 0, or
 * 1 if a bounded wait inside the sort gave up, in which case
 * the output is not sorted. The call returns before the GPU work ends, so
 * without device_status such a give-up goes unreported. */
#define HP_NOALLOC_SORT_MAX_KEYS 262144
hp_status hp_radix_sort_noalloc(const void* keys_in, const int32_t* vals_in,
                                void* keys_out, int32_t* vals_out, int64_t n,
                                int32_t key_bytes, int32_t bits, int32_t* device_status,
                                void* stream);

/* ---- environment files (Environment / AppEnvironment) ------------------- */
typedef struct hp_env hp_env;
hp_status hp_env_create(hp_env** out);      /* registers the reference's options */
hp_status hp_env_destroy(hp_env* env);
/* Parse a block-structured env file; unknown keys and malformed values make
 * the parse fail (HP_ERR_PARSE) like Environment::readEnvFile. */
hp_status hp_env_read_file(hp_env* env, const char* path);
hp_status hp_env_read_string(hp_env* env, const char* text);
/* First value of an option (or its default); HP_ERR_ARG if unknown or unset. */
hp_status hp_env_get_int(const hp_env* env, const char* name, int32_t* value);
hp_status hp_env_get_float(const hp_env* env, const char* name, float* value);
hp_status hp_env_get_bool(const hp_env* env, const char* name, int32_t* value);
hp_status hp_env_get_string(const hp_env* env, const char* name, char* buf, int64_t buf_size);
/* Fill build parameters from the Bvh.* keys with the builders' range checks
 * (out-of-range values keep the default, as the reference setters do). */
hp_status hp_env_build_params(const hp_env* env, hp_build_params* p);

/* ---- synthetic inputs (host memory, deterministic, thread-count independent) */
/* Uniform triangle soup: centre ~ U[0,1]^3, vertex = centre + U[-h,h]^3. */
hp_status hp_gen_uniform_mesh(uint64_t seed, int64_t n, float half_extent,
                              float* vertices, int32_t* triangles);
/* Clustered soup: n_clusters centres ~ U[0,1]^3, triangle i in cluster i % n_clusters,
 * centre = cluster centre + N(0, sigma^2)^3, vertex = centre + U[-h,h]^3. */
hp_status hp_gen_clustered_mesh(uint64_t seed, int64_t n, int32_t n_clusters, float sigma,
                                float half_extent, float* vertices, int32_t* triangles);
/* Heightfield nx*ny vertices on [0,1]x[0,ny/(nx)] ... see implementation notes:
 * domain [0,sx]x[0,sy], z = sum of n_waves sinusoids; 2 triangles per cell. */
hp_status hp_gen_heightfield(uint64_t seed, int32_t nx, int32_t ny, float sx, float sy,
                             int32_t n_waves, float* vertices, int32_t* triangles);
/* Rays aimed at targets: origin ~ U[lo,hi]^3, target ~ U[0,1]^3, tmin 0, tmax inf. */
hp_status hp_gen_rays_targeted(uint64_t seed, int64_t n, float lo, float hi, float* rays);
/* Rays with origin ~ U(box) and direction uniform on the sphere. */
hp_status hp_gen_rays_sphere(uint64_t seed, int64_t n, const float* box6, float* rays);
/* Downward rays on a jittered nx*ny grid over [0,sx]x[0,sy], origin z = z0. */
hp_status hp_gen_rays_grid_down(uint64_t seed, int32_t nx, int32_t ny, float sx, float sy,
                                float z0, float* rays);

#ifdef __cplusplus
}
#endif

#endif /* HIPPIE_B200_H_ */
