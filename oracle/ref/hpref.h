// Launch wrappers around the reference's kernels (one translation unit per
// reference kernel file; see w_*.cu) and the host harness that sequences them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// Occupancy-derived default block size, as HipKernel::getDefaultBlockSize.
int hpref_default_block(const void* kernel);

// w_lbvh.cu
void hpref_set_scene_box(const float* box6);
void hpref_setup_boxes(int n, int* tri_idx, const int* tris, const float* verts, float4* bmin, float4* bmax);
void hpref_morton60(int n, int bits, unsigned long long* keys, int* refs, float4* bmin, float4* bmax);
void hpref_setup_leaves(int n, int* refs0, int* refs1, int* tri0, int* tri1, int* left, int* right,
                        float4* nbmin, float4* nbmax, float4* bmin, float4* bmax);
void hpref_construct60(int n, int* parent, int* left, int* right, unsigned long long* keys);
void hpref_refit(int nodes, int* counters, int* parent, int* left, int* right, float4* nbmin, float4* nbmax);

// w_ploc.cu
void hpref_ploc_neighbours(int clusters, int r, float* dist, int* nbr, float4* nbmin, float4* nbmax, int* nodes);
void hpref_ploc_merge(int clusters, int offset, int* nbr, int* in, int* out, int* parent, int* left, int* right,
                      float4* nbmin, float4* nbmax);
int hpref_ploc_merged(void);
void hpref_ploc_reset(void);
void hpref_ploc_scan_compact(int clusters, int* in, int* out, int* thread_offsets, int* block_offsets);

// w_collapse.cu
void hpref_collapse_sizes(int nodes, int* counters, int* parent, int* left, int* right, int* sizes);
void hpref_collapse_states(int n, float ci, float ct, int* counters, float* costs, int* parent, int* left,
                           int* right, int* sizes, int* states, float4* nbmin, float4* nbmax);
void hpref_collapse_leaf_indices(int n, int* leaf_idx, int* parent, int* states);
void hpref_collapse_invalidate(int n, int* counters, int* leaf_idx, int* parent, int* states);
void hpref_collapse_offsets_begin(void);
void hpref_collapse_offsets(int task_offset, int tasks, int* left, int* right, int* node_idx, int* node_off,
                            int* states);
int hpref_collapse_interiors(void);
int hpref_collapse_leaves(void);
void hpref_collapse_ref_offsets(int nodes, int* states, int* sizes, int* ref_off);
void hpref_collapse_compact(int nodes, int n_int, int* states, int* node_off, int* parent, int* left, int* right,
                            int* sizes, int* ref_off, float4* nbmin, float4* nbmax, void* out_nodes);
void hpref_collapse_reorder(int n, int* left, int* ref_off, int* tri_in, int* tri_out, int* leaf_idx);

// w_atr.cu
void hpref_atr_areas(int nodes, float* areas, float4* nbmin, float4* nbmax);
void hpref_atr_optimize(int n, int treelet, int schedule_size, int dist_size, int gamma, float ci, float ct,
                        float* costs, float* areas, float* dist_mats, int* left, int* right, float4* nbmin,
                        float4* nbmax, int* counters, int* parent, int* subtree_refs, int* schedule, int smem);

// w_hlbvh.cu
void hpref_hl_node_states(int n, int bits, int sah, int* counters, int* parent, int* left, int* right, int* states,
                          unsigned long long* keys);
void hpref_hl_leaf_clusters(int n, int* leaf_cluster, int* parent, int* states);
void hpref_hl_invalidate(int n, int* counters, int* leaf_cluster, int* parent, int* states);
void hpref_hl_set_counter(int v);
int hpref_hl_counter(void);
void hpref_hl_node_offsets(int n, int* offsets, int* states);
void hpref_hl_compact(int n, int* offsets, int* states, int* in_parent, int* in_left, int* in_right, int* out_parent,
                      int* out_left, int* out_right);
void hpref_hl_clusters(int n, int bits, int sah, int* states, int* offsets, int* lbvh_left, int* cluster_nodes,
                       int4* cluster_bins, unsigned long long* keys);
void hpref_hl_reset_bins(int all_bins, float4* bmin, float4* bmax);
void hpref_hl_bin(int tasks, int bins, int clusters, int* cluster_tasks, int* cluster_nodes, int4* cluster_bins,
                  float4* nbmin, float4* nbmax, float4* bmin, float4* bmax);
void hpref_hl_split(int bins, int tasks, int* out_size, int* new_tasks, int* split_idx, int* parent, int* left,
                    int* right, float4* nbmin, float4* nbmax, float4* bmin, float4* bmax, int2* in_q, int2* out_q);
void hpref_hl_distribute(int tasks, int bins, int clusters, int* new_tasks, int* split_idx, int* parent, int* left,
                         int* right, int* cluster_tasks, int* cluster_nodes, int4* cluster_bins, float4* bmin,
                         float4* bmax, int2* in_q);

// w_bvh.cu
void hpref_woopify(int n, int* tri_idx, const int* tris, const float* verts, float4* woop);
float hpref_cost(int nodes, float scene_area, float ct, float ci, void* bin_nodes);

// w_trace.cu
void hpref_trace_launch(int rays, bool any_hit, float4* rays_buf, int4* results, float4* nodes, float4* tris,
                        int2* stats, int* tri_idx);
