/*
 * dynoracle.h -- CPU oracle for the rigid mapping path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * in libdynamap_b200.so: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm call it, nothing in the product does.
 *
 * It restates the reference kernels serially on the CPU, function by
 * function (citations in dynoracle.cpp), with the defect fixes the CUDA path
 * also applies.  Built with -ffp-contract=off so every float operation is a
 * single IEEE-rounded operation in source order: the FP32 instantiation
 * reproduces the reference's own FP32 arithmetic, and a second
 * instantiation runs the same algorithm in FP64 (the FP64 oracle used for
 * ATE / SDF error).
 *
 * All images are row-major.  Poses are row-major float[16] camera-to-world.
 */
#ifndef DYNORACLE_H
#define DYNORACLE_H

#include <stdint.h>
#include "../include/dynamap.h"

#ifdef __cplusplus
extern "C" {
#endif

/* counters[] layout shared by allocate / integrate / raycast */
enum {
  DYO_C_NEW_BLOCKS = 0,    /* blocks allocated by the call */
  DYO_C_BUCKET_FULL = 1,   /* AllocateBlock returned -1 */
  DYO_C_HEAP_EXHAUSTED = 2,
  DYO_C_DDA_OVERRUNS = 3,
  DYO_C_VISIBLE = 4,       /* blocks passing the frustum test */
  DYO_C_REHASH_MISMATCH = 5, /* integration: world round trip left the voxel */
  DYO_C_RAYCAST_OVERRUNS = 6,
  DYO_C_UNIQUE_PROBED = 7, /* distinct blocks visited by allocation rays */
  DYO_C_N = 8
};

void dyo_set_threads(int n);
int dyo_get_threads(void);

/* HashTable::Hash, hashTable.cu:152-163 (returns the first slot index). */
int32_t dyo_hash(int32_t x, int32_t y, int32_t z, int32_t num_buckets,
                 int32_t bucket_size);

/* The DDA of AllocateFromDepthKernel (tsdf.cu:346-453) for one ray: writes
 * up to max_out visited block coordinates (x,y,z triples) and returns how
 * many were visited (negative: the step cap cut the ray). */
int32_t dyo_dda_blocks(const float start[3], const float point[3], float trunc,
                       float block_size, int32_t cap, int32_t* out_xyz,
                       int32_t max_out);
/* Voxel::mergeVoxel (geom_Types.h:79-103) on one voxel: rgbw[4], sdf in/out. */
void dyo_merge_voxel(uint8_t rgbw[4], float* sdf, float new_sdf,
                     const uint8_t new_rgb[3], int32_t new_w, int32_t max_w);

/* Level sensor for a pyramid scale (1, 2, 4, 8). */
void dyo_level_sensor(const dyn_sensor* s, int32_t scale, dyn_sensor* out);

/* ---- images (FP32) ---- */
void dyo_depth_from_raw(const uint16_t* raw, int64_t n, float scaler,
                        float* out);
void dyo_bilateral(const float* src, float* dst, int32_t rows, int32_t cols,
                   const dyn_bilateral_params* p);
void dyo_downsample_depth(const float* src, int32_t rows, int32_t cols,
                          float* dst);
void dyo_intensity(const uint8_t* rgb, int64_t n, float* out);
void dyo_downsample_intensity(const float* src, int32_t rows, int32_t cols,
                              float* dst);
void dyo_maps(const float* depth, const dyn_sensor* level, float* vertex4,
              float* normal4);
void dyo_icp_normal_equations(const float* src_depth, const float* src_n4,
                              const float* src_i, const float* tgt_depth,
                              const float* tgt_n4, const float* tgt_i,
                              const dyn_sensor* level, const dyn_gn_params* gn,
                              const float T[16], double out[29]);
/* The same terms as the reference's buildNLSKernel accumulates them on one
 * thread (gnSolver.cu:192-193): FP32 sums of the full 6x6 A and of -b in
 * pixel order.  Returns the number of pixels with a correspondence. */
int64_t dyo_icp_normal_equations_refsum(const float* src_depth, const float* src_n4,
                                        const float* src_i, const float* tgt_depth,
                                        const float* tgt_n4, const float* tgt_i,
                                        const dyn_sensor* level, const dyn_gn_params* gn,
                                        const float T[16], float A_out[36], float b_out[6]);
/* gnSolver::solve's loop on full-resolution images with those sums
 * (gnSolver.cu:340-430): the final increment xi from zero. */
void dyo_gn_solve_refsum(const float* src_depth, const float* src_n4, const float* tgt_depth,
                         const float* tgt_n4, const dyn_sensor* level, const dyn_gn_params* gn,
                         double inc_out[6]);
/* float4x4::getInverse, utils_matrix.h:970-1086 */
void dyo_inverse4(const float m[16], float out[16]);
/* closed-form SE(3) exponential of xi = [w; t] (double), row-major */
void dyo_se3_exp(const double xi[6], double out[16]);
/* 6x6 LDL^T solve of A x = b (double) */
int dyo_ldlt_solve6(const double A[36], const double b[6], double x[6]);

/* ---- volume (FP32 faithful, or FP64 when fp64 != 0) ---- */
void* dyo_volume_create(const dyn_tsdf_params* p, int32_t fp64);
void dyo_volume_destroy(void* v);
void dyo_volume_allocate(void* v, const float* depth, const dyn_sensor* s,
                         const float pose[16], int64_t counters[DYO_C_N]);
void dyo_volume_integrate(void* v, const float* depth, const uint8_t* rgb,
                          const dyn_sensor* s, const float pose[16],
                          int64_t counters[DYO_C_N]);
void dyo_volume_raycast(void* v, const float pose[16], const dyn_sensor* s,
                        float* depth_out, uint8_t* rgb_out,
                        int64_t counters[DYO_C_N]);
int64_t dyo_volume_num_blocks(void* v);
/* MeshExtractor::ExtractMesh over the box [lo, hi] up to its vertices
 * (meshExtractor.cu:22-214, 364-407): {x, y, z, r, g, b} of every vertex its
 * triangles use, per grid cell in grid order (FP32 volumes; -1 otherwise). */
int64_t dyo_mesh_vertices(void* v, const float lo[3], const float hi[3], float* out,
                          int64_t cap);
/* The mesh of the same cells with this project's marching-cubes table
 * (dynamap_b200/csrc/mc_tables.h): 18 floats per triangle. */
int64_t dyo_mesh_triangles(void* v, const float lo[3], const float hi[3], float* out,
                           int64_t cap);
/* sdf_out: float (fp32 volume) or double (fp64 volume) per voxel; voxels in
 * x-major order.  Any output may be NULL. */
int64_t dyo_volume_download(void* v, int32_t* coords, uint8_t* rgbw,
                            void* sdf_out, int64_t capacity);
/* The inverse for FP32 volumes: blocks allocated in the order given, voxels
 * set (rgbw and sdf as dyo_volume_download writes them).  Returns the blocks
 * placed (fewer when one does not fit), -1 for an FP64 volume. */
int64_t dyo_volume_upload(void* v, const int32_t* coords, const uint8_t* rgbw,
                          const float* sdf, int64_t n);

/* ---- full per-frame pipeline (builder::buildModelLS with fixes) ---- */
void* dyo_session_create(const dyn_tsdf_params* t, const dyn_gn_params* g,
                         const dyn_bilateral_params* b, const dyn_sensor* s,
                         int32_t fp64);
void dyo_session_destroy(void* s);
void dyo_session_set_pose(void* s, const float pose[16]);
void dyo_session_get_pose(void* s, float pose[16]);
void dyo_session_get_pose_f64(void* s, double pose[16]);
void dyo_session_frame(void* s, const uint16_t* depth, const uint8_t* rgb,
                       float pose_out[16], dyn_frame_stats* stats);
void dyo_session_integrate_with_pose(void* s, const uint16_t* depth,
                                     const uint8_t* rgb, const float pose[16]);
void* dyo_session_volume(void* s);
/* which/level as dyn_debug_image (fp32 sessions only) */
int dyo_session_image(void* s, int32_t which, int32_t level, void* out,
                      int64_t bytes);

#ifdef __cplusplus
}
#endif
#endif
