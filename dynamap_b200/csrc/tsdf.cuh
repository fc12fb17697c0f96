// tsdf.cuh -- voxel-hashed TSDF: allocation, visibility, integration, raycast.
// The per-frame stages run as fused launches over a table of sessions
// (sessdev.cuh); the raycast also has a one-session form for
// tsdfVolume::GenerateDepth / GenerateRgb.
#pragma once
#include "common.cuh"
#include "icp.cuh"

namespace dyn {

struct VolumeDev {
  Entry* entries;                 // num_buckets * bucket_size
  unsigned long long* block_keys; // key of each heap index
  dyn_voxel* voxels;              // FP32 form: num_blocks * 512, x-major per block
  unsigned* vox16;                // mixed form: {f16 sdf | u16 weight << 16} per voxel
  uchar4* colors;                 // mixed form: r,g,b per voxel (null: no colour kept)
  int fp16;                       // 1: mixed-precision voxels (vox16 [+ colors])
  Counters* cnt;
  DTsdf t;
  // Free-space summaries per heap index, kept for the mixed form (null in
  // the FP32 form, whose raycast evaluates every sample, and with band
  // allocation, which allocates no free space to step through): nonsat = voxels
  // that are observed and not saturated, kept exact by the integration;
  // freecell = 1 when every voxel a trilinear cell keyed in the block can
  // read (the block and its seven upper neighbours, missing neighbours
  // included) is unobserved or saturated, so the raycast's interpolated sdf
  // there is the truncation distance.  freecell may be 0 where it could be
  // 1, never the reverse.  A mixed voxel is saturated when its f16 value is
  // exactly 1 (free space); an FP32 voxel (the upload's count, for a volume
  // that keeps summaries) when sdf >= sat_lo, the truncation distance to
  // within 1e-6 relative.  free_ok: sat_lo >= vs, so a saturated sample
  // never ends a march (flags are set only then).
  int* nonsat;
  unsigned char* freecell;
  float sat_lo;
  int free_ok;
};

void launch_volume_clear(const VolumeDev& v, cudaStream_t st);
// GenerateDepthKernel / GenerateRgbKernel (tsdf.cu:471-526).  pose_override
// (device float[16]) replaces the session pose when non-null.
void launch_raycast(const VolumeDev& v, const DSensor& s, const PoseState* ps,
                    const float* pose_override, float* depth_out, uint8_t* rgb_out,
                    cudaStream_t st);
// Download helpers: block coordinates of heap indices [0, n).
void launch_block_coords(const VolumeDev& v, int n, int* coords, cudaStream_t st);
// Heap index (or -1) of each of n block coordinates (x, y, z triples).
void launch_find_blocks(const VolumeDev& v, const int* coords, int n, int* ptr_out,
                        cudaStream_t st);

}  // namespace dyn
