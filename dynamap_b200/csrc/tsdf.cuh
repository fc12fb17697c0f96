// tsdf.cuh -- voxel-hashed TSDF: allocation, visibility, integration, raycast.
#pragma once
#include "common.cuh"
#include "icp.cuh"

namespace dyn {

struct VolumeDev {
  Entry* entries;                 // num_buckets * bucket_size
  unsigned long long* block_keys; // key of each heap index
  dyn_voxel* voxels;              // num_blocks * 512, x-major per block
  int* visible;                   // heap indices of this frame's visible blocks
  Counters* cnt;
  DTsdf t;
};

void launch_volume_clear(const VolumeDev& v, cudaStream_t st);
// AllocateFromDepthKernel (tsdf.cu:346-453) for 'depth' seen from the
// session pose; blocks touched are stamped with the pose's frame number.
void launch_allocate(const VolumeDev& v, const float* depth, const DSensor& s,
                     const PoseState* ps, cudaStream_t st);
// Frustum test of every allocated block (tsdf.cu:283-300), compacted.
void launch_visible(const VolumeDev& v, const DSensor& s, const PoseState* ps,
                    cudaStream_t st);
// IntegrateScanKernel body (tsdf.cu:301-341) for the visible blocks.
void launch_integrate(const VolumeDev& v, const float* depth, const uint8_t* rgb,
                      const DSensor& s, const PoseState* ps, cudaStream_t st);
// GenerateDepthKernel / GenerateRgbKernel (tsdf.cu:471-526).  pose_override
// (device float[16]) replaces the session pose when non-null.
void launch_raycast(const VolumeDev& v, const DSensor& s, const PoseState* ps,
                    const float* pose_override, float* depth_out, uint8_t* rgb_out,
                    cudaStream_t st);
// Download helpers: block coordinates of heap indices [0, n).
void launch_block_coords(const VolumeDev& v, int n, int* coords, cudaStream_t st);

}  // namespace dyn
