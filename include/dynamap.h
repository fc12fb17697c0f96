/*
 * dynamap.h -- C ABI of the B200 rigid-mapping library (libdynamap_b200.so).
 *
 * This is the drop-in boundary for DynaMap's per-frame rigid mapping path:
 * depth ingest -> bilateral filter -> vertex/normal pyramids -> projective
 * point-to-plane (+photometric) Gauss-Newton ICP -> voxel-hashed TSDF
 * allocation + integration -> raycast of the model for the next frame.
 *
 * Every entry point takes plain pointers and sizes, returns a dyn_status and
 * never throws.  Citations name the reference interface each item replaces
 * (paths are relative to the alirezaahmadi/dynamap source tree).
 *
 * Conventions
 *   - Poses are camera-to-world rigid transforms stored as 16 floats in
 *     ROW-major order (m11 m12 m13 m14 m21 ...), the layout of the
 *     reference's device-side float4x4 (include/math/utils_matrix.h:816-839,
 *     built from Eigen at include/builder/builder.cu:102).
 *   - Depth frames are uint16 raw sensor units, row-major rows*cols;
 *     metres = raw / depth_scaler.  0 = invalid.
 *   - RGB frames are uint8 R,G,B interleaved, row-major rows*cols*3.
 *   - "_host" buffers are caller-owned host memory (pageable or pinned);
 *     "_dev" buffers are device pointers on the session's device.
 *   - All calls on one session must be serialised by the caller; different
 *     sessions may be driven from different host threads.
 */
#ifndef DYNAMAP_B200_H
#define DYNAMAP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DYN_ABI_VERSION 1

/* Status codes.  The reference reports failures with printf + return
 * (include/solver/gnSolver/gnSolver.cu:329-343) or silent -1 returns
 * (include/dataStructure/hashTable/hashTable.cu:109); here every call
 * returns one of these. */
typedef enum dyn_status {
  DYN_OK = 0,
  DYN_ERR_INVALID_ARG = 1,
  DYN_ERR_OOM = 2,
  DYN_ERR_BUDGET_EXCEEDED = 3,
  DYN_ERR_HASH_FULL = 4,       /* a bucket overflowed (block not stored) */
  DYN_ERR_HEAP_EXHAUSTED = 5,  /* more blocks requested than num_blocks */
  DYN_ERR_ICP_DIVERGED = 6,
  DYN_ERR_TIMEOUT = 7,
  DYN_ERR_CUDA = 8,
  DYN_ERR_NOT_READY = 9,
  DYN_ERR_NO_DEVICE = 10
} dyn_status;

/* Pinhole sensor.  Replaces DynaMap::rgbdSensor
 * (include/image/sensor/rgbdSensor.h:13-19: rows, cols, f, c, depthScaler). */
typedef struct dyn_sensor {
  uint32_t rows;
  uint32_t cols;
  float fx, fy;          /* rgbdSensor::f */
  float cx, cy;          /* rgbdSensor::c */
  float depth_scaler;    /* raw units per metre (TUM 5000, millimetres 1000) */
} dyn_sensor;

/* TSDF / voxel-hash configuration.  Replaces tsdf::tsdfProperties
 * (include/geometry/tsdf/tsdf.h:19-35) and the keys of
 * config/tsdfParams.yaml (voxelSize, numBuckets, bucketSize, numBlocks,
 * blockSize, maxSDFWeight, truncationDistance, maxSensorDepth,
 * minSensorDepth). */
typedef struct dyn_tsdf_params {
  float voxel_size;           /* metres */
  int32_t num_buckets;
  int32_t bucket_size;        /* slots per bucket, no overflow list */
  int32_t num_blocks;         /* voxel-block pool size (heap) */
  int32_t block_size;         /* voxels per block edge; must be 8 */
  int32_t max_sdf_weight;     /* weight cap, <= 255 (uint8 weight) */
  float truncation_distance;  /* metres */
  float max_sensor_depth;     /* metres */
  float min_sensor_depth;     /* metres */
} dyn_tsdf_params;

/* Gauss-Newton ICP configuration.  Replaces solver::Properties
 * (include/solver/gnSolver/gnSolver.h:47-55) and config/gnOptimParams.yaml
 * (lvlIterationNum[i], lvlScale[i], minIncrement, maxIncrement,
 * regularization, huberConstant).  The fields after huber_constant are
 * additive: the reference hard-codes them at the cited lines. */
typedef struct dyn_gn_params {
  int32_t lvl_iteration_num[3]; /* level i runs lvl_iteration_num[i]-1
                                   iterations (gnSolver.cu:370) */
  int32_t lvl_scale[3];         /* 1, 2, 4 or 8; level order as given */
  int32_t max_iteration;        /* unused by the reference; kept */
  float min_increment;          /* stop when |delta xi| <= this */
  float max_increment;          /* zero the increment if sum(xi) >= this */
  float regularization;         /* damping: A += (reg*max(A)/it) I */
  float huber_constant;         /* parsed, unused (gnSolver.cu:116-119) */
  float color_weight;           /* photometric blend, gnSolver.cu:180 (0) */
  float icp_min_depth;          /* DEPTH_MIN, pyramid.h:16 (0.15) */
  float icp_max_depth;          /* DEPTH_MAX, pyramid.h:15 (2.0) */
  float normal_cos_thresh;      /* |n.ns| gate, gnSolver.cu:108 cos(pi/10) */
  int32_t mode;                 /* builder Mode: 0 frame-to-frame,
                                   1 frame-to-model (raycast target) */
  int32_t compose_left;         /* 1: pose = exp(xi) * pose as at
                                   gnSolver.cu:429; 0: pose = pose * exp(xi) */
} dyn_gn_params;

/* Bilateral filter.  Replaces DynaMap::gaussianKernal
 * (include/image/kernel2D/kernel2D.h:20-43) and config/bilateralFParams.yaml
 * (diameter, sigmaI, sigmaS).  The window is 2*diameter taps per axis
 * (pyramid.cu:250). */
typedef struct dyn_bilateral_params {
  int32_t diameter;
  float sigma_i;   /* range sigma (metres) */
  float sigma_s;   /* spatial sigma (pixels) */
  int32_t enabled; /* 0: ICP uses the unfiltered depth */
} dyn_bilateral_params;

typedef enum dyn_precision {
  DYN_PRECISION_FP32 = 0,   /* 8-byte voxels {r,g,b,w,f32 sdf}: the drop-in */
  DYN_PRECISION_MIXED = 1,  /* f16 sdf + u16 weight, compensated-f32 normal eqns */
  /* DYN_PRECISION_MIXED, and each depth ray allocates only the blocks
   * within the truncation band of its surface point (the reference
   * allocates every block from the camera to the surface,
   * tsdf.cu:346-453): free space farther than a block from any surface is
   * left unobserved instead of carved, which the raycast steps through
   * exactly as it steps through carved free space (one truncation
   * distance per sample).  No counterpart in the reference. */
  DYN_PRECISION_MIXED_BAND = 2
} dyn_precision;

/* One voxel as downloaded.  Same 8-byte layout as geometry::Voxel
 * (include/geometry/geom_Types.h:72-76: uchar3 color, uchar weight,
 * float sdf). */
typedef struct dyn_voxel {
  uint8_t r, g, b;
  uint8_t weight;
  float sdf;
} dyn_voxel;

/* Per-frame counters, read back with dyn_frame_result. */
typedef struct dyn_frame_stats {
  int32_t frame_index;
  int32_t icp_iterations[3];    /* executed iterations per level */
  int32_t icp_inliers[3];       /* correspondences, last iteration per level */
  float icp_rms[3];             /* point-to-plane RMS residual (m) */
  int32_t icp_reset;            /* 1 if the NaN / max_increment guard fired */
  int32_t blocks_total;         /* allocated blocks after this frame */
  int32_t blocks_new;           /* blocks allocated by this frame */
  int32_t blocks_visible;       /* blocks integrated this frame */
  int32_t unique_blocks_probed; /* distinct blocks the rays touched */
  int32_t bucket_full;          /* inserts refused: bucket full */
  int32_t heap_exhausted;       /* inserts refused: no free block */
  int32_t dda_overruns;         /* rays cut at the step limit */
  int32_t raycast_overruns;     /* raycast pixels cut at the step limit */
  double pose_increment[6];     /* final xi = [w; t] of this frame */
} dyn_frame_stats;

typedef struct dyn_session dyn_session;

/* ---- library ---------------------------------------------------------- */
int32_t dyn_abi_version(void);
const char* dyn_status_string(dyn_status s);
/* Fills the defaults of the reference config files (tsdfParams.yaml,
 * gnOptimParams.yaml, bilateralFParams.yaml, cameraParams.yaml) and of
 * include/image/pyramid/pyramid.h. */
dyn_status dyn_default_params(dyn_tsdf_params* tsdf, dyn_gn_params* gn,
                              dyn_bilateral_params* bil, dyn_sensor* sensor);
/* Parses the reference's flat "- key: value" YAML files
 * (config/tsdfParams.yaml, gnOptimParams.yaml, bilateralFParams.yaml,
 * cameraParams.yaml).  Any pointer may be NULL; unknown keys are ignored,
 * missing keys keep the value already in the struct. */
dyn_status dyn_load_yaml(const char* path, dyn_tsdf_params* tsdf,
                         dyn_gn_params* gn, dyn_bilateral_params* bil,
                         dyn_sensor* sensor);
/* Bytes of device memory a session with these parameters holds. */
dyn_status dyn_session_bytes(const dyn_tsdf_params* tsdf,
                             const dyn_sensor* sensor, int32_t precision,
                             size_t* bytes_out);

/* ---- session (builder, include/builder/builder.h:49-117) -------------- */
/* builder::init (builder.cu:11-49) + tsdfVolume::init (tsdf.cu:18) +
 * HashTable::Init (hashTable.cu:41-70).  All device memory is allocated
 * here, once; no call below allocates. */
dyn_status dyn_session_create(const dyn_tsdf_params* tsdf,
                              const dyn_gn_params* gn,
                              const dyn_bilateral_params* bil,
                              const dyn_sensor* sensor, int32_t precision,
                              int32_t device, dyn_session** out);
/* builder::~builder (builder.cu:50-65). */
dyn_status dyn_session_destroy(dyn_session* s);
/* Clears the map and the pose (HashTable::Init semantics, no realloc). */
dyn_status dyn_session_reset(dyn_session* s);

/* Pose of the last processed frame (builder::getCurrentPose, builder.cu:284)
 * and an explicit initial pose (builder::setInitialPose, builder.cu:263). */
dyn_status dyn_session_get_pose(dyn_session* s, float pose_out[16]);
dyn_status dyn_session_set_pose(dyn_session* s, const float pose[16]);

/* builder::buildModelLS (builder.cu:70-139) for one frame: track against
 * the model (or the previous frame in mode 0), integrate, raycast the
 * target for the next frame.  Enqueued; returns before the GPU finishes.
 * Pageable host buffers are copied before return (they may be reused at
 * once); page-locked ones (cudaHostAlloc / cudaHostRegister) are read by
 * the device copy after return and must stay unchanged until the frame's
 * dyn_frame_result.  Two frames may be in flight: submitting frame k+1
 * before reading frame k's result overlaps frame k+1's host->device copy
 * (on the session's copy stream, into a second input slot) with frame k's
 * work; dyn_frame_result returns results in submission order.  A third
 * submit gives up the oldest unread result. */
dyn_status dyn_frame_submit(dyn_session* s, const uint16_t* depth_host,
                            const uint8_t* rgb_host /* nullable */);
/* Same, with the frame already resident on the device. */
dyn_status dyn_frame_submit_device(dyn_session* s, const uint16_t* depth_dev,
                                   const uint8_t* rgb_dev /* nullable */);
/* dyn_frame_submit with an initial estimate of the new camera pose
 * (row-major camera-to-world, e.g. from odometry): tracking starts from
 * the motion it implies relative to the current pose instead of from no
 * motion.  A null hint is dyn_frame_submit.  No counterpart in the
 * reference (its ICP always starts from the previous pose). */
dyn_status dyn_frame_submit_hint(dyn_session* s, const uint16_t* depth_host,
                                 const uint8_t* rgb_host /* nullable */,
                                 const float pose_hint[16] /* nullable */);
/* Waits for the oldest frame in flight; returns its pose and counters
 * (DYN_ERR_NOT_READY when no frame is in flight). */
dyn_status dyn_frame_result(dyn_session* s, float pose_out[16],
                            dyn_frame_stats* stats /* nullable */);

/* builder::buildModelGT (builder.cu:140-160): integrate a frame at a given
 * pose (no tracking), then raycast the target at that pose.  Synchronous. */
dyn_status dyn_integrate_with_pose(dyn_session* s, const uint16_t* depth_host,
                                   const uint8_t* rgb_host /* nullable */,
                                   const float pose[16]);

/* gnSolver::solve (gnSolver.cu:317-438) on caller images: registers the
 * source depth (metres, rows*cols of the session sensor, optional RGB)
 * against the target depth (same size, in the target camera's frame) with
 * the session's pyramid and GN parameters; pose_inout (row-major) is
 * composed with the increment as dyn_gn_params.compose_left says, and the
 * final increment xi = [w; t] is returned.  Uses the session's image and
 * solver buffers only: its map is not touched.  Synchronous. */
dyn_status dyn_solver_solve(dyn_session* s, const float* target_depth_host,
                            const uint8_t* target_rgb_host /* nullable */,
                            const float* source_depth_host,
                            const uint8_t* source_rgb_host /* nullable */,
                            float pose_inout[16], double increment_out[6],
                            dyn_frame_stats* stats /* nullable */);

/* tsdfVolume::GenerateDepth / GenerateRgb (tsdf.cu:527-550; kernels
 * tsdf.cu:471-526) into caller buffers.  'virt' may be NULL for the session
 * sensor; otherwise its rows*cols must not exceed the session sensor's.
 * Synchronous. */
dyn_status dyn_raycast(dyn_session* s, const float pose[16],
                       const dyn_sensor* virt, float* depth_host,
                       uint8_t* rgb_host /* nullable */);

/* dyn_raycast plus the raycast's vertex and normal maps in the camera frame
 * (rgbdImage::getPointCloudXYZ / getNormalsfromVertices, rgbdImage.cu:23-167,
 * applied to the raycast depth with misses as invalid): float4 per pixel,
 * zero where invalid.  Any output may be NULL.  Uses the session's source
 * image buffers as scratch (they are rewritten by the next frame).
 * Synchronous. */
dyn_status dyn_raycast_maps(dyn_session* s, const float pose[16], const dyn_sensor* virt,
                            float* depth_host, float* vertex4_host, float* normal4_host,
                            uint8_t* rgb_host);

/* Number of allocated blocks (HashTable::GetNumAllocatedBlocks,
 * hashTable.cu:165). */
dyn_status dyn_num_blocks(dyn_session* s, int64_t* n_out);

/* HashTable::FindHashEntry (hashTable.cu:136-150) for n block coordinates
 * (coords[3*i..]): the heap index of each block, or -1 where none is
 * allocated.  Waits for the session's frames. */
dyn_status dyn_find_blocks(dyn_session* s, const int32_t* coords, int64_t n,
                           int32_t* heap_index_out);
/* Copies every allocated block: coords_out[3*i..] = block coordinate
 * (HashEntry::position, hashTable.h:22), voxels_out[512*i..] = its voxels in
 * the reference's x-major order (VoxelBlock::at, geom_Types.h:116-119).
 * Blocks come in heap order (the order dyn_extract_mesh walks them and
 * eviction hands them out).  voxels_out may be NULL. */
dyn_status dyn_download_blocks(dyn_session* s, int32_t* coords_out,
                               dyn_voxel* voxels_out, int64_t capacity,
                               int64_t* n_out);

/* Triangle mesh of the volume over the box between 'lower' and 'upper'
 * (tsdfVolume::ExtractMesh, tsdf.cu:551-560; MeshExtractor::ExtractMesh,
 * meshExtractor.cu:364-407): the reference's cells (|upper - lower| / vs * 2
 * per axis from 'lower', corners at +-vs/2, each sampled by trilinear
 * interpolation that gives up at an unobserved voxel), vertices by its edge
 * interpolation coloured by the cell's centre voxel, triangles from a
 * generated marching-cubes table.  18 floats per triangle: three vertices
 * {x, y, z, r, g, b}, colour in 0..1.  *n_out = the number of triangles;
 * min(*n_out, capacity) are written, in a fixed order (allocated blocks in
 * heap order, cells x-fastest within a block).  triangles_host may be NULL
 * (count only).  Synchronous.  DYN_ERR_INVALID_ARG for a box that is not
 * finite or has 2^24 or more cells along an axis. */
dyn_status dyn_extract_mesh(dyn_session* s, const float lower[3], const float upper[3],
                            float* triangles_host, int64_t capacity, int64_t* n_out);

/* ---- block eviction and streaming ----------------------------------------
 * The reference has HashTable::DeleteBlock (hashTable.cu:112-134) but never
 * calls it; these remove blocks between frames so that a session stays
 * inside its memory, can hand them to the host first, and put blocks back.
 * Removal keeps the heap dense (survivors move into the freed slots, the
 * rest is cleared), so dyn_download_blocks afterwards lists exactly the
 * survivors and the next frames allocate from the freed space.  The
 * removed blocks' coordinates and voxels (the 8-byte form of
 * dyn_download_blocks) go to coords_out / voxels_out (either may be NULL),
 * at most 'capacity' of them, in heap order; *n_out = the blocks removed.
 * Synchronous; not for a session whose frames a batch or server is running
 * at the same time. */
/* Blocks the allocation has not touched in the last frame or the
 * max_age_frames frames before it (0: keep only the last frame's). */
dyn_status dyn_evict_blocks(dyn_session* s, int32_t max_age_frames, int32_t* coords_out,
                            dyn_voxel* voxels_out, int64_t capacity, int64_t* n_out);
/* The blocks at n_coords block coordinates (coords[3*i..]); coordinates
 * without a block are ignored, repeats count once. */
dyn_status dyn_delete_blocks(dyn_session* s, const int32_t* coords, int64_t n_coords,
                             int32_t* coords_out, dyn_voxel* voxels_out, int64_t capacity,
                             int64_t* n_out);
/* n blocks (coordinates, 512 voxels each in the 8-byte form) into the
 * volume, as touched by the last frame; a block whose key is present is
 * left as it is.  counts_out = {placed, already present, bucket full, heap
 * exhausted}.  The mixed form stores sdf / truncation as f16 and the weight
 * as u16 (the round trip through dyn_download_blocks is exact for weights
 * up to 255). */
dyn_status dyn_upload_blocks(dyn_session* s, const int32_t* coords, const dyn_voxel* voxels,
                             int64_t n, int64_t counts_out[4]);

/* Internal images of the last frame, for inspection and parity tests.
 * which: 0 raw depth (f32, level 0), 1 filtered depth (f32, level 0),
 *        2 source depth pyramid level L (f32), 3 source vertices level L
 *        (float4), 4 source normals level L (float4), 5 target depth level L,
 *        6 target vertices L, 7 target normals L, 8 target rgb (u8x3, level 0),
 *        9 source intensity level L (f32), 10 target intensity level L (f32).
 * 'level' is the pyramid level (0 = full resolution). */
dyn_status dyn_debug_image(dyn_session* s, int32_t which, int32_t level,
                           void* host_out, size_t bytes);

/* ---- measurement --------------------------------------------------------
 * The reference times frames with gettimeofday around the whole loop
 * (src/dynaMap.cpp:220,295-299, include/utils/utils_Timer.h:15-33); these
 * expose device-side timing of each stage instead. */
enum {
  DYN_STAGE_INGEST = 0,     /* u16 -> metres (+ intensity) */
  DYN_STAGE_BILATERAL = 1,
  DYN_STAGE_SOURCE_MAPS = 2, /* pyramid + normal maps of the new frame */
  DYN_STAGE_ICP = 3,         /* all GN iterations + pose update */
  DYN_STAGE_ALLOCATE = 4,
  DYN_STAGE_VISIBLE = 5,
  DYN_STAGE_INTEGRATE = 6,
  DYN_STAGE_RAYCAST = 7,
  DYN_STAGE_TARGET_MAPS = 8, /* pyramid + normal maps of the raycast */
  DYN_STAGE_FRAME = 9,       /* whole frame, first to last kernel */
  DYN_NUM_STAGES = 10
};
/* The session's CUDA stream (a cudaStream_t), for callers that record their
 * own events around dyn_frame_submit. */
dyn_status dyn_session_stream(dyn_session* s, void** stream_out);
/* enable != 0: every frame records a CUDA event between stages (inside the
 * frame's graph); dyn_frame_result accumulates the stage times. */
dyn_status dyn_session_profile(dyn_session* s, int32_t enable);
/* Accumulated device milliseconds per stage since the last reset and the
 * number of frames they cover; reset != 0 clears the accumulators. */
dyn_status dyn_session_stage_times(dyn_session* s, double ms_out[DYN_NUM_STAGES],
                                   int64_t* frames_out, int32_t reset);
/* Kernels one frame launches (nodes of the frame graph). */
dyn_status dyn_session_kernels_per_frame(dyn_session* s, int32_t* n_out);
/* Bytes each submitted frame copies device -> host (pose, solver state and
 * counters read back by dyn_frame_result). */
size_t dyn_frame_d2h_bytes(void);

/* ---- stage entry points on caller device buffers ----------------------
 * These run one stage of the path on caller-owned device memory, on
 * 'stream' (a cudaStream_t, NULL = legacy default stream), and return once
 * the work is enqueued (no host synchronisation) unless noted. */

/* pyramid::bilateralFilter (pyramid.cu:253-282 -> applyBilateralFilter
 * :213-233).  Out-of-image and invalid (<= 0) taps are skipped; an invalid
 * centre stays 0. */
dyn_status dyn_bilateral_filter(const float* depth_dev, float* out_dev,
                                uint32_t rows, uint32_t cols,
                                const dyn_bilateral_params* p, void* stream);

/* rgbdImage::getPointCloudXYZ + getNormalsfromVertices (rgbdImage.cu:23-49,
 * :126-167) for one level: vertex (x,y,z,1 | 0 if invalid) and normal
 * (nx,ny,nz,0 | 0 if invalid) as float4 per pixel. */
dyn_status dyn_depth_to_maps(const float* depth_dev, const dyn_sensor* level,
                             float* vertex4_dev, float* normal4_dev,
                             void* stream);

/* The same maps for a depth image in host memory (rgbdImage's own buffers,
 * as the reference's managed images are): depth_host and the float4 maps
 * are rows*cols host arrays; vertex4_host may be NULL.  The device buffers
 * are taken and released inside the call, on the calling thread's default
 * stream; synchronous. */
dyn_status dyn_depth_to_maps_host(const float* depth_host, const dyn_sensor* level,
                                  float* vertex4_host, float* normal4_host);

/* The 6x6 normal equations of one ICP iteration (buildNLSKernel,
 * gnSolver.cu:26-196): for source pixels (depth, normals, intensity) and a
 * target (depth, normals, intensity, all on the same level sensor), under
 * the transform T (row-major float[16]) computes
 *   out[0..20]  upper triangle of A = sum J^T J (row-major, i<=j)
 *   out[21..26] -sum J r   (the reference's acc_b)
 *   out[27]     sum r^2 (point-to-plane residuals)
 *   out[28]     number of correspondences
 * in a fixed-order reduction (FP32 per pixel, FP64 across thread blocks).
 * intensity pointers may be NULL when gn->color_weight == 0.
 * Synchronous: out_host is filled on return. */
dyn_status dyn_icp_normal_equations(
    const float* src_depth_dev, const float* src_normal4_dev,
    const float* src_intensity_dev, const float* tgt_depth_dev,
    const float* tgt_normal4_dev, const float* tgt_intensity_dev,
    const dyn_sensor* level, const dyn_gn_params* gn, const float T[16],
    double out_host[29], void* stream);

/* The same normal equations for callers that cannot allocate device memory
 * (a host that reserves a fixed GPU-memory budget up front and forbids later
 * cudaMalloc, e.g. a real-time executor running the tracker in its control
 * loop).  No counterpart in the reference: this entry point exists for such
 * callers.  Its scratch is one fixed file-scope device array (~465 KiB per
 * GPU that loads the library, held until exit) instead of allocated
 * buffers; it calls no cudaMalloc/cudaFree.  Levels up to 2,097,152 pixels
 * (1920x1080 fits); larger ones return DYN_ERR_INVALID_ARG.  All calls on a
 * device share the array: calls whose GPU work overlaps race and must be
 * serialised by the caller.  The first call on a device does a one-time
 * set-up (looks up the array's address with that device current); make it
 * before any stream capture.  That address is kept until exit: do not use
 * the library across a cudaDeviceReset of the device.  Levels are checked
 * as dyn_icp_normal_equations checks them.  Results equal
 * dyn_icp_normal_equations' to rounding (the partial sums are grouped
 * differently).  Synchronous. */
dyn_status dyn_icp_normal_equations_noalloc(
    const float* src_depth_dev, const float* src_normal4_dev,
    const float* src_intensity_dev, const float* tgt_depth_dev,
    const float* tgt_normal4_dev, const float* tgt_intensity_dev,
    const dyn_sensor* level, const dyn_gn_params* gn, const float T[16],
    double out_host[29], void* stream);

/* The bounded grid-wide barrier of the persistent ICP (one cooperative
 * launch per frame walks every level and iteration; its blocks meet at one
 * barrier per iteration), run alone on 'device': 'blocks' blocks, all
 * resident at once, wait for blocks + missing arrivals.  DYN_OK when the
 * barrier completes; DYN_ERR_TIMEOUT when its bounded wait (half a second)
 * runs out, as it must when missing > 0 -- the blocks give up and return,
 * the device stays usable; DYN_ERR_INVALID_ARG when the blocks cannot all
 * be resident (refused before anything runs).  A frame whose ICP barrier
 * timed out reports DYN_ERR_TIMEOUT.  For tests of that failure path; no
 * counterpart in the reference. */
dyn_status dyn_barrier_selftest(int32_t device, int32_t blocks, int32_t missing);

/* ---- multi-session stepping ---------------------------------------------
 * No counterpart in the reference (its builder drives one stream).
 *
 * dyn_sessions_submit: one frame for each of n sessions, each replayed as
 * that session's own frame graph on its own stream (the streams overlap on
 * the device).  Frames are host pointers, copied before return; results are
 * read with dyn_frame_result per session. */
dyn_status dyn_sessions_submit(dyn_session* const* sessions, int32_t n,
                               const uint16_t* const* depth_host,
                               const uint8_t* const* rgb_host /* nullable */);

/* dyn_batch: a fixed set of sessions on one device stepped together.  Each
 * stage of a frame is ONE kernel launch over all members (a member uses
 * only its own part of the grid, so its results are bit-identical to
 * stepping it alone) and the whole frame is one CUDA graph on the batch's
 * stream, followed by one device->host copy of every member's results.
 * Members may differ in sensor size, volume, parameters and precision.
 * While a session belongs to a batch its frames go only through the batch
 * (dyn_frame_submit, dyn_frame_submit_device, dyn_integrate_with_pose and
 * dyn_solver_solve return DYN_ERR_INVALID_ARG); its other calls (pose,
 * raycast, download, images) first wait for the batch's work in flight.
 * Destroying a member makes the batch refuse further frames. */
typedef struct dyn_batch dyn_batch;
dyn_status dyn_batch_create(dyn_session* const* sessions, int32_t n, dyn_batch** out);
dyn_status dyn_batch_destroy(dyn_batch* b);
/* One frame per member: depth_host[i] (rows_i x cols_i u16), rgb_host
 * nullable, or rgb_host[i] nullable per member.  Host buffers may be
 * reused when the call returns. */
dyn_status dyn_batch_submit(dyn_batch* b, const uint16_t* const* depth_host,
                            const uint8_t* const* rgb_host);
/* The same with device buffers (read on the batch's stream). */
dyn_status dyn_batch_submit_device(dyn_batch* b, const uint16_t* const* depth_dev,
                                   const uint8_t* const* rgb_dev);
/* Waits for the frame; poses_out n x 16 floats, stats_out n entries and
 * status_out n entries are each nullable.  Returns the first member error
 * (DYN_ERR_HEAP_EXHAUSTED / DYN_ERR_HASH_FULL) or DYN_OK. */
dyn_status dyn_batch_result(dyn_batch* b, float* poses_out, dyn_frame_stats* stats_out,
                            dyn_status* status_out);
dyn_status dyn_batch_size(dyn_batch* b, int32_t* n_out);
dyn_status dyn_batch_stream(dyn_batch* b, void** stream_out);
dyn_status dyn_batch_profile(dyn_batch* b, int32_t enable);
dyn_status dyn_batch_stage_times(dyn_batch* b, double ms_out[DYN_NUM_STAGES],
                                 int64_t* frames_out, int32_t reset);
dyn_status dyn_batch_kernels_per_frame(dyn_batch* b, int32_t* n_out);
/* Autotuner: over the next frames the batch times each candidate launch
 * shape -- integration grid 592 / 1184 / 2368 CTAs x raycast tile 16x16 /
 * 32x8 / 8x8 pixels, shapes that change no result -- for
 * frames_per_candidate frames (the first of each not counted; at least 2),
 * then keeps the fastest.  0 restores the default shape.  No counterpart in
 * the reference. */
dyn_status dyn_batch_autotune(dyn_batch* b, int32_t frames_per_candidate);
/* done: tuning finished; the shape in use (ray_tile: 0 16x16, 1 32x8, 2 8x8). */
dyn_status dyn_batch_tuning(dyn_batch* b, int32_t* done, int32_t* integrate_ctas,
                            int32_t* ray_tile);

/* dyn_server: the serving loop's device side.  Sessions are admitted while
 * their device bytes (dyn_session_bytes, with a mixed session's colour only
 * when its photometric weight is nonzero) fit the budget and a slot is free
 * (else DYN_ERR_BUDGET_EXCEEDED: retry when a session has been released),
 * and released at any time.  dyn_server_push copies a host frame into the
 * session's pinned staging buffers; dyn_server_step then runs one frame of
 * every session that has one waiting, all of them fused into one launch per
 * stage on the server's stream, and returns without waiting: frames pushed
 * while a step runs join the next step (continuous batching).  A session's
 * results are the same whichever sessions share its steps.
 * dyn_server_result waits for the last step that processed the slot and
 * returns its latest result.  A served session takes frames only through
 * the server; its other calls (raycast, download, pose, images) wait for
 * the server's work in flight.  Calls on one server are not thread-safe.
 * The server reserves its whole budget at creation: the first budget/258
 * bytes hold the batch visible list (one entry for every block the rest of
 * the budget can hold: a block costs at least 2,064 bytes), the rest is
 * carved into sessions.  It also makes its sessions' streams ahead of time
 * (a pool of up to 64, more on demand, reused after release), so neither
 * admission nor a step allocates device memory or creates a stream. */
typedef struct dyn_server dyn_server;
typedef struct {
  size_t budget_bytes;   /* device bytes for sessions and the batch visible list
                            (0: 90% of free memory) */
  int32_t max_sessions;  /* slots (0: 256) */
  int32_t device;
} dyn_server_params;
typedef struct {
  size_t budget_bytes;
  size_t used_bytes;
  int32_t capacity;
  int32_t sessions;
  int64_t steps;       /* steps submitted */
  int64_t steps_done;  /* steps completed on the device (they complete in order) */
  int64_t frames;
} dyn_server_usage;
dyn_status dyn_server_create(const dyn_server_params* p, dyn_server** out);
dyn_status dyn_server_destroy(dyn_server* sv);
dyn_status dyn_server_admit(dyn_server* sv, const dyn_tsdf_params* tsdf,
                            const dyn_gn_params* gn, const dyn_bilateral_params* bil,
                            const dyn_sensor* sensor, int32_t precision,
                            const float pose0[16] /* nullable */, int32_t* slot_out);
dyn_status dyn_server_release(dyn_server* sv, int32_t slot);
/* DYN_ERR_NOT_READY: the slot's previous frame has not been stepped yet.
 * Page-locked buffers (cudaHostAlloc / cudaHostRegister) are not copied
 * here: the next dyn_server_step reads them, so they must stay unchanged
 * until that step has completed (dyn_server_poll / dyn_server_result).
 * Other buffers are copied into the session's staging buffers and may be
 * reused when the call returns. */
dyn_status dyn_server_push(dyn_server* sv, int32_t slot, const uint16_t* depth_host,
                           const uint8_t* rgb_host /* nullable */);
dyn_status dyn_server_step(dyn_server* sv, int32_t* n_out /* frames in the step */);
dyn_status dyn_server_poll(dyn_server* sv, int32_t slot, int32_t* ready_out);
dyn_status dyn_server_result(dyn_server* sv, int32_t slot, float pose_out[16],
                             dyn_frame_stats* stats);
dyn_status dyn_server_sync(dyn_server* sv);
dyn_status dyn_server_session(dyn_server* sv, int32_t slot, dyn_session** out);
dyn_status dyn_server_info(dyn_server* sv, dyn_server_usage* out);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* DYNAMAP_B200_H */
