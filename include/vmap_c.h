/*
 * vmap_c.h - C ABI of the B200 voxel-hashing TSDF library (libvmap_b200.so).
 *
 * Drop-in boundary for xingruiyang/VoxelMapping. The reference exposes a C++
 * pimpl class (include/vmapping.h:10-27) over templated CUDA launchers
 * (src/device_functions.h:11-66); this header flattens that surface into plain
 * functions over an opaque map handle so any FFI (ctypes, cgo, JNI, N-API) can
 * bind it. include/vmapping.h (this repository) rebuilds the reference's class
 * on top of these functions.
 *
 * Conventions
 *  - Poses are camera-to-world, row-major 4x4 doubles; the library composes and
 *    inverts them in FP64 and hands FP32 copies to the kernels.
 *  - Device pointers (`_dev`) must be CUDA device memory; `_host` pointers host
 *    memory (pinned for asynchronous copies). Pitches are in bytes.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    All calls are asynchronous on that stream unless documented otherwise.
 *    The fuse / render / mesh / batch-step path never synchronises; the calls
 *    that do are marked at their declaration: vmap_create / vmap_destroy,
 *    vmap_get_stats, vmap_polygonize_host, the host-buffer variants, the block
 *    exports, the snapshot calls and the batch reconfiguration calls.
 *  - Errors: every call returns a vmap_status. Conditions detected on the GPU
 *    (pool or hash table full, coordinates out of range, mesh buffer full) are
 *    accumulated as sticky flags read by vmap_get_stats. Nothing calls exit().
 *  - Not thread-safe per map; distinct maps may be driven from distinct
 *    threads and streams.
 */
#ifndef VMAP_C_H
#define VMAP_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VMAP_ABI_VERSION 1

typedef enum vmap_status {
    VMAP_OK = 0,
    VMAP_ERR_INVALID_ARG = 1,
    VMAP_ERR_CUDA = 2,          /* a CUDA runtime call failed (see vmap_last_error) */
    VMAP_ERR_OUT_OF_MEMORY = 3, /* device or host allocation failed              */
    VMAP_ERR_POOL_FULL = 4,     /* voxel-block pool exhausted                    */
    VMAP_ERR_HASH_FULL = 5,     /* probe limit reached in the block hash table   */
    VMAP_ERR_RANGE = 6,         /* block coordinate outside +-2^20               */
    VMAP_ERR_BUFFER_FULL = 7,   /* mesh output buffer too small                  */
    VMAP_ERR_NO_DEVICE = 8      /* no CUDA device / wrong architecture           */
} vmap_status;

/* sticky device-side error flags (vmap_stats.error_flags) */
#define VMAP_FLAG_POOL_FULL 1u
#define VMAP_FLAG_HASH_FULL 2u
#define VMAP_FLAG_RANGE 4u
#define VMAP_FLAG_BUFFER_FULL 8u
#define VMAP_FLAG_BAD_SNAPSHOT 16u /* a loaded snapshot held an invalid or repeated block key */
#define VMAP_FLAG_STEP_STALLED 32u /* a persistent batch step saw no progress for 2 s and stopped: that step's
                                     * maps and outputs are incomplete */

/* Voxel storage formats. REF is the reference's Voxel (int16 TSDF x32767,
 * uint8 weight, map_struct.h:17-21); F32 is the plain single-precision map;
 * F16 / I16 are the reduced-precision formats with uint16 weights. */
typedef enum vmap_voxel_format {
    VMAP_VOXEL_REF = 0, /* int16 tsdf, uint8 weight   : 4 B/voxel, 3 used (+3 colour) */
    VMAP_VOXEL_F32 = 1, /* float tsdf, float weight   : 8 B/voxel (+3 colour) */
    VMAP_VOXEL_F16 = 2, /* half tsdf, uint16 weight   : 4 B/voxel (+3 colour) */
    VMAP_VOXEL_I16 = 3  /* int16 tsdf, uint16 weight  : 4 B/voxel (+3 colour) */
} vmap_voxel_format;

typedef enum vmap_depth_type {
    VMAP_DEPTH_F32 = 0, /* float metres (reference GpuMat CV_32FC1)        */
    VMAP_DEPTH_U16 = 1  /* uint16 scaled by depth_scale (e.g. 0.001 = mm)  */
} vmap_depth_type;

typedef struct vmap_config {
    /* camera: reference VoxelMapping(int w, int h, const Matrix3f& K) */
    int width, height;
    float fx, fy, cx, cy;
    /* map: reference CreateMap(int numEntries, int numVoxels, float voxelSize) */
    int num_entries;          /* hash entries requested (>= 0; must fit 4 * num_buckets) */
    int num_blocks;           /* voxel-block pool capacity ("numVoxels")        */
    float voxel_size;         /* metres, >= 1e-4                                */
    /* extensions (0 selects the reference default) */
    int num_buckets;          /* 0: int(0.9 * num_blocks) as the reference       */
    float truncation;         /* 0: 4 * voxel_size; at most 1024 * voxel_size   */
    int voxel_format;         /* vmap_voxel_format                              */
    int max_weight;           /* 0: 255                                         */
    int with_color;           /* keep uint8x3 colour per voxel                  */
    int raycast_mode;         /* 0: z-range bounded march (default), 1: full march from 0.1 m */
} vmap_config;

typedef struct vmap_stats {
    uint32_t allocated_blocks;  /* blocks in use                                 */
    uint32_t capacity_blocks;
    uint32_t visible_blocks;    /* visible blocks of the last fuse (numVisBlock) */
    uint32_t error_flags;       /* VMAP_FLAG_* (sticky until vmap_clear_errors)  */
    uint32_t failed_allocs;     /* allocations refused because the pool was full */
    uint32_t last_triangles;    /* triangles found by the last polygonize (unclamped) */
    uint64_t pool_bytes;        /* device bytes of the voxel pool                */
    uint64_t device_bytes;      /* all device bytes owned by the map            */
} vmap_stats;

typedef struct vmap_map vmap_map;

/* ---- lifetime ------------------------------------------------------------ */
/* VoxelMapping(w,h,K) + CreateMap (vmapping.cpp:57-75, map_struct.cu:44-66):
 * allocates the hash table, block pool and work buffers on the current device
 * and resets them. Synchronous. */
vmap_status vmap_create(const vmap_config* cfg, vmap_map** out);
/* Maps in caller-owned device memory (no counterpart in the reference): a
 * server that keeps many maps resident and swaps them in and out places them
 * in memory it manages, so creating and destroying a map allocates and frees
 * no device memory. vmap_required_bytes gives the size for a configuration;
 * vmap_create_in builds the map inside device_mem (256-byte aligned, at
 * least that many bytes) and resets it asynchronously on `stream`. The
 * memory must stay valid until vmap_destroy, which then frees only what the
 * map allocated itself (host-call staging, mesh buffers) and does not
 * synchronise the device: the caller first finishes the work on the map. */
vmap_status vmap_required_bytes(const vmap_config* cfg, uint64_t* bytes);
vmap_status vmap_create_in(const vmap_config* cfg, void* device_mem, uint64_t bytes, void* stream,
                           vmap_map** out);
/* ~VoxelMapping / MapStruct::release (map_struct.cu:68-79). Synchronous. */
vmap_status vmap_destroy(vmap_map* map);
/* VoxelMapping::reset / MapStruct::reset (map_struct.cu:29-42): empties the
 * map, keeps the allocations. */
vmap_status vmap_reset(vmap_map* map, void* stream);
vmap_status vmap_get_config(const vmap_map* map, vmap_config* out);

/* ---- fusion -------------------------------------------------------------- */
/* VoxelMapping::FuseDepth (vmapping.cpp:162 -> FuseImage, depth_fusion.cu:199-301):
 * allocate blocks along each depth ray, select visible blocks, update
 * TSDF/weight. depth_dev has the map's width x height. */
vmap_status vmap_fuse_depth(vmap_map* map, const void* depth_dev, int depth_type, size_t depth_pitch,
                            float depth_scale, const double pose[16], void* stream);
/* VoxelMapping::FuseDepthAndImage (vmapping.cpp:167, FuseDepthAndImage
 * depth_fusion.cu:383-488): as above plus colour (uint8x3 per pixel, blended
 * 0.7 old + 0.3 new). Requires with_color. */
vmap_status vmap_fuse_depth_rgb(vmap_map* map, const void* depth_dev, int depth_type, size_t depth_pitch,
                                float depth_scale, const uint8_t* rgb_dev, size_t rgb_pitch,
                                const double pose[16], void* stream);
/* Host-buffer variant (the reference's FuseDepthAndImage takes cv::Mat):
 * copies depth (and rgb, may be NULL) into device staging, then fuses. */
vmap_status vmap_fuse_host(vmap_map* map, const void* depth_host, int depth_type, float depth_scale,
                           const uint8_t* rgb_host, const double pose[16], void* stream);
/* CheckVisibleBlocks (depth_fusion.cu:494-539): visible-block selection at a
 * pose; count readable through vmap_get_stats. */
vmap_status vmap_check_visible_blocks(vmap_map* map, const double pose[16], void* stream);

/* ---- raycast ------------------------------------------------------------- */
/* VoxelMapping::RenderScene (vmapping.cpp:83-104; ProjectRenderingBlocks
 * ray_tracing.cu:171-234 + RenderScene :403-437) fused with computeNormal
 * (image_proc.cu:95-104): vertex map (float4, camera frame, w = 1, all-NaN on
 * a miss) and, if nmap_dev != NULL, normal map (float4, all-NaN where
 * undefined). */
vmap_status vmap_render_scene(vmap_map* map, const double pose[16], float* vmap_dev, size_t vmap_pitch,
                              float* nmap_dev, size_t nmap_pitch, void* stream);
/* Host-buffer variant: results copied into host buffers (w*h*4 floats each,
 * nmap_host may be NULL). Asynchronous for pinned memory. */
vmap_status vmap_render_scene_host(vmap_map* map, const double pose[16], float* vmap_host, float* nmap_host,
                                   void* stream);
/* computeNormal (image_proc.h:11, image_proc.cu:74-104) on any float4 map. */
vmap_status vmap_compute_normal(const float* vmap_dev, size_t vmap_pitch, float* nmap_dev, size_t nmap_pitch,
                                int width, int height, void* stream);
/* renderScene (image_proc.h:10, image_proc.cu:8-72): Phong shading of vertex
 * + normal maps into RGBA8. */
vmap_status vmap_render_phong(const float* vmap_dev, size_t vmap_pitch, const float* nmap_dev,
                              size_t nmap_pitch, uint8_t* rgba_dev, size_t rgba_pitch, int width, int height,
                              void* stream);

/* ---- pipelined host frames (no counterpart in the reference, whose host
 * path copies, computes and copies back one frame at a time). Enqueues one
 * frame: its depth (and colour) are copied from host memory to one of two
 * staging sets on an internal copy stream, fused and, when vmap_host is not
 * NULL, rendered on `stream`, and the vertex (and normal) maps copied to host
 * memory on a second internal copy stream. Returns at once; consecutive frames
 * overlap their copies with each other's kernels. The host buffers must stay
 * untouched until vmap_host_wait(map, stream) and then a synchronisation of
 * `stream`: after vmap_host_wait, work on `stream` follows every copy of the
 * frames enqueued so far. Pinned host buffers make the copies asynchronous. */
typedef struct vmap_host_frame {
    const void* depth_host;  /* width x height, packed                        */
    int depth_type;          /* vmap_depth_type                               */
    float depth_scale;       /* uint16 -> metres                              */
    const uint8_t* rgb_host; /* uint8x3 packed, or NULL                       */
    double pose[16];         /* camera-to-world, row-major                    */
    float* vmap_host;        /* float4 vertex map out, or NULL (fuse only)    */
    float* nmap_host;        /* float4 normal map out, or NULL                */
} vmap_host_frame;
vmap_status vmap_frame_host_async(vmap_map* map, const vmap_host_frame* frame, void* stream);
vmap_status vmap_host_wait(vmap_map* map, void* stream);

/* ---- meshing ------------------------------------------------------------- */
/* Polygonize (marching_cubes.cu:251-305): marching cubes over all allocated
 * blocks. Writes at most max_tris triangles (9 floats each for verts and
 * norms, world metres); the unclamped count goes to *n_tris_dev (device
 * uint32, may be NULL) and to vmap_stats.last_triangles. With verts_dev NULL
 * the call only counts; otherwise a count above max_tris sets
 * VMAP_FLAG_BUFFER_FULL. */
vmap_status vmap_polygonize(vmap_map* map, float* verts_dev, float* norms_dev, uint32_t max_tris,
                            uint32_t* n_tris_dev, void* stream);
/* VoxelMapping::Polygonize (vmapping.cpp:119-132, 182): mesh into library-owned
 * device buffers, copied to library-owned host buffers; *verts / *norms point
 * at them until the next call. Synchronous. Returns the triangle count in
 * *n_tris (clamped to the buffer). */
vmap_status vmap_polygonize_host(vmap_map* map, const float** verts, const float** norms, uint32_t* n_tris,
                                 void* stream);
/* GetSurfacePoints (marching_cubes.cu:314-344, vmapping.cpp:134-147): triangle
 * centroids, 3 floats each. */
vmap_status vmap_surface_points(const float* verts_dev, uint32_t n_tris, float* points_dev, void* stream);

/* ---- batches (no counterpart in the reference, which drives one map per call)
 * A batch fuses and raycasts many independent maps per step: frame i goes into
 * maps[i], which is then raycast at the same pose. Every stage is one launch
 * covering all maps; the ray marcher is one persistent launch draining a
 * device-side queue of pixel tiles from every map. On a non-default stream the
 * first two steps record the step as CUDA graphs that later steps replay (the
 * per-map descriptors are refreshed by one pinned-memory copy per step).
 * Maps keep their own sizes, cameras, voxel sizes and pools; all maps of a
 * batch share one voxel format. A map may belong to several batches but only
 * one step may use it at a time. */
typedef struct vmap_batch vmap_batch;
/* A NULL depth_dev skips the map's fusion this step (rgb_dev must then be
 * NULL), a NULL vmap_dev its render (nmap_dev must then be NULL); with both
 * NULL the map is idle for the step. */
typedef struct vmap_batch_frame {
    const void* depth_dev;   /* map-sized depth image or NULL (no fusion)    */
    int depth_type;          /* vmap_depth_type                              */
    size_t depth_pitch;      /* bytes, 0 = packed                            */
    float depth_scale;       /* uint16 -> metres                             */
    const uint8_t* rgb_dev;  /* uint8x3 or NULL (no colour this step)        */
    size_t rgb_pitch;
    double pose[16];         /* camera-to-world, row-major                   */
    float* vmap_dev;         /* float4 vertex map out (16-byte aligned) or NULL */
    size_t vmap_pitch;
    float* nmap_dev;         /* float4 normal map out or NULL                */
    size_t nmap_pitch;
} vmap_batch_frame;

#define VMAP_MAX_BATCH 256
vmap_status vmap_batch_create(vmap_map* const* maps, int n_maps, vmap_batch** out);
/* A batch of n_slots empty slots for maps of one voxel format. Slots are
 * filled and emptied between steps with vmap_batch_set_map (NULL empties a
 * slot); the recorded graphs stay valid, so a server can swap maps in and
 * out of a long-lived batch. An empty slot's frame must have all pointers
 * NULL. Calling vmap_batch_set_map on a batch made by vmap_batch_create
 * synchronises the device once and records its graphs again. */
vmap_status vmap_batch_create_slots(int n_slots, int voxel_format, vmap_batch** out);
vmap_status vmap_batch_set_map(vmap_batch* batch, int slot, vmap_map* map);
vmap_status vmap_batch_destroy(vmap_batch* batch);
/* frames: n_maps entries. Asynchronous on `stream`; may block only until the
 * step before last has copied its descriptors. */
vmap_status vmap_batch_step(vmap_batch* batch, const vmap_batch_frame* frames, void* stream);
/* Test of the persistent step's bounded wait (no counterpart in the
 * reference): stages `frames` as vmap_batch_step does, then runs the step as
 * the persistent launch with one task-ring entry reserved and never written,
 * so no warp can take work. After stall_ms (1 .. 10000) without progress every
 * warp raises VMAP_FLAG_STEP_STALLED in every map of the batch and the launch
 * ends; the maps are left mid-step (reset them). Asynchronous on `stream`;
 * never captured into the batch's graphs. */
vmap_status vmap_batch_stall_probe(vmap_batch* batch, const vmap_batch_frame* frames, uint32_t stall_ms,
                                   void* stream);

/* ---- launch shapes (no counterpart in the reference, which hard-codes its
 * grids). Every stage's grid in CTAs per SM; each kernel strides over its work
 * items, so any shape gives the same results and only the time changes.
 * 0 in a field selects the library default (alloc 8, visibility 2, fuse 16,
 * zrange 4, normals 8, mesh 8; raycast 0 = as many CTAs as fit on an SM, the
 * ray marcher being persistent). Values above 64 (tile orders above 2) are
 * refused. Setting a batch's shapes synchronises the device and records its
 * graphs again. */
typedef struct vmap_launch_config {
    int alloc_ctas_per_sm;
    int visibility_ctas_per_sm;
    int fuse_ctas_per_sm;
    int zrange_ctas_per_sm;
    int raycast_ctas_per_sm;
    int normals_ctas_per_sm;
    int mesh_ctas_per_sm;
    /* order in which the ray marcher hands out each image's pixel tiles:
     * 0 = default (bottom rows first), 1 = top rows first, 2 = alternating
     * from both ends. Tiles are independent, so only the time changes: the
     * slowest tiles are best started first. */
    int raycast_tile_order;
    /* ray-marcher tile: a warp marches a tile of 32 neighbouring rays,
     * raycast_tile_width pixels wide (4, 8 or 16; 0 = 8) and 32 / width
     * high; raycast_threads_per_cta is 128 or 256 (0 = 256). Only the time
     * changes. */
    int raycast_tile_width;
    int raycast_threads_per_cta;
    /* how vmap_batch_step runs a batch: 1 = one launch per stage (six, replayed
     * as a CUDA graph); 2 = one persistent launch whose warps take the items of
     * every map's stages from a device-side queue, each map's next stage
     * opening as soon as its previous one finishes; 0 = the default (1). Only
     * the time changes. Single maps always use the stage launches; the
     * persistent launch uses raycast_ctas_per_sm for its grid and 256 threads
     * per CTA. */
    int batch_schedule;
} vmap_launch_config;
vmap_status vmap_get_launch_config(const vmap_map* map, vmap_launch_config* out);
vmap_status vmap_set_launch_config(vmap_map* map, const vmap_launch_config* cfg);
vmap_status vmap_batch_get_launch_config(const vmap_batch* batch, vmap_launch_config* out);
vmap_status vmap_batch_set_launch_config(vmap_batch* batch, const vmap_launch_config* cfg);

/* ---- inspection (no counterpart in the reference: it reports no counters,
 * and its SafeCall, src/cuda_utils.h:11-26, ends the process on a CUDA
 * error while capacity failures pass silently) -------------------------------- */
/* Synchronises `stream`, then reads the device counters. */
vmap_status vmap_get_stats(vmap_map* map, void* stream, vmap_stats* out);
vmap_status vmap_clear_errors(vmap_map* map, void* stream);
/* Asynchronous copy of the raw device counters (16 x uint32: [0] blocks
 * handed out, may exceed capacity; [1] visible blocks; [2] error flags;
 * [3] triangles; [4] refused allocations) to dst (device or pinned host
 * memory), ordered on `stream`; for monitoring without a synchronisation. */
vmap_status vmap_copy_counters(vmap_map* map, uint32_t* dst, void* stream);
/* Dense export of the allocated blocks in pool order (also the snapshot
 * format): coords int32 x3 per block, tsdf float x512 (dequantised), weight
 * float x512, rgb uint8 x3x512 (may be NULL). Voxel index x + 8y + 64z.
 * Buffers are host memory sized for max_blocks. Synchronous. */
vmap_status vmap_export_blocks(vmap_map* map, int32_t* coords, float* tsdf, float* weight, uint8_t* rgb,
                               uint32_t max_blocks, uint32_t* n_blocks, void* stream);

/* ---- snapshots (no counterpart in the reference; its nearest operations are
 * reset/release, map_struct.cu:29-79). A snapshot is the map's used blocks in
 * pool order plus their keys: enough to evict a map from the GPU (to pinned
 * host memory) and bring it back, or to checkpoint and resume it. Loading
 * rebuilds the hash table, so the target map may have a different number of
 * buckets; it needs the same voxel format, colour setting, voxel size,
 * truncation and weight cap, and capacity for the blocks. A loaded map gives
 * bit-identical fusion, raycast and mesh results to the map it was saved from.
 *
 * Layout (little-endian): this 64-byte header, at keys_offset n_blocks uint64
 * keys (block x, y, z as 21-bit two's-complement fields at bits 42, 21 and 0),
 * at pool_offset (a multiple of 256) n_blocks blocks of block_bytes each, in the
 * pool layout [tsdf/weight word x512][r x512][g x512][b x512] (voxel x + 8y + 64z;
 * colour planes only with colour). */
typedef struct vmap_snapshot_header {
    char magic[8];          /* "VMAPSNAP"                                   */
    uint32_t version;       /* 1                                            */
    uint32_t header_bytes;  /* 64                                           */
    int32_t voxel_format;
    int32_t with_color;
    uint32_t block_bytes;   /* vmap_block_bytes(voxel_format, with_color)   */
    uint32_t n_blocks;
    float voxel_size;
    float truncation;
    int32_t max_weight;
    uint32_t error_flags;   /* sticky flags of the saved map                */
    uint64_t keys_offset;
    uint64_t pool_offset;
} vmap_snapshot_header;

/* Writes the snapshot to dst (host memory, pinned or not, or device memory).
 * *bytes receives the snapshot size; with dst NULL nothing is written (a size
 * query), and a capacity below the size fails with VMAP_ERR_INVALID_ARG.
 * Synchronous: returns once dst holds the snapshot. */
vmap_status vmap_snapshot_save(vmap_map* map, void* dst, uint64_t capacity, uint64_t* bytes, void* stream);
/* Replaces the map's content by the snapshot at src (host or device memory,
 * `bytes` long). Synchronous: src may be reused on return. Invalid or
 * mismatched snapshots fail with VMAP_ERR_INVALID_ARG and leave the map as it
 * was; a snapshot whose keys do not fit the target's hash table fails with
 * VMAP_ERR_HASH_FULL (the map is then reset). */
vmap_status vmap_snapshot_load(vmap_map* map, const void* src, uint64_t bytes, void* stream);

/* Block export that allocates nothing. No counterpart in the reference.
 *
 * Same output as vmap_export_blocks for the blocks [first, first + count) in
 * pool order: count <= VMAP_EXPORT_STATIC_MAX_BLOCKS; *n_blocks receives how
 * many exist from `first` on. It is for callers that must not call cudaMalloc
 * or cudaFree once running: loops under a no-allocation policy (an allocation
 * can stall or fail mid-run), plugins whose host owns all device memory.
 * vmap_export_blocks stages through device buffers it allocates on
 * every call; this entry point stages through one fixed device array of
 * VMAP_EXPORT_STATIC_MAX_BLOCKS blocks (about 1.4 MiB) that every GPU loading
 * the library holds until the process exits.
 *  - count > VMAP_EXPORT_STATIC_MAX_BLOCKS is rejected with
 *    VMAP_ERR_INVALID_ARG (text in vmap_last_error); loop over `first`.
 *  - The map's device must be the current device (else
 *    VMAP_ERR_INVALID_ARG); the array's device address is looked up on
 *    every call.
 *  - All calls share the one array: calls whose work overlaps on the GPU (other
 *    threads, streams or maps at the same time) race. Each call overwrites what
 *    it uses, so nothing needs clearing between calls.
 *  - Synchronises `stream` (it reads the block count first) and returns
 *    after the host buffers are filled, so it cannot be captured. */
#define VMAP_EXPORT_STATIC_MAX_BLOCKS 256
vmap_status vmap_export_blocks_static(vmap_map* map, uint32_t first, uint32_t count, int32_t* coords, float* tsdf,
                                      float* weight, uint8_t* rgb, uint32_t* n_blocks, void* stream);

/* ---- stage timing (no counterpart in the reference, which has no timers) --
 * When enabled, every kernel launch of the map is bracketed by CUDA events on
 * the caller's stream; vmap_timing_read synchronises on them and returns the
 * summed device time and launch count per stage since the last read. */
typedef enum vmap_stage {
    VMAP_STAGE_ALLOC = 0,      /* block allocation along depth rays     */
    VMAP_STAGE_VISIBILITY = 1, /* visible-block selection               */
    VMAP_STAGE_FUSE = 2,       /* TSDF / weight / colour update         */
    VMAP_STAGE_ZRANGE = 3,     /* per-tile depth bounds                 */
    VMAP_STAGE_RAYCAST = 4,    /* ray marching                          */
    VMAP_STAGE_NORMALS = 5,    /* normal map                            */
    VMAP_STAGE_MESH = 6,       /* marching cubes                        */
    VMAP_NUM_STAGES = 7
} vmap_stage;
/* max_records: event pairs to keep (0 disables timing). */
vmap_status vmap_timing_enable(vmap_map* map, uint32_t max_records);
vmap_status vmap_timing_read(vmap_map* map, double ms[VMAP_NUM_STAGES], uint32_t launches[VMAP_NUM_STAGES]);

/* ---- utilities ----------------------------------------------------------- */
/* The library's pose inverse (FP64, affine), exposed for parity tests; it
 * replaces the reference's camToWorld.inverse() in float
 * (src/depth_fusion.cu:251, src/ray_tracing.cu:414). */
void vmap_pose_inverse(const double pose[16], double inv[16]);
/* hash (map_struct.h:104-109), exposed for parity tests. */
int vmap_block_hash(int x, int y, int z, int n_buckets);
/* The same hash evaluated on the GPU by the code the hash table uses, for n
 * block coordinates (xyz_dev: n x 3 int32, device) into out_dev (n int32). */
vmap_status vmap_block_hash_device(const int32_t* xyz_dev, uint32_t n, int n_buckets, int32_t* out_dev,
                                   void* stream);
/* Bytes per voxel block for a format. */
size_t vmap_block_bytes(int voxel_format, int with_color);
const char* vmap_status_string(vmap_status s);
/* Text of the last CUDA error seen by this thread. */
const char* vmap_last_error(void);
int vmap_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* VMAP_C_H */
