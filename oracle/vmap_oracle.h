/*
 * CPU oracle for the voxel-hashing TSDF pipeline (fuse / raycast / normals /
 * marching cubes). TEST INFRASTRUCTURE ONLY: the product never links or calls
 * this code; tests, the smoke check and the CPU-baseline leg of the benchmark
 * use it as the checker and as the timed CPU baseline.
 *
 * It restates the algorithm of xingruiyang/VoxelMapping:
 *   allocation        src/depth_fusion.cu:32-59   (CreateBlockLineTracingFunctor)
 *   visibility        include/map_struct.h:204-244 + src/depth_fusion.cu:82-126
 *   TSDF update       src/depth_fusion.cu:148-196 (+ colour :328-380)
 *   raycast           src/ray_tracing.cu:272-400
 *   normal map        src/image_proc.cu:74-93
 *   marching cubes    src/marching_cubes.cu:52-242
 *   coordinate math   include/map_struct.h:72-202
 *
 * Two arithmetic modes:
 *   ORC_FP32 - the reference's single-precision arithmetic. Where nvcc's default
 *              FMA contraction fuses a multiply into an add in the reference
 *              (Eigen's coefficient-wise products, running averages), this code
 *              calls fmaf() at the same place; everything else is compiled with
 *              -ffp-contract=off. TSDF storage is quantised exactly like the
 *              selected voxel format (int16 x32767 for the reference's Voxel).
 *   ORC_FP64 - the same algorithm in double precision with unquantised storage:
 *              the accuracy oracle.
 *
 * Parity pinning: the reference's marching-cubes tables are loaded from the
 * golden fixture parsed out of the reference (tests/golden/mc_tables.json) and
 * the constants are checked against the ones parsed from the reference
 * headers. The floating-point arithmetic itself is unpinned: the reference
 * needs Eigen and OpenCV-with-CUDA, neither of which exists here, so it cannot
 * be built or run to produce fixtures.
 */
#ifndef VMAP_ORACLE_H
#define VMAP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FP32 = 0, ORC_FP64 = 1 };
/* stored TSDF / weight formats (FP32 mode only; FP64 stores doubles) */
enum { ORC_STORE_REF = 0, /* int16 x32767 + uint8 weight (reference Voxel) */
       ORC_STORE_F32 = 1, /* float + float weight                          */
       ORC_STORE_F16 = 2, /* IEEE half + uint16 weight                     */
       ORC_STORE_I16 = 3  /* int16 x32767 + uint16 weight                  */ };

typedef struct orc_config {
    int width, height;       /* camera image size                       */
    float fx, fy, cx, cy;    /* pinhole intrinsics                      */
    int num_blocks;          /* voxel-block pool capacity               */
    float voxel_size;        /* metres                                  */
    float truncation;        /* mu, metres (reference: 4 * voxel_size)  */
    int precision;           /* ORC_FP32 / ORC_FP64                     */
    int storage;             /* ORC_STORE_*                             */
    int max_weight;          /* weight cap (reference: 255)             */
    int with_color;          /* fuse uint8x3 colour                     */
} orc_config;

typedef struct orc_map orc_map;

/* Tables: tri_table is the reference's triTable[256][16] (-1 terminated). */
void orc_set_mc_tables(const int* tri_table_256x16);

orc_map* orc_create(const orc_config* cfg);
void orc_destroy(orc_map* m);
void orc_reset(orc_map* m);
void orc_set_threads(int n);
int orc_get_threads(void);

/* Fuse one frame. depth: float metres, row-major width*height (NaN or out of
 * [0.1, 5] = invalid). rgb: uint8x3 row-major or NULL. pose: camera-to-world
 * row-major 4x4 (double). Returns the visible-block count (reference
 * numVisBlock) or -1 on error. *n_new receives blocks allocated this frame,
 * *n_failed allocation attempts that failed because the pool is full. */
int orc_fuse(orc_map* m, const float* depth, const uint8_t* rgb, const double pose[16],
             int* n_new, int* n_failed);

/* Allocation only (reference K3), for block-set parity tests. */
int orc_allocate(orc_map* m, const float* depth, const double pose[16], int* n_failed);

/* Raycast at pose into vmap (width*height*4 floats, camera frame, x=NaN on a
 * miss). Returns the number of hits. */
int orc_raycast(orc_map* m, const double pose[16], float* vmap);

/* Unique allocated blocks the last orc_raycast read (U of the raycast's
 * algorithmic bytes: U x 512 voxels are all the voxel data rays can touch). */
int orc_last_raycast_blocks(const orc_map* m);

/* Unique allocated blocks the last fused frame's allocation samples touched
 * (A of the fused frame's algorithmic bytes). */
int orc_last_alloc_blocks(const orc_map* m);

/* The reference build's arithmetic probe shapes (oracle/ref_harness.cu)
 * through this oracle's FP32 helpers: in 20 floats, out 4 floats per item. */
void orc_probe(int which, const float* in, int n, float* out);

/* Reference computeNormal on a width*height float4 vertex map. Pixels in the
 * last row/column, or with a NaN neighbour, come out NaN. */
void orc_compute_normal(const float* vmap, int width, int height, float* nmap);

/* Phong preview of vertex + normal maps into RGBA8 (reference renderScene). */
void orc_render_phong(const float* vmap, const float* nmap, int width, int height, uint8_t* rgba);

/* Marching cubes over all allocated blocks. verts/norms: 9 floats per
 * triangle (may be NULL to count only). Returns the triangle count (not
 * clamped); writes at most max_tris triangles, in block-allocation order. */
long orc_polygonize(orc_map* m, float* verts, float* norms, long max_tris);

/* Triangle centroids (reference GetSurfacePoints). */
void orc_surface_points(const float* verts, long n_tris, float* points);

/* Map inspection. */
int orc_num_blocks(const orc_map* m);
/* coords: n*3 int32 block coordinates; tsdf/weight: n*512 doubles (the
 * dequantised stored values), rgb: n*512*3 (may be NULL). Voxel index inside a
 * block is x + 8*y + 64*z. */
void orc_export(const orc_map* m, int32_t* coords, double* tsdf, double* weight, uint8_t* rgb);

/* Helpers exposed for unit tests. */
int orc_hash(int x, int y, int z, int n_buckets);
void orc_pose_inverse(const double pose[16], double inv[16]);
/* Constants the oracle uses, for pinning against the reference headers:
 * [block_size, min_depth*1000, max_depth*1000, trunc_factor, weight_cap_ref,
 *  hash_p0, hash_p1, hash_p2, subsample] */
void orc_constants(int out[9]);

#ifdef __cplusplus
}
#endif
#endif
