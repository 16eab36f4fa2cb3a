// Host-side launchers of the libvmap_b200 kernels (internal interface between
// the C ABI glue in map.cu / batch.cu and the kernel translation units). The
// stage launchers take a view source: OneView (single map, by value) or
// ManyViews (device array of MapView for a batch).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <type_traits>
#include <utility>

#include "vmap_internal.cuh"

struct vmap_map;

namespace vmapb {

// Grid shape of every stage, in CTAs per SM (vmap_launch_config). Each kernel
// strides over its work items, so any grid gives the same result; the
// defaults are measured choices, the autotuner may pick others.
struct Launcher {
    int numSMs;
    int alloc = 8, visibility = 2, fuse = 16, zrange = 4;
    int raycast = 0;  // persistent ray marcher: 0 = as many CTAs as fit on an SM
    int normals = 8, mesh = 8;
    int tileOrder = 0;  // ray-marcher tile order (vmap_launch_config.raycast_tile_order)
    int tileW = 8;       // ray-marcher tile width; the tile is 32 rays
    int rayThreads = 256;  // ray-marcher threads per CTA
    int batchSchedule = 1;  // vmap_launch_config.batch_schedule
};

// vmap_launch_config <-> Launcher (0 in a field: the default)
inline bool launch_config_ok(const vmap_launch_config* c)
{
    const int v[7] = {c->alloc_ctas_per_sm, c->visibility_ctas_per_sm, c->fuse_ctas_per_sm, c->zrange_ctas_per_sm,
                      c->raycast_ctas_per_sm, c->normals_ctas_per_sm, c->mesh_ctas_per_sm};
    for (int x : v)
        if (x < 0 || x > 64) return false;
    const int tw = c->raycast_tile_width, tt = c->raycast_threads_per_cta;
    return c->raycast_tile_order >= 0 && c->raycast_tile_order <= 2 && (tw == 0 || tw == 4 || tw == 8 || tw == 16) &&
           (tt == 0 || tt == 128 || tt == 256) && c->batch_schedule >= 0 && c->batch_schedule <= 2;
}

inline void launch_config_to(const vmap_launch_config* c, Launcher& l)
{
    const Launcher d = Launcher();
    l.alloc = c->alloc_ctas_per_sm ? c->alloc_ctas_per_sm : d.alloc;
    l.visibility = c->visibility_ctas_per_sm ? c->visibility_ctas_per_sm : d.visibility;
    l.fuse = c->fuse_ctas_per_sm ? c->fuse_ctas_per_sm : d.fuse;
    l.zrange = c->zrange_ctas_per_sm ? c->zrange_ctas_per_sm : d.zrange;
    l.raycast = c->raycast_ctas_per_sm;
    l.normals = c->normals_ctas_per_sm ? c->normals_ctas_per_sm : d.normals;
    l.mesh = c->mesh_ctas_per_sm ? c->mesh_ctas_per_sm : d.mesh;
    l.tileOrder = c->raycast_tile_order;
    l.tileW = c->raycast_tile_width ? c->raycast_tile_width : d.tileW;
    l.rayThreads = c->raycast_threads_per_cta ? c->raycast_threads_per_cta : d.rayThreads;
    l.batchSchedule = c->batch_schedule ? c->batch_schedule : d.batchSchedule;
}

inline void launch_config_from(const Launcher& l, vmap_launch_config* c)
{
    c->alloc_ctas_per_sm = l.alloc;
    c->visibility_ctas_per_sm = l.visibility;
    c->fuse_ctas_per_sm = l.fuse;
    c->zrange_ctas_per_sm = l.zrange;
    c->raycast_ctas_per_sm = l.raycast;
    c->normals_ctas_per_sm = l.normals;
    c->mesh_ctas_per_sm = l.mesh;
    c->raycast_tile_order = l.tileOrder;
    c->raycast_tile_width = l.tileW;
    c->raycast_threads_per_cta = l.rayThreads;
    c->batch_schedule = l.batchSchedule;
}

// grid of `per_sm` CTAs per SM, or fewer when there are fewer work items
inline int stage_grid(const Launcher& l, int per_sm, long long items = -1)
{
    const long long g = (long long)l.numSMs * per_sm;
    if (items >= 0 && items < g) return items > 0 ? (int)items : 1;
    return (int)g;
}

// Launch of a per-frame stage kernel (which calls stage_entry() first) over
// the view source V: single maps with programmatic stream serialization,
// batches without (their multi-wave launches measured 1.7 % slower with it,
// a single map's 4 % faster).
template <class V, typename... KArgs, typename... Args>
cudaError_t launch_stage(void (*kernel)(KArgs...), int grid, int block, cudaStream_t s, Args&&... args)
{
    constexpr bool pdl = std::is_same<V, OneView>::value;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// fusion.cu
template <class V>
cudaError_t launch_alloc(const V& views, int totalTiles, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_visibility(const V& views, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_fuse(const V& views, int fmt, const Launcher& l, cudaStream_t s);
cudaError_t launch_reset(const DevMap& m, size_t poolBytes, const Launcher& l, cudaStream_t s);

// raycast.cu
template <class V>
cudaError_t launch_zrange(const V& views, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_raycast(const V& views, int fmt, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_normals(const V& views, int totalTiles, const Launcher& l, cudaStream_t s);
cudaError_t launch_phong(const float4* vmap, size_t vpitch, const float4* nmap, size_t npitch, uchar4* rgba,
                         size_t rpitch, int W, int H, cudaStream_t s);

// mesh.cu
cudaError_t launch_mesh(const DevMap& m, int fmt, float* verts, float* norms, unsigned maxTris,
                        unsigned* ntrisOut, const Launcher& l, cudaStream_t s);
cudaError_t launch_surface_points(const float* verts, unsigned n, float* pts, cudaStream_t s);
cudaError_t launch_export(const DevMap& m, int fmt, bool color, int first, int count, int* coords, float* tsdf,
                          float* weight, uint8_t* rgb, cudaStream_t s);

// map.cu: device view of a map and the text behind vmap_last_error().
const DevMap& map_device_view(const vmap_map* m);
int map_device(const vmap_map* m);  // CUDA device the map was created on
void set_last_error(const std::string& msg);

// Allocation and normal-map kernels work on 32 x kStageTileH-pixel tiles, one
// 256-thread CTA each (kStageTileH / 8 pixels per thread). 16-row tiles (600
// per 640x480 frame, one wave on 148 SMs, where 8-row tiles leave a second
// wave of 16 CTAs) measured slower: allocation 31.3 against 21.3 us, since
// each thread then walks two bands one after the other.
constexpr int kStageTileH = 8;
inline int stage_tiles(int W, int H) { return ((W + 31) / 32) * ((H + kStageTileH - 1) / kStageTileH); }

}  // namespace vmapb
