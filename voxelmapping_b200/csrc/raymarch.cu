// Ray marching (MapRenderingDelegate, src/ray_tracing.cu:255-401) for one map
// or a batch.
//
// Every ray follows the reference's sample sequence: start at z = 0.1 m (or,
// with z-range tiles, at the last 1-voxel step before the tile's nearest
// allocated block), SDF-proportional steps near surfaces, one-voxel steps
// where a sample is unobserved, trilinear interpolation within 0.5 of the
// surface, two refinement steps after the zero crossing. Work that cannot
// change the result is skipped:
//   * inside an unallocated block, where the reference reads "invalid, 1.0"
//     and steps one voxel at a time, the steps up to the block's exit are
//     taken as one integer jump; before the tile's nearest allocated block
//     these jumps need no lookup and are taken when the ray starts;
//   * when the 8 trilinear corners sit in the current block, the 7 besides
//     the centre sample are read with independent loads (no lookups between);
//   * hash lookups are cached per ray (current block + one neighbour).
//
// Scheduling: the kernel is persistent. Each warp takes 8x4-pixel tiles from
// one device-side queue shared by every map of the batch until it runs dry.
// A map's tiles are handed out in a selectable order: starting with the
// slowest tiles shortens the tail of the launch (bottom rows first measured
// 5 % faster than top rows first on the room sequences, whose lower rows see
// the floor and the nearest surfaces).
// (Refilling lanes from a larger group as their rays finish was measured
// 2.8x slower: lanes at different depths scatter their loads and lookups.)
#include "march.cuh"

namespace vmapb {

// 4 CTAs per SM (at most 64 registers) measured faster than the 3 that 76
// registers allow: latency hiding outweighs a small register spill.
template <class V, int FMT>
__global__ void __launch_bounds__(256, 4) raycast_kernel(const __grid_constant__ V views, int order, int tw)
{
    stage_entry();
    __shared__ int pre[kMaxBatch + 1];
    __shared__ unsigned long long s_wkey[8][kWarpCache];
    __shared__ int s_wslot[8][kWarpCache];
    map_prefix(views, [tw](const MapView& v) { return ray_tiles(v, tw); }, pre);
    // the z-range pass before this launch linked every allocated block of the
    // maps it renders
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int mi = 0; mi < views.count(); ++mi)
            if (views[mi].out.vmap) views[mi].m.ctr[C_LINKED] = (unsigned)allocated_blocks(views[mi].m);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    const int lane = threadIdx.x & 31;
    unsigned long long* wkey = s_wkey[threadIdx.x >> 5];
    int* wslot = s_wslot[threadIdx.x >> 5];
    int wmap = -1;  // map whose blocks the warp cache holds
    for (;;) {
        int item = 0;
        if (lane == 0) item = (int)atomicAdd(views.queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        const int mi = map_of(pre, nmaps, item);
        if (mi != wmap) {
            warp_cache_clear(wkey, lane);
            wmap = mi;
        }
        march_tile<FMT, true>(views[mi], mi, item - pre[mi], pre[mi + 1] - pre[mi], order, tw, wkey, wslot, lane);
    }
}

template <class V, int FMT>
static cudaError_t raycast_persistent(const V& views, const Launcher& l, cudaStream_t s)
{
    // resident CTAs per SM of this instantiation at 128 and 256 threads (a
    // static initialiser runs once, thread-safely, on the first launch)
    static const int occ[2] = {[] {
                                   int o = 0;
                                   if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, raycast_kernel<V, FMT>, 128,
                                                                                     0) != cudaSuccess || o < 1)
                                       o = 1;
                                   return o;
                               }(),
                               [] {
                                   int o = 0;
                                   if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, raycast_kernel<V, FMT>, 256,
                                                                                     0) != cudaSuccess || o < 1)
                                       o = 1;
                                   return o;
                               }()};
    const int threads = l.rayThreads == 128 ? 128 : 256;
    const int fit = occ[threads == 256];
    // CTAs beyond those resident would only start once others finish: cap at occupancy
    const int per_sm = l.raycast > 0 && l.raycast < fit ? l.raycast : fit;
    return launch_stage<V>(raycast_kernel<V, FMT>, stage_grid(l, per_sm), threads, s, views, l.tileOrder, l.tileW);
}

template <class V>
cudaError_t launch_raycast(const V& views, int fmt, const Launcher& l, cudaStream_t s)
{
    switch (fmt) {
    case VMAP_VOXEL_REF: return raycast_persistent<V, VMAP_VOXEL_REF>(views, l, s);
    case VMAP_VOXEL_F32: return raycast_persistent<V, VMAP_VOXEL_F32>(views, l, s);
    case VMAP_VOXEL_F16: return raycast_persistent<V, VMAP_VOXEL_F16>(views, l, s);
    case VMAP_VOXEL_I16: return raycast_persistent<V, VMAP_VOXEL_I16>(views, l, s);
    default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_raycast<OneView>(const OneView&, int, const Launcher&, cudaStream_t);
template cudaError_t launch_raycast<ManyViews>(const ManyViews&, int, const Launcher&, cudaStream_t);

}  // namespace vmapb
