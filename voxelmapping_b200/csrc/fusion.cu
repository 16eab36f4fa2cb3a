// Fusion path: block allocation along depth rays, visible-block selection and
// the projective TSDF / weight / colour update, for one map or a batch.
//
// Reference: src/depth_fusion.cu (FuseImage :199-301, FuseDepthAndImage
// :383-488, CheckVisibleBlocks :494-539) and the device helpers of
// include/map_struct.h. The reference synchronises the device three times and
// copies the visible count to the host on every fuse; here the three kernels
// run back to back on one stream, over every map of a batch at once, and the
// counts stay in device memory.
#include "stages.cuh"

namespace vmapb {

// ---------------------------------------------------------------- allocation
// A 256-thread CTA per 32 x kStageTileH-pixel tile, kStageTileH / 8 depth
// pixels per thread. The
// samples of a pixel's band are walked without touching global memory: each
// block a pixel enters is staged in a CTA-wide shared-memory set, and once
// the whole tile has been walked its distinct blocks (a few dozen) are
// inserted into the hash table in parallel, one thread per block. A warp so
// waits on one table round trip per tile instead of one per sample step, and
// the block set is the one a per-sample insertion gives. The CTA of item 0
// also clears the visible counters the next kernel accumulates into.
// 8 resident CTAs per SM (at most 32 registers) measured faster than the 6
// that 38 registers allow (20.9 against 22.1 us per 640x480 frame).
constexpr int kTileSet = 1024;  // open-addressed set of one tile's blocks (8 KB)

template <class V>
__global__ void __launch_bounds__(256, 8) alloc_kernel(V views)
{
    stage_entry();
    __shared__ int pre[kMaxBatch + 1];
    __shared__ unsigned long long set[kTileSet];
    for (int i = threadIdx.x; i < kTileSet; i += blockDim.x) set[i] = kEmptyKey;
    map_prefix(views, [](const MapView& v) { return alloc_tiles<kStageTileH>(v); }, pre);  // ends with __syncthreads
    const int nmaps = views.count();
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < nmaps; i += blockDim.x)
            if (views[i].in.active) views[i].m.ctr[C_VISIBLE] = 0u;
    const int total = pre[nmaps];
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int mi = map_of(pre, nmaps, item);
        const MapView& v = views[mi];
        const DevMap& m = v.m;
        const int t = item - pre[mi];
        const int tx = (v.cam.W + 31) >> 5;
        const int x = (t % tx) * 32 + (threadIdx.x & 31);
        const int y0 = (t / tx) * kStageTileH + (threadIdx.x >> 5);
        float d[kStageTileH / 8];  // this thread's pixels (x, y0 + 8 r), depths loaded first
#pragma unroll
        for (int r = 0; r < kStageTileH / 8; ++r)
            d[r] = x < v.cam.W && y0 + 8 * r < v.cam.H ? read_depth(v.in, x, y0 + 8 * r) : __int_as_float(0x7fffffff);
#pragma unroll 1
        for (int r = 0; r < kStageTileH / 8; ++r)
            band_blocks_at(v, x, y0 + 8 * r, d[r], [&](unsigned long long key, int bx, int by, int bz) {
                stage_block<kTileSet>(set, m, key, bx, by, bz);
            });
        __syncthreads();
        insert_staged<kTileSet>(set, m, threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- visibility
// CheckEntryVisibilityFunctor without the full hash-table scan: allocated
// blocks are dense in pool order, so only min(alloc, capacity) 8-byte keys
// are read. Work items are 32-block groups of one map, one per warp. The
// map's visible counter must be zero on entry (cleared by alloc_kernel or the
// host).
template <class V>
__global__ void __launch_bounds__(256) visibility_kernel(V views)
{
    stage_entry();
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return v.in.active ? (allocated_blocks(v.m) + 31) >> 5 : 0; }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = warp; w < total; w += nwarps) {
        const int mi = map_of(pre, nmaps, w);
        visibility_group(views[mi], w - pre[mi], threadIdx.x & 31);
    }
}

// ----------------------------------------------------------------- fusion
// A team of 512 / kFuseVoxels threads per visible block, kFuseVoxels voxels
// of an x-row per thread; 256 / team blocks per CTA, grid-stride over the
// visible blocks of all maps. 6 resident CTAs per SM (at most 40 registers)
// measured faster than the 5 that 48 registers allow (56.9 against 59.4 us
// at 22.7k visible blocks) and than 8 voxels per thread at 4 CTAs per SM.
constexpr int kFuseVoxels = 4;
constexpr int kFuseTeam = kBlockVoxels / kFuseVoxels;

template <class V, int FMT>
__global__ void __launch_bounds__(256, 6) fuse_kernel(V views)
{
    stage_entry();
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return v.in.active ? (int)v.m.ctr[C_VISIBLE] : 0; }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    constexpr int teams = 256 / kFuseTeam;
    const int team = threadIdx.x / kFuseTeam;
    const int v0 = (threadIdx.x % kFuseTeam) * kFuseVoxels;  // first voxel index of this thread
    for (int i = blockIdx.x * teams + team; i < total; i += gridDim.x * teams) {
        const int mi = map_of(pre, nmaps, i);
        const MapView& v = views[mi];
        fuse_voxels<FMT, kFuseVoxels>(v, v.m.visList[i - pre[mi]], v0);
    }
}

// ------------------------------------------------------------------- reset
// MapStruct::reset (map_struct.cu:29-42): empty hash slots, pool pointer 0,
// zeroed voxels.
__global__ void reset_hash_kernel(DevMap m)
{
    const size_t n = (size_t)m.nBucket * kSlots;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        m.slots[i] = make_ulonglong2(kEmptyKey, ~0ull);
    }
}

// ------------------------------------------------------------------ launchers
template <class V>
cudaError_t launch_alloc(const V& views, int totalTiles, const Launcher& l, cudaStream_t s)
{
    return launch_stage<V>(alloc_kernel<V>, stage_grid(l, l.alloc, totalTiles), 256, s, views);
}

template <class V>
cudaError_t launch_visibility(const V& views, const Launcher& l, cudaStream_t s)
{
    return launch_stage<V>(visibility_kernel<V>, stage_grid(l, l.visibility), 256, s, views);
}

template <class V>
cudaError_t launch_fuse(const V& views, int fmt, const Launcher& l, cudaStream_t s)
{
    const int grid = stage_grid(l, l.fuse);
    switch (fmt) {
    case VMAP_VOXEL_REF: return launch_stage<V>(fuse_kernel<V, VMAP_VOXEL_REF>, grid, 256, s, views);
    case VMAP_VOXEL_F32: return launch_stage<V>(fuse_kernel<V, VMAP_VOXEL_F32>, grid, 256, s, views);
    case VMAP_VOXEL_F16: return launch_stage<V>(fuse_kernel<V, VMAP_VOXEL_F16>, grid, 256, s, views);
    case VMAP_VOXEL_I16: return launch_stage<V>(fuse_kernel<V, VMAP_VOXEL_I16>, grid, 256, s, views);
    default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_alloc<OneView>(const OneView&, int, const Launcher&, cudaStream_t);
template cudaError_t launch_alloc<ManyViews>(const ManyViews&, int, const Launcher&, cudaStream_t);
template cudaError_t launch_visibility<OneView>(const OneView&, const Launcher&, cudaStream_t);
template cudaError_t launch_visibility<ManyViews>(const ManyViews&, const Launcher&, cudaStream_t);
template cudaError_t launch_fuse<OneView>(const OneView&, int, const Launcher&, cudaStream_t);
template cudaError_t launch_fuse<ManyViews>(const ManyViews&, int, const Launcher&, cudaStream_t);

cudaError_t launch_reset(const DevMap& m, size_t poolBytes, const Launcher& l, cudaStream_t s)
{
    reset_hash_kernel<<<l.numSMs * 4, 256, 0, s>>>(m);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(m.ctr, 0, C_COUNT * sizeof(unsigned), s)) != cudaSuccess) return e;
    return cudaMemsetAsync(m.pool, 0, poolBytes, s);
}

}  // namespace vmapb
