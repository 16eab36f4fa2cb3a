// Fusion path: block allocation along depth rays, visible-block selection and
// the projective TSDF / weight / colour update, for one map or a batch.
//
// Reference: src/depth_fusion.cu (FuseImage :199-301, FuseDepthAndImage
// :383-488, CheckVisibleBlocks :494-539) and the device helpers of
// include/map_struct.h. The reference synchronises the device three times and
// copies the visible count to the host on every fuse; here the three kernels
// run back to back on one stream, over every map of a batch at once, and the
// counts stay in device memory.
#include "vmap_launch.h"

namespace vmapb {

template <int DT>
__device__ __forceinline__ float read_depth_t(const FrameIn& f, int x, int y)
{
    const char* row = reinterpret_cast<const char*>(f.depth) + (size_t)y * f.dpitch;
    if constexpr (DT == VMAP_DEPTH_F32) {
        return __ldg(reinterpret_cast<const float*>(row) + x);
    } else {
        return __fmul_rn(__uint2float_rn(__ldg(reinterpret_cast<const unsigned short*>(row) + x)), f.dscale);
    }
}

__device__ __forceinline__ float read_depth(const FrameIn& f, int x, int y)
{
    return f.dtype == VMAP_DEPTH_U16 ? read_depth_t<VMAP_DEPTH_U16>(f, x, y) : read_depth_t<VMAP_DEPTH_F32>(f, x, y);
}

// maps without fusion work this step (no frame) contribute no items
__device__ __forceinline__ int alloc_tiles(const MapView& v)
{
    return v.in.active ? ((v.cam.W + 31) >> 5) * ((v.cam.H + 7) >> 3) : 0;
}

// ---------------------------------------------------------------- allocation
// One thread per depth pixel, a 256-thread CTA per 32x8-pixel tile
// (CreateBlockLineTracingFunctor, depth_fusion.cu:32-59): the band
// [d - mu/2, d + mu/2] is unprojected to world voxel coordinates, sampled at
// ceil(2 |far - near|) points and every sampled block is inserted.
// The samples of a pixel are walked without touching global memory: each
// block a pixel enters is staged in a CTA-wide shared-memory set, and once
// the whole tile has been walked its distinct blocks (a few dozen) are
// inserted into the hash table in parallel, one thread per block. A warp so
// waits on one table round trip per tile instead of one per sample step, and
// the resulting block set is the one a per-sample insertion gives. The CTA
// of item 0 also clears the visible counters the next kernel accumulates
// into.
constexpr int kTileSet = 1024;  // open-addressed set of one tile's blocks (8 KB)

// Stage block key (bx, by, bz) in the tile's set; after 32 occupied probes the
// block goes straight into the hash table, which leaves the block set unchanged.
__device__ __forceinline__ void stage_block(unsigned long long* set, const DevMap& m, unsigned long long key, int bx,
                                            int by, int bz)
{
    unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 54);
#pragma unroll 1
    for (int p = 0; p < 32; ++p) {
        const unsigned long long cur = atomicCAS(set + h, kEmptyKey, key);
        if (cur == kEmptyKey || cur == key) return;
        h = (h + 1) & (kTileSet - 1);
    }
    hash_insert(m, bx, by, bz);
}

template <class V>
__global__ void __launch_bounds__(256) alloc_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    __shared__ unsigned long long set[kTileSet];
    for (int i = threadIdx.x; i < kTileSet; i += blockDim.x) set[i] = kEmptyKey;
    map_prefix(views, [](const MapView& v) { return alloc_tiles(v); }, pre);  // ends with __syncthreads
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
        const int y = (t / tx) * 8 + (threadIdx.x >> 5);
        if (x < v.cam.W && y < v.cam.H) {
            const float d = read_depth(v.in, x, y);
            if (!(isnan(d) || d < kMinDepth || d > kMaxDepth)) {
                const float tdh = __fmul_rn(m.mu, 0.5f);
                const float dn = fmaxf(kMinDepth, __fsub_rn(d, tdh));
                const float df = fmaxf(kMinDepth, __fadd_rn(d, tdh));
                if (dn < df) {
                    const float3 a = unproject(x, y, dn, v.cam.ifx, v.cam.ify, v.cam.cx, v.cam.cy);
                    const float3 wa = xf_apply(v.T, a.x, a.y, a.z);
                    const float3 b = unproject(x, y, df, v.cam.ifx, v.cam.ify, v.cam.cx, v.cam.cy);
                    const float3 wb = xf_apply(v.T, b.x, b.y, b.z);
                    // worldPtToVoxelPos: (int)floor(p / voxelSize)
                    const int nx = __float2int_rz(floorf(__fdiv_rn(wa.x, m.vs)));
                    const int ny = __float2int_rz(floorf(__fdiv_rn(wa.y, m.vs)));
                    const int nz = __float2int_rz(floorf(__fdiv_rn(wa.z, m.vs)));
                    const int fx = __float2int_rz(floorf(__fdiv_rn(wb.x, m.vs)));
                    const int fy = __float2int_rz(floorf(__fdiv_rn(wb.y, m.vs)));
                    const int fz = __float2int_rz(floorf(__fdiv_rn(wb.z, m.vs)));
                    // band end points outside the +-2^23-voxel (+-2^20-block) key range
                    // cannot be stored: flag and skip the pixel (every sample lies
                    // between the two end points)
                    if (!voxel_ok(nx, ny, nz) || !voxel_ok(fx, fy, fz)) {
                        atomicOr(m.ctr + C_ERR, VMAP_FLAG_RANGE);
                    } else {
                        float3 dir =
                            make_float3(__int2float_rn(fx - nx), __int2float_rn(fy - ny), __int2float_rn(fz - nz));
                        const float len = __fsqrt_rn(sqnorm(dir));
                        // (int)ceil(2.0 * len): the double product of a float by 2 is exact
                        const int n = __float2int_rz(ceilf(__fmul_rn(2.f, len)));
                        const float den = __int2float_rn(n - 1);
                        const float dx = __fdiv_rn(dir.x, den);
                        const float dy = __fdiv_rn(dir.y, den);
                        const float dz = __fdiv_rn(dir.z, den);
                        float px = __int2float_rn(nx), py = __int2float_rn(ny), pz = __int2float_rn(nz);
                        int lbx = INT_MIN, lby = INT_MIN, lbz = INT_MIN;
#pragma unroll 1
                        for (int s = 0; s < n; ++s) {
                            // pt_start.cast<int>() truncates toward zero, then voxelPosToBlockPos
                            const int bx = vox2blk(__float2int_rz(px));
                            const int by = vox2blk(__float2int_rz(py));
                            const int bz = vox2blk(__float2int_rz(pz));
                            if (bx != lbx || by != lby || bz != lbz) {  // consecutive samples share blocks
                                lbx = bx;
                                lby = by;
                                lbz = bz;
                                if (coord_ok(bx, by, bz)) stage_block(set, m, pack_key(bx, by, bz), bx, by, bz);
                                else atomicOr(m.ctr + C_ERR, VMAP_FLAG_RANGE);
                            }
                            px = __fadd_rn(px, dx);
                            py = __fadd_rn(py, dy);
                            pz = __fadd_rn(pz, dz);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // insert the tile's distinct blocks and empty the set for the next tile
        for (int i = threadIdx.x; i < kTileSet; i += blockDim.x) {
            const unsigned long long key = set[i];
            if (key != kEmptyKey) {
                set[i] = kEmptyKey;
                const int3 c = unpack_key(key);
                hash_insert(m, c.x, c.y, c.z);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- visibility
// CheckEntryVisibilityFunctor (depth_fusion.cu:82-126) without the full
// hash-table scan: allocated blocks are dense in pool order, so only
// min(alloc, capacity) 8-byte keys are read. Work items are 32-block groups of
// one map; visible slots are compacted with one atomic per warp. The map's
// visible counter must be zero on entry (cleared by alloc_kernel or the host).
template <class V>
__global__ void __launch_bounds__(256) visibility_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return v.in.active ? (allocated_blocks(v.m) + 31) >> 5 : 0; }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = warp; w < total; w += nwarps) {
        const int mi = map_of(pre, nmaps, w);
        const MapView& v = views[mi];
        const DevMap& m = v.m;
        const int i = (w - pre[mi]) * 32 + lane;
        bool vis = false;
        if (i < allocated_blocks(m)) {
            const int3 b = unpack_key(m.blockKeys[i]);
            vis = block_visible(b.x, b.y, b.z, v.Ti, __fmul_rn(m.vs, 8.f), v.cam.W, v.cam.H, v.cam.fx, v.cam.fy,
                                v.cam.cx, v.cam.cy);
        }
        const unsigned mask = __ballot_sync(0xffffffffu, vis);
        if (mask == 0) continue;
        unsigned first = 0;
        if (lane == 0) first = atomicAdd(m.ctr + C_VISIBLE, (unsigned)__popc(mask));
        first = __shfl_sync(0xffffffffu, first, 0);
        if (vis) m.visList[first + __popc(mask & ((1u << lane) - 1))] = i;
    }
}

// ----------------------------------------------------------------- fusion
// DepthFusionFunctor / ImageFusionFunctor (depth_fusion.cu:148-196, 328-380)
// for one visible block: 128 threads, each owning 4 consecutive voxels of an
// x-row (one 16- or 32-byte vector of voxel words, one 4-byte word per colour
// plane). The voxel words are loaded before the projections so the load
// overlaps the arithmetic; a thread writes only when one of its voxels updates.
template <int FMT, bool COLOR, int DT>
__device__ __forceinline__ void fuse_block(const MapView& v, int slot, int v0)
{
    typedef Layout<FMT> L;
    typedef typename L::Word Word;
    typedef Fmt<FMT> F;
    const DevMap& m = v.m;
    const int lx0 = v0 & 7, ly = (v0 >> 3) & 7, lz = v0 >> 6;
    const int3 bp = unpack_key(m.blockKeys[slot]);
    Word* blk = L::words_rw(m, slot);
    Word w[4];
    load_vec<4 * sizeof(Word)>(blk + v0, w);
    const int vx0 = bp.x * 8 + lx0;
    const float wy = __fmul_rn(__int2float_rn(bp.y * 8 + ly), m.vs);
    const float wz = __fmul_rn(__int2float_rn(bp.z * 8 + lz), m.vs);
    float sdfv[4];
    int pu[4], pv[4];
    unsigned mask = 0;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        const float3 p = xf_apply(v.Ti, __fmul_rn(__int2float_rn(vx0 + x), m.vs), wy, wz);
        // __float2int_rd(fx * p0 / p2 + cx + 0.5)
        const int u = __float2int_rd(__fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(v.cam.fx, p.x), p.z), v.cam.cx), 0.5f));
        const int vv = __float2int_rd(__fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(v.cam.fy, p.y), p.z), v.cam.cy), 0.5f));
        pu[x] = u;
        pv[x] = vv;
        sdfv[x] = 0.f;
        if (u < 0 || vv < 0 || u > v.cam.W - 1 || vv > v.cam.H - 1) continue;
        const float d = read_depth_t<DT>(v.in, u, vv);
        if (isnan(d) || d > kMaxDepth || d < kMinDepth) continue;
        const float sdf = __fsub_rn(d, p.z);
        if (sdf < -m.mu) continue;
        sdfv[x] = fminf(1.f, __fdiv_rn(sdf, m.mu));
        mask |= 1u << x;
    }
    if (!mask) return;
    unsigned char c[3][4];
    unsigned char* crow = reinterpret_cast<unsigned char*>(blk) + L::kRgbOff + v0;
    if constexpr (COLOR) {
#pragma unroll
        for (int k = 0; k < 3; ++k) load_vec<4>(crow + k * kBlockVoxels, c[k]);
    }
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        if (!(mask & (1u << x))) continue;
        const float ow = F::weight(w[x]);
        const uint8_t* px = nullptr;
        if constexpr (COLOR) px = v.in.rgb + (size_t)pv[x] * v.in.rgbPitch + 3 * pu[x];
        if (ow == 0.f) {
            w[x] = F::make(sdfv[x], 1.f);
            if constexpr (COLOR) {
#pragma unroll
                for (int k = 0; k < 3; ++k) c[k][x] = __ldg(px + k);
            }
        } else {
            const float os = F::tsdf(w[x]);
            w[x] = F::make(__fdiv_rn(__fmaf_rn(os, ow, sdfv[x]), __fadd_rn(ow, 1.f)), fminf(__fadd_rn(ow, 1.f), m.wmax));
            if constexpr (COLOR) {
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    c[k][x] = (unsigned char)__float2int_rz(
                        __fmaf_rn(0.7f, __uint2float_rn(c[k][x]), __fmul_rn(0.3f, __uint2float_rn(__ldg(px + k)))));
            }
        }
    }
    store_vec<4 * sizeof(Word)>(blk + v0, w);
    if constexpr (COLOR) {
#pragma unroll
        for (int k = 0; k < 3; ++k) store_vec<4>(crow + k * kBlockVoxels, c[k]);
    }
}

// 2 blocks per 256-thread CTA, grid-stride over the visible blocks of all maps.
// Colour is fused when the frame carries it (the map must keep colour).
template <class V, int FMT>
__global__ void __launch_bounds__(256) fuse_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return v.in.active ? (int)v.m.ctr[C_VISIBLE] : 0; }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    const int team = threadIdx.x >> 7;
    const int v0 = (threadIdx.x & 127) * 4;  // first voxel index of this thread
    for (int i = blockIdx.x * 2 + team; i < total; i += gridDim.x * 2) {
        const int mi = map_of(pre, nmaps, i);
        const MapView& v = views[mi];
        const int slot = v.m.visList[i - pre[mi]];
        const bool color = v.in.rgb != nullptr;
        if (v.in.dtype == VMAP_DEPTH_U16) {
            if (color) fuse_block<FMT, true, VMAP_DEPTH_U16>(v, slot, v0);
            else fuse_block<FMT, false, VMAP_DEPTH_U16>(v, slot, v0);
        } else {
            if (color) fuse_block<FMT, true, VMAP_DEPTH_F32>(v, slot, v0);
            else fuse_block<FMT, false, VMAP_DEPTH_F32>(v, slot, v0);
        }
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
    alloc_kernel<V><<<stage_grid(l, l.alloc, totalTiles), 256, 0, s>>>(views);
    return cudaGetLastError();
}

template <class V>
cudaError_t launch_visibility(const V& views, const Launcher& l, cudaStream_t s)
{
    visibility_kernel<V><<<stage_grid(l, l.visibility), 256, 0, s>>>(views);
    return cudaGetLastError();
}

template <class V>
cudaError_t launch_fuse(const V& views, int fmt, const Launcher& l, cudaStream_t s)
{
    const int grid = stage_grid(l, l.fuse);
    switch (fmt) {
    case VMAP_VOXEL_REF: fuse_kernel<V, VMAP_VOXEL_REF><<<grid, 256, 0, s>>>(views); break;
    case VMAP_VOXEL_F32: fuse_kernel<V, VMAP_VOXEL_F32><<<grid, 256, 0, s>>>(views); break;
    case VMAP_VOXEL_F16: fuse_kernel<V, VMAP_VOXEL_F16><<<grid, 256, 0, s>>>(views); break;
    case VMAP_VOXEL_I16: fuse_kernel<V, VMAP_VOXEL_I16><<<grid, 256, 0, s>>>(views); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
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
