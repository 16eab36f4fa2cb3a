// Raycast path: per-tile depth bounds, ray marching with trilinear
// interpolation, normal map and Phong preview, for one map or a batch.
//
// Reference: src/ray_tracing.cu (RenderingBlockDelegate :13-137,
// FillRenderingBlockFunctor :139-169, MapRenderingDelegate :255-401) and
// src/image_proc.cu (renderSceneKernel :8-61, computeNormalKernel :74-93).
//
// The reference marches every ray from z = 0.1 m to 5 m, one voxel per step
// through unallocated space, with a full hash-chain walk per sample; it
// computes per-tile z ranges but never reads them (ray_tracing.cu:335-341).
// This implementation keeps the reference's sample lattice (start point,
// direction, 1-voxel steps in empty space, SDF-proportional steps near
// surfaces, two refinement steps) and skips work that cannot change the
// result:
//   * tiles of 8x8 pixels start at the nearest allocated block that can
//     cover them and stop after the farthest one (bounds computed over all
//     allocated blocks, conservatively, so no block a ray can enter is
//     missed);
//   * inside an unallocated block, where the reference reads "invalid, 1.0"
//     and steps 1 voxel at a time, the steps up to the block's exit are taken
//     as one integer jump;
//   * block lookups are cached per thread.
// The ray marcher itself lives in raymarch.cu.
#include "vmap_launch.h"

namespace vmapb {

// ------------------------------------------------------------------ z-range
// Per allocated block: the part of the block in front of the plane z = zc
// (corners in front, plus the points where its 12 edges cross the plane) is
// projected; its pixel bounding box (+1 px) and depth range (+-1 voxel) are
// folded into the 8x8-pixel tile maps with 64-bit atomics on epoch-tagged
// values (depths are positive, so float order == bit order). Every point of a
// block is a convex combination of its corners, so the box and range bound
// every ray sample that can fall inside the block. Block 0 also rewinds the
// raycast work queue for the kernel that follows.
//
// The same pass, in both raycast modes, sets the forward neighbour links of
// the blocks allocated since the last pass, [ctr[C_LINKED], allocated): pool
// slots are dense, so those are the newest. Each new block is 14 independent
// tasks spread over the grid, one lookup each: its 7 links, and the link of
// each of its 7 backward neighbours that points at it. Two new neighbours
// write each other's link with the same value, so the order of the writes
// does not matter. The ray marcher, which always follows, reads the links for
// trilinear corners in neighbouring blocks and advances C_LINKED.
constexpr float kClipZ = 0.05f;  // below the ray start depth of 0.1 m

__device__ __forceinline__ int links_pending(const MapView& v)
{
    if (!v.out.vmap) return 0;
    const int done = (int)*((volatile const unsigned*)(v.m.ctr + C_LINKED));
    const int n = allocated_blocks(v.m);
    return n > done ? 14 * (n - done) : 0;
}

template <class V>
__global__ void __launch_bounds__(256) zrange_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    const int nmaps = views.count();
    // neighbour links of the new blocks
    map_prefix(views, [](const MapView& v) { return links_pending(v); }, pre);
    const int ntasks = pre[nmaps];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntasks; i += gridDim.x * blockDim.x) {
        const int mi = map_of(pre, nmaps, i);
        const DevMap& m = views[mi].m;
        const int t = i - pre[mi];
        const int slot = (int)*((volatile const unsigned*)(m.ctr + C_LINKED)) + t / 14;
        const int k = 1 + (t % 14) / 2, dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        const int3 b = unpack_key(m.blockKeys[slot]);
        if (t & 1) {  // a backward neighbour's link to this block
            const int e = hash_find(m, b.x - dx, b.y - dy, b.z - dz);
            if (e >= 0) m.nbr[7 * (size_t)e + k - 1] = slot;
        } else {
            m.nbr[7 * (size_t)slot + k - 1] = hash_find(m, b.x + dx, b.y + dy, b.z + dz);
        }
    }
    __syncthreads();  // `pre` is reused
    map_prefix(views, [](const MapView& v) { return v.out.vmap && v.out.mode == 0 ? allocated_blocks(v.m) : 0; }, pre);
    if (blockIdx.x == 0 && threadIdx.x == 0) views.queue[0] = 0u;
    const int total = pre[nmaps];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int mi = map_of(pre, nmaps, i);
        const MapView& v = views[mi];
        const DevMap& m = v.m;
        const RenderOut& r = v.out;
        const int3 b = unpack_key(m.blockKeys[i - pre[mi]]);
        const float scale = m.vs * 8.f;
        float3 p[8];
        float zlo = 1e30f, zhi = -1e30f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            p[c] = xf_apply(v.Ti, (float)(b.x + (c & 1)) * scale, (float)(b.y + ((c >> 1) & 1)) * scale,
                            (float)(b.z + ((c >> 2) & 1)) * scale);
            zlo = fminf(zlo, p[c].z);
            zhi = fmaxf(zhi, p[c].z);
        }
        if (zhi <= kClipZ || zhi < kMinDepth - m.vs || zlo > kMaxDepth + m.vs) continue;
        float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
        auto add = [&](float3 q) {
            const float iz = 1.f / q.z;
            const float u = v.cam.fx * q.x * iz + v.cam.cx, w = v.cam.fy * q.y * iz + v.cam.cy;
            umin = fminf(umin, u);
            umax = fmaxf(umax, u);
            vmin = fminf(vmin, w);
            vmax = fmaxf(vmax, w);
        };
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (p[c].z > kClipZ) add(p[c]);
        if (zlo <= kClipZ) {  // the block crosses the clip plane: add the edge crossings
#pragma unroll
            for (int c = 0; c < 8; ++c)
#pragma unroll
                for (int bit = 1; bit < 8; bit <<= 1) {
                    if (c & bit) continue;
                    const float3 a = p[c], e = p[c | bit];
                    if ((a.z > kClipZ) == (e.z > kClipZ)) continue;
                    const float t = (kClipZ - a.z) / (e.z - a.z);
                    add(make_float3(a.x + t * (e.x - a.x), a.y + t * (e.y - a.y), kClipZ));
                }
        }
        const int W = v.cam.W, H = v.cam.H;
        if (umax < -1.f || vmax < -1.f || umin > (float)W || vmin > (float)H) continue;
        const int tx0 = max(0, (int)floorf(fmaxf(umin - 1.f, -8.f)) >> 3);
        const int tx1 = min(r.tilesX - 1, (int)floorf(fminf(umax + 1.f, (float)W + 8.f)) >> 3);
        const int ty0 = max(0, (int)floorf(fmaxf(vmin - 1.f, -8.f)) >> 3);
        const int ty1 = min(r.tilesY - 1, (int)floorf(fminf(vmax + 1.f, (float)H + 8.f)) >> 3);
        const unsigned long long lo =
            ((unsigned long long)(~r.epoch) << 32) | __float_as_uint(fmaxf(zlo - m.vs, 0.f));
        const unsigned long long hi = ((unsigned long long)r.epoch << 32) | __float_as_uint(zhi + m.vs);
        for (int ty = ty0; ty <= ty1; ++ty)
            for (int tx = tx0; tx <= tx1; ++tx) {
                const int t = ty * r.tilesX + tx;
                atomicMin(r.zmin + t, lo);
                atomicMax(r.zmax + t, hi);
            }
    }
}

// ------------------------------------------------------------------ normals
// computeNormalKernel (image_proc.cu:74-93): normalize((v[x+1] - v[x-1]) x
// (v[y+1] - v[y-1])), w = 1. Undefined pixels (last row / column, NaN
// neighbour) are written all-NaN. 32x8-pixel tiles of every map that wants a
// normal map.
__device__ __forceinline__ int normal_tiles(const MapView& v)
{
    return v.out.nmap ? ((v.cam.W + 31) >> 5) * ((v.cam.H + 7) >> 3) : 0;
}

template <class V>
__global__ void __launch_bounds__(256) normals_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return normal_tiles(v); }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int mi = map_of(pre, nmaps, item);
        const MapView& v = views[mi];
        const int t = item - pre[mi];
        const int W = v.cam.W, H = v.cam.H;
        const int tx = (W + 31) >> 5;
        const int x = (t % tx) * 32 + (threadIdx.x & 31);
        const int y = (t / tx) * 8 + (threadIdx.x >> 5);
        if (x >= W || y >= H) continue;
        const float qnan = __int_as_float(0x7fffffff);
        float4 res = make_float4(qnan, qnan, qnan, qnan);
        if (x < W - 1 && y < H - 1) {
            const char* vm = reinterpret_cast<const char*>(v.out.vmap);
            const size_t vp = v.out.vpitch;
            auto at = [&](int xx, int yy) { return __ldg(reinterpret_cast<const float4*>(vm + (size_t)yy * vp) + xx); };
            const float4 v00 = at(max(x - 1, 0), y), v01 = at(x + 1, y), v10 = at(x, max(y - 1, 0)), v11 = at(x, y + 1);
            if (!(isnan(v00.x) || isnan(v01.x) || isnan(v10.x) || isnan(v11.x))) {
                const float3 a = make_float3(__fsub_rn(v01.x, v00.x), __fsub_rn(v01.y, v00.y), __fsub_rn(v01.z, v00.z));
                const float3 b = make_float3(__fsub_rn(v11.x, v10.x), __fsub_rn(v11.y, v10.y), __fsub_rn(v11.z, v10.z));
                const float3 n = normalized(cross3(a, b));
                res = make_float4(n.x, n.y, n.z, 1.f);
            }
        }
        *(reinterpret_cast<float4*>(reinterpret_cast<char*>(v.out.nmap) + (size_t)y * v.out.npitch) + x) = res;
    }
}

// -------------------------------------------------------------------- Phong
// renderPoint (image_proc.cu:8-44): light at (5,5,5), Ka 0.3, Kd 0.5, Ks 0.2,
// exponent 20, unit material colour; background (4,2,2)/255.
__global__ void __launch_bounds__(256) phong_kernel(const float4* vmap, size_t vpitch, const float4* nmap,
                                                    size_t npitch, uchar4* rgba, size_t rpitch, int W, int H)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= W || y >= H) return;
    const float4 p = __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(vmap) + (size_t)y * vpitch) + x);
    const float4 n = __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(nmap) + (size_t)y * npitch) + x);
    float c0 = 4.f / 255.f, c1 = 2.f / 255.f, c2 = 2.f / 255.f;
    if (!isnan(p.x)) {
        const float3 L = normalized(make_float3(__fsub_rn(5.f, p.x), __fsub_rn(5.f, p.y), __fsub_rn(5.f, p.z)));
        const float3 V = normalized(make_float3(__fsub_rn(0.f, p.x), __fsub_rn(0.f, p.y), __fsub_rn(0.f, p.z)));
        const float nl = __fmaf_rn(n.x, L.x, __fmaf_rn(n.y, L.y, __fmul_rn(n.z, L.z)));
        const float3 R = normalized(make_float3(__fmaf_rn(__fmul_rn(2.f, n.x), nl, -L.x),
                                                __fmaf_rn(__fmul_rn(2.f, n.y), nl, -L.y),
                                                __fmaf_rn(__fmul_rn(2.f, n.z), nl, -L.z)));
        const float rv = __fmaf_rn(R.x, V.x, __fmaf_rn(R.y, V.y, __fmul_rn(R.z, V.z)));
        const float I = __fmaf_rn(0.2f, powf(fmaxf(0.f, rv), 20.f), __fmaf_rn(0.5f, fmaxf(0.f, nl), 0.3f));
        c0 = c1 = c2 = I;
    }
    uchar4 o;
    o.x = (unsigned char)__float2uint_rz(__saturatef(c0) * 255.f);
    o.y = (unsigned char)__float2uint_rz(__saturatef(c1) * 255.f);
    o.z = (unsigned char)__float2uint_rz(__saturatef(c2) * 255.f);
    o.w = 255;
    *(reinterpret_cast<uchar4*>(reinterpret_cast<char*>(rgba) + (size_t)y * rpitch) + x) = o;
}

// ------------------------------------------------------------------ launchers
template <class V>
cudaError_t launch_zrange(const V& views, const Launcher& l, cudaStream_t s)
{
    zrange_kernel<V><<<stage_grid(l, l.zrange), 256, 0, s>>>(views);
    return cudaGetLastError();
}

template <class V>
cudaError_t launch_normals(const V& views, int totalTiles, const Launcher& l, cudaStream_t s)
{
    normals_kernel<V><<<stage_grid(l, l.normals, totalTiles), 256, 0, s>>>(views);
    return cudaGetLastError();
}

template cudaError_t launch_zrange<OneView>(const OneView&, const Launcher&, cudaStream_t);
template cudaError_t launch_zrange<ManyViews>(const ManyViews&, const Launcher&, cudaStream_t);
template cudaError_t launch_normals<OneView>(const OneView&, int, const Launcher&, cudaStream_t);
template cudaError_t launch_normals<ManyViews>(const ManyViews&, int, const Launcher&, cudaStream_t);

cudaError_t launch_phong(const float4* vmap, size_t vpitch, const float4* nmap, size_t npitch, uchar4* rgba,
                         size_t rpitch, int W, int H, cudaStream_t s)
{
    dim3 grid((W + 31) / 32, (H + 7) / 8);
    phong_kernel<<<grid, 256, 0, s>>>(vmap, vpitch, nmap, npitch, rgba, rpitch, W, H);
    return cudaGetLastError();
}

}  // namespace vmapb
