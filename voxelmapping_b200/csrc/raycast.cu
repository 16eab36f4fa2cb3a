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
#include "stages.cuh"

namespace vmapb {

// ------------------------------------------------------------------ z-range
// One thread per task, in one index space per map: first the neighbour links
// of the blocks allocated since the last pass, [ctr[C_LINKED], allocated) (in
// both raycast modes: the ray marcher, which always follows, reads the links
// for trilinear corners in neighbouring blocks and advances C_LINKED), then
// one z-range fold per allocated block of the maps rendered in mode 0. The
// two kinds of task are independent, so they share one pass. Block 0 also
// rewinds the raycast work queue for the kernel that follows.
template <class V>
__global__ void __launch_bounds__(256) zrange_kernel(V views)
{
    stage_entry();
    __shared__ int pre[kMaxBatch + 1];
    const int nmaps = views.count();
    map_prefix(views, [](const MapView& v) { return links_pending(v) + zrange_blocks(v); }, pre);
    if (blockIdx.x == 0 && threadIdx.x == 0) views.queue[0] = 0u;
    const int total = pre[nmaps];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int mi = map_of(pre, nmaps, i);
        const MapView& v = views[mi];
        const int t = i - pre[mi], nlink = links_pending(v);
        if (t < nlink) link_task<true>(v.m, t);
        else zrange_block(v, t - nlink);
    }
}

// ------------------------------------------------------------------ normals
// One 256-thread CTA per 32 x kStageTileH-pixel tile, kStageTileH / 8 pixels
// per thread.
template <class V>
__global__ void __launch_bounds__(256) normals_kernel(V views)
{
    stage_entry();
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return normal_tiles<kStageTileH>(v); }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int mi = map_of(pre, nmaps, item);
        const MapView& v = views[mi];
        const int t = item - pre[mi];
        const int tx = (v.cam.W + 31) >> 5;
        const int x = (t % tx) * 32 + (threadIdx.x & 31), y0 = (t / tx) * kStageTileH + (threadIdx.x >> 5);
#pragma unroll
        for (int r = 0; r < kStageTileH / 8; ++r) normal_pixel<true>(v, x, y0 + 8 * r);
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
    return launch_stage<V>(zrange_kernel<V>, stage_grid(l, l.zrange), 256, s, views);
}

template <class V>
cudaError_t launch_normals(const V& views, int totalTiles, const Launcher& l, cudaStream_t s)
{
    return launch_stage<V>(normals_kernel<V>, stage_grid(l, l.normals, totalTiles), 256, s, views);
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
