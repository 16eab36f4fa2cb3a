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
// The ray kernel is persistent: its warps take 8x4-pixel tiles of every map
// of the batch from one device-side queue until the queue runs dry.
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
constexpr float kClipZ = 0.05f;  // below the ray start depth of 0.1 m

template <class V>
__global__ void __launch_bounds__(256) zrange_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return v.out.mode == 0 ? allocated_blocks(v.m) : 0; }, pre);
    if (blockIdx.x == 0 && threadIdx.x == 0) views.queue[0] = 0u;
    const int nmaps = views.count();
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

// ------------------------------------------------------------------ raycast
template <int FMT>
struct RayCtx {
    const DevMap& m;
    int cbx, cby, cbz, cblk;  // block of the current sample
    int obx, oby, obz, oblk;  // last other block (trilinear corners)

    __device__ __forceinline__ RayCtx(const DevMap& mm)
        : m(mm), cbx(INT_MIN), cby(0), cbz(0), cblk(-1), obx(INT_MIN), oby(0), obz(0), oblk(-1)
    {
    }

    __device__ __forceinline__ int block_of(int bx, int by, int bz)
    {
        if (bx == cbx && by == cby && bz == cbz) return cblk;
        if (bx == obx && by == oby && bz == obz) return oblk;
        obx = bx;
        oby = by;
        obz = bz;
        oblk = hash_find(m, bx, by, bz);
        return oblk;
    }

    // read_sdf (ray_tracing.cu:272-286): voxel at integer coordinates;
    // unallocated or zero weight -> invalid, 1.0
    __device__ __forceinline__ float voxel(int slot, int vx, int vy, int vz, bool& valid) const
    {
        if (slot >= 0) {
            const typename Fmt<FMT>::Word w = __ldg(Layout<FMT>::words(m, slot) + local_idx(vx, vy, vz));
            if (Fmt<FMT>::observed(w)) {
                valid = true;
                return Fmt<FMT>::tsdf(w);
            }
        }
        valid = false;
        return 1.f;
    }

    // read_sdf_interped (ray_tracing.cu:288-321). When `have0` is set, s0/v0
    // are the value and validity of corner 0 (the voxel at floor(p)), already
    // read by the caller.
    __device__ float interp(float3 p, bool& valid, bool have0 = false, float s0 = 1.f, bool v0 = false)
    {
        const float flx = floorf(p.x), fly = floorf(p.y), flz = floorf(p.z);
        const float ax = __fsub_rn(p.x, flx), ay = __fsub_rn(p.y, fly), az = __fsub_rn(p.z, flz);
        const int x0 = __float2int_rz(flx), y0 = __float2int_rz(fly), z0 = __float2int_rz(flz);
        const int x1 = __float2int_rz(floorf(__fadd_rn(p.x, 1.f)));
        const int y1 = __float2int_rz(floorf(__fadd_rn(p.y, 1.f)));
        const int z1 = __float2int_rz(floorf(__fadd_rn(p.z, 1.f)));
        float s[8];
        bool ok = true;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            bool v;
            if (c == 0 && have0) {
                s[0] = s0;
                v = v0;
            } else {
                const int vx = (c & 1) ? x1 : x0, vy = (c & 2) ? y1 : y0, vz = (c & 4) ? z1 : z0;
                s[c] = voxel(block_of(vox2blk(vx), vox2blk(vy), vox2blk(vz)), vx, vy, vz, v);
            }
            ok &= v;
        }
        const float bx = __fsub_rn(1.f, ax), by = __fsub_rn(1.f, ay), bz = __fsub_rn(1.f, az);
        const float r0 = __fmaf_rn(bx, s[0], __fmul_rn(ax, s[1]));
        const float r1 = __fmaf_rn(bx, s[2], __fmul_rn(ax, s[3]));
        const float r2 = __fmaf_rn(by, r0, __fmul_rn(ay, r1));
        const float r4 = __fmaf_rn(bx, s[4], __fmul_rn(ax, s[5]));
        const float r5 = __fmaf_rn(bx, s[6], __fmul_rn(ax, s[7]));
        const float r3 = __fmaf_rn(by, r4, __fmul_rn(ay, r5));
        valid = ok;
        return __fmaf_rn(bz, r2, __fmul_rn(az, r3));
    }
};

__device__ __forceinline__ float3 fma3(float k, float3 d, float3 r)
{
    return make_float3(__fmaf_rn(k, d.x, r.x), __fmaf_rn(k, d.y, r.y), __fmaf_rn(k, d.z, r.z));
}

// MapRenderingDelegate::operator() (ray_tracing.cu:323-400) for pixel (x, y).
template <int FMT>
__device__ __forceinline__ void trace_ray(const MapView& v, int x, int y)
{
    const RenderOut& r = v.out;
    const CamParams& c = v.cam;
    float4* out = reinterpret_cast<float4*>(reinterpret_cast<char*>(r.vmap) + (size_t)y * r.vpitch) + x;
    const float qnan = __int_as_float(0x7fffffff);
    const float4 miss = make_float4(qnan, qnan, qnan, qnan);

    float zn = 0.f, zf = kMaxDepth;
    if (r.mode == 0) {
        const int t = (y >> 3) * r.tilesX + (x >> 3);
        const unsigned long long kn = __ldg(r.zmin + t), kf = __ldg(r.zmax + t);
        if ((unsigned)(kn >> 32) != ~r.epoch || (unsigned)(kf >> 32) != r.epoch) {
            *out = miss;  // no allocated block projects into this tile
            return;
        }
        zn = __uint_as_float((unsigned)kn);
        zf = __uint_as_float((unsigned)kf);
    }

    const float3 p0 = unproject(x, y, kMinDepth, c.ifx, c.ify, c.cx, c.cy);
    const float dist0 = __fmul_rn(__fsqrt_rn(sqnorm(p0)), r.vsinv);
    float3 bs = xf_apply(v.T, p0.x, p0.y, p0.z);
    bs = make_float3(__fmul_rn(bs.x, r.vsinv), __fmul_rn(bs.y, r.vsinv), __fmul_rn(bs.z, r.vsinv));
    const float3 p1 = unproject(x, y, kMaxDepth, c.ifx, c.ify, c.cx, c.cy);
    const float dist_e = __fmul_rn(__fsqrt_rn(sqnorm(p1)), r.vsinv);
    float3 be = xf_apply(v.T, p1.x, p1.y, p1.z);
    be = make_float3(__fmul_rn(be.x, r.vsinv), __fmul_rn(be.y, r.vsinv), __fmul_rn(be.z, r.vsinv));
    const float3 dir = normalized(make_float3(__fsub_rn(be.x, bs.x), __fsub_rn(be.y, bs.y), __fsub_rn(be.z, bs.z)));
    // exit faces: +8 along axes the ray runs up (and +0), +0 along axes it runs
    // down (and -0), so a zero component gives an infinite exit distance
    const float3 inv = make_float3(__frcp_rn(dir.x), __frcp_rn(dir.y), __frcp_rn(dir.z));
    const int ox = signbit(dir.x) ? 0 : 8, oy = signbit(dir.y) ? 0 : 8, oz = signbit(dir.z) ? 0 : 8;

    float3 res = bs;
    float dist_s = dist0;
    float dist_lim = dist_e;
    if (r.mode == 0) {
        // ray length (voxels) is proportional to camera depth along a ray
        const float g = dist_e / kMaxDepth;
        const float k0 = floorf(g * zn - dist0) - 2.f;
        if (k0 > 0.f) {
            res = fma3(k0, dir, res);
            dist_s = dist0 + k0;
        }
        dist_lim = fminf(dist_e, g * zf + 2.f);
    }

    RayCtx<FMT> ctx(v.m);
    float sdf = 1.f, step;
    bool valid = false;
    while (dist_s < dist_lim) {
        const float flx = floorf(res.x), fly = floorf(res.y), flz = floorf(res.z);
        const int vx = __float2int_rz(flx), vy = __float2int_rz(fly), vz = __float2int_rz(flz);
        const int bx = vox2blk(vx), by = vox2blk(vy), bz = vox2blk(vz);
        if (bx != ctx.cbx || by != ctx.cby || bz != ctx.cbz) {
            const int s = (bx == ctx.obx && by == ctx.oby && bz == ctx.obz) ? ctx.oblk : hash_find(v.m, bx, by, bz);
            ctx.cbx = bx;
            ctx.cby = by;
            ctx.cbz = bz;
            ctx.cblk = s;
        }
        if (ctx.cblk < 0) {
            // every 1-voxel step inside this unallocated block reads (1.0, invalid):
            // jump to the last step that is still inside (at least one step)
            const float tx = ((float)(bx * 8 + ox) - res.x) * inv.x;
            const float ty = ((float)(by * 8 + oy) - res.y) * inv.y;
            const float tz = ((float)(bz * 8 + oz) - res.z) * inv.z;
            const float t = fminf(fminf(tx, ty), tz);  // fminf drops the NaN of 0 * inf
            const float k = fmaxf(1.f, ceilf(t - 1e-3f));
            res = fma3(k, dir, res);
            dist_s = __fadd_rn(dist_s, k);
            sdf = 1.f;
            valid = false;
            continue;
        }
        sdf = ctx.voxel(ctx.cblk, vx, vy, vz, valid);
        if (sdf <= 0.5f && sdf >= -0.5f) sdf = ctx.interp(res, valid, true, sdf, valid);
        if (sdf <= 0.f) break;
        step = valid ? fmaxf(__fmul_rn(sdf, r.rts), 1.f) : 1.f;
        res = fma3(step, dir, res);
        dist_s = __fadd_rn(dist_s, step);
    }

    bool found = false;
    if (sdf <= 0.f) {
        step = __fmul_rn(sdf, r.rts);
        res = fma3(step, dir, res);
        sdf = ctx.interp(res, valid);
        step = __fmul_rn(sdf, r.rts);
        res = fma3(step, dir, res);
        found = valid;
    }
    if (found) {
        const float3 o = xf_apply(v.Ti, __fdiv_rn(res.x, r.vsinv), __fdiv_rn(res.y, r.vsinv), __fdiv_rn(res.z, r.vsinv));
        *out = make_float4(o.x, o.y, o.z, 1.f);
    } else {
        *out = miss;
    }
}

__device__ __forceinline__ int ray_tiles(const MapView& v) { return ((v.cam.W + 7) >> 3) * ((v.cam.H + 3) >> 2); }

// Persistent: each warp takes one 8x4-pixel tile at a time from the queue
// (rewound by zrange_kernel) until every tile of every map is done.
template <class V, int FMT>
__global__ void __launch_bounds__(256) raycast_kernel(V views)
{
    __shared__ int pre[kMaxBatch + 1];
    map_prefix(views, [](const MapView& v) { return ray_tiles(v); }, pre);
    const int nmaps = views.count();
    const int total = pre[nmaps];
    const int lane = threadIdx.x & 31;
    for (;;) {
        int item = 0;
        if (lane == 0) item = (int)atomicAdd(views.queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        const int mi = map_of(pre, nmaps, item);
        const MapView& v = views[mi];
        const int t = item - pre[mi];
        const int tx = (v.cam.W + 7) >> 3;
        const int x = (t % tx) * 8 + (lane & 7);
        const int y = (t / tx) * 4 + (lane >> 3);
        if (x < v.cam.W && y < v.cam.H) trace_ray<FMT>(v, x, y);
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
    zrange_kernel<V><<<l.numSMs * 4, 256, 0, s>>>(views);
    return cudaGetLastError();
}

template <class V, int FMT>
static cudaError_t raycast_persistent(const V& views, const Launcher& l, cudaStream_t s)
{
    static int occ = 0;  // resident CTAs per SM of this instantiation
    if (occ == 0) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, raycast_kernel<V, FMT>, 256, 0);
        if (e != cudaSuccess || occ < 1) occ = 1;
    }
    raycast_kernel<V, FMT><<<l.numSMs * occ, 256, 0, s>>>(views);
    return cudaGetLastError();
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

template <class V>
cudaError_t launch_normals(const V& views, int totalTiles, const Launcher& l, cudaStream_t s)
{
    const int grid = totalTiles < l.numSMs * 8 ? (totalTiles > 0 ? totalTiles : 1) : l.numSMs * 8;
    normals_kernel<V><<<grid, 256, 0, s>>>(views);
    return cudaGetLastError();
}

template cudaError_t launch_zrange<OneView>(const OneView&, const Launcher&, cudaStream_t);
template cudaError_t launch_zrange<ManyViews>(const ManyViews&, const Launcher&, cudaStream_t);
template cudaError_t launch_raycast<OneView>(const OneView&, int, const Launcher&, cudaStream_t);
template cudaError_t launch_raycast<ManyViews>(const ManyViews&, int, const Launcher&, cudaStream_t);
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
