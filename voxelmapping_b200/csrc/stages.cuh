// Per-item bodies of the fusion and render stages, shared by the stage
// kernels (one launch per stage, fusion.cu and raycast.cu) and the persistent
// batch step (step.cu): one depth pixel's block band, one visibility group,
// four voxels of a fused block, one neighbour-link or z-range task, one
// normal-map pixel. Both schedules run the same arithmetic, so their results
// are identical.
//
// Reference: src/depth_fusion.cu (CreateBlockLineTracingFunctor :32-59,
// CheckEntryVisibilityFunctor :82-126, DepthFusionFunctor / ImageFusionFunctor
// :148-196, 328-380), src/ray_tracing.cu (RenderingBlockDelegate :13-137) and
// src/image_proc.cu (computeNormalKernel :74-93).
#pragma once

#include <climits>

#include "vmap_launch.h"

namespace vmapb {

// ---------------------------------------------------------------- frames
// Depth and colour frames are inputs: nothing writes them while a kernel runs.
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

// ---------------------------------------------------------------- allocation
// 32 x TH-pixel tiles of a map's frame; maps without fusion work this step
// (no frame) contribute none.
template <int TH>
__device__ __forceinline__ int alloc_tiles(const MapView& v)
{
    return v.in.active ? ((v.cam.W + 31) >> 5) * ((v.cam.H + TH - 1) / TH) : 0;
}

constexpr int ilog2(int n) { return n > 1 ? 1 + ilog2(n >> 1) : 0; }

// Stage block key (bx, by, bz) in an open-addressed shared-memory set of SET
// keys; after 32 occupied probes the block goes straight into the hash
// table, which leaves the block set unchanged.
template <int SET>
__device__ __forceinline__ void stage_block(unsigned long long* set, const DevMap& m, unsigned long long key, int bx,
                                            int by, int bz)
{
    static_assert((SET & (SET - 1)) == 0, "power of two");
    unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> (64 - ilog2(SET)));
#pragma unroll 1
    for (int p = 0; p < 32; ++p) {
        const unsigned long long cur = atomicCAS(set + h, kEmptyKey, key);
        if (cur == kEmptyKey || cur == key) return;
        h = (h + 1) & (SET - 1);
    }
    hash_insert(m, bx, by, bz);
}

// Insert the staged blocks into the hash table and empty the set; threads
// t, t + nt, ... of the set's users take one entry each.
template <int SET>
__device__ __forceinline__ void insert_staged(unsigned long long* set, const DevMap& m, int t, int nt)
{
    for (int i = t; i < SET; i += nt) {
        const unsigned long long key = set[i];
        if (key != kEmptyKey) {
            set[i] = kEmptyKey;
            const int3 c = unpack_key(key);
            hash_insert(m, c.x, c.y, c.z);
        }
    }
}

// CreateBlockLineTracingFunctor for pixel (x, y) of depth d: the band
// [d - mu/2, d + mu/2] is unprojected to world voxel coordinates and sampled
// at ceil(2 |far - near|) points; `stage` is called with each block the
// samples enter (once per run of consecutive samples inside one block).
template <class Stage>
__device__ __forceinline__ void band_blocks_at(const MapView& v, int x, int y, float d, Stage stage)
{
    const DevMap& m = v.m;
    if (isnan(d) || d < kMinDepth || d > kMaxDepth) return;
    const float tdh = __fmul_rn(m.mu, 0.5f);
    const float dn = fmaxf(kMinDepth, __fsub_rn(d, tdh));
    const float df = fmaxf(kMinDepth, __fadd_rn(d, tdh));
    if (!(dn < df)) return;
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
    // band end points outside the +-2^23-voxel (+-2^20-block) key range cannot
    // be stored: flag and skip the pixel (every sample lies between the two
    // end points)
    if (!voxel_ok(nx, ny, nz) || !voxel_ok(fx, fy, fz)) {
        atomicOr(m.ctr + C_ERR, VMAP_FLAG_RANGE);
        return;
    }
    float3 dir = make_float3(__int2float_rn(fx - nx), __int2float_rn(fy - ny), __int2float_rn(fz - nz));
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
        if (bx != lbx || by != lby || bz != lbz) {
            lbx = bx;
            lby = by;
            lbz = bz;
            if (coord_ok(bx, by, bz)) stage(pack_key(bx, by, bz), bx, by, bz);
            else atomicOr(m.ctr + C_ERR, VMAP_FLAG_RANGE);
        }
        px = __fadd_rn(px, dx);
        py = __fadd_rn(py, dy);
        pz = __fadd_rn(pz, dz);
    }
}

// the same with the pixel's depth read here
template <class Stage>
__device__ __forceinline__ void band_blocks(const MapView& v, int x, int y, Stage stage)
{
    band_blocks_at(v, x, y, read_depth(v.in, x, y), stage);
}

// ---------------------------------------------------------------- visibility
// checkBlockVisible over allocated blocks [32 g, 32 g + 32) of one map, one
// warp (every lane calls): visible slots are appended to the map's visible
// list with one atomic per warp.
__device__ __forceinline__ void visibility_group(const MapView& v, int g, int lane)
{
    const DevMap& m = v.m;
    const int i = g * 32 + lane;
    bool vis = false;
    if (i < allocated_blocks(m)) {
        const int3 b = unpack_key(m.blockKeys[i]);
        vis = block_visible(b.x, b.y, b.z, v.Ti, __fmul_rn(m.vs, 8.f), v.cam.W, v.cam.H, v.cam.fx, v.cam.fy, v.cam.cx,
                            v.cam.cy);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, vis);
    if (mask == 0) return;
    unsigned first = 0;
    if (lane == 0) first = atomicAdd(m.ctr + C_VISIBLE, (unsigned)__popc(mask));
    first = __shfl_sync(0xffffffffu, first, 0);
    if (vis) m.visList[first + __popc(mask & ((1u << lane) - 1))] = i;
}

// ----------------------------------------------------------------- fusion
// DepthFusionFunctor / ImageFusionFunctor for the NV (4 or 8) consecutive
// voxels v0 .. v0 + NV - 1 of an x-row of block `slot` (one vector of NV
// voxel words, one NV-byte word per colour plane). The projections come
// first: each projected pixel's depth and colour are loaded right after its
// projection, and the group's voxel words and colour planes only when one of
// its voxels updates, so groups behind the surface or outside the frame move
// no voxel bytes. Nothing is written unless a voxel updates.
template <int FMT, bool COLOR, int DT, int NV = 4>
__device__ __forceinline__ void fuse_block(const MapView& v, int slot, int v0)
{
    typedef Layout<FMT> L;
    typedef typename L::Word Word;
    typedef Fmt<FMT> F;
    const DevMap& m = v.m;
    const int lx0 = v0 & 7, ly = (v0 >> 3) & 7, lz = v0 >> 6;
    const int3 bp = unpack_key(m.blockKeys[slot]);
    Word* blk = L::words_rw(m, slot);
    static_assert(NV == 4 || NV == 8, "4 or 8 voxels of an x-row");
    Word w[NV];
    unsigned char c[3][NV];
    unsigned char* crow = reinterpret_cast<unsigned char*>(blk) + L::kRgbOff + v0;
    const int vx0 = bp.x * 8 + lx0;
    const float wy = __fmul_rn(__int2float_rn(bp.y * 8 + ly), m.vs);
    const float wz = __fmul_rn(__int2float_rn(bp.z * 8 + lz), m.vs);
    float sdfv[NV];
    unsigned pix[NV];  // the projected pixel's colour, r | g << 8 | b << 16
    unsigned mask = 0;
#pragma unroll
    for (int x = 0; x < NV; ++x) {
        const float3 p = xf_apply(v.Ti, __fmul_rn(__int2float_rn(vx0 + x), m.vs), wy, wz);
        // __float2int_rd(fx * p0 / p2 + cx + 0.5)
        const int u = __float2int_rd(__fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(v.cam.fx, p.x), p.z), v.cam.cx), 0.5f));
        const int vv = __float2int_rd(__fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(v.cam.fy, p.y), p.z), v.cam.cy), 0.5f));
        sdfv[x] = 0.f;
        pix[x] = 0u;
        if (u < 0 || vv < 0 || u > v.cam.W - 1 || vv > v.cam.H - 1) continue;
        const float d = read_depth_t<DT>(v.in, u, vv);
        if constexpr (COLOR) {
            const uint8_t* px = v.in.rgb + (size_t)vv * v.in.rgbPitch + 3 * u;
            pix[x] = (unsigned)__ldg(px) | ((unsigned)__ldg(px + 1) << 8) | ((unsigned)__ldg(px + 2) << 16);
        }
        if (isnan(d) || d > kMaxDepth || d < kMinDepth) continue;
        const float sdf = __fsub_rn(d, p.z);
        if (sdf < -m.mu) continue;
        sdfv[x] = fminf(1.f, __fdiv_rn(sdf, m.mu));
        mask |= 1u << x;
    }
    if (!mask) return;
    load_vec<NV * sizeof(Word)>(blk + v0, w);
    if constexpr (COLOR) {
#pragma unroll
        for (int k = 0; k < 3; ++k) load_vec<NV>(crow + k * kBlockVoxels, c[k]);
    }
#pragma unroll
    for (int x = 0; x < NV; ++x) {
        if (!(mask & (1u << x))) continue;
        const float ow = F::weight(w[x]);
        if (ow == 0.f) {
            w[x] = F::make(sdfv[x], 1.f);
            if constexpr (COLOR) {
#pragma unroll
                for (int k = 0; k < 3; ++k) c[k][x] = (unsigned char)(pix[x] >> (8 * k));
            }
        } else {
            const float os = F::tsdf(w[x]);
            w[x] = F::make(__fdiv_rn(__fmaf_rn(os, ow, sdfv[x]), __fadd_rn(ow, 1.f)), fminf(__fadd_rn(ow, 1.f), m.wmax));
            if constexpr (COLOR) {
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    c[k][x] = (unsigned char)__float2int_rz(__fmaf_rn(
                        0.7f, __uint2float_rn(c[k][x]), __fmul_rn(0.3f, __uint2float_rn((pix[x] >> (8 * k)) & 0xffu))));
            }
        }
    }
    store_vec<NV * sizeof(Word)>(blk + v0, w);
    if constexpr (COLOR) {
#pragma unroll
        for (int k = 0; k < 3; ++k) store_vec<NV>(crow + k * kBlockVoxels, c[k]);
    }
}

// fuse_block for the frame's depth type; colour when the frame carries it
// (the map must keep colour).
template <int FMT, int NV = 4>
__device__ __forceinline__ void fuse_voxels(const MapView& v, int slot, int v0)
{
    const bool color = v.in.rgb != nullptr;
    if (v.in.dtype == VMAP_DEPTH_U16) {
        if (color) fuse_block<FMT, true, VMAP_DEPTH_U16, NV>(v, slot, v0);
        else fuse_block<FMT, false, VMAP_DEPTH_U16, NV>(v, slot, v0);
    } else {
        if (color) fuse_block<FMT, true, VMAP_DEPTH_F32, NV>(v, slot, v0);
        else fuse_block<FMT, false, VMAP_DEPTH_F32, NV>(v, slot, v0);
    }
}

// ------------------------------------------------------------------ z-range
// Neighbour links of the blocks allocated since the last render,
// [ctr[C_LINKED], allocated): each new block is 14 independent tasks, one
// lookup each - its 7 forward links, and the link of each of its 7 backward
// neighbours that points at it. Two new neighbours write each other's link
// with the same value, so the order of the writes does not matter.
__device__ __forceinline__ int links_pending(const MapView& v)
{
    if (!v.out.vmap) return 0;
    const int done = (int)*((volatile const unsigned*)(v.m.ctr + C_LINKED));
    const int n = allocated_blocks(v.m);
    return n > done ? 14 * (n - done) : 0;
}

template <bool NC>
__device__ __forceinline__ void link_task(const DevMap& m, int t)
{
    const int slot = (int)*((volatile const unsigned*)(m.ctr + C_LINKED)) + t / 14;
    const int k = 1 + (t % 14) / 2, dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
    const int3 b = unpack_key(m.blockKeys[slot]);
    if (t & 1) {  // a backward neighbour's link to this block
        const int e = hash_find<NC>(m, b.x - dx, b.y - dy, b.z - dz);
        if (e >= 0) m.nbr[7 * (size_t)e + k - 1] = slot;
    } else {
        m.nbr[7 * (size_t)slot + k - 1] = hash_find<NC>(m, b.x + dx, b.y + dy, b.z + dz);
    }
}

// z-range tiles are folded from every allocated block of a map rendered in
// mode 0
__device__ __forceinline__ int zrange_blocks(const MapView& v)
{
    return v.out.vmap && v.out.mode == 0 ? allocated_blocks(v.m) : 0;
}

constexpr float kClipZ = 0.05f;  // below the ray start depth of 0.1 m

// Block `slot`: the part of the block in front of the plane z = kClipZ
// (corners in front, plus the points where its 12 edges cross the plane) is
// projected; its pixel bounding box (+1 px) and depth range (+-1 voxel) are
// folded into the 8x8-pixel tile maps with 64-bit atomics on epoch-tagged
// values (depths are positive, so float order == bit order). Every point of a
// block is a convex combination of its corners, so the box and range bound
// every ray sample that can fall inside the block.
__device__ __forceinline__ void zrange_block(const MapView& v, int slot)
{
    const DevMap& m = v.m;
    const RenderOut& r = v.out;
    const int3 b = unpack_key(m.blockKeys[slot]);
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
    if (zhi <= kClipZ || zhi < kMinDepth - m.vs || zlo > kMaxDepth + m.vs) return;
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
    if (umax < -1.f || vmax < -1.f || umin > (float)W || vmin > (float)H) return;
    const int tx0 = max(0, (int)floorf(fmaxf(umin - 1.f, -8.f)) >> 3);
    const int tx1 = min(r.tilesX - 1, (int)floorf(fminf(umax + 1.f, (float)W + 8.f)) >> 3);
    const int ty0 = max(0, (int)floorf(fmaxf(vmin - 1.f, -8.f)) >> 3);
    const int ty1 = min(r.tilesY - 1, (int)floorf(fminf(vmax + 1.f, (float)H + 8.f)) >> 3);
    const unsigned long long lo = ((unsigned long long)(~r.epoch) << 32) | __float_as_uint(fmaxf(zlo - m.vs, 0.f));
    const unsigned long long hi = ((unsigned long long)r.epoch << 32) | __float_as_uint(zhi + m.vs);
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int t = ty * r.tilesX + tx;
            atomicMin(r.zmin + t, lo);
            atomicMax(r.zmax + t, hi);
        }
}

// ------------------------------------------------------------------ normals
// computeNormalKernel: normalize((v[x+1] - v[x-1]) x (v[y+1] - v[y-1])),
// w = 1. Undefined pixels (last row / column, NaN neighbour) are written
// all-NaN. Work is split into 32-pixel-wide tiles of every map that wants a
// normal map.
template <int TH>
__device__ __forceinline__ int normal_tiles(const MapView& v)
{
    return v.out.nmap ? ((v.cam.W + 31) >> 5) * ((v.cam.H + TH - 1) / TH) : 0;
}

template <bool NC>
__device__ __forceinline__ void normal_pixel(const MapView& v, int x, int y)
{
    const int W = v.cam.W, H = v.cam.H;
    if (x >= W || y >= H) return;
    const float qnan = __int_as_float(0x7fffffff);
    float4 res = make_float4(qnan, qnan, qnan, qnan);
    if (x < W - 1 && y < H - 1) {
        const char* vm = reinterpret_cast<const char*>(v.out.vmap);
        const size_t vp = v.out.vpitch;
        auto at = [&](int xx, int yy) { return ld_map<NC>(reinterpret_cast<const float4*>(vm + (size_t)yy * vp) + xx); };
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

}  // namespace vmapb
