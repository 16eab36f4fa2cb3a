// Ray marcher device code (MapRenderingDelegate, src/ray_tracing.cu:255-401)
// shared by the ray-marching kernel and the persistent batch step: per-ray
// state, the sample loop, the per-warp block cache and one warp's tile.
#pragma once

#include "vmap_launch.h"

namespace vmapb {

// A warp marches one tile of 32 neighbouring rays (tw x 32/tw pixels, 8 x 4
// by default): neighbouring rays sample neighbouring voxels at similar
// depths, so a warp's loads and hash lookups share sectors.
__device__ __forceinline__ int ray_tiles(const MapView& v, int tw)
{
    const int th = 32 / tw;
    return v.out.vmap ? ((v.cam.W + tw - 1) / tw) * ((v.cam.H + th - 1) / th) : 0;
}

__device__ __forceinline__ float3 fma3(float k, float3 d, float3 r)
{
    return make_float3(__fmaf_rn(k, d.x, r.x), __fmaf_rn(k, d.y, r.y), __fmaf_rn(k, d.z, r.z));
}

// Per-lane state of one ray.
struct Ray {
    int mi;            // map index, -1 = lane idle
    int x, y;
    float3 res, dir, inv;
    float dist_s, dist_lim;
    float sdf;
    bool valid;
    int cbx, cby, cbz, cblk;  // block of the current sample
    int obx, oby, obz, oblk;  // last other block (trilinear corners)
};

template <int FMT, bool NC = true>
struct March {
    typedef Fmt<FMT> F;
    typedef typename F::Word Word;

    // read_sdf (ray_tracing.cu:272-286) on a loaded word
    static __device__ __forceinline__ float value(Word w, bool& valid)
    {
        valid = F::observed(w);
        return valid ? F::tsdf(w) : 1.f;
    }

    static __device__ __forceinline__ float voxel(const DevMap& m, int slot, int vx, int vy, int vz, bool& valid)
    {
        if (slot >= 0) return value(ld_map<NC>(Layout<FMT>::words(m, slot) + local_idx(vx, vy, vz)), valid);
        valid = false;
        return 1.f;
    }

    static __device__ __forceinline__ int block_of(const DevMap& m, Ray& r, int bx, int by, int bz)
    {
        if (bx == r.cbx && by == r.cby && bz == r.cbz) return r.cblk;
        if (bx == r.obx && by == r.oby && bz == r.obz) return r.oblk;
        r.obx = bx;
        r.oby = by;
        r.obz = bz;
        r.oblk = hash_find<NC>(m, bx, by, bz);
        return r.oblk;
    }

    // read_sdf_interped (ray_tracing.cu:288-321): corners floor(p + {0,1}^3),
    // x fastest; lerps contracted as fma((1 - a), s0, a * s1).
    static __device__ __forceinline__ float lerp8(const float* s, float ax, float ay, float az)
    {
        const float bx = __fsub_rn(1.f, ax), by = __fsub_rn(1.f, ay), bz = __fsub_rn(1.f, az);
        const float r0 = __fmaf_rn(bx, s[0], __fmul_rn(ax, s[1]));
        const float r1 = __fmaf_rn(bx, s[2], __fmul_rn(ax, s[3]));
        const float r2 = __fmaf_rn(by, r0, __fmul_rn(ay, r1));
        const float r4 = __fmaf_rn(bx, s[4], __fmul_rn(ax, s[5]));
        const float r5 = __fmaf_rn(bx, s[6], __fmul_rn(ax, s[7]));
        const float r3 = __fmaf_rn(by, r4, __fmul_rn(ay, r5));
        return __fmaf_rn(bz, r2, __fmul_rn(az, r3));
    }

    struct Corners {
        float ax, ay, az;
        int x0, y0, z0, x1, y1, z1;
        __device__ __forceinline__ bool inner() const  // all 8 corners in the block of (x0, y0, z0)
        {
            return x1 == x0 + 1 && y1 == y0 + 1 && z1 == z0 + 1 && (x0 & 7) != 7 && (y0 & 7) != 7 && (z0 & 7) != 7;
        }
    };

    // The voxel floor(p) of a sample: all the loop head needs (the block
    // lookup and the first read). The trilinear fractions and far corners are
    // computed from the same position only on the samples that interpolate,
    // so they are not live across the warp's block lookup.
    struct Cell {
        int x0, y0, z0;
    };

    static __device__ __forceinline__ Cell cell(float3 p)
    {
        Cell c;
        c.x0 = __float2int_rz(floorf(p.x));
        c.y0 = __float2int_rz(floorf(p.y));
        c.z0 = __float2int_rz(floorf(p.z));
        return c;
    }

    static __device__ __forceinline__ Corners corners(float3 p)
    {
        Corners c;
        const float flx = floorf(p.x), fly = floorf(p.y), flz = floorf(p.z);
        c.ax = __fsub_rn(p.x, flx);
        c.ay = __fsub_rn(p.y, fly);
        c.az = __fsub_rn(p.z, flz);
        c.x0 = __float2int_rz(flx);
        c.y0 = __float2int_rz(fly);
        c.z0 = __float2int_rz(flz);
        c.x1 = __float2int_rz(floorf(__fadd_rn(p.x, 1.f)));
        c.y1 = __float2int_rz(floorf(__fadd_rn(p.y, 1.f)));
        c.z1 = __float2int_rz(floorf(__fadd_rn(p.z, 1.f)));
        return c;
    }

    // 8 corner values from one block with independent loads; returns the
    // mask of observed corners (bit k = corner k)
    static __device__ __forceinline__ unsigned load8(const DevMap& m, int slot, const Corners& c, float* s)
    {
        const Word* w = Layout<FMT>::words(m, slot) + local_idx(c.x0, c.y0, c.z0);
        const Word w0 = ld_map<NC>(w), w1 = ld_map<NC>(w + 1), w2 = ld_map<NC>(w + 8), w3 = ld_map<NC>(w + 9);
        const Word w4 = ld_map<NC>(w + 64), w5 = ld_map<NC>(w + 65), w6 = ld_map<NC>(w + 72), w7 = ld_map<NC>(w + 73);
        unsigned mask = 0;
        bool v;
        s[0] = value(w0, v); mask |= (unsigned)v;
        s[1] = value(w1, v); mask |= (unsigned)v << 1;
        s[2] = value(w2, v); mask |= (unsigned)v << 2;
        s[3] = value(w3, v); mask |= (unsigned)v << 3;
        s[4] = value(w4, v); mask |= (unsigned)v << 4;
        s[5] = value(w5, v); mask |= (unsigned)v << 5;
        s[6] = value(w6, v); mask |= (unsigned)v << 6;
        s[7] = value(w7, v); mask |= (unsigned)v << 7;
        return mask;
    }

    // corners across block boundaries, from the block of corner 0 (slot0)
    // and its forward neighbour links: floor(p + 1) is floor(p) + 1 or + 2,
    // so the other corners lie in that block or in a block one step up on
    // each axis that crosses; the needed links are independent loads
    static __device__ __forceinline__ bool load8_linked(const DevMap& m, int slot0, const Corners& c, float* s)
    {
        const int mask = (vox2blk(c.x1) != vox2blk(c.x0) ? 1 : 0) | (vox2blk(c.y1) != vox2blk(c.y0) ? 2 : 0) |
                         (vox2blk(c.z1) != vox2blk(c.z0) ? 4 : 0);
        const int* L = m.nbr + 7 * (size_t)slot0;
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int vx = (k & 1) ? c.x1 : c.x0, vy = (k & 2) ? c.y1 : c.y0, vz = (k & 4) ? c.z1 : c.z0;
            const int o = k & mask;  // corner k's block, as an offset from corner 0's
            bool v;
            s[k] = voxel(m, o ? ld_map<NC>(L + o - 1) : slot0, vx, vy, vz, v);
            ok &= v;
        }
        return ok;
    }

    // corners across block boundaries when corner 0's block is not allocated:
    // one lookup per distinct block
    static __device__ __forceinline__ bool load8_general(const DevMap& m, Ray& r, const Corners& c, float* s)
    {
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int vx = (k & 1) ? c.x1 : c.x0, vy = (k & 2) ? c.y1 : c.y0, vz = (k & 4) ? c.z1 : c.z0;
            bool v;
            s[k] = voxel(m, block_of(m, r, vox2blk(vx), vox2blk(vy), vox2blk(vz)), vx, vy, vz, v);
            ok &= v;
        }
        return ok;
    }

    static __device__ __forceinline__ float interp(const DevMap& m, Ray& r, float3 p, bool& valid)
    {
        const Corners c = corners(p);
        float s[8];
        const int slot = block_of(m, r, vox2blk(c.x0), vox2blk(c.y0), vox2blk(c.z0));
        if (slot >= 0) {
            valid = c.inner() ? load8(m, slot, c, s) == 0xffu : load8_linked(m, slot, c, s);
        } else if (c.inner()) {
            valid = false;
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] = 1.f;
        } else {
            valid = load8_general(m, r, c, s);
        }
        return lerp8(s, c.ax, c.ay, c.az);
    }

    // Every 1-voxel step inside the unallocated block (bx, by, bz) reads
    // (1.0, invalid): jump to the first step past the block's exit (at least
    // one step). Exit faces: +8 where the ray runs up (and +0), +0 where it
    // runs down (and -0), so a zero component gives an infinite distance.
    static __device__ __forceinline__ void empty_jump(Ray& r, int bx, int by, int bz)
    {
        const float tx = ((float)(bx * 8 + (signbit(r.dir.x) ? 0 : 8)) - r.res.x) * r.inv.x;
        const float ty = ((float)(by * 8 + (signbit(r.dir.y) ? 0 : 8)) - r.res.y) * r.inv.y;
        const float tz = ((float)(bz * 8 + (signbit(r.dir.z) ? 0 : 8)) - r.res.z) * r.inv.z;
        const float t = fminf(fminf(tx, ty), tz);  // fminf drops the NaN of 0 * inf
        const float k = fmaxf(1.f, ceilf(t - 1e-3f));
        r.res = fma3(k, r.dir, r.res);
        r.dist_s = __fadd_rn(r.dist_s, k);
    }

    // Start a ray at pixel (x, y); false when it finishes at once (tile with
    // no allocated block: written as a miss).
    static __device__ __forceinline__ bool init(const MapView& v, Ray& r, int mi, int x, int y)
    {
        const RenderOut& o = v.out;
        const CamParams& c = v.cam;
        float zn = 0.f, zf = kMaxDepth;
        if (o.mode == 0) {
            const int t = (y >> 3) * o.tilesX + (x >> 3);
            const unsigned long long kn = ld_map<NC>(o.zmin + t), kf = ld_map<NC>(o.zmax + t);
            if ((unsigned)(kn >> 32) != ~o.epoch || (unsigned)(kf >> 32) != o.epoch) {
                const float qnan = __int_as_float(0x7fffffff);
                *(reinterpret_cast<float4*>(reinterpret_cast<char*>(o.vmap) + (size_t)y * o.vpitch) + x) =
                    make_float4(qnan, qnan, qnan, qnan);
                return false;
            }
            zn = __uint_as_float((unsigned)kn);
            zf = __uint_as_float((unsigned)kf);
        }
        const float3 p0 = unproject(x, y, kMinDepth, c.ifx, c.ify, c.cx, c.cy);
        const float dist0 = __fmul_rn(__fsqrt_rn(sqnorm(p0)), o.vsinv);
        float3 bs = xf_apply(v.T, p0.x, p0.y, p0.z);
        bs = make_float3(__fmul_rn(bs.x, o.vsinv), __fmul_rn(bs.y, o.vsinv), __fmul_rn(bs.z, o.vsinv));
        const float3 p1 = unproject(x, y, kMaxDepth, c.ifx, c.ify, c.cx, c.cy);
        const float dist_e = __fmul_rn(__fsqrt_rn(sqnorm(p1)), o.vsinv);
        float3 be = xf_apply(v.T, p1.x, p1.y, p1.z);
        be = make_float3(__fmul_rn(be.x, o.vsinv), __fmul_rn(be.y, o.vsinv), __fmul_rn(be.z, o.vsinv));
        r.dir = normalized(make_float3(__fsub_rn(be.x, bs.x), __fsub_rn(be.y, bs.y), __fsub_rn(be.z, bs.z)));
        // reciprocals only bound the empty-block jump (taken with a 1e-3 margin):
        // approximate ones suffice; 1/(+-0) stays +-inf
        r.inv = make_float3(__fdividef(1.f, r.dir.x), __fdividef(1.f, r.dir.y), __fdividef(1.f, r.dir.z));
        r.res = bs;
        r.dist_s = dist0;
        r.dist_lim = dist_e;
        if (o.mode == 0) {
            // ray length (voxels) is proportional to camera depth along a ray
            const float g = dist_e / kMaxDepth;
            const float k0 = floorf(g * zn - dist0) - 2.f;
            if (k0 > 0.f) {
                r.res = fma3(k0, r.dir, r.res);
                r.dist_s = dist0 + k0;
            }
            r.dist_lim = fminf(dist_e, g * zf + 2.f);
            // A sample nearer than zn (the nearest depth of any allocated block
            // whose projection covers this tile, less a voxel) cannot lie in an
            // allocated block: the loop would look its block up, find it empty
            // and jump. Those jumps are taken here without lookups, with the
            // loop's jump arithmetic: the same blocks and sample lattice (an
            // instrumented run found every skipped block empty; positions agree
            // with the lookup path to float rounding).
            const float lim = g * zn - 1.f;
            while (r.dist_s < lim && r.dist_s < r.dist_lim)
                empty_jump(r, vox2blk(__float2int_rz(floorf(r.res.x))), vox2blk(__float2int_rz(floorf(r.res.y))),
                           vox2blk(__float2int_rz(floorf(r.res.z))));
        }
        r.mi = mi;
        r.x = x;
        r.y = y;
        r.sdf = 1.f;
        r.valid = false;
        r.cbx = r.obx = INT_MIN;
        r.cblk = r.oblk = -1;
        return true;
    }

    // First half of a loop iteration: the key of the block the sample at res
    // falls in when that block is not the ray's current one and not its
    // cached second block (kEmptyKey otherwise: no lookup needed). The block
    // the ray leaves becomes the cached second block: the refinement step
    // after the zero crossing steps back by up to half a truncation band, and
    // at 640x480 / 5 mm it lands in that block on 27 % of rays (69 % stay in
    // the current block; an oracle count over 3.1 M crossings).
    static __device__ __forceinline__ unsigned long long lookup_key(Ray& r, const Cell& c)
    {
        const int bx = vox2blk(c.x0), by = vox2blk(c.y0), bz = vox2blk(c.z0);
        if (bx == r.cbx && by == r.cby && bz == r.cbz) return kEmptyKey;
        const bool second = bx == r.obx && by == r.oby && bz == r.obz;
        const int oblk = r.oblk;
        r.obx = r.cbx;
        r.oby = r.cby;
        r.obz = r.cbz;
        r.oblk = r.cblk;
        r.cbx = bx;
        r.cby = by;
        r.cbz = bz;
        if (second) {
            r.cblk = oblk;
            return kEmptyKey;
        }
        if (!coord_ok(bx, by, bz)) {
            r.cblk = -1;
            return kEmptyKey;
        }
        return pack_key(bx, by, bz);
    }

    // An unobserved voxel of an allocated block reads (1.0, invalid), and the
    // reference steps one voxel (ray_tracing.cu:372-378). Most rays meet none,
    // but runs of them make the slowest rays: at 640x480 / 5 mm the slowest
    // rays of the 200 slowest 8x4 tiles of a frame spend on average 13 of
    // their 19 iterations on them (an oracle count; 0.03 per ray over all
    // rays), and a tile lasts as long as its slowest ray.
    // So from an unobserved sample the next kRunAhead one-voxel samples inside
    // the same block are loaded together, and the unobserved ones that lead
    // are consumed in this iteration. The ray lands on the first sample that
    // is observed, lies outside the block or is past dist_lim, and the next
    // iteration takes it; positions and distances are the one-at-a-time
    // steps' own (the same fma and add chains).
    static constexpr int kRunAhead = 4;

    static __device__ __forceinline__ void unobserved_run(const MapView& v, Ray& r)
    {
        const Word* blk = Layout<FMT>::words(v.m, r.cblk);
        float3 q = r.res;
        float ds = r.dist_s;
        bool ok[kRunAhead];
        Word w[kRunAhead];
#pragma unroll
        for (int k = 0; k < kRunAhead; ++k) {
            q = fma3(1.f, r.dir, q);
            ds = __fadd_rn(ds, 1.f);
            const Cell c = cell(q);
            ok[k] = ds < r.dist_lim && vox2blk(c.x0) == r.cbx && vox2blk(c.y0) == r.cby && vox2blk(c.z0) == r.cbz;
            w[k] = Word();
            if (ok[k]) w[k] = ld_map<NC>(blk + local_idx(c.x0, c.y0, c.z0));
        }
        int n = 1;  // samples consumed: this one, then the leading unobserved ones ahead
        bool run = true;
#pragma unroll
        for (int k = 0; k < kRunAhead; ++k) {
            run = run && ok[k] && !F::observed(w[k]);
            n += run ? 1 : 0;
        }
        for (int k = 0; k < n; ++k) {
            r.res = fma3(1.f, r.dir, r.res);
            r.dist_s = __fadd_rn(r.dist_s, 1.f);
        }
        r.sdf = 1.f;
        r.valid = false;
    }

    // Second half: one iteration of the reference loop with the sample's block
    // (r.cblk) known; true when the ray leaves the loop.
    static __device__ __forceinline__ bool advance(const MapView& v, Ray& r, const Cell& p)
    {
        const DevMap& m = v.m;
        const int bx = r.cbx, by = r.cby, bz = r.cbz;
        if (r.cblk < 0) {
            empty_jump(r, bx, by, bz);
            r.sdf = 1.f;
            r.valid = false;
            return false;
        }
        bool valid;
        float sdf = voxel(m, r.cblk, p.x0, p.y0, p.z0, valid);  // read_sdf at floor(res)
        if (!valid) {
            unobserved_run(v, r);
            return false;
        }
        if (sdf <= 0.5f && sdf >= -0.5f) {
            float s[8];
            const Corners c = corners(r.res);  // c.x0 == p.x0 (same position)
            if (c.inner()) {
                // corner 0 is the sample just read; the other 7 are independent
                // loads (loading all 8 with every sample was measured slower)
                const Word* w = Layout<FMT>::words(m, r.cblk) + local_idx(c.x0, c.y0, c.z0);
                const Word w1 = ld_map<NC>(w + 1), w2 = ld_map<NC>(w + 8), w3 = ld_map<NC>(w + 9), w4 = ld_map<NC>(w + 64);
                const Word w5 = ld_map<NC>(w + 65), w6 = ld_map<NC>(w + 72), w7 = ld_map<NC>(w + 73);
                bool v;
                s[0] = sdf;
                s[1] = value(w1, v); valid &= v;
                s[2] = value(w2, v); valid &= v;
                s[3] = value(w3, v); valid &= v;
                s[4] = value(w4, v); valid &= v;
                s[5] = value(w5, v); valid &= v;
                s[6] = value(w6, v); valid &= v;
                s[7] = value(w7, v); valid &= v;
            } else {
                valid = load8_linked(m, r.cblk, c, s);
            }
            sdf = lerp8(s, c.ax, c.ay, c.az);
        }
        r.sdf = sdf;
        r.valid = valid;
        if (sdf <= 0.f) return true;
        const float st = valid ? fmaxf(__fmul_rn(sdf, v.out.rts), 1.f) : 1.f;
        r.res = fma3(st, r.dir, r.res);
        r.dist_s = __fadd_rn(r.dist_s, st);
        return false;
    }

    // After the loop: two refinement steps when the zero crossing was found
    // (ray_tracing.cu:381-393), then the camera-frame vertex or a miss. The
    // first step is taken here; the block of the interpolation's first corner
    // becomes the ray's current block, and its key is returned when it is
    // neither the block the ray is in nor the one it came from (4 % of
    // crossings at 640x480 / 5 mm) and has to be looked up.
    static __device__ __forceinline__ unsigned long long refine_key(const MapView& v, Ray& r)
    {
        if (!(r.sdf <= 0.f)) return kEmptyKey;
        r.res = fma3(__fmul_rn(r.sdf, v.out.rts), r.dir, r.res);
        return lookup_key(r, cell(r.res));
    }

    // The rest, with the current block's slot (r.cblk) known.
    static __device__ __forceinline__ void finish(const MapView& v, Ray& r)
    {
        const RenderOut& o = v.out;
        bool found = false;
        if (r.sdf <= 0.f) {
            bool valid;
            const float s = interp(v.m, r, r.res, valid);  // first corner's block: r.cblk
            r.res = fma3(__fmul_rn(s, o.rts), r.dir, r.res);
            found = valid;
        }
        float4 out;
        if (found) {
            const float3 q = xf_apply(v.Ti, __fdiv_rn(r.res.x, o.vsinv), __fdiv_rn(r.res.y, o.vsinv),
                                      __fdiv_rn(r.res.z, o.vsinv));
            out = make_float4(q.x, q.y, q.z, 1.f);
        } else {
            const float qnan = __int_as_float(0x7fffffff);
            out = make_float4(qnan, qnan, qnan, qnan);
        }
        *(reinterpret_cast<float4*>(reinterpret_cast<char*>(o.vmap) + (size_t)r.y * o.vpitch) + r.x) = out;
    }
};

// Per-warp block cache in shared memory (64 direct-mapped entries), shared by
// the 32 rays of the warp's tile and kept across the warp's tiles of one map.
// Called by all lanes together: lanes that miss look their block up once per
// distinct key (__match_any_sync), and each cache line gets one writer, so an
// entry's key and slot always belong together.
constexpr int kWarpCache = 64;

template <bool NC>
__device__ __forceinline__ int warp_lookup(const DevMap& m, unsigned long long key, unsigned long long* wkey,
                                           int* wslot, int lane)
{
    const unsigned full = 0xffffffffu;
    const bool need = key != kEmptyKey;
    if (!__ballot_sync(full, need)) return -1;
    const unsigned idx = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 58);
    int slot = -1;
    bool miss = false;
    if (need) {
        if (wkey[idx] == key) slot = wslot[idx];
        else miss = true;
    }
    if (__ballot_sync(full, miss)) {
        const unsigned grp = __match_any_sync(full, miss ? key : kEmptyKey);
        const int leader = __ffs(grp) - 1;
        int s = -1;
        if (miss && lane == leader) {
            const int3 b = unpack_key(key);
            s = hash_find<NC>(m, b.x, b.y, b.z);
        }
        s = __shfl_sync(full, s, leader);
        if (miss) slot = s;
        const bool writer = miss && lane == leader;
        const unsigned ig = __match_any_sync(full, writer ? (int)idx : -1);
        __syncwarp();
        if (writer && lane == __ffs(ig) - 1) {
            wkey[idx] = key;
            wslot[idx] = s;
        }
        __syncwarp();
    }
    return slot;
}

// One warp marches tile q of the nt tiles of map mi (q counts in the order
// the tiles are handed out). The warp's block cache must hold blocks of this
// map only.
template <int FMT, bool NC>
__device__ __forceinline__ void march_tile(const MapView& v, int mi, int q, int nt, int order, int tw,
                                           unsigned long long* wkey, int* wslot, int lane)
{
    typedef March<FMT, NC> M;
    typedef typename M::Cell Cell;
    const unsigned full = 0xffffffffu;
    // the map's q-th tile in the requested order (row-major tile index t):
    // 0 bottom rows first, 1 top rows first, 2 alternating from both ends
    const int t = order == 1 ? q : order == 2 ? ((q & 1) ? nt - 1 - (q >> 1) : (q >> 1)) : nt - 1 - q;
    const int tx = (v.cam.W + tw - 1) / tw;
    const int x = (t % tx) * tw + (lane % tw), y = (t / tx) * (32 / tw) + (lane / tw);
    Ray r;
    bool live = x < v.cam.W && y < v.cam.H && M::init(v, r, mi, x, y);
    const bool started = live;
    // warp-synchronous march: every lane reaches the shared lookup each
    // iteration; finished lanes idle until the tile is done, then all
    // finish together
    while (__ballot_sync(full, live)) {
        Cell c;
        unsigned long long key = kEmptyKey;
        if (live) {
            if (!(r.dist_s < r.dist_lim)) live = false;
            else {
                c = M::cell(r.res);
                key = M::lookup_key(r, c);
            }
        }
        const int slot = warp_lookup<NC>(v.m, key, wkey, wslot, lane);
        if (key != kEmptyKey) r.cblk = slot;
        if (live && M::advance(v, r, c)) live = false;
    }
    // the first refinement step's block, looked up per lane when the ray's
    // two cached blocks miss it (measured faster on the batched step than the
    // same lookup through the warp's block cache)
    if (started) {
        const unsigned long long key = M::refine_key(v, r);
        if (key != kEmptyKey) {
            const int3 b = unpack_key(key);
            r.cblk = hash_find<NC>(v.m, b.x, b.y, b.z);
        }
        M::finish(v, r);
    }
}

// Empty the warp's block cache (all lanes of the warp).
__device__ __forceinline__ void warp_cache_clear(unsigned long long* wkey, int lane)
{
    wkey[lane] = kEmptyKey;
    wkey[lane + 32] = kEmptyKey;
    __syncwarp();
}

}  // namespace vmapb
