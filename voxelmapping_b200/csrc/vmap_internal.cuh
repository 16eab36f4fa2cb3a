// Device-side building blocks shared by the kernels of libvmap_b200.
//
// Floating-point policy: every operation whose rounding decides a result that
// must match the reference's algorithm bit for bit (block coordinates,
// visibility, projective TSDF updates, marching-cubes vertices) is written
// with explicit round-to-nearest intrinsics (__fmul_rn, __fadd_rn, __fmaf_rn,
// __fdiv_rn, __fsqrt_rn). The compiler never contracts or reorders those, so
// the FP32 operation sequence is the one documented beside each helper: the
// reference's Eigen expression with nvcc's default multiply-add contraction.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cooperative_groups.h>
#include <stdint.h>

#include "../../include/vmap_c.h"

namespace vmapb {

namespace cg = cooperative_groups;

// Reference constants (include/map_struct.h:6-10).
constexpr int kBlockSide = 8;
constexpr int kBlockVoxels = 512;
constexpr float kMinDepth = 0.1f;
constexpr float kMaxDepth = 5.f;
// Slots per hash bucket: four 64-bit keys = one 32-byte L2 sector per probe.
constexpr int kSlots = 4;
constexpr int kMaxProbe = 64;  // buckets visited before VMAP_FLAG_HASH_FULL
constexpr unsigned long long kEmptyKey = ~0ull;
constexpr int kCoordLimit = 1 << 20;  // block coordinates in [-2^20, 2^20)
constexpr int kZTile = 8;             // z-range tile edge (reference SubSample 8)

// device counters (uint32 array in device memory)
enum {
    C_ALLOC = 0,   // pool bump pointer (may run past capacity on failure)
    C_VISIBLE = 1, // visible blocks of the last selection
    C_ERR = 2,     // VMAP_FLAG_* bits
    C_TRI = 3,     // triangles counted by the last polygonize
    C_FAILED = 4,  // allocations refused (pool full)
    C_RAYQ = 8,    // raycast work queue of the single-map path
    C_LINKED = 9,  // blocks [0, C_LINKED) have their neighbour links set
    C_COUNT = 16
};

// 3x4 affine transform, row-major; passed by value as a kernel argument.
struct Xf {
    float m[3][4];
};

struct DevMap {
    ulonglong2* slots;             // nBucket * kSlots: {packed block coordinates, pool slot or -1}
    unsigned long long* blockKeys; // capacity: key of each allocated block
    unsigned char* pool;           // capacity * blockBytes
    unsigned* ctr;                 // C_COUNT counters
    int* visList;                  // capacity: visible block slots
    // forward neighbour links: nbr[7 * s + k - 1] = pool slot of the block at
    // (bx + (k & 1), by + (k >> 1 & 1), bz + (k >> 2 & 1)) for block slot s,
    // or -1 while that block is not allocated; set for the blocks below
    // ctr[C_LINKED] (all of them once a z-range pass has run)
    int* nbr;                      // capacity * 7
    unsigned long long bucketMagic;  // ceil(2^64 / nBucket): remainder by multiplication
    int nBucket;
    int capacity;
    int blockBytes;
    float vs;   // voxel size
    float mu;   // truncation distance
    float wmax; // weight cap
};

// ---------------------------------------------------------------- FP32 math
// Transform<float,3,Affine> * Vector3f (map_struct.h:201,212): Eigen 3.3
// multiplies the 4x4 matrix by (v, 1), each row reduced in halves,
// (m_i0 v0 + m_i1 v1) + (m_i2 v2 + m_i3); nvcc contracts the first product of
// each half (measured on the reference's own build).
__device__ __forceinline__ float3 xf_apply(const Xf& t, float v0, float v1, float v2)
{
    float3 o;
    o.x = __fadd_rn(__fmaf_rn(t.m[0][0], v0, __fmul_rn(t.m[0][1], v1)), __fmaf_rn(t.m[0][2], v2, t.m[0][3]));
    o.y = __fadd_rn(__fmaf_rn(t.m[1][0], v0, __fmul_rn(t.m[1][1], v1)), __fmaf_rn(t.m[1][2], v2, t.m[1][3]));
    o.z = __fadd_rn(__fmaf_rn(t.m[2][0], v0, __fmul_rn(t.m[2][1], v1)), __fmaf_rn(t.m[2][2], v2, t.m[2][3]));
    return o;
}

// unproject (map_struct.h:189-194): ((ifx * (x - cx)) * z, (ify * (y - cy)) * z, z)
__device__ __forceinline__ float3 unproject(int x, int y, float z, float ifx, float ify, float cx, float cy)
{
    return make_float3(__fmul_rn(__fmul_rn(ifx, __fsub_rn(__int2float_rn(x), cx)), z),
                       __fmul_rn(__fmul_rn(ify, __fsub_rn(__int2float_rn(y), cy)), z), z);
}

// Eigen squaredNorm: v0^2 + (v1^2 + v2^2), contracted.
__device__ __forceinline__ float sqnorm(float3 v)
{
    return __fmaf_rn(v.x, v.x, __fmaf_rn(v.y, v.y, __fmul_rn(v.z, v.z)));
}

// Eigen normalized(): v / sqrt(|v|^2) if |v|^2 > 0 else v. Inside
// normalized() nvcc contracts the squared norm's inner sum the other way,
// v0^2 + (v2^2 + v1^2) (measured on the reference's own build).
__device__ __forceinline__ float3 normalized(float3 v)
{
    const float s = __fmaf_rn(v.x, v.x, __fmaf_rn(v.z, v.z, __fmul_rn(v.y, v.y)));
    if (s > 0.f) {
        const float n = __fsqrt_rn(s);
        v.x = __fdiv_rn(v.x, n);
        v.y = __fdiv_rn(v.y, n);
        v.z = __fdiv_rn(v.z, n);
    }
    return v;
}

// Eigen cross(): a1 b2 - a2 b1, ... contracted as fma(a1, b2, -(a2 b1)).
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return make_float3(__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
                       __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}

// ------------------------------------------------------- coordinate helpers
// voxelPosToBlockPos (map_struct.h:131-141) == floor division by 8.
__device__ __forceinline__ int vox2blk(int v) { return v >> 3; }
// localPosToLocalIdx(voxelPosToLocalPos(v)) (map_struct.h:148-180).
__device__ __forceinline__ int local_idx(int vx, int vy, int vz)
{
    return ((vz & 7) << 6) | ((vy & 7) << 3) | (vx & 7);
}

__device__ __forceinline__ bool coord_ok(int x, int y, int z)
{
    return x >= -kCoordLimit && x < kCoordLimit && y >= -kCoordLimit && y < kCoordLimit && z >= -kCoordLimit &&
           z < kCoordLimit;
}

// voxel coordinates whose blocks are representable: [-2^23, 2^23)
__device__ __forceinline__ bool voxel_ok(int x, int y, int z)
{
    constexpr int lim = kCoordLimit * kBlockSide;
    return x >= -lim && x < lim && y >= -lim && y < lim && z >= -lim && z < lim;
}

__device__ __forceinline__ unsigned long long pack_key(int x, int y, int z)
{
    return ((unsigned long long)(x & 0x1FFFFF) << 42) | ((unsigned long long)(y & 0x1FFFFF) << 21) |
           (unsigned long long)(z & 0x1FFFFF);
}

__device__ __forceinline__ int3 unpack_key(unsigned long long k)
{
    return make_int3((int)((long long)(k << 1) >> 43), (int)((long long)(k << 22) >> 43),
                     (int)((long long)(k << 43) >> 43));
}

// hash (map_struct.h:104-109): int32 wrap-around products, C remainder,
// shifted non-negative.
__device__ __forceinline__ int ref_hash(int x, int y, int z, int nb)
{
    int r = (int)(((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^ ((unsigned)z * 83492791u));
    r %= nb;
    return r < 0 ? r + nb : r;
}

// The same value with the remainder taken by multiplication (Lemire, Kaser and
// Kurz, "Faster remainder by direct computation", 2019): for 32-bit a and d,
// a mod d = hi64((M * a mod 2^64) * d) with M = ceil(2^64 / d). C's remainder
// of a negative r has the sign of r, so |r| mod d is negated and shifted.
__host__ __device__ __forceinline__ unsigned long long bucket_magic(unsigned d)
{
    return ~0ull / d + 1ull;
}

__device__ __forceinline__ int ref_hash_fast(int x, int y, int z, int nb, unsigned long long magic)
{
    const int r = (int)(((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^ ((unsigned)z * 83492791u));
    const unsigned a = r < 0 ? 0u - (unsigned)r : (unsigned)r;
    const unsigned mod = (unsigned)__umul64hi(magic * a, (unsigned long long)nb);
    return r < 0 ? (mod ? nb - (int)mod : 0) : (int)mod;
}

// checkBlockVisible (map_struct.h:219-244): any of the 8 block corners
// projects inside [0, cols-1] x [0, rows-1] with depth in [0.1, 5].
__device__ __forceinline__ bool block_visible(int bx, int by, int bz, const Xf& ti, float scale, int cols,
                                              int rows, float fx, float fy, float cx, float cy)
{
    const float cmax = __int2float_rn(cols - 1), rmax = __int2float_rn(rows - 1);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float3 p = xf_apply(ti, __fmul_rn(__int2float_rn(bx + (c & 1)), scale),
                                  __fmul_rn(__int2float_rn(by + ((c >> 1) & 1)), scale),
                                  __fmul_rn(__int2float_rn(bz + ((c >> 2) & 1)), scale));
        const float px = __fadd_rn(__fdiv_rn(__fmul_rn(fx, p.x), p.z), cx);
        const float py = __fadd_rn(__fdiv_rn(__fmul_rn(fy, p.y), p.z), cy);
        if (!(px < 0.f || py < 0.f || px > cmax || py > rmax || p.z < kMinDepth || p.z > kMaxDepth)) return true;
    }
    return false;
}

// ------------------------------------------------ programmatic dependent launch
// A single map's per-frame stage kernels are launched with programmatic
// stream serialization (launch_stage): a stage's CTAs may be scheduled while
// the previous kernel on the stream drains, hiding the launch between
// dependent stages. Every stage kernel calls stage_entry() first, before it reads or
// writes anything: griddepcontrol.wait returns once the previous kernel has
// completed and its writes are visible (at once for a launch without a
// programmatic dependency), and launch_dependents then lets the next stage be
// scheduled. Each stage waits for its predecessor, so completion is ordered
// along the whole chain.
__device__ __forceinline__ void stage_entry()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ------------------------------------------------------------- map loads
// Stage kernels read map data that no thread writes while the kernel runs
// (hash slots, voxels, links, tile bounds, vertex maps) through the read-only
// path (NC = true). The persistent batch step writes such data in one stage
// and reads it in a later one of the same launch, so it reads with plain
// loads (NC = false), ordered after the acquire that opened the stage.
template <bool NC, class T>
__device__ __forceinline__ T ld_map(const T* p)
{
    if constexpr (NC) return __ldg(p);
    else return *p;
}

// ------------------------------------------------------------- hash table
// Bucketed open hashing: bucket = reference hash of the block coordinates,
// 4 slots per bucket (key and pool slot side by side: one 64-byte read per
// probe, no second round trip for the value), linear probing into the next
// bucket when all 4 are taken. Slots go EMPTY -> key exactly once, so the
// filled slots of a bucket always form a prefix: a lookup stops at the first
// EMPTY slot.
template <bool NC = true>
__device__ __forceinline__ int hash_find(const DevMap& m, int bx, int by, int bz)
{
    if (!coord_ok(bx, by, bz)) return -1;
    const unsigned long long key = pack_key(bx, by, bz);
    int b = ref_hash_fast(bx, by, bz, m.nBucket, m.bucketMagic);
#pragma unroll 1
    for (int p = 0; p < kMaxProbe; ++p) {
        const ulonglong2* s = m.slots + (size_t)b * kSlots;
        const ulonglong2 a0 = ld_map<NC>(s), a1 = ld_map<NC>(s + 1), a2 = ld_map<NC>(s + 2), a3 = ld_map<NC>(s + 3);
        if (a0.x == key) return (int)a0.y;
        if (a0.x == kEmptyKey) return -1;
        if (a1.x == key) return (int)a1.y;
        if (a1.x == kEmptyKey) return -1;
        if (a2.x == key) return (int)a2.y;
        if (a2.x == kEmptyKey) return -1;
        if (a3.x == key) return (int)a3.y;
        if (a3.x == kEmptyKey) return -1;
        b = (b + 1 == m.nBucket) ? 0 : b + 1;
    }
    return -1;
}

// Insert a block if absent (createBlock, map_struct.h:304-354, without its
// lock: a compare-and-swap claims an empty slot, losers re-read). The winner
// takes the next pool slot from a warp-aggregated bump counter, which hands
// out blocks in the reference's heap order 0, 1, 2, ...
__device__ __forceinline__ void hash_insert(const DevMap& m, int bx, int by, int bz)
{
    const unsigned long long key = pack_key(bx, by, bz);
    int b = ref_hash_fast(bx, by, bz, m.nBucket, m.bucketMagic);
#pragma unroll 1
    for (int p = 0; p < kMaxProbe; ++p) {
        ulonglong2* s = m.slots + (size_t)b * kSlots;
        const unsigned long long k[4] = {__ldcg(&s[0].x), __ldcg(&s[1].x), __ldcg(&s[2].x), __ldcg(&s[3].x)};
#pragma unroll
        for (int i = 0; i < kSlots; ++i) {
            unsigned long long cur = k[i];
            if (cur == kEmptyKey) cur = atomicCAS(&s[i].x, kEmptyKey, key);
            if (cur == key) return;  // present (or inserted by another thread)
            if (cur == kEmptyKey) {  // this thread won the slot
                cg::coalesced_group g = cg::coalesced_threads();
                unsigned first = 0;
                if (g.thread_rank() == 0) first = atomicAdd(m.ctr + C_ALLOC, g.size());
                const unsigned slot = g.shfl(first, 0) + g.thread_rank();
                if (slot < (unsigned)m.capacity) {
                    m.blockKeys[slot] = key;
                    s[i].y = (unsigned long long)slot;
                } else {
                    atomicOr(m.ctr + C_ERR, VMAP_FLAG_POOL_FULL);
                    atomicAdd(m.ctr + C_FAILED, 1u);
                }
                return;
            }
        }
        b = (b + 1 == m.nBucket) ? 0 : b + 1;
    }
    atomicOr(m.ctr + C_ERR, VMAP_FLAG_HASH_FULL);
}

__device__ __forceinline__ int allocated_blocks(const DevMap& m)
{
    const unsigned n = *((volatile const unsigned*)(m.ctr + C_ALLOC));
    return n < (unsigned)m.capacity ? (int)n : m.capacity;
}

// ------------------------------------------------------------ voxel formats
// Each voxel's TSDF and weight share one word so a sample is one load:
// 4 bytes (REF, F16, I16) or 8 bytes (F32). Block layout in the pool:
// [word x512][r x512][g x512][b x512], voxel index x + 8y + 64z; colour
// planes only when the map keeps colour. A voxel with weight 0 is unobserved.
template <int FMT>
struct Fmt;

template <>
struct Fmt<VMAP_VOXEL_REF> {  // reference Voxel: int16 x32767 tsdf, uint8 weight
    typedef unsigned Word;      // bits 0-15 tsdf code, 16-23 weight
    // unpackFloat (map_struct.h:72-75): val / 32767.f
    static __device__ __forceinline__ float tsdf(Word w) { return __fdiv_rn(__int2float_rn((short)(w & 0xffffu)), 32767.f); }
    static __device__ __forceinline__ float weight(Word w) { return __uint2float_rn((w >> 16) & 0xffu); }
    static __device__ __forceinline__ bool observed(Word w) { return (w >> 16) != 0u; }
    // packFloat (map_struct.h:77-80): (short)(val * 32767), truncation
    static __device__ __forceinline__ Word make(float t, float wt)
    {
        return (unsigned)(unsigned short)(short)__float2int_rz(__fmul_rn(t, 32767.f)) | (__float2uint_rz(wt) << 16);
    }
};

template <>
struct Fmt<VMAP_VOXEL_F32> {
    typedef float2 Word;  // x tsdf, y weight
    static __device__ __forceinline__ float tsdf(Word w) { return w.x; }
    static __device__ __forceinline__ float weight(Word w) { return w.y; }
    static __device__ __forceinline__ bool observed(Word w) { return w.y != 0.f; }
    static __device__ __forceinline__ Word make(float t, float wt) { return make_float2(t, wt); }
};

template <>
struct Fmt<VMAP_VOXEL_F16> {
    typedef unsigned Word;  // bits 0-15 IEEE half tsdf, 16-31 uint16 weight
    static __device__ __forceinline__ float tsdf(Word w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu))); }
    static __device__ __forceinline__ float weight(Word w) { return __uint2float_rn(w >> 16); }
    static __device__ __forceinline__ bool observed(Word w) { return (w >> 16) != 0u; }
    static __device__ __forceinline__ Word make(float t, float wt)
    {
        return (unsigned)__half_as_ushort(__float2half_rn(t)) | (__float2uint_rz(wt) << 16);
    }
};

template <>
struct Fmt<VMAP_VOXEL_I16> {
    typedef unsigned Word;  // bits 0-15 int16 x32767 tsdf, 16-31 uint16 weight
    static __device__ __forceinline__ float tsdf(Word w) { return __fdiv_rn(__int2float_rn((short)(w & 0xffffu)), 32767.f); }
    static __device__ __forceinline__ float weight(Word w) { return __uint2float_rn(w >> 16); }
    static __device__ __forceinline__ bool observed(Word w) { return (w >> 16) != 0u; }
    static __device__ __forceinline__ Word make(float t, float wt)
    {
        return (unsigned)(unsigned short)(short)__float2int_rz(__fmul_rn(t, 32767.f)) | (__float2uint_rz(wt) << 16);
    }
};

template <int FMT>
struct Layout {
    typedef typename Fmt<FMT>::Word Word;
    static constexpr int kWordBytes = (int)sizeof(Word);
    static constexpr int kRgbOff = kBlockVoxels * kWordBytes;
    static __host__ __device__ constexpr int bytes(bool color)
    {
        return kBlockVoxels * kWordBytes + (color ? 3 * kBlockVoxels : 0);
    }
    static __device__ __forceinline__ const Word* words(const DevMap& m, int slot)
    {
        return reinterpret_cast<const Word*>(m.pool + (size_t)slot * m.blockBytes);
    }
    static __device__ __forceinline__ Word* words_rw(const DevMap& m, int slot)
    {
        return reinterpret_cast<Word*>(m.pool + (size_t)slot * m.blockBytes);
    }
};

// 16-byte vectorised copies of NBYTES (a multiple of 4; 16-byte aligned when >= 16).
template <int NBYTES>
__device__ __forceinline__ void load_vec(const void* src, void* dst)
{
    static_assert(NBYTES == 4 || NBYTES == 8 || NBYTES % 16 == 0, "vector size");
    if constexpr (NBYTES == 4) {
        *reinterpret_cast<unsigned*>(dst) = *reinterpret_cast<const unsigned*>(src);
    } else if constexpr (NBYTES == 8) {
        *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(src);
    } else {
#pragma unroll
        for (int i = 0; i < NBYTES / 16; ++i)
            reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
    }
}

template <int NBYTES>
__device__ __forceinline__ void store_vec(void* dst, const void* src)
{
    if constexpr (NBYTES == 4) {
        *reinterpret_cast<unsigned*>(dst) = *reinterpret_cast<const unsigned*>(src);
    } else if constexpr (NBYTES == 8) {
        *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(src);
    } else {
#pragma unroll
        for (int i = 0; i < NBYTES / 16; ++i)
            reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
    }
}

}  // namespace vmapb

namespace vmapb {

// ------------------------------------------------------------- map views
// Everything one stage kernel needs about one map for one step. Kernels are
// written over a "view source": OneView (a single map, passed by value as the
// kernel argument) or ManyViews (an array of views in device memory, one per
// map of a batch). Work of a stage is split over the maps with per-map item
// counts and a prefix sum computed at kernel start.
struct CamParams {
    int W, H;
    float fx, fy, cx, cy;
    float ifx, ify;  // (float)(1.0 / (double)f), as the reference's host code
};

struct FrameIn {
    int active;      // this map selects visible blocks / fuses this step
    const void* depth;
    size_t dpitch;
    int dtype;       // VMAP_DEPTH_*
    float dscale;    // uint16 -> metres
    const uint8_t* rgb;  // uint8x3 per pixel or NULL
    size_t rgbPitch;
};

struct RenderOut {
    float4* vmap;
    size_t vpitch;
    float4* nmap;    // may be NULL
    size_t npitch;
    // tile depth bounds, tagged with the render epoch in the high word:
    // zmin = (~epoch << 32 | float bits), folded with atomicMin; zmax =
    // (epoch << 32 | float bits), folded with atomicMax. A newer epoch always
    // wins, so the tiles never need clearing between renders.
    unsigned long long* zmin;
    unsigned long long* zmax;
    unsigned epoch;  // 1 .. 2^32 - 2
    int tilesX, tilesY;
    float vsinv;     // (float)(1.0 / (double)voxel_size)
    float rts;       // truncation / voxel_size (raytraceStep)
    int mode;        // 0: z-range bounded, 1: full march
};

struct MapView {
    DevMap m;
    CamParams cam;
    FrameIn in;
    RenderOut out;
    Xf T;   // camera -> world
    Xf Ti;  // world -> camera
};

constexpr int kMaxBatch = 256;

struct OneView {
    MapView v;
    unsigned* queue;  // work-queue counters of this step
    __device__ __forceinline__ int count() const { return 1; }
    __device__ __forceinline__ const MapView& operator[](int) const { return v; }
};

struct ManyViews {
    const MapView* v;
    int n;
    unsigned* queue;
    __device__ __forceinline__ int count() const { return n; }
    __device__ __forceinline__ const MapView& operator[](int i) const { return v[i]; }
};

// Exclusive prefix of per-map item counts in shared memory (pre[0..n]),
// computed by the first warp; the CTA must call it uniformly.
template <class V, class F>
__device__ __forceinline__ void map_prefix(const V& views, F items, int* pre)
{
    const int n = views.count();
    if (threadIdx.x < 32) {
        int run = 0;
        for (int base = 0; base < n; base += 32) {
            const int i = base + (int)threadIdx.x;
            int v = i < n ? items(views[i]) : 0;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, d);
                if ((int)threadIdx.x >= d) v += u;
            }
            if (i < n) pre[i + 1] = run + v;
            run += __shfl_sync(0xffffffffu, v, 31);
        }
        if (threadIdx.x == 0) pre[0] = 0;
    }
    __syncthreads();
}

// Map owning item i: largest m with pre[m] <= i (pre is non-decreasing).
__device__ __forceinline__ int map_of(const int* pre, int n, int i)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace vmapb
