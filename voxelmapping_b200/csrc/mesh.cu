// Marching cubes over all allocated blocks, triangle centroids and the dense
// block export.
//
// Reference: src/marching_cubes.cu (select_blocks :25-50, read_sdf_list
// :68-104, interpolateLinear :106-115, make_vertex :117-207, emit loop
// :209-242, compute_surface_point_kernel :314-328). The reference runs 64
// threads per block, looks every cube corner up through the hash table (8
// chain walks per cube) and takes one global atomic per triangle. Here a
// 256-thread CTA stages the block plus its +x/+y/+z halo (9x9x9 voxels, 7
// neighbour lookups) in shared memory, counts triangles from the packed
// table, reserves the CTA's output range with one atomic and emits with one
// thread per triangle.
#include "vmap_launch.h"
#include "mc_table.inc"

namespace vmapb {

__device__ const unsigned long long kMcTri[256] = VMAP_MC_TRI_PACKED_INIT;

// interpolateLinear: |v| < 1e-6 (a double literal) is |v| <= 1e-6f for floats
__device__ __forceinline__ float mc_interp(float v1, float v2)
{
    if (fabsf(v1) <= 1e-6f) return 0.f;
    if (fabsf(v2) <= 1e-6f) return 1.f;
    if (fabsf(__fsub_rn(v1, v2)) <= 1e-6f) return 0.f;
    return __fdiv_rn(__fsub_rn(0.f, v1), __fsub_rn(v2, v1));
}

// make_vertex (marching_cubes.cu:145-204): edge e of the cube at integer
// voxel coordinates (bx, by, bz); corner sdf s[0..7] in the reference order.
__device__ __forceinline__ float3 edge_vertex(int e, const float* s, float bx, float by, float bz)
{
    switch (e) {
    case 0: { const float t = mc_interp(s[0], s[1]); return make_float3(__fadd_rn(bx, t), by, bz); }
    case 1: { const float t = mc_interp(s[1], s[2]); return make_float3(__fadd_rn(bx, 1.f), __fadd_rn(by, t), bz); }
    case 2: { const float t = mc_interp(s[2], s[3]); return make_float3(__fadd_rn(bx, __fsub_rn(1.f, t)), __fadd_rn(by, 1.f), bz); }
    case 3: { const float t = mc_interp(s[3], s[0]); return make_float3(bx, __fadd_rn(by, __fsub_rn(1.f, t)), bz); }
    case 4: { const float t = mc_interp(s[4], s[5]); return make_float3(__fadd_rn(bx, t), by, __fadd_rn(bz, 1.f)); }
    case 5: { const float t = mc_interp(s[5], s[6]); return make_float3(__fadd_rn(bx, 1.f), __fadd_rn(by, t), __fadd_rn(bz, 1.f)); }
    case 6: { const float t = mc_interp(s[6], s[7]); return make_float3(__fadd_rn(bx, __fsub_rn(1.f, t)), __fadd_rn(by, 1.f), __fadd_rn(bz, 1.f)); }
    case 7: { const float t = mc_interp(s[7], s[4]); return make_float3(bx, __fadd_rn(by, __fsub_rn(1.f, t)), __fadd_rn(bz, 1.f)); }
    case 8: { const float t = mc_interp(s[0], s[4]); return make_float3(bx, by, __fadd_rn(bz, t)); }
    case 9: { const float t = mc_interp(s[1], s[5]); return make_float3(__fadd_rn(bx, 1.f), by, __fadd_rn(bz, t)); }
    case 10: { const float t = mc_interp(s[2], s[6]); return make_float3(__fadd_rn(bx, 1.f), __fadd_rn(by, 1.f), __fadd_rn(bz, t)); }
    default: { const float t = mc_interp(s[3], s[7]); return make_float3(bx, __fadd_rn(by, 1.f), __fadd_rn(bz, t)); }
    }
}

constexpr int kHalo = 9;  // 8 voxels + 1 halo layer per axis

template <int FMT>
__global__ void __launch_bounds__(256) mesh_kernel(DevMap m, float* verts, float* norms, unsigned maxTris)
{
    __shared__ unsigned long long s_tab[256];
    __shared__ float s_sdf[kHalo * kHalo * kHalo];
    __shared__ unsigned char s_ok[kHalo * kHalo * kHalo];
    __shared__ int s_nb[8];
    __shared__ unsigned s_wsum[8];
    __shared__ unsigned s_base, s_total;
    __shared__ unsigned short s_start[512];  // first triangle of each cube rank within the block
    __shared__ unsigned char s_ci[512];      // case index of each cube rank
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    s_tab[tid] = kMcTri[tid];
    const int n = allocated_blocks(m);
    for (int blk = blockIdx.x; blk < n; blk += gridDim.x) {
        __syncthreads();
        const int3 bp = unpack_key(m.blockKeys[blk]);
        if (tid < 8)
            s_nb[tid] = tid == 0 ? blk : hash_find(m, bp.x + (tid & 1), bp.y + ((tid >> 1) & 1), bp.z + ((tid >> 2) & 1));
        __syncthreads();
        for (int e = tid; e < kHalo * kHalo * kHalo; e += 256) {
            const int lx = e % kHalo, ly = (e / kHalo) % kHalo, lz = e / (kHalo * kHalo);
            const int slot = s_nb[(lx >> 3) | ((ly >> 3) << 1) | ((lz >> 3) << 2)];
            float v = 1.f;
            unsigned char ok = 0;
            if (slot >= 0) {
                const int li = ((lz & 7) << 6) | ((ly & 7) << 3) | (lx & 7);
                const typename Fmt<FMT>::Word w = Layout<FMT>::words(m, slot)[li];
                if (Fmt<FMT>::observed(w)) {
                    ok = 1;
                    v = Fmt<FMT>::tsdf(w);
                }
            }
            s_sdf[e] = v;
            s_ok[e] = ok;
        }
        __syncthreads();
        // two cubes per thread; cube c -> local (c & 7, (c >> 3) & 7, c >> 6)
        int ci[2];
        unsigned cnt = 0;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int c = tid + 256 * j;
            const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
            const int e0 = (z * kHalo + y) * kHalo + x;
            // reference corner order (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1)
            const int off[8] = {0, 1, kHalo + 1, kHalo, 81, 82, 81 + kHalo + 1, 81 + kHalo};
            int idx = 0;
            bool ok = true;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                ok &= s_ok[e0 + off[k]] != 0;
                if (s_sdf[e0 + off[k]] < 0.f) idx |= 1 << k;
            }
            ci[j] = ok ? idx : 0;
            cnt += (unsigned)(s_tab[ci[j]] >> 60);
        }
        // CTA exclusive scan of the per-thread triangle counts
        unsigned incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) s_wsum[wid] = incl;
        __syncthreads();
        if (tid == 0) {
            unsigned run = 0;
            for (int w = 0; w < 8; ++w) {
                const unsigned t = s_wsum[w];
                s_wsum[w] = run;
                run += t;
            }
            s_base = run ? atomicAdd(m.ctr + C_TRI, run) : 0u;
            s_total = run;
        }
        __syncthreads();
        if (verts == nullptr) continue;
        // emission: triangles, not cubes, are spread over the threads, so every
        // lane writes (a cube-per-thread loop leaves most lanes idle: few cubes
        // of a block cross the surface). Cube rank r = 2 * tid + j keeps the
        // scan's order; s_start[r] is its first triangle within the block.
        {
            const unsigned first = s_wsum[wid] + incl - cnt;
            const unsigned n0 = (unsigned)(s_tab[ci[0]] >> 60);
            s_start[2 * tid] = (unsigned short)first;
            s_start[2 * tid + 1] = (unsigned short)(first + n0);
            s_ci[2 * tid] = (unsigned char)ci[0];
            s_ci[2 * tid + 1] = (unsigned char)ci[1];
        }
        __syncthreads();
        const unsigned total = s_total;
        for (unsigned q = tid; q < total; q += 256) {
            const unsigned t = s_base + q;
            if (t >= maxTris) break;
            // the last cube rank whose start is <= q (zero-triangle cubes share
            // their successor's start and precede it)
            int lo = 0, hi = 511;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_start[mid] <= q) lo = mid;
                else hi = mid - 1;
            }
            const int r = lo, k = (int)(q - s_start[r]);
            const int c = (r >> 1) + 256 * (r & 1);
            const unsigned long long code = s_tab[s_ci[r]];
            const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
            const int e0 = (z * kHalo + y) * kHalo + x;
            const float s[8] = {s_sdf[e0], s_sdf[e0 + 1], s_sdf[e0 + kHalo + 1], s_sdf[e0 + kHalo],
                                s_sdf[e0 + 81], s_sdf[e0 + 82], s_sdf[e0 + 81 + kHalo + 1], s_sdf[e0 + 81 + kHalo]};
            const float fbx = __int2float_rn(bp.x * 8 + x), fby = __int2float_rn(bp.y * 8 + y),
                        fbz = __int2float_rn(bp.z * 8 + z);
            const int ea = (int)((code >> (12 * k)) & 15), eb = (int)((code >> (12 * k + 4)) & 15),
                      ec = (int)((code >> (12 * k + 8)) & 15);
            // reversed winding: tri[2] = v[a], tri[1] = v[b], tri[0] = v[c], all * voxel size
            const float3 va = edge_vertex(ea, s, fbx, fby, fbz), vb = edge_vertex(eb, s, fbx, fby, fbz),
                         vc = edge_vertex(ec, s, fbx, fby, fbz);
            const float3 t2 = make_float3(__fmul_rn(va.x, m.vs), __fmul_rn(va.y, m.vs), __fmul_rn(va.z, m.vs));
            const float3 t1 = make_float3(__fmul_rn(vb.x, m.vs), __fmul_rn(vb.y, m.vs), __fmul_rn(vb.z, m.vs));
            const float3 t0 = make_float3(__fmul_rn(vc.x, m.vs), __fmul_rn(vc.y, m.vs), __fmul_rn(vc.z, m.vs));
            const float3 nrm = normalized(cross3(make_float3(__fsub_rn(t1.x, t0.x), __fsub_rn(t1.y, t0.y), __fsub_rn(t1.z, t0.z)),
                                                 make_float3(__fsub_rn(t2.x, t0.x), __fsub_rn(t2.y, t0.y), __fsub_rn(t2.z, t0.z))));
            float* vo = verts + 9 * (size_t)t;
            vo[0] = t0.x; vo[1] = t0.y; vo[2] = t0.z;
            vo[3] = t1.x; vo[4] = t1.y; vo[5] = t1.z;
            vo[6] = t2.x; vo[7] = t2.y; vo[8] = t2.z;
            if (norms) {
                float* no = norms + 9 * (size_t)t;
#pragma unroll
                for (int w = 0; w < 3; ++w) {
                    no[3 * w] = nrm.x;
                    no[3 * w + 1] = nrm.y;
                    no[3 * w + 2] = nrm.z;
                }
            }
        }
    }
}

// A pass without an output buffer only counts: it flags nothing.
__global__ void mesh_finish_kernel(DevMap m, unsigned maxTris, unsigned* ntrisOut, bool emitting)
{
    const unsigned n = m.ctr[C_TRI];
    if (emitting && n > maxTris) atomicOr(m.ctr + C_ERR, VMAP_FLAG_BUFFER_FULL);
    if (ntrisOut) *ntrisOut = n;
}

// compute_surface_point_kernel (marching_cubes.cu:314-328): (a + b + c) / 3
__global__ void surface_points_kernel(const float* v, unsigned n, float* pts)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        pts[3 * (size_t)t + i] =
            __fdiv_rn(__fadd_rn(__fadd_rn(v[9 * (size_t)t + i], v[9 * (size_t)t + 3 + i]), v[9 * (size_t)t + 6 + i]), 3.f);
}

// Dense export of blocks [first, first + count) in pool order.
template <int FMT, bool COLOR>
__global__ void export_kernel(DevMap m, int first, int count, int* coords, float* tsdf, float* weight, uint8_t* rgb)
{
    typedef Layout<FMT> L;
    for (int b = blockIdx.x; b < count; b += gridDim.x) {
        const int slot = first + b;
        if (threadIdx.x == 0) {
            const int3 p = unpack_key(m.blockKeys[slot]);
            coords[3 * b] = p.x;
            coords[3 * b + 1] = p.y;
            coords[3 * b + 2] = p.z;
        }
        for (int i = threadIdx.x; i < kBlockVoxels; i += blockDim.x) {
            const size_t o = (size_t)b * kBlockVoxels + i;
            const typename Fmt<FMT>::Word w = L::words(m, slot)[i];
            tsdf[o] = Fmt<FMT>::tsdf(w);
            weight[o] = Fmt<FMT>::weight(w);
            if constexpr (COLOR) {
                if (rgb) {
                    const unsigned char* c = m.pool + (size_t)slot * m.blockBytes + L::kRgbOff;
                    rgb[3 * o] = c[i];
                    rgb[3 * o + 1] = c[kBlockVoxels + i];
                    rgb[3 * o + 2] = c[2 * kBlockVoxels + i];
                }
            }
        }
    }
}

cudaError_t launch_mesh(const DevMap& m, int fmt, float* verts, float* norms, unsigned maxTris, unsigned* ntrisOut,
                        const Launcher& l, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(m.ctr + C_TRI, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    const int grid = stage_grid(l, l.mesh);
    switch (fmt) {
    case VMAP_VOXEL_REF: mesh_kernel<VMAP_VOXEL_REF><<<grid, 256, 0, s>>>(m, verts, norms, maxTris); break;
    case VMAP_VOXEL_F32: mesh_kernel<VMAP_VOXEL_F32><<<grid, 256, 0, s>>>(m, verts, norms, maxTris); break;
    case VMAP_VOXEL_F16: mesh_kernel<VMAP_VOXEL_F16><<<grid, 256, 0, s>>>(m, verts, norms, maxTris); break;
    case VMAP_VOXEL_I16: mesh_kernel<VMAP_VOXEL_I16><<<grid, 256, 0, s>>>(m, verts, norms, maxTris); break;
    default: return cudaErrorInvalidValue;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    mesh_finish_kernel<<<1, 1, 0, s>>>(m, maxTris, ntrisOut, verts != nullptr);
    return cudaGetLastError();
}

cudaError_t launch_surface_points(const float* verts, unsigned n, float* pts, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    surface_points_kernel<<<(n + 255) / 256, 256, 0, s>>>(verts, n, pts);
    return cudaGetLastError();
}

template <int FMT>
static void export_dispatch(const DevMap& m, bool color, int first, int count, int* coords, float* tsdf,
                            float* weight, uint8_t* rgb, cudaStream_t s)
{
    const int grid = count < 4096 ? count : 4096;
    if (color) export_kernel<FMT, true><<<grid, 256, 0, s>>>(m, first, count, coords, tsdf, weight, rgb);
    else export_kernel<FMT, false><<<grid, 256, 0, s>>>(m, first, count, coords, tsdf, weight, rgb);
}

cudaError_t launch_export(const DevMap& m, int fmt, bool color, int first, int count, int* coords, float* tsdf,
                          float* weight, uint8_t* rgb, cudaStream_t s)
{
    if (count <= 0) return cudaSuccess;
    switch (fmt) {
    case VMAP_VOXEL_REF: export_dispatch<VMAP_VOXEL_REF>(m, color, first, count, coords, tsdf, weight, rgb, s); break;
    case VMAP_VOXEL_F32: export_dispatch<VMAP_VOXEL_F32>(m, color, first, count, coords, tsdf, weight, rgb, s); break;
    case VMAP_VOXEL_F16: export_dispatch<VMAP_VOXEL_F16>(m, color, first, count, coords, tsdf, weight, rgb, s); break;
    case VMAP_VOXEL_I16: export_dispatch<VMAP_VOXEL_I16>(m, color, first, count, coords, tsdf, weight, rgb, s); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace vmapb
