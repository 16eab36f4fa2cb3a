// C ABI of libvmap_b200 (include/vmap_c.h): map lifetime, argument checking,
// pose handling (FP64 on the host) and kernel sequencing. No call here
// synchronises the device except the documented synchronous entry points.
//
// Reference: src/vmapping.cpp (VoxelizationImpl :10-148), src/map_struct.cu
// (create / reset / release :29-79).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "vmap_launch.h"

using namespace vmapb;

struct vmap_map {
    vmap_config cfg;
    DevMap dm;
    Launcher launcher;
    int device;
    bool external;            // device buffers live in caller memory (vmap_create_in)
    size_t poolBytes;
    size_t deviceBytes;
    unsigned* hCtr;           // pinned readback of the counters
    unsigned long long* zmin; // z-range tiles (epoch-tagged)
    unsigned long long* zmax;
    unsigned epoch;           // render epoch of the tiles
    int tilesX, tilesY;
    void* dDepth;             // staging for host-buffer calls
    uint8_t* dRgb;
    float4* dVmap;
    float4* dNmap;
    float* dVerts;            // mesh buffers of vmap_polygonize_host
    float* dNorms;
    float* hVerts;
    float* hNorms;
    unsigned meshCap;
    unsigned* dNtri;
    // pipelined host frames (vmap_frame_host_async): two staging sets, a copy
    // stream each way, events ordering copies and kernels per set
    struct HostPipe {
        bool ready;
        unsigned next;
        cudaStream_t h2d, d2h;
        void* depth[2];
        uint8_t* rgb[2];
        float4* vmap[2];
        float4* nmap[2];
        cudaEvent_t inReady[2], inFree[2], outReady[2], outFree[2];
    } pipe;
    // stage timing: event pairs on the caller's stream
    unsigned tCap, tUsed;
    cudaEvent_t* tEv;
    int* tStage;
};

namespace {

thread_local std::string g_last_error;

vmap_status cuda_fail(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? VMAP_ERR_OUT_OF_MEMORY : VMAP_ERR_CUDA;
}

#define VMAP_CK(expr)                                          \
    do {                                                       \
        cudaError_t e_ = (expr);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr);    \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

void to_xf(const double p[16], Xf& t)
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) t.m[r][c] = (float)p[4 * r + c];
}

bool pose_ok(const double p[16])
{
    if (!p) return false;
    for (int i = 0; i < 12; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

}  // namespace

namespace vmapb {
// The per-step view of a map: storage, camera, pose (FP64 inverse rounded to
// FP32), no frame inputs and no render outputs yet.
void make_view(const vmap_map* m, const double pose[16], MapView& v)
{
    std::memset(&v, 0, sizeof(v));
    v.m = m->dm;
    v.cam.W = m->cfg.width;
    v.cam.H = m->cfg.height;
    v.cam.fx = m->cfg.fx;
    v.cam.fy = m->cfg.fy;
    v.cam.cx = m->cfg.cx;
    v.cam.cy = m->cfg.cy;
    v.cam.ifx = (float)(1.0 / (double)m->cfg.fx);
    v.cam.ify = (float)(1.0 / (double)m->cfg.fy);
    v.in.active = 1;
    v.in.dscale = 1.f;
    if (pose) {
        double inv[16];
        vmap_pose_inverse(pose, inv);
        to_xf(pose, v.T);
        to_xf(inv, v.Ti);
    }
    v.out.tilesX = m->tilesX;
    v.out.tilesY = m->tilesY;
    v.out.zmin = m->zmin;
    v.out.zmax = m->zmax;
    v.out.vsinv = (float)(1.0 / (double)m->cfg.voxel_size);
    v.out.rts = m->cfg.truncation / m->cfg.voxel_size;
    v.out.mode = m->cfg.raycast_mode;
}

// Next render epoch of a map's z-range tiles; on wrap-around the tiles are
// re-initialised (all-ones near, zero far) so no stale tag can match.
cudaError_t next_epoch(vmap_map* m, cudaStream_t s, unsigned* epoch)
{
    if (m->epoch >= 0xFFFFFFFEu) {
        const size_t nt = (size_t)m->tilesX * m->tilesY * sizeof(unsigned long long);
        cudaError_t e = cudaMemsetAsync(m->zmin, 0xff, nt, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(m->zmax, 0, nt, s);
        if (e != cudaSuccess) return e;
        m->epoch = 0;
    }
    *epoch = ++m->epoch;
    return cudaSuccess;
}
}  // namespace vmapb

namespace {

template <typename T>
cudaError_t dalloc(vmap_map* m, T** p, size_t bytes)
{
    cudaError_t e = cudaMalloc((void**)p, bytes ? bytes : 16);
    if (e == cudaSuccess) m->deviceBytes += bytes;
    return e;
}

// Staging buffers of the host-buffer calls, allocated on the first such call
// (maps driven only through device pointers never hold them).
cudaError_t ensure_staging(vmap_map* m)
{
    if (m->dDepth) return cudaSuccess;
    const size_t npix = (size_t)m->cfg.width * m->cfg.height, before = m->deviceBytes;
    cudaError_t e = dalloc(m, &m->dDepth, npix * sizeof(float));
    if (e == cudaSuccess) e = dalloc(m, &m->dRgb, npix * 3);
    if (e == cudaSuccess) e = dalloc(m, &m->dVmap, npix * sizeof(float4));
    if (e == cudaSuccess) e = dalloc(m, &m->dNmap, npix * sizeof(float4));
    if (e != cudaSuccess) {
        for (void* p : {m->dDepth, (void*)m->dRgb, (void*)m->dVmap, (void*)m->dNmap}) cudaFree(p);
        m->deviceBytes = before;
        m->dDepth = nullptr;
        m->dRgb = nullptr;
        m->dVmap = m->dNmap = nullptr;
    }
    return e;
}

void timing_free(vmap_map* m)
{
    for (unsigned i = 0; i < 2 * m->tCap; ++i) cudaEventDestroy(m->tEv[i]);
    delete[] m->tEv;
    delete[] m->tStage;
    m->tEv = nullptr;
    m->tStage = nullptr;
    m->tCap = m->tUsed = 0;
}

// Runs one kernel launcher, bracketed by timing events when timing is on.
template <typename F>
cudaError_t staged(vmap_map* m, int stage, cudaStream_t s, F&& launch)
{
    const bool rec = m->tUsed < m->tCap;
    if (rec) cudaEventRecord(m->tEv[2 * m->tUsed], s);
    cudaError_t e = launch();
    if (rec && e == cudaSuccess) {
        cudaEventRecord(m->tEv[2 * m->tUsed + 1], s);
        m->tStage[m->tUsed++] = stage;
    }
    return e;
}

void pipe_free(vmap_map* m)
{
    vmap_map::HostPipe& p = m->pipe;
    if (p.h2d) cudaStreamSynchronize(p.h2d);
    if (p.d2h) cudaStreamSynchronize(p.d2h);
    for (int b = 0; b < 2; ++b) {
        cudaFree(p.depth[b]);
        cudaFree(p.rgb[b]);
        cudaFree(p.vmap[b]);
        cudaFree(p.nmap[b]);
        for (cudaEvent_t e : {p.inReady[b], p.inFree[b], p.outReady[b], p.outFree[b]})
            if (e) cudaEventDestroy(e);
    }
    if (p.h2d) cudaStreamDestroy(p.h2d);
    if (p.d2h) cudaStreamDestroy(p.d2h);
    std::memset(&p, 0, sizeof(p));
}

void free_all(vmap_map* m)
{
    timing_free(m);
    pipe_free(m);
    if (!m->external) {  // buffers carved from caller memory stay with the caller
        cudaFree(m->dm.slots);
        cudaFree(m->dm.blockKeys);
        cudaFree(m->dm.pool);
        cudaFree(m->dm.ctr);
        cudaFree(m->dm.visList);
        cudaFree(m->zmin);
        cudaFree(m->zmax);
        cudaFree(m->dNtri);
        cudaFree(m->dm.nbr);
    }
    cudaFree(m->dDepth);
    cudaFree(m->dRgb);
    cudaFree(m->dVmap);
    cudaFree(m->dNmap);
    cudaFree(m->dVerts);
    cudaFree(m->dNorms);
    if (m->hCtr) cudaFreeHost(m->hCtr);
    if (m->hVerts) cudaFreeHost(m->hVerts);
    if (m->hNorms) cudaFreeHost(m->hNorms);
}

}  // namespace

extern "C" {

int vmap_abi_version(void) { return VMAP_ABI_VERSION; }

const char* vmap_last_error(void) { return g_last_error.c_str(); }

const char* vmap_status_string(vmap_status s)
{
    switch (s) {
    case VMAP_OK: return "ok";
    case VMAP_ERR_INVALID_ARG: return "invalid argument";
    case VMAP_ERR_CUDA: return "CUDA error";
    case VMAP_ERR_OUT_OF_MEMORY: return "out of memory";
    case VMAP_ERR_POOL_FULL: return "voxel-block pool full";
    case VMAP_ERR_HASH_FULL: return "hash table full";
    case VMAP_ERR_RANGE: return "block coordinate out of range";
    case VMAP_ERR_BUFFER_FULL: return "mesh buffer full";
    case VMAP_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    }
    return "unknown status";
}

// hash (map_struct.h:104-109), host copy for tests
int vmap_block_hash(int x, int y, int z, int nb)
{
    int r = (int)(((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^ ((unsigned)z * 83492791u));
    r %= nb;
    return r < 0 ? r + nb : r;
}

}  // extern "C"

namespace {
__global__ void block_hash_kernel(const int* xyz, unsigned n, int nb, unsigned long long magic, int* out)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = ref_hash_fast(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], nb, magic);
}
}  // namespace

extern "C" {

vmap_status vmap_block_hash_device(const int32_t* xyz_dev, uint32_t n, int n_buckets, int32_t* out_dev, void* stream)
{
    if ((!xyz_dev || !out_dev) && n) return VMAP_ERR_INVALID_ARG;
    if (n_buckets < 1) return VMAP_ERR_INVALID_ARG;
    if (n == 0) return VMAP_OK;
    block_hash_kernel<<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(xyz_dev, n, n_buckets,
                                                                      bucket_magic((unsigned)n_buckets), out_dev);
    VMAP_CK(cudaGetLastError());
    return VMAP_OK;
}

// Affine inverse of a row-major camera-to-world pose in double:
// inv(A) = adj(A) / det(A), t' = -inv(A) t (the reference inverts the 4x4 in
// float with Eigen, depth_fusion.cu:251, ray_tracing.cu:414).
void vmap_pose_inverse(const double p[16], double o[16])
{
    const double a = p[0], b = p[1], c = p[2], d = p[4], e = p[5], f = p[6], g = p[8], h = p[9], i = p[10];
    const double A = e * i - f * h, B = f * g - d * i, C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double r = 1.0 / det;
    o[0] = A * r;
    o[1] = (c * h - b * i) * r;
    o[2] = (b * f - c * e) * r;
    o[4] = B * r;
    o[5] = (a * i - c * g) * r;
    o[6] = (c * d - a * f) * r;
    o[8] = C * r;
    o[9] = (b * g - a * h) * r;
    o[10] = (a * e - b * d) * r;
    for (int k = 0; k < 3; ++k) o[4 * k + 3] = -(o[4 * k] * p[3] + o[4 * k + 1] * p[7] + o[4 * k + 2] * p[11]);
    o[12] = o[13] = o[14] = 0.0;
    o[15] = 1.0;
}

size_t vmap_block_bytes(int fmt, int color)
{
    switch (fmt) {
    case VMAP_VOXEL_REF: return Layout<VMAP_VOXEL_REF>::bytes(color != 0);
    case VMAP_VOXEL_F32: return Layout<VMAP_VOXEL_F32>::bytes(color != 0);
    case VMAP_VOXEL_F16: return Layout<VMAP_VOXEL_F16>::bytes(color != 0);
    case VMAP_VOXEL_I16: return Layout<VMAP_VOXEL_I16>::bytes(color != 0);
    }
    return 0;
}

}  // extern "C"

namespace {

// Validates a configuration and fills in its defaults (vmapping.cpp:57-75).
vmap_status resolve_config(const vmap_config* cfg_in, vmap_config& cfg)
{
    if (!cfg_in) return VMAP_ERR_INVALID_ARG;
    cfg = *cfg_in;
    if (cfg.width <= 0 || cfg.height <= 0 || !(cfg.fx > 0) || !(cfg.fy > 0) || !std::isfinite(cfg.cx) ||
        !std::isfinite(cfg.cy) || cfg.num_blocks <= 0 || !(cfg.voxel_size > 0) || cfg.num_entries < 0 ||
        cfg.num_buckets < 0 || cfg.truncation < 0 || cfg.max_weight < 0 || cfg.raycast_mode < 0 ||
        cfg.raycast_mode > 1)
        return VMAP_ERR_INVALID_ARG;
    if (vmap_block_bytes(cfg.voxel_format, cfg.with_color) == 0) return VMAP_ERR_INVALID_ARG;
    if (cfg.num_buckets == 0) cfg.num_buckets = (int)(cfg.num_blocks * 0.9);  // vmapping.cpp:59
    if (cfg.num_buckets < 1) cfg.num_buckets = 1;
    if ((long long)cfg.num_buckets * kSlots < (long long)cfg.num_entries)
        cfg.num_buckets = (int)(((long long)cfg.num_entries + kSlots - 1) / kSlots);
    if (cfg.truncation == 0) cfg.truncation = cfg.voxel_size * 4;  // vmapping.cpp:59
    // voxel size >= 0.1 mm keeps ray distances (in voxels, up to 5 m) below 2^24 so
    // unit steps always advance a float; truncation <= 1024 voxels bounds the
    // samples per depth pixel
    if (cfg.voxel_size < 1e-4f || cfg.truncation > 1024.f * cfg.voxel_size) return VMAP_ERR_INVALID_ARG;
    if (cfg.max_weight == 0) cfg.max_weight = 255;                 // depth_fusion.cu:193
    if (cfg.voxel_format == VMAP_VOXEL_REF && cfg.max_weight > 255) return VMAP_ERR_INVALID_ARG;
    if (cfg.max_weight > 65535) return VMAP_ERR_INVALID_ARG;
    return VMAP_OK;
}

// Device buffers of a map, in order, each starting on a 256-byte boundary:
// hash slots, block keys, voxel pool, counters, visible list, z-range tiles
// (min, max), triangle count.
struct MapLayout {
    enum { SLOTS, KEYS, POOL, CTR, VIS, ZMIN, ZMAX, NTRI, NBR, N };
    size_t off[N + 1];
};

MapLayout map_layout(const vmap_config& cfg)
{
    const size_t nslots = (size_t)cfg.num_buckets * kSlots, cap = (size_t)cfg.num_blocks;
    const size_t ntiles = (size_t)((cfg.width + kZTile - 1) / kZTile) * ((cfg.height + kZTile - 1) / kZTile);
    const size_t sz[MapLayout::N] = {nslots * sizeof(ulonglong2), cap * sizeof(unsigned long long),
                                     cap * vmap_block_bytes(cfg.voxel_format, cfg.with_color),
                                     C_COUNT * sizeof(unsigned), cap * sizeof(int),
                                     ntiles * sizeof(unsigned long long), ntiles * sizeof(unsigned long long),
                                     sizeof(unsigned), cap * 7 * sizeof(int)};
    MapLayout l;
    l.off[0] = 0;
    for (int i = 0; i < MapLayout::N; ++i) l.off[i + 1] = (l.off[i] + sz[i] + 255) / 256 * 256;
    return l;
}

// Builds a map for a resolved configuration. With `base` non-NULL its device
// buffers are carved from the caller's memory (MapLayout) and the reset runs
// asynchronously on `stream`; otherwise they are cudaMalloc'ed and the reset
// is synchronous.
vmap_status build_map(const vmap_config& cfg, unsigned char* base, cudaStream_t stream, vmap_map** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (cuda_fail(e, "cudaGetDevice"), VMAP_ERR_NO_DEVICE);
    int major = 0, sms = 0;
    if ((e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    if (major != 10) {
        g_last_error = "libvmap_b200 is built for sm_100a; device is sm_" + std::to_string(major * 10);
        return VMAP_ERR_NO_DEVICE;
    }
    vmap_map* m = new (std::nothrow) vmap_map();
    if (!m) return VMAP_ERR_OUT_OF_MEMORY;
    std::memset(m, 0, sizeof(*m));
    m->cfg = cfg;
    m->device = dev;
    m->external = base != nullptr;
    m->launcher = Launcher();  // the memset above cleared the default grid shapes
    m->launcher.numSMs = sms;
    m->tilesX = (cfg.width + kZTile - 1) / kZTile;
    m->tilesY = (cfg.height + kZTile - 1) / kZTile;
    const size_t blockBytes = vmap_block_bytes(cfg.voxel_format, cfg.with_color);
    m->poolBytes = (size_t)cfg.num_blocks * blockBytes;
    const MapLayout l = map_layout(cfg);
    void** ptrs[MapLayout::N] = {(void**)&m->dm.slots, (void**)&m->dm.blockKeys, (void**)&m->dm.pool,
                                 (void**)&m->dm.ctr, (void**)&m->dm.visList, (void**)&m->zmin, (void**)&m->zmax,
                                 (void**)&m->dNtri, (void**)&m->dm.nbr};
    for (int i = 0; i < MapLayout::N; ++i) {
        const size_t bytes = l.off[i + 1] - l.off[i];
        if (base) {
            *ptrs[i] = base + l.off[i];
            m->deviceBytes += bytes;
        } else if ((e = dalloc(m, (unsigned char**)ptrs[i], bytes)) != cudaSuccess) {
            vmap_status st = cuda_fail(e, "cudaMalloc");
            free_all(m);
            delete m;
            return st;
        }
    }
    if ((e = cudaHostAlloc((void**)&m->hCtr, C_COUNT * sizeof(unsigned), cudaHostAllocDefault)) != cudaSuccess) {
        vmap_status st = cuda_fail(e, "cudaHostAlloc");
        free_all(m);
        delete m;
        return st;
    }
    m->dm.nBucket = cfg.num_buckets;
    m->dm.bucketMagic = bucket_magic((unsigned)cfg.num_buckets);
    m->dm.capacity = cfg.num_blocks;
    m->dm.blockBytes = (int)blockBytes;
    m->dm.vs = cfg.voxel_size;
    m->dm.mu = cfg.truncation;
    m->dm.wmax = (float)cfg.max_weight;
    m->epoch = 0xFFFFFFFEu;  // the first render re-initialises the tiles
    vmap_status st = vmap_reset(m, stream);
    if (st == VMAP_OK && !base && (e = cudaStreamSynchronize(stream)) != cudaSuccess) st = cuda_fail(e, "create sync");
    if (st != VMAP_OK) {
        free_all(m);
        delete m;
        return st;
    }
    *out = m;
    return VMAP_OK;
}

}  // namespace

extern "C" {

vmap_status vmap_create(const vmap_config* cfg_in, vmap_map** out)
{
    if (!cfg_in || !out) return VMAP_ERR_INVALID_ARG;
    *out = nullptr;
    vmap_config cfg;
    vmap_status st = resolve_config(cfg_in, cfg);
    if (st != VMAP_OK) return st;
    return build_map(cfg, nullptr, nullptr, out);
}

vmap_status vmap_required_bytes(const vmap_config* cfg_in, uint64_t* bytes)
{
    if (!cfg_in || !bytes) return VMAP_ERR_INVALID_ARG;
    vmap_config cfg;
    vmap_status st = resolve_config(cfg_in, cfg);
    if (st != VMAP_OK) return st;
    *bytes = map_layout(cfg).off[MapLayout::N];
    return VMAP_OK;
}

vmap_status vmap_create_in(const vmap_config* cfg_in, void* device_mem, uint64_t bytes, void* stream,
                           vmap_map** out)
{
    if (!cfg_in || !out || !device_mem || ((uintptr_t)device_mem & 255)) return VMAP_ERR_INVALID_ARG;
    *out = nullptr;
    vmap_config cfg;
    vmap_status st = resolve_config(cfg_in, cfg);
    if (st != VMAP_OK) return st;
    if (bytes < map_layout(cfg).off[MapLayout::N]) {
        g_last_error = "vmap_create_in: " + std::to_string(bytes) + " bytes given, " +
                       std::to_string(map_layout(cfg).off[MapLayout::N]) + " needed";
        return VMAP_ERR_INVALID_ARG;
    }
    return build_map(cfg, static_cast<unsigned char*>(device_mem), as_stream(stream), out);
}

vmap_status vmap_destroy(vmap_map* m)
{
    if (!m) return VMAP_ERR_INVALID_ARG;
    if (!m->external) cudaDeviceSynchronize();
    free_all(m);
    delete m;
    return VMAP_OK;
}

vmap_status vmap_get_launch_config(const vmap_map* m, vmap_launch_config* out)
{
    if (!m || !out) return VMAP_ERR_INVALID_ARG;
    launch_config_from(m->launcher, out);
    return VMAP_OK;
}

vmap_status vmap_set_launch_config(vmap_map* m, const vmap_launch_config* cfg)
{
    if (!m || !cfg || !launch_config_ok(cfg)) return VMAP_ERR_INVALID_ARG;
    launch_config_to(cfg, m->launcher);
    return VMAP_OK;
}

vmap_status vmap_get_config(const vmap_map* m, vmap_config* out)
{
    if (!m || !out) return VMAP_ERR_INVALID_ARG;
    *out = m->cfg;
    return VMAP_OK;
}

vmap_status vmap_reset(vmap_map* m, void* stream)
{
    if (!m) return VMAP_ERR_INVALID_ARG;
    VMAP_CK(launch_reset(m->dm, m->poolBytes, m->launcher, as_stream(stream)));
    return VMAP_OK;
}

static vmap_status fuse_impl(vmap_map* m, const void* depth, int dtype, size_t dpitch, float dscale,
                             const uint8_t* rgb, size_t rgbPitch, const double pose[16], cudaStream_t s)
{
    if (!m || !depth || !pose_ok(pose)) return VMAP_ERR_INVALID_ARG;
    if (dtype != VMAP_DEPTH_F32 && dtype != VMAP_DEPTH_U16) return VMAP_ERR_INVALID_ARG;
    const size_t elem = dtype == VMAP_DEPTH_F32 ? 4 : 2;
    if (dpitch == 0) dpitch = elem * m->cfg.width;
    if (dpitch < elem * m->cfg.width || dpitch % elem) return VMAP_ERR_INVALID_ARG;
    if (dtype == VMAP_DEPTH_U16 && !(dscale > 0)) return VMAP_ERR_INVALID_ARG;
    if (rgb) {
        if (!m->cfg.with_color) return VMAP_ERR_INVALID_ARG;
        if (rgbPitch == 0) rgbPitch = 3 * (size_t)m->cfg.width;
        if (rgbPitch < 3 * (size_t)m->cfg.width) return VMAP_ERR_INVALID_ARG;
    }
    OneView ov;
    make_view(m, pose, ov.v);
    ov.v.in.depth = depth;
    ov.v.in.dpitch = dpitch;
    ov.v.in.dtype = dtype;
    ov.v.in.dscale = dscale;
    ov.v.in.rgb = rgb;
    ov.v.in.rgbPitch = rgbPitch;
    ov.queue = m->dm.ctr + C_RAYQ;
    const int tiles = stage_tiles(m->cfg.width, m->cfg.height);
    // alloc_kernel clears the visible counter the visibility kernel fills
    VMAP_CK(staged(m, VMAP_STAGE_ALLOC, s, [&] { return launch_alloc(ov, tiles, m->launcher, s); }));
    VMAP_CK(staged(m, VMAP_STAGE_VISIBILITY, s, [&] { return launch_visibility(ov, m->launcher, s); }));
    VMAP_CK(staged(m, VMAP_STAGE_FUSE, s, [&] { return launch_fuse(ov, m->cfg.voxel_format, m->launcher, s); }));
    return VMAP_OK;
}

vmap_status vmap_fuse_depth(vmap_map* m, const void* depth_dev, int depth_type, size_t depth_pitch,
                            float depth_scale, const double pose[16], void* stream)
{
    return fuse_impl(m, depth_dev, depth_type, depth_pitch, depth_scale, nullptr, 0, pose, as_stream(stream));
}

vmap_status vmap_fuse_depth_rgb(vmap_map* m, const void* depth_dev, int depth_type, size_t depth_pitch,
                                float depth_scale, const uint8_t* rgb_dev, size_t rgb_pitch, const double pose[16],
                                void* stream)
{
    if (!rgb_dev) return VMAP_ERR_INVALID_ARG;
    return fuse_impl(m, depth_dev, depth_type, depth_pitch, depth_scale, rgb_dev, rgb_pitch, pose,
                     as_stream(stream));
}

vmap_status vmap_fuse_host(vmap_map* m, const void* depth_host, int depth_type, float depth_scale,
                           const uint8_t* rgb_host, const double pose[16], void* stream)
{
    if (!m || !depth_host) return VMAP_ERR_INVALID_ARG;
    if (depth_type != VMAP_DEPTH_F32 && depth_type != VMAP_DEPTH_U16) return VMAP_ERR_INVALID_ARG;
    if (rgb_host && !m->cfg.with_color) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    const size_t npix = (size_t)m->cfg.width * m->cfg.height;
    const size_t elem = depth_type == VMAP_DEPTH_F32 ? 4 : 2;
    VMAP_CK(ensure_staging(m));
    VMAP_CK(cudaMemcpyAsync(m->dDepth, depth_host, npix * elem, cudaMemcpyHostToDevice, s));
    if (rgb_host) VMAP_CK(cudaMemcpyAsync(m->dRgb, rgb_host, npix * 3, cudaMemcpyHostToDevice, s));
    return fuse_impl(m, m->dDepth, depth_type, elem * m->cfg.width, depth_scale, rgb_host ? m->dRgb : nullptr,
                     3 * (size_t)m->cfg.width, pose, s);
}

vmap_status vmap_check_visible_blocks(vmap_map* m, const double pose[16], void* stream)
{
    if (!m || !pose_ok(pose)) return VMAP_ERR_INVALID_ARG;
    OneView ov;
    make_view(m, pose, ov.v);
    ov.queue = m->dm.ctr + C_RAYQ;
    cudaStream_t s = as_stream(stream);
    VMAP_CK(cudaMemsetAsync(m->dm.ctr + C_VISIBLE, 0, sizeof(unsigned), s));
    VMAP_CK(staged(m, VMAP_STAGE_VISIBILITY, s, [&] { return launch_visibility(ov, m->launcher, s); }));
    return VMAP_OK;
}

vmap_status vmap_render_scene(vmap_map* m, const double pose[16], float* vmap_dev, size_t vmap_pitch,
                              float* nmap_dev, size_t nmap_pitch, void* stream)
{
    if (!m || !vmap_dev || !pose_ok(pose)) return VMAP_ERR_INVALID_ARG;
    const size_t row = sizeof(float4) * (size_t)m->cfg.width;
    if (vmap_pitch == 0) vmap_pitch = row;
    if (nmap_pitch == 0) nmap_pitch = row;
    if (vmap_pitch < row || vmap_pitch % 16 || (nmap_dev && (nmap_pitch < row || nmap_pitch % 16)) ||
        ((uintptr_t)vmap_dev & 15) || ((uintptr_t)nmap_dev & 15))
        return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    OneView ov;
    make_view(m, pose, ov.v);
    ov.queue = m->dm.ctr + C_RAYQ;
    ov.v.out.vmap = reinterpret_cast<float4*>(vmap_dev);
    ov.v.out.vpitch = vmap_pitch;
    ov.v.out.nmap = reinterpret_cast<float4*>(nmap_dev);
    ov.v.out.npitch = nmap_pitch;
    VMAP_CK(next_epoch(m, s, &ov.v.out.epoch));
    // the z-range kernel also rewinds the raycast work queue, so it runs in
    // both raycast modes (with no work in mode 1)
    VMAP_CK(staged(m, VMAP_STAGE_ZRANGE, s, [&] { return launch_zrange(ov, m->launcher, s); }));
    VMAP_CK(staged(m, VMAP_STAGE_RAYCAST, s, [&] { return launch_raycast(ov, m->cfg.voxel_format, m->launcher, s); }));
    if (nmap_dev)
        VMAP_CK(staged(m, VMAP_STAGE_NORMALS, s, [&] {
            return launch_normals(ov, stage_tiles(m->cfg.width, m->cfg.height), m->launcher, s);
        }));
    return VMAP_OK;
}

vmap_status vmap_render_scene_host(vmap_map* m, const double pose[16], float* vmap_host, float* nmap_host,
                                   void* stream)
{
    if (!m || !vmap_host) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    VMAP_CK(ensure_staging(m));
    vmap_status st = vmap_render_scene(m, pose, (float*)m->dVmap, 0, nmap_host ? (float*)m->dNmap : nullptr, 0, stream);
    if (st != VMAP_OK) return st;
    const size_t bytes = (size_t)m->cfg.width * m->cfg.height * sizeof(float4);
    VMAP_CK(cudaMemcpyAsync(vmap_host, m->dVmap, bytes, cudaMemcpyDeviceToHost, s));
    if (nmap_host) VMAP_CK(cudaMemcpyAsync(nmap_host, m->dNmap, bytes, cudaMemcpyDeviceToHost, s));
    return VMAP_OK;
}

// Buffers, streams and events of the host pipeline, on its first use.
static cudaError_t ensure_pipe(vmap_map* m)
{
    vmap_map::HostPipe& p = m->pipe;
    if (p.ready) return cudaSuccess;
    const size_t npix = (size_t)m->cfg.width * m->cfg.height;
    cudaError_t e = cudaStreamCreateWithFlags(&p.h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p.d2h, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMalloc(&p.depth[b], npix * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc((void**)&p.rgb[b], npix * 3);
        if (e == cudaSuccess) e = cudaMalloc((void**)&p.vmap[b], npix * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc((void**)&p.nmap[b], npix * sizeof(float4));
        for (cudaEvent_t* ev : {&p.inReady[b], &p.inFree[b], &p.outReady[b], &p.outFree[b]})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        pipe_free(m);
        return e;
    }
    m->deviceBytes += 2 * npix * (sizeof(float) + 3 + 2 * sizeof(float4));
    p.ready = true;
    return cudaSuccess;
}

vmap_status vmap_frame_host_async(vmap_map* m, const vmap_host_frame* f, void* stream)
{
    if (!m || !f || !f->depth_host || !pose_ok(f->pose)) return VMAP_ERR_INVALID_ARG;
    if (f->depth_type != VMAP_DEPTH_F32 && f->depth_type != VMAP_DEPTH_U16) return VMAP_ERR_INVALID_ARG;
    if (f->depth_type == VMAP_DEPTH_U16 && !(f->depth_scale > 0)) return VMAP_ERR_INVALID_ARG;
    if ((f->rgb_host && !m->cfg.with_color) || (f->nmap_host && !f->vmap_host)) return VMAP_ERR_INVALID_ARG;
    VMAP_CK(ensure_pipe(m));
    vmap_map::HostPipe& p = m->pipe;
    cudaStream_t s = as_stream(stream);
    const int b = (int)(p.next & 1u);
    const size_t npix = (size_t)m->cfg.width * m->cfg.height;
    const size_t elem = f->depth_type == VMAP_DEPTH_F32 ? 4 : 2;
    // inputs: into staging set b once the fusion two frames back has read it
    VMAP_CK(cudaStreamWaitEvent(p.h2d, p.inFree[b], 0));
    VMAP_CK(cudaMemcpyAsync(p.depth[b], f->depth_host, npix * elem, cudaMemcpyHostToDevice, p.h2d));
    if (f->rgb_host) VMAP_CK(cudaMemcpyAsync(p.rgb[b], f->rgb_host, npix * 3, cudaMemcpyHostToDevice, p.h2d));
    VMAP_CK(cudaEventRecord(p.inReady[b], p.h2d));
    // kernels on the caller's stream
    VMAP_CK(cudaStreamWaitEvent(s, p.inReady[b], 0));
    vmap_status st = fuse_impl(m, p.depth[b], f->depth_type, elem * m->cfg.width, f->depth_scale,
                               f->rgb_host ? p.rgb[b] : nullptr, 3 * (size_t)m->cfg.width, f->pose, s);
    if (st != VMAP_OK) return st;
    VMAP_CK(cudaEventRecord(p.inFree[b], s));
    if (f->vmap_host) {
        // render into output set b once its copy-out two frames back is done
        VMAP_CK(cudaStreamWaitEvent(s, p.outFree[b], 0));
        st = vmap_render_scene(m, f->pose, (float*)p.vmap[b], 0, f->nmap_host ? (float*)p.nmap[b] : nullptr, 0,
                               stream);
        if (st != VMAP_OK) return st;
        VMAP_CK(cudaEventRecord(p.outReady[b], s));
        VMAP_CK(cudaStreamWaitEvent(p.d2h, p.outReady[b], 0));
        VMAP_CK(cudaMemcpyAsync(f->vmap_host, p.vmap[b], npix * sizeof(float4), cudaMemcpyDeviceToHost, p.d2h));
        if (f->nmap_host)
            VMAP_CK(cudaMemcpyAsync(f->nmap_host, p.nmap[b], npix * sizeof(float4), cudaMemcpyDeviceToHost, p.d2h));
        VMAP_CK(cudaEventRecord(p.outFree[b], p.d2h));
    }
    ++p.next;
    return VMAP_OK;
}

vmap_status vmap_host_wait(vmap_map* m, void* stream)
{
    if (!m) return VMAP_ERR_INVALID_ARG;
    if (!m->pipe.ready) return VMAP_OK;
    cudaStream_t s = as_stream(stream);
    for (int b = 0; b < 2; ++b) VMAP_CK(cudaStreamWaitEvent(s, m->pipe.outFree[b], 0));
    return VMAP_OK;
}

vmap_status vmap_compute_normal(const float* vmap_dev, size_t vmap_pitch, float* nmap_dev, size_t nmap_pitch,
                                int width, int height, void* stream)
{
    if (!vmap_dev || !nmap_dev || width <= 0 || height <= 0) return VMAP_ERR_INVALID_ARG;
    const size_t row = sizeof(float4) * (size_t)width;
    if (vmap_pitch == 0) vmap_pitch = row;
    if (nmap_pitch == 0) nmap_pitch = row;
    if (vmap_pitch < row || nmap_pitch < row || vmap_pitch % 16 || nmap_pitch % 16) return VMAP_ERR_INVALID_ARG;
    OneView ov;
    std::memset(&ov, 0, sizeof(ov));
    ov.v.cam.W = width;
    ov.v.cam.H = height;
    ov.v.out.vmap = const_cast<float4*>(reinterpret_cast<const float4*>(vmap_dev));
    ov.v.out.vpitch = vmap_pitch;
    ov.v.out.nmap = reinterpret_cast<float4*>(nmap_dev);
    ov.v.out.npitch = nmap_pitch;
    int dev = 0, sms = 1;
    VMAP_CK(cudaGetDevice(&dev));
    VMAP_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    Launcher l;
    l.numSMs = sms;
    VMAP_CK(launch_normals(ov, stage_tiles(width, height), l, as_stream(stream)));
    return VMAP_OK;
}

vmap_status vmap_render_phong(const float* vmap_dev, size_t vmap_pitch, const float* nmap_dev, size_t nmap_pitch,
                              uint8_t* rgba_dev, size_t rgba_pitch, int width, int height, void* stream)
{
    if (!vmap_dev || !nmap_dev || !rgba_dev || width <= 0 || height <= 0) return VMAP_ERR_INVALID_ARG;
    const size_t row = sizeof(float4) * (size_t)width;
    if (vmap_pitch == 0) vmap_pitch = row;
    if (nmap_pitch == 0) nmap_pitch = row;
    if (rgba_pitch == 0) rgba_pitch = 4 * (size_t)width;
    if (vmap_pitch < row || nmap_pitch < row || rgba_pitch < 4 * (size_t)width || rgba_pitch % 4)
        return VMAP_ERR_INVALID_ARG;
    VMAP_CK(launch_phong(reinterpret_cast<const float4*>(vmap_dev), vmap_pitch,
                         reinterpret_cast<const float4*>(nmap_dev), nmap_pitch, reinterpret_cast<uchar4*>(rgba_dev),
                         rgba_pitch, width, height, as_stream(stream)));
    return VMAP_OK;
}

vmap_status vmap_polygonize(vmap_map* m, float* verts_dev, float* norms_dev, uint32_t max_tris, uint32_t* n_tris_dev,
                            void* stream)
{
    if (!m || (norms_dev && !verts_dev)) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    VMAP_CK(staged(m, VMAP_STAGE_MESH, s, [&] {
        return launch_mesh(m->dm, m->cfg.voxel_format, verts_dev, norms_dev, verts_dev ? max_tris : 0u, n_tris_dev,
                           m->launcher, s);
    }));
    return VMAP_OK;
}

vmap_status vmap_polygonize_host(vmap_map* m, const float** verts, const float** norms, uint32_t* n_tris, void* stream)
{
    if (!m || !verts || !norms || !n_tris) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    unsigned count = 0;
    VMAP_CK(launch_mesh(m->dm, m->cfg.voxel_format, nullptr, nullptr, 0u, m->dNtri, m->launcher, s));
    VMAP_CK(cudaMemcpyAsync(&count, m->dNtri, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    VMAP_CK(cudaStreamSynchronize(s));
    if (count > m->meshCap) {
        cudaFree(m->dVerts);
        cudaFree(m->dNorms);
        if (m->hVerts) cudaFreeHost(m->hVerts);
        if (m->hNorms) cudaFreeHost(m->hNorms);
        m->dVerts = m->dNorms = m->hVerts = m->hNorms = nullptr;
        m->meshCap = 0;
        const unsigned cap = count + count / 8 + 1024;
        const size_t bytes = (size_t)cap * 9 * sizeof(float);
        VMAP_CK(cudaMalloc((void**)&m->dVerts, bytes));
        VMAP_CK(cudaMalloc((void**)&m->dNorms, bytes));
        VMAP_CK(cudaHostAlloc((void**)&m->hVerts, bytes, cudaHostAllocDefault));
        VMAP_CK(cudaHostAlloc((void**)&m->hNorms, bytes, cudaHostAllocDefault));
        m->meshCap = cap;
    }
    if (count > 0) {
        VMAP_CK(launch_mesh(m->dm, m->cfg.voxel_format, m->dVerts, m->dNorms, m->meshCap, m->dNtri, m->launcher, s));
        VMAP_CK(cudaMemcpyAsync(&count, m->dNtri, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        VMAP_CK(cudaStreamSynchronize(s));
        if (count > m->meshCap) count = m->meshCap;
        const size_t bytes = (size_t)count * 9 * sizeof(float);
        VMAP_CK(cudaMemcpyAsync(m->hVerts, m->dVerts, bytes, cudaMemcpyDeviceToHost, s));
        VMAP_CK(cudaMemcpyAsync(m->hNorms, m->dNorms, bytes, cudaMemcpyDeviceToHost, s));
        VMAP_CK(cudaStreamSynchronize(s));
    }
    *verts = m->hVerts;
    *norms = m->hNorms;
    *n_tris = count;
    return VMAP_OK;
}

vmap_status vmap_surface_points(const float* verts_dev, uint32_t n_tris, float* points_dev, void* stream)
{
    if ((!verts_dev || !points_dev) && n_tris) return VMAP_ERR_INVALID_ARG;
    VMAP_CK(launch_surface_points(verts_dev, n_tris, points_dev, as_stream(stream)));
    return VMAP_OK;
}

vmap_status vmap_get_stats(vmap_map* m, void* stream, vmap_stats* out)
{
    if (!m || !out) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    VMAP_CK(cudaMemcpyAsync(m->hCtr, m->dm.ctr, C_COUNT * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    VMAP_CK(cudaStreamSynchronize(s));
    const unsigned alloc = m->hCtr[C_ALLOC];
    out->allocated_blocks = alloc < (unsigned)m->cfg.num_blocks ? alloc : (unsigned)m->cfg.num_blocks;
    out->capacity_blocks = (unsigned)m->cfg.num_blocks;
    out->visible_blocks = m->hCtr[C_VISIBLE];
    out->error_flags = m->hCtr[C_ERR];
    out->failed_allocs = m->hCtr[C_FAILED];
    out->last_triangles = m->hCtr[C_TRI];
    out->pool_bytes = m->poolBytes;
    out->device_bytes = m->deviceBytes;
    return VMAP_OK;
}

vmap_status vmap_clear_errors(vmap_map* m, void* stream)
{
    if (!m) return VMAP_ERR_INVALID_ARG;
    VMAP_CK(cudaMemsetAsync(m->dm.ctr + C_ERR, 0, sizeof(unsigned), as_stream(stream)));
    VMAP_CK(cudaMemsetAsync(m->dm.ctr + C_FAILED, 0, sizeof(unsigned), as_stream(stream)));
    return VMAP_OK;
}

vmap_status vmap_copy_counters(vmap_map* m, uint32_t* dst, void* stream)
{
    if (!m || !dst) return VMAP_ERR_INVALID_ARG;
    VMAP_CK(cudaMemcpyAsync(dst, m->dm.ctr, C_COUNT * sizeof(unsigned), cudaMemcpyDefault, as_stream(stream)));
    return VMAP_OK;
}

vmap_status vmap_timing_enable(vmap_map* m, uint32_t max_records)
{
    if (!m) return VMAP_ERR_INVALID_ARG;
    timing_free(m);
    if (max_records == 0) return VMAP_OK;
    m->tEv = new (std::nothrow) cudaEvent_t[2 * (size_t)max_records];
    m->tStage = new (std::nothrow) int[max_records];
    if (!m->tEv || !m->tStage) {
        timing_free(m);
        return VMAP_ERR_OUT_OF_MEMORY;
    }
    for (uint32_t i = 0; i < 2 * max_records; ++i) {
        cudaError_t e = cudaEventCreate(&m->tEv[i]);
        if (e != cudaSuccess) {
            m->tCap = i / 2;
            timing_free(m);
            return cuda_fail(e, "cudaEventCreate");
        }
        m->tCap = (i + 1) / 2;
    }
    m->tCap = max_records;
    m->tUsed = 0;
    return VMAP_OK;
}

vmap_status vmap_timing_read(vmap_map* m, double ms[VMAP_NUM_STAGES], uint32_t launches[VMAP_NUM_STAGES])
{
    if (!m || !ms || !launches) return VMAP_ERR_INVALID_ARG;
    for (int i = 0; i < VMAP_NUM_STAGES; ++i) {
        ms[i] = 0.0;
        launches[i] = 0;
    }
    for (unsigned i = 0; i < m->tUsed; ++i) {
        VMAP_CK(cudaEventSynchronize(m->tEv[2 * i + 1]));
        float t = 0.f;
        VMAP_CK(cudaEventElapsedTime(&t, m->tEv[2 * i], m->tEv[2 * i + 1]));
        ms[m->tStage[i]] += t;
        launches[m->tStage[i]]++;
    }
    m->tUsed = 0;
    return VMAP_OK;
}

vmap_status vmap_export_blocks(vmap_map* m, int32_t* coords, float* tsdf, float* weight, uint8_t* rgb,
                               uint32_t max_blocks, uint32_t* n_blocks, void* stream)
{
    if (!m || !n_blocks) return VMAP_ERR_INVALID_ARG;
    if (rgb && !m->cfg.with_color) return VMAP_ERR_INVALID_ARG;
    vmap_stats st;
    vmap_status r = vmap_get_stats(m, stream, &st);
    if (r != VMAP_OK) return r;
    *n_blocks = st.allocated_blocks;
    const uint32_t n = st.allocated_blocks < max_blocks ? st.allocated_blocks : max_blocks;
    if (n == 0 || (!coords && !tsdf && !weight && !rgb)) return VMAP_OK;
    cudaStream_t s = as_stream(stream);
    const int chunk = 8192;
    int* dc = nullptr;
    float *dt = nullptr, *dw = nullptr;
    uint8_t* drgb = nullptr;
    cudaError_t e = cudaMalloc((void**)&dc, (size_t)chunk * 3 * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dt, (size_t)chunk * 512 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&dw, (size_t)chunk * 512 * sizeof(float));
    if (e == cudaSuccess && rgb) e = cudaMalloc((void**)&drgb, (size_t)chunk * 512 * 3);
    for (uint32_t first = 0; e == cudaSuccess && first < n; first += chunk) {
        const int cnt = (int)((n - first) < (uint32_t)chunk ? (n - first) : (uint32_t)chunk);
        e = launch_export(m->dm, m->cfg.voxel_format, rgb != nullptr, (int)first, cnt, dc, dt, dw, drgb, s);
        if (e == cudaSuccess && coords)
            e = cudaMemcpyAsync(coords + 3 * (size_t)first, dc, (size_t)cnt * 3 * sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && tsdf)
            e = cudaMemcpyAsync(tsdf + 512 * (size_t)first, dt, (size_t)cnt * 512 * sizeof(float), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && weight)
            e = cudaMemcpyAsync(weight + 512 * (size_t)first, dw, (size_t)cnt * 512 * sizeof(float), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && rgb)
            e = cudaMemcpyAsync(rgb + 3 * 512 * (size_t)first, drgb, (size_t)cnt * 512 * 3, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFree(dc);
    cudaFree(dt);
    cudaFree(dw);
    cudaFree(drgb);
    if (e != cudaSuccess) return cuda_fail(e, "vmap_export_blocks");
    return VMAP_OK;
}

}  // extern "C"

// Internal accessors for other translation units of the library.
namespace vmapb {
const DevMap& map_device_view(const vmap_map* m) { return m->dm; }
int map_device(const vmap_map* m) { return m->device; }
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace vmapb
