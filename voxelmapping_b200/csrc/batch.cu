// Batched fuse + raycast over many independent maps.
//
// One step fuses frame i into map i and raycasts map i at the same pose, for
// every map of the batch: each stage (allocation, visibility, fusion, z-range,
// ray marching, normals) is ONE launch covering all maps, and the ray marcher
// is a persistent kernel whose warps drain a single device-side queue of
// 8x4-pixel tiles from every map. Per-map descriptors (MapView: storage,
// camera, frame pointers, FP32 poses, outputs) live in device memory and are
// refreshed by one host-to-device copy per step from pinned staging, so the
// whole step - copy plus six kernels - is recorded once as a CUDA graph and
// replayed. Two staging buffers and two graphs alternate, so the host never
// rewrites descriptors a replay still has to copy.
//
// The reference has no counterpart: VoxelMapping drives one map per call.
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "step.h"

using namespace vmapb;

namespace vmapb {
void make_view(const vmap_map* m, const double pose[16], MapView& v);
cudaError_t next_epoch(vmap_map* m, cudaStream_t s, unsigned* epoch);
}  // namespace vmapb

struct vmap_batch {
    std::vector<vmap_map*> maps;
    int fmt;
    int totalAllocTiles;
    int totalNormalTiles;
    Launcher launcher;
    MapView* dViews[2];      // device descriptors, one set per buffer
    MapView* hViews[2];      // pinned staging
    unsigned* dQueue;        // raycast work queue
    StepSched* dSched;       // scheduler of the persistent step
    cudaEvent_t copied[2];   // the copy out of staging b has executed
    bool eventUsed[2];
    cudaGraphExec_t exec[2];
    cudaStream_t graphStream[2];  // stream each graph was recorded for
    int next;                // buffer of the next step
};

namespace {

vmap_status fail(cudaError_t e, const char* what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VMAP_ERR_OUT_OF_MEMORY : VMAP_ERR_CUDA;
}

#define VMAP_BCK(expr)                                      \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return fail(e_, #expr);      \
    } while (0)

void release(vmap_batch* b)
{
    for (int i = 0; i < 2; ++i) {
        if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
        if (b->copied[i]) cudaEventDestroy(b->copied[i]);
        cudaFree(b->dViews[i]);
        if (b->hViews[i]) cudaFreeHost(b->hViews[i]);
    }
    cudaFree(b->dQueue);
    cudaFree(b->dSched);
}

// Work-item count that makes the alloc and normals launches use their full
// grid (their kernels stride over the items of every map, so any grid is
// correct): slot batches change maps between steps without new graphs.
constexpr int kFullGrid = 1 << 30;

vmap_status finish_create(vmap_batch* b, vmap_batch** out)
{
    int dev = 0, sms = 1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->launcher.numSMs = sms;
    const size_t bytes = sizeof(MapView) * b->maps.size();
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaMalloc((void**)&b->dViews[i], bytes);
        if (e == cudaSuccess) e = cudaHostAlloc((void**)&b->hViews[i], bytes, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->copied[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->dQueue, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->dSched, sizeof(StepSched));
    if (e != cudaSuccess) {
        vmap_status st = fail(e, "vmap_batch_create");
        release(b);
        delete b;
        return st;
    }
    *out = b;
    return VMAP_OK;
}

// One step over the descriptors in dViews[buf]: the persistent launch, or
// the six stage launches.
cudaError_t enqueue_stages(vmap_batch* b, int buf, cudaStream_t s)
{
    ManyViews mv{b->dViews[buf], (int)b->maps.size(), b->dQueue};
    if (b->launcher.batchSchedule == 2) return launch_step(mv, b->dSched, b->fmt, b->launcher, s);
    cudaError_t e;
    if ((e = launch_alloc(mv, b->totalAllocTiles, b->launcher, s)) != cudaSuccess) return e;
    if ((e = launch_visibility(mv, b->launcher, s)) != cudaSuccess) return e;
    if ((e = launch_fuse(mv, b->fmt, b->launcher, s)) != cudaSuccess) return e;
    if ((e = launch_zrange(mv, b->launcher, s)) != cudaSuccess) return e;
    if ((e = launch_raycast(mv, b->fmt, b->launcher, s)) != cudaSuccess) return e;
    return launch_normals(mv, b->totalNormalTiles, b->launcher, s);
}

}  // namespace

extern "C" {

vmap_status vmap_batch_create(vmap_map* const* maps, int n_maps, vmap_batch** out)
{
    if (!maps || !out || n_maps < 1 || n_maps > kMaxBatch) return VMAP_ERR_INVALID_ARG;
    *out = nullptr;
    vmap_config c0;
    if (!maps[0] || vmap_get_config(maps[0], &c0) != VMAP_OK) return VMAP_ERR_INVALID_ARG;
    vmap_batch* b = new (std::nothrow) vmap_batch();
    if (!b) return VMAP_ERR_OUT_OF_MEMORY;
    b->fmt = c0.voxel_format;
    for (int i = 0; i < n_maps; ++i) {
        vmap_config c;
        if (!maps[i] || vmap_get_config(maps[i], &c) != VMAP_OK || c.voxel_format != b->fmt) {
            delete b;
            set_last_error("vmap_batch_create: every map needs the same voxel format");
            return VMAP_ERR_INVALID_ARG;
        }
        for (int j = 0; j < i; ++j)
            if (maps[j] == maps[i]) {
                delete b;
                set_last_error("vmap_batch_create: a map appears twice");
                return VMAP_ERR_INVALID_ARG;
            }
        b->maps.push_back(maps[i]);
        b->totalAllocTiles += stage_tiles(c.width, c.height);
    }
    b->totalNormalTiles = b->totalAllocTiles;
    return finish_create(b, out);
}

vmap_status vmap_batch_create_slots(int n_slots, int voxel_format, vmap_batch** out)
{
    if (!out || n_slots < 1 || n_slots > kMaxBatch || vmap_block_bytes(voxel_format, 0) == 0)
        return VMAP_ERR_INVALID_ARG;
    *out = nullptr;
    vmap_batch* b = new (std::nothrow) vmap_batch();
    if (!b) return VMAP_ERR_OUT_OF_MEMORY;
    b->fmt = voxel_format;
    b->maps.assign(n_slots, nullptr);
    b->totalAllocTiles = b->totalNormalTiles = kFullGrid;
    return finish_create(b, out);
}

vmap_status vmap_batch_set_map(vmap_batch* b, int slot, vmap_map* map)
{
    if (!b || slot < 0 || slot >= (int)b->maps.size()) return VMAP_ERR_INVALID_ARG;
    if (map) {
        vmap_config c;
        if (vmap_get_config(map, &c) != VMAP_OK || c.voxel_format != b->fmt) {
            set_last_error("vmap_batch_set_map: the map's voxel format differs from the batch's");
            return VMAP_ERR_INVALID_ARG;
        }
        for (int j = 0; j < (int)b->maps.size(); ++j)
            if (j != slot && b->maps[j] == map) {
                set_last_error("vmap_batch_set_map: the map is already in slot " + std::to_string(j));
                return VMAP_ERR_INVALID_ARG;
            }
    }
    if (b->totalAllocTiles != kFullGrid) {
        // grids were sized for the original maps: from now on launch full
        // grids, and record the graphs again once the steps in flight are done
        VMAP_BCK(cudaDeviceSynchronize());
        for (int i = 0; i < 2; ++i)
            if (b->exec[i]) {
                cudaGraphExecDestroy(b->exec[i]);
                b->exec[i] = nullptr;
            }
        b->totalAllocTiles = b->totalNormalTiles = kFullGrid;
    }
    b->maps[slot] = map;
    return VMAP_OK;
}

vmap_status vmap_batch_get_launch_config(const vmap_batch* b, vmap_launch_config* out)
{
    if (!b || !out) return VMAP_ERR_INVALID_ARG;
    launch_config_from(b->launcher, out);
    return VMAP_OK;
}

vmap_status vmap_batch_set_launch_config(vmap_batch* b, const vmap_launch_config* cfg)
{
    if (!b || !cfg || !launch_config_ok(cfg)) return VMAP_ERR_INVALID_ARG;
    // the recorded graphs hold the old grids: record again once the steps in flight are done
    VMAP_BCK(cudaDeviceSynchronize());
    for (int i = 0; i < 2; ++i)
        if (b->exec[i]) {
            cudaGraphExecDestroy(b->exec[i]);
            b->exec[i] = nullptr;
        }
    launch_config_to(cfg, b->launcher);
    return VMAP_OK;
}

vmap_status vmap_batch_destroy(vmap_batch* b)
{
    if (!b) return VMAP_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    release(b);
    delete b;
    return VMAP_OK;
}

}  // extern "C"

namespace {

// Validates the step's frames and writes their descriptors into staging
// buffer `buf` (after the copy out of it, recorded in the step before last,
// has run).
vmap_status stage_frames(vmap_batch* b, const vmap_batch_frame* frames, cudaStream_t s, int buf)
{
    const int n = (int)b->maps.size();
    if (b->eventUsed[buf]) VMAP_BCK(cudaEventSynchronize(b->copied[buf]));
    for (int i = 0; i < n; ++i) {
        const vmap_batch_frame& f = frames[i];
        vmap_map* m = b->maps[i];
        MapView& v = b->hViews[buf][i];
        if (!m) {  // an empty slot takes no frame and contributes no work
            if (f.depth_dev || f.vmap_dev || f.nmap_dev || f.rgb_dev) {
                set_last_error("vmap_batch_step: frame " + std::to_string(i) + " given for an empty slot");
                return VMAP_ERR_INVALID_ARG;
            }
            std::memset(&v, 0, sizeof(v));
            continue;
        }
        vmap_config c;
        vmap_get_config(m, &c);
        // a NULL depth frame skips this map's fusion, a NULL vertex map its
        // render; a frame with neither leaves the map idle for the step
        const bool fuse = f.depth_dev != nullptr, render = f.vmap_dev != nullptr;
        bool ok = (!fuse || f.depth_type == VMAP_DEPTH_F32 || f.depth_type == VMAP_DEPTH_U16) &&
                  (render || !f.nmap_dev) && (fuse || !f.rgb_dev);
        for (int k = 0; k < 12 && ok; ++k) ok = std::isfinite(f.pose[k]);
        const size_t elem = f.depth_type == VMAP_DEPTH_F32 ? 4 : 2;
        const size_t dp = f.depth_pitch ? f.depth_pitch : elem * c.width;
        const size_t row = sizeof(float4) * (size_t)c.width;
        const size_t vp = f.vmap_pitch ? f.vmap_pitch : row, np = f.nmap_pitch ? f.nmap_pitch : row;
        const size_t rp = f.rgb_pitch ? f.rgb_pitch : 3 * (size_t)c.width;
        ok = ok && (!fuse || (dp >= elem * c.width && dp % elem == 0 &&
                              (f.depth_type != VMAP_DEPTH_U16 || f.depth_scale > 0))) &&
             (!render || (vp >= row && vp % 16 == 0 && ((uintptr_t)f.vmap_dev & 15) == 0)) &&
             (!f.nmap_dev || (np >= row && np % 16 == 0)) && ((uintptr_t)f.nmap_dev & 15) == 0 &&
             (!f.rgb_dev || (c.with_color && rp >= 3 * (size_t)c.width));
        if (!ok) {
            set_last_error("vmap_batch_step: invalid frame " + std::to_string(i));
            return VMAP_ERR_INVALID_ARG;
        }
        make_view(m, f.pose, v);
        v.in.active = fuse;
        v.in.depth = f.depth_dev;
        v.in.dpitch = dp;
        v.in.dtype = f.depth_type;
        v.in.dscale = f.depth_scale;
        v.in.rgb = f.rgb_dev;
        v.in.rgbPitch = rp;
        v.out.vmap = reinterpret_cast<float4*>(f.vmap_dev);
        v.out.vpitch = vp;
        v.out.nmap = reinterpret_cast<float4*>(f.nmap_dev);
        v.out.npitch = np;
        if (render) VMAP_BCK(next_epoch(m, s, &v.out.epoch));
    }
    return VMAP_OK;
}

}  // namespace

extern "C" {

vmap_status vmap_batch_step(vmap_batch* b, const vmap_batch_frame* frames, void* stream)
{
    if (!b || !frames) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int n = (int)b->maps.size();
    const int buf = b->next;
    const vmap_status st = stage_frames(b, frames, s, buf);
    if (st != VMAP_OK) return st;
    const size_t bytes = sizeof(MapView) * (size_t)n;
    if (s == nullptr) {  // the legacy stream cannot be captured: launch directly
        VMAP_BCK(cudaMemcpyAsync(b->dViews[buf], b->hViews[buf], bytes, cudaMemcpyHostToDevice, s));
        VMAP_BCK(cudaEventRecord(b->copied[buf], s));
        VMAP_BCK(enqueue_stages(b, buf, s));
    } else {
        if (b->exec[buf] && b->graphStream[buf] != s) {
            cudaGraphExecDestroy(b->exec[buf]);
            b->exec[buf] = nullptr;
        }
        if (!b->exec[buf]) {
            cudaGraph_t g = nullptr;
            VMAP_BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = cudaMemcpyAsync(b->dViews[buf], b->hViews[buf], bytes, cudaMemcpyHostToDevice, s);
            // an external record becomes a graph node the host can wait on
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->copied[buf], s, cudaEventRecordExternal);
            if (e == cudaSuccess) e = enqueue_stages(b, buf, s);
            cudaError_t e2 = cudaStreamEndCapture(s, &g);
            if (e == cudaSuccess) e = e2;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[buf], g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(e, "vmap_batch_step capture");
            b->graphStream[buf] = s;
        }
        VMAP_BCK(cudaGraphLaunch(b->exec[buf], s));
    }
    b->eventUsed[buf] = true;
    b->next = buf ^ 1;
    return VMAP_OK;
}

vmap_status vmap_batch_stall_probe(vmap_batch* b, const vmap_batch_frame* frames, uint32_t stall_ms, void* stream)
{
    if (!b || !frames || stall_ms == 0 || stall_ms > 10000) return VMAP_ERR_INVALID_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int buf = b->next;
    const vmap_status st = stage_frames(b, frames, s, buf);
    if (st != VMAP_OK) return st;
    ManyViews mv{b->dViews[buf], (int)b->maps.size(), b->dQueue};
    VMAP_BCK(cudaMemcpyAsync(b->dViews[buf], b->hViews[buf], sizeof(MapView) * b->maps.size(),
                             cudaMemcpyHostToDevice, s));
    VMAP_BCK(cudaEventRecord(b->copied[buf], s));
    VMAP_BCK(launch_step(mv, b->dSched, b->fmt, b->launcher, s, 1000000ull * stall_ms, true));
    b->eventUsed[buf] = true;
    b->next = buf ^ 1;
    return VMAP_OK;
}

}  // extern "C"
