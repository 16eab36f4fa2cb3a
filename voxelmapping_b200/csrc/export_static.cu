// vmap_export_blocks_static: block export that allocates no memory.
//
// vmap_export_blocks stages each chunk of blocks in device buffers it
// cudaMalloc's and frees on every call. Some callers must not allocate once
// they are running: a real-time loop under a no-allocation policy (an
// allocation can stall or fail mid-run), a plugin whose host application owns
// all device memory. This entry point stages through one fixed array in device
// global memory instead, sized for VMAP_EXPORT_STATIC_MAX_BLOCKS blocks, and
// copies the result into the caller's host buffers.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds it (about 1.4 MiB) until the process exits. In host code its
// name is only a host-side stand-in, so its device address is looked up with
// cudaGetSymbolAddress on every call, on the map's device (a lookup: it
// allocates nothing, and it stays right if the application tears its context
// down and the module is loaded again at another address).
#include <string>

#include "vmap_launch.h"

using namespace vmapb;

namespace {

// Per-block staging: coordinates, dequantised tsdf, weight and colour.
constexpr size_t kStageCoords = sizeof(int) * 3;
constexpr size_t kStageTsdf = sizeof(float) * kBlockVoxels;
constexpr size_t kStageWeight = sizeof(float) * kBlockVoxels;
constexpr size_t kStageRgb = 3 * kBlockVoxels;
constexpr size_t kMaxBlocks = VMAP_EXPORT_STATIC_MAX_BLOCKS;
constexpr size_t kStageBytes = kMaxBlocks * (kStageCoords + kStageTsdf + kStageWeight + kStageRgb);

static __device__ __align__(256) unsigned char g_export_stage[kStageBytes];

// Device address of the staging array on the current device.
cudaError_t stage_address(unsigned char** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_export_stage);
    if (e == cudaSuccess) *out = static_cast<unsigned char*>(p);
    return e;
}

}  // namespace

extern "C" vmap_status vmap_export_blocks_static(vmap_map* map, uint32_t first, uint32_t count, int32_t* coords,
                                                 float* tsdf, float* weight, uint8_t* rgb, uint32_t* n_blocks,
                                                 void* stream)
{
    if (!map || !n_blocks) return VMAP_ERR_INVALID_ARG;
    if (count > kMaxBlocks) {
        set_last_error("vmap_export_blocks_static: count " + std::to_string(count) + " exceeds the staging limit of " +
                       std::to_string(kMaxBlocks) + " blocks per call");
        return VMAP_ERR_INVALID_ARG;
    }
    vmap_config cfg;
    vmap_status st = vmap_get_config(map, &cfg);
    if (st != VMAP_OK) return st;
    if (rgb && !cfg.with_color) return VMAP_ERR_INVALID_ARG;
    // the staging array used is the current device's: it must be the map's
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != map_device(map)) {
        set_last_error("vmap_export_blocks_static: the current device (" + std::to_string(cur) +
                       ") is not the map's device (" + std::to_string(map_device(map)) + ")");
        return VMAP_ERR_INVALID_ARG;
    }
    vmap_stats s;
    if ((st = vmap_get_stats(map, stream, &s)) != VMAP_OK) return st;  // synchronises `stream`
    const uint32_t n = first >= s.allocated_blocks ? 0u
                       : (s.allocated_blocks - first < count ? s.allocated_blocks - first : count);
    *n_blocks = n;
    if (n == 0 || (!coords && !tsdf && !weight && !rgb)) return VMAP_OK;

    unsigned char* base = nullptr;
    cudaError_t e = stage_address(&base);
    if (e != cudaSuccess) {
        set_last_error(std::string("vmap_export_blocks_static: ") + cudaGetErrorString(e));
        return VMAP_ERR_CUDA;
    }
    int* d_coords = reinterpret_cast<int*>(base);
    float* d_tsdf = reinterpret_cast<float*>(base + kMaxBlocks * kStageCoords);
    float* d_weight = reinterpret_cast<float*>(base + kMaxBlocks * (kStageCoords + kStageTsdf));
    uint8_t* d_rgb = base + kMaxBlocks * (kStageCoords + kStageTsdf + kStageWeight);
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    // the export kernel writes every staged entry it covers, so nothing in the
    // shared array has to be cleared first
    e = launch_export(map_device_view(map), cfg.voxel_format, rgb != nullptr, (int)first, (int)n, d_coords, d_tsdf,
                      d_weight, rgb ? d_rgb : nullptr, cs);
    if (e == cudaSuccess && coords)
        e = cudaMemcpyAsync(coords, d_coords, (size_t)n * kStageCoords, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess && tsdf)
        e = cudaMemcpyAsync(tsdf, d_tsdf, (size_t)n * kStageTsdf, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess && weight)
        e = cudaMemcpyAsync(weight, d_weight, (size_t)n * kStageWeight, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess && rgb) e = cudaMemcpyAsync(rgb, d_rgb, (size_t)n * kStageRgb, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) {
        set_last_error(std::string("vmap_export_blocks_static: ") + cudaGetErrorString(e));
        return VMAP_ERR_CUDA;
    }
    return VMAP_OK;
}
