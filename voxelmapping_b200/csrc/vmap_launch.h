// Host-side launchers of the libvmap_b200 kernels (internal interface between
// the C ABI glue in map.cu and the kernel translation units).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "vmap_internal.cuh"

namespace vmapb {

struct FrameParams {
    int W, H;
    float fx, fy, cx, cy;
    float ifx, ify;      // (float)(1.0 / (double)f), as the reference's host code
    const void* depth;
    size_t dpitch;
    int dtype;           // VMAP_DEPTH_*
    float dscale;        // uint16 -> metres
    const uint8_t* rgb;  // uint8x3 per pixel or NULL
    size_t rgbPitch;
    Xf T;                // camera -> world
    Xf Ti;               // world -> camera
};

struct RenderParams {
    int W, H;
    float fx, fy, cx, cy;
    float ifx, ify;
    float vsinv;   // (float)(1.0 / (double)voxel_size)
    float rts;     // truncation / voxel_size (raytraceStep)
    Xf T, Ti;
    int mode;      // 0: z-range bounded, 1: full march
    int tilesX, tilesY;
    unsigned* zmin; // tilesX * tilesY float bits
    unsigned* zmax;
};

struct Launcher {
    int numSMs;
};

cudaError_t launch_alloc(const DevMap& m, const FrameParams& f, const Launcher& l, cudaStream_t s);
cudaError_t launch_visibility(const DevMap& m, const FrameParams& f, const Launcher& l, cudaStream_t s);
cudaError_t launch_fuse(const DevMap& m, int fmt, bool color, const FrameParams& f, const Launcher& l,
                        cudaStream_t s);
cudaError_t launch_reset(const DevMap& m, size_t poolBytes, const Launcher& l, cudaStream_t s);

cudaError_t launch_zrange(const DevMap& m, const RenderParams& r, const Launcher& l, cudaStream_t s);
cudaError_t launch_raycast(const DevMap& m, int fmt, const RenderParams& r, float4* vmap, size_t vpitch,
                           const Launcher& l, cudaStream_t s);
cudaError_t launch_normals(const float4* vmap, size_t vpitch, float4* nmap, size_t npitch, int W, int H,
                           cudaStream_t s);
cudaError_t launch_phong(const float4* vmap, size_t vpitch, const float4* nmap, size_t npitch, uchar4* rgba,
                         size_t rpitch, int W, int H, cudaStream_t s);

cudaError_t launch_mesh(const DevMap& m, int fmt, float* verts, float* norms, unsigned maxTris,
                        unsigned* ntrisOut, const Launcher& l, cudaStream_t s);
cudaError_t launch_surface_points(const float* verts, unsigned n, float* pts, cudaStream_t s);

cudaError_t launch_export(const DevMap& m, int fmt, bool color, int first, int count, int* coords, float* tsdf,
                          float* weight, uint8_t* rgb, cudaStream_t s);

}  // namespace vmapb

struct vmap_map;
#include <string>
namespace vmapb {
// map.cu: device view of a map and the text behind vmap_last_error().
const DevMap& map_device_view(const vmap_map* m);
void set_last_error(const std::string& msg);
}  // namespace vmapb
