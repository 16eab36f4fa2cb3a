// Host-side launchers of the libvmap_b200 kernels (internal interface between
// the C ABI glue in map.cu / batch.cu and the kernel translation units). The
// stage launchers take a view source: OneView (single map, by value) or
// ManyViews (device array of MapView for a batch).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "vmap_internal.cuh"

struct vmap_map;

namespace vmapb {

struct Launcher {
    int numSMs;
};

// fusion.cu
template <class V>
cudaError_t launch_alloc(const V& views, int totalTiles, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_visibility(const V& views, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_fuse(const V& views, int fmt, const Launcher& l, cudaStream_t s);
cudaError_t launch_reset(const DevMap& m, size_t poolBytes, const Launcher& l, cudaStream_t s);

// raycast.cu
template <class V>
cudaError_t launch_zrange(const V& views, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_raycast(const V& views, int fmt, const Launcher& l, cudaStream_t s);
template <class V>
cudaError_t launch_normals(const V& views, int totalTiles, const Launcher& l, cudaStream_t s);
cudaError_t launch_phong(const float4* vmap, size_t vpitch, const float4* nmap, size_t npitch, uchar4* rgba,
                         size_t rpitch, int W, int H, cudaStream_t s);

// mesh.cu
cudaError_t launch_mesh(const DevMap& m, int fmt, float* verts, float* norms, unsigned maxTris,
                        unsigned* ntrisOut, const Launcher& l, cudaStream_t s);
cudaError_t launch_surface_points(const float* verts, unsigned n, float* pts, cudaStream_t s);
cudaError_t launch_export(const DevMap& m, int fmt, bool color, int first, int count, int* coords, float* tsdf,
                          float* weight, uint8_t* rgb, cudaStream_t s);

// map.cu: device view of a map and the text behind vmap_last_error().
const DevMap& map_device_view(const vmap_map* m);
void set_last_error(const std::string& msg);

// 32x8-pixel tiles of a W x H image (alloc and normal-map work items)
inline int tiles_32x8(int W, int H) { return ((W + 31) / 32) * ((H + 7) / 8); }

}  // namespace vmapb
