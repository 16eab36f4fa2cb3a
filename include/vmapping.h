// vmapping.h - C++ drop-in for the reference's vmap::VoxelMapping
// (xingruiyang/VoxelMapping include/vmapping.h:10-27, image_proc.h:10-11),
// implemented over the C ABI in vmap_c.h (libvmap_b200.so).
//
// Same class, method names, argument meaning and ownership rules. Eigen and
// OpenCV types are replaced by small PODs so the header has no dependency:
//   Eigen::Matrix3f / Matrix4f  -> Mat3f / Mat4f (row-major values; with Eigen,
//                                  pass m.transpose().data() or copy (r, c))
//   cv::cuda::GpuMat             -> DeviceImage (device pointer, pitch, size)
//   cv::Mat                      -> host pointers (tightly packed rows)
// Differences from the reference: failures throw vmap::Error (the reference
// calls exit(0)); FuseDepthAndImage is implemented (a stub there); misses in
// the vertex map are NaN in all four lanes; calls are asynchronous on the
// object's stream (set_stream) instead of synchronising the device.
#ifndef VMAP_VMAPPING_H
#define VMAP_VMAPPING_H

#include <stdexcept>
#include <string>
#include <vector>

#include "vmap_c.h"

namespace vmap {

struct Mat3f {
    float m[9];  // row-major
    float operator()(int r, int c) const { return m[3 * r + c]; }
};

struct Mat4f {
    float m[16];  // row-major, camera-to-world
    float operator()(int r, int c) const { return m[4 * r + c]; }
};

struct Vector3f {
    float x, y, z;
};

// A device image: `data` in CUDA device memory, `pitch` in bytes.
struct DeviceImage {
    void* data = nullptr;
    size_t pitch = 0;
    int rows = 0, cols = 0;
    bool empty() const { return data == nullptr; }
};

class Error : public std::runtime_error {
public:
    Error(vmap_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    vmap_status status;
};

class VoxelMapping {
public:
    // reference VoxelMapping(int w, int h, const Eigen::Matrix3f& K); the
    // extension arguments select the voxel format (REF = the reference's
    // int16 TSDF + uint8 weight) and whether colour is kept.
    VoxelMapping(int w, int h, const Mat3f& K, vmap_voxel_format format = VMAP_VOXEL_REF, bool with_color = true);
    ~VoxelMapping();
    VoxelMapping(const VoxelMapping&) = delete;
    VoxelMapping& operator=(const VoxelMapping&) = delete;

    void reset();
    void CreateMap(int numEntries, int numVoxels, float voxelSize);
    // depth: float metres (CV_32FC1); camToWorld: row-major
    void FuseDepth(const DeviceImage& depth, const Mat4f& camToWorld);
    // host images: rgb uint8x3 (may be NULL), depth float metres, both w x h
    void FuseDepthAndImage(const unsigned char* rgb, const float* depth, const Mat4f& camToWorld);
    // vmap: float4 per pixel (CV_32FC4), camera frame; allocated by the
    // object when empty (valid until the object is destroyed), as the
    // reference allocates the GpuMat
    void RenderScene(DeviceImage& vmap, const Mat4f& camToWorld);
    // triangle count; verts_out / norms_out point at library-owned host
    // buffers of 9 floats per triangle, valid until the next call
    int Polygonize(float*& verts_out, float*& norms_out);
    std::vector<Vector3f> GetSurfacePoints();

    // extensions
    void set_stream(void* cuda_stream) { stream_ = cuda_stream; }
    vmap_map* handle() const { return map_; }
    vmap_stats stats() const;

private:
    int width_, height_;
    Mat3f K_;
    vmap_voxel_format format_;
    bool with_color_;
    vmap_map* map_ = nullptr;
    void* stream_ = nullptr;
    void* vmap_owned_ = nullptr;
    void* points_dev_ = nullptr;
    size_t points_cap_ = 0;
};

// image_proc.h:10-11
void computeNormal(const DeviceImage& vmap, DeviceImage& nmap, void* stream = nullptr);
void renderScene(const DeviceImage& vmap, const DeviceImage& nmap, DeviceImage& image, void* stream = nullptr);

}  // namespace vmap

#endif  // VMAP_VMAPPING_H
