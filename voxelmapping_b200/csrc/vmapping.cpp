// The C++ drop-in class of include/vmapping.h over the C ABI.
// Reference: src/vmapping.cpp (VoxelizationImpl :10-148, public methods :150-191).
#include "../../include/vmapping.h"

#include <cuda_runtime.h>

#include <cstring>

namespace vmap {

namespace {

void check(vmap_status s, const char* what)
{
    if (s != VMAP_OK) {
        std::string msg = std::string(what) + ": " + vmap_status_string(s);
        const char* detail = vmap_last_error();
        if (detail && *detail && (s == VMAP_ERR_CUDA || s == VMAP_ERR_OUT_OF_MEMORY || s == VMAP_ERR_NO_DEVICE))
            msg += std::string(" (") + detail + ")";
        throw Error(s, msg);
    }
}

void check_cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw Error(VMAP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void to_pose(const Mat4f& m, double* p)
{
    for (int i = 0; i < 16; ++i) p[i] = (double)m.m[i];
}

}  // namespace

VoxelMapping::VoxelMapping(int w, int h, const Mat3f& K, vmap_voxel_format format, bool with_color)
    : width_(w), height_(h), K_(K), format_(format), with_color_(with_color)
{
}

VoxelMapping::~VoxelMapping()
{
    if (map_) vmap_destroy(map_);
    if (vmap_owned_) cudaFree(vmap_owned_);
    if (points_dev_) cudaFree(points_dev_);
}

void VoxelMapping::CreateMap(int numEntries, int numVoxels, float voxelSize)
{
    if (map_) {
        vmap_destroy(map_);
        map_ = nullptr;
    }
    vmap_config c;
    std::memset(&c, 0, sizeof(c));
    c.width = width_;
    c.height = height_;
    c.fx = K_(0, 0);
    c.fy = K_(1, 1);
    c.cx = K_(0, 2);
    c.cy = K_(1, 2);
    c.num_entries = numEntries;
    c.num_blocks = numVoxels;
    c.voxel_size = voxelSize;
    c.voxel_format = format_;
    c.with_color = with_color_ ? 1 : 0;
    check(vmap_create(&c, &map_), "CreateMap");
}

void VoxelMapping::reset()
{
    check(map_ ? vmap_reset(map_, stream_) : VMAP_ERR_INVALID_ARG, "reset");
}

void VoxelMapping::FuseDepth(const DeviceImage& depth, const Mat4f& camToWorld)
{
    if (!map_ || depth.rows != height_ || depth.cols != width_) check(VMAP_ERR_INVALID_ARG, "FuseDepth");
    double p[16];
    to_pose(camToWorld, p);
    check(vmap_fuse_depth(map_, depth.data, VMAP_DEPTH_F32, depth.pitch, 1.f, p, stream_), "FuseDepth");
}

void VoxelMapping::FuseDepthAndImage(const unsigned char* rgb, const float* depth, const Mat4f& camToWorld)
{
    if (!map_) check(VMAP_ERR_INVALID_ARG, "FuseDepthAndImage");
    double p[16];
    to_pose(camToWorld, p);
    check(vmap_fuse_host(map_, depth, VMAP_DEPTH_F32, 1.f, with_color_ ? rgb : nullptr, p, stream_),
          "FuseDepthAndImage");
    // the host images belong to the caller once this returns
    check_cuda(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream_)), "FuseDepthAndImage");
}

void VoxelMapping::RenderScene(DeviceImage& vmap, const Mat4f& camToWorld)
{
    if (!map_) check(VMAP_ERR_INVALID_ARG, "RenderScene");
    if (vmap.empty()) {  // vmapping.cpp:90-91: create(height, width, CV_32FC4)
        if (!vmap_owned_)
            check_cuda(cudaMalloc(&vmap_owned_, sizeof(float) * 4 * (size_t)width_ * height_), "RenderScene");
        vmap.data = vmap_owned_;
        vmap.pitch = sizeof(float) * 4 * (size_t)width_;
        vmap.rows = height_;
        vmap.cols = width_;
    }
    if (vmap.rows != height_ || vmap.cols != width_) check(VMAP_ERR_INVALID_ARG, "RenderScene");
    double p[16];
    to_pose(camToWorld, p);
    check(vmap_render_scene(map_, p, static_cast<float*>(vmap.data), vmap.pitch, nullptr, 0, stream_), "RenderScene");
}

int VoxelMapping::Polygonize(float*& verts_out, float*& norms_out)
{
    if (!map_) check(VMAP_ERR_INVALID_ARG, "Polygonize");
    const float *v = nullptr, *n = nullptr;
    uint32_t count = 0;
    check(vmap_polygonize_host(map_, &v, &n, &count, stream_), "Polygonize");
    verts_out = const_cast<float*>(v);
    norms_out = const_cast<float*>(n);
    return (int)count;
}

std::vector<Vector3f> VoxelMapping::GetSurfacePoints()
{
    if (!map_) check(VMAP_ERR_INVALID_ARG, "GetSurfacePoints");
    float *v = nullptr, *n = nullptr;
    const int count = Polygonize(v, n);
    std::vector<Vector3f> out((size_t)count);
    if (count == 0) return out;
    // centroids on the device from the mesh just copied out
    const size_t tri_bytes = sizeof(float) * 9 * (size_t)count, pt_bytes = sizeof(float) * 3 * (size_t)count;
    if (points_cap_ < tri_bytes + pt_bytes) {
        if (points_dev_) cudaFree(points_dev_);
        points_dev_ = nullptr;
        points_cap_ = 0;
        check_cuda(cudaMalloc(&points_dev_, tri_bytes + pt_bytes), "GetSurfacePoints");
        points_cap_ = tri_bytes + pt_bytes;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_);
    float* dv = static_cast<float*>(points_dev_);
    float* dp = dv + 9 * (size_t)count;
    check_cuda(cudaMemcpyAsync(dv, v, tri_bytes, cudaMemcpyHostToDevice, s), "GetSurfacePoints");
    check(vmap_surface_points(dv, (uint32_t)count, dp, stream_), "GetSurfacePoints");
    check_cuda(cudaMemcpyAsync(out.data(), dp, pt_bytes, cudaMemcpyDeviceToHost, s), "GetSurfacePoints");
    check_cuda(cudaStreamSynchronize(s), "GetSurfacePoints");
    return out;
}

vmap_stats VoxelMapping::stats() const
{
    vmap_stats st;
    std::memset(&st, 0, sizeof(st));
    if (map_) check(vmap_get_stats(map_, stream_, &st), "stats");
    return st;
}

void computeNormal(const DeviceImage& vmap, DeviceImage& nmap, void* stream)
{
    if (nmap.empty()) check(VMAP_ERR_INVALID_ARG, "computeNormal: nmap must be allocated");
    check(vmap_compute_normal(static_cast<const float*>(vmap.data), vmap.pitch, static_cast<float*>(nmap.data),
                              nmap.pitch, vmap.cols, vmap.rows, stream),
          "computeNormal");
}

void renderScene(const DeviceImage& vmap, const DeviceImage& nmap, DeviceImage& image, void* stream)
{
    if (image.empty()) check(VMAP_ERR_INVALID_ARG, "renderScene: image must be allocated");
    check(vmap_render_phong(static_cast<const float*>(vmap.data), vmap.pitch, static_cast<const float*>(nmap.data),
                            nmap.pitch, static_cast<unsigned char*>(image.data), image.pitch, vmap.cols, vmap.rows,
                            stream),
          "renderScene");
}

}  // namespace vmap
