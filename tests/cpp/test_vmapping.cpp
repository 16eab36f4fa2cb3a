// Drives the C++ drop-in class (include/vmapping.h) the way the reference's
// example drives vmap::VoxelMapping: fuse frames, render, compute normals,
// polygonize, surface points. Input/output are raw little-endian files written
// and checked by tests/test_gpu_cpp.py.
//
//   in : int32 w, h, nframes, num_entries, num_blocks; float fx, fy, cx, cy, voxel_size;
//        per frame: float pose[16] (row-major camera-to-world), float depth[h*w] (metres),
//        uint8 rgb[h*w*3]
//   out: float vmap[h*w*4], float nmap[h*w*4], int32 ntri, float verts[ntri*9],
//        float norms[ntri*9], int32 npoints, float points[npoints*3]
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "vmapping.h"

static void die(const char* msg)
{
    std::fprintf(stderr, "%s\n", msg);
    std::exit(1);
}

template <typename T>
static void rd(FILE* f, T* p, size_t n)
{
    if (std::fread(p, sizeof(T), n, f) != n) die("short read");
}

template <typename T>
static void wr(FILE* f, const T* p, size_t n)
{
    if (n && std::fwrite(p, sizeof(T), n, f) != n) die("short write");
}

int main(int argc, char** argv)
{
    if (argc != 3) die("usage: test_vmapping in.bin out.bin");
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) die("cannot open input");
    int hdr[5];
    float cam[5];
    rd(in, hdr, 5);
    rd(in, cam, 5);
    const int w = hdr[0], h = hdr[1], nframes = hdr[2];
    vmap::Mat3f K = {{cam[0], 0.f, cam[2], 0.f, cam[1], cam[3], 0.f, 0.f, 1.f}};
    try {
        vmap::VoxelMapping vm(w, h, K, VMAP_VOXEL_REF, true);
        vm.CreateMap(hdr[3], hdr[4], cam[4]);
        std::vector<float> depth((size_t)w * h);
        std::vector<unsigned char> rgb((size_t)w * h * 3);
        vmap::Mat4f pose;
        void* ddepth = nullptr;
        if (cudaMalloc(&ddepth, depth.size() * sizeof(float)) != cudaSuccess) die("cudaMalloc");
        for (int i = 0; i < nframes; ++i) {
            rd(in, pose.m, 16);
            rd(in, depth.data(), depth.size());
            rd(in, rgb.data(), rgb.size());
            if (i + 1 < nframes) {
                vm.FuseDepthAndImage(rgb.data(), depth.data(), pose);  // host images (cv::Mat path)
            } else {  // device image (GpuMat path)
                cudaMemcpy(ddepth, depth.data(), depth.size() * sizeof(float), cudaMemcpyHostToDevice);
                vmap::DeviceImage d;
                d.data = ddepth;
                d.pitch = sizeof(float) * w;
                d.rows = h;
                d.cols = w;
                vm.FuseDepth(d, pose);
            }
        }
        std::fclose(in);
        vmap::DeviceImage vmap;  // empty: allocated by RenderScene
        vm.RenderScene(vmap, pose);
        vmap::DeviceImage nmap;
        if (cudaMalloc(&nmap.data, sizeof(float) * 4 * (size_t)w * h) != cudaSuccess) die("cudaMalloc");
        nmap.pitch = sizeof(float) * 4 * w;
        nmap.rows = h;
        nmap.cols = w;
        vmap::computeNormal(vmap, nmap);
        std::vector<float> hv((size_t)w * h * 4), hn((size_t)w * h * 4);
        cudaMemcpy(hv.data(), vmap.data, hv.size() * sizeof(float), cudaMemcpyDeviceToHost);
        cudaMemcpy(hn.data(), nmap.data, hn.size() * sizeof(float), cudaMemcpyDeviceToHost);
        float *verts = nullptr, *norms = nullptr;
        const int ntri = vm.Polygonize(verts, norms);
        std::vector<vmap::Vector3f> pts = vm.GetSurfacePoints();
        FILE* out = std::fopen(argv[2], "wb");
        if (!out) die("cannot open output");
        wr(out, hv.data(), hv.size());
        wr(out, hn.data(), hn.size());
        wr(out, &ntri, 1);
        wr(out, verts, (size_t)ntri * 9);
        wr(out, norms, (size_t)ntri * 9);
        const int np = (int)pts.size();
        wr(out, &np, 1);
        wr(out, reinterpret_cast<const float*>(pts.data()), (size_t)np * 3);
        std::fclose(out);
        // errors surface as exceptions, not exit(0)
        bool threw = false;
        try {
            vmap::DeviceImage wrong;
            wrong.data = ddepth;
            wrong.rows = h + 1;
            wrong.cols = w;
            vm.FuseDepth(wrong, pose);
        } catch (const vmap::Error& e) {
            threw = e.status == VMAP_ERR_INVALID_ARG;
        }
        if (!threw) die("size mismatch was not reported");
        cudaFree(ddepth);
        cudaFree(nmap.data);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    std::printf("ok\n");
    return 0;
}
