/*
 * OpenCV subset for compiling the reference's CUDA sources without OpenCV
 * (TEST INFRASTRUCTURE ONLY, like eigen_subset.h).
 *
 * The reference uses OpenCV for containers only: cv::cuda::GpuMat (device
 * image with a row pitch, shared by copies), PtrStep / PtrStepSz (the kernel
 * views of a GpuMat), cv::divUp, GpuMat::setTo for CV_32FC1, and cv::Mat in
 * one unimplemented signature. No OpenCV arithmetic reaches its results.
 */
#ifndef VMAP_REF_SHIM_OPENCV_SUBSET_H
#define VMAP_REF_SHIM_OPENCV_SUBSET_H

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstddef>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <vector>

typedef unsigned char uchar;

#define CV_8UC3 16
#define CV_8UC4 24
#define CV_32FC1 5
#define CV_32FC4 29

namespace cv {

static inline int divUp(int total, unsigned grain) { return (total + int(grain) - 1) / int(grain); }
static inline std::size_t divUp(std::size_t total, unsigned grain) { return (total + grain - 1) / grain; }

struct Scalar {
    double val[4];
    Scalar(double v0 = 0, double v1 = 0, double v2 = 0, double v3 = 0) : val{v0, v1, v2, v3} {}
};

struct Size {
    int width, height;
    Size(int w = 0, int h = 0) : width(w), height(h) {}
};

struct Mat {
    int rows = 0, cols = 0;
    void* data = nullptr;
};

static inline std::size_t elem_size(int type)
{
    switch (type) {
    case CV_8UC3: return 3;
    case CV_8UC4: return 4;
    case CV_32FC1: return 4;
    case CV_32FC4: return 16;
    default: throw std::runtime_error("opencv subset: unsupported type");
    }
}

namespace cuda {

template <typename T>
struct PtrStep {
    T* data;
    std::size_t step;
    __host__ __device__ PtrStep() : data(nullptr), step(0) {}
    __host__ __device__ PtrStep(T* d, std::size_t s) : data(d), step(s) {}
    __host__ __device__ __forceinline__ T* ptr(int y = 0) { return (T*)((unsigned char*)data + y * step); }
    __host__ __device__ __forceinline__ const T* ptr(int y = 0) const
    {
        return (const T*)((const unsigned char*)data + y * step);
    }
};

template <typename T>
struct PtrStepSz : public PtrStep<T> {
    int cols, rows;
    __host__ __device__ PtrStepSz() : PtrStep<T>(), cols(0), rows(0) {}
    __host__ __device__ PtrStepSz(int r, int c, T* d, std::size_t s) : PtrStep<T>(d, s), cols(c), rows(r) {}
};

void fill_f32(void* data, std::size_t step, int rows, int cols, float value);

// Device image with a row pitch; copies share the memory (reference counted
// when this object allocated it, borrowed when it wraps caller memory).
class GpuMat {
public:
    int rows = 0, cols = 0, kind = 0;
    unsigned char* data = nullptr;
    std::size_t step = 0;

    GpuMat() {}
    GpuMat(int r, int c, int type, void* d, std::size_t s)
        : rows(r), cols(c), kind(type), data((unsigned char*)d), step(s)
    {
    }

    bool empty() const { return data == nullptr; }
    int type() const { return kind; }
    Size size() const { return Size(cols, rows); }

    void create(int r, int c, int type)
    {
        if (data && r == rows && c == cols && type == kind) return;
        void* p = nullptr;
        const std::size_t s = std::size_t(c) * elem_size(type);
        if (cudaMalloc(&p, s * std::size_t(r)) != cudaSuccess) throw std::runtime_error("GpuMat: cudaMalloc failed");
        owner_.reset(p, [](void* q) { cudaFree(q); });
        data = (unsigned char*)p;
        rows = r;
        cols = c;
        kind = type;
        step = s;
    }
    void create(Size sz, int type) { create(sz.height, sz.width, type); }

    GpuMat& setTo(Scalar s)
    {
        if (kind != CV_32FC1) throw std::runtime_error("GpuMat::setTo: CV_32FC1 only");
        fill_f32(data, step, rows, cols, float(s.val[0]));
        return *this;
    }

    template <typename T>
    operator PtrStepSz<T>() const
    {
        return PtrStepSz<T>(rows, cols, (T*)data, step);
    }
    template <typename T>
    operator PtrStep<T>() const
    {
        return PtrStep<T>((T*)data, step);
    }

private:
    std::shared_ptr<void> owner_;
};

} // namespace cuda
} // namespace cv

#endif
