/*
 * Eigen subset for compiling the reference's CUDA sources without Eigen
 * (TEST INFRASTRUCTURE ONLY: used by oracle/ref_harness.cu to build the
 * reference as a parity anchor; the product never includes it).
 *
 * Only what the reference uses (map_struct.h, depth_fusion.cu, ray_tracing.cu,
 * marching_cubes.cu, image_proc.cu, vmapping.h): fixed-size column vectors and
 * square matrices, element access, element-wise arithmetic, cast, norm,
 * normalized, dot, cross, head<N>, Matrix4f::inverse, and
 * Transform<float,3,Affine> applied to a 3-vector.
 *
 * Arithmetic follows Eigen 3.3's evaluation order, written out as plain
 * expressions so that nvcc sees the same operation tree after inlining (and
 * contracts multiplies into adds exactly as it would inside Eigen):
 *   * reductions (sum, dot, squaredNorm, the coefficients of a small product)
 *     split in halves: three terms c0 + (c1 + c2), four (c0 + c1) + (c2 + c3)
 *     (Eigen's redux_novec_unroller; no vectorisation in device code);
 *   * Transform<T,3,Affine> * Vector3 appends a homogeneous 1 and multiplies
 *     the 4x4 matrix by it (Eigen 3.3 Transform.h, transform_right_product_impl
 *     for a rhs vector of size Dim): row i is (m_i0 v0 + m_i1 v1) +
 *     (m_i2 v2 + m_i3 * 1), and the multiply by one folds away;
 *   * cross: (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0);
 *   * normalized: v / sqrt(|v|^2) when |v|^2 > 0, else v; a scalar divide
 *     divides each coefficient.
 * One departure: Matrix4f::inverse (host only, rigid poses only) is the
 * affine inverse computed in double and rounded to float, the arithmetic of
 * the library's vmap_pose_inverse, so both builds see the same inverse pose;
 * Eigen inverts in float with its own cofactor schedule, which can differ in
 * the last bit.
 * Eigen itself is not present on this machine, so this order is a reading
 * of Eigen 3.3's source, not a measurement of it.
 */
#ifndef VMAP_REF_SHIM_EIGEN_SUBSET_H
#define VMAP_REF_SHIM_EIGEN_SUBSET_H

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <type_traits>

#define SHIM_HD __host__ __device__ __forceinline__

namespace Eigen {

enum TransformTraits { Isometry = 0x1, Affine = 0x2, AffineCompact = 0x10 | 0x2, Projective = 0x20 };

namespace shim {
template <typename T, int N>
struct align_of {
    // Eigen aligns fixed-size float/int/double objects whose size is a
    // multiple of 16 bytes to 16 bytes (Vector4f, Matrix4f); others keep the
    // scalar's alignment.
    static constexpr std::size_t value =
        ((sizeof(T) * N) % 16 == 0 && (std::is_same<T, float>::value || std::is_same<T, double>::value ||
                                       std::is_same<T, int>::value))
            ? 16
            : alignof(T);
};

// Sum of f(0) .. f(N-1) in halves, as Eigen's unrolled redux does.
template <int Start, int Len>
struct redux {
    template <typename T, typename F>
    static SHIM_HD T run(const F& f)
    {
        return redux<Start, Len / 2>::template run<T>(f) + redux<Start + Len / 2, Len - Len / 2>::template run<T>(f);
    }
};
template <int Start>
struct redux<Start, 1> {
    template <typename T, typename F>
    static SHIM_HD T run(const F& f)
    {
        return f(Start);
    }
};
} // namespace shim

template <typename T, int N>
struct Segment;

template <typename T, int R, int C>
struct alignas(shim::align_of<T, R * C>::value) Matrix {
    static constexpr int Size = R * C;
    typedef T Scalar;
    T v[R * C]; // column-major: (i, j) -> v[i + j * R]

    SHIM_HD Matrix() {}
    template <typename A, typename B>
    SHIM_HD Matrix(const A& a, const B& b)
    {
        static_assert(R * C == 2, "two coefficients");
        v[0] = T(a);
        v[1] = T(b);
    }
    template <typename A, typename B, typename D>
    SHIM_HD Matrix(const A& a, const B& b, const D& c)
    {
        static_assert(R * C == 3, "three coefficients");
        v[0] = T(a);
        v[1] = T(b);
        v[2] = T(c);
    }
    template <typename A, typename B, typename D, typename E>
    SHIM_HD Matrix(const A& a, const B& b, const D& c, const E& d)
    {
        static_assert(R * C == 4, "four coefficients");
        v[0] = T(a);
        v[1] = T(b);
        v[2] = T(c);
        v[3] = T(d);
    }
    template <int N>
    SHIM_HD Matrix(const Segment<T, N>& s);

    SHIM_HD T& operator()(int i) { return v[i]; }
    SHIM_HD const T& operator()(int i) const { return v[i]; }
    SHIM_HD T& operator[](int i) { return v[i]; }
    SHIM_HD const T& operator[](int i) const { return v[i]; }
    SHIM_HD T& operator()(int i, int j) { return v[i + j * R]; }
    SHIM_HD const T& operator()(int i, int j) const { return v[i + j * R]; }

    template <typename U>
    SHIM_HD Matrix<U, R, C> cast() const
    {
        Matrix<U, R, C> o;
        for (int i = 0; i < Size; ++i) o.v[i] = static_cast<U>(v[i]);
        return o;
    }

    SHIM_HD Matrix& operator+=(const Matrix& b)
    {
        for (int i = 0; i < Size; ++i) v[i] = v[i] + b.v[i];
        return *this;
    }
    SHIM_HD Matrix& operator-=(const Matrix& b)
    {
        for (int i = 0; i < Size; ++i) v[i] = v[i] - b.v[i];
        return *this;
    }

    SHIM_HD T dot(const Matrix& b) const
    {
        return shim::redux<0, Size>::template run<T>([&](int i) { return v[i] * b.v[i]; });
    }
    SHIM_HD T squaredNorm() const
    {
        return shim::redux<0, Size>::template run<T>([&](int i) { return v[i] * v[i]; });
    }
    SHIM_HD T norm() const
    {
        using std::sqrt;
        return sqrt(squaredNorm());
    }
    SHIM_HD Matrix normalized() const
    {
        using std::sqrt;
        T z = squaredNorm();
        if (z > T(0)) {
            T n = sqrt(z);
            Matrix o;
            for (int i = 0; i < Size; ++i) o.v[i] = v[i] / n;
            return o;
        }
        return *this;
    }
    SHIM_HD Matrix cross(const Matrix& b) const
    {
        static_assert(R == 3 && C == 1, "cross of 3-vectors");
        return Matrix(v[1] * b.v[2] - v[2] * b.v[1], v[2] * b.v[0] - v[0] * b.v[2], v[0] * b.v[1] - v[1] * b.v[0]);
    }

    template <int N>
    SHIM_HD Segment<T, N> head()
    {
        static_assert(C == 1 && N <= R, "head of a vector");
        return Segment<T, N>{v};
    }
    template <int N>
    SHIM_HD Matrix<T, N, 1> head() const
    {
        static_assert(C == 1 && N <= R, "head of a vector");
        Matrix<T, N, 1> o;
        for (int i = 0; i < N; ++i) o.v[i] = v[i];
        return o;
    }

    // host only: inverse of a 4x4 in double, rounded to T (see file header)
    Matrix inverse() const;
};

// Writable view of the first N coefficients of a vector (head<N>()).
template <typename T, int N>
struct Segment {
    T* p;
    SHIM_HD operator Matrix<T, N, 1>() const
    {
        Matrix<T, N, 1> o;
        for (int i = 0; i < N; ++i) o.v[i] = p[i];
        return o;
    }
    SHIM_HD Segment& operator=(const Matrix<T, N, 1>& m)
    {
        for (int i = 0; i < N; ++i) p[i] = m.v[i];
        return *this;
    }
};

template <typename T, int R, int C>
template <int N>
SHIM_HD Matrix<T, R, C>::Matrix(const Segment<T, N>& s)
{
    static_assert(N == R * C, "segment size");
    for (int i = 0; i < N; ++i) v[i] = s.p[i];
}

// element-wise arithmetic
template <typename T, int R, int C>
SHIM_HD Matrix<T, R, C> operator+(const Matrix<T, R, C>& a, const Matrix<T, R, C>& b)
{
    Matrix<T, R, C> o;
    for (int i = 0; i < R * C; ++i) o.v[i] = a.v[i] + b.v[i];
    return o;
}
template <typename T, int R, int C>
SHIM_HD Matrix<T, R, C> operator-(const Matrix<T, R, C>& a, const Matrix<T, R, C>& b)
{
    Matrix<T, R, C> o;
    for (int i = 0; i < R * C; ++i) o.v[i] = a.v[i] - b.v[i];
    return o;
}
template <typename T, int R, int C>
SHIM_HD Matrix<T, R, C> operator-(const Matrix<T, R, C>& a)
{
    Matrix<T, R, C> o;
    for (int i = 0; i < R * C; ++i) o.v[i] = -a.v[i];
    return o;
}
template <typename T, int R, int C, typename S,
          typename = typename std::enable_if<std::is_arithmetic<S>::value>::type>
SHIM_HD Matrix<T, R, C> operator*(const Matrix<T, R, C>& a, const S& s)
{
    Matrix<T, R, C> o;
    const T t = T(s);
    for (int i = 0; i < R * C; ++i) o.v[i] = a.v[i] * t;
    return o;
}
template <typename T, int R, int C, typename S,
          typename = typename std::enable_if<std::is_arithmetic<S>::value>::type>
SHIM_HD Matrix<T, R, C> operator*(const S& s, const Matrix<T, R, C>& a)
{
    Matrix<T, R, C> o;
    const T t = T(s);
    for (int i = 0; i < R * C; ++i) o.v[i] = t * a.v[i];
    return o;
}
template <typename T, int R, int C, typename S,
          typename = typename std::enable_if<std::is_arithmetic<S>::value>::type>
SHIM_HD Matrix<T, R, C> operator/(const Matrix<T, R, C>& a, const S& s)
{
    Matrix<T, R, C> o;
    const T t = T(s);
    for (int i = 0; i < R * C; ++i) o.v[i] = a.v[i] / t;
    return o;
}

typedef Matrix<float, 2, 1> Vector2f;
typedef Matrix<float, 3, 1> Vector3f;
typedef Matrix<float, 4, 1> Vector4f;
typedef Matrix<int, 3, 1> Vector3i;
typedef Matrix<float, 3, 3> Matrix3f;
typedef Matrix<float, 4, 4> Matrix4f;

template <typename T, int R, int C>
Matrix<T, R, C> Matrix<T, R, C>::inverse() const
{
    static_assert(R == 4 && C == 4, "4x4 inverse only");
    // The reference inverts rigid camera poses only (last row 0 0 0 1):
    // the affine inverse in double, by cofactors of the 3x3 part, the same
    // arithmetic as the library's vmap_pose_inverse, rounded to T.
    const Matrix& M = *this;
    if (!(M(3, 0) == 0 && M(3, 1) == 0 && M(3, 2) == 0 && M(3, 3) == 1))
        throw std::domain_error("eigen subset: inverse of a non-affine 4x4");
    const double a = M(0, 0), b = M(0, 1), c = M(0, 2), d = M(1, 0), e = M(1, 1), f = M(1, 2), g = M(2, 0),
                 h = M(2, 1), i = M(2, 2);
    const double A = e * i - f * h, B = f * g - d * i, Cc = d * h - e * g;
    const double r = 1.0 / (a * A + b * B + c * Cc);
    double o[3][3] = {{A * r, (c * h - b * i) * r, (b * f - c * e) * r},
                      {B * r, (a * i - c * g) * r, (c * d - a * f) * r},
                      {Cc * r, (b * g - a * h) * r, (a * e - b * d) * r}};
    Matrix out;
    for (int k = 0; k < 3; ++k) {
        for (int j = 0; j < 3; ++j) out(k, j) = T(o[k][j]);
        out(k, 3) = T(-(o[k][0] * double(M(0, 3)) + o[k][1] * double(M(1, 3)) + o[k][2] * double(M(2, 3))));
        out(3, k) = T(0);
    }
    out(3, 3) = T(1);
    return out;
}

template <typename T, int Dim, int Mode, int Options = 0>
struct Transform {
    Matrix<T, Dim + 1, Dim + 1> m;

    SHIM_HD Transform() {}
    SHIM_HD Transform(const Matrix<T, Dim + 1, Dim + 1>& mm) : m(mm) {}
    SHIM_HD Transform& operator=(const Matrix<T, Dim + 1, Dim + 1>& mm)
    {
        m = mm;
        return *this;
    }
    SHIM_HD const Matrix<T, Dim + 1, Dim + 1>& matrix() const { return m; }

    // Eigen 3.3: homogeneous (p, 1), 4x4 product, head<3>; each row reduced
    // in halves with the multiply by one folded (see file header)
    SHIM_HD Matrix<T, Dim, 1> operator*(const Matrix<T, Dim, 1>& p) const
    {
        static_assert(Dim == 3, "3-D transforms only");
        Matrix<T, Dim, 1> o;
        for (int i = 0; i < 3; ++i) o.v[i] = (m(i, 0) * p.v[0] + m(i, 1) * p.v[1]) + (m(i, 2) * p.v[2] + m(i, 3));
        return o;
    }
};

} // namespace Eigen

#endif
