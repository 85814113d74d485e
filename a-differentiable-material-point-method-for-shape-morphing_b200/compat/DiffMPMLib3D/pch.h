// pch.h -- value types of the DiffMPMLib3D-compatible C++ API (compat layer
// over libdmpm.so).
//
// Where Eigen is on the include path (the reference's callers always have it),
// Vec3 and Mat3 are the reference's own typedefs, Eigen::Vector3f and
// Eigen::Matrix3f (pch.h:24-25), so caller code that does Eigen arithmetic on
// MaterialPoint fields compiles unchanged; such callers link
// libdmpm_compat_eigen.so.  Without Eigen (or with DMPM_COMPAT_NO_EIGEN
// defined) Vec3 and Mat3 are small structs with the same storage -- 3 and 9
// floats, matrices column-major, no padding -- and only the operations the API
// needs; those callers link libdmpm_compat.so.  Either way MaterialPoint and
// GridNode keep the reference's byte layout.  DMPM_COMPAT_EIGEN forces the
// Eigen types.
#pragma once
#include <cmath>
#include <memory>
#include <vector>

#if !defined(DMPM_COMPAT_EIGEN) && !defined(DMPM_COMPAT_NO_EIGEN) && defined(__has_include)
#if __has_include(<Eigen/Dense>)
#define DMPM_COMPAT_EIGEN 1
#endif
#endif

#ifdef DMPM_COMPAT_EIGEN
#include <Eigen/Dense>

namespace DiffMPMLib3D {

typedef Eigen::Vector3f Vec3;
typedef Eigen::Matrix3f Mat3;

// A:B (pch.h:27-30)
inline float InnerProduct(const Mat3& A, const Mat3& B) { return (A.array() * B.array()).sum(); }

static_assert(sizeof(Vec3) == 12 && sizeof(Mat3) == 36, "Eigen::Vector3f / Matrix3f storage");

}  // namespace DiffMPMLib3D

#else

namespace DiffMPMLib3D {

struct Vec3 {
    float d[3];
    Vec3() : d{0.f, 0.f, 0.f} {}
    Vec3(float x, float y, float z) : d{x, y, z} {}
    static Vec3 Zero() { return Vec3(); }
    float& operator[](int i) { return d[i]; }
    float operator[](int i) const { return d[i]; }
    float& operator()(int i) { return d[i]; }
    float operator()(int i) const { return d[i]; }
    float* data() { return d; }
    const float* data() const { return d; }
    Vec3 operator+(const Vec3& o) const { return Vec3(d[0] + o.d[0], d[1] + o.d[1], d[2] + o.d[2]); }
    Vec3 operator-(const Vec3& o) const { return Vec3(d[0] - o.d[0], d[1] - o.d[1], d[2] - o.d[2]); }
    Vec3 operator*(float s) const { return Vec3(d[0] * s, d[1] * s, d[2] * s); }
    Vec3& operator+=(const Vec3& o) { d[0] += o.d[0]; d[1] += o.d[1]; d[2] += o.d[2]; return *this; }
    float dot(const Vec3& o) const { return d[0] * o.d[0] + d[1] * o.d[1] + d[2] * o.d[2]; }
    float squaredNorm() const { return dot(*this); }
    float norm() const { return std::sqrt(squaredNorm()); }
    void setZero() { d[0] = d[1] = d[2] = 0.f; }
};
inline Vec3 operator*(float s, const Vec3& v) { return v * s; }

struct Mat3 {
    float d[9];  // column-major: (i, j) at d[i + 3 j]
    Mat3() { setZero(); }
    static Mat3 Zero() { return Mat3(); }
    static Mat3 Identity() { Mat3 m; m(0, 0) = m(1, 1) = m(2, 2) = 1.f; return m; }
    float& operator()(int i, int j) { return d[i + 3 * j]; }
    float operator()(int i, int j) const { return d[i + 3 * j]; }
    float* data() { return d; }
    const float* data() const { return d; }
    void setZero() { for (float& x : d) x = 0.f; }
    Mat3 operator+(const Mat3& o) const { Mat3 r; for (int k = 0; k < 9; k++) r.d[k] = d[k] + o.d[k]; return r; }
    Mat3 operator-(const Mat3& o) const { Mat3 r; for (int k = 0; k < 9; k++) r.d[k] = d[k] - o.d[k]; return r; }
    Mat3 operator*(float s) const { Mat3 r; for (int k = 0; k < 9; k++) r.d[k] = d[k] * s; return r; }
    Mat3 operator*(const Mat3& o) const {
        Mat3 r;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) r(i, j) = (*this)(i, 0) * o(0, j) + (*this)(i, 1) * o(1, j) + (*this)(i, 2) * o(2, j);
        return r;
    }
    Mat3 transpose() const { Mat3 r; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r(i, j) = (*this)(j, i); return r; }
    float squaredNorm() const { float s = 0.f; for (float x : d) s += x * x; return s; }
    float norm() const { return std::sqrt(squaredNorm()); }
};
inline Mat3 operator*(float s, const Mat3& m) { return m * s; }

// A:B (pch.h:27-30)
inline float InnerProduct(const Mat3& A, const Mat3& B) {
    float s = 0.f;
    for (int k = 0; k < 9; k++) s += A.d[k] * B.d[k];
    return s;
}

static_assert(sizeof(Vec3) == 12 && sizeof(Mat3) == 36, "Eigen::Vector3f / Matrix3f storage");

}  // namespace DiffMPMLib3D

#endif  // DMPM_COMPAT_EIGEN
