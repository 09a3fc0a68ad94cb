// dem_math.cuh -- FP64 vector/quaternion helpers for the DEM kernels.
//
// Every helper evaluates its expression in the same operation order as the
// reference's Vec3D / Quaternion / MatrixSymmetric3D code
// (Kernel/Math/Vector.h:166-245,332-335, Vector.cc:77-80,164-167,
//  Quaternion.cc:107-170,223-226,406-438, MatrixSymmetric.cc:132-137).
// The engine is compiled with --fmad=false, so each line is a sequence of
// correctly rounded IEEE operations exactly like the reference's x86-64
// build; that makes a single contact or integration step bit-comparable.
#pragma once
#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
// plain C++ build of the same arithmetic (the CPU oracle); -ffp-contract=off
#include <cmath>
using std::fabs;
using std::sqrt;
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace dem {

struct V3 {
    double x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
// Vec3D * scalar and scalar * Vec3D both multiply each component by the scalar.
__host__ __device__ __forceinline__ V3 operator*(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator*(double s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator/(V3 a, double s) { return V3{a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__host__ __device__ __forceinline__ V3& operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__host__ __device__ __forceinline__ V3& operator*=(V3& a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }
__host__ __device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ double len2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__host__ __device__ __forceinline__ double len(V3 a) { return sqrt(len2(a)); }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ V3 zero3() { return V3{0.0, 0.0, 0.0}; }

// Unit quaternion q = (q0, q1, q2, q3).
struct Q4 {
    double q0, q1, q2, q3;
};

// Quaternion::updateAngularDisplacement (Quaternion.cc:425-438):
// q += 0.5 * C(q) * (omega dt), then q /= |q|.
__host__ __device__ __forceinline__ Q4 quat_rotate(Q4 q, V3 w)
{
    const double d0 = (-q.q1 * w.x - q.q2 * w.y - q.q3 * w.z) * 0.5;
    const double d1 = (q.q0 * w.x + q.q3 * w.y - q.q2 * w.z) * 0.5;
    const double d2 = (-q.q3 * w.x + q.q0 * w.y + q.q1 * w.z) * 0.5;
    const double d3 = (q.q2 * w.x - q.q1 * w.y + q.q0 * w.z) * 0.5;
    Q4 r{q.q0 + d0, q.q1 + d1, q.q2 + d2, q.q3 + d3};
    const double l = sqrt(r.q0 * r.q0 + r.q1 * r.q1 + r.q2 * r.q2 + r.q3 * r.q3);
    r.q0 /= l; r.q1 /= l; r.q2 /= l; r.q3 /= l;
    return r;
}

// Symmetric 3x3 (XX XY XZ YY YZ ZZ).
struct S33 {
    double xx, xy, xz, yy, yz, zz;
};

__host__ __device__ __forceinline__ V3 operator*(const S33& A, V3 b)
{
    return V3{A.xx * b.x + A.xy * b.y + A.xz * b.z,
              A.xy * b.x + A.yy * b.y + A.yz * b.z,
              A.xz * b.x + A.yz * b.y + A.zz * b.z};
}

// R * invI * R^T with R the rotation matrix of q, written out entry by entry
// in the order of Quaternion::rotateInverseInertiaTensor (Quaternion.cc:677-702).
__host__ __device__ __forceinline__ S33 rotate_inverse_inertia(Q4 q, const S33& I)
{
    const double a = 1 - 2 * q.q2 * q.q2 - 2 * q.q3 * q.q3;
    const double b = 2 * q.q1 * q.q2 - 2 * q.q0 * q.q3;
    const double c = 2 * q.q1 * q.q3 + 2 * q.q0 * q.q2;
    const double d = 2 * q.q1 * q.q2 + 2 * q.q0 * q.q3;
    const double e = 1 - 2 * q.q1 * q.q1 - 2 * q.q3 * q.q3;
    const double f = 2 * q.q2 * q.q3 - 2 * q.q0 * q.q1;
    const double g = 2 * q.q1 * q.q3 - 2 * q.q0 * q.q2;
    const double h = 2 * q.q2 * q.q3 + 2 * q.q0 * q.q1;
    const double i = 1 - 2 * q.q1 * q.q1 - 2 * q.q2 * q.q2;
    S33 r;
    r.xx = I.xx * a * a + 2 * I.xy * a * b + 2 * I.xz * a * c + I.yy * b * b + 2 * I.yz * b * c + I.zz * c * c;
    r.xy = d * (I.xx * a + I.xy * b + I.xz * c) + e * (I.xy * a + I.yy * b + I.yz * c) +
           f * (I.xz * a + I.yz * b + I.zz * c);
    r.xz = g * (I.xx * a + I.xy * b + I.xz * c) + h * (I.xy * a + I.yy * b + I.yz * c) +
           i * (I.xz * a + I.yz * b + I.zz * c);
    r.yy = I.xx * d * d + 2 * I.xy * d * e + 2 * I.xz * d * f + I.yy * e * e + 2 * I.yz * e * f + I.zz * f * f;
    r.yz = g * (I.xx * d + I.xy * e + I.xz * f) + h * (I.xy * d + I.yy * e + I.yz * f) +
           i * (I.xz * d + I.yz * e + I.zz * f);
    r.zz = I.xx * g * g + 2 * I.xy * g * h + 2 * I.xz * g * i + I.yy * h * h + 2 * I.yz * h * i + I.zz * i * i;
    return r;
}

// Signed distance of p from the plane through p0 whose outward normal is the
// first rotated axis of q (Quaternion::getDistance, Quaternion.cc:658-670).
__host__ __device__ __forceinline__ double quat_plane_distance(Q4 q, V3 p, V3 p0)
{
    const double q00 = q.q0 * q.q0;
    const double q02 = 2 * q.q0 * q.q2;
    const double q03 = 2 * q.q0 * q.q3;
    const double q11 = q.q1 * q.q1;
    const double q12 = 2 * q.q1 * q.q2;
    const double q13 = 2 * q.q1 * q.q3;
    const double q22 = q.q2 * q.q2;
    const double q33 = q.q3 * q.q3;
    return (q00 + q11 - q22 - q33) * (p0.x - p.x) + ((q12 + q03) * (p0.y - p.y) + (q13 - q02) * (p0.z - p.z));
}

// First rotated axis of q (Quaternion::getAxis, Quaternion.cc:501-512).
__host__ __device__ __forceinline__ V3 quat_axis(Q4 q)
{
    const double q00 = q.q0 * q.q0;
    const double q11 = q.q1 * q.q1;
    const double q22 = q.q2 * q.q2;
    const double q33 = q.q3 * q.q3;
    const double q12 = q.q1 * q.q2;
    const double q30 = q.q3 * q.q0;
    const double q13 = q.q1 * q.q3;
    const double q20 = q.q2 * q.q0;
    return V3{q00 - q33 + q11 - q22, 2.0 * (q12 + q30), 2.0 * (q13 - q20)};
}

} // namespace dem
