// Forward-mode dual numbers of the tangent-linear kernels: a value and its directional derivative.
// The value part performs exactly the double operations of the plain expression, in the same order,
// so a dual kernel compiled with -fmad=false reproduces the FP64 step's values bit for bit.
#pragma once
#include "common.cuh"

namespace mhd
{
struct Dual
{
    double v, d;
};
__device__ __forceinline__ Dual dl(double v) { return {v, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b)
{
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}
__device__ __forceinline__ Dual &operator+=(Dual &a, Dual b) { return a = a + b; }
__device__ __forceinline__ Dual &operator-=(Dual &a, Dual b) { return a = a - b; }
__device__ __forceinline__ Dual dsqrt(Dual a)
{
    const double s = sqrt(a.v);
    return {s, s > 0 ? a.d / (2.0 * s) : 0.0};
}
__device__ __forceinline__ Dual dabs(Dual a) { return a.v < 0 ? -a : a; }
// std::max / std::min of the reference (first argument wins ties): the derivative follows the value chosen
__device__ __forceinline__ Dual dmax(Dual a, Dual b) { return (a.v < b.v) ? b : a; }
__device__ __forceinline__ Dual dmin(Dual a, Dual b) { return (b.v < a.v) ? b : a; }

struct DV3
{
    Dual x, y, z;
};
__device__ __forceinline__ DV3 dmk(Dual x, Dual y, Dual z) { return {x, y, z}; }
__device__ __forceinline__ DV3 dmk(V3 a) { return {dl(a.x), dl(a.y), dl(a.z)}; }
__device__ __forceinline__ DV3 operator+(DV3 a, DV3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ DV3 operator-(DV3 a, DV3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ DV3 operator*(Dual s, DV3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ DV3 operator*(double s, DV3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ Dual dot(DV3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Dual dot(DV3 a, DV3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DV3 cross(V3 a, DV3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// value and tangent arrays of one dual field
struct DPtr
{
    double *v, *d;
    __device__ __forceinline__ Dual get(int64_t i) const { return {v[i], d[i]}; }
    __device__ __forceinline__ void put(int64_t i, Dual a) const
    {
        v[i] = a.v;
        d[i] = a.d;
    }
};
struct DCPtr
{
    const double *v, *d;
    __device__ __forceinline__ Dual get(int64_t i) const { return {v[i], d[i]}; }
};
__device__ __forceinline__ DV3 dld3(DCPtr a, int64_t i) { return {a.get(3 * i), a.get(3 * i + 1), a.get(3 * i + 2)}; }
__device__ __forceinline__ void dst3(DPtr a, int64_t i, DV3 x)
{
    a.put(3 * i, x.x);
    a.put(3 * i + 1, x.y);
    a.put(3 * i + 2, x.z);
}
} // namespace mhd
