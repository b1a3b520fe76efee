// dual.cuh -- forward-mode dual numbers for the adjoint: a value and N
// partial derivatives, FP64.  The node physics of lbm_common.cuh is written
// for any compute type C; instantiated with Dual<N> it yields the Jacobian of
// a node's collision with respect to N seeded inputs in one pass, from which
// the adjoint kernel takes the vector-Jacobian product.
#pragma once

#include <cuda_runtime.h>

namespace ippi {

// the sqrt overload below must not hide the FP32 / FP64 ones for code in
// this namespace
using ::sqrt;

template <int N>
struct Dual {
    double v;
    double d[N];
    __host__ __device__ constexpr Dual() : v(0), d{} {}
    __host__ __device__ constexpr Dual(double x) : v(x), d{} {}
    __device__ static Dual seed(double x, int i)
    {
        Dual r(x);
        r.d[i] = 1.0;
        return r;
    }
    __device__ Dual& operator+=(const Dual& b)
    {
        v += b.v;
#pragma unroll
        for (int i = 0; i < N; i++) d[i] += b.d[i];
        return *this;
    }
    __device__ Dual& operator-=(const Dual& b)
    {
        v -= b.v;
#pragma unroll
        for (int i = 0; i < N; i++) d[i] -= b.d[i];
        return *this;
    }
    __device__ Dual& operator*=(const Dual& b)
    {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = d[i] * b.v + v * b.d[i];
        v *= b.v;
        return *this;
    }
};

template <int N>
__device__ __forceinline__ Dual<N> operator+(Dual<N> a, const Dual<N>& b) { return a += b; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(Dual<N> a, const Dual<N>& b) { return a -= b; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(Dual<N> a, const Dual<N>& b) { return a *= b; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a)
{
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    const double inv = 1.0 / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
// a function of one value with derivative dv: chain rule
template <int N>
__device__ __forceinline__ Dual<N> chain(const Dual<N>& a, double fv, double dv)
{
    Dual<N> r;
    r.v = fv;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = dv * a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a)
{
    const double s = ::sqrt(a.v);
    return chain(a, s, s > 0 ? 0.5 / s : 0.0);
}
template <int N> __device__ __forceinline__ bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> __device__ __forceinline__ bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> __device__ __forceinline__ bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N> __device__ __forceinline__ bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }

}  // namespace ippi
