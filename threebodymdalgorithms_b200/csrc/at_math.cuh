// Per-triplet Axilrod-Teller math shared by every kernel.
//
// The reference (src/potential/AxilrodTeller.cpp:23-129) works from the three side lengths and
// about 36 divisions per triplet.  Here the triplet is written in three scalars of two edge
// vectors that share the vertex i:
//   u = x_j - x_i,  v = x_k - x_i,  a = u.u,  b = v.v,  p = u.v
//   c = |x_k - x_j|^2 = a + b - 2p,  q = u.(x_k - x_j) = p - a,  s = v.(x_k - x_j) = b - p
//   D = p q s,  t = (a b c)^(-1/2)
//   E = nu (1 + 3 cos g1 cos g2 cos g3) / (r1 r2 r3)^3 = nu t^3 (1 - 3 D t^2)
// and the gradient of E(a, b, p) (c, q, s eliminated) is
//   grad_j E = alpha u + gamma v,   grad_k E = beta v + gamma u,   grad_i E = -(grad_j E + grad_k E)
// with alpha = 2 dE/da, beta = 2 dE/db, gamma = dE/dp:
//   m = -3 nu t^5,  B2 = m + 15 nu t^5 D t^2
//   alpha = B2 b (a + c) - 2 m p s
//   beta  = B2 a (b + c) + 2 m p q
//   gamma = m (q s + p s - p q) - B2 a b
// One reciprocal square root and no division per triplet.  The reference stores f = +grad E
// (it subtracts -grad E into f), which these coefficients produce directly.
#pragma once

#include <cuda_runtime.h>

namespace tbmd {

// Forward-mode dual number: value and tangent.  at_coef<Dual<T>> yields the directional
// derivatives of alpha, beta, gamma used by the Hessian-vector product.
template <class T>
struct Dual {
    T v, d;
};
template <class T>
__device__ __forceinline__ Dual<T> operator+(Dual<T> a, Dual<T> b) { return {a.v + b.v, a.d + b.d}; }
template <class T>
__device__ __forceinline__ Dual<T> operator-(Dual<T> a, Dual<T> b) { return {a.v - b.v, a.d - b.d}; }
template <class T>
__device__ __forceinline__ Dual<T> operator-(Dual<T> a) { return {-a.v, -a.d}; }
template <class T>
__device__ __forceinline__ Dual<T> operator*(Dual<T> a, Dual<T> b) { return {a.v * b.v, a.v * b.d + a.d * b.v}; }
template <class T>
__device__ __forceinline__ Dual<T> operator*(T s, Dual<T> a) { return {s * a.v, s * a.d}; }

__device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
template <class T>
__device__ __forceinline__ Dual<T> fma_(Dual<T> a, Dual<T> b, Dual<T> c) { return a * b + c; }

__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_(double x) { return rsqrt(x); }
template <class T>
__device__ __forceinline__ Dual<T> rsqrt_(Dual<T> x)
{
    T t = rsqrt_(x.v);
    return {t, T(-0.5) * t * t * t * x.d};
}

template <class T>
__device__ __forceinline__ T zero_like(T) { return T(0); }
template <class T>
__device__ __forceinline__ Dual<T> zero_like(Dual<T>) { return {T(0), T(0)}; }
template <class T>
__device__ __forceinline__ T cst(T, double c) { return T(c); }
template <class T>
__device__ __forceinline__ Dual<T> cst(Dual<T>, double c) { return {T(c), T(0)}; }

template <class S>
struct ATCoef {
    S alpha, beta, gamma;
};

// Coefficients of one triplet.  `valid` false gives exact zeros (masked lanes, k <= j, padding)
// without evaluating anything that could be inf or NaN in the result.  nu3 = -3 nu, nu15 = 15 nu.
// ENERGY adds the triplet energy nu t^3 (1 - 3 D t^2) to `e`.
template <bool ENERGY, class S>
__device__ __forceinline__ ATCoef<S> at_coef(S a, S b, S p, S nu, S nu3, S nu15, bool valid, S &e)
{
    S c = fma_(cst(a, -2.0), p, a + b);
    S q = p - a;
    S s = b - p;
    S ab = a * b;
    S t = rsqrt_(ab * c);
    if (!valid) t = zero_like(t);
    S t2 = t * t;
    S t5 = t2 * t2 * t;
    S pq = p * q;
    S ps = p * s;
    S D = pq * s;
    S Dt2 = D * t2;
    S m = nu3 * t5;
    S B2 = t5 * fma_(nu15, Dt2, nu3);
    S m2 = m + m;
    ATCoef<S> r;
    r.alpha = fma_(B2, b * (a + c), -(m2 * ps));
    r.beta = fma_(B2, a * (b + c), m2 * pq);
    r.gamma = fma_(m, fma_(q, s, ps - pq), -(B2 * ab));
    if (ENERGY) e = e + t2 * t * fma_(nu3, Dt2, nu);
    return r;
}

}  // namespace tbmd
