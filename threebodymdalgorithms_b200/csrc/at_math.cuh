// Per-triplet Axilrod-Teller math shared by every kernel.
//
// The reference (src/potential/AxilrodTeller.cpp:23-129) works from the three side lengths and
// about 36 divisions per triplet.  Here the triplet is written in three scalars of two edge
// vectors that share the vertex i:
//   u = x_j - x_i,  v = x_k - x_i,  a = u.u,  b = v.v,  p = u.v
//   c = |x_k - x_j|^2 = a + b - 2p,  q = u.(x_k - x_j) = p - a,  s = v.(x_k - x_j) = b - p
//   D = p q s,  t = (a b c)^(-1/2)
//   E = nu (1 + 3 cos g1 cos g2 cos g3) / (r1 r2 r3)^3 = nu t^3 (1 - 3 D t^2)
// and, with E a function of the three squared sides a, b, c, the gradient is written along the two
// sides that meet at each particle (the reference's form, AxilrodTeller.cpp:83-93):
//   grad_j E = alpha u + gamma w,   grad_k E = beta v - gamma w,   grad_i E = -(alpha u + beta v)
// with w = x_k - x_j and alpha = 2 dE/da, beta = 2 dE/db, gamma = -2 dE/dc:
//   m = -3 nu t^5,  B2 = m + 15 nu t^5 D t^2
//   alpha = B2 b c + m (q s - p s - p q)
//   beta  = B2 a c + m (q s + p s + p q)
//   gamma = m (q s + p s - p q) - B2 a b
// Writing grad_j in the basis (u, v) instead would need alpha + gamma and gamma separately, which
// are large and nearly opposite when j and k are close and i is far: their rounding error is then
// amplified by |u| / |w|.  Along the sides, no term cancels that way.
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

// FP32: the hardware approximation (PTX rsqrt.approx.ftz.f32, relative error about 2^-23).  The
// arguments a*b*c are products of squared distances and never denormal in this code.
__device__ __forceinline__ float rsqrt_(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
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

// Shared core of one triplet from the six scalars a = u.u, b = v.v, c = w.w, p = u.v, q = u.w,
// s = v.w with w = x_k - x_j, passed as ab = a b, c, p and qs = q s.  Callers form each scalar as a
// direct dot product of accurate edge vectors (never c = a + b - 2p, which cancels when j and k are
// close but far from i).  `valid` false gives exact zeros (masked lanes, k <= j, padding) without
// anything inf or NaN reaching the result.  nu3 = -3 nu, nu15 = 15 nu.  Returns m = -3 nu t^5 and
// B2 = m + 15 nu t^5 D t^2; ENERGY adds the triplet energy nu t^3 (1 - 3 D t^2) to `e`.
// One Newton step for x^(-1/2): t (1.5 - 0.5 x t^2).  Used for FP32 when the energy is also wanted:
// the energy sum of a small system can cancel, so its terms get the refined value.
__device__ __forceinline__ float refine_rsqrt(float x, float t) { return t * fmaf(-0.5f * x, t * t, 1.5f); }
__device__ __forceinline__ double refine_rsqrt(double, double t) { return t; }
template <class T>
__device__ __forceinline__ Dual<T> refine_rsqrt(Dual<T>, Dual<T> t) { return t; }

template <bool ENERGY, class S>
__device__ __forceinline__ void at_core(S ab, S c, S p, S qs, S nu, S nu3, S nu15, bool valid, S &e, S &m, S &B2)
{
    const S x = ab * c;
    S t = rsqrt_(x);
    if (ENERGY) t = refine_rsqrt(x, t);
    if (!valid) t = zero_like(t);
    S t2 = t * t;
    S t5 = t2 * t2 * t;
    S Dt2 = p * qs * t2;
    m = nu3 * t5;
    B2 = t5 * fma_(nu15, Dt2, nu3);
    if (ENERGY) e = e + t2 * t * fma_(nu3, Dt2, nu);
}

// Gradient coefficients for all three particles (see the top of this file).  With P2 = p (q + s) and
// s - q = (v - u).w = c, the three combinations are qs - ps - pq = qs - P2, qs + ps + pq = qs + P2 and
// qs + ps - pq = qs + p c (c is the directly formed w.w, the more accurate of the two equal values).
template <bool ENERGY, class S>
__device__ __forceinline__ ATCoef<S> at_coef(S a, S b, S c, S p, S q, S s, S nu, S nu3, S nu15, bool valid, S &e)
{
    S m, B2;
    const S ab = a * b, qs = q * s;
    at_core<ENERGY>(ab, c, p, qs, nu, nu3, nu15, valid, e, m, B2);
    const S P2 = p * (q + s);
    ATCoef<S> r;
    r.alpha = fma_(B2, b * c, m * (qs - P2));
    r.beta = fma_(B2, a * c, m * (qs + P2));
    r.gamma = fma_(m, fma_(p, c, qs), -(B2 * ab));
    return r;
}

// Gradient on particle i alone: grad_i E = -(alpha u + beta v) = -(sigma u + beta w)
// = -(sigma v - alpha w) with sigma = alpha + beta in closed form,
//   sigma = B2 c (a + b) + 2 m q s.
// Each of the three forms cancels in one geometry: the side form when w is the shortest side (i far
// from a close pair j, k: alpha ~ -beta, u ~ v), the (u, w) form when v is (beta w ~ -beta u), the
// (v, w) form when u is.  The caller takes (u, w) when |u| <= |v| (ub) and (v, w) otherwise; the
// side left out of the basis is then never the shortest, and no term exceeds the result by more
// than the triangle's aspect ratio of 2.  kappa is the coefficient of w: beta, or -alpha.
template <class S>
struct ATSelf {
    S sigma, kappa;
};
template <bool ENERGY, class S>
__device__ __forceinline__ ATSelf<S> at_self(S a, S b, S c, S p, S q, S s, S nu, S nu3, S nu15, bool valid, bool ub,
                                             S &e)
{
    S m, B2;
    const S qs = q * s;
    at_core<ENERGY>(a * b, c, p, qs, nu, nu3, nu15, valid, e, m, B2);
    ATSelf<S> r;
    r.sigma = fma_(B2, c * (a + b), (m + m) * qs);
    // beta = B2 a c + m (q s + p (q + s)),  -alpha = B2 (-b) c + m (-q s + p (q + s))
    const S x = ub ? a : -b, y = ub ? qs : -qs;
    r.kappa = fma_(B2, x * c, m * fma_(p, q + s, y));
    return r;
}

}  // namespace tbmd
