// fj_physics.cuh -- per-cell / per-face physics of the famrdp_jax hot path as
// device functions, templated on the flux arithmetic type T (double for the
// drop-in FP64 path, float for the FP32-flux path).
//
// Each function restates the reference expression it cites (famrdp_jax,
// path:line) in the same operation order; nvcc may contract a*b+c into one
// FMA, which changes results by at most one rounding per contraction.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fj {

// Clamp constants of the reference (flux/roe.py:6,23-24,33,39; rhs/invscd.py:93,
// 126; rhs/viscous.py:36).  FP32 cannot represent 1e-300 / 1e-150, so the float
// path uses the smallest normal-range values that keep the same role.
template <typename T> struct Tiny;
template <> struct Tiny<double> {
  static __device__ __forceinline__ double rho() { return 1e-300; }
  static __device__ __forceinline__ double ss() { return 1e-150; }
  static __device__ __forceinline__ double c2() { return 1e-30; }
  static __device__ __forceinline__ double nmag() { return 1e-300; }
};
template <> struct Tiny<float> {
  static __device__ __forceinline__ float rho() { return 1e-37f; }
  static __device__ __forceinline__ float ss() { return 1e-18f; }
  static __device__ __forceinline__ float c2() { return 1e-30f; }
  static __device__ __forceinline__ float nmag() { return 1e-37f; }
};

__device__ __forceinline__ double fj_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float fj_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double fj_abs(double x) { return fabs(x); }
__device__ __forceinline__ float fj_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double fj_max(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fj_max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fj_min(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float fj_min(float a, float b) { return fminf(a, b); }

// jnp.sign: -1, 0 or +1 (NaN propagates; not reached on finite data).
template <typename T> __device__ __forceinline__ T fj_sign(T x) {
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0));
}

template <typename T> struct Prim { T rho, u, v, w, p; };
template <typename T> struct Cons { T r, ru, rv, rw, rE; };
template <typename T> struct Vec5 { T a[5]; };

// physics/eos.py:12-17 (no density clamp)
template <typename T>
__device__ __forceinline__ Prim<T> cons_to_prim(T r, T ru, T rv, T rw, T rE, T gm1) {
  Prim<T> o;
  o.rho = r;
  o.u = ru / r;
  o.v = rv / r;
  o.w = rw / r;
  T ke = T(0.5) * (o.u * o.u + o.v * o.v + o.w * o.w);
  o.p = gm1 * (rE - r * ke);
  return o;
}

// physics/eos.py:5-9
template <typename T>
__device__ __forceinline__ Cons<T> prim_to_cons(const Prim<T>& pv, T gm1) {
  Cons<T> o;
  T ke = T(0.5) * (pv.u * pv.u + pv.v * pv.v + pv.w * pv.w);
  o.r = pv.rho;
  o.ru = pv.rho * pv.u;
  o.rv = pv.rho * pv.v;
  o.rw = pv.rho * pv.w;
  o.rE = pv.p / gm1 + pv.rho * ke;
  return o;
}

// physics/reconstruct/muscl2.py:5-7
template <typename T> __device__ __forceinline__ T minmod(T a, T b) {
  T sa = fj_sign(a);
  T s = sa * fj_max(sa * fj_sign(b), T(0));
  return s * fj_min(fj_abs(a), fj_abs(b));
}

// physics/reconstruct/muscl2.py:10-12
template <typename T> __device__ __forceinline__ T vanleer(T a, T b) {
  T sd = fj_abs(a + b) > T(1e-30) ? a + b : T(1);
  return a * b > T(0) ? T(2) * a * b / sd : T(0);
}

template <typename T> __device__ __forceinline__ T limit(T a, T b, int limiter) {
  return limiter == 0 ? minmod(a, b) : vanleer(a, b);
}

// physics/reconstruct/muscl2.py:18-37 for one face between cells c1 and c2:
// pL = c1 + 0.5*lim(c1-c0, c2-c1), pR = c2 - 0.5*lim(c2-c1, c3-c2)
template <typename T>
__device__ __forceinline__ void muscl2(T c0, T c1, T c2, T c3, int limiter, T& L, T& R) {
  T sL = limit(c1 - c0, c2 - c1, limiter);
  T sR = limit(c2 - c1, c3 - c2, limiter);
  L = c1 + T(0.5) * sL;
  R = c2 - T(0.5) * sR;
}

// flux/roe.py:5-18
template <typename T>
__device__ __forceinline__ void physical_flux(const Cons<T>& U, T n0, T n1, T n2, T gm1,
                                              T F[5]) {
  T rho = fj_max(U.r, Tiny<T>::rho());
  T u = U.ru / rho, v = U.rv / rho, w = U.rw / rho;
  T ke = T(0.5) * (u * u + v * v + w * w);
  T p = gm1 * (U.rE - rho * ke);
  T un = u * n0 + v * n1 + w * n2;
  T H = (U.rE + p) / rho;
  F[0] = rho * un;
  F[1] = rho * u * un + p * n0;
  F[2] = rho * v * un + p * n1;
  F[3] = rho * w * un + p * n2;
  F[4] = rho * H * un;
}

// flux/roe.py:21-85: Roe flux along the unit normal (n0, n1, n2) with the
// Harten fix on lambda_1 and lambda_5 and the reference's shear term.
template <typename T>
__device__ __forceinline__ void roe_flux(const Cons<T>& UL, const Cons<T>& UR, T n0, T n1,
                                         T n2, T gm1, T eps_entropy, T F[5]) {
  const T rhoL = fj_max(UL.r, Tiny<T>::rho());
  const T rhoR = fj_max(UR.r, Tiny<T>::rho());
  const T uL = UL.ru / rhoL, vL = UL.rv / rhoL, wL = UL.rw / rhoL;
  const T uR = UR.ru / rhoR, vR = UR.rv / rhoR, wR = UR.rw / rhoR;
  const T keL = T(0.5) * (uL * uL + vL * vL + wL * wL);
  const T keR = T(0.5) * (uR * uR + vR * vR + wR * wR);
  const T pL = gm1 * (UL.rE - rhoL * keL);
  const T pR = gm1 * (UR.rE - rhoR * keR);
  const T HL = (UL.rE + pL) / rhoL;
  const T HR = (UR.rE + pR) / rhoR;

  const T sqL = fj_sqrt(rhoL), sqR = fj_sqrt(rhoR);
  const T ss = fj_max(sqL + sqR, Tiny<T>::ss());
  const T u_h = (sqL * uL + sqR * uR) / ss;
  const T v_h = (sqL * vL + sqR * vR) / ss;
  const T w_h = (sqL * wL + sqR * wR) / ss;
  const T H_h = (sqL * HL + sqR * HR) / ss;
  const T q2 = u_h * u_h + v_h * v_h + w_h * w_h;
  const T c2 = fj_max(gm1 * (H_h - T(0.5) * q2), Tiny<T>::c2());
  const T c_h = fj_sqrt(c2);
  const T un_h = u_h * n0 + v_h * n1 + w_h * n2;
  const T rho_h = sqL * sqR;

  const T eps = eps_entropy * (fj_abs(un_h) + c_h);
  const T lam1 = un_h - c_h, lam5 = un_h + c_h;
  const T al1 = fj_abs(lam1) >= eps ? fj_abs(lam1) : T(0.5) * (lam1 * lam1 / eps + eps);
  const T al5 = fj_abs(lam5) >= eps ? fj_abs(lam5) : T(0.5) * (lam5 * lam5 / eps + eps);
  const T al2 = fj_abs(un_h);

  const T d0 = UR.r - UL.r, d1 = UR.ru - UL.ru, d2 = UR.rv - UL.rv, d3 = UR.rw - UL.rw,
          d4 = UR.rE - UL.rE;
  const T dp = gm1 * (d4 - u_h * d1 - v_h * d2 - w_h * d3 + T(0.5) * q2 * d0);
  const T dun = (d1 * n0 + d2 * n1 + d3 * n2) - un_h * d0;
  const T a1 = (dp - rho_h * c_h * dun) / (T(2) * c2);
  const T a5 = (dp + rho_h * c_h * dun) / (T(2) * c2);
  const T a23 = d0 - dp / c2;

  const T du_t = d1 / rho_h - u_h * d0 / rho_h;
  const T dv_t = d2 / rho_h - v_h * d0 / rho_h;
  const T dw_t = d3 / rho_h - w_h * d0 / rho_h;
  const T dun_full = du_t * n0 + dv_t * n1 + dw_t * n2;
  const T tu = du_t - dun_full * n0, tv = dv_t - dun_full * n1, tw = dw_t - dun_full * n2;
  const T dvt1 = rho_h * tu, dvt2 = rho_h * tv, dvt3 = rho_h * tw;
  const T dvt4 = rho_h * (u_h * tu + v_h * tv + w_h * tw);

  const T s1 = al1 * a1, s5 = al5 * a5;
  T A[5];
  A[0] = s1 + s5 + al2 * a23;
  A[1] = s1 * (u_h - c_h * n0) + s5 * (u_h + c_h * n0) + al2 * (a23 * u_h + dvt1);
  A[2] = s1 * (v_h - c_h * n1) + s5 * (v_h + c_h * n1) + al2 * (a23 * v_h + dvt2);
  A[3] = s1 * (w_h - c_h * n2) + s5 * (w_h + c_h * n2) + al2 * (a23 * w_h + dvt3);
  A[4] = s1 * (H_h - c_h * un_h) + s5 * (H_h + c_h * un_h) + al2 * (a23 * (T(0.5) * q2) + dvt4);

  T FL[5], FR[5];
  physical_flux(UL, n0, n1, n2, gm1, FL);
  physical_flux(UR, n0, n1, n2, gm1, FR);
#pragma unroll
  for (int v = 0; v < 5; ++v) F[v] = T(0.5) * (FL[v] + FR[v]) - T(0.5) * A[v];
}

// One inviscid face of rhs/invscd.py:62-100 between cells c1 and c2 along an
// axis: MUSCL on the primitives of the four cells c0..c3, prim->cons, face
// normal = 0.5*(kxyz row of c1 + row of c2), |n| + tiny, Roe, times |n|.
template <typename T>
__device__ __forceinline__ void invscd_face(const Prim<T> c[4], T kl0, T kl1, T kl2, T kr0,
                                            T kr1, T kr2, T gm1, T eps_entropy, int limiter,
                                            T F[5]) {
  Prim<T> L, R;
  muscl2(c[0].rho, c[1].rho, c[2].rho, c[3].rho, limiter, L.rho, R.rho);
  muscl2(c[0].u, c[1].u, c[2].u, c[3].u, limiter, L.u, R.u);
  muscl2(c[0].v, c[1].v, c[2].v, c[3].v, limiter, L.v, R.v);
  muscl2(c[0].w, c[1].w, c[2].w, c[3].w, limiter, L.w, R.w);
  muscl2(c[0].p, c[1].p, c[2].p, c[3].p, limiter, L.p, R.p);
  const Cons<T> UL = prim_to_cons(L, gm1);
  const Cons<T> UR = prim_to_cons(R, gm1);
  const T nf0 = T(0.5) * (kl0 + kr0), nf1 = T(0.5) * (kl1 + kr1), nf2 = T(0.5) * (kl2 + kr2);
  const T nmag = fj_sqrt(nf0 * nf0 + nf1 * nf1 + nf2 * nf2) + Tiny<T>::nmag();
  roe_flux(UL, UR, nf0 / nmag, nf1 / nmag, nf2 / nmag, gm1, eps_entropy, F);
#pragma unroll
  for (int v = 0; v < 5; ++v) F[v] = F[v] * nmag;
}

// ---------------------------------------------------------------------------
// Reformulated face flux for the fused kernels.  Same mathematics as
// roe_flux + prim_to_cons above, rearranged to cut divisions and recomputation:
//   * the face states stay primitive (the reference rebuilds u = (rho u)/rho,
//     p = (g-1)(rhoE - rho ke) from the conserved states it just built, which
//     returns the same values up to rounding);
//   * one reciprocal per divisor (1/(sqL+sqR), 1/c^2, 1/eps, 1/rho);
//   * the shear term rho_h (du_t - (du_t . n) n) of flux/roe.py:69-79 equals
//     (dU_m - u_h,m dU_0) - dun n_m with dun the normal-velocity jump of
//     flux/roe.py:57, so it needs no division by rho_h.
// For T = float the reciprocals and square roots use the fast MUFU-based
// intrinsics (__fdividef, rsqrtf); the FP32-flux path's tolerance is 1e-5.
// ---------------------------------------------------------------------------
template <typename T> struct FastMath;
template <> struct FastMath<double> {
  // __drcp_rn: the IEEE round-to-nearest reciprocal, the same value as 1.0 / x
  static __device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
  static __device__ __forceinline__ double sqrt_pos(double x) { return sqrt(x); }
  static __device__ __forceinline__ double sqrt_nn(double x) { return sqrt(x); }
};
template <> struct FastMath<float> {
  static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
  // x must be > 0
  static __device__ __forceinline__ float sqrt_pos(float x) { return x * rsqrtf(x); }
  // x >= 0
  static __device__ __forceinline__ float sqrt_nn(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
};

// minmod(a, b) of muscl2.py:5-7 without sign products: the smaller-magnitude
// argument when both have the same strict sign (a*b > 0), else 0.  (For
// |a*b| below the smallest normal the product rounds to 0 and the result is
// 0 where the reference returns the tiny min(|a|, |b|).)
template <typename T> __device__ __forceinline__ T minmod_sel(T a, T b) {
  const T m = fj_abs(a) < fj_abs(b) ? a : b;
  return a * b > T(0) ? m : T(0);
}

template <typename T>
__device__ __forceinline__ void muscl2_fast(T c0, T c1, T c2, T c3, int limiter, T& L, T& R) {
  const T d0 = c1 - c0, d1 = c2 - c1, d2 = c3 - c2;
  T sL, sR;
  if (limiter == 0) {
    sL = minmod_sel(d0, d1);
    sR = minmod_sel(d1, d2);
  } else {
    sL = vanleer(d0, d1);
    sR = vanleer(d1, d2);
  }
  L = c1 + T(0.5) * sL;
  R = c2 - T(0.5) * sR;
}

// Roe flux (flux/roe.py:21-85) of the primitive face states L, R along the unit
// normal n; inv_gm1 = 1/(gamma-1).
//
// POFF (the FP32-flux split path): the states carry the pressure OFFSET
// p' = p - p_ref instead of p.  The energies and enthalpies add p_ref back as
// constants, energy differences use p' differences, and the momentum
// components leave out the constant part p_ref n of their pressure term
// (p n = p' n + p_ref n), which the caller adds in FP64.  In FP32 that keeps
// the rounding of the large, nearly uniform pressure out of the small
// momentum fluxes and pressure jumps.  The two forms are equal in exact
// arithmetic; POFF = false is the reference arrangement.
template <typename T, bool POFF = false>
__device__ __forceinline__ void roe_prim(const Prim<T>& L, const Prim<T>& R, T n0, T n1, T n2,
                                         T gm1, T inv_gm1, T eps_entropy, T F[5], T p_ref = T(0)) {
  using M = FastMath<T>;
  const T rhoL = fj_max(L.rho, Tiny<T>::rho()), rhoR = fj_max(R.rho, Tiny<T>::rho());
  const T keL = T(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w);
  const T keR = T(0.5) * (R.u * R.u + R.v * R.v + R.w * R.w);
  // conserved energies (eos.py:8) and enthalpies
  const T eL = L.p * inv_gm1 + L.rho * keL, eR = R.p * inv_gm1 + R.rho * keR;
  const T Ec = POFF ? p_ref * inv_gm1 : T(0), Hc = POFF ? p_ref * (inv_gm1 + T(1)) : T(0);
  const T EL = POFF ? eL + Ec : eL;
  const T ER = POFF ? eR + Ec : eR;
  const T irL = M::rcp(rhoL), irR = M::rcp(rhoR);
  const T HL = (POFF ? (eL + L.p) + Hc : EL + L.p) * irL;
  const T HR = (POFF ? (eR + R.p) + Hc : ER + R.p) * irR;
  // Roe weights sqL / (sqL + sqR), sqR / (sqL + sqR) and rho_h = sqL sqR.  In
  // FP64 from one square root, t = sqrt(rhoR / rhoL): wl = 1 / (1 + t),
  // wr = t / (1 + t), rho_h = rhoL t (the same values; the reference's clamp
  // of sqL + sqR at 1e-150 cannot bind once rho >= 1e-300).  FP32 keeps the
  // two MUFU square roots.
  T wl, wr, rho_h;
  if constexpr (sizeof(T) == 8) {
    const T t = sqrt(rhoR * irL);
    wl = M::rcp(T(1) + t);
    wr = t * wl;
    rho_h = rhoL * t;
  } else {
    const T sqL = M::sqrt_pos(rhoL), sqR = M::sqrt_pos(rhoR);
    const T inv_ss = M::rcp(fj_max(sqL + sqR, Tiny<T>::ss()));
    wl = sqL * inv_ss;
    wr = sqR * inv_ss;
    rho_h = sqL * sqR;
  }
  const T u_h = wl * L.u + wr * R.u;
  const T v_h = wl * L.v + wr * R.v;
  const T w_h = wl * L.w + wr * R.w;
  const T H_h = wl * HL + wr * HR;
  const T q2 = u_h * u_h + v_h * v_h + w_h * w_h;
  const T c2 = fj_max(gm1 * (H_h - T(0.5) * q2), Tiny<T>::c2());
  T c_h, inv_c2;
  if constexpr (sizeof(T) == 8) {
    // one reciprocal square root for c and 1/c^2 (c2 >= 1e-30 > 0)
    const T ic = rsqrt(c2);
    c_h = c2 * ic;
    inv_c2 = ic * ic;
  } else {
    c_h = M::sqrt_pos(c2);
    inv_c2 = M::rcp(c2);
  }
  const T un_h = u_h * n0 + v_h * n1 + w_h * n2;

  const T eps = eps_entropy * (fj_abs(un_h) + c_h);
  const T lam1 = un_h - c_h, lam5 = un_h + c_h;
  T al1 = fj_abs(lam1), al5 = fj_abs(lam5);
  if constexpr (sizeof(T) == 8) {
    // Harten's fix (flux/roe.py:45-52) only where |lambda| < eps: the FP64
    // reciprocal of eps is taken only then
    if (al1 < eps || al5 < eps) {
      const T inv_eps = M::rcp(eps);
      if (al1 < eps) al1 = T(0.5) * (lam1 * lam1 * inv_eps + eps);
      if (al5 < eps) al5 = T(0.5) * (lam5 * lam5 * inv_eps + eps);
    }
  } else {
    const T inv_eps = M::rcp(eps);
    al1 = al1 >= eps ? al1 : T(0.5) * (lam1 * lam1 * inv_eps + eps);
    al5 = al5 >= eps ? al5 : T(0.5) * (lam5 * lam5 * inv_eps + eps);
  }
  const T al2 = fj_abs(un_h);

  const T d0 = R.rho - L.rho;
  const T d1 = R.rho * R.u - L.rho * L.u;
  const T d2 = R.rho * R.v - L.rho * L.v;
  const T d3 = R.rho * R.w - L.rho * L.w;
  const T d4 = POFF ? eR - eL : ER - EL;
  const T dp = gm1 * (d4 - u_h * d1 - v_h * d2 - w_h * d3 + T(0.5) * q2 * d0);
  const T dun = (d1 * n0 + d2 * n1 + d3 * n2) - un_h * d0;
  const T rcd = rho_h * c_h * dun;
  const T hc2 = T(0.5) * inv_c2;
  const T a1 = (dp - rcd) * hc2;
  const T a5 = (dp + rcd) * hc2;
  const T a23 = d0 - dp * inv_c2;
  const T t1 = (d1 - u_h * d0) - dun * n0;
  const T t2 = (d2 - v_h * d0) - dun * n1;
  const T t3 = (d3 - w_h * d0) - dun * n2;
  const T t4 = u_h * t1 + v_h * t2 + w_h * t3;

  const T s1 = al1 * a1, s5 = al5 * a5;
  const T cn0 = c_h * n0, cn1 = c_h * n1, cn2 = c_h * n2, cun = c_h * un_h;
  const T unL = L.u * n0 + L.v * n1 + L.w * n2;
  const T unR = R.u * n0 + R.v * n1 + R.w * n2;
  const T mL = rhoL * unL, mR = rhoR * unR;
  F[0] = T(0.5) * (mL + mR) - T(0.5) * (s1 + s5 + al2 * a23);
  const T pL = L.p, pR = R.p;  // p' with POFF: the p_ref n part is the caller's
  F[1] = T(0.5) * ((mL * L.u + pL * n0) + (mR * R.u + pR * n0)) -
         T(0.5) * (s1 * (u_h - cn0) + s5 * (u_h + cn0) + al2 * (a23 * u_h + t1));
  F[2] = T(0.5) * ((mL * L.v + pL * n1) + (mR * R.v + pR * n1)) -
         T(0.5) * (s1 * (v_h - cn1) + s5 * (v_h + cn1) + al2 * (a23 * v_h + t2));
  F[3] = T(0.5) * ((mL * L.w + pL * n2) + (mR * R.w + pR * n2)) -
         T(0.5) * (s1 * (w_h - cn2) + s5 * (w_h + cn2) + al2 * (a23 * w_h + t3));
  F[4] = T(0.5) * (mL * HL + mR * HR) -
         T(0.5) * (s1 * (H_h - cun) + s5 * (H_h + cun) + al2 * (a23 * (T(0.5) * q2) + t4));
}

// One inviscid face (rhs/invscd.py:62-100) in the reformulated arithmetic:
// MUSCL on the four cells' primitives, face normal from the two adjacent
// cells' kxyz rows, Roe, times |n|.
template <typename T, bool POFF = false>
__device__ __forceinline__ void invscd_face_fast(const Prim<T> c[4], T kl0, T kl1, T kl2, T kr0,
                                                 T kr1, T kr2, T gm1, T inv_gm1, T eps_entropy,
                                                 int limiter, T F[5], T p_ref = T(0)) {
  Prim<T> L, R;
  muscl2_fast(c[0].rho, c[1].rho, c[2].rho, c[3].rho, limiter, L.rho, R.rho);
  muscl2_fast(c[0].u, c[1].u, c[2].u, c[3].u, limiter, L.u, R.u);
  muscl2_fast(c[0].v, c[1].v, c[2].v, c[3].v, limiter, L.v, R.v);
  muscl2_fast(c[0].w, c[1].w, c[2].w, c[3].w, limiter, L.w, R.w);
  muscl2_fast(c[0].p, c[1].p, c[2].p, c[3].p, limiter, L.p, R.p);
  const T nf0 = T(0.5) * (kl0 + kr0), nf1 = T(0.5) * (kl1 + kr1), nf2 = T(0.5) * (kl2 + kr2);
  const T nmag = FastMath<T>::sqrt_nn(nf0 * nf0 + nf1 * nf1 + nf2 * nf2) + Tiny<T>::nmag();
  const T inv = FastMath<T>::rcp(nmag);
  roe_prim<T, POFF>(L, R, nf0 * inv, nf1 * inv, nf2 * inv, gm1, inv_gm1, eps_entropy, F, p_ref);
#pragma unroll
  for (int v = 0; v < 5; ++v) F[v] = F[v] * nmag;
}

// physics/eos.py:24-25 (or the constant law)
template <typename T>
__device__ __forceinline__ T viscosity(T Tt, int law, T mu0, T T0, T Ts) {
  if (law == 1) return mu0;
  const T r = Tt / T0;
  return mu0 * (r * fj_sqrt(r)) * (T0 + Ts) / (Tt + Ts);
}

}  // namespace fj
