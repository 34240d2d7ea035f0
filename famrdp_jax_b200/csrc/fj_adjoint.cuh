// fj_adjoint.cuh -- reverse-mode (vector-Jacobian) counterparts of the face
// flux, written by hand from the forward code in fj_physics.cuh
// (muscl2_fast, roe_prim, invscd_face_fast).  Each reverse statement undoes one
// forward statement; branches take the forward branch (max/min/abs/select
// have the derivative of the branch taken; d|x|/dx at 0 is 0, as in jax.grad
// and torch.autograd).
#pragma once

#include "fj_physics.cuh"

namespace fj {

template <typename T> __device__ __forceinline__ T dsign(T x) {
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0));
}

// Reverse of muscl2_fast for one variable: lamL, lamR -> lamc[0..3] (added).
template <typename T>
__device__ __forceinline__ void muscl2_vjp(T c0, T c1, T c2, T c3, int limiter, T lamL, T lamR,
                                           T lamc[4]) {
  const T d0 = c1 - c0, d1 = c2 - c1, d2 = c3 - c2;
  // partials of lim(a, b) wrt a and b
  T pa0, pb0, pa1, pb1;
  if (limiter == 0) {  // minmod: picks a when a*b > 0 and |a| < |b|, b when a*b > 0 otherwise
    const bool s0 = d0 * d1 > T(0), s1 = d1 * d2 > T(0);
    const bool a0 = fj_abs(d0) < fj_abs(d1), a1 = fj_abs(d1) < fj_abs(d2);
    pa0 = (s0 && a0) ? T(1) : T(0);
    pb0 = (s0 && !a0) ? T(1) : T(0);
    pa1 = (s1 && a1) ? T(1) : T(0);
    pb1 = (s1 && !a1) ? T(1) : T(0);
  } else {  // van Leer 2ab/(a+b) where ab > 0
    const bool s0 = d0 * d1 > T(0), s1 = d1 * d2 > T(0);
    const T e0 = d0 + d1, e1 = d1 + d2;
    pa0 = s0 ? T(2) * d1 * d1 / (e0 * e0) : T(0);
    pb0 = s0 ? T(2) * d0 * d0 / (e0 * e0) : T(0);
    pa1 = s1 ? T(2) * d2 * d2 / (e1 * e1) : T(0);
    pb1 = s1 ? T(2) * d1 * d1 / (e1 * e1) : T(0);
  }
  // L = c1 + 0.5 sL(d0, d1); R = c2 - 0.5 sR(d1, d2)
  const T lsL = T(0.5) * lamL, lsR = T(-0.5) * lamR;
  const T ld0 = lsL * pa0;
  const T ld1 = lsL * pb0 + lsR * pa1;
  const T ld2 = lsR * pb1;
  lamc[0] += -ld0;
  lamc[1] += lamL + ld0 - ld1;
  lamc[2] += lamR + ld1 - ld2;
  lamc[3] += ld2;
}

// Reverse of roe_prim: lamF (5) -> lamL, lamR (primitive face states, set).
template <typename T>
__device__ __forceinline__ void roe_prim_vjp(const Prim<T>& L, const Prim<T>& R, T n0, T n1, T n2,
                                             T gm1, T ig, T eps_e, const T g[5], Prim<T>& lL,
                                             Prim<T>& lR) {
  using M = FastMath<T>;
  // ---- forward recomputation (same statements as roe_prim) ----
  const bool clL = L.rho > Tiny<T>::rho(), clR = R.rho > Tiny<T>::rho();
  const T rhoL = clL ? L.rho : Tiny<T>::rho(), rhoR = clR ? R.rho : Tiny<T>::rho();
  const T keL = T(0.5) * (L.u * L.u + L.v * L.v + L.w * L.w);
  const T keR = T(0.5) * (R.u * R.u + R.v * R.v + R.w * R.w);
  const T EL = L.p * ig + L.rho * keL, ER = R.p * ig + R.rho * keR;
  const T irL = M::rcp(rhoL), irR = M::rcp(rhoR);
  const T HL = (EL + L.p) * irL, HR = (ER + R.p) * irR;
  const T sqL = M::sqrt_pos(rhoL), sqR = M::sqrt_pos(rhoR);
  const T ssum = sqL + sqR;
  const bool css = ssum > Tiny<T>::ss();
  const T iss = M::rcp(css ? ssum : Tiny<T>::ss());
  const T wl = sqL * iss, wr = sqR * iss;
  const T uh = wl * L.u + wr * R.u, vh = wl * L.v + wr * R.v, wh = wl * L.w + wr * R.w;
  const T Hh = wl * HL + wr * HR;
  const T q2 = uh * uh + vh * vh + wh * wh;
  const T c2r = gm1 * (Hh - T(0.5) * q2);
  const bool cc2 = c2r > Tiny<T>::c2();
  const T c2 = cc2 ? c2r : Tiny<T>::c2();
  const T ch = M::sqrt_pos(c2);
  const T ic2 = M::rcp(c2);
  const T unh = uh * n0 + vh * n1 + wh * n2;
  const T rhoh = sqL * sqR;
  const T eps = eps_e * (fj_abs(unh) + ch);
  const T ieps = M::rcp(eps);
  const T lam1 = unh - ch, lam5 = unh + ch;
  const bool h1 = fj_abs(lam1) >= eps, h5 = fj_abs(lam5) >= eps;
  const T al1 = h1 ? fj_abs(lam1) : T(0.5) * (lam1 * lam1 * ieps + eps);
  const T al5 = h5 ? fj_abs(lam5) : T(0.5) * (lam5 * lam5 * ieps + eps);
  const T al2 = fj_abs(unh);
  const T d0 = R.rho - L.rho;
  const T d1 = R.rho * R.u - L.rho * L.u, d2 = R.rho * R.v - L.rho * L.v, d3 = R.rho * R.w - L.rho * L.w;
  const T d4 = ER - EL;
  const T dp = gm1 * (d4 - uh * d1 - vh * d2 - wh * d3 + T(0.5) * q2 * d0);
  const T dun = (d1 * n0 + d2 * n1 + d3 * n2) - unh * d0;
  const T rcd = rhoh * ch * dun;
  const T hc2 = T(0.5) * ic2;
  const T a1 = (dp - rcd) * hc2, a5 = (dp + rcd) * hc2, a23 = d0 - dp * ic2;
  const T t1 = (d1 - uh * d0) - dun * n0, t2 = (d2 - vh * d0) - dun * n1, t3 = (d3 - wh * d0) - dun * n2;
  const T t4 = uh * t1 + vh * t2 + wh * t3;
  const T s1 = al1 * a1, s5 = al5 * a5;
  const T cn0 = ch * n0, cn1 = ch * n1, cn2 = ch * n2, cun = ch * unh;
  const T unL = L.u * n0 + L.v * n1 + L.w * n2, unR = R.u * n0 + R.v * n1 + R.w * n2;
  const T mL = rhoL * unL, mR = rhoR * unR;

  // ---- reverse ----
  const T h = T(0.5);
  T lmL = 0, lmR = 0, ls1 = 0, ls5 = 0, lal2 = 0, la23 = 0, luh = 0, lvh = 0, lwh = 0, lHh = 0;
  T lcn0 = 0, lcn1 = 0, lcn2 = 0, lcun = 0, lt1 = 0, lt2 = 0, lt3 = 0, lt4 = 0, lq2 = 0;
  T luL = 0, lvL = 0, lwL = 0, lpL = 0, luR = 0, lvR = 0, lwR = 0, lpR = 0, lHL = 0, lHR = 0;
  // F0
  lmL += h * g[0];
  lmR += h * g[0];
  ls1 -= h * g[0];
  ls5 -= h * g[0];
  lal2 -= h * g[0] * a23;
  la23 -= h * g[0] * al2;
  // F1..F3
  {
    const T gv[3] = {g[1], g[2], g[3]};
    const T uLv[3] = {L.u, L.v, L.w}, uRv[3] = {R.u, R.v, R.w};
    const T nv[3] = {n0, n1, n2}, hv[3] = {uh, vh, wh}, cnv[3] = {cn0, cn1, cn2}, tv[3] = {t1, t2, t3};
    T lh[3] = {0, 0, 0}, lcn[3] = {0, 0, 0}, lt[3] = {0, 0, 0}, luLv[3] = {0, 0, 0}, luRv[3] = {0, 0, 0};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const T gg = gv[m];
      lmL += h * gg * uLv[m];
      luLv[m] += h * gg * mL;
      lpL += h * gg * nv[m];
      lmR += h * gg * uRv[m];
      luRv[m] += h * gg * mR;
      lpR += h * gg * nv[m];
      ls1 -= h * gg * (hv[m] - cnv[m]);
      ls5 -= h * gg * (hv[m] + cnv[m]);
      lh[m] -= h * gg * (s1 + s5 + al2 * a23);
      lcn[m] -= h * gg * (s5 - s1);
      lal2 -= h * gg * (a23 * hv[m] + tv[m]);
      la23 -= h * gg * al2 * hv[m];
      lt[m] -= h * gg * al2;
    }
    luh += lh[0];
    lvh += lh[1];
    lwh += lh[2];
    lcn0 += lcn[0];
    lcn1 += lcn[1];
    lcn2 += lcn[2];
    lt1 += lt[0];
    lt2 += lt[1];
    lt3 += lt[2];
    luL += luLv[0];
    lvL += luLv[1];
    lwL += luLv[2];
    luR += luRv[0];
    lvR += luRv[1];
    lwR += luRv[2];
  }
  // F4
  lmL += h * g[4] * HL;
  lHL += h * g[4] * mL;
  lmR += h * g[4] * HR;
  lHR += h * g[4] * mR;
  ls1 -= h * g[4] * (Hh - cun);
  ls5 -= h * g[4] * (Hh + cun);
  lHh -= h * g[4] * (s1 + s5);
  lcun -= h * g[4] * (s5 - s1);
  lal2 -= h * g[4] * (a23 * (h * q2) + t4);
  la23 -= h * g[4] * al2 * (h * q2);
  lq2 -= h * g[4] * al2 * a23 * h;
  lt4 -= h * g[4] * al2;
  // mL = rhoL unL, mR = rhoR unR
  T lrhoL = lmL * unL, lrhoR = lmR * unR;
  const T lunL = lmL * rhoL, lunR = lmR * rhoR;
  luL += lunL * n0;
  lvL += lunL * n1;
  lwL += lunL * n2;
  luR += lunR * n0;
  lvR += lunR * n1;
  lwR += lunR * n2;
  // cn = ch n, cun = ch unh
  T lch = lcn0 * n0 + lcn1 * n1 + lcn2 * n2 + lcun * unh;
  T lunh = lcun * ch;
  // s1 = al1 a1, s5 = al5 a5
  T lal1 = ls1 * a1, la1 = ls1 * al1, lal5 = ls5 * a5, la5 = ls5 * al5;
  // t4 = uh t1 + vh t2 + wh t3
  luh += lt4 * t1;
  lt1 += lt4 * uh;
  lvh += lt4 * t2;
  lt2 += lt4 * vh;
  lwh += lt4 * t3;
  lt3 += lt4 * wh;
  // t_m = (d_m - uh_m d0) - dun n_m
  T ld0 = 0, ld1 = 0, ld2 = 0, ld3 = 0, ld4 = 0, ldun = 0, ldp = 0, lic2 = 0, lhc2 = 0, lrcd = 0;
  ld1 += lt1;
  luh -= lt1 * d0;
  ld0 -= lt1 * uh;
  ldun -= lt1 * n0;
  ld2 += lt2;
  lvh -= lt2 * d0;
  ld0 -= lt2 * vh;
  ldun -= lt2 * n1;
  ld3 += lt3;
  lwh -= lt3 * d0;
  ld0 -= lt3 * wh;
  ldun -= lt3 * n2;
  // a23 = d0 - dp ic2
  ld0 += la23;
  ldp -= la23 * ic2;
  lic2 -= la23 * dp;
  // a1 = (dp - rcd) hc2, a5 = (dp + rcd) hc2
  ldp += la1 * hc2 + la5 * hc2;
  lrcd += -la1 * hc2 + la5 * hc2;
  lhc2 += la1 * (dp - rcd) + la5 * (dp + rcd);
  lic2 += h * lhc2;
  // rcd = rhoh ch dun
  T lrhoh = lrcd * ch * dun;
  lch += lrcd * rhoh * dun;
  ldun += lrcd * rhoh * ch;
  // dun = (d1 n0 + d2 n1 + d3 n2) - unh d0
  ld1 += ldun * n0;
  ld2 += ldun * n1;
  ld3 += ldun * n2;
  lunh -= ldun * d0;
  ld0 -= ldun * unh;
  // dp = gm1 (d4 - uh d1 - vh d2 - wh d3 + 0.5 q2 d0)
  {
    const T G = gm1 * ldp;
    ld4 += G;
    luh -= G * d1;
    ld1 -= G * uh;
    lvh -= G * d2;
    ld2 -= G * vh;
    lwh -= G * d3;
    ld3 -= G * wh;
    lq2 += G * h * d0;
    ld0 += G * h * q2;
  }
  // d4 = ER - EL; d_m = R.rho R.u_m - L.rho L.u_m; d0 = R.rho - L.rho
  T lER = ld4, lEL = -ld4;
  T lLr = -ld0 - ld1 * L.u - ld2 * L.v - ld3 * L.w;
  T lRr = ld0 + ld1 * R.u + ld2 * R.v + ld3 * R.w;
  luL -= ld1 * L.rho;
  lvL -= ld2 * L.rho;
  lwL -= ld3 * L.rho;
  luR += ld1 * R.rho;
  lvR += ld2 * R.rho;
  lwR += ld3 * R.rho;
  // al2 = |unh|; al1, al5 (Harten)
  lunh += lal2 * dsign(unh);
  T llam1 = 0, llam5 = 0, lieps = 0, leps = 0;
  if (h1) {
    llam1 += lal1 * dsign(lam1);
  } else {
    llam1 += lal1 * lam1 * ieps;
    lieps += lal1 * h * lam1 * lam1;
    leps += lal1 * h;
  }
  if (h5) {
    llam5 += lal5 * dsign(lam5);
  } else {
    llam5 += lal5 * lam5 * ieps;
    lieps += lal5 * h * lam5 * lam5;
    leps += lal5 * h;
  }
  lunh += llam1 + llam5;
  lch += -llam1 + llam5;
  leps -= lieps * ieps * ieps;
  lunh += leps * eps_e * dsign(unh);
  lch += leps * eps_e;
  // rhoh = sqL sqR
  T lsqL = lrhoh * sqR, lsqR = lrhoh * sqL;
  // unh = uh n0 + vh n1 + wh n2
  luh += lunh * n0;
  lvh += lunh * n1;
  lwh += lunh * n2;
  // ic2 = 1/c2; ch = sqrt(c2); c2 = max(c2r, tiny)
  T lc2 = -lic2 * ic2 * ic2 + lch * h * (ch * ic2);  // 1/ch = ch / c2
  const T lc2r = cc2 ? lc2 : T(0);
  // c2r = gm1 (Hh - 0.5 q2)
  lHh += gm1 * lc2r;
  lq2 -= h * gm1 * lc2r;
  // q2 = uh^2 + vh^2 + wh^2
  luh += T(2) * uh * lq2;
  lvh += T(2) * vh * lq2;
  lwh += T(2) * wh * lq2;
  // Hh = wl HL + wr HR; uh = wl uL + wr uR; ...
  T lwl = lHh * HL + luh * L.u + lvh * L.v + lwh * L.w;
  T lwr = lHh * HR + luh * R.u + lvh * R.v + lwh * R.w;
  lHL += lHh * wl;
  lHR += lHh * wr;
  luL += luh * wl;
  luR += luh * wr;
  lvL += lvh * wl;
  lvR += lvh * wr;
  lwL += lwh * wl;
  lwR += lwh * wr;
  // wl = sqL iss, wr = sqR iss; iss = 1/max(ssum, tiny); ssum = sqL + sqR
  lsqL += lwl * iss;
  lsqR += lwr * iss;
  const T liss = lwl * sqL + lwr * sqR;
  const T lss = -liss * iss * iss;
  const T lssum = css ? lss : T(0);
  lsqL += lssum;
  lsqR += lssum;
  // sq = sqrt(rho)
  lrhoL += lsqL * h * (sqL * irL);  // 1/sqL = sqL / rhoL
  lrhoR += lsqR * h * (sqR * irR);
  // H = (E + p) ir; ir = 1/rho
  lEL += lHL * irL;
  lpL += lHL * irL;
  lrhoL -= lHL * (EL + L.p) * irL * irL;
  lER += lHR * irR;
  lpR += lHR * irR;
  lrhoR -= lHR * (ER + R.p) * irR * irR;
  // E = p ig + rho ke; ke = 0.5 |u|^2
  lpL += lEL * ig;
  lLr += lEL * keL;
  const T lkeL = lEL * L.rho;
  lpR += lER * ig;
  lRr += lER * keR;
  const T lkeR = lER * R.rho;
  luL += lkeL * L.u;
  lvL += lkeL * L.v;
  lwL += lkeL * L.w;
  luR += lkeR * R.u;
  lvR += lkeR * R.v;
  lwR += lkeR * R.w;
  // rho = max(L.rho, tiny)
  lLr += clL ? lrhoL : T(0);
  lRr += clR ? lrhoR : T(0);
  lL.rho = lLr;
  lL.u = luL;
  lL.v = lvL;
  lL.w = lwL;
  lL.p = lpL;
  lR.rho = lRr;
  lR.u = luR;
  lR.v = lvR;
  lR.w = lwR;
  lR.p = lpR;
}

// Reverse of invscd_face_fast: lamF (5, on the |n|-scaled flux) -> lamc[4]
// (primitives of the four cells, added).
template <typename T>
__device__ __forceinline__ void invscd_face_vjp(const Prim<T> c[4], T kl0, T kl1, T kl2, T kr0, T kr1,
                                                T kr2, T gm1, T ig, T eps_e, int limiter,
                                                const T lamF[5], Prim<T> lamc[4]) {
  Prim<T> L, R;
  muscl2_fast(c[0].rho, c[1].rho, c[2].rho, c[3].rho, limiter, L.rho, R.rho);
  muscl2_fast(c[0].u, c[1].u, c[2].u, c[3].u, limiter, L.u, R.u);
  muscl2_fast(c[0].v, c[1].v, c[2].v, c[3].v, limiter, L.v, R.v);
  muscl2_fast(c[0].w, c[1].w, c[2].w, c[3].w, limiter, L.w, R.w);
  muscl2_fast(c[0].p, c[1].p, c[2].p, c[3].p, limiter, L.p, R.p);
  const T nf0 = T(0.5) * (kl0 + kr0), nf1 = T(0.5) * (kl1 + kr1), nf2 = T(0.5) * (kl2 + kr2);
  const T nmag = FastMath<T>::sqrt_nn(nf0 * nf0 + nf1 * nf1 + nf2 * nf2) + Tiny<T>::nmag();
  const T inv = FastMath<T>::rcp(nmag);
  T g[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) g[v] = lamF[v] * nmag;  // F_out = nmag F
  Prim<T> lL, lR;
  roe_prim_vjp(L, R, nf0 * inv, nf1 * inv, nf2 * inv, gm1, ig, eps_e, g, lL, lR);
  T lc[4];
#define FJ_MUSCL_VJP(field)                                                                    \
  lc[0] = lc[1] = lc[2] = lc[3] = T(0);                                                        \
  muscl2_vjp(c[0].field, c[1].field, c[2].field, c[3].field, limiter, lL.field, lR.field, lc); \
  lamc[0].field += lc[0];                                                                      \
  lamc[1].field += lc[1];                                                                      \
  lamc[2].field += lc[2];                                                                      \
  lamc[3].field += lc[3];
  FJ_MUSCL_VJP(rho)
  FJ_MUSCL_VJP(u)
  FJ_MUSCL_VJP(v)
  FJ_MUSCL_VJP(w)
  FJ_MUSCL_VJP(p)
#undef FJ_MUSCL_VJP
}

}  // namespace fj
