// fj_adjoint.cu -- hand-written reverse mode of the RHS and of the TVD-RK3
// step (the reference differentiates its step with jax.grad,
// tests/solver/test_grad.py:30-35; there is no hand-written adjoint there).
//
// RHS vector-Jacobian product lam -> (dL/dq)^T lam for one block, four kernels:
//   k_adj_prims    primitives (rho, u, v, w, p, T) of q                 (forward)
//   k_adj_faces    per cell c and axis a with a face c | c+e_a: the face's
//                  adjoint  lamF = -lam(c)/vol(c) [c in range] + lam(c+e_a)/
//                  vol(c+e_a) [c+e_a in range]  (reverse of rhs/invscd.py:
//                  119-131), then the reverse of MUSCL + Roe; the primitive
//                  adjoints of the four cells are atomically added to lamP
//   k_adj_visc     per cell y: lamG(y) gathered from the six neighbours'
//                  lam and kxyz (reverse of the divergence, rhs/viscous.py:
//                  86-117), then the reverse of the viscous fluxes at y:
//                  lamD[s][l] (adjoint of the central difference of u, v, w, T
//                  along l) and the local adjoints of u, v, w, T at y
//   k_adj_final    per cell: lamP + local + the neighbours' lamD gathered back
//                  through the central differences, the reverse of
//                  T = p/(rho R) and of cons_to_prim (physics/eos.py:12-17)
// All neighbour indices wrap around the padded block like the forward.
//
// The step adjoint recomputes q0' (copy + halo + BC), q1 and q2 with the
// forward kernels, then applies the transposed stage combines and RHS VJPs
// in reverse (solver/step.py:45-53) and finally the transposed boundary
// conditions and halo fill (mesh/halo.py:56-92, physics/bc/*.py).
#include <algorithm>
#include <vector>

#include "fj_adjoint.cuh"
#include "fj_common.cuh"
#include "fj_rhs.cuh"

namespace fj {

namespace {

constexpr int kAT = 256;

struct ADims {
  int ni, nj, nk;
};

__device__ __forceinline__ void dec(int c, const ADims& d, int& i, int& j, int& k) {
  k = c % d.nk;
  const int t = c / d.nk;
  j = t % d.nj;
  i = t / d.nj;
}

__device__ __forceinline__ void wrapped(int c, int i, int j, int k, const ADims& d, int nb[6]) {
  const int si = d.nj * d.nk, sj = d.nk;
  nb[0] = i + 1 == d.ni ? c - (d.ni - 1) * si : c + si;
  nb[1] = i == 0 ? c + (d.ni - 1) * si : c - si;
  nb[2] = j + 1 == d.nj ? c - (d.nj - 1) * sj : c + sj;
  nb[3] = j == 0 ? c + (d.nj - 1) * sj : c - sj;
  nb[4] = k + 1 == d.nk ? c - (d.nk - 1) : c + 1;
  nb[5] = k == 0 ? c + (d.nk - 1) : c - 1;
}

// The primitives (rho, u, v, w, p, T) of the forward evaluation: in FP32 one
// 32-byte record per cell (two pad values), moved with one 256-bit load or
// store that covers whole sectors; in FP64 six field-major arrays.
template <typename T>
constexpr int kPVals = sizeof(T) == 4 ? 8 : 6;  // values per cell in the primitive buffer

template <typename T>
__device__ __forceinline__ void load_prims(const T* __restrict__ P, int N, int c, T x[6]) {
  if constexpr (sizeof(T) == 4) {
    float v6, v7;
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(x[0]), "=f"(x[1]), "=f"(x[2]), "=f"(x[3]), "=f"(x[4]), "=f"(x[5]), "=f"(v6), "=f"(v7)
        : "l"(P + (size_t)c * 8));
  } else {
#pragma unroll
    for (int f = 0; f < 6; ++f) x[f] = P[(size_t)f * N + c];
  }
}

template <typename T>
__device__ __forceinline__ void store_prims(T* __restrict__ P, int N, int c, const T x[6]) {
  if constexpr (sizeof(T) == 4) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(P + (size_t)c * 8), "f"(x[0]),
                 "f"(x[1]), "f"(x[2]), "f"(x[3]), "f"(x[4]), "f"(x[5]), "f"(0.0f), "f"(0.0f)
                 : "memory");
  } else {
#pragma unroll
    for (int f = 0; f < 6; ++f) P[(size_t)f * N + c] = x[f];
  }
}

// q -> (rho, u, v, w, p, T) of cell c, in the primitive buffer's layout
template <typename T>
__device__ __forceinline__ void write_prims(const double* __restrict__ q, T* __restrict__ P, int N, int c,
                                            double gm1, double R) {
  const double r = q[c], ir = 1.0 / r;
  const double u = q[N + c] * ir, v = q[2 * N + c] * ir, w = q[3 * N + c] * ir;
  const double p = gm1 * (q[4 * N + c] - r * (0.5 * (u * u + v * v + w * w)));
  const T x[6] = {(T)r, (T)u, (T)v, (T)w, (T)p, (T)(r * R > 1e-300 ? p * ir * (1.0 / R) : p * 1e300)};
  store_prims<T>(P, N, c, x);
}

// With lv, also lv = lam / (vol + 1e-300) per cell, in FP64: the face adjoint
// -lam(c)/vol(c) + lam(c+e_a)/vol(c+e_a) of every axis then costs one FP64
// subtraction per face instead of two divisions.
template <typename T>
__global__ void k_adj_prims(const double* __restrict__ q, T* __restrict__ P, int N, double gm1,
                            double R, const double* __restrict__ lam, const double* __restrict__ vol,
                            double* __restrict__ lv, T* __restrict__ lamP) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  if (lamP)  // cleared here for the face kernel's atomic sums
#pragma unroll
    for (int v = 0; v < 5; ++v) lamP[v * N + c] = T(0);
  if (lv) {
    const double iv = 1.0 / (vol[c] + 1e-300);
#pragma unroll
    for (int v = 0; v < 5; ++v) lv[v * N + c] = lam[v * N + c] * iv;
  }
  write_prims<T>(q, P, N, c, gm1, R);
}

__device__ __forceinline__ void atomic_add(float* a, float v) { atomicAdd(a, v); }
__device__ __forceinline__ void atomic_add(double* a, double v) { atomicAdd(a, v); }

// Face c | c+e_a (stride sa): loads the four MUSCL cells and the two cells'
// metric rows, then the reverse of MUSCL + Roe; lc[s][v] = adjoint of the
// primitive v (rho, u, v, w, p) of cell c + (s-1) e_a.
template <typename T>
__device__ __forceinline__ void face_vjp_cells(const T* __restrict__ P, const double* __restrict__ K, int N,
                                               int c, int sa, const T lF[5], const Phys& ph, T lc[4][5]) {
  Prim<T> cell[4], l4[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int cc = c + (s - 1) * sa;
    T x[6];
    load_prims<T>(P, N, cc, x);
    cell[s] = Prim<T>{x[0], x[1], x[2], x[3], x[4]};
    l4[s] = Prim<T>{T(0), T(0), T(0), T(0), T(0)};
  }
  const int cr = c + sa;
  invscd_face_vjp<T>(cell, (T)K[c], (T)K[N + c], (T)K[2 * N + c], (T)K[cr], (T)K[N + cr], (T)K[2 * N + cr],
                     (T)ph.gm1, (T)ph.inv_gm1, (T)ph.eps_entropy, ph.limiter, lF, l4);
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    lc[s][0] = l4[s].rho;
    lc[s][1] = l4[s].u;
    lc[s][2] = l4[s].v;
    lc[s][3] = l4[s].w;
    lc[s][4] = l4[s].p;
  }
}

template <typename T>
__device__ __forceinline__ void add_cell(T* __restrict__ lamP, int N, int c, const T v[5]) {
#pragma unroll
  for (int f = 0; f < 5; ++f)
    if (v[f] != T(0)) atomic_add(lamP + f * N + c, v[f]);
}

// The inviscid part of the RHS VJP (reverse of rhs/invscd.py:119-131 and of
// MUSCL + Roe), accumulated into lamP.  One thread per face c | c+e_a over the
// linear cell index c, blockIdx.y = the face axis a.  Face adjoint
// lamF = -lam(c)/vol(c) [2 <= c_a <= n_a-3] + lam(c+e_a)/vol(c+e_a)
// [c_a+1 <= n_a-3] for faces 1 <= c_a <= n_a-3, in FP64 as the forward's flux
// difference.  Along k (a = 2) the four contributions to a cell x come from
// lanes x+1, x, x-1, x-2 of the same warp and are combined by shuffles, so only
// each cell's total and the contributions that leave the warp use atomics
// (faces at the ends of a k row are invalid and contribute zero, so a warp that
// spans two rows combines correctly); along i and j each face adds its four
// cells' adjoints atomically.
// (a, bx) = the face axis and the block of faces this CTA takes.
template <typename T>
__device__ __forceinline__ void adj_faces_body(const T* __restrict__ P, const double* __restrict__ kxyz,
                                               const double* __restrict__ lv, T* __restrict__ lamP,
                                               const ADims& d, const Phys& ph, int a, int bx) {
  const int N = d.ni * d.nj * d.nk;
  if (bx * (int)blockDim.x >= N) return;  // whole block past the end (uniform)
  const int c = bx * blockDim.x + threadIdx.x;
  const int n_a = a == 0 ? d.ni : (a == 1 ? d.nj : d.nk);
  const int sa = a == 0 ? d.nj * d.nk : (a == 1 ? d.nk : 1);
  if (threadIdx.x == 0) {
    // L2 fills of the ranges this CTA reaches first: lam/vol and the metric
    // row one cell ahead along a, the primitives two ahead
    const int c0 = bx * blockDim.x, n = min((int)blockDim.x, N - c0);
    const int a1 = c0 + sa, m1 = min(n, N - a1), a2 = c0 + 2 * sa, m2 = min(n, N - a2);
    if (m1 > 0) {
      for (int v = 0; v < 5; ++v) l2_prefetch(lv + (size_t)v * N + a1, m1 * 8);
      for (int m = 0; m < 3; ++m) l2_prefetch(kxyz + (size_t)(3 * a + m) * N + a1, m1 * 8);
    }
    if (m2 > 0)
      if constexpr (sizeof(T) == 4)
        l2_prefetch(P + (size_t)a2 * 8, m2 * 32);
      else
        for (int v = 0; v < 5; ++v) l2_prefetch(P + (size_t)v * N + a2, m2 * (int)sizeof(T));
  }
  T lc[4][5];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int f = 0; f < 5; ++f) lc[s][f] = T(0);
  if (c < N) {
    const int ia = a == 0 ? c / (d.nj * d.nk) : (a == 1 ? (c / d.nk) % d.nj : c % d.nk);
    if (ia >= 1 && ia <= n_a - 3) {
      const bool inL = ia >= 2, inR = ia + 1 <= n_a - 3;
      const int cr = c + sa;
      T lF[5];
      bool any = false;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double x = (inL ? -lv[v * N + c] : 0.0) + (inR ? lv[v * N + cr] : 0.0);
        lF[v] = (T)x;
        any |= x != 0.0;
      }
      if (any) face_vjp_cells<T>(P, kxyz + (size_t)(3 * a) * N, N, c, sa, lF, ph, lc);
    }
  }
  if (a != 2) {
    if (c < N)
#pragma unroll
      for (int s = 0; s < 4; ++s) add_cell<T>(lamP, N, c + (s - 1) * sa, lc[s]);
    return;
  }
  const int lane = threadIdx.x & 31;
  T own[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const T from_right = __shfl_down_sync(0xffffffffu, lc[0][f], 1);  // lane x+1's face, cell x
    const T from_left = __shfl_up_sync(0xffffffffu, lc[2][f], 1);     // lane x-1's face, cell x
    const T from_left2 = __shfl_up_sync(0xffffffffu, lc[3][f], 2);    // lane x-2's face, cell x
    own[f] = lc[1][f] + (lane < 31 ? from_right : T(0)) + (lane >= 1 ? from_left : T(0)) +
             (lane >= 2 ? from_left2 : T(0));
  }
  if (c < N) add_cell<T>(lamP, N, c, own);
  if (lane == 0) add_cell<T>(lamP, N, c - 1, lc[0]);  // nonzero only for a valid face, so c >= 1
  if (lane == 31) add_cell<T>(lamP, N, c + 1, lc[2]);
  if (lane >= 30) add_cell<T>(lamP, N, c + 2, lc[3]);
}

template <typename T, int NT, int MB>
__global__ void __launch_bounds__(NT, MB) k_adj_faces(const T* __restrict__ P, const double* __restrict__ kxyz,
                                                      const double* __restrict__ lv, T* __restrict__ lamP, ADims d,
                                                      Phys ph) {
  adj_faces_body<T>(P, kxyz, lv, lamP, d, ph, blockIdx.y, blockIdx.x);
}

// lamD: 12 x N (s-major: u, v, w, T; l = 0..2), lamL: 4 x N (local u, v, w, T).
// If dmu is set, also *dmu += mu_scale * sum_y lamG(y) . G(y): the viscous RHS
// is L_vis = D G with G linear in mu0, so lam . dL_vis/dmu0 = (D^T lam) . G / mu0.
template <typename T>
__device__ __forceinline__ double adj_visc_cell(const T* __restrict__ P, const double* __restrict__ kxyz,
                                                const double* __restrict__ lam, T* __restrict__ lamD,
                                                T* __restrict__ lamL, const ADims& d, const Phys& ph, int y,
                                                bool want_dot) {
  using M = FastMath<T>;
  const int N = d.ni * d.nj * d.nk;
  int i, j, k;
  dec(y, d, i, j, k);
  int nb[6];
  wrapped(y, i, j, k, d, nb);
  // ---- lamG(y): reverse of rhs_vis(c) = sum_jj sum_l 0.5 k[l][jj](c) (G(c+e_l) - G(c-e_l))
  double lG[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int l = 0; l < 3; ++l) {
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      // side 0: c = y - e_l (y is its + neighbour, weight +0.5); side 1: c = y + e_l (-0.5)
      const int c = side == 0 ? nb[2 * l + 1] : nb[2 * l];
      const double wgt = side == 0 ? 0.5 : -0.5;
      const double k0 = kxyz[(3 * l + 0) * N + c], k1 = kxyz[(3 * l + 1) * N + c],
                   k2 = kxyz[(3 * l + 2) * N + c];
      const double L1 = lam[N + c], L2 = lam[2 * N + c], L3 = lam[3 * N + c], L4 = lam[4 * N + c];
      // comp(e, jj): tau_00 tau_01 tau_02 tau_11 tau_12 tau_22 Ge_0 Ge_1 Ge_2
      lG[0] += wgt * (k0 * L1);
      lG[1] += wgt * (k1 * L1 + k0 * L2);
      lG[2] += wgt * (k2 * L1 + k0 * L3);
      lG[3] += wgt * (k1 * L2);
      lG[4] += wgt * (k2 * L2 + k1 * L3);
      lG[5] += wgt * (k2 * L3);
      lG[6] += wgt * (k0 * L4);
      lG[7] += wgt * (k1 * L4);
      lG[8] += wgt * (k2 * L4);
    }
  }
  // ---- forward of the viscous fluxes at y (rhs/viscous.py:36-105)
  const int fld[4] = {1, 2, 3, 5};
  T dd[4][3];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    T xp[6], xm[6];
    load_prims<T>(P, N, nb[2 * l], xp);
    load_prims<T>(P, N, nb[2 * l + 1], xm);
#pragma unroll
    for (int s = 0; s < 4; ++s) dd[s][l] = T(0.5) * (xp[fld[s]] - xm[fld[s]]);
  }
  T kk[9];
#pragma unroll
  for (int lm = 0; lm < 9; ++lm) kk[lm] = (T)kxyz[lm * N + y];
  T g[4][3];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int m = 0; m < 3; ++m) g[s][m] = dd[s][0] * kk[m] + dd[s][1] * kk[3 + m] + dd[s][2] * kk[6 + m];
  T xy[6];
  load_prims<T>(P, N, y, xy);
  const T u = xy[1], v = xy[2], w = xy[3], Tt = xy[5];
  T mu = (T)ph.mu0, dmu_dT = T(0);
  if (ph.visc_law == 0) {
    const T r = Tt * (T)ph.inv_T0;
    mu = (T)ph.mu0 * (r * M::sqrt_pos(r)) * (T)ph.sfac * M::rcp(Tt + (T)ph.Ts);
    dmu_dT = mu * (T(1.5) * M::rcp(Tt) - M::rcp(Tt + (T)ph.Ts));
  }
  const T kap = (T)ph.kap_fac;
  const T kappa = kap * mu;
  const T third = (T)(1.0 / 3.0);
  const T div_u = g[0][0] + g[1][1] + g[2][2];
  const T t00 = T(2) * mu * (g[0][0] - div_u * third), t11 = T(2) * mu * (g[1][1] - div_u * third),
          t22 = T(2) * mu * (g[2][2] - div_u * third);
  const T t01 = mu * (g[0][1] + g[1][0]), t02 = mu * (g[0][2] + g[2][0]), t12 = mu * (g[1][2] + g[2][1]);
  double dot = 0.0;
  if (want_dot) {
    const T ge0 = u * t00 + v * t01 + w * t02 + kappa * g[3][0];
    const T ge1 = u * t01 + v * t11 + w * t12 + kappa * g[3][1];
    const T ge2 = u * t02 + v * t12 + w * t22 + kappa * g[3][2];
    dot = lG[0] * t00 + lG[1] * t01 + lG[2] * t02 + lG[3] * t11 + lG[4] * t12 + lG[5] * t22 + lG[6] * ge0 +
          lG[7] * ge1 + lG[8] * ge2;
  }
  // ---- reverse
  const T lGe0 = (T)lG[6], lGe1 = (T)lG[7], lGe2 = (T)lG[8];
  T lt00 = (T)lG[0] + lGe0 * u, lt01 = (T)lG[1] + lGe0 * v + lGe1 * u, lt02 = (T)lG[2] + lGe0 * w + lGe2 * u;
  T lt11 = (T)lG[3] + lGe1 * v, lt12 = (T)lG[4] + lGe1 * w + lGe2 * v, lt22 = (T)lG[5] + lGe2 * w;
  const T lu = lGe0 * t00 + lGe1 * t01 + lGe2 * t02;
  const T lv = lGe0 * t01 + lGe1 * t11 + lGe2 * t12;
  const T lw = lGe0 * t02 + lGe1 * t12 + lGe2 * t22;
  T lkappa = lGe0 * g[3][0] + lGe1 * g[3][1] + lGe2 * g[3][2];
  T lg[4][3];
  lg[3][0] = lGe0 * kappa;
  lg[3][1] = lGe1 * kappa;
  lg[3][2] = lGe2 * kappa;
  T lmu = lt00 * T(2) * (g[0][0] - div_u * third) + lt11 * T(2) * (g[1][1] - div_u * third) +
          lt22 * T(2) * (g[2][2] - div_u * third) + lt01 * (g[0][1] + g[1][0]) +
          lt02 * (g[0][2] + g[2][0]) + lt12 * (g[1][2] + g[2][1]) + kap * lkappa;
  const T ldiv = -(lt00 + lt11 + lt22) * T(2) * mu * third;
  lg[0][0] = lt00 * T(2) * mu + ldiv;
  lg[1][1] = lt11 * T(2) * mu + ldiv;
  lg[2][2] = lt22 * T(2) * mu + ldiv;
  lg[0][1] = lt01 * mu;
  lg[1][0] = lt01 * mu;
  lg[0][2] = lt02 * mu;
  lg[2][0] = lt02 * mu;
  lg[1][2] = lt12 * mu;
  lg[2][1] = lt12 * mu;
  const T lT = lmu * dmu_dT;
  // g[s][m] = sum_l d[s][l] k[l][m]  ->  lamD[s][l] = sum_m lg[s][m] k[l][m]
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int l = 0; l < 3; ++l)
      lamD[(s * 3 + l) * N + y] = lg[s][0] * kk[3 * l] + lg[s][1] * kk[3 * l + 1] + lg[s][2] * kk[3 * l + 2];
  lamL[y] = lu;
  lamL[N + y] = lv;
  lamL[2 * N + y] = lw;
  lamL[3 * N + y] = lT;
  return dot;
}

// bx = the block of cells this CTA takes (blockDim.x a multiple of 32)
template <typename T>
__device__ __forceinline__ void adj_visc_body(const T* __restrict__ P, const double* __restrict__ kxyz,
                                              const double* __restrict__ lam, T* __restrict__ lamD,
                                              T* __restrict__ lamL, const ADims& d, const Phys& ph,
                                              double* __restrict__ dmu, double mu_scale, int bx) {
  const int N = d.ni * d.nj * d.nk;
  const int y = bx * blockDim.x + threadIdx.x;
  if (threadIdx.x == 0) {
    // L2 fills one i-plane ahead (nearer neighbours were fetched by earlier CTAs)
    const int a1 = bx * blockDim.x + d.nj * d.nk, m1 = min((int)blockDim.x, N - a1);
    if (m1 > 0) {
      for (int v = 1; v < 5; ++v) l2_prefetch(lam + (size_t)v * N + a1, m1 * 8);
      for (int lm = 0; lm < 9; ++lm) l2_prefetch(kxyz + (size_t)lm * N + a1, m1 * 8);
      if constexpr (sizeof(T) == 4) {
        l2_prefetch(P + (size_t)a1 * 8, m1 * 32);
      } else {
        const int fld[4] = {1, 2, 3, 5};
        for (int s = 0; s < 4; ++s) l2_prefetch(P + (size_t)fld[s] * N + a1, m1 * (int)sizeof(T));
      }
    }
  }
  double dot = 0.0;
  if (y < N) dot = adj_visc_cell<T>(P, kxyz, lam, lamD, lamL, d, ph, y, dmu != nullptr);
  if (dmu) {  // warp reduction (all lanes take part), one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
    if ((threadIdx.x & 31) == 0 && dot != 0.0) atomicAdd(dmu, mu_scale * dot);
  }
}

template <typename T, int MB = 1>
__global__ void __launch_bounds__(kAT, MB) k_adj_visc(const T* __restrict__ P, const double* __restrict__ kxyz,
                                                     const double* __restrict__ lam, T* __restrict__ lamD,
                                                     T* __restrict__ lamL, ADims d, Phys ph,
                                                     double* __restrict__ dmu, double mu_scale) {
  adj_visc_body<T>(P, kxyz, lam, lamD, lamL, d, ph, dmu, mu_scale, blockIdx.x);
}

// The face VJPs of the three axes and the viscous VJP in one launch of NT-
// thread CTAs: CTA b takes task b % 4 (face axis 0, 1, 2, or the viscous VJP)
// over block b / 4 of cells, so every residency wave mixes the issue-bound
// face work with the load-bound viscous work on the same SMs and reads the
// same primitive, metric and adjoint ranges for all four tasks.  The tasks
// write disjoint arrays (lamP by atomics; lamD, lamL), so their order does not
// matter.
template <typename T, int NT, int MB>
__global__ void __launch_bounds__(NT, MB)
    k_adj_faces_visc(const T* __restrict__ P, const double* __restrict__ kxyz, const double* __restrict__ lv,
                     T* __restrict__ lamP, const double* __restrict__ lam, T* __restrict__ lamD,
                     T* __restrict__ lamL, ADims d, Phys ph, double* __restrict__ dmu, double mu_scale) {
  const int task = blockIdx.x & 3, bx = blockIdx.x >> 2;
  if (task < 3)
    adj_faces_body<T>(P, kxyz, lv, lamP, d, ph, task, bx);
  else
    adj_visc_body<T>(P, kxyz, lam, lamD, lamL, d, ph, dmu, mu_scale, bx);
}

template <typename T>
__global__ void k_adj_final(const double* __restrict__ q, T* lamP, const T* __restrict__ lamD,
                            const T* __restrict__ lamL, double* __restrict__ out, T* __restrict__ P,
                            double* __restrict__ lam_vol, ADims d, Phys ph, int flags, VjpEpilogue e) {
  const int N = d.ni * d.nj * d.nk;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= N) return;
  if (threadIdx.x == 0) {
    // L2 fills of this CTA's own ranges, and of lamD one i-plane ahead
    const int c0 = x, n = min((int)blockDim.x, N - c0);
    const int a1 = c0 + d.nj * d.nk, m1 = min(n, N - a1);
    for (int f = 0; f < 5; ++f) l2_prefetch(q + (size_t)f * N + c0, n * 8);
    if (flags & kRhsInvscd)
      for (int f = 0; f < 5; ++f) l2_prefetch(lamP + (size_t)f * N + c0, n * (int)sizeof(T));
    if (flags & kRhsViscous) {
      for (int s = 0; s < 4; ++s) l2_prefetch(lamL + (size_t)s * N + c0, n * (int)sizeof(T));
      if (m1 > 0)
        for (int f = 0; f < 12; ++f) l2_prefetch(lamD + (size_t)f * N + a1, m1 * (int)sizeof(T));
    }
    const double* ep[6] = {e.x1, e.y1, e.z1, e.x2, e.y2, e.next_q};
    for (int t = 0; t < 6; ++t)
      if ((t < 3 || t == 5 ? e.o1 : e.o2) && ep[t])
        for (int f = 0; f < 5; ++f) l2_prefetch(ep[t] + (size_t)f * N + c0, n * 8);
    if (e.o1 && e.next_q && (flags & kRhsInvscd)) l2_prefetch(e.next_vol + c0, n * 8);
  }
  double lr = 0, lu = 0, lv = 0, lw = 0, lp = 0, lT = 0;
  if (flags & kRhsInvscd) {
    lr = lamP[x];
    lu = lamP[N + x];
    lv = lamP[2 * N + x];
    lw = lamP[3 * N + x];
    lp = lamP[4 * N + x];
  }
  if (flags & kRhsViscous) {
    int i, j, k;
    dec(x, d, i, j, k);
    int nb[6];
    wrapped(x, i, j, k, d, nb);
    double ls[4] = {(double)lamL[x], (double)lamL[N + x], (double)lamL[2 * N + x], (double)lamL[3 * N + x]};
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int l = 0; l < 3; ++l)
        ls[s] += 0.5 * ((double)lamD[(s * 3 + l) * N + nb[2 * l + 1]] - (double)lamD[(s * 3 + l) * N + nb[2 * l]]);
    lu += ls[0];
    lv += ls[1];
    lw += ls[2];
    lT = ls[3];
  }
  // reverse of T = p / max(rho R, 1e-300) and of cons_to_prim
  const double r = q[x], ir = 1.0 / r;
  const double u = q[N + x] * ir, v = q[2 * N + x] * ir, w = q[3 * N + x] * ir;
  const double ke = 0.5 * (u * u + v * v + w * w);
  const double p = ph.gm1 * (q[4 * N + x] - r * ke);
  if (r * ph.R > 1e-300) {
    lp += lT * ir / ph.R;
    lr -= lT * p * ir * ir / ph.R;
  } else {
    lp += lT * 1e300;
  }
  // p = gm1 (q4 - rho ke); ke = 0.5 |u|^2; u = q1 / rho
  const double lq4 = ph.gm1 * lp;
  lr -= ph.gm1 * lp * ke;
  const double lke = -ph.gm1 * lp * r;
  lu += lke * u;
  lv += lke * v;
  lw += lke * w;
  const double V[5] = {lr - (lu * u + lv * v + lw * w) * ir, lu * ir, lv * ir, lw * ir, lq4};
  if (!e.o1) {
#pragma unroll
    for (int f = 0; f < 5; ++f) out[f * N + x] = V[f];
    return;
  }
  double o1[5], o2[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const int t = f * N + x;
    o1[f] = e.a1 * e.x1[t] + e.e1 * V[f];
    if (e.y1) o1[f] += e.b1 * e.y1[t];
    if (e.z1) o1[f] += e.c1 * e.z1[t];
    if (e.o2) {
      o2[f] = e.a2 * e.x2[t];
      if (e.y2) o2[f] += e.b2 * e.y2[t];
    }
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    e.o1[f * N + x] = o1[f];
    if (e.o2) e.o2[f * N + x] = o2[f];
  }
  if (e.next_q) {
    // what the next RHS VJP of this block reads first (its k_adj_prims
    // launch is skipped); this cell's lamP was read above, by this thread only
    write_prims<T>(e.next_q, P, N, x, ph.gm1, ph.R);
    if (flags & kRhsInvscd) {
      const double iv = 1.0 / (e.next_vol[x] + 1e-300);
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        lam_vol[f * N + x] = o1[f] * iv;
        lamP[f * N + x] = T(0);
      }
    }
  }
}

// dJ/dq of J = sum_interior vol * 0.5 |m|^2 / rho
__global__ void k_ke_grad(const double* __restrict__ q, const double* __restrict__ vol,
                          double* __restrict__ grad, int ni, int nj, int nk, int g) {
  const int N = ni * nj * nk;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int k = c % nk, j = (c / nk) % nj, i = c / (nk * nj);
  const bool in = i >= g && i < ni - g && j >= g && j < nj - g && k >= g && k < nk - g;
  if (!in) {
#pragma unroll
    for (int v = 0; v < 5; ++v) grad[v * N + c] = 0.0;
    return;
  }
  const double r = q[c], m1 = q[N + c], m2 = q[2 * N + c], m3 = q[3 * N + c], V = vol[c];
  const double ir = 1.0 / r;
  grad[c] = -V * 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) * ir * ir;
  grad[N + c] = V * m1 * ir;
  grad[2 * N + c] = V * m2 * ir;
  grad[3 * N + c] = V * m3 * ir;
  grad[4 * N + c] = 0.0;
}

template <typename T>
size_t vjp_ws(int64_t N) {
  return ((kPVals<T> + 5 + 12 + 4) * (size_t)N) * sizeof(T) + 5 * (size_t)N * sizeof(double) + 5 * 256;
}

template <typename T>
int rhs_vjp_impl(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
                 const double* lam, double* out, int ni, int nj, int nk, const Phys& ph, int flags,
                 void* ws, cudaStream_t st, double* dmu, double mu_scale, const VjpEpilogue* epi) {
  const int N = ni * nj * nk;
  auto al = [](char* p) { return (char*)(((uintptr_t)p + 255) & ~(uintptr_t)255); };
  char* p = al((char*)ws);
  T* P = (T*)p;
  p = al(p + kPVals<T> * (size_t)N * sizeof(T));
  T* lamP = (T*)p;
  p = al(p + 5 * (size_t)N * sizeof(T));
  T* lamD = (T*)p;
  p = al(p + 12 * (size_t)N * sizeof(T));
  T* lamL = (T*)p;
  p = al(p + 4 * (size_t)N * sizeof(T));
  double* lv = (double*)p;
  const ADims d{ni, nj, nk};
  const int grid = grid_for(N, kAT);
  const bool inv = (flags & kRhsInvscd) != 0;
  if (!(epi && epi->ws_ready)) {
    k_adj_prims<T><<<grid, kAT, 0, st>>>(q, P, N, ph.gm1, ph.R, lam, vol, inv ? lv : nullptr, inv ? lamP : nullptr);
    ctx->launches += 1;
  }
  int rest = flags;  // the parts still to launch
  if constexpr (sizeof(T) == 4) {
    if (ctx->adj_variant == 0 && (flags & kRhsInvscd) && (flags & kRhsViscous)) {
      // FP32 default: both VJPs in one launch (80 registers, 3 CTAs of 256 per
      // SM).  FP64 keeps two launches: its face VJP is bound by the FP64 pipe at
      // the 128-register cap, and the fused form (128 x 4) measured 4 % slower
      // on the reverse sweep
      k_adj_faces_visc<T, kAT, 3><<<4 * (unsigned)grid, kAT, 0, st>>>(P, kxyz, lv, lamP, lam, lamD, lamL, d, ph,
                                                                     dmu, mu_scale);
      ctx->launches += 1;
      rest &= ~(kRhsInvscd | kRhsViscous);
    }
  }
  if (rest & kRhsInvscd) {
    // register caps (threads per CTA, minimum CTAs per SM): the FP64 face VJP
    // needs ~180 registers uncapped.  Variant 0 is the fastest measured on
    // B200 (TGV 96^3 adjoint sweep): FP64 128 x 4 (128 registers), FP32
    // 256 x 3 (80 registers, a few spilled values)
    auto launch = [&](auto kern, int nt) {
      kern<<<dim3((unsigned)((N + nt - 1) / nt), 3), nt, 0, st>>>(P, kxyz, lv, lamP, d, ph);
    };
    constexpr bool f64 = sizeof(T) == 8;
    switch (ctx->adj_variant) {
      case 1: launch(k_adj_faces<T, 256, 1>, 256); break;
      case 2:
      case 4:
        if (f64) launch(k_adj_faces<T, 128, 3>, 128);
        else launch(k_adj_faces<T, 256, 2>, 256);
        break;
      default:
        if (f64) launch(k_adj_faces<T, 128, 4>, 128);
        else launch(k_adj_faces<T, 256, 3>, 256);
    }
    ctx->launches += 1;
  }
  if (rest & kRhsViscous) {
    // variants 0 and 2 cap the viscous VJP at 64 registers (4 CTAs per SM)
    if (ctx->adj_variant == 0 || ctx->adj_variant == 2)
      k_adj_visc<T, 4><<<grid, kAT, 0, st>>>(P, kxyz, lam, lamD, lamL, d, ph, dmu, mu_scale);
    else
      k_adj_visc<T><<<grid, kAT, 0, st>>>(P, kxyz, lam, lamD, lamL, d, ph, dmu, mu_scale);
    ctx->launches += 1;
  }
  k_adj_final<T><<<grid, kAT, 0, st>>>(q, lamP, lamD, lamL, out, P, lv, d, ph, flags, epi ? *epi : VjpEpilogue{});
  ctx->launches += 1;
  return launch_status(ctx, "rhs vjp launch");
}

}  // namespace

size_t rhs_vjp_ws_bytes(int precision, int ni, int nj, int nk) {
  const int64_t N = (int64_t)ni * nj * nk;
  return precision == FJ_PREC_F32FLUX ? vjp_ws<float>(N) : vjp_ws<double>(N);
}

int rhs_vjp(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol, const double* lam,
            double* out, int ni, int nj, int nk, const fj_params* p, int flags, void* ws,
            cudaStream_t st, double* dmu, double mu_scale, const VjpEpilogue* epi) {
  const Phys ph = make_phys(p);
  if (p->precision == FJ_PREC_F32FLUX)
    return rhs_vjp_impl<float>(ctx, q, kxyz, vol, lam, out, ni, nj, nk, ph, flags, ws, st, dmu, mu_scale, epi);
  return rhs_vjp_impl<double>(ctx, q, kxyz, vol, lam, out, ni, nj, nk, ph, flags, ws, st, dmu, mu_scale, epi);
}

int ke_grad(fj_ctx* ctx, const double* q, const double* vol, double* grad, int ni, int nj, int nk, int g,
            cudaStream_t st) {
  k_ke_grad<<<grid_for((int64_t)ni * nj * nk), kThreads, 0, st>>>(q, vol, grad, ni, nj, nk, g);
  ctx->launches += 1;
  return launch_status(ctx, "ke grad launch");
}

}  // namespace fj
