// fj_stage_split.cu -- one TVD-RK3 stage (or one RHS) of MANY blocks in three
// barrier-free, high-occupancy kernels, each launched once for all blocks:
//
//   k_split_prims    q -> primitives (rho, u, v, w, p, T) per padded cell
//                    (physics/eos.py:12-17; T = p / max(rho R, 1e-300),
//                    rhs/viscous.py:36)
//   k_split_fluxes   per cell c: the viscous flux components G(c)
//                    (rhs/viscous.py:36-105, neighbours wrap around the padded
//                    block like jnp.roll) and the three Roe faces c | c+e_a
//                    (rhs/invscd.py:53-100) for c_a in [1, n_a-3]
//   k_split_assemble per cell: -(F_a(c) - F_a(c-e_a)) / (vol + 1e-300) over
//                    the axes where c_a in [2, n_a-3] (rhs/invscd.py:119-131),
//                    the viscous divergence of G with the cell's own kxyz
//                    (rhs/viscous.py:86-117) and the TVD-RK3 combine
//                    (solver/step.py:45-53)
//
// Intermediates live in scratch in the flux type T (float on the FP32-flux
// path, double on the FP64 path) as per-cell RECORDS, so that a cell's fields
// sit at compile-time offsets from one address and move with 16-byte vector
// loads and stores:
//   P  8 T per cell: rho u v w p T (2 pad)
//   F 16 T per cell: the faces c | c+e_i, c | c+e_j, c | c+e_k, 5 T each (1 pad)
//   G 12 T per cell: tau_00 tau_01 tau_02 tau_11 tau_12 tau_22, the energy
//     flux components 0..2 (3 pad)
// A plan also keeps the metrics as records (kRecK<T> T per cell: the nine
// kxyz[l][m], l-major, then pad), converted once from the caller's FP64
// field-major kxyz; without one the kernels read kxyz field by field.
// Each launch covers every block of a table; a CTA handles 256 consecutive
// cells of one block, and neighbours are read through L1/L2.
#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_rhs.cuh"
#include "fj_split.cuh"

#include "fj_split_dev.cuh"

namespace fj {

namespace {

using namespace sd;

// NW: warps per CTA.  8 normally; 2 for tables too small to give every SM two
// 256-thread CTAs (the 32^3 block: 183 CTAs of 256 would leave a fifth of the
// SMs with twice the work), whose flux and assembly work runs in
// k_split_fluxes_roles and k_split_assemble_kmem over the same 64-cell ranges.
template <typename T, int NW = 8>
__global__ void __launch_bounds__(32 * NW) k_split_prims(const Table tab, const double gm1, const double R,
                                                         const double iR, const double p_ref) {
  const int b = find_block(tab, blockIdx.x);
  if (threadIdx.x == 0) prefetch_state(tab.b[b], blockIdx.x, 32 * NW);
  grid_dep_wait();
  const SplitBlock& B = tab.b[b].blk;
  const int32_t c = (blockIdx.x - B.cta_begin) * (32 * NW) + threadIdx.x;
  if (c >= B.ni * B.nj * B.nk) return;
  prims_cell<T>(B, c, gm1, R, iR, p_ref);
}

template <typename T, bool K_AOS, int OCC = SplitOcc<T>::fluxes>
__global__ void __launch_bounds__(kSplitThreads, OCC) k_split_fluxes(const Table tab, const Phys ph,
                                                                     const int flags) {
  const int b = find_block(tab, blockIdx.x);
  if (threadIdx.x == 0) prefetch_fluxes<T, K_AOS, false>(tab.b[b], blockIdx.x);
  grid_dep_wait();
  Cell x;
  if (!decode(tab.b[b], blockIdx.x, x)) return;
  flux_cell<T, K_AOS, true>(tab.b[b].blk, tab.b[b].blk.prim, x, ph, flags);
}

// The flux work of small FP32 tables split by warp roles: a CTA of 256 threads
// takes the 64 cells of one 2-warp flux CTA; warps 0-1 evaluate their cells'
// i faces, warps 2-3 the j faces, warps 4-5 the viscous components and warps
// 6-7 the k faces (into Fk, which k_split_assemble_kmem reads instead of
// evaluating them).  Each thread's dependency chain is about a third of
// k_split_fluxes' (a small table leaves most of the GPU's warp slots free,
// and its kernels' times are set by those chains).
template <typename T, bool K_AOS>
__global__ void __launch_bounds__(256, 4) k_split_fluxes_roles(const Table tab, const Phys ph, const int flags) {
  const int b = find_block(tab, blockIdx.x);
  if (threadIdx.x == 0) prefetch_fluxes<T, K_AOS, false>(tab.b[b], blockIdx.x, 64);
  grid_dep_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const SplitBlock& B = tab.b[b].blk;
  Cell x;
  if (!decode_cell(tab.b[b], (int64_t)(blockIdx.x - B.cta_begin) * 64 + (warp & 1) * 32 + lane, x)) return;
  if (warp < 2) {
    if (flags & kRhsInvscd) flux_face_part<T, K_AOS, 0>(B, B.prim, x, ph);
  } else if (warp < 4) {
    if (flags & kRhsInvscd) flux_face_part<T, K_AOS, 1>(B, B.prim, x, ph);
  } else if (warp < 6) {
    if (flags & kRhsViscous) flux_visc_part<T, K_AOS>(B, B.prim, x, ph);
  } else if (flags & kRhsInvscd) {
    flux_face_part<T, K_AOS, 2>(B, B.prim, x, ph);
  }
}

// The assembly of small FP32 tables: asm_chunk with the k faces read from Fk
// (2-warp CTAs of 62 cells; a small table puts about five of them on an SM,
// so the register cap is loose).
template <typename T, bool K_AOS>
__global__ void __launch_bounds__(64, 8) k_split_assemble_kmem(const Table tab, const int flags, const int stage,
                                                                 const int next_prims, const double gm1,
                                                                 const double R, const double iR, const Phys ph) {
  const int b = find_block_asm(tab, blockIdx.x);
  const Dev& d = tab.b[b];
  const SplitBlock& B = d.blk;
  if (threadIdx.x == 0) prefetch_assembly<T, K_AOS, false>(d, blockIdx.x, flags, stage, 62, B.cta_begin_asm);
  grid_dep_wait();
  asm_chunk_kmem<T, K_AOS>(d, TablePtrs{B}, (int64_t)(blockIdx.x - B.cta_begin_asm) * 62, flags, stage, next_prims,
                           gm1, R, iR, ph);
}

template <typename T, bool K_AOS, int OCC = SplitOcc<T>::assemble>
__global__ void __launch_bounds__(kSplitThreads, OCC) k_split_assemble(const Table tab, const int flags,
                                                                       const int stage, const int next_prims,
                                                                       const double gm1, const double R,
                                                                       const double iR, const Phys ph) {
  const int b = find_block_asm(tab, blockIdx.x);
  const Dev& d = tab.b[b];
  const SplitBlock& B = d.blk;
  if (threadIdx.x == 0) prefetch_assembly<T, K_AOS, false>(d, blockIdx.x, flags, stage, kAsmCells, B.cta_begin_asm);
  grid_dep_wait();
  asm_chunk<T, K_AOS, true>(d, TablePtrs{B}, (int64_t)(blockIdx.x - B.cta_begin_asm) * kAsmCells, flags, stage,
                            next_prims, gm1, R, iR, ph);
}

// ---- field-major variant (the FP64 path) ----------------------------------
// The FP64 path keeps its primitives as 48-byte records (three 16-byte loads
// per neighbour) and its face and viscous fluxes field-major (10 + 9 arrays of
// N): flux records would cost FP64 more registers (two doubles per vector
// lane) and padding bytes than the index arithmetic they save.
namespace fm {

template <typename T, int NW = 8>
__global__ void __launch_bounds__(32 * NW) k_fm_prims(const Table tab, const double gm1,
                                                              const double R, const double iR) {
  const int b = find_block(tab, blockIdx.x);
  if (threadIdx.x == 0) prefetch_state(tab.b[b], blockIdx.x, 32 * NW);
  grid_dep_wait();
  const SplitBlock& B = tab.b[b].blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c = (int64_t)(blockIdx.x - B.cta_begin) * (32 * NW) + threadIdx.x;
  if (c >= N) return;
  const double* q = B.q;
  const double r = q[c];
  const double ir = __drcp_rn(r);
  const double u = q[N + c] * ir, v = q[2 * N + c] * ir, w = q[3 * N + c] * ir;
  const double p = gm1 * (q[4 * N + c] - r * (0.5 * (u * u + v * v + w * w)));
  const double Tt = r * R > 1e-300 ? p * ir * iR : p * 1e300;
  const T rec[kRecP64] = {(T)r, (T)u, (T)v, (T)w, (T)p, (T)Tt};
  st_rec<T, kRecP64>((T*)B.prim + c * kRecP64, rec);
}

template <typename T>
__device__ __forceinline__ T metric(const SplitBlock& B, int64_t N, int lm, int64_t c) {
  return (T)__ldg(B.kxyz + lm * N + c);
}

// Primitives (rho, u, v, w, p[, T]) of one cell from the field-major scratch.
template <typename T>
struct Cell6 {
  T r, u, v, w, p, t;
};

template <typename T, bool WITH_T>
__device__ __forceinline__ Cell6<T> load_cell(const T* __restrict__ P, int32_t N, int32_t c) {
  (void)N;
  T x[kRecP64];
  ld_rec<T, kRecP64>(P + (size_t)c * kRecP64, x);
  return Cell6<T>{x[0], x[1], x[2], x[3], x[4], WITH_T ? x[5] : T(0)};
}

// Roe face c | c+e_a from the primitives of c-e_a, c, c+e_a, c+2e_a and the
// kxyz rows of c and c+e_a (rhs/invscd.py:62-100).
template <typename T>
__device__ __forceinline__ void face_from_cells(const Cell6<T>& a0, const Cell6<T>& a1, const Cell6<T>& a2,
                                                const Cell6<T>& a3, const T kl[3], const T kr[3],
                                                const Phys& ph, T F[5]) {
  Prim<T> cell[4] = {{a0.r, a0.u, a0.v, a0.w, a0.p}, {a1.r, a1.u, a1.v, a1.w, a1.p},
                     {a2.r, a2.u, a2.v, a2.w, a2.p}, {a3.r, a3.u, a3.v, a3.w, a3.p}};
  invscd_face_fast<T>(cell, kl[0], kl[1], kl[2], kr[0], kr[1], kr[2], (T)ph.gm1, (T)ph.inv_gm1,
                      (T)ph.eps_entropy, ph.limiter, F);
}

template <typename T>
__device__ __forceinline__ void metric_row(const SplitBlock& B, int32_t N, int row, int32_t c, T k[3]) {
  const double* K = B.kxyz + 3 * row * N;
  k[0] = (T)__ldg(K + c);
  k[1] = (T)__ldg(K + N + c);
  k[2] = (T)__ldg(K + 2 * N + c);
}

template <typename T, int OCC = 2>
__global__ void __launch_bounds__(kSplitThreads, OCC) k_fm_fluxes(const Table tab, const Phys ph,
                                                                 const int flags) {
  using M = FastMath<T>;
  const int b = find_block(tab, blockIdx.x);
  if (threadIdx.x == 0) prefetch_fluxes<T, false, true>(tab.b[b], blockIdx.x);
  grid_dep_wait();
  Cell x;
  if (!decode(tab.b[b], blockIdx.x, x)) return;
  const SplitBlock& B = tab.b[b].blk;
  // 32-bit offsets: 15 N < 2^31 is checked on the host
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int32_t si = x.nj * x.nk, sj = x.nk;
  const T* __restrict__ P = (const T*)B.prim;
  const bool vis = (flags & kRhsViscous) != 0, inv = (flags & kRhsInvscd) != 0;

  // neighbour offsets with the padded-array wrap (jnp.roll) for the viscous
  // stencil; faces exist only where no wrap is involved
  const int32_t ip = x.i + 1 == x.ni ? c - (x.ni - 1) * si : c + si;
  const int32_t im = x.i == 0 ? c + (x.ni - 1) * si : c - si;
  const int32_t jp = x.j + 1 == x.nj ? c - (x.nj - 1) * sj : c + sj;
  const int32_t jm = x.j == 0 ? c + (x.nj - 1) * sj : c - sj;
  const int32_t kp = x.k + 1 == x.nk ? c - (x.nk - 1) : c + 1;
  const int32_t km = x.k == 0 ? c + (x.nk - 1) : c - 1;

  const Cell6<T> C0 = load_cell<T, true>(P, N, c);
  const Cell6<T> Im = load_cell<T, true>(P, N, im), Ip = load_cell<T, true>(P, N, ip);
  const Cell6<T> Jm = load_cell<T, true>(P, N, jm), Jp = load_cell<T, true>(P, N, jp);
  const Cell6<T> Km = load_cell<T, true>(P, N, km), Kp = load_cell<T, true>(P, N, kp);

  if (vis) {
    // viscous flux components at c (rhs/viscous.py:36-105)
    const T h = T(0.5);
    const T d[4][3] = {{h * (Ip.u - Im.u), h * (Jp.u - Jm.u), h * (Kp.u - Km.u)},
                       {h * (Ip.v - Im.v), h * (Jp.v - Jm.v), h * (Kp.v - Km.v)},
                       {h * (Ip.w - Im.w), h * (Jp.w - Jm.w), h * (Kp.w - Km.w)},
                       {h * (Ip.t - Im.t), h * (Jp.t - Jm.t), h * (Kp.t - Km.t)}};
    T kk[9];
    metric_row<T>(B, N, 0, c, kk);
    metric_row<T>(B, N, 1, c, kk + 3);
    metric_row<T>(B, N, 2, c, kk + 6);
    T g[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[m] + d[s][1] * kk[3 + m] + d[s][2] * kk[6 + m];
    T mu = (T)B.mu0;
    if (ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
      const T r = C0.t * (T)ph.inv_T0;
      mu = (T)B.mu0 * (r * M::sqrt_pos(r)) * (T)ph.sfac * M::rcp(C0.t + (T)ph.Ts);
    }
    const T kappa = (T)ph.kap_fac * mu;
    const T third = (T)(1.0 / 3.0);
    const T div_u = g[0][0] + g[1][1] + g[2][2];
    const T t00 = T(2) * mu * (g[0][0] - div_u * third);
    const T t01 = mu * (g[0][1] + g[1][0]);
    const T t02 = mu * (g[0][2] + g[2][0]);
    const T t11 = T(2) * mu * (g[1][1] - div_u * third);
    const T t12 = mu * (g[1][2] + g[2][1]);
    const T t22 = T(2) * mu * (g[2][2] - div_u * third);
    T* __restrict__ G = (T*)B.G;
    G[c] = t00;
    G[N + c] = t01;
    G[2 * N + c] = t02;
    G[3 * N + c] = t11;
    G[4 * N + c] = t12;
    G[5 * N + c] = t22;
    G[6 * N + c] = C0.u * t00 + C0.v * t01 + C0.w * t02 + kappa * g[3][0];
    G[7 * N + c] = C0.u * t01 + C0.v * t11 + C0.w * t12 + kappa * g[3][1];
    G[8 * N + c] = C0.u * t02 + C0.v * t12 + C0.w * t22 + kappa * g[3][2];
  }
  if (inv) {
    // the three faces c | c+e_a with face index c_a - 1 in [0, n_a - 4]
    T* __restrict__ F = (T*)B.F;
    T kc[3], kn[3], Fo[5];
    if (x.i >= 1 && x.i <= x.ni - 3) {
      const Cell6<T> I2 = load_cell<T, false>(P, N, c + 2 * si);
      metric_row<T>(B, N, 0, c, kc);
      metric_row<T>(B, N, 0, c + si, kn);
      face_from_cells<T>(Im, C0, Ip, I2, kc, kn, ph, Fo);
#pragma unroll
      for (int v = 0; v < 5; ++v) F[v * N + c] = Fo[v];
    }
    if (x.j >= 1 && x.j <= x.nj - 3) {
      const Cell6<T> J2 = load_cell<T, false>(P, N, c + 2 * sj);
      metric_row<T>(B, N, 1, c, kc);
      metric_row<T>(B, N, 1, c + sj, kn);
      face_from_cells<T>(Jm, C0, Jp, J2, kc, kn, ph, Fo);
#pragma unroll
      for (int v = 0; v < 5; ++v) F[(5 + v) * N + c] = Fo[v];
    }
    // the k faces are evaluated in the assembly (this kernel is bound by the
    // FP64 pipe, the assembly by memory latency)
  }
}

// The FP64 flux work of small tables split by warp roles (192-thread CTAs over
// the 64 cells of one 2-warp CTA: warps 0-1 the i faces, 2-3 the j faces, 4-5
// the viscous components), the same arithmetic and stores as k_fm_fluxes.
template <typename T, int AXIS>
__device__ __forceinline__ void fm_face_role(const SplitBlock& B, const Cell& x, const Phys& ph) {
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int ia = AXIS == 0 ? x.i : x.j, na = AXIS == 0 ? x.ni : x.nj;
  if (ia < 1 || ia > na - 3) return;
  const int32_t sa = AXIS == 0 ? x.nj * x.nk : x.nk;
  const T* __restrict__ P = (const T*)B.prim;
  const Cell6<T> a0 = load_cell<T, false>(P, N, c - sa), a1 = load_cell<T, false>(P, N, c),
                 a2 = load_cell<T, false>(P, N, c + sa), a3 = load_cell<T, false>(P, N, c + 2 * sa);
  T kc[3], kn[3], Fo[5];
  metric_row<T>(B, N, AXIS, c, kc);
  metric_row<T>(B, N, AXIS, c + sa, kn);
  face_from_cells<T>(a0, a1, a2, a3, kc, kn, ph, Fo);
  T* __restrict__ F = (T*)B.F;
#pragma unroll
  for (int v = 0; v < 5; ++v) F[(5 * AXIS + v) * N + c] = Fo[v];
}

template <typename T>
__device__ __forceinline__ void fm_visc_role(const SplitBlock& B, const Cell& x, const Phys& ph) {
  using M = FastMath<T>;
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int32_t si = x.nj * x.nk, sj = x.nk;
  const T* __restrict__ P = (const T*)B.prim;
  const int32_t ip = x.i + 1 == x.ni ? c - (x.ni - 1) * si : c + si;
  const int32_t im = x.i == 0 ? c + (x.ni - 1) * si : c - si;
  const int32_t jp = x.j + 1 == x.nj ? c - (x.nj - 1) * sj : c + sj;
  const int32_t jm = x.j == 0 ? c + (x.nj - 1) * sj : c - sj;
  const int32_t kp = x.k + 1 == x.nk ? c - (x.nk - 1) : c + 1;
  const int32_t km = x.k == 0 ? c + (x.nk - 1) : c - 1;
  const Cell6<T> C0 = load_cell<T, true>(P, N, c);
  const Cell6<T> Im = load_cell<T, true>(P, N, im), Ip = load_cell<T, true>(P, N, ip);
  const Cell6<T> Jm = load_cell<T, true>(P, N, jm), Jp = load_cell<T, true>(P, N, jp);
  const Cell6<T> Km = load_cell<T, true>(P, N, km), Kp = load_cell<T, true>(P, N, kp);
  const T h = T(0.5);
  const T d[4][3] = {{h * (Ip.u - Im.u), h * (Jp.u - Jm.u), h * (Kp.u - Km.u)},
                     {h * (Ip.v - Im.v), h * (Jp.v - Jm.v), h * (Kp.v - Km.v)},
                     {h * (Ip.w - Im.w), h * (Jp.w - Jm.w), h * (Kp.w - Km.w)},
                     {h * (Ip.t - Im.t), h * (Jp.t - Jm.t), h * (Kp.t - Km.t)}};
  T kk[9];
  metric_row<T>(B, N, 0, c, kk);
  metric_row<T>(B, N, 1, c, kk + 3);
  metric_row<T>(B, N, 2, c, kk + 6);
  T g[4][3];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[m] + d[s][1] * kk[3 + m] + d[s][2] * kk[6 + m];
  T mu = (T)B.mu0;
  if (ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
    const T r = C0.t * (T)ph.inv_T0;
    mu = (T)B.mu0 * (r * M::sqrt_pos(r)) * (T)ph.sfac * M::rcp(C0.t + (T)ph.Ts);
  }
  const T kappa = (T)ph.kap_fac * mu;
  const T third = (T)(1.0 / 3.0);
  const T div_u = g[0][0] + g[1][1] + g[2][2];
  const T t00 = T(2) * mu * (g[0][0] - div_u * third);
  const T t01 = mu * (g[0][1] + g[1][0]);
  const T t02 = mu * (g[0][2] + g[2][0]);
  const T t11 = T(2) * mu * (g[1][1] - div_u * third);
  const T t12 = mu * (g[1][2] + g[2][1]);
  const T t22 = T(2) * mu * (g[2][2] - div_u * third);
  T* __restrict__ G = (T*)B.G;
  G[c] = t00;
  G[N + c] = t01;
  G[2 * N + c] = t02;
  G[3 * N + c] = t11;
  G[4 * N + c] = t12;
  G[5 * N + c] = t22;
  G[6 * N + c] = C0.u * t00 + C0.v * t01 + C0.w * t02 + kappa * g[3][0];
  G[7 * N + c] = C0.u * t01 + C0.v * t11 + C0.w * t12 + kappa * g[3][1];
  G[8 * N + c] = C0.u * t02 + C0.v * t12 + C0.w * t22 + kappa * g[3][2];
}

template <typename T>
__global__ void __launch_bounds__(192, 2) k_fm_fluxes_roles(const Table tab, const Phys ph, const int flags) {
  const int b = find_block(tab, blockIdx.x);
  if (threadIdx.x == 0) prefetch_fluxes<T, false, true>(tab.b[b], blockIdx.x, 64);
  grid_dep_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const SplitBlock& B = tab.b[b].blk;
  Cell x;
  if (!decode_cell(tab.b[b], (int64_t)(blockIdx.x - B.cta_begin) * 64 + (warp & 1) * 32 + lane, x)) return;
  if (warp < 2) {
    if (flags & kRhsInvscd) fm_face_role<T, 0>(B, x, ph);
  } else if (warp < 4) {
    if (flags & kRhsInvscd) fm_face_role<T, 1>(B, x, ph);
  } else if (flags & kRhsViscous) {
    fm_visc_role<T>(B, x, ph);
  }
}

// The k face c-1 | c (rhs/invscd.py:62-100) of the FP64 path from the
// primitive records of c-2 .. c+1 and the k rows of kxyz at c-1 and c.
template <typename T>
__device__ __forceinline__ void fm_k_face_left(const SplitBlock& B, int32_t N, int32_t c, const Phys& ph, T F[5]) {
  const T* __restrict__ P = (const T*)B.prim;
  const Cell6<T> a0 = load_cell<T, false>(P, N, c - 2), a1 = load_cell<T, false>(P, N, c - 1),
                 a2 = load_cell<T, false>(P, N, c), a3 = load_cell<T, false>(P, N, c + 1);
  T kl[3], kr[3];
  metric_row<T>(B, N, 2, c - 1, kl);
  metric_row<T>(B, N, 2, c, kr);
  face_from_cells<T>(a0, a1, a2, a3, kl, kr, ph, F);
}

// Each warp assembles 31 consecutive cells; lane l evaluates the k face on the
// left of its cell and takes the one on its right from lane l+1 by shuffle
// (lane 31's cell is the next warp's first, for which it only supplies the
// face), as in the FP32 assembly.
// NW: warps per CTA (8; 2 for the small tables of launch_tab, with a looser
// register cap since such a table puts few CTAs on an SM).
template <typename T, int OCC = 3, int NW = 8>
__global__ void __launch_bounds__(32 * NW, NW == 8 ? OCC : 8) k_fm_assemble(const Table tab, const int flags,
                                                                 const int stage, const int next_prims,
                                                                 const double gm1, const double R,
                                                                 const double iR, const Phys ph) {
  const int b = find_block_asm(tab, blockIdx.x);
  const Dev& dv = tab.b[b];
  const SplitBlock& B = dv.blk;
  if (threadIdx.x == 0) prefetch_assembly<T, false, true>(dv, blockIdx.x, flags, stage, 31 * NW, B.cta_begin_asm);
  grid_dep_wait();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Cell x;
  x.N = (int64_t)B.ni * B.nj * B.nk;
  x.c = (int64_t)(blockIdx.x - B.cta_begin_asm) * (31 * NW) + warp * 31 + lane;
  const bool alive = x.c < x.N;
  if (alive) {
    const uint32_t t1 = dv.dk.div((uint32_t)x.c);
    x.k = (int)((uint32_t)x.c - t1 * (uint32_t)B.nk);
    x.i = (int)dv.dj.div(t1);
    x.j = (int)(t1 - (uint32_t)x.i * (uint32_t)B.nj);
    x.ni = B.ni;
    x.nj = B.nj;
    x.nk = B.nk;
  }
  T fl[5] = {T(0), T(0), T(0), T(0), T(0)}, fr[5];
  // face c-1 | c exists for k-1 in [1, nk-3]
  if ((flags & kRhsInvscd) && alive && x.k >= 2 && x.k <= x.nk - 2)
    fm_k_face_left<T>(B, (int32_t)x.N, (int32_t)x.c, ph, fl);
#pragma unroll
  for (int v = 0; v < 5; ++v) fr[v] = __shfl_down_sync(0xffffffffu, fl[v], 1);
  if (lane == 31 || !alive) return;
  const int64_t N = x.N, c = x.c;
  const int64_t si = (int64_t)x.nj * x.nk, sj = x.nk;
  const int n[3] = {x.ni, x.nj, x.nk};
  const int idx[3] = {x.i, x.j, x.k};
  const int64_t st[3] = {si, sj, 1};
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (flags & kRhsInvscd) {
    const T* F = (const T*)B.F;
    const double ivd = __drcp_rn(B.vol[c] + 1e-300);
    const bool on[3] = {idx[0] >= 2 && idx[0] <= n[0] - 3, idx[1] >= 2 && idx[1] <= n[1] - 3,
                        idx[2] >= 2 && idx[2] <= n[2] - 3};
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      double dsum;
      if (sizeof(T) == sizeof(double)) {
        dsum = 0.0;  // axis by axis like the reference
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (on[a]) {
            if (a == 2) {
              dsum += (double)(fr[v] - fl[v]);
            } else {
              const T* Fa = F + (int64_t)(a * 5 + v) * N;
              dsum += (double)(Fa[c] - Fa[c - st[a]]);
            }
          }
      } else {
        T s = T(0);
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (on[a]) {
            if (a == 2) {
              s += fr[v] - fl[v];
            } else {
              const T* Fa = F + (int64_t)(a * 5 + v) * N;
              s += Fa[c] - Fa[c - st[a]];
            }
          }
        dsum = (double)s;
      }
      r[v] = -dsum * ivd;
    }
  }
  if (flags & kRhsViscous) {
    const T* G = (const T*)B.G;
    int64_t cp[3], cm[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      cp[l] = idx[l] + 1 == n[l] ? c - (int64_t)(n[l] - 1) * st[l] : c + st[l];
      cm[l] = idx[l] == 0 ? c + (int64_t)(n[l] - 1) * st[l] : c - st[l];
    }
    T kk[9];
#pragma unroll
    for (int lm = 0; lm < 9; ++lm) kk[lm] = metric<T>(B, N, lm, c);
    // D[comp][l] = 0.5 (G(c+e_l) - G(c-e_l))
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      T res = T(0);
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) {
        int comp;
        if (e == 3) {
          comp = 6 + jj;
        } else {
          const int lo = e < jj ? e : jj, hi = e < jj ? jj : e;
          comp = lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
        }
        const T* Gc = G + (int64_t)comp * N;
        res += T(0.5) * ((Gc[cp[0]] - Gc[cm[0]]) * kk[jj] + (Gc[cp[1]] - Gc[cm[1]]) * kk[3 + jj] +
                         (Gc[cp[2]] - Gc[cm[2]]) * kk[6 + jj]);
      }
      r[e + 1] += (double)res;
    }
  }
  if (stage == 0) {
#pragma unroll
    for (int v = 0; v < 5; ++v) B.out[v * N + c] = r[v];
  } else {
    const double ca = stage == 2 ? 0.75 : 1.0 / 3.0;
    const double cb = stage == 2 ? 0.25 : 2.0 / 3.0;
    double qn[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const int64_t o = v * N + c;
      const double t = B.q[o] + B.dt * r[v];
      qn[v] = stage == 1 ? t : ca * B.q0[o] + cb * t;
      B.out[o] = qn[v];
    }
    if (next_prims) {
      double pv[6];
      prims_of(qn, gm1, R, iR, pv);
      T rec[kRecP64];
#pragma unroll
      for (int v = 0; v < kRecP64; ++v) rec[v] = (T)pv[v];
      st_rec<T, kRecP64>((T*)B.prim_next + c * kRecP64, rec);
    }
  }
}


}  // namespace fm

// Record of cell c: the nine kxyz[l][m], then (FP32 records) the three
// gcl[m] = sum over the axes a with c_a in [2, n_a-3] of
// 0.5 (kxyz[a][m](c+e_a) - kxyz[a][m](c-e_a)), evaluated in FP64: the sum of
// the face-normal differences n_a(c) - n_a(c-e_a) the assembly multiplies by
// p_ref (rhs/invscd.py:87-89, 119-131).
template <typename T>
__global__ void k_metric_records(const double* __restrict__ kxyz, T* __restrict__ out, int ni, int nj, int nk) {
  const int64_t N = (int64_t)ni * nj * nk;
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  T rec[kRecK<T>];
#pragma unroll
  for (int lm = 0; lm < 9; ++lm) rec[lm] = (T)kxyz[lm * N + c];
#pragma unroll
  for (int lm = 9; lm < kRecK<T>; ++lm) rec[lm] = T(0);
  if (kRecK<T> >= 12) {
    const int k = (int)(c % nk), j = (int)((c / nk) % nj), i = (int)(c / ((int64_t)nk * nj));
    const int idx[3] = {i, j, k}, n[3] = {ni, nj, nk};
    const int64_t st[3] = {(int64_t)nj * nk, nk, 1};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double g = 0.0;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (idx[a] >= 2 && idx[a] <= n[a] - 3)
          g += 0.5 * (kxyz[(3 * a + m) * N + c + st[a]] - kxyz[(3 * a + m) * N + c - st[a]]);
      if (9 + m < kRecK<T>) rec[9 + m] = (T)g;
    }
  }
  st_rec<T, kRecK<T>>(out + c * kRecK<T>, rec);
}

// Sum of (pressure) over a block, one partial per CTA (fixed grid, fixed
// summation order: the result does not depend on scheduling).
constexpr int kPsumCtas = 592, kPsumThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}

__global__ void k_pressure_partial(const double* __restrict__ q, int64_t N, double gm1, double* __restrict__ part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
    const double r = q[c], u = q[N + c] / r, v = q[2 * N + c] / r, w = q[3 * N + c] / r;
    s += gm1 * (q[4 * N + c] - r * (0.5 * (u * u + v * v + w * w)));
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_fold_sum(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int t = threadIdx.x; t < n; t += blockDim.x) s += part[t];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

// Launch shapes of the split kernels, selected per plan by the autotuner
// (index 0 is the default): the minimum resident CTAs per SM of the flux and
// assembly kernels, i.e. their register caps.  These are the FP32 record
// kernels' shapes; kSplitVariants64 below are the FP64 kernels'.
struct SplitShape {
  int flux_occ, asm_occ;
};
constexpr SplitShape kSplitVariants[] = {{4, 4}, {3, 4}, {3, 6}, {3, 5}, {4, 3}, {2, 4}};
static_assert(sizeof(kSplitVariants) / sizeof(kSplitVariants[0]) == FJ_NUM_SPLIT_VARIANTS, "variant table");

// Launch shapes of the FP64 field-major kernels (the same variant index; FP64
// face arithmetic needs more registers at the same occupancy).
constexpr SplitShape kSplitVariants64[] = {{2, 3}, {2, 4}, {3, 3}, {2, 2}, {3, 4}, {3, 2}};
static_assert(sizeof(kSplitVariants64) / sizeof(kSplitVariants64[0]) == FJ_NUM_SPLIT_VARIANTS, "variant table");

template <int V>
void launch_pair64(const Table& tab, int ctas, int asm_ctas, const Phys& ph, int flags, int stage, int np,
                   cudaStream_t st, cudaEvent_t after_fluxes) {
  constexpr SplitShape sh = kSplitVariants64[V];
  pdl_launch(fm::k_fm_fluxes<double, sh.flux_occ>, ctas, kSplitThreads, 0, st, tab, ph, flags);
  if (after_fluxes) cudaEventRecord(after_fluxes, st);
  pdl_launch(fm::k_fm_assemble<double, sh.asm_occ>, asm_ctas, kSplitThreads, 0, st, tab, flags, stage, np, ph.gm1,
             ph.R, 1.0 / ph.R, ph);
}

template <typename T, bool K_AOS, int V>
void launch_pair(const Table& tab, int ctas, int asm_ctas, const Phys& ph, int flags, int stage, int np,
                 cudaStream_t st, cudaEvent_t after_fluxes) {
  constexpr SplitShape sh = kSplitVariants[V];
  pdl_launch(k_split_fluxes<T, K_AOS, sh.flux_occ>, ctas, kSplitThreads, 0, st, tab, ph, flags);
  if (after_fluxes) cudaEventRecord(after_fluxes, st);
  pdl_launch(k_split_assemble<T, K_AOS, sh.asm_occ>, asm_ctas, kSplitThreads, 0, st, tab, flags, stage, np, ph.gm1,
             ph.R, 1.0 / ph.R, ph);
}

template <typename T, bool K_AOS>
int launch_tab(const Table& tab, int ctas, int asm_ctas, const Phys& ph, int flags, int stage, bool prims_ready,
               bool next_prims, int variant, cudaStream_t st, cudaEvent_t after_fluxes, int nw = 8) {
  const int np = next_prims ? 1 : 0;
  if constexpr (sizeof(T) == 4) {
    if (nw == 2) {  // a small table: the role-split flux kernel and 2-warp assembly CTAs
      if (!prims_ready)
        pdl_launch(k_split_prims<T, 2>, ctas, 64, 0, st, tab, ph.gm1, ph.R, 1.0 / ph.R, K_AOS ? ph.p_ref : 0.0);
      pdl_launch(k_split_fluxes_roles<T, K_AOS>, ctas, 256, 0, st, tab, ph, flags);
      if (after_fluxes) cudaEventRecord(after_fluxes, st);
      pdl_launch(k_split_assemble_kmem<T, K_AOS>, asm_ctas, 64, 0, st, tab, flags, stage, np, ph.gm1, ph.R,
                 1.0 / ph.R, ph);
      return prims_ready ? 2 : 3;
    }
  }
  if constexpr (sizeof(T) == 8) {
    if (nw == 2) {  // a small table: the role-split flux kernel and 2-warp CTAs
      if (!prims_ready) pdl_launch(fm::k_fm_prims<double, 2>, ctas, 64, 0, st, tab, ph.gm1, ph.R, 1.0 / ph.R);
      pdl_launch(fm::k_fm_fluxes_roles<double>, ctas, 192, 0, st, tab, ph, flags);
      if (after_fluxes) cudaEventRecord(after_fluxes, st);
      pdl_launch(fm::k_fm_assemble<double, 3, 2>, asm_ctas, 64, 0, st, tab, flags, stage, np, ph.gm1, ph.R,
                 1.0 / ph.R, ph);
      return prims_ready ? 2 : 3;
    }
    if (!prims_ready) pdl_launch(fm::k_fm_prims<double>, ctas, kSplitThreads, 0, st, tab, ph.gm1, ph.R, 1.0 / ph.R);
    switch (variant) {
      case 1: launch_pair64<1>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 2: launch_pair64<2>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 3: launch_pair64<3>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 4: launch_pair64<4>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 5: launch_pair64<5>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      default: launch_pair64<0>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes);
    }
  } else {
    if (!prims_ready)
      pdl_launch(k_split_prims<T>, ctas, kSplitThreads, 0, st, tab, ph.gm1, ph.R, 1.0 / ph.R, K_AOS ? ph.p_ref : 0.0);
    switch (K_AOS ? variant : 0) {
      case 1: launch_pair<T, K_AOS, 1>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 2: launch_pair<T, K_AOS, 2>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 3: launch_pair<T, K_AOS, 3>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 4: launch_pair<T, K_AOS, 4>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      case 5: launch_pair<T, K_AOS, 5>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes); break;
      default: launch_pair<T, K_AOS, 0>(tab, ctas, asm_ctas, ph, flags, stage, np, st, after_fluxes);
    }
  }
  return prims_ready ? 2 : 3;
}

template <typename T>
int launch_split(fj_ctx* ctx, const SplitBlock* blocks, int nblocks, const Phys& ph, int flags,
                 int stage, bool prims_ready, bool next_prims, int variant, cudaStream_t st,
                 cudaEvent_t after_fluxes) {
  static int sms = 0;  // SMs of the device (B200: 148)
  if (sms == 0 && (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess || sms <= 0))
    sms = 148;
  for (int base = 0; base < nblocks; base += kMaxSplitBlocks) {
    Table tab;
    tab.n = std::min(kMaxSplitBlocks, nblocks - base);
    // tables with fewer 256-thread flux CTAs than two per SM run 2-warp CTAs
    int nw = 8;
    {
      int64_t wide = 0;
      for (int t = 0; t < tab.n; ++t) {
        const SplitBlock& sb = blocks[base + t];
        wide += ((int64_t)sb.ni * sb.nj * sb.nk + kSplitThreads - 1) / kSplitThreads;
      }
      if (wide < 2 * (int64_t)sms) nw = 2;
    }
    const int fcells = 32 * nw, acells = 31 * nw;
    int ctas = 0, asm_ctas = 0;
    const bool k_aos = blocks[base].kaos != nullptr;
    for (int t = 0; t < tab.n; ++t) {
      const SplitBlock& sb = blocks[base + t];
      // the kernels index cells and records with 32-bit offsets
      if ((int64_t)kRecF * sb.ni * sb.nj * sb.nk > INT32_MAX)
        return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block too large for the split pipeline");
      if ((sb.kaos != nullptr) != k_aos)
        return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "metric records on some blocks only");
      tab.b[t].blk = sb;
      tab.b[t].blk.cta_begin = ctas;
      tab.b[t].blk.cta_begin_asm = asm_ctas;
      tab.b[t].dk.init((uint32_t)sb.nk);
      tab.b[t].dj.init((uint32_t)sb.nj);
      const int64_t N = (int64_t)sb.ni * sb.nj * sb.nk;
      ctas += (int)((N + fcells - 1) / fcells);
      asm_ctas += (int)((N + acells - 1) / acells);
    }
    if (k_aos && sizeof(T) == 8)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "the FP64 split path reads kxyz directly");
    // the event marks the first chunk's flux launch
    cudaEvent_t ev = base == 0 ? after_fluxes : nullptr;
    ctx->launches += k_aos ? launch_tab<T, true>(tab, ctas, asm_ctas, ph, flags, stage, prims_ready, next_prims,
                                                 variant, st, ev, nw)
                           : launch_tab<T, false>(tab, ctas, asm_ctas, ph, flags, stage, prims_ready, next_prims,
                                                  variant, st, ev, nw);
    int s = launch_status(ctx, "split stage launch");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

}  // namespace

int split_metric_records(const double* kxyz, void* out, int ni, int nj, int nk, int precision, cudaStream_t st) {
  const int64_t N = (int64_t)ni * nj * nk;
  if (N <= 0) return FJ_OK;
  const int grid = (int)((N + 255) / 256);
  if (precision == FJ_PREC_F32FLUX)
    k_metric_records<float><<<grid, 256, 0, st>>>(kxyz, (float*)out, ni, nj, nk);
  else
    k_metric_records<double><<<grid, 256, 0, st>>>(kxyz, (double*)out, ni, nj, nk);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

size_t mean_pressure_scratch_bytes(int nblocks) { return ((size_t)kPsumCtas * nblocks + 1) * sizeof(double); }

int mean_pressure(const fj_block* blocks, int nblocks, double gm1, double* scratch, cudaStream_t st, double* out) {
  double* part = scratch;
  const size_t n = (size_t)kPsumCtas * nblocks;
  int64_t cells = 0;
  for (int b = 0; b < nblocks; ++b) {
    const int64_t N = (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
    cells += N;
    k_pressure_partial<<<kPsumCtas, kPsumThreads, 0, st>>>(blocks[b].q, N, gm1, part + (size_t)b * kPsumCtas);
  }
  k_fold_sum<<<1, 1024, 0, st>>>(part, (int)n, part + n);
  double h = 0.0;
  cudaError_t e = cudaMemcpyAsync(&h, part + n, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return FJ_ERR_CUDA;
  *out = cells > 0 ? h / (double)cells : 0.0;
  return FJ_OK;
}

size_t split_metric_record_bytes(int precision, int64_t N) {
  return precision == FJ_PREC_F32FLUX ? (size_t)N * kRecK<float> * sizeof(float)
                                      : (size_t)N * kRecK<double> * sizeof(double);
}

// Values per cell of each intermediate: records (FP32-flux) or field-major
// arrays (FP64).
static void split_counts(int precision, int& nP, int& nF, int& nG) {
  const bool rec = precision == FJ_PREC_F32FLUX;
  // the stage input's primitives and the next stage's: the assembly reads the
  // first (its k faces) while writing the second
  nP = rec ? 2 * kRecP : 2 * kRecP64;
  // FP32: the i/j face records and, for the kernels of small tables, the k
  // faces (Fk, 5 per cell); FP64: the i and j faces, field-major (the k faces
  // stay in the assembly)
  nF = rec ? kRecFA + kRecFB + 5 : 10;
  nG = 9;  // records: kRecG per cell in G, then one per cell in Gz
}

size_t split_scratch_bytes(int precision, int64_t cells) {
  const size_t t = precision == FJ_PREC_F32FLUX ? sizeof(float) : sizeof(double);
  int nP, nF, nG;
  split_counts(precision, nP, nF, nG);
  return (size_t)(nP + nF + nG) * (size_t)cells * t + 3 * 256;
}

void split_assign_scratch(int precision, SplitBlock* blocks, int nblocks, void* scratch) {
  const size_t t = precision == FJ_PREC_F32FLUX ? sizeof(float) : sizeof(double);
  int nP, nF, nG;
  split_counts(precision, nP, nF, nG);
  char* p = (char*)scratch;
  auto al = [](char* x) { return (char*)(((uintptr_t)x + 255) & ~(uintptr_t)255); };
  int64_t total = 0;
  for (int b = 0; b < nblocks; ++b) total += (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
  char* prim = al(p);
  char* F = al(prim + nP * total * t);
  char* G = al(F + nF * total * t);
  int64_t off = 0;
  for (int b = 0; b < nblocks; ++b) {
    const int64_t N = (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
    // records are multiples of 16 bytes: [input | next] primitive records
    const int rp = precision == FJ_PREC_F32FLUX ? kRecP : kRecP64;
    blocks[b].prim = prim + rp * off * t;
    blocks[b].prim_next = prim + (rp * total + rp * off) * t;
    if (precision == FJ_PREC_F32FLUX) {
      blocks[b].F = F + kRecFA * off * t;
      blocks[b].Fz = F + (kRecFA * total + kRecFB * off) * t;
      blocks[b].Fk = F + ((kRecFA + kRecFB) * total + 5 * off) * t;
    } else {
      blocks[b].F = F + nF * off * t;
      blocks[b].Fz = nullptr;
      blocks[b].Fk = nullptr;
    }
    if (precision == FJ_PREC_F32FLUX) {
      blocks[b].G = G + kRecG * off * t;
      blocks[b].Gz = G + (kRecG * total + off) * t;
    } else {
      blocks[b].G = G + nG * off * t;
      blocks[b].Gz = nullptr;
    }
    off += N;
  }
}

int split_stage(fj_ctx* ctx, const SplitBlock* blocks, int nblocks, const Phys& ph, int flags,
                int stage, int precision, cudaStream_t st, bool prims_ready, bool next_prims, int variant,
                cudaEvent_t after_fluxes) {
  if (next_prims && (stage < 1 || stage > 2)) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "next_prims needs stage 1 or 2");
  if (variant < 0 || variant >= FJ_NUM_SPLIT_VARIANTS) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown variant");
  if (precision == FJ_PREC_F32FLUX)
    return launch_split<float>(ctx, blocks, nblocks, ph, flags, stage, prims_ready, next_prims, variant, st,
                               after_fluxes);
  return launch_split<double>(ctx, blocks, nblocks, ph, flags, stage, prims_ready, next_prims, variant, st,
                              after_fluxes);
}

}  // namespace fj
