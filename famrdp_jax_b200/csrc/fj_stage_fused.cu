// fj_stage_fused.cu -- one TVD-RK3 stage (or one RHS) of one block in ONE
// kernel: the reference's inviscid sweeps (rhs/invscd.py:53-131), viscous
// fluxes and divergence (rhs/viscous.py:36-117) and the stage combine
// (solver/step.py:45-53), with no intermediate in global memory.
//
// Decomposition (2.5-D streaming): a CTA owns a TJ x TK tile of (j, k)
// columns and marches along i over a segment of planes.  Shared memory holds
//   P   ring of 4 planes of primitives (rho, u, v, w, p, T) on the tile plus a
//       2-cell halo in j and k (indices wrap around the padded block, as the
//       reference's jnp.roll does for the viscous terms);
//   K   ring of 2 planes of metrics kxyz on the tile plus a 1-cell halo;
//   G   ring of 3 planes of viscous flux components (tau_00 tau_01 tau_02
//       tau_11 tau_12 tau_22 Ge_0 Ge_1 Ge_2) on the tile plus a 1-cell halo;
//   FJ, FK the Roe face fluxes of the current plane along j and k
// (the i-face flux of a column stays in its thread's registers).
// Iteration i (two barriers):
//   A  primitives of plane i+2, metrics of plane i+1                 | sync
//   B  one balanced work list: i faces (i|i+1), j and k faces of plane i,
//      G of plane i+1; each thread also reads its own cell's metrics  | sync
//   C  per-cell assembly + stage combine of plane i.
// The segment's first two iterations only fill the rings (i = ib-2, ib-1).
//
// Inputs are read from HBM once per stage (halo re-reads hit L2); the only
// write is the stage result.  T is the flux arithmetic type: double (the
// drop-in FP64 path) or float (FP32-flux path: state, volume reciprocal,
// accumulation and combine stay FP64; metrics may come as an FP32 copy).
#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_rhs.cuh"
#include "fj_stage.cuh"

namespace fj {

namespace {

// x mod n for the small overshoots of halo indices (|x| < a few n).
__device__ __forceinline__ int wrap(int x, int n) {
  while (x < 0) x += n;
  while (x >= n) x -= n;
  return x;
}

__device__ __forceinline__ int slot4(int p) { return p & 3; }  // two's complement: p mod 4
__device__ __forceinline__ int slot3(int p) { return ((p % 3) + 3) % 3; }

template <typename T, int TJ, int TK>
struct Tile {
  static constexpr int NT = TJ * TK;
  static constexpr int HJ = TJ + 4, HK = TK + 4, HN = HJ * HK;  // primitive plane
  static constexpr int GJ = TJ + 2, GK = TK + 2, GN = GJ * GK;  // viscous-flux / metric plane
  static constexpr int NFI = NT, NFJ = (TJ + 1) * TK, NFK = TJ * (TK + 1);
  static constexpr int NW = NFI + NFJ + NFK + GN;                // phase-B work items
  static constexpr size_t kP = (size_t)4 * 6 * HN;
  static constexpr size_t kG = (size_t)3 * 9 * GN;
  static constexpr size_t kK = (size_t)2 * 9 * GN;
  static constexpr size_t bytes() { return (kP + kG + kK + 5 * (NFJ + NFK)) * sizeof(T); }
  // CTAs per SM the launch bounds ask the register allocator to allow
  static constexpr int kMinBlocks = sizeof(T) == 8 ? 1 : (NT <= 128 ? 3 : (NT <= 256 ? 2 : 1));
  // per-thread points of the next plane's loads held in registers
  static constexpr int NPP = (HN + NT - 1) / NT, NKP = (GN + NT - 1) / NT;
};

// Raw state of plane p on the tile + 2-halo: each thread loads its points
// (t, t + NT, ...) into registers; store_plane turns them into primitives.
template <typename T, int TJ, int TK>
__device__ __forceinline__ void issue_plane(const StageArgs& a, int p, int j0, int k0,
                                            double (&qr)[Tile<T, TJ, TK>::NPP][5]) {
  using TL = Tile<T, TJ, TK>;
  const int64_t N = (int64_t)a.ni * a.nj * a.nk;
  const int64_t base = (int64_t)wrap(p, a.ni) * a.nj * a.nk;
#pragma unroll
  for (int s = 0; s < TL::NPP; ++s) {
    const int t = threadIdx.x + s * TL::NT;
    if (t < TL::HN) {
      const int hj = t / TL::HK, hk = t - (t / TL::HK) * TL::HK;
      const int j = wrap(j0 - 2 + hj, a.nj), k = wrap(k0 - 2 + hk, a.nk);
      const double* qc = a.q + base + (int64_t)j * a.nk + k;
#pragma unroll
      for (int v = 0; v < 5; ++v) qr[s][v] = __ldg(qc + v * N);
    }
  }
}

// Primitives (rho, u, v, w, p, T) of the issued plane into P ring slot slot4(p)
// (physics/eos.py:12-17; T = p / max(rho R, 1e-300), rhs/viscous.py:36).
template <typename T, int TJ, int TK>
__device__ __forceinline__ void store_plane(const StageArgs& a, T* __restrict__ P, int p,
                                            const double (&qr)[Tile<T, TJ, TK>::NPP][5]) {
  using TL = Tile<T, TJ, TK>;
  T* dst = P + (size_t)slot4(p) * 6 * TL::HN;
  const double gm1 = a.ph.gm1, R = a.ph.R, inv_R = 1.0 / a.ph.R;
#pragma unroll
  for (int s = 0; s < TL::NPP; ++s) {
    const int t = threadIdx.x + s * TL::NT;
    if (t < TL::HN) {
      const double r = qr[s][0];
      const double ir = 1.0 / r;
      const double u = qr[s][1] * ir, v = qr[s][2] * ir, w = qr[s][3] * ir;
      const double p_ = gm1 * (qr[s][4] - r * (0.5 * (u * u + v * v + w * w)));
      const double Tt = r * R > 1e-300 ? p_ * ir * inv_R : p_ * 1e300;
      dst[t] = (T)r;
      dst[TL::HN + t] = (T)u;
      dst[2 * TL::HN + t] = (T)v;
      dst[3 * TL::HN + t] = (T)w;
      dst[4 * TL::HN + t] = (T)p_;
      dst[5 * TL::HN + t] = (T)Tt;
    }
  }
}

// Metrics of plane p on the tile + 1-halo into registers, then into K ring
// slot p & 1.
template <typename T, int TJ, int TK>
__device__ __forceinline__ void issue_metrics(const StageArgs& a, int p, int j0, int k0,
                                              T (&kr)[Tile<T, TJ, TK>::NKP][9]) {
  using TL = Tile<T, TJ, TK>;
  const int64_t N = (int64_t)a.ni * a.nj * a.nk;
  const int64_t base = (int64_t)wrap(p, a.ni) * a.nj * a.nk;
#pragma unroll
  for (int s = 0; s < TL::NKP; ++s) {
    const int t = threadIdx.x + s * TL::NT;
    if (t < TL::GN) {
      const int gj = t / TL::GK, gk = t - (t / TL::GK) * TL::GK;
      const int64_t c = base + (int64_t)wrap(j0 - 1 + gj, a.nj) * a.nk + wrap(k0 - 1 + gk, a.nk);
      if (a.kxyz32) {
#pragma unroll
        for (int lm = 0; lm < 9; ++lm) kr[s][lm] = (T)__ldg(a.kxyz32 + lm * N + c);
      } else {
#pragma unroll
        for (int lm = 0; lm < 9; ++lm) kr[s][lm] = (T)__ldg(a.kxyz + lm * N + c);
      }
    }
  }
}

template <typename T, int TJ, int TK>
__device__ __forceinline__ void store_metrics(T* __restrict__ K, int p,
                                              const T (&kr)[Tile<T, TJ, TK>::NKP][9]) {
  using TL = Tile<T, TJ, TK>;
  T* dst = K + (size_t)(p & 1) * 9 * TL::GN;
#pragma unroll
  for (int s = 0; s < TL::NKP; ++s) {
    const int t = threadIdx.x + s * TL::NT;
    if (t < TL::GN) {
#pragma unroll
      for (int lm = 0; lm < 9; ++lm) dst[lm * TL::GN + t] = kr[s][lm];
    }
  }
}

template <typename T, int TJ, int TK>
__global__ void __launch_bounds__(TJ* TK, (Tile<T, TJ, TK>::kMinBlocks)) k_stage_fused(const StageArgs a) {
  using TL = Tile<T, TJ, TK>;
  using M = FastMath<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* P = (T*)smem_raw;
  T* G = P + TL::kP;
  T* K = G + TL::kG;
  T* FJ = K + TL::kK;
  T* FK = FJ + 5 * TL::NFJ;

  const int tile = blockIdx.x;
  const int tj = tile / a.ntk, tk = tile - tj * a.ntk;
  const int j0 = tj * TJ, k0 = tk * TK;
  const int ib = blockIdx.y * a.seg;
  const int ie = min(a.ni, ib + a.seg);
  const int lj = threadIdx.x / TK, lk = threadIdx.x - (threadIdx.x / TK) * TK;
  const int j = j0 + lj, k = k0 + lk;
  const bool active = j < a.nj && k < a.nk;
  const int64_t N = (int64_t)a.ni * a.nj * a.nk;
  const int ni = a.ni, nj = a.nj, nk = a.nk;
  const bool do_inv = (a.flags & kRhsInvscd) != 0, do_vis = (a.flags & kRhsViscous) != 0;
  const T gm1 = (T)a.ph.gm1, inv_gm1 = (T)(1.0 / a.ph.gm1), eps_e = (T)a.ph.eps_entropy;
  const T mu0 = (T)a.ph.mu0, Ts = (T)a.ph.Ts;
  const T inv_T0 = (T)(1.0 / a.ph.T0), sfac = (T)(a.ph.T0 + a.ph.Ts);
  const T kap_fac = (T)(a.ph.cp / a.ph.Pr);
  const T third = (T)(1.0 / 3.0);
  const int gown = (lj + 1) * TL::GK + (lk + 1);

  T Fprev[5] = {T(0), T(0), T(0), T(0), T(0)};
  T Fnext[5] = {T(0), T(0), T(0), T(0), T(0)};
  T kown[9];

  // C: assembly + stage combine of plane i (face fluxes from the previous
  // phase B: Fnext = face i|i+1, Fprev = face i-1|i, FJ/FK, G ring, kown)
  auto assemble = [&](const int i) {
    if (active) {
      const int64_t c = ((int64_t)i * nj + j) * nk + k;
      double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      if (do_inv) {
        // face-flux differences along i, j, k (cells [2, n-3] of each axis);
        // summed in T, then scaled by 1/(vol + 1e-300) in FP64
        const bool ii = i >= 2 && i <= ni - 3, jj = j >= 2 && j <= nj - 3, kk = k >= 2 && k <= nk - 3;
        const int jR = (lj + 1) * TK + lk, jL = lj * TK + lk;
        const int kR = lj * (TK + 1) + lk + 1, kL = lj * (TK + 1) + lk;
        const double ivd = 1.0 / (a.vol[c] + 1e-300);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          double dsum;
          if (sizeof(T) == sizeof(double)) {
            // FP64: accumulate axis by axis like the reference
            dsum = 0.0;
            if (ii) dsum += (double)(Fnext[v] - Fprev[v]);
            if (jj) dsum += (double)(FJ[v * TL::NFJ + jR] - FJ[v * TL::NFJ + jL]);
            if (kk) dsum += (double)(FK[v * TL::NFK + kR] - FK[v * TL::NFK + kL]);
          } else {
            T s = T(0);
            if (ii) s += Fnext[v] - Fprev[v];
            if (jj) s += FJ[v * TL::NFJ + jR] - FJ[v * TL::NFJ + jL];
            if (kk) s += FK[v * TL::NFK + kR] - FK[v * TL::NFK + kL];
            dsum = (double)s;
          }
          r[v] = -dsum * ivd;
        }
      }
      if (do_vis) {
        const T* Gm = G + (size_t)slot3(i - 1) * 9 * TL::GN;
        const T* Gc = G + (size_t)slot3(i) * 9 * TL::GN;
        const T* Gp = G + (size_t)slot3(i + 1) * 9 * TL::GN;
        // rows 0..2: momentum (tau row e), row 3: energy
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
            const size_t o = (size_t)comp * TL::GN + gown;
            res += T(0.5) * ((Gp[o] - Gm[o]) * kown[jj] + (Gc[o + TL::GK] - Gc[o - TL::GK]) * kown[3 + jj] +
                             (Gc[o + 1] - Gc[o - 1]) * kown[6 + jj]);
          }
          r[e + 1] += (double)res;
        }
      }
      if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a.out[v * N + c] = r[v];
      } else {
        const double ca = a.stage == 2 ? 0.75 : 1.0 / 3.0;
        const double cb = a.stage == 2 ? 0.25 : 2.0 / 3.0;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const int64_t o = v * N + c;
          const double t = a.q[o] + a.dt * r[v];
          a.out[o] = a.stage == 1 ? t : ca * a.q0[o] + cb * t;
        }
      }
    }
  };

  {
    double qr[TL::NPP][5];
    T kr[TL::NKP][9];
    issue_plane<T, TJ, TK>(a, ib - 2, j0, k0, qr);
    store_plane<T, TJ, TK>(a, P, ib - 2, qr);
    issue_plane<T, TJ, TK>(a, ib - 1, j0, k0, qr);
    store_plane<T, TJ, TK>(a, P, ib - 1, qr);
    issue_metrics<T, TJ, TK>(a, ib - 2, j0, k0, kr);
    store_metrics<T, TJ, TK>(K, ib - 2, kr);
  }

  for (int i = ib - 2; i < ie; ++i) {
    // ---- A: loads of plane i+2 (state) and i+1 (metrics) in flight while
    //      the previous plane is assembled (C of plane i-1), then stored
    {
      double qr[TL::NPP][5];
      T kr[TL::NKP][9];
      issue_plane<T, TJ, TK>(a, i + 2, j0, k0, qr);
      issue_metrics<T, TJ, TK>(a, i + 1, j0, k0, kr);
      if (i - 1 >= ib) assemble(i - 1);
#pragma unroll
      for (int v = 0; v < 5; ++v) Fprev[v] = Fnext[v];
      store_plane<T, TJ, TK>(a, P, i + 2, qr);
      store_metrics<T, TJ, TK>(K, i + 1, kr);
    }
    __syncthreads();

    // ---- B: faces of plane i, viscous fluxes of plane i+1 (one work list)
    const T* Ki = K + (size_t)(i & 1) * 9 * TL::GN;
    const T* Kn = K + (size_t)((i + 1) & 1) * 9 * TL::GN;
#pragma unroll
    for (int v = 0; v < 5; ++v) Fnext[v] = T(0);
#pragma unroll
    for (int lm = 0; lm < 9; ++lm) kown[lm] = Ki[lm * TL::GN + gown];
    for (int w = threadIdx.x; w < TL::NW; w += TL::NT) {
      if (w < TL::NFI + TL::NFJ + TL::NFK) {
        // face item: cells c0..c3 in P, the two adjacent cells' metric rows in K
        int ax, h0, hstep, ps0, gl, gstep, o_idx;
        bool valid;
        const T* Kl;
        if (w < TL::NFI) {  // i face between planes i and i+1, column w
          const int wj = w / TK, wk = w - (w / TK) * TK;
          valid = do_inv && j0 + wj < nj && k0 + wk < nk && i >= ib - 1 && i - 1 >= 0 && i - 1 <= ni - 4;
          ax = 0;
          h0 = (wj + 2) * TL::HK + wk + 2;
          hstep = 0;
          ps0 = i - 1;
          gl = (wj + 1) * TL::GK + wk + 1;
          gstep = 0;
          Kl = Ki;
          o_idx = -1;
        } else if (w < TL::NFI + TL::NFJ) {  // j face between j0-1+fj and j0+fj
          const int t = w - TL::NFI;
          const int fj = t / TK, fk = t - (t / TK) * TK;
          const int jl = j0 - 1 + fj;
          valid = do_inv && i >= ib && jl - 1 >= 0 && jl - 1 <= nj - 4 && k0 + fk < nk;
          ax = 1;
          h0 = fj * TL::HK + fk + 2;
          hstep = TL::HK;
          ps0 = i;
          gl = fj * TL::GK + fk + 1;
          gstep = TL::GK;
          Kl = Ki;
          o_idx = t;
        } else {  // k face between k0-1+fk and k0+fk
          const int t = w - TL::NFI - TL::NFJ;
          const int fj = t / (TK + 1), fk = t - (t / (TK + 1)) * (TK + 1);
          const int kl = k0 - 1 + fk;
          valid = do_inv && i >= ib && kl - 1 >= 0 && kl - 1 <= nk - 4 && j0 + fj < nj;
          ax = 2;
          h0 = (fj + 2) * TL::HK + fk;
          hstep = 1;
          ps0 = i;
          gl = (fj + 1) * TL::GK + fk;
          gstep = 1;
          Kl = Ki;
          o_idx = t;
        }
        T F[5] = {T(0), T(0), T(0), T(0), T(0)};
        if (valid) {
          Prim<T> cell[4];
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            // i faces step through ring slots, j/k faces through the plane
            const T* ps = P + (size_t)slot4(ax == 0 ? ps0 + s : ps0) * 6 * TL::HN + h0 + s * hstep;
            cell[s].rho = ps[0];
            cell[s].u = ps[TL::HN];
            cell[s].v = ps[2 * TL::HN];
            cell[s].w = ps[3 * TL::HN];
            cell[s].p = ps[4 * TL::HN];
          }
          const T* Kr = ax == 0 ? Kn : Kl;
          const int gr = gl + gstep;
          const int m0 = 3 * ax * TL::GN;
          invscd_face_fast<T>(cell, Kl[m0 + gl], Kl[m0 + TL::GN + gl], Kl[m0 + 2 * TL::GN + gl], Kr[m0 + gr],
                              Kr[m0 + TL::GN + gr], Kr[m0 + 2 * TL::GN + gr], gm1, inv_gm1, eps_e,
                              a.ph.limiter, F);
        }
        if (o_idx < 0) {
#pragma unroll
          for (int v = 0; v < 5; ++v) Fnext[v] = F[v];
        } else if (ax == 1) {
#pragma unroll
          for (int v = 0; v < 5; ++v) FJ[v * TL::NFJ + o_idx] = F[v];
        } else {
#pragma unroll
          for (int v = 0; v < 5; ++v) FK[v * TL::NFK + o_idx] = F[v];
        }
      } else if (do_vis) {
        // viscous flux components at plane i+1, point (j0-1+gj, k0-1+gk)
        const int t = w - TL::NFI - TL::NFJ - TL::NFK;
        const int gj = t / TL::GK, gk = t - (t / TL::GK) * TL::GK;
        if ((gj == 0 || gj == TL::GJ - 1) && (gk == 0 || gk == TL::GK - 1)) continue;
        const int p = i + 1;
        const int h = (gj + 1) * TL::HK + (gk + 1);
        const T* Pm = P + (size_t)slot4(p - 1) * 6 * TL::HN;
        const T* Pc = P + (size_t)slot4(p) * 6 * TL::HN;
        const T* Pp = P + (size_t)slot4(p + 1) * 6 * TL::HN;
        T d[4][3];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const int f = s < 3 ? s + 1 : 5;  // u, v, w, T
          const size_t o = (size_t)f * TL::HN;
          d[s][0] = T(0.5) * (Pp[o + h] - Pm[o + h]);
          d[s][1] = T(0.5) * (Pc[o + h + TL::HK] - Pc[o + h - TL::HK]);
          d[s][2] = T(0.5) * (Pc[o + h + 1] - Pc[o + h - 1]);
        }
        T g[4][3];
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int m = 0; m < 3; ++m)
            g[s][m] = d[s][0] * Kn[m * TL::GN + t] + d[s][1] * Kn[(3 + m) * TL::GN + t] +
                      d[s][2] * Kn[(6 + m) * TL::GN + t];
        const T u = Pc[TL::HN + h], v = Pc[2 * TL::HN + h], wv = Pc[3 * TL::HN + h];
        T mu = mu0;
        if (a.ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
          const T Tt = Pc[5 * TL::HN + h];
          const T r = Tt * inv_T0;
          mu = mu0 * (r * M::sqrt_pos(r)) * sfac * M::rcp(Tt + Ts);
        }
        const T kappa = kap_fac * mu;
        const T div_u = g[0][0] + g[1][1] + g[2][2];
        const T t00 = T(2) * mu * (g[0][0] - div_u * third);
        const T t01 = mu * (g[0][1] + g[1][0]);
        const T t02 = mu * (g[0][2] + g[2][0]);
        const T t11 = T(2) * mu * (g[1][1] - div_u * third);
        const T t12 = mu * (g[1][2] + g[2][1]);
        const T t22 = T(2) * mu * (g[2][2] - div_u * third);
        T* dst = G + (size_t)slot3(p) * 9 * TL::GN + t;
        dst[0] = t00;
        dst[TL::GN] = t01;
        dst[2 * TL::GN] = t02;
        dst[3 * TL::GN] = t11;
        dst[4 * TL::GN] = t12;
        dst[5 * TL::GN] = t22;
        dst[6 * TL::GN] = u * t00 + v * t01 + wv * t02 + kappa * g[3][0];
        dst[7 * TL::GN] = u * t01 + v * t11 + wv * t12 + kappa * g[3][1];
        dst[8 * TL::GN] = u * t02 + v * t12 + wv * t22 + kappa * g[3][2];
      }
    }
    __syncthreads();

  }
  if (ie - 1 >= ib) assemble(ie - 1);
}

template <typename T, int TJ, int TK>
int launch_tiled(fj_ctx* ctx, StageArgs a, int seg, cudaStream_t st) {
  using TL = Tile<T, TJ, TK>;
  cudaError_t e = cudaFuncSetAttribute(k_stage_fused<T, TJ, TK>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TL::bytes());
  if (e != cudaSuccess) return cuda_status(ctx, e, "fused stage: shared memory attribute");
  a.ntj = (a.nj + TJ - 1) / TJ;
  a.ntk = (a.nk + TK - 1) / TK;
  if (seg <= 0) {
    // enough CTAs for two waves at the kernel's residency, segments >= 8 planes
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_fused<T, TJ, TK>, TL::NT, TL::bytes());
    const int tiles = a.ntj * a.ntk;
    const int target = 2 * nsm * (per_sm > 0 ? per_sm : 1);
    const int nseg = (target + tiles - 1) / tiles;
    seg = (a.ni + nseg - 1) / nseg;
    if (seg < 8) seg = 8;
  }
  a.seg = seg;
  dim3 grid(a.ntj * a.ntk, (a.ni + a.seg - 1) / a.seg);
  k_stage_fused<T, TJ, TK><<<grid, TL::NT, TL::bytes(), st>>>(a);
  ctx->launches += 1;
  return launch_status(ctx, "fused stage launch");
}

}  // namespace

int fused_stage(fj_ctx* ctx, const StageArgs& a, int seg, int precision, int tile, cudaStream_t st) {
  if (precision == FJ_PREC_F32FLUX) {
    switch (tile) {
      case 1: return launch_tiled<float, 4, 32>(ctx, a, seg, st);
      case 2: return launch_tiled<float, 6, 32>(ctx, a, seg, st);
      case 3: return launch_tiled<float, 8, 16>(ctx, a, seg, st);
      case 4: return launch_tiled<float, 16, 32>(ctx, a, seg, st);
      case 5: return launch_tiled<float, 8, 64>(ctx, a, seg, st);
      case 6: return launch_tiled<float, 16, 16>(ctx, a, seg, st);
      default: return launch_tiled<float, 8, 32>(ctx, a, seg, st);
    }
  }
  // FP64 tiles must fit 227 KB of shared memory: the 512-thread shapes do not
  switch (tile) {
    case 1: return launch_tiled<double, 4, 32>(ctx, a, seg, st);
    case 2: return launch_tiled<double, 6, 32>(ctx, a, seg, st);
    case 3: case 6: return launch_tiled<double, 8, 16>(ctx, a, seg, st);
    default: return launch_tiled<double, 8, 32>(ctx, a, seg, st);
  }
}

}  // namespace fj
