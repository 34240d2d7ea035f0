// fj_stage_tile.cu -- one TVD-RK3 stage of MANY blocks with FP32 fluxes and
// FP64 state in ONE persistent launch: the reference's inviscid sweeps
// (rhs/invscd.py:53-131), viscous fluxes and divergence
// (rhs/viscous.py:36-117) and the stage combine (solver/step.py:45-53), with
// no intermediate in global memory.
//
// Work-list.  A tile is TJ = 8 rows (j) x TK = 30 columns (k) of one block;
// a work item is one segment of consecutive i-planes of one tile (segments
// of 24..48 planes when that gives the grid several items per CTA, else the
// whole i extent).  Items are ordered segment-slowest (segment, block, tile),
// and the CTAs of the persistent grid (two per SM) take them in that order
// from a work counter, so the CTAs busy at one time hold neighbouring tiles of
// the same plane range and share their halo rows in L2.  A CTA streams along
// i through each segment.
//
// Shared memory (one CTA, 8 warps; warp w owns row j0 + w, lane l column
// k0 - 1 + l, so lanes 1..30 are the tile's columns and lanes 0 and 31 its
// k-halo):
//   P   ring of 4 planes of primitives (rho u v w p', FP32) on the tile plus
//       its 2-cell ghost layers in j and k, each plane ONE TMA box
//       (cp.async.bulk.tensor, 36 x 12 x 5 floats) of the padded primitive
//       array, which already holds the periodic images at the block's j and k
//       ends; a producer thread keeps the ring 2 planes ahead;
//   G   ring of 4 planes of viscous flux components on the tile + 1 ring;
//   Sj  the limited j-slopes of the next plane on the tile + 1 ring;
//   Fj  the j-face fluxes of the current plane.
// Registers carry what stays in a thread's own column: its i-slope, its two
// i-face fluxes and its left k-face flux.
//
// Iteration p (one barrier):
//   A(p)  all from data already in shared memory: G(p+1); the k-slopes and
//         the k-face on the left of each column (lane l-1's slope by shuffle);
//         the j-slopes of plane p+1; the j-face (r | r+1) of plane p from the
//         j-slopes of plane p (written in A(p-1)); the i-slope of plane p+1 and
//         the i-face (p | p+1); the ring rows' work rotates over the warps.
//   ----- __syncthreads; the producer refills the slot of plane p with p+4
//   B(p)  assembly of plane p: face-flux differences / vol over the active
//         axes (+ the FP64 pressure-offset term), viscous divergence of G,
//         TVD-RK3 combine in FP64, and the primitives of the result written to
//         the next stage's padded array (with its periodic images).
// B(p) and A(p+1) run in the same barrier interval: their shared-memory slots
// are disjoint (G: 4 planes, Sj and Fj: 2).
//
// Cell-centred slopes: the face c | c+e uses pL = P(c) + s(c)/2 and
// pR = P(c+e) - s(c+e)/2 with s(c) = lim(P(c) - P(c-e), P(c+e) - P(c)), which
// is muscl2.py:18-37 (limiter arguments in the reference's order); each slope
// is evaluated once per cell and axis instead of once per face side.
//
// Bounded waits: every mbarrier wait gives up after a limit; a CTA whose wait
// gave up sets the error word, stops issuing loads and computing, waits for
// its copies in flight and exits.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>
#include <new>

#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_tile.cuh"

namespace fj {

namespace {

constexpr int TJ = 8, TK = 30;
constexpr int NW = TJ, NT = 32 * NW;
constexpr int BW = 36, BH = TJ + 4, NF = 5;
constexpr int PSLOT = NF * BH * BW;           // floats of one primitive plane box
constexpr int PSLOT_STRIDE = 2176;            // slot pitch: 8704 bytes, a multiple of 128
constexpr uint32_t kBoxBytes = PSLOT * 4;     // bytes one TMA box delivers
constexpr int RS = 4;                         // primitive planes in the ring
constexpr int GR = TJ + 2, GC = 32;           // rows / columns of G and Sj planes
constexpr int GSLOT = 9 * GR * GC;
constexpr int SSLOT = 5 * GR * GC;
constexpr int FR = TJ + 1;
constexpr int FSLOT = 5 * FR * GC;
constexpr int kSmemFloats = RS * PSLOT_STRIDE + 4 * GSLOT + 2 * SSLOT + 2 * FSLOT;
constexpr size_t kSmemBytes = (size_t)kSmemFloats * 4 + RS * 8 + 16 + 128;  // + mbarriers, flags, alignment
constexpr int kDefaultWaitLimit = 1 << 22;
constexpr int kDrainWaitLimit = 1 << 26;
static_assert(PSLOT <= PSLOT_STRIDE, "slot pitch");
static_assert(kSmemBytes <= 113 * 1024, "two CTAs per SM");

struct __align__(64) TileParams {
  CUtensorMap map[kTileMaxBlocks];
  TileBlock blk[kTileMaxBlocks];
  Phys ph;
  int* err;
  int* next;            // work counter (zeroed before the launch)
  int nb, stage, wait_limit;
  int seg_len;          // planes per segment
  int max_seg;          // segments of the block with the most planes
  int items;            // work items: (segment, block, tile) with the segment slowest
};
static_assert(sizeof(TileParams) <= 32764, "kernel parameter space");

__device__ __forceinline__ uint32_t s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(s32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of parity `parity` to complete, at most `limit` tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int limit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try(b, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_plane(float* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s32(bar)), "r"(kBoxBytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(s32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(s32(bar))
      : "memory");
}

__device__ __forceinline__ int wrap1(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

struct F5 {
  float v[5];
};

__device__ __forceinline__ F5 ldP(const float* S, int by, int bx) {
  F5 o;
#pragma unroll
  for (int f = 0; f < NF; ++f) o.v[f] = S[(f * BH + by) * BW + bx];
  return o;
}

__device__ __forceinline__ float lim(float a, float b, int limiter) {
  return limiter == 0 ? minmod_sel(a, b) : vanleer(a, b);
}

// Limited slopes lim(c - m, p - c) of the five primitives.
__device__ __forceinline__ F5 slope(const F5& m, const F5& c, const F5& p, int limiter) {
  F5 s;
#pragma unroll
  for (int f = 0; f < NF; ++f) s.v[f] = lim(c.v[f] - m.v[f], p.v[f] - c.v[f], limiter);
  return s;
}

// FP32 constants of the face and viscous arithmetic.
struct Consts {
  float gm1, inv_gm1, eps, p_ref, R, inv_T0, sfac, Ts, kap_fac;
  int limiter, visc_law;
};

// One inviscid face (rhs/invscd.py:62-100) between cells c1 and c2 from their
// primitives and limited slopes: MUSCL face states, normal from the two
// cells' kxyz rows, Roe (pressure offset form), times |n|.
__device__ __forceinline__ void face_flux(const F5& c1, const F5& s1, const F5& c2, const F5& s2, const float kl[3],
                                          const float kr[3], const Consts& C, float F[5]) {
  const Prim<float> L{c1.v[0] + 0.5f * s1.v[0], c1.v[1] + 0.5f * s1.v[1], c1.v[2] + 0.5f * s1.v[2],
                      c1.v[3] + 0.5f * s1.v[3], c1.v[4] + 0.5f * s1.v[4]};
  const Prim<float> R{c2.v[0] - 0.5f * s2.v[0], c2.v[1] - 0.5f * s2.v[1], c2.v[2] - 0.5f * s2.v[2],
                      c2.v[3] - 0.5f * s2.v[3], c2.v[4] - 0.5f * s2.v[4]};
  const float nf0 = 0.5f * (kl[0] + kr[0]), nf1 = 0.5f * (kl[1] + kr[1]), nf2 = 0.5f * (kl[2] + kr[2]);
  const float nmag = FastMath<float>::sqrt_nn(nf0 * nf0 + nf1 * nf1 + nf2 * nf2) + Tiny<float>::nmag();
  const float inv = FastMath<float>::rcp(nmag);
  roe_prim<float, true>(L, R, nf0 * inv, nf1 * inv, nf2 * inv, C.gm1, C.inv_gm1, C.eps, F, C.p_ref);
#pragma unroll
  for (int v = 0; v < 5; ++v) F[v] *= nmag;
}

// u, v, w and T = p / max(rho R, tiny) of the box cell (by, bx) of plane S
// (rhs/viscous.py:36; p = p' + p_ref).
__device__ __forceinline__ void uvwT(const float* S, int by, int bx, const Consts& C, float o[4]) {
  const float rho = S[(0 * BH + by) * BW + bx];
  o[0] = S[(1 * BH + by) * BW + bx];
  o[1] = S[(2 * BH + by) * BW + bx];
  o[2] = S[(3 * BH + by) * BW + bx];
  o[3] = __fdividef(S[(4 * BH + by) * BW + bx] + C.p_ref, fmaxf(rho * C.R, 1e-37f));
}

// The nine viscous flux components at box cell (by, bx) of plane S0, with
// the i-neighbours in planes Sm / Sp (rhs/viscous.py:36-105; central
// differences over the wrapped neighbours, which the padded array and the
// plane wrap provide): tau_00 tau_01 tau_02 tau_11 tau_12 tau_22 and the
// energy flux components u_i tau_ij - heat_j.
__device__ __forceinline__ void visc_flux(const float* Sm, const float* S0, const float* Sp, int by, int bx,
                                          const float kk[9], float mu0, const Consts& C, float G[9]) {
  float a[4], b[4], d[4][3];
  uvwT(Sp, by, bx, C, a);
  uvwT(Sm, by, bx, C, b);
#pragma unroll
  for (int s = 0; s < 4; ++s) d[s][0] = 0.5f * (a[s] - b[s]);
  uvwT(S0, by + 1, bx, C, a);
  uvwT(S0, by - 1, bx, C, b);
#pragma unroll
  for (int s = 0; s < 4; ++s) d[s][1] = 0.5f * (a[s] - b[s]);
  uvwT(S0, by, bx + 1, C, a);
  uvwT(S0, by, bx - 1, C, b);
#pragma unroll
  for (int s = 0; s < 4; ++s) d[s][2] = 0.5f * (a[s] - b[s]);
  float c0[4];
  uvwT(S0, by, bx, C, c0);
  float g[4][3];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[m] + d[s][1] * kk[3 + m] + d[s][2] * kk[6 + m];
  float mu = mu0;
  if (C.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
    const float r = c0[3] * C.inv_T0;
    mu = mu0 * (r * FastMath<float>::sqrt_pos(r)) * C.sfac * FastMath<float>::rcp(c0[3] + C.Ts);
  }
  const float kappa = C.kap_fac * mu;
  const float third = 1.0f / 3.0f;
  const float div_u = g[0][0] + g[1][1] + g[2][2];
  G[0] = 2.0f * mu * (g[0][0] - div_u * third);
  G[1] = mu * (g[0][1] + g[1][0]);
  G[2] = mu * (g[0][2] + g[2][0]);
  G[3] = 2.0f * mu * (g[1][1] - div_u * third);
  G[4] = mu * (g[1][2] + g[2][1]);
  G[5] = 2.0f * mu * (g[2][2] - div_u * third);
  G[6] = c0[0] * G[0] + c0[1] * G[1] + c0[2] * G[2] + kappa * g[3][0];
  G[7] = c0[0] * G[1] + c0[1] * G[3] + c0[2] * G[4] + kappa * g[3][1];
  G[8] = c0[0] * G[2] + c0[1] * G[4] + c0[2] * G[5] + kappa * g[3][2];
}

__device__ __forceinline__ void ld_rec12(const float* __restrict__ p, float* v) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float4 x = __ldg(reinterpret_cast<const float4*>(p) + i);
    v[4 * i] = x.x;
    v[4 * i + 1] = x.y;
    v[4 * i + 2] = x.z;
    v[4 * i + 3] = x.w;
  }
}

__device__ __forceinline__ void ld_row(const float* __restrict__ rec, int l, float k[3]) {
  k[0] = __ldg(rec + 3 * l);
  k[1] = __ldg(rec + 3 * l + 1);
  k[2] = __ldg(rec + 3 * l + 2);
}

// The primitives (rho, u, v, w, p - p_ref) of cell (i, j, k) into the padded
// array and its periodic images (physics/eos.py:12-17 in FP64, then FP32).
__device__ __forceinline__ void write_prims(float* __restrict__ dst, const TileBlock& B, int i, int j, int k,
                                            const double q[5], double gm1, double p_ref) {
  const double r = q[0];
  const double ir = __drcp_rn(r);
  const double u = q[1] * ir, v = q[2] * ir, w = q[3] * ir;
  const double p = gm1 * (q[4] - r * (0.5 * (u * u + v * v + w * w)));
  const float val[5] = {(float)r, (float)u, (float)v, (float)w, (float)(p - p_ref)};
  const int64_t fs = (int64_t)B.ni * B.njp * B.nkp;
  const int rows[2] = {j + 2, j < 2 ? j + 2 + B.nj : (j >= B.nj - 2 ? j + 2 - B.nj : -1)};
  const int cols[2] = {k + 2, k < 2 ? k + 2 + B.nk : (k >= B.nk - 2 ? k + 2 - B.nk : -1)};
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    if (rows[a] < 0) continue;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (cols[c] < 0) continue;
      const int64_t o = ((int64_t)i * B.njp + rows[a]) * B.nkp + cols[c];
#pragma unroll
      for (int f = 0; f < NF; ++f) dst[f * fs + o] = val[f];
    }
  }
}

__global__ void k_tile_prims(const TileBlock B, const double* __restrict__ q, float* __restrict__ dst, double gm1,
                             double p_ref) {
  grid_dep_wait();
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int k = (int)(c % B.nk);
  const int64_t t = c / B.nk;
  const int j = (int)(t % B.nj), i = (int)(t / B.nj);
  const double qc[5] = {q[c], q[N + c], q[2 * N + c], q[3 * N + c], q[4 * N + c]};
  write_prims(dst, B, i, j, k, qc, gm1, p_ref);
}

__global__ void __launch_bounds__(NT, 2) k_tile_stage(const __grid_constant__ TileParams P) {
  extern __shared__ unsigned char smem_raw[];
  grid_dep_wait();
  float* const base = (float*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  float* const Pr = base;
  float* const Gs = Pr + RS * PSLOT_STRIDE;
  float* const Sj = Gs + 4 * GSLOT;
  float* const Fj = Sj + 2 * SSLOT;
  uint64_t* const bar = (uint64_t*)(Fj + 2 * FSLOT);
  int* const fail = (int*)(bar + RS);
  const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < RS; ++s) mbar_init(bar + s);
    *fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const Phys& ph = P.ph;
  Consts C;
  C.gm1 = (float)ph.gm1;
  C.inv_gm1 = (float)ph.inv_gm1;
  C.eps = (float)ph.eps_entropy;
  C.p_ref = (float)ph.p_ref;
  C.R = (float)ph.R;
  C.inv_T0 = (float)ph.inv_T0;
  C.sfac = (float)ph.sfac;
  C.Ts = (float)ph.Ts;
  C.kap_fac = (float)ph.kap_fac;
  C.limiter = ph.limiter;
  C.visc_law = ph.visc_law;
  const int limit = P.wait_limit;
  const int stage = P.stage;
  const double ca = stage == 2 ? 0.75 : 1.0 / 3.0;
  const double cb = stage == 2 ? 0.25 : 2.0 / 3.0;

  uint32_t wpar = 0;   // per slot: parity of the next wait
  uint32_t ipar = 0;   // per slot (thread 0): parity of the loads issued
  uint32_t used = 0;   // per slot (thread 0): a load was ever issued
  bool stop = false;

  int* const item_sh = fail + 1;
  while (!stop) {
    // ---- next work item (segment, block, tile), segment slowest, so that the
    // CTAs busy at one time hold neighbouring tiles of the same plane range
    // and their halo rows meet in L2
    __syncthreads();  // the previous segment's readers of G / Fj and item_sh are done
    if (tid == 0) *item_sh = atomicAdd(P.next, 1);
    __syncthreads();
    const int item = *item_sh;
    if (item >= P.items) break;
    // blocks hold contiguous item ranges per segment: unit_begin is the block's
    // first item within a segment's range, ntj * ntk its tile count
    int seg = 0, b = 0, tile = 0;
    {
      int rem = item;
      for (seg = 0; seg < P.max_seg; ++seg) {
        int cnt = 0;
        for (int t = 0; t < P.nb; ++t)
          if (seg * P.seg_len < P.blk[t].ni) cnt += P.blk[t].ntj * P.blk[t].ntk;
        if (rem < cnt) break;
        rem -= cnt;
      }
      for (b = 0; b < P.nb; ++b) {
        if (seg * P.seg_len >= P.blk[b].ni) continue;
        const int cnt = P.blk[b].ntj * P.blk[b].ntk;
        if (rem < cnt) break;
        rem -= cnt;
      }
      tile = rem;
    }
    const TileBlock& B = P.blk[b];
    const CUtensorMap* map = &P.map[b];
    const int ib = seg * P.seg_len;
    const int ie = min(B.ni, ib + P.seg_len);
    const int ni = B.ni, nj = B.nj, nk = B.nk;
    const int jt = tile / B.ntk, kt = tile - jt * B.ntk;
    const int j0 = jt * TJ, k0 = kt * TK;
    const int nrows = min(TJ, nj - j0), ncols = min(TK, nk - k0);
    const int x0 = k0 & ~3, ko = k0 - x0;
    const int r = j0 + w;
    const bool row_ok = w < nrows;
    const int k = k0 - 1 + l;
    const bool lane_own = l >= 1 && l <= ncols;
    const bool own = row_ok && lane_own;
    const int by0 = w + 2, bx0 = l + 1 + ko;
    const int kc = wrap1(min(k, nk), nk);  // metric column (wrapped; clamped for unused lanes)
    const int64_t N = (int64_t)ni * nj * nk;
    const float mu0 = (float)B.mu0;
    const double dt = B.dt;
    // metric record of (plane x, own row, column kc): krow + x * kplane
    const int64_t kplane = (int64_t)nj * nk * 12;
    const float* const krow = B.kaos + ((int64_t)min(r, nj - 1) * nk + kc) * 12;

    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      for (int x = ib - 2; x <= min(ib + 1, ie + 1); ++x) {
        const int s = x & (RS - 1);
        tma_plane(Pr + s * PSLOT_STRIDE, map, bar + s, x0, j0, wrap1(x, ni));
        ipar ^= 1u << s;
        used |= 1u << s;
      }
    }

    F5 si{};                                    // i-slope of the own cell at plane p (A5: at p+1)
    float Fim[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // i-face (p-1 | p), set in A5 of plane p
    float Fip[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // i-face (p | p+1), set in A5 of plane p
    float Fk[5] = {0.f, 0.f, 0.f, 0.f, 0.f};   // k-face (k-1 | k) of plane p

    for (int p = ib - 2; p < ie; ++p) {
      // ---- the planes A(p) reads: p, p+1, p+2 ----------------------------
      bool ok = true;
      for (int x = (p == ib - 2 ? p : p + 2); x <= p + 2; ++x) {
        const int s = x & (RS - 1);
        ok = mbar_wait(bar + s, (wpar >> s) & 1u, limit) && ok;
        wpar ^= 1u << s;
      }
      if (!ok) atomicOr(fail, 1);
      const float* S0 = Pr + (p & (RS - 1)) * PSLOT_STRIDE;
      const float* S1 = Pr + ((p + 1) & (RS - 1)) * PSLOT_STRIDE;
      const float* S2 = Pr + ((p + 2) & (RS - 1)) * PSLOT_STRIDE;
      const bool full = p >= ib, pre1 = p >= ib - 1;
      const int pw = wrap1(p, ni), pw1 = wrap1(p + 1, ni);
      float* const Gn = Gs + ((p + 1) & 3) * GSLOT;           // G(p+1)
      float* const Sjn = Sj + ((p + 1) & 1) * SSLOT;          // j-slopes of plane p+1
      const float* const Sjc = Sj + (p & 1) * SSLOT;          // j-slopes of plane p
      float* const Fjc = Fj + (p & 1) * FSLOT;                // j-faces of plane p

      // own metric records of planes p and p+1 (rows 0, 1, 2: the face
      // normals; p+1: also G(p+1))
      float kp[12], kn[12];
      if (row_ok) {
        ld_rec12(krow + pw * kplane, kp);
        ld_rec12(krow + pw1 * kplane, kn);
      }
      // ---- A1: G(p+1) on the own row, every lane (lanes 0 / 31: k-halo) ----
      if (row_ok) {
        float Gv[9];
        visc_flux(S0, S1, S2, by0, bx0, kn, mu0, C, Gv);
#pragma unroll
        for (int c = 0; c < 9; ++c) Gn[(c * GR + w + 1) * GC + l] = Gv[c];
      }
      // ---- A2: k-slopes and the k-face on the left of each column ---------
      if (full && row_ok) {
        const F5 c = ldP(S0, by0, bx0), m = ldP(S0, by0, bx0 - 1), pp = ldP(S0, by0, bx0 + 1);
        const F5 sk = slope(m, c, pp, C.limiter);
        float kr[3] = {kp[6], kp[7], kp[8]}, kl[3];
        F5 skm;
#pragma unroll
        for (int f = 0; f < NF; ++f) skm.v[f] = __shfl_up_sync(0xffffffffu, sk.v[f], 1);
#pragma unroll
        for (int a = 0; a < 3; ++a) kl[a] = __shfl_up_sync(0xffffffffu, kr[a], 1);
#pragma unroll
        for (int v = 0; v < 5; ++v) Fk[v] = 0.f;
        // face (k-1 | k) exists for k-1 in [1, nk-3]
        if (l >= 1 && k - 1 >= 1 && k - 1 <= nk - 3) face_flux(m, skm, c, sk, kl, kr, C, Fk);
      }
      // ---- A3: j-slopes of plane p+1 on the own row ------------------------
      if (pre1 && own) {
        const F5 sj = slope(ldP(S1, by0 - 1, bx0), ldP(S1, by0, bx0), ldP(S1, by0 + 1, bx0), C.limiter);
#pragma unroll
        for (int f = 0; f < NF; ++f) Sjn[(f * GR + w + 1) * GC + l] = sj.v[f];
      }
      // ---- A4: the j-face (r | r+1) of plane p ------------------------------
      if (full && own && r >= 1 && r <= nj - 3) {
        F5 sL, sR;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          sL.v[f] = Sjc[(f * GR + w + 1) * GC + l];
          sR.v[f] = Sjc[(f * GR + w + 2) * GC + l];
        }
        const float kl[3] = {kp[3], kp[4], kp[5]};
        float kr[3];
        ld_row(krow + pw * kplane + nk * 12, 1, kr);
        float F[5];
        face_flux(ldP(S0, by0, bx0), sL, ldP(S0, by0 + 1, bx0), sR, kl, kr, C, F);
#pragma unroll
        for (int v = 0; v < 5; ++v) Fjc[(v * FR + w + 1) * GC + l] = F[v];
      }
      // ---- A5: i-slope of plane p+1 and the i-face (p | p+1) ----------------
      if (own) {
        const F5 a0 = ldP(S0, by0, bx0), a1 = ldP(S1, by0, bx0), a2 = ldP(S2, by0, bx0);
        const F5 sn = slope(a0, a1, a2, C.limiter);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          Fim[v] = Fip[v];  // (p-1 | p)
          Fip[v] = 0.f;
        }
        // face (p | p+1) exists for p in [1, ni-3]
        if (pre1 && p >= 1 && p <= ni - 3) {
          const float kl[3] = {kp[0], kp[1], kp[2]}, kr[3] = {kn[0], kn[1], kn[2]};
          face_flux(a0, si, a1, sn, kl, kr, C, Fip);
        }
        si = sn;
      }
      // ---- A6: the ring rows' work, rotated over the warps -------------------
      // e0 / e1: j-slopes of plane p+1 at rows j0-1 / j0+nrows; e2 / e3: G(p+1)
      // at those rows; e4: the j-face (j0-1 | j0) of plane p
      if (lane_own) {
        const int rot = p & (NW - 1);
#pragma unroll 1
        for (int e = 0; e < 5; ++e) {
          if (w != ((e + rot) & (NW - 1))) continue;
          const bool up = (e & 1) != 0;
          const int gr = up ? nrows + 1 : 0;   // G / Sj row
          const int by = gr + 1;               // box row
          const int rr = j0 - 1 + gr;          // block row (may be -1 or nj: periodic images)
          if (e < 2) {
            if (!pre1) continue;
            const F5 sj = slope(ldP(S1, by - 1, bx0), ldP(S1, by, bx0), ldP(S1, by + 1, bx0), C.limiter);
#pragma unroll
            for (int f = 0; f < NF; ++f) Sjn[(f * GR + gr) * GC + l] = sj.v[f];
          } else if (e < 4) {
            float kk[12];
            ld_rec12(B.kaos + (((int64_t)pw1 * nj + wrap1(rr, nj)) * nk + k) * 12, kk);
            float Gv[9];
            visc_flux(S0, S1, S2, by, bx0, kk, mu0, C, Gv);
#pragma unroll
            for (int c = 0; c < 9; ++c) Gn[(c * GR + gr) * GC + l] = Gv[c];
          } else {
            if (!full || j0 - 1 < 1 || j0 - 1 > nj - 3) continue;
            F5 sL, sR;
#pragma unroll
            for (int f = 0; f < NF; ++f) {
              sL.v[f] = Sjc[(f * GR + 0) * GC + l];
              sR.v[f] = Sjc[(f * GR + 1) * GC + l];
            }
            float kl[3], kr[3];
            ld_row(B.kaos + (((int64_t)pw * nj + j0 - 1) * nk + k) * 12, 1, kl);
            ld_row(B.kaos + (((int64_t)pw * nj + j0) * nk + k) * 12, 1, kr);
            float F[5];
            face_flux(ldP(S0, 1, bx0), sL, ldP(S0, 2, bx0), sR, kl, kr, C, F);
#pragma unroll
            for (int v = 0; v < 5; ++v) Fjc[(v * FR + 0) * GC + l] = F[v];
          }
        }
      }

      __syncthreads();
      if (*fail) {
        stop = true;
        break;
      }
      // ---- refill: the slot of plane p (no longer read) takes plane p+4 ----
      if (tid == 0 && p + 4 <= ie + 1) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const int x = p + 4, s = x & (RS - 1);
        tma_plane(Pr + s * PSLOT_STRIDE, map, bar + s, x0, j0, wrap1(x, ni));
        ipar ^= 1u << s;
        used |= 1u << s;
      }


      if (full) {
        // ---- B(p): assembly of plane p -------------------------------------
        float Fkr[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) Fkr[v] = __shfl_down_sync(0xffffffffu, Fk[v], 1);
        if (own) {
          const int64_t c = ((int64_t)p * nj + r) * nk + k;
          double qv[5], q0v[5];
#pragma unroll
          for (int v = 0; v < 5; ++v) qv[v] = B.q[v * N + c];
          if (stage >= 2) {
#pragma unroll
            for (int v = 0; v < 5; ++v) q0v[v] = B.q0[v * N + c];
          }
          const double vol = B.vol[c];
          float kk[12];
          ld_rec12(krow + pw * kplane, kk);
          double rv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
          const bool on_i = p >= 2 && p <= ni - 3, on_j = r >= 2 && r <= nj - 3, on_k = k >= 2 && k <= nk - 3;
          if (on_i || on_j || on_k) {
            const double ivd = __drcp_rn(vol + 1e-300);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
              float s = 0.f;
              if (on_i) s += Fip[v] - Fim[v];
              if (on_j) s += Fjc[(v * FR + w + 1) * GC + l] - Fjc[(v * FR + w) * GC + l];
              if (on_k) s += Fkr[v] - Fk[v];
              double ds = (double)s;
              // the p_ref n part the face fluxes left out (see roe_prim)
              if (v >= 1 && v <= 3) ds += ph.p_ref * (double)kk[8 + v];
              rv[v] = -ds * ivd;
            }
          }
          // viscous divergence: sum_l 0.5 kxyz[l][.] (G(c+e_l) - G(c-e_l))
          // (rhs/viscous.py:86-117), neighbour by neighbour
          const float* Gc = Gs + (p & 3) * GSLOT;
          const float* Gm = Gs + ((p - 1) & 3) * GSLOT;
          const float* Gp = Gs + ((p + 1) & 3) * GSLOT;
          float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int la = 0; la < 3; ++la) {
#pragma unroll
            for (int side = 0; side < 2; ++side) {
              const float* src;
              int row = w + 1, col = l;
              if (la == 0) src = side == 0 ? Gp : Gm;
              else if (la == 1) { src = Gc; row += side == 0 ? 1 : -1; }
              else { src = Gc; col += side == 0 ? 1 : -1; }
              float g[9];
#pragma unroll
              for (int cc = 0; cc < 9; ++cc) g[cc] = src[(cc * GR + row) * GC + col];
              const float sg = side == 0 ? 0.5f : -0.5f;
              const float m0 = sg * kk[3 * la], m1 = sg * kk[3 * la + 1], m2 = sg * kk[3 * la + 2];
              acc[0] += g[0] * m0 + g[1] * m1 + g[2] * m2;
              acc[1] += g[1] * m0 + g[3] * m1 + g[4] * m2;
              acc[2] += g[2] * m0 + g[4] * m1 + g[5] * m2;
              acc[3] += g[6] * m0 + g[7] * m1 + g[8] * m2;
            }
          }
#pragma unroll
          for (int e = 0; e < 4; ++e) rv[e + 1] += (double)acc[e];
          // TVD-RK3 combine (solver/step.py:45-53)
          double qn[5];
#pragma unroll
          for (int v = 0; v < 5; ++v) {
            const double t = qv[v] + dt * rv[v];
            qn[v] = stage == 1 ? t : ca * q0v[v] + cb * t;
            B.out[v * N + c] = qn[v];
          }
          if (B.prim_next) write_prims(B.prim_next, B, p, r, k, qn, ph.gm1, ph.p_ref);
        }
      }
    }
  }
  // ---- drain: no copy may be in flight when the CTA exits -------------------
  if (tid == 0) {
    bool ok = true;
    for (int s = 0; s < RS; ++s)
      if (used & (1u << s)) ok = mbar_wait(bar + s, ((ipar >> s) & 1u) ^ 1u, kDrainWaitLimit) && ok;
    if (*fail || !ok) atomicOr(P.err, *fail ? 1 : 2);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
    cudaGetLastError();
  });
  return fn;
}

int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cudaGetLastError();
  }
  return n;
}

}  // namespace

size_t tile_scratch_bytes(const fj_block* blocks, int nblocks) {
  size_t t = 0;
  for (int b = 0; b < nblocks; ++b) t += 2 * tile_prims_bytes(blocks[b].ni, blocks[b].nj, blocks[b].nk);
  return t;
}

bool tile_setup(const fj_block* blocks, int nblocks, void* scratch, TileMaps& tm) {
  tm.ok = false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encoder();
  if (!enc || !scratch) return false;
  // the kernel's dynamic shared memory (two CTAs per SM), set on the current
  // device at plan creation, never during a stream capture
  if (cudaFuncSetAttribute(k_tile_stage, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  // the error word lives apart from the scratch, which the halo fill reuses
  if (!tm.err) {
    if (cudaMalloc(&tm.err, 2 * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      tm.err = nullptr;
      return false;
    }
  }
  char* p = (char*)scratch;
  for (int w = 0; w < 2; ++w) {
    tm.map[w].assign(nblocks, {});
    tm.prim[w].assign(nblocks, nullptr);
  }
  for (int b = 0; b < nblocks; ++b) {
    const fj_block& B = blocks[b];
    for (int w = 0; w < 2; ++w) {
      tm.prim[w][b] = (float*)p;
      p += tile_prims_bytes(B.ni, B.nj, B.nk);
      const int njp = tile_njp(B.nj), nkp = tile_nkp(B.nk);
      const cuuint64_t dims[4] = {(cuuint64_t)nkp, (cuuint64_t)njp, (cuuint64_t)B.ni, 5};
      const cuuint64_t strides[3] = {(cuuint64_t)nkp * 4, (cuuint64_t)nkp * njp * 4,
                                     (cuuint64_t)nkp * njp * B.ni * 4};
      const cuuint32_t box[4] = {BW, BH, 1, NF};
      const cuuint32_t estr[4] = {1, 1, 1, 1};
      CUtensorMap m;
      const CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, tm.prim[w][b], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return false;
      static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
      std::memcpy(tm.map[w][b].data(), &m, sizeof(m));
    }
  }
  tm.ok = true;
  return true;
}

int tile_prims(fj_ctx* ctx, const TileMaps& tm, int which, const double* const* q, const fj_block* blocks,
               int nblocks, double gm1, double R, double p_ref, cudaStream_t st) {
  (void)R;
  for (int b = 0; b < nblocks; ++b) {
    TileBlock B{};
    B.ni = blocks[b].ni;
    B.nj = blocks[b].nj;
    B.nk = blocks[b].nk;
    B.njp = tile_njp(B.nj);
    B.nkp = tile_nkp(B.nk);
    const int64_t N = (int64_t)B.ni * B.nj * B.nk;
    pdl_launch(k_tile_prims, grid_for(N), kThreads, 0, st, B, q[b], tm.prim[which][b], gm1, p_ref);
    ctx->launches += 1;
  }
  return launch_status(ctx, "tile primitive launch");
}

int tile_stage(fj_ctx* ctx, const TileMaps& tm, int which, TileBlock* blocks, int nblocks, const Phys& ph,
               int stage, cudaStream_t st, int wait_limit) {
  for (int base = 0; base < nblocks; base += kTileMaxBlocks) {
    TileParams* prm = new (std::nothrow) TileParams();
    if (!prm) return FJ_ERR_NO_MEMORY;
    prm->nb = std::min(kTileMaxBlocks, nblocks - base);
    int64_t tiles = 0;
    int max_ni = 0;
    for (int t = 0; t < prm->nb; ++t) {
      TileBlock& B = prm->blk[t];
      B = blocks[base + t];
      B.njp = tile_njp(B.nj);
      B.nkp = tile_nkp(B.nk);
      B.ntj = (B.nj + TJ - 1) / TJ;
      B.ntk = (B.nk + TK - 1) / TK;
      B.prim_next = stage < 3 ? tm.prim[1 - which][base + t] : nullptr;
      tiles += (int64_t)B.ntj * B.ntk;
      max_ni = std::max(max_ni, B.ni);
      std::memcpy(&prm->map[t], tm.map[which][base + t].data(), sizeof(CUtensorMap));
    }
    // persistent grid of two CTAs per SM; segments of about 24..48 planes,
    // fewer (longer) when that already gives every CTA several items
    const int grid_max = 2 * num_sms();
    int seg = max_ni;
    while (seg > 24 && tiles * ((max_ni + seg - 1) / seg) < 4 * (int64_t)grid_max) seg = (seg + 1) / 2;
    int64_t items = 0;
    const int max_seg = (max_ni + seg - 1) / seg;
    for (int t = 0; t < prm->nb; ++t)
      items += (int64_t)prm->blk[t].ntj * prm->blk[t].ntk * ((prm->blk[t].ni + seg - 1) / seg);
    prm->ph = ph;
    prm->err = tm.err;
    prm->next = tm.err + 1;
    prm->stage = stage;
    prm->wait_limit = wait_limit < 0 ? kDefaultWaitLimit : wait_limit;
    prm->seg_len = seg;
    prm->max_seg = max_seg;
    prm->items = (int)items;
    const int64_t g = std::min<int64_t>(grid_max, std::max<int64_t>(1, items));
    int s = cuda_status(ctx, cudaMemsetAsync(prm->next, 0, sizeof(int), st), "tile work counter");
    if (s != FJ_OK) {
      delete prm;
      return s;
    }
    pdl_launch(k_tile_stage, (int)g, NT, kSmemBytes, st, *prm);
    delete prm;
    ctx->launches += 1;
    s = launch_status(ctx, "tile stage launch");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

int tile_read_error(const TileMaps& tm, int* out, cudaStream_t st) {
  if (!tm.err) return FJ_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaMemcpyAsync(out, tm.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

int tile_clear_error(const TileMaps& tm, cudaStream_t st) {
  if (!tm.err) return FJ_ERR_INVALID_ARGUMENT;
  return cudaMemsetAsync(tm.err, 0, sizeof(int), st) == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

}  // namespace fj

namespace fj {
TileMaps::~TileMaps() {
  if (err) cudaFree(err);
}
}  // namespace fj
