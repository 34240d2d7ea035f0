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
// path, double on the FP64 path): 6 primitives + 15 face-flux + 9 viscous
// components per cell.  Each launch covers every block of a table; a CTA
// handles 256 consecutive cells of one block, and neighbours are read through
// L1/L2 (consecutive threads touch consecutive cells).
#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_rhs.cuh"
#include "fj_split.cuh"

namespace fj {

namespace {

constexpr int kSplitThreads = 256;

// Division of a non-negative int by a run-time constant (multiply-high form).
struct FastDiv {
  uint32_t d, m, s;
  __host__ void init(uint32_t dd) {
    d = dd;
    s = 0;
    while ((1u << s) < d) ++s;
    m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << s) - d)) / d + 1);
  }
  __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi(n, m) + n) >> s; }
};

struct Dev {
  SplitBlock blk;
  FastDiv dk, dj;  // n / nk, n / nj
};

struct Table {
  int n;
  Dev b[kMaxSplitBlocks];
};

// Locates the block of CTA `cta` (blocks own contiguous CTA ranges).
__device__ __forceinline__ int find_block(const Table& t, int cta) {
  int b = 0;
  while (b + 1 < t.n && t.b[b + 1].blk.cta_begin <= cta) ++b;
  return b;
}

struct Cell {
  int i, j, k;
  int64_t c, N;
  int ni, nj, nk;
};

__device__ __forceinline__ bool decode(const Dev& d, int cta, Cell& x) {
  const SplitBlock& B = d.blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c = (int64_t)(cta - B.cta_begin) * kSplitThreads + threadIdx.x;
  if (c >= N) return false;
  const uint32_t t1 = d.dk.div((uint32_t)c);
  x.k = (int)((uint32_t)c - t1 * (uint32_t)B.nk);
  x.i = (int)d.dj.div(t1);
  x.j = (int)(t1 - (uint32_t)x.i * (uint32_t)B.nj);
  x.c = c;
  x.N = N;
  x.ni = B.ni;
  x.nj = B.nj;
  x.nk = B.nk;
  return true;
}

template <typename T>
__global__ void __launch_bounds__(kSplitThreads) k_split_prims(const Table tab, const double gm1,
                                                              const double R) {
  const int b = find_block(tab, blockIdx.x);
  const SplitBlock& B = tab.b[b].blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c = (int64_t)(blockIdx.x - B.cta_begin) * kSplitThreads + threadIdx.x;
  if (c >= N) return;
  const double* q = B.q;
  const double r = q[c];
  const double ir = 1.0 / r;
  const double u = q[N + c] * ir, v = q[2 * N + c] * ir, w = q[3 * N + c] * ir;
  const double p = gm1 * (q[4 * N + c] - r * (0.5 * (u * u + v * v + w * w)));
  const double Tt = r * R > 1e-300 ? p * ir * (1.0 / R) : p * 1e300;
  T* P = (T*)B.prim;
  P[c] = (T)r;
  P[N + c] = (T)u;
  P[2 * N + c] = (T)v;
  P[3 * N + c] = (T)w;
  P[4 * N + c] = (T)p;
  P[5 * N + c] = (T)Tt;
}

template <typename T>
__device__ __forceinline__ T metric(const SplitBlock& B, int64_t N, int lm, int64_t c) {
  return B.kxyz32 ? (T)__ldg(B.kxyz32 + lm * N + c) : (T)__ldg(B.kxyz + lm * N + c);
}

template <typename T>
__global__ void __launch_bounds__(kSplitThreads) k_split_fluxes(const Table tab, const Phys ph,
                                                               const int flags) {
  using M = FastMath<T>;
  const int b = find_block(tab, blockIdx.x);
  Cell x;
  if (!decode(tab.b[b], blockIdx.x, x)) return;
  const SplitBlock& B = tab.b[b].blk;
  const int64_t N = x.N, c = x.c;
  const int64_t si = (int64_t)x.nj * x.nk, sj = x.nk;
  const T* P = (const T*)B.prim;
  const int n[3] = {x.ni, x.nj, x.nk};
  const int idx[3] = {x.i, x.j, x.k};
  const int64_t st[3] = {si, sj, 1};

  if (flags & kRhsViscous) {
    // viscous flux components at c (rhs/viscous.py:36-105)
    int64_t cp[3], cm[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      cp[l] = idx[l] + 1 == n[l] ? c - (int64_t)(n[l] - 1) * st[l] : c + st[l];
      cm[l] = idx[l] == 0 ? c + (int64_t)(n[l] - 1) * st[l] : c - st[l];
    }
    T d[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int64_t o = (int64_t)(s < 3 ? s + 1 : 5) * N;  // u, v, w, T
#pragma unroll
      for (int l = 0; l < 3; ++l) d[s][l] = T(0.5) * (P[o + cp[l]] - P[o + cm[l]]);
    }
    T kk[9];
#pragma unroll
    for (int lm = 0; lm < 9; ++lm) kk[lm] = metric<T>(B, N, lm, c);
    T g[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[m] + d[s][1] * kk[3 + m] + d[s][2] * kk[6 + m];
    const T u = P[N + c], v = P[2 * N + c], w = P[3 * N + c];
    T mu = (T)ph.mu0;
    if (ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
      const T Tt = P[5 * N + c];
      const T r = Tt * (T)(1.0 / ph.T0);
      mu = (T)ph.mu0 * (r * M::sqrt_pos(r)) * (T)(ph.T0 + ph.Ts) * M::rcp(Tt + (T)ph.Ts);
    }
    const T kappa = (T)(ph.cp / ph.Pr) * mu;
    const T third = (T)(1.0 / 3.0);
    const T div_u = g[0][0] + g[1][1] + g[2][2];
    const T t00 = T(2) * mu * (g[0][0] - div_u * third);
    const T t01 = mu * (g[0][1] + g[1][0]);
    const T t02 = mu * (g[0][2] + g[2][0]);
    const T t11 = T(2) * mu * (g[1][1] - div_u * third);
    const T t12 = mu * (g[1][2] + g[2][1]);
    const T t22 = T(2) * mu * (g[2][2] - div_u * third);
    T* G = (T*)B.G;
    G[c] = t00;
    G[N + c] = t01;
    G[2 * N + c] = t02;
    G[3 * N + c] = t11;
    G[4 * N + c] = t12;
    G[5 * N + c] = t22;
    G[6 * N + c] = u * t00 + v * t01 + w * t02 + kappa * g[3][0];
    G[7 * N + c] = u * t01 + v * t11 + w * t12 + kappa * g[3][1];
    G[8 * N + c] = u * t02 + v * t12 + w * t22 + kappa * g[3][2];
  }
  if (flags & kRhsInvscd) {
    const T gm1 = (T)ph.gm1, inv_gm1 = (T)(1.0 / ph.gm1), eps_e = (T)ph.eps_entropy;
    T* F = (T*)B.F;
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
      // face c | c+e_a (face index c_a - 1 of rhs/invscd.py:62-100)
      if (idx[a] < 1 || idx[a] > n[a] - 3) continue;
      Prim<T> cell[4];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int64_t cc = c + (int64_t)(s - 1) * st[a];
        cell[s].rho = P[cc];
        cell[s].u = P[N + cc];
        cell[s].v = P[2 * N + cc];
        cell[s].w = P[3 * N + cc];
        cell[s].p = P[4 * N + cc];
      }
      const int64_t cr = c + st[a];
      T Fo[5];
      invscd_face_fast<T>(cell, metric<T>(B, N, 3 * a, c), metric<T>(B, N, 3 * a + 1, c),
                          metric<T>(B, N, 3 * a + 2, c), metric<T>(B, N, 3 * a, cr),
                          metric<T>(B, N, 3 * a + 1, cr), metric<T>(B, N, 3 * a + 2, cr), gm1, inv_gm1,
                          eps_e, ph.limiter, Fo);
#pragma unroll
      for (int v = 0; v < 5; ++v) F[(int64_t)(a * 5 + v) * N + c] = Fo[v];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kSplitThreads) k_split_assemble(const Table tab, const int flags,
                                                                 const int stage, const double dt) {
  const int b = find_block(tab, blockIdx.x);
  Cell x;
  if (!decode(tab.b[b], blockIdx.x, x)) return;
  const SplitBlock& B = tab.b[b].blk;
  const int64_t N = x.N, c = x.c;
  const int64_t si = (int64_t)x.nj * x.nk, sj = x.nk;
  const int n[3] = {x.ni, x.nj, x.nk};
  const int idx[3] = {x.i, x.j, x.k};
  const int64_t st[3] = {si, sj, 1};
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (flags & kRhsInvscd) {
    const T* F = (const T*)B.F;
    const double ivd = 1.0 / (B.vol[c] + 1e-300);
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
            const T* Fa = F + (int64_t)(a * 5 + v) * N;
            dsum += (double)(Fa[c] - Fa[c - st[a]]);
          }
      } else {
        T s = T(0);
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (on[a]) {
            const T* Fa = F + (int64_t)(a * 5 + v) * N;
            s += Fa[c] - Fa[c - st[a]];
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
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const int64_t o = v * N + c;
      const double t = B.q[o] + dt * r[v];
      B.out[o] = stage == 1 ? t : ca * B.q0[o] + cb * t;
    }
  }
}

template <typename T>
int launch_split(fj_ctx* ctx, const SplitBlock* blocks, int nblocks, const Phys& ph, int flags,
                 int stage, double dt, cudaStream_t st) {
  for (int base = 0; base < nblocks; base += kMaxSplitBlocks) {
    Table tab;
    tab.n = std::min(kMaxSplitBlocks, nblocks - base);
    int ctas = 0;
    for (int t = 0; t < tab.n; ++t) {
      tab.b[t].blk = blocks[base + t];
      tab.b[t].blk.cta_begin = ctas;
      tab.b[t].dk.init((uint32_t)blocks[base + t].nk);
      tab.b[t].dj.init((uint32_t)blocks[base + t].nj);
      const int64_t N = (int64_t)blocks[base + t].ni * blocks[base + t].nj * blocks[base + t].nk;
      ctas += (int)((N + kSplitThreads - 1) / kSplitThreads);
    }
    k_split_prims<T><<<ctas, kSplitThreads, 0, st>>>(tab, ph.gm1, ph.R);
    k_split_fluxes<T><<<ctas, kSplitThreads, 0, st>>>(tab, ph, flags);
    k_split_assemble<T><<<ctas, kSplitThreads, 0, st>>>(tab, flags, stage, dt);
    ctx->launches += 3;
    int s = launch_status(ctx, "split stage launch");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

}  // namespace

size_t split_scratch_bytes(int precision, int64_t cells) {
  const size_t t = precision == FJ_PREC_F32FLUX ? sizeof(float) : sizeof(double);
  return (size_t)(6 + 15 + 9) * (size_t)cells * t + 3 * 256;
}

void split_assign_scratch(int precision, SplitBlock* blocks, int nblocks, void* scratch) {
  const size_t t = precision == FJ_PREC_F32FLUX ? sizeof(float) : sizeof(double);
  char* p = (char*)scratch;
  auto al = [](char* x) { return (char*)(((uintptr_t)x + 255) & ~(uintptr_t)255); };
  int64_t total = 0;
  for (int b = 0; b < nblocks; ++b) total += (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
  char* prim = al(p);
  char* F = al(prim + 6 * total * t);
  char* G = al(F + 15 * total * t);
  int64_t off = 0;
  for (int b = 0; b < nblocks; ++b) {
    const int64_t N = (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
    blocks[b].prim = prim + 6 * off * t;
    blocks[b].F = F + 15 * off * t;
    blocks[b].G = G + 9 * off * t;
    off += N;
  }
}

int split_stage(fj_ctx* ctx, const SplitBlock* blocks, int nblocks, const Phys& ph, int flags,
                int stage, double dt, int precision, cudaStream_t st) {
  if (precision == FJ_PREC_F32FLUX)
    return launch_split<float>(ctx, blocks, nblocks, ph, flags, stage, dt, st);
  return launch_split<double>(ctx, blocks, nblocks, ph, flags, stage, dt, st);
}

}  // namespace fj
