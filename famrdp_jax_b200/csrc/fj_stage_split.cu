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

// Primitives (rho, u, v, w, p[, T]) of one cell from the field-major scratch.
template <typename T>
struct Cell6 {
  T r, u, v, w, p, t;
};

template <typename T, bool WITH_T>
__device__ __forceinline__ Cell6<T> load_cell(const T* __restrict__ P, int32_t N, int32_t c) {
  Cell6<T> x;
  x.r = P[c];
  x.u = P[N + c];
  x.v = P[2 * N + c];
  x.w = P[3 * N + c];
  x.p = P[4 * N + c];
  x.t = WITH_T ? P[5 * N + c] : T(0);
  return x;
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
  if (B.kxyz32) {
    const float* K = B.kxyz32 + 3 * row * N;
    k[0] = (T)__ldg(K + c);
    k[1] = (T)__ldg(K + N + c);
    k[2] = (T)__ldg(K + 2 * N + c);
  } else {
    const double* K = B.kxyz + 3 * row * N;
    k[0] = (T)__ldg(K + c);
    k[1] = (T)__ldg(K + N + c);
    k[2] = (T)__ldg(K + 2 * N + c);
  }
}

template <typename T>
__global__ void __launch_bounds__(kSplitThreads) k_split_fluxes(const Table tab, const Phys ph,
                                                               const int flags) {
  using M = FastMath<T>;
  const int b = find_block(tab, blockIdx.x);
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
    T mu = (T)ph.mu0;
    if (ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
      const T r = C0.t * (T)ph.inv_T0;
      mu = (T)ph.mu0 * (r * M::sqrt_pos(r)) * (T)ph.sfac * M::rcp(C0.t + (T)ph.Ts);
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
    if (x.k >= 1 && x.k <= x.nk - 3) {
      const Cell6<T> K2 = load_cell<T, false>(P, N, c + 2);
      metric_row<T>(B, N, 2, c, kc);
      metric_row<T>(B, N, 2, c + 1, kn);
      face_from_cells<T>(Km, C0, Kp, K2, kc, kn, ph, Fo);
#pragma unroll
      for (int v = 0; v < 5; ++v) F[(10 + v) * N + c] = Fo[v];
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
      // the kernels index the 15 face-flux fields with 32-bit offsets
      if (15 * (int64_t)blocks[base + t].ni * blocks[base + t].nj * blocks[base + t].nk > INT32_MAX)
        return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block too large for the split pipeline");
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
