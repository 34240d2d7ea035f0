// fj_rhs_staged.cu -- the staged RHS pipeline of one block: the reference's
// RHS (rhs/invscd.py:18-133 + rhs/viscous.py:19-119) as four kernel kinds that
// pass primitives, viscous fluxes and face fluxes through scratch memory:
//
//   k_prim      q -> primitives pv (every padded cell)            eos.py:12-17
//   k_vflux     pv, kxyz -> viscous flux components G (every cell) viscous.py:36-105
//   k_iflux<a>  pv, kxyz -> Roe face flux * |n| along axis a       invscd.py:53-100
//   k_combine   face-flux differences / vol + viscous divergence
//               (+ the RK3 stage combine of solver/step.py:45-53)  invscd.py:119-131
//                                                                  viscous.py:86-117
//
// It is the straightforward decomposition, kept as the cross-check of the
// fused stage kernel (fj_stage_fused.cu) and as the general fallback for
// blocks the fused kernels do not tile.
#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_rhs.cuh"

namespace fj {

template <typename T>
__global__ void k_prim(const double* __restrict__ q, T* __restrict__ pv, int N, double gm1) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  Prim<double> p = cons_to_prim<double>(q[c], q[(int64_t)N + c], q[2 * (int64_t)N + c],
                                        q[3 * (int64_t)N + c], q[4 * (int64_t)N + c], gm1);
  pv[c] = (T)p.rho;
  pv[(int64_t)N + c] = (T)p.u;
  pv[2 * (int64_t)N + c] = (T)p.v;
  pv[3 * (int64_t)N + c] = (T)p.w;
  pv[4 * (int64_t)N + c] = (T)p.p;
}

// rhs/viscous.py:36-105 at one padded cell.  Neighbours wrap around the padded
// array (jnp.roll, :12-16).  G = [t00 t01 t02 t11 t12 t22 Ge0 Ge1 Ge2].
template <typename T>
__global__ void k_vflux(const T* __restrict__ pv, const double* __restrict__ kxyz,
                        T* __restrict__ G, int ni, int nj, int nk, Phys ph) {
  const int N = ni * nj * nk;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int k = c % nk;
  const int j = (c / nk) % nj;
  const int i = c / (nk * nj);
  const int sj = nk, si = nj * nk;
  // neighbour offsets with wrap
  const int cip = (i + 1 == ni) ? c - (ni - 1) * si : c + si;
  const int cim = (i == 0) ? c + (ni - 1) * si : c - si;
  const int cjp = (j + 1 == nj) ? c - (nj - 1) * sj : c + sj;
  const int cjm = (j == 0) ? c + (nj - 1) * sj : c - sj;
  const int ckp = (k + 1 == nk) ? c - (nk - 1) : c + 1;
  const int ckm = (k == 0) ? c + (nk - 1) : c - 1;
  const int nb[6] = {cip, cim, cjp, cjm, ckp, ckm};

  const T R = (T)ph.R;
  auto temp = [&](int cc) {
    T rho = pv[cc];
    T p = pv[4 * (int64_t)N + cc];
    return p / fj_max(rho * R, Tiny<T>::rho());
  };
  // d/dxi_l of u, v, w, T (0.5*(f[+1] - f[-1]))
  T d[4][3];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    const int cp = nb[2 * l], cm = nb[2 * l + 1];
#pragma unroll
    for (int s = 0; s < 3; ++s)
      d[s][l] = T(0.5) * (pv[(int64_t)(s + 1) * N + cp] - pv[(int64_t)(s + 1) * N + cm]);
    d[3][l] = T(0.5) * (temp(cp) - temp(cm));
  }
  T kk[3][3];
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) kk[l][m] = (T)kxyz[(int64_t)(l * 3 + m) * N + c];
  // physical gradients (einsum "lijk,lmijk->mijk")
  T g[4][3];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[0][m] + d[s][1] * kk[1][m] + d[s][2] * kk[2][m];

  const T u = pv[(int64_t)N + c], v = pv[2 * (int64_t)N + c], w = pv[3 * (int64_t)N + c];
  const T Tc = temp(c);
  const T mu = viscosity<T>(Tc, ph.visc_law, (T)ph.mu0, (T)ph.T0, (T)ph.Ts);
  const T kappa = (T)ph.cp * mu / (T)ph.Pr;
  const T div_u = g[0][0] + g[1][1] + g[2][2];
  const T t00 = T(2) * mu * (g[0][0] - div_u / T(3));
  const T t01 = mu * (g[0][1] + g[1][0]);
  const T t02 = mu * (g[0][2] + g[2][0]);
  const T t11 = T(2) * mu * (g[1][1] - div_u / T(3));
  const T t12 = mu * (g[1][2] + g[2][1]);
  const T t22 = T(2) * mu * (g[2][2] - div_u / T(3));
  const T h0 = -kappa * g[3][0], h1 = -kappa * g[3][1], h2 = -kappa * g[3][2];
  const T ge0 = u * t00 + v * t01 + w * t02 - h0;
  const T ge1 = u * t01 + v * t11 + w * t12 - h1;
  const T ge2 = u * t02 + v * t12 + w * t22 - h2;
  G[c] = t00;
  G[(int64_t)N + c] = t01;
  G[2 * (int64_t)N + c] = t02;
  G[3 * (int64_t)N + c] = t11;
  G[4 * (int64_t)N + c] = t12;
  G[5 * (int64_t)N + c] = t22;
  G[6 * (int64_t)N + c] = ge0;
  G[7 * (int64_t)N + c] = ge1;
  G[8 * (int64_t)N + c] = ge2;
}

// One Roe face per thread along axis AX (0 = i, 1 = j, 2 = k).  Faces f in
// [0, n_AX - 4] lie between cells f+1 and f+2; every index of the other two
// axes is a face row (rhs/invscd.py:62-100).
template <typename T, int AX>
__global__ void k_iflux(const T* __restrict__ pv, const double* __restrict__ kxyz,
                        T* __restrict__ F, int ni, int nj, int nk, Phys ph) {
  const int N = ni * nj * nk;
  const int fi = ni - (AX == 0 ? 3 : 0), fj = nj - (AX == 1 ? 3 : 0), fk = nk - (AX == 2 ? 3 : 0);
  const int NF = fi * fj * fk;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NF) return;
  const int k = t % fk;
  const int j = (t / fk) % fj;
  const int i = t / (fk * fj);
  const int stride = AX == 0 ? nj * nk : (AX == 1 ? nk : 1);
  const int c0 = i * nj * nk + j * nk + k;  // face f -> cell f (the first of c0..c3)
  Prim<T> cell[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int cc = c0 + s * stride;
    cell[s].rho = pv[cc];
    cell[s].u = pv[(int64_t)N + cc];
    cell[s].v = pv[2 * (int64_t)N + cc];
    cell[s].w = pv[3 * (int64_t)N + cc];
    cell[s].p = pv[4 * (int64_t)N + cc];
  }
  const int cl = c0 + stride, cr = c0 + 2 * stride;
  const double* ka = kxyz + (int64_t)(AX * 3) * N;
  T Fo[5];
  invscd_face<T>(cell, (T)ka[cl], (T)ka[(int64_t)N + cl], (T)ka[2 * (int64_t)N + cl], (T)ka[cr],
                 (T)ka[(int64_t)N + cr], (T)ka[2 * (int64_t)N + cr], (T)ph.gm1,
                 (T)ph.eps_entropy, ph.limiter, Fo);
#pragma unroll
  for (int v = 0; v < 5; ++v) F[(int64_t)v * NF + t] = Fo[v];
}

__device__ __forceinline__ int sym_index(int a, int b) {
  // (0,0)->0 (0,1)->1 (0,2)->2 (1,1)->3 (1,2)->4 (2,2)->5
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

// Per-cell assembly: inviscid face differences (rhs/invscd.py:119-131, axis
// order i, j, k, only at cells [2, n-3] along each axis), the viscous
// divergence (rhs/viscous.py:86-117, wrapped central differences of G with
// the cell's own kxyz), their sum (solver/step.py:15) and the RK3 combine.
template <typename T>
__global__ void k_combine(const T* __restrict__ Fi, const T* __restrict__ Fj,
                          const T* __restrict__ Fk, const T* __restrict__ G,
                          const double* __restrict__ kxyz, const double* __restrict__ vol,
                          const double* __restrict__ qs, const double* __restrict__ q0,
                          double* __restrict__ out, int ni, int nj, int nk, int flags,
                          int stage, double dt) {
  const int N = ni * nj * nk;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int k = c % nk;
  const int j = (c / nk) % nj;
  const int i = c / (nk * nj);
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (flags & kRhsInvscd) {
    const double vd = vol[c] + 1e-300;
    if (i >= 2 && i <= ni - 3) {
      const int NF = (ni - 3) * nj * nk;
      const int fR = (i - 1) * nj * nk + j * nk + k, fL = fR - nj * nk;
#pragma unroll
      for (int v = 0; v < 5; ++v)
        r[v] += -((double)Fi[(int64_t)v * NF + fR] - (double)Fi[(int64_t)v * NF + fL]) / vd;
    }
    if (j >= 2 && j <= nj - 3) {
      const int NF = ni * (nj - 3) * nk;
      const int fR = i * (nj - 3) * nk + (j - 1) * nk + k, fL = fR - nk;
#pragma unroll
      for (int v = 0; v < 5; ++v)
        r[v] += -((double)Fj[(int64_t)v * NF + fR] - (double)Fj[(int64_t)v * NF + fL]) / vd;
    }
    if (k >= 2 && k <= nk - 3) {
      const int NF = ni * nj * (nk - 3);
      const int fR = i * nj * (nk - 3) + j * (nk - 3) + (k - 1), fL = fR - 1;
#pragma unroll
      for (int v = 0; v < 5; ++v)
        r[v] += -((double)Fk[(int64_t)v * NF + fR] - (double)Fk[(int64_t)v * NF + fL]) / vd;
    }
  }
  if (flags & kRhsViscous) {
    const int sj = nk, si = nj * nk;
    const int nb[6] = {(i + 1 == ni) ? c - (ni - 1) * si : c + si,
                       (i == 0) ? c + (ni - 1) * si : c - si,
                       (j + 1 == nj) ? c - (nj - 1) * sj : c + sj,
                       (j == 0) ? c + (nj - 1) * sj : c - sj,
                       (k + 1 == nk) ? c - (nk - 1) : c + 1,
                       (k == 0) ? c + (nk - 1) : c - 1};
    T kk[3][3];
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m) kk[l][m] = (T)kxyz[(int64_t)(l * 3 + m) * N + c];
    // rows 0..2: momentum (tau row), row 3: energy
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      T res = T(0);
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) {
        const int gi = e < 3 ? sym_index(e, jj) : 6 + jj;
        const T* Gc = G + (int64_t)gi * N;
        T s = T(0);
#pragma unroll
        for (int l = 0; l < 3; ++l) s = s + T(0.5) * (Gc[nb[2 * l]] - Gc[nb[2 * l + 1]]) * kk[l][jj];
        res = res + s;
      }
      r[e + 1] += (double)res;
    }
  }
  if (stage == 0) {
#pragma unroll
    for (int v = 0; v < 5; ++v) out[(int64_t)v * N + c] = r[v];
    return;
  }
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const int64_t o = (int64_t)v * N + c;
    const double t = qs[o] + dt * r[v];
    double res;
    if (stage == 1)
      res = t;
    else if (stage == 2)
      res = 0.75 * q0[o] + 0.25 * t;
    else
      res = (1.0 / 3.0) * q0[o] + (2.0 / 3.0) * t;
    out[o] = res;
  }
}

template <typename T>
size_t staged_ws_bytes(int ni, int nj, int nk) {
  const size_t N = (size_t)ni * nj * nk;
  const size_t fI = (size_t)(ni - 3) * nj * nk, fJ = (size_t)ni * (nj - 3) * nk,
               fK = (size_t)ni * nj * (nk - 3);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return al(5 * N * sizeof(T)) + al(9 * N * sizeof(T)) + al(5 * fI * sizeof(T)) +
         al(5 * fJ * sizeof(T)) + al(5 * fK * sizeof(T));
}

template <typename T>
int staged_rhs(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
               const double* q0, double* out, int ni, int nj, int nk, const Phys& ph,
               int flags, int stage, double dt, void* ws, cudaStream_t st) {
  const int N = ni * nj * nk;
  const size_t fI = (size_t)(ni - 3) * nj * nk, fJ = (size_t)ni * (nj - 3) * nk,
               fK = (size_t)ni * nj * (nk - 3);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  char* p = (char*)ws;
  T* pv = (T*)p;  p += al(5 * (size_t)N * sizeof(T));
  T* G = (T*)p;   p += al(9 * (size_t)N * sizeof(T));
  T* Fi = (T*)p;  p += al(5 * fI * sizeof(T));
  T* Fj = (T*)p;  p += al(5 * fJ * sizeof(T));
  T* Fk = (T*)p;
  k_prim<T><<<grid_for(N), kThreads, 0, st>>>(q, pv, N, ph.gm1);
  ctx->launches += 2;
  if (flags & kRhsViscous) {
    k_vflux<T><<<grid_for(N), kThreads, 0, st>>>(pv, kxyz, G, ni, nj, nk, ph);
    ctx->launches += 1;
  }
  if (flags & kRhsInvscd) {
    k_iflux<T, 0><<<grid_for(fI), kThreads, 0, st>>>(pv, kxyz, Fi, ni, nj, nk, ph);
    k_iflux<T, 1><<<grid_for(fJ), kThreads, 0, st>>>(pv, kxyz, Fj, ni, nj, nk, ph);
    k_iflux<T, 2><<<grid_for(fK), kThreads, 0, st>>>(pv, kxyz, Fk, ni, nj, nk, ph);
    ctx->launches += 3;
  }
  k_combine<T><<<grid_for(N), kThreads, 0, st>>>(Fi, Fj, Fk, G, kxyz, vol, q, q0, out, ni, nj,
                                                 nk, flags, stage, dt);
  return launch_status(ctx, "staged rhs launch");
}

// The same RHS launch sequence without a context (no launch counting, no
// error text): used by the entry point whose scratch is a static device array.
template <typename T>
cudaError_t staged_rhs_noctx(const double* q, const double* kxyz, const double* vol,
                             double* out, int ni, int nj, int nk, const Phys& ph, void* ws,
                             cudaStream_t st) {
  const int N = ni * nj * nk;
  const size_t fI = (size_t)(ni - 3) * nj * nk, fJ = (size_t)ni * (nj - 3) * nk,
               fK = (size_t)ni * nj * (nk - 3);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  char* p = (char*)ws;
  T* pv = (T*)p;  p += al(5 * (size_t)N * sizeof(T));
  T* G = (T*)p;   p += al(9 * (size_t)N * sizeof(T));
  T* Fi = (T*)p;  p += al(5 * fI * sizeof(T));
  T* Fj = (T*)p;  p += al(5 * fJ * sizeof(T));
  T* Fk = (T*)p;
  k_prim<T><<<grid_for(N), kThreads, 0, st>>>(q, pv, N, ph.gm1);
  k_vflux<T><<<grid_for(N), kThreads, 0, st>>>(pv, kxyz, G, ni, nj, nk, ph);
  k_iflux<T, 0><<<grid_for(fI), kThreads, 0, st>>>(pv, kxyz, Fi, ni, nj, nk, ph);
  k_iflux<T, 1><<<grid_for(fJ), kThreads, 0, st>>>(pv, kxyz, Fj, ni, nj, nk, ph);
  k_iflux<T, 2><<<grid_for(fK), kThreads, 0, st>>>(pv, kxyz, Fk, ni, nj, nk, ph);
  k_combine<T><<<grid_for(N), kThreads, 0, st>>>(Fi, Fj, Fk, G, kxyz, vol, q, nullptr, out, ni,
                                                 nj, nk, kRhsInvscd | kRhsViscous, 0, 0.0);
  return cudaGetLastError();
}

template cudaError_t staged_rhs_noctx<double>(const double*, const double*, const double*,
                                              double*, int, int, int, const Phys&, void*,
                                              cudaStream_t);
template cudaError_t staged_rhs_noctx<float>(const double*, const double*, const double*,
                                             double*, int, int, int, const Phys&, void*,
                                             cudaStream_t);

template size_t staged_ws_bytes<double>(int, int, int);
template size_t staged_ws_bytes<float>(int, int, int);
template int staged_rhs<double>(fj_ctx*, const double*, const double*, const double*,
                                const double*, double*, int, int, int, const Phys&, int, int,
                                double, void*, cudaStream_t);
template int staged_rhs<float>(fj_ctx*, const double*, const double*, const double*,
                               const double*, double*, int, int, int, const Phys&, int, int,
                               double, void*, cudaStream_t);

}  // namespace fj
