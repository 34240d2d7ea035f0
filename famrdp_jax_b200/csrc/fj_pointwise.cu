// fj_pointwise.cu -- the per-cell / per-face building blocks of the hot path
// exposed on their own (EOS, MUSCL-2, Roe, the RK3 combine), running the same
// device functions the RHS kernels inline -- and the plan step's state copy.
#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_rhs.cuh"

#include <algorithm>

namespace fj {

__global__ void k_cons_to_prim(const double* __restrict__ q, double* __restrict__ pv, int64_t n,
                               double gm1) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  Prim<double> p = cons_to_prim<double>(q[c], q[n + c], q[2 * n + c], q[3 * n + c], q[4 * n + c], gm1);
  pv[c] = p.rho;
  pv[n + c] = p.u;
  pv[2 * n + c] = p.v;
  pv[3 * n + c] = p.w;
  pv[4 * n + c] = p.p;
}

__global__ void k_prim_to_cons(const double* __restrict__ pv, double* __restrict__ q, int64_t n,
                               double gm1) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  Prim<double> p{pv[c], pv[n + c], pv[2 * n + c], pv[3 * n + c], pv[4 * n + c]};
  Cons<double> u = prim_to_cons(p, gm1);
  q[c] = u.r;
  q[n + c] = u.ru;
  q[2 * n + c] = u.rv;
  q[3 * n + c] = u.rw;
  q[4 * n + c] = u.rE;
}

__global__ void k_roe(const double* __restrict__ UL, const double* __restrict__ UR,
                      const double* __restrict__ nx, double* __restrict__ F, int64_t n,
                      double gm1, double eps) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  Cons<double> L{UL[c], UL[n + c], UL[2 * n + c], UL[3 * n + c], UL[4 * n + c]};
  Cons<double> R{UR[c], UR[n + c], UR[2 * n + c], UR[3 * n + c], UR[4 * n + c]};
  double f[5];
  roe_flux<double>(L, R, nx[c], nx[n + c], nx[2 * n + c], gm1, eps, f);
#pragma unroll
  for (int v = 0; v < 5; ++v) F[v * n + c] = f[v];
}

// pv (nv, n1, n2, n3); outputs have extent n_axis - 3 along `axis` (1..3).
__global__ void k_muscl2(const double* __restrict__ pv, double* __restrict__ L,
                         double* __restrict__ R, int nv, int n1, int n2, int n3, int axis,
                         int limiter) {
  const int o1 = n1 - (axis == 1 ? 3 : 0), o2 = n2 - (axis == 2 ? 3 : 0),
            o3 = n3 - (axis == 3 ? 3 : 0);
  const int64_t NO = (int64_t)o1 * o2 * o3;
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= NO * nv) return;
  const int v = (int)(t / NO);
  const int64_t r = t - v * NO;
  const int c = (int)(r % o3);
  const int b = (int)((r / o3) % o2);
  const int a = (int)(r / ((int64_t)o3 * o2));
  const int64_t stride = axis == 1 ? (int64_t)n2 * n3 : (axis == 2 ? n3 : 1);
  const int64_t base = (int64_t)v * n1 * n2 * n3 + ((int64_t)a * n2 + b) * n3 + c;
  double l, rr;
  muscl2<double>(pv[base], pv[base + stride], pv[base + 2 * stride], pv[base + 3 * stride],
                 limiter, l, rr);
  L[t] = l;
  R[t] = rr;
}

__global__ void k_limiter(const double* __restrict__ a, const double* __restrict__ b,
                          double* __restrict__ out, int64_t n, int limiter) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  out[c] = limit<double>(a[c], b[c], limiter);
}

int pw_limiter(const double* a, const double* b, double* out, int64_t n, int limiter,
               cudaStream_t st) {
  k_limiter<<<grid_for(n), kThreads, 0, st>>>(a, b, out, n, limiter);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

// Copies of whole state arrays (one per block, src[b] -> dst[b], len[b]
// doubles) in one launch: blockIdx.y is the block, 16-byte accesses where both
// pointers allow.  Launched with pdl_launch: the sources may be the previous
// step's results.
__global__ void k_copy_states(const CopyTable t) {
  grid_dep_wait();
  const int b = blockIdx.y;
  const double* __restrict__ s = t.src[b];
  double* __restrict__ d = t.dst[b];
  const int64_t n = t.len[b];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d)) & 15) == 0) {
    const int64_t n2 = n >> 1;
    for (int64_t i = i0; i < n2; i += stride)
      reinterpret_cast<double2*>(d)[i] = reinterpret_cast<const double2*>(s)[i];
    if ((n & 1) && i0 == 0) d[n - 1] = s[n - 1];
  } else {
    for (int64_t i = i0; i < n; i += stride) d[i] = s[i];
  }
}

int copy_states(const double* const* src, double* const* dst, const int64_t* len, int n, cudaStream_t st,
                int64_t* launches) {
  for (int base = 0; base < n; base += kMaxCopyBlocks) {
    CopyTable t;
    t.n = std::min(kMaxCopyBlocks, n - base);
    int64_t longest = 0;
    for (int i = 0; i < t.n; ++i) {
      t.src[i] = src[base + i];
      t.dst[i] = dst[base + i];
      t.len[i] = len[base + i];
      longest = std::max(longest, t.len[i]);
    }
    if (longest == 0) continue;
    // about eight 256-thread CTAs per SM over all blocks of the launch, at most
    // one per 512 doubles of the longest block
    const int64_t per_block = std::max<int64_t>(1, 148 * 8 / t.n);
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>(per_block, (longest + 511) / 512));
    cudaError_t e = pdl_launch(k_copy_states, dim3(gx, (unsigned)t.n), kThreads, 0, st, t);
    if (e != cudaSuccess) return FJ_ERR_CUDA;
    if (launches) *launches += 1;
  }
  return FJ_OK;
}

__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < n) out[c] = (float)in[c];
}

int convert_f64_f32(const double* in, float* out, int64_t n, cudaStream_t st) {
  k_f64_to_f32<<<grid_for(n), kThreads, 0, st>>>(in, out, n);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

__global__ void k_rk3_combine(const double* __restrict__ q0, const double* __restrict__ qs,
                              const double* __restrict__ Lr, double* __restrict__ out, int64_t n,
                              double dt, int stage) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const double t = qs[c] + dt * Lr[c];
  if (stage == 1)
    out[c] = t;
  else if (stage == 2)
    out[c] = 0.75 * q0[c] + 0.25 * t;
  else
    out[c] = (1.0 / 3.0) * q0[c] + (2.0 / 3.0) * t;
}

int pw_cons_to_prim(const double* q, double* pv, int64_t n, double gamma, cudaStream_t st) {
  k_cons_to_prim<<<grid_for(n), kThreads, 0, st>>>(q, pv, n, gamma - 1.0);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}
int pw_prim_to_cons(const double* pv, double* q, int64_t n, double gamma, cudaStream_t st) {
  k_prim_to_cons<<<grid_for(n), kThreads, 0, st>>>(pv, q, n, gamma - 1.0);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}
int pw_roe(const double* UL, const double* UR, const double* nx, double* F, int64_t n,
           double gamma, double eps, cudaStream_t st) {
  k_roe<<<grid_for(n), kThreads, 0, st>>>(UL, UR, nx, F, n, gamma - 1.0, eps);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}
int pw_muscl2(const double* pv, double* L, double* R, int nv, int n1, int n2, int n3, int axis,
              int limiter, cudaStream_t st) {
  const int64_t no = (int64_t)nv * (n1 - (axis == 1 ? 3 : 0)) * (n2 - (axis == 2 ? 3 : 0)) *
                     (n3 - (axis == 3 ? 3 : 0));
  k_muscl2<<<grid_for(no), kThreads, 0, st>>>(pv, L, R, nv, n1, n2, n3, axis, limiter);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}
int pw_rk3_combine(const double* q0, const double* qs, const double* Lr, double* out, int64_t n,
                   double dt, int stage, cudaStream_t st) {
  k_rk3_combine<<<grid_for(n), kThreads, 0, st>>>(q0, qs, Lr, out, n, dt, stage);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

}  // namespace fj
