// fj_reduce.cu -- FP64 global reductions over all blocks: the CFL time step,
// the kinetic-energy integral, the state check (finite values, minimum
// density and pressure) and the per-component residual RMS of dq/dt.  None of these exists in the reference, which takes
// dt as an argument (solver/step.py:18) and declares but never reads
// Config.cfl / Config.nan_check (core/types.py:187-189).
//
// Each kernel runs a fixed grid (a multiple of the SM count), reduces each CTA
// with warp shuffles and writes one partial per CTA; a single-CTA kernel folds
// the partials in a fixed order, so results are bitwise reproducible.
#include <vector>

#include "fj_common.cuh"

namespace fj {

namespace {

constexpr int kRedBlocks = 592;  // 4 x 148 SMs

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// op: 0 sum, 1 max, 2 min
template <int OP>
__device__ __forceinline__ double block_reduce(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = OP == 0 ? warp_sum(v) : (OP == 1 ? warp_max(v) : warp_min(v));
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  double r = OP == 0 ? 0.0 : (OP == 1 ? -INFINITY : INFINITY);
  if (wid == 0) {
    r = lane < nw ? sh[lane] : r;
    r = OP == 0 ? warp_sum(r) : (OP == 1 ? warp_max(r) : warp_min(r));
  }
  __syncthreads();
  return r;
}

struct Dims {
  int ni, nj, nk, g;
};

__device__ __forceinline__ bool interior_cell(int64_t t, const Dims& d, int64_t& c) {
  const int jj = d.nj - 2 * d.g, kk = d.nk - 2 * d.g;
  const int k = (int)(t % kk) + d.g;
  const int j = (int)((t / kk) % jj) + d.g;
  const int i = (int)(t / ((int64_t)kk * jj)) + d.g;
  c = ((int64_t)i * d.nj + j) * d.nk + k;
  return true;
}

// max over interior cells of sum_a (|u.n_a| + c) |k_a| / vol
__global__ void k_cfl_partial(const double* __restrict__ q, const double* __restrict__ kxyz,
                              const double* __restrict__ vol, Dims d, double gamma,
                              double* __restrict__ part) {
  __shared__ double sh[32];
  const int64_t N = (int64_t)d.ni * d.nj * d.nk;
  const int64_t NI = (int64_t)(d.ni - 2 * d.g) * (d.nj - 2 * d.g) * (d.nk - 2 * d.g);
  double m = 0.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < NI;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c;
    interior_cell(t, d, c);
    const double rho = q[c];
    const double u = q[N + c] / rho, v = q[2 * N + c] / rho, w = q[3 * N + c] / rho;
    const double ke = 0.5 * (u * u + v * v + w * w);
    const double p = (gamma - 1.0) * (q[4 * N + c] - rho * ke);
    const double cs = sqrt(gamma * p / rho);
    double lam = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double k0 = kxyz[(3 * a + 0) * N + c], k1 = kxyz[(3 * a + 1) * N + c],
                   k2 = kxyz[(3 * a + 2) * N + c];
      const double kmag = sqrt(k0 * k0 + k1 * k1 + k2 * k2);
      const double un = (u * k0 + v * k1 + w * k2) / kmag;
      lam = lam + (fabs(un) + cs) * kmag;
    }
    m = fmax(m, lam / vol[c]);
  }
  m = block_reduce<1>(m, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = m;
}

__global__ void k_ke_partial(const double* __restrict__ q, const double* __restrict__ vol, Dims d,
                             double* __restrict__ part) {
  __shared__ double sh[32];
  const int64_t N = (int64_t)d.ni * d.nj * d.nk;
  const int64_t NI = (int64_t)(d.ni - 2 * d.g) * (d.nj - 2 * d.g) * (d.nk - 2 * d.g);
  double s = 0.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < NI;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c;
    interior_cell(t, d, c);
    const double r1 = q[N + c], r2 = q[2 * N + c], r3 = q[3 * N + c];
    s += vol[c] * (0.5 * (r1 * r1 + r2 * r2 + r3 * r3) / q[c]);
  }
  s = block_reduce<0>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// part layout per CTA: sum over interior cells of ((q - q_prev) / dt)^2 per
// component (5 values)
__global__ void k_res_partial(const double* __restrict__ q, const double* __restrict__ qp, Dims d,
                              double inv_dt, double* __restrict__ part) {
  __shared__ double sh[32];
  const int64_t N = (int64_t)d.ni * d.nj * d.nk;
  const int64_t NI = (int64_t)(d.ni - 2 * d.g) * (d.nj - 2 * d.g) * (d.nk - 2 * d.g);
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < NI;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c;
    interior_cell(t, d, c);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double r = (q[v * N + c] - qp[v * N + c]) * inv_dt;
      s[v] += r * r;
    }
  }
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const double x = block_reduce<0>(s[v], sh);
    if (threadIdx.x == 0) part[5 * blockIdx.x + v] = x;
  }
}

// part layout per CTA: [nonfinite count, min rho, min p]
__global__ void k_check_partial(const double* __restrict__ q, int64_t N, double gamma,
                                double* __restrict__ part) {
  __shared__ double sh[32];
  double bad = 0.0, mr = INFINITY, mp = INFINITY;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N;
       c += (int64_t)gridDim.x * blockDim.x) {
    const double r0 = q[c], r1 = q[N + c], r2 = q[2 * N + c], r3 = q[3 * N + c],
                 r4 = q[4 * N + c];
    bad += (double)(!isfinite(r0)) + (double)(!isfinite(r1)) + (double)(!isfinite(r2)) +
           (double)(!isfinite(r3)) + (double)(!isfinite(r4));
    const double u = r1 / r0, v = r2 / r0, w = r3 / r0;
    const double p = (gamma - 1.0) * (r4 - r0 * (0.5 * (u * u + v * v + w * w)));
    mr = fmin(mr, r0);
    mp = fmin(mp, p);
  }
  bad = block_reduce<0>(bad, sh);
  mr = block_reduce<2>(mr, sh);
  mp = block_reduce<2>(mp, sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = bad;
    part[3 * blockIdx.x + 1] = mr;
    part[3 * blockIdx.x + 2] = mp;
  }
}

// Folds n partials (stride `stride`, component `comp`) with OP into out[0].
template <int OP>
__global__ void k_fold(const double* __restrict__ part, int n, int stride, int comp,
                       double* __restrict__ out) {
  __shared__ double sh[32];
  double v = OP == 0 ? 0.0 : (OP == 1 ? -INFINITY : INFINITY);
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const double x = part[(int64_t)t * stride + comp];
    v = OP == 0 ? v + x : (OP == 1 ? fmax(v, x) : fmin(v, x));
  }
  v = block_reduce<OP>(v, sh);
  if (threadIdx.x == 0) out[0] = v;
}

int check_blocks(fj_ctx* ctx, const fj_block* blocks, int nblocks, int g) {
  if (!blocks || nblocks <= 0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "no blocks");
  for (int b = 0; b < nblocks; ++b) {
    if (!blocks[b].q) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block q is NULL");
    if (blocks[b].ni <= 2 * g || blocks[b].nj <= 2 * g || blocks[b].nk <= 2 * g)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block has no interior cells");
  }
  return FJ_OK;
}

}  // namespace

int reduce_cfl_dt(fj_ctx* ctx, const fj_block* blocks, int nblocks, double gamma, int g,
                  double cfl, double* dt_out, cudaStream_t st) {
  int s = check_blocks(ctx, blocks, nblocks, g);
  if (s != FJ_OK) return s;
  for (int b = 0; b < nblocks; ++b)
    if (!blocks[b].kxyz || !blocks[b].vol)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block metrics are NULL");
  s = ensure_red(ctx, sizeof(double) * (3 * (size_t)kRedBlocks * nblocks + 8));
  if (s != FJ_OK) return s;
  double* part = (double*)ctx->red;
  double* out = part + 3 * (size_t)kRedBlocks * nblocks;
  for (int b = 0; b < nblocks; ++b) {
    Dims d{blocks[b].ni, blocks[b].nj, blocks[b].nk, g};
    k_cfl_partial<<<kRedBlocks, kThreads, 0, st>>>(blocks[b].q, blocks[b].kxyz, blocks[b].vol, d,
                                                   gamma, part + (size_t)b * kRedBlocks);
  }
  k_fold<1><<<1, 1024, 0, st>>>(part, kRedBlocks * nblocks, 1, 0, out);
  double lam = 0.0;
  s = cuda_status(ctx, cudaMemcpyAsync(&lam, out, sizeof(double), cudaMemcpyDeviceToHost, st),
                  "cfl copy");
  if (s != FJ_OK) return s;
  s = cuda_status(ctx, cudaStreamSynchronize(st), "cfl sync");
  if (s != FJ_OK) return s;
  if (!(lam > 0.0) || !isfinite(lam))
    return set_err(ctx, FJ_ERR_NONFINITE, "CFL spectral radius is not finite and positive");
  *dt_out = cfl / lam;
  return FJ_OK;
}

int reduce_kinetic_energy(fj_ctx* ctx, const fj_block* blocks, int nblocks, int g, double* res,
                          cudaStream_t st) {
  int s = check_blocks(ctx, blocks, nblocks, g);
  if (s != FJ_OK) return s;
  for (int b = 0; b < nblocks; ++b)
    if (!blocks[b].vol) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block vol is NULL");
  s = ensure_red(ctx, sizeof(double) * (3 * (size_t)kRedBlocks * nblocks + 8));
  if (s != FJ_OK) return s;
  double* part = (double*)ctx->red;
  double* out = part + 3 * (size_t)kRedBlocks * nblocks;
  for (int b = 0; b < nblocks; ++b) {
    Dims d{blocks[b].ni, blocks[b].nj, blocks[b].nk, g};
    k_ke_partial<<<kRedBlocks, kThreads, 0, st>>>(blocks[b].q, blocks[b].vol, d,
                                                  part + (size_t)b * kRedBlocks);
  }
  k_fold<0><<<1, 1024, 0, st>>>(part, kRedBlocks * nblocks, 1, 0, out);
  s = cuda_status(ctx, cudaMemcpyAsync(res, out, sizeof(double), cudaMemcpyDeviceToHost, st),
                  "ke copy");
  if (s != FJ_OK) return s;
  return cuda_status(ctx, cudaStreamSynchronize(st), "ke sync");
}

int reduce_check_state(fj_ctx* ctx, const fj_block* blocks, int nblocks, double gamma,
                       int64_t* nonfinite, double* min_rho, double* min_p, cudaStream_t st) {
  int s = check_blocks(ctx, blocks, nblocks, 0);
  if (s != FJ_OK) return s;
  s = ensure_red(ctx, sizeof(double) * (3 * (size_t)kRedBlocks * nblocks + 8));
  if (s != FJ_OK) return s;
  double* part = (double*)ctx->red;
  double* out = part + 3 * (size_t)kRedBlocks * nblocks;
  for (int b = 0; b < nblocks; ++b) {
    const int64_t N = (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
    k_check_partial<<<kRedBlocks, kThreads, 0, st>>>(blocks[b].q, N, gamma,
                                                     part + 3 * (size_t)b * kRedBlocks);
  }
  const int n = kRedBlocks * nblocks;
  k_fold<0><<<1, 1024, 0, st>>>(part, n, 3, 0, out);
  k_fold<2><<<1, 1024, 0, st>>>(part, n, 3, 1, out + 1);
  k_fold<2><<<1, 1024, 0, st>>>(part, n, 3, 2, out + 2);
  double h[3];
  s = cuda_status(ctx, cudaMemcpyAsync(h, out, 3 * sizeof(double), cudaMemcpyDeviceToHost, st),
                  "check copy");
  if (s != FJ_OK) return s;
  s = cuda_status(ctx, cudaStreamSynchronize(st), "check sync");
  if (s != FJ_OK) return s;
  *nonfinite = (int64_t)h[0];
  *min_rho = h[1];
  *min_p = h[2];
  if (h[0] > 0.0 || !(h[1] > 0.0) || !(h[2] > 0.0))
    return set_err(ctx, FJ_ERR_NONFINITE, "state has non-finite values or non-positive rho/p");
  return FJ_OK;
}

int reduce_residual(fj_ctx* ctx, const fj_block* blocks, const double* const* prev, int nblocks, int g,
                    double dt, double* res5, cudaStream_t st) {
  int s = check_blocks(ctx, blocks, nblocks, g);
  if (s != FJ_OK) return s;
  if (!prev || !(dt > 0.0)) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad previous states or dt");
  for (int b = 0; b < nblocks; ++b)
    if (!prev[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "previous state is NULL");
  s = ensure_red(ctx, sizeof(double) * (5 * (size_t)kRedBlocks * nblocks + 8));
  if (s != FJ_OK) return s;
  double* part = (double*)ctx->red;
  double* out = part + 5 * (size_t)kRedBlocks * nblocks;
  int64_t cells = 0;
  for (int b = 0; b < nblocks; ++b) {
    Dims d{blocks[b].ni, blocks[b].nj, blocks[b].nk, g};
    cells += (int64_t)(d.ni - 2 * g) * (d.nj - 2 * g) * (d.nk - 2 * g);
    k_res_partial<<<kRedBlocks, kThreads, 0, st>>>(blocks[b].q, prev[b], d, 1.0 / dt,
                                                   part + 5 * (size_t)b * kRedBlocks);
  }
  for (int v = 0; v < 5; ++v) k_fold<0><<<1, 1024, 0, st>>>(part, kRedBlocks * nblocks, 5, v, out + v);
  ctx->launches += nblocks + 5;
  double h[5];
  s = cuda_status(ctx, cudaMemcpyAsync(h, out, 5 * sizeof(double), cudaMemcpyDeviceToHost, st), "residual copy");
  if (s != FJ_OK) return s;
  s = cuda_status(ctx, cudaStreamSynchronize(st), "residual sync");
  if (s != FJ_OK) return s;
  for (int v = 0; v < 5; ++v) res5[v] = sqrt(h[v] / (double)cells);
  return FJ_OK;
}

}  // namespace fj
