// fj_metrics.cu -- grid metrics of one block (mesh/metric.py:18-70).
//
// Per cell: J[m][l] = d x_m / d xi_l by the 4th-order central difference
// (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2]) / 12 with indices wrapping around the
// array ends (jnp.roll, mesh/metric.py:24-28); jac = det(J); kxyz = inv(J)
// (kxyz[l][m] = d xi_l / d x_m); vol = |jac|.  The 3x3 determinant and inverse
// use cofactors (the reference uses LU; both are exact to a few ulp for the
// well-conditioned matrices of a valid grid).
#include "fj_common.cuh"

namespace fj {

__global__ void k_metrics(const double* __restrict__ xyz, double* __restrict__ jac,
                          double* __restrict__ kxyz, double* __restrict__ vol, int ni, int nj,
                          int nk) {
  const int N = ni * nj * nk;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int k = c % nk;
  const int j = (c / nk) % nj;
  const int i = c / (nk * nj);
  const int n[3] = {ni, nj, nk};
  const int idx[3] = {i, j, k};
  const int stride[3] = {nj * nk, nk, 1};
  double M[3][3];  // M[m][l]
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    int off[4];
    const int sh[4] = {2, 1, -1, -2};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      int t = idx[l] + sh[s];
      t = t >= n[l] ? t - n[l] : (t < 0 ? t + n[l] : t);
      off[s] = c + (t - idx[l]) * stride[l];
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const double* f = xyz + (int64_t)m * N;
      M[m][l] = (-f[off[0]] + 8.0 * f[off[1]] - 8.0 * f[off[2]] + f[off[3]]) / 12.0;
    }
  }
  const double c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
  const double c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
  const double c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
  const double det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
  const double c10 = M[0][2] * M[2][1] - M[0][1] * M[2][2];
  const double c11 = M[0][0] * M[2][2] - M[0][2] * M[2][0];
  const double c12 = M[0][1] * M[2][0] - M[0][0] * M[2][1];
  const double c20 = M[0][1] * M[1][2] - M[0][2] * M[1][1];
  const double c21 = M[0][2] * M[1][0] - M[0][0] * M[1][2];
  const double c22 = M[0][0] * M[1][1] - M[0][1] * M[1][0];
  // inv[l][m] = cofactor[m][l] / det
  const double cof[3][3] = {{c00, c01, c02}, {c10, c11, c12}, {c20, c21, c22}};
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) kxyz[(int64_t)(l * 3 + m) * N + c] = cof[m][l] / det;
  jac[c] = det;
  vol[c] = fabs(det);
}

int metrics(const double* xyz, double* jac, double* kxyz, double* vol, int ni, int nj, int nk,
            cudaStream_t st) {
  const int N = ni * nj * nk;
  k_metrics<<<grid_for(N), kThreads, 0, st>>>(xyz, jac, kxyz, vol, ni, nj, nk);
  return cudaGetLastError() == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

}  // namespace fj
