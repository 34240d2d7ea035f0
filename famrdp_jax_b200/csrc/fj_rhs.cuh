// fj_rhs.cuh -- internal interfaces between the C ABI (fj_capi.cu) and the
// RHS / step kernels.
#pragma once

#include <cuda_runtime.h>

#include "fj_common.cuh"

namespace fj {

// Which parts of the RHS a call evaluates (solver/step.py:10-15 = both).
constexpr int kRhsInvscd = 1;
constexpr int kRhsViscous = 2;

// Staged pipeline (fj_rhs_staged.cu).  stage 0 writes the RHS to `out`;
// stages 1..3 write the TVD-RK3 stage value (solver/step.py:45-53) computed
// from q (the stage input), q0 (the step's start state) and dt.
template <typename T>
size_t staged_ws_bytes(int ni, int nj, int nk);
template <typename T>
int staged_rhs(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
               const double* q0, double* out, int ni, int nj, int nk, const Phys& ph,
               int flags, int stage, double dt, void* ws, cudaStream_t st);

// The RHS (stage 0) launch sequence without a context, on caller-given scratch
// of staged_ws_bytes<T> bytes.
template <typename T>
cudaError_t staged_rhs_noctx(const double* q, const double* kxyz, const double* vol,
                             double* out, int ni, int nj, int nk, const Phys& ph, void* ws,
                             cudaStream_t st);

// Whole-array copies src[b] -> dst[b] (len[b] doubles each, non-overlapping)
// as SM kernels (fj_pointwise.cu), kMaxCopyBlocks arrays per launch;
// *launches (if set) counts the launches.
constexpr int kMaxCopyBlocks = 64;
struct CopyTable {
  int n;
  const double* src[kMaxCopyBlocks];
  double* dst[kMaxCopyBlocks];
  int64_t len[kMaxCopyBlocks];
};
int copy_states(const double* const* src, double* const* dst, const int64_t* len, int n, cudaStream_t st,
                int64_t* launches);

// Halo fill + boundary conditions (fj_halo.cu), in place on blocks[].q.
// `scratch` holds the gathered source slabs (halo_ws_bytes of them).
int halo_exchange(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links,
                  int nlinks, int ghost, double* scratch, size_t scratch_bytes,
                  cudaStream_t st);
int apply_bc(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_bc* bcs, int nbcs,
             const fj_params* p, cudaStream_t st);
// The step's start state blocks[b].q -> dst[b] with the halo fill of `links`
// folded in (one kernel over all blocks; dst must not overlap blocks[].q).
// *done = false, without launching, when the link or block count exceeds one
// launch's table: the caller then copies and fills separately.
int copy_fill(fj_ctx* ctx, const fj_block* blocks, double* const* dst, int nblocks, const fj_link* links, int nlinks,
              int ghost, cudaStream_t st, bool* done);
// Bytes of scratch the halo gather needs for these links (0 on shape errors).
size_t halo_ws_bytes(const fj_block* blocks, const fj_link* links, int nlinks, int ghost);
// One device's part of a halo fill whose blocks live on several devices: the
// links sel[0..nsel) have their source slabs gathered into buf (pack) or the
// slabs in buf written into their targets in selection order (unpack), slab i
// at buf + off[i] (5 x the target's ghost box, in the gather's order).  Blocks
// whose q this call does not touch may have q == NULL.
int halo_pack_unpack(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks, int ghost,
                     const int* sel, const int64_t* off, int nsel, double* buf, int64_t buf_doubles, bool unpack,
                     cudaStream_t st);

// ---- adjoint (fj_adjoint.cu, fj_halo.cu) ----
// Elementwise epilogue of an RHS VJP V = (dL/dq)^T lam, applied in the kernel
// that produces V instead of writing V:
//   o1 = a1 x1 + b1 y1 + c1 z1 + e1 V   (y1, z1 may be NULL)
//   o2 = a2 x2 + b2 y2               (o2 may be NULL; y2 may be NULL)
// Every input is read at a cell before any output is written there, so an
// output may alias an input.  With next_q set, the kernel also leaves in the
// workspace what the next RHS VJP of the same block (state next_q, adjoint
// o1, cell volumes next_vol, same flags) reads first: the primitives, lam/vol
// and the cleared face sums; that call is then made with ws_ready and skips
// its primitive launch.
struct VjpEpilogue {
  double* o1 = nullptr;
  const double* x1 = nullptr;
  double a1 = 0.0;
  const double* y1 = nullptr;
  double b1 = 0.0;
  const double* z1 = nullptr;
  double c1 = 0.0;
  double e1 = 1.0;
  double* o2 = nullptr;
  const double* x2 = nullptr;
  double a2 = 0.0;
  const double* y2 = nullptr;
  double b2 = 0.0;
  const double* next_q = nullptr;
  const double* next_vol = nullptr;
  bool ws_ready = false;
};
// out = (dL/dq)^T lam for one block (L = the RHS parts selected by flags), or
// with epi the epilogue's outputs instead (out unused); with dmu set, also
// *dmu += mu_scale * lam . L_vis(q) (device accumulator).
size_t rhs_vjp_ws_bytes(int precision, int ni, int nj, int nk);
int rhs_vjp(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol, const double* lam,
            double* out, int ni, int nj, int nk, const fj_params* p, int flags, void* ws,
            cudaStream_t st, double* dmu = nullptr, double mu_scale = 0.0, const VjpEpilogue* epi = nullptr);
// grad = dJ/dq of the interior kinetic-energy integral
int ke_grad(fj_ctx* ctx, const double* q, const double* vol, double* grad, int ni, int nj, int nk, int g,
            cudaStream_t st);
// In-place transposes of the halo fill and of the (linear) boundary conditions
// on per-block adjoint arrays; the blocks' q pointers hold the adjoints.
int halo_transpose(fj_ctx* ctx, const fj_block* lam, int nblocks, const fj_link* links, int nlinks,
                   int ghost, double* scratch, size_t scratch_bytes, cudaStream_t st);
int bc_transpose(fj_ctx* ctx, const fj_block* lam, int nblocks, const fj_bc* bcs, int nbcs,
                 const fj_params* p, cudaStream_t st);

}  // namespace fj
