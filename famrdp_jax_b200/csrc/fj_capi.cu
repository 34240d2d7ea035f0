// fj_capi.cu -- the extern "C" entry points of libfamrdp_cuda.so
// (declared in include/famrdp_cuda.h).  Validation, scratch sizing and
// dispatch only; the kernels live in the other translation units.
#include <algorithm>
#include <new>
#include <vector>

#include "famrdp_cuda.h"
#include "fj_common.cuh"
#include "fj_rhs.cuh"
#include "fj_stage.cuh"

namespace fj {
int metrics(const double* xyz, double* jac, double* kxyz, double* vol, int ni, int nj, int nk,
            cudaStream_t st);
int pw_cons_to_prim(const double* q, double* pv, int64_t n, double gamma, cudaStream_t st);
int pw_prim_to_cons(const double* pv, double* q, int64_t n, double gamma, cudaStream_t st);
int pw_roe(const double* UL, const double* UR, const double* nx, double* F, int64_t n,
           double gamma, double eps, cudaStream_t st);
int pw_muscl2(const double* pv, double* L, double* R, int nv, int n1, int n2, int n3, int axis,
              int limiter, cudaStream_t st);
int pw_rk3_combine(const double* q0, const double* qs, const double* Lr, double* out, int64_t n,
                   double dt, int stage, cudaStream_t st);
int pw_limiter(const double* a, const double* b, double* out, int64_t n, int limiter,
               cudaStream_t st);
int reduce_cfl_dt(fj_ctx* ctx, const fj_block* blocks, int nblocks, double gamma, int g,
                  double cfl, double* dt_out, cudaStream_t st);
int reduce_kinetic_energy(fj_ctx* ctx, const fj_block* blocks, int nblocks, int g, double* res,
                          cudaStream_t st);
int reduce_check_state(fj_ctx* ctx, const fj_block* blocks, int nblocks, double gamma,
                       int64_t* nonfinite, double* min_rho, double* min_p, cudaStream_t st);
}  // namespace fj

using namespace fj;

namespace {

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Scratch of one RHS/stage evaluation: none for the fused kernel, the
// intermediates for the staged pipeline.
size_t rhs_scratch_bytes(const fj_ctx* ctx, int precision, int ni, int nj, int nk) {
  if (ctx->pipeline == FJ_PIPELINE_FUSED) return 0;
  return precision == FJ_PREC_F32FLUX ? staged_ws_bytes<float>(ni, nj, nk)
                                      : staged_ws_bytes<double>(ni, nj, nk);
}

int run_rhs(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
            const double* q0, double* out, int ni, int nj, int nk, const fj_params* p, int flags,
            int stage, double dt, void* ws, cudaStream_t st) {
  Phys ph = make_phys(p);
  if (ctx->pipeline == FJ_PIPELINE_FUSED) {
    StageArgs a{};
    a.q = q;
    a.q0 = q0;
    a.kxyz = kxyz;
    a.kxyz32 = nullptr;
    a.vol = vol;
    a.out = out;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.flags = flags;
    a.stage = stage;
    a.dt = dt;
    a.ph = ph;
    return fused_stage(ctx, a, ctx->seg, p->precision, st);
  }
  if (p->precision == FJ_PREC_F32FLUX)
    return staged_rhs<float>(ctx, q, kxyz, vol, q0, out, ni, nj, nk, ph, flags, stage, dt, ws, st);
  return staged_rhs<double>(ctx, q, kxyz, vol, q0, out, ni, nj, nk, ph, flags, stage, dt, ws, st);
}

int rhs_entry(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol, double* rhs,
              int ni, int nj, int nk, const fj_params* p, int flags, void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  int s = check_params(ctx, p);
  if (s != FJ_OK) return s;
  s = check_dims(ctx, ni, nj, nk);
  if (s != FJ_OK) return s;
  if (!q || !kxyz || !rhs || ((flags & kRhsInvscd) && !vol))
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "NULL array argument");
  s = ensure_ws(ctx, rhs_scratch_bytes(ctx, p->precision, ni, nj, nk));
  if (s != FJ_OK) return s;
  return run_rhs(ctx, q, kxyz, vol, nullptr, rhs, ni, nj, nk, p, flags, 0, 0.0, ctx->ws, S(stream));
}

int check_blockset(fj_ctx* ctx, const fj_block* blocks, int nblocks, bool need_metrics) {
  if (!blocks || nblocks <= 0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "no blocks");
  for (int b = 0; b < nblocks; ++b) {
    if (!blocks[b].q) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block q is NULL");
    if (need_metrics && (!blocks[b].kxyz || !blocks[b].vol))
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block metrics are NULL");
    int s = check_dims(ctx, blocks[b].ni, blocks[b].nj, blocks[b].nk);
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

}  // namespace

extern "C" {

int fj_abi_version(void) { return FJ_ABI_VERSION; }

const char* fj_status_string(int status) {
  switch (status) {
    case FJ_OK: return "ok";
    case FJ_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FJ_ERR_CUDA: return "CUDA error";
    case FJ_ERR_NOT_IMPLEMENTED: return "not implemented";
    case FJ_ERR_SHAPE: return "shape mismatch";
    case FJ_ERR_NONFINITE: return "non-finite or non-physical state";
    case FJ_ERR_NO_MEMORY: return "out of device memory";
    case FJ_ERR_SCRATCH_LIMIT: return "block exceeds the fixed scratch of the no-allocation entry point";
    default: return "unknown status";
  }
}

int fj_ctx_create(fj_ctx** out) {
  if (!out) return FJ_ERR_INVALID_ARGUMENT;
  fj_ctx* c = new (std::nothrow) fj_ctx();
  if (!c) return FJ_ERR_NO_MEMORY;
  if (cudaGetDevice(&c->device) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return FJ_ERR_CUDA;
  }
  *out = c;
  return FJ_OK;
}

int fj_ctx_destroy(fj_ctx* ctx) {
  if (!ctx) return FJ_OK;
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->red) cudaFree(ctx->red);
  delete ctx;
  return FJ_OK;
}

const char* fj_last_error(const fj_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int fj_ctx_set_pipeline(fj_ctx* ctx, int pipeline, int seg) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (pipeline != FJ_PIPELINE_FUSED && pipeline != FJ_PIPELINE_STAGED)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown pipeline");
  if (seg < 0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "segment length must be >= 0");
  ctx->pipeline = pipeline;
  ctx->seg = seg;
  return FJ_OK;
}

int fj_launch_count(const fj_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return FJ_ERR_INVALID_ARGUMENT;
  *out = ctx->launches;
  return FJ_OK;
}

int fj_rk_stage_f64(fj_ctx* ctx, const double* q, const double* q0, const double* kxyz,
                    const double* vol, double* out, int ni, int nj, int nk, const fj_params* p,
                    double dt, int stage, void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  int s = check_params(ctx, p);
  if (s != FJ_OK) return s;
  s = check_dims(ctx, ni, nj, nk);
  if (s != FJ_OK) return s;
  if (stage < 1 || stage > 3) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "stage must be 1, 2 or 3");
  if (!q || !kxyz || !vol || !out || (stage > 1 && !q0))
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "NULL array argument");
  if (out == q) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "out must not alias q");
  s = ensure_ws(ctx, rhs_scratch_bytes(ctx, p->precision, ni, nj, nk));
  if (s != FJ_OK) return s;
  return run_rhs(ctx, q, kxyz, vol, q0, out, ni, nj, nk, p, kRhsInvscd | kRhsViscous, stage, dt,
                 ctx->ws, S(stream));
}

int fj_cons_to_prim_f64(const double* q, double* pv, int64_t ncell, double gamma, void* stream) {
  if (!q || !pv || ncell < 0) return FJ_ERR_INVALID_ARGUMENT;
  if (ncell == 0) return FJ_OK;
  return pw_cons_to_prim(q, pv, ncell, gamma, S(stream));
}

int fj_prim_to_cons_f64(const double* pv, double* q, int64_t ncell, double gamma, void* stream) {
  if (!q || !pv || ncell < 0) return FJ_ERR_INVALID_ARGUMENT;
  if (ncell == 0) return FJ_OK;
  return pw_prim_to_cons(pv, q, ncell, gamma, S(stream));
}

int fj_roe_flux_f64(const double* UL, const double* UR, const double* nxyz, double* F,
                    int64_t nface, double gamma, double eps_entropy, void* stream) {
  if (!UL || !UR || !nxyz || !F || nface < 0) return FJ_ERR_INVALID_ARGUMENT;
  if (nface == 0) return FJ_OK;
  return pw_roe(UL, UR, nxyz, F, nface, gamma, eps_entropy, S(stream));
}

int fj_limiter_f64(const double* a, const double* b, double* out, int64_t n, int limiter,
                   void* stream) {
  if (!a || !b || !out || n < 0) return FJ_ERR_INVALID_ARGUMENT;
  if (limiter != FJ_LIM_MINMOD && limiter != FJ_LIM_VANLEER) return FJ_ERR_INVALID_ARGUMENT;
  if (n == 0) return FJ_OK;
  return pw_limiter(a, b, out, n, limiter, S(stream));
}

int fj_muscl2_f64(const double* pv, double* pvL, double* pvR, int nv, int n1, int n2, int n3,
                  int axis, int limiter, void* stream) {
  if (!pv || !pvL || !pvR || nv < 1 || n1 < 1 || n2 < 1 || n3 < 1) return FJ_ERR_INVALID_ARGUMENT;
  if (axis < 1 || axis > 3) return FJ_ERR_INVALID_ARGUMENT;
  if (limiter != FJ_LIM_MINMOD && limiter != FJ_LIM_VANLEER) return FJ_ERR_INVALID_ARGUMENT;
  const int n = axis == 1 ? n1 : (axis == 2 ? n2 : n3);
  if (n < 4) return FJ_ERR_INVALID_ARGUMENT;
  return pw_muscl2(pv, pvL, pvR, nv, n1, n2, n3, axis, limiter, S(stream));
}

int fj_invscd_rhs_f64(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
                      double* rhs, int ni, int nj, int nk, const fj_params* p, void* stream) {
  return rhs_entry(ctx, q, kxyz, vol, rhs, ni, nj, nk, p, kRhsInvscd, stream);
}

int fj_viscous_rhs_f64(fj_ctx* ctx, const double* q, const double* kxyz, double* rhs, int ni,
                       int nj, int nk, const fj_params* p, void* stream) {
  return rhs_entry(ctx, q, kxyz, nullptr, rhs, ni, nj, nk, p, kRhsViscous, stream);
}

int fj_rhs_f64(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol, double* rhs,
               int ni, int nj, int nk, const fj_params* p, void* stream) {
  return rhs_entry(ctx, q, kxyz, vol, rhs, ni, nj, nk, p, kRhsInvscd | kRhsViscous, stream);
}

int fj_halo_exchange_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links,
                         int nlinks, int ghost, void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (ghost != 2) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "the kernels require ghost == 2");
  int s = check_blockset(ctx, blocks, nblocks, false);
  if (s != FJ_OK) return s;
  if (nlinks < 0 || (nlinks > 0 && !links))
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad link list");
  for (int L = 0; L < nlinks; ++L)
    if (links[L].tgt_block < 0 || links[L].tgt_block >= nblocks || links[L].tgt_face < 0 ||
        links[L].tgt_face > 5)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "link target out of range");
  const size_t hb = halo_ws_bytes(blocks, links, nlinks, ghost);
  s = ensure_ws(ctx, std::max<size_t>(hb, 256));
  if (s != FJ_OK) return s;
  return halo_exchange(ctx, blocks, nblocks, links, nlinks, ghost, (double*)ctx->ws, ctx->ws_bytes,
                       S(stream));
}

int fj_apply_bc_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_bc* bcs, int nbcs,
                    const fj_params* p, void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  int s = check_params(ctx, p);
  if (s != FJ_OK) return s;
  s = check_blockset(ctx, blocks, nblocks, false);
  if (s != FJ_OK) return s;
  if (nbcs < 0 || (nbcs > 0 && !bcs)) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad bc list");
  return apply_bc(ctx, blocks, nblocks, bcs, nbcs, p, S(stream));
}

int fj_step_f64(fj_ctx* ctx, const fj_block* blocks, double* const* q_out, int nblocks,
                const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs, const fj_params* p,
                double dt, void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  int s = check_params(ctx, p);
  if (s != FJ_OK) return s;
  s = check_blockset(ctx, blocks, nblocks, true);
  if (s != FJ_OK) return s;
  if (!q_out) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "q_out is NULL");
  if (nlinks < 0 || (nlinks > 0 && !links) || nbcs < 0 || (nbcs > 0 && !bcs))
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad link or bc list");
  for (int L = 0; L < nlinks; ++L)
    if (links[L].tgt_block < 0 || links[L].tgt_block >= nblocks || links[L].tgt_face < 0 ||
        links[L].tgt_face > 5)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "link target out of range");
  cudaStream_t st = S(stream);
  size_t maxN = 0, rhs_b = 0;
  for (int b = 0; b < nblocks; ++b) {
    if (!q_out[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "q_out entry is NULL");
    maxN = std::max(maxN, (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk);
    rhs_b = std::max(rhs_b, rhs_scratch_bytes(ctx, p->precision, blocks[b].ni, blocks[b].nj, blocks[b].nk));
  }
  const size_t stage_b = align256(5 * maxN * sizeof(double));
  const size_t halo_b = halo_ws_bytes(blocks, links, nlinks, p->ghost);
  s = ensure_ws(ctx, 2 * stage_b + std::max(rhs_b, halo_b));
  if (s != FJ_OK) return s;
  double* q1 = (double*)ctx->ws;
  double* q2 = (double*)((char*)ctx->ws + stage_b);
  void* tail = (char*)ctx->ws + 2 * stage_b;
  const size_t tail_b = ctx->ws_bytes - 2 * stage_b;

  // q0 := q (the functional copy), then halo + BC in place on q0
  std::vector<fj_block> out(blocks, blocks + nblocks);
  for (int b = 0; b < nblocks; ++b) {
    out[b].q = q_out[b];
    if (q_out[b] != blocks[b].q) {
      const size_t bytes = 5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double);
      s = cuda_status(ctx, cudaMemcpyAsync(q_out[b], blocks[b].q, bytes, cudaMemcpyDeviceToDevice, st),
                      "state copy");
      if (s != FJ_OK) return s;
    }
  }
  s = halo_exchange(ctx, out.data(), nblocks, links, nlinks, p->ghost, (double*)tail, tail_b, st);
  if (s != FJ_OK) return s;
  s = apply_bc(ctx, out.data(), nblocks, bcs, nbcs, p, st);
  if (s != FJ_OK) return s;
  // Blocks do not interact between the halo fill and the end of the step
  // (solver/step.py:40-53), so each block runs its three stages back to back.
  const int flags = kRhsInvscd | kRhsViscous;
  for (int b = 0; b < nblocks; ++b) {
    const fj_block& B = out[b];
    s = run_rhs(ctx, B.q, B.kxyz, B.vol, B.q, q1, B.ni, B.nj, B.nk, p, flags, 1, dt, tail, st);
    if (s != FJ_OK) return s;
    s = run_rhs(ctx, q1, B.kxyz, B.vol, B.q, q2, B.ni, B.nj, B.nk, p, flags, 2, dt, tail, st);
    if (s != FJ_OK) return s;
    s = run_rhs(ctx, q2, B.kxyz, B.vol, B.q, B.q, B.ni, B.nj, B.nk, p, flags, 3, dt, tail, st);
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

int fj_rk3_combine_f64(const double* q0, const double* qs, const double* L, double* out, int64_t n,
                       double dt, int stage, void* stream) {
  if (!qs || !L || !out || n < 0 || stage < 1 || stage > 3 || (stage > 1 && !q0))
    return FJ_ERR_INVALID_ARGUMENT;
  if (n == 0) return FJ_OK;
  return pw_rk3_combine(q0, qs, L, out, n, dt, stage, S(stream));
}

int fj_metrics_f64(const double* xyz, double* jac, double* kxyz, double* vol, int ni, int nj,
                   int nk, void* stream) {
  if (!xyz || !jac || !kxyz || !vol || ni < 1 || nj < 1 || nk < 1) return FJ_ERR_INVALID_ARGUMENT;
  if ((int64_t)ni * nj * nk > (int64_t)INT32_MAX / 9) return FJ_ERR_INVALID_ARGUMENT;
  return metrics(xyz, jac, kxyz, vol, ni, nj, nk, S(stream));
}

int fj_cfl_dt_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_params* p,
                  double cfl, double* dt_out, void* stream) {
  if (!ctx || !dt_out) return FJ_ERR_INVALID_ARGUMENT;
  int s = check_params(ctx, p);
  if (s != FJ_OK) return s;
  return reduce_cfl_dt(ctx, blocks, nblocks, p->gamma, p->ghost, cfl, dt_out, S(stream));
}

int fj_kinetic_energy_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, int ghost, double* out,
                          void* stream) {
  if (!ctx || !out || ghost < 0) return FJ_ERR_INVALID_ARGUMENT;
  return reduce_kinetic_energy(ctx, blocks, nblocks, ghost, out, S(stream));
}

int fj_check_state_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, double gamma,
                       int64_t* nonfinite_out, double* min_rho_out, double* min_p_out,
                       void* stream) {
  if (!ctx || !nonfinite_out || !min_rho_out || !min_p_out) return FJ_ERR_INVALID_ARGUMENT;
  return reduce_check_state(ctx, blocks, nblocks, gamma, nonfinite_out, min_rho_out, min_p_out,
                            S(stream));
}

}  // extern "C"
