// fj_capi.cu -- the extern "C" entry points of libfamrdp_cuda.so
// (declared in include/famrdp_cuda.h).  Validation, scratch sizing and
// dispatch only; the kernels live in the other translation units.
#include <algorithm>
#include <new>
#include <vector>

#include "famrdp_cuda.h"
#include "fj_common.cuh"
#include "fj_rhs.cuh"
#include "fj_split.cuh"
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
int convert_f64_f32(const double* in, float* out, int64_t n, cudaStream_t st);
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

// Scratch of one RHS/stage evaluation of one block: none for the fused
// kernel, the intermediates for the split and staged pipelines.
size_t rhs_scratch_bytes(const fj_ctx* ctx, int precision, int ni, int nj, int nk) {
  if (ctx->pipeline == FJ_PIPELINE_FUSED) return 0;
  if (ctx->pipeline == FJ_PIPELINE_SPLIT) return split_scratch_bytes(precision, (int64_t)ni * nj * nk);
  return precision == FJ_PREC_F32FLUX ? staged_ws_bytes<float>(ni, nj, nk)
                                      : staged_ws_bytes<double>(ni, nj, nk);
}

SplitBlock split_block(const double* q, const double* q0, double* out, const double* kxyz,
                       const float* kxyz32, const double* vol, int ni, int nj, int nk) {
  SplitBlock b{};
  b.q = q;
  b.q0 = q0;
  b.out = out;
  b.kxyz = kxyz;
  b.kxyz32 = kxyz32;
  b.vol = vol;
  b.ni = ni;
  b.nj = nj;
  b.nk = nk;
  return b;
}

int run_rhs(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
            const double* q0, double* out, int ni, int nj, int nk, const fj_params* p, int flags,
            int stage, double dt, void* ws, cudaStream_t st, const float* kxyz32 = nullptr) {
  Phys ph = make_phys(p);
  if (ctx->pipeline == FJ_PIPELINE_SPLIT) {
    SplitBlock b = split_block(q, q0, out, kxyz, p->precision == FJ_PREC_F32FLUX ? kxyz32 : nullptr,
                               vol, ni, nj, nk);
    split_assign_scratch(p->precision, &b, 1, ws);
    return split_stage(ctx, &b, 1, ph, flags, stage, dt, p->precision, st);
  }
  if (ctx->pipeline == FJ_PIPELINE_FUSED) {
    StageArgs a{};
    a.q = q;
    a.q0 = q0;
    a.kxyz = kxyz;
    a.kxyz32 = p->precision == FJ_PREC_F32FLUX ? kxyz32 : nullptr;
    a.vol = vol;
    a.out = out;
    a.ni = ni;
    a.nj = nj;
    a.nk = nk;
    a.flags = flags;
    a.stage = stage;
    a.dt = dt;
    a.ph = ph;
    return fused_stage(ctx, a, ctx->seg, p->precision, ctx->tile, st);
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


int check_step_args(fj_ctx* ctx, const fj_block* blocks, double* const* q_out, int nblocks,
                    const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs, const fj_params* p) {
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
  for (int b = 0; b < nblocks; ++b)
    if (!q_out[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "q_out entry is NULL");
  return FJ_OK;
}

// Scratch layout of one step: [q1 | q2 | tail].  The split pipeline runs all
// blocks per launch, so q1/q2 hold every block and the tail every block's
// intermediates; the other pipelines run block by block and size everything
// for the largest block.  The halo slabs reuse the tail (the halo runs first).
size_t step_layout(const fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links,
                   int nlinks, const fj_params* p, size_t* stage_b, size_t* tail_b) {
  size_t maxN = 0, sumStage = 0, rhs_b = 0;
  int64_t cells = 0;
  for (int b = 0; b < nblocks; ++b) {
    const size_t N = (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
    maxN = std::max(maxN, N);
    sumStage += align256(5 * N * sizeof(double));
    cells += (int64_t)N;
    rhs_b = std::max(rhs_b, rhs_scratch_bytes(ctx, p->precision, blocks[b].ni, blocks[b].nj, blocks[b].nk));
  }
  const bool split = ctx->pipeline == FJ_PIPELINE_SPLIT;
  *stage_b = split ? sumStage : align256(5 * maxN * sizeof(double));
  const size_t work = split ? split_scratch_bytes(p->precision, cells) : rhs_b;
  *tail_b = align256(std::max(std::max(work, halo_ws_bytes(blocks, links, nlinks, p->ghost)), (size_t)256));
  return 2 * *stage_b + *tail_b;
}

// solver/step.py:18-56 on the device: q_out := q, halo + BC in place on q_out,
// then the three stages of each block (blocks do not interact between the halo
// fill and the end of the step, solver/step.py:40-53).
int step_body(fj_ctx* ctx, const fj_block* blocks, double* const* q_out, int nblocks,
              const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs, const fj_params* p,
              double dt, float* const* kxyz32, double* q1, double* q2, void* tail, size_t tail_b,
              cudaStream_t st) {
  std::vector<fj_block> out(blocks, blocks + nblocks);
  int s;
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
  const int flags = kRhsInvscd | kRhsViscous;
  if (ctx->pipeline == FJ_PIPELINE_SPLIT) {
    // all blocks per launch: q1/q2 hold every block (step_layout), the tail
    // holds the intermediates of every block
    std::vector<SplitBlock> sb(nblocks);
    std::vector<double*> b1(nblocks), b2(nblocks);
    size_t off = 0;
    for (int b = 0; b < nblocks; ++b) {
      const fj_block& B = out[b];
      b1[b] = (double*)((char*)q1 + off);
      b2[b] = (double*)((char*)q2 + off);
      off += align256(5 * (size_t)B.ni * B.nj * B.nk * sizeof(double));
      sb[b] = split_block(B.q, B.q, b1[b], B.kxyz,
                          (p->precision == FJ_PREC_F32FLUX && kxyz32) ? kxyz32[b] : nullptr, B.vol, B.ni,
                          B.nj, B.nk);
    }
    split_assign_scratch(p->precision, sb.data(), nblocks, tail);
    const Phys ph = make_phys(p);
    s = split_stage(ctx, sb.data(), nblocks, ph, flags, 1, dt, p->precision, st);
    if (s != FJ_OK) return s;
    for (int b = 0; b < nblocks; ++b) {
      sb[b].q = b1[b];
      sb[b].out = b2[b];
    }
    s = split_stage(ctx, sb.data(), nblocks, ph, flags, 2, dt, p->precision, st);
    if (s != FJ_OK) return s;
    for (int b = 0; b < nblocks; ++b) {
      sb[b].q = b2[b];
      sb[b].out = out[b].q;
    }
    return split_stage(ctx, sb.data(), nblocks, ph, flags, 3, dt, p->precision, st);
  }
  for (int b = 0; b < nblocks; ++b) {
    const fj_block& B = out[b];
    const float* k32 = kxyz32 ? kxyz32[b] : nullptr;
    s = run_rhs(ctx, B.q, B.kxyz, B.vol, B.q, q1, B.ni, B.nj, B.nk, p, flags, 1, dt, tail, st, k32);
    if (s != FJ_OK) return s;
    s = run_rhs(ctx, q1, B.kxyz, B.vol, B.q, q2, B.ni, B.nj, B.nk, p, flags, 2, dt, tail, st, k32);
    if (s != FJ_OK) return s;
    s = run_rhs(ctx, q2, B.kxyz, B.vol, B.q, B.q, B.ni, B.nj, B.nk, p, flags, 3, dt, tail, st, k32);
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

int fj_ctx_set_pipeline(fj_ctx* ctx, int pipeline, int seg, int tile) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (pipeline != FJ_PIPELINE_FUSED && pipeline != FJ_PIPELINE_STAGED && pipeline != FJ_PIPELINE_SPLIT)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown pipeline");
  if (seg < 0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "segment length must be >= 0");
  if (tile < 0 || tile >= FJ_NUM_TILES) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown tile shape");
  ctx->pipeline = pipeline;
  ctx->seg = seg;
  ctx->tile = tile;
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
  int s = check_step_args(ctx, blocks, q_out, nblocks, links, nlinks, bcs, nbcs, p);
  if (s != FJ_OK) return s;
  size_t stage_b = 0, tail_b = 0;
  s = ensure_ws(ctx, step_layout(ctx, blocks, nblocks, links, nlinks, p, &stage_b, &tail_b));
  if (s != FJ_OK) return s;
  double* q1 = (double*)ctx->ws;
  double* q2 = (double*)((char*)ctx->ws + stage_b);
  void* tail = (char*)ctx->ws + 2 * stage_b;
  return step_body(ctx, blocks, q_out, nblocks, links, nlinks, bcs, nbcs, p, dt, nullptr, q1, q2, tail,
                   tail_b, S(stream));
}

int fj_plan_create(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                   const fj_bc* bcs, int nbcs, const fj_params* p, fj_plan** out) {
  if (!ctx || !out) return FJ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::vector<double*> dummy_out(nblocks > 0 ? nblocks : 1, nullptr);
  for (int b = 0; b < nblocks; ++b) dummy_out[b] = blocks ? blocks[b].q : nullptr;
  int s = check_step_args(ctx, blocks, dummy_out.data(), nblocks, links, nlinks, bcs, nbcs, p);
  if (s != FJ_OK) return s;
  fj_plan* pl = new (std::nothrow) fj_plan();
  if (!pl) return FJ_ERR_NO_MEMORY;
  pl->ctx = ctx;
  pl->blocks.assign(blocks, blocks + nblocks);
  pl->links.assign(links, links + nlinks);
  pl->bcs.assign(bcs, bcs + nbcs);
  pl->p = *p;
  // the plan keeps the context's pipeline choice of its creation time
  pl->pipeline = ctx->pipeline;
  const size_t total = step_layout(ctx, blocks, nblocks, links, nlinks, p, &pl->stage_bytes, &pl->halo_bytes);
  cudaError_t e = cudaMalloc(&pl->scratch, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete pl;
    return set_err(ctx, FJ_ERR_NO_MEMORY, "plan scratch allocation failed");
  }
  if (p->precision == FJ_PREC_F32FLUX) {
    pl->kxyz32.assign(nblocks, nullptr);
    for (int b = 0; b < nblocks; ++b) {
      const size_t n9 = 9 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
      e = cudaMalloc(&pl->kxyz32[b], n9 * sizeof(float));
      if (e != cudaSuccess) {
        cudaGetLastError();
        fj_plan_destroy(pl);
        return set_err(ctx, FJ_ERR_NO_MEMORY, "plan FP32 metric allocation failed");
      }
      s = convert_f64_f32(blocks[b].kxyz, pl->kxyz32[b], (int64_t)n9, nullptr);
      if (s != FJ_OK) {
        fj_plan_destroy(pl);
        return set_err(ctx, s, "plan FP32 metric conversion failed");
      }
    }
    e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) {
      fj_plan_destroy(pl);
      return cuda_status(ctx, e, "plan metric conversion");
    }
  }
  *out = pl;
  return FJ_OK;
}

int fj_plan_step(fj_plan* pl, double* const* q_in, double* const* q_out, double dt, void* stream) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  fj_ctx* ctx = pl->ctx;
  const int nb = (int)pl->blocks.size();
  if (!q_in || !q_out) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "q_in/q_out is NULL");
  std::vector<fj_block> in(pl->blocks);
  for (int b = 0; b < nb; ++b) {
    if (!q_in[b] || !q_out[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "state pointer is NULL");
    in[b].q = q_in[b];
  }
  double* q1 = (double*)pl->scratch;
  double* q2 = (double*)((char*)pl->scratch + pl->stage_bytes);
  void* tail = (char*)pl->scratch + 2 * pl->stage_bytes;
  const int saved = ctx->pipeline;
  ctx->pipeline = pl->pipeline;  // the scratch was laid out for this pipeline
  int s = step_body(ctx, in.data(), q_out, nb, pl->links.data(), (int)pl->links.size(), pl->bcs.data(),
                    (int)pl->bcs.size(), &pl->p, dt, pl->kxyz32.empty() ? nullptr : pl->kxyz32.data(), q1, q2,
                    tail, pl->halo_bytes, S(stream));
  ctx->pipeline = saved;
  return s;
}

int fj_plan_stage(fj_plan* pl, double* const* q, double* const* q0, double* const* out, double dt,
                  int stage, void* stream) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  fj_ctx* ctx = pl->ctx;
  const int nb = (int)pl->blocks.size();
  if (!q || !out || (stage > 1 && !q0)) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "NULL state list");
  if (stage < 1 || stage > 3) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "stage must be 1, 2 or 3");
  for (int b = 0; b < nb; ++b)
    if (!q[b] || !out[b] || (stage > 1 && !q0[b]) || out[b] == q[b])
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad state pointer");
  void* tail = (char*)pl->scratch + 2 * pl->stage_bytes;
  const int flags = kRhsInvscd | kRhsViscous;
  const int saved = ctx->pipeline;
  ctx->pipeline = pl->pipeline;
  int s = FJ_OK;
  if (pl->pipeline == FJ_PIPELINE_SPLIT) {
    std::vector<SplitBlock> sb(nb);
    for (int b = 0; b < nb; ++b) {
      const fj_block& B = pl->blocks[b];
      sb[b] = split_block(q[b], stage > 1 ? q0[b] : q[b], out[b], B.kxyz,
                          pl->kxyz32.empty() ? nullptr : pl->kxyz32[b], B.vol, B.ni, B.nj, B.nk);
    }
    split_assign_scratch(pl->p.precision, sb.data(), nb, tail);
    s = split_stage(ctx, sb.data(), nb, make_phys(&pl->p), flags, stage, dt, pl->p.precision, S(stream));
  } else {
    for (int b = 0; b < nb && s == FJ_OK; ++b) {
      const fj_block& B = pl->blocks[b];
      s = run_rhs(ctx, q[b], B.kxyz, B.vol, stage > 1 ? q0[b] : q[b], out[b], B.ni, B.nj, B.nk, &pl->p, flags,
                  stage, dt, tail, S(stream), pl->kxyz32.empty() ? nullptr : pl->kxyz32[b]);
    }
  }
  ctx->pipeline = saved;
  return s;
}

int fj_rhs_vjp_f64(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
                   const double* lam, double* out, int ni, int nj, int nk, const fj_params* p,
                   void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  int s = check_params(ctx, p);
  if (s != FJ_OK) return s;
  s = check_dims(ctx, ni, nj, nk);
  if (s != FJ_OK) return s;
  if (!q || !kxyz || !vol || !lam || !out) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "NULL array argument");
  s = ensure_ws(ctx, rhs_vjp_ws_bytes(p->precision, ni, nj, nk));
  if (s != FJ_OK) return s;
  return rhs_vjp(ctx, q, kxyz, vol, lam, out, ni, nj, nk, p, kRhsInvscd | kRhsViscous, ctx->ws, S(stream));
}

static int step_vjp_impl(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                         double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                         const fj_bc* bcs, int nbcs, const fj_params* p, double dt, double* dmu,
                         void* stream);

int fj_step_vjp_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                    double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                    const fj_bc* bcs, int nbcs, const fj_params* p, double dt, void* stream) {
  return step_vjp_impl(ctx, blocks, lam_in, lam_out, nblocks, links, nlinks, bcs, nbcs, p, dt, nullptr, stream);
}

int fj_step_vjp_mu_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                       double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                       const fj_bc* bcs, int nbcs, const fj_params* p, double dt, double* dJ_dmu0,
                       void* stream) {
  if (!dJ_dmu0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "dJ_dmu0 is NULL");
  return step_vjp_impl(ctx, blocks, lam_in, lam_out, nblocks, links, nlinks, bcs, nbcs, p, dt, dJ_dmu0, stream);
}

int fj_kinetic_energy_grad_f64(fj_ctx* ctx, const fj_block* blocks, double* const* grad, int nblocks,
                               int ghost, void* stream) {
  if (!ctx || !blocks || !grad || nblocks <= 0 || ghost < 0) return FJ_ERR_INVALID_ARGUMENT;
  for (int b = 0; b < nblocks; ++b) {
    if (!blocks[b].q || !blocks[b].vol || !grad[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "NULL array");
    int s = ke_grad(ctx, blocks[b].q, blocks[b].vol, grad[b], blocks[b].ni, blocks[b].nj, blocks[b].nk, ghost,
                    S(stream));
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

static int step_vjp_impl(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                         double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                         const fj_bc* bcs, int nbcs, const fj_params* p, double dt, double* dmu,
                         void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (!lam_in || !lam_out) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "adjoint lists are NULL");
  std::vector<double*> dummy(nblocks > 0 ? nblocks : 1, nullptr);
  for (int b = 0; b < nblocks; ++b) dummy[b] = blocks ? blocks[b].q : nullptr;
  int s = check_step_args(ctx, blocks, dummy.data(), nblocks, links, nlinks, bcs, nbcs, p);
  if (s != FJ_OK) return s;
  for (int b = 0; b < nblocks; ++b)
    if (!lam_in[b] || !lam_out[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "adjoint pointer is NULL");
  for (int b = 0; b < nbcs; ++b)
    if (bcs[b].type == FJ_BC_WALL && bcs[b].isothermal)
      return set_err(ctx, FJ_ERR_NOT_IMPLEMENTED, "the adjoint of the isothermal wall is not implemented");
  cudaStream_t st = S(stream);
  // layout: [Q0 all blocks][L0 all blocks][Q1][Q2][LA][LB][V][work]
  size_t sum5 = 0, max5 = 0, work = 256;
  for (int b = 0; b < nblocks; ++b) {
    const size_t by = align256(5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double));
    sum5 += by;
    max5 = std::max(max5, by);
    work = std::max(work, rhs_scratch_bytes(ctx, p->precision, blocks[b].ni, blocks[b].nj, blocks[b].nk));
    work = std::max(work, rhs_vjp_ws_bytes(p->precision, blocks[b].ni, blocks[b].nj, blocks[b].nk));
  }
  work = std::max(work, halo_ws_bytes(blocks, links, nlinks, p->ghost));
  work = align256(work);
  s = ensure_ws(ctx, 2 * sum5 + 6 * max5 + work);
  if (s != FJ_OK) return s;
  char* base = (char*)ctx->ws;
  std::vector<fj_block> q0(blocks, blocks + nblocks), l0(blocks, blocks + nblocks);
  size_t off = 0;
  for (int b = 0; b < nblocks; ++b) {
    q0[b].q = (double*)(base + off);
    l0[b].q = (double*)(base + sum5 + off);
    off += align256(5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double));
  }
  double* Q1 = (double*)(base + 2 * sum5);
  double* Q2 = (double*)(base + 2 * sum5 + max5);
  double* LA = (double*)(base + 2 * sum5 + 2 * max5);
  double* LB = (double*)(base + 2 * sum5 + 3 * max5);
  double* V = (double*)(base + 2 * sum5 + 4 * max5);
  double* W = (double*)(base + 2 * sum5 + 5 * max5);  // viscous RHS for dJ/dmu0
  void* wk = base + 2 * sum5 + 6 * max5;
  const double inv_mu = p->mu0 != 0.0 ? 1.0 / p->mu0 : 0.0;
  // c_s dt lam_{s+1} . L_vis(q_s) / mu0
  auto mu_term = [&](const fj_block& B, const double* qs, const double* lam_next, double coef) -> int {
    if (!dmu) return FJ_OK;
    int r = run_rhs(ctx, qs, B.kxyz, B.vol, nullptr, W, B.ni, B.nj, B.nk, p, kRhsViscous, 0, 0.0, wk, st);
    if (r != FJ_OK) return r;
    return dot_acc(ctx, lam_next, W, 5 * (int64_t)B.ni * B.nj * B.nk, coef * dt * inv_mu, dmu, st);
  };
  // ---- forward recompute of q0' (copy + halo + BC)
  for (int b = 0; b < nblocks; ++b) {
    const size_t bytes = 5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double);
    s = cuda_status(ctx, cudaMemcpyAsync(q0[b].q, blocks[b].q, bytes, cudaMemcpyDeviceToDevice, st), "copy");
    if (s != FJ_OK) return s;
  }
  s = halo_exchange(ctx, q0.data(), nblocks, links, nlinks, p->ghost, (double*)wk, work, st);
  if (s != FJ_OK) return s;
  s = apply_bc(ctx, q0.data(), nblocks, bcs, nbcs, p, st);
  if (s != FJ_OK) return s;
  // ---- per block: recompute q1, q2; reverse the three stages
  const int flags = kRhsInvscd | kRhsViscous;
  for (int b = 0; b < nblocks; ++b) {
    const fj_block& B = q0[b];
    const int64_t n5 = 5 * (int64_t)B.ni * B.nj * B.nk;
    double* L0 = l0[b].q;
    s = run_rhs(ctx, B.q, B.kxyz, B.vol, B.q, Q1, B.ni, B.nj, B.nk, p, flags, 1, dt, wk, st);
    if (s == FJ_OK) s = run_rhs(ctx, Q1, B.kxyz, B.vol, B.q, Q2, B.ni, B.nj, B.nk, p, flags, 2, dt, wk, st);
    // stage 3: q3 = 1/3 q0 + 2/3 (q2 + dt L(q2))
    if (s == FJ_OK) s = mu_term(B, Q2, lam_in[b], 2.0 / 3.0);
    if (s == FJ_OK) s = rhs_vjp(ctx, Q2, B.kxyz, B.vol, lam_in[b], V, B.ni, B.nj, B.nk, p, flags, wk, st);
    if (s == FJ_OK) s = axpy3(ctx, LB, lam_in[b], 2.0 / 3.0, V, 2.0 / 3.0 * dt, nullptr, 0.0, n5, st);
    if (s == FJ_OK) s = axpy3(ctx, L0, lam_in[b], 1.0 / 3.0, nullptr, 0.0, nullptr, 0.0, n5, st);
    // stage 2: q2 = 3/4 q0 + 1/4 (q1 + dt L(q1))
    if (s == FJ_OK) s = mu_term(B, Q1, LB, 0.25);
    if (s == FJ_OK) s = rhs_vjp(ctx, Q1, B.kxyz, B.vol, LB, V, B.ni, B.nj, B.nk, p, flags, wk, st);
    if (s == FJ_OK) s = axpy3(ctx, LA, LB, 0.25, V, 0.25 * dt, nullptr, 0.0, n5, st);
    if (s == FJ_OK) s = axpy3(ctx, L0, L0, 1.0, LB, 0.75, nullptr, 0.0, n5, st);
    // stage 1: q1 = q0 + dt L(q0)
    if (s == FJ_OK) s = mu_term(B, B.q, LA, 1.0);
    if (s == FJ_OK) s = rhs_vjp(ctx, B.q, B.kxyz, B.vol, LA, V, B.ni, B.nj, B.nk, p, flags, wk, st);
    if (s == FJ_OK) s = axpy3(ctx, L0, L0, 1.0, LA, 1.0, V, dt, n5, st);
    if (s != FJ_OK) return s;
  }
  // ---- transposed boundary conditions, then transposed halo fill
  s = bc_transpose(ctx, l0.data(), nblocks, bcs, nbcs, p, st);
  if (s != FJ_OK) return s;
  s = halo_transpose(ctx, l0.data(), nblocks, links, nlinks, p->ghost, (double*)wk, work, st);
  if (s != FJ_OK) return s;
  for (int b = 0; b < nblocks; ++b) {
    const size_t bytes = 5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double);
    s = cuda_status(ctx, cudaMemcpyAsync(lam_out[b], l0[b].q, bytes, cudaMemcpyDeviceToDevice, st), "copy");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

int fj_plan_destroy(fj_plan* pl) {
  if (!pl) return FJ_OK;
  for (float* k : pl->kxyz32)
    if (k) cudaFree(k);
  if (pl->scratch) cudaFree(pl->scratch);
  delete pl;
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
