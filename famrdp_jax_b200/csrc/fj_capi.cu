// fj_capi.cu -- the extern "C" entry points of libfamrdp_cuda.so
// (declared in include/famrdp_cuda.h).  Validation, scratch sizing and
// dispatch only; the kernels live in the other translation units.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "famrdp_cuda.h"
#include "fj_common.cuh"
#include "fj_rhs.cuh"
#include "fj_split.cuh"
#include "fj_persist.cuh"
#include "fj_tile.cuh"
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
int reduce_residual(fj_ctx* ctx, const fj_block* blocks, const double* const* prev, int nblocks, int g,
                    double dt, double* res5, cudaStream_t st);
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
                       const void* kaos, const double* vol, int ni, int nj, int nk, double mu0, double dt) {
  SplitBlock b{};
  b.mu0 = mu0;
  b.dt = dt;
  b.q = q;
  b.q0 = q0;
  b.out = out;
  b.kxyz = kxyz;
  b.kaos = kaos;
  b.vol = vol;
  b.ni = ni;
  b.nj = nj;
  b.nk = nk;
  return b;
}

int run_rhs(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
            const double* q0, double* out, int ni, int nj, int nk, const fj_params* p, int flags,
            int stage, double dt, void* ws, cudaStream_t st, const void* kmet = nullptr) {
  // kmet: a plan's metric copy for this block and pipeline (split: records
  // in the flux type; fused, FP32-flux: field-major FP32), or nullptr
  Phys ph = make_phys(p);
  if (ctx->pipeline == FJ_PIPELINE_SPLIT) {
    SplitBlock b = split_block(q, q0, out, kxyz, kmet,
                               vol, ni, nj, nk, p->mu0, dt);
    split_assign_scratch(p->precision, &b, 1, ws);
    return split_stage(ctx, &b, 1, ph, flags, stage, p->precision, st);
  }
  if (ctx->pipeline == FJ_PIPELINE_FUSED) {
    StageArgs a{};
    a.q = q;
    a.q0 = q0;
    a.kxyz = kxyz;
    a.kxyz32 = p->precision == FJ_PREC_F32FLUX ? (const float*)kmet : nullptr;
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
                   int nlinks, const fj_params* p, size_t* stage_b, size_t* tail_b, bool with_tile = false) {
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
  size_t work = split ? split_scratch_bytes(p->precision, cells) : rhs_b;
  // FP32-flux split plans may run the tile kernel, whose padded primitive
  // buffers share the tail with the split intermediates, or the persistent
  // step, whose halo slabs follow the intermediates
  if (split && with_tile && p->precision == FJ_PREC_F32FLUX)
    work = std::max({work, tile_scratch_bytes(blocks, nblocks),
                     persist_tail_bytes(blocks, nblocks, links, nlinks, p->ghost)});
  *tail_b = align256(std::max(std::max(work, halo_ws_bytes(blocks, links, nlinks, p->ghost)), (size_t)256));
  return 2 * *stage_b + *tail_b;
}

// solver/step.py:18-56 on the device: q0p := q, halo + BC in place on q0p,
// then the three stages of each block (blocks do not interact between the halo
// fill and the end of the step, solver/step.py:40-53): q1s := stage 1 of q0p,
// q2s := stage 2, q_out := stage 3.  q0p may equal q_out (the stage-3 kernels
// read q0 only at the cell they write).
// mu0_b / dt_b (nullable): per-block viscosity scale and time step that
// replace p->mu0 and dt (independent instances of an ensemble).
// Plan settings a step runs with (defaults: a plain one-stream step).
struct StepOpts {
  const double* mu0_b = nullptr;  // per-block mu0 / dt (ensembles), or nullptr
  const double* dt_b = nullptr;
  double p_ref = 0.0;             // FP32-flux pressure offset
  int variant = 0;                // FP32 split launch shape
  // two streams: the blocks are split into two groups of about equal cells,
  // each running its three stages on its own stream (blocks are independent
  // between the halo fill and the end of the step), so the groups' launches
  // overlap at kernel boundaries (measured 1-2 % faster on 4 x 128^3; starting
  // the second group half a stage later was slower)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // FP32-flux split plans: run the stages with the fused TMA-tile kernel, or
  // the whole step with the persistent kernel
  const TileMaps* tile = nullptr;
  const PersistPlan* persist = nullptr;
  // split kernels for the stages, the halo, BCs and stage-1 primitives as one
  // persistent launch (the persistent step's work-list head)
  const PersistPlan* fill = nullptr;
  int wait_limit = -1;
};

// The three stages of all blocks with the tile kernel: the primitives of the
// halo-filled start state into padded buffer 0, then stage 1 (buffer 0 ->
// stage result q1 + its primitives in buffer 1), stage 2 (1 -> 0), stage 3.
int tile_step(fj_ctx* ctx, const std::vector<fj_block>& out, double* const* q1s, double* const* q2s,
              double* const* q_out, const fj_params* p, double dt, void* const* kmet, cudaStream_t st,
              const StepOpts& o) {
  const int nb = (int)out.size();
  std::vector<const double*> q0v(nb);
  for (int b = 0; b < nb; ++b) q0v[b] = out[b].q;
  int s = tile_prims(ctx, *o.tile, 0, q0v.data(), out.data(), nb, p->gamma - 1.0, p->R, o.p_ref, st);
  Phys ph = make_phys(p);
  ph.p_ref = o.p_ref;
  std::vector<TileBlock> tb(nb);
  for (int stage = 1; stage <= 3 && s == FJ_OK; ++stage) {
    for (int b = 0; b < nb; ++b) {
      TileBlock& B = tb[b];
      B = TileBlock{};
      B.q = stage == 1 ? out[b].q : (stage == 2 ? q1s[b] : q2s[b]);
      B.q0 = out[b].q;
      B.out = stage == 1 ? q1s[b] : (stage == 2 ? q2s[b] : q_out[b]);
      B.kaos = (const float*)kmet[b];
      B.vol = out[b].vol;
      B.mu0 = o.mu0_b ? o.mu0_b[b] : p->mu0;
      B.dt = o.dt_b ? o.dt_b[b] : dt;
      B.ni = out[b].ni;
      B.nj = out[b].nj;
      B.nk = out[b].nk;
    }
    s = tile_stage(ctx, *o.tile, stage == 2 ? 1 : 0, tb.data(), nb, ph, stage, st, o.wait_limit);
  }
  return s;
}

int step_body(fj_ctx* ctx, const fj_block* blocks, double* const* q0p, double* const* q1s,
              double* const* q2s, double* const* q_out, int nblocks, const fj_link* links, int nlinks,
              const fj_bc* bcs, int nbcs, const fj_params* p, double dt, void* const* kmet, void* tail,
              size_t tail_b, cudaStream_t st, const StepOpts& o = StepOpts{}) {
  const double* mu0_b = o.mu0_b;
  const double* dt_b = o.dt_b;
  const int variant = o.variant;
  std::vector<fj_block> out(blocks, blocks + nblocks);
  int s;
  const bool persist = ctx->pipeline == FJ_PIPELINE_SPLIT && o.persist && p->precision == FJ_PREC_F32FLUX && kmet;
  const bool fused_fill = ctx->pipeline == FJ_PIPELINE_SPLIT && o.fill && p->precision == FJ_PREC_F32FLUX && kmet;
  // the copy and the halo fill as one kernel where the step is not in place
  // (its sources are then the untouched input states); the persistent and
  // fused-fill paths fill the halo themselves
  bool filled = false;
  bool apart = nlinks > 0 && !persist && !fused_fill;
  for (int b = 0; b < nblocks && apart; ++b) apart = q0p[b] != blocks[b].q;
  if (apart) {
    s = copy_fill(ctx, blocks, q0p, nblocks, links, nlinks, p->ghost, st, &filled);
    if (s != FJ_OK) return s;
  }
  for (int b = 0; b < nblocks; ++b) out[b].q = q0p[b];
  if (!filled) {
    // the step's start state into q0p (where the halo, the BCs and the stages
    // work) by an SM copy kernel: captured into a step graph, a memcpy node
    // made graph replays 2-4 % slower than plain launches
    std::vector<const double*> src;
    std::vector<double*> dst;
    std::vector<int64_t> len;
    for (int b = 0; b < nblocks; ++b) {
      out[b].q = q0p[b];
      if (q0p[b] != blocks[b].q) {
        src.push_back(blocks[b].q);
        dst.push_back(q0p[b]);
        len.push_back(5 * (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk);
      }
    }
    if (copy_states(src.data(), dst.data(), len.data(), (int)src.size(), st, &ctx->launches) != FJ_OK)
      return cuda_status(ctx, cudaGetLastError(), "state copy");
  }
  // the persistent kernel: halo, BCs and the three stages in one launch
  if (persist)
    return persist_step(ctx, *o.persist, out.data(), nblocks, q1s, q2s, q_out, p, o.p_ref, mu0_b, dt_b, dt, kmet,
                        tail, o.wait_limit, st);
  if (fused_fill) {
    s = persist_step(ctx, *o.fill, out.data(), nblocks, q1s, q2s, q_out, p, o.p_ref, mu0_b, dt_b, dt, kmet, tail,
                     o.wait_limit, st, true);
  } else {
    if (!filled) {
      s = halo_exchange(ctx, out.data(), nblocks, links, nlinks, p->ghost, (double*)tail, tail_b, st);
      if (s != FJ_OK) return s;
    }
    s = apply_bc(ctx, out.data(), nblocks, bcs, nbcs, p, st);
  }
  if (s != FJ_OK) return s;
  const int flags = kRhsInvscd | kRhsViscous;
  if (ctx->pipeline == FJ_PIPELINE_SPLIT && o.tile && p->precision == FJ_PREC_F32FLUX && kmet)
    return tile_step(ctx, out, q1s, q2s, q_out, p, dt, kmet, st, o);
  if (ctx->pipeline == FJ_PIPELINE_SPLIT) {
    // all blocks per launch; the tail holds the intermediates of every block
    std::vector<SplitBlock> sb(nblocks);
    for (int b = 0; b < nblocks; ++b) {
      const fj_block& B = out[b];
      sb[b] = split_block(B.q, B.q, q1s[b], B.kxyz,
                          kmet ? kmet[b] : nullptr, B.vol, B.ni,
                          B.nj, B.nk, mu0_b ? mu0_b[b] : p->mu0, dt_b ? dt_b[b] : dt);
    }
    split_assign_scratch(p->precision, sb.data(), nblocks, tail);
    Phys ph = make_phys(p);
    ph.p_ref = o.p_ref;
    // the blocks of each stream group; one group unless two streams are set up
    std::vector<int> groups[2];
    const bool two = o.side && nblocks >= 2;
    if (two) {
      std::vector<int> order(nblocks);
      for (int b = 0; b < nblocks; ++b) order[b] = b;
      auto cells = [&](int b) { return (int64_t)out[b].ni * out[b].nj * out[b].nk; };
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
      int64_t load[2] = {0, 0};
      for (int b : order) {
        const int g = load[0] <= load[1] ? 0 : 1;
        groups[g].push_back(b);
        load[g] += cells(b);
      }
      for (auto& g : groups) std::sort(g.begin(), g.end());
    } else {
      for (int b = 0; b < nblocks; ++b) groups[0].push_back(b);
    }
    // stage k of group g: input q_k, output the next stage buffer
    auto stage_group = [&](int g, int stage, cudaStream_t gs, cudaEvent_t after_fluxes) -> int {
      std::vector<SplitBlock> v;
      for (int b : groups[g]) {
        SplitBlock e = sb[b];
        // the primitives alternate between the two buffers from stage to stage
        if (stage == 2) std::swap(e.prim, e.prim_next);
        e.q = stage == 1 ? out[b].q : (stage == 2 ? q1s[b] : q2s[b]);
        e.out = stage == 1 ? q1s[b] : (stage == 2 ? q2s[b] : q_out[b]);
        v.push_back(e);
      }
      if (v.empty()) return FJ_OK;
      // the assembly of stages 1 and 2 also writes the next stage's primitives
      // (the fused ghost fill writes stage 1's)
      return split_stage(ctx, v.data(), (int)v.size(), ph, flags, stage, p->precision, gs, stage > 1 || fused_fill,
                         stage < 3, variant, after_fluxes);
    };
    if (two) {
      s = cuda_status(ctx, cudaEventRecord(o.fork, st), "fork");
      if (s == FJ_OK) s = cuda_status(ctx, cudaStreamWaitEvent(o.side, o.fork, 0), "fork wait");
      if (s != FJ_OK) return s;
    }
    for (int stage = 1; stage <= 3 && s == FJ_OK; ++stage) {
      s = stage_group(0, stage, st, nullptr);
      if (s == FJ_OK && two) s = stage_group(1, stage, o.side, nullptr);
    }
    if (two) {
      // join even after an error so the side stream is not left forked
      const int j = cuda_status(ctx, cudaEventRecord(o.join, o.side), "join");
      const int w = j == FJ_OK ? cuda_status(ctx, cudaStreamWaitEvent(st, o.join, 0), "join wait") : j;
      if (s == FJ_OK) s = w;
    }
    return s;
  }
  for (int b = 0; b < nblocks; ++b) {
    const fj_block& B = out[b];
    const void* k32 = kmet ? kmet[b] : nullptr;
    fj_params pb = *p;
    if (mu0_b) pb.mu0 = mu0_b[b];
    const double dtb = dt_b ? dt_b[b] : dt;
    s = run_rhs(ctx, B.q, B.kxyz, B.vol, B.q, q1s[b], B.ni, B.nj, B.nk, &pb, flags, 1, dtb, tail, st, k32);
    if (s != FJ_OK) return s;
    s = run_rhs(ctx, q1s[b], B.kxyz, B.vol, B.q, q2s[b], B.ni, B.nj, B.nk, &pb, flags, 2, dtb, tail, st, k32);
    if (s != FJ_OK) return s;
    s = run_rhs(ctx, q2s[b], B.kxyz, B.vol, B.q, q_out[b], B.ni, B.nj, B.nk, &pb, flags, 3, dtb, tail, st, k32);
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

// Per-block stage pointers into a [q1 all blocks | q2 all blocks] scratch of
// step_layout's stage_b bytes each (the non-split pipelines run block by block
// and share one block-sized q1/q2).
void stage_ptrs(const fj_ctx* ctx, const fj_block* blocks, int nblocks, void* scratch, size_t stage_b,
                std::vector<double*>& q1s, std::vector<double*>& q2s) {
  q1s.resize(nblocks);
  q2s.resize(nblocks);
  size_t off = 0;
  const bool split = ctx->pipeline == FJ_PIPELINE_SPLIT;
  for (int b = 0; b < nblocks; ++b) {
    q1s[b] = (double*)((char*)scratch + (split ? off : 0));
    q2s[b] = (double*)((char*)scratch + stage_b + (split ? off : 0));
    off += align256(5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double));
  }
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

int fj_ctx_set_adjoint_variant(fj_ctx* ctx, int variant) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (variant < 0 || variant >= FJ_NUM_ADJ_VARIANTS) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown variant");
  ctx->adj_variant = variant;
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

// Shared checks of fj_halo_pack_f64 / fj_halo_unpack_f64: every block's
// dimensions (q may be NULL), the link list and the selection arrays.
static int check_halo_part(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                           int ghost, const int* sel, const int64_t* off, int nsel, const void* buf,
                           int64_t buf_doubles) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (ghost != 2) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "the kernels require ghost == 2");
  if (!blocks || nblocks <= 0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "no blocks");
  for (int b = 0; b < nblocks; ++b) {
    int s = check_dims(ctx, blocks[b].ni, blocks[b].nj, blocks[b].nk);
    if (s != FJ_OK) return s;
  }
  if (nlinks < 0 || (nlinks > 0 && !links)) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad link list");
  if (nsel < 0 || (nsel > 0 && (!sel || !off || !buf)) || buf_doubles < 0)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bad selection or buffer");
  return FJ_OK;
}

int fj_halo_pack_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks, int ghost,
                     const int* sel, const int64_t* off, int nsel, double* buf, int64_t buf_doubles, void* stream) {
  int s = check_halo_part(ctx, blocks, nblocks, links, nlinks, ghost, sel, off, nsel, buf, buf_doubles);
  if (s != FJ_OK) return s;
  return halo_pack_unpack(ctx, blocks, nblocks, links, nlinks, ghost, sel, off, nsel, buf, buf_doubles, false,
                          S(stream));
}

int fj_halo_unpack_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                       int ghost, const int* sel, const int64_t* off, int nsel, const double* buf,
                       int64_t buf_doubles, void* stream) {
  int s = check_halo_part(ctx, blocks, nblocks, links, nlinks, ghost, sel, off, nsel, buf, buf_doubles);
  if (s != FJ_OK) return s;
  return halo_pack_unpack(ctx, blocks, nblocks, links, nlinks, ghost, sel, off, nsel, const_cast<double*>(buf),
                          buf_doubles, true, S(stream));
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
  std::vector<double*> q1s, q2s;
  stage_ptrs(ctx, blocks, nblocks, ctx->ws, stage_b, q1s, q2s);
  void* tail = (char*)ctx->ws + 2 * stage_b;
  return step_body(ctx, blocks, q_out, q1s.data(), q2s.data(), q_out, nblocks, links, nlinks, bcs, nbcs, p, dt,
                   nullptr, tail, tail_b, S(stream));
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
  const size_t total =
      step_layout(ctx, blocks, nblocks, links, nlinks, p, &pl->stage_bytes, &pl->halo_bytes, true);
  cudaError_t e = cudaMalloc(&pl->scratch, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete pl;
    return set_err(ctx, FJ_ERR_NO_MEMORY, "plan scratch allocation failed");
  }
  // metric copies for the FP32-flux path: per-cell FP32 records for the split
  // pipeline, field-major FP32 for the fused kernel (the FP64 kernels read
  // the caller's kxyz)
  const bool split = pl->pipeline == FJ_PIPELINE_SPLIT;
  // the plan's own stream: set-up kernels and later graph captures run on it,
  // never on the legacy stream.  The caller's pending writes of the states
  // and metrics (on any stream) complete first: creation synchronises the
  // device once.
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&pl->capture_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    pl->capture_stream = nullptr;
    fj_plan_destroy(pl);
    return cuda_status(ctx, e, "plan stream creation");
  }
  if (p->precision == FJ_PREC_F32FLUX &&
      (pl->pipeline == FJ_PIPELINE_SPLIT || pl->pipeline == FJ_PIPELINE_FUSED)) {
    pl->kmet.assign(nblocks, nullptr);
    for (int b = 0; b < nblocks; ++b) {
      const int64_t N = (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
      const size_t bytes = split ? split_metric_record_bytes(p->precision, N) : 9 * (size_t)N * sizeof(float);
      e = cudaMalloc(&pl->kmet[b], bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        fj_plan_destroy(pl);
        return set_err(ctx, FJ_ERR_NO_MEMORY, "plan metric copy allocation failed");
      }
      s = split ? split_metric_records(blocks[b].kxyz, pl->kmet[b], blocks[b].ni, blocks[b].nj, blocks[b].nk,
                                       p->precision, pl->capture_stream)
                : convert_f64_f32(blocks[b].kxyz, (float*)pl->kmet[b], 9 * N, pl->capture_stream);
      if (s != FJ_OK) {
        fj_plan_destroy(pl);
        return set_err(ctx, s, "plan metric conversion failed");
      }
    }
    e = cudaStreamSynchronize(pl->capture_stream);
    if (e != cudaSuccess) {
      fj_plan_destroy(pl);
      return cuda_status(ctx, e, "plan metric conversion");
    }
    // the FP32-flux split path offsets the momentum fluxes' pressure by the
    // mean pressure of the state the plan is created with (partial sums in
    // the plan's scratch, which no step has used yet)
    if (split) {
      if (mean_pressure_scratch_bytes(nblocks) <= total)
        s = mean_pressure(blocks, nblocks, p->gamma - 1.0, (double*)pl->scratch, pl->capture_stream, &pl->p_ref);
      else
        s = FJ_ERR_NO_MEMORY;
      if (s != FJ_OK || !std::isfinite(pl->p_ref)) pl->p_ref = 0.0;
    }
    // the fused TMA-tile kernel: padded primitive buffers in the tail and
    // their tensor maps (absent when the driver's encoder is unavailable)
    if (split) {
      TileMaps* tm = new (std::nothrow) TileMaps();
      if (tm && tile_setup(blocks, nblocks, (char*)pl->scratch + 2 * pl->stage_bytes, *tm) &&
          tile_clear_error(*tm, pl->capture_stream) == FJ_OK &&
          cudaStreamSynchronize(pl->capture_stream) == cudaSuccess) {
        pl->tile = tm;
      } else {
        delete tm;
        cudaGetLastError();
      }
      // the persistent step: its work-list and tables (absent when the plan
      // does not qualify, e.g. more than 64 blocks)
      PersistPlan* pp = new (std::nothrow) PersistPlan();
      std::string why;
      if (pp && persist_setup(ctx, blocks, nblocks, links, nlinks, bcs, nbcs, p, *pp, &why)) {
        pl->persist = pp;
      } else {
        delete pp;
        cudaGetLastError();
      }
    }
  }
  *out = pl;
  return FJ_OK;
}

static int plan_step_impl(fj_plan* pl, double* const* q_in, double* const* q_out, double* const* q0_save,
                          double* const* q1_save, double* const* q2_save, double dt, void* stream) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  fj_ctx* ctx = pl->ctx;
  const int nb = (int)pl->blocks.size();
  if (!q_in || !q_out) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "q_in/q_out is NULL");
  std::vector<fj_block> in(pl->blocks);
  for (int b = 0; b < nb; ++b) {
    if (!q_in[b] || !q_out[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "state pointer is NULL");
    in[b].q = q_in[b];
  }
  const int saved = ctx->pipeline;
  ctx->pipeline = pl->pipeline;  // the scratch was laid out for this pipeline
  std::vector<double*> q1s, q2s;
  if (q0_save) {
    q1s.assign(q1_save, q1_save + nb);
    q2s.assign(q2_save, q2_save + nb);
  } else {
    stage_ptrs(ctx, pl->blocks.data(), nb, pl->scratch, pl->stage_bytes, q1s, q2s);
  }
  void* tail = (char*)pl->scratch + 2 * pl->stage_bytes;
  StepOpts opts;
  opts.mu0_b = pl->mu0_b.empty() ? nullptr : pl->mu0_b.data();
  opts.dt_b = pl->dt_b.empty() ? nullptr : pl->dt_b.data();
  opts.p_ref = pl->p_ref;
  opts.variant = pl->variant;
  if (pl->kernel == FJ_KERNEL_TILE && pl->tile) {
    opts.tile = (const TileMaps*)pl->tile;
    opts.wait_limit = pl->wait_limit;
  }
  if (pl->kernel == FJ_KERNEL_PERSIST && pl->persist) {
    opts.persist = (const PersistPlan*)pl->persist;
    opts.wait_limit = pl->wait_limit;
  }
  if (pl->kernel == FJ_KERNEL_SPLIT_FILL && pl->persist) {
    opts.fill = (const PersistPlan*)pl->persist;
    opts.wait_limit = pl->wait_limit;
  }
  if (pl->streams == 2) {
    opts.side = pl->side_stream;
    opts.fork = pl->ev_fork;
    opts.join = pl->ev_join;
  }
  int s = step_body(ctx, in.data(), q0_save ? q0_save : q_out, q1s.data(), q2s.data(), q_out, nb,
                    pl->links.data(), (int)pl->links.size(), pl->bcs.data(), (int)pl->bcs.size(), &pl->p, dt,
                    pl->kmet.empty() ? nullptr : pl->kmet.data(), tail, pl->halo_bytes, S(stream), opts);
  ctx->pipeline = saved;
  return s;
}

int fj_plan_step(fj_plan* pl, double* const* q_in, double* const* q_out, double dt, void* stream) {
  return plan_step_impl(pl, q_in, q_out, nullptr, nullptr, nullptr, dt, stream);
}

static void drop_graphs(fj_plan* pl) {
  for (fj_graph_entry& g : pl->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  pl->graphs.clear();
}

int fj_plan_set_ensemble(fj_plan* pl, const double* mu0, const double* dt) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  const size_t nb = pl->blocks.size();
  if (mu0)
    for (size_t b = 0; b < nb; ++b)
      if (!(mu0[b] >= 0.0)) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "mu0 must be >= 0");
  if (dt)
    for (size_t b = 0; b < nb; ++b)
      if (!(dt[b] >= 0.0) || dt[b] == INFINITY) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "bad dt");
  pl->mu0_b.clear();
  pl->dt_b.clear();
  if (mu0) pl->mu0_b.assign(mu0, mu0 + nb);
  if (dt) pl->dt_b.assign(dt, dt + nb);
  drop_graphs(pl);
  return FJ_OK;
}

int fj_plan_p_ref(const fj_plan* pl, double* out) {
  if (!pl || !out) return FJ_ERR_INVALID_ARGUMENT;
  *out = pl->p_ref;
  return FJ_OK;
}

int fj_plan_set_p_ref(fj_plan* pl, double p_ref) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(p_ref)) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "p_ref must be finite");
  if (p_ref != pl->p_ref) drop_graphs(pl);
  pl->p_ref = p_ref;
  return FJ_OK;
}

int fj_plan_set_variant(fj_plan* pl, int variant) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (variant < 0 || variant >= FJ_NUM_SPLIT_VARIANTS)
    return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "unknown launch-shape variant");
  if (variant != pl->variant) drop_graphs(pl);
  pl->variant = variant;
  return FJ_OK;
}

int fj_plan_set_streams(fj_plan* pl, int n) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (n != 1 && n != 2) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "streams must be 1 or 2");
  if (n == 2 && !pl->side_stream) {
    int s = cuda_status(pl->ctx, cudaStreamCreateWithFlags(&pl->side_stream, cudaStreamNonBlocking), "side stream");
    if (s == FJ_OK)
      s = cuda_status(pl->ctx, cudaEventCreateWithFlags(&pl->ev_fork, cudaEventDisableTiming), "fork event");
    if (s == FJ_OK)
      s = cuda_status(pl->ctx, cudaEventCreateWithFlags(&pl->ev_join, cudaEventDisableTiming), "join event");
    if (s != FJ_OK) return s;
  }
  if (n != pl->streams) drop_graphs(pl);
  pl->streams = n;
  return FJ_OK;
}

int fj_plan_set_kernel(fj_plan* pl, int kernel) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (kernel != FJ_KERNEL_SPLIT && kernel != FJ_KERNEL_TILE && kernel != FJ_KERNEL_PERSIST &&
      kernel != FJ_KERNEL_SPLIT_FILL)
    return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "unknown stage kernel");
  if (kernel == FJ_KERNEL_TILE && !pl->tile)
    return set_err(pl->ctx, FJ_ERR_NOT_IMPLEMENTED,
                   "the tile kernel needs an FP32-flux split plan and the driver's tensor-map encoder");
  if ((kernel == FJ_KERNEL_PERSIST || kernel == FJ_KERNEL_SPLIT_FILL) && !pl->persist)
    return set_err(pl->ctx, FJ_ERR_NOT_IMPLEMENTED,
                   "the persistent step needs an FP32-flux split plan of at most 64 blocks");
  if (kernel != pl->kernel) drop_graphs(pl);
  pl->kernel = kernel;
  return FJ_OK;
}

int fj_plan_set_persist_shape(fj_plan* pl, int shape) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (shape < 0 || shape >= FJ_NUM_PERSIST_SHAPES) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "unknown shape");
  if (!pl->persist)
    return set_err(pl->ctx, FJ_ERR_NOT_IMPLEMENTED,
                   "the persistent step needs an FP32-flux split plan of at most 64 blocks");
  if (shape == pl->persist_shape) return FJ_OK;
  PersistPlan& pp = *(PersistPlan*)pl->persist;
  // the work-list is re-laid out and uploaded: no step of this plan may be in flight
  int s = cuda_status(pl->ctx, cudaDeviceSynchronize(), "persistent shape");
  if (s != FJ_OK) return s;
  if (!persist_reshape(pp, pl->blocks.data(), (int)pl->blocks.size(), kPersistShapes[shape].occ,
                       kPersistShapes[shape].lag_scale))
    return set_err(pl->ctx, FJ_ERR_CUDA, "persistent step work-list upload failed");
  drop_graphs(pl);
  pl->persist_shape = shape;
  return FJ_OK;
}

int fj_plan_get_kernel(const fj_plan* pl, int* kernel) {
  if (!pl || !kernel) return FJ_ERR_INVALID_ARGUMENT;
  *kernel = pl->kernel;
  return FJ_OK;
}

int fj_plan_set_wait_limit(fj_plan* pl, int limit) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (limit < -1) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "limit must be >= -1");
  if (limit != pl->wait_limit) drop_graphs(pl);
  pl->wait_limit = limit;
  return FJ_OK;
}

int fj_plan_check(fj_plan* pl, int* word, void* stream) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  int w = 0, wp = 0;
  int s = FJ_OK;
  if (pl->tile) {
    const TileMaps& tm = *(const TileMaps*)pl->tile;
    s = tile_read_error(tm, &w, S(stream));
    if (s == FJ_OK && w != 0) s = tile_clear_error(tm, S(stream));
  }
  if (s == FJ_OK && pl->persist) {
    const PersistPlan& pp = *(const PersistPlan*)pl->persist;
    s = persist_read_error(pp, &wp, S(stream));
    if (s == FJ_OK && wp != 0) s = persist_clear_error(pp, S(stream));
  }
  if (s == FJ_OK) s = cuda_status(pl->ctx, cudaStreamSynchronize(S(stream)), "plan check");
  if (s != FJ_OK) return s;
  // bit 0: the tile kernel's word; bit 1: the persistent step's
  const int all = (w != 0 ? 1 : 0) | (wp != 0 ? 2 : 0);
  if (word) *word = all;
  if (all == 0) return FJ_OK;
  return set_err(pl->ctx, FJ_ERR_CUDA,
                 std::string("a bounded wait of the ") + (w != 0 ? "tile kernel" : "persistent step") +
                     " gave up (error word " + std::to_string(w != 0 ? w : wp) + ")");
}

int fj_plan_autotune(fj_plan* pl, double* const* q_in, double* const* q_out, double dt, int reps, int* chosen,
                     double* ms_out, void* stream) {
  if (!pl || !chosen || reps < 1) return FJ_ERR_INVALID_ARGUMENT;
  fj_ctx* ctx = pl->ctx;
  const bool split = pl->pipeline == FJ_PIPELINE_SPLIT;
  // the launch shapes of the split kernels, in both precisions
  const bool tunable = split;
  const int nv = tunable ? FJ_NUM_SPLIT_VARIANTS : 1;
  const int ns = split && pl->blocks.size() >= 2 ? 2 : 1;
  const bool with_tile = tunable && pl->p.precision == FJ_PREC_F32FLUX && pl->tile != nullptr;
  const bool with_persist = tunable && pl->p.precision == FJ_PREC_F32FLUX && pl->persist != nullptr;
  if (ms_out)
    for (int i = 0; i < FJ_AUTOTUNE_CANDIDATES; ++i) ms_out[i] = 0.0;
  cudaStream_t st = S(stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int s = cuda_status(ctx, cudaEventCreate(&e0), "event");
  if (s == FJ_OK) s = cuda_status(ctx, cudaEventCreate(&e1), "event");
  const int keep_v = pl->variant, keep_s = pl->streams, keep_k = pl->kernel, keep_p = pl->persist_shape;
  int best_v = keep_v, best_s = keep_s, best_k = keep_k, best_p = keep_p;
  float best_ms = -1.0f;
  // mean step time of the plan's current settings over `reps` steps
  auto time_steps = [&](float& ms) -> int {
    int t = plan_step_impl(pl, q_in, q_out, nullptr, nullptr, nullptr, dt, stream);  // untimed
    if (t == FJ_OK) t = cuda_status(ctx, cudaEventRecord(e0, st), "event record");
    for (int r = 0; r < reps && t == FJ_OK; ++r) t = plan_step_impl(pl, q_in, q_out, nullptr, nullptr, nullptr, dt, stream);
    if (t == FJ_OK) t = cuda_status(ctx, cudaEventRecord(e1, st), "event record");
    if (t == FJ_OK) t = cuda_status(ctx, cudaEventSynchronize(e1), "event sync");
    if (t == FJ_OK) t = cuda_status(ctx, cudaEventElapsedTime(&ms, e0, e1), "event time");
    return t;
  };
  if (s == FJ_OK) s = fj_plan_set_kernel(pl, FJ_KERNEL_SPLIT);
  for (int sn = 1; sn <= ns && s == FJ_OK; ++sn) {
    for (int v = 0; v < nv && s == FJ_OK; ++v) {
      s = fj_plan_set_variant(pl, tunable ? v : keep_v);
      if (s == FJ_OK) s = fj_plan_set_streams(pl, sn);
      float ms = 0.0f;
      if (s == FJ_OK) s = time_steps(ms);
      if (s == FJ_OK) {
        if (ms_out) ms_out[(sn - 1) * FJ_NUM_SPLIT_VARIANTS + v] = ms / reps;
        if (best_ms < 0.0f || ms < best_ms) {
          best_ms = ms;
          best_v = tunable ? v : keep_v;
          best_s = sn;
          best_k = FJ_KERNEL_SPLIT;
        }
      }
    }
  }
  if (with_tile && s == FJ_OK) {
    s = fj_plan_set_streams(pl, 1);
    if (s == FJ_OK) s = fj_plan_set_kernel(pl, FJ_KERNEL_TILE);
    float ms = 0.0f;
    if (s == FJ_OK) s = time_steps(ms);
    if (s == FJ_OK) {
      if (ms_out) ms_out[2 * FJ_NUM_SPLIT_VARIANTS] = ms / reps;
      if (best_ms < 0.0f || ms < best_ms) {
        best_ms = ms;
        best_s = 1;
        best_k = FJ_KERNEL_TILE;
      }
    }
  }
  // the split kernels behind the fused ghost fill, in the best split shape so far
  if (with_persist && s == FJ_OK && best_k == FJ_KERNEL_SPLIT) {
    s = fj_plan_set_variant(pl, best_v);
    if (s == FJ_OK) s = fj_plan_set_streams(pl, best_s);
    if (s == FJ_OK) s = fj_plan_set_kernel(pl, FJ_KERNEL_SPLIT_FILL);
    float ms = 0.0f;
    if (s == FJ_OK) s = time_steps(ms);
    if (s == FJ_OK) {
      if (ms_out) ms_out[2 * FJ_NUM_SPLIT_VARIANTS + 1 + FJ_NUM_PERSIST_SHAPES] = ms / reps;
      if (ms < best_ms) {
        best_ms = ms;
        best_k = FJ_KERNEL_SPLIT_FILL;
      }
    }
  }
  for (int k = 0; with_persist && k < FJ_NUM_PERSIST_SHAPES && s == FJ_OK; ++k) {
    s = fj_plan_set_streams(pl, 1);
    if (s == FJ_OK) s = fj_plan_set_kernel(pl, FJ_KERNEL_PERSIST);
    if (s == FJ_OK) s = fj_plan_set_persist_shape(pl, k);
    float ms = 0.0f;
    if (s == FJ_OK) s = time_steps(ms);
    if (s == FJ_OK) {
      if (ms_out) ms_out[2 * FJ_NUM_SPLIT_VARIANTS + 1 + k] = ms / reps;
      if (best_ms < 0.0f || ms < best_ms) {
        best_ms = ms;
        best_s = 1;
        best_k = FJ_KERNEL_PERSIST;
        best_p = k;
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  int r = fj_plan_set_variant(pl, s == FJ_OK ? best_v : keep_v);
  if (r == FJ_OK) r = fj_plan_set_streams(pl, s == FJ_OK ? best_s : keep_s);
  if (r == FJ_OK) r = fj_plan_set_kernel(pl, s == FJ_OK ? best_k : keep_k);
  if (r == FJ_OK && pl->persist) r = fj_plan_set_persist_shape(pl, s == FJ_OK ? best_p : keep_p);
  if (s == FJ_OK) s = r;
  *chosen = pl->kernel == FJ_KERNEL_TILE         ? 2 * FJ_NUM_SPLIT_VARIANTS
            : pl->kernel == FJ_KERNEL_PERSIST    ? 2 * FJ_NUM_SPLIT_VARIANTS + 1 + pl->persist_shape
            : pl->kernel == FJ_KERNEL_SPLIT_FILL ? 2 * FJ_NUM_SPLIT_VARIANTS + 1 + FJ_NUM_PERSIST_SHAPES
                                                 : pl->variant + FJ_NUM_SPLIT_VARIANTS * (pl->streams - 1);
  return s;
}

int fj_plan_step_graph(fj_plan* pl, double* const* q_in, double* const* q_out, double dt, void* stream) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  fj_ctx* ctx = pl->ctx;
  const int nb = (int)pl->blocks.size();
  if (!q_in || !q_out) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "q_in/q_out is NULL");
  std::vector<double*> in(q_in, q_in + nb), out(q_out, q_out + nb);
  for (int b = 0; b < nb; ++b)
    if (!in[b] || !out[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "state pointer is NULL");
  size_t hit = pl->graphs.size();
  for (size_t g = 0; g < pl->graphs.size(); ++g)
    if (pl->graphs[g].q_in == in && pl->graphs[g].q_out == out && pl->graphs[g].dt == dt) hit = g;
  if (hit == pl->graphs.size()) {
    if (!pl->capture_stream) {
      int s = cuda_status(ctx, cudaStreamCreateWithFlags(&pl->capture_stream, cudaStreamNonBlocking),
                          "capture stream");
      if (s != FJ_OK) return s;
    }
    int s = cuda_status(ctx, cudaStreamBeginCapture(pl->capture_stream, cudaStreamCaptureModeThreadLocal),
                        "begin capture");
    if (s != FJ_OK) return s;
    const int64_t before = ctx->launches;
    s = plan_step_impl(pl, q_in, q_out, nullptr, nullptr, nullptr, dt, pl->capture_stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(pl->capture_stream, &graph);
    const int64_t nlaunch = ctx->launches - before;
    ctx->launches = before;  // nothing has run yet
    if (s == FJ_OK) s = cuda_status(ctx, e, "end capture");
    fj_graph_entry ent;
    if (s == FJ_OK) s = cuda_status(ctx, cudaGraphInstantiate(&ent.exec, graph, 0), "graph instantiate");
    if (graph) cudaGraphDestroy(graph);
    if (s != FJ_OK) {
      cudaGetLastError();
      return s;
    }
    ent.q_in = in;
    ent.q_out = out;
    ent.dt = dt;
    ent.launches = nlaunch;
    if ((int)pl->graphs.size() >= FJ_PLAN_MAX_GRAPHS) {
      cudaGraphExecDestroy(pl->graphs.front().exec);
      pl->graphs.erase(pl->graphs.begin());
    }
    pl->graphs.push_back(ent);
    hit = pl->graphs.size() - 1;
  } else if (hit + 1 != pl->graphs.size()) {
    std::rotate(pl->graphs.begin() + hit, pl->graphs.begin() + hit + 1, pl->graphs.end());
    hit = pl->graphs.size() - 1;
  }
  int s = cuda_status(ctx, cudaGraphLaunch(pl->graphs[hit].exec, S(stream)), "graph launch");
  if (s == FJ_OK) ctx->launches += pl->graphs[hit].launches;
  return s;
}

int fj_plan_step_save(fj_plan* pl, double* const* q_in, double* const* q_out, double* const* q0_save,
                      double* const* q1_save, double* const* q2_save, double dt, void* stream) {
  if (!pl) return FJ_ERR_INVALID_ARGUMENT;
  if (!q0_save || !q1_save || !q2_save) return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "save lists are NULL");
  for (size_t b = 0; b < pl->blocks.size(); ++b)
    if (!q0_save[b] || !q1_save[b] || !q2_save[b])
      return set_err(pl->ctx, FJ_ERR_INVALID_ARGUMENT, "save pointer is NULL");
  return plan_step_impl(pl, q_in, q_out, q0_save, q1_save, q2_save, dt, stream);
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
  if (pl->pipeline == FJ_PIPELINE_SPLIT && pl->kernel == FJ_KERNEL_TILE && pl->tile && !pl->kmet.empty()) {
    // the tile kernel: the primitives of q into padded buffer 0, then the stage
    // (which, for stages 1 and 2, also writes its result's primitives)
    const TileMaps& tm = *(const TileMaps*)pl->tile;
    std::vector<fj_block> in(pl->blocks);
    for (int b = 0; b < nb; ++b) in[b].q = q[b];
    std::vector<const double*> qv(q, q + nb);
    s = tile_prims(ctx, tm, 0, qv.data(), in.data(), nb, pl->p.gamma - 1.0, pl->p.R, pl->p_ref, S(stream));
    Phys ph = make_phys(&pl->p);
    ph.p_ref = pl->p_ref;
    std::vector<TileBlock> tb(nb);
    for (int b = 0; b < nb; ++b) {
      const fj_block& B = pl->blocks[b];
      tb[b] = TileBlock{};
      tb[b].q = q[b];
      tb[b].q0 = stage > 1 ? q0[b] : q[b];
      tb[b].out = out[b];
      tb[b].kaos = (const float*)pl->kmet[b];
      tb[b].vol = B.vol;
      tb[b].mu0 = pl->mu0_b.empty() ? pl->p.mu0 : pl->mu0_b[b];
      tb[b].dt = pl->dt_b.empty() ? dt : pl->dt_b[b];
      tb[b].ni = B.ni;
      tb[b].nj = B.nj;
      tb[b].nk = B.nk;
    }
    if (s == FJ_OK) s = tile_stage(ctx, tm, 0, tb.data(), nb, ph, stage, S(stream), pl->wait_limit);
  } else if (pl->pipeline == FJ_PIPELINE_SPLIT) {
    std::vector<SplitBlock> sb(nb);
    for (int b = 0; b < nb; ++b) {
      const fj_block& B = pl->blocks[b];
      sb[b] = split_block(q[b], stage > 1 ? q0[b] : q[b], out[b], B.kxyz,
                          pl->kmet.empty() ? nullptr : pl->kmet[b], B.vol, B.ni, B.nj, B.nk,
                          pl->mu0_b.empty() ? pl->p.mu0 : pl->mu0_b[b], pl->dt_b.empty() ? dt : pl->dt_b[b]);
    }
    split_assign_scratch(pl->p.precision, sb.data(), nb, tail);
    Phys ph = make_phys(&pl->p);
    ph.p_ref = pl->p_ref;
    s = split_stage(ctx, sb.data(), nb, ph, flags, stage, pl->p.precision, S(stream), false, false, pl->variant);
  } else {
    for (int b = 0; b < nb && s == FJ_OK; ++b) {
      const fj_block& B = pl->blocks[b];
      fj_params pb = pl->p;
      if (!pl->mu0_b.empty()) pb.mu0 = pl->mu0_b[b];
      s = run_rhs(ctx, q[b], B.kxyz, B.vol, stage > 1 ? q0[b] : q[b], out[b], B.ni, B.nj, B.nk, &pb, flags,
                  stage, pl->dt_b.empty() ? dt : pl->dt_b[b], tail, S(stream),
                  pl->kmet.empty() ? nullptr : pl->kmet[b]);
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

static int step_vjp_impl(fj_ctx* ctx, const fj_block* blocks, const double* const* q1_saved,
                         const double* const* q2_saved, const double* const* lam_in, double* const* lam_out,
                         int nblocks, const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs,
                         const fj_params* p, double dt, double* dmu, void* stream, const double* mu0_b = nullptr,
                         const double* dt_b = nullptr, bool dmu_per_block = false);

int fj_step_vjp_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                    double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                    const fj_bc* bcs, int nbcs, const fj_params* p, double dt, void* stream) {
  return step_vjp_impl(ctx, blocks, nullptr, nullptr, lam_in, lam_out, nblocks, links, nlinks, bcs, nbcs, p, dt,
                       nullptr, stream);
}

int fj_step_vjp_mu_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                       double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                       const fj_bc* bcs, int nbcs, const fj_params* p, double dt, double* dJ_dmu0,
                       void* stream) {
  if (!dJ_dmu0) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "dJ_dmu0 is NULL");
  return step_vjp_impl(ctx, blocks, nullptr, nullptr, lam_in, lam_out, nblocks, links, nlinks, bcs, nbcs, p, dt,
                       dJ_dmu0, stream);
}

int fj_step_vjp_saved_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* q1,
                          const double* const* q2, const double* const* lam_in, double* const* lam_out,
                          int nblocks, const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs,
                          const fj_params* p, double dt, double* dJ_dmu0, void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (!q1 || !q2) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "saved stage lists are NULL");
  for (int b = 0; b < nblocks; ++b)
    if (!q1[b] || !q2[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "saved stage pointer is NULL");
  return step_vjp_impl(ctx, blocks, q1, q2, lam_in, lam_out, nblocks, links, nlinks, bcs, nbcs, p, dt, dJ_dmu0,
                       stream);
}

int fj_step_vjp_ensemble_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* q1,
                             const double* const* q2, const double* const* lam_in, double* const* lam_out,
                             int nblocks, const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs,
                             const fj_params* p, double dt, const double* mu0, const double* dts, double* dJ_dmu0,
                             void* stream) {
  if (!ctx) return FJ_ERR_INVALID_ARGUMENT;
  if (!q1 || !q2) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "saved stage lists are NULL");
  for (int b = 0; b < nblocks; ++b)
    if (!q1[b] || !q2[b]) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "saved stage pointer is NULL");
  return step_vjp_impl(ctx, blocks, q1, q2, lam_in, lam_out, nblocks, links, nlinks, bcs, nbcs, p, dt, dJ_dmu0,
                       stream, mu0, dts, true);
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

// Reverse of one step.  Without saved states, q0' (copy + halo + BC), q1 and
// q2 are recomputed first; with them, blocks[b].q is q0' and q1/q2 are read.
// mu0_b / dt_b: per-block overrides (ensembles); dmu_per_block: dmu holds one
// accumulator per block instead of one in total.
static int step_vjp_impl(fj_ctx* ctx, const fj_block* blocks, const double* const* q1_saved,
                         const double* const* q2_saved, const double* const* lam_in, double* const* lam_out,
                         int nblocks, const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs,
                         const fj_params* p, double dt, double* dmu, void* stream, const double* mu0_b,
                         const double* dt_b, bool dmu_per_block) {
  const double dt_all = dt;
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
  const bool saved = q1_saved != nullptr;
  cudaStream_t st = S(stream);
  // layout: [Q0 all blocks, unless saved][L0 all blocks][Q1][Q2][LA][LB][work]
  // (Q1/Q2 only without saved states)
  size_t sum5 = 0, max5 = 0, work = 256;
  for (int b = 0; b < nblocks; ++b) {
    const size_t by = align256(5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double));
    sum5 += by;
    max5 = std::max(max5, by);
    if (!saved) work = std::max(work, rhs_scratch_bytes(ctx, p->precision, blocks[b].ni, blocks[b].nj, blocks[b].nk));
    work = std::max(work, rhs_vjp_ws_bytes(p->precision, blocks[b].ni, blocks[b].nj, blocks[b].nk));
  }
  work = std::max(work, halo_ws_bytes(blocks, links, nlinks, p->ghost));
  work = align256(work);
  const size_t q0_bytes = saved ? 0 : sum5;
  const int nstage = saved ? 0 : 2;
  s = ensure_ws(ctx, q0_bytes + sum5 + (nstage + 2) * max5 + work);
  if (s != FJ_OK) return s;
  char* base = (char*)ctx->ws;
  std::vector<fj_block> q0(blocks, blocks + nblocks), l0(blocks, blocks + nblocks);
  // The adjoint accumulates in lam_out itself when no lam_out array overlaps
  // any array the sweep reads (lam_in, the states); else in scratch, copied
  // out at the end.
  auto bytes5 = [&](int b) { return 5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double); };
  auto overlap = [](const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return b != nullptr && x < y + nb && y < x + na;
  };
  bool direct = true;
  for (int b = 0; b < nblocks && direct; ++b)
    for (int c = 0; c < nblocks && direct; ++c) {
      const size_t nb = bytes5(b), nc = bytes5(c);
      if (overlap(lam_out[b], nb, lam_in[c], nc) || overlap(lam_out[b], nb, blocks[c].q, nc) ||
          (saved && (overlap(lam_out[b], nb, q1_saved[c], nc) || overlap(lam_out[b], nb, q2_saved[c], nc))) ||
          (c != b && overlap(lam_out[b], nb, lam_out[c], nc)))
        direct = false;
    }
  size_t off = 0;
  for (int b = 0; b < nblocks; ++b) {
    if (!saved) q0[b].q = (double*)(base + off);
    l0[b].q = direct ? lam_out[b] : (double*)(base + q0_bytes + off);
    off += align256(bytes5(b));
  }
  char* tail = base + q0_bytes + sum5;
  double* Q1w = saved ? nullptr : (double*)tail;
  double* Q2w = saved ? nullptr : (double*)(tail + max5);
  double* LA = (double*)(tail + nstage * max5);
  double* LB = (double*)(tail + (nstage + 1) * max5);
  void* wk = tail + (nstage + 2) * max5;
  if (!saved) {
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
  }
  // ---- per block: q1, q2 (recomputed or saved); reverse the three stages
  const int flags = kRhsInvscd | kRhsViscous;
  for (int b = 0; b < nblocks; ++b) {
    const fj_block& B = q0[b];
    double* L0 = l0[b].q;
    const double* Q1 = saved ? q1_saved[b] : Q1w;
    const double* Q2 = saved ? q2_saved[b] : Q2w;
    fj_params pb = *p;
    if (mu0_b) pb.mu0 = mu0_b[b];
    const double dt = dt_b ? dt_b[b] : dt_all;
    double* dmu_b = dmu ? (dmu_per_block ? dmu + b : dmu) : nullptr;
    // dJ/dmu0 = sum over stages of c_s dt lam_{s+1} . L_vis(q_s) / mu0 (L_vis is
    // linear in mu0); the viscous VJP kernel accumulates it with this scale.
    const double inv_mu = pb.mu0 != 0.0 ? 1.0 / pb.mu0 : 0.0;
    const fj_params* const pp = &pb;
    if (!saved) {
      s = run_rhs(ctx, B.q, B.kxyz, B.vol, B.q, Q1w, B.ni, B.nj, B.nk, pp, flags, 1, dt, wk, st);
      if (s == FJ_OK) s = run_rhs(ctx, Q1w, B.kxyz, B.vol, B.q, Q2w, B.ni, B.nj, B.nk, pp, flags, 2, dt, wk, st);
      if (s != FJ_OK) return s;
    }
    // stage 3: q3 = 1/3 q0 + 2/3 (q2 + dt L(q2)):
    //   LB = 2/3 lam + 2/3 dt V3   (q0 receives 1/3 lam, added at stage 1)
    VjpEpilogue e3;
    e3.o1 = LB, e3.x1 = lam_in[b], e3.a1 = 2.0 / 3.0, e3.e1 = 2.0 / 3.0 * dt;
    e3.next_q = Q1, e3.next_vol = B.vol;  // leaves the stage-2 VJP's inputs in wk
    s = rhs_vjp(ctx, Q2, B.kxyz, B.vol, lam_in[b], nullptr, B.ni, B.nj, B.nk, pp, flags, wk, st, dmu_b,
                2.0 / 3.0 * dt * inv_mu, &e3);
    // stage 2: q2 = 3/4 q0 + 1/4 (q1 + dt L(q1)):
    //   LA = 1/4 LB + dt/4 V2      (q0 receives 3/4 LB, added at stage 1)
    VjpEpilogue e2;
    e2.o1 = LA, e2.x1 = LB, e2.a1 = 0.25, e2.e1 = 0.25 * dt;
    e2.next_q = B.q, e2.next_vol = B.vol, e2.ws_ready = true;
    if (s == FJ_OK)
      s = rhs_vjp(ctx, Q1, B.kxyz, B.vol, LB, nullptr, B.ni, B.nj, B.nk, pp, flags, wk, st, dmu_b,
                  0.25 * dt * inv_mu, &e2);
    // stage 1: q1 = q0 + dt L(q0):  L0 = 1/3 lam + 3/4 LB + LA + dt V1
    // (L0 is read by no stage, so each of its cells is written once)
    VjpEpilogue e1;
    e1.o1 = L0, e1.x1 = lam_in[b], e1.a1 = 1.0 / 3.0, e1.y1 = LB, e1.b1 = 0.75, e1.z1 = LA, e1.c1 = 1.0;
    e1.e1 = dt, e1.ws_ready = true;
    if (s == FJ_OK)
      s = rhs_vjp(ctx, B.q, B.kxyz, B.vol, LA, nullptr, B.ni, B.nj, B.nk, pp, flags, wk, st, dmu_b, dt * inv_mu,
                  &e1);
    if (s != FJ_OK) return s;
  }
  // ---- transposed boundary conditions, then transposed halo fill
  s = bc_transpose(ctx, l0.data(), nblocks, bcs, nbcs, p, st);
  if (s != FJ_OK) return s;
  s = halo_transpose(ctx, l0.data(), nblocks, links, nlinks, p->ghost, (double*)wk, work, st);
  if (s != FJ_OK) return s;
  if (direct) return FJ_OK;
  for (int b = 0; b < nblocks; ++b) {
    const size_t bytes = 5 * (size_t)blocks[b].ni * blocks[b].nj * blocks[b].nk * sizeof(double);
    s = cuda_status(ctx, cudaMemcpyAsync(lam_out[b], l0[b].q, bytes, cudaMemcpyDeviceToDevice, st), "copy");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

int fj_plan_destroy(fj_plan* pl) {
  if (!pl) return FJ_OK;
  for (fj_graph_entry& g : pl->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (pl->capture_stream) cudaStreamDestroy(pl->capture_stream);
  if (pl->side_stream) cudaStreamDestroy(pl->side_stream);
  if (pl->ev_fork) cudaEventDestroy(pl->ev_fork);
  if (pl->ev_join) cudaEventDestroy(pl->ev_join);
  for (void* k : pl->kmet)
    if (k) cudaFree(k);
  if (pl->scratch) cudaFree(pl->scratch);
  delete (TileMaps*)pl->tile;
  delete (PersistPlan*)pl->persist;
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

int fj_residual_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* q_prev, int nblocks, int ghost,
                    double dt, double* res_out, void* stream) {
  if (!ctx || !res_out || ghost < 0) return FJ_ERR_INVALID_ARGUMENT;
  return reduce_residual(ctx, blocks, q_prev, nblocks, ghost, dt, res_out, S(stream));
}

}  // extern "C"
