// fj_common.cuh -- shared host/device plumbing of libfamrdp_cuda.so: the
// context, status handling and launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <utility>
#include <vector>

#include "famrdp_cuda.h"

struct fj_ctx {
  int device = 0;
  void* ws = nullptr;        // scratch owned by the context (stage buffers, fluxes)
  size_t ws_bytes = 0;
  void* red = nullptr;       // small reduction scratch (partials + counters)
  size_t red_bytes = 0;
  std::string last_error;
  int64_t launches = 0;      // kernels launched through this context
  int pipeline = FJ_PIPELINE_SPLIT;
  int seg = 0;               // fused kernel: planes per CTA along i (0 = automatic)
  int tile = 0;              // fused kernel: tile shape index (FJ_NUM_TILES shapes)
  int adj_variant = 0;       // face-VJP register cap (FJ_NUM_ADJ_VARIANTS)
};

// One captured step (fj_plan_step_graph) for a fixed set of state pointers
// and dt.
struct fj_graph_entry {
  std::vector<double*> q_in, q_out;
  double dt = 0.0;
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;  // kernels in the graph
};

// A prepared step of one block set (fj_plan_create): tables, the metric
// pointers, metric copies in the layout of the plan's pipeline, and owned
// scratch.
struct fj_plan {
  fj_ctx* ctx = nullptr;
  std::vector<fj_block> blocks;
  std::vector<fj_link> links;
  std::vector<fj_bc> bcs;
  fj_params p{};
  std::vector<void*> kmet;  // per-block metric copy for the plan's pipeline (or empty)
  void* scratch = nullptr;   // q1 | q2 | tail (intermediates, halo slabs)
  size_t stage_bytes = 0, halo_bytes = 0;  // halo_bytes: size of the tail
  int pipeline = 0;
  std::vector<double> mu0_b, dt_b;        // per-block overrides (ensembles), empty = none
  double p_ref = 0.0;                     // FP32-flux split path: momentum-flux pressure offset
  int variant = 0;                        // launch shape of the FP32 split kernels
  int streams = 1;                        // 1, or 2: block groups on two streams
  cudaStream_t side_stream = nullptr;     // the second stream and its fork/join events
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t capture_stream = nullptr;  // private stream for graph capture
  std::vector<fj_graph_entry> graphs;     // most recently used last
  // FP32-flux split plans: which stage kernels run (FJ_KERNEL_SPLIT: the three
  // split kernels; FJ_KERNEL_TILE: the fused TMA-tile kernel), the tile
  // kernel's plan data (fj::TileMaps, owned; nullptr when unavailable) and its
  // bounded-wait limit (-1: the default)
  int kernel = FJ_KERNEL_SPLIT;
  void* tile = nullptr;
  void* persist = nullptr;  // FJ_KERNEL_PERSIST's plan data (fj::PersistPlan, owned; nullptr when unavailable)
  int persist_shape = 0;    // its launch shape (FJ_NUM_PERSIST_SHAPES)
  int wait_limit = -1;
};

namespace fj {

constexpr int kThreads = 256;

inline int set_err(fj_ctx* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

inline int cuda_status(fj_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FJ_OK;
  if (ctx) ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return FJ_ERR_CUDA;
}

// Status of the last launch (cudaGetLastError clears the sticky-free error).
inline int launch_status(fj_ctx* ctx, const char* what) {
  return cuda_status(ctx, cudaGetLastError(), what);
}

inline int grid_for(int64_t n, int threads = kThreads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (1LL << 30)) b = (1LL << 30);
  return (int)b;
}

// Grows the context's scratch to at least `bytes` (contents not preserved).
inline int ensure_ws(fj_ctx* ctx, size_t bytes) {
  if (ctx->ws_bytes >= bytes) return FJ_OK;
  if (ctx->ws) {
    cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
  }
  cudaError_t e = cudaMalloc(&ctx->ws, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, FJ_ERR_NO_MEMORY,
                   "scratch allocation of " + std::to_string(bytes) + " bytes failed: " +
                       cudaGetErrorString(e));
  }
  ctx->ws_bytes = bytes;
  return FJ_OK;
}

inline int ensure_red(fj_ctx* ctx, size_t bytes) {
  if (ctx->red_bytes >= bytes) return FJ_OK;
  if (ctx->red) {
    cudaFree(ctx->red);
    ctx->red = nullptr;
    ctx->red_bytes = 0;
  }
  cudaError_t e = cudaMalloc(&ctx->red, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, FJ_ERR_NO_MEMORY, "reduction scratch allocation failed");
  }
  ctx->red_bytes = bytes;
  return FJ_OK;
}

inline int check_params(fj_ctx* ctx, const fj_params* p) {
  if (!p) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "params is NULL");
  if (p->ghost != 2)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "the kernels require ghost == 2");
  if (p->limiter != FJ_LIM_MINMOD && p->limiter != FJ_LIM_VANLEER)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown limiter");
  if (p->visc_law != FJ_VISC_SUTHERLAND && p->visc_law != FJ_VISC_CONSTANT)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown viscosity law");
  if (p->precision != FJ_PREC_F64 && p->precision != FJ_PREC_F32FLUX)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unknown precision");
  return FJ_OK;
}

inline int check_dims(fj_ctx* ctx, int ni, int nj, int nk) {
  // The widest stencil (MUSCL + face difference) needs 5 cells per axis.
  if (ni < 5 || nj < 5 || nk < 5)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "every padded extent must be >= 5");
  if ((int64_t)ni * nj * nk > (int64_t)INT32_MAX / 9)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "block too large for 32-bit cell indexing");
  return FJ_OK;
}

// Physics constants passed by value to kernels.
struct Phys {
  double gm1, eps_entropy, R, mu0, T0, Ts, cp, Pr;
  // derived once on the host: 1/(gamma-1), 1/T0, T0+Ts, cp/Pr
  double inv_gm1, inv_T0, sfac, kap_fac;
  int limiter, visc_law;
  // FP32-flux split path with metric records only: the pressure offset of the
  // momentum fluxes (roe_prim), added back in FP64 in the assembly; 0 elsewhere
  double p_ref = 0.0;
};

inline Phys make_phys(const fj_params* p) {
  Phys f;
  f.gm1 = p->gamma - 1.0;
  f.eps_entropy = p->eps_entropy;
  f.R = p->R;
  f.mu0 = p->mu0;
  f.T0 = p->T0;
  f.Ts = p->Ts;
  // kappa = cp * mu / Pr with cp = gamma R / (gamma - 1) (rhs/viscous.py:38-39)
  f.cp = p->gamma * p->R / (p->gamma - 1.0);
  f.Pr = p->Pr;
  f.inv_gm1 = 1.0 / f.gm1;
  f.inv_T0 = 1.0 / f.T0;
  f.sfac = f.T0 + f.Ts;
  f.kap_fac = f.cp / f.Pr;
  f.limiter = p->limiter;
  f.visc_law = p->visc_law;
  return f;
}

// Programmatic dependent launch.  A kernel launched with pdl_launch may be
// scheduled while the previous kernel on its stream drains; it calls
// grid_dep_wait() before its first load or store of data another kernel
// writes (L2 prefetches may come first: L2 is coherent with the writes still
// in flight), which blocks until the previous grid has completed and its
// writes are visible.  Only the launch latency overlaps; without the launch
// attribute the wait returns at once.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... Exp, typename... Act>
inline cudaError_t pdl_launch(void (*k)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Act&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Act>(args)...);
}

// Starts an L2 fill of the bytes [p, p + n) of one contiguous range, clipped
// inward to 16-byte boundaries so that nothing outside the range is touched.
// Issued by one thread for a CTA's whole cell range, it puts every stream the
// CTA will read in flight at once; the threads' own loads then hit L2 (or
// join the fill) instead of each waiting for DRAM in turn.
__device__ __forceinline__ void l2_prefetch(const void* p, int64_t n) {
  const uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15;
  const uintptr_t e = ((uintptr_t)p + n) & ~(uintptr_t)15;
  if (e > a)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

}  // namespace fj
