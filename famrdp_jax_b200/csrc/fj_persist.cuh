// fj_persist.cuh -- the persistent step kernel (fj_step_persist.cu): one
// whole TVD-RK3 step of all blocks (FP32 fluxes, FP64 state) in ONE launch
// over a work-list whose items are the halo gathers and scatters, the
// boundary-condition faces, the primitives and the flux and assembly chunks
// of the three stages, ordered so that each item only waits for items ahead
// of it (device-side completion counters, bounded waits).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "fj_common.cuh"

namespace fj {

constexpr int kPersistMaxBlocks = 64;

// Launch shapes (FJ_NUM_PERSIST_SHAPES): resident CTAs per SM and the lag of
// the assembly chunks behind the flux chunks they read, in units of half the
// resident CTAs (about the flux chunks in flight); a negative lag mixes each
// sweep's assembly chunks into the next sweep's (another block's) flux chunks.
struct PersistShape {
  int occ;
  double lag_scale;
};
// Shape 0 (each sweep's assembly chunks after all its flux chunks) measured
// fastest: any mixing of the two kinds of chunks made the step slower.
constexpr PersistShape kPersistShapes[] = {{4, 1e6}, {3, 1e6}, {4, -1.0}, {4, 3.0}};
static_assert(sizeof(kPersistShapes) / sizeof(kPersistShapes[0]) == FJ_NUM_PERSIST_SHAPES, "shape table");

// Host-side plan data of the persistent step: the work-list and the
// pointer-free halo and BC descriptor tables in device memory, the control
// block (per-launch counters and a sticky error word) and the launch shape.
struct PersistPlan {
  void* items = nullptr;  // uint2 per item, device
  int n_items = 0;
  void* links = nullptr;  // hd::HaloDesc per link, device
  void* bcs = nullptr;    // hd::BcDesc per boundary face, device
  int nlinks = 0, nbcs = 0;
  int* ctl = nullptr;      // control block, device (ctl_ints ints)
  int ctl_ints = 0, reset_from = 0;  // the per-launch part: [reset_from, ctl_ints)
  int n_gather = 0;        // gather items (the scatters wait for all of them)
  std::vector<uint2> head;  // the halo, BC and primitive items (the part of the list the shape leaves alone)
  std::vector<int> scatter_total, bc_prefix, plane_base;  // per block (bc_prefix: 7 per block)
  std::vector<int> link_tgt, bc_block;  // per link its target block, per boundary entry its block
  int total_planes = 0;
  size_t split_bytes = 0;  // offset of the halo slabs in the tail (after the intermediates)
  int grid = 0;            // resident CTAs (occupancy x SMs)
  int occ = 4;             // CTAs per SM the kernel instantiation is built for
  int lag = 0;             // flux chunks an assembly chunk trails the last flux chunk it needs by
  PersistPlan() = default;
  PersistPlan(const PersistPlan&) = delete;
  PersistPlan& operator=(const PersistPlan&) = delete;
  ~PersistPlan();
};

// Bytes of plan scratch tail the persistent step needs: the split
// intermediates of all blocks and, after them, the halo slabs (the halo
// items run while other blocks' flux items already write intermediates).
size_t persist_tail_bytes(const fj_block* blocks, int nblocks, const fj_link* links, int nlinks, int ghost);
// Builds the work-list and tables of a plan (FP32-flux split plans with
// metric records, at most kPersistMaxBlocks blocks).  Returns false with the
// reason in *why when the plan does not qualify or set-up failed.
bool persist_setup(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                   const fj_bc* bcs, int nbcs, const fj_params* p, PersistPlan& pp, std::string* why);
// Rebuilds the work-list with another launch shape: occ CTAs per SM (3 or 4)
// and lag_scale (see kPersistShapes).  Refuses (false) a list in which an
// item would wait for one behind it.
bool persist_reshape(PersistPlan& pp, const fj_block* blocks, int nblocks, int occ, double lag_scale);
// One step: blocks[b].q is the step's start state (written in place by the
// halo and BC items), q1s / q2s / q_out the stage results.  tail: the plan
// tail (persist_tail_bytes); kmet: the FP32 metric records.  fill_only: only
// the list's head -- halo gathers and scatters, BC faces and the stage-1
// primitives (into the split layout's first primitive buffer) -- in one
// launch; the caller runs the stages with the split kernels.
int persist_step(fj_ctx* ctx, const PersistPlan& pp, const fj_block* blocks, int nblocks, double* const* q1s,
                 double* const* q2s, double* const* q_out, const fj_params* p, double p_ref, const double* mu0_b,
                 const double* dt_b, double dt, void* const* kmet, void* tail, int wait_limit, cudaStream_t st,
                 bool fill_only = false);
// The sticky error word (nonzero: a bounded wait gave up); clear resets it.
int persist_read_error(const PersistPlan& pp, int* out, cudaStream_t st);
int persist_clear_error(const PersistPlan& pp, cudaStream_t st);

}  // namespace fj
