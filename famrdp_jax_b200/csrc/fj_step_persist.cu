// fj_step_persist.cu -- one TVD-RK3 step of all blocks (FP32 fluxes, FP64
// state; solver/step.py:18-56) in ONE persistent launch.
//
// Work-list.  The host lays out, once per plan, the items of a step in an
// order in which every item depends only on items ahead of it:
//   1. halo gathers of every CUT1TO1 link into scratch (mesh/halo.py:89-90:
//      all sources are read before any target is written);
//   2. halo scatters, in link order (the later link wins where slabs overlap);
//   3. boundary-condition faces in Face order (physics/bc/dispatch.py:15),
//      each after every scatter into its block and its block's earlier faces;
//   4. the primitives of each block's halo-filled state;
//   5. per stage, per block, a wavefront of flux chunks (224 cells: the
//      viscous components and the i and j faces, k_split_fluxes) and
//      assembly chunks (217 cells: the k faces, the flux differences, the
//      viscous divergence and the RK3 combine, k_split_assemble), each
//      assembly chunk trailing the last flux chunk it reads by `lag` chunks,
//      so that flux work (issue-bound) and assembly work (bound by loads)
//      share the SMs and the intermediates are read back while still in L2.
// A grid of resident CTAs takes items from an atomic counter; in each CTA a
// scheduler warp claims items, waits (bounded) for the completion counters
// of what an item reads and publishes completions, while seven worker warps
// compute the items it hands over (k_step_persist).  An item waits for:
//   scatter   all gathers;
//   BC face   all scatters into its block, its block's BC items of earlier faces;
//   primitive all scatters into and BC items of its block;
//   flux s    stage 1: all primitive chunks of its block; stages 2, 3: all
//             assembly chunks of the previous stage of its block (the
//             periodic i wrap of the viscous stencil makes plane 0 depend on
//             plane ni-1, so a stage cannot start on a block before the
//             previous stage is done with all of it);
//   assembly  the flux chunks of the i-planes next to its own (p-1 .. p+1,
//             and the far end plane for the wrap at planes 0 and ni-1);
// then is computed, and its counter is bumped (release).  Because every wait
// is for an item taken earlier, by a CTA that is running, no item waits for
// an item that cannot start: the launch needs no co-residency guarantee
// (schedule() keeps this true for the items a CTA holds back).
// The arithmetic is the split kernels' (fj_split_dev.cuh) with plain loads
// in place of the read-only path (the intermediates are written within the
// launch), so a step is bit-identical to the three-kernel pipeline's.
// Bounded waits: a wait that runs out sets the sticky error word and an abort
// flag; every CTA then stops taking items and exits.  No trap, no hang.
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>

#include "fj_halo_dev.cuh"
#include "fj_persist.cuh"
#include "fj_split_dev.cuh"

namespace fj {

namespace {

using namespace sd;
using hd::BcDesc;
using hd::HaloDesc;

// Control block (ints).  [0] the sticky error word; from kCtlReset on,
// zeroed before every launch: the work counter, the abort flag and the
// completion counters.
constexpr int kCtlErr = 0;
constexpr int kCtlReset = 32;
constexpr int kCtlNext = 32, kCtlAbort = 33, kCtlGather = 34;
constexpr int kCtlScatter = 64;   // + block
constexpr int kCtlBc = 128;       // + block
constexpr int kCtlPrims = 192;    // + block
constexpr int kCtlAsm = 256;      // + 64 (stage - 1) + block
constexpr int kCtlFlux = 448;     // + (stage - 1) total_planes + plane_base[block] + plane
static_assert(kCtlAsm + 3 * kPersistMaxBlocks <= kCtlFlux, "control block layout");
static_assert(kPersistMaxBlocks <= kMaxSplitBlocks, "block table");

// Item codes: type | stage << 4 | face << 8 | index << 12 (block, link or BC
// entry); the second word is the chunk.
enum : uint32_t { kItGather = 0, kItScatter = 1, kItBc = 2, kItPrims = 3, kItFlux = 4, kItAsm = 5 };
constexpr int kHaloChunk = 2048;  // slab elements per halo / BC item
// A CTA is seven worker warps and one scheduler warp (see k_step_persist).
constexpr int kWorkWarps = 7;
constexpr int kWorkThreads = kWorkWarps * 32;
constexpr int kCtaThreads = kWorkThreads + 32;
static_assert(kCtaThreads == kSplitThreads, "launch bounds");
constexpr int kFluxCells = kWorkThreads;       // cells per flux / primitive chunk (one per worker thread)
constexpr int kAsmCellsP = kWorkWarps * 31;    // cells per assembly chunk (31 per worker warp)
constexpr int kFlags = kRhsInvscd | kRhsViscous;
// Waits give up after this many polls (64-256 ns apart: about a second)
// unless the plan sets a limit.
constexpr long long kDefaultWaitPolls = 1ll << 22;

inline uint32_t item_code(uint32_t type, int stage, int face, int idx) {
  return type | (uint32_t)stage << 4 | (uint32_t)face << 8 | (uint32_t)idx << 12;
}

struct PersistParams {
  Table tab;  // q = q0 = the step's start state; prim: buffer 0, prim_next: buffer 1
  double* qs[kPersistMaxBlocks][3];  // stage results q1, q2, q_out
  Phys ph;
  double gamma, gm1, R, iR;
  const uint2* items;
  const HaloDesc* links;
  const BcDesc* bcs;
  double* halo;
  int* ctl;
  int n_items, nlinks, ghost, wait_limit, n_gather, total_planes;
  int scatter_total[kPersistMaxBlocks];
  int bc_prefix[kPersistMaxBlocks][7];  // BC items of the block's faces before face f; [6]: all
  int plane_base[kPersistMaxBlocks];
};
static_assert(sizeof(PersistParams) <= 32764, "kernel parameter space");

__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__host__ __device__ __forceinline__ int64_t chunks_of(int64_t n, int64_t per) { return (n + per - 1) / per; }

// Flux chunks (kFluxCells cells) that overlap i-plane q of a block with si
// cells per plane (32-bit: a block's cell count is below 2^27).
__device__ __forceinline__ int flux_chunks_in_plane(uint32_t si, int q) {
  return (int)(((uint32_t)(q + 1) * si - 1) / kFluxCells - ((uint32_t)q * si) / kFluxCells + 1);
}

__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void red_add(int* p, int v) {
  asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The completion counters an item waits for (see the file comment), as
// (counter, target) pairs 0 .. n-1; dep_pair returns n and, for i < n, pair i.
__device__ int dep_pair(const PersistParams& P, uint32_t code, int chunk, int i, const int*& p, int& target) {
  const int type = code & 15, stage = (code >> 4) & 15, face = (code >> 8) & 15, idx = (int)(code >> 12);
  const int* const ctl = P.ctl;
  p = nullptr;
  target = 0;
  switch (type) {
    case kItGather:
      return 0;
    case kItScatter:
      if (i == 0) p = ctl + kCtlGather, target = P.n_gather;
      return 1;
    case kItBc: {
      const int X = P.bcs[idx].block;
      if (i == 0) p = ctl + kCtlScatter + X, target = P.scatter_total[X];
      if (i == 1) p = ctl + kCtlBc + X, target = P.bc_prefix[X][face];
      return 2;
    }
    case kItPrims:
      if (i == 0) p = ctl + kCtlScatter + idx, target = P.scatter_total[idx];
      if (i == 1) p = ctl + kCtlBc + idx, target = P.bc_prefix[idx][6];
      return 2;
    case kItFlux: {
      const SplitBlock& B = P.tab.b[idx].blk;
      const uint32_t N = (uint32_t)B.ni * B.nj * B.nk;
      if (i == 0) {
        if (stage == 1) p = ctl + kCtlPrims + idx, target = (int)((N + kFluxCells - 1) / kFluxCells);
        else p = ctl + kCtlAsm + kPersistMaxBlocks * (stage - 2) + idx, target = (int)((N + kAsmCellsP - 1) / kAsmCellsP);
      }
      return 1;
    }
    default: {  // kItAsm: the flux planes lo .. hi, then the periodic i wrap's far plane
      // (32-bit: a block's cell count is below 2^27)
      const SplitBlock& B = P.tab.b[idx].blk;
      const uint32_t si = (uint32_t)B.nj * B.nk, N = si * B.ni;
      const uint32_t c0 = (uint32_t)chunk * kAsmCellsP, c1 = min(c0 + kAsmCellsP, N) - 1;
      const int pl0 = (int)(c0 / si), pl1 = (int)(c1 / si);
      const int lo = max(pl0 - 1, 0), hi = min(pl1 + 1, B.ni - 1);
      const bool wrap_hi = pl0 == 0 && hi < B.ni - 1, wrap_lo = pl1 == B.ni - 1 && lo > 0;
      const int n = hi - lo + 1 + (wrap_hi ? 1 : 0) + (wrap_lo ? 1 : 0);
      int q = -1;
      if (i <= hi - lo) q = lo + i;
      else if (i == hi - lo + 1) q = wrap_hi ? B.ni - 1 : 0;
      else if (i == hi - lo + 2) q = 0;
      if (q >= 0 && i < n) {
        p = ctl + kCtlFlux + (stage - 1) * P.total_planes + P.plane_base[idx] + q;
        target = flux_chunks_in_plane(si, q);
      }
      return n;
    }
  }
}

// Scheduler warp: whether every counter the item waits for has reached its
// target, the lanes polling the (counter, target) pairs in parallel (relaxed
// loads; the caller fences once they have).  The pairs are set up once.
// soft: at most `looks` looks 128 ns apart that neither wait longer nor
// record anything (false: not yet).  Otherwise each lane polls at most the
// wait limit times (0: give up at once if there is anything to wait for;
// negative: the default); giving up records the error and raises the abort
// flag, and an abort raised elsewhere ends the wait as well.
__device__ bool deps_wait(const PersistParams& P, uint2 it, bool soft, int looks) {
  const unsigned all = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int* p0;
  int t0;
  const int n = dep_pair(P, it.x, (int)it.y, 0, p0, t0);
  const long long lim = P.wait_limit < 0 ? kDefaultWaitPolls : (long long)P.wait_limit;
  for (int base = 0; base < n; base += 32) {
    const int* p = nullptr;
    int target = 0;
    if (base + lane < n) dep_pair(P, it.x, (int)it.y, base + lane, p, target);
    const bool need = p != nullptr && target > 0;
    bool ok = !need || ld_relaxed(p) >= target;
    if (soft) {
      for (int look = 1; look < looks && !__all_sync(all, ok); ++look) {
        __nanosleep(128);
        if (!ok) ok = ld_relaxed(p) >= target;
      }
      if (!__all_sync(all, ok)) return false;
      continue;
    }
    if (lim == 0 && __any_sync(all, need)) ok = false;  // give up at once
    for (long long poll = 0; !__all_sync(all, ok); ++poll) {
      int give_up = poll >= lim;
      if (lane == 0 && !give_up && ld_relaxed(P.ctl + kCtlAbort) != 0) give_up = 2;
      give_up = __shfl_sync(all, give_up, 0);
      if (give_up) {
        if (lane == 0 && give_up == 1) {
          atomicOr(P.ctl + kCtlErr, 1);
          atomicExch(P.ctl + kCtlAbort, 1);
        }
        return false;
      }
      __nanosleep(poll < 64 ? 64 : 256);
      if (!ok) ok = ld_relaxed(p) >= target;
    }
  }
  return true;
}

// Scheduler lane 0, once the workers are done with the item: publish its
// completion (the workers' writes are ordered before this by the named
// barrier; the fence makes them visible at device scope before the counts).
__device__ void item_done(const PersistParams& P, uint2 it) {
  const uint32_t code = it.x;
  const int chunk = (int)it.y;
  const int type = code & 15, stage = (code >> 4) & 15, idx = (int)(code >> 12);
  int* const ctl = P.ctl;
  fence_acq_rel();
  switch (type) {
    case kItGather: red_add(ctl + kCtlGather, 1); break;
    case kItScatter: red_add(ctl + kCtlScatter + P.links[idx].tgt_block, 1); break;
    case kItBc: red_add(ctl + kCtlBc + P.bcs[idx].block, 1); break;
    case kItPrims: red_add(ctl + kCtlPrims + idx, 1); break;
    case kItFlux: {
      const SplitBlock& B = P.tab.b[idx].blk;
      const uint32_t si = (uint32_t)B.nj * B.nk, N = si * B.ni;
      const uint32_t c0 = (uint32_t)chunk * kFluxCells, c1 = min(c0 + kFluxCells, N) - 1;
      int* f = ctl + kCtlFlux + (stage - 1) * P.total_planes + P.plane_base[idx];
      for (int q = (int)(c0 / si); q <= (int)(c1 / si); ++q) red_add(f + q, 1);
      break;
    }
    default: red_add(ctl + kCtlAsm + kPersistMaxBlocks * (stage - 1) + idx, 1);
  }
}

// Worker threads (threadIdx.x < kWorkThreads): the item's work.
__device__ __forceinline__ void item_work(const PersistParams& P, uint32_t code, int chunk) {
  const int type = code & 15, stage = (code >> 4) & 15, idx = (int)(code >> 12);
  if (type == kItFlux) {
    const Dev& d = P.tab.b[idx];
    // the primitives alternate between two buffers
    const void* prim = stage == 2 ? d.blk.prim_next : d.blk.prim;
    Cell x;
    if (decode_cell(d, (int64_t)chunk * kFluxCells + threadIdx.x, x))
      flux_cell<float, true, false>(d.blk, prim, x, P.ph, kFlags);
  } else if (type == kItAsm) {
    const Dev& d = P.tab.b[idx];
    const StagePtrs sp{stage == 1 ? d.blk.q : P.qs[idx][stage - 2], P.qs[idx][stage - 1],
                       stage == 2 ? d.blk.prim_next : d.blk.prim,
                       stage == 2 ? const_cast<void*>(d.blk.prim) : d.blk.prim_next};
    asm_chunk<float, true, false>(d, sp, (int64_t)chunk * kAsmCellsP, kFlags, stage, stage < 3 ? 1 : 0, P.gm1, P.R,
                                  P.iR, P.ph);
  } else if (type == kItPrims) {
    const SplitBlock& B = P.tab.b[idx].blk;
    const int64_t c = (int64_t)chunk * kFluxCells + threadIdx.x;
    if (c < (int64_t)B.ni * B.nj * B.nk) prims_cell<float>(B, (int32_t)c, P.gm1, P.R, P.iR, P.ph.p_ref);
  } else if (type == kItGather) {
    const HaloDesc& d = P.links[idx];
    const double* src = P.tab.b[d.src_block].blk.q;
    const int64_t V = (int64_t)d.ext[0] * d.ext[1] * d.ext[2];
    const int64_t NS = (int64_t)d.sn[0] * d.sn[1] * d.sn[2];
    const int64_t t1 = min((int64_t)(chunk + 1) * kHaloChunk, 5 * V);
    for (int64_t t = (int64_t)chunk * kHaloChunk + threadIdx.x; t < t1; t += kWorkThreads) {
      const int v = (int)(t / V);
      int a, b, c;
      hd::slab_coords(d, t - v * V, a, b, c);
      P.halo[d.off + t] = src[v * NS + d.s0 + a * d.sstr[0] + b * d.sstr[1] + c * d.sstr[2]];
    }
  } else if (type == kItScatter) {
    const HaloDesc& d = P.links[idx];
    double* tgt = const_cast<double*>(P.tab.b[d.tgt_block].blk.q);
    const int64_t V = (int64_t)d.ext[0] * d.ext[1] * d.ext[2];
    const int64_t NT = (int64_t)d.tn[0] * d.tn[1] * d.tn[2];
    const int64_t r1 = min((int64_t)(chunk + 1) * kHaloChunk, V);
    for (int64_t r = (int64_t)chunk * kHaloChunk + threadIdx.x; r < r1; r += kWorkThreads) {
      int a, b, c;
      hd::slab_coords(d, r, a, b, c);
      const int ti = d.tlo[0] + a, tj = d.tlo[1] + b, tk = d.tlo[2] + c;
      bool later = false;
      for (int L2 = idx + 1; L2 < P.nlinks && !later; ++L2)
        later = P.links[L2].tgt_block == d.tgt_block && hd::slab_covers(P.links[L2], ti, tj, tk);
      if (later) continue;
      const int64_t tc = hd::cell_index(d.tn, ti, tj, tk);
#pragma unroll
      for (int v = 0; v < 5; ++v) tgt[v * NT + tc] = P.halo[d.off + v * V + r];
    }
  } else {  // kItBc
    const BcDesc& d = P.bcs[idx];
    double* q = const_cast<double*>(P.tab.b[d.block].blk.q);
    const int ax = d.face >> 1;
    const int oa = ax == 0 ? 1 : 0, ob = ax == 2 ? 1 : 2;
    const int64_t V = (int64_t)P.ghost * d.n[oa] * d.n[ob];
    const int64_t r1 = min((int64_t)(chunk + 1) * kHaloChunk, V);
    for (int64_t r = (int64_t)chunk * kHaloChunk + threadIdx.x; r < r1; r += kWorkThreads) {
      const int y = (int)(r % d.n[ob]);
      const int x = (int)((r / d.n[ob]) % d.n[oa]);
      const int o = (int)(r / ((int64_t)d.n[ob] * d.n[oa]));
      hd::bc_cell(d, q, ax, oa, ob, o, x, y, P.ghost, P.gamma, P.R);
    }
  }
}

// Named barriers of the hand-over between the scheduler warp and the workers:
// slot b (two slots) is "full" when the scheduler has put an item there and
// "empty" when the workers are done with it.
__device__ __forceinline__ void named_sync(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kCtaThreads) : "memory");
}
__device__ __forceinline__ void named_arrive(int id) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(kCtaThreads) : "memory");
}
constexpr int kBarFull = 1, kBarEmpty = 3;  // + slot

// The scheduler warp.  Lane 0 keeps two claims ahead of the item in hand
// (the next item's list entry already loaded, the one after it claimed), so
// the claim's atomic and the entry's load complete while the workers compute.
// Per item k (slot k & 1): make sure the workers are done with item k-2 (its
// slot is reused); look at the item's counters once and, if they are not all
// there, first publish every item handed out before (the one the workers are
// on may be among those waited for) and then wait; hand the item over; then
// publish item k-2.  So the claims, the waits and the publication overlap
// the workers' compute, and the scheduler never waits for an item that it
// holds back itself.
__device__ void schedule(const PersistParams& P, uint2* slot, int* end) {
  const unsigned all = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool l0 = lane == 0;
  int c1 = 0, c2 = 0, aborted = 0;  // lane 0: the next item's index and the one after it
  uint2 it1 = make_uint2(0u, 0u);   // lane 0: the next item's entry
  if (l0) {
    c1 = atomicAdd(P.ctl + kCtlNext, 1);
    c2 = atomicAdd(P.ctl + kCtlNext, 1);
    if (c1 < P.n_items) it1 = P.items[c1];
  }
  uint2 held0 = make_uint2(0u, 0u), held1 = make_uint2(0u, 0u);  // the items in the slots (lane 0)
  uint2 pend_it = make_uint2(0u, 0u);
  bool pend = false;  // the workers are done with pend_it, its completion is not published yet
  int done = -1;      // the workers are done with the items handed out up to this one
  for (int k = 0;; ++k) {
    const int b = k & 1;
    if (k >= 2 && done < k - 2) {
      named_sync(kBarEmpty + b);
      pend = true;
      pend_it = b ? held1 : held0;
      done = k - 2;
    }
    int cur = 0;
    uint2 it = make_uint2(0u, 0u);
    if (l0) {
      cur = c1;
      it = it1;
      // advance the claims: the entry after this one, and a new claim
      c1 = c2;
      if (cur < P.n_items) {
        if (c1 < P.n_items) it1 = P.items[c1];
        c2 = atomicAdd(P.ctl + kCtlNext, 1);
      }
    }
    cur = __shfl_sync(all, cur, 0);
    it = make_uint2(__shfl_sync(all, it.x, 0), __shfl_sync(all, it.y, 0));
    bool stop = cur >= P.n_items || aborted;
    if (!stop) {
      // a few looks while the workers are still on item k-1, before giving
      // up the overlap and publishing it
      const bool ready = P.wait_limit != 0 && deps_wait(P, it, true, 13);
      if (!ready) {
        if (pend) {
          if (l0) item_done(P, pend_it);
          pend = false;
        }
        if (k >= 1 && done < k - 1) {
          named_sync(kBarEmpty + (b ^ 1));
          if (l0) item_done(P, b ? held0 : held1);
          done = k - 1;
        }
        stop = !deps_wait(P, it, false, 0);
      }
      if (!stop && l0) fence_acq_rel();  // acquire: what the counters published is visible from here on
    }
    if (l0) {
      end[b] = stop ? 1 : 0;
      slot[b] = it;
      if (b) held1 = it;
      else held0 = it;
    }
    __syncwarp();
    named_arrive(kBarFull + b);
    if (pend) {
      if (l0) item_done(P, pend_it);
      pend = false;
    }
    if (stop) {
      // the workers finish item k-1 before they see the end mark
      if (k >= 1 && done < k - 1) {
        named_sync(kBarEmpty + (b ^ 1));
        if (l0) item_done(P, b ? held0 : held1);
      }
      return;
    }
    // an abort raised elsewhere ends this CTA at its next item (looked at
    // every 16 items, and by every wait)
    if ((k & 15) == 15) {
      if (l0) aborted = ld_relaxed(P.ctl + kCtlAbort);
      aborted = __shfl_sync(all, aborted, 0);
    }
  }
}

// One CTA = seven worker warps + one scheduler warp (warp 7).  Items are
// handed over through two shared-memory slots behind named barriers.  Every
// wait is bounded (the scheduler's counter polls) or ends when bounded work
// ends (the barriers), and a wait that gives up raises the abort flag, on
// which every scheduler hands its workers the end mark.
template <int OCC>
__global__ void __launch_bounds__(kCtaThreads, OCC) k_step_persist(const __grid_constant__ PersistParams P) {
  __shared__ uint2 s_slot[2];
  __shared__ int s_end[2];
  if (threadIdx.x >= kWorkThreads) {
    schedule(P, s_slot, s_end);
    return;
  }
  for (int k = 0;; ++k) {
    const int b = k & 1;
    named_sync(kBarFull + b);
    if (*(volatile int*)&s_end[b]) return;
    const uint2 it = s_slot[b];
    item_work(P, it.x, (int)it.y);
    named_arrive(kBarEmpty + b);
  }
}

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cudaGetLastError();
  }
  return n;
}

int resident_grid(int occ) {
  int per_sm = 0;
  const cudaError_t e = occ == 3
                            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_persist<3>, kSplitThreads, 0)
                            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_persist<4>, kSplitThreads, 0);
  if (e != cudaSuccess || per_sm <= 0) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sm_count();
}

// The stage part of the work-list: per stage, per block, the flux / assembly
// wavefront (see the file comment).
void stage_items(const fj_block* blocks, int nblocks, int lag, std::vector<uint2>& out) {
  for (int s = 1; s <= 3; ++s)
    for (int X = 0; X < nblocks; ++X) {
      const int64_t si = (int64_t)blocks[X].nj * blocks[X].nk, N = si * blocks[X].ni;
      const int ni = blocks[X].ni;
      const int nF = (int)chunks_of(N, kFluxCells), nA = (int)chunks_of(N, kAsmCellsP);
      // slot[a]: the flux chunk after which assembly chunk a is taken
      std::vector<std::vector<int>> after(nF);
      for (int a = 0; a < nA; ++a) {
        const int64_t c0 = (int64_t)a * kAsmCellsP, c1 = std::min<int64_t>(c0 + kAsmCellsP, N) - 1;
        const int pl0 = (int)(c0 / si), pl1 = (int)(c1 / si);
        // the last flux chunk of plane min(pl1 + 1, ni - 1); all of them for plane 0 (wrap)
        const int need_plane = std::min(pl1 + 1, ni - 1);
        int64_t f_need = (pl0 == 0 && ni > 1) ? nF - 1 : ((int64_t)(need_plane + 1) * si - 1) / kFluxCells;
        const int slot = (int)std::min<int64_t>(f_need + lag, nF - 1);
        after[slot].push_back(a);
      }
      for (int f = 0; f < nF; ++f) {
        out.push_back(make_uint2(item_code(kItFlux, s, 0, X), (unsigned)f));
        for (int a : after[f]) out.push_back(make_uint2(item_code(kItAsm, s, 0, X), (unsigned)a));
      }
    }
}

// The stage part of the work-list with the mixing across blocks: the sweeps
// (stage, block) in stage-major order, each sweep's flux chunks in order and,
// spread evenly among them, the previous sweep's assembly chunks, which come
// after all of that sweep's flux chunks (so an assembly chunk never waits on
// a flux chunk near it in the list).  A sweep whose next sweep is the same
// block's next stage (one block) keeps its assembly chunks to itself, after
// its flux chunks: that stage's flux chunks wait for all of them.
void stage_items_across(const fj_block* blocks, int nblocks, std::vector<uint2>& out) {
  int prev_X = -1, prev_s = 0, prev_nA = 0;
  auto flush_prev = [&]() {
    for (int a = 0; a < prev_nA; ++a) out.push_back(make_uint2(item_code(kItAsm, prev_s, 0, prev_X), (unsigned)a));
    prev_nA = 0;
  };
  for (int s = 1; s <= 3; ++s)
    for (int X = 0; X < nblocks; ++X) {
      const int64_t N = (int64_t)blocks[X].ni * blocks[X].nj * blocks[X].nk;
      const int nF = (int)chunks_of(N, kFluxCells), nA = (int)chunks_of(N, kAsmCellsP);
      if (prev_nA > 0 && prev_X == X) flush_prev();  // one block: its next stage waits for all of them
      // the previous sweep's assembly chunk a follows flux chunk floor(a nF / nA)
      int a = 0;
      for (int f = 0; f < nF; ++f) {
        out.push_back(make_uint2(item_code(kItFlux, s, 0, X), (unsigned)f));
        for (; a < prev_nA && (int64_t)a * nF / prev_nA <= f; ++a)
          out.push_back(make_uint2(item_code(kItAsm, prev_s, 0, prev_X), (unsigned)a));
      }
      for (; a < prev_nA; ++a) out.push_back(make_uint2(item_code(kItAsm, prev_s, 0, prev_X), (unsigned)a));
      prev_X = X;
      prev_s = s;
      prev_nA = nA;
    }
  flush_prev();
}

// Whether every item of the list waits only for items ahead of it: in a
// sequential run, item by item, the counters must already have reached every
// target an item waits for (the host restatement of dep_pair and item_done).
// A list that passes cannot deadlock the launch.
bool list_is_ordered(const PersistPlan& pp, const fj_block* blocks, int nblocks, const std::vector<uint2>& items) {
  std::vector<int64_t> scatter(nblocks, 0), bc(nblocks, 0), prims(nblocks, 0), asmc(3 * nblocks, 0),
      flux(3 * (size_t)pp.total_planes, 0);
  int64_t gather = 0;
  auto chunks_in_plane = [](int64_t si, int q) {
    return ((int64_t)(q + 1) * si - 1) / kFluxCells - ((int64_t)q * si) / kFluxCells + 1;
  };
  for (const uint2& it : items) {
    const uint32_t code = it.x;
    const int type = code & 15, stage = (code >> 4) & 15, face = (code >> 8) & 15, idx = (int)(code >> 12);
    const int64_t chunk = it.y;
    switch (type) {
      case kItGather:
        ++gather;
        break;
      case kItScatter:
        if (gather < pp.n_gather) return false;
        ++scatter[pp.link_tgt[idx]];
        break;
      case kItBc: {
        const int X = pp.bc_block[idx];
        if (scatter[X] < pp.scatter_total[X] || bc[X] < pp.bc_prefix[X * 7 + face]) return false;
        ++bc[X];
        break;
      }
      case kItPrims:
        if (scatter[idx] < pp.scatter_total[idx] || bc[idx] < pp.bc_prefix[idx * 7 + 6]) return false;
        ++prims[idx];
        break;
      case kItFlux: {
        const int64_t si = (int64_t)blocks[idx].nj * blocks[idx].nk, N = si * blocks[idx].ni;
        if (stage == 1 ? prims[idx] < chunks_of(N, kFluxCells)
                       : asmc[(stage - 2) * nblocks + idx] < chunks_of(N, kAsmCellsP))
          return false;
        const int64_t c0 = chunk * kFluxCells, c1 = std::min<int64_t>(c0 + kFluxCells, N) - 1;
        for (int64_t q = c0 / si; q <= c1 / si; ++q) ++flux[(stage - 1) * (size_t)pp.total_planes + pp.plane_base[idx] + q];
        break;
      }
      case kItAsm: {
        const int ni = blocks[idx].ni;
        const int64_t si = (int64_t)blocks[idx].nj * blocks[idx].nk, N = si * ni;
        const int64_t c0 = chunk * kAsmCellsP, c1 = std::min<int64_t>(c0 + kAsmCellsP, N) - 1;
        const int pl0 = (int)(c0 / si), pl1 = (int)(c1 / si);
        const int64_t* f = flux.data() + (stage - 1) * (size_t)pp.total_planes + pp.plane_base[idx];
        for (int q = std::max(pl0 - 1, 0); q <= std::min(pl1 + 1, ni - 1); ++q)
          if (f[q] < chunks_in_plane(si, q)) return false;
        if (pl0 == 0 && f[ni - 1] < chunks_in_plane(si, ni - 1)) return false;
        if (pl1 == ni - 1 && f[0] < chunks_in_plane(si, 0)) return false;
        ++asmc[(stage - 1) * nblocks + idx];
        break;
      }
      default:
        return false;
    }
  }
  return true;
}

}  // namespace

PersistPlan::~PersistPlan() {
  if (items) cudaFree(items);
  if (links) cudaFree(links);
  if (bcs) cudaFree(bcs);
  if (ctl) cudaFree(ctl);
}

size_t persist_tail_bytes(const fj_block* blocks, int nblocks, const fj_link* links, int nlinks, int ghost) {
  int64_t cells = 0;
  for (int b = 0; b < nblocks; ++b) cells += (int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk;
  const size_t split = (split_scratch_bytes(FJ_PREC_F32FLUX, cells) + 255) & ~(size_t)255;
  return split + halo_ws_bytes(blocks, links, nlinks, ghost);
}

namespace {

// The host part of the set-up: validation, the halo and BC descriptor tables,
// the halo / BC / primitive items and the counters' targets.  No device work.
bool persist_tables(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                    const fj_bc* bcs, int nbcs, const fj_params* p, PersistPlan& pp, std::vector<HaloDesc>& descs,
                    std::vector<BcDesc>& bds, std::string* why) {
  auto fail = [&](const std::string& w) {
    if (why) *why = w;
    return false;
  };
  if (p->precision != FJ_PREC_F32FLUX) return fail("the persistent step is the FP32-flux path's");
  if (nblocks < 1 || nblocks > kPersistMaxBlocks) return fail("the persistent step takes 1..64 blocks");
  for (int b = 0; b < nblocks; ++b) {
    if ((int64_t)16 * blocks[b].ni * blocks[b].nj * blocks[b].nk > INT32_MAX)
      return fail("block too large for 32-bit record offsets");
    if (blocks[b].ni < 1 || blocks[b].nj < 1 || blocks[b].nk < 1) return fail("empty block");
  }
  descs.clear();
  bds.clear();
  size_t nd = 0;
  if (hd::build_links(ctx, blocks, nblocks, links, nlinks, p->ghost, descs, nd) != FJ_OK)
    return fail("halo links: " + (ctx ? ctx->last_error : std::string()));
  if (descs.size() >= (1u << 20)) return fail("too many links");
  pp.scatter_total.assign(kPersistMaxBlocks, 0);
  pp.bc_prefix.assign(kPersistMaxBlocks * 7, 0);
  pp.plane_base.assign(kPersistMaxBlocks, 0);
  std::vector<uint2> head;
  // 1. gathers, 2. scatters (link order)
  pp.n_gather = 0;
  for (size_t L = 0; L < descs.size(); ++L) {
    descs[L].tgt = nullptr;
    descs[L].src = nullptr;
    const int64_t V = (int64_t)descs[L].ext[0] * descs[L].ext[1] * descs[L].ext[2];
    const int64_t g = chunks_of(5 * V, kHaloChunk);
    for (int64_t c = 0; c < g; ++c) head.push_back(make_uint2(item_code(kItGather, 0, 0, (int)L), (unsigned)c));
    pp.n_gather += (int)g;
  }
  for (size_t L = 0; L < descs.size(); ++L) {
    const int64_t V = (int64_t)descs[L].ext[0] * descs[L].ext[1] * descs[L].ext[2];
    const int64_t n = chunks_of(V, kHaloChunk);
    for (int64_t c = 0; c < n; ++c) head.push_back(make_uint2(item_code(kItScatter, 0, 0, (int)L), (unsigned)c));
    pp.scatter_total[descs[L].tgt_block] += (int)n;
    pp.link_tgt.push_back(descs[L].tgt_block);
  }
  // 3. boundary conditions, Face order, list order within a face
  std::vector<int64_t> bc_chunks(nbcs, 0);
  for (int e = 0; e < nbcs; ++e) {
    const fj_bc& bc = bcs[e];
    if (bc.block < 0 || bc.block >= nblocks || bc.face < 0 || bc.face > 5) return fail("bc entry out of range");
    if (bc.type != FJ_BC_WALL && bc.type != FJ_BC_SYMMETRY && bc.type != FJ_BC_FARFIELD)
      return fail("unsupported bc type");
    const fj_block& blk = blocks[bc.block];
    BcDesc d;
    std::memset(&d, 0, sizeof(d));
    d.q = nullptr;
    d.n[0] = blk.ni;
    d.n[1] = blk.nj;
    d.n[2] = blk.nk;
    d.face = bc.face;
    d.type = bc.type;
    d.iso = bc.isothermal;
    d.T_wall = bc.T_wall;
    for (int v = 0; v < 5; ++v) d.qinf[v] = bc.q_inf[v];
    d.block = bc.block;
    bds.push_back(d);
    pp.bc_block.push_back(bc.block);
    const int ax = bc.face >> 1;
    const int64_t area = (int64_t)blk.ni * blk.nj * blk.nk / d.n[ax];
    bc_chunks[e] = chunks_of(area * p->ghost, kHaloChunk);
  }
  for (int face = 0; face < 6; ++face)
    for (int e = 0; e < nbcs; ++e) {
      if (bcs[e].face != face) continue;
      for (int64_t c = 0; c < bc_chunks[e]; ++c) head.push_back(make_uint2(item_code(kItBc, 0, face, e), (unsigned)c));
      // later faces of this block wait for these items
      for (int f = face + 1; f <= 6; ++f) pp.bc_prefix[bcs[e].block * 7 + f] += (int)bc_chunks[e];
    }
  // 4. primitives, block order
  int planes = 0;
  for (int X = 0; X < nblocks; ++X) {
    const int64_t N = (int64_t)blocks[X].ni * blocks[X].nj * blocks[X].nk;
    for (int64_t c = 0; c < chunks_of(N, kFluxCells); ++c)
      head.push_back(make_uint2(item_code(kItPrims, 0, 0, X), (unsigned)c));
    pp.plane_base[X] = planes;
    planes += blocks[X].ni;
  }
  pp.total_planes = planes;
  pp.reset_from = kCtlReset;
  pp.ctl_ints = kCtlFlux + 3 * planes;
  pp.nlinks = (int)descs.size();
  pp.nbcs = (int)bds.size();
  pp.split_bytes = persist_tail_bytes(blocks, nblocks, nullptr, 0, p->ghost);
  pp.head.swap(head);
  return true;
}

// The whole work-list for a grid of `grid` resident CTAs: the head and the
// stage items in the shape's order.
void build_list(const PersistPlan& pp, const fj_block* blocks, int nblocks, int grid, double lag_scale,
                std::vector<uint2>& items, int* lag_out) {
  items = pp.head;
  const int lag = std::max(0, (int)(lag_scale * grid / 2));
  if (lag_scale < 0)
    stage_items_across(blocks, nblocks, items);
  else
    stage_items(blocks, nblocks, lag, items);
  if (lag_out) *lag_out = lag;
}

}  // namespace

bool persist_setup(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                   const fj_bc* bcs, int nbcs, const fj_params* p, PersistPlan& pp, std::string* why) {
  auto fail = [&](const std::string& w) {
    if (why) *why = w;
    return false;
  };
  std::vector<HaloDesc> descs;
  std::vector<BcDesc> bds;
  if (!persist_tables(ctx, blocks, nblocks, links, nlinks, bcs, nbcs, p, pp, descs, bds, why)) return false;
  // device tables
  auto upload = [](void** dst, const void* src, size_t bytes) {
    if (bytes == 0) return true;
    if (cudaMalloc(dst, bytes) != cudaSuccess) {
      *dst = nullptr;
      cudaGetLastError();
      return false;
    }
    return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  if (!upload(&pp.links, descs.data(), descs.size() * sizeof(HaloDesc)) ||
      !upload(&pp.bcs, bds.data(), bds.size() * sizeof(BcDesc)))
    return fail("persistent step tables: device allocation failed");
  if (cudaMalloc((void**)&pp.ctl, (size_t)pp.ctl_ints * sizeof(int)) != cudaSuccess ||
      cudaMemset(pp.ctl, 0, (size_t)pp.ctl_ints * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return fail("persistent step control block: device allocation failed");
  }
  if (!persist_reshape(pp, blocks, nblocks, kPersistShapes[0].occ, kPersistShapes[0].lag_scale))
    return fail("persistent step work-list: set-up failed");
  return true;
}

bool persist_reshape(PersistPlan& pp, const fj_block* blocks, int nblocks, int occ, double lag_scale) {
  if (occ != 3 && occ != 4) return false;
  const int grid = resident_grid(occ);
  if (grid <= 0) return false;
  std::vector<uint2> items;
  int lag = 0;
  build_list(pp, blocks, nblocks, grid, lag_scale, items, &lag);
  if (items.size() >= (size_t)INT32_MAX) return false;
  if (!list_is_ordered(pp, blocks, nblocks, items)) return false;
  if (pp.items && (int)items.size() != pp.n_items) {
    cudaFree(pp.items);
    pp.items = nullptr;
  }
  if (!pp.items && cudaMalloc(&pp.items, items.size() * sizeof(uint2)) != cudaSuccess) {
    pp.items = nullptr;
    cudaGetLastError();
    return false;
  }
  if (cudaMemcpy(pp.items, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  pp.n_items = (int)items.size();
  pp.grid = std::min<int64_t>(grid, pp.n_items);
  pp.occ = occ;
  pp.lag = lag;
  return true;
}

int persist_step(fj_ctx* ctx, const PersistPlan& pp, const fj_block* blocks, int nblocks, double* const* q1s,
                 double* const* q2s, double* const* q_out, const fj_params* p, double p_ref, const double* mu0_b,
                 const double* dt_b, double dt, void* const* kmet, void* tail, int wait_limit, cudaStream_t st,
                 bool fill_only) {
  if (nblocks < 1 || nblocks > kPersistMaxBlocks || !kmet || !pp.items || !pp.ctl)
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "persistent step: plan not set up");
  std::unique_ptr<PersistParams> hold(new (std::nothrow) PersistParams());  // 14 KB: off the stack
  if (!hold) return set_err(ctx, FJ_ERR_NO_MEMORY, "persistent step parameters");
  PersistParams& P = *hold;
  std::vector<SplitBlock> sb(nblocks);
  for (int b = 0; b < nblocks; ++b) {
    SplitBlock& e = sb[b];
    e = SplitBlock{};
    e.q = blocks[b].q;
    e.q0 = blocks[b].q;
    e.out = nullptr;
    e.kxyz = blocks[b].kxyz;
    e.kaos = kmet[b];
    e.vol = blocks[b].vol;
    e.mu0 = mu0_b ? mu0_b[b] : p->mu0;
    e.dt = dt_b ? dt_b[b] : dt;
    e.ni = blocks[b].ni;
    e.nj = blocks[b].nj;
    e.nk = blocks[b].nk;
    if (!e.kaos) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "persistent step: metric records missing");
  }
  split_assign_scratch(FJ_PREC_F32FLUX, sb.data(), nblocks, tail);
  P.tab.n = nblocks;
  for (int b = 0; b < nblocks; ++b) {
    P.tab.b[b].blk = sb[b];
    P.tab.b[b].dk.init((uint32_t)sb[b].nk);
    P.tab.b[b].dj.init((uint32_t)sb[b].nj);
    P.qs[b][0] = q1s[b];
    P.qs[b][1] = q2s[b];
    P.qs[b][2] = q_out[b];
    P.scatter_total[b] = pp.scatter_total[b];
    for (int f = 0; f < 7; ++f) P.bc_prefix[b][f] = pp.bc_prefix[b * 7 + f];
    P.plane_base[b] = pp.plane_base[b];
  }
  P.ph = make_phys(p);
  P.ph.p_ref = p_ref;
  P.gamma = p->gamma;
  P.gm1 = p->gamma - 1.0;
  P.R = p->R;
  P.iR = 1.0 / p->R;
  P.items = (const uint2*)pp.items;
  P.links = (const HaloDesc*)pp.links;
  P.bcs = (const BcDesc*)pp.bcs;
  P.halo = (double*)((char*)tail + pp.split_bytes);
  P.ctl = pp.ctl;
  // the list's head (halo, BCs, primitives) is a prefix that depends on nothing after it
  P.n_items = fill_only ? (int)pp.head.size() : pp.n_items;
  P.nlinks = pp.nlinks;
  P.ghost = p->ghost;
  P.wait_limit = wait_limit;
  P.n_gather = pp.n_gather;
  P.total_planes = pp.total_planes;
  int s = cuda_status(ctx,
                      cudaMemsetAsync(pp.ctl + pp.reset_from, 0, (size_t)(pp.ctl_ints - pp.reset_from) * sizeof(int), st),
                      "persistent step counters");
  if (s != FJ_OK) return s;
  const int grid = std::max(1, std::min(pp.grid, P.n_items));
  if (pp.occ == 3)
    k_step_persist<3><<<grid, kSplitThreads, 0, st>>>(P);
  else
    k_step_persist<4><<<grid, kSplitThreads, 0, st>>>(P);
  ctx->launches += 1;
  return launch_status(ctx, "persistent step launch");
}

int persist_read_error(const PersistPlan& pp, int* out, cudaStream_t st) {
  *out = 0;
  if (!pp.ctl) return FJ_OK;
  cudaError_t e = cudaMemcpyAsync(out, pp.ctl + kCtlErr, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

int persist_clear_error(const PersistPlan& pp, cudaStream_t st) {
  if (!pp.ctl) return FJ_OK;
  return cudaMemsetAsync(pp.ctl + kCtlErr, 0, sizeof(int), st) == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}

}  // namespace fj

extern "C" int fj_persist_list_check(const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                                     const fj_bc* bcs, int nbcs, const fj_params* p, int grid, int shape,
                                     int64_t* n_items) {
  using namespace fj;
  if (!blocks || !p || grid < 1 || shape < 0 || shape >= FJ_NUM_PERSIST_SHAPES || (nlinks > 0 && !links) ||
      (nbcs > 0 && !bcs) || nlinks < 0 || nbcs < 0)
    return FJ_ERR_INVALID_ARGUMENT;
  PersistPlan pp;
  std::vector<hd::HaloDesc> descs;
  std::vector<hd::BcDesc> bds;
  if (!persist_tables(nullptr, blocks, nblocks, links, nlinks, bcs, nbcs, p, pp, descs, bds, nullptr))
    return FJ_ERR_NOT_IMPLEMENTED;
  std::vector<uint2> items;
  build_list(pp, blocks, nblocks, grid, kPersistShapes[shape].lag_scale, items, nullptr);
  if (n_items) *n_items = (int64_t)items.size();
  return list_is_ordered(pp, blocks, nblocks, items) ? FJ_OK : FJ_ERR_INVALID_ARGUMENT;
}
