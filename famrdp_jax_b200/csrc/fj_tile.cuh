// fj_tile.cuh -- the fused TMA-tile stage kernel (fj_stage_tile.cu): one
// TVD-RK3 stage of all blocks (FP32 fluxes, FP64 state) in one persistent
// launch over a work-list of (tile, i-plane segment) items.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <array>
#include <vector>

#include "fj_common.cuh"

namespace fj {

constexpr int kTileMaxBlocks = 64;  // blocks per launch (more are chunked)

// The padded primitive arrays the tile kernel streams with TMA: per block
// (5, ni, njp, nkp) FP32 (rho, u, v, w, p - p_ref), where padded row
// jj = j + 2 and column kk = k + 2, the two rows / columns on either side
// holding the periodic images (row -1 = row nj - 1, row nj = row 0, ...), so
// that a tile's 2-cell halo is one box even where it wraps around the block
// (the reference's jnp.roll in the viscous terms).  nkp = nk + 4 rounded up to
// a multiple of 4 (16-byte TMA row pitch) and njp = nj + 4, both at least the
// TMA box (36 columns, 12 rows) so that tiny blocks need no special case.
inline int tile_nkp(int nk) { return std::max((nk + 4 + 3) & ~3, 36); }
inline int tile_njp(int nj) { return std::max(nj + 4, 12); }
inline size_t tile_prims_bytes(int ni, int nj, int nk) {
  return ((size_t)5 * ni * tile_njp(nj) * tile_nkp(nk) * sizeof(float) + 255) & ~(size_t)255;
}

// One block of a tile-stage launch.
struct TileBlock {
  const double* q;     // stage input (5, ni, nj, nk)
  const double* q0;    // step start state (stages 2, 3)
  double* out;         // stage result; may alias q0, never q
  const float* kaos;   // FP32 metric records, 12 per cell (kxyz[l][m] l-major, 3 pressure-offset sums)
  const double* vol;   // (ni, nj, nk)
  float* prim_next;    // padded primitives of the stage result (nullptr: not written)
  double mu0, dt;
  int ni, nj, nk, njp, nkp;
  int ntj, ntk;         // tiles along j and k
};

// Host-side plan data of the tile path: one TMA descriptor per block and
// padded primitive buffer (two buffers alternate between stages).
struct TileMaps {
  std::vector<std::array<unsigned long long, 16>> map[2];  // CUtensorMap images (128 B)
  std::vector<float*> prim[2];                             // per block, padded primitives
  int* err = nullptr;                                      // device error word (bounded waits), owned
  bool ok = false;
  TileMaps() = default;
  TileMaps(const TileMaps&) = delete;
  TileMaps& operator=(const TileMaps&) = delete;
  ~TileMaps();
};

// Bytes of plan scratch the tile path needs for these blocks (both padded
// primitive buffers).
size_t tile_scratch_bytes(const fj_block* blocks, int nblocks);
// Lays the padded buffers out in `scratch`, encodes the TMA descriptors and
// allocates the error word; returns false when the driver's encoder is
// unavailable or refuses a block.
bool tile_setup(const fj_block* blocks, int nblocks, void* scratch, TileMaps& tm);
// Primitives of q (the stage-1 input) into padded buffer `which` of every block.
int tile_prims(fj_ctx* ctx, const TileMaps& tm, int which, const double* const* q, const fj_block* blocks,
               int nblocks, double gm1, double R, double p_ref, cudaStream_t st);
// One stage (1..3) of all blocks: reads padded buffer `which`, writes the
// stage result and (stages 1, 2) the next stage's primitives into buffer
// 1 - which.  blocks[b].prim_next is set by the launcher.
int tile_stage(fj_ctx* ctx, const TileMaps& tm, int which, TileBlock* blocks, int nblocks, const Phys& ph,
               int stage, cudaStream_t st, int wait_limit = -1);
// The error word (nonzero: a bounded wait of the tile kernel gave up).
int tile_read_error(const TileMaps& tm, int* out, cudaStream_t st);
int tile_clear_error(const TileMaps& tm, cudaStream_t st);

}  // namespace fj
