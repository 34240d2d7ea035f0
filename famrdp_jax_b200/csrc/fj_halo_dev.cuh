// fj_halo_dev.cuh -- halo-link and boundary-condition descriptors and their
// per-cell device code, shared by the halo / BC kernels (fj_halo.cu) and the
// persistent step kernel (fj_step_persist.cu).
#pragma once

#include <vector>

#include "fj_common.cuh"

namespace fj {
namespace hd {

// One CUT1TO1 link reduced to an affine map from the target slab's
// coordinates to a source cell index (mesh/halo.py:36-53).  The launch-table
// kernels address the blocks through tgt / src; the persistent kernel's
// copies carry nullptr there and address them by tgt_block / src_block.
struct HaloDesc {
  double* tgt;
  const double* src;
  long long off;      // slab offset in scratch (doubles)
  long long s0;       // source cell index of the slab's first element
  long long sstr[3];  // source index step per step along target slab axis 0, 1, 2
  int tn[3], sn[3];
  int tlo[3], ext[3];
  int tgt_block;
  int src_block;
};

// One face's boundary condition; the persistent kernel's copies carry
// q = nullptr and address the block by `block`.
struct BcDesc {
  double* q;
  double qinf[5];
  double T_wall;
  int n[3];
  int face, type, iso;
  int block;
};

__device__ __forceinline__ int64_t cell_index(const int n[3], int i, int j, int k) {
  return ((int64_t)i * n[1] + j) * n[2] + k;
}

// Slab element r (of ext[0] x ext[1] x ext[2], last axis fastest) of link d:
// its offsets a, b, c along the target slab's axes.
__device__ __forceinline__ void slab_coords(const HaloDesc& d, int64_t r, int& a, int& b, int& c) {
  c = (int)(r % d.ext[2]);
  b = (int)((r / d.ext[2]) % d.ext[1]);
  a = (int)(r / ((int64_t)d.ext[2] * d.ext[1]));
}

// Whether target cell (ti, tj, tk) lies in link e's target slab.
__device__ __forceinline__ bool slab_covers(const HaloDesc& e, int ti, int tj, int tk) {
  return ti >= e.tlo[0] && ti < e.tlo[0] + e.ext[0] && tj >= e.tlo[1] && tj < e.tlo[1] + e.ext[1] &&
         tk >= e.tlo[2] && tk < e.tlo[2] + e.ext[2];
}

// physics/bc/base.py:15-27 ghost_indices: outer layer o (0..g-1 counted from
// the face) pairs with the mirrored inner layer.
__device__ __forceinline__ void bc_layers(int face, int n, int g, int o, int& outer, int& inner) {
  if ((face & 1) == 0) {
    outer = o;
    inner = 2 * g - 1 - o;
  } else {
    outer = n - 1 - o;
    inner = n - 2 * g + o;
  }
}

// The boundary condition d on ghost layer o, cell (x, y) of the face's two
// other axes oa, ob (ax: the face's axis), in place on q (5, n0, n1, n2).
__device__ __forceinline__ void bc_cell(const BcDesc& d, double* q, int ax, int oa, int ob, int o, int x, int y,
                                        int g, double gamma, double R) {
  const int64_t NT = (int64_t)d.n[0] * d.n[1] * d.n[2];
  int outer, inner;
  bc_layers(d.face, d.n[ax], g, o, outer, inner);
  int io[3], ii[3];
  io[ax] = outer; ii[ax] = inner;
  io[oa] = x; ii[oa] = x;
  io[ob] = y; ii[ob] = y;
  const int64_t co = cell_index(d.n, io[0], io[1], io[2]);
  const int64_t ci = cell_index(d.n, ii[0], ii[1], ii[2]);
  if (d.type == FJ_BC_FARFIELD) {  // physics/bc/farfield.py:7-21
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v * NT + co] = d.qinf[v];
  } else if (d.type == FJ_BC_WALL && d.iso) {  // physics/bc/wall.py:32-55
    const double r0 = q[ci], r1 = q[NT + ci], r2 = q[2 * NT + ci], r3 = q[3 * NT + ci], r4 = q[4 * NT + ci];
    const double gm1 = gamma - 1.0;
    const double ke_i = 0.5 * (r1 * r1 + r2 * r2 + r3 * r3) / r0;
    const double p_g = gm1 * (r4 - ke_i);
    const double rho_g = p_g / (R * d.T_wall);
    const double scale = rho_g / r0;
    const double u_g = -r1 * scale, v_g = -r2 * scale, w_g = -r3 * scale;
    const double ke_g = 0.5 * (u_g * u_g + v_g * v_g + w_g * w_g) / rho_g;
    q[co] = rho_g;
    q[NT + co] = u_g;
    q[2 * NT + co] = v_g;
    q[3 * NT + co] = w_g;
    q[4 * NT + co] = p_g / gm1 + ke_g;
  } else {  // mirror: adiabatic wall (wall.py:27-29) or symmetry (symmetry.py:8-11)
    double s[5] = {1.0, 1.0, 1.0, 1.0, 1.0};
    if (d.type == FJ_BC_WALL) {
      s[1] = s[2] = s[3] = -1.0;
    } else {
      s[1 + ax] = -1.0;
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v * NT + co] = q[v * NT + ci] * s[v];
  }
}

// The halo links of a step (fj_halo.cu): validated, with slab offsets into a
// scratch of scratch_doubles doubles, in list order.
int build_links(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks, int ghost,
                std::vector<HaloDesc>& out, size_t& scratch_doubles);

}  // namespace hd
}  // namespace fj
