// fj_halo.cu -- inter-block halo fill (mesh/halo.py:36-92) and physical
// boundary conditions (physics/bc/*.py), in place on the blocks' q arrays.
//
// Halo semantics kept from the reference:
//   * every CUT1TO1 link copies the source block's 2-layer slab next to the
//     source face ([g, 2g) or [n-2g, n-g) along its axis, FULL extent along the
//     other two axes) into the target's ghost slab ([0, g) or [n-g, n) along
//     the target face's axis, full extent along the others), element by
//     element in array order (mesh/halo.py:36-53);
//   * all sources are read from the PRE-exchange arrays (mesh/halo.py:89-90):
//     one kernel gathers every source slab into scratch before any target is
//     written;
//   * links apply in list order, so where two target slabs overlap (edges and
//     corners) the later link wins: the scatter kernel skips a cell that a
//     later link of the same target block also writes.
// Orientation: 0 is the reference's element-by-element slab copy; 1 (the
// marker the reference's topology reader stores) is rejected as there.  Codes
// 8..15 are this library's face-to-face mapping (the reference has none): the
// ghost layer at distance d from the interface takes the source's interior
// layer at distance d, and the target's two tangential axes (in i, j, k
// order) map onto the source's with bit 0 = swapped, bit 1 / bit 2 = the
// first / second target tangential axis runs backwards on the source.  Each
// link is reduced on the host to an affine map from the target slab's
// coordinates to a source cell index (base + signed stride per axis).
// Boundary conditions run after the halo, one launch per face in Face enum
// order (physics/bc/dispatch.py:15), each launch covering that face of every
// block (blocks are independent).
#include <vector>

#include "fj_common.cuh"
#include "fj_halo_dev.cuh"
#include "fj_rhs.cuh"

namespace fj {

namespace {

constexpr int kMaxLinksPerLaunch = 192;
constexpr int kMaxBcPerLaunch = 128;

using namespace hd;

struct HaloTable {
  int n;
  HaloDesc d[kMaxLinksPerLaunch];
};

struct BcTable {
  int n;
  double gamma, R;
  BcDesc d[kMaxBcPerLaunch];
};

__global__ void k_halo_gather(const HaloTable tab, double* __restrict__ scratch) {
  grid_dep_wait();
  const HaloDesc& d = tab.d[blockIdx.y];
  const int64_t V = (int64_t)d.ext[0] * d.ext[1] * d.ext[2];
  const int64_t NS = (int64_t)d.sn[0] * d.sn[1] * d.sn[2];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 5 * V;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(t / V);
    int a, b, c;
    slab_coords(d, t - v * V, a, b, c);
    scratch[d.off + t] = d.src[v * NS + d.s0 + a * d.sstr[0] + b * d.sstr[1] + c * d.sstr[2]];
  }
}

__global__ void k_halo_scatter(const HaloTable tab, const double* __restrict__ scratch) {
  grid_dep_wait();
  const int L = blockIdx.y;
  const HaloDesc& d = tab.d[L];
  const int64_t V = (int64_t)d.ext[0] * d.ext[1] * d.ext[2];
  const int64_t NT = (int64_t)d.tn[0] * d.tn[1] * d.tn[2];
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < V;
       r += (int64_t)gridDim.x * blockDim.x) {
    int a, b, c;
    slab_coords(d, r, a, b, c);
    const int ti = d.tlo[0] + a, tj = d.tlo[1] + b, tk = d.tlo[2] + c;
    bool later = false;
    for (int L2 = L + 1; L2 < tab.n && !later; ++L2)
      later = tab.d[L2].tgt_block == d.tgt_block && slab_covers(tab.d[L2], ti, tj, tk);
    if (later) continue;
    const int64_t tc = cell_index(d.tn, ti, tj, tk);
#pragma unroll
    for (int v = 0; v < 5; ++v) d.tgt[v * NT + tc] = scratch[d.off + v * V + r];
  }
}

__global__ void k_bc(const BcTable tab, int g) {
  grid_dep_wait();
  const BcDesc& d = tab.d[blockIdx.y];
  const int ax = d.face >> 1;
  const int oa = ax == 0 ? 1 : 0, ob = ax == 2 ? 1 : 2;  // the two other axes
  const int64_t V = (int64_t)g * d.n[oa] * d.n[ob];
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < V;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(r % d.n[ob]);
    const int x = (int)((r / d.n[ob]) % d.n[oa]);
    const int o = (int)(r / ((int64_t)d.n[ob] * d.n[oa]));
    bc_cell(d, d.q, ax, oa, ob, o, x, y, g, tab.gamma, tab.R);
  }
}

bool face_box(int face, const int n[3], int g, bool source, int lo[3], int ext[3]) {
  if (face < 0 || face > 5) return false;
  const int ax = face >> 1;
  for (int a = 0; a < 3; ++a) {
    lo[a] = 0;
    ext[a] = n[a];
  }
  ext[ax] = g;
  if (source)
    lo[ax] = (face & 1) == 0 ? g : n[ax] - 2 * g;
  else
    lo[ax] = (face & 1) == 0 ? 0 : n[ax] - g;
  return true;
}

}  // namespace

namespace hd {

int build_links(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links,
                int nlinks, int ghost, std::vector<HaloDesc>& out, size_t& scratch_doubles) {
  out.clear();
  scratch_doubles = 0;
  for (int L = 0; L < nlinks; ++L) {
    const fj_link& l = links[L];
    if (l.tgt_block < 0 || l.tgt_block >= nblocks || l.src_block < 0 || l.src_block >= nblocks)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "link block index out of range");
    if (l.tgt_face < 0 || l.tgt_face > 5 || l.src_face < 0 || l.src_face > 5)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "link face out of range");
    const bool mapped = (l.orient & ~7) == 8;
    if (l.orient != 0 && !mapped)
      return set_err(ctx, FJ_ERR_NOT_IMPLEMENTED,
                     "orient=" + std::to_string(l.orient) + " not supported in stage 1");
    const fj_block& tb = blocks[l.tgt_block];
    const fj_block& sb = blocks[l.src_block];
    HaloDesc d;
    d.tgt = tb.q;
    d.src = sb.q;
    d.tn[0] = tb.ni; d.tn[1] = tb.nj; d.tn[2] = tb.nk;
    d.sn[0] = sb.ni; d.sn[1] = sb.nj; d.sn[2] = sb.nk;
    const long long sst[3] = {(long long)d.sn[1] * d.sn[2], d.sn[2], 1};  // source array strides
    face_box(l.tgt_face, d.tn, ghost, false, d.tlo, d.ext);
    if (!mapped) {  // the reference's element-by-element copy of equal-shaped slabs
      int slo[3], sext[3];
      face_box(l.src_face, d.sn, ghost, true, slo, sext);
      if (sext[0] != d.ext[0] || sext[1] != d.ext[1] || sext[2] != d.ext[2])
        return set_err(ctx, FJ_ERR_SHAPE,
                       "halo slab shape mismatch: target (5," + std::to_string(d.ext[0]) + "," +
                           std::to_string(d.ext[1]) + "," + std::to_string(d.ext[2]) +
                           ") vs source (5," + std::to_string(sext[0]) + "," +
                           std::to_string(sext[1]) + "," + std::to_string(sext[2]) + ")");
      d.s0 = slo[0] * sst[0] + slo[1] * sst[1] + slo[2];
      for (int a = 0; a < 3; ++a) d.sstr[a] = sst[a];
    } else {
      const int aT = l.tgt_face >> 1, aS = l.src_face >> 1;
      const bool tmin = (l.tgt_face & 1) == 0, smin = (l.src_face & 1) == 0;
      if (d.sn[aS] < 2 * ghost)
        return set_err(ctx, FJ_ERR_SHAPE, "halo source block thinner than two ghost widths");
      // normal axis: target layer r (0..g-1 from the slab's low end) is at
      // distance d = g - r (MIN face) or r + 1 (MAX face) from the interface;
      // the source layer at distance d is g + d - 1 (MIN) or n - g - d (MAX)
      long long base, dir;
      if (tmin && smin) base = 2 * ghost - 1, dir = -1;
      else if (tmin) base = d.sn[aS] - 2 * ghost, dir = 1;
      else if (smin) base = ghost, dir = 1;
      else base = d.sn[aS] - ghost - 1, dir = -1;
      d.s0 = base * sst[aS];
      d.sstr[aT] = dir * sst[aS];
      int tt[2], ss[2], nt = 0, ns = 0;  // tangential axes in i, j, k order
      for (int a = 0; a < 3; ++a) {
        if (a != aT) tt[nt++] = a;
        if (a != aS) ss[ns++] = a;
      }
      const bool swap = (l.orient & 1) != 0;
      for (int m = 0; m < 2; ++m) {
        const int t = tt[m], sa = ss[swap ? 1 - m : m];
        const bool rev = (l.orient & (2 << m)) != 0;
        if (d.ext[t] != d.sn[sa])
          return set_err(ctx, FJ_ERR_SHAPE,
                         "halo slab shape mismatch: target tangential extent " + std::to_string(d.ext[t]) +
                             " vs source " + std::to_string(d.sn[sa]));
        d.s0 += (rev ? (long long)(d.sn[sa] - 1) : 0) * sst[sa];
        d.sstr[t] = (rev ? -1 : 1) * sst[sa];
      }
    }
    d.tgt_block = l.tgt_block;
    d.src_block = l.src_block;
    d.off = (long long)scratch_doubles;
    scratch_doubles += 5ull * d.ext[0] * d.ext[1] * d.ext[2];
    scratch_doubles = (scratch_doubles + 31) & ~31ull;  // 256-byte aligned slabs
    out.push_back(d);
  }
  return FJ_OK;
}

}  // namespace hd

size_t halo_ws_bytes(const fj_block* blocks, const fj_link* links, int nlinks, int ghost) {
  size_t total = 0;
  for (int L = 0; L < nlinks; ++L) {
    const fj_block& tb = blocks[links[L].tgt_block];
    int n[3] = {tb.ni, tb.nj, tb.nk}, lo[3], ext[3];
    if (!face_box(links[L].tgt_face, n, ghost, false, lo, ext)) return 0;
    total += 5ull * ext[0] * ext[1] * ext[2];
    total = (total + 31) & ~31ull;
  }
  return total * sizeof(double);
}

int halo_exchange(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links,
                  int nlinks, int ghost, double* scratch, size_t scratch_bytes,
                  cudaStream_t st) {
  if (nlinks == 0) return FJ_OK;
  std::vector<HaloDesc> descs;
  size_t nd = 0;
  int s = build_links(ctx, blocks, nblocks, links, nlinks, ghost, descs, nd);
  if (s != FJ_OK) return s;
  if (scratch_bytes < nd * sizeof(double))
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "halo scratch too small");
  const int nl = (int)descs.size();
  // gather all sources first (pre-exchange values), then scatter in order
  for (int pass = 0; pass < 2; ++pass) {
    for (int base = 0; base < nl; base += kMaxLinksPerLaunch) {
      HaloTable tab;
      tab.n = std::min(kMaxLinksPerLaunch, nl - base);
      int64_t vmax = 0;
      for (int t = 0; t < tab.n; ++t) {
        tab.d[t] = descs[base + t];
        vmax = std::max<int64_t>(vmax, (int64_t)tab.d[t].ext[0] * tab.d[t].ext[1] * tab.d[t].ext[2]);
      }
      dim3 grid((unsigned)std::min<int64_t>(grid_for(pass == 0 ? 5 * vmax : vmax), 4096), tab.n);
      if (pass == 0)
        pdl_launch(k_halo_gather, grid, kThreads, 0, st, tab, scratch);
      else
        pdl_launch(k_halo_scatter, grid, kThreads, 0, st, tab, (const double*)scratch);
      ctx->launches += 1;
      s = launch_status(ctx, "halo launch");
      if (s != FJ_OK) return s;
    }
  }
  return FJ_OK;
}

int halo_pack_unpack(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks, int ghost,
                     const int* sel, const int64_t* off, int nsel, double* buf, int64_t buf_doubles, bool unpack,
                     cudaStream_t st) {
  if (nsel == 0) return FJ_OK;
  std::vector<fj_link> chosen((size_t)nsel);
  for (int i = 0; i < nsel; ++i) {
    if (sel[i] < 0 || sel[i] >= nlinks) return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "selected link out of range");
    chosen[(size_t)i] = links[sel[i]];
  }
  std::vector<HaloDesc> descs;
  size_t nd = 0;
  int s = build_links(ctx, blocks, nblocks, chosen.data(), nsel, ghost, descs, nd);
  if (s != FJ_OK) return s;
  for (int i = 0; i < nsel; ++i) {
    HaloDesc& d = descs[(size_t)i];
    const int64_t len = 5ll * d.ext[0] * d.ext[1] * d.ext[2];
    if (off[i] < 0 || off[i] > buf_doubles - len)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "slab offset outside the buffer");
    // the block this call reads (pack: the source) or writes (unpack: the target)
    if (!(unpack ? d.tgt : d.src))
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, unpack ? "link target q is NULL" : "link source q is NULL");
    d.off = off[i];
  }
  // one table per kMaxLinksPerLaunch links in selection order: a later table
  // runs after an earlier one, so its slabs overwrite the earlier ones
  for (int base = 0; base < nsel; base += kMaxLinksPerLaunch) {
    HaloTable tab;
    tab.n = std::min(kMaxLinksPerLaunch, nsel - base);
    int64_t vmax = 0;
    for (int t = 0; t < tab.n; ++t) {
      tab.d[t] = descs[(size_t)(base + t)];
      vmax = std::max<int64_t>(vmax, (int64_t)tab.d[t].ext[0] * tab.d[t].ext[1] * tab.d[t].ext[2]);
    }
    dim3 grid((unsigned)std::min<int64_t>(grid_for(unpack ? vmax : 5 * vmax), 4096), tab.n);
    if (unpack)
      pdl_launch(k_halo_scatter, grid, kThreads, 0, st, tab, (const double*)buf);
    else
      pdl_launch(k_halo_gather, grid, kThreads, 0, st, tab, buf);
    ctx->launches += 1;
    s = launch_status(ctx, unpack ? "halo unpack launch" : "halo pack launch");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

namespace {

// The step's state copy with the halo fill folded in (copy_fill): per block
// the source and destination state, its dimensions and its links (indices
// into the HaloTable, grouped by target block, in list order within a block).
// Block b owns the CTAs [cta_begin[b], cta_begin[b+1]), `cells` cells each
// (CTAs in proportion to the block's cells): one per thread for tables that
// would not give every SM 16 CTAs so (their time is the per-thread latency),
// else four.
constexpr int kMaxFillBlocks = 64;
struct CopyFillTable {
  int nb, ghost, cells;
  const double* src[kMaxFillBlocks];
  double* dst[kMaxFillBlocks];
  int n[kMaxFillBlocks][3];
  int cta_begin[kMaxFillBlocks + 1];
  short first[kMaxFillBlocks], count[kMaxFillBlocks];
  short order[kMaxLinksPerLaunch];
};
static_assert(sizeof(HaloTable) + sizeof(CopyFillTable) <= 32000, "kernel parameter space");

// dst[b] := src[b] cell by cell, except the ghost cells a link of block b
// covers: those take the source cell of the LAST such link (list order), read
// from the source block's src, i.e. from the pre-exchange states (src is
// never written here).  The same values as a copy followed by the gather and
// the ordered scatter.
__global__ void k_copy_fill(const HaloTable tab, const CopyFillTable ct) {
  grid_dep_wait();
  int b = 0;
  while (b + 1 < ct.nb && ct.cta_begin[b + 1] <= (int)blockIdx.x) ++b;
  const int ni = ct.n[b][0], nj = ct.n[b][1], nk = ct.n[b][2], g = ct.ghost;
  const uint32_t N = (uint32_t)ni * nj * nk;  // < 2^31, checked on the host
  const double* __restrict__ s = ct.src[b];
  double* __restrict__ d = ct.dst[b];
  const int e0 = ct.first[b], e1 = ct.first[b] + ct.count[b];
  const uint32_t c0 = (uint32_t)(blockIdx.x - ct.cta_begin[b]) * (uint32_t)ct.cells;
  for (uint32_t c = c0 + threadIdx.x; c < N && c < c0 + (uint32_t)ct.cells; c += kThreads) {
    const uint32_t t = c / (uint32_t)nk;
    const int k = (int)(c - t * (uint32_t)nk);
    const int i = (int)(t / (uint32_t)nj), j = (int)(t - (uint32_t)i * (uint32_t)nj);
    int L = -1;
    if (i < g || i >= ni - g || j < g || j >= nj - g || k < g || k >= nk - g)
      for (int e = e1 - 1; e >= e0 && L < 0; --e)
        if (slab_covers(tab.d[ct.order[e]], i, j, k)) L = ct.order[e];
    if (L < 0) {
#pragma unroll
      for (int v = 0; v < 5; ++v) d[(size_t)v * N + c] = s[(size_t)v * N + c];
    } else {
      const HaloDesc& h = tab.d[L];
      const int64_t NS = (int64_t)h.sn[0] * h.sn[1] * h.sn[2];
      const int64_t si = h.s0 + (i - h.tlo[0]) * h.sstr[0] + (j - h.tlo[1]) * h.sstr[1] + (k - h.tlo[2]) * h.sstr[2];
#pragma unroll
      for (int v = 0; v < 5; ++v) d[(size_t)v * N + c] = h.src[v * NS + si];
    }
  }
}

}  // namespace

int copy_fill(fj_ctx* ctx, const fj_block* blocks, double* const* dst, int nblocks, const fj_link* links, int nlinks,
              int ghost, cudaStream_t st, bool* done) {
  *done = false;
  if (nblocks > kMaxFillBlocks || nlinks > kMaxLinksPerLaunch) return FJ_OK;  // the separate copy and fill
  for (int b = 0; b < nblocks; ++b)
    if ((int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk >= ((int64_t)1 << 31)) return FJ_OK;
  std::vector<HaloDesc> descs;
  size_t nd = 0;
  int s = build_links(ctx, blocks, nblocks, links, nlinks, ghost, descs, nd);
  if (s != FJ_OK) return s;
  HaloTable tab;
  tab.n = (int)descs.size();
  for (int L = 0; L < tab.n; ++L) tab.d[L] = descs[(size_t)L];
  CopyFillTable ct;
  ct.nb = nblocks;
  ct.ghost = ghost;
  int pos = 0;
  int64_t ctas = 0, narrow = 0;
  for (int b = 0; b < nblocks; ++b) narrow += ((int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk + kThreads - 1) / kThreads;
  ct.cells = narrow < 16 * 148 ? kThreads : 4 * kThreads;
  for (int b = 0; b < nblocks; ++b) {
    ct.src[b] = blocks[b].q;
    ct.dst[b] = dst[b];
    ct.n[b][0] = blocks[b].ni;
    ct.n[b][1] = blocks[b].nj;
    ct.n[b][2] = blocks[b].nk;
    ct.first[b] = (short)pos;
    for (int L = 0; L < tab.n; ++L)
      if (tab.d[L].tgt_block == b) ct.order[pos++] = (short)L;
    ct.count[b] = (short)(pos - ct.first[b]);
    ct.cta_begin[b] = (int)ctas;
    ctas += ((int64_t)blocks[b].ni * blocks[b].nj * blocks[b].nk + ct.cells - 1) / ct.cells;
  }
  ct.cta_begin[nblocks] = (int)ctas;
  if (ctas == 0) return FJ_OK;
  pdl_launch(k_copy_fill, dim3((unsigned)ctas), kThreads, 0, st, tab, ct);
  ctx->launches += 1;
  s = launch_status(ctx, "copy-fill launch");
  if (s == FJ_OK) *done = true;
  return s;
}

int apply_bc(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_bc* bcs, int nbcs,
             const fj_params* p, cudaStream_t st) {
  for (int b = 0; b < nbcs; ++b) {
    const fj_bc& e = bcs[b];
    if (e.block < 0 || e.block >= nblocks)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bc block index out of range");
    if (e.face < 0 || e.face > 5)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bc face out of range");
    if (e.type != FJ_BC_WALL && e.type != FJ_BC_SYMMETRY && e.type != FJ_BC_FARFIELD)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "unsupported bc type");
  }
  for (int face = 0; face < 6; ++face) {
    std::vector<BcDesc> ds;
    for (int b = 0; b < nbcs; ++b) {
      const fj_bc& e = bcs[b];
      if (e.face != face) continue;
      const fj_block& blk = blocks[e.block];
      BcDesc d;
      d.q = blk.q;
      d.n[0] = blk.ni; d.n[1] = blk.nj; d.n[2] = blk.nk;
      d.face = face;
      d.type = e.type;
      d.iso = e.isothermal;
      d.T_wall = e.T_wall;
      for (int v = 0; v < 5; ++v) d.qinf[v] = e.q_inf[v];
      ds.push_back(d);
    }
    for (size_t base = 0; base < ds.size(); base += kMaxBcPerLaunch) {
      BcTable tab;
      tab.n = (int)std::min<size_t>(kMaxBcPerLaunch, ds.size() - base);
      tab.gamma = p->gamma;
      tab.R = p->R;
      int64_t vmax = 0;
      for (int t = 0; t < tab.n; ++t) {
        tab.d[t] = ds[base + t];
        const int ax = face >> 1;
        int64_t area = (int64_t)tab.d[t].n[0] * tab.d[t].n[1] * tab.d[t].n[2] / tab.d[t].n[ax];
        vmax = std::max<int64_t>(vmax, area * p->ghost);
      }
      dim3 grid((unsigned)std::min<int64_t>(grid_for(vmax), 4096), tab.n);
      pdl_launch(k_bc, grid, kThreads, 0, st, tab, p->ghost);
      ctx->launches += 1;
      int s = launch_status(ctx, "bc launch");
      if (s != FJ_OK) return s;
    }
  }
  return FJ_OK;
}

// ---------------------------------------------------------------------------
// Transposes (adjoint) of the halo fill and of the linear boundary conditions,
// applied in place to per-block adjoint arrays laid out like q.
// ---------------------------------------------------------------------------
namespace {

// A target cell's value after the fill comes from its last writer's source
// cell; the cell's own original value is discarded.
__device__ __forceinline__ bool later_link_covers(const HaloTable& tab, int L, int ti, int tj, int tk) {
  const HaloDesc& d = tab.d[L];
  for (int L2 = L + 1; L2 < tab.n; ++L2) {
    if (tab.d[L2].tgt_block == d.tgt_block && slab_covers(tab.d[L2], ti, tj, tk)) return true;
  }
  return false;
}

// pass 0: scratch := lam at last-writer target cells (else 0); pass 1: zero
// every target cell; pass 2: lam[source] += scratch.
__global__ void k_halo_transpose(const HaloTable tab, double* __restrict__ scratch, int pass) {
  const int L = blockIdx.y;
  const HaloDesc& d = tab.d[L];
  const int64_t V = (int64_t)d.ext[0] * d.ext[1] * d.ext[2];
  const int64_t NT = (int64_t)d.tn[0] * d.tn[1] * d.tn[2];
  const int64_t NS = (int64_t)d.sn[0] * d.sn[1] * d.sn[2];
  double* tgt = d.tgt;
  double* src = const_cast<double*>(d.src);
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < V;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(r % d.ext[2]);
    const int b = (int)((r / d.ext[2]) % d.ext[1]);
    const int a = (int)(r / ((int64_t)d.ext[2] * d.ext[1]));
    const int ti = d.tlo[0] + a, tj = d.tlo[1] + b, tk = d.tlo[2] + c;
    const int64_t tc = cell_index(d.tn, ti, tj, tk);
    if (pass == 0) {
      const bool last = !later_link_covers(tab, L, ti, tj, tk);
#pragma unroll
      for (int v = 0; v < 5; ++v) scratch[d.off + v * V + r] = last ? tgt[v * NT + tc] : 0.0;
    } else if (pass == 1) {
#pragma unroll
      for (int v = 0; v < 5; ++v) tgt[v * NT + tc] = 0.0;
    } else {
      const int64_t sc = d.s0 + a * d.sstr[0] + b * d.sstr[1] + c * d.sstr[2];
#pragma unroll
      for (int v = 0; v < 5; ++v) atomicAdd(src + v * NS + sc, scratch[d.off + v * V + r]);
    }
  }
}

// Transpose of one face's farfield (lam(outer) := 0) or mirror BC
// (lam(inner) += s lam(outer); lam(outer) := 0).
__global__ void k_bc_transpose(const BcTable tab, int g) {
  const BcDesc& d = tab.d[blockIdx.y];
  const int ax = d.face >> 1;
  const int oa = ax == 0 ? 1 : 0, ob = ax == 2 ? 1 : 2;
  const int64_t NT = (int64_t)d.n[0] * d.n[1] * d.n[2];
  const int64_t V = (int64_t)d.n[oa] * d.n[ob];
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < V;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(r % d.n[ob]);
    const int x = (int)(r / d.n[ob]);
    // the layers of one (x, y) line in one thread: outer and inner sets are disjoint
    for (int o = 0; o < g; ++o) {
      int outer, inner;
      bc_layers(d.face, d.n[ax], g, o, outer, inner);
      int io[3], ii[3];
      io[ax] = outer; ii[ax] = inner;
      io[oa] = x; ii[oa] = x;
      io[ob] = y; ii[ob] = y;
      const int64_t co = cell_index(d.n, io[0], io[1], io[2]);
      const int64_t ci = cell_index(d.n, ii[0], ii[1], ii[2]);
      if (d.type != FJ_BC_FARFIELD) {
        double s[5] = {1.0, 1.0, 1.0, 1.0, 1.0};
        if (d.type == FJ_BC_WALL) {
          s[1] = s[2] = s[3] = -1.0;
        } else {
          s[1 + ax] = -1.0;
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) d.q[v * NT + ci] += s[v] * d.q[v * NT + co];
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) d.q[v * NT + co] = 0.0;
    }
  }
}

}  // namespace

int halo_transpose(fj_ctx* ctx, const fj_block* lam, int nblocks, const fj_link* links, int nlinks,
                   int ghost, double* scratch, size_t scratch_bytes, cudaStream_t st) {
  if (nlinks == 0) return FJ_OK;
  if (nlinks > kMaxLinksPerLaunch)
    return set_err(ctx, FJ_ERR_NOT_IMPLEMENTED, "adjoint halo limited to 192 links");
  std::vector<HaloDesc> descs;
  size_t nd = 0;
  int s = build_links(ctx, lam, nblocks, links, nlinks, ghost, descs, nd);
  if (s != FJ_OK) return s;
  if (scratch_bytes < nd * sizeof(double))
    return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "halo scratch too small");
  HaloTable tab;
  tab.n = (int)descs.size();
  int64_t vmax = 0;
  for (int t = 0; t < tab.n; ++t) {
    tab.d[t] = descs[t];
    vmax = std::max<int64_t>(vmax, (int64_t)tab.d[t].ext[0] * tab.d[t].ext[1] * tab.d[t].ext[2]);
  }
  dim3 grid((unsigned)std::min<int64_t>(grid_for(vmax), 4096), tab.n);
  for (int pass = 0; pass < 3; ++pass) {
    k_halo_transpose<<<grid, kThreads, 0, st>>>(tab, scratch, pass);
    ctx->launches += 1;
    s = launch_status(ctx, "halo transpose launch");
    if (s != FJ_OK) return s;
  }
  return FJ_OK;
}

int bc_transpose(fj_ctx* ctx, const fj_block* lam, int nblocks, const fj_bc* bcs, int nbcs,
                 const fj_params* p, cudaStream_t st) {
  for (int b = 0; b < nbcs; ++b) {
    if (bcs[b].block < 0 || bcs[b].block >= nblocks || bcs[b].face < 0 || bcs[b].face > 5)
      return set_err(ctx, FJ_ERR_INVALID_ARGUMENT, "bc entry out of range");
    if (bcs[b].type == FJ_BC_WALL && bcs[b].isothermal)
      return set_err(ctx, FJ_ERR_NOT_IMPLEMENTED, "the adjoint of the isothermal wall is not implemented");
  }
  for (int face = 5; face >= 0; --face) {  // reverse of the Face-order application
    std::vector<BcDesc> ds;
    for (int b = 0; b < nbcs; ++b) {
      if (bcs[b].face != face) continue;
      const fj_block& blk = lam[bcs[b].block];
      BcDesc d;
      d.q = blk.q;
      d.n[0] = blk.ni; d.n[1] = blk.nj; d.n[2] = blk.nk;
      d.face = face;
      d.type = bcs[b].type;
      d.iso = 0;
      d.T_wall = 0.0;
      for (int v = 0; v < 5; ++v) d.qinf[v] = 0.0;
      ds.push_back(d);
    }
    for (size_t base = 0; base < ds.size(); base += kMaxBcPerLaunch) {
      BcTable tab;
      tab.n = (int)std::min<size_t>(kMaxBcPerLaunch, ds.size() - base);
      tab.gamma = p->gamma;
      tab.R = p->R;
      int64_t vmax = 0;
      for (int t = 0; t < tab.n; ++t) {
        tab.d[t] = ds[base + t];
        const int ax = face >> 1;
        vmax = std::max<int64_t>(vmax, (int64_t)tab.d[t].n[0] * tab.d[t].n[1] * tab.d[t].n[2] / tab.d[t].n[ax]);
      }
      dim3 grid((unsigned)std::min<int64_t>(grid_for(vmax), 4096), tab.n);
      k_bc_transpose<<<grid, kThreads, 0, st>>>(tab, p->ghost);
      ctx->launches += 1;
      int s = launch_status(ctx, "bc transpose launch");
      if (s != FJ_OK) return s;
    }
  }
  return FJ_OK;
}

}  // namespace fj
