// fj_split_dev.cuh -- device code of the split stage pipeline shared by its
// three kernels (fj_stage_split.cu) and the persistent step kernel
// (fj_step_persist.cu): the block table, cell decoding, record access, the
// L2 fills and the per-cell / per-chunk bodies of the primitive, flux and
// assembly kernels.
//
// NC template arguments select the load path of the intermediates: true for
// the read-only (non-coherent) path, which is valid while no kernel of the
// same launch writes them (the three-kernel pipeline); false for plain
// loads, which the persistent kernel needs because its own items write the
// primitives and fluxes other items read after a device-scope acquire.
#pragma once

#include "fj_common.cuh"
#include "fj_physics.cuh"
#include "fj_rhs.cuh"
#include "fj_split.cuh"

namespace fj {
namespace sd {

constexpr int kSplitThreads = 256;

// Division of a non-negative int by a run-time constant (multiply-high form).
struct FastDiv {
  uint32_t d, m, s;
  __host__ void init(uint32_t dd) {
    d = dd;
    s = 0;
    while ((1u << s) < d) ++s;
    m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << s) - d)) / d + 1);
  }
  __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi(n, m) + n) >> s; }
};

struct Dev {
  SplitBlock blk;
  FastDiv dk, dj;  // n / nk, n / nj
};

struct Table {
  int n;
  Dev b[kMaxSplitBlocks];
};
static_assert(sizeof(Table) <= 32764, "kernel parameter space (sm_70+, CUDA 12.1+)");

// Locates the block of CTA `cta` (blocks own contiguous, increasing CTA
// ranges): the last b with cta_begin <= cta, by bisection.
__device__ __forceinline__ int find_block(const Table& t, int cta) {
  int lo = 0, hi = t.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.b[mid].blk.cta_begin <= cta) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct Cell {
  int i, j, k;
  int64_t c, N;
  int ni, nj, nk;
};

// The pointers of a block that change from stage to stage: the stage input,
// the stage result, the input's primitive records and where the result's go.
// The split kernels read them from the block table where they are used
// (TablePtrs); the persistent step passes them alongside it (StagePtrs).
struct StagePtrs {
  const double* q_;
  double* out_;
  const void* prim_;
  void* prim_next_;
  __device__ __forceinline__ const double* q() const { return q_; }
  __device__ __forceinline__ double* out() const { return out_; }
  __device__ __forceinline__ const void* prim() const { return prim_; }
  __device__ __forceinline__ void* prim_next() const { return prim_next_; }
};

struct TablePtrs {
  const SplitBlock& B;
  __device__ __forceinline__ const double* q() const { return B.q; }
  __device__ __forceinline__ double* out() const { return B.out; }
  __device__ __forceinline__ const void* prim() const { return B.prim; }
  __device__ __forceinline__ void* prim_next() const { return B.prim_next; }
};

// Coordinates of cell c of block d; false past the block's end.
__device__ __forceinline__ bool decode_cell(const Dev& d, int64_t c, Cell& x) {
  const SplitBlock& B = d.blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  if (c >= N) return false;
  const uint32_t t1 = d.dk.div((uint32_t)c);
  x.k = (int)((uint32_t)c - t1 * (uint32_t)B.nk);
  x.i = (int)d.dj.div(t1);
  x.j = (int)(t1 - (uint32_t)x.i * (uint32_t)B.nj);
  x.c = c;
  x.N = N;
  x.ni = B.ni;
  x.nj = B.nj;
  x.nk = B.nk;
  return true;
}

// The cell of this thread in flux / primitive CTA `cta` of the table.
__device__ __forceinline__ bool decode(const Dev& d, int cta, Cell& x) {
  return decode_cell(d, (int64_t)(cta - d.blk.cta_begin) * kSplitThreads + threadIdx.x, x);
}

// ---- record access -------------------------------------------------------
constexpr int kRecP = 8, kRecF = 16, kRecG = 8;  // G: 8 components per record + 1 in Gz
// FP32 face fluxes (the k faces are evaluated in the assembly): a 32-byte record
// (i face 0..4, j face 0..2) and a pair (j face 3..4) per cell
constexpr int kRecFA = 8, kRecFB = 2;
constexpr int kRecP64 = 6;  // FP64 primitive record: rho, u, v, w, p, T (48 bytes)

// The L2 fills of the flux CTA `cta` of block d (thread 0 only): the
// primitives two i-planes ahead (MUSCL's farthest upwind cell) and the
// metrics one i-plane ahead (the right cell of the i-face); nearer ranges were
// fetched by earlier CTAs.  FIELD: the FP64 path (48-byte primitive records,
// FP64 field-major kxyz).
template <typename T, bool K_AOS, bool FIELD>
__device__ __forceinline__ void prefetch_fluxes(const Dev& d, int cta, int cells = kSplitThreads) {
  const SplitBlock& B = d.blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk, si = (int64_t)B.nj * B.nk;
  const int64_t c0 = (int64_t)(cta - B.cta_begin) * cells;
  const int64_t n = min((int64_t)cells, N - c0);
  const int64_t a2 = c0 + 2 * si, m2 = min(n, N - a2);
  const int rec = FIELD ? kRecP64 : kRecP;
  if (m2 > 0) l2_prefetch((const T*)B.prim + a2 * rec, m2 * rec * (int64_t)sizeof(T));
  const int64_t a1 = c0 + si, m1 = min(n, N - a1);
  if (m1 > 0) {
    if (K_AOS && !FIELD)
      l2_prefetch((const T*)B.kaos + a1 * kRecK<T>, m1 * kRecK<T> * (int64_t)sizeof(T));
    else
      for (int lm = 0; lm < 9; ++lm) l2_prefetch(B.kxyz + lm * N + a1, m1 * 8);
  }
}

// The L2 fill of the state range of primitive CTA `cta` (thread 0 only).
__device__ __forceinline__ void prefetch_state(const Dev& d, int cta, int cells = kSplitThreads) {
  const SplitBlock& B = d.blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c0 = (int64_t)(cta - B.cta_begin) * cells;
  const int64_t n = min((int64_t)cells, N - c0);
  for (int v = 0; v < 5; ++v) l2_prefetch(B.q + v * N + c0, n * 8);
}

// The L2 fills of the assembly CTA `cta` of block d (thread 0 only): its own
// range of q, q0, vol, metrics and face fluxes, and the viscous components
// one i-plane ahead (the ones behind were fetched by earlier CTAs).  FIELD:
// field-major intermediates and FP64 kxyz (the FP64 path), else records.
template <typename T, bool K_AOS, bool FIELD>
__device__ __forceinline__ void prefetch_assembly(const Dev& d, int cta, int flags, int stage,
                                                  int cells = kSplitThreads, int begin = -1) {
  const SplitBlock& B = d.blk;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c0 = (int64_t)(cta - (begin < 0 ? B.cta_begin : begin)) * cells;
  const int64_t n = min((int64_t)cells, N - c0);
  if (n <= 0) return;
  if (stage != 0)
    for (int v = 0; v < 5; ++v) l2_prefetch(B.q + v * N + c0, n * 8);
  if (stage == 2 || stage == 3)
    for (int v = 0; v < 5; ++v) l2_prefetch(B.q0 + v * N + c0, n * 8);
  const int64_t a = c0 + (int64_t)B.nj * B.nk, m = min(n, N - a);
  if (FIELD) {
    if (flags & kRhsInvscd) {
      l2_prefetch(B.vol + c0, n * 8);
      // the i and j faces (the assembly evaluates the k faces itself)
      for (int v = 0; v < 10; ++v) l2_prefetch((const T*)B.F + v * N + c0, n * (int64_t)sizeof(T));
    }
    if (flags & kRhsViscous) {
      for (int lm = 0; lm < 9; ++lm) l2_prefetch(B.kxyz + lm * N + c0, n * 8);
      if (m > 0)
        for (int v = 0; v < 9; ++v) l2_prefetch((const T*)B.G + v * N + a, m * (int64_t)sizeof(T));
    }
  } else {
    if (K_AOS) l2_prefetch((const T*)B.kaos + c0 * kRecK<T>, n * kRecK<T> * (int64_t)sizeof(T));
    if (flags & kRhsInvscd) {
      l2_prefetch(B.vol + c0, n * 8);
      l2_prefetch((const T*)B.F + c0 * kRecFA, n * kRecFA * (int64_t)sizeof(T));
      l2_prefetch((const T*)B.Fz + c0 * kRecFB, n * kRecFB * (int64_t)sizeof(T));
    }
    if ((flags & kRhsViscous) && m > 0) {
      l2_prefetch((const T*)B.G + a * kRecG, m * kRecG * (int64_t)sizeof(T));
      l2_prefetch((const T*)B.Gz + a, m * (int64_t)sizeof(T));
    }
  }
}

// Minimum resident CTAs per SM (register caps): FP64 face arithmetic needs
// more registers than FP32 at the same occupancy.
template <typename T>
struct SplitOcc {
  static constexpr int fluxes = sizeof(T) == 8 ? 2 : 3;
  static constexpr int assemble = sizeof(T) == 8 ? 3 : 4;
};

// One value through the read-only path (NC) or a plain load.
template <bool NC, typename V>
__device__ __forceinline__ V ldv(const V* p) {
  if constexpr (NC) return __ldg(p);
  else return *p;
}

// n values of a 16-byte aligned record (n a multiple of 16 / sizeof(T)).
template <typename T, int n, bool NC = true>
__device__ __forceinline__ void ld_rec(const T* __restrict__ p, T* v) {
  if constexpr (sizeof(T) == 4 && n % 8 == 0) {
    // 32-byte records (32-byte aligned): one 256-bit load per 8 floats
#pragma unroll
    for (int i = 0; i < n / 8; ++i) {
      if constexpr (NC)
        asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=f"(v[8 * i]), "=f"(v[8 * i + 1]), "=f"(v[8 * i + 2]), "=f"(v[8 * i + 3]), "=f"(v[8 * i + 4]),
              "=f"(v[8 * i + 5]), "=f"(v[8 * i + 6]), "=f"(v[8 * i + 7])
            : "l"(p + 8 * i));
      else
        asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=f"(v[8 * i]), "=f"(v[8 * i + 1]), "=f"(v[8 * i + 2]), "=f"(v[8 * i + 3]),
                       "=f"(v[8 * i + 4]), "=f"(v[8 * i + 5]), "=f"(v[8 * i + 6]), "=f"(v[8 * i + 7])
                     : "l"(p + 8 * i)
                     : "memory");
    }
  } else if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int i = 0; i < n / 4; ++i) {
      const float4 x = ldv<NC>(reinterpret_cast<const float4*>(p) + i);
      v[4 * i] = x.x;
      v[4 * i + 1] = x.y;
      v[4 * i + 2] = x.z;
      v[4 * i + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < n / 2; ++i) {
      const double2 x = ldv<NC>(reinterpret_cast<const double2*>(p) + i);
      v[2 * i] = x.x;
      v[2 * i + 1] = x.y;
    }
  }
}

template <typename T, int n>
__device__ __forceinline__ void st_rec(T* __restrict__ p, const T* v) {
  if constexpr (sizeof(T) == 4 && n % 8 == 0) {
    // one 256-bit store per 8 floats: whole 32-byte sectors per instruction
#pragma unroll
    for (int i = 0; i < n / 8; ++i)
      asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p + 8 * i), "f"(v[8 * i]),
                   "f"(v[8 * i + 1]), "f"(v[8 * i + 2]), "f"(v[8 * i + 3]), "f"(v[8 * i + 4]), "f"(v[8 * i + 5]),
                   "f"(v[8 * i + 6]), "f"(v[8 * i + 7])
                   : "memory");
  } else if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int i = 0; i < n / 4; ++i)
      reinterpret_cast<float4*>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < n / 2; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
  }
}

template <typename T>
struct Cell6 {
  T r, u, v, w, p, t;
};

template <typename T, bool NC = true>
__device__ __forceinline__ Cell6<T> load_cell(const T* __restrict__ P, int32_t c) {
  T x[kRecP];
  ld_rec<T, kRecP, NC>(P + (size_t)c * kRecP, x);
  return Cell6<T>{x[0], x[1], x[2], x[3], x[4], x[5]};
}

// The nine kxyz[l][m] of cell c, from the record copy (K_AOS) or from the
// caller's field-major FP64 array.
template <typename T, bool K_AOS>
__device__ __forceinline__ void metric9(const SplitBlock& B, int32_t N, int32_t c, T kk[9], T* gcl = nullptr) {
  if constexpr (K_AOS) {
    T x[kRecK<T>];
    ld_rec<T, kRecK<T>>((const T*)B.kaos + (size_t)c * kRecK<T>, x);
#pragma unroll
    for (int lm = 0; lm < 9; ++lm) kk[lm] = x[lm];
    if (gcl) {
      gcl[0] = x[9];
      gcl[1] = x[10];
      gcl[2] = x[11];
    }
  } else {
#pragma unroll
    for (int lm = 0; lm < 9; ++lm) kk[lm] = (T)__ldg(B.kxyz + (size_t)lm * N + c);
  }
}

// Row l (kxyz[l][0..2]) of cell c.
template <typename T, bool K_AOS>
__device__ __forceinline__ void metric_row(const SplitBlock& B, int32_t N, int l, int32_t c, T k[3]) {
  if constexpr (K_AOS) {
    const T* K = (const T*)B.kaos + (size_t)c * kRecK<T> + 3 * l;
    k[0] = __ldg(K);
    k[1] = __ldg(K + 1);
    k[2] = __ldg(K + 2);
  } else {
    const double* K = B.kxyz + (size_t)(3 * l) * N + c;
    k[0] = (T)__ldg(K);
    k[1] = (T)__ldg(K + N);
    k[2] = (T)__ldg(K + 2 * (size_t)N);
  }
}

// Primitives rho u v w p T of one cell from its conserved values, in FP64
// (physics/eos.py:12-17; T = p / max(rho R, 1e-300), rhs/viscous.py:36).
// (iR = 1/R from the host; __drcp_rn is the IEEE round-to-nearest reciprocal,
// the same value as 1.0 / r without a general division.)
__device__ __forceinline__ void prims_of(const double q[5], double gm1, double R, double iR, double out[6]) {
  const double r = q[0];
  const double ir = __drcp_rn(r);
  const double u = q[1] * ir, v = q[2] * ir, w = q[3] * ir;
  const double p = gm1 * (q[4] - r * (0.5 * (u * u + v * v + w * w)));
  out[0] = r;
  out[1] = u;
  out[2] = v;
  out[3] = w;
  out[4] = p;
  out[5] = r * R > 1e-300 ? p * ir * iR : p * 1e300;
}

// Roe face c | c+e_a from the primitives of c-e_a, c, c+e_a, c+2e_a and the
// kxyz rows of c and c+e_a (rhs/invscd.py:62-100).
// POFF: the cells carry p' = p - p_ref (see roe_prim).
template <typename T, bool POFF>
__device__ __forceinline__ void face_from_cells(const Cell6<T>& a0, const Cell6<T>& a1, const Cell6<T>& a2,
                                                const Cell6<T>& a3, const T kl[3], const T kr[3],
                                                const Phys& ph, T* F, T p_ref) {
  Prim<T> cell[4] = {{a0.r, a0.u, a0.v, a0.w, a0.p}, {a1.r, a1.u, a1.v, a1.w, a1.p},
                     {a2.r, a2.u, a2.v, a2.w, a2.p}, {a3.r, a3.u, a3.v, a3.w, a3.p}};
  invscd_face_fast<T, POFF>(cell, kl[0], kl[1], kl[2], kr[0], kr[1], kr[2], (T)ph.gm1, (T)ph.inv_gm1,
                            (T)ph.eps_entropy, ph.limiter, F, p_ref);
}

// With next_prims, also writes the primitives of the stage result (the next
// stage's input) in place of a separate k_split_prims launch.
// Where the assembly reads the intermediates of a cell from: the scratch
// arrays through L1/L2 (the interface lets another source, e.g. a
// shared-memory copy, feed the same arithmetic).
template <typename T, bool K_AOS, bool NC = true>
struct GlobalSrc {
  const SplitBlock& B;
  int32_t N;
  // the i and j faces of cell c: o[0..9]
  __device__ __forceinline__ void F_rec(int32_t c, T* o) const {
    ld_rec<T, kRecFA, NC>((const T*)B.F + (size_t)c * kRecFA, o);
    const float2 z = ldv<NC>(reinterpret_cast<const float2*>(B.Fz) + c);
    o[8] = z.x;
    o[9] = z.y;
  }
  // the five components of face a (0: i, 1: j) of cell c
  __device__ __forceinline__ void F_axis(int32_t c, int a, T* o) const {
    const T* p = (const T*)B.F + (size_t)c * kRecFA;
    if (a == 0) {  // one 256-bit load of the record
      float w[8];
      ld_rec<T, 8, NC>(p, w);
#pragma unroll
      for (int v = 0; v < 5; ++v) o[v] = w[v];
    } else {  // floats 5..7 of the record and the pair
      const float4 x = ldv<NC>(reinterpret_cast<const float4*>(p) + 1);  // floats 4..7
      const float2 z = ldv<NC>(reinterpret_cast<const float2*>(B.Fz) + c);
      o[0] = x.y;
      o[1] = x.z;
      o[2] = x.w;
      o[3] = z.x;
      o[4] = z.y;
    }
  }
  __device__ __forceinline__ void G_rec(int32_t c, T* o) const {
    ld_rec<T, kRecG, NC>((const T*)B.G + (size_t)c * kRecG, o);
  }
  __device__ __forceinline__ void K9(int32_t c, T* kk, T* gcl) const { metric9<T, K_AOS>(B, N, c, kk, gcl); }
};

// The assembly of one cell (rhs/invscd.py:119-131, rhs/viscous.py:86-117,
// solver/step.py:45-53) from the intermediates Src provides.
// fk_m / fk_p: the k faces c-1 | c and c | c+1 (the flux records hold only the
// i and j faces); kk / gcl: the metric record of c, loaded by the caller.
template <typename T, bool K_AOS, class Src, class SP>
__device__ __forceinline__ void assemble_cell(const SplitBlock& B, const SP& sp, const Cell& x, const Src& src,
                                              int flags,
                                              int stage, int next_prims, double gm1, double R, double iR,
                                              double ph_p_ref, const T fk_m[5], const T fk_p[5], const T kk[9],
                                              const T gcl[3]) {
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int32_t si = x.nj * x.nk, sj = x.nk;
  const int n[3] = {x.ni, x.nj, x.nk};
  const int idx[3] = {x.i, x.j, x.k};
  const int32_t st[3] = {si, sj, 1};
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (flags & kRhsInvscd) {
    const bool on[3] = {idx[0] >= 2 && idx[0] <= n[0] - 3, idx[1] >= 2 && idx[1] <= n[1] - 3,
                        idx[2] >= 2 && idx[2] <= n[2] - 3};
    if (on[0] || on[1] || on[2]) {
      const double ivd = __drcp_rn(B.vol[c] + 1e-300);
      T Fc[kRecF];
      src.F_rec(c, Fc);
#pragma unroll
      for (int v = 0; v < 5; ++v) Fc[10 + v] = fk_p[v];
      // the p_ref n part the face fluxes left out: p_ref times the sum over
      // the active axes of the face-normal differences, evaluated in FP64 when
      // the records were built
      const double pg[3] = {ph_p_ref * (double)gcl[0], ph_p_ref * (double)gcl[1], ph_p_ref * (double)gcl[2]};
      T Fm[3][5];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (on[a] && a == 2) {
#pragma unroll
          for (int v = 0; v < 5; ++v) Fm[2][v] = fk_m[v];
        } else if (on[a]) {
          src.F_axis(c - st[a], a, Fm[a]);
        } else {
#pragma unroll
          for (int v = 0; v < 5; ++v) Fm[a][v] = T(0);
        }
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        double dsum;
        if (sizeof(T) == sizeof(double)) {
          dsum = 0.0;  // axis by axis like the reference
#pragma unroll
          for (int a = 0; a < 3; ++a)
            if (on[a]) dsum += (double)(Fc[5 * a + v] - Fm[a][v]);
        } else {
          T s = T(0);
#pragma unroll
          for (int a = 0; a < 3; ++a)
            if (on[a]) s += Fc[5 * a + v] - Fm[a][v];
          dsum = (double)s;
          if (K_AOS && v >= 1 && v <= 3) dsum += pg[v - 1];
        }
        r[v] = -dsum * ivd;
      }
    }
  }
  if (flags & kRhsViscous) {
    // sum_l 0.5 kxyz[l][jj] (G(c+e_l) - G(c-e_l)) per equation, one
    // neighbour record at a time (rhs/viscous.py:86-117)
    const T* Gz = (const T*)B.Gz;
    T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
    for (int l = 0; l < 3; ++l) {
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const int32_t nb = side == 0 ? (idx[l] + 1 == n[l] ? c - (n[l] - 1) * st[l] : c + st[l])
                                     : (idx[l] == 0 ? c + (n[l] - 1) * st[l] : c - st[l]);
        const T s = side == 0 ? T(0.5) : T(-0.5);
        T g[kRecG];
        src.G_rec(nb, g);
        const T gz = Gz[nb];
        const T k0 = s * kk[3 * l], k1 = s * kk[3 * l + 1], k2 = s * kk[3 * l + 2];
        acc[0] += g[0] * k0 + g[1] * k1 + g[2] * k2;
        acc[1] += g[1] * k0 + g[3] * k1 + g[4] * k2;
        acc[2] += g[2] * k0 + g[4] * k1 + g[5] * k2;
        acc[3] += g[6] * k0 + g[7] * k1 + gz * k2;
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) r[e + 1] += (double)acc[e];
  }
  double* out = sp.out() + c;
  if (stage == 0) {
#pragma unroll
    for (int v = 0; v < 5; ++v) out[(size_t)v * N] = r[v];
  } else {
    const double ca = stage == 2 ? 0.75 : 1.0 / 3.0;
    const double cb = stage == 2 ? 0.25 : 2.0 / 3.0;
    const double* q = sp.q() + c;
    const double* q0 = B.q0 + c;
    double qn[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double t = q[(size_t)v * N] + B.dt * r[v];
      qn[v] = stage == 1 ? t : ca * q0[(size_t)v * N] + cb * t;
      out[(size_t)v * N] = qn[v];
    }
    if (next_prims) {
      double pv[6];
      prims_of(qn, gm1, R, iR, pv);
      const T rec[kRecP] = {(T)pv[0], (T)pv[1], (T)pv[2], (T)pv[3], (T)(pv[4] - ph_p_ref), (T)pv[5], T(0), T(0)};
      st_rec<T, kRecP>((T*)sp.prim_next() + (size_t)c * kRecP, rec);
    }
  }
}

// With next_prims, also writes the primitives of the stage result (the next
// stage's input) in place of a separate k_split_prims launch.
// The k face c-1 | c (rhs/invscd.py:62-100) from the stage input's primitive
// records of c-2 .. c+1, the k row of the metrics of c-1 and kr, that of c.
template <typename T, bool K_AOS, bool NC = true>
__device__ __forceinline__ void k_face_left(const SplitBlock& B, const void* prim, int32_t N, int32_t c,
                                            const T kr[3], const Phys& ph, T F[5]) {
  const T* __restrict__ P = (const T*)prim;
  const Cell6<T> a0 = load_cell<T, NC>(P, c - 2), a1 = load_cell<T, NC>(P, c - 1), a2 = load_cell<T, NC>(P, c),
                 a3 = load_cell<T, NC>(P, c + 1);
  T kl[3];
  metric_row<T, K_AOS>(B, N, 2, c - 1, kl);
  face_from_cells<T, K_AOS>(a0, a1, a2, a3, kl, kr, ph, F, K_AOS ? (T)ph.p_ref : T(0));
}

// Cells per assembly CTA: each warp assembles 31 consecutive cells; its 32nd
// lane only evaluates the k face its 31st cell needs on the right.
constexpr int kAsmCells = kSplitThreads / 32 * 31;

// The last b with cta_begin_asm <= cta (the assembly's CTA ranges).
__device__ __forceinline__ int find_block_asm(const Table& t, int cta) {
  int lo = 0, hi = t.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.b[mid].blk.cta_begin_asm <= cta) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ---- the kernels' bodies ---------------------------------------------------

// Primitive record of cell c of B from its state (k_split_prims).
// p_ref != 0 (the record path): the pressure slot holds p - p_ref.
template <typename T>
__device__ __forceinline__ void prims_cell(const SplitBlock& B, int32_t c, double gm1, double R, double iR,
                                           double p_ref) {
  const int32_t N = B.ni * B.nj * B.nk;
  const double* q = B.q + c;
  const double qc[5] = {q[0], q[N], q[2 * (size_t)N], q[3 * (size_t)N], q[4 * (size_t)N]};
  double pv[6];
  prims_of(qc, gm1, R, iR, pv);
  const T rec[kRecP] = {(T)pv[0], (T)pv[1], (T)pv[2], (T)pv[3], (T)(pv[4] - p_ref), (T)pv[5], T(0), T(0)};
  st_rec<T, kRecP>((T*)B.prim + (size_t)c * kRecP, rec);
}

// Flux work of cell x of B (k_split_fluxes): the viscous flux components G(c)
// (rhs/viscous.py:36-105, neighbours wrap around the padded block like
// jnp.roll) and the Roe faces c | c+e_i and c | c+e_j (rhs/invscd.py:53-100)
// for c_a in [1, n_a-3].
template <typename T, bool K_AOS, bool NC>
__device__ __forceinline__ void flux_cell(const SplitBlock& B, const void* prim, const Cell& x, const Phys& ph,
                                          int flags) {
  using M = FastMath<T>;
  // 32-bit cell indices: kRecF N < 2^31 is checked on the host
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int32_t si = x.nj * x.nk, sj = x.nk;
  const T* __restrict__ P = (const T*)prim;
  const bool vis = (flags & kRhsViscous) != 0, inv = (flags & kRhsInvscd) != 0;

  // neighbour offsets with the padded-array wrap (jnp.roll) for the viscous
  // stencil; faces exist only where no wrap is involved
  const int32_t ip = x.i + 1 == x.ni ? c - (x.ni - 1) * si : c + si;
  const int32_t im = x.i == 0 ? c + (x.ni - 1) * si : c - si;
  const int32_t jp = x.j + 1 == x.nj ? c - (x.nj - 1) * sj : c + sj;
  const int32_t jm = x.j == 0 ? c + (x.nj - 1) * sj : c - sj;
  const int32_t kp = x.k + 1 == x.nk ? c - (x.nk - 1) : c + 1;
  const int32_t km = x.k == 0 ? c + (x.nk - 1) : c - 1;

  const Cell6<T> C0 = load_cell<T, NC>(P, c);
  const Cell6<T> Im = load_cell<T, NC>(P, im), Ip = load_cell<T, NC>(P, ip);
  const Cell6<T> Jm = load_cell<T, NC>(P, jm), Jp = load_cell<T, NC>(P, jp);
  const Cell6<T> Km = load_cell<T, NC>(P, km), Kp = load_cell<T, NC>(P, kp);
  T kk[9];
  metric9<T, K_AOS>(B, N, c, kk);

  if (vis) {
    // viscous flux components at c (rhs/viscous.py:36-105)
    const T h = T(0.5);
    const T d[4][3] = {{h * (Ip.u - Im.u), h * (Jp.u - Jm.u), h * (Kp.u - Km.u)},
                       {h * (Ip.v - Im.v), h * (Jp.v - Jm.v), h * (Kp.v - Km.v)},
                       {h * (Ip.w - Im.w), h * (Jp.w - Jm.w), h * (Kp.w - Km.w)},
                       {h * (Ip.t - Im.t), h * (Jp.t - Jm.t), h * (Kp.t - Km.t)}};
    T g[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[m] + d[s][1] * kk[3 + m] + d[s][2] * kk[6 + m];
    T mu = (T)B.mu0;
    if (ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
      const T r = C0.t * (T)ph.inv_T0;
      mu = (T)B.mu0 * (r * M::sqrt_pos(r)) * (T)ph.sfac * M::rcp(C0.t + (T)ph.Ts);
    }
    const T kappa = (T)ph.kap_fac * mu;
    const T third = (T)(1.0 / 3.0);
    const T div_u = g[0][0] + g[1][1] + g[2][2];
    const T t00 = T(2) * mu * (g[0][0] - div_u * third);
    const T t01 = mu * (g[0][1] + g[1][0]);
    const T t02 = mu * (g[0][2] + g[2][0]);
    const T t11 = T(2) * mu * (g[1][1] - div_u * third);
    const T t12 = mu * (g[1][2] + g[2][1]);
    const T t22 = T(2) * mu * (g[2][2] - div_u * third);
    const T rec[kRecG] = {t00, t01, t02, t11, t12, t22,
                          C0.u * t00 + C0.v * t01 + C0.w * t02 + kappa * g[3][0],
                          C0.u * t01 + C0.v * t11 + C0.w * t12 + kappa * g[3][1]};
    st_rec<T, kRecG>((T*)B.G + (size_t)c * kRecG, rec);
    ((T*)B.Gz)[c] = C0.u * t02 + C0.v * t12 + C0.w * t22 + kappa * g[3][2];
  }
  if (inv) {
    // the faces c | c+e_i and c | c+e_j for c_a in [1, n_a - 3]; invalid faces
    // are stored as zeros (never read).  The k faces are left to the
    // assembly, whose issue slots are mostly idle (the flux work is issue-bound)
    T Fr[kRecFA + kRecFB];
#pragma unroll
    for (int v = 0; v < kRecFA + kRecFB; ++v) Fr[v] = T(0);
    T kn[3];
    // with metric records the primitives carry p' = p - p_ref and the FP64
    // correction of the momentum fluxes is in the records
    const T p_ref = K_AOS ? (T)ph.p_ref : T(0);
    if (x.i >= 1 && x.i <= x.ni - 3) {
      const Cell6<T> I2 = load_cell<T, NC>(P, c + 2 * si);
      metric_row<T, K_AOS>(B, N, 0, c + si, kn);
      face_from_cells<T, K_AOS>(Im, C0, Ip, I2, kk, kn, ph, Fr, p_ref);
    }
    if (x.j >= 1 && x.j <= x.nj - 3) {
      const Cell6<T> J2 = load_cell<T, NC>(P, c + 2 * sj);
      metric_row<T, K_AOS>(B, N, 1, c + sj, kn);
      face_from_cells<T, K_AOS>(Jm, C0, Jp, J2, kk + 3, kn, ph, Fr + 5, p_ref);
    }
    st_rec<T, kRecFA>((T*)B.F + (size_t)c * kRecFA, Fr);
    reinterpret_cast<float2*>(B.Fz)[c] = make_float2(Fr[8], Fr[9]);
  }
}

// The flux work of cell x split into three independent parts for the
// role-split kernel of small FP32 tables (k_split_fluxes_roles): each part
// loads only its own operands and writes only its own values, with the
// same arithmetic as flux_cell (bit-identical results).
// The viscous flux components G(c) (the record and Gz).
template <typename T, bool K_AOS>
__device__ __forceinline__ void flux_visc_part(const SplitBlock& B, const void* prim, const Cell& x,
                                               const Phys& ph) {
  static_assert(sizeof(T) == 4, "the role-split flux kernel is the FP32 records path");
  using M = FastMath<T>;
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int32_t si = x.nj * x.nk, sj = x.nk;
  const T* __restrict__ P = (const T*)prim;
  const int32_t ip = x.i + 1 == x.ni ? c - (x.ni - 1) * si : c + si;
  const int32_t im = x.i == 0 ? c + (x.ni - 1) * si : c - si;
  const int32_t jp = x.j + 1 == x.nj ? c - (x.nj - 1) * sj : c + sj;
  const int32_t jm = x.j == 0 ? c + (x.nj - 1) * sj : c - sj;
  const int32_t kp = x.k + 1 == x.nk ? c - (x.nk - 1) : c + 1;
  const int32_t km = x.k == 0 ? c + (x.nk - 1) : c - 1;
  const Cell6<T> C0 = load_cell<T, true>(P, c);
  const Cell6<T> Im = load_cell<T, true>(P, im), Ip = load_cell<T, true>(P, ip);
  const Cell6<T> Jm = load_cell<T, true>(P, jm), Jp = load_cell<T, true>(P, jp);
  const Cell6<T> Km = load_cell<T, true>(P, km), Kp = load_cell<T, true>(P, kp);
  T kk[9];
  metric9<T, K_AOS>(B, N, c, kk);
  const T h = T(0.5);
  const T d[4][3] = {{h * (Ip.u - Im.u), h * (Jp.u - Jm.u), h * (Kp.u - Km.u)},
                     {h * (Ip.v - Im.v), h * (Jp.v - Jm.v), h * (Kp.v - Km.v)},
                     {h * (Ip.w - Im.w), h * (Jp.w - Jm.w), h * (Kp.w - Km.w)},
                     {h * (Ip.t - Im.t), h * (Jp.t - Jm.t), h * (Kp.t - Km.t)}};
  T g[4][3];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int m = 0; m < 3; ++m) g[s][m] = d[s][0] * kk[m] + d[s][1] * kk[3 + m] + d[s][2] * kk[6 + m];
  T mu = (T)B.mu0;
  if (ph.visc_law == 0) {  // Sutherland (physics/eos.py:24-25)
    const T r = C0.t * (T)ph.inv_T0;
    mu = (T)B.mu0 * (r * M::sqrt_pos(r)) * (T)ph.sfac * M::rcp(C0.t + (T)ph.Ts);
  }
  const T kappa = (T)ph.kap_fac * mu;
  const T third = (T)(1.0 / 3.0);
  const T div_u = g[0][0] + g[1][1] + g[2][2];
  const T t00 = T(2) * mu * (g[0][0] - div_u * third);
  const T t01 = mu * (g[0][1] + g[1][0]);
  const T t02 = mu * (g[0][2] + g[2][0]);
  const T t11 = T(2) * mu * (g[1][1] - div_u * third);
  const T t12 = mu * (g[1][2] + g[2][1]);
  const T t22 = T(2) * mu * (g[2][2] - div_u * third);
  const T rec[kRecG] = {t00, t01, t02, t11, t12, t22,
                        C0.u * t00 + C0.v * t01 + C0.w * t02 + kappa * g[3][0],
                        C0.u * t01 + C0.v * t11 + C0.w * t12 + kappa * g[3][1]};
  st_rec<T, kRecG>((T*)B.G + (size_t)c * kRecG, rec);
  ((T*)B.Gz)[c] = C0.u * t02 + C0.v * t12 + C0.w * t22 + kappa * g[3][2];
}

// The Roe face c | c+e_AXIS for c_a in [1, n_a-3], zeros elsewhere: AXIS 0
// (i) writes floats 0..4 of the cell's face record, AXIS 1 (j) floats 5..7
// and the Fz pair, AXIS 2 (k) the cell's 5 values of Fk.
template <typename T, bool K_AOS, int AXIS>
__device__ __forceinline__ void flux_face_part(const SplitBlock& B, const void* prim, const Cell& x,
                                               const Phys& ph) {
  static_assert(sizeof(T) == 4, "the role-split flux kernel is the FP32 records path");
  const int32_t N = (int32_t)x.N, c = (int32_t)x.c;
  const int32_t sa = AXIS == 0 ? x.nj * x.nk : (AXIS == 1 ? x.nk : 1);
  const int ia = AXIS == 0 ? x.i : (AXIS == 1 ? x.j : x.k), na = AXIS == 0 ? x.ni : (AXIS == 1 ? x.nj : x.nk);
  const T* __restrict__ P = (const T*)prim;
  T F[5] = {T(0), T(0), T(0), T(0), T(0)};
  if (ia >= 1 && ia <= na - 3) {
    const Cell6<T> A0 = load_cell<T, true>(P, c - sa), A1 = load_cell<T, true>(P, c),
                   A2 = load_cell<T, true>(P, c + sa), A3 = load_cell<T, true>(P, c + 2 * sa);
    T kc[3], kn[3];
    metric_row<T, K_AOS>(B, N, AXIS, c, kc);
    metric_row<T, K_AOS>(B, N, AXIS, c + sa, kn);
    face_from_cells<T, K_AOS>(A0, A1, A2, A3, kc, kn, ph, F, K_AOS ? (T)ph.p_ref : T(0));
  }
  if (AXIS == 2) {
    T* fk = (T*)B.Fk + (size_t)c * 5;
#pragma unroll
    for (int v = 0; v < 5; ++v) fk[v] = F[v];
    return;
  }
  T* rec = (T*)B.F + (size_t)c * kRecFA;
  if (AXIS == 0) {
    reinterpret_cast<float4*>(rec)[0] = make_float4(F[0], F[1], F[2], F[3]);
    rec[4] = F[4];
  } else {
    rec[5] = F[0];
    reinterpret_cast<float2*>(rec + 6)[0] = make_float2(F[1], F[2]);
    reinterpret_cast<float2*>(B.Fz)[c] = make_float2(F[3], F[4]);
  }
}

// Assembly of the kAsmCells cells from c0 of B (k_split_assemble; all 256
// threads of the CTA call it).  The k faces are evaluated here: lane l of a
// warp evaluates the face on the left of its cell (c-1 | c) and takes the one
// on its right from lane l+1 by shuffle, so no face is evaluated twice and no
// barrier is needed; lane 31's cell is the next warp's first, for which it
// only supplies the face.  With next_prims, also writes the primitives of the
// stage result (the next stage's input).
template <typename T, bool K_AOS, bool NC, class SP>
__device__ __forceinline__ void asm_chunk(const Dev& d, const SP& sp, int64_t c0, int flags, int stage,
                                          int next_prims, double gm1, double R, double iR, const Phys& ph) {
  const SplitBlock& B = d.blk;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c = c0 + warp * 31 + lane;
  Cell x;
  const bool alive = c < N;
  if (alive) {
    const uint32_t t1 = d.dk.div((uint32_t)c);
    x.k = (int)((uint32_t)c - t1 * (uint32_t)B.nk);
    x.i = (int)d.dj.div(t1);
    x.j = (int)(t1 - (uint32_t)x.i * (uint32_t)B.nj);
    x.c = c;
    x.N = N;
    x.ni = B.ni;
    x.nj = B.nj;
    x.nk = B.nk;
  }
  const GlobalSrc<T, K_AOS, NC> src{B, (int32_t)N};
  T kk[9], gcl[3] = {T(0), T(0), T(0)};
  if (alive) src.K9((int32_t)c, kk, K_AOS ? gcl : nullptr);
  T fl[5] = {T(0), T(0), T(0), T(0), T(0)}, fr[5];
  // face c-1 | c exists for k-1 in [1, nk-3]
  if ((flags & kRhsInvscd) && alive && x.k >= 2 && x.k <= x.nk - 2)
    k_face_left<T, K_AOS, NC>(B, sp.prim(), (int32_t)N, (int32_t)c, kk + 6, ph, fl);
#pragma unroll
  for (int v = 0; v < 5; ++v) fr[v] = __shfl_down_sync(0xffffffffu, fl[v], 1);
  if (lane == 31 || !alive) return;
  assemble_cell<T, K_AOS>(B, sp, x, src, flags, stage, next_prims, gm1, R, iR, K_AOS ? ph.p_ref : 0.0, fl, fr, kk,
                          gcl);
}

// asm_chunk with the k faces read from Fk (written by the k-face role of
// k_split_fluxes_roles) instead of evaluated: the face c-1 | c (for k-1 in
// [1, nk-3]) is Fk of c-1, the face c | c+1 is Fk of c (zero where it does not
// exist).  The same values as asm_chunk's shuffled ones, so the same result.
template <typename T, bool K_AOS, class SP>
__device__ __forceinline__ void asm_chunk_kmem(const Dev& d, const SP& sp, int64_t c0, int flags, int stage,
                                               int next_prims, double gm1, double R, double iR, const Phys& ph) {
  const SplitBlock& B = d.blk;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t N = (int64_t)B.ni * B.nj * B.nk;
  const int64_t c = c0 + warp * 31 + lane;
  if (lane == 31 || c >= N) return;
  Cell x;
  const uint32_t t1 = d.dk.div((uint32_t)c);
  x.k = (int)((uint32_t)c - t1 * (uint32_t)B.nk);
  x.i = (int)d.dj.div(t1);
  x.j = (int)(t1 - (uint32_t)x.i * (uint32_t)B.nj);
  x.c = c;
  x.N = N;
  x.ni = B.ni;
  x.nj = B.nj;
  x.nk = B.nk;
  const GlobalSrc<T, K_AOS, true> src{B, (int32_t)N};
  T kk[9], gcl[3] = {T(0), T(0), T(0)};
  src.K9((int32_t)c, kk, K_AOS ? gcl : nullptr);
  T fl[5] = {T(0), T(0), T(0), T(0), T(0)}, fr[5] = {T(0), T(0), T(0), T(0), T(0)};
  if (flags & kRhsInvscd) {
    const T* fk = (const T*)B.Fk;
    if (x.k >= 2 && x.k <= x.nk - 2)
#pragma unroll
      for (int v = 0; v < 5; ++v) fl[v] = __ldg(fk + (c - 1) * 5 + v);
#pragma unroll
    for (int v = 0; v < 5; ++v) fr[v] = __ldg(fk + c * 5 + v);
  }
  assemble_cell<T, K_AOS>(B, sp, x, src, flags, stage, next_prims, gm1, R, iR, K_AOS ? ph.p_ref : 0.0, fl, fr, kk,
                          gcl);
}

}  // namespace sd
}  // namespace fj
