/*
 * famrdp_cuda.h -- C ABI of libfamrdp_cuda.so, the sm_100a kernels behind the
 * famrdp_jax RHS + TVD-RK3 step path.
 *
 * Conventions
 *   - Every array argument is a DEVICE pointer to contiguous float64 data in
 *     the reference's C-order layout (famrdp_jax core/types.py:26-89):
 *       q    (5, ni, nj, nk)   [rho, rho*u, rho*v, rho*w, rho*E], ghosts embedded
 *       xyz  (3, ni, nj, nk)
 *       kxyz (3, 3, ni, nj, nk)  kxyz[l][m] = d xi_l / d x_m
 *       jac, vol (ni, nj, nk)
 *     so k is the contiguous axis.  The caller owns all of them.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls are stream-ordered and asynchronous unless stated otherwise.
 *   - Every entry point returns an int status (FJ_OK = 0).  A context-taking
 *     call records a message retrievable with fj_last_error(ctx).  No C++
 *     exception crosses this boundary.
 *   - A context (fj_ctx) owns only scratch memory (stage buffers and
 *     intermediate fluxes) and must be used from one host thread and one stream
 *     at a time.
 *
 * The reference is pure Python/JAX and has no FFI; each entry point replaces
 * one Python function of famrdp_jax (cited beside it, path:line relative to
 * that project), and the Python shim in famrdp_jax_b200 keeps that function's
 * name, signature and error behaviour.
 */
#ifndef FAMRDP_CUDA_H
#define FAMRDP_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FJ_ABI_VERSION 1

enum fj_status {
  FJ_OK = 0,
  FJ_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad enum value   */
  FJ_ERR_CUDA = 2,             /* a CUDA runtime call or launch failed      */
  FJ_ERR_NOT_IMPLEMENTED = 3,  /* e.g. orient != 0 (mesh/halo.py:86-87)     */
  FJ_ERR_SHAPE = 4,            /* halo slab extents differ (mesh/halo.py:53) */
  FJ_ERR_NONFINITE = 5,        /* a reduction found NaN/Inf                  */
  FJ_ERR_NO_MEMORY = 6,        /* scratch allocation failed                  */
  FJ_ERR_SCRATCH_LIMIT = 7     /* block too large for the fixed scratch of
                                  fj_rhs_noalloc_f64                         */
};

/* Size of the fixed device scratch behind fj_rhs_noalloc_f64 (64 MiB). */
#define FJ_NOALLOC_SCRATCH_BYTES (64u << 20)

enum fj_pipeline { FJ_PIPELINE_FUSED = 0, FJ_PIPELINE_STAGED = 1, FJ_PIPELINE_SPLIT = 2 };
enum fj_visc_law { FJ_VISC_SUTHERLAND = 0, FJ_VISC_CONSTANT = 1 };
enum fj_limiter { FJ_LIM_MINMOD = 0, FJ_LIM_VANLEER = 1 };
enum fj_precision { FJ_PREC_F64 = 0, FJ_PREC_F32FLUX = 1 };
enum fj_face { FJ_IMIN = 0, FJ_IMAX = 1, FJ_JMIN = 2, FJ_JMAX = 3, FJ_KMIN = 4, FJ_KMAX = 5 };
enum fj_bc_type { FJ_BC_WALL = 2, FJ_BC_SYMMETRY = 3, FJ_BC_FARFIELD = 4 };

/* Gas model + scheme (GasModel core/types.py:159-167, SchemeChoice :170-176). */
typedef struct fj_params {
  double gamma;
  double R;
  double mu0;
  double T0;
  double Ts;
  double Pr;            /* GasModel.Pr_lam                                  */
  double eps_entropy;   /* Harten parameter; the reference always uses 0.1  */
  int visc_law;         /* enum fj_visc_law                                 */
  int limiter;          /* enum fj_limiter                                  */
  int ghost;            /* ghost layers; the kernels require 2              */
  int precision;        /* enum fj_precision                                */
} fj_params;

/* One block of a multi-block state. */
typedef struct fj_block {
  double* q;            /* (5, ni, nj, nk)                                  */
  const double* kxyz;   /* (3, 3, ni, nj, nk)                               */
  const double* vol;    /* (ni, nj, nk)                                     */
  int ni, nj, nk;       /* padded extents                                   */
} fj_block;

/* One CUT1TO1 face (a BlockTopology.neighbors entry, mesh/halo.py:79-90).
 * Links are applied in array order; the caller lists them in the reference's
 * (block, neighbors-dict) iteration order.
 * orient:
 *   0      the reference's copy (mesh/halo.py:36-53): the source's 2-layer
 *          slab next to src_face, element by element in array order, into
 *          the target's ghost slab; the two slabs must have equal shapes;
 *   1      the marker the reference's topology reader stores for every
 *          interface (mesh/io_top.py:183): FJ_ERR_NOT_IMPLEMENTED, as the
 *          reference's halo fill raises (mesh/halo.py:86-87);
 *   8..15  FJ_ORIENT_MAPPED | bits (no counterpart in the reference): the
 *          ghost layer at distance d from the interface takes the source's
 *          interior layer at distance d (any pair of faces), and the target
 *          face's two tangential axes, in i, j, k order, map onto the source
 *          face's: FJ_ORIENT_SWAP pairs the first with the second,
 *          FJ_ORIENT_REV_A / FJ_ORIENT_REV_B run the target's first / second
 *          tangential axis backwards on the source.  Tangential extents must
 *          match (full extents, ghosts included), else FJ_ERR_SHAPE;
 *   other  FJ_ERR_NOT_IMPLEMENTED. */
#define FJ_ORIENT_MAPPED 8
#define FJ_ORIENT_SWAP 1
#define FJ_ORIENT_REV_A 2
#define FJ_ORIENT_REV_B 4
typedef struct fj_link {
  int tgt_block, tgt_face;
  int src_block, src_face;
  int orient;
} fj_link;

/* One physical boundary face (physics/bc/dispatch.py:11-32).  The caller lists
 * them per block in Face enum order; blocks are independent. */
typedef struct fj_bc {
  int block, face, type;   /* type: enum fj_bc_type                         */
  int isothermal;          /* WALL only: 1 = isothermal, 0 = adiabatic      */
  double T_wall;           /* WALL isothermal only                          */
  double q_inf[5];         /* FARFIELD only                                 */
} fj_bc;

typedef struct fj_ctx fj_ctx;

/* ---- library / context --------------------------------------------------- */
int fj_abi_version(void);
const char* fj_status_string(int status);
int fj_ctx_create(fj_ctx** out);             /* on the current CUDA device  */
int fj_ctx_destroy(fj_ctx* ctx);
const char* fj_last_error(const fj_ctx* ctx);
/* Selects how the context evaluates RHS / RK stages (no counterpart in the
 * reference): FJ_PIPELINE_SPLIT (default) runs three barrier-free kernels per
 * stage over all blocks at once (primitives; face fluxes + viscous fluxes;
 * assembly + combine) through scratch; FJ_PIPELINE_FUSED runs one
 * shared-memory streaming kernel per stage and block; FJ_PIPELINE_STAGED runs
 * the six-kernel reference decomposition (kept as a cross-check).  A plan
 * keeps the pipeline chosen when it was created.  For the fused kernel, `seg` = planes per CTA
 * along i (0 = chosen from the block size and the SM count) and `tile` picks
 * the (j, k) tile shape, 0 .. FJ_NUM_TILES-1: 8x32, 4x32, 6x32, 8x16, 16x32,
 * 8x64, 16x16 (the last three FP32-flux only; FP64 maps them to 8x32/8x16). */
#define FJ_NUM_TILES 7
int fj_ctx_set_pipeline(fj_ctx* ctx, int pipeline, int seg, int tile);
/* Launch shape of the RHS adjoint's face and viscous kernels (a tuning knob;
 * results agree to the rounding of atomic accumulation order): 0 = the
 * fastest measured (default; face kernel register-capped per precision,
 * viscous kernel capped at 64 registers; with FP32 fluxes both VJPs in one
 * launch of interleaved CTAs), 1 = face kernel uncapped, 2 = the
 * other face cap, 3 = 0 and 4 = 2 with the viscous kernel uncapped.  The
 * reference has no counterpart. */
#define FJ_NUM_ADJ_VARIANTS 5
int fj_ctx_set_adjoint_variant(fj_ctx* ctx, int variant);
/* Number of kernels launched through this context so far (instrumentation;
 * the reference has no counterpart). */
int fj_launch_count(const fj_ctx* ctx, int64_t* out);

/* ---- pointwise building blocks ------------------------------------------- */
/* physics/eos.py:12-17 cons_to_prim over ncell cells, (5, ncell) -> (5, ncell) */
int fj_cons_to_prim_f64(const double* q, double* pv, int64_t ncell, double gamma,
                        void* stream);
/* physics/eos.py:5-9 prim_to_cons */
int fj_prim_to_cons_f64(const double* pv, double* q, int64_t ncell, double gamma,
                        void* stream);
/* flux/roe.py:21-85 roe_flux: UL, UR (5, nface), nxyz (3, nface) -> F (5, nface) */
int fj_roe_flux_f64(const double* UL, const double* UR, const double* nxyz, double* F,
                    int64_t nface, double gamma, double eps_entropy, void* stream);
/* physics/reconstruct/muscl2.py:5-12 minmod / vanleer elementwise over n values */
int fj_limiter_f64(const double* a, const double* b, double* out, int64_t n, int limiter,
                   void* stream);
/* physics/reconstruct/muscl2.py:18-37 on pv (nv, n1, n2, n3) along axis 1..3;
 * pvL/pvR have extent n_axis-3 along that axis. */
int fj_muscl2_f64(const double* pv, double* pvL, double* pvR, int nv, int n1, int n2,
                  int n3, int axis, int limiter, void* stream);

/* ---- right-hand side (one block) ------------------------------------------ */
/* rhs/invscd.py:18-133 compute_invscd_rhs */
int fj_invscd_rhs_f64(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
                      double* rhs, int ni, int nj, int nk, const fj_params* p,
                      void* stream);
/* rhs/viscous.py:19-119 compute_viscous_rhs */
int fj_viscous_rhs_f64(fj_ctx* ctx, const double* q, const double* kxyz, double* rhs,
                       int ni, int nj, int nk, const fj_params* p, void* stream);
/* solver/step.py:10-15 _rhs_block = inviscid + viscous */
int fj_rhs_f64(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
               double* rhs, int ni, int nj, int nk, const fj_params* p, void* stream);

/* The same result as fj_rhs_f64 for callers that cannot allocate device
 * memory.  No counterpart in the reference.  It takes no context and never
 * calls cudaMalloc/cudaFree: its intermediates live in one fixed device array
 * of FJ_NOALLOC_SCRATCH_BYTES inside the library.  The array is reserved on a
 * device when its module loads there -- at first use under lazy module
 * loading (the CUDA default), at context creation on every device that uses
 * the library under CUDA_MODULE_LOADING=EAGER -- and kept until the process
 * exits.  Meant for callers whose device memory is
 * owned by a framework (e.g. an XLA custom call under JAX, whose allocator has
 * reserved most of the GPU) or by a fixed start-up budget.
 *   - Limit: the intermediates need about 232 bytes per padded cell in FP64
 *     (116 with precision FJ_PREC_F32FLUX), so blocks of up to ~289,000 padded
 *     cells (e.g. 66^3) in FP64; larger blocks return FJ_ERR_SCRATCH_LIMIT
 *     before any device work.
 *   - The first call on a device looks up the array's device address (with
 *     that device current); make that first call before any stream capture.
 *   - All calls share the one array: calls that can run at the same time on
 *     one device (different streams, or different host threads) race on it
 *     and must be ordered by the caller.  The array keeps the last call's
 *     contents; no call depends on them.
 *   - A call that finds a CUDA error pending on the calling thread returns
 *     FJ_ERR_CUDA without launching and leaves that error in place.
 *   - The array's device address is cached per device for the process's
 *     life: cudaDeviceReset while the library is in use is not supported. */
int fj_rhs_noalloc_f64(const double* q, const double* kxyz, const double* vol, double* rhs,
                       int ni, int nj, int nk, const fj_params* p, void* stream);

/* ---- halo fill and boundary conditions (in place) ------------------------- */
/* mesh/halo.py:56-92 halo_exchange: every link reads its source slab from the
 * pre-exchange arrays; later links overwrite earlier ones. */
int fj_halo_exchange_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks,
                         const fj_link* links, int nlinks, int ghost, void* stream);
/* One device's part of mesh/halo.py:56-92 when the blocks of a topology live
 * on several devices (block sharding; the reference is single-device and has
 * no counterpart).  `blocks` lists EVERY block of the topology (dimensions
 * always; q may be NULL for a block this call neither reads nor writes) and
 * `links` the whole link list.  sel[0..nsel) selects links by index; slab i
 * occupies buf[off[i] .. off[i] + 5*V_i), V_i = the cells of the target face's
 * ghost box (g layers x the target block's two other extents), values in
 * (variable, a, b, c) order over that box.
 *   fj_halo_pack_f64:   gathers each selected link's source slab (the source
 *                       blocks' q must be set) into buf;
 *   fj_halo_unpack_f64: writes the slabs into the selected links' targets
 *                       (their q must be set) in selection order; where the
 *                       ghost boxes of two selected links of one target block
 *                       overlap, the later one wins.
 * A sharded fill is: pack every link whose source is local (before any
 * unpack, so that all sources are pre-exchange values), move the slabs of
 * links whose target lives elsewhere to that device, then unpack every link
 * whose target is local in list order.  Returns FJ_ERR_INVALID_ARGUMENT for a
 * slab outside [0, buf_doubles) or a NULL q the call needs. */
int fj_halo_pack_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                     int ghost, const int* sel, const int64_t* off, int nsel, double* buf,
                     int64_t buf_doubles, void* stream);
int fj_halo_unpack_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                       int ghost, const int* sel, const int64_t* off, int nsel, const double* buf,
                       int64_t buf_doubles, void* stream);
/* physics/bc/dispatch.py:11-32 apply_bc for all blocks */
int fj_apply_bc_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_bc* bcs,
                    int nbcs, const fj_params* p, void* stream);

/* ---- the time step ------------------------------------------------------- */
/* solver/step.py:18-56 step: halo + BC once, then three TVD-RK3 stages.
 * Reads blocks[b].q (unchanged) and writes the new state to q_out[b], which
 * must not alias any blocks[b].q. */
int fj_step_f64(fj_ctx* ctx, const fj_block* blocks, double* const* q_out, int nblocks,
                const fj_link* links, int nlinks, const fj_bc* bcs, int nbcs,
                const fj_params* p, double dt, void* stream);

/* One TVD-RK3 stage of one block, RHS and combine together (solver/step.py:
 * 45-53 for a single block, without the halo fill):
 *   stage 1: out = q + dt*L(q)
 *   stage 2: out = 0.75*q0 + 0.25*(q + dt*L(q))
 *   stage 3: out = (1/3)*q0 + (2/3)*(q + dt*L(q))
 * `out` must not alias `q`; it may alias `q0` (each cell of q0 is read only by
 * the thread that writes the same cell of out). */
int fj_rk_stage_f64(fj_ctx* ctx, const double* q, const double* q0, const double* kxyz,
                    const double* vol, double* out, int ni, int nj, int nk, const fj_params* p,
                    double dt, int stage, void* stream);

/* A prepared step (solver/step.py:18-56 for a fixed block set): the link and
 * boundary tables are copied and checked once, the metrics are bound (they
 * must stay valid and unchanged while the plan lives) and, for the FP32-flux
 * precision, an FP32 copy of every block's kxyz is built in the layout of the
 * context's pipeline (split: per-cell records, 48 B per cell; fused:
 * field-major).  The plan owns its scratch,
 * so fj_plan_step allocates nothing.  Creation synchronises the device. */
typedef struct fj_plan fj_plan;
int fj_plan_create(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_link* links,
                   int nlinks, const fj_bc* bcs, int nbcs, const fj_params* p, fj_plan** out);
/* One step: reads q_in[b] (unchanged) and writes q_out[b]; q_out[b] may equal
 * q_in[b] (in-place step), but must not partially overlap any state. */
int fj_plan_step(fj_plan* plan, double* const* q_in, double* const* q_out, double dt,
                 void* stream);
/* As fj_plan_step, and also keeps the step's intermediate states for a later
 * fj_step_vjp_saved_f64: q0_save[b] = q_in[b] after the halo fill and the
 * boundary conditions, q1_save[b] and q2_save[b] = the first two stage values.
 * The three saves are distinct (5, ni, nj, nk) arrays that overlap no state. */
int fj_plan_step_save(fj_plan* plan, double* const* q_in, double* const* q_out,
                      double* const* q0_save, double* const* q1_save, double* const* q2_save,
                      double dt, void* stream);
/* Per-block viscosity scale and time step for ensembles of independent
 * instances: with mu0 non-NULL, block b uses mu0[b] in place of p->mu0; with
 * dt non-NULL, block b advances by dt[b] and the dt argument of the step and
 * stage calls is ignored.  NULL restores the plan-wide value.  The arrays are
 * host arrays of nblocks values, copied; captured graphs are dropped. */
int fj_plan_set_ensemble(fj_plan* plan, const double* mu0, const double* dt);
/* fj_plan_step through a CUDA graph: the first call for a given (q_in, q_out,
 * dt) captures the step's launches (copy, halo fill, boundary conditions and
 * the three stages) on a private stream and instantiates them; later calls
 * with the same pointers and dt replay the graph on `stream`.  The plan keeps
 * the FJ_PLAN_MAX_GRAPHS most recently used graphs (a ping-pong loop uses
 * two). */
#define FJ_PLAN_MAX_GRAPHS 4
/* The FP32-flux pressure offset p_ref (the mean pressure over the plan's
 * padded cells at creation; 0 for FP64 plans, which do not use it).  Setting
 * it (any finite value) changes only the rounding of FP32-flux results; plans
 * that hold the shards of one topology set the same value so that their steps
 * match one plan over all blocks bit for bit.  Changing it drops captured
 * graphs.  The reference has no counterpart. */
int fj_plan_p_ref(const fj_plan* plan, double* out);
int fj_plan_set_p_ref(fj_plan* plan, double p_ref);
/* Launch shape of the plan's split kernels (either precision; the shapes
 * differ between FP32-flux and FP64): the register caps (minimum resident CTAs
 * per SM) of the flux and assembly kernels, one of FJ_NUM_SPLIT_VARIANTS; 0 is
 * the default.  Changing it drops captured graphs.  Results do not depend on
 * it. */
#define FJ_NUM_SPLIT_VARIANTS 6
int fj_plan_set_variant(fj_plan* plan, int variant);
/* Stage kernels of an FP32-flux split plan (no counterpart in the reference,
 * whose rhs/step are one XLA program): FJ_KERNEL_SPLIT runs each stage as the
 * three split kernels through scratch; FJ_KERNEL_TILE runs it as ONE
 * persistent launch over a work-list of (8 x 30 (j, k) tile, i-plane) units
 * of all blocks, each CTA streaming along i with its primitive planes staged
 * by TMA (cp.async.bulk.tensor) from a padded FP32 copy that holds the
 * periodic images, every intermediate in shared memory or registers.  The
 * results agree to FP32 rounding (the face arithmetic is the same; the
 * temperature is formed in FP32).  FJ_KERNEL_TILE returns
 * FJ_ERR_NOT_IMPLEMENTED for FP64 or non-split plans and when the driver's
 * tensor-map encoder is unavailable.
 * FJ_KERNEL_PERSIST runs the WHOLE step (halo gathers and scatters, boundary
 * faces, primitives and the three stages of all blocks) as ONE persistent
 * launch over a work-list fixed at plan creation; every item waits on device
 * completion counters for the items it reads (a halo scatter for all gathers,
 * a block's BC faces for the scatters into it and its earlier faces, an
 * assembly chunk for the flux chunks of its neighbouring i-planes, a stage of
 * a block for the previous stage of that block), and the flux and assembly
 * chunks of a stage are interleaved so both kinds of work share the SMs.  Its
 * arithmetic is the split kernels', and its results are bit-identical to
 * FJ_KERNEL_SPLIT's.  FJ_ERR_NOT_IMPLEMENTED for FP64 or non-split plans and
 * plans of more than 64 blocks.  fj_plan_stage runs the split kernels for it.
 * FJ_KERNEL_SPLIT_FILL runs the stages with the split kernels and the step's
 * ghost fill -- halo gathers and scatters, boundary faces in Face order and
 * the stage-1 primitives -- as ONE launch of FJ_KERNEL_PERSIST's work-list
 * head (the boundary conditions fused with the halo); bit-identical to
 * FJ_KERNEL_SPLIT, same conditions as FJ_KERNEL_PERSIST.
 * Changing the kernel drops captured graphs. */
#define FJ_KERNEL_SPLIT 0
#define FJ_KERNEL_TILE 1
#define FJ_KERNEL_PERSIST 2
#define FJ_KERNEL_SPLIT_FILL 3
int fj_plan_set_kernel(fj_plan* plan, int kernel);
int fj_plan_get_kernel(const fj_plan* plan, int* kernel);
/* Launch shape of FJ_KERNEL_PERSIST, one of FJ_NUM_PERSIST_SHAPES (0 is the
 * default): resident CTAs per SM (its register cap) and how many flux chunks
 * an assembly chunk trails the last flux chunk it reads by.  Results do not
 * depend on it.  Drops captured graphs. */
#define FJ_NUM_PERSIST_SHAPES 4
int fj_plan_set_persist_shape(fj_plan* plan, int shape);
/* Diagnostic of FJ_KERNEL_PERSIST's work-list, host only (no device work; the
 * q / kxyz / vol pointers of blocks are not read): builds the list the plan of
 * these blocks, links and boundary entries would run for `grid` resident CTAs
 * in launch shape `shape`, stores its length in *n_items (may be NULL) and
 * returns FJ_OK when every item waits only for items ahead of it (the
 * property that makes the launch deadlock-free), FJ_ERR_INVALID_ARGUMENT
 * when not (or for bad arguments), FJ_ERR_NOT_IMPLEMENTED when the persistent
 * step does not apply to the configuration. */
int fj_persist_list_check(const fj_block* blocks, int nblocks, const fj_link* links, int nlinks,
                          const fj_bc* bcs, int nbcs, const fj_params* p, int grid, int shape,
                          int64_t* n_items);
/* Diagnostics of the bounded waits of the tile kernel (every wait for a TMA
 * copy) and of the persistent step (every wait on a completion counter): a
 * wait gives up after `limit` tries (-1 restores the default, about a
 * second); a CTA whose wait gave up records it in the plan's error word and
 * exits (the tile kernel after its copies in flight have landed; the
 * persistent step raises an abort flag on which every other CTA stops taking
 * items) -- never a trap or a hang.  fj_plan_check waits for `stream`, stores
 * the words (bit 0: the tile kernel's, bit 1: the persistent step's; 0 = no
 * wait gave up) in *word, clears them, and returns FJ_ERR_CUDA when one was
 * nonzero.  limit = 0 makes every wait give up at once (used by the tests;
 * the persistent step's results are then incomplete). */
int fj_plan_set_wait_limit(fj_plan* plan, int limit);
int fj_plan_check(fj_plan* plan, int* word, void* stream);
/* Split-pipeline plans of two or more blocks: n = 2 splits the blocks into two
 * groups of about equal cells whose three stages run on two streams (forked
 * from and joined back into the step's stream), so one group's flux kernels
 * overlap the other group's assemblies; n = 1 (default) runs all blocks per
 * launch on one stream.  Results do not depend on it.  Drops captured graphs. */
int fj_plan_set_streams(fj_plan* plan, int n);
/* The autotuner: times `reps` steps q_in -> q_out (after one untimed step) for
 * every launch shape (split plans, both precisions) and stream count (split plans of
 * two or more blocks) with CUDA events on `stream`, keeps the fastest in the
 * plan and reports it as shape + FJ_NUM_SPLIT_VARIANTS * (streams - 1),
 * 2 * FJ_NUM_SPLIT_VARIANTS for the tile kernel,
 * 2 * FJ_NUM_SPLIT_VARIANTS + 1 + k for the persistent step in shape k, or
 * 2 * FJ_NUM_SPLIT_VARIANTS + 1 + FJ_NUM_PERSIST_SHAPES for FJ_KERNEL_SPLIT_FILL
 * in the best split shape (FP32-flux plans where those kernels are available:
 * more candidates) (and,
 * if ms_out is non-NULL, the FJ_AUTOTUNE_CANDIDATES mean step times at those
 * indices; 0 where not timed).  q_out is overwritten; q_in is not changed.
 * Synchronises the stream. */
#define FJ_AUTOTUNE_CANDIDATES (2 * FJ_NUM_SPLIT_VARIANTS + 2 + FJ_NUM_PERSIST_SHAPES)
int fj_plan_autotune(fj_plan* plan, double* const* q_in, double* const* q_out, double dt, int reps,
                     int* chosen, double* ms_out, void* stream);
int fj_plan_step_graph(fj_plan* plan, double* const* q_in, double* const* q_out, double dt,
                       void* stream);
int fj_plan_destroy(fj_plan* plan);
/* One TVD-RK3 stage (1..3) of every block of the plan, without the halo fill
 * (solver/step.py:45-53): out[b] from q[b] (stage input) and q0[b] (step start
 * state); out[b] may alias q0[b], never q[b].  With the split pipeline this is
 * three launches over all blocks. */
int fj_plan_stage(fj_plan* plan, double* const* q, double* const* q0, double* const* out,
                  double dt, int stage, void* stream);

/* ---- adjoint (the reference differentiates step with jax.grad,
 *      tests/solver/test_grad.py:30-35; these are hand-written reverse modes) -- */
/* out = (dL/dq)^T lam for one block, L = _rhs_block (solver/step.py:10-15);
 * lam and out are (5, ni, nj, nk).  Flux arithmetic follows p->precision. */
int fj_rhs_vjp_f64(fj_ctx* ctx, const double* q, const double* kxyz, const double* vol,
                   const double* lam, double* out, int ni, int nj, int nk, const fj_params* p,
                   void* stream);
/* Reverse of one step (solver/step.py:18-56): given lam_in[b] = dJ/dq_new[b]
 * for the state the step produced from blocks[b].q, writes
 * lam_out[b] = dJ/dq[b].  The step's intermediate states are recomputed from
 * blocks[b].q.  Supports CUT1TO1, FARFIELD, SYMMETRY and adiabatic WALL faces
 * (an isothermal wall returns FJ_ERR_NOT_IMPLEMENTED).  lam_out may alias
 * lam_in. */
int fj_step_vjp_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                    double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                    const fj_bc* bcs, int nbcs, const fj_params* p, double dt, void* stream);
/* As fj_step_vjp_f64, and also adds to *dJ_dmu0 (a device double) the
 * derivative of J with respect to the viscosity scale mu0 through this step:
 * the viscous RHS is linear in mu0 for both viscosity laws, so each stage
 * contributes c_s dt lam_{s+1} . L_vis(q_s) / mu0 (c = 1, 1/4, 2/3). */
int fj_step_vjp_mu_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* lam_in,
                       double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                       const fj_bc* bcs, int nbcs, const fj_params* p, double dt, double* dJ_dmu0,
                       void* stream);
/* fj_step_vjp_f64 / fj_step_vjp_mu_f64 on states kept by fj_plan_step_save:
 * blocks[b].q = q0_save[b], and q1[b], q2[b] = q1_save[b], q2_save[b], so the
 * step's forward is not recomputed.  dJ_dmu0 may be NULL. */
int fj_step_vjp_saved_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* q1,
                          const double* const* q2, const double* const* lam_in,
                          double* const* lam_out, int nblocks, const fj_link* links, int nlinks,
                          const fj_bc* bcs, int nbcs, const fj_params* p, double dt,
                          double* dJ_dmu0, void* stream);
/* fj_step_vjp_saved_f64 for an ensemble (fj_plan_set_ensemble): block b uses
 * mu0[b] and dt[b] (host arrays of nblocks values; NULL = p->mu0 / dt), and
 * dJ_dmu0 (device, nblocks doubles, or NULL) receives each block's own
 * dJ/dmu0[b]. */
int fj_step_vjp_ensemble_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* q1,
                             const double* const* q2, const double* const* lam_in,
                             double* const* lam_out, int nblocks, const fj_link* links,
                             int nlinks, const fj_bc* bcs, int nbcs, const fj_params* p,
                             double dt, const double* mu0, const double* dts, double* dJ_dmu0,
                             void* stream);
/* grad[b] = dJ/dq[b] for J = sum over interior cells of vol * 0.5 |rho u|^2 / rho
 * (the objective of fj_kinetic_energy_f64); ghost cells get 0. */
int fj_kinetic_energy_grad_f64(fj_ctx* ctx, const fj_block* blocks, double* const* grad,
                               int nblocks, int ghost, void* stream);

/* time/rk.py:5-20 one Shu-Osher stage combine, elementwise over n values:
 *   stage 1: out = qs + dt*L
 *   stage 2: out = 0.75*q0 + 0.25*(qs + dt*L)
 *   stage 3: out = (1/3)*q0 + (2/3)*(qs + dt*L)                               */
int fj_rk3_combine_f64(const double* q0, const double* qs, const double* L, double* out,
                       int64_t n, double dt, int stage, void* stream);

/* ---- grid metrics --------------------------------------------------------- */
/* mesh/metric.py:31-70 compute_metrics (4th-order central, roll wrap) */
int fj_metrics_f64(const double* xyz, double* jac, double* kxyz, double* vol, int ni,
                   int nj, int nk, void* stream);

/* ---- reductions (FP64; block until the host result is ready) ------------- */
/* Global dt = cfl / max_interior sum_a (|u.n_a| + c) |kxyz[a,:]| / vol. */
int fj_cfl_dt_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, const fj_params* p,
                  double cfl, double* dt_out, void* stream);
/* J = sum_interior vol * 0.5 * (q1^2 + q2^2 + q3^2) / q0 over all blocks. */
int fj_kinetic_energy_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, int ghost,
                          double* out, void* stream);
/* Residual of one step for logging: res_out[v] = sqrt(mean over interior
 * cells of ((blocks[b].q - q_prev[b]) / dt)^2) for each conserved component v
 * (rho, rho u, rho v, rho w, rho E), over all blocks.  Synchronises the
 * stream.  The reference plans such a log (one line per step) but has none. */
int fj_residual_f64(fj_ctx* ctx, const fj_block* blocks, const double* const* q_prev, int nblocks,
                    int ghost, double dt, double* res_out, void* stream);
/* Counts non-finite values of q over all padded cells of all blocks and the
 * minimum density and pressure; returns FJ_ERR_NONFINITE when count > 0 or
 * min rho <= 0 or min p <= 0. */
int fj_check_state_f64(fj_ctx* ctx, const fj_block* blocks, int nblocks, double gamma,
                       int64_t* nonfinite_out, double* min_rho_out, double* min_p_out,
                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FAMRDP_CUDA_H */
