/*
 * mfgpu -- B200 (sm_100a) implementation of the MiniFS iteration hot path.
 *
 * C ABI: plain pointers and sizes, an opaque context, int status codes.
 * Each entry point below names the reference routine it replaces
 * (paths relative to the MiniFS project root).
 *
 * Array conventions follow the reference's PolyGrid after PreprocessGrid:
 *   - C = n_cell, G = n_bface, F = n_face, N = n_node, n = C + G;
 *   - faces [0, G) are boundary faces; the ghost cell of boundary face k is
 *     C + k (SpecifyBC, src/Kernels/load_grid.cpp:893-901);
 *   - flow fields are SoA blocks: q = [rho | u | v | w | p], each block n
 *     long; res is 5 blocks of C; dqdx/dqdy/dqdz and DQ are 5 blocks of n.
 *   - floating point is IEEE double; indices are int32 (number_type.h:26-39).
 *
 * Calls on one context are not reentrant (the reference is single-threaded,
 * main.cpp:201-291).  All device work is issued on the context's stream;
 * entry points that hand data to the host synchronise that stream.
 */
#ifndef MFGPU_H
#define MFGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MFG_OK 0
#define MFG_ERR_INVALID (-1)     /* bad argument, size or field id */
#define MFG_ERR_CUDA (-2)        /* CUDA runtime error (see mfg_last_cuda_error) */
#define MFG_ERR_NOMEM (-3)       /* device or host allocation failed */
#define MFG_ERR_TIMEOUT (-4)     /* a bounded device-side wait gave up */
#define MFG_ERR_NONFINITE (-5)   /* NaN/Inf found in residual or state */
#define MFG_ERR_UNSUPPORTED (-6) /* LU-SGS order inconsistent with layers, etc. */
#define MFG_ERR_BADMESH (-7)     /* degenerate volume, bad connectivity */
#define MFG_ERR_NODEVICE (-8)    /* no CUDA device / wrong architecture */
#define MFG_ERR_IO (-9)          /* file missing, unreadable, truncated or malformed */

/* Boundary-condition codes (src/Base/constant.h:47-51). */
#define MFG_BC_WALL 3
#define MFG_BC_SYMM 4
#define MFG_BC_FAR_FIELD 6
#define MFG_BC_FAR_FIELD_MOD 61
#define MFG_BC_INTERFACE 10

/* Field ids for mfg_download / mfg_upload. */
#define MFG_FIELD_Q 0    /* [5n] rho,u,v,w,p (download/upload) */
#define MFG_FIELD_RES 1  /* [5C] residual (download) */
#define MFG_FIELD_DT 2   /* [C] local time step (download) */
#define MFG_FIELD_DQ 3   /* [5n] LU-SGS increment (download) */
#define MFG_FIELD_DQDX 4 /* [5n] gradient x (download) */
#define MFG_FIELD_DQDY 5 /* [5n] gradient y (download) */
#define MFG_FIELD_DQDZ 6 /* [5n] gradient z (download) */
#define MFG_FIELD_DIAG 7 /* [C] LU-SGS diagonal of the last sweep (download) */
#define MFG_FIELD_LIMITER 8 /* [5C] reconstruction limiter of the last flux (order 3, 4) */

/* Precision modes. */
#define MFG_PREC_FP64 0  /* the drop-in: every operation in FP64, bit-faithful */
#define MFG_PREC_MIXED 1 /* FP32 Roe flux, gradient, LU-SGS off-diagonal terms */

/* Solver parameters: the globals of src/Base/para_field_global.cpp.
 * Fill the inputs (mach ... ratio_dtmax) and call mfg_params_derive to set
 * the dependent values with the formulas of para_field_global.cpp:150-209. */
typedef struct mfg_params {
  /* inputs */
  double mach, alpha, beita, re, T, gam, gascon;
  double cfl_start, cfl_end;
  int32_t cfl_nstep;
  double lhs_omga, epsa_r, ratio_dtmax;
  /* derived */
  double amu, ainf, uqq, u_s, v_s, w_s, p_s, rho_s, p_bar, gamm1;
  double p_stag, e_stag, p_min, p_max, rho_min, rho_max, p_break, e_stag_max;
  double cfl_min, cfl_ratio, alf_l;
} mfg_params;

/* Grid as the reference holds it after PreprocessGrid (load_grid.cpp:405-540).
 * Node-weight arrays are those of ComputeWeight3D_Node and FindNodeSYMM
 * (grid_polyhedra_auxiliary_functions.cpp:831-1049, :2060-2140). */
typedef struct mfg_mesh {
  int32_t n_node, n_face, n_cell, n_bface;
  const int32_t *f2c;    /* [2F]; ghost of boundary face k = C + k */
  const int32_t *nnpf;   /* [F] nodes per face */
  const int32_t *f2n;    /* [sum nnpf] */
  const int32_t *bctype; /* [G] BC type of each boundary face */
  const double *xfn, *yfn, *zfn, *area, *xfc, *yfc, *zfc; /* [F] */
  const double *xcc, *ycc, *zcc, *vol;                   /* [n] */
  const double *wnode;   /* WeightNodeDist [N] */
  const int32_t *nmark;  /* Nmark [N] */
  const double *wbface;  /* WeightNodeBFace2C, f2n layout of faces [0, G) */
  const int32_t *nnpc;   /* nNPC [C] */
  const int32_t *c2n;    /* C2N [sum nnpc] */
  const double *wc2n;    /* WeightNodeC2N [sum nnpc] */
  const int32_t *nodesymm;                            /* [N] */
  const double *xfn_n_symm, *yfn_n_symm, *zfn_n_symm; /* [N] */
  const int32_t *lusgs_order; /* LUSGSCellOrder [C], NULL = identity */
  const int32_t *lusgs_layer; /* LUSGSLayer [n], NULL = identity */
} mfg_mesh;

typedef struct mfg_ctx mfg_ctx;

/* Statistics of a context (level sets, memory). */
typedef struct mfg_info {
  int32_t n_cell, n_face, n_node, n_bface;
  int32_t fw_levels, bw_levels;     /* LU-SGS level-set counts */
  int32_t max_level_cells;          /* widest level */
  int32_t precision;
  int64_t device_bytes;             /* device memory held by the context */
  int32_t sweep_mode;               /* 0 = one launch per level, 1 = persistent */
  int32_t graph_ready;
  int32_t ncase;                    /* independent cases in the context (1 unless batched) */
  int32_t sweep_chunks;             /* persistent sweeps: chunks (= resident blocks) */
  int32_t sweep_lanes;              /* persistent sweeps: lanes per cell */
  int32_t sweep_records;            /* persistent sweeps: record slots per cell (4 or 8) */
  int32_t sweep_chunking;           /* persistent sweeps: chunk assignment (MFG_CHUNK_*) */
  /* records of the [forward, backward] sweep whose neighbour increment is
   * read from the block's shared-memory ring, from global memory (same
   * chunk, older than the ring) and from another chunk (polled in L2) */
  int32_t sweep_ring_records[2], sweep_global_records[2], sweep_cross_records[2];
  double sweep_model_us[2];         /* modelled duration of each sweep with its chunks */
  int32_t sweep_kernel;             /* persistent sweep kernels (MFG_SWEEP_*) */
} mfg_info;

/* ---- parameters -------------------------------------------------------- */
/* Reference defaults (para_field_global.cpp:37-221), then derived values. */
void mfg_params_default(mfg_params *p);
/* para_field_global.cpp:150-209 evaluated at run time. */
int mfg_params_derive(mfg_params *p);

/* ---- context ----------------------------------------------------------- */
/* Uploads the grid and the initial state q0 [5n] (ghost states included) to
 * `device` and builds the CSR gathers and LU-SGS level sets.  Replaces the
 * lazy allocations of ZeroResiduals / ComputeTimeStep / ForwardLUSGS
 * (cal_flux.cpp:57-63, compute_timestep.cpp:77-84, forward_lusgs.cpp:112-117)
 * and AllocAndCalQuantityGradient's storage (cal_gradient.cpp:50-78); the
 * gradient itself is computed by the first mfg_calculate_gradient. */
int mfg_create(const mfg_mesh *mesh, const mfg_params *params, const double *q0,
               int32_t device, int32_t precision, mfg_ctx **out);
/* Batched cases: ncase independent grids (each a complete mfg_mesh with its
 * own mfg_params and initial state q0s[k] [5 n_k]) solved together in one
 * context, so that every launch and every level of the LU-SGS sweeps covers
 * all cases at once -- the reference's whole main loop run once per case
 * (main.cpp:170-291), as many cases as fit the device.  The context holds the
 * union grid: the cells of case 0, 1, ..., then the ghosts of case 0, 1, ...
 * (mfg_batch_layout gives the offsets); downloads and uploads use that order.
 * Each case computes exactly what it would alone: same bits, its own CFL
 * ramp, its own dt_max/dt_min, its own first cell of the LU-SGS order.
 * Meshes must use the identity LU-SGS order (lusgs_order = lusgs_layer =
 * NULL); mfg_set_params is not available on a batch. */
int mfg_create_batch(int32_t ncase, const mfg_mesh *meshes, const mfg_params *params,
                     const double *const *q0s, int32_t device, int32_t precision,
                     mfg_ctx **out);
/* cell0[k] = first cell of case k in the union, bface0[k] = its first
 * boundary face (its ghosts start at n_cell + bface0[k]); both [ncase + 1]. */
int mfg_batch_layout(mfg_ctx *ctx, int32_t *cell0, int32_t *bface0);
/* dt_max, dt_min of every case: ext[2k], ext[2k + 1]. */
int mfg_batch_dt_extrema(mfg_ctx *ctx, double *ext);
/* Residual L2 norms per case: out[5k + v]. */
int mfg_batch_residual_norm(mfg_ctx *ctx, double *out);
/* Frees the context's device and pinned host memory, streams, events and
 * graphs. */
int mfg_destroy(mfg_ctx *ctx);
/* Issue all further work on this cudaStream_t (NULL = the context's own). */
int mfg_set_stream(mfg_ctx *ctx, void *cuda_stream);
/* New flow parameters (e.g. another CFL ramp) for the following calls;
 * the captured iteration graphs are rebuilt on the next mfg_iterate.
 * MFG_ERR_UNSUPPORTED for a batch (its cases fix theirs at creation). */
int mfg_set_params(mfg_ctx *ctx, const mfg_params *params);
/* Sizes, level counts, precision, device bytes, and the sweep choices and
 * their record counts (mfg_info above); host-side only. */
int mfg_info_get(mfg_ctx *ctx, mfg_info *info);
/* Sweep strategy: 0 = one kernel per LU-SGS level; 1 (default when the
 * device supports cooperative launch) = one persistent kernel per sweep: the
 * LU-SGS order is cut into one contiguous chunk per resident block, a block
 * walks its chunk level by level, and a cell that depends on another chunk
 * waits, with a bounded spin, for that neighbour's ready flag.  Both modes
 * give identical results. */
int mfg_set_sweep_mode(mfg_ctx *ctx, int32_t mode);
/* Face gather and gradient face sums: lanes = 0, one thread per cell (the
 * default), or one lane per face of a cell with the per-cell sums passed
 * from lane to lane in ascending face order (lanes = 4 where every cell has
 * at most 4 faces, 8 where at most 8; other values MFG_ERR_UNSUPPORTED).
 * Identical results, norms included; the autotuner times both. */
int mfg_set_gather_lanes(mfg_ctx *ctx, int32_t lanes);
/* Persistent sweeps: lanes per cell; the record slots per cell W is the
 * only value the current kernels take (others: MFG_ERR_UNSUPPORTED). */
int mfg_set_sweep_lanes(mfg_ctx *ctx, int32_t lanes);
/* Chunk assignments of the persistent sweeps (one chunk per block).
 * MFG_CHUNK_VOTE: level by level a cell joins the chunk most of its
 * dependencies are in, up to its share of the level (every level spread
 * evenly, many dependencies between chunks).  MFG_CHUNK_TRANSVERSE_*: a
 * grid of chunks over two centroid axes, each cell's label the maximum of
 * its own bucket and its dependencies' labels, so that any dependency path
 * crosses few chunk boundaries.  By default each context takes, per sweep,
 * the assignment with the shortest modelled sweep; mfg_set_chunking(kind)
 * forces one for contexts created afterwards (-1 restores the default).
 * Results are identical with every assignment. */
#define MFG_CHUNK_VOTE 0
#define MFG_CHUNK_TRANSVERSE_XY 1
#define MFG_CHUNK_TRANSVERSE_XZ 2
#define MFG_CHUNK_TRANSVERSE_YZ 3
#define MFG_CHUNK_TRANSVERSE_ANY 4 /* the best transverse grid over any axis pair */
int mfg_set_chunking(int32_t kind);
/* The chunk assignment a context makes for one sweep, on the host (no
 * device; for inspection and tests).  The sweep: L levels over C cells,
 * lptr [L + 1] the level bounds in cells [C] (cells in level order, a
 * permutation of 0..C-1), and the dependencies of the cell at position i
 * in nbs[sptr[i] .. sptr[i + 1]) (cell ids; ids >= C, ghosts, are not
 * dependencies).  xc, yc, zc: cell centroids [C] for the transverse
 * assignments (NULL: the vote only).  P chunks of G lane groups each;
 * force: -1 (the model's choice, as a context makes it) or MFG_CHUNK_*.
 * assign [C]: each cell's chunk; grid (optional, [2]): the transverse
 * grid Pa, Pb (a cell's chunk is la + Pa * lb), 0, 0 for the vote;
 * est_us (optional): the modelled sweep duration.  Returns the assignment
 * made (MFG_CHUNK_*), MFG_ERR_INVALID for inconsistent tables. */
int mfg_plan_chunks(int32_t C, int32_t L, const int32_t *lptr, const int32_t *cells,
                    const int32_t *sptr, const int32_t *nbs, const double *xc,
                    const double *yc, const double *zc, int32_t P, int32_t G, int32_t force,
                    int32_t *assign, int32_t *grid, double *est_us);
/* The persistent sweep kernels.  MFG_SWEEP_DEEP: one block per SM, producer
 * warps staging each cell's static terms ahead for consumer lane pairs that
 * run only the dependent chain -- short per-level latency, for levels of up
 * to about 128 cells per SM.  MFG_SWEEP_WIDE: many 64-thread blocks per SM
 * with small chunks -- for wider levels, whose latency one block hides
 * behind another's work.  A context takes WIDE when its widest level would
 * give a DEEP block more than two passes per level; mfg_set_sweep_kernel
 * forces a kind for contexts created afterwards (-1 restores the default).
 * Identical results either way. */
#define MFG_SWEEP_DEEP 0
#define MFG_SWEEP_WIDE 1
int mfg_set_sweep_kernel(int32_t kind);
/* Times n_trial fused iterations with each lane count the persistent
 * sweeps take on this context's own grid and keeps the faster (ms_out[2],
 * optional, receives the ms per iteration of W and W / 2 lanes; the
 * current kernels take W only, so ms_out[1] is -1).  mfg_autotune covers
 * this and the other launch parameters.  The state and the dt extrema are
 * restored afterwards; res, dt, Diag, DQ and the gradient hold the last
 * trial iteration's values.  iter_done: the CFL ramp position to time at. */
int mfg_autotune_sweeps(mfg_ctx *ctx, int32_t n_trial, int32_t iter_done, double *ms_out);
/* Launch parameters chosen by measurement on the context's own grid (the
 * reference's counterpart is TDTree's fixed partition sizes,
 * grid_polyhedra.cpp:380,405): one pass of coordinate descent over the
 * knobs below, each candidate timed over n_trial fused iterations after two
 * warm-up ones, the fastest kept.  The state and the dt extrema are restored
 * after every trial; res, dt, Diag, DQ and the gradient hold the last
 * trial's values.  iter_done: the CFL ramp position to time at.  rep
 * (optional) receives every trial.  Knobs:
 *   MFG_KNOB_SWEEP_KERNEL  persistent sweep kernels (MFG_SWEEP_*; the
 *                          chunk tables are rebuilt for each)
 *   MFG_KNOB_CHUNKING      chunk assignment: MFG_CHUNK_VOTE or
 *                          MFG_CHUNK_TRANSVERSE_ANY (tables rebuilt)
 * (flags & MFG_TUNE_NO_REBUILD leaves these two as the context has them:
 * a rebuild of a grid of many millions of cells takes seconds)
 *   MFG_KNOB_SWEEP_MODE    1 persistent, 0 one launch per level
 *   MFG_KNOB_GATHER_BLOCKS resident blocks per SM the fused face gather is
 *                          compiled for (its register cap): 2, 3, 4
 *   MFG_KNOB_FLUX_BLOCKS   the same for the per-face Roe flux
 *   MFG_KNOB_NODE_BLOCK    threads per block of the node values
 *   MFG_KNOB_GRAD_BLOCK    threads per block of the gradient face sums
 *   MFG_KNOB_GATHER_LANES  lanes per cell of the face gather and the
 *                          gradient face sums: one lane per face of a cell
 *                          (4 or 8, as the grid's cells allow) or 0 (one
 *                          thread per cell)
 * Results are identical with every choice. */
#define MFG_KNOB_SWEEP_KERNEL 0
#define MFG_KNOB_CHUNKING 1
#define MFG_KNOB_SWEEP_MODE 2
#define MFG_KNOB_GATHER_BLOCKS 3
#define MFG_KNOB_FLUX_BLOCKS 4
#define MFG_KNOB_NODE_BLOCK 5
#define MFG_KNOB_GRAD_BLOCK 6
#define MFG_KNOB_GATHER_LANES 7
#define MFG_TUNE_KNOBS 8
#define MFG_TUNE_CANDS 4
typedef struct mfg_tune_report {
  int32_t n_knobs;
  int32_t knob[MFG_TUNE_KNOBS];                 /* MFG_KNOB_* of each row */
  int32_t n_cand[MFG_TUNE_KNOBS];
  int32_t cand[MFG_TUNE_KNOBS][MFG_TUNE_CANDS]; /* candidate values */
  double ms[MFG_TUNE_KNOBS][MFG_TUNE_CANDS];    /* ms per fused iteration; < 0: not usable */
  int32_t chosen[MFG_TUNE_KNOBS];               /* the value kept */
  double ms_initial, ms_final;                  /* before and after */
} mfg_tune_report;
#define MFG_TUNE_NO_REBUILD 1
int mfg_autotune(mfg_ctx *ctx, int32_t n_trial, int32_t iter_done, int32_t flags,
                 mfg_tune_report *rep);
/* Failure-detection self-test of the bounded waits: runs a forward sweep
 * whose first chunk is withheld, so the cells that depend on it wait for
 * flags that are never set; each wait gives up after spin_cycles SM cycles.
 * Returns MFG_ERR_TIMEOUT and leaves the context's state unchanged and
 * usable (MFG_ERR_UNSUPPORTED when the grid has a single chunk). */
int mfg_selftest_sweep_timeout(mfg_ctx *ctx, int64_t spin_cycles);
/* Self-test of the sweeps' division by a precomputed reciprocal (no
 * counterpart in the reference): n pseudo-random dividend/divisor pairs
 * (seeded, exponents across [-600, 600]) divided both ways on the current
 * device; *mismatches receives the number of results whose bits differ
 * from the division's (0 expected). */
int mfg_selftest_division(int64_t n, uint64_t seed, int64_t *mismatches);
/* Known-answer self-test of the device arithmetic (test hook; the inputs
 * are the reference functions' own arguments): runs the device functions
 * the iteration kernels use on n given inputs, one GPU thread each, and
 * copies the results back to the host.  consts = {gam, p_bar, alf_l
 * (= epsa_r), lhs_omga, rho_min, rho_max, p_min, p_max}; in/out are host
 * arrays.
 *   mode 0 [RoeFlux_noprec, cal_flux.cpp:676-834]: in = ql[5][n], qr[5][n],
 *          nx[n], ny[n], nz[n], area[n]; out = flux[5][n]
 *   mode 1 [FluxLUSGS3D, forward_lusgs.cpp:1271-1324]: in = [n][13]
 *          (q[5], dq[5], normal[3]); out = [n][5]
 *   mode 2 [UpdateFlowField3D_CFL3d, forward_lusgs.cpp:1335-1488]: in =
 *          q[5][n], dq[5][n]; out = updated q[5][n]
 *   mode 3 as mode 1, in the persistent sweeps' form with branch-free
 *          divisions (mfg_selftest_division_fast) */
int mfg_selftest_functions(int32_t mode, int32_t n, const double *consts, const double *in,
                           double *out);
/* Self-test of the persistent sweeps' branch-free reciprocal and quotient
 * (a single-precision seed, Newton-Raphson steps on the FMA and Markstein's
 * correction steps; no counterpart in the reference): n pseudo-random
 * divisor/dividend pairs (seeded; divisor exponents across [-130, 130],
 * every eighth significand all ones) on the current device.  counts[0]:
 * reciprocals, counts[1]: quotients whose bits differ from the division's
 * (0 expected); counts[2]: divisors the fast path leaves to the division. */
int mfg_selftest_division_fast(int64_t n, uint64_t seed, int64_t *counts);

/* ---- the iteration path (reference routine replaced in brackets) -------- */
/* [ZeroResiduals, cal_flux.cpp:54-72] */
int mfg_zero_residuals(mfg_ctx *ctx);
/* [InviscidFlux, cal_flux.cpp:84-192: SetQlQrWithQ + RoeFlux_noprec + LoadFlux]
 * res += sum of first-order Roe face fluxes (cell-centric gather, no atomics). */
int mfg_inviscid_flux(mfg_ctx *ctx);
/* [ComputeTimeStep, compute_timestep.cpp:66-121: TimeStepNormal_new +
 * CellIsMG + LimitTimeStep]; iter_done is the reference's global counter. */
int mfg_compute_timestep(mfg_ctx *ctx, int32_t iter_done);
/* [ForwardLUSGS, forward_lusgs.cpp:67-162: Diag, CalDiagLUSGS, SolveLUSGS3D
 * forward/backward sweeps, UpdateFlowField3D_CFL3d] */
int mfg_forward_lusgs(mfg_ctx *ctx);
/* [CalculateGradient, cal_gradient.cpp:87-167: CompNodeVar3D_dist +
 * CompGradientQ_Gauss_Node for rho,u,v,w,p] */
int mfg_calculate_gradient(mfg_ctx *ctx);
/* [SetGhostVariables, load_grid.cpp:953-1212, inviscid steady case]: the
 * ghost state of every boundary face from its inner cell's current state
 * (WALL and SYMM mirror the velocity, FAR_FIELD from Riemann invariants,
 * INTERFACE untouched, other types keep their ghost; then the rho and p
 * clamps).  The reference calls it once, in PreprocessGrid (its main loop
 * has the call commented out, main.cpp:286); mfg_prep_init_flow does that
 * one.  The subsonic far-field branches use CUDA's pow where the reference
 * uses the C library's, so those ghosts may differ in the last bit. */
int mfg_set_ghost_variables(mfg_ctx *ctx);
/* on = 1: mfg_iterate (and mfg_iterate_host, mfg_profile_phases) call
 * mfg_set_ghost_variables after the LU-SGS update and before the gradient
 * of every iteration, where main.cpp:286 would; on = 0 (the default, the
 * reference's frozen ghosts): they do not. */
int mfg_set_live_bc(mfg_ctx *ctx, int32_t on);
/* Mixed form only (no counterpart in the reference): on = 1 computes the Roe
 * flux wholly in FP64 (the face kernel of the FP64 form; the rest of the
 * iteration stays mixed), on = 0 (the default) its dissipation in FP32.  The
 * FP32 dissipation's rounding leaves a residual floor (near 4e-8 of the
 * initial residual on the wall channel); with the FP64 flux the residual is
 * evaluated in FP64 and converges like the FP64 form's.  The FP64 form
 * accepts on = 1 (its flux is FP64) and rejects on = 0. */
int mfg_set_flux_fp64(mfg_ctx *ctx, int32_t on);
/* The reference's `order` switch (para_field_global.cpp:100: 1 first
 * order; 2 second order without limiter; 3 with Barth's limiter; 4 with
 * Venkatakrishnan's), which the reference declares but does not implement
 * (its reconstruction call is commented out, cal_flux.cpp:175): order >= 2
 * reconstructs each face's inner-cell states linearly from the cell's
 * Green-Gauss gradient to the face centroid, limited per cell and variable
 * for 3 (Barth-Jespersen) and 4 (Venkatakrishnan, eps^2 = (venkat_k h)^3,
 * h = vol^(1/3)); ghost states stay first order; a face whose
 * reconstructed density or absolute pressure is not positive keeps its
 * first-order states.  The flux reads the gradient the previous
 * CalculateGradient left (main.cpp's order of calls); this call and
 * mfg_upload compute it for the current state.  LU-SGS stays first order.
 * No reference output exists for order >= 2.  Default 1. */
int mfg_set_order(mfg_ctx *ctx, int32_t order, double venkat_k);
/* The whole main-loop body (main.cpp:201-291) n times, fused kernels in a
 * CUDA graph.  Each iteration's gradient is computed once, as in the loop;
 * all but the last run beside the next iteration's face kernels (same
 * values; on return the gradient is that of the final state).  norms (optional, host) receives 5 residual L2 norms per
 * iteration (main.cpp:294-317 evaluated every iteration); for a batch
 * norms[(i * ncase + k) * 5 + v]. */
int mfg_iterate(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done, double *norms);
/* End-to-end form with host buffers: copies q_in [5n] (host) in, runs
 * n_iter iterations, copies the state to q_out [5n] and the residual to
 * res_out [5C] (either may be NULL).  Pinned host memory is fastest.  The
 * copies out overlap the last iteration: the residual leaves during its
 * LU-SGS sweeps, the state during its gradient (on a second stream of the
 * context); the call returns when both are in host memory. */
int mfg_iterate_host(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done, const double *q_in,
                     double *q_out, double *res_out, double *norms);
/* Phases of one fused iteration, for mfg_profile_phases. */
#define MFG_NPHASES 6 /* face gather (flux+dt+Diag), forward sweep, backward sweep +
                         update, node values, gradient face sums, norm reduction */
/* Same work as mfg_iterate without the graph, with CUDA events recorded on
 * the context's stream between phases; phase_ms[MFG_NPHASES] receives the
 * summed device time of each phase over the n_iter iterations. */
int mfg_profile_phases(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done, double *phase_ms);
/* [main.cpp:294-317] L2 norm of each residual component. */
int mfg_residual_norm(mfg_ctx *ctx, double out[5]);

/* Allocation-free residual norm (no counterpart in the reference: an extra
 * entry point of this library).  For callers that must not allocate device
 * memory -- code that holds only device pointers and no mfgpu context
 * (creating one allocates), or an application whose device memory budget is
 * owned by another allocator.  res: device pointer to the residual, 5 SoA
 * blocks of n_cell doubles; norms: device pointer receiving 5 doubles (the
 * L2 norm of each component).  Runs on `stream` (a cudaStream_t, NULL = the
 * default stream) on the current device; allocates nothing (no cudaMalloc,
 * cudaFree or allocating library call).
 *   - The block partial sums go to a file-scope __device__ array sized for
 *     MFG_NORM_STATIC_MAX_CELLS cells (2.5 MiB); every device that loads the
 *     library holds it until the process exits.  Larger n_cell is rejected
 *     with MFG_ERR_INVALID (message in mfg_last_cuda_error).
 *   - The first call on a device resolves the array's device address
 *     (cudaGetSymbolAddress, once per device and context); make that first
 *     call before any stream capture.  Under CUDA's lazy module loading
 *     (the default since CUDA 12) that first call may also be the one that
 *     loads this library's device code onto the device and reserves the
 *     2.5 MiB array there, so it can fail with an out-of-memory error when
 *     the device is already full: a caller whose memory is managed by
 *     another allocator should make it early (e.g. once at start-up with
 *     n_cell = 0) while there is room.
 *   - The address is cached per device with the id of the context it was
 *     resolved in; after cudaDeviceReset, or with another context current
 *     (a caller's own driver-API context), the next call resolves it again
 *     in the new context -- make that call outside stream capture too.
 *   - All calls on a device share the one array: calls that overlap on the
 *     GPU (different streams, no ordering between them) race and may return
 *     wrong norms.  Every partial read is written by the same call first, so
 *     no clearing is needed between calls. */
#define MFG_NORM_STATIC_MAX_CELLS (1 << 24)
int mfg_residual_norm_static(const double *res, int32_t n_cell, double *norms, void *stream);
/* The running extrema dt_max / dt_min (para_field_global.cpp:220-221,
 * updated in LimitTimeStep, compute_timestep.cpp:914-918).  For a batch, get
 * returns case 0's and set sets every case's. */
int mfg_get_dt_extrema(mfg_ctx *ctx, double *dt_max, double *dt_min);
int mfg_set_dt_extrema(mfg_ctx *ctx, double dt_max, double dt_min);

/* ---- one mesh over several contexts (the reference's MPI mode) ---------- */
/* A context created from one part of a partitioned mesh, whose faces on a
 * partition cut are boundary faces of type MFG_BC_INTERFACE (their ghost
 * holds the neighbouring part's cell), iterates as the reference's MPI
 * build does when the caller moves the exchange buffers between the parts
 * (NCCL, peer copies, CUDA-aware MPI) between the phases of
 * mfg_halo_phase.  One iteration, every part in step:
 *   MFG_HALO_FACE      ZeroResiduals, InviscidFlux, the part's dt and Diag;
 *                      dt extrema -> ext, squared residual sums -> norm_sq
 *     caller: ext[0] = max over parts, ext[1] = min over parts
 *             (compute_timestep.cpp:921-925)
 *   MFG_HALO_FORWARD   dt limited with ext; forward sweep; DQ* of the sent
 *                      cells -> send_rows
 *     caller: each neighbour's send_rows -> recv_rows
 *             (forward_lusgs.cpp:1030-1053)
 *   MFG_HALO_BACKWARD  recv_rows -> ghost DQ; backward sweep and update; the
 *                      new states of the sent cells -> send_rows
 *     caller: send_rows -> recv_rows (PassInterfaceData, main.cpp:280)
 *   MFG_HALO_NODES     recv_rows -> ghost states; node values, the shared
 *                      nodes' left as partial sums -> node_send
 *     caller: each neighbour's node_send -> node_recv
 *             (CommInternodeDataMPI, cal_gradient.cpp:2293-2301)
 *   MFG_HALO_GRADIENT  shared nodes: own + received partial sums, divided by
 *                      the node weight; Green-Gauss face sums
 *     caller: norm_sq summed over parts (main.cpp:311-312), sqrt
 * Before the first iteration: MFG_HALO_PACK_Q (current states of the sent
 * cells -> send_rows), exchange, then MFG_HALO_NODES and MFG_HALO_GRADIENT
 * for the gradient of the initial state.  MFG_HALO_CHECK synchronises and
 * reports a sweep timeout (MFG_ERR_TIMEOUT).  At second order (mfg_set_order
 * >= 2, the halo registered with grad_send/grad_recv) each iteration starts
 * with MFG_HALO_LIMIT (the limiter of the part's cells; their gradient,
 * limiter and centroid rows -> grad_send), the caller moves each
 * neighbour's grad_send to grad_recv, and MFG_HALO_FACE first places the
 * received rows in the interface ghosts, whose face states are then
 * reconstructed as the neighbouring cells' own (other ghosts stay first
 * order).  The LU-SGS sweeps of a part
 * see a neighbour's increment only through the ghost DQ of the backward
 * sweep, as in the reference, so several parts converge along another
 * path than one mesh does; one part with no neighbours gives mfg_iterate's
 * bits.  The node weights, marks and symmetry normals of the part's mesh
 * must be those of the whole mesh (the reference sums them over parts,
 * grid_polyhedra_auxiliary_functions.cpp:951-1047).  Single-case contexts
 * only, FP64 or mixed (MFG_ERR_UNSUPPORTED for a batch); a context with
 * a halo refuses mfg_iterate, mfg_iterate_host, mfg_forward_lusgs,
 * mfg_calculate_gradient, mfg_profile_phases and mfg_autotune_sweeps. */
typedef struct mfg_halo {
  int32_t n_send;             /* rows sent, all neighbours' segments concatenated */
  const int32_t *send_cells;  /* host [n_send]: local cell of each sent row */
  int32_t n_recv;             /* rows received */
  const int32_t *recv_bfaces; /* host [n_recv]: boundary face (type MFG_BC_INTERFACE)
                                 whose ghost each received row fills */
  int32_t n_node;             /* node entries: a shared node once per neighbour
                                 holding it; sent and received alike */
  const int32_t *nodes;       /* host [n_node]: local node of each entry; a node's
                                 received partial sums are added in entry order */
  double *send_rows;          /* device [n_send][8] (state record: rho,u,v,w,p and
                                 three derived words; DQ rows use the first 5) */
  double *recv_rows;          /* device [n_recv][8] */
  double *node_send;          /* device [n_node][8] (first 5 words used) */
  double *node_recv;          /* device [n_node][8] */
  int64_t *ext;               /* device [2]: dt_max, dt_min as the bits of positive
                                 doubles (their order is that of the int64 values) */
  double *norm_sq;            /* device [5]: the part's sums of squared residuals */
  double *grad_send;          /* device [n_send][24] (second order only, else NULL): the
                                 sent cells' gradients (x, y, z of rho,u,v,w,p), limiter
                                 (1 when unlimited) and centroid (x, y, z, vol^(1/3)) */
  double *grad_recv;          /* device [n_recv][24] */
} mfg_halo;
#define MFG_HALO_PACK_Q 0
#define MFG_HALO_FACE 1
#define MFG_HALO_FORWARD 2
#define MFG_HALO_BACKWARD 3
#define MFG_HALO_NODES 4
#define MFG_HALO_GRADIENT 5
#define MFG_HALO_CHECK 6
#define MFG_HALO_LIMIT 7
/* Registers the exchange lists (copied) and the caller's device buffers
 * (kept; on the context's device, alive while the context is), once per
 * context.  MFG_ERR_INVALID for an index out of range or a received row
 * whose boundary face is not of type MFG_BC_INTERFACE. */
int mfg_halo_set(mfg_ctx *ctx, const mfg_halo *halo);
/* Launches one phase on the context's stream (mfg_set_stream shares it
 * with the communication library); iter_done sets the CFL of
 * MFG_HALO_FACE as in mfg_compute_timestep.  Asynchronous except
 * MFG_HALO_CHECK. */
int mfg_halo_phase(mfg_ctx *ctx, int32_t phase, int32_t iter_done);

/* ---- data movement ----------------------------------------------------- */
int mfg_download(mfg_ctx *ctx, int32_t field, double *host);
int mfg_upload(mfg_ctx *ctx, int32_t field, const double *host);
/* Waits for the work issued on the context's stream. */
int mfg_sync(mfg_ctx *ctx);

/* ---- diagnostics ------------------------------------------------------- */
const char *mfg_error_string(int32_t code);
const char *mfg_last_cuda_error(void);
/* Number of kernels this library launched (all contexts), for accounting. */
int64_t mfg_kernel_launches(void);

/* ---- host preprocessing (restatements of the reference's setup) -------- */
/* Raw grid as read from a FlowStar binary file (ReadMFlowGrid_binary,
 * load_grid.cpp:129-273): boundary faces first, f2c[2k+1] = -patch id. */
typedef struct mfg_raw_grid {
  int32_t n_node, n_face, n_cell, n_bface;
  const double *x, *y, *z;
  const int32_t *nnpf, *f2n;
  int32_t *f2c; /* rewritten in place by mfg_prep_specify_bc */
} mfg_raw_grid;

/* [SpecifyBC, load_grid.cpp:804-902]: bctype[k] = patch_types[patch(k) - 1],
 * f2c[2k+1] = C + k. */
int mfg_prep_specify_bc(mfg_raw_grid *g, int32_t n_patch, const int32_t *patch_types,
                        int32_t *bctype);
/* [PolyGrid::ComputeMetrics, grid_polyhedra.cpp:1071-1118]: outputs sized
 * [F] for face arrays and [n] for cell arrays. */
int mfg_prep_metrics(const mfg_raw_grid *g, double *xfn, double *yfn, double *zfn, double *area,
                     double *xfc, double *yfc, double *zfc, double *xcc, double *ycc,
                     double *zcc, double *vol);
/* [AllocAndInitFlowfield + SetGhostVariables, load_grid.cpp:571-601,
 * :953-1212] with an optional Gaussian density bump at the cell centroids
 * rho = rho_s*(1 + amp*exp(-|x - x0|^2 / (2 sigma^2))) applied in between. */
int mfg_prep_init_flow(const mfg_raw_grid *g, const mfg_params *p, const int32_t *bctype,
                       const double *xfn, const double *yfn, const double *zfn,
                       const double *xcc, const double *ycc, const double *zcc,
                       double bump_amp, double bump_sigma, double bump_x0, double bump_y0,
                       double bump_z0, double *q);
/* Sizes for mfg_prep_node_weights: *n_c2n = sum over cells of distinct nodes. */
int mfg_prep_c2n_size(const mfg_raw_grid *g, int64_t *n_c2n);
/* [CalnNPC/CalC2N + ComputeWeight3D_Node + FindNodeSYMM]. */
int mfg_prep_node_weights(const mfg_raw_grid *g, const int32_t *bctype, const double *xfn,
                          const double *yfn, const double *zfn, const double *xfc,
                          const double *yfc, const double *zfc, const double *xcc,
                          const double *ycc, const double *zcc, double *wnode, int32_t *nmark,
                          double *wbface, int32_t *nnpc, int32_t *c2n, double *wc2n,
                          int32_t *nodesymm, double *xfn_n_symm, double *yfn_n_symm,
                          double *zfn_n_symm);

/* ---- FlowStar files ----------------------------------------------------- */
/* A binary grid file as ReadMFlowGrid_binary (load_grid.cpp:129-273) reads
 * it: int32 n_node, n_face, n_cell; double x[n_node], y[], z[]; int32
 * nnpf[n_face], f2n[sum nnpf], f2c[2 n_face]; then, in a partitioned file,
 * the interface block int32 n_iface, nbz[n_iface] (zone of the face's other
 * side), nbf[n_iface] (its face there), int32 n_inode, nbsn[n_inode] (own
 * node), nbzn[] (zone), nbrn[] (node there).  A serial file ends with
 * n_iface = n_inode = 0 (the reference reads the block unless the stream
 * has already hit its end, which an exact read never does); a file that
 * ends right after f2c reads as having no interfaces.  On reading, a face
 * whose first cell is a boundary (f2c[2i] < 0) has its node order reversed
 * after the first node and its two cells swapped, and n_bface counts the
 * faces with a negative neighbour, as the reference does (:209-229); the
 * boundary faces must come first for SpecifyBC, as in the format.  The
 * fields n_node ... f2c are mfg_raw_grid's, in the same order. */
typedef struct mfg_mfl {
  int32_t n_node, n_face, n_cell, n_bface;
  double *x, *y, *z;
  int32_t *nnpf, *f2n, *f2c;
  int32_t n_iface;
  int32_t *nbz, *nbf;
  int32_t n_inode;
  int32_t *nbsn, *nbzn, *nbrn;
} mfg_mfl;
/* Allocates *out (free with mfg_mfl_free).  MFG_ERR_IO for a missing,
 * truncated or inconsistent file (negative counts, nnpf < 1, extra bytes
 * after the interface block). */
int mfg_mfl_read(const char *path, mfg_mfl **out);
/* Writes the arrays as given, with the interface block (zeros when
 * n_iface = n_inode = 0).  n_bface is not stored: the reader recounts it. */
int mfg_mfl_write(const char *path, const mfg_mfl *g);
int mfg_mfl_free(mfg_mfl *g);
/* bc.para (ReadMFlowBoundaryCondition, load_grid.cpp:282-314): the patch
 * count, then one "patch_id type" pair per patch, in file order (SpecifyBC
 * indexes this table by position: patch p is record p - 1).  Reads at most
 * `cap` records; *n_patch is the file's count (MFG_ERR_INVALID if above
 * cap, MFG_ERR_IO if the file is short or malformed). */
int mfg_bc_read(const char *path, int32_t cap, int32_t *n_patch, int32_t *patch_id,
                int32_t *type);
int mfg_bc_write(const char *path, int32_t n_patch, const int32_t *patch_id,
                 const int32_t *type);

/* Checkpoint of a run (no counterpart in the reference, which has none):
 * the whole solver state between iterations -- the states of cells and
 * ghosts q [5n] (mfg_download of MFG_FIELD_Q), the iteration count that
 * sets the CFL ramp, and the running dt extrema (mfg_get_dt_extrema).  A
 * context restored from it (mfg_upload, mfg_set_dt_extrema, the count
 * passed on) continues with the bits of the uninterrupted run.  Read checks
 * the magic word, the sizes against n_cell / n (MFG_ERR_INVALID for
 * another grid) and the length (MFG_ERR_IO). */
int mfg_checkpoint_write(const char *path, int64_t n_cell, int64_t n, int32_t iter_done,
                         double dt_max, double dt_min, const double *q);
int mfg_checkpoint_read(const char *path, int64_t n_cell, int64_t n, int32_t *iter_done,
                        double *dt_max, double *dt_min, double *q);

/* ---- the same preprocessing on a GPU ------------------------------------ */
/* ComputeMetrics, CalnNPC/CalC2N, ComputeWeight3D_Node and FindNodeSYMM run
 * on `device`: every output is bit-identical to mfg_prep_metrics,
 * mfg_prep_c2n_size and mfg_prep_node_weights on the same raw grid.
 * mfg_prep_gpu_run copies the raw grid (host arrays, f2c as rewritten by
 * mfg_prep_specify_bc) and bctype to the device, checks every node and cell
 * index there (MFG_ERR_BADMESH, nothing computed, if one is out of range),
 * and computes all outputs; it returns MFG_ERR_BADMESH for a cell volume
 * below 1e-40, as mfg_prep_metrics does.  The getters copy the results into
 * host arrays sized and laid out as the host entries' outputs.  The
 * initial flow field (mfg_prep_init_flow) stays on the host: its exp and pow
 * are the C library's. */
typedef struct mfg_prep_gpu mfg_prep_gpu;
int mfg_prep_gpu_run(const mfg_raw_grid *g, const int32_t *bctype, int32_t device,
                     mfg_prep_gpu **out);
int mfg_prep_gpu_c2n_size(const mfg_prep_gpu *p, int64_t *n_c2n);
int mfg_prep_gpu_metrics(mfg_prep_gpu *p, double *xfn, double *yfn, double *zfn, double *area,
                         double *xfc, double *yfc, double *zfc, double *xcc, double *ycc,
                         double *zcc, double *vol);
int mfg_prep_gpu_node_weights(mfg_prep_gpu *p, double *wnode, int32_t *nmark, double *wbface,
                              int32_t *nnpc, int32_t *c2n, double *wc2n, int32_t *nodesymm,
                              double *xfn_n_symm, double *yfn_n_symm, double *zfn_n_symm);
/* Device time of the preprocessing kernels of the last mfg_prep_gpu_run, ms
 * (CUDA events around them; the copies of the raw grid are outside). */
int mfg_prep_gpu_kernel_ms(const mfg_prep_gpu *p, double *ms);
int mfg_prep_gpu_destroy(mfg_prep_gpu *p);
/* mfg_prep_init_flow for a device-resident preprocessing: the boundary
 * normals, cell centroids, boundary f2c and BC types it reads are copied to
 * the host and the host routine fills q [5n] (host memory). */
int mfg_prep_gpu_init_flow(mfg_prep_gpu *p, const mfg_params *params, double bump_amp,
                           double bump_sigma, double bump_x0, double bump_y0, double bump_z0,
                           double *q);
/* A context built on the device from a device-resident preprocessing, for
 * the identity LU-SGS order: the context mfg_create makes from the arrays
 * of that preprocessing (the same tables, the same results), without their
 * round trip through the host.  Slots, face records, level sets, sweep
 * records and node lists are built by device kernels; the chunk assignment
 * of the persistent sweeps runs on the host (both sweeps at once).  q0 [5n]
 * is host memory; the device is the preprocessing's, which stays valid. */
int mfg_create_from_prep(const mfg_prep_gpu *prep, const mfg_params *params, const double *q0,
                         int32_t precision, mfg_ctx **out);

#ifdef __cplusplus
}
#endif
#endif /* MFGPU_H */
