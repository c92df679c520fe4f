/* TEST INFRASTRUCTURE ONLY -- the CPU oracle.  Only tests/, the smoke check
 * and the CPU-baseline leg of bench.py load it; the product never does.
 *
 * Plain-C restatement of the MiniFS iteration path (src/main.cpp:201-291):
 * Roe flux + residual scatter, local time step, LU-SGS sweeps + update, and
 * the node-based Green-Gauss gradient.  It keeps the reference's own loop
 * structure (face loops that scatter into cells, boundary faces first), so a
 * match between it and the GPU's per-cell gathers is evidence that the gather
 * order reproduces the reference's summation order.
 *
 * Parity of this restatement is pinned bit-for-bit against the reference
 * compiled from its own sources (oracle/_ref/minifs_ref) through the golden
 * fixtures in tests/golden/.
 */
#ifndef MINIFS_ORACLE_H
#define MINIFS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Grid after PreprocessGrid: ghost cell of boundary face k is nTCell + k. */
typedef struct {
  int32_t n_node, n_face, n_cell, n_bface;
  const int32_t *f2c;    /* [2*n_face] */
  const int32_t *nnpf;   /* [n_face] */
  const int32_t *f2n;    /* [sum nnpf] */
  const int32_t *bctype; /* [n_bface] */
  const double *xfn, *yfn, *zfn, *area, *xfc, *yfc, *zfc; /* [n_face] */
  const double *xcc, *ycc, *zcc, *vol;                   /* [n_cell + n_bface] */
  const double *wnode;   /* WeightNodeDist [n_node] */
  const int32_t *nmark;  /* Nmark [n_node] */
  const double *wbface;  /* WeightNodeBFace2C, f2n layout of faces [0, n_bface) */
  const int32_t *nnpc;   /* [n_cell] */
  const int32_t *c2n;    /* [sum nnpc] */
  const double *wc2n;    /* WeightNodeC2N [sum nnpc] */
  const int32_t *nodesymm;                          /* [n_node] */
  const double *xfn_n_symm, *yfn_n_symm, *zfn_n_symm; /* [n_node] */
} mfo_grid;

/* Solver globals of para_field_global.cpp (derived values already set). */
typedef struct {
  double gam, gamm1, p_bar, alf_l, lhs_omga;
  double rho_s, rho_min, rho_max, p_min, p_max, p_break;
  double cfl_start, cfl_end, cfl_ratio, ratio_dtmax;
  int32_t cfl_nstep;
} mfo_params;

/* Mutable solver state; arrays are the reference's SoA blocks. */
typedef struct {
  double *q;     /* rho,u,v,w,p blocks of n = n_cell + n_bface  [5n] */
  double *res;   /* [5*n_cell] */
  double *dt;    /* [n_cell] */
  double *dq;    /* DQ [5n] */
  double *diag;  /* [n_cell], LU-SGS diagonal of the last ForwardLUSGS */
  double *dqdx, *dqdy, *dqdz; /* [5n] each */
  double dt_max, dt_min, cfl_min;
  int32_t iter_done;
} mfo_state;

void mfo_zero_residuals(const mfo_grid *g, mfo_state *s);
void mfo_inviscid_flux(const mfo_grid *g, const mfo_params *p, mfo_state *s);
void mfo_compute_timestep(const mfo_grid *g, const mfo_params *p, mfo_state *s);
void mfo_forward_lusgs(const mfo_grid *g, const mfo_params *p, mfo_state *s);
void mfo_calculate_gradient(const mfo_grid *g, const mfo_params *p, mfo_state *s);
void mfo_residual_norm(const mfo_grid *g, const mfo_state *s, double out[5]);
/* n iterations of main.cpp:201-291; norms[5*it + k] gets the L2 norm of
 * residual component k after iteration it (may be NULL). */
void mfo_iterate(const mfo_grid *g, const mfo_params *p, mfo_state *s, int32_t n, double *norms);
/* One matrix-free LU-SGS flux (forward_lusgs.cpp:1271-1324), for unit tests. */
void mfo_flux_lusgs(double flux[5], const double q[5], const double dq[5], const double n[3],
                    double gam, double p_bar, double lhs_omga);
/* UpdateFlowField3D_CFL3d (forward_lusgs.cpp:1335-1488) on the first C cells
 * of q [5][n] (primitive) with DQ [5][n] (conservative), for unit tests. */
void mfo_update_flow(const mfo_params *p, int32_t C, int64_t n, double *q, const double *DQ);
/* One Roe face flux with the 1/2*area factor (cal_flux.cpp:676-834). */
void mfo_roe_flux(double flux[5], const double ql[5], const double qr[5], double nx, double ny,
                  double nz, double area, double gam, double gamm1, double p_bar, double alf_l);

#ifdef __cplusplus
}
#endif
#endif
