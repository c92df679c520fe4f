/* TEST INFRASTRUCTURE ONLY -- the CPU oracle (see minifs_oracle.h).
 *
 * Every function restates one reference routine with the same loop order and
 * the same floating-point expression order; the citation in front of each
 * names the lines it follows.  Build: oracle/Makefile (gcc -O2
 * -ffp-contract=off, so no fused multiply-adds, like the reference's x86-64
 * g++ -O3 build).
 */
#include "minifs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MFO_TINY 1.e-40 /* number_type.h:29 */
#define MFO_BIG 1.e40   /* number_type.h:28 */
#define MFO_WALL 3      /* constant.h:47-51 */
#define MFO_SYMM 4
#define MFO_FAR_FIELD 6
#define MFO_INTERFACE 10

/* std::min / std::max semantics: min(a,b) = (b < a) ? b : a */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

static inline int64_t nq(const mfo_grid *g) { return (int64_t)g->n_cell + g->n_bface; }

void mfo_zero_residuals(const mfo_grid *g, mfo_state *s) {
  /* cal_flux.cpp:54-72 */
  memset(s->res, 0, sizeof(double) * 5 * (size_t)g->n_cell);
}

/* cal_flux.cpp:676-834 (serial body of RoeFlux_noprec), one face. */
void mfo_roe_flux(double flux[5], const double ql[5], const double qr[5], double areax,
                  double areay, double areaz, double area, double gam, double gamm1,
                  double p_bar, double alf_l) {
  (void)gam;
  double rho_a, u_a, v_a, w_a, h_a, c_a, c2_a, vn_a, q2;
  double vn_l, et_l, ht_l, vn_r, et_r, ht_r;
  double tmp0, tmp1, tmp2, alpha1, alpha2, alpha3, eigv1, eigv2, eigv3;
  double drho, du, dv, dw, dp, dvn, dq2;
  double spectral, epsaa, epsbb, epscc, epsa_r;

  et_l = (ql[4] + p_bar) / gamm1 + 0.5 * ql[0] * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
  et_r = (qr[4] + p_bar) / gamm1 + 0.5 * qr[0] * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
  ht_l = et_l + ql[4] + p_bar;
  ht_r = et_r + qr[4] + p_bar;

  vn_l = areax * ql[1] + areay * ql[2] + areaz * ql[3];
  vn_r = areax * qr[1] + areay * qr[2] + areaz * qr[3];

  tmp0 = vn_l * ql[0];
  tmp1 = vn_r * qr[0];
  flux[0] = tmp0 + tmp1;
  flux[1] = tmp0 * ql[1] + areax * ql[4] + tmp1 * qr[1] + areax * qr[4];
  flux[2] = tmp0 * ql[2] + areay * ql[4] + tmp1 * qr[2] + areay * qr[4];
  flux[3] = tmp0 * ql[3] + areaz * ql[4] + tmp1 * qr[3] + areaz * qr[4];
  flux[4] = ht_l * vn_l + ht_r * vn_r;

  tmp0 = sqrt(qr[0] / ql[0]);
  tmp1 = 1.0 / (1.0 + tmp0);
  rho_a = sqrt(qr[0] * ql[0]);
  u_a = (ql[1] + qr[1] * tmp0) * tmp1;
  v_a = (ql[2] + qr[2] * tmp0) * tmp1;
  w_a = (ql[3] + qr[3] * tmp0) * tmp1;
  vn_a = u_a * areax + v_a * areay + w_a * areaz;
  h_a = (ht_l / ql[0] + ht_r / qr[0] * tmp0) * tmp1;

  q2 = 0.5 * (u_a * u_a + v_a * v_a + w_a * w_a);
  c2_a = gamm1 * (h_a - q2);
  c2_a = fabs(c2_a);
  c_a = sqrt(c2_a);

  eigv1 = fabs(vn_a);
  eigv2 = fabs(vn_a + c_a);
  eigv3 = fabs(vn_a - c_a);

  epsa_r = alf_l;
  spectral = fabs(u_a) + fabs(v_a) + fabs(w_a) + c_a;
  epsaa = epsa_r * spectral;
  epsbb = 0.25 / smax(epsaa, MFO_TINY);
  epscc = 2.0 * epsaa;
  if (eigv1 < epscc) eigv1 = eigv1 * eigv1 * epsbb + epsaa;
  if (eigv2 < epscc) eigv2 = eigv2 * eigv2 * epsbb + epsaa;
  if (eigv3 < epscc) eigv3 = eigv3 * eigv3 * epsbb + epsaa;

  drho = qr[0] - ql[0];
  du = qr[1] - ql[1];
  dv = qr[2] - ql[2];
  dw = qr[3] - ql[3];
  dp = qr[4] - ql[4];
  dvn = vn_r - vn_l;

  dq2 = u_a * du + v_a * dv + w_a * dw;

  tmp0 = dp / c2_a;
  tmp1 = rho_a * dvn / c_a;
  alpha1 = (drho - tmp0) * eigv1;
  alpha2 = 0.5 * (tmp0 + tmp1) * eigv2;
  alpha3 = 0.5 * (tmp0 - tmp1) * eigv3;

  tmp0 = alpha1 + alpha2 + alpha3;
  tmp1 = eigv1 * rho_a;
  tmp2 = -tmp1 * dvn + (alpha2 - alpha3) * c_a;
  flux[0] -= tmp0;
  flux[1] -= tmp0 * u_a + tmp1 * du + tmp2 * areax;
  flux[2] -= tmp0 * v_a + tmp1 * dv + tmp2 * areay;
  flux[3] -= tmp0 * w_a + tmp1 * dw + tmp2 * areaz;
  flux[4] -= alpha1 * q2 + (alpha2 + alpha3) * h_a + tmp1 * dq2 + tmp2 * vn_a;

  tmp0 = 0.5 * area;
  for (int k = 0; k < 5; k++) flux[k] *= tmp0;
}

/* InviscidFlux (cal_flux.cpp:84-192): SetQlQrWithQ copies the cell states
 * (first order, :207-243), RoeFlux_noprec, then LoadFlux scatters in face
 * order (:1219-1255).  The SEG_LEN chunking does not change that order. */
void mfo_inviscid_flux(const mfo_grid *g, const mfo_params *p, mfo_state *s) {
  const int64_t n = nq(g);
  const int32_t C = g->n_cell;
  double ql[5], qr[5], f[5];
  for (int32_t face = 0; face < g->n_face; face++) {
    const int32_t c1 = g->f2c[2 * face], c2 = g->f2c[2 * face + 1];
    for (int k = 0; k < 5; k++) {
      ql[k] = s->q[k * n + c1];
      qr[k] = s->q[k * n + c2];
    }
    mfo_roe_flux(f, ql, qr, g->xfn[face], g->yfn[face], g->zfn[face], g->area[face], p->gam,
                 p->gamm1, p->p_bar, p->alf_l);
    for (int k = 0; k < 5; k++) s->res[(int64_t)k * C + c1] -= f[k];
    if (face >= g->n_bface)
      for (int k = 0; k < 5; k++) s->res[(int64_t)k * C + c2] += f[k];
  }
}

/* CellIsMG serial body (compute_timestep.cpp:1009-1340, :1315-1339). */
static void cell_is_mg(const mfo_grid *g, const mfo_params *p, const double *pr, int32_t *det) {
  const double stind = 0.1;
  for (int32_t i = 0; i < g->n_cell; i++) det[i] = 1;
  for (int32_t i = 0; i < g->n_bface; i++) {
    const int32_t c1 = g->f2c[i + i], c2 = g->f2c[i + i + 1];
    double dp = fabs(pr[c2] - pr[c1]) / (pr[c2] + pr[c1] + p->p_bar + p->p_bar);
    if (dp > stind) det[c1] = 0;
  }
  for (int32_t i = g->n_bface; i < g->n_face; i++) {
    const int32_t c1 = g->f2c[i + i], c2 = g->f2c[i + i + 1];
    double dp = fabs(pr[c2] - pr[c1]) / (pr[c2] + pr[c1] + p->p_bar + p->p_bar);
    if (dp > stind) {
      det[c1] = 0;
      det[c2] = 0;
    }
  }
}

/* ComputeTimeStep (compute_timestep.cpp:66-121) = TimeStepNormal_new serial
 * body (:756-824) + LimitTimeStep (:836-1000). */
void mfo_compute_timestep(const mfo_grid *g, const mfo_params *p, mfo_state *s) {
  const int64_t n = nq(g);
  const double *rho = s->q, *u = s->q + n, *v = s->q + 2 * n, *w = s->q + 3 * n,
               *pr = s->q + 4 * n;
  double *dt = s->dt;
  for (int32_t i = 0; i < g->n_cell; i++) dt[i] = MFO_BIG;
  for (int32_t i = 0; i < g->n_face; i++) {
    const int32_t c1 = g->f2c[i + i];
    double c2tmp = p->gam * (pr[c1] + p->p_bar) / rho[c1];
    double dn = fabs((g->xfc[i] - g->xcc[c1]) * g->xfn[i] + (g->yfc[i] - g->ycc[c1]) * g->yfn[i] +
                     (g->zfc[i] - g->zcc[c1]) * g->zfn[i]);
    double vn = u[c1] * g->xfn[i] + v[c1] * g->yfn[i] + w[c1] * g->zfn[i];
    vn = fabs(vn);
    double eigv = vn + sqrt(c2tmp);
    dt[c1] = smin(dt[c1], dn / eigv);
    if (i < g->n_bface) continue;
    const int32_t c2 = g->f2c[i + i + 1];
    c2tmp = p->gam * (pr[c2] + p->p_bar) / rho[c2];
    dn = fabs((g->xfc[i] - g->xcc[c2]) * g->xfn[i] + (g->yfc[i] - g->ycc[c2]) * g->yfn[i] +
              (g->zfc[i] - g->zcc[c2]) * g->zfn[i]);
    vn = u[c2] * g->xfn[i] + v[c2] * g->yfn[i] + w[c2] * g->zfn[i];
    vn = fabs(vn);
    eigv = vn + sqrt(c2tmp);
    dt[c2] = smin(dt[c2], dn / eigv);
  }

  /* LimitTimeStep */
  double cfl, cfl_tmp;
  if (s->iter_done > p->cfl_nstep)
    cfl = p->cfl_end;
  else
    cfl = p->cfl_start * pow(p->cfl_ratio, (double)s->iter_done / p->cfl_nstep);
  int32_t *det = (int32_t *)malloc(sizeof(int32_t) * (size_t)g->n_cell);
  cell_is_mg(g, p, pr, det);
  s->cfl_min = 0.5 * cfl;
  const double cfl_min = s->cfl_min;
  for (int32_t i = 0; i < g->n_cell; i++) {
    if (pr[i] > p->p_break)
      cfl_tmp = cfl;
    else if (pr[i] < p->p_min)
      cfl_tmp = cfl_min;
    else
      cfl_tmp = (pr[i] - p->p_min) / (p->p_break - p->p_min) * (cfl - cfl_min) + cfl_min;
    if (!det[i]) cfl_tmp = cfl_min;
    dt[i] *= cfl_tmp;
  }
  free(det);
  for (int32_t i = 0; i < g->n_cell; i++) {
    s->dt_max = smax(s->dt_max, dt[i]);
    s->dt_min = smin(s->dt_min, dt[i]);
  }
  double ratio_max = s->dt_max / s->dt_min;
  if (ratio_max > p->ratio_dtmax) {
    double dt_max_lim = p->ratio_dtmax * s->dt_min;
    for (int32_t i = 0; i < g->n_cell; i++)
      if (dt[i] > dt_max_lim) dt[i] = dt_max_lim;
  }
}

/* FluxLUSGS3D (forward_lusgs.cpp:1271-1324). */
void mfo_flux_lusgs(double flux[5], const double q[5], const double DQ[5], const double fa_n[3],
                    double gam, double p_bar, double lhs_omga) {
  double Q[5], rv2, v_n, p, peff, c2, eig, gam1 = gam - 1.;
  const double nx = fa_n[0], ny = fa_n[1], nz = fa_n[2];
  Q[0] = q[0];
  Q[1] = q[0] * q[1];
  Q[2] = q[0] * q[2];
  Q[3] = q[0] * q[3];
  rv2 = 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  p = q[4];
  Q[4] = p / gam1 + rv2;

  v_n = q[1] * nx + q[2] * ny + q[3] * nz;
  c2 = gam * (p + p_bar) / q[0];
  eig = fabs(v_n) + sqrt(c2);
  eig *= lhs_omga;

  peff = gam * p_bar / gam1;
  flux[1] = -Q[1] * v_n - p * nx;
  flux[2] = -Q[2] * v_n - p * ny;
  flux[3] = -Q[3] * v_n - p * nz;
  flux[4] = -(Q[4] + p + peff) * v_n;

  for (int i = 0; i < 5; i++) Q[i] += DQ[i];
  rv2 = 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0];
  p = gam1 * (Q[4] - rv2);

  flux[0] = DQ[1] * nx + DQ[2] * ny + DQ[3] * nz;
  v_n *= q[0];
  v_n += flux[0];
  v_n /= Q[0];
  flux[1] += Q[1] * v_n + p * nx;
  flux[2] += Q[2] * v_n + p * ny;
  flux[3] += Q[3] * v_n + p * nz;
  flux[4] += (Q[4] + p + peff) * v_n;

  for (int i = 0; i < 5; i++) flux[i] -= eig * DQ[i];
}

/* The DQ_limit == 2 positivity limiter (forward_lusgs.cpp:939-973 and
 * :1184-1218): two x0.1 stages, then zero. */
static void dq_limit(const mfo_params *p, const double *q, int64_t n, int32_t cell, double *DQ) {
  const double q0 = q[cell], q1 = q[n + cell], q2 = q[2 * n + cell], q3 = q[3 * n + cell],
               q4 = q[4 * n + cell];
  double *d0 = &DQ[cell], *d1 = &DQ[n + cell], *d2 = &DQ[2 * n + cell], *d3 = &DQ[3 * n + cell],
         *d4 = &DQ[4 * n + cell];
  double dp, vv;
  vv = q1 * q1 + q2 * q2 + q3 * q3;
  for (int stage = 0; stage < 3; stage++) {
    dp = *d4 + 0.5 * *d0 * vv - (*d1 * q1 + *d2 * q2 + *d3 * q3);
    dp *= p->gamm1;
    if ((q0 + *d0) < p->rho_min || (q0 + *d0) > p->rho_max || (q4 + dp) < p->p_min ||
        (q4 + dp) > p->p_max) {
      if (stage < 2) {
        *d0 *= 0.1; *d1 *= 0.1; *d2 *= 0.1; *d3 *= 0.1; *d4 *= 0.1;
      } else {
        *d0 = 0.0; *d1 = 0.0; *d2 = 0.0; *d3 = 0.0; *d4 = 0.0;
      }
    }
  }
}

/* CalnFPC + CalC2F (grid_polyhedra_auxiliary_functions.cpp:1293-1392):
 * faces of each cell in ascending face order. */
static void build_c2f(const mfo_grid *g, int32_t **ptr_out, int32_t **c2f_out) {
  const int32_t C = g->n_cell;
  int32_t *ptr = (int32_t *)calloc((size_t)C + 1, sizeof(int32_t));
  for (int32_t i = 0; i < g->n_face; i++) {
    ptr[g->f2c[2 * i] + 1]++;
    if (i >= g->n_bface) ptr[g->f2c[2 * i + 1] + 1]++;
  }
  for (int32_t i = 0; i < C; i++) ptr[i + 1] += ptr[i];
  int32_t *fill = (int32_t *)malloc(sizeof(int32_t) * (size_t)C);
  memcpy(fill, ptr, sizeof(int32_t) * (size_t)C);
  int32_t *c2f = (int32_t *)malloc(sizeof(int32_t) * (size_t)ptr[C]);
  for (int32_t i = 0; i < g->n_face; i++) {
    c2f[fill[g->f2c[2 * i]]++] = i;
    if (i >= g->n_bface) c2f[fill[g->f2c[2 * i + 1]]++] = i;
  }
  free(fill);
  *ptr_out = ptr;
  *c2f_out = c2f;
}

/* ForwardLUSGS (forward_lusgs.cpp:67-162) with CalDiagLUSGS (:554-595),
 * SolveLUSGS3D (:710-1255) and UpdateFlowField3D_CFL3d (:1335-1488).  The
 * serial build's LU-SGS order is the identity (ReorderCellforLUSGS_0,
 * grid_polyhedra.cpp:1127-1142), so layer[i] == i. */
void mfo_forward_lusgs(const mfo_grid *g, const mfo_params *p, mfo_state *s) {
  const int64_t n = nq(g);
  const int32_t C = g->n_cell;
  const double *q = s->q;
  const double *rho = q, *u = q + n, *v = q + 2 * n, *w = q + 3 * n, *pr = q + 4 * n;
  double *Diag = s->diag;
  double *DQ = s->dq;
  int32_t *ptr, *c2f;
  build_c2f(g, &ptr, &c2f);

  for (int32_t i = 0; i < C; i++) Diag[i] = g->vol[i] / s->dt[i];
  for (int32_t i = 0; i < g->n_face; i++) {
    const int32_t c1 = g->f2c[2 * i];
    double vn_1 = u[c1] * g->xfn[i] + v[c1] * g->yfn[i] + w[c1] * g->zfn[i];
    vn_1 = fabs(vn_1);
    double ss_1 = p->gam * (pr[c1] + p->p_bar) / rho[c1];
    double eig = vn_1 + sqrt(ss_1);
    Diag[c1] += 0.5 * g->area[i] * eig * p->lhs_omga;
    if (i < g->n_bface) continue;
    const int32_t c2 = g->f2c[2 * i + 1];
    double vn_2 = u[c2] * g->xfn[i] + v[c2] * g->yfn[i] + w[c2] * g->zfn[i];
    vn_2 = fabs(vn_2);
    double ss_2 = p->gam * (pr[c2] + p->p_bar) / rho[c2];
    eig = vn_2 + sqrt(ss_2);
    Diag[c2] += 0.5 * g->area[i] * eig * p->lhs_omga;
  }

  for (int64_t j = 0; j < 5 * n; j++) DQ[j] = 0.;
  for (int k = 0; k < 5; k++)
    for (int32_t j = 0; j < C; j++) DQ[k * n + j] = s->res[(int64_t)k * C + j];

  double flux[5], q_loc[5], DQ_loc[5], face_n[3];
  /* forward sweep */
  for (int k = 0; k < 5; k++) DQ[k * n + 0] /= Diag[0];
  for (int32_t cell = 1; cell < C; cell++) {
    for (int32_t j = ptr[cell]; j < ptr[cell + 1]; j++) {
      const int32_t face = c2f[j];
      int32_t c1 = g->f2c[2 * face], c2 = g->f2c[2 * face + 1];
      if (c1 > cell || c2 > cell) continue;
      face_n[0] = g->xfn[face];
      face_n[1] = g->yfn[face];
      face_n[2] = g->zfn[face];
      if (c2 == cell) {
        c2 = c1;
        c1 = cell;
        face_n[0] = -face_n[0];
        face_n[1] = -face_n[1];
        face_n[2] = -face_n[2];
      }
      for (int i = 0; i < 5; i++) {
        q_loc[i] = q[i * n + c2];
        DQ_loc[i] = DQ[i * n + c2];
      }
      mfo_flux_lusgs(flux, q_loc, DQ_loc, face_n, p->gam, p->p_bar, p->lhs_omga);
      const double tmp = 0.5 * g->area[face];
      for (int i = 0; i < 5; i++) DQ[i * n + cell] -= tmp * flux[i];
    }
    for (int i = 0; i < 5; i++) DQ[i * n + cell] /= Diag[cell];
    dq_limit(p, q, n, cell, DQ);
  }
  /* backward sweep */
  for (int32_t cell = C - 1; cell >= 0; cell--) {
    double flux_s[5] = {0., 0., 0., 0., 0.};
    for (int32_t j = ptr[cell]; j < ptr[cell + 1]; j++) {
      const int32_t face = c2f[j];
      int32_t c1 = g->f2c[2 * face], c2 = g->f2c[2 * face + 1];
      if (c1 < cell || c2 < cell) continue;
      face_n[0] = g->xfn[face];
      face_n[1] = g->yfn[face];
      face_n[2] = g->zfn[face];
      if (c2 == cell) {
        c2 = c1;
        c1 = cell;
        face_n[0] = -face_n[0];
        face_n[1] = -face_n[1];
        face_n[2] = -face_n[2];
      }
      for (int i = 0; i < 5; i++) {
        q_loc[i] = q[i * n + c2];
        DQ_loc[i] = DQ[i * n + c2];
      }
      mfo_flux_lusgs(flux, q_loc, DQ_loc, face_n, p->gam, p->p_bar, p->lhs_omga);
      const double tmp = g->area[face];
      for (int i = 0; i < 5; i++) flux_s[i] += tmp * flux[i];
    }
    const double tmp = 2.0 * Diag[cell];
    for (int i = 0; i < 5; i++) DQ[i * n + cell] -= flux_s[i] / tmp;
    dq_limit(p, q, n, cell, DQ);
  }
  free(ptr);
  free(c2f);

  mfo_update_flow(p, C, n, s->q, DQ);
}

/* UpdateFlowField3D_CFL3d (forward_lusgs.cpp:1335-1488): the conservative
 * update of the C cells of q [5][n] by DQ [5][n], with the density and
 * pressure relaxation and the clamps; ghosts untouched. */
void mfo_update_flow(const mfo_params *p, int32_t C, int64_t n, double *q,
                     const double *DQ) {
  double *qr = q, *qu = q + n, *qv = q + 2 * n, *qw = q + 3 * n, *qp = q + 4 * n;
  const double gam1 = p->gam - 1.;
  const double p00 = p->p_bar;
  const double alpq = -0.2, phiq = 1. / 0.5;
  const double betq = 1.0 + alpq * phiq;
  for (int32_t i = 0; i < C; i++) {
    double rhot, rhotr, ru, rv, rw, re, rho_del, p_del, rho_rat, p_rat, ptmp;
    rhot = qr[i];
    ru = rhot * qu[i];
    rv = rhot * qv[i];
    rw = rhot * qw[i];
    re = qp[i] / gam1 + 0.5 * rhot * (qu[i] * qu[i] + qv[i] * qv[i] + qw[i] * qw[i]);
    rhot += DQ[i];
    ru += DQ[n + i];
    rv += DQ[2 * n + i];
    rw += DQ[3 * n + i];
    re += DQ[4 * n + i];
    rhotr = 1. / (rhot + MFO_TINY);
    qu[i] = ru * rhotr;
    qv[i] = rv * rhotr;
    qw[i] = rw * rhotr;
    rho_del = DQ[i];
    rho_rat = rho_del / qr[i];
    if (rho_rat < alpq) rho_del /= betq + fabs(rho_rat) * phiq;
    qr[i] += rho_del;
    qr[i] = smax(qr[i], p->rho_min);
    qr[i] = smin(qr[i], p->rho_max);
    ptmp = gam1 * (re - 0.5 * (qu[i] * qu[i] + qv[i] * qv[i] + qw[i] * qw[i]) * qr[i]);
    p_del = ptmp - qp[i];
    p_rat = p_del / (qp[i] + p00);
    if (p_rat < alpq) p_del /= betq + fabs(p_rat) * phiq;
    qp[i] += p_del;
    qp[i] = smax(qp[i], p->p_min);
    qp[i] = smin(qp[i], p->p_max);
  }
}

/* CompNodeVar3D_dist serial path (cal_gradient.cpp:1922-2372). */
static void node_values(const mfo_grid *g, const double *qv, int name, double *q_n, double *u_n,
                        double *v_n, double *w_n, const double *u, const double *v,
                        const double *w, const int32_t *fptr) {
  const int32_t N = g->n_node, G = g->n_bface;
  double *facu = NULL, *facv = NULL, *facw = NULL;
  if (name == 1) {
    for (int32_t i = 0; i < N; i++) u_n[i] = v_n[i] = w_n[i] = 0.0;
    facu = (double *)malloc(sizeof(double) * (size_t)(G ? G : 1));
    facv = (double *)malloc(sizeof(double) * (size_t)(G ? G : 1));
    facw = (double *)malloc(sizeof(double) * (size_t)(G ? G : 1));
  }
  for (int32_t i = 0; i < N; i++) q_n[i] = 0.0;
  double *facq = (double *)malloc(sizeof(double) * (size_t)(G ? G : 1));
  for (int32_t i = 0; i < G; i++) {
    facq[i] = 0.0;
    const int type = g->bctype[i];
    if (type == MFO_INTERFACE || type == MFO_SYMM) continue;
    const int32_t c1 = g->f2c[2 * i], c2 = g->f2c[2 * i + 1];
    facq[i] = qv[c1] + qv[c2];
    facq[i] *= 0.5;
    if (name == 1) {
      facu[i] = u[c1] + u[c2];
      facu[i] *= 0.5;
      facv[i] = v[c1] + v[c2];
      facv[i] *= 0.5;
      facw[i] = w[c1] + w[c2];
      facw[i] *= 0.5;
    }
  }
  /* three passes over boundary faces: WALL, FAR_FIELD, then the other types */
  for (int pass = 0; pass < 3; pass++) {
    for (int32_t i = 0; i < G; i++) {
      const int type = g->bctype[i];
      if (pass == 0 && type != MFO_WALL) continue;
      if (pass == 1 && type != MFO_FAR_FIELD) continue;
      if (pass == 2 && (type == MFO_WALL || type == MFO_SYMM || type == MFO_FAR_FIELD ||
                        type == MFO_INTERFACE))
        continue;
      for (int32_t j = 0; j < g->nnpf[i]; j++) {
        const int32_t p1 = g->f2n[fptr[i] + j];
        if (pass == 1 && g->nmark[p1] == MFO_WALL) continue;
        if (pass == 2 && (g->nmark[p1] == MFO_WALL || g->nmark[p1] == MFO_FAR_FIELD)) continue;
        const double wr = g->wbface[fptr[i] + j];
        q_n[p1] += facq[i] * wr;
        if (name == 1 && g->nodesymm[p1] == 1) {
          u_n[p1] += facu[i] * wr;
          v_n[p1] += facv[i] * wr;
          w_n[p1] += facw[i] * wr;
        }
      }
    }
  }
  int64_t k = 0;
  for (int32_t i = 0; i < g->n_cell; i++) {
    for (int32_t j = 0; j < g->nnpc[i]; j++, k++) {
      const int32_t p1 = g->c2n[k];
      if (g->nmark[p1] != 0) continue;
      q_n[p1] += qv[i] * g->wc2n[k];
      if (name == 1 && g->nodesymm[p1] == 1) {
        u_n[p1] += u[i] * g->wc2n[k];
        v_n[p1] += v[i] * g->wc2n[k];
        w_n[p1] += w[i] * g->wc2n[k];
      }
    }
  }
  for (int32_t i = 0; i < N; i++) {
    q_n[i] /= (g->wnode[i] + MFO_TINY);
    if (name == 1 && g->nodesymm[i] == 1) {
      u_n[i] /= (g->wnode[i] + MFO_TINY);
      v_n[i] /= (g->wnode[i] + MFO_TINY);
      w_n[i] /= (g->wnode[i] + MFO_TINY);
    }
  }
  if (name > 0 && name < 4) {
    for (int32_t i = 0; i < N; i++) {
      if (g->nodesymm[i] != 1) continue;
      double vn = u_n[i] * g->xfn_n_symm[i] + v_n[i] * g->yfn_n_symm[i] + w_n[i] * g->zfn_n_symm[i];
      if (name == 1)
        q_n[i] = u_n[i] - vn * g->xfn_n_symm[i];
      else if (name == 2)
        q_n[i] = v_n[i] - vn * g->yfn_n_symm[i];
      else
        q_n[i] = w_n[i] - vn * g->zfn_n_symm[i];
    }
  }
  free(facq);
  free(facu);
  free(facv);
  free(facw);
}

/* CalculateGradient (cal_gradient.cpp:87-167) -> CompGradientQ_Gauss_Node
 * serial face loops (:1740-1897) for each of rho, u, v, w, p. */
void mfo_calculate_gradient(const mfo_grid *g, const mfo_params *p, mfo_state *s) {
  (void)p;
  const int64_t n = nq(g);
  const int32_t N = g->n_node;
  for (int64_t i = 0; i < 5 * n; i++) s->dqdx[i] = s->dqdy[i] = s->dqdz[i] = 0.;
  int32_t *fptr = (int32_t *)malloc(sizeof(int32_t) * ((size_t)g->n_face + 1));
  fptr[0] = 0;
  for (int32_t i = 0; i < g->n_face; i++) fptr[i + 1] = fptr[i] + g->nnpf[i];
  double *u_n = (double *)malloc(sizeof(double) * (size_t)N);
  double *v_n = (double *)malloc(sizeof(double) * (size_t)N);
  double *w_n = (double *)malloc(sizeof(double) * (size_t)N);
  double *q_n = (double *)malloc(sizeof(double) * (size_t)N);
  const double *u = s->q + n, *v = s->q + 2 * n, *w = s->q + 3 * n;
  for (int name = 0; name < 5; name++) {
    const double *qv = s->q + name * n;
    double *dqdx = s->dqdx + name * n, *dqdy = s->dqdy + name * n, *dqdz = s->dqdz + name * n;
    node_values(g, qv, name, q_n, u_n, v_n, w_n, u, v, w, fptr);
    for (int32_t i = 0; i < g->n_bface; i++) {
      const int32_t c1 = g->f2c[2 * i], c2 = g->f2c[2 * i + 1];
      const int type = g->bctype[i];
      double qsum = 0.0;
      if (type == MFO_INTERFACE || type == MFO_SYMM) {
        for (int32_t j = 0; j < g->nnpf[i]; j++) qsum += q_n[g->f2n[fptr[i] + j]];
        qsum /= (double)g->nnpf[i];
      } else {
        qsum = 0.5 * (qv[c1] + qv[c2]);
      }
      qsum *= g->area[i];
      dqdx[c1] += qsum * g->xfn[i];
      dqdy[c1] += qsum * g->yfn[i];
      dqdz[c1] += qsum * g->zfn[i];
    }
    for (int32_t i = g->n_bface; i < g->n_face; i++) {
      const int32_t c1 = g->f2c[2 * i], c2 = g->f2c[2 * i + 1];
      double qsum = 0.0;
      for (int32_t j = 0; j < g->nnpf[i]; j++) qsum += q_n[g->f2n[fptr[i] + j]];
      qsum /= (double)g->nnpf[i];
      qsum *= g->area[i];
      const double tmpx = qsum * g->xfn[i], tmpy = qsum * g->yfn[i], tmpz = qsum * g->zfn[i];
      dqdx[c1] += tmpx;
      dqdy[c1] += tmpy;
      dqdz[c1] += tmpz;
      dqdx[c2] -= tmpx;
      dqdy[c2] -= tmpy;
      dqdz[c2] -= tmpz;
    }
    for (int32_t i = 0; i < g->n_cell; i++) {
      dqdx[i] /= g->vol[i];
      dqdy[i] /= g->vol[i];
      dqdz[i] /= g->vol[i];
    }
  }
  free(fptr);
  free(u_n);
  free(v_n);
  free(w_n);
  free(q_n);
}

/* main.cpp:294-317 */
void mfo_residual_norm(const mfo_grid *g, const mfo_state *s, double out[5]) {
  const int32_t C = g->n_cell;
  for (int j = 0; j < 5; j++) {
    double acc = 0.;
    for (int32_t i = 0; i < C; i++) acc += s->res[(int64_t)j * C + i] * s->res[(int64_t)j * C + i];
    out[j] = sqrt(acc);
  }
}

/* main.cpp:201-291 */
void mfo_iterate(const mfo_grid *g, const mfo_params *p, mfo_state *s, int32_t n, double *norms) {
  for (int32_t it = 0; it < n; it++) {
    mfo_zero_residuals(g, s);
    mfo_inviscid_flux(g, p, s);
    mfo_compute_timestep(g, p, s);
    mfo_forward_lusgs(g, p, s);
    mfo_calculate_gradient(g, p, s);
    s->iter_done++;
    if (norms) mfo_residual_norm(g, s, norms + 5 * (int64_t)it);
  }
}
