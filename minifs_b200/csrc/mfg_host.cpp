// Host-side setup for the mfgpu hot path: solver parameters and the mesh
// preprocessing the reference performs once before its iteration loop.
//
// Every routine keeps the reference's loop order and floating-point
// expression order, because the iteration path is checked bit-for-bit and it
// consumes these values.  Compiled with -ffp-contract=off (no fused
// multiply-add), the rounding of the reference's x86-64 g++ -O3 build.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mfgpu.h"

namespace {

const double kTiny = 1.e-40;  // number_type.h:29
const double kBig = 1.e40;    // number_type.h:28
const double kPi = 3.14159265358979323846;  // constant.h:23

inline double smin(double a, double b) { return (b < a) ? b : a; }  // std::min
inline double smax(double a, double b) { return (a < b) ? b : a; }  // std::max

}  // namespace

extern "C" void mfg_params_default(mfg_params *p) {
  std::memset(p, 0, sizeof(*p));
  // para_field_global.cpp:37-130
  p->cfl_start = 100.0;
  p->cfl_end = 100.0;
  p->cfl_nstep = 2000;
  p->re = 1.8140449177e7;
  p->T = 288.15;
  p->mach = 0.8395;
  p->alpha = 3.06;
  p->beita = 0.0;
  p->epsa_r = 0.1;
  p->lhs_omga = 1.0;
  p->ratio_dtmax = 1.0e80;
  p->gam = 1.4;
  p->gascon = 287.053;
  mfg_params_derive(p);
}

// para_field_global.cpp:150-209 (tref, sref, amuref and the ratio_* factors
// are the reference's fixed intermediate constants).
extern "C" int mfg_params_derive(mfg_params *p) {
  if (!p) return MFG_ERR_INVALID;
  const double tref = 288.15, sref = 110.4, amuref = 1.78938e-5;
  const double ratio_rhop_max = 10.0, ratio_rhop_min = 1.0e-4, ratio_p_break = 0.01;
  // volatile keeps the compiler from folding libm calls at compile time when
  // the inputs happen to be constants: the values must be glibc's.
  volatile double T = p->T, gam = p->gam, gascon = p->gascon, mach = p->mach;
  volatile double alpha = p->alpha, beita = p->beita, re = p->re;
  const double trat = (T / tref);
  p->amu = amuref * trat * sqrt(trat) * (tref + sref) / (T + sref);
  p->ainf = sqrt(gam * gascon * T);
  p->uqq = p->ainf * mach;
  const double alpha_t = (alpha * kPi / 180.);
  const double beita_t = (beita * kPi / 180.);
  p->u_s = p->uqq * cos(alpha_t) * cos(-1. * beita_t);
  p->v_s = p->uqq * sin(-1. * beita_t);
  p->w_s = p->uqq * sin(alpha_t) * cos(-1. * beita_t);
  p->p_s = 0.00;
  p->rho_s = re * p->amu / p->uqq;
  p->p_bar = p->rho_s * gascon * T;
  p->gamm1 = gam - 1.0;
  const double temp = 1.0 + 0.5 * p->gamm1 * mach * mach;
  const double p_stag_t = pow(temp, gam / p->gamm1);
  const double rho_stag = pow(temp, 1.0 / p->gamm1) * p->rho_s;
  p->p_stag = (p_stag_t - 1.0) * p->p_bar;
  p->e_stag = p->p_bar / p->gamm1 +
              0.5 * p->rho_s * (p->u_s * p->u_s + p->v_s * p->v_s + p->w_s * p->w_s);
  p->p_min = ratio_rhop_min * p->p_bar - p->p_bar;
  p->p_max = ratio_rhop_max * (p->p_stag + p->p_bar) - p->p_bar;
  p->rho_min = ratio_rhop_min * p->rho_s;
  p->rho_max = ratio_rhop_max * rho_stag;
  p->p_break = ratio_p_break * p->p_bar - p->p_bar;
  p->e_stag_max = 1.0e5 * p->e_stag;
  p->cfl_min = 0.5 * p->cfl_start;
  p->cfl_ratio = p->cfl_end / p->cfl_start;
  p->alf_l = p->epsa_r;
  return MFG_OK;
}

// SpecifyBC (load_grid.cpp:804-902), serial case (no interface patches).
extern "C" int mfg_prep_specify_bc(mfg_raw_grid *g, int32_t n_patch, const int32_t *patch_types,
                                   int32_t *bctype) {
  if (!g || !g->f2c || (!patch_types && n_patch > 0) || !bctype) return MFG_ERR_INVALID;
  for (int32_t k = 0; k < g->n_bface; k++) {
    const int32_t c2 = -g->f2c[k * 2 + 1];
    if (c2 < 1 || c2 > n_patch) return MFG_ERR_BADMESH;
    bctype[k] = patch_types[c2 - 1];
    g->f2c[k * 2 + 1] = k + g->n_cell;
  }
  return MFG_OK;
}

namespace {

// FaceCellCenterbyAverage (grid_polyhedra_auxiliary_functions.cpp:271-351).
void face_cell_center_by_average(const mfg_raw_grid *g, double *xfc, double *yfc, double *zfc,
                                 double *xcc, double *ycc, double *zcc) {
  const int32_t nF = g->n_face, nB = g->n_bface, nC = g->n_cell;
  int64_t node = 0;
  for (int32_t i = 0; i < nF; i++) {
    xfc[i] = 0.0;
    yfc[i] = 0.0;
    zfc[i] = 0.0;
    for (int32_t j = 0; j < g->nnpf[i]; j++) {
      const int32_t p1 = g->f2n[node++];
      xfc[i] += g->x[p1];
      yfc[i] += g->y[p1];
      zfc[i] += g->z[p1];
    }
    xfc[i] /= g->nnpf[i];
    yfc[i] /= g->nnpf[i];
    zfc[i] /= g->nnpf[i];
  }
  for (int32_t i = 0; i < nC; i++) xcc[i] = ycc[i] = zcc[i] = 0.0;
  std::vector<int32_t> nface(nC, 0);
  for (int32_t i = 0; i < nB; i++) {
    const int32_t c1 = g->f2c[2 * i];
    xcc[c1] += xfc[i];
    ycc[c1] += yfc[i];
    zcc[c1] += zfc[i];
    nface[c1]++;
  }
  for (int32_t i = nB; i < nF; i++) {
    const int32_t c1 = g->f2c[2 * i], c2 = g->f2c[2 * i + 1];
    xcc[c1] += xfc[i];
    ycc[c1] += yfc[i];
    zcc[c1] += zfc[i];
    xcc[c2] += xfc[i];
    ycc[c2] += yfc[i];
    zcc[c2] += zfc[i];
    nface[c1]++;
    nface[c2]++;
  }
  for (int32_t i = 0; i < nC; i++) {
    xcc[i] /= nface[i];
    ycc[i] /= nface[i];
    zcc[i] /= nface[i];
  }
}

// FaceAreaNormalCentroid_cycle (:68-265): four centroid refinements, then
// normals and areas from the triangle fan about the refined centroid.
void face_area_normal_centroid(const mfg_raw_grid *g, double *area, double *xfn, double *yfn,
                               double *zfn, double *xfc, double *yfc, double *zfc,
                               const double *xcc, const double *ycc, const double *zcc) {
  const int32_t nF = g->n_face;
  const double *x = g->x, *y = g->y, *z = g->z;
  std::vector<double> xfct(nF), yfct(nF), zfct(nF);
  for (int k = 0; k <= 4; k++) {
    const bool last = (k == 4);
    int64_t count = 0;
    for (int32_t i = 0; i < nF; i++) {
      if (last) {
        xfn[i] = 0.0;
        yfn[i] = 0.0;
        zfn[i] = 0.0;
      }
      area[i] = 0.0;
      xfct[i] = 0.0;
      yfct[i] = 0.0;
      zfct[i] = 0.0;
      const int32_t p1 = g->f2n[count];
      for (int32_t j = 0; j < g->nnpf[i]; j++) {
        const int32_t p2 = g->f2n[count++];
        const int32_t p3 = (j == g->nnpf[i] - 1) ? p1 : g->f2n[count];
        const double x21 = x[p2] - xfc[i], y21 = y[p2] - yfc[i], z21 = z[p2] - zfc[i];
        const double x31 = x[p3] - xfc[i], y31 = y[p3] - yfc[i], z31 = z[p3] - zfc[i];
        const double xn = y21 * z31 - y31 * z21;
        const double yn = z21 * x31 - z31 * x21;
        const double zn = x21 * y31 - x31 * y21;
        const double art = sqrt(xn * xn + yn * yn + zn * zn);
        const double xt = x[p2] + x[p3] + xfc[i];
        const double yt = y[p2] + y[p3] + yfc[i];
        const double zt = z[p2] + z[p3] + zfc[i];
        area[i] += art;
        xfct[i] += art * xt;
        yfct[i] += art * yt;
        zfct[i] += art * zt;
        if (last) {
          xfn[i] += xn;
          yfn[i] += yn;
          zfn[i] += zn;
        }
      }
      if (!last) {
        if (area[i] > kTiny) {
          const double art = 1.0 / area[i] / 3.0;
          xfct[i] *= art;
          yfct[i] *= art;
          zfct[i] *= art;
          xfc[i] = xfct[i];
          yfc[i] = yfct[i];
          zfc[i] = zfct[i];
        }
      } else {
        if (area[i] > kTiny) {
          const double art = 1.0 / area[i] / 3.0;
          xfc[i] = xfct[i] * art;
          yfc[i] = yfct[i] * art;
          zfc[i] = zfct[i] * art;
        }
        double art = sqrt(xfn[i] * xfn[i] + yfn[i] * yfn[i] + zfn[i] * zfn[i]);
        area[i] = art * 0.5;
        if (art > kTiny) {
          xfn[i] /= art;
          yfn[i] /= art;
          zfn[i] /= art;
        } else {
          const int32_t c1 = g->f2c[i + i];
          const double xn = xfc[i] - xcc[c1], yn = yfc[i] - ycc[c1], zn = zfc[i] - zcc[c1];
          art = sqrt(xn * xn + yn * yn + zn * zn);
          xfn[i] = xn / art;
          yfn[i] = yn / art;
          zfn[i] = zn / art;
        }
      }
    }
  }
}

// CellVolCentroid (:357-613).  Returns false on a volume below TINY (the
// reference prints and exits, :528-536).
bool cell_vol_centroid(const mfg_raw_grid *g, double *vol, double *xcc, double *ycc, double *zcc,
                       const double *xfc, const double *yfc, const double *zfc,
                       const double *xfn, const double *yfn, const double *zfn,
                       const double *area) {
  const int32_t nF = g->n_face, nB = g->n_bface, nC = g->n_cell;
  const double *x = g->x, *y = g->y, *z = g->z;
  std::vector<double> xcct(nC, 0.0), ycct(nC, 0.0), zcct(nC, 0.0);
  for (int32_t i = 0; i < nC; i++) vol[i] = 0.0;
  int64_t node = 0;
  for (int32_t i = 0; i < nF; i++) {
    const bool interior = i >= nB;
    const int32_t c1 = g->f2c[2 * i];
    const int32_t c2 = interior ? g->f2c[2 * i + 1] : -1;
    const int32_t p1 = g->f2n[node];
    for (int32_t j = 0; j < g->nnpf[i]; j++) {
      const int32_t p2 = g->f2n[node++];
      const int32_t p3 = (j == g->nnpf[i] - 1) ? p1 : g->f2n[node];
      const double x21 = x[p2] - xfc[i], y21 = y[p2] - yfc[i], z21 = z[p2] - zfc[i];
      const double x31 = x[p3] - xfc[i], y31 = y[p3] - yfc[i], z31 = z[p3] - zfc[i];
      const double nx = y21 * z31 - y31 * z21;
      const double ny = z21 * x31 - z31 * x21;
      const double nz = x21 * y31 - x31 * y21;
      {
        const double x41 = xcc[c1] - xfc[i], y41 = ycc[c1] - yfc[i], z41 = zcc[c1] - zfc[i];
        const double xt = x[p2] + x[p3] + xfc[i] + xcc[c1];
        const double yt = y[p2] + y[p3] + yfc[i] + ycc[c1];
        const double zt = z[p2] + z[p3] + zfc[i] + zcc[c1];
        double volt = nx * x41 + ny * y41 + nz * z41;
        volt = -volt;
        xcct[c1] += volt * xt;
        ycct[c1] += volt * yt;
        zcct[c1] += volt * zt;
        vol[c1] += volt;
      }
      if (interior) {
        const double x41 = xcc[c2] - xfc[i], y41 = ycc[c2] - yfc[i], z41 = zcc[c2] - zfc[i];
        const double xt = x[p2] + x[p3] + xfc[i] + xcc[c2];
        const double yt = y[p2] + y[p3] + yfc[i] + ycc[c2];
        const double zt = z[p2] + z[p3] + zfc[i] + zcc[c2];
        const double volt = nx * x41 + ny * y41 + nz * z41;
        xcct[c2] += volt * xt;
        ycct[c2] += volt * yt;
        zcct[c2] += volt * zt;
        vol[c2] += volt;
      }
    }
  }
  int32_t bad = 0;
  for (int32_t i = 0; i < nC; i++) {
    const double tmp = 1.0 / (4.0 * vol[i] + kTiny);
    xcct[i] *= tmp;
    ycct[i] *= tmp;
    zcct[i] *= tmp;
    vol[i] /= 6.0;
    if (vol[i] < kTiny) bad++;
  }
  if (bad > 0) return false;
  std::vector<int32_t> mark(nC, 1);
  for (int32_t i = 0; i < nB; i++) {
    const int32_t c1 = g->f2c[i + i];
    const double x21 = xcct[c1] - xfc[i], y21 = ycct[c1] - yfc[i], z21 = zcct[c1] - zfc[i];
    const double dot = x21 * xfn[i] + y21 * yfn[i] + z21 * zfn[i];
    if (dot > 0.0) mark[c1] = 0;
  }
  for (int32_t i = nB; i < nF; i++) {
    const int32_t c1 = g->f2c[i + i], c2 = g->f2c[i + i + 1];
    double x21 = xcct[c1] - xfc[i], y21 = ycct[c1] - yfc[i], z21 = zcct[c1] - zfc[i];
    double dot = x21 * xfn[i] + y21 * yfn[i] + z21 * zfn[i];
    if (dot > 0.0) mark[c1] = 0;
    x21 = xcct[c2] - xfc[i];
    y21 = ycct[c2] - yfc[i];
    z21 = zcct[c2] - zfc[i];
    dot = x21 * xfn[i] + y21 * yfn[i] + z21 * zfn[i];
    if (dot < 0.0) mark[c2] = 0;
  }
  for (int32_t i = 0; i < nC; i++) {
    if (mark[i] == 1) {
      xcc[i] = xcct[i];
      ycc[i] = ycct[i];
      zcc[i] = zcct[i];
    }
  }
  for (int32_t i = 0; i < nB; i++) {
    const int32_t c1 = g->f2c[2 * i];
    const int32_t c2 = i + nC;
    if (area[i] > kTiny) {
      const double tmp = 2. * ((xcc[c1] - xfc[i]) * xfn[i] + (ycc[c1] - yfc[i]) * yfn[i] +
                               (zcc[c1] - zfc[i]) * zfn[i]);
      xcc[c2] = xcc[c1] - xfn[i] * tmp;
      ycc[c2] = ycc[c1] - yfn[i] * tmp;
      zcc[c2] = zcc[c1] - zfn[i] * tmp;
    } else {
      xcc[c2] = -xcc[c1] + 2. * xfc[i];
      ycc[c2] = -ycc[c1] + 2. * yfc[i];
      zcc[c2] = -zcc[c1] + 2. * zfc[i];
    }
    vol[c2] = vol[c1];
  }
  return true;
}

// CorrectFaceNormal (:619-671): faces of (near) zero area.
void correct_face_normal(const mfg_raw_grid *g, double *xfn, double *yfn, double *zfn,
                         const double *xfc, const double *yfc, const double *zfc,
                         const double *xcc, const double *ycc, const double *zcc,
                         const double *area) {
  int64_t node = 0;
  for (int32_t i = 0; i < g->n_face; i++) {
    const int32_t p1 = g->f2n[node];
    node += g->nnpf[i];
    if (area[i] < kTiny) {
      const int32_t c1 = g->f2c[i + i];
      double x21 = xcc[c1] - xfc[i], y21 = ycc[c1] - yfc[i], z21 = zcc[c1] - zfc[i];
      const double x31 = g->x[p1] - xfc[i], y31 = g->y[p1] - yfc[i], z31 = g->z[p1] - zfc[i];
      const double dot = x21 * x31 + y21 * y31 + z21 * z31;
      double nn = x31 * x31 + y31 * y31 + z31 * z31;
      double ratio = 0.0;
      if (nn > kTiny) ratio = dot / nn;
      x21 -= ratio * x31;
      y21 -= ratio * y31;
      z21 -= ratio * z31;
      nn = sqrt(x21 * x21 + y21 * y21 + z21 * z21);
      xfn[i] = -x21 / nn;
      yfn[i] = -y21 / nn;
      zfn[i] = -z21 / nn;
    }
  }
}

inline double abs_max_sign_first(double a, double b) {  // AbsMaxSignFirst (:812-823)
  const int sign = (a > 0) ? 1 : -1;
  double c = smax(fabs(a), fabs(b));
  c *= sign;
  return c;
}

// CorrectCellCentroid (:679-807): nudge centroids closer than 1e-10 to a face.
void correct_cell_centroid(const mfg_raw_grid *g, double *xcc, double *ycc, double *zcc,
                           const double *xfc, const double *yfc, const double *zfc,
                           const double *xfn, const double *yfn, const double *zfn) {
  const int iexp = 16;
  volatile double ten = 10.0;
  const double scale = pow(ten, -iexp + 1);
  const double minDn = 1.0e-10;
  auto fix = [&](int32_t c, int32_t i) {
    const double x21 = xcc[c] - xfc[i], y21 = ycc[c] - yfc[i], z21 = zcc[c] - zfc[i];
    const double dot = x21 * xfn[i] + y21 * yfn[i] + z21 * zfn[i];
    if (fabs(dot) < minDn) {
      double dx = minDn * xfn[i], dy = minDn * yfn[i], dz = minDn * zfn[i];
      dx = abs_max_sign_first(dx, scale * xcc[c]);
      dy = abs_max_sign_first(dy, scale * ycc[c]);
      dz = abs_max_sign_first(dz, scale * zcc[c]);
      const int sign = (dot > 0.0) ? 1 : -1;
      xcc[c] += sign * dx;
      ycc[c] += sign * dy;
      zcc[c] += sign * dz;
    }
  };
  for (int32_t i = 0; i < g->n_bface; ++i) fix(g->f2c[i + i], i);
  for (int32_t i = g->n_bface; i < g->n_face; i++) {
    fix(g->f2c[i + i], i);
    fix(g->f2c[i + i + 1], i);
  }
}

}  // namespace

extern "C" int mfg_prep_metrics(const mfg_raw_grid *g, double *xfn, double *yfn, double *zfn,
                                double *area, double *xfc, double *yfc, double *zfc, double *xcc,
                                double *ycc, double *zcc, double *vol) {
  if (!g || !xfn || !yfn || !zfn || !area || !xfc || !yfc || !zfc || !xcc || !ycc || !zcc || !vol)
    return MFG_ERR_INVALID;
  face_cell_center_by_average(g, xfc, yfc, zfc, xcc, ycc, zcc);
  face_area_normal_centroid(g, area, xfn, yfn, zfn, xfc, yfc, zfc, xcc, ycc, zcc);
  if (!cell_vol_centroid(g, vol, xcc, ycc, zcc, xfc, yfc, zfc, xfn, yfn, zfn, area))
    return MFG_ERR_BADMESH;
  correct_face_normal(g, xfn, yfn, zfn, xfc, yfc, zfc, xcc, ycc, zcc, area);
  correct_cell_centroid(g, xcc, ycc, zcc, xfc, yfc, zfc, xfn, yfn, zfn);
  return MFG_OK;
}

extern "C" int mfg_prep_init_flow(const mfg_raw_grid *g, const mfg_params *p,
                                  const int32_t *bctype, const double *xfn, const double *yfn,
                                  const double *zfn, const double *xcc, const double *ycc,
                                  const double *zcc, double bump_amp, double bump_sigma,
                                  double bump_x0, double bump_y0, double bump_z0, double *q) {
  if (!g || !p || !bctype || !q) return MFG_ERR_INVALID;
  const int32_t nC = g->n_cell, nB = g->n_bface;
  const int64_t n = (int64_t)nC + nB;
  double *rho = q, *u = q + n, *v = q + 2 * n, *w = q + 3 * n, *pr = q + 4 * n;
  // AllocAndInitFlowfield (load_grid.cpp:571-601)
  for (int64_t i = 0; i < n; i++) {
    rho[i] = p->rho_s;
    u[i] = p->u_s;
    v[i] = p->v_s;
    w[i] = p->w_s;
    pr[i] = p->p_s;
  }
  if (bump_amp != 0.0) {
    for (int32_t i = 0; i < nC; i++) {
      const double dx = xcc[i] - bump_x0, dy = ycc[i] - bump_y0, dz = zcc[i] - bump_z0;
      const double r2 = dx * dx + dy * dy + dz * dz;
      rho[i] = p->rho_s * (1.0 + bump_amp * exp(-r2 / (2.0 * bump_sigma * bump_sigma)));
    }
  }
  // SetGhostVariables (load_grid.cpp:953-1212), inviscid steady case.
  const double gam = p->gam, p_bar = p->p_bar;
  const double rho00 = p->rho_s, u00 = p->u_s, v00 = p->v_s, w00 = p->w_s, p00 = p->p_s;
  const double norm_of_uvw = sqrt(u00 * u00 + v00 * v00 + w00 * w00);
  const double eps_of_farfield_vn = 0.0;
  for (int32_t i = 0; i < nB; i++) {
    const int type = bctype[i];
    const int32_t c1 = g->f2c[2 * i], c2 = g->f2c[2 * i + 1];
    if (type == MFG_BC_INTERFACE) continue;
    switch (type) {
      case MFG_BC_WALL:
      case MFG_BC_SYMM: {
        if (type == MFG_BC_WALL) {
          pr[c2] = pr[c1];
          rho[c2] = rho[c1];
        } else {
          rho[c2] = rho[c1];
          pr[c2] = pr[c1];
        }
        const double vn = 2. * (xfn[i] * u[c1] + yfn[i] * v[c1] + zfn[i] * w[c1]);
        u[c2] = u[c1] - vn * xfn[i];
        v[c2] = v[c1] - vn * yfn[i];
        w[c2] = w[c1] - vn * zfn[i];
        break;
      }
      case MFG_BC_FAR_FIELD: {
        const double um = u00, vm = v00, wm = w00;
        const double up = u[c1], vp = v[c1], wp = w[c1];
        const double rhom = rho00, pm = p00 + p_bar;
        const double rhop = rho[c1], pp = pr[c1] + p_bar;
        const double vnm = xfn[i] * um + yfn[i] * vm + zfn[i] * wm;
        const double vnp = xfn[i] * up + yfn[i] * vp + zfn[i] * wp;
        const double cm = sqrt(gam * pm / rhom);
        const double cp = sqrt(gam * pp / rhop);
        const double riemm = vnm - 2. * cm / (gam - 1.);
        const double riemp = vnp + 2. * cp / (gam - 1.);
        const double vnb = 0.5 * (riemp + riemm);
        const double cb = 0.25 * (riemp - riemm) * (gam - 1.);
        if (fabs(vnb / cb) > 1.) {
          if (vnb <= 0.0) {
            rho[c2] = rhom;
            u[c2] = um;
            v[c2] = vm;
            w[c2] = wm;
            pr[c2] = pm;
          } else {
            rho[c2] = rhop;
            u[c2] = up;
            v[c2] = vp;
            w[c2] = wp;
            pr[c2] = pp;
          }
        } else {
          const double rela_vnb = vnb / norm_of_uvw;
          if (rela_vnb <= -eps_of_farfield_vn) {
            const double vtx = um - vnm * xfn[i], vty = vm - vnm * yfn[i], vtz = wm - vnm * zfn[i];
            const double entr = pm / pow(rhom, gam);
            rho[c2] = pow((cb * cb / (entr * gam)), double(1. / (gam - 1.)));
            u[c2] = vtx + vnb * xfn[i];
            v[c2] = vty + vnb * yfn[i];
            w[c2] = vtz + vnb * zfn[i];
            pr[c2] = cb * cb * rho[c2] / gam;
          } else if (rela_vnb > eps_of_farfield_vn) {
            const double vtx = up - vnp * xfn[i], vty = vp - vnp * yfn[i], vtz = wp - vnp * zfn[i];
            const double entr = pp / pow(rhop, gam);
            rho[c2] = pow((cb * cb / (entr * gam)), double(1. / (gam - 1.)));
            u[c2] = vtx + vnb * xfn[i];
            v[c2] = vty + vnb * yfn[i];
            w[c2] = vtz + vnb * zfn[i];
            pr[c2] = cb * cb * rho[c2] / gam;
          } else {
            rho[c2] = 0.5 * (rhop + rhom);
            u[c2] = 0.5 * (up + um);
            v[c2] = 0.5 * (vp + vm);
            w[c2] = 0.5 * (wp + wm);
            pr[c2] = 0.5 * (pp + pm);
          }
        }
        rho[c2] = 2 * rho[c2] - rhop;
        u[c2] = 2 * u[c2] - up;
        v[c2] = 2 * v[c2] - vp;
        w[c2] = 2 * w[c2] - wp;
        pr[c2] = 2 * pr[c2] - pp;
        pr[c2] -= p_bar;
        break;
      }
      default:
        // The reference prints "Error in SetGhostVariables 001" and keeps the
        // freestream ghost state; the clamps below still apply.
        break;
    }
    rho[c2] = smax(rho[c2], p->rho_min);
    rho[c2] = smin(rho[c2], p->rho_max);
    pr[c2] = smax(pr[c2], p->p_min);
    pr[c2] = smin(pr[c2], p->p_max);
  }
  return MFG_OK;
}

namespace {

// Distinct nodes of each cell in order of first appearance over its faces
// (C2F order), the generic branch of CalC2N (:1438-1830).  Only the set of
// nodes of a cell matters downstream: each node receives one contribution
// per cell, in ascending cell order.
void build_c2n(const mfg_raw_grid *g, std::vector<int32_t> &ptr, std::vector<int32_t> &c2n) {
  const int32_t nC = g->n_cell, nF = g->n_face, nB = g->n_bface;
  std::vector<int64_t> fptr(nF + 1, 0);
  for (int32_t i = 0; i < nF; i++) fptr[i + 1] = fptr[i] + g->nnpf[i];
  std::vector<int32_t> cf_ptr(nC + 1, 0);
  for (int32_t i = 0; i < nF; i++) {
    cf_ptr[g->f2c[2 * i] + 1]++;
    if (i >= nB) cf_ptr[g->f2c[2 * i + 1] + 1]++;
  }
  for (int32_t i = 0; i < nC; i++) cf_ptr[i + 1] += cf_ptr[i];
  std::vector<int32_t> cf(cf_ptr[nC]), fill(cf_ptr.begin(), cf_ptr.end() - 1);
  for (int32_t i = 0; i < nF; i++) {
    cf[fill[g->f2c[2 * i]]++] = i;
    if (i >= nB) cf[fill[g->f2c[2 * i + 1]]++] = i;
  }
  ptr.assign(nC + 1, 0);
  c2n.clear();
  c2n.reserve((size_t)nC * 4);
  for (int32_t c = 0; c < nC; c++) {
    const size_t start = c2n.size();
    for (int32_t j = cf_ptr[c]; j < cf_ptr[c + 1]; j++) {
      const int32_t f = cf[j];
      for (int64_t k = fptr[f]; k < fptr[f + 1]; k++) {
        const int32_t pnode = g->f2n[k];
        bool seen = false;
        for (size_t m = start; m < c2n.size(); m++)
          if (c2n[m] == pnode) { seen = true; break; }
        if (!seen) c2n.push_back(pnode);
      }
    }
    ptr[c + 1] = (int32_t)c2n.size();
  }
}

}  // namespace

extern "C" int mfg_prep_c2n_size(const mfg_raw_grid *g, int64_t *n_c2n) {
  if (!g || !n_c2n) return MFG_ERR_INVALID;
  std::vector<int32_t> ptr, c2n;
  build_c2n(g, ptr, c2n);
  *n_c2n = (int64_t)c2n.size();
  return MFG_OK;
}

// ComputeWeight3D_Node (:831-1049) and FindNodeSYMM (:2060-2140).
extern "C" int mfg_prep_node_weights(const mfg_raw_grid *g, const int32_t *bctype,
                                     const double *xfn, const double *yfn, const double *zfn,
                                     const double *xfc, const double *yfc, const double *zfc,
                                     const double *xcc, const double *ycc, const double *zcc,
                                     double *wnode, int32_t *nmark, double *wbface, int32_t *nnpc,
                                     int32_t *c2n_out, double *wc2n, int32_t *nodesymm,
                                     double *xfn_n_symm, double *yfn_n_symm,
                                     double *zfn_n_symm) {
  if (!g || !bctype || !wnode || !nmark || !wbface || !nnpc || !c2n_out || !wc2n || !nodesymm ||
      !xfn_n_symm || !yfn_n_symm || !zfn_n_symm)
    return MFG_ERR_INVALID;
  const int32_t nN = g->n_node, nB = g->n_bface, nC = g->n_cell;
  const double *x = g->x, *y = g->y, *z = g->z;
  std::vector<int32_t> ptr, c2n;
  build_c2n(g, ptr, c2n);
  for (int32_t i = 0; i < nN; i++) {
    nmark[i] = 0;
    wnode[i] = 0.;
  }
  std::vector<int64_t> fptr(nB + 1, 0);
  for (int32_t i = 0; i < nB; i++) fptr[i + 1] = fptr[i] + g->nnpf[i];
  for (int64_t k = 0; k < fptr[nB]; k++) wbface[k] = 0.0;
  for (size_t k = 0; k < c2n.size(); k++) wc2n[k] = 0.0;
  auto face_pass = [&](int pass) {
    for (int32_t i = 0; i < nB; i++) {
      const int type = bctype[i];
      if (pass == 0 && type != MFG_BC_WALL) continue;
      if (pass == 1 && type != MFG_BC_FAR_FIELD && type != MFG_BC_FAR_FIELD_MOD) continue;
      if (pass == 2 && (type == MFG_BC_WALL || type == MFG_BC_SYMM || type == MFG_BC_FAR_FIELD ||
                        type == MFG_BC_FAR_FIELD_MOD || type == MFG_BC_INTERFACE))
        continue;
      for (int32_t j = 0; j < g->nnpf[i]; j++) {
        const int32_t p1 = g->f2n[fptr[i] + j];
        if (pass == 1 && nmark[p1] == MFG_BC_WALL) continue;
        if (pass == 2 && (nmark[p1] == MFG_BC_WALL || nmark[p1] == MFG_BC_FAR_FIELD)) continue;
        const double dx = x[p1] - xfc[i], dy = y[p1] - yfc[i], dz = z[p1] - zfc[i];
        double wr = dx * dx + dy * dy + dz * dz;
        wr = sqrt(wr);
        wr = 1. / wr;
        wbface[fptr[i] + j] = wr;
        wnode[p1] += wr;
        nmark[p1] = pass == 0 ? MFG_BC_WALL : (pass == 1 ? MFG_BC_FAR_FIELD : 101);
      }
    }
  };
  face_pass(0);
  face_pass(1);
  face_pass(2);
  for (int32_t i = 0; i < nC; i++) {
    nnpc[i] = ptr[i + 1] - ptr[i];
    for (int32_t j = ptr[i]; j < ptr[i + 1]; j++) {
      const int32_t p1 = c2n[j];
      c2n_out[j] = p1;
      if (nmark[p1] != 0) continue;
      const double dx = x[p1] - xcc[i], dy = y[p1] - ycc[i], dz = z[p1] - zcc[i];
      double wr = dx * dx + dy * dy + dz * dz;
      wr = sqrt(wr);
      wr = 1. / wr;
      wc2n[j] = wr;
      wnode[p1] += wr;
    }
  }
  // FindNodeSYMM
  std::vector<double> nface(nN, 0.0);
  for (int32_t i = 0; i < nN; i++) {
    nodesymm[i] = 2;
    xfn_n_symm[i] = 0.0;
    yfn_n_symm[i] = 0.0;
    zfn_n_symm[i] = 0.0;
  }
  for (int32_t i = 0; i < nB; i++) {
    if (bctype[i] != MFG_BC_SYMM) continue;
    for (int32_t j = 0; j < g->nnpf[i]; j++) {
      const int32_t p1 = g->f2n[fptr[i] + j];
      nodesymm[p1] = 1;
      xfn_n_symm[p1] += xfn[i];
      yfn_n_symm[p1] += yfn[i];
      zfn_n_symm[p1] += zfn[i];
      nface[p1] += 1.0;
    }
  }
  for (int32_t i = 0; i < nN; i++) {
    if (nodesymm[i] == 2) nodesymm[i] = 0;
    if (nodesymm[i] == 1) {
      xfn_n_symm[i] /= nface[i];
      yfn_n_symm[i] /= nface[i];
      zfn_n_symm[i] /= nface[i];
    }
  }
  return MFG_OK;
}
