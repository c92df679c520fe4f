// TEST INFRASTRUCTURE ONLY.
//
// Known-answer harness: calls single reference functions on caller-chosen
// inputs, so that the fixtures under tests/golden/ pin the oracle's per-face
// arithmetic (the whole-routine dumps of ref_harness.cpp pin the loops).
// Linked with the unmodified MiniFS Base and Kernels sources by
// oracle/Makefile into oracle/_ref/minifs_kat.
//
//   minifs_kat roe   <in> <out>   RoeFlux_noprec (cal_flux.cpp:301-834)
//   minifs_kat lusgs <in> <out>   FluxLUSGS3D (forward_lusgs.cpp:1271-1324)
//   minifs_kat update <in> <out>  UpdateFlowField3D_CFL3d (forward_lusgs.cpp:1335-1488)
//
// <in> is raw float64.  roe: len, gam, p_bar, alf_l, then ql[5][len],
// qr[5][len], xfn[len], yfn[len], zfn[len], area[len] (SoA, as the
// reference's face chunks); <out> is flux[5][len].  lusgs: len, gam, p_bar,
// lhs_omga, then per case q[5], dq[5], n[3]; <out> is flux[5] per case.
// update: len (cells), gam, p_bar, unused, then rho_s, rho_min, rho_max,
// p_min, p_max, q[5][len] (primitive), DQ[5][len]; <out> is the updated
// q[5][len] (a grid of len cells and no ghosts).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "grid_polyhedra.h"
#include "para_field_global.h"
#include "cal_flux.h"
#include "forward_lusgs.h"

static std::vector<double> read_all(const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  std::vector<double> v;
  double buf[4096];
  size_t got;
  while ((got = fread(buf, sizeof(double), 4096, f)) > 0) v.insert(v.end(), buf, buf + got);
  fclose(f);
  return v;
}

static void write_all(const char *path, const std::vector<double> &v) {
  FILE *f = fopen(path, "wb");
  if (!f || fwrite(v.data(), sizeof(double), v.size(), f) != v.size()) { perror(path); exit(2); }
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s roe|lusgs <in> <out>\n", argv[0]);
    return 2;
  }
  std::vector<double> in = read_all(argv[2]);
  if (in.size() < 4) { fprintf(stderr, "short input\n"); return 2; }
  const long len = (long)in[0];
  gam = in[1];
  gamm1 = gam - 1.0;
  p_bar = in[2];
  const double *d = in.data() + 4;
  std::vector<double> out;
  if (!strcmp(argv[1], "roe")) {
    if (in.size() != 4 + 14 * (size_t)len) { fprintf(stderr, "bad roe input size\n"); return 2; }
    std::vector<double> ql(d, d + 5 * len), qr(d + 5 * len, d + 10 * len);
    std::vector<double> xfn(d + 10 * len, d + 11 * len), yfn(d + 11 * len, d + 12 * len),
        zfn(d + 12 * len, d + 13 * len), area(d + 13 * len, d + 14 * len);
    out.assign(5 * len, 0.0);
    RealFlow *pl[5], *pr[5], *pf[5];
    for (int k = 0; k < 5; k++) {
      pl[k] = ql.data() + k * len;
      pr[k] = qr.data() + k * len;
      pf[k] = out.data() + k * len;
    }
    // the steady first-order path reads only the grid's counts and f2c
    // (unused for the flux itself); a default grid serves.  Never freed:
    // the process ends right after.
    PolyGrid *grid = new PolyGrid();
    const double alf = in[3];
    RoeFlux_noprec(grid, pl, pr, pf, xfn.data(), yfn.data(), zfn.data(), area.data(), NULL, gam,
                   p_bar, alf, alf, 0, (IntType)len);
  } else if (!strcmp(argv[1], "lusgs")) {
    if (in.size() != 4 + 13 * (size_t)len) { fprintf(stderr, "bad lusgs input size\n"); return 2; }
    const double lhs = in[3];
    out.assign(5 * len, 0.0);
    for (long i = 0; i < len; i++) {
      RealFlow q[5], dq[5], flux[5];
      RealGeom n[3];
      const double *c = d + 13 * i;
      for (int k = 0; k < 5; k++) { q[k] = c[k]; dq[k] = c[5 + k]; }
      for (int k = 0; k < 3; k++) n[k] = c[10 + k];
      FluxLUSGS3D(flux, q, dq, n, gam, p_bar, lhs);
      for (int k = 0; k < 5; k++) out[5 * i + k] = flux[k];
    }
  } else if (!strcmp(argv[1], "update")) {
    if (in.size() != 9 + 10 * (size_t)len) { fprintf(stderr, "bad update input size\n"); return 2; }
    rho_s = d[0];
    rho_min = d[1];
    rho_max = d[2];
    p_min = d[3];
    p_max = d[4];
    const double *q = d + 5, *dq = d + 5 + 5 * len;
    // the grid owns its state arrays (new[]); never freed: the process ends
    PolyGrid *grid = new PolyGrid();
    grid->SetNTCell((IntType)len);
    grid->SetNBFace(0);
    RealFlow *prim[5], *DQ[5];
    for (int k = 0; k < 5; k++) {
      prim[k] = new RealFlow[len];
      DQ[k] = new RealFlow[len];
      memcpy(prim[k], q + k * len, len * sizeof(double));
      memcpy(DQ[k], dq + k * len, len * sizeof(double));
    }
    grid->SetRho(prim[0]);
    grid->SetU(prim[1]);
    grid->SetV(prim[2]);
    grid->SetW(prim[3]);
    grid->SetP(prim[4]);
    UpdateFlowField3D_CFL3d(grid, DQ);
    out.resize(5 * len);
    for (int k = 0; k < 5; k++) memcpy(out.data() + k * len, prim[k], len * sizeof(double));
  } else {
    fprintf(stderr, "unknown mode %s\n", argv[1]);
    return 2;
  }
  write_all(argv[3], out);
  return 0;
}
