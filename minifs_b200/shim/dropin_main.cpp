// The reference's own driver sequence (src/main.cpp:160-291 with
// PreprocessGrid, load_grid.cpp:405-540) running on libmfgpu through
// mfgpu_shim.cpp: the demonstration that the C ABI drops in under the
// reference's unmodified Base and load_grid code.
//
// main.cpp hard-codes its grid path and parameters, so this driver takes
// them from the command line (--mesh grid.mfl --bc bc.para --params file,
// one "key value" per line; the density bump of the synthetic cases is
// applied between AllocAndInitFlowfield and SetGhostVariables), runs the
// loop in main.cpp's call order, and writes the residual norms of every
// iteration and the final state, residual, gradients and dt extrema to
// --out in a tagged binary form (8-byte magic "MFDUMP01", then records of
// name length, name, type code 'd'/'i', count, data).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <string>
#include <vector>

#include "cal_flux.h"
#include "cal_gradient.h"
#include "compute_timestep.h"
#include "forward_lusgs.h"
#include "grid_polyhedra.h"
#include "load_grid.h"
#include "para_field_global.h"

// Globals para_field_global.cpp defines without declaring them.
extern RealFlow tref, sref, amuref, trat, alpha_t, beita_t, temp, p_stag_t, rho_stag,
    ratio_rhop_max, ratio_rhop_min, ratio_p_break;

namespace {

struct Out {
  FILE *f = nullptr;
  void put(const std::string &name, const void *p, long long n, char code, size_t size) {
    const int len = (int)name.size();
    fwrite(&len, 4, 1, f);
    fwrite(name.data(), 1, len, f);
    fwrite(&code, 1, 1, f);
    fwrite(&n, 8, 1, f);
    if (n) fwrite(p, size, n, f);
  }
  void d(const std::string &name, const double *p, long long n) { put(name, p, n, 'd', 8); }
};

std::map<std::string, double> read_params(const char *path) {
  std::map<std::string, double> kv;
  FILE *f = fopen(path, "r");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  char key[128];
  double val;
  while (fscanf(f, "%127s %lf", key, &val) == 2) kv[key] = val;
  fclose(f);
  return kv;
}

// The dependent globals of para_field_global.cpp:150-209, after overrides.
void derive() {
  trat = (T / tref);
  amu = amuref * trat * sqrt(trat) * (tref + sref) / (T + sref);
  ainf = sqrt(gam * gascon * T);
  uqq = ainf * mach;
  alpha_t = (alpha * PI / 180.);
  beita_t = (beita * PI / 180.);
  u_s = uqq * cos(alpha_t) * cos(-1. * beita_t);
  v_s = uqq * sin(-1. * beita_t);
  w_s = uqq * sin(alpha_t) * cos(-1. * beita_t);
  p_s = 0.00;
  rho_s = re * amu / uqq;
  p_bar = rho_s * gascon * T;
  gamm1 = gam - 1.0;
  temp = 1.0 + 0.5 * gamm1 * mach * mach;
  p_stag_t = pow(temp, gam / gamm1);
  rho_stag = pow(temp, 1.0 / gamm1) * rho_s;
  p_stag = (p_stag_t - 1.0) * p_bar;
  e_stag = p_bar / gamm1 + 0.5 * rho_s * (u_s * u_s + v_s * v_s + w_s * w_s);
  p_min = ratio_rhop_min * p_bar - p_bar;
  p_max = ratio_rhop_max * (p_stag + p_bar) - p_bar;
  rho_min = ratio_rhop_min * rho_s;
  rho_max = ratio_rhop_max * rho_stag;
  p_break = ratio_p_break * p_bar - p_bar;
  e_stag_max = 1.0e5 * e_stag;
  cfl_min = 0.5 * cfl_start;
  cfl_ratio = cfl_end / cfl_start;
  alf_l = epsa_r;
  alf_n = epsa_r;
}

double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

}  // namespace

int main(int argc, char **argv) {
  const char *mesh = nullptr, *bcf = nullptr, *params = nullptr, *out = nullptr;
  for (int a = 1; a + 1 < argc; a += 2) {
    const std::string k = argv[a];
    if (k == "--mesh") mesh = argv[a + 1];
    else if (k == "--bc") bcf = argv[a + 1];
    else if (k == "--params") params = argv[a + 1];
    else if (k == "--out") out = argv[a + 1];
    else {
      fprintf(stderr, "unknown argument %s\n", k.c_str());
      return 2;
    }
  }
  if (!mesh || !bcf || !params || !out) {
    fprintf(stderr, "usage: %s --mesh g.mfl --bc bc.para --params p.txt --out dump.bin\n",
            argv[0]);
    return 2;
  }
  std::map<std::string, double> kv = read_params(params);
  auto get = [&](const char *key, double dflt) { return kv.count(key) ? kv[key] : dflt; };
  mach = get("mach", mach);
  alpha = get("alpha", alpha);
  beita = get("beita", beita);
  re = get("re", re);
  T = get("T", T);
  gam = get("gam", gam);
  gascon = get("gascon", gascon);
  cfl_start = get("cfl_start", cfl_start);
  cfl_end = get("cfl_end", cfl_end);
  cfl_nstep = (IntType)get("cfl_nstep", cfl_nstep);
  n_steps = (IntType)get("n_steps", n_steps);
  lhs_omga = get("lhs_omga", lhs_omga);
  epsa_r = get("epsa_r", epsa_r);
  ratio_dtmax = get("ratio_dtmax", ratio_dtmax);
  const double amp = get("bump_amp", 0.0), sig = get("bump_sigma", 0.1);
  const double x0 = get("bump_x0", 0.5), y0 = get("bump_y0", 0.5), z0 = get("bump_z0", 0.5);
  derive();

  PolyGrid *grid = new PolyGrid();
  BCond *bc = new BCond();
  ReadMFlowGrid_binary(grid, mesh);
  ReadMFlowBoundaryCondition(bc, bcf);
  Decoupling(grid);
  // PreprocessGrid (load_grid.cpp:405-540) with the density bump inserted
  const double t0 = now_s();
  SpecifyNeighbors(grid);
  SpecifyBC(grid, bc);
  grid->ComputeMetrics();
  ReorderCellforLUSGS(grid);
  AllocAndInitFlowfield(grid);
  if (amp != 0.0) {
    const int nc = grid->GetNTCell();
    RealFlow *rho = grid->GetRho();
    const RealGeom *xc = grid->GetXcc(), *yc = grid->GetYcc(), *zc = grid->GetZcc();
    for (int i = 0; i < nc; i++) {
      const double dx = xc[i] - x0, dy = yc[i] - y0, dz = zc[i] - z0;
      const double r2 = dx * dx + dy * dy + dz * dz;
      rho[i] = rho_s * (1.0 + amp * exp(-r2 / (2.0 * sig * sig)));
    }
  }
  PassInterfaceData(grid);
  SetGhostVariables(grid);
  ComputeWeight3D_Node(grid);
  FindNodeSYMM(grid);
  AllocAndCalQuantityGradient(grid);  // the context is created here (shim)
  const double t_pre = now_s() - t0;

  // main.cpp:201-291
  const int nc = grid->GetNTCell();
  const long long n = (long long)nc + grid->GetNBFace();
  std::vector<double> norms;
  const double t1 = now_s();
  for (IntType inner_iter = 0; inner_iter < n_steps; ++inner_iter) {
    ZeroResiduals(grid);
    InviscidFlux(grid, NULL, 0);
    ComputeTimeStep(grid);
    ForwardLUSGS(grid, 0);
    PassInterfaceData(grid);
    CalculateGradient(grid);
    iter_done++;
    if (getenv("MFGPU_SYNC_EVERY_CALL")) {  // main.cpp:294-317 on every iteration
      const RealFlow *res = grid->GetRes();
      for (int j = 0; j < 5; j++) {
        double s = 0.0;
        for (int i = 0; i < nc; i++) s += res[(long long)j * nc + i] * res[(long long)j * nc + i];
        norms.push_back(sqrt(s));
      }
    }
  }
  const double t_loop = now_s() - t1;

  Out o;
  o.f = fopen(out, "wb");
  if (!o.f) {
    fprintf(stderr, "cannot open %s\n", out);
    return 2;
  }
  fwrite("MFDUMP01", 1, 8, o.f);
  o.d("norms", norms.data(), (long long)norms.size());
  std::vector<double> q(5 * n);
  const double *src[5] = {grid->GetRho(), grid->GetU(), grid->GetV(), grid->GetW(), grid->GetP()};
  for (int k = 0; k < 5; k++) memcpy(&q[k * n], src[k], sizeof(double) * n);
  o.d("final.q", q.data(), 5 * n);
  o.d("final.res", grid->GetRes(), 5LL * nc);
  o.d("final.dqdx", grid->GetDqdx(), 5 * n);
  o.d("final.dqdy", grid->GetDqdy(), 5 * n);
  o.d("final.dqdz", grid->GetDqdz(), 5 * n);
  double ext[2] = {dt_max, dt_min};
  o.d("final.dt_extrema", ext, 2);
  fclose(o.f);
  printf("{\"cells\": %d, \"iters\": %d, \"loop_s\": %.6f, \"preprocess_s\": %.6f}\n", nc,
         (int)n_steps, t_loop, t_pre);
  return 0;
}
