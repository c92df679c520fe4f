// TEST INFRASTRUCTURE ONLY -- never linked into, loaded by, or called from the
// product library.  This driver is compiled together with the UNMODIFIED
// MiniFS sources (src/Base/*.cpp, src/Kernels/*.cpp; for the TDTree variant
// also src/src/*.cpp and libmetis.a) by oracle/Makefile into oracle/_ref/.
//
// It replaces only what src/main.cpp hard-codes:
//   * the grid path (load_grid.cpp:86) -> --mesh / --bc arguments;
//   * the parameter block (para_field_global.cpp:37-221) -> --params file,
//     re-deriving every dependent global with the formulas of
//     para_field_global.cpp:150-209;
//   * the seeded initial state: a Gaussian density bump at the cell
//     centroids, applied between AllocAndInitFlowfield and SetGhostVariables
//     in the PreprocessGrid sequence (load_grid.cpp:443-531).
// The iteration loop is main.cpp:201-291 verbatim in call order (with
// --live-bc, also the SetGhostVariables call that main.cpp:286 comments
// out).  Arrays are dumped to a simple tagged binary file for the Python
// tests.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "grid_polyhedra.h"
#include "para_field_global.h"
#include "load_grid.h"
#include "cal_flux.h"
#include "compute_timestep.h"
#include "forward_lusgs.h"
#include "cal_gradient.h"

#if defined(TDTREE)
#include <omp.h>
#endif

// Globals of para_field_global.cpp that its header does not declare.
extern RealFlow tref, sref, amuref, trat, alpha_t, beita_t, temp, p_stag_t,
    rho_stag, ratio_rhop_max, ratio_rhop_min, ratio_p_break;

namespace {

struct Dump {
  FILE *f = nullptr;
  void open(const char *path) {
    f = fopen(path, "wb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    fwrite("MFDUMP01", 1, 8, f);
  }
  template <typename T>
  void put(const std::string &name, const T *p, long long n, char code) {
    if (!f) return;
    int len = (int)name.size();
    fwrite(&len, 4, 1, f);
    fwrite(name.data(), 1, len, f);
    fwrite(&code, 1, 1, f);
    fwrite(&n, 8, 1, f);
    if (n) fwrite(p, sizeof(T), n, f);
  }
  void d(const std::string &name, const double *p, long long n) { put(name, p, n, 'd'); }
  void i(const std::string &name, const int *p, long long n) { put(name, p, n, 'i'); }
  void close() { if (f) fclose(f); f = nullptr; }
};

double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

std::map<std::string, double> read_params(const char *path) {
  std::map<std::string, double> kv;
  FILE *f = fopen(path, "r");
  if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  char key[128];
  double val;
  while (fscanf(f, "%127s %lf", key, &val) == 2) kv[key] = val;
  fclose(f);
  return kv;
}

// para_field_global.cpp:150-209, re-evaluated at run time after overrides.
void derive_globals() {
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

void write_mfl(PolyGrid *g, const char *path) {
  FILE *f = fopen(path, "wb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  int nn = g->GetNTNode(), nf = g->GetNTFace(), nc = g->GetNTCell();
  int hdr[3] = {nn, nf, nc};
  fwrite(hdr, 4, 3, f);
  fwrite(g->GetX(), 8, nn, f);
  fwrite(g->GetY(), 8, nn, f);
  fwrite(g->GetZ(), 8, nn, f);
  fwrite(g->GetnNPF(), 4, nf, f);
  long long s = 0;
  for (int i = 0; i < nf; i++) s += g->GetnNPF()[i];
  fwrite(g->Getf2n(), 4, s, f);
  fwrite(g->Getf2c(), 4, 2LL * nf, f);
  int tail[2] = {0, 0};
  fwrite(tail, 4, 2, f);
  fclose(f);
}

void dump_state(Dump &D, PolyGrid *g, const std::string &pfx) {
  long long n = (long long)g->GetNTCell() + g->GetNBFace();
  std::vector<double> q(5 * n);
  const double *src[5] = {g->GetRho(), g->GetU(), g->GetV(), g->GetW(), g->GetP()};
  for (int k = 0; k < 5; k++) memcpy(&q[k * n], src[k], n * sizeof(double));
  D.d(pfx + "q", q.data(), 5 * n);
}

void dump_grad(Dump &D, PolyGrid *g, const std::string &pfx) {
  long long n = (long long)g->GetNTCell() + g->GetNBFace();
  D.d(pfx + "dqdx", g->GetDqdx(), 5 * n);
  D.d(pfx + "dqdy", g->GetDqdy(), 5 * n);
  D.d(pfx + "dqdz", g->GetDqdz(), 5 * n);
}

void dump_preprocessing(Dump &D, PolyGrid *g) {
  int nc = g->GetNTCell(), nb = g->GetNBFace(), nf = g->GetNTFace(), nn = g->GetNTNode();
  long long n = (long long)nc + nb;
  int dims[4] = {nn, nf, nc, nb};
  D.i("dims", dims, 4);
  D.i("f2c", g->Getf2c(), 2LL * nf);
  D.i("nnpf", g->GetnNPF(), nf);
  long long s = 0;
  for (int i = 0; i < nf; i++) s += g->GetnNPF()[i];
  D.i("f2n", g->Getf2n(), s);
  D.d("x", g->GetX(), nn);
  D.d("y", g->GetY(), nn);
  D.d("z", g->GetZ(), nn);
  D.d("xfn", g->GetXfn(), nf);
  D.d("yfn", g->GetYfn(), nf);
  D.d("zfn", g->GetZfn(), nf);
  D.d("area", g->GetFaceArea(), nf);
  D.d("xfc", g->GetXfc(), nf);
  D.d("yfc", g->GetYfc(), nf);
  D.d("zfc", g->GetZfc(), nf);
  D.d("xcc", g->GetXcc(), n);
  D.d("ycc", g->GetYcc(), n);
  D.d("zcc", g->GetZcc(), n);
  D.d("vol", g->GetCellVol(), n);
  std::vector<int> bct(nb);
  BCRecord **bcr = g->Getbcr();
  for (int i = 0; i < nb; i++) bct[i] = bcr[i]->GetType();
  D.i("bctype", bct.data(), nb);
  D.d("wnode", g->GetWeightNodeDist(), nn);
  D.i("nmark", g->GetNodeType(), nn);
  long long sb = 0;
  for (int i = 0; i < nb; i++) sb += g->GetnNPF()[i];
  D.d("wbface", g->GetWeightNodeBFace2C()[0], sb);
  IntType *nnpc = CalnNPC(g);
  IntType **c2n = CalC2N(g);
  long long sc = 0;
  for (int i = 0; i < nc; i++) sc += nnpc[i];
  D.i("nnpc", nnpc, nc);
  D.i("c2n", c2n[0], sc);
  D.d("wc2n", g->GetWeightNodeC2N()[0], sc);
  D.i("nodesymm", g->GetNodeSymm(), nn);
  D.d("xfn_n_symm", g->GetXfnNSymm(), nn);
  D.d("yfn_n_symm", g->GetYfnNSymm(), nn);
  D.d("zfn_n_symm", g->GetZfnNSymm(), nn);
}

}  // namespace

int main(int argc, char **argv) {
  const char *mesh = nullptr, *bcf = nullptr, *params = nullptr, *out = nullptr,
             *write_mesh = nullptr;
  std::set<int> dump_iters;
  bool dump_all_iters = false;
  bool light = false;  // timings and norms only
  bool live_bc = false;  // SetGhostVariables in the loop, where main.cpp:286 has it commented out
  for (int a = 1; a < argc; a++) {
    std::string k = argv[a];
    auto need = [&](void) -> const char * {
      if (a + 1 >= argc) { fprintf(stderr, "missing value for %s\n", k.c_str()); exit(2); }
      return argv[++a];
    };
    if (k == "--mesh") mesh = need();
    else if (k == "--bc") bcf = need();
    else if (k == "--params") params = need();
    else if (k == "--out") out = need();
    else if (k == "--write-mesh") write_mesh = need();
    else if (k == "--light") light = true;
    else if (k == "--live-bc") live_bc = true;
    else if (k == "--dump-iters") {
      std::string v = need();
      if (v == "all") dump_all_iters = true;
      else {
        size_t p = 0;
        while (p < v.size()) {
          size_t q = v.find(',', p);
          if (q == std::string::npos) q = v.size();
          dump_iters.insert(atoi(v.substr(p, q - p).c_str()));
          p = q + 1;
        }
      }
    } else { fprintf(stderr, "unknown argument %s\n", k.c_str()); return 2; }
  }
  if (!mesh || !bcf || !params) {
    fprintf(stderr, "usage: %s --mesh f.mfl --bc bc.para --params p.txt [--out dump.bin] "
                    "[--dump-iters 0,1,5|all] [--write-mesh renumbered.mfl] [--light] "
                    "[--live-bc]\n", argv[0]);
    return 2;
  }
  std::map<std::string, double> kv = read_params(params);
  auto getd = [&](const char *key, double dflt) { return kv.count(key) ? kv[key] : dflt; };
  mach = getd("mach", mach);
  alpha = getd("alpha", alpha);
  beita = getd("beita", beita);
  re = getd("re", re);
  T = getd("T", T);
  gam = getd("gam", gam);
  gascon = getd("gascon", gascon);
  cfl_start = getd("cfl_start", cfl_start);
  cfl_end = getd("cfl_end", cfl_end);
  cfl_nstep = (IntType)getd("cfl_nstep", cfl_nstep);
  n_steps = (IntType)getd("n_steps", n_steps);
  lhs_omga = getd("lhs_omga", lhs_omga);
  epsa_r = getd("epsa_r", epsa_r);
  ratio_dtmax = getd("ratio_dtmax", ratio_dtmax);
  const double bump_amp = getd("bump_amp", 0.0), bump_sigma = getd("bump_sigma", 0.1);
  const double bx0 = getd("bump_x0", 0.5), by0 = getd("bump_y0", 0.5), bz0 = getd("bump_z0", 0.5);
  derive_globals();

  Dump D;
  if (out) D.open(out);
  double par[] = {mach, alpha, beita, re, T, gam, gascon, cfl_start, cfl_end, (double)cfl_nstep,
                  lhs_omga, alf_l, ratio_dtmax, amu, ainf, uqq, u_s, v_s, w_s, p_s, rho_s,
                  p_bar, gamm1, p_stag, e_stag, p_min, p_max, rho_min, rho_max, p_break,
                  e_stag_max, cfl_min, cfl_ratio};
  D.d("params", par, sizeof(par) / sizeof(double));

  PolyGrid *grid = new PolyGrid();
  BCond *bc = new BCond();
  ReadMFlowGrid_binary(grid, mesh);
  ReadMFlowBoundaryCondition(bc, bcf);
  double t0 = now_s();
  Decoupling(grid);  // main.cpp:169 (TDTree renumbering when built with TDTREE)
  double t_decouple = now_s() - t0;
  if (write_mesh) write_mfl(grid, write_mesh);

  // PreprocessGrid (load_grid.cpp:405-540) with the initial bump inserted.
  t0 = now_s();
  SpecifyNeighbors(grid);
  SpecifyBC(grid, bc);
  grid->ComputeMetrics();
  ReorderCellforLUSGS(grid);
  AllocAndInitFlowfield(grid);
  {
    const int nc = grid->GetNTCell();
    RealFlow *rho = grid->GetRho();
    const RealGeom *xcc = grid->GetXcc(), *ycc = grid->GetYcc(), *zcc = grid->GetZcc();
    if (bump_amp != 0.0) {
      for (int i = 0; i < nc; i++) {
        double dx = xcc[i] - bx0, dy = ycc[i] - by0, dz = zcc[i] - bz0;
        double r2 = dx * dx + dy * dy + dz * dz;
        rho[i] = rho_s * (1.0 + bump_amp * exp(-r2 / (2.0 * bump_sigma * bump_sigma)));
      }
    }
  }
  PassInterfaceData(grid);
  SetGhostVariables(grid);
  ComputeWeight3D_Node(grid);
  FindNodeSYMM(grid);
  AllocAndCalQuantityGradient(grid);
  double t_pre = now_s() - t0;
  if (!light) {
    dump_preprocessing(D, grid);
    dump_state(D, grid, "init.");
    dump_grad(D, grid, "init.");
  }
  std::vector<double> iter_times;

  const int nc = grid->GetNTCell();
  const long long n = (long long)nc + grid->GetNBFace();
  std::vector<double> norms;
  std::vector<double> diag(nc);
  double t_loop = 0.0, t_phase[4] = {0, 0, 0, 0};  // inviscid, lusgs, gradient, timestep
  double loop_before = 0.0;
  for (IntType inner_iter = 0; inner_iter < n_steps; ++inner_iter) {
    const bool dump_it = out && (dump_all_iters || dump_iters.count(inner_iter));
    const std::string pfx = "it" + std::to_string(inner_iter) + ".";
    double t_a = now_s();
    ZeroResiduals(grid);
#ifdef TDTREE
    InviscidFlux_TDTree(grid, NULL, 0);
#else
    InviscidFlux(grid, NULL, 0);
#endif
    double t_b = now_s();
    ComputeTimeStep(grid);
    double t_c = now_s();
    t_phase[0] += t_b - t_a;
    t_phase[3] += t_c - t_b;
    t_loop += t_c - t_a;
    if (dump_it) {
      // Diag exactly as ForwardLUSGS forms it (forward_lusgs.cpp:91-101);
      // CalDiagLUSGS only reads the flow field, so the extra call is inert.
      const RealGeom *vol = grid->GetCellVol();
      const RealFlow *dt = grid->GetDt();
      for (int i = 0; i < nc; i++) diag[i] = vol[i] / dt[i];
#ifdef TDTREE
      CalDiagLUSGS_TDTree(grid, diag.data(), 0);
#else
      CalDiagLUSGS(grid, diag.data(), 0);
#endif
      D.d(pfx + "res", grid->GetRes(), 5LL * nc);
      D.d(pfx + "dt", grid->GetDt(), nc);
      D.d(pfx + "diag", diag.data(), nc);
    }
    t_a = now_s();
    ForwardLUSGS(grid, 0);
    PassInterfaceData(grid);
    if (live_bc) SetGhostVariables(grid);
    t_b = now_s();
    CalculateGradient(grid);
    iter_done++;
    t_c = now_s();
    t_phase[1] += t_b - t_a;
    t_phase[2] += t_c - t_b;
    t_loop += t_c - t_a;
    iter_times.push_back(t_loop - loop_before);
    loop_before = t_loop;
    // residual norm exactly as main.cpp:294-317 (on the residual of this step)
    const RealFlow *res = grid->GetRes();
    for (int j = 0; j < 5; j++) {
      double s = 0.0;
      for (int i = 0; i < nc; i++) s += res[(long long)j * nc + i] * res[(long long)j * nc + i];
      norms.push_back(sqrt(s));
    }
    if (dump_it) {
      D.d(pfx + "dq_lusgs", grid->GetDQ(), 5 * n);
      dump_state(D, grid, pfx);
      dump_grad(D, grid, pfx);
      double ext[2] = {dt_max, dt_min};
      D.d(pfx + "dt_extrema", ext, 2);
    }
  }
  D.d("norms", norms.data(), (long long)norms.size());
  D.d("iter_times", iter_times.data(), (long long)iter_times.size());
  double ext[2] = {dt_max, dt_min};
  D.d("final.dt_extrema", ext, 2);
  if (!light) {
    D.d("final.res", grid->GetRes(), 5LL * nc);
    dump_state(D, grid, "final.");
    dump_grad(D, grid, "final.");
  }
  double tim[8] = {t_loop, t_pre, t_decouple, t_phase[0], t_phase[1], t_phase[2], t_phase[3],
                   (double)n_steps};
  D.d("timing", tim, 8);
  D.close();
  int threads = 1;
#if defined(TDTREE)
  threads = omp_get_max_threads();
#endif
  printf("{\"cells\": %d, \"iters\": %d, \"loop_s\": %.6f, \"preprocess_s\": %.6f, "
         "\"decouple_s\": %.6f, \"threads\": %d, \"inviscid_s\": %.6f, \"lusgs_s\": %.6f, "
         "\"gradient_s\": %.6f, \"timestep_s\": %.6f, \"norm0\": %.17g, \"dt_max\": %.17g, "
         "\"dt_min\": %.17g}\n",
         nc, (int)n_steps, t_loop, t_pre, t_decouple, threads, t_phase[0], t_phase[1], t_phase[2],
         t_phase[3], norms.empty() ? 0.0 : norms[norms.size() - 5], dt_max, dt_min);
  return 0;
}
