// The reference's kernel entry points on top of libmfgpu's C ABI.
//
// Linked in place of src/Kernels/cal_flux.cpp, compute_timestep.cpp,
// forward_lusgs.cpp and cal_gradient.cpp, this file defines the symbols
// src/main.cpp and PreprocessGrid call -- ZeroResiduals and InviscidFlux
// (cal_flux.h:24,27), ComputeTimeStep (compute_timestep.h:24), ForwardLUSGS
// (forward_lusgs.h:23), AllocAndCalQuantityGradient and CalculateGradient
// (cal_gradient.h:22-23) -- with the reference's signatures, lazy host
// allocations and globals.  The grid and the flow field live on the GPU
// from AllocAndCalQuantityGradient (the last step of PreprocessGrid) on.
//
// The host arrays of the grid (res, q, dt, DQ, gradients) and the globals
// dt_max / dt_min are refreshed from the device at the end of the last
// iteration of main.cpp's loop (iter_done + 1 == n_steps, main.cpp:198,290:
// the loop has no other hook), or after every CalculateGradient when the
// environment sets MFGPU_SYNC_EVERY_CALL=1 (for parity dumps).
// MFGPU_DEVICE picks the CUDA device (default 0).  A failing call prints the
// library's error and exits(1), as the reference does on its own errors.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cal_flux.h"
#include "cal_gradient.h"
#include "compute_timestep.h"
#include "forward_lusgs.h"
#include "grid_polyhedra.h"
#include "memory_util.h"
#include "mfgpu.h"
#include "para_field_global.h"

namespace {

mfg_ctx *g_ctx = nullptr;

void must(int rc, const char *what) {
  if (rc == MFG_OK) return;
  fprintf(stderr, "%s: %s %s\n", what, mfg_error_string(rc), mfg_last_cuda_error());
  exit(1);
}

bool sync_every_call() {
  const char *v = getenv("MFGPU_SYNC_EVERY_CALL");
  return v && v[0] == '1';
}

int device_id() {
  const char *v = getenv("MFGPU_DEVICE");
  return v ? atoi(v) : 0;
}

// The reference's globals (para_field_global.h) as an mfg_params: the
// inputs and the values the reference derived from them, taken as they are.
mfg_params params_from_globals() {
  mfg_params p;
  memset(&p, 0, sizeof(p));
  p.mach = mach;
  p.alpha = alpha;
  p.beita = beita;
  p.re = re;
  p.T = T;
  p.gam = gam;
  p.gascon = gascon;
  p.cfl_start = cfl_start;
  p.cfl_end = cfl_end;
  p.cfl_nstep = cfl_nstep;
  p.lhs_omga = lhs_omga;
  p.epsa_r = epsa_r;
  p.ratio_dtmax = ratio_dtmax;
  p.amu = amu;
  p.ainf = ainf;
  p.uqq = uqq;
  p.u_s = u_s;
  p.v_s = v_s;
  p.w_s = w_s;
  p.p_s = p_s;
  p.rho_s = rho_s;
  p.p_bar = p_bar;
  p.gamm1 = gamm1;
  p.p_stag = p_stag;
  p.e_stag = e_stag;
  p.p_min = p_min;
  p.p_max = p_max;
  p.rho_min = rho_min;
  p.rho_max = rho_max;
  p.p_break = p_break;
  p.e_stag_max = e_stag_max;
  p.cfl_min = cfl_min;
  p.cfl_ratio = cfl_ratio;
  p.alf_l = alf_l;
  return p;
}

// The grid's arrays after PreprocessGrid, as the context's mesh.
void create_context(PolyGrid *g) {
  const int nc = g->GetNTCell(), nb = g->GetNBFace(), nf = g->GetNTFace(), nn = g->GetNTNode();
  const long long n = (long long)nc + nb;
  std::vector<int32_t> bct(nb > 0 ? nb : 1, 0);
  BCRecord **bcr = g->Getbcr();
  for (int i = 0; i < nb; i++) bct[i] = bcr[i]->GetType();
  IntType *nnpc = CalnNPC(g);
  IntType **c2n = CalC2N(g);
  mfg_mesh m;
  memset(&m, 0, sizeof(m));
  m.n_node = nn;
  m.n_face = nf;
  m.n_cell = nc;
  m.n_bface = nb;
  m.f2c = g->Getf2c();
  m.nnpf = g->GetnNPF();
  m.f2n = g->Getf2n();
  m.bctype = bct.data();
  m.xfn = g->GetXfn();
  m.yfn = g->GetYfn();
  m.zfn = g->GetZfn();
  m.area = g->GetFaceArea();
  m.xfc = g->GetXfc();
  m.yfc = g->GetYfc();
  m.zfc = g->GetZfc();
  m.xcc = g->GetXcc();
  m.ycc = g->GetYcc();
  m.zcc = g->GetZcc();
  m.vol = g->GetCellVol();
  m.wnode = g->GetWeightNodeDist();
  m.nmark = g->GetNodeType();
  m.wbface = g->GetWeightNodeBFace2C()[0];
  m.nnpc = nnpc;
  m.c2n = c2n[0];
  m.wc2n = g->GetWeightNodeC2N()[0];
  m.nodesymm = g->GetNodeSymm();
  m.xfn_n_symm = g->GetXfnNSymm();
  m.yfn_n_symm = g->GetYfnNSymm();
  m.zfn_n_symm = g->GetZfnNSymm();
  m.lusgs_order = g->GetLUSGSCellOrder();
  m.lusgs_layer = g->GetLUSGSLayer();
  std::vector<double> q0(5 * n);
  const RealFlow *src[5] = {g->GetRho(), g->GetU(), g->GetV(), g->GetW(), g->GetP()};
  for (int k = 0; k < 5; k++) memcpy(&q0[k * n], src[k], sizeof(double) * n);
  const mfg_params p = params_from_globals();
  must(mfg_create(&m, &p, q0.data(), device_id(), MFG_PREC_FP64, &g_ctx), "mfg_create");
}

// Device -> the grid's host arrays and the dt extrema globals.
void sync_to_host(PolyGrid *g) {
  const int nc = g->GetNTCell(), nb = g->GetNBFace();
  const long long n = (long long)nc + nb;
  std::vector<double> q(5 * n);
  must(mfg_download(g_ctx, MFG_FIELD_Q, q.data()), "mfg_download q");
  RealFlow *dst[5] = {g->GetRho(), g->GetU(), g->GetV(), g->GetW(), g->GetP()};
  for (int k = 0; k < 5; k++) memcpy(dst[k], &q[k * n], sizeof(double) * n);
  if (g->GetRes()) must(mfg_download(g_ctx, MFG_FIELD_RES, g->GetRes()), "mfg_download res");
  if (g->GetDt()) must(mfg_download(g_ctx, MFG_FIELD_DT, g->GetDt()), "mfg_download dt");
  if (g->GetDQ()) must(mfg_download(g_ctx, MFG_FIELD_DQ, g->GetDQ()), "mfg_download DQ");
  must(mfg_download(g_ctx, MFG_FIELD_DQDX, g->GetDqdx()), "mfg_download dqdx");
  must(mfg_download(g_ctx, MFG_FIELD_DQDY, g->GetDqdy()), "mfg_download dqdy");
  must(mfg_download(g_ctx, MFG_FIELD_DQDZ, g->GetDqdz()), "mfg_download dqdz");
  double mx = 0.0, mn = 0.0;
  must(mfg_get_dt_extrema(g_ctx, &mx, &mn), "mfg_get_dt_extrema");
  dt_max = mx;
  dt_min = mn;
}

}  // namespace

void AllocAndCalQuantityGradient(PolyGrid *grid) {
  const long long n = (long long)grid->GetNTCell() + grid->GetNBFace();
  RealFlow *dqdx = NULL, *dqdy = NULL, *dqdz = NULL;
  snew_array_1D(dqdx, 5 * n);
  snew_array_1D(dqdy, 5 * n);
  snew_array_1D(dqdz, 5 * n);
  grid->SetDqdx(dqdx);
  grid->SetDqdy(dqdy);
  grid->SetDqdz(dqdz);
  if (g_ctx) must(mfg_destroy(g_ctx), "mfg_destroy");
  create_context(grid);
  CalculateGradient(grid);
}

void ZeroResiduals(PolyGrid *grid) {
  if (!grid->GetRes()) {
    RealFlow *res = NULL;
    snew_array_1D(res, 5 * (size_t)grid->GetNTCell());
    grid->SetRes(res);
  }
  must(mfg_zero_residuals(g_ctx), "ZeroResiduals");
}

void InviscidFlux(PolyGrid *grid, RealFlow **limit, IntType level) {
  (void)grid;
  (void)limit;
  (void)level;
  must(mfg_inviscid_flux(g_ctx), "InviscidFlux");
}

void ComputeTimeStep(PolyGrid *grid) {
  if (!grid->GetDt()) {
    RealFlow *dt = NULL;
    snew_array_1D(dt, (size_t)grid->GetNTCell());
    grid->SetDt(dt);
  }
  must(mfg_compute_timestep(g_ctx, iter_done), "ComputeTimeStep");
}

void ForwardLUSGS(PolyGrid *grid, IntType level) {
  (void)level;
  if (!grid->GetDQ()) {
    RealFlow *dq = NULL;
    snew_array_1D(dq, 5 * ((size_t)grid->GetNTCell() + grid->GetNBFace()));
    grid->SetDQ(dq);
  }
  must(mfg_forward_lusgs(g_ctx), "ForwardLUSGS");
}

void CalculateGradient(PolyGrid *grid) {
  must(mfg_calculate_gradient(g_ctx), "CalculateGradient");
  if (sync_every_call() || iter_done + 1 == n_steps) sync_to_host(grid);
}
