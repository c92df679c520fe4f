// mfgpu: the MiniFS iteration hot path on B200 (sm_100a), behind the C ABI
// of include/mfgpu.h.
//
// Layout in HBM (C cells, G ghosts, n = C + G, S = sum of faces per cell):
//   q8[2][n][8]     two state buffers (the backward sweep writes the update
//                   into the other one; ghosts are frozen and held by both)
//   dq8[n][8]       LU-SGS increments (ghost rows stay zero)
//   res[5][C], dt[C], diag[C]            SoA, as the reference
//   dqdx/dqdy/dqdz[5][n]                 SoA, as the reference
//   qn8[N][8]       node values of the gradient
//   slots[S]        (cell, face) records in ascending face order per cell
//   fw_*/bw_*       LU-SGS level sets: cells sorted by (level, index) and
//                   their lower / upper neighbour records in that order
//   node lists      per node, its contributions in the reference's order
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <thread>

#include "mfg_internal.h"
#include "mfg_kernels.cuh"
#include "mfgpu.h"

using namespace mfg;

namespace {

thread_local std::string g_cuda_error;
std::atomic<long long> g_launches{0};

constexpr int kBlock = 256;
// Block sizes of the gradient kernels, measured: node values (one thread per
// node over ~24 dependent loads) gain from 512-thread blocks, the face sums
// from 128-thread ones (0.137 -> 0.117 and 0.250 -> 0.240 ms at 64^3).
constexpr int kNodeBlock = 512;
constexpr int kGradBlock = 128;
constexpr int kGradBlockMax = 256;  // the largest block mfg_autotune tries
constexpr int kNormBlocks = 1184;  // 8 x 148 SMs, fixed so the norm reduction order is fixed
constexpr int kSegBlocks = 32;     // blocks per case of the batched norm reduction

#define MFG_CUDA(call)                                                            \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      g_cuda_error = std::string(#call) + ": " + cudaGetErrorString(e_);          \
      return MFG_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

// The same inside a context build: the partly built context is released.
#define MFG_CUDA_OR(call)                                                         \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      g_cuda_error = std::string(#call) + ": " + cudaGetErrorString(e_);          \
      return fail(MFG_ERR_CUDA);                                                  \
    }                                                                             \
  } while (0)

inline int grid_for(int64_t n, int block = kBlock) {
  return (int)std::max<int64_t>(1, (n + block - 1) / block);
}
// Lanes per cell of the face gather for cells of at most max_slots faces.
inline int gather_lanes_for(int32_t max_slots) {
  return max_slots <= 4 ? 4 : (max_slots <= 8 ? 8 : 0);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Scatter SoA q (5 blocks of n) into both state buffers and derive per-cell
// quantities.
__global__ void k_upload_q(const double *__restrict__ soa, double *__restrict__ qa,
                           double *__restrict__ qb, float *__restrict__ q4a,
                           float *__restrict__ q4b, int64_t n, Params P0, Cases cs) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double q[Q_STRIDE];
  for (int k = 0; k < 5; k++) q[k] = soa[k * n + i];
  cell_props(q, params_of(P0, cs, i));
  store_q(qa, i, q);
  if (qb) store_q(qb, i, q);
  if (q4a) store_q4(q4a, i, q);
  if (q4b) store_q4(q4b, i, q);
}

__global__ void k_download_rec(const double *__restrict__ rec, double *__restrict__ soa,
                               int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = 0; k < 5; k++) soa[k * n + i] = rec[i * Q_STRIDE + k];
}

// SetGhostVariables (load_grid.cpp:953-1212), inviscid steady case: the
// ghost state of every boundary face from its inner cell's current state,
// one thread per boundary face, written into both state buffers (which keep
// identical ghost rows) and, in the mixed form, both single-precision
// copies.  The same expressions as the reference; its only libm calls whose
// arguments change with the flow are the two pow of the subsonic far-field
// branches, which here are CUDA's pow.
__global__ void k_ghost_bc(int32_t G, int32_t C, const FaceRec *__restrict__ faces,
                           const int32_t *__restrict__ bctype, double *__restrict__ qa,
                           double *__restrict__ qb, float *__restrict__ q4a,
                           float *__restrict__ q4b, Params P0, Cases cs) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G) return;
  const int type = bctype[i];
  if (type == MFG_BC_INTERFACE) return;  // :1030-1031
  const FaceRec fr = faces[i];
  const int32_t c1 = fr.c1;
  const int64_t c2 = (int64_t)C + i;
  const Params P = params_of(P0, cs, c1);
  const double xfn = fr.nx, yfn = fr.ny, zfn = fr.nz;
  double q1[Q_STRIDE], g[Q_STRIDE];
  load_q(qa, c1, q1);
  load_q(qa, c2, g);  // kept by types the reference does not handle
  const double gam = P.gam, p_bar = P.p_bar;
  switch (type) {
    case MFG_BC_WALL:
    case MFG_BC_SYMM: {  // :1036-1044, :1084-1095 (same assignments)
      g[4] = q1[4];
      g[0] = q1[0];
      const double vn = 2. * (xfn * q1[1] + yfn * q1[2] + zfn * q1[3]);
      g[1] = q1[1] - vn * xfn;
      g[2] = q1[2] - vn * yfn;
      g[3] = q1[3] - vn * zfn;
      break;
    }
    case MFG_BC_FAR_FIELD: {  // :1097-1194
      const double um = P.ref[1], vm = P.ref[2], wm = P.ref[3];
      const double up = q1[1], vp = q1[2], wp = q1[3];
      const double rhom = P.ref[0], pm = P.ref[4] + p_bar;
      const double rhop = q1[0], pp = q1[4] + p_bar;
      const double vnm = xfn * um + yfn * vm + zfn * wm;
      const double vnp = xfn * up + yfn * vp + zfn * wp;
      const double cm = sqrt(gam * pm / rhom);
      const double cp = sqrt(gam * pp / rhop);
      const double riemm = vnm - 2. * cm / (gam - 1.);
      const double riemp = vnp + 2. * cp / (gam - 1.);
      const double vnb = 0.5 * (riemp + riemm);
      const double cb = 0.25 * (riemp - riemm) * (gam - 1.);
      if (fabs(vnb / cb) > 1.) {
        if (vnb <= 0.0) {
          g[0] = rhom;
          g[1] = um;
          g[2] = vm;
          g[3] = wm;
          g[4] = pm;
        } else {
          g[0] = rhop;
          g[1] = up;
          g[2] = vp;
          g[3] = wp;
          g[4] = pp;
        }
      } else {
        const double rela_vnb = vnb / P.uvw_norm;
        const double eps_of_farfield_vn = 0.0;
        if (rela_vnb <= -eps_of_farfield_vn) {
          const double vtx = um - vnm * xfn, vty = vm - vnm * yfn, vtz = wm - vnm * zfn;
          g[0] = pow((cb * cb / (P.entr_m * gam)), double(1. / (gam - 1.)));
          g[1] = vtx + vnb * xfn;
          g[2] = vty + vnb * yfn;
          g[3] = vtz + vnb * zfn;
          g[4] = cb * cb * g[0] / gam;
        } else if (rela_vnb > eps_of_farfield_vn) {
          const double vtx = up - vnp * xfn, vty = vp - vnp * yfn, vtz = wp - vnp * zfn;
          const double entr = pp / pow(rhop, gam);
          g[0] = pow((cb * cb / (entr * gam)), double(1. / (gam - 1.)));
          g[1] = vtx + vnb * xfn;
          g[2] = vty + vnb * yfn;
          g[3] = vtz + vnb * zfn;
          g[4] = cb * cb * g[0] / gam;
        } else {
          g[0] = 0.5 * (rhop + rhom);
          g[1] = 0.5 * (up + um);
          g[2] = 0.5 * (vp + vm);
          g[3] = 0.5 * (wp + wm);
          g[4] = 0.5 * (pp + pm);
        }
      }
      g[0] = 2 * g[0] - rhop;
      g[1] = 2 * g[1] - up;
      g[2] = 2 * g[2] - vp;
      g[3] = 2 * g[3] - wp;
      g[4] = 2 * g[4] - pp;
      g[4] -= p_bar;
      break;
    }
    default:
      break;  // the reference reports "Error in SetGhostVariables 001" and goes on
  }
  g[0] = smax(g[0], P.rho_min);  // :1204-1208
  g[0] = smin(g[0], P.rho_max);
  g[4] = smax(g[4], P.p_min);
  g[4] = smin(g[4], P.p_max);
  cell_props(g, P);
  store_q(qa, c2, g);
  store_q(qb, c2, g);
  if (q4a) store_q4(q4a, c2, g);
  if (q4b) store_q4(q4b, c2, g);
}

// Interior rows of an increment array set to the "not yet written" sentinel.
__global__ void k_arm_sentinel(int32_t C, double *__restrict__ dq8) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < C) store_sentinel(dq8, c);
}

// End of a face gather, one cell per thread: the running dt extrema
// (compute_timestep.cpp:914-918) and the block partial sums of res^2 for the
// residual norm, reduced in a fixed order.
template <bool FLUX, bool DT>
__device__ __forceinline__ void gather_epilogue(bool live, int32_t cse, double dtc,
                                                const double *r,
                                                unsigned long long *__restrict__ dt_ext,
                                                double *__restrict__ norm_part) {
  if (DT) {
    // dt >= 0, so the bit patterns order like the values
    unsigned long long mx = live ? dbits(dtc) : 0ull;
    unsigned long long mn = live ? dbits(dtc) : ~0ull;
    // one atomic pair per warp when the warp's cells share a case (the
    // extrema are per case), else one per cell
    const int32_t c0 = __shfl_sync(0xffffffffu, cse, 0);
    if (__all_sync(0xffffffffu, !live || cse == c0)) {
      for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      }
      if ((threadIdx.x & 31) == 0) {
        atomicMax(dt_ext + 2 * c0, mx);
        atomicMin(dt_ext + 2 * c0 + 1, mn);
      }
    } else if (live) {
      atomicMax(dt_ext + 2 * cse, mx);
      atomicMin(dt_ext + 2 * cse + 1, mn);
    }
  }
  if (FLUX && norm_part) {
    __shared__ double sh[kBlock / 32][5];
    double s2[5];
    for (int k = 0; k < 5; k++) s2[k] = live ? r[k] * r[k] : 0.0;
    for (int o = 16; o > 0; o >>= 1)
      for (int k = 0; k < 5; k++) s2[k] += __shfl_down_sync(0xffffffffu, s2[k], o);
    if ((threadIdx.x & 31) == 0)
      for (int k = 0; k < 5; k++) sh[threadIdx.x >> 5][k] = s2[k];
    __syncthreads();
    if (threadIdx.x < 5) {
      double acc = 0.0;
      for (int wgi = 0; wgi < kBlock / 32; wgi++) acc += sh[wgi][threadIdx.x];
      norm_part[(int64_t)blockIdx.x * 5 + threadIdx.x] = acc;
    }
  }
}

// A face's row of the per-face flux array: the five fluxes and CellIsMG's
// pressure test of its two cells (1.0 when |p2 - p1| / (p2 + p1 + 2 p_bar)
// exceeds 0.1, compute_timestep.cpp:1009-1340; the expression is symmetric
// in the two sides, so either cell's gather reads the same outcome).
constexpr int kFluxRow = 6;
// Cells per slice of the sliced slot records (one warp).
constexpr int kSlice = 32;
// RN(1/3), folded by the compiler: the reciprocal of a triangle's node count.
constexpr double kRcp3 = 1.0 / 3.0;
// The sliced slot records of the one-thread-per-cell kernels, each holding
// what its kernel reads (48 bytes, so that a warp reads 1.5 KB per face
// position).  The face gathers': the normal, area, dn, the neighbour, and
// the face with the side in bit 31 (set where the cell is the face's second
// cell).
struct __align__(16) GatherSlot {
  double nx, ny, nz, area, dn;
  int32_t nb;
  uint32_t face_c2;
};
// The gradient's: the normal, area, flags and n0..n2 = a triangle's nodes
// (SLOT_TRI), else n0 = the ghost (a boundary face averaged with its ghost)
// or the face (its nodes through the face -> node lists).
struct __align__(16) GradSlot {
  double nx, ny, nz, area;
  int32_t n0, n1, n2, flags;
};
static_assert(sizeof(GatherSlot) == 48 && sizeof(GradSlot) == 48, "sliced slot records");
// One entry of a node's list (a cell, or a boundary face), with its weight.
struct __align__(16) NodeEnt {
  int32_t src, pad;
  double w;
};
static_assert(kBlock % kSlice == 0, "blocks hold whole slices");

// Per-cell face gather: Roe flux into the residual, local time step with
// CellIsMG and LimitTimeStep, and the LU-SGS diagonal.  One thread per cell,
// faces in ascending order (see the file header for why that is exact).
// Resident blocks of the face gathers and the face flux (register caps).
#ifndef MFG_GATHER_MINB
#define MFG_GATHER_MINB 3
#endif
#ifndef MFG_FLUX_MINB
#define MFG_FLUX_MINB 3
#endif

template <bool FLUX, bool DT, bool DIAG, bool PRE>
__device__ __forceinline__ void face_gather_cell(
    int32_t c, int32_t C, const int32_t *__restrict__ cptr, const GatherSlot *__restrict__ gslots,
    const int32_t *__restrict__ sptr32, const double *__restrict__ q8, const double *__restrict__ vol, double *__restrict__ res,
    int res_zero, double *__restrict__ dt, double *__restrict__ diag,
    const double *__restrict__ cfl_tab, const int32_t *__restrict__ iter_counter, double cfl_arg,
    const Params &P0, unsigned long long *__restrict__ dt_ext, double *__restrict__ norm_part,
    const Cases &cs, const double *__restrict__ fflux, int32_t F) {
  const bool live = c < C;
  const int32_t cse = live ? case_of(cs, c) : 0;
  // the parameters the gather reads, field by field: a batch's case table
  // or the kernel argument
  const Params *Pc = (live && cs.P) ? cs.P + cse : nullptr;
  const double p_bar = Pc ? Pc->p_bar : P0.p_bar;
  const double lhs_omga = Pc ? Pc->lhs_omga : P0.lhs_omga;
  double qc[Q_STRIDE];
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double dtc = 0.0;
  if (live) {
    load_q(q8, c, qc);
    if (FLUX && !res_zero)
      for (int k = 0; k < 5; k++) r[k] = res[(int64_t)k * C + c];
    const int32_t ns = __ldg(cptr + c + 1) - __ldg(cptr + c);
    const GatherSlot *sl = gslots + __ldg(sptr32 + c / kSlice) + c % kSlice;  // sliced
    double dtl = kBig;
    int det = 1;
    // Diag's terms 0.5 area eig lhs_omga of the first four faces, formed with
    // the time step's eigenvalue (the same expression), so that Diag's pass
    // reads no slot record again for them
    double dg0 = 0.0, dg1 = 0.0, dg2 = 0.0, dg3 = 0.0;
    for (int32_t j = 0; j < ns; j++) {
      const GatherSlot sr = sl[(int64_t)j * kSlice];
      if (FLUX || DT) {
        // the neighbour's state: its pressure for CellIsMG and, without the
        // per-face rows, the flux; with them (PRE) the row holds both
        double qn[Q_STRIDE], mgf = 0.0;
        if (!PRE) load_q(q8, sr.nb, qn);
        if (FLUX) {
          double f[5];
          if (PRE) {  // the face's flux, computed once by k_face_flux
            const double2 *row =
                reinterpret_cast<const double2 *>(fflux + (int64_t)(sr.face_c2 & 0x7FFFFFFFu) * kFluxRow);
            const double2 a = __ldg(row), b = __ldg(row + 1), e = __ldg(row + 2);
            f[0] = a.x; f[1] = a.y; f[2] = b.x; f[3] = b.y; f[4] = e.x;
            mgf = e.y;
          } else if (sr.face_c2 >> 31) {
            roe_flux(qn, qc, sr.nx, sr.ny, sr.nz, sr.area, params_of(P0, cs, c), f);
          } else {
            roe_flux(qc, qn, sr.nx, sr.ny, sr.nz, sr.area, params_of(P0, cs, c), f);
          }
          if (sr.face_c2 >> 31) {
            for (int k = 0; k < 5; k++) r[k] += f[k];
          } else {
            for (int k = 0; k < 5; k++) r[k] -= f[k];
          }
        }
        if (DT) {
          double vn = qc[1] * sr.nx + qc[2] * sr.ny + qc[3] * sr.nz;
          vn = fabs(vn);
          const double eigv = vn + qc[Q_A];
          dtl = smin(dtl, sr.dn / eigv);
          if (DIAG) {
            const double t = 0.5 * sr.area * eigv * lhs_omga;
            dg0 = j == 0 ? t : dg0;
            dg1 = j == 1 ? t : dg1;
            dg2 = j == 2 ? t : dg2;
            dg3 = j == 3 ? t : dg3;
          }
          // CellIsMG: |p2-p1| and p2+p1 are symmetric in the two sides.
          if (PRE) {
            if (mgf != 0.0) det = 0;
          } else {
            const double dp = fabs(qn[4] - qc[4]) / (qn[4] + qc[4] + p_bar + p_bar);
            if (dp > 0.1) det = 0;
          }
        }
      }
    }
    if (DT) {
      const double cfl =
          cfl_tab ? cfl_tab[(int64_t)(*iter_counter) * max(cs.ncase, 1) + cse] : cfl_arg;
      const double cfl_min = 0.5 * cfl;
      dtc = dtl * local_cfl_pb(qc[4], det, cfl, cfl_min, Pc ? Pc->p_break : P0.p_break,
                               Pc ? Pc->p_min : P0.p_min);
      dt[c] = dtc;
    }
    if (DIAG) {
      const double dtv = DT ? dtc : dt[c];
      double d = vol[c] / dtv;
      int32_t j0 = 0;
      if (DT) {
        if (ns > 0) d += dg0;
        if (ns > 1) d += dg1;
        if (ns > 2) d += dg2;
        if (ns > 3) d += dg3;
        j0 = ns < 4 ? ns : 4;
      }
      for (int32_t j = j0; j < ns; j++) {
        const GatherSlot sr = sl[(int64_t)j * kSlice];
        double vn = qc[1] * sr.nx + qc[2] * sr.ny + qc[3] * sr.nz;
        vn = fabs(vn);
        const double eig = vn + qc[Q_A];
        d += 0.5 * sr.area * eig * lhs_omga;
      }
      diag[c] = d;
    }
    if (FLUX)
      for (int k = 0; k < 5; k++) res[(int64_t)k * C + c] = r[k];
  }
  gather_epilogue<FLUX, DT>(live, cse, dtc, r, dt_ext, norm_part);
}

template <bool FLUX, bool DT, bool DIAG, bool PRE, int MINB = MFG_GATHER_MINB>
__global__ void __launch_bounds__(kBlock, MINB)
k_face_gather(int32_t C, const int32_t *__restrict__ cptr, const GatherSlot *__restrict__ gslots,
              const int32_t *__restrict__ sptr32, const double *__restrict__ q8,
              const double *__restrict__ vol,
              double *__restrict__ res, int res_zero, double *__restrict__ dt,
              double *__restrict__ diag, const double *__restrict__ cfl_tab,
              const int32_t *__restrict__ iter_counter, double cfl_arg, Params P0,
              unsigned long long *__restrict__ dt_ext, double *__restrict__ norm_part, Cases cs,
              const double *__restrict__ fflux, int32_t F) {
  face_gather_cell<FLUX, DT, DIAG, PRE>(blockIdx.x * blockDim.x + threadIdx.x, C, cptr, gslots,
                                        sptr32, q8, vol, res, res_zero, dt, diag, cfl_tab, iter_counter,
                                        cfl_arg, P0, dt_ext, norm_part, cs, fflux, F);
}

// Mixed form of the face gather: the Roe flux in the mixed form above; the
// local time step and its CellIsMG switch (a discrete decision, kept in FP64
// so that both forms take it alike), the Diag terms and all sums in FP64 in
// the same face order.
template <bool FLUX, bool DT, bool DIAG, bool PRE, int MINB = MFG_GATHER_MINB>
__global__ void __launch_bounds__(kBlock, MINB)
k_face_gather_mx(int32_t C, const int32_t *__restrict__ cptr,
                 const GatherSlot *__restrict__ gslots, const int32_t *__restrict__ sptr32,
                 const double *__restrict__ q8, const double *__restrict__ vol,
                 double *__restrict__ res, int res_zero, double *__restrict__ dt,
                 double *__restrict__ diag, const double *__restrict__ cfl_tab,
                 const int32_t *__restrict__ iter_counter, double cfl_arg, Params P0,
                 unsigned long long *__restrict__ dt_ext, double *__restrict__ norm_part,
                 Cases cs, const double *__restrict__ fflux, int32_t F) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = c < C;
  const int32_t cse = live ? case_of(cs, c) : 0;
  const Params *Pc = (live && cs.P) ? cs.P + cse : nullptr;  // as in face_gather_cell
  const double p_bar = Pc ? Pc->p_bar : P0.p_bar;
  const double lhs_omga = Pc ? Pc->lhs_omga : P0.lhs_omga;
  double qd[Q_STRIDE];
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double dtc = 0.0;
  if (live) {
    load_q(q8, c, qd);
    if (FLUX && !res_zero)
      for (int k = 0; k < 5; k++) r[k] = res[(int64_t)k * C + c];
    const int32_t ns = __ldg(cptr + c + 1) - __ldg(cptr + c);
    const GatherSlot *sl = gslots + __ldg(sptr32 + c / kSlice) + c % kSlice;  // sliced
    double dtl = kBig;
    int det = 1;
    double dg0 = 0.0, dg1 = 0.0, dg2 = 0.0, dg3 = 0.0;  // as in face_gather_cell
    for (int32_t j = 0; j < ns; j++) {
      const GatherSlot sr = sl[(int64_t)j * kSlice];
      if (FLUX || DT) {
        double qn[Q_STRIDE], mgf = 0.0;
        if (!PRE) load_q(q8, sr.nb, qn);
        if (FLUX) {
          double f[5];
          if (PRE) {  // the face's flux, computed once by k_face_flux
            const double2 *row =
                reinterpret_cast<const double2 *>(fflux + (int64_t)(sr.face_c2 & 0x7FFFFFFFu) * kFluxRow);
            const double2 a = __ldg(row), b = __ldg(row + 1), e = __ldg(row + 2);
            f[0] = a.x; f[1] = a.y; f[2] = b.x; f[3] = b.y; f[4] = e.x;
            mgf = e.y;
          } else if (sr.face_c2 >> 31) {
            const Params P = params_of(P0, cs, c);
            roe_flux_mx(qn, qd, sr.nx, sr.ny, sr.nz, sr.area, P, flux_params<float>(P), f);
          } else {
            const Params P = params_of(P0, cs, c);
            roe_flux_mx(qd, qn, sr.nx, sr.ny, sr.nz, sr.area, P, flux_params<float>(P), f);
          }
          if (sr.face_c2 >> 31) {
            for (int k = 0; k < 5; k++) r[k] += f[k];
          } else {
            for (int k = 0; k < 5; k++) r[k] -= f[k];
          }
        }
        if (DT) {  // as in k_face_gather
          double vn = qd[1] * sr.nx + qd[2] * sr.ny + qd[3] * sr.nz;
          vn = fabs(vn);
          const double eigv = vn + qd[Q_A];
          dtl = smin(dtl, sr.dn / eigv);
          if (DIAG) {
            const double t = 0.5 * sr.area * eigv * lhs_omga;
            dg0 = j == 0 ? t : dg0;
            dg1 = j == 1 ? t : dg1;
            dg2 = j == 2 ? t : dg2;
            dg3 = j == 3 ? t : dg3;
          }
          if (PRE) {
            if (mgf != 0.0) det = 0;
          } else {
            const double dp = fabs(qn[4] - qd[4]) / (qn[4] + qd[4] + p_bar + p_bar);
            if (dp > 0.1) det = 0;
          }
        }
      }
    }
    if (DT) {
      const double cfl =
          cfl_tab ? cfl_tab[(int64_t)(*iter_counter) * max(cs.ncase, 1) + cse] : cfl_arg;
      dtc = dtl * local_cfl_pb(qd[4], det, cfl, 0.5 * cfl, Pc ? Pc->p_break : P0.p_break,
                               Pc ? Pc->p_min : P0.p_min);
      dt[c] = dtc;
    }
    if (DIAG) {
      const double dtv = DT ? dtc : dt[c];
      double d = vol[c] / dtv;
      int32_t j0 = 0;
      if (DT) {
        if (ns > 0) d += dg0;
        if (ns > 1) d += dg1;
        if (ns > 2) d += dg2;
        if (ns > 3) d += dg3;
        j0 = ns < 4 ? ns : 4;
      }
      for (int32_t j = j0; j < ns; j++) {
        const GatherSlot sr = sl[(int64_t)j * kSlice];
        double vn = qd[1] * sr.nx + qd[2] * sr.ny + qd[3] * sr.nz;
        vn = fabs(vn);
        d += 0.5 * sr.area * (vn + qd[Q_A]) * lhs_omga;
      }
      diag[c] = d;
    }
    if (FLUX)
      for (int k = 0; k < 5; k++) res[(int64_t)k * C + c] = r[k];
  }
  gather_epilogue<FLUX, DT>(live, cse, dtc, r, dt_ext, norm_part);
}

// Face gather with one lane per (cell, face) slot: L lanes per cell (L at
// least the cell's slot count), so that a cell's slot records and face rows
// are loaded side by side instead of one after another.  The per-cell
// results are folds over the slots in ascending face order passed from lane
// to lane: the residual r := r - F_f (r + F_f where the cell is the face's
// second cell; a difference is the sum with the negated term, exactly), the
// time step min(dt, dn_f / eig_f), CellIsMG's switch, then Diag := vol / dt
// + sum 0.5 area_f eig_f lhs_omga -- the operations and order of the
// one-thread gather, so the same bits.  The flux comes from the per-face
// rows (FLUX, either precision's flux kernel); without them (the time step
// alone) CellIsMG reads the neighbour's pressure.
template <int L>
__device__ __forceinline__ double lane_prev(double x) {
  return __shfl_up_sync(0xffffffffu, x, 1, L);
}

template <int L, bool FLUX, bool DT, bool DIAG, int MINB = MFG_GATHER_MINB>
__global__ void __launch_bounds__(kBlock, MINB)
k_face_gather_lanes(int32_t C, const int32_t *__restrict__ cptr,
                    const SlotRec *__restrict__ slots, const double *__restrict__ q8,
                    const double *__restrict__ vol, double *__restrict__ res, int res_zero,
                    double *__restrict__ dt, double *__restrict__ diag,
                    const double *__restrict__ cfl_tab, const int32_t *__restrict__ iter_counter,
                    double cfl_arg, Params P0, unsigned long long *__restrict__ dt_ext,
                    double *__restrict__ norm_part, Cases cs, const double *__restrict__ fflux) {
  static_assert((L & (L - 1)) == 0 && L >= 2 && L <= 32 && kBlock % L == 0, "lanes per cell");
  const int64_t cl = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / L;
  const bool live = cl < C;
  const int32_t c = live ? (int32_t)cl : 0;
  const int lane = threadIdx.x & (L - 1);
  const bool last = lane == L - 1;
  int32_t s0 = 0, ns = 0;
  if (live) {
    s0 = __ldg(cptr + c);
    ns = __ldg(cptr + c + 1) - s0;
  }
  const bool has = live && lane < ns;
  const int32_t cse = live ? case_of(cs, c) : 0;
  const Params P = live ? params_of(P0, cs, c) : P0;
  double qc[Q_STRIDE];
  load_q(q8, c, qc);
  // this lane's slot
  double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double dtt = 0.0, dgt = 0.0;
  int bad = 0;
  if (has) {
    const SlotRec sr = slots[s0 + lane];
    if (FLUX) {
      const double2 *row = reinterpret_cast<const double2 *>(fflux + (int64_t)sr.face * kFluxRow);
      const double2 a = __ldg(row), b = __ldg(row + 1), e = __ldg(row + 2);
      const double f[5] = {a.x, a.y, b.x, b.y, e.x};
      const bool plus = (sr.flags & SLOT_IS_C2) != 0;
#pragma unroll
      for (int k = 0; k < 5; k++) t[k] = plus ? f[k] : -f[k];
      if (DT) bad = e.y != 0.0;
    }
    if (DT || DIAG) {
      double vn = qc[1] * sr.nx + qc[2] * sr.ny + qc[3] * sr.nz;
      vn = fabs(vn);
      const double eig = vn + qc[Q_A];
      if (DT) {
        dtt = sr.dn / eig;
        if (!FLUX) {
          const double pn = __ldg(q8 + (int64_t)sr.nb * Q_STRIDE + 4);
          const double dp = fabs(pn - qc[4]) / (pn + qc[4] + P.p_bar + P.p_bar);
          bad = dp > 0.1;
        }
      }
      if (DIAG) dgt = 0.5 * sr.area * eig * P.lhs_omga;
    }
  }
  // the folds, lane 0 from the initial values
  double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double dtl = kBig;
  if (lane == 0) {
    if (FLUX && live && !res_zero)
#pragma unroll
      for (int k = 0; k < 5; k++) r[k] = res[(int64_t)k * C + c];
    if (has) {
      if (FLUX)
#pragma unroll
        for (int k = 0; k < 5; k++) r[k] += t[k];
      if (DT) dtl = smin(dtl, dtt);
    }
  }
#pragma unroll
  for (int j = 1; j < L; j++) {
    double pr[5], pd = 0.0;
    if (FLUX)
#pragma unroll
      for (int k = 0; k < 5; k++) pr[k] = lane_prev<L>(r[k]);
    if (DT) pd = lane_prev<L>(dtl);
    if (lane == j) {
      if (FLUX)
#pragma unroll
        for (int k = 0; k < 5; k++) r[k] = has ? pr[k] + t[k] : pr[k];
      if (DT) dtl = has ? smin(pd, dtt) : pd;
    }
  }
  double dtc = 0.0;
  if (DT) {
#pragma unroll
    for (int o = 1; o < L; o <<= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o, L);
    if (last && live) {
      const double cfl =
          cfl_tab ? cfl_tab[(int64_t)(*iter_counter) * max(cs.ncase, 1) + cse] : cfl_arg;
      const double cfl_min = 0.5 * cfl;
      dtc = dtl * local_cfl(qc[4], bad ? 0 : 1, cfl, cfl_min, P);
      dt[c] = dtc;
    }
  }
  if (DIAG) {
    double dtv;
    if (DT)
      dtv = __shfl_sync(0xffffffffu, dtc, L - 1, L);
    else
      dtv = live ? dt[c] : 1.0;
    double d = 0.0;
    if (lane == 0 && live) {
      d = vol[c] / dtv;
      if (has) d += dgt;
    }
#pragma unroll
    for (int j = 1; j < L; j++) {
      const double pd = lane_prev<L>(d);
      if (lane == j) d = has ? pd + dgt : pd;
    }
    if (last && live) diag[c] = d;
  }
  if (FLUX && last && live)
#pragma unroll
    for (int k = 0; k < 5; k++) res[(int64_t)k * C + c] = r[k];
  gather_epilogue<FLUX, DT>(live && last, cse, dtc, r, dt_ext, norm_part);
}

// Second-order face state (RECON): q + phi * grad(q) . (x_f - x_c) for an
// inner cell, the ghost's own state otherwise (the reference's switch
// `order`, para_field_global.cpp:100, has no implementation behind it, so
// this is this library's own reconstruction: linear from the Green-Gauss
// gradient of the state the face kernel reads, limited per cell).
// gflag (a partitioned mesh at second order): the ghosts that hold another
// part's cell, with that cell's gradient, limiter and centroid, reconstruct
// as the cell would; other ghosts stay first order.
__device__ __forceinline__ void reconstruct(double *q, int32_t c, int32_t C, int64_t n,
                                            const Cen &fc, const Cen *__restrict__ ccen,
                                            const double *__restrict__ dqdx,
                                            const double *__restrict__ dqdy,
                                            const double *__restrict__ dqdz,
                                            const double *__restrict__ phi,
                                            const int32_t *__restrict__ gflag) {
  if (c >= C && !(gflag && gflag[c - C])) return;
  const Cen cc = ccen[c];
  const double rx = fc.x - cc.x, ry = fc.y - cc.y, rz = fc.z - cc.z;
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const int64_t k = (int64_t)v * n + c;
    const double d = dqdx[k] * rx + dqdy[k] * ry + dqdz[k] * rz;
    q[v] += (phi ? phi[(int64_t)v * n + c] : 1.0) * d;
  }
}

// RoeFlux_noprec once per face (the reference's own face loop,
// cal_flux.cpp:84-192), from q[c1] and q[c2] with the stored normal, into
// row f of fflux[F][kFluxRow]; the face gathers then add each face's flux to
// its cells in ascending face order.  The arguments are those the per-cell form passes
// from either side, so the sums are the same bits with half the flux work.
// RECON:
// the face states reconstructed to second order first (a face whose
// reconstructed density or absolute pressure is not positive keeps its
// first-order states).
template <bool MX, bool RECON, int MINB = MFG_FLUX_MINB>
__global__ void __launch_bounds__(kBlock, MINB)
k_face_flux(int32_t F, const FaceRec *__restrict__ faces, const double *__restrict__ q8,
            Params P0, Cases cs, double *__restrict__ fflux, int32_t C, int64_t n,
            const Cen *__restrict__ fcen, const Cen *__restrict__ ccen,
            const double *__restrict__ dqdx, const double *__restrict__ dqdy,
            const double *__restrict__ dqdz, const double *__restrict__ phi,
            const int32_t *__restrict__ gflag) {
  const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const FaceRec fr = faces[f];
  const Params P = params_of(P0, cs, fr.c1);
  double ql[Q_STRIDE], qr[Q_STRIDE], fl[5];
  load_q_w(q8, fr.c1, ql);
  load_q_w(q8, fr.c2, qr);
  // CellIsMG's test of the two cells' states (first order, as the gathers)
  const double dp = fabs(qr[4] - ql[4]) / (qr[4] + ql[4] + P.p_bar + P.p_bar);
  const double mg = dp > 0.1 ? 1.0 : 0.0;
  if (RECON) {
    double al[Q_STRIDE], ar[Q_STRIDE];
#pragma unroll
    for (int v = 0; v < Q_STRIDE; v++) {
      al[v] = ql[v];
      ar[v] = qr[v];
    }
    const Cen fc = fcen[f];
    reconstruct(al, fr.c1, C, n, fc, ccen, dqdx, dqdy, dqdz, phi, gflag);
    reconstruct(ar, fr.c2, C, n, fc, ccen, dqdx, dqdy, dqdz, phi, gflag);
    if (al[0] > 0.0 && ar[0] > 0.0 && al[4] + P.p_bar > 0.0 && ar[4] + P.p_bar > 0.0) {
      cell_props(al, P);
      cell_props(ar, P);
#pragma unroll
      for (int v = 0; v < Q_STRIDE; v++) {
        ql[v] = al[v];
        qr[v] = ar[v];
      }
    }
  }
  if (MX)
    roe_flux_mx(ql, qr, fr.nx, fr.ny, fr.nz, fr.area, P, flux_params<float>(P), fl);
  else
    roe_flux(ql, qr, fr.nx, fr.ny, fr.nz, fr.area, P, fl);
  double2 *row = reinterpret_cast<double2 *>(fflux + (int64_t)f * kFluxRow);
  row[0] = make_double2(fl[0], fl[1]);
  row[1] = make_double2(fl[2], fl[3]);
  row[2] = make_double2(fl[4], mg);
}

// Per-cell limiter of the reconstruction, per variable: the minimum over the
// cell's faces of the bound on the face's extrapolated change that keeps it
// within the range of the cell and its face neighbours (ghosts included) --
// Barth and Jespersen (AIAA 89-0366) -- or Venkatakrishnan's smooth form of
// the same bound (AIAA 93-0880; eps^2 = (K h)^3, h = vol^(1/3)).
template <bool VENKAT>
__global__ void __launch_bounds__(kBlock)
k_limiter(int32_t C, int64_t n, const int32_t *__restrict__ cptr,
          const SlotRec *__restrict__ slots, const double *__restrict__ q8,
          const double *__restrict__ dqdx, const double *__restrict__ dqdy,
          const double *__restrict__ dqdz, const Cen *__restrict__ fcen,
          const Cen *__restrict__ ccen, double venkat_k, double *__restrict__ phi) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double qc[Q_STRIDE], qmin[5], qmax[5], lim[5], gx[5], gy[5], gz[5];
  load_q(q8, c, qc);
  for (int v = 0; v < 5; v++) {
    qmin[v] = qc[v];
    qmax[v] = qc[v];
    lim[v] = 1.0;
    const int64_t k = (int64_t)v * n + c;
    gx[v] = dqdx[k];
    gy[v] = dqdy[k];
    gz[v] = dqdz[k];
  }
  const int32_t s0 = cptr[c], s1 = cptr[c + 1];
  for (int32_t s = s0; s < s1; s++) {
    double qn[Q_STRIDE];
    load_q(q8, slots[s].nb, qn);
    for (int v = 0; v < 5; v++) {
      qmin[v] = fmin(qmin[v], qn[v]);
      qmax[v] = fmax(qmax[v], qn[v]);
    }
  }
  const Cen cc = ccen[c];
  const double eps2 = VENKAT ? (venkat_k * cc.h) * (venkat_k * cc.h) * (venkat_k * cc.h) : 0.0;
  for (int32_t s = s0; s < s1; s++) {
    const Cen fc = fcen[slots[s].face];
    const double rx = fc.x - cc.x, ry = fc.y - cc.y, rz = fc.z - cc.z;
    for (int v = 0; v < 5; v++) {
      const double d2 = gx[v] * rx + gy[v] * ry + gz[v] * rz;
      if (d2 == 0.0) continue;
      const double d1 = (d2 > 0.0 ? qmax[v] : qmin[v]) - qc[v];
      double psi;
      if (VENKAT) {
        const double a = d1 * d1 + eps2;
        psi = (a + 2.0 * d2 * d1) / (a + 2.0 * d2 * d2 + d1 * d2);
      } else {
        psi = fmin(1.0, d1 / d2);
      }
      lim[v] = fmin(lim[v], psi);
    }
  }
  for (int v = 0; v < 5; v++) phi[(int64_t)v * n + c] = fmax(0.0, fmin(1.0, lim[v]));
}

// Centroids for the reconstruction: faces and cells (with h = vol^(1/3)).
__global__ void k_centroids(int32_t F, int64_t n, const double *__restrict__ xfc,
                            const double *__restrict__ yfc, const double *__restrict__ zfc,
                            const double *__restrict__ xcc, const double *__restrict__ ycc,
                            const double *__restrict__ zcc, const double *__restrict__ vol,
                            Cen *__restrict__ fcen, Cen *__restrict__ ccen) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < F) fcen[i] = Cen{xfc[i], yfc[i], zfc[i], 0.0};
  if (i < n) ccen[i] = Cen{xcc[i], ycc[i], zcc[i], cbrt(fabs(vol[i]))};
}

// LimitTimeStep's ratio clamp (compute_timestep.cpp:929-944), per case.
__global__ void k_dt_clamp(int32_t C, double *__restrict__ dt,
                           const unsigned long long *__restrict__ dt_ext, Params P0, Cases cs) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const int32_t cse = case_of(cs, c);
  const double ratio_dtmax = params_of(P0, cs, c).ratio_dtmax;
  const double dt_max = __longlong_as_double((long long)dt_ext[2 * cse]);
  const double dt_min = __longlong_as_double((long long)dt_ext[2 * cse + 1]);
  const double ratio_max = dt_max / dt_min;
  if (!(ratio_max > ratio_dtmax)) return;
  const double lim = ratio_dtmax * dt_min;
  if (dt[c] > lim) dt[c] = lim;
}

// Forward (lower) sweep of one level: cells [l0, l1) of the level order.
// Increments of the forward sweep go to dqf, those of the backward sweep to
// dqb (the final DQ); each sweep re-arms the other array's row of its cell
// with the sentinel (see mfg_kernels.cuh), the protocol the persistent
// sweeps rely on.  In the fused path the ratio clamp of LimitTimeStep is
// applied here: a cell whose dt exceeds the limit gets the limited dt and
// its Diag rebuilt.
__device__ __forceinline__ void clamp_diag(int32_t c, const double *qc, double &dg,
                                           const Params &P, double *__restrict__ dt,
                                           const unsigned long long *__restrict__ dt_ext,
                                           const int32_t *__restrict__ cptr,
                                           const SlotRec *__restrict__ slots,
                                           const double *__restrict__ vol,
                                           double *__restrict__ diag) {
  const double dt_max = __longlong_as_double((long long)dt_ext[0]);
  const double dt_min = __longlong_as_double((long long)dt_ext[1]);
  if (dt_max / dt_min > P.ratio_dtmax) {
    const double lim = P.ratio_dtmax * dt_min;
    if (dt[c] > lim) {
      dt[c] = lim;
      dg = vol[c] / lim;
      for (int32_t s = cptr[c]; s < cptr[c + 1]; s++) {
        const SlotRec sr = slots[s];
        double vn = qc[1] * sr.nx + qc[2] * sr.ny + qc[3] * sr.nz;
        vn = fabs(vn);
        dg += 0.5 * sr.area * (vn + qc[Q_A]) * P.lhs_omga;
      }
      diag[c] = dg;
    }
  }
}

// The mixed form (MX) evaluates each record's product as the persistent
// sweeps' mixed form does: FluxLUSGS3D in difference form in FP32 from the
// neighbour's single-precision state record q4 and the record's normal and
// weight rounded to FP32, the weighted product widened to FP64 and summed in
// record order.  Same operations, same bits as those sweeps.
template <bool MX>
__device__ __forceinline__ void level_rec_product(const SweepRec &r, int32_t nb,
                                                  const double *__restrict__ q8,
                                                  const float *__restrict__ q4, const double *dn,
                                                  const Params &P, double *wf) {
  if constexpr (MX) {
    float qf[Q_STRIDE], df[5], ff[5];
    load_q4(q4, nb, qf);
#pragma unroll
    for (int k = 0; k < 5; k++) df[k] = (float)dn[k];
    flux_lusgs_diff(qf, df, (float)r.nx, (float)r.ny, (float)r.nz, flux_params<float>(P), ff);
    const float w = (float)r.w;
#pragma unroll
    for (int k = 0; k < 5; k++) wf[k] = (double)(w * ff[k]);
  } else {
    double qn[Q_STRIDE], f[5];
    load_q(q8, nb, qn);
    flux_lusgs(qn, dn, r.nx, r.ny, r.nz, P, f);
#pragma unroll
    for (int k = 0; k < 5; k++) wf[k] = r.w * f[k];
  }
}

template <bool MX>
__global__ void __launch_bounds__(kBlock)
k_sweep_fwd(int32_t l0, int32_t l1, const int32_t *__restrict__ cells,
            const int32_t *__restrict__ sptr, const SweepRec *__restrict__ recs,
            const int32_t *__restrict__ nbs, const double *__restrict__ q8,
            const float *__restrict__ q4,
            double *__restrict__ dqf, double *__restrict__ dqb, const double *__restrict__ res,
            int32_t C, double *__restrict__ diag, int32_t first_cell, Params P0, int clamp_check,
            double *__restrict__ dt, const unsigned long long *__restrict__ dt_ext,
            const int32_t *__restrict__ cptr, const SlotRec *__restrict__ slots,
            const double *__restrict__ vol, Cases cs) {
  const int32_t i = l0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= l1) return;
  const int32_t c = cells[i];
  const int32_t cse = case_of(cs, c);
  const Params P = params_of(P0, cs, c);
  const int32_t first = cs.P ? cs.first[cse] : first_cell;
  double d[5];
  for (int k = 0; k < 5; k++) d[k] = res[(int64_t)k * C + c];
  const int32_t s1 = sptr[i + 1];
  for (int32_t s = sptr[i]; s < s1; s++) {
    const SweepRec r = recs[s];
    const int32_t nb = nbs[s];
    double dn[5], wf[5];
    load_dq_cg(dqf, nb, dn);
    level_rec_product<MX>(r, nb, q8, q4, dn, P, wf);
    for (int k = 0; k < 5; k++) d[k] -= wf[k];
  }
  double dg = diag[c];
  double qc[Q_STRIDE];
  load_q(q8, c, qc);
  if (clamp_check) clamp_diag(c, qc, dg, P, dt, dt_ext + 2 * cse, cptr, slots, vol, diag);
  for (int k = 0; k < 5; k++) d[k] /= dg;
  if (c != first) dq_limit(qc, d, P);
  store_dq(dqf, c, d);
  store_sentinel(dqb, c);
}

// Backward (upper) sweep of one level, fused with the state update: the new
// state of the cell goes to the other buffer, so later levels of this sweep
// still read the old state (the reference updates after the sweep).
template <bool MX>
__global__ void __launch_bounds__(kBlock)
k_sweep_bwd(int32_t l0, int32_t l1, const int32_t *__restrict__ cells,
            const int32_t *__restrict__ sptr, const SweepRec *__restrict__ recs,
            const int32_t *__restrict__ nbs, const double *__restrict__ q8,
            const float *__restrict__ q4, double *__restrict__ q8_new,
            float *__restrict__ q4_new, double *__restrict__ dqf, double *__restrict__ dqb,
            const double *__restrict__ diag, Params P0, Cases cs) {
  const int32_t i = l0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= l1) return;
  const int32_t c = cells[i];
  const Params P = params_of(P0, cs, c);
  double d[5], fs[5] = {0., 0., 0., 0., 0.};
  load_dq_cg(dqf, c, d);
  const int32_t s1 = sptr[i + 1];
  for (int32_t s = sptr[i]; s < s1; s++) {
    const SweepRec r = recs[s];
    const int32_t nb = nbs[s];
    double dn[5], wf[5];
    load_dq_cg(dqb, nb, dn);
    level_rec_product<MX>(r, nb, q8, q4, dn, P, wf);
    for (int k = 0; k < 5; k++) fs[k] += wf[k];
  }
  const double tmp = 2.0 * diag[c];
  for (int k = 0; k < 5; k++) d[k] -= fs[k] / tmp;
  double qc[Q_STRIDE];
  load_q(q8, c, qc);
  dq_limit(qc, d, P);
  store_dq(dqb, c, d);
  store_sentinel(dqf, c);
  update_cell(qc, d, P);
  cell_props(qc, P);
  store_q(q8_new, c, qc);
  if (MX) store_q4(q4_new, c, qc);
}

// ---------------------------------------------------------------------------
// Persistent chunked sweeps, warp-specialised.
//
// The cells are split into chunks, one per block and one block per SM
// (cooperative launch).  A block walks the levels of its chunk in increasing
// order; a level with more cells than the block has lane groups takes several
// passes, and every (level, pass) is one work item.  The block's warps have
// two roles:
//
//  * producer warps, in kWsTeams teams taking the items in turn, read what an
//    item's cells need that no sweep writes -- the cell's state, Diag and
//    right-hand side, and for each of its neighbour records the neighbour's
//    state and the face -- and evaluate the neighbour-state half of
//    FluxLUSGS3D (flux_lusgs_pre), the reciprocal of the diagonal term and
//    the limiter's velocity square into the team's shared-memory stage slot
//    (an mbarrier pair per slot hands it over and back);
//  * consumer warps take an item from its stage into registers, wait at the
//    level barrier (a named barrier over the consumer warps alone) and run
//    only the dependent chain: the neighbours' increments, the rest of
//    FluxLUSGS3D, the ordered sums, the division, the limiter and the stores.
//
// A dependency inside the chunk is read from the block's shared-memory ring
// of its last kRing positions (or, when older, from global memory); a
// dependency on another chunk is polled in L2 until it is no longer the
// sentinel (bounded wait).  In the backward sweep the producers also apply
// the state update of an item's cells (UpdateFlowField3D_CFL3d) once the
// consumers have released its slot, from the slot's state record and the
// ring: the update is off the dependent chain and reads nothing twice.  The
// consumer warps are then at most kWsTeams - 1 items further (a slot is
// refilled only after every consumer warp has released it), fewer than kRing
// positions, so the item's ring entries are still there.  Progress: a cell
// waits only for cells of lower levels, each block visits its levels in
// increasing order, and every block is resident, so by induction over the
// levels every cell completes.  Every wait is bounded; one that gives up
// sets the error word, after which every other wait returns at once and the
// kernel runs to its end.
// ---------------------------------------------------------------------------
constexpr uint32_t kMark = 0x80000000u;    // neighbour flag: in another chunk (wait in L2)
constexpr uint32_t kInRing = 0x40000000u;  // neighbour flag: increment in the block's ring
constexpr uint32_t kIdMask = 0x3FFFFFFFu;  // neighbour id bits
constexpr int kMinChunk = 64;              // no chunk smaller than this many cells
// Increments of the last kRing positions of a chunk stay in shared memory, so
// that a dependency inside the chunk is read on the SM instead of from L2.
#ifndef MFG_SWEEP_RING
#define MFG_SWEEP_RING 512
#endif
constexpr int kRing = MFG_SWEEP_RING;
static_assert((kRing & (kRing - 1)) == 0, "ring size must be a power of two");

constexpr int kWsTeams = 4;  // producer teams; team t fills stage slot t
// Segment starts of a chunk kept in shared memory (longer chunks read the
// rest from global memory).
constexpr int kSegCache = 512;
// Cases whose LimitTimeStep clamp state is kept in shared memory.
constexpr int kCaseCache = 128;

// Position-major sweep tables.  Position p (chunk-major, level-sorted) holds
// one cell; its records sit at [p * W, p * W + ns).  W = 4 (tetrahedra) or 8
// (any cell with at most 8 lower or upper neighbours).
struct __align__(8) PosCell {
  int32_t cell, ns;
};

// A cell is swept by a pair of consumer lanes: lane h of the pair owns the
// records [h W / 2, (h + 1) W / 2), whose products are independent
// (instruction-level parallelism); lane 0 sums its records into the
// right-hand side in record order and hands the partial sums to lane 1,
// which adds its own in order, divides, limits and stores -- the operations
// and order of the reference's loop, so the same bits.  An item holds
// kGroups cells: 64 (four consumer warps, one per SM sub-partition) for W =
// 4, 32 for W = 8, whose stage records are twice the size; a producer
// thread stages one cell.
template <int W>
struct WsGeom {
  static constexpr int kGroups = W == 8 ? 32 : 64;      // cells per item
  static constexpr int kRh = W / 2;                     // records per consumer lane
  static constexpr int kConsumers = 2 * kGroups;        // consumer threads
  static constexpr int kTeamThreads = kGroups;          // producer threads per team
  static constexpr int kThreads = kConsumers + kWsTeams * kTeamThreads;
};

template <bool MX>
struct SweepTypes {
  using Q = double;
  using Rec = SweepRec;
};
template <>
struct SweepTypes<true> {
  using Q = float;
  using Rec = SweepRecF;
};

// One stage slot: what the producers stage for the cells of one item, each
// field an array over the item's G cells, so that the consumer warps (one
// thread per cell) read 32 consecutive words per field without bank
// conflicts.  A record's fields -- FP64: the neighbour-state half of
// FluxLUSGS3D (LusgsPre, 11 values), the face normal and the weight;
// mixed: the neighbour's single-precision state record (8 values), the
// normal and the weight.  A cell's: its state record, the right-hand side
// (res, forward; the forward increment, backward), the diagonal term it
// divides by with its reciprocal, the limiter's velocity square, and the
// indices.
template <int W, bool MX>
struct WsSlot {
  static constexpr int G = WsGeom<W>::kGroups;
  static constexpr int kRF = MX ? Q_STRIDE + 4 : 15;
  typename SweepTypes<MX>::Q rec[W][kRF][G];
  double qc[Q_STRIDE][G];
  double in5[5][G];
  double den[G], rden[G], vv[G];
  int32_t cell[G], ns[G], first[G], pos[G];
  uint32_t nb[W][G];
  int32_t nslot[W][G];
};

template <int W, bool MX>
constexpr size_t ws_smem_bytes() {
  return sizeof(WsSlot<W, MX>) * kWsTeams + sizeof(double) * kRing * 5 +
         sizeof(int32_t) * (kSegCache + 2) + sizeof(double) * kCaseCache +
         sizeof(uint64_t) * 2 * kWsTeams;
}
// the producers' update reads an item's ring entries up to kWsTeams items on
static_assert(kWsTeams * WsGeom<4>::kGroups < kRing && kWsTeams * WsGeom<8>::kGroups < kRing,
              "ring longer than the stage");
static_assert(sizeof(WsSlot<4, false>) % 16 == 0 && sizeof(WsSlot<8, false>) % 16 == 0 &&
                  sizeof(WsSlot<4, true>) % 16 == 0 && sizeof(WsSlot<8, true>) % 16 == 0,
              "slot alignment");
static_assert(ws_smem_bytes<4, false>() <= 227 * 1024 && ws_smem_bytes<8, false>() <= 227 * 1024 &&
                  ws_smem_bytes<4, true>() <= 227 * 1024 && ws_smem_bytes<8, true>() <= 227 * 1024,
              "stage fits in shared memory");

// Asynchronous copies global -> shared (.cg: from L2, never a stale L1 line).
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// mbarrier hand-off between the producer teams and the consumer warps.
__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                   smem_addr(b))
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the completion of the phase of the given parity; gives up
// (setting *err) after `spin` cycles, or soon after another wait gave up.
// The error word and the clock are read every 64th try only, and a waiter
// with slack (the producers) sleeps between tries, so that waiting warps
// take neither issue slots nor L2 requests from the ones that compute.
__device__ __forceinline__ void mbar_wait(uint64_t *b, unsigned parity, int *err,
                                          long long spin, unsigned sleep_ns) {
  if (mbar_test(b, parity)) return;
  const long long t0 = clock64();
  for (unsigned tries = 1;; tries++) {
    if (sleep_ns) __nanosleep(sleep_ns);
    if (mbar_test(b, parity)) return;
    if ((tries & 63) == 0) {
      if (ld_relaxed(err)) return;
      if (clock64() - t0 > spin) {
        atomicExch(err, 1);
        return;
      }
    }
  }
}
// The level barrier of the consumer warps (named barrier 1; the producers
// never take part).
template <int N>
__device__ __forceinline__ void consumers_sync() {
  if (N > 32)
    asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory");
  else
    __syncwarp();
}

// Diag of a cell whose dt LimitTimeStep clamps to lim (compute_timestep.cpp
// :929-944, then Diag = vol / dt + the face sum of CalDiagLUSGS,
// forward_lusgs.cpp:96 and :175-260, with that dt).
__device__ __forceinline__ double clamped_diag(int32_t c, const double *qc, const Params &P,
                                               double lim, const int32_t *__restrict__ cptr,
                                               const SlotRec *__restrict__ slots,
                                               const double *__restrict__ vol) {
  double dg = vol[c] / lim;
  for (int32_t s = cptr[c]; s < cptr[c + 1]; s++) {
    const SlotRec sr = slots[s];
    double vn = qc[1] * sr.nx + qc[2] * sr.ny + qc[3] * sr.nz;
    vn = fabs(vn);
    dg += 0.5 * sr.area * (vn + qc[Q_A]) * P.lhs_omga;
  }
  return dg;
}

// Per-case clamp state: lim > 0 when dt_max / dt_min exceeds ratio_dtmax.
__device__ __forceinline__ double clamp_limit(const Params &P,
                                              const unsigned long long *__restrict__ ext) {
  const double dt_max = __longlong_as_double((long long)ext[0]);
  const double dt_min = __longlong_as_double((long long)ext[1]);
  return (dt_max / dt_min > P.ratio_dtmax) ? P.ratio_dtmax * dt_min : -1.0;
}

// Producer: one item's cells into a stage slot; thread g of the team stages
// cell g of the item.
template <int W, bool FWD, bool MX>
__device__ __forceinline__ void ws_produce(
    WsSlot<W, MX> &S, int32_t g, int32_t p0, int32_t pend, const PosCell *__restrict__ pcs,
    const typename SweepTypes<MX>::Rec *__restrict__ prec, const int32_t *__restrict__ pnb,
    const int32_t *__restrict__ pslot, const double *__restrict__ q8,
    const typename SweepTypes<MX>::Q *__restrict__ qnb, const double *__restrict__ res,
    const double *__restrict__ dqf_own, int32_t C, const double *__restrict__ diag,
    int32_t first_cell, const Params &P0, const Cases &cs) {
  const int32_t p = p0 + g;
  if (p >= pend) {
    S.cell[g] = -1;
    return;
  }
  const PosCell x = pcs[p];
  const Params P = params_of(P0, cs, x.cell);
  // the records' indices, then the states, then the products (the padding
  // slots past ns are not read)
  uint32_t e[W];
  int32_t sl[W];
  typename SweepTypes<MX>::Rec rc[W];
#pragma unroll
  for (int j = 0; j < W; j++) {
    const int64_t o = (int64_t)p * W + j;
    if (j >= x.ns) continue;
    e[j] = (uint32_t)pnb[o];
    sl[j] = pslot[o];
    rc[j] = prec[o];
  }
  {
    double qc[Q_STRIDE];
    load_q(q8, x.cell, qc);
    const double dg = diag[x.cell];
    double in5[5];
#pragma unroll
    for (int k = 0; k < 5; k++)
      in5[k] = FWD ? res[(int64_t)k * C + x.cell] : dqf_own[(int64_t)x.cell * Q_STRIDE + k];
    const double den = FWD ? dg : 2.0 * dg;
#pragma unroll
    for (int k = 0; k < Q_STRIDE; k++) S.qc[k][g] = qc[k];
#pragma unroll
    for (int k = 0; k < 5; k++) S.in5[k][g] = in5[k];
    S.den[g] = den;
    S.rden[g] = 1.0 / den;
    S.vv[g] = qc[1] * qc[1] + qc[2] * qc[2] + qc[3] * qc[3];
    S.cell[g] = x.cell;
    S.ns[g] = x.ns;
    S.first[g] = FWD && x.cell == (cs.P ? cs.first[case_of(cs, x.cell)] : first_cell);
    S.pos[g] = p;
  }
#pragma unroll
  for (int j = 0; j < W; j++) {
    if (j >= x.ns) continue;
    S.nb[j][g] = e[j];
    S.nslot[j][g] = sl[j];
    const int64_t nb = (int64_t)(e[j] & kIdMask);
    if constexpr (MX) {
      const float4 *qs = reinterpret_cast<const float4 *>(qnb + nb * Q_STRIDE);
      const float4 a = __ldg(qs), b = __ldg(qs + 1);
      const float v[Q_STRIDE] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int k = 0; k < Q_STRIDE; k++) S.rec[j][k][g] = v[k];
      S.rec[j][Q_STRIDE][g] = rc[j].nx;
      S.rec[j][Q_STRIDE + 1][g] = rc[j].ny;
      S.rec[j][Q_STRIDE + 2][g] = rc[j].nz;
      S.rec[j][Q_STRIDE + 3][g] = rc[j].w;
    } else {
      double qn[Q_STRIDE];
      load_q(qnb, nb, qn);
      const LusgsPre<double> a =
          flux_lusgs_pre(qn, rc[j].nx, rc[j].ny, rc[j].nz, flux_params<double>(P));
      const double v[15] = {a.Q0, a.Q1, a.Q2, a.Q3, a.Q4, a.vq, a.eig, a.f1,
                            a.f2, a.f3, a.f4, rc[j].nx, rc[j].ny, rc[j].nz, rc[j].w};
#pragma unroll
      for (int k = 0; k < 15; k++) S.rec[j][k][g] = v[k];
    }
  }
}

// Consumer: the dependent chain of one cell on its lane pair (lane h, see
// WsGeom), c < 0 when the pair has no cell in this item.  e[u]: the
// neighbour word of the lane's record u, dn[u]: its increment as read when
// the item was taken (unless it is in the ring).  FWD: DQ* = (res - sum_j
// 0.5 area_j F_j) / Diag, limited except for the first cell (SolveLUSGS3D
// forward, forward_lusgs.cpp:803-1014); backward: DQ = DQ* - (sum_j area_j
// F_j) / (2 Diag), limited (:1060-1249).
template <int W, bool FWD, bool MX>
__device__ __forceinline__ void ws_cell(
    const WsSlot<W, MX> &S, int32_t g, int32_t h, int32_t c, int32_t ns, const uint32_t *e,
    double (*dn)[5], int32_t pbase, double *ring, const double *src, double *dst,
    double *rearm, const Params &P0, const double *s_lim, int clamp_check,
    double *__restrict__ dt, double *__restrict__ diag,
    const unsigned long long *__restrict__ dt_ext, const int32_t *__restrict__ cptr,
    const SlotRec *__restrict__ slots, const double *__restrict__ vol, int *err, long long spin,
    const Cases &cs) {
  constexpr int R = WsGeom<W>::kRh;
  const bool live = c >= 0;
  // the neighbour increments: from the ring, else as read when the item was
  // taken, polled again in L2 while one is the sentinel.  The warp polls in
  // one converged, bounded loop.
  bool have[R];
#pragma unroll
  for (int u = 0; u < R; u++) {
    const int j = h * R + u;
    have[u] = true;
    if (!live || j >= ns) continue;
    if (e[u] & kInRing) {
      const int32_t sl = S.nslot[j][g];
#pragma unroll
      for (int k = 0; k < 5; k++) dn[u][k] = ring[sl * 5 + k];
    } else {
      have[u] = rec5_ready(dn[u]);
    }
  }
  bool all = true;
#pragma unroll
  for (int u = 0; u < R; u++) all = all && have[u];
  if (__any_sync(0xffffffffu, !all)) {
    const long long t0 = clock64();
    for (int polls = 1;; polls++) {
      if (polls > 64) __nanosleep(64);
      if (!all) {
        const int gave_up = ld_relaxed(err);
        all = true;
#pragma unroll
        for (int u = 0; u < R; u++) {
          if (have[u]) continue;
          load_rec5_l2(src + (int64_t)(e[u] & kIdMask) * Q_STRIDE, dn[u]);
          have[u] = rec5_ready(dn[u]);
          all = all && have[u];
        }
        if (!all && (gave_up || clock64() - t0 > spin)) {
          if (!gave_up) atomicExch(err, 1);
          all = true;  // results invalid; the host reports MFG_ERR_TIMEOUT
        }
      }
      if (!__any_sync(0xffffffffu, !all)) break;
    }
  }
  const int32_t cse = live ? case_of(cs, c) : 0;
  const Params P = live ? params_of(P0, cs, c) : P0;
  // w_j * FluxLUSGS3D(q[nb_j], DQ[nb_j], n_j) of the lane's records, their
  // products overlapping (FP64: branch-free divisions, the exact form redone
  // for the lane's records when one is out of its window)
  double wf[R][5];
  if constexpr (!MX) {
    auto pre_of = [&](int j) {
      LusgsPre<double> a;
      a.Q0 = S.rec[j][0][g];
      a.Q1 = S.rec[j][1][g];
      a.Q2 = S.rec[j][2][g];
      a.Q3 = S.rec[j][3][g];
      a.Q4 = S.rec[j][4][g];
      a.vq = S.rec[j][5][g];
      a.eig = S.rec[j][6][g];
      a.f1 = S.rec[j][7][g];
      a.f2 = S.rec[j][8][g];
      a.f3 = S.rec[j][9][g];
      a.f4 = S.rec[j][10][g];
      return a;
    };
    bool ok = true;
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int j = h * R + u;
      if (!live || j >= ns) continue;
      double f[5];
      bool oku;
      flux_lusgs_fin_fast(pre_of(j), dn[u], S.rec[j][11][g], S.rec[j][12][g], S.rec[j][13][g],
                          flux_params<double>(P), f, oku);
      ok = ok && oku;
      const double w = S.rec[j][14][g];
#pragma unroll
      for (int k = 0; k < 5; k++) wf[u][k] = w * f[k];
    }
    if (!ok) {
#pragma unroll
      for (int u = 0; u < R; u++) {
        const int j = h * R + u;
        if (!live || j >= ns) continue;
        double f[5];
        flux_lusgs_fin(pre_of(j), dn[u], S.rec[j][11][g], S.rec[j][12][g], S.rec[j][13][g],
                       flux_params<double>(P), f);
        const double w = S.rec[j][14][g];
#pragma unroll
        for (int k = 0; k < 5; k++) wf[u][k] = w * f[k];
      }
    }
  } else {
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int j = h * R + u;
      if (!live || j >= ns) continue;
      // off-diagonal product in FP32, accumulated in FP64
      float qf[Q_STRIDE], df[5], ff[5];
#pragma unroll
      for (int k = 0; k < Q_STRIDE; k++) qf[k] = S.rec[j][k][g];
#pragma unroll
      for (int k = 0; k < 5; k++) df[k] = (float)dn[u][k];
      flux_lusgs_diff(qf, df, S.rec[j][Q_STRIDE][g], S.rec[j][Q_STRIDE + 1][g],
                      S.rec[j][Q_STRIDE + 2][g], flux_params<float>(P), ff);
      const float w = S.rec[j][Q_STRIDE + 3][g];
#pragma unroll
      for (int k = 0; k < 5; k++) wf[u][k] = (double)(w * ff[k]);
    }
  }
  // the sum over the records in record order: lane 0 from the right-hand
  // side through its records, lane 1 on from lane 0's partial sums
  double part[5];
#pragma unroll
  for (int k = 0; k < 5; k++) part[k] = (FWD && h == 0 && live) ? S.in5[k][g] : 0.0;
#pragma unroll
  for (int u = 0; u < R; u++) {
    const int j = h * R + u;
    if (!live || j >= ns || h != 0) continue;
#pragma unroll
    for (int k = 0; k < 5; k++) {
      if (FWD)
        part[k] -= wf[u][k];
      else
        part[k] += wf[u][k];
    }
  }
#pragma unroll
  for (int k = 0; k < 5; k++) part[k] = __shfl_sync(0xffffffffu, part[k], threadIdx.x & ~1);
#pragma unroll
  for (int u = 0; u < R; u++) {
    const int j = h * R + u;
    if (!live || j >= ns || h != 1) continue;
#pragma unroll
    for (int k = 0; k < 5; k++) {
      if (FWD)
        part[k] -= wf[u][k];
      else
        part[k] += wf[u][k];
    }
  }
  if (!live || h != 1) return;
  double qc[Q_STRIDE];
#pragma unroll
  for (int k = 0; k < Q_STRIDE; k++) qc[k] = S.qc[k][g];
  const double den = S.den[g], rden = S.rden[g];
  // LimitTimeStep's clamp (forward sweep of a fused iteration, only when some
  // case's dt ratio exceeds its limit)
  double dg = den, lim = -1.0;  // forward: den is Diag itself
  bool clamped = false;
  if (FWD && clamp_check) {
    lim = (cse < kCaseCache) ? s_lim[cse] : clamp_limit(P, dt_ext + 2 * cse);
    if (lim > 0.0 && dt[c] > lim) {
      dg = clamped_diag(c, qc, P, lim, cptr, slots, vol);
      clamped = true;
    }
  }
  // the five quotients overlapping (branch-free; div_by_recip for all when
  // one of them is out of its window)
  double d[5];
  bool okq = true;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    bool okk;
    const double qk = div_recip_fast(part[k], den, rden, okk);
    okq = okq && okk;
    d[k] = FWD ? qk : S.in5[k][g] - qk;
  }
  if (!okq)
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const double qk = div_by_recip(part[k], den, rden);
      d[k] = FWD ? qk : S.in5[k][g] - qk;
    }
  if (FWD && clamped)
#pragma unroll
    for (int k = 0; k < 5; k++) d[k] = part[k] / dg;
  if (!FWD || !S.first[g]) dq_limit_vv(qc, S.vv[g], d, P);
  if (FWD && clamped) {
    dt[c] = lim;
    diag[c] = dg;
  }
  store_dq(dst, c, d);
  store_sentinel(rearm, c);  // armed for the other sweep
  const int32_t slot = (S.pos[g] - pbase) & (kRing - 1);
#pragma unroll
  for (int k = 0; k < 5; k++) ring[slot * 5 + k] = d[k];
}

// Backward sweep, producer thread g: UpdateFlowField3D_CFL3d of cell g of the
// item whose slot the consumers have just released, from the slot's state
// record and the cell's final increment in the ring (forward_lusgs.cpp:
// 1335-1488); the new state goes to the other state buffer.
template <int W, bool MX>
__device__ __forceinline__ void ws_update(const WsSlot<W, MX> &S, int32_t g, int32_t pbase,
                                          const double *ring, double *__restrict__ q8_new,
                                          float *__restrict__ q4_new, const Params &P0,
                                          const Cases &cs) {
  const int32_t c = S.cell[g];
  if (c < 0) return;
  double qc[Q_STRIDE], d[5];
#pragma unroll
  for (int k = 0; k < Q_STRIDE; k++) qc[k] = S.qc[k][g];
  const int32_t sl = (S.pos[g] - pbase) & (kRing - 1);
#pragma unroll
  for (int k = 0; k < 5; k++) d[k] = ring[sl * 5 + k];
  const Params P = params_of(P0, cs, c);
  update_cell(qc, d, P);
  cell_props(qc, P);
  store_q(q8_new, c, qc);
  if (MX) store_q4(q4_new, c, qc);
}

// One persistent sweep over chunk blockIdx.x (see the section comment).
template <int W, bool FWD, bool MX>
__device__ __forceinline__ void ws_sweep(
    const int32_t *__restrict__ seg_begin, const int32_t *__restrict__ segs,
    const PosCell *__restrict__ pcs, const typename SweepTypes<MX>::Rec *__restrict__ prec,
    const int32_t *__restrict__ pnb, const int32_t *__restrict__ pslot,
    const double *__restrict__ q8, const typename SweepTypes<MX>::Q *__restrict__ qnb,
    const double *src, double *dst, double *rearm, const double *__restrict__ res,
    const double *__restrict__ dqf_own, int32_t C, double *__restrict__ diag, int32_t first_cell,
    const Params &P0, int clamp_check, double *__restrict__ dt,
    const unsigned long long *__restrict__ dt_ext, const int32_t *__restrict__ cptr,
    const SlotRec *__restrict__ slots, const double *__restrict__ vol, int *err, long long spin,
    const Cases &cs, double *__restrict__ q8_new, float *__restrict__ q4_new) {
  using Geo = WsGeom<W>;
  constexpr int G = Geo::kGroups;
  extern __shared__ __align__(16) unsigned char ws_smem[];
  WsSlot<W, MX> *stage = reinterpret_cast<WsSlot<W, MX> *>(ws_smem);  // [kWsTeams]
  double *ring = reinterpret_cast<double *>(stage + kWsTeams);         // [kRing][5]
  int32_t *s_segs = reinterpret_cast<int32_t *>(ring + kRing * 5);       // [kSegCache + 1]
  double *s_lim = reinterpret_cast<double *>(s_segs + kSegCache + 2);    // [kCaseCache]
  uint64_t *full = reinterpret_cast<uint64_t *>(s_lim + kCaseCache);     // [kWsTeams]
  uint64_t *empty = full + kWsTeams;                                      // [kWsTeams]
  __shared__ int s_clamp_any;
  const int32_t sg0 = seg_begin[blockIdx.x], sg1 = seg_begin[blockIdx.x + 1];
  for (int32_t i = threadIdx.x; i <= sg1 - sg0 && i <= kSegCache; i += blockDim.x)
    s_segs[i] = segs[sg0 + i];
  if (threadIdx.x == 0) {
    s_clamp_any = 0;
    for (int t = 0; t < kWsTeams; t++) {
      mbar_init(&full[t], Geo::kTeamThreads);
      mbar_init(&empty[t], Geo::kConsumers / 32);
    }
  }
  __syncthreads();
  if (FWD && clamp_check)
    for (int32_t k = threadIdx.x; k < cs.ncase && k < kCaseCache; k += blockDim.x) {
      s_lim[k] = clamp_limit(cs.P ? cs.P[k] : P0, dt_ext + 2 * k);
      if (s_lim[k] > 0.0) s_clamp_any = 1;
    }
  if (FWD && clamp_check && cs.ncase > kCaseCache && threadIdx.x == 0) s_clamp_any = 1;
  __syncthreads();
  // the per-cell clamp test only when some case needs it
  clamp_check = (FWD && clamp_check && s_clamp_any) ? 1 : 0;
  const int32_t pbase = sg1 > sg0 ? s_segs[0] : 0;
  auto seg_at = [&](int32_t sg) {
    const int32_t i = sg - sg0;
    return i <= kSegCache ? s_segs[i] : segs[sg];
  };
  if (threadIdx.x >= Geo::kConsumers) {
    // producer team t: items t, t + kWsTeams, ... into stage slot t
    const int32_t t = (threadIdx.x - Geo::kConsumers) / Geo::kTeamThreads;
    const int32_t r = (threadIdx.x - Geo::kConsumers) % Geo::kTeamThreads;
    WsSlot<W, MX> &S = stage[t];
    int32_t item = 0, last_use = -1;
    for (int32_t sg = sg0; sg < sg1; sg++) {
      const int32_t a = seg_at(sg), b = seg_at(sg + 1);
      const int32_t np = (b - a + G - 1) / G;
      for (int32_t pass = 0; pass < np; pass++, item++) {
        if (item % kWsTeams != t) continue;
        const int32_t use = item / kWsTeams;
        if (use >= 1) {
          mbar_wait(&empty[t], (unsigned)((use - 1) & 1), err, spin, 256);
          if (!FWD) ws_update<W, MX>(S, r, pbase, ring, q8_new, q4_new, P0, cs);
        }
        ws_produce<W, FWD, MX>(S, r, a + pass * G, b, pcs, prec, pnb, pslot, q8, qnb, res,
                               dqf_own, C, diag, first_cell, P0, cs);
        mbar_arrive(&full[t]);
        last_use = use;
      }
    }
    if (!FWD && last_use >= 0) {  // the slot's last item
      mbar_wait(&empty[t], (unsigned)(last_use & 1), err, spin, 256);
      ws_update<W, MX>(S, r, pbase, ring, q8_new, q4_new, P0, cs);
    }
    return;
  }
  // consumers: lane pair g takes cell g of every item
  constexpr int R = Geo::kRh;
  const int32_t g = threadIdx.x >> 1, h = threadIdx.x & 1;
  int32_t item = 0;
  for (int32_t sg = sg0; sg < sg1; sg++) {
    const int32_t a = seg_at(sg), b = seg_at(sg + 1);
    const int32_t np = (b - a + G - 1) / G;
    for (int32_t pass = 0; pass < np; pass++, item++) {
      const int32_t t = item % kWsTeams;
      mbar_wait(&full[t], (unsigned)((item / kWsTeams) & 1), err, spin, 0);
      const WsSlot<W, MX> &S = stage[t];
      const int32_t c = S.cell[g];
      const int32_t ns = c >= 0 ? S.ns[g] : 0;
      uint32_t e[R];
      double dn[R][5];
      // increments read from L2 (older than the ring, or produced by another
      // chunk) are requested now, so that their round trips overlap the
      // level barrier; one still holding the sentinel is polled in ws_cell
#pragma unroll
      for (int u = 0; u < R; u++) {
        const int j = h * R + u;
        e[u] = j < ns ? S.nb[j][g] : kInRing;
        if (!(e[u] & kInRing)) load_rec5_l2(src + (int64_t)(e[u] & kIdMask) * Q_STRIDE, dn[u]);
      }
      if (pass == 0 && item > 0) consumers_sync<Geo::kConsumers>();  // the previous level is stored
      ws_cell<W, FWD, MX>(S, g, h, c, ns, e, dn, pbase, ring, src, dst, rearm, P0, s_lim,
                          clamp_check,
                          dt, diag, dt_ext, cptr, slots, vol, err, spin, cs);
      __syncwarp();
      if ((threadIdx.x & 31) == 0) mbar_arrive(&empty[t]);  // the slot is free again
    }
  }
}

#ifndef MFG_PERSIST_MINB
#define MFG_PERSIST_MINB 1
#endif

// Forward sweep.  chunk_skip > 0 withholds the first chunk_skip chunks
// (failure-detection self-test only: the cells that depend on them wait
// until the bound runs out).
template <int W, bool MX>
__global__ void __launch_bounds__(WsGeom<W>::kThreads, MFG_PERSIST_MINB)
k_sweep_fwd_chunk(const int32_t *__restrict__ seg_begin, const int32_t *__restrict__ segs,
                  const PosCell *__restrict__ pcs,
                  const typename SweepTypes<MX>::Rec *__restrict__ prec,
                  const int32_t *__restrict__ pnb, const int32_t *__restrict__ pslot,
                  const double *__restrict__ q8,
                  const typename SweepTypes<MX>::Q *__restrict__ qnb, double *dqf,
                  double *__restrict__ dqb, const double *__restrict__ res, int32_t C,
                  double *__restrict__ diag, int32_t first_cell, Params P0, int clamp_check,
                  double *__restrict__ dt, const unsigned long long *__restrict__ dt_ext,
                  const int32_t *__restrict__ cptr, const SlotRec *__restrict__ slots,
                  const double *__restrict__ vol, int *err, long long spin,
                  int32_t chunk_skip, Cases cs) {
  if ((int32_t)blockIdx.x < chunk_skip) return;
  ws_sweep<W, true, MX>(seg_begin, segs, pcs, prec, pnb, pslot, q8, qnb, dqf, dqf, dqb, res,
                        nullptr, C, diag, first_cell, P0, clamp_check, dt, dt_ext, cptr, slots,
                        vol, err, spin, cs, nullptr, nullptr);
}

// Backward sweep with the state update (by the producers, see the section
// comment).
template <int W, bool MX>
__global__ void __launch_bounds__(WsGeom<W>::kThreads, MFG_PERSIST_MINB)
k_sweep_bwd_chunk(const int32_t *__restrict__ seg_begin, const int32_t *__restrict__ segs,
                  const PosCell *__restrict__ pcs,
                  const typename SweepTypes<MX>::Rec *__restrict__ prec,
                  const int32_t *__restrict__ pnb, const int32_t *__restrict__ pslot,
                  const double *__restrict__ q8,
                  const typename SweepTypes<MX>::Q *__restrict__ qnb,
                  double *__restrict__ q8_new, float *__restrict__ q4_new,
                  double *__restrict__ dqf, double *dqb, const double *__restrict__ diag,
                  Params P0, int *err, long long spin, Cases cs) {
  ws_sweep<W, false, MX>(seg_begin, segs, pcs, prec, pnb, pslot, q8, qnb, dqb, dqb, dqf, nullptr,
                         dqf, 0, const_cast<double *>(diag), 0, P0, 0, nullptr, nullptr, nullptr,
                         nullptr, nullptr, err, spin, cs, q8_new, q4_new);
}

// ---------------------------------------------------------------------------
// Persistent chunked sweeps for wide levels.  The same tables with many
// small chunks -- several blocks of 64 threads per SM, kWideRing positions
// in each block's ring -- so that a level of many cells is spread over many
// blocks and an SM hides one block's waits behind another's work.  A cell is
// swept by a group of W lanes: lane j computes the flux of record j and owns
// the components k = j, j + W, ... < 5 of the increment (the ordered sum over
// the records and the division); every lane applies the limiter.  The
// operations and their order per component are those of the one-thread
// form, so the results are the same bits.  A block walks its chunk level by
// level with __syncthreads between levels; a group's work items (level,
// pass) are pipelined: indices loaded two items ahead, the read-only data
// staged into shared memory by cp.async one item ahead.
// ---------------------------------------------------------------------------
constexpr int kWideBlock = 64;  // threads per block
constexpr int kWideMinB = 6;    // resident blocks per SM (register cap)
constexpr int kWideRing = 128;  // positions of a block's ring
static_assert((kWideRing & (kWideRing - 1)) == 0, "ring size must be a power of two");

// What a lane knows about its group's position on a future level: the
// position, its ring slot, the cell, the record count, this lane's
// neighbours (flags kMark / kInRing) and their ring slots; cell < 0 = none.
template <int R>
struct WideRegs {
  int32_t p, slot, cell, ns;
  uint32_t nb[R];
  int32_t nslot[R];
};

// Everything a group reads for one cell that no sweep writes, staged into
// shared memory by cp.async one item ahead: neighbour states and records
// (by the lane of the record), the cell's state and Diag (lane 0), and res
// (forward) or the cell's forward increment (backward), component k by the
// lane that owns it.  The mixed form (MX) stages the single-precision
// neighbour records.
// Padding of a stage so that consecutive groups' stages start 16 bytes
// apart modulo 128: the groups of a warp then read their records from
// different shared-memory banks (without it every group's record k sits in
// the same bank and a warp's stage reads are 4- to 8-way conflicts).
constexpr int wide_pad_bytes(int raw) {
  const int a16 = (raw + 15) / 16 * 16;
  return a16 - raw + ((16 - a16 % 128) % 128 + 128) % 128;
}
template <int W, bool MX>
struct __align__(16) WideStage {
  typename SweepTypes<MX>::Q qn[W][Q_STRIDE];
  typename SweepTypes<MX>::Rec rec[W];
  double qc[Q_STRIDE];
  double in5[5];
  double diag;
  char pad[wide_pad_bytes(int(sizeof(typename SweepTypes<MX>::Q)) * W * Q_STRIDE +
                           int(sizeof(typename SweepTypes<MX>::Rec)) * W + 8 * (Q_STRIDE + 6))];
};
static_assert(sizeof(WideStage<4, false>) % 128 == 16 && sizeof(WideStage<4, true>) % 128 == 16 &&
                  sizeof(WideStage<8, false>) % 128 == 16 && sizeof(WideStage<8, true>) % 128 == 16,
              "stage stride");

template <int W, int L>
__device__ __forceinline__ void wide_fetch(const int32_t *s_segs, const int32_t *__restrict__ segs,
                                           int32_t sg0, int32_t sg, int32_t sg1, int32_t pbase,
                                           int32_t pos_in_level, int32_t lane,
                                           const PosCell *__restrict__ pcs,
                                           const int32_t *__restrict__ pnb,
                                           const int32_t *__restrict__ pslot,
                                           WideRegs<W / L> &o) {
  o.cell = -1;
  o.ns = 0;
#pragma unroll
  for (int r = 0; r < W / L; r++) {
    o.nb[r] = 0;
    o.nslot[r] = 0;
  }
  if (sg >= sg1) return;
  const int32_t i = sg - sg0;
  const int32_t a = i < kSegCache ? s_segs[i] : segs[sg];
  const int32_t b = i + 1 <= kSegCache ? s_segs[i + 1] : segs[sg + 1];
  const int32_t p = a + pos_in_level;
  if (p >= b) return;
  const PosCell x = pcs[p];
  o.p = p;
  o.slot = (p - pbase) & (kWideRing - 1);
  o.cell = x.cell;
  o.ns = x.ns;
#pragma unroll
  for (int r = 0; r < W / L; r++) {  // padding reads 0
    o.nb[r] = (uint32_t)pnb[(int64_t)p * W + lane + L * r];
    o.nslot[r] = pslot[(int64_t)p * W + lane + L * r];
  }
}

template <int W, int L, bool FWD, bool MX>
__device__ __forceinline__ void wide_stage_copy(const WideRegs<W / L> &o, int32_t lane,
                                           WideStage<W, MX> &st, const double *q8,
                                           const typename SweepTypes<MX>::Q *qnb,
                                           const typename SweepTypes<MX>::Rec *prec,
                                           const double *res, const double *diag,
                                           const double *dqf, int32_t C) {
  if (o.cell < 0) return;
  // 16-byte pieces of the neighbour record (64 B FP64, 32 B FP32) and of the
  // sweep record (32 B, 16 B)
  constexpr int kQ = sizeof(st.qn[0]) / 16, kR = sizeof(st.rec[0]) / 16;
#pragma unroll
  for (int r = 0; r < W / L; r++) {
    const int j = lane + L * r;
    if (j < o.ns) {
      const char *qs =
          reinterpret_cast<const char *>(qnb + (int64_t)(o.nb[r] & kIdMask) * Q_STRIDE);
      char *qd = reinterpret_cast<char *>(&st.qn[j][0]);
#pragma unroll
      for (int i = 0; i < kQ; i++) cp_async16(qd + 16 * i, qs + 16 * i);
      const char *rs = reinterpret_cast<const char *>(prec + (int64_t)o.p * W + j);
      char *rd = reinterpret_cast<char *>(&st.rec[j]);
#pragma unroll
      for (int i = 0; i < kR; i++) cp_async16(rd + 16 * i, rs + 16 * i);
    }
  }
  if (lane == 0) {
    const double *qs = q8 + (int64_t)o.cell * Q_STRIDE;
#pragma unroll
    for (int i = 0; i < 4; i++) cp_async16(&st.qc[2 * i], qs + 2 * i);
    cp_async8(&st.diag, diag + o.cell);
  }
  for (int k = lane; k < 5; k += L)
    cp_async8(&st.in5[k], FWD ? res + (int64_t)k * C + o.cell : dqf + (int64_t)o.cell * Q_STRIDE + k);
}

// One cell of one sweep level on a lane group, from its stage (the group's
// lanes only wait for one another: a cell is stored as soon as its own
// inputs are in).  sh: the group's scratch (W * 5 + 5 doubles); ring: the
// block's increments of its last kWideRing positions.  FWD: DQ* = (res - sum_j
// 0.5 area_j F_j) / Diag, limited except for the first cell (SolveLUSGS3D
// forward, forward_lusgs.cpp:799-870); backward: DQ = DQ* - (sum_j area_j
// F_j) / (2 Diag), limited (:871-940).
template <int W, int L, bool FWD, bool MX>
__device__ __forceinline__ void wide_cell(
    const WideRegs<W / L> &o, int32_t lane, const WideStage<W, MX> &st, double *sh, double *ring,
    const double (*pre)[5],
    const double *src, double *dst, double *rearm, int32_t first_cell, const Params &P0,
    const double *s_lim, int clamp_check, double *__restrict__ dt, double *__restrict__ diag,
    const unsigned long long *__restrict__ dt_ext, const int32_t *__restrict__ cptr,
    const SlotRec *__restrict__ slots, const double *__restrict__ vol, int *err,
    long long spin, const Cases &cs) {
  if (o.cell < 0) return;  // the whole group
  const unsigned gmask = ((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1));
  const int32_t c = o.cell;
  const int32_t cse = case_of(cs, c);
  const Params P = params_of(P0, cs, c);
  // what the cell's own staged data give, formed while its neighbours'
  // increments are still awaited: the reciprocal of the diagonal term the
  // increment is divided by, and the velocity square of the limiter
  const double den = FWD ? st.diag : 2.0 * st.diag;
  const double rden = 1.0 / den;
  const double vv = st.qc[1] * st.qc[1] + st.qc[2] * st.qc[2] + st.qc[3] * st.qc[3];
  // record j = lane + L r < ns: w_j * FluxLUSGS3D(q[nb_j], DQ[nb_j], n_j)
#pragma unroll
  for (int r = 0; r < W / L; r++) {
    const int j = lane + L * r;
    if (j < o.ns) {
      const uint32_t b = o.nb[r];
      // FP64: the part of the product the neighbour's state and the face
      // give, before the increment is waited for
      LusgsPre<double> a{};
      if constexpr (!MX) {
        double qn[Q_STRIDE];
#pragma unroll
        for (int k = 0; k < Q_STRIDE; k++) qn[k] = st.qn[j][k];
        a = flux_lusgs_pre(qn, st.rec[j].nx, st.rec[j].ny, st.rec[j].nz, flux_params<double>(P));
      }
      double dn[5];
      if (b & kInRing) {
#pragma unroll
        for (int k = 0; k < 5; k++) dn[k] = ring[o.nslot[r] * 5 + k];
      } else if ((b & kMark) && !rec5_ready(pre[r])) {
        wait_rec(src + (int64_t)(b & kIdMask) * Q_STRIDE, dn, err, spin);
      } else {  // read at the start of the item (see wide_chunk)
#pragma unroll
        for (int k = 0; k < 5; k++) dn[k] = pre[r][k];
      }
      if constexpr (MX) {
        // off-diagonal product in FP32, accumulated in FP64 below
        float qf[Q_STRIDE], df[5], ff[5];
#pragma unroll
        for (int k = 0; k < Q_STRIDE; k++) qf[k] = st.qn[j][k];
#pragma unroll
        for (int k = 0; k < 5; k++) df[k] = (float)dn[k];
        const SweepRecF rr = st.rec[j];
        flux_lusgs_diff(qf, df, rr.nx, rr.ny, rr.nz, flux_params<float>(P), ff);
#pragma unroll
        for (int k = 0; k < 5; k++) sh[j * 5 + k] = (double)(rr.w * ff[k]);
      } else {
        double f[5];
        const SweepRec rr = st.rec[j];
        flux_lusgs_fin(a, dn, rr.nx, rr.ny, rr.nz, flux_params<double>(P), f);
#pragma unroll
        for (int k = 0; k < 5; k++) sh[j * 5 + k] = rr.w * f[k];
      }
    }
  }
  // LimitTimeStep's clamp (fused forward sweep, and only when some case's
  // dt ratio exceeds its limit): every component lane reads dt[c] before
  // lane 0 may write it below
  double dg = st.diag, lim = -1.0;
  bool clamped = false;
  if (FWD && clamp_check && lane < 5) {
    lim = (cse < kCaseCache) ? s_lim[cse] : clamp_limit(P, dt_ext + 2 * cse);
    if (lim > 0.0 && dt[c] > lim) {
      double qc[Q_STRIDE];
#pragma unroll
      for (int i = 0; i < Q_STRIDE; i++) qc[i] = st.qc[i];
      dg = clamped_diag(c, qc, P, lim, cptr, slots, vol);
      clamped = true;
    }
  }
  __syncwarp(gmask);
  // components k = lane, lane + L, ... < 5 (at most two per lane, as two
  // independent chains); records summed in order
  {
    constexpr int kC = (5 + L - 1) / L;
    double acc[kC];
#pragma unroll
    for (int i = 0; i < kC; i++) {
      const int k = lane + L * i;
      acc[i] = (FWD && k < 5) ? st.in5[k] : 0.0;
    }
    for (int32_t j = 0; j < o.ns; j++) {
#pragma unroll
      for (int i = 0; i < kC; i++) {
        const int k = lane + L * i;
        if (k < 5) {
          if (FWD)
            acc[i] -= sh[j * 5 + k];
          else
            acc[i] += sh[j * 5 + k];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kC; i++) {
      const int k = lane + L * i;
      if (k < 5)
        sh[W * 5 + k] = FWD ? (clamped ? acc[i] / dg : div_by_recip(acc[i], den, rden))
                            : st.in5[k] - div_by_recip(acc[i], den, rden);
    }
  }
  __syncwarp(gmask);
  // the limiter on every lane (same values), the stores spread over the lanes
  double d[5], qc[Q_STRIDE];
#pragma unroll
  for (int k = 0; k < 5; k++) d[k] = sh[W * 5 + k];
#pragma unroll
  for (int i = 0; i < Q_STRIDE; i++) qc[i] = st.qc[i];
  if (!FWD || c != (cs.P ? cs.first[cse] : first_cell)) dq_limit_vv(qc, vv, d, P);
  if (lane == 0) {
    if (FWD && clamped) {
      dt[c] = lim;
      diag[c] = dg;
    }
    store_dq(dst, c, d);
  }
  if (lane == (L > 1 ? 1 : 0)) store_sentinel(rearm, c);  // armed for the other sweep
#pragma unroll
  for (int k = 0; k < 5; k++)
    if (k % L == lane) ring[o.slot * 5 + k] = d[k];
  __syncwarp(gmask);  // sh is free for the group's next cell
}

// One persistent sweep: block b walks chunk b level by level.  A level of
// more cells than the block has groups takes several passes; the group's
// work items (level, pass) form one sequence, pipelined as a whole: indices
// loaded two items ahead, read-only data staged into shared memory one item
// ahead (cp.async), so that an item's critical path holds the increments it
// depends on and one cell's arithmetic.  Blocks synchronise only between
// levels.
template <int W, int L, bool FWD, bool MX>
__device__ __forceinline__ void wide_chunk(
    const int32_t *__restrict__ seg_begin, const int32_t *__restrict__ segs,
    const PosCell *__restrict__ pcs, const typename SweepTypes<MX>::Rec *__restrict__ prec,
    const int32_t *__restrict__ pnb, const int32_t *__restrict__ pslot,
    const double *__restrict__ q8, const typename SweepTypes<MX>::Q *__restrict__ qnb,
    const double *src, double *dst, double *rearm,
    const double *__restrict__ res, const double *__restrict__ dqf_own, int32_t C,
    double *__restrict__ diag, int32_t first_cell, const Params &P0, int clamp_check,
    double *__restrict__ dt, const unsigned long long *__restrict__ dt_ext,
    const int32_t *__restrict__ cptr, const SlotRec *__restrict__ slots,
    const double *__restrict__ vol, int *err, long long spin, const Cases &cs) {
  constexpr int kGroups = kWideBlock / L;
  __shared__ WideStage<W, MX> stg[2][kGroups];
  __shared__ double shm[kGroups][W * 5 + 5];
  __shared__ double ring[kWideRing * 5];
  __shared__ int32_t s_segs[kSegCache + 1];
  __shared__ double s_lim[FWD ? kCaseCache : 1];
  const int32_t sg0 = seg_begin[blockIdx.x], sg1 = seg_begin[blockIdx.x + 1];
  const int32_t lane = threadIdx.x & (L - 1);
  const int32_t grp = threadIdx.x / L;
  for (int32_t i = threadIdx.x; i <= sg1 - sg0 && i <= kSegCache; i += blockDim.x)
    s_segs[i] = segs[sg0 + i];
  __shared__ int s_clamp_any;
  if (threadIdx.x == 0) s_clamp_any = 0;
  __syncthreads();
  if (FWD && clamp_check)
    for (int32_t k = threadIdx.x; k < cs.ncase && k < kCaseCache; k += blockDim.x) {
      s_lim[k] = clamp_limit(cs.P ? cs.P[k] : P0, dt_ext + 2 * k);
      if (s_lim[k] > 0.0) s_clamp_any = 1;
    }
  if (FWD && clamp_check && cs.ncase > kCaseCache && threadIdx.x == 0) s_clamp_any = 1;
  __syncthreads();
  // the per-cell clamp test only when some case needs it
  clamp_check = (FWD && clamp_check && s_clamp_any) ? 1 : 0;
  const unsigned gmask = ((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1));
  double *sh = shm[grp];
  const int32_t pbase = sg1 > sg0 ? s_segs[0] : 0;
  // work items (level sg, pass): the same sequence in every thread of the block
  auto seg_at = [&](int32_t sg) {
    const int32_t i = sg - sg0;
    return i <= kSegCache ? s_segs[i] : segs[sg];
  };
  auto advance = [&](int32_t &sg, int32_t &pass) {
    if (sg >= sg1) return;
    const int32_t np = (seg_at(sg + 1) - seg_at(sg) + kGroups - 1) / kGroups;
    if (++pass >= np) {
      ++sg;
      pass = 0;
    }
  };
  auto fetch = [&](int32_t sg, int32_t pass, WideRegs<W / L> &o) {
    wide_fetch<W, L>(s_segs, segs, sg0, sg, sg1, pbase, grp + pass * kGroups, lane, pcs, pnb,
                     pslot, o);
  };
  int32_t sg = sg0, pass = 0;              // this item
  int32_t sgn = sg, passn = pass;          // the next
  advance(sgn, passn);
  int32_t sgf = sgn, passf = passn;        // the one after
  advance(sgf, passf);
  WideRegs<W / L> cur, nxt, far;
  fetch(sg, pass, cur);
  fetch(sgn, passn, nxt);
  wide_stage_copy<W, L, FWD, MX>(cur, lane, stg[0][grp], q8, qnb, prec, res, diag, dqf_own, C);
  cp_async_commit();
  int par = 0;
  while (sg < sg1) {
    // increments this item reads from L2 (older than the ring, or produced by
    // another chunk): requested first, so that their round trip overlaps the
    // staging of the next items; one that still holds the sentinel is waited
    // for in wide_cell
    double pre[W / L][5];
#pragma unroll
    for (int r = 0; r < W / L; r++) {
      const int j = lane + L * r;
      if (cur.cell >= 0 && j < cur.ns && !(cur.nb[r] & kInRing))
        load_rec5_l2(src + (int64_t)(cur.nb[r] & kIdMask) * Q_STRIDE, pre[r]);
    }
    fetch(sgf, passf, far);
    wide_stage_copy<W, L, FWD, MX>(nxt, lane, stg[par ^ 1][grp], q8, qnb, prec, res, diag, dqf_own,
                              C);
    cp_async_commit();
    cp_async_wait<1>();  // this item's stage
    __syncwarp(gmask);
    wide_cell<W, L, FWD, MX>(cur, lane, stg[par][grp], sh, ring, pre, src, dst, rearm, first_cell,
                              P0, s_lim, clamp_check, dt, diag, dt_ext, cptr, slots, vol, err,
                              spin, cs);
    if (sgn != sg) __syncthreads();  // end of a level
    sg = sgn;
    pass = passn;
    sgn = sgf;
    passn = passf;
    advance(sgf, passf);
    cur = nxt;
    nxt = far;
    par ^= 1;
  }
  cp_async_wait<0>();
}

// Forward sweep.  chunk_skip > 0 withholds the first chunk_skip chunks
// (failure-detection self-test only: the cells that depend on them wait
// until the bound runs out).
template <int W, int L, bool MX>
__global__ void __launch_bounds__(kWideBlock, kWideMinB)
k_sweep_fwd_wide(const int32_t *__restrict__ seg_begin, const int32_t *__restrict__ segs,
                  const PosCell *__restrict__ pcs,
                  const typename SweepTypes<MX>::Rec *__restrict__ prec,
                  const int32_t *__restrict__ pnb, const int32_t *__restrict__ pslot,
                  const double *__restrict__ q8,
                  const typename SweepTypes<MX>::Q *__restrict__ qnb, double *dqf,
                  double *__restrict__ dqb, const double *__restrict__ res, int32_t C,
                  double *__restrict__ diag, int32_t first_cell, Params P0, int clamp_check,
                  double *__restrict__ dt, const unsigned long long *__restrict__ dt_ext,
                  const int32_t *__restrict__ cptr, const SlotRec *__restrict__ slots,
                  const double *__restrict__ vol, int *err, long long spin,
                  int32_t chunk_skip, Cases cs) {
  if ((int32_t)blockIdx.x < chunk_skip) return;
  wide_chunk<W, L, true, MX>(seg_begin, segs, pcs, prec, pnb, pslot, q8, qnb, dqf, dqf, dqb, res,
                              nullptr, C, diag, first_cell, P0, clamp_check, dt, dt_ext, cptr,
                              slots, vol, err, spin, cs);
}

// Backward sweep.  The state update is k_update_cells, launched after it:
// a separate streaming pass reads each cell's state and increment once in
// cell order, where an update by each block after its chunk (cells in
// chunk order, one after another per thread) took 0.79 ms of the 128^3
// iteration against 0.35 ms.  q8_new and q4_new are unused here (the
// argument list is the deep kernels').
template <int W, int L, bool MX>
__global__ void __launch_bounds__(kWideBlock, kWideMinB)
k_sweep_bwd_wide(const int32_t *__restrict__ seg_begin, const int32_t *__restrict__ segs,
                  const PosCell *__restrict__ pcs,
                  const typename SweepTypes<MX>::Rec *__restrict__ prec,
                  const int32_t *__restrict__ pnb, const int32_t *__restrict__ pslot,
                  const double *__restrict__ q8,
                  const typename SweepTypes<MX>::Q *__restrict__ qnb,
                  double *__restrict__ q8_new, float *__restrict__ q4_new,
                  double *__restrict__ dqf, double *dqb, const double *__restrict__ diag,
                  Params P0, int *err, long long spin, Cases cs) {
  wide_chunk<W, L, false, MX>(seg_begin, segs, pcs, prec, pnb, pslot, q8, qnb, dqb, dqb, dqf,
                               nullptr, dqf, 0, const_cast<double *>(diag), 0, P0, 0, nullptr,
                               nullptr, nullptr, nullptr, nullptr, err, spin, cs);
}

// UpdateFlowField3D_CFL3d (forward_lusgs.cpp:1335-1488) of every cell from
// its state and backward increment, the new state (with a, H, E; and the
// single-precision record of the mixed form) into the other state buffer:
// the update of the wide backward sweeps, one thread per cell.
template <bool MX>
__global__ void __launch_bounds__(kBlock)
k_update_cells(int32_t C, const double *__restrict__ q8, const double *__restrict__ dqb,
               double *__restrict__ q8_new, float *__restrict__ q4_new, Params P0, Cases cs) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double d[5], qc[Q_STRIDE];
  const double2 *pp = reinterpret_cast<const double2 *>(dqb + (int64_t)c * Q_STRIDE);
  const double2 x = pp[0], y = pp[1], z = pp[2];
  d[0] = x.x; d[1] = x.y; d[2] = y.x; d[3] = y.y; d[4] = z.x;
  load_q(q8, c, qc);
  const Params P = params_of(P0, cs, c);
  update_cell(qc, d, P);
  cell_props(qc, P);
  store_q(q8_new, c, qc);
  if (MX) store_q4(q4_new, c, qc);
}

// A node's weighted sums divided by its weight (cal_gradient.cpp:2314-2324),
// then the symmetry-plane projection of the velocity (:2330-2350).
__device__ __forceinline__ void node_finish(int32_t nd, int32_t info,
                                            const double *__restrict__ wnode,
                                            const double *__restrict__ nsym, double acc[5]) {
  const double den = wnode[nd] + kTiny;
  for (int v = 0; v < 5; v++) acc[v] /= den;
  if (info & 2) {
    const double xs = nsym[3 * nd], ys = nsym[3 * nd + 1], zs = nsym[3 * nd + 2];
    const double un = acc[1], vn_ = acc[2], wn = acc[3];
    const double vn = un * xs + vn_ * ys + wn * zs;
    acc[1] = un - vn * xs;
    acc[2] = vn_ - vn * ys;
    acc[3] = wn - vn * zs;
  }
}

// Node values of all five variables (CompNodeVar3D_dist, cal_gradient.cpp
// :1922-2372): boundary-marked nodes average their boundary-face states,
// the others their cells, each in the reference's accumulation order; then
// the symmetry-plane projection of the velocity.
__global__ void __launch_bounds__(kNodeBlock)
k_node_values(int32_t N, int32_t C, const int32_t *__restrict__ nptr,
              const NodeEnt *__restrict__ nsl, const int32_t *__restrict__ nsptr32,
              const int32_t *__restrict__ ninfo, const double *__restrict__ wnode,
              const double *__restrict__ nsym, const int32_t *__restrict__ bface_c1,
              const double *__restrict__ q8, double *__restrict__ qn8) {
  const int32_t nd = blockIdx.x * blockDim.x + threadIdx.x;
  if (nd >= N) return;
  const int32_t info = ninfo[nd];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int32_t ne = nptr[nd + 1] - nptr[nd];
  const NodeEnt *el = nsl + nsptr32[nd / kSlice] + nd % kSlice;  // sliced
  if (info & 1) {
    for (int32_t j = 0; j < ne; j++) {
      const NodeEnt en = el[(int64_t)j * kSlice];
      const int32_t k = en.src;
      const double w = en.w;
      double qa[Q_STRIDE], qb[Q_STRIDE];
      load_q5_w(q8, bface_c1[k], qa);
      load_q5_w(q8, (int64_t)C + k, qb);
      for (int v = 0; v < 5; v++) {
        double facq = qa[v] + qb[v];
        facq *= 0.5;
        acc[v] += facq * w;
      }
    }
  } else {
    for (int32_t j = 0; j < ne; j++) {
      const NodeEnt en = el[(int64_t)j * kSlice];
      double qa[Q_STRIDE];
      load_q5_w(q8, en.src, qa);
      const double w = en.w;
      for (int v = 0; v < 5; v++) acc[v] += qa[v] * w;
    }
  }
  // a node shared with other parts of a partitioned mesh keeps its partial
  // sum until theirs are added (k_halo_nodes)
  if (!(info & 4)) node_finish(nd, info, wnode, nsym, acc);
  double *o = qn8 + (int64_t)nd * Q_STRIDE;
  reinterpret_cast<double2 *>(o)[0] = make_double2(acc[0], acc[1]);
  reinterpret_cast<double2 *>(o)[1] = make_double2(acc[2], acc[3]);
  reinterpret_cast<double2 *>(o)[2] = make_double2(acc[4], 0.0);
}

// Green-Gauss face sums per cell (CompGradientQ_Gauss_Node face loops,
// cal_gradient.cpp:1740-1897), divided by the volume.
__device__ __forceinline__ void grad_faces_cell(
    int32_t c, int32_t C, int64_t n, const int32_t *__restrict__ cptr,
    const GradSlot *__restrict__ rslots, const int32_t *__restrict__ sptr32,
    const int32_t *__restrict__ fnptr,
    const int32_t *__restrict__ fnodes, const double *__restrict__ qn8,
    const double *__restrict__ q8, const double *__restrict__ vol, double *__restrict__ dqdx,
    double *__restrict__ dqdy, double *__restrict__ dqdz) {
  if (c >= C) return;
  double gx[5] = {0., 0., 0., 0., 0.}, gy[5] = {0., 0., 0., 0., 0.},
         gz[5] = {0., 0., 0., 0., 0.};
  const int32_t ns = cptr[c + 1] - cptr[c];
  const GradSlot *sl = rslots + sptr32[c / kSlice] + c % kSlice;  // sliced
  for (int32_t j = 0; j < ns; j++) {
    const GradSlot sr = sl[(int64_t)j * kSlice];
    double qs[5];
    if ((sr.flags & SLOT_BOUNDARY) && !(sr.flags & SLOT_NODE_AVG)) {
      double qc[Q_STRIDE], qg[Q_STRIDE];
      load_q(q8, c, qc);
      load_q(q8, sr.n0, qg);
      for (int v = 0; v < 5; v++) qs[v] = 0.5 * (qc[v] + qg[v]);
    } else {
      for (int v = 0; v < 5; v++) qs[v] = 0.0;
      auto add = [&](int32_t node) {
        double r[5];
        load_q5_w(qn8, node, r);
        qs[0] += r[0];
        qs[1] += r[1];
        qs[2] += r[2];
        qs[3] += r[3];
        qs[4] += r[4];
      };
      int32_t nn = 3;
      if (sr.flags & SLOT_TRI) {
        add(sr.n0);
        add(sr.n1);
        add(sr.n2);
      } else {
        const int32_t j0 = fnptr[sr.n0], j1 = fnptr[sr.n0 + 1];
        for (int32_t j = j0; j < j1; j++) add(fnodes[j]);
        nn = j1 - j0;
      }
      // the mean: a triangle's sums times RN(1/3) with Markstein's
      // correction (the quotient's bits), else the divisions
      const double cnt = (double)nn;
      bool ok = nn == 3;
      double t[5];
      for (int v = 0; v < 5; v++) t[v] = quot_pos(qs[v], 3.0, kRcp3, ok);
      if (ok) {
        for (int v = 0; v < 5; v++) qs[v] = t[v];
      } else {
        for (int v = 0; v < 5; v++) qs[v] /= cnt;
      }
    }
    const bool minus = (sr.flags & SLOT_IS_C2) != 0;
    for (int v = 0; v < 5; v++) {
      const double qsum = qs[v] * sr.area;
      const double tx = qsum * sr.nx, ty = qsum * sr.ny, tz = qsum * sr.nz;
      if (minus) {
        gx[v] -= tx;
        gy[v] -= ty;
        gz[v] -= tz;
      } else {
        gx[v] += tx;
        gy[v] += ty;
        gz[v] += tz;
      }
    }
  }
  // the 15 quotients by the volume from one reciprocal (the divisions when
  // an operand is outside the window)
  const double vc = vol[c];
  bool ok;
  const double y = rcp_rn_fast(vc, ok);
  double tx[5], ty[5], tz[5];
  for (int v = 0; v < 5; v++) {
    tx[v] = quot_pos(gx[v], vc, y, ok);
    ty[v] = quot_pos(gy[v], vc, y, ok);
    tz[v] = quot_pos(gz[v], vc, y, ok);
  }
  if (!(vc > 0.0)) ok = false;
  if (!ok) {
    for (int v = 0; v < 5; v++) {
      tx[v] = gx[v] / vc;
      ty[v] = gy[v] / vc;
      tz[v] = gz[v] / vc;
    }
  }
  for (int v = 0; v < 5; v++) {
    dqdx[v * n + c] = tx[v];
    dqdy[v * n + c] = ty[v];
    dqdz[v * n + c] = tz[v];
  }
}

__global__ void __launch_bounds__(kGradBlockMax)
k_grad_faces(int32_t C, int64_t n, const int32_t *__restrict__ cptr,
             const GradSlot *__restrict__ rslots, const int32_t *__restrict__ sptr32,
             const int32_t *__restrict__ fnptr,
             const int32_t *__restrict__ fnodes, const double *__restrict__ qn8,
             const double *__restrict__ q8, const double *__restrict__ vol,
             double *__restrict__ dqdx, double *__restrict__ dqdy, double *__restrict__ dqdz) {
  grad_faces_cell(blockIdx.x * blockDim.x + threadIdx.x, C, n, cptr, rslots, sptr32, fnptr,
                  fnodes, qn8, q8, vol, dqdx, dqdy, dqdz);
}

// Mixed form of node_finish: the sums (deviations from the freestream) times
// the reciprocal of the weight, then the symmetry-plane projection of the
// velocity (of value = freestream + deviation).
__device__ __forceinline__ void node_finish_mx(int32_t nd, int32_t info,
                                               const double *__restrict__ wnode,
                                               const double *__restrict__ nsym, const Params &P,
                                               float acc[5]) {
  const float rden = __fdividef(1.0f, (float)(wnode[nd] + kTiny));
  for (int v = 0; v < 5; v++) acc[v] *= rden;
  if (info & 2) {
    const float xs = (float)nsym[3 * nd], ys = (float)nsym[3 * nd + 1], zs = (float)nsym[3 * nd + 2];
    const float vn = acc[1] * xs + acc[2] * ys + acc[3] * zs +
                     (float)(P.ref[1] * nsym[3 * nd] + P.ref[2] * nsym[3 * nd + 1] +
                             P.ref[3] * nsym[3 * nd + 2]);
    acc[1] -= vn * xs;
    acc[2] -= vn * ys;
    acc[3] -= vn * zs;
  }
}

// Mixed form of the gradient: node values and Green-Gauss face sums in FP32
// over the same loops as the FP64 kernels above, carried as deviations from
// the freestream state (formed in FP64 from the FP64 records): the reference
// state drops out of a closed cell's face sum, so FP32 rounding scales with
// the deviations instead of with the values.  Gradients stored in FP64.
__global__ void __launch_bounds__(kNodeBlock)
k_node_values_mx(int32_t N, int32_t C, const int32_t *__restrict__ nptr,
                 const NodeEnt *__restrict__ nsl, const int32_t *__restrict__ nsptr32,
                 const int32_t *__restrict__ ninfo, const double *__restrict__ wnode,
                 const double *__restrict__ nsym, const int32_t *__restrict__ bface_c1,
                 const double *__restrict__ q8, float *__restrict__ qn4, Params P0, Cases cs) {
  const int32_t nd = blockIdx.x * blockDim.x + threadIdx.x;
  if (nd >= N) return;
  const int32_t info = ninfo[nd];
  float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  const int32_t ne = nptr[nd + 1] - nptr[nd];
  const NodeEnt *el = nsl + nsptr32[nd / kSlice] + nd % kSlice;  // sliced
  // the case of a node is that of any cell it touches
  const Params P = ne > 0 ? params_of(P0, cs, (info & 1) ? bface_c1[el[0].src] : el[0].src) : P0;
  if (info & 1) {
    for (int32_t j = 0; j < ne; j++) {
      const NodeEnt en = el[(int64_t)j * kSlice];
      const int32_t k = en.src;
      const float w = (float)en.w;
      double qa[Q_STRIDE], qb[Q_STRIDE];
      load_q5_w(q8, bface_c1[k], qa);
      load_q5_w(q8, (int64_t)C + k, qb);
      for (int v = 0; v < 5; v++)
        acc[v] += (float)(0.5 * ((qa[v] - P.ref[v]) + (qb[v] - P.ref[v]))) * w;
    }
  } else {
    for (int32_t j = 0; j < ne; j++) {
      const NodeEnt en = el[(int64_t)j * kSlice];
      double qa[Q_STRIDE];
      load_q5_w(q8, en.src, qa);
      const float w = (float)en.w;
      for (int v = 0; v < 5; v++) acc[v] += (float)(qa[v] - P.ref[v]) * w;
    }
  }
  // a node shared with other parts keeps its partial sum (k_halo_nodes_mx)
  if (!(info & 4)) node_finish_mx(nd, info, wnode, nsym, P, acc);
  float4 *o = reinterpret_cast<float4 *>(qn4 + (int64_t)nd * Q_STRIDE);
  o[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
  o[1] = make_float4(acc[4], 0.f, 0.f, 0.f);
}

__global__ void __launch_bounds__(kGradBlockMax)
k_grad_faces_mx(int32_t C, int64_t n, const int32_t *__restrict__ cptr,
                const GradSlot *__restrict__ rslots, const int32_t *__restrict__ sptr32,
                const int32_t *__restrict__ fnptr,
                const int32_t *__restrict__ fnodes, const float *__restrict__ qn4,
                const double *__restrict__ q8, const double *__restrict__ vol,
                double *__restrict__ dqdx, double *__restrict__ dqdy, double *__restrict__ dqdz,
                Params P0, Cases cs) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const Params P = params_of(P0, cs, c);
  float gx[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, gy[5] = {0.f, 0.f, 0.f, 0.f, 0.f},
        gz[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  const int32_t ns = cptr[c + 1] - cptr[c];
  const GradSlot *sl = rslots + sptr32[c / kSlice] + c % kSlice;  // sliced
  for (int32_t j = 0; j < ns; j++) {
    const GradSlot sr = sl[(int64_t)j * kSlice];
    float qs[5];
    if ((sr.flags & SLOT_BOUNDARY) && !(sr.flags & SLOT_NODE_AVG)) {
      double qc[Q_STRIDE], qg[Q_STRIDE];
      load_q(q8, c, qc);
      load_q(q8, sr.n0, qg);
      for (int v = 0; v < 5; v++) qs[v] = (float)(0.5 * ((qc[v] - P.ref[v]) + (qg[v] - P.ref[v])));
    } else {
      for (int v = 0; v < 5; v++) qs[v] = 0.f;
      auto add = [&](int32_t node) {
        float r[8];
        ldg_v8f(qn4 + (int64_t)node * Q_STRIDE, r);
        qs[0] += r[0];
        qs[1] += r[1];
        qs[2] += r[2];
        qs[3] += r[3];
        qs[4] += r[4];
      };
      int32_t nn = 3;
      if (sr.flags & SLOT_TRI) {
        add(sr.n0);
        add(sr.n1);
        add(sr.n2);
      } else {
        const int32_t j0 = fnptr[sr.n0], j1 = fnptr[sr.n0 + 1];
        for (int32_t j = j0; j < j1; j++) add(fnodes[j]);
        nn = j1 - j0;
      }
      const float rc = __fdividef(1.0f, (float)nn);
      for (int v = 0; v < 5; v++) qs[v] *= rc;
    }
    const float sg = (sr.flags & SLOT_IS_C2) ? -(float)sr.area : (float)sr.area;
    const float nx = (float)sr.nx, ny = (float)sr.ny, nz = (float)sr.nz;
    for (int v = 0; v < 5; v++) {
      const float qsum = qs[v] * sg;
      gx[v] += qsum * nx;
      gy[v] += qsum * ny;
      gz[v] += qsum * nz;
    }
  }
  const float rv = __fdividef(1.0f, (float)vol[c]);
  for (int v = 0; v < 5; v++) {
    dqdx[v * n + c] = (double)(gx[v] * rv);
    dqdy[v * n + c] = (double)(gy[v] * rv);
    dqdz[v * n + c] = (double)(gz[v] * rv);
  }
}

// Green-Gauss face sums with one lane per (cell, face) slot (L lanes per
// cell, L at least its face count): each lane forms its face's value (the
// mean of the face's node values, or of the cell and ghost states) and its
// area-weighted normal components; the 15 sums are folds over the slots in
// ascending face order passed from lane to lane (a difference as the sum with
// the negated term, exactly), so the same bits as grad_faces_cell (FP64) and
// k_grad_faces_mx (mixed: FP32 sums of deviations from the freestream).
template <int L, bool MX>
__global__ void __launch_bounds__(kGradBlockMax)
k_grad_faces_lanes(int32_t C, int64_t n, const int32_t *__restrict__ cptr,
                   const SlotRec *__restrict__ slots, const int32_t *__restrict__ fnptr,
                   const int32_t *__restrict__ fnodes, const double *__restrict__ qn8,
                   const float *__restrict__ qn4, const double *__restrict__ q8,
                   const double *__restrict__ vol, double *__restrict__ dqdx,
                   double *__restrict__ dqdy, double *__restrict__ dqdz, Params P0, Cases cs) {
  using T = typename std::conditional<MX, float, double>::type;
  static_assert((L & (L - 1)) == 0 && L >= 2 && L <= 32, "lanes per cell");
  const int64_t cl = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / L;
  const bool live = cl < C;
  const int32_t c = live ? (int32_t)cl : 0;
  const int lane = threadIdx.x & (L - 1);
  int32_t s0 = 0, ns = 0;
  if (live) {
    s0 = __ldg(cptr + c);
    ns = __ldg(cptr + c + 1) - s0;
  }
  const bool has = live && lane < ns;
  // this lane's face: value qs and weight a n (sign folded in)
  T qs[5] = {0, 0, 0, 0, 0};
  T ax = 0, ay = 0, az = 0, aw = 0;
  bool minus = false;
  double dnx = 0.0, dny = 0.0, dnz = 0.0, darea = 0.0;
  if (has) {
    const SlotRec sr = slots[s0 + lane];
    if ((sr.flags & SLOT_BOUNDARY) && !(sr.flags & SLOT_NODE_AVG)) {
      double qc[Q_STRIDE], qg[Q_STRIDE];
      load_q(q8, c, qc);
      load_q(q8, sr.nb, qg);
      if (MX) {
        const Params P = params_of(P0, cs, c);
#pragma unroll
        for (int v = 0; v < 5; v++)
          qs[v] = (T)(0.5 * ((qc[v] - P.ref[v]) + (qg[v] - P.ref[v])));
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) qs[v] = (T)(0.5 * (qc[v] + qg[v]));
      }
    } else {
      auto add = [&](int32_t node) {
        if (MX) {
          const float4 *p = reinterpret_cast<const float4 *>(qn4 + (int64_t)node * Q_STRIDE);
          const float4 a = __ldg(p), b = __ldg(p + 1);
          qs[0] += (T)a.x;
          qs[1] += (T)a.y;
          qs[2] += (T)a.z;
          qs[3] += (T)a.w;
          qs[4] += (T)b.x;
        } else {
          const double2 *p = reinterpret_cast<const double2 *>(qn8 + (int64_t)node * Q_STRIDE);
          const double2 a = __ldg(p), b = __ldg(p + 1), e = __ldg(p + 2);
          qs[0] += (T)a.x;
          qs[1] += (T)a.y;
          qs[2] += (T)b.x;
          qs[3] += (T)b.y;
          qs[4] += (T)e.x;
        }
      };
      int32_t nn = 3;
      if (sr.flags & SLOT_TRI) {
        add(sr.tri[0]);
        add(sr.tri[1]);
        add(sr.tri[2]);
      } else {
        const int32_t j0 = fnptr[sr.face], j1 = fnptr[sr.face + 1];
        for (int32_t j = j0; j < j1; j++) add(fnodes[j]);
        nn = j1 - j0;
      }
      if (MX) {
        const float rc = __fdividef(1.0f, (float)nn);
#pragma unroll
        for (int v = 0; v < 5; v++) qs[v] = (T)((float)qs[v] * rc);
      } else {
        const double cnt = (double)nn;
#pragma unroll
        for (int v = 0; v < 5; v++) qs[v] = (T)((double)qs[v] / cnt);
      }
    }
    minus = (sr.flags & SLOT_IS_C2) != 0;
    if (MX) {
      aw = (T)(minus ? -(float)sr.area : (float)sr.area);
      ax = (T)(float)sr.nx;
      ay = (T)(float)sr.ny;
      az = (T)(float)sr.nz;
    } else {
      darea = sr.area;
      dnx = sr.nx;
      dny = sr.ny;
      dnz = sr.nz;
    }
  }
  // this lane's 15 terms: FP64 (qs area) n, negated for the second cell;
  // mixed (qs (+-area)) n
  auto terms = [&](int v, T &tx, T &ty, T &tz) {
    if (MX) {
      const T qsum = qs[v] * aw;
      tx = qsum * ax;
      ty = qsum * ay;
      tz = qsum * az;
    } else {
      const double qsum = (double)qs[v] * darea;
      const double x = qsum * dnx, y = qsum * dny, z = qsum * dnz;
      tx = (T)(minus ? -x : x);
      ty = (T)(minus ? -y : y);
      tz = (T)(minus ? -z : z);
    }
  };
  T gx[5], gy[5], gz[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    T tx, ty, tz;
    terms(v, tx, ty, tz);
    gx[v] = (lane == 0 && has) ? (T)0 + tx : (T)0;
    gy[v] = (lane == 0 && has) ? (T)0 + ty : (T)0;
    gz[v] = (lane == 0 && has) ? (T)0 + tz : (T)0;
  }
#pragma unroll
  for (int j = 1; j < L; j++) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const T px = __shfl_up_sync(0xffffffffu, gx[v], 1, L);
      const T py = __shfl_up_sync(0xffffffffu, gy[v], 1, L);
      const T pz = __shfl_up_sync(0xffffffffu, gz[v], 1, L);
      if (lane == j) {
        T tx, ty, tz;
        terms(v, tx, ty, tz);
        gx[v] = has ? px + tx : px;
        gy[v] = has ? py + ty : py;
        gz[v] = has ? pz + tz : pz;
      }
    }
  }
  if (lane != L - 1 || !live) return;
  if (MX) {
    const float rv = __fdividef(1.0f, (float)vol[c]);
#pragma unroll
    for (int v = 0; v < 5; v++) {
      dqdx[v * n + c] = (double)((float)gx[v] * rv);
      dqdy[v * n + c] = (double)((float)gy[v] * rv);
      dqdz[v * n + c] = (double)((float)gz[v] * rv);
    }
  } else {
    const double vc = vol[c];
#pragma unroll
    for (int v = 0; v < 5; v++) {
      dqdx[v * n + c] = (double)gx[v] / vc;
      dqdy[v * n + c] = (double)gy[v] / vc;
      dqdz[v * n + c] = (double)gz[v] / vc;
    }
  }
}

// Residual norm from res (main.cpp:294-317) as fixed-order block partials.
__global__ void k_norm_partial(int32_t C, const double *__restrict__ res,
                               double *__restrict__ part) {
  __shared__ double sh[kBlock / 32][5];
  double s2[5] = {0., 0., 0., 0., 0.};
  for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x)
    for (int k = 0; k < 5; k++) {
      const double r = res[(int64_t)k * C + c];
      s2[k] += r * r;
    }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 5; k++) s2[k] += __shfl_down_sync(0xffffffffu, s2[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 5; k++) sh[threadIdx.x >> 5][k] = s2[k];
  __syncthreads();
  if (threadIdx.x < 5) {
    double acc = 0.0;
    for (int w = 0; w < kBlock / 32; w++) acc += sh[w][threadIdx.x];
    part[(int64_t)blockIdx.x * 5 + threadIdx.x] = acc;
  }
}

// Final reduction of the partials; also advances the fused-loop counter.
// The sums over b < nparts of part[b][k] (k < 5) in a fixed order: thread t
// of the block (kNormThreads) adds b = t, t + kNormThreads, ... in turn, then
// a tree over the threads halves them in fixed pairs.  sh[k][0] holds sum k.
constexpr int kNormThreads = 1024;
__device__ __forceinline__ void norm_parts_sum(int32_t nparts, const double *__restrict__ part,
                                               double (*sh)[kNormThreads]) {
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
  for (int32_t b = threadIdx.x; b < nparts; b += kNormThreads)
#pragma unroll
    for (int k = 0; k < 5; k++) acc[k] += part[(int64_t)b * 5 + k];
#pragma unroll
  for (int k = 0; k < 5; k++) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = kNormThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 5; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kNormThreads)
k_norm_final(int32_t nparts, const double *__restrict__ part, double *__restrict__ out,
             int32_t *__restrict__ iter_counter, double *__restrict__ hist) {
  __shared__ double sh[5][kNormThreads];
  norm_parts_sum(nparts, part, sh);
  if (threadIdx.x < 5) {
    const double v = sqrt(sh[threadIdx.x][0]);
    out[threadIdx.x] = v;
    if (hist) hist[(int64_t)(*iter_counter) * 5 + threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0 && iter_counter) *iter_counter += 1;
}

// Batched cases: residual norms per case.  Block (x, k) reduces cells
// [cell0[k], cell0[k+1]) with stride gridDim.x * blockDim.x; fixed order.
__global__ void k_norm_seg_partial(int32_t C, const double *__restrict__ res,
                                   const int32_t *__restrict__ cell0, double *__restrict__ part) {
  __shared__ double sh[kBlock / 32][5];
  const int32_t k = blockIdx.y;
  double s2[5] = {0., 0., 0., 0., 0.};
  for (int32_t c = cell0[k] + blockIdx.x * blockDim.x + threadIdx.x; c < cell0[k + 1];
       c += gridDim.x * blockDim.x)
    for (int v = 0; v < 5; v++) {
      const double r = res[(int64_t)v * C + c];
      s2[v] += r * r;
    }
  for (int o = 16; o > 0; o >>= 1)
    for (int v = 0; v < 5; v++) s2[v] += __shfl_down_sync(0xffffffffu, s2[v], o);
  if ((threadIdx.x & 31) == 0)
    for (int v = 0; v < 5; v++) sh[threadIdx.x >> 5][v] = s2[v];
  __syncthreads();
  if (threadIdx.x < 5) {
    double acc = 0.0;
    for (int w = 0; w < kBlock / 32; w++) acc += sh[w][threadIdx.x];
    part[((int64_t)k * gridDim.x + blockIdx.x) * 5 + threadIdx.x] = acc;
  }
}

__global__ void k_norm_seg_final(int32_t nparts, const double *__restrict__ part,
                                 double *__restrict__ out, const int32_t *__restrict__ iter_counter,
                                 double *__restrict__ hist) {
  const int32_t k = blockIdx.x;
  if (threadIdx.x < 5) {
    double acc = 0.0;
    for (int32_t b = 0; b < nparts; b++) acc += part[((int64_t)k * nparts + b) * 5 + threadIdx.x];
    const double v = sqrt(acc);
    out[k * 5 + threadIdx.x] = v;
    if (hist) hist[((int64_t)(*iter_counter) * gridDim.x + k) * 5 + threadIdx.x] = v;
  }
}

__global__ void k_counter_inc(int32_t *__restrict__ counter) { *counter += 1; }

// Self-test of div_by_recip against the division: n dividend/divisor pairs
// from a splitmix64 stream, significands uniform, exponents uniform in
// [-600, 600] (both sides of div_by_recip's window) and random signs; every
// fourth divisor has an all-ones significand.  Counts the pairs whose bits
// differ.
__device__ __forceinline__ uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double draw_double(uint64_t &x, bool all_ones) {
  const uint64_t r = splitmix64(x), e = splitmix64(x);
  const uint64_t mant = all_ones ? 0xFFFFFFFFFFFFFull : (r & 0xFFFFFFFFFFFFFull);
  const uint64_t expo = (uint64_t)(1023 - 600 + (int64_t)(e % 1201));
  return __longlong_as_double((long long)(((r >> 63) << 63) | (expo << 52) | mant));
}

__global__ void k_selftest_division(int64_t n, uint64_t seed,
                                    unsigned long long *__restrict__ bad) {
  unsigned long long local = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t x = seed ^ ((uint64_t)i * 0xD1B54A32D192ED03ull);
    const double a = draw_double(x, false);
    const double b = draw_double(x, (i & 3) == 3);
    const double y = 1.0 / b;
    const double q = div_by_recip(a, b, y), ref = a / b;
    if (__double_as_longlong(q) != __double_as_longlong(ref)) local++;
  }
  if (local) atomicAdd(bad, local);
}

// Known-answer self-test of the device arithmetic: the device functions the
// iteration kernels call (roe_flux, flux_lusgs through its pre/fin split,
// update_cell with cell_props before each) on caller-given inputs, one
// thread per input.  mode 0: RoeFlux_noprec, in = ql[5][n], qr[5][n],
// nx[n], ny[n], nz[n], area[n] -> out[5][n]; mode 1: FluxLUSGS3D, in =
// [n][13] (q[5], dq[5], normal[3]) -> out[n][5]; mode 2:
// UpdateFlowField3D_CFL3d, in = q[5][n], dq[5][n] -> out[5][n].
__global__ void k_selftest_functions(int mode, int32_t n, Params P, const double *__restrict__ in,
                                     double *__restrict__ out) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t m = n;
  if (mode == 0) {
    double ql[Q_STRIDE], qr[Q_STRIDE], f[5];
    for (int k = 0; k < 5; k++) {
      ql[k] = in[k * m + i];
      qr[k] = in[(5 + k) * m + i];
    }
    cell_props(ql, P);
    cell_props(qr, P);
    roe_flux(ql, qr, in[10 * m + i], in[11 * m + i], in[12 * m + i], in[13 * m + i], P, f);
    for (int k = 0; k < 5; k++) out[k * m + i] = f[k];
  } else if (mode == 1 || mode == 3) {
    const double *c = in + 13 * (int64_t)i;
    double q[Q_STRIDE], dq[5], f[5];
    for (int k = 0; k < 5; k++) {
      q[k] = c[k];
      dq[k] = c[5 + k];
    }
    cell_props(q, P);
    const FluxP<double> fp = flux_params<double>(P);
    const LusgsPre<double> a = flux_lusgs_pre(q, c[10], c[11], c[12], fp);
    bool ok = false;
    if (mode == 3) flux_lusgs_fin_fast(a, dq, c[10], c[11], c[12], fp, f, ok);
    if (!ok) flux_lusgs_fin(a, dq, c[10], c[11], c[12], fp, f);
    for (int k = 0; k < 5; k++) out[5 * (int64_t)i + k] = f[k];
  } else {
    double q[Q_STRIDE], dq[5];
    for (int k = 0; k < 5; k++) {
      q[k] = in[k * m + i];
      dq[k] = in[(5 + k) * m + i];
    }
    cell_props(q, P);
    update_cell(q, dq, P);
    for (int k = 0; k < 5; k++) out[k * m + i] = q[k];
  }
}

// Self-test of the branch-free reciprocal and quotient against the division:
// divisors with exponents across [-130, 130] (both sides of rcp_rn_fast's
// window), significands uniform, and every eighth one all ones (routed to
// the division), every eighth + 1 all ones but the last bit, every eighth +
// 2 a power of two.  Counts bad[0] reciprocals and bad[1] quotients (both
// fast forms taken) whose bits differ from the division's, bad[2] divisors
// outside the fast path.
__global__ void k_selftest_division_fast(int64_t n, uint64_t seed,
                                         unsigned long long *__restrict__ bad) {
  unsigned long long b0 = 0, b1 = 0, b2 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t x = seed ^ ((uint64_t)i * 0xD1B54A32D192ED03ull);
    const uint64_t r = splitmix64(x), e = splitmix64(x), ra = splitmix64(x), ea = splitmix64(x);
    uint64_t mant = r & 0xFFFFFFFFFFFFFull;
    if ((i & 7) == 0) mant = 0xFFFFFFFFFFFFFull;
    if ((i & 7) == 1) mant = 0xFFFFFFFFFFFFEull;
    if ((i & 7) == 2) mant = 0;
    const uint64_t expo = (uint64_t)(1023 - 130 + (int64_t)(e % 261));
    const double b = __longlong_as_double((long long)(((r >> 63) << 63) | (expo << 52) | mant));
    const uint64_t expa = (uint64_t)(1023 - 400 + (int64_t)(ea % 801));
    const double a = __longlong_as_double(
        (long long)(((ra >> 63) << 63) | (expa << 52) | (ra & 0xFFFFFFFFFFFFFull)));
    bool ok;
    const double y = rcp_rn_fast(b, ok);
    if (!ok) {
      b2++;
      continue;
    }
    if (__double_as_longlong(y) != __double_as_longlong(1.0 / b)) b0++;
    bool okq;
    const double q = div_recip_fast(a, b, y, okq);
    if (okq && __double_as_longlong(q) != __double_as_longlong(a / b)) b1++;
  }
  if (b0) atomicAdd(bad, b0);
  if (b1) atomicAdd(bad + 1, b1);
  if (b2) atomicAdd(bad + 2, b2);
}

// ---- one part of a partitioned mesh (the reference's MPI mode) ------------

// The partials of k_norm_final, summed in its order, left squared: a part's
// share of main.cpp:311-312's MPI_Reduce.
__global__ void __launch_bounds__(kNormThreads)
k_norm_sums(int32_t nparts, const double *__restrict__ part, double *__restrict__ out) {
  __shared__ double sh[5][kNormThreads];
  norm_parts_sum(nparts, part, sh);
  if (threadIdx.x < 5) out[threadIdx.x] = sh[threadIdx.x][0];
}

// Rows (Q_STRIDE doubles) of the listed records into a packed buffer [n][8];
// words from `width` on are written as 0.  One thread per word.
__global__ void k_halo_gather(int32_t n, int32_t width, const int32_t *__restrict__ idx,
                              const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * Q_STRIDE) return;
  const int32_t i = (int32_t)(t / Q_STRIDE), k = (int32_t)(t % Q_STRIDE);
  dst[t] = k < width ? src[(int64_t)idx[i] * Q_STRIDE + k] : 0.0;
}

// A packed buffer [n][8] into the listed rows of one or two arrays (words
// below `width`).
// (the mixed form's state records: also the single-precision mirrors fa, fb)
__global__ void k_halo_scatter(int32_t n, int32_t width, const int32_t *__restrict__ rows,
                               const double *__restrict__ src, double *__restrict__ a,
                               double *__restrict__ b, float *__restrict__ fa,
                               float *__restrict__ fb) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * Q_STRIDE) return;
  const int32_t i = (int32_t)(t / Q_STRIDE), k = (int32_t)(t % Q_STRIDE);
  if (k >= width) return;
  const int64_t o = (int64_t)rows[i] * Q_STRIDE + k;
  const double v = src[t];
  a[o] = v;
  if (b) b[o] = v;
  if (fa) fa[o] = (float)v;
  if (fb) fb[o] = (float)v;
}

// Mixed form: single-precision node rows into a packed double buffer.
__global__ void k_halo_gather_f(int32_t n, int32_t width, const int32_t *__restrict__ idx,
                                const float *__restrict__ src, double *__restrict__ dst) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * Q_STRIDE) return;
  const int32_t i = (int32_t)(t / Q_STRIDE), k = (int32_t)(t % Q_STRIDE);
  dst[t] = k < width ? (double)src[(int64_t)idx[i] * Q_STRIDE + k] : 0.0;
}

// Second order across parts: a sent cell's gradient rows (x, y, z of the
// five variables), limiter (1 without one) and centroid into a packed row of
// kGradRow doubles, and a received row into the ghost's places.
constexpr int kGradRow = 24;

__global__ void k_halo_pack_grad(int32_t m, const int32_t *__restrict__ cells, int64_t n,
                                 const double *__restrict__ dqdx, const double *__restrict__ dqdy,
                                 const double *__restrict__ dqdz, const double *__restrict__ phi,
                                 const Cen *__restrict__ ccen, double *__restrict__ out) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t c = cells[i];
  double *o = out + (int64_t)i * kGradRow;
  for (int v = 0; v < 5; v++) {
    o[v] = dqdx[(int64_t)v * n + c];
    o[5 + v] = dqdy[(int64_t)v * n + c];
    o[10 + v] = dqdz[(int64_t)v * n + c];
    o[15 + v] = phi ? phi[(int64_t)v * n + c] : 1.0;
  }
  const Cen cc = ccen[c];
  o[20] = cc.x;
  o[21] = cc.y;
  o[22] = cc.z;
  o[23] = cc.h;
}

__global__ void k_halo_unpack_grad(int32_t m, const int32_t *__restrict__ rows, int64_t n,
                                   const double *__restrict__ in, double *__restrict__ dqdx,
                                   double *__restrict__ dqdy, double *__restrict__ dqdz,
                                   double *__restrict__ phi, Cen *__restrict__ ccen) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t g = rows[i];
  const double *r = in + (int64_t)i * kGradRow;
  for (int v = 0; v < 5; v++) {
    dqdx[(int64_t)v * n + g] = r[v];
    dqdy[(int64_t)v * n + g] = r[5 + v];
    dqdz[(int64_t)v * n + g] = r[10 + v];
    if (phi) phi[(int64_t)v * n + g] = r[15 + v];
  }
  ccen[g] = Cen{r[20], r[21], r[22], r[23]};
}

// Shared nodes: the local partial sums plus each neighbour's (in entry
// order, RecvSendVarNeighbor_Node, parallel_mpi.cpp:1997-2004), then the
// division and projection of every node (cal_gradient.cpp:2314-2350).
__global__ void k_halo_nodes(int32_t nu, const int32_t *__restrict__ unodes,
                             const int32_t *__restrict__ eptr, const int32_t *__restrict__ eidx,
                             const double *__restrict__ recv, const int32_t *__restrict__ ninfo,
                             const double *__restrict__ wnode, const double *__restrict__ nsym,
                             double *__restrict__ qn8) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nu) return;
  const int32_t nd = unodes[i];
  double *o = qn8 + (int64_t)nd * Q_STRIDE;
  double acc[5];
  for (int v = 0; v < 5; v++) acc[v] = o[v];
  for (int32_t e = eptr[i]; e < eptr[i + 1]; e++) {
    const double *r = recv + (int64_t)eidx[e] * Q_STRIDE;
    for (int v = 0; v < 5; v++) acc[v] += r[v];
  }
  node_finish(nd, ninfo[nd], wnode, nsym, acc);
  for (int v = 0; v < 5; v++) o[v] = acc[v];
}

// Mixed form of k_halo_nodes (partial sums in single precision).
__global__ void k_halo_nodes_mx(int32_t nu, const int32_t *__restrict__ unodes,
                                const int32_t *__restrict__ eptr,
                                const int32_t *__restrict__ eidx, const double *__restrict__ recv,
                                const int32_t *__restrict__ ninfo,
                                const double *__restrict__ wnode,
                                const double *__restrict__ nsym, Params P,
                                float *__restrict__ qn4) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nu) return;
  const int32_t nd = unodes[i];
  float *o = qn4 + (int64_t)nd * Q_STRIDE;
  float acc[5];
  for (int v = 0; v < 5; v++) acc[v] = o[v];
  for (int32_t e = eptr[i]; e < eptr[i + 1]; e++) {
    const double *r = recv + (int64_t)eidx[e] * Q_STRIDE;
    for (int v = 0; v < 5; v++) acc[v] += (float)r[v];
  }
  node_finish_mx(nd, ninfo[nd], wnode, nsym, P, acc);
  for (int v = 0; v < 5; v++) o[v] = acc[v];
}

}  // namespace

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

// The persistent sweep kernel for (W, precision) and its dynamic shared
// memory.
// kind MFG_SWEEP_DEEP: the warp-specialised kernels (one block per SM);
// MFG_SWEEP_WIDE: the many-block kernels for wide levels.
static const void *sweep_kernel(bool fwd, int w, bool mx, int kind = MFG_SWEEP_DEEP) {
#define MFG_SK(W_)                                                                           \
  if (w == W_ && kind == MFG_SWEEP_DEEP)                                                     \
    return fwd ? (mx ? (const void *)k_sweep_fwd_chunk<W_, true>                               \
                     : (const void *)k_sweep_fwd_chunk<W_, false>)                             \
               : (mx ? (const void *)k_sweep_bwd_chunk<W_, true>                               \
                     : (const void *)k_sweep_bwd_chunk<W_, false>);                            \
  if (w == W_ && kind == MFG_SWEEP_WIDE)                                                     \
    return fwd ? (mx ? (const void *)k_sweep_fwd_wide<W_, W_, true>                            \
                     : (const void *)k_sweep_fwd_wide<W_, W_, false>)                          \
               : (mx ? (const void *)k_sweep_bwd_wide<W_, W_, true>                            \
                     : (const void *)k_sweep_bwd_wide<W_, W_, false>);
  MFG_SK(4)
  MFG_SK(8)
#undef MFG_SK
  return nullptr;
}
static int sweep_threads(int w, int kind = MFG_SWEEP_DEEP) {
  if (kind == MFG_SWEEP_WIDE) return kWideBlock;
  return w == 8 ? WsGeom<8>::kThreads : WsGeom<4>::kThreads;
}
static size_t sweep_smem(int w, bool mx, int kind = MFG_SWEEP_DEEP) {
  if (kind == MFG_SWEEP_WIDE) return 0;
  if (w == 8) return mx ? ws_smem_bytes<8, true>() : ws_smem_bytes<8, false>();
  return mx ? ws_smem_bytes<4, true>() : ws_smem_bytes<4, false>();
}
// Cells per work item (lane groups of a block) and ring positions of a
// kernel kind.
static int32_t sweep_groups(int w, int kind = MFG_SWEEP_DEEP) {
  if (kind == MFG_SWEEP_WIDE) return kWideBlock / std::max(w, 1);
  return w == 8 ? WsGeom<8>::kGroups : WsGeom<4>::kGroups;
}
static int32_t sweep_ring(int kind) { return kind == MFG_SWEEP_WIDE ? kWideRing : kRing; }

struct ChunkSweep {
  int32_t *seg_begin = nullptr, *segs = nullptr, *nbs = nullptr, *nslots = nullptr;
  PosCell *cells = nullptr;
  SweepRec *recs = nullptr;
  SweepRecF *recs_f = nullptr;  // mixed form
  int32_t nseg = 0;
};

struct mfg_ctx {
  int device = 0;
  int precision = MFG_PREC_FP64;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  // mfg_iterate_host: results copied out on a second stream while the last
  // iteration's later kernels run
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_res = nullptr, ev_state = nullptr;
  // fused iterations: the gradient of the state an iteration starts from
  // runs on a second stream beside that iteration's face kernels
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int32_t C = 0, G = 0, F = 0, N = 0;
  int64_t n = 0, S = 0;
  mfg_params hp{};
  Params P{};
  int first_cell = 0;
  bool res_zero = true;
  int cur = 0;
  int sweep_mode = 0;
  // device arrays
  double *q8[2] = {nullptr, nullptr};
  // mixed form: single-precision state records (kept with q8[cur]) and node
  // values
  float *q4[2] = {nullptr, nullptr};
  float *qn4 = nullptr;
  double *dq8 = nullptr, *res = nullptr, *dt = nullptr, *diag = nullptr;
  double *dqdx = nullptr, *dqdy = nullptr, *dqdz = nullptr, *qn8 = nullptr;
  double *vol = nullptr, *staging = nullptr;
  int32_t *cptr = nullptr;
  SlotRec *slots = nullptr;
  // the slots again, sliced: the cells in slices of kSlice (a warp), slot j
  // of the slice's lane t at sptr32[slice] + j kSlice + t, so that a warp's
  // one-thread-per-cell gathers read consecutive records
  GatherSlot *gslots = nullptr;
  GradSlot *rslots = nullptr;
  int32_t *sptr32 = nullptr;
  FaceRec *faces = nullptr;  // per-face flux: normal, area, cells
  double *fflux = nullptr;   // per-face flux rows [F][kFluxRow]
  int32_t *bctype_d = nullptr;  // BC type of each boundary face [G]
  int32_t live_bc = 0;          // ghost states recomputed every iteration
  int32_t flux_fp64 = 0;        // mixed form: the Roe flux wholly in FP64
  // second-order reconstruction (the reference's `order`: 1 first order, 2
  // unlimited, 3 Barth-Jespersen, 4 Venkatakrishnan)
  int32_t order = 1;
  double venkat_k = 5.0;
  Cen *fcen = nullptr, *ccen = nullptr;  // face centroids [F], cell centroids + h [n]
  double *phi = nullptr;                 // limiter [5][C]
  int32_t *fnptr = nullptr, *fnodes = nullptr;
  int32_t *nptr = nullptr, *nsrc = nullptr, *ninfo = nullptr, *bface_c1 = nullptr;
  // the node lists again, sliced like the slot records (entry j of the
  // slice's lane t at nsptr32[slice] + j kSlice + t)
  NodeEnt *nsl = nullptr;
  int32_t *nsptr32 = nullptr;
  double *nw = nullptr, *wnode = nullptr, *nsym = nullptr;
  int32_t *fw_cells = nullptr, *fw_sptr = nullptr, *fw_nb = nullptr;
  SweepRec *fw_recs = nullptr;
  int32_t *bw_cells = nullptr, *bw_sptr = nullptr, *bw_nb = nullptr;
  SweepRec *bw_recs = nullptr;
  std::vector<int32_t> fw_lptr, bw_lptr;
  // persistent sweeps: chunked level order, ready flags, error word
  ChunkSweep fwc, bwc;
  int32_t nchunks = 0;
  bool chunk0_exported = false;
  double *dqf = nullptr;  // forward-sweep increments (dq8 holds the backward ones = DQ)
  int *sweep_err = nullptr;
  int persist_grid = 0;
  int sweep_w = 0;               // records per position of the persistent sweeps (4 or 8)
  int sweep_lanes = 0;           // lanes per cell of the persistent sweeps (= W)
  int persist_occ[2][2] = {{0, 0}, {0, 0}};  // resident blocks per SM [kind][W = 4, 8]
  int sweep_kind = MFG_SWEEP_DEEP;  // persistent sweep kernels in use (MFG_SWEEP_*)
  // launch knobs of the other kernels (mfg_autotune): resident blocks per SM
  // the fused face gather and the face flux are compiled for (their register
  // caps), and the block sizes of the two gradient kernels
  int gather_minb = MFG_GATHER_MINB, flux_minb = MFG_FLUX_MINB;
  // lanes per cell of the face gather and the gradient face sums (one lane
  // per face; 0: one thread per cell), and the most the grid's cells allow
  // (0 for cells of more than 8 faces)
  int gather_lanes = 0, gather_lanes_fit = 0;
  int node_block = kNodeBlock, grad_block = kGradBlock;
  int ring = kRing;                 // ring positions the tables were built for
  int chunking = 0;              // chunk assignment of the forward sweep (MFG_CHUNK_*)
  double chunk_est_us[2] = {0.0, 0.0};  // modelled duration of each sweep with its chunks
  // records of each sweep [forward, backward] whose increment comes from the
  // block's ring, from global memory (same chunk, older than the ring), or
  // from another chunk
  int32_t sweep_stats[2][3] = {{0, 0, 0}, {0, 0, 0}};
  int n_sm = 0;
  unsigned long long *dt_ext = nullptr;
  double *norm_part = nullptr, *norm_out = nullptr, *norm_hist = nullptr, *cfl_tab = nullptr;
  int32_t *iter_counter = nullptr;
  int32_t hist_cap = 0, cfl_cap = 0;
  // batched cases (ncase == 1: a single grid, kernels use P)
  int32_t ncase = 1;
  std::vector<mfg_params> hps;          // per-case host parameters
  std::vector<int32_t> case_cell0;      // first cell of each case [ncase+1]
  std::vector<int32_t> case_bface0;     // first boundary face (= ghost - C) [ncase+1]
  Params *ptab = nullptr;               // per-case device parameters
  int32_t *case_of_d = nullptr, *case_first_d = nullptr, *case_cell0_d = nullptr;
  double *seg_part = nullptr;
  double *h_pinned = nullptr;  // small pinned scratch for scalars
  std::vector<void *> allocs;
  int64_t device_bytes = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int64_t graph_nodes = 0;
  int max_level_cells = 0;
  // one part of a partitioned mesh (mfg_halo_set): the caller's exchange
  // buffers and the device copies of the exchange lists
  bool halo = false;
  mfg_halo hb{};
  int32_t *h_send = nullptr;            // local cell of each sent row
  int32_t *h_recv = nullptr;            // ghost record (C + boundary face) of each received row
  int32_t *h_nodes = nullptr;           // local node of each node entry
  int32_t *h_unodes = nullptr, *h_eptr = nullptr, *h_eidx = nullptr;  // entries per shared node
  int32_t h_nu = 0;
  int32_t *h_gflag = nullptr;  // [G] 1 for the ghosts received rows fill (second order)
};

namespace {

template <typename T>
int dalloc(mfg_ctx *ctx, T **p, size_t count) {
  size_t bytes = std::max<size_t>(1, count) * sizeof(T);
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e != cudaSuccess) {
    g_cuda_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return MFG_ERR_NOMEM;
  }
  ctx->allocs.push_back((void *)*p);
  ctx->device_bytes += (int64_t)bytes;
  return MFG_OK;
}

template <typename T>
int dupload(mfg_ctx *ctx, T **p, const std::vector<T> &h) {
  int rc = dalloc(ctx, p, h.size());
  if (rc) return rc;
  if (!h.empty()) MFG_CUDA(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return MFG_OK;
}

Params make_params(const mfg_params &p) {
  Params P;
  P.gam = p.gam;
  P.gamm1 = p.gamm1;
  P.p_bar = p.p_bar;
  P.alf_l = p.alf_l;
  P.lhs_omga = p.lhs_omga;
  const double gam1 = p.gam - 1.;
  P.peff = p.gam * p.p_bar / gam1;  // forward_lusgs.cpp:1295
  P.rho_min = p.rho_min;
  P.rho_max = p.rho_max;
  P.p_min = p.p_min;
  P.p_max = p.p_max;
  P.p_break = p.p_break;
  P.ratio_dtmax = p.ratio_dtmax;
  P.ref[0] = p.rho_s;
  P.ref[1] = p.u_s;
  P.ref[2] = p.v_s;
  P.ref[3] = p.w_s;
  P.ref[4] = p.p_s;
  P.uvw_norm = sqrt(p.u_s * p.u_s + p.v_s * p.v_s + p.w_s * p.w_s);
  {
    const double pm = p.p_s + p.p_bar, rhom = p.rho_s;
    P.entr_m = pm / pow(rhom, p.gam);
  }
  return P;
}

inline void count_launch(int64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

Cases cases_of(const mfg_ctx *ctx) {
  if (ctx->ncase <= 1) return Cases{nullptr, nullptr, nullptr, 1};
  return Cases{ctx->ptab, ctx->case_of_d, ctx->case_first_d, ctx->ncase};
}

int check_kernel() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_cuda_error = std::string("kernel launch: ") + cudaGetErrorString(e);
    return MFG_ERR_CUDA;
  }
  return MFG_OK;
}

// host: CSR of faces per cell, ascending (CalnFPC + CalC2F order).
void build_c2f(const mfg_mesh *m, std::vector<int32_t> &ptr, std::vector<int32_t> &c2f) {
  const int32_t C = m->n_cell;
  ptr.assign(C + 1, 0);
  for (int32_t f = 0; f < m->n_face; f++) {
    ptr[m->f2c[2 * f] + 1]++;
    if (f >= m->n_bface) ptr[m->f2c[2 * f + 1] + 1]++;
  }
  for (int32_t c = 0; c < C; c++) ptr[c + 1] += ptr[c];
  c2f.resize(ptr[C]);
  std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
  for (int32_t f = 0; f < m->n_face; f++) {
    c2f[fill[m->f2c[2 * f]]++] = f;
    if (f >= m->n_bface) c2f[fill[m->f2c[2 * f + 1]]++] = f;
  }
}

int validate_mesh(const mfg_mesh *m) {
  if (!m || m->n_cell <= 0 || m->n_face <= 0 || m->n_node <= 0 || m->n_bface < 0 ||
      m->n_bface > m->n_face)
    return MFG_ERR_INVALID;
  if (!m->f2c || !m->nnpf || !m->f2n || (!m->bctype && m->n_bface) || !m->xfn || !m->yfn ||
      !m->zfn || !m->area || !m->xfc || !m->yfc || !m->zfc || !m->xcc || !m->ycc || !m->zcc ||
      !m->vol || !m->wnode || !m->nmark || !m->wbface || !m->nnpc || !m->c2n || !m->wc2n ||
      !m->nodesymm || !m->xfn_n_symm || !m->yfn_n_symm || !m->zfn_n_symm)
    return MFG_ERR_INVALID;
  const int64_t n = (int64_t)m->n_cell + m->n_bface;
  for (int32_t f = 0; f < m->n_face; f++) {
    const int32_t c1 = m->f2c[2 * f], c2 = m->f2c[2 * f + 1];
    if (c1 < 0 || c1 >= m->n_cell) return MFG_ERR_BADMESH;
    if (f < m->n_bface) {
      if (c2 != m->n_cell + f) return MFG_ERR_BADMESH;
    } else if (c2 < 0 || c2 >= m->n_cell || c2 == c1) {
      return MFG_ERR_BADMESH;
    }
    if (m->nnpf[f] <= 0) return MFG_ERR_BADMESH;
  }
  (void)n;
  return MFG_OK;
}

}  // namespace

// Shared with the other translation units of the library (mesh
// preprocessing): the thread's last CUDA error text and the launch count.
namespace mfg {
void note_cuda_error(const char *what, int code) {
  g_cuda_error = std::string(what) + ": " + cudaGetErrorString((cudaError_t)code);
}
void note_launches(int64_t k) { count_launch(k); }
}  // namespace mfg

// ---------------------------------------------------------------------------
// Context tables built on the device from a device-resident preprocessing
// (mfg_create_from_prep): the arrays create_impl builds on the host, for the
// identity LU-SGS order, from the preprocessing's own lists.
// ---------------------------------------------------------------------------
namespace {

// create_impl's slot loop, one thread per cell
__global__ void k_dev_slots(int32_t C, int32_t B, const int32_t *__restrict__ cptr,
                            const int32_t *__restrict__ cf, const int32_t *__restrict__ fptr,
                            const int32_t *__restrict__ f2n, const int32_t *__restrict__ f2c,
                            const int32_t *__restrict__ bctype, const double *__restrict__ xfn,
                            const double *__restrict__ yfn, const double *__restrict__ zfn,
                            const double *__restrict__ area, const double *__restrict__ xfc,
                            const double *__restrict__ yfc, const double *__restrict__ zfc,
                            const double *__restrict__ xcc, const double *__restrict__ ycc,
                            const double *__restrict__ zcc, SlotRec *__restrict__ slots,
                            int32_t *__restrict__ bad, int32_t *__restrict__ max_slots) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  atomicMax(max_slots, cptr[c + 1] - cptr[c]);
  const double cx = xcc[c], cy = ycc[c], cz = zcc[c];
  for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
    const int32_t f = cf[j];
    SlotRec sr;
    const bool is_c1 = f2c[2 * f] == c;
    sr.nx = xfn[f];
    sr.ny = yfn[f];
    sr.nz = zfn[f];
    sr.area = area[f];
    // compute_timestep.cpp:762, the same expression for either side
    sr.dn = fabs((xfc[f] - cx) * sr.nx + (yfc[f] - cy) * sr.ny + (zfc[f] - cz) * sr.nz);
    sr.nb = is_c1 ? f2c[2 * f + 1] : f2c[2 * f];
    if (sr.nb == c) atomicAdd(bad, 1);  // the cell on both sides of a face
    sr.face = f;
    sr.flags = is_c1 ? 0 : SLOT_IS_C2;
    if (f < B) {
      sr.flags |= SLOT_BOUNDARY;
      const int t = bctype[f];
      if (t == MFG_BC_INTERFACE || t == MFG_BC_SYMM) sr.flags |= SLOT_NODE_AVG;
    }
    const int32_t k0 = fptr[f];
    const bool tri = fptr[f + 1] - k0 == 3;
    if (tri) sr.flags |= SLOT_TRI;
    for (int t = 0; t < 3; t++) sr.tri[t] = tri ? f2n[k0 + t] : 0;
    slots[j] = sr;
  }
}

__global__ void k_dev_faces(int32_t F, const int32_t *__restrict__ f2c,
                            const double *__restrict__ xfn, const double *__restrict__ yfn,
                            const double *__restrict__ zfn, const double *__restrict__ area,
                            FaceRec *__restrict__ faces) {
  const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  faces[f] = FaceRec{xfn[f], yfn[f], zfn[f], area[f], f2c[2 * f], f2c[2 * f + 1], 0, 0};
}

// Records per cell of each sweep (forward: the neighbours before the cell in
// the identity order; backward: those after it, ghosts included) and the
// in-degrees of the level computation (interior dependencies only).
__global__ void k_dev_counts(int32_t C, const int32_t *__restrict__ cptr,
                             const SlotRec *__restrict__ slots, int32_t *__restrict__ fw_cnt,
                             int32_t *__restrict__ bw_cnt, int32_t *__restrict__ fw_deg,
                             int32_t *__restrict__ bw_deg, int32_t *__restrict__ maxns) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  int32_t fw = 0, bw = 0, bwi = 0;
  for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
    const int32_t nb = slots[j].nb;
    if (nb < c) {
      fw++;
    } else {
      bw++;
      if (nb < C) bwi++;
    }
  }
  fw_cnt[c] = fw;
  bw_cnt[c] = bw;
  fw_deg[c] = fw;
  bw_deg[c] = bwi;
  atomicMax(maxns, max(fw, bw));
}

// Level sets as a breadth-first release: a cell joins level l + 1 when the
// last of its dependencies (all on levels <= l) has been processed, which is
// 1 + the longest dependency chain below it, the level create_impl computes.
__global__ void k_dev_level_seed(int32_t C, const int32_t *__restrict__ deg,
                                 int32_t *__restrict__ lvl, int32_t *__restrict__ front,
                                 int32_t *__restrict__ count) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  if (deg[c] == 0) {
    lvl[c] = 0;
    front[atomicAdd(count, 1)] = c;
  }
}

__global__ void k_dev_level_step(int32_t nf, const int32_t *__restrict__ front, int32_t level,
                                 int fwd, int32_t C, const int32_t *__restrict__ cptr,
                                 const SlotRec *__restrict__ slots, int32_t *__restrict__ deg,
                                 int32_t *__restrict__ lvl, int32_t *__restrict__ next,
                                 int32_t *__restrict__ next_count) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int32_t c = front[i];
  for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
    const int32_t nb = slots[j].nb;
    if (nb >= C || (fwd ? nb <= c : nb >= c)) continue;  // not a dependant of c
    if (atomicSub(&deg[nb], 1) == 1) {
      lvl[nb] = level + 1;
      next[atomicAdd(next_count, 1)] = nb;
    }
  }
}

__global__ void k_dev_iota(int32_t C, int32_t *__restrict__ v) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < C) v[i] = i;
}

// g[i] = cnt[cells[i]] (and g[C] = 0), for the record offsets of the
// level-sorted cells
__global__ void k_dev_gather_cnt(int32_t C, const int32_t *__restrict__ cells,
                                 const int32_t *__restrict__ cnt, int32_t *__restrict__ g) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < C) g[i] = cnt[cells[i]];
  if (i == C) g[C] = 0;
}

// build_levels' per-level sweep records, one thread per level-sorted cell
__global__ void k_dev_level_records(int32_t C, const int32_t *__restrict__ cells,
                                    const int32_t *__restrict__ sptr,
                                    const int32_t *__restrict__ cptr,
                                    const SlotRec *__restrict__ slots, int fwd,
                                    SweepRec *__restrict__ recs, int32_t *__restrict__ nbs) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C) return;
  const int32_t c = cells[i];
  if (fwd && c == 0) return;  // the first cell of the order only divides by Diag
  int32_t o = sptr[i];
  for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
    const SlotRec sr = slots[j];
    const int32_t nb = sr.nb;
    if (fwd ? nb > c : nb < c) continue;
    const bool is_c1 = (sr.flags & SLOT_IS_C2) == 0;
    SweepRec r;
    r.nx = is_c1 ? sr.nx : -sr.nx;
    r.ny = is_c1 ? sr.ny : -sr.ny;
    r.nz = is_c1 ? sr.nz : -sr.nz;
    r.w = fwd ? 0.5 * sr.area : sr.area;
    recs[o] = r;
    nbs[o] = nb;
    o++;
  }
}

// chunk of each level-sorted position (sort key) and its index (value)
__global__ void k_dev_chunk_keys(int32_t C, const int32_t *__restrict__ cells,
                                 const int32_t *__restrict__ assign, int32_t *__restrict__ keys,
                                 int32_t *__restrict__ idx, int32_t *__restrict__ chunk_cnt) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C) return;
  const int32_t p = assign[cells[i]];
  keys[i] = p;
  idx[i] = i;
  atomicAdd(&chunk_cnt[p], 1);
}

// chunk-major positions: cell, position of each cell, segment heads
// (chunk start or level change)
__global__ void k_dev_positions(int32_t C, const int32_t *__restrict__ order,
                                const int32_t *__restrict__ cells,
                                const int32_t *__restrict__ pchunk, const int32_t *__restrict__ lvl,
                                int32_t *__restrict__ ccells, int32_t *__restrict__ posof,
                                int32_t *__restrict__ head) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > C) return;
  if (k == C) {
    head[C] = 0;
    return;
  }
  const int32_t c = cells[order[k]];
  ccells[k] = c;
  posof[c] = k;
  head[k] = (k == 0 || pchunk[k] != pchunk[k - 1] || lvl[c] != lvl[cells[order[k - 1]]]) ? 1 : 0;
}

__global__ void k_dev_segs(int32_t C, const int32_t *__restrict__ head,
                           const int32_t *__restrict__ hscan, int32_t *__restrict__ segs) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > C) return;
  if (k == C)
    segs[hscan[C]] = C;
  else if (head[k])
    segs[hscan[k]] = k;
}

__global__ void k_dev_seg_begin(int32_t P, const int32_t *__restrict__ chunk_ptr,
                                const int32_t *__restrict__ hscan,
                                int32_t *__restrict__ seg_begin) {
  const int32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p <= P) seg_begin[p] = hscan[chunk_ptr[p]];
}

// build_levels' position-major tables, one thread per chunk-major position
template <bool MX>
__global__ void k_dev_pack(int32_t C, int32_t W, int with_recs, const int32_t *__restrict__ order,
                           const int32_t *__restrict__ ccells, const int32_t *__restrict__ pchunk,
                           const int32_t *__restrict__ head, const int32_t *__restrict__ hscan,
                           const int32_t *__restrict__ segs, const int32_t *__restrict__ chunk_ptr,
                           const int32_t *__restrict__ posof, const int32_t *__restrict__ assign,
                           const int32_t *__restrict__ sptr, const int32_t *__restrict__ nbs,
                           const SweepRec *__restrict__ recs, PosCell *__restrict__ packed,
                           int32_t *__restrict__ cnbs, SweepRec *__restrict__ crecs,
                           SweepRecF *__restrict__ crecs_f, int32_t *__restrict__ cslot,
                           int32_t *__restrict__ chunk0_exported, int32_t *__restrict__ stats,
                           int32_t ring) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= C) return;
  const int32_t gi = order[k];
  const int32_t c = ccells[k];
  const int32_t s0 = sptr[gi], ns = sptr[gi + 1] - s0;
  packed[k] = PosCell{c, ns};
  if (!with_recs) return;
  const int32_t p = pchunk[k];
  const int32_t seg_end = segs[hscan[k] + head[k]];  // next segment head
  for (int32_t j = 0; j < ns; j++) {
    const int32_t nb = nbs[s0 + j];
    const int64_t o = (int64_t)k * W + j;
    const bool cross = nb < C && assign[nb] != p;
    if (cross && assign[nb] == 0) *chunk0_exported = 1;
    uint32_t e = (uint32_t)nb;
    if (cross) {
      e |= kMark;
      atomicAdd(&stats[2], 1);
    } else if (nb < C && posof[nb] >= seg_end - ring) {
      e |= kInRing;
      cslot[o] = (posof[nb] - chunk_ptr[p]) & (ring - 1);
      atomicAdd(&stats[0], 1);
    } else if (nb < C) {
      atomicAdd(&stats[1], 1);
    }
    cnbs[o] = (int32_t)e;
    const SweepRec r = recs[s0 + j];
    if (MX)
      crecs_f[o] = SweepRecF{(float)r.nx, (float)r.ny, (float)r.nz, (float)r.w};
    else
      crecs[o] = r;
  }
}

// build_node_lists' passes (CompNodeVar3D_dist, cal_gradient.cpp:2041-2125,
// :2261-2279): a boundary entry of pass 0 (walls), 1 (far field) or 2
// (other types), and whether the node's mark lets it through
__device__ __forceinline__ bool node_pass_takes(int pass, int t, int mark) {
  if (pass == 0) return t == MFG_BC_WALL;
  if (pass == 1) return t == MFG_BC_FAR_FIELD && mark != MFG_BC_WALL;
  return !(t == MFG_BC_WALL || t == MFG_BC_SYMM || t == MFG_BC_FAR_FIELD ||
           t == MFG_BC_INTERFACE) &&
         mark != MFG_BC_WALL && mark != MFG_BC_FAR_FIELD;
}

template <bool FILL>
__global__ void k_dev_node_lists(int32_t N, const int32_t *__restrict__ nbptr,
                                 const int32_t *__restrict__ nblist,
                                 const int32_t *__restrict__ bent_face,
                                 const int32_t *__restrict__ bctype,
                                 const int32_t *__restrict__ ncptr,
                                 const int32_t *__restrict__ nclist,
                                 const int32_t *__restrict__ c2n_cell,
                                 const int32_t *__restrict__ nmark,
                                 const double *__restrict__ wbface,
                                 const double *__restrict__ wc2n, int32_t *__restrict__ cnt,
                                 int32_t *__restrict__ bad, const int32_t *__restrict__ nptr,
                                 int32_t *__restrict__ nsrc, double *__restrict__ nw) {
  const int32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int mark = nmark[p];
  const int32_t o0 = FILL ? nptr[p] : 0;
  int32_t o = o0;
  for (int pass = 0; pass < 3; pass++)
    for (int32_t s = nbptr[p]; s < nbptr[p + 1]; s++) {
      const int32_t k = nblist[s];
      const int32_t i = bent_face[k];
      if (!node_pass_takes(pass, bctype[i], mark)) continue;
      if (FILL) {
        nsrc[o] = i;
        nw[o] = wbface[k];
      }
      o++;
    }
  const int32_t nbnd = o - o0;
  if (mark == 0) {
    for (int32_t s = ncptr[p]; s < ncptr[p + 1]; s++) {
      const int32_t m = nclist[s];
      if (FILL) {
        nsrc[o] = c2n_cell[m];
        nw[o] = wc2n[m];
      }
      o++;
    }
  }
  if (!FILL) {
    cnt[p] = o;
    if (nbnd > 0 && o > nbnd) atomicAdd(bad, 1);  // both kinds of entry
  }
}

__global__ void k_dev_node_info(int32_t N, const int32_t *__restrict__ nmark,
                                const int32_t *__restrict__ nodesymm,
                                const double *__restrict__ xs, const double *__restrict__ ys,
                                const double *__restrict__ zs, int32_t *__restrict__ info,
                                double *__restrict__ nsym) {
  const int32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  int32_t v = nmark[p] != 0 ? 1 : 0;
  const bool sym = nodesymm[p] == 1;
  if (sym) v |= 2;
  info[p] = v;
  nsym[3 * (int64_t)p] = sym ? xs[p] : 0.0;
  nsym[3 * (int64_t)p + 1] = sym ? ys[p] : 0.0;
  nsym[3 * (int64_t)p + 2] = sym ? zs[p] : 0.0;
}

__global__ void k_dev_bface_c1(int32_t G, const int32_t *__restrict__ f2c,
                               int32_t *__restrict__ bc1) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < G) bc1[k] = f2c[2 * k];
}

}  // namespace

extern "C" {

const char *mfg_error_string(int32_t code) {
  switch (code) {
    case MFG_OK: return "ok";
    case MFG_ERR_INVALID: return "invalid argument";
    case MFG_ERR_CUDA: return "CUDA error";
    case MFG_ERR_NOMEM: return "out of memory";
    case MFG_ERR_TIMEOUT: return "device wait timed out";
    case MFG_ERR_NONFINITE: return "non-finite value";
    case MFG_ERR_UNSUPPORTED: return "unsupported configuration";
    case MFG_ERR_BADMESH: return "bad mesh";
    case MFG_ERR_NODEVICE: return "no usable CUDA device";
    case MFG_ERR_IO: return "file missing, truncated or malformed";
    default: return "unknown error";
  }
}

const char *mfg_last_cuda_error(void) { return g_cuda_error.c_str(); }

int64_t mfg_kernel_launches(void) { return g_launches.load(); }

static void free_ctx(mfg_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (int k = 0; k < 2; k++)
    if (ctx->graph[k]) cudaGraphExecDestroy(ctx->graph[k]);
  for (void *p : ctx->allocs) cudaFree(p);
  if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
  if (ctx->ev_res) cudaEventDestroy(ctx->ev_res);
  if (ctx->ev_state) cudaEventDestroy(ctx->ev_state);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

int mfg_destroy(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  free_ctx(ctx);
  return MFG_OK;
}

// Chunk assignment and persistent sweep kernels forced for contexts created
// from now on (-1: chosen by the model), set by mfg_set_chunking and
// mfg_set_sweep_kernel.
static std::atomic<int> g_chunking{-1};
static std::atomic<int> g_sweep_kind{-1};

// Records per position (W), persistent-sweep kernel kind, grid and chunk
// count of a new context: one chunk per resident block, no chunk under
// kMinChunk cells.  The kind follows the widest level (max_level_cells,
// both sweeps): where it would give a deep block more than two passes of
// its lane groups per level, the many small blocks of the wide kernels.
static void setup_sweep_grid(mfg_ctx *ctx, int32_t maxns, int force_kind = -1) {
  const int32_t C = ctx->C;
  ctx->sweep_w = maxns <= 4 ? 4 : (maxns <= 8 ? 8 : 0);
  if (ctx->n > (int64_t)kIdMask) ctx->sweep_w = 0;  // neighbour ids share their word with flags
  const int wi = ctx->sweep_w == 8 ? 1 : 0;
  auto grid_of = [&](int kind) {
    return ctx->sweep_w ? ctx->persist_occ[kind][wi] * ctx->n_sm : 0;
  };
  int kind = force_kind >= 0 ? force_kind : g_sweep_kind.load();
  if (kind < 0) {
    const int32_t pdeep = std::max(1, std::min(grid_of(MFG_SWEEP_DEEP), (C + kMinChunk - 1) / kMinChunk));
    kind = (int64_t)ctx->max_level_cells > 2LL * sweep_groups(ctx->sweep_w) * pdeep
               ? MFG_SWEEP_WIDE
               : MFG_SWEEP_DEEP;
  }
  if (grid_of(kind) <= 0) kind = kind == MFG_SWEEP_WIDE ? MFG_SWEEP_DEEP : MFG_SWEEP_WIDE;
  ctx->sweep_kind = kind;
  ctx->ring = sweep_ring(kind);
  ctx->persist_grid = grid_of(kind);
  ctx->nchunks = std::max(1, std::min(ctx->persist_grid, (C + kMinChunk - 1) / kMinChunk));
  ctx->sweep_mode = ctx->persist_grid > 0 ? 1 : 0;
  ctx->sweep_lanes = ctx->sweep_w;
}

// Chunks for the persistent sweeps, one per resident block.  Level by level
// (lptr over the level-sorted cells, sptr/nbs their dependencies), a cell
// joins the chunk that most of its dependencies are in, unless that chunk
// already holds its share of the level; the remaining cells fill the chunks
// in order.  Every level is thereby spread evenly over the chunks while
// dependency chains mostly stay in one chunk.
static void assign_chunks(int32_t C, int32_t P, const std::vector<int32_t> &lptr,
                          const int32_t *cells, const int32_t *sptr, const int32_t *nbs,
                          std::vector<int32_t> &assign) {
  const int32_t L = (int32_t)lptr.size() - 1;
  assign.assign(C, -1);
  std::vector<int32_t> load(P), pending;
  for (int32_t l = 0; l < L; l++) {
    const int32_t a0 = lptr[l], a1 = lptr[l + 1];
    const int32_t quota = (a1 - a0 + P - 1) / P;
    std::fill(load.begin(), load.end(), 0);
    pending.clear();
    for (int32_t i = a0; i < a1; i++) {
      int32_t best = -1, bestn = 0;
      for (int32_t s0 = sptr[i]; s0 < sptr[i + 1]; s0++) {
        if (nbs[s0] >= C) continue;
        const int32_t ch = assign[nbs[s0]];
        int32_t votes = 0;
        for (int32_t t = sptr[i]; t < sptr[i + 1]; t++)
          if (nbs[t] < C && assign[nbs[t]] == ch) votes++;
        if (votes > bestn) {
          best = ch;
          bestn = votes;
        }
      }
      if (best >= 0 && load[best] < quota) {
        assign[cells[i]] = best;
        load[best]++;
      } else {
        pending.push_back(cells[i]);
      }
    }
    int32_t pp = 0;
    for (int32_t c : pending) {
      while (load[pp] >= quota) pp++;
      assign[c] = pp;
      load[pp]++;
    }
  }
}

// Chunks across the level sets, monotone along the dependencies.  Every
// cell gets a label (la, lb) on a Pa x Pb grid: its seed is the equal-count
// bucket of its centroid along two axes, and per axis the label is the
// maximum of the seed and the labels of the cells it depends on (cells in
// level order, so those are labelled first) -- the minimum instead along an
// axis on which a sweep's dependencies lie mostly above the cell (the
// backward sweep's).  Labels are therefore monotone along every dependency:
// a dependency path crosses at most Pa + Pb - 2 chunk boundaries, and where
// the level sets run across the two axes (the levels of a lexicographically
// numbered box follow its slowest axis) every level spreads over all the
// chunks.
// rank: each cell's position in the centroid order along an axis.
static void assign_chunks_transverse(int32_t C, int32_t Pa, int32_t Pb, int ax, int bx,
                                     const std::vector<int32_t> &lptr, const int32_t *cells,
                                     const int32_t *sptr, const int32_t *nbs,
                                     const double *const xyz[3],
                                     const std::vector<int32_t> *rank,
                                     std::vector<int32_t> &assign) {
  const double *ca = xyz[ax], *cb = xyz[bx];
  std::vector<int32_t> la(C), lb(C);
  for (int32_t c = 0; c < C; c++) {
    la[c] = (int32_t)((int64_t)rank[ax][c] * Pa / C);
    lb[c] = (int32_t)((int64_t)rank[bx][c] * Pb / C);
  }
  const int32_t L = (int32_t)lptr.size() - 1;
  // per axis: do the dependencies lie mostly above (then labels take the
  // minimum) or below the cell (the maximum)?
  int64_t up_a = 0, up_b = 0;
  for (int32_t i = 0; i < lptr[L]; i++) {
    const int32_t c = cells[i];
    for (int32_t s0 = sptr[i]; s0 < sptr[i + 1]; s0++) {
      const int32_t d = nbs[s0];
      if (d >= C) continue;
      up_a += (ca[d] > ca[c]) - (ca[d] < ca[c]);
      up_b += (cb[d] > cb[c]) - (cb[d] < cb[c]);
    }
  }
  for (int32_t i = 0; i < lptr[L]; i++) {
    const int32_t c = cells[i];
    for (int32_t s0 = sptr[i]; s0 < sptr[i + 1]; s0++) {
      const int32_t d = nbs[s0];
      if (d >= C) continue;
      la[c] = up_a > 0 ? std::min(la[c], la[d]) : std::max(la[c], la[d]);
      lb[c] = up_b > 0 ? std::min(lb[c], lb[d]) : std::max(lb[c], lb[d]);
    }
  }
  assign.resize(C);
  for (int32_t c = 0; c < C; c++) assign[c] = la[c] + Pa * lb[c];
}

// Modelled duration (SM cycles) of a persistent sweep over the chunks
// `assign`: per level, a chunk starts after its previous level plus a
// barrier; its k-th cell of the level waits k / G lane-group passes; a cell
// waits for each dependency in another chunk until that one is done plus the
// L2 round trip; a cell takes one dependent chain.  Used to choose between
// chunk assignments.
static double model_sweep_cycles(int32_t C, int32_t P, int32_t G,
                                 const std::vector<int32_t> &lptr, const int32_t *cells,
                                 const int32_t *sptr, const int32_t *nbs,
                                 const std::vector<int32_t> &assign) {
  const double kChain = 800.0, kCross = 1500.0, kBarrier = 60.0;
  std::vector<double> done(C, 0.0), tch(P, 0.0), nxt(P, 0.0);
  std::vector<int32_t> cnt(P, 0);
  const int32_t L = (int32_t)lptr.size() - 1;
  double tmax = 0.0;
  for (int32_t l = 0; l < L; l++) {
    for (int32_t i = lptr[l]; i < lptr[l + 1]; i++) {
      const int32_t c = cells[i], ch = assign[c];
      double t = tch[ch] + kBarrier + (double)(cnt[ch]++ / G) * kChain;
      for (int32_t s0 = sptr[i]; s0 < sptr[i + 1]; s0++) {
        const int32_t d = nbs[s0];
        if (d < C && assign[d] != ch) t = std::max(t, done[d] + kCross);
      }
      done[c] = t + kChain;
      nxt[ch] = std::max(nxt[ch], done[c]);
      tmax = std::max(tmax, done[c]);
    }
    for (int32_t i = lptr[l]; i < lptr[l + 1]; i++) {
      const int32_t ch = assign[cells[i]];
      tch[ch] = nxt[ch];
      cnt[ch] = 0;
    }
  }
  return tmax;
}

// Most cells any chunk holds on any level (more than the block's lane
// groups take two passes over that level).
static int32_t max_chunk_level(int32_t P, const std::vector<int32_t> &lptr, const int32_t *cells,
                               const std::vector<int32_t> &assign) {
  std::vector<int32_t> cnt(P, 0);
  int32_t mx = 0;
  const int32_t L = (int32_t)lptr.size() - 1;
  for (int32_t l = 0; l < L; l++) {
    for (int32_t i = lptr[l]; i < lptr[l + 1]; i++) mx = std::max(mx, ++cnt[assign[cells[i]]]);
    for (int32_t i = lptr[l]; i < lptr[l + 1]; i++) cnt[assign[cells[i]]] = 0;
  }
  return mx;
}

// The chunk assignment of a sweep: the balanced vote (assign_chunks) and the
// transverse monotone one over each pair of axes and each Pa x Pb <= P grid
// whose aspect is within a factor two of the pair's extents.  Grids that
// keep every level of every chunk within one pass of the lane groups come
// first (else the fewest cells per chunk and level); among those the
// shortest modelled sweep is kept.  Returns the choice (MFG_CHUNK_VOTE or
// MFG_CHUNK_TRANSVERSE_*) and its modelled duration in microseconds at
// 1.9 GHz; grid (optional) receives the transverse grid Pa, Pb (0, 0 for
// the vote).
static int choose_chunks(int32_t C, int32_t P, int32_t G, const std::vector<int32_t> &lptr,
                         const int32_t *cells, const int32_t *sptr, const int32_t *nbs,
                         const double *const xyz[3], int force, std::vector<int32_t> &assign,
                         double *est_us, int32_t *grid = nullptr) {
  std::vector<int32_t> best, cand;
  double tbest = 1e300;
  int32_t lbest = INT32_MAX;
  int choice = MFG_CHUNK_VOTE;
  int32_t pa_best = 0;
  // MFG_CHUNK_TRANSVERSE_ANY: the transverse grids of every axis pair, no vote
  const bool any_t = force == MFG_CHUNK_TRANSVERSE_ANY;
  if (any_t) force = -1;
  if ((force < 0 && !any_t) || force == MFG_CHUNK_VOTE) {
    assign_chunks(C, P, lptr, cells, sptr, nbs, cand);
    lbest = std::max(max_chunk_level(P, lptr, cells, cand), G);  // <= G: one pass
    tbest = model_sweep_cycles(C, P, G, lptr, cells, sptr, nbs, cand);
    choice = MFG_CHUNK_VOTE;
    best.swap(cand);
  }
  const bool geo = xyz[0] && xyz[1] && xyz[2] &&
                   (force < 0 || force >= MFG_CHUNK_TRANSVERSE_XY);
  if (geo) {
    // each axis's centroid order once; the axis pairs on threads of their own
    std::vector<int32_t> rank[3];
    double ext[3];
    for (int a = 0; a < 3; a++) {
      std::vector<int32_t> idx(C);
      for (int32_t c = 0; c < C; c++) idx[c] = c;
      std::stable_sort(idx.begin(), idx.end(),
                       [&](int32_t x, int32_t y) { return xyz[a][x] < xyz[a][y]; });
      rank[a].resize(C);
      for (int32_t r = 0; r < C; r++) rank[a][idx[r]] = r;
      ext[a] = std::max(C ? xyz[a][idx[C - 1]] - xyz[a][idx[0]] : 0.0, 1e-300);
    }
    struct Best {
      int32_t load = INT32_MAX;
      double t = 1e300;
      int32_t pa = 0;
      std::vector<int32_t> assign;
    } pb[3];
    auto pair_search = [&](int kind) {
      const int ax = kind == MFG_CHUNK_TRANSVERSE_YZ ? 1 : 0;
      const int bx = kind == MFG_CHUNK_TRANSVERSE_XY ? 1 : 2;
      Best &b = pb[kind - MFG_CHUNK_TRANSVERSE_XY];
      // the grids' balance first (one pass over the cells each), the model
      // on the best-balanced three
      std::vector<std::pair<int32_t, int32_t>> grids;  // (load, Pa)
      std::vector<int32_t> a;
      for (int32_t Pa = 1; Pa <= P; Pa++) {
        const int32_t Pb = P / Pa;
        if (Pb < 1 || (Pa > 1 && P / (Pa - 1) == Pb)) continue;  // the largest Pa per Pb
        const double r = (double)Pa / Pb / (ext[ax] / ext[bx]);
        if (r > 2.0 || r < 0.5) continue;
        assign_chunks_transverse(C, Pa, Pb, ax, bx, lptr, cells, sptr, nbs, xyz, rank, a);
        grids.push_back({std::max(max_chunk_level(P, lptr, cells, a), G), Pa});
      }
      std::sort(grids.begin(), grids.end());
      for (size_t i = 0; i < grids.size() && i < 3; i++) {
        const int32_t load = grids[i].first, Pa = grids[i].second, Pb = P / Pa;
        if (load > b.load) break;
        assign_chunks_transverse(C, Pa, Pb, ax, bx, lptr, cells, sptr, nbs, xyz, rank, a);
        const double t = model_sweep_cycles(C, P, G, lptr, cells, sptr, nbs, a);
        if (load < b.load || t < b.t) {
          b.load = load;
          b.t = t;
          b.pa = Pa;
          b.assign.swap(a);
        }
      }
    };
    std::vector<std::thread> th;
    for (int kind = MFG_CHUNK_TRANSVERSE_XY; kind <= MFG_CHUNK_TRANSVERSE_YZ; kind++)
      if (force < 0 || force == kind) th.emplace_back(pair_search, kind);
    for (auto &t : th) t.join();
    for (int kind = MFG_CHUNK_TRANSVERSE_XY; kind <= MFG_CHUNK_TRANSVERSE_YZ; kind++) {
      Best &b = pb[kind - MFG_CHUNK_TRANSVERSE_XY];
      if (b.assign.empty() || b.load > lbest || (b.load == lbest && b.t >= tbest)) continue;
      lbest = b.load;
      tbest = b.t;
      choice = kind;
      pa_best = b.pa;
      best.swap(b.assign);
    }
  }
  if (best.empty()) {  // a forced transverse assignment without centroids
    assign_chunks(C, P, lptr, cells, sptr, nbs, best);
    tbest = model_sweep_cycles(C, P, G, lptr, cells, sptr, nbs, best);
    choice = MFG_CHUNK_VOTE;
    pa_best = 0;
  }
  (void)lbest;
  assign.swap(best);
  if (est_us) *est_us = tbest / 1900.0;
  if (grid) {
    grid[0] = choice == MFG_CHUNK_VOTE ? 0 : pa_best;
    grid[1] = choice == MFG_CHUNK_VOTE ? 0 : P / pa_best;
  }
  return choice;
}

static int build_levels(mfg_ctx *ctx, const mfg_mesh *m, const std::vector<int32_t> &cptr,
                        const std::vector<int32_t> &c2f) {
  const int32_t C = m->n_cell;
  const int64_t n = ctx->n;
  std::vector<int32_t> order(C), pos(C);
  for (int32_t i = 0; i < C; i++) order[i] = m->lusgs_order ? m->lusgs_order[i] : i;
  std::vector<char> seen(C, 0);
  for (int32_t i = 0; i < C; i++) {
    if (order[i] < 0 || order[i] >= C || seen[order[i]]) return MFG_ERR_INVALID;
    seen[order[i]] = 1;
    pos[order[i]] = i;
  }
  auto layer = [&](int64_t c) -> int64_t { return m->lusgs_layer ? m->lusgs_layer[c] : c; };
  ctx->first_cell = order[0];
  // forward: neighbour used iff layer[nb] <= layer[c] (forward_lusgs.cpp:838)
  std::vector<int32_t> lvl(C, 0);
  std::vector<int32_t> fw_cnt(C, 0);
  for (int32_t i = 0; i < C; i++) {
    const int32_t c = order[i];
    if (i == 0) continue;  // the first cell only divides by Diag (:803-804)
    int32_t l = 0;
    for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
      const int32_t f = c2f[j];
      const int32_t nb = (m->f2c[2 * f] == c) ? m->f2c[2 * f + 1] : m->f2c[2 * f];
      if (layer(nb) > layer(c)) continue;
      fw_cnt[c]++;
      if (nb >= C) continue;  // ghost: DQ stays zero, no dependency
      if (pos[nb] > pos[c]) return MFG_ERR_UNSUPPORTED;
      l = std::max(l, lvl[nb] + 1);
    }
    lvl[c] = l;
  }
  std::vector<int32_t> blvl(C, 0), bw_cnt(C, 0);
  for (int32_t i = C - 1; i >= 0; i--) {
    const int32_t c = order[i];
    int32_t l = 0;
    for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
      const int32_t f = c2f[j];
      const int32_t nb = (m->f2c[2 * f] == c) ? m->f2c[2 * f + 1] : m->f2c[2 * f];
      if (layer(nb) < layer(c)) continue;
      bw_cnt[c]++;
      if (nb >= C) continue;
      if (pos[nb] < pos[c]) return MFG_ERR_UNSUPPORTED;
      l = std::max(l, blvl[nb] + 1);
    }
    blvl[c] = l;
  }
  // persistent sweeps: records per position and chunk count
  {
    int32_t maxns = 0;
    for (int32_t c = 0; c < C; c++) maxns = std::max(maxns, std::max(fw_cnt[c], bw_cnt[c]));
    for (const std::vector<int32_t> *lv : {&lvl, &blvl}) {
      std::vector<int32_t> width;
      for (int32_t c = 0; c < C; c++) {
        if ((int32_t)width.size() <= (*lv)[c]) width.resize((*lv)[c] + 1, 0);
        ctx->max_level_cells = std::max(ctx->max_level_cells, ++width[(*lv)[c]]);
      }
    }
    setup_sweep_grid(ctx, maxns);
  }
  const int W = std::max(ctx->sweep_w, 1);
  auto make = [&](const std::vector<int32_t> &lv, const std::vector<int32_t> &cnt, bool fwd,
                  std::vector<int32_t> &lptr, int32_t **d_cells, int32_t **d_sptr,
                  SweepRec **d_recs, int32_t **d_nb) -> int {
    int32_t L = 0;
    for (int32_t c = 0; c < C; c++) L = std::max(L, lv[c] + 1);
    lptr.assign(L + 1, 0);
    for (int32_t c = 0; c < C; c++) lptr[lv[c] + 1]++;
    for (int32_t l = 0; l < L; l++) {
      ctx->max_level_cells = std::max(ctx->max_level_cells, lptr[l + 1]);
      lptr[l + 1] += lptr[l];
    }
    std::vector<int32_t> cells(C), fill(lptr.begin(), lptr.end() - 1);
    for (int32_t c = 0; c < C; c++) cells[fill[lv[c]]++] = c;  // ascending index per level
    std::vector<int32_t> sptr(C + 1, 0);
    for (int32_t i = 0; i < C; i++) sptr[i + 1] = sptr[i] + cnt[cells[i]];
    std::vector<SweepRec> recs(sptr[C]);
    std::vector<int32_t> nbs(sptr[C]);
    for (int32_t i = 0; i < C; i++) {
      const int32_t c = cells[i];
      int32_t s = sptr[i];
      if (fwd && c == order[0]) continue;
      for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
        const int32_t f = c2f[j];
        const bool is_c1 = m->f2c[2 * f] == c;
        const int32_t nb = is_c1 ? m->f2c[2 * f + 1] : m->f2c[2 * f];
        if (fwd ? (layer(nb) > layer(c)) : (layer(nb) < layer(c))) continue;
        SweepRec r;
        r.nx = is_c1 ? m->xfn[f] : -m->xfn[f];
        r.ny = is_c1 ? m->yfn[f] : -m->yfn[f];
        r.nz = is_c1 ? m->zfn[f] : -m->zfn[f];
        r.w = fwd ? 0.5 * m->area[f] : m->area[f];
        recs[s] = r;
        nbs[s] = nb;
        s++;
      }
    }
    const int32_t P = ctx->nchunks;
    std::vector<int32_t> assign, chunk_cnt(P, 0);
    {
      const double *xyz[3] = {m->xcc, m->ycc, m->zcc};
      const int kind = choose_chunks(C, P, sweep_groups(ctx->sweep_w, ctx->sweep_kind), lptr,
                                     cells.data(),
                                     sptr.data(), nbs.data(), xyz, g_chunking.load(), assign,
                                     &ctx->chunk_est_us[fwd ? 0 : 1]);
      if (fwd) ctx->chunking = kind;
    }
    // chunk-major, level-sorted cell lists (the level order is already sorted)
    for (int32_t c = 0; c < C; c++) chunk_cnt[assign[c]]++;
    std::vector<int32_t> chunk_ptr(P + 1, 0);
    for (int32_t p = 0; p < P; p++) chunk_ptr[p + 1] = chunk_ptr[p] + chunk_cnt[p];
    std::vector<int32_t> slot_of(C), cfill(chunk_ptr.begin(), chunk_ptr.end() - 1);
    std::vector<int32_t> ccells(C);
    for (int32_t i = 0; i < C; i++) {
      const int32_t c = cells[i];
      slot_of[i] = cfill[assign[c]]++;
      ccells[slot_of[i]] = c;
    }
    std::vector<int32_t> gpos(C);
    for (int32_t i = 0; i < C; i++) gpos[cells[i]] = i;
    std::vector<int32_t> segs, seg_begin;
    // position-major: the records of position k at [k * W, k * W + ns)
    std::vector<int32_t> cnbs((size_t)C * W, 0);
    std::vector<SweepRec> crecs((size_t)C * W, SweepRec{0.0, 0.0, 0.0, 0.0});
    std::vector<int32_t> cslot((size_t)C * W, 0), posof(C);
    for (int32_t k = 0; k < C; k++) posof[ccells[k]] = k;
    std::vector<PosCell> packed(C);
    bool chunk0_exported = false;
    for (int32_t p = 0; p < P; p++) {
      seg_begin.push_back((int32_t)segs.size());
      int32_t seg_end = chunk_ptr[p];
      for (int32_t k = chunk_ptr[p]; k < chunk_ptr[p + 1]; k++) {
        const int32_t c = ccells[k];
        if (k == chunk_ptr[p] || lv[c] != lv[ccells[k - 1]]) {
          segs.push_back(k);
          seg_end = k;
          while (seg_end < chunk_ptr[p + 1] && lv[ccells[seg_end]] == lv[c]) seg_end++;
        }
        const int32_t gi = gpos[c];
        packed[k] = PosCell{c, sptr[gi + 1] - sptr[gi]};
        if (!ctx->sweep_w) continue;  // no persistent sweeps for this grid
        int64_t o = (int64_t)k * W;
        for (int32_t s0 = sptr[gi]; s0 < sptr[gi + 1]; s0++, o++) {
          const int32_t nb = nbs[s0];
          const bool cross = nb < C && assign[nb] != p;
          if (cross && assign[nb] == 0) chunk0_exported = true;
          uint32_t e = (uint32_t)nb;
          int32_t *stat = ctx->sweep_stats[fwd ? 0 : 1];
          if (cross) {
            e |= kMark;
            stat[2]++;
          } else if (nb < C && posof[nb] >= seg_end - ctx->ring) {
            // still in the ring when this level reads it: overwritten only by
            // position posof[nb] + ring, which lies in a later level
            e |= kInRing;
            cslot[o] = (posof[nb] - chunk_ptr[p]) & (ctx->ring - 1);
            stat[0]++;
          } else if (nb < C) {
            stat[1]++;  // in the chunk, older than the ring: read from global memory
          }
          cnbs[o] = (int32_t)e;
          crecs[o] = recs[s0];
        }
      }
    }
    seg_begin.push_back((int32_t)segs.size());
    segs.push_back(C);
    if (fwd) ctx->chunk0_exported = chunk0_exported;
    int rc;
    if ((rc = dupload(ctx, d_cells, cells))) return rc;
    if ((rc = dupload(ctx, d_sptr, sptr))) return rc;
    if ((rc = dupload(ctx, d_recs, recs))) return rc;
    if ((rc = dupload(ctx, d_nb, nbs))) return rc;
    ChunkSweep &cs = fwd ? ctx->fwc : ctx->bwc;
    cs.nseg = (int32_t)segs.size() - 1;
    if ((rc = dupload(ctx, &cs.seg_begin, seg_begin))) return rc;
    if ((rc = dupload(ctx, &cs.segs, segs))) return rc;
    if ((rc = dupload(ctx, &cs.cells, packed))) return rc;
    if (ctx->precision == MFG_PREC_MIXED) {
      std::vector<SweepRecF> rf(crecs.size());
      for (size_t i = 0; i < crecs.size(); i++)
        rf[i] = SweepRecF{(float)crecs[i].nx, (float)crecs[i].ny, (float)crecs[i].nz,
                          (float)crecs[i].w};
      if ((rc = dupload(ctx, &cs.recs_f, rf))) return rc;
    } else {
      if ((rc = dupload(ctx, &cs.recs, crecs))) return rc;
    }
    if ((rc = dupload(ctx, &cs.nbs, cnbs))) return rc;
    if ((rc = dupload(ctx, &cs.nslots, cslot))) return rc;
    return MFG_OK;
  };
  (void)n;
  int rc = make(lvl, fw_cnt, true, ctx->fw_lptr, &ctx->fw_cells, &ctx->fw_sptr, &ctx->fw_recs,
                &ctx->fw_nb);
  if (rc) return rc;
  return make(blvl, bw_cnt, false, ctx->bw_lptr, &ctx->bw_cells, &ctx->bw_sptr, &ctx->bw_recs,
              &ctx->bw_nb);
}

// Node contribution lists that replay CompNodeVar3D_dist's loops
// (cal_gradient.cpp:2041-2125 boundary passes, :2261-2279 cell pass).
static int build_node_lists(mfg_ctx *ctx, const mfg_mesh *m) {
  const int32_t N = m->n_node, G = m->n_bface, C = m->n_cell;
  std::vector<int64_t> fptr(m->n_face + 1, 0);
  for (int32_t f = 0; f < m->n_face; f++) fptr[f + 1] = fptr[f] + m->nnpf[f];
  std::vector<int32_t> cnt(N, 0);
  auto bpass = [&](int pass, auto &&emit) {
    for (int32_t i = 0; i < G; i++) {
      const int type = m->bctype[i];
      if (pass == 0 && type != MFG_BC_WALL) continue;
      if (pass == 1 && type != MFG_BC_FAR_FIELD) continue;
      if (pass == 2 && (type == MFG_BC_WALL || type == MFG_BC_SYMM ||
                        type == MFG_BC_FAR_FIELD || type == MFG_BC_INTERFACE))
        continue;
      for (int32_t j = 0; j < m->nnpf[i]; j++) {
        const int32_t p1 = m->f2n[fptr[i] + j];
        if (pass == 1 && m->nmark[p1] == MFG_BC_WALL) continue;
        if (pass == 2 && (m->nmark[p1] == MFG_BC_WALL || m->nmark[p1] == MFG_BC_FAR_FIELD))
          continue;
        emit(p1, i, m->wbface[fptr[i] + j]);
      }
    }
  };
  auto cpass = [&](auto &&emit) {
    int64_t k = 0;
    for (int32_t i = 0; i < C; i++)
      for (int32_t j = 0; j < m->nnpc[i]; j++, k++) {
        const int32_t p1 = m->c2n[k];
        if (m->nmark[p1] != 0) continue;
        emit(p1, i, m->wc2n[k]);
      }
  };
  // A boundary pass only touches marked nodes and the cell pass only
  // unmarked ones (the weights loops mark every node the face passes reach),
  // so each node has entries of one kind.
  std::vector<char> kind(N, 0);
  for (int pass = 0; pass < 3; pass++)
    bpass(pass, [&](int32_t p1, int32_t, double) { cnt[p1]++; kind[p1] |= 1; });
  cpass([&](int32_t p1, int32_t, double) { cnt[p1]++; kind[p1] |= 2; });
  std::vector<int32_t> ptr(N + 1, 0);
  for (int32_t i = 0; i < N; i++) {
    if (kind[i] == 3) return MFG_ERR_UNSUPPORTED;
    ptr[i + 1] = ptr[i] + cnt[i];
  }
  std::vector<int32_t> src(ptr[N]), fill(ptr.begin(), ptr.end() - 1);
  std::vector<double> w(ptr[N]);
  for (int pass = 0; pass < 3; pass++)
    bpass(pass, [&](int32_t p1, int32_t face, double wr) {
      src[fill[p1]] = face;
      w[fill[p1]++] = wr;
    });
  cpass([&](int32_t p1, int32_t cell, double wr) {
    src[fill[p1]] = cell;
    w[fill[p1]++] = wr;
  });
  std::vector<int32_t> info(N, 0);
  std::vector<double> nsym(3 * (size_t)N, 0.0), wnode(m->wnode, m->wnode + N);
  for (int32_t i = 0; i < N; i++) {
    if (m->nmark[i] != 0) info[i] |= 1;
    if (m->nodesymm[i] == 1) {
      info[i] |= 2;
      nsym[3 * i] = m->xfn_n_symm[i];
      nsym[3 * i + 1] = m->yfn_n_symm[i];
      nsym[3 * i + 2] = m->zfn_n_symm[i];
    }
  }
  std::vector<int32_t> bc1(std::max(G, 1), 0);
  for (int32_t k = 0; k < G; k++) bc1[k] = m->f2c[2 * k];
  int rc;
  if ((rc = dupload(ctx, &ctx->nptr, ptr))) return rc;
  if ((rc = dupload(ctx, &ctx->nsrc, src))) return rc;
  if ((rc = dupload(ctx, &ctx->nw, w))) return rc;
  if ((rc = dupload(ctx, &ctx->ninfo, info))) return rc;
  if ((rc = dupload(ctx, &ctx->nsym, nsym))) return rc;
  if ((rc = dupload(ctx, &ctx->wnode, wnode))) return rc;
  if ((rc = dupload(ctx, &ctx->bface_c1, bc1))) return rc;
  std::vector<int32_t> fnp(m->n_face + 1), fns(fptr[m->n_face]);
  for (int32_t f = 0; f <= m->n_face; f++) fnp[f] = (int32_t)fptr[f];
  std::memcpy(fns.data(), m->f2n, sizeof(int32_t) * fns.size());
  if ((rc = dupload(ctx, &ctx->fnptr, fnp))) return rc;
  if ((rc = dupload(ctx, &ctx->fnodes, fns))) return rc;
  return MFG_OK;
}

// Case layout of a context: offsets of each case's cells and boundary faces
// in the concatenated grid, the case of every cell and ghost, and the first
// cell of each case's LU-SGS order.
struct CaseLayout {
  int32_t ncase = 1;
  std::vector<int32_t> cell0, bface0, of, first;
};

// Device, stream, sizes, parameters, case tables and sweep occupancy of a
// new context (whatever builds its grid tables next).
static int ctx_begin(int32_t n_node, int32_t n_face, int32_t n_cell, int32_t n_bface,
                     const mfg_params *params, const CaseLayout &cl, int32_t device,
                     int32_t precision, mfg_ctx **out) {
  *out = nullptr;
  if (precision != MFG_PREC_FP64 && precision != MFG_PREC_MIXED) return MFG_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) {
    g_cuda_error = "no CUDA device";
    return MFG_ERR_NODEVICE;
  }
  mfg_ctx *ctx = new mfg_ctx();
  int rc;
  ctx->device = device;
  ctx->precision = precision;
  auto fail = [&](int code) {
    free_ctx(ctx);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail(MFG_ERR_NODEVICE);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10)
    return fail(MFG_ERR_NODEVICE);
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(MFG_ERR_CUDA);
  ctx->stream = ctx->own_stream;
  ctx->C = n_cell;
  ctx->G = n_bface;
  ctx->F = n_face;
  ctx->N = n_node;
  ctx->n = (int64_t)n_cell + n_bface;
  ctx->hp = *params;
  ctx->P = make_params(*params);
  ctx->ncase = cl.ncase;
  ctx->hps.assign(params, params + cl.ncase);
  const int32_t C = ctx->C;
  if (cl.ncase > 1) {
    ctx->case_cell0 = cl.cell0;
    ctx->case_bface0 = cl.bface0;
    std::vector<Params> pt(cl.ncase);
    for (int32_t k = 0; k < cl.ncase; k++) pt[k] = make_params(params[k]);
    if ((rc = dupload(ctx, &ctx->ptab, pt))) return fail(rc);
    if ((rc = dupload(ctx, &ctx->case_of_d, cl.of))) return fail(rc);
    if ((rc = dupload(ctx, &ctx->case_first_d, cl.first))) return fail(rc);
    if ((rc = dupload(ctx, &ctx->case_cell0_d, cl.cell0))) return fail(rc);
    if ((rc = dalloc(ctx, &ctx->seg_part, (size_t)5 * kSegBlocks * cl.ncase))) return fail(rc);
  } else {
    ctx->case_cell0 = {0, C};
    ctx->case_bface0 = {0, ctx->G};
  }

  {
    // persistent sweeps need every block resident: one chunk per block, at
    // most as many blocks as the occupancy of the heavier kernel allows
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    // resident blocks per SM of each kernel pair (both sweeps), with the
    // stage's dynamic shared memory allowed first
    const bool mx = precision == MFG_PREC_MIXED;
    for (int kind = 0; kind < 2; kind++)
      for (int wi = 0; wi < 2; wi++) {
        const int w = wi ? 8 : 4;
        int per_sm = 1 << 30;
        for (bool fwd : {true, false}) {
          const void *fn = sweep_kernel(fwd, w, mx, kind);
          const size_t smem = sweep_smem(w, mx, kind);
          if (smem &&
              cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                  cudaSuccess)
            return fail(MFG_ERR_CUDA);
          int b = 0;
          if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, sweep_threads(w, kind),
                                                            smem) != cudaSuccess)
            return fail(MFG_ERR_CUDA);
          per_sm = std::min(per_sm, b);
        }
        ctx->persist_occ[kind][wi] = coop ? per_sm : 0;
      }
    ctx->n_sm = prop.multiProcessorCount;
  }
  *out = ctx;
  return MFG_OK;
}

namespace {
int build_sliced_slots(mfg_ctx *ctx);  // defined with the device-build helpers
}  // namespace

// Partials of the residual norm a face gather leaves: one per 256 cells in
// either gather form (the lane-per-face form has them formed by
// k_norm_partial from res, in the one-thread gather's order).
static int gather_blocks(const mfg_ctx *ctx) { return grid_for(ctx->C); }

// Buffers of the iteration, their initial contents and the initial state:
// the end of every context creation.
static int ctx_finish(mfg_ctx *ctx, const double *q0, const CaseLayout &cl) {
  const int32_t C = ctx->C;
  const int64_t n = ctx->n;
  const int32_t precision = ctx->precision;
  int rc;
  if ((rc = build_sliced_slots(ctx))) return rc;
  if (precision == MFG_PREC_MIXED) {
    for (int k = 0; k < 2; k++)
      if ((rc = dalloc(ctx, &ctx->q4[k], (size_t)n * Q_STRIDE))) return rc;
    if ((rc = dalloc(ctx, &ctx->qn4, (size_t)ctx->N * Q_STRIDE))) return rc;
  }
  for (int k = 0; k < 2; k++)
    if ((rc = dalloc(ctx, &ctx->q8[k], (size_t)n * Q_STRIDE))) return rc;
  if ((rc = dalloc(ctx, &ctx->dq8, (size_t)n * Q_STRIDE))) return rc;
  if ((rc = dalloc(ctx, &ctx->res, (size_t)5 * C))) return rc;
  if ((rc = dalloc(ctx, &ctx->dt, (size_t)C))) return rc;
  if ((rc = dalloc(ctx, &ctx->diag, (size_t)C))) return rc;
  if ((rc = dalloc(ctx, &ctx->dqdx, (size_t)5 * n))) return rc;
  if ((rc = dalloc(ctx, &ctx->dqdy, (size_t)5 * n))) return rc;
  if ((rc = dalloc(ctx, &ctx->dqdz, (size_t)5 * n))) return rc;
  if ((rc = dalloc(ctx, &ctx->qn8, (size_t)ctx->N * Q_STRIDE))) return rc;
  if ((rc = dalloc(ctx, &ctx->staging, (size_t)5 * n))) return rc;
  if ((rc = dalloc(ctx, &ctx->dt_ext, (size_t)2 * cl.ncase))) return rc;
  const int nparts = std::max(gather_blocks(ctx), kNormBlocks);
  if ((rc = dalloc(ctx, &ctx->norm_part, (size_t)5 * nparts))) return rc;
  if ((rc = dalloc(ctx, &ctx->norm_out, (size_t)5 * cl.ncase))) return rc;
  if ((rc = dalloc(ctx, &ctx->iter_counter, 1))) return rc;
  if ((rc = dalloc(ctx, &ctx->dqf, (size_t)n * Q_STRIDE))) return rc;
  if ((rc = dalloc(ctx, &ctx->sweep_err, 1))) return rc;
  if (cudaMallocHost((void **)&ctx->h_pinned, (64 + 5 * (size_t)cl.ncase) * sizeof(double)) !=
      cudaSuccess)
    return MFG_ERR_NOMEM;

  cudaStream_t st = ctx->stream;
  if (cudaMemsetAsync(ctx->dq8, 0, sizeof(double) * n * Q_STRIDE, st) ||
      cudaMemsetAsync(ctx->res, 0, sizeof(double) * 5 * C, st) ||
      cudaMemsetAsync(ctx->dt, 0, sizeof(double) * C, st) ||
      cudaMemsetAsync(ctx->diag, 0, sizeof(double) * C, st) ||
      cudaMemsetAsync(ctx->dqdx, 0, sizeof(double) * 5 * n, st) ||
      cudaMemsetAsync(ctx->dqdy, 0, sizeof(double) * 5 * n, st) ||
      cudaMemsetAsync(ctx->dqdz, 0, sizeof(double) * 5 * n, st) ||
      cudaMemsetAsync(ctx->qn8, 0, sizeof(double) * ctx->N * Q_STRIDE, st) ||
      cudaMemsetAsync(ctx->dqf, 0, sizeof(double) * n * Q_STRIDE, st) ||
      cudaMemsetAsync(ctx->sweep_err, 0, sizeof(int), st) ||
      cudaMemsetAsync(ctx->iter_counter, 0, sizeof(int32_t), st))
    return MFG_ERR_CUDA;
  k_arm_sentinel<<<grid_for(C), kBlock, 0, st>>>(C, ctx->dqf);  // ready for a forward sweep
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return MFG_ERR_CUDA;
  if ((rc = mfg_set_dt_extrema(ctx, 0.0, kBig))) return rc;  // para_field_global.cpp:220-221
  if ((rc = mfg_upload(ctx, MFG_FIELD_Q, q0))) return rc;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MFG_ERR_CUDA;
  return MFG_OK;
}

static int create_impl(const mfg_mesh *m, const mfg_params *params, const CaseLayout &cl,
                       const double *q0, int32_t device, int32_t precision, mfg_ctx **out) {
  if (!out || !params || !q0) return MFG_ERR_INVALID;
  *out = nullptr;
  int rc = validate_mesh(m);
  if (rc) return rc;
  mfg_ctx *ctx = nullptr;
  if ((rc = ctx_begin(m->n_node, m->n_face, m->n_cell, m->n_bface, params, cl, device, precision,
                      &ctx)))
    return rc;
  auto fail = [&](int code) {
    free_ctx(ctx);
    return code;
  };
  const int32_t C = ctx->C;
  const int64_t n = ctx->n;
  std::vector<int32_t> cptr, c2f;
  build_c2f(m, cptr, c2f);
  ctx->S = cptr[C];
  std::vector<int64_t> fnp((size_t)m->n_face + 1, 0);
  for (int32_t f = 0; f < m->n_face; f++) fnp[f + 1] = fnp[f] + m->nnpf[f];
  std::vector<SlotRec> slots(ctx->S);
  for (int32_t c = 0; c < C; c++) {
    for (int32_t j = cptr[c]; j < cptr[c + 1]; j++) {
      const int32_t f = c2f[j];
      SlotRec s;
      const bool is_c1 = m->f2c[2 * f] == c;
      s.nx = m->xfn[f];
      s.ny = m->yfn[f];
      s.nz = m->zfn[f];
      s.area = m->area[f];
      // compute_timestep.cpp:762, the same expression for either side
      s.dn = std::fabs((m->xfc[f] - m->xcc[c]) * m->xfn[f] + (m->yfc[f] - m->ycc[c]) * m->yfn[f] +
                       (m->zfc[f] - m->zcc[c]) * m->zfn[f]);
      s.nb = is_c1 ? m->f2c[2 * f + 1] : m->f2c[2 * f];
      s.face = f;
      s.flags = 0;
      if (!is_c1) s.flags |= SLOT_IS_C2;
      if (f < m->n_bface) {
        s.flags |= SLOT_BOUNDARY;
        const int t = m->bctype[f];
        if (t == MFG_BC_INTERFACE || t == MFG_BC_SYMM) s.flags |= SLOT_NODE_AVG;
      }
      const bool tri = m->nnpf[f] == 3;
      if (tri) s.flags |= SLOT_TRI;
      for (int t = 0; t < 3; t++) s.tri[t] = tri ? m->f2n[fnp[f] + t] : 0;
      slots[j] = s;
    }
  }
  if ((rc = dupload(ctx, &ctx->cptr, cptr))) return fail(rc);
  if ((rc = dupload(ctx, &ctx->slots, slots))) return fail(rc);
  {
    int32_t max_slots = 0;
    for (int32_t c = 0; c < C; c++) max_slots = std::max(max_slots, cptr[c + 1] - cptr[c]);
    ctx->gather_lanes_fit = gather_lanes_for(max_slots);
  }
  {
    std::vector<FaceRec> fr(m->n_face);
    for (int32_t f = 0; f < m->n_face; f++)
      fr[f] = FaceRec{m->xfn[f], m->yfn[f], m->zfn[f], m->area[f], m->f2c[2 * f],
                      m->f2c[2 * f + 1], 0, 0};
    if ((rc = dupload(ctx, &ctx->faces, fr))) return fail(rc);
    if ((rc = dalloc(ctx, &ctx->fflux, (size_t)kFluxRow * m->n_face))) return fail(rc);
    std::vector<int32_t> bt(m->bctype, m->bctype + m->n_bface);
    if ((rc = dupload(ctx, &ctx->bctype_d, bt))) return fail(rc);
  }
  slots.clear();
  slots.shrink_to_fit();
  std::vector<double> volv(m->vol, m->vol + n);
  if ((rc = dupload(ctx, &ctx->vol, volv))) return fail(rc);
  {
    std::vector<Cen> fc(m->n_face), cc(n);
    for (int32_t f = 0; f < m->n_face; f++) fc[f] = Cen{m->xfc[f], m->yfc[f], m->zfc[f], 0.0};
    for (int64_t i = 0; i < n; i++)
      cc[i] = Cen{m->xcc[i], m->ycc[i], m->zcc[i], std::cbrt(std::fabs(m->vol[i]))};
    if ((rc = dupload(ctx, &ctx->fcen, fc)) || (rc = dupload(ctx, &ctx->ccen, cc)))
      return fail(rc);
  }
  if ((rc = build_levels(ctx, m, cptr, c2f))) return fail(rc);
  if ((rc = build_node_lists(ctx, m))) return fail(rc);
  if ((rc = ctx_finish(ctx, q0, cl))) return fail(rc);
  *out = ctx;
  return MFG_OK;
}

int mfg_create(const mfg_mesh *m, const mfg_params *params, const double *q0, int32_t device,
               int32_t precision, mfg_ctx **out) {
  CaseLayout cl;
  return create_impl(m, params, cl, q0, device, precision, out);
}

// Concatenation of independent grids into one: cells of case 0, 1, ...; then
// the boundary faces of all cases (so that faces [0, G) stay the boundary
// faces and the ghost of union boundary face K is C + K), then the interior
// faces of all cases; nodes likewise.  No face joins two cases, so every
// gather, level set and sweep of the union computes each case exactly as it
// would alone.
int mfg_create_batch(int32_t ncase, const mfg_mesh *ms, const mfg_params *params,
                     const double *const *q0s, int32_t device, int32_t precision,
                     mfg_ctx **out) {
  if (!out || ncase <= 0 || !ms || !params || !q0s) return MFG_ERR_INVALID;
  if (ncase == 1) return mfg_create(&ms[0], &params[0], q0s[0], device, precision, out);
  CaseLayout cl;
  cl.ncase = ncase;
  cl.cell0.assign(ncase + 1, 0);
  cl.bface0.assign(ncase + 1, 0);
  std::vector<int64_t> node0(ncase + 1, 0), iface0(ncase + 1, 0), fnode0(ncase + 1, 0),
      bnode0(ncase + 1, 0), c2n0(ncase + 1, 0);
  for (int32_t k = 0; k < ncase; k++) {
    const mfg_mesh &m = ms[k];
    int rc = validate_mesh(&m);
    if (rc) return rc;
    if (m.lusgs_order || m.lusgs_layer) return MFG_ERR_UNSUPPORTED;
    cl.cell0[k + 1] = cl.cell0[k] + m.n_cell;
    cl.bface0[k + 1] = cl.bface0[k] + m.n_bface;
    node0[k + 1] = node0[k] + m.n_node;
    iface0[k + 1] = iface0[k] + (m.n_face - m.n_bface);
    int64_t sb = 0, sf = 0, sc = 0;
    for (int32_t f = 0; f < m.n_face; f++) (f < m.n_bface ? sb : sf) += m.nnpf[f];
    for (int32_t c = 0; c < m.n_cell; c++) sc += m.nnpc[c];
    bnode0[k + 1] = bnode0[k] + sb;
    fnode0[k + 1] = fnode0[k] + sf;
    c2n0[k + 1] = c2n0[k] + sc;
  }
  const int64_t C = cl.cell0[ncase], G = cl.bface0[ncase], N = node0[ncase];
  const int64_t F = G + iface0[ncase], n = C + G;
  if (n > INT32_MAX || F > INT32_MAX || bnode0[ncase] + fnode0[ncase] > INT32_MAX ||
      c2n0[ncase] > INT32_MAX)
    return MFG_ERR_INVALID;
  std::vector<int32_t> f2c(2 * F), nnpf(F), f2n(bnode0[ncase] + fnode0[ncase]), bct(G);
  std::vector<double> fa[7], ca[4], na[5];
  for (auto &v : fa) v.resize(F);
  for (auto &v : ca) v.resize(n);
  for (auto &v : na) v.resize(N);
  std::vector<int32_t> nmark(N), nsym(N), nnpc(C), c2n(c2n0[ncase]);
  std::vector<double> wbface(bnode0[ncase]), wc2n(c2n0[ncase]);
  std::vector<double> q0((size_t)5 * n);
  cl.of.resize(n);
  cl.first.resize(ncase);
  for (int32_t k = 0; k < ncase; k++) {
    const mfg_mesh &m = ms[k];
    const int64_t cb = cl.cell0[k], gb = cl.bface0[k], nb = node0[k];
    const int64_t mc = m.n_cell, mg = m.n_bface, mn = (int64_t)m.n_cell + m.n_bface;
    auto cell_map = [&](int64_t c) -> int64_t { return c < mc ? cb + c : C + gb + (c - mc); };
    auto face_map = [&](int64_t f) -> int64_t {
      return f < mg ? gb + f : G + iface0[k] + (f - mg);
    };
    const double *fsrc[7] = {m.xfn, m.yfn, m.zfn, m.area, m.xfc, m.yfc, m.zfc};
    int64_t pb = bnode0[k], pi = bnode0[ncase] + fnode0[k], off = 0;
    for (int32_t f = 0; f < m.n_face; f++) {
      const int64_t g = face_map(f);
      f2c[2 * g] = (int32_t)cell_map(m.f2c[2 * f]);
      f2c[2 * g + 1] = (int32_t)cell_map(m.f2c[2 * f + 1]);
      nnpf[g] = m.nnpf[f];
      for (int j = 0; j < 7; j++) fa[j][g] = fsrc[j][f];
      for (int32_t j = 0; j < m.nnpf[f]; j++) {
        const int64_t dst = (f < m.n_bface ? pb : pi) + j;
        f2n[dst] = (int32_t)(nb + m.f2n[off + j]);
        if (f < m.n_bface) wbface[dst] = m.wbface[off + j];
      }
      (f < m.n_bface ? pb : pi) += m.nnpf[f];
      off += m.nnpf[f];
      if (f < m.n_bface) bct[gb + f] = m.bctype[f];
    }
    const double *csrc[4] = {m.xcc, m.ycc, m.zcc, m.vol};
    for (int64_t c = 0; c < mn; c++) {
      const int64_t g = cell_map(c);
      for (int j = 0; j < 4; j++) ca[j][g] = csrc[j][c];
      cl.of[g] = k;
      for (int v = 0; v < 5; v++) q0[(size_t)v * n + g] = q0s[k][(size_t)v * mn + c];
    }
    const double *nsrc[5] = {m.wnode, m.xfn_n_symm, m.yfn_n_symm, m.zfn_n_symm, nullptr};
    for (int64_t p = 0; p < m.n_node; p++) {
      for (int j = 0; j < 4; j++) na[j][nb + p] = nsrc[j][p];
      nmark[nb + p] = m.nmark[p];
      nsym[nb + p] = m.nodesymm[p];
    }
    for (int64_t c = 0, o = 0; c < mc; c++) {
      nnpc[cb + c] = m.nnpc[c];
      for (int32_t j = 0; j < m.nnpc[c]; j++, o++) {
        c2n[c2n0[k] + o] = (int32_t)(nb + m.c2n[o]);
        wc2n[c2n0[k] + o] = m.wc2n[o];
      }
    }
    cl.first[k] = (int32_t)cb;  // identity LU-SGS order
  }
  // boundary-face node lists must precede interior ones in f2n order: the
  // union keeps face order, and faces [0, G) are the boundary faces of all
  // cases in case order, whose node lists were written at [0, sum bnode)
  mfg_mesh u = {};
  u.n_node = (int32_t)N;
  u.n_face = (int32_t)F;
  u.n_cell = (int32_t)C;
  u.n_bface = (int32_t)G;
  u.f2c = f2c.data();
  u.nnpf = nnpf.data();
  u.f2n = f2n.data();
  u.bctype = bct.data();
  u.xfn = fa[0].data();
  u.yfn = fa[1].data();
  u.zfn = fa[2].data();
  u.area = fa[3].data();
  u.xfc = fa[4].data();
  u.yfc = fa[5].data();
  u.zfc = fa[6].data();
  u.xcc = ca[0].data();
  u.ycc = ca[1].data();
  u.zcc = ca[2].data();
  u.vol = ca[3].data();
  u.wnode = na[0].data();
  u.nmark = nmark.data();
  u.wbface = wbface.data();
  u.nnpc = nnpc.data();
  u.c2n = c2n.data();
  u.wc2n = wc2n.data();
  u.nodesymm = nsym.data();
  u.xfn_n_symm = na[1].data();
  u.yfn_n_symm = na[2].data();
  u.zfn_n_symm = na[3].data();
  return create_impl(&u, params, cl, q0.data(), device, precision, out);
}

}  // extern "C"

namespace {

// Scratch device memory of a context build, freed on every exit.
struct DevScratch {
  std::vector<void *> ptrs;
  ~DevScratch() {
    for (void *q : ptrs) cudaFree(q);
  }
  template <typename T>
  int get(T **p, int64_t count) {
    const size_t bytes = std::max<size_t>(1, (size_t)std::max<int64_t>(count, 0)) * sizeof(T);
    const cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
      g_cuda_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return MFG_ERR_NOMEM;
    }
    ptrs.push_back((void *)*p);
    return MFG_OK;
  }
};

int dev_read_i32(const int32_t *d, int32_t *h, cudaStream_t st) {
  MFG_CUDA(cudaMemcpyAsync(h, d, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  MFG_CUDA(cudaStreamSynchronize(st));
  return MFG_OK;
}

int dev_scan(DevScratch &sc, const int32_t *in, int32_t *out, int32_t m, cudaStream_t st) {
  size_t bytes = 0;
  MFG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, m, st));
  char *tmp = nullptr;
  const int rc = sc.get(&tmp, (int64_t)bytes);
  if (rc) return rc;
  MFG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, m, st));
  return MFG_OK;
}

// stable: equal keys keep the order of their values' input positions
int dev_sort_pairs(DevScratch &sc, const int32_t *kin, int32_t *kout, const int32_t *vin,
                   int32_t *vout, int32_t m, int32_t max_key, cudaStream_t st) {
  int bits = 1;
  while (bits < 31 && (1 << bits) <= max_key) bits++;
  size_t bytes = 0;
  MFG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, m, 0, bits, st));
  char *tmp = nullptr;
  const int rc = sc.get(&tmp, (int64_t)bytes);
  if (rc) return rc;
  MFG_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, m, 0, bits, st));
  return MFG_OK;
}

// One thread per slice: kSlice times the most slots of its cells.
__global__ void k_slice_width(int32_t C, const int32_t *__restrict__ cptr,
                              int32_t *__restrict__ width) {
  const int32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t nsl = (C + kSlice - 1) / kSlice;
  if (b > nsl) return;
  int32_t w = 0;
  if (b < nsl)
    for (int32_t c = b * kSlice; c < min(C, (b + 1) * kSlice); c++)
      w = max(w, cptr[c + 1] - cptr[c]);
  width[b] = w * kSlice;
}

__global__ void k_slice_fill(int32_t C, const int32_t *__restrict__ cptr,
                             const SlotRec *__restrict__ slots, const int32_t *__restrict__ sptr32,
                             GatherSlot *__restrict__ gslots, GradSlot *__restrict__ rslots) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const int64_t o = sptr32[c / kSlice] + c % kSlice;
  const int32_t s0 = cptr[c], ns = cptr[c + 1] - s0;
  for (int32_t j = 0; j < ns; j++) {
    const SlotRec sr = slots[s0 + j];
    const int64_t k = o + (int64_t)j * kSlice;
    gslots[k] = GatherSlot{sr.nx, sr.ny, sr.nz, sr.area, sr.dn, sr.nb,
                           (uint32_t)sr.face | ((sr.flags & SLOT_IS_C2) ? 0x80000000u : 0u)};
    GradSlot g{sr.nx, sr.ny, sr.nz, sr.area, sr.tri[0], sr.tri[1], sr.tri[2], sr.flags};
    if ((sr.flags & SLOT_BOUNDARY) && !(sr.flags & SLOT_NODE_AVG))
      g.n0 = sr.nb;  // averaged with the ghost
    else if (!(sr.flags & SLOT_TRI))
      g.n0 = sr.face;  // nodes through the face -> node lists
    rslots[k] = g;
  }
}

__global__ void k_node_slice_fill(int32_t N, const int32_t *__restrict__ nptr,
                                  const int32_t *__restrict__ nsrc, const double *__restrict__ nw,
                                  const int32_t *__restrict__ nsptr32, NodeEnt *__restrict__ nsl) {
  const int32_t nd = blockIdx.x * blockDim.x + threadIdx.x;
  if (nd >= N) return;
  NodeEnt *o = nsl + nsptr32[nd / kSlice] + nd % kSlice;
  const int32_t e0 = nptr[nd], ne = nptr[nd + 1] - e0;
  for (int32_t j = 0; j < ne; j++) o[(int64_t)j * kSlice] = NodeEnt{nsrc[e0 + j], 0, nw[e0 + j]};
}

// The sliced copies of the slot records and of the node lists (see
// mfg_ctx::gslots, rslots, nsl), from the plain ones on the device.
int build_sliced_slots(mfg_ctx *ctx) {
  const int32_t C = ctx->C, nsl = (C + kSlice - 1) / kSlice;
  cudaStream_t st = ctx->stream;
  DevScratch sc;
  int32_t *width = nullptr;
  int rc;
  if ((rc = sc.get(&width, (int64_t)nsl + 1))) return rc;
  if ((rc = dalloc(ctx, &ctx->sptr32, (size_t)nsl + 1))) return rc;
  k_slice_width<<<grid_for((int64_t)nsl + 1), kBlock, 0, st>>>(C, ctx->cptr, width);
  if ((rc = dev_scan(sc, width, ctx->sptr32, nsl + 1, st))) return rc;
  int32_t total = 0;
  if ((rc = dev_read_i32(ctx->sptr32 + nsl, &total, st))) return rc;
  if ((rc = dalloc(ctx, &ctx->gslots, (size_t)std::max(total, 1))) ||
      (rc = dalloc(ctx, &ctx->rslots, (size_t)std::max(total, 1))))
    return rc;
  k_slice_fill<<<grid_for(C), kBlock, 0, st>>>(C, ctx->cptr, ctx->slots, ctx->sptr32,
                                                 ctx->gslots, ctx->rslots);
  // the node lists
  const int32_t N = ctx->N, nsn = (N + kSlice - 1) / kSlice;
  int32_t *nwidth = nullptr;
  if ((rc = sc.get(&nwidth, (int64_t)nsn + 1))) return rc;
  if ((rc = dalloc(ctx, &ctx->nsptr32, (size_t)nsn + 1))) return rc;
  k_slice_width<<<grid_for((int64_t)nsn + 1), kBlock, 0, st>>>(N, ctx->nptr, nwidth);
  if ((rc = dev_scan(sc, nwidth, ctx->nsptr32, nsn + 1, st))) return rc;
  int32_t ntotal = 0;
  if ((rc = dev_read_i32(ctx->nsptr32 + nsn, &ntotal, st))) return rc;
  if ((rc = dalloc(ctx, &ctx->nsl, (size_t)std::max(ntotal, 1)))) return rc;
  k_node_slice_fill<<<grid_for(N), kBlock, 0, st>>>(N, ctx->nptr, ctx->nsrc, ctx->nw,
                                                      ctx->nsptr32, ctx->nsl);
  MFG_CUDA(cudaGetLastError());
  MFG_CUDA(cudaStreamSynchronize(st));
  return MFG_OK;
}

template <typename T>
int d2h(std::vector<T> &h, const T *d, int64_t count, cudaStream_t st) {
  h.resize((size_t)std::max<int64_t>(count, 0));
  if (count > 0)
    MFG_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost, st));
  return MFG_OK;
}

// One sweep direction of build_levels on the device: levels, level-sorted
// cells and their per-level records, then (after the chunk assignment) the
// chunk-major persistent tables.
struct DevSweep {
  bool fwd = true;
  int32_t *cnt = nullptr, *deg = nullptr, *lvl = nullptr;  // device scratch
  std::vector<int32_t> lptr;                              // level starts
  int32_t L = 0;
  std::vector<int32_t> h_cells, h_sptr, h_nbs, h_assign;  // for the chunk assignment
};

int dev_levels(mfg_ctx *ctx, DevScratch &sc, DevSweep &d, int32_t *front, int32_t *next,
               int32_t *counter) {
  const int32_t C = ctx->C;
  cudaStream_t st = ctx->stream;
  MFG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
  k_dev_level_seed<<<grid_for(C), kBlock, 0, st>>>(C, d.deg, d.lvl, front, counter);
  count_launch();
  MFG_CUDA(cudaGetLastError());
  int32_t nf = 0;
  int rc;
  if ((rc = dev_read_i32(counter, &nf, st))) return rc;
  d.lptr.assign(1, 0);
  int64_t done = 0;
  int32_t level = 0;
  while (nf > 0) {
    d.lptr.push_back(d.lptr.back() + nf);
    ctx->max_level_cells = std::max(ctx->max_level_cells, nf);
    done += nf;
    MFG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
    k_dev_level_step<<<grid_for(nf), kBlock, 0, st>>>(nf, front, level, d.fwd ? 1 : 0, C,
                                                     ctx->cptr, ctx->slots, d.deg, d.lvl, next,
                                                     counter);
    count_launch();
    MFG_CUDA(cudaGetLastError());
    if ((rc = dev_read_i32(counter, &nf, st))) return rc;
    std::swap(front, next);
    if (++level > C) return MFG_ERR_BADMESH;
  }
  if (done != C) return MFG_ERR_BADMESH;  // a dependency cycle
  d.L = level;
  // level-sorted cells (ascending index within a level) and their records
  int32_t *idx = nullptr, *keys = nullptr, *g = nullptr;
  int32_t **cells = d.fwd ? &ctx->fw_cells : &ctx->bw_cells;
  int32_t **sptr = d.fwd ? &ctx->fw_sptr : &ctx->bw_sptr;
  int32_t **nbs = d.fwd ? &ctx->fw_nb : &ctx->bw_nb;
  SweepRec **recs = d.fwd ? &ctx->fw_recs : &ctx->bw_recs;
  if ((rc = sc.get(&idx, C)) || (rc = sc.get(&keys, C)) || (rc = sc.get(&g, (int64_t)C + 1)) ||
      (rc = dalloc(ctx, cells, C)) || (rc = dalloc(ctx, sptr, (size_t)C + 1)))
    return rc;
  k_dev_iota<<<grid_for(C), kBlock, 0, st>>>(C, idx);
  count_launch();
  if ((rc = dev_sort_pairs(sc, d.lvl, keys, idx, *cells, C, d.L, st))) return rc;
  k_dev_gather_cnt<<<grid_for((int64_t)C + 1), kBlock, 0, st>>>(C, *cells, d.cnt, g);
  count_launch();
  if ((rc = dev_scan(sc, g, *sptr, C + 1, st))) return rc;
  int32_t S = 0;
  if ((rc = dev_read_i32(*sptr + C, &S, st))) return rc;
  if ((rc = dalloc(ctx, recs, S)) || (rc = dalloc(ctx, nbs, S))) return rc;
  k_dev_level_records<<<grid_for(C), kBlock, 0, st>>>(C, *cells, *sptr, ctx->cptr, ctx->slots,
                                                       d.fwd ? 1 : 0, *recs, *nbs);
  count_launch();
  MFG_CUDA(cudaGetLastError());
  // what the chunk assignment on the host reads
  if ((rc = d2h(d.h_cells, (const int32_t *)*cells, C, st)) ||
      (rc = d2h(d.h_sptr, (const int32_t *)*sptr, (int64_t)C + 1, st)) ||
      (rc = d2h(d.h_nbs, (const int32_t *)*nbs, S, st)))
    return rc;
  MFG_CUDA(cudaStreamSynchronize(st));
  return MFG_OK;
}

int dev_pack(mfg_ctx *ctx, DevScratch &sc, DevSweep &d) {
  const int32_t C = ctx->C, P = ctx->nchunks, W = std::max(ctx->sweep_w, 1);
  cudaStream_t st = ctx->stream;
  int rc;
  int32_t *assign = nullptr, *keys = nullptr, *idx = nullptr, *pchunk = nullptr, *order = nullptr;
  int32_t *chunk_cnt = nullptr, *chunk_ptr = nullptr, *ccells = nullptr, *posof = nullptr;
  int32_t *head = nullptr, *hscan = nullptr, *exported = nullptr;
  if ((rc = sc.get(&assign, C)) || (rc = sc.get(&keys, C)) || (rc = sc.get(&idx, C)) ||
      (rc = sc.get(&pchunk, C)) || (rc = sc.get(&order, C)) ||
      (rc = sc.get(&chunk_cnt, (int64_t)P + 1)) || (rc = sc.get(&chunk_ptr, (int64_t)P + 1)) ||
      (rc = sc.get(&ccells, C)) || (rc = sc.get(&posof, C)) ||
      (rc = sc.get(&head, (int64_t)C + 1)) || (rc = sc.get(&hscan, (int64_t)C + 1)) ||
      (rc = sc.get(&exported, 4)))
    return rc;
  MFG_CUDA(cudaMemcpyAsync(assign, d.h_assign.data(), sizeof(int32_t) * C,
                           cudaMemcpyHostToDevice, st));
  MFG_CUDA(cudaMemsetAsync(chunk_cnt, 0, sizeof(int32_t) * ((size_t)P + 1), st));
  MFG_CUDA(cudaMemsetAsync(exported, 0, 4 * sizeof(int32_t), st));
  const int32_t *cells = d.fwd ? ctx->fw_cells : ctx->bw_cells;
  const int32_t *sptr = d.fwd ? ctx->fw_sptr : ctx->bw_sptr;
  const int32_t *nbs = d.fwd ? ctx->fw_nb : ctx->bw_nb;
  const SweepRec *recs = d.fwd ? ctx->fw_recs : ctx->bw_recs;
  k_dev_chunk_keys<<<grid_for(C), kBlock, 0, st>>>(C, cells, assign, keys, idx, chunk_cnt);
  count_launch();
  if ((rc = dev_sort_pairs(sc, keys, pchunk, idx, order, C, P, st))) return rc;
  if ((rc = dev_scan(sc, chunk_cnt, chunk_ptr, P + 1, st))) return rc;
  k_dev_positions<<<grid_for((int64_t)C + 1), kBlock, 0, st>>>(C, order, cells, pchunk, d.lvl,
                                                               ccells, posof, head);
  count_launch();
  if ((rc = dev_scan(sc, head, hscan, C + 1, st))) return rc;
  int32_t nseg = 0;
  if ((rc = dev_read_i32(hscan + C, &nseg, st))) return rc;
  ChunkSweep &cs = d.fwd ? ctx->fwc : ctx->bwc;
  cs.nseg = nseg;
  if ((rc = dalloc(ctx, &cs.seg_begin, (size_t)P + 1)) ||
      (rc = dalloc(ctx, &cs.segs, (size_t)nseg + 1)) || (rc = dalloc(ctx, &cs.cells, C)))
    return rc;
  k_dev_segs<<<grid_for((int64_t)C + 1), kBlock, 0, st>>>(C, head, hscan, cs.segs);
  k_dev_seg_begin<<<grid_for((int64_t)P + 1), kBlock, 0, st>>>(P, chunk_ptr, hscan, cs.seg_begin);
  count_launch(2);
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const bool with_recs = ctx->sweep_w != 0;
  const size_t nrec = with_recs ? (size_t)C * W : 0;
  const size_t nrec1 = std::max<size_t>(nrec, 1);
  if ((rc = dalloc(ctx, &cs.nbs, nrec)) || (rc = dalloc(ctx, &cs.nslots, nrec))) return rc;
  if (mx) {
    if ((rc = dalloc(ctx, &cs.recs_f, nrec))) return rc;
    MFG_CUDA(cudaMemsetAsync(cs.recs_f, 0, sizeof(SweepRecF) * nrec1, st));
  } else {
    if ((rc = dalloc(ctx, &cs.recs, nrec))) return rc;
    MFG_CUDA(cudaMemsetAsync(cs.recs, 0, sizeof(SweepRec) * nrec1, st));
  }
  MFG_CUDA(cudaMemsetAsync(cs.nbs, 0, sizeof(int32_t) * nrec1, st));
  MFG_CUDA(cudaMemsetAsync(cs.nslots, 0, sizeof(int32_t) * nrec1, st));
  if (mx)
    k_dev_pack<true><<<grid_for(C), kBlock, 0, st>>>(
        C, W, with_recs, order, ccells, pchunk, head, hscan, cs.segs, chunk_ptr, posof, assign,
        sptr, nbs, recs, cs.cells, cs.nbs, nullptr, cs.recs_f, cs.nslots, exported, exported + 1,
        ctx->ring);
  else
    k_dev_pack<false><<<grid_for(C), kBlock, 0, st>>>(
        C, W, with_recs, order, ccells, pchunk, head, hscan, cs.segs, chunk_ptr, posof, assign,
        sptr, nbs, recs, cs.cells, cs.nbs, cs.recs, nullptr, cs.nslots, exported, exported + 1,
        ctx->ring);
  count_launch();
  MFG_CUDA(cudaGetLastError());
  int32_t ex[4] = {0, 0, 0, 0};
  MFG_CUDA(cudaMemcpyAsync(ex, exported, sizeof(ex), cudaMemcpyDeviceToHost, st));
  MFG_CUDA(cudaStreamSynchronize(st));
  if (d.fwd) ctx->chunk0_exported = ex[0] != 0;
  for (int k = 0; k < 3; k++) ctx->sweep_stats[d.fwd ? 0 : 1][k] = ex[1 + k];
  (d.fwd ? ctx->fw_lptr : ctx->bw_lptr) = d.lptr;
  return MFG_OK;
}

int create_from_prep_impl(const mfg_prep_gpu *pp, const mfg_params *params, const double *q0,
                          int32_t precision, mfg_ctx **out) {
  if (!out || !pp || !params || !q0) return MFG_ERR_INVALID;
  *out = nullptr;
  CaseLayout cl;
  mfg_ctx *ctx = nullptr;
  int rc = ctx_begin(pp->N, pp->F, pp->C, pp->B, params, cl, pp->device, precision, &ctx);
  if (rc) return rc;
  auto fail = [&](int code) {
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    return code;
  };
  const int32_t C = ctx->C, F = ctx->F, G = ctx->G, N = ctx->N;
  const int64_t n = ctx->n;
  cudaStream_t st = ctx->stream;
  DevScratch sc;
  // [0] bad slot, [1] most records of a cell, [2] bad node list, [3] most faces of a cell
  int32_t *flags = nullptr;
  if ((rc = sc.get(&flags, 4))) return fail(rc);
  MFG_CUDA_OR(cudaMemsetAsync(flags, 0, 4 * sizeof(int32_t), st));
  // slots, faces, volumes, BC types
  ctx->S = pp->S;
  if ((rc = dalloc(ctx, &ctx->cptr, (size_t)C + 1)) || (rc = dalloc(ctx, &ctx->slots, pp->S)) ||
      (rc = dalloc(ctx, &ctx->faces, F)) || (rc = dalloc(ctx, &ctx->fflux, (size_t)kFluxRow * F)) ||
      (rc = dalloc(ctx, &ctx->bctype_d, G)) || (rc = dalloc(ctx, &ctx->vol, n)))
    return fail(rc);
  MFG_CUDA_OR(cudaMemcpyAsync(ctx->cptr, pp->cptr, sizeof(int32_t) * ((size_t)C + 1),
                              cudaMemcpyDeviceToDevice, st));
  if (G > 0)
    MFG_CUDA_OR(cudaMemcpyAsync(ctx->bctype_d, pp->bctype, sizeof(int32_t) * G,
                                cudaMemcpyDeviceToDevice, st));
  MFG_CUDA_OR(
      cudaMemcpyAsync(ctx->vol, pp->vol, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  k_dev_slots<<<grid_for(C), kBlock, 0, st>>>(C, G, pp->cptr, pp->cf, pp->fptr, pp->f2n,
                                              pp->f2c, pp->bctype,
                                              pp->xfn, pp->yfn, pp->zfn, pp->area, pp->xfc,
                                              pp->yfc, pp->zfc, pp->xcc, pp->ycc, pp->zcc,
                                              ctx->slots, flags, flags + 3);
  k_dev_faces<<<grid_for(F), kBlock, 0, st>>>(F, pp->f2c, pp->xfn, pp->yfn, pp->zfn, pp->area,
                                              ctx->faces);
  if ((rc = dalloc(ctx, &ctx->fcen, F)) || (rc = dalloc(ctx, &ctx->ccen, n))) return fail(rc);
  k_centroids<<<grid_for(std::max<int64_t>(F, n)), kBlock, 0, st>>>(
      F, n, pp->xfc, pp->yfc, pp->zfc, pp->xcc, pp->ycc, pp->zcc, pp->vol, ctx->fcen, ctx->ccen);
  count_launch(3);
  // record counts, the record width W and the chunk grid
  DevSweep fw, bw;
  fw.fwd = true;
  bw.fwd = false;
  if ((rc = sc.get(&fw.cnt, C)) || (rc = sc.get(&bw.cnt, C)) || (rc = sc.get(&fw.deg, C)) ||
      (rc = sc.get(&bw.deg, C)) || (rc = sc.get(&fw.lvl, C)) || (rc = sc.get(&bw.lvl, C)))
    return fail(rc);
  k_dev_counts<<<grid_for(C), kBlock, 0, st>>>(C, ctx->cptr, ctx->slots, fw.cnt, bw.cnt, fw.deg,
                                               bw.deg, flags + 1);
  count_launch();
  MFG_CUDA_OR(cudaGetLastError());
  int32_t h_flags[4] = {0, 0, 0, 0};
  MFG_CUDA_OR(cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
  MFG_CUDA_OR(cudaStreamSynchronize(st));
  if (h_flags[0]) return fail(MFG_ERR_BADMESH);
  ctx->gather_lanes_fit = gather_lanes_for(h_flags[3]);
  {
    // the choices of build_levels (the kernel kind once the levels are known)
    setup_sweep_grid(ctx, h_flags[1]);
    ctx->first_cell = 0;
  }
  const int32_t maxns_dev = h_flags[1];
  {
    int32_t *front = nullptr, *next = nullptr, *counter = nullptr;
    if ((rc = sc.get(&front, C)) || (rc = sc.get(&next, C)) || (rc = sc.get(&counter, 1)))
      return fail(rc);
    if ((rc = dev_levels(ctx, sc, fw, front, next, counter))) return fail(rc);
    if ((rc = dev_levels(ctx, sc, bw, front, next, counter))) return fail(rc);
  }
  setup_sweep_grid(ctx, maxns_dev);
  // the chunk assignment runs on the host, both sweeps at once, from the
  // cell centroids
  {
    const int32_t P = ctx->nchunks;
    std::vector<double> cx, cy, cz;
    if ((rc = d2h(cx, pp->xcc, C, st)) || (rc = d2h(cy, pp->ycc, C, st)) ||
        (rc = d2h(cz, pp->zcc, C, st)))
      return fail(rc);
    MFG_CUDA_OR(cudaStreamSynchronize(st));
    const double *xyz[3] = {cx.data(), cy.data(), cz.data()};
    const int force = g_chunking.load();
    const int32_t G = sweep_groups(ctx->sweep_w, ctx->sweep_kind);
    std::thread tb([&] {
      choose_chunks(C, P, G, bw.lptr, bw.h_cells.data(), bw.h_sptr.data(), bw.h_nbs.data(), xyz,
                    force, bw.h_assign, &ctx->chunk_est_us[1]);
    });
    ctx->chunking = choose_chunks(C, P, G, fw.lptr, fw.h_cells.data(), fw.h_sptr.data(),
                                  fw.h_nbs.data(), xyz, force, fw.h_assign, &ctx->chunk_est_us[0]);
    tb.join();
  }
  if ((rc = dev_pack(ctx, sc, fw))) return fail(rc);
  if ((rc = dev_pack(ctx, sc, bw))) return fail(rc);
  // node lists
  {
    int32_t *cnt = nullptr;
    if ((rc = sc.get(&cnt, (int64_t)N + 1))) return fail(rc);
    MFG_CUDA_OR(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ((size_t)N + 1), st));
    k_dev_node_lists<false><<<grid_for(N), kBlock, 0, st>>>(
        N, pp->nbptr, pp->nblist, pp->bent_face, pp->bctype, pp->ncptr, pp->nclist,
        pp->c2n_cell, pp->nmark, pp->wbface, pp->wc2n, cnt, flags + 2, nullptr, nullptr, nullptr);
    count_launch();
    if ((rc = dalloc(ctx, &ctx->nptr, (size_t)N + 1))) return fail(rc);
    if ((rc = dev_scan(sc, cnt, ctx->nptr, N + 1, st))) return fail(rc);
    int32_t tot = 0, badn = 0;
    if ((rc = dev_read_i32(ctx->nptr + N, &tot, st))) return fail(rc);
    if ((rc = dev_read_i32(flags + 2, &badn, st))) return fail(rc);
    if (badn) return fail(MFG_ERR_UNSUPPORTED);  // as build_node_lists
    if ((rc = dalloc(ctx, &ctx->nsrc, tot)) || (rc = dalloc(ctx, &ctx->nw, tot)) ||
        (rc = dalloc(ctx, &ctx->ninfo, N)) || (rc = dalloc(ctx, &ctx->nsym, 3 * (size_t)N)) ||
        (rc = dalloc(ctx, &ctx->wnode, N)) ||
        (rc = dalloc(ctx, &ctx->bface_c1, (size_t)std::max(G, 1))) ||
        (rc = dalloc(ctx, &ctx->fnptr, (size_t)F + 1)) || (rc = dalloc(ctx, &ctx->fnodes, pp->L)))
      return fail(rc);
    k_dev_node_lists<true><<<grid_for(N), kBlock, 0, st>>>(
        N, pp->nbptr, pp->nblist, pp->bent_face, pp->bctype, pp->ncptr, pp->nclist,
        pp->c2n_cell, pp->nmark, pp->wbface, pp->wc2n, nullptr, nullptr, ctx->nptr, ctx->nsrc,
        ctx->nw);
    k_dev_node_info<<<grid_for(N), kBlock, 0, st>>>(N, pp->nmark, pp->nodesymm, pp->xsym,
                                                    pp->ysym, pp->zsym, ctx->ninfo, ctx->nsym);
    MFG_CUDA_OR(cudaMemsetAsync(ctx->bface_c1, 0, sizeof(int32_t), st));
    k_dev_bface_c1<<<grid_for(std::max(G, 1)), kBlock, 0, st>>>(G, pp->f2c, ctx->bface_c1);
    count_launch(3);
    MFG_CUDA_OR(cudaMemcpyAsync(ctx->wnode, pp->wnode, sizeof(double) * N,
                                cudaMemcpyDeviceToDevice, st));
    MFG_CUDA_OR(cudaMemcpyAsync(ctx->fnptr, pp->fptr, sizeof(int32_t) * ((size_t)F + 1),
                                cudaMemcpyDeviceToDevice, st));
    if (pp->L > 0)
      MFG_CUDA_OR(cudaMemcpyAsync(ctx->fnodes, pp->f2n, sizeof(int32_t) * pp->L,
                                  cudaMemcpyDeviceToDevice, st));
    MFG_CUDA_OR(cudaGetLastError());
  }
  MFG_CUDA_OR(cudaStreamSynchronize(st));
  if ((rc = ctx_finish(ctx, q0, cl))) return fail(rc);
  *out = ctx;
  return MFG_OK;
}

}  // namespace

extern "C" {

int mfg_create_from_prep(const mfg_prep_gpu *prep, const mfg_params *params, const double *q0,
                         int32_t precision, mfg_ctx **out) {
  return create_from_prep_impl(prep, params, q0, precision, out);
}

int mfg_set_stream(mfg_ctx *ctx, void *s) {
  if (!ctx) return MFG_ERR_INVALID;
  ctx->stream = s ? (cudaStream_t)s : ctx->own_stream;
  return MFG_OK;
}

int mfg_set_params(mfg_ctx *ctx, const mfg_params *p) {
  if (!ctx || !p) return MFG_ERR_INVALID;
  if (ctx->ncase > 1) return MFG_ERR_UNSUPPORTED;  // a batch fixes its cases at creation
  ctx->hp = *p;
  ctx->hps[0] = *p;
  ctx->P = make_params(*p);
  for (int k = 0; k < 2; k++)
    if (ctx->graph[k]) {
      cudaGraphExecDestroy(ctx->graph[k]);
      ctx->graph[k] = nullptr;
    }
  return MFG_OK;
}

int mfg_set_sweep_mode(mfg_ctx *ctx, int32_t mode) {
  if (!ctx || (mode != 0 && mode != 1)) return MFG_ERR_INVALID;
  if (mode == 1 && ctx->persist_grid <= 0) return MFG_ERR_UNSUPPORTED;
  ctx->sweep_mode = mode;
  for (int k = 0; k < 2; k++)
    if (ctx->graph[k]) {
      cudaGraphExecDestroy(ctx->graph[k]);
      ctx->graph[k] = nullptr;
    }
  return MFG_OK;
}

int mfg_info_get(mfg_ctx *ctx, mfg_info *info) {
  if (!ctx || !info) return MFG_ERR_INVALID;
  info->n_cell = ctx->C;
  info->n_face = ctx->F;
  info->n_node = ctx->N;
  info->n_bface = ctx->G;
  info->fw_levels = (int32_t)ctx->fw_lptr.size() - 1;
  info->bw_levels = (int32_t)ctx->bw_lptr.size() - 1;
  info->max_level_cells = ctx->max_level_cells;
  info->precision = ctx->precision;
  info->device_bytes = ctx->device_bytes;
  info->sweep_mode = ctx->sweep_mode;
  info->graph_ready = ctx->graph[0] != nullptr;
  info->ncase = ctx->ncase;
  info->sweep_chunks = ctx->sweep_mode == 1 ? ctx->nchunks : 0;
  info->sweep_lanes = ctx->sweep_mode == 1 ? ctx->sweep_lanes : 0;
  info->sweep_records = ctx->sweep_w;
  info->sweep_chunking = ctx->chunking;
  info->sweep_kernel = ctx->sweep_kind;
  for (int k = 0; k < 2; k++) {
    info->sweep_ring_records[k] = ctx->sweep_stats[k][0];
    info->sweep_global_records[k] = ctx->sweep_stats[k][1];
    info->sweep_cross_records[k] = ctx->sweep_stats[k][2];
    info->sweep_model_us[k] = ctx->chunk_est_us[k];
  }
  return MFG_OK;
}

int mfg_set_chunking(int32_t kind) {
  if (kind < -1 || kind > MFG_CHUNK_TRANSVERSE_ANY) return MFG_ERR_INVALID;
  g_chunking.store(kind);
  return MFG_OK;
}

int mfg_plan_chunks(int32_t C, int32_t L, const int32_t *lptr, const int32_t *cells,
                    const int32_t *sptr, const int32_t *nbs, const double *xc,
                    const double *yc, const double *zc, int32_t P, int32_t G, int32_t force,
                    int32_t *assign, int32_t *grid, double *est_us) {
  if (C < 0 || L < 0 || P < 1 || G < 1 || !lptr || (C > 0 && (!cells || !sptr || !nbs || !assign)))
    return MFG_ERR_INVALID;
  if (force < -1 || force > MFG_CHUNK_TRANSVERSE_ANY) return MFG_ERR_INVALID;
  // the tables are indexed by what they hold: check them all first
  if (lptr[0] != 0 || lptr[L] != C) return MFG_ERR_INVALID;
  for (int32_t l = 0; l < L; l++)
    if (lptr[l + 1] < lptr[l]) return MFG_ERR_INVALID;
  std::vector<char> seen(C, 0);
  for (int32_t i = 0; i < C; i++) {
    if (cells[i] < 0 || cells[i] >= C || seen[cells[i]]) return MFG_ERR_INVALID;
    seen[cells[i]] = 1;
  }
  if (C > 0 && sptr[0] != 0) return MFG_ERR_INVALID;
  for (int32_t i = 0; i < C; i++)
    if (sptr[i + 1] < sptr[i]) return MFG_ERR_INVALID;
  for (int32_t s0 = 0; C > 0 && s0 < sptr[C]; s0++)
    if (nbs[s0] < 0) return MFG_ERR_INVALID;
  const std::vector<int32_t> lp(lptr, lptr + L + 1);
  const double *const xyz[3] = {xc, yc, zc};
  std::vector<int32_t> a;
  int32_t g[2] = {0, 0};
  double us = 0.0;
  const int choice = choose_chunks(C, P, G, lp, cells, sptr, nbs, xyz, force, a, &us, g);
  if (C > 0) std::copy(a.begin(), a.end(), assign);
  if (grid) {
    grid[0] = g[0];
    grid[1] = g[1];
  }
  if (est_us) *est_us = us;
  return choice;
}

int mfg_set_sweep_kernel(int32_t kind) {
  if (kind < -1 || kind > MFG_SWEEP_WIDE) return MFG_ERR_INVALID;
  g_sweep_kind.store(kind);
  return MFG_OK;
}

static void drop_graphs(mfg_ctx *ctx) {
  for (int k = 0; k < 2; k++)
    if (ctx->graph[k]) {
      cudaGraphExecDestroy(ctx->graph[k]);
      ctx->graph[k] = nullptr;
    }
}

int mfg_set_gather_lanes(mfg_ctx *ctx, int32_t lanes) {
  if (!ctx || lanes < 0) return MFG_ERR_INVALID;
  if (lanes != 0 && lanes != ctx->gather_lanes_fit) return MFG_ERR_UNSUPPORTED;
  ctx->gather_lanes = lanes;
  drop_graphs(ctx);
  return MFG_OK;
}


static int launch_ghost_bc(mfg_ctx *ctx, cudaStream_t st) {
  if (ctx->G == 0) return MFG_OK;
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  k_ghost_bc<<<grid_for(ctx->G), kBlock, 0, st>>>(
      ctx->G, ctx->C, ctx->faces, ctx->bctype_d, ctx->q8[ctx->cur], ctx->q8[ctx->cur ^ 1],
      mx ? ctx->q4[ctx->cur] : nullptr, mx ? ctx->q4[ctx->cur ^ 1] : nullptr, ctx->P,
      cases_of(ctx));
  count_launch();
  return check_kernel();
}

int mfg_set_ghost_variables(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  return launch_ghost_bc(ctx, ctx->stream);
}

int mfg_set_flux_fp64(mfg_ctx *ctx, int32_t on) {
  if (!ctx || (on != 0 && on != 1)) return MFG_ERR_INVALID;
  if (ctx->precision != MFG_PREC_MIXED) return on ? MFG_OK : MFG_ERR_UNSUPPORTED;
  if (ctx->flux_fp64 != on) {
    ctx->flux_fp64 = on;
    drop_graphs(ctx);
  }
  return MFG_OK;
}

static int launch_gradient(mfg_ctx *ctx);

int mfg_set_order(mfg_ctx *ctx, int32_t order, double venkat_k) {
  if (!ctx || order < 1 || order > 4 || !(venkat_k > 0.0)) return MFG_ERR_INVALID;
  // across parts, second order needs the gradient rows' exchange buffers
  if (ctx->halo && order != 1 && ctx->hb.n_send + ctx->hb.n_recv > 0 &&
      (!ctx->hb.grad_send || !ctx->hb.grad_recv))
    return MFG_ERR_UNSUPPORTED;
  MFG_CUDA(cudaSetDevice(ctx->device));
  int rc;
  if (order >= 3 && !ctx->phi && (rc = dalloc(ctx, &ctx->phi, (size_t)5 * ctx->n))) return rc;
  if (order != ctx->order) drop_graphs(ctx);
  ctx->order = order;
  ctx->venkat_k = venkat_k;
  if (order >= 3)
    MFG_CUDA(cudaMemsetAsync(ctx->phi, 0, sizeof(double) * 5 * ctx->n, ctx->stream));
  // the next flux reads the gradient of the current state (a part's comes
  // from its GRADIENT phase)
  return order >= 2 && !ctx->halo ? launch_gradient(ctx) : MFG_OK;
}

int mfg_set_live_bc(mfg_ctx *ctx, int32_t on) {
  if (!ctx || (on != 0 && on != 1)) return MFG_ERR_INVALID;
  if (ctx->live_bc != on) {
    ctx->live_bc = on;
    drop_graphs(ctx);  // the captured iteration gains or loses the ghost update
  }
  return MFG_OK;
}

int mfg_set_sweep_lanes(mfg_ctx *ctx, int32_t lanes) {
  if (!ctx) return MFG_ERR_INVALID;
  if (!ctx->sweep_w || ctx->sweep_mode != 1 || lanes != ctx->sweep_w) return MFG_ERR_UNSUPPORTED;
  ctx->sweep_lanes = lanes;
  for (int k = 0; k < 2; k++)
    if (ctx->graph[k]) {
      cudaGraphExecDestroy(ctx->graph[k]);
      ctx->graph[k] = nullptr;
    }
  return MFG_OK;
}

int mfg_batch_layout(mfg_ctx *ctx, int32_t *cell0, int32_t *bface0) {
  if (!ctx || !cell0 || !bface0) return MFG_ERR_INVALID;
  for (int32_t k = 0; k <= ctx->ncase; k++) {
    cell0[k] = ctx->case_cell0[k];
    bface0[k] = ctx->case_bface0[k];
  }
  return MFG_OK;
}

int mfg_batch_dt_extrema(mfg_ctx *ctx, double *ext) {
  if (!ctx || !ext) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  MFG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->dt_ext, 2 * sizeof(double) * ctx->ncase,
                           cudaMemcpyDeviceToHost, ctx->stream));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(ext, ctx->h_pinned, 2 * sizeof(double) * ctx->ncase);
  return MFG_OK;
}

int mfg_zero_residuals(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  ctx->res_zero = true;  // the next flux gather writes instead of accumulating
  return MFG_OK;
}

static int launch_face(mfg_ctx *ctx, bool flux, bool dtp, bool diag, double cfl,
                       bool use_table, bool limiter = true) {
  cudaStream_t st = ctx->stream;
  const int g = grid_for(ctx->C);
  const double *q = ctx->q8[ctx->cur];
  const double *tab = use_table ? ctx->cfl_tab : nullptr;
  double *np = (flux && ctx->ncase == 1) ? ctx->norm_part : nullptr;
  const Cases cs = cases_of(ctx);
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  if (flux) {  // each face's Roe flux once, then gathered per cell
    const bool recon = ctx->order >= 2;
    const double *phi = ctx->order >= 3 ? ctx->phi : nullptr;
    if (ctx->order >= 3 && limiter) {
      if (ctx->order == 4)
        k_limiter<true><<<g, kBlock, 0, st>>>(ctx->C, ctx->n, ctx->cptr, ctx->slots, q,
                                              ctx->dqdx, ctx->dqdy, ctx->dqdz, ctx->fcen,
                                              ctx->ccen, ctx->venkat_k, ctx->phi);
      else
        k_limiter<false><<<g, kBlock, 0, st>>>(ctx->C, ctx->n, ctx->cptr, ctx->slots, q,
                                               ctx->dqdx, ctx->dqdy, ctx->dqdz, ctx->fcen,
                                               ctx->ccen, ctx->venkat_k, ctx->phi);
      count_launch();
    }
#define MFG_FLUX(MX_, R_, M_)                                                                 \
  k_face_flux<MX_, R_, M_><<<grid_for(ctx->F), kBlock, 0, st>>>(                               \
      ctx->F, ctx->faces, q, ctx->P, cs, ctx->fflux, ctx->C, ctx->n, ctx->fcen, ctx->ccen,     \
      ctx->dqdx, ctx->dqdy, ctx->dqdz, phi, ctx->halo ? ctx->h_gflag : nullptr)
    const bool fmx = mx && !ctx->flux_fp64;
    const int fm = ctx->flux_minb;
    if (fmx && recon)
      MFG_FLUX(true, true, MFG_FLUX_MINB);
    else if (recon)
      MFG_FLUX(false, true, MFG_FLUX_MINB);
    else if (fmx && fm == 2)
      MFG_FLUX(true, false, 2);
    else if (fmx && fm == 4)
      MFG_FLUX(true, false, 4);
    else if (fmx)
      MFG_FLUX(true, false, 3);
    else if (fm == 2)
      MFG_FLUX(false, false, 2);
    else if (fm == 4)
      MFG_FLUX(false, false, 4);
    else
      MFG_FLUX(false, false, 3);
#undef MFG_FLUX
    count_launch();
  }
  if (ctx->gather_lanes == 4 || ctx->gather_lanes == 8) {
    const int gl = grid_for((int64_t)ctx->C * ctx->gather_lanes);
#define MFG_LANES(L_, F_, D_, G_, M_)                                                          \
  k_face_gather_lanes<L_, F_, D_, G_, M_><<<gl, kBlock, 0, st>>>(                              \
      ctx->C, ctx->cptr, ctx->slots, q, ctx->vol, ctx->res, ctx->res_zero ? 1 : 0, ctx->dt,    \
      ctx->diag, tab, ctx->iter_counter, cfl, ctx->P, ctx->dt_ext, nullptr, cs, ctx->fflux)
#define MFG_LANES_L(F_, D_, G_, M_)                                                            \
  if (ctx->gather_lanes == 4)                                                                 \
    MFG_LANES(4, F_, D_, G_, M_);                                                             \
  else                                                                                        \
    MFG_LANES(8, F_, D_, G_, M_)
    if (flux && dtp && diag) {
      if (ctx->gather_minb == 2) {
        MFG_LANES_L(true, true, true, 2);
      } else if (ctx->gather_minb == 4) {
        MFG_LANES_L(true, true, true, 4);
      } else {
        MFG_LANES_L(true, true, true, 3);
      }
    } else if (flux && !dtp && !diag) {
      MFG_LANES_L(true, false, false, MFG_GATHER_MINB);
    } else if (!flux && dtp && !diag) {
      MFG_LANES_L(false, true, false, MFG_GATHER_MINB);
    } else if (!flux && !dtp && diag) {
      MFG_LANES_L(false, false, true, MFG_GATHER_MINB);
    } else {
      return MFG_ERR_INVALID;
    }
#undef MFG_LANES_L
#undef MFG_LANES
    count_launch();
    if (np) {  // the norm partials, from res in the one-thread gather's order
      k_norm_partial<<<gather_blocks(ctx), kBlock, 0, st>>>(ctx->C, ctx->res, np);
      count_launch();
    }
    if (flux) ctx->res_zero = false;
    return check_kernel();
  }
#define MFG_FACE_M(F_, D_, G_, M_)                                                            \
  if (mx)                                                                                     \
    k_face_gather_mx<F_, D_, G_, F_, M_><<<g, kBlock, 0, st>>>(                               \
        ctx->C, ctx->cptr, ctx->gslots, ctx->sptr32, q, ctx->vol, ctx->res, ctx->res_zero ? 1 : 0, ctx->dt,  \
        ctx->diag, tab, ctx->iter_counter, cfl, ctx->P, ctx->dt_ext, np, cs, ctx->fflux,       \
        ctx->F);                                                                              \
  else                                                                                        \
    k_face_gather<F_, D_, G_, F_, M_><<<g, kBlock, 0, st>>>(                                  \
        ctx->C, ctx->cptr, ctx->gslots, ctx->sptr32, q, ctx->vol, ctx->res, ctx->res_zero ? 1 : 0, ctx->dt,  \
        ctx->diag, tab, ctx->iter_counter, cfl, ctx->P, ctx->dt_ext, np, cs, ctx->fflux,       \
        ctx->F)
#define MFG_FACE(F_, D_, G_) MFG_FACE_M(F_, D_, G_, MFG_GATHER_MINB)
  if (flux && dtp && diag) {
    if (ctx->gather_minb == 2) {
      MFG_FACE_M(true, true, true, 2);
    } else if (ctx->gather_minb == 4) {
      MFG_FACE_M(true, true, true, 4);
    } else {
      MFG_FACE_M(true, true, true, 3);
    }
  } else if (flux && !dtp && !diag) {
    MFG_FACE(true, false, false);
  } else if (!flux && dtp && !diag) {
    MFG_FACE(false, true, false);
  } else if (!flux && !dtp && diag) {
    MFG_FACE(false, false, true);
  } else {
    return MFG_ERR_INVALID;
  }
#undef MFG_FACE
#undef MFG_FACE_M
  count_launch();
  if (flux) ctx->res_zero = false;
  return check_kernel();
}

int mfg_inviscid_flux(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  return launch_face(ctx, true, false, false, 0.0, false);
}

// LimitTimeStep's CFL (compute_timestep.cpp:865-873), evaluated with glibc.
static double cfl_for(const mfg_params &p, int32_t iter_done) {
  if (iter_done > p.cfl_nstep) return p.cfl_end;
  return p.cfl_start * pow(p.cfl_ratio, (double)iter_done / p.cfl_nstep);
}

static int fill_cfl_table(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done);

int mfg_compute_timestep(mfg_ctx *ctx, int32_t iter_done) {
  if (!ctx) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  const double cfl = cfl_for(ctx->hp, iter_done);
  ctx->hp.cfl_min = 0.5 * cfl;
  int rc;
  if (ctx->ncase > 1) {
    // one CFL per case (their ramps differ): through the CFL table, slot 0
    if ((rc = fill_cfl_table(ctx, 1, iter_done))) return rc;
    rc = launch_face(ctx, false, true, false, cfl, true);
  } else {
    rc = launch_face(ctx, false, true, false, cfl, false);
  }
  if (rc) return rc;
  k_dt_clamp<<<grid_for(ctx->C), kBlock, 0, ctx->stream>>>(ctx->C, ctx->dt, ctx->dt_ext, ctx->P,
                                                           cases_of(ctx));
  count_launch();
  return check_kernel();
}

static int launch_coop(const void *fn, int blocks, int threads, size_t smem, cudaStream_t st,
                       void **args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MFG_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
  count_launch();
  return MFG_OK;
}

static int launch_fwd_persist(mfg_ctx *ctx, bool clamp_check, int32_t chunk_skip,
                              long long spin) {
  const double *q = ctx->q8[ctx->cur];
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const void *qnb = mx ? (const void *)ctx->q4[ctx->cur] : (const void *)q;
  int32_t C = ctx->C, first = ctx->first_cell, skip = chunk_skip;
  int clamp = clamp_check ? 1 : 0;
  Params P = ctx->P;
  Cases cs = cases_of(ctx);
  ChunkSweep &w = ctx->fwc;
  void *recs = mx ? (void *)w.recs_f : (void *)w.recs;
  void *args[] = {&w.seg_begin, &w.segs, &w.cells, &recs, &w.nbs, &w.nslots, (void *)&q,
                  (void *)&qnb, &ctx->dqf, &ctx->dq8, &ctx->res, &C, &ctx->diag, &first, &P,
                  &clamp, &ctx->dt, &ctx->dt_ext, &ctx->cptr, &ctx->slots, &ctx->vol,
                  &ctx->sweep_err, &spin, &skip, &cs};
  const void *fn = sweep_kernel(true, ctx->sweep_w, mx, ctx->sweep_kind);
  if (!fn) return MFG_ERR_UNSUPPORTED;
  return launch_coop(fn, ctx->nchunks, sweep_threads(ctx->sweep_w, ctx->sweep_kind),
                     sweep_smem(ctx->sweep_w, mx, ctx->sweep_kind), ctx->stream, args);
}

static int launch_bwd_persist(mfg_ctx *ctx, long long spin) {
  const double *q = ctx->q8[ctx->cur];
  double *qn = ctx->q8[ctx->cur ^ 1];
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const void *qnb = mx ? (const void *)ctx->q4[ctx->cur] : (const void *)q;
  float *q4n = mx ? ctx->q4[ctx->cur ^ 1] : nullptr;
  Params P = ctx->P;
  Cases cs = cases_of(ctx);
  ChunkSweep &w = ctx->bwc;
  void *recs = mx ? (void *)w.recs_f : (void *)w.recs;
  void *args[] = {&w.seg_begin, &w.segs, &w.cells, &recs, &w.nbs, &w.nslots, (void *)&q,
                  (void *)&qnb, &qn, &q4n, &ctx->dqf, &ctx->dq8, &ctx->diag, &P,
                  &ctx->sweep_err, &spin, &cs};
  const void *fn = sweep_kernel(false, ctx->sweep_w, mx, ctx->sweep_kind);
  if (!fn) return MFG_ERR_UNSUPPORTED;
  const int rc = launch_coop(fn, ctx->nchunks, sweep_threads(ctx->sweep_w, ctx->sweep_kind),
                             sweep_smem(ctx->sweep_w, mx, ctx->sweep_kind), ctx->stream, args);
  if (rc || ctx->sweep_kind != MFG_SWEEP_WIDE) return rc;
  // the wide sweeps leave the update to a streaming pass
  if (mx)
    k_update_cells<true><<<grid_for(ctx->C), kBlock, 0, ctx->stream>>>(ctx->C, q, ctx->dq8, qn,
                                                                         q4n, P, cs);
  else
    k_update_cells<false><<<grid_for(ctx->C), kBlock, 0, ctx->stream>>>(ctx->C, q, ctx->dq8, qn,
                                                                          q4n, P, cs);
  count_launch();
  return MFG_OK;
}

// Reads the sweeps' error word; on a timeout, re-arms the flags so that the
// context stays usable, and reports MFG_ERR_TIMEOUT.  Synchronises.
static int check_sweep_error(mfg_ctx *ctx) {
  if (ctx->sweep_mode != 1) return MFG_OK;
  int *h = reinterpret_cast<int *>(ctx->h_pinned + 32);
  MFG_CUDA(cudaMemcpyAsync(h, ctx->sweep_err, sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*h == 0) return MFG_OK;
  k_arm_sentinel<<<grid_for(ctx->C), kBlock, 0, ctx->stream>>>(ctx->C, ctx->dqf);
  count_launch();
  MFG_CUDA(cudaMemsetAsync(ctx->sweep_err, 0, sizeof(int), ctx->stream));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  g_cuda_error = "an LU-SGS sweep gave up waiting for a neighbour (results invalid)";
  return MFG_ERR_TIMEOUT;
}

// One LU-SGS sweep: forward (DQ* into dqf) or backward (DQ into dq8 and the
// updated state into the other state buffer).
// One sweep as one launch per level (cells with more records than the
// persistent sweeps take, or sweep mode 0), either precision.
static void launch_level_sweep(mfg_ctx *ctx, bool fwd, bool clamp_check, cudaStream_t st) {
  const double *q = ctx->q8[ctx->cur];
  double *qn = ctx->q8[ctx->cur ^ 1];
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const float *q4 = mx ? ctx->q4[ctx->cur] : nullptr;
  float *q4n = mx ? ctx->q4[ctx->cur ^ 1] : nullptr;
  const Cases cs = cases_of(ctx);
  if (fwd) {
    const int Lf = (int)ctx->fw_lptr.size() - 1;
    auto kf = mx ? k_sweep_fwd<true> : k_sweep_fwd<false>;
    for (int l = 0; l < Lf; l++) {
      const int32_t a = ctx->fw_lptr[l], b = ctx->fw_lptr[l + 1];
      kf<<<grid_for(b - a), kBlock, 0, st>>>(a, b, ctx->fw_cells, ctx->fw_sptr, ctx->fw_recs,
                                             ctx->fw_nb, q, q4, ctx->dqf, ctx->dq8, ctx->res,
                                             ctx->C, ctx->diag, ctx->first_cell, ctx->P,
                                             clamp_check ? 1 : 0, ctx->dt, ctx->dt_ext,
                                             ctx->cptr, ctx->slots, ctx->vol, cs);
    }
    count_launch(Lf);
  } else {
    const int Lb = (int)ctx->bw_lptr.size() - 1;
    auto kb = mx ? k_sweep_bwd<true> : k_sweep_bwd<false>;
    for (int l = 0; l < Lb; l++) {
      const int32_t a = ctx->bw_lptr[l], b = ctx->bw_lptr[l + 1];
      kb<<<grid_for(b - a), kBlock, 0, st>>>(a, b, ctx->bw_cells, ctx->bw_sptr, ctx->bw_recs,
                                             ctx->bw_nb, q, q4, qn, q4n, ctx->dqf, ctx->dq8,
                                             ctx->diag, ctx->P, cs);
    }
    count_launch(Lb);
  }
}

static int launch_sweep(mfg_ctx *ctx, bool fwd, bool clamp_check) {
  if (ctx->sweep_mode == 1)
    return fwd ? launch_fwd_persist(ctx, clamp_check, 0, kSpinCycles)
               : launch_bwd_persist(ctx, kSpinCycles);
  launch_level_sweep(ctx, fwd, clamp_check, ctx->stream);
  return check_kernel();
}

static int launch_sweeps(mfg_ctx *ctx, bool clamp_check) {
  const int rc = launch_sweep(ctx, true, clamp_check);
  if (rc) return rc;
  return launch_sweep(ctx, false, clamp_check);
}

int mfg_forward_lusgs(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  MFG_CUDA(cudaSetDevice(ctx->device));
  int rc = launch_face(ctx, false, false, true, 0.0, false);
  if (rc) return rc;
  rc = launch_sweeps(ctx, false);
  if (rc) return rc;
  ctx->cur ^= 1;
  return check_sweep_error(ctx);
}

// Failure-detection self-test: a forward sweep whose first chunk is never
// run, so the cells that depend on it wait for flags nobody sets.  The
// bounded waits give up after spin_cycles; the call must return
// MFG_ERR_TIMEOUT and leave the context usable.  State is not changed.
int mfg_selftest_sweep_timeout(mfg_ctx *ctx, int64_t spin_cycles) {
  if (!ctx || spin_cycles <= 0) return MFG_ERR_INVALID;
  if (ctx->sweep_mode != 1 || ctx->nchunks < 2 || !ctx->chunk0_exported)
    return MFG_ERR_UNSUPPORTED;
  MFG_CUDA(cudaSetDevice(ctx->device));
  // keep DQ intact: the test sweep writes only cells of later levels, so
  // save and restore the whole increment array around it
  double *save = nullptr;
  int rc = dalloc(ctx, &save, (size_t)ctx->n * Q_STRIDE);
  if (rc) return rc;
  MFG_CUDA(cudaMemcpyAsync(save, ctx->dq8, sizeof(double) * ctx->n * Q_STRIDE,
                           cudaMemcpyDeviceToDevice, ctx->stream));
  rc = launch_fwd_persist(ctx, false, 1, (long long)spin_cycles);
  const int rc2 = check_sweep_error(ctx);
  cudaMemcpyAsync(ctx->dq8, save, sizeof(double) * ctx->n * Q_STRIDE, cudaMemcpyDeviceToDevice,
                  ctx->stream);
  k_arm_sentinel<<<grid_for(ctx->C), kBlock, 0, ctx->stream>>>(ctx->C, ctx->dqf);
  count_launch();
  cudaStreamSynchronize(ctx->stream);
  ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)save));
  ctx->device_bytes -= (int64_t)sizeof(double) * ctx->n * Q_STRIDE;
  cudaFree(save);
  if (rc) return rc;
  return rc2;
}

static void launch_node_values(mfg_ctx *ctx, cudaStream_t st) {
  const int nb = ctx->node_block;
  if (ctx->precision == MFG_PREC_MIXED)
    k_node_values_mx<<<grid_for(ctx->N, nb), nb, 0, st>>>(
        ctx->N, ctx->C, ctx->nptr, ctx->nsl, ctx->nsptr32, ctx->ninfo, ctx->wnode, ctx->nsym,
        ctx->bface_c1, ctx->q8[ctx->cur], ctx->qn4, ctx->P, cases_of(ctx));
  else
    k_node_values<<<grid_for(ctx->N, nb), nb, 0, st>>>(
        ctx->N, ctx->C, ctx->nptr, ctx->nsl, ctx->nsptr32, ctx->ninfo, ctx->wnode, ctx->nsym,
        ctx->bface_c1, ctx->q8[ctx->cur], ctx->qn8);
  count_launch();
}

static void launch_grad_faces(mfg_ctx *ctx, cudaStream_t st) {
  const int gb = ctx->grad_block;
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const int L = ctx->gather_lanes;
  if (L == 4 || L == 8) {
    const int g = grid_for((int64_t)ctx->C * L, gb);
    const double *q = ctx->q8[ctx->cur];
#define MFG_GRAD_LANES(L_, MX_)                                                                \
  k_grad_faces_lanes<L_, MX_><<<g, gb, 0, st>>>(ctx->C, ctx->n, ctx->cptr, ctx->slots,           \
                                                ctx->fnptr, ctx->fnodes, ctx->qn8, ctx->qn4, q,  \
                                                ctx->vol, ctx->dqdx, ctx->dqdy, ctx->dqdz,       \
                                                ctx->P, cases_of(ctx))
    if (L == 4 && mx)
      MFG_GRAD_LANES(4, true);
    else if (L == 4)
      MFG_GRAD_LANES(4, false);
    else if (mx)
      MFG_GRAD_LANES(8, true);
    else
      MFG_GRAD_LANES(8, false);
#undef MFG_GRAD_LANES
    count_launch();
    return;
  }
  if (ctx->precision == MFG_PREC_MIXED)
    k_grad_faces_mx<<<grid_for(ctx->C, gb), gb, 0, st>>>(
        ctx->C, ctx->n, ctx->cptr, ctx->rslots, ctx->sptr32, ctx->fnptr, ctx->fnodes, ctx->qn4,
        ctx->q8[ctx->cur], ctx->vol, ctx->dqdx, ctx->dqdy, ctx->dqdz, ctx->P, cases_of(ctx));
  else
    k_grad_faces<<<grid_for(ctx->C, gb), gb, 0, st>>>(
        ctx->C, ctx->n, ctx->cptr, ctx->rslots, ctx->sptr32, ctx->fnptr, ctx->fnodes, ctx->qn8,
        ctx->q8[ctx->cur], ctx->vol, ctx->dqdx, ctx->dqdy, ctx->dqdz);
  count_launch();
}

static int launch_gradient(mfg_ctx *ctx) {
  launch_node_values(ctx, ctx->stream);
  launch_grad_faces(ctx, ctx->stream);
  return check_kernel();
}

int mfg_calculate_gradient(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  MFG_CUDA(cudaSetDevice(ctx->device));
  return launch_gradient(ctx);
}

// End of a fused iteration: the residual norm into norm_hist[counter] and the
// counter advanced.  One grid reduces the flux gather's block partials; a
// batch reduces each case's cell range.
static int launch_norm_tail(mfg_ctx *ctx, cudaStream_t st) {
  if (ctx->ncase == 1) {
    k_norm_final<<<1, kNormThreads, 0, st>>>(gather_blocks(ctx), ctx->norm_part, ctx->norm_out,
                                    ctx->iter_counter, ctx->norm_hist);
    count_launch();
  } else {
    k_norm_seg_partial<<<dim3(kSegBlocks, ctx->ncase), kBlock, 0, st>>>(
        ctx->C, ctx->res, ctx->case_cell0_d, ctx->seg_part);
    k_norm_seg_final<<<ctx->ncase, 32, 0, st>>>(kSegBlocks, ctx->seg_part, ctx->norm_out,
                                                ctx->iter_counter, ctx->norm_hist);
    k_counter_inc<<<1, 1, 0, st>>>(ctx->iter_counter);
    count_launch(3);
  }
  return check_kernel();
}

// Per-iteration tables of a fused run: CFL [n_iter][ncase] and norms
// [n_iter][ncase][5].  Captured graphs hold their pointers, so growing them
// drops the graphs.
static int ensure_tables(mfg_ctx *ctx, int32_t n_iter) {
  if (n_iter <= ctx->hist_cap) return MFG_OK;
  for (int k = 0; k < 2; k++)
    if (ctx->graph[k]) {
      cudaGraphExecDestroy(ctx->graph[k]);
      ctx->graph[k] = nullptr;
    }
  const int32_t cap = std::max(n_iter, 256);
  int rc;
  if ((rc = dalloc(ctx, &ctx->norm_hist, (size_t)5 * cap * ctx->ncase))) return rc;
  if ((rc = dalloc(ctx, &ctx->cfl_tab, (size_t)cap * ctx->ncase))) return rc;
  ctx->hist_cap = cap;
  return MFG_OK;
}

// CFL of iterations iter_done .. iter_done + n_iter - 1 of every case (each
// case ramps with its own cfl_start/cfl_end/cfl_nstep) into cfl_tab, and the
// fused-loop counter reset.
static int fill_cfl_table(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done) {
  int rc = ensure_tables(ctx, n_iter);
  if (rc) return rc;
  const int32_t K = ctx->ncase;
  std::vector<double> tab((size_t)n_iter * K);
  for (int32_t i = 0; i < n_iter; i++)
    for (int32_t k = 0; k < K; k++) tab[(size_t)i * K + k] = cfl_for(ctx->hps[k], iter_done + i);
  ctx->hp.cfl_min = 0.5 * cfl_for(ctx->hp, iter_done + n_iter - 1);
  for (int32_t k = 0; k < K; k++) ctx->hps[k].cfl_min = 0.5 * tab[(size_t)(n_iter - 1) * K + k];
  // the copy must finish before tab goes out of scope
  MFG_CUDA(cudaMemcpyAsync(ctx->cfl_tab, tab.data(), sizeof(double) * tab.size(),
                           cudaMemcpyHostToDevice, ctx->stream));
  MFG_CUDA(cudaMemsetAsync(ctx->iter_counter, 0, sizeof(int32_t), ctx->stream));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  return MFG_OK;
}

// One fused iteration: flux + dt + Diag in one gather, level sweeps with the
// update, gradient, residual norm.  Reads the CFL from cfl_tab[counter].
// Optional hooks for a caller that copies results out while the iteration
// runs on: `after_face` is recorded once the residual is final (nothing
// later in the iteration writes it), `after_update` once the new state has
// been unpacked into the SoA staging buffer.
//
// Where the iteration's gradient goes (`grad`): GRAD_AT_END after the update,
// as the reference orders it; GRAD_DEFER not in this iteration; GRAD_LEAD
// the gradient of the state the iteration starts from -- the one the
// previous, deferred, iteration owes -- on the side stream beside this
// iteration's face kernels (both only read that state; neither reads what
// the other writes).  A run of n iterations defers the first, leads the
// others and ends with one gradient of the final state (run_iterations):
// every iteration's gradient is computed once, with the same kernels and
// values, the n - 1 inner ones overlapping the next iteration's face phase.
static int ensure_side_stream(mfg_ctx *ctx) {
  if (ctx->side_stream) return MFG_OK;
  MFG_CUDA(cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking));
  MFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  MFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  return MFG_OK;
}

enum : int { GRAD_AT_END = 0, GRAD_DEFER = 1, GRAD_LEAD = 2 };

static int launch_iteration(mfg_ctx *ctx, cudaEvent_t after_face = nullptr,
                            cudaEvent_t after_update = nullptr, int grad = GRAD_AT_END) {
  const bool lead_gradient = grad == GRAD_LEAD;
  if (lead_gradient) {
    MFG_CUDA(cudaEventRecord(ctx->ev_fork, ctx->stream));
    MFG_CUDA(cudaStreamWaitEvent(ctx->side_stream, ctx->ev_fork, 0));
    launch_node_values(ctx, ctx->side_stream);
    launch_grad_faces(ctx, ctx->side_stream);
    MFG_CUDA(cudaGetLastError());
    MFG_CUDA(cudaEventRecord(ctx->ev_join, ctx->side_stream));
  }
  int rc = launch_face(ctx, true, true, true, 0.0, true);
  if (rc) return rc;
  if (after_face) MFG_CUDA(cudaEventRecord(after_face, ctx->stream));
  // the persistent sweeps need every SM: the gradient ends before them
  if (lead_gradient) MFG_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
  rc = launch_sweeps(ctx, true);
  if (rc) return rc;
  ctx->cur ^= 1;
  if (ctx->live_bc) {
    // main.cpp:286 with its SetGhostVariables call enabled
    rc = launch_ghost_bc(ctx, ctx->stream);
    if (rc) return rc;
  }
  if (after_update) {
    k_download_rec<<<grid_for(ctx->n), kBlock, 0, ctx->stream>>>(ctx->q8[ctx->cur],
                                                                  ctx->staging, ctx->n);
    count_launch();
    MFG_CUDA(cudaGetLastError());
    MFG_CUDA(cudaEventRecord(after_update, ctx->stream));
  }
  if (grad == GRAD_AT_END) {
    rc = launch_gradient(ctx);
    if (rc) return rc;
  }
  return launch_norm_tail(ctx, ctx->stream);
}

static int ensure_graphs(mfg_ctx *ctx) {
  if (ctx->graph[0] && ctx->graph[1]) return MFG_OK;
  int rc0 = ensure_side_stream(ctx);
  if (rc0) return rc0;
  const int start = ctx->cur;
  for (int k = 0; k < 2; k++) {
    const int par = start ^ k;
    ctx->cur = par;
    ctx->res_zero = true;  // each captured iteration starts with ZeroResiduals
    cudaGraph_t g = nullptr;
    MFG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = g_launches.load();
    // second order: the flux reads the gradient of the state it starts
    // from, so each iteration keeps its gradient at its end
    int rc = launch_iteration(ctx, nullptr, nullptr, ctx->order >= 2 ? GRAD_AT_END : GRAD_LEAD);
    const long long nodes = g_launches.load() - before;
    g_launches.fetch_sub(nodes);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      ctx->cur = start;
      return rc;
    }
    if (e != cudaSuccess) {
      g_cuda_error = std::string("capture: ") + cudaGetErrorString(e);
      ctx->cur = start;
      return MFG_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&ctx->graph[par], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      g_cuda_error = std::string("instantiate: ") + cudaGetErrorString(e);
      ctx->cur = start;
      return MFG_ERR_CUDA;
    }
    ctx->graph_nodes = nodes;
  }
  ctx->cur = start;
  return MFG_OK;
}

// n_iter >= 1 fused iterations after fill_cfl_table: the first launched
// plainly with its gradient deferred, the inner ones as captured graphs that
// lead with the previous iteration's gradient, the last one plainly when it
// carries the copy hooks, then the gradient of the final state.
static int run_iterations(mfg_ctx *ctx, int32_t n_iter, cudaEvent_t after_face = nullptr,
                          cudaEvent_t after_update = nullptr) {
  cudaStream_t st = ctx->stream;
  const bool hooks = after_face || after_update;
  const int32_t n_graph = n_iter - 1 - ((hooks && n_iter > 1) ? 1 : 0);
  int rc;
  if ((rc = ensure_side_stream(ctx))) return rc;
  if (n_graph > 0 && (rc = ensure_graphs(ctx))) return rc;
  ctx->res_zero = true;  // ZeroResiduals at the top of each iteration
  const bool second = ctx->order >= 2;
  rc = launch_iteration(ctx, n_iter == 1 ? after_face : nullptr,
                        n_iter == 1 ? after_update : nullptr, second ? GRAD_AT_END : GRAD_DEFER);
  for (int32_t i = 0; rc == MFG_OK && i < n_graph; i++) {
    const cudaError_t e = cudaGraphLaunch(ctx->graph[ctx->cur], st);
    if (e != cudaSuccess) {
      g_cuda_error = std::string("cudaGraphLaunch: ") + cudaGetErrorString(e);
      rc = MFG_ERR_CUDA;
      break;
    }
    count_launch(ctx->graph_nodes);
    ctx->cur ^= 1;
  }
  if (rc == MFG_OK && hooks && n_iter > 1) {
    ctx->res_zero = true;
    rc = launch_iteration(ctx, after_face, after_update, second ? GRAD_AT_END : GRAD_LEAD);
  }
  if (rc == MFG_OK && !second) rc = launch_gradient(ctx);  // of the final state
  ctx->res_zero = false;
  return rc;
}

int mfg_iterate(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done, double *norms) {
  if (!ctx || n_iter < 0) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  if (n_iter == 0) return MFG_OK;
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  int rc = fill_cfl_table(ctx, n_iter, iter_done);
  if (rc) return rc;
  if ((rc = run_iterations(ctx, n_iter))) {
    cudaStreamSynchronize(st);
    return rc;
  }
  if (norms) {
    MFG_CUDA(cudaMemcpyAsync(norms, ctx->norm_hist, sizeof(double) * 5 * n_iter * ctx->ncase,
                             cudaMemcpyDeviceToHost, st));
    MFG_CUDA(cudaStreamSynchronize(st));
  }
  MFG_CUDA(cudaGetLastError());
  return check_sweep_error(ctx);
}

}  // extern "C"

// Rebuild the persistent sweeps' chunk tables of a context with another
// kernel kind and chunk assignment (-1: the model's), for mfg_autotune's
// trials: the level order and records of both sweeps stay on the device;
// the assignment is chosen on the host from them and the cell centroids,
// then packed on the device as at creation.
static int rechunk(mfg_ctx *ctx, int kind, int chunking) {
  if (!ctx->sweep_w || !ctx->fw_cells || !ctx->bw_cells || ctx->halo) return MFG_ERR_UNSUPPORTED;
  cudaStream_t st = ctx->stream;
  const int32_t C = ctx->C, W = ctx->sweep_w;
  int rc;
  std::vector<Cen> cc;
  if ((rc = d2h(cc, ctx->ccen, C, st))) return rc;
  DevSweep d[2];
  d[0].fwd = true;
  d[1].fwd = false;
  for (int k = 0; k < 2; k++) {
    d[k].lptr = k ? ctx->bw_lptr : ctx->fw_lptr;
    if ((rc = d2h(d[k].h_cells, (const int32_t *)(k ? ctx->bw_cells : ctx->fw_cells), C, st)) ||
        (rc = d2h(d[k].h_sptr, (const int32_t *)(k ? ctx->bw_sptr : ctx->fw_sptr), (int64_t)C + 1,
                  st)))
      return rc;
  }
  MFG_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < 2; k++)
    if ((rc = d2h(d[k].h_nbs, (const int32_t *)(k ? ctx->bw_nb : ctx->fw_nb), d[k].h_sptr[C], st)))
      return rc;
  MFG_CUDA(cudaStreamSynchronize(st));
  std::vector<double> xyz3[3];
  for (int a = 0; a < 3; a++) xyz3[a].resize(C);
  for (int32_t c = 0; c < C; c++) {
    xyz3[0][c] = cc[c].x;
    xyz3[1][c] = cc[c].y;
    xyz3[2][c] = cc[c].z;
  }
  const double *xyz[3] = {xyz3[0].data(), xyz3[1].data(), xyz3[2].data()};
  const int old_kind = ctx->sweep_kind;
  const int32_t old_chunks = ctx->nchunks;
  setup_sweep_grid(ctx, W, kind);
  if (ctx->persist_grid <= 0 || ctx->sweep_kind != kind) {
    setup_sweep_grid(ctx, W, old_kind);
    return MFG_ERR_UNSUPPORTED;
  }
  const int32_t P = ctx->nchunks, G = sweep_groups(W, ctx->sweep_kind);
  for (int k = 0; k < 2; k++) {
    const int ch = choose_chunks(C, P, G, d[k].lptr, d[k].h_cells.data(), d[k].h_sptr.data(),
                                 d[k].h_nbs.data(), xyz, chunking, d[k].h_assign,
                                 &ctx->chunk_est_us[k]);
    if (k == 0) ctx->chunking = ch;
  }
  // the previous tables go; the new ones are packed as at creation
  auto dfree = [&](void *ptr, size_t bytes) {
    if (!ptr) return;
    auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), ptr);
    if (it != ctx->allocs.end()) {
      ctx->allocs.erase(it);
      ctx->device_bytes -= (int64_t)std::max<size_t>(bytes, 1);
    }
    cudaFree(ptr);
  };
  MFG_CUDA(cudaStreamSynchronize(st));
  for (ChunkSweep *cs : {&ctx->fwc, &ctx->bwc}) {
    const size_t nrec = (size_t)C * W;
    dfree(cs->seg_begin, sizeof(int32_t) * ((size_t)old_chunks + 1));
    dfree(cs->segs, sizeof(int32_t) * ((size_t)cs->nseg + 1));
    dfree(cs->cells, sizeof(PosCell) * C);
    dfree(cs->nbs, sizeof(int32_t) * nrec);
    dfree(cs->nslots, sizeof(int32_t) * nrec);
    dfree(cs->recs, sizeof(SweepRec) * nrec);
    dfree(cs->recs_f, sizeof(SweepRecF) * nrec);
    *cs = ChunkSweep{};
  }
  DevScratch sc;
  for (int k = 0; k < 2; k++) {
    std::vector<int32_t> lv(C, 0);
    for (size_t l = 0; l + 1 < d[k].lptr.size(); l++)
      for (int32_t i = d[k].lptr[l]; i < d[k].lptr[l + 1]; i++) lv[d[k].h_cells[i]] = (int32_t)l;
    if ((rc = sc.get(&d[k].lvl, C))) return rc;
    MFG_CUDA(cudaMemcpyAsync(d[k].lvl, lv.data(), sizeof(int32_t) * C, cudaMemcpyHostToDevice, st));
    for (int a = 0; a < 2; a++) ctx->sweep_stats[k][a] = 0;
    ctx->sweep_stats[k][2] = 0;
    if ((rc = dev_pack(ctx, sc, d[k]))) return rc;
  }
  MFG_CUDA(cudaStreamSynchronize(st));
  drop_graphs(ctx);
  return MFG_OK;
}

extern "C" {

int mfg_autotune(mfg_ctx *ctx, int32_t n_trial, int32_t iter_done, int32_t flags,
                 mfg_tune_report *rep) {
  if (!ctx || n_trial <= 0) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const size_t qbytes = sizeof(double) * ctx->n * Q_STRIDE;
  const size_t q4bytes = sizeof(float) * ctx->n * Q_STRIDE;
  // every trial leaves the state as it was: the current records and the
  // running dt extrema are saved once and restored after each
  void *save = nullptr;
  if (cudaMalloc(&save, qbytes + (mx ? q4bytes : 0)) != cudaSuccess) {
    g_cuda_error = "cudaMalloc: autotune scratch";
    return MFG_ERR_NOMEM;
  }
  std::vector<unsigned long long> ext(2 * ctx->ncase);
  cudaMemcpyAsync(save, ctx->q8[ctx->cur], qbytes, cudaMemcpyDeviceToDevice, st);
  if (mx)
    cudaMemcpyAsync((char *)save + qbytes, ctx->q4[ctx->cur], q4bytes, cudaMemcpyDeviceToDevice,
                    st);
  cudaMemcpyAsync(ext.data(), ctx->dt_ext, sizeof(unsigned long long) * ext.size(),
                  cudaMemcpyDeviceToHost, st);
  const int cur0 = ctx->cur;
  const bool res_zero0 = ctx->res_zero;
  int rc = cudaStreamSynchronize(st) == cudaSuccess ? MFG_OK : MFG_ERR_CUDA;
  auto restore = [&]() {
    ctx->cur = cur0;
    cudaMemcpyAsync(ctx->q8[ctx->cur], save, qbytes, cudaMemcpyDeviceToDevice, st);
    if (mx)
      cudaMemcpyAsync(ctx->q4[ctx->cur], (char *)save + qbytes, q4bytes, cudaMemcpyDeviceToDevice,
                      st);
    cudaMemcpyAsync(ctx->dt_ext, ext.data(), sizeof(unsigned long long) * ext.size(),
                    cudaMemcpyHostToDevice, st);
    return cudaStreamSynchronize(st) == cudaSuccess ? MFG_OK : MFG_ERR_CUDA;
  };
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rc == MFG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    rc = MFG_ERR_CUDA;
  // ms per fused iteration of the context as it stands (-1: it cannot run)
  auto trial = [&]() -> double {
    if (mfg_iterate(ctx, 2, iter_done, nullptr) != MFG_OK) {  // builds the graphs
      restore();
      return -1.0;
    }
    cudaEventRecord(e0, st);
    const int r = mfg_iterate(ctx, n_trial, iter_done + 2, nullptr);
    cudaEventRecord(e1, st);
    float t = 0.f;
    const bool ok = r == MFG_OK && cudaEventSynchronize(e1) == cudaSuccess &&
                    cudaEventElapsedTime(&t, e0, e1) == cudaSuccess;
    if (restore() != MFG_OK) return -1.0;
    return ok ? (double)t / n_trial : -1.0;
  };
  mfg_tune_report local{};
  mfg_tune_report &R = rep ? *rep : local;
  R = mfg_tune_report{};
  if (rc == MFG_OK) R.ms_initial = trial();
  // knob k: candidates, how to apply one, how to read the current value
  struct Knob {
    int id;
    std::vector<int> cand;
  };
  std::vector<Knob> knobs;
  if (ctx->sweep_w && ctx->sweep_mode == 1 && !(flags & MFG_TUNE_NO_REBUILD)) {
    knobs.push_back({MFG_KNOB_SWEEP_KERNEL, {MFG_SWEEP_DEEP, MFG_SWEEP_WIDE}});
    knobs.push_back({MFG_KNOB_CHUNKING, {MFG_CHUNK_VOTE, MFG_CHUNK_TRANSVERSE_ANY}});
  }
  if (ctx->sweep_w) knobs.push_back({MFG_KNOB_SWEEP_MODE, {1, 0}});
  knobs.push_back({MFG_KNOB_GATHER_BLOCKS, {3, 2, 4}});
  knobs.push_back({MFG_KNOB_FLUX_BLOCKS, {3, 2, 4}});
  knobs.push_back({MFG_KNOB_NODE_BLOCK, {512, 256, 128}});
  knobs.push_back({MFG_KNOB_GRAD_BLOCK, {128, 64, 256}});
  if (ctx->gather_lanes_fit) knobs.push_back({MFG_KNOB_GATHER_LANES, {0, ctx->gather_lanes_fit}});
  auto current = [&](int id) {
    switch (id) {
      case MFG_KNOB_SWEEP_KERNEL: return ctx->sweep_kind;
      case MFG_KNOB_CHUNKING:  // the transverse candidate stands for any axis pair
        return ctx->chunking == MFG_CHUNK_VOTE ? MFG_CHUNK_VOTE : MFG_CHUNK_TRANSVERSE_ANY;
      case MFG_KNOB_SWEEP_MODE: return ctx->sweep_mode;
      case MFG_KNOB_GATHER_BLOCKS: return ctx->gather_minb;
      case MFG_KNOB_FLUX_BLOCKS: return ctx->flux_minb;
      case MFG_KNOB_NODE_BLOCK: return ctx->node_block;
      case MFG_KNOB_GATHER_LANES: return ctx->gather_lanes;
      default: return ctx->grad_block;
    }
  };
  auto apply = [&](int id, int v) -> int {
    switch (id) {
      case MFG_KNOB_SWEEP_KERNEL:
        return v == ctx->sweep_kind ? MFG_OK : rechunk(ctx, v, -1);
      case MFG_KNOB_CHUNKING:
        return v == current(MFG_KNOB_CHUNKING) ? MFG_OK : rechunk(ctx, ctx->sweep_kind, v);
      case MFG_KNOB_SWEEP_MODE: return mfg_set_sweep_mode(ctx, v);
      case MFG_KNOB_GATHER_BLOCKS: ctx->gather_minb = v; break;
      case MFG_KNOB_FLUX_BLOCKS: ctx->flux_minb = v; break;
      case MFG_KNOB_NODE_BLOCK: ctx->node_block = v; break;
      case MFG_KNOB_GATHER_LANES: ctx->gather_lanes = v; break;
      default: ctx->grad_block = v; break;
    }
    drop_graphs(ctx);
    return MFG_OK;
  };
  for (size_t k = 0; k < knobs.size() && k < MFG_TUNE_KNOBS && rc == MFG_OK; k++) {
    const Knob &kb = knobs[k];
    R.knob[k] = kb.id;
    const int v0 = current(kb.id);
    int best = v0;
    double tbest = 1e300;
    R.n_cand[k] = (int32_t)std::min<size_t>(kb.cand.size(), MFG_TUNE_CANDS);
    for (int i = 0; i < R.n_cand[k]; i++) {
      const int v = kb.cand[i];
      R.cand[k][i] = v;
      R.ms[k][i] = -1.0;
      if (apply(kb.id, v) != MFG_OK) continue;
      // a rebuild may settle on another value than asked (a kind without a
      // grid): the trial is recorded under the value asked only when taken
      if (current(kb.id) != v) continue;
      R.ms[k][i] = trial();
      if (R.ms[k][i] > 0.0 && R.ms[k][i] < tbest) {
        tbest = R.ms[k][i];
        best = v;
      }
    }
    if (apply(kb.id, best) != MFG_OK) rc = MFG_ERR_CUDA;
    R.chosen[k] = current(kb.id);
    R.n_knobs = (int32_t)k + 1;
  }
  if (rc == MFG_OK) R.ms_final = trial();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(save);
  ctx->res_zero = res_zero0;
  drop_graphs(ctx);
  return rc;
}

int mfg_autotune_sweeps(mfg_ctx *ctx, int32_t n_trial, int32_t iter_done, double *ms_out) {
  if (!ctx || n_trial <= 0) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  if (ctx->sweep_mode != 1 || !ctx->sweep_w) return MFG_ERR_UNSUPPORTED;
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const bool mx = ctx->precision == MFG_PREC_MIXED;
  const size_t qbytes = sizeof(double) * ctx->n * Q_STRIDE;
  const size_t q4bytes = sizeof(float) * ctx->n * Q_STRIDE;
  // the trial iterations must leave the state as it was: save the current
  // records and the running dt extrema
  void *save = nullptr;
  if (cudaMalloc(&save, qbytes + (mx ? q4bytes : 0)) != cudaSuccess) {
    g_cuda_error = "cudaMalloc: autotune scratch";
    return MFG_ERR_NOMEM;
  }
  std::vector<unsigned long long> ext(2 * ctx->ncase);
  int rc = MFG_OK;
  auto save_state = [&]() {
    cudaMemcpyAsync(save, ctx->q8[ctx->cur], qbytes, cudaMemcpyDeviceToDevice, st);
    if (mx)
      cudaMemcpyAsync((char *)save + qbytes, ctx->q4[ctx->cur], q4bytes, cudaMemcpyDeviceToDevice,
                      st);
    cudaMemcpyAsync(ext.data(), ctx->dt_ext, sizeof(unsigned long long) * ext.size(),
                    cudaMemcpyDeviceToHost, st);
    return cudaStreamSynchronize(st) == cudaSuccess ? MFG_OK : MFG_ERR_CUDA;
  };
  auto restore_state = [&]() {
    cudaMemcpyAsync(ctx->q8[ctx->cur], save, qbytes, cudaMemcpyDeviceToDevice, st);
    if (mx)
      cudaMemcpyAsync(ctx->q4[ctx->cur], (char *)save + qbytes, q4bytes, cudaMemcpyDeviceToDevice,
                      st);
    cudaMemcpyAsync(ctx->dt_ext, ext.data(), sizeof(unsigned long long) * ext.size(),
                    cudaMemcpyHostToDevice, st);
    return cudaStreamSynchronize(st) == cudaSuccess ? MFG_OK : MFG_ERR_CUDA;
  };
  const bool res_zero0 = ctx->res_zero;
  rc = save_state();
  const int cand[2] = {ctx->sweep_w, ctx->sweep_w / 2};
  double ms[2] = {0.0, 0.0};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rc == MFG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    rc = MFG_ERR_CUDA;
  double ms_best = 1e300;
  int best = ctx->sweep_lanes;
  for (int k = 0; k < 2 && rc == MFG_OK; k++) {
    ms[k] = -1.0;  // not usable with this context's kernels
    if (cand[k] != ctx->sweep_w) continue;
    if ((rc = mfg_set_sweep_lanes(ctx, cand[k]))) break;
    if ((rc = mfg_iterate(ctx, 2, iter_done, nullptr))) break;  // builds the graphs
    cudaEventRecord(e0, st);
    if ((rc = mfg_iterate(ctx, n_trial, iter_done + 2, nullptr))) break;
    cudaEventRecord(e1, st);
    float t = 0.f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
      rc = MFG_ERR_CUDA;
    ms[k] = (double)t / n_trial;
    if (ms[k] < ms_best) {
      ms_best = ms[k];
      best = cand[k];
    }
    if (rc == MFG_OK) rc = restore_state();
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(save);
  ctx->res_zero = res_zero0;
  if (rc) return rc;
  if (ms_out) {
    ms_out[0] = ms[0];
    ms_out[1] = ms[1];
  }
  return mfg_set_sweep_lanes(ctx, best);
}

int mfg_profile_phases(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done, double *phase_ms) {
  if (!ctx || n_iter <= 0 || !phase_ms) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  {
    int rc = fill_cfl_table(ctx, n_iter, iter_done);
    if (rc) return rc;
  }
  cudaEvent_t ev[MFG_NPHASES + 1];
  for (auto &e : ev) MFG_CUDA(cudaEventCreate(&e));
  for (int k = 0; k < MFG_NPHASES; k++) phase_ms[k] = 0.0;
  int rc = MFG_OK;
  for (int32_t it = 0; it < n_iter && rc == MFG_OK; it++) {
    ctx->res_zero = true;
    cudaEventRecord(ev[0], st);
    rc = launch_face(ctx, true, true, true, 0.0, true);
    cudaEventRecord(ev[1], st);
    if (ctx->sweep_mode == 1) {
      if (rc == MFG_OK) rc = launch_fwd_persist(ctx, true, 0, kSpinCycles);
      cudaEventRecord(ev[2], st);
      if (rc == MFG_OK) rc = launch_bwd_persist(ctx, kSpinCycles);
    } else if (rc == MFG_OK) {
      launch_level_sweep(ctx, true, true, st);
      cudaEventRecord(ev[2], st);
      launch_level_sweep(ctx, false, true, st);
    } else {
      cudaEventRecord(ev[2], st);
    }
    ctx->cur ^= 1;
    if (ctx->live_bc && rc == MFG_OK) rc = launch_ghost_bc(ctx, st);  // with the update
    cudaEventRecord(ev[3], st);
    launch_node_values(ctx, st);
    cudaEventRecord(ev[4], st);
    launch_grad_faces(ctx, st);
    cudaEventRecord(ev[5], st);
    const int rn = launch_norm_tail(ctx, st);
    cudaEventRecord(ev[6], st);
    if (rc == MFG_OK) rc = rn;
    if (rc == MFG_OK) rc = check_kernel();
    if (cudaEventSynchronize(ev[6]) != cudaSuccess) rc = MFG_ERR_CUDA;
    for (int k = 0; k < MFG_NPHASES && rc == MFG_OK; k++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      phase_ms[k] += ms;
    }
  }
  ctx->res_zero = false;
  for (auto &e : ev) cudaEventDestroy(e);
  if (rc) return rc;
  return check_sweep_error(ctx);
}

// The state and the residual of the last iteration leave on a second stream
// as soon as each is final: the residual (written only by the face gather)
// during the sweeps, the state during the gradient.  The first n_iter - 1
// iterations run as graphs, the last one as plain launches with two event
// hooks (the same kernels in the same order as the graph).
int mfg_iterate_host(mfg_ctx *ctx, int32_t n_iter, int32_t iter_done, const double *q_in,
                     double *q_out, double *res_out, double *norms) {
  if (!ctx || n_iter < 0) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_UNSUPPORTED;  // a part iterates through mfg_halo_phase
  int rc;
  if (q_in && (rc = mfg_upload(ctx, MFG_FIELD_Q, q_in))) return rc;
  if (n_iter == 0 || (!q_out && !res_out)) {
    if ((rc = mfg_iterate(ctx, n_iter, iter_done, norms))) return rc;
    if (q_out && (rc = mfg_download(ctx, MFG_FIELD_Q, q_out))) return rc;
    if (res_out && (rc = mfg_download(ctx, MFG_FIELD_RES, res_out))) return rc;
    return MFG_OK;
  }
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (!ctx->copy_stream) {
    MFG_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    MFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_res, cudaEventDisableTiming));
    MFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_state, cudaEventDisableTiming));
  }
  if ((rc = fill_cfl_table(ctx, n_iter, iter_done))) return rc;
  rc = run_iterations(ctx, n_iter, res_out ? ctx->ev_res : nullptr,
                      q_out ? ctx->ev_state : nullptr);
  if (rc) {
    cudaStreamSynchronize(st);
    return rc;
  }
  cudaStream_t cp = ctx->copy_stream;
  if (res_out) {
    MFG_CUDA(cudaStreamWaitEvent(cp, ctx->ev_res, 0));
    MFG_CUDA(cudaMemcpyAsync(res_out, ctx->res, sizeof(double) * 5 * ctx->C,
                             cudaMemcpyDeviceToHost, cp));
  }
  if (q_out) {
    MFG_CUDA(cudaStreamWaitEvent(cp, ctx->ev_state, 0));
    MFG_CUDA(cudaMemcpyAsync(q_out, ctx->staging, sizeof(double) * 5 * ctx->n,
                             cudaMemcpyDeviceToHost, cp));
  }
  if (norms)
    MFG_CUDA(cudaMemcpyAsync(norms, ctx->norm_hist, sizeof(double) * 5 * n_iter * ctx->ncase,
                             cudaMemcpyDeviceToHost, st));
  MFG_CUDA(cudaStreamSynchronize(st));
  MFG_CUDA(cudaStreamSynchronize(cp));
  return check_sweep_error(ctx);
}

int mfg_residual_norm(mfg_ctx *ctx, double out[5]) {
  if (!ctx || !out) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (ctx->res_zero) {
    for (int k = 0; k < 5; k++) out[k] = 0.0;
    return MFG_OK;
  }
  k_norm_partial<<<kNormBlocks, kBlock, 0, st>>>(ctx->C, ctx->res, ctx->norm_part);
  k_norm_final<<<1, kNormThreads, 0, st>>>(kNormBlocks, ctx->norm_part, ctx->norm_out, nullptr, nullptr);
  count_launch(2);
  MFG_CUDA(cudaGetLastError());
  MFG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->norm_out, 5 * sizeof(double),
                           cudaMemcpyDeviceToHost, st));
  MFG_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < 5; k++) out[k] = ctx->h_pinned[k];
  return MFG_OK;
}

int mfg_batch_residual_norm(mfg_ctx *ctx, double *out) {
  if (!ctx || !out) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  if (ctx->ncase == 1) return mfg_residual_norm(ctx, out);
  cudaStream_t st = ctx->stream;
  const size_t nb = sizeof(double) * 5 * ctx->ncase;
  if (ctx->res_zero) {
    std::memset(out, 0, nb);
    return MFG_OK;
  }
  k_norm_seg_partial<<<dim3(kSegBlocks, ctx->ncase), kBlock, 0, st>>>(
      ctx->C, ctx->res, ctx->case_cell0_d, ctx->seg_part);
  k_norm_seg_final<<<ctx->ncase, 32, 0, st>>>(kSegBlocks, ctx->seg_part, ctx->norm_out, nullptr,
                                              nullptr);
  count_launch(2);
  MFG_CUDA(cudaGetLastError());
  MFG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->norm_out, nb, cudaMemcpyDeviceToHost, st));
  MFG_CUDA(cudaStreamSynchronize(st));
  std::memcpy(out, ctx->h_pinned, nb);
  return MFG_OK;
}

int mfg_get_dt_extrema(mfg_ctx *ctx, double *dt_max, double *dt_min) {
  if (!ctx || !dt_max || !dt_min) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  MFG_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->dt_ext, 2 * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  *dt_max = ctx->h_pinned[0];
  *dt_min = ctx->h_pinned[1];
  return MFG_OK;
}

int mfg_set_dt_extrema(mfg_ctx *ctx, double dt_max, double dt_min) {
  if (!ctx || !(dt_max >= 0.0) || !(dt_min >= 0.0)) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int32_t k = 0; k < ctx->ncase; k++) {
    ctx->h_pinned[2 * k] = dt_max;
    ctx->h_pinned[2 * k + 1] = dt_min;
  }
  MFG_CUDA(cudaMemcpyAsync(ctx->dt_ext, ctx->h_pinned, 2 * sizeof(double) * ctx->ncase,
                           cudaMemcpyHostToDevice, ctx->stream));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  return MFG_OK;
}

int mfg_sync(mfg_ctx *ctx) {
  if (!ctx) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  MFG_CUDA(cudaStreamSynchronize(ctx->stream));
  return MFG_OK;
}

int mfg_download(mfg_ctx *ctx, int32_t field, double *host) {
  if (!ctx || !host) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n, C = ctx->C;
  const double *src = nullptr;
  size_t count = 0;
  switch (field) {
    case MFG_FIELD_Q:
    case MFG_FIELD_DQ: {
      const double *rec = field == MFG_FIELD_Q ? ctx->q8[ctx->cur] : ctx->dq8;
      k_download_rec<<<grid_for(n), kBlock, 0, st>>>(rec, ctx->staging, n);
      count_launch();
      MFG_CUDA(cudaGetLastError());
      src = ctx->staging;
      count = 5 * n;
      break;
    }
    case MFG_FIELD_RES:
      if (ctx->res_zero) MFG_CUDA(cudaMemsetAsync(ctx->res, 0, sizeof(double) * 5 * C, st));
      src = ctx->res;
      count = 5 * C;
      break;
    case MFG_FIELD_DT: src = ctx->dt; count = C; break;
    case MFG_FIELD_DIAG: src = ctx->diag; count = C; break;
    case MFG_FIELD_LIMITER:  // [5][n] on the device: the cells' rows
      if (!ctx->phi) return MFG_ERR_INVALID;
      for (int v = 0; v < 5; v++)
        MFG_CUDA(cudaMemcpyAsync(host + (int64_t)v * C, ctx->phi + (int64_t)v * n,
                                 sizeof(double) * C, cudaMemcpyDeviceToHost, st));
      MFG_CUDA(cudaStreamSynchronize(st));
      return MFG_OK;
    case MFG_FIELD_DQDX: src = ctx->dqdx; count = 5 * n; break;
    case MFG_FIELD_DQDY: src = ctx->dqdy; count = 5 * n; break;
    case MFG_FIELD_DQDZ: src = ctx->dqdz; count = 5 * n; break;
    default: return MFG_ERR_INVALID;
  }
  MFG_CUDA(cudaMemcpyAsync(host, src, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
  MFG_CUDA(cudaStreamSynchronize(st));
  return MFG_OK;
}

int mfg_upload(mfg_ctx *ctx, int32_t field, const double *host) {
  if (!ctx || !host) return MFG_ERR_INVALID;
  if (field != MFG_FIELD_Q) return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  MFG_CUDA(cudaMemcpyAsync(ctx->staging, host, sizeof(double) * 5 * n, cudaMemcpyHostToDevice,
                           st));
  k_upload_q<<<grid_for(n), kBlock, 0, st>>>(ctx->staging, ctx->q8[ctx->cur],
                                            ctx->q8[ctx->cur ^ 1], ctx->q4[ctx->cur],
                                            ctx->q4[ctx->cur ^ 1], n, ctx->P, cases_of(ctx));
  count_launch();
  MFG_CUDA(cudaGetLastError());
  // second order: the next flux reads the gradient of the uploaded state
  return ctx->order >= 2 ? launch_gradient(ctx) : MFG_OK;
}


// ---------------------------------------------------------------------------
// one part of a partitioned mesh: the reference's MPI mode in phases, the
// exchanges between them left to the caller
// ---------------------------------------------------------------------------

int mfg_halo_set(mfg_ctx *ctx, const mfg_halo *h) {
  if (!ctx || !h) return MFG_ERR_INVALID;
  if (ctx->halo) return MFG_ERR_INVALID;  // once per context
  if (ctx->ncase != 1) return MFG_ERR_UNSUPPORTED;
  if (ctx->order != 1 && h->n_send + h->n_recv > 0 && (!h->grad_send || !h->grad_recv))
    return MFG_ERR_UNSUPPORTED;  // second order needs the gradient rows' buffers
  if (h->n_send < 0 || h->n_recv < 0 || h->n_node < 0 || !h->ext || !h->norm_sq)
    return MFG_ERR_INVALID;
  if ((h->n_send && (!h->send_cells || !h->send_rows)) ||
      (h->n_recv && (!h->recv_bfaces || !h->recv_rows)) ||
      (h->n_node && (!h->nodes || !h->node_send || !h->node_recv)))
    return MFG_ERR_INVALID;
  MFG_CUDA(cudaSetDevice(ctx->device));
  for (int32_t i = 0; i < h->n_send; i++)
    if (h->send_cells[i] < 0 || h->send_cells[i] >= ctx->C) return MFG_ERR_INVALID;
  for (int32_t i = 0; i < h->n_node; i++)
    if (h->nodes[i] < 0 || h->nodes[i] >= ctx->N) return MFG_ERR_INVALID;
  std::vector<int32_t> bct(std::max(ctx->G, 1));
  if (ctx->G)
    MFG_CUDA(cudaMemcpy(bct.data(), ctx->bctype_d, sizeof(int32_t) * ctx->G,
                        cudaMemcpyDeviceToHost));
  std::vector<int32_t> recv(h->n_recv);
  for (int32_t i = 0; i < h->n_recv; i++) {
    const int32_t k = h->recv_bfaces[i];
    if (k < 0 || k >= ctx->G || bct[k] != MFG_BC_INTERFACE) return MFG_ERR_INVALID;
    recv[i] = ctx->C + k;
  }
  // the entries of each shared node, in entry order
  std::vector<int32_t> order(h->n_node);
  for (int32_t i = 0; i < h->n_node; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t a, int32_t b) { return h->nodes[a] < h->nodes[b]; });
  std::vector<int32_t> unodes, eptr(1, 0), eidx;
  for (int32_t j = 0; j < h->n_node; j++) {
    const int32_t e = order[j];
    if (unodes.empty() || unodes.back() != h->nodes[e]) {
      if (!unodes.empty()) eptr.push_back((int32_t)eidx.size());
      unodes.push_back(h->nodes[e]);
    }
    eidx.push_back(e);
  }
  if (!unodes.empty()) eptr.push_back((int32_t)eidx.size());
  int rc;
  std::vector<int32_t> send(h->send_cells, h->send_cells + h->n_send),
      nodes(h->nodes, h->nodes + h->n_node);
  if ((rc = dupload(ctx, &ctx->h_send, send))) return rc;
  if ((rc = dupload(ctx, &ctx->h_recv, recv))) return rc;
  if ((rc = dupload(ctx, &ctx->h_nodes, nodes))) return rc;
  if ((rc = dupload(ctx, &ctx->h_unodes, unodes))) return rc;
  if ((rc = dupload(ctx, &ctx->h_eptr, eptr))) return rc;
  if ((rc = dupload(ctx, &ctx->h_eidx, eidx))) return rc;
  std::vector<int32_t> gflag(std::max(ctx->G, 1), 0);
  for (int32_t i = 0; i < h->n_recv; i++) gflag[h->recv_bfaces[i]] = 1;
  if ((rc = dupload(ctx, &ctx->h_gflag, gflag))) return rc;
  // shared nodes keep their partial sums in k_node_values (info bit 4)
  std::vector<int32_t> info(ctx->N);
  MFG_CUDA(cudaMemcpy(info.data(), ctx->ninfo, sizeof(int32_t) * ctx->N, cudaMemcpyDeviceToHost));
  for (int32_t nd : unodes) info[nd] |= 4;
  MFG_CUDA(cudaMemcpy(ctx->ninfo, info.data(), sizeof(int32_t) * ctx->N, cudaMemcpyHostToDevice));
  ctx->h_nu = (int32_t)unodes.size();
  ctx->hb = *h;
  ctx->hb.send_cells = ctx->hb.recv_bfaces = ctx->hb.nodes = nullptr;  // not kept
  ctx->halo = true;
  drop_graphs(ctx);
  return MFG_OK;
}

static void halo_gather(mfg_ctx *ctx, int32_t n, int32_t width, const int32_t *idx,
                        const double *src, double *dst) {
  if (n == 0) return;
  k_halo_gather<<<grid_for((int64_t)n * Q_STRIDE), kBlock, 0, ctx->stream>>>(n, width, idx, src,
                                                                             dst);
  count_launch();
}

static void halo_scatter(mfg_ctx *ctx, int32_t n, int32_t width, const double *src, double *a,
                         double *b, float *fa = nullptr, float *fb = nullptr) {
  if (n == 0) return;
  k_halo_scatter<<<grid_for((int64_t)n * Q_STRIDE), kBlock, 0, ctx->stream>>>(
      n, width, ctx->h_recv, src, a, b, fa, fb);
  count_launch();
}

int mfg_halo_phase(mfg_ctx *ctx, int32_t phase, int32_t iter_done) {
  if (!ctx) return MFG_ERR_INVALID;
  if (!ctx->halo) return MFG_ERR_UNSUPPORTED;
  MFG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const mfg_halo &h = ctx->hb;
  int rc = MFG_OK;
  switch (phase) {
    case MFG_HALO_PACK_Q:
      halo_gather(ctx, h.n_send, Q_STRIDE, ctx->h_send, ctx->q8[ctx->cur], h.send_rows);
      break;
    case MFG_HALO_LIMIT: {  // second order: the limiter, then the gradient rows out
      if (ctx->order < 2) return MFG_ERR_INVALID;
      if (ctx->order >= 3) {
        const int g = grid_for(ctx->C);
        if (ctx->order == 4)
          k_limiter<true><<<g, kBlock, 0, st>>>(ctx->C, ctx->n, ctx->cptr, ctx->slots,
                                                ctx->q8[ctx->cur], ctx->dqdx, ctx->dqdy,
                                                ctx->dqdz, ctx->fcen, ctx->ccen, ctx->venkat_k,
                                                ctx->phi);
        else
          k_limiter<false><<<g, kBlock, 0, st>>>(ctx->C, ctx->n, ctx->cptr, ctx->slots,
                                                 ctx->q8[ctx->cur], ctx->dqdx, ctx->dqdy,
                                                 ctx->dqdz, ctx->fcen, ctx->ccen, ctx->venkat_k,
                                                 ctx->phi);
        count_launch();
      }
      if (h.n_send) {
        k_halo_pack_grad<<<grid_for(h.n_send), kBlock, 0, st>>>(
            h.n_send, ctx->h_send, ctx->n, ctx->dqdx, ctx->dqdy, ctx->dqdz,
            ctx->order >= 3 ? ctx->phi : nullptr, ctx->ccen, h.grad_send);
        count_launch();
      }
      break;
    }
    case MFG_HALO_FACE: {
      const bool second = ctx->order >= 2;
      if (second && h.n_recv) {  // the neighbours' rows from MFG_HALO_LIMIT
        k_halo_unpack_grad<<<grid_for(h.n_recv), kBlock, 0, st>>>(
            h.n_recv, ctx->h_recv, ctx->n, h.grad_recv, ctx->dqdx, ctx->dqdy, ctx->dqdz,
            ctx->order >= 3 ? ctx->phi : nullptr, ctx->ccen);
        count_launch();
      }
      ctx->res_zero = true;
      rc = launch_face(ctx, true, true, true, cfl_for(ctx->hp, iter_done), false, !second);
      if (rc) return rc;
      k_norm_sums<<<1, kNormThreads, 0, st>>>(gather_blocks(ctx), ctx->norm_part, h.norm_sq);
      count_launch();
      MFG_CUDA(cudaMemcpyAsync(h.ext, ctx->dt_ext, 2 * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                               st));
      break;
    }
    case MFG_HALO_FORWARD:
      MFG_CUDA(cudaMemcpyAsync(ctx->dt_ext, h.ext, 2 * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                               st));
      rc = launch_sweep(ctx, true, true);
      if (rc) return rc;
      halo_gather(ctx, h.n_send, 5, ctx->h_send, ctx->dqf, h.send_rows);
      break;
    case MFG_HALO_BACKWARD:
      halo_scatter(ctx, h.n_recv, 5, h.recv_rows, ctx->dq8, nullptr);
      rc = launch_sweep(ctx, false, false);
      if (rc) return rc;
      ctx->cur ^= 1;
      if (ctx->live_bc && (rc = launch_ghost_bc(ctx, st))) return rc;
      halo_gather(ctx, h.n_send, Q_STRIDE, ctx->h_send, ctx->q8[ctx->cur], h.send_rows);
      break;
    case MFG_HALO_NODES: {
      const bool mx = ctx->precision == MFG_PREC_MIXED;
      halo_scatter(ctx, h.n_recv, Q_STRIDE, h.recv_rows, ctx->q8[0], ctx->q8[1],
                   mx ? ctx->q4[0] : nullptr, mx ? ctx->q4[1] : nullptr);
      launch_node_values(ctx, st);
      if (!h.n_node) break;
      if (mx) {
        k_halo_gather_f<<<grid_for((int64_t)h.n_node * Q_STRIDE), kBlock, 0, st>>>(
            h.n_node, 5, ctx->h_nodes, ctx->qn4, h.node_send);
        count_launch();
      } else {
        halo_gather(ctx, h.n_node, 5, ctx->h_nodes, ctx->qn8, h.node_send);
      }
      break;
    }
    case MFG_HALO_GRADIENT:
      if (ctx->h_nu && ctx->precision == MFG_PREC_MIXED) {
        k_halo_nodes_mx<<<grid_for(ctx->h_nu), kBlock, 0, st>>>(
            ctx->h_nu, ctx->h_unodes, ctx->h_eptr, ctx->h_eidx, h.node_recv, ctx->ninfo,
            ctx->wnode, ctx->nsym, ctx->P, ctx->qn4);
        count_launch();
      } else if (ctx->h_nu) {
        k_halo_nodes<<<grid_for(ctx->h_nu), kBlock, 0, st>>>(
            ctx->h_nu, ctx->h_unodes, ctx->h_eptr, ctx->h_eidx, h.node_recv, ctx->ninfo,
            ctx->wnode, ctx->nsym, ctx->qn8);
        count_launch();
      }
      launch_grad_faces(ctx, st);
      break;
    case MFG_HALO_CHECK:
      MFG_CUDA(cudaStreamSynchronize(st));
      return check_sweep_error(ctx);
    default:
      return MFG_ERR_INVALID;
  }
  return check_kernel();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free residual norm.
//
// For callers that may not allocate device memory themselves: code that
// only holds device pointers (no mfgpu context, whose creation allocates),
// or a host application whose device memory budget is owned by another
// allocator, where an extra cudaMalloc/cudaFree would fail or fragment it.
// The per-block partial sums live in a fixed file-scope device array instead
// of a context buffer.  The array stays resident on every device that loads
// this library until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr int kStaticNormBlocks = MFG_NORM_STATIC_MAX_CELLS / kBlock;
static_assert(MFG_NORM_STATIC_MAX_CELLS % kBlock == 0, "whole blocks");

// One partial (5 doubles) per 256-cell block: 65536 x 5 x 8 B = 2.5 MiB.
__device__ __align__(256) double g_norm_scratch[kStaticNormBlocks * 5];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
// The array's device address as resolved in one CUDA context: a context
// has its own copy of the module, so the address is cached per device
// together with the unique id of the context it was resolved in (the
// driver never reuses a context id within a process).  A device reset or a
// different current context (a caller's own driver-API context) changes the
// id, and the address is resolved again there.
struct ScratchAddr {
  unsigned long long ctx_id = 0;
  double *ptr = nullptr;
};
ScratchAddr g_scratch_dev[kMaxDevices];

// Driver entry points for the current context and its id, fetched through
// the runtime (the library does not link libcuda itself).
using CtxGetCurrentFn = int (*)(void **);
using CtxGetIdFn = int (*)(void *, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Id of the context current on this thread, 0 where none can be had.  With
// no context current yet, the device's primary context is made current
// first (cudaSetDevice on the current device; it allocates nothing).
unsigned long long current_context_id(int dev) {
  if (!g_ctx_get_current || !g_ctx_get_id) {
    void *a = nullptr, *b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qb != cudaDriverEntryPointSuccess)
      return 0;
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(a);
    g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(b);
  }
  void *ctx = nullptr;
  if (g_ctx_get_current(&ctx) != 0) return 0;
  if (!ctx) {
    if (cudaSetDevice(dev) != cudaSuccess || g_ctx_get_current(&ctx) != 0 || !ctx) return 0;
  }
  unsigned long long id = 0;
  return g_ctx_get_id(ctx, &id) == 0 ? id : 0;
}

}  // namespace

extern "C" int mfg_selftest_division(int64_t n, uint64_t seed, int64_t *mismatches) {
  if (n < 0 || !mismatches) return MFG_ERR_INVALID;
  unsigned long long *d = nullptr;
  MFG_CUDA(cudaMalloc(&d, sizeof(unsigned long long)));
  cudaError_t e = cudaMemset(d, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) {
    k_selftest_division<<<4 * 148, kBlock>>>(n, seed, d);
    count_launch();
    e = cudaGetLastError();
  }
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    g_cuda_error = std::string("division self-test: ") + cudaGetErrorString(e);
    return MFG_ERR_CUDA;
  }
  *mismatches = (int64_t)h;
  return MFG_OK;
}

extern "C" int mfg_selftest_division_fast(int64_t n, uint64_t seed, int64_t *counts) {
  if (n < 0 || !counts) return MFG_ERR_INVALID;
  unsigned long long *d = nullptr;
  MFG_CUDA(cudaMalloc(&d, 3 * sizeof(unsigned long long)));
  cudaError_t e = cudaMemset(d, 0, 3 * sizeof(unsigned long long));
  if (e == cudaSuccess) {
    k_selftest_division_fast<<<8 * 148, kBlock>>>(n, seed, d);
    count_launch();
    e = cudaGetLastError();
  }
  unsigned long long h[3] = {0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    g_cuda_error = std::string("division self-test: ") + cudaGetErrorString(e);
    return MFG_ERR_CUDA;
  }
  for (int k = 0; k < 3; k++) counts[k] = (int64_t)h[k];
  return MFG_OK;
}

extern "C" int mfg_selftest_functions(int32_t mode, int32_t n, const double *consts,
                                      const double *in, double *out) {
  if (mode < 0 || mode > 3 || n < 0 || !consts || (n > 0 && (!in || !out)))
    return MFG_ERR_INVALID;
  if (n == 0) return MFG_OK;
  Params P{};
  P.gam = consts[0];
  P.p_bar = consts[1];
  P.gamm1 = P.gam - 1.0;
  P.alf_l = consts[2];
  P.lhs_omga = consts[3];
  P.peff = P.gam * P.p_bar / (P.gam - 1.);  // forward_lusgs.cpp:1295
  P.rho_min = consts[4];
  P.rho_max = consts[5];
  P.p_min = consts[6];
  P.p_max = consts[7];
  const size_t nin = (size_t)n * (mode == 0 ? 14 : (mode == 1 || mode == 3) ? 13 : 10);
  const size_t nout = (size_t)n * 5;
  double *d = nullptr;
  MFG_CUDA(cudaMalloc(&d, sizeof(double) * (nin + nout)));
  cudaError_t e = cudaMemcpy(d, in, sizeof(double) * nin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_selftest_functions<<<grid_for(n), kBlock>>>(mode, n, P, d, d + nin);
    count_launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + nin, sizeof(double) * nout, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    g_cuda_error = std::string("function self-test: ") + cudaGetErrorString(e);
    return MFG_ERR_CUDA;
  }
  return MFG_OK;
}

extern "C" int mfg_residual_norm_static(const double *res, int32_t n_cell, double *norms,
                                        void *stream) {
  if (!res || !norms || n_cell < 0) return MFG_ERR_INVALID;
  if (n_cell > MFG_NORM_STATIC_MAX_CELLS) {
    g_cuda_error = "mfg_residual_norm_static: n_cell " + std::to_string(n_cell) +
                   " exceeds the static scratch limit of " +
                   std::to_string(MFG_NORM_STATIC_MAX_CELLS) + " cells";
    return MFG_ERR_INVALID;
  }
  int dev = 0;
  MFG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return MFG_ERR_INVALID;
  double *scratch = nullptr;
  {
    // Host code cannot use the symbol itself (it names a host-side shadow),
    // so resolve its device address at the first call on a device, with it
    // current, and again only if the current context has changed since.
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    const unsigned long long id = current_context_id(dev);
    if (!id) {
      g_cuda_error = "mfg_residual_norm_static: no CUDA context current on device " +
                     std::to_string(dev);
      return MFG_ERR_CUDA;
    }
    ScratchAddr &a = g_scratch_dev[dev];
    if (!a.ptr || a.ctx_id != id) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_norm_scratch);
      if (e != cudaSuccess) {
        g_cuda_error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return MFG_ERR_CUDA;
      }
      a.ptr = static_cast<double *>(p);
      a.ctx_id = id;
    }
    scratch = a.ptr;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nblocks = grid_for(n_cell);  // <= kStaticNormBlocks by the check above
  // every partial that k_norm_final reads is written first, so nothing in
  // the scratch needs clearing between calls
  k_norm_partial<<<nblocks, kBlock, 0, st>>>(n_cell, res, scratch);
  k_norm_final<<<1, kNormThreads, 0, st>>>(nblocks, scratch, norms, nullptr, nullptr);
  count_launch(2);
  MFG_CUDA(cudaGetLastError());
  return MFG_OK;
}
