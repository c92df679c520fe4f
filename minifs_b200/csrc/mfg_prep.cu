// Mesh preprocessing on the GPU: the same arrays as the host restatements
// in mfg_host.cpp (ComputeMetrics, CalnNPC/CalC2N, ComputeWeight3D_Node,
// FindNodeSYMM), bit for bit.
//
// The reference computes these with serial loops that scatter into cells
// and nodes (grid_polyhedra_auxiliary_functions.cpp).  Here every scatter
// becomes a gather: each cell (or node) walks its own list of contributions
// in the order the reference's loop would have delivered them, and adds them
// with the same expressions, so the sums round identically and no atomics
// touch floating-point values.  The lists are built on the device:
//   cell -> faces        ascending face index (the face loops' order);
//   cell -> nodes (c2n)  distinct nodes in order of first appearance over the
//                        cell's faces (CalC2N's generic branch);
//   node -> boundary face-node positions, ascending (face, then node slot);
//   node -> c2n positions, ascending (= ascending cell).
// Integer counts go through atomics and CUB's exclusive scan; each list is
// then sorted per segment, which makes the result independent of the order
// the atomics ran in.
//
// Division and square root are IEEE correctly rounded on both sides and the
// file is compiled with --fmad=false, so each expression rounds as in the
// host build (-ffp-contract=off).
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "mfg_internal.h"
#include "mfg_kernels.cuh"
#include "mfgpu.h"

using mfg::kTiny;

namespace {

constexpr int kPrepBlock = 256;

inline int blocks_for(int64_t n) {
  return (int)std::max<int64_t>(1, (n + kPrepBlock - 1) / kPrepBlock);
}

__device__ __forceinline__ int64_t gtid() {
  return (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
}

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

// --------------------------------------------------------------------------
// index checks: nothing below indexes with an unchecked value
// --------------------------------------------------------------------------

__global__ void k_check_nodes(int32_t L, const int32_t *__restrict__ f2n, int32_t N,
                              int32_t *__restrict__ err) {
  const int64_t k = gtid();
  if (k >= L) return;
  const int32_t p = f2n[k];
  if (p < 0 || p >= N) atomicAdd(err, 1);
}

__global__ void k_check_cells(int32_t F, int32_t B, int32_t C, const int32_t *__restrict__ f2c,
                              int32_t *__restrict__ err) {
  const int64_t i = gtid();
  if (i >= F) return;
  const int32_t c1 = f2c[2 * i];
  bool bad = c1 < 0 || c1 >= C;
  if (i >= B) {
    const int32_t c2 = f2c[2 * i + 1];
    bad = bad || c2 < 0 || c2 >= C;
  }
  if (bad) atomicAdd(err, 1);
}

// --------------------------------------------------------------------------
// lists
// --------------------------------------------------------------------------

// faces per cell (CalnFPC): both sides of interior faces, the inner side of
// boundary faces
__global__ void k_count_cell_faces(int32_t F, int32_t B, const int32_t *__restrict__ f2c,
                                   int32_t *__restrict__ cnt) {
  const int64_t i = gtid();
  if (i >= F) return;
  atomicAdd(&cnt[f2c[2 * i]], 1);
  if (i >= B) atomicAdd(&cnt[f2c[2 * i + 1]], 1);
}

__global__ void k_fill_cell_faces(int32_t F, int32_t B, const int32_t *__restrict__ f2c,
                                  const int32_t *__restrict__ ptr, int32_t *__restrict__ cur,
                                  int32_t *__restrict__ cf) {
  const int64_t i = gtid();
  if (i >= F) return;
  const int32_t c1 = f2c[2 * i];
  cf[ptr[c1] + atomicAdd(&cur[c1], 1)] = (int32_t)i;
  if (i >= B) {
    const int32_t c2 = f2c[2 * i + 1];
    cf[ptr[c2] + atomicAdd(&cur[c2], 1)] = (int32_t)i;
  }
}

// ascending order within each segment (short: a cell's faces, a node's cells)
__global__ void k_sort_segments(int32_t nseg, const int32_t *__restrict__ ptr,
                                int32_t *__restrict__ v) {
  const int64_t s = gtid();
  if (s >= nseg) return;
  const int32_t b = ptr[s], e = ptr[s + 1];
  for (int32_t i = b + 1; i < e; i++) {
    const int32_t x = v[i];
    int32_t j = i - 1;
    while (j >= b && v[j] > x) {
      v[j + 1] = v[j];
      j--;
    }
    v[j + 1] = x;
  }
}

// Distinct nodes of cell c in order of first appearance over its faces
// (ascending face order, each face's nodes in file order): the generic
// branch of CalC2N (grid_polyhedra_auxiliary_functions.cpp:1438-1830).  A
// node is new when no earlier position of the walk holds it.  FILL=false
// counts, FILL=true writes the list from ptr[c].
template <bool FILL>
__global__ void k_cell_nodes(int32_t C, const int32_t *__restrict__ cptr,
                             const int32_t *__restrict__ cf, const int32_t *__restrict__ fptr,
                             const int32_t *__restrict__ f2n, int32_t *__restrict__ cnt,
                             const int32_t *__restrict__ ptr, int32_t *__restrict__ c2n,
                             int32_t *__restrict__ c2n_cell, int32_t *__restrict__ nnpc) {
  const int64_t c = gtid();
  if (c >= C) return;
  const int32_t sb = cptr[c], se = cptr[c + 1];
  int32_t m = 0;
  for (int32_t s = sb; s < se; s++) {
    const int32_t f = cf[s];
    for (int32_t k = fptr[f]; k < fptr[f + 1]; k++) {
      const int32_t p = f2n[k];
      bool seen = false;
      for (int32_t s2 = sb; s2 <= s && !seen; s2++) {
        const int32_t f2 = cf[s2];
        const int32_t kend = (s2 == s) ? k : fptr[f2 + 1];
        for (int32_t k2 = fptr[f2]; k2 < kend; k2++)
          if (f2n[k2] == p) {
            seen = true;
            break;
          }
      }
      if (seen) continue;
      if (FILL) {
        c2n[ptr[c] + m] = p;
        c2n_cell[ptr[c] + m] = (int32_t)c;
      }
      m++;
    }
  }
  if (FILL)
    nnpc[c] = m;
  else
    cnt[c] = m;
}

// node -> boundary face-node positions k < fptr[B]; bent_face[k] = face
__global__ void k_count_bnodes(int32_t B, const int32_t *__restrict__ fptr,
                               const int32_t *__restrict__ f2n, int32_t *__restrict__ cnt,
                               int32_t *__restrict__ bent_face) {
  const int64_t i = gtid();
  if (i >= B) return;
  for (int32_t k = fptr[i]; k < fptr[i + 1]; k++) {
    atomicAdd(&cnt[f2n[k]], 1);
    bent_face[k] = (int32_t)i;
  }
}

// node -> positions of `key` (f2n over boundary faces, or c2n), unordered
__global__ void k_fill_by_node(int32_t L, const int32_t *__restrict__ key,
                               const int32_t *__restrict__ ptr, int32_t *__restrict__ cur,
                               int32_t *__restrict__ list) {
  const int64_t k = gtid();
  if (k >= L) return;
  const int32_t p = key[k];
  list[ptr[p] + atomicAdd(&cur[p], 1)] = (int32_t)k;
}

__global__ void k_count_by_node(int32_t L, const int32_t *__restrict__ key,
                                int32_t *__restrict__ cnt) {
  const int64_t k = gtid();
  if (k >= L) return;
  atomicAdd(&cnt[key[k]], 1);
}

// --------------------------------------------------------------------------
// metrics (grid_polyhedra_auxiliary_functions.cpp, via ComputeMetrics,
// grid_polyhedra.cpp:1071-1118)
// --------------------------------------------------------------------------

// FaceCellCenterbyAverage, face part (:271-290)
__global__ void k_face_average(int32_t F, const int32_t *__restrict__ fptr,
                               const int32_t *__restrict__ f2n, const double *__restrict__ x,
                               const double *__restrict__ y, const double *__restrict__ z,
                               double *__restrict__ xfc, double *__restrict__ yfc,
                               double *__restrict__ zfc) {
  const int64_t i = gtid();
  if (i >= F) return;
  const int32_t b = fptr[i], e = fptr[i + 1];
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int32_t k = b; k < e; k++) {
    const int32_t p = f2n[k];
    sx += x[p];
    sy += y[p];
    sz += z[p];
  }
  const int32_t m = e - b;
  xfc[i] = sx / m;
  yfc[i] = sy / m;
  zfc[i] = sz / m;
}

// FaceCellCenterbyAverage, cell part (:292-351): the face centres of the
// cell summed in ascending face order, divided by its face count
__global__ void k_cell_average(int32_t C, const int32_t *__restrict__ cptr,
                               const int32_t *__restrict__ cf, const double *__restrict__ xfc,
                               const double *__restrict__ yfc, const double *__restrict__ zfc,
                               double *__restrict__ xcc, double *__restrict__ ycc,
                               double *__restrict__ zcc) {
  const int64_t c = gtid();
  if (c >= C) return;
  const int32_t sb = cptr[c], se = cptr[c + 1];
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int32_t s = sb; s < se; s++) {
    const int32_t f = cf[s];
    sx += xfc[f];
    sy += yfc[f];
    sz += zfc[f];
  }
  const int32_t m = se - sb;
  xcc[c] = sx / m;
  ycc[c] = sy / m;
  zcc[c] = sz / m;
}

// FaceAreaNormalCentroid_cycle (:68-265): four refinements of the face
// centroid from the area-weighted triangle fan about the current one, then
// the normal and area from the fan about the refined centroid.
__global__ void k_face_metrics(int32_t F, const int32_t *__restrict__ fptr,
                               const int32_t *__restrict__ f2n, const int32_t *__restrict__ f2c,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ xcc,
                               const double *__restrict__ ycc, const double *__restrict__ zcc,
                               double *__restrict__ xfc, double *__restrict__ yfc,
                               double *__restrict__ zfc, double *__restrict__ xfn,
                               double *__restrict__ yfn, double *__restrict__ zfn,
                               double *__restrict__ area) {
  const int64_t i = gtid();
  if (i >= F) return;
  const int32_t b = fptr[i], m = fptr[i + 1] - b;
  double fx = xfc[i], fy = yfc[i], fz = zfc[i];
  double ar = 0.0, nxo = 0.0, nyo = 0.0, nzo = 0.0;
  for (int k = 0; k <= 4; k++) {
    const bool last = (k == 4);
    double a = 0.0, tx = 0.0, ty = 0.0, tz = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    const int32_t p1 = f2n[b];
    for (int32_t j = 0; j < m; j++) {
      const int32_t p2 = f2n[b + j];
      const int32_t p3 = (j == m - 1) ? p1 : f2n[b + j + 1];
      const double x2 = x[p2], y2 = y[p2], z2 = z[p2];
      const double x3 = x[p3], y3 = y[p3], z3 = z[p3];
      const double x21 = x2 - fx, y21 = y2 - fy, z21 = z2 - fz;
      const double x31 = x3 - fx, y31 = y3 - fy, z31 = z3 - fz;
      const double xn = y21 * z31 - y31 * z21;
      const double yn = z21 * x31 - z31 * x21;
      const double zn = x21 * y31 - x31 * y21;
      const double art = sqrt(xn * xn + yn * yn + zn * zn);
      const double xt = x2 + x3 + fx;
      const double yt = y2 + y3 + fy;
      const double zt = z2 + z3 + fz;
      a += art;
      tx += art * xt;
      ty += art * yt;
      tz += art * zt;
      if (last) {
        sx += xn;
        sy += yn;
        sz += zn;
      }
    }
    if (a > kTiny) {
      const double r = 1.0 / a / 3.0;
      fx = tx * r;
      fy = ty * r;
      fz = tz * r;
    }
    if (last) {
      double art = sqrt(sx * sx + sy * sy + sz * sz);
      ar = art * 0.5;
      if (art > kTiny) {
        nxo = sx / art;
        nyo = sy / art;
        nzo = sz / art;
      } else {
        const int32_t c1 = f2c[2 * i];
        const double xn = fx - xcc[c1], yn = fy - ycc[c1], zn = fz - zcc[c1];
        art = sqrt(xn * xn + yn * yn + zn * zn);
        nxo = xn / art;
        nyo = yn / art;
        nzo = zn / art;
      }
    }
  }
  xfc[i] = fx;
  yfc[i] = fy;
  zfc[i] = fz;
  xfn[i] = nxo;
  yfn[i] = nyo;
  zfn[i] = nzo;
  area[i] = ar;
}

// CellVolCentroid (:357-613), inner cells: volume and centroid from the
// tetrahedra (face triangle, cell centre), summed over the cell's faces in
// ascending order (the inner side of a face negates the signed volume),
// then the centroid is kept only if it lies inside every face plane.
// A face listed twice for one cell (both sides the same cell) counts as its
// first side, then its second, as the reference's loop does.
__global__ void k_cell_volume(int32_t C, const int32_t *__restrict__ cptr,
                              const int32_t *__restrict__ cf, const int32_t *__restrict__ fptr,
                              const int32_t *__restrict__ f2n, const int32_t *__restrict__ f2c,
                              const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ xfc,
                              const double *__restrict__ yfc, const double *__restrict__ zfc,
                              const double *__restrict__ xfn, const double *__restrict__ yfn,
                              const double *__restrict__ zfn, double *__restrict__ xcc,
                              double *__restrict__ ycc, double *__restrict__ zcc,
                              double *__restrict__ vol, int32_t *__restrict__ bad) {
  const int64_t c = gtid();
  if (c >= C) return;
  const int32_t sb = cptr[c], se = cptr[c + 1];
  const double cx = xcc[c], cy = ycc[c], cz = zcc[c];
  double tx = 0.0, ty = 0.0, tz = 0.0, v = 0.0;
  int32_t prev = -1;
  for (int32_t s = sb; s < se; s++) {
    const int32_t f = cf[s];
    const bool first = f2c[2 * f] == c && f != prev;
    prev = f;
    const double fx = xfc[f], fy = yfc[f], fz = zfc[f];
    const int32_t b = fptr[f], m = fptr[f + 1] - b;
    const int32_t p1 = f2n[b];
    for (int32_t j = 0; j < m; j++) {
      const int32_t p2 = f2n[b + j];
      const int32_t p3 = (j == m - 1) ? p1 : f2n[b + j + 1];
      const double x2 = x[p2], y2 = y[p2], z2 = z[p2];
      const double x3 = x[p3], y3 = y[p3], z3 = z[p3];
      const double x21 = x2 - fx, y21 = y2 - fy, z21 = z2 - fz;
      const double x31 = x3 - fx, y31 = y3 - fy, z31 = z3 - fz;
      const double nx = y21 * z31 - y31 * z21;
      const double ny = z21 * x31 - z31 * x21;
      const double nz = x21 * y31 - x31 * y21;
      const double x41 = cx - fx, y41 = cy - fy, z41 = cz - fz;
      const double xt = x2 + x3 + fx + cx;
      const double yt = y2 + y3 + fy + cy;
      const double zt = z2 + z3 + fz + cz;
      double volt = nx * x41 + ny * y41 + nz * z41;
      if (first) volt = -volt;
      tx += volt * xt;
      ty += volt * yt;
      tz += volt * zt;
      v += volt;
    }
  }
  const double tmp = 1.0 / (4.0 * v + kTiny);
  tx *= tmp;
  ty *= tmp;
  tz *= tmp;
  v /= 6.0;
  if (v < kTiny) atomicAdd(bad, 1);
  bool inside = true;
  prev = -1;
  for (int32_t s = sb; s < se; s++) {
    const int32_t f = cf[s];
    const bool first = f2c[2 * f] == c && f != prev;
    prev = f;
    const double x21 = tx - xfc[f], y21 = ty - yfc[f], z21 = tz - zfc[f];
    const double dot = x21 * xfn[f] + y21 * yfn[f] + z21 * zfn[f];
    if (first ? dot > 0.0 : dot < 0.0) inside = false;
  }
  if (inside) {
    xcc[c] = tx;
    ycc[c] = ty;
    zcc[c] = tz;
  }
  vol[c] = v;
}

// Per face, after k_cell_volume: the ghost cell of a boundary face mirrored
// through the face plane (CellVolCentroid :588-611, with the normal before
// CorrectFaceNormal), then CorrectFaceNormal (:619-671) for a face of
// (near) zero area.
__global__ void k_face_fix(int32_t F, int32_t B, int32_t C, const int32_t *__restrict__ fptr,
                           const int32_t *__restrict__ f2n, const int32_t *__restrict__ f2c,
                           const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, const double *__restrict__ xfc,
                           const double *__restrict__ yfc, const double *__restrict__ zfc,
                           const double *__restrict__ area, double *__restrict__ xfn,
                           double *__restrict__ yfn, double *__restrict__ zfn,
                           double *__restrict__ xcc, double *__restrict__ ycc,
                           double *__restrict__ zcc, double *__restrict__ vol) {
  const int64_t i = gtid();
  if (i >= F) return;
  const int32_t c1 = f2c[2 * i];
  const double fx = xfc[i], fy = yfc[i], fz = zfc[i];
  const double a = area[i];
  const double cx = xcc[c1], cy = ycc[c1], cz = zcc[c1];
  if (i < B) {
    const int64_t c2 = i + C;
    const double nx = xfn[i], ny = yfn[i], nz = zfn[i];
    if (a > kTiny) {
      const double tmp = 2. * ((cx - fx) * nx + (cy - fy) * ny + (cz - fz) * nz);
      xcc[c2] = cx - nx * tmp;
      ycc[c2] = cy - ny * tmp;
      zcc[c2] = cz - nz * tmp;
    } else {
      xcc[c2] = -cx + 2. * fx;
      ycc[c2] = -cy + 2. * fy;
      zcc[c2] = -cz + 2. * fz;
    }
    vol[c2] = vol[c1];
  }
  if (a < kTiny) {
    const int32_t p1 = f2n[fptr[i]];
    double x21 = cx - fx, y21 = cy - fy, z21 = cz - fz;
    const double x31 = x[p1] - fx, y31 = y[p1] - fy, z31 = z[p1] - fz;
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

// AbsMaxSignFirst (:812-823)
__device__ __forceinline__ double abs_max_sign_first(double a, double b) {
  const int sign = (a > 0) ? 1 : -1;
  double c = dmax(fabs(a), fabs(b));
  c *= sign;
  return c;
}

// CorrectCellCentroid (:679-807): a centroid closer than 1e-10 to one of its
// face planes moves off it; the cell's faces apply in ascending order, each
// seeing the moves of the ones before.
__global__ void k_cell_fix(int32_t C, const int32_t *__restrict__ cptr,
                           const int32_t *__restrict__ cf, const double *__restrict__ xfc,
                           const double *__restrict__ yfc, const double *__restrict__ zfc,
                           const double *__restrict__ xfn, const double *__restrict__ yfn,
                           const double *__restrict__ zfn, double *__restrict__ xcc,
                           double *__restrict__ ycc, double *__restrict__ zcc, double scale) {
  const int64_t c = gtid();
  if (c >= C) return;
  const double minDn = 1.0e-10;
  double cx = xcc[c], cy = ycc[c], cz = zcc[c];
  bool moved = false;
  for (int32_t s = cptr[c]; s < cptr[c + 1]; s++) {
    const int32_t f = cf[s];
    const double nx = xfn[f], ny = yfn[f], nz = zfn[f];
    const double x21 = cx - xfc[f], y21 = cy - yfc[f], z21 = cz - zfc[f];
    const double dot = x21 * nx + y21 * ny + z21 * nz;
    if (fabs(dot) < minDn) {
      double dx = minDn * nx, dy = minDn * ny, dz = minDn * nz;
      dx = abs_max_sign_first(dx, scale * cx);
      dy = abs_max_sign_first(dy, scale * cy);
      dz = abs_max_sign_first(dz, scale * cz);
      const int sign = (dot > 0.0) ? 1 : -1;
      cx += sign * dx;
      cy += sign * dy;
      cz += sign * dz;
      moved = true;
    }
  }
  if (moved) {
    xcc[c] = cx;
    ycc[c] = cy;
    zcc[c] = cz;
  }
}

// --------------------------------------------------------------------------
// node weights: ComputeWeight3D_Node (:831-1049) and FindNodeSYMM
// (:2060-2140)
// --------------------------------------------------------------------------

// The pass in which a boundary face's nodes take inverse-distance weights:
// walls first, then far field, then the other types; symmetry and interface
// faces never (3).
__device__ __forceinline__ int weight_pass(int32_t t) {
  if (t == MFG_BC_WALL) return 0;
  if (t == MFG_BC_FAR_FIELD || t == MFG_BC_FAR_FIELD_MOD) return 1;
  if (t == MFG_BC_SYMM || t == MFG_BC_INTERFACE) return 3;
  return 2;
}

// Per node.  In the reference a node marked by an earlier pass is skipped by
// the later ones, so its weight sums exactly the faces of its first pass, in
// face order; an unmarked node sums its cells in ascending cell order.
__global__ void k_node_weights(int32_t N, const int32_t *__restrict__ nbptr,
                               const int32_t *__restrict__ nblist,
                               const int32_t *__restrict__ bent_face,
                               const int32_t *__restrict__ bctype,
                               const int32_t *__restrict__ ncptr,
                               const int32_t *__restrict__ nclist,
                               const int32_t *__restrict__ c2n_cell, const double *__restrict__ x,
                               const double *__restrict__ y, const double *__restrict__ z,
                               const double *__restrict__ xfc, const double *__restrict__ yfc,
                               const double *__restrict__ zfc, const double *__restrict__ xfn,
                               const double *__restrict__ yfn, const double *__restrict__ zfn,
                               const double *__restrict__ xcc, const double *__restrict__ ycc,
                               const double *__restrict__ zcc, double *__restrict__ wnode,
                               int32_t *__restrict__ nmark, double *__restrict__ wbface,
                               double *__restrict__ wc2n, int32_t *__restrict__ nodesymm,
                               double *__restrict__ xsym, double *__restrict__ ysym,
                               double *__restrict__ zsym) {
  const int64_t p = gtid();
  if (p >= N) return;
  const int32_t bb = nbptr[p], be = nbptr[p + 1];
  const double px = x[p], py = y[p], pz = z[p];
  int pass = 3;
  for (int32_t s = bb; s < be; s++) pass = min(pass, weight_pass(bctype[bent_face[nblist[s]]]));
  double w = 0.0;
  double sx = 0.0, sy = 0.0, sz = 0.0, nf = 0.0;
  bool symm = false;
  for (int32_t s = bb; s < be; s++) {
    const int32_t k = nblist[s];
    const int32_t i = bent_face[k];
    const int32_t t = bctype[i];
    if (pass < 3 && weight_pass(t) == pass) {
      const double dx = px - xfc[i], dy = py - yfc[i], dz = pz - zfc[i];
      double wr = dx * dx + dy * dy + dz * dz;
      wr = sqrt(wr);
      wr = 1. / wr;
      wbface[k] = wr;
      w += wr;
    } else {
      wbface[k] = 0.0;
    }
    if (t == MFG_BC_SYMM) {
      symm = true;
      sx += xfn[i];
      sy += yfn[i];
      sz += zfn[i];
      nf += 1.0;
    }
  }
  nmark[p] = pass == 0 ? MFG_BC_WALL : (pass == 1 ? MFG_BC_FAR_FIELD : (pass == 2 ? 101 : 0));
  for (int32_t s = ncptr[p]; s < ncptr[p + 1]; s++) {
    const int32_t m = nclist[s];
    if (pass == 3) {
      const int32_t c = c2n_cell[m];
      const double dx = px - xcc[c], dy = py - ycc[c], dz = pz - zcc[c];
      double wr = dx * dx + dy * dy + dz * dz;
      wr = sqrt(wr);
      wr = 1. / wr;
      wc2n[m] = wr;
      w += wr;
    } else {
      wc2n[m] = 0.0;
    }
  }
  wnode[p] = w;
  nodesymm[p] = symm ? 1 : 0;
  xsym[p] = symm ? sx / nf : 0.0;
  ysym[p] = symm ? sy / nf : 0.0;
  zsym[p] = symm ? sz / nf : 0.0;
}

}  // namespace



namespace {

#define PREP_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) {                             \
      mfg::note_cuda_error(#call, (int)e_);              \
      return e_ == cudaErrorMemoryAllocation ? MFG_ERR_NOMEM : MFG_ERR_CUDA; \
    }                                                    \
  } while (0)

template <typename T>
int palloc(mfg_prep_gpu *p, T **ptr, int64_t count) {
  const size_t bytes = std::max<size_t>(1, (size_t)count) * sizeof(T);
  PREP_CUDA(cudaMalloc((void **)ptr, bytes));
  p->allocs.push_back((void *)*ptr);
  return MFG_OK;
}

template <typename T>
int pupload(mfg_prep_gpu *p, T **ptr, const T *host, int64_t count) {
  int rc = palloc(p, ptr, count);
  if (rc) return rc;
  if (count > 0) PREP_CUDA(cudaMemcpy(*ptr, host, (size_t)count * sizeof(T), cudaMemcpyHostToDevice));
  return MFG_OK;
}

template <typename T>
int pdownload(T *host, const T *dev, int64_t count) {
  if (count > 0) PREP_CUDA(cudaMemcpy(host, dev, (size_t)count * sizeof(T), cudaMemcpyDeviceToHost));
  return MFG_OK;
}

void free_prep(mfg_prep_gpu *p) {
  if (!p) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(p->device);
  for (void *a : p->allocs) cudaFree(a);
  if (prev >= 0) cudaSetDevice(prev);
  delete p;
}

int launched() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    mfg::note_cuda_error("kernel launch", (int)e);
    return MFG_ERR_CUDA;
  }
  mfg::note_launches(1);
  return MFG_OK;
}

// exclusive scan of cnt[0, m) (cnt[m - 1] must be 0 to give the total in
// out[m - 1])
int scan(void *tmp, size_t tmp_bytes, const int32_t *cnt, int32_t *out, int32_t m) {
  size_t bytes = tmp_bytes;
  PREP_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, cnt, out, m));
  return MFG_OK;
}

int read_i32(const int32_t *dev, int32_t *host) {
  PREP_CUDA(cudaMemcpy(host, dev, sizeof(int32_t), cudaMemcpyDeviceToHost));
  return MFG_OK;
}

int run_impl(mfg_prep_gpu *p, const mfg_raw_grid *g, const int32_t *bctype) {
  const int32_t N = p->N, F = p->F, C = p->C, B = p->B;
  const int64_t n = p->n;
  int rc;
  // raw grid
  if ((rc = pupload(p, &p->x, g->x, N)) || (rc = pupload(p, &p->y, g->y, N)) ||
      (rc = pupload(p, &p->z, g->z, N)) || (rc = pupload(p, &p->f2n, g->f2n, p->L)) ||
      (rc = pupload(p, &p->f2c, (const int32_t *)g->f2c, 2 * (int64_t)F)) ||
      (rc = pupload(p, &p->bctype, bctype, B)))
    return rc;
  if ((rc = palloc(p, &p->nnpf, (int64_t)F + 1))) return rc;
  if (F > 0) PREP_CUDA(cudaMemcpy(p->nnpf, g->nnpf, sizeof(int32_t) * F, cudaMemcpyHostToDevice));
  PREP_CUDA(cudaMemset(p->nnpf + F, 0, sizeof(int32_t)));

  // scratch: counters (reused), cursors, the two error counts, scan storage
  const int64_t big = std::max<int64_t>(std::max<int64_t>(F, C), N) + 1;
  int32_t *cnt = nullptr, *cur = nullptr, *err = nullptr;
  if ((rc = palloc(p, &cnt, big)) || (rc = palloc(p, &cur, big)) || (rc = palloc(p, &err, 2)))
    return rc;
  size_t tmp_bytes = 0;
  PREP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, cur, (int)big));
  void *tmp = nullptr;
  if ((rc = palloc(p, (char **)&tmp, (int64_t)tmp_bytes))) return rc;

  cudaEvent_t ev0, ev1;
  PREP_CUDA(cudaEventCreate(&ev0));
  if (cudaEventCreate(&ev1) != cudaSuccess) {
    cudaEventDestroy(ev0);
    PREP_CUDA(cudaGetLastError());
    return MFG_ERR_CUDA;
  }
  struct Events {
    cudaEvent_t a, b;
    ~Events() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evs{ev0, ev1};
  PREP_CUDA(cudaEventRecord(ev0, 0));

  // 1. every index in range, before anything indexes with one
  PREP_CUDA(cudaMemset(err, 0, 2 * sizeof(int32_t)));
  k_check_nodes<<<blocks_for(p->L), kPrepBlock>>>(p->L, p->f2n, N, err);
  if ((rc = launched())) return rc;
  k_check_cells<<<blocks_for(F), kPrepBlock>>>(F, B, C, p->f2c, err);
  if ((rc = launched())) return rc;
  int32_t nbad = 0;
  if ((rc = read_i32(err, &nbad))) return rc;
  if (nbad) return MFG_ERR_BADMESH;

  // 2. face -> node offsets, cell -> faces
  if ((rc = palloc(p, &p->fptr, (int64_t)F + 1))) return rc;
  if ((rc = scan(tmp, tmp_bytes, p->nnpf, p->fptr, F + 1))) return rc;
  if ((rc = palloc(p, &p->cptr, (int64_t)C + 1))) return rc;
  PREP_CUDA(cudaMemset(cnt, 0, sizeof(int32_t) * ((size_t)C + 1)));
  k_count_cell_faces<<<blocks_for(F), kPrepBlock>>>(F, B, p->f2c, cnt);
  if ((rc = launched())) return rc;
  if ((rc = scan(tmp, tmp_bytes, cnt, p->cptr, C + 1))) return rc;
  if ((rc = read_i32(p->cptr + C, &p->S))) return rc;
  if ((rc = palloc(p, &p->cf, p->S))) return rc;
  PREP_CUDA(cudaMemset(cur, 0, sizeof(int32_t) * (size_t)C));
  k_fill_cell_faces<<<blocks_for(F), kPrepBlock>>>(F, B, p->f2c, p->cptr, cur, p->cf);
  if ((rc = launched())) return rc;
  k_sort_segments<<<blocks_for(C), kPrepBlock>>>(C, p->cptr, p->cf);
  if ((rc = launched())) return rc;

  // 3. metrics
  if ((rc = palloc(p, &p->xfn, F)) || (rc = palloc(p, &p->yfn, F)) ||
      (rc = palloc(p, &p->zfn, F)) || (rc = palloc(p, &p->area, F)) ||
      (rc = palloc(p, &p->xfc, F)) || (rc = palloc(p, &p->yfc, F)) ||
      (rc = palloc(p, &p->zfc, F)) || (rc = palloc(p, &p->xcc, n)) ||
      (rc = palloc(p, &p->ycc, n)) || (rc = palloc(p, &p->zcc, n)) ||
      (rc = palloc(p, &p->vol, n)))
    return rc;
  k_face_average<<<blocks_for(F), kPrepBlock>>>(F, p->fptr, p->f2n, p->x, p->y, p->z, p->xfc,
                                                 p->yfc, p->zfc);
  if ((rc = launched())) return rc;
  k_cell_average<<<blocks_for(C), kPrepBlock>>>(C, p->cptr, p->cf, p->xfc, p->yfc, p->zfc,
                                                 p->xcc, p->ycc, p->zcc);
  if ((rc = launched())) return rc;
  k_face_metrics<<<blocks_for(F), kPrepBlock>>>(F, p->fptr, p->f2n, p->f2c, p->x, p->y, p->z,
                                                 p->xcc, p->ycc, p->zcc, p->xfc, p->yfc, p->zfc,
                                                 p->xfn, p->yfn, p->zfn, p->area);
  if ((rc = launched())) return rc;
  k_cell_volume<<<blocks_for(C), kPrepBlock>>>(C, p->cptr, p->cf, p->fptr, p->f2n, p->f2c, p->x,
                                                p->y, p->z, p->xfc, p->yfc, p->zfc, p->xfn,
                                                p->yfn, p->zfn, p->xcc, p->ycc, p->zcc, p->vol,
                                                err + 1);
  if ((rc = launched())) return rc;
  if ((rc = read_i32(err + 1, &nbad))) return rc;
  if (nbad) return MFG_ERR_BADMESH;  // CellVolCentroid stops here (:528-536)
  k_face_fix<<<blocks_for(F), kPrepBlock>>>(F, B, C, p->fptr, p->f2n, p->f2c, p->x, p->y, p->z,
                                             p->xfc, p->yfc, p->zfc, p->area, p->xfn, p->yfn,
                                             p->zfn, p->xcc, p->ycc, p->zcc, p->vol);
  if ((rc = launched())) return rc;
  // CorrectCellCentroid's 10^(1-16) from the C library's pow, as the host
  volatile double ten = 10.0;
  const double scale = pow(ten, -16 + 1);
  k_cell_fix<<<blocks_for(C), kPrepBlock>>>(C, p->cptr, p->cf, p->xfc, p->yfc, p->zfc, p->xfn,
                                             p->yfn, p->zfn, p->xcc, p->ycc, p->zcc, scale);
  if ((rc = launched())) return rc;

  // 4. cell -> distinct nodes
  if ((rc = palloc(p, &p->c2n_ptr, (int64_t)C + 1)) || (rc = palloc(p, &p->nnpc, C))) return rc;
  PREP_CUDA(cudaMemset(cnt, 0, sizeof(int32_t) * ((size_t)C + 1)));
  k_cell_nodes<false><<<blocks_for(C), kPrepBlock>>>(C, p->cptr, p->cf, p->fptr, p->f2n, cnt,
                                                      nullptr, nullptr, nullptr, nullptr);
  if ((rc = launched())) return rc;
  if ((rc = scan(tmp, tmp_bytes, cnt, p->c2n_ptr, C + 1))) return rc;
  if ((rc = read_i32(p->c2n_ptr + C, &p->K))) return rc;
  if ((rc = palloc(p, &p->c2n, p->K)) || (rc = palloc(p, &p->c2n_cell, p->K))) return rc;
  k_cell_nodes<true><<<blocks_for(C), kPrepBlock>>>(C, p->cptr, p->cf, p->fptr, p->f2n, nullptr,
                                                     p->c2n_ptr, p->c2n, p->c2n_cell, p->nnpc);
  if ((rc = launched())) return rc;

  // 5. node -> boundary face-node positions, node -> c2n positions
  if ((rc = palloc(p, &p->nbptr, (int64_t)N + 1)) || (rc = palloc(p, &p->nblist, p->LB)) ||
      (rc = palloc(p, &p->bent_face, p->LB)) || (rc = palloc(p, &p->ncptr, (int64_t)N + 1)) ||
      (rc = palloc(p, &p->nclist, p->K)))
    return rc;
  PREP_CUDA(cudaMemset(cnt, 0, sizeof(int32_t) * ((size_t)N + 1)));
  k_count_bnodes<<<blocks_for(B), kPrepBlock>>>(B, p->fptr, p->f2n, cnt, p->bent_face);
  if ((rc = launched())) return rc;
  if ((rc = scan(tmp, tmp_bytes, cnt, p->nbptr, N + 1))) return rc;
  PREP_CUDA(cudaMemset(cur, 0, sizeof(int32_t) * (size_t)N));
  k_fill_by_node<<<blocks_for(p->LB), kPrepBlock>>>(p->LB, p->f2n, p->nbptr, cur, p->nblist);
  if ((rc = launched())) return rc;
  k_sort_segments<<<blocks_for(N), kPrepBlock>>>(N, p->nbptr, p->nblist);
  if ((rc = launched())) return rc;
  PREP_CUDA(cudaMemset(cnt, 0, sizeof(int32_t) * ((size_t)N + 1)));
  k_count_by_node<<<blocks_for(p->K), kPrepBlock>>>(p->K, p->c2n, cnt);
  if ((rc = launched())) return rc;
  if ((rc = scan(tmp, tmp_bytes, cnt, p->ncptr, N + 1))) return rc;
  PREP_CUDA(cudaMemset(cur, 0, sizeof(int32_t) * (size_t)N));
  k_fill_by_node<<<blocks_for(p->K), kPrepBlock>>>(p->K, p->c2n, p->ncptr, cur, p->nclist);
  if ((rc = launched())) return rc;
  k_sort_segments<<<blocks_for(N), kPrepBlock>>>(N, p->ncptr, p->nclist);
  if ((rc = launched())) return rc;

  // 6. weights
  if ((rc = palloc(p, &p->wnode, N)) || (rc = palloc(p, &p->nmark, N)) ||
      (rc = palloc(p, &p->wbface, p->LB)) || (rc = palloc(p, &p->wc2n, p->K)) ||
      (rc = palloc(p, &p->nodesymm, N)) || (rc = palloc(p, &p->xsym, N)) ||
      (rc = palloc(p, &p->ysym, N)) || (rc = palloc(p, &p->zsym, N)))
    return rc;
  k_node_weights<<<blocks_for(N), kPrepBlock>>>(
      N, p->nbptr, p->nblist, p->bent_face, p->bctype, p->ncptr, p->nclist, p->c2n_cell, p->x,
      p->y, p->z, p->xfc, p->yfc, p->zfc, p->xfn, p->yfn, p->zfn, p->xcc, p->ycc, p->zcc,
      p->wnode, p->nmark, p->wbface, p->wc2n, p->nodesymm, p->xsym, p->ysym, p->zsym);
  if ((rc = launched())) return rc;
  PREP_CUDA(cudaEventRecord(ev1, 0));
  PREP_CUDA(cudaEventSynchronize(ev1));
  float ms = 0.f;
  PREP_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  p->kernel_ms = ms;
  return MFG_OK;
}

struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int d) {
    cudaGetDevice(&prev);
    cudaSetDevice(d);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

int mfg_prep_gpu_run(const mfg_raw_grid *g, const int32_t *bctype, int32_t device,
                     mfg_prep_gpu **out) {
  if (!out) return MFG_ERR_INVALID;
  *out = nullptr;
  if (!g || !g->x || !g->y || !g->z || !g->nnpf || !g->f2n || !g->f2c) return MFG_ERR_INVALID;
  if (g->n_node < 1 || g->n_cell < 1 || g->n_face < 0 || g->n_bface < 0 ||
      g->n_bface > g->n_face || (g->n_bface > 0 && !bctype))
    return MFG_ERR_INVALID;
  // sizes: every list index below stays within int32
  if (2 * (int64_t)g->n_face > INT32_MAX || (int64_t)g->n_cell + g->n_bface > INT32_MAX)
    return MFG_ERR_UNSUPPORTED;
  int64_t L = 0, LB = 0;
  for (int32_t i = 0; i < g->n_face; i++) {
    if (g->nnpf[i] < 1) return MFG_ERR_BADMESH;
    L += g->nnpf[i];
    if (i + 1 == g->n_bface) LB = L;
  }
  if (2 * L > INT32_MAX) return MFG_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) {
    cudaGetLastError();
    return MFG_ERR_NODEVICE;
  }
  DeviceScope scope(device);
  mfg_prep_gpu *p = new mfg_prep_gpu();
  p->device = device;
  p->N = g->n_node;
  p->F = g->n_face;
  p->C = g->n_cell;
  p->B = g->n_bface;
  p->n = (int64_t)g->n_cell + g->n_bface;
  p->L = (int32_t)L;
  p->LB = (int32_t)LB;
  const int rc = run_impl(p, g, bctype);
  if (rc != MFG_OK) {
    cudaDeviceSynchronize();
    free_prep(p);
    return rc;
  }
  *out = p;
  return MFG_OK;
}

int mfg_prep_gpu_c2n_size(const mfg_prep_gpu *p, int64_t *n_c2n) {
  if (!p || !n_c2n) return MFG_ERR_INVALID;
  *n_c2n = p->K;
  return MFG_OK;
}

int mfg_prep_gpu_kernel_ms(const mfg_prep_gpu *p, double *ms) {
  if (!p || !ms) return MFG_ERR_INVALID;
  *ms = p->kernel_ms;
  return MFG_OK;
}

int mfg_prep_gpu_metrics(mfg_prep_gpu *p, double *xfn, double *yfn, double *zfn, double *area,
                         double *xfc, double *yfc, double *zfc, double *xcc, double *ycc,
                         double *zcc, double *vol) {
  if (!p || !xfn || !yfn || !zfn || !area || !xfc || !yfc || !zfc || !xcc || !ycc || !zcc ||
      !vol)
    return MFG_ERR_INVALID;
  DeviceScope scope(p->device);
  int rc;
  const int64_t F = p->F, n = p->n;
  if ((rc = pdownload(xfn, p->xfn, F)) || (rc = pdownload(yfn, p->yfn, F)) ||
      (rc = pdownload(zfn, p->zfn, F)) || (rc = pdownload(area, p->area, F)) ||
      (rc = pdownload(xfc, p->xfc, F)) || (rc = pdownload(yfc, p->yfc, F)) ||
      (rc = pdownload(zfc, p->zfc, F)) || (rc = pdownload(xcc, p->xcc, n)) ||
      (rc = pdownload(ycc, p->ycc, n)) || (rc = pdownload(zcc, p->zcc, n)) ||
      (rc = pdownload(vol, p->vol, n)))
    return rc;
  return MFG_OK;
}

int mfg_prep_gpu_node_weights(mfg_prep_gpu *p, double *wnode, int32_t *nmark, double *wbface,
                              int32_t *nnpc, int32_t *c2n, double *wc2n, int32_t *nodesymm,
                              double *xfn_n_symm, double *yfn_n_symm, double *zfn_n_symm) {
  if (!p || !wnode || !nmark || (!wbface && p->LB > 0) || !nnpc || (!c2n && p->K > 0) ||
      (!wc2n && p->K > 0) || !nodesymm || !xfn_n_symm || !yfn_n_symm || !zfn_n_symm)
    return MFG_ERR_INVALID;
  DeviceScope scope(p->device);
  int rc;
  const int64_t N = p->N;
  if ((rc = pdownload(wnode, p->wnode, N)) || (rc = pdownload(nmark, p->nmark, N)) ||
      (rc = pdownload(wbface, p->wbface, (int64_t)p->LB)) ||
      (rc = pdownload(nnpc, p->nnpc, (int64_t)p->C)) ||
      (rc = pdownload(c2n, p->c2n, (int64_t)p->K)) ||
      (rc = pdownload(wc2n, p->wc2n, (int64_t)p->K)) ||
      (rc = pdownload(nodesymm, p->nodesymm, N)) || (rc = pdownload(xfn_n_symm, p->xsym, N)) ||
      (rc = pdownload(yfn_n_symm, p->ysym, N)) || (rc = pdownload(zfn_n_symm, p->zsym, N)))
    return rc;
  return MFG_OK;
}

int mfg_prep_gpu_init_flow(mfg_prep_gpu *p, const mfg_params *params, double bump_amp,
                           double bump_sigma, double bump_x0, double bump_y0, double bump_z0,
                           double *q) {
  if (!p || !params || !q) return MFG_ERR_INVALID;
  DeviceScope scope(p->device);
  const int64_t n = p->n, B = p->B, B1 = std::max<int64_t>(B, 1);
  std::vector<int32_t> f2c(2 * (size_t)B1, 0), bt((size_t)B1, 0);
  std::vector<double> nx(B1), ny(B1), nz(B1), cx(n), cy(n), cz(n);
  int rc;
  if ((rc = pdownload(f2c.data(), p->f2c, 2 * B)) || (rc = pdownload(bt.data(), p->bctype, B)) ||
      (rc = pdownload(nx.data(), p->xfn, B)) || (rc = pdownload(ny.data(), p->yfn, B)) ||
      (rc = pdownload(nz.data(), p->zfn, B)) || (rc = pdownload(cx.data(), p->xcc, n)) ||
      (rc = pdownload(cy.data(), p->ycc, n)) || (rc = pdownload(cz.data(), p->zcc, n)))
    return rc;
  // the host routine reads the sizes and, of boundary faces only, f2c, the
  // normals and the BC types
  mfg_raw_grid g{};
  g.n_node = p->N;
  g.n_face = p->F;
  g.n_cell = p->C;
  g.n_bface = p->B;
  g.f2c = f2c.data();
  return mfg_prep_init_flow(&g, params, bt.data(), nx.data(), ny.data(), nz.data(), cx.data(),
                            cy.data(), cz.data(), bump_amp, bump_sigma, bump_x0, bump_y0, bump_z0,
                            q);
}

int mfg_prep_gpu_destroy(mfg_prep_gpu *p) {
  free_prep(p);
  return MFG_OK;
}

}  // extern "C"
