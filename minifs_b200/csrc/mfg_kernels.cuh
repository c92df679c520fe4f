// Device code of the mfgpu hot path (sm_100a, FP64).
//
// Bit-faithfulness rules, kept throughout:
//  * every arithmetic expression has the operand order of the reference
//    routine it restates (cited per function); the file is compiled with
//    --fmad=false so no multiply-add is contracted;
//  * per-cell sums run over the cell's faces in ascending face order, the
//    order in which the reference's face loops scatter into that cell, so
//    gathers reproduce the scatter sums exactly and no atomics are needed;
//  * per-cell values that the reference recomputes at every face from the
//    same operands (sound speed, total enthalpy, conserved energy) are
//    computed once per cell with the same expression, which yields the same
//    bits.
#pragma once

#include <cstdint>

namespace mfg {

constexpr double kTiny = 1.e-40;  // number_type.h:29
constexpr double kBig = 1.e40;    // number_type.h:28

// Host-side state shared by the library's translation units (defined with
// the iteration path): record a CUDA error for mfg_last_cuda_error, and
// count kernel launches for mfg_kernel_launches.
void note_cuda_error(const char *what, int code);
void note_launches(int64_t k);

// Per-cell state record, 64 bytes: the five primitive variables of the
// reference's SoA arrays plus three derived per-cell quantities.
enum : int {
  Q_RHO = 0, Q_U, Q_V, Q_W, Q_P,
  Q_A,   // sqrt(gam*(p+p_bar)/rho): compute_timestep.cpp:763-768, forward_lusgs.cpp:566-570, :1291-1293
  Q_HT,  // total enthalpy et + p + p_bar: cal_flux.cpp:688-693
  Q_E,   // p/gam1 + 0.5*rho*|v|^2: forward_lusgs.cpp:1285-1289
  Q_STRIDE = 8
};

// One (cell, face) slot in ascending face order of the cell: the face normal
// as stored (pointing out of the face's first cell), the face area, the
// distance of the face centroid to this cell's centroid along the normal
// (compute_timestep.cpp:762), the other cell, and flags.
struct __align__(16) SlotRec {
  double nx, ny, nz, area, dn;
  int32_t nb;      // neighbour cell (ghost C+k for boundary face k)
  int32_t face;    // face index
  int32_t flags;   // SLOT_*
  int32_t tri[3];  // a triangular face's nodes in file order (SLOT_TRI), else 0
};
static_assert(sizeof(SlotRec) == 64, "slot record: one 64-byte line");
// SLOT_TRI: the gradient reads the face's nodes from the slot instead of
// through the face -> node offsets
enum : int32_t { SLOT_IS_C2 = 1, SLOT_BOUNDARY = 2, SLOT_NODE_AVG = 4, SLOT_TRI = 8 };

// A centroid (face or cell) and, for a cell, its length scale vol^(1/3)
// (second-order reconstruction and its limiters).
struct __align__(16) Cen {
  double x, y, z, h;
};

// LU-SGS sweep record: normal oriented out of the swept cell and the
// multiplier of the flux (0.5*area forward, area backward).
struct __align__(16) SweepRec {
  double nx, ny, nz, w;
};

// One face for the per-face flux: the stored normal and area, and its cells.
struct __align__(16) FaceRec {
  double nx, ny, nz, area;
  int32_t c1, c2, pad0, pad1;
};

// Mixed form: single-precision LU-SGS sweep record.
struct __align__(16) SweepRecF {
  float nx, ny, nz, w;
};

struct Params {
  double gam, gamm1, p_bar, alf_l, lhs_omga, peff;
  double rho_min, rho_max, p_min, p_max, p_break, ratio_dtmax;
  double ref[5];  // freestream rho, u, v, w, gauge p (mixed gradient: values kept as deviations)
  // SetGhostVariables' far-field constants (load_grid.cpp:1000-1003, :1105):
  // |freestream velocity| and the freestream entropy pm / pow(rhom, gam),
  // evaluated on the host with the C library's sqrt and pow
  double uvw_norm, entr_m;
};

// Batched cases: several independent grids concatenated into one (cells,
// then ghosts, each in case order).  Kernels read the case of a cell and that
// case's parameters; with P == nullptr there is a single case whose
// parameters come as a kernel argument.
struct Cases {
  const Params *P;        // [ncase]
  const int32_t *of;      // case of each cell and ghost [n]
  const int32_t *first;   // first cell of each case's LU-SGS order [ncase]
  int32_t ncase;
};

__device__ __forceinline__ int32_t case_of(const Cases &cs, int64_t c) {
  return cs.P ? cs.of[c] : 0;
}
__device__ __forceinline__ Params params_of(const Params &P0, const Cases &cs, int64_t c) {
  return cs.P ? cs.P[cs.of[c]] : P0;
}

__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

// Single-precision state record of the mixed form (32 bytes, same fields as
// the FP64 record, rounded from it after every update).
__device__ __forceinline__ void load_q4(const float *__restrict__ q4, int64_t c, float *q) {
  const float4 *p = reinterpret_cast<const float4 *>(q4 + c * Q_STRIDE);
  const float4 a = __ldg(p), b = __ldg(p + 1);
  q[0] = a.x; q[1] = a.y; q[2] = a.z; q[3] = a.w;
  q[4] = b.x; q[5] = b.y; q[6] = b.z; q[7] = b.w;
}
__device__ __forceinline__ void store_q4(float *q4, int64_t c, const double *q) {
  float4 *p = reinterpret_cast<float4 *>(q4 + c * Q_STRIDE);
  p[0] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
  p[1] = make_float4((float)q[4], (float)q[5], (float)q[6], (float)q[7]);
}
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ void load_q(const double *__restrict__ q8, int64_t c, double *q) {
  const double2 *p = reinterpret_cast<const double2 *>(q8 + c * Q_STRIDE);
  double2 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2), e = __ldg(p + 3);
  q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y;
  q[4] = d.x; q[5] = d.y; q[6] = e.x; q[7] = e.y;
}

// 32-byte rows of the library's own allocations (cudaMalloc's 256-byte
// alignment, rows of 64 or 32 bytes) read with one 256-bit load per 32 bytes
// (PTX .v4.f64 / .v8.f32, sm_100): fewer load instructions per gathered row
// than 16-byte loads, the same bytes.  Never for caller-supplied buffers,
// whose alignment is only 16 bytes.
__device__ __forceinline__ void ldg_v4(const double *p, double &a, double &b, double &c,
                                       double &d) {
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void ldg_v8f(const float *p, float *q) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(q[0]), "=f"(q[1]), "=f"(q[2]), "=f"(q[3]), "=f"(q[4]), "=f"(q[5]), "=f"(q[6]),
        "=f"(q[7])
      : "l"(p));
}
// load_q of an own array: the whole record
__device__ __forceinline__ void load_q_w(const double *__restrict__ q8, int64_t c, double *q) {
  const double *p = q8 + c * Q_STRIDE;
  ldg_v4(p, q[0], q[1], q[2], q[3]);
  ldg_v4(p + 4, q[4], q[5], q[6], q[7]);
}
// the five primitive variables only
__device__ __forceinline__ void load_q5_w(const double *__restrict__ q8, int64_t c, double *q) {
  const double *p = q8 + c * Q_STRIDE;
  ldg_v4(p, q[0], q[1], q[2], q[3]);
  q[4] = __ldg(p + 4);
}

__device__ __forceinline__ void store_q(double *__restrict__ q8, int64_t c, const double *q) {
  double2 *p = reinterpret_cast<double2 *>(q8 + c * Q_STRIDE);
  p[0] = make_double2(q[0], q[1]);
  p[1] = make_double2(q[2], q[3]);
  p[2] = make_double2(q[4], q[5]);
  p[3] = make_double2(q[6], q[7]);
}

// Loads that must observe writes of earlier levels of the same sweep in a
// persistent kernel: bypass the non-coherent path.
__device__ __forceinline__ void load_dq_cg(const double *dq8, int64_t c, double *d) {
  const double2 *p = reinterpret_cast<const double2 *>(dq8 + c * Q_STRIDE);
  double2 a = __ldcg(p), b = __ldcg(p + 1), e = __ldcg(p + 2);
  d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y; d[4] = e.x;
}

// Plain (write-through) stores: readers in the same block see them after
// __syncthreads, readers on other SMs through L2 after the release flag.
__device__ __forceinline__ void store_dq(double *dq8, int64_t c, const double *d) {
  double2 *p = reinterpret_cast<double2 *>(dq8 + c * Q_STRIDE);
  p[0] = make_double2(d[0], d[1]);
  p[1] = make_double2(d[2], d[3]);
  p[2] = make_double2(d[4], 0.0);
}

// Derived per-cell quantities from the primitive variables.
__device__ __forceinline__ void cell_props(double *q, const Params &P) {
  const double rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  // compute_timestep.cpp:763 c2tmp = gam * (p[c1] + p_bar) / rho[c1]; eigv = vn + sqrt(c2tmp)
  q[Q_A] = sqrt(P.gam * (p + P.p_bar) / rho);
  // cal_flux.cpp:688-693
  const double et = (p + P.p_bar) / P.gamm1 + 0.5 * rho * (u * u + v * v + w * w);
  q[Q_HT] = et + p + P.p_bar;
  // forward_lusgs.cpp:1285-1289 (gam1 = gam - 1. equals gamm1 = gam - 1.0)
  const double rv2 = 0.5 * rho * (u * u + v * v + w * w);
  q[Q_E] = p / P.gamm1 + rv2;
}

// Arithmetic of the flux routines in T = double (the FP64 form: exactly the
// reference's operations) or T = float (the mixed form: single-precision
// flux arithmetic with hardware reciprocal-based division).
template <typename T>
struct Num;
template <>
struct Num<double> {
  __device__ static __forceinline__ double div(double a, double b) { return a / b; }
  __device__ static __forceinline__ double sqrt_(double a) { return sqrt(a); }
};
template <>
struct Num<float> {
  __device__ static __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
  __device__ static __forceinline__ float sqrt_(float a) { return sqrtf(a); }
};

// The parameters the flux routines read, in T.
template <typename T>
struct FluxP {
  T gamm1, alf_l, lhs_omga, peff, tiny;
};
template <typename T>
__device__ __forceinline__ FluxP<T> flux_params(const Params &P) {
  return FluxP<T>{(T)P.gamm1, (T)P.alf_l, (T)P.lhs_omga, (T)P.peff, (T)kTiny};
}

// RoeFlux_noprec serial body (cal_flux.cpp:676-834) for one face with
// first-order face states ql = q[c1], qr = q[c2]; includes the 0.5*area
// factor.  ht_l / ht_r come precomputed from the cell records.
template <typename T>
__device__ __forceinline__ void roe_flux_t(const T *ql, const T *qr, T areax, T areay, T areaz,
                                           T area, const FluxP<T> &P, T *flux) {
  using N = Num<T>;
  const T ht_l = ql[Q_HT], ht_r = qr[Q_HT];
  const T vn_l = areax * ql[1] + areay * ql[2] + areaz * ql[3];
  const T vn_r = areax * qr[1] + areay * qr[2] + areaz * qr[3];
  T tmp0 = vn_l * ql[0];
  T tmp1 = vn_r * qr[0];
  T f0 = tmp0 + tmp1;
  T f1 = tmp0 * ql[1] + areax * ql[4] + tmp1 * qr[1] + areax * qr[4];
  T f2 = tmp0 * ql[2] + areay * ql[4] + tmp1 * qr[2] + areay * qr[4];
  T f3 = tmp0 * ql[3] + areaz * ql[4] + tmp1 * qr[3] + areaz * qr[4];
  T f4 = ht_l * vn_l + ht_r * vn_r;

  tmp0 = N::sqrt_(N::div(qr[0], ql[0]));
  tmp1 = N::div(T(1.0), T(1.0) + tmp0);
  const T rho_a = N::sqrt_(qr[0] * ql[0]);
  const T u_a = (ql[1] + qr[1] * tmp0) * tmp1;
  const T v_a = (ql[2] + qr[2] * tmp0) * tmp1;
  const T w_a = (ql[3] + qr[3] * tmp0) * tmp1;
  const T vn_a = u_a * areax + v_a * areay + w_a * areaz;
  const T h_a = (N::div(ht_l, ql[0]) + N::div(ht_r, qr[0]) * tmp0) * tmp1;

  const T q2 = T(0.5) * (u_a * u_a + v_a * v_a + w_a * w_a);
  T c2_a = P.gamm1 * (h_a - q2);
  c2_a = fabs(c2_a);
  const T c_a = N::sqrt_(c2_a);

  T eigv1 = fabs(vn_a);
  T eigv2 = fabs(vn_a + c_a);
  T eigv3 = fabs(vn_a - c_a);

  const T spectral = fabs(u_a) + fabs(v_a) + fabs(w_a) + c_a;
  const T epsaa = P.alf_l * spectral;
  const T epsbb = N::div(T(0.25), (epsaa < P.tiny) ? P.tiny : epsaa);  // smax(epsaa, tiny)
  const T epscc = T(2.0) * epsaa;
  if (eigv1 < epscc) eigv1 = eigv1 * eigv1 * epsbb + epsaa;
  if (eigv2 < epscc) eigv2 = eigv2 * eigv2 * epsbb + epsaa;
  if (eigv3 < epscc) eigv3 = eigv3 * eigv3 * epsbb + epsaa;

  const T drho = qr[0] - ql[0];
  const T du = qr[1] - ql[1];
  const T dv = qr[2] - ql[2];
  const T dw = qr[3] - ql[3];
  const T dp = qr[4] - ql[4];
  const T dvn = vn_r - vn_l;
  const T dq2 = u_a * du + v_a * dv + w_a * dw;

  tmp0 = N::div(dp, c2_a);
  tmp1 = N::div(rho_a * dvn, c_a);
  const T alpha1 = (drho - tmp0) * eigv1;
  const T alpha2 = T(0.5) * (tmp0 + tmp1) * eigv2;
  const T alpha3 = T(0.5) * (tmp0 - tmp1) * eigv3;

  tmp0 = alpha1 + alpha2 + alpha3;
  tmp1 = eigv1 * rho_a;
  const T tmp2 = -tmp1 * dvn + (alpha2 - alpha3) * c_a;
  f0 -= tmp0;
  f1 -= tmp0 * u_a + tmp1 * du + tmp2 * areax;
  f2 -= tmp0 * v_a + tmp1 * dv + tmp2 * areay;
  f3 -= tmp0 * w_a + tmp1 * dw + tmp2 * areaz;
  f4 -= alpha1 * q2 + (alpha2 + alpha3) * h_a + tmp1 * dq2 + tmp2 * vn_a;

  const T half = T(0.5) * area;
  flux[0] = f0 * half;
  flux[1] = f1 * half;
  flux[2] = f2 * half;
  flux[3] = f3 * half;
  flux[4] = f4 * half;
}

__device__ __forceinline__ void roe_flux(const double *ql, const double *qr, double areax,
                                         double areay, double areaz, double area,
                                         const Params &P, double *flux) {
  roe_flux_t<double>(ql, qr, areax, areay, areaz, area, flux_params<double>(P), flux);
}

// Correctly rounded a / b from y = RN(1 / b), for a divisor known before
// the dividend (the LU-SGS diagonal): the quotient's dependent chain is one
// product and four fused multiply-adds instead of a division.  Markstein's
// theorem (P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990): for y within
// half an ulp of 1/b and q within one ulp of a/b, r = a - b q is exact and
// RN(q + r y) = RN(a / b).  q0 = RN(a y) is within two ulps; one correction
// step makes it faithful, the second rounds correctly.  Exponents outside
// [2^-500, 2^500] (zeros, subnormals, overflow risks, non-finite values)
// take the division itself.
__device__ __forceinline__ double div_by_recip(double a, double b, double y) {
  const int ea = (__double2hiint(a) >> 20) & 0x7FF;
  const int eb = (__double2hiint(b) >> 20) & 0x7FF;
  if (ea < 523 || ea > 1523 || eb < 523 || eb > 1523) return a / b;
  const double q0 = __dmul_rn(a, y);
  const double r0 = __fma_rn(-b, q0, a);
  const double q1 = __fma_rn(r0, y, q0);
  const double r1 = __fma_rn(-b, q1, a);
  return __fma_rn(r1, y, q1);
}

// Branch-free forms of the correctly rounded reciprocal and quotient, so
// that the divisions of a cell's several records (and the five components'
// quotients) can overlap instead of running one after another.
//
// rcp_rn_fast(b) = RN(1 / b) without a division: a single-precision seed
// (hardware approximate reciprocal of b rounded to single, relative error
// below 2^-22) refined by Newton-Raphson steps on the FMA -- e = 1 - b y is
// exact once y is close, y' = y + y e squares the relative error (2^-44,
// then below half an ulp) -- and a final step of the same form, which for a
// reciprocal within one ulp rounds correctly (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990) except when the significand of b is all ones.  ok is
// false for that significand and outside the window 2^+-120 (zeros,
// subnormals, non-finite values): the caller then takes 1 / b.
__device__ __forceinline__ double rcp_rn_fast(double b, bool &ok) {
  const int hb = __double2hiint(b);
  const int eb = (hb >> 20) & 0x7FF;
  ok = eb > 1023 - 120 && eb < 1023 + 120 &&
       !((hb & 0xFFFFF) == 0xFFFFF && (unsigned)__double2loint(b) == 0xFFFFFFFFu);
  const float bf = __double2float_rn(b);
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(bf));
  double y = (double)r;
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  return __fma_rn(y, e, y);
}
// The quotient steps of div_by_recip without its branch: ok is false when
// an exponent lies outside [2^-500, 2^500]; the caller then takes a / b.
__device__ __forceinline__ double div_recip_fast(double a, double b, double y, bool &ok) {
  const int ea = (__double2hiint(a) >> 20) & 0x7FF;
  const int eb = (__double2hiint(b) >> 20) & 0x7FF;
  ok = ea >= 523 && ea <= 1523 && eb >= 523 && eb <= 1523;
  const double q0 = __dmul_rn(a, y);
  const double r0 = __fma_rn(-b, q0, a);
  const double q1 = __fma_rn(r0, y, q0);
  const double r1 = __fma_rn(-b, q1, a);
  return __fma_rn(r1, y, q1);
}

// a / b for b > 0 with y = rcp_rn_fast(b): a zero a is its own quotient
// (with its sign); otherwise div_recip_fast, which clears ok outside its
// window (the caller then divides).
__device__ __forceinline__ double quot_pos(double a, double b, double y, bool &ok) {
  bool okq;
  const double q = div_recip_fast(a, b, y, okq);
  if (a == 0.0) return a;
  ok = ok && okq;
  return q;
}

// FluxLUSGS3D (forward_lusgs.cpp:1271-1324) with the neighbour's sound speed
// and conserved energy taken from its record (same expressions), in two
// parts: what the neighbour's state and the face give, which an LU-SGS sweep
// evaluates while it still waits for the neighbour's increment, and the rest.
template <typename T>
struct LusgsPre {
  T Q0, Q1, Q2, Q3, Q4, vq, eig, f1, f2, f3, f4;
};

template <typename T>
__device__ __forceinline__ LusgsPre<T> flux_lusgs_pre(const T *q, T nx, T ny, T nz,
                                                      const FluxP<T> &P) {
  LusgsPre<T> a;
  a.Q0 = q[0];
  a.Q1 = q[0] * q[1];
  a.Q2 = q[0] * q[2];
  a.Q3 = q[0] * q[3];
  a.Q4 = q[Q_E];
  const T p = q[4];
  const T v_n = q[1] * nx + q[2] * ny + q[3] * nz;
  T eig = fabs(v_n) + q[Q_A];
  eig *= P.lhs_omga;
  a.eig = eig;
  const T peff = P.peff;
  a.f1 = -a.Q1 * v_n - p * nx;
  a.f2 = -a.Q2 * v_n - p * ny;
  a.f3 = -a.Q3 * v_n - p * nz;
  a.f4 = -(a.Q4 + p + peff) * v_n;
  a.vq = v_n * q[0];
  return a;
}

template <typename T>
__device__ __forceinline__ void flux_lusgs_fin(const LusgsPre<T> &a, const T *DQ, T nx, T ny,
                                               T nz, const FluxP<T> &P, T *flux) {
  using N = Num<T>;
  const T gam1 = P.gamm1;
  const T peff = P.peff;
  const T Q0 = a.Q0 + DQ[0];
  const T Q1 = a.Q1 + DQ[1];
  const T Q2 = a.Q2 + DQ[2];
  const T Q3 = a.Q3 + DQ[3];
  const T Q4 = a.Q4 + DQ[4];
  const T rv2 = N::div(T(0.5) * (Q1 * Q1 + Q2 * Q2 + Q3 * Q3), Q0);
  const T p = gam1 * (Q4 - rv2);
  const T f0 = DQ[1] * nx + DQ[2] * ny + DQ[3] * nz;
  T v_n = a.vq;
  v_n += f0;
  v_n = N::div(v_n, Q0);
  const T f1 = a.f1 + (Q1 * v_n + p * nx);
  const T f2 = a.f2 + (Q2 * v_n + p * ny);
  const T f3 = a.f3 + (Q3 * v_n + p * nz);
  const T f4 = a.f4 + ((Q4 + p + peff) * v_n);
  flux[0] = f0 - a.eig * DQ[0];
  flux[1] = f1 - a.eig * DQ[1];
  flux[2] = f2 - a.eig * DQ[2];
  flux[3] = f3 - a.eig * DQ[3];
  flux[4] = f4 - a.eig * DQ[4];
}

// flux_lusgs_fin<double> with its two divisions by Q0 as rcp_rn_fast +
// div_recip_fast: the same bits when ok comes back true (else the caller
// takes flux_lusgs_fin).
__device__ __forceinline__ void flux_lusgs_fin_fast(const LusgsPre<double> &a, const double *DQ,
                                                    double nx, double ny, double nz,
                                                    const FluxP<double> &P, double *flux,
                                                    bool &ok) {
  const double gam1 = P.gamm1;
  const double peff = P.peff;
  const double Q0 = a.Q0 + DQ[0];
  const double Q1 = a.Q1 + DQ[1];
  const double Q2 = a.Q2 + DQ[2];
  const double Q3 = a.Q3 + DQ[3];
  const double Q4 = a.Q4 + DQ[4];
  bool ok0, ok1, ok2;
  const double y = rcp_rn_fast(Q0, ok0);
  const double rv2 = div_recip_fast(0.5 * (Q1 * Q1 + Q2 * Q2 + Q3 * Q3), Q0, y, ok1);
  const double p = gam1 * (Q4 - rv2);
  const double f0 = DQ[1] * nx + DQ[2] * ny + DQ[3] * nz;
  double v_n = a.vq;
  v_n += f0;
  v_n = div_recip_fast(v_n, Q0, y, ok2);
  ok = ok0 && ok1 && ok2;
  const double f1 = a.f1 + (Q1 * v_n + p * nx);
  const double f2 = a.f2 + (Q2 * v_n + p * ny);
  const double f3 = a.f3 + (Q3 * v_n + p * nz);
  const double f4 = a.f4 + ((Q4 + p + peff) * v_n);
  flux[0] = f0 - a.eig * DQ[0];
  flux[1] = f1 - a.eig * DQ[1];
  flux[2] = f2 - a.eig * DQ[2];
  flux[3] = f3 - a.eig * DQ[3];
  flux[4] = f4 - a.eig * DQ[4];
}

template <typename T>
__device__ __forceinline__ void flux_lusgs_t(const T *q, const T *DQ, T nx, T ny, T nz,
                                             const FluxP<T> &P, T *flux) {
  flux_lusgs_fin(flux_lusgs_pre(q, nx, ny, nz, P), DQ, nx, ny, nz, P, flux);
}

__device__ __forceinline__ void flux_lusgs(const double *q, const double *DQ, double nx, double ny,
                                           double nz, const Params &P, double *flux) {
  flux_lusgs_t<double>(q, DQ, nx, ny, nz, flux_params<double>(P), flux);
}

// Mixed form of RoeFlux_noprec: the central part (the two one-sided fluxes)
// in FP64 with the FP64 expressions above, so that a closed cell of uniform
// state still sums to zero; the Roe average, eigenvalues and dissipation (the
// square roots and divisions) in FP32 from state differences formed in FP64,
// so that the FP32 rounding scales with the jump across the face.
__device__ __forceinline__ void roe_flux_mx(const double *ql, const double *qr, double areax,
                                           double areay, double areaz, double area,
                                           const Params &P, const FluxP<float> &F,
                                           double *flux) {
  const double vn_l = areax * ql[1] + areay * ql[2] + areaz * ql[3];
  const double vn_r = areax * qr[1] + areay * qr[2] + areaz * qr[3];
  double tmp0 = vn_l * ql[0];
  double tmp1 = vn_r * qr[0];
  double f0 = tmp0 + tmp1;
  double f1 = tmp0 * ql[1] + areax * ql[4] + tmp1 * qr[1] + areax * qr[4];
  double f2 = tmp0 * ql[2] + areay * ql[4] + tmp1 * qr[2] + areay * qr[4];
  double f3 = tmp0 * ql[3] + areaz * ql[4] + tmp1 * qr[3] + areaz * qr[4];
  double f4 = ql[Q_HT] * vn_l + qr[Q_HT] * vn_r;

  const float nx = (float)areax, ny = (float)areay, nz = (float)areaz;
  const float rl = (float)ql[0], rr = (float)qr[0];
  const float t0 = sqrtf(__fdividef(rr, rl));
  const float t1 = __fdividef(1.0f, 1.0f + t0);
  const float rho_a = sqrtf(rr * rl);
  const float u_a = ((float)ql[1] + (float)qr[1] * t0) * t1;
  const float v_a = ((float)ql[2] + (float)qr[2] * t0) * t1;
  const float w_a = ((float)ql[3] + (float)qr[3] * t0) * t1;
  const float vn_a = u_a * nx + v_a * ny + w_a * nz;
  const float h_a =
      (__fdividef((float)ql[Q_HT], rl) + __fdividef((float)qr[Q_HT], rr) * t0) * t1;
  const float q2 = 0.5f * (u_a * u_a + v_a * v_a + w_a * w_a);
  const float c2_a = fabsf(F.gamm1 * (h_a - q2));
  const float c_a = sqrtf(c2_a);
  float eigv1 = fabsf(vn_a);
  float eigv2 = fabsf(vn_a + c_a);
  float eigv3 = fabsf(vn_a - c_a);
  const float spectral = fabsf(u_a) + fabsf(v_a) + fabsf(w_a) + c_a;
  const float epsaa = F.alf_l * spectral;
  const float epsbb = __fdividef(0.25f, fmaxf(epsaa, F.tiny));
  const float epscc = 2.0f * epsaa;
  if (eigv1 < epscc) eigv1 = eigv1 * eigv1 * epsbb + epsaa;
  if (eigv2 < epscc) eigv2 = eigv2 * eigv2 * epsbb + epsaa;
  if (eigv3 < epscc) eigv3 = eigv3 * eigv3 * epsbb + epsaa;
  const float drho = (float)(qr[0] - ql[0]);
  const float du = (float)(qr[1] - ql[1]);
  const float dv = (float)(qr[2] - ql[2]);
  const float dw = (float)(qr[3] - ql[3]);
  const float dp = (float)(qr[4] - ql[4]);
  const float dvn = (float)(vn_r - vn_l);
  const float dq2 = u_a * du + v_a * dv + w_a * dw;
  const float a0 = __fdividef(dp, c2_a);
  const float a1 = __fdividef(rho_a * dvn, c_a);
  const float alpha1 = (drho - a0) * eigv1;
  const float alpha2 = 0.5f * (a0 + a1) * eigv2;
  const float alpha3 = 0.5f * (a0 - a1) * eigv3;
  const float s0 = alpha1 + alpha2 + alpha3;
  const float s1 = eigv1 * rho_a;
  const float s2 = -s1 * dvn + (alpha2 - alpha3) * c_a;
  f0 -= (double)s0;
  f1 -= (double)(s0 * u_a + s1 * du + s2 * nx);
  f2 -= (double)(s0 * v_a + s1 * dv + s2 * ny);
  f3 -= (double)(s0 * w_a + s1 * dw + s2 * nz);
  f4 -= (double)(alpha1 * q2 + (alpha2 + alpha3) * h_a + s1 * dq2 + s2 * vn_a);
  const double half = 0.5 * area;
  flux[0] = f0 * half;
  flux[1] = f1 * half;
  flux[2] = f2 * half;
  flux[3] = f3 * half;
  flux[4] = f4 * half;
}

// Mixed form of FluxLUSGS3D: F(Q + DQ) - F(Q) - eig DQ (forward_lusgs.cpp
// :1271-1324) in FP32, written in difference form so that every term is
// formed from DQ directly: a zero increment gives exactly zero and the
// rounding scales with the increment instead of with F.  With m = rho vn and
// M = rho (u, v, w): vn' - vn = (DQ.n - vn DQ0) / Q0', rv2' - rv2 = (rho u.dM
// + |dM|^2 / 2 - rho |u|^2 DQ0 / 2) / Q0', p' - p = gam1 (DQ4 - (rv2' - rv2)).
__device__ __forceinline__ void flux_lusgs_diff(const float *q, const float *DQ, float nx,
                                               float ny, float nz, const FluxP<float> &P,
                                               float *flux) {
  const float rho = q[0], u = q[1], v = q[2], w = q[3];
  const float vn = u * nx + v * ny + w * nz;
  const float eig = (fabsf(vn) + q[Q_A]) * P.lhs_omga;
  const float rq0n = __fdividef(1.0f, rho + DQ[0]);
  const float f0 = DQ[1] * nx + DQ[2] * ny + DQ[3] * nz;
  const float dvn = (f0 - vn * DQ[0]) * rq0n;
  const float vnn = vn + dvn;
  const float udm = u * DQ[1] + v * DQ[2] + w * DQ[3];
  const float dm2 = DQ[1] * DQ[1] + DQ[2] * DQ[2] + DQ[3] * DQ[3];
  const float uu = u * u + v * v + w * w;
  const float drv2 = (rho * udm + 0.5f * dm2 - 0.5f * rho * uu * DQ[0]) * rq0n;
  const float dp = P.gamm1 * (DQ[4] - drv2);
  const float H = q[Q_E] + q[4] + P.peff;
  const float dH = DQ[4] + dp;
  flux[0] = f0 - eig * DQ[0];
  flux[1] = rho * u * dvn + DQ[1] * vnn + dp * nx - eig * DQ[1];
  flux[2] = rho * v * dvn + DQ[2] * vnn + dp * ny - eig * DQ[2];
  flux[3] = rho * w * dvn + DQ[3] * vnn + dp * nz - eig * DQ[3];
  flux[4] = H * dvn + dH * vnn - eig * DQ[4];
}

// DQ_limit == 2 positivity limiter (forward_lusgs.cpp:939-973, :1184-1218);
// vv = u^2 + v^2 + w^2 of the cell, which the sweeps form before the
// increment is known.
__device__ __forceinline__ void dq_limit_vv(const double *q, double vv, double *d,
                                            const Params &P) {
#pragma unroll
  for (int stage = 0; stage < 3; stage++) {
    double dp = d[4] + 0.5 * d[0] * vv - (d[1] * q[1] + d[2] * q[2] + d[3] * q[3]);
    dp *= P.gamm1;
    if ((q[0] + d[0]) < P.rho_min || (q[0] + d[0]) > P.rho_max || (q[4] + dp) < P.p_min ||
        (q[4] + dp) > P.p_max) {
      if (stage < 2) {
#pragma unroll
        for (int k = 0; k < 5; k++) d[k] *= 0.1;
      } else {
#pragma unroll
        for (int k = 0; k < 5; k++) d[k] = 0.0;
      }
    } else {
      break;  // d unchanged: the later stages repeat this test and pass too
    }
  }
}

__device__ __forceinline__ void dq_limit(const double *q, double *d, const Params &P) {
  dq_limit_vv(q, q[1] * q[1] + q[2] * q[2] + q[3] * q[3], d, P);
}

// UpdateFlowField3D_CFL3d (forward_lusgs.cpp:1335-1488) for one cell; q is
// updated in place (primitive part).
__device__ __forceinline__ void update_cell(double *q, const double *DQ, const Params &P) {
  const double gam1 = P.gamm1;
  const double p00 = P.p_bar;
  const double alpq = -0.2;
  const double phiq = 1. / 0.5;
  const double betq = 1.0 + alpq * phiq;
  double rhot = q[0];
  double ru = rhot * q[1];
  double rv = rhot * q[2];
  double rw = rhot * q[3];
  double re = q[4] / gam1 + 0.5 * rhot * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  rhot += DQ[0];
  ru += DQ[1];
  rv += DQ[2];
  rw += DQ[3];
  re += DQ[4];
  const double rhotr = 1. / (rhot + kTiny);
  const double u = ru * rhotr, v = rv * rhotr, w = rw * rhotr;
  double rho_del = DQ[0];
  const double rho_rat = rho_del / q[0];
  if (rho_rat < alpq) rho_del /= betq + fabs(rho_rat) * phiq;
  double rho = q[0] + rho_del;
  rho = smax(rho, P.rho_min);
  rho = smin(rho, P.rho_max);
  const double ptmp = gam1 * (re - 0.5 * (u * u + v * v + w * w) * rho);
  double p_del = ptmp - q[4];
  const double p_rat = p_del / (q[4] + p00);
  if (p_rat < alpq) p_del /= betq + fabs(p_rat) * phiq;
  double p = q[4] + p_del;
  p = smax(p, P.p_min);
  p = smin(p, P.p_max);
  q[0] = rho;
  q[1] = u;
  q[2] = v;
  q[3] = w;
  q[4] = p;
}

// LimitTimeStep's local CFL (compute_timestep.cpp:881-906).
__device__ __forceinline__ double local_cfl_pb(double p, int det, double cfl, double cfl_min,
                                               double p_break, double p_min) {
  double cfl_tmp;
  if (p > p_break)
    cfl_tmp = cfl;
  else if (p < p_min)
    cfl_tmp = cfl_min;
  else
    cfl_tmp = (p - p_min) / (p_break - p_min) * (cfl - cfl_min) + cfl_min;
  if (!det) cfl_tmp = cfl_min;
  return cfl_tmp;
}
__device__ __forceinline__ double local_cfl(double p, int det, double cfl, double cfl_min,
                                            const Params &P) {
  return local_cfl_pb(p, det, cfl, cfl_min, P.p_break, P.p_min);
}

// Order-preserving bit pattern of a non-negative double for atomic max/min.
__device__ __forceinline__ unsigned long long dbits(double x) {
  return static_cast<unsigned long long>(__double_as_longlong(x));
}

// ---- readiness of LU-SGS increments -----------------------------------------
// The forward and backward increments live in separate arrays whose interior
// rows hold this signalling-NaN pattern until written.  IEEE arithmetic only
// produces quiet NaNs, so a computed increment never equals it, and every
// 8-byte word is written and read atomically: a reader may use a record as
// soon as none of its five words is the sentinel, with no flag or fence.
constexpr unsigned long long kSentinelBits = 0x7FF40000DEADBEEFull;

__device__ __forceinline__ bool is_sentinel(double x) {
  return (unsigned long long)__double_as_longlong(x) == kSentinelBits;
}

// Five words of a record straight from L2 (the point of coherence), never a
// stale L1 line; asm volatile keeps the loads inside a polling loop.
__device__ __forceinline__ void load_rec5_l2(const double *rec, double *d) {
  double a0, a1, b0, b1, e0;
  asm volatile("ld.global.cg.v2.f64 {%0, %1}, [%2];" : "=d"(a0), "=d"(a1) : "l"(rec) : "memory");
  asm volatile("ld.global.cg.v2.f64 {%0, %1}, [%2];" : "=d"(b0), "=d"(b1) : "l"(rec + 2) : "memory");
  asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(e0) : "l"(rec + 4) : "memory");
  d[0] = a0; d[1] = a1; d[2] = b0; d[3] = b1; d[4] = e0;
}

__device__ __forceinline__ bool rec5_ready(const double *d) {
  return !(is_sentinel(d[0]) || is_sentinel(d[1]) || is_sentinel(d[2]) || is_sentinel(d[3]) ||
           is_sentinel(d[4]));
}

__device__ __forceinline__ int ld_relaxed(const int *p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Cycles a lane may wait for one neighbour (~2 s at 1.9 GHz) before it gives
// up, records the failure in *err and lets the sweep run to its end.
constexpr long long kSpinCycles = 4000000000LL;

// Bounded wait for a neighbour increment produced on another SM: poll the
// record in L2 until none of its words is the sentinel.  Returns false when
// it gave up (or another lane did); d then holds whatever was read.
__device__ __forceinline__ bool wait_rec(const double *rec, double *d, int *err,
                                         long long max_cycles) {
  load_rec5_l2(rec, d);
  if (rec5_ready(d)) return true;
  const long long t0 = clock64();
  // the error word is read on every poll: polling faster (reading it every
  // 16th poll, two polls in flight, one word per poll) or backing off with
  // __nanosleep each measured slower on the 64^3 x 6 cube
  int polls = 0;
  for (;;) {
    if (polls > 64) __nanosleep(64);
    ++polls;
    load_rec5_l2(rec, d);
    const int gave_up = ld_relaxed(err);  // in flight beside the record's words
    if (rec5_ready(d)) return true;
    if (gave_up) return false;  // another lane gave up: finish quickly
    if (clock64() - t0 > max_cycles) {
      atomicExch(err, 1);
      return false;
    }
  }
}

__device__ __forceinline__ void store_sentinel(double *dq8, int64_t c) {
  const double s = __longlong_as_double((long long)kSentinelBits);
  double2 *p = reinterpret_cast<double2 *>(dq8 + c * Q_STRIDE);
  p[0] = make_double2(s, s);
  p[1] = make_double2(s, s);
  p[2] = make_double2(s, 0.0);
}

}  // namespace mfg
