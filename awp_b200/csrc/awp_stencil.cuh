// Per-cell arithmetic shared by the stencil kernels (awp_kernels.cu, awp_tma.cu).
#pragma once

#include <math.h>

// Q(f) weight (kernel.cu:974-1040) before its division by wwo.  The reference
// switches on 1./(q*2.0) <= 200.0 evaluated in double; for float q that is
// exactly (2q >= qthr) for positive q, true for negative q and -0, false for
// +0/NaN.  The reference evaluates the polynomial c0 (2q)^2 + c1 (2q) in
// double; here it is float (the two differ by about one float ulp, far below
// the 1e-5 parity bar, at a fraction of the instructions).
__device__ __forceinline__ float awp_qf_weight_num(float q, float wwo, float c0, float c1,
                                               float qthr) {
  const float x = __fmul_rn(2.0f, q);
  const bool low = (x >= qthr) || (x < 0.f) || (x == 0.f && signbit(x));
  return low ? __fmaf_rn(__fmul_rn(c0, x), x, __fmul_rn(c1, x))
             : __fmul_rn(__fmul_rn(2.0f, wwo), q);
}

__device__ __forceinline__ float awp_qf_weight(float q, float wwo, float c0, float c1,
                                           float qthr) {
  return awp_qf_weight_num(q, wwo, c0, c1, qthr) / wwo;  // the build's division mode
}

// ---------------------------------------------------------------------------
// Rounding discipline.  The per-cell arithmetic below is written with explicit
// rounding intrinsics, so every kernel family that calls it (read-only-path,
// TMA-pipelined, fused) produces the same bits: left to the compiler, the
// contraction of a*b + c into an FMA is chosen per kernel and differs between
// kernels that spell the same expression.  The association follows the
// reference's left-to-right order (kernel.cu:222-253, 1041-1086).
// ---------------------------------------------------------------------------

// c1*(a - b) + c2*(c - d): one 4th-order staggered difference.
__device__ __forceinline__ float awp_d4(float c1, float c2, float a, float b, float c, float d) {
  return __fmaf_rn(c2, __fsub_rn(c, d), __fmul_rn(c1, __fsub_rn(a, b)));
}

// Velocity update of dvelcx (kernel.cu:222-253):
// (v + fd*(c1*x0 + c2*x1 + c1*y0 + c2*y1 + c1*z0 + c2*z1)) * dcrj, where
// x0..z1 are the six differences of the three stress derivatives.
__device__ __forceinline__ float awp_vel_update(float v, float fd, float c1, float c2, float x0,
                                                float x1, float y0, float y1, float z0,
                                                float z1, float dcrj) {
  float s = __fmul_rn(c1, x0);
  s = __fmaf_rn(c2, x1, s);
  s = __fmaf_rn(c1, y0, s);
  s = __fmaf_rn(c2, y1, s);
  s = __fmaf_rn(c1, z0, s);
  s = __fmaf_rn(c2, z1, s);
  return __fmul_rn(__fmaf_rn(fd, s, v), dcrj);
}

// dth / (0.25 * (a + b + c + d)): the density-averaged velocity factor
// (kernel.cu:218-221).
__device__ __forceinline__ float awp_vel_factor(float dth, float a, float b, float c, float d) {
  return dth / __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d));
}

// Material coefficients of one stress cell (kernel.cu:962-1040, 1041-1070).
struct AwpStrCoef {
  float xl, xm, xmu1, xmu2, xmu3, h, h1, h2, h3, qpa, vx1;
};

// L8, M8, QP8, QS8: the eight-cell sums of lam, mu, qp, qs in the reference's
// order; mu0 = mu(i,j,k), muk = mu(i,j,k-1), muj = mu(i,j-1,k), mui = mu(i+1,j,k)
// (same for qs).  The reference divides in double ((float)(8.0/(double)x),
// the correctly rounded quotient); here the five harmonic-mean quotients and
// the five Q(f) weights use the hardware reciprocal (within two ulp of the
// correctly rounded value), which keeps the stress update off the division
// slow path; the parity tests hold the result to the reference build at
// relative L2 1e-5.
template <bool ELASTIC>
__device__ __forceinline__ AwpStrCoef awp_stress_coef(float L8, float M8, float mu0, float muk,
                                                      float muj, float mui, float QP8, float QS8,
                                                      float qs0, float qsk, float qsj, float qsi,
                                                      float f_vx1, float f_vx2, float f_wwo,
                                                      float cc0, float cc1, float qthr,
                                                      float dth, float dh1, float DT) {
  AwpStrCoef r;
  float xl = __fdividef(8.0f, L8);
  float xm = __fdividef(16.0f, M8);
  float xmu1 = __fdividef(2.0f, __fadd_rn(mu0, muk));
  float xmu2 = __fdividef(2.0f, __fadd_rn(mu0, muj));
  float xmu3 = __fdividef(2.0f, __fadd_rn(mu0, mui));
  xl = __fadd_rn(xl, xm);
  float h = 0.f, h1 = 0.f, h2 = 0.f, h3 = 0.f, qpa = 0.f;
  if (!ELASTIC) {
    const float iw = __fdividef(1.0f, f_wwo);
    const float qpaw =
        __fmul_rn(awp_qf_weight_num(__fmul_rn(0.0625f, QP8), f_wwo, cc0, cc1, qthr), iw);
    const float hw =
        __fmul_rn(awp_qf_weight_num(__fmul_rn(0.0625f, QS8), f_wwo, cc0, cc1, qthr), iw);
    const float h1w = __fmul_rn(
        awp_qf_weight_num(__fmul_rn(0.25f, __fadd_rn(qs0, qsk)), f_wwo, cc0, cc1, qthr), iw);
    const float h2w = __fmul_rn(
        awp_qf_weight_num(__fmul_rn(0.25f, __fadd_rn(qs0, qsj)), f_wwo, cc0, cc1, qthr), iw);
    const float h3w = __fmul_rn(
        awp_qf_weight_num(__fmul_rn(0.25f, __fadd_rn(qs0, qsi)), f_wwo, cc0, cc1, qthr), iw);
    h = __fmul_rn(__fmul_rn(-xm, hw), dh1);
    h1 = __fmul_rn(__fmul_rn(-xmu1, h1w), dh1);
    h2 = __fmul_rn(__fmul_rn(-xmu2, h2w), dh1);
    h3 = __fmul_rn(__fmul_rn(-xmu3, h3w), dh1);
    qpa = __fmul_rn(__fmul_rn(-qpaw, xl), dh1);
  }
  xm = __fmul_rn(xm, dth);
  xmu1 = __fmul_rn(xmu1, dth);
  xmu2 = __fmul_rn(xmu2, dth);
  xmu3 = __fmul_rn(xmu3, dth);
  xl = __fmul_rn(xl, dth);
  float vx1 = 0.f;
  if (!ELASTIC) {
    h = __fmul_rn(h, f_vx1);
    h1 = __fmul_rn(h1, f_vx1);
    h2 = __fmul_rn(h2, f_vx1);
    h3 = __fmul_rn(h3, f_vx1);
    qpa = __fmul_rn(qpa, f_vx1);
    xm = __fmaf_rn(DT, h, xm);
    xmu1 = __fmaf_rn(DT, h1, xmu1);
    xmu2 = __fmaf_rn(DT, h2, xmu2);
    xmu3 = __fmaf_rn(DT, h3, xmu3);
    vx1 = __fmul_rn(DT, __fmaf_rn(f_vx2, f_vx1, 1.0f));
  }
  r.xl = xl; r.xm = xm; r.xmu1 = xmu1; r.xmu2 = xmu2; r.xmu3 = xmu3;
  r.h = h; r.h1 = h1; r.h2 = h2; r.h3 = h3; r.qpa = qpa; r.vx1 = vx1;
  return r;
}

// One stress/memory-variable update of a cell (dstrqc, kernel.cu:1114-1179),
// the state passed in and out through registers.
//   sg: xx yy zz xy xz yz; rr: r1..r6
//   d:  vs1 vs2 vs3 (normal strain rates), then the xy, xz, yz difference pairs
// Memory-variable step of one component (kernel.cu:1116-1124):
//   t     = base + vx1*r                     (base: the elastic increment)
//   r'    = vx2*r + wwo*f
//   f'    = f*(wwo - 1) + vx2*r*(1 - vx1)
//   sigma = (t [* dcrj] + DT*f') * dcrj
__device__ __forceinline__ float awp_mem_step(float base, float& r, float f, float vx1,
                                              float f_vx1, float f_vx2, float f_wwo, float DT,
                                              float dcrj, bool twice) {
  const float f_r = r;
  float t = __fmaf_rn(vx1, f_r, base);
  if (twice) t = __fmul_rn(t, dcrj);
  const float vr = __fmul_rn(f_vx2, f_r);
  r = __fmaf_rn(f_wwo, f, vr);
  const float f2 = __fmaf_rn(f, __fsub_rn(f_wwo, 1.0f), __fmul_rn(vr, __fsub_rn(1.0f, f_vx1)));
  return __fmul_rn(__fmaf_rn(DT, f2, t), dcrj);
}

template <bool ELASTIC>
__device__ __forceinline__ void awp_stress_update(float (&sg)[6], float (&rr)[6],
                                                  const AwpStrCoef& q, float f_vx1, float f_vx2,
                                                  float f_wwo, float DT, float dcrj,
                                                  const float (&d)[9]) {
  const float vs1 = d[0], vs2 = d[1], vs3 = d[2];
  const float s123 = __fadd_rn(__fadd_rn(vs1, vs2), vs3);
  const float s23 = __fadd_rn(vs2, vs3), s13 = __fadd_rn(vs1, vs3), s12 = __fadd_rn(vs1, vs2);
  const float dxy = __fadd_rn(d[3], d[4]), dxz = __fadd_rn(d[5], d[6]),
              dyz = __fadd_rn(d[7], d[8]);
  const float a1 = __fmul_rn(q.qpa, s123);
  const float tmp = __fmaf_rn(DT, a1, __fmul_rn(q.xl, s123));
  // normal components: sigma + tmp - xm*(sum of the other two)
  const float b0 = __fmaf_rn(-q.xm, s23, __fadd_rn(sg[0], tmp));
  const float b1 = __fmaf_rn(-q.xm, s13, __fadd_rn(sg[1], tmp));
  const float b2 = __fmaf_rn(-q.xm, s12, __fadd_rn(sg[2], tmp));
  const float b3 = __fmaf_rn(q.xmu1, dxy, sg[3]);
  const float b4 = __fmaf_rn(q.xmu2, dxz, sg[4]);
  const float b5 = __fmaf_rn(q.xmu3, dyz, sg[5]);
  if (ELASTIC) {
    // the reference multiplies yy and zz by the sponge factor twice (kernel.cu:1130-1150)
    sg[0] = __fmul_rn(b0, dcrj);
    sg[1] = __fmul_rn(__fmul_rn(b1, dcrj), dcrj);
    sg[2] = __fmul_rn(__fmul_rn(b2, dcrj), dcrj);
    sg[3] = __fmul_rn(b3, dcrj);
    sg[4] = __fmul_rn(b4, dcrj);
    sg[5] = __fmul_rn(b5, dcrj);
    return;
  }
  sg[0] = awp_mem_step(b0, rr[0], __fmaf_rn(-q.h, s23, a1), q.vx1, f_vx1, f_vx2, f_wwo, DT, dcrj,
                       false);
  sg[1] = awp_mem_step(b1, rr[1], __fmaf_rn(-q.h, s13, a1), q.vx1, f_vx1, f_vx2, f_wwo, DT, dcrj,
                       true);
  sg[2] = awp_mem_step(b2, rr[2], __fmaf_rn(-q.h, s12, a1), q.vx1, f_vx1, f_vx2, f_wwo, DT, dcrj,
                       true);
  sg[3] = awp_mem_step(b3, rr[3], __fmul_rn(q.h1, dxy), q.vx1, f_vx1, f_vx2, f_wwo, DT, dcrj,
                       false);
  sg[4] = awp_mem_step(b4, rr[4], __fmul_rn(q.h2, dxz), q.vx1, f_vx1, f_vx2, f_wwo, DT, dcrj,
                       false);
  sg[5] = awp_mem_step(b5, rr[5], __fmul_rn(q.h3, dyz), q.vx1, f_vx1, f_vx2, f_wwo, DT, dcrj,
                       false);
}

// TY = 8: 256 threads held to 128 registers (2 CTAs / SM);
// TY = 4: 128 threads without a register cap (3 CTAs / SM).
