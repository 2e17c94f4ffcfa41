// Per-cell arithmetic shared by the stencil kernels (awp_kernels.cu, awp_tma.cu).
#pragma once

#include <math.h>

// Q(f) weight (kernel.cu:974-1040).  The reference switches on
// 1./(q*2.0) <= 200.0 evaluated in double; for float q that is exactly
// (2q >= qthr) for positive q, true for negative q and -0, false for +0/NaN.
__device__ __forceinline__ float awp_qf_weight(float q, float wwo, float c0, float c1,
                                           float qthr) {
  const float x = 2.0f * q;
  const bool low = (x >= qthr) || (x < 0.f) || (x == 0.f && signbit(x));
  float w;
  if (low) {
    const double xd = 2.0 * (double)q;
    w = (float)((double)c0 * xd * xd + (double)c1 * xd);
  } else {
    w = 2.0f * wwo * q;
  }
  return w / wwo;
}

// One stress/memory-variable update of a cell (dstrqc, kernel.cu:1114-1179),
// the state passed in and out through registers.
template <bool ELASTIC>
__device__ __forceinline__ void awp_stress_update(float (&sg)[6], float (&rr)[6], float xl, float xm,
                                              float xmu1, float xmu2, float xmu3, float h,
                                              float h1, float h2, float h3, float qpa,
                                              float vx1, float f_vx1, float f_vx2,
                                              float f_wwo, float DT, float dcrj,
                                              const float (&d)[9]) {
  // d: vs1 vs2 vs3 (normal), xy pair, xz pair, yz pair
  const float vs1 = d[0], vs2 = d[1], vs3 = d[2];
  float tmp = xl * (vs1 + vs2 + vs3);
  const float a1 = qpa * (vs1 + vs2 + vs3);
  tmp = tmp + DT * a1;
  if (ELASTIC) {
    sg[0] = (sg[0] + tmp - xm * (vs2 + vs3)) * dcrj;
    sg[1] = ((sg[1] + tmp - xm * (vs1 + vs3)) * dcrj) * dcrj;
    sg[2] = ((sg[2] + tmp - xm * (vs1 + vs2)) * dcrj) * dcrj;
    sg[3] = (sg[3] + xmu1 * (d[3] + d[4])) * dcrj;
    sg[4] = (sg[4] + xmu2 * (d[5] + d[6])) * dcrj;
    sg[5] = (sg[5] + xmu3 * (d[7] + d[8])) * dcrj;
    return;
  }
  float f_r, f_rtmp, t;
  f_r = rr[0];
  f_rtmp = -h * (vs2 + vs3) + a1;
  t = sg[0] + tmp - xm * (vs2 + vs3) + vx1 * f_r;
  rr[0] = f_vx2 * f_r + f_wwo * f_rtmp;
  f_rtmp = f_rtmp * (f_wwo - 1) + f_vx2 * f_r * (1 - f_vx1);
  sg[0] = (t + DT * f_rtmp) * dcrj;

  f_r = rr[1];
  f_rtmp = -h * (vs1 + vs3) + a1;
  t = (sg[1] + tmp - xm * (vs1 + vs3) + vx1 * f_r) * dcrj;
  rr[1] = f_vx2 * f_r + f_wwo * f_rtmp;
  f_rtmp = f_rtmp * (f_wwo - 1) + f_vx2 * f_r * (1 - f_vx1);
  sg[1] = (t + DT * f_rtmp) * dcrj;

  f_r = rr[2];
  f_rtmp = -h * (vs1 + vs2) + a1;
  t = (sg[2] + tmp - xm * (vs1 + vs2) + vx1 * f_r) * dcrj;
  rr[2] = f_vx2 * f_r + f_wwo * f_rtmp;
  f_rtmp = f_rtmp * (f_wwo - 1) + f_vx2 * f_r * (1 - f_vx1);
  sg[2] = (t + DT * f_rtmp) * dcrj;

  f_r = rr[3];
  f_rtmp = h1 * (d[3] + d[4]);
  t = sg[3] + xmu1 * (d[3] + d[4]) + vx1 * f_r;
  rr[3] = f_vx2 * f_r + f_wwo * f_rtmp;
  f_rtmp = f_rtmp * (f_wwo - 1) + f_vx2 * f_r * (1 - f_vx1);
  sg[3] = (t + DT * f_rtmp) * dcrj;

  f_r = rr[4];
  f_rtmp = h2 * (d[5] + d[6]);
  t = sg[4] + xmu2 * (d[5] + d[6]) + vx1 * f_r;
  rr[4] = f_vx2 * f_r + f_wwo * f_rtmp;
  f_rtmp = f_rtmp * (f_wwo - 1) + f_vx2 * f_r * (1 - f_vx1);
  sg[4] = (t + DT * f_rtmp) * dcrj;

  f_r = rr[5];
  f_rtmp = h3 * (d[7] + d[8]);
  t = sg[5] + xmu3 * (d[7] + d[8]) + vx1 * f_r;
  rr[5] = f_vx2 * f_r + f_wwo * f_rtmp;
  f_rtmp = f_rtmp * (f_wwo - 1) + f_vx2 * f_r * (1 - f_vx1);
  sg[5] = (t + DT * f_rtmp) * dcrj;
}

// TY = 8: 256 threads held to 128 registers (2 CTAs / SM);
// TY = 4: 128 threads without a register cap (3 CTAs / SM).
