// Curvilinear (topography) velocity and stress kernels of the top grid.
#pragma once

#include <cuda_runtime.h>

#include "awp_common.h"

struct TopoArgs {
  // wavefield and memory variables (padded layout of awp_common.h)
  float *u1, *v1, *w1, *xx, *yy, *zz, *xy, *xz, *yz;
  float *r1, *r2, *r3, *r4, *r5, *r6;
  // media (rho, 1/lambda, 1/mu, 1/Qp, 1/Qs) and the sponge
  const float *d1, *lam, *mu, *qp, *qs, *dcrjx, *dcrjy, *dcrjz;
  // metrics: 2-D f arrays (ld = ny + 4 + 2 ngsl + 2 align) and 1-D g arrays
  const float *f, *f_1, *f_2, *f_c, *f1_1, *f1_2, *f1_c, *f2_1, *f2_2, *f2_c;
  const float *g, *g_c, *g3, *g3_c;
  AwpTexture tex;
  float coeff[16];
  int nx, ny, nz, slice, yline, fld;
  float nu;              // velocity: dt/h (topo_t.dth)
  float DT, dth, dh1;    // stress: (dt/h)*h, DT/h, 1/h (topo_set_constants)
  float qthr;            // smallest float x with 1/(double)x <= 200 (Q(f) switch)
  int s_i, e_i, s_j, e_j;  // stress window, relative indices, ends exclusive
};

// dtopo_vel_111_unroll + dtopo_vel_112 (velocity_unroll.cu, optimized_velocity.cu:1040-1629)
cudaError_t awp_launch_topo_velocity(const TopoArgs& a, cudaStream_t st);
// dtopo_str_111 + dtopo_str_112 (kernels/stress_attenuation.cu:73-1415)
cudaError_t awp_launch_topo_stress(const TopoArgs& a, bool elastic, cudaStream_t st);
