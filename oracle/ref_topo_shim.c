/* Test-only checker glue: drives the reference's own curvilinear topography
 * code (src/topography/{topography.c,geometry.c,velocity.cu,
 * stress_attenuation.cu}, kernels/{optimized_velocity.cu,
 * stress_attenuation.cu}, compiled in place by oracle/Makefile) for one rank
 * on the device arrays the caller owns, in pmcl3d's order:
 *   set-up  topo_init / topo_bind / topo_init_metrics / topo_init_grid /
 *           topo_init_geometry / topo_build / topo_set_constants
 *           (pmcl3d.c:1522-1548)
 *   step    topo_velocity_interior_H (pmcl3d.c:1693-1698; at one rank the
 *           front/back launchers only fill the MPI send buffers);
 *           topo_stress_interior_H, topo_stress_left_H, topo_stress_right_H
 *           (pmcl3d.c:1855-1922).
 * Nothing of the product links this file. */
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <topography/topography.h>

void topo_velocity_interior_H(topo_t *T);
void topo_velocity_front_H(topo_t *T);
void topo_velocity_back_H(topo_t *T);
void topo_stress_interior_H(topo_t *T);
void topo_stress_left_H(topo_t *T);
void topo_stress_right_H(topo_t *T);
void topo_set_constants(topo_t *T);

/* fields: rho lam mu qp coeff qs vx1 vx2 ww wwo xx yy zz xy xz yz r1..r6 u1 v1
 * w1 dcrjx dcrjy dcrjz (device pointers, 28 of them) */
void *ref_topo_create(const char *intopo, int nx, int ny, int nz, float dt, float h,
                      void **d) {
  int coord[2] = {0, 0};
  topo_t *T = (topo_t *)calloc(1, sizeof(topo_t));
  *T = topo_init(1, intopo, 0, -1, -1, -1, -1, coord, 1, 1, nx, ny, nz, dt, h, 0, 0, 0);
  float **f = (float **)d;
  topo_bind(T, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], (int *)d[8], f[9], f[10],
            f[11], f[12], f[13], f[14], f[15], f[16], f[17], f[18], f[19], f[20], f[21],
            f[22], f[23], f[24], NULL, NULL, NULL, NULL, NULL, NULL, f[25], f[26], f[27]);
  topo_init_metrics(T);
  topo_init_grid(T);
  topo_init_geometry(T);
  topo_build(T);
  topo_set_constants(T);
  cudaDeviceSynchronize();
  return T;
}

void ref_topo_velocity(void *t) {
  topo_t *T = (topo_t *)t;
  topo_velocity_interior_H(T);
  cudaDeviceSynchronize();
}

void ref_topo_stress(void *t) {
  topo_t *T = (topo_t *)t;
  topo_set_constants(T); /* the Cartesian library shares no symbols with it */
  topo_stress_interior_H(T);
  topo_stress_left_H(T);
  topo_stress_right_H(T);
  cudaDeviceSynchronize();
}

/* device metric pointers: f f_1 f_2 f_c (for the curvilinear source add) and
 * g3 g3_c; plus the f line length */
void ref_topo_metric_ptrs(void *t, void **out, int *ld) {
  topo_t *T = (topo_t *)t;
  out[0] = T->metrics_f.d_f;
  out[1] = T->metrics_f.d_f_1;
  out[2] = T->metrics_f.d_f_2;
  out[3] = T->metrics_f.d_f_c;
  out[4] = T->metrics_g.d_g3;
  out[5] = T->metrics_g.d_g3_c;
  *ld = T->metrics_f.slice;
}

void ref_topo_destroy(void *t) {
  topo_t *T = (topo_t *)t;
  if (!T) return;
  topo_free(T);
  free(T);
}
