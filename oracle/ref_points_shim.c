/*
 * Test infrastructure only: drives the reference's own point-set device code
 * (src/interpolation/interpolation.cu: cuinterp_init / cuinterp_interp_H, the
 * receiver gather; src/topography/sources/source.cu: cusource_add_cartesian_H,
 * the SOURCEFILE add, and cusource_add_force_H, the FORCEFILE add) on caller
 * device buffers, for GPU parity checks.  Built
 * into oracle/_ref/libawpref_points.so by oracle/Makefile from the reference
 * sources where they lie.
 *
 * Set-up at one rank, one grid block (optionally the curvilinear top block): the reference's reader
 * (input_init), grids_init / grids_select, dist_indices, grid_init_metric_grid
 * and grid_data_init do the work; the glue restates source.c:193-205 and
 * 288-360 (offset by -h/2 in x, zero DM offsets, vertical mapping).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <awp/definitions.h>
#include <grid/grid_3d.h>
#include <interpolation/interpolation.cuh>
#include <mpi/distribute.h>
#include <readers/input.h>
#include <topography/grids.h>
#include <topography/sources/source.cuh>
#include <topography/sources/source.h>
#include <topography/metrics/metrics.h>
#include <grid/shift.h>

typedef struct {
  cu_interp_t I;
  int length;
} ref_pts_t;

/* Returns a handle (NULL on failure); *count = owned points.  With `ftopo`
 * (the normalised surface function of the topography metrics, host copy of
 * f_grid_t.f) the block is curvilinear: closed top boundary and the vertical
 * map of source.c:268-340 through metrics_interpolate_f_point. */
static void *pts_create(const char *path, int grid_type, int nxt, int nyt, int nzt, float h,
                        const float *ftopo, int *count) {
  input_t in;
  memset(&in, 0, sizeof(in));
  if (input_init(&in, path) != 0) return NULL;
  grids_t grids = grids_init(nxt, nyt, nzt, 0, 0, 0, ftopo != NULL, h);
  grid3_t grid = grids_select((enum grid_types)grid_type, &grids);
  size_t n = in.length;
  prec dm0 = 0;
  prec *x = malloc(sizeof(prec) * n), *y = malloc(sizeof(prec) * n),
       *z = malloc(sizeof(prec) * n);
  for (size_t i = 0; i < n; ++i) {
    x[i] = in.x[i] + SOURCE_OFFSET_X * grid.gridspacing;
    y[i] = in.y[i];
    z[i] = in.z[i];
    x[i] = x[i] + dm0;
    y[i] = y[i] + dm0;
    z[i] = z[i] + dm0;
  }
  int *idx = NULL;
  size_t len = 0;
  if (dist_indices(&idx, &len, x, y, n, grid) != 0 || len == 0) return NULL;
  prec block_height = grid.gridspacing * (grid.size.z - (ftopo ? 2 : 1));
  prec lower = 0 - block_height + 0;
  prec *qx = malloc(sizeof(prec) * len), *qy = malloc(sizeof(prec) * len),
       *qz = malloc(sizeof(prec) * len);
  int *ridx = malloc(sizeof(int) * len);
  for (size_t q = 0; q < len; ++q) {
    int s = idx[q];
    qx[q] = x[s];
    qy[q] = y[s];
    qz[q] = z[s];
    if (!ftopo) {
      if (in.type[s] == INPUT_VOLUME_COORD) qz[q] = qz[q] - lower;
      else if (in.type[s] == INPUT_SURFACE_COORD) qz[q] = block_height;
    }
    ridx[q] = (int)q;
  }
  if (ftopo) {
    grid3_t mg = grid_init_metric_grid(grid.inner_size, grid_node(), grid.coordinate,
                                       grid.boundary1, grid.boundary2, grid.gridspacing);
    grid1_t xg = grid_grid1_x(mg), yg = grid_grid1_y(mg), zg = grid_grid1_z(mg);
    prec *x1 = malloc(sizeof(prec) * xg.size), *y1 = malloc(sizeof(prec) * yg.size),
         *z1 = malloc(sizeof(prec) * zg.size);
    grid_fill1(x1, xg);
    grid_fill1(y1, yg);
    grid_fill1(z1, zg);
    int size[3] = {nxt, nyt, nzt};
    f_grid_t fg = metrics_init_f(size, h);
    memcpy(fg.f, ftopo, sizeof(float) * fg.mem[0] * fg.mem[1]);
    prec *fi = malloc(sizeof(prec) * len);
    metrics_interpolate_f_point(&fg, fi, fg.f, x1, y1, mg, qx, qy, (int)len, in.degree);
    for (size_t q = 0; q < len; ++q) {
      int s = idx[q];
      if (in.type[s] == INPUT_VOLUME_COORD) qz[q] = (block_height + qz[q]) / fi[q];
      else if (in.type[s] == INPUT_SURFACE_COORD) qz[q] = z1[zg.size - 2];
    }
    metrics_free_f(&fg);
    free(fi); free(x1); free(y1); free(z1);
  }
  grid3_t full = grid_init_metric_grid(grid.inner_size, grid.shift, grid.coordinate,
                                       grid.boundary1, grid.boundary2, grid.gridspacing);
  grid_data_t xyz;
  grid_data_init(&xyz, full);
  ref_pts_t *p = calloc(1, sizeof(ref_pts_t));
  /* the reference aborts on a non-zero status here (AWPCHK, source.c:376-379) */
  int err = cuinterp_init(&p->I, xyz.x, xyz.y, xyz.z, full, qx, qy, qz, ridx, (int)len,
                          in.degree);
  grid_data_free(&xyz);
  free(x); free(y); free(z); free(idx); free(qx); free(qy); free(qz); free(ridx);
  input_finalize(&in);
  if (err) {
    free(p);
    return NULL;
  }
  p->length = (int)len;
  *count = (int)len;
  return p;
}

void *ref_pts_create(const char *path, int grid_type, int nxt, int nyt, int nzt, float h,
                     int *count) {
  return pts_create(path, grid_type, nxt, nyt, nzt, h, NULL, count);
}

void *ref_pts_create_topo(const char *path, int grid_type, int nxt, int nyt, int nzt, float h,
                          const float *ftopo, int *count) {
  return pts_create(path, grid_type, nxt, nyt, nzt, h, ftopo, count);
}

/* cuinterp_interp_H: d_out[q] = sum l * d_in (the receiver gather). */
void ref_pts_interp(void *h, float *d_out, const float *d_in) {
  ref_pts_t *p = (ref_pts_t *)h;
  cuinterp_interp_H(&p->I, d_out, d_in);
}

/* cusource_add_cartesian_H: d_field -= dt/h^3 * l * d_values[q]. */
void ref_pts_srcadd(void *h, float *d_field, const float *d_values, float hh, float dt) {
  ref_pts_t *p = (ref_pts_t *)h;
  cusource_add_cartesian_H(&p->I, d_field, d_values, hh, dt);
}

/* cusource_add_curvilinear_H: as above, divided by the cell Jacobian f dg. */
void ref_pts_srcadd_curv(void *h, float *d_field, const float *d_values, float hh, float dt,
                         const float *d_f, int ny, const float *d_dg) {
  ref_pts_t *p = (ref_pts_t *)h;
  cusource_add_curvilinear_H(&p->I, d_field, d_values, hh, dt, d_f, ny, d_dg);
}

/* cusource_add_force_H (FORCEFILE, forces.c:74-94): the force rate into a
 * velocity component, scaled by -quad_weight / (f dg rho). */
void ref_pts_force(void *h, float *d_field, const float *d_values, const float *d_d1, float hh,
                   float dt, float quad_weight, const float *d_f, int nx, int ny, int nz,
                   const float *d_dg) {
  ref_pts_t *p = (ref_pts_t *)h;
  cusource_add_force_H(&p->I, d_field, d_values, d_d1, hh, dt, quad_weight, d_f, nx, ny, nz,
                       d_dg);
}

void ref_pts_destroy(void *h) {
  ref_pts_t *p = (ref_pts_t *)h;
  if (!p) return;
  cuinterp_finalize(&p->I);
  free(p);
}
