/*
 * Flat-array entry points around the reference's own host set-up code.
 *
 * Test infrastructure only.  This file is compiled together with the
 * reference's src/awp/mesh.c, src/awp/cerjan.c and src/awp/grid.c (read in
 * place, never copied) into oracle/_ref/libawpref_host.so.  The tests call it
 * through ctypes to pin the product's C++ re-statement of the same set-up
 * (Q(f) tables, relaxation times, the media/modulus mapping, the memory-
 * variable parity pattern and the Cerjan sponge) against the reference
 * itself.
 *
 * Every output array is flat and uses the reference's padded layout
 * (i slowest, k fastest): (nxt+4+2*ngsl) x (nyt+4+2*ngsl) x (nzt+2*align).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <awp/pmcl3d.h>

Grid3D Alloc3D(int nx, int ny, int nz);
Grid3Dww Alloc3Dww(int nx, int ny, int nz);
Grid1D Alloc1D(int nx);
void Delloc3D(Grid3D U);
void Delloc3Dww(Grid3Dww U);
void Delloc1D(Grid1D U);
void tausub(Grid3D tau, _prec taumin, _prec taumax);
void weights_sub(Grid3D weights, Grid1D coeff, _prec ex, _prec fac);
void init_texture(int nxt, int nyt, int nzt, Grid3D tau1, Grid3D tau2, Grid3D vx1,
                  Grid3D vx2, Grid3D weights, Grid3Dww ww, Grid3D wwo, int xls,
                  int xre, int yls, int yre);
void inicrj(_prec ARBC, int *coords, int nxt, int nyt, int nzt, int NX, int NY,
            int ND, Grid1D dcrjx, Grid1D dcrjy, Grid1D dcrjz, int islowest,
            int NPC);
void hoek_brown(_prec sigma_0, _prec sigma_ci, _prec GSI, _prec mi, _prec D,
                int tunnel, _prec *phi, _prec *cohes);

static void copy8(Grid3D g, float *out) {
  int i, j, k;
  for (i = 0; i < 2; i++)
    for (j = 0; j < 2; j++)
      for (k = 0; k < 2; k++) out[i * 4 + j * 2 + k] = g[i][j][k];
}

/* tausub (mesh.c:684-710): 8 relaxation times between taumin and taumax. */
void ref_tausub(float taumin, float taumax, float *tau8) {
  Grid3D tau = Alloc3D(2, 2, 2);
  tausub(tau, taumin, taumax);
  copy8(tau, tau8);
  free(tau);
}

/* weights_sub (mesh.c:713-1097): Q(f) weights (already divided by FAC^EX)
 * and the 16-entry coefficient table. */
void ref_weights_sub(float ex, float fac, float *w8, float *coeff16) {
  Grid3D w = Alloc3D(2, 2, 2);
  Grid1D c = Alloc1D(16);
  weights_sub(w, c, ex, fac);
  copy8(w, w8);
  memcpy(coeff16, c, 16 * sizeof(float));
  free(w);
  free(c);
}

/* inimesh (mesh.c:23-614) with MEDIASTART=1/2 reading INVEL at PX=PY=1.
 * Outputs the padded d1, mu, lam, qp, qs arrays plus the relaxation times,
 * the Q(f) weights/coefficients and the vs/vp/rho extrema. */
void ref_inimesh(const char *invel, int nvar, float fp, float fac, float q0,
                 float ex, int nxt, int nyt, int nzt, int nve, int socalq,
                 float *d1, float *mu, float *lam, float *qp, float *qs,
                 float *taumax, float *taumin, float *tau8, float *w8,
                 float *coeff16, float *vse, float *vpe, float *dde) {
  int nx = nxt + 4 + ngsl2, ny = nyt + 4 + ngsl2, nz = nzt + 2 * align;
  size_t n = (size_t)nx * ny * nz;
  Grid3D gd1 = Alloc3D(nx, ny, nz), gmu = Alloc3D(nx, ny, nz),
         glam = Alloc3D(nx, ny, nz), gqp = Alloc3D(nx, ny, nz),
         gqs = Alloc3D(nx, ny, nz);
  Grid3D tau = Alloc3D(2, 2, 2), weights = Alloc3D(2, 2, 2);
  Grid1D coeff = Alloc1D(16);
  int coords[2] = {0, 0};
  char path[512];
  weights_sub(weights, coeff, ex, fac);
  strncpy(path, invel, sizeof(path) - 1);
  path[sizeof(path) - 1] = 0;
  inimesh(0, 1, gd1, gmu, glam, gqp, gqs, taumax, taumin, tau, weights, coeff,
          nvar, fp, fac, q0, ex, nxt, nyt, nzt, 1, 1, nxt, nyt, nzt, coords,
          MPI_COMM_WORLD, 0, nve, socalq, path, vse, vpe, dde);
  memcpy(d1, &gd1[0][0][0], n * sizeof(float));
  memcpy(mu, &gmu[0][0][0], n * sizeof(float));
  memcpy(lam, &glam[0][0][0], n * sizeof(float));
  memcpy(qp, &gqp[0][0][0], n * sizeof(float));
  memcpy(qs, &gqs[0][0][0], n * sizeof(float));
  copy8(tau, tau8);
  copy8(weights, w8);
  memcpy(coeff16, coeff, 16 * sizeof(float));
  free(gd1); free(gmu); free(glam); free(gqp); free(gqs);
  free(tau); free(weights); free(coeff);
}

/* init_texture (mesh.c:1103-1137) given tau1/tau2/weights as 8-vectors. */
void ref_init_texture(int nxt, int nyt, int nzt, const float *tau1_8,
                      const float *tau2_8, const float *w8, int xls, int xre,
                      int yls, int yre, float *vx1, float *vx2, int *ww,
                      float *wwo) {
  int nx = nxt + 4 + ngsl2, ny = nyt + 4 + ngsl2, nz = nzt + 2 * align;
  size_t n = (size_t)nx * ny * nz;
  Grid3D t1 = Alloc3D(2, 2, 2), t2 = Alloc3D(2, 2, 2), w = Alloc3D(2, 2, 2);
  Grid3D g1 = Alloc3D(nx, ny, nz), g2 = Alloc3D(nx, ny, nz), gwo = Alloc3D(nx, ny, nz);
  Grid3Dww gww = Alloc3Dww(nx, ny, nz);
  int i, j, k;
  for (i = 0; i < 2; i++)
    for (j = 0; j < 2; j++)
      for (k = 0; k < 2; k++) {
        t1[i][j][k] = tau1_8[i * 4 + j * 2 + k];
        t2[i][j][k] = tau2_8[i * 4 + j * 2 + k];
        w[i][j][k] = w8[i * 4 + j * 2 + k];
      }
  init_texture(nxt, nyt, nzt, t1, t2, g1, g2, w, gww, gwo, xls, xre, yls, yre);
  memcpy(vx1, &g1[0][0][0], n * sizeof(float));
  memcpy(vx2, &g2[0][0][0], n * sizeof(float));
  memcpy(wwo, &gwo[0][0][0], n * sizeof(float));
  memcpy(ww, &gww[0][0][0], n * sizeof(int));
  free(t1); free(t2); free(w); free(g1); free(g2); free(gwo); free(gww);
}

/* inicrj (cerjan.c:5-64) at coords (0,0). */
void ref_inicrj(float arbc, int nxt, int nyt, int nzt, int NX, int NY, int ND,
                int islowest, int npc, float *dcrjx, float *dcrjy,
                float *dcrjz) {
  int coords[2] = {0, 0};
  int i;
  for (i = 0; i < nxt + 4 + ngsl2; i++) dcrjx[i] = 1.0f;
  for (i = 0; i < nyt + 4 + ngsl2; i++) dcrjy[i] = 1.0f;
  for (i = 0; i < nzt + 2 * align; i++) dcrjz[i] = 1.0f;
  inicrj(arbc, coords, nxt, nyt, nzt, NX, NY, ND, dcrjx, dcrjy, dcrjz, islowest,
         npc);
}

/* hoek_brown (mesh.c:1139-1176). */
void ref_hoek_brown(float sigma_0, float sigma_ci, float gsi, float mi, float d,
                    int tunnel, float *phi, float *cohes) {
  hoek_brown(sigma_0, sigma_ci, gsi, mi, d, tunnel, phi, cohes);
}

/* rotation_matrix (mesh.c:1370-1401): principal-stress rotation from the
 * strike and dip angles (degrees) of nonlinear.dat. */
void rotation_matrix(_prec *strike, _prec *dip, _prec *Rz, _prec *RzT);
void ref_rotation_matrix(const float *strike, const float *dip, float *Rz, float *RzT) {
  float s[3], d[3];
  memcpy(s, strike, sizeof(s));
  memcpy(d, dip, sizeof(d));
  rotation_matrix(s, d, Rz, RzT);
}

/* ------------------------------------------------------------------------ */
/* Point sets (RECVFILE / SOURCEFILE): the reference's ASCII v2 reader and   */
/* its interpolation set-up, one rank, one grid block, no topography.        */
/* ------------------------------------------------------------------------ */
#include <readers/input.h>
#include <grid/grid_3d.h>
#include <grid/shift.h>
#include <topography/grids.h>
#include <interpolation/interpolation.h>
#include <mpi/distribute.h>
#include <topography/sources/source.h> /* SOURCE_OFFSET_X */

static input_t g_input;
static int g_input_ok = 0;

/* input_init (readers/input.c:35-42).  hdr[] = length, gpu_buffer_size,
 * cpu_buffer_size, steps, num_writes, stride, degree, major version. */
int ref_input_read(const char *path, long long *hdr, char *file, int filecap) {
  if (g_input_ok) input_finalize(&g_input);
  memset(&g_input, 0, sizeof(g_input));
  int err = input_init(&g_input, path);
  g_input_ok = (err == 0);
  if (err) return err;
  hdr[0] = (long long)g_input.length;
  hdr[1] = (long long)g_input.gpu_buffer_size;
  hdr[2] = (long long)g_input.cpu_buffer_size;
  hdr[3] = (long long)g_input.steps;
  hdr[4] = (long long)g_input.num_writes;
  hdr[5] = g_input.stride;
  hdr[6] = g_input.degree;
  hdr[7] = g_input.version.major;
  snprintf(file, filecap, "%s", g_input.file);
  return 0;
}

void ref_input_data(float *x, float *y, float *z, int *type) {
  for (size_t i = 0; i < g_input.length; ++i) {
    x[i] = g_input.x[i];
    y[i] = g_input.y[i];
    z[i] = g_input.z[i];
    type[i] = g_input.type[i];
  }
}

/* The interpolation set-up of source_init_common (topography/sources/
 * source.c:137-400) for the last file read, at one rank, one grid block,
 * no topography.  grid_type follows enum grid_types (X=0, Y, Z, XX, YY, ZZ,
 * XY, XZ, YZ).  The reference's building blocks do the work (grids_init,
 * dist_indices, grid_init_metric_grid, grid_data_init,
 * interp_lagrange1_coef); the few lines of glue restate source.c:193-205 and
 * 288-360.  Returns the number of owned points, or -err. */
static int point_coefs(int grid_type, int nxt, int nyt, int nzt, float h, const float *ftopo,
                       int *indices, int *ix, int *iy, int *iz, float *lx, float *ly,
                       float *lz);
int ref_point_coefs(int grid_type, int nxt, int nyt, int nzt, float h, int *indices,
                    int *ix, int *iy, int *iz, float *lx, float *ly, float *lz) {
  return point_coefs(grid_type, nxt, nyt, nzt, h, NULL, indices, ix, iy, iz, lx, ly, lz);
}
/* The curvilinear top block: ftopo = the normalised surface function (host
 * layout of f_grid_t.f); the vertical map of source.c:268-340. */
int ref_point_coefs_topo(int grid_type, int nxt, int nyt, int nzt, float h, const float *ftopo,
                         int *indices, int *ix, int *iy, int *iz, float *lx, float *ly,
                         float *lz) {
  return point_coefs(grid_type, nxt, nyt, nzt, h, ftopo, indices, ix, iy, iz, lx, ly, lz);
}
static int point_coefs(int grid_type, int nxt, int nyt, int nzt, float h, const float *ftopo,
                       int *indices, int *ix, int *iy, int *iz, float *lx, float *ly,
                       float *lz) {
  grids_t grids = grids_init(nxt, nyt, nzt, 0, 0, 0, ftopo != NULL, h);
  grid3_t grid = grids_select((enum grid_types)grid_type, &grids);
  size_t n = g_input.length;
  prec dm0 = 0;
  prec *x = malloc(sizeof(prec) * n), *y = malloc(sizeof(prec) * n),
       *z = malloc(sizeof(prec) * n);
  for (size_t i = 0; i < n; ++i) {
    x[i] = g_input.x[i] + SOURCE_OFFSET_X * grid.gridspacing;
    y[i] = g_input.y[i];
    z[i] = g_input.z[i];
    /* DM offsets of the top block are zero, but adding them turns -0 into +0
     * (source.c:201-203) */
    x[i] = x[i] + dm0;
    y[i] = y[i] + dm0;
    z[i] = z[i] + dm0;
  }
  int *idx = NULL;
  size_t len = 0;
  int err = dist_indices(&idx, &len, x, y, n, grid);
  if (err) return -err;
  prec block_height = grid.gridspacing * (grid.size.z - (ftopo ? 2 : 1));
  prec lower = 0 - block_height + 0;
  grid3_t full = grid_init_metric_grid(grid.inner_size, grid.shift, grid.coordinate,
                                       grid.boundary1, grid.boundary2, grid.gridspacing);
  grid_data_t xyz;
  grid_data_init(&xyz, full);
  int deg = g_input.degree, nb = deg + 1;
  prec *xloc = calloc(sizeof(prec), nb);
  prec *fi = NULL, *z1 = NULL;
  int zsize = 0;
  if (ftopo) {
    /* f_grid_t of metrics_init_f (metrics.c:14-33) on the caller's host f */
    f_grid_t fg;
    memset(&fg, 0, sizeof(fg));
    fg.offset[0] = 2 + ngsl;
    fg.offset[1] = 2 + ngsl + align;
    fg.bounds_x[0] = -ngsl;
    fg.bounds_y[0] = -ngsl;
    fg.slice = (nyt + 4 + 2 * ngsl + 2 * align) * 1;
    fg.f = (prec *)ftopo;
    grid3_t mg = grid_init_metric_grid(grid.inner_size, grid_node(), grid.coordinate,
                                       grid.boundary1, grid.boundary2, grid.gridspacing);
    grid1_t xg = grid_grid1_x(mg), yg = grid_grid1_y(mg), zg = grid_grid1_z(mg);
    prec *x1 = malloc(sizeof(prec) * xg.size), *y1 = malloc(sizeof(prec) * yg.size);
    z1 = malloc(sizeof(prec) * zg.size);
    zsize = zg.size;
    grid_fill1(x1, xg);
    grid_fill1(y1, yg);
    grid_fill1(z1, zg);
    prec *qx = malloc(sizeof(prec) * len), *qy = malloc(sizeof(prec) * len);
    for (size_t q = 0; q < len; ++q) {
      qx[q] = x[idx[q]];
      qy[q] = y[idx[q]];
    }
    fi = malloc(sizeof(prec) * len);
    metrics_interpolate_f_point(&fg, fi, fg.f, x1, y1, mg, qx, qy, (int)len, deg);
    free(x1); free(y1); free(qx); free(qy);
  }
  for (size_t q = 0; q < len; ++q) {
    int s = idx[q];
    prec zz = z[s];
    if (ftopo) {
      if (g_input.type[s] == INPUT_VOLUME_COORD) zz = (block_height + zz) / fi[q];
      else if (g_input.type[s] == INPUT_SURFACE_COORD) zz = z1[zsize - 2];
    } else if (g_input.type[s] == INPUT_VOLUME_COORD) zz = zz - lower;
    else if (g_input.type[s] == INPUT_SURFACE_COORD) zz = block_height;
    indices[q] = s;
    err = interp_lagrange1_coef(xloc, &lx[q * nb], &ix[q], xyz.x, grid_boundary_size(full).x,
                                x[s], deg);
    err = interp_lagrange1_coef(xloc, &ly[q * nb], &iy[q], xyz.y, grid_boundary_size(full).y,
                                y[s], deg);
    err = interp_lagrange1_coef(xloc, &lz[q * nb], &iz[q], xyz.z, grid_boundary_size(full).z,
                                zz, deg);
  }
  free(xloc);
  free(fi);
  free(z1);
  grid_data_free(&xyz);
  free(x); free(y); free(z); free(idx);
  return (int)len;
}

/* checkmesh / checkmesh_ww (mesh.c:1404-1478) on flat padded arrays: the
 * coarse grid "l" takes the fine grid "h"'s values at its top three levels. */
int checkmesh(int nxtl, int nytl, int nztl, int nxth, int nyth, int nzth, Grid3D varl,
              Grid3D varh, int pl, int ph, char *varname);
int checkmesh_ww(int nxtl, int nytl, int nztl, int nxth, int nyth, int nzth, Grid3Dww varl,
                 Grid3Dww varh, int pl, int ph, char *varname);
int ref_checkmesh(int nxtl, int nytl, int nztl, int nxth, int nyth, int nzth, float *varl,
                  const float *varh) {
  int nxl = nxtl + 4 + ngsl2, nyl = nytl + 4 + ngsl2, nzl = nztl + 2 * align;
  int nxh = nxth + 4 + ngsl2, nyh = nyth + 4 + ngsl2, nzh = nzth + 2 * align;
  Grid3D l = Alloc3D(nxl, nyl, nzl), h = Alloc3D(nxh, nyh, nzh);
  memcpy(&l[0][0][0], varl, sizeof(float) * (size_t)nxl * nyl * nzl);
  memcpy(&h[0][0][0], varh, sizeof(float) * (size_t)nxh * nyh * nzh);
  int c = checkmesh(nxtl, nytl, nztl, nxth, nyth, nzth, l, h, 1, 0, "var");
  memcpy(varl, &l[0][0][0], sizeof(float) * (size_t)nxl * nyl * nzl);
  free(l);
  free(h);
  return c;
}
int ref_checkmesh_ww(int nxtl, int nytl, int nztl, int nxth, int nyth, int nzth, int *varl,
                     const int *varh) {
  int nxl = nxtl + 4 + ngsl2, nyl = nytl + 4 + ngsl2, nzl = nztl + 2 * align;
  int nxh = nxth + 4 + ngsl2, nyh = nyth + 4 + ngsl2, nzh = nzth + 2 * align;
  Grid3Dww l = Alloc3Dww(nxl, nyl, nzl), h = Alloc3Dww(nxh, nyh, nzh);
  memcpy(&l[0][0][0], varl, sizeof(int) * (size_t)nxl * nyl * nzl);
  memcpy(&h[0][0][0], varh, sizeof(int) * (size_t)nxh * nyh * nzh);
  int c = checkmesh_ww(nxtl, nytl, nztl, nxth, nyth, nzth, l, h, 1, 0, "ww");
  memcpy(varl, &l[0][0][0], sizeof(int) * (size_t)nxl * nyl * nzl);
  free(l);
  free(h);
  return c;
}

/* ------------------------------------------------------------------------ */
/* Topography metrics: the reference's reader, geometry and metric code      */
/* (readers/serial_reader.c, geometry/geometry.c, metrics/metrics.c,         */
/* metrics/kernel.c) in the order of topo_init_metrics / topo_init_geometry / */
/* topo_build (topography.c:238-262), one rank.  The f_grid_t / g_grid_t set- */
/* up restates metrics_init_f / metrics_init_g (metrics.c:14-37, 194-211)     */
/* with zero-filled host arrays and no device copies.                         */
/* out: f, f_1, f_2, f_c, f1_1, f1_2, f1_c, f2_1, f2_2, f2_c (each mx*my),     */
/* then g, g_c, g3, g3_c (each nz + 2 align).  Returns the reader's status.   */
/* ------------------------------------------------------------------------ */
#include <topography/metrics/metrics.h>
#include <topography/geometry/geometry.h>
#include <topography/readers/serial_reader.h>

int ref_topo_metrics(const char *path, int nx, int ny, int nz, float h, float *out) {
  f_grid_t f;
  memset(&f, 0, sizeof(f));
  f.size[0] = nx; f.size[1] = ny; f.size[2] = 1;
  f.mem[0] = nx + 4 + 2 * ngsl; f.mem[1] = ny + 4 + 2 * ngsl + 2 * align; f.mem[2] = 1;
  f.bounds_x[0] = -ngsl; f.bounds_x[1] = nx + ngsl;
  f.bounds_y[0] = -ngsl; f.bounds_y[1] = ny + ngsl;
  f.bounds_stress_x[0] = -ngsl / 2; f.bounds_stress_x[1] = nx + ngsl / 2;
  f.bounds_stress_y[0] = -ngsl / 2; f.bounds_stress_y[1] = ny + ngsl / 2;
  f.offset[0] = 2 + ngsl; f.offset[1] = 2 + ngsl + align; f.offset[2] = 0;
  f.hi = 1.0 / h;
  f.line = f.mem[2];
  f.slice = f.mem[1] * f.mem[2];
  size_t nf = (size_t)f.mem[0] * f.mem[1];
  prec **farr[10] = {&f.f, &f.f_1, &f.f_2, &f.f_c, &f.f1_1, &f.f1_2, &f.f1_c, &f.f2_1,
                     &f.f2_2, &f.f2_c};
  for (int q = 0; q < 10; ++q) *farr[q] = calloc(nf, sizeof(prec));
  g_grid_t g;
  memset(&g, 0, sizeof(g));
  g.size = nz; g.mem = nz + 2 * align; g.bounds_z[0] = 0; g.bounds_z[1] = nz;
  g.offset = align; g.hi = 1.0 / h; g.line = g.mem;
  prec **garr[4] = {&g.g, &g.g_c, &g.g3, &g.g3_c};
  for (int q = 0; q < 4; ++q) *garr[q] = calloc(g.mem, sizeof(prec));
  int coord[2] = {0, 0};
  int err = topo_read_serial(path, 0, 1, 1, coord, nx, ny, 0, &f.f);
  if (err) return err;
  geom_no_grid_stretching(&g);
  int3_t size = {.x = nx, .y = ny, .z = nz};
  int3_t shift = {.x = 1, .y = 0, .z = 0};
  int3_t c3 = {.x = 0, .y = 0, .z = 0};
  int3_t b1 = {.x = 0, .y = 0, .z = 0};
  int3_t b2 = {.x = 0, .y = 0, .z = 1};
  grid3_t tg = grid_init_metric_grid(size, shift, c3, b1, b2, h);
  geom_custom(&f, tg, 1, 1, f.f);
  metrics_interpolate_f(&f);
  metrics_differentiate_f(&f);
  metrics_interpolate_g(&g);
  metrics_differentiate_g(&g);
  for (int q = 0; q < 10; ++q) {
    memcpy(out + q * nf, *farr[q], nf * sizeof(float));
    free(*farr[q]);
  }
  for (int q = 0; q < 4; ++q) {
    memcpy(out + 10 * nf + (size_t)q * g.mem, *garr[q], g.mem * sizeof(float));
    free(*garr[q]);
  }
  return 0;
}
