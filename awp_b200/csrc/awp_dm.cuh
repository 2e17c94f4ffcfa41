// Discontinuous-mesh (DM) coupling of a vertical stack of grids, each 3x
// coarser than the one above it (pmcl3d.c:370-378).  Grid p = 0 is the top
// (finest) block; "hi" is the finer grid above an interface, "lo" the coarser
// one below it.
#pragma once

#include <cuda_runtime.h>

#include "awp_common.h"

struct DmGrid {  // the nine wavefield arrays and the geometry of one grid
  float *u1, *v1, *w1, *xx, *yy, *zz, *xy, *xz, *yz;
  int nxt, nyt, nzt, slice, yline;
};

// dvelc2 (kernel.cu:2289-2356): 2nd-order velocity at k = align+2 of a grid
// that has a coarser grid below it.
struct DmVel2Args {
  DmGrid g;
  const float *d1, *dcrjx, *dcrjy, *dcrjz;
  float dth;
};

// dstrqc2 (kernel.cu:2564-2784): 2nd-order stress and memory variables at
// k = align+2 of a grid that has a coarser grid below it.
struct DmStr2Args {
  DmGrid g;
  float *r1, *r2, *r3, *r4, *r5, *r6;
  const float *lam, *mu, *qp, *qs, *dcrjx, *dcrjy, *dcrjz;
  // memory-variable coefficients: explicit arrays (reference ABI) or the
  // parity pattern when vx1 is null
  const float *vx1, *vx2, *wwo;
  const int* ww;
  AwpTexture tex;
  float coeff[16];
  const float* coeff_dev;
  int i0, i1, j0, j1;
  float dth, dh1, dt;
};

// intp3d (kernel.cu:2359-2561) coarse -> fine and swap3 (kernel.cu:3032-3217)
// fine -> coarse across one interface.
struct DmPairArgs {
  DmGrid lo, hi;
};

// checkmesh (mesh.c:1404-1443): the coarse grid's values at its top three
// levels are replaced by the fine grid's at the co-located points.
struct DmCheckArgs {
  float* lo[5];
  const float* hi[5];
  int nf;
  DmGrid glo, ghi;
};

cudaError_t awp_launch_dvelc2(const DmVel2Args& a, cudaStream_t st);
cudaError_t awp_launch_dstrqc2(const DmStr2Args& a, cudaStream_t st);
cudaError_t awp_launch_intp3d(const DmPairArgs& a, cudaStream_t st);
cudaError_t awp_launch_swap3(const DmPairArgs& a, cudaStream_t st);
cudaError_t awp_launch_checkmesh(const DmCheckArgs& a, cudaStream_t st);
