// Discrete adjoint of the single-grid time step (velocity, stress with memory
// variables, free-surface images) and the gradient of a seismogram misfit with
// respect to the materials.
#pragma once

#include <cuda_runtime.h>

#include "awp_common.h"

// Layout of the stored forward velocities: the box of padded cells
// [i0, i0+ni) x [j0, j0+nj) x [k0, k0+nk) that the adjoint kernels read, rows
// of ld >= nk floats.  Padded cell (i, j, k) sits at i*S + j*Y + k - off.
struct VelBox {
  int i0, j0, k0, ni, nj, nk, ld;
  long long S, Y, off;
  size_t cells() const { return (size_t)ni * nj * ld; }
};

struct AdjArgs {
  // forward state: velocities before the step (velocity half) and after it
  // (both halves; free-surface images included), in the VelBox layout vb
  const float *bu, *bv, *bw;
  const float *fu, *fv, *fw;
  VelBox vb;
  // adjoint state, updated in place (u v w xx yy zz xy xz yz r1..r6)
  float* L[15];
  // temporaries (zero outside the ranges that write them)
  // stress half: adjoint strain rates (6), material weights of the moduli (5)
  // and of the inverse quality factors (5: the Qp^-1 and Qs^-1 eight-cell
  // sums and the three Qs^-1 pair sums); velocity half: weighted adjoint
  // velocities (3) and density weights (3).  The weights are summed over the
  // steps and turned into gradients once, by awp_launch_adjoint_fold.
  float* E[16];
  float* V[6];
  // image-adjoint increments of the surface columns and their one-column
  // ring: 4 planes of (si1 - si0 + 3) x (sj1 - sj0 + 3), (i, j) row-major
  float* img;
  // gradients on the padded kernel arrays: rho, 1/lambda, 1/mu, Qp^-1,
  // Qs^-1, and the surface Lame ratio lam_mu (2-D)
  float *gd, *glam, *gmu, *gqp, *gqs, *glm;
  // media and constants of the forward step
  const float *d1, *lam, *mu, *qp, *qs, *lam_mu;
  const float *dcrjx, *dcrjy, *dcrjz;
  AwpTexture tex;
  float coeff[16];
  float dth, dh1, dt, c1, c2, qthr;
  int elastic;
  int want_q;  // accumulate the Q^-1 weights (the caller asked for g_qpinv / g_qsinv)
  AwpGeom g;
  int vi0, vi1, vj0, vj1, vk0, vk1;  // velocity update range (inclusive, padded)
  int si0, si1, sj0, sj1, sk0, sk1;  // stress update range
  int fj1;                           // last j row of the free-surface imaging
  int gx_lim, gy_min, lam_mu_ld;
};

// One step backwards: imaging, stress (+ memory variables, images), velocity;
// accumulates the material gradients of that step.
cudaError_t awp_launch_adjoint_step(const AdjArgs& a, cudaStream_t st);

// The forward velocities u, v, w (padded layout) into the VelBox layout.
cudaError_t awp_launch_pack_vel(const float* u, const float* v, const float* w, float* du,
                                float* dv, float* dw, const VelBox& b, const AwpGeom& g,
                                cudaStream_t st);

// Receiver terms: L[comp][idx[r]] += res[r], one thread per distinct
// (component, cell) c adding the receivers order[first[c] .. first[c+1]) in order.
cudaError_t awp_launch_adjoint_inject(float* const L[3], const long long* idx, const int* comp,
                                      const int* first, const int* order, int ncell,
                                      const float* res, cudaStream_t st);
// Seismogram samples of the current state: out[r] = field(comp[r])[idx[r]].
cudaError_t awp_launch_sample(const float* u, const float* v, const float* w,
                              const long long* idx, const int* comp, int nrec, float* out,
                              cudaStream_t st);

// The summed material weights -> gradients on the padded arrays -> interior
// lambda, mu, rho (layout [nz][ny][nx], surface first): the border-fill
// copies folded back, the reciprocal moduli and the surface Lame ratio
// chained through.
cudaError_t awp_launch_adjoint_fold(const AdjArgs& a, float* g_lambda, float* g_mu,
                                    float* g_rho, cudaStream_t st);
// The summed Q weights -> interior gradients with respect to Qp^-1 and Qs^-1
// (layout [nz][ny][nx], surface first), the border-fill copies folded back.
// Runs after awp_launch_adjoint_fold (which forms the padded gradients).
cudaError_t awp_launch_adjoint_fold_q(const AdjArgs& a, float* g_qpinv, float* g_qsinv,
                                      cudaStream_t st);
// Qp^-1 and Qs^-1 from interior arrays into the padded kernel arrays, one-cell
// border included.
cudaError_t awp_launch_set_qinv(const float* qpinv, const float* qsinv, float* qp, float* qs,
                                const AwpGeom& g, cudaStream_t st);

// Moduli and density from interior arrays ([nz][ny][nx], surface first) into
// the padded kernel arrays (1/lambda, 1/mu, rho), one-cell border included.
cudaError_t awp_launch_set_moduli(const float* lambda, const float* mu_, const float* rho,
                                  float* lam, float* mu, float* d1, const AwpGeom& g,
                                  cudaStream_t st);
