// Kernel argument blocks and launch helpers for the B200 time-step library.
#pragma once

#include <cuda_runtime.h>

#include "awp_common.h"

// ---------------------------------------------------------------------------
// Velocity half-step (reference: dvelcx_opt, kernel.cu:125-268).
// ---------------------------------------------------------------------------
struct VelArgs {
  float* u1;
  float* v1;
  float* w1;
  const float *xx, *yy, *zz, *xy, *xz, *yz;
  const float *dcrjx, *dcrjy, *dcrjz, *d1;
  int slice, yline;
  int i0, i1, j0, j1, k0, k1;  // inclusive update ranges
  float dth, c1, c2;
};

// ---------------------------------------------------------------------------
// Stress + memory-variable half-step with the free-surface velocity images
// (reference: dstrqc, kernel.cu:880-1197).
// ---------------------------------------------------------------------------
struct StrArgs {
  float *xx, *yy, *zz, *xy, *xz, *yz;
  float *r1, *r2, *r3, *r4, *r5, *r6;
  float *u1, *v1, *w1;
  const float *lam, *mu, *qp, *qs;
  const float *dcrjx, *dcrjy, *dcrjz, *lam_mu;
  // Optional explicit memory-variable arrays (reference ABI); when vx1 is null
  // the parity pattern in `tex` is used instead.
  const float *vx1, *vx2, *wwo;
  const int* ww;
  AwpTexture tex;
  float coeff[16];
  const float* coeff_dev;  // when set, the Q(f) table is read from device memory
  int slice, yline, lam_mu_ld;
  int i0, i1, j0, j1, k0, k1;
  int fs;        // 1: free-surface images at k = ktop (grid 0)
  int ktop;
  int gx_lim;    // image at i+1 exists while i < gx_lim   (kernel.cu:1092)
  int gy_min;    // image at j-1 exists while j >= gy_min  (kernel.cu:1097)
  float dth, dh1, dt, c1, c2;
  float qthr;    // smallest float x with 1/(double)x <= 200 (Q(f) switch)
};

// ---------------------------------------------------------------------------
// Free-surface stress imaging (reference: fstr, kernel.cu:1616-1647).
// ---------------------------------------------------------------------------
struct FstrArgs {
  float *zz, *xz, *yz;
  int slice, yline, ktop;
  int i0, i1, j0, j1;
};

// ---------------------------------------------------------------------------
// Point moment-rate source (reference: addsrc_cu, kernel.cu:1780-1806).
// Sources are grouped by target cell on the host; one thread owns one cell and
// applies its sources in file order, so duplicates accumulate deterministically.
// ---------------------------------------------------------------------------
struct SrcArgs {
  float *xx, *yy, *zz, *xy, *yz, *xz;
  const int* cell_pos;     // [ncell] linear padded index
  const int* cell_first;   // [ncell+1] offsets into order[]
  const int* order;        // source ids grouped by cell
  // Direct mode (reference ABI): cell_pos == nullptr, one thread per source
  // reading its (x, y, z) from psrc[s*dim + 0..2] (kernel.cu:1793-1795).
  const int* psrc;
  int dim, slice, yline;
  const float *axx, *ayy, *azz, *axz, *ayz, *axy;  // [nsrc][stride]
  int ncell, stride, tidx;
  float vtst;              // DT / DH^3
};

// Kinematic finite-fault source (reference: addkinsrc_cu, kernel.cu:3775-3858).
struct KinSrcArgs {
  float *xx, *yy, *zz, *xy, *yz, *xz;
  const float* mu;
  const int* cell_pos;
  const int* cell_first;
  const int* order;
  const int* psrc;  // direct mode as in SrcArgs
  int dim, slice, yline;
  const float *axx, *ayy, *azz, *axz, *ayz, *axy;  // [nsrc][2] subfault params
  float* mom;               // [nsrc] accumulated moment
  double* filt_state;       // [nsrc][filtorder+1] (null if no filter)
  double filt_b[AWP_MAXFILT], filt_a[AWP_MAXFILT];
  int filtorder;
  int ncell, step;
  float dt, vtst;
};

// ---------------------------------------------------------------------------
// Drucker-Prager plasticity (reference: drprecpc_calc_opt, drprecpc_app and
// rotate_principal, kernel.cu:43-64, 1253-1463, 1650-1778).
// ---------------------------------------------------------------------------
struct PlastParams {
  float fmajor, fminor;
  float Rz[9], RzT[9];
  float dh, dt;
  int ktop;  // surface index nzt + ALIGN - 1
};

struct PlastCalcArgs {
  const float *xx, *yy, *zz, *xy, *xz, *yz, *mu, *d1, *sigma2, *cohes, *phi;
  float* yldfac;
  float* neta;
  const unsigned char* neta_mult;  // per-(i,j) visit count of the reference's
                                   // overlapping strip launches (null: 1)
  int neta_ld;
  PlastParams p;
  int slice, yline;
  int i0, i1, j0, j1, k0, k1;
};

struct PlastAppArgs {
  float *xx, *yy, *zz, *xy, *xz, *yz;
  const float *mu, *sigma2, *yldfac;
  PlastParams p;
  int slice, yline;
  int i0, i1, j0, j1, k0, k1;
};

// ---------------------------------------------------------------------------
// Surface / volume output gather (reference: velbuffer, kernel.cu:3948-4011).
// ---------------------------------------------------------------------------
struct VelBufArgs {
  const float *u1, *v1, *w1, *neta;
  float *bufx, *bufy, *bufz, *bufeta;
  int nve, nbgx, nedx, nskpx, nbgy, nedy, nskpy, nbgz, nedz, nskpz;
  int rec_nxt, rec_nyt, rec_nzt;
  int slice, yline, ktop, w_shift;  // w_shift = 1 on grid 0 (w sampled one cell lower)
  const int* bathy;                 // FOLLOWBATHY surface index per (i, j), or null
  int bathy_ld;                     // nxt + 4 + 2*NGSL (bathy is [j][i])
};

// ---------------------------------------------------------------------------
// Media set-up (reference: inimesh, mesh.c:222-466): per-cell unrelaxed-modulus
// correction, inverse moduli and placement into the padded arrays.
// ---------------------------------------------------------------------------
struct MediaArgs {
  const float* media;  // [nz][ny][nx][nvar], surface first
  float *d1, *mu, *lam, *qp, *qs;
  float tau[8], weights[8], coeff[16];
  float w0, facex;
  int nvar, var_offset, nve, socalq;
  int nxt, nyt, nzt;
  int slice, yline;
  // extrema of the corrected vs, vp, rho as float bits (mesh.c:455-460):
  // [vs_min (vs > 1 only), vs_max, vp_min, vp_max, rho_min, rho_max]
  unsigned int* ext;
};

// Launch-shape tuning (awp_kernels.cu): "ichunk" (x-planes marched per CTA) and
// "tma" (kernel family of the context API).  Returns 0 on success.
int awp_tuning_set(const char* key, int value);
int awp_tuning_get(const char* key);

// addplanesrc_cu (kernel.cu:3897-3925): a plane-wave source (IFAULT 6) on the
// level k = align + ND + 1 of the bottom grid, every (i, j) from 4 to
// 3 + nx (ny), sample n of the three input series.
struct PlaneSrcArgs {
  int n, nx, ny, k;
  const float *mu, *lambda, *axx, *ayy, *azz;
  float *xx, *yy, *zz, *xz, *yz;
  int slice, yline;
  float DT, DH;
};

// frcvel_cu (kernel.cu:1836-1934): prescribed velocities at the source points
// (IFAULT 4), linearly interpolated between input samples tskp steps apart;
// on the last prescribed step the restoring force is stored in the source
// arrays and applied on every later step.  One thread per source point.
struct FrcvelArgs {
  int i, read_step, dim, npsrc, tskp, xmin, xmax;
  const int* psrc;
  float *axx, *ayy, *azz, *u1, *v1, *w1;
  int slice, yline;
  float DT;
};

// Up to 32 device-to-device copies in one launch (the halo planes of a
// decomposition): segment q copies n[q] floats, 16-byte aligned, src -> dst.
struct CopySegs {
  const float* src[32];
  float* dst[32];
  long long n[32];
  int nseg;
};

// Launchers (awp_kernels.cu).  All are asynchronous on `st`.
cudaError_t awp_launch_copy_segments(const CopySegs& s, cudaStream_t st);
cudaError_t awp_launch_planesrc(const PlaneSrcArgs& a, cudaStream_t st);
cudaError_t awp_launch_frcvel(const FrcvelArgs& a, cudaStream_t st);
cudaError_t awp_launch_velocity(const VelArgs& a, cudaStream_t st);
cudaError_t awp_launch_stress(const StrArgs& a, bool elastic, cudaStream_t st);
cudaError_t awp_launch_fstr(const FstrArgs& a, cudaStream_t st);
cudaError_t awp_launch_addsrc(const SrcArgs& a, cudaStream_t st);
cudaError_t awp_launch_addkinsrc(const KinSrcArgs& a, cudaStream_t st);
cudaError_t awp_launch_plast_calc(const PlastCalcArgs& a, cudaStream_t st);
cudaError_t awp_launch_plast_app(const PlastAppArgs& a, cudaStream_t st);
cudaError_t awp_launch_velbuffer(const VelBufArgs& a, cudaStream_t st);
cudaError_t awp_launch_media(const MediaArgs& a, cudaStream_t st);
cudaError_t awp_launch_media_borders(float* d1, float* mu, float* lam, float* qp,
                                     float* qs, const AwpGeom& g, int nve,
                                     cudaStream_t st);
cudaError_t awp_launch_lam_mu(const float* lam, const float* mu, float* lam_mu,
                              const AwpGeom& g, int xls, int xre, int yls,
                              int yre, cudaStream_t st);
cudaError_t awp_launch_fill(float* p, float v, long long n, cudaStream_t st);
cudaError_t awp_launch_anynonzero(const float* p, long long n, unsigned int* flag,
                                  cudaStream_t st);
cudaError_t awp_launch_nonfinite(const float* p, long long n, unsigned int* flag,
                                 cudaStream_t st);

// ---------------------------------------------------------------------------
// Batched instances: the per-step launches of many independent single-grid
// simulations (awp_batch_* of the C ABI).  Each instance carries the argument
// blocks its one-simulation launches would take; tiles index into them.
// ---------------------------------------------------------------------------
struct BatchInst {
  VelArgs v;
  StrArgs s;
  FstrArgs f;
  SrcArgs src;
  KinSrcArgs kin;
  int elastic;  // stress without memory variables (Q^-1 == 0)
  int ifault, nst;
};

struct BatchLaunch {
  const BatchInst* inst;
  const int4* vtiles;  // (instance, tile x, tile y, tile z) of the velocity launch
  const int4* stiles;     // same for the stress launch of the anelastic instances
  const int4* stiles_el;  // ... and of the elastic ones
  const int2* src_cells;  // (instance, source cell)
  const int2* rows;       // (instance, padded x index) of the free-surface rows
  int nvtiles, nstiles, nstiles_el, nsrc, nrows;
  int* counters;  // [3] tile counters (reset by the launcher)
  int* step;      // steps taken so far (advanced on the device)
  int ty, ichunk, grid_vel, grid_str;
};

// One time step of every instance: velocity, stress (anelastic, elastic),
// sources, free-surface images and the step counter; a 12-byte memset and up
// to five kernels, all capturable in a CUDA graph.
cudaError_t awp_launch_batch_step(const BatchLaunch& b, cudaStream_t st);
// Resident CTAs per SM of the persistent kernels for tiles 32 x ty (ty = 4, 8).
int awp_batch_blocks_per_sm(int ty, int* vel, int* str);
// Sources of one instance at the step held in device memory (*step + 1), for
// graphs replayed step after step; either argument block may be null.
cudaError_t awp_launch_sources_dev(const SrcArgs* a, const KinSrcArgs* k, const int* step,
                                   int nst, cudaStream_t st);
cudaError_t awp_launch_step_advance(int* step, cudaStream_t st);
