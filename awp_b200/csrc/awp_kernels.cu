// B200 kernels for the AWP-ODC time step.
//
// Design (all HBM-bound; nothing here is a dense contraction):
//  * Each CTA owns a tile of 32 consecutive k (one warp row = one 128-byte
//    line per field) by TY consecutive j, and marches a chunk of x planes.
//    Values the x-stencil needs at i-2..i+2 live in a per-thread register
//    queue, so every x-plane of a field is loaded from HBM once per chunk.
//  * j- and k-neighbours are read through the read-only path (LDG.NC); they
//    are served by L1/L2 because the 32 x TY tile and its neighbours in the
//    same wave touch the same lines.
//  * The memory-variable coefficients (vx1, vx2, ww, wwo) are recomputed from
//    the parity of (i, j, k) instead of being read (4 arrays, 16 B/cell saved).
//  * The arithmetic of every update follows the reference expression by
//    expression (including its double-precision divisions and its Q(f)
//    switch), so results agree with the reference CUDA build to rounding.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <string.h>

#include "awp_kernels.cuh"
#include "awp_stencil.cuh"
#include "awp_tma.cuh"

#define LDG(p) __ldg(p)

namespace {

// Launch shape (tuned on B200; adjustable through awp_set_tuning).  Tiles are
// 32 k x 8 j for every kernel; the chunk of x planes and the kernel family vary.
int g_ichunk = 32;
// context API kernel family per half-step: TMA-pipelined (1) or read-only path (0)
int g_tma_vel = 1;
int g_tma_str = 1;

// ===========================================================================
// Velocity (dvelcx_opt, kernel.cu:125-268)
// ===========================================================================
// One 32 k x TY j x ichunk i tile (tile coordinates bx, by, bz), thread (tx, ty).
template <int TY>
__device__ __forceinline__ void vel_tile(const VelArgs& a, const int bx, const int by,
                                         const int bz, const int ichunk, const int tx,
                                         const int ty) {
  const int k = a.k0 + bx * 32 + tx;
  const int j = a.j0 + by * TY + ty;
  if (k > a.k1 || j > a.j1) return;
  const int ib = a.i0 + bz * ichunk;
  const int ie = min(ib + ichunk - 1, a.i1);
  const int S = a.slice, Y = a.yline;
  const float c1 = a.c1, c2 = a.c2, dth = a.dth;
  const float dcy = LDG(a.dcrjy + j), dcz = LDG(a.dcrjz + k);
  const long long col = (long long)j * Y + k;

  const float* __restrict__ XX = a.xx + col;
  const float* __restrict__ YY = a.yy + col;
  const float* __restrict__ ZZ = a.zz + col;
  const float* __restrict__ XY = a.xy + col;
  const float* __restrict__ XZ = a.xz + col;
  const float* __restrict__ YZ = a.yz + col;
  const float* __restrict__ D = a.d1 + col;
  float* __restrict__ U = a.u1 + col;
  float* __restrict__ V = a.v1 + col;
  float* __restrict__ W = a.w1 + col;

  long long o = (long long)ib * S;
  // register queues along x
  float xx_m2 = LDG(XX + o - 2 * S), xx_m1 = LDG(XX + o - S), xx_0 = LDG(XX + o);
  float xy_m1 = LDG(XY + o - S), xy_0 = LDG(XY + o), xy_p1 = LDG(XY + o + S);
  float xz_m1 = LDG(XZ + o - S), xz_0 = LDG(XZ + o), xz_p1 = LDG(XZ + o + S);
  float d_0 = LDG(D + o), d_0k = LDG(D + o - 1), d_0j = LDG(D + o - Y);

  for (int i = ib; i <= ie; ++i, o += S) {
    const float xx_p1 = LDG(XX + o + S);
    const float xy_p2 = LDG(XY + o + 2 * S);
    const float xz_p2 = LDG(XZ + o + 2 * S);
    const float d_p = LDG(D + o + S), d_pk = LDG(D + o + S - 1),
                d_pj = LDG(D + o + S - Y);
    const float d_0jk = LDG(D + o - Y - 1);
    const float yz_0 = LDG(YZ + o);

    const float fd1 = awp_vel_factor(dth, d_0, d_0j, d_0k, d_0jk);
    const float fd2 = awp_vel_factor(dth, d_0, d_p, d_0k, d_pk);
    const float fd3 = awp_vel_factor(dth, d_0, d_p, d_0j, d_pj);
    const float dcrj = LDG(a.dcrjx + i) * dcy * dcz;

    U[o] = awp_vel_update(U[o], fd1, c1, c2, xx_0 - xx_m1, xx_p1 - xx_m2,
                          xy_0 - LDG(XY + o - Y), LDG(XY + o + Y) - LDG(XY + o - 2 * Y),
                          xz_0 - LDG(XZ + o - 1), LDG(XZ + o + 1) - LDG(XZ + o - 2), dcrj);
    V[o] = awp_vel_update(V[o], fd2, c1, c2, xy_p1 - xy_0, xy_p2 - xy_m1,
                          LDG(YY + o + Y) - LDG(YY + o), LDG(YY + o + 2 * Y) - LDG(YY + o - Y),
                          yz_0 - LDG(YZ + o - 1), LDG(YZ + o + 1) - LDG(YZ + o - 2), dcrj);
    W[o] = awp_vel_update(W[o], fd3, c1, c2, xz_p1 - xz_0, xz_p2 - xz_m1,
                          yz_0 - LDG(YZ + o - Y), LDG(YZ + o + Y) - LDG(YZ + o - 2 * Y),
                          LDG(ZZ + o + 1) - LDG(ZZ + o), LDG(ZZ + o + 2) - LDG(ZZ + o - 1), dcrj);

    xx_m2 = xx_m1; xx_m1 = xx_0; xx_0 = xx_p1;
    xy_m1 = xy_0; xy_0 = xy_p1; xy_p1 = xy_p2;
    xz_m1 = xz_0; xz_0 = xz_p1; xz_p1 = xz_p2;
    d_0 = d_p; d_0k = d_pk; d_0j = d_pj;
  }
}

template <int TY>
__global__ void __launch_bounds__(32 * TY)
    k_velocity(const VelArgs a, const int ichunk) {
  vel_tile<TY>(a, blockIdx.x, blockIdx.y, blockIdx.z, ichunk, threadIdx.x, threadIdx.y);
}

// ===========================================================================
// Stress + attenuation (dstrqc, kernel.cu:880-1197)
// ===========================================================================

struct Plane4 {  // one field at (j,k), (j-1,k), (j,k-1), (j-1,k-1) of a plane
  float a, b, c, d;
};

__device__ __forceinline__ Plane4 load4(const float* __restrict__ p, int Y) {
  Plane4 r;
  r.a = LDG(p);
  r.b = LDG(p - Y);
  r.c = LDG(p - 1);
  r.d = LDG(p - Y - 1);
  return r;
}

// Sum of the 8 cell values around an edge in the reference's order:
// pos, ip1, jm1, ijk, km1, ik1, jk1, ijk1.
__device__ __forceinline__ float sum8(const Plane4& c, const Plane4& n) {
  return c.a + n.a + c.b + n.b + c.c + n.c + c.d + n.d;
}

template <bool ELASTIC, bool TEXARR, int TY>
__device__ __forceinline__ void str_tile(const StrArgs& a, const int bx, const int by,
                                         const int bz, const int ichunk, const int tx,
                                         const int ty) {
  const int k = a.k0 + bx * 32 + tx;
  const int j = a.j0 + by * TY + ty;
  if (k > a.k1 || j > a.j1) return;
  const int ib = a.i0 + bz * ichunk;
  const int ie = min(ib + ichunk - 1, a.i1);
  const int S = a.slice, Y = a.yline;
  const float c1 = a.c1, c2 = a.c2, DT = a.dt, dth = a.dth, dh1 = a.dh1;
  const float dcy = LDG(a.dcrjy + j), dcz = LDG(a.dcrjz + k);
  const long long col = (long long)j * Y + k;
  const bool top = a.fs && (k == a.ktop);
  const bool top1 = a.fs && (k == a.ktop - 1);

  const float* __restrict__ U = a.u1 + col;
  const float* __restrict__ V = a.v1 + col;
  const float* __restrict__ W = a.w1 + col;
  const float* __restrict__ LAM = a.lam + col;
  const float* __restrict__ MU = a.mu + col;
  const float* __restrict__ QP = a.qp + col;
  const float* __restrict__ QS = a.qs + col;
  float* __restrict__ SG[6] = {a.xx + col, a.yy + col, a.zz + col,
                               a.xy + col, a.xz + col, a.yz + col};
  float* __restrict__ RR[6] = {a.r1 + col, a.r2 + col, a.r3 + col,
                               a.r4 + col, a.r5 + col, a.r6 + col};

  long long o = (long long)ib * S;
  float u_m1 = LDG(U + o - S), u_0 = LDG(U + o), u_p1 = LDG(U + o + S);
  float v_m2 = LDG(V + o - 2 * S), v_m1 = LDG(V + o - S), v_0 = LDG(V + o);
  float w_m2 = LDG(W + o - 2 * S), w_m1 = LDG(W + o - S), w_0 = LDG(W + o);
  Plane4 lam_c = load4(LAM + o, Y), mu_c = load4(MU + o, Y);
  Plane4 qp_c{0.f, 0.f, 0.f, 0.f}, qs_c{0.f, 0.f, 0.f, 0.f};
  if (!ELASTIC) {
    qp_c = load4(QP + o, Y);
    qs_c = load4(QS + o, Y);
  }

  for (int i = ib; i <= ie; ++i, o += S) {
    // ---- every load of this iteration first (independent, all in flight) ----
    float sg[6], rr[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) sg[q] = SG[q][o];
    if (!ELASTIC) {
#pragma unroll
      for (int q = 0; q < 6; ++q) rr[q] = RR[q][o];
    }
    const float u_p2 = LDG(U + o + 2 * S);
    const float v_p1 = LDG(V + o + S);
    const float w_p1 = LDG(W + o + S);
    const Plane4 lam_n = load4(LAM + o + S, Y), mu_n = load4(MU + o + S, Y);
    Plane4 qp_n{0.f, 0.f, 0.f, 0.f}, qs_n{0.f, 0.f, 0.f, 0.f};
    if (!ELASTIC) {
      qp_n = load4(QP + o + S, Y);
      qs_n = load4(QS + o + S, Y);
    }
    const float u_jp1 = LDG(U + o + Y), u_jp2 = LDG(U + o + 2 * Y), u_jm1 = LDG(U + o - Y);
    const float u_km1 = LDG(U + o - 1);
    const float v_jm1 = LDG(V + o - Y), v_jp1 = LDG(V + o + Y), v_jm2 = LDG(V + o - 2 * Y);
    const float v_km1 = LDG(V + o - 1);
    const float w_km1 = LDG(W + o - 1), w_km2 = LDG(W + o - 2);
    const float w_jp1 = LDG(W + o + Y), w_jp2 = LDG(W + o + 2 * Y), w_jm1 = LDG(W + o - Y);
    float uk1 = LDG(U + o + 1), vk1 = LDG(V + o + 1), wk1 = LDG(W + o + 1);
    float uk2 = LDG(U + o + 2), vk2 = LDG(V + o + 2);

    // memory-variable coefficients for this cell
    float f_vx1, f_vx2, f_wwo;
    int cidx;
    if (TEXARR) {
      const long long p = col + o;
      f_vx1 = LDG(a.vx1 + p);
      f_vx2 = LDG(a.vx2 + p);
      f_wwo = LDG(a.wwo + p);
      cidx = 2 * LDG(a.ww + p) - 2;
    } else {
      const int t = awp_tex_index(a.tex, i, j, k);
      f_vx1 = a.tex.tau1[t];
      f_vx2 = a.tex.tau2[t];
      f_wwo = a.tex.wwo8[t];
      cidx = 2 * t;
    }
    const float dcrj = LDG(a.dcrjx + i) * dcy * dcz;

    float cc0 = 0.f, cc1 = 0.f;
    if (!ELASTIC) {
      if (a.coeff_dev) {
        cc0 = LDG(a.coeff_dev + cidx);
        cc1 = LDG(a.coeff_dev + cidx + 1);
      } else {
        cc0 = a.coeff[cidx];
        cc1 = a.coeff[cidx + 1];
      }
    }
    const AwpStrCoef cf = awp_stress_coef<ELASTIC>(
        sum8(lam_c, lam_n), sum8(mu_c, mu_n), mu_c.a, mu_c.c, mu_c.b, mu_n.a,
        sum8(qp_c, qp_n), sum8(qs_c, qs_n), qs_c.a, qs_c.c, qs_c.b, qs_n.a, f_vx1, f_vx2, f_wwo,
        cc0, cc1, a.qthr, dth, dh1, DT);

    // velocities at k+1 / k+2 that fall on the free-surface image layer
    // (computed here in registers; kernel.cu:1087-1112)
    if (top) {
      const float uimg = u_0 - (w_0 - w_m1);
      const float vimg = v_0 - (w_jp1 - w_0);
      const float vs1 = (i < a.gx_lim) ? u_p1 - (w_p1 - w_0) : 0.0f;
      const float vs2 = (j >= a.gy_min) ? v_jm1 - (w_0 - w_jm1) : 0.0f;
      const float wimg = __fmaf_rn(
          -LDG(a.lam_mu + (long long)i * a.lam_mu_ld + j),
          __fadd_rn(__fadd_rn(__fadd_rn(vs1 - uimg, u_p1 - u_0), vimg - vs2), v_0 - v_jm1), w_km1);
      a.u1[col + o + 1] = uimg;
      a.v1[col + o + 1] = vimg;
      a.w1[col + o + 1] = wimg;
      uk1 = uimg;
      vk1 = vimg;
      wk1 = wimg;
    } else if (top1) {
      uk2 = uk1 - (wk1 - LDG(W + o - S + 1));
      vk2 = vk1 - (LDG(W + o + Y + 1) - wk1);
    }

    float d[9];
    d[0] = awp_d4(c1, c2, u_p1, u_0, u_p2, u_m1);
    d[1] = awp_d4(c1, c2, v_0, v_jm1, v_jp1, v_jm2);
    d[2] = awp_d4(c1, c2, w_0, w_km1, wk1, w_km2);
    d[3] = awp_d4(c1, c2, u_jp1, u_0, u_jp2, u_jm1);
    d[4] = awp_d4(c1, c2, v_0, v_m1, v_p1, v_m2);
    d[5] = awp_d4(c1, c2, uk1, u_0, uk2, u_km1);
    d[6] = awp_d4(c1, c2, w_0, w_m1, w_p1, w_m2);
    d[7] = awp_d4(c1, c2, vk1, v_0, vk2, v_km1);
    d[8] = awp_d4(c1, c2, w_jp1, w_0, w_jp2, w_jm1);

    awp_stress_update<ELASTIC>(sg, rr, cf, f_vx1, f_vx2, f_wwo, DT, dcrj, d);
#pragma unroll
    for (int q = 0; q < 6; ++q) SG[q][o] = sg[q];
    if (!ELASTIC) {
#pragma unroll
      for (int q = 0; q < 6; ++q) RR[q][o] = rr[q];
    }

    u_m1 = u_0; u_0 = u_p1; u_p1 = u_p2;
    v_m2 = v_m1; v_m1 = v_0; v_0 = v_p1;
    w_m2 = w_m1; w_m1 = w_0; w_0 = w_p1;
    lam_c = lam_n;
    mu_c = mu_n;
    if (!ELASTIC) {
      qp_c = qp_n;
      qs_c = qs_n;
    }
  }
}

template <bool ELASTIC, bool TEXARR, int TY>
__global__ void __launch_bounds__(32 * TY, TY == 8 ? 2 : 1)
    k_stress(const StrArgs a, const int ichunk) {
  str_tile<ELASTIC, TEXARR, TY>(a, blockIdx.x, blockIdx.y, blockIdx.z, ichunk, threadIdx.x,
                                threadIdx.y);
}

// ===========================================================================
// Free-surface stress imaging (fstr, kernel.cu:1616-1647)
// ===========================================================================
__device__ __forceinline__ void fstr_cell(const FstrArgs& a, const int i, const int j) {
  if (j > a.j1 || i > a.i1) return;
  const long long p = (long long)i * a.slice + (long long)j * a.yline + a.ktop;
  // all six reads before the first write (each write could alias a later
  // read, so in store order every read would wait a full memory round trip)
  const float zz0 = a.zz[p], zz1 = a.zz[p - 1];
  const float xz1 = a.xz[p - 1], xz2 = a.xz[p - 2];
  const float yz1 = a.yz[p - 1], yz2 = a.yz[p - 2];
  a.zz[p + 1] = -zz0;
  a.zz[p + 2] = -zz1;
  a.xz[p + 1] = -xz1;
  a.xz[p + 2] = -xz2;
  a.yz[p + 1] = -yz1;
  a.yz[p + 2] = -yz2;
  a.xz[p] = 0.0f;
  a.yz[p] = 0.0f;
}

__global__ void k_fstr(const FstrArgs a) {
  fstr_cell(a, a.i0 + blockIdx.y, a.j0 + blockIdx.x * blockDim.x + threadIdx.x);
}

// ===========================================================================
// Point sources (addsrc_cu, kernel.cu:1780-1806)
// ===========================================================================
__device__ __forceinline__ long long src_cell(const int* psrc, int s, int dim, int S, int Y) {
  const int idx = psrc[s * dim] + 1 + AWP_NGSL;
  const int idy = psrc[s * dim + 1] + 1 + AWP_NGSL;
  const int idz = psrc[s * dim + 2] + AWP_ALIGN - 1;
  return (long long)idx * S + (long long)idy * Y + idz;
}

__global__ void k_addsrc_direct(const SrcArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.ncell) return;
  const long long p = src_cell(a.psrc, s, a.dim, a.slice, a.yline);
  const long long t = (long long)s * a.stride + a.tidx;
  a.xx[p] = a.xx[p] - a.vtst * a.axx[t];
  a.yy[p] = a.yy[p] - a.vtst * a.ayy[t];
  a.zz[p] = a.zz[p] - a.vtst * a.azz[t];
  a.xz[p] = a.xz[p] - a.vtst * a.axz[t];
  a.yz[p] = a.yz[p] - a.vtst * a.ayz[t];
  a.xy[p] = a.xy[p] - a.vtst * a.axy[t];
}

__device__ __forceinline__ void addsrc_cell(const SrcArgs& a, const int c) {
  const long long p = a.cell_pos[c];
  float sxx = a.xx[p], syy = a.yy[p], szz = a.zz[p];
  float sxz = a.xz[p], syz = a.yz[p], sxy = a.xy[p];
  for (int n = a.cell_first[c]; n < a.cell_first[c + 1]; ++n) {
    const long long s = (long long)a.order[n] * a.stride + a.tidx;
    sxx = sxx - a.vtst * a.axx[s];
    syy = syy - a.vtst * a.ayy[s];
    szz = szz - a.vtst * a.azz[s];
    sxz = sxz - a.vtst * a.axz[s];
    syz = syz - a.vtst * a.ayz[s];
    sxy = sxy - a.vtst * a.axy[s];
  }
  a.xx[p] = sxx;
  a.yy[p] = syy;
  a.zz[p] = szz;
  a.xz[p] = sxz;
  a.yz[p] = syz;
  a.xy[p] = sxy;
}

__global__ void k_addsrc(const SrcArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  addsrc_cell(a, c);
}

// ===========================================================================
// Kinematic finite-fault source (addkinsrc_cu + compmt/brune/liu/lfilter,
// kernel.cu:3706-3858)
// ===========================================================================
__device__ void compmt(float str, float dip, float rake, float* xx, float* yy,
                       float* zz, float* xz, float* yz, float* xy) {
  *yy = -(sinf(dip) * cosf(rake) * sinf(2. * str) +
          sinf(2. * dip) * sinf(rake) * sinf(str) * sinf(str));
  *xy = sinf(dip) * cosf(rake) * cosf(2. * str) +
        0.5 * (sinf(2. * dip) * sinf(rake) * sinf(2. * str));
  *yz = (cosf(dip) * cosf(rake) * cosf(str) + cosf(2. * dip) * sinf(rake) * sinf(str));
  *xx = sinf(dip) * cosf(rake) * sinf(2. * str) -
        sinf(2. * dip) * sinf(rake) * cosf(str) * cosf(str);
  *xz = (cosf(dip) * cosf(rake) * sinf(str) - cosf(2. * dip) * sinf(rake) * cosf(str));
  *zz = sinf(2. * dip) * sinf(rake);
}

__device__ float stf_brune(float freq, float time) {
  const float omega = freq * M_PI * 2.;
  return (time > 0.) ? powf(omega, 2.) * time * expf(-omega * time) : 0.f;
}

__device__ float stf_liu(float tau, float time) {
  const float tau1 = 0.13 * tau;
  const float tau2 = tau - tau1;
  const float CN = M_PI / (1.4 * M_PI * tau1 + 1.2 * tau1 + 0.3 * M_PI * tau2);
  float stf;
  if (time < tau1)
    stf = CN * (0.7 - 0.7 * cosf(M_PI * time / tau1) + 0.6 * sinf(0.5 * M_PI * time / tau1));
  else if (time < 2 * tau1)
    stf = CN * (1.0 - 0.7 * cosf(M_PI * time / tau1) + 0.3 * cosf(M_PI * (time - tau1) / tau2));
  else if (time < tau)
    stf = CN * (0.3 + 0.3 * cosf(M_PI * (time - tau1) / tau2));
  else
    stf = 0.;
  return stf;
}

// Direct-form II transposed IIR/FIR step (same recursion as scipy lfilter).
__device__ double iir_step(int order, const double* b, const double* aa, double x,
                           double* d) {
  const double y = (b[0] * x + d[0]) / aa[0];
  for (int n = 0; n < order - 1; n++) d[n] = b[n + 1] * x - aa[n + 1] * y + d[n + 1];
  d[order - 1] = b[order] * x - aa[order] * y;
  return y;
}

__device__ __forceinline__ void addkinsrc_cell(const KinSrcArgs& a, const int c, const int step) {
  const bool direct = a.cell_pos == nullptr;
  const long long p = direct ? src_cell(a.psrc, c, a.dim, a.slice, a.yline) : a.cell_pos[c];
  const float atime = step * a.dt;
  float sxx = a.xx[p], syy = a.yy[p], szz = a.zz[p];
  float sxz = a.xz[p], syz = a.yz[p], sxy = a.xy[p];
  const int n0 = direct ? 0 : a.cell_first[c], n1 = direct ? 1 : a.cell_first[c + 1];
  for (int n = n0; n < n1; ++n) {
    const int s = direct ? c : a.order[n];
    const int stf_type = (int)a.axx[2 * s];
    const float slip = a.ayy[2 * s];
    const float ruptime = a.azz[2 * s];
    const float risetime = a.axz[2 * s];
    if (!(atime > ruptime)) continue;
    const float area = a.ayz[2 * s];
    const float strike = a.axx[2 * s + 1] / 180. * M_PI;
    const float dip = a.ayy[2 * s + 1] / 180. * M_PI;
    const float rake = a.azz[2 * s + 1] / 180. * M_PI;
    float mxx, myy, mzz, mxz, myz, mxy;
    compmt(strike, dip, rake, &mxx, &myy, &mzz, &mxz, &myz, &mxy);
    float stf;
    if (stf_type == 1.0f) {
      const float freq = 1. / risetime;
      stf = stf_brune(freq, atime - ruptime);
    } else if (stf_type == 2.0f) {
      stf = stf_liu(risetime, atime - ruptime);
    } else {
      stf = 0.;
    }
    if (a.filtorder > 0)
      stf = (float)iir_step(a.filtorder, a.filt_b, a.filt_a, (double)stf,
                            a.filt_state + (long long)s * (a.filtorder + 1));
    stf *= slip * area / a.mu[p];
    a.mom[s] += stf * a.dt;
    stf *= a.vtst;
    sxx = sxx - stf * mxx;
    syy = syy - stf * myy;
    szz = szz - stf * mzz;
    sxz = sxz - stf * mxz;
    syz = syz - stf * myz;
    sxy = sxy - stf * mxy;
  }
  a.xx[p] = sxx;
  a.yy[p] = syy;
  a.zz[p] = szz;
  a.xz[p] = sxz;
  a.yz[p] = syz;
  a.xy[p] = sxy;
}

__global__ void k_addkinsrc(const KinSrcArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  addkinsrc_cell(a, c, a.step);
}

// ===========================================================================
// Plasticity (drprecpc_calc_opt / drprecpc_app / rotate_principal)
// ===========================================================================
// One component (I, J) of rotate_principal (the initial stress in the model
// frame): ssp = Rz^T diag(s fmajor, s, s fminor) Rz - pfluid I with
// s = sigma2 + pfluid, both products summed over k = 0, 1, 2 in order as the
// reference's matmul.  In the first product the two off-diagonal terms of
// each sum multiply an exact zero and add +-0, so its entry (I, k) is the one
// rounded product RzT[I][k] * diag[k]; forming only that product and only the
// components a kernel uses gives the same bits as the full 3 x 3 products.
template <int I, int J>
__device__ __forceinline__ float principal(const PlastParams& pp, float sigma2, float pfluid) {
  const float s = sigma2 + pfluid;
  const float d0 = s * pp.fmajor, d2 = s * pp.fminor;
  const float t0 = pp.RzT[I * 3 + 0] * d0, t1 = pp.RzT[I * 3 + 1] * s,
              t2 = pp.RzT[I * 3 + 2] * d2;
  float c = 0.f;
  c += t0 * pp.Rz[0 * 3 + J];
  c += t1 * pp.Rz[1 * 3 + J];
  c += t2 * pp.Rz[2 * 3 + J];
  if (I == J) c -= pfluid;
  return c;
}

__device__ __forceinline__ float pfluid_at(const PlastParams& pp, int k) {
  const float depth = (float)(pp.ktop - k) * pp.dh;
  return (depth > 0) ? (depth + pp.dh * 0.5) * 9.81e3 : pp.dh / 2. * 9.81e3;
}

__global__ void k_plast_calc(const PlastCalcArgs a) {
  const int k = a.k0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = a.j0 + blockIdx.y * blockDim.y + threadIdx.y;
  const int i = a.i0 + blockIdx.z;
  if (k > a.k1 || j > a.j1 || i > a.i1) return;
  const PlastParams& pp = a.p;
  const int S = a.slice, Y = a.yline;
  const long long pos = (long long)i * S + (long long)j * Y + k;
  const long long pos_ip1 = pos + S, pos_jm1 = pos - Y, pos_km1 = pos - 1;
  const float pfluid = pfluid_at(pp, k);
  const float s2 = a.sigma2[pos], s2_ip1 = a.sigma2[pos_ip1];
  const float iixx = 0.5f * (principal<0, 0>(pp, s2, pfluid) + principal<0, 0>(pp, s2_ip1, pfluid));
  const float iiyy = 0.5f * (principal<1, 1>(pp, s2, pfluid) + principal<1, 1>(pp, s2_ip1, pfluid));
  const float iizz = 0.5f * (principal<2, 2>(pp, s2, pfluid) + principal<2, 2>(pp, s2_ip1, pfluid));
  float Sxx = a.xx[pos] + iixx;
  float Syy = a.yy[pos] + iiyy;
  float Szz = a.zz[pos] + iizz;
  float Sxz = 0.25f * (a.xz[pos] + a.xz[pos_ip1] + a.xz[pos_km1] + a.xz[pos_ip1 - 1]) +
              0.5f * (principal<0, 2>(pp, s2, pfluid) + principal<0, 2>(pp, s2_ip1, pfluid));
  float Syz = 0.25f * (a.yz[pos] + a.yz[pos_jm1] + a.yz[pos_km1] + a.yz[pos_jm1 - 1]) +
              0.5f * (principal<1, 2>(pp, s2, pfluid) + principal<1, 2>(pp, s2_ip1, pfluid));
  float Sxy = 0.25f * (a.xy[pos] + a.xy[pos_ip1] + a.xy[pos_jm1] + a.xy[pos_ip1 - Y]) +
              0.5f * (principal<0, 1>(pp, s2, pfluid) + principal<0, 1>(pp, s2_ip1, pfluid));
  const float mu_i = a.mu[pos], mu_ip1 = a.mu[pos_ip1];
  const float Tv = pp.dh / sqrt(1.0f / (mu_i * a.d1[pos]));
  const float Sxxp = Sxx, Syyp = Syy, Szzp = Szz, Sxyp = Sxy, Sxzp = Sxz, Syzp = Syz;
  const float rphi = a.phi[pos] * 0.017453292519943295f;
  const float sigma_m = (Sxx + Syy + Szz) / 3.0f;
  const float SDxx = Sxx - sigma_m, SDyy = Syy - sigma_m, SDzz = Szz - sigma_m;
  const float secinv =
      0.5f * (SDxx * SDxx + SDyy * SDyy + SDzz * SDzz) + Sxz * Sxz + Sxy * Sxy + Syz * Syz;
  const float sqrtSecinv = sqrt(secinv);
  const float taulim2 = a.cohes[pos] * cos(rphi) - (sigma_m + pfluid) * sin(rphi);
  const float taulim = (taulim2 > 0.0f) ? taulim2 : 0.0f;
  float iyldfac;
  if (sqrtSecinv > taulim) {
    iyldfac = taulim / sqrtSecinv + (1.0f - taulim / sqrtSecinv) * exp(-pp.dt / Tv);
    Sxx = SDxx * iyldfac + sigma_m;
    Syy = SDyy * iyldfac + sigma_m;
    Szz = SDzz * iyldfac + sigma_m;
    Sxz = Sxz * iyldfac;
    Sxy = Sxy * iyldfac;
    Syz = Syz * iyldfac;
  } else {
    iyldfac = 1.0f;
  }
  if (iyldfac < 1.0f) {
    const float xm = 2.0f / (mu_i + mu_ip1);
    const float depxx = (Sxx - Sxxp) / xm, depyy = (Syy - Syyp) / xm,
                depzz = (Szz - Szzp) / xm, depxy = (Sxy - Sxyp) / xm,
                depxz = (Sxz - Sxzp) / xm, depyz = (Syz - Syzp) / xm;
    const float inc = sqrt(0.5f * (depxx * depxx + depyy * depyy + depzz * depzz) +
                           2.0f * (depxy * depxy + depxz * depxz + depyz * depyz));
    const int mult = a.neta_mult ? a.neta_mult[(long long)i * a.neta_ld + j] : 1;
    float eta = a.neta[pos];
    for (int m = 0; m < mult; ++m) eta = eta + inc;
    a.neta[pos] = eta;
    a.yldfac[pos] = iyldfac;
  } else {
    a.yldfac[pos] = 1.0f;
  }
}

__global__ void k_plast_app(const PlastAppArgs a) {
  const int k = a.k0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = a.j0 + blockIdx.y * blockDim.y + threadIdx.y;
  const int i = a.i0 + blockIdx.z;
  if (k > a.k1 || j > a.j1 || i > a.i1) return;
  const PlastParams& pp = a.p;
  const int S = a.slice, Y = a.yline;
  const long long pos = (long long)i * S + (long long)j * Y + k;
  const long long pos_im1 = pos - S, pos_ip1 = pos + S, pos_jp1 = pos + Y,
                  pos_kp1 = pos + 1;
  const long long pos_im1jp1 = pos_im1 + Y, pos_im1kp1 = pos_im1 + 1,
                  pos_ip1jp1 = pos_ip1 + Y, pos_ip1kp1 = pos_ip1 + 1,
                  pos_jp1kp1 = pos_jp1 + 1, pos_ip1jp1kp1 = pos_ip1 + Y + 1;
  const float depth = (float)(pp.ktop - k) * pp.dh;
  const float depth_kp1 = (float)(pp.ktop - k + 1) * pp.dh;
  const float pfluid = (depth > 0) ? (depth + pp.dh / 2.) * 9.81e3 : pp.dh / 2. * 9.81e3;
  const float pfluid_kp1 =
      (depth_kp1 > 0) ? (depth_kp1 + pp.dh / 2.) * 9.81e3 : pp.dh / 2. * 9.81e3;
  // every input first (the yield factors, the cell's stresses and the eight
  // sigma2 of its stencil), so the loads overlap instead of following the
  // branches one after another; the branches then read registers.  The
  // reference's double-precision scalings here (0.5, 0.25, 0.125 and the
  // division by 3 of a float sum, rounded back to float) are formed in float:
  // the scalings are exact, and for float operands the double quotient
  // rounded to float is the correctly rounded float quotient (double rounding
  // is innocuous for division at 53 >= 2 * 24 + 2 bits; Figueroa 1995).
  const float yf = a.yldfac[pos], y_im1 = a.yldfac[pos_im1], y_kp1 = a.yldfac[pos_kp1],
              y_jp1 = a.yldfac[pos_jp1], y_im1kp1 = a.yldfac[pos_im1kp1],
              y_jp1kp1 = a.yldfac[pos_jp1kp1], y_im1jp1 = a.yldfac[pos_im1jp1];
  const float sxx = a.xx[pos], syy = a.yy[pos], szz = a.zz[pos], sxz = a.xz[pos],
              syz = a.yz[pos], sxy = a.xy[pos];
  const float s2 = a.sigma2[pos], s2_ip1 = a.sigma2[pos_ip1], s2_kp1 = a.sigma2[pos_kp1],
              s2_jp1 = a.sigma2[pos_jp1], s2_ip1kp1 = a.sigma2[pos_ip1kp1],
              s2_ip1jp1 = a.sigma2[pos_ip1jp1], s2_jp1kp1 = a.sigma2[pos_jp1kp1],
              s2_ip1jp1kp1 = a.sigma2[pos_ip1jp1kp1];
  if (yf < 1.f) {
    const float iixx =
        0.5f * (principal<0, 0>(pp, s2, pfluid) + principal<0, 0>(pp, s2_ip1, pfluid_kp1));
    const float iiyy =
        0.5f * (principal<1, 1>(pp, s2, pfluid) + principal<1, 1>(pp, s2_ip1, pfluid_kp1));
    const float iizz =
        0.5f * (principal<2, 2>(pp, s2, pfluid) + principal<2, 2>(pp, s2_ip1, pfluid_kp1));
    const float Sxx = sxx + iixx, Syy = syy + iiyy, Szz = szz + iizz;
    const float sigma_m = __fdiv_rn(Sxx + Syy + Szz, 3.0f);
    const float SDxx = sxx + iixx - sigma_m;
    const float SDyy = syy + iiyy - sigma_m;
    const float SDzz = szz + iizz - sigma_m;
    a.xx[pos] = SDxx * yf + sigma_m - iixx;
    a.yy[pos] = SDyy * yf + sigma_m - iiyy;
    a.zz[pos] = SDzz * yf + sigma_m - iizz;
  }
  float iyldfac = 0.25f * (y_im1 + yf + y_im1kp1 + y_kp1);
  if (iyldfac < 1.f) {
    const float iist =
        0.5f * (principal<0, 2>(pp, s2, pfluid) + principal<0, 2>(pp, s2_kp1, pfluid_kp1));
    a.xz[pos] = (sxz + iist) * iyldfac - iist;
  }
  iyldfac = 0.25f * (yf + y_jp1 + y_jp1kp1 + y_kp1);
  if (iyldfac < 1.f) {
    const float iist = 0.125f * (principal<1, 2>(pp, s2, pfluid) +
                                principal<1, 2>(pp, s2_ip1, pfluid) +
                                principal<1, 2>(pp, s2_kp1, pfluid_kp1) +
                                principal<1, 2>(pp, s2_ip1kp1, pfluid_kp1) +
                                principal<1, 2>(pp, s2_jp1, pfluid) +
                                principal<1, 2>(pp, s2_ip1jp1, pfluid) +
                                principal<1, 2>(pp, s2_jp1kp1, pfluid_kp1) +
                                principal<1, 2>(pp, s2_ip1jp1kp1, pfluid_kp1));
    a.yz[pos] = (syz + iist) * iyldfac - iist;
  }
  iyldfac = 0.25f * (yf + y_jp1 + y_im1 + y_im1jp1);
  if (iyldfac < 1.f) {
    const float iist =
        0.5f * (principal<0, 1>(pp, s2, pfluid) + principal<0, 1>(pp, s2_jp1, pfluid));
    a.xy[pos] = (sxy + iist) * iyldfac - iist;
  }
}

// ===========================================================================
// Plane-wave source (IFAULT 6)
// ===========================================================================
// addplanesrc_cu (kernel.cu:3897-3925): a plane-wave source (IFAULT 6) on the
// level k = align + ND + 1 of every (i, j) from 4 to nxt+7 (nyt+7), the
// launched rows rounded up to the shipped 2 x 2 blocks.  The reference forms
// the increments in double.
__global__ void k_addplanesrc(const PlaneSrcArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.nx || j >= a.ny) return;
  const long long pos = (long long)(i + 4) * a.slice + (long long)(j + 4) * a.yline + a.k;
  const float vtst = a.DT / a.DH;  // float quotient, as the reference forms it
  const double v2 = __dmul_rn((double)vtst, 2.0);
  const double mu = a.mu[pos], la = a.lambda[pos];
  a.xz[pos] = (float)__fma_rn(-__ddiv_rn(v2, mu), (double)a.axx[a.n], (double)a.xz[pos]);
  a.yz[pos] = (float)__fma_rn(-__ddiv_rn(v2, mu), (double)a.ayy[a.n], (double)a.yz[pos]);
  a.xx[pos] = (float)__fma_rn(-__ddiv_rn(v2, la), (double)a.azz[a.n], (double)a.xx[pos]);
  a.yy[pos] = (float)__fma_rn(-__ddiv_rn(v2, la), (double)a.azz[a.n], (double)a.yy[pos]);
  a.zz[pos] = (float)__fma_rn(-__ddiv_rn(v2, __fma_rn(2.0, mu, la)), (double)a.azz[a.n],
                              (double)a.zz[pos]);
}

// ===========================================================================
// Output gather (velbuffer, kernel.cu:3948-4011)
// ===========================================================================
__global__ void k_velbuffer(const VelBufArgs a) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z * blockDim.z + threadIdx.z;
  const int i = 2 + AWP_NGSL + a.nbgx + ix * a.nskpx;
  const int j = 2 + AWP_NGSL + a.nbgy + iy * a.nskpy;
  const int k = a.nbgz + iz * a.nskpz;
  if (i > 2 + AWP_NGSL + a.nedx || j > 2 + AWP_NGSL + a.nedy || k > a.nedz) return;
  int ko, koz;
  if (a.bathy) {
    const int b = a.bathy[(long long)j * a.bathy_ld + i];
    ko = b - k;
    koz = (b == a.ktop) ? ko - 1 : ko;
  } else {
    ko = a.ktop - k;
    koz = ko - a.w_shift;
  }
  const long long col = (long long)i * a.slice + (long long)j * a.yline;
  const long long pos = col + ko;
  const long long idx = (long long)iz * a.rec_nxt * a.rec_nyt + (long long)iy * a.rec_nxt + ix;
  a.bufx[idx] = a.u1[pos];
  a.bufy[idx] = a.v1[pos];
  a.bufz[idx] = a.w1[col + koz];
  if (a.nve == 3 && a.bufeta) a.bufeta[idx] = a.neta[pos];
}

// ===========================================================================
// Media mapping (inimesh per-cell body, mesh.c:222-466)
//
// The reference runs this on the host, compiled without FMA contraction and
// with IEEE float division.  Every rounding step is therefore spelled out with
// the _rn intrinsics so that the device result is the same bit pattern.
// ===========================================================================
struct cplx {
  double re, im;
};
// Complex division in the scaled form used by C99 (libgcc __divdc3).
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  if (fabs(b.re) < fabs(b.im)) {
    const double r = __ddiv_rn(b.re, b.im);
    const double den = __dadd_rn(__dmul_rn(b.re, r), b.im);
    return {__ddiv_rn(__dadd_rn(__dmul_rn(a.re, r), a.im), den),
            __ddiv_rn(__dsub_rn(__dmul_rn(a.im, r), a.re), den)};
  } else {
    const double r = __ddiv_rn(b.im, b.re);
    const double den = __dadd_rn(__dmul_rn(b.im, r), b.re);
    return {__ddiv_rn(__dadd_rn(__dmul_rn(a.im, r), a.re), den),
            __ddiv_rn(__dsub_rn(a.im, __dmul_rn(a.re, r)), den)};
  }
}

// Unrelaxed modulus for one wave type (mesh.c:313-351 / 359-391).
__device__ float q_modulus(const MediaArgs& a, float dd, float v, float q) {
  const float ddvv = __fmul_rn(__fmul_rn(dd, v), v);
  if (q > 200.0) {
    float val0 = 0.0f;
    for (int t = 0; t < 8; ++t) {
      const float wt2 =
          __fmul_rn(__fmul_rn(__fmul_rn(a.w0, a.w0), a.tau[t]), a.tau[t]);
      const float denom = (float)__dmul_rn(
          __dmul_rn(__dadd_rn((double)wt2, 1.0), (double)q), (double)a.facex);
      val0 = __fadd_rn(val0, __fdiv_rn(a.weights[t], denom));
    }
    return (float)__ddiv_rn((double)ddvv, __dsub_rn(1.0, (double)val0));
  } else if (q > 0.) {
    cplx value{0.0, 0.0};
    for (int t = 0; t < 8; ++t) {
      const float wl = __fadd_rn(__fdiv_rn(a.coeff[2 * t], __fmul_rn(q, q)),
                                 __fdiv_rn(a.coeff[2 * t + 1], q));
      const cplx den{1.0, __dmul_rn((double)a.w0, (double)a.tau[t])};
      const cplx frac = cdiv(cplx{(double)wl, 0.0}, den);
      const cplx r = cdiv(cplx{1.0, 0.0}, cplx{__dsub_rn(1.0, frac.re), -frac.im});
      value.re = __dadd_rn(value.re, r.re);
      value.im = __dadd_rn(value.im, r.im);
    }
    value = cdiv(cplx{1.0, 0.0}, value);
    return (float)__ddiv_rn((double)ddvv, __dmul_rn(8., value.re));
  }
  return ddvv;
}

__device__ __forceinline__ unsigned int warp_min_u(unsigned int v) {
  for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned int warp_max_u(unsigned int v) {
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void k_media(const MediaArgs a) {
  const long long n = (long long)a.nxt * a.nyt * a.nzt;
  // non-negative floats order like their bit patterns
  unsigned int e[6] = {0x7f800000u, 0u, 0x7f800000u, 0u, 0x7f800000u, 0u};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % a.nxt);
    const int j = (int)((c / a.nxt) % a.nyt);
    const int k = (int)(c / ((long long)a.nxt * a.nyt));
    const float* m = a.media + c * a.nvar + a.var_offset;
    float vp = m[0], vs = m[1], dd = m[2];
    float pq = 0.f, sq = 0.f;
    if (a.nvar > 3) {
      pq = m[3];
      sq = m[4];
    } else if (a.nve == 1 || a.nve == 3) {
      sq = (float)__dmul_rn(0.05, (double)vs);
      pq = (float)__dmul_rn(2.0, (double)sq);
    }
    vp = (float)sqrt((double)__fdiv_rn(q_modulus(a, dd, vp, pq), dd));
    vs = (float)sqrt((double)__fdiv_rn(q_modulus(a, dd, vs, sq), dd));
    if (vs == 0.f) {
      sq = 50.;
      pq = 100.;
    }
    if (a.socalq == 1) {
      const float vpvs = __fdiv_rn(vp, vs);
      if (vpvs < 1.45) vs = (float)__ddiv_rn((double)vp, 1.45);
    }
    const long long p = (long long)(i + 2 + AWP_NGSL) * a.slice +
                        (long long)(j + 2 + AWP_NGSL) * a.yline +
                        (a.nzt + AWP_ALIGN - 1 - k);
    if (vs > 1.0f) e[0] = min(e[0], __float_as_uint(vs));
    e[1] = max(e[1], __float_as_uint(fmaxf(vs, 0.f)));
    e[2] = min(e[2], __float_as_uint(fmaxf(vp, 0.f)));
    e[3] = max(e[3], __float_as_uint(fmaxf(vp, 0.f)));
    e[4] = min(e[4], __float_as_uint(fmaxf(dd, 0.f)));
    e[5] = max(e[5], __float_as_uint(fmaxf(dd, 0.f)));
    a.mu[p] = (float)__ddiv_rn(1., (double)__fmul_rn(__fmul_rn(dd, vs), vs));
    const double vp2 = (double)__fmul_rn(vp, vp);
    const double vs2 = __dmul_rn(__dmul_rn(2., (double)vs), (double)vs);
    a.lam[p] = (float)__ddiv_rn(1., __dmul_rn((double)dd, __dsub_rn(vp2, vs2)));
    a.d1[p] = dd;
    if (a.nve == 1 || a.nve == 3) {
      float qpinv, qsinv;
      if (pq <= 0.0) {
        qpinv = 0.0;
        qsinv = 0.0;
      } else {
        qpinv = (float)__ddiv_rn(1., (double)pq);
        qsinv = (float)__ddiv_rn(1., (double)sq);
      }
      a.qp[p] = __fdiv_rn(qpinv, a.facex);
      a.qs[p] = __fdiv_rn(qsinv, a.facex);
    }
  }
  if (a.ext) {
    for (int q = 0; q < 6; q += 2) {
      const unsigned int lo = warp_min_u(e[q]), hi = warp_max_u(e[q + 1]);
      if ((threadIdx.x & 31) == 0) {
        atomicMin(a.ext + q, lo);
        atomicMax(a.ext + q + 1, hi);
      }
    }
  }
}

// Ghost-layer fill of d1/mu/lam one cell beyond the interior and the qp/qs copy
// above the surface (mesh.c:468-591).  One thread per (i,j) column of the
// padded plane; each writes only cells of its own column.
__global__ void k_media_borders(float* d1, float* mu, float* lam, float* qp, float* qs,
                                const AwpGeom g, int nve) {
  const int i = blockIdx.y;                                   // 0 .. nx_pad-1
  const int j = blockIdx.x * blockDim.x + threadIdx.x;        // 0 .. ny_pad-1
  if (i >= g.nx_pad() || j >= g.ny_pad()) return;
  const int lo = 2 + AWP_NGSL, hix = g.nxt + 1 + AWP_NGSL, hiy = g.nyt + 1 + AWP_NGSL;
  const int kb = AWP_ALIGN, kt = g.nzt + AWP_ALIGN - 1;
  const bool xin = (i >= lo && i <= hix), yin = (j >= lo && j <= hiy);
  const bool xg = (i == lo - 1 || i == hix + 1), yg = (j == lo - 1 || j == hiy + 1);
  // source column for ghost columns: clamp into the interior
  const int si = (i == lo - 1) ? lo : (i == hix + 1 ? hix : i);
  const int sj = (j == lo - 1) ? lo : (j == hiy + 1 ? hiy : j);
  const long long dst = (long long)i * g.slice + (long long)j * g.yline;
  const long long src = (long long)si * g.slice + (long long)sj * g.yline;
  if (xin && yin) {
    // interior column: bottom ghost (align-1) and top ghost (nzt+align)
    d1[dst + kb - 1] = d1[dst + kb];
    mu[dst + kb - 1] = mu[dst + kb];
    lam[dst + kb - 1] = lam[dst + kb];
    d1[dst + kt + 1] = d1[dst + kt];
    mu[dst + kt + 1] = mu[dst + kt];
    lam[dst + kt + 1] = lam[dst + kt];
    if (nve == 1 || nve == 3) {
      qp[dst + kt + 1] = qp[dst + kt];
      qs[dst + kt + 1] = qs[dst + kt];
    }
    return;
  }
  if (!((xg && (yin || yg)) || (yg && xin))) return;
  // Side planes, edge lines and corners (mesh.c:468-571) together make every
  // ghost column of the one-cell border a copy of the nearest interior column,
  // with its own bottom/top ghost taken from that column's bottom/top cell.
  for (int k = kb; k <= kt; ++k) {
    d1[dst + k] = d1[src + k];
    mu[dst + k] = mu[src + k];
    lam[dst + k] = lam[src + k];
  }
  d1[dst + kb - 1] = d1[src + kb];
  mu[dst + kb - 1] = mu[src + kb];
  lam[dst + kb - 1] = lam[src + kb];
  d1[dst + kt + 1] = d1[src + kt];
  mu[dst + kt + 1] = mu[src + kt];
  lam[dst + kt + 1] = lam[src + kt];
}

__global__ void k_lam_mu(const float* lam, const float* mu, float* lam_mu, const AwpGeom g,
                         int xls, int xre, int yls, int yre) {
  const int j = yls + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = xls + blockIdx.y;
  if (j > yre || i > xre) return;
  const long long p = (long long)i * g.slice + (long long)j * g.yline + g.top();
  // pmcl3d.c:944-951 runs on the host with IEEE float division
  const float t_xl = __ddiv_rn(1.0, (double)lam[p]);
  const float t_xl2m = __dadd_rn(__ddiv_rn(2.0, (double)mu[p]), (double)t_xl);
  lam_mu[(long long)i * g.ny_pad() + j] = __fdiv_rn(t_xl, t_xl2m);
}

__global__ void k_fill(float* p, float v, long long n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    p[c] = v;
}

__global__ void k_nonfinite(const float* p, long long n, unsigned int* flag) {
  unsigned int bad = 0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(p[c]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

__global__ void k_anynonzero(const float* p, long long n, unsigned int* flag) {
  unsigned int nz = 0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    nz |= (p[c] != 0.0f);
  if (__any_sync(0xffffffffu, nz) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

inline unsigned cdiv_u(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

// ===========================================================================
// Batched instances (many independent simulations, one persistent launch per
// half-step).  CTAs pull tiles (instance, tile coordinates) from a global
// counter and run the same per-tile bodies as the one-simulation kernels, so
// each instance's arithmetic is unchanged.
// ===========================================================================
__device__ __forceinline__ int next_tile(int* counter, int* s_tile) {
  __syncthreads();  // every thread has read the previous tile
  if (threadIdx.x == 0 && threadIdx.y == 0) *s_tile = atomicAdd(counter, 1);
  __syncthreads();
  return *s_tile;
}

template <int TY>
__global__ void __launch_bounds__(32 * TY)
    k_batch_velocity(const BatchInst* __restrict__ inst, const int4* __restrict__ tiles,
                     const int ntiles, int* counter, const int ichunk) {
  __shared__ int s_tile;
  for (;;) {
    const int t = next_tile(counter, &s_tile);
    if (t >= ntiles) return;
    const int4 d = tiles[t];
    const VelArgs a = inst[d.x].v;
    vel_tile<TY>(a, d.y, d.z, d.w, ichunk, threadIdx.x, threadIdx.y);
  }
}

// Elastic and anelastic instances have separate tile lists and launches, so
// each launch carries one stress variant (register pressure as k_stress).
template <bool ELASTIC, int TY>
__global__ void __launch_bounds__(32 * TY, TY == 8 ? 2 : 1)
    k_batch_stress(const BatchInst* __restrict__ inst, const int4* __restrict__ tiles,
                   const int ntiles, int* counter, const int ichunk) {
  __shared__ int s_tile;
  for (;;) {
    const int t = next_tile(counter, &s_tile);
    if (t >= ntiles) return;
    const int4 d = tiles[t];
    const StrArgs& a = inst[d.x].s;  // read in place (dynamically indexed tables)
    str_tile<ELASTIC, false, TY>(a, d.y, d.z, d.w, ichunk, threadIdx.x, threadIdx.y);
  }
}

// Sources of every instance at step *step + 1 (the step being taken), with the
// schedule of one_step: IFAULT < 4 while the step is below NST, IFAULT 5 always.
__global__ void k_batch_sources(const BatchInst* __restrict__ inst,
                                const int2* __restrict__ cells, const int n,
                                const int* __restrict__ step) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int2 e = cells[q];
  const BatchInst& I = inst[e.x];
  const int cur = *step + 1;
  if (I.ifault == 5) {
    addkinsrc_cell(I.kin, e.y, cur);
  } else if (I.ifault < 4 && cur < I.nst) {
    SrcArgs a = I.src;
    a.tidx = cur;
    addsrc_cell(a, e.y);
  }
}

// Sources of one instance at step *step + 1 read from device memory (replayable
// graphs): the schedule of one_step, IFAULT < 4 while the step is below NST.
__global__ void k_addsrc_dev(const SrcArgs a, const int* __restrict__ step, const int nst) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int cur = *step + 1;
  if (c >= a.ncell || cur >= nst) return;
  SrcArgs b = a;
  b.tidx = cur;
  addsrc_cell(b, c);
}

__global__ void k_addkinsrc_dev(const KinSrcArgs a, const int* __restrict__ step) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  addkinsrc_cell(a, c, *step + 1);
}

__global__ void k_step_advance(int* step) { *step = *step + 1; }

// Free-surface imaging of every instance (one CTA per (instance, x row)); the
// first thread then advances the batch's step counter.
__global__ void k_batch_fstr(const BatchInst* __restrict__ inst, const int2* __restrict__ rows,
                             const int n, int* step) {
  for (int r = blockIdx.x; r < n; r += gridDim.x) {
    const int2 e = rows[r];
    const FstrArgs& a = inst[e.x].f;
    for (int j = a.j0 + threadIdx.x; j <= a.j1; j += blockDim.x) fstr_cell(a, e.y, j);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *step = *step + 1;
}

// ===========================================================================
// launchers
// ===========================================================================
cudaError_t awp_launch_velocity(const VelArgs& a, cudaStream_t st) {
  const int nk = a.k1 - a.k0 + 1, nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nk <= 0 || nj <= 0 || ni <= 0) return cudaSuccess;
  const dim3 block(32, 8, 1);
  const dim3 grid(cdiv_u(nk, 32), cdiv_u(nj, 8), cdiv_u(ni, g_ichunk));
  k_velocity<8><<<grid, block, 0, st>>>(a, g_ichunk);
  return cudaGetLastError();
}

template <int TY>
static void launch_stress_ty(const StrArgs& a, bool elastic, bool texarr, dim3 grid,
                             cudaStream_t st) {
  const dim3 block(32, TY, 1);
  if (elastic) {
    if (texarr)
      k_stress<true, true, TY><<<grid, block, 0, st>>>(a, g_ichunk);
    else
      k_stress<true, false, TY><<<grid, block, 0, st>>>(a, g_ichunk);
  } else {
    if (texarr)
      k_stress<false, true, TY><<<grid, block, 0, st>>>(a, g_ichunk);
    else
      k_stress<false, false, TY><<<grid, block, 0, st>>>(a, g_ichunk);
  }
}

cudaError_t awp_launch_stress(const StrArgs& a, bool elastic, cudaStream_t st) {
  const int nk = a.k1 - a.k0 + 1, nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nk <= 0 || nj <= 0 || ni <= 0) return cudaSuccess;
  const dim3 grid(cdiv_u(nk, 32), cdiv_u(nj, 8), cdiv_u(ni, g_ichunk));
  launch_stress_ty<8>(a, elastic, a.vx1 != nullptr, grid, st);
  return cudaGetLastError();
}

int awp_tuning_set(const char* key, int value) {
  if (!strcmp(key, "ichunk") && value >= 4 && value <= 1024) { g_ichunk = value; return 0; }
  if (!strcmp(key, "spin_limit")) return awp_tma_set_spin_limit(value);
  if (!strcmp(key, "l2_promotion")) return awp_tma_set_l2_promotion(value);
  if (value == 0 || value == 1) {
    if (!strcmp(key, "tma")) { g_tma_vel = g_tma_str = value; return 0; }  // both half-steps
    if (!strcmp(key, "tma_vel")) { g_tma_vel = value; return 0; }
    if (!strcmp(key, "tma_str")) { g_tma_str = value; return 0; }
  }
  return 1;
}

int awp_tuning_get(const char* key) {
  if (!strcmp(key, "ichunk")) return g_ichunk;
  if (!strcmp(key, "tma")) return g_tma_vel == g_tma_str ? g_tma_str : -1;
  if (!strcmp(key, "tma_vel")) return g_tma_vel;
  if (!strcmp(key, "tma_str")) return g_tma_str;
  if (!strcmp(key, "spin_limit")) return (int)awp_tma_get_spin_limit();
  if (!strcmp(key, "l2_promotion")) return awp_tma_get_l2_promotion();
  return -1;
}

cudaError_t awp_launch_fstr(const FstrArgs& a, cudaStream_t st) {
  const int nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nj <= 0 || ni <= 0) return cudaSuccess;
  k_fstr<<<dim3(cdiv_u(nj, 128), ni, 1), 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_addsrc(const SrcArgs& a, cudaStream_t st) {
  if (a.ncell <= 0) return cudaSuccess;
  if (a.cell_pos)
    k_addsrc<<<cdiv_u(a.ncell, 128), 128, 0, st>>>(a);
  else
    k_addsrc_direct<<<cdiv_u(a.ncell, 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

__global__ void k_frcvel(const FrcvelArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.npsrc) return;
  const int i = a.i - 1;
  const float ts = (float)a.tskp;
  int i0 = (int)((float)a.tskp * floorf((float)((double)i + 1.0) / ts));
  int i1 = (int)((float)a.tskp * ceilf((float)((double)i + 1.0) / ts));
  const float pfact = (float)(i + 1 - i0) / ts;
  i0 /= a.tskp;
  i1 /= a.tskp;
  const int idx = a.psrc[j * a.dim] + 1 + AWP_NGSL;
  const int idy = a.psrc[j * a.dim + 1] + 1 + AWP_NGSL;
  const int idz = a.psrc[j * a.dim + 2] + AWP_ALIGN - 1;
  const long long pos = (long long)idx * a.slice + (long long)idy * a.yline + idz;
  const bool above = (a.xmin == -1) || (idx >= a.xmin);
  const bool below = (a.xmax == -1) || (idx <= a.xmax);
  if (!(above && below)) return;
  const int n = a.npsrc;
  if (i < a.read_step * a.tskp) {
    const float up = a.axx[i0 * n + j], vp = a.ayy[i0 * n + j], wp = a.azz[i0 * n + j];
    const float un = a.axx[i1 * n + j], vn = a.ayy[i1 * n + j], wn = a.azz[i1 * n + j];
    const float ui = __fmaf_rn(__fsub_rn(un, up), pfact, up);
    const float vi = __fmaf_rn(__fsub_rn(vn, vp), pfact, vp);
    const float wi = __fmaf_rn(__fsub_rn(wn, wp), pfact, wp);
    if (i == a.read_step * a.tskp - 1) {
      a.axx[j] = a.axx[i1 * n + j];
      a.ayy[j] = a.ayy[i1 * n + j];
      a.azz[j] = a.azz[i1 * n + j];
      a.axx[i1 * n + j] = (un - a.u1[pos]) / a.DT;
      a.ayy[i1 * n + j] = (vn - a.v1[pos]) / a.DT;
      a.azz[i1 * n + j] = (wn - a.w1[pos]) / a.DT;
    }
    a.u1[pos] = ui;
    a.v1[pos] = vi;
    a.w1[pos] = wi;
  } else {
    a.u1[pos] = __fmaf_rn(a.axx[a.read_step * n + j], a.DT, a.u1[pos]);
    a.v1[pos] = __fmaf_rn(a.ayy[a.read_step * n + j], a.DT, a.v1[pos]);
    a.w1[pos] = __fmaf_rn(a.azz[a.read_step * n + j], a.DT, a.w1[pos]);
  }
}

// Halo planes: whole planes of the padded layout, so every segment is a
// multiple of 4 floats on 16-byte boundaries; one block row per segment.
__global__ void k_copy_segments(const CopySegs s) {
  const int q = blockIdx.y;
  const float4* __restrict__ src = reinterpret_cast<const float4*>(s.src[q]);
  float4* __restrict__ dst = reinterpret_cast<float4*>(s.dst[q]);
  const long long n4 = s.n[q] >> 2;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n4;
       v += (long long)gridDim.x * blockDim.x)
    dst[v] = src[v];
}

cudaError_t awp_launch_copy_segments(const CopySegs& s, cudaStream_t st) {
  if (s.nseg <= 0) return cudaSuccess;
  if (s.nseg > 32) return cudaErrorInvalidValue;
  long long mx = 0;
  for (int q = 0; q < s.nseg; ++q) {
    if ((s.n[q] & 3) || (reinterpret_cast<uintptr_t>(s.src[q]) & 15) ||
        (reinterpret_cast<uintptr_t>(s.dst[q]) & 15))
      return cudaErrorInvalidValue;
    mx = s.n[q] > mx ? s.n[q] : mx;
  }
  const unsigned bx = (unsigned)std::min<long long>(cdiv_u(mx >> 2, 256), 148 * 4 / s.nseg + 1);
  k_copy_segments<<<dim3(bx, s.nseg), 256, 0, st>>>(s);
  return cudaGetLastError();
}

cudaError_t awp_launch_frcvel(const FrcvelArgs& a, cudaStream_t st) {
  if (a.npsrc <= 0) return cudaSuccess;
  k_frcvel<<<cdiv_u(a.npsrc, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_planesrc(const PlaneSrcArgs& a, cudaStream_t st) {
  if (a.nx <= 0 || a.ny <= 0) return cudaSuccess;
  k_addplanesrc<<<dim3(cdiv_u(a.nx, 16), cdiv_u(a.ny, 16)), dim3(16, 16), 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_addkinsrc(const KinSrcArgs& a, cudaStream_t st) {
  if (a.ncell <= 0) return cudaSuccess;
  k_addkinsrc<<<cdiv_u(a.ncell, 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_plast_calc(const PlastCalcArgs& a, cudaStream_t st) {
  const int nk = a.k1 - a.k0 + 1, nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nk <= 0 || nj <= 0 || ni <= 0) return cudaSuccess;
  k_plast_calc<<<dim3(cdiv_u(nk, 32), cdiv_u(nj, 4), ni), dim3(32, 4, 1), 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_plast_app(const PlastAppArgs& a, cudaStream_t st) {
  const int nk = a.k1 - a.k0 + 1, nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nk <= 0 || nj <= 0 || ni <= 0) return cudaSuccess;
  k_plast_app<<<dim3(cdiv_u(nk, 32), cdiv_u(nj, 4), ni), dim3(32, 4, 1), 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_velbuffer(const VelBufArgs& a, cudaStream_t st) {
  if (a.rec_nxt <= 0 || a.rec_nyt <= 0 || a.rec_nzt <= 0) return cudaSuccess;
  const dim3 block(32, 4, 1);
  const dim3 grid(cdiv_u(a.rec_nxt, 32), cdiv_u(a.rec_nyt, 4), a.rec_nzt);
  k_velbuffer<<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_media(const MediaArgs& a, cudaStream_t st) {
  k_media<<<148 * 8, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_media_borders(float* d1, float* mu, float* lam, float* qp, float* qs,
                                     const AwpGeom& g, int nve, cudaStream_t st) {
  const dim3 grid(cdiv_u(g.ny_pad(), 128), (unsigned)g.nx_pad(), 1);
  k_media_borders<<<grid, 128, 0, st>>>(d1, mu, lam, qp, qs, g, nve);
  return cudaGetLastError();
}

cudaError_t awp_launch_lam_mu(const float* lam, const float* mu, float* lam_mu,
                              const AwpGeom& g, int xls, int xre, int yls, int yre,
                              cudaStream_t st) {
  const dim3 grid(cdiv_u(yre - yls + 1, 128), xre - xls + 1, 1);
  k_lam_mu<<<grid, 128, 0, st>>>(lam, mu, lam_mu, g, xls, xre, yls, yre);
  return cudaGetLastError();
}

cudaError_t awp_launch_fill(float* p, float v, long long n, cudaStream_t st) {
  k_fill<<<148 * 8, 256, 0, st>>>(p, v, n);
  return cudaGetLastError();
}

cudaError_t awp_launch_anynonzero(const float* p, long long n, unsigned int* flag,
                                  cudaStream_t st) {
  k_anynonzero<<<148 * 8, 256, 0, st>>>(p, n, flag);
  return cudaGetLastError();
}

cudaError_t awp_launch_nonfinite(const float* p, long long n, unsigned int* flag,
                                 cudaStream_t st) {
  k_nonfinite<<<148 * 8, 256, 0, st>>>(p, n, flag);
  return cudaGetLastError();
}

int awp_batch_blocks_per_sm(int ty, int* vel, int* str) {
  cudaError_t e;
  if (ty == 8) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(vel, k_batch_velocity<8>, 256, 0);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(str, k_batch_stress<false, 8>, 256, 0);
  } else if (ty == 4) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(vel, k_batch_velocity<4>, 128, 0);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(str, k_batch_stress<false, 4>, 128, 0);
  } else {
    return 1;
  }
  return e == cudaSuccess ? 0 : 2;
}

template <int TY>
static void launch_batch_halfsteps(const BatchLaunch& b, cudaStream_t st) {
  const dim3 block(32, TY);
  k_batch_velocity<TY><<<b.grid_vel, block, 0, st>>>(b.inst, b.vtiles, b.nvtiles, b.counters,
                                                     b.ichunk);
  if (b.nstiles > 0)
    k_batch_stress<false, TY><<<b.grid_str, block, 0, st>>>(b.inst, b.stiles, b.nstiles,
                                                            b.counters + 1, b.ichunk);
  if (b.nstiles_el > 0)
    k_batch_stress<true, TY><<<b.grid_str, block, 0, st>>>(b.inst, b.stiles_el, b.nstiles_el,
                                                           b.counters + 2, b.ichunk);
}

cudaError_t awp_launch_batch_step(const BatchLaunch& b, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(b.counters, 0, 3 * sizeof(int), st);
  if (e != cudaSuccess) return e;
  if (b.ty == 8)
    launch_batch_halfsteps<8>(b, st);
  else
    launch_batch_halfsteps<4>(b, st);
  if (b.nsrc > 0)
    k_batch_sources<<<cdiv_u(b.nsrc, 128), 128, 0, st>>>(b.inst, b.src_cells, b.nsrc, b.step);
  k_batch_fstr<<<b.nrows > 0 ? b.nrows : 1, 128, 0, st>>>(b.inst, b.rows, b.nrows, b.step);
  return cudaGetLastError();
}

cudaError_t awp_launch_sources_dev(const SrcArgs* a, const KinSrcArgs* k, const int* step,
                                   int nst, cudaStream_t st) {
  if (a && a->ncell > 0)
    k_addsrc_dev<<<cdiv_u(a->ncell, 128), 128, 0, st>>>(*a, step, nst);
  if (k && k->ncell > 0) k_addkinsrc_dev<<<cdiv_u(k->ncell, 128), 128, 0, st>>>(*k, step);
  return cudaGetLastError();
}

cudaError_t awp_launch_step_advance(int* step, cudaStream_t st) {
  k_step_advance<<<1, 1, 0, st>>>(step);
  return cudaGetLastError();
}
