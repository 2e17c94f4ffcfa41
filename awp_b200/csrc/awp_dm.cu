// Discontinuous-mesh coupling kernels (reference: src/awp/kernel.cu:2289-3234,
// src/awp/mesh.c:1404-1443).  All are 2-D over an interface (a few planes of
// work per step), so they run one thread per horizontal point; the
// arithmetic follows the reference expression by expression with explicit
// rounding intrinsics.
//
// At one rank the reference's swap-area exchanges (swap.c:549-583,
// kernel.cu:3320-3676) return at once and bgcaccess (kernel.cu:2809-2852)
// only ever reads the grid itself: every index swap3 forms lies inside the
// padded fine grid, so the window average reads the fine grid directly.
#include <cuda_runtime.h>

#include "awp_dm.cuh"
#include "awp_stencil.cuh"

namespace {

__device__ __forceinline__ long long at(const DmGrid& g, int i, int j, int k) {
  return (long long)i * g.slice + (long long)j * g.yline + k;
}

// ===========================================================================
// dvelc2 (kernel.cu:2289-2343)
// ===========================================================================
__global__ void k_dvelc2(const DmVel2Args a) {
  const int j = 2 + AWP_NGSL + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = 2 + AWP_NGSL + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.g.nxt + 2 + AWP_NGSL || j >= a.g.nyt + 2 + AWP_NGSL) return;
  const int S = a.g.slice, Y = a.g.yline;
  const int k = 2 + AWP_ALIGN;
  const long long pos = at(a.g, i, j, k);
  const float* d = a.d1;
  const float dcrj = __fmul_rn(__fmul_rn(a.dcrjz[k], a.dcrjx[i]), a.dcrjy[j]);
  // w along the first line
  {
    const float fd3 = a.dth / __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(d[pos], d[pos + S]),
                                                                   d[pos - Y]),
                                                         d[pos + S - Y]));
    const float s = __fadd_rn(__fadd_rn(__fsub_rn(a.g.xz[pos + S], a.g.xz[pos]),
                                        __fsub_rn(a.g.yz[pos], a.g.yz[pos - Y])),
                              __fsub_rn(a.g.zz[pos + 1], a.g.zz[pos]));
    a.g.w1[pos] = __fmul_rn(__fmaf_rn(fd3, s, a.g.w1[pos]), dcrj);
  }
  // u, v along the second line (same k in the reference)
  {
    const float fd1 = a.dth / __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(d[pos], d[pos - Y]),
                                                                   d[pos - 1]),
                                                         d[pos - Y - 1]));
    const float fd2 = a.dth / __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(d[pos], d[pos + S]),
                                                                   d[pos - 1]),
                                                         d[pos + S - 1]));
    const float su = __fadd_rn(__fadd_rn(__fsub_rn(a.g.xx[pos], a.g.xx[pos - S]),
                                         __fsub_rn(a.g.xy[pos], a.g.xy[pos - Y])),
                               __fsub_rn(a.g.xz[pos], a.g.xz[pos - 1]));
    const float sv = __fadd_rn(__fadd_rn(__fsub_rn(a.g.xy[pos + S], a.g.xy[pos]),
                                         __fsub_rn(a.g.yy[pos + Y], a.g.yy[pos])),
                               __fsub_rn(a.g.yz[pos], a.g.yz[pos - 1]));
    a.g.u1[pos] = __fmul_rn(__fmaf_rn(fd1, su, a.g.u1[pos]), dcrj);
    a.g.v1[pos] = __fmul_rn(__fmaf_rn(fd2, sv, a.g.v1[pos]), dcrj);
  }
}

// ===========================================================================
// dstrqc2 (kernel.cu:2564-2767), anelastic form (ELA2 undefined)
// ===========================================================================
// Q(f) weight of dstrqc2: double switch 1/(2q) <= 200, low-Q polynomial in
// double, otherwise wwo*q (dstrqc uses 2*wwo*q there), then / wwo.
__device__ __forceinline__ float qf2(float q, float wwo, float c0, float c1) {
  float w;
  if (1. / ((double)q * 2.0) <= 200.0) {
    const double x = 2. * (double)q;
    w = (float)__fma_rn(__dmul_rn((double)c0, x), x, __dmul_rn((double)c1, x));
  } else {
    w = __fmul_rn(wwo, q);
  }
  return w / wwo;
}

__global__ void k_dstrqc2(const DmStr2Args a) {
  const int j = a.j0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = a.i0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > a.i1 || j > a.j1) return;
  const int S = a.g.slice, Y = a.g.yline;
  const int k = AWP_ALIGN + 2;
  const long long pos = at(a.g, i, j, k);
  const float dcrj = __fmul_rn(__fmul_rn(a.dcrjz[k], a.dcrjx[i]), a.dcrjy[j]);
  float f_vx1, f_vx2, f_wwo;
  int cidx;
  if (a.vx1) {
    f_vx1 = a.vx1[pos];
    f_vx2 = a.vx2[pos];
    f_wwo = a.wwo[pos];
    cidx = 2 * a.ww[pos] - 2;
  } else {
    const int t = awp_tex_index(a.tex, i, j, k);
    f_vx1 = a.tex.tau1[t];
    f_vx2 = a.tex.tau2[t];
    f_wwo = a.tex.wwo8[t];
    cidx = 2 * t;
  }
  const float c0 = a.coeff_dev ? a.coeff_dev[cidx] : a.coeff[cidx];
  const float c1 = a.coeff_dev ? a.coeff_dev[cidx + 1] : a.coeff[cidx + 1];
  // eight-cell sums in the reference's order: pos, ip1, jm1, ijk, km1, ik1, jk1, ijk1
  auto sum8 = [&](const float* f) {
    float s = __fadd_rn(f[pos], f[pos + S]);
    s = __fadd_rn(s, f[pos - Y]);
    s = __fadd_rn(s, f[pos + S - Y]);
    s = __fadd_rn(s, f[pos - 1]);
    s = __fadd_rn(s, f[pos + S - 1]);
    s = __fadd_rn(s, f[pos - Y - 1]);
    return __fadd_rn(s, f[pos + S - Y - 1]);
  };
  const float* mu = a.mu;
  float xl = __fdiv_rn(8.0f, sum8(a.lam));   // = (float)(8.0/(double)x), see k_stress
  float xm = __fdiv_rn(16.0f, sum8(mu));
  float xmu1 = __fdiv_rn(2.0f, __fadd_rn(mu[pos], mu[pos - 1]));
  float xmu2 = __fdiv_rn(2.0f, __fadd_rn(mu[pos], mu[pos - Y]));
  float xmu3 = __fdiv_rn(2.0f, __fadd_rn(mu[pos], mu[pos + S]));
  xl = __fadd_rn(xl, xm);
  // qpa: float switch 1.0f/(2q) <= 200.0f
  float qpa = __fmul_rn(0.0625f, sum8(a.qp));
  float qpaw;
  if (1.0f / (qpa * 2.0f) <= 200.0f) {
    const double x = 2. * (double)qpa;
    qpaw = (float)__fma_rn(__dmul_rn((double)c0, x), x, __dmul_rn((double)c1, x));
  } else {
    qpaw = __fmul_rn(f_wwo, qpa);
  }
  qpaw = qpaw / f_wwo;
  const float* qs = a.qs;
  const float hw = qf2(__fmul_rn(0.0625f, sum8(qs)), f_wwo, c0, c1);
  const float h1w = qf2(__fmul_rn(0.25f, __fadd_rn(qs[pos], qs[pos - 1])), f_wwo, c0, c1);
  const float h2w = qf2(__fmul_rn(0.25f, __fadd_rn(qs[pos], qs[pos - Y])), f_wwo, c0, c1);
  const float h3w = qf2(__fmul_rn(0.25f, __fadd_rn(qs[pos], qs[pos + S])), f_wwo, c0, c1);
  AwpStrCoef cf;
  float h = __fmul_rn(__fmul_rn(-xm, hw), a.dh1);
  float h1 = __fmul_rn(__fmul_rn(-xmu1, h1w), a.dh1);
  float h2 = __fmul_rn(__fmul_rn(-xmu2, h2w), a.dh1);
  float h3 = __fmul_rn(__fmul_rn(-xmu3, h3w), a.dh1);
  qpa = __fmul_rn(__fmul_rn(-qpaw, xl), a.dh1);
  xm = __fmul_rn(xm, a.dth);
  xmu1 = __fmul_rn(xmu1, a.dth);
  xmu2 = __fmul_rn(xmu2, a.dth);
  xmu3 = __fmul_rn(xmu3, a.dth);
  xl = __fmul_rn(xl, a.dth);
  h = __fmul_rn(h, f_vx1);
  h1 = __fmul_rn(h1, f_vx1);
  h2 = __fmul_rn(h2, f_vx1);
  h3 = __fmul_rn(h3, f_vx1);
  qpa = __fmul_rn(qpa, f_vx1);
  const float DT = a.dt;
  cf.xl = xl;
  cf.xm = __fmaf_rn(DT, h, xm);
  cf.xmu1 = __fmaf_rn(DT, h1, xmu1);
  cf.xmu2 = __fmaf_rn(DT, h2, xmu2);
  cf.xmu3 = __fmaf_rn(DT, h3, xmu3);
  cf.h = h; cf.h1 = h1; cf.h2 = h2; cf.h3 = h3; cf.qpa = qpa;
  cf.vx1 = __fmul_rn(DT, __fmaf_rn(f_vx2, f_vx1, 1.0f));

  const DmGrid& g = a.g;
  float d[9];
  d[0] = __fsub_rn(g.u1[pos + S], g.u1[pos]);  // normal: x, y, z
  d[1] = __fsub_rn(g.v1[pos], g.v1[pos - Y]);
  d[2] = __fsub_rn(g.w1[pos], g.w1[pos - 1]);
  d[3] = __fsub_rn(g.u1[pos + Y], g.u1[pos]);  // xy pair
  d[4] = __fsub_rn(g.v1[pos], g.v1[pos - S]);
  d[5] = __fsub_rn(g.u1[pos + 1], g.u1[pos]);  // xz pair
  d[6] = __fsub_rn(g.w1[pos], g.w1[pos - S]);
  d[7] = __fsub_rn(g.v1[pos + 1], g.v1[pos]);  // yz pair
  d[8] = __fsub_rn(g.w1[pos + Y], g.w1[pos]);
  float sg[6] = {g.xx[pos], g.yy[pos], g.zz[pos], g.xy[pos], g.xz[pos], g.yz[pos]};
  float rr[6] = {a.r1[pos], a.r2[pos], a.r3[pos], a.r4[pos], a.r5[pos], a.r6[pos]};
  awp_stress_update<false>(sg, rr, cf, f_vx1, f_vx2, f_wwo, DT, dcrj, d);
  g.xx[pos] = sg[0]; g.yy[pos] = sg[1]; g.zz[pos] = sg[2];
  g.xy[pos] = sg[3]; g.xz[pos] = sg[4]; g.yz[pos] = sg[5];
  a.r1[pos] = rr[0]; a.r2[pos] = rr[1]; a.r3[pos] = rr[2];
  a.r4[pos] = rr[3]; a.r5[pos] = rr[4]; a.r6[pos] = rr[5];
}

// ===========================================================================
// intp3d (kernel.cu:2359-2561): bilinear weights (1, 2/3, 1/3, 0) spread each
// coarse cell's four corners over a 4 x 4 fine patch at kh = align+1.
// Neighbouring patches share an edge where the weight is 0 on one side, and
// both threads store the same value there, as in the reference.
// ===========================================================================
__global__ void k_intp3d(const DmPairArgs a) {
  const int j = AWP_NGSL + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = AWP_NGSL + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > a.lo.nxt + 3 + AWP_NGSL || j > a.lo.nyt + 3 + AWP_NGSL) return;
  const float w[4] = {1.0f, (float)(2. / 3.), (float)(1. / 3.), 0.0f};
  const DmGrid &lo = a.lo, &hi = a.hi;
  const long long pl = at(lo, i, j, lo.nzt + AWP_ALIGN - 3);
  const long long pip = pl + lo.slice, pjp = pl + lo.yline, pij = pl + lo.slice + lo.yline;
  const int ih = (i - 2 - AWP_NGSL) * 3 + 2 + AWP_NGSL;
  const int jh = (j - 2 - AWP_NGSL) * 3 + 2 + AWP_NGSL;
  const long long ph = at(hi, ih, jh, AWP_ALIGN + 1);
  // field, its fine patch offset in i and j
  auto patch = [&](const float* L, float* H, int oi, int oj) {
    const float v0 = L[pl], v1 = L[pip], v2 = L[pjp], v3 = L[pij];
    for (int jj = 1; jj <= 4; ++jj)
      for (int ii = 1; ii <= 4; ++ii) {
        const float wa = w[ii - 1], wb = w[jj - 1], wc = w[4 - ii], wd = w[4 - jj];
        float s = __fmul_rn(__fmul_rn(v0, wa), wb);
        s = __fmaf_rn(__fmul_rn(v1, wc), wb, s);
        s = __fmaf_rn(__fmul_rn(v2, wa), wd, s);
        s = __fmaf_rn(__fmul_rn(v3, wc), wd, s);
        H[ph + (long long)(ii - 1 + oi) * hi.slice + (long long)(jj - 1 + oj) * hi.yline] = s;
      }
  };
  // one field per blockIdx.z (the nine patches of a column are independent)
  switch (blockIdx.z) {
    case 0: patch(lo.xz, hi.xz, 0, 0); break;
    case 1: patch(lo.yz, hi.yz, 1, 1); break;
    case 2: patch(lo.w1, hi.w1, 1, 0); break;
    case 3: patch(lo.xx, hi.xx, 1, 0); break;
    case 4: patch(lo.yy, hi.yy, 1, 0); break;
    case 5: patch(lo.zz, hi.zz, 1, 0); break;
    case 6: patch(lo.u1, hi.u1, 0, 0); break;
    case 7: patch(lo.v1, hi.v1, 1, 1); break;
    default: patch(lo.xy, hi.xy, 0, 1); break;
  }
}

// ===========================================================================
// swap3 (kernel.cu:3032-3217): tent-weighted 5 x 5 x 5 window average of the
// fine grid (WWL = 2) into the coarse grid's top two layers.  Weights and
// products in double, each partial sum rounded to float like the reference's
// float accumulator.
// ===========================================================================
// A CTA takes 2 (i) x 32 (j) coarse columns of one field (blockIdx.z): it
// copies the fine-grid box the field's windows read
// (9 x 99 x 8 points: fine i2-2 .. i3+2 and j2-2 .. j3+2 of its columns,
// levels align+1 .. align+8) into shared memory with k-contiguous,
// sector-wide loads, then each of its threads forms one window of one column
// (a field has one or two: levels nzt-2 and nzt-1), its 125 terms in the
// reference's order from shared memory.  Read straight from global memory the
// windows' stride-3 j columns cost a sector per 4-byte load; the box copy
// reads each sector once.
constexpr int kSwTI = 2, kSwTJ = 32;
constexpr int kSwBI = 3 * (kSwTI - 1) + 6, kSwBJ = 3 * (kSwTJ - 1) + 6, kSwBK = 8;
constexpr int kSwKS = 9;  // padded k stride: lanes 3 j apart fall in distinct banks

// The 125 tent weights of a window in the sum's order (jj, ii, kk), formed on
// the host as the reference forms them on the device, in double:
// (1 / total) * (3 - |ii|) * (3 - |jj|) * (3 - |kk|) left to right.
struct SwapWeights {
  double w[125];
};

__global__ void __launch_bounds__(128) k_swap3(const DmPairArgs a, const SwapWeights sw) {
  __shared__ float box[kSwBI * kSwBJ * kSwKS];
  const DmGrid &lo = a.lo, &hi = a.hi;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int i0 = AWP_NGSL + blockIdx.y * kSwTI, j0 = AWP_NGSL + blockIdx.x * kSwTJ;
  const int imax = lo.nxt + AWP_NGSL + 4, jmax = lo.nyt + AWP_NGSL + 4;
  // fine box origin (i2 - 2, j2 - 2 of the first column) and the extent the
  // valid columns read
  const int fi0 = (i0 - 2 - AWP_NGSL) * 3 + AWP_NGSL, fj0 = (j0 - 2 - AWP_NGSL) * 3 + AWP_NGSL;
  const int nbi = 3 * (min(i0 + kSwTI - 1, imax) - i0) + 6;
  const int nbj = 3 * (min(j0 + kSwTJ - 1, jmax) - j0) + 6;
  // this thread's column and window slot (level 0 or 1)
  const int c = tid & 63, lev = tid >> 6;
  const int ci = c >> 5, cj = c & 31;
  const int i = i0 + ci, j = j0 + cj;
  const bool valid = i <= imax && j <= jmax;
  {
    const int f = blockIdx.z;  // one field per CTA
    float* dst;
    const float* src;
    int kh0, nwin, di, dj;  // level-0 window at kh0 (level 1 at 6); source i3 / j3 if di / dj
    switch (f) {
      case 0: dst = lo.u1; src = hi.u1; kh0 = 3; nwin = 2; di = 0; dj = 0; break;
      case 1: dst = lo.v1; src = hi.v1; kh0 = 3; nwin = 2; di = 1; dj = 1; break;
      case 2: dst = lo.xy; src = hi.xy; kh0 = 3; nwin = 2; di = 0; dj = 1; break;
      case 3: dst = lo.xx; src = hi.xx; kh0 = 3; nwin = 2; di = 1; dj = 0; break;
      case 4: dst = lo.yy; src = hi.yy; kh0 = 3; nwin = 2; di = 1; dj = 0; break;
      case 5: dst = lo.zz; src = hi.zz; kh0 = 3; nwin = 2; di = 1; dj = 0; break;
      case 6: dst = lo.xz; src = hi.xz; kh0 = 4; nwin = 1; di = 0; dj = 0; break;
      case 7: dst = lo.w1; src = hi.w1; kh0 = 4; nwin = 1; di = 1; dj = 0; break;
      default: dst = lo.yz; src = hi.yz; kh0 = 4; nwin = 1; di = 1; dj = 1; break;
    }
    for (int t = tid; t < nbi * nbj * kSwBK; t += 128) {
      const int bk = t % kSwBK, r = t / kSwBK, bj = r % nbj, bi = r / nbj;
      box[(bi * kSwBJ + bj) * kSwKS + bk] = src[at(hi, fi0 + bi, fj0 + bj, AWP_ALIGN + 1 + bk)];
    }
    __syncthreads();
    if (valid && lev < nwin) {
      const int kh = lev ? 6 : kh0;
      const int bi = 3 * ci + di + 2, bj = 3 * cj + dj + 2, bk = kh - 1;
      float sum = 0.0f;
      int q = 0;
      for (int jj = -AWP_WWL; jj <= AWP_WWL; ++jj)
        for (int ii = -AWP_WWL; ii <= AWP_WWL; ++ii)
#pragma unroll
          for (int kk = -AWP_WWL; kk <= AWP_WWL; ++kk, ++q) {
            const float h = box[((bi + ii) * kSwBJ + bj + jj) * kSwKS + bk + kk];
            sum = (float)__fma_rn(sw.w[q], (double)h, (double)sum);
          }
      dst[at(lo, i, j, AWP_ALIGN + lo.nzt - 2 + lev)] = sum;
    }
  }
}

// ===========================================================================
// checkmesh (mesh.c:1404-1443)
// ===========================================================================
__global__ void k_checkmesh(const DmCheckArgs a) {
  const int j = 2 + AWP_NGSL + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = 2 + AWP_NGSL + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.glo.nxt + 2 + AWP_NGSL || j >= a.glo.nyt + 2 + AWP_NGSL) return;
  const int ih = (i - 2 - AWP_NGSL) * 3 + 2 + AWP_NGSL;
  const int jh = (j - 2 - AWP_NGSL) * 3 + 3 + AWP_NGSL;
  for (int l = 0; l < 3; ++l) {
    const long long pl = at(a.glo, i, j, AWP_ALIGN + a.glo.nzt - 3 + l);
    const long long ph = at(a.ghi, ih, jh, AWP_ALIGN + 1 + 3 * l);
    for (int f = 0; f < a.nf; ++f)
      if (a.lo[f][pl] != a.hi[f][ph]) a.lo[f][pl] = a.hi[f][ph];
  }
}

inline unsigned cdiv(int a, int b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

cudaError_t awp_launch_dvelc2(const DmVel2Args& a, cudaStream_t st) {
  const dim3 block(32, 4);
  k_dvelc2<<<dim3(cdiv(a.g.nyt, 32), cdiv(a.g.nxt, 4)), block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_dstrqc2(const DmStr2Args& a, cudaStream_t st) {
  if (a.i1 < a.i0 || a.j1 < a.j0) return cudaSuccess;
  const dim3 block(32, 4);
  k_dstrqc2<<<dim3(cdiv(a.j1 - a.j0 + 1, 32), cdiv(a.i1 - a.i0 + 1, 4)), block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_intp3d(const DmPairArgs& a, cudaStream_t st) {
  const dim3 block(32, 4);
  k_intp3d<<<dim3(cdiv(a.lo.nyt + 4, 32), cdiv(a.lo.nxt + 4, 4), 9), block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_swap3(const DmPairArgs& a, cudaStream_t st) {
  double total = 0.;  // ttlwght2 = ttlwght3 = ttlwght4 for WWL = 2 (kernel.cu:3052-3061)
  for (int jj = -AWP_WWL; jj <= AWP_WWL; jj++)
    for (int ii = -AWP_WWL; ii <= AWP_WWL; ii++)
      for (int kk = -AWP_WWL; kk <= AWP_WWL; kk++)
        total += (1. + AWP_WWL - abs(jj)) * (1. + AWP_WWL - abs(ii)) * (1. + AWP_WWL - abs(kk));
  const double inv_total = 1. / total;
  SwapWeights sw;
  int q = 0;
  for (int jj = -AWP_WWL; jj <= AWP_WWL; jj++)
    for (int ii = -AWP_WWL; ii <= AWP_WWL; ii++)
      for (int kk = -AWP_WWL; kk <= AWP_WWL; kk++)
        sw.w[q++] = inv_total * (1. + AWP_WWL - abs(ii)) * (1. + AWP_WWL - abs(jj)) *
                    (1. + AWP_WWL - abs(kk));
  k_swap3<<<dim3(cdiv(a.lo.nyt + 5, kSwTJ), cdiv(a.lo.nxt + 5, kSwTI), 9), dim3(32, 4), 0, st>>>(
      a, sw);
  return cudaGetLastError();
}

cudaError_t awp_launch_checkmesh(const DmCheckArgs& a, cudaStream_t st) {
  const dim3 block(32, 4);
  k_checkmesh<<<dim3(cdiv(a.glo.nyt, 32), cdiv(a.glo.nxt, 4)), block, 0, st>>>(a);
  return cudaGetLastError();
}
