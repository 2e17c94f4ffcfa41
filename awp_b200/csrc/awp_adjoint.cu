// Discrete adjoint of the single-grid time step and the material gradient of
// a seismogram misfit.
//
// The forward step (one_step: dvelcx, dstrqc with its free-surface velocity
// images, point sources, fstr) is linear in the wavefield state for fixed
// materials, so its adjoint is the transpose of each map in reverse order:
//
//   fstr^T -> stress^T (memory variables, strain rates, then the images) ->
//   velocity^T
//
// (the fstr transpose is folded into the stress kernel's top three cells; the
// imaged values above the surface are cleared with the velocity images).  The
// free-surface imaging of the rows beyond the stress range (the extra row of
// an odd ny) acts on values that stay zero, so it has no transpose to apply.
//
// The density term needs the stress divergence the velocity update applied;
// it is recovered from the velocities before and after the step
// (fd * D(sigma) = u'/dc - u), so the segment store holds velocities only.
// Every transpose is written in gather form (each thread owns one output
// cell and reads the neighbours whose forward stencils touched it), so no
// atomics are needed and the result is deterministic.  The gradient terms use
// the forward state of the same step (stresses before it for the density
// term, velocities after it for the moduli terms).  Derivation, per map:
//
//   velocity  u' = (u + fd(rho) * D(sigma)) * dc          (dvelcx, kernel.cu:222-253)
//   stress    s' = K (s + P(e) + a r + DT (Q(e)(w-1) + g r)),  r' = b r + w Q(e)
//             (yy, zz carry K twice; dstrqc, kernel.cu:1114-1179)
//   images    u(top+1) = u - (w - w_{i-1}), v(top+1) = v - (w_{j+1} - w),
//             w(top+1) = w(top-1) - lam_mu * Z(u, v, w)     (kernel.cu:1087-1112)
//   fstr      zz(top+1) = -zz(top), ..., xz(top) = yz(top) = 0  (kernel.cu:1616-1647)
#include "awp_adjoint.cuh"

#include "awp_stencil.cuh"

namespace {

enum { LU, LV, LW, LXX, LYY, LZZ, LXY, LXZ, LYZ, LR1, LR2, LR3, LR4, LR5, LR6 };
enum { E1, E2, E3, E4, E5, E6, GL8, GM8, GP1, GP2, GP3, GQP8, GQS8, GQ1, GQ2, GQ3 };

// d(weight)/dq of the Q(f) weight awp_qf_weight(q, ...): the polynomial
// c0 (2q)^2 + c1 (2q) over wwo on the low-Q branch, 2 q otherwise (the branch
// held fixed, as the forward takes it at q)
__device__ __forceinline__ float qf_dweight(float q, float wwo, float c0, float c1,
                                            float qthr) {
  const float x = 2.0f * q;
  const bool low = (x >= qthr) || (x < 0.f) || (x == 0.f && signbit(x));
  return low ? (8.0f * c0 * q + 2.0f * c1) / wwo : 2.0f;
}
enum { VA, VB, VC, VEA, VEB, VEC };

// Per-thread asynchronous 4-byte copy global -> shared (cp.async); a thread
// reads back only its own slots, after cp.async.wait_all.
__device__ __forceinline__ void cpa4(float* s, const float* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(s)),
               "l"(g)
               : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

#ifndef AWP_ADJ_STAGE
#define AWP_ADJ_STAGE 1  // stage the stress transpose's once-read values
#endif
#ifndef AWP_ADJ_MINB
#define AWP_ADJ_MINB 7  // CTAs per SM the stress transpose's registers allow
#endif

// ---------------------------------------------------------------------------
// stress^T, pointwise part: memory variables and stresses in place, adjoint
// strain rates of the cell into E[], its material weights added to the sums
// in E[].  Seven 128-thread CTAs per SM (72 registers) run it faster than
// four without spills: the kernel waits on HBM latency.  The values it reads
// once and late (the cell's adjoint stresses, memory variables and weight
// sums) are copied to shared memory by cp.async when a thread starts, which
// takes them out of the registers (840 against 860 ms for a 600-step
// gradient at 256 x 256 x 128).
// ---------------------------------------------------------------------------
// WANTQ: also accumulate the Q^-1 weights (anelastic runs that ask for the
// Q^-1 gradients); without it the five Q sums are neither read nor written.
template <bool ELASTIC, bool WANTQ>
__global__ void __launch_bounds__(128, AWP_ADJ_MINB) k_adj_stress_cell(const AdjArgs a) {
  // the cell's own adjoint stresses and memory variables and its weight sums,
  // read once and late: copied to shared memory when the thread starts
  // (slots 0-5 stresses, 6-11 memory variables, 12-16 moduli sums, 17-21 Q sums)
  __shared__ float stg[AWP_ADJ_STAGE ? 22 : 1][128];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  // the relaxation tables in shared memory: the lanes of a warp alternate the
  // table entry with the parity of k, which a constant-bank read would serve
  // in two passes
  __shared__ float tab[40];  // tau1[8], tau2[8], wwo8[8], coeff[16]
  {
    if (tid < 8) {
      tab[tid] = a.tex.tau1[tid];
      tab[8 + tid] = a.tex.tau2[tid];
      tab[16 + tid] = a.tex.wwo8[tid];
    }
    if (!ELASTIC && tid < 16) tab[24 + tid] = a.coeff[tid];
    __syncthreads();
  }
  const int k = a.sk0 + blockIdx.x * 32 + threadIdx.x;
  const int j = a.sj0 + blockIdx.y * 4 + threadIdx.y;
  const int i = a.si0 + blockIdx.z;
  if (k > a.sk1 || j > a.sj1 || i > a.si1) return;
  // stencil neighbours as 32-bit offsets from per-array pointers at the cell
  const int S = a.g.slice, Y = a.g.yline;
  const long long p = (long long)i * S + (long long)j * Y + k;
  const float c1 = a.c1, c2 = a.c2, DT = a.dt;
  if (AWP_ADJ_STAGE) {
#pragma unroll
    for (int q = 0; q < 6; ++q) cpa4(&stg[q][tid], a.L[LXX + q] + p);
    if (!ELASTIC) {
#pragma unroll
      for (int q = 0; q < 6; ++q) cpa4(&stg[6 + q][tid], a.L[LR1 + q] + p);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) cpa4(&stg[12 + q][tid], a.E[GL8 + q] + p);
    if (!ELASTIC && WANTQ) {
#pragma unroll
      for (int q = 0; q < 5; ++q) cpa4(&stg[17 + q][tid], a.E[GQP8 + q] + p);
    }
  }
  // the cell's value of a staged array
  auto own = [&](int slot, const float* f) { return AWP_ADJ_STAGE ? stg[slot][tid] : f[p]; };

  // forward strain rates from the velocities after the step (VelBox layout)
  const int VS = (int)a.vb.S, VY = (int)a.vb.Y;
  const long long pv = (long long)i * a.vb.S + (long long)j * a.vb.Y + k - a.vb.off;
  const float* u = a.fu + pv;
  const float* v = a.fv + pv;
  const float* w = a.fw + pv;
  const float vs1 = c1 * (u[VS] - u[0]) + c2 * (u[2 * VS] - u[-VS]);
  const float vs2 = c1 * (v[0] - v[-VY]) + c2 * (v[VY] - v[-(2 * VY)]);
  const float vs3 = c1 * (w[0] - w[-1]) + c2 * (w[1] - w[-2]);
  const float e4 = c1 * (u[VY] - u[0]) + c2 * (u[2 * VY] - u[-VY]) +
                   c1 * (v[0] - v[-VS]) + c2 * (v[VS] - v[-(2 * VS)]);
  const float e5 = c1 * (u[1] - u[0]) + c2 * (u[2] - u[-1]) +
                   c1 * (w[0] - w[-VS]) + c2 * (w[VS] - w[-(2 * VS)]);
  const float e6 = c1 * (v[1] - v[0]) + c2 * (v[2] - v[-1]) +
                   c1 * (w[VY] - w[0]) + c2 * (w[2 * VY] - w[-VY]);

  // materials of the cell (kernel.cu:962-1070)
  auto sum8 = [&](const float* m0) {
    const float* m = m0 + p;
    return m[0] + m[S] + m[-Y] + m[S - Y] + m[-1] + m[S - 1] + m[-Y - 1] + m[S - Y - 1];
  };
  const float* mu = a.mu + p;
  const float L8 = sum8(a.lam), M8 = sum8(a.mu);
  const float P1 = mu[0] + mu[-1], P2 = mu[0] + mu[-Y], P3 = mu[0] + mu[S];
  const float xm_raw = 16.0f / M8;
  const float xl_raw = 8.0f / L8 + xm_raw;
  const float m1_raw = 2.0f / P1, m2_raw = 2.0f / P2, m3_raw = 2.0f / P3;
  const int t = awp_tex_index(a.tex, i, j, k);
  const float fvx1 = tab[t], fvx2 = tab[8 + t], wwo = tab[16 + t];
  float c_xm = a.dth, c_h = 0.f, c_q = 0.f, c_m[3] = {a.dth, a.dth, a.dth}, c_hh[3] = {0, 0, 0};
  // derivatives of the Q weights with respect to their averaged arguments
  float dqpaw = 0.f, dhw = 0.f, dhiw[3] = {0.f, 0.f, 0.f};
  if (!ELASTIC) {
    const float cc0 = tab[24 + 2 * t], cc1 = tab[25 + 2 * t];
    const float qs8 = 0.0625f * sum8(a.qs), qp8 = 0.0625f * sum8(a.qp);
    const float hw = awp_qf_weight(qs8, wwo, cc0, cc1, a.qthr);
    const float qpaw = awp_qf_weight(qp8, wwo, cc0, cc1, a.qthr);
    const float* qs = a.qs + p;
    const float qsp[3] = {0.25f * (qs[0] + qs[-1]), 0.25f * (qs[0] + qs[-Y]),
                          0.25f * (qs[0] + qs[S])};
    const float hiw[3] = {awp_qf_weight(qsp[0], wwo, cc0, cc1, a.qthr),
                          awp_qf_weight(qsp[1], wwo, cc0, cc1, a.qthr),
                          awp_qf_weight(qsp[2], wwo, cc0, cc1, a.qthr)};
    dhw = qf_dweight(qs8, wwo, cc0, cc1, a.qthr);
    dqpaw = qf_dweight(qp8, wwo, cc0, cc1, a.qthr);
    for (int q = 0; q < 3; ++q) dhiw[q] = qf_dweight(qsp[q], wwo, cc0, cc1, a.qthr);
    c_h = -hw * a.dh1 * fvx1;
    c_xm = a.dth + DT * c_h;
    c_q = -qpaw * a.dh1 * fvx1;
    for (int q = 0; q < 3; ++q) {
      c_hh[q] = -hiw[q] * a.dh1 * fvx1;
      c_m[q] = a.dth + DT * c_hh[q];
    }
  }
  const float xm = xm_raw * c_xm, h = xm_raw * c_h, xl = xl_raw * a.dth, qpa = xl_raw * c_q;
  const float xmu[3] = {m1_raw * c_m[0], m2_raw * c_m[1], m3_raw * c_m[2]};
  const float hh[3] = {m1_raw * c_hh[0], m2_raw * c_hh[1], m3_raw * c_hh[2]};
  const float K = a.dcrjx[i] * a.dcrjy[j] * a.dcrjz[k];
  const float al = DT * (1.0f + fvx2 * fvx1);   // coefficient of r in sigma
  const float be = fvx2, ga = fvx2 * (1.0f - fvx1);

  // fstr^T of this column's top three cells (the imaged values above the
  // surface are cleared later, in k_adj_vel_cell): zz(t) += -zz(t+1),
  // zz(t-1) += -zz(t+2), xz/yz(t-1) += -xz/yz(t+1), xz/yz(t-2) += -xz/yz(t+2),
  // xz/yz(t) after the imaging is zero
  const int top = a.g.top();
  auto fs = [&](int f) -> float {  // adjoint of the field after the stress update
    const float* Lf = a.L[f];
    float v = own(f - LXX, Lf);
    if (k == top) {
      if (f == LZZ) v -= Lf[p + 1];
      if (f == LXZ || f == LYZ) v = 0.f;
    } else if (k == top - 1) {
      if (f == LZZ) v -= Lf[p + 3];
      if (f == LXZ || f == LYZ) v -= Lf[p + 2];
    } else if (k == top - 2) {
      if (f == LXZ || f == LYZ) v -= Lf[p + 4];
    }
    return v;
  };
  // every load of the adjoint state before the first store: the stores below
  // go to other arrays (or other cells of the same array), and issuing the
  // loads together keeps them from waiting on one another
  if (AWP_ADJ_STAGE) cpa_wait();
  const float lx = own(0, a.L[LXX]), ly = own(1, a.L[LYY]), lz = fs(LZZ);
  const float ls[3] = {fs(LXY), fs(LXZ), fs(LYZ)};
  float rv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (!ELASTIC)
    for (int q = 0; q < 6; ++q) rv[q] = own(6 + q, a.L[LR1 + q]);
  // material weights, summed over the time steps (their spatial transposes
  // are linear and time-invariant, so k_adj_material applies them once)
  float wacc[5], qacc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int q = 0; q < 5; ++q) wacc[q] = own(12 + q, a.E[GL8 + q]);
  if (!ELASTIC && WANTQ)
    for (int q = 0; q < 5; ++q) qacc[q] = own(17 + q, a.E[GQP8 + q]);
  // normal components
  float PX, PY, PZ, QX = 0.f, QY = 0.f, QZ = 0.f;
  PX = K * lx;
  PY = K * K * ly;
  PZ = K * K * lz;
  if (!ELASTIC) {
    QX = DT * (wwo - 1.0f) * K * lx + wwo * rv[0];
    QY = DT * (wwo - 1.0f) * K * ly + wwo * rv[1];
    QZ = DT * (wwo - 1.0f) * K * lz + wwo * rv[2];
  }
  const float sP = PX + PY + PZ, sQ = QX + QY + QZ;
  const float A = xl + DT * qpa;
  const float s123 = vs1 + vs2 + vs3;
  const float G_xl = s123 * sP;
  const float G_qpa = DT * s123 * sP + s123 * sQ;
  const float G_xm = -((vs2 + vs3) * PX + (vs1 + vs3) * PY + (vs1 + vs2) * PZ);
  const float G_h = -((vs2 + vs3) * QX + (vs1 + vs3) * QY + (vs1 + vs2) * QZ);

  // shear components
  const float es[3] = {e4, e5, e6};
  const float mraw[3] = {m1_raw, m2_raw, m3_raw};
  float GP[3], ES[3], GQP[3];
  for (int q = 0; q < 3; ++q) {
    const float l = ls[q], lrv = rv[3 + q];
    ES[q] = (xmu[q] + DT * hh[q] * (wwo - 1.0f)) * K * l + wwo * hh[q] * lrv;
    const float G_xmu = es[q] * K * l;
    const float G_hq = es[q] * (DT * (wwo - 1.0f) * K * l + wwo * lrv);
    const float Pq = q == 0 ? P1 : (q == 1 ? P2 : P3);
    GP[q] = -2.0f / (Pq * Pq) * (G_xmu * c_m[q] + G_hq * c_hh[q]);
    // Qs^-1 pair: hh = m_raw c_hh, xmu = m_raw (dth + DT c_hh), c_hh = -hiw dh1 vx1
    GQP[q] = (G_hq + DT * G_xmu) * mraw[q] * (-a.dh1 * fvx1) * dhiw[q] * 0.25f;
  }

  // stores: the adjoint state in place, then the temporaries
  a.L[LXX][p] = K * lx;
  a.L[LYY][p] = K * K * ly;
  a.L[LZZ][p] = K * K * lz;
  a.L[LXY][p] = K * ls[0];
  a.L[LXZ][p] = K * ls[1];
  a.L[LYZ][p] = K * ls[2];
  if (!ELASTIC) {
    a.L[LR1][p] = (al + DT * ga) * K * lx + be * rv[0];
    a.L[LR2][p] = al * K * K * ly + DT * ga * K * ly + be * rv[1];
    a.L[LR3][p] = al * K * K * lz + DT * ga * K * lz + be * rv[2];
    for (int q = 0; q < 3; ++q) a.L[LR4 + q][p] = (al + DT * ga) * K * ls[q] + be * rv[3 + q];
  }
  float* const* E = a.E;
  E[E1][p] = A * sP - xm * (PY + PZ) + qpa * sQ - h * (QY + QZ);
  E[E2][p] = A * sP - xm * (PX + PZ) + qpa * sQ - h * (QX + QZ);
  E[E3][p] = A * sP - xm * (PX + PY) + qpa * sQ - h * (QX + QY);
  for (int q = 0; q < 3; ++q) E[E4 + q][p] = ES[q];
  // chain to the eight-cell sums
  const float G_xlraw = G_xl * a.dth + G_qpa * c_q;
  const float G_xmraw = G_xm * c_xm + G_h * c_h + G_xlraw;
  E[GL8][p] = wacc[0] + -8.0f / (L8 * L8) * G_xlraw;
  E[GM8][p] = wacc[1] + -16.0f / (M8 * M8) * G_xmraw;
  E[GP1][p] = wacc[2] + GP[0];
  E[GP2][p] = wacc[3] + GP[1];
  E[GP3][p] = wacc[4] + GP[2];
  if (!ELASTIC && WANTQ) {
    // Qp^-1 eight-cell sum: qpa = xl_raw c_q, c_q = -qpaw dh1 vx1
    E[GQP8][p] = qacc[0] + G_qpa * xl_raw * (-a.dh1 * fvx1) * dqpaw * 0.0625f;
    // Qs^-1 eight-cell sum: h = xm_raw c_h, xm = xm_raw (dth + DT c_h)
    E[GQS8][p] = qacc[1] + (G_h + DT * G_xm) * xm_raw * (-a.dh1 * fvx1) * dhw * 0.0625f;
    E[GQ1][p] = qacc[2] + GQP[0];
    E[GQ2][p] = qacc[3] + GQP[1];
    E[GQ3][p] = qacc[4] + GQP[2];
  }
}

// ---------------------------------------------------------------------------
// stress^T, gather part: adjoint strain rates -> adjoint velocities (images
// and the untouched k = top+2 values included); material weights -> the
// gradients of 1/lambda and 1/mu
// ---------------------------------------------------------------------------
constexpr int kGch = 4;  // x planes a gather thread marches (register queues along x)

__global__ void k_adj_stress_gather(const AdjArgs a) {
  const int k = a.sk0 - 2 + blockIdx.x * 32 + threadIdx.x;
  const int j = a.sj0 - 2 + blockIdx.y * 4 + threadIdx.y;
  const int ib = a.si0 - 2 + blockIdx.z * kGch;
  const int ie = min(ib + kGch - 1, a.si1 + 2);
  if (k > a.sk1 + 2 || j > a.sj1 + 2) return;
  const int S = a.g.slice, Y = a.g.yline;
  const long long q = (long long)ib * S + (long long)j * Y + k;
  const float c1 = a.c1, c2 = a.c2;
  const float* e1 = a.E[E1] + q;
  const float* e2 = a.E[E2] + q;
  const float* e3 = a.E[E3] + q;
  const float* e4 = a.E[E4] + q;
  const float* e5 = a.E[E5] + q;
  const float* e6 = a.E[E6] + q;
  float* Lu = a.L[LU] + q;
  float* Lv = a.L[LV] + q;
  float* Lw = a.L[LW] + q;
  // x queues: e1 at x-2, x-1, x; e4, e5 at x-1, x, x+1
  float e1m2 = e1[-(2 * S)], e1m1 = e1[-S], e1c = e1[0];
  float e4m1 = e4[-S], e4c = e4[0], e4p1 = e4[S];
  float e5m1 = e5[-S], e5c = e5[0], e5p1 = e5[S];
#pragma unroll 1
  for (int i = ib; i <= ie; ++i) {
    // the sums first, then the read-modify-writes, so that no load waits
    // behind a store
    const float e1p1 = e1[S], e4p2 = e4[2 * S], e5p2 = e5[2 * S];
    const float du = c1 * (e1m1 - e1c) + c2 * (e1m2 - e1p1) +
                     c1 * (e4[-Y] - e4c) + c2 * (e4[-(2 * Y)] - e4[Y]) +
                     c1 * (e5[-1] - e5c) + c2 * (e5[-2] - e5[1]);
    const float dv = c1 * (e2[0] - e2[Y]) + c2 * (e2[-Y] - e2[2 * Y]) +
                     c1 * (e4c - e4p1) + c2 * (e4m1 - e4p2) +
                     c1 * (e6[-1] - e6[0]) + c2 * (e6[-2] - e6[1]);
    const float dw = c1 * (e3[0] - e3[1]) + c2 * (e3[-1] - e3[2]) +
                     c1 * (e5c - e5p1) + c2 * (e5m1 - e5p2) +
                     c1 * (e6[-Y] - e6[0]) + c2 * (e6[-(2 * Y)] - e6[Y]);
    const float lu = Lu[0], lv = Lv[0], lw = Lw[0];
    Lu[0] = lu + du;
    Lv[0] = lv + dv;
    Lw[0] = lw + dw;
    e1m2 = e1m1; e1m1 = e1c; e1c = e1p1;
    e4m1 = e4c; e4c = e4p1; e4p1 = e4p2;
    e5m1 = e5c; e5c = e5p1; e5p1 = e5p2;
    e1 += S; e2 += S; e3 += S; e4 += S; e5 += S; e6 += S;
    Lu += S; Lv += S; Lw += S;
  }
}

// ---------------------------------------------------------------------------
// images^T over the imaged columns: the adjoint of the image values (top+1)
// goes to the velocities they were made from, and to lam_mu; the images are
// overwritten each step, so their adjoint is cleared
// ---------------------------------------------------------------------------
// image-adjoint scratch: column (i, j) of the ring-extended surface window
__device__ __forceinline__ long long img_plane(const AdjArgs& a) {
  return (long long)(a.si1 - a.si0 + 3) * (a.sj1 - a.sj0 + 3);
}
__device__ __forceinline__ long long img_index(const AdjArgs& a, int i, int j) {
  return (long long)(i - a.si0 + 1) * (a.sj1 - a.sj0 + 3) + (j - a.sj0 + 1);
}

__global__ void k_adj_images(const AdjArgs a) {
  // targets: the imaged columns and the one-column ring the images also read
  const int j = a.sj0 - 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = a.si0 - 1 + blockIdx.y;
  if (j > a.sj1 + 1 || i > a.si1 + 1) return;
  const long long S = a.g.slice, Y = a.g.yline;
  const long long p = (long long)i * S + (long long)j * Y + a.g.top();
  const float* Lu = a.L[LU];
  const float* Lv = a.L[LV];
  const float* Lw = a.L[LW];
  // adjoints of the images of column (ii, jj), zero outside the imaged window
  auto win = [&](int ii, int jj) { return ii >= a.si0 && ii <= a.si1 && jj >= a.sj0 && jj <= a.sj1; };
  auto col = [&](int ii, int jj) { return (long long)ii * S + (long long)jj * Y + a.g.top(); };
  auto Au = [&](int ii, int jj) { return win(ii, jj) ? Lu[col(ii, jj) + 1] : 0.f; };
  auto Av = [&](int ii, int jj) { return win(ii, jj) ? Lv[col(ii, jj) + 1] : 0.f; };
  auto Aw = [&](int ii, int jj) { return win(ii, jj) ? Lw[col(ii, jj) + 1] : 0.f; };
  auto lm = [&](int ii, int jj) { return a.lam_mu[(long long)ii * a.lam_mu_ld + jj]; };
  auto m1 = [&](int ii) { return ii < a.gx_lim ? 1.0f : 0.0f; };
  auto m2 = [&](int jj) { return jj >= a.gy_min ? 1.0f : 0.0f; };
  // lZ(ii, jj) = adjoint of Z at column (ii, jj): -lam_mu * A_w
  auto lZ = [&](int ii, int jj) { return win(ii, jj) ? -lm(ii, jj) * Aw(ii, jj) : 0.f; };
  // Z = m1 (u_{i+1} - w_{i+1} + w) - (u - w + w_{i-1}) + (u_{i+1} - u)
  //     + (v - w_{j+1} + w) - m2 (v_{j-1} - w + w_{j-1}) + (v - v_{j-1})
  const float du = Au(i, j) - 2.0f * lZ(i, j) + (m1(i - 1) + 1.0f) * lZ(i - 1, j);
  const float dv = Av(i, j) + 2.0f * lZ(i, j) - (m2(j + 1) + 1.0f) * lZ(i, j + 1);
  const float dw = -Au(i, j) + Au(i + 1, j) + Av(i, j) - Av(i, j - 1) +
                   (m1(i) + 2.0f + m2(j)) * lZ(i, j) - m1(i - 1) * lZ(i - 1, j) -
                   lZ(i + 1, j) - lZ(i, j - 1) - m2(j + 1) * lZ(i, j + 1);
  // lam_mu gradient: d wimg / d lam_mu = -Z
  if (win(i, j)) {
    const float* u = a.fu;
    const float* v = a.fv;
    const float* w = a.fw;
    const long long VS = a.vb.S, VY = a.vb.Y;
    const long long q = (long long)i * VS + (long long)j * VY + a.g.top() - a.vb.off;
    const float Z = m1(i) * (u[q + VS] - w[q + VS] + w[q]) - (u[q] - w[q] + w[q - VS]) +
                    (u[q + VS] - u[q]) + (v[q] - w[q + VY] + w[q]) -
                    m2(j) * (v[q - VY] - w[q] + w[q - VY]) + (v[q] - v[q - VY]);
    a.glm[(long long)i * a.lam_mu_ld + j] += -Z * Aw(i, j);
  }
  // neighbouring columns read this column's image adjoints, so the updates
  // wait for the next kernel (k_adj_vel_cell)
  const long long ip = img_index(a, i, j), np = img_plane(a);
  a.img[ip] = du;
  a.img[ip + np] = dv;
  a.img[ip + 2 * np] = dw;
  a.img[ip + 3 * np] = Aw(i, j);  // to w(top-1)
}


// ---------------------------------------------------------------------------
// velocity^T, pointwise part
// ---------------------------------------------------------------------------
__global__ void k_adj_vel_cell(const AdjArgs a) {
  const int k = a.vk0 + blockIdx.x * 32 + threadIdx.x;
  const int j = a.vj0 + blockIdx.y * 4 + threadIdx.y;
  const int i = a.vi0 + blockIdx.z;
  if (k > a.vk1 || j > a.vj1 || i > a.vi1) return;
  const long long S = a.g.slice, Y = a.g.yline;
  const long long p = (long long)i * S + (long long)j * Y + k;
  const float* d = a.d1;
  const float r1 = 0.25f * (d[p] + d[p - Y] + d[p - 1] + d[p - Y - 1]);
  const float r2 = 0.25f * (d[p] + d[p + S] + d[p - 1] + d[p + S - 1]);
  const float r3 = 0.25f * (d[p] + d[p + S] + d[p - Y] + d[p + S - Y]);
  const float fd1 = a.dth / r1, fd2 = a.dth / r2, fd3 = a.dth / r3;
  const float dc = a.dcrjx[i] * a.dcrjy[j] * a.dcrjz[k];
  // fd * D(sigma) * dc of the forward update = u' - dc u
  const long long pv = (long long)i * a.vb.S + (long long)j * a.vb.Y + k - a.vb.off;
  const float su = a.fu[pv] - dc * a.bu[pv];
  const float sv = a.fv[pv] - dc * a.bv[pv];
  const float sw = a.fw[pv] - dc * a.bw[pv];
  float lu = a.L[LU][p], lv = a.L[LV][p], lw = a.L[LW][p];
  const float wa = a.V[VEA][p], wb = a.V[VEB][p], wc = a.V[VEC][p];
  // the image adjoints of the surface columns (k_adj_images) enter here:
  // u, v, w(top) of the window and its ring, w(top-1) of the window; the
  // imaged velocities and stresses above the surface return to zero (fstr
  // and the images rewrite them every step; their transposes went below)
  const int top = a.g.top();
  if (k >= top - 1 && k <= top + 2) {
    const bool ring = i >= a.si0 - 1 && i <= a.si1 + 1 && j >= a.sj0 - 1 && j <= a.sj1 + 1;
    const bool in = i >= a.si0 && i <= a.si1 && j >= a.sj0 && j <= a.sj1;
    if (k == top && ring) {
      const long long ip = img_index(a, i, j), np = img_plane(a);
      lu += a.img[ip];
      lv += a.img[ip + np];
      lw += a.img[ip + 2 * np];
    } else if (k == top - 1 && in) {
      lw += a.img[img_index(a, i, j) + 3 * img_plane(a)];
    } else if (k > top && in) {
      lu = lv = lw = 0.f;
    }
    if (k == top && in) {
      for (int d = 1; d <= 2; ++d) {
        if (top + d > a.vk1) {  // cells no thread of this kernel owns
          a.L[LU][p + d] = 0.f;
          a.L[LV][p + d] = 0.f;
          a.L[LW][p + d] = 0.f;
        }
        a.L[LZZ][p + d] = 0.f;
        a.L[LXZ][p + d] = 0.f;
        a.L[LYZ][p + d] = 0.f;
      }
    }
  }
  a.L[LU][p] = dc * lu;
  a.L[LV][p] = dc * lv;
  a.L[LW][p] = dc * lw;
  a.V[VA][p] = fd1 * dc * lu;
  a.V[VB][p] = fd2 * dc * lv;
  a.V[VC][p] = fd3 * dc * lw;
  // d fd / d rho_avg = -fd / rho_avg, each of the four densities weighs 1/4:
  // d u' / d d(q) = -1/4 * (fd D dc) / rho_avg
  // summed over the time steps (k_adj_material applies their transposes)
  a.V[VEA][p] = wa + -0.25f / r1 * su * lu;
  a.V[VEB][p] = wb + -0.25f / r2 * sv * lv;
  a.V[VEC][p] = wc + -0.25f / r3 * sw * lw;
}

// ---------------------------------------------------------------------------
// velocity^T, gather part: weighted adjoint velocities -> adjoint stresses;
// density weights -> the density gradient
// ---------------------------------------------------------------------------
__global__ void k_adj_vel_gather(const AdjArgs a) {
  const int k = a.vk0 - 2 + blockIdx.x * 32 + threadIdx.x;
  const int j = a.vj0 - 2 + blockIdx.y * 4 + threadIdx.y;
  const int ib = a.vi0 - 2 + blockIdx.z * kGch;
  const int ie = min(ib + kGch - 1, a.vi1 + 2);
  if (k > a.vk1 + 2 || j > a.vj1 + 2) return;
  const int S = a.g.slice, Y = a.g.yline;
  const long long q = (long long)ib * S + (long long)j * Y + k;
  const float c1 = a.c1, c2 = a.c2;
  const float* A = a.V[VA] + q;
  const float* B = a.V[VB] + q;
  const float* C = a.V[VC] + q;
  float* L[6] = {a.L[LXX] + q, a.L[LXY] + q, a.L[LXZ] + q,
                 a.L[LYY] + q, a.L[LYZ] + q, a.L[LZZ] + q};
  // x queues: A at x-1, x, x+1; B, C at x-2, x-1, x
  float Am1 = A[-S], Ac = A[0], Ap1 = A[S];
  float Bm2 = B[-(2 * S)], Bm1 = B[-S], Bc = B[0];
  float Cm2 = C[-(2 * S)], Cm1 = C[-S], Cc = C[0];
#pragma unroll 1
  for (int i = ib; i <= ie; ++i) {
    // the sums first, then the read-modify-writes (no load behind a store)
    const float Ap2 = A[2 * S], Bp1 = B[S], Cp1 = C[S];
    const float dxx = c1 * (Ac - Ap1) + c2 * (Am1 - Ap2);
    const float dxy = c1 * (Ac - A[Y]) + c2 * (A[-Y] - A[2 * Y]) +
                      c1 * (Bm1 - Bc) + c2 * (Bm2 - Bp1);
    const float dxz = c1 * (Ac - A[1]) + c2 * (A[-1] - A[2]) +
                      c1 * (Cm1 - Cc) + c2 * (Cm2 - Cp1);
    const float dyy = c1 * (B[-Y] - Bc) + c2 * (B[-(2 * Y)] - B[Y]);
    const float dyz = c1 * (Bc - B[1]) + c2 * (B[-1] - B[2]) +
                      c1 * (Cc - C[Y]) + c2 * (C[-Y] - C[2 * Y]);
    const float dzz = c1 * (C[-1] - Cc) + c2 * (C[-2] - C[1]);
    const float l0 = L[0][0], l1 = L[1][0], l2 = L[2][0];
    const float l3 = L[3][0], l4 = L[4][0], l5 = L[5][0];
    L[0][0] = l0 + dxx;
    L[1][0] = l1 + dxy;
    L[2][0] = l2 + dxz;
    L[3][0] = l3 + dyy;
    L[4][0] = l4 + dyz;
    L[5][0] = l5 + dzz;
    Am1 = Ac; Ac = Ap1; Ap1 = Ap2;
    Bm2 = Bm1; Bm1 = Bc; Bc = Bp1;
    Cm2 = Cm1; Cm1 = Cc; Cc = Cp1;
    A += S; B += S; C += S;
#pragma unroll
    for (int f = 0; f < 6; ++f) L[f] += S;
  }
}

// ---------------------------------------------------------------------------
// the material weights summed over the steps -> gradients on the padded
// arrays, once per sweep: each cell's weight goes to every material value its
// forward averages read
//   1/lambda, 1/mu : eight-cell sums at the normal-stress node (box8), mu
//                    pairs at the shear nodes (xy: k-1, xz: j-1, yz: i+1)
//   rho            : four-cell averages of the three velocity nodes
// ---------------------------------------------------------------------------
__global__ void k_adj_material(const AdjArgs a, int i0, int j0, int k0, int ni, int nj,
                               int nk) {
  const int k = k0 + blockIdx.x * 32 + threadIdx.x;
  const int j = j0 + blockIdx.y * 4 + threadIdx.y;
  const int i = i0 + blockIdx.z;
  if (k >= k0 + nk || j >= j0 + nj || i >= i0 + ni) return;
  const long long S = a.g.slice, Y = a.g.yline;
  const long long q = (long long)i * S + (long long)j * Y + k;
  // box8(p) = {p, p+S, p-Y, p+S-Y, p-1, p+S-1, p-Y-1, p+S-Y-1} contains q for
  // p in {q, q-S, q+Y, q-S+Y, q+1, q-S+1, q+Y+1, q-S+Y+1}
  auto box = [&](const float* x) {
    return x[q] + x[q - S] + x[q + Y] + x[q - S + Y] + x[q + 1] + x[q - S + 1] + x[q + Y + 1] +
           x[q - S + Y + 1];
  };
  a.glam[q] = box(a.E[GL8]);
  a.gmu[q] = box(a.E[GM8]) + a.E[GP1][q] + a.E[GP1][q + 1] + a.E[GP2][q] + a.E[GP2][q + Y] +
             a.E[GP3][q] + a.E[GP3][q - S];
  if (a.gqp) {  // the inverse quality factors follow the same averages
    a.gqp[q] = box(a.E[GQP8]);
    a.gqs[q] = box(a.E[GQS8]) + a.E[GQ1][q] + a.E[GQ1][q + 1] + a.E[GQ2][q] +
               a.E[GQ2][q + Y] + a.E[GQ3][q] + a.E[GQ3][q - S];
  }
  const float* ea = a.V[VEA];
  const float* eb = a.V[VEB];
  const float* ec = a.V[VEC];
  a.gd[q] = ea[q] + ea[q + Y] + ea[q + 1] + ea[q + Y + 1] + eb[q] + eb[q - S] + eb[q + 1] +
            eb[q - S + 1] + ec[q] + ec[q - S] + ec[q + Y] + ec[q - S + Y];
}

// One thread per distinct (component, cell); receivers sharing a cell are
// added in receiver order (first[c] .. first[c+1] of order[]).
__global__ void k_adj_inject(float* Lu, float* Lv, float* Lw, const long long* idx,
                             const int* comp, const int* first, const int* order, int ncell,
                             const float* res) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int r0 = order[first[c]];
  float* L = comp[r0] == 0 ? Lu : (comp[r0] == 1 ? Lv : Lw);
  float acc = L[idx[r0]];
  for (int n = first[c]; n < first[c + 1]; ++n) acc += res[order[n]];
  L[idx[r0]] = acc;
}

__global__ void k_sample(const float* u, const float* v, const float* w, const long long* idx,
                         const int* comp, int n, float* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float* f = comp[r] == 0 ? u : (comp[r] == 1 ? v : w);
  out[r] = f[idx[r]];
}

// ---------------------------------------------------------------------------
// gradients on the padded arrays -> interior lambda, mu, rho
// ---------------------------------------------------------------------------
__global__ void k_adj_fold(const AdjArgs a, float* g_lambda, float* g_mu, float* g_rho) {
  const long long n = (long long)a.g.nxt * a.g.nyt * a.g.nzt;
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int x = (int)(c % a.g.nxt), y = (int)((c / a.g.nxt) % a.g.nyt),
            z = (int)(c / ((long long)a.g.nxt * a.g.nyt));
  const int lo = 2 + AWP_NGSL, hix = a.g.nxt + 1 + AWP_NGSL, hiy = a.g.nyt + 1 + AWP_NGSL;
  const int kb = AWP_ALIGN, kt = a.g.nzt + AWP_ALIGN - 1;
  const int i = x + lo, j = y + lo, k = kt - z;
  // the border fill copies (i, j, k) into the ghost cells that clamp onto it
  int is[2] = {i, 0}, js[2] = {j, 0}, ks[2] = {k, 0};
  int ni = 1, nj = 1, nk = 1;
  if (i == lo) is[ni++] = lo - 1;
  if (i == hix) is[ni++] = hix + 1;
  if (j == lo) js[nj++] = lo - 1;
  if (j == hiy) js[nj++] = hiy + 1;
  if (k == kb) ks[nk++] = kb - 1;
  if (k == kt) ks[nk++] = kt + 1;
  float gl = 0.f, gm = 0.f, gr = 0.f;
  for (int ii = 0; ii < ni; ++ii)
    for (int jj = 0; jj < nj; ++jj)
      for (int kk = 0; kk < nk; ++kk) {
        const long long p = (long long)is[ii] * a.g.slice + (long long)js[jj] * a.g.yline + ks[kk];
        gl += a.glam[p];
        gm += a.gmu[p];
        gr += a.gd[p];
      }
  const long long p0 = (long long)i * a.g.slice + (long long)j * a.g.yline + k;
  const float il = a.lam[p0], im = a.mu[p0];  // 1/lambda, 1/mu
  float g_l = -il * il * gl;                  // d(1/lambda)/d lambda = -1/lambda^2
  float g_m = -im * im * gm;
  if (k == kt && i >= a.si0 && i <= a.si1 && j >= a.sj0 && j <= a.sj1) {
    // lam_mu = lambda / (lambda + 2 mu)
    const float lm = 1.0f / il, mm = 1.0f / im, den = lm + 2.0f * mm;
    const float glm = a.glm[(long long)i * a.lam_mu_ld + j];
    g_l += glm * 2.0f * mm / (den * den);
    g_m += -glm * 2.0f * lm / (den * den);
  }
  g_lambda[c] = g_l;
  g_mu[c] = g_m;
  g_rho[c] = gr;
}

// padded Qp^-1 / Qs^-1 gradients -> interior cells, border-fill copies folded
__global__ void k_adj_fold_q(const AdjArgs a, float* g_qp, float* g_qs) {
  const long long n = (long long)a.g.nxt * a.g.nyt * a.g.nzt;
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int x = (int)(c % a.g.nxt), y = (int)((c / a.g.nxt) % a.g.nyt),
            z = (int)(c / ((long long)a.g.nxt * a.g.nyt));
  const int lo = 2 + AWP_NGSL, hix = a.g.nxt + 1 + AWP_NGSL, hiy = a.g.nyt + 1 + AWP_NGSL;
  const int kb = AWP_ALIGN, kt = a.g.nzt + AWP_ALIGN - 1;
  const int i = x + lo, j = y + lo, k = kt - z;
  int is[2] = {i, 0}, js[2] = {j, 0}, ks[2] = {k, 0};
  int ni = 1, nj = 1, nk = 1;
  if (i == lo) is[ni++] = lo - 1;
  if (i == hix) is[ni++] = hix + 1;
  if (j == lo) js[nj++] = lo - 1;
  if (j == hiy) js[nj++] = hiy + 1;
  if (k == kb) ks[nk++] = kb - 1;
  if (k == kt) ks[nk++] = kt + 1;
  float gp = 0.f, gs = 0.f;
  for (int ii = 0; ii < ni; ++ii)
    for (int jj = 0; jj < nj; ++jj)
      for (int kk = 0; kk < nk; ++kk) {
        const long long p = (long long)is[ii] * a.g.slice + (long long)js[jj] * a.g.yline + ks[kk];
        gp += a.gqp[p];
        gs += a.gqs[p];
      }
  g_qp[c] = gp;
  g_qs[c] = gs;
}

__global__ void k_set_qinv(const float* qpinv, const float* qsinv, float* qp, float* qs,
                           const AwpGeom g) {
  const int lo = 2 + AWP_NGSL, hix = g.nxt + 1 + AWP_NGSL, hiy = g.nyt + 1 + AWP_NGSL;
  const int kb = AWP_ALIGN, kt = g.nzt + AWP_ALIGN - 1;
  const int k = kb - 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = lo - 1 + blockIdx.y;
  const int i = lo - 1 + blockIdx.z;
  if (k > kt + 1 || j > hiy + 1 || i > hix + 1) return;
  const int ci = min(max(i, lo), hix), cj = min(max(j, lo), hiy), ck = min(max(k, kb), kt);
  const long long c = (long long)(kt - ck) * g.nxt * g.nyt + (long long)(cj - lo) * g.nxt + (ci - lo);
  const long long p = (long long)i * g.slice + (long long)j * g.yline + k;
  qp[p] = qpinv[c];
  qs[p] = qsinv[c];
}

__global__ void k_set_moduli(const float* lambda, const float* mu_, const float* rho, float* lam,
                             float* mu, float* d1, const AwpGeom g) {
  // every cell of the one-cell shell around the interior takes the clamped
  // interior value (the border fill of the media set-up)
  const int lo = 2 + AWP_NGSL, hix = g.nxt + 1 + AWP_NGSL, hiy = g.nyt + 1 + AWP_NGSL;
  const int kb = AWP_ALIGN, kt = g.nzt + AWP_ALIGN - 1;
  const int k = kb - 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = lo - 1 + blockIdx.y;
  const int i = lo - 1 + blockIdx.z;
  if (k > kt + 1 || j > hiy + 1 || i > hix + 1) return;
  const int ci = min(max(i, lo), hix), cj = min(max(j, lo), hiy), ck = min(max(k, kb), kt);
  const long long c = (long long)(kt - ck) * g.nxt * g.nyt + (long long)(cj - lo) * g.nxt + (ci - lo);
  const long long p = (long long)i * g.slice + (long long)j * g.yline + k;
  lam[p] = __frcp_rn(lambda[c]);  // correctly rounded (the build divides approximately)
  mu[p] = __frcp_rn(mu_[c]);
  d1[p] = rho[c];
}

// padded velocities -> VelBox rows; rows beyond nk (up to ld) are not read
__global__ void k_pack_vel(const float* __restrict__ u, const float* __restrict__ v,
                           const float* __restrict__ w, float* __restrict__ du,
                           float* __restrict__ dv, float* __restrict__ dw, const VelBox b,
                           long long S, long long Y) {
  const int kk = blockIdx.x * 32 + threadIdx.x;
  const int jj = blockIdx.y * 4 + threadIdx.y;
  const int ii = blockIdx.z;
  if (kk >= b.nk || jj >= b.nj) return;
  const long long p = (long long)(b.i0 + ii) * S + (long long)(b.j0 + jj) * Y + b.k0 + kk;
  const long long q = (long long)ii * b.S + (long long)jj * b.Y + kk;
  du[q] = u[p];
  dv[q] = v[p];
  dw[q] = w[p];
}

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

cudaError_t awp_launch_pack_vel(const float* u, const float* v, const float* w, float* du,
                                float* dv, float* dw, const VelBox& b, const AwpGeom& g,
                                cudaStream_t st) {
  if (b.ni <= 0 || b.nj <= 0 || b.nk <= 0) return cudaSuccess;
  k_pack_vel<<<dim3(cdiv(b.nk, 32), cdiv(b.nj, 4), b.ni), dim3(32, 4), 0, st>>>(
      u, v, w, du, dv, dw, b, g.slice, g.yline);
  return cudaGetLastError();
}

cudaError_t awp_launch_adjoint_step(const AdjArgs& a, cudaStream_t st) {
  const int si = a.si1 - a.si0 + 1, sj = a.sj1 - a.sj0 + 1, sk = a.sk1 - a.sk0 + 1;
  const dim3 blk(32, 4);
  // the imaging (fstr) transpose runs inside k_adj_stress_cell
  const dim3 sgrid(cdiv(sk, 32), cdiv(sj, 4), si);
  if (a.elastic)
    k_adj_stress_cell<true, false><<<sgrid, blk, 0, st>>>(a);
  else if (a.want_q)
    k_adj_stress_cell<false, true><<<sgrid, blk, 0, st>>>(a);
  else
    k_adj_stress_cell<false, false><<<sgrid, blk, 0, st>>>(a);
  k_adj_stress_gather<<<dim3(cdiv(sk + 4, 32), cdiv(sj + 4, 4), cdiv(si + 4, kGch)), blk, 0,
                        st>>>(a);
  k_adj_images<<<dim3(cdiv(sj + 2, 128), si + 2), 128, 0, st>>>(a);
  const int vi = a.vi1 - a.vi0 + 1, vj = a.vj1 - a.vj0 + 1, vk = a.vk1 - a.vk0 + 1;
  k_adj_vel_cell<<<dim3(cdiv(vk, 32), cdiv(vj, 4), vi), blk, 0, st>>>(a);
  k_adj_vel_gather<<<dim3(cdiv(vk + 4, 32), cdiv(vj + 4, 4), cdiv(vi + 4, kGch)), blk, 0,
                     st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_adjoint_inject(float* const L[3], const long long* idx, const int* comp,
                                      const int* first, const int* order, int ncell,
                                      const float* res, cudaStream_t st) {
  if (ncell <= 0) return cudaSuccess;
  k_adj_inject<<<cdiv(ncell, 128), 128, 0, st>>>(L[0], L[1], L[2], idx, comp, first, order,
                                                 ncell, res);
  return cudaGetLastError();
}

cudaError_t awp_launch_sample(const float* u, const float* v, const float* w,
                              const long long* idx, const int* comp, int nrec, float* out,
                              cudaStream_t st) {
  if (nrec <= 0) return cudaSuccess;
  k_sample<<<cdiv(nrec, 128), 128, 0, st>>>(u, v, w, idx, comp, nrec, out);
  return cudaGetLastError();
}

cudaError_t awp_launch_adjoint_fold(const AdjArgs& a, float* g_lambda, float* g_mu,
                                    float* g_rho, cudaStream_t st) {
  {
    // every cell a weight can reach: the stress and velocity ranges +-2
    const int i0 = min(a.si0, a.vi0) - 2, i1 = max(a.si1, a.vi1) + 2;
    const int j0 = min(a.sj0, a.vj0) - 2, j1 = max(a.sj1, a.vj1) + 2;
    const int k0 = min(a.sk0, a.vk0) - 2, k1 = max(a.sk1, a.vk1) + 2;
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    k_adj_material<<<dim3(cdiv(nk, 32), cdiv(nj, 4), ni), dim3(32, 4), 0, st>>>(a, i0, j0, k0,
                                                                                ni, nj, nk);
  }
  const long long n = (long long)a.g.nxt * a.g.nyt * a.g.nzt;
  k_adj_fold<<<cdiv(n, 256), 256, 0, st>>>(a, g_lambda, g_mu, g_rho);
  return cudaGetLastError();
}

cudaError_t awp_launch_set_moduli(const float* lambda, const float* mu_, const float* rho,
                                  float* lam, float* mu, float* d1, const AwpGeom& g,
                                  cudaStream_t st) {
  const dim3 grid(cdiv(g.nzt + 2, 64), g.nyt + 2, g.nxt + 2);
  k_set_moduli<<<grid, 64, 0, st>>>(lambda, mu_, rho, lam, mu, d1, g);
  return cudaGetLastError();
}

cudaError_t awp_launch_adjoint_fold_q(const AdjArgs& a, float* g_qpinv, float* g_qsinv,
                                      cudaStream_t st) {
  if (!a.gqp || !a.gqs) return cudaErrorInvalidValue;
  const long long n = (long long)a.g.nxt * a.g.nyt * a.g.nzt;
  k_adj_fold_q<<<cdiv(n, 256), 256, 0, st>>>(a, g_qpinv, g_qsinv);
  return cudaGetLastError();
}

cudaError_t awp_launch_set_qinv(const float* qpinv, const float* qsinv, float* qp, float* qs,
                                const AwpGeom& g, cudaStream_t st) {
  const dim3 grid(cdiv(g.nzt + 2, 64), g.nyt + 2, g.nxt + 2);
  k_set_qinv<<<grid, 64, 0, st>>>(qpinv, qsinv, qp, qs, g);
  return cudaGetLastError();
}
