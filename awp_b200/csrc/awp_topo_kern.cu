// Curvilinear (topography) velocity and stress half-steps of the top grid.
//
// The reference spells these operators out as generated code, one kernel for
// the interior (k below the top six points) and one for the six boundary rows
// next to the free surface:
//   velocity: dtopo_vel_111_unroll (kernels/velocity_unroll.cu:1-428) and
//             dtopo_vel_112 (kernels/optimized_velocity.cu:1040-1629),
//   stress:   dtopo_str_111 / dtopo_str_112 (kernels/stress_attenuation.cu:73-1415),
// launched by topo_velocity_*_H (velocity.cu) and topo_stress_*_H
// (stress_attenuation.cu).  Here each half-step is one kernel.  A warp owns 32
// consecutive k of one (i, j) column and every lane loads the values of its
// own level only: the vertical operators (7-point differences of horizontal
// interpolants, 4-point differences) take the neighbouring levels from the
// neighbouring lanes by warp shuffles, so each value crosses the memory system
// once per column instead of once per stencil point.  Warps overlap by three
// levels on each side (tiles of 26 output levels; the top tile outputs its 29
// levels under the surface), the halo lanes only feeding their neighbours.
// The boundary-closure rows r = nz-1-k of the summation-by-parts tables
// (awp_topo_tables.h) read the top levels of the column, which all sit in the
// top tile, by broadcast shuffles.
//
// Latency: a CTA (four warps = four j columns) takes AWP_TOPO_MARCH
// consecutive x planes one after another, so x-neighbour reads find the
// earlier planes in L1.  The values a thread reads only once are copied to
// shared memory by cp.async when the thread starts on a plane: in the
// velocity kernel all 31 of its 3-D operands, in the stress kernel the
// stresses and memory variables the update reads at the end.  Both kernels
// are then bound by instruction issue (ncu: issue active ~80 %, "not
// selected" the largest stall), not by memory latency.
//
// Term structure (f = surface function interpolants, g = vertical metric;
// relative indices, k = 0 the bottom point of the grid):
//   u_t = (A / (f g3 rho)) * [ D_x(f g3 sigma_x) + D_y(f g3 sigma_y) + D_z sigma_z
//                              - f1 * Dz(g P_x sigma_x) - f2 * Dz(g P_y sigma_y) ]
//   sigma_t from strain rates  D_x u - J^-1 g P_x(f1 Dz u)  etc.
// and the memory-variable / sponge update shared with the Cartesian kernels
// (awp_stress_coef / awp_stress_update).  Products and sums follow the
// reference's left-to-right order; the reference build contracts them into
// FMAs at its compiler's choice, so agreement is to rounding, not bitwise.
#include "awp_topo_kern.cuh"

#include "awp_stencil.cuh"
#include "awp_topo_tables.h"

namespace {

// interior 4-point interpolation / difference and the 7-point vertical
// difference of the interpolant (the reference's double literals as float)
constexpr float kP0 = (float)-0.0625, kP1 = (float)0.5625;
constexpr float kD0 = (float)0.0416666666666667, kD1 = (float)-1.1250000000000000;
constexpr float kZ0 = (float)-0.0026041666666667, kZ1 = (float)0.0937500000000000,
                kZ2 = (float)-0.6796875000000000;
constexpr unsigned kAll = 0xffffffffu;
constexpr int kTileOut = 26;  // output levels of a tile below the top one

__device__ __forceinline__ float gk(const float* __restrict__ g, int k) {
  return __ldg(g + k + AWP_ALIGN);
}
// The reference forms these reciprocals and quotients in double and rounds
// the result to float.  For float operands the double quotient (53 bits)
// rounded again to 24 bits equals the correctly rounded float quotient
// (double rounding is innocuous for division when the wider format has at
// least 2p + 2 bits; Figueroa, "When is double rounding innocuous?", 1995),
// so the IEEE float division gives the same bits without the FP64 pipe.
__device__ __forceinline__ float inv(float x) { return __frcp_rn(x); }
__device__ __forceinline__ float quot(float x, float y) { return __fdiv_rn(x, y); }

// Per-thread asynchronous 4-byte copies global -> shared (cp.async), issued at
// the start of a kernel for the values it reads only at its end, so their
// latency overlaps the stencil arithmetic.  Each thread reads back its own
// slots after cp.async.wait_all; no block barrier is needed.
__device__ __forceinline__ void cpa4(float* s, const float* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(s)),
               "l"(g)
               : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Column position of a warp: tile t = 0 holds the top 32 levels, tile t > 0
// the 32 levels starting 26 t lower.  A lane outputs its level when it is not
// a halo lane (three at each end; the top tile has no upper halo) and k >= 3
// (the reference leaves the three bottom points to the mesh coupling,
// dm_offset = 3).
struct ColPos {
  int k, r, lane;
  bool top, out;
  __device__ ColPos(int nz, int tile) {
    lane = threadIdx.x;
    top = (tile == 0);
    k = nz - 32 - kTileOut * tile + lane;
    r = (top && lane >= 26) ? 31 - lane : -1;  // boundary row nz-1-k of the top six
    out = lane >= 3 && (top || lane <= 28) && k >= 3;
  }
};

// Boundary-closure rows of the top tile: lane 31 - r holds row r of T
// applied to the top NT levels (lanes 31, 30, ...), other lanes keep s.  Every
// row is formed with compile-time table indices (constant-bank operands, no
// per-lane indexed constant loads) and the lane picks its own.
template <int NT>
__device__ __forceinline__ float closure(float v, const ColPos& c, const float (&T)[6][NT]) {
  float top[NT];
#pragma unroll
  for (int m = 0; m < NT; ++m) top[m] = __shfl_sync(kAll, v, 31 - m);
  float s = 0.f;
#pragma unroll
  for (int rr = 0; rr < 6; ++rr) {
    float b = 0.f;
#pragma unroll
    for (int m = NT - 1; m >= 0; --m) b += T[rr][m] * top[m];
    if (c.r == rr) s = b;
  }
  return s;
}

// 7-point vertical difference at the lane's level of a value v(k) held one
// level per lane (interior coefficients), or boundary row r of T in the top
// tile.  Summation order as the reference's operators.
template <int NT>
__device__ __forceinline__ float zd7(float v, const ColPos& c, const float (&T)[6][NT]) {
  const float m3 = __shfl_up_sync(kAll, v, 3), m2 = __shfl_up_sync(kAll, v, 2),
              m1 = __shfl_up_sync(kAll, v, 1), p1 = __shfl_down_sync(kAll, v, 1),
              p2 = __shfl_down_sync(kAll, v, 2), p3 = __shfl_down_sync(kAll, v, 3);
  float s = kZ0 * m3 + kZ1 * m2 + kZ2 * m1 - kZ2 * p1 - kZ1 * p2 - kZ0 * p3;
  if (c.top) {  // warp-uniform branch
    const float b = closure(v, c, T);
    if (c.r >= 0) s = b;
  }
  return s;
}

// 4-point vertical difference: half-point form (k-2..k+1) or node form
// (k-1..k+2), or boundary row r.
template <int NT>
__device__ __forceinline__ float zd4(float v, const ColPos& c, bool half,
                                     const float (&T)[6][NT]) {
  const float m2 = __shfl_up_sync(kAll, v, 2), m1 = __shfl_up_sync(kAll, v, 1),
              p1 = __shfl_down_sync(kAll, v, 1), p2 = __shfl_down_sync(kAll, v, 2);
  float s = half ? kD0 * m2 + kD1 * m1 - kD1 * v - kD0 * p1
                 : kD0 * m1 + kD1 * v - kD1 * p1 - kD0 * p2;
  if (c.top) {
    const float b = closure(v, c, T);
    if (c.r >= 0) s = b;
  }
  return s;
}

struct Cell {
  long long o;   // padded index of (i, j, k)
  long long of;  // index of (i, j) in the 2-D metric arrays
  int S, Y, F;
  __device__ Cell(const TopoArgs& a, int i, int j, int k)
      : o((long long)(i + AWP_NGSL + 2) * a.slice + (long long)(j + AWP_NGSL + 2) * a.yline +
          (k + AWP_ALIGN)),
        of((long long)(i + AWP_NGSL + 2) * a.fld + (j + AWP_NGSL + 2 + AWP_ALIGN)),
        S(a.slice), Y(a.yline), F(a.fld) {}
  // 2-D metric at (i+di, j+dj)
  __device__ __forceinline__ float fm(const float* __restrict__ f, int di, int dj) const {
    return __ldg(f + of + (di * F + dj));
  }
};

}  // namespace

// ===========================================================================
// Velocity
// ===========================================================================
// CTAs per SM the register allocation is held to (64 and 48 registers), and
// x planes per CTA; chosen by timing at 512 x 512 x 256 with a hill.
#ifndef AWP_TOPO_VEL_MINB
#define AWP_TOPO_VEL_MINB 8
#endif
#ifndef AWP_TOPO_STR_MINB
#define AWP_TOPO_STR_MINB 10
#endif
#ifndef AWP_TOPO_MARCH
#define AWP_TOPO_MARCH 4
#endif

// every 3-D value a velocity thread reads, staged by cp.async in one batch
enum VelSlot {
  kU, kV, kW, kR00, kR0m, kRm0, kRmm,
  kX11_0, kX11_m2, kX11_m1, kX11_p1,
  kY12_0, kY12_m2, kY12_m1, kY12_p1, kX12_m1, kX12_p1, kX12_p2,
  kX13_0, kX13_m1, kX13_p1, kX13_p2,
  kY22_0, kY22_m1, kY22_p1, kY22_p2,
  kY23_0, kY23_m2, kY23_m1, kY23_p1,
  kZ33, kVelPre
};

// One column tile of plane i, column j (the lanes' levels).
__device__ __forceinline__ void velocity_column(const TopoArgs& a, const ColPos& c, int i, int j,
                                                float (&pre)[kVelPre][128]) {
  const int k = c.k;
  const Cell X(a, i, j, k);
  const int tid = threadIdx.y * 32 + threadIdx.x;
  {
    auto cp = [&](int slot, const float* f, int di, int dj) {
      cpa4(&pre[slot][tid], f + X.o + ((long long)di * X.S + dj * X.Y));
    };
    cp(kU, a.u1, 0, 0); cp(kV, a.v1, 0, 0); cp(kW, a.w1, 0, 0);
    cp(kR00, a.d1, 0, 0); cp(kR0m, a.d1, 0, -1); cp(kRm0, a.d1, -1, 0); cp(kRmm, a.d1, -1, -1);
    cp(kX11_0, a.xx, 0, 0); cp(kX11_m2, a.xx, -2, 0); cp(kX11_m1, a.xx, -1, 0);
    cp(kX11_p1, a.xx, 1, 0);
    cp(kY12_0, a.xy, 0, 0); cp(kY12_m2, a.xy, 0, -2); cp(kY12_m1, a.xy, 0, -1);
    cp(kY12_p1, a.xy, 0, 1); cp(kX12_m1, a.xy, -1, 0); cp(kX12_p1, a.xy, 1, 0);
    cp(kX12_p2, a.xy, 2, 0);
    cp(kX13_0, a.xz, 0, 0); cp(kX13_m1, a.xz, -1, 0); cp(kX13_p1, a.xz, 1, 0);
    cp(kX13_p2, a.xz, 2, 0);
    cp(kY22_0, a.yy, 0, 0); cp(kY22_m1, a.yy, 0, -1); cp(kY22_p1, a.yy, 0, 1);
    cp(kY22_p2, a.yy, 0, 2);
    cp(kY23_0, a.yz, 0, 0); cp(kY23_m2, a.yz, 0, -2); cp(kY23_m1, a.yz, 0, -1);
    cp(kY23_p1, a.yz, 0, 1);
    cp(kZ33, a.zz, 0, 0);
  }
  auto P = [&](int slot) { return pre[slot][tid]; };
  const float g3c = gk(a.g3_c, k), g3 = gk(a.g3, k), gc = gk(a.g_c, k), gg = gk(a.g, k);
  const float fc = X.fm(a.f_c, 0, 0), ff = X.fm(a.f, 0, 0), f1 = X.fm(a.f_1, 0, 0),
              f2 = X.fm(a.f_2, 0, 0);
  const float dcrj = __ldg(a.dcrjx + i + AWP_NGSL + 2) * __ldg(a.dcrjy + j + AWP_NGSL + 2) *
                     __ldg(a.dcrjz + k + AWP_ALIGN);
  cpa_wait();

  // density at the staggered velocity points (velocity_unroll.cu:140-152); the
  // k-1 values from the lane below
  const float r00 = P(kR00), r0m = P(kR0m), rm0 = P(kRm0), rmm = P(kRmm);
  const float r00k = __shfl_up_sync(kAll, r00, 1), r0mk = __shfl_up_sync(kAll, r0m, 1),
              rm0k = __shfl_up_sync(kAll, rm0, 1);
  const float rho1 = 0.25f * (r00k + r0mk) + 0.25f * (r00 + r0m);
  const float rho2 = 0.25f * (r00k + rm0k) + 0.25f * (r00 + rm0);
  const float rho3 = 0.25f * (r00 + rm0) + 0.25f * (r0m + rmm);
  const float Ai1 = quot(a.nu, f1 * g3c * rho1);
  const float Ai2 = quot(a.nu, f2 * g3c * rho2);
  const float Ai3 = quot(a.nu, fc * g3 * rho3);

  // --- u1 -------------------------------------------------------------------
  float s1 = -kD1 * fc * g3c * P(kX11_0) + kD0 * X.fm(a.f_c, -2, 0) * g3c * P(kX11_m2) +
             kD1 * X.fm(a.f_c, -1, 0) * g3c * P(kX11_m1) -
             kD0 * X.fm(a.f_c, 1, 0) * g3c * P(kX11_p1);
  s1 += -kD1 * ff * g3c * P(kY12_0) + kD0 * X.fm(a.f, 0, -2) * g3c * P(kY12_m2) +
        kD1 * X.fm(a.f, 0, -1) * g3c * P(kY12_m1) - kD0 * X.fm(a.f, 0, 1) * g3c * P(kY12_p1);
  s1 += zd4(P(kX13_0), c, true, kTopoVelDhz4r);
  {
    const float px =
        gc * (kP1 * P(kX11_0) + kP0 * P(kX11_m2) + kP1 * P(kX11_m1) + kP0 * P(kX11_p1));
    const float py =
        gc * (kP1 * P(kY12_0) + kP0 * P(kY12_m2) + kP1 * P(kY12_m1) + kP0 * P(kY12_p1));
    s1 = s1 - X.fm(a.f1_1, 0, 0) * zd7(px, c, kTopoVelDhpz4r);
    s1 = s1 - X.fm(a.f2_1, 0, 0) * zd7(py, c, kTopoVelDhpz4r);
  }
  // --- u2 -------------------------------------------------------------------
  float s2 = zd4(P(kY23_0), c, true, kTopoVelDhz4r);
  s2 += kD1 * ff * g3c * P(kY12_0) + kD0 * X.fm(a.f, -1, 0) * g3c * P(kX12_m1) -
        kD1 * X.fm(a.f, 1, 0) * g3c * P(kX12_p1) - kD0 * X.fm(a.f, 2, 0) * g3c * P(kX12_p2);
  s2 += kD1 * fc * g3c * P(kY22_0) + kD0 * X.fm(a.f_c, 0, -1) * g3c * P(kY22_m1) -
        kD1 * X.fm(a.f_c, 0, 1) * g3c * P(kY22_p1) -
        kD0 * X.fm(a.f_c, 0, 2) * g3c * P(kY22_p2);
  {
    const float px =
        gc * (kP1 * P(kY12_0) + kP0 * P(kX12_m1) + kP1 * P(kX12_p1) + kP0 * P(kX12_p2));
    const float py =
        gc * (kP1 * P(kY22_0) + kP0 * P(kY22_m1) + kP1 * P(kY22_p1) + kP0 * P(kY22_p2));
    s2 = s2 - X.fm(a.f1_2, 0, 0) * zd7(px, c, kTopoVelDhpz4r);
    s2 = s2 - X.fm(a.f2_2, 0, 0) * zd7(py, c, kTopoVelDhpz4r);
  }
  // --- u3 -------------------------------------------------------------------
  float s3 = -kD1 * f2 * g3 * P(kY23_0) + kD0 * X.fm(a.f_2, 0, -2) * g3 * P(kY23_m2) +
             kD1 * X.fm(a.f_2, 0, -1) * g3 * P(kY23_m1) -
             kD0 * X.fm(a.f_2, 0, 1) * g3 * P(kY23_p1);
  s3 += kD1 * f1 * g3 * P(kX13_0) + kD0 * X.fm(a.f_1, -1, 0) * g3 * P(kX13_m1) -
        kD1 * X.fm(a.f_1, 1, 0) * g3 * P(kX13_p1) - kD0 * X.fm(a.f_1, 2, 0) * g3 * P(kX13_p2);
  s3 += zd4(P(kZ33), c, false, kTopoVelDz4r);
  {
    const float px =
        gg * (kP1 * P(kX13_0) + kP0 * P(kX13_m1) + kP1 * P(kX13_p1) + kP0 * P(kX13_p2));
    const float py =
        gg * (kP1 * P(kY23_0) + kP0 * P(kY23_m2) + kP1 * P(kY23_m1) + kP0 * P(kY23_p1));
    s3 = s3 - X.fm(a.f1_c, 0, 0) * zd7(px, c, kTopoVelDphz4r);
    s3 = s3 - X.fm(a.f2_c, 0, 0) * zd7(py, c, kTopoVelDphz4r);
  }

  if (!c.out) return;
  const long long o = X.o;
  a.u1[o] = (P(kU) + Ai1 * s1) * dcrj;
  a.v1[o] = (P(kV) + Ai2 * s2) * dcrj;
  a.w1[o] = (P(kW) + Ai3 * s3) * dcrj;
}

// A CTA takes four columns of AWP_TOPO_MARCH consecutive x planes, one plane
// after another, so that the x-neighbour reads of a plane find the previous
// planes' values in L1.
__global__ void __launch_bounds__(128, AWP_TOPO_VEL_MINB) k_topo_velocity(const TopoArgs a) {
  const ColPos c(a.nz, blockIdx.x);
  const int j = blockIdx.y * 4 + threadIdx.y;
  if (j >= a.ny) return;  // whole warps
  __shared__ float pre[kVelPre][128];
  const int i0 = blockIdx.z * AWP_TOPO_MARCH, i1 = min(i0 + AWP_TOPO_MARCH, a.nx);
#pragma unroll 1
  for (int i = i0; i < i1; ++i) velocity_column(a, c, i, j, pre);
}

// ===========================================================================
// Stress and memory variables
// ===========================================================================
// A stress thread stages the stresses and memory variables of its cell by
// cp.async at its start (read only by the update at its end); the velocity
// stencil and the media are read where they are used, through L1.
template <bool ELASTIC>
struct StrStage {
  static constexpr int kRows = ELASTIC ? 6 : 12;
};

template <bool ELASTIC>
__device__ __forceinline__ void stress_column(const TopoArgs& a, const ColPos& c, int i, int j,
                                              float (&pre)[StrStage<ELASTIC>::kRows][128]) {
  const int k = c.k, r = c.r;
  const Cell X(a, i, j, k);
  const int S1 = a.slice, Y1 = a.yline;
  const long long o = X.o;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  float* const SG[6] = {a.xx, a.yy, a.zz, a.xy, a.xz, a.yz};
  float* const RR[6] = {a.r1, a.r2, a.r3, a.r4, a.r5, a.r6};
#pragma unroll
  for (int q = 0; q < 6; ++q) cpa4(&pre[q][tid], SG[q] + o);
  if (!ELASTIC) {
#pragma unroll
    for (int q = 0; q < 6; ++q) cpa4(&pre[6 + q][tid], RR[q] + o);
  }
  // the 21 velocity stencil points: (field, di, dj)
  constexpr signed char kStencil[21][3] = {
      {0, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 2, 0}, {0, 0, -1}, {0, 0, 1}, {0, 0, 2},
      {1, 0, 0}, {1, 0, -2}, {1, 0, -1}, {1, 0, 1}, {1, -2, 0}, {1, -1, 0}, {1, 1, 0},
      {2, 0, 0}, {2, -2, 0}, {2, -1, 0}, {2, 1, 0}, {2, 0, -1}, {2, 0, 1}, {2, 0, 2}};
  const float* const V[3] = {a.u1, a.v1, a.w1};
  auto P = [&](int n) {
    return __ldg(V[kStencil[n][0]] + o + (kStencil[n][1] * S1 + kStencil[n][2] * Y1));
  };
  const float gc = gk(a.g_c, k), g = gk(a.g, k);

  // every vertical difference of a horizontal interpolant is one difference
  // of the interpolated column (the metric weights do not depend on k)
  float d[9];
  // ---- normal components: Jii = 1 / (f_c g3_c) (stress_attenuation.cu:340-431)
  const float Jii = inv(X.fm(a.f_c, 0, 0) * gk(a.g3_c, k));
  const float u_0 = P(0), u_xm1 = P(1), u_xp1 = P(2),
              u_xp2 = P(3);
  const float v_0 = P(7), v_ym2 = P(8), v_ym1 = P(9),
              v_yp1 = P(10);
  const float w_0 = P(14);
  {
    const float iu = kP0 * X.fm(a.f1_1, -1, 0) * u_xm1 + kP1 * X.fm(a.f1_1, 0, 0) * u_0 +
                     kP1 * X.fm(a.f1_1, 1, 0) * u_xp1 + kP0 * X.fm(a.f1_1, 2, 0) * u_xp2;
    d[0] = kD1 * u_0 + kD0 * u_xm1 - kD1 * u_xp1 - kD0 * u_xp2 -
           Jii * gc * zd7(iu, c, kTopoStrPhdz4r);
    const float iv = kP1 * X.fm(a.f2_2, 0, 0) * v_0 + kP0 * X.fm(a.f2_2, 0, -2) * v_ym2 +
                     kP1 * X.fm(a.f2_2, 0, -1) * v_ym1 + kP0 * X.fm(a.f2_2, 0, 1) * v_yp1;
    d[1] = -kD1 * v_0 + kD0 * v_ym2 + kD1 * v_ym1 - kD0 * v_yp1 -
           Jii * gc * zd7(iv, c, kTopoStrPhdz4r);
    d[2] = Jii * zd4(w_0, c, true, kTopoStrDhz4r);
  }
  // ---- xy: J12i = 1 / (f g3_c); the interior rows read g3_c six points
  // higher (stress_attenuation.cu:471), the boundary rows at k (:1149)
  {
    const float J12i = inv(X.fm(a.f, 0, 0) * gk(a.g3_c, r < 0 ? k + 6 : k));
    const float u_ym1 = P(4), u_yp1 = P(5), u_yp2 = P(6);
    const float iu = kP1 * X.fm(a.f2_1, 0, 0) * u_0 + kP0 * X.fm(a.f2_1, 0, -1) * u_ym1 +
                     kP1 * X.fm(a.f2_1, 0, 1) * u_yp1 + kP0 * X.fm(a.f2_1, 0, 2) * u_yp2;
    d[3] = kD1 * u_0 + kD0 * u_ym1 - kD1 * u_yp1 - kD0 * u_yp2 -
           J12i * gc * zd7(iu, c, kTopoStrPhdz4r);
    const float v_xm2 = P(11), v_xm1 = P(12), v_xp1 = P(13);
    const float iv = kP1 * X.fm(a.f1_2, 0, 0) * v_0 + kP0 * X.fm(a.f1_2, -2, 0) * v_xm2 +
                     kP1 * X.fm(a.f1_2, -1, 0) * v_xm1 + kP0 * X.fm(a.f1_2, 1, 0) * v_xp1;
    d[4] = -kD1 * v_0 + kD0 * v_xm2 + kD1 * v_xm1 - kD0 * v_xp1 -
           J12i * gc * zd7(iv, c, kTopoStrPhdz4r);
  }
  // ---- xz: J13i = 1 / (f_1 g3) (:550-598, :1254-1317)
  {
    const float J13i = inv(X.fm(a.f_1, 0, 0) * gk(a.g3, k));
    d[5] = J13i * zd4(u_0, c, false, kTopoStrDz4r);
    const float w_xm2 = P(15), w_xm1 = P(16), w_xp1 = P(17);
    const float iw = kP1 * X.fm(a.f1_c, 0, 0) * w_0 + kP0 * X.fm(a.f1_c, -2, 0) * w_xm2 +
                     kP1 * X.fm(a.f1_c, -1, 0) * w_xm1 + kP0 * X.fm(a.f1_c, 1, 0) * w_xp1;
    d[6] = -kD1 * w_0 + kD0 * w_xm2 + kD1 * w_xm1 - kD0 * w_xp1 -
           J13i * g * zd7(iw, c, kTopoStrPdhz4r);
  }
  // ---- yz: J23i = 1 / (f_2 g3) (:600-650, :1319-1380)
  {
    const float J23i = inv(X.fm(a.f_2, 0, 0) * gk(a.g3, k));
    d[7] = J23i * zd4(v_0, c, false, kTopoStrDz4r);
    const float w_ym1 = P(18), w_yp1 = P(19), w_yp2 = P(20);
    const float iw = kP1 * X.fm(a.f2_c, 0, 0) * w_0 + kP0 * X.fm(a.f2_c, 0, -1) * w_ym1 +
                     kP1 * X.fm(a.f2_c, 0, 1) * w_yp1 + kP0 * X.fm(a.f2_c, 0, 2) * w_yp2;
    d[8] = kD1 * w_0 + kD0 * w_ym1 - kD1 * w_yp1 - kD0 * w_yp2 -
           J23i * g * zd7(iw, c, kTopoStrPdhz4r);
  }

  // ---- material coefficients and the update (as the Cartesian dstrqc); the
  // k-1 neighbours of the eight-cell sums from the lane below
  const float* const MT[4] = {a.lam, a.mu, a.qp, a.qs};
  const long long corner[4] = {o, o + S1, o - Y1, o + S1 - Y1};
  auto mat = [&](int m, int q) { return __ldg(MT[m] + corner[q]); };
  auto sum8 = [&](int m) {
    const float q0 = mat(m, 0), q1 = mat(m, 1), q2 = mat(m, 2), q3 = mat(m, 3);
    return q0 + q1 + q2 + q3 + __shfl_up_sync(kAll, q0, 1) + __shfl_up_sync(kAll, q1, 1) +
           __shfl_up_sync(kAll, q2, 1) + __shfl_up_sync(kAll, q3, 1);
  };
  const float L8 = sum8(0), M8 = sum8(1);
  const float QP8 = ELASTIC ? 0.f : sum8(2), QS8 = ELASTIC ? 0.f : sum8(3);
  const float mu0 = mat(1, 0), muk = __shfl_up_sync(kAll, mu0, 1);
  const float qs0 = ELASTIC ? 0.f : mat(3, 0);
  const float qsk = __shfl_up_sync(kAll, qs0, 1);
  cpa_wait();
  if (!c.out) return;
  const int ia = i + AWP_NGSL + 2, ja = j + AWP_NGSL + 2, ka = k + AWP_ALIGN;
  const int t = awp_tex_index(a.tex, ia, ja, ka);
  const float f_vx1 = a.tex.tau1[t], f_vx2 = a.tex.tau2[t], f_wwo = a.tex.wwo8[t];
  const float cc0 = ELASTIC ? 0.f : a.coeff[2 * t], cc1 = ELASTIC ? 0.f : a.coeff[2 * t + 1];
  const AwpStrCoef cf = awp_stress_coef<ELASTIC>(
      L8, M8, mu0, muk, mat(1, 2), mat(1, 1), QP8, QS8, qs0, qsk,
      ELASTIC ? 0.f : mat(3, 2), ELASTIC ? 0.f : mat(3, 1), f_vx1, f_vx2,
      f_wwo, cc0, cc1, a.qthr, a.dth, a.dh1, a.DT);
  const float dcrj = __ldg(a.dcrjx + ia) * __ldg(a.dcrjy + ja) * __ldg(a.dcrjz + ka);
  float sg[6], rr[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    sg[q] = pre[q][tid];
    rr[q] = ELASTIC ? 0.f : pre[6 + q][tid];
  }
  awp_stress_update<ELASTIC>(sg, rr, cf, f_vx1, f_vx2, f_wwo, a.DT, dcrj, d);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    SG[q][o] = sg[q];
    if (!ELASTIC) RR[q][o] = rr[q];
  }
}

template <bool ELASTIC>
__global__ void __launch_bounds__(128, AWP_TOPO_STR_MINB) k_topo_stress(const TopoArgs a) {
  const ColPos c(a.nz, blockIdx.x);
  const int j = a.s_j + blockIdx.y * 4 + threadIdx.y;
  if (j >= a.e_j) return;  // whole warps
  __shared__ float pre[StrStage<ELASTIC>::kRows][128];
  const int i0 = a.s_i + blockIdx.z * AWP_TOPO_MARCH, i1 = min(i0 + AWP_TOPO_MARCH, a.e_i);
#pragma unroll 1
  for (int i = i0; i < i1; ++i) stress_column<ELASTIC>(a, c, i, j, pre);
}

// Tiles of a column: the top one, then one per 26 levels below it until a
// tile reaches level 0.
static unsigned column_tiles(int nz) {
  return 1u + (nz > 32 ? (unsigned)((nz - 32 + kTileOut - 1) / kTileOut) : 0u);
}

cudaError_t awp_launch_topo_velocity(const TopoArgs& a, cudaStream_t st) {
  if (a.nz < 12 || a.nx < 1 || a.ny < 1) return cudaErrorInvalidValue;
  const dim3 block(32, 4, 1);
  const dim3 grid(column_tiles(a.nz), (a.ny + 3) / 4,
                  (a.nx + AWP_TOPO_MARCH - 1) / AWP_TOPO_MARCH);
  k_topo_velocity<<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_topo_stress(const TopoArgs& a, bool elastic, cudaStream_t st) {
  if (a.nz < 12) return cudaErrorInvalidValue;
  if (a.e_i <= a.s_i || a.e_j <= a.s_j) return cudaSuccess;
  const dim3 block(32, 4, 1);
  const dim3 grid(column_tiles(a.nz), (a.e_j - a.s_j + 3) / 4,
                  (a.e_i - a.s_i + AWP_TOPO_MARCH - 1) / AWP_TOPO_MARCH);
  if (elastic)
    k_topo_stress<true><<<grid, block, 0, st>>>(a);
  else
    k_topo_stress<false><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}
