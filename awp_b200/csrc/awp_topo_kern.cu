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
__device__ __forceinline__ float inv(float x) { return (float)(1.0 / (double)x); }

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

// 7-point vertical difference at the lane's level of a value v(k) held one
// level per lane (interior coefficients), or boundary row r of T in the top
// tile.  Summation order as the reference's operators.
template <int NT>
__device__ __forceinline__ float zd7(float v, const ColPos& c, const float (&T)[6][NT]) {
  const float m3 = __shfl_up_sync(kAll, v, 3), m2 = __shfl_up_sync(kAll, v, 2),
              m1 = __shfl_up_sync(kAll, v, 1), p1 = __shfl_down_sync(kAll, v, 1),
              p2 = __shfl_down_sync(kAll, v, 2), p3 = __shfl_down_sync(kAll, v, 3);
  float s = kZ0 * m3 + kZ1 * m2 + kZ2 * m1 - kZ2 * p1 - kZ1 * p2 - kZ0 * p3;
  if (c.top) {  // warp-uniform: the closure rows of the top six levels
    const int rr = c.r < 0 ? 0 : c.r;
    float b = 0.f;
#pragma unroll
    for (int m = NT - 1; m >= 0; --m) b += T[rr][m] * __shfl_sync(kAll, v, 31 - m);
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
    const int rr = c.r < 0 ? 0 : c.r;
    float b = 0.f;
#pragma unroll
    for (int m = NT - 1; m >= 0; --m) b += T[rr][m] * __shfl_sync(kAll, v, 31 - m);
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
  // 3-D field at (i+di, j+dj, k); 2-D metric at (i+di, j+dj)
  __device__ __forceinline__ float at(const float* __restrict__ s, int di, int dj) const {
    return __ldg(s + o + (di * S + dj * Y));
  }
  __device__ __forceinline__ float fm(const float* __restrict__ f, int di, int dj) const {
    return __ldg(f + of + (di * F + dj));
  }
};

}  // namespace

// ===========================================================================
// Velocity
// ===========================================================================
__global__ void __launch_bounds__(128) k_topo_velocity(const TopoArgs a) {
  const ColPos c(a.nz, blockIdx.x);
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= a.ny || i >= a.nx) return;  // whole warps
  const int k = c.k;
  const Cell X(a, i, j, k);
  const float *__restrict__ s11 = a.xx, *__restrict__ s12 = a.xy, *__restrict__ s13 = a.xz,
              *__restrict__ s22 = a.yy, *__restrict__ s23 = a.yz, *__restrict__ s33 = a.zz;

  // density at the staggered velocity points (velocity_unroll.cu:140-152); the
  // k-1 values from the lane below
  const float r00 = X.at(a.d1, 0, 0), r0m = X.at(a.d1, 0, -1), rm0 = X.at(a.d1, -1, 0),
              rmm = X.at(a.d1, -1, -1);
  const float r00k = __shfl_up_sync(kAll, r00, 1), r0mk = __shfl_up_sync(kAll, r0m, 1),
              rm0k = __shfl_up_sync(kAll, rm0, 1);
  const float rho1 = 0.25f * (r00k + r0mk) + 0.25f * (r00 + r0m);
  const float rho2 = 0.25f * (r00k + rm0k) + 0.25f * (r00 + rm0);
  const float rho3 = 0.25f * (r00 + rm0) + 0.25f * (r0m + rmm);
  const float g3c = gk(a.g3_c, k), g3 = gk(a.g3, k), gc = gk(a.g_c, k), gg = gk(a.g, k);
  const float fc = X.fm(a.f_c, 0, 0);
  const float Ai1 = (float)((double)a.nu / (double)(X.fm(a.f_1, 0, 0) * g3c * rho1));
  const float Ai2 = (float)((double)a.nu / (double)(X.fm(a.f_2, 0, 0) * g3c * rho2));
  const float Ai3 = (float)((double)a.nu / (double)(fc * g3 * rho3));
  const float dcrj = __ldg(a.dcrjx + i + AWP_NGSL + 2) * __ldg(a.dcrjy + j + AWP_NGSL + 2) *
                     __ldg(a.dcrjz + k + AWP_ALIGN);

  // --- u1 -------------------------------------------------------------------
  const float x11_0 = X.at(s11, 0, 0), x11_m2 = X.at(s11, -2, 0), x11_m1 = X.at(s11, -1, 0),
              x11_p1 = X.at(s11, 1, 0);
  const float y12_0 = X.at(s12, 0, 0), y12_m2 = X.at(s12, 0, -2), y12_m1 = X.at(s12, 0, -1),
              y12_p1 = X.at(s12, 0, 1);
  float s1 = -kD1 * fc * g3c * x11_0 + kD0 * X.fm(a.f_c, -2, 0) * g3c * x11_m2 +
             kD1 * X.fm(a.f_c, -1, 0) * g3c * x11_m1 - kD0 * X.fm(a.f_c, 1, 0) * g3c * x11_p1;
  const float ff = X.fm(a.f, 0, 0);
  s1 += -kD1 * ff * g3c * y12_0 + kD0 * X.fm(a.f, 0, -2) * g3c * y12_m2 +
        kD1 * X.fm(a.f, 0, -1) * g3c * y12_m1 - kD0 * X.fm(a.f, 0, 1) * g3c * y12_p1;
  const float x13_0 = X.at(s13, 0, 0);
  s1 += zd4(x13_0, c, true, kTopoVelDhz4r);
  {
    const float px = gc * (kP1 * x11_0 + kP0 * x11_m2 + kP1 * x11_m1 + kP0 * x11_p1);
    const float py = gc * (kP1 * y12_0 + kP0 * y12_m2 + kP1 * y12_m1 + kP0 * y12_p1);
    s1 = s1 - X.fm(a.f1_1, 0, 0) * zd7(px, c, kTopoVelDhpz4r);
    s1 = s1 - X.fm(a.f2_1, 0, 0) * zd7(py, c, kTopoVelDhpz4r);
  }
  // --- u2 -------------------------------------------------------------------
  const float x23_0 = X.at(s23, 0, 0);
  float s2 = zd4(x23_0, c, true, kTopoVelDhz4r);
  const float x12_m1 = X.at(s12, -1, 0), x12_p1 = X.at(s12, 1, 0), x12_p2 = X.at(s12, 2, 0);
  s2 += kD1 * ff * g3c * y12_0 + kD0 * X.fm(a.f, -1, 0) * g3c * x12_m1 -
        kD1 * X.fm(a.f, 1, 0) * g3c * x12_p1 - kD0 * X.fm(a.f, 2, 0) * g3c * x12_p2;
  const float y22_0 = X.at(s22, 0, 0), y22_m1 = X.at(s22, 0, -1), y22_p1 = X.at(s22, 0, 1),
              y22_p2 = X.at(s22, 0, 2);
  s2 += kD1 * fc * g3c * y22_0 + kD0 * X.fm(a.f_c, 0, -1) * g3c * y22_m1 -
        kD1 * X.fm(a.f_c, 0, 1) * g3c * y22_p1 - kD0 * X.fm(a.f_c, 0, 2) * g3c * y22_p2;
  {
    const float px = gc * (kP1 * y12_0 + kP0 * x12_m1 + kP1 * x12_p1 + kP0 * x12_p2);
    const float py = gc * (kP1 * y22_0 + kP0 * y22_m1 + kP1 * y22_p1 + kP0 * y22_p2);
    s2 = s2 - X.fm(a.f1_2, 0, 0) * zd7(px, c, kTopoVelDhpz4r);
    s2 = s2 - X.fm(a.f2_2, 0, 0) * zd7(py, c, kTopoVelDhpz4r);
  }
  // --- u3 -------------------------------------------------------------------
  const float f2 = X.fm(a.f_2, 0, 0), f1 = X.fm(a.f_1, 0, 0);
  const float y23_m2 = X.at(s23, 0, -2), y23_m1 = X.at(s23, 0, -1), y23_p1 = X.at(s23, 0, 1);
  float s3 = -kD1 * f2 * g3 * x23_0 + kD0 * X.fm(a.f_2, 0, -2) * g3 * y23_m2 +
             kD1 * X.fm(a.f_2, 0, -1) * g3 * y23_m1 - kD0 * X.fm(a.f_2, 0, 1) * g3 * y23_p1;
  const float x13_m1 = X.at(s13, -1, 0), x13_p1 = X.at(s13, 1, 0), x13_p2 = X.at(s13, 2, 0);
  s3 += kD1 * f1 * g3 * x13_0 + kD0 * X.fm(a.f_1, -1, 0) * g3 * x13_m1 -
        kD1 * X.fm(a.f_1, 1, 0) * g3 * x13_p1 - kD0 * X.fm(a.f_1, 2, 0) * g3 * x13_p2;
  s3 += zd4(X.at(s33, 0, 0), c, false, kTopoVelDz4r);
  {
    const float px = gg * (kP1 * x13_0 + kP0 * x13_m1 + kP1 * x13_p1 + kP0 * x13_p2);
    const float py = gg * (kP1 * x23_0 + kP0 * y23_m2 + kP1 * y23_m1 + kP0 * y23_p1);
    s3 = s3 - X.fm(a.f1_c, 0, 0) * zd7(px, c, kTopoVelDphz4r);
    s3 = s3 - X.fm(a.f2_c, 0, 0) * zd7(py, c, kTopoVelDphz4r);
  }

  if (!c.out) return;
  const long long o = X.o;
  a.u1[o] = (a.u1[o] + Ai1 * s1) * dcrj;
  a.v1[o] = (a.v1[o] + Ai2 * s2) * dcrj;
  a.w1[o] = (a.w1[o] + Ai3 * s3) * dcrj;
}

// ===========================================================================
// Stress and memory variables
// ===========================================================================
template <bool ELASTIC>
__global__ void __launch_bounds__(128) k_topo_stress(const TopoArgs a) {
  const ColPos c(a.nz, blockIdx.x);
  const int j = a.s_j + blockIdx.y * 4 + threadIdx.y;
  const int i = a.s_i + blockIdx.z;
  if (j >= a.e_j || i >= a.e_i) return;  // whole warps
  const int k = c.k, r = c.r;
  const Cell X(a, i, j, k);
  const float *__restrict__ u1 = a.u1, *__restrict__ v1 = a.v1, *__restrict__ w1 = a.w1;
  const float gc = gk(a.g_c, k), g = gk(a.g, k);

  // every vertical difference of a horizontal interpolant is one difference
  // of the interpolated column (the metric weights do not depend on k)
  float d[9];
  // ---- normal components: Jii = 1 / (f_c g3_c) (stress_attenuation.cu:340-431)
  const float Jii = inv(X.fm(a.f_c, 0, 0) * gk(a.g3_c, k));
  const float u_0 = X.at(u1, 0, 0), u_xm1 = X.at(u1, -1, 0), u_xp1 = X.at(u1, 1, 0),
              u_xp2 = X.at(u1, 2, 0);
  const float v_0 = X.at(v1, 0, 0), v_ym2 = X.at(v1, 0, -2), v_ym1 = X.at(v1, 0, -1),
              v_yp1 = X.at(v1, 0, 1);
  const float w_0 = X.at(w1, 0, 0);
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
    const float u_ym1 = X.at(u1, 0, -1), u_yp1 = X.at(u1, 0, 1), u_yp2 = X.at(u1, 0, 2);
    const float iu = kP1 * X.fm(a.f2_1, 0, 0) * u_0 + kP0 * X.fm(a.f2_1, 0, -1) * u_ym1 +
                     kP1 * X.fm(a.f2_1, 0, 1) * u_yp1 + kP0 * X.fm(a.f2_1, 0, 2) * u_yp2;
    d[3] = kD1 * u_0 + kD0 * u_ym1 - kD1 * u_yp1 - kD0 * u_yp2 -
           J12i * gc * zd7(iu, c, kTopoStrPhdz4r);
    const float v_xm2 = X.at(v1, -2, 0), v_xm1 = X.at(v1, -1, 0), v_xp1 = X.at(v1, 1, 0);
    const float iv = kP1 * X.fm(a.f1_2, 0, 0) * v_0 + kP0 * X.fm(a.f1_2, -2, 0) * v_xm2 +
                     kP1 * X.fm(a.f1_2, -1, 0) * v_xm1 + kP0 * X.fm(a.f1_2, 1, 0) * v_xp1;
    d[4] = -kD1 * v_0 + kD0 * v_xm2 + kD1 * v_xm1 - kD0 * v_xp1 -
           J12i * gc * zd7(iv, c, kTopoStrPhdz4r);
  }
  // ---- xz: J13i = 1 / (f_1 g3) (:550-598, :1254-1317)
  {
    const float J13i = inv(X.fm(a.f_1, 0, 0) * gk(a.g3, k));
    d[5] = J13i * zd4(u_0, c, false, kTopoStrDz4r);
    const float w_xm2 = X.at(w1, -2, 0), w_xm1 = X.at(w1, -1, 0), w_xp1 = X.at(w1, 1, 0);
    const float iw = kP1 * X.fm(a.f1_c, 0, 0) * w_0 + kP0 * X.fm(a.f1_c, -2, 0) * w_xm2 +
                     kP1 * X.fm(a.f1_c, -1, 0) * w_xm1 + kP0 * X.fm(a.f1_c, 1, 0) * w_xp1;
    d[6] = -kD1 * w_0 + kD0 * w_xm2 + kD1 * w_xm1 - kD0 * w_xp1 -
           J13i * g * zd7(iw, c, kTopoStrPdhz4r);
  }
  // ---- yz: J23i = 1 / (f_2 g3) (:600-650, :1319-1380)
  {
    const float J23i = inv(X.fm(a.f_2, 0, 0) * gk(a.g3, k));
    d[7] = J23i * zd4(v_0, c, false, kTopoStrDz4r);
    const float w_ym1 = X.at(w1, 0, -1), w_yp1 = X.at(w1, 0, 1), w_yp2 = X.at(w1, 0, 2);
    const float iw = kP1 * X.fm(a.f2_c, 0, 0) * w_0 + kP0 * X.fm(a.f2_c, 0, -1) * w_ym1 +
                     kP1 * X.fm(a.f2_c, 0, 1) * w_yp1 + kP0 * X.fm(a.f2_c, 0, 2) * w_yp2;
    d[8] = kD1 * w_0 + kD0 * w_ym1 - kD1 * w_yp1 - kD0 * w_yp2 -
           J23i * g * zd7(iw, c, kTopoStrPdhz4r);
  }

  // ---- material coefficients and the update (as the Cartesian dstrqc); the
  // k-1 neighbours of the eight-cell sums from the lane below
  const int S1 = a.slice, Y1 = a.yline;
  const long long o = X.o;
  auto sum8 = [&](const float* __restrict__ m) {
    const float q0 = __ldg(m + o), q1 = __ldg(m + o + S1), q2 = __ldg(m + o - Y1),
                q3 = __ldg(m + o + S1 - Y1);
    return q0 + q1 + q2 + q3 + __shfl_up_sync(kAll, q0, 1) + __shfl_up_sync(kAll, q1, 1) +
           __shfl_up_sync(kAll, q2, 1) + __shfl_up_sync(kAll, q3, 1);
  };
  const float L8 = sum8(a.lam), M8 = sum8(a.mu);
  const float QP8 = ELASTIC ? 0.f : sum8(a.qp), QS8 = ELASTIC ? 0.f : sum8(a.qs);
  const float mu0 = __ldg(a.mu + o), muk = __shfl_up_sync(kAll, mu0, 1);
  const float qs0 = ELASTIC ? 0.f : __ldg(a.qs + o);
  const float qsk = __shfl_up_sync(kAll, qs0, 1);
  if (!c.out) return;
  const int ia = i + AWP_NGSL + 2, ja = j + AWP_NGSL + 2, ka = k + AWP_ALIGN;
  const int t = awp_tex_index(a.tex, ia, ja, ka);
  const float f_vx1 = a.tex.tau1[t], f_vx2 = a.tex.tau2[t], f_wwo = a.tex.wwo8[t];
  const float cc0 = ELASTIC ? 0.f : a.coeff[2 * t], cc1 = ELASTIC ? 0.f : a.coeff[2 * t + 1];
  const AwpStrCoef cf = awp_stress_coef<ELASTIC>(
      L8, M8, mu0, muk, __ldg(a.mu + o - Y1), __ldg(a.mu + o + S1), QP8, QS8, qs0, qsk,
      ELASTIC ? 0.f : __ldg(a.qs + o - Y1), ELASTIC ? 0.f : __ldg(a.qs + o + S1), f_vx1, f_vx2,
      f_wwo, cc0, cc1, a.qthr, a.dth, a.dh1, a.DT);
  const float dcrj = __ldg(a.dcrjx + ia) * __ldg(a.dcrjy + ja) * __ldg(a.dcrjz + ka);
  float* const SG[6] = {a.xx, a.yy, a.zz, a.xy, a.xz, a.yz};
  float* const RR[6] = {a.r1, a.r2, a.r3, a.r4, a.r5, a.r6};
  float sg[6], rr[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    sg[q] = SG[q][o];
    rr[q] = ELASTIC ? 0.f : RR[q][o];
  }
  awp_stress_update<ELASTIC>(sg, rr, cf, f_vx1, f_vx2, f_wwo, a.DT, dcrj, d);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    SG[q][o] = sg[q];
    if (!ELASTIC) RR[q][o] = rr[q];
  }
}

// Tiles of a column: the top one, then one per 26 levels below it until a
// tile reaches level 0.
static unsigned column_tiles(int nz) {
  return 1u + (nz > 32 ? (unsigned)((nz - 32 + kTileOut - 1) / kTileOut) : 0u);
}

cudaError_t awp_launch_topo_velocity(const TopoArgs& a, cudaStream_t st) {
  if (a.nz < 12 || a.nx < 1 || a.ny < 1) return cudaErrorInvalidValue;
  const dim3 block(32, 4, 1);
  const dim3 grid(column_tiles(a.nz), (a.ny + 3) / 4, a.nx);
  k_topo_velocity<<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_topo_stress(const TopoArgs& a, bool elastic, cudaStream_t st) {
  if (a.nz < 12) return cudaErrorInvalidValue;
  if (a.e_i <= a.s_i || a.e_j <= a.s_j) return cudaSuccess;
  const dim3 block(32, 4, 1);
  const dim3 grid(column_tiles(a.nz), (a.e_j - a.s_j + 3) / 4, a.e_i - a.s_i);
  if (elastic)
    k_topo_stress<true><<<grid, block, 0, st>>>(a);
  else
    k_topo_stress<false><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}
