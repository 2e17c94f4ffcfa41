// Curvilinear (topography) velocity and stress half-steps of the top grid.
//
// The reference spells these operators out as generated code, one kernel for
// the interior (k below the top six points) and one for the six boundary rows
// next to the free surface:
//   velocity: dtopo_vel_111_unroll (kernels/velocity_unroll.cu:1-428) and
//             dtopo_vel_112 (kernels/optimized_velocity.cu:1040-1629),
//   stress:   dtopo_str_111 / dtopo_str_112 (kernels/stress_attenuation.cu:73-1415),
// launched by topo_velocity_*_H (velocity.cu) and topo_stress_*_H
// (stress_attenuation.cu).  Here each half-step is one kernel: a thread owns
// one (i, j, k) cell, k fastest across the warp for coalesced loads, and the
// vertical operators switch between the interior stencil and the boundary
// closure row r = nz-1-k (tables in awp_topo_tables.h) per thread.
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

struct Idx {
  int slice, yline, fld;
  __device__ __forceinline__ long long p(int i, int j, int k) const {
    return (long long)(i + AWP_NGSL + 2) * slice + (long long)(j + AWP_NGSL + 2) * yline +
           (k + AWP_ALIGN);
  }
  __device__ __forceinline__ long long f(int i, int j) const {
    return (long long)(i + AWP_NGSL + 2) * fld + (j + AWP_NGSL + 2 + AWP_ALIGN);
  }
};

__device__ __forceinline__ float ld(const float* __restrict__ a, long long o) { return __ldg(a + o); }
__device__ __forceinline__ float gk(const float* __restrict__ g, int k) {
  return __ldg(g + k + AWP_ALIGN);
}
__device__ __forceinline__ float inv(float x) { return (float)(1.0 / (double)x); }

// 7-point vertical difference at k (interior: c[n] at k-3+n, the centre
// weight is zero) or boundary row r (T[r][m] at nz-1-m, m = NT-1 .. 0).
template <int NT, class Fn>
__device__ __forceinline__ float zdiff7(int k, int r, int nz, const float (&T)[6][NT], Fn v) {
  if (r < 0)
    return kZ0 * v(k - 3) + kZ1 * v(k - 2) + kZ2 * v(k - 1) - kZ2 * v(k + 1) - kZ1 * v(k + 2) -
           kZ0 * v(k + 3);
  float s = 0.f;
#pragma unroll
  for (int m = NT - 1; m >= 0; --m) s += T[r][m] * v(nz - 1 - m);
  return s;
}

// 4-point vertical difference: half-point form (dhz4: k-2..k+1) or node form
// (dz4: k-1..k+2), or the boundary row.
template <int NT, class Fn>
__device__ __forceinline__ float zdiff4(int k, int r, int nz, bool half, const float (&T)[6][NT],
                                        Fn v) {
  if (r < 0) {
    const int b = half ? k - 2 : k - 1;
    return kD0 * v(b) + kD1 * v(b + 1) - kD1 * v(b + 2) - kD0 * v(b + 3);
  }
  float s = 0.f;
#pragma unroll
  for (int m = NT - 1; m >= 0; --m) s += T[r][m] * v(nz - 1 - m);
  return s;
}

}  // namespace

// ===========================================================================
// Velocity
// ===========================================================================
__global__ void __launch_bounds__(128) k_topo_velocity(const TopoArgs a) {
  const int k = 3 + blockIdx.x * 32 + threadIdx.x;  // dm_offset = 3 (velocity_unroll.cu:420)
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int i = blockIdx.z;
  const int nz = a.nz;
  if (k >= nz || j >= a.ny || i >= a.nx) return;
  const int r = (k >= nz - 6) ? nz - 1 - k : -1;
  const Idx X{a.slice, a.yline, a.fld};
  const float *__restrict__ s11 = a.xx, *__restrict__ s12 = a.xy, *__restrict__ s13 = a.xz,
              *__restrict__ s22 = a.yy, *__restrict__ s23 = a.yz, *__restrict__ s33 = a.zz;
  const float* __restrict__ rho = a.d1;
  // neighbours as 32-bit offsets from this cell (the offsets are constants
  // times the strides, so each distinct one costs one multiply-add, not a
  // 64-bit index per load)
  const long long oc = X.p(i, j, k), ofc = X.f(i, j);
  auto S = [&](const float* __restrict__ s, int ii, int jj, int kk) {
    return __ldg(s + oc + ((ii - i) * a.slice + (jj - j) * a.yline + (kk - k)));
  };
  auto F = [&](const float* __restrict__ f, int ii, int jj) {
    return __ldg(f + ofc + ((ii - i) * a.fld + (jj - j)));
  };

  // density at the staggered velocity points (velocity_unroll.cu:140-152)
  const float rho1 = 0.25f * (S(rho, i, j, k - 1) + S(rho, i, j - 1, k - 1)) +
                     0.25f * (S(rho, i, j, k) + S(rho, i, j - 1, k));
  const float rho2 = 0.25f * (S(rho, i, j, k - 1) + S(rho, i - 1, j, k - 1)) +
                     0.25f * (S(rho, i, j, k) + S(rho, i - 1, j, k));
  const float rho3 = 0.25f * (S(rho, i, j, k) + S(rho, i - 1, j, k)) +
                     0.25f * (S(rho, i, j - 1, k) + S(rho, i - 1, j - 1, k));
  const float g3c = gk(a.g3_c, k), g3 = gk(a.g3, k);
  const float Ai1 = (float)((double)a.nu / (double)(F(a.f_1, i, j) * g3c * rho1));
  const float Ai2 = (float)((double)a.nu / (double)(F(a.f_2, i, j) * g3c * rho2));
  const float Ai3 = (float)((double)a.nu / (double)(F(a.f_c, i, j) * g3 * rho3));
  const float dcrj = ld(a.dcrjx, i + AWP_NGSL + 2) * ld(a.dcrjy, j + AWP_NGSL + 2) *
                     ld(a.dcrjz, k + AWP_ALIGN);

  // --- u1 -------------------------------------------------------------------
  float s1 = -kD1 * F(a.f_c, i, j) * g3c * S(s11, i, j, k) + kD0 * F(a.f_c, i - 2, j) * g3c * S(s11, i - 2, j, k) +
       kD1 * F(a.f_c, i - 1, j) * g3c * S(s11, i - 1, j, k) -
       kD0 * F(a.f_c, i + 1, j) * g3c * S(s11, i + 1, j, k);
  s1 += -kD1 * F(a.f, i, j) * g3c * S(s12, i, j, k) + kD0 * F(a.f, i, j - 2) * g3c * S(s12, i, j - 2, k) +
        kD1 * F(a.f, i, j - 1) * g3c * S(s12, i, j - 1, k) -
        kD0 * F(a.f, i, j + 1) * g3c * S(s12, i, j + 1, k);
  s1 += zdiff4(k, r, nz, true, kTopoVelDhz4r, [&](int kk) { return S(s13, i, j, kk); });
  {
    auto px = [&](int kk) {  // phx4 on s11 at i-2..i+1
      return gk(a.g_c, kk) * (kP1 * S(s11, i, j, kk) + kP0 * S(s11, i - 2, j, kk) +
                              kP1 * S(s11, i - 1, j, kk) + kP0 * S(s11, i + 1, j, kk));
    };
    auto py = [&](int kk) {  // phy4 on s12 at j-2..j+1
      return gk(a.g_c, kk) * (kP1 * S(s12, i, j, kk) + kP0 * S(s12, i, j - 2, kk) +
                              kP1 * S(s12, i, j - 1, kk) + kP0 * S(s12, i, j + 1, kk));
    };
    s1 = s1 - F(a.f1_1, i, j) * zdiff7(k, r, nz, kTopoVelDhpz4r, px);
    s1 = s1 - F(a.f2_1, i, j) * zdiff7(k, r, nz, kTopoVelDhpz4r, py);
  }
  // --- u2 -------------------------------------------------------------------
  float s2 = zdiff4(k, r, nz, true, kTopoVelDhz4r, [&](int kk) { return S(s23, i, j, kk); });
  s2 += kD1 * F(a.f, i, j) * g3c * S(s12, i, j, k) + kD0 * F(a.f, i - 1, j) * g3c * S(s12, i - 1, j, k) -
        kD1 * F(a.f, i + 1, j) * g3c * S(s12, i + 1, j, k) -
        kD0 * F(a.f, i + 2, j) * g3c * S(s12, i + 2, j, k);
  s2 += kD1 * F(a.f_c, i, j) * g3c * S(s22, i, j, k) +
        kD0 * F(a.f_c, i, j - 1) * g3c * S(s22, i, j - 1, k) -
        kD1 * F(a.f_c, i, j + 1) * g3c * S(s22, i, j + 1, k) -
        kD0 * F(a.f_c, i, j + 2) * g3c * S(s22, i, j + 2, k);
  {
    auto px = [&](int kk) {  // px4 on s12 at i-1..i+2
      return gk(a.g_c, kk) * (kP1 * S(s12, i, j, kk) + kP0 * S(s12, i - 1, j, kk) +
                              kP1 * S(s12, i + 1, j, kk) + kP0 * S(s12, i + 2, j, kk));
    };
    auto py = [&](int kk) {  // py4 on s22 at j-1..j+2
      return gk(a.g_c, kk) * (kP1 * S(s22, i, j, kk) + kP0 * S(s22, i, j - 1, kk) +
                              kP1 * S(s22, i, j + 1, kk) + kP0 * S(s22, i, j + 2, kk));
    };
    s2 = s2 - F(a.f1_2, i, j) * zdiff7(k, r, nz, kTopoVelDhpz4r, px);
    s2 = s2 - F(a.f2_2, i, j) * zdiff7(k, r, nz, kTopoVelDhpz4r, py);
  }
  // --- u3 -------------------------------------------------------------------
  float s3 = -kD1 * F(a.f_2, i, j) * g3 * S(s23, i, j, k) +
             kD0 * F(a.f_2, i, j - 2) * g3 * S(s23, i, j - 2, k) +
             kD1 * F(a.f_2, i, j - 1) * g3 * S(s23, i, j - 1, k) -
             kD0 * F(a.f_2, i, j + 1) * g3 * S(s23, i, j + 1, k);
  s3 += kD1 * F(a.f_1, i, j) * g3 * S(s13, i, j, k) + kD0 * F(a.f_1, i - 1, j) * g3 * S(s13, i - 1, j, k) -
        kD1 * F(a.f_1, i + 1, j) * g3 * S(s13, i + 1, j, k) -
        kD0 * F(a.f_1, i + 2, j) * g3 * S(s13, i + 2, j, k);
  s3 += zdiff4(k, r, nz, false, kTopoVelDz4r, [&](int kk) { return S(s33, i, j, kk); });
  {
    auto px = [&](int kk) {  // px4 on s13 at i-1..i+2, weighted by g
      return gk(a.g, kk) * (kP1 * S(s13, i, j, kk) + kP0 * S(s13, i - 1, j, kk) +
                            kP1 * S(s13, i + 1, j, kk) + kP0 * S(s13, i + 2, j, kk));
    };
    auto py = [&](int kk) {  // phy4 on s23 at j-2..j+1
      return gk(a.g, kk) * (kP1 * S(s23, i, j, kk) + kP0 * S(s23, i, j - 2, kk) +
                            kP1 * S(s23, i, j - 1, kk) + kP0 * S(s23, i, j + 1, kk));
    };
    s3 = s3 - F(a.f1_c, i, j) * zdiff7(k, r, nz, kTopoVelDphz4r, px);
    s3 = s3 - F(a.f2_c, i, j) * zdiff7(k, r, nz, kTopoVelDphz4r, py);
  }

  const long long o = X.p(i, j, k);
  a.u1[o] = (a.u1[o] + Ai1 * s1) * dcrj;
  a.v1[o] = (a.v1[o] + Ai2 * s2) * dcrj;
  a.w1[o] = (a.w1[o] + Ai3 * s3) * dcrj;
}

// ===========================================================================
// Stress and memory variables
// ===========================================================================
template <bool ELASTIC>
__global__ void __launch_bounds__(128) k_topo_stress(const TopoArgs a) {
  const int k = 3 + blockIdx.x * 32 + threadIdx.x;  // dm_offset = 3 (stress_attenuation.cu:177)
  const int j = a.s_j + blockIdx.y * 4 + threadIdx.y;
  const int i = a.s_i + blockIdx.z;
  const int nz = a.nz;
  if (k >= nz || j >= a.e_j || i >= a.e_i) return;
  const int r = (k >= nz - 6) ? nz - 1 - k : -1;
  const Idx X{a.slice, a.yline, a.fld};
  const float *__restrict__ u1 = a.u1, *__restrict__ v1 = a.v1, *__restrict__ w1 = a.w1;
  // neighbours as 32-bit offsets from this cell (the offsets are constants
  // times the strides, so each distinct one costs one multiply-add, not a
  // 64-bit index per load)
  const long long oc = X.p(i, j, k), ofc = X.f(i, j);
  auto S = [&](const float* __restrict__ s, int ii, int jj, int kk) {
    return __ldg(s + oc + ((ii - i) * a.slice + (jj - j) * a.yline + (kk - k)));
  };
  auto F = [&](const float* __restrict__ f, int ii, int jj) {
    return __ldg(f + ofc + ((ii - i) * a.fld + (jj - j)));
  };
  const float gc = gk(a.g_c, k), g = gk(a.g, k);

  // ---- normal components: Jii = 1 / (f_c g3_c) (stress_attenuation.cu:340-431)
  const float Jii = inv(F(a.f_c, i, j) * gk(a.g3_c, k));
  float d[9];
  {
    auto zu = [&](int ii, int jj) {
      return zdiff7(k, r, nz, kTopoStrPhdz4r, [&](int kk) { return S(u1, ii, jj, kk); });
    };
    auto zv = [&](int ii, int jj) {
      return zdiff7(k, r, nz, kTopoStrPhdz4r, [&](int kk) { return S(v1, ii, jj, kk); });
    };
    d[0] = kD1 * S(u1, i, j, k) + kD0 * S(u1, i - 1, j, k) - kD1 * S(u1, i + 1, j, k) -
           kD0 * S(u1, i + 2, j, k) -
           Jii * gc *
               (kP0 * F(a.f1_1, i - 1, j) * zu(i - 1, j) + kP1 * F(a.f1_1, i, j) * zu(i, j) +
                kP1 * F(a.f1_1, i + 1, j) * zu(i + 1, j) + kP0 * F(a.f1_1, i + 2, j) * zu(i + 2, j));
    d[1] = -kD1 * S(v1, i, j, k) + kD0 * S(v1, i, j - 2, k) + kD1 * S(v1, i, j - 1, k) -
           kD0 * S(v1, i, j + 1, k) -
           Jii * gc *
               (kP1 * F(a.f2_2, i, j) * zv(i, j) + kP0 * F(a.f2_2, i, j - 2) * zv(i, j - 2) +
                kP1 * F(a.f2_2, i, j - 1) * zv(i, j - 1) + kP0 * F(a.f2_2, i, j + 1) * zv(i, j + 1));
    d[2] = Jii * zdiff4(k, r, nz, true, kTopoStrDhz4r, [&](int kk) { return S(w1, i, j, kk); });
  }
  // ---- xy: J12i = 1 / (f g3_c); the interior rows read g3_c six points
  // higher (stress_attenuation.cu:471), the boundary rows at k (:1149)
  {
    const float J12i = inv(F(a.f, i, j) * gk(a.g3_c, r < 0 ? k + 6 : k));
    auto zu = [&](int ii, int jj) {
      return zdiff7(k, r, nz, kTopoStrPhdz4r, [&](int kk) { return S(u1, ii, jj, kk); });
    };
    auto zv = [&](int ii, int jj) {
      return zdiff7(k, r, nz, kTopoStrPhdz4r, [&](int kk) { return S(v1, ii, jj, kk); });
    };
    d[3] = kD1 * S(u1, i, j, k) + kD0 * S(u1, i, j - 1, k) - kD1 * S(u1, i, j + 1, k) -
           kD0 * S(u1, i, j + 2, k) -
           J12i * gc *
               (kP1 * F(a.f2_1, i, j) * zu(i, j) + kP0 * F(a.f2_1, i, j - 1) * zu(i, j - 1) +
                kP1 * F(a.f2_1, i, j + 1) * zu(i, j + 1) + kP0 * F(a.f2_1, i, j + 2) * zu(i, j + 2));
    d[4] = -kD1 * S(v1, i, j, k) + kD0 * S(v1, i - 2, j, k) + kD1 * S(v1, i - 1, j, k) -
           kD0 * S(v1, i + 1, j, k) -
           J12i * gc *
               (kP1 * F(a.f1_2, i, j) * zv(i, j) + kP0 * F(a.f1_2, i - 2, j) * zv(i - 2, j) +
                kP1 * F(a.f1_2, i - 1, j) * zv(i - 1, j) + kP0 * F(a.f1_2, i + 1, j) * zv(i + 1, j));
  }
  // ---- xz: J13i = 1 / (f_1 g3) (:550-598, :1254-1317)
  {
    const float J13i = inv(F(a.f_1, i, j) * gk(a.g3, k));
    auto zw = [&](int ii, int jj) {
      return zdiff7(k, r, nz, kTopoStrPdhz4r, [&](int kk) { return S(w1, ii, jj, kk); });
    };
    d[5] = J13i * zdiff4(k, r, nz, false, kTopoStrDz4r, [&](int kk) { return S(u1, i, j, kk); });
    d[6] = -kD1 * S(w1, i, j, k) + kD0 * S(w1, i - 2, j, k) + kD1 * S(w1, i - 1, j, k) -
           kD0 * S(w1, i + 1, j, k) -
           J13i * g *
               (kP1 * F(a.f1_c, i, j) * zw(i, j) + kP0 * F(a.f1_c, i - 2, j) * zw(i - 2, j) +
                kP1 * F(a.f1_c, i - 1, j) * zw(i - 1, j) + kP0 * F(a.f1_c, i + 1, j) * zw(i + 1, j));
  }
  // ---- yz: J23i = 1 / (f_2 g3) (:600-650, :1319-1380)
  {
    const float J23i = inv(F(a.f_2, i, j) * gk(a.g3, k));
    auto zw = [&](int ii, int jj) {
      return zdiff7(k, r, nz, kTopoStrPdhz4r, [&](int kk) { return S(w1, ii, jj, kk); });
    };
    d[7] = J23i * zdiff4(k, r, nz, false, kTopoStrDz4r, [&](int kk) { return S(v1, i, j, kk); });
    d[8] = kD1 * S(w1, i, j, k) + kD0 * S(w1, i, j - 1, k) - kD1 * S(w1, i, j + 1, k) -
           kD0 * S(w1, i, j + 2, k) -
           J23i * g *
               (kP1 * F(a.f2_c, i, j) * zw(i, j) + kP0 * F(a.f2_c, i, j - 1) * zw(i, j - 1) +
                kP1 * F(a.f2_c, i, j + 1) * zw(i, j + 1) + kP0 * F(a.f2_c, i, j + 2) * zw(i, j + 2));
  }

  // ---- material coefficients and the update (as the Cartesian dstrqc)
  const long long o = X.p(i, j, k);
  const int S1 = a.slice, Y1 = a.yline;
  auto sum8 = [&](const float* __restrict__ m) {
    return ld(m, o) + ld(m, o + S1) + ld(m, o - Y1) + ld(m, o + S1 - Y1) + ld(m, o - 1) +
           ld(m, o + S1 - 1) + ld(m, o - Y1 - 1) + ld(m, o + S1 - Y1 - 1);
  };
  const int ia = i + AWP_NGSL + 2, ja = j + AWP_NGSL + 2, ka = k + AWP_ALIGN;
  const int t = awp_tex_index(a.tex, ia, ja, ka);
  const float f_vx1 = a.tex.tau1[t], f_vx2 = a.tex.tau2[t], f_wwo = a.tex.wwo8[t];
  const float cc0 = ELASTIC ? 0.f : a.coeff[2 * t], cc1 = ELASTIC ? 0.f : a.coeff[2 * t + 1];
  const AwpStrCoef cf = awp_stress_coef<ELASTIC>(
      sum8(a.lam), sum8(a.mu), ld(a.mu, o), ld(a.mu, o - 1), ld(a.mu, o - Y1), ld(a.mu, o + S1),
      ELASTIC ? 0.f : sum8(a.qp), ELASTIC ? 0.f : sum8(a.qs), ld(a.qs, o), ld(a.qs, o - 1),
      ld(a.qs, o - Y1), ld(a.qs, o + S1), f_vx1, f_vx2, f_wwo, cc0, cc1, a.qthr, a.dth, a.dh1,
      a.DT);
  const float dcrj = ld(a.dcrjx, ia) * ld(a.dcrjy, ja) * ld(a.dcrjz, ka);
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

cudaError_t awp_launch_topo_velocity(const TopoArgs& a, cudaStream_t st) {
  if (a.nz < 12 || a.nx < 1 || a.ny < 1) return cudaErrorInvalidValue;
  const dim3 block(32, 4, 1);
  const dim3 grid((a.nz - 3 + 31) / 32, (a.ny + 3) / 4, a.nx);
  k_topo_velocity<<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_topo_stress(const TopoArgs& a, bool elastic, cudaStream_t st) {
  if (a.nz < 12) return cudaErrorInvalidValue;
  if (a.e_i <= a.s_i || a.e_j <= a.s_j) return cudaSuccess;
  const dim3 block(32, 4, 1);
  const dim3 grid((a.nz - 3 + 31) / 32, (a.e_j - a.s_j + 3) / 4, a.e_i - a.s_i);
  if (elastic)
    k_topo_stress<true><<<grid, block, 0, st>>>(a);
  else
    k_topo_stress<false><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}
