// Curvilinear (topography) velocity and stress half-steps of the top grid.
//
// The reference spells these operators out as generated code, one kernel for
// the interior (k below the top six points) and one for the six boundary rows
// next to the free surface:
//   velocity: dtopo_vel_111_unroll (kernels/velocity_unroll.cu:1-428) and
//             dtopo_vel_112 (kernels/optimized_velocity.cu:1040-1629),
//   stress:   dtopo_str_111 / dtopo_str_112 (kernels/stress_attenuation.cu:73-1415),
// launched by topo_velocity_*_H (velocity.cu) and topo_stress_*_H
// (stress_attenuation.cu).  Here each half-step is one kernel.  A warp owns 64
// consecutive levels of one (i, j) column, two adjacent levels per lane, and
// every lane loads the values of its own two levels only (one 8-byte access
// per field where the layout is 8-byte aligned): the vertical operators
// (7-point differences of horizontal interpolants, 4-point differences) take
// the neighbouring levels from the neighbouring lanes by warp shuffles -- six
// shuffles give a 7-point difference at both of a lane's levels -- so each
// value crosses the memory system once per column instead of once per stencil
// point.  Warps overlap by two lanes (four levels, the operators reach three)
// on each side: tiles of 56 output levels, the top tile outputting its 60
// levels under the surface.  The boundary-closure rows r = nz-1-k of the
// summation-by-parts tables (awp_topo_tables.h) read the top levels of the
// column, which all sit in the top tile's last lanes, by broadcast shuffles.
//
// Latency: a CTA (four warps = four j columns) takes AWP_TOPO_MARCH
// consecutive x planes one after another, so x-neighbour reads find the
// earlier planes in L1.  The values a thread reads only once are copied to
// shared memory by cp.async when the thread starts on a plane: in the
// velocity kernel all 31 of its 3-D operands, in the stress kernel the
// stresses and memory variables the update reads at the end.
//
// Term structure (f = surface function interpolants, g = vertical metric;
// relative indices, k = 0 the bottom point of the grid):
//   u_t = (A / (f g3 rho)) * [ D_x(f g3 sigma_x) + D_y(f g3 sigma_y) + D_z sigma_z
//                              - f1 * Dz(g P_x sigma_x) - f2 * Dz(g P_y sigma_y) ]
//   sigma_t from strain rates  D_x u - J^-1 g P_x(f1 Dz u)  etc.
// and the memory-variable / sponge update shared with the Cartesian kernels
// (awp_stress_coef / awp_stress_update).  Every level evaluates the same
// expressions in the same order (products and sums left to right as the
// reference's operators); the reference build contracts them into FMAs at its
// compiler's choice, so agreement with it is to rounding, not bitwise.
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
constexpr int kSpan = 64;     // levels of a warp
constexpr int kTileOut = 56;  // output levels of a tile below the top one

// Component-wise float2 arithmetic: each of a lane's two levels evaluates the
// scalar expression, with C++'s left-to-right grouping, unchanged.
__device__ __forceinline__ float2 operator+(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float2 operator-(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ float2 operator*(float2 a, float2 b) {
  return make_float2(a.x * b.x, a.y * b.y);
}
__device__ __forceinline__ float2 operator*(float a, float2 b) {
  return make_float2(a * b.x, a * b.y);
}

// The reference forms these reciprocals and quotients in double and rounds
// the result to float.  For float operands the double quotient (53 bits)
// rounded again to 24 bits equals the correctly rounded float quotient
// (double rounding is innocuous for division when the wider format has at
// least 2p + 2 bits; Figueroa, "When is double rounding innocuous?", 1995),
// so the IEEE float division gives the same bits without the FP64 pipe.
__device__ __forceinline__ float inv(float x) { return __frcp_rn(x); }
__device__ __forceinline__ float quot(float x, float y) { return __fdiv_rn(x, y); }

// Asynchronous copies global -> shared (cp.async) of a lane's two levels,
// issued when a thread starts on a plane for the values it reads once, so
// their latency overlaps the stencil arithmetic.  Each thread reads back its
// own slots after cp.async.wait_all; no block barrier is needed.  V2: one
// 8-byte copy (both addresses 8-byte aligned), else two 4-byte copies.
__device__ __forceinline__ void cpa(void* s, const float* g, int bytes_is_8) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  if (bytes_is_8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(g) : "memory");
}
template <bool V2>
__device__ __forceinline__ void cpa2(float2* s, const float* g) {
  if (V2) {
    cpa(s, g, 1);
  } else {
    cpa(&s->x, g, 0);
    cpa(&s->y, g + 1, 0);
  }
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <bool V2>
__device__ __forceinline__ float2 ld2(const float* __restrict__ p) {
  if (V2) return __ldg(reinterpret_cast<const float2*>(p));
  return make_float2(__ldg(p), __ldg(p + 1));
}

// 1-D vertical metric at a level, and at the lane's two levels
__device__ __forceinline__ float gk(const float* __restrict__ g, int k) {
  return __ldg(g + k + AWP_ALIGN);
}
__device__ __forceinline__ float2 gk2(const float* __restrict__ g, int k) {
  return make_float2(__ldg(g + k + AWP_ALIGN), __ldg(g + k + 1 + AWP_ALIGN));
}

// Column position of a warp: tile t = 0 holds the top 64 levels, tile t > 0
// the 64 levels starting 56 t lower; lane L holds levels kb + 2L and
// kb + 2L + 1.  A level is output when its lane is not a halo lane (two at
// each end; the top tile has no upper halo) and k >= 3 (the reference leaves
// the three bottom points to the mesh coupling, dm_offset = 3).  Loads read
// level max(kb + 2L, -32): the levels below the grid are padding and only
// ever feed halo lanes, and the clamp keeps a short grid's reads inside it.
struct ColPos2 {
  int k, ld, lane, r0, r1;
  bool top, out0, out1;
  __device__ ColPos2(int nz, int tile) {
    lane = threadIdx.x;
    top = (tile == 0);
    k = nz - kSpan - kTileOut * tile + 2 * lane;
    ld = k < -AWP_ALIGN ? -AWP_ALIGN : k;
    const bool in = lane >= 2 && (top || lane <= 29);
    out0 = in && k >= 3;
    out1 = in && k + 1 >= 3;
    // boundary rows nz-1-k of the top six levels (lanes 29..31)
    r0 = (top && lane >= 29) ? nz - 1 - k : -1;
    r1 = (top && lane >= 29) ? nz - 2 - k : -1;
  }
};

// Boundary-closure rows of the top tile: row r of T applied to the top NT
// levels (level nz-1-m = lane 31 - m/2, .y for even m).  Every row is formed
// with compile-time table indices (constant-bank operands, no per-lane indexed
// constant loads) and each level of lanes 29..31 picks its own row.
template <int NT>
__device__ __forceinline__ void closure(float2 v, const ColPos2& c, const float (&T)[6][NT],
                                        float2& s) {
  float top[NT];
#pragma unroll
  for (int m = 0; m < NT; ++m) top[m] = __shfl_sync(kAll, (m & 1) ? v.x : v.y, 31 - (m >> 1));
#pragma unroll
  for (int rr = 0; rr < 6; ++rr) {
    float b = 0.f;
#pragma unroll
    for (int m = NT - 1; m >= 0; --m) b += T[rr][m] * top[m];
    if (c.r0 == rr) s.x = b;
    if (c.r1 == rr) s.y = b;
  }
}

// 7-point vertical difference at the lane's two levels l, l+1 of a value held
// two levels per lane (interior coefficients), or the boundary rows of T in
// the top tile.  Summation order as the reference's operators.
template <int NT>
__device__ __forceinline__ float2 zd7(float2 v, const ColPos2& c, const float (&T)[6][NT]) {
  const float m3 = __shfl_up_sync(kAll, v.y, 2);    // l-3
  const float m2 = __shfl_up_sync(kAll, v.x, 1);    // l-2
  const float m1 = __shfl_up_sync(kAll, v.y, 1);    // l-1
  const float p2 = __shfl_down_sync(kAll, v.x, 1);  // l+2
  const float p3 = __shfl_down_sync(kAll, v.y, 1);  // l+3
  const float p4 = __shfl_down_sync(kAll, v.x, 2);  // l+4
  float2 s;
  s.x = kZ0 * m3 + kZ1 * m2 + kZ2 * m1 - kZ2 * v.y - kZ1 * p2 - kZ0 * p3;
  s.y = kZ0 * m2 + kZ1 * m1 + kZ2 * v.x - kZ2 * p2 - kZ1 * p3 - kZ0 * p4;
  if (c.top) closure(v, c, T, s);  // warp-uniform branch
  return s;
}

// 4-point vertical difference: half-point form (k-2..k+1) or node form
// (k-1..k+2), or the boundary rows.
template <int NT>
__device__ __forceinline__ float2 zd4(float2 v, const ColPos2& c, bool half,
                                      const float (&T)[6][NT]) {
  float2 s;
  if (half) {
    const float m2 = __shfl_up_sync(kAll, v.x, 1), m1 = __shfl_up_sync(kAll, v.y, 1),
                p2 = __shfl_down_sync(kAll, v.x, 1);
    s.x = kD0 * m2 + kD1 * m1 - kD1 * v.x - kD0 * v.y;
    s.y = kD0 * m1 + kD1 * v.x - kD1 * v.y - kD0 * p2;
  } else {
    const float m1 = __shfl_up_sync(kAll, v.y, 1), p2 = __shfl_down_sync(kAll, v.x, 1),
                p3 = __shfl_down_sync(kAll, v.y, 1);
    s.x = kD0 * m1 + kD1 * v.x - kD1 * v.y - kD0 * p2;
    s.y = kD0 * v.x + kD1 * v.y - kD1 * p2 - kD0 * p3;
  }
  if (c.top) closure(v, c, T, s);
  return s;
}

// The value at level - 1 of each of a lane's two levels
__device__ __forceinline__ float2 below(float2 v) {
  return make_float2(__shfl_up_sync(kAll, v.y, 1), v.x);
}

struct Cell {
  long long o;   // padded index of (i, j, ld): the lane's first load level
  long long of;  // index of (i, j) in the 2-D metric arrays
  int S, Y, F;
  __device__ Cell(const TopoArgs& a, int i, int j, int ld)
      : o((long long)(i + AWP_NGSL + 2) * a.slice + (long long)(j + AWP_NGSL + 2) * a.yline +
          (ld + AWP_ALIGN)),
        of((long long)(i + AWP_NGSL + 2) * a.fld + (j + AWP_NGSL + 2 + AWP_ALIGN)),
        S(a.slice), Y(a.yline), F(a.fld) {}
  // 2-D metric at (i+di, j+dj)
  __device__ __forceinline__ float fm(const float* __restrict__ f, int di, int dj) const {
    return __ldg(f + of + (di * F + dj));
  }
};

// Store a lane's two output levels at p (8-byte store where aligned and both
// are output).
template <bool V2>
__device__ __forceinline__ void st2(float* p, float2 v, bool o0, bool o1) {
  if (V2 && o0 && o1) {
    *reinterpret_cast<float2*>(p) = v;
  } else {
    if (o0) p[0] = v.x;
    if (o1) p[1] = v.y;
  }
}

}  // namespace

// CTAs per SM the register allocation is held to, and x planes per CTA;
// chosen by timing at 512 x 512 x 256 with a hill.
#ifndef AWP_TOPO_VEL_MINB
#define AWP_TOPO_VEL_MINB 6
#endif
#ifndef AWP_TOPO_STR_MINB
#define AWP_TOPO_STR_MINB 6
#endif
#ifndef AWP_TOPO_MARCH
#define AWP_TOPO_MARCH 4
#endif

// ===========================================================================
// Velocity
// ===========================================================================
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

// One column tile of plane i, column j.
template <bool V2>
__device__ __forceinline__ void velocity_column(const TopoArgs& a, const ColPos2& c, int i,
                                                int j, float2 (&pre)[kVelPre][128]) {
  const Cell X(a, i, j, c.ld);
  const int tid = threadIdx.y * 32 + threadIdx.x;
  {
    auto cp = [&](int slot, const float* f, int di, int dj) {
      cpa2<V2>(&pre[slot][tid], f + X.o + ((long long)di * X.S + dj * X.Y));
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
  const int k = c.ld;
  const float2 g3c = gk2(a.g3_c, k), g3 = gk2(a.g3, k), gc = gk2(a.g_c, k), gg = gk2(a.g, k);
  const float fc = X.fm(a.f_c, 0, 0), ff = X.fm(a.f, 0, 0), f1 = X.fm(a.f_1, 0, 0),
              f2 = X.fm(a.f_2, 0, 0);
  const float dcx = __ldg(a.dcrjx + i + AWP_NGSL + 2) * __ldg(a.dcrjy + j + AWP_NGSL + 2);
  const float2 dcrj = dcx * gk2(a.dcrjz, k);
  cpa_wait();

  // density at the staggered velocity points (velocity_unroll.cu:140-152)
  const float2 r00 = P(kR00), r0m = P(kR0m), rm0 = P(kRm0), rmm = P(kRmm);
  const float2 r00k = below(r00), r0mk = below(r0m), rm0k = below(rm0);
  const float2 rho1 = 0.25f * (r00k + r0mk) + 0.25f * (r00 + r0m);
  const float2 rho2 = 0.25f * (r00k + rm0k) + 0.25f * (r00 + rm0);
  const float2 rho3 = 0.25f * (r00 + rm0) + 0.25f * (r0m + rmm);
  const float2 d1a = f1 * g3c * rho1, d2a = f2 * g3c * rho2, d3a = fc * g3 * rho3;
  const float2 Ai1 = make_float2(quot(a.nu, d1a.x), quot(a.nu, d1a.y));
  const float2 Ai2 = make_float2(quot(a.nu, d2a.x), quot(a.nu, d2a.y));
  const float2 Ai3 = make_float2(quot(a.nu, d3a.x), quot(a.nu, d3a.y));

  // --- u1 -------------------------------------------------------------------
  float2 s1 = -kD1 * fc * g3c * P(kX11_0) + kD0 * X.fm(a.f_c, -2, 0) * g3c * P(kX11_m2) +
              kD1 * X.fm(a.f_c, -1, 0) * g3c * P(kX11_m1) -
              kD0 * X.fm(a.f_c, 1, 0) * g3c * P(kX11_p1);
  s1 = s1 + (-kD1 * ff * g3c * P(kY12_0) + kD0 * X.fm(a.f, 0, -2) * g3c * P(kY12_m2) +
             kD1 * X.fm(a.f, 0, -1) * g3c * P(kY12_m1) - kD0 * X.fm(a.f, 0, 1) * g3c * P(kY12_p1));
  s1 = s1 + zd4(P(kX13_0), c, true, kTopoVelDhz4r);
  {
    const float2 px =
        gc * (kP1 * P(kX11_0) + kP0 * P(kX11_m2) + kP1 * P(kX11_m1) + kP0 * P(kX11_p1));
    const float2 py =
        gc * (kP1 * P(kY12_0) + kP0 * P(kY12_m2) + kP1 * P(kY12_m1) + kP0 * P(kY12_p1));
    s1 = s1 - X.fm(a.f1_1, 0, 0) * zd7(px, c, kTopoVelDhpz4r);
    s1 = s1 - X.fm(a.f2_1, 0, 0) * zd7(py, c, kTopoVelDhpz4r);
  }
  // --- u2 -------------------------------------------------------------------
  float2 s2 = zd4(P(kY23_0), c, true, kTopoVelDhz4r);
  s2 = s2 + (kD1 * ff * g3c * P(kY12_0) + kD0 * X.fm(a.f, -1, 0) * g3c * P(kX12_m1) -
             kD1 * X.fm(a.f, 1, 0) * g3c * P(kX12_p1) - kD0 * X.fm(a.f, 2, 0) * g3c * P(kX12_p2));
  s2 = s2 + (kD1 * fc * g3c * P(kY22_0) + kD0 * X.fm(a.f_c, 0, -1) * g3c * P(kY22_m1) -
             kD1 * X.fm(a.f_c, 0, 1) * g3c * P(kY22_p1) -
             kD0 * X.fm(a.f_c, 0, 2) * g3c * P(kY22_p2));
  {
    const float2 px =
        gc * (kP1 * P(kY12_0) + kP0 * P(kX12_m1) + kP1 * P(kX12_p1) + kP0 * P(kX12_p2));
    const float2 py =
        gc * (kP1 * P(kY22_0) + kP0 * P(kY22_m1) + kP1 * P(kY22_p1) + kP0 * P(kY22_p2));
    s2 = s2 - X.fm(a.f1_2, 0, 0) * zd7(px, c, kTopoVelDhpz4r);
    s2 = s2 - X.fm(a.f2_2, 0, 0) * zd7(py, c, kTopoVelDhpz4r);
  }
  // --- u3 -------------------------------------------------------------------
  float2 s3 = -kD1 * f2 * g3 * P(kY23_0) + kD0 * X.fm(a.f_2, 0, -2) * g3 * P(kY23_m2) +
              kD1 * X.fm(a.f_2, 0, -1) * g3 * P(kY23_m1) -
              kD0 * X.fm(a.f_2, 0, 1) * g3 * P(kY23_p1);
  s3 = s3 + (kD1 * f1 * g3 * P(kX13_0) + kD0 * X.fm(a.f_1, -1, 0) * g3 * P(kX13_m1) -
             kD1 * X.fm(a.f_1, 1, 0) * g3 * P(kX13_p1) - kD0 * X.fm(a.f_1, 2, 0) * g3 * P(kX13_p2));
  s3 = s3 + zd4(P(kZ33), c, false, kTopoVelDz4r);
  {
    const float2 px =
        gg * (kP1 * P(kX13_0) + kP0 * P(kX13_m1) + kP1 * P(kX13_p1) + kP0 * P(kX13_p2));
    const float2 py =
        gg * (kP1 * P(kY23_0) + kP0 * P(kY23_m2) + kP1 * P(kY23_m1) + kP0 * P(kY23_p1));
    s3 = s3 - X.fm(a.f1_c, 0, 0) * zd7(px, c, kTopoVelDphz4r);
    s3 = s3 - X.fm(a.f2_c, 0, 0) * zd7(py, c, kTopoVelDphz4r);
  }

  if (!(c.out0 || c.out1)) return;
  st2<V2>(a.u1 + X.o, (P(kU) + Ai1 * s1) * dcrj, c.out0, c.out1);
  st2<V2>(a.v1 + X.o, (P(kV) + Ai2 * s2) * dcrj, c.out0, c.out1);
  st2<V2>(a.w1 + X.o, (P(kW) + Ai3 * s3) * dcrj, c.out0, c.out1);
}

// A CTA takes four columns of AWP_TOPO_MARCH consecutive x planes, one plane
// after another, so that the x-neighbour reads of a plane find the previous
// planes' values in L1.
template <bool V2>
__global__ void __launch_bounds__(128, AWP_TOPO_VEL_MINB) k_topo_velocity(const TopoArgs a) {
  const ColPos2 c(a.nz, blockIdx.x);
  const int j = blockIdx.y * 4 + threadIdx.y;
  if (j >= a.ny) return;  // whole warps
  __shared__ float2 pre[kVelPre][128];
  const int i0 = blockIdx.z * AWP_TOPO_MARCH, i1 = min(i0 + AWP_TOPO_MARCH, a.nx);
#pragma unroll 1
  for (int i = i0; i < i1; ++i) velocity_column<V2>(a, c, i, j, pre);
}

// ===========================================================================
// Stress and memory variables
// ===========================================================================
// A stress thread stages the stresses and memory variables of its two levels
// by cp.async when it starts on a plane (read only by the update at its end);
// the velocity stencil and the media are read where they are used, through L1.
template <bool ELASTIC>
struct StrStage {
  static constexpr int kRows = ELASTIC ? 6 : 12;
};

template <bool ELASTIC, bool V2>
__device__ __forceinline__ void stress_column(const TopoArgs& a, const ColPos2& c, int i, int j,
                                              float2 (&pre)[StrStage<ELASTIC>::kRows][128]) {
  const Cell X(a, i, j, c.ld);
  const int k = c.ld;
  const int S1 = a.slice, Y1 = a.yline;
  const long long o = X.o;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  float* const SG[6] = {a.xx, a.yy, a.zz, a.xy, a.xz, a.yz};
  float* const RR[6] = {a.r1, a.r2, a.r3, a.r4, a.r5, a.r6};
#pragma unroll
  for (int q = 0; q < 6; ++q) cpa2<V2>(&pre[q][tid], SG[q] + o);
  if (!ELASTIC) {
#pragma unroll
    for (int q = 0; q < 6; ++q) cpa2<V2>(&pre[6 + q][tid], RR[q] + o);
  }
  // the 21 velocity stencil points: (field, di, dj)
  constexpr signed char kStencil[21][3] = {
      {0, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 2, 0}, {0, 0, -1}, {0, 0, 1}, {0, 0, 2},
      {1, 0, 0}, {1, 0, -2}, {1, 0, -1}, {1, 0, 1}, {1, -2, 0}, {1, -1, 0}, {1, 1, 0},
      {2, 0, 0}, {2, -2, 0}, {2, -1, 0}, {2, 1, 0}, {2, 0, -1}, {2, 0, 1}, {2, 0, 2}};
  const float* const V[3] = {a.u1, a.v1, a.w1};
  auto P = [&](int n) {
    return ld2<V2>(V[kStencil[n][0]] + o + (kStencil[n][1] * S1 + kStencil[n][2] * Y1));
  };
  const float2 gc = gk2(a.g_c, k), g = gk2(a.g, k);

  // every vertical difference of a horizontal interpolant is one difference
  // of the interpolated column (the metric weights do not depend on k)
  float2 d[9];
  // ---- normal components: Jii = 1 / (f_c g3_c) (stress_attenuation.cu:340-431)
  const float2 jii = X.fm(a.f_c, 0, 0) * gk2(a.g3_c, k);
  const float2 Jii = make_float2(inv(jii.x), inv(jii.y));
  const float2 u_0 = P(0), u_xm1 = P(1), u_xp1 = P(2), u_xp2 = P(3);
  const float2 v_0 = P(7), v_ym2 = P(8), v_ym1 = P(9), v_yp1 = P(10);
  const float2 w_0 = P(14);
  {
    const float2 iu = kP0 * X.fm(a.f1_1, -1, 0) * u_xm1 + kP1 * X.fm(a.f1_1, 0, 0) * u_0 +
                      kP1 * X.fm(a.f1_1, 1, 0) * u_xp1 + kP0 * X.fm(a.f1_1, 2, 0) * u_xp2;
    d[0] = kD1 * u_0 + kD0 * u_xm1 - kD1 * u_xp1 - kD0 * u_xp2 -
           Jii * gc * zd7(iu, c, kTopoStrPhdz4r);
    const float2 iv = kP1 * X.fm(a.f2_2, 0, 0) * v_0 + kP0 * X.fm(a.f2_2, 0, -2) * v_ym2 +
                      kP1 * X.fm(a.f2_2, 0, -1) * v_ym1 + kP0 * X.fm(a.f2_2, 0, 1) * v_yp1;
    d[1] = -kD1 * v_0 + kD0 * v_ym2 + kD1 * v_ym1 - kD0 * v_yp1 -
           Jii * gc * zd7(iv, c, kTopoStrPhdz4r);
    d[2] = Jii * zd4(w_0, c, true, kTopoStrDhz4r);
  }
  // ---- xy: J12i = 1 / (f g3_c); the interior rows read g3_c six points
  // higher (stress_attenuation.cu:471), the boundary rows at k (:1149)
  {
    const float f0 = X.fm(a.f, 0, 0);
    const float2 J12i = make_float2(inv(f0 * gk(a.g3_c, c.r0 < 0 ? k + 6 : k)),
                                    inv(f0 * gk(a.g3_c, c.r1 < 0 ? k + 7 : k + 1)));
    const float2 u_ym1 = P(4), u_yp1 = P(5), u_yp2 = P(6);
    const float2 iu = kP1 * X.fm(a.f2_1, 0, 0) * u_0 + kP0 * X.fm(a.f2_1, 0, -1) * u_ym1 +
                      kP1 * X.fm(a.f2_1, 0, 1) * u_yp1 + kP0 * X.fm(a.f2_1, 0, 2) * u_yp2;
    d[3] = kD1 * u_0 + kD0 * u_ym1 - kD1 * u_yp1 - kD0 * u_yp2 -
           J12i * gc * zd7(iu, c, kTopoStrPhdz4r);
    const float2 v_xm2 = P(11), v_xm1 = P(12), v_xp1 = P(13);
    const float2 iv = kP1 * X.fm(a.f1_2, 0, 0) * v_0 + kP0 * X.fm(a.f1_2, -2, 0) * v_xm2 +
                      kP1 * X.fm(a.f1_2, -1, 0) * v_xm1 + kP0 * X.fm(a.f1_2, 1, 0) * v_xp1;
    d[4] = -kD1 * v_0 + kD0 * v_xm2 + kD1 * v_xm1 - kD0 * v_xp1 -
           J12i * gc * zd7(iv, c, kTopoStrPhdz4r);
  }
  // ---- xz: J13i = 1 / (f_1 g3) (:550-598, :1254-1317)
  {
    const float2 j13 = X.fm(a.f_1, 0, 0) * gk2(a.g3, k);
    const float2 J13i = make_float2(inv(j13.x), inv(j13.y));
    d[5] = J13i * zd4(u_0, c, false, kTopoStrDz4r);
    const float2 w_xm2 = P(15), w_xm1 = P(16), w_xp1 = P(17);
    const float2 iw = kP1 * X.fm(a.f1_c, 0, 0) * w_0 + kP0 * X.fm(a.f1_c, -2, 0) * w_xm2 +
                      kP1 * X.fm(a.f1_c, -1, 0) * w_xm1 + kP0 * X.fm(a.f1_c, 1, 0) * w_xp1;
    d[6] = -kD1 * w_0 + kD0 * w_xm2 + kD1 * w_xm1 - kD0 * w_xp1 -
           J13i * g * zd7(iw, c, kTopoStrPdhz4r);
  }
  // ---- yz: J23i = 1 / (f_2 g3) (:600-650, :1319-1380)
  {
    const float2 j23 = X.fm(a.f_2, 0, 0) * gk2(a.g3, k);
    const float2 J23i = make_float2(inv(j23.x), inv(j23.y));
    d[7] = J23i * zd4(v_0, c, false, kTopoStrDz4r);
    const float2 w_ym1 = P(18), w_yp1 = P(19), w_yp2 = P(20);
    const float2 iw = kP1 * X.fm(a.f2_c, 0, 0) * w_0 + kP0 * X.fm(a.f2_c, 0, -1) * w_ym1 +
                      kP1 * X.fm(a.f2_c, 0, 1) * w_yp1 + kP0 * X.fm(a.f2_c, 0, 2) * w_yp2;
    d[8] = kD1 * w_0 + kD0 * w_ym1 - kD1 * w_yp1 - kD0 * w_yp2 -
           J23i * g * zd7(iw, c, kTopoStrPdhz4r);
  }

  // ---- material coefficients and the update (as the Cartesian dstrqc); the
  // level-1 neighbours of the eight-cell sums from the lane's first level and
  // the lane below
  const float* const MT[4] = {a.lam, a.mu, a.qp, a.qs};
  const long long corner[4] = {o, o + S1, o - Y1, o + S1 - Y1};
  auto mat = [&](int m, int q) { return ld2<V2>(MT[m] + corner[q]); };
  auto sum8 = [&](int m) {
    const float2 q0 = mat(m, 0), q1 = mat(m, 1), q2 = mat(m, 2), q3 = mat(m, 3);
    return q0 + q1 + q2 + q3 + below(q0) + below(q1) + below(q2) + below(q3);
  };
  const float2 L8 = sum8(0), M8 = sum8(1);
  const float2 QP8 = ELASTIC ? make_float2(0.f, 0.f) : sum8(2);
  const float2 QS8 = ELASTIC ? make_float2(0.f, 0.f) : sum8(3);
  const float2 mu0 = mat(1, 0), muk = below(mu0);
  const float2 qs0 = ELASTIC ? make_float2(0.f, 0.f) : mat(3, 0);
  const float2 qsk = below(qs0);
  cpa_wait();
  if (!(c.out0 || c.out1)) return;
  const float2 mu_j = mat(1, 2), mu_i = mat(1, 1);
  const float2 qs_j = ELASTIC ? make_float2(0.f, 0.f) : mat(3, 2);
  const float2 qs_i = ELASTIC ? make_float2(0.f, 0.f) : mat(3, 1);
  const int ia = i + AWP_NGSL + 2, ja = j + AWP_NGSL + 2;
  const float dcx = __ldg(a.dcrjx + ia) * __ldg(a.dcrjy + ja);
  float2 sg2[6], rr2[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    sg2[q] = pre[q][tid];
    rr2[q] = ELASTIC ? make_float2(0.f, 0.f) : pre[6 + q][tid];
  }
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    auto el = [e](float2 v) { return e ? v.y : v.x; };
    const int ka = k + e + AWP_ALIGN;
    const int t = awp_tex_index(a.tex, ia, ja, ka);
    const float f_vx1 = a.tex.tau1[t], f_vx2 = a.tex.tau2[t], f_wwo = a.tex.wwo8[t];
    const float cc0 = ELASTIC ? 0.f : a.coeff[2 * t], cc1 = ELASTIC ? 0.f : a.coeff[2 * t + 1];
    const AwpStrCoef cf = awp_stress_coef<ELASTIC>(
        el(L8), el(M8), el(mu0), el(muk), el(mu_j), el(mu_i), el(QP8), el(QS8), el(qs0),
        el(qsk), el(qs_j), el(qs_i), f_vx1, f_vx2, f_wwo, cc0, cc1, a.qthr, a.dth, a.dh1, a.DT);
    const float dcrj = dcx * __ldg(a.dcrjz + ka);
    float sg[6], rr[6], de[9];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      sg[q] = el(sg2[q]);
      rr[q] = el(rr2[q]);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) de[q] = el(d[q]);
    awp_stress_update<ELASTIC>(sg, rr, cf, f_vx1, f_vx2, f_wwo, a.DT, dcrj, de);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      if (e) {
        sg2[q].y = sg[q];
        rr2[q].y = rr[q];
      } else {
        sg2[q].x = sg[q];
        rr2[q].x = rr[q];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    st2<V2>(SG[q] + o, sg2[q], c.out0, c.out1);
    if (!ELASTIC) st2<V2>(RR[q] + o, rr2[q], c.out0, c.out1);
  }
}

template <bool ELASTIC, bool V2>
__global__ void __launch_bounds__(128, AWP_TOPO_STR_MINB) k_topo_stress(const TopoArgs a) {
  const ColPos2 c(a.nz, blockIdx.x);
  const int j = a.s_j + blockIdx.y * 4 + threadIdx.y;
  if (j >= a.e_j) return;  // whole warps
  __shared__ float2 pre[StrStage<ELASTIC>::kRows][128];
  const int i0 = a.s_i + blockIdx.z * AWP_TOPO_MARCH, i1 = min(i0 + AWP_TOPO_MARCH, a.e_i);
#pragma unroll 1
  for (int i = i0; i < i1; ++i) stress_column<ELASTIC, V2>(a, c, i, j, pre);
}

// Tiles of a column: the top one (outputs nz-60 .. nz-1), then one per 56
// levels below it until a tile outputs level 3.
static unsigned column_tiles(int nz) {
  return 1u + (nz > 63 ? (unsigned)((nz - 63 + kTileOut - 1) / kTileOut) : 0u);
}

// 8-byte accesses need an even column length (yline = nz + 64, so every
// level pair starts on an even index) and 8-byte aligned fields.
static bool pairs_aligned(const TopoArgs& a) {
  const void* p[] = {a.u1, a.v1, a.w1, a.xx, a.yy, a.zz, a.xy, a.xz, a.yz, a.r1, a.r2,
                     a.r3, a.r4, a.r5, a.r6, a.d1, a.lam, a.mu, a.qp, a.qs};
  if (a.yline % 2 || a.slice % 2) return false;
  for (const void* q : p)
    if (q && ((size_t)q & 7)) return false;
  return true;
}

cudaError_t awp_launch_topo_velocity(const TopoArgs& a, cudaStream_t st) {
  if (a.nz < 12 || a.nx < 1 || a.ny < 1) return cudaErrorInvalidValue;
  const dim3 block(32, 4, 1);
  const dim3 grid(column_tiles(a.nz), (a.ny + 3) / 4,
                  (a.nx + AWP_TOPO_MARCH - 1) / AWP_TOPO_MARCH);
  if (pairs_aligned(a))
    k_topo_velocity<true><<<grid, block, 0, st>>>(a);
  else
    k_topo_velocity<false><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t awp_launch_topo_stress(const TopoArgs& a, bool elastic, cudaStream_t st) {
  if (a.nz < 12) return cudaErrorInvalidValue;
  if (a.e_i <= a.s_i || a.e_j <= a.s_j) return cudaSuccess;
  const dim3 block(32, 4, 1);
  const dim3 grid(column_tiles(a.nz), (a.e_j - a.s_j + 3) / 4,
                  (a.e_i - a.s_i + AWP_TOPO_MARCH - 1) / AWP_TOPO_MARCH);
  const bool v2 = pairs_aligned(a);
  if (elastic) {
    if (v2)
      k_topo_stress<true, true><<<grid, block, 0, st>>>(a);
    else
      k_topo_stress<true, false><<<grid, block, 0, st>>>(a);
  } else {
    if (v2)
      k_topo_stress<false, true><<<grid, block, 0, st>>>(a);
    else
      k_topo_stress<false, false><<<grid, block, 0, st>>>(a);
  }
  return cudaGetLastError();
}
