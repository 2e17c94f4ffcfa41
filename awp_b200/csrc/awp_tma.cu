// TMA-pipelined stencil kernels for the context API (sm_100a).
//
// Each CTA owns a tile of 32 k (one 128-byte line) x 8 j and marches a chunk of
// x planes.  Per plane, one elected thread issues cp.async.bulk.tensor loads of
// the plane's tiles (with the j/k halo the stencil needs) into shared-memory
// rings; completion is tracked by one mbarrier per ring slot.  The loads run
// several planes ahead of the arithmetic, so the HBM latency is hidden by the
// pipeline rather than by occupancy, and every x plane of every field is read
// from HBM once per chunk.  Results are stored straight from registers with
// coalesced 128-byte rows.
//
// Tile boxes (x = k fastest, y = j, z = i), all 16-byte aligned in x:
//   halo   : k in [kb-4, kb+36), j in [jb-2, jb+10)   40 x 12 floats
//   media  : k in [kb-4, kb+32), j in [jb-1, jb+8)    36 x  9 floats
//   own    : k in [kb,   kb+32), j in [jb,   jb+8)    32 x  8 floats
//
// Every wait on an mbarrier is bounded; a wait that runs out sets the
// context's error word and the whole CTA leaves the march together.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include "awp_kernels.cuh"
#include "awp_stencil.cuh"
#include "awp_tma.cuh"

#define LDG(p) __ldg(p)

namespace {

constexpr int TZ = 32, TY = 8, NT = TZ * TY;
constexpr int HX = 40, HY = 12, HTILE = HX * HY;     // halo tile (floats)
constexpr int MX = 36, MY = 9, MTILE_B = MX * MY * 4; // media tile bytes (1296)
constexpr int MTILE = 352;                            // media tile stride (floats, 1408 B)
constexpr int OTILE = TZ * TY;                        // own tile (floats)
constexpr int DH_ = 7;                                // halo ring depth (planes i-2..i+2 + 2)
constexpr int DM_ = 4;                                // media ring depth (planes i, i+1 + 2)
constexpr int DO_ = 3;                                // own ring depth (plane i + 2)
// Poll limit of the pipeline waits: the default, and the one the drain of an
// aborted march always uses (copies already issued must land before the CTA
// releases its shared memory, whatever limit the march itself ran with).
constexpr unsigned kSpinLimit = 1u << 26;
// velocity kernel: each stress field is staged with only the halo its
// differences read (xx none, yy and xy j, zz and xz k, yz both), one slot of
// the ring holding the six tiles at 128-byte multiples
constexpr int VT_XX = 0, VT_YY = 256, VT_ZZ = 640, VT_XY = 960, VT_XZ = 1344, VT_YZ = 1664,
              VT_SLOT = 2144;
constexpr int VJ = TZ;  // row stride of the j-halo tiles (32 x 12)
constexpr int VK = HX;  // row stride of the k-halo tiles (40 x 8) and of yz (40 x 12)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned limit = kSpinLimit) {
  for (unsigned n = 0; n < limit; ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load3(void* dst, const CUtensorMap* map, uint64_t* bar,
                                          int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// One ring of per-plane slots with their mbarriers.
struct Ring {
  float* buf;
  uint64_t* bar;
  int depth, slot_floats, base;  // base = first plane of the march for this ring
  __device__ int slot(int p) const { return (p - base) % depth; }
  __device__ unsigned parity(int p) const { return ((p - base) / depth) & 1; }
  __device__ uint64_t* b(int p) const { return bar + slot(p); }
};

// Slot and mbarrier phase of one plane in a ring: plane p of a march lives in
// slot (p - base) % depth with phase ((p - base) / depth) & 1; the march
// advances these incrementally instead of dividing.
struct Cursor {
  int slot;
  unsigned phase;
  __device__ void next(int depth) {
    if (++slot == depth) {
      slot = 0;
      phase ^= 1u;
    }
  }
};
__device__ __forceinline__ int wrap_add(int s, int d, int depth) {
  s += d;
  return s >= depth ? s - depth : s;
}

// ===========================================================================
// Stress + memory variables (dstrqc, kernel.cu:880-1197), same arithmetic as
// k_stress in awp_kernels.cu (see there for the term-by-term citation).
// ===========================================================================
template <bool ELASTIC>
__global__ void __launch_bounds__(NT, 2)
    k_stress_tma(const StrArgs a, const __grid_constant__ TmaMaps tm, const int ichunk,
                 int* err, const unsigned spin) {
  constexpr int NM = ELASTIC ? 2 : 4;   // lam, mu (, qp, qs)
  constexpr int NO = ELASTIC ? 6 : 12;  // xx..yz (, r1..r6)
  extern __shared__ __align__(128) float smem[];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tx;
  const int kb = AWP_ALIGN + blockIdx.x * TZ;
  const int jb = a.j0 + blockIdx.y * TY;
  const int k = kb + tx, j = jb + ty;
  const int ib = a.i0 + blockIdx.z * ichunk;
  const int ie = min(ib + ichunk - 1, a.i1);
  const bool active = (k >= a.k0) && (k <= a.k1) && (j <= a.j1);

  Ring rh{smem, nullptr, DH_, 3 * HTILE, ib - 2};
  Ring rm{rh.buf + DH_ * 3 * HTILE, nullptr, DM_, NM * MTILE, ib};
  Ring ro{rm.buf + DM_ * NM * MTILE, nullptr, DO_, NO * OTILE, ib};
  uint64_t* bars = reinterpret_cast<uint64_t*>(ro.buf + DO_ * NO * OTILE);
  rh.bar = bars;
  rm.bar = bars + DH_;
  ro.bar = bars + DH_ + DM_;

  // producer: one thread issues a plane's tiles and arms its barrier
  // producer (thread 0): slot of the next plane each ring receives
  int ish = 0, ism = 0, iso = 0;
  auto issue_halo = [&](int p) {
    if (p > ie + 2) return;
    uint64_t* b = rh.bar + ish;
    mbar_expect_tx(b, 3 * HTILE * 4);
    float* d = rh.buf + ish * rh.slot_floats;
    for (int f = 0; f < 3; ++f) tma_load3(d + f * HTILE, &tm.halo[f], b, kb - 4, jb - 2, p);
    ish = wrap_add(ish, 1, DH_);
  };
  auto issue_media = [&](int p) {
    if (p > ie + 1) return;
    uint64_t* b = rm.bar + ism;
    mbar_expect_tx(b, NM * MTILE_B);
    float* d = rm.buf + ism * rm.slot_floats;
    for (int f = 0; f < NM; ++f) tma_load3(d + f * MTILE, &tm.media[f], b, kb - 4, jb - 1, p);
    ism = wrap_add(ism, 1, DM_);
  };
  auto issue_own = [&](int p) {
    if (p > ie) return;
    uint64_t* b = ro.bar + iso;
    mbar_expect_tx(b, NO * OTILE * 4);
    float* d = ro.buf + iso * ro.slot_floats;
    for (int f = 0; f < NO; ++f) tma_load3(d + f * OTILE, &tm.own[f], b, kb, jb, p);
    iso = wrap_add(iso, 1, DO_);
  };

  if (tid == 0) {
    for (int q = 0; q < DH_ + DM_ + DO_; ++q) mbar_init(bars + q, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // next plane to issue per ring (meaningful in the producer thread only)
  int nh = ib - 2, nm = ib, no = ib;
  if (tid == 0) {
    for (; nh < ib - 2 + DH_; ++nh) issue_halo(nh);
    for (; nm < ib + DM_; ++nm) issue_media(nm);
    for (; no < ib + DO_; ++no) issue_own(no);
  }

  const int S = a.slice, Y = a.yline;
  const float c1 = a.c1, c2 = a.c2, DT = a.dt, dth = a.dth, dh1 = a.dh1;
  const float dcy = LDG(a.dcrjy + min(j, a.j1)), dcz = LDG(a.dcrjz + min(max(k, a.k0), a.k1));
  const long long col = (long long)j * Y + k;
  const bool top = a.fs && (k == a.ktop);
  const bool top1 = a.fs && (k == a.ktop - 1);
  float* __restrict__ SG[6] = {a.xx, a.yy, a.zz, a.xy, a.xz, a.yz};
  float* __restrict__ RR[6] = {a.r1, a.r2, a.r3, a.r4, a.r5, a.r6};
  const int hoff = (ty + 2) * HX + (tx + 4);
  const int moff = (ty + 1) * MX + (tx + 4);
  const int ooff = ty * TZ + tx;
  bool ok = true, aborted = false;

  // consumers: the plane each ring waits for next (halo i+2, media i+1, own i)
  // and the slots of the oldest planes read (halo i-2, media i)
  Cursor wh{4, 0u}, wm{1, 0u}, wo{0, 0u};
  int sh = 0, sm = 0;
  // media of the current x plane at (j,k), (j-1,k), (j,k-1), (j-1,k-1): the
  // next plane's values of one step are the current plane's of the next
  float cl[4], cmu[4], cqp[4], cqs[4];
  // relaxation-table entries of this (j, k) column.  The table index depends
  // on the parity of i only (period 2 along the march), so both are read once
  // here instead of per plane, where the lanes of a warp (alternating k
  // parity) would split each constant-bank read in two.
  float tv1[2], tv2[2], twwo[2], tc0[2] = {0.f, 0.f}, tc1[2] = {0.f, 0.f};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int t = awp_tex_index(a.tex, ib + q, j, k);
    tv1[q] = a.tex.tau1[t];
    tv2[q] = a.tex.tau2[t];
    twwo[q] = a.tex.wwo8[t];
    if (!ELASTIC) {
      tc0[q] = a.coeff[2 * t];
      tc1[q] = a.coeff[2 * t + 1];
    }
  }
  for (int i = ib; i <= ie; ++i) {
    // ---- wait for the planes this step reads for the first time ------------
    if (i == ib) {
      for (int q = 0; q < 4 && ok; ++q) ok = mbar_wait(rh.bar + q, 0u, spin);  // ib-2..ib+1
      if (ok) ok = mbar_wait(rm.bar, 0u, spin);                                  // plane ib
    }
    if (ok) ok = mbar_wait(rh.bar + wh.slot, wh.phase, spin);
    if (ok) ok = mbar_wait(rm.bar + wm.slot, wm.phase, spin);
    if (ok) ok = mbar_wait(ro.bar + wo.slot, wo.phase, spin);
    // one barrier per plane: it also tells the producer that every thread is
    // done with the previous step's oldest planes, whose slots it refills
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    if (tid == 0 && i > ib) {
      issue_halo(nh++);
      issue_media(nm++);
      issue_own(no++);
    }
    const int sh1 = wrap_add(sh, 1, DH_), sh2 = wrap_add(sh, 2, DH_), sh3 = wrap_add(sh, 3, DH_),
              sh4 = wrap_add(sh, 4, DH_), sm1 = wrap_add(sm, 1, DM_);

    const float* Hm2 = rh.buf + sh * rh.slot_floats + hoff;
    const float* Hm1 = rh.buf + sh1 * rh.slot_floats + hoff;
    const float* H0 = rh.buf + sh2 * rh.slot_floats + hoff;
    const float* Hp1 = rh.buf + sh3 * rh.slot_floats + hoff;
    const float* Hp2 = rh.buf + sh4 * rh.slot_floats + hoff;
    // field f of a halo plane: + f * HTILE; neighbour (dj, dk): + dj * HX + dk
    const float u_m1 = Hm1[0], u_0 = H0[0], u_p1 = Hp1[0], u_p2 = Hp2[0];
    const float v_m2 = Hm2[HTILE], v_m1 = Hm1[HTILE], v_0 = H0[HTILE], v_p1 = Hp1[HTILE];
    const float w_m2 = Hm2[2 * HTILE], w_m1 = Hm1[2 * HTILE], w_0 = H0[2 * HTILE],
                w_p1 = Hp1[2 * HTILE];
    const float* U0 = H0;
    const float* V0 = H0 + HTILE;
    const float* W0 = H0 + 2 * HTILE;
    const float u_jp1 = U0[HX], u_jp2 = U0[2 * HX], u_jm1 = U0[-HX], u_km1 = U0[-1];
    const float v_jm1 = V0[-HX], v_jp1 = V0[HX], v_jm2 = V0[-2 * HX], v_km1 = V0[-1];
    const float w_km1 = W0[-1], w_km2 = W0[-2], w_jp1 = W0[HX], w_jp2 = W0[2 * HX],
                w_jm1 = W0[-HX];
    float uk1 = U0[1], vk1 = V0[1], wk1 = W0[1], uk2 = U0[2], vk2 = V0[2];

    const float* Mc = rm.buf + sm * rm.slot_floats + moff;
    const float* Mn = rm.buf + sm1 * rm.slot_floats + moff;
    // (j,k), (j-1,k), (j,k-1), (j-1,k-1) of a media tile
    auto m4 = [&](const float* m, int f, float& pa, float& pb, float& pc, float& pd) {
      const float* q = m + f * MTILE;
      pa = q[0];
      pb = q[-MX];
      pc = q[-1];
      pd = q[-MX - 1];
    };
    if (i == ib) {
      m4(Mc, 0, cl[0], cl[1], cl[2], cl[3]);
      m4(Mc, 1, cmu[0], cmu[1], cmu[2], cmu[3]);
      if (!ELASTIC) {
        m4(Mc, 2, cqp[0], cqp[1], cqp[2], cqp[3]);
        m4(Mc, 3, cqs[0], cqs[1], cqs[2], cqs[3]);
      }
    }
    float nl[4], nmu[4], nqp[4], nqs[4];
    m4(Mn, 0, nl[0], nl[1], nl[2], nl[3]);
    m4(Mn, 1, nmu[0], nmu[1], nmu[2], nmu[3]);
    const bool odd = ((i - ib) & 1) != 0;
    const float f_vx1 = odd ? tv1[1] : tv1[0], f_vx2 = odd ? tv2[1] : tv2[0],
                f_wwo = odd ? twwo[1] : twwo[0];
    float QP8 = 0.f, QS8 = 0.f;
    const float cc0 = odd ? tc0[1] : tc0[0], cc1 = odd ? tc1[1] : tc1[0];
    if (!ELASTIC) {
      m4(Mn, 2, nqp[0], nqp[1], nqp[2], nqp[3]);
      m4(Mn, 3, nqs[0], nqs[1], nqs[2], nqs[3]);
      QP8 = cqp[0] + nqp[0] + cqp[1] + nqp[1] + cqp[2] + nqp[2] + cqp[3] + nqp[3];
      QS8 = cqs[0] + nqs[0] + cqs[1] + nqs[1] + cqs[2] + nqs[2] + cqs[3] + nqs[3];
    }
    // eight-cell sums in the reference's order: pos, ip1, jm1, ijk, km1, ik1, jk1, ijk1
    const AwpStrCoef cf = awp_stress_coef<ELASTIC>(
        cl[0] + nl[0] + cl[1] + nl[1] + cl[2] + nl[2] + cl[3] + nl[3],
        cmu[0] + nmu[0] + cmu[1] + nmu[1] + cmu[2] + nmu[2] + cmu[3] + nmu[3], cmu[0], cmu[2],
        cmu[1], nmu[0], QP8, QS8, cqs[0], cqs[2], cqs[1], nqs[0], f_vx1, f_vx2, f_wwo, cc0, cc1,
        a.qthr, dth, dh1, DT);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      cl[q] = nl[q];
      cmu[q] = nmu[q];
      if (!ELASTIC) {
        cqp[q] = nqp[q];
        cqs[q] = nqs[q];
      }
    }
    const float dcrj = LDG(a.dcrjx + i) * dcy * dcz;
    const long long o = (long long)i * S;

    if (top && active) {
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
      uk2 = uk1 - (wk1 - Hm1[2 * HTILE + 1]);
      vk2 = vk1 - (W0[HX + 1] - wk1);
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

    const float* O = ro.buf + wo.slot * ro.slot_floats + ooff;
    float sg[6], rr[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) sg[q] = O[q * OTILE];
    if (!ELASTIC) {
#pragma unroll
      for (int q = 0; q < 6; ++q) rr[q] = O[(6 + q) * OTILE];
    }
    awp_stress_update<ELASTIC>(sg, rr, cf, f_vx1, f_vx2, f_wwo, DT, dcrj, d);
    if (active) {
#pragma unroll
      for (int q = 0; q < 6; ++q) SG[q][col + o] = sg[q];
      if (!ELASTIC) {
#pragma unroll
        for (int q = 0; q < 6; ++q) RR[q][col + o] = rr[q];
      }
    }

    wh.next(DH_);
    wm.next(DM_);
    wo.next(DO_);
    sh = sh1;
    sm = sm1;
  }
  if (aborted) {
    if (tid == 0) {
      atomicExch(err, 1);
      // let copies still in flight land before the CTA's shared memory is released
      for (int p = max(nh - DH_, ib - 2); p < nh && p <= ie + 2; ++p)
        (void)mbar_wait(rh.b(p), rh.parity(p));
      for (int p = max(nm - DM_, ib); p < nm && p <= ie + 1; ++p)
        (void)mbar_wait(rm.b(p), rm.parity(p));
      for (int p = max(no - DO_, ib); p < no && p <= ie; ++p)
        (void)mbar_wait(ro.b(p), ro.parity(p));
    }
    __syncthreads();
  }
}

// ===========================================================================
// Velocity (dvelcx_opt, kernel.cu:125-268), same arithmetic as k_velocity.
// Rings: stress halo tiles (6 fields, planes i-2..i+2), density (planes i,
// i+1), own velocity tiles (plane i).
// ===========================================================================
__global__ void __launch_bounds__(NT, 3)
    k_velocity_tma(const VelArgs a, const __grid_constant__ TmaMaps tm, const int ichunk,
                   int* err, const unsigned spin) {
  extern __shared__ __align__(128) float smem[];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tx;
  const int kb = AWP_ALIGN + blockIdx.x * TZ;
  const int jb = a.j0 + blockIdx.y * TY;
  const int k = kb + tx, j = jb + ty;
  const int ib = a.i0 + blockIdx.z * ichunk;
  const int ie = min(ib + ichunk - 1, a.i1);
  const bool active = (k >= a.k0) && (k <= a.k1) && (j <= a.j1);

  Ring rh{smem, nullptr, DH_, VT_SLOT, ib - 2};
  Ring rm{rh.buf + DH_ * VT_SLOT, nullptr, DM_, MTILE, ib};
  Ring ro{rm.buf + DM_ * MTILE, nullptr, DO_, 3 * OTILE, ib};
  uint64_t* bars = reinterpret_cast<uint64_t*>(ro.buf + DO_ * 3 * OTILE);
  rh.bar = bars;
  rm.bar = bars + DH_;
  ro.bar = bars + DH_ + DM_;

  // producer (thread 0): slot of the next plane each ring receives
  int ish = 0, ism = 0, iso = 0;
  auto issue_halo = [&](int p) {
    if (p > ie + 2) return;
    uint64_t* b = rh.bar + ish;
    mbar_expect_tx(b, VT_SLOT * 4);
    float* d = rh.buf + ish * rh.slot_floats;
    tma_load3(d + VT_XX, &tm.halo[0], b, kb, jb, p);
    tma_load3(d + VT_YY, &tm.halo[1], b, kb, jb - 2, p);
    tma_load3(d + VT_ZZ, &tm.halo[2], b, kb - 4, jb, p);
    tma_load3(d + VT_XY, &tm.halo[3], b, kb, jb - 2, p);
    tma_load3(d + VT_XZ, &tm.halo[4], b, kb - 4, jb, p);
    tma_load3(d + VT_YZ, &tm.halo[5], b, kb - 4, jb - 2, p);
    ish = wrap_add(ish, 1, DH_);
  };
  auto issue_media = [&](int p) {
    if (p > ie + 1) return;
    uint64_t* b = rm.bar + ism;
    mbar_expect_tx(b, MTILE_B);
    tma_load3(rm.buf + ism * rm.slot_floats, &tm.media[0], b, kb - 4, jb - 1, p);
    ism = wrap_add(ism, 1, DM_);
  };
  auto issue_own = [&](int p) {
    if (p > ie) return;
    uint64_t* b = ro.bar + iso;
    mbar_expect_tx(b, 3 * OTILE * 4);
    float* d = ro.buf + iso * ro.slot_floats;
    for (int f = 0; f < 3; ++f) tma_load3(d + f * OTILE, &tm.own[f], b, kb, jb, p);
    iso = wrap_add(iso, 1, DO_);
  };

  if (tid == 0) {
    for (int q = 0; q < DH_ + DM_ + DO_; ++q) mbar_init(bars + q, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // next plane to issue per ring (meaningful in the producer thread only)
  int nh = ib - 2, nm = ib, no = ib;
  if (tid == 0) {
    for (; nh < ib - 2 + DH_; ++nh) issue_halo(nh);
    for (; nm < ib + DM_; ++nm) issue_media(nm);
    for (; no < ib + DO_; ++no) issue_own(no);
  }

  const int S = a.slice, Y = a.yline;
  const float c1 = a.c1, c2 = a.c2, dth = a.dth;
  const float dcy = LDG(a.dcrjy + min(j, a.j1)), dcz = LDG(a.dcrjz + min(k, a.k1));
  const long long col = (long long)j * Y + k;
  const int o_xx = VT_XX + ty * TZ + tx;             // no halo
  const int o_yy = VT_YY + (ty + 2) * VJ + tx;       // j halo
  const int o_zz = VT_ZZ + ty * VK + tx + 4;         // k halo
  const int o_xy = VT_XY + (ty + 2) * VJ + tx;
  const int o_xz = VT_XZ + ty * VK + tx + 4;
  const int o_yz = VT_YZ + (ty + 2) * VK + tx + 4;   // both
  const int moff = (ty + 1) * MX + (tx + 4);
  const int ooff = ty * TZ + tx;
  bool ok = true, aborted = false;

  // consumers: the plane each ring waits for next (halo i+2, media i+1, own i)
  // and the slots of the oldest planes read (halo i-2, media i)
  Cursor wh{4, 0u}, wm{1, 0u}, wo{0, 0u};
  int sh = 0, sm = 0;
  for (int i = ib; i <= ie; ++i) {
    // ---- wait for the planes this step reads for the first time ------------
    if (i == ib) {
      for (int q = 0; q < 4 && ok; ++q) ok = mbar_wait(rh.bar + q, 0u, spin);  // ib-2..ib+1
      if (ok) ok = mbar_wait(rm.bar, 0u, spin);                                  // plane ib
    }
    if (ok) ok = mbar_wait(rh.bar + wh.slot, wh.phase, spin);
    if (ok) ok = mbar_wait(rm.bar + wm.slot, wm.phase, spin);
    if (ok) ok = mbar_wait(ro.bar + wo.slot, wo.phase, spin);
    // one barrier per plane: it also tells the producer that every thread is
    // done with the previous step's oldest planes, whose slots it refills
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    if (tid == 0 && i > ib) {
      issue_halo(nh++);
      issue_media(nm++);
      issue_own(no++);
    }
    const int sh1 = wrap_add(sh, 1, DH_), sh2 = wrap_add(sh, 2, DH_), sh3 = wrap_add(sh, 3, DH_),
              sh4 = wrap_add(sh, 4, DH_), sm1 = wrap_add(sm, 1, DM_);

    // halo fields: 0 xx, 1 yy, 2 zz, 3 xy, 4 xz, 5 yz
    const float* Hm2 = rh.buf + sh * rh.slot_floats;
    const float* Hm1 = rh.buf + sh1 * rh.slot_floats;
    const float* H0 = rh.buf + sh2 * rh.slot_floats;
    const float* Hp1 = rh.buf + sh3 * rh.slot_floats;
    const float* Hp2 = rh.buf + sh4 * rh.slot_floats;
    const float xx_m2 = Hm2[o_xx], xx_m1 = Hm1[o_xx], xx_0 = H0[o_xx], xx_p1 = Hp1[o_xx];
    const float xy_m1 = Hm1[o_xy], xy_0 = H0[o_xy], xy_p1 = Hp1[o_xy], xy_p2 = Hp2[o_xy];
    const float xz_m1 = Hm1[o_xz], xz_0 = H0[o_xz], xz_p1 = Hp1[o_xz], xz_p2 = Hp2[o_xz];
    const float* YY = H0 + o_yy;
    const float* ZZ = H0 + o_zz;
    const float* XY = H0 + o_xy;
    const float* XZ = H0 + o_xz;
    const float* YZ = H0 + o_yz;
    const float yz_0 = YZ[0];

    const float* Dc = rm.buf + sm * rm.slot_floats + moff;
    const float* Dn = rm.buf + sm1 * rm.slot_floats + moff;
    const float d_0 = Dc[0], d_0j = Dc[-MX], d_0k = Dc[-1], d_0jk = Dc[-MX - 1];
    const float d_p = Dn[0], d_pj = Dn[-MX], d_pk = Dn[-1];

    const float fd1 = awp_vel_factor(dth, d_0, d_0j, d_0k, d_0jk);
    const float fd2 = awp_vel_factor(dth, d_0, d_p, d_0k, d_pk);
    const float fd3 = awp_vel_factor(dth, d_0, d_p, d_0j, d_pj);
    const float dcrj = LDG(a.dcrjx + i) * dcy * dcz;

    const float* O = ro.buf + wo.slot * ro.slot_floats + ooff;
    const float u = awp_vel_update(O[0], fd1, c1, c2, xx_0 - xx_m1, xx_p1 - xx_m2,
                                   xy_0 - XY[-VJ], XY[VJ] - XY[-2 * VJ], xz_0 - XZ[-1],
                                   XZ[1] - XZ[-2], dcrj);
    const float v = awp_vel_update(O[OTILE], fd2, c1, c2, xy_p1 - xy_0, xy_p2 - xy_m1,
                                   YY[VJ] - YY[0], YY[2 * VJ] - YY[-VJ], yz_0 - YZ[-1],
                                   YZ[1] - YZ[-2], dcrj);
    const float w = awp_vel_update(O[2 * OTILE], fd3, c1, c2, xz_p1 - xz_0, xz_p2 - xz_m1,
                                   yz_0 - YZ[-VK], YZ[VK] - YZ[-2 * VK], ZZ[1] - ZZ[0],
                                   ZZ[2] - ZZ[-1], dcrj);
    if (active) {
      const long long o = (long long)i * S + col;
      a.u1[o] = u;
      a.v1[o] = v;
      a.w1[o] = w;
    }
    wh.next(DH_);
    wm.next(DM_);
    wo.next(DO_);
    sh = sh1;
    sm = sm1;
  }
  if (aborted) {
    if (tid == 0) {
      atomicExch(err, 1);
      for (int p = max(nh - DH_, ib - 2); p < nh && p <= ie + 2; ++p)
        (void)mbar_wait(rh.b(p), rh.parity(p));
      for (int p = max(nm - DM_, ib); p < nm && p <= ie + 1; ++p)
        (void)mbar_wait(rm.b(p), rm.parity(p));
      for (int p = max(no - DO_, ib); p < no && p <= ie; ++p)
        (void)mbar_wait(ro.b(p), ro.parity(p));
    }
    __syncthreads();
  }
}

inline unsigned cdiv_u(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// Poll limit the next launches give their pipeline waits (process-wide).
unsigned g_spin_limit = kSpinLimit;

size_t stress_smem(bool elastic) {
  const int nm = elastic ? 2 : 4, no = elastic ? 6 : 12;
  return sizeof(float) * ((size_t)DH_ * 3 * HTILE + (size_t)DM_ * nm * MTILE +
                          (size_t)DO_ * no * OTILE) +
         sizeof(uint64_t) * (DH_ + DM_ + DO_);
}
size_t velocity_smem() {
  return sizeof(float) * ((size_t)DH_ * VT_SLOT + (size_t)DM_ * MTILE + (size_t)DO_ * 3 * OTILE) +
         sizeof(uint64_t) * (DH_ + DM_ + DO_);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

// L2 promotion of the tensor maps' fetches (process-wide; a context encodes
// its maps with the value of the moment and re-encodes them when it changes):
// 0 none, 1 64 B, 2 128 B, 3 256 B.
static int g_l2_promotion = 3;

int awp_tma_set_l2_promotion(int mode) {
  if (mode < 0 || mode > 3) return 1;
  g_l2_promotion = mode;
  return 0;
}

int awp_tma_get_l2_promotion() { return g_l2_promotion; }

int awp_tma_encode(CUtensorMap* map, const float* base, const AwpGeom& g, int box_x, int box_y) {
  auto fn = encode_fn();
  if (!fn) return 1;
  const cuuint64_t dims[3] = {(cuuint64_t)g.nz_pad(), (cuuint64_t)g.ny_pad(),
                              (cuuint64_t)g.nx_pad()};
  const cuuint64_t strides[2] = {(cuuint64_t)g.yline * 4, (cuuint64_t)g.slice * 4};
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r =
      fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
         g_l2_promotion == 0   ? CU_TENSOR_MAP_L2_PROMOTION_NONE
         : g_l2_promotion == 1 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
         : g_l2_promotion == 2 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B
                               : CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : 2;
}

int awp_tma_box(int group, int* bx, int* by) {
  switch (group) {
    case 0: *bx = HX; *by = HY; return 0;   // halo
    case 1: *bx = MX; *by = MY; return 0;   // media
    case 2: *bx = TZ; *by = TY; return 0;   // own
    case 3: *bx = TZ; *by = HY; return 0;   // j halo only
    case 4: *bx = HX; *by = TY; return 0;   // k halo only
  }
  return 1;
}

cudaError_t awp_launch_stress_tma(const StrArgs& a, const TmaMaps& tm, bool elastic, int ichunk,
                                  int* err, cudaStream_t st) {
  const int nk = a.k1 - AWP_ALIGN + 1, nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nk <= 0 || nj <= 0 || ni <= 0) return cudaSuccess;
  const dim3 block(TZ, TY, 1);
  const dim3 grid(cdiv_u(nk, TZ), cdiv_u(nj, TY), cdiv_u(ni, ichunk));
  const size_t sm = stress_smem(elastic);
  cudaError_t e;
  if (elastic) {
    e = cudaFuncSetAttribute(k_stress_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
    if (e != cudaSuccess) return e;
    k_stress_tma<true><<<grid, block, sm, st>>>(a, tm, ichunk, err, g_spin_limit);
  } else {
    e = cudaFuncSetAttribute(k_stress_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
    if (e != cudaSuccess) return e;
    k_stress_tma<false><<<grid, block, sm, st>>>(a, tm, ichunk, err, g_spin_limit);
  }
  return cudaGetLastError();
}

cudaError_t awp_launch_velocity_tma(const VelArgs& a, const TmaMaps& tm, int ichunk, int* err,
                                    cudaStream_t st) {
  const int nk = a.k1 - AWP_ALIGN + 1, nj = a.j1 - a.j0 + 1, ni = a.i1 - a.i0 + 1;
  if (nk <= 0 || nj <= 0 || ni <= 0) return cudaSuccess;
  const dim3 block(TZ, TY, 1);
  const dim3 grid(cdiv_u(nk, TZ), cdiv_u(nj, TY), cdiv_u(ni, ichunk));
  const size_t sm = velocity_smem();
  cudaError_t e =
      cudaFuncSetAttribute(k_velocity_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_velocity_tma<<<grid, block, sm, st>>>(a, tm, ichunk, err, g_spin_limit);
  return cudaGetLastError();
}

int awp_tma_set_spin_limit(long long polls) {
  if (polls < 0 || polls > (1ll << 30)) return 1;
  g_spin_limit = (unsigned)polls;
  return 0;
}

long long awp_tma_get_spin_limit() { return g_spin_limit; }
