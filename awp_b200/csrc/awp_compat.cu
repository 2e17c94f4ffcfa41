// Reference-named launchers (include/awp/kernel_launch.h:10-190) on top of the
// B200 kernels.  The reference keeps per-grid constants in __constant__ memory
// set by SetDeviceConstValue (kernel.cu:68-117); here they live in a host-side
// table and travel to the kernels by value, which keeps every kernel launch
// independent of global device state.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <climits>

#include "../../include/awp_b200.h"
#include "awp_common.h"
#include "awp_dm.cuh"
#include "awp_host.h"
#include "awp_kernels.cuh"

namespace {

struct GridConsts {
  float dth, dh1, DH;
  int nxt, nyt, nzt;
  int slice, yline;
};

struct CompatState {
  int ngrids = 0;
  GridConsts g[AWP_MAXGRIDS];
  float DT = 0.f;
  float c1 = 9.0 / 8.0, c2 = -1.0 / 24.0;
  float fmajor = 0.f, fminor = 0.f, Rz[9] = {}, RzT[9] = {};
  int filtorder = 0;
  double filt_b[AWP_MAXFILT] = {}, filt_a[AWP_MAXFILT] = {};
  float qthr = 0.f;
  int exit_on_error = 1;
  int last_error = 0;
};

CompatState& S() {
  static CompatState s;
  return s;
}

inline int round_up(int n, int m) { return (n + m - 1) / m * m; }

// CUCHK semantics (include/awp/pmcl3d_cons.h:43-54): report and exit, unless
// the caller asked for "record and return".
void check(cudaError_t e, const char* func) {
  if (e == cudaSuccess) return;
  CompatState& s = S();
  s.last_error = (int)e;
  if (s.exit_on_error) {
    fprintf(stderr, "CUDA error in %s(): %s.\n", func, cudaGetErrorString(e));
    fflush(stderr);
    exit(EXIT_FAILURE);
  }
}

bool grid_ok(int d_i, const char* func) {
  if (d_i >= 0 && d_i < S().ngrids) return true;
  fprintf(stderr, "%s(): grid %d has no constants (call SetDeviceConstValue)\n", func, d_i);
  check(cudaErrorInvalidValue, func);
  return false;
}

PlastParams plast_params(int d_i) {
  CompatState& s = S();
  PlastParams p;
  p.fmajor = s.fmajor;
  p.fminor = s.fminor;
  memcpy(p.Rz, s.Rz, sizeof(p.Rz));
  memcpy(p.RzT, s.RzT, sizeof(p.RzT));
  p.dh = s.g[d_i].DH;
  p.dt = s.DT;
  p.ktop = s.g[d_i].nzt + AWP_ALIGN - 1;
  return p;
}

void stress_common(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz,
                   float* r1, float* r2, float* r3, float* r4, float* r5, float* r6,
                   float* u1, float* v1, float* w1, float* lam, float* mu, float* qp,
                   float* coeff, float* qs, float* dcrjx, float* dcrjy, float* dcrjz,
                   int nyt, int nzt, cudaStream_t St, float* lam_mu, float* vx1, float* vx2,
                   int* ww, float* wwo, int NX, int NPC, int rankx, int ranky, int s_i,
                   int e_i, int s_j, int e_j, int d_i, const char* func) {
  (void)nyt;
  if (!grid_ok(d_i, func)) return;
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  StrArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = xx; a.yy = yy; a.zz = zz; a.xy = xy; a.xz = xz; a.yz = yz;
  a.r1 = r1; a.r2 = r2; a.r3 = r3; a.r4 = r4; a.r5 = r5; a.r6 = r6;
  a.u1 = u1; a.v1 = v1; a.w1 = w1;
  a.lam = lam; a.mu = mu; a.qp = qp; a.qs = qs;
  a.dcrjx = dcrjx; a.dcrjy = dcrjy; a.dcrjz = dcrjz; a.lam_mu = lam_mu;
  a.vx1 = vx1; a.vx2 = vx2; a.ww = ww; a.wwo = wwo;
  a.coeff_dev = coeff;
  a.slice = gc.slice; a.yline = gc.yline;
  a.lam_mu_ld = gc.nyt + 4 + AWP_NGSL2;
  a.i0 = s_i; a.i1 = e_i; a.j0 = s_j; a.j1 = e_j;
  // dstrqc: k from align+3 to maxk, within the launched rows (kernel.cu:900-913)
  const int maxk = (d_i == 0) ? nzt + AWP_ALIGN - 1 : nzt + AWP_ALIGN - 3;
  a.k0 = AWP_ALIGN + 3;
  a.k1 = maxk < AWP_ALIGN + round_up(nzt, 4) - 1 ? maxk : AWP_ALIGN + round_up(nzt, 4) - 1;
  a.fs = (d_i == 0) ? 1 : 0;
  a.ktop = gc.nzt + AWP_ALIGN - 1;
  a.gx_lim = NX + AWP_NGSL + 1 - gc.nxt * rankx;
  a.gy_min = (NPC == 2) ? INT_MIN : AWP_NGSL + 3 - gc.nyt * ranky;
  a.dth = gc.dth; a.dh1 = gc.dh1; a.dt = s.DT; a.c1 = s.c1; a.c2 = s.c2;
  a.qthr = s.qthr;
  check(awp_launch_stress(a, false, St), func);
}

DmGrid dm_grid(int d_i, float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
               float* xy, float* xz, float* yz) {
  const GridConsts& gc = S().g[d_i];
  DmGrid g;
  g.u1 = u1; g.v1 = v1; g.w1 = w1;
  g.xx = xx; g.yy = yy; g.zz = zz; g.xy = xy; g.xz = xz; g.yz = yz;
  g.nxt = gc.nxt; g.nyt = gc.nyt; g.nzt = gc.nzt;
  g.slice = gc.slice; g.yline = gc.yline;
  return g;
}

// Halo exchanges between ranks: at world size 1 every neighbour rank is -1 and
// the reference returns at once (kernel.cu:331-333, 2036-2038, 2100-2102,
// 2162-2164, 2225-2227, 3320-3322, 3408-3410, 3499-3501, 3587-3589); more than
// one rank is outside this library.
void single_rank_only(int rank_a, int rank_b, const char* func) {
  if (rank_a == -1 && rank_b == -1) return;
  fprintf(stderr, "%s(): multi-rank halo exchange is not part of this library\n", func);
  check(cudaErrorNotSupported, func);
}

// fvel (kernel.cu:1949-2033): free-surface velocity images at k = top + 1 of
// grid 0 from the velocities at and below the surface.  Every (i, j) of the
// launch reads only levels top and top - 1, so the reference's sequential
// march over i is one thread per cell here.
struct FvelArgs {
  float *u1, *v1, *w1;
  const float* lam_mu;
  int lam_mu_ld, slice, yline, ktop;
  int i0, i1, j0, nj, gx_lim, gy_min;
};

__global__ void k_fvel(const FvelArgs a) {
  const int j = a.j0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = a.i0 + blockIdx.y;
  if (j >= a.j0 + a.nj || i > a.i1) return;
  const long long S = a.slice, Y = a.yline;
  const long long pos = (long long)i * S + (long long)j * Y + a.ktop;
  const float u0 = a.u1[pos], up1 = a.u1[pos + S];
  const float v0 = a.v1[pos], vjm1 = a.v1[pos - Y];
  const float w0 = a.w1[pos], wm1 = a.w1[pos - S], wp1 = a.w1[pos + S];
  const float wjp1 = a.w1[pos + Y], wjm1 = a.w1[pos - Y], wkm1 = a.w1[pos - 1];
  const float uimg = __fsub_rn(u0, __fsub_rn(w0, wm1));
  const float vimg = __fsub_rn(v0, __fsub_rn(wjp1, w0));
  const float vs1 = (i < a.gx_lim) ? __fsub_rn(up1, __fsub_rn(wp1, w0)) : 0.0f;
  const float vs2 = (j >= a.gy_min) ? __fsub_rn(vjm1, __fsub_rn(w0, wjm1)) : 0.0f;
  const float sum = __fadd_rn(__fadd_rn(__fadd_rn(__fsub_rn(vs1, uimg), __fsub_rn(up1, u0)),
                                        __fsub_rn(vimg, vs2)),
                              __fsub_rn(v0, vjm1));
  a.u1[pos + 1] = uimg;
  a.v1[pos + 1] = vimg;
  a.w1[pos + 1] = __fmaf_rn(-a.lam_mu[(long long)i * a.lam_mu_ld + j], sum, wkm1);
}

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

extern "C" {

void awp_compat_exit_on_error(int exit_on_error) { S().exit_on_error = exit_on_error; }

int awp_compat_last_error(void) {
  const int e = S().last_error;
  S().last_error = 0;
  return e;
}

void SetDeviceConstValue(float* DH, float DT, int* nxt, int* nyt, int* nzt, int ngrids,
                         float fmajor, float fminor, float* Rz, float* RzT) {
  CompatState& s = S();
  if (ngrids < 1 || ngrids > AWP_MAXGRIDS) {
    check(cudaErrorInvalidValue, "SetDeviceConstValue");
    return;
  }
  s.ngrids = ngrids;
  s.DT = DT;
  for (int k = 0; k < ngrids; ++k) {
    GridConsts& g = s.g[k];
    g.dth = DT / DH[k];
    g.dh1 = 1.0 / DH[k];
    g.DH = DH[k];
    g.nxt = nxt[k];
    g.nyt = nyt[k];
    g.nzt = nzt[k];
    g.yline = nzt[k] + 2 * AWP_ALIGN;
    g.slice = (nyt[k] + 4 + AWP_NGSL2) * g.yline;
  }
  s.fmajor = fmajor;
  s.fminor = fminor;
  if (Rz) memcpy(s.Rz, Rz, sizeof(s.Rz));
  if (RzT) memcpy(s.RzT, RzT, sizeof(s.RzT));
  s.qthr = awp::qf_threshold();
}

void SetDeviceFilterParameters(int filtorder, double* srcfilt_b, double* srcfilt_a) {
  CompatState& s = S();
  if (filtorder < 0 || filtorder >= AWP_MAXFILT) {
    check(cudaErrorInvalidValue, "SetDeviceFilterParameters");
    return;
  }
  s.filtorder = filtorder;
  for (int k = 0; k <= filtorder && filtorder > 0; ++k) {
    s.filt_b[k] = srcfilt_b[k];
    s.filt_a[k] = srcfilt_a[k];
  }
}

void dvelcx_H_opt(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz, float* xy,
                  float* xz, float* yz, float* dcrjx, float* dcrjy, float* dcrjz, float* d_1,
                  int nyt, int nzt, awp_stream_t St, int s_i, int e_i, int d_i, int ngrids) {
  if (!grid_ok(d_i, "dvelcx_H_opt")) return;
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  VelArgs a;
  a.u1 = u1; a.v1 = v1; a.w1 = w1;
  a.xx = xx; a.yy = yy; a.zz = zz; a.xy = xy; a.xz = xz; a.yz = yz;
  a.dcrjx = dcrjx; a.dcrjy = dcrjy; a.dcrjz = dcrjz; a.d1 = d_1;
  a.slice = gc.slice; a.yline = gc.yline;
  a.i0 = s_i; a.i1 = e_i;
  // launched rows: 2x2/4-thread blocks round j and k up (kernel.cu:300-301)
  a.j0 = 2 + AWP_NGSL; a.j1 = 2 + AWP_NGSL + round_up(nyt, 2) - 1;
  a.k0 = AWP_ALIGN; a.k1 = AWP_ALIGN + round_up(nzt, 4) - 1;
  // DM interface layers are left to dvelc2 (kernel.cu:146-147)
  if (d_i > 0 && a.k1 > gc.nzt + AWP_ALIGN - 3) a.k1 = gc.nzt + AWP_ALIGN - 3;
  if (d_i < ngrids - 1 && a.k0 < AWP_ALIGN + 3) a.k0 = AWP_ALIGN + 3;
  a.dth = gc.dth; a.c1 = s.c1; a.c2 = s.c2;
  check(awp_launch_velocity(a, St), "dvelcx_H_opt");
}

void dvelcy_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz, float* xy,
              float* xz, float* yz, float* dcrjx, float* dcrjy, float* dcrjz, float* d_1,
              int nxt, int nzt, float* s_u1, float* s_v1, float* s_w1, awp_stream_t St,
              int s_j, int e_j, int rank, int d_i) {
  (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;
  (void)dcrjx; (void)dcrjy; (void)dcrjz; (void)d_1; (void)nxt; (void)nzt; (void)s_u1;
  (void)s_v1; (void)s_w1; (void)St; (void)s_j; (void)e_j; (void)d_i;
  if (rank == -1) return;  // no neighbour at one rank (kernel.cu:321)
  fprintf(stderr, "dvelcy_H(): multi-rank halo strips are not part of this library\n");
  check(cudaErrorNotSupported, "dvelcy_H");
}

void dstrqc_H(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz, float* r1,
              float* r2, float* r3, float* r4, float* r5, float* r6, float* u1, float* v1,
              float* w1, float* lam, float* mu, float* qp, float* coeff, float* qs,
              float* dcrjx, float* dcrjy, float* dcrjz, int nyt, int nzt, awp_stream_t St,
              float* lam_mu, float* vx1, float* vx2, int* ww, float* wwo, int NX, int NPC,
              int rankx, int ranky, int s_i, int e_i, int s_j, int e_j, int d_i) {
  stress_common(xx, yy, zz, xy, xz, yz, r1, r2, r3, r4, r5, r6, u1, v1, w1, lam, mu, qp, coeff,
                qs, dcrjx, dcrjy, dcrjz, nyt, nzt, St, lam_mu, vx1, vx2, ww, wwo, NX, NPC,
                rankx, ranky, s_i, e_i, s_j, e_j, d_i, "dstrqc_H");
}

void dstrqc_H_new(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz, float* r1,
                  float* r2, float* r3, float* r4, float* r5, float* r6, float* u1, float* v1,
                  float* w1, float* lam, float* mu, float* qp, float* coeff, float* qs,
                  float* dcrjx, float* dcrjy, float* dcrjz, int nyt, int nzt, awp_stream_t St,
                  float* lam_mu, float* vx1, float* vx2, int* ww, float* wwo, int NX, int NPC,
                  int rankx, int ranky, int s_i, int e_i, int s_j, int e_j, int d_i) {
  stress_common(xx, yy, zz, xy, xz, yz, r1, r2, r3, r4, r5, r6, u1, v1, w1, lam, mu, qp, coeff,
                qs, dcrjx, dcrjy, dcrjz, nyt, nzt, St, lam_mu, vx1, vx2, ww, wwo, NX, NPC,
                rankx, ranky, s_i, e_i, s_j, e_j, d_i, "dstrqc_H_new");
}

void fstr_H(float* zz, float* xz, float* yz, awp_stream_t St, int s_i, int e_i, int s_j,
            int e_j) {
  if (!grid_ok(0, "fstr_H")) return;
  const GridConsts& gc = S().g[0];
  FstrArgs a;
  a.zz = zz; a.xz = xz; a.yz = yz;
  a.slice = gc.slice; a.yline = gc.yline; a.ktop = gc.nzt + AWP_ALIGN - 1;
  a.i0 = s_i; a.i1 = e_i;
  a.j0 = s_j; a.j1 = s_j + round_up(e_j - s_j + 1, 2) - 1;  // kernel.cu:1246-1247
  check(awp_launch_fstr(a, St), "fstr_H");
}

void drprecpc_calc_H_opt(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz,
                         float* mu, float* d1, float* sigma2, float* yldfac, float* cohes,
                         float* phi, float* neta, int nzt, int xls, int xre, int yls, int yre,
                         awp_stream_t St, int d_i) {
  if (!grid_ok(d_i, "drprecpc_calc_H_opt")) return;
  const GridConsts& gc = S().g[d_i];
  PlastCalcArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = xx; a.yy = yy; a.zz = zz; a.xy = xy; a.xz = xz; a.yz = yz;
  a.mu = mu; a.d1 = d1; a.sigma2 = sigma2; a.cohes = cohes; a.phi = phi;
  a.yldfac = yldfac; a.neta = neta; a.neta_mult = nullptr;
  a.p = plast_params(d_i);
  a.slice = gc.slice; a.yline = gc.yline;
  a.i0 = xls; a.i1 = xre; a.j0 = yls; a.j1 = yre;
  a.k0 = AWP_ALIGN;
  a.k1 = AWP_ALIGN + round_up(nzt, 4) - 1;
  if (a.k1 > nzt + AWP_ALIGN + 1) a.k1 = nzt + AWP_ALIGN + 1;
  check(awp_launch_plast_calc(a, St), "drprecpc_calc_H_opt");
}

void drprecpc_app_H(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz, float* mu,
                    float* sigma2, float* yldfac, int nzt, int xls, int xre, int yls, int yre,
                    awp_stream_t St, int d_i) {
  if (!grid_ok(d_i, "drprecpc_app_H")) return;
  const GridConsts& gc = S().g[d_i];
  PlastAppArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = xx; a.yy = yy; a.zz = zz; a.xy = xy; a.xz = xz; a.yz = yz;
  a.mu = mu; a.sigma2 = sigma2; a.yldfac = yldfac;
  a.p = plast_params(d_i);
  a.slice = gc.slice; a.yline = gc.yline;
  a.i0 = xls; a.i1 = xre;
  a.j0 = yls; a.j1 = yls + round_up(yre - yls + 1, 2) - 1;
  a.k0 = AWP_ALIGN; a.k1 = AWP_ALIGN + round_up(nzt, 4) - 1;
  check(awp_launch_plast_app(a, St), "drprecpc_app_H");
}

void addsrc_H(int i, int READ_STEP, int dim, int* psrc, int npsrc, awp_stream_t St, float* axx,
              float* ayy, float* azz, float* axz, float* ayz, float* axy, float* xx, float* yy,
              float* zz, float* xy, float* yz, float* xz, int d_i) {
  if (!grid_ok(d_i, "addsrc_H")) return;
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  SrcArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = xx; a.yy = yy; a.zz = zz; a.xy = xy; a.yz = yz; a.xz = xz;
  a.psrc = psrc; a.dim = dim; a.slice = gc.slice; a.yline = gc.yline;
  a.axx = axx; a.ayy = ayy; a.azz = azz; a.axz = axz; a.ayz = ayz; a.axy = axy;
  a.ncell = npsrc;
  a.stride = READ_STEP;
  a.tidx = i - 1;
  a.vtst = (float)s.DT / (gc.DH * gc.DH * gc.DH);
  check(awp_launch_addsrc(a, St), "addsrc_H");
}

void addkinsrc_H(int i, int dim, int* psrc, int npsrc, awp_stream_t St, float* mu, float* axx,
                 float* ayy, float* azz, float* axz, float* ayz, float* axy, float* xx, float* yy,
                 float* zz, float* xy, float* yz, float* xz, float* mom, double* d_srcfilt_d,
                 int d_i) {
  if (!grid_ok(d_i, "addkinsrc_H")) return;
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  KinSrcArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = xx; a.yy = yy; a.zz = zz; a.xy = xy; a.yz = yz; a.xz = xz;
  a.mu = mu;
  a.psrc = psrc; a.dim = dim; a.slice = gc.slice; a.yline = gc.yline;
  a.axx = axx; a.ayy = ayy; a.azz = azz; a.axz = axz; a.ayz = ayz; a.axy = axy;
  a.mom = mom;
  a.filt_state = d_srcfilt_d;
  a.filtorder = s.filtorder;
  memcpy(a.filt_b, s.filt_b, sizeof(a.filt_b));
  memcpy(a.filt_a, s.filt_a, sizeof(a.filt_a));
  a.ncell = npsrc;
  a.step = i;
  a.dt = s.DT;
  a.vtst = (float)s.DT / (gc.DH * gc.DH * gc.DH);
  check(awp_launch_addkinsrc(a, St), "addkinsrc_H");
}

void velbuffer_H(const float* u1, const float* v1, const float* w1, const float* neta,
                 float* Bufx, float* Bufy, float* Bufz, float* Bufeta, int NVE, int nbgx,
                 int nedx, int nskpx, int nbgy, int nedy, int nskpy, int nbgz, int nedz,
                 int nskpz, int rec_nxt, int rec_nyt, int rec_nzt, awp_stream_t St,
                 int FOLLOWBATHY, const int* bathy, int d_i) {
  if (!grid_ok(d_i, "velbuffer_H")) return;
  const GridConsts& gc = S().g[d_i];
  VelBufArgs a;
  memset(&a, 0, sizeof(a));
  a.u1 = u1; a.v1 = v1; a.w1 = w1; a.neta = neta;
  a.bufx = Bufx; a.bufy = Bufy; a.bufz = Bufz; a.bufeta = Bufeta;
  a.nve = NVE;
  a.nbgx = nbgx; a.nedx = nedx; a.nskpx = nskpx;
  a.nbgy = nbgy; a.nedy = nedy; a.nskpy = nskpy;
  a.nbgz = nbgz; a.nedz = nedz; a.nskpz = nskpz;
  a.rec_nxt = rec_nxt; a.rec_nyt = rec_nyt; a.rec_nzt = rec_nzt;
  a.slice = gc.slice; a.yline = gc.yline; a.ktop = gc.nzt + AWP_ALIGN - 1;
  a.w_shift = (d_i == 0) ? 1 : 0;
  if (d_i == 0 && FOLLOWBATHY == 1) {
    a.bathy = bathy;
    a.bathy_ld = gc.nxt + 4 + AWP_NGSL2;
  }
  check(awp_launch_velbuffer(a, St), "velbuffer_H");
}

// ---- discontinuous mesh (kernel.cu:2289-3234) ------------------------------

void dvelc2_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz, float* xy,
              float* xz, float* yz, float* dcrjx, float* dcrjy, float* dcrjz, float* d_1, int nxt,
              int nyt, awp_stream_t St, int d_i) {
  if (!grid_ok(d_i, "dvelc2_H")) return;
  (void)nxt; (void)nyt;
  DmVel2Args a;
  a.g = dm_grid(d_i, u1, v1, w1, xx, yy, zz, xy, xz, yz);
  a.d1 = d_1;
  a.dcrjx = dcrjx; a.dcrjy = dcrjy; a.dcrjz = dcrjz;
  a.dth = S().g[d_i].dth;
  check(awp_launch_dvelc2(a, St), "dvelc2_H");
}

void dstrqc2_H(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz, float* r1,
               float* r2, float* r3, float* r4, float* r5, float* r6, float* u1, float* v1,
               float* w1, float* lam, float* mu, float* qp, float* qs, float* dcrjx,
               float* dcrjy, float* dcrjz, int nxt, int nyt, awp_stream_t St, float* coeff,
               float* d_vx1, float* d_vx2, int* d_ww, float* d_wwo, int s_i, int e_i, int s_j,
               int e_j, int d_i) {
  if (!grid_ok(d_i, "dstrqc2_H")) return;
  (void)nxt; (void)nyt;
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  DmStr2Args a;
  memset(&a, 0, sizeof(a));
  a.g = dm_grid(d_i, u1, v1, w1, xx, yy, zz, xy, xz, yz);
  a.r1 = r1; a.r2 = r2; a.r3 = r3; a.r4 = r4; a.r5 = r5; a.r6 = r6;
  a.lam = lam; a.mu = mu; a.qp = qp; a.qs = qs;
  a.dcrjx = dcrjx; a.dcrjy = dcrjy; a.dcrjz = dcrjz;
  a.vx1 = d_vx1; a.vx2 = d_vx2; a.ww = d_ww; a.wwo = d_wwo;  // the caller's arrays
  a.coeff_dev = coeff;
  a.i0 = s_i; a.i1 = e_i; a.j0 = s_j; a.j1 = e_j;
  a.dth = gc.dth; a.dh1 = gc.dh1; a.dt = s.DT;
  check(awp_launch_dstrqc2(a, St), "dstrqc2_H");
}

// d_i is the coarse ("low") grid; its finer neighbour above is d_i - 1
// (kernel.cu:2792).
void intp3d_H(float* u1l, float* v1l, float* w1l, float* xxl, float* yyl, float* zzl,
              float* xyl, float* xzl, float* yzl, float* u1h, float* v1h, float* w1h, float* xxh,
              float* yyh, float* zzh, float* xyh, float* xzh, float* yzh, int nxtl, int nytl,
              int rank, awp_stream_t St, int d_i) {
  (void)nxtl; (void)nytl; (void)rank;
  if (!grid_ok(d_i, "intp3d_H") || !grid_ok(d_i - 1, "intp3d_H")) return;
  DmPairArgs a{dm_grid(d_i, u1l, v1l, w1l, xxl, yyl, zzl, xyl, xzl, yzl),
               dm_grid(d_i - 1, u1h, v1h, w1h, xxh, yyh, zzh, xyh, xzh, yzh)};
  check(awp_launch_intp3d(a, St), "intp3d_H");
}

// d_i is the fine ("high") grid; the coarse one below it is d_i + 1
// (kernel.cu:3223).  At world size 1 every point of the window average lies in
// the fine grid itself, so the swap-area buffers (zero at one rank,
// pmcl3d.c:1434-1508) are never read.
void swap_H(float* xxl, float* yyl, float* zzl, float* xyl, float* xzl, float* yzl, float* u1l,
            float* v1l, float* w1l, float* xxh, float* yyh, float* zzh, float* xyh, float* xzh,
            float* yzh, float* u1h, float* v1h, float* w1h, int nxtl, int nytl, float* buf_L,
            float* buf_R, float* buf_F, float* buf_B, int rank, awp_stream_t St, int d_i) {
  (void)nxtl; (void)nytl; (void)buf_L; (void)buf_R; (void)buf_F; (void)buf_B; (void)rank;
  if (!grid_ok(d_i, "swap_H") || !grid_ok(d_i + 1, "swap_H")) return;
  DmPairArgs a{dm_grid(d_i + 1, u1l, v1l, w1l, xxl, yyl, zzl, xyl, xzl, yzl),
               dm_grid(d_i, u1h, v1h, w1h, xxh, yyh, zzh, xyh, xzh, yzh)};
  check(awp_launch_swap3(a, St), "swap_H");
}

// ---- other sources (kernel.cu:1808-1834, 3860-3895) ---------------------------

void frcvel_H(int i, int READ_STEP, int dim, int* psrc, int npsrc, int tskp, awp_stream_t St,
              float* axx, float* ayy, float* azz, float* axz, float* ayz, float* axy, float* u1,
              float* v1, float* w1, int ymin, int ymax, int d_i) {
  (void)axz; (void)ayz; (void)axy;
  if (!grid_ok(d_i, "frcvel_H")) return;
  if (npsrc <= 0) return;
  if (tskp <= 0) {
    check(cudaErrorInvalidValue, "frcvel_H");
    return;
  }
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  FrcvelArgs a;
  a.i = i; a.read_step = READ_STEP; a.dim = dim; a.npsrc = npsrc; a.tskp = tskp;
  a.xmin = ymin; a.xmax = ymax;
  a.psrc = psrc;
  a.axx = axx; a.ayy = ayy; a.azz = azz; a.u1 = u1; a.v1 = v1; a.w1 = w1;
  a.slice = gc.slice; a.yline = gc.yline;
  a.DT = s.DT;
  check(awp_launch_frcvel(a, St), "frcvel_H");
}

void addplanesrc_H(int i, int dim, int NST, awp_stream_t St, float* mu, float* lambda, int ND,
                   int nxt, int nyt, float* axx, float* ayy, float* azz, float* xx, float* yy,
                   float* zz, float* xy, float* yz, float* xz, int d_i) {
  (void)dim; (void)NST; (void)xy;
  if (!grid_ok(d_i, "addplanesrc_H")) return;
  CompatState& s = S();
  const GridConsts& gc = s.g[d_i];
  PlaneSrcArgs a;
  a.n = i;
  a.nx = round_up(nxt + 4, 2);  // launched rows of the shipped 2 x 2 blocks
  a.ny = round_up(nyt + 4, 2);
  a.k = AWP_ALIGN + ND + 1;
  a.mu = mu; a.lambda = lambda; a.axx = axx; a.ayy = ayy; a.azz = azz;
  a.xx = xx; a.yy = yy; a.zz = zz; a.xz = xz; a.yz = yz;
  a.slice = gc.slice; a.yline = gc.yline;
  a.DT = s.DT;
  a.DH = gc.DH;
  check(awp_launch_planesrc(a, St), "addplanesrc_H");
}

void fvel_H(float* u1, float* v1, float* w1, awp_stream_t St, float* lam_mu, int NX, int rankx,
            int ranky, int s_i, int e_i, int s_j, int e_j) {
  if (!grid_ok(0, "fvel_H")) return;
  const GridConsts& gc = S().g[0];
  if (e_i < s_i || e_j < s_j) return;
  FvelArgs a;
  a.u1 = u1; a.v1 = v1; a.w1 = w1; a.lam_mu = lam_mu;
  a.lam_mu_ld = gc.nyt + 4 + AWP_NGSL2;
  a.slice = gc.slice; a.yline = gc.yline; a.ktop = gc.nzt + AWP_ALIGN - 1;
  a.i0 = s_i; a.i1 = e_i; a.j0 = s_j;
  a.nj = round_up(e_j - s_j + 1, 2);  // launched rows of the shipped 2-row blocks
  a.gx_lim = NX + AWP_NGSL + 1 - gc.nxt * rankx;  // g_i < NX
  a.gy_min = AWP_NGSL + 3 - gc.nyt * ranky;       // g_j > 1
  k_fvel<<<dim3(cdiv(a.nj, 128), e_i - s_i + 1), 128, 0, St>>>(a);
  check(cudaGetLastError(), "fvel_H");
}

// ---- halo exchanges: single rank only ----------------------------------------

void update_bound_y_H(float* u1, float* v1, float* w1, float* f_u1, float* f_v1, float* f_w1,
                      float* b_u1, float* b_v1, float* b_w1, int nxt, int nzt, awp_stream_t St1,
                      awp_stream_t St2, int rank_f, int rank_b, int d_i) {
  (void)u1; (void)v1; (void)w1; (void)f_u1; (void)f_v1; (void)f_w1; (void)b_u1; (void)b_v1;
  (void)b_w1; (void)nxt; (void)nzt; (void)St1; (void)St2; (void)d_i;
  single_rank_only(rank_f, rank_b, "update_bound_y_H");
}

void update_yldfac_buffer_x_H(float* yldfac, float* buf_L, float* buf_R, int nyt, int nzt,
                              awp_stream_t St1, awp_stream_t St2, int rank_L, int rank_R,
                              int d_i) {
  (void)yldfac; (void)buf_L; (void)buf_R; (void)nyt; (void)nzt; (void)St1; (void)St2; (void)d_i;
  single_rank_only(rank_L, rank_R, "update_yldfac_buffer_x_H");
}

void update_yldfac_data_x_H(float* yldfac, float* buf_L, float* buf_R, int nyt, int nzt,
                            awp_stream_t St1, awp_stream_t St2, int rank_L, int rank_R, int d_i) {
  (void)yldfac; (void)buf_L; (void)buf_R; (void)nyt; (void)nzt; (void)St1; (void)St2; (void)d_i;
  single_rank_only(rank_L, rank_R, "update_yldfac_data_x_H");
}

void update_yldfac_buffer_y_H(float* yldfac, float* buf_F, float* buf_B, int nxt, int nzt,
                              awp_stream_t St1, awp_stream_t St2, int rank_F, int rank_B,
                              int d_i) {
  (void)yldfac; (void)buf_F; (void)buf_B; (void)nxt; (void)nzt; (void)St1; (void)St2; (void)d_i;
  single_rank_only(rank_F, rank_B, "update_yldfac_buffer_y_H");
}

void update_yldfac_data_y_H(float* yldfac, float* buf_F, float* buf_B, int nxt, int nzt,
                            awp_stream_t St1, awp_stream_t St2, int rank_F, int rank_B, int d_i) {
  (void)yldfac; (void)buf_F; (void)buf_B; (void)nxt; (void)nzt; (void)St1; (void)St2; (void)d_i;
  single_rank_only(rank_F, rank_B, "update_yldfac_data_y_H");
}

void update_swapzone_buffer_x_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                                float* xy, float* xz, float* yz, float* buf_L, float* buf_R,
                                int nyt, awp_stream_t St1, awp_stream_t St2, int rank_L,
                                int rank_R, int zs, int ze, int meshtp) {
  (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;
  (void)buf_L; (void)buf_R; (void)nyt; (void)St1; (void)St2; (void)zs; (void)ze; (void)meshtp;
  single_rank_only(rank_L, rank_R, "update_swapzone_buffer_x_H");
}

void update_swapzone_data_x_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                              float* xy, float* xz, float* yz, float* buf_L, float* buf_R, int nyt,
                              awp_stream_t St1, awp_stream_t St2, int rank_L, int rank_R, int zs,
                              int ze, int meshtp) {
  (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;
  (void)buf_L; (void)buf_R; (void)nyt; (void)St1; (void)St2; (void)zs; (void)ze; (void)meshtp;
  single_rank_only(rank_L, rank_R, "update_swapzone_data_x_H");
}

void update_swapzone_buffer_y_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                                float* xy, float* xz, float* yz, float* buf_F, float* buf_B,
                                int nxt, awp_stream_t St1, awp_stream_t St2, int rank_F,
                                int rank_B, int zs, int ze, int d_i) {
  (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;
  (void)buf_F; (void)buf_B; (void)nxt; (void)St1; (void)St2; (void)zs; (void)ze; (void)d_i;
  single_rank_only(rank_F, rank_B, "update_swapzone_buffer_y_H");
}

void update_swapzone_data_y_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                              float* xy, float* xz, float* yz, float* buf_F, float* buf_B, int nxt,
                              awp_stream_t St1, awp_stream_t St2, int rank_F, int rank_B, int zs,
                              int ze, int d_i) {
  (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;
  (void)buf_F; (void)buf_B; (void)nxt; (void)St1; (void)St2; (void)zs; (void)ze; (void)d_i;
  single_rank_only(rank_F, rank_B, "update_swapzone_data_y_H");
}

// ---- debug printing ------------------------------------------------------------
// The reference's device-side printing is commented out (kernel.cu:270-296,
// 3236-3318): these launch nothing and print nothing, as there.

void print_const_H(int ngrids) { (void)ngrids; }

void print_nonzero_H(float* array, int nx, int ny, int nz, int d_i, int rank) {
  (void)array; (void)nx; (void)ny; (void)nz; (void)d_i; (void)rank;
}

void print_nonzero_mat_H(float* array, int nx, int ny, int nz, int d_i, float* d1, float* mu,
                         float* lam, float* qp, float* qs, int rank) {
  (void)array; (void)nx; (void)ny; (void)nz; (void)d_i; (void)d1; (void)mu; (void)lam; (void)qp;
  (void)qs; (void)rank;
}

void print_nan_H(float* array, int nx, int ny, int nz, char* vname) {
  (void)array; (void)nx; (void)ny; (void)nz; (void)vname;
}

}  // extern "C"
