// C ABI of libawpb200: the re-entrant context API and the reference-named
// launchers.  See include/awp_b200.h for the contract of every entry point.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <map>
#include <vector>

#include "../../include/awp_b200.h"
#include "awp_common.h"
#include "awp_dm.cuh"
#include "awp_host.h"
#include "awp_kernels.cuh"
#include "awp_pointsets.h"
#include "awp_points.h"
#include "awp_tma.cuh"
#include "awp_topo.h"
#include "awp_topo_kern.cuh"
#include "awp_adjoint.cuh"

namespace {

thread_local char g_errmsg[512] = "";

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_errmsg, sizeof(g_errmsg), fmt, ap);
  va_end(ap);
  return status;
}

#define CU_TRY(call)                                                              \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return set_error(AWP_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                       cudaGetErrorString(e_));                                   \
  } while (0)

inline int round_up(int n, int m) { return (n + m - 1) / m * m; }

}  // namespace

// Lets other translation units of the library report through awp_last_error.
void awp_internal_set_error(const char* msg) {
  snprintf(g_errmsg, sizeof(g_errmsg), "%s", msg);
}

// ===========================================================================
// Context
// ===========================================================================
struct awp_ctx {
  awp_params p;
  AwpGeom g;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  float* f[AWP_NFIELDS] = {};
  float *dcrjx = nullptr, *dcrjy = nullptr, *dcrjz = nullptr, *lam_mu = nullptr;
  AwpTexture tex{};
  float coeff[16] = {}, tau8[8] = {}, w8[8] = {};
  float taumax = 0.f, taumin = 0.f;
  float qthr = 0.f;
  float c1 = 9.0 / 8.0, c2 = -1.0 / 24.0;
  float dth = 0.f, dh1 = 0.f;
  int xls = 0, xre = 0, yls = 0, yre = 0;  // stress / output window (pmcl3d.c:573-631)
  bool media_ready = false;
  bool elastic = false;  // Q^-1 == 0 everywhere and memory variables zero
  // sources
  int nsrc = 0, ncell = 0, src_stride = 0;
  int *d_cell_pos = nullptr, *d_cell_first = nullptr, *d_order = nullptr;
  float* d_src[6] = {};
  float* d_mom = nullptr;
  double* d_filt = nullptr;
  float* d_plane[3] = {};  // IFAULT 6 plane-wave series (x, y, z), plane_n samples each
  int plane_n = 0;
  // IFAULT 4: velocities prescribed at points (frcvel_cu), windows of frc_w
  // frames with one carry slot in front (pmcl3d.c:714-722, 792-805, 1821-1826)
  int frc_n = 0, frc_frames = 0, frc_tskp = 1, frc_w = 0, frc_next = 0;
  long long frc_s = 0;  // source_step of pmcl3d
  int* d_frc_pos = nullptr;
  float* d_frc[3] = {};
  float* h_frc = nullptr;  // pinned staging of one window, 3 * frc_w * frc_n
  cudaEvent_t frc_h2d = nullptr;
  bool frc_pending = false;
  awp_frame_reader frc_read = nullptr;
  void* frc_user = nullptr;
  // x-slab sub-domain of a decomposed grid: global width and offset of this
  // part (0 = the whole grid), and the caller's halo exchange hook
  int sub_nxg = 0, sub_x0 = 0;
  awp_exchange_fn xch = nullptr;
  void* xch_user = nullptr;
  // FOLLOWBATHY surface level per padded (i, j) column, [j][i] (pmcl3d.c:905-930)
  int* d_bathy = nullptr;
  std::vector<int> bathy;
  int filtorder = 0;
  double filt_b[AWP_MAXFILT] = {}, filt_a[AWP_MAXFILT] = {};
  // plasticity
  bool plast_ready = false;
  PlastParams pp{};
  unsigned char* d_neta_mult = nullptr;
  unsigned int* d_flag = nullptr;
  unsigned int* d_ext = nullptr;  // media extrema (6 float bit patterns)
  int* d_err = nullptr;           // pipeline-wait error word of the TMA kernels
  bool tma_ok = false;            // tensor maps encoded for this context
  int tma_promo = -1;             // L2 promotion the maps were encoded with
  TmaMaps vel_maps{}, str_maps{};
  long long cur_step = 0;
  bool initial_src_done = false;
  RecvState* recv = nullptr;     // RECVFILE receivers
  RecvState* sgt = nullptr;      // SGTFILE stress receivers
  RecvState* sgt_mat = nullptr;  // SGTFILE material output (one write)
  SrcFileState* srcf = nullptr;  // SOURCEFILE moment-tensor sources
  SrcFileState* forcef = nullptr;  // FORCEFILE boundary forces (curvilinear block)
  // curvilinear topography of the top grid (topo_t of the reference)
  awp::TopoMetrics* topo = nullptr;  // host metrics (point-set set-up)
  float* d_topo = nullptr;           // f arrays then g arrays, one allocation
  TopoArgs targs{};                  // device pointers and constants
  // NVE 3 on a curvilinear top grid: 0 = the reference's single-rank
  // behaviour (only the middle band is stress-updated, Cartesian), 1 = the
  // curvilinear stress everywhere before the plasticity return
  int topo_plastic_consistent = 0;
  // adjoint workspace, kept between gradient calls of the same size
  float* adj_slab = nullptr;
  size_t adj_slab_floats = 0;
  long long dev_bytes = 0;
  long long launches = 0;
  // phase timing
  bool profile = false;
  struct PhaseEv {
    int phase;
    cudaEvent_t a, b;
  };
  std::vector<PhaseEv> ev_used, ev_free;
};

namespace {

int ctx_alloc(awp_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(AWP_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  c->dev_bytes += (long long)bytes;
  return AWP_OK;
}

bool field_needed(const awp_params& p, int f) {
  if (f >= AWP_SIGMA2 && f <= AWP_YLDFAC) return p.nve == 3;
  return true;  // neta is always allocated (velbuffer reads it, pmcl3d.c:1218)
}

StrArgs make_str_args(awp_ctx* c) {
  StrArgs a;
  memset(&a, 0, sizeof(a));
  float** f = c->f;
  a.xx = f[AWP_XX]; a.yy = f[AWP_YY]; a.zz = f[AWP_ZZ];
  a.xy = f[AWP_XY]; a.xz = f[AWP_XZ]; a.yz = f[AWP_YZ];
  a.r1 = f[AWP_R1]; a.r2 = f[AWP_R2]; a.r3 = f[AWP_R3];
  a.r4 = f[AWP_R4]; a.r5 = f[AWP_R5]; a.r6 = f[AWP_R6];
  a.u1 = f[AWP_U1]; a.v1 = f[AWP_V1]; a.w1 = f[AWP_W1];
  a.lam = f[AWP_LAM]; a.mu = f[AWP_MU]; a.qp = f[AWP_QP]; a.qs = f[AWP_QS];
  a.dcrjx = c->dcrjx; a.dcrjy = c->dcrjy; a.dcrjz = c->dcrjz; a.lam_mu = c->lam_mu;
  a.tex = c->tex;
  memcpy(a.coeff, c->coeff, sizeof(a.coeff));
  a.slice = c->g.slice;
  a.yline = c->g.yline;
  a.lam_mu_ld = (int)c->g.ny_pad();
  a.i0 = c->xls; a.i1 = c->xre; a.j0 = c->yls; a.j1 = c->yre;
  // dstrqc: k from align+3 to maxk (kernel.cu:900-911); the free-surface
  // images belong to the top grid only
  a.k0 = AWP_ALIGN + 3;
  a.k1 = (c->p.grid == 0) ? c->g.top() : c->g.top() - 2;
  a.fs = (c->p.grid == 0) ? 1 : 0;
  a.ktop = c->g.top();
  // g_i < NX (rankx = 0): the global last column, in this part's indices
  a.gx_lim = (c->sub_nxg ? c->sub_nxg - c->sub_x0 : c->p.nx) + AWP_NGSL + 1;
  a.gy_min = (c->p.npc == 2) ? INT_MIN : AWP_NGSL + 3;     // g_j > 1 || NPC == 2
  a.dth = c->dth; a.dh1 = c->dh1; a.dt = c->p.dt; a.c1 = c->c1; a.c2 = c->c2;
  a.qthr = c->qthr;
  return a;
}

KinSrcArgs make_kin_args(awp_ctx* c, int step) {
  KinSrcArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = c->f[AWP_XX]; a.yy = c->f[AWP_YY]; a.zz = c->f[AWP_ZZ];
  a.xy = c->f[AWP_XY]; a.yz = c->f[AWP_YZ]; a.xz = c->f[AWP_XZ];
  a.mu = c->f[AWP_MU];
  a.cell_pos = c->d_cell_pos; a.cell_first = c->d_cell_first; a.order = c->d_order;
  a.axx = c->d_src[0]; a.ayy = c->d_src[1]; a.azz = c->d_src[2];
  a.axz = c->d_src[3]; a.ayz = c->d_src[4]; a.axy = c->d_src[5];
  a.mom = c->d_mom;
  a.filt_state = c->d_filt;
  a.filtorder = c->filtorder;
  memcpy(a.filt_b, c->filt_b, sizeof(a.filt_b));
  memcpy(a.filt_a, c->filt_a, sizeof(a.filt_a));
  a.ncell = c->ncell;
  a.step = step;
  a.dt = c->p.dt;
  a.vtst = (float)c->p.dt / (c->p.dh * c->p.dh * c->p.dh);
  return a;
}

SrcArgs make_src_args(awp_ctx* c, int tidx) {
  SrcArgs a;
  memset(&a, 0, sizeof(a));
  a.xx = c->f[AWP_XX]; a.yy = c->f[AWP_YY]; a.zz = c->f[AWP_ZZ];
  a.xy = c->f[AWP_XY]; a.yz = c->f[AWP_YZ]; a.xz = c->f[AWP_XZ];
  a.cell_pos = c->d_cell_pos; a.cell_first = c->d_cell_first; a.order = c->d_order;
  a.axx = c->d_src[0]; a.ayy = c->d_src[1]; a.azz = c->d_src[2];
  a.axz = c->d_src[3]; a.ayz = c->d_src[4]; a.axy = c->d_src[5];
  a.ncell = c->ncell;
  a.stride = c->src_stride;
  a.tidx = tidx;
  a.vtst = (float)c->p.dt / (c->p.dh * c->p.dh * c->p.dh);
  return a;
}

int launch_sources(awp_ctx* c, int tidx) {
  if (c->ncell == 0) return AWP_OK;
  if (c->p.ifault == 5)
    CU_TRY(awp_launch_addkinsrc(make_kin_args(c, tidx), c->stream));
  else
    CU_TRY(awp_launch_addsrc(make_src_args(c, tidx), c->stream));
  return AWP_OK;
}

int launch_plasticity(awp_ctx* c) {
  // Yield factor over the union of the five strip launches of pmcl3d.c:2121-2181
  // (xlsp..xrep x ylsp..yrep at one rank); neta counts each strip visit.
  PlastCalcArgs a;
  memset(&a, 0, sizeof(a));
  float** f = c->f;
  a.xx = f[AWP_XX]; a.yy = f[AWP_YY]; a.zz = f[AWP_ZZ];
  a.xy = f[AWP_XY]; a.xz = f[AWP_XZ]; a.yz = f[AWP_YZ];
  a.mu = f[AWP_MU]; a.d1 = f[AWP_D1]; a.sigma2 = f[AWP_SIGMA2];
  a.cohes = f[AWP_COHES]; a.phi = f[AWP_PHI];
  a.yldfac = f[AWP_YLDFAC]; a.neta = f[AWP_NETA];
  a.neta_mult = c->d_neta_mult;
  a.neta_ld = (int)c->g.ny_pad();
  a.p = c->pp;
  a.slice = c->g.slice; a.yline = c->g.yline;
  a.i0 = c->xls; a.i1 = c->xre; a.j0 = c->yls; a.j1 = c->yre;
  a.k0 = AWP_ALIGN;
  a.k1 = AWP_ALIGN + round_up(c->g.nzt, 4) - 1;
  CU_TRY(awp_launch_plast_calc(a, c->stream));
  return AWP_OK;
}

// drprecpc_app (kernel.cu:1650-1778) over the same window: reads the yield
// factors of the cell and of its -x, +y, +z neighbours
int launch_plast_app(awp_ctx* c) {
  float** f = c->f;
  PlastAppArgs b;
  memset(&b, 0, sizeof(b));
  b.xx = f[AWP_XX]; b.yy = f[AWP_YY]; b.zz = f[AWP_ZZ];
  b.xy = f[AWP_XY]; b.xz = f[AWP_XZ]; b.yz = f[AWP_YZ];
  b.mu = f[AWP_MU]; b.sigma2 = f[AWP_SIGMA2]; b.yldfac = f[AWP_YLDFAC];
  b.p = c->pp;
  b.slice = c->g.slice; b.yline = c->g.yline;
  b.i0 = c->xls; b.i1 = c->xre; b.j0 = c->yls;
  b.j1 = c->yls + round_up(c->yre - c->yls + 1, 2) - 1;  // grid rounds j up (kernel.cu:1451)
  b.k0 = AWP_ALIGN;
  b.k1 = AWP_ALIGN + round_up(c->g.nzt, 4) - 1;
  CU_TRY(awp_launch_plast_app(b, c->stream));
  return AWP_OK;
}

// Tensor maps over the context's fields for the TMA-pipelined kernels.
bool build_tma_maps(awp_ctx* c) {
  int hx, hy, mx, my, ox, oy, jx, jy, kx, ky;
  awp_tma_box(0, &hx, &hy);
  awp_tma_box(1, &mx, &my);
  awp_tma_box(2, &ox, &oy);
  awp_tma_box(3, &jx, &jy);
  awp_tma_box(4, &kx, &ky);
  float** f = c->f;
  const int vh[6] = {AWP_XX, AWP_YY, AWP_ZZ, AWP_XY, AWP_XZ, AWP_YZ};
  const int vo[3] = {AWP_U1, AWP_V1, AWP_W1};
  const int sm[4] = {AWP_LAM, AWP_MU, AWP_QP, AWP_QS};
  const int so[12] = {AWP_XX, AWP_YY, AWP_ZZ, AWP_XY, AWP_XZ, AWP_YZ,
                      AWP_R1, AWP_R2, AWP_R3, AWP_R4, AWP_R5, AWP_R6};
  int bad = 0;
  // velocity: each stress field with the halo its differences read
  const int vbx[6] = {ox, jx, kx, jx, kx, hx}, vby[6] = {oy, jy, ky, jy, ky, hy};
  for (int q = 0; q < 6; ++q)
    bad |= awp_tma_encode(&c->vel_maps.halo[q], f[vh[q]], c->g, vbx[q], vby[q]);
  bad |= awp_tma_encode(&c->vel_maps.media[0], f[AWP_D1], c->g, mx, my);
  for (int q = 0; q < 3; ++q) bad |= awp_tma_encode(&c->vel_maps.own[q], f[vo[q]], c->g, ox, oy);
  for (int q = 0; q < 3; ++q) bad |= awp_tma_encode(&c->str_maps.halo[q], f[vo[q]], c->g, hx, hy);
  for (int q = 0; q < 4; ++q) bad |= awp_tma_encode(&c->str_maps.media[q], f[sm[q]], c->g, mx, my);
  for (int q = 0; q < 12; ++q) bad |= awp_tma_encode(&c->str_maps.own[q], f[so[q]], c->g, ox, oy);
  return bad == 0;
}

// The maps carry the process-wide L2 promotion of the moment they were
// encoded; a tuning change re-encodes them before the next TMA launch (host
// only: the fields and boxes stay the same, so results are unchanged).
bool tma_ready(awp_ctx* c) {
  const int promo = awp_tuning_get("l2_promotion");
  if (c->tma_promo != promo) {
    c->tma_ok = build_tma_maps(c);
    c->tma_promo = promo;
  }
  return c->tma_ok;
}

struct PhaseScope {
  awp_ctx* c;
  awp_ctx::PhaseEv ev{};
  bool on;
  PhaseScope(awp_ctx* c_, int phase) : c(c_), on(c_->profile) {
    if (!on) return;
    if (c->ev_free.empty()) {
      awp_ctx::PhaseEv e{};
      cudaEventCreate(&e.a);
      cudaEventCreate(&e.b);
      c->ev_free.push_back(e);
    }
    ev = c->ev_free.back();
    c->ev_free.pop_back();
    ev.phase = phase;
    cudaEventRecord(ev.a, c->stream);
  }
  ~PhaseScope() {
    if (!on) return;
    cudaEventRecord(ev.b, c->stream);
    c->ev_used.push_back(ev);
  }
};

// ---- one time step in phases (pmcl3d.c:1628-2487 at one rank) --------------
// A single grid runs them in order (one_step); a discontinuous mesh
// interleaves them with the coupling kernels (mesh_step).

// The step-1 source sample is added before the loop (pmcl3d.c:1175-1187).
int initial_source(awp_ctx* c) {
  if (c->cur_step == 0 && !c->initial_src_done) {
    if (c->p.ifault < 4) {
      int s = launch_sources(c, 0);
      if (s) return s;
      if (c->ncell) c->launches++;
    }
    c->initial_src_done = true;
  }
  return AWP_OK;
}

int phase_begin(awp_ctx* c) {
  const int s = initial_source(c);
  if (s) return s;
  c->cur_step += 1;
  return AWP_OK;
}

// Kernel arguments of the curvilinear half-steps: the wavefield, media and
// texture of the context plus the metric arrays of awp_topography_init.
TopoArgs topo_args(awp_ctx* c) {
  TopoArgs a = c->targs;
  float** f = c->f;
  a.u1 = f[AWP_U1]; a.v1 = f[AWP_V1]; a.w1 = f[AWP_W1];
  a.xx = f[AWP_XX]; a.yy = f[AWP_YY]; a.zz = f[AWP_ZZ];
  a.xy = f[AWP_XY]; a.xz = f[AWP_XZ]; a.yz = f[AWP_YZ];
  a.r1 = f[AWP_R1]; a.r2 = f[AWP_R2]; a.r3 = f[AWP_R3];
  a.r4 = f[AWP_R4]; a.r5 = f[AWP_R5]; a.r6 = f[AWP_R6];
  a.d1 = f[AWP_D1]; a.lam = f[AWP_LAM]; a.mu = f[AWP_MU]; a.qp = f[AWP_QP]; a.qs = f[AWP_QS];
  a.dcrjx = c->dcrjx; a.dcrjy = c->dcrjy; a.dcrjz = c->dcrjz;
  a.tex = c->tex;
  memcpy(a.coeff, c->coeff, sizeof(a.coeff));
  a.qthr = c->qthr;
  a.slice = c->g.slice; a.yline = c->g.yline;
  a.nx = c->g.nxt; a.ny = c->g.nyt; a.nz = c->g.nzt;
  return a;
}

VelArgs make_vel_args(awp_ctx* c) {
  float** f = c->f;
  VelArgs v;
  v.u1 = f[AWP_U1]; v.v1 = f[AWP_V1]; v.w1 = f[AWP_W1];
  v.xx = f[AWP_XX]; v.yy = f[AWP_YY]; v.zz = f[AWP_ZZ];
  v.xy = f[AWP_XY]; v.xz = f[AWP_XZ]; v.yz = f[AWP_YZ];
  v.dcrjx = c->dcrjx; v.dcrjy = c->dcrjy; v.dcrjz = c->dcrjz; v.d1 = f[AWP_D1];
  v.slice = c->g.slice; v.yline = c->g.yline;
  v.i0 = 2 + AWP_NGSL; v.i1 = c->g.nxt + AWP_NGSL + 1;          // xvs..xve
  v.j0 = 2 + AWP_NGSL; v.j1 = 2 + AWP_NGSL + round_up(c->g.nyt, 2) - 1;
  // dvelcx_opt leaves the interface layers of a mesh to dvelc2 / intp3d /
  // swap3: k <= nzt+align-3 below the top grid, k >= align+3 above the
  // bottom grid (kernel.cu:146-147)
  v.k0 = (c->p.grid < c->p.ngrids - 1) ? AWP_ALIGN + 3 : AWP_ALIGN;
  v.k1 = AWP_ALIGN + round_up(c->g.nzt, 4) - 1;
  if (c->p.grid > 0) v.k1 = std::min(v.k1, c->g.nzt + AWP_ALIGN - 3);
  v.dth = c->dth; v.c1 = c->c1; v.c2 = c->c2;
  return v;
}

int phase_velocity(awp_ctx* c) {
  const VelArgs v = make_vel_args(c);
  if (c->topo) {  // topo_velocity_*_H replace dvelc[xy] on the top grid (pmcl3d.c:1661-1698)
    PhaseScope ps(c, 0);
    CU_TRY(awp_launch_topo_velocity(topo_args(c), c->stream));
    c->launches++;
    return AWP_OK;
  }
  const bool tma = awp_tuning_get("tma_vel") == 1 && tma_ready(c);
  PhaseScope ps(c, 0);
  if (tma)
    CU_TRY(awp_launch_velocity_tma(v, c->vel_maps, awp_tuning_get("ichunk"), c->d_err,
                                   c->stream));
  else
    CU_TRY(awp_launch_velocity(v, c->stream));
  c->launches++;
  return AWP_OK;
}

// Middle band of the NVE = 3 stress split at one rank: xss2..xse2 x
// yls2..yre2 (pmcl3d.c:573-631; ylsp = yls, yrep = yre at one rank).
void middle_band(const awp_ctx* c, int* i0, int* i1, int* j0, int* j1) {
  const int yls = c->yls, yre = c->yre;
  int yls2 = (int)(yls + (int)(yre - yls) * 0.25);
  if (yls2 % 2 != 0) yls2 += 1;
  int yre2 = (int)(yls + (int)(yre - yls) * 0.75);
  if (yre2 % 2 == 0) yre2 -= 1;
  // x range of the whole grid, in this part's indices when it is a sub-domain
  const int x0 = c->sub_nxg ? c->sub_x0 : 0, nxg = c->sub_nxg ? c->sub_nxg : c->g.nxt;
  *i0 = std::max(AWP_NGSL + 4 - x0, c->sub_nxg ? c->xls : 0);
  *i1 = std::min(nxg + AWP_NGSL - 1 - x0, c->sub_nxg ? c->xre : INT_MAX);
  *j0 = std::max(yls2, yls + AWP_NGSL + 2);
  *j1 = std::min(yre2, yre - AWP_NGSL - 2);
}

// Cartesian stress (+ memory variables) over i0..i1 x j0..j1 of the stress
// window, with the kernel family the tuning selects.
int launch_cart_stress(awp_ctx* c, int i0, int i1, int j0, int j1) {
  if (i1 < i0 || j1 < j0) return AWP_OK;
  const bool tma = awp_tuning_get("tma_str") == 1 && tma_ready(c);
  StrArgs s = make_str_args(c);
  s.i0 = i0; s.i1 = i1; s.j0 = j0; s.j1 = j1;
  if (tma)
    CU_TRY(awp_launch_stress_tma(s, c->str_maps, c->elastic, awp_tuning_get("ichunk"),
                                 c->d_err, c->stream));
  else
    CU_TRY(awp_launch_stress(s, c->elastic, c->stream));
  c->launches++;
  return AWP_OK;
}

// NVE = 3 splits the stress update (pmcl3d.c:1858-1924, 2139-2148): the
// middle band xss2..xse2 x yls2..yre2 is updated in the plasticity section,
// after the sources and the mesh-interface exchanges, the rest here.  On a
// curvilinear grid 0 the reference at one rank runs no other stress at all:
// its band loops start at grid `usetopo` (pmcl3d.c:1858-1879), the interior
// topography stress belongs to the NVE < 3 branch (:1855) and
// topo_stress_left/right_H return without a neighbour rank
// (src/topography/stress_attenuation.cu:323-325, 430-432).
bool stress_split(const awp_ctx* c) {
  return c->p.nve == 3 && (!c->topo || !c->topo_plastic_consistent);
}

int phase_stress(awp_ctx* c) {
  if (c->topo && c->p.nve == 3 && !c->topo_plastic_consistent) return AWP_OK;
  if (c->topo) {  // topo_stress_*_H replace dstrqc on the top grid (pmcl3d.c:1843-1924)
    PhaseScope ps(c, 1);
    CU_TRY(awp_launch_topo_stress(topo_args(c), c->elastic, c->stream));
    c->launches++;
    return AWP_OK;
  }
  PhaseScope ps(c, 1);
  if (!stress_split(c)) return launch_cart_stress(c, c->xls, c->xre, c->yls, c->yre);
  int i0, i1, j0, j1, st;
  middle_band(c, &i0, &i1, &j0, &j1);
  if ((st = launch_cart_stress(c, i0, i1, c->yls, j0 - 1))) return st;  // xss2, front
  if ((st = launch_cart_stress(c, i0, i1, j1 + 1, c->yre))) return st;  // xss2, back
  if ((st = launch_cart_stress(c, c->xls, i0 - 1, c->yls, c->yre))) return st;  // xss1
  return launch_cart_stress(c, i1 + 1, c->xre, c->yls, c->yre);                 // xss3
}

int phase_sources(awp_ctx* c) {
  float** f = c->f;
  if (c->srcf) {  // sources_read + sources_add_cartesian (pmcl3d.c:1987-2004)
    PhaseScope ps(c, 2);
    float* const stress[6] = {f[AWP_XX], f[AWP_YY], f[AWP_ZZ], f[AWP_XY], f[AWP_XZ], f[AWP_YZ]};
    if (awp_srcf_read(c->srcf, c->cur_step, c->stream, g_errmsg, sizeof(g_errmsg)) ||
        awp_srcf_add(c->srcf, c->cur_step, stress, c->stream, &c->launches, g_errmsg,
                     sizeof(g_errmsg)))
      return AWP_ERR_IO;
  }
  if (c->forcef) {  // forces_read + forces_add after the moments (pmcl3d.c:1989-1994)
    PhaseScope ps(c, 2);
    float* const vel[3] = {f[AWP_U1], f[AWP_V1], f[AWP_W1]};
    if (awp_srcf_read(c->forcef, c->cur_step, c->stream, g_errmsg, sizeof(g_errmsg)) ||
        awp_forcef_add(c->forcef, c->cur_step, vel, f[AWP_D1], c->stream, &c->launches,
                       g_errmsg, sizeof(g_errmsg)))
      return AWP_ERR_IO;
  }
  if ((c->p.ifault < 4 && c->cur_step < c->p.nst) || c->p.ifault == 5) {
    PhaseScope ps(c, 2);
    int st = launch_sources(c, (int)c->cur_step);
    if (st) return st;
    if (c->ncell) c->launches++;
  }
  // IFAULT 6: addplanesrc_H(cur_step, ...) while cur_step < NST, on the grid
  // that holds the plane wave (the bottom one, pmcl3d.c:2035-2041); the loop
  // counter starts at 1, so sample 0 of the series is never applied
  if (c->p.ifault == 6 && c->plane_n > 0 && c->cur_step < c->plane_n) {
    PhaseScope ps(c, 2);
    PlaneSrcArgs a;
    a.n = (int)c->cur_step;
    a.nx = c->p.nx + 4 + (c->p.nx % 2);  // rows of the shipped 2 x 2 launch blocks
    a.ny = c->p.ny + 4 + (c->p.ny % 2);
    a.k = AWP_ALIGN + c->p.nd + 1;
    a.mu = c->f[AWP_MU]; a.lambda = c->f[AWP_LAM];
    a.axx = c->d_plane[0]; a.ayy = c->d_plane[1]; a.azz = c->d_plane[2];
    a.xx = c->f[AWP_XX]; a.yy = c->f[AWP_YY]; a.zz = c->f[AWP_ZZ];
    a.xz = c->f[AWP_XZ]; a.yz = c->f[AWP_YZ];
    a.slice = c->g.slice; a.yline = c->g.yline;
    a.DT = c->p.dt; a.DH = c->p.dh;
    CU_TRY(awp_launch_planesrc(a, c->stream));
    c->launches++;
  }
  return AWP_OK;
}

// The caller's halo exchange of a sub-domain (awp_set_exchange): at the start
// of a step the stresses and velocities (the last step's stress update wrote
// the free-surface velocity images, and the first step's starts from the
// source sample added before the loop), after the velocity update the
// velocities.
int exchange(awp_ctx* c, int set) {
  if (!c->xch) return AWP_OK;
  const int r = c->xch(c->xch_user, set);
  if (r) return set_error(AWP_ERR_IO, "halo exchange hook failed (%d)", r);
  return AWP_OK;
}

int phase_plasticity(awp_ctx* c) {
  if (c->p.nve != 3) return AWP_OK;
  int st;
  if (stress_split(c)) {  // the middle band of the stress split (pmcl3d.c:2139-2148)
    PhaseScope ps(c, 1);
    int i0, i1, j0, j1;
    middle_band(c, &i0, &i1, &j0, &j1);
    if ((st = launch_cart_stress(c, i0, i1, j0, j1))) return st;
  }
  PhaseScope ps(c, 3);
  // a sub-domain's ghost planes take the neighbours' updated stresses (the
  // yield factor averages xz and xy over x) and then their yield factors
  // (the return averages them over x)
  if ((st = exchange(c, AWP_HALO_STRESS))) return st;
  if ((st = launch_plasticity(c))) return st;
  c->launches++;
  if ((st = exchange(c, AWP_HALO_YLDFAC))) return st;
  if ((st = launch_plast_app(c))) return st;
  c->launches++;
  return AWP_OK;
}

FstrArgs make_fstr_args(awp_ctx* c) {
  float** f = c->f;
  FstrArgs fs;
  fs.zz = f[AWP_ZZ]; fs.xz = f[AWP_XZ]; fs.yz = f[AWP_YZ];
  fs.slice = c->g.slice; fs.yline = c->g.yline; fs.ktop = c->g.top();
  fs.i0 = c->xls; fs.i1 = c->xre;
  fs.j0 = c->yls; fs.j1 = c->yls + round_up(c->yre - c->yls + 1, 2) - 1;
  return fs;
}

int phase_fstr(awp_ctx* c) {
  if (c->p.grid != 0) return AWP_OK;  // fstr_H on grid 0 only (pmcl3d.c:2243)
  const FstrArgs fs = make_fstr_args(c);
  PhaseScope ps(c, 4);
  CU_TRY(awp_launch_fstr(fs, c->stream));
  c->launches++;
  return AWP_OK;
}

// sgt_write (receivers/sgt.c:92-127) of the six stresses at the current step
int sgt_record(awp_ctx* c) {
  float** f = c->f;
  const float* const stress[6] = {f[AWP_XX], f[AWP_YY], f[AWP_ZZ],
                                  f[AWP_XY], f[AWP_XZ], f[AWP_YZ]};
  if (c->sgt && awp_recv_record_fields(c->sgt, c->cur_step, stress, c->stream, &c->launches,
                                       g_errmsg, sizeof(g_errmsg)))
    return AWP_ERR_IO;
  return AWP_OK;
}

int phase_receivers(awp_ctx* c) {
  float** f = c->f;
  if (c->recv &&  // receivers_write (pmcl3d.c:2246-2247)
      awp_recv_record(c->recv, c->cur_step, f[AWP_U1], f[AWP_V1], f[AWP_W1], c->stream,
                      &c->launches, g_errmsg, sizeof(g_errmsg)))
    return AWP_ERR_IO;
  return sgt_record(c);  // pmcl3d.c:2248-2249
}

// IFAULT 4: the next window of frames from the caller's reader into slots
// 1..frc_w of the device arrays (read_src_ifault_4 + Cpy2Device_source,
// source.c:469-680, swap.c:323-353); slot 0 carries the last frame of the
// window before, which frcvel_cu itself moves there.
int frc_fill(awp_ctx* c) {
  if (c->frc_pending) {  // the staging buffer of the window before has been copied
    CU_TRY(cudaEventSynchronize(c->frc_h2d));
    c->frc_pending = false;
  }
  const size_t n = (size_t)c->frc_w * c->frc_n;
  float* h = c->h_frc;
  const int first = c->frc_next * c->frc_w;
  const int r = c->frc_read(c->frc_user, first, c->frc_w, h, h + n, h + 2 * n);
  if (r) return set_error(AWP_ERR_IO, "velocity frame reader failed on frames %d..%d (%d)", first,
                          first + c->frc_w - 1, r);
  for (int q = 0; q < 3; ++q)
    CU_TRY(cudaMemcpyAsync(c->d_frc[q] + c->frc_n, h + (size_t)q * n, n * sizeof(float),
                           cudaMemcpyHostToDevice, c->stream));
  CU_TRY(cudaEventRecord(c->frc_h2d, c->stream));
  c->frc_pending = true;
  c->frc_next++;
  return AWP_OK;
}

// frcvel_H on grid 0 after the velocity update and its mesh coupling
// (pmcl3d.c:1821-1826): the step counter advances, then the kernel sets (or,
// past the last frame, pushes) the velocities at the points.
int phase_forcing(awp_ctx* c) {
  if (!c->d_frc_pos) return AWP_OK;
  PhaseScope ps(c, 2);
  c->frc_s += 1;
  FrcvelArgs a;
  memset(&a, 0, sizeof(a));
  a.i = (int)c->frc_s;
  a.read_step = c->frc_w;
  a.dim = 3;
  a.npsrc = c->frc_n;
  a.tskp = c->frc_tskp;
  a.xmin = -1;
  a.xmax = -1;
  a.psrc = c->d_frc_pos;
  a.axx = c->d_frc[0]; a.ayy = c->d_frc[1]; a.azz = c->d_frc[2];
  a.u1 = c->f[AWP_U1]; a.v1 = c->f[AWP_V1]; a.w1 = c->f[AWP_W1];
  a.slice = c->g.slice; a.yline = c->g.yline;
  a.DT = c->p.dt;
  CU_TRY(awp_launch_frcvel(a, c->stream));
  c->launches++;
  return AWP_OK;
}

// End of a step: a new window every frc_w * tskp steps while frames remain,
// and the step counter restarts (pmcl3d.c:2442-2486).
int phase_forcing_window(awp_ctx* c) {
  if (!c->d_frc_pos) return AWP_OK;
  const long long cs = c->cur_step, wt = (long long)c->frc_w * c->frc_tskp;
  if (cs < (long long)c->frc_frames * c->frc_tskp - 1 && (cs + 1) % wt == 0) {
    const int st = frc_fill(c);
    if (st) return st;
    c->frc_s = 0;
  }
  return AWP_OK;
}

int one_step(awp_ctx* c) {
  int st;
  if ((st = phase_begin(c))) return st;
  if ((st = exchange(c, AWP_HALO_VELOCITY | AWP_HALO_STRESS))) return st;
  if ((st = phase_velocity(c))) return st;
  if ((st = phase_forcing(c))) return st;
  if ((st = exchange(c, AWP_HALO_VELOCITY))) return st;
  if ((st = phase_stress(c))) return st;
  if ((st = phase_sources(c))) return st;
  if ((st = phase_plasticity(c))) return st;
  if ((st = phase_fstr(c))) return st;
  if ((st = phase_receivers(c))) return st;
  return phase_forcing_window(c);
}

// Fields of a halo set, in enum order.
int halo_fields(int set, int* out) {
  int n = 0;
  if (set & AWP_HALO_VELOCITY)
    for (int f = AWP_U1; f <= AWP_W1; ++f) out[n++] = f;
  if (set & AWP_HALO_STRESS)
    for (int f = AWP_XX; f <= AWP_YZ; ++f) out[n++] = f;
  if (set & AWP_HALO_MEDIA)
    for (int f = AWP_D1; f <= AWP_QS; ++f) out[n++] = f;
  if (set & AWP_HALO_YLDFAC) out[n++] = AWP_YLDFAC;
  return n;
}

// First plane of a halo: the `planes` interior planes next to `side` (send),
// or the ghost planes beyond it (receive).
long long halo_plane(const awp_ctx* c, int side, bool ghost, int planes) {
  const long long lo = 2 + AWP_NGSL, hi = c->p.nx + 2 + AWP_NGSL;  // first / one-past interior
  if (side == 0) return ghost ? lo - planes : lo;
  return ghost ? hi : hi - planes;
}

}  // namespace

namespace {

DmGrid dm_grid(awp_ctx* c) {
  DmGrid g;
  float** f = c->f;
  g.u1 = f[AWP_U1]; g.v1 = f[AWP_V1]; g.w1 = f[AWP_W1];
  g.xx = f[AWP_XX]; g.yy = f[AWP_YY]; g.zz = f[AWP_ZZ];
  g.xy = f[AWP_XY]; g.xz = f[AWP_XZ]; g.yz = f[AWP_YZ];
  g.nxt = c->g.nxt; g.nyt = c->g.nyt; g.nzt = c->g.nzt;
  g.slice = c->g.slice; g.yline = c->g.yline;
  return g;
}

int dm_interfaces(awp_ctx* const* g, int n, cudaStream_t st) {
  for (int p = 1; p < n; ++p) {  // coarse -> fine (pmcl3d.c:1767-1772, 2057-2062)
    DmPairArgs a{dm_grid(g[p]), dm_grid(g[p - 1])};
    CU_TRY(awp_launch_intp3d(a, st));
    g[p]->launches++;
  }
  for (int p = 0; p < n - 1; ++p) {  // fine -> coarse (pmcl3d.c:1802-1806, 2085-2090)
    DmPairArgs a{dm_grid(g[p + 1]), dm_grid(g[p])};
    CU_TRY(awp_launch_swap3(a, st));
    g[p]->launches++;
  }
  return AWP_OK;
}

int dm_velocity(awp_ctx* c) {  // dvelc2 (pmcl3d.c:1729-1732)
  DmVel2Args a;
  a.g = dm_grid(c);
  a.d1 = c->f[AWP_D1];
  a.dcrjx = c->dcrjx; a.dcrjy = c->dcrjy; a.dcrjz = c->dcrjz;
  a.dth = c->dth;
  CU_TRY(awp_launch_dvelc2(a, c->stream));
  c->launches++;
  return AWP_OK;
}

int dm_stress(awp_ctx* c) {  // dstrqc2 over xss1..xse3 x yls..yre (pmcl3d.c:1936-1948)
  DmStr2Args a;
  memset(&a, 0, sizeof(a));
  float** f = c->f;
  a.g = dm_grid(c);
  a.r1 = f[AWP_R1]; a.r2 = f[AWP_R2]; a.r3 = f[AWP_R3];
  a.r4 = f[AWP_R4]; a.r5 = f[AWP_R5]; a.r6 = f[AWP_R6];
  a.lam = f[AWP_LAM]; a.mu = f[AWP_MU]; a.qp = f[AWP_QP]; a.qs = f[AWP_QS];
  a.dcrjx = c->dcrjx; a.dcrjy = c->dcrjy; a.dcrjz = c->dcrjz;
  a.tex = c->tex;
  memcpy(a.coeff, c->coeff, sizeof(a.coeff));
  a.i0 = c->xls; a.i1 = c->xre; a.j0 = c->yls; a.j1 = c->yre;
  a.dth = c->dth; a.dh1 = c->dh1; a.dt = c->p.dt;
  CU_TRY(awp_launch_dstrqc2(a, c->stream));
  c->launches++;
  return AWP_OK;
}

}  // namespace

struct awp_mesh {
  int ngrids = 0;
  awp_ctx* g[AWP_MAXGRIDS] = {};
  cudaStream_t stream = nullptr;      // the stream every block runs on
  cudaStream_t own_stream = nullptr;  // created with the mesh, destroyed with it
  bool prepared = false;
};

namespace {

// checkmesh of the media (pmcl3d.c:892-899): the coarse grid's top three
// levels take the finer grid's values; then each grid's elastic
// specialisation is decided on the corrected Q.
int mesh_prepare(awp_mesh* m) {
  for (int p = 0; p < m->ngrids; ++p)
    if (!m->g[p]->media_ready)
      return set_error(AWP_ERR_STATE, "grid %d has no media (awp_upload_media first)", p);
  for (int p = 1; p < m->ngrids; ++p) {
    awp_ctx *lo = m->g[p], *hi = m->g[p - 1];
    DmCheckArgs a;
    const int fid[5] = {AWP_D1, AWP_MU, AWP_LAM, AWP_QP, AWP_QS};
    for (int q = 0; q < 5; ++q) {
      a.lo[q] = lo->f[fid[q]];
      a.hi[q] = hi->f[fid[q]];
    }
    a.nf = 5;
    a.glo = dm_grid(lo);
    a.ghi = dm_grid(hi);
    CU_TRY(awp_launch_checkmesh(a, m->stream));
  }
  for (int p = 1; p < m->ngrids; ++p) {
    awp_ctx* c = m->g[p];
    unsigned int hflag = 1;
    CU_TRY(cudaMemsetAsync(c->d_flag, 0, sizeof(unsigned int), m->stream));
    CU_TRY(awp_launch_anynonzero(c->f[AWP_QP], c->g.cells_pad(), c->d_flag, m->stream));
    CU_TRY(awp_launch_anynonzero(c->f[AWP_QS], c->g.cells_pad(), c->d_flag, m->stream));
    CU_TRY(cudaMemcpyAsync(&hflag, c->d_flag, sizeof(hflag), cudaMemcpyDeviceToHost, m->stream));
    CU_TRY(cudaStreamSynchronize(m->stream));
    c->elastic = (hflag == 0);
  }
  m->prepared = true;
  return AWP_OK;
}

// One time step of the whole stack in pmcl3d's order (pmcl3d.c:1628-2490).
int mesh_step(awp_mesh* m) {
  awp_ctx* const* g = m->g;
  const int n = m->ngrids;
  int st;
  for (int p = 0; p < n; ++p)
    if ((st = phase_begin(g[p]))) return st;
  for (int p = 0; p < n; ++p)
    if ((st = phase_velocity(g[p]))) return st;
  for (int p = 0; p < n - 1; ++p)
    if ((st = dm_velocity(g[p]))) return st;
  if ((st = dm_interfaces(g, n, m->stream))) return st;
  if ((st = phase_forcing(g[0]))) return st;
  for (int p = 0; p < n; ++p)
    if ((st = phase_stress(g[p]))) return st;
  for (int p = 0; p < n - 1; ++p)
    if ((st = dm_stress(g[p]))) return st;
  for (int p = 0; p < n; ++p)
    if ((st = phase_sources(g[p]))) return st;
  if ((st = dm_interfaces(g, n, m->stream))) return st;
  for (int p = 0; p < n; ++p)
    if ((st = phase_plasticity(g[p]))) return st;
  if ((st = phase_fstr(g[0]))) return st;
  for (int p = 0; p < n; ++p)
    if ((st = phase_receivers(g[p]))) return st;
  return phase_forcing_window(g[0]);
}

}  // namespace

extern "C" {

void awp_params_default(awp_params* p) {
  memset(p, 0, sizeof(*p));
  p->nx = 256; p->ny = 256; p->nz = 1024;
  p->dh = 200.0f; p->dt = 0.01f;
  p->arbc = 0.92f; p->npc = 0; p->nd = 20;
  p->nve = 1;
  p->fac = 0.005f; p->q0 = 5.0f; p->ex = 0.0f; p->fp = 2.5f;
  p->socalq = 1;
  p->ifault = 1;
  p->nst = 91;
  p->read_step = 91;
  p->grid = 0;
  p->ngrids = 1;
}

const char* awp_status_string(int status) {
  switch (status) {
    case AWP_OK: return "ok";
    case AWP_ERR_ARG: return "invalid argument";
    case AWP_ERR_CUDA: return "CUDA error";
    case AWP_ERR_STATE: return "call out of order";
    case AWP_ERR_IO: return "I/O error";
    case AWP_ERR_NOMEM: return "out of memory";
    case AWP_ERR_NUMERIC: return "non-finite wavefield";
    case AWP_ERR_UNSUPPORTED: return "unsupported option";
  }
  return "unknown status";
}

const char* awp_last_error(void) { return g_errmsg; }

int awp_ctx_destroy(awp_ctx* c) {
  if (!c) return AWP_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  awp_recv_destroy(c->recv);
  awp_recv_destroy(c->sgt);
  awp_recv_destroy(c->sgt_mat);
  awp_srcf_destroy(c->srcf);
  awp_srcf_destroy(c->forcef);
  delete c->topo;
  cudaFree(c->d_topo);
  cudaFree(c->adj_slab);
  for (int i = 0; i < AWP_NFIELDS; ++i) cudaFree(c->f[i]);
  cudaFree(c->dcrjx); cudaFree(c->dcrjy); cudaFree(c->dcrjz); cudaFree(c->lam_mu);
  cudaFree(c->d_cell_pos); cudaFree(c->d_cell_first); cudaFree(c->d_order);
  for (int i = 0; i < 6; ++i) cudaFree(c->d_src[i]);
  cudaFree(c->d_mom); cudaFree(c->d_filt); cudaFree(c->d_neta_mult); cudaFree(c->d_flag);
  for (int q = 0; q < 3; ++q) cudaFree(c->d_plane[q]);
  cudaFree(c->d_bathy);
  cudaFree(c->d_frc_pos);
  for (int q = 0; q < 3; ++q) cudaFree(c->d_frc[q]);
  if (c->h_frc) cudaFreeHost(c->h_frc);
  if (c->frc_h2d) cudaEventDestroy(c->frc_h2d);
  cudaFree(c->d_ext);
  cudaFree(c->d_err);
  for (auto& e : c->ev_used) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  for (auto& e : c->ev_free) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return AWP_OK;
}

int awp_ctx_create(const awp_params* p, awp_ctx** out) {
  if (!p || !out) return set_error(AWP_ERR_ARG, "null argument");
  *out = nullptr;
  if (p->nx < 4 || p->ny < 4 || p->nz < 8)
    return set_error(AWP_ERR_ARG, "grid %dx%dx%d too small", p->nx, p->ny, p->nz);
  if (p->nz % 4 != 0)
    return set_error(AWP_ERR_ARG, "NZ=%d is not divisible by 4 (pmcl3d.c:380-391)", p->nz);
  if (!(p->dh > 0) || !(p->dt > 0)) return set_error(AWP_ERR_ARG, "DH and DT must be > 0");
  if (p->ngrids < 1 || p->ngrids > AWP_MAXGRIDS || p->grid < 0 || p->grid >= p->ngrids)
    return set_error(AWP_ERR_ARG, "grid %d of %d (at most %d grids)", p->grid, p->ngrids,
                     AWP_MAXGRIDS);
  if (p->nve != 1 && p->nve != 3)
    return set_error(AWP_ERR_UNSUPPORTED,
                     "NVE=%d: the time loop runs only for NVE 1 or 3 (pmcl3d.c:1624)", p->nve);
  if (p->npc != 0 && p->npc != 2)
    return set_error(AWP_ERR_UNSUPPORTED, "NPC=%d (only 0 and 2 run the loop)", p->npc);
  if (p->ifault < 0 || p->ifault > 6 || p->ifault == 3)
    return set_error(AWP_ERR_UNSUPPORTED, "IFAULT=%d", p->ifault);
  const long long cells = (long long)(p->nx + 20) * (p->ny + 20) * (p->nz + 64);
  if (cells >= (1LL << 31))
    return set_error(AWP_ERR_ARG, "padded grid of %lld cells exceeds the 32-bit index range", cells);

  awp_ctx* c = new awp_ctx();
  c->p = *p;
  c->g = awp_make_geom(p->nx, p->ny, p->nz);
  c->xls = 2 + AWP_NGSL;
  c->xre = p->nx + AWP_NGSL + 1;
  c->yls = 2 + AWP_NGSL;
  c->yre = p->ny + AWP_NGSL + 1;
  c->dth = p->dt / p->dh;
  c->dh1 = 1.0 / p->dh;
  c->qthr = awp::qf_threshold();
  int st;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return set_error(AWP_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  c->own_stream = true;
  const size_t fbytes = sizeof(float) * (size_t)c->g.cells_pad();
  for (int i = 0; i < AWP_NFIELDS; ++i) {
    if (!field_needed(*p, i)) continue;
    if ((st = ctx_alloc(c, (void**)&c->f[i], fbytes))) goto fail;
    if (cudaMemsetAsync(c->f[i], 0, fbytes, c->stream) != cudaSuccess) {
      st = set_error(AWP_ERR_CUDA, "memset");
      goto fail;
    }
  }
  if (p->nve == 3) {
    // yldfac starts at 1 (pmcl3d.c:842-849)
    if (awp_launch_fill(c->f[AWP_YLDFAC], 1.0f, c->g.cells_pad(), c->stream) != cudaSuccess) {
      st = set_error(AWP_ERR_CUDA, "fill");
      goto fail;
    }
  }
  {
    const int nxp = (int)c->g.nx_pad(), nyp = (int)c->g.ny_pad(), nzp = (int)c->g.nz_pad();
    std::vector<float> cx(nxp, 1.0f), cy(nyp, 1.0f), cz(nzp, 1.0f);
    // the bottom sponge belongs to the lowest grid only (pmcl3d.c:1026-1028)
    awp::inicrj(p->arbc, p->nx, p->ny, p->nz, p->nx, p->ny, p->nd,
                p->grid == p->ngrids - 1 ? 1 : 0, p->npc, cx.data(),
                cy.data(), cz.data());
    if ((st = ctx_alloc(c, (void**)&c->dcrjx, nxp * sizeof(float)))) goto fail;
    if ((st = ctx_alloc(c, (void**)&c->dcrjy, nyp * sizeof(float)))) goto fail;
    if ((st = ctx_alloc(c, (void**)&c->dcrjz, nzp * sizeof(float)))) goto fail;
    if ((st = ctx_alloc(c, (void**)&c->lam_mu, (size_t)nxp * nyp * sizeof(float)))) goto fail;
    if (cudaMemcpy(c->dcrjx, cx.data(), nxp * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->dcrjy, cy.data(), nyp * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->dcrjz, cz.data(), nzp * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemsetAsync(c->lam_mu, 0, (size_t)nxp * nyp * 4, c->stream) != cudaSuccess) {
      st = set_error(AWP_ERR_CUDA, "sponge upload");
      goto fail;
    }
    if (!awp::tau_range(p->ex, p->fac, &c->taumax, &c->taumin)) {
      st = set_error(AWP_ERR_UNSUPPORTED, "EX=%g >= 0.95 has no relaxation-time range", p->ex);
      goto fail;
    }
    awp::tausub(c->taumin, c->taumax, c->tau8);
    awp::weights_sub(p->ex, p->fac, c->w8, c->coeff);
    awp::texture_tables(c->tau8, c->w8, p->dt, &c->tex);
    c->tex.xls = c->xls;
    c->tex.yls = c->yls;
    c->tex.ny = c->yre - c->yls + 1;
    c->tex.nzt = p->nz;
  }
  if ((st = ctx_alloc(c, (void**)&c->d_flag, sizeof(unsigned int)))) goto fail;
  if ((st = ctx_alloc(c, (void**)&c->d_ext, 6 * sizeof(unsigned int)))) goto fail;
  if ((st = ctx_alloc(c, (void**)&c->d_err, sizeof(int)))) goto fail;
  if (cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream) != cudaSuccess) {
    st = set_error(AWP_ERR_CUDA, "memset");
    goto fail;
  }
  c->tma_ok = build_tma_maps(c);
  c->tma_promo = awp_tuning_get("l2_promotion");
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    st = set_error(AWP_ERR_CUDA, "initialisation");
    goto fail;
  }
  *out = c;
  return AWP_OK;
fail:
  awp_ctx_destroy(c);
  return st;
}

int awp_set_stream(awp_ctx* c, void* s) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (c->own_stream && c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  c->own_stream = false;
  c->stream = (cudaStream_t)s;  // NULL selects the legacy default stream
  return AWP_OK;
}

int awp_padded_dims(const awp_ctx* c, long long dims[3]) {
  if (!c || !dims) return set_error(AWP_ERR_ARG, "null argument");
  dims[0] = c->g.nx_pad();
  dims[1] = c->g.ny_pad();
  dims[2] = c->g.nz_pad();
  return AWP_OK;
}

static int upload_media_impl(awp_ctx* c, int nvar, const float* media, bool device) {
  if (!c || !media) return set_error(AWP_ERR_ARG, "null argument");
  if (nvar != 3 && nvar != 5 && nvar != 8)
    return set_error(AWP_ERR_ARG, "NVAR=%d (mesh.c:122 reads 3, 5 or 8)", nvar);
  const size_t n = (size_t)c->p.nx * c->p.ny * c->p.nz * nvar;
  const float* dmedia = media;
  float* tmp = nullptr;
  if (!device) {
    CU_TRY(cudaMallocAsync((void**)&tmp, n * sizeof(float), c->stream));
    CU_TRY(cudaMemcpyAsync(tmp, media, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    dmedia = tmp;
  }
  MediaArgs a;
  memset(&a, 0, sizeof(a));
  a.media = dmedia;
  a.d1 = c->f[AWP_D1]; a.mu = c->f[AWP_MU]; a.lam = c->f[AWP_LAM];
  a.qp = c->f[AWP_QP]; a.qs = c->f[AWP_QS];
  memcpy(a.tau, c->tau8, sizeof(a.tau));
  memcpy(a.weights, c->w8, sizeof(a.weights));
  memcpy(a.coeff, c->coeff, sizeof(a.coeff));
  const float pi = 4. * atan(1.);
  a.w0 = 2 * pi * c->p.fp;
  a.facex = (float)pow((double)c->p.fac, (double)c->p.ex);
  a.nvar = nvar;
  a.var_offset = (nvar == 8) ? 3 : 0;
  a.nve = c->p.nve;
  a.socalq = c->p.socalq;
  a.nxt = c->p.nx; a.nyt = c->p.ny; a.nzt = c->p.nz;
  a.slice = c->g.slice; a.yline = c->g.yline;
  {
    const unsigned int init[6] = {0x7f800000u, 0u, 0x7f800000u, 0u, 0x7f800000u, 0u};
    CU_TRY(cudaMemcpyAsync(c->d_ext, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  }
  a.ext = c->d_ext;
  CU_TRY(awp_launch_media(a, c->stream));
  CU_TRY(awp_launch_media_borders(c->f[AWP_D1], c->f[AWP_MU], c->f[AWP_LAM], c->f[AWP_QP],
                                  c->f[AWP_QS], c->g, c->p.nve, c->stream));
  CU_TRY(awp_launch_lam_mu(c->f[AWP_LAM], c->f[AWP_MU], c->lam_mu, c->g, c->xls, c->xre,
                           c->yls, c->yre, c->stream));
  if (tmp) CU_TRY(cudaFreeAsync(tmp, c->stream));
  // Elastic specialisation: with Q^-1 identically zero the memory variables
  // stay zero and the anelastic update reduces exactly to the elastic one, so
  // the stress kernel may skip the six r arrays and the two Q arrays.
  CU_TRY(cudaMemsetAsync(c->d_flag, 0, sizeof(unsigned int), c->stream));
  CU_TRY(awp_launch_anynonzero(c->f[AWP_QP], c->g.cells_pad(), c->d_flag, c->stream));
  CU_TRY(awp_launch_anynonzero(c->f[AWP_QS], c->g.cells_pad(), c->d_flag, c->stream));
  unsigned int hflag = 1;
  CU_TRY(cudaMemcpyAsync(&hflag, c->d_flag, sizeof(hflag), cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  const bool any_q = hflag != 0;
  c->elastic = !any_q;
  c->media_ready = true;
  return AWP_OK;
}

int awp_media_extrema(awp_ctx* c, float vse[2], float vpe[2], float dde[2]) {
  if (!c || !vse || !vpe || !dde) return set_error(AWP_ERR_ARG, "null argument");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "no media uploaded");
  unsigned int h[6];
  CU_TRY(cudaMemcpyAsync(h, c->d_ext, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  float v[6];
  memcpy(v, h, sizeof(v));
  vse[0] = (h[0] == 0x7f800000u) ? 1.0e10f : v[0];
  vse[1] = v[1];
  vpe[0] = v[2];
  vpe[1] = v[3];
  dde[0] = v[4];
  dde[1] = v[5];
  return AWP_OK;
}

int awp_alloc_host_pinned(void** ptr, size_t bytes) {
  if (!ptr) return set_error(AWP_ERR_ARG, "null argument");
  cudaError_t e = cudaMallocHost(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return set_error(AWP_ERR_NOMEM, "cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return AWP_OK;
}

int awp_free_host_pinned(void* ptr) {
  CU_TRY(cudaFreeHost(ptr));
  return AWP_OK;
}

int awp_upload_media(awp_ctx* c, int nvar, const float* host_media) {
  return upload_media_impl(c, nvar, host_media, false);
}
int awp_upload_media_device(awp_ctx* c, int nvar, const float* dev_media) {
  return upload_media_impl(c, nvar, dev_media, true);
}

int awp_upload_plane_wave(awp_ctx* c, int nst, const float* vx, const float* vy,
                          const float* vz) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (c->p.ifault != 6) return set_error(AWP_ERR_STATE, "the context runs IFAULT=%d, not 6", c->p.ifault);
  if (nst < 1 || !vx || !vy || !vz) return set_error(AWP_ERR_ARG, "bad plane-wave series");
  if (nst != c->p.nst)
    return set_error(AWP_ERR_ARG, "the series holds %d samples, NST is %d (ini_plane_wave)", nst,
                     c->p.nst);
  const float* in[3] = {vx, vy, vz};
  for (int q = 0; q < 3; ++q) {
    cudaFree(c->d_plane[q]);
    c->d_plane[q] = nullptr;
  }
  c->plane_n = 0;
  int st;
  for (int q = 0; q < 3; ++q) {
    if ((st = ctx_alloc(c, (void**)&c->d_plane[q], (size_t)nst * 4))) return st;
    CU_TRY(cudaMemcpy(c->d_plane[q], in[q], (size_t)nst * 4, cudaMemcpyDefault));
  }
  c->plane_n = nst;
  return AWP_OK;
}

int awp_upload_sources(awp_ctx* c, int nsrc, const int* pos, const float* data) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (nsrc < 0 || (nsrc > 0 && (!pos || !data))) return set_error(AWP_ERR_ARG, "bad sources");
  const int rs = c->p.read_step;
  if ((c->p.ifault == 1 || c->p.ifault == 2) && rs < c->p.nst)
    return set_error(AWP_ERR_UNSUPPORTED,
                     "IFAULT=%d holds all NST samples on the device (READ_STEP >= NST)",
                     c->p.ifault);
  const int stride = (c->p.ifault == 5) ? 2 : rs;
  // group by target cell (file order kept inside a cell)
  std::map<long long, std::vector<int>> cells;
  for (int s = 0; s < nsrc; ++s) {
    // inisource (source.c:172-174, 228-230) then addsrc (source.c:285-287)
    const int x = pos[3 * s], y = pos[3 * s + 1], zf = pos[3 * s + 2];
    const int z = c->p.nz + 1 - zf;
    if (x < -1 || x > c->p.nx + 2 || y < -1 || y > c->p.ny + 2 || z < 1 || z > c->p.nz)
      continue;  // outside this rank's index window: skipped as inisource does
    const long long p = (long long)(x + 1 + AWP_NGSL) * c->g.slice +
                        (long long)(y + 1 + AWP_NGSL) * c->g.yline + (z + AWP_ALIGN - 1);
    cells[p].push_back(s);
  }
  std::vector<int> cpos, cfirst, order;
  for (auto& kv : cells) {
    cpos.push_back((int)kv.first);
    cfirst.push_back((int)order.size());
    for (int s : kv.second) order.push_back(s);
  }
  cfirst.push_back((int)order.size());
  // de-interleave the time series: [comp][nsrc][stride]
  std::vector<float> comp((size_t)6 * nsrc * stride);
  for (int s = 0; s < nsrc; ++s)
    for (int t = 0; t < stride; ++t)
      for (int q = 0; q < 6; ++q)
        comp[((size_t)q * nsrc + s) * stride + t] = data[((size_t)s * rs + t) * 6 + q];
  cudaFree(c->d_cell_pos); cudaFree(c->d_cell_first); cudaFree(c->d_order);
  for (int q = 0; q < 6; ++q) cudaFree(c->d_src[q]);
  cudaFree(c->d_mom);
  c->d_cell_pos = c->d_cell_first = c->d_order = nullptr;
  c->d_mom = nullptr;
  for (int q = 0; q < 6; ++q) c->d_src[q] = nullptr;
  c->nsrc = nsrc;
  c->ncell = (int)cpos.size();
  c->src_stride = stride;
  if (nsrc == 0) return AWP_OK;
  int st;
  if ((st = ctx_alloc(c, (void**)&c->d_cell_pos, cpos.size() * 4 + 4))) return st;
  if ((st = ctx_alloc(c, (void**)&c->d_cell_first, cfirst.size() * 4))) return st;
  if ((st = ctx_alloc(c, (void**)&c->d_order, order.size() * 4 + 4))) return st;
  CU_TRY(cudaMemcpy(c->d_cell_pos, cpos.data(), cpos.size() * 4, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(c->d_cell_first, cfirst.data(), cfirst.size() * 4, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(c->d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
  for (int q = 0; q < 6; ++q) {
    if ((st = ctx_alloc(c, (void**)&c->d_src[q], (size_t)nsrc * stride * 4))) return st;
    CU_TRY(cudaMemcpy(c->d_src[q], comp.data() + (size_t)q * nsrc * stride,
                      (size_t)nsrc * stride * 4, cudaMemcpyHostToDevice));
  }
  if (c->p.ifault == 5) {
    if ((st = ctx_alloc(c, (void**)&c->d_mom, (size_t)nsrc * 4))) return st;
    CU_TRY(cudaMemset(c->d_mom, 0, (size_t)nsrc * 4));
    if (c->filtorder > 0) {
      cudaFree(c->d_filt);
      c->d_filt = nullptr;
      const size_t b = (size_t)nsrc * (c->filtorder + 1) * sizeof(double);
      if ((st = ctx_alloc(c, (void**)&c->d_filt, b))) return st;
      CU_TRY(cudaMemset(c->d_filt, 0, b));
    }
  }
  return AWP_OK;
}

int awp_set_source_filter(awp_ctx* c, int order, const double* b, const double* a) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (order < 0 || order >= AWP_MAXFILT) return set_error(AWP_ERR_ARG, "filter order %d", order);
  c->filtorder = order;
  for (int i = 0; i <= order && order > 0; ++i) {
    c->filt_b[i] = b[i];
    c->filt_a[i] = a[i];
  }
  if (c->nsrc > 0 && c->p.ifault == 5 && order > 0) {
    cudaFree(c->d_filt);
    c->d_filt = nullptr;
    const size_t bytes = (size_t)c->nsrc * (order + 1) * sizeof(double);
    int st;
    if ((st = ctx_alloc(c, (void**)&c->d_filt, bytes))) return st;
    CU_TRY(cudaMemset(c->d_filt, 0, bytes));
  }
  return AWP_OK;
}

int awp_download_moment(awp_ctx* c, float* host_mom) {
  if (!c || !host_mom) return set_error(AWP_ERR_ARG, "null argument");
  if (!c->d_mom) return set_error(AWP_ERR_STATE, "no kinematic source");
  CU_TRY(cudaStreamSynchronize(c->stream));
  CU_TRY(cudaMemcpy(host_mom, c->d_mom, (size_t)c->nsrc * 4, cudaMemcpyDeviceToHost));
  return AWP_OK;
}

int awp_upload_plasticity(awp_ctx* c, const float* sigma2, const float* cohes,
                          const float* phi, float fmajor, float fminor,
                          const float strike[3], const float dip[3]) {
  if (!c || !sigma2 || !cohes || !phi || !strike || !dip)
    return set_error(AWP_ERR_ARG, "null argument");
  if (c->p.nve != 3) return set_error(AWP_ERR_STATE, "plasticity needs NVE=3");
  const size_t bytes = sizeof(float) * (size_t)c->g.cells_pad();
  CU_TRY(cudaMemcpy(c->f[AWP_SIGMA2], sigma2, bytes, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(c->f[AWP_COHES], cohes, bytes, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(c->f[AWP_PHI], phi, bytes, cudaMemcpyHostToDevice));
  c->pp.fmajor = fmajor;
  c->pp.fminor = fminor;
  awp::rotation_matrix(strike, dip, c->pp.Rz, c->pp.RzT);
  c->pp.dh = c->p.dh;
  c->pp.dt = c->p.dt;
  c->pp.ktop = c->g.top();
  // visit count of the five drprecpc_calc strips (pmcl3d.c:2121-2181)
  const int nxp = (int)c->g.nx_pad(), nyp = (int)c->g.ny_pad();
  std::vector<unsigned char> mult((size_t)nxp * nyp, 0);
  // the whole grid's strips, in this part's indices when it is a sub-domain
  const int xo = c->sub_nxg ? c->sub_x0 : 0;
  const int xl = c->xls - xo, xr = (c->sub_nxg ? c->sub_nxg : c->p.nx) + AWP_NGSL + 1 - xo,
            yl = c->yls, yr = c->yre;
  auto add = [&](int i0, int i1, int j0, int j1) {
    for (int i = i0; i <= i1; ++i)
      for (int j = j0; j <= j1; ++j)
        if (i >= 0 && i < nxp && j >= 0 && j < nyp) mult[(size_t)i * nyp + j]++;
  };
  add(xl, xr, yl, yl + AWP_NGSL);
  add(xl, xr, yr - AWP_NGSL, yr);
  add(xl, xl + AWP_NGSL, yl, yr);
  add(xr - AWP_NGSL, xr, yl, yr);
  add(xl + AWP_NGSL, xr - AWP_NGSL, yl + AWP_NGSL, yr - AWP_NGSL);
  cudaFree(c->d_neta_mult);
  c->d_neta_mult = nullptr;
  int st;
  if ((st = ctx_alloc(c, (void**)&c->d_neta_mult, mult.size()))) return st;
  CU_TRY(cudaMemcpy(c->d_neta_mult, mult.data(), mult.size(), cudaMemcpyHostToDevice));
  c->plast_ready = true;
  return AWP_OK;
}

int awp_step(awp_ctx* c, int nsteps) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "awp_step before media upload");
  if (c->p.nve == 3 && !c->plast_ready)
    return set_error(AWP_ERR_STATE, "NVE=3 needs awp_upload_plasticity first");
  if (c->p.ngrids > 1)
    return set_error(AWP_ERR_STATE, "grid %d of a mesh: step the mesh (awp_mesh_step)", c->p.grid);
  for (int n = 0; n < nsteps; ++n) {
    int st = one_step(c);
    if (st) return st;
  }
  return AWP_OK;
}

int awp_synchronize(awp_ctx* c) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  CU_TRY(cudaStreamSynchronize(c->stream));
  int err = 0;
  CU_TRY(cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    // reported once: the word is cleared so that later steps report afresh
    CU_TRY(cudaMemset(c->d_err, 0, sizeof(int)));
    return set_error(AWP_ERR_CUDA, "a TMA pipeline wait ran out of its iteration limit");
  }
  return AWP_OK;
}

int awp_current_step(const awp_ctx* c, long long* step) {
  if (!c || !step) return set_error(AWP_ERR_ARG, "null argument");
  *step = c->cur_step;
  return AWP_OK;
}

int awp_field_device_ptr(awp_ctx* c, int field, float** dev_ptr) {
  if (!c || !dev_ptr || field < 0 || field >= AWP_NFIELDS)
    return set_error(AWP_ERR_ARG, "bad field %d", field);
  if (!c->f[field]) return set_error(AWP_ERR_STATE, "field %d not allocated (NVE)", field);
  *dev_ptr = c->f[field];
  return AWP_OK;
}

int awp_field_download(awp_ctx* c, int field, float* host) {
  float* d;
  int st = awp_field_device_ptr(c, field, &d);
  if (st) return st;
  if (!host) return set_error(AWP_ERR_ARG, "null host buffer");
  CU_TRY(cudaMemcpyAsync(host, d, sizeof(float) * (size_t)c->g.cells_pad(),
                         cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  return AWP_OK;
}

int awp_field_upload(awp_ctx* c, int field, const float* host) {
  float* d;
  int st = awp_field_device_ptr(c, field, &d);
  if (st) return st;
  if (!host) return set_error(AWP_ERR_ARG, "null host buffer");
  CU_TRY(cudaMemcpyAsync(d, host, sizeof(float) * (size_t)c->g.cells_pad(),
                         cudaMemcpyHostToDevice, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  if ((field >= AWP_R1 && field <= AWP_R6) || field == AWP_QP || field == AWP_QS)
    c->elastic = false;  // explicit memory-variable / Q state: use the full update
  if (field == AWP_D1 || field == AWP_MU || field == AWP_LAM) {
    if (field == AWP_LAM || field == AWP_MU)
      CU_TRY(awp_launch_lam_mu(c->f[AWP_LAM], c->f[AWP_MU], c->lam_mu, c->g, c->xls, c->xre,
                               c->yls, c->yre, c->stream));
    c->media_ready = true;
  }
  return AWP_OK;
}

int awp_gather_output(awp_ctx* c, int nbgx, int nedx, int nskpx, int nbgy, int nedy,
                      int nskpy, int nbgz, int nedz, int nskpz, float* bufx, float* bufy,
                      float* bufz, float* bufeta) {
  if (!c || !bufx || !bufy || !bufz) return set_error(AWP_ERR_ARG, "null argument");
  if (nskpx < 1 || nskpy < 1 || nskpz < 1) return set_error(AWP_ERR_ARG, "skip < 1");
  // every read inside the padded arrays: columns 2+ngsl+nbg .. 2+ngsl+ned, and
  // the levels top-k (w one lower on grid 0) or bathy-k
  const int shift = (c->p.grid == 0) ? 1 : 0;
  const bool follow = c->p.grid == 0 && c->d_bathy;
  if (nbgx < 0 || nbgy < 0 || nbgz < 0 || nedx < nbgx || nedy < nbgy || nedz < nbgz ||
      2 + AWP_NGSL + nedx >= c->g.nx_pad() || 2 + AWP_NGSL + nedy >= c->g.ny_pad() ||
      (!follow && c->g.top() - nedz - shift < 0))
    return set_error(AWP_ERR_ARG, "output window outside the grid");
  if (follow) {  // koz = bathy - k (- 1 at the top level) >= 0 at every recorded column
    const long long ld = c->g.nx_pad();
    for (int j = nbgy; j <= nedy; j += nskpy)
      for (int i = nbgx; i <= nedx; i += nskpx) {
        const int b = c->bathy[(size_t)(2 + AWP_NGSL + j) * ld + 2 + AWP_NGSL + i];
        if (b - nedz - (b == c->g.top() ? 1 : 0) < 0)
          return set_error(AWP_ERR_ARG,
                           "recorded depth %d is below the bathymetry level %d at column "
                           "(%d, %d)", nedz, b, i, j);
      }
  }
  VelBufArgs a;
  memset(&a, 0, sizeof(a));
  a.u1 = c->f[AWP_U1]; a.v1 = c->f[AWP_V1]; a.w1 = c->f[AWP_W1]; a.neta = c->f[AWP_NETA];
  a.bufx = bufx; a.bufy = bufy; a.bufz = bufz; a.bufeta = bufeta;
  a.nve = c->p.nve;
  a.nbgx = nbgx; a.nedx = nedx; a.nskpx = nskpx;
  a.nbgy = nbgy; a.nedy = nedy; a.nskpy = nskpy;
  a.nbgz = nbgz; a.nedz = nedz; a.nskpz = nskpz;
  a.rec_nxt = (nedx - nbgx) / nskpx + 1;
  a.rec_nyt = (nedy - nbgy) / nskpy + 1;
  a.rec_nzt = (nedz - nbgz) / nskpz + 1;
  a.slice = c->g.slice; a.yline = c->g.yline; a.ktop = c->g.top();
  // w one cell below the recorded level on grid 0 only (kernel.cu:3975-3986)
  a.w_shift = shift;
  if (follow) {
    a.bathy = c->d_bathy;
    a.bathy_ld = (int)c->g.nx_pad();
  }
  CU_TRY(awp_launch_velbuffer(a, c->stream));
  return AWP_OK;
}

int awp_velocity_forcing_init(awp_ctx* c, int npsrc, const int* pos, int nframes, int tskp,
                              int window, awp_frame_reader read, void* user) {
  if (!c || !pos || !read) return set_error(AWP_ERR_ARG, "null argument");
  if (c->p.ifault != 4) return set_error(AWP_ERR_STATE, "the context runs IFAULT=%d, not 4", c->p.ifault);
  if (c->p.grid != 0) return set_error(AWP_ERR_STATE, "frcvel acts on grid 0 (pmcl3d.c:1821)");
  if (c->d_frc_pos) return set_error(AWP_ERR_STATE, "velocity forcing already initialised");
  if (c->cur_step != 0) return set_error(AWP_ERR_STATE, "velocity forcing before the first step");
  if (npsrc < 1 || tskp < 1 || window < 1 || nframes < window || nframes % window)
    return set_error(AWP_ERR_ARG,
                     "npsrc, tskp, window >= 1 and frames a multiple of the window required "
                     "(%d points, tskp %d, %d frames, window %d)", npsrc, tskp, nframes, window);
  // frcvel_cu's cell of a point: (x + 1 + ngsl, y + 1 + ngsl, z + align - 1)
  for (int j = 0; j < npsrc; ++j) {
    const long long ix = pos[3 * j] + 1 + AWP_NGSL, iy = pos[3 * j + 1] + 1 + AWP_NGSL,
                    iz = pos[3 * j + 2] + AWP_ALIGN - 1;
    if (ix < 0 || ix >= c->g.nx_pad() || iy < 0 || iy >= c->g.ny_pad() || iz < 0 ||
        iz >= c->g.yline)
      return set_error(AWP_ERR_ARG, "point %d (%d, %d, %d) lies outside the padded grid", j,
                       pos[3 * j], pos[3 * j + 1], pos[3 * j + 2]);
  }
  int st;
  const size_t slots = (size_t)(window + 1) * npsrc;
  if ((st = ctx_alloc(c, (void**)&c->d_frc_pos, (size_t)npsrc * 3 * sizeof(int)))) return st;
  CU_TRY(cudaMemcpy(c->d_frc_pos, pos, (size_t)npsrc * 3 * sizeof(int), cudaMemcpyHostToDevice));
  for (int q = 0; q < 3; ++q) {
    if ((st = ctx_alloc(c, (void**)&c->d_frc[q], slots * sizeof(float)))) return st;
    CU_TRY(cudaMemset(c->d_frc[q], 0, slots * sizeof(float)));  // carry slot of window 1: zero
  }
  CU_TRY(cudaMallocHost((void**)&c->h_frc, 3 * (size_t)window * npsrc * sizeof(float)));
  CU_TRY(cudaEventCreateWithFlags(&c->frc_h2d, cudaEventDisableTiming));
  c->frc_n = npsrc;
  c->frc_frames = nframes;
  c->frc_tskp = tskp;
  c->frc_w = window;
  c->frc_next = 0;
  c->frc_read = read;
  c->frc_user = user;
  c->frc_s = 1;  // source_step before the loop (pmcl3d.c:1175)
  return frc_fill(c);
}

int awp_set_subdomain(awp_ctx* c, int nx_global, int x0) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (c->media_ready || c->cur_step != 0)
    return set_error(AWP_ERR_STATE, "sub-domain before the media and the first step");
  if (c->topo) return set_error(AWP_ERR_STATE, "sub-domain before the topography");
  if (c->p.ngrids != 1 || c->p.npc >= 2 || c->p.ifault == 4 || c->p.ifault == 6)
    return set_error(AWP_ERR_UNSUPPORTED,
                     "x-slab sub-domains cover single-grid runs without periodic sides, "
                     "prescribed velocities or plane waves");
  if (c->plast_ready)
    return set_error(AWP_ERR_STATE, "sub-domain before the plasticity inputs");
  if (x0 < 0 || x0 % 2 || nx_global < c->p.nx || x0 + c->p.nx > nx_global)
    return set_error(AWP_ERR_ARG,
                     "sub-domain x0=%d (even, >= 0) of width %d outside a grid of %d", x0,
                     c->p.nx, nx_global);
  // the sponge of the whole grid, this part's planes of it (inicrj, cerjan.c:5-64)
  const int nxp = (int)c->g.nx_pad(), nyp = (int)c->g.ny_pad(), nzp = (int)c->g.nz_pad();
  std::vector<float> cx(nx_global + 4 + AWP_NGSL2, 1.0f), cy(nyp, 1.0f), cz(nzp, 1.0f);
  awp::inicrj(c->p.arbc, nx_global, c->p.ny, c->p.nz, nx_global, c->p.ny, c->p.nd,
              c->p.grid == c->p.ngrids - 1 ? 1 : 0, c->p.npc, cx.data(), cy.data(), cz.data());
  CU_TRY(cudaMemcpy(c->dcrjx, cx.data() + x0, (size_t)nxp * 4, cudaMemcpyHostToDevice));
  c->sub_nxg = nx_global;
  c->sub_x0 = x0;
  return AWP_OK;
}

int awp_set_exchange(awp_ctx* c, awp_exchange_fn fn, void* user) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (fn && !c->sub_nxg) return set_error(AWP_ERR_STATE, "halo exchange without a sub-domain");
  c->xch = fn;
  c->xch_user = user;
  return AWP_OK;
}

int awp_halo_copy(awp_ctx* c, int unpack, int side, int set, int planes, float* buf) {
  if (!c || !buf) return set_error(AWP_ERR_ARG, "null argument");
  if ((side != 0 && side != 1) || set <= 0 || set > 15 || planes < 1 || planes > AWP_NGSL ||
      planes > c->p.nx)
    return set_error(AWP_ERR_ARG, "halo side %d, set %d, planes %d (1..%d)", side, set, planes,
                     AWP_NGSL);
  int fid[16];
  const int nf = halo_fields(set, fid);
  for (int q = 0; q < nf; ++q)
    if (!c->f[fid[q]]) return set_error(AWP_ERR_STATE, "field %d not allocated (NVE)", fid[q]);
  const long long plane0 = halo_plane(c, side, unpack != 0, planes);
  const size_t n = (size_t)planes * c->g.slice;
  cudaPointerAttributes at;
  const bool dev_buf = cudaPointerGetAttributes(&at, buf) == cudaSuccess &&
                       at.type == cudaMemoryTypeDevice && !(reinterpret_cast<uintptr_t>(buf) & 15);
  cudaGetLastError();  // a host pointer may leave a sticky "invalid value" here
  if (dev_buf) {  // one launch for every field of the set
    CopySegs cs;
    cs.nseg = nf;
    for (int q = 0; q < nf; ++q) {
      float* field = c->f[fid[q]] + plane0 * c->g.slice;
      float* b = buf + (size_t)q * n;
      cs.src[q] = unpack ? b : field;
      cs.dst[q] = unpack ? field : b;
      cs.n[q] = (long long)n;
    }
    CU_TRY(awp_launch_copy_segments(cs, c->stream));
    c->launches++;
    return AWP_OK;
  }
  for (int q = 0; q < nf; ++q) {  // host staging: one copy per field
    float* field = c->f[fid[q]] + plane0 * c->g.slice;
    float* b = buf + (size_t)q * n;
    CU_TRY(cudaMemcpyAsync(unpack ? field : b, unpack ? b : field, n * sizeof(float),
                           cudaMemcpyDefault, c->stream));
  }
  return AWP_OK;
}

int awp_compute_bathymetry(awp_ctx* c, int* bathy) {
  if (!c || !bathy) return set_error(AWP_ERR_ARG, "null argument");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "media not uploaded");
  const size_t n = (size_t)c->g.cells_pad();
  std::vector<float> mu(n), d1(n);
  CU_TRY(cudaStreamSynchronize(c->stream));
  CU_TRY(cudaMemcpy(mu.data(), c->f[AWP_MU], n * 4, cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(d1.data(), c->f[AWP_D1], n * 4, cudaMemcpyDeviceToHost));
  const long long nxp = c->g.nx_pad(), nyp = c->g.ny_pad();
  // pmcl3d.c:909-925: the highest level below the top with vs above 1 mm/s
  for (long long i = 0; i < nxp; ++i)
    for (long long j = 0; j < nyp; ++j) {
      int level = 0;
      for (int k = c->g.top(); k > AWP_ALIGN; --k) {
        const size_t q = (size_t)(i * c->g.slice + j * c->g.yline + k);
        const float prod = mu[q] * d1[q];
        const float vs = (float)sqrt(1. / (double)prod);
        if (vs > 0.001f) {
          level = k;
          break;
        }
      }
      bathy[j * nxp + i] = level;
    }
  return AWP_OK;
}

int awp_set_bathymetry(awp_ctx* c, const int* bathy) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  cudaFree(c->d_bathy);
  cudaFree(c->d_frc_pos);
  for (int q = 0; q < 3; ++q) cudaFree(c->d_frc[q]);
  if (c->h_frc) cudaFreeHost(c->h_frc);
  if (c->frc_h2d) cudaEventDestroy(c->frc_h2d);
  c->d_bathy = nullptr;
  c->bathy.clear();
  if (!bathy) return AWP_OK;
  if (c->p.grid != 0) return set_error(AWP_ERR_STATE, "FOLLOWBATHY applies to grid 0 only");
  const size_t n = (size_t)(c->g.nx_pad() * c->g.ny_pad());
  for (size_t q = 0; q < n; ++q)
    if (bathy[q] < 0 || bathy[q] > c->g.top())
      return set_error(AWP_ERR_ARG, "bathymetry level %d outside 0..%d at column %zu", bathy[q],
                       c->g.top(), q);
  int st;
  if ((st = ctx_alloc(c, (void**)&c->d_bathy, n * sizeof(int)))) return st;
  CU_TRY(cudaMemcpy(c->d_bathy, bathy, n * sizeof(int), cudaMemcpyHostToDevice));
  c->bathy.assign(bathy, bathy + n);
  return AWP_OK;
}

int awp_receivers_init(awp_ctx* c, const char* recvfile, long long nt) {
  if (!c || !recvfile) return set_error(AWP_ERR_ARG, "null argument");
  if (c->sub_nxg)
    return set_error(AWP_ERR_UNSUPPORTED, "point sets on an x-slab sub-domain");
  if (nt < 1) return set_error(AWP_ERR_ARG, "nt must be >= 1");
  if (c->recv) return set_error(AWP_ERR_STATE, "receivers already initialised");
  RecvState* r = nullptr;
  const int e = awp_recv_create(recvfile, nt, c->g, c->p.dh, c->topo, &r, g_errmsg,
                                sizeof(g_errmsg));
  if (e) return e < 0 ? AWP_ERR_CUDA : AWP_ERR_IO;
  c->recv = r;
  // the reference records the state before the first step (pmcl3d.c:1603-1605)
  if (awp_recv_record(c->recv, c->cur_step, c->f[AWP_U1], c->f[AWP_V1], c->f[AWP_W1], c->stream,
                      &c->launches, g_errmsg, sizeof(g_errmsg)))
    return AWP_ERR_IO;
  return AWP_OK;
}

int awp_sgt_init(awp_ctx* c, const char* sgtfile, long long nt) {
  if (!c || !sgtfile) return set_error(AWP_ERR_ARG, "null argument");
  if (c->sub_nxg)
    return set_error(AWP_ERR_UNSUPPORTED, "point sets on an x-slab sub-domain");
  if (nt < 1) return set_error(AWP_ERR_ARG, "nt must be >= 1");
  if (c->sgt) return set_error(AWP_ERR_STATE, "SGT output already initialised");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "media not uploaded");
  RecvState *r = nullptr, *m = nullptr;
  const int e = awp_sgt_create(sgtfile, nt, c->g, c->p.dh, c->topo, &r, &m, g_errmsg,
                               sizeof(g_errmsg));
  if (e) return e < 0 ? AWP_ERR_CUDA : AWP_ERR_IO;
  c->sgt = r;
  c->sgt_mat = m;
  // sgt_write_material_properties (sgt.c:70-90, pmcl3d.c:1575-1578): the
  // reference writes the inverse-lambda array to the "d1" file as well, and so
  // does this build; then "lami" (1/lambda) and "mui" (1/mu)
  const std::string base = awp_recv_base(c->sgt_mat, 0);
  const struct {
    const char* suffix;
    const float* field;
  } out[3] = {{"d1", c->f[AWP_LAM]}, {"lami", c->f[AWP_LAM]}, {"mui", c->f[AWP_MU]}};
  for (const auto& o : out)
    if (awp_recv_write_once(c->sgt_mat, o.field, (base + o.suffix).c_str(), c->stream,
                            &c->launches, g_errmsg, sizeof(g_errmsg)))
      return AWP_ERR_IO;
  // the state before the first step (pmcl3d.c:1605), which holds the step-1
  // source sample the reference adds before the loop (pmcl3d.c:1175-1187)
  if (c->ncell) {
    const int s = initial_source(c);
    if (s) return s;
  }
  return sgt_record(c);
}

int awp_receivers_count(awp_ctx* c, int counts[3]) {
  if (!c || !counts) return set_error(AWP_ERR_ARG, "null argument");
  for (int q = 0; q < 3; ++q) counts[q] = awp_recv_length(c->recv, q);
  return AWP_OK;
}

int awp_sourcefile_init(awp_ctx* c, const char* sourcefile) {
  if (!c || !sourcefile) return set_error(AWP_ERR_ARG, "null argument");
  if (c->sub_nxg)
    return set_error(AWP_ERR_UNSUPPORTED, "point sets on an x-slab sub-domain");
  if (c->srcf) return set_error(AWP_ERR_STATE, "SOURCEFILE already initialised");
  SrcFileState* s = nullptr;
  const int e = awp_srcf_create(sourcefile, c->g, c->p.dh, c->p.dt, c->topo, &s, g_errmsg,
                                sizeof(g_errmsg));
  if (e) return e < 0 ? AWP_ERR_CUDA : AWP_ERR_IO;
  c->srcf = s;
  // sources_read(0) before the loop (pmcl3d.c:1607)
  if (awp_srcf_read(c->srcf, c->cur_step, c->stream, g_errmsg, sizeof(g_errmsg)))
    return AWP_ERR_IO;
  return AWP_OK;
}

int awp_forcefile_init(awp_ctx* c, const char* forcefile) {
  if (!c || !forcefile) return set_error(AWP_ERR_ARG, "null argument");
  if (c->sub_nxg)
    return set_error(AWP_ERR_UNSUPPORTED, "point sets on an x-slab sub-domain");
  if (c->forcef) return set_error(AWP_ERR_STATE, "FORCEFILE already initialised");
  if (!c->topo)
    return set_error(AWP_ERR_STATE,
                     "FORCEFILE forces act on a curvilinear top block: initialise the "
                     "topography first");
  SrcFileState* s = nullptr;
  const int e = awp_forcef_create(forcefile, c->g, c->p.dh, c->p.dt, c->topo, &s, g_errmsg,
                                  sizeof(g_errmsg));
  if (e) return e < 0 ? AWP_ERR_CUDA : AWP_ERR_IO;
  c->forcef = s;
  // forces_read(0) before the loop (pmcl3d.c:1608)
  if (awp_srcf_read(c->forcef, c->cur_step, c->stream, g_errmsg, sizeof(g_errmsg)))
    return AWP_ERR_IO;
  return AWP_OK;
}

int awp_input_read(const char* path, long long hdr[8], char* file, int filecap, float* x,
                   float* y, float* z, int* type, long long cap) {
  if (!path || !hdr) return AWP_ERR_ARG;
  awp::InputFile in;
  const int e = awp::read_input(path, &in);
  if (e) return e;
  hdr[0] = (long long)in.length;
  hdr[1] = (long long)in.gpu_buffer_size;
  hdr[2] = (long long)in.cpu_buffer_size;
  hdr[3] = (long long)in.steps;
  hdr[4] = (long long)in.num_writes;
  hdr[5] = in.stride;
  hdr[6] = in.degree;
  hdr[7] = in.major;
  if (file && filecap > 0) snprintf(file, (size_t)filecap, "%s", in.file.c_str());
  for (size_t i = 0; i < in.length && (long long)i < cap; ++i) {
    if (x) x[i] = in.x[i];
    if (y) y[i] = in.y[i];
    if (z) z[i] = in.z[i];
    if (type) type[i] = in.type[i];
  }
  return 0;
}

static int point_coefs(const char* path, const char* intopo, int grid_type, int nxt, int nyt,
                       int nzt, float h, long long cap, int* count, int* indices, int* ix,
                       int* iy, int* iz, float* lx, float* ly, float* lz) {
  if (!path || !count || grid_type < 0 || grid_type > 9) return AWP_ERR_ARG;
  awp::InputFile in;
  int e = awp::read_input(path, &in);
  if (e) return e;
  awp::TopoMetrics m;
  if (intopo) {
    if (nzt < 12) return AWP_ERR_ARG;
    awp::topo_init_metrics(&m, nxt, nyt, nzt, h);
    e = awp::topo_read_file(intopo, nxt, nyt, &m.f);
    if (e) return e;
    awp::topo_build_metrics(&m);
  }
  awp::BlockDesc b{nxt, nyt, nzt, h, intopo ? 1 : 0};
  awp::PointSet ps;
  e = awp::point_set_init(in, (awp::GridType)grid_type, &b, 1, &ps, intopo ? &m : nullptr);
  if (e) return e;
  const awp::BlockInterp& bi = ps.block[0];
  *count = bi.num_query;
  const int nb = bi.num_basis;
  for (int q = 0; q < bi.num_query && q < cap; ++q) {
    indices[q] = ps.indices[bi.ridx[q]];
    ix[q] = bi.ix[q];
    iy[q] = bi.iy[q];
    iz[q] = bi.iz[q];
    for (int d = 0; d < nb; ++d) {
      lx[(size_t)q * nb + d] = bi.lx[(size_t)q * nb + d];
      ly[(size_t)q * nb + d] = bi.ly[(size_t)q * nb + d];
      lz[(size_t)q * nb + d] = bi.lz[(size_t)q * nb + d];
    }
  }
  return 0;
}

int awp_point_coefs(const char* path, int grid_type, int nxt, int nyt, int nzt, float h,
                    long long cap, int* count, int* indices, int* ix, int* iy, int* iz, float* lx,
                    float* ly, float* lz) {
  return point_coefs(path, nullptr, grid_type, nxt, nyt, nzt, h, cap, count, indices, ix, iy, iz,
                     lx, ly, lz);
}

int awp_point_coefs_topo(const char* path, const char* intopo, int grid_type, int nxt, int nyt,
                         int nzt, float h, long long cap, int* count, int* indices, int* ix,
                         int* iy, int* iz, float* lx, float* ly, float* lz) {
  if (!intopo) return AWP_ERR_ARG;
  return point_coefs(path, intopo, grid_type, nxt, nyt, nzt, h, cap, count, indices, ix, iy, iz,
                     lx, ly, lz);
}

int awp_mesh_destroy(awp_mesh* m) {
  if (!m) return AWP_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (int p = 0; p < m->ngrids; ++p) awp_ctx_destroy(m->g[p]);
  if (m->own_stream) cudaStreamDestroy(m->own_stream);
  delete m;
  return AWP_OK;
}

int awp_mesh_set_stream(awp_mesh* m, void* stream) {
  if (!m) return set_error(AWP_ERR_ARG, "null mesh");
  CU_TRY(cudaStreamSynchronize(m->stream));
  m->stream = static_cast<cudaStream_t>(stream);
  for (int p = 0; p < m->ngrids; ++p) {
    const int st = awp_set_stream(m->g[p], stream);
    if (st) return st;
  }
  return AWP_OK;
}

int awp_mesh_create(const awp_params* grids, int ngrids, awp_mesh** out) {
  if (!grids || !out) return set_error(AWP_ERR_ARG, "null argument");
  *out = nullptr;
  if (ngrids < 1 || ngrids > AWP_MAXGRIDS)
    return set_error(AWP_ERR_ARG, "ngrids=%d (1..%d)", ngrids, AWP_MAXGRIDS);
  for (int p = 0; p < ngrids; ++p) {
    const awp_params& q = grids[p];
    if (q.grid != p || q.ngrids != ngrids)
      return set_error(AWP_ERR_ARG, "grid %d: params.grid/ngrids must be %d/%d", p, p, ngrids);
    if (p > 0) {  // each block 3x coarser than the one above (pmcl3d.c:370-378)
      const awp_params& f = grids[p - 1];
      if (f.nx != 3 * q.nx || f.ny != 3 * q.ny)
        return set_error(AWP_ERR_ARG, "grid %d: NX, NY must be 1/3 of grid %d's", p, p - 1);
      if (f.dt != q.dt) return set_error(AWP_ERR_ARG, "grids must share DT");
      if (q.nz < 8) return set_error(AWP_ERR_ARG, "grid %d: NZ too small for the interface", p);
    }
    if (p < ngrids - 1 && q.nz < 12)
      return set_error(AWP_ERR_ARG, "grid %d: NZ too small for the interface", p);
  }
  awp_mesh* m = new awp_mesh();
  cudaError_t e = cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete m;
    return set_error(AWP_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  m->stream = m->own_stream;
  for (int p = 0; p < ngrids; ++p) {
    int st = awp_ctx_create(&grids[p], &m->g[p]);
    if (st) {
      awp_mesh_destroy(m);
      return st;
    }
    m->ngrids = p + 1;
    awp_set_stream(m->g[p], m->stream);
    if (p > 0) {
      AwpTexture& t = m->g[p]->tex;
      t.dm = 1;
      t.nx = grids[p].nx;
      t.f_ny = grids[p - 1].ny;
      t.f_nzt = grids[p - 1].nz;
    }
  }
  *out = m;
  return AWP_OK;
}

int awp_mesh_grid(awp_mesh* m, int p, awp_ctx** ctx) {
  if (!m || !ctx || p < 0 || p >= m->ngrids) return set_error(AWP_ERR_ARG, "bad grid %d", p);
  *ctx = m->g[p];
  return AWP_OK;
}

int awp_mesh_step(awp_mesh* m, int nsteps) {
  if (!m) return set_error(AWP_ERR_ARG, "null mesh");
  if (!m->prepared) {
    int st = mesh_prepare(m);
    if (st) return st;
  }
  for (int p = 0; p < m->ngrids; ++p)
    if (m->g[p]->p.nve == 3 && !m->g[p]->plast_ready)
      return set_error(AWP_ERR_STATE, "grid %d: NVE=3 needs awp_upload_plasticity first", p);
  for (int s = 0; s < nsteps; ++s) {
    int st = mesh_step(m);
    if (st) return st;
  }
  return AWP_OK;
}

// ---------------------------------------------------------------------------
// x-slab decomposition stepped in lockstep on one device: the parts' phases in
// order, the halo planes copied between neighbours in device memory.
// ---------------------------------------------------------------------------
struct awp_decomp {
  int n = 0;
  awp_ctx* part[AWP_MAXPARTS] = {};
  int planes = AWP_HALO_PLANES;
  cudaStream_t stream = nullptr;  // created with the decomposition, destroyed with it
  cudaStream_t run = nullptr;     // a caller's stream (awp_decomp_set_stream)
  bool use_run = false;
  bool prepared = false;
  cudaStream_t active() const { return use_run ? run : stream; }
};

namespace {

int decomp_exchange(awp_decomp* d, int set) {
  int fid[16];
  const int nf = halo_fields(set, fid);
  const int H = d->planes;
  // one launch per interface: both directions of every field of the set
  for (int p = 0; p + 1 < d->n; ++p) {
    awp_ctx *L = d->part[p], *R = d->part[p + 1];
    const long long n = (long long)H * L->g.slice;
    CopySegs cs;
    cs.nseg = 0;
    for (int q = 0; q < nf; ++q) {
      const int f = fid[q];
      cs.src[cs.nseg] = L->f[f] + halo_plane(L, 1, false, H) * L->g.slice;
      cs.dst[cs.nseg] = R->f[f] + halo_plane(R, 0, true, H) * R->g.slice;
      cs.n[cs.nseg++] = n;
      cs.src[cs.nseg] = R->f[f] + halo_plane(R, 0, false, H) * R->g.slice;
      cs.dst[cs.nseg] = L->f[f] + halo_plane(L, 1, true, H) * L->g.slice;
      cs.n[cs.nseg++] = n;
    }
    CU_TRY(awp_launch_copy_segments(cs, d->active()));
    L->launches++;
  }
  return AWP_OK;
}

int decomp_step(awp_decomp* d) {
  int st;
  awp_ctx* const* c = d->part;
  for (int p = 0; p < d->n; ++p)
    if ((st = phase_begin(c[p]))) return st;
  if ((st = decomp_exchange(d, AWP_HALO_VELOCITY | AWP_HALO_STRESS))) return st;
  for (int p = 0; p < d->n; ++p)
    if ((st = phase_velocity(c[p]))) return st;
  if ((st = decomp_exchange(d, AWP_HALO_VELOCITY))) return st;
  for (int p = 0; p < d->n; ++p)
    if ((st = phase_stress(c[p]))) return st;
  for (int p = 0; p < d->n; ++p)
    if ((st = phase_sources(c[p]))) return st;
  if (c[0]->p.nve == 3) {  // the middle band, the stress halo, the yield factors, their
                           // halo, the return
    for (int p = 0; p < d->n; ++p) {
      if (!stress_split(c[p])) continue;
      int i0, i1, j0, j1;
      middle_band(c[p], &i0, &i1, &j0, &j1);
      if ((st = launch_cart_stress(c[p], i0, i1, j0, j1))) return st;
    }
    if ((st = decomp_exchange(d, AWP_HALO_STRESS))) return st;
    for (int p = 0; p < d->n; ++p) {
      if ((st = launch_plasticity(c[p]))) return st;
      c[p]->launches++;
    }
    if ((st = decomp_exchange(d, AWP_HALO_YLDFAC))) return st;
    for (int p = 0; p < d->n; ++p) {
      if ((st = launch_plast_app(c[p]))) return st;
      c[p]->launches++;
    }
  }
  for (int p = 0; p < d->n; ++p)
    if ((st = phase_fstr(c[p]))) return st;
  return AWP_OK;
}

}  // namespace

int awp_decomp_create(awp_ctx** parts, int n, awp_decomp** out) {
  if (!parts || !out) return set_error(AWP_ERR_ARG, "null argument");
  *out = nullptr;
  if (n < 1 || n > AWP_MAXPARTS) return set_error(AWP_ERR_ARG, "%d parts (1..%d)", n, AWP_MAXPARTS);
  int dev0 = -1;
  for (int p = 0; p < n; ++p) {
    awp_ctx* c = parts[p];
    if (!c || !c->sub_nxg) return set_error(AWP_ERR_STATE, "part %d has no sub-domain", p);
    if (c->xch) return set_error(AWP_ERR_STATE, "part %d has its own exchange hook", p);
    if (c->p.ny != parts[0]->p.ny || c->p.nz != parts[0]->p.nz ||
        c->sub_nxg != parts[0]->sub_nxg || c->p.nve != parts[0]->p.nve)
      return set_error(AWP_ERR_ARG, "part %d: ny, nz, NVE and the global nx must agree", p);
    const int want = p == 0 ? 0 : parts[p - 1]->sub_x0 + parts[p - 1]->p.nx;
    if (c->sub_x0 != want)
      return set_error(AWP_ERR_ARG, "part %d starts at x=%d, not %d", p, c->sub_x0, want);
    if (c->p.nx < AWP_NGSL / 2) return set_error(AWP_ERR_ARG, "part %d narrower than its halo", p);
    int dev = -1;
    cudaPointerAttributes at;
    CU_TRY(cudaPointerGetAttributes(&at, c->f[AWP_U1]));
    dev = at.device;
    if (p == 0) dev0 = dev;
    else if (dev != dev0) return set_error(AWP_ERR_ARG, "part %d is on another device", p);
  }
  if (parts[n - 1]->sub_x0 + parts[n - 1]->p.nx != parts[0]->sub_nxg)
    return set_error(AWP_ERR_ARG, "the parts do not cover the grid");
  awp_decomp* d = new awp_decomp();
  d->n = n;
  for (int p = 0; p < n; ++p) d->part[p] = parts[p];
  if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete d;
    return set_error(AWP_ERR_CUDA, "stream");
  }
  for (int p = 0; p < n; ++p) {
    cudaStreamSynchronize(parts[p]->stream);
    awp_set_stream(parts[p], d->stream);
  }
  *out = d;
  return AWP_OK;
}

int awp_decomp_destroy(awp_decomp* d) {
  if (!d) return AWP_OK;
  cudaStreamSynchronize(d->active());
  cudaStreamSynchronize(d->stream);
  for (int p = 0; p < d->n; ++p) awp_set_stream(d->part[p], nullptr);
  cudaStreamDestroy(d->stream);
  delete d;
  return AWP_OK;
}

int awp_decomp_step(awp_decomp* d, int nsteps) {
  if (!d) return set_error(AWP_ERR_ARG, "null decomposition");
  if (!d->prepared) {
    // the media halos once; each part keeps its own elastic specialisation
    // (with Q^-1 identically zero the anelastic update reduces exactly to it)
    for (int p = 0; p < d->n; ++p) {
      if (!d->part[p]->media_ready) return set_error(AWP_ERR_STATE, "part %d has no media", p);
      if (d->part[p]->p.nve == 3 && !d->part[p]->plast_ready)
        return set_error(AWP_ERR_STATE, "part %d: NVE=3 needs awp_upload_plasticity", p);
    }
    const int st = decomp_exchange(d, AWP_HALO_MEDIA);
    if (st) return st;
    d->prepared = true;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int st = decomp_step(d);
    if (st) return st;
  }
  return AWP_OK;
}

int awp_decomp_set_stream(awp_decomp* d, void* stream) {
  if (!d) return set_error(AWP_ERR_ARG, "null decomposition");
  CU_TRY(cudaStreamSynchronize(d->active()));
  for (int p = 0; p < d->n; ++p) {
    const int st = awp_set_stream(d->part[p], stream);
    if (st) return st;
  }
  d->run = static_cast<cudaStream_t>(stream);
  d->use_run = true;
  return AWP_OK;
}

int awp_decomp_synchronize(awp_decomp* d) {
  if (!d) return set_error(AWP_ERR_ARG, "null decomposition");
  for (int p = 0; p < d->n; ++p) {
    const int st = awp_synchronize(d->part[p]);
    if (st) return st;
  }
  return AWP_OK;
}

int awp_mesh_synchronize(awp_mesh* m) {
  if (!m) return set_error(AWP_ERR_ARG, "null mesh");
  for (int p = 0; p < m->ngrids; ++p) {
    int st = awp_synchronize(m->g[p]);
    if (st) return st;
  }
  return AWP_OK;
}

int awp_topo_metrics(const char* path, int nx, int ny, int nz, float h, float* out) {
  if (!path || !out || nx < 1 || ny < 1 || nz < 12) return AWP_ERR_ARG;
  awp::TopoMetrics m;
  awp::topo_init_metrics(&m, nx, ny, nz, h);
  const int e = awp::topo_read_file(path, nx, ny, &m.f);
  if (e) return e;
  awp::topo_build_metrics(&m);
  const size_t nf = m.f.size(), ng = m.g.size();
  const std::vector<float>* fa[10] = {&m.f, &m.f_1, &m.f_2, &m.f_c, &m.f1_1,
                                      &m.f1_2, &m.f1_c, &m.f2_1, &m.f2_2, &m.f2_c};
  for (int q = 0; q < 10; ++q) memcpy(out + q * nf, fa[q]->data(), nf * sizeof(float));
  const std::vector<float>* ga[4] = {&m.g, &m.g_c, &m.g3, &m.g3_c};
  for (int q = 0; q < 4; ++q) memcpy(out + 10 * nf + q * ng, ga[q]->data(), ng * sizeof(float));
  return 0;
}

}  // extern "C"

// ===========================================================================
// Batched instances
// ===========================================================================
struct awp_batch {
  std::vector<awp_ctx*> ctx;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  BatchInst* d_inst = nullptr;
  int4 *d_vt = nullptr, *d_st = nullptr, *d_ste = nullptr;
  int2 *d_src = nullptr, *d_rows = nullptr;
  int* d_cnt = nullptr;   // [3] tile counters
  int* d_step = nullptr;  // steps taken (device copy of cur_step)
  BatchLaunch L{};
  int ty = 8, ichunk = 16;
  int mode = 0;  // 0: persistent tile-queue launches; 1: graph of each instance's own launches
  int branches = 0;  // mode 1: parallel graph branches (0: one per instance)
  std::vector<cudaStream_t> cs;   // mode 1: one capture stream per instance
  std::vector<cudaEvent_t> join;  // mode 1: branch joins
  cudaEvent_t fork = nullptr;
  long long launches_per_step = 0;
  bool use_graph = true;
  bool dirty = true;  // tile lists / graph to rebuild
  long long step = 0;
  long long cells = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

void batch_free_lists(awp_batch* b) {
  cudaFree(b->d_vt); cudaFree(b->d_st); cudaFree(b->d_ste);
  b->d_vt = b->d_st = b->d_ste = nullptr;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

template <class T>
int upload_vec(T** d, const std::vector<T>& h) {
  *d = nullptr;
  if (h.empty()) return AWP_OK;
  CU_TRY(cudaMalloc((void**)d, sizeof(T) * h.size()));
  CU_TRY(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return AWP_OK;
}

// Mode 1: one step of every instance as parallel branches of one graph, each
// branch the instance's own tuned launches (velocity, stress, sources at the
// device step, free-surface images); the step counter advances after the join.
int batch_capture_instances(awp_batch* b) {
  if (b->cs.empty()) {
    b->cs.assign(b->ctx.size(), nullptr);
    b->join.assign(b->ctx.size(), nullptr);
    for (size_t q = 0; q < b->ctx.size(); ++q) {
      CU_TRY(cudaStreamCreateWithFlags(&b->cs[q], cudaStreamNonBlocking));
      CU_TRY(cudaEventCreateWithFlags(&b->join[q], cudaEventDisableTiming));
    }
    CU_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  }
  CU_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int st = AWP_OK;
  long long l0 = 0;
  for (awp_ctx* c : b->ctx) l0 += c->launches;
  cudaError_t ce = cudaEventRecord(b->fork, b->stream);
  // branches in decreasing size: the largest instances start first, so the
  // small ones fill the tail (capture order is the graph's launch order)
  std::vector<size_t> ord(b->ctx.size());
  for (size_t q = 0; q < ord.size(); ++q) ord[q] = q;
  std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
    return b->ctx[x]->g.cells_pad() > b->ctx[y]->g.cells_pad();
  });
  // instances dealt round-robin (largest first) onto nb branches
  const size_t nb = b->branches > 0 ? std::min((size_t)b->branches, ord.size()) : ord.size();
  std::vector<char> used(nb, 0);
  for (size_t n = 0; n < ord.size() && !st && ce == cudaSuccess; ++n) {
    const size_t q = ord[n], br = n % nb;
    awp_ctx* c = b->ctx[q];
    cudaStream_t saved = c->stream;
    const bool prof = c->profile;
    c->stream = b->cs[br];
    c->profile = false;
    if (!used[br]) {
      ce = cudaStreamWaitEvent(b->cs[br], b->fork, 0);
      used[br] = 1;
    }
    if (ce == cudaSuccess) st = phase_velocity(c);
    if (!st && ce == cudaSuccess) st = phase_stress(c);
    if (!st && ce == cudaSuccess && c->ncell > 0) {
      if (c->p.ifault == 5) {
        const KinSrcArgs k = make_kin_args(c, 0);
        ce = awp_launch_sources_dev(nullptr, &k, b->d_step, 0, c->stream);
        c->launches++;
      } else if (c->p.ifault < 4) {
        const SrcArgs a = make_src_args(c, 0);
        ce = awp_launch_sources_dev(&a, nullptr, b->d_step, c->p.nst, c->stream);
        c->launches++;
      }
    }
    if (!st && ce == cudaSuccess) st = phase_fstr(c);
    c->stream = saved;
    c->profile = prof;
  }
  for (size_t br = 0; br < nb && !st && ce == cudaSuccess; ++br) {
    if (!used[br]) continue;
    ce = cudaEventRecord(b->join[br], b->cs[br]);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->join[br], 0);
  }
  if (!st && ce == cudaSuccess) {
    ce = awp_launch_step_advance(b->d_step, b->stream);
    b->ctx[0]->launches++;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
  long long l1 = 0;
  for (awp_ctx* c : b->ctx) l1 += c->launches;
  b->ctx[0]->launches -= (l1 - l0);  // counted per replay instead
  b->launches_per_step = l1 - l0;
  if (st || ce != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (st) return st;
    return set_error(AWP_ERR_CUDA, "batch graph capture: %s",
                     cudaGetErrorString(ce != cudaSuccess ? ce : ee));
  }
  b->graph = g;
  CU_TRY(cudaGraphInstantiate(&b->exec, g, 0));
  return AWP_OK;
}

// Tile lists for the current shape (tile 32 k x ty j x ichunk i), the
// persistent grid sizes, and the captured one-step graph.
int batch_build(awp_batch* b) {
  batch_free_lists(b);
  if (b->mode == 1) {
    const int e = batch_capture_instances(b);
    if (!e) b->dirty = false;
    return e;
  }
  std::vector<int4> vt, st, ste;
  for (size_t n = 0; n < b->ctx.size(); ++n) {
    awp_ctx* c = b->ctx[n];
    const VelArgs v = make_vel_args(c);
    const int gx = (v.k1 - v.k0 + 32) / 32, gy = (v.j1 - v.j0 + b->ty) / b->ty,
              gz = (v.i1 - v.i0 + b->ichunk) / b->ichunk;
    for (int z = 0; z < gz; ++z)
      for (int y = 0; y < gy; ++y)
        for (int x = 0; x < gx; ++x) vt.push_back(make_int4((int)n, x, y, z));
    const StrArgs a = make_str_args(c);
    const int sx = (a.k1 - a.k0 + 32) / 32, sy = (a.j1 - a.j0 + b->ty) / b->ty,
              sz = (a.i1 - a.i0 + b->ichunk) / b->ichunk;
    std::vector<int4>& dst = c->elastic ? ste : st;
    for (int z = 0; z < sz; ++z)
      for (int y = 0; y < sy; ++y)
        for (int x = 0; x < sx; ++x) dst.push_back(make_int4((int)n, x, y, z));
  }
  int e;
  if ((e = upload_vec(&b->d_vt, vt)) || (e = upload_vec(&b->d_st, st)) ||
      (e = upload_vec(&b->d_ste, ste)))
    return e;
  int bv = 0, bs = 0;
  if (awp_batch_blocks_per_sm(b->ty, &bv, &bs))
    return set_error(AWP_ERR_CUDA, "batch occupancy query failed");
  int dev = 0, nsm = 0;
  CU_TRY(cudaGetDevice(&dev));
  CU_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  BatchLaunch& L = b->L;
  L.inst = b->d_inst;
  L.vtiles = b->d_vt; L.stiles = b->d_st; L.stiles_el = b->d_ste;
  L.nvtiles = (int)vt.size(); L.nstiles = (int)st.size(); L.nstiles_el = (int)ste.size();
  L.counters = b->d_cnt; L.step = b->d_step;
  L.ty = b->ty; L.ichunk = b->ichunk;
  L.grid_vel = std::max(1, std::min(nsm * std::max(bv, 1), L.nvtiles));
  L.grid_str = std::max(1, std::min(nsm * std::max(bs, 1), std::max(L.nstiles, L.nstiles_el)));
  b->launches_per_step = 1 + (L.nstiles > 0) + (L.nstiles_el > 0) + (L.nsrc > 0) + 1;
  if (b->use_graph) {
    CU_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = awp_launch_batch_step(L, b->stream);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return set_error(AWP_ERR_CUDA, "batch graph capture: %s",
                       cudaGetErrorString(le != cudaSuccess ? le : ce));
    }
    b->graph = g;
    CU_TRY(cudaGraphInstantiate(&b->exec, g, 0));
  }
  b->dirty = false;
  return AWP_OK;
}

}  // namespace

extern "C" {

int awp_batch_destroy(awp_batch* b) {
  if (!b) return AWP_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_free_lists(b);
  cudaFree(b->d_inst); cudaFree(b->d_src); cudaFree(b->d_rows);
  cudaFree(b->d_cnt); cudaFree(b->d_step);
  for (cudaStream_t x : b->cs) if (x) cudaStreamDestroy(x);
  for (cudaEvent_t x : b->join) if (x) cudaEventDestroy(x);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return AWP_OK;
}

int awp_batch_create(awp_ctx* const* ctxs, int n, awp_batch** out) {
  if (!ctxs || !out || n < 1) return set_error(AWP_ERR_ARG, "null argument or n < 1");
  *out = nullptr;
  for (int q = 0; q < n; ++q) {
    awp_ctx* c = ctxs[q];
    if (!c) return set_error(AWP_ERR_ARG, "instance %d is null", q);
    if (!c->media_ready) return set_error(AWP_ERR_STATE, "instance %d: media not uploaded", q);
    if (c->p.ngrids != 1 || c->p.nve == 3 || c->topo || c->recv || c->srcf || c->forcef ||
        c->sgt || c->p.ifault == 6 || c->p.ifault == 4 || c->sub_nxg)
      return set_error(AWP_ERR_UNSUPPORTED,
                       "instance %d: a batch holds single-grid Cartesian runs without "
                       "plasticity, receivers, SOURCEFILE, plane-wave or prescribed-velocity "
                       "sources", q);
    if (c->cur_step != ctxs[0]->cur_step)
      return set_error(AWP_ERR_STATE, "instances must start at the same step");
    for (int r = 0; r < q; ++r)
      if (ctxs[r] == c) return set_error(AWP_ERR_ARG, "instance %d appears twice", q);
  }
  awp_batch* b = new awp_batch();
  b->ctx.assign(ctxs, ctxs + n);
  b->step = ctxs[0]->cur_step;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) {
    awp_batch_destroy(b);
    return set_error(AWP_ERR_CUDA, "batch stream/event creation failed");
  }
  std::vector<BatchInst> inst(n);
  std::vector<int2> src, rows;
  for (int q = 0; q < n; ++q) {
    awp_ctx* c = ctxs[q];
    BatchInst& I = inst[q];
    memset(&I, 0, sizeof(I));
    I.v = make_vel_args(c);
    I.s = make_str_args(c);
    I.f = make_fstr_args(c);
    I.src = make_src_args(c, 0);
    I.kin = make_kin_args(c, 0);
    I.elastic = c->elastic ? 1 : 0;
    I.ifault = c->p.ifault;
    I.nst = c->p.nst;
    if (c->ncell > 0 && (c->p.ifault < 4 || c->p.ifault == 5))
      for (int k = 0; k < c->ncell; ++k) src.push_back(make_int2(q, k));
    for (int i = I.f.i0; i <= I.f.i1; ++i) rows.push_back(make_int2(q, i));
    b->cells += (long long)c->p.nx * c->p.ny * c->p.nz;
  }
  int e;
  if ((e = upload_vec(&b->d_inst, inst)) || (e = upload_vec(&b->d_src, src)) ||
      (e = upload_vec(&b->d_rows, rows))) {
    awp_batch_destroy(b);
    return e;
  }
  if (cudaMalloc((void**)&b->d_cnt, 3 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_step, sizeof(int)) != cudaSuccess) {
    awp_batch_destroy(b);
    return set_error(AWP_ERR_NOMEM, "batch counters");
  }
  b->L.src_cells = b->d_src;
  b->L.nsrc = (int)src.size();
  b->L.rows = b->d_rows;
  b->L.nrows = (int)rows.size();
  const int st = (int)b->step;
  if (cudaMemcpy(b->d_step, &st, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
    awp_batch_destroy(b);
    return set_error(AWP_ERR_CUDA, "batch step upload");
  }
  *out = b;
  return AWP_OK;
}

int awp_batch_set_shape(awp_batch* b, int ty, int ichunk) {
  if (!b) return set_error(AWP_ERR_ARG, "null batch");
  if ((ty != 4 && ty != 8) || ichunk < 1 || ichunk > 1024)
    return set_error(AWP_ERR_ARG, "tile shape: ty 4 or 8, ichunk 1..1024");
  if (ty != b->ty || ichunk != b->ichunk) {
    b->ty = ty;
    b->ichunk = ichunk;
    b->dirty = true;
  }
  return AWP_OK;
}

int awp_batch_set_mode(awp_batch* b, int mode) {
  if (!b) return set_error(AWP_ERR_ARG, "null batch");
  if (mode != 0 && mode != 1) return set_error(AWP_ERR_ARG, "batch mode 0 or 1");
  if (mode != b->mode) {
    b->mode = mode;
    b->dirty = true;
  }
  return AWP_OK;
}

int awp_batch_get_mode(const awp_batch* b) { return b ? b->mode : -1; }

int awp_batch_set_branches(awp_batch* b, int branches) {
  if (!b) return set_error(AWP_ERR_ARG, "null batch");
  if (branches < 0) return set_error(AWP_ERR_ARG, "branches >= 0");
  if (branches != b->branches) {
    b->branches = branches;
    b->dirty = true;
  }
  return AWP_OK;
}

int awp_batch_get_shape(const awp_batch* b, int* ty, int* ichunk) {
  if (!b || !ty || !ichunk) return set_error(AWP_ERR_ARG, "null argument");
  *ty = b->ty;
  *ichunk = b->ichunk;
  return AWP_OK;
}

int awp_batch_set_graph(awp_batch* b, int use_graph) {
  if (!b) return set_error(AWP_ERR_ARG, "null batch");
  if ((use_graph != 0) != b->use_graph) {
    b->use_graph = use_graph != 0;
    b->dirty = true;
  }
  return AWP_OK;
}

int awp_batch_step(awp_batch* b, int nsteps) {
  if (!b) return set_error(AWP_ERR_ARG, "null batch");
  if (nsteps < 0) return set_error(AWP_ERR_ARG, "nsteps < 0");
  for (awp_ctx* c : b->ctx)
    if (c->cur_step != b->step)
      return set_error(AWP_ERR_STATE, "an instance was stepped outside the batch");
  if (nsteps == 0) return AWP_OK;
  // order after each instance's earlier work; the step-1 source sample of
  // IFAULT < 4 is added before the first step (pmcl3d.c:1175-1187)
  for (awp_ctx* c : b->ctx) {
    if (c->cur_step == 0 && !c->initial_src_done) {
      if (c->p.ifault < 4) {
        int s = launch_sources(c, 0);
        if (s) return s;
        if (c->ncell) c->launches++;
      }
      c->initial_src_done = true;
    }
    CU_TRY(cudaEventRecord(b->ev, c->stream));
    CU_TRY(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  if (b->dirty) {
    int e = batch_build(b);
    if (e) return e;
  }
  for (int n = 0; n < nsteps; ++n) {
    if (b->use_graph || b->mode == 1)
      CU_TRY(cudaGraphLaunch(b->exec, b->stream));
    else
      CU_TRY(awp_launch_batch_step(b->L, b->stream));
  }
  CU_TRY(cudaEventRecord(b->ev, b->stream));
  for (awp_ctx* c : b->ctx) {
    CU_TRY(cudaStreamWaitEvent(c->stream, b->ev, 0));
    c->cur_step += nsteps;
  }
  b->ctx[0]->launches += b->launches_per_step * nsteps;
  b->step += nsteps;
  return AWP_OK;
}

int awp_batch_synchronize(awp_batch* b) {
  if (!b) return set_error(AWP_ERR_ARG, "null batch");
  CU_TRY(cudaStreamSynchronize(b->stream));
  return AWP_OK;
}

int awp_batch_info(awp_batch* b, long long info[6]) {
  if (!b || !info) return set_error(AWP_ERR_ARG, "null argument");
  if (b->dirty) {
    int e = batch_build(b);
    if (e) return e;
  }
  info[0] = (long long)b->ctx.size();
  info[1] = b->cells;
  info[2] = b->L.nvtiles;
  info[3] = (long long)b->L.nstiles + b->L.nstiles_el;
  info[4] = b->L.grid_vel;
  info[5] = b->L.grid_str;
  return AWP_OK;
}

int awp_set_topo_plasticity(awp_ctx* c, int consistent) {
  if (!c || (consistent != 0 && consistent != 1))
    return set_error(AWP_ERR_ARG, "null context or mode not 0/1");
  c->topo_plastic_consistent = consistent;
  return AWP_OK;
}

int awp_topography_init(awp_ctx* c, const char* intopo) {
  if (!c || !intopo) return set_error(AWP_ERR_ARG, "null argument");
  if (c->topo) return set_error(AWP_ERR_STATE, "topography already initialised");
  if (c->recv || c->srcf || c->forcef || c->sgt)
    return set_error(AWP_ERR_STATE,
                     "topography must be initialised before receivers, SGT output, "
                     "SOURCEFILE sources and FORCEFILE forces");
  if (c->p.grid != 0)
    return set_error(AWP_ERR_ARG, "topography belongs to the top grid (grid 0) only");
  const int nx = c->g.nxt, ny = c->g.nyt, nz = c->g.nzt;
  if (nz < 12) return set_error(AWP_ERR_ARG, "topography needs nzt >= 12 (got %d)", nz);
  // a sub-domain builds the whole grid's metrics and keeps its own planes
  const int nxg = c->sub_nxg ? c->sub_nxg : nx, x0 = c->sub_nxg ? c->sub_x0 : 0;
  awp::TopoMetrics* m = new awp::TopoMetrics();
  awp::topo_init_metrics(m, nxg, ny, nz, c->p.dh);
  const int e = awp::topo_read_file(intopo, nxg, ny, &m->f);
  if (e) {
    delete m;
    return set_error(e == 902 ? AWP_ERR_ARG : AWP_ERR_IO,
                     e == 902 ? "%s: grid size or padding inconsistent with the context"
                              : "%s: cannot read the topography file",
                     intopo);
  }
  awp::topo_build_metrics(m);
  if (c->sub_nxg) {
    awp::TopoMetrics* part = new awp::TopoMetrics();
    awp::topo_init_metrics(part, nx, ny, nz, c->p.dh);
    std::vector<float>* dst[10] = {&part->f, &part->f_1, &part->f_2, &part->f_c, &part->f1_1,
                                   &part->f1_2, &part->f1_c, &part->f2_1, &part->f2_2,
                                   &part->f2_c};
    const std::vector<float>* src[10] = {&m->f, &m->f_1, &m->f_2, &m->f_c, &m->f1_1,
                                         &m->f1_2, &m->f1_c, &m->f2_1, &m->f2_2, &m->f2_c};
    const size_t row = (size_t)m->ld, rows = (size_t)nx + 4 + AWP_NGSL2;
    for (int q = 0; q < 10; ++q) {
      dst[q]->assign(src[q]->begin() + (size_t)x0 * row, src[q]->begin() + (size_t)x0 * row +
                                                             rows * row);
    }
    part->g = m->g; part->g_c = m->g_c; part->g3 = m->g3; part->g3_c = m->g3_c;
    delete m;
    m = part;
  }
  const size_t nf = m->f.size(), ng = m->g.size();
  float* d = nullptr;
  if (ctx_alloc(c, (void**)&d, sizeof(float) * (10 * nf + 4 * ng))) {
    delete m;
    return AWP_ERR_NOMEM;
  }
  const std::vector<float>* fa[10] = {&m->f, &m->f_1, &m->f_2, &m->f_c, &m->f1_1,
                                      &m->f1_2, &m->f1_c, &m->f2_1, &m->f2_2, &m->f2_c};
  const std::vector<float>* ga[4] = {&m->g, &m->g_c, &m->g3, &m->g3_c};
  cudaError_t ce = cudaSuccess;
  for (int q = 0; q < 10 && ce == cudaSuccess; ++q)
    ce = cudaMemcpy(d + q * nf, fa[q]->data(), nf * sizeof(float), cudaMemcpyHostToDevice);
  for (int q = 0; q < 4 && ce == cudaSuccess; ++q)
    ce = cudaMemcpy(d + 10 * nf + q * ng, ga[q]->data(), ng * sizeof(float),
                    cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    cudaFree(d);
    delete m;
    return set_error(AWP_ERR_CUDA, "topography upload: %s", cudaGetErrorString(ce));
  }
  TopoArgs& t = c->targs;
  t = TopoArgs{};
  t.f = d; t.f_1 = d + nf; t.f_2 = d + 2 * nf; t.f_c = d + 3 * nf;
  t.f1_1 = d + 4 * nf; t.f1_2 = d + 5 * nf; t.f1_c = d + 6 * nf;
  t.f2_1 = d + 7 * nf; t.f2_2 = d + 8 * nf; t.f2_c = d + 9 * nf;
  t.g = d + 10 * nf; t.g_c = d + 10 * nf + ng; t.g3 = d + 10 * nf + 2 * ng;
  t.g3_c = d + 10 * nf + 3 * ng;
  t.fld = m->ld;
  // topo_init (topography.c:69) and topo_set_constants (stress_attenuation.cu:19-23)
  const float h = c->p.dh, dt = c->p.dt;
  t.nu = dt / h;
  t.DT = t.nu * h;
  t.dth = t.DT / h;
  t.dh1 = (float)(1.0 / (double)h);
  // stress window of a rank on every domain boundary: ngsl/2 cells in from
  // each side (topo_set_stress_bounds_*, topography.c:379-420)
  t.s_i = std::max(AWP_NGSL / 2 - x0, 0); t.e_i = std::min(nxg - AWP_NGSL / 2 - x0, nx);
  t.s_j = AWP_NGSL / 2; t.e_j = ny - AWP_NGSL / 2;
  c->d_topo = d;
  c->topo = m;
  return AWP_OK;
}

// ===========================================================================
// Materials, reset, seismograms and the adjoint gradient
// ===========================================================================
}  // extern "C"

namespace {

int check_adjoint_ctx(awp_ctx* c) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "media not uploaded");
  if (c->p.ngrids != 1 || c->p.nve == 3 || c->topo || c->recv || c->srcf || c->forcef ||
      c->sgt)
    return set_error(AWP_ERR_UNSUPPORTED,
                     "the adjoint covers single-grid Cartesian runs without plasticity, "
                     "receiver or SGT files or SOURCEFILE sources");
  if (c->d_frc_pos || c->sub_nxg)
    return set_error(AWP_ERR_UNSUPPORTED,
                     "the adjoint covers neither prescribed velocities nor sub-domains");
  if (c->ncell > 0 && c->p.ifault != 1 && c->p.ifault != 2)
    return set_error(AWP_ERR_UNSUPPORTED,
                     "the adjoint takes IFAULT 1 or 2 sources (the kinematic source depends on "
                     "mu)");
  return AWP_OK;
}

// device copies of receiver positions (padded linear index) and components
int upload_receivers(awp_ctx* c, int nrec, const int* xyz, const int* comp, long long** d_idx,
                     int** d_comp) {
  std::vector<long long> idx(nrec);
  for (int r = 0; r < nrec; ++r) {
    const int x = xyz[3 * r], y = xyz[3 * r + 1], z = xyz[3 * r + 2];
    if (x < 0 || x >= c->g.nxt || y < 0 || y >= c->g.nyt || z < 0 || z >= c->g.nzt ||
        comp[r] < 0 || comp[r] > 2)
      return set_error(AWP_ERR_ARG, "receiver %d outside the grid or bad component", r);
    idx[r] = (long long)(x + 2 + AWP_NGSL) * c->g.slice +
             (long long)(y + 2 + AWP_NGSL) * c->g.yline + (c->g.top() - z);
  }
  CU_TRY(cudaMalloc((void**)d_idx, sizeof(long long) * std::max(nrec, 1)));
  CU_TRY(cudaMalloc((void**)d_comp, sizeof(int) * std::max(nrec, 1)));
  CU_TRY(cudaMemcpy(*d_idx, idx.data(), sizeof(long long) * nrec, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(*d_comp, comp, sizeof(int) * nrec, cudaMemcpyHostToDevice));
  return AWP_OK;
}

struct DevBuf {  // owned device allocations of one call
  std::vector<void*> p;
  ~DevBuf() {
    for (void* q : p) cudaFree(q);
  }
  float* f(size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, n * sizeof(float)) != cudaSuccess) return nullptr;
    p.push_back(q);
    return (float*)q;
  }
};

}  // namespace

extern "C" {

int awp_set_moduli(awp_ctx* c, const float* lambda, const float* mu, const float* rho) {
  if (!c || !lambda || !mu || !rho) return set_error(AWP_ERR_ARG, "null argument");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "upload media first (Q and layout)");
  const size_t n = (size_t)c->g.nxt * c->g.nyt * c->g.nzt;
  DevBuf b;
  float *dl = b.f(n), *dm = b.f(n), *dr = b.f(n);
  if (!dl || !dm || !dr) return set_error(AWP_ERR_NOMEM, "moduli staging");
  // host or device arrays alike (unified addressing picks the direction)
  CU_TRY(cudaMemcpyAsync(dl, lambda, n * sizeof(float), cudaMemcpyDefault, c->stream));
  CU_TRY(cudaMemcpyAsync(dm, mu, n * sizeof(float), cudaMemcpyDefault, c->stream));
  CU_TRY(cudaMemcpyAsync(dr, rho, n * sizeof(float), cudaMemcpyDefault, c->stream));
  CU_TRY(awp_launch_set_moduli(dl, dm, dr, c->f[AWP_LAM], c->f[AWP_MU], c->f[AWP_D1], c->g,
                               c->stream));
  CU_TRY(awp_launch_lam_mu(c->f[AWP_LAM], c->f[AWP_MU], c->lam_mu, c->g, c->xls, c->xre, c->yls,
                           c->yre, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  return AWP_OK;
}

int awp_set_qinv(awp_ctx* c, const float* qpinv, const float* qsinv) {
  if (!c || !qpinv || !qsinv) return set_error(AWP_ERR_ARG, "null argument");
  if (!c->media_ready) return set_error(AWP_ERR_STATE, "upload media first (layout)");
  const size_t n = (size_t)c->g.nxt * c->g.nyt * c->g.nzt;
  bool any = false;
  for (size_t q = 0; q < n && !any; ++q) any = (qpinv[q] != 0.f) || (qsinv[q] != 0.f);
  DevBuf b;
  float *dp = b.f(n), *ds = b.f(n);
  if (!dp || !ds) return set_error(AWP_ERR_NOMEM, "Q staging");
  CU_TRY(cudaMemcpyAsync(dp, qpinv, n * sizeof(float), cudaMemcpyDefault, c->stream));
  CU_TRY(cudaMemcpyAsync(ds, qsinv, n * sizeof(float), cudaMemcpyDefault, c->stream));
  CU_TRY(awp_launch_set_qinv(dp, ds, c->f[AWP_QP], c->f[AWP_QS], c->g, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  // the elastic specialisation holds exactly when every Q^-1 is zero
  c->elastic = !any;
  return AWP_OK;
}

int awp_reset(awp_ctx* c) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  const size_t bytes = sizeof(float) * (size_t)c->g.cells_pad();
  for (int fld = AWP_U1; fld <= AWP_R6; ++fld)
    CU_TRY(cudaMemsetAsync(c->f[fld], 0, bytes, c->stream));
  c->cur_step = 0;
  c->initial_src_done = false;
  CU_TRY(cudaStreamSynchronize(c->stream));
  return AWP_OK;
}

int awp_seismograms(awp_ctx* c, int nsteps, int nrec, const int* rec_xyz, const int* rec_comp,
                    float* seis) {
  int e = check_adjoint_ctx(c);
  if (e) return e;
  if (nsteps < 0 || nrec < 1 || !rec_xyz || !rec_comp || !seis)
    return set_error(AWP_ERR_ARG, "bad receiver arguments");
  long long* d_idx = nullptr;
  int* d_comp = nullptr;
  e = upload_receivers(c, nrec, rec_xyz, rec_comp, &d_idx, &d_comp);
  DevBuf b;
  b.p.push_back(d_idx);
  b.p.push_back(d_comp);
  if (e) return e;
  float* d_seis = b.f((size_t)std::max(nsteps, 1) * nrec);
  if (!d_seis) return set_error(AWP_ERR_NOMEM, "seismogram buffer");
  for (int n = 0; n < nsteps; ++n) {
    if ((e = one_step(c))) return e;
    CU_TRY(awp_launch_sample(c->f[AWP_U1], c->f[AWP_V1], c->f[AWP_W1], d_idx, d_comp, nrec,
                             d_seis + (size_t)n * nrec, c->stream));
  }
  CU_TRY(cudaMemcpyAsync(seis, d_seis, sizeof(float) * (size_t)nsteps * nrec,
                         cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  return AWP_OK;
}

// Forward-state storage of the misfit gradient (two levels).  The last M
// steps keep their velocities from the first forward pass (no
// recomputation); the first H = N - M steps are covered by snapshots every
// L = ceil(sqrt(H)) steps and run forward again, one segment at a time,
// before their backward sweep.  nsnap > 0 fixes the snapshot count and
// stores no tail; nsnap = 0 takes the largest M that fits in 90 % of the free
// device memory (counting the workspace already held).
struct AdjPlan {
  VelBox vb;
  int M = 0, L = 1, nseg = 0;
  size_t floats = 0;  // workspace, slab pieces on 256-byte boundaries
};
static inline size_t slab_round(size_t n) { return (n + 63) / 64 * 64; }

static int adjoint_plan(awp_ctx* c, int nsteps, int nsnap, AdjPlan* out) {
  const size_t cp = (size_t)c->g.cells_pad();
  // the stored velocities cover what the adjoint kernels read of them
  // (velocity range, stress range +-2)
  const VelArgs va = make_vel_args(c);
  const StrArgs sa = make_str_args(c);
  VelBox& vb = out->vb;
  {
    const int i0 = std::min(va.i0, sa.i0 - 2), i1 = std::max(va.i1, sa.i1 + 2);
    const int j0 = std::min(va.j0, sa.j0 - 2), j1 = std::max(va.j1, sa.j1 + 2);
    const int k0 = std::min(va.k0, sa.k0 - 2) / 4 * 4, k1 = std::max(va.k1, sa.k1 + 2);
    vb.i0 = i0; vb.j0 = j0; vb.k0 = k0;
    vb.ni = i1 - i0 + 1; vb.nj = j1 - j0 + 1; vb.nk = k1 - k0 + 1;
    vb.ld = (vb.nk + 7) / 8 * 8;
    vb.Y = vb.ld;
    vb.S = (long long)vb.nj * vb.ld;
    vb.off = (long long)i0 * vb.S + (long long)j0 * vb.Y + k0;
  }
  const size_t cv = vb.cells();
  auto plan = [&](int M, int* Lp, int* nsegp) -> size_t {  // floats
    const int H = nsteps - M;
    int Lh = H > 0 ? (nsnap > 0 ? (H + nsnap - 1) / nsnap : (int)ceil(sqrt((double)H))) : 1;
    Lh = std::max(1, std::min(Lh, std::max(H, 1)));
    *Lp = Lh;
    *nsegp = H > 0 ? (H + Lh - 1) / Lh : 0;
    // snapshots, adjoint state (15), temporaries (16 + 6), gradients (5)
    return ((size_t)(*nsegp + 1) * 15 + 15 + 22 + 5) * slab_round(cp) +
           ((size_t)(H > 0 ? Lh + 1 : 0) + (size_t)(M > 0 ? M + 1 : 0)) * 3 * slab_round(cv);
  };
  int M = 0;
  out->floats = plan(0, &out->L, &out->nseg);
  if (nsnap <= 0) {
    size_t freeb = 0, totb = 0;
    CU_TRY(cudaMemGetInfo(&freeb, &totb));
    const double budget =
        0.9 * (double)(freeb + c->adj_slab_floats * sizeof(float)) - (256u << 20);
    int lo = 0, hi = nsteps;  // largest M whose plan fits the budget
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      int Lm, nm;
      if ((double)plan(mid, &Lm, &nm) * sizeof(float) <= budget)
        lo = mid;
      else
        hi = mid - 1;
    }
    M = lo;
    out->floats = plan(M, &out->L, &out->nseg);
  }
  out->M = M;
  return AWP_OK;
}

// The workspace of a plan: one slab, kept in the context for later calls.
static int ensure_adjoint_slab(awp_ctx* c, const AdjPlan& pl) {
  if (c->adj_slab_floats >= pl.floats) return AWP_OK;
  cudaFree(c->adj_slab);
  c->adj_slab = nullptr;
  c->adj_slab_floats = 0;
  size_t freeb = 0, totb = 0;
  CU_TRY(cudaMemGetInfo(&freeb, &totb));
  const double gb = pl.floats * sizeof(float) / 1e9;
  if (pl.floats * sizeof(float) + (64u << 20) > freeb)
    return set_error(AWP_ERR_NOMEM,
                     "adjoint needs %.1f GB (%d snapshots of %.1f MB fields, %d-step "
                     "segments), %.1f GB free",
                     gb, pl.nseg + 1, c->g.cells_pad() * 4.0 / 1e6, pl.L, freeb / 1e9);
  if (cudaMalloc((void**)&c->adj_slab, pl.floats * sizeof(float)) != cudaSuccess) {
    c->adj_slab = nullptr;
    return set_error(AWP_ERR_NOMEM, "adjoint workspace of %.1f GB", gb);
  }
  c->adj_slab_floats = pl.floats;
  // touch every page once here, so that the first gradient does not pay the
  // first-use mapping of the workspace
  CU_TRY(cudaMemsetAsync(c->adj_slab, 0, pl.floats * sizeof(float), c->stream));
  return AWP_OK;
}

int awp_adjoint_reserve(awp_ctx* c, int nsteps, int nsnap) {
  int e = check_adjoint_ctx(c);
  if (e) return e;
  if (nsteps < 1) return set_error(AWP_ERR_ARG, "nsteps < 1");
  AdjPlan pl;
  if ((e = adjoint_plan(c, nsteps, nsnap, &pl))) return e;
  return ensure_adjoint_slab(c, pl);
}

int awp_adjoint_plan(awp_ctx* c, int nsteps, int nsnap, int* tail_steps, int* segment_steps,
                     int* snapshots, double* workspace_gb) {
  int e = check_adjoint_ctx(c);
  if (e) return e;
  if (nsteps < 1) return set_error(AWP_ERR_ARG, "nsteps < 1");
  AdjPlan pl;
  if ((e = adjoint_plan(c, nsteps, nsnap, &pl))) return e;
  if (tail_steps) *tail_steps = pl.M;
  if (segment_steps) *segment_steps = pl.L;
  if (snapshots) *snapshots = pl.nseg + 1;
  if (workspace_gb) *workspace_gb = pl.floats * sizeof(float) / 1e9;
  return AWP_OK;
}

int awp_misfit_gradient(awp_ctx* c, int nsteps, int nrec, const int* rec_xyz, const int* rec_comp,
                        const float* d_obs, int nsnap, double* misfit, float* seis,
                        float* g_lambda, float* g_mu, float* g_rho) {
  return awp_misfit_gradient_q(c, nsteps, nrec, rec_xyz, rec_comp, d_obs, nsnap, misfit, seis,
                               g_lambda, g_mu, g_rho, nullptr, nullptr);
}

int awp_misfit_gradient_q(awp_ctx* c, int nsteps, int nrec, const int* rec_xyz,
                          const int* rec_comp, const float* d_obs, int nsnap, double* misfit,
                          float* seis, float* g_lambda, float* g_mu, float* g_rho,
                          float* g_qpinv, float* g_qsinv) {
  int e = check_adjoint_ctx(c);
  if (e) return e;
  if (nsteps < 1 || nrec < 1 || !rec_xyz || !rec_comp || !d_obs || !misfit)
    return set_error(AWP_ERR_ARG, "bad arguments");
  const size_t cp = (size_t)c->g.cells_pad();
  const size_t fb = cp * sizeof(float);
  AdjPlan pl;
  if ((e = adjoint_plan(c, nsteps, nsnap, &pl))) return e;
  const VelBox vb = pl.vb;
  const size_t cv = vb.cells();
  const int M = pl.M, L = pl.L, nseg = pl.nseg;
  const VelArgs va = make_vel_args(c);
  const StrArgs sa = make_str_args(c);
  auto rnd = slab_round;
  const int H = nsteps - M;
  // one slab for snapshots, stores, adjoint state, temporaries and gradients,
  // kept in the context for the next call
  if ((e = ensure_adjoint_slab(c, pl))) return e;
  size_t slab_next = 0;  // floats
  auto take_n = [&](size_t n) -> float* {
    float* q = c->adj_slab + slab_next;
    slab_next += rnd(n);
    return q;
  };
  auto take = [&]() -> float* { return take_n(cp); };
  auto take_v = [&]() -> float* { return take_n(cv); };
  DevBuf b;
  long long* d_idx = nullptr;
  int* d_comp = nullptr;
  e = upload_receivers(c, nrec, rec_xyz, rec_comp, &d_idx, &d_comp);
  b.p.push_back(d_idx);
  b.p.push_back(d_comp);
  if (e) return e;
  float* d_seis = b.f((size_t)nsteps * nrec);
  float* d_res = b.f((size_t)nsteps * nrec);
  if (!d_seis || !d_res) return set_error(AWP_ERR_NOMEM, "seismogram buffers");
  cudaStream_t st = c->stream;

  // ---- forward pass with snapshots X_{sL} and the final state ---------------------
  std::vector<float*> snap((size_t)(nseg + 1) * 15, nullptr);
  for (auto& q : snap) q = take();
  std::vector<long long> snap_step(nseg + 1);
  std::vector<char> snap_init(nseg + 1);
  auto save = [&](int s) -> int {
    for (int fld = 0; fld < 15; ++fld)
      CU_TRY(cudaMemcpyAsync(snap[(size_t)s * 15 + fld], c->f[fld], fb, cudaMemcpyDeviceToDevice, st));
    snap_step[s] = c->cur_step;
    snap_init[s] = c->initial_src_done;
    return AWP_OK;
  };
  auto restore = [&](int s) -> int {
    for (int fld = 0; fld < 15; ++fld)
      CU_TRY(cudaMemcpyAsync(c->f[fld], snap[(size_t)s * 15 + fld], fb, cudaMemcpyDeviceToDevice, st));
    c->cur_step = snap_step[s];
    c->initial_src_done = snap_init[s] != 0;
    return AWP_OK;
  };
  // tail store: the velocities at step H and after each later step
  std::vector<float*> tail((size_t)(M > 0 ? M + 1 : 0) * 3, nullptr);
  for (auto& q : tail) q = take_v();
  auto keep_vel = [&](float** dst) -> int {
    CU_TRY(awp_launch_pack_vel(c->f[AWP_U1], c->f[AWP_V1], c->f[AWP_W1], dst[0], dst[1], dst[2],
                               vb, c->g, st));
    return AWP_OK;
  };
  for (int n = 0; n < nsteps; ++n) {
    if (n < H && n % L == 0 && (e = save(n / L))) return e;
    if (n == H && M > 0 && (e = keep_vel(&tail[0]))) return e;
    if ((e = one_step(c))) return e;
    if (n >= H && (e = keep_vel(&tail[(size_t)(n - H + 1) * 3]))) return e;
    CU_TRY(awp_launch_sample(c->f[AWP_U1], c->f[AWP_V1], c->f[AWP_W1], d_idx, d_comp, nrec,
                             d_seis + (size_t)n * nrec, st));
  }
  if ((e = save(nseg))) return e;  // the final state, restored at the end

  // ---- misfit and residuals ---------------------------------------------------------
  std::vector<float> hs((size_t)nsteps * nrec), hr((size_t)nsteps * nrec);
  CU_TRY(cudaMemcpyAsync(hs.data(), d_seis, sizeof(float) * hs.size(), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  double J = 0.0;
  for (size_t q = 0; q < hs.size(); ++q) {
    hr[q] = hs[q] - d_obs[q];
    J += 0.5 * (double)hr[q] * (double)hr[q];
  }
  *misfit = J;
  if (seis) memcpy(seis, hs.data(), sizeof(float) * hs.size());
  CU_TRY(cudaMemcpyAsync(d_res, hr.data(), sizeof(float) * hr.size(), cudaMemcpyHostToDevice, st));

  // ---- adjoint state, temporaries, gradients (zeroed) --------------------------------
  AdjArgs a;
  memset(&a, 0, sizeof(a));
  // adjoint state, temporaries, gradients: 42 consecutive fields of the slab
  float* const zero0 = c->adj_slab + slab_next;
  for (int q = 0; q < 15; ++q) a.L[q] = take();
  for (int q = 0; q < 16; ++q) a.E[q] = take();
  for (int q = 0; q < 6; ++q) a.V[q] = take();
  a.gd = take();
  a.glam = take();
  a.gmu = take();
  a.gqp = take();
  a.gqs = take();
  CU_TRY(cudaMemsetAsync(zero0, 0, (size_t)(c->adj_slab + slab_next - zero0) * sizeof(float), st));
  if (!(a.glm = b.f((size_t)c->g.nx_pad() * c->g.ny_pad())))
    return set_error(AWP_ERR_NOMEM, "gradients");
  CU_TRY(cudaMemsetAsync(a.glm, 0, sizeof(float) * c->g.nx_pad() * c->g.ny_pad(), st));
  a.d1 = c->f[AWP_D1]; a.lam = c->f[AWP_LAM]; a.mu = c->f[AWP_MU];
  a.qp = c->f[AWP_QP]; a.qs = c->f[AWP_QS]; a.lam_mu = c->lam_mu;
  a.dcrjx = c->dcrjx; a.dcrjy = c->dcrjy; a.dcrjz = c->dcrjz;
  a.tex = c->tex;
  memcpy(a.coeff, c->coeff, sizeof(a.coeff));
  a.dth = c->dth; a.dh1 = c->dh1; a.dt = c->p.dt; a.c1 = c->c1; a.c2 = c->c2; a.qthr = c->qthr;
  a.elastic = c->elastic ? 1 : 0;
  a.want_q = (!c->elastic && (g_qpinv || g_qsinv)) ? 1 : 0;
  a.g = c->g;
  a.vb = vb;
  a.vi0 = va.i0; a.vi1 = va.i1; a.vj0 = va.j0; a.vj1 = va.j1; a.vk0 = va.k0; a.vk1 = va.k1;
  a.si0 = sa.i0; a.si1 = sa.i1; a.sj0 = sa.j0; a.sj1 = sa.j1; a.sk0 = sa.k0; a.sk1 = sa.k1;
  a.gx_lim = sa.gx_lim; a.gy_min = sa.gy_min; a.lam_mu_ld = sa.lam_mu_ld;
  a.fj1 = make_fstr_args(c).j1;
  if (!(a.img = b.f((size_t)4 * (a.si1 - a.si0 + 3) * (a.sj1 - a.sj0 + 3))))
    return set_error(AWP_ERR_NOMEM, "image scratch");
  // segment store: the velocities at the start of a segment and after each
  // of its steps (slot 0 = start)
  std::vector<float*> seg((size_t)(H > 0 ? L + 1 : 0) * 3, nullptr);
  for (auto& q : seg) q = take_v();
  float* const Lvel[3] = {a.L[0], a.L[1], a.L[2]};
  // receivers grouped by (component, cell) for the residual injection
  int* d_first = nullptr;
  int* d_order = nullptr;
  int ncell_rec = 0;
  {
    std::vector<std::pair<long long, int>> key(nrec);
    for (int r = 0; r < nrec; ++r) {
      const int x = rec_xyz[3 * r], y = rec_xyz[3 * r + 1], z = rec_xyz[3 * r + 2];
      key[r] = {((long long)rec_comp[r] << 48) | (((long long)x * c->g.nyt + y) * c->g.nzt + z), r};
    }
    std::stable_sort(key.begin(), key.end(),
                     [](const std::pair<long long, int>& u, const std::pair<long long, int>& v) {
                       return u.first < v.first;
                     });
    std::vector<int> first, order(nrec);
    for (int r = 0; r < nrec; ++r) {
      if (r == 0 || key[r].first != key[r - 1].first) first.push_back(r);
      order[r] = key[r].second;
    }
    ncell_rec = (int)first.size();
    first.push_back(nrec);
    CU_TRY(cudaMalloc((void**)&d_first, sizeof(int) * first.size()));
    b.p.push_back(d_first);
    CU_TRY(cudaMalloc((void**)&d_order, sizeof(int) * order.size()));
    b.p.push_back(d_order);
    CU_TRY(cudaMemcpy(d_first, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice));
    CU_TRY(cudaMemcpy(d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
  }

  // ---- backward sweep: the stored tail, then the recomputed segments ---------------
  auto back_step = [&](int n, float** before, float** after) -> int {
    // the misfit term of the state after step n (its sample index is n)
    CU_TRY(awp_launch_adjoint_inject(Lvel, d_idx, d_comp, d_first, d_order, ncell_rec,
                                     d_res + (size_t)n * nrec, st));
    a.bu = before[0]; a.bv = before[1]; a.bw = before[2];
    a.fu = after[0]; a.fv = after[1]; a.fw = after[2];
    CU_TRY(awp_launch_adjoint_step(a, st));
    return AWP_OK;
  };
  for (int n = nsteps - 1; n >= H; --n)
    if ((e = back_step(n, &tail[(size_t)(n - H) * 3], &tail[(size_t)(n - H + 1) * 3]))) return e;
  for (int s = nseg - 1; s >= 0; --s) {
    const int n0 = s * L, n1 = std::min(H, n0 + L);
    if ((e = restore(s))) return e;
    if ((e = keep_vel(&seg[0]))) return e;
    for (int n = n0; n < n1; ++n) {
      if ((e = one_step(c))) return e;
      if ((e = keep_vel(&seg[(size_t)(n - n0 + 1) * 3]))) return e;
    }
    for (int n = n1 - 1; n >= n0; --n)
      if ((e = back_step(n, &seg[(size_t)(n - n0) * 3], &seg[(size_t)(n - n0 + 1) * 3])))
        return e;
  }

  // ---- gradients to the host; the context ends on the final forward state -----------
  // staged in three strain-rate temporaries of the slab, free after the sweep
  // (no allocation per call on a device the workspace nearly fills)
  const size_t ni = (size_t)c->g.nxt * c->g.nyt * c->g.nzt;
  float *gl = a.E[0], *gm = a.E[1], *gr = a.E[2], *gqp = a.E[3], *gqs = a.E[4];
  CU_TRY(awp_launch_adjoint_fold(a, gl, gm, gr, st));
  if (g_qpinv || g_qsinv) CU_TRY(awp_launch_adjoint_fold_q(a, gqp, gqs, st));
  // host or device targets alike (unified addressing picks the direction)
  if (g_lambda) CU_TRY(cudaMemcpyAsync(g_lambda, gl, ni * sizeof(float), cudaMemcpyDefault, st));
  if (g_mu) CU_TRY(cudaMemcpyAsync(g_mu, gm, ni * sizeof(float), cudaMemcpyDefault, st));
  if (g_rho) CU_TRY(cudaMemcpyAsync(g_rho, gr, ni * sizeof(float), cudaMemcpyDefault, st));
  if (g_qpinv) CU_TRY(cudaMemcpyAsync(g_qpinv, gqp, ni * sizeof(float), cudaMemcpyDefault, st));
  if (g_qsinv) CU_TRY(cudaMemcpyAsync(g_qsinv, gqs, ni * sizeof(float), cudaMemcpyDefault, st));
  if ((e = restore(nseg))) return e;
  CU_TRY(cudaStreamSynchronize(st));
  return AWP_OK;
}

int awp_check_finite(awp_ctx* c, int* ok) {
  if (!c || !ok) return set_error(AWP_ERR_ARG, "null argument");
  CU_TRY(cudaMemsetAsync(c->d_flag, 0, sizeof(unsigned int), c->stream));
  for (int fld = AWP_U1; fld <= AWP_YZ; ++fld)
    CU_TRY(awp_launch_nonfinite(c->f[fld], c->g.cells_pad(), c->d_flag, c->stream));
  unsigned int h = 0;
  CU_TRY(cudaMemcpyAsync(&h, c->d_flag, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  *ok = h ? 0 : 1;
  return AWP_OK;
}

int awp_profile_phases(awp_ctx* c, int enable) {
  if (!c) return set_error(AWP_ERR_ARG, "null context");
  c->profile = enable != 0;
  return AWP_OK;
}

int awp_phase_times(awp_ctx* c, double ms[AWP_NPHASES], long long launches[AWP_NPHASES]) {
  if (!c || !ms || !launches) return set_error(AWP_ERR_ARG, "null argument");
  CU_TRY(cudaStreamSynchronize(c->stream));
  for (int p = 0; p < AWP_NPHASES; ++p) {
    ms[p] = 0.0;
    launches[p] = 0;
  }
  for (auto& e : c->ev_used) {
    float t = 0.f;
    CU_TRY(cudaEventElapsedTime(&t, e.a, e.b));
    ms[e.phase] += t;
    launches[e.phase] += 1;
    c->ev_free.push_back(e);
  }
  c->ev_used.clear();
  return AWP_OK;
}

int awp_set_tuning(const char* key, int value) {
  if (!key || awp_tuning_set(key, value))
    return set_error(AWP_ERR_ARG, "tuning %s=%d not accepted", key ? key : "(null)", value);
  return AWP_OK;
}

int awp_get_tuning(const char* key) { return key ? awp_tuning_get(key) : -1; }

int awp_kernel_launches(const awp_ctx* c, long long* launches) {
  if (!c || !launches) return set_error(AWP_ERR_ARG, "null argument");
  *launches = c->launches;
  return AWP_OK;
}

int awp_device_bytes(const awp_ctx* c, long long* bytes) {
  if (!c || !bytes) return set_error(AWP_ERR_ARG, "null argument");
  *bytes = c->dev_bytes;
  return AWP_OK;
}

// --------------------------------------------------------------------------
// host set-up helpers
// --------------------------------------------------------------------------
int awp_q_tau(float ex, float fac, float* taumax, float* taumin, float tau8[8]) {
  if (!awp::tau_range(ex, fac, taumax, taumin))
    return set_error(AWP_ERR_UNSUPPORTED, "EX=%g has no relaxation-time range", ex);
  awp::tausub(*taumin, *taumax, tau8);
  return AWP_OK;
}

int awp_q_weights(float ex, float fac, float w8[8], float coeff16[16]) {
  awp::weights_sub(ex, fac, w8, coeff16);
  return AWP_OK;
}

int awp_cerjan(float arbc, int nxt, int nyt, int nzt, int nd, int islowest, int npc,
               float* dcrjx, float* dcrjy, float* dcrjz) {
  for (int i = 0; i < nxt + 4 + AWP_NGSL2; ++i) dcrjx[i] = 1.0f;
  for (int i = 0; i < nyt + 4 + AWP_NGSL2; ++i) dcrjy[i] = 1.0f;
  for (int i = 0; i < nzt + 2 * AWP_ALIGN; ++i) dcrjz[i] = 1.0f;
  awp::inicrj(arbc, nxt, nyt, nzt, nxt, nyt, nd, islowest, npc, dcrjx, dcrjy, dcrjz);
  return AWP_OK;
}

int awp_texture_at(const float tau8[8], const float w8[8], float dt, int xls, int yls, int ny,
                   int nzt, int i, int j, int k, float* vx1, float* vx2, int* ww, float* wwo) {
  AwpTexture t{};
  awp::texture_tables(tau8, w8, dt, &t);
  t.xls = xls;
  t.yls = yls;
  t.ny = ny;
  t.nzt = nzt;
  const int idx = awp_tex_index(t, i, j, k);
  *vx1 = t.tau1[idx];
  *vx2 = t.tau2[idx];
  *wwo = t.wwo8[idx];
  *ww = idx + 1;
  return AWP_OK;
}

}  // extern "C"
