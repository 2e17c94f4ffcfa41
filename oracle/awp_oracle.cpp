// CPU oracle for the AWP-ODC time step -- TEST INFRASTRUCTURE ONLY.
//
// Each routine restates one reference kernel point by point, citing the
// reference lines it follows.  Arithmetic is carried out in T throughout
// (T = double: FP64 oracle; T = float: OpenMP CPU baseline).
#include "awp_oracle.h"

#include <math.h>
#include <omp.h>
#include <xmmintrin.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <vector>

namespace {

constexpr int NGSL = 8, NGSL2 = 16, ALIGN = 32, MAXFILT = 20;

// Dual number (value, tangent) in double: the oracle instantiated on it
// carries the exact derivative of every state value along one direction of
// the materials (tangent-linear mode), the discrete derivative the adjoint
// gradient must reproduce.  Branches compare values.
struct Dual {
  double v = 0.0, d = 0.0;
  Dual() = default;
  Dual(double x) : v(x) {}  // NOLINT (implicit from constants and floats)
  Dual(double x, double y) : v(x), d(y) {}
  explicit operator double() const { return v; }
  explicit operator float() const { return (float)v; }
  explicit operator int() const { return (int)v; }
  Dual& operator+=(const Dual& b) { v += b.v; d += b.d; return *this; }
  Dual& operator-=(const Dual& b) { v -= b.v; d -= b.d; return *this; }
  Dual& operator*=(const Dual& b) { d = d * b.v + v * b.d; v *= b.v; return *this; }
  Dual& operator/=(const Dual& b) { d = (d * b.v - v * b.d) / (b.v * b.v); v /= b.v; return *this; }
};
inline Dual operator+(Dual a, const Dual& b) { return a += b; }
inline Dual operator-(Dual a, const Dual& b) { return a -= b; }
inline Dual operator*(Dual a, const Dual& b) { return a *= b; }
inline Dual operator/(Dual a, const Dual& b) { return a /= b; }
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
using ::cos;  // keep the double overloads visible beside the Dual ones
using ::exp;
using ::sin;
using ::sqrt;
inline Dual sin(const Dual& a) { return Dual(::sin(a.v), ::cos(a.v) * a.d); }
inline Dual cos(const Dual& a) { return Dual(::cos(a.v), -::sin(a.v) * a.d); }
inline Dual exp(const Dual& a) { const double e = ::exp(a.v); return Dual(e, e * a.d); }
inline Dual sqrt(const Dual& a) { const double r = ::sqrt(a.v); return Dual(r, a.d / (2.0 * r)); }
inline double tangent(const Dual& a) { return a.d; }
inline double tangent(double) { return 0.0; }
inline double tangent(float) { return 0.0; }
inline void set_tangent(Dual& a, double t) { a.d = t; }
inline void set_tangent(double&, double) {}
inline void set_tangent(float&, double) {}

struct Base {
  virtual ~Base() {}
  virtual void set_field(int f, const float* s) = 0;
  virtual void get_field(int f, float* d) = 0;
  virtual void get_field64(int f, double* d) = 0;
  virtual void set_ww(const int* w) = 0;
  virtual void set_sponge(const float* x, const float* y, const float* z) = 0;
  virtual void set_coeff(const float* c) = 0;
  virtual void compute_lam_mu() = 0;
  virtual void set_sources(int ifault, int nsrc, const int* psrc, int stride, int nst,
                           const float* const a[6]) = 0;
  virtual void set_filter(int order, const double* b, const double* a) = 0;
  virtual void get_moment(float* m) = 0;
  virtual void set_plasticity(float fmajor, float fminor, const float* Rz, const float* RzT) = 0;
  virtual void set_plane_wave(int n, int nd, const float* vx, const float* vy,
                              const float* vz) = 0;
  virtual void add_point_sources(int field, int nq, int nb, const int* ix, const int* iy,
                                 const int* iz, const float* lx, const float* ly, const float* lz,
                                 int nsamples, const float* values, int stride) = 0;
  virtual void step(int nve, int n) = 0;
  virtual long long current() = 0;
  virtual void gather(int nbgx, int nedx, int nskpx, int nbgy, int nedy, int nskpy, int nbgz,
                      int nedz, int nskpz, float* bx, float* by, float* bz) = 0;
  virtual void set_tangent_field(int f, const double* t) = 0;
  virtual void get_tangent_field(int f, double* t) = 0;
};

template <typename T>
struct Oracle : Base {
  int nxt, nyt, nzt, npc, nthreads;
  long long slice, yline, ncell;
  T DH, DT, dth, dh1, c1, c2;
  std::vector<T> f[28];
  std::vector<int> ww;
  std::vector<T> dcrjx, dcrjy, dcrjz, lam_mu;
  T coeff[16] = {};
  // sources
  int ifault = 0, nsrc = 0, stride = 0, nst = 0;
  std::vector<int> psrc;
  std::vector<T> src[6];
  std::vector<T> mom;
  int filtorder = 0;
  double fb[MAXFILT] = {}, fa[MAXFILT] = {};
  std::vector<double> filt_state;
  // plasticity
  T fmajor = 0, fminor = 0, Rz[9] = {}, RzT[9] = {};
  // IFAULT 6 plane wave (ini_plane_wave) and the level it enters
  std::vector<T> plane[3];
  int plane_n = 0, plane_nd = 0;
  // SOURCEFILE moment tensors, one entry per stress component
  struct PointSrc {
    int field, nq, nb, nsamples, stride;
    std::vector<int> ix, iy, iz;
    std::vector<float> lx, ly, lz, values;  // values[nsamples][nq]
  };
  std::vector<PointSrc> psrcs;
  long long cur = 0;
  bool initial_done = false;

  enum { U1, V1, W1, XX, YY, ZZ, XY, XZ, YZ, R1, R2, R3, R4, R5, R6, D1, MU, LAM, QP, QS,
         SIGMA2, COHES, PHI, YLDFAC, NETA, VX1, VX2, WWO };

  Oracle(int nx_, int ny_, int nz_, float dh, float dt, int npc_, int nth)
      : nxt(nx_), nyt(ny_), nzt(nz_), npc(npc_), nthreads(nth) {
    yline = nzt + 2 * ALIGN;
    slice = (long long)(nyt + 4 + NGSL2) * yline;
    ncell = (long long)(nxt + 4 + NGSL2) * slice;
    for (auto& v : f) v.assign(ncell, T(0));
    f[YLDFAC].assign(ncell, T(1));  // pmcl3d.c:842-849
    ww.assign(ncell, 0);
    dcrjx.assign(nxt + 4 + NGSL2, T(1));
    dcrjy.assign(nyt + 4 + NGSL2, T(1));
    dcrjz.assign(nzt + 2 * ALIGN, T(1));
    lam_mu.assign((long long)(nxt + 4 + NGSL2) * (nyt + 4 + NGSL2), T(0));
    DH = dh;
    DT = dt;
    // SetDeviceConstValue (kernel.cu:68-100)
    dth = DT / DH;
    dh1 = T(1) / DH;
    c1 = T(9) / T(8);
    c2 = T(-1) / T(24);
  }

  long long idx(int i, int j, int k) const { return i * slice + j * yline + k; }

  void set_field(int fi, const float* s) override {
    for (long long n = 0; n < ncell; ++n) f[fi][n] = (T)s[n];
  }
  void get_field(int fi, float* d) override {
    for (long long n = 0; n < ncell; ++n) d[n] = (float)f[fi][n];
  }
  void get_field64(int fi, double* d) override {
    for (long long n = 0; n < ncell; ++n) d[n] = (double)f[fi][n];
  }
  void set_ww(const int* w) override { memcpy(ww.data(), w, sizeof(int) * ncell); }
  void set_tangent_field(int fi, const double* t) override {
    for (long long n = 0; n < ncell; ++n) set_tangent(f[fi][n], t[n]);
  }
  void get_tangent_field(int fi, double* t) override {
    for (long long n = 0; n < ncell; ++n) t[n] = tangent(f[fi][n]);
  }
  void set_sponge(const float* x, const float* y, const float* z) override {
    for (size_t n = 0; n < dcrjx.size(); ++n) dcrjx[n] = x[n];
    for (size_t n = 0; n < dcrjy.size(); ++n) dcrjy[n] = y[n];
    for (size_t n = 0; n < dcrjz.size(); ++n) dcrjz[n] = z[n];
  }
  void set_coeff(const float* c) override {
    for (int n = 0; n < 16; ++n) coeff[n] = c[n];
  }
  // pmcl3d.c:944-951 (over xls..xre x yls..yre at one rank)
  void compute_lam_mu() override {
    const int ktop = nzt + ALIGN - 1;
    for (int i = 2 + NGSL; i <= nxt + NGSL + 1; i++)
      for (int j = 2 + NGSL; j <= nyt + NGSL + 1; j++) {
        const T t_xl = T(1) / f[LAM][idx(i, j, ktop)];
        const T t_xl2m = T(2) / f[MU][idx(i, j, ktop)] + t_xl;
        lam_mu[(long long)i * (nyt + 4 + NGSL2) + j] = t_xl / t_xl2m;
      }
  }
  void set_sources(int ifault_, int nsrc_, const int* ps, int stride_, int nst_,
                   const float* const a[6]) override {
    ifault = ifault_;
    nsrc = nsrc_;
    stride = stride_;
    nst = nst_;
    psrc.assign(ps, ps + 3 * nsrc);
    for (int q = 0; q < 6; ++q) {
      src[q].resize((size_t)nsrc * stride);
      for (size_t n = 0; n < src[q].size(); ++n) src[q][n] = a[q][n];
    }
    mom.assign(nsrc, T(0));
    filt_state.assign((size_t)nsrc * (filtorder + 1), 0.0);
  }
  void set_filter(int order, const double* b, const double* a) override {
    filtorder = order;
    for (int n = 0; n <= order && order > 0; ++n) {
      fb[n] = b[n];
      fa[n] = a[n];
    }
    filt_state.assign((size_t)nsrc * (filtorder + 1), 0.0);
  }
  void get_moment(float* m) override {
    for (int s = 0; s < nsrc; ++s) m[s] = (float)mom[s];
  }
  void set_plasticity(float fmaj, float fmin, const float* rz, const float* rzt) override {
    fmajor = fmaj;
    fminor = fmin;
    for (int n = 0; n < 9; ++n) {
      Rz[n] = rz[n];
      RzT[n] = rzt[n];
    }
  }
  long long current() override { return cur; }

  // ---- dvelcx_opt (kernel.cu:125-268), i = xvs..xve, full launched j/k rows
  void velocity() {
    T* u1 = f[U1].data(); T* v1 = f[V1].data(); T* w1 = f[W1].data();
    const T* xx = f[XX].data(); const T* yy = f[YY].data(); const T* zz = f[ZZ].data();
    const T* xy = f[XY].data(); const T* xz = f[XZ].data(); const T* yz = f[YZ].data();
    const T* d1 = f[D1].data();
    const int j0 = 2 + NGSL, j1 = 2 + NGSL + (nyt + 1) / 2 * 2 - 1;
    const int k0 = ALIGN, k1 = ALIGN + (nzt + 3) / 4 * 4 - 1;
    const long long S = slice, Y = yline;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 2 + NGSL; i <= nxt + NGSL + 1; i++)
      for (int j = j0; j <= j1; j++) {
        const T dcrjyz_y = dcrjy[j];
#pragma omp simd
        for (int k = k0; k <= k1; k++) {
          const long long p = i * S + j * Y + k;
          const T f_dcrj = dcrjx[i] * dcrjyz_y * dcrjz[k];
          T f_d1 = T(0.25) * (d1[p] + d1[p - Y] + d1[p - 1] + d1[p - Y - 1]);
          T f_d2 = T(0.25) * (d1[p] + d1[p + S] + d1[p - 1] + d1[p + S - 1]);
          T f_d3 = T(0.25) * (d1[p] + d1[p + S] + d1[p - Y] + d1[p + S - Y]);
          f_d1 = dth / f_d1;
          f_d2 = dth / f_d2;
          f_d3 = dth / f_d3;
          u1[p] = (u1[p] + f_d1 * (c1 * (xx[p] - xx[p - S]) + c2 * (xx[p + S] - xx[p - 2 * S]) +
                                   c1 * (xy[p] - xy[p - Y]) + c2 * (xy[p + Y] - xy[p - 2 * Y]) +
                                   c1 * (xz[p] - xz[p - 1]) + c2 * (xz[p + 1] - xz[p - 2]))) *
                  f_dcrj;
          v1[p] = (v1[p] + f_d2 * (c1 * (xy[p + S] - xy[p]) + c2 * (xy[p + 2 * S] - xy[p - S]) +
                                   c1 * (yy[p + Y] - yy[p]) + c2 * (yy[p + 2 * Y] - yy[p - Y]) +
                                   c1 * (yz[p] - yz[p - 1]) + c2 * (yz[p + 1] - yz[p - 2]))) *
                  f_dcrj;
          w1[p] = (w1[p] + f_d3 * (c1 * (xz[p + S] - xz[p]) + c2 * (xz[p + 2 * S] - xz[p - S]) +
                                   c1 * (yz[p] - yz[p - Y]) + c2 * (yz[p + Y] - yz[p - 2 * Y]) +
                                   c1 * (zz[p + 1] - zz[p]) + c2 * (zz[p + 2] - zz[p - 1]))) *
                  f_dcrj;
        }
      }
  }

  // Q(f) weight, kernel.cu:974-1040
  T qfw(T q, T wwo, int w) const {
    T r;
    if (T(1) / (q * T(2)) <= T(200))
      r = coeff[w * 2 - 2] * (T(2) * q) * (T(2) * q) + coeff[w * 2 - 1] * (T(2) * q);
    else
      r = T(2) * wwo * q;
    return r / wwo;
  }

  // ---- dstrqc (kernel.cu:880-1197) at one cell
  void stress_cell(int i, int j, int k, int NX) {
    T* xx = f[XX].data(); T* yy = f[YY].data(); T* zz = f[ZZ].data();
    T* xy = f[XY].data(); T* xz = f[XZ].data(); T* yz = f[YZ].data();
    T* r1 = f[R1].data(); T* r2 = f[R2].data(); T* r3 = f[R3].data();
    T* r4 = f[R4].data(); T* r5 = f[R5].data(); T* r6 = f[R6].data();
    T* u1 = f[U1].data(); T* v1 = f[V1].data(); T* w1 = f[W1].data();
    const T* lam = f[LAM].data(); const T* mu = f[MU].data();
    const T* qp = f[QP].data(); const T* qs = f[QS].data();
    const long long S = slice, Y = yline;
    const long long pos = i * S + j * Y + k;
    const long long ip1 = pos + S, jm1 = pos - Y, km1 = pos - 1, ijk = pos + S - Y,
                    ik1 = pos + S - 1, jk1 = pos - Y - 1, ijk1 = pos + S - Y - 1;
    const T f_vx1 = f[VX1][pos], f_vx2 = f[VX2][pos], f_wwo = f[WWO][pos];
    const int f_ww = ww[pos];
    const T f_dcrj = dcrjx[i] * dcrjy[j] * dcrjz[k];
    T xl = T(8) / (lam[pos] + lam[ip1] + lam[jm1] + lam[ijk] + lam[km1] + lam[ik1] + lam[jk1] +
                   lam[ijk1]);
    T xm = T(16) / (mu[pos] + mu[ip1] + mu[jm1] + mu[ijk] + mu[km1] + mu[ik1] + mu[jk1] +
                    mu[ijk1]);
    T xmu1 = T(2) / (mu[pos] + mu[km1]);
    T xmu2 = T(2) / (mu[pos] + mu[jm1]);
    T xmu3 = T(2) / (mu[pos] + mu[ip1]);
    xl = xl + xm;
    T qpa = T(0.0625) * (qp[pos] + qp[ip1] + qp[jm1] + qp[ijk] + qp[km1] + qp[ik1] + qp[jk1] +
                         qp[ijk1]);
    const T qpaw = qfw(qpa, f_wwo, f_ww);
    T h = T(0.0625) * (qs[pos] + qs[ip1] + qs[jm1] + qs[ijk] + qs[km1] + qs[ik1] + qs[jk1] +
                       qs[ijk1]);
    const T hw = qfw(h, f_wwo, f_ww);
    T h1 = T(0.25) * (qs[pos] + qs[km1]);
    const T h1w = qfw(h1, f_wwo, f_ww);
    T h2 = T(0.25) * (qs[pos] + qs[jm1]);
    const T h2w = qfw(h2, f_wwo, f_ww);
    T h3 = T(0.25) * (qs[pos] + qs[ip1]);
    const T h3w = qfw(h3, f_wwo, f_ww);
    h = -xm * hw * dh1;
    h1 = -xmu1 * h1w * dh1;
    h2 = -xmu2 * h2w * dh1;
    h3 = -xmu3 * h3w * dh1;
    qpa = -qpaw * xl * dh1;
    xm = xm * dth;
    xmu1 = xmu1 * dth;
    xmu2 = xmu2 * dth;
    xmu3 = xmu3 * dth;
    xl = xl * dth;
    h = h * f_vx1;
    h1 = h1 * f_vx1;
    h2 = h2 * f_vx1;
    h3 = h3 * f_vx1;
    qpa = qpa * f_vx1;
    xm = xm + DT * h;
    xmu1 = xmu1 + DT * h1;
    xmu2 = xmu2 + DT * h2;
    xmu3 = xmu3 + DT * h3;
    const T vx1 = DT * (T(1) + f_vx2 * f_vx1);

    const T u1_ip2 = u1[pos + 2 * S], u1_ip1 = u1[pos + S], f_u1 = u1[pos], u1_im1 = u1[pos - S];
    const T v1_ip1 = v1[pos + S], f_v1 = v1[pos], v1_im1 = v1[pos - S], v1_im2 = v1[pos - 2 * S];
    const T w1_ip1 = w1[pos + S], f_w1 = w1[pos], w1_im1 = w1[pos - S], w1_im2 = w1[pos - 2 * S];
    const int ktop = nzt + ALIGN - 1;
    // free-surface velocity images on grid 0 (kernel.cu:1087-1112)
    if (k == ktop) {
      u1[pos + 1] = f_u1 - (f_w1 - w1_im1);
      v1[pos + 1] = f_v1 - (w1[pos + Y] - f_w1);
      int g_i = i - NGSL - 1;
      const T vs1 = (g_i < NX) ? u1_ip1 - (w1_ip1 - f_w1) : T(0);
      g_i = j - NGSL - 1;
      const T vs2 = (g_i > 1 || npc == 2) ? v1[jm1] - (f_w1 - w1[jm1]) : T(0);
      w1[pos + 1] = w1[km1] - lam_mu[(long long)i * (nyt + 4 + NGSL2) + j] *
                                  ((vs1 - u1[pos + 1]) + (u1_ip1 - f_u1) + (v1[pos + 1] - vs2) +
                                   (f_v1 - v1[jm1]));
    } else if (k == ktop - 1) {
      u1[pos + 2] = u1[pos + 1] - (w1[pos + 1] - w1[pos - S + 1]);
      v1[pos + 2] = v1[pos + 1] - (w1[pos + Y + 1] - w1[pos + 1]);
    }

    T vs1 = c1 * (u1_ip1 - f_u1) + c2 * (u1_ip2 - u1_im1);
    T vs2 = c1 * (f_v1 - v1[jm1]) + c2 * (v1[pos + Y] - v1[pos - 2 * Y]);
    T vs3 = c1 * (f_w1 - w1[km1]) + c2 * (w1[pos + 1] - w1[pos - 2]);
    T tmp = xl * (vs1 + vs2 + vs3);
    const T a1 = qpa * (vs1 + vs2 + vs3);
    tmp = tmp + DT * a1;

    T f_r = r1[pos];
    T f_rtmp = -h * (vs2 + vs3) + a1;
    xx[pos] = xx[pos] + tmp - xm * (vs2 + vs3) + vx1 * f_r;
    r1[pos] = f_vx2 * f_r + f_wwo * f_rtmp;
    f_rtmp = f_rtmp * (f_wwo - T(1)) + f_vx2 * f_r * (T(1) - f_vx1);
    xx[pos] = (xx[pos] + DT * f_rtmp) * f_dcrj;

    f_r = r2[pos];
    f_rtmp = -h * (vs1 + vs3) + a1;
    yy[pos] = (yy[pos] + tmp - xm * (vs1 + vs3) + vx1 * f_r) * f_dcrj;
    r2[pos] = f_vx2 * f_r + f_wwo * f_rtmp;
    f_rtmp = f_rtmp * (f_wwo - T(1)) + f_vx2 * f_r * (T(1) - f_vx1);
    yy[pos] = (yy[pos] + DT * f_rtmp) * f_dcrj;

    f_r = r3[pos];
    f_rtmp = -h * (vs1 + vs2) + a1;
    zz[pos] = (zz[pos] + tmp - xm * (vs1 + vs2) + vx1 * f_r) * f_dcrj;
    r3[pos] = f_vx2 * f_r + f_wwo * f_rtmp;
    f_rtmp = f_rtmp * (f_wwo - T(1)) + f_vx2 * f_r * (T(1) - f_vx1);
    zz[pos] = (zz[pos] + DT * f_rtmp) * f_dcrj;

    vs1 = c1 * (u1[pos + Y] - f_u1) + c2 * (u1[pos + 2 * Y] - u1[jm1]);
    vs2 = c1 * (f_v1 - v1_im1) + c2 * (v1_ip1 - v1_im2);
    f_r = r4[pos];
    f_rtmp = h1 * (vs1 + vs2);
    xy[pos] = xy[pos] + xmu1 * (vs1 + vs2) + vx1 * f_r;
    r4[pos] = f_vx2 * f_r + f_wwo * f_rtmp;
    f_rtmp = f_rtmp * (f_wwo - T(1)) + f_vx2 * f_r * (T(1) - f_vx1);
    xy[pos] = (xy[pos] + DT * f_rtmp) * f_dcrj;

    vs1 = c1 * (u1[pos + 1] - f_u1) + c2 * (u1[pos + 2] - u1[km1]);
    vs2 = c1 * (f_w1 - w1_im1) + c2 * (w1_ip1 - w1_im2);
    f_r = r5[pos];
    f_rtmp = h2 * (vs1 + vs2);
    xz[pos] = xz[pos] + xmu2 * (vs1 + vs2) + vx1 * f_r;
    r5[pos] = f_vx2 * f_r + f_wwo * f_rtmp;
    f_rtmp = f_rtmp * (f_wwo - T(1)) + f_vx2 * f_r * (T(1) - f_vx1);
    xz[pos] = (xz[pos] + DT * f_rtmp) * f_dcrj;

    vs1 = c1 * (v1[pos + 1] - f_v1) + c2 * (v1[pos + 2] - v1[km1]);
    vs2 = c1 * (w1[pos + Y] - f_w1) + c2 * (w1[pos + 2 * Y] - w1[jm1]);
    f_r = r6[pos];
    f_rtmp = h3 * (vs1 + vs2);
    yz[pos] = yz[pos] + xmu3 * (vs1 + vs2) + vx1 * f_r;
    r6[pos] = f_vx2 * f_r + f_wwo * f_rtmp;
    f_rtmp = f_rtmp * (f_wwo - T(1)) + f_vx2 * f_r * (T(1) - f_vx1);
    yz[pos] = (yz[pos] + DT * f_rtmp) * f_dcrj;
  }

  // dstrqc over xls..xre x yls..yre, k = align+3 .. nzt+align-1 (grid 0)
  void stress() {
    const int NX = nxt;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 2 + NGSL; i <= nxt + NGSL + 1; i++)
      for (int j = 2 + NGSL; j <= nyt + NGSL + 1; j++)
        for (int k = ALIGN + 3; k <= nzt + ALIGN - 1; k++) stress_cell(i, j, k, NX);
  }

  // fstr (kernel.cu:1616-1647), j rows rounded up to the 2-row blocks
  void fstr() {
    T* zz = f[ZZ].data(); T* xz = f[XZ].data(); T* yz = f[YZ].data();
    const int k = nzt + ALIGN - 1;
    const int j0 = 2 + NGSL, j1 = j0 + (nyt + 1) / 2 * 2 - 1;
    for (int i = 2 + NGSL; i <= nxt + NGSL + 1; i++)
      for (int j = j0; j <= j1; j++) {
        const long long pos = idx(i, j, k);
        zz[pos + 1] = -zz[pos];
        zz[pos + 2] = -zz[pos - 1];
        xz[pos + 1] = -xz[pos - 1];
        xz[pos + 2] = -xz[pos - 2];
        yz[pos + 1] = -yz[pos - 1];
        yz[pos + 2] = -yz[pos - 2];
        xz[pos] = T(0);
        yz[pos] = T(0);
      }
  }

  long long src_pos(int s) const {
    return idx(psrc[3 * s] + 1 + NGSL, psrc[3 * s + 1] + 1 + NGSL, psrc[3 * s + 2] + ALIGN - 1);
  }

  // addsrc_cu (kernel.cu:1780-1806), sources applied in file order
  void addsrc(int ti) {
    const T vtst = DT / (DH * DH * DH);
    T* o[6] = {f[XX].data(), f[YY].data(), f[ZZ].data(), f[XZ].data(), f[YZ].data(),
               f[XY].data()};
    for (int s = 0; s < nsrc; ++s) {
      const long long pos = src_pos(s);
      for (int q = 0; q < 6; ++q) o[q][pos] = o[q][pos] - vtst * src[q][(size_t)s * stride + ti];
    }
  }

  // compmt / brune / liu / lfilter / addkinsrc_cu (kernel.cu:3706-3858)
  static void compmt(T str, T dip, T rake, T* m) {
    const T sd = sin(dip), cd = cos(dip), sr = sin(rake), cr = cos(rake);
    m[1] = -(sd * cr * sin(T(2) * str) + sin(T(2) * dip) * sr * sin(str) * sin(str));   // yy
    m[5] = sd * cr * cos(T(2) * str) + T(0.5) * (sin(T(2) * dip) * sr * sin(T(2) * str));  // xy
    m[4] = (cd * cr * cos(str) + cos(T(2) * dip) * sr * sin(str));                      // yz
    m[0] = sd * cr * sin(T(2) * str) - sin(T(2) * dip) * sr * cos(str) * cos(str);       // xx
    m[3] = (cd * cr * sin(str) - cos(T(2) * dip) * sr * cos(str));                      // xz
    m[2] = sin(T(2) * dip) * sr;                                                        // zz
  }
  static T brune(T freq, T time) {
    const T omega = freq * T(M_PI) * T(2);
    return (time > T(0)) ? omega * omega * time * exp(-omega * time) : T(0);
  }
  static T liu(T tau, T time) {
    const T PI = T(M_PI);
    const T tau1 = T(0.13) * tau, tau2 = tau - tau1;
    const T CN = PI / (T(1.4) * PI * tau1 + T(1.2) * tau1 + T(0.3) * PI * tau2);
    if (time < tau1)
      return CN * (T(0.7) - T(0.7) * cos(PI * time / tau1) + T(0.6) * sin(T(0.5) * PI * time / tau1));
    if (time < T(2) * tau1)
      return CN * (T(1.0) - T(0.7) * cos(PI * time / tau1) + T(0.3) * cos(PI * (time - tau1) / tau2));
    if (time < tau) return CN * (T(0.3) + T(0.3) * cos(PI * (time - tau1) / tau2));
    return T(0);
  }
  double lfilter(double x, double* d) const {
    const double y = (fb[0] * x + d[0]) / fa[0];
    for (int n = 0; n < filtorder - 1; n++) d[n] = fb[n + 1] * x - fa[n + 1] * y + d[n + 1];
    d[filtorder - 1] = fb[filtorder] * x - fa[filtorder] * y;
    return y;
  }
  void addkinsrc(int step) {
    const T atime = step * DT;
    const T vtst = DT / (DH * DH * DH);
    T* o[6] = {f[XX].data(), f[YY].data(), f[ZZ].data(), f[XZ].data(), f[YZ].data(),
               f[XY].data()};
    for (int s = 0; s < nsrc; ++s) {
      const size_t b = (size_t)s * stride;
      const int stf_type = (int)src[0][b];
      const T slip = src[1][b], ruptime = src[2][b], risetime = src[3][b];
      if (!(atime > ruptime)) continue;
      const T area = src[4][b];
      const T strike = src[0][b + 1] / T(180) * T(M_PI);
      const T dip = src[1][b + 1] / T(180) * T(M_PI);
      const T rake = src[2][b + 1] / T(180) * T(M_PI);
      T m[6];
      compmt(strike, dip, rake, m);
      T stf;
      if (stf_type == 1)
        stf = brune(T(1) / risetime, atime - ruptime);
      else if (stf_type == 2)
        stf = liu(risetime, atime - ruptime);
      else
        stf = T(0);
      if (filtorder > 0) stf = (T)lfilter((double)stf, filt_state.data() + (size_t)s * (filtorder + 1));
      const long long pos = src_pos(s);
      stf *= slip * area / f[MU][pos];
      mom[s] += stf * DT;
      stf *= vtst;
      for (int q = 0; q < 6; ++q) o[q][pos] = o[q][pos] - stf * m[q];
    }
  }

  // rotate_principal (kernel.cu:43-64)
  void rotate_principal(T sigma2, T pfluid, T* ssp) const {
    T ss[9] = {}, tmp[9] = {};
    for (int k = 0; k < 9; k++) ssp[k] = 0;
    ss[0] = (sigma2 + pfluid) * fmajor;
    ss[4] = sigma2 + pfluid;
    ss[8] = (sigma2 + pfluid) * fminor;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) tmp[i * 3 + j] += RzT[i * 3 + k] * ss[k * 3 + j];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) ssp[i * 3 + j] += tmp[i * 3 + k] * Rz[k * 3 + j];
    ssp[0] -= pfluid;
    ssp[4] -= pfluid;
    ssp[8] -= pfluid;
  }
  T pfluid_at(int k) const {
    const T depth = (T)((nzt + ALIGN - 1) - k) * DH;
    return (depth > 0) ? (depth + DH * T(0.5)) * T(9.81e3) : DH / T(2) * T(9.81e3);
  }

  // drprecpc_calc_opt (kernel.cu:1253-1422) at one cell
  void plast_calc_cell(int i, int j, int k) {
    const long long S = slice, Y = yline;
    const long long pos = idx(i, j, k), ip1 = pos + S, jm1 = pos - Y, km1 = pos - 1;
    const T* xx = f[XX].data(); const T* yy = f[YY].data(); const T* zz = f[ZZ].data();
    const T* xy = f[XY].data(); const T* xz = f[XZ].data(); const T* yz = f[YZ].data();
    const T pfluid = pfluid_at(k);
    T ini[9], ini_ip1[9];
    rotate_principal(f[SIGMA2][pos], pfluid, ini);
    rotate_principal(f[SIGMA2][ip1], pfluid, ini_ip1);
    const T iixx = T(0.5) * (ini[0] + ini_ip1[0]);
    const T iiyy = T(0.5) * (ini[4] + ini_ip1[4]);
    const T iizz = T(0.5) * (ini[8] + ini_ip1[8]);
    T Sxx = xx[pos] + iixx, Syy = yy[pos] + iiyy, Szz = zz[pos] + iizz;
    T Sxz = T(0.25) * (xz[pos] + xz[ip1] + xz[km1] + xz[ip1 - 1]) + T(0.5) * (ini[2] + ini_ip1[2]);
    T Syz = T(0.25) * (yz[pos] + yz[jm1] + yz[km1] + yz[jm1 - 1]) + T(0.5) * (ini[5] + ini_ip1[5]);
    T Sxy = T(0.25) * (xy[pos] + xy[ip1] + xy[jm1] + xy[ip1 - Y]) + T(0.5) * (ini[1] + ini_ip1[1]);
    const T mu_i = f[MU][pos], mu_ip1 = f[MU][ip1];
    const T Tv = DH / sqrt(T(1) / (mu_i * f[D1][pos]));
    const T Sxxp = Sxx, Syyp = Syy, Szzp = Szz, Sxyp = Sxy, Sxzp = Sxz, Syzp = Syz;
    const T rphi = f[PHI][pos] * T(0.017453292519943295);
    const T sigma_m = (Sxx + Syy + Szz) / T(3);
    const T SDxx = Sxx - sigma_m, SDyy = Syy - sigma_m, SDzz = Szz - sigma_m;
    const T secinv =
        T(0.5) * (SDxx * SDxx + SDyy * SDyy + SDzz * SDzz) + Sxz * Sxz + Sxy * Sxy + Syz * Syz;
    const T sq = sqrt(secinv);
    const T taulim2 = f[COHES][pos] * cos(rphi) - (sigma_m + pfluid) * sin(rphi);
    const T taulim = taulim2 > T(0) ? taulim2 : T(0);
    T y;
    if (sq > taulim) {
      y = taulim / sq + (T(1) - taulim / sq) * exp(-DT / Tv);
      Sxx = SDxx * y + sigma_m;
      Syy = SDyy * y + sigma_m;
      Szz = SDzz * y + sigma_m;
      Sxz = Sxz * y;
      Sxy = Sxy * y;
      Syz = Syz * y;
    } else {
      y = T(1);
    }
    f[YLDFAC][pos] = y;
    if (y < T(1)) {
      const T xm = T(2) / (mu_i + mu_ip1);
      const T a = (Sxx - Sxxp) / xm, b = (Syy - Syyp) / xm, c = (Szz - Szzp) / xm,
              d = (Sxy - Sxyp) / xm, e = (Sxz - Sxzp) / xm, g = (Syz - Syzp) / xm;
      f[NETA][pos] = f[NETA][pos] + sqrt(T(0.5) * (a * a + b * b + c * c) + T(2) * (d * d + e * e + g * g));
    } else {
      f[YLDFAC][pos] = T(1);
    }
  }

  // drprecpc_app (kernel.cu:1650-1778) at one cell
  void plast_app_cell(int i, int j, int k) {
    const long long S = slice, Y = yline;
    const long long pos = idx(i, j, k), im1 = pos - S, ip1 = pos + S, jp1 = pos + Y, kp1 = pos + 1;
    T* xx = f[XX].data(); T* yy = f[YY].data(); T* zz = f[ZZ].data();
    T* xy = f[XY].data(); T* xz = f[XZ].data(); T* yz = f[YZ].data();
    const T* yl = f[YLDFAC].data();
    const T* s2 = f[SIGMA2].data();
    const T depth = (T)((nzt + ALIGN - 1) - k) * DH;
    const T depth_kp1 = (T)((nzt + ALIGN - 1) - k + 1) * DH;
    const T pfluid = depth > 0 ? (depth + DH / T(2)) * T(9.81e3) : DH / T(2) * T(9.81e3);
    const T pfluid_kp1 = depth_kp1 > 0 ? (depth_kp1 + DH / T(2)) * T(9.81e3) : DH / T(2) * T(9.81e3);
    T a[9], b[9], c[9], d[9], e[9], g[9], h[9], q[9];
    if (yl[pos] < T(1)) {
      rotate_principal(s2[pos], pfluid, a);
      rotate_principal(s2[ip1], pfluid_kp1, b);
      const T iixx = T(0.5) * (a[0] + b[0]), iiyy = T(0.5) * (a[4] + b[4]),
              iizz = T(0.5) * (a[8] + b[8]);
      const T Sxx = xx[pos] + iixx, Syy = yy[pos] + iiyy, Szz = zz[pos] + iizz;
      const T sigma_m = (Sxx + Syy + Szz) / T(3);
      const T SDxx = xx[pos] + iixx - sigma_m, SDyy = yy[pos] + iiyy - sigma_m,
              SDzz = zz[pos] + iizz - sigma_m;
      xx[pos] = SDxx * yl[pos] + sigma_m - iixx;
      yy[pos] = SDyy * yl[pos] + sigma_m - iiyy;
      zz[pos] = SDzz * yl[pos] + sigma_m - iizz;
    }
    T iy = T(0.25) * (yl[im1] + yl[pos] + yl[im1 + 1] + yl[kp1]);
    if (iy < T(1)) {
      rotate_principal(s2[pos], pfluid, a);
      rotate_principal(s2[kp1], pfluid_kp1, c);
      const T iist = T(0.5) * (a[2] + c[2]);
      xz[pos] = (xz[pos] + iist) * iy - iist;
    }
    iy = T(0.25) * (yl[pos] + yl[jp1] + yl[jp1 + 1] + yl[kp1]);
    if (iy < T(1)) {
      rotate_principal(s2[pos], pfluid, a);
      rotate_principal(s2[ip1], pfluid, b);
      rotate_principal(s2[kp1], pfluid_kp1, c);
      rotate_principal(s2[ip1 + 1], pfluid_kp1, d);
      rotate_principal(s2[jp1], pfluid, e);
      rotate_principal(s2[ip1 + Y], pfluid, g);
      rotate_principal(s2[jp1 + 1], pfluid_kp1, h);
      rotate_principal(s2[ip1 + Y + 1], pfluid_kp1, q);
      const T iist = T(0.125) * (a[5] + b[5] + c[5] + d[5] + e[5] + g[5] + h[5] + q[5]);
      yz[pos] = (yz[pos] + iist) * iy - iist;
    }
    iy = T(0.25) * (yl[pos] + yl[jp1] + yl[im1] + yl[im1 + Y]);
    if (iy < T(1)) {
      rotate_principal(s2[pos], pfluid, a);
      rotate_principal(s2[jp1], pfluid, e);
      const T iist = T(0.5) * (a[1] + e[1]);
      xy[pos] = (xy[pos] + iist) * iy - iist;
    }
  }

  // NVE=3 section of the time loop at one rank (pmcl3d.c:2110-2209):
  // five drprecpc_calc strip launches (overlapping rows visited twice), then
  // drprecpc_app over xlsp..xrep x ylsp..yrep (j rounded up to 2 rows).
  void plasticity() {
    const int xl = 2 + NGSL, xr = nxt + NGSL + 1, yl = 2 + NGSL, yr = nyt + NGSL + 1;
    const int kc1 = ALIGN + (nzt + 3) / 4 * 4 - 1;
    auto calc = [&](int i0, int i1, int j0, int j1) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
      for (int i = i0; i <= i1; i++)
        for (int j = j0; j <= j1; j++)
          for (int k = ALIGN; k <= kc1; k++) plast_calc_cell(i, j, k);
    };
    calc(xl, xr, yl, yl + NGSL);
    calc(xl, xr, yr - NGSL, yr);
    calc(xl, xl + NGSL, yl, yr);
    calc(xr - NGSL, xr, yl, yr);
    calc(xl + NGSL, xr - NGSL, yl + NGSL, yr - NGSL);
    const int ja1 = yl + (yr - yl + 2) / 2 * 2 - 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = xl; i <= xr; i++)
      for (int j = yl; j <= ja1; j++)
        for (int k = ALIGN; k <= kc1; k++) plast_app_cell(i, j, k);
  }

  void add_point_sources(int field, int nq, int nb, const int* ix, const int* iy, const int* iz,
                         const float* lx, const float* ly, const float* lz, int nsamples,
                         const float* values, int stride) override {
    PointSrc p;
    p.field = field; p.nq = nq; p.nb = nb; p.nsamples = nsamples; p.stride = stride;
    p.ix.assign(ix, ix + nq); p.iy.assign(iy, iy + nq); p.iz.assign(iz, iz + nq);
    p.lx.assign(lx, lx + (size_t)nq * nb); p.ly.assign(ly, ly + (size_t)nq * nb);
    p.lz.assign(lz, lz + (size_t)nq * nb);
    p.values.assign(values, values + (size_t)nsamples * nq);
    psrcs.push_back(p);
  }

  // cusource_add_cartesian (topography/sources/source.cu:24-49): every
  // `stride` steps, sigma(cell) -= dt/h^3 * lx*ly*lz * M(step/stride), in
  // query order; cells of the metric grid sit at (2 + ix, 2 + iy, align + iz).
  void point_sources() {
    const T dthh = DT / (DH * DH * DH);
    for (const PointSrc& p : psrcs) {
      if (cur % p.stride != 0) continue;
      const long long smp = cur / p.stride;
      if (smp >= p.nsamples) continue;
      T* F = f[p.field].data();
      for (int q = 0; q < p.nq; ++q) {
        const T v = (T)p.values[(size_t)smp * p.nq + q];
        for (int i = 0; i < p.nb; ++i)
          for (int j = 0; j < p.nb; ++j)
            for (int k = 0; k < p.nb; ++k) {
              const long long pos =
                  idx(2 + p.ix[q] + i, 2 + p.iy[q] + j, ALIGN + p.iz[q] + k);
              F[pos] -= dthh * (T)p.lx[(size_t)q * p.nb + i] * (T)p.ly[(size_t)q * p.nb + j] *
                        (T)p.lz[(size_t)q * p.nb + k] * v;
            }
      }
    }
  }

  void set_plane_wave(int n, int nd, const float* vx, const float* vy,
                      const float* vz) override {
    const float* in[3] = {vx, vy, vz};
    for (int q = 0; q < 3; ++q) plane[q].assign(in[q], in[q] + n);
    plane_n = n;
    plane_nd = nd;
  }

  // addplanesrc_cu (kernel.cu:3897-3925): sample ti of the plane wave on level
  // align + ND + 1, every (i, j) of the reference's launch (rows 4 .. 3 + nx
  // rounded up to its 2 x 2 blocks); the kernel arrays hold 1/mu and 1/lambda
  void addplanesrc(int ti) {
    const int nx = nxt + 4 + (nxt % 2), ny = nyt + 4 + (nyt % 2);
    const T vtst = DT / DH;
    const int k = ALIGN + plane_nd + 1;
    for (int i = 4; i < 4 + nx; ++i)
      for (int j = 4; j < 4 + ny; ++j) {
        const long long pos = idx(i, j, k);
        const T mu = f[MU][pos], la = f[LAM][pos];
        f[XZ][pos] = f[XZ][pos] - vtst * T(2) / mu * plane[0][ti];
        f[YZ][pos] = f[YZ][pos] - vtst * T(2) / mu * plane[1][ti];
        f[XX][pos] = f[XX][pos] - vtst * T(2) / la * plane[2][ti];
        f[YY][pos] = f[YY][pos] - vtst * T(2) / la * plane[2][ti];
        f[ZZ][pos] = f[ZZ][pos] - vtst * T(2) / (la + T(2) * mu) * plane[2][ti];
      }
  }

  void step(int nve, int n) override {
    for (int s = 0; s < n; ++s) {
      if (cur == 0 && !initial_done) {
        if (ifault == 1 && nsrc > 0) addsrc(0);  // pmcl3d.c:1175-1187
        initial_done = true;
      }
      cur += 1;
      velocity();
      stress();
      point_sources();  // sources_add_cartesian (pmcl3d.c:1987-2004)
      if (ifault == 1 && cur < nst) addsrc((int)cur);
      if (ifault == 5) addkinsrc((int)cur);
      if (ifault == 6 && cur < plane_n) addplanesrc((int)cur);
      if (nve == 3) plasticity();
      fstr();
    }
  }

  void gather(int nbgx, int nedx, int nskpx, int nbgy, int nedy, int nskpy, int nbgz, int nedz,
              int nskpz, float* bx, float* by, float* bz) override {
    const int rnx = (nedx - nbgx) / nskpx + 1, rny = (nedy - nbgy) / nskpy + 1;
    for (int k = nbgz; k <= nedz; k += nskpz)
      for (int j = 2 + NGSL + nbgy; j <= 2 + NGSL + nedy; j += nskpy)
        for (int i = 2 + NGSL + nbgx; i <= 2 + NGSL + nedx; i += nskpx) {
          const int ko = nzt + ALIGN - 1 - k;
          const long long t = (long long)(k - nbgz) / nskpz * rnx * rny +
                              (long long)(j - 2 - NGSL - nbgy) / nskpy * rnx +
                              (i - 2 - NGSL - nbgx) / nskpx;
          bx[t] = (float)f[U1][idx(i, j, ko)];
          by[t] = (float)f[V1][idx(i, j, ko)];
          bz[t] = (float)f[W1][idx(i, j, ko - 1)];
        }
  }
};

}  // namespace

struct oracle {
  Base* impl;
  int nthreads = 1;
  int flush = 0;  // FTZ/DAZ on the stepping threads (CPU baseline mode)
};

namespace {
// Flush-to-zero and denormals-are-zero (MXCSR bits 15 and 6) on every thread of
// the team the stepping loops use, and on the calling thread: the reference's
// CUDA build compiles with -use_fast_math, which flushes FP32 subnormals, so the
// CPU baseline times the same arithmetic without the x86 subnormal slow path.
void set_ftz_daz(int nthreads, bool on) {
#pragma omp parallel num_threads(nthreads)
  {
    const unsigned m = _mm_getcsr();
    _mm_setcsr(on ? (m | 0x8040u) : (m & ~0x8040u));
  }
  const unsigned m = _mm_getcsr();
  _mm_setcsr(on ? (m | 0x8040u) : (m & ~0x8040u));
}
}  // namespace

extern "C" {

oracle* oracle_create(int precision, int nxt, int nyt, int nzt, float dh, float dt, int npc,
                      int nthreads) {
  oracle* o = new oracle;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  o->nthreads = nthreads;
  if (precision == 32)
    o->impl = new Oracle<float>(nxt, nyt, nzt, dh, dt, npc, nthreads);
  else if (precision == 65)
    o->impl = new Oracle<Dual>(nxt, nyt, nzt, dh, dt, npc, nthreads);
  else
    o->impl = new Oracle<double>(nxt, nyt, nzt, dh, dt, npc, nthreads);
  return o;
}
void oracle_destroy(oracle* o) {
  if (!o) return;
  delete o->impl;
  delete o;
}
void oracle_set_field(oracle* o, int field, const float* src) { o->impl->set_field(field, src); }
void oracle_get_field(oracle* o, int field, float* dst) { o->impl->get_field(field, dst); }
void oracle_get_field_f64(oracle* o, int field, double* dst) { o->impl->get_field64(field, dst); }
void oracle_set_ww(oracle* o, const int* ww) { o->impl->set_ww(ww); }
void oracle_set_sponge(oracle* o, const float* x, const float* y, const float* z) {
  o->impl->set_sponge(x, y, z);
}
void oracle_set_coeff(oracle* o, const float* c) { o->impl->set_coeff(c); }
void oracle_compute_lam_mu(oracle* o) { o->impl->compute_lam_mu(); }
void oracle_set_sources(oracle* o, int ifault, int nsrc, const int* psrc, int stride, int nst,
                        const float* axx, const float* ayy, const float* azz, const float* axz,
                        const float* ayz, const float* axy) {
  const float* a[6] = {axx, ayy, azz, axz, ayz, axy};
  o->impl->set_sources(ifault, nsrc, psrc, stride, nst, a);
}
void oracle_set_filter(oracle* o, int order, const double* b, const double* a) {
  o->impl->set_filter(order, b, a);
}
void oracle_get_moment(oracle* o, float* m) { o->impl->get_moment(m); }
void oracle_set_plane_wave(oracle* o, int n, int nd, const float* vx, const float* vy,
                           const float* vz) {
  o->impl->set_plane_wave(n, nd, vx, vy, vz);
}
void oracle_set_plasticity(oracle* o, float fmajor, float fminor, const float* Rz,
                           const float* RzT) {
  o->impl->set_plasticity(fmajor, fminor, Rz, RzT);
}
void oracle_add_point_sources(oracle* o, int field, int nq, int nb, const int* ix,
                              const int* iy, const int* iz, const float* lx, const float* ly,
                              const float* lz, int nsamples, const float* values, int stride) {
  o->impl->add_point_sources(field, nq, nb, ix, iy, iz, lx, ly, lz, nsamples, values, stride);
}
void oracle_step(oracle* o, int nve, int n) {
  if (o->flush) set_ftz_daz(o->nthreads, true);
  o->impl->step(nve, n);
  if (o->flush) set_ftz_daz(o->nthreads, false);
}
void oracle_set_flush_denormals(oracle* o, int on) { o->flush = on ? 1 : 0; }
void oracle_set_tangent(oracle* o, int field, const double* t) {
  o->impl->set_tangent_field(field, t);
}
void oracle_get_tangent(oracle* o, int field, double* t) { o->impl->get_tangent_field(field, t); }
long long oracle_current_step(oracle* o) { return o->impl->current(); }
void oracle_gather(oracle* o, int nbgx, int nedx, int nskpx, int nbgy, int nedy, int nskpy,
                   int nbgz, int nedz, int nskpz, float* bx, float* by, float* bz) {
  o->impl->gather(nbgx, nedx, nskpx, nbgy, nedy, nskpy, nbgz, nedz, nskpz, bx, by, bz);
}

}  // extern "C"
