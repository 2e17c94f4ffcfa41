/*
 * CPU oracle for the AWP-ODC time step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference kernels (src/awp/kernel.cu) in
 * the reference's own update order (src/awp/pmcl3d.c:1628-2487), templated on
 * the arithmetic type: precision 64 is the FP64 oracle every parity test
 * compares against, precision 32 (OpenMP) is the timed CPU baseline.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this library, and only as a checker / reference timing; the product never
 * links it.
 *
 * All 3-D inputs and outputs are float arrays in the reference's padded
 * layout ((nxt+20) x (nyt+20) x (nzt+64), k fastest).
 */
#ifndef AWP_ORACLE_H
#define AWP_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle oracle;

/* precision: 32, 64, or 65 = FP64 dual numbers (value + tangent: the exact
 * derivative of the discrete scheme along one direction, tangent-linear
 * mode).  nx, ny: global sizes for the free-surface edge test
 * (kernel.cu:1092-1097); npc: 0 sponge, 2 periodic. */
oracle* oracle_create(int precision, int nxt, int nyt, int nzt, float dh, float dt,
                      int npc, int nthreads);
void oracle_destroy(oracle* o);

/* field ids: 0..2 u1 v1 w1, 3..8 xx yy zz xy xz yz, 9..14 r1..r6,
 * 15 d1, 16 mu, 17 lam, 18 qp, 19 qs, 20 sigma2, 21 cohes, 22 phi,
 * 23 yldfac, 24 neta, 25 vx1, 26 vx2, 27 wwo, 28 ww (int stored as float) */
void oracle_set_field(oracle* o, int field, const float* src);
void oracle_get_field(oracle* o, int field, float* dst);
void oracle_get_field_f64(oracle* o, int field, double* dst);
void oracle_set_ww(oracle* o, const int* ww);
void oracle_set_sponge(oracle* o, const float* dcrjx, const float* dcrjy, const float* dcrjz);
void oracle_set_coeff(oracle* o, const float* coeff16);
/* lam_mu of pmcl3d.c:944-951 computed from the current lam/mu arrays. */
void oracle_compute_lam_mu(oracle* o);

/* Point (ifault 1) or kinematic (ifault 5) sources, already mapped to padded
 * cells (x, y, z as addsrc expects: psrc + 1 + ngsl, psrc + align - 1);
 * a*: [nsrc][stride] per component. */
void oracle_set_sources(oracle* o, int ifault, int nsrc, const int* psrc, int stride,
                        int nst, const float* axx, const float* ayy, const float* azz,
                        const float* axz, const float* ayz, const float* axy);
void oracle_set_filter(oracle* o, int order, const double* b, const double* a);
void oracle_get_moment(oracle* o, float* mom);

/* Plasticity (NVE=3): principal-stress frame; sigma2/cohes/phi via set_field. */
void oracle_set_plane_wave(oracle* o, int n, int nd, const float* vx, const float* vy,
                           const float* vz);
void oracle_set_plasticity(oracle* o, float fmajor, float fminor, const float* Rz,
                           const float* RzT);

/* nve: 1 or 3.  Advances n steps in pmcl3d order. */
/* SOURCEFILE moment-tensor component on stress field `field` (oracle field
 * index): queries with first indices ix/iy/iz on the metric grid and Lagrange
 * weights l*[nq][nb]; values[nsamples][nq] applied every `stride` steps. */
void oracle_add_point_sources(oracle* o, int field, int nq, int nb, const int* ix,
                              const int* iy, const int* iz, const float* lx, const float* ly,
                              const float* lz, int nsamples, const float* values, int stride);
void oracle_step(oracle* o, int nve, int n);
/* FP32 subnormals flushed to zero while stepping (as the reference's
 * -use_fast_math CUDA build does); for the CPU baseline, off by default. */
void oracle_set_flush_denormals(oracle* o, int on);
/* Tangent part of a field (precision 65; a no-op / zeros otherwise). */
void oracle_set_tangent(oracle* o, int field, const double* t);
void oracle_get_tangent(oracle* o, int field, double* t);
long long oracle_current_step(oracle* o);

/* velbuffer gather (kernel.cu:3948-4011) for grid 0 without FOLLOWBATHY. */
void oracle_gather(oracle* o, int nbgx, int nedx, int nskpx, int nbgy, int nedy,
                   int nskpy, int nbgz, int nedz, int nskpz, float* bx, float* by,
                   float* bz);

#ifdef __cplusplus
}
#endif
#endif
