/*
 * awp_b200.h -- C ABI of the B200 time-step library (libawpb200.so).
 *
 * Two groups of entry points:
 *
 *  1. A re-entrant context API.  All state of one simulation lives in an
 *     opaque awp_ctx; every call returns an int status (AWP_OK = 0).  It
 *     replaces the host orchestration of pmcl3d's time loop
 *     (src/awp/pmcl3d.c:1624-2490) together with the per-run set-up that
 *     loop depends on (pmcl3d.c:370-1372).
 *
 *  2. Drop-in launchers with the reference's names and signatures
 *     (include/awp/kernel_launch.h:10-190).  A pmcl3d-style caller links
 *     against them unchanged: raw device float* per field in the reference's
 *     padded layout, integer bounds in padded coordinates, a grid index d_i
 *     into state installed by SetDeviceConstValue, void returns.  Like the
 *     reference (CUCHK, include/awp/pmcl3d_cons.h:43-54) a CUDA error inside
 *     one of them prints the error and exits the process; awp_compat_exit_on_error(0)
 *     switches that to "record and return", readable via awp_compat_last_error().
 *
 * Field layout (both groups): index(i,j,k) = i*slice + j*yline + k with
 * yline = nzt+64, slice = (nyt+20)*yline, extents (nxt+20) x (nyt+20) x (nzt+64);
 * interior i,j in [10, 10+n), k in [32, 32+nzt); the free surface is the top,
 * k = nzt+31.
 */
#ifndef AWP_B200_H
#define AWP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
#define AWP_OK 0
#define AWP_ERR_ARG 1
#define AWP_ERR_CUDA 2
#define AWP_ERR_STATE 3
#define AWP_ERR_IO 4
#define AWP_ERR_NOMEM 5
#define AWP_ERR_NUMERIC 6
#define AWP_ERR_UNSUPPORTED 7

/* Field identifiers for awp_field_* (padded 3-D fields). */
enum awp_field_id {
  AWP_U1 = 0, AWP_V1, AWP_W1,                      /* velocities          */
  AWP_XX, AWP_YY, AWP_ZZ, AWP_XY, AWP_XZ, AWP_YZ,  /* stresses            */
  AWP_R1, AWP_R2, AWP_R3, AWP_R4, AWP_R5, AWP_R6,  /* memory variables    */
  AWP_D1, AWP_MU, AWP_LAM, AWP_QP, AWP_QS,         /* media (rho, 1/mu,   */
                                                   /*  1/lambda, Q^-1)    */
  AWP_SIGMA2, AWP_COHES, AWP_PHI, AWP_YLDFAC, AWP_NETA, /* plasticity     */
  AWP_NFIELDS
};

typedef struct awp_ctx awp_ctx;

/* Run parameters.  Names and meaning follow pmcl3d's command line
 * (src/awp/command.c:71-136, 228-504).  Single rank, single grid. */
typedef struct awp_params {
  int nx, ny, nz;    /* -X -Y -Z   interior cells (nz % 4 == 0, as pmcl3d.c:380) */
  float dh, dt;      /* -H -t      grid spacing (m), time step (s)                */
  float arbc;        /* -A         Cerjan sponge coefficient                      */
  int npc;           /* -M         0 = Cerjan sponge, 2 = periodic                */
  int nd;            /* -D         sponge width (cells)                           */
  int nve;           /* -V         1 = anelastic, 3 = anelastic + plasticity      */
  float fac, q0, ex, fp; /* -l -h --EX -p   Q(f) parameters                       */
  int socalq;        /* -s         SoCal vp/vs floor (1 = on)                     */
  int ifault;        /* -I         1 = point moment-rate source, 2 = the same from
                                   split files, 4 = prescribed velocities,
                                   5 = kinematic, 6 = plane wave                  */
  int nst;           /* -N         source time samples                            */
  int read_step;     /* -R/-Q      samples held per source (IFAULT 1, 2: >= nst)   */
  int grid;          /*            block of a discontinuous mesh, 0 = top (finest)  */
  int ngrids;        /* -G         blocks of the mesh (1 = a single grid)          */
} awp_params;

/* Fill *p with pmcl3d's defaults (command.c:71-136). */
void awp_params_default(awp_params* p);

/* Human-readable message for a status code, and the last error's detail. */
const char* awp_status_string(int status);
const char* awp_last_error(void);

/* ------------------------------------------------------------------------ */
/* Context API                                                               */
/* ------------------------------------------------------------------------ */

/* Allocate a simulation on the current CUDA device.  Fields start at zero,
 * the sponge (inicrj, cerjan.c:5) and the Q(f) tables (weights_sub/tausub,
 * mesh.c:684-1097) are set up here. */
int awp_ctx_create(const awp_params* p, awp_ctx** out);
int awp_ctx_destroy(awp_ctx* ctx);

/* Run every subsequent kernel on this cudaStream_t (NULL = the legacy default
 * stream).  A new context runs on a stream of its own. */
int awp_set_stream(awp_ctx* ctx, void* cuda_stream);

/* Padded extents (nxt+20, nyt+20, nzt+64). */
int awp_padded_dims(const awp_ctx* ctx, long long dims[3]);

/* Media from a host buffer in the mesh-file layout float[nz][ny][nx][nvar],
 * surface first, nvar in {3, 5, 8} (mesh.c:122-222).  Applies inimesh's
 * unrelaxed-modulus correction and inverse-modulus mapping (mesh.c:222-466)
 * on the device, fills the one-cell ghost border (mesh.c:468-591) and the
 * surface Lame ratio (pmcl3d.c:944-951). */
int awp_upload_media(awp_ctx* ctx, int nvar, const float* host_media);
/* Same, with the media buffer already in device memory. */
int awp_upload_media_device(awp_ctx* ctx, int nvar, const float* dev_media);
/* Extrema of the corrected vs (vs > 1 m/s only), vp and rho of the last media
 * upload, as inimesh reports them for the CHK file (mesh.c:455-460, io.c:23-31). */
int awp_media_extrema(awp_ctx* ctx, float vse[2], float vpe[2], float dde[2]);

/* Page-locked host buffers (for awp_gather_output targets). */
int awp_alloc_host_pinned(void** ptr, size_t bytes);
int awp_free_host_pinned(void* ptr);

/* Point / kinematic sources in the INSRC layout (source.c:165-181):
 * pos[nsrc][3] = (x, y, z) 1-based with z counted down from the surface;
 * data[nsrc][read_step][6] = (xx, yy, zz, xz, yz, xy) per time sample.  For
 * IFAULT=5 only samples 0 and 1 are used and hold the subfault parameters
 * (kernel.cu:3788-3809).  IFAULT=2 adds as IFAULT=1 (addsrc, pmcl3d.c:2008-2016);
 * its split files (read_src_ifault_2, source.c:15-128) are assembled by the
 * caller into all NST samples. */
int awp_upload_sources(awp_ctx* ctx, int nsrc, const int* pos, const float* data);
/* Plane-wave input (IFAULT=6; ini_plane_wave, source.c:797-833, and
 * addplanesrc_H, pmcl3d.c:2035-2041): three series of NST samples (vx, vy, vz,
 * the three columns of the INSRC text file), host or device pointers.  Every
 * step with cur_step < NST subtracts 2 dt/h times sample cur_step, scaled by
 * mu (xz, yz from vx, vy) and by lambda / lambda + 2 mu (xx, yy, zz from vz),
 * from the stresses of level align + ND + 1 of the grid -- the bottom grid of
 * a mesh.  Sample 0 is never applied (the loop counter starts at 1). */
int awp_upload_plane_wave(awp_ctx* ctx, int nst, const float* vx, const float* vy,
                          const float* vz);
/* Optional IIR/FIR filter of the kinematic source time function
 * (sourcefilter.dat, pmcl3d.c:651-673): b[order+1], a[order+1]. */
int awp_set_source_filter(awp_ctx* ctx, int order, const double* b, const double* a);
/* Accumulated moment per subfault (IFAULT=5), host buffer of nsrc floats. */
int awp_download_moment(awp_ctx* ctx, float* host_mom);

/* Plasticity inputs (NVE=3): padded sigma2/cohes/phi arrays (host) and the
 * principal-stress frame of nonlinear.dat (mesh.c:1178-1401). */
int awp_upload_plasticity(awp_ctx* ctx, const float* sigma2, const float* cohes,
                          const float* phi, float fmajor, float fminor,
                          const float strike[3], const float dip[3]);

/* Receivers of an ASCII v2 RECVFILE (replaces receivers_init,
 * src/topography/receivers/receivers.c:22-42, and the receivers_write calls of
 * pmcl3d.c:1603-1605 and 2246-2247).  The velocities are interpolated with
 * Lagrange weights of the file's degree every `stride` steps, staged through
 * a device ring of gpu_buffer_size samples and a host ring of cpu_buffer_size
 * device rings, and written as "<file>_<x|y|z>_<step>" (float32, receiver-major,
 * num_writes rings per file, receiver.c:47-113).  nt = number of time steps of
 * the run (pmcl3d's TMAX/DT + 1), used only for the zero padding of the file
 * step.  The current state is recorded at once (step 0 before the first
 * awp_step).  Set-up errors of the reference (unreadable or malformed file,
 * AWP error codes 101..901 of include/awp/error.h) return AWP_ERR_IO with the
 * code in awp_last_error(). */
int awp_receivers_init(awp_ctx* ctx, const char* recvfile, long long nt);
/* Receivers inside the domain per component (x, y, z). */
int awp_receivers_count(awp_ctx* ctx, int counts[3]);

/* Strain Green tensor output of an ASCII v2 SGTFILE (replaces sgt_init /
 * sgt_write_material_properties / sgt_write, src/topography/receivers/sgt.c,
 * and their calls at pmcl3d.c:1572-1578, 1605, 2248-2249): receivers of the six
 * stresses on their staggered grids, written like awp_receivers_init's as
 * "<file>_<Gxx|Gyy|Gzz|Gxy|Gxz|Gyz>_<step>", and once, at this call, the
 * material on the node grid as "<file>_d1", "<file>_lami" and "<file>_mui"
 * (1/lambda and 1/mu; "_d1" holds 1/lambda too, as the reference writes it).
 * Needs the media; the current stresses are recorded at once, after the
 * step-1 source sample of IFAULT < 4 that the reference adds before its loop
 * (pmcl3d.c:1175-1187), so upload the sources first. */
int awp_sgt_init(awp_ctx* ctx, const char* sgtfile, long long nt);

/* IFAULT=4 prescribed velocities (frcvel_cu, kernel.cu:1836-1934; read_src_ifault_4,
 * source.c:469-680; pmcl3d.c:714-722, 792-805, 1821-1826, 2442-2486): on grid
 * 0, after the velocity update, the velocities at `npsrc` points
 * (pos[npsrc][3] as read_src_ifault_4 forms them: the cell is (x + 1 + ngsl,
 * y + 1 + ngsl, z + align - 1)) take the frames of a previous run,
 * interpolated linearly over `tskp` steps per frame; after the last of
 * `nframes` frames the restoring force of the last prescribed step is added
 * every step.  Frames arrive in windows of `window` frames: `read` fills
 * vx, vy, vz [nframes_asked][npsrc] with frames first..first+n-1 (0 = ok),
 * at set-up and whenever the step loop reaches the end of a window, as
 * pmcl3d's reader rank delivers them.  nframes must be a multiple of
 * `window`.  Before the first step. */
typedef int (*awp_frame_reader)(void* user, int first, int n, float* vx, float* vy, float* vz);
int awp_velocity_forcing_init(awp_ctx* ctx, int npsrc, const int* pos, int nframes, int tskp,
                              int window, awp_frame_reader read, void* user);

/* Moment-tensor sources of an ASCII v2 SOURCEFILE (replaces sources_init /
 * sources_read / sources_add_cartesian, src/topography/sources/sources.c:27-78,
 * and their calls at pmcl3d.c:1563-1565, 1607, 1987-2004).  Rates are read
 * from "<file>_<xx|yy|zz|xy|xz|yz>" (float32, source-major, `steps` samples
 * each) in blocks of gpu_buffer_size*cpu_buffer_size samples and added every
 * `stride` steps with Lagrange weights: sigma -= dt/h^3 * w * M(t). */
int awp_sourcefile_init(awp_ctx* ctx, const char* sourcefile);

/* Boundary forces of an ASCII v2 FORCEFILE on the curvilinear top block
 * (replaces forces_init / forces_read / forces_add,
 * src/topography/sources/forces.c:24-96, cusource_add_force_H,
 * src/topography/sources/source.cu:101-157, and their calls at
 * pmcl3d.c:1569-1571, 1608, 1989-1994).  Every point must be a boundary point
 * (type 1).  Rates "<file>_<fx|fy|fz>" as for SOURCEFILE, added to u1, v1, w1
 * after the stress update: v += dt/h^3 * w * F(t) * q / (f dg rho), with the
 * SBP boundary weight q, the staggered metric f dg of the component and rho
 * read ngsl cells further in x and y than the cell, as the reference indexes
 * it.  Needs the topography first; refused where that density index would
 * leave the grid. */
int awp_forcefile_init(awp_ctx* ctx, const char* forcefile);

/* Host-only helpers (no context, no GPU) that expose the point-set set-up for
 * checks: the ASCII v2 reader (readers/input.c:35-42; hdr = length,
 * gpu_buffer_size, cpu_buffer_size, steps, num_writes, stride, degree, major
 * version) and the Lagrange interpolation of one staggered component
 * (grid_type 0..9 = x, y, z, xx, yy, zz, xy, xz, yz, material node) on one grid block
 * (source.c:137-400).  They return 0 or the reference's error code. */
int awp_input_read(const char* path, long long hdr[8], char* file, int filecap, float* x,
                   float* y, float* z, int* type, long long cap);
int awp_point_coefs(const char* path, int grid_type, int nxt, int nyt, int nzt, float h,
                    long long cap, int* count, int* indices, int* ix, int* iy, int* iz,
                    float* lx, float* ly, float* lz);
/* The same on the curvilinear top block of the topography file `intopo`
 * (vertical coordinate mapped through the surface function, source.c:283-340). */
int awp_point_coefs_topo(const char* path, const char* intopo, int grid_type, int nxt, int nyt,
                         int nzt, float h, long long cap, int* count, int* indices, int* ix,
                         int* iy, int* iz, float* lx, float* ly, float* lz);

/* ------------------------------------------------------------------------ */
/* Discontinuous mesh (DM): a vertical stack of grids, grid 0 on top, each   */
/* block 3x coarser in x and y than the one above (pmcl3d.c:370-378).        */
/* ------------------------------------------------------------------------ */
typedef struct awp_mesh awp_mesh;
/* grids[p] describes block p (params.grid = p, params.ngrids = ngrids; NX, NY,
 * DH, ND already scaled per block as pmcl3d does: NX*3^(ngrids-1-p), ...).
 * Every block shares one stream. */
int awp_mesh_create(const awp_params* grids, int ngrids, awp_mesh** out);
int awp_mesh_destroy(awp_mesh* mesh);
/* The context of block p, for its uploads (media, sources, plasticity) and
 * field access.  awp_step on it is refused; step the mesh instead. */
int awp_mesh_grid(awp_mesh* mesh, int p, awp_ctx** ctx);
/* Advance the whole mesh (pmcl3d.c:1628-2490 with ngrids > 1): velocity of
 * every block; the 2nd-order interface update dvelc2 (kernel.cu:2289-2343);
 * coarse-to-fine interpolation intp3d (kernel.cu:2359-2561) and fine-to-coarse
 * window average swap3 (kernel.cu:3032-3217); stress of every block; dstrqc2
 * (kernel.cu:2564-2767); sources; intp3d and swap3 again; plasticity; the
 * free-surface images of block 0.  The first call applies checkmesh
 * (mesh.c:1404-1443) to the media of every coarser block. */
int awp_mesh_step(awp_mesh* mesh, int nsteps);
/* Run every block of the mesh on this cudaStream_t (NULL = the legacy default
 * stream) from now on; the mesh's own stream stays until awp_mesh_destroy. */
int awp_mesh_set_stream(awp_mesh* mesh, void* cuda_stream);
int awp_mesh_synchronize(awp_mesh* mesh);

/* x-slab domain decomposition (the multi-rank path of pmcl3d.c:1657-1721,
 * 1838-1924 and swap.c, rebuilt for contiguous slabs: the padded layout's
 * slowest axis is x, so every halo is a run of whole x planes).  A part is a
 * context of width nx (its awp_params.nx) at global offset x0 (even, so that
 * the attenuation parity pattern is the global one) in a grid of nx_global;
 * awp_set_subdomain is called after awp_ctx_create and before the media,
 * which are uploaded per part ([nz][ny][nx] of the part).  The sponge is the
 * whole grid's; sources are given to their owning part in its own
 * coordinates; the plasticity inputs are the part's planes of the whole
 * padded arrays (x0 .. x0 + nx + 4 + 2*ngsl - 1), uploaded after
 * awp_set_subdomain.  Single-grid Cartesian runs without point-set files,
 * prescribed velocities or plane waves.  At the start of a step the
 * stresses and velocities (the stress update writes the free-surface
 * velocity images; before the first step the source sample of the loop's
 * start is added), after the velocity update the velocities, and once before
 * the first step the media must reach the neighbours' ghost planes, and with
 * NVE 3 the stresses before the yield factors and the yield factors before
 * the return (the two plasticity kernels average over x); a 4th-order
 * stencil reads two planes across, AWP_HALO_PLANES = 4 are sent. */
#define AWP_HALO_VELOCITY 1 /* u1 v1 w1 */
#define AWP_HALO_STRESS 2   /* xx yy zz xy xz yz */
#define AWP_HALO_MEDIA 4    /* d1 mu lam qp qs */
#define AWP_HALO_YLDFAC 8   /* yldfac (NVE 3: between the two plasticity kernels) */
#define AWP_HALO_PLANES 4
#define AWP_MAXPARTS 16
int awp_set_subdomain(awp_ctx* ctx, int nx_global, int x0);
/* Copy the halo of `set` (fields in enum order, `planes` x planes each, x
 * fastest within a plane as the padded layout) between the context and `buf`
 * (device or page-locked host memory, nfields * planes * (ny+4+2*ngsl) *
 * (nz+2*align) floats) on the context's stream: unpack = 0 reads the planes
 * inside `side` (0 = low x, 1 = high x) into buf, unpack = 1 writes buf into
 * the ghost planes beyond it. */
int awp_halo_copy(awp_ctx* ctx, int unpack, int side, int set, int planes, float* buf);
/* One process per GPU: awp_step calls `fn(user, set)` at the two exchange
 * points of every step; it exchanges with the neighbours (awp_halo_copy and
 * the caller's transport, e.g. NCCL) and returns 0.  NULL removes it. */
typedef int (*awp_exchange_fn)(void* user, int set);
int awp_set_exchange(awp_ctx* ctx, awp_exchange_fn fn, void* user);
/* Several parts on one device stepped in lockstep, the halos copied in device
 * memory on one stream the decomposition owns (destroy it before the parts). */
typedef struct awp_decomp awp_decomp;
int awp_decomp_create(awp_ctx** parts, int nparts, awp_decomp** out);
int awp_decomp_step(awp_decomp* d, int nsteps);
int awp_decomp_synchronize(awp_decomp* d);
/* Run the parts and the halo copies on this cudaStream_t from now on. */
int awp_decomp_set_stream(awp_decomp* d, void* cuda_stream);
int awp_decomp_destroy(awp_decomp* d);

/* ------------------------------------------------------------------------ */
/* Batched instances: many independent single-grid simulations of uneven     */
/* sizes (source ensembles, shots) advanced together.                        */
/* ------------------------------------------------------------------------ */
typedef struct awp_batch awp_batch;
/* The instances are ordinary contexts, set up as for awp_step (media,
 * sources); single grid, Cartesian, NVE 1/2, no receivers or SOURCEFILE
 * (AWP_ERR_UNSUPPORTED otherwise), all at the same step.  The batch keeps
 * pointers to them; destroy the batch before its contexts. */
int awp_batch_create(awp_ctx* const* ctxs, int n, awp_batch** out);
int awp_batch_destroy(awp_batch* batch);
/* Advance every instance nsteps, each step one persistent launch per
 * half-step over a tile queue of all instances (CTAs pull 32 k x ty j x ichunk
 * i tiles from a global counter), then the sources and free-surface images of
 * all instances; the step is one CUDA graph replayed nsteps times.  Each
 * instance's arithmetic is that of awp_step, bit for bit.  Ordered after
 * earlier work on the contexts' streams and before later work on them. */
int awp_batch_step(awp_batch* batch, int nsteps);
int awp_batch_synchronize(awp_batch* batch);
/* Tile shape (ty = 4 or 8 j rows, ichunk x planes per tile; default 8, 16)
 * and graph replay (1, default) or direct launches (0). */
int awp_batch_set_shape(awp_batch* batch, int ty, int ichunk);
int awp_batch_get_shape(const awp_batch* batch, int* ty, int* ichunk);
int awp_batch_set_graph(awp_batch* batch, int use_graph);
/* Execution mode: 0 (default) the persistent tile-queue launches above;
 * 1 one graph per step whose parallel branches are each instance's own tuned
 * launches (velocity, stress, sources at the device-held step, free-surface
 * images), the step counter advanced after the join.  Same results. */
int awp_batch_set_mode(awp_batch* batch, int mode);
int awp_batch_get_mode(const awp_batch* batch);
/* Mode 1: the instances' launches are dealt, largest first, round-robin onto
 * `branches` parallel graph branches (0, the default: one branch per
 * instance). */
int awp_batch_set_branches(awp_batch* batch, int branches);
/* info = instances, interior cells, velocity tiles, stress tiles, persistent
 * CTAs of the velocity and stress launches. */
int awp_batch_info(awp_batch* batch, long long info[6]);

/* ------------------------------------------------------------------------ */
/* Materials, seismograms and the adjoint gradient (single grid, Cartesian,  */
/* NVE 1/2, IFAULT 1 sources)                                                */
/* ------------------------------------------------------------------------ */
/* Lame moduli and density of the interior, arrays [nz][ny][nx] in host or
 * device memory (surface first, the mesh-file order), into the kernel arrays (1/lambda, 1/mu, rho
 * with the one-cell border copy of the media set-up) and the surface ratio
 * lambda/(lambda+2mu).  Q and the memory-variable set-up of the last media
 * upload stay (upload media first). */
int awp_set_moduli(awp_ctx* ctx, const float* lambda, const float* mu, const float* rho);
/* Wavefield and memory variables to zero, step counter to 0 (sources start
 * over). */
int awp_reset(awp_ctx* ctx);
/* nsteps forward steps, sampling after each step the velocity component
 * rec_comp[r] (0 u, 1 v, 2 w) at interior cell rec_xyz[r] = (x, y, z), z counted
 * from the surface: seis[nsteps][nrec] (host). */
int awp_seismograms(awp_ctx* ctx, int nsteps, int nrec, const int* rec_xyz, const int* rec_comp,
                    float* seis);
/* The same forward run with the misfit J = 1/2 sum_n sum_r (seis - d_obs)^2
 * and its gradient with respect to lambda, mu, rho of every interior cell
 * (arrays [nz][ny][nx] in host or device memory, surface first; Q held
 * fixed), by the discrete
 * adjoint of the time step: hand-written transposes of the velocity, stress,
 * memory-variable, free-surface-image and imaging updates.  Forward states:
 * with nsnap > 0, nsnap full-state snapshots in device memory, each segment
 * between them run forward again before its backward sweep (revolve-style,
 * about sqrt(nsteps) snapshots); with nsnap = 0, the velocities of as many of
 * the last steps as fit in 90 % of the free device memory are kept from the
 * first forward pass and only the earlier steps are snapshotted (every
 * ceil(sqrt) steps) and recomputed.  The workspace stays allocated in the
 * context for the next call.  The context ends on the state after nsteps
 * steps.  seis (optional) receives the samples.  AWP_ERR_NOMEM when the
 * snapshots do not fit, with the size in awp_last_error. */
int awp_misfit_gradient(awp_ctx* ctx, int nsteps, int nrec, const int* rec_xyz, const int* rec_comp,
                        const float* d_obs, int nsnap, double* misfit, float* seis,
                        float* g_lambda, float* g_mu, float* g_rho);
/* The same gradient plus, where attenuation is on, the gradient with respect
 * to the inverse quality factors Qp^-1 and Qs^-1 of every interior cell (host
 * arrays [nz][ny][nx], surface first; lambda, mu, rho held fixed): the
 * adjoint of the memory-variable coefficients through the Q(f) weights of
 * dstrqc (kernel.cu:974-1040), each weight's branch (low-Q polynomial or
 * linear) held as the forward takes it.  g_qpinv / g_qsinv may be NULL; on
 * an elastic context (every Q^-1 zero) they come back zero. */
int awp_misfit_gradient_q(awp_ctx* ctx, int nsteps, int nrec, const int* rec_xyz,
                          const int* rec_comp, const float* d_obs, int nsnap, double* misfit,
                          float* seis, float* g_lambda, float* g_mu, float* g_rho,
                          float* g_qpinv, float* g_qsinv);
/* Inverse quality factors Qp^-1, Qs^-1 of the interior (host arrays
 * [nz][ny][nx], surface first) into the kernel arrays with the one-cell
 * border copy of the media set-up; moduli and density stay. */
int awp_set_qinv(awp_ctx* ctx, const float* qpinv, const float* qsinv);
/* The forward-state storage awp_misfit_gradient would use for nsteps steps
 * and this nsnap, from the free device memory now: tail_steps steps keep
 * their velocities, the others run again in segments of segment_steps steps
 * from snapshots full states; workspace_gb is the slab it allocates.  Any
 * output may be NULL. */
int awp_adjoint_plan(awp_ctx* ctx, int nsteps, int nsnap, int* tail_steps, int* segment_steps,
                     int* snapshots, double* workspace_gb);
/* Allocate now the workspace awp_misfit_gradient(nsteps, nsnap) would
 * allocate on its first call (it stays in the context), so that an inversion
 * loop or a timing excludes the allocation. */
int awp_adjoint_reserve(awp_ctx* ctx, int nsteps, int nsnap);

/* Host-only helper (no context, no GPU): the metric arrays of a topography
 * file (INTOPO) for an nx x ny x nz grid of spacing h, as topo_init_metrics /
 * topo_init_geometry / topo_build compute them (src/topography/topography.c:
 * 238-262).  out = the ten f arrays f, f_1, f_2, f_c, f1_1, f1_2, f1_c, f2_1,
 * f2_2, f2_c ((nx+20) x (ny+84) each), then g, g_c, g3, g3_c (nz+64 each).
 * Returns 0 or the reference's error code (101 unreadable, 902 sizes). */
int awp_topo_metrics(const char* path, int nx, int ny, int nz, float h, float* out);

/* Curvilinear topography of the top grid (INTOPO; replaces topo_init /
 * topo_bind / topo_init_metrics / topo_init_grid / topo_init_geometry /
 * topo_build / topo_set_constants, pmcl3d.c:1522-1550).  Reads the elevation
 * file (int32 nx, ny, padding; float32 [nx+2 padding][ny+2 padding], y
 * fastest), builds the metrics and from then on the context's velocity and
 * stress half-steps are the curvilinear ones (topo_velocity_*_H,
 * topo_stress_*_H: interior operators below the top six points, boundary
 * closures on them, stress window ngsl/2 cells in from each side).  Receivers
 * and SOURCEFILE sources initialised afterwards are placed through the
 * surface function and the SOURCEFILE moments divided by the cell Jacobian
 * (sources_add_curvilinear).  Only on grid 0, nzt >= 12, and before
 * awp_receivers_init / awp_sourcefile_init (AWP_ERR_STATE otherwise).
 * Returns AWP_ERR_IO for an unreadable file, AWP_ERR_ARG for sizes or padding
 * that do not fit the context. */
int awp_topography_init(awp_ctx* ctx, const char* intopo);
/* Stress update of a curvilinear top grid with plasticity (NVE = 3).
 * consistent = 0 (default): the reference's single-rank behaviour -- with
 * NVE = 3 pmcl3d skips the curvilinear interior stress and runs the Cartesian
 * dstrqc only over the middle band xss2..xse2 x yls2..yre2 of grid 0
 * (pmcl3d.c:1855-1879, 2139-2148; topo_stress_left/right_H return at one
 * rank, src/topography/stress_attenuation.cu:323-325, 430-432).
 * consistent = 1: a documented change of behaviour -- the curvilinear stress
 * (and memory variables) on the whole window, then the plasticity return, as
 * NVE 1/2 do plus the return. */
int awp_set_topo_plasticity(awp_ctx* ctx, int consistent);

/* Advance nsteps time steps (pmcl3d.c:1628-2487 order: velocity, stress +
 * attenuation, SOURCEFILE and INSRC sources, plasticity, free-surface stress
 * images, receivers).  Asynchronous with respect to the host except when a
 * receiver ring is written to disk or a source ring is refilled from disk;
 * call awp_synchronize to wait. */
int awp_step(awp_ctx* ctx, int nsteps);
int awp_synchronize(awp_ctx* ctx);
/* Number of completed time steps. */
int awp_current_step(const awp_ctx* ctx, long long* step);

/* Whole padded fields: host copies and raw device pointers. */
int awp_field_download(awp_ctx* ctx, int field, float* host);
int awp_field_upload(awp_ctx* ctx, int field, const float* host);
int awp_field_device_ptr(awp_ctx* ctx, int field, float** dev_ptr);

/* Surface / volume output gather of velbuffer (kernel.cu:3948-4011) into
 * caller buffers (device or pinned host), one value per recording point (on
 * grid 0 the w component one cell below the recorded level, as velbuffer),
 * x fastest: rec_n = ((ned-nbg)/nskp+1) per axis, indices 0-based as
 * calcRecordingPoints (calc.c:9-72) returns them. */
int awp_gather_output(awp_ctx* ctx, int nbgx, int nedx, int nskpx, int nbgy,
                      int nedy, int nskpy, int nbgz, int nedz, int nskpz,
                      float* bufx, float* bufy, float* bufz, float* bufeta);

/* FOLLOWBATHY=1 (pmcl3d.c:905-930, kernel.cu:3975-3983): the surface level of
 * every padded (i, j) column of grid 0, int[ny+4+2*ngsl][nx+4+2*ngsl] (x
 * fastest).  awp_compute_bathymetry fills it from the context's media as
 * pmcl3d does (the highest level k > align, from the top down, whose
 * sqrt(1/(mu*d1)) exceeds 0.001; 0 where none does); awp_set_bathymetry makes
 * awp_gather_output on this grid read level bathy-k of each column (w one cell
 * lower where the level is the top one), or clears it with NULL.  A gather
 * whose depth reaches below level 0 of a recorded column is refused. */
int awp_compute_bathymetry(awp_ctx* ctx, int* bathy);
int awp_set_bathymetry(awp_ctx* ctx, const int* bathy);

/* Device-side non-finite sentinel over velocities and stresses: *ok = 1 when
 * every value is finite. */
int awp_check_finite(awp_ctx* ctx, int* ok);

/* Allocation-free non-finite check -- no counterpart in the reference.
 *
 * For callers that own all the device memory they may use and cannot ask the
 * CUDA allocator for more (a host code running the wavefield in its own
 * pre-reserved pool, or a watchdog thread checking a running simulation
 * between steps, where cudaMalloc could fail on a full device and cudaFree
 * would wait for the whole device).  awp_check_finite needs a context, which
 * allocates; this call allocates nothing.
 *
 * fields: host array of nfields device pointers, each to n floats.  On return
 * ok[f] = 1 when every value of field f is finite, else 0.  Work is queued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and the call waits
 * for it.  nfields above AWP_NOALLOC_MAX_FIELDS is rejected with AWP_ERR_ARG.
 *
 * Scratch is one fixed device array of AWP_NOALLOC_MAX_FIELDS flags per GPU,
 * held by every GPU that loads the library until the process exits.  The
 * first call on a device looks its address up (and caches it), so make that
 * first call before any stream capture.  All calls share the array: calls
 * whose work overlaps on the GPU (other threads or streams) race on it. */
#define AWP_NOALLOC_MAX_FIELDS 32
int awp_check_finite_noalloc(const float* const* fields, int nfields, long long n, int* ok,
                             void* stream);

/* Per-phase device timing: when enabled, every subsequent awp_step records
 * CUDA events around each of its phases on the context's stream.
 * awp_phase_times waits for the stream and returns, per phase, the summed
 * milliseconds and the number of launches since the last call:
 * 0 velocity, 1 stress, 2 sources, 3 plasticity, 4 free-surface stress. */
#define AWP_NPHASES 5
int awp_profile_phases(awp_ctx* ctx, int enable);
int awp_phase_times(awp_ctx* ctx, double ms[AWP_NPHASES], long long launches[AWP_NPHASES]);
/* Launch-shape tuning of the stencil kernels (process-wide): key "ichunk"
 * (x planes marched per CTA, 4..1024), "tma_vel" / "tma_str" (1: the context
 * API runs the TMA-pipelined velocity / stress kernel, 0: the read-only-path
 * one; results are bit-identical), "tma" (sets both; reads -1 when they
 * differ) and "spin_limit" (0 .. 2^30, default 2^26: polls of each pipeline
 * wait of the TMA kernels before it gives up, 0 = give up at once; a wait that
 * gives up makes the CTA drain its issued copies and leave, and the next
 * awp_synchronize of the context returns AWP_ERR_CUDA once) and
 * "l2_promotion" (0 none, 1 64 B, 2 128 B, 3 256 B (default): the L2 fetch
 * granule of the TMA tiles; a context re-encodes its tensor maps before its
 * next TMA launch after a change; results do not change).  Returns AWP_OK or
 * AWP_ERR_ARG;
 * awp_get_tuning returns the value or -1 for an unknown key. */
int awp_set_tuning(const char* key, int value);
int awp_get_tuning(const char* key);

/* Kernels this context has launched so far. */
int awp_kernel_launches(const awp_ctx* ctx, long long* launches);

/* Bytes of device memory the context holds. */
int awp_device_bytes(const awp_ctx* ctx, long long* bytes);

/* ------------------------------------------------------------------------ */
/* Host set-up helpers (exported for tests and the pmcl3d driver)           */
/* ------------------------------------------------------------------------ */
/* tausub (mesh.c:684-710) after inimesh's tau range (mesh.c:36-57);
 * returns AWP_ERR_UNSUPPORTED for EX >= 0.95 (range left unset there). */
int awp_q_tau(float ex, float fac, float* taumax, float* taumin, float tau8[8]);
/* weights_sub (mesh.c:713-1097). */
int awp_q_weights(float ex, float fac, float w8[8], float coeff16[16]);
/* inicrj (cerjan.c:5-64), single rank; arrays pre-sized to the padded axes. */
int awp_cerjan(float arbc, int nxt, int nyt, int nzt, int nd, int islowest, int npc,
               float* dcrjx, float* dcrjy, float* dcrjz);
/* The eight vx1/vx2/wwo values and ww of init_texture (mesh.c:1103-1137) at
 * one padded cell, from the pattern the kernels use. */
int awp_texture_at(const float tau8[8], const float w8[8], float dt, int xls,
                   int yls, int ny, int nzt, int i, int j, int k, float* vx1,
                   float* vx2, int* ww, float* wwo);

/* ------------------------------------------------------------------------ */
/* Reference-compatible launchers (include/awp/kernel_launch.h)             */
/* ------------------------------------------------------------------------ */
typedef struct CUstream_st* awp_stream_t; /* == cudaStream_t */

/* kernel_launch.h:24 */
void SetDeviceConstValue(float* DH, float DT, int* nxt, int* nyt, int* nzt,
                         int ngrids, float fmajor, float fminor, float* Rz,
                         float* RzT);
/* kernel_launch.h:28 */
void SetDeviceFilterParameters(int filtorder, double* srcfilt_b, double* srcfilt_a);
/* kernel_launch.h:31 */
void dvelcx_H_opt(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                  float* xy, float* xz, float* yz, float* dcrjx, float* dcrjy,
                  float* dcrjz, float* d_1, int nyt, int nzt, awp_stream_t St,
                  int s_i, int e_i, int d_i, int ngrids);
/* kernel_launch.h:36 (single rank: returns at rank == -1 like the reference) */
void dvelcy_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
              float* xy, float* xz, float* yz, float* dcrjx, float* dcrjy,
              float* dcrjz, float* d_1, int nxt, int nzt, float* s_u1,
              float* s_v1, float* s_w1, awp_stream_t St, int s_j, int e_j,
              int rank, int d_i);
/* kernel_launch.h:51 */
void dstrqc_H(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz,
              float* r1, float* r2, float* r3, float* r4, float* r5, float* r6,
              float* u1, float* v1, float* w1, float* lam, float* mu, float* qp,
              float* coeff, float* qs, float* dcrjx, float* dcrjy, float* dcrjz,
              int nyt, int nzt, awp_stream_t St, float* lam_mu, float* vx1,
              float* vx2, int* ww, float* wwo, int NX, int NPC, int rankx,
              int ranky, int s_i, int e_i, int s_j, int e_j, int d_i);
/* kernel_launch.h:42 (same arithmetic as dstrqc_H) */
void dstrqc_H_new(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz,
                  float* r1, float* r2, float* r3, float* r4, float* r5, float* r6,
                  float* u1, float* v1, float* w1, float* lam, float* mu, float* qp,
                  float* coeff, float* qs, float* dcrjx, float* dcrjy, float* dcrjz,
                  int nyt, int nzt, awp_stream_t St, float* lam_mu, float* vx1,
                  float* vx2, int* ww, float* wwo, int NX, int NPC, int rankx,
                  int ranky, int s_i, int e_i, int s_j, int e_j, int d_i);
/* kernel_launch.h:58 */
void fstr_H(float* zz, float* xz, float* yz, awp_stream_t St, int s_i, int e_i,
            int s_j, int e_j);
/* kernel_launch.h:61 */
void drprecpc_calc_H_opt(float* xx, float* yy, float* zz, float* xy, float* xz,
                         float* yz, float* mu, float* d1, float* sigma2,
                         float* yldfac, float* cohes, float* phi, float* neta,
                         int nzt, int xls, int xre, int yls, int yre,
                         awp_stream_t St, int d_i);
/* kernel_launch.h:67 */
void drprecpc_app_H(float* xx, float* yy, float* zz, float* xy, float* xz,
                    float* yz, float* mu, float* sigma2, float* yldfac, int nzt,
                    int xls, int xre, int yls, int yre, awp_stream_t St, int d_i);
/* kernel_launch.h:72 */
void addsrc_H(int i, int READ_STEP, int dim, int* psrc, int npsrc, awp_stream_t St,
              float* axx, float* ayy, float* azz, float* axz, float* ayz,
              float* axy, float* xx, float* yy, float* zz, float* xy, float* yz,
              float* xz, int d_i);
/* kernel_launch.h:150 */
void addkinsrc_H(int i, int dim, int* psrc, int npsrc, awp_stream_t St, float* mu,
                 float* axx, float* ayy, float* azz, float* axz, float* ayz,
                 float* axy, float* xx, float* yy, float* zz, float* xy, float* yz,
                 float* xz, float* mom, double* d_srcfilt_d, int d_i);
/* kernel_launch.h:182 */
void velbuffer_H(const float* u1, const float* v1, const float* w1,
                 const float* neta, float* Bufx, float* Bufy, float* Bufz,
                 float* Bufeta, int NVE, int nbgx, int nedx, int nskpx, int nbgy,
                 int nedy, int nskpy, int nbgz, int nedz, int nskpz, int rec_nxt,
                 int rec_nyt, int rec_nzt, awp_stream_t St, int FOLLOWBATHY,
                 const int* bathy, int d_i);

/* kernel_launch.h:92 -- 2nd-order velocity of the interface layer of grid d_i */
void dvelc2_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz, float* xy,
              float* xz, float* yz, float* dcrjx, float* dcrjy, float* dcrjz, float* d_1,
              int nxt, int nyt, awp_stream_t St, int d_i);
/* kernel_launch.h:97 -- 2nd-order stress of the interface layer of grid d_i,
 * memory-variable coefficients from the caller's vx1/vx2/ww/wwo arrays */
void dstrqc2_H(float* xx, float* yy, float* zz, float* xy, float* xz, float* yz, float* r1,
               float* r2, float* r3, float* r4, float* r5, float* r6, float* u1, float* v1,
               float* w1, float* lam, float* mu, float* qp, float* qs, float* dcrjx,
               float* dcrjy, float* dcrjz, int nxt, int nyt, awp_stream_t St, float* coeff,
               float* d_vx1, float* d_vx2, int* d_ww, float* d_wwo, int s_i, int e_i, int s_j,
               int e_j, int d_i);
/* kernel_launch.h:105 -- coarse (grid d_i, "l") to fine (grid d_i-1, "h") */
void intp3d_H(float* u1l, float* v1l, float* w1l, float* xxl, float* yyl, float* zzl,
              float* xyl, float* xzl, float* yzl, float* u1h, float* v1h, float* w1h, float* xxh,
              float* yyh, float* zzh, float* xyh, float* xzh, float* yzh, int nxtl, int nytl,
              int rank, awp_stream_t St, int d_i);
/* kernel_launch.h:111 -- fine (grid d_i, "h") to coarse (grid d_i+1, "l") window
 * average; at one rank the swap-area buffers are not read */
void swap_H(float* xxl, float* yyl, float* zzl, float* xyl, float* xzl, float* yzl, float* u1l,
            float* v1l, float* w1l, float* xxh, float* yyh, float* zzh, float* xyh, float* xzh,
            float* yzh, float* u1h, float* v1h, float* w1h, int nxtl, int nytl, float* buf_L,
            float* buf_R, float* buf_F, float* buf_B, int rank, awp_stream_t St, int d_i);
/* kernel_launch.h:74 -- prescribed velocities at the source points (IFAULT 4) */
void frcvel_H(int i, int READ_STEP, int dim, int* psrc, int npsrc, int tskp, awp_stream_t St,
              float* axx, float* ayy, float* azz, float* axz, float* ayz, float* axy, float* u1,
              float* v1, float* w1, int ymin, int ymax, int d_i);
/* kernel_launch.h:127 -- plane-wave source (IFAULT 6) at k = align+ND+1 */
void addplanesrc_H(int i, int dim, int NST, awp_stream_t St, float* mu, float* lambda, int ND,
                   int nxt, int nyt, float* axx, float* ayy, float* azz, float* xx, float* yy,
                   float* zz, float* xy, float* yz, float* xz, int d_i);
/* kernel_launch.h:79 -- free-surface velocity images of grid 0 */
void fvel_H(float* u1, float* v1, float* w1, awp_stream_t St, float* lam_mu, int NX, int rankx,
            int ranky, int s_i, int e_i, int s_j, int e_j);
/* kernel_launch.h:82-91, 132-178 -- halo exchanges between ranks: return at
 * once when both neighbour ranks are -1 (world size 1), like the reference;
 * any other rank is refused with the launchers' error behaviour */
void update_bound_y_H(float* u1, float* v1, float* w1, float* f_u1, float* f_v1, float* f_w1,
                      float* b_u1, float* b_v1, float* b_w1, int nxt, int nzt, awp_stream_t St1,
                      awp_stream_t St2, int rank_f, int rank_b, int d_i);
void update_yldfac_buffer_x_H(float* yldfac, float* buf_L, float* buf_R, int nyt, int nzt,
                              awp_stream_t St1, awp_stream_t St2, int rank_L, int rank_R,
                              int d_i);
void update_yldfac_data_x_H(float* yldfac, float* buf_L, float* buf_R, int nyt, int nzt,
                            awp_stream_t St1, awp_stream_t St2, int rank_L, int rank_R, int d_i);
void update_yldfac_buffer_y_H(float* yldfac, float* buf_F, float* buf_B, int nxt, int nzt,
                              awp_stream_t St1, awp_stream_t St2, int rank_F, int rank_B,
                              int d_i);
void update_yldfac_data_y_H(float* yldfac, float* buf_F, float* buf_B, int nxt, int nzt,
                            awp_stream_t St1, awp_stream_t St2, int rank_F, int rank_B, int d_i);
void update_swapzone_buffer_x_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                                float* xy, float* xz, float* yz, float* buf_L, float* buf_R,
                                int nyt, awp_stream_t St1, awp_stream_t St2, int rank_L,
                                int rank_R, int zs, int ze, int meshtp);
void update_swapzone_data_x_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                              float* xy, float* xz, float* yz, float* buf_L, float* buf_R, int nyt,
                              awp_stream_t St1, awp_stream_t St2, int rank_L, int rank_R, int zs,
                              int ze, int meshtp);
void update_swapzone_buffer_y_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                                float* xy, float* xz, float* yz, float* buf_F, float* buf_B,
                                int nxt, awp_stream_t St1, awp_stream_t St2, int rank_F,
                                int rank_B, int zs, int ze, int d_i);
void update_swapzone_data_y_H(float* u1, float* v1, float* w1, float* xx, float* yy, float* zz,
                              float* xy, float* xz, float* yz, float* buf_F, float* buf_B, int nxt,
                              awp_stream_t St1, awp_stream_t St2, int rank_F, int rank_B, int zs,
                              int ze, int d_i);
/* kernel_launch.h:11-19 -- device-side debug printing, compiled out in the
 * reference (kernel.cu:270-296, 3236-3318): no output, no launch */
void print_const_H(int ngrids);
void print_nonzero_H(float* array, int nx, int ny, int nz, int d_i, int rank);
void print_nonzero_mat_H(float* array, int nx, int ny, int nz, int d_i, float* d1, float* mu,
                         float* lam, float* qp, float* qs, int rank);
void print_nan_H(float* array, int nx, int ny, int nz, char* vname);

/* Error mode of the launchers above: 1 (default) = print and exit like the
 * reference's CUCHK; 0 = record the error and return. */
void awp_compat_exit_on_error(int exit_on_error);
/* Last error recorded by a launcher (0 = none); reading clears it. */
int awp_compat_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* AWP_B200_H */
