// Receivers (RECVFILE) and SOURCEFILE sources: device tables, ring buffers
// and the per-step hooks.
//
// Reference behaviour restated here (one rank, one grid block):
//  * receivers: every `stride` steps the three velocity components are
//    interpolated at the receivers into a device ring of gpu_buffer_size
//    slots (cuinterp_dinterp, interpolation/interpolation.cu:177-199); a full
//    device ring is copied into the host ring of cpu_buffer_size blocks; a
//    full host ring is transposed to receiver-major order and written to
//    "<file>_<x|y|z>_<step>" (topography/receivers/receiver.c:47-75).
//  * SOURCEFILE: the binary moment-rate series "<file>_<xx..yz>" are read in
//    blocks of gpu*cpu samples (source.c:449-472), staged through the same
//    rings, and every `stride` steps added with Lagrange weights
//    (cusource_add_cartesian, sources/source.cu:24-49).
// The device ring copies are asynchronous on the context's stream; the host
// waits only when a host ring is written to disk or refilled from disk.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "awp_pointsets.h"
#include "awp_points.h"
#include "awp_topo.h"

namespace {

constexpr int kMaxBasis = 8;  // degree <= 7

// The fields a receiver set reads, indexed by component.
struct GatherFields {
  const float* f[6];
};

__global__ void k_recv_gather(const int4* __restrict__ q, const float* __restrict__ l, int nq,
                              int nb, const GatherFields F, int slice, int yline,
                              float* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const int4 qi = q[t];  // ix, iy, iz, (component << 24) | output index
  const int comp = qi.w >> 24, oi = qi.w & 0xffffff;
  const float* __restrict__ in = F.f[comp];
  const float* lx = l + (size_t)t * 3 * nb;
  const float* ly = lx + nb;
  const float* lz = ly + nb;
  float acc = 0.0f;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j)
      for (int k = 0; k < nb; ++k) {
        // grid_index of the metric grid: offsets (2, 2, align) (grid/grid_3d.h:113)
        const long long pos = (long long)(2 + qi.x + i) * slice +
                              (long long)(2 + qi.y + j) * yline + (AWP_ALIGN + qi.z + k);
        acc = __fmaf_rn(__fmul_rn(__fmul_rn(lx[i], ly[j]), lz[k]), in[pos], acc);
      }
  out[oi] = acc;
}

struct SrcCellArgs {
  float* f[6];
  const long long* pos;
  const int* comp;
  const int* first;
  const float* w;
  const int* src;
  const float* vals;  // one ring slot
  int ncell;
};

__global__ void k_srcfile_add(const SrcCellArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  float* F = a.f[a.comp[c]];
  const long long p = a.pos[c];
  float acc = F[p];
  for (int n = a.first[c]; n < a.first[c + 1]; ++n) acc = __fmaf_rn(a.w[n], a.vals[a.src[n]], acc);
  F[p] = acc;
}

// FORCEFILE (cusource_add_force, source.cu:118-157): per cell of a velocity
// component, the contributions w * rate * Ji in file order, Ji = -q / (f dg rho)
// with rho read ngsl cells further in x and y than the cell, as the
// reference's _rho macro indexes it.
struct ForceCellArgs {
  float* f[3];
  const float* d1;
  const long long* pos;
  const int* comp;
  const int* first;
  const float* w;
  const float* fdg;
  const long long* rho;
  const int* src;
  const float* vals;  // one ring slot
  float qw[3];
  int ncell;
};

__global__ void k_force_add(const ForceCellArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int comp = a.comp[c];
  float* F = a.f[comp];
  const long long p = a.pos[c];
  const float nq = -a.qw[comp];
  float acc = F[p];
  for (int n = a.first[c]; n < a.first[c + 1]; ++n) {
    const float Ji = __fdiv_rn(nq, __fmul_rn(a.fdg[n], a.d1[a.rho[n]]));
    acc = __fmaf_rn(__fmul_rn(a.w[n], a.vals[a.src[n]]), Ji, acc);
  }
  F[p] = acc;
}

int fail(char* msg, size_t cap, int status, const char* what) {
  snprintf(msg, cap, "%s", what);
  return status;
}
int failf(char* msg, size_t cap, int status, const char* fmt, const char* what) {
  snprintf(msg, cap, fmt, what);
  return status;
}

#define CU_OK(call, msg, cap)                                                        \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      snprintf(msg, cap, "%s: %s", #call, cudaGetErrorString(e_));                   \
      return -1;                                                                     \
    }                                                                                \
  } while (0)

template <typename T>
int upload(T** d, const std::vector<T>& h, char* msg, size_t cap) {
  *d = nullptr;
  if (h.empty()) return 0;
  CU_OK(cudaMalloc((void**)d, h.size() * sizeof(T)), msg, cap);
  CU_OK(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), msg, cap);
  return 0;
}

awp::BlockDesc block_of(const AwpGeom& g, float h, const awp::TopoMetrics* topo) {
  awp::BlockDesc b;
  b.nxt = g.nxt;
  b.nyt = g.nyt;
  b.nzt = g.nzt;
  b.h = h;
  b.topography = topo ? 1 : 0;
  return b;
}

int setup_error(int e, const char* what, char* msg, size_t cap) {
  snprintf(msg, cap, "%s: AWP error %d (%s)", what, e,
           e == awp::PE_FILE_READ ? "cannot read file"
           : e == awp::PE_FILE_WRITE ? "cannot write file"
           : e == awp::PE_WRONG_VERSION ? "unsupported input version"
           : e == awp::PE_PARSE_UNKNOWN_ARG ? "unknown header argument"
           : e == awp::PE_PARSE_ARG ? "malformed header line"
           : e == awp::PE_NOT_DIVISIBLE ? "steps not divisible by the buffer sizes"
           : e == awp::PE_BUFFER_SIZES ? "zero buffer size"
           : e == awp::PE_DATA_READ_ELEMENT ? "malformed coordinate line"
           : e == awp::PE_GRID_ASSIGN ? "point outside every grid block"
           : (e == awp::PE_OUT_OF_BOUNDS_LOWER || e == awp::PE_OUT_OF_BOUNDS_UPPER)
               ? "last point lies outside the interpolation grid"
           : (e == awp::PE_LAGRANGE_LOWER || e == awp::PE_LAGRANGE_UPPER)
               ? "Lagrange extrapolation"
               : "set-up failed");
  return e;
}

}  // namespace

// ===========================================================================
// Receivers
// ===========================================================================
struct RecvState {
  awp::InputFile in;
  int ncomp = 0;
  awp::PointSet ps[6];
  awp::RingSchedule ring;
  long long nt = 0;
  std::string base[6];
  int len[6] = {}, off[6] = {}, total = 0;
  int nq = 0, nb = 1;
  int slice = 0, yline = 0;
  size_t current_write = 0;
  int4* d_q = nullptr;
  float* d_l = nullptr;
  float* d_ring = nullptr;  // [num_device][total]
  float* h_ring = nullptr;  // pinned [num_host][num_device][total]
};

void awp_recv_destroy(RecvState* r) {
  if (!r) return;
  cudaFree(r->d_q);
  cudaFree(r->d_l);
  cudaFree(r->d_ring);
  if (r->h_ring) cudaFreeHost(r->h_ring);
  delete r;
}

int awp_recv_length(const RecvState* r, int comp) {
  return (r && comp >= 0 && comp < r->ncomp) ? r->len[comp] : 0;
}

std::string awp_recv_base(const RecvState* r, int comp) {
  return (r && comp >= 0 && comp < r->ncomp) ? r->base[comp] : std::string();
}

// receiver_init (receivers/receiver.c:17-41) for each of `ncomp` components
// of one input: component c on the staggered grid types[c], its files named
// `<file>_<names[c]>`.
static int recv_create(const awp::InputFile& in, long long nt, const AwpGeom& g, float h,
                       const awp::TopoMetrics* topo, int ncomp, const awp::GridType* types,
                       const char* const* names, const char* what, RecvState** out,
                       char* msg, size_t cap) {
  *out = nullptr;
  RecvState* r = new RecvState();
  r->in = in;
  r->ncomp = ncomp;
  if (r->in.degree < 0 || r->in.degree + 1 > kMaxBasis || r->in.stride < 1 ||
      r->in.gpu_buffer_size < 1 || r->in.cpu_buffer_size < 1 || r->in.num_writes < 1) {
    delete r;
    return failf(msg, cap, awp::PE_PARSE_ARG,
                 "%s: degree 0..7, stride >= 1 and nonzero buffer sizes are required", what);
  }
  const awp::BlockDesc b = block_of(g, h, topo);
  std::vector<int4> q;
  std::vector<float> l;
  r->nb = r->in.degree + 1;
  for (int c = 0; c < ncomp; ++c) {
    const int e = awp::point_set_init(r->in, types[c], &b, 1, &r->ps[c], topo);
    if (e) {
      awp_recv_destroy(r);
      return setup_error(e, what, msg, cap);
    }
    r->base[c] = r->in.file + "_" + names[c];
    r->len[c] = (int)r->ps[c].indices.size();
    r->off[c] = r->total;
    r->total += r->len[c];
    const awp::BlockInterp& bi = r->ps[c].block[0];
    for (int k = 0; k < bi.num_query; ++k) {
      q.push_back(make_int4(bi.ix[k], bi.iy[k], bi.iz[k], (c << 24) | (r->off[c] + bi.ridx[k])));
      for (int d = 0; d < r->nb; ++d) l.push_back(bi.lx[(size_t)k * r->nb + d]);
      for (int d = 0; d < r->nb; ++d) l.push_back(bi.ly[(size_t)k * r->nb + d]);
      for (int d = 0; d < r->nb; ++d) l.push_back(bi.lz[(size_t)k * r->nb + d]);
    }
  }
  r->nq = (int)q.size();
  r->nt = nt;
  r->slice = g.slice;
  r->yline = g.yline;
  r->ring.num_device = r->in.gpu_buffer_size;
  r->ring.num_host = r->in.cpu_buffer_size;
  r->ring.stride = (size_t)r->in.stride;
  if (upload(&r->d_q, q, msg, cap) || upload(&r->d_l, l, msg, cap)) {
    awp_recv_destroy(r);
    return -1;
  }
  const size_t slot = (size_t)std::max(r->total, 1);
  if (cudaMalloc((void**)&r->d_ring, sizeof(float) * slot * r->ring.num_device) != cudaSuccess ||
      cudaMemset(r->d_ring, 0, sizeof(float) * slot * r->ring.num_device) != cudaSuccess ||
      cudaMallocHost((void**)&r->h_ring,
                     sizeof(float) * slot * r->ring.num_device * r->ring.num_host) != cudaSuccess) {
    awp_recv_destroy(r);
    return failf(msg, cap, -1, "%s: ring buffer allocation failed", what);
  }
  memset(r->h_ring, 0, sizeof(float) * slot * r->ring.num_device * r->ring.num_host);
  *out = r;
  return 0;
}

int awp_recv_create(const char* path, long long nt, const AwpGeom& g, float h,
                    const awp::TopoMetrics* topo, RecvState** out,
                    char* msg, size_t cap) {
  *out = nullptr;
  awp::InputFile in;
  const int e = awp::read_input(path, &in);
  if (e) return setup_error(e, "RECVFILE", msg, cap);
  // receivers_init (receivers/receivers.c:38-40)
  const awp::GridType t[3] = {awp::GT_X, awp::GT_Y, awp::GT_Z};
  const char* names[3] = {"x", "y", "z"};
  return recv_create(in, nt, g, h, topo, 3, t, names, "RECVFILE", out, msg, cap);
}

int awp_sgt_create(const char* path, long long nt, const AwpGeom& g, float h,
                   const awp::TopoMetrics* topo, RecvState** out, RecvState** mat,
                   char* msg, size_t cap) {
  *out = *mat = nullptr;
  awp::InputFile in;
  int e = awp::read_input(path, &in);
  if (e) return setup_error(e, "SGTFILE", msg, cap);
  // sgt_init (receivers/sgt.c:29-58): the six stresses, then the material
  // properties on the node grid, written once without buffering
  const awp::GridType t[6] = {awp::GT_XX, awp::GT_YY, awp::GT_ZZ,
                              awp::GT_XY, awp::GT_XZ, awp::GT_YZ};
  const char* names[6] = {"Gxx", "Gyy", "Gzz", "Gxy", "Gxz", "Gyz"};
  e = recv_create(in, nt, g, h, topo, 6, t, names, "SGTFILE", out, msg, cap);
  if (e) return e;
  awp::InputFile min = in;
  min.gpu_buffer_size = 1;
  min.cpu_buffer_size = 1;
  min.steps = 1;
  min.num_writes = 1;
  const awp::GridType tn[1] = {awp::GT_NODE};
  const char* nn[1] = {""};
  e = recv_create(min, 1, g, h, topo, 1, tn, nn, "SGTFILE", mat, msg, cap);
  if (e) {
    awp_recv_destroy(*out);
    *out = nullptr;
  }
  return e;
}

// receiver_write (receivers/receiver.c:48-75) of every component at `step`;
// `name` replaces the file name of component 0 (the one-shot material output).
static int recv_write(RecvState* r, long long step, const float* const* fields,
                      const char* name0, cudaStream_t st, long long* launches, char* msg,
                      size_t cap) {
  if (!r || r->total == 0 || step < 0) return 0;
  const size_t s = (size_t)step;
  const size_t T = (size_t)r->total, nd = r->ring.num_device;
  if (!r->ring.device_ready(s)) return 0;
  if (r->nq > 0) {
    float* slot = r->d_ring + r->ring.device_slot(s) * T;
    GatherFields F{};
    for (int c = 0; c < r->ncomp; ++c) F.f[c] = fields[c];
    k_recv_gather<<<(r->nq + 127) / 128, 128, 0, st>>>(r->d_q, r->d_l, r->nq, r->nb, F,
                                                       r->slice, r->yline, slot);
    CU_OK(cudaGetLastError(), msg, cap);
    if (launches) ++*launches;
  }
  if (r->ring.device_full(s)) {  // buffer_copy_to_host (buffers/buffer.c:98-104)
    float* dst = r->h_ring + r->ring.host_slot(s) * nd * T;
    CU_OK(cudaMemcpyAsync(dst, r->d_ring, sizeof(float) * nd * T, cudaMemcpyDeviceToHost, st),
          msg, cap);
  }
  if (r->ring.host_full(s)) {  // transpose and indexed write (receiver.c:62-74)
    CU_OK(cudaStreamSynchronize(st), msg, cap);
    const size_t rows = r->ring.num_host * nd;
    for (int c = 0; c < r->ncomp; ++c) {
      if (r->len[c] == 0) continue;
      std::vector<float> data((size_t)r->len[c] * rows);
      for (size_t t = 0; t < rows; ++t)
        for (int i = 0; i < r->len[c]; ++i)
          data[(size_t)i * rows + t] = r->h_ring[t * T + r->off[c] + i];
      const std::string name =
          (c == 0 && name0)
              ? std::string(name0)
              : awp::receiver_filename(r->base[c], r->in.gpu_buffer_size, r->in.cpu_buffer_size,
                                       r->in.num_writes, r->in.stride, s, (size_t)r->nt);
      const int e = awp::indexed_write(name.c_str(), r->ps[c].indices, rows, r->in.num_writes,
                                       r->current_write, data.data());
      if (e) return setup_error(e, name.c_str(), msg, cap);
    }
    r->current_write = (r->current_write + 1) % r->in.num_writes;
  }
  return 0;
}

int awp_recv_record(RecvState* r, long long step, const float* u, const float* v, const float* w,
                    cudaStream_t st, long long* launches, char* msg, size_t cap) {
  const float* f[3] = {u, v, w};
  return recv_write(r, step, f, nullptr, st, launches, msg, cap);
}

int awp_recv_record_fields(RecvState* r, long long step, const float* const* fields,
                           cudaStream_t st, long long* launches, char* msg, size_t cap) {
  return recv_write(r, step, fields, nullptr, st, launches, msg, cap);
}

int awp_recv_write_once(RecvState* r, const float* field, const char* filename, cudaStream_t st,
                        long long* launches, char* msg, size_t cap) {
  const float* f[1] = {field};
  return recv_write(r, 0, f, filename, st, launches, msg, cap);
}

// ===========================================================================
// SOURCEFILE sources
// ===========================================================================
struct SrcFileState {
  awp::InputFile in;
  int ncomp = 6;
  bool force = false;  // FORCEFILE: three forces on the velocity grids
  awp::PointSet ps[6];
  awp::RingSchedule ring;
  std::string name[6];
  int len[6] = {}, off[6] = {}, total = 0;
  int ncell = 0;
  size_t ne = 1, num_reads = 1, reads_done = 0;
  long long* d_pos = nullptr;
  int *d_comp = nullptr, *d_first = nullptr, *d_src = nullptr;
  float* d_w = nullptr;
  float* d_fdg = nullptr;      // force: f * dg of each contribution
  long long* d_rho = nullptr;  // force: density index of each contribution
  float qw[3] = {};            // force: SBP quadrature weight per component
  float* d_ring = nullptr;  // [num_device][total]
  float* h_ring = nullptr;  // pinned [num_host * num_device][total] (time-major)
  cudaEvent_t h2d_done = nullptr;
  bool h2d_pending = false;
};

void awp_srcf_destroy(SrcFileState* s) {
  if (!s) return;
  cudaFree(s->d_pos);
  cudaFree(s->d_comp);
  cudaFree(s->d_first);
  cudaFree(s->d_src);
  cudaFree(s->d_w);
  cudaFree(s->d_fdg);
  cudaFree(s->d_rho);
  cudaFree(s->d_ring);
  if (s->h_ring) cudaFreeHost(s->h_ring);
  if (s->h2d_done) cudaEventDestroy(s->h2d_done);
  delete s;
}

// sources_init (sources.c:27-50) or, with `force`, forces_init (forces.c:24-50):
// the point sets of every component, their cell-grouped contributions and the
// rate ring buffers.
static int srcf_create(const char* path, const AwpGeom& g, float h, float dt,
                       const awp::TopoMetrics* topo, bool force, SrcFileState** out,
                       char* msg, size_t cap) {
  *out = nullptr;
  const char* what = force ? "FORCEFILE" : "SOURCEFILE";
  SrcFileState* s = new SrcFileState();
  s->force = force;
  s->ncomp = force ? 3 : 6;
  int e = awp::read_input(path, &s->in);
  if (e) {
    delete s;
    return setup_error(e, what, msg, cap);
  }
  if (s->in.degree < 0 || s->in.degree + 1 > kMaxBasis || s->in.stride < 1 ||
      s->in.gpu_buffer_size < 1 || s->in.cpu_buffer_size < 1) {
    delete s;
    return failf(msg, cap, awp::PE_PARSE_ARG,
                 "%s: degree 0..7, stride >= 1 and nonzero buffer sizes are required", what);
  }
  if (force && !topo) {
    delete s;
    return fail(msg, cap, awp::PE_PARSE_ARG,
                "FORCEFILE: the forces act on a curvilinear top block (pmcl3d.c:1988-1994)");
  }
  const awp::BlockDesc b = block_of(g, h, topo);
  const char* mnames[6] = {"xx", "yy", "zz", "xy", "xz", "yz"};
  const char* fnames[3] = {"fx", "fy", "fz"};
  // SBP quadrature weights of the boundary node (forces.c:84-90): the
  // node-centred grids of fx, fy and the nodal grid of fz
  const float qh = 2.9022824945274315f, qn = 3.55599789310935f;
  std::vector<long long> pos, rho;
  std::vector<int> comp, first, src;
  std::vector<float> w, fdg;
  for (int c = 0; c < s->ncomp; ++c) {
    const awp::GridType t =
        force ? (awp::GridType)(awp::GT_X + c) : (awp::GridType)(awp::GT_XX + c);
    e = awp::point_set_init(s->in, t, &b, 1, &s->ps[c], topo);
    if (e) {
      awp_srcf_destroy(s);
      return setup_error(e, what, msg, cap);
    }
    if (force && c == 0) {  // forces_boundary_check (forces.c:52-65)
      for (int i : s->ps[0].indices)
        if (s->in.type[i] != 1) {
          awp_srcf_destroy(s);
          return fail(msg, cap, awp::PE_PARSE_ARG,
                      "FORCEFILE: every force must be placed on the boundary (type 1)");
        }
    }
    s->name[c] = s->in.file + "_" + (force ? fnames[c] : mnames[c]);
    s->len[c] = (int)s->ps[c].indices.size();
    s->off[c] = s->total;
    s->total += s->len[c];
    awp::CellAdds ca;
    awp::source_cell_adds(s->ps[c].block[0], dt, h, g.slice, g.yline, &ca);
    for (size_t n = 0; n + 1 < ca.first.size(); ++n) {
      pos.push_back(ca.cell_pos[n]);
      comp.push_back(c);
      first.push_back((int)w.size() + ca.first[n] - ca.first[0]);
    }
    // sources_add_curvilinear (sources.c:79-101, source.cu:65-100): each
    // contribution is divided by the Jacobian f g of its cell, with the
    // component's staggered f and vertical metric
    if (force) {
      // forces.c:91-96: fx with f_1 and g3_c, fy with f_2 and g3_c, fz with
      // f_c and g3
      const std::vector<float>* F[3] = {&topo->f_1, &topo->f_2, &topo->f_c};
      const std::vector<float>* G[3] = {&topo->g3_c, &topo->g3_c, &topo->g3};
      s->qw[c] = c < 2 ? qh : qn;
      for (size_t n = 0; n + 1 < ca.first.size(); ++n)
        for (int m = ca.first[n]; m < ca.first[n + 1]; ++m) {
          const long long p = ca.cell_pos[n];
          const long long ia = p / g.slice, jb = (p % g.slice) / g.yline, kk = p % g.yline;
          if (ia + AWP_NGSL >= g.nx_pad() || jb + AWP_NGSL >= g.ny_pad()) {
            awp_srcf_destroy(s);
            return fail(msg, cap, awp::PE_PARSE_ARG,
                        "FORCEFILE: a force lies within ngsl cells of the high x or y edge, "
                        "where the density it reads would lie outside the grid");
          }
          fdg.push_back((*F[c])[(size_t)(ia * topo->ld + jb + AWP_ALIGN)] * (*G[c])[(size_t)kk]);
          rho.push_back((ia + AWP_NGSL) * g.slice + (jb + AWP_NGSL) * g.yline + kk);
          w.push_back(ca.w[m]);
          src.push_back(s->off[c] + ca.src[m]);
        }
      continue;
    }
    const std::vector<float>* jf[6] = {nullptr};
    const std::vector<float>* jg[6] = {nullptr};
    if (topo) {
      const std::vector<float>* F[6] = {&topo->f_c, &topo->f_c, &topo->f_c,
                                        &topo->f,   &topo->f_1, &topo->f_2};
      const std::vector<float>* G[6] = {&topo->g3_c, &topo->g3_c, &topo->g3_c,
                                        &topo->g3_c, &topo->g3,   &topo->g3};
      jf[c] = F[c];
      jg[c] = G[c];
    }
    for (size_t n = 0; n + 1 < ca.first.size(); ++n)
      for (int m = ca.first[n]; m < ca.first[n + 1]; ++m) {
        float wm = ca.w[m];
        if (topo) {
          const long long p = ca.cell_pos[n];
          const long long ia = p / g.slice, jb = (p % g.slice) / g.yline, kk = p % g.yline;
          const float J = (*jf[c])[(size_t)(ia * topo->ld + jb + AWP_ALIGN)] * (*jg[c])[(size_t)kk];
          wm = wm * (float)(1.0 / (double)J);
        }
        w.push_back(wm);
        src.push_back(s->off[c] + ca.src[m]);
      }
  }
  first.push_back((int)w.size());
  s->ncell = (int)pos.size();
  s->ring.num_device = s->in.gpu_buffer_size;
  s->ring.num_host = s->in.cpu_buffer_size;
  s->ring.stride = (size_t)s->in.stride;
  s->ne = s->in.gpu_buffer_size * s->in.cpu_buffer_size;
  s->num_reads = s->in.steps / s->ne;  // source_init (source.c:40-41)
  if (s->num_reads == 0) s->num_reads = 1;
  if (upload(&s->d_pos, pos, msg, cap) || upload(&s->d_comp, comp, msg, cap) ||
      upload(&s->d_first, first, msg, cap) || upload(&s->d_src, src, msg, cap) ||
      upload(&s->d_w, w, msg, cap) || upload(&s->d_fdg, fdg, msg, cap) ||
      upload(&s->d_rho, rho, msg, cap)) {
    awp_srcf_destroy(s);
    return -1;
  }
  const size_t slot = (size_t)std::max(s->total, 1);
  if (cudaMalloc((void**)&s->d_ring, sizeof(float) * slot * s->ring.num_device) != cudaSuccess ||
      cudaMemset(s->d_ring, 0, sizeof(float) * slot * s->ring.num_device) != cudaSuccess ||
      cudaMallocHost((void**)&s->h_ring, sizeof(float) * slot * s->ne) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->h2d_done, cudaEventDisableTiming) != cudaSuccess) {
    awp_srcf_destroy(s);
    return failf(msg, cap, -1, "%s: ring buffer allocation failed", what);
  }
  memset(s->h_ring, 0, sizeof(float) * slot * s->ne);
  *out = s;
  return 0;
}

int awp_srcf_create(const char* path, const AwpGeom& g, float h, float dt,
                    const awp::TopoMetrics* topo, SrcFileState** out, char* msg, size_t cap) {
  return srcf_create(path, g, h, dt, topo, false, out, msg, cap);
}

int awp_forcef_create(const char* path, const AwpGeom& g, float h, float dt,
                      const awp::TopoMetrics* topo, SrcFileState** out, char* msg, size_t cap) {
  return srcf_create(path, g, h, dt, topo, true, out, msg, cap);
}

int awp_srcf_read(SrcFileState* s, long long step, cudaStream_t st, char* msg, size_t cap) {
  if (!s || s->total == 0 || step < 0) return 0;
  const size_t t = (size_t)step, T = (size_t)s->total, nd = s->ring.num_device;
  if (s->ring.host_empty(t)) {  // mpi_io_idx_read + transpose (source.c:449-466)
    if (s->h2d_pending) {       // the previous block must have reached the device
      CU_OK(cudaEventSynchronize(s->h2d_done), msg, cap);
      s->h2d_pending = false;
    }
    for (int c = 0; c < s->ncomp; ++c) {
      if (s->len[c] == 0) continue;
      std::vector<float> data((size_t)s->len[c] * s->ne);
      const int e = awp::indexed_read(s->name[c].c_str(), s->ps[c].indices, s->ne,
                                      s->ne * s->num_reads, s->reads_done, data.data());
      if (e) return setup_error(e, s->name[c].c_str(), msg, cap);
      for (size_t r = 0; r < s->ne; ++r)
        for (int i = 0; i < s->len[c]; ++i)
          s->h_ring[r * T + s->off[c] + i] = data[(size_t)i * s->ne + r];
    }
    s->reads_done++;
  }
  if (s->ring.device_empty(t)) {  // buffer_copy_to_device (buffers/buffer.c:90-96)
    const float* src = s->h_ring + s->ring.host_slot(t) * nd * T;
    CU_OK(cudaMemcpyAsync(s->d_ring, src, sizeof(float) * nd * T, cudaMemcpyHostToDevice, st),
          msg, cap);
    CU_OK(cudaEventRecord(s->h2d_done, st), msg, cap);
    s->h2d_pending = true;
  }
  return 0;
}

int awp_forcef_add(SrcFileState* s, long long step, float* const vel[3], const float* d1,
                   cudaStream_t st, long long* launches, char* msg, size_t cap) {
  if (!s || !s->force || s->ncell == 0 || step < 0) return 0;
  const size_t t = (size_t)step;
  if (!s->ring.device_ready(t)) return 0;
  ForceCellArgs a;
  for (int c = 0; c < 3; ++c) {
    a.f[c] = vel[c];
    a.qw[c] = s->qw[c];
  }
  a.d1 = d1;
  a.pos = s->d_pos;
  a.comp = s->d_comp;
  a.first = s->d_first;
  a.w = s->d_w;
  a.fdg = s->d_fdg;
  a.rho = s->d_rho;
  a.src = s->d_src;
  a.vals = s->d_ring + s->ring.device_slot(t) * (size_t)s->total;
  a.ncell = s->ncell;
  k_force_add<<<(s->ncell + 127) / 128, 128, 0, st>>>(a);
  CU_OK(cudaGetLastError(), msg, cap);
  if (launches) ++*launches;
  return 0;
}

int awp_srcf_add(SrcFileState* s, long long step, float* const stress[6], cudaStream_t st,
                 long long* launches, char* msg, size_t cap) {
  if (!s || s->force || s->ncell == 0 || step < 0) return 0;
  const size_t t = (size_t)step;
  if (!s->ring.device_ready(t)) return 0;
  SrcCellArgs a;
  for (int c = 0; c < 6; ++c) a.f[c] = stress[c];
  a.pos = s->d_pos;
  a.comp = s->d_comp;
  a.first = s->d_first;
  a.w = s->d_w;
  a.src = s->d_src;
  a.vals = s->d_ring + s->ring.device_slot(t) * (size_t)s->total;
  a.ncell = s->ncell;
  k_srcfile_add<<<(s->ncell + 127) / 128, 128, 0, st>>>(a);
  CU_OK(cudaGetLastError(), msg, cap);
  if (launches) ++*launches;
  return 0;
}
