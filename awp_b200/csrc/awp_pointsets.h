// Receivers (RECVFILE) and SOURCEFILE sources of a context: device tables,
// ring buffers and the per-step hooks of the time loop.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "awp_common.h"

struct RecvState;
struct SrcFileState;
namespace awp {
struct TopoMetrics;
}

// receivers_init (topography/receivers/receivers.c:22-42) for one grid block
// (`topo`: the metrics when the block is curvilinear, else null).
// Returns a PointErr-coded or CUDA status through `status`; message in `msg`.
int awp_recv_create(const char* path, long long nt, const AwpGeom& g, float h,
                    const awp::TopoMetrics* topo, RecvState** out, char* msg, size_t msgcap);
// receivers_write (receivers.c:52-77) at `step` from the grid's velocities.
int awp_recv_record(RecvState* r, long long step, const float* u, const float* v,
                    const float* w, cudaStream_t st, long long* launches, char* msg,
                    size_t msgcap);
void awp_recv_destroy(RecvState* r);
int awp_recv_length(const RecvState* r, int comp);
// The file name stem of component `comp` (<file>_<name>).
std::string awp_recv_base(const RecvState* r, int comp);
// sgt_init (topography/receivers/sgt.c:29-58) for one grid block: receivers
// of the six stresses (files <file>_Gxx ... _Gyz) and the one-shot material
// recorder on the node grid (`mat`).
int awp_sgt_create(const char* path, long long nt, const AwpGeom& g, float h,
                   const awp::TopoMetrics* topo, RecvState** out, RecvState** mat, char* msg,
                   size_t msgcap);
// receiver_write of every component of `r` at `step` from fields[component].
int awp_recv_record_fields(RecvState* r, long long step, const float* const* fields,
                           cudaStream_t st, long long* launches, char* msg, size_t msgcap);
// One unbuffered write of a one-component recorder at step 0 into `filename`
// (sgt_write_material_properties, sgt.c:70-90).
int awp_recv_write_once(RecvState* r, const float* field, const char* filename, cudaStream_t st,
                        long long* launches, char* msg, size_t msgcap);

// sources_init (topography/sources/sources.c:27-50) for one grid block.
int awp_srcf_create(const char* path, const AwpGeom& g, float h, float dt,
                    const awp::TopoMetrics* topo, SrcFileState** out, char* msg, size_t msgcap);
// sources_read (sources.c:52-63) at `step`.
int awp_srcf_read(SrcFileState* s, long long step, cudaStream_t st, char* msg, size_t msgcap);
// sources_add_cartesian (sources.c:65-78) at `step`; stress = xx yy zz xy xz yz.
int awp_srcf_add(SrcFileState* s, long long step, float* const stress[6], cudaStream_t st,
                 long long* launches, char* msg, size_t msgcap);
void awp_srcf_destroy(SrcFileState* s);
// forces_init (topography/sources/forces.c:24-50) on the curvilinear top block:
// fx, fy, fz on the velocity grids, every point a boundary point (type 1).
// Read with awp_srcf_read (forces_read), added with awp_forcef_add.
int awp_forcef_create(const char* path, const AwpGeom& g, float h, float dt,
                      const awp::TopoMetrics* topo, SrcFileState** out, char* msg, size_t msgcap);
// forces_add (forces.c:67-96) at `step`: vel = u1 v1 w1, d1 the density.
int awp_forcef_add(SrcFileState* s, long long step, float* const vel[3], const float* d1,
                   cudaStream_t st, long long* launches, char* msg, size_t msgcap);
