// Receivers (RECVFILE) and SOURCEFILE sources of a context: device tables,
// ring buffers and the per-step hooks of the time loop.
#pragma once

#include <cuda_runtime.h>

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

// sources_init (topography/sources/sources.c:27-50) for one grid block.
int awp_srcf_create(const char* path, const AwpGeom& g, float h, float dt,
                    const awp::TopoMetrics* topo, SrcFileState** out, char* msg, size_t msgcap);
// sources_read (sources.c:52-63) at `step`.
int awp_srcf_read(SrcFileState* s, long long step, cudaStream_t st, char* msg, size_t msgcap);
// sources_add_cartesian (sources.c:65-78) at `step`; stress = xx yy zz xy xz yz.
int awp_srcf_add(SrcFileState* s, long long step, float* const stress[6], cudaStream_t st,
                 long long* launches, char* msg, size_t msgcap);
void awp_srcf_destroy(SrcFileState* s);
