// TMA-pipelined stencil kernels (awp_tma.cu): tensor maps and launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "awp_common.h"
#include "awp_kernels.cuh"

// Tensor maps of the fields one kernel streams, grouped by tile shape:
//   halo  (40 x 12 box): fields read with their j/k neighbours
//   media (36 x  9 box): fields read at (j|j-1, k|k-1) of planes i and i+1
//   own   (32 x  8 box): fields read and written at the cell itself
// velocity kernel: halo = xx (own box), yy, xy (32 x 12: j halo), zz, xz
//                  (40 x 8: k halo), yz (40 x 12); media = d1; own = u1 v1 w1
// stress kernel  : halo = u1 v1 w1, media = lam mu qp qs, own = xx..yz r1..r6
struct TmaMaps {
  CUtensorMap halo[6];
  CUtensorMap media[4];
  CUtensorMap own[12];
};

// Encode one 3-D tensor map over a padded field; box groups: 0 halo (40 x 12),
// 1 media (36 x 9), 2 own (32 x 8), 3 j halo (32 x 12), 4 k halo (40 x 8).
int awp_tma_box(int group, int* box_x, int* box_y);
int awp_tma_encode(CUtensorMap* map, const float* base, const AwpGeom& g, int box_x, int box_y);

cudaError_t awp_launch_stress_tma(const StrArgs& a, const TmaMaps& tm, bool elastic, int ichunk,
                                  int* err, cudaStream_t st);
cudaError_t awp_launch_velocity_tma(const VelArgs& a, const TmaMaps& tm, int ichunk, int* err,
                                    cudaStream_t st);
// Poll limit of the TMA kernels' pipeline waits (0 .. 2^30; default 2^26; 0
// makes every wait give up at once, which exercises the failure path).  A wait
// that runs out sets the context's error word; the CTA then drains its issued
// copies with the default limit and leaves.  Returns 0 or 1 (refused).
int awp_tma_set_spin_limit(long long polls);
long long awp_tma_get_spin_limit();
// L2 promotion of the TMA fetches for tensor maps encoded from now on (0 none,
// 1 64 B, 2 128 B, 3 256 B, the default).  Returns 0 or 1 (refused).
int awp_tma_set_l2_promotion(int mode);
int awp_tma_get_l2_promotion();
