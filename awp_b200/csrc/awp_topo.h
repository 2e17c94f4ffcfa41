// Curvilinear topography: host-side set-up of the metric arrays.
//
// Restates, for one rank:
//   topography/readers/serial_reader.c:9-62   -- the topography file reader
//   topography/geometry/geometry.c:33-43, 188-210 -- geom_no_grid_stretching, geom_custom
//   topography/metrics/metrics.c:14-37, 141-167, 194-305 and metrics/kernel.c
//                                              -- f and g interpolation / differentiation
// with the reference's float/double rounding points (the host code is
// compiled without FMA contraction), so the arrays are bit-identical to the
// reference's (pinned by the CPU tests against the reference's own code).
//
// Layouts (relative indices: i, j = 0 the first interior cell, k = 0 the
// bottom cell of the grid):
//   2-D f arrays: (nx + 4 + 2*ngsl) x (ny + 4 + 2*ngsl + 2*align), element
//     (i, j) at (i + ngsl + 2) * ld + (j + ngsl + 2 + align), ld the second extent;
//   1-D g arrays: nz + 2*align, element k at k + align.
#pragma once

#include <vector>

namespace awp {

struct TopoMetrics {
  int nx = 0, ny = 0, nz = 0;
  int ld = 0;  // second extent of the f arrays
  float h = 0.f;
  // f (the surface function), its interpolants to the staggered positions
  // (f_1, f_2, f_c) and derivatives (f1_* in x, f2_* in y)
  std::vector<float> f, f_1, f_2, f_c, f1_1, f1_2, f1_c, f2_1, f2_2, f2_c;
  // g (vertical coordinate), interpolant g_c and derivatives g3, g3_c
  std::vector<float> g, g_c, g3, g3_c;
  long long fidx(int i, int j) const;  // index of relative (i, j) in an f array
};

// topo_read_serial: reads int32 gnx, gny, padding and float32
// data[gnx + 2 padding][gny + 2 padding] (y fastest); the first
// nx + 2*ngsl rows and columns land in f at relative -ngsl...  Returns 0,
// 101 (unreadable) or 902 (sizes inconsistent with nx, ny, or padding < ngsl).
int topo_read_file(const char* path, int nx, int ny, std::vector<float>* f);

// The whole set-up of topo_init_metrics / topo_init_geometry / topo_build
// from the raw elevation (as the file holds it, already in `f`): geom_custom,
// the unstretched g and every interpolant and derivative.
void topo_build_metrics(TopoMetrics* m);

// Allocate the arrays of an nx x ny x nz grid with spacing h (f zero).
void topo_init_metrics(TopoMetrics* m, int nx, int ny, int nz, float h);

}  // namespace awp
