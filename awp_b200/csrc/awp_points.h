// Point sets on the staggered grids: receivers (RECVFILE) and moment-tensor
// sources (SOURCEFILE) of the ASCII "input v2" format.
//
// Host-side restatement of the reference's set-up for these point sets:
//   readers/input.c, readers/version.c     -- the ASCII v2 reader
//   grid/grid_3d.c, grid/shift.c, topography/grids.c -- staggered coordinates
//   interpolation/interpolation.c, interpolation/lagrange.c -- Lagrange weights
//   mpi/distribute.c                        -- which points this rank owns
//   topography/sources/source.c:71-520      -- grid assignment, DM offsets,
//                                              vertical mapping, coefficients
//   buffers/buffer.c, mpi/io.c              -- ring schedule and file layout
// Every floating-point step keeps the reference's float/double rounding
// points (the host code is compiled without FMA contraction), so indices and
// weights are bit-identical to the reference's; the CPU tests pin them against
// the reference's own sources.
#pragma once

#include <stddef.h>

#include <string>
#include <vector>

namespace awp {

// Status codes of the reference's error.h that the point-set set-up reports.
enum PointErr {
  PE_OK = 0,
  PE_FILE_READ = 101,
  PE_FILE_WRITE = 102,
  PE_GET_VERSION = 200,
  PE_WRONG_VERSION = 201,
  PE_DATA_MALLOC = 304,
  PE_DATA_READ_ELEMENT = 305,
  PE_PARSE_ARG = 308,
  PE_PARSE_UNKNOWN_ARG = 309,
  PE_NOT_DIVISIBLE = 311,
  PE_LAGRANGE_LOWER = 600,
  PE_LAGRANGE_UPPER = 601,
  PE_OUT_OF_BOUNDS_LOWER = 700,
  PE_OUT_OF_BOUNDS_UPPER = 701,
  PE_NON_POSITIVE = 800,
  PE_GRID_ASSIGN = 1100,  // a point lies in no grid block (source.c:120-129 exits)
  PE_BUFFER_SIZES = 1101, // steps > 1 with a zero buffer size (the reference divides by it)
};

// Contents of an ASCII v2 input file (readers/input.h:56-72).
struct InputFile {
  int major = 0, minor = 0, patch = 0;
  std::string file = "default";
  size_t length = 0;
  size_t gpu_buffer_size = 0, cpu_buffer_size = 0;
  size_t steps = 1, num_writes = 1;
  int stride = 1, degree = 0;
  std::vector<float> x, y, z;
  std::vector<int> type;  // 0 volume coordinates, 1 surface coordinates
};

// _input_read (readers/input.c:249-290), including the version check
// (major 2), the writability check of `file` and the divisibility check of
// `steps` by the buffer sizes.  Returns a PointErr.
int read_input(const char* path, InputFile* out);

// Staggered component of a point set (topography/grids.c:45-90, grid/shift.c).
enum GridType { GT_X = 0, GT_Y, GT_Z, GT_XX, GT_YY, GT_ZZ, GT_XY, GT_XZ, GT_YZ, GT_NODE };
void grid_shift(GridType t, int shift[3]);

// One grid block of a (possibly discontinuous) mesh, top block first.
struct BlockDesc {
  int nxt, nyt, nzt;
  float h;
  int topography;  // closed top boundary (only the top block with topography)
};

// grid_fill1 (grid/grid_3d.c:258-278) for one direction of a grid with
// `size` points, the given shift and padding, at MPI coordinate 0.
void grid_fill1(float* out, int size, int shift, int padding, int boundary1, int boundary2,
                float h);

// interp_lagrange1_coef (interpolation/interpolation.c:93-130): first index
// and deg+1 Lagrange weights for query q on the nodes x[0..n).  Returns the
// reference's error bits (out-of-bounds queries are clamped and flagged).
int lagrange_coef(float* l, int* first, const float* x, int n, float q, int deg);

// Interpolation of one point set on one grid block (cu_interp_t).
struct BlockInterp {
  int num_query = 0, num_basis = 0;
  std::vector<int> ix, iy, iz, ridx;
  std::vector<float> lx, ly, lz;  // [num_query][num_basis]
};

// source_init_common (topography/sources/source.c:137-520) at one rank:
// which points lie in the domain (`indices`, into the input), their grid
// block, and the interpolation on each block.  With `topo` (the metrics of a
// curvilinear top block, blocks[0].topography = 1) the vertical coordinate of
// the top block's points is mapped to parameter space through the surface
// function interpolated at the point (source.c:283-340):
//   volume points  z' = (h (nz - 2) + z) / f(x, y),  surface points z' = h (nz - 2).
struct TopoMetrics;
struct PointSet {
  GridType type = GT_X;
  int ngrids = 0;
  std::vector<int> indices;        // input index of each owned point
  BlockInterp block[10];           // per grid block
};
int point_set_init(const InputFile& in, GridType type, const BlockDesc* blocks, int ngrids,
                   PointSet* out, const TopoMetrics* topo = nullptr);

// Ring-buffer schedule of buffers/buffer.c:44-95.
struct RingSchedule {
  size_t num_device = 1, num_host = 1, stride = 1;
  bool device_ready(size_t step) const { return step % stride == 0; }
  size_t device_slot(size_t step) const { return (step / stride) % num_device; }
  size_t host_slot(size_t step) const { return (step / stride / num_device) % num_host; }
  bool device_full(size_t step) const {
    return device_ready(step) && device_slot(step) == num_device - 1;
  }
  bool device_empty(size_t step) const { return device_ready(step) && device_slot(step) == 0; }
  bool host_full(size_t step) const { return device_full(step) && host_slot(step) == num_host - 1; }
  bool host_empty(size_t step) const { return device_empty(step) && host_slot(step) == 0; }
};

// Output file name of receiver.c:95-113: "<base>_<step>" zero-padded to
// ceil(log10(maxsteps)) + 1 digits, step rounded up to the next multiple of
// gpu*cpu*num_writes*stride.
std::string receiver_filename(const std::string& base, size_t gpu, size_t cpu, size_t num_writes,
                              int stride, size_t step, size_t maxsteps);

// mpi_io_idx_write (mpi/io.c:77-104) at one rank: writes, for owned point i,
// `ne` contiguous floats of `data` (point-major) at element
// indices[i]*ne*num_writes + write_index*ne of `path`, creating the file if
// needed and never truncating it.  Returns a PointErr.
int indexed_write(const char* path, const std::vector<int>& indices, size_t ne, size_t num_writes,
                  size_t write_index, const float* data);

// mpi_io_idx_read (mpi/io.c:106-124) at one rank for a source component:
// reads, for owned point i, `ne` floats at element indices[i]*steps + read_index*ne.
int indexed_read(const char* path, const std::vector<int>& indices, size_t ne, size_t steps,
                 size_t read_index, float* data);

}  // namespace awp

namespace awp {

// Per-cell contributions of a SOURCEFILE component (cusource_add_cartesian,
// topography/sources/source.cu:24-49): every (query, i, j, k) adds
// w * value(query) to cell pos with w = ((-dt/h^3 * lx) * ly) * lz in float.
// Contributions are grouped by cell, in query order, so one thread applies
// a cell's sources in the order the reference's threads would (the reference
// lets threads of overlapping sources race on a cell).
struct CellAdds {
  std::vector<long long> cell_pos;   // padded linear index of each cell
  std::vector<int> first;            // [ncell + 1] offsets into w / src
  std::vector<float> w;
  std::vector<int> src;              // owned-point index of each contribution
};
void source_cell_adds(const BlockInterp& bi, float dt, float h, int slice, int yline,
                      CellAdds* out);

}  // namespace awp
