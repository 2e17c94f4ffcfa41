// Point sets on the staggered grids (receivers and SOURCEFILE sources).
// See awp_points.h for the reference routines each function restates.
#include "awp_points.h"

#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>

#include "awp_common.h"
#include "awp_topo.h"

namespace awp {

namespace {

constexpr double kFltol = 1e-5;          // FLTOL (awp/definitions.h:43)
constexpr double kSourceOffsetX = -0.5;  // SOURCE_OFFSET_X (sources/source.h:25)
constexpr int kDmOffsetX = 0;            // SOURCE_DM_OFFSET_X (sources/source.h:19)
constexpr int kDmOffsetY = -1;           // SOURCE_DM_OFFSET_Y (sources/source.h:20)
constexpr double kOverlap = 7.0;         // OVERLAP (sources/source.c:19)

// input_parse / input_parse_arg (readers/input.c:126-190)
int parse_line(InputFile* out, const char* line) {
  std::string s(line);
  std::vector<char> buf(s.begin(), s.end());
  buf.push_back('\0');
  char* save = nullptr;
  char* var = strtok_r(buf.data(), "=", &save);
  if (!var) return PE_PARSE_ARG;
  char* val = strtok_r(nullptr, "=", &save);
  if (!val) return PE_PARSE_ARG;
  if (!strcmp(var, "file")) out->file = val;
  else if (!strcmp(var, "length")) out->length = (size_t)atof(val);
  else if (!strcmp(var, "stride")) out->stride = (int)(size_t)atof(val);
  else if (!strcmp(var, "steps")) out->steps = (size_t)atof(val);
  else if (!strcmp(var, "num_writes")) out->num_writes = (size_t)atof(val);
  else if (!strcmp(var, "degree")) out->degree = atoi(val);
  else if (!strcmp(var, "gpu_buffer_size")) out->gpu_buffer_size = (size_t)atoi(val);
  else if (!strcmp(var, "cpu_buffer_size")) out->cpu_buffer_size = (size_t)atoi(val);
  else {
    fprintf(stderr, "Unknown argument: %s \n", var);
    return PE_PARSE_UNKNOWN_ARG;
  }
  return PE_OK;
}

// input_file_writeable (readers/input.c:108-124): an existing file, or one
// that can be created (and is removed again).
int file_writeable(const char* path) {
  FILE* fh = fopen(path, "r");
  if (fh) {
    fclose(fh);
    return PE_OK;
  }
  fh = fopen(path, "w");
  if (!fh) return PE_FILE_WRITE;
  fclose(fh);
  remove(path);
  return PE_OK;
}

// interp_argnearest (interpolation/interpolation.c:14-38)
int argnearest(int* nearest, const float* points, int n, float query) {
  if (query < points[0]) {
    *nearest = 0;
    return PE_OUT_OF_BOUNDS_LOWER;
  }
  if (query > points[n - 1]) {
    *nearest = n - 1;
    return PE_OUT_OF_BOUNDS_UPPER;
  }
  int argmin = n + 1;
  float dist = INFINITY;
  for (int i = 0; i < n; ++i) {
    const float d = (float)fabs((double)(query - points[i]));
    if (d < dist) {
      dist = d;
      argmin = i;
    }
  }
  *nearest = argmin;
  return PE_OK;
}

// lagrange_node_poly (interpolation/lagrange.c:66-74)
double node_poly(float x0, const float* x, int n) {
  double l = 1.0;
  for (int i = 0; i < n; ++i) l *= (double)(x0 - x[i]);
  return l;
}

// lagrange_basis (interpolation/lagrange.c:20-52)
int lagrange_basis(float* l, int n, const float* x, float x0) {
  if (n == 1) {
    l[0] = 1.0f;
    return PE_OK;
  }
  if ((double)(x0 - x[0]) < -kFltol) return PE_LAGRANGE_LOWER;
  if ((double)(x0 - x[n - 1]) > kFltol) return PE_LAGRANGE_UPPER;
  const double L = node_poly(x0, x, n);
  for (int j = 0; j < n; ++j) {
    l[j] = 1.0f;
    if (fabs((double)(x0 - x[j])) < kFltol) continue;
    double denom = 1.0;
    for (int k = 0; k < n; ++k) {
      if (j == k) continue;
      denom *= (double)(x[j] - x[k]);
    }
    const double lambda = 1.0 / denom;
    l[j] = (float)((double)(float)L * lambda / (double)(x0 - x[j]));
  }
  return PE_OK;
}

struct CompGrid {  // one staggered component grid of one block (grid3_t subset)
  int size[3];     // points per direction (padding included in x, y)
  int shift[3];
  int padding;
  int b2z;         // closed top boundary
  float h;
};

CompGrid comp_grid(const BlockDesc& b, GridType t, int padding) {
  CompGrid g;
  grid_shift(t, g.shift);
  g.padding = padding;
  g.size[0] = b.nxt + 2 * padding;
  g.size[1] = b.nyt + 2 * padding;
  g.size[2] = b.nzt;
  g.b2z = b.topography;
  g.h = b.h;
  return g;
}

void fill_dir(std::vector<float>& out, const CompGrid& g, int d) {
  out.resize(g.size[d]);
  grid_fill1(out.data(), g.size[d], g.shift[d], d < 2 ? g.padding : 0, 0, d == 2 ? g.b2z : 0,
             g.h);
}

// grid_in_bounds_ext1 (grid/grid_3d.c:301-311)
bool in_bounds_ext(const std::vector<float>& x, float q, float h) {
  const float hh = h / 2;
  if (q - (x[0] - hh) < 0) return false;
  if (q - (x[x.size() - 1] + hh) >= 0) return false;
  return true;
}

// source_find_grid_number (topography/sources/source.c:71-130)
int find_grid_numbers(const InputFile& in, const BlockDesc* blocks, int ngrids,
                      const std::vector<int>& idx, std::vector<int>& gn) {
  gn.assign(idx.size(), -1);
  float lower = 0.f, upper = 0.f, overlap = 0.f;
  for (int i = 0; i < ngrids; ++i) {
    // velocity grid of the w component (grids.z): shift (0, 1, 0), no padding
    CompGrid g = comp_grid(blocks[i], GT_Z, 0);
    std::vector<float> z1;
    fill_dir(z1, g, 2);
    const int end = g.size[2] - 1 - g.b2z;
    upper = lower;
    lower = lower - z1[end];
    for (size_t j = 0; j < idx.size(); ++j) {
      const float z = in.z[idx[j]];
      if (in.type[idx[j]] == 1) {
        gn[j] = 0;
        continue;
      } else if (z > 0) {
        gn[j] = 0;
      } else if (z > lower && z <= upper - overlap) {
        gn[j] = i;
      }
    }
    overlap = (i + 1 != ngrids) ? (float)((double)g.h * kOverlap) : 0.0f;
    lower = lower + overlap;
  }
  for (size_t j = 0; j < idx.size(); ++j)
    if (gn[j] == -1) {
      fprintf(stderr, "Failed to assign source/receiver id=%zu  to a grid.\n", j);
      return PE_GRID_ASSIGN;
    }
  return PE_OK;
}

// padding of the component grids of grids_init (topography/grids.c:24-37)
// topography/grids.c:26-40: velocity and material grids without padding,
// stress grids with ngsl / 2
int component_padding(GridType t) { return (t <= GT_Z || t == GT_NODE) ? 0 : AWP_NGSL / 2; }

}  // namespace

int read_input(const char* path, InputFile* out) {
  *out = InputFile();
  FILE* fp = fopen(path, "r");
  if (!fp) return PE_FILE_READ;
  char vs[1024];
  if (!fgets(vs, sizeof(vs), fp)) {
    fclose(fp);
    return PE_GET_VERSION;
  }
  {  // version_init (readers/version.c:8-19)
    char* save = nullptr;
    char* t = strtok_r(vs, ".", &save);
    if (t) out->major = atoi(t);
    t = strtok_r(nullptr, ".", &save);
    if (t) out->minor = atoi(t);
    t = strtok_r(nullptr, ".", &save);
    if (t) out->patch = atoi(t);
  }
  if (out->major != 2) {  // version_check_compatibility: same major as 2.1.0
    fclose(fp);
    return PE_WRONG_VERSION;
  }
  int parse_arg = PE_OK;
  int match = 1;
  char line[2048];
  line[0] = '\0';
  while (parse_arg == PE_OK && match == 1) {
    match = fscanf(fp, "#%2047[^\n]", line);
    if (match) {  // a comment line (or the end of the file)
      getc(fp);
      continue;
    }
    match = fscanf(fp, "%2047s\n", line);
    if (match != 1) break;
    if (!strcmp(line, "coordinates")) break;
    parse_arg = parse_line(out, line);
  }
  int err = file_writeable(out->file.c_str());
  if (!err) err = parse_arg;
  if (!err && out->steps > 1) {  // input_check_header (readers/input.c:318-329)
    const size_t bs = out->gpu_buffer_size * out->cpu_buffer_size;
    if (bs == 0) err = PE_BUFFER_SIZES;
    else if (out->steps % bs != 0) err = PE_NOT_DIVISIBLE;
  }
  if (!err) {
    out->x.resize(out->length);
    out->y.resize(out->length);
    out->z.resize(out->length);
    out->type.resize(out->length);
    for (size_t id = 0; id < out->length; ++id) {  // _read_data (readers/input.c:346-366)
      float x, y, z;
      int type;
      if (fscanf(fp, "%d %g %g %g\n", &type, &x, &y, &z) != 4) {
        err = PE_DATA_READ_ELEMENT;
        break;
      }
      out->x[id] = x;
      out->y[id] = y;
      out->z[id] = z;
      out->type[id] = type;
    }
  }
  fclose(fp);
  return err;
}

void grid_shift(GridType t, int s[3]) {
  // grid/shift.c:76-151: u1 (1,1,1), u2 (0,0,1), u3 (0,1,0), normal stresses
  // (0,1,1), xy (1,0,1), xz (1,1,0), yz (0,0,0), material node (1,0,0)
  static const int tab[10][3] = {{1, 1, 1}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1}, {0, 1, 1},
                                 {0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {0, 0, 0}, {1, 0, 0}};
  s[0] = tab[t][0];
  s[1] = tab[t][1];
  s[2] = tab[t][2];
}

void grid_fill1(float* out, int size, int shift, int padding, int boundary1, int boundary2,
                float h) {
  for (int i = 0; i < size; ++i)
    out[i] = (float)((double)h * (((double)i - 0.5 * (double)shift) - (double)padding));
  if (shift && boundary1) out[0] = h * 0 * size;
  if (shift && boundary2) out[size - 1] = h * ((size - 2 * padding) - 2 - padding);
  if (!shift && boundary2) out[size - 1] = 0.0f;
}

int lagrange_coef(float* l, int* first, const float* x, int n, float query, int deg) {
  int err = 0, nearest = 0;
  int lower = (int)ceil((double)deg * 0.5);
  int upper = (int)ceil((double)deg * 0.5);
  float q = query;
  err = argnearest(&nearest, x, n, query);
  if (err == PE_OUT_OF_BOUNDS_LOWER) q = x[0];
  if (err == PE_OUT_OF_BOUNDS_UPPER) q = x[n - 1];
  if (deg % 2 == 1) {
    if (x[nearest] - query > 0) {
      lower = (int)ceil((double)deg * 0.5);
      upper = (int)floor((double)deg * 0.5);
    } else {
      lower = (int)floor((double)deg * 0.5);
      upper = (int)ceil((double)deg * 0.5);
    }
  }
  // interp_argnearest_range (interpolation.c:49-63)
  const int diffleft = nearest - lower;
  const int diffright = n - nearest - upper - 1;
  const int ileft = std::max(diffleft, 0) + std::min(diffright, 0);
  *first = ileft;
  std::vector<float> xloc(deg + 1);
  for (int j = 0; j < deg + 1; ++j) xloc[j] = x[ileft + j];
  err |= lagrange_basis(l, deg + 1, xloc.data(), q);
  return err;
}

int point_set_init(const InputFile& in, GridType type, const BlockDesc* blocks, int ngrids,
                   PointSet* out, const TopoMetrics* topo) {
  *out = PointSet();
  out->type = type;
  out->ngrids = ngrids;
  if (ngrids < 1 || ngrids > 10) return PE_NON_POSITIVE;
  const size_t n = in.length;
  std::vector<int> all(n);
  for (size_t i = 0; i < n; ++i) all[i] = (int)i;
  std::vector<int> gn;
  int err = find_grid_numbers(in, blocks, ngrids, all, gn);
  if (err) return err;

  // DM offsets of source_init_common (source.c:155-176)
  const int pad = component_padding(type);
  std::vector<CompGrid> cg(ngrids);
  for (int j = 0; j < ngrids; ++j) cg[j] = comp_grid(blocks[j], type, pad);
  std::vector<float> dmx(ngrids, 0.f), dmy(ngrids, 0.f), dmz(ngrids, 0.f);
  for (int j = 1; j < ngrids; ++j) {
    const CompGrid &pre = cg[j - 1], &cur = cg[j];
    const float ax = dmx[j - 1] + kDmOffsetX * pre.h;
    dmx[j] = (float)((double)ax - ((double)cur.shift[0] * 0.5 * (double)cur.h -
                                   (double)pre.shift[0] * 0.5 * (double)pre.h));
    const float ay = dmy[j - 1] + kDmOffsetY * pre.h;
    dmy[j] = (float)((double)ay - ((double)cur.shift[1] * 0.5 * (double)cur.h -
                                   (double)pre.shift[1] * 0.5 * (double)pre.h));
    dmz[j] = (float)((double)cg[0].shift[2] * 0.5 * (double)cg[0].h -
                     (double)cur.shift[2] * 0.5 * (double)cur.h);
  }
  std::vector<float> x(n), y(n), z(n);
  for (size_t i = 0; i < n; ++i) {
    x[i] = (float)((double)in.x[i] + kSourceOffsetX * (double)cg[0].h);
    y[i] = in.y[i];
    z[i] = in.z[i];
    x[i] = x[i] + dmx[gn[i]];
    y[i] = y[i] + dmy[gn[i]];
    z[i] = z[i] + dmz[gn[i]];
  }

  // dist_indices (mpi/distribute.c:9-52) on the component grid of the top block
  {
    std::vector<float> gx, gy;
    fill_dir(gx, cg[0], 0);
    fill_dir(gy, cg[0], 1);
    for (size_t i = 0; i < n; ++i)
      if (in_bounds_ext(gx, x[i], cg[0].h) && in_bounds_ext(gy, y[i], cg[0].h))
        out->indices.push_back((int)i);
  }
  const size_t len = out->indices.size();
  if (len == 0) return PE_OK;
  std::vector<int> gown;
  err = find_grid_numbers(in, blocks, ngrids, out->indices, gown);
  if (err) return err;

  float overlap = 0.f, lower = 0.f;
  for (int j = 0; j < ngrids; ++j) {
    const CompGrid& g = cg[j];
    const bool curv = topo != nullptr && j == 0;
    // the curvilinear block's height excludes its ghost point (source.c:268-273)
    const float block_height = g.h * (g.size[2] - (curv ? 2 : 1));
    lower = lower - block_height + overlap;
    std::vector<float> qx, qy, qz;
    std::vector<int> ridx;
    for (size_t i = 0; i < len; ++i) {
      if (gown[i] != j) continue;
      const int src = out->indices[i];
      ridx.push_back((int)i);
      qx.push_back(x[src]);
      qy.push_back(y[src]);
      qz.push_back(z[src]);
    }
    if (curv && !ridx.empty()) {
      // metrics_interpolate_f_point (metrics/metrics.c:171-204) on the
      // topography grid with ngsl padding -- grid_node(), shift (1, 0, 0)
      // (grid/shift.c:76-80) -- then the map to parameter space
      CompGrid mg = comp_grid(blocks[0], GT_YZ, AWP_NGSL);
      mg.shift[0] = 1;
      std::vector<float> mx, my, mz;
      fill_dir(mx, mg, 0);
      fill_dir(my, mg, 1);
      fill_dir(mz, mg, 2);
      const int nb = in.degree + 1;
      std::vector<float> lx(nb), ly(nb);
      for (size_t q = 0; q < ridx.size(); ++q) {
        int ix = 0, iy = 0;
        lagrange_coef(lx.data(), &ix, mx.data(), mg.size[0], qx[q], in.degree);
        lagrange_coef(ly.data(), &iy, my.data(), mg.size[1], qy[q], in.degree);
        float fq = 0.0f;
        for (int a = 0; a < nb; ++a)
          for (int b = 0; b < nb; ++b)
            fq += lx[a] * ly[b] * topo->f[(size_t)topo->fidx(ix + a - AWP_NGSL, iy + b - AWP_NGSL)];
        const int src = out->indices[ridx[q]];
        if (in.type[src] == 0)
          qz[q] = (block_height + qz[q]) / fq;
        else if (in.type[src] == 1)
          qz[q] = mz[mg.size[2] - 2];
      }
    } else {
      for (size_t q = 0; q < ridx.size(); ++q) {
        const int src = out->indices[ridx[q]];
        if (in.type[src] == 1)
          qz[q] = block_height;  // surface coordinates (only in the top block)
        else if (in.type[src] == 0)
          qz[q] = qz[q] - lower;
      }
    }
    overlap = (float)((double)g.h * kOverlap);
    if (ridx.empty()) continue;
    // interpolation on the full (metric) grid: padding ngsl in x and y
    CompGrid full = comp_grid(blocks[j], type, AWP_NGSL);
    std::vector<float> fx, fy, fz;
    fill_dir(fx, full, 0);
    fill_dir(fy, full, 1);
    fill_dir(fz, full, 2);
    const int nbx = full.size[0] - ((full.shift[0] == 0 && 0) ? 1 : 0);
    const int nby = full.size[1] - ((full.shift[1] == 0 && 0) ? 1 : 0);
    const int nbz = full.size[2] - ((full.shift[2] == 0 && full.b2z == 1) ? 1 : 0);
    BlockInterp& bi = out->block[j];
    const int nb = in.degree + 1;
    bi.num_query = (int)ridx.size();
    bi.num_basis = nb;
    bi.ridx = ridx;
    bi.ix.assign(bi.num_query, 0);
    bi.iy.assign(bi.num_query, 0);
    bi.iz.assign(bi.num_query, 0);
    bi.lx.assign((size_t)bi.num_query * nb, 0.f);
    bi.ly.assign((size_t)bi.num_query * nb, 0.f);
    bi.lz.assign((size_t)bi.num_query * nb, 0.f);
    int cerr = 0;
    for (int q = 0; q < bi.num_query; ++q) {  // cuinterp_lagrange_h (interpolation.cu:42-64)
      cerr = lagrange_coef(&bi.lx[(size_t)q * nb], &bi.ix[q], fx.data(), nbx, qx[q], in.degree);
      cerr = lagrange_coef(&bi.ly[(size_t)q * nb], &bi.iy[q], fy.data(), nby, qy[q], in.degree);
      cerr = lagrange_coef(&bi.lz[(size_t)q * nb], &bi.iz[q], fz.data(), nbz, qz[q], in.degree);
    }
    // the reference checks only the status of the last query's z weights
    if (cerr) return cerr;
    if (ngrids > 1) {  // overlap-zone clamps (source.c:384-420)
      for (int q = 0; q < bi.num_query; ++q) {
        int& iz = bi.iz[q];
        if (j == 0) {
          if (iz < 2) iz = 2;
        } else if (j != ngrids - 1) {
          if (iz < 2) iz = 2;
          else if (iz > g.size[2] - 3) iz = g.size[2] - 3;
        } else {
          if (iz > g.size[2] - 3) iz = g.size[2] - 3;
        }
      }
    }
  }
  return PE_OK;
}

std::string receiver_filename(const std::string& base, size_t gpu, size_t cpu, size_t num_writes,
                              int stride, size_t step, size_t maxsteps) {
  const size_t unit = gpu * cpu * num_writes * (size_t)stride;
  const size_t filestep = (1 + step / unit) * unit;
  const int zeros = (int)ceil(log10((double)maxsteps)) + 1;
  char buf[4096];
  snprintf(buf, sizeof(buf), "%s_%0*ld", base.c_str(), zeros, (long)filestep);
  return buf;
}

int indexed_write(const char* path, const std::vector<int>& indices, size_t ne, size_t num_writes,
                  size_t write_index, const float* data) {
  const int fd = open(path, O_WRONLY | O_CREAT, 0644);
  if (fd < 0) return PE_FILE_WRITE;
  int err = PE_OK;
  for (size_t i = 0; i < indices.size() && !err; ++i) {
    const off_t off =
        (off_t)sizeof(float) * ((off_t)indices[i] * ne * num_writes + (off_t)write_index * ne);
    const size_t bytes = ne * sizeof(float);
    if (pwrite(fd, data + i * ne, bytes, off) != (ssize_t)bytes) err = PE_FILE_WRITE;
  }
  if (close(fd) != 0) err = PE_FILE_WRITE;
  return err;
}

int indexed_read(const char* path, const std::vector<int>& indices, size_t ne, size_t steps,
                 size_t read_index, float* data) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return PE_FILE_READ;
  int err = PE_OK;
  for (size_t i = 0; i < indices.size() && !err; ++i) {
    const off_t off =
        (off_t)sizeof(float) * ((off_t)indices[i] * steps + (off_t)read_index * ne);
    const size_t bytes = ne * sizeof(float);
    if (pread(fd, data + i * ne, bytes, off) != (ssize_t)bytes) err = PE_FILE_READ;
  }
  close(fd);
  return err;
}

}  // namespace awp

namespace awp {

void source_cell_adds(const BlockInterp& bi, float dt, float h, int slice, int yline,
                      CellAdds* out) {
  *out = CellAdds();
  const float dth = dt / (h * h * h);
  const int nb = bi.num_basis;
  struct C {
    long long pos;
    int order;
    float w;
    int src;
  };
  std::vector<C> all;
  all.reserve((size_t)bi.num_query * nb * nb * nb);
  int order = 0;
  for (int q = 0; q < bi.num_query; ++q)
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        for (int k = 0; k < nb; ++k) {
          // grid_index of the metric grid: offsets (2, 2, align) (grid/grid_3d.h:113)
          const long long pos = (long long)(2 + bi.ix[q] + i) * slice +
                                (long long)(2 + bi.iy[q] + j) * yline + (AWP_ALIGN + bi.iz[q] + k);
          const float w = ((-dth * bi.lx[(size_t)q * nb + i]) * bi.ly[(size_t)q * nb + j]) *
                          bi.lz[(size_t)q * nb + k];
          all.push_back({pos, order++, w, bi.ridx[q]});
        }
  std::stable_sort(all.begin(), all.end(), [](const C& a, const C& b) { return a.pos < b.pos; });
  for (size_t n = 0; n < all.size(); ++n) {
    if (n == 0 || all[n].pos != all[n - 1].pos) {
      out->cell_pos.push_back(all[n].pos);
      out->first.push_back((int)n);
    }
    out->w.push_back(all[n].w);
    out->src.push_back(all[n].src);
  }
  out->first.push_back((int)all.size());
}

}  // namespace awp
