// Curvilinear topography: metric arrays (see awp_topo.h for the reference
// routines restated here).
#include "awp_topo.h"

#include <stdio.h>

#include "awp_common.h"
#include "awp_points.h"
#include "awp_topo_tables.h"

namespace awp {

namespace {

// 4th-order staggered interpolation and difference (the interior stencils of
// the generated metric kernels, metrics/kernel.c): (-1, 9, 9, -1)/16 and
// (1, -27, 27, -1)/24 as the reference's double literals converted to float.
constexpr float kP4[4] = {-0.0625, 0.5625, 0.5625, -0.0625};
constexpr float kD4[4] = {0.0416666666666667, -1.1250000000000000, 1.1250000000000000,
                          -0.0416666666666667};

}  // namespace

long long TopoMetrics::fidx(int i, int j) const {
  return (long long)(i + AWP_NGSL + 2) * ld + (j + AWP_NGSL + 2 + AWP_ALIGN);
}

void topo_init_metrics(TopoMetrics* m, int nx, int ny, int nz, float h) {
  m->nx = nx;
  m->ny = ny;
  m->nz = nz;
  m->h = h;
  m->ld = ny + 4 + 2 * AWP_NGSL + 2 * AWP_ALIGN;
  const size_t nf = (size_t)(nx + 4 + 2 * AWP_NGSL) * m->ld;
  for (auto* v : {&m->f, &m->f_1, &m->f_2, &m->f_c, &m->f1_1, &m->f1_2, &m->f1_c, &m->f2_1,
                  &m->f2_2, &m->f2_c})
    v->assign(nf, 0.f);
  const size_t ng = (size_t)nz + 2 * AWP_ALIGN;
  for (auto* v : {&m->g, &m->g_c, &m->g3, &m->g3_c}) v->assign(ng, 0.f);
}

int topo_read_file(const char* path, int nx, int ny, std::vector<float>* f) {
  FILE* fh = fopen(path, "rb");
  if (!fh) return PE_FILE_READ;
  int hdr[3];
  if (fread(hdr, sizeof(int), 3, fh) != 3) {
    fclose(fh);
    return PE_FILE_READ;
  }
  const int gnx = hdr[0], gny = hdr[1], padding = hdr[2];
  if (nx != gnx || ny != gny || padding < AWP_NGSL) {
    fclose(fh);
    return 902;  // ERR_INCONSISTENT_SIZE
  }
  const long long gmx = gnx + 2LL * padding, gmy = gny + 2LL * padding;
  std::vector<float> data((size_t)(gmx * gmy));
  const size_t got = fread(data.data(), sizeof(float), data.size(), fh);
  fclose(fh);
  if (got != data.size()) return PE_FILE_READ;
  const long long lmy = 4 + ny + 2 * AWP_NGSL + 2 * AWP_ALIGN;
  for (int i = 0; i < nx + 2 * AWP_NGSL; ++i)
    for (int j = 0; j < ny + 2 * AWP_NGSL; ++j)
      (*f)[(size_t)(2 + AWP_ALIGN + j + (2 + i) * lmy)] = data[(size_t)(j + i * gmy)];
  return 0;
}

void topo_build_metrics(TopoMetrics* m) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  const float h = m->h;
  // geom_custom (geometry.c:188-210): f = 1 + f / (h (nz - 2)) over the
  // topography window (nx + 2 ngsl) x (ny + 2 ngsl) from relative -ngsl
  {
    const float normalize = (float)(1.0 / (double)h / (double)(nz - 2));
    for (int i = -AWP_NGSL; i < nx + AWP_NGSL; ++i)
      for (int j = -AWP_NGSL; j < ny + AWP_NGSL; ++j) {
        float& v = m->f[(size_t)m->fidx(i, j)];
        v = (float)(1.0 + (double)(v * normalize));
      }
  }
  // f interpolants and derivatives (metrics_interpolate_f /
  // metrics_differentiate_f), each over relative [-ngsl + 2, n + ngsl - 2)
  const float hi = (float)(1.0 / (double)h);
  auto F = [&](std::vector<float>& a, int i, int j) -> float& { return a[(size_t)m->fidx(i, j)]; };
  const int i0 = -AWP_NGSL + 2, i1 = nx + AWP_NGSL - 2, j0 = -AWP_NGSL + 2,
            j1 = ny + AWP_NGSL - 2;
  for (int j = j0; j < j1; ++j)
    for (int i = i0; i < i1; ++i) {
      F(m->f_1, i, j) = kP4[0] * F(m->f, i, j - 2) + kP4[1] * F(m->f, i, j - 1) +
                        kP4[2] * F(m->f, i, j) + kP4[3] * F(m->f, i, j + 1);
      F(m->f_2, i, j) = kP4[0] * F(m->f, i - 1, j) + kP4[1] * F(m->f, i, j) +
                        kP4[2] * F(m->f, i + 1, j) + kP4[3] * F(m->f, i + 2, j);
      auto row = [&](int jj) {
        return kP4[0] * F(m->f, i - 1, jj) + kP4[1] * F(m->f, i, jj) +
               kP4[2] * F(m->f, i + 1, jj) + kP4[3] * F(m->f, i + 2, jj);
      };
      F(m->f_c, i, j) =
          kP4[0] * row(j - 2) + kP4[1] * row(j - 1) + kP4[2] * row(j) + kP4[3] * row(j + 1);
    }
  auto dx_h = [&](std::vector<float>& out, std::vector<float>& in) {  // to the half point
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i)
        F(out, i, j) = hi * (kD4[0] * F(in, i - 2, j) + kD4[1] * F(in, i - 1, j) +
                             kD4[2] * F(in, i, j) + kD4[3] * F(in, i + 1, j));
  };
  auto dx_n = [&](std::vector<float>& out, std::vector<float>& in) {  // to the node
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i)
        F(out, i, j) = hi * (kD4[0] * F(in, i - 1, j) + kD4[1] * F(in, i, j) +
                             kD4[2] * F(in, i + 1, j) + kD4[3] * F(in, i + 2, j));
  };
  auto dy_h = [&](std::vector<float>& out, std::vector<float>& in) {
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i)
        F(out, i, j) = hi * (kD4[0] * F(in, i, j - 2) + kD4[1] * F(in, i, j - 1) +
                             kD4[2] * F(in, i, j) + kD4[3] * F(in, i, j + 1));
  };
  auto dy_n = [&](std::vector<float>& out, std::vector<float>& in) {
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i)
        F(out, i, j) = hi * (kD4[0] * F(in, i, j - 1) + kD4[1] * F(in, i, j) +
                             kD4[2] * F(in, i, j + 1) + kD4[3] * F(in, i, j + 2));
  };
  dx_h(m->f1_1, m->f_c);
  dx_n(m->f1_2, m->f);
  dx_n(m->f1_c, m->f_1);
  dy_h(m->f2_1, m->f);
  dy_n(m->f2_2, m->f_c);
  dy_h(m->f2_c, m->f_2);

  // g: unstretched vertical coordinate (geom_no_grid_stretching with
  // metrics_grid_g, metrics.c:316-339): spacing 1/(1/h) in float, the top
  // point set to 0 by the closed upper boundary of grid_fill1
  const float hg = (float)(1.0 / (double)hi);
  std::vector<float>& g = m->g;
  const int A = AWP_ALIGN;
  grid_fill1(&g[A], nz, 0, 0, 0, 1, hg);
  std::vector<float>& gc = m->g_c;
  std::vector<float>& g3 = m->g3;
  std::vector<float>& g3c = m->g3_c;
  // g_c (metrics_g_interp_110/111/112)
  for (int k = 0; k < 6; ++k) {
    float s = 0.f;
    s = kTopoGPhzl[k][0] * g[A + 0] + kTopoGPhzl[k][1] * g[A + 1] + kTopoGPhzl[k][2] * g[A + 2] +
        kTopoGPhzl[k][3] * g[A + 3] + kTopoGPhzl[k][4] * g[A + 4] + kTopoGPhzl[k][5] * g[A + 5] +
        kTopoGPhzl[k][6] * g[A + 6];
    gc[A + k] = s;
  }
  for (int k = 0; k < nz - 12; ++k)
    gc[A + k + 6] = kP4[0] * g[A + k + 4] + kP4[1] * g[A + k + 5] + kP4[2] * g[A + k + 6] +
                    kP4[3] * g[A + k + 7];
  for (int k = 0; k < 6; ++k) {
    float s = kTopoGPhzr[k][7] * g[A + nz - 8];
    for (int q = 6; q >= 0; --q) s = s + kTopoGPhzr[k][q] * g[A + nz - 1 - q];
    gc[A + nz - 1 - k] = s;
  }
  // g3 = d g_c / dz at the nodes (metrics_g_diff_3_110/111/112)
  for (int k = 0; k < 6; ++k) {
    float s = kTopoGDzl[k][0] * gc[A + 0];
    for (int q = 1; q < 8; ++q) s = s + kTopoGDzl[k][q] * gc[A + q];
    g3[A + k] = hi * s;
  }
  for (int k = 0; k < nz - 12; ++k)
    g3[A + k + 6] = hi * (kD4[0] * gc[A + k + 5] + kD4[1] * gc[A + k + 6] +
                          kD4[2] * gc[A + k + 7] + kD4[3] * gc[A + k + 8]);
  for (int k = 0; k < 6; ++k) {
    float s = kTopoGDzr[k][6] * gc[A + nz - 7];
    for (int q = 5; q >= 0; --q) s = s + kTopoGDzr[k][q] * gc[A + nz - 1 - q];
    g3[A + nz - 1 - k] = hi * s;
  }
  g3[A + nz - 1] = 1.0f;  // metrics.c:294-297: the ghost point must not be 0
  // g3_c = d g / dz at the cell centres (metrics_g_diff_c_110/111/112)
  for (int k = 0; k < 6; ++k) {
    float s = kTopoGDhzl[k][0] * g[A + 0];
    for (int q = 1; q < 7; ++q) s = s + kTopoGDhzl[k][q] * g[A + q];
    g3c[A + k] = hi * s;
  }
  for (int k = 0; k < nz - 12; ++k)
    g3c[A + k + 6] = hi * (kD4[0] * g[A + k + 4] + kD4[1] * g[A + k + 5] +
                           kD4[2] * g[A + k + 6] + kD4[3] * g[A + k + 7]);
  for (int k = 0; k < 6; ++k) {
    float s = kTopoGDhzr[k][7] * g[A + nz - 8];
    for (int q = 6; q >= 0; --q) s = s + kTopoGDhzr[k][q] * g[A + nz - 1 - q];
    g3c[A + nz - 1 - k] = hi * s;
  }
}

}  // namespace awp
