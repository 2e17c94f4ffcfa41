// Shared definitions for the B200 time-step library (host + device).
//
// Field layout in HBM is the reference's padded layout, so that pointers can be
// exchanged with pmcl3d-style callers unchanged (pmcl3d.c:827, kernel.cu:87-94):
//
//   index(i, j, k) = i * slice + j * yline + k          (k fastest)
//   extents        = (nxt + 4 + 2*NGSL) x (nyt + 4 + 2*NGSL) x (nzt + 2*ALIGN)
//   interior       = i, j in [2+NGSL, 2+NGSL+n), k in [ALIGN, ALIGN+nzt)
//   free surface   = k = nzt + ALIGN - 1 (the top)
//
// With ALIGN = 32 every z column starts on a 128-byte boundary, so a warp
// spanning 32 consecutive k reads one full 128-byte line per field.
#pragma once

#include <stddef.h>
#include <stdint.h>

#define AWP_NGSL 8
#define AWP_NGSL2 16
#define AWP_ALIGN 32
#define AWP_MAXGRIDS 10
#define AWP_MAXFILT 20
#define AWP_WWL 2

#ifdef __CUDACC__
#define AWP_HD __host__ __device__ __forceinline__
#else
#define AWP_HD inline
#endif

struct AwpGeom {
  int nxt, nyt, nzt;  // interior cells of this grid
  int yline;          // nzt + 2*ALIGN
  int slice;          // (nyt + 4 + 2*NGSL) * yline
  AWP_HD long long nx_pad() const { return nxt + 4 + AWP_NGSL2; }
  AWP_HD long long ny_pad() const { return nyt + 4 + AWP_NGSL2; }
  AWP_HD long long nz_pad() const { return nzt + 2 * AWP_ALIGN; }
  AWP_HD long long cells_pad() const { return nx_pad() * ny_pad() * nz_pad(); }
  AWP_HD int top() const { return nzt + AWP_ALIGN - 1; }
};

inline AwpGeom awp_make_geom(int nxt, int nyt, int nzt) {
  AwpGeom g;
  g.nxt = nxt;
  g.nyt = nyt;
  g.nzt = nzt;
  g.yline = nzt + 2 * AWP_ALIGN;
  g.slice = (nyt + 4 + AWP_NGSL2) * g.yline;
  return g;
}

// Memory-variable parity pattern.  The reference stores vx1/vx2/ww/wwo as four
// full 3-D arrays (init_texture, mesh.c:1103-1137), but every value is one of
// eight entries selected by the parity of the visit counters of that loop, so
// the kernels recompute them from (i, j, k) and read no array.
struct AwpTexture {
  float tau1[8];   // 0.5*(1 - exp(-DT/tau))      -> vx1
  float tau2[8];   // exp(-DT/tau)                -> vx2
  float wwo8[8];   // 8 * weight                  -> wwo
  int xls, yls;    // first (i, j) visited by init_texture
  int ny;          // yre - yls + 1
  int nzt;         // z cells of the grid
  // Discontinuous mesh: on a grid with a finer grid above it, the top three
  // levels hold the finer grid's values at the co-located points (checkmesh
  // of the texture arrays, pmcl3d.c:1051-1057 with mesh.c:1404-1443).
  int dm;          // 1 on such a grid
  int nx;          // interior cells in x of this grid
  int f_ny, f_nzt; // the finer grid's interior cells in y and z
};

// Parity index of init_texture's visit counters (mesh.c:1103-1137) for the
// cell (di, dj, kk) relative to the loop start: itx = parity of di + 1, ity =
// parity of di*ny + dj + 1, itz = parity of nzt*(di*ny + dj + 1) + kk.  Only
// the low bits matter, so the products reduce to bit operations.
AWP_HD int awp_tex_index_base(long long di, long long dj, int ny, int nzt, int kk) {
  const int pdi = (int)(di & 1);
  const int pij1 = ((pdi & ny) + (int)(dj & 1) + 1) & 1;  // parity of di*ny + dj + 1
  const int itx = pdi ^ 1;
  const int itz = ((nzt & pij1) + kk) & 1;
  return 4 * itx + 2 * pij1 + itz;
}

// Index into the eight-entry tables (= ww - 1 of the reference).
AWP_HD int awp_tex_index(const AwpTexture& t, int i, int j, int k) {
  if (t.dm) {
    const int l = k - (AWP_ALIGN + t.nzt - 3);
    if (l >= 0 && l < 3 && i >= t.xls && i < t.xls + t.nx && j >= t.yls && j < t.yls + t.ny) {
      const int ih = (i - 2 - AWP_NGSL) * 3 + 2 + AWP_NGSL;
      const int jh = (j - 2 - AWP_NGSL) * 3 + 3 + AWP_NGSL;
      return awp_tex_index_base(ih - (2 + AWP_NGSL), jh - (2 + AWP_NGSL), t.f_ny, t.f_nzt,
                                1 + 3 * l);
    }
  }
  return awp_tex_index_base(i - t.xls, j - t.yls, t.ny, t.nzt, k - AWP_ALIGN);
}

// Status codes are the AWP_OK / AWP_ERR_* values of include/awp_b200.h.
