// Shared definitions for the bbFMM B200 kernels.
//
// Cell numbering. Cells of level l are addressed two ways:
//  * Morton order (the reference's order): local index m in [0, 8^l); the global
//    reference index is levsta(l) + m and the children of A are 8A+1..8A+8
//    (cell.h:27-28). Sibling bits are (4*xbit + 2*ybit + zbit) at each depth
//    (anotherFMMDistribute.c:239-253).
//  * Class-major parent grid ("cpg"): index ((c*P + pz)*P + py)*P + px with
//    c = m & 7 the sibling class, (px,py,pz) the grid coordinate of the parent and
//    P = 2^(l-1). For a target class and a translation offset v, the source cells
//    of a box of targets form a box of the same shape in one class grid, which is
//    what lets the M2L kernels stage them with single tiled copies.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define BBFMM_MINLEV 2
#define BBFMM_NUM_OFFSETS 316

#define BBFMM_CUDA_OK(call)                                                  \
  do {                                                                       \
    cudaError_t e__ = (call);                                                \
    if (e__ != cudaSuccess) return bbfmm_set_cuda_error(e__, #call, __FILE__, __LINE__); \
  } while (0)

// Error plumbing shared by every entry point (defined in solver.cu).
int bbfmm_set_cuda_error(cudaError_t e, const char *what, const char *file, int line);
int bbfmm_set_error(int code, const char *msg);

enum {
  BBFMM_OK = 0,
  BBFMM_ERR_ARG = 1,
  BBFMM_ERR_CUDA = 2,
  BBFMM_ERR_NOMEM = 3,
  BBFMM_ERR_UNSUPPORTED = 4,
  BBFMM_ERR_STATE = 5,
};

__host__ __device__ inline int64_t pow8i(int l) { return (int64_t)1 << (3 * l); }
__host__ __device__ inline int64_t levsta(int l) { return (pow8i(l) - 1) / 7; }

// Morton (reference order) -> grid coordinates at level l.
__host__ __device__ inline void morton_to_grid(int64_t m, int l, int &ix, int &iy, int &iz) {
  ix = iy = iz = 0;
  for (int b = 0; b < l; ++b) {
    int t = (int)((m >> (3 * b)) & 7);
    ix |= ((t >> 2) & 1) << b;
    iy |= ((t >> 1) & 1) << b;
    iz |= (t & 1) << b;
  }
}

__host__ __device__ inline int64_t grid_to_morton(int ix, int iy, int iz, int l) {
  int64_t m = 0;
  for (int b = l - 1; b >= 0; --b)
    m = m * 8 + (((ix >> b) & 1) << 2) + (((iy >> b) & 1) << 1) + ((iz >> b) & 1);
  return m;
}

// Grid coordinates at level l >= 1 -> class-major parent-grid index.
__host__ __device__ inline int64_t grid_to_cpg(int ix, int iy, int iz, int l) {
  const int64_t P = (int64_t)1 << (l - 1);
  const int c = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
  return ((c * P + (iz >> 1)) * P + (iy >> 1)) * P + (ix >> 1);
}

// Cell (stacked Morton row) of local row t of a pass: rows[t] when the pass runs over a row
// list (a local solve), else the slab's first row row0 + t.
__host__ __device__ inline int64_t pass_cell(const int64_t *rows, int64_t row0, int64_t t) {
  return rows ? rows[t] : row0 + t;
}

// Class-major row of stacked Morton row m of level l: set base + in-set cpg index.
__host__ __device__ inline int64_t morton_to_cpg_row(int64_t m, int l) {
  int ix, iy, iz;
  morton_to_grid(m, l, ix, iy, iz);  // the set index above bit 3 l is ignored
  return (m & ~(pow8i(l) - 1)) + grid_to_cpg(ix, iy, iz, l);
}

// Centre of a cell exactly as the reference accumulates it from the root
// (anotherFMMDistribute.c:191-255, 336-344): c_l = c_{l-1} +/- celeng[l]/2, with
// celeng[l] = L * 0.5^l obtained by repeated halving.
template <typename T>
__host__ __device__ inline T cell_center_1d(int i, int l, T L) {
  T c = (T)0;
  T len = L;
  for (int k = 1; k <= l; ++k) {
    len *= (T)0.5;
    const T h = len / (T)2;
    const int bit = (i >> (l - k)) & 1;
    c = bit ? c + h : c - h;
  }
  return c;
}

template <typename T>
__host__ __device__ inline T cell_length(int l, T L) {
  T len = L;
  for (int k = 1; k <= l; ++k) len *= (T)0.5;
  return len;
}

namespace bbfmm {
// Device copies of the Chebyshev tables (only the working precision is filled).
struct Tables {
  const double *tkz_d, *cw_d, *kw_d;
  const float *tkz_f, *cw_f, *kw_f;
};
// Row remapping of the projection GEMMs between Morton and cpg order.
enum { MAP_NONE = 0, MAP_IN_CPG = 1, MAP_OUT_CPG = 2 };
}  // namespace bbfmm
