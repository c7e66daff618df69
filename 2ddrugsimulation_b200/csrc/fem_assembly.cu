// Device assembly of the monodomain operators on a structured grid:
// A = M/dt + D K and B = M with Q1 quadrilaterals (2D) or trilinear
// hexahedra (3D), written both as CSR and as column-major ELL.
//
// Element integrals follow Cfem::set_amat_bmat (fem.cpp:628-661): Gauss
// points at +-0.57735 with unit weights (fem.cpp:231-271), the reference's
// shape functions and local node order (fem.cpp:398-478), and
//   A_e[j][k] = sum_g Phi_j Phi_k detJ/dt + grad Phi_j . D grad Phi_k detJ
//   B_e[j][k] = sum_g Phi_j Phi_k detJ.
// D is one scalar per element (the reference's DE, fem.cpp:656) or a
// symmetric tensor per element (anisotropic extension).
//
// One thread per node (row). For every stencil neighbour in ascending column
// order it sums the entry over the elements that share both nodes in
// ascending element order, which is the order in which element-by-element
// scatter assembly adds them. This file is compiled without FMA contraction
// so each entry is the same IEEE expression as a scalar assembly.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace cep {
namespace fem {

constexpr double kGauss = 0.57735;  // fem.cpp:231-271 (truncated 1/sqrt(3))

__device__ __forceinline__ void gauss_point(int dim, int g, double &s, double &t, double &z) {
  if (dim == 2) {
    // (-,-), (+,-), (+,+), (-,+)
    s = (g == 0 || g == 3) ? -kGauss : kGauss;
    t = (g < 2) ? -kGauss : kGauss;
    z = 0.0;
  } else {
    // g = 4*ix + 2*iy + iz over {-,+}^3
    s = (g & 4) ? kGauss : -kGauss;
    t = (g & 2) ? kGauss : -kGauss;
    z = (g & 1) ? kGauss : -kGauss;
  }
}

// Shape function of local node a and its reference-space gradient.
__device__ __forceinline__ void shape(int dim, int a, double s, double t, double z, double &phi, double ds[3]) {
  if (dim == 2) {
    switch (a) {
      case 0: phi = (1. - s) * (1. - t) / 4.; ds[0] = -(1. - t) / 4.; ds[1] = -(1. - s) / 4.; break;
      case 1: phi = (1. + s) * (1. - t) / 4.; ds[0] = +(1. - t) / 4.; ds[1] = -(1. + s) / 4.; break;
      case 2: phi = (1. + s) * (1. + t) / 4.; ds[0] = +(1. + t) / 4.; ds[1] = +(1. + s) / 4.; break;
      default: phi = (1. - s) * (1. + t) / 4.; ds[0] = -(1. + t) / 4.; ds[1] = +(1. - s) / 4.; break;
    }
    ds[2] = 0.0;
    return;
  }
  // local node a: x bit from {0:-,1:+,2:+,3:-}, y bit from {0,1:-; 2,3:+}, z from a >= 4
  const int q = a & 3;
  const double sx = (q == 1 || q == 2) ? 1.0 : -1.0;
  const double sy = (q >= 2) ? 1.0 : -1.0;
  const double sz = (a >= 4) ? 1.0 : -1.0;
  const double fs = sx > 0 ? 1 + s : 1 - s, ft = sy > 0 ? 1 + t : 1 - t, fz = sz > 0 ? 1 + z : 1 - z;
  phi = fs * ft * fz / 8.;
  const double gs = 1 + sx * s, gt = 1 + sy * t, gz = 1 + sz * z;
  ds[0] = sx * gt * gz / 8.;
  ds[1] = sy * gs * gz / 8.;
  ds[2] = sz * gs * gt / 8.;
}

// Entry (a, b) of the element matrices of an axis-aligned element of edge h.
__device__ void element_entry(int dim, double h, double dt, const double (&Dm)[3][3], int a, int b, double &ae,
                              double &be) {
  const double jac = 0.5 * h;
  const double detJ = dim == 2 ? jac * jac : jac * jac * jac;
  const double inv = 1.0 / jac;
  const int ng = dim == 2 ? 4 : 8;
  ae = 0.0;
  be = 0.0;
  for (int g = 0; g < ng; ++g) {
    double s, t, z;
    gauss_point(dim, g, s, t, z);
    double pa, pb, dsa[3], dsb[3];
    shape(dim, a, s, t, z, pa, dsa);
    shape(dim, b, s, t, z, pb, dsb);
    double dxa[3], dxb[3];
    for (int d = 0; d < dim; ++d) {
      dxa[d] = dsa[d] * inv;
      dxb[d] = dsb[d] * inv;
    }
    double gdg = 0.0;
    for (int u = 0; u < dim; ++u)
      for (int v = 0; v < dim; ++v) gdg += dxa[u] * Dm[u][v] * dxb[v];
    ae += pa * pb * detJ / dt + gdg * detJ;
    be += pa * pb * detJ;
  }
}

__device__ __forceinline__ void tensor_of(int dim, const double *D, int n_d, double (&Dm)[3][3]) {
  for (int u = 0; u < 3; ++u)
    for (int v = 0; v < 3; ++v) Dm[u][v] = 0.0;
  if (n_d == 1) {
    for (int u = 0; u < dim; ++u) Dm[u][u] = D[0];
  } else if (dim == 2) {
    Dm[0][0] = D[0]; Dm[0][1] = Dm[1][0] = D[1]; Dm[1][1] = D[2];
  } else {
    Dm[0][0] = D[0]; Dm[0][1] = Dm[1][0] = D[1]; Dm[0][2] = Dm[2][0] = D[2];
    Dm[1][1] = D[3]; Dm[1][2] = Dm[2][1] = D[4]; Dm[2][2] = D[5];
  }
}

// local index of the node at offset (ox, oy, oz) of its element
__device__ __forceinline__ int local_index(int ox, int oy, int oz) {
  const int q = oy == 0 ? ox : 3 - ox;  // (0,0)->0 (1,0)->1 (1,1)->2 (0,1)->3
  return q + 4 * oz;
}

struct GridArgs {
  int dim, nx, ny, nz;
  double h, dt;
  const double *D;  // [n_elem][n_d]
  int n_d;
  const int *rp;    // CSR row pointers (host-computed)
  int *col;
  double *a, *b;
  int width;
  int64_t ld;
  int *ecol;        // ELL [width][ld]
  double *ea, *eb;
  double *dinv;
};

__global__ void assemble_grid_kernel(GridArgs g) {
  const int64_t n = (int64_t)g.nx * g.ny * g.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ix = (int)(i % g.nx);
  const int iy = (int)((i / g.nx) % g.ny);
  const int iz = (int)(i / ((int64_t)g.nx * g.ny));
  const int ex_n = g.nx - 1, ey_n = g.ny - 1, ez_n = g.dim == 3 ? g.nz - 1 : 1;
  int64_t q = g.rp[i];
  int slot = 0;
  double diag = 1.0;
  const int dk0 = g.dim == 3 ? -1 : 0, dk1 = g.dim == 3 ? 1 : 0;
  for (int dk = dk0; dk <= dk1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        const int jx = ix + di, jy = iy + dj, jz = iz + dk;
        if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) continue;
        const int64_t j = (int64_t)jx + (int64_t)g.nx * ((int64_t)jy + (int64_t)g.ny * jz);
        double av = 0.0, bv = 0.0;
        // elements holding both nodes, ascending element index (z, y, x order)
        const int z_lo = max(max(iz, jz) - 1, 0), z_hi = min(min(iz, jz), ez_n - 1);
        const int y_lo = max(max(iy, jy) - 1, 0), y_hi = min(min(iy, jy), ey_n - 1);
        const int x_lo = max(max(ix, jx) - 1, 0), x_hi = min(min(ix, jx), ex_n - 1);
        for (int ez = (g.dim == 3 ? z_lo : 0); ez <= (g.dim == 3 ? z_hi : 0); ++ez)
          for (int ey = y_lo; ey <= y_hi; ++ey)
            for (int ex = x_lo; ex <= x_hi; ++ex) {
              const int64_t e = (int64_t)ex + (int64_t)ex_n * ((int64_t)ey + (int64_t)ey_n * ez);
              double Dm[3][3];
              tensor_of(g.dim, g.D + e * g.n_d, g.n_d, Dm);
              const int la = local_index(ix - ex, iy - ey, g.dim == 3 ? iz - ez : 0);
              const int lb = local_index(jx - ex, jy - ey, g.dim == 3 ? jz - ez : 0);
              double ae, be;
              element_entry(g.dim, g.h, g.dt, Dm, la, lb, ae, be);
              av += ae;
              bv += be;
            }
        g.col[q] = (int)j;
        g.a[q] = av;
        g.b[q] = bv;
        ++q;
        g.ecol[(int64_t)slot * g.ld + i] = (int)j;
        g.ea[(int64_t)slot * g.ld + i] = av;
        g.eb[(int64_t)slot * g.ld + i] = bv;
        ++slot;
        if (j == i) diag = av;
      }
  for (; slot < g.width; ++slot) {  // padding: the row's own column with zero weight
    g.ecol[(int64_t)slot * g.ld + i] = (int)i;
    g.ea[(int64_t)slot * g.ld + i] = 0.0;
    g.eb[(int64_t)slot * g.ld + i] = 0.0;
  }
  g.dinv[i] = 1.0 / diag;
}

}  // namespace fem
}  // namespace cep

extern "C" int cep_internal_fem_assemble_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *d_D,
                                              int n_d, const int *d_rp, int *d_col, double *d_a, double *d_b,
                                              int width, int64_t ld, int *d_ecol, double *d_ea, double *d_eb,
                                              double *d_dinv, void *stream) {
  cep::fem::GridArgs g{dim, nx, ny, dim == 3 ? nz : 1, h, dt, d_D, n_d, d_rp, d_col, d_a, d_b,
                       width, ld, d_ecol, d_ea, d_eb, d_dinv};
  const int64_t n = (int64_t)g.nx * g.ny * g.nz;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  cep::fem::assemble_grid_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
