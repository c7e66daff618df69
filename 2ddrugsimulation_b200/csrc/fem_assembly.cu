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

// Per-Gauss-point geometry of an element with node coordinates x[nn][dim],
// in the reference's sequence of operations (Cfem::set_amat_bmat,
// fem.cpp:628-661 with inverseMat, fem.cpp:557-589): the Jacobian
// J[r][c] = sum_a dS[a][r] x[a][c] over the nodes in order, its determinant
// and cofactor inverse xJ, and the physical gradient of node a,
// dX[i] = sum_j dS[a][j] xJ[i][j].
struct ElemGeom {
  double det, xJ[3][3];
};

__device__ void elem_geom(int dim, int nn, const double (*dS)[3], const double *x, ElemGeom &eg) {
  double J[3][3];
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) {
      double acc = 0.0;
      for (int a = 0; a < nn; ++a) acc += dS[a][r] * x[a * dim + c];
      J[r][c] = acc;
    }
  if (dim == 3) {
    const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    eg.det = det;
    eg.xJ[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    eg.xJ[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) / det;
    eg.xJ[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    eg.xJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) / det;
    eg.xJ[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    eg.xJ[2][1] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]) / det;
    eg.xJ[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    eg.xJ[1][2] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]) / det;
    eg.xJ[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  } else {
    const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    eg.det = det;
    eg.xJ[0][0] = J[1][1] / det;
    eg.xJ[0][1] = -J[0][1] / det;
    eg.xJ[1][0] = -J[1][0] / det;
    eg.xJ[1][1] = J[0][0] / det;
  }
}

__device__ __forceinline__ void phys_grad(int dim, const double ds[3], const ElemGeom &eg, double dx[3]) {
  for (int i = 0; i < dim; ++i) {
    double acc = 0.0;
    for (int j = 0; j < dim; ++j) acc += ds[j] * eg.xJ[i][j];
    dx[i] = acc;
  }
}

// The stiffness contribution of one Gauss point: with a scalar D the
// reference's (sum_i dX_a[i] dX_b[i]) detJ D; with a tensor (the
// anisotropic extension) grad Phi_a . D grad Phi_b detJ.
__device__ __forceinline__ double stiffness(int dim, const double dxa[3], const double dxb[3], const double *D,
                                            int n_d, const double (&Dm)[3][3], double det) {
  if (n_d == 1) {
    double acc = 0.0;
    for (int i = 0; i < dim; ++i) acc += dxa[i] * dxb[i];
    return acc * det * D[0];
  }
  double gdg = 0.0;
  for (int u = 0; u < dim; ++u)
    for (int v = 0; v < dim; ++v) gdg += dxa[u] * Dm[u][v] * dxb[v];
  return gdg * det;
}

// Entry (a, b) of the element matrices of the axis-aligned grid element of
// edge h with its first node at the origin (every element of the grid uses
// these), Gauss point by Gauss point with unit weights:
//   A_e[a][b] += Phi_a Phi_b detJ / dt + stiffness,  B_e[a][b] += Phi_a Phi_b detJ.
__device__ void element_entry(int dim, double h, double dt, const double *D, int n_d, const double (&Dm)[3][3],
                              int a, int b, double &ae, double &be) {
  const int ng = dim == 2 ? 4 : 8;
  double x[24];
  for (int n = 0; n < ng; ++n) {
    const int q = n & 3;
    x[n * dim + 0] = (q == 1 || q == 2) ? 1.0 * h : 0.0 * h;
    x[n * dim + 1] = (q >= 2) ? 1.0 * h : 0.0 * h;
    if (dim == 3) x[n * dim + 2] = (n >= 4) ? 1.0 * h : 0.0 * h;
  }
  ae = 0.0;
  be = 0.0;
  for (int g = 0; g < ng; ++g) {
    double s, t, z;
    gauss_point(dim, g, s, t, z);
    double dS[8][3], phi[8];
    for (int n = 0; n < ng; ++n) shape(dim, n, s, t, z, phi[n], dS[n]);
    ElemGeom eg;
    elem_geom(dim, ng, dS, x, eg);
    double dxa[3], dxb[3];
    phys_grad(dim, dS[a], eg, dxa);
    phys_grad(dim, dS[b], eg, dxb);
    ae += phi[a] * phi[b] * eg.det / dt + stiffness(dim, dxa, dxb, D, n_d, Dm, eg.det);
    be += phi[a] * phi[b] * eg.det;
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
  // A row range of the grid (a slab part): rows row0 .. row0 + n_rows - 1
  // (n_rows 0: every row), stored at local index row - row0 with columns
  // shifted by -col_off; D holds elements e_off onwards.
  int64_t row0, n_rows, col_off, e_off;
};

__global__ void assemble_grid_kernel(GridArgs g) {
  const int64_t n = g.n_rows > 0 ? g.n_rows : (int64_t)g.nx * g.ny * g.nz;
  const int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= n) return;
  const int64_t i = g.row0 + li;  // global row
  const int ix = (int)(i % g.nx);
  const int iy = (int)((i / g.nx) % g.ny);
  const int iz = (int)(i / ((int64_t)g.nx * g.ny));
  const int ex_n = g.nx - 1, ey_n = g.ny - 1, ez_n = g.dim == 3 ? g.nz - 1 : 1;
  int64_t q = g.rp[li];
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
              const double *De = g.D + (e - g.e_off) * g.n_d;
              double Dm[3][3];
              tensor_of(g.dim, De, g.n_d, Dm);
              const int la = local_index(ix - ex, iy - ey, g.dim == 3 ? iz - ez : 0);
              const int lb = local_index(jx - ex, jy - ey, g.dim == 3 ? jz - ez : 0);
              double ae, be;
              element_entry(g.dim, g.h, g.dt, De, g.n_d, Dm, la, lb, ae, be);
              av += ae;
              bv += be;
            }
        g.col[q] = (int)(j - g.col_off);
        g.a[q] = av;
        g.b[q] = bv;
        ++q;
        g.ecol[(int64_t)slot * g.ld + li] = (int)(j - g.col_off);
        g.ea[(int64_t)slot * g.ld + li] = av;
        g.eb[(int64_t)slot * g.ld + li] = bv;
        ++slot;
        if (j == i) diag = av;
      }
  for (; slot < g.width; ++slot) {  // padding: the row's own column with zero weight
    g.ecol[(int64_t)slot * g.ld + li] = (int)(i - g.col_off);
    g.ea[(int64_t)slot * g.ld + li] = 0.0;
    g.eb[(int64_t)slot * g.ld + li] = 0.0;
  }
  g.dinv[li] = 1.0 / diag;
}

}  // namespace fem
}  // namespace cep

extern "C" int cep_internal_fem_assemble_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *d_D,
                                              int n_d, const int *d_rp, int *d_col, double *d_a, double *d_b,
                                              int width, int64_t ld, int *d_ecol, double *d_ea, double *d_eb,
                                              double *d_dinv, void *stream) {
  cep::fem::GridArgs g{dim, nx, ny, dim == 3 ? nz : 1, h, dt, d_D, n_d, d_rp, d_col, d_a, d_b,
                       width, ld, d_ecol, d_ea, d_eb, d_dinv, 0, 0, 0, 0};
  const int64_t n = (int64_t)g.nx * g.ny * g.nz;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  cep::fem::assemble_grid_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Rows row0 .. row0 + n_rows - 1 of the same operator (a slab part), with
// the same kernel and so the same bits; columns shifted by -col_off, D
// starting at element e_off.
extern "C" int cep_internal_fem_assemble_grid_rows(int dim, int nx, int ny, int nz, double h, double dt,
                                                   const double *d_D, int n_d, int64_t e_off, int64_t row0,
                                                   int64_t n_rows, int64_t col_off, const int *d_rp, int *d_col,
                                                   double *d_a, double *d_b, int width, int64_t ld, int *d_ecol,
                                                   double *d_ea, double *d_eb, double *d_dinv, void *stream) {
  cep::fem::GridArgs g{dim, nx, ny, dim == 3 ? nz : 1, h, dt, d_D, n_d, d_rp, d_col, d_a, d_b,
                       width, ld, d_ecol, d_ea, d_eb, d_dinv, row0, n_rows, col_off, e_off};
  const int block = 128;
  const unsigned grid = (unsigned)((n_rows + block - 1) / block);
  cep::fem::assemble_grid_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ------------------------------------------------ P1 tetrahedral meshes
// Unstructured meshes of linear tetrahedra (the reference's "tet" meshes:
// Gauss points fem.cpp:209-229, shape functions fem.cpp:342-373, element
// matrices fem.cpp:628-661 with unit Gauss weights). One thread per node
// (row): its incident elements in ascending order, each adding its row of
// the element matrices to the row's sorted columns, local nodes in order.
namespace cep {
namespace fem {

// Row la of the element matrices of tetrahedron x[4][3] in the reference's
// sequence of operations (the constant Jacobian is recomputed at each of
// the four Gauss points, as fem.cpp:640-651 does).
__device__ void tet_row(const double x[4][3], const double *D, int n_d, double dt, int la, double *arow,
                        double *brow) {
  const double aaa = (5. - sqrt(5.)) / 20., bbb = (5. + 3. * sqrt(5.)) / 20.;
  const double gp[4][3] = {{aaa, aaa, aaa}, {aaa, aaa, bbb}, {aaa, bbb, aaa}, {bbb, aaa, aaa}};
  const double dS[4][3] = {{-1., -1., -1.}, {1., 0., 0.}, {0., 1., 0.}, {0., 0., 1.}};
  double Dm[3][3];
  tensor_of(3, D, n_d, Dm);
  for (int k = 0; k < 4; ++k) {
    arow[k] = 0.;
    brow[k] = 0.;
  }
  for (int g = 0; g < 4; ++g) {
    ElemGeom eg;
    elem_geom(3, 4, dS, &x[0][0], eg);
    const double s = gp[g][0], t = gp[g][1], z = gp[g][2];
    const double phi[4] = {1. - s - t - z, s, t, z};
    double dxa[3];
    phys_grad(3, dS[la], eg, dxa);
    for (int k = 0; k < 4; ++k) {
      double dxb[3];
      phys_grad(3, dS[k], eg, dxb);
      arow[k] += phi[la] * phi[k] * eg.det / dt + stiffness(3, dxa, dxb, D, n_d, Dm, eg.det);
      brow[k] += phi[la] * phi[k] * eg.det;
    }
  }
}

__global__ void assemble_tet_kernel(int n_nodes, const double *xyz, const int *conn, const double *D, int n_d,
                                    double dt, const int *inc_ptr, const int *inc, const int *rp, const int *col,
                                    double *a, double *b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_nodes) return;
  const int r0 = rp[i], r1 = rp[i + 1];
  for (int q = r0; q < r1; ++q) {
    a[q] = 0.;
    b[q] = 0.;
  }
  for (int p = inc_ptr[i]; p < inc_ptr[i + 1]; ++p) {
    const int e = inc[2 * p], la = inc[2 * p + 1];
    double x[4][3], ar[4], br[4];
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 3; ++c) x[k][c] = xyz[3 * (int64_t)conn[4 * (int64_t)e + k] + c];
    tet_row(x, D + (int64_t)e * n_d, n_d, dt, la, ar, br);
    for (int k = 0; k < 4; ++k) {
      const int j = conn[4 * (int64_t)e + k];
      int q = r0;
      while (q < r1 - 1 && col[q] != j) ++q;
      a[q] += ar[k];
      b[q] += br[k];
    }
  }
}

}  // namespace fem
}  // namespace cep

extern "C" int cep_internal_fem_assemble_tet(int n_nodes, const double *d_xyz, const int *d_conn, const double *d_D,
                                             int n_d, double dt, const int *d_inc_ptr, const int *d_inc,
                                             const int *d_rp, const int *d_col, double *d_a, double *d_b,
                                             void *stream) {
  cep::fem::assemble_tet_kernel<<<(n_nodes + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      n_nodes, d_xyz, d_conn, d_D, n_d, dt, d_inc_ptr, d_inc, d_rp, d_col, d_a, d_b);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
