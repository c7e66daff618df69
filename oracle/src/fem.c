/*
 * TEST INFRASTRUCTURE ONLY. CPU restatement of the reference's monodomain
 * FEM diffusion solve (fem.cpp / heart.cpp) on structured grids.
 *
 * Elements: Q1 quadrilaterals (2D), trilinear hexahedra (3D) and P1
 * tetrahedra with the reference's local node order and shape functions
 * (fem.cpp:342-478), its Gauss points (+-0.57735 with unit weights,
 * fem.cpp:209-271), and its element matrices (fem.cpp:628-661) in its own
 * sequence of floating-point operations (cepo_element):
 *   A_e[j][k] = sum_g Phi_j Phi_k detJ/dt + grad Phi_j . grad Phi_k detJ D
 *   B_e[j][k] = sum_g Phi_j Phi_k detJ
 * D per element is the reference's scalar DE (n_d == 1) or, as an
 * extension for anisotropic tissue, a symmetric tensor. The global solve
 * A V = B V* / dt uses Jacobi-preconditioned CG from a zero initial guess
 * (fem.cpp:705-718, 753-760; PETSc KSPCG + PCJACOBI, KSPSetInitialGuessNonzero
 * is never called). PETSc itself is not in the reference tree, so the
 * stopping rule is stated here: ||M^-1 r||_2 <= rtol ||M^-1 b||_2 (PETSc's
 * default preconditioned norm for CG) or ||r||_2 <= rtol ||b||_2.
 * Parity of the solve with PETSc is unpinned.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "cep_oracle.h"

static const double GA = 0.57735;

long cepo_fem_nnz(int dim, int nx, int ny, int nz) {
  /* stencil neighbours of every node, (3 or 2 per axis) */
  long cx = 3L * nx - 2, cy = 3L * ny - 2, cz = dim == 3 ? 3L * nz - 2 : 1;
  return cx * cy * cz;
}

/* local node offsets of the reference's node order */
static void local_offsets(int dim, int off[8][3]) {
  static const int q4[4][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
  static const int h8[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  memcpy(off, dim == 2 ? (const void *)q4 : (const void *)h8, sizeof(int) * 3 * (dim == 2 ? 4 : 8));
}

/* Gauss points, shape functions and their reference-space gradients of the
 * reference's element types: kind 0 Q1 square (fem.cpp:256-271,398-425),
 * kind 1 trilinear hex (fem.cpp:231-248,427-478), kind 2 P1 tetrahedron
 * (fem.cpp:209-229,342-373); nodes in the reference's local order. */
static void element_basis(int kind, int g, double Phi[8], double dS[8][3]) {
  if (kind == 0) {
    const double g4[4][2] = {{-GA, -GA}, {GA, -GA}, {GA, GA}, {-GA, GA}};
    const double s = g4[g][0], t = g4[g][1];
    Phi[0] = (1. - s) * (1. - t) / 4.; Phi[1] = (1. + s) * (1. - t) / 4.;
    Phi[2] = (1. + s) * (1. + t) / 4.; Phi[3] = (1. - s) * (1. + t) / 4.;
    dS[0][0] = -(1. - t) / 4.; dS[0][1] = -(1. - s) / 4.;
    dS[1][0] = +(1. - t) / 4.; dS[1][1] = -(1. + s) / 4.;
    dS[2][0] = +(1. + t) / 4.; dS[2][1] = +(1. + s) / 4.;
    dS[3][0] = -(1. + t) / 4.; dS[3][1] = +(1. - s) / 4.;
  } else if (kind == 1) {
    const double aa[2] = {-GA, GA};
    const double s = aa[(g >> 2) & 1], t = aa[(g >> 1) & 1], z = aa[g & 1];
    const double sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                             {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    for (int n = 0; n < 8; ++n) {
      const double fs = 1 + sg[n][0] * s, ft = 1 + sg[n][1] * t, fz = 1 + sg[n][2] * z;
      Phi[n] = fs * ft * fz / 8.;
      dS[n][0] = sg[n][0] * ft * fz / 8.; dS[n][1] = sg[n][1] * fs * fz / 8.; dS[n][2] = sg[n][2] * fs * ft / 8.;
    }
  } else {
    const double aaa = (5. - sqrt(5.)) / 20., bbb = (5. + 3. * sqrt(5.)) / 20.;
    const double gp[4][3] = {{aaa, aaa, aaa}, {aaa, aaa, bbb}, {aaa, bbb, aaa}, {bbb, aaa, aaa}};
    const double s = gp[g][0], t = gp[g][1], z = gp[g][2];
    Phi[0] = 1. - s - t - z; Phi[1] = s; Phi[2] = t; Phi[3] = z;
    const double d4[4][3] = {{-1., -1., -1.}, {1., 0., 0.}, {0., 1., 0.}, {0., 0., 1.}};
    memcpy(dS, d4, sizeof(d4));
  }
}

/* Element matrices of one element with node coordinates x[nn][dim]
 * (fem.cpp:628-661), in the reference's sequence of operations: per Gauss
 * point the Jacobian J[r][c] = sum_a dS[a][r] x[a][c] summed over the nodes
 * in order, its determinant and cofactor inverse (fem.cpp:544-589), the
 * physical gradients dX[a][i] = sum_j dS[a][j] xJ[i][j] and
 * K[j][k] = sum_i dX[j][i] dX[k][i]; then, Gauss point by Gauss point,
 *   A_e[j][k] += Phi_j Phi_k detJ / dt + K[j][k] detJ D
 *   B_e[j][k] += Phi_j Phi_k detJ
 * with unit weights. D: the reference's scalar DE (n_d == 1); a symmetric
 * tensor (2D: xx,xy,yy; 3D: xx,xy,xz,yy,yz,zz) is an extension for
 * anisotropic tissue, whose stiffness term is grad Phi_j . D grad Phi_k
 * detJ. */
void cepo_element(int kind, const double *x, const double *D, int n_d, double dt, double *Ae, double *Be) {
  const int dim = kind == 0 ? 2 : 3, nn = kind == 1 ? 8 : 4;
  double Dm[3][3] = {{0}};
  if (n_d > 1 && dim == 2) {
    Dm[0][0] = D[0]; Dm[0][1] = Dm[1][0] = D[1]; Dm[1][1] = D[2];
  } else if (n_d > 1) {
    Dm[0][0] = D[0]; Dm[0][1] = Dm[1][0] = D[1]; Dm[0][2] = Dm[2][0] = D[2];
    Dm[1][1] = D[3]; Dm[1][2] = Dm[2][1] = D[4]; Dm[2][2] = D[5];
  }
  for (int j = 0; j < nn * nn; ++j) { Ae[j] = 0; Be[j] = 0; }
  for (int g = 0; g < nn; ++g) {
    double Phi[8], dS[8][3], J[3][3], xJ[3][3], det;
    element_basis(kind, g, Phi, dS);
    for (int r = 0; r < dim; ++r)
      for (int c = 0; c < dim; ++c) {
        double acc = 0.;
        for (int a = 0; a < nn; ++a) acc += dS[a][r] * x[a * dim + c];
        J[r][c] = acc;
      }
    if (dim == 3) {
      det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
            J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      xJ[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
      xJ[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) / det;
      xJ[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
      xJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) / det;
      xJ[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
      xJ[2][1] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]) / det;
      xJ[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
      xJ[1][2] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]) / det;
      xJ[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    } else {
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      xJ[0][0] = J[1][1] / det; xJ[0][1] = -J[0][1] / det;
      xJ[1][0] = -J[1][0] / det; xJ[1][1] = J[0][0] / det;
    }
    double dX[8][3];
    for (int a = 0; a < nn; ++a)
      for (int i = 0; i < dim; ++i) {
        double acc = 0.;
        for (int j = 0; j < dim; ++j) acc += dS[a][j] * xJ[i][j];
        dX[a][i] = acc;
      }
    for (int j = 0; j < nn; ++j)
      for (int k = 0; k < nn; ++k) {
        double stiff;
        if (n_d == 1) {
          double acc = 0.;
          for (int i = 0; i < dim; ++i) acc += dX[j][i] * dX[k][i];
          stiff = acc * det * D[0];
        } else {
          double gdg = 0.;
          for (int u = 0; u < dim; ++u)
            for (int v = 0; v < dim; ++v) gdg += dX[j][u] * Dm[u][v] * dX[k][v];
          stiff = gdg * det;
        }
        Ae[j * nn + k] += Phi[j] * Phi[k] * det / dt + stiff;
        Be[j * nn + k] += Phi[j] * Phi[k] * det;
      }
  }
}

/* Element matrices of the axis-aligned grid element of edge h with its
 * first node at the origin; every element of a structured grid uses these
 * (the reference's own matrices of translated elements differ from them
 * only by the rounding of its node coordinates). */
void cepo_fem_element(int dim, double h, double dt, const double *D, int n_d, double *Ae, double *Be) {
  int off[8][3];
  local_offsets(dim, off);
  const int nn = dim == 2 ? 4 : 8;
  double x[24];
  for (int a = 0; a < nn; ++a)
    for (int c = 0; c < dim; ++c) x[a * dim + c] = off[a][c] * h;
  cepo_element(dim == 2 ? 0 : 1, x, D, n_d, dt, Ae, Be);
}

/* Shape-function gradients (reference coordinates) at Gauss point g of the
 * reference's element (fem.cpp:398-478), as cepo_fem_element uses them. */
static void gauss_gradients(int dim, int g, double dS[8][3]) {
  double s, t, z = 0.0;
  if (dim == 2) {
    const double g4[4][2] = {{-GA, -GA}, {GA, -GA}, {GA, GA}, {-GA, GA}};
    s = g4[g][0]; t = g4[g][1];
    dS[0][0] = -(1. - t) / 4.; dS[0][1] = -(1. - s) / 4.;
    dS[1][0] = +(1. - t) / 4.; dS[1][1] = -(1. + s) / 4.;
    dS[2][0] = +(1. + t) / 4.; dS[2][1] = +(1. + s) / 4.;
    dS[3][0] = -(1. + t) / 4.; dS[3][1] = +(1. - s) / 4.;
    return;
  }
  const double aa[2] = {-GA, GA};
  s = aa[(g >> 2) & 1]; t = aa[(g >> 1) & 1]; z = aa[g & 1];
  const double sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  for (int n = 0; n < 8; ++n) {
    const double fs = 1 + sg[n][0] * s, ft = 1 + sg[n][1] * t, fz = 1 + sg[n][2] * z;
    dS[n][0] = sg[n][0] * ft * fz / 8.; dS[n][1] = sg[n][1] * fs * fz / 8.; dS[n][2] = sg[n][2] * fs * ft / 8.;
  }
}

/* Pseudo-ECG of a structured-grid tissue at n_el electrodes (Cheart::Radiate,
 * heart.cpp:640-690): for every element, r = centroid - electrode, and for
 * every Gauss point bsp -= (D grad V) . r detJ w / |r|^3 with w = 1/6; the
 * electrode's value is -sum over elements of bsp. Node (i, j, k) sits at
 * (i h, j h, k h). The reference's Gauss counter is uninitialised and its
 * accumulator is never reset between calls; here the loop starts at 0 and
 * every call starts from 0. */
void cepo_pseudo_ecg(int dim, int nx, int ny, int nz, double h, const double *D, int n_d, const double *V,
                     int n_el, const double *xyz, double *phi) {
  if (dim == 2) nz = 1;
  const int nn = dim == 2 ? 4 : 8;
  int off[8][3];
  local_offsets(dim, off);
  const double jac = 0.5 * h, inv = 1.0 / jac;
  const double detJ = dim == 2 ? jac * jac : jac * jac * jac;
  const double w = 1.0 / 6.0;
  for (int k = 0; k < n_el; ++k) phi[k] = 0.0;
  const long nex = nx - 1, ney = ny - 1, nez = dim == 3 ? nz - 1 : 1;
  for (long ez = 0; ez < nez; ++ez)
    for (long ey = 0; ey < ney; ++ey)
      for (long ex = 0; ex < nex; ++ex) {
        const long e = ex + nex * (ey + ney * ez);
        const double *d = D + e * n_d;
        double Dm[3][3] = {{0}};
        if (n_d == 1) {
          for (int a = 0; a < dim; ++a) Dm[a][a] = d[0];
        } else if (dim == 2) {
          Dm[0][0] = d[0]; Dm[0][1] = Dm[1][0] = d[1]; Dm[1][1] = d[2];
        } else {
          Dm[0][0] = d[0]; Dm[0][1] = Dm[1][0] = d[1]; Dm[0][2] = Dm[2][0] = d[2];
          Dm[1][1] = d[3]; Dm[1][2] = Dm[2][1] = d[4]; Dm[2][2] = d[5];
        }
        double ve[8], c[3] = {0, 0, 0};
        for (int a = 0; a < nn; ++a) {
          const long i = ex + off[a][0], j = ey + off[a][1], kk = ez + off[a][2];
          ve[a] = V[i + (long)nx * (j + (long)ny * kk)];
          c[0] += (double)i * h / nn; c[1] += (double)j * h / nn; c[2] += dim == 3 ? (double)kk * h / nn : 0.0;
        }
        for (int g = 0; g < nn; ++g) {
          double dS[8][3];
          gauss_gradients(dim, g, dS);
          double vd[3] = {0, 0, 0}, vel[3] = {0, 0, 0};
          for (int a = 0; a < nn; ++a)
            for (int q = 0; q < dim; ++q) vd[q] += dS[a][q] * inv * ve[a];
          for (int q = 0; q < dim; ++q)
            for (int p2 = 0; p2 < dim; ++p2) vel[q] += Dm[q][p2] * vd[p2];
          for (int k = 0; k < n_el; ++k) {
            const double r[3] = {c[0] - xyz[3 * k], c[1] - xyz[3 * k + 1], c[2] - xyz[3 * k + 2]};
            const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            const double bsp = -(vel[0] * r[0] + vel[1] * r[1] + vel[2] * r[2]) * detJ * w / pow(rr, 3);
            phi[k] -= bsp;
          }
        }
      }
}

static long node_id(int dim, int nx, int ny, int i, int j, int k) {
  (void)dim;
  return (long)i + (long)nx * ((long)j + (long)ny * (long)k);
}

/* CSR over the structured grid: every row lists its stencil neighbours in
 * ascending column order; values summed over the elements sharing both
 * nodes. D holds n_d values per element (element-major). */
int cepo_fem_assemble(int dim, int nx, int ny, int nz, double h, double dt, const double *D, int n_d,
                      int *row_ptr, int *col_idx, double *a_val, double *b_val) {
  if (dim == 2) nz = 1;
  const long n = (long)nx * ny * nz;
  long p = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        row_ptr[node_id(dim, nx, ny, i, j, k)] = (int)p;
        for (int dk = (dim == 3 ? -1 : 0); dk <= (dim == 3 ? 1 : 0); ++dk)
          for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di) {
              const int ii = i + di, jj = j + dj, kk = k + dk;
              if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) continue;
              col_idx[p] = (int)node_id(dim, nx, ny, ii, jj, kk);
              a_val[p] = 0;
              b_val[p] = 0;
              ++p;
            }
      }
  row_ptr[n] = (int)p;
  int off[8][3];
  local_offsets(dim, off);
  const int nn = dim == 2 ? 4 : 8;
  const int ex = nx - 1, ey = ny - 1, ez = dim == 3 ? nz - 1 : 1;
  double Ae[64], Be[64];
  for (int ek = 0; ek < ez; ++ek)
    for (int ej = 0; ej < ey; ++ej)
      for (int ei = 0; ei < ex; ++ei) {
        const long e = (long)ei + (long)ex * ((long)ej + (long)ey * ek);
        cepo_fem_element(dim, h, dt, D + e * n_d, n_d, Ae, Be);
        long gid[8];
        for (int a = 0; a < nn; ++a) gid[a] = node_id(dim, nx, ny, ei + off[a][0], ej + off[a][1], ek + off[a][2]);
        for (int a = 0; a < nn; ++a)
          for (int b = 0; b < nn; ++b) {
            int q = row_ptr[gid[a]];
            while (col_idx[q] != gid[b]) ++q;
            a_val[q] += Ae[a * nn + b];
            b_val[q] += Be[a * nn + b];
          }
      }
  return 0;
}

void cepo_spmv(int n, const int *row_ptr, const int *col_idx, const double *val, const double *x, double *y) {
  for (int i = 0; i < n; ++i) {
    double s = 0;
    for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) s += val[q] * x[col_idx[q]];
    y[i] = s;
  }
}

static double dot(int n, const double *a, const double *b) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* Jacobi-PCG from x = 0. precond_norm: 1 -> ||M^-1 r|| / ||M^-1 b||
 * (PETSc default for CG), 0 -> ||r|| / ||b||. Returns iterations (or
 * -max_iter if not converged). */
int cepo_pcg2(int n, const int *row_ptr, const int *col_idx, const double *a_val, const double *b, double *x,
              double rtol, int max_iter, int precond_norm, double *rel_res) {
  double *dinv = malloc(sizeof(double) * n), *r = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n);
  double *pv = malloc(sizeof(double) * n), *q = malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) {
    double d = 1.0;
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
      if (col_idx[k] == i) d = a_val[k];
    dinv[i] = 1.0 / d;
    x[i] = 0.0;
    r[i] = b[i];
    z[i] = dinv[i] * r[i];
    pv[i] = z[i];
  }
  double rz = dot(n, r, z);
  const double n0 = precond_norm ? sqrt(dot(n, z, z)) : sqrt(dot(n, r, r));
  int it = 0;
  double res = n0 > 0 ? 1.0 : 0.0;
  if (n0 == 0.0) goto done;
  for (it = 1; it <= max_iter; ++it) {
    cepo_spmv(n, row_ptr, col_idx, a_val, pv, q);
    const double alpha = rz / dot(n, pv, q);
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * pv[i];
      r[i] -= alpha * q[i];
      z[i] = dinv[i] * r[i];
    }
    const double rz_new = dot(n, r, z);
    const double nr = precond_norm ? sqrt(dot(n, z, z)) : sqrt(dot(n, r, r));
    res = nr / n0;
    if (nr <= rtol * n0) break;
    const double beta = rz_new / rz;
    rz = rz_new;
    for (int i = 0; i < n; ++i) pv[i] = z[i] + beta * pv[i];
  }
done:
  if (rel_res) *rel_res = res;
  free(dinv); free(r); free(z); free(pv); free(q);
  return it > max_iter ? -max_iter : it;
}

int cepo_pcg(int n, const int *row_ptr, const int *col_idx, const double *a_val, const double *b, double *x,
             double rtol, int max_iter, double *rel_res) {
  return cepo_pcg2(n, row_ptr, col_idx, a_val, b, x, rtol, max_iter, 1, rel_res);
}

/* Tissue: Godunov split of heart.cpp:127-165 / 274-430 on a structured grid.
 * Per step: every node's ionic update (cepo_step with the tissue stimulus
 * flag) at time t, then A V = B V* / dt by PCG. The S1 region is stimulated
 * while iia*bcl + t_crt < t < iia*bcl + t_crt + dur for pace iia < n_pace
 * (the "square" mesh rule, heart.cpp:309-323). Returns total CG iterations;
 * V (n) receives the final potential, iters_out (n_steps, may be NULL) the
 * iterations per step, t_act (n, may be NULL) the first step end at which
 * V >= act_thr (-1 if never). */
long cepo_tissue_run(int model, int dim, int nx, int ny, int nz, double h, const double *D, int n_d, double dt,
                     long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                     double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                     const double *celltype, double *V, int *iters_out, double act_thr, double *t_act) {
  return cepo_tissue_run_s2(model, dim, nx, ny, nz, h, D, n_d, dt, n_steps, s1, bcl, t_crt, dur, n_pace, conc, hill,
                            n_hill, rtol, precond_norm, celltype, V, iters_out, act_thr, t_act, 0, 0, 0.0, NULL, 0.0);
}

/* The same with an S1-S2 protocol (Cheart::apply_s2 / apply_ectopic,
 * heart.cpp:452-501, called before the node loop of every step of the last
 * S1 pace, heart.cpp:322-323): s2_kind 1 resets the region's nodes to their
 * initial states once node `target` has gone above thr and back below it;
 * s2_kind 2 instead drives the region with the S1 current (isEctopic) for
 * ecto_dur ms. After the protocol fires the S1 stimulus stays off (the
 * "square" mesh branch runs only while idid is false, heart.cpp:300). */
static long tissue_loop(int model, int n, const int *rp, const int *ci, const double *av, const double *bv, double dt,
                        long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                        double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                        const double *celltype, double *V, int *iters_out, double act_thr, double *t_act,
                        int s2_kind, int target, double thr, const unsigned char *region, double ecto_dur) {
  const int ns = cepo_n_states(model);
  cepo_cell *cells = malloc(sizeof(cepo_cell) * n);
  double *y = malloc(sizeof(double) * (size_t)n * CEPO_MAX_STATES);
  double *vs = malloc(sizeof(double) * n), *b = malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) {
    cepo_init(&cells[i], model, celltype ? celltype[i] : 0.0, conc, hill, n_hill, 0, celltype ? 0 : 1);
    cells[i].tissue_stim = 1;
    cepo_init_states(&cells[i], y + (size_t)i * CEPO_MAX_STATES);
  }
  double t = 0.0;
  long total = 0;
  if (t_act)
    for (int i = 0; i < n; ++i) t_act[i] = -1.0;
  double *y0 = NULL;  /* initial states, for the S2 reset */
  if (s2_kind == 1) {
    y0 = malloc(sizeof(double) * (size_t)n * CEPO_MAX_STATES);
    memcpy(y0, y, sizeof(double) * (size_t)n * CEPO_MAX_STATES);
  }
  int depol = 0, repol = 0, fired = 0, ecto = 0;
  double t_fire = 0.0;
  for (long st = 0; st < n_steps; ++st) {
    if (s2_kind && (int)(t / bcl) == n_pace - 1) {
      const double vt = y[(size_t)target * CEPO_MAX_STATES];
      if (vt > thr) depol = 1;
      if (depol && vt < thr) repol = 1;
      if (repol && !fired) {
        fired = 1;
        t_fire = t;
        if (s2_kind == 1)
          for (int i = 0; i < n; ++i)
            if (region[i]) memcpy(y + (size_t)i * CEPO_MAX_STATES, y0 + (size_t)i * CEPO_MAX_STATES, sizeof(double) * ns);
        if (s2_kind == 2) ecto = 1;
      }
      if (s2_kind == 2 && fired && t - t_fire > ecto_dur) ecto = 0;
    }
    const int iia = (int)(t / bcl);
    const int on = !fired && iia < n_pace && t < (double)iia * bcl + dur + t_crt && t > (double)iia * bcl + t_crt;
    for (int i = 0; i < n; ++i) {
      cells[i].is_s1 = (on && s1[i]) || (ecto && region[i]);
      cepo_step(&cells[i], t, dt, y + (size_t)i * CEPO_MAX_STATES, NULL);
      vs[i] = y[(size_t)i * CEPO_MAX_STATES];
    }
    cepo_spmv(n, rp, ci, bv, vs, b);
    for (int i = 0; i < n; ++i) b[i] /= dt;
    double rr;
    const int it = cepo_pcg2(n, rp, ci, av, b, vs, rtol, 10000, precond_norm, &rr);
    total += it < 0 ? -it : it;
    if (iters_out) iters_out[st] = it;
    for (int i = 0; i < n; ++i) y[(size_t)i * CEPO_MAX_STATES] = vs[i];
    t += dt;
    if (t_act)
      for (int i = 0; i < n; ++i)
        if (t_act[i] < 0.0 && vs[i] >= act_thr) t_act[i] = t;
  }
  (void)ns;
  for (int i = 0; i < n; ++i) V[i] = y[(size_t)i * CEPO_MAX_STATES];
  free(cells); free(y); free(vs); free(b); free(y0);
  return total;
}

long cepo_tissue_run_s2(int model, int dim, int nx, int ny, int nz, double h, const double *D, int n_d, double dt,
                        long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                        double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                        const double *celltype, double *V, int *iters_out, double act_thr, double *t_act,
                        int s2_kind, int target, double thr, const unsigned char *region, double ecto_dur) {
  if (dim == 2) nz = 1;
  const int n = nx * ny * nz;
  const long nnz = cepo_fem_nnz(dim, nx, ny, nz);
  int *rp = malloc(sizeof(int) * (n + 1)), *ci = malloc(sizeof(int) * nnz);
  double *av = malloc(sizeof(double) * nnz), *bv = malloc(sizeof(double) * nnz);
  cepo_fem_assemble(dim, nx, ny, nz, h, dt, D, n_d, rp, ci, av, bv);
  const long total = tissue_loop(model, n, rp, ci, av, bv, dt, n_steps, s1, bcl, t_crt, dur, n_pace, conc, hill,
                                 n_hill, rtol, precond_norm, celltype, V, iters_out, act_thr, t_act, s2_kind, target,
                                 thr, region, ecto_dur);
  free(rp); free(ci); free(av); free(bv);
  return total;
}

/* The Godunov tissue loop on a caller's CSR operator (any mesh). */
long cepo_tissue_run_csr(int model, int n, const int *rp, const int *ci, const double *av, const double *bv, double dt,
                         long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                         double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                         const double *celltype, double *V, int *iters_out, double act_thr, double *t_act) {
  return tissue_loop(model, n, rp, ci, av, bv, dt, n_steps, s1, bcl, t_crt, dur, n_pace, conc, hill, n_hill, rtol,
                     precond_norm, celltype, V, iters_out, act_thr, t_act, 0, 0, 0.0, NULL, 0.0);
}

/* ---- unstructured P1 tetrahedra (fem.cpp:209-229 Gauss points,
 * 342-373 shape functions, 628-661 element matrices) ---- */

/* Row la of the element matrices of tetrahedron x[4][3] (cepo_element,
 * kind 2; D scalar (n_d 1) or xx,xy,xz,yy,yz,zz (6)). */
void cepo_tet_row(const double x[4][3], const double *D, int n_d, double dt, int la, double *arow, double *brow) {
  double Ae[16], Be[16];
  cepo_element(2, &x[0][0], D, n_d, dt, Ae, Be);
  for (int k = 0; k < 4; ++k) {
    arow[k] = Ae[la * 4 + k];
    brow[k] = Be[la * 4 + k];
  }
}

/* CSR of a tetrahedral mesh: columns of row i = the nodes sharing an element
 * with i, ascending; each row sums its incident elements in ascending
 * element order, local nodes in order. row_ptr must hold n_nodes + 1
 * entries; col/a/b the returned nnz (call with col == NULL to count). */
long cepo_fem_assemble_tet(int n_nodes, const double *xyz, int n_elem, const int *conn, const double *D, int n_d,
                           double dt, int *row_ptr, int *col, double *a, double *b) {
  /* incidence, node -> (element, local) in ascending element order */
  int *cnt = calloc((size_t)n_nodes + 1, sizeof(int));
  for (long e = 0; e < n_elem; ++e)
    for (int k = 0; k < 4; ++k) cnt[conn[4 * e + k] + 1]++;
  for (int i = 0; i < n_nodes; ++i) cnt[i + 1] += cnt[i];
  int *fill = calloc((size_t)n_nodes, sizeof(int));
  int *inc = malloc(sizeof(int) * 2 * (size_t)cnt[n_nodes]);
  for (long e = 0; e < n_elem; ++e)
    for (int k = 0; k < 4; ++k) {
      const int i = conn[4 * e + k];
      const int p = cnt[i] + fill[i]++;
      inc[2 * p] = (int)e;
      inc[2 * p + 1] = k;
    }
  /* sparsity */
  long nnz = 0;
  int *nb = malloc(sizeof(int) * 64);
  for (int i = 0; i < n_nodes; ++i) {
    int m = 0;
    for (int p = cnt[i]; p < cnt[i + 1]; ++p)
      for (int k = 0; k < 4; ++k) {
        const int j = conn[4 * inc[2 * p] + k];
        int seen = 0;
        for (int q = 0; q < m; ++q) seen |= nb[q] == j;
        if (!seen) {
          if (m % 64 == 0 && m) nb = realloc(nb, sizeof(int) * (size_t)(m + 64));
          nb[m++] = j;
        }
      }
    for (int u = 1; u < m; ++u)  /* insertion sort */
      for (int v = u; v > 0 && nb[v - 1] > nb[v]; --v) { const int tmp = nb[v]; nb[v] = nb[v - 1]; nb[v - 1] = tmp; }
    if (row_ptr) row_ptr[i] = (int)nnz;
    if (col) {
      for (int q = 0; q < m; ++q) { col[nnz + q] = nb[q]; a[nnz + q] = 0.; b[nnz + q] = 0.; }
      for (int p = cnt[i]; p < cnt[i + 1]; ++p) {
        const int e = inc[2 * p], la = inc[2 * p + 1];
        double x[4][3], ar[4], br[4];
        for (int k = 0; k < 4; ++k)
          for (int c = 0; c < 3; ++c) x[k][c] = xyz[3 * (long)conn[4 * e + k] + c];
        cepo_tet_row(x, D + (long)e * n_d, n_d, dt, la, ar, br);
        for (int k = 0; k < 4; ++k) {
          const int j = conn[4 * e + k];
          int q = 0;
          while (col[nnz + q] != j) ++q;
          a[nnz + q] += ar[k];
          b[nnz + q] += br[k];
        }
      }
    }
    nnz += m;
  }
  if (row_ptr) row_ptr[n_nodes] = (int)nnz;
  free(cnt); free(fill); free(inc); free(nb);
  return nnz;
}
