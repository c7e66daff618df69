/* TEST INFRASTRUCTURE: exercises every entry point of the CPU oracle once on
 * small cases so that a build with -fsanitize=address,undefined reports any
 * out-of-bounds access, use of freed memory, leak or undefined arithmetic in
 * the host code that checks the device kernels. Prints "ok" and exits 0 when
 * nothing was reported (the sanitizers abort otherwise). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../oracle/src/cep_oracle.h"

static void fail(const char *what) {
  fprintf(stderr, "oracle check failed: %s\n", what);
  exit(2);
}

static void models(void) {
  double hill[CEPO_MAX_HILL];
  for (int k = 0; k < 14; ++k) hill[k] = (k % 2) ? 1.0 : 5.0 + k;
  hill[14] = 2e4; hill[15] = 1e-3; hill[16] = 0.9; hill[17] = 1e4; hill[18] = -50.0; hill[19] = 3.5e-5;
  for (int model = 0; model < 5; ++model) {
    cepo_cell c;
    if (cepo_init(&c, model, 1.0, 0.5, hill, 20, 1, 1) != 0) fail("init");
    cepo_set_pacing(&c, 300.0, -1.0, -1.0, 1.0);
    double y[CEPO_MAX_STATES], dy[CEPO_MAX_STATES];
    cepo_init_states(&c, y);
    cepo_currents cur;
    cepo_rates(&c, 0.0, y, dy, &cur);
    double t = 0.0, vt[64];
    cepo_run(&c, &t, 0.01, 3000, y, vt, 50);
    if (!isfinite(y[0])) fail("run");
    cepo_biomarkers bm;
    cepo_init_states(&c, y);
    double vt2[4096];
    if (cepo_run_biomarkers(&c, y, 0.01, 2, 1, 1.0, -1e300, &bm, vt2, 20, 4096) != 0) fail("biomarkers");
    double v[500], out[500];
    for (int k = 0; k < 500; ++k) v[k] = k < 100 ? -85.0 : 10.0;
    cepo_clamp(&c, y, v, 500, 0.0, 0.01, 3, out);
  }
  double ct[3] = {0, 1, 2}, conc[3] = {0, 1, 2}, rows[3 * 14];
  for (int k = 0; k < 42; ++k) rows[k] = (k % 2) ? 1.0 : 3.0;
  double states[3 * CEPO_MAX_STATES];
  cepo_run_batch(CEPO_ORD2011, 3, ct, conc, rows, 14, 0, 1, 1000.0, 0.005, 2000, states, 2);
  cepo_cell c;
  cepo_init(&c, CEPO_TT2004, 0.0, 0.0, NULL, 0, 0, 1);
  cepo_tt04_mcell(&c, 0.0, NULL);
  double y[CEPO_MAX_STATES];
  cepo_init_states(&c, y);
  const double bcls[2] = {300.0, 250.0};
  cepo_apdr_record rec[16];
  int n_rec = 0;
  if (cepo_restitution(&c, y, bcls, 2, 4, 0.02, rec, 16, &n_rec) != 0 || n_rec != 4) fail("restitution");
}

static void fem(void) {
  for (int dim = 2; dim <= 3; ++dim) {
    const int nx = dim == 2 ? 8 : 5, ny = dim == 2 ? 7 : 4, nz = dim == 2 ? 1 : 3;
    const int n = nx * ny * nz, ne = (nx - 1) * (ny - 1) * (dim == 3 ? nz - 1 : 1), nd = dim == 2 ? 3 : 6;
    const long nnz = cepo_fem_nnz(dim, nx, ny, nz);
    int *rp = malloc(sizeof(int) * (size_t)(n + 1)), *ci = malloc(sizeof(int) * (size_t)nnz);
    double *a = malloc(sizeof(double) * (size_t)nnz), *b = malloc(sizeof(double) * (size_t)nnz);
    double *D = malloc(sizeof(double) * (size_t)ne * nd);
    for (int e = 0; e < ne; ++e)
      for (int k = 0; k < nd; ++k) D[e * nd + k] = (k == 0 || k == (dim == 2 ? 2 : 3) || k == 5) ? 0.0013 : 0.0002;
    if (cepo_fem_assemble(dim, nx, ny, nz, 0.025, 0.01, D, nd, rp, ci, a, b) != 0) fail("assemble");
    double *x = calloc((size_t)n, sizeof(double)), *rhs = malloc(sizeof(double) * (size_t)n), res = 0;
    for (int i = 0; i < n; ++i) x[i] = sin(0.3 * i);
    cepo_spmv(n, rp, ci, b, x, rhs);
    memset(x, 0, sizeof(double) * (size_t)n);
    if (cepo_pcg2(n, rp, ci, a, rhs, x, 1e-10, 1000, 1, &res) <= 0) fail("pcg");
    double Ae[64], Be[64], el[6] = {0.1, 0.2, 0.3, 0.4, 0.5, 0.6}, phi[2];
    cepo_fem_element(dim, 0.025, 0.01, D, nd, Ae, Be);
    cepo_pseudo_ecg(dim, nx, ny, nz, 0.025, D, nd, x, 2, el, phi);
    unsigned char *s1 = calloc((size_t)n, 1), *region = calloc((size_t)n, 1);
    s1[0] = s1[1] = 1;
    region[n - 1] = 1;
    double *V = malloc(sizeof(double) * (size_t)n), *tact = malloc(sizeof(double) * (size_t)n);
    int iters[200];  /* one per step */
    double hill[14] = {0};
    cepo_tissue_run(CEPO_TT2006, dim, nx, ny, nz, 0.025, D, nd, 0.01, 200, s1, 1000.0, 0.0, 1.0, 1, 0.0, hill, 14,
                    1e-8, 1, NULL, V, iters, -30.0, tact);
    cepo_tissue_run_s2(CEPO_TT2006, dim, nx, ny, nz, 0.025, D, nd, 0.01, 200, s1, 100.0, 0.0, 1.0, 2, 0.0, hill, 14,
                       1e-8, 1, NULL, V, iters, -30.0, tact, 2, n - 1, -45.0, region, 2.0);
    cepo_tissue_run_csr(CEPO_TT2006, n, rp, ci, a, b, 0.01, 100, s1, 1000.0, 0.0, 1.0, 1, 0.0, hill, 14, 1e-8, 1,
                        NULL, V, iters, -30.0, tact);
    free(rp); free(ci); free(a); free(b); free(D); free(x); free(rhs); free(s1); free(region); free(V); free(tact);
  }
  /* two tetrahedra sharing a face */
  const double xyz[5 * 3] = {0, 0, 0, 0.1, 0, 0, 0, 0.1, 0, 0, 0, 0.1, 0.1, 0.1, 0.1};
  const int conn[2 * 4] = {0, 1, 2, 3, 1, 2, 3, 4};
  const double Dt[2] = {0.0013, 0.0013};  /* one per element */
  const long nnz = cepo_fem_assemble_tet(5, xyz, 2, conn, Dt, 1, 0.01, NULL, NULL, NULL, NULL);
  int rp[6], *ci = malloc(sizeof(int) * (size_t)nnz);
  double *a = malloc(sizeof(double) * (size_t)nnz), *b = malloc(sizeof(double) * (size_t)nnz);
  if (cepo_fem_assemble_tet(5, xyz, 2, conn, Dt, 1, 0.01, rp, ci, a, b) != nnz) fail("tet");
  free(ci); free(a); free(b);
}

int main(void) {
  models();
  fem();
  printf("ok\n");
  return 0;
}
