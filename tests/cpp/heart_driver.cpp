// A heart.cpp-style tissue driver written against the C ABI alone: the
// reference's Cheart set-up (a "square" mesh, one TT2006 cell per node, the
// drug as a Hill row, the corner S1 nodes, an ECG electrode) and its time
// loop (cellular_reaction, then solve_Bmat, every step), with every status
// checked where the reference would exit(). Prints the final V of every
// node, then the activation times, then the electrode's last ECG value, one
// value per line.
//   heart_driver <nx> <ny> <n_steps> <conc> <ic50_kr> <h_kr>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cep_b200.h"

static void check(int rc, const char *what) {
  if (rc != CEP_OK) {
    std::fprintf(stderr, "%s: %s\n", what, cep_last_error());
    std::exit(1);
  }
}

int main(int argc, char **argv) {
  if (argc < 7) return 2;
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]);
  const long n_steps = std::atol(argv[3]);
  const double conc = std::atof(argv[4]);
  const int n = nx * ny;
  const double h = 0.025, dt = 0.01, D = 0.0013;
  // cells: one TT2006 epi cell per node with the IKr Hill pair (columns 12, 13)
  cep_batch_t cells = nullptr;
  check(cep_batch_create(CEP_MODEL_TT2006, n, CEP_PREC_FP64, nullptr, &cells), "cep_batch_create");
  std::vector<double> c(n, conc), hill((size_t)n * 14, 0.0);
  for (int i = 0; i < n; ++i) {
    hill[(size_t)i * 14 + 12] = std::atof(argv[5]);
    hill[(size_t)i * 14 + 13] = std::atof(argv[6]);
  }
  check(cep_batch_init(cells, nullptr, c.data(), hill.data(), 14, CEP_FLAG_QUIRKS), "cep_batch_init");
  // Cfem: the square mesh's operator, scalar conductivity per element
  std::vector<double> De((size_t)(nx - 1) * (ny - 1), D);
  cep_fem_t fem = nullptr;
  check(cep_fem_create_grid(2, nx, ny, 1, h, dt, De.data(), 1, CEP_FEM_AUTO, nullptr, &fem), "cep_fem_create_grid");
  check(cep_fem_set_solver(fem, 1e-10, 10000, 1), "cep_fem_set_solver");
  // Cheart: S1 on the first two columns, one pace at BCL 1000 ms, 1 ms
  cep_tissue_t heart = nullptr;
  check(cep_tissue_create(cells, fem, dt, &heart), "cep_tissue_create");
  std::vector<unsigned char> s1(n, 0);
  for (int y = 0; y < ny; ++y) s1[(size_t)y * nx] = s1[(size_t)y * nx + 1] = 1;
  check(cep_tissue_set_stimulus(heart, s1.data(), 1000.0, 0.0, 1.0, 1), "cep_tissue_set_stimulus");
  const double electrode[3] = {0.5 * (nx - 1) * h, -0.5, 1.0};
  check(cep_tissue_set_electrodes(heart, 1, electrode, 1, n_steps), "cep_tissue_set_electrodes");
  check(cep_tissue_run(heart, n_steps), "cep_tissue_run");
  check(cep_tissue_sync(heart), "cep_tissue_sync");
  std::vector<double> v(n), t_act(n), ecg((size_t)n_steps);
  long n_rec = 0;
  check(cep_tissue_get_v(heart, v.data()), "cep_tissue_get_v");
  check(cep_tissue_get_activation(heart, t_act.data()), "cep_tissue_get_activation");
  check(cep_tissue_get_ecg(heart, ecg.data(), &n_rec), "cep_tissue_get_ecg");
  for (double x : v) std::printf("%.17g\n", x);
  for (double x : t_act) std::printf("%.17g\n", x);
  std::printf("%.17g\n", n_rec > 0 ? ecg[(size_t)n_rec - 1] : 0.0);
  cep_tissue_destroy(heart);
  cep_fem_destroy(fem);
  cep_batch_destroy(cells);
  return 0;
}
