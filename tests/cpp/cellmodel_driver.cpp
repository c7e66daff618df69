// A reference-style driver written against the Cellmodel members: the
// explicit loop of the reference's fixed-step benches (computeRates(t);
// solveAnalytical(dt); t += dt) on cep::Cellmodel. Prints V every `stride`
// steps, one value per line.
//   cellmodel_driver ord <n_steps> <stride> <bcl>
//   cellmodel_driver cipa_rates <n_steps> <stride> <bcl>
//   cellmodel_driver tt06_tissue <n_on> <n_off> <stride>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "cep_cellmodel.hpp"

int main(int argc, char **argv) {
  if (argc < 5) return 2;
  try {
    if (!std::strcmp(argv[1], "ord")) {
      const long n = std::atol(argv[2]), stride = std::atol(argv[3]);
      cep::Cellmodel *p_cell = new cep::Cellmodel(CEP_MODEL_ORD2011);
      double hill[14] = {1.5, 0.9, 20.0, 1.1, 0, 0, 3.0, 1.3, 5.0, 0.8, 12.0, 1.0, 0.7, 1.2};
      p_cell->initConsts(0.0, 0.4, hill, false);
      p_cell->CONSTANTS[140] = std::atof(argv[4]);  // CONSTANTS[BCL], as the benches set it
      double t = 0.0, dt = 0.005;
      for (long k = 1; k <= n; ++k) {
        p_cell->computeRates(t, p_cell->CONSTANTS, p_cell->RATES, p_cell->STATES, p_cell->ALGEBRAIC);
        p_cell->solveAnalytical(dt);
        t += dt;
        if (k % stride == 0) std::printf("%.17g\n", p_cell->STATES[0]);
      }
      delete p_cell;
    } else if (!std::strcmp(argv[1], "cipa_rates")) {
      // CiPA-ORd with a drug, the bench's call-site writes (CONSTANTS[BCL],
      // CONSTANTS[GNa] *= gna_scale: cipa_drug_bench.cpp:146-148), the
      // explicit loop; every `stride` steps one line: STATES then RATES.
      const long n = std::atol(argv[2]), stride = std::atol(argv[3]);
      cep::Cellmodel cell(CEP_MODEL_CIPA2017);
      double hill[20] = {1.5, 0.9, 20.0, 1.1, 0, 0, 3.0, 1.3, 5.0, 0.8, 12.0, 1.0, 0, 0,
                         5e3, 2e-3, 0.9, 1e4, -40.0, 3.5e-5};
      cell.initConsts(0.0, 0.4, hill);
      cell.CONSTANTS[15] = std::atof(argv[4]);  // CONSTANTS[BCL]
      cell.CONSTANTS[45] *= 0.7;                // CONSTANTS[GNa] *= gna_scale
      double t = 0.0, dt = 0.005;
      for (long k = 1; k <= n; ++k) {
        cell.computeRates(t, cell.CONSTANTS, cell.RATES, cell.STATES, cell.ALGEBRAIC);
        if (k % stride == 0) {
          for (int q = 0; q < cell.states_size; ++q) std::printf("%.17g ", cell.STATES[q]);
          for (int q = 0; q < cell.states_size; ++q) std::printf("%.17g ", cell.RATES[q]);
          std::printf("%.17g\n", t);
        }
        cell.solveAnalytical(dt);
        t += dt;
      }
    } else if (!std::strcmp(argv[1], "tt06_tissue")) {
      const long n_on = std::atol(argv[2]), n_off = std::atol(argv[3]), stride = std::atol(argv[4]);
      cep::Cellmodel cell(CEP_MODEL_TT2006, CEP_PREC_FP64, true);
      cell.initConsts();
      double t = 0.0, dt = 0.01;
      for (long k = 1; k <= n_on + n_off; ++k) {
        cell.isS1 = k <= n_on;
        cell.computeRates(t, cell.CONSTANTS, cell.RATES, cell.STATES, cell.ALGEBRAIC);
        cell.solveAnalytical(dt);
        t += dt;
        if (k % stride == 0) std::printf("%.17g\n", cell.STATES[0]);
      }
    } else {
      return 2;
    }
  } catch (const cep::Error &e) {
    std::fprintf(stderr, "cep error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
