/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * C-ABI access to the reference's FEM element routines, compiled unmodified
 * from the reference's fem.cpp (with the inert PETSc stand-ins of
 * ref_shim/petsc and the reference's CEPCell_NEO/modules/globals.cpp): for
 * one element of a given type and node coordinates, the reference's own
 * set_gpt / set_Phi_dPhiS (fem.cpp:830-860) and set_amat_bmat
 * (fem.cpp:628-661) produce the element matrices amat (M/dt + DE K) and
 * bmat (M). The tests pin the oracle's element arithmetic to these.
 */
#include <cstring>

#include "fem.h"

/* Cmesh's constructor (mesh.cpp) reads an .inp file; the shim fills the
 * one-element mesh itself. */
Cmesh::Cmesh(char *) {}
cCalcException::cCalcException(const char *) {}

namespace {
/* The reference allocates dPhiX2 as [node][node][dimension]
 * (fem.cpp:141-147) but set_amat_bmat fills and reads it as a [node][node]
 * matrix per Gauss point (fem.cpp:647,658): each row gets `node` values in
 * room for `dimension`. With glibc's allocator the extra values land in the
 * slack and the headers of neighbouring chunks (ASan: heap-buffer-overflow
 * at fem.cpp:611; glibc aborts later with "corrupted size"), and for hex
 * elements (8 nodes, 3 dimensions) a row's overflow reaches the next row's
 * storage. The shim gives every row the `node` values the arithmetic uses,
 * so the element matrices are the ones the code means, deterministically. */
class PinFem : public Cfem {
 public:
  explicit PinFem(Cmesh *m) : Cfem(m) {
    for (int g = 0; g < m->node; ++g)
      for (int i = 0; i < m->node; ++i) {
        delete[] dPhiX2[g][i];
        dPhiX2[g][i] = new double[m->node];
      }
  }
  int processing(int, char **, param_t) { return 0; }
  void writeVTK() {}
  void writeoutput() {}
  double **amat_rows() { return amat; }
  double **bmat_rows() { return bmat; }
};
}  // namespace

extern "C" {

/* type: "square" (dim 2, 4 nodes), "hex" (dim 3, 8 nodes) or "tet" (dim 3,
 * 4 nodes); xy: the element's node coordinates [nn][dim] in the
 * reference's local node order; de: the element's scalar conductivity DE;
 * ae, be: [nn][nn] row-major outputs. Returns 0, or -1 for an unknown
 * type. */
int ref_fem_element(const char *type, const double *xy, double de, double dt, double *ae, double *be) {
  int dim, nn;
  if (!std::strcmp(type, "square")) { dim = 2; nn = 4; }
  else if (!std::strcmp(type, "hex")) { dim = 3; nn = 8; }
  else if (!std::strcmp(type, "tet")) { dim = 3; nn = 4; }
  else return -1;
  Cmesh m((char *)"");
  m.dimension = dim;
  std::strcpy(m.type, type);
  m.node = nn;
  m.all_nodes = nn;
  m.all_elements = 1;
  m.XY = new double *[nn];
  m.EC = new int *[1];
  m.EC[0] = new int[nn];
  for (int a = 0; a < nn; ++a) {
    m.XY[a] = new double[dim];
    for (int d = 0; d < dim; ++d) m.XY[a][d] = xy[a * dim + d];
    m.EC[0][a] = a;
  }
  PinFem f(&m);
  f.set_gpt();
  f.set_Phi_dPhiS();
  f.DE[0] = de;
  f.set_amat_bmat(0, dt, f.amat_rows(), f.bmat_rows());
  for (int j = 0; j < nn; ++j)
    for (int k = 0; k < nn; ++k) {
      ae[j * nn + k] = f.amat_rows()[j][k];
      be[j * nn + k] = f.bmat_rows()[j][k];
    }
  return 0;
}

}  // extern "C"
