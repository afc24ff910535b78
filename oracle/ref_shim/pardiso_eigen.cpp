// pardiso_eigen.cpp -- the PARDISO entry points the reference declares in
// StepperCPU/include/pardiso_sym.hpp (and the two of SparseLin.hpp), written
// over the reference's vendored Eigen 3.2.2 sparse LU because the PARDISO
// library is not in the tree (StepperCPU/src/pardiso_sym.cpp:23-30 compiles
// them only with PARDISO_AVAILABLE).  TEST INFRASTRUCTURE ONLY: it lets
// oracle/build_ref.sh link the reference's NumericalCoarsening into
// oracle/_ref/libnc_ref.so.
//
// Same contract as the reference's PARDISO wrapper for mtype -2 (real
// symmetric, indefinite: the periodic-jump and rigid-motion multiplier rows
// of femlib's system, femlib/src/EMeshStiffness.cpp:53-274): ia/ja are the
// 1-based CSR pattern of the upper triangle (NumericalCoarsening.cpp:97-102),
// val its values; the factorisation lives in state->pt[0] between
// pardisoNumericalFactorize and pardisoFree.
#include <cstdio>
#include <vector>

#include <Eigen/Sparse>
#include <Eigen/SparseLU>

#include "SparseLin.hpp"
#include "pardiso_sym.hpp"

namespace {
typedef Eigen::SparseMatrix<double> SpMat;
typedef Eigen::SparseLU<SpMat, Eigen::COLAMDOrdering<int> > LU;

SpMat full_from_upper(const int* ia, const int* ja, const double* val, int n) {
  std::vector<Eigen::Triplet<double> > t;
  t.reserve(2 * (ia[n] - 1));
  for (int i = 0; i < n; ++i)
    for (int p = ia[i] - 1; p < ia[i + 1] - 1; ++p) {
      const int j = ja[p] - 1;
      t.push_back(Eigen::Triplet<double>(i, j, val[p]));
      if (j != i) t.push_back(Eigen::Triplet<double>(j, i, val[p]));
    }
  SpMat A(n, n);
  A.setFromTriplets(t.begin(), t.end());
  A.makeCompressed();
  return A;
}
}  // namespace

void pardisoInit(PardisoState* state) {
  for (int i = 0; i < 64; ++i) state->pt[i] = 0;
  state->mtype = -2;
}

int pardisoSymbolicFactorize(int*, int*, int, PardisoState*) { return 0; }

int pardisoNumericalFactorize(int* ia, int* ja, double* val, int n, PardisoState* state) {
  delete static_cast<LU*>(state->pt[0]);
  LU* lu = new LU();
  SpMat A = full_from_upper(ia, ja, val, n);
  lu->analyzePattern(A);
  lu->factorize(A);
  state->pt[0] = lu;
  if (lu->info() != Eigen::Success) {
    std::fprintf(stderr, "pardiso_eigen: factorisation failed\n");
    return 1;
  }
  return 0;
}

int pardisoBackSubstitute(int*, int*, double*, int n, double* x, double* b, PardisoState* state) {
  LU* lu = static_cast<LU*>(state->pt[0]);
  if (!lu) return 1;
  Eigen::Map<Eigen::VectorXd> bv(b, n), xv(x, n);
  xv = lu->solve(bv);
  return lu->info() == Eigen::Success ? 0 : 1;
}

int pardisoSolve(int* ia, int* ja, double* val, int n, double* x, double* b, PardisoState* state) {
  const int e = pardisoNumericalFactorize(ia, ja, val, n, state);
  return e ? e : pardisoBackSubstitute(ia, ja, val, n, x, b, state);
}

void pardisoFree(int*, int*, int, PardisoState* state) {
  delete static_cast<LU*>(state->pt[0]);
  state->pt[0] = 0;
}

void sparseInit() {}

int sparseSolve(int* ia, int* ja, double* val, int n, double* x, double* b) {
  PardisoState s;
  pardisoInit(&s);
  const int e = pardisoSolve(ia, ja, val, n, x, b, &s);
  pardisoFree(ia, ja, n, &s);
  return e;
}
