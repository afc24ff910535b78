// femlib_k0.cpp -- C entry point into the reference's own femlib element code
// (compiled from the reference sources by oracle/build_ref.sh into
// oracle/_ref/libfemlib_ref.so; TEST INFRASTRUCTURE ONLY).
//
// femlib_k0(E, nu, K): stiffness of the unit hex8 element of a 1x1x1
// ElementRegGrid with a MaterialQuad(StrainLin) material, exactly as the
// reference assembles it (femlib/src/MaterialQuad.cpp:68-105, ElementHex.cpp,
// StrainLin.cpp:29-37, Quadrature.cpp Gauss2), built in FP64
// (USE_DOUBLE_FOR_SCALAR).  Output: row-major 24x24 in femlib's vertex order.
#include "ElementRegGrid.hpp"
#include "Element.hpp"
#include "MaterialQuad.hpp"
#include "StrainLin.hpp"

extern "C" int femlib_k0(double E, double nu, double* K) {
  ElementRegGrid grid(1, 1, 1);
  StrainLin ene;
  const double mu = E / (2.0 * (1.0 + nu));
  const double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  ene.param[0] = mu;
  ene.param[1] = lambda;
  MaterialQuad mat(&ene);
  grid.m.clear();
  grid.addMaterial(&mat);
  for (auto& me : grid.me) me = 0;
  mat.init(&grid);
  MatrixXS Ke = mat.getStiffness(grid.e[0], &grid);
  if (Ke.rows() != 24 || Ke.cols() != 24) return 1;
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) K[i * 24 + j] = (double)Ke(i, j);
  return 0;
}
