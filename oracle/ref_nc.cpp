// ref_nc.cpp -- C entry into the reference's own force-driven coarsening,
// NumericalCoarsening::computeCoarsenedElasticityTensorAndParameters3D
// (SamplesGenerator/NumericalCoarsening.cpp:266-340), compiled from the
// reference sources in place by oracle/build_ref.sh into
// oracle/_ref/libnc_ref.so together with femlib, Utilities, StepperCPU's
// Newton stepper and oracle/ref_shim/pardiso_eigen.cpp (Eigen's sparse LU in
// place of the absent PARDISO).  TEST INFRASTRUCTURE ONLY.
//
// Built as the reference ships it: cfgScalar = float (Utilities/include/cfgDefs.h),
// the 1 + 1e-5 diagonal scaling of NumericalCoarsening.cpp:1278 included.
//
// ref_nc_coarsen3d: nx*ny*nz material indices (voxel (i*ny + j)*nz + k), nmat
// base materials (E, nu) with their densities, structure type (0 General,
// 1 Cubic, 2 Orthotropic); writes the 21 appended tensor values and the
// appended parameters (4 for Cubic, 10 otherwise), returns their count or < 0.
#include <vector>

#include "ElementRegGrid.hpp"
#include "MaterialQuad.hpp"
#include "NumericalCoarsening.h"
#include "StrainLin.hpp"

extern "C" int ref_nc_coarsen3d(int nx, int ny, int nz, const int* materials, int nmat, const double* E,
                                const double* nu, const double* densities, int type, double* tensor21,
                                double* params) {
  if (nx < 1 || ny < 1 || nz < 1 || nmat < 1) return -1;
  std::vector<StrainLin> ene(nmat);
  for (int m = 0; m < nmat; ++m) {
    ene[m].param[0] = (cfgScalar)(E[m] / (2.0 * (1.0 + nu[m])));                          // mu
    ene[m].param[1] = (cfgScalar)(E[m] * nu[m] / ((1.0 + nu[m]) * (1.0 - 2.0 * nu[m])));  // lambda
  }
  std::vector<MaterialQuad> mats;
  for (int m = 0; m < nmat; ++m) mats.push_back(MaterialQuad(&ene[m]));
  int N[3] = {nx, ny, nz};
  NumericalCoarsening nc;
  nc.init(N, 1, 1, mats);
  std::vector<int> cellMaterials(materials, materials + (long)nx * ny * nz);
  std::vector<cfgScalar> dens(densities, densities + nmat);
  std::vector<cfgScalar> tv, pv;
  nc.computeCoarsenedElasticityTensorAndParameters3D(cellMaterials, N, dens,
                                                     (NumericalCoarsening::StructureType)type, tv, pv);
  if (tv.size() != 21) return -2;
  for (int i = 0; i < 21; ++i) tensor21[i] = tv[i];
  for (size_t i = 0; i < pv.size(); ++i) params[i] = pv[i];
  return (int)pv.size();
}
