// Homogenization.h -- stand-in for topoOptLib's Homogenization<3>
// (fast_fem/FEM3DFun.hpp:7, used at fast_fem/FEM3DFun.cpp:154,160).  TEST
// INFRASTRUCTURE ONLY.  Homogenize() solves the six periodic unit-strain load
// cases on the coefficient field that FEM3DFun::setParam wrote, with the
// oracle's FP64 multigrid PCG (oracle/femh_oracle_mg.c) to a relative residual
// of 1e-12, and hands back what fast_fem reads: unit_test_u[i] = the total
// displacement eps^i x + chi^i on the n^3 periodic nodes (index
// 3 (i n^2 + j n + k) + d, as copyPeriodicU reads it, FEM3DFun.cpp:31-56) and
// unit_test_strains[i] = the unit macro strain (Voigt xx,yy,zz,yz,xz,xy,
// engineering shear: tensor entries 1/2).
#ifndef FEMH_REF_SHIM_HOMOGENIZATION_H
#define FEMH_REF_SHIM_HOMOGENIZATION_H
#include <vector>

#include <Eigen/Dense>

#include "ElasticHexFEM.h"
#include "femh_oracle.h"

template <int d>
struct Homogenization {
  ElasticHexFEM<d>& fem;
  std::vector<Eigen::VectorXd> unit_test_u;
  std::vector<Eigen::Matrix3d> unit_test_strains;
  int status = -1;
  explicit Homogenization(ElasticHexFEM<d>& f) : fem(f) {}
  void Initialize() {}
  void Homogenize() {
    const Field<T, d>& c = *fem.variable_coef;
    const int n0 = c.n[0], n1 = c.n[1], n2 = c.n[2];
    const long nv = (long)n0 * n1 * n2;
    // coefficient field as densities of the linear law c(rho) = rho
    fo_material lin = {0, 1.0, 0.0, 1.0, fem.nu, 1.0, 0.0};
    std::vector<double> chi(18 * nv);
    double C[36], rel[6];
    int it[6];
    status = fo_mg_homogenize(n0, n1, n2, fem.lattice.dx, c.a.data(), &lin, 1e-12, 100000, 3, 3, 64.0, 64, C,
                              chi.data(), it, rel);
    unit_test_u.assign(6, Eigen::VectorXd::Zero(3 * nv));
    unit_test_strains.assign(6, Eigen::Matrix3d::Zero());
    for (int I = 0; I < 6; ++I) {
      Eigen::Matrix3d& e = unit_test_strains[I];
      if (I < 3) e(I, I) = 1.0;
      else {
        const int a = I == 3 ? 1 : 0, b = I == 5 ? 1 : 2;
        e(a, b) = e(b, a) = 0.5;
      }
      for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j)
          for (int k = 0; k < n2; ++k) {
            const long node = ((long)i * n1 + j) * n2 + k;
            const Eigen::Vector3d X(i * fem.lattice.dx, j * fem.lattice.dx, k * fem.lattice.dx);
            const Eigen::Vector3d y = e * X;
            for (int q = 0; q < 3; ++q) unit_test_u[I][3 * node + q] = y[q] + chi[(long)I * 3 * nv + 3 * node + q];
          }
    }
  }
};
#endif
