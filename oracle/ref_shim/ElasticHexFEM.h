// ElasticHexFEM.h -- stand-in for the topoOptLib header that fast_fem includes
// (fast_fem/FEM3DFun.hpp:6; the library itself is absent from the reference
// tree: SamplesGenerator/CMakeLists.txt:57, ReadMe.txt:9-19).  TEST
// INFRASTRUCTURE ONLY: it declares exactly the members, types and helpers that
// fast_fem/FEM3DFun.cpp uses, so that the reference's own setParam energy loop,
// f, df and field chain rule compile unchanged (oracle/build_ref.sh).  The
// solve behind Homogenize() is the oracle's (Homogenization.h).
#ifndef FEMH_REF_SHIM_ELASTIC_HEX_FEM_H
#define FEMH_REF_SHIM_ELASTIC_HEX_FEM_H
#include <vector>

#include <Eigen/Dense>

typedef double T;
typedef Eigen::VectorXd VectorX;
#define Type_Define_VectorD_Outside_Class(d) typedef Eigen::Matrix<double, d, 1> VectorD
#define Type_Define_VectorDi_Outside_Class(d) typedef Eigen::Matrix<int, d, 1> VectorDi
#define Type_Define_MatrixD_Outside_Class(d) typedef Eigen::Matrix<double, d, d> MatrixD

template <class S>
inline S Clamp(const S& x, const S& lo, const S& hi) {
  return x < lo ? lo : (hi < x ? hi : x);
}

template <int d>
struct Lattice {
  double dx = 1.0;   // voxel edge
};

// per-voxel scalar field, x slowest
template <class S, int d>
struct Field {
  int n[3] = {0, 0, 0};
  std::vector<S> a;
  void Resize(const Eigen::Vector3i& s) {
    for (int i = 0; i < 3; ++i) n[i] = s[i];
    a.assign((size_t)n[0] * n[1] * n[2], S(0));
  }
  void Fill(const S& v) { std::fill(a.begin(), a.end(), v); }
  S& operator()(int i, int j, int k) { return a[((size_t)i * n[1] + j) * n[2] + k]; }
};

template <int d>
struct ElasticHexFEM {
  Lattice<d> lattice;
  Field<T, d>* variable_coef = nullptr;   // per-voxel stiffness multiplier (setParam writes femCoef)
  Eigen::VectorXd u, f;
  std::vector<int> psi_D, nodal_forces;
  Eigen::MatrixXd Ke;                      // element stiffness of a voxel (edge lattice.dx)
  double nu = 0.3;                         // Poisson ratio of the base material (stand-in only)
  void Update_Matrices() {}
};
#endif
