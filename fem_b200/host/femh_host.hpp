// femh_host.hpp -- C++ host layer over the C ABI (include/femh.h) that mirrors
// the reference's homogenization interfaces, so reference callers switch by
// relinking:
//   - RealFun / RealField / PiecewiseConstant3D / FEM3DFun
//       (fast_fem/RealFun.hpp:13-50, fast_fem/RealField.hpp, fast_fem/PiecewiseConstant3D.cpp,
//        fast_fem/FEM3DFun.hpp:13-92 / FEM3DFun.cpp:128-268)
//   - NumericalCoarseningUsingMultigrid
//       (SamplesGenerator/NumericalCoarseningUsingMultigrid.h:11-48,
//        NumericalCoarseningUsingMultiGrid.cpp:134-345)
//   - computeParametersAndTensorValues (the sample generator's batch call,
//       SamplesGenerator/SamplesGeneratorImpl.cpp:3683-3752) and the level*.bin
//       file format (Utilities/include/cfgUtilities.h:780-870).
// Eigen types of the reference become std::vector<double>; names, argument
// meaning and outputs are kept.  Every numeric step runs in libfemh.
#pragma once
#include <array>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/femh.h"

namespace femh_host {

// Error thrown when the engine reports a failure (the reference asserts or prints).
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ------------------------------------------------------------- fast_fem ---
class RealFun {
 public:
  std::vector<double> param;
  std::vector<double> lowerBounds, upperBounds;
  virtual void init(const std::vector<double>& x0) { param = x0; }
  virtual void setParam(const std::vector<double>& x0) { param = x0; }
  virtual double f() = 0;
  virtual std::vector<double> df() { return {}; }
  virtual ~RealFun() {}
};

// Sparse derivative entry (index, value) of a field value w.r.t. its parameters.
using SparseEntry = std::pair<int, double>;

class RealField {
 public:
  std::vector<double> param;
  virtual double f(const std::array<double, 3>& x) = 0;
  virtual std::vector<SparseEntry> df(const std::array<double, 3>& x) = 0;
  virtual void setParam(int i, double v) { param.at(i) = v; }
  // For fields whose df at every voxel centre is one parameter with weight 1
  // (piecewise-constant fields): that parameter per voxel of an n[0] x n[1] x
  // n[2] grid, voxel (i*n1 + j)*n2 + k; false for other fields.  FEM3DFun::df
  // then runs the field chain rule on the device (femh_field_gradient).
  virtual bool voxelMap(const int n[3], std::vector<int>& map) const { (void)n; (void)map; return false; }
  virtual ~RealField() {}
};

// One parameter per grid cell (fast_fem/PiecewiseConstant3D.cpp).
class PiecewiseConstant3D : public RealField {
 public:
  int gridSize[3] = {0, 0, 0};
  void allocate(int nx, int ny, int nz);
  double f(const std::array<double, 3>& x) override;
  std::vector<SparseEntry> df(const std::array<double, 3>& x) override;
  bool voxelMap(const int n[3], std::vector<int>& map) const override;

 private:
  int index(const std::array<double, 3>& x) const;
};

// Mirror-symmetric field (fast_fem/PiecewiseConstantSym3D.cpp): every
// coordinate in [0, 1] is reflected into the lower half (c -> 2c, then 2 - 2c
// above 1) and mapped onto an nx x ny x nz parameter grid -- the parameters of
// one octant, mirrored into the other seven.
class PiecewiseConstantSym3D : public RealField {
 public:
  int gridSize[3] = {0, 0, 0};
  void allocate(int nx, int ny, int nz);
  double f(const std::array<double, 3>& x) override;
  std::vector<SparseEntry> df(const std::array<double, 3>& x) override;
  bool voxelMap(const int n[3], std::vector<int>& map) const override;

 protected:
  virtual int index(const std::array<double, 3>& x) const;
};

// Cubic-symmetric field (fast_fem/PiecewiseConstantCubic3D.cpp, the field of
// fast_fem/run3d.cpp:176-182): reflected as the mirror-symmetric field, then
// the three coordinates sorted so that x >= y >= z (the 48 symmetries of the
// cube map onto one parameter).
class PiecewiseConstantCubic3D : public PiecewiseConstantSym3D {
 protected:
  int index(const std::array<double, 3>& x) const override;
};

// Homogenized-stiffness objective on a periodic voxel cell.  G is C^H (both
// triangles); f = 0.5 sum wG (G-G0)^2 + 0.5 mw (density-m0)^2; df is the
// adjoint gradient w.r.t. the field parameters.
class FEM3DFun : public RealFun {
 public:
  FEM3DFun();
  ~FEM3DFun() override;
  FEM3DFun(const FEM3DFun&) = delete;
  FEM3DFun& operator=(const FEM3DFun&) = delete;

  // material of the solid (fast_fem: ElasticMaterial(E, nu)), precision/solver
  double E = 1.0, nu = 0.3;
  int precision = FEMH_FP64, solver = FEMH_GMG_PCG;
  // start each solve from the previous one's fluctuation fields (consecutive
  // setParam calls of a line search / descent differ little); off by default
  bool warmStart = false;

  std::array<double, 36> G{}, G0{}, wG{};
  double density = 0, m0 = 0, mw = 0;
  std::vector<int> gridSize{0, 0, 0};
  RealField* field = nullptr;          // not owned (as in the reference)
  std::vector<double> distribution;    // per voxel, clamped to [1e-3, 1]
  femh_solve_info lastInfo{};

  void init(const std::vector<double>& x0) override;
  void setParam(const std::vector<double>& x0) override;
  double f() override;
  std::vector<double> df() override;

 private:
  femh_handle* h_ = nullptr;
  void ensure_handle();
};

// Optimisation loop around the objective (fast_fem/run3d.cpp:238-289): steepest
// descent with a halving line search on the bounds-clamped step x - h*grad.
void clampVector(std::vector<double>& x, const std::vector<double>& lo, const std::vector<double>& hi);
// Returns 0 and updates x0 when f decreased within 10 halvings of h, else -1.
int lineSearch(RealFun* fun, std::vector<double>& x0, const std::vector<double>& dir, double& h);
// nSteps of descent from x0 with initial step maxStep / ||grad||_inf; x0 holds
// the last accepted point.  Returns the number of accepted steps.
int gradientDescent(RealFun* fun, std::vector<double>& x0, int nSteps, double maxStep);

// --------------------------------------------------------- SamplesGenerator ---
struct BaseMaterial {   // StrainLin parameters: param[0] = mu, param[1] = lambda
  double mu, lambda;
};

class NumericalCoarseningUsingMultigrid {
 public:
  enum StructureType { General, Cubic, Orthotropic };

  NumericalCoarseningUsingMultigrid();
  ~NumericalCoarseningUsingMultigrid();
  NumericalCoarseningUsingMultigrid(const NumericalCoarseningUsingMultigrid&) = delete;
  NumericalCoarseningUsingMultigrid& operator=(const NumericalCoarseningUsingMultigrid&) = delete;

  void setUseVariableDensity(bool v) { m_useVariableDensity = v; }
  void init(int N[3], int iNbBlockRep, int iNbSubdiv, const std::vector<BaseMaterial>& iBaseMaterials,
            StructureType iType);
  // Appends the 21 lower-triangle entries of C^H and, for Cubic, (rho, E, nu_xy, G).
  void computeCoarsenedElasticityTensorAndParameters3D(const std::vector<int>& iMaterials, int N[3],
                                                       const std::vector<double>& iBaseMaterialDensities,
                                                       StructureType iType, std::vector<double>& ioTensorValues,
                                                       std::vector<double>& ioParameters);
  // Many structures in batched engine calls (the sample generator's batch).
  // maxNodesPerCall > 0 caps the voxels of one call; 0 (default) splits by
  // what fits the device (femh_batch_memory).  The outputs are appended only
  // once every call has succeeded: on an error they are left as they were.
  void computeBatch(const std::vector<std::vector<int>>& iMaterials, int N[3],
                    const std::vector<double>& iBaseMaterialDensities, StructureType iType,
                    std::vector<double>& ioTensorValues, std::vector<double>& ioParameters);

  femh_solve_info lastInfo{};
  long long maxNodesPerCall = 0;
  // The reference fills only the upper triangle of its C but appends the
  // entries C(i, j), j <= i (NumericalCoarseningUsingMultiGrid.cpp:296-324), so
  // its 15 off-diagonal tensor values are 0.  false (default): append the
  // symmetric tensor's values; true: append those zeros, as the reference's
  // tensor files hold them (the parameters use C(0,1) either way, as there).
  bool referenceLowerTriangle = false;

 private:
  femh_handle* h_ = nullptr;
  int m_nbBlockRep = 1, m_nbSubdiv = 1;
  bool m_useVariableDensity = true;
  double m_densityMin = 1e-4;
  double m_E = 1.0, m_nu = 0.3;
  void append(const double C[36], const std::vector<int>& mats, const std::vector<double>& dens,
              StructureType t, std::vector<double>& tv, std::vector<double>& pv);
};

// femlib's force-driven coarsening, NumericalCoarsening
// (SamplesGenerator/NumericalCoarsening.h:20-90, .cpp:116-133, 266-340): the
// same init / computeCoarsenedElasticityTensorAndParameters3D calls and
// outputs.  The reference applies unit face forces, solves the multiplier
// system with PARDISO and reads C and the parameters off the harmonic
// displacements; here one strain-driven solve gives C^H and the fields, and
// femh_force_tensors evaluates femlib's tensor formula on them.  Appends the
// 21 lower-triangle entries of that tensor and (rho, Y, nu_xy, G) for Cubic,
// (rho, Yx, Yy, Yz, nu_xy, nu_xz, nu_yz, G_yz, G_xz, G_xy) otherwise, with
// Y_a = f / eps_aa and nu_ab = -eps_bb / eps_aa of the coarse strains eps =
// (C^H)^-1 sigma under the unit face force f on faces of area A_a (sigma_aa =
// f / A_a; the mesh spans 1 along its longest side) and G_i = C(3+i, 3+i).
// Cells must be cubic (n = N * rep * subdiv equal on all axes; femh_force_tensors).
// Every base material must have the same Poisson ratio (the engine scales one
// element matrix per voxel) and a positive stiffness (femlib's fixing of
// isolated vertices of a zero-stiffness void is not needed then).  femlib also
// scales the diagonal of K by 1 + 1e-5; these are the exact values, from which
// femlib's outputs differ at about that level.
class NumericalCoarsening {
 public:
  enum StructureType { General, Cubic, Orthotropic };

  NumericalCoarsening() = default;
  ~NumericalCoarsening();
  NumericalCoarsening(const NumericalCoarsening&) = delete;
  NumericalCoarsening& operator=(const NumericalCoarsening&) = delete;

  void init(int N[3], int iNbBlockRep, int iNbSubdiv, const std::vector<BaseMaterial>& iBaseMaterials);
  void computeCoarsenedElasticityTensorAndParameters3D(const std::vector<int>& iMaterials, int N[3],
                                                       const std::vector<double>& iBaseMaterialDensities,
                                                       StructureType iType, std::vector<double>& ioTensorValues,
                                                       std::vector<double>& ioParameters);
  // Many structures in batched engine calls; maxNodesPerCall as in
  // NumericalCoarseningUsingMultigrid::computeBatch (0: what fits the device);
  // outputs appended only once every call has succeeded.
  void computeBatch(const std::vector<std::vector<int>>& iMaterials, int N[3],
                    const std::vector<double>& iBaseMaterialDensities, StructureType iType,
                    std::vector<double>& ioTensorValues, std::vector<double>& ioParameters);

  femh_solve_info lastInfo{};
  long long maxNodesPerCall = 0;

 private:
  femh_handle* h_ = nullptr;
  int m_nbBlockRep = 1, m_nbSubdiv = 1;
  std::vector<double> m_E;   // Young's modulus of each base material
  void rho_of(const std::vector<int>& cells, std::vector<double>& rho) const;
  void append(const double CH[36], const double Cf[36], const int n[3], const std::vector<int>& mats,
              const std::vector<double>& dens, StructureType t, std::vector<double>& tv,
              std::vector<double>& pv) const;
};

// cfgMaterialUtilities::repMaterialAssignment (Utilities/src/cfgMaterialUtilities.cpp:914-956)
void repMaterialAssignment(int nx, int ny, int nz, const std::vector<int>& iMaterialCombIndices, int repX,
                           int repY, int repZ, int iNbSubdivisions, std::vector<int>& oMaterials);
// Lame -> (E, nu)  (Utilities/src/cfgMaterialUtilities.cpp:2945-2949)
void fromLamesParametersToYoungModulusPoissonRatio(double lambda, double mu, double& E, double& nu);

// level*.bin files: int32 count + raw values; nested vectors count-prefixed.
template <class T> bool writeBinary(const std::string& file, const std::vector<T>& v);
template <class T> bool readBinary(const std::string& file, std::vector<T>& v);
template <class T> bool writeBinary(const std::string& file, const std::vector<std::vector<T>>& v);
template <class T> bool readBinary(const std::string& file, std::vector<std::vector<T>>& v);

}  // namespace femh_host
