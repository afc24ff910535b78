// femh_host.cpp -- the reference-facing C++ layer over the C ABI (see
// femh_host.hpp for the interfaces it mirrors).
#include "femh_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>

namespace femh_host {

namespace {
void check(femh_handle* h, int st, bool allow_unconverged = false) {
  if (st == FEMH_OK || (allow_unconverged && st == FEMH_E_NOT_CONVERGED)) return;
  char buf[512] = {0};
  if (h) femh_last_error(h, buf, sizeof buf);
  else std::snprintf(buf, sizeof buf, "engine creation failed (no CUDA device or bad config)");
  throw Error(st, "femh error " + std::to_string(st) + ": " + buf);
}

// Structures of n[0] x n[1] x n[2] voxels per batched engine call, at least
// one: a voxel budget when max_nodes > 0, else what fits the device -- the
// engine's estimate of one cell's memory against 92% of the memory available
// to the handle (femh_batch_memory).
size_t batch_cells_per_call(femh_handle* h, const int n[3], long long max_nodes) {
  const long long cell = (long long)n[0] * n[1] * n[2];
  if (max_nodes > 0) return (size_t)std::max(1LL, max_nodes / std::max(1LL, cell));
  femh_cell c{n[0], n[1], n[2], 1.0, nullptr};
  double need = 0.0, avail = 0.0;
  check(h, femh_batch_memory(h, 1, &c, &need, &avail));
  return (size_t)std::max(1.0, std::floor(0.92 * avail / std::max(need, 1.0)));
}
}  // namespace

// ---------------------------------------------------------- PiecewiseConstant3D
void PiecewiseConstant3D::allocate(int nx, int ny, int nz) {
  gridSize[0] = nx;
  gridSize[1] = ny;
  gridSize[2] = nz;
  param.assign((size_t)nx * ny * nz, 1.0);
}

int PiecewiseConstant3D::index(const std::array<double, 3>& x) const {
  int idx[3];
  for (int d = 0; d < 3; ++d) idx[d] = std::min(std::max((int)(x[d] * gridSize[d]), 0), gridSize[d] - 1);
  return (idx[0] * gridSize[1] + idx[1]) * gridSize[2] + idx[2];
}

double PiecewiseConstant3D::f(const std::array<double, 3>& x) { return param[index(x)]; }

std::vector<SparseEntry> PiecewiseConstant3D::df(const std::array<double, 3>& x) { return {{index(x), 1.0}}; }

bool PiecewiseConstant3D::voxelMap(const int n[3], std::vector<int>& map) const {
  map.resize((size_t)n[0] * n[1] * n[2]);
  for (int i = 0; i < n[0]; ++i)
    for (int j = 0; j < n[1]; ++j)
      for (int k = 0; k < n[2]; ++k)
        map[((size_t)i * n[1] + j) * n[2] + k] = index({(i + 0.5) / n[0], (j + 0.5) / n[1], (k + 0.5) / n[2]});
  return true;
}

// ------------------------------------------- PiecewiseConstantSym3D / Cubic3D
void PiecewiseConstantSym3D::allocate(int nx, int ny, int nz) {
  gridSize[0] = nx;
  gridSize[1] = ny;
  gridSize[2] = nz;
  param.assign((size_t)nx * ny * nz, 1.0);
}

namespace {
double reflect(double c) {
  c *= 2.0;
  return c > 1.0 ? 2.0 - c : c;
}
int cell_of(double c, int n) { return std::min(std::max((int)(c * n), 0), n - 1); }
}  // namespace

int PiecewiseConstantSym3D::index(const std::array<double, 3>& x) const {
  int idx[3];
  for (int d = 0; d < 3; ++d) idx[d] = cell_of(reflect(x[d]), gridSize[d]);
  return (idx[0] * gridSize[1] + idx[1]) * gridSize[2] + idx[2];
}

int PiecewiseConstantCubic3D::index(const std::array<double, 3>& x) const {
  double c[3] = {reflect(x[0]), reflect(x[1]), reflect(x[2])};
  if (c[0] < c[1]) std::swap(c[0], c[1]);   // x >= y >= z
  if (c[0] < c[2]) std::swap(c[0], c[2]);
  if (c[1] < c[2]) std::swap(c[1], c[2]);
  int idx[3];
  for (int d = 0; d < 3; ++d) idx[d] = cell_of(c[d], gridSize[d]);
  return (idx[0] * gridSize[1] + idx[1]) * gridSize[2] + idx[2];
}

double PiecewiseConstantSym3D::f(const std::array<double, 3>& x) { return param[index(x)]; }

std::vector<SparseEntry> PiecewiseConstantSym3D::df(const std::array<double, 3>& x) { return {{index(x), 1.0}}; }

bool PiecewiseConstantSym3D::voxelMap(const int n[3], std::vector<int>& map) const {
  map.resize((size_t)n[0] * n[1] * n[2]);
  for (int i = 0; i < n[0]; ++i)
    for (int j = 0; j < n[1]; ++j)
      for (int k = 0; k < n[2]; ++k)
        map[((size_t)i * n[1] + j) * n[2] + k] = index({(i + 0.5) / n[0], (j + 0.5) / n[1], (k + 0.5) / n[2]});
  return true;
}

// -------------------------------------------------------------------- FEM3DFun
FEM3DFun::FEM3DFun() {}

FEM3DFun::~FEM3DFun() {
  if (h_) femh_destroy(h_);
}

void FEM3DFun::ensure_handle() {
  if (h_) return;
  femh_config c;
  femh_config_default(&c);
  c.interp = FEMH_INTERP_RAMP3;   // coef x/(3-2x) of fast_fem/FEM3DFun.cpp:20-27
  c.E_s = E;
  c.nu = nu;
  c.rho_min = 1e-3;               // Clamp(field->f, 1e-3, 1), FEM3DFun.cpp:147
  c.rho_max = 1.0;
  c.precision = precision;
  c.solver = solver;
  c.warm_start = warmStart ? 1 : 0;
  check(nullptr, femh_create(&h_, &c));
}

void FEM3DFun::init(const std::vector<double>& x0) {
  param = x0;
  ensure_handle();
}

void FEM3DFun::setParam(const std::vector<double>& x0) {
  if (!field) throw Error(FEMH_E_STATE, "FEM3DFun::setParam needs a field");
  ensure_handle();
  param = x0;
  for (size_t i = 0; i < field->param.size() && i < x0.size(); ++i) field->setParam((int)i, x0[i]);
  const int nx = gridSize[0], ny = gridSize[1], nz = gridSize[2];
  distribution.assign((size_t)nx * ny * nz, 0.0);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const std::array<double, 3> x = {(i + 0.5) / nx, (j + 0.5) / ny, (k + 0.5) / nz};
        distribution[((size_t)i * ny + j) * nz + k] = std::min(std::max(field->f(x), 1e-3), 1.0);
      }
  check(h_, femh_homogenize(h_, nx, ny, nz, 1.0 / nx, distribution.data(), 0, G.data(), &lastInfo), true);
  density = 0.0;
  for (double d : distribution) density += d;
  density /= (double)distribution.size();
}

double FEM3DFun::f() {
  double sum = 0.0;
  for (int t = 0; t < 36; ++t) sum += wG[t] * (G[t] - G0[t]) * (G[t] - G0[t]);
  return 0.5 * sum + 0.5 * mw * (density - m0) * (density - m0);
}

std::vector<double> FEM3DFun::df() {
  const int nx = gridSize[0], ny = gridSize[1], nz = gridSize[2];
  const size_t nv = (size_t)nx * ny * nz;
  double dLdC[36];
  for (int t = 0; t < 36; ++t) dLdC[t] = wG[t] * (G[t] - G0[t]);
  const double dm = (mw / (double)nv) * (density - m0);
  std::vector<double> grad(param.size(), 0.0);
  std::vector<int> map;
  if (!grad.empty() && field->voxelMap(gridSize.data(), map)) {   // chain rule on the device
    for (int& p : map)
      if (p < 0 || (size_t)p >= grad.size()) p = -1;
    check(h_, femh_field_gradient(h_, dLdC, dm, (int)grad.size(), map.data(), grad.data()));
    return grad;
  }
  std::vector<double> dfddist(nv, 0.0);
  check(h_, femh_homogenize_grad(h_, dLdC, dfddist.data(), 0));
  for (auto& v : dfddist) v += dm;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const std::array<double, 3> x = {(i + 0.5) / nx, (j + 0.5) / ny, (k + 0.5) / nz};
        const double g = dfddist[((size_t)i * ny + j) * nz + k];
        for (const auto& e : field->df(x))
          if (e.first >= 0 && (size_t)e.first < grad.size()) grad[e.first] += g * e.second;
      }
  return grad;
}

// ------------------------------------------------------------ descent loop
void clampVector(std::vector<double>& x, const std::vector<double>& lo, const std::vector<double>& hi) {
  for (size_t i = 0; i < x.size(); ++i) {
    if (i < lo.size()) x[i] = std::max(x[i], lo[i]);
    if (i < hi.size()) x[i] = std::min(x[i], hi[i]);
  }
}

int lineSearch(RealFun* fun, std::vector<double>& x0, const std::vector<double>& dir, double& h) {
  const double f0 = fun->f();
  for (int step = 0; step < 10; ++step) {
    std::vector<double> x(x0.size());
    for (size_t i = 0; i < x.size(); ++i) x[i] = x0[i] - h * dir[i];
    clampVector(x, fun->lowerBounds, fun->upperBounds);
    fun->setParam(x);
    if (fun->f() < f0) {
      x0 = x;
      return 0;
    }
    h /= 2;
  }
  fun->setParam(x0);   // leave the objective at the last accepted point
  return -1;
}

int gradientDescent(RealFun* fun, std::vector<double>& x0, int nSteps, double maxStep) {
  std::vector<double> x = x0;
  fun->setParam(x);
  int accepted = 0;
  for (int it = 0; it < nSteps; ++it) {
    const std::vector<double> grad = fun->df();
    double norm = 0.0;
    for (double g : grad) norm = std::max(norm, std::fabs(g));
    if (!(norm > 0.0)) break;
    double h = maxStep / norm;
    if (lineSearch(fun, x, grad, h) < 0) break;
    x0 = x;
    ++accepted;
  }
  return accepted;
}

// ----------------------------------------------- NumericalCoarseningUsingMultigrid
void fromLamesParametersToYoungModulusPoissonRatio(double lambda, double mu, double& E, double& nu) {
  E = mu * (3 * lambda + 2 * mu) / (lambda + mu);
  nu = lambda / (2 * (lambda + mu));
}

void repMaterialAssignment(int nx, int ny, int nz, const std::vector<int>& in, int repX, int repY, int repZ,
                           int sub, std::vector<int>& out) {
  const int NX = repX * nx * sub, NY = repY * ny * sub, NZ = repZ * nz * sub;
  out.assign((size_t)NX * NY * NZ, -1);
  for (int m = 0; m < nx; ++m)
    for (int n = 0; n < ny; ++n)
      for (int p = 0; p < nz; ++p) {
        const int v = in[((size_t)m * ny + n) * nz + p];
        for (int i = 0; i < repX; ++i)
          for (int j = 0; j < repY; ++j)
            for (int k = 0; k < repZ; ++k)
              for (int a = 0; a < sub; ++a)
                for (int b = 0; b < sub; ++b)
                  for (int c = 0; c < sub; ++c) {
                    const int X = i * sub * nx + m * sub + a;
                    const int Y = j * sub * ny + n * sub + b;
                    const int Z = k * sub * nz + p * sub + c;
                    out[((size_t)X * NY + Y) * NZ + Z] = v;
                  }
      }
}

NumericalCoarseningUsingMultigrid::NumericalCoarseningUsingMultigrid() {}

NumericalCoarseningUsingMultigrid::~NumericalCoarseningUsingMultigrid() {
  if (h_) femh_destroy(h_);
}

void NumericalCoarseningUsingMultigrid::init(int N[3], int iNbBlockRep, int iNbSubdiv,
                                             const std::vector<BaseMaterial>& mats, StructureType) {
  if (mats.size() < 2) throw Error(FEMH_E_ARG, "two base materials are required");
  m_nbBlockRep = iNbBlockRep;
  m_nbSubdiv = iNbSubdiv;
  // The reference swaps materials 0 and 1 and assigns material id 0 to every
  // cell, so K0 is the stiffness of base material 1; the per-cell coefficient
  // is 1 for material 1 and m_densityMin otherwise
  // (NumericalCoarseningUsingMultiGrid.cpp:170-193, 229-241).
  fromLamesParametersToYoungModulusPoissonRatio(mats[1].lambda, mats[1].mu, m_E, m_nu);
  if (h_) femh_destroy(h_);
  h_ = nullptr;
  femh_config c;
  femh_config_default(&c);
  c.interp = FEMH_INTERP_BINARY;
  c.bin_hi = m_E;
  c.bin_lo = m_E * (m_useVariableDensity ? m_densityMin : 1.0);
  c.nu = m_nu;
  check(nullptr, femh_create(&h_, &c));
  (void)N;
}

void NumericalCoarseningUsingMultigrid::append(const double C[36], const std::vector<int>& mats,
                                               const std::vector<double>& dens, StructureType t,
                                               std::vector<double>& tv, std::vector<double>& pv) {
  if (t != Cubic) throw Error(FEMH_E_ARG, "only Cubic structures derive (rho, E, nu, G), as in the reference");
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) tv.push_back(referenceLowerTriangle && j < i ? 0.0 : C[i * 6 + j]);
  double r = 0.0;
  for (int m : mats) r += dens.at(m);
  r /= (double)mats.size();
  const double Gs = C[3 * 6 + 3];
  const double a = C[0 * 6 + 1] / C[0];
  const double nuxy = a / (1 + a);
  const double Ey = C[0 * 6 + 1] * (1 + nuxy) * (1 - 2 * nuxy) / nuxy;
  pv.push_back(r);
  pv.push_back(Ey);
  pv.push_back(nuxy);
  pv.push_back(Gs);
}

void NumericalCoarseningUsingMultigrid::computeCoarsenedElasticityTensorAndParameters3D(
    const std::vector<int>& iMaterials, int N[3], const std::vector<double>& iDens, StructureType t,
    std::vector<double>& tv, std::vector<double>& pv) {
  if (!h_) throw Error(FEMH_E_STATE, "init() first");
  std::vector<int> cells;
  repMaterialAssignment(N[0], N[1], N[2], iMaterials, m_nbBlockRep, m_nbBlockRep, m_nbBlockRep, m_nbSubdiv, cells);
  const int n[3] = {N[0] * m_nbBlockRep * m_nbSubdiv, N[1] * m_nbBlockRep * m_nbSubdiv,
                    N[2] * m_nbBlockRep * m_nbSubdiv};
  std::vector<double> rho(cells.size());
  for (size_t i = 0; i < cells.size(); ++i) rho[i] = cells[i] == 1 ? 1.0 : 0.0;
  double C[36];
  check(h_, femh_homogenize(h_, n[0], n[1], n[2], 1.0 / n[0], rho.data(), 0, C, &lastInfo), true);
  append(C, iMaterials, iDens, t, tv, pv);
}

void NumericalCoarseningUsingMultigrid::computeBatch(const std::vector<std::vector<int>>& iMaterials, int N[3],
                                                     const std::vector<double>& iDens, StructureType t,
                                                     std::vector<double>& tv, std::vector<double>& pv) {
  if (!h_) throw Error(FEMH_E_STATE, "init() first");
  const size_t nc = iMaterials.size();
  if (nc == 0) return;
  const int n[3] = {N[0] * m_nbBlockRep * m_nbSubdiv, N[1] * m_nbBlockRep * m_nbSubdiv,
                    N[2] * m_nbBlockRep * m_nbSubdiv};
  const size_t per = batch_cells_per_call(h_, n, maxNodesPerCall);
  std::vector<double> tv_new, pv_new;   // appended to the caller's vectors once every call succeeded
  for (size_t c0 = 0; c0 < nc; c0 += per) {
    const size_t m = std::min(per, nc - c0);
    std::vector<std::vector<double>> rho(m);
    std::vector<femh_cell> cells(m);
    for (size_t c = 0; c < m; ++c) {
      std::vector<int> mm;
      repMaterialAssignment(N[0], N[1], N[2], iMaterials[c0 + c], m_nbBlockRep, m_nbBlockRep, m_nbBlockRep,
                            m_nbSubdiv, mm);
      rho[c].resize(mm.size());
      for (size_t i = 0; i < mm.size(); ++i) rho[c][i] = mm[i] == 1 ? 1.0 : 0.0;
      cells[c] = femh_cell{n[0], n[1], n[2], 1.0 / n[0], rho[c].data()};
    }
    std::vector<double> C(36 * m);
    std::vector<femh_solve_info> infos(m);
    check(h_, femh_homogenize_batch(h_, (int)m, cells.data(), C.data(), nullptr, nullptr, infos.data()), true);
    for (size_t c = 0; c < m; ++c) append(&C[36 * c], iMaterials[c0 + c], iDens, t, tv_new, pv_new);
    lastInfo = infos.back();
  }
  tv.insert(tv.end(), tv_new.begin(), tv_new.end());
  pv.insert(pv.end(), pv_new.begin(), pv_new.end());
}

// ---------------------------------------------------------- NumericalCoarsening
namespace {

// Inverse of a nonsingular 6x6 matrix (Gauss-Jordan with partial pivoting).
bool invert6(const double A[36], double Ai[36]) {
  double M[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      M[i][j] = A[6 * i + j];
      M[i][6 + j] = i == j ? 1.0 : 0.0;
    }
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
    if (!(std::fabs(M[p][c]) > 0.0)) return false;
    if (p != c)
      for (int j = 0; j < 12; ++j) std::swap(M[p][j], M[c][j]);
    const double inv = 1.0 / M[c][c];
    for (int j = 0; j < 12; ++j) M[c][j] *= inv;
    for (int r = 0; r < 6; ++r) {
      if (r == c || M[r][c] == 0.0) continue;
      const double f = M[r][c];
      for (int j = 0; j < 12; ++j) M[r][j] -= f * M[c][j];
    }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ai[6 * i + j] = M[i][6 + j];
  return true;
}
}  // namespace

NumericalCoarsening::~NumericalCoarsening() {
  if (h_) femh_destroy(h_);
}

void NumericalCoarsening::init(int N[3], int iNbBlockRep, int iNbSubdiv, const std::vector<BaseMaterial>& mats) {
  if (mats.size() != 2) throw Error(FEMH_E_ARG, "two base materials are required (the engine's two-material law)");
  m_nbBlockRep = iNbBlockRep;
  m_nbSubdiv = iNbSubdiv;
  m_E.assign(2, 0.0);
  double nu[2];
  for (int i = 0; i < 2; ++i) fromLamesParametersToYoungModulusPoissonRatio(mats[i].lambda, mats[i].mu, m_E[i], nu[i]);
  if (!(m_E[0] > 0.0 && m_E[1] > 0.0)) throw Error(FEMH_E_ARG, "base materials need a positive stiffness");
  if (std::fabs(nu[0] - nu[1]) > 1e-12) throw Error(FEMH_E_ARG, "base materials must share one Poisson ratio");
  if (h_) femh_destroy(h_);
  h_ = nullptr;
  femh_config c;
  femh_config_default(&c);
  c.interp = FEMH_INTERP_BINARY;   // material index 1 -> bin_hi, 0 -> bin_lo
  c.bin_hi = m_E[1];
  c.bin_lo = m_E[0];
  c.nu = nu[1];
  check(nullptr, femh_create(&h_, &c));
  (void)N;
}

void NumericalCoarsening::rho_of(const std::vector<int>& cells, std::vector<double>& rho) const {
  rho.resize(cells.size());
  for (size_t i = 0; i < cells.size(); ++i) {
    if (cells[i] != 0 && cells[i] != 1) throw Error(FEMH_E_ARG, "material indices must be 0 or 1");
    rho[i] = cells[i] == 1 ? 1.0 : 0.0;
  }
}

void NumericalCoarsening::append(const double CH[36], const double Cf[36], const int n[3],
                                 const std::vector<int>& mats, const std::vector<double>& dens, StructureType t,
                                 std::vector<double>& tv, std::vector<double>& pv) const {
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) tv.push_back(Cf[i * 6 + j]);
  double r = 0.0;   // computeMaterialDensity (Utilities/src/cfgMaterialUtilities.cpp:660-671)
  for (int m : mats) r += dens.at(m);
  r /= (double)mats.size();
  double S[36];   // compliance: the coarse strain under a macro stress sigma is S sigma
  if (!invert6(CH, S)) throw Error(FEMH_E_ARG, "C^H is singular");
  const double dx = 1.0 / std::max(n[0], std::max(n[1], n[2]));   // ElementRegGrid: longest side 1
  const double area[3] = {n[1] * n[2] * dx * dx, n[0] * n[2] * dx * dx, n[0] * n[1] * dx * dx};
  const int naxis = t == Cubic ? 1 : 3;
  pv.push_back(r);
  for (int a = 0; a < naxis; ++a) pv.push_back(area[a] / S[7 * a]);   // f / eps_aa, eps_aa = S_aa f / A_a
  pv.push_back(-S[6 * 1 + 0] / S[0]);                                 // nu_xy = -eps_yy / eps_xx (x load)
  if (t != Cubic) {
    pv.push_back(-S[6 * 2 + 0] / S[0]);   // nu_xz (x load)
    pv.push_back(-S[6 * 2 + 1] / S[7]);   // nu_yz (y load)
  }
  for (int i = 0; i < naxis; ++i) pv.push_back(Cf[(3 + i) * 6 + 3 + i]);
}

void NumericalCoarsening::computeCoarsenedElasticityTensorAndParameters3D(
    const std::vector<int>& iMaterials, int N[3], const std::vector<double>& iDens, StructureType t,
    std::vector<double>& tv, std::vector<double>& pv) {
  if (!h_) throw Error(FEMH_E_STATE, "init() first");
  std::vector<int> cells;
  repMaterialAssignment(N[0], N[1], N[2], iMaterials, m_nbBlockRep, m_nbBlockRep, m_nbBlockRep, m_nbSubdiv, cells);
  const int n[3] = {N[0] * m_nbBlockRep * m_nbSubdiv, N[1] * m_nbBlockRep * m_nbSubdiv,
                    N[2] * m_nbBlockRep * m_nbSubdiv};
  std::vector<double> rho;
  rho_of(cells, rho);
  double CH[36], Cf[36];
  const double dx = 1.0 / std::max(n[0], std::max(n[1], n[2]));
  check(h_, femh_homogenize(h_, n[0], n[1], n[2], dx, rho.data(), 0, CH, &lastInfo), true);
  check(h_, femh_force_tensors(h_, Cf));
  append(CH, Cf, n, iMaterials, iDens, t, tv, pv);
}

void NumericalCoarsening::computeBatch(const std::vector<std::vector<int>>& iMaterials, int N[3],
                                       const std::vector<double>& iDens, StructureType t,
                                       std::vector<double>& tv, std::vector<double>& pv) {
  if (!h_) throw Error(FEMH_E_STATE, "init() first");
  const size_t nc = iMaterials.size();
  if (nc == 0) return;
  const int n[3] = {N[0] * m_nbBlockRep * m_nbSubdiv, N[1] * m_nbBlockRep * m_nbSubdiv,
                    N[2] * m_nbBlockRep * m_nbSubdiv};
  const double dx = 1.0 / std::max(n[0], std::max(n[1], n[2]));
  const size_t per = batch_cells_per_call(h_, n, maxNodesPerCall);
  std::vector<double> tv_new, pv_new;   // appended to the caller's vectors once every call succeeded
  for (size_t c0 = 0; c0 < nc; c0 += per) {
    const size_t m = std::min(per, nc - c0);
    std::vector<std::vector<double>> rho(m);
    std::vector<femh_cell> cells(m);
    for (size_t c = 0; c < m; ++c) {
      std::vector<int> mm;
      repMaterialAssignment(N[0], N[1], N[2], iMaterials[c0 + c], m_nbBlockRep, m_nbBlockRep, m_nbBlockRep,
                            m_nbSubdiv, mm);
      rho_of(mm, rho[c]);
      cells[c] = femh_cell{n[0], n[1], n[2], dx, rho[c].data()};
    }
    std::vector<double> CH(36 * m), Cf(36 * m);
    std::vector<femh_solve_info> infos(m);
    check(h_, femh_homogenize_batch(h_, (int)m, cells.data(), CH.data(), nullptr, nullptr, infos.data()), true);
    check(h_, femh_force_tensors(h_, Cf.data()));
    for (size_t c = 0; c < m; ++c)
      append(&CH[36 * c], &Cf[36 * c], n, iMaterials[c0 + c], iDens, t, tv_new, pv_new);
    lastInfo = infos.back();
  }
  tv.insert(tv.end(), tv_new.begin(), tv_new.end());
  pv.insert(pv.end(), pv_new.begin(), pv_new.end());
}

// ------------------------------------------------------------ binary files
template <class T>
bool writeBinary(const std::string& file, const std::vector<T>& v) {
  std::ofstream f(file, std::ios::binary);
  if (!f) return false;
  const int32_t n = (int32_t)v.size();
  f.write((const char*)&n, sizeof n);
  if (n > 0) f.write((const char*)v.data(), sizeof(T) * n);
  return (bool)f;
}

template <class T>
bool readBinary(const std::string& file, std::vector<T>& v) {
  std::ifstream f(file, std::ios::binary);
  if (!f) return false;
  int32_t n = 0;
  f.read((char*)&n, sizeof n);
  if (!f || n < 0) return false;
  v.resize(n);
  if (n > 0) f.read((char*)v.data(), sizeof(T) * n);
  return (bool)f;
}

template <class T>
bool writeBinary(const std::string& file, const std::vector<std::vector<T>>& v) {
  std::ofstream f(file, std::ios::binary);
  if (!f) return false;
  const int32_t n = (int32_t)v.size();
  f.write((const char*)&n, sizeof n);
  for (const auto& row : v) {
    const int32_t m = (int32_t)row.size();
    f.write((const char*)&m, sizeof m);
    if (m > 0) f.write((const char*)row.data(), sizeof(T) * m);
  }
  return (bool)f;
}

template <class T>
bool readBinary(const std::string& file, std::vector<std::vector<T>>& v) {
  std::ifstream f(file, std::ios::binary);
  if (!f) return false;
  int32_t n = 0;
  f.read((char*)&n, sizeof n);
  if (!f || n < 0) return false;
  v.assign(n, {});
  for (auto& row : v) {
    int32_t m = 0;
    f.read((char*)&m, sizeof m);
    if (!f || m < 0) return false;
    row.resize(m);
    if (m > 0) f.read((char*)row.data(), sizeof(T) * m);
  }
  return (bool)f;
}

template bool writeBinary<float>(const std::string&, const std::vector<float>&);
template bool writeBinary<int>(const std::string&, const std::vector<int>&);
template bool writeBinary<double>(const std::string&, const std::vector<double>&);
template bool readBinary<float>(const std::string&, std::vector<float>&);
template bool readBinary<int>(const std::string&, std::vector<int>&);
template bool readBinary<double>(const std::string&, std::vector<double>&);
template bool writeBinary<float>(const std::string&, const std::vector<std::vector<float>>&);
template bool writeBinary<int>(const std::string&, const std::vector<std::vector<int>>&);
template bool readBinary<float>(const std::string&, std::vector<std::vector<float>>&);
template bool readBinary<int>(const std::string&, std::vector<std::vector<int>>&);

}  // namespace femh_host
