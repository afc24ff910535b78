// engine.cu -- host side of libfemh: cell hierarchy, PCG / multigrid / defect
// correction drivers, energy reductions and the C ABI of include/femh.h.
//
// The reference path this replaces (desaic/fem): fast_fem/FEM3DFun.cpp:128-268
// (setParam -> topoOptLib Homogenize -> copyPeriodicU -> energy loop; df) and
// SamplesGenerator/NumericalCoarseningUsingMultiGrid.cpp:221-345.  There is no
// CPU fallback: every numeric step below is one of this library's kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/femh.h"
#include "kernels.cuh"

using namespace femh;

namespace {

struct FemhError {
  int code;
  std::string msg;
};

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) {                                                               \
      char b_[512];                                                                        \
      snprintf(b_, sizeof b_, "%s failed: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, \
               __LINE__);                                                                  \
      throw FemhError{e_ == cudaErrorMemoryAllocation ? FEMH_E_OOM : FEMH_E_CUDA, b_};      \
    }                                                                                      \
  } while (0)

// ------------------------------------------------------------ host math ---
// Element matrix of a unit cube (h = 1) for the engineering-Voigt material
// matrix D (xx,yy,zz,yz,xz,xy), 2x2x2 Gauss, local node a = 4ax+2ay+az.
void host_k0_voigt(const double D[6][6], double K[576]) {
  std::fill(K, K + 576, 0.0);
  const double g = 1.0 / std::sqrt(3.0);
  for (int q = 0; q < 8; ++q) {
    const double xi[3] = {(q & 4) ? g : -g, (q & 2) ? g : -g, (q & 1) ? g : -g};
    double B[6][24] = {};
    for (int a = 0; a < 8; ++a) {
      const double s[3] = {(a & 4) ? 1.0 : -1.0, (a & 2) ? 1.0 : -1.0, (a & 1) ? 1.0 : -1.0};
      double dN[3];
      for (int d = 0; d < 3; ++d) {
        double v = s[d] / 8.0;
        for (int e = 0; e < 3; ++e)
          if (e != d) v *= 1.0 + s[e] * xi[e];
        dN[d] = 2.0 * v;
      }
      B[0][3 * a] = dN[0];
      B[1][3 * a + 1] = dN[1];
      B[2][3 * a + 2] = dN[2];
      B[3][3 * a + 1] = dN[2]; B[3][3 * a + 2] = dN[1];
      B[4][3 * a] = dN[2];     B[4][3 * a + 2] = dN[0];
      B[5][3 * a] = dN[1];     B[5][3 * a + 1] = dN[0];
    }
    for (int p = 0; p < 24; ++p)
      for (int r = 0; r < 24; ++r) {
        double acc = 0;
        for (int m = 0; m < 6; ++m) {
          double t = 0;
          for (int n = 0; n < 6; ++n) t += D[m][n] * B[n][r];
          acc += B[m][p] * t;
        }
        K[p * 24 + r] += 0.125 * acc;
      }
  }
}

// Isotropic material matrix, E = 1.
void iso_voigt(double nu, double D[6][6]) {
  const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 1.0 / (2.0 * (1.0 + nu));
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) D[a][b] = 0.0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) D[a][b] = lam;
  for (int a = 0; a < 3; ++a) D[a][a] += 2 * mu;
  D[3][3] = D[4][4] = D[5][5] = mu;
}

void host_k0(double nu, double K[576]) {
  double D[6][6];
  iso_voigt(nu, D);
  host_k0_voigt(D, K);
}

// Element matrix of femlib's force-driven coarse tensor: that tensor
// (meshUtil::computeCoarsenedElasticityTensor, femlib/src/MeshUtilities.cpp:960-1060)
// contracts tensor-shear strains (eps_yz, not 2 eps_yz) with the engineering
// matrix StrainLin::EMatrix (femlib/src/StrainLin.cpp:39-58), i.e. its energy
// is that of the matrix S D S, S = diag(1, 1, 1, 1/2, 1/2, 1/2), on
// engineering strains -- a cubic material with the shear modulus divided by 4.
void host_k0_force(double nu, double K[576]) {
  double D[6][6];
  iso_voigt(nu, D);
  for (int a = 3; a < 6; ++a) D[a][a] *= 0.25;
  host_k0_voigt(D, K);
}

inline double chi_k(int k, int a) {  // Hadamard character
  double v = 1.0;
  for (int s = 0; s < 3; ++s)
    if ((k >> s) & 1) v *= ((a >> s) & 1) ? 1.0 : -1.0;
  return v;
}

// Kh = T K0 T^T / 64 in (k, c) indexing; returns its 8 distinct values after
// checking that every other entry vanishes and the structure holds.
HadK host_hadk(const double K[576]) {
  double Kh[24][24];
  for (int k1 = 0; k1 < 8; ++k1)
    for (int c1 = 0; c1 < 3; ++c1)
      for (int k2 = 0; k2 < 8; ++k2)
        for (int c2 = 0; c2 < 3; ++c2) {
          double s = 0;
          for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) s += chi_k(k1, a) * K[(3 * a + c1) * 24 + 3 * b + c2] * chi_k(k2, b);
          Kh[3 * k1 + c1][3 * k2 + c2] = s / 64.0;
        }
  auto at = [&](int k1, int c1, int k2, int c2) { return Kh[3 * k1 + c1][3 * k2 + c2]; };
  HadK h;
  h.A = at(1, 0, 1, 0);
  h.Bd = at(4, 0, 4, 0);
  h.Bo = at(4, 0, 2, 1);
  h.D1 = at(3, 0, 3, 0);
  h.O1 = at(3, 0, 5, 1);
  h.D2 = at(3, 1, 3, 1);
  h.O2 = at(3, 1, 5, 0);
  h.G = at(7, 0, 7, 0);
  h.diag = K[0];
  // rebuild the model and compare
  double M[24][24] = {};
  auto set = [&](int k1, int c1, int k2, int c2, double v) { M[3 * k1 + c1][3 * k2 + c2] = v; };
  const int N[3][2] = {{4, 0}, {2, 1}, {1, 2}};
  const int T3[3][2] = {{3, 0}, {5, 1}, {6, 2}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      set(N[i][0], N[i][1], N[j][0], N[j][1], i == j ? h.Bd : h.Bo);
      set(T3[i][0], T3[i][1], T3[j][0], T3[j][1], i == j ? h.D1 : h.O1);
    }
  const int S[3][2][2] = {{{1, 0}, {4, 2}}, {{1, 1}, {2, 2}}, {{2, 0}, {4, 1}}};
  const int Pp[3][2][2] = {{{3, 1}, {5, 0}}, {{3, 2}, {6, 0}}, {{5, 2}, {6, 1}}};
  for (int t = 0; t < 3; ++t)
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        set(S[t][i][0], S[t][i][1], S[t][j][0], S[t][j][1], h.A);
        set(Pp[t][i][0], Pp[t][i][1], Pp[t][j][0], Pp[t][j][1], i == j ? h.D2 : h.O2);
      }
  for (int c = 0; c < 3; ++c) set(7, c, 7, c, h.G);
  double err = 0, mx = 0;
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) {
      err = std::max(err, std::fabs(M[i][j] - Kh[i][j]));
      mx = std::max(mx, std::fabs(Kh[i][j]));
    }
  for (int i = 1; i < 24; ++i)
    if (std::fabs(K[i * 24 + i] - K[0]) > 1e-13 * std::fabs(K[0])) err = 1.0;
  if (err > 1e-12 * mx) throw FemhError{FEMH_E_ARG, "element stiffness lacks cube symmetry (nu out of range?)"};
  return h;
}

// Largest eigenvalue of diag(K0)^-1 K0, by cyclic Jacobi rotations of the
// symmetric diag^-1/2 K0 diag^-1/2.  For K = sum_e c_e K0_e with c_e >= 0,
// u.K u <= lambda u.D u holds element by element, so this bounds the spectrum
// of D^-1 K for every coefficient field, on every rediscretised level (5.318
// for nu = 0.3, the volumetric mode of one element).
// Largest eigenvalue of D^-1 K0 for the Jacobi smoother's diagonal D: the
// point diagonal, or (block) the 3x3 node blocks.  K = sum_e K_e and
// D = sum_e D_e with K_e <= lambda D_e for every element, so the bound holds
// for every coefficient field.  Symmetric form L^-1 K0 L^-T (L the Cholesky
// factor of D), cyclic Jacobi eigenvalue sweeps.
double host_jacobi_bound(const double K[576], bool block = false) {
  double S[24][24];
  if (!block) {
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) S[i][j] = K[i * 24 + j] / std::sqrt(K[i * 24 + i] * K[j * 24 + j]);
  } else {
    double Li[24][24] = {};   // block-diagonal inverse Cholesky factor of the node blocks
    for (int a = 0; a < 8; ++a) {
      double L[3][3] = {}, I[3][3] = {};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) {
          double v = K[(3 * a + i) * 24 + 3 * a + j];
          for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k];
          L[i][j] = (i == j) ? std::sqrt(v) : v / L[j][j];
        }
      for (int c = 0; c < 3; ++c)   // forward substitution: L I = e_c
        for (int i = 0; i < 3; ++i) {
          double v = (i == c) ? 1.0 : 0.0;
          for (int k = 0; k < i; ++k) v -= L[i][k] * I[k][c];
          I[i][c] = v / L[i][i];
        }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Li[3 * a + i][3 * a + j] = I[i][j];
    }
    double T[24][24];
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double v = 0.0;
        for (int k = 0; k < 24; ++k) v += Li[i][k] * K[k * 24 + j];
        T[i][j] = v;
      }
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double v = 0.0;
        for (int k = 0; k < 24; ++k) v += T[i][k] * Li[j][k];
        S[i][j] = v;
      }
  }
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < 24; ++i)
      for (int j = i + 1; j < 24; ++j) off += S[i][j] * S[i][j];
    if (off < 1e-28) break;
    for (int p = 0; p < 24; ++p)
      for (int q = p + 1; q < 24; ++q) {
        if (std::fabs(S[p][q]) < 1e-300) continue;
        const double th = (S[q][q] - S[p][p]) / (2.0 * S[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 24; ++k) {
          const double a = S[k][p], b = S[k][q];
          S[k][p] = c * a - s * b;
          S[k][q] = s * a + c * b;
        }
        for (int k = 0; k < 24; ++k) {
          const double a = S[p][k], b = S[q][k];
          S[p][k] = c * a - s * b;
          S[q][k] = s * a + c * b;
        }
      }
  }
  double m = 0.0;
  for (int i = 0; i < 24; ++i) m = std::max(m, S[i][i]);
  return m;
}

// Damping weights of an m-sweep smoothing pass.  ratio > 0: the reciprocal
// roots of the degree-m Chebyshev polynomial on [lmax/ratio, lmax], smallest
// weight first (the pass then multiplies the error by the scaled Chebyshev
// polynomial, below 1 in magnitude on all of (0, lmax]); ratio == 0: omega for
// every sweep.
std::vector<double> smooth_weights(int m, double lmax, double ratio, double omega) {
  std::vector<double> w;
  for (int k = 1; k <= m; ++k) {
    if (ratio > 0.0) {
      const double a = lmax / ratio, c = 0.5 * (lmax + a), h = 0.5 * (lmax - a);
      w.push_back(1.0 / (c + h * std::cos(M_PI * (2 * k - 1) / (2.0 * m))));
    } else {
      w.push_back(omega);
    }
  }
  return w;
}

ElemConst host_elemconst(const double K[576]) {
  ElemConst ec{};
  for (int I = 0; I < kNumRhs; ++I) {
    double eps[3][3] = {};
    if (I < 3) eps[I][I] = 1;
    if (I == 3) eps[1][2] = eps[2][1] = 0.5;
    if (I == 4) eps[0][2] = eps[2][0] = 0.5;
    if (I == 5) eps[0][1] = eps[1][0] = 0.5;
    double ue[24];
    for (int a = 0; a < 8; ++a) {
      const double x[3] = {double((a >> 2) & 1), double((a >> 1) & 1), double(a & 1)};
      for (int c = 0; c < 3; ++c) ue[3 * a + c] = eps[c][0] * x[0] + eps[c][1] * x[1] + eps[c][2] * x[2];
    }
    for (int p = 0; p < 24; ++p) {
      double s = 0;
      for (int q = 0; q < 24; ++q) s += K[p * 24 + q] * ue[q];
      ec.g1[I][p] = s;
    }
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 8; ++k) {
        double s = 0;
        for (int a = 0; a < 8; ++a) s += chi_k(k, a) * ue[3 * a + c];
        ec.uhat0[I][c][k] = s;
      }
  }
  return ec;
}

// ------------------------------------------------------------- device mem ---
struct Arena {
  std::vector<void*> ptrs;
  size_t held = 0;            // bytes allocated
  size_t limit = SIZE_MAX;    // FEMH_ARENA_LIMIT_BYTES (tests only): fail like a full device beyond it
  void* get(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (bytes > limit - held) throw FemhError{FEMH_E_OOM, "device memory limit of this handle reached"};
    void* p = nullptr;
    CK(cudaMalloc(&p, bytes));
    ptrs.push_back(p);
    held += bytes;
    return p;
  }
  template <typename T> T* arr(size_t n) { return static_cast<T*>(get(n * sizeof(T))); }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
    held = 0;
  }
  ~Arena() { release(); }
};

template <typename T>
T* upload(Arena& ar, const std::vector<T>& v, cudaStream_t s) {
  T* d = ar.arr<T>(std::max<size_t>(v.size(), 1));
  if (!v.empty()) CK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return d;
}

struct UnitList {
  std::vector<StencilUnit> su;
  StencilUnit* d_su = nullptr;
  std::vector<NodeUnit> nu;
  NodeUnit* d_nu = nullptr;
  // persistent staged kernel (variant 7): CTA b runs units [cta[b], cta[b+1])
  std::vector<int> cta;
  int* d_cta = nullptr;
  int cta_cap = 0;   // entries allocated at d_cta
};

// Stencil units of one z extent: entries [b, e) of a unit list sorted by z extent.
struct UnitGroups {
  std::vector<int> nz, b, e;
};

struct Level {
  std::vector<CellDesc> cells;
  CellDesc* d_cells = nullptr;
  long long ntot = 0, nodes_smooth = 0;
  int level = 0;
  int NT = 256, maxnz = 1;
  int nz_spec = 0;   // > 0: every cell of the level has this z extent (specialised kernel)
  int chunk = 0;     // x-chunk length of the stencil units (0 = heuristic), set by the autotuner
  int variant = 2;   // stencil kernel (femh_config::stencil_variant numbering)
  bool bulk_ok = false;     // the bulk-copy staged FP32 kernel (variant 5) can run on this level
  bool bulk_ok64 = false;   // the bulk-copy staged FP64 kernel (variant 6) can run on this level
  // cells of several z extents, each one with a compile-time kernel (a batch
  // of uneven cells): the unit lists are sorted by z extent and each extent
  // launches its own specialised kernel
  bool grouped = false;
  UnitGroups gall, gsmooth, g64;
  // level 0 of the mixed modes also runs FP64 operator applies (CG / true
  // residual): they get their own tuned layout (FP64 kernels spill in the
  // layout that suits FP32)
  bool use64 = false;
  int variant64 = 1, chunk64 = 0;
  std::vector<StencilUnit> su64;
  StencilUnit* d_su64 = nullptr;
  std::vector<int> su64_sb, su64_se;
  int *d_su64_sb = nullptr, *d_su64_se = nullptr;
  UnitList all, smooth;      // all cells / cells that continue to a coarser level
  std::vector<int> su_sb, su_se, nu_sb, nu_se;   // slot ranges per cell (all lists)
  int *d_su_sb = nullptr, *d_su_se = nullptr, *d_nu_sb = nullptr, *d_nu_se = nullptr;
  std::vector<int> coarse_list;                  // cells whose coarsest level this is
  int* d_coarse_list = nullptr;
  long long* d_aoff = nullptr;
  double* d_A = nullptr;
  double* d_Awork = nullptr;
  int* d_cstat = nullptr;
  int coarse_maxm = 0;
  void* kc = nullptr;     // TC
  float* invd = nullptr;
  float* binv = nullptr;  // node-block Jacobi: [node][6] symmetric 3x3 inverses (block_jacobi)
  void* xa = nullptr;     // level vectors (TV)
  void* xb = nullptr;
  void* bv = nullptr;
};

int pow2ceil(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace

// ============================================================== handle ===
struct femh_handle {
  femh_config cfg{};
  int device = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  std::string err;
  long long launches = 0;
  double K0[576];
  HadK hk{};
  HadK hk_force{};   // Hadamard factors of host_k0_force (femh_force_tensors)
  ElemConst ec{};
  ElemConst* d_ec = nullptr;
  double* d_K0 = nullptr;
  std::vector<double> w_pre, w_post;   // damping weight of each smoothing sweep
  Arena perm;   // lives as long as the handle

  // setup cache
  std::vector<int> shape_key;
  std::vector<double> h_key;
  int prec_key = -1, solver_key = -1, bf16_key = -1;
  Arena setup;
  std::vector<Level> levels;
  std::map<std::string, int> tune_cache;   // autotuned x-chunk per level signature
  int ncells = 0;
  std::vector<long long> cell_vox;   // voxels per cell
  std::vector<long long> cell_off;   // fine offsets
  long long nvox = 0;
  // fine-level FP64 arrays
  double* rho_in = nullptr;     // packed input rho
  double* rho_used = nullptr;
  double* kc64 = nullptr;
  double* b64 = nullptr;        // [6][3][nvox]
  double* x64 = nullptr;        // solution chi
  double* r64 = nullptr;
  void* cg_x = nullptr;         // inner CG vectors (TV / TP)
  void* cg_r = nullptr;
  void* cg_p = nullptr;
  void* cg_q = nullptr;
  void* cg_rm = nullptr;        // FP32 copy of the FP64 residual (level-0 rhs of an FP32 V-cycle)
  CGState* d_state = nullptr;
  BlockCG* d_bcg = nullptr;     // block PCG step matrices per cell
  double* d_part_g = nullptr;   // block PCG 6x6 partials [2][sub-slots][36]
  double* d_part_b = nullptr;   // block PCG ||r||^2 partials [sub-slots][6]
  size_t part_g_slots = 0;      // slots of level 0 before any compaction (units keep their slot)
  int bsub = 1;                 // block PCG update / direction: CTAs per level-0 node unit
  int bsub_g = 1;               // block PCG Gram kernels: CTAs per level-0 node unit
  std::vector<CGState> state;
  double* d_part_s = nullptr;   // stencil partials [slots][6]
  double* d_part_n = nullptr;   // node partials [slots][6][2]
  double* d_part_z = nullptr;   // node partials [slots][6]
  double* d_part_e = nullptr;   // energy partials [slots][21]
  double* d_C = nullptr;        // [ncells][36]
  double* d_W = nullptr;        // [ncells][21]
  double* d_stage = nullptr;    // output staging (dCdrho, fields, apply), allocated on first use
  size_t stage_n = 0;           // doubles in d_stage
  // field chain rule: voxels of each field parameter (CSR), cached by the map's hash
  int* d_fmap = nullptr;        // [nparam + 1] offsets, then [nmapped] voxel indices
  size_t fmap_n = 0;            // ints allocated
  unsigned long long fmap_key = 0;
  int fmap_nparam = -1;
  double* d_nrm = nullptr;      // [ncells][6]
  bool solved = false;
  bool have_x = false;   // x64 holds the last solution of these cells (warm starts)
  std::vector<double> C_last;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int wait_limit = kWaitLimit;   // try_wait rounds of the staged kernels' stage waits
  int nsm = 1;                   // multiprocessors of the device (persistent stencil CTAs)
  // persistent stencil CTAs are split evenly over the six load cases; the inner
  // solves of defect correction finish their load cases at different times
  // (the CTAs of a finished one would idle), so they run one CTA per unit
  bool persist_ok = true;
  int* d_loop = nullptr;         // CG iterations run on the device in the current solve (WHILE-node count)
  int* d_err = nullptr;   // [0] set by a stencil kernel whose bounded wait ran out,
                          // [1] by k_coef on a NaN, infinite or negative density

  // measurement: per-kernel-class CUDA-event timing (femh_profile), and the
  // count of kernel executions including CUDA-graph replays
  bool prof = false;
  bool capturing = false;
  long long cap_count = 0;
  struct KStat {
    long long launches = 0;
    double ms = 0, bytes = 0;
  };
  std::map<std::string, KStat> kstats;
  struct Pend {
    std::string name;
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<Pend> pend;
  std::vector<cudaEvent_t> evpool;
};

namespace {

#define LAUNCH_CHECK(H)                          \
  do {                                           \
    CK(cudaGetLastError());                      \
    if ((H)->capturing) (H)->cap_count++;        \
    else (H)->launches++;                        \
  } while (0)

cudaEvent_t pool_event(femh_handle* H) {
  if (!H->evpool.empty()) {
    cudaEvent_t e = H->evpool.back();
    H->evpool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}

// Times the launches issued in its scope when profiling is on (graphs are
// not captured then, so every launch is timed on the handle's stream).
struct Prof {
  femh_handle* H;
  const char* name;
  double bytes;
  cudaEvent_t a = nullptr;
  Prof(femh_handle* h, const char* n, double b) : H(h), name(n), bytes(b) {
    if (H->prof && !H->capturing) {
      a = pool_event(H);
      CK(cudaEventRecord(a, H->stream));
    }
  }
  ~Prof() {
    if (a) {
      cudaEvent_t b = pool_event(H);
      if (cudaEventRecord(b, H->stream) == cudaSuccess) H->pend.push_back({name, a, b, bytes});
    }
  }
};

void prof_resolve(femh_handle* H) {
  if (H->pend.empty()) return;
  CK(cudaStreamSynchronize(H->stream));
  for (auto& p : H->pend) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, p.a, p.b));
    auto& k = H->kstats[p.name];
    k.launches++;
    k.ms += ms;
    k.bytes += p.bytes;
    H->evpool.push_back(p.a);
    H->evpool.push_back(p.b);
  }
  H->pend.clear();
}

void set_err(femh_handle* h, const std::string& m) {
  if (h) h->err = m;
}

MatLaw make_law(const femh_config& c) {
  MatLaw m{};
  m.interp = c.interp;
  m.rho_bf16 = (c.precision != FEMH_FP64 && c.store_bf16) ? 1 : 0;
  m.E_s = c.E_s;
  m.E_min = c.E_min;
  m.penal = c.penal;
  m.bin_hi = c.bin_hi;
  m.bin_lo = c.bin_lo;
  m.rho_min = c.rho_min;
  m.rho_max = c.rho_max;
  return m;
}

// Stencil work units of one cell: tiles of up to R-1 rows, x-chunks of len.
void add_stencil_units(std::vector<StencilUnit>& out, int cellidx, const CellDesc& cd, int NT,
                       int& slot, int chunk_req = 0, int variant = 2) {
  const int R = NT / cd.nz;
  const bool two_rows = variant == 2 || variant == 4 || variant == 5 || variant == 7;
  const int maxrows = std::max(1, std::min(two_rows ? 2 * R - 1 : R - 1, cd.ny));
  const int ntiles = (cd.ny + maxrows - 1) / maxrows;
  const int chunk = chunk_req > 0 ? std::min(chunk_req, cd.nx)
                                  : (cd.nx >= 128 ? 32 : (cd.nx >= 64 ? 16 : (cd.nx >= 16 ? 8 : cd.nx)));
  const int nchunks = (cd.nx + chunk - 1) / chunk;
  int j = 0;
  for (int t = 0; t < ntiles; ++t) {
    const int rows = (cd.ny - j + (ntiles - t) - 1) / (ntiles - t);
    int i = 0;
    for (int c = 0; c < nchunks; ++c) {
      const int len = (cd.nx - i + (nchunks - c) - 1) / (nchunks - c);
      out.push_back(StencilUnit{cellidx, j, rows, i, len, slot++});
      i += len;
    }
    j += rows;
  }
}

// Node work units of chunk nodes (even, so node pairs never straddle units).
// Level 0 (whose CG reductions keep per-unit partial sums) uses 2048; the
// coarser levels' node kernels are latency-bound, and smaller units give them
// more CTAs.
void add_node_units(std::vector<NodeUnit>& out, int cellidx, long long nn, int& slot, long long chunk) {
  for (long long b = 0; b < nn; b += chunk)
    out.push_back(NodeUnit{cellidx, slot++, b, std::min(nn, b + chunk)});
}

template <typename T> size_t esize() { return sizeof(T); }

// Threads per CTA of a stencil variant on a level: the packed two-row kernel
// needs up to ~160 registers a thread, so it runs 384-thread CTAs where its
// tiles still hold at least two thread rows.
int variant_nt(int level_nt, int maxnz, int variant) {
  if ((variant == 4 || variant == 5 || variant == 7) && level_nt > 384 && 384 >= 2 * maxnz) return 384;
  return level_nt;
}

// z extents with compile-time kernels, and their threads per CTA.
bool spec_nz(int nz) { return nz == 16 || nz == 24 || nz == 32 || nz == 48 || nz == 64 || nz == 128 || nz == 256; }
int spec_nt(int nz) { return (nz == 24 || nz == 48) ? 480 : 512; }

// Threads per CTA that a cell's stencil units are cut for.
int cell_nt(const Level& L, const CellDesc& cd, int variant) {
  return L.grouped ? variant_nt(spec_nt(cd.nz), cd.nz, variant) : variant_nt(L.NT, L.maxnz, variant);
}

// On grouped levels: sort a unit list by z extent (stable, so each cell's
// units stay in order; slots travel with their units) and record the groups.
void group_units(const Level& L, std::vector<StencilUnit>& su, UnitGroups& g, bool sort) {
  g.nz.clear();
  g.b.clear();
  g.e.clear();
  if (!L.grouped) return;
  if (sort)
    std::stable_sort(su.begin(), su.end(), [&](const StencilUnit& x, const StencilUnit& y) {
      return L.cells[x.cell].nz < L.cells[y.cell].nz;
    });
  for (int i = 0; i < (int)su.size(); ++i) {
    const int nz = L.cells[su[i].cell].nz;
    if (g.nz.empty() || g.nz.back() != nz) {
      g.nz.push_back(nz);
      g.b.push_back(i);
      g.e.push_back(i + 1);
    } else {
      g.e.back() = i + 1;
    }
  }
}

// Persistent staged kernel (variant 7): one CTA per multiprocessor, the six
// load cases in blockIdx.y, so P = SMs / 6 CTAs per load case; CTA b runs the
// consecutive units [cta[b], cta[b+1]) of the list, the cut points balancing
// x planes (the kernel's steps).  The table lives at a fixed device address
// (capacity P + 1), rewritten in place when the list changes (batch
// compaction), so captured launches stay valid for the same P.
void build_cta_table(femh_handle* H, const Level& L, UnitList& ul, bool upload_new) {
  if (L.variant != 7 || L.grouped) {
    ul.cta.clear();
    return;
  }
  const int P = std::max(1, std::min(H->nsm / kNumRhs, (int)ul.su.size()));
  long long tot = 0;
  for (const auto& u : ul.su) tot += u.len;
  ul.cta.assign(P + 1, (int)ul.su.size());
  ul.cta[0] = 0;
  long long acc = 0;
  int p = 1;
  for (int k = 0; k < (int)ul.su.size() && p < P; ++k) {
    acc += ul.su[k].len;
    while (p < P && acc * P >= tot * p) ul.cta[p++] = k + 1;
  }
  if (upload_new || ul.d_cta == nullptr || ul.cta_cap < P + 1) {
    ul.cta_cap = std::max(P + 1, H->nsm / kNumRhs + 1);
    ul.d_cta = H->setup.arr<int>(ul.cta_cap);
  }
  CK(cudaMemcpyAsync(ul.d_cta, ul.cta.data(), sizeof(int) * ul.cta.size(), cudaMemcpyHostToDevice, H->stream));
}

}  // namespace

// ======================================================== kernel launch ===
namespace {

template <typename T, int NT, int OUT, int NZ, typename TIn, typename TOut, typename TB, typename TC>
void stencil_go(femh_handle* H, dim3 grid, size_t smem, const StencilArgs<TIn, TOut, TB, TC>& a, int variant) {
  static bool attr1 = false, attr2 = false, attr3 = false;
  if constexpr (std::is_same<T, float>::value) {
    if (variant == 3) {   // two load cases per CTA in packed FP32x2 lanes
      auto fn3 = stencilp_kernel<NT, OUT, NZ, TIn, TOut, TB, TC>;
      if (!attr3) {
        CK(cudaFuncSetAttribute(fn3, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        attr3 = true;
      }
      fn3<<<dim3(grid.x, kNumRhs / 2), NT, smem, H->stream>>>(a);
      LAUNCH_CHECK(H);
      return;
    }
  }
  if (variant == 2) {
    auto fn2 = stencil2_kernel<T, NT, OUT, NZ, TIn, TOut, TB, TC>;
    if (!attr2) {
      CK(cudaFuncSetAttribute(fn2, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr2 = true;
    }
    fn2<<<grid, NT, smem, H->stream>>>(a);
    LAUNCH_CHECK(H);
    return;
  }
  bool& attr = attr1;
  auto fn = stencil_kernel<T, NT, OUT, NZ, TIn, TOut, TB, TC>;
  if (!attr) {
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  fn<<<grid, NT, smem, H->stream>>>(a);
  LAUNCH_CHECK(H);
}

// Two voxel rows per thread in packed FP32x2 lanes (variant 4).
template <int NT, int OUT, int NZ, typename TIn, typename TOut, typename TB, typename TC>
void stencil_go4(femh_handle* H, dim3 grid, size_t smem, const StencilArgs<TIn, TOut, TB, TC>& a) {
  static bool attr = false;
  auto fn = stencil2p_kernel<NT, OUT, NZ, TIn, TOut, TB, TC>;
  if (!attr) {
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  fn<<<grid, NT, smem, H->stream>>>(a);
  LAUNCH_CHECK(H);
}

// Two voxel rows per thread in packed FP32x2 lanes, inputs staged by bulk copies (variant 5).
template <int NT, int OUT, int NZ>
void stencil_go5(femh_handle* H, dim3 grid, size_t smem, const StencilArgs<float, float, float, float>& a) {
  static bool attr = false;
  auto fn = stencil2b_kernel<NT, OUT, NZ>;
  if (!attr) {   // (a few bytes of static shared memory come on top)
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  fn<<<grid, NT, smem, H->stream>>>(a);
  LAUNCH_CHECK(H);
}

// FP64 operator, one voxel row per thread, inputs staged by bulk copies (variant 6).
template <int NT, int OUT, int NZ, typename TIn>
void stencil_go6(femh_handle* H, dim3 grid, size_t smem, const StencilArgs<TIn, double, double, double>& a) {
  static bool attr = false;
  auto fn = stencil1b_kernel<NT, OUT, NZ, TIn>;
  if (!attr) {   // (a few bytes of static shared memory come on top)
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    attr = true;
  }
  fn<<<grid, NT, smem, H->stream>>>(a);
  LAUNCH_CHECK(H);
}

// T = arithmetic type; in/out/b storage types as given.
template <typename T, int OUT, typename TIn, typename TOut, typename TB, typename TC>
void stencil(femh_handle* H, Level& L, bool smooth_only, const TIn* in, TOut* out, const TB* b,
             const TC* kc, double* part, const CGState* stt, double omega) {
  const bool use64 = sizeof(T) == 8 && L.use64 && !smooth_only;
  UnitList& ul = smooth_only ? L.smooth : L.all;
  const std::vector<StencilUnit>& units = use64 ? L.su64 : ul.su;
  if (units.empty()) return;
  int variant = use64 ? L.variant64 : L.variant;
  if (!std::is_same<T, float>::value) {   // packed-FP32 kernels: FP64 twin with the same units
    if (variant == 3) variant = 1;
    if (variant == 4 || variant == 5 || variant == 7) variant = 2;
  } else if (variant == 6) {   // the staged FP64 kernel's FP32 twin has the same units
    variant = 1;
  }
  if (variant == 6) {   // bulk-copy staging: FP64 output / rhs / coefficients, aligned rows
    const bool ok = std::is_same<TOut, double>::value && std::is_same<TB, double>::value &&
                    std::is_same<TC, double>::value &&
                    (std::is_same<TIn, double>::value || std::is_same<TIn, float>::value);
    auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    if (!(ok && L.bulk_ok64 && al(in) && al(out) && al(kc) && al(L.invd) && (!b || al(b)) && L.ntot % 4 == 0))
      variant = 1;
  }
  bool persistent = false;
  if (variant == 7) {   // the staged kernel as persistent CTAs over the list's CTA table
    persistent = !use64 && !L.grouped && ul.cta.size() >= 2 && H->persist_ok;
    variant = 5;
  }
  if (variant == 5) {   // bulk-copy staging: FP32 storage, 16-byte aligned rows, eligible level
    const bool f32 = std::is_same<TIn, float>::value && std::is_same<TOut, float>::value &&
                     std::is_same<TB, float>::value && std::is_same<TC, float>::value;
    auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    if (!(f32 && L.bulk_ok && al(in) && al(out) && al(kc) && al(L.invd) && (!b || al(b)) && L.ntot % 4 == 0)) {
      variant = 4;
      persistent = false;
    }
  }
  StencilArgs<TIn, TOut, TB, TC> a;
  a.cells = L.d_cells;
  a.units = use64 ? L.d_su64 : ul.d_su;
  a.u = in;
  a.out = out;
  a.b = b;
  a.kc = kc;
  a.invd = L.invd;
  a.partials = part;
  a.stt = stt;
  a.ntot = L.ntot;
  a.k = H->hk;
  a.omega = omega;
  a.err = H->d_err;
  a.wait_limit = H->wait_limit;
  a.cta_units = persistent ? ul.d_cta : nullptr;
  a.binv = (OUT == OUT_JACOBI || OUT == OUT_JACOBI_DOT) ? L.binv : nullptr;
  {
    const HadK& k = H->hk;
    const double kv[8] = {k.A, k.Bd - k.Bo, k.Bo, k.D1 - k.O1, k.O1, k.D2 - k.O2, k.O2, k.G};
    for (int i = 0; i < 8; ++i) a.kp[i] = make_float2((float)kv[i], (float)kv[i]);
  }
  dim3 grid((unsigned)(persistent ? ul.cta.size() - 1 : units.size()), kNumRhs);
  static const char* mode_names[] = {"apply", "apply_dot", "jacobi", "jacobi_dot", "resid"};
  char nm[64];
  snprintf(nm, sizeof nm, "stencil_%s_%s_L%d", sizeof(T) == 8 ? "f64" : "f32", mode_names[OUT], L.level);
  // algorithmic bytes: only (cell, load case) pairs still iterating move data
  double nodes = 0.0;
  if (H->prof) {
    for (const auto& cd : L.cells) {
      if (smooth_only && cd.child < 0) continue;
      int act = kNumRhs;
      if (stt) {
        act = 0;
        for (int q = 0; q < kNumRhs; ++q) act += H->state[cd.id * kNumRhs + q].active ? 1 : 0;
      }
      nodes += (double)cd.nx * cd.ny * cd.nz * act / kNumRhs;
    }
  }
  double per = 18.0 * (sizeof(TIn) + sizeof(TOut)) + sizeof(TC);
  if (OUT >= OUT_JACOBI) per += 18.0 * sizeof(TB) + (OUT == OUT_RESID ? 0.0 : (L.binv ? 24.0 : 4.0));
  std::string key(nm);
  Prof prof_(H, H->prof ? H->kstats.emplace(key, femh_handle::KStat{}).first->first.c_str() : nm, nodes * per);
  // launch on units of one z extent (nz_spec > 0: compile-time kernels) or on
  // the level's runtime-z kernels (nz_spec = 0), lnt threads per CTA
  auto launch = [&](int nz_spec, int lnt, int maxnz, dim3 grid, const StencilArgs<TIn, TOut, TB, TC>& a) {
    const size_t smem =
        variant == 3 ? sizeof(float4) * 12 * (size_t)lnt + 2 * sizeof(float2) * (size_t)(12 * lnt + 3 * maxnz) +
                             64 * sizeof(double)
        : variant == 2 ? sizeof(T) * (size_t)(2 * (6 * lnt + 3 * maxnz) + 24 * lnt) + 16 + 64 * sizeof(double)
                       : 2 * sizeof(T) * (size_t)(15 * lnt + 3 * maxnz) + 16 + 64 * sizeof(double);
    if constexpr (std::is_same<T, double>::value && std::is_same<TOut, double>::value &&
                  std::is_same<TB, double>::value && std::is_same<TC, double>::value &&
                  (std::is_same<TIn, double>::value || std::is_same<TIn, float>::value)) {
      if (variant == 6) {
        const size_t sm6 = stencil1b_smem_bytes(lnt, nz_spec, (int)sizeof(TIn));
        switch (nz_spec) {
          case 16: stencil_go6<512, OUT, 16>(H, grid, sm6, a); return;
          case 24: stencil_go6<480, OUT, 24>(H, grid, sm6, a); return;
          case 32: stencil_go6<512, OUT, 32>(H, grid, sm6, a); return;
          case 48: stencil_go6<480, OUT, 48>(H, grid, sm6, a); return;
          case 64: stencil_go6<512, OUT, 64>(H, grid, sm6, a); return;
          case 128: stencil_go6<512, OUT, 128>(H, grid, sm6, a); return;
          case 256: stencil_go6<512, OUT, 256>(H, grid, sm6, a); return;
          default: throw FemhError{FEMH_E_ARG, "staged FP64 stencil on an ineligible level"};
        }
      }
    }
    if constexpr (std::is_same<TIn, float>::value && std::is_same<TOut, float>::value &&
                  std::is_same<TB, float>::value && std::is_same<TC, float>::value) {
      if (variant == 5) {   // eligible levels have a compile-time z extent and 384-thread tiles
        const int nt = variant_nt(lnt, maxnz, 5);
        const size_t sm5 = stencil2b_smem_bytes(nt, nz_spec);
        switch (nz_spec) {
          case 16: stencil_go5<384, OUT, 16>(H, grid, sm5, a); return;
          case 24: stencil_go5<384, OUT, 24>(H, grid, sm5, a); return;
          case 32: stencil_go5<384, OUT, 32>(H, grid, sm5, a); return;
          case 48: stencil_go5<384, OUT, 48>(H, grid, sm5, a); return;
          case 64: stencil_go5<384, OUT, 64>(H, grid, sm5, a); return;
          case 128: stencil_go5<384, OUT, 128>(H, grid, sm5, a); return;
          default: throw FemhError{FEMH_E_ARG, "bulk-copy stencil on an ineligible level"};
        }
      }
    }
    if constexpr (std::is_same<T, float>::value) {
      if (variant == 4) {
        const int nt = variant_nt(lnt, maxnz, 4);
        const size_t sm4 =
            sizeof(float2) * 18 * (size_t)nt + sizeof(float) * (6 * (size_t)maxnz + 2) + 64 * sizeof(double);
        if (nt == 384) {
          switch (nz_spec) {
            case 16: stencil_go4<384, OUT, 16>(H, grid, sm4, a); return;
            case 24: stencil_go4<384, OUT, 24>(H, grid, sm4, a); return;
            case 32: stencil_go4<384, OUT, 32>(H, grid, sm4, a); return;
            case 48: stencil_go4<384, OUT, 48>(H, grid, sm4, a); return;
            case 64: stencil_go4<384, OUT, 64>(H, grid, sm4, a); return;
            case 128: stencil_go4<384, OUT, 128>(H, grid, sm4, a); return;
            default: stencil_go4<384, OUT, 0>(H, grid, sm4, a); return;
          }
        }
        if (nz_spec == 256) {
          stencil_go4<512, OUT, 256>(H, grid, sm4, a);
          return;
        }
        switch (nt) {
          case 128: stencil_go4<128, OUT, 0>(H, grid, sm4, a); return;
          case 256: stencil_go4<256, OUT, 0>(H, grid, sm4, a); return;
          case 512: stencil_go4<512, OUT, 0>(H, grid, sm4, a); return;
          default: throw FemhError{FEMH_E_ARG, "unsupported stencil block size"};
        }
      }
    }
    switch (nz_spec) {   // compile-time z extent (threads fixed per extent)
      case 16: stencil_go<T, 512, OUT, 16>(H, grid, smem, a, variant); return;
      case 24: stencil_go<T, 480, OUT, 24>(H, grid, smem, a, variant); return;
      case 32: stencil_go<T, 512, OUT, 32>(H, grid, smem, a, variant); return;
      case 48: stencil_go<T, 480, OUT, 48>(H, grid, smem, a, variant); return;
      case 64: stencil_go<T, 512, OUT, 64>(H, grid, smem, a, variant); return;
      case 128: stencil_go<T, 512, OUT, 128>(H, grid, smem, a, variant); return;
      case 256: stencil_go<T, 512, OUT, 256>(H, grid, smem, a, variant); return;
      default: break;
    }
    switch (lnt) {
      case 128: stencil_go<T, 128, OUT, 0>(H, grid, smem, a, variant); break;
      case 256: stencil_go<T, 256, OUT, 0>(H, grid, smem, a, variant); break;
      case 512: stencil_go<T, 512, OUT, 0>(H, grid, smem, a, variant); break;
      default: throw FemhError{FEMH_E_ARG, "unsupported stencil block size"};
    }
  };
  if (!L.grouped) {
    launch(L.nz_spec, L.NT, L.maxnz, grid, a);
    return;
  }
  // cells of several compile-time z extents: one launch per extent
  const UnitGroups& gr = use64 ? L.g64 : (smooth_only ? L.gsmooth : L.gall);
  for (size_t gi = 0; gi < gr.nz.size(); ++gi) {
    StencilArgs<TIn, TOut, TB, TC> ag = a;
    ag.units = a.units + gr.b[gi];
    launch(gr.nz[gi], spec_nt(gr.nz[gi]), gr.nz[gi], dim3((unsigned)(gr.e[gi] - gr.b[gi]), kNumRhs), ag);
  }
}

#define NODE_GRID(ul) dim3((unsigned)(ul).nu.size(), kNumRhs)


inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

// ====================================================== setup / solve ===
namespace {

template <typename T>
void autotune_levels(femh_handle* H, bool mg);
void autotune_level0_fp64(femh_handle* H);

// Device staging for outputs that the solver's own buffers cannot hold (the
// 21 x nvox dC/drho table, full fields, layouts): allocated on first use and
// kept until the cell set changes, so a batch that never asks for them never
// pays their memory (21 x 8 B per voxel for dC/drho).
void release_stage(femh_handle* H) {
  if (H->d_stage) cudaFree(H->d_stage);
  H->d_stage = nullptr;
  H->stage_n = 0;
  if (H->d_fmap) cudaFree(H->d_fmap);
  H->d_fmap = nullptr;
  H->fmap_n = 0;
  H->fmap_key = 0;
  H->fmap_nparam = -1;
}

double* stage(femh_handle* H, size_t n) {
  if (H->stage_n < n) {
    release_stage(H);
    CK(cudaMalloc(&H->d_stage, n * sizeof(double)));
    H->stage_n = n;
  }
  return H->d_stage;
}

// Where a gradient is written before it goes to the caller: the caller's own
// device buffer, else the CG direction-product buffer q, dead between solves
// and at least 18 x 4 B per voxel (>= the 8 B per voxel of a gradient).
double* grad_target(femh_handle* H, double* user, int user_on_device) {
  return user_on_device ? user : (double*)H->cg_q;
}

// Extents of every multigrid level of one cell (x, y, z per level, finest
// first): halve while every extent is even and >= 4 and the level has more
// than coarse_max_nodes nodes.  Jacobi-PCG: the cell alone.
// Block PCG over the load cases (config block_cg) applies to the multigrid
// PCG with FP64 CG vectors; its search directions are kept in FP64 (FP32 or
// BF16 directions lose the conjugacy of the block's weak directions: at 128^3
// the block stalled for hundreds of iterations with FP32 directions).
bool block_pcg(const femh_config& c) {
  return c.block_cg && c.solver == FEMH_GMG_PCG && (c.precision == FEMH_FP64 || c.precision == FEMH_MIXED_PC);
}

std::vector<int> level_dims(const femh_config& c, int nx, int ny, int nz) {
  std::vector<int> d = {nx, ny, nz};
  if (c.solver != FEMH_GMG_PCG) return d;
  while ((long long)nx * ny * nz > c.coarse_max_nodes && nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && nx >= 4 &&
         ny >= 4 && nz >= 4) {
    nx /= 2; ny /= 2; nz /= 2;
    d.insert(d.end(), {nx, ny, nz});
  }
  if ((long long)nx * ny * nz * 3 > 3 * 1536)
    throw FemhError{FEMH_E_ARG, "multigrid needs cells that halve down to <= 1536 coarse nodes; use Jacobi-PCG"};
  return d;
}

// Device bytes that build_setup allocates for one cell under config c: its
// multigrid levels, dense coarse matrices and fine-level solver vectors (unit
// tables and per-unit partial sums add well under 1%).  Mirrors build_setup.
double cell_setup_bytes(const femh_config& c, int nx, int ny, int nz) {
  const bool mixed = c.precision == FEMH_MIXED;
  const bool gmg = c.solver == FEMH_GMG_PCG;
  const bool mg32 = c.precision != FEMH_FP64;
  const double vsz = mixed ? 4 : 8, msz = mg32 ? 4 : 8, csz = mg32 ? 4 : 8;
  const double psz = (c.precision == FEMH_FP64 || block_pcg(c)) ? 8 : (c.store_bf16 ? 2 : 4);
  const std::vector<int> d = level_dims(c, nx, ny, nz);
  const int nl = (int)d.size() / 3;
  double b = 0.0;
  for (int l = 0; l < nl; ++l) {
    const double n = (double)d[3 * l] * d[3 * l + 1] * d[3 * l + 2];
    b += n * (csz + 4.0);                                   // kc, invd
    if (gmg && c.block_jacobi) b += n * 24.0;              // node-block inverses
    if (l > 0 || gmg) b += n * 36.0 * msz;                 // xa, xb
    if (l > 0) b += n * 18.0 * msz;                        // bv
    if (gmg && l == nl - 1) b += 2.0 * (3.0 * n) * (3.0 * n) * 8.0;   // coarse A, Awork
  }
  const double nv = (double)nx * ny * nz;
  b += nv * (3 * 8.0 + 18 * 8.0 * 2);                      // rho_in, rho_used, kc64, b64, x64
  if (mixed) b += nv * 18 * (8.0 + vsz);                   // r64, cg_x
  b += nv * 18 * (2 * vsz + psz);                          // cg_r, cg_q, cg_p
  if (c.precision == FEMH_MIXED_PC && gmg) b += nv * 18 * 4.0;   // cg_rm
  return b;
}

void build_setup(femh_handle* H, const std::vector<int>& shapes, const std::vector<double>& hs) {
  const femh_config& c = H->cfg;
  const bool mixed = c.precision == FEMH_MIXED;
  const bool gmg = c.solver == FEMH_GMG_PCG;
  if (H->shape_key == shapes && H->h_key == hs && H->prec_key == c.precision && H->solver_key == c.solver &&
      H->bf16_key == c.store_bf16)
    return;
  H->setup.release();
  release_stage(H);
  H->levels.clear();
  H->solved = false;
  H->have_x = false;
  Arena& ar = H->setup;
  cudaStream_t s = H->stream;
  const int nc = (int)shapes.size() / 3;
  H->ncells = nc;
  H->cell_vox.assign(nc, 0);
  H->cell_off.assign(nc, 0);
  long long off = 0;
  for (int i = 0; i < nc; ++i) {
    const int nx = shapes[3 * i], ny = shapes[3 * i + 1], nz = shapes[3 * i + 2];
    if (nx < 2 || ny < 2 || nz < 2) throw FemhError{FEMH_E_ARG, "each cell needs >= 2 voxels per axis"};
    if (nz > 256) throw FemhError{FEMH_E_ARG, "nz > 256 is not supported"};
    if (!(hs[i] > 0.0)) throw FemhError{FEMH_E_ARG, "voxel edge h must be positive"};
    H->cell_vox[i] = (long long)nx * ny * nz;
    H->cell_off[i] = off;
    off += H->cell_vox[i];
  }
  H->nvox = off;
  const bool mg32 = c.precision != FEMH_FP64;   // multigrid hierarchy in FP32
  const size_t vsz = mixed ? sizeof(float) : sizeof(double);   // CG vectors
  const size_t psz = (c.precision == FEMH_FP64 || block_pcg(c)) ? sizeof(double)
                     : (c.store_bf16 ? sizeof(__nv_bfloat16) : sizeof(float));   // search directions
  const size_t msz = mg32 ? sizeof(float) : sizeof(double);

  // ---- levels
  std::vector<std::vector<int>> dims(nc);   // per cell: level dims
  for (int i = 0; i < nc; ++i) dims[i] = level_dims(c, shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2]);
  int nlev = 1;
  for (int i = 0; i < nc; ++i) nlev = std::max(nlev, (int)dims[i].size() / 3);
  H->levels.resize(nlev);
  std::vector<std::vector<int>> idx_at(nlev, std::vector<int>(nc, -1));
  for (int l = 0; l < nlev; ++l) {
    Level& L = H->levels[l];
    long long loff = 0;
    for (int i = 0; i < nc; ++i) {
      if ((int)dims[i].size() / 3 <= l) continue;
      CellDesc cd{};
      cd.nx = dims[i][3 * l];
      cd.ny = dims[i][3 * l + 1];
      cd.nz = dims[i][3 * l + 2];
      cd.id = i;
      cd.parent = l > 0 ? idx_at[l - 1][i] : -1;
      cd.child = -1;
      cd.off = loff;
      cd.h = hs[i] * (double)(1 << l);
      idx_at[l][i] = (int)L.cells.size();
      L.cells.push_back(cd);
      loff += (long long)cd.nx * cd.ny * cd.nz;
      L.maxnz = std::max(L.maxnz, cd.nz);
    }
    L.ntot = loff;
  }
  for (int l = 0; l + 1 < nlev; ++l)
    for (auto& cd : H->levels[l].cells) cd.child = idx_at[l + 1][cd.id];
  for (int l = 0; l < nlev; ++l) {
    Level& L = H->levels[l];
    int maxrow = 1;
    for (auto& cd : L.cells) maxrow = std::max(maxrow, (std::min(cd.ny, 16) + 1) * cd.nz);
    L.NT = std::min(512, std::max(128, pow2ceil(maxrow)));
    if (L.NT < 2 * L.maxnz) L.NT = pow2ceil(2 * L.maxnz);
    if (L.NT > 512) throw FemhError{FEMH_E_ARG, "nz too large for the stencil block"};
    {
      bool same = true;
      for (auto& cd : L.cells) same &= (cd.nz == L.cells[0].nz);
      const int z0 = L.cells[0].nz;
      if (same && (z0 == 16 || z0 == 24 || z0 == 32 || z0 == 48 || z0 == 64 || z0 == 128 || z0 == 256)) {
        L.nz_spec = z0;
        L.NT = (z0 == 24 || z0 == 48) ? 480 : 512;
      }
    }
    {
      bool all_spec = true, same = true;
      for (auto& cd : L.cells) {
        all_spec = all_spec && spec_nz(cd.nz);
        same = same && cd.nz == L.cells[0].nz;
      }
      L.grouped = L.nz_spec == 0 && all_spec && !same;
    }
    // bulk-copy staging needs compile-time z extents with 16-byte rows (all in
    // the compile-time set are multiples of 4); a tile never has more rows than
    // its cell, so each staged array takes at most three row segments (20
    // copies per stage at most, within warp 0's lanes)
    L.bulk_ok = (L.nz_spec > 0 || L.grouped) && L.maxnz <= 128;
    L.bulk_ok64 = L.nz_spec > 0 || L.grouped;
    if (c.stencil_variant > 0) L.variant = c.stencil_variant;
    if (L.variant == 7 && L.grouped) L.variant = 5;   // persistent CTAs need one z extent
    if ((L.variant == 5 || L.variant == 7) && !L.bulk_ok) L.variant = 4;
    int ss = 0, sn = 0;
    for (int ci = 0; ci < (int)L.cells.size(); ++ci) {
      const CellDesc& cd = L.cells[ci];
      L.su_sb.push_back(ss);
      add_stencil_units(L.all.su, ci, cd, cell_nt(L, cd, L.variant), ss, 0, L.variant);
      L.su_se.push_back(ss);
      L.nu_sb.push_back(sn);
      add_node_units(L.all.nu, ci, (long long)cd.nx * cd.ny * cd.nz, sn, l == 0 ? 2048 : 256);
      L.nu_se.push_back(sn);
    }
    L.level = l;
    for (auto& cd : L.cells)
      if (cd.child >= 0) L.nodes_smooth += (long long)cd.nx * cd.ny * cd.nz;
    group_units(L, L.all.su, L.gall, true);
    for (auto& u : L.all.su)
      if (L.cells[u.cell].child >= 0) L.smooth.su.push_back(u);
    group_units(L, L.smooth.su, L.gsmooth, false);
    for (auto& u : L.all.nu)
      if (L.cells[u.cell].child >= 0) L.smooth.nu.push_back(u);
    if (gmg)
      for (int ci = 0; ci < (int)L.cells.size(); ++ci)
        if (L.cells[ci].child < 0) L.coarse_list.push_back(ci);
    L.d_cells = upload(ar, L.cells, s);
    L.all.d_su = upload(ar, L.all.su, s);
    L.all.d_nu = upload(ar, L.all.nu, s);
    L.smooth.d_su = upload(ar, L.smooth.su, s);
    L.smooth.d_nu = upload(ar, L.smooth.nu, s);
    build_cta_table(H, L, L.all, true);
    build_cta_table(H, L, L.smooth, true);
    L.d_su_sb = upload(ar, L.su_sb, s);
    L.d_su_se = upload(ar, L.su_se, s);
    L.d_nu_sb = upload(ar, L.nu_sb, s);
    L.d_nu_se = upload(ar, L.nu_se, s);
    // arrays
    const size_t csz = mg32 ? sizeof(float) : sizeof(double);
    L.kc = ar.get(csz * L.ntot);
    L.invd = ar.arr<float>(L.ntot);
    L.binv = (gmg && c.block_jacobi) ? ar.arr<float>(6 * L.ntot) : nullptr;
    if (l > 0 || gmg) {
      L.xa = ar.get(msz * 18 * L.ntot);
      L.xb = ar.get(msz * 18 * L.ntot);
      if (l > 0) L.bv = ar.get(msz * 18 * L.ntot);
    }
    if (!L.coarse_list.empty()) {
      std::vector<long long> aoff;
      long long o = 0;
      for (int ci : L.coarse_list) {
        const long long m = 3LL * L.cells[ci].nx * L.cells[ci].ny * L.cells[ci].nz;
        aoff.push_back(o);
        o += m * m;
        L.coarse_maxm = std::max<int>(L.coarse_maxm, (int)m);
      }
      L.d_coarse_list = upload(ar, L.coarse_list, s);
      L.d_aoff = upload(ar, aoff, s);
      L.d_A = ar.arr<double>(o);
      L.d_Awork = ar.arr<double>(o);
      L.d_cstat = ar.arr<int>(L.coarse_list.size());
    }
  }
  // ---- fine-level arrays
  const long long nv = H->nvox;
  H->rho_in = ar.arr<double>(nv);
  H->rho_used = ar.arr<double>(nv);
  H->kc64 = ar.arr<double>(nv);
  H->b64 = ar.arr<double>(18 * nv);
  H->x64 = ar.arr<double>(18 * nv);
  if (mixed) H->r64 = ar.arr<double>(18 * nv);
  H->cg_x = mixed ? ar.get(vsz * 18 * nv) : (void*)H->x64;
  H->cg_r = ar.get(vsz * 18 * nv);
  H->cg_p = ar.get(psz * 18 * nv);
  H->cg_q = ar.get(vsz * 18 * nv);
  H->cg_rm = (c.precision == FEMH_MIXED_PC && gmg) ? ar.get(sizeof(float) * 18 * nv) : nullptr;
  H->d_state = ar.arr<CGState>(nc * kNumRhs);
  H->state.assign(nc * kNumRhs, CGState{});
  if (c.autotune) {
    if (mg32 || (mixed && !gmg)) autotune_levels<float>(H, gmg);
    else autotune_levels<double>(H, gmg);
  }
  if (mg32 || mixed) autotune_level0_fp64(H);   // FP64 operator of the mixed modes
  const Level& L0 = H->levels[0];
  H->d_part_s = ar.arr<double>(std::max(L0.all.su.size(), L0.su64.size()) * kNumRhs);
  H->d_part_n = ar.arr<double>(L0.all.nu.size() * kNumRhs * 2);
  H->part_g_slots = L0.all.nu.size();
  // CTAs per level-0 node unit in the block PCG's kernels.  The update and
  // direction kernels (three 256-thread CTAs per SM) get >= 16 CTAs per SM, so
  // the last wave is a small part of the launch (128^3: 1024 units -> 4096
  // CTAs; ncu showed 1024 CTAs in 2.3 waves at 23-33% of the SMs' warps);
  // the Gram kernels only enough for two per SM, because every extra CTA adds
  // 21-36 partial sums that the per-cell finalisation reads back.
  const long long nsm = std::max(H->nsm, 1);
  H->bsub = H->bsub_g = 1;
  while (H->bsub < 32 && (long long)H->part_g_slots * H->bsub < 16 * nsm) H->bsub *= 2;
  while (H->bsub_g < 32 && (long long)H->part_g_slots * H->bsub_g < 2 * nsm) H->bsub_g *= 2;
  H->d_part_g = ar.arr<double>(H->part_g_slots * H->bsub_g * 72);
  H->d_part_b = ar.arr<double>(H->part_g_slots * H->bsub * kNumRhs);
  H->d_bcg = ar.arr<BlockCG>(nc);
  H->d_part_z = ar.arr<double>(std::max(L0.all.nu.size(), L0.all.su.size()) * kNumRhs);
  H->d_part_e = ar.arr<double>(L0.all.nu.size() * 22);   // 21 pair energies + sum of rho per slot
  H->d_C = ar.arr<double>(nc * 36);
  H->d_W = ar.arr<double>(nc * 21);
  H->d_nrm = ar.arr<double>(nc * kNumRhs);
  H->shape_key = shapes;
  H->h_key = hs;
  H->prec_key = c.precision;
  H->solver_key = c.solver;
  H->bf16_key = c.store_bf16;
}


bool verbose() {
  static const int v = [] {
    const char* e = std::getenv("FEMH_VERBOSE");
    return (e && *e && *e != '0') ? 1 : 0;
  }();
  return v != 0;
}


// Batch compaction: restrict every level's unit lists to cells that still
// have an iterating load case (slots keep their numbers, so partial sums and
// per-cell slot ranges stay valid), or restore the full lists.
struct FullLists {
  std::vector<StencilUnit> all_su, smooth_su, su64;
  std::vector<NodeUnit> all_nu, smooth_nu;
};

void set_units(femh_handle* H, Level& L, const FullLists& F, const std::vector<char>* keep) {
  auto filt_s = [&](const std::vector<StencilUnit>& in) {
    std::vector<StencilUnit> out;
    for (const auto& u : in)
      if (!keep || (*keep)[L.cells[u.cell].id]) out.push_back(u);
    return out;
  };
  auto filt_n = [&](const std::vector<NodeUnit>& in) {
    std::vector<NodeUnit> out;
    for (const auto& u : in)
      if (!keep || (*keep)[L.cells[u.cell].id]) out.push_back(u);
    return out;
  };
  cudaStream_t s = H->stream;
  // copies come from the level's own (persistent) host vectors
  auto put_s = [&](std::vector<StencilUnit>& dst, StencilUnit* d, std::vector<StencilUnit> v) {
    dst.swap(v);
    if (!dst.empty())
      CK(cudaMemcpyAsync(d, dst.data(), sizeof(StencilUnit) * dst.size(), cudaMemcpyHostToDevice, s));
  };
  auto put_n = [&](std::vector<NodeUnit>& dst, NodeUnit* d, std::vector<NodeUnit> v) {
    dst.swap(v);
    if (!dst.empty()) CK(cudaMemcpyAsync(d, dst.data(), sizeof(NodeUnit) * dst.size(), cudaMemcpyHostToDevice, s));
  };
  put_s(L.all.su, L.all.d_su, filt_s(F.all_su));
  put_s(L.smooth.su, L.smooth.d_su, filt_s(F.smooth_su));
  build_cta_table(H, L, L.all, false);
  build_cta_table(H, L, L.smooth, false);
  if (L.use64) put_s(L.su64, L.d_su64, filt_s(F.su64));
  group_units(L, L.all.su, L.gall, false);   // filtering keeps the z-extent order
  group_units(L, L.smooth.su, L.gsmooth, false);
  if (L.use64) group_units(L, L.su64, L.g64, false);
  put_n(L.all.nu, L.all.d_nu, filt_n(F.all_nu));
  put_n(L.smooth.nu, L.smooth.d_nu, filt_n(F.smooth_nu));
}

// (Re)build a level's stencil unit lists for an x-chunk length.
void build_stencil_units(femh_handle* H, Level& L, int chunk) {
  L.chunk = chunk;
  L.all.su.clear();
  L.smooth.su.clear();
  L.su_sb.clear();
  L.su_se.clear();
  int ss = 0;
  for (int ci = 0; ci < (int)L.cells.size(); ++ci) {
    L.su_sb.push_back(ss);
    add_stencil_units(L.all.su, ci, L.cells[ci], cell_nt(L, L.cells[ci], L.variant), ss, chunk, L.variant);
    L.su_se.push_back(ss);
  }
  group_units(L, L.all.su, L.gall, true);
  for (auto& u : L.all.su)
    if (L.cells[u.cell].child >= 0) L.smooth.su.push_back(u);
  group_units(L, L.smooth.su, L.gsmooth, false);
  cudaStream_t s = H->stream;
  Arena& ar = H->setup;
  L.all.d_su = upload(ar, L.all.su, s);
  L.smooth.d_su = upload(ar, L.smooth.su, s);
  L.d_su_sb = upload(ar, L.su_sb, s);
  L.d_su_se = upload(ar, L.su_se, s);
  build_cta_table(H, L, L.all, true);
  build_cta_table(H, L, L.smooth, true);
}

void build_stencil_units64(femh_handle* H, Level& L, int chunk, int variant) {
  L.use64 = true;
  L.variant64 = variant;
  L.chunk64 = chunk;
  L.su64.clear();
  L.su64_sb.clear();
  L.su64_se.clear();
  int ss = 0;
  for (int ci = 0; ci < (int)L.cells.size(); ++ci) {
    L.su64_sb.push_back(ss);
    add_stencil_units(L.su64, ci, L.cells[ci], cell_nt(L, L.cells[ci], variant), ss, chunk, variant);
    L.su64_se.push_back(ss);
  }
  group_units(L, L.su64, L.g64, true);
  cudaStream_t s = H->stream;
  Arena& ar = H->setup;
  L.d_su64 = upload(ar, L.su64, s);
  L.d_su64_sb = upload(ar, L.su64_sb, s);
  L.d_su64_se = upload(ar, L.su64_se, s);
}

// FP64 layout of level 0 (mixed modes): variant x chunk timed with the FP64 operator.
void autotune_level0_fp64(femh_handle* H) {
  Level& L = H->levels[0];
  cudaStream_t s = H->stream;
  std::string key = "f64L0:" + std::to_string(L.NT) + ":" + std::to_string(H->cfg.stencil_variant);
  int maxnx = 1;
  for (auto& cd : L.cells) {
    key += ":" + std::to_string(cd.nx) + "x" + std::to_string(cd.ny) + "x" + std::to_string(cd.nz);
    maxnx = std::max(maxnx, cd.nx);
  }
  auto it = H->tune_cache.find(key);
  if (it != H->tune_cache.end()) {
    build_stencil_units64(H, L, it->second / 16, it->second % 16);
    return;
  }
  if (!H->cfg.autotune || L.ntot < 4096) {
    build_stencil_units64(H, L, 0, 1);
    H->tune_cache[key] = 0 * 16 + 1;
    return;
  }
  double* in = H->x64;
  double* out = H->b64;
  CK(cudaMemsetAsync(H->kc64, 0, sizeof(double) * L.ntot, s));
  CK(cudaMemsetAsync(in, 0, sizeof(double) * 18 * L.ntot, s));
  int best = 0, best_var = 1;
  float best_ms = 1e30f;
  std::vector<int> cands;
  for (int cand : {4, 8, 16, 32, 64, maxnx})
    if (cand <= maxnx && std::find(cands.begin(), cands.end(), cand) == cands.end()) cands.push_back(cand);
  // large levels favour long chunks: scan from the longest, so the 25% rule
  // stops before the slow short ones
  if (L.ntot > (1 << 20)) std::reverse(cands.begin(), cands.end());
  std::vector<int> vars64 = {1, 2};
  if (L.bulk_ok64) vars64.push_back(6);
  if (H->cfg.stencil_variant == 6 && L.bulk_ok64) vars64 = {6};
  for (int var : vars64) {   // pruned as in autotune_levels
    float var_best = 1e30f;
    for (int cand : cands) {
      build_stencil_units64(H, L, cand, var);
      float ms_min = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        CK(cudaEventRecord(H->ev0, s));
        stencil<double, OUT_APPLY>(H, L, false, (const double*)in, out, (const double*)nullptr,
                                   (const double*)H->kc64, nullptr, nullptr, 0.0);
        CK(cudaEventRecord(H->ev1, s));
        CK(cudaEventSynchronize(H->ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
        ms_min = std::min(ms_min, ms);
        if (ms_min > 8.0f || (rep >= 1 && ms_min > 2.0f)) break;   // one sample of a long launch suffices
      }
      if (verbose()) std::fprintf(stderr, "[femh] tune level 0 fp64 variant %d chunk %d: %.4f ms\n", var, cand, ms_min);
      if (ms_min < best_ms) {
        best_ms = ms_min;
        best = cand;
        best_var = var;
      }
      var_best = std::min(var_best, ms_min);
      if (ms_min > 1.25f * var_best) break;
    }
  }
  build_stencil_units64(H, L, best, best_var);
  H->tune_cache[key] = best * 16 + best_var;
}

// Project autotuner for the stencil's tile shape: for every level whose
// stencil runs, time the damped-Jacobi sweep (the most launched mode) for
// x-chunk lengths {1, 2, 4, 8, 16, 32, 64, whole cell} on the level's own buffers
// and keep the fastest.  Results are cached per level signature in the handle.
template <typename T>
void autotune_levels(femh_handle* H, bool mg) {
  cudaStream_t s = H->stream;
  for (size_t l = 0; l < H->levels.size(); ++l) {
    Level& L = H->levels[l];
    const bool smooth = mg && l > 0;   // coarse levels only run smoothing sweeps
    if ((smooth ? L.smooth.su : L.all.su).empty()) continue;
    std::string key = std::to_string(l) + ":" + std::to_string(L.NT) + ":" + std::to_string(sizeof(T)) + ":" +
                      std::to_string(H->cfg.stencil_variant);
    int maxnx = 1;
    for (auto& cd : L.cells) {
      key += ":" + std::to_string(cd.nx) + "x" + std::to_string(cd.ny) + "x" + std::to_string(cd.nz);
      maxnx = std::max(maxnx, cd.nx);
    }
    auto it = H->tune_cache.find(key);
    if (it != H->tune_cache.end()) {   // cached: chunk * 16 + variant
      L.variant = it->second % 16;
      build_stencil_units(H, L, it->second / 16);
      continue;
    }
    T* in = (T*)(L.xa ? L.xa : H->cg_r);
    T* out = (T*)(L.xb ? L.xb : H->cg_q);
    CK(cudaMemsetAsync(L.kc, 0, sizeof(T) * L.ntot, s));
    CK(cudaMemsetAsync(L.invd, 0, sizeof(float) * L.ntot, s));
    CK(cudaMemsetAsync(in, 0, sizeof(T) * 18 * L.ntot, s));
    int best = L.chunk, best_var = L.variant;
    float best_ms = 1e30f;
    // short x-chunks give small, latency-bound levels more CTAs of fewer steps
    std::vector<int> cands;
    for (int cand : {1, 2, 4, 8, 16, 32, 64, maxnx})
      if (cand <= maxnx && std::find(cands.begin(), cands.end(), cand) == cands.end()) cands.push_back(cand);
    // large levels favour long chunks: scan from the longest (the 25% rule below
    // then stops before the slow short ones); small levels from the shortest
    if (L.ntot > (1 << 20)) std::reverse(cands.begin(), cands.end());
    const int reps = L.ntot < 65536 ? 7 : 3;   // small levels time in microseconds: more samples
    std::vector<int> vars = {1, 2};
    if (std::is_same<T, float>::value) vars = {2, 3, 4};
    if (std::is_same<T, float>::value && L.bulk_ok) vars.push_back(5);
    // persistent CTAs (statically balanced) on single-cell levels: in a batch the
    // cells converge at different iterations and one CTA per unit balances itself
    if (std::is_same<T, float>::value && L.bulk_ok && !L.grouped && L.cells.size() == 1) vars.push_back(7);
    if (std::is_same<T, double>::value && L.bulk_ok64) vars.push_back(6);
    if (H->cfg.stencil_variant > 0) vars = {H->cfg.stencil_variant};
    // a variant's scan stops once a chunk is 25% slower than its best so far
    // (the time is unimodal in the chunk); launches of a few
    // milliseconds are stable after two samples, launches over 8 ms after one
    for (int var : vars) {
    float var_best = 1e30f;
    for (int cand : cands) {
      // persistent CTAs stream across units; their dot sums close per unit, so
      // units shorter than 8 planes would add reductions without balancing better
      if (var == 7 && cand < 8 && cand < maxnx) continue;
      L.variant = var;
      build_stencil_units(H, L, cand);
      float ms_min = 1e30f;
      for (int rep = 0; rep < reps; ++rep) {
        CK(cudaEventRecord(H->ev0, s));
        stencil<T, OUT_JACOBI>(H, L, smooth, (const T*)in, out, (const T*)in, (const T*)L.kc, nullptr, nullptr,
                               0.5);
        CK(cudaEventRecord(H->ev1, s));
        CK(cudaEventSynchronize(H->ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
        ms_min = std::min(ms_min, ms);
        if (ms_min > 8.0f || (rep >= 1 && ms_min > 2.0f)) break;   // one sample of a long launch suffices
      }
      if (verbose()) std::fprintf(stderr, "[femh] tune level %zu variant %d chunk %d: %.4f ms\n", l, var, cand, ms_min);
      if (ms_min < best_ms) {
        best_ms = ms_min;
        best = cand;
        best_var = var;
      }
      var_best = std::min(var_best, ms_min);
      if (ms_min > 1.25f * var_best) break;
    }
    }
    L.variant = best_var;
    build_stencil_units(H, L, best);
    H->tune_cache[key] = best * 16 + best_var;
  }
}

// coefficients on all levels + inverse diagonals + coarse factorisations
template <typename TC>
void prepare_operator(femh_handle* H) {
  const femh_config& c = H->cfg;
  cudaStream_t s = H->stream;
  Level& L0 = H->levels[0];
  const MatLaw law = make_law(c);
  {
    Prof prof_(H, "k_coef", 0.0);
    k_coef<TC><<<(unsigned)L0.all.nu.size(), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, H->rho_in, law, H->kc64,
                                                        std::is_same<TC, double>::value ? nullptr : (TC*)L0.kc,
                                                        H->rho_used, H->d_err + 1);
    LAUNCH_CHECK(H);
  }
  if (std::is_same<TC, double>::value)
    CK(cudaMemcpyAsync(L0.kc, H->kc64, sizeof(double) * H->nvox, cudaMemcpyDeviceToDevice, s));
  for (size_t l = 1; l < H->levels.size(); ++l) {
    Level& L = H->levels[l];
    Level& F = H->levels[l - 1];
    {
      Prof prof_(H, "k_coarsen_coef", 0.0);
      k_coarsen_coef<TC, TC><<<(unsigned)L.all.nu.size(), 256, 0, s>>>(F.d_cells, L.d_cells, L.all.d_nu,
                                                                     (const TC*)F.kc, (TC*)L.kc, c.coarse_avg);
      LAUNCH_CHECK(H);
    }
  }
  for (auto& L : H->levels) {
    {
      Prof prof_(H, "k_invdiag", 0.0);
      k_invdiag<TC><<<(unsigned)L.all.nu.size(), 256, 0, s>>>(L.d_cells, L.all.d_nu, (const TC*)L.kc,
                                                            H->hk.diag, L.invd);
      LAUNCH_CHECK(H);
    }
    if (L.binv) {
      Prof prof_(H, "k_invblock", 0.0);
      k_invblock<TC><<<(unsigned)L.all.nu.size(), 256, 0, s>>>(L.d_cells, L.all.d_nu, (const TC*)L.kc, H->K0[0],
                                                             H->K0[1], L.binv);
      LAUNCH_CHECK(H);
    }
    if (!L.coarse_list.empty()) {
      const unsigned n = (unsigned)L.coarse_list.size();
      {
        Prof prof_(H, "k_coarse_assemble", 0.0);
        k_coarse_assemble<TC><<<n, 256, 0, s>>>(L.d_cells, L.d_coarse_list, (const TC*)L.kc, H->d_K0, L.d_A,
                                              L.d_aoff);
        LAUNCH_CHECK(H);
      }
      {
        Prof prof_(H, "k_coarse_factor", 0.0);
        if (L.coarse_maxm <= kCoarseSmemM) {   // packed triangle in shared memory
          static bool attr = false;
          if (!attr) {
            CK(cudaFuncSetAttribute(k_coarse_factor_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)coarse_factor_smem_bytes(kCoarseSmemM)));
            attr = true;
          }
          k_coarse_factor_smem<<<n, 1024, coarse_factor_smem_bytes(L.coarse_maxm), s>>>(
              L.d_cells, L.d_coarse_list, L.d_A, L.d_aoff, L.d_cstat);
        } else {
          k_coarse_factor<<<n, 256, 0, s>>>(L.d_cells, L.d_coarse_list, L.d_A, L.d_Awork, L.d_aoff, L.d_cstat);
        }
        LAUNCH_CHECK(H);
      }
    }
  }
  // loads
  {
    Prof prof_(H, "k_rhs", 0.0);
    k_rhs<double><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, H->kc64, H->d_ec, H->b64, L0.ntot);
    LAUNCH_CHECK(H);
  }
}


unsigned fin_blocks(int nc) { return cdiv((long long)nc * kNumRhs * 32, 128); }   // a warp per (cell, rhs)

// The z . r product of the multigrid preconditioner comes out of the last
// level-0 post-smoothing sweep when every level-0 cell is smoothed there (no
// cell is solved directly on level 0) and there is such a sweep.
bool fuse_rz(const femh_handle* H) {
  const Level& L0 = H->levels[0];
  return H->cfg.solver == FEMH_GMG_PCG && H->cfg.post_smooth > 0 && L0.coarse_list.empty() &&
         L0.smooth.su.size() == L0.all.su.size();
}

// One V-cycle of the multigrid preconditioner: z = V(r0), levels in TM
// arithmetic/storage with coefficients TMC; r0 (level-0 right-hand side) may
// be of another type (FP64 CG residual feeding an FP32 V-cycle).  Level 0's xa
// must already hold the first damped-Jacobi sweep w_pre[0]*invd*r0 (written by
// the CG update kernel); each coarser level's xa is written by the restriction
// that forms its right-hand side.  Buffer roles are fixed by the sweep counts, so the
// launch sequence is identical every iteration (graph capture).
// Profile name of a per-level kernel ("<base>_L<level>"), interned in the
// handle's statistics map so that the pointer stays valid.
const char* level_name(femh_handle* H, const char* base, int level) {
  if (!H->prof) return base;
  const std::string k = std::string(base) + "_L" + std::to_string(level);
  return H->kstats.emplace(k, femh_handle::KStat{}).first->first.c_str();
}

template <typename TM, typename TMC, typename TB>
void vcycle_level_down(femh_handle* H, int l, const TB* b, TM* cur, TM* oth, TM* sol) {
  const femh_config& c = H->cfg;
  cudaStream_t s = H->stream;
  const std::vector<double>& w = H->w_pre;
  const CGState* stt = H->d_state;
  Level& L = H->levels[l];
  if (!L.coarse_list.empty()) {
    dim3 g((unsigned)L.coarse_list.size(), kNumRhs);
    Prof prof_(H, "k_coarse_solve", 0.0);
    k_coarse_solve<TB, TM><<<g, 1024, sizeof(double) * L.coarse_maxm, s>>>(
        L.d_cells, L.d_coarse_list, L.d_A, L.d_aoff, b, sol, stt, L.ntot);
    LAUNCH_CHECK(H);
  }
  if (L.smooth.su.empty()) return;
  for (int sw = 1; sw < c.pre_smooth; ++sw) {
    stencil<TM, OUT_JACOBI>(H, L, true, (const TM*)cur, oth, b, (const TMC*)L.kc, nullptr, stt, w[sw]);
    std::swap(cur, oth);
  }
  stencil<TM, OUT_RESID>(H, L, true, (const TM*)cur, oth, b, (const TMC*)L.kc, nullptr, stt, w[0]);
  Level& C = H->levels[l + 1];
  const bool c_smooth = !C.smooth.su.empty();   // also C's first sweep from a zero guess
  Prof prof_(H, level_name(H, "k_restrict", l),
             18.0 * sizeof(TM) * (L.nodes_smooth + C.ntot) + (c_smooth ? (18.0 * sizeof(TM) + (C.binv ? 24.0 : 4.0)) * C.nodes_smooth : 0.0));
  k_restrict<TM, TM><<<NODE_GRID(C.all), 256, 0, s>>>(L.d_cells, C.d_cells, C.all.d_nu, oth, (TM*)C.bv,
                                                      c_smooth ? (TM*)C.xa : (TM*)nullptr, C.invd, w[0], stt,
                                                      L.ntot, C.ntot, C.binv);
  LAUNCH_CHECK(H);
}

template <typename TM, typename TMC, typename TB>
void vcycle_level_up(femh_handle* H, int l, const TB* b, TM* x, TM* t, const TM* coarse_sol, double* dot_part) {
  const femh_config& c = H->cfg;
  cudaStream_t s = H->stream;
  const CGState* stt = H->d_state;
  Level& L = H->levels[l];
  if (L.smooth.su.empty()) return;
  Level& C = H->levels[l + 1];
  {
    Prof prof_(H, level_name(H, "k_prolong_add", l), 18.0 * sizeof(TM) * (2.0 * L.nodes_smooth + C.ntot));
    k_prolong_add<TM, TM><<<NODE_GRID(L.smooth), 256, 0, s>>>(L.d_cells, C.d_cells, L.smooth.d_nu, x, coarse_sol,
                                                              stt, L.ntot, C.ntot);
    LAUNCH_CHECK(H);
  }
  for (int sw = 0; sw < c.post_smooth; ++sw) {
    if (dot_part && sw + 1 == c.post_smooth)   // last sweep also forms z . b
      stencil<TM, OUT_JACOBI_DOT>(H, L, true, (const TM*)x, t, b, (const TMC*)L.kc, dot_part, stt, H->w_post[sw]);
    else
      stencil<TM, OUT_JACOBI>(H, L, true, (const TM*)x, t, b, (const TMC*)L.kc, nullptr, stt, H->w_post[sw]);
    std::swap(x, t);
  }
}

// dot_part != nullptr: the last level-0 sweep writes the z . r0 partials
// there (per stencil unit slot).
template <typename TM, typename TMC, typename TR>
TM* vcycle(femh_handle* H, const TR* r0, double* dot_part) {
  const femh_config& c = H->cfg;
  const int nlev = (int)H->levels.size();
  std::vector<TM*> sm(nlev), tmp(nlev), sol(nlev);
  for (int l = 0; l < nlev; ++l) {
    Level& L = H->levels[l];
    TM* cur = (TM*)L.xa;
    TM* oth = (TM*)L.xb;
    if ((c.pre_smooth - 1) % 2 == 1) std::swap(cur, oth);   // where the pre-smoothed iterate ends
    sm[l] = cur;
    tmp[l] = oth;
    sol[l] = (c.post_smooth % 2 == 0) ? cur : oth;
  }
  for (int l = 0; l < nlev; ++l) {
    if (l == 0) vcycle_level_down<TM, TMC, TR>(H, 0, r0, (TM*)H->levels[0].xa, (TM*)H->levels[0].xb, sol[0]);
    else vcycle_level_down<TM, TMC, TM>(H, l, (const TM*)H->levels[l].bv, (TM*)H->levels[l].xa,
                                         (TM*)H->levels[l].xb, sol[l]);
  }
  for (int l = nlev - 2; l >= 0; --l) {
    if (l == 0) vcycle_level_up<TM, TMC, TR>(H, 0, r0, sm[0], tmp[0], sol[1], dot_part);
    else vcycle_level_up<TM, TMC, TM>(H, l, (const TM*)H->levels[l].bv, sm[l], tmp[l], sol[l + 1], nullptr);
  }
  return sol[0];
}

// Solver precisions: TV = CG vectors, TP = search direction storage, TK = CG
// operator coefficients, TM / TMC = multigrid level vectors / coefficients.
template <typename TV, typename TP, typename TK, typename TM, typename TMC>
struct Prec {
  using V = TV;
  using P = TP;
  using K = TK;
  using M = TM;
  using MC = TMC;
};

// Block PCG: directions dropped from G = P^T K P below this pivot ratio
// (dependent to the accuracy of the preconditioned block: an FP32 V-cycle
// resolves ~1e-4 in angle, an FP64 one ~1e-6 is still meaningful).
template <typename TM> constexpr double block_drop() { return sizeof(TM) == 8 ? 1e-12 : 1e-8; }

// Partials of a 6x6 product A^T B of each cell's block: the upper triangle
// (SYM) or all 36 entries, per node slot, into `part`.
template <bool SYM, typename TA, typename TB>
void block_gram(femh_handle* H, const char* name, const TA* a, const TB* b, double* part) {
  Level& L0 = H->levels[0];
  const dim3 grid((unsigned)(L0.all.nu.size() * H->bsub_g));
  Prof prof_(H, name, 18.0 * (sizeof(TA) + sizeof(TB)) * (double)L0.ntot);
  k_bgram<SYM, TA, TB><<<grid, 256, 0, H->stream>>>(L0.d_cells, L0.all.d_nu, a, b, H->d_bcg, part, L0.ntot,
                                                    H->bsub_g);
  LAUNCH_CHECK(H);
}

// One block PCG iteration of the multigrid PCG (all live cells).
template <class PR>
void pcg_iteration_block(femh_handle* H, const typename PR::K* kcg) {
  using TV = typename PR::V;
  using TP = typename PR::P;
  using TM = typename PR::M;
  using TMC = typename PR::MC;
  cudaStream_t s = H->stream;
  Level& L0 = H->levels[0];
  const int nc = H->ncells;
  const int nsub = H->bsub;
  const dim3 grid((unsigned)(L0.all.nu.size() * nsub));
  TV* x = (TV*)H->cg_x;
  TV* r = (TV*)H->cg_r;
  TP* p = (TP*)H->cg_p;
  TV* q = (TV*)H->cg_q;
  TM* rm = (sizeof(TM) != sizeof(TV)) ? (TM*)H->cg_rm : nullptr;
  CGState* stt = H->d_state;
  const int nsub_g = H->bsub_g;
  double* part_a = H->d_part_g;                                        // [Gram sub-slots][36]
  double* part_b = H->d_part_g + H->part_g_slots * nsub_g * 36;        // [Gram sub-slots][36]
  stencil<TV, OUT_APPLY_DOT>(H, L0, false, (const TP*)p, q, (const TV*)nullptr, kcg, H->d_part_s, stt, 0.0);
  block_gram<true, TP, TV>(H, "k_bgram_pq", (const TP*)p, (const TV*)q, part_a);
  {
    Prof prof_(H, "k_bfin_alpha", 0.0);
    k_bfin_alpha<<<nc, 256, 0, s>>>(H->d_bcg, stt, L0.d_nu_sb, L0.d_nu_se, part_a, nc, block_drop<TM>(), nsub_g);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_bupdate",
               18.0 * (5 * sizeof(TV) + sizeof(TP) + sizeof(TM) + (rm ? sizeof(TM) : 0)) * (double)L0.ntot +
                   (L0.binv ? 24.0 : 4.0) * (double)L0.ntot);
    k_bupdate<TV, TP, TV, TM><<<grid, 256, 0, s>>>(L0.d_cells, L0.all.d_nu, x, r, p, q, L0.invd, (TM*)L0.xa, rm,
                                                   H->w_pre[0], H->d_bcg, H->d_part_b, L0.ntot, L0.binv, nsub);
    LAUNCH_CHECK(H);
  }
  TM* z = rm ? vcycle<TM, TMC, TM>(H, rm, nullptr) : vcycle<TM, TMC, TV>(H, r, nullptr);
  block_gram<false, TM, TV>(H, "k_bgram_zr", (const TM*)z, (const TV*)r, part_a);
  block_gram<false, TV, TM>(H, "k_bgram_qz", (const TV*)q, (const TM*)z, part_b);
  {
    Prof prof_(H, "k_bfin_beta", 0.0);
    k_bfin_beta<<<nc, 256, 0, s>>>(H->d_bcg, stt, L0.d_nu_sb, L0.d_nu_se, H->d_part_b, part_a, part_b, nc,
                                   block_drop<TM>(), nsub_g, nsub);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_bdir", 18.0 * (sizeof(TM) + 2 * sizeof(TP)) * (double)L0.ntot);
    k_bdir<TP, TM><<<grid, 256, 0, s>>>(L0.d_cells, L0.all.d_nu, p, (const TM*)z, H->d_bcg, L0.ntot, 0, nsub);
    LAUNCH_CHECK(H);
  }
}

// One PCG iteration (all cells / load cases; inactive ones skip their work).
template <class PR>
void pcg_iteration(femh_handle* H, const typename PR::K* kcg, bool blk) {
  if (blk) return pcg_iteration_block<PR>(H, kcg);
  using TV = typename PR::V;
  using TP = typename PR::P;
  using TM = typename PR::M;
  using TMC = typename PR::MC;
  const femh_config& c = H->cfg;
  cudaStream_t s = H->stream;
  Level& L0 = H->levels[0];
  const int nc = H->ncells;
  const bool gmg = c.solver == FEMH_GMG_PCG;
  TV* x = (TV*)H->cg_x;
  TV* r = (TV*)H->cg_r;
  TP* p = (TP*)H->cg_p;
  TV* q = (TV*)H->cg_q;
  TM* rm = (gmg && sizeof(TM) != sizeof(TV)) ? (TM*)H->cg_rm : nullptr;
  CGState* stt = H->d_state;
  stencil<TV, OUT_APPLY_DOT>(H, L0, false, (const TP*)p, q, (const TV*)nullptr, kcg, H->d_part_s, stt, 0.0);
  {
    Prof prof_(H, "k_fin_alpha", 0.0);
    const bool l64 = sizeof(TV) == 8 && L0.use64;   // the apply above used the FP64 layout
    k_fin_alpha<<<fin_blocks(nc), 128, 0, s>>>(stt, l64 ? L0.d_su64_sb : L0.d_su_sb,
                                               l64 ? L0.d_su64_se : L0.d_su_se, H->d_part_s, nc);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_cg_update",
               (18.0 * (5 * sizeof(TV) + sizeof(TP) + (gmg ? sizeof(TM) : 0) + (rm ? sizeof(TM) : 0)) + 4.0) *
                   (double)L0.ntot);
    k_cg_update<TV, TP, TV, TM><<<NODE_GRID(L0.all), 256, 0, s>>>(
        L0.d_cells, L0.all.d_nu, x, r, p, q, L0.invd, gmg ? (TM*)L0.xa : (TM*)nullptr, rm, H->w_pre[0], stt,
        H->d_part_n, L0.ntot, L0.binv);
    LAUNCH_CHECK(H);
  }
  TM* z = nullptr;
  const bool fuse = fuse_rz(H);
  if (gmg) {
    double* dp = fuse ? H->d_part_z : nullptr;
    z = rm ? vcycle<TM, TMC, TM>(H, rm, dp) : vcycle<TM, TMC, TV>(H, r, dp);
    if (!fuse) {
      Prof prof_(H, "k_dot", 0.0);
      k_dot<TM, TV><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, z, r, stt, H->d_part_z, L0.ntot);
      LAUNCH_CHECK(H);
    }
  }
  {
    Prof prof_(H, "k_fin_beta", 0.0);
    k_fin_beta<<<fin_blocks(nc), 128, 0, s>>>(stt, L0.d_nu_sb, L0.d_nu_se, fuse ? L0.d_su_sb : L0.d_nu_sb,
                                              fuse ? L0.d_su_se : L0.d_nu_se, H->d_part_n, H->d_part_z, nc,
                                              gmg ? 0 : 1);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_cg_dir", 18.0 * (sizeof(TM) + 2 * sizeof(TP)) * (double)L0.ntot);
    k_cg_dir<TP, TM, TV><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, p, (const TM*)z,
                                                           (const TV*)r, L0.invd, stt, L0.ntot);
    LAUNCH_CHECK(H);
  }
}

// PCG on K x = scale*b for every (cell, rhs) whose state is active.
// warm: x already holds the starting iterate and b is its residual; the
// relative residual is measured against ||b_orig||^2 in H->d_nrm.
// block: the GMG-PCG of the FP64 CG modes runs as block PCG over each cell's
// load cases (config block_cg); a cell whose block fails is solved again one
// load case at a time, from zero on the unreduced right-hand side H->b64.
template <class PR, typename TB>
void pcg(femh_handle* H, const TB* b, const typename PR::K* kcg, int max_iter, double tol, int iters_out[],
         bool warm = false, bool block = true) {
  using TV = typename PR::V;
  using TP = typename PR::P;
  using TM = typename PR::M;
  using TMC = typename PR::MC;
  const femh_config& c = H->cfg;
  cudaStream_t s = H->stream;
  Level& L0 = H->levels[0];
  const int nc = H->ncells;
  const bool gmg = c.solver == FEMH_GMG_PCG;
  TV* x = (TV*)H->cg_x;
  TV* r = (TV*)H->cg_r;
  TP* p = (TP*)H->cg_p;
  TM* rm = (gmg && sizeof(TM) != sizeof(TV)) ? (TM*)H->cg_rm : nullptr;
  CGState* stt = H->d_state;
  const bool blk = block && block_pcg(c) && sizeof(TV) == 8 && sizeof(TP) == 8;
  for (auto& S : H->state) {
    S.tol = tol;
    S.max_iter = max_iter;
    S.iters = 0;
  }
  CK(cudaMemcpyAsync(stt, H->state.data(), sizeof(CGState) * H->state.size(), cudaMemcpyHostToDevice, s));
  {
    Prof prof_(H, "k_cg_init", 0.0);
    k_cg_init<TB, TV, TP><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, b, x, r, p, L0.invd, stt,
                                                            H->d_part_n, L0.ntot, gmg ? 0 : 1, warm ? 1 : 0);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_fin_init", 0.0);
    k_fin_init<<<fin_blocks(nc), 128, 0, s>>>(stt, L0.d_nu_sb, L0.d_nu_se, H->d_part_n, nc, gmg ? 0 : 1,
                                              warm ? H->d_nrm : nullptr);
    LAUNCH_CHECK(H);
  }
  if (gmg) {
    {
      Prof prof_(H, "k_jacobi0", 0.0);
      k_jacobi0<TV, TM><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, r, (TM*)L0.xa, rm,
                                                          L0.invd, H->w_pre[0], stt, L0.ntot, L0.binv);
      LAUNCH_CHECK(H);
    }
    if (blk) {   // block PCG: Z^T R of the start, P = Z
      {
        Prof prof_(H, "k_binit", 0.0);
        k_binit<<<cdiv(nc, 128), 128, 0, s>>>(H->d_bcg, stt, nc);
        LAUNCH_CHECK(H);
      }
      TM* z = rm ? vcycle<TM, TMC, TM>(H, rm, nullptr) : vcycle<TM, TMC, TV>(H, r, nullptr);
      block_gram<false, TM, TV>(H, "k_bgram_zr", (const TM*)z, (const TV*)r, H->d_part_g);
      {
        Prof prof_(H, "k_bfin_rz", 0.0);
        k_bfin_rz<<<nc, 256, 0, s>>>(H->d_bcg, stt, L0.d_nu_sb, L0.d_nu_se, H->d_part_g, nc, H->bsub_g);
        LAUNCH_CHECK(H);
      }
      {
        Prof prof_(H, "k_bdir", 0.0);
        k_bdir<TP, TM><<<dim3((unsigned)(L0.all.nu.size() * H->bsub)), 256, 0, s>>>(
            L0.d_cells, L0.all.d_nu, p, (const TM*)z, H->d_bcg, L0.ntot, 1, H->bsub);
        LAUNCH_CHECK(H);
      }
    }
  }
  if (gmg && !blk) {
    const bool fuse = fuse_rz(H);
    double* dp = fuse ? H->d_part_z : nullptr;
    TM* z = rm ? vcycle<TM, TMC, TM>(H, rm, dp) : vcycle<TM, TMC, TV>(H, r, dp);
    if (!fuse) {
      Prof prof_(H, "k_dot", 0.0);
      k_dot<TM, TV><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, z, r, stt, H->d_part_z, L0.ntot);
      LAUNCH_CHECK(H);
    }
    {
      Prof prof_(H, "k_fin_rz", 0.0);
      k_fin_rz<<<fin_blocks(nc), 128, 0, s>>>(stt, L0.d_nu_sb, L0.d_nu_se, fuse ? L0.d_su_sb : L0.d_nu_sb,
                                              fuse ? L0.d_su_se : L0.d_nu_se, H->d_part_z, H->d_part_n, nc);
      LAUNCH_CHECK(H);
    }
    {   // p = z (beta = 0; Jacobi z for pairs that fell back)
      Prof prof_(H, "k_cg_dir", 0.0);
      k_cg_dir<TP, TM, TV><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, p, (const TM*)z,
                                                             (const TV*)r, L0.invd, stt, L0.ntot);
      LAUNCH_CHECK(H);
    }
  }
  const int chunk = H->prof ? 1 : std::max(1, c.graph_chunk > 0 ? c.graph_chunk : 8);
  // The iterations run on the device without the host: a CUDA graph whose
  // WHILE node repeats `chunk` captured iterations while k_while_cond finds
  // live cells (and, for a batch, more than half of the listed ones); the host
  // wakes only to compact a batch's unit lists or at the end.
  cudaGraphExec_t exec = nullptr;
  long long graph_kernels = 0;   // kernels of one pass of the loop body
  int listed = nc;               // cells covered by the current unit lists
  const int limit = max_iter + chunk;
  CK(cudaMemsetAsync(H->d_loop, 0, sizeof(int), s));
  auto capture = [&]() {
    if (!(c.graph_chunk > 0 && !H->prof)) return;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    cudaGraph_t body = nullptr;
    try {
      CK(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = cond;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      CK(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
      body = cp.conditional.phGraph_out[0];
    } catch (...) {
      cudaGraphDestroy(g);
      throw;
    }
    H->capturing = true;
    H->cap_count = 0;
    CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
      for (int i = 0; i < chunk; ++i) pcg_iteration<PR>(H, kcg, blk);
      k_while_cond<<<1, 1024, 0, s>>>(cond, H->d_state, nc, listed, H->d_loop, chunk, limit);
      LAUNCH_CHECK(H);
    } catch (...) {
      H->capturing = false;
      cudaGraph_t tmp = nullptr;
      cudaStreamEndCapture(s, &tmp);
      cudaGraphDestroy(g);
      throw;
    }
    H->capturing = false;
    graph_kernels = H->cap_count;
    cudaGraph_t got = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &got);
    if (ee != cudaSuccess) {
      cudaGraphDestroy(g);
      CK(ee);
    }
    const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
  };
  // batch compaction bookkeeping
  std::vector<FullLists> full;
  auto restore = [&]() {
    if (full.empty()) return;
    for (size_t l = 0; l < H->levels.size(); ++l) set_units(H, H->levels[l], full[l], nullptr);
    full.clear();
  };
  capture();
  int done = 0;
  const auto t_start = std::chrono::steady_clock::now();
  try {
    while (true) {
      if (exec) {
        int loop_now = done;
        CK(cudaGraphLaunch(exec, s));
        CK(cudaMemcpyAsync(&loop_now, H->d_loop, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(H->state.data(), stt, sizeof(CGState) * H->state.size(), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        H->launches += graph_kernels * (long long)std::max(1, (loop_now - done) / chunk);
        done = loop_now;
      } else {
        for (int i = 0; i < chunk; ++i) pcg_iteration<PR>(H, kcg, blk);
        done += chunk;
        CK(cudaMemcpyAsync(H->state.data(), stt, sizeof(CGState) * H->state.size(), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
      }
      prof_resolve(H);
      std::vector<char> keep(nc, 0);
      int alive = 0;
      for (int t = 0; t < nc * kNumRhs; ++t)
        if (H->state[t].active) keep[t / kNumRhs] = 1;
      for (int ci = 0; ci < nc; ++ci) alive += keep[ci];
      if (alive == 0 || done > max_iter + chunk) break;
      if (verbose())
        std::fprintf(stderr, "[femh] pcg: %.3f s, %d iterations, %d of %d cells iterating\n",
                     std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count(), done,
                     alive, nc);
      if (nc > 1 && 2 * alive <= listed) {   // at least half of the listed cells finished: compact
        if (full.empty()) {
          full.resize(H->levels.size());
          for (size_t l = 0; l < H->levels.size(); ++l) {
            Level& L = H->levels[l];
            full[l] = FullLists{L.all.su, L.smooth.su, L.su64, L.all.nu, L.smooth.nu};
          }
        }
        for (size_t l = 0; l < H->levels.size(); ++l) set_units(H, H->levels[l], full[l], &keep);
        listed = alive;
        if (exec) {
          CK(cudaGraphExecDestroy(exec));
          exec = nullptr;
        }
        capture();
      }
    }
  } catch (...) {
    if (exec) cudaGraphExecDestroy(exec);
    restore();
    throw;
  }
  if (exec) CK(cudaGraphExecDestroy(exec));
  restore();
  for (int t = 0; t < nc * kNumRhs; ++t) iters_out[t] += H->state[t].iters;
  if (blk) {   // cells whose block step matrices turned indefinite: one load case at a time
    bool again = false;
    for (auto& S : H->state) {
      if (S.status != CG_BLOCK_FAIL) continue;
      const double sc = S.scale;
      S = CGState{};
      S.active = 1;
      S.scale = sc;
      again = true;
    }
    if (again) pcg<PR>(H, (const TB*)H->b64, kcg, max_iter, tol, iters_out, false, false);
  }
}

// FP64 true residual r64 = b64 - K x64 and its norm per (cell, rhs) -> host.
void true_residual(femh_handle* H, std::vector<double>& rn2) {
  Level& L0 = H->levels[0];
  cudaStream_t s = H->stream;
  double* r = H->r64 ? H->r64 : (double*)H->cg_r;
  stencil<double, OUT_RESID>(H, L0, false, (const double*)H->x64, r, (const double*)H->b64,
                             (const double*)H->kc64, nullptr, nullptr, 0.0);
  {
    Prof prof_(H, "k_norm2", 0.0);
    k_norm2<double><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, r, H->d_part_z, L0.ntot);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_sum_slots", 0.0);
    k_sum_slots<<<fin_blocks(H->ncells), 128, 0, s>>>(L0.d_nu_sb, L0.d_nu_se, H->d_part_z, H->d_nrm, H->ncells);
    LAUNCH_CHECK(H);
  }
  rn2.assign(H->ncells * kNumRhs, 0.0);
  CK(cudaMemcpyAsync(rn2.data(), H->d_nrm, sizeof(double) * rn2.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

void norms_of(femh_handle* H, const double* v, std::vector<double>& n2) {
  Level& L0 = H->levels[0];
  cudaStream_t s = H->stream;
  {
    Prof prof_(H, "k_norm2", 0.0);
    k_norm2<double><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, v, H->d_part_z, L0.ntot);
    LAUNCH_CHECK(H);
  }
  {
    Prof prof_(H, "k_sum_slots", 0.0);
    k_sum_slots<<<fin_blocks(H->ncells), 128, 0, s>>>(L0.d_nu_sb, L0.d_nu_se, H->d_part_z, H->d_nrm, H->ncells);
    LAUNCH_CHECK(H);
  }
  n2.assign(H->ncells * kNumRhs, 0.0);
  CK(cudaMemcpyAsync(n2.data(), H->d_nrm, sizeof(double) * n2.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

// k_coef flags a NaN, infinite or negative density (d_err[1]): an argument
// error, reported before any solve uses the clamped stand-in value.
void check_density(femh_handle* H) {
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, H->d_err + 1, sizeof(int), cudaMemcpyDeviceToHost, H->stream));
  CK(cudaStreamSynchronize(H->stream));
  if (bad) {
    CK(cudaMemsetAsync(H->d_err + 1, 0, sizeof(int), H->stream));
    H->have_x = false;
    H->solved = false;
    throw FemhError{FEMH_E_ARG, "density is NaN, infinite or negative in at least one voxel"};
  }
}

// Solve all six load cases of all cells; fills per-cell infos (status etc.).
void solve_all(femh_handle* H, std::vector<femh_solve_info>& infos) {
  const femh_config& c = H->cfg;
  const int nc = H->ncells;
  cudaStream_t s = H->stream;
  Level& L0 = H->levels[0];
  infos.assign(nc, femh_solve_info{});
  std::vector<int> iters(nc * kNumRhs, 0);
  CK(cudaEventRecord(H->ev0, s));
  if (c.precision == FEMH_FP64) prepare_operator<double>(H);
  else prepare_operator<float>(H);
  const float* kc32 = (const float*)L0.kc;
  std::vector<double> bn2;
  norms_of(H, H->b64, bn2);   // synchronises: the density check below costs no extra wait
  check_density(H);
  std::vector<double> rn2;
  int outer_done = 0;
  std::vector<int> final_status(nc * kNumRhs, CG_CONVERGED);
  // warm start: the previous solution of this handle (same cells) is the
  // starting iterate; its residual b - K x0 replaces b (d_nrm keeps ||b||^2)
  const bool warm = c.warm_start && H->have_x;
  if (c.precision == FEMH_FP64 || c.precision == FEMH_MIXED_PC) {
    for (auto& S : H->state) {
      S = CGState{};
      S.active = 1;
      S.scale = 1.0;
    }
    const double* b0 = H->b64;
    if (warm) {
      double* r0 = (double*)H->cg_q;   // free until the first CG apply
      stencil<double, OUT_RESID>(H, L0, false, (const double*)H->x64, r0, (const double*)H->b64,
                                 (const double*)H->kc64, nullptr, nullptr, 0.0);
      b0 = r0;
    }
    if (c.precision == FEMH_FP64)
      pcg<Prec<double, double, double, double, double>>(H, b0, H->kc64, c.max_iter, c.tol, iters.data(), warm);
    else if (block_pcg(c))   // block PCG: FP64 search directions
      pcg<Prec<double, double, double, float, float>>(H, b0, H->kc64, c.max_iter, c.tol, iters.data(), warm);
    else if (c.store_bf16)   // FP64 CG and operator, FP32 multigrid, bf16 search directions
      pcg<Prec<double, __nv_bfloat16, double, float, float>>(H, b0, H->kc64, c.max_iter, c.tol, iters.data(), warm);
    else   // FP64 CG and operator, FP32 multigrid preconditioner and search directions
      pcg<Prec<double, float, double, float, float>>(H, b0, H->kc64, c.max_iter, c.tol, iters.data(), warm);
    for (int t = 0; t < nc * kNumRhs; ++t) final_status[t] = H->state[t].status;
    outer_done = 1;
    true_residual(H, rn2);
  } else {
    if (warm) {   // defect correction continues from the previous solution
      true_residual(H, rn2);
    } else {
      CK(cudaMemsetAsync(H->x64, 0, sizeof(double) * 18 * H->nvox, s));
      CK(cudaMemcpyAsync(H->r64, H->b64, sizeof(double) * 18 * H->nvox, cudaMemcpyDeviceToDevice, s));
      rn2 = bn2;
    }
    std::vector<int> outer_on(nc * kNumRhs, 1);
    for (int t = 0; t < nc * kNumRhs; ++t)
      if (!(bn2[t] > 0.0) || (warm && std::sqrt(rn2[t] / bn2[t]) < c.tol)) outer_on[t] = 0;
    for (int o = 0; o < c.max_outer; ++o) {
      bool any = false;
      for (int t = 0; t < nc * kNumRhs; ++t) {
        CGState S{};
        S.active = outer_on[t];
        S.outer = outer_on[t];
        S.scale = outer_on[t] ? 1.0 / std::sqrt(rn2[t]) : 1.0;
        H->state[t] = S;
        any |= outer_on[t] != 0;
      }
      if (!any) break;
      outer_done++;
      H->persist_ok = false;
      struct Restore {
        femh_handle* h;
        ~Restore() { h->persist_ok = true; }
      } restore_{H};
      if (c.store_bf16)
        pcg<Prec<float, __nv_bfloat16, float, float, float>>(H, H->r64, kc32, c.max_iter, c.inner_tol, iters.data());
      else
        pcg<Prec<float, float, float, float, float>>(H, H->r64, kc32, c.max_iter, c.inner_tol, iters.data());
      for (int t = 0; t < nc * kNumRhs; ++t)
        if (H->state[t].status == CG_BREAKDOWN && H->state[t].iters == 0) outer_on[t] = 0;
      {
        Prof prof_(H, "k_dc_accum", 0.0);
        k_dc_accum<float><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, H->x64, (const float*)H->cg_x,
                                                          H->d_state, L0.ntot);
        LAUNCH_CHECK(H);
      }
      true_residual(H, rn2);
      for (int t = 0; t < nc * kNumRhs; ++t) {
        const double rel = bn2[t] > 0 ? std::sqrt(rn2[t] / bn2[t]) : 0.0;
        if (rel < c.tol) outer_on[t] = 0;
      }
      if (verbose()) {
        std::fprintf(stderr, "[femh] outer %d:", outer_done);
        for (int t = 0; t < std::min(nc * kNumRhs, 6); ++t)
          std::fprintf(stderr, " (%d it, inner %.1e, true %.2e)", H->state[t].iters, H->state[t].rel,
                       bn2[t] > 0 ? std::sqrt(rn2[t] / bn2[t]) : 0.0);
        std::fprintf(stderr, "\n");
      }
    }
    for (int t = 0; t < nc * kNumRhs; ++t) {
      const double rel = bn2[t] > 0 ? std::sqrt(rn2[t] / bn2[t]) : 0.0;
      final_status[t] = rel < c.tol ? CG_CONVERGED : CG_MAXITER;
    }
  }
  CK(cudaEventRecord(H->ev1, s));
  CK(cudaEventSynchronize(H->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
  for (int ci = 0; ci < nc; ++ci) {
    femh_solve_info& I = infos[ci];
    I.status = FEMH_OK;
    I.outer_iterations = outer_done;
    I.solve_ms = ms;
    for (int r = 0; r < kNumRhs; ++r) {
      const int t = ci * kNumRhs + r;
      I.iterations[r] = iters[t];
      I.rel_residual[r] = bn2[t] > 0 ? std::sqrt(rn2[t] / bn2[t]) : 0.0;
      if (final_status[t] == CG_BREAKDOWN && I.status == FEMH_OK) I.status = FEMH_E_BREAKDOWN;
      if (I.rel_residual[r] >= c.tol && I.status == FEMH_OK) I.status = FEMH_E_NOT_CONVERGED;
    }
  }
}

// Energy pairs of the resident fields: C^H with the element matrix's Hadamard
// factors k = H->hk; other factors give other bilinear forms on the same fields.
void energy_C(femh_handle* H, std::vector<double>& C, std::vector<double>& dens, const HadK* k = nullptr) {
  Level& L0 = H->levels[0];
  cudaStream_t s = H->stream;
  EnergyArgs a{};
  a.cells = L0.d_cells;
  a.units = L0.all.d_nu;
  a.chi = H->x64;
  a.kc64 = H->kc64;
  a.rho = H->rho_used;
  a.ec = H->d_ec;
  a.part = H->d_part_e;
  a.ntot = L0.ntot;
  a.k = k ? *k : H->hk;
  a.law = make_law(H->cfg);
  {
    Prof prof_(H, "k_energy", 0.0);
    k_energy<EN_C><<<(unsigned)L0.all.nu.size(), 128, 0, s>>>(a);
    LAUNCH_CHECK(H);
  }
  double* d_dens = H->d_nrm;
  {
    Prof prof_(H, "k_energy_fin", 0.0);
    k_energy_fin<<<cdiv((long long)H->ncells * 22, 128), 128, 0, s>>>(L0.d_cells, L0.d_nu_sb, L0.d_nu_se,
                                                                   H->d_part_e, H->d_C, d_dens, H->ncells);
    LAUNCH_CHECK(H);
  }
  C.assign(H->ncells * 36, 0.0);
  dens.assign(H->ncells, 0.0);
  CK(cudaMemcpyAsync(C.data(), H->d_C, sizeof(double) * C.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(dens.data(), d_dens, sizeof(double) * dens.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

// Common path of single-cell and batched calls.  rho_ptrs[i] host or device.
// A kernel whose bounded wait ran out leaves its work undone and sets the
// handle's error flag: report it (and clear it) at the end of a solve.
void check_kernel_error(femh_handle* H) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, H->d_err, sizeof(int), cudaMemcpyDeviceToHost, H->stream));
  CK(cudaStreamSynchronize(H->stream));
  if (e) {
    CK(cudaMemsetAsync(H->d_err, 0, sizeof(int), H->stream));
    throw FemhError{FEMH_E_CUDA, "a stencil kernel's copy pipeline timed out"};
  }
}

void run_cells(femh_handle* H, const std::vector<int>& shapes, const std::vector<double>& hs,
               const std::vector<const double*>& rho, bool rho_dev, std::vector<double>& C,
               std::vector<femh_solve_info>& infos) {
  build_setup(H, shapes, hs);
  cudaStream_t s = H->stream;
  for (int i = 0; i < H->ncells; ++i) {
    if (!rho[i]) throw FemhError{FEMH_E_ARG, "null rho"};
    CK(cudaMemcpyAsync(H->rho_in + H->cell_off[i], rho[i], sizeof(double) * H->cell_vox[i],
                       rho_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  }
  solve_all(H, infos);
  check_kernel_error(H);
  H->have_x = true;
  std::vector<double> dens;
  energy_C(H, C, dens);
  for (int i = 0; i < H->ncells; ++i) infos[i].density = dens[i];
  H->solved = true;
  H->C_last = C;
}


}  // namespace

// ================================================================ C ABI ===
namespace {
template <typename F>
femh_status guard(femh_handle* H, F&& f) {
  try {
    f();
    return FEMH_OK;
  } catch (const FemhError& e) {
    set_err(H, e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_err(H, "host allocation failed");
    return FEMH_E_OOM;
  } catch (const std::exception& e) {
    set_err(H, e.what());
    return FEMH_E_CUDA;
  }
}

void to_host_or_dev(femh_handle* H, double* dst, const double* src, size_t n, int on_device) {
  CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     H->stream));
  CK(cudaStreamSynchronize(H->stream));
}

void check_config(const femh_config& c) {
  if (c.interp < 0 || c.interp > 2) throw FemhError{FEMH_E_ARG, "interp must be SIMP, RAMP3 or BINARY"};
  if (!(c.nu > -1.0 && c.nu < 0.5)) throw FemhError{FEMH_E_ARG, "nu must lie in (-1, 0.5)"};
  if (c.precision != FEMH_FP64 && c.precision != FEMH_MIXED && c.precision != FEMH_MIXED_PC)
    throw FemhError{FEMH_E_ARG, "bad precision"};
  if (c.solver != FEMH_JACOBI_PCG && c.solver != FEMH_GMG_PCG) throw FemhError{FEMH_E_ARG, "bad solver"};
  if (c.solver == FEMH_GMG_PCG && (c.pre_smooth < 1 || c.post_smooth < 0))
    throw FemhError{FEMH_E_ARG, "pre_smooth >= 1 and post_smooth >= 0 are required"};
  if (!(c.tol > 0.0) || c.max_iter < 1) throw FemhError{FEMH_E_ARG, "tol > 0 and max_iter >= 1 are required"};
  if (c.precision == FEMH_MIXED && (!(c.inner_tol > 0.0) || c.max_outer < 1))
    throw FemhError{FEMH_E_ARG, "inner_tol > 0 and max_outer >= 1 are required"};
  if (c.stencil_variant < 0 || c.stencil_variant > 7) throw FemhError{FEMH_E_ARG, "stencil_variant must be 0..7"};
  if (!(c.cheb_ratio == 0.0 || c.cheb_ratio > 1.0)) throw FemhError{FEMH_E_ARG, "cheb_ratio must be 0 or > 1"};
  if (c.block_jacobi != 0 && c.block_jacobi != 1) throw FemhError{FEMH_E_ARG, "block_jacobi must be 0 or 1"};
  if (c.block_cg != 0 && c.block_cg != 1) throw FemhError{FEMH_E_ARG, "block_cg must be 0 or 1"};
  if (c.coarse_avg < 0 || c.coarse_avg > 2) throw FemhError{FEMH_E_ARG, "coarse_avg must be 0, 1 or 2"};
  if (!(c.E_s > 0.0) || c.E_min < 0.0 || !(c.rho_max >= c.rho_min))
    throw FemhError{FEMH_E_ARG, "bad material law parameters"};
}
}  // namespace

extern "C" {

femh_status femh_config_default(femh_config* c) {
  if (!c) return FEMH_E_ARG;
  std::memset(c, 0, sizeof(*c));
  c->device = 0;
  c->interp = FEMH_INTERP_SIMP;
  c->E_s = 1.0;
  c->E_min = 1e-6;
  c->penal = 3.0;
  c->nu = 0.3;
  c->bin_hi = 1.0;
  c->bin_lo = 1e-4;
  c->rho_min = 0.0;
  c->rho_max = 1.0;
  c->precision = FEMH_FP64;
  c->solver = FEMH_GMG_PCG;
  c->pre_smooth = 3;
  c->post_smooth = 3;
  c->omega = 0.35;   // < 2 / 5.32: damped Jacobi stable for any coefficient field (nu = 0.3)
  c->coarse_max_nodes = 64;
  c->tol = 1e-10;
  c->max_iter = 20000;
  c->inner_tol = 1e-5;
  c->max_outer = 8;
  c->store_bf16 = 0;
  c->graph_chunk = 8;
  c->coarse_avg = 0;
  c->autotune = 1;
  c->stencil_variant = 0;
  c->warm_start = 0;
  c->cheb_ratio = 64.0;   // 128^3 smooth cell, mixed: 146 iterations (2+2, omega) -> 86
  c->block_jacobi = 1;   // 128^3 smooth cell, mixed: 87 iterations -> 75, 219 -> 204 ms
  c->block_cg = 1;
  return FEMH_OK;
}

femh_status femh_create(femh_handle** out, const femh_config* cfg) {
  if (!out || !cfg) return FEMH_E_ARG;
  *out = nullptr;
  femh_handle* H = new (std::nothrow) femh_handle();
  if (!H) return FEMH_E_OOM;
  const femh_status st = guard(H, [&] {
    check_config(*cfg);
    H->cfg = *cfg;
    H->device = cfg->device;
    CK(cudaSetDevice(cfg->device));
    CK(cudaDeviceGetAttribute(&H->nsm, cudaDevAttrMultiProcessorCount, cfg->device));
    CK(cudaStreamCreateWithFlags(&H->own_stream, cudaStreamNonBlocking));
    H->stream = H->own_stream;
    CK(cudaEventCreate(&H->ev0));
    CK(cudaEventCreate(&H->ev1));
    host_k0(cfg->nu, H->K0);
    H->hk = host_hadk(H->K0);
    {
      double Kf[576];
      host_k0_force(cfg->nu, Kf);
      H->hk_force = host_hadk(Kf);
    }
    H->ec = host_elemconst(H->K0);
    {
      const double lmax = host_jacobi_bound(H->K0, cfg->block_jacobi != 0);
      H->w_pre = smooth_weights(std::max(cfg->pre_smooth, 1), lmax, cfg->cheb_ratio, cfg->omega);
      H->w_post = smooth_weights(std::max(cfg->post_smooth, 1), lmax, cfg->cheb_ratio, cfg->omega);
      std::reverse(H->w_post.begin(), H->w_post.end());   // the pre-smoother's factors in reverse
    }
    H->d_ec = H->perm.arr<ElemConst>(1);
    H->d_K0 = H->perm.arr<double>(576);
    CK(cudaMemcpy(H->d_ec, &H->ec, sizeof(ElemConst), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(H->d_K0, H->K0, sizeof(double) * 576, cudaMemcpyHostToDevice));
    H->d_err = H->perm.arr<int>(2);
    CK(cudaMemset(H->d_err, 0, 2 * sizeof(int)));
    H->d_loop = H->perm.arr<int>(1);
    // FEMH_STAGE_WAIT_LIMIT=0 (tests only): every stage wait of the bulk-copy
    // staged kernels gives up at once, although its copies complete -- the
    // kernel then drains them with the full limit, flags the handle and
    // returns, and the call reports FEMH_E_CUDA
    if (const char* w = std::getenv("FEMH_STAGE_WAIT_LIMIT")) {
      if (std::strtol(w, nullptr, 10) == 0) H->wait_limit = 0;
    }
    // FEMH_ARENA_LIMIT_BYTES (tests only): the handle's set-up allocations fail
    // with FEMH_E_OOM beyond this many bytes, as on a device without room
    if (const char* w = std::getenv("FEMH_ARENA_LIMIT_BYTES")) {
      const long long v = std::strtoll(w, nullptr, 10);
      if (v > 0) H->setup.limit = (size_t)v;
    }
  });
  if (st != FEMH_OK) {
    femh_destroy(H);
    return st;
  }
  *out = H;
  return FEMH_OK;
}

femh_status femh_destroy(femh_handle* H) {
  if (!H) return FEMH_E_ARG;
  cudaSetDevice(H->device);
  if (H->stream) cudaStreamSynchronize(H->stream);
  H->setup.release();
  release_stage(H);
  H->perm.release();
  if (H->ev0) cudaEventDestroy(H->ev0);
  if (H->ev1) cudaEventDestroy(H->ev1);
  if (H->own_stream) cudaStreamDestroy(H->own_stream);
  delete H;
  return FEMH_OK;
}

femh_status femh_homogenize(femh_handle* H, int nx, int ny, int nz, double hvox, const double* rho,
                            int rho_on_device, double C_out[36], femh_solve_info* info) {
  if (!H) return FEMH_E_ARG;
  femh_status code = FEMH_OK;
  const femh_status st = guard(H, [&] {
    if (!rho || !C_out) throw FemhError{FEMH_E_ARG, "rho and C_out must not be NULL"};
    CK(cudaSetDevice(H->device));
    std::vector<double> C;
    std::vector<femh_solve_info> infos;
    run_cells(H, {nx, ny, nz}, {hvox}, {rho}, rho_on_device != 0, C, infos);
    std::memcpy(C_out, C.data(), sizeof(double) * 36);
    if (info) *info = infos[0];
    code = infos[0].status;
    if (code != FEMH_OK) set_err(H, code == FEMH_E_BREAKDOWN ? "CG breakdown" : "not converged to tol");
  });
  return st != FEMH_OK ? st : code;
}

femh_status femh_homogenize_batch(femh_handle* H, int ncell, const femh_cell* cells, double* C_out,
                                  const double* dLdC, double* dLdrho, femh_solve_info* infos_out) {
  if (!H) return FEMH_E_ARG;
  femh_status code = FEMH_OK;
  const femh_status st = guard(H, [&] {
    if (ncell < 1 || !cells || !C_out) throw FemhError{FEMH_E_ARG, "ncell >= 1, cells and C_out are required"};
    if ((dLdC == nullptr) != (dLdrho == nullptr)) throw FemhError{FEMH_E_ARG, "dLdC and dLdrho go together"};
    CK(cudaSetDevice(H->device));
    std::vector<int> shapes;
    std::vector<double> hs;
    std::vector<const double*> rho;
    for (int i = 0; i < ncell; ++i) {
      shapes.insert(shapes.end(), {cells[i].nx, cells[i].ny, cells[i].nz});
      hs.push_back(cells[i].h);
      rho.push_back(cells[i].rho);
    }
    std::vector<double> C;
    std::vector<femh_solve_info> infos;
    run_cells(H, shapes, hs, rho, false, C, infos);
    std::memcpy(C_out, C.data(), sizeof(double) * 36 * ncell);
    if (infos_out) std::memcpy(infos_out, infos.data(), sizeof(femh_solve_info) * ncell);
    for (auto& I : infos)
      if (I.status != FEMH_OK) code = I.status;
    if (dLdC) {
      Level& L0 = H->levels[0];
      std::vector<double> W(21 * ncell);
      for (int ci = 0; ci < ncell; ++ci) {
        int t = 0;
        for (int I = 0; I < 6; ++I)
          for (int J = 0; J <= I; ++J)
            W[ci * 21 + t++] = (I == J) ? dLdC[ci * 36 + I * 6 + I] : dLdC[ci * 36 + I * 6 + J] + dLdC[ci * 36 + J * 6 + I];
      }
      CK(cudaMemcpyAsync(H->d_W, W.data(), sizeof(double) * W.size(), cudaMemcpyHostToDevice, H->stream));
      EnergyArgs a{};
      a.cells = L0.d_cells;
      a.units = L0.all.d_nu;
      a.chi = H->x64;
      a.kc64 = H->kc64;
      a.rho = H->rho_used;
      a.ec = H->d_ec;
      a.W = H->d_W;
      a.out = grad_target(H, dLdrho, 0);
      a.ntot = L0.ntot;
      a.k = H->hk;
      a.law = make_law(H->cfg);
      {
        Prof prof_(H, "k_energy", 0.0);
        k_energy<EN_GRAD><<<(unsigned)L0.all.nu.size(), 128, 0, H->stream>>>(a);
        LAUNCH_CHECK(H);
      }
      to_host_or_dev(H, dLdrho, a.out, H->nvox, 0);
    }
  });
  return st != FEMH_OK ? st : code;
}

femh_status femh_homogenize_grad(femh_handle* H, const double dLdC[36], double* dLdrho, int out_on_device) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!H->solved || H->ncells != 1) throw FemhError{FEMH_E_STATE, "call femh_homogenize first"};
    if (!dLdC || !dLdrho) throw FemhError{FEMH_E_ARG, "dLdC and dLdrho must not be NULL"};
    CK(cudaSetDevice(H->device));
    Level& L0 = H->levels[0];
    double W[21];
    int t = 0;
    for (int I = 0; I < 6; ++I)
      for (int J = 0; J <= I; ++J) W[t++] = (I == J) ? dLdC[I * 6 + I] : dLdC[I * 6 + J] + dLdC[J * 6 + I];
    CK(cudaMemcpyAsync(H->d_W, W, sizeof W, cudaMemcpyHostToDevice, H->stream));
    EnergyArgs a{};
    a.cells = L0.d_cells;
    a.units = L0.all.d_nu;
    a.chi = H->x64;
    a.kc64 = H->kc64;
    a.rho = H->rho_used;
    a.ec = H->d_ec;
    a.W = H->d_W;
    a.out = grad_target(H, dLdrho, out_on_device);
    a.ntot = L0.ntot;
    a.k = H->hk;
    a.law = make_law(H->cfg);
    {
      Prof prof_(H, "k_energy", 0.0);
      k_energy<EN_GRAD><<<(unsigned)L0.all.nu.size(), 128, 0, H->stream>>>(a);
      LAUNCH_CHECK(H);
    }
    if (!out_on_device) to_host_or_dev(H, dLdrho, a.out, H->nvox, 0);
  });
}

femh_status femh_field_gradient(femh_handle* H, const double dLdC[36], double dLdrho_add, int nparam,
                                const int* voxel_param, double* grad_out) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!H->solved || H->ncells != 1) throw FemhError{FEMH_E_STATE, "call femh_homogenize first"};
    if (!dLdC || !voxel_param || !grad_out || nparam < 1)
      throw FemhError{FEMH_E_ARG, "dLdC, voxel_param, grad_out and nparam >= 1 are required"};
    CK(cudaSetDevice(H->device));
    const long long nv = H->nvox;
    // voxels of each parameter, in voxel order (FNV-1a hash of the map decides reuse)
    unsigned long long key = 1469598103934665603ULL ^ (unsigned long long)nparam;
    for (long long e = 0; e < nv; ++e) {
      const int p = voxel_param[e];
      if (p < -1 || p >= nparam) throw FemhError{FEMH_E_ARG, "voxel_param entries must lie in [-1, nparam)"};
      key = (key ^ (unsigned long long)(unsigned)p) * 1099511628211ULL;
    }
    if (key != H->fmap_key || nparam != H->fmap_nparam) {
      std::vector<int> ptr(nparam + 1, 0);
      for (long long e = 0; e < nv; ++e)
        if (voxel_param[e] >= 0) ptr[voxel_param[e] + 1]++;
      for (int p = 0; p < nparam; ++p) ptr[p + 1] += ptr[p];
      std::vector<int> vox(std::max(ptr[nparam], 1));
      std::vector<int> fill(ptr.begin(), ptr.end() - 1);
      for (long long e = 0; e < nv; ++e)
        if (voxel_param[e] >= 0) vox[fill[voxel_param[e]]++] = (int)e;
      const size_t need = (size_t)nparam + 1 + vox.size();
      if (H->fmap_n < need) {
        if (H->d_fmap) cudaFree(H->d_fmap);
        H->d_fmap = nullptr;
        H->fmap_n = 0;
        CK(cudaMalloc(&H->d_fmap, need * sizeof(int)));
        H->fmap_n = need;
      }
      CK(cudaMemcpyAsync(H->d_fmap, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, H->stream));
      CK(cudaMemcpyAsync(H->d_fmap + nparam + 1, vox.data(), vox.size() * sizeof(int), cudaMemcpyHostToDevice,
                         H->stream));
      CK(cudaStreamSynchronize(H->stream));   // host vectors go out of scope
      H->fmap_key = key;
      H->fmap_nparam = nparam;
    }
    Level& L0 = H->levels[0];
    double W[21];
    int t = 0;
    for (int I = 0; I < 6; ++I)
      for (int J = 0; J <= I; ++J) W[t++] = (I == J) ? dLdC[I * 6 + I] : dLdC[I * 6 + J] + dLdC[J * 6 + I];
    CK(cudaMemcpyAsync(H->d_W, W, sizeof W, cudaMemcpyHostToDevice, H->stream));
    EnergyArgs a{};
    a.cells = L0.d_cells;
    a.units = L0.all.d_nu;
    a.chi = H->x64;
    a.kc64 = H->kc64;
    a.rho = H->rho_used;
    a.ec = H->d_ec;
    a.W = H->d_W;
    // the voxel gradient and then the parameter sums, in the dead CG buffer q
    // when they fit (18 x nvox FP64 or FP32 values), else in the staging buffer
    const size_t qd = (size_t)18 * nv * (H->cfg.precision == FEMH_MIXED ? 4 : 8) / sizeof(double);
    a.out = ((size_t)nv + nparam <= qd) ? grad_target(H, nullptr, 0) : stage(H, (size_t)nv + nparam);
    a.ntot = L0.ntot;
    a.k = H->hk;
    a.law = make_law(H->cfg);
    {
      Prof prof_(H, "k_energy", 0.0);
      k_energy<EN_GRAD><<<(unsigned)L0.all.nu.size(), 128, 0, H->stream>>>(a);
      LAUNCH_CHECK(H);
    }
    double* pg = a.out + nv;
    {
      Prof prof_(H, "k_param_sum", 0.0);
      k_param_sum<<<cdiv((long long)nparam * 32, 256), 256, 0, H->stream>>>(H->d_fmap, H->d_fmap + nparam + 1,
                                                                           a.out, dLdrho_add, pg, nparam);
      LAUNCH_CHECK(H);
    }
    to_host_or_dev(H, grad_out, pg, nparam, 0);
  });
}

femh_status femh_force_tensors(femh_handle* H, double* C_out) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!H->solved) throw FemhError{FEMH_E_STATE, "call femh_homogenize or femh_homogenize_batch first"};
    if (!C_out) throw FemhError{FEMH_E_ARG, "C_out must not be NULL"};
    // femlib's shear loads put f/2 on faces of different areas when the cell
    // is not cubic: out of moment balance, the rotation multipliers then load
    // the cell in the interior and its fields leave the periodic + affine space
    for (const CellDesc& cd : H->levels[0].cells)
      if (cd.nx != cd.ny || cd.ny != cd.nz)
        throw FemhError{FEMH_E_ARG, "the force-driven tensor needs cubic cells (nx = ny = nz)"};
    CK(cudaSetDevice(H->device));
    std::vector<double> W, dens;
    energy_C(H, W, dens, &H->hk_force);
    // unit tensor-shear coarse strains instead of unit engineering ones: the
    // shear rows and columns scale by 2 (coarseGv = S, inverted, :1000-1060)
    const double sc[6] = {1, 1, 1, 2, 2, 2};
    for (int c = 0; c < H->ncells; ++c)
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) C_out[36 * c + 6 * i + j] = sc[i] * sc[j] * W[36 * c + 6 * i + j];
  });
}

femh_status femh_dCdrho(femh_handle* H, double* out, int out_on_device) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!H->solved || H->ncells != 1) throw FemhError{FEMH_E_STATE, "call femh_homogenize first"};
    if (!out) throw FemhError{FEMH_E_ARG, "out must not be NULL"};
    CK(cudaSetDevice(H->device));
    Level& L0 = H->levels[0];
    EnergyArgs a{};
    a.cells = L0.d_cells;
    a.units = L0.all.d_nu;
    a.chi = H->x64;
    a.kc64 = H->kc64;
    a.rho = H->rho_used;
    a.ec = H->d_ec;
    a.out = out_on_device ? out : stage(H, 21 * (size_t)H->nvox);
    a.ntot = L0.ntot;
    a.k = H->hk;
    a.law = make_law(H->cfg);
    {
      Prof prof_(H, "k_energy", 0.0);
      k_energy<EN_DCDRHO><<<(unsigned)L0.all.nu.size(), 128, 0, H->stream>>>(a);
      LAUNCH_CHECK(H);
    }
    if (!out_on_device) to_host_or_dev(H, out, a.out, 21 * H->nvox, 0);
  });
}

femh_status femh_full_field(femh_handle* H, int I, double* u_out, int out_on_device) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!H->solved || H->ncells != 1) throw FemhError{FEMH_E_STATE, "call femh_homogenize first"};
    if (I < 0 || I > 5 || !u_out) throw FemhError{FEMH_E_ARG, "load case must be 0..5 and u_out non-NULL"};
    CK(cudaSetDevice(H->device));
    const CellDesc& cd = H->levels[0].cells[0];
    const long long n = 3LL * (cd.nx + 1) * (cd.ny + 1) * (cd.nz + 1);
    double* tmp = stage(H, (size_t)n);
    {
      Prof prof_(H, "k_full_field", 0.0);
      k_full_field<<<cdiv(n / 3, 256), 256, 0, H->stream>>>(H->levels[0].d_cells, 0, H->x64, I, tmp,
                                                          H->levels[0].ntot);
      LAUNCH_CHECK(H);
    }
    to_host_or_dev(H, u_out, tmp, n, out_on_device);
  });
}

femh_status femh_fluctuation(femh_handle* H, double* chi_out, int out_on_device) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!H->solved || H->ncells != 1) throw FemhError{FEMH_E_STATE, "call femh_homogenize first"};
    if (!chi_out) throw FemhError{FEMH_E_ARG, "chi_out must not be NULL"};
    CK(cudaSetDevice(H->device));
    const long long nn = H->nvox;
    double* tmp = stage(H, 18 * (size_t)nn);
    {
      Prof prof_(H, "k_layout", 0.0);
      k_layout<true><<<cdiv(18 * nn, 256), 256, 0, H->stream>>>(H->x64, tmp, 0, nn, H->levels[0].ntot);
      LAUNCH_CHECK(H);
    }
    to_host_or_dev(H, chi_out, tmp, 18 * nn, out_on_device);
  });
}

femh_status femh_apply_operator(femh_handle* H, int nx, int ny, int nz, double hvox, const double* rho,
                                const double* u, double* y, int on_device) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (!rho || !u || !y) throw FemhError{FEMH_E_ARG, "rho, u and y must not be NULL"};
    CK(cudaSetDevice(H->device));
    build_setup(H, {nx, ny, nz}, {hvox});
    cudaStream_t s = H->stream;
    const long long nn = H->nvox;
    const cudaMemcpyKind k_in = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(H->rho_in, rho, sizeof(double) * nn, k_in, s));
    Level& L0 = H->levels[0];
    const MatLaw law = make_law(H->cfg);
    // FP32 operator (the arithmetic of the mixed modes' multigrid sweeps) when
    // the handle is configured for a mixed precision with FP32 storage
    const bool f32 = H->cfg.precision != FEMH_FP64 && !H->cfg.store_bf16;
    {
      Prof prof_(H, "k_coef", 0.0);
      if (f32)
        k_coef<float><<<(unsigned)L0.all.nu.size(), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, H->rho_in, law, H->kc64,
                                                               (float*)L0.kc, H->rho_used, H->d_err + 1);
      else
        k_coef<double><<<(unsigned)L0.all.nu.size(), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, H->rho_in, law,
                                                                H->kc64, (double*)nullptr, H->rho_used,
                                                                H->d_err + 1);
      LAUNCH_CHECK(H);
    }
    check_density(H);
    double* tmp = stage(H, 18 * (size_t)nn);
    H->have_x = false;   // x64 serves as the input buffer below
    CK(cudaMemcpyAsync(tmp, u, sizeof(double) * 18 * nn, k_in, s));
    {
      Prof prof_(H, "k_layout", 0.0);
      k_layout<false><<<cdiv(18 * nn, 256), 256, 0, s>>>(tmp, H->x64, 0, nn, L0.ntot);
      LAUNCH_CHECK(H);
    }
    if (f32) {
      float* uf = (float*)H->cg_r;
      float* yf = (float*)H->cg_q;
      k_copy<float, double><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, uf, H->x64, nullptr,
                                                              L0.ntot);
      LAUNCH_CHECK(H);
      stencil<float, OUT_APPLY>(H, L0, false, (const float*)uf, yf, (const float*)nullptr, (const float*)L0.kc,
                                nullptr, nullptr, 0.0);
      check_kernel_error(H);
      k_copy<double, float><<<NODE_GRID(L0.all), 256, 0, s>>>(L0.d_cells, L0.all.d_nu, H->b64, yf, nullptr,
                                                              L0.ntot);
      LAUNCH_CHECK(H);
    } else {
      stencil<double, OUT_APPLY>(H, L0, false, (const double*)H->x64, H->b64, (const double*)nullptr,
                                 (const double*)H->kc64, nullptr, nullptr, 0.0);
    }
    {
      Prof prof_(H, "k_layout", 0.0);
      k_layout<true><<<cdiv(18 * nn, 256), 256, 0, s>>>(H->b64, tmp, 0, nn, L0.ntot);
      LAUNCH_CHECK(H);
    }
    to_host_or_dev(H, y, tmp, 18 * nn, on_device);
    H->solved = false;
  });
}

femh_status femh_batch_memory(femh_handle* H, int ncell, const femh_cell* cells, double* need_bytes,
                              double* avail_bytes) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    if (ncell < 0 || (ncell > 0 && !cells)) throw FemhError{FEMH_E_ARG, "ncell >= 0 and cells are required"};
    double need = 0.0;
    for (int i = 0; i < ncell; ++i) need += cell_setup_bytes(H->cfg, cells[i].nx, cells[i].ny, cells[i].nz);
    if (need_bytes) *need_bytes = need;
    if (avail_bytes) {
      CK(cudaSetDevice(H->device));
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      *avail_bytes = (double)fr + (double)H->setup.held + (double)H->stage_n * sizeof(double);
    }
  });
}

femh_status femh_last_error(const femh_handle* H, char* buf, size_t n) {
  if (!H || !buf || n == 0) return FEMH_E_ARG;
  std::snprintf(buf, n, "%s", H->err.c_str());
  return FEMH_OK;
}

femh_status femh_set_stream(femh_handle* H, void* stream) {
  if (!H) return FEMH_E_ARG;
  H->stream = stream ? (cudaStream_t)stream : H->own_stream;
  return FEMH_OK;
}

long long femh_kernel_launches(const femh_handle* H) { return H ? H->launches : -1; }

femh_status femh_profile(femh_handle* H, int enable) {
  if (!H) return FEMH_E_ARG;
  return guard(H, [&] {
    prof_resolve(H);
    H->prof = enable != 0;
    H->kstats.clear();
  });
}

femh_status femh_profile_read(femh_handle* H, femh_kernel_stat* out, int max, int* n) {
  if (!H || !n || (max > 0 && !out)) return FEMH_E_ARG;
  return guard(H, [&] {
    prof_resolve(H);
    int i = 0;
    for (auto& kv : H->kstats) {
      if (kv.second.launches == 0) continue;
      if (i < max) {
        std::snprintf(out[i].name, sizeof out[i].name, "%s", kv.first.c_str());
        out[i].launches = kv.second.launches;
        out[i].total_ms = kv.second.ms;
        out[i].bytes = kv.second.bytes;
      }
      ++i;
    }
    *n = i;
  });
}

}  // extern "C"

// ============================================= allocation-free energy entry ===
// femh_energy_noalloc: C^H of one cell from a caller-provided density and
// periodic fluctuation, for callers that cannot call cudaMalloc.  Its per-CTA
// partial sums live in the file-scope device array below instead of in
// handle-owned memory.
namespace {

constexpr int kNoAllocSlots = 2048;                          // CTAs of the partial pass
constexpr long long kNoAllocMaxVoxels = 256LL * 256 * 256;   // largest accepted cell
// 2048 slots x 21 doubles = 336 KiB on every device that loads the library.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots * 21];

std::mutex g_noalloc_mu;
double* g_noalloc_addr[256] = {};   // device address of g_noalloc_scratch, per device

// Per voxel u^I = ue0^I(h) + chi^I with chi in the [6][node][3] layout of
// femh_fluctuation; slot sums of kc_e u^I.K0(1) u^J (21 pairs) into part.
__global__ void __launch_bounds__(128)
k_energy_noalloc_partial(int nx, int ny, int nz, double h, const double* __restrict__ rho,
                         const double* __restrict__ chi, MatLaw law, HadK K, ElemConst ec,
                         double* __restrict__ part, long long per) {
  const long long nv = (long long)nx * ny * nz;
  const long long b = (long long)blockIdx.x * per, e_end = min(nv, b + per);
  double acc[21];
#pragma unroll
  for (int t = 0; t < 21; ++t) acc[t] = 0.0;
  for (long long e = b + threadIdx.x; e < e_end; e += blockDim.x) {
    int i, j, k;
    node_ijk(e, ny, nz, i, j, k);
    long long nd[8];
#pragma unroll
    for (int a8 = 0; a8 < 8; ++a8)
      nd[a8] = lin(wrap(i + ((a8 >> 2) & 1), nx), wrap(j + ((a8 >> 1) & 1), ny), wrap(k + (a8 & 1), nz), ny, nz);
    double uh[kNumRhs][3][8];
#pragma unroll
    for (int I = 0; I < kNumRhs; ++I)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int a8 = 0; a8 < 8; ++a8) uh[I][c][a8] = chi[((long long)I * nv + nd[a8]) * 3 + c];
        fwht8_fwd(uh[I][c]);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) uh[I][c][kk] += h * ec.uhat0[I][c][kk];
      }
    double r = fmin(fmax(rho[e], law.rho_min), law.rho_max);
    const double ke = law_coef(law, r) * h;
#pragma unroll
    for (int J = 0; J < kNumRhs; ++J) {
      double w[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) w[c][kk] = uh[J][c][kk];
      had_block(w, K, 1.0);
#pragma unroll
      for (int I = J; I < kNumRhs; ++I) {
        double d = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int kk = 1; kk < 8; ++kk) d += uh[I][c][kk] * w[c][kk];
        acc[I * (I + 1) / 2 + J] += ke * d;
      }
    }
  }
  __shared__ double red[32 * 21];
  block_reduce<21>(acc, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int t = 0; t < 21; ++t) part[(long long)blockIdx.x * 21 + t] = acc[t];
}

// C (6x6, both triangles) from the slot sums, fixed summation order.
__global__ void k_energy_noalloc_final(double vol, const double* __restrict__ part, int nslots,
                                       double* __restrict__ C) {
  const int q = threadIdx.x;
  if (q >= 21) return;
  double s = 0.0;
  for (int sl = 0; sl < nslots; ++sl) s += part[(long long)sl * 21 + q];
  int I = 0;
  while ((I + 1) * (I + 2) / 2 <= q) ++I;
  const int J = q - I * (I + 1) / 2;
  C[I * 6 + J] = s / vol;
  C[J * 6 + I] = s / vol;
}

}  // namespace

extern "C" femh_status femh_energy_noalloc(const femh_config* cfg, int nx, int ny, int nz, double hvox,
                                           const double* rho, const double* chi, double* C_out,
                                           void* stream) {
  if (!cfg || !rho || !chi || !C_out) return FEMH_E_ARG;
  if (nx < 2 || ny < 2 || nz < 2 || !(hvox > 0.0)) return FEMH_E_ARG;
  const long long nv = (long long)nx * ny * nz;
  if (nv > kNoAllocMaxVoxels) return FEMH_E_ARG;   // beyond the scratch array's design limit
  try {
    check_config(*cfg);
  } catch (const FemhError&) {
    return FEMH_E_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return FEMH_E_CUDA;
  if (dev != cfg->device) return FEMH_E_ARG;   // runs on the caller's current device only
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      // set-up, once per device: the host-side symbol is only a stand-in; its
      // device address must be looked up with the device current
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return FEMH_E_CUDA;
      g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_noalloc_addr[dev];
  }
  double K[576];
  host_k0(cfg->nu, K);
  HadK hk;
  try {
    hk = host_hadk(K);
  } catch (const FemhError&) {
    return FEMH_E_ARG;
  }
  const ElemConst ec = host_elemconst(K);
  MatLaw law = make_law(*cfg);
  law.rho_bf16 = 0;
  const long long per = (nv + kNoAllocSlots - 1) / kNoAllocSlots;
  const int nslots = (int)((nv + per - 1) / per);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_energy_noalloc_partial<<<nslots, 128, 0, s>>>(nx, ny, nz, hvox, rho, chi, law, hk, ec, scratch, per);
  if (cudaGetLastError() != cudaSuccess) return FEMH_E_CUDA;
  const double vol = (double)nv * hvox * hvox * hvox;
  k_energy_noalloc_final<<<1, 32, 0, s>>>(vol, scratch, nslots, C_out);
  if (cudaGetLastError() != cudaSuccess) return FEMH_E_CUDA;
  return FEMH_OK;
}
