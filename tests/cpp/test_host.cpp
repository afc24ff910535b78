// test_host.cpp -- exercises the reference-facing C++ layer (femh_host) the way
// the reference exercises FEM3DFun / NumericalCoarseningUsingMultigrid:
//   1. FEM3DFun::setParam / f / df with a PiecewiseConstant3D field and the
//      central-difference check of df (fast_fem/run3d.cpp:291-323 check_df);
//   2. NumericalCoarseningUsingMultigrid init + computeCoarsened... on a
//      replicated/subdivided structure (21 tensor values + 4 parameters), and
//      the batched call against the one-at-a-time call; the same for femlib's
//      force-driven NumericalCoarsening (Cubic and General parameters, a
//      non-cubic cell rejected);
//   3. level*.bin round trip (cfgUtil::writeBinary / readBinary format).
// Prints one JSON object; tests/test_gpu_host.py checks it (also against the
// oracle).  Exit code != 0 on a failed in-program check.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../fem_b200/host/femh_host.hpp"

using namespace femh_host;

static void print_vec(const char* key, const std::vector<double>& v, bool last = false) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i]);
  std::printf("]%s\n", last ? "" : ",");
}

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";   // where the level file round trip writes
  int fails = 0;
  std::printf("{\n");
  // ---------------------------------------------------------------- 1
  const int n = 8;
  PiecewiseConstant3D field;
  field.allocate(n, n, n);
  std::mt19937 rng(7);
  std::uniform_real_distribution<double> U(0.2, 0.95);
  std::vector<double> x0(n * n * n);
  for (auto& v : x0) v = U(rng);
  FEM3DFun fun;
  fun.gridSize = {n, n, n};
  fun.field = &field;
  fun.E = 1.0;
  fun.nu = 0.3;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      fun.wG[i * 6 + j] = (i <= 2 && j <= 2) ? 1.0 : 0.5;
      fun.G0[i * 6 + j] = (i == j) ? 0.05 : 0.0;
    }
  fun.m0 = 0.4;
  fun.mw = 0.1;
  fun.init(x0);
  fun.setParam(x0);
  const double f0 = fun.f();
  std::vector<double> G(fun.G.begin(), fun.G.end());
  std::vector<double> g = fun.df();
  const double hstep = 1e-6;
  std::vector<double> fd, an;
  for (int t = 0; t < 4; ++t) {
    const int k = (int)(rng() % x0.size());
    std::vector<double> xp = x0, xm = x0;
    xp[k] += hstep;
    xm[k] -= hstep;
    fun.setParam(xp);
    const double fp = fun.f();
    fun.setParam(xm);
    const double fm = fun.f();
    fd.push_back((fp - fm) / (2 * hstep));
    an.push_back(g[k]);
  }
  fun.setParam(x0);
  // a few descent steps (fast_fem/run3d.cpp:268-289): f must decrease
  std::vector<double> xo = x0;
  fun.lowerBounds.assign(x0.size(), 1e-3);
  fun.upperBounds.assign(x0.size(), 1.0);
  const int accepted = gradientDescent(&fun, xo, 3, 0.05);
  const double f_after = fun.f();
  if (accepted < 1 || !(f_after < f0)) ++fails;
  std::printf("\"descent_f\": [%.17g, %.17g], \"descent_steps\": %d,\n", f0, f_after, accepted);
  fun.setParam(x0);
  std::printf("\"f\": %.17g,\n", f0);
  std::printf("\"density\": %.17g,\n", fun.density);
  print_vec("G", G);
  print_vec("x0", x0);
  print_vec("df_fd", fd);
  print_vec("df_adjoint", an);
  // ------------------------------------------------------------- 1b
  // an 8^3 cell over a 4^3 PiecewiseConstant3D field (the field chain rule sums
  // eight voxels per parameter), parameters partly outside [1e-3, 1] (setParam
  // clamps), upper-triangular weights: the test compares G, f and df with the
  // reference's own FEM3DFun (oracle/_ref/libfastfem_ref.so)
  {
    PiecewiseConstant3D f4;
    f4.allocate(4, 4, 4);
    std::vector<double> x4(64);
    for (int i = 0; i < 64; ++i) x4[i] = -0.1 + 1.2 * ((i * 37 + 11) % 64) / 63.0;
    FEM3DFun fb;
    fb.gridSize = {n, n, n};
    fb.field = &f4;
    fb.E = 1.0;
    fb.nu = 0.3;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        fb.wG[i * 6 + j] = j >= i ? 0.5 + ((i * 5 + j * 3) % 7) / 7.0 : 0.0;
        fb.G0[i * 6 + j] = (i == j) ? (i < 3 ? 0.1 : 0.03) : (j > i ? 0.01 : 0.0);
      }
    fb.m0 = 0.4;
    fb.mw = 0.1;
    fb.init(x4);
    fb.setParam(x4);
    const double fv = fb.f();
    std::vector<double> gb = fb.df();
    std::printf("\"ff_f\": %.17g,\n", fv);
    print_vec("ff_x0", x4);
    print_vec("ff_G", std::vector<double>(fb.G.begin(), fb.G.end()));
    print_vec("ff_G0", std::vector<double>(fb.G0.begin(), fb.G0.end()));
    print_vec("ff_wG", std::vector<double>(fb.wG.begin(), fb.wG.end()));
    print_vec("ff_df", gb);
    // the same with run3D's cubic-symmetric field (fast_fem/run3d.cpp:176-182)
    PiecewiseConstantCubic3D fc;
    fc.allocate(4, 4, 4);
    fb.field = &fc;
    fb.setParam(x4);
    const double fvc = fb.f();
    std::vector<double> gc = fb.df();
    std::printf("\"ffc_f\": %.17g,\n", fvc);
    print_vec("ffc_G", std::vector<double>(fb.G.begin(), fb.G.end()));
    print_vec("ffc_df", gc);
  }
  // ---------------------------------------------------------------- 2
  NumericalCoarseningUsingMultigrid nc;
  int N[3] = {4, 4, 4};
  std::vector<BaseMaterial> mats = {{0.1, 0.15}, {1.0 / 2.6, 0.3 / (1.3 * 0.4)}};  // (mu, lambda)
  nc.init(N, 1, 2, mats, NumericalCoarseningUsingMultigrid::Cubic);
  std::vector<std::vector<int>> structs(3, std::vector<int>(64));
  for (auto& s : structs)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 4; ++k) {   // x<->y symmetric so the cubic relations are meaningful
          const int a = std::min(i, j), b = std::max(i, j);
          s[(i * 4 + j) * 4 + k] = ((a * 7 + b * 3 + k * 5 + (int)(&s - &structs[0])) % 3) != 0;
        }
  std::vector<double> dens = {0.0, 1.0};
  std::vector<double> tv, pv, tvb, pvb;
  for (auto& s : structs)
    nc.computeCoarsenedElasticityTensorAndParameters3D(s, N, dens, NumericalCoarseningUsingMultigrid::Cubic, tv, pv);
  nc.computeBatch(structs, N, dens, NumericalCoarseningUsingMultigrid::Cubic, tvb, pvb);
  double dmax = 0;
  for (size_t i = 0; i < tv.size(); ++i) dmax = std::fmax(dmax, std::fabs(tv[i] - tvb[i]));
  if (tv.size() != 63 || pv.size() != 12 || dmax > 1e-9) ++fails;
  print_vec("coarsened_tensors", tv);
  print_vec("coarsened_params", pv);
  std::printf("\"batch_max_diff\": %.3g,\n", dmax);
  std::vector<double> mat0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) mat0.push_back(structs[0][(i * 4 + j) * 4 + k]);
  print_vec("struct0", mat0);
  // ------------------------------------------------------------- 2b
  // femlib's force-driven NumericalCoarsening on the same structures and
  // materials (both base materials have nu = 0.3)
  NumericalCoarsening fc;
  fc.init(N, 1, 2, mats);
  std::vector<double> ftv, fpv, ftvb, fpvb;
  for (auto& s : structs)
    fc.computeCoarsenedElasticityTensorAndParameters3D(s, N, dens, NumericalCoarsening::Cubic, ftv, fpv);
  fc.computeBatch(structs, N, dens, NumericalCoarsening::Cubic, ftvb, fpvb);
  double fmax = 0;
  for (size_t i = 0; i < ftv.size(); ++i) fmax = std::fmax(fmax, std::fabs(ftv[i] - ftvb[i]));
  for (size_t i = 0; i < fpv.size(); ++i) fmax = std::fmax(fmax, std::fabs(fpv[i] - fpvb[i]));
  if (ftv.size() != 63 || fpv.size() != 12 || fpvb.size() != 12 || fmax > 1e-9) ++fails;
  std::vector<double> gtv, gpv;   // General: three Y, three nu, three G
  fc.computeCoarsenedElasticityTensorAndParameters3D(structs[0], N, dens, NumericalCoarsening::General, gtv, gpv);
  if (gpv.size() != 10) ++fails;
  bool rejected = false;   // a non-cubic cell is an argument error
  try {
    int M[3] = {4, 4, 2};
    std::vector<int> flat(32, 1);
    std::vector<double> t2, p2;
    fc.computeCoarsenedElasticityTensorAndParameters3D(flat, M, dens, NumericalCoarsening::Cubic, t2, p2);
  } catch (const Error& e) {
    rejected = e.code == FEMH_E_ARG;
  }
  if (!rejected) ++fails;
  print_vec("force_tensors", ftv);
  print_vec("force_params", fpv);
  print_vec("force_params_general", gpv);
  std::printf("\"force_batch_max_diff\": %.3g,\n", fmax);
  std::printf("\"force_noncubic_rejected\": %s,\n", rejected ? "true" : "false");
  // ---------------------------------------------------------------- 3
  const std::string tmp = dir + "/femh_level0_elasticityTensors.bin";
  std::vector<float> tf(tv.begin(), tv.end()), back;
  std::vector<std::vector<int>> back2;
  bool ok = writeBinary(tmp, tf) && readBinary(tmp, back) && back == tf;
  ok = ok && writeBinary(tmp, structs) && readBinary(tmp, back2) && back2 == structs;
  if (!ok) ++fails;
  std::printf("\"binary_roundtrip\": %s,\n", ok ? "true" : "false");
  std::printf("\"fails\": %d\n}\n", fails);
  return fails ? 1 : 0;
}
