// The C++ host layer on the CPU, linked against tests/cpp/fake_femh.cpp (a
// stand-in for the engine's C ABI): femlib's force-driven NumericalCoarsening
// (Cubic and General parameters, batch = one at a time, argument errors),
// NumericalCoarseningUsingMultigrid's parameters, and FEM3DFun's objective and
// chain rule.  Prints one JSON object; tests/test_host_logic.py recomputes
// every value from the fake's tensors.
#include <cstdio>
#include <random>
#include <vector>

#include "../../fem_b200/host/femh_host.hpp"

using namespace femh_host;

extern int g_batch_calls;   // tests/cpp/fake_femh.cpp
extern int g_fail_batch_call;
extern double g_fake_avail;

static void print_vec(const char* key, const std::vector<double>& v) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i]);
  std::printf("],\n");
}

template <class F>
static int error_code(F&& f) {
  try {
    f();
  } catch (const Error& e) {
    return e.code;
  }
  return 0;
}

int main() {
  std::printf("{\n");
  // femlib's force-driven class: 2^3 structures, subdivided twice -> 4^3 cells
  int N[3] = {2, 2, 2};
  std::vector<BaseMaterial> mats = {{0.1, 0.15}, {1.0 / 2.6, 0.3 / (1.3 * 0.4)}};   // nu = 0.3 both
  std::vector<std::vector<int>> structs = {{0, 1, 1, 0, 1, 0, 0, 1}, {1, 1, 1, 0, 1, 1, 0, 1}, {0, 0, 1, 0, 0, 1, 0, 0}};
  std::vector<double> dens = {0.1, 0.9};
  NumericalCoarsening fc;
  fc.init(N, 1, 2, mats);
  std::vector<double> tv, pv, tvb, pvb, tvg, pvg;
  for (auto& s : structs)
    fc.computeCoarsenedElasticityTensorAndParameters3D(s, N, dens, NumericalCoarsening::Cubic, tv, pv);
  fc.computeBatch(structs, N, dens, NumericalCoarsening::Cubic, tvb, pvb);
  fc.computeCoarsenedElasticityTensorAndParameters3D(structs[0], N, dens, NumericalCoarsening::General, tvg, pvg);
  print_vec("force_tensors", tv);
  print_vec("force_params", pv);
  print_vec("force_tensors_batch", tvb);
  print_vec("force_params_batch", pvb);
  print_vec("force_params_general", pvg);
  {   // split into calls of one 4^3 structure each: same outputs, one call per structure
    std::vector<double> ts, ps;
    fc.maxNodesPerCall = 64;
    const int before = g_batch_calls;
    fc.computeBatch(structs, N, dens, NumericalCoarsening::Cubic, ts, ps);
    std::printf("\"force_split_calls\": %d,\n", g_batch_calls - before);
    std::printf("\"force_split_equal\": %s,\n", (ts == tvb && ps == pvb) ? "true" : "false");
    // default split: what fits the device -- 0.92 x 150 kB over 64 kB a cell = 2 cells per call
    std::vector<double> ta, pa;
    fc.maxNodesPerCall = 0;
    g_fake_avail = 150e3;
    const int before_auto = g_batch_calls;
    fc.computeBatch(structs, N, dens, NumericalCoarsening::Cubic, ta, pa);
    std::printf("\"force_auto_calls\": %d,\n", g_batch_calls - before_auto);
    std::printf("\"force_auto_equal\": %s,\n", (ta == tvb && pa == pvb) ? "true" : "false");
    // a failing second call (FEMH_E_OOM) leaves the caller's vectors as they were
    std::vector<double> tk = {7.0}, pk = {8.0, 9.0};
    fc.maxNodesPerCall = 64;
    g_fail_batch_call = g_batch_calls + 2;
    const int code = error_code([&] { fc.computeBatch(structs, N, dens, NumericalCoarsening::Cubic, tk, pk); });
    g_fail_batch_call = -1;
    std::printf("\"force_failed_code\": %d,\n", code);
    std::printf("\"force_failed_untouched\": %s,\n",
                (tk == std::vector<double>{7.0} && pk == std::vector<double>{8.0, 9.0}) ? "true" : "false");
    g_fake_avail = 1e12;
    fc.maxNodesPerCall = 0;
  }
  std::vector<double> cell0;   // structure 0 after repMaterialAssignment
  {
    std::vector<int> m;
    repMaterialAssignment(2, 2, 2, structs[0], 1, 1, 1, 2, m);
    for (int v : m) cell0.push_back(v);
  }
  print_vec("cell0", cell0);
  std::vector<double> t2, p2;
  int M[3] = {2, 2, 1};
  std::printf("\"err_noncubic\": %d,\n", error_code([&] {
    fc.computeCoarsenedElasticityTensorAndParameters3D(std::vector<int>(4, 1), M, dens, NumericalCoarsening::Cubic,
                                                       t2, p2);
  }));
  std::printf("\"err_material_index\": %d,\n", error_code([&] {
    fc.computeCoarsenedElasticityTensorAndParameters3D({0, 1, 2, 0, 1, 0, 0, 1}, N, dens, NumericalCoarsening::Cubic,
                                                       t2, p2);
  }));
  std::printf("\"err_nu_mismatch\": %d,\n", error_code([&] {
    NumericalCoarsening bad;
    bad.init(N, 1, 1, {{0.1, 0.3}, {1.0, 1.0}});
  }));
  std::printf("\"err_void\": %d,\n", error_code([&] {
    NumericalCoarsening bad;
    bad.init(N, 1, 1, {{0.0, 0.0}, {1.0, 1.0}});
  }));
  std::printf("\"err_uninitialised\": %d,\n", error_code([&] {
    NumericalCoarsening bad;
    bad.computeCoarsenedElasticityTensorAndParameters3D(structs[0], N, dens, NumericalCoarsening::Cubic, t2, p2);
  }));
  // NumericalCoarseningUsingMultigrid
  NumericalCoarseningUsingMultigrid mg;
  mg.init(N, 1, 2, mats, NumericalCoarseningUsingMultigrid::Cubic);
  std::vector<double> mtv, mpv;
  mg.computeCoarsenedElasticityTensorAndParameters3D(structs[0], N, dens, NumericalCoarseningUsingMultigrid::Cubic,
                                                     mtv, mpv);
  print_vec("mg_tensors", mtv);
  print_vec("mg_params", mpv);
  {
    std::vector<double> t1, p1, t2, p2;
    mg.computeBatch(structs, N, dens, NumericalCoarseningUsingMultigrid::Cubic, t1, p1);
    mg.maxNodesPerCall = 128;   // two 4^3 structures per call
    const int before = g_batch_calls;
    mg.computeBatch(structs, N, dens, NumericalCoarseningUsingMultigrid::Cubic, t2, p2);
    std::printf("\"mg_split_calls\": %d,\n", g_batch_calls - before);
    std::printf("\"mg_split_equal\": %s,\n", (t1 == t2 && p1 == p2) ? "true" : "false");
    std::vector<double> tk = {1.0}, pk = {2.0};
    g_fail_batch_call = g_batch_calls + 2;
    const int code = error_code([&] { mg.computeBatch(structs, N, dens, NumericalCoarseningUsingMultigrid::Cubic, tk, pk); });
    g_fail_batch_call = -1;
    std::printf("\"mg_failed_code\": %d,\n", code);
    std::printf("\"mg_failed_untouched\": %s,\n",
                (tk == std::vector<double>{1.0} && pk == std::vector<double>{2.0}) ? "true" : "false");
    mg.maxNodesPerCall = 0;
  }
  {   // the reference's tensor files: the 15 off-diagonal lower-triangle values are 0
    std::vector<double> tr, pr;
    mg.referenceLowerTriangle = true;
    mg.computeCoarsenedElasticityTensorAndParameters3D(structs[0], N, dens, NumericalCoarseningUsingMultigrid::Cubic,
                                                       tr, pr);
    mg.referenceLowerTriangle = false;
    print_vec("mg_tensors_reference_triangle", tr);
    print_vec("mg_params_reference_triangle", pr);
  }
  // FEM3DFun objective and chain rule through a piecewise-constant field
  const int n = 4;
  PiecewiseConstant3D field;
  field.allocate(2, 2, 2);
  FEM3DFun fun;
  fun.gridSize = {n, n, n};
  fun.field = &field;
  fun.E = 2.0;
  fun.nu = 0.25;
  for (int i = 0; i < 36; ++i) {
    fun.wG[i] = 1.0 + 0.1 * (i % 7);
    fun.G0[i] = (i % 7 == 0) ? 0.3 : 0.01;
  }
  fun.m0 = 0.4;
  fun.mw = 0.7;
  std::vector<double> x0 = {0.2, 0.5, 0.9, 0.0005, 0.6, 0.3, 1.2, 0.45};   // two clamped
  fun.init(x0);
  fun.setParam(x0);
  std::vector<double> G(fun.G.begin(), fun.G.end());
  print_vec("fun_x0", x0);
  print_vec("fun_G", G);
  print_vec("fun_distribution", fun.distribution);
  std::printf("\"fun_density\": %.17g,\n", fun.density);
  std::printf("\"fun_f\": %.17g,\n", fun.f());
  print_vec("fun_df", fun.df());
  {   // voxel -> parameter maps of the symmetric fields (3^3 parameters on a 7 x 8 x 9 grid)
    const int n3[3] = {7, 8, 9};
    PiecewiseConstantSym3D sym;
    sym.allocate(3, 3, 3);
    PiecewiseConstantCubic3D cub;
    cub.allocate(3, 3, 3);
    std::vector<int> ms, mc;
    sym.voxelMap(n3, ms);
    cub.voxelMap(n3, mc);
    print_vec("map_sym", std::vector<double>(ms.begin(), ms.end()));
    print_vec("map_cubic", std::vector<double>(mc.begin(), mc.end()));
  }
  std::printf("\"ok\": true\n}\n");
  return 0;
}
