// ref_fastfem.cpp -- C entry into the reference's own fast_fem FEM3DFun
// (fast_fem/FEM3DFun.cpp:128-268: setParam's field read, clamp and energy loop
// to G, f, and df with its field chain rule), over a PiecewiseConstant3D field
// (fast_fem/PiecewiseConstant3D.cpp), compiled from the reference sources in
// place by oracle/build_ref.sh into oracle/_ref/libfastfem_ref.so.  topoOptLib
// is absent from the reference tree: oracle/ref_shim/ holds stand-in headers
// whose Homogenize() runs the oracle's solve.  TEST INFRASTRUCTURE ONLY.
//
// ref_ff_eval: an n^3 cell, an m^3 field of `kind` (0 PiecewiseConstant3D,
// 1 PiecewiseConstantSym3D, 2 PiecewiseConstantCubic3D) with parameters x0, targets
// G0 / weights wG (6x6 row major), density target m0 and weight mw; set up as
// fast_fem/run3d.cpp:117-164 (initFEM) and :166-202 (run3D) set up the
// function -- lattice edge 1/n, Ke0 = the element stiffness of that edge
// (E = 1, nu), six (n+1)^3 displacement fields -- then setParam(x0), f(), df().
// Outputs G (6x6 as the reference fills it: upper triangle only), f, df (m^3),
// the clamped distribution (n^3) and the mean density.  Returns the stand-in
// solve's status (0 = converged).
#include <vector>

#include "FEM3DFun.hpp"
#include "PiecewiseConstant3D.hpp"
#include "PiecewiseConstantCubic3D.hpp"
#include "PiecewiseConstantSym3D.hpp"
#include "femh_oracle.h"

namespace {
// field kind 0: PiecewiseConstant3D, 1: PiecewiseConstantSym3D, 2: PiecewiseConstantCubic3D
RealField* make_field(int kind, int m) {
  if (kind == 1) {
    PiecewiseConstantSym3D* f = new PiecewiseConstantSym3D();
    f->allocate(m, m, m);
    return f;
  }
  if (kind == 2) {
    PiecewiseConstantCubic3D* f = new PiecewiseConstantCubic3D();
    f->allocate(m, m, m);
    return f;
  }
  PiecewiseConstant3D* f = new PiecewiseConstant3D();
  f->allocate(m, m, m);
  return f;
}
}  // namespace

// Parameter index that the reference's field of this kind (m^3 parameters)
// gives the point x (its df(x): one index, weight 1), or -1.
extern "C" int ref_field_index(int kind, int m, double x, double y, double z) {
  RealField* f = make_field(kind, m);
  Eigen::VectorXd c(3);
  c << x, y, z;
  Eigen::SparseVector<double> d = f->df(c);
  int idx = -1;
  for (Eigen::SparseVector<double>::InnerIterator it(d); it; ++it)
    if (it.value() == 1.0) idx = (int)it.index();
  delete f;
  return idx;
}

extern "C" int ref_ff_eval(int n, int m, int kind, double nu, const double* x0, const double* G0, const double* wG, double m0,
                           double mw, double* G_out, double* f_out, double* df_out, double* dist_out,
                           double* density_out) {
  const int nv = n * n * n;
  FEM3DFun fun;
  fun.lattice.dx = 1.0 / n;
  fun.fem.lattice.dx = 1.0 / n;
  fun.fem.nu = nu;
  fun.fem.Ke = Eigen::MatrixXd(24, 24);
  double K[576];
  fo_k0(1.0, nu, 1.0 / n, K);
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) fun.fem.Ke(i, j) = K[i * 24 + j];
  fun.Ke0.assign(1, fun.fem.Ke);
  fun.u.assign(6, Eigen::VectorXd::Zero(3 * (n + 1) * (n + 1) * (n + 1)));
  Homogenization<3> hom(fun.fem);
  fun.hom = &hom;
  Field<T, 3> coef;
  coef.Resize(Eigen::Vector3i(n, n, n));
  fun.fem.variable_coef = &coef;
  RealField* field = make_field(kind, m);
  fun.field = field;
  fun.gridSize[0] = fun.gridSize[1] = fun.gridSize[2] = n;
  fun.distribution.resize(nv);
  fun.param = field->param;
  fun.initArrays();
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      fun.G0(i, j) = G0[i * 6 + j];
      fun.wG(i, j) = wG[i * 6 + j];
    }
  fun.m0 = m0;
  fun.mw = mw;
  const int np = m * m * m;
  Eigen::VectorXd x(np);
  for (int i = 0; i < np; ++i) x[i] = x0[i];
  fun.setParam(x);
  *f_out = fun.f();
  Eigen::VectorXd g = fun.df();
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) G_out[i * 6 + j] = fun.G(i, j);
  for (int i = 0; i < np; ++i) df_out[i] = g[i];
  for (int i = 0; i < nv; ++i) dist_out[i] = fun.distribution[i];
  *density_out = fun.density;
  fun.hom = 0;
  delete field;
  return hom.status;
}
