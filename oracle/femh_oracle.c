/*
 * femh_oracle.c -- CPU FP64 restatement of the reference's periodic voxel
 * homogenization (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  The engine in fem_b200/ never
 * links or calls it.
 *
 * What it restates (paths are relative to the desaic/fem tree):
 *   - element stiffness K0: trilinear hex8, isotropic (E, nu), 2x2x2 Gauss
 *     (femlib/src/MaterialQuad.cpp:68-105, femlib/src/ElementHex.cpp:74-89,
 *     femlib/src/StrainLin.cpp:29-58, femlib/src/Quadrature.cpp:63-75; the
 *     closed form matlab/homogenize.m:121-167 is the same matrix).  Node order
 *     is the z-fastest `oneV` order of fast_fem/FEM3DFun.cpp:58-60
 *     (a = 4*ax + 2*ay + az), DOF 3*a + c.
 *   - per-voxel coefficient: SIMP E_min + rho^p (E_s - E_min)
 *     (MaterialOpt/src/FEM3DFun.cpp:244-257),
 *     x/(3-2x) (fast_fem/FEM3DFun.cpp:20-27) and the two-material coefficient
 *     {hi, lo} (SamplesGenerator/NumericalCoarseningUsingMultiGrid.cpp:235-241).
 *   - periodic six-load-case problem: total displacement u^I = eps^I x + chi^I
 *     with chi periodic (fast_fem/FEM3DFun.cpp:31-56 copyPeriodicU), unit
 *     macro strains in Voigt order xx,yy,zz,yz,xz,xy with engineering shear
 *     (MaterialOpt/src/Homogenize3D.cpp:196-201).
 *   - solve: Jacobi-preconditioned CG in FP64, node 0 pinned, relative 2-norm
 *     residual tolerance; loop shape of pcgsolver/pcg_solver.h:243-285.
 *   - C^H_IJ = (1/|Y|) sum_e c_e u^I_e . K0 u^J_e
 *     (fast_fem/FEM3DFun.cpp:163-180, NumericalCoarseningUsingMultiGrid.cpp:289-313).
 *   - dC^H_IJ/drho_e = c'(rho_e) u^I_e . K0 u^J_e / |Y| and the chain rule for a
 *     loss on C^H (fast_fem/FEM3DFun.cpp:222-268).
 *
 * Layouts: voxel/node index (i*ny + j)*nz + k (x slowest, z fastest, as
 * fast_fem/ArrayUtil.cpp gridToLinearIdx); voxel (i,j,k) has lower corner node
 * (i,j,k); fields are [rhs][node][3].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "femh_oracle.h"

static inline long nidx(int i, int j, int k, int ny, int nz) {
  return ((long)i * ny + j) * nz + k;
}

/* ---------------------------------------------------------------- K0 --- */
void fo_k0(double E, double nu, double h, double K[576]) {
  const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double mu = E / (2.0 * (1.0 + nu));
  double D[6][6];
  memset(D, 0, sizeof(D));
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) D[a][b] = lam;
  for (int a = 0; a < 3; ++a) D[a][a] += 2.0 * mu;
  D[3][3] = D[4][4] = D[5][5] = mu;
  memset(K, 0, 576 * sizeof(double));
  const double g = 1.0 / sqrt(3.0);
  const double gp[2] = {-g, g};
  for (int qx = 0; qx < 2; ++qx)
    for (int qy = 0; qy < 2; ++qy)
      for (int qz = 0; qz < 2; ++qz) {
        const double xi[3] = {gp[qx], gp[qy], gp[qz]};
        double B[6][24];
        memset(B, 0, sizeof(B));
        for (int a = 0; a < 8; ++a) {
          const double s[3] = {(double)(2 * ((a >> 2) & 1) - 1),
                               (double)(2 * ((a >> 1) & 1) - 1),
                               (double)(2 * (a & 1) - 1)};
          double dN[3];
          for (int d = 0; d < 3; ++d) {
            double v = s[d] / 8.0;
            for (int e = 0; e < 3; ++e)
              if (e != d) v *= (1.0 + s[e] * xi[e]);
            dN[d] = v * 2.0 / h; /* d/dx = (2/h) d/dxi */
          }
          B[0][3 * a + 0] = dN[0];
          B[1][3 * a + 1] = dN[1];
          B[2][3 * a + 2] = dN[2];
          B[3][3 * a + 1] = dN[2]; /* gamma_yz */
          B[3][3 * a + 2] = dN[1];
          B[4][3 * a + 0] = dN[2]; /* gamma_xz */
          B[4][3 * a + 2] = dN[0];
          B[5][3 * a + 0] = dN[1]; /* gamma_xy */
          B[5][3 * a + 1] = dN[0];
        }
        const double w = (h / 2.0) * (h / 2.0) * (h / 2.0);
        for (int p = 0; p < 24; ++p)
          for (int q = 0; q < 24; ++q) {
            double acc = 0.0;
            for (int m = 0; m < 6; ++m) {
              double dq = 0.0;
              for (int n = 0; n < 6; ++n) dq += D[m][n] * B[n][q];
              acc += B[m][p] * dq;
            }
            K[p * 24 + q] += w * acc;
          }
      }
}

/* ------------------------------------------------------ coefficients --- */
double fo_coef(const fo_material* m, double rho) {
  switch (m->interp) {
    case FO_INTERP_SIMP:
      return m->E_min + pow(rho, m->penal) * (m->E_s - m->E_min);
    case FO_INTERP_RAMP3:
      return m->E_s * rho / (3.0 - 2.0 * rho);
    case FO_INTERP_BINARY:
      return rho >= 0.5 ? m->bin_hi : m->bin_lo;
  }
  return 0.0;
}

double fo_dcoef(const fo_material* m, double rho) {
  switch (m->interp) {
    case FO_INTERP_SIMP:
      return m->penal * pow(rho, m->penal - 1.0) * (m->E_s - m->E_min);
    case FO_INTERP_RAMP3: {
      const double d = 3.0 - 2.0 * rho;
      return m->E_s * 3.0 / (d * d);
    }
    case FO_INTERP_BINARY:
      return 0.0;
  }
  return 0.0;
}

/* unit macro strain I as a symmetric 3x3 tensor (engineering shear) */
static void unit_strain(int I, double eps[3][3]) {
  memset(eps, 0, 9 * sizeof(double));
  switch (I) {
    case 0: eps[0][0] = 1; break;
    case 1: eps[1][1] = 1; break;
    case 2: eps[2][2] = 1; break;
    case 3: eps[1][2] = eps[2][1] = 0.5; break;
    case 4: eps[0][2] = eps[2][0] = 0.5; break;
    case 5: eps[0][1] = eps[1][0] = 0.5; break;
  }
}

void fo_affine(double h, double ue0[6][24]) {
  for (int I = 0; I < 6; ++I) {
    double eps[3][3];
    unit_strain(I, eps);
    for (int a = 0; a < 8; ++a) {
      const double x[3] = {h * ((a >> 2) & 1), h * ((a >> 1) & 1), h * (a & 1)};
      for (int c = 0; c < 3; ++c)
        ue0[I][3 * a + c] = eps[c][0] * x[0] + eps[c][1] * x[1] + eps[c][2] * x[2];
    }
  }
}

/* nodes of voxel (i,j,k) in oneV order */
static inline void elem_nodes(int i, int j, int k, int nx, int ny, int nz, long nd[8]) {
  for (int a = 0; a < 8; ++a) {
    const int ii = (i + ((a >> 2) & 1)) % nx;
    const int jj = (j + ((a >> 1) & 1)) % ny;
    const int kk = (k + (a & 1)) % nz;
    nd[a] = nidx(ii, jj, kk, ny, nz);
  }
}

/* y = K(coef) u for one right-hand side ([node][3]); work holds 24*nvox. */
void fo_apply1(int nx, int ny, int nz, const double* K0, const double* coef,
               const double* u, double* y, double* work) {
  const long nv = (long)nx * ny * nz;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < nv; ++e) {
    const int i = (int)(e / ((long)ny * nz));
    const int j = (int)((e / nz) % ny);
    const int k = (int)(e % nz);
    long nd[8];
    elem_nodes(i, j, k, nx, ny, nz, nd);
    double ue[24];
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * nd[a] + c];
    double* w = work + 24 * e;
    for (int p = 0; p < 24; ++p) {
      double acc = 0.0;
      for (int q = 0; q < 24; ++q) acc += K0[p * 24 + q] * ue[q];
      w[p] = coef[e] * acc;
    }
  }
  /* gather: node (i,j,k) is local node a of voxel (i-ax, j-ay, k-az) */
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n) {
    const int i = (int)(n / ((long)ny * nz));
    const int j = (int)((n / nz) % ny);
    const int k = (int)(n % nz);
    double acc[3] = {0, 0, 0};
    for (int a = 0; a < 8; ++a) {
      const int ei = (i - ((a >> 2) & 1) + nx) % nx;
      const int ej = (j - ((a >> 1) & 1) + ny) % ny;
      const int ek = (k - (a & 1) + nz) % nz;
      const double* w = work + 24 * nidx(ei, ej, ek, ny, nz);
      for (int c = 0; c < 3; ++c) acc[c] += w[3 * a + c];
    }
    for (int c = 0; c < 3; ++c) y[3 * n + c] = acc[c];
  }
}

void fo_apply(int nx, int ny, int nz, const double* K0, const double* coef,
              const double* u, double* y, int nrhs) {
  const long nv = (long)nx * ny * nz;
  double* work = (double*)malloc(sizeof(double) * 24 * nv);
  for (int r = 0; r < nrhs; ++r)
    fo_apply1(nx, ny, nz, K0, coef, u + 3 * nv * r, y + 3 * nv * r, work);
  free(work);
}

/* b^I = -sum_e c_e K0 ue0^I scattered to the voxel's nodes */
void fo_rhs(int nx, int ny, int nz, double h, const double* K0, const double* coef, double* b) {
  const long nv = (long)nx * ny * nz;
  double ue0[6][24], g[6][24];
  fo_affine(h, ue0);
  for (int I = 0; I < 6; ++I)
    for (int p = 0; p < 24; ++p) {
      double acc = 0.0;
      for (int q = 0; q < 24; ++q) acc += K0[p * 24 + q] * ue0[I][q];
      g[I][p] = acc;
    }
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n) {
    const int i = (int)(n / ((long)ny * nz));
    const int j = (int)((n / nz) % ny);
    const int k = (int)(n % nz);
    double acc[6][3];
    memset(acc, 0, sizeof(acc));
    for (int a = 0; a < 8; ++a) {
      const int ei = (i - ((a >> 2) & 1) + nx) % nx;
      const int ej = (j - ((a >> 1) & 1) + ny) % ny;
      const int ek = (k - (a & 1) + nz) % nz;
      const double ce = coef[nidx(ei, ej, ek, ny, nz)];
      for (int I = 0; I < 6; ++I)
        for (int c = 0; c < 3; ++c) acc[I][c] += ce * g[I][3 * a + c];
    }
    for (int I = 0; I < 6; ++I)
      for (int c = 0; c < 3; ++c) b[3 * nv * I + 3 * n + c] = -acc[I][c];
  }
}

/* inverse of the operator diagonal per DOF; node 0 (the pinned node) gets 0 */
void fo_inv_diag(int nx, int ny, int nz, const double* K0, const double* coef, double* dinv) {
  const long nv = (long)nx * ny * nz;
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n) {
    const int i = (int)(n / ((long)ny * nz));
    const int j = (int)((n / nz) % ny);
    const int k = (int)(n % nz);
    double acc[3] = {0, 0, 0};
    for (int a = 0; a < 8; ++a) {
      const int ei = (i - ((a >> 2) & 1) + nx) % nx;
      const int ej = (j - ((a >> 1) & 1) + ny) % ny;
      const int ek = (k - (a & 1) + nz) % nz;
      const double ce = coef[nidx(ei, ej, ek, ny, nz)];
      for (int c = 0; c < 3; ++c) acc[c] += ce * K0[(3 * a + c) * 24 + 3 * a + c];
    }
    for (int c = 0; c < 3; ++c) dinv[3 * n + c] = (n == 0) ? 0.0 : 1.0 / acc[c];
  }
}

static double dot(const double* a, const double* b, long n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* Jacobi-PCG for one RHS, node 0 pinned (x[0..2] = 0).  Returns iterations
 * (negative if max_iter was hit).  rel_out receives ||r||/||b||. */
int fo_pcg1(int nx, int ny, int nz, const double* K0, const double* coef, const double* dinv,
            const double* b, double* x, double tol, int max_iter, double* rel_out) {
  const long nv = (long)nx * ny * nz;
  const long nd = 3 * nv;
  double* r = (double*)malloc(sizeof(double) * nd);
  double* z = (double*)malloc(sizeof(double) * nd);
  double* p = (double*)malloc(sizeof(double) * nd);
  double* q = (double*)malloc(sizeof(double) * nd);
  double* work = (double*)malloc(sizeof(double) * 24 * nv);
  memset(x, 0, sizeof(double) * nd);
  memcpy(r, b, sizeof(double) * nd);
  r[0] = r[1] = r[2] = 0.0;
  const double bnorm = sqrt(dot(r, r, nd));
  int it = 0;
  double rel = 0.0;
  if (bnorm == 0.0) {
    *rel_out = 0.0;
    free(r); free(z); free(p); free(q); free(work);
    return 0;
  }
  for (long i = 0; i < nd; ++i) z[i] = dinv[i] * r[i];
  memcpy(p, z, sizeof(double) * nd);
  double rz = dot(r, z, nd);
  int converged = 0;
  for (it = 1; it <= max_iter; ++it) {
    fo_apply1(nx, ny, nz, K0, coef, p, q, work);
    q[0] = q[1] = q[2] = 0.0;
    const double pq = dot(p, q, nd);
    const double alpha = rz / pq;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nd; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rel = sqrt(dot(r, r, nd)) / bnorm;
    if (rel < tol) { converged = 1; break; }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nd; ++i) z[i] = dinv[i] * r[i];
    const double rz_new = dot(r, z, nd);
    const double beta = rz_new / rz;
    rz = rz_new;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nd; ++i) p[i] = z[i] + beta * p[i];
  }
  *rel_out = rel;
  free(r); free(z); free(p); free(q); free(work);
  return converged ? it : -max_iter;
}

/* per-voxel energies s_e[IJ] = u^I_e . K0 u^J_e (21 lower-triangle pairs,
 * row-major: (0,0),(1,0),(1,1),(2,0),...) ; u = affine + chi */
static void voxel_energies(int nx, int ny, int nz, double h, const double* K0, const double* chi,
                           long e, double s[21]) {
  const long nv = (long)nx * ny * nz;
  const int i = (int)(e / ((long)ny * nz));
  const int j = (int)((e / nz) % ny);
  const int k = (int)(e % nz);
  long nd[8];
  elem_nodes(i, j, k, nx, ny, nz, nd);
  double ue0[6][24];
  fo_affine(h, ue0);
  double u[6][24], w[6][24];
  for (int I = 0; I < 6; ++I)
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c)
        u[I][3 * a + c] = ue0[I][3 * a + c] + chi[3 * nv * I + 3 * nd[a] + c];
  for (int I = 0; I < 6; ++I)
    for (int p = 0; p < 24; ++p) {
      double acc = 0.0;
      for (int q = 0; q < 24; ++q) acc += K0[p * 24 + q] * u[I][q];
      w[I][p] = acc;
    }
  int t = 0;
  for (int I = 0; I < 6; ++I)
    for (int J = 0; J <= I; ++J) {
      double acc = 0.0;
      for (int p = 0; p < 24; ++p) acc += u[I][p] * w[J][p];
      s[t++] = acc;
    }
}

void fo_energy(int nx, int ny, int nz, double h, const double* K0, const double* coef,
               const double* chi, double C[36]) {
  const long nv = (long)nx * ny * nz;
  const double vol = (double)nv * h * h * h;
  double acc[21];
  memset(acc, 0, sizeof(acc));
#pragma omp parallel
  {
    double loc[21];
    memset(loc, 0, sizeof(loc));
#pragma omp for schedule(static)
    for (long e = 0; e < nv; ++e) {
      double s[21];
      voxel_energies(nx, ny, nz, h, K0, chi, e, s);
      for (int t = 0; t < 21; ++t) loc[t] += coef[e] * s[t];
    }
#pragma omp critical
    for (int t = 0; t < 21; ++t) acc[t] += loc[t];
  }
  int t = 0;
  for (int I = 0; I < 6; ++I)
    for (int J = 0; J <= I; ++J) {
      C[I * 6 + J] = C[J * 6 + I] = acc[t] / vol;
      ++t;
    }
}

void fo_dCdrho(int nx, int ny, int nz, double h, const double* K0, const fo_material* m,
               const double* rho, const double* chi, double* out /* [21][nv] */) {
  const long nv = (long)nx * ny * nz;
  const double vol = (double)nv * h * h * h;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < nv; ++e) {
    double s[21];
    voxel_energies(nx, ny, nz, h, K0, chi, e, s);
    const double dc = fo_dcoef(m, rho[e]) / vol;
    for (int t = 0; t < 21; ++t) out[(long)t * nv + e] = dc * s[t];
  }
}

void fo_grad(int nx, int ny, int nz, double h, const double* K0, const fo_material* m,
             const double* rho, const double* chi, const double dLdC[36], double* dLdrho) {
  const long nv = (long)nx * ny * nz;
  const double vol = (double)nv * h * h * h;
  /* symmetric weight per lower-triangle pair: G_IJ + G_JI off the diagonal */
  double wgt[21];
  int t = 0;
  for (int I = 0; I < 6; ++I)
    for (int J = 0; J <= I; ++J) {
      wgt[t++] = (I == J) ? dLdC[I * 6 + I] : dLdC[I * 6 + J] + dLdC[J * 6 + I];
    }
#pragma omp parallel for schedule(static)
  for (long e = 0; e < nv; ++e) {
    double s[21];
    voxel_energies(nx, ny, nz, h, K0, chi, e, s);
    double acc = 0.0;
    for (int q = 0; q < 21; ++q) acc += wgt[q] * s[q];
    dLdrho[e] = fo_dcoef(m, rho[e]) * acc / vol;
  }
}

int fo_homogenize(int nx, int ny, int nz, double h, const double* rho, const fo_material* m,
                  double tol, int max_iter, double C[36], double* chi_out, int iters[6],
                  double rel[6]) {
  const long nv = (long)nx * ny * nz;
  double K0[576];
  fo_k0(1.0, m->nu, h, K0);
  double* coef = (double*)malloc(sizeof(double) * nv);
  for (long e = 0; e < nv; ++e) coef[e] = fo_coef(m, rho[e]);
  double* b = (double*)malloc(sizeof(double) * 18 * nv);
  double* dinv = (double*)malloc(sizeof(double) * 3 * nv);
  double* chi = chi_out ? chi_out : (double*)malloc(sizeof(double) * 18 * nv);
  fo_rhs(nx, ny, nz, h, K0, coef, b);
  fo_inv_diag(nx, ny, nz, K0, coef, dinv);
  int status = 0;
  for (int I = 0; I < 6; ++I) {
    double rr = 0.0;
    const int it = fo_pcg1(nx, ny, nz, K0, coef, dinv, b + 3 * nv * I, chi + 3 * nv * I, tol,
                           max_iter, &rr);
    if (iters) iters[I] = it;
    if (rel) rel[I] = rr;
    if (it < 0) status = 1;
  }
  fo_energy(nx, ny, nz, h, K0, coef, chi, C);
  free(coef); free(b); free(dinv);
  if (!chi_out) free(chi);
  return status;
}

int fo_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
