/*
 * femh_oracle_mg.c -- CPU FP64 geometric-multigrid PCG for the periodic voxel
 * homogenization (TEST INFRASTRUCTURE ONLY: the checker and the timed CPU
 * baseline, never the product; the engine in fem_b200/ never links or calls it).
 *
 * Same problem and outputs as fo_homogenize in femh_oracle.c (which restates
 * the reference's plain method with Jacobi-PCG); this file solves it with the
 * method the reference runs for this path -- topoOptLib's geometric multigrid
 * preconditioned Krylov solve, configured in fast_fem/run3d.cpp:118-137 and
 * SamplesGenerator/NumericalCoarseningUsingMultiGrid.cpp:147-168 (levels,
 * V-cycles, Krylov iterations) -- so that 128^3 and 256^3 cells converge to
 * 1e-10 in seconds to minutes on the host cores:
 *   - levels: the cell halves while every extent is even and the level has
 *     more than `coarse_max` nodes; coarse modulus = arithmetic mean of the 8
 *     children, voxel edge doubled (rediscretisation);
 *   - smoother: damped Jacobi, `pre` sweeps down and `post` sweeps up, weights
 *     the reciprocal roots of the Chebyshev polynomial of that degree on
 *     [lmax/ratio, lmax], lmax = the largest eigenvalue of diag(K0)^-1 K0
 *     (ratio 0: every sweep damped by 0.35);
 *   - transfers: trilinear prolongation P and full-weighting restriction P^T;
 *   - coarsest level: dense FP64 Cholesky of the operator with node 0 removed;
 *   - node 0 of every level is pinned (the three translations);
 *   - CG: x0 = 0, relative 2-norm residual ||b - K x|| / ||b|| < tol per load
 *     case (loop shape of pcgsolver/pcg_solver.h:243-285 with a V-cycle as the
 *     preconditioner).
 * The operator apply is the element-by-element product with K0 written in the
 * Hadamard basis of the element's 2x2x2 nodes, K0 = T^T Kh T / 64 (T the +-1
 * characters of the 8 corners, Kh = T K0 T^T computed numerically from K0 and
 * kept sparse), vectorised along z rows.  It equals fo_apply (dense K0) to
 * rounding, which tests/test_oracle_mg.py checks.
 *
 * Layout inside this file: [rhs][comp][node], node (i*ny + j)*nz + k.  The
 * fluctuation handed back uses femh_oracle.c's [rhs][node][comp].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "femh_oracle.h"

#define NR 6
#define MAXLEV 16
static const double kPi = 3.14159265358979323846;

typedef struct {
  int nnz;
  int cnt[24];        /* nonzeros of output row P (at most 3: Kh is block diagonal) */
  int q[24][24];
  double v[24][24];
} hadk_t;

typedef struct {
  int nx, ny, nz;
  long nv;
  double* kc;     /* [nv] modulus x voxel edge: the voxel's K0(1) multiplier */
  double* dinv;   /* [3][nv] inverse operator diagonal, 0 at node 0 */
  double* binv;   /* node-block smoother: [nv][6] inverse 3x3 diagonal blocks (xx yy zz xy xz yz), or NULL */
  double* x;      /* [6][3][nv] */
  double* b;
  double* t;
  int m;          /* coarsest level: unknowns (3 (nv - 1)), else 0 */
  double* L;      /* coarsest level: Cholesky factor, m x m row major */
} mglev_t;

typedef struct {
  int nlev;
  mglev_t lv[MAXLEV];
  hadk_t hk;
  double K0[576];   /* K0(1) */
  int pre, post;
  int block;        /* node-block Jacobi sweeps */
  double wpre[16], wpost[16];
} mg_t;

static inline int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

/* ------------------------------------------------ Hadamard form of K0 --- */
static inline int hchar(int kk, int a) { return (__builtin_popcount(kk & a) & 1) ? -1 : 1; }

static void hadamard_k(const double K0[576], hadk_t* H) {
  double Kh[24][24];
  double mx = 0.0;
  for (int P = 0; P < 24; ++P)
    for (int Q = 0; Q < 24; ++Q) {
      const int kk = P / 3, c = P % 3, kk2 = Q / 3, c2 = Q % 3;
      double s = 0.0;
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) s += hchar(kk, a) * hchar(kk2, b) * K0[(3 * a + c) * 24 + 3 * b + c2];
      Kh[P][Q] = s;
      if (fabs(s) > mx) mx = fabs(s);
    }
  H->nnz = 0;
  for (int P = 0; P < 24; ++P) {
    H->cnt[P] = 0;
    for (int Q = 0; Q < 24; ++Q)
      if (fabs(Kh[P][Q]) > 1e-13 * mx) {
        H->q[P][H->cnt[P]] = Q;
        H->v[P][H->cnt[P]] = Kh[P][Q] / 64.0;
        H->cnt[P]++;
        H->nnz++;
      }
  }
}

/* +-1 butterfly stages over the corner bits `bits` (4 = ax, 2 = ay, 1 = az)
 * of 24 rows (8 corners x 3 comps, a = 4ax + 2ay + az) of a block of KB
 * voxels.  The Hadamard transform is its own transpose, so the same stages
 * map corner values to characters and back. */
#define KB 64
static inline void bfly2(double* restrict lo, double* restrict hi) {
  for (int k = 0; k < KB; ++k) {
    const double s = lo[k] + hi[k], d = lo[k] - hi[k];
    lo[k] = s;
    hi[k] = d;
  }
}

static void butterfly_xy(double (*v)[KB]) {
  for (int bit = 2; bit <= 4; bit <<= 1)
    for (int a = 0; a < 8; ++a) {
      if (a & bit) continue;
      for (int c = 0; c < 3; ++c) bfly2(v[3 * a + c], v[3 * (a | bit) + c]);
    }
}

/* ------------------------------------------------------------- apply --- */
/* one voxel row (i, j) of load case r: the row's element products added to
 * the node-plane accumulators lo (node plane i) and hi (node plane i+1),
 * each [3][ny*nz]; a NULL accumulator drops that half.  Blocks of KB voxels
 * along z keep the 24 corner rows in L1; the z stage of the transform is
 * fused into the gather and the scatter, the kc scale into the Kh product. */
static void apply_row(const mglev_t* L, const hadk_t* H, const double* u, int r, int i, int j, double* lo,
                      double* hi) {
  const int ny = L->ny, nz = L->nz;
  const long nv = L->nv, plane = (long)ny * nz;
  const double* kc = L->kc + ((long)i * ny + j) * nz;
  const double* urow[4];
  double* orow[4];
  for (int ax = 0; ax < 2; ++ax)
    for (int ay = 0; ay < 2; ++ay) {
      const long prow = (long)wrapi(j + ay, ny) * nz;
      urow[2 * ax + ay] = u + (long)r * 3 * nv + (long)wrapi(i + ax, L->nx) * plane + prow;
      double* acc = ax ? hi : lo;
      orow[2 * ax + ay] = acc ? acc + prow : NULL;
    }
  double V[24][KB], W[24][KB], up[KB + 1];
  for (int k0 = 0; k0 < nz; k0 += KB) {
    const int kn = nz - k0 < KB ? nz - k0 : KB;
    /* gather + z stage: corners (.., az=0) and (.., az=1) of node row (ax, ay) */
    for (int g = 0; g < 4; ++g)
      for (int c = 0; c < 3; ++c) {
        const double* src = urow[g] + (long)c * nv;
        for (int k = 0; k < kn; ++k) up[k] = src[k0 + k];
        up[kn] = src[k0 + kn < nz ? k0 + kn : 0];
        for (int k = kn + 1; k <= KB; ++k) up[k] = 0.0;
        double* restrict s0 = V[3 * (2 * g) + c];
        double* restrict s1 = V[3 * (2 * g + 1) + c];
        for (int k = 0; k < KB; ++k) {
          s0[k] = up[k] + up[k + 1];
          s1[k] = up[k] - up[k + 1];
        }
      }
    butterfly_xy(V);
    for (int P = 0; P < 24; ++P) {
      double* restrict w = W[P];
      const int n = H->cnt[P];
      if (n == 0) {
        for (int k = 0; k < KB; ++k) w[k] = 0.0;
        continue;
      }
      const double* restrict v0 = V[H->q[P][0]];
      const double h0 = H->v[P][0];
      if (n == 1) {
        for (int k = 0; k < kn; ++k) w[k] = kc[k0 + k] * (h0 * v0[k]);
      } else if (n == 2) {
        const double* restrict v1 = V[H->q[P][1]];
        const double h1 = H->v[P][1];
        for (int k = 0; k < kn; ++k) w[k] = kc[k0 + k] * (h0 * v0[k] + h1 * v1[k]);
      } else if (n == 3) {
        const double* restrict v1 = V[H->q[P][1]];
        const double* restrict v2 = V[H->q[P][2]];
        const double h1 = H->v[P][1], h2 = H->v[P][2];
        for (int k = 0; k < kn; ++k) w[k] = kc[k0 + k] * (h0 * v0[k] + h1 * v1[k] + h2 * v2[k]);
      } else {   /* not reached for an isotropic K0 (blocks of at most 3) */
        for (int k = 0; k < kn; ++k) {
          double acc = 0.0;
          for (int t = 0; t < n; ++t) acc += H->v[P][t] * V[H->q[P][t]][k];
          w[k] = kc[k0 + k] * acc;
        }
      }
      for (int k = kn; k < KB; ++k) w[k] = 0.0;
    }
    butterfly_xy(W);
    /* z stage + scatter: corner az=0 -> node k, az=1 -> node k+1 */
    for (int g = 0; g < 4; ++g) {
      double* out = orow[g];
      if (!out) continue;
      for (int c = 0; c < 3; ++c) {
        double* dst = out + (long)c * plane;
        const double* restrict f0 = W[3 * (2 * g) + c];
        const double* restrict f1 = W[3 * (2 * g + 1) + c];
        /* node k0 + k gets (f0 + f1)[k] + (f0 - f1)[k - 1] */
        for (int k = 0; k < kn; ++k) dst[k0 + k] += f0[k] + f1[k];
        for (int k = 0; k + 1 < kn; ++k) dst[k0 + k + 1] += f0[k] - f1[k];
        dst[k0 + kn < nz ? k0 + kn : 0] += f0[kn - 1] - f1[kn - 1];
      }
    }
  }
}

/* y = K u for the six load cases of a level; y[node 0] = 0 (pinned).
 * Each thread owns a slab of node planes [i0, i1): it runs the voxel planes
 * i0-1 .. i1-1 (plane i0-1 only for its upper half, which lands on node plane
 * i0) through two node-plane accumulators, and writes every node plane of y
 * once. */
static void mg_apply(const mglev_t* L, const hadk_t* H, const double* u, double* y) {
  const int nx = L->nx, ny = L->ny;
  const long nv = L->nv, plane = (long)ny * L->nz;
#pragma omp parallel
  {
#ifdef _OPENMP
    const int nt = omp_get_num_threads(), tid = omp_get_thread_num();
#else
    const int nt = 1, tid = 0;
#endif
    const int ns = nt < nx ? nt : nx;
    double* cur = (double*)malloc(sizeof(double) * 3 * plane);
    double* nxt = (double*)malloc(sizeof(double) * 3 * plane);
    for (int sl = tid; sl < ns; sl += nt) {
      const int i0 = (int)((long)sl * nx / ns), i1 = (int)((long)(sl + 1) * nx / ns);
      for (int r = 0; r < NR; ++r) {
        memset(cur, 0, sizeof(double) * 3 * plane);
        const int ip = wrapi(i0 - 1, nx);
        for (int j = 0; j < ny; ++j) apply_row(L, H, u, r, ip, j, NULL, cur);
        for (int p = i0; p < i1; ++p) {
          const int last = p + 1 == i1;
          if (!last) memset(nxt, 0, sizeof(double) * 3 * plane);
          for (int j = 0; j < ny; ++j) apply_row(L, H, u, r, p, j, cur, last ? NULL : nxt);
          for (int c = 0; c < 3; ++c)
            memcpy(y + ((long)r * 3 + c) * nv + (long)p * plane, cur + (long)c * plane, sizeof(double) * plane);
          double* t = cur;
          cur = nxt;
          nxt = t;
        }
      }
    }
    free(cur);
    free(nxt);
  }
  for (int r = 0; r < NR; ++r)
    for (int c = 0; c < 3; ++c) y[((long)r * 3 + c) * nv] = 0.0;
}

/* ------------------------------------------------------------- levels --- */
static double lmax_bound(const double K0[576], int block) {
  /* largest eigenvalue of D^-1 K0 (D the diagonal, or with block the 3x3 node
     blocks) by power iteration on the symmetric L^-1 K0 L^-T, L = chol(D) */
  double Li[576];
  memset(Li, 0, sizeof(Li));
  for (int a = 0; a < 8; ++a) {
    if (!block) {
      for (int c = 0; c < 3; ++c) Li[(3 * a + c) * 25] = 1.0 / sqrt(K0[(3 * a + c) * 25]);
      continue;
    }
    double L[3][3] = {{0}}, I[3][3] = {{0}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j <= i; ++j) {
        double v = K0[(3 * a + i) * 24 + 3 * a + j];
        for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k];
        L[i][j] = (i == j) ? sqrt(v) : v / L[j][j];
      }
    for (int c = 0; c < 3; ++c)
      for (int i = 0; i < 3; ++i) {
        double v = (i == c) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) v -= L[i][k] * I[k][c];
        I[i][c] = v / L[i][i];
      }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Li[(3 * a + i) * 24 + 3 * a + j] = I[i][j];
  }
  double S[576], T[576];
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) {
      double v = 0.0;
      for (int k = 0; k < 24; ++k) v += Li[i * 24 + k] * K0[k * 24 + j];
      T[i * 24 + j] = v;
    }
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) {
      double v = 0.0;
      for (int k = 0; k < 24; ++k) v += T[i * 24 + k] * Li[j * 24 + k];
      S[i * 24 + j] = v;
    }
  double x[24], y[24];
  for (int p = 0; p < 24; ++p) x[p] = 1.0 + 0.01 * p;
  double lam = 0.0;
  for (int it = 0; it < 2000; ++it) {
    double nrm = 0.0;
    for (int p = 0; p < 24; ++p) {
      double sacc = 0.0;
      for (int q = 0; q < 24; ++q) sacc += S[p * 24 + q] * x[q];
      y[p] = sacc;
      nrm += sacc * sacc;
    }
    nrm = sqrt(nrm);
    double dotv = 0.0, xn = 0.0;
    for (int p = 0; p < 24; ++p) {
      dotv += x[p] * y[p];
      xn += x[p] * x[p];
    }
    lam = dotv / xn;
    for (int p = 0; p < 24; ++p) x[p] = y[p] / nrm;
  }
  return lam;
}

static void weights(int m, double lmax, double ratio, double* w) {
  if (ratio <= 0.0) {
    for (int s = 0; s < m; ++s) w[s] = 0.35;
    return;
  }
  const double a = lmax / ratio, b = lmax;
  for (int s = 0; s < m; ++s) {
    /* roots in decreasing order -> weights in increasing order */
    const double root = 0.5 * (a + b) + 0.5 * (b - a) * cos((2.0 * s + 1.0) * kPi / (2.0 * m));
    w[s] = 1.0 / root;
  }
}

static void level_diag(mglev_t* L, const double K0[576]) {
  const long nv = L->nv;
  const int nx = L->nx, ny = L->ny, nz = L->nz;
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n) {
    const int i = (int)(n / ((long)ny * nz)), j = (int)((n / nz) % ny), k = (int)(n % nz);
    double acc[3] = {0, 0, 0};
    for (int a = 0; a < 8; ++a) {
      const long e = ((long)wrapi(i - ((a >> 2) & 1), nx) * ny + wrapi(j - ((a >> 1) & 1), ny)) * nz +
                     wrapi(k - (a & 1), nz);
      for (int c = 0; c < 3; ++c) acc[c] += L->kc[e] * K0[(3 * a + c) * 25];
    }
    for (int c = 0; c < 3; ++c) L->dinv[(long)c * nv + n] = n == 0 ? 0.0 : 1.0 / acc[c];
  }
}

/* node-block smoother: D_n = sum over the 8 voxels at n of kc_e K0_aa (the
   3x3 diagonal block of K at n), inverted; 0 at node 0 */
static void level_block(mglev_t* L, const double K0[576]) {
  const long nv = L->nv;
  const int nx = L->nx, ny = L->ny, nz = L->nz;
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n) {
    const int i = (int)(n / ((long)ny * nz)), j = (int)((n / nz) % ny), k = (int)(n % nz);
    double D[3][3] = {{0}};
    for (int a = 0; a < 8; ++a) {
      const long e = ((long)wrapi(i - ((a >> 2) & 1), nx) * ny + wrapi(j - ((a >> 1) & 1), ny)) * nz +
                     wrapi(k - (a & 1), nz);
      for (int c1 = 0; c1 < 3; ++c1)
        for (int c2 = 0; c2 < 3; ++c2) D[c1][c2] += L->kc[e] * K0[(3 * a + c1) * 24 + 3 * a + c2];
    }
    double* o = L->binv + 6 * n;
    if (n == 0) {
      for (int q = 0; q < 6; ++q) o[q] = 0.0;
      continue;
    }
    const double c00 = D[1][1] * D[2][2] - D[1][2] * D[2][1], c01 = D[1][2] * D[2][0] - D[1][0] * D[2][2],
                 c02 = D[1][0] * D[2][1] - D[1][1] * D[2][0];
    const double det = D[0][0] * c00 + D[0][1] * c01 + D[0][2] * c02;
    o[0] = c00 / det;
    o[1] = (D[0][0] * D[2][2] - D[0][2] * D[2][0]) / det;
    o[2] = (D[0][0] * D[1][1] - D[0][1] * D[1][0]) / det;
    o[3] = c01 / det;
    o[4] = c02 / det;
    o[5] = (D[0][2] * D[1][0] - D[0][0] * D[1][2]) / det;
  }
}

/* x (+)= w D^-1 v for the 3 components of every node: v = b - t, or b alone
   when t == NULL (with from_zero the sweep starts x from zero) */
static void block_sweep(const mglev_t* L, double* x, const double* b, const double* t, double w, int from_zero) {
  const long nv = L->nv;
#pragma omp parallel for schedule(static)
  for (long rn = 0; rn < 6 * nv; ++rn) {
    const long rr = rn / nv, n = rn % nv;
    const double* B = L->binv + 6 * n;
    double v[3];
    for (int c = 0; c < 3; ++c) {
      const long q = (rr * 3 + c) * nv + n;
      v[c] = t ? b[q] - t[q] : b[q];
    }
    const double d0 = B[0] * v[0] + B[3] * v[1] + B[4] * v[2];
    const double d1 = B[3] * v[0] + B[1] * v[1] + B[5] * v[2];
    const double d2 = B[4] * v[0] + B[5] * v[1] + B[2] * v[2];
    const long q0 = (rr * 3) * nv + n;
    if (from_zero) {
      x[q0] = w * d0;
      x[q0 + nv] = w * d1;
      x[q0 + 2 * nv] = w * d2;
    } else {
      x[q0] += w * d0;
      x[q0 + nv] += w * d1;
      x[q0 + 2 * nv] += w * d2;
    }
  }
}

/* dense operator of the coarsest level without node 0, Cholesky-factorised */
static int level_coarse(mglev_t* L, const double K0[576]) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long nv = L->nv;
  const int m = (int)(3 * (nv - 1));
  L->m = m;
  if (m <= 0) return 0;
  double* A = (double*)calloc((size_t)m * m, sizeof(double));
  for (long e = 0; e < nv; ++e) {
    const int i = (int)(e / ((long)ny * nz)), j = (int)((e / nz) % ny), k = (int)(e % nz);
    long nd[8];
    for (int a = 0; a < 8; ++a)
      nd[a] = ((long)wrapi(i + ((a >> 2) & 1), nx) * ny + wrapi(j + ((a >> 1) & 1), ny)) * nz + wrapi(k + (a & 1), nz);
    for (int a = 0; a < 8; ++a) {
      if (nd[a] == 0) continue;
      for (int b = 0; b < 8; ++b) {
        if (nd[b] == 0) continue;
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d)
            A[(3 * (nd[a] - 1) + c) * (long)m + 3 * (nd[b] - 1) + d] += L->kc[e] * K0[(3 * a + c) * 24 + 3 * b + d];
      }
    }
  }
  for (int j = 0; j < m; ++j) {
    double s = A[(long)j * m + j];
    for (int p = 0; p < j; ++p) s -= A[(long)j * m + p] * A[(long)j * m + p];
    if (!(s > 0.0)) {
      free(A);
      return -1;
    }
    const double d = sqrt(s);
    A[(long)j * m + j] = d;
    for (int i = j + 1; i < m; ++i) {
      double t = A[(long)i * m + j];
      for (int p = 0; p < j; ++p) t -= A[(long)i * m + p] * A[(long)j * m + p];
      A[(long)i * m + j] = t / d;
    }
  }
  L->L = A;
  return 0;
}

static void coarse_solve(const mglev_t* L, const double* b, double* x) {
  const long nv = L->nv;
  const int m = L->m;
  double* y = (double*)malloc(sizeof(double) * (m > 0 ? m : 1));
  for (int r = 0; r < NR; ++r) {
    for (int c = 0; c < 3; ++c) x[((long)r * 3 + c) * nv] = 0.0;
    for (int p = 0; p < m; ++p) y[p] = b[((long)r * 3 + p % 3) * nv + 1 + p / 3];
    for (int i = 0; i < m; ++i) {
      double s = y[i];
      for (int p = 0; p < i; ++p) s -= L->L[(long)i * m + p] * y[p];
      y[i] = s / L->L[(long)i * m + i];
    }
    for (int i = m - 1; i >= 0; --i) {
      double s = y[i];
      for (int p = i + 1; p < m; ++p) s -= L->L[(long)p * m + i] * y[p];
      y[i] = s / L->L[(long)i * m + i];
    }
    for (int p = 0; p < m; ++p) x[((long)r * 3 + p % 3) * nv + 1 + p / 3] = y[p];
  }
  free(y);
}

/* ---------------------------------------------------------- transfers --- */
static void restrict_fw(const mglev_t* F, const mglev_t* C, const double* rf, double* bc) {
  const long nvf = F->nv, nvc = C->nv;
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nvc; ++n) {
    const int i = (int)(n / ((long)C->ny * C->nz)), j = (int)((n / C->nz) % C->ny), k = (int)(n % C->nz);
    double acc[NR][3];
    memset(acc, 0, sizeof(acc));
    if (n != 0)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            const double w = (dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0);
            const long g = ((long)wrapi(2 * i + dx, F->nx) * F->ny + wrapi(2 * j + dy, F->ny)) * F->nz +
                           wrapi(2 * k + dz, F->nz);
            for (int r = 0; r < NR; ++r)
              for (int c = 0; c < 3; ++c) acc[r][c] += w * rf[((long)r * 3 + c) * nvf + g];
          }
    for (int r = 0; r < NR; ++r)
      for (int c = 0; c < 3; ++c) bc[((long)r * 3 + c) * nvc + n] = acc[r][c];
  }
}

static void prolong_add(const mglev_t* F, const mglev_t* C, double* xf, const double* ec) {
  const long nvf = F->nv, nvc = C->nv;
#pragma omp parallel for schedule(static)
  for (long n = 1; n < nvf; ++n) {
    const int i = (int)(n / ((long)F->ny * F->nz)), j = (int)((n / F->nz) % F->ny), k = (int)(n % F->nz);
    const int ci[2] = {i >> 1, wrapi((i >> 1) + 1, C->nx)};
    const int cj[2] = {j >> 1, wrapi((j >> 1) + 1, C->ny)};
    const int ck[2] = {k >> 1, wrapi((k >> 1) + 1, C->nz)};
    const int ni = (i & 1) ? 2 : 1, nj = (j & 1) ? 2 : 1, nk = (k & 1) ? 2 : 1;
    const double w = 1.0 / (ni * nj * nk);
    for (int r = 0; r < NR; ++r)
      for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int a = 0; a < ni; ++a)
          for (int b = 0; b < nj; ++b)
            for (int d = 0; d < nk; ++d)
              s += ec[((long)r * 3 + c) * nvc + ((long)ci[a] * C->ny + cj[b]) * C->nz + ck[d]];
        xf[((long)r * 3 + c) * nvf + n] += w * s;
      }
  }
}

/* x += w D^-1 (b - t) */
static void jacobi_update(const mglev_t* L, double* x, const double* b, const double* t, double w) {
  if (L->binv) {
    block_sweep(L, x, b, t, w, 0);
    return;
  }
  const long nv = L->nv;
#pragma omp parallel for schedule(static)
  for (long q = 0; q < 18 * nv; ++q) {
    const long cn = q % (3 * nv);
    x[q] += w * L->dinv[cn] * (b[q] - t[q]);
  }
}

static void vcycle(mg_t* M, int l) {
  mglev_t* L = &M->lv[l];
  const long n18 = 18 * L->nv;
  if (l == M->nlev - 1) {
    coarse_solve(L, L->b, L->x);
    return;
  }
  /* first pre-sweep from x = 0 */
  if (L->binv) {
    block_sweep(L, L->x, L->b, NULL, M->wpre[0], 1);
  } else {
#pragma omp parallel for schedule(static)
    for (long q = 0; q < n18; ++q) L->x[q] = M->wpre[0] * L->dinv[q % (3 * L->nv)] * L->b[q];
  }
  for (int s = 1; s < M->pre; ++s) {
    mg_apply(L, &M->hk, L->x, L->t);
    jacobi_update(L, L->x, L->b, L->t, M->wpre[s]);
  }
  mg_apply(L, &M->hk, L->x, L->t);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n18; ++q) L->t[q] = L->b[q] - L->t[q];
  mglev_t* C = &M->lv[l + 1];
  restrict_fw(L, C, L->t, C->b);
  vcycle(M, l + 1);
  prolong_add(L, C, L->x, C->x);
  for (int s = 0; s < M->post; ++s) {
    mg_apply(L, &M->hk, L->x, L->t);
    jacobi_update(L, L->x, L->b, L->t, M->wpost[s]);
  }
}

static void mg_free(mg_t* M) {
  for (int l = 0; l < M->nlev; ++l) {
    free(M->lv[l].kc);
    free(M->lv[l].dinv);
    free(M->lv[l].binv);
    free(M->lv[l].x);
    free(M->lv[l].b);
    free(M->lv[l].t);
    free(M->lv[l].L);
  }
  M->nlev = 0;
}

static int mg_setup(mg_t* M, int nx, int ny, int nz, double h, const double* coef, int pre, int post,
                    double ratio, int coarse_max, double nu, int block) {
  memset(M, 0, sizeof(*M));
  fo_k0(1.0, nu, 1.0, M->K0);
  hadamard_k(M->K0, &M->hk);
  M->pre = pre < 1 ? 1 : (pre > 16 ? 16 : pre);
  M->post = post < 0 ? 0 : (post > 16 ? 16 : post);
  M->block = block != 0;
  const double lmax = lmax_bound(M->K0, M->block);
  weights(M->pre, lmax, ratio, M->wpre);
  double wp[16];
  weights(M->post, lmax, ratio, wp);
  for (int s = 0; s < M->post; ++s) M->wpost[s] = wp[M->post - 1 - s];
  int dims[3] = {nx, ny, nz};
  for (int l = 0; l < MAXLEV; ++l) {
    mglev_t* L = &M->lv[l];
    L->nx = dims[0];
    L->ny = dims[1];
    L->nz = dims[2];
    L->nv = (long)dims[0] * dims[1] * dims[2];
    L->kc = (double*)malloc(sizeof(double) * L->nv);
    L->dinv = (double*)malloc(sizeof(double) * 3 * L->nv);
    L->binv = M->block ? (double*)malloc(sizeof(double) * 6 * L->nv) : NULL;
    L->x = (double*)calloc(18 * L->nv, sizeof(double));
    L->b = (double*)calloc(18 * L->nv, sizeof(double));
    L->t = (double*)calloc(18 * L->nv, sizeof(double));
    M->nlev = l + 1;
    if (l == 0) {
      for (long e = 0; e < L->nv; ++e) L->kc[e] = coef[e] * h;
    } else {
      const mglev_t* F = &M->lv[l - 1];
#pragma omp parallel for schedule(static)
      for (long e = 0; e < L->nv; ++e) {
        const int i = (int)(e / ((long)L->ny * L->nz)), j = (int)((e / L->nz) % L->ny), k = (int)(e % L->nz);
        double s = 0.0;
        for (int a = 0; a < 8; ++a)
          s += F->kc[((long)(2 * i + ((a >> 2) & 1)) * F->ny + 2 * j + ((a >> 1) & 1)) * F->nz + 2 * k + (a & 1)];
        L->kc[e] = 2.0 * s / 8.0;   /* mean modulus x doubled edge */
      }
    }
    level_diag(L, M->K0);
    if (L->binv) level_block(L, M->K0);
    const int halve = L->nv > coarse_max && dims[0] % 2 == 0 && dims[1] % 2 == 0 && dims[2] % 2 == 0 &&
                      dims[0] >= 4 && dims[1] >= 4 && dims[2] >= 4 && l + 1 < MAXLEV;
    if (!halve) break;
    dims[0] /= 2;
    dims[1] /= 2;
    dims[2] /= 2;
  }
  mglev_t* Lc = &M->lv[M->nlev - 1];
  if (Lc->nv > 4096 || level_coarse(Lc, M->K0) != 0) {
    mg_free(M);
    return -1;
  }
  return 0;
}

/* ----------------------------------------------------------------- PCG --- */
static void dots(const double* a, const double* b, long n3, double out[NR]) {
  for (int r = 0; r < NR; ++r) {
    const double* pa = a + (long)r * n3;
    const double* pb = b + (long)r * n3;
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long q = 0; q < n3; ++q) s += pa[q] * pb[q];
    out[r] = s;
  }
}

/* right-hand sides b^I = -K(c) (eps^I x), element by element: the affine
 * field of a voxel is eps^I (h * corner), so with kc = c h (the K0(1)
 * multiplier) b_n = -h sum_{voxels e at n} kc_e (K0(1) eps^I corner)_a */
static void mg_rhs(const mglev_t* L, const double K0[576], double h, double* b) {
  double ue0[6][24], g[6][24];
  fo_affine(1.0, ue0);
  for (int I = 0; I < 6; ++I)
    for (int p = 0; p < 24; ++p) {
      double acc = 0.0;
      for (int q = 0; q < 24; ++q) acc += K0[p * 24 + q] * ue0[I][q];
      g[I][p] = acc * h;
    }
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long nv = L->nv;
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n) {
    const int i = (int)(n / ((long)ny * nz)), j = (int)((n / nz) % ny), k = (int)(n % nz);
    double acc[6][3];
    memset(acc, 0, sizeof(acc));
    for (int a = 0; a < 8; ++a) {
      const long e = ((long)wrapi(i - ((a >> 2) & 1), nx) * ny + wrapi(j - ((a >> 1) & 1), ny)) * nz +
                     wrapi(k - (a & 1), nz);
      for (int I = 0; I < 6; ++I)
        for (int c = 0; c < 3; ++c) acc[I][c] += L->kc[e] * g[I][3 * a + c];
    }
    for (int I = 0; I < 6; ++I)
      for (int c = 0; c < 3; ++c) b[((long)I * 3 + c) * nv + n] = n == 0 ? 0.0 : -acc[I][c];
  }
}

int fo_mg_homogenize(int nx, int ny, int nz, double h, const double* rho, const fo_material* mat, double tol,
                     int max_iter, int pre, int post, double cheb_ratio, int coarse_max, double C[36],
                     double* chi_out, int iters[6], double rel[6]) {
  return fo_mg_homogenize_b(nx, ny, nz, h, rho, mat, tol, max_iter, pre, post, cheb_ratio, coarse_max, 0, C,
                            chi_out, iters, rel);
}

int fo_mg_homogenize_b(int nx, int ny, int nz, double h, const double* rho, const fo_material* mat, double tol,
                       int max_iter, int pre, int post, double cheb_ratio, int coarse_max, int block, double C[36],
                       double* chi_out, int iters[6], double rel[6]) {
  const long nv = (long)nx * ny * nz;
  const long n3 = 3 * nv, n18 = 18 * nv;
  if (nx < 2 || ny < 2 || nz < 2 || nz > 256) return -2;
  double* coef = (double*)malloc(sizeof(double) * nv);
  for (long e = 0; e < nv; ++e) coef[e] = fo_coef(mat, rho[e]);
  mg_t* M = (mg_t*)malloc(sizeof(mg_t));
  if (mg_setup(M, nx, ny, nz, h, coef, pre, post, cheb_ratio, coarse_max, mat->nu, block) != 0) {
    free(coef);
    free(M);
    return -3;
  }
  mglev_t* L0 = &M->lv[0];
  double* b = (double*)malloc(sizeof(double) * n18);
  double* x = (double*)calloc(n18, sizeof(double));
  double* r = (double*)malloc(sizeof(double) * n18);
  double* p = (double*)malloc(sizeof(double) * n18);
  double* q = (double*)malloc(sizeof(double) * n18);
  mg_rhs(L0, M->K0, h, b);
  memcpy(r, b, sizeof(double) * n18);
  double bn[NR], rr[NR], rz[NR], pq[NR], rzn[NR];
  int active[NR], it_done[NR];
  dots(r, r, n3, bn);
  int status = 0;
  for (int I = 0; I < NR; ++I) {
    active[I] = bn[I] > 0.0;
    it_done[I] = 0;
    rel[I] = 0.0;
  }
  /* z = V(r) -> p */
  memcpy(L0->b, r, sizeof(double) * n18);
  if (M->nlev == 1) coarse_solve(L0, L0->b, L0->x);
  else vcycle(M, 0);
  memcpy(p, L0->x, sizeof(double) * n18);
  dots(r, L0->x, n3, rz);
  for (int it = 1; it <= max_iter; ++it) {
    int any = 0;
    for (int I = 0; I < NR; ++I) any |= active[I];
    if (!any) break;
    mg_apply(L0, &M->hk, p, q);
    dots(p, q, n3, pq);
    double alpha[NR];
    for (int I = 0; I < NR; ++I) {
      if (active[I] && !(pq[I] > 0.0)) {   /* breakdown */
        active[I] = 0;
        status = 2;
      }
      alpha[I] = active[I] ? rz[I] / pq[I] : 0.0;
    }
#pragma omp parallel for schedule(static)
    for (long t = 0; t < n18; ++t) {
      const int I = (int)(t / n3);
      x[t] += alpha[I] * p[t];
      r[t] -= alpha[I] * q[t];
    }
    dots(r, r, n3, rr);
    for (int I = 0; I < NR; ++I) {
      if (!active[I]) continue;
      it_done[I] = it;
      rel[I] = sqrt(rr[I] / bn[I]);
      if (rel[I] < tol) active[I] = 0;
    }
    memcpy(L0->b, r, sizeof(double) * n18);
    if (M->nlev == 1) coarse_solve(L0, L0->b, L0->x);
    else vcycle(M, 0);
    dots(r, L0->x, n3, rzn);
    double beta[NR];
    for (int I = 0; I < NR; ++I) {
      beta[I] = active[I] ? rzn[I] / rz[I] : 0.0;
      if (active[I]) rz[I] = rzn[I];
    }
    const double* z = L0->x;
#pragma omp parallel for schedule(static)
    for (long t = 0; t < n18; ++t) {
      const int I = (int)(t / n3);
      if (active[I]) p[t] = z[t] + beta[I] * p[t];
    }
  }
  for (int I = 0; I < NR; ++I) {
    if (iters) iters[I] = it_done[I];
    if (bn[I] > 0.0 && !(rel[I] < tol) && status == 0) status = 1;
  }
  /* fluctuation in [rhs][node][comp] and C^H by the plain energy reduction */
  double* chi = chi_out ? chi_out : (double*)malloc(sizeof(double) * n18);
#pragma omp parallel for schedule(static)
  for (long n = 0; n < nv; ++n)
    for (int I = 0; I < NR; ++I)
      for (int c = 0; c < 3; ++c) chi[(long)I * n3 + 3 * n + c] = x[((long)I * 3 + c) * nv + n];
  double K0h[576];
  fo_k0(1.0, mat->nu, h, K0h);
  fo_energy(nx, ny, nz, h, K0h, coef, chi, C);
  if (!chi_out) free(chi);
  free(b); free(x); free(r); free(p); free(q); free(coef);
  mg_free(M);
  free(M);
  return status;
}

/* y = K(coef) u through the multigrid file's apply (input/output in the
 * [rhs][node][comp] layout of fo_apply, six load cases), for the tests. */
void fo_mg_apply(int nx, int ny, int nz, double h, const double* coef, double nu, const double* u, double* y) {
  mglev_t L;
  memset(&L, 0, sizeof(L));
  L.nx = nx;
  L.ny = ny;
  L.nz = nz;
  L.nv = (long)nx * ny * nz;
  const long nv = L.nv, n3 = 3 * nv;
  L.kc = (double*)malloc(sizeof(double) * nv);
  for (long e = 0; e < nv; ++e) L.kc[e] = coef[e] * h;
  double K0[576];
  hadk_t H;
  fo_k0(1.0, nu, 1.0, K0);
  hadamard_k(K0, &H);
  double* us = (double*)malloc(sizeof(double) * 18 * nv);
  double* ys = (double*)malloc(sizeof(double) * 18 * nv);
  for (int I = 0; I < NR; ++I)
    for (long n = 0; n < nv; ++n)
      for (int c = 0; c < 3; ++c) us[((long)I * 3 + c) * nv + n] = u[(long)I * n3 + 3 * n + c];
  mg_apply(&L, &H, us, ys);   /* rows of node 0 come back 0 (pinned) */
  for (int I = 0; I < NR; ++I)
    for (long n = 0; n < nv; ++n)
      for (int c = 0; c < 3; ++c) y[(long)I * n3 + 3 * n + c] = ys[((long)I * 3 + c) * nv + n];
  free(us);
  free(ys);
  free(L.kc);
}
