// kernels.cuh -- node-parallel kernels of the femh engine: coefficients, the
// strain-driven right-hand sides, fused CG vector updates with FP64 partial
// sums, per-(cell, load case) scalar finalisation, multigrid transfers, the
// dense FP64 coarse solve, and the FP64 energy reductions (C^H, dC^H/drho,
// dL/drho).
//
// All node-parallel kernels take a NodeUnit table: one CTA per (unit, load
// case), a unit being a contiguous node range of one cell, so that thousands
// of cells of different sizes run in the same launch.
#pragma once
#include "femh_common.cuh"
#include "stencil.cuh"

namespace femh {

// Material law of the per-voxel modulus E(rho) (K0 is built for E = 1).
enum Interp : int { INTERP_SIMP = 0, INTERP_RAMP3 = 1, INTERP_BINARY = 2 };
struct MatLaw {
  int interp;
  int rho_bf16;   // round rho to bf16 before the law (mixed-precision option)
  double E_s, E_min, penal, bin_hi, bin_lo, rho_min, rho_max;
};

__host__ __device__ inline double law_coef(const MatLaw& m, double rho) {
  if (m.interp == INTERP_SIMP) return m.E_min + pow(rho, m.penal) * (m.E_s - m.E_min);
  if (m.interp == INTERP_RAMP3) return m.E_s * rho / (3.0 - 2.0 * rho);
  return rho >= 0.5 ? m.bin_hi : m.bin_lo;
}
__host__ __device__ inline double law_dcoef(const MatLaw& m, double rho) {
  if (m.interp == INTERP_SIMP) return m.penal * pow(rho, m.penal - 1.0) * (m.E_s - m.E_min);
  if (m.interp == INTERP_RAMP3) {
    const double d = 3.0 - 2.0 * rho;
    return m.E_s * 3.0 / (d * d);
  }
  return 0.0;
}

// Constants of the load and energy kernels, for h = 1 (scaled by h inside).
struct ElemConst {
  double g1[kNumRhs][24];      // K0(E=1,h=1) ue0^I(h=1), DOF 3a+c
  double uhat0[kNumRhs][3][8]; // Hadamard transform of ue0^I(h=1)
};

// (i, j, k) of node n of a cell; n < nx*ny*nz < 2^32, so 32-bit unsigned
// division (far cheaper than 64-bit) is exact.
__device__ __forceinline__ void node_ijk(long long n, int ny, int nz, int& i, int& j, int& k) {
  const unsigned nn = (unsigned)n, p = (unsigned)ny * (unsigned)nz;
  const unsigned ii = nn / p, rem = nn - ii * p, jj = rem / (unsigned)nz;
  i = (int)ii;
  j = (int)jj;
  k = (int)(rem - jj * (unsigned)nz);
}
__device__ __forceinline__ long long lin(int i, int j, int k, int ny, int nz) {
  return ((long long)i * ny + j) * nz + k;
}
__device__ __forceinline__ int wrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

// ---------------------------------------------------------------- setup ---
// Fine-level stiffness scale kc[e] = E(clamp(rho_e)) * h and the rho actually used.
// A density that is NaN, infinite or negative is not clamped into range but
// reported: *bad = 1 (the host turns it into FEMH_E_ARG before solving).
template <typename TC2>
__global__ void k_coef(const CellDesc* cells, const NodeUnit* units, const double* rho, MatLaw law,
                       double* kc64, TC2* kc2, double* rho_used, int* bad) {
  const NodeUnit u = units[blockIdx.x];
  const CellDesc cd = cells[u.cell];
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    double r = rho[cd.off + n];
    if (!(r >= 0.0) || isinf(r)) {
      *bad = 1;
      r = 0.0;
    }
    r = fmin(fmax(r, law.rho_min), law.rho_max);
    const double kc = law_coef(law, r) * cd.h;
    if (rho_used) rho_used[cd.off + n] = r;
    if (kc64) kc64[cd.off + n] = kc;
    if (kc2) {
      // the inner (FP32) operator may see rho rounded to bf16; the FP64
      // operator that defines the solution always uses rho as given
      const double rb = law.rho_bf16 ? (double)__bfloat162float(__float2bfloat16_rn((float)r)) : r;
      kc2[cd.off + n] = (TC2)(law.rho_bf16 ? law_coef(law, rb) * cd.h : kc);
    }
  }
}

// Rediscretised coarse scale: the coarse voxel's modulus is the mean of its 8
// children's moduli and its edge is 2h, so kc_c = mean(kc_f / h) * 2h =
// 2 mean(kc_f).  avg: 0 arithmetic mean, 1 geometric, 2 harmonic.
template <typename TF, typename TCo>
__global__ void k_coarsen_coef(const CellDesc* fine, const CellDesc* coarse, const NodeUnit* units,
                               const TF* kcf, TCo* kcc, int avg) {
  const NodeUnit u = units[blockIdx.x];
  const CellDesc cc = coarse[u.cell], cf = fine[cc.parent];
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    int i, j, k;
    node_ijk(n, cc.ny, cc.nz, i, j, k);
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double v = (double)kcf[cf.off + lin(2 * i + ((a >> 2) & 1), 2 * j + ((a >> 1) & 1), 2 * k + (a & 1),
                                                cf.ny, cf.nz)];
      s += (avg == 0) ? v : (avg == 1 ? log(v) : 1.0 / v);
    }
    const double m = (avg == 0) ? s / 8.0 : (avg == 1 ? exp(s / 8.0) : 8.0 / s);
    kcc[cc.off + n] = (TCo)(2.0 * m);
  }
}

// Point-Jacobi inverse diagonal: all 24 diagonal entries of the cube's K0 are
// equal, so diag(K)_n = K0diag * sum_{8 voxels at n} kc_e for all 3 components.
template <typename TC>
__global__ void k_invdiag(const CellDesc* cells, const NodeUnit* units, const TC* kc, double diag,
                          float* invd) {
  const NodeUnit u = units[blockIdx.x];
  const CellDesc cd = cells[u.cell];
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    int i, j, k;
    node_ijk(n, cd.ny, cd.nz, i, j, k);
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a)
      s += (double)kc[cd.off + lin(wrap(i - ((a >> 2) & 1), cd.nx), wrap(j - ((a >> 1) & 1), cd.ny),
                                   wrap(k - (a & 1), cd.nz), cd.ny, cd.nz)];
    invd[cd.off + n] = (n == 0) ? 0.f : (float)(1.0 / (diag * s));
  }
}

// Node-block Jacobi: D_n = the 3x3 diagonal block of K at node n = sum over
// the 8 voxels at n of kc_e K0(1)_aa, a = the node's corner in voxel e.  The
// cube's corner blocks are d I + o S_a, S_a(c1, c2) = sigma_c1 sigma_c2 off the
// diagonal, sigma_c = 1 - 2 bit_c(a) (d = K0 diagonal, o = K0[0][1]), so
// D_n = d (sum kc) I + o T_n with T_n(c1, c2) = sum_e kc_e sigma_c1 sigma_c2.
// binv[6 (cd.off + n) + k] = the symmetric inverse, k = xx, yy, zz, xy, xz, yz
// (FP32; 0 at the pinned node 0).
template <typename TC>
__global__ void k_invblock(const CellDesc* cells, const NodeUnit* units, const TC* kc, double d, double o,
                           float* binv) {
  const NodeUnit u = units[blockIdx.x];
  const CellDesc cd = cells[u.cell];
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    int i, j, k;
    node_ijk(n, cd.ny, cd.nz, i, j, k);
    double sum = 0.0, txy = 0.0, txz = 0.0, tyz = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int ax = (a >> 2) & 1, ay = (a >> 1) & 1, az = a & 1;
      const double ke = (double)kc[cd.off + lin(wrap(i - ax, cd.nx), wrap(j - ay, cd.ny), wrap(k - az, cd.nz), cd.ny,
                                                cd.nz)];
      const double sx = 1.0 - 2.0 * ax, sy = 1.0 - 2.0 * ay, sz = 1.0 - 2.0 * az;
      sum += ke;
      txy += ke * sx * sy;
      txz += ke * sx * sz;
      tyz += ke * sy * sz;
    }
    const double A = d * sum, X = o * txy, Y = o * txz, Z = o * tyz;   // [[A X Y] [X A Z] [Y Z A]]
    const double c00 = A * A - Z * Z, c11 = A * A - Y * Y, c22 = A * A - X * X;
    const double c01 = Y * Z - X * A, c02 = X * Z - Y * A, c12 = X * Y - A * Z;
    const double det = A * c00 + X * c01 + Y * c02;
    const double r = (n == 0) ? 0.0 : 1.0 / det;
    float* out = binv + 6 * (cd.off + n);
    out[0] = (float)(c00 * r);
    out[1] = (float)(c11 * r);
    out[2] = (float)(c22 * r);
    out[3] = (float)(c01 * r);
    out[4] = (float)(c02 * r);
    out[5] = (float)(c12 * r);
  }
}

// Strain-driven load b^I_n = -sum_{e at n} c_e (K0(h) ue0^I(h))[a_n(e)]
//   = -h * sum_e kc_e g1^I[a_n(e)]  (K0(h) = h K0(1), ue0(h) = h ue0(1), kc = c h).
// Pinned node 0 gets 0.  One CTA per (unit, load case).
template <typename TB>
__global__ void k_rhs(const CellDesc* cells, const NodeUnit* units, const double* kc64,
                      const ElemConst* ec, TB* b, long long ntot) {
  const NodeUnit u = units[blockIdx.x];
  const int I = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    int i, j, k;
    node_ijk(n, cd.ny, cd.nz, i, j, k);
    double acc[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double ke = kc64[cd.off + lin(wrap(i - ((a >> 2) & 1), cd.nx), wrap(j - ((a >> 1) & 1), cd.ny),
                                          wrap(k - (a & 1), cd.nz), cd.ny, cd.nz)];
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] += ke * ec->g1[I][3 * a + c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
      st_val(b + ((long long)I * 3 + c) * ntot + cd.off + n, (n == 0) ? 0.0 : -cd.h * acc[c]);
  }
}

// ------------------------------------------------------------- CG pieces ---
// Start of PCG: x = 0 (kept as it is when keep_x: a warm start, with b the
// residual of that x), r = s*b (s = per (cell,rhs) scale), partial ||r||^2.
// With jacobi != 0 also partial r.(invd r) for the Jacobi-preconditioned rz and
// p = invd r.  Partials: [slot][6][2].
template <typename TB, typename TV, typename TP>
__global__ void k_cg_init(const CellDesc* cells, const NodeUnit* units, const TB* __restrict__ b, TV* __restrict__ x, TV* __restrict__ r,
                          TP* __restrict__ p, const float* __restrict__ invd, const CGState* stt, double* __restrict__ part, long long ntot,
                          int jacobi, int keep_x) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  const CGState S = stt[cd.id * kNumRhs + rhs];
  double v[2] = {0.0, 0.0};
  if (S.active) {
    #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
      const long long g = cd.off + n;
      const float id = invd[g];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const long long o = ((long long)rhs * 3 + c) * ntot + g;
        const double rv = (n == 0) ? 0.0 : S.scale * (double)ld_val(b + o);
        if (!keep_x) st_val(x + o, 0.0);
        st_val(r + o, rv);
        v[0] += rv * rv;
        const double z = (double)id * rv;
        v[1] += rv * z;
        if (jacobi) st_val(p + o, z);
      }
    }
  }
  __shared__ double red[64];
  block_reduce<2>(v, red);
  if (threadIdx.x == 0) {
    part[((long long)u.slot * kNumRhs + rhs) * 2 + 0] = v[0];
    part[((long long)u.slot * kNumRhs + rhs) * 2 + 1] = v[1];
  }
}

// x += alpha p ; r -= alpha q (r = 0 at node 0) ; partial ||r||^2 and, for
// Jacobi, r.(invd r).  For the multigrid preconditioner (z0 != nullptr) it
// also writes the first damped-Jacobi sweep from zero: z0 = omega invd r, and,
// when rm != nullptr, r in the V-cycle's storage type (the level-0 right-hand
// side its sweeps read).
template <typename TV, typename TP, typename TQ, typename TZ>
__global__ void k_cg_update(const CellDesc* cells, const NodeUnit* units, TV* __restrict__ x, TV* __restrict__ r, const TP* __restrict__ p,
                            const TQ* __restrict__ q, const float* __restrict__ invd, TZ* __restrict__ z0,
                            TZ* __restrict__ rm, double omega, const CGState* stt,
                            double* __restrict__ part, long long ntot, const float* __restrict__ binv) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  const CGState S = stt[cd.id * kNumRhs + rhs];
  double v[2] = {0.0, 0.0};
  if (S.active) {
    const double al = S.alpha;
    #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
      const long long g = cd.off + n;
      const double id = (double)invd[g];
      double rvs[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const long long o = ((long long)rhs * 3 + c) * ntot + g;
        const double pv = (double)ld_val(p + o);
        const double xv = (double)ld_val(x + o) + al * pv;
        const double rv = (n == 0) ? 0.0 : (double)ld_val(r + o) - al * (double)ld_val(q + o);
        st_val(x + o, xv);
        st_val(r + o, rv);
        v[0] += rv * rv;
        v[1] += rv * id * rv;
        if (z0 && !binv) st_val(z0 + o, omega * id * rv);
        if (rm) st_val(rm + o, rv);
        rvs[c] = rv;
      }
      if (z0 && binv) {   // node-block Jacobi: z0 = omega B r
        jacobi_dir<double>(binv, g, 0.0, rvs);
#pragma unroll
        for (int c = 0; c < 3; ++c) st_val(z0 + ((long long)rhs * 3 + c) * ntot + g, omega * rvs[c]);
      }
    }
  }
  __shared__ double red[64];
  block_reduce<2>(v, red);
  if (threadIdx.x == 0) {
    part[((long long)u.slot * kNumRhs + rhs) * 2 + 0] = v[0];
    part[((long long)u.slot * kNumRhs + rhs) * 2 + 1] = v[1];
  }
}

// p = z + beta p, with z = invd r (Jacobi) or z read from zvec (multigrid).
template <typename TP, typename TZ, typename TR>
__global__ void k_cg_dir(const CellDesc* cells, const NodeUnit* units, TP* __restrict__ p, const TZ* __restrict__ zvec,
                         const TR* __restrict__ r, const float* __restrict__ invd, const CGState* stt, long long ntot) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  const CGState S = stt[cd.id * kNumRhs + rhs];
  if (!S.active) return;
  const double be = S.beta;
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    const long long g = cd.off + n;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long o = ((long long)rhs * 3 + c) * ntot + g;
      const double z = (zvec && !S.fallback) ? (double)ld_val(zvec + o) : (double)invd[g] * (double)ld_val(r + o);
      st_val(p + o, be == 0.0 ? z : z + be * (double)ld_val(p + o));
    }
  }
}

// Sum of the partials of one (cell, rhs) over the cell's slot range: one warp,
// lane-strided then a shuffle tree (fixed order: deterministic).  Valid in all lanes.
__device__ __forceinline__ double sum_slots(const double* part, int b, int e, int rhs, int stride,
                                            int comp) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int t = b + lane; t < e; t += 32) s += part[((long long)t * kNumRhs + rhs) * stride + comp];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// ------------------------------------------------------ block PCG ---
// Block conjugate gradients over the six load cases of a cell (O'Leary,
// Linear Algebra Appl. 29, 1980): they share the operator and the
// preconditioner, so one Krylov space serves all six and the scalar steps
// become 6x6 matrices.  Each new search block is made K-conjugate to the
// previous one explicitly (the flexible form, as in Notay's flexible CG,
// SIAM J. Sci. Comput. 22, 2000), so an FP32 V-cycle that is symmetric only to
// its rounding keeps the directions conjugate:
//   G = P^T K P,  alpha = G^+ (Z^T R),  X += P alpha,  R -= (K P) alpha,
//   Z = M R,      beta = -G^+ ((K P)^T Z),  P = Z + P beta.
// G^+ solves by Cholesky and drops a direction whose pivot falls below `drop`
// of its diagonal (dependent on the earlier ones to the accuracy of the
// preconditioned block: 1e-12 with an FP64 V-cycle, 1e-8 with an FP32 one).
// Load cases that are not live at the start (a zero right-hand side) stay out
// of every product.
struct BlockCG {
  double g[36];       // P^T K P of the current search block, symmetric, row-major
  double zr[36];      // zr[k * 6 + j] = z_k . r_j
  double alpha[36];   // alpha[i * 6 + j]: weight of direction i in load case j
  double beta[36];    // beta[i * 6 + j]: weight of old direction i in new direction j
  double best;        // smallest worst-case relative residual of the block so far
  int since;          // iterations since that last halved
  int mask;           // load cases in the block (bit j)
  int live;           // 1 while the block iterates
};
// A block whose worst relative residual has not halved for this many
// iterations has stalled: its cell is solved again one load case at a time.
constexpr int kBlockStallWindow = 200;

// Index of (i, j), i <= j, in the 21 upper-triangle entries of a 6x6 matrix.
__host__ __device__ constexpr int sym6(int i, int j) { return i * 6 - i * (i - 1) / 2 + (j - i); }

// G X = s B (6x6, row-major) by Cholesky on the columns in mask, a column
// with a pivot below drop times its diagonal dropped (its row of X is 0).
// Returns false if a pivot is below -1e-8 times its diagonal (G indefinite
// beyond rounding), not finite, or no column is kept.
__device__ __noinline__ bool chol_solve6(const double* __restrict__ G, const double* __restrict__ B, double sgn,
                                         double* __restrict__ X, int mask, double drop) {
  double L[6][6];
  int keep = 0;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double gkk = G[k * 6 + k];
    double d = gkk;
#pragma unroll
    for (int j = 0; j < k; ++j)
      if (keep >> j & 1) d -= L[k][j] * L[k][j];
    const bool in = mask >> k & 1;
    if (in && (!isfinite(d) || d < -1e-8 * fabs(gkk))) ok = false;
    const bool use = in && gkk > 0.0 && d > drop * gkk;
    const double lkk = use ? sqrt(d) : 1.0;
    L[k][k] = lkk;
#pragma unroll
    for (int i = k + 1; i < 6; ++i) {
      double v = G[i * 6 + k];
#pragma unroll
      for (int j = 0; j < k; ++j)
        if (keep >> j & 1) v -= L[i][j] * L[k][j];
      L[i][k] = use ? v / lkk : 0.0;
    }
    if (use) keep |= 1 << k;
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double y[6], x[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double v = sgn * B[k * 6 + c];
#pragma unroll
      for (int j = 0; j < k; ++j)
        if (keep >> j & 1) v -= L[k][j] * y[j];
      y[k] = (keep >> k & 1) ? v / L[k][k] : 0.0;
    }
#pragma unroll
    for (int k = 5; k >= 0; --k) {
      double v = y[k];
#pragma unroll
      for (int j = k + 1; j < 6; ++j)
        if (keep >> j & 1) v -= L[j][k] * x[j];
      x[k] = (keep >> k & 1) ? v / L[k][k] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) X[k * 6 + c] = x[k];
  }
  return ok && keep != 0;
}

// The block kernels split each node unit into S sub-ranges, one CTA each (S
// > 1 gives small cells enough CTAs); partial sums go to sub-slot slot*S + s.
struct SubUnit {
  NodeUnit u;
  long long begin, end;
  long long sub;   // partial-sum index
};
__device__ __forceinline__ SubUnit sub_unit(const NodeUnit* units, int S) {
  const int s = (int)(blockIdx.x % (unsigned)S);
  SubUnit r;
  r.u = units[blockIdx.x / (unsigned)S];
  const long long len = r.u.end - r.u.begin;
  r.begin = r.u.begin + len * s / S;
  r.end = r.u.begin + len * (s + 1) / S;
  r.sub = (long long)r.u.slot * S + s;
  return r;
}

// Partials of the 6x6 matrix A^T B of one cell's block per sub-slot: its
// upper triangle (SYM, 21 values) or all 36 entries a_i . b_j (i * 6 + j);
// columns outside the block's mask read as 0.
template <bool SYM, typename TA, typename TB>
__global__ void __launch_bounds__(256, 2)
k_bgram(const CellDesc* cells, const NodeUnit* units, const TA* __restrict__ a, const TB* __restrict__ b,
        const BlockCG* bst, double* __restrict__ part, long long ntot, int nsub) {
  constexpr int NV = SYM ? 21 : 36;
  const SubUnit su = sub_unit(units, nsub);
  const CellDesc cd = cells[su.u.cell];
  const int mask = bst[cd.id].live ? bst[cd.id].mask : 0;
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  if (mask) {
    for (long long n = su.begin + threadIdx.x; n < su.end; n += blockDim.x) {
      const long long g = cd.off + n;
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        double av[6], bv[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const long long o = ((long long)j * 3 + c) * ntot + g;
          const bool in = mask >> j & 1;
          av[j] = in ? (double)ld_val(a + o) : 0.0;
          bv[j] = in ? (double)ld_val(b + o) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
          for (int j = SYM ? i : 0; j < 6; ++j) v[SYM ? sym6(i, j) : i * 6 + j] += av[i] * bv[j];
      }
    }
  }
  __shared__ double red[32 * NV];
  block_reduce<NV>(v, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) part[su.sub * NV + k] = v[k];
}

// Sum of a cell's per-slot partials over its slot range [b, e) by a
// 256-thread CTA in a fixed order (deterministic): thread t adds value
// t % NV of the slots b + t / NV, b + t / NV + G, ... (G = 256 / NV groups,
// coalesced rows), then thread k < NV adds the G group sums of value k.
// out[k] (shared memory) is valid after the call in every thread.
template <int NV>
__device__ __forceinline__ void cta_sum_slots(const double* __restrict__ part, int b, int e, double* red,
                                              double* out) {
  constexpr int G = 256 / NV;
  const int t = threadIdx.x, k = t % NV, grp = t / NV;
  if (grp < G) {
    double acc = 0.0;
    for (int sl = b + grp; sl < e; sl += G) acc += part[(long long)sl * NV + k];
    red[grp * NV + k] = acc;
  }
  __syncthreads();
  if (t < NV) {
    double acc = 0.0;
    for (int g2 = 0; g2 < G; ++g2) acc += red[g2 * NV + t];
    out[t] = acc;
  }
  __syncthreads();
}

// Full 6x6 matrix from 21 upper-triangle values (sym) or 36 row-major ones.
__device__ __forceinline__ void expand6(const double* v, bool sym, double* M) {
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) M[i * 6 + j] = sym ? v[i <= j ? sym6(i, j) : sym6(j, i)] : v[i * 6 + j];
}

// The block stops: its load cases leave the loop with `status`.
__device__ void block_stop(BlockCG& B, CGState* stt, int cell, int status) {
  B.live = 0;
#pragma unroll 1
  for (int j = 0; j < kNumRhs; ++j)
    if (B.mask >> j & 1) {
      CGState& S = stt[cell * kNumRhs + j];
      S.active = 0;
      S.status = status == CG_MAXITER && S.rel < S.tol ? CG_CONVERGED : status;
    }
}

// z_j . r_j of every load case of the block positive: the preconditioner is
// positive on the current residuals.
__device__ __forceinline__ bool zr_positive(const double* Z, int mask) {
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 6; ++j)
    if (mask >> j & 1) ok = ok && Z[j * 7] > 0.0 && isfinite(Z[j * 7]);
  return ok;
}

// After k_fin_init: the block of each cell is its live load cases.
__global__ void k_binit(BlockCG* bst, const CGState* stt, int ncells) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  int mask = 0;
  for (int j = 0; j < kNumRhs; ++j)
    if (stt[cell * kNumRhs + j].active) mask |= 1 << j;
  BlockCG& B = bst[cell];
  B.mask = mask;
  B.live = mask != 0;
  B.best = INFINITY;
  B.since = 0;
  for (int k = 0; k < 36; ++k) B.alpha[k] = B.beta[k] = 0.0;
}

// After the first preconditioner application: Z^T R of the start (beta = 0).
// One 256-thread CTA per cell.
__global__ void __launch_bounds__(256) k_bfin_rz(BlockCG* bst, CGState* stt, const int* sb, const int* se,
                                                 const double* part_zr, int ncells, int nsub) {
  const int cell = blockIdx.x;
  BlockCG& B = bst[cell];
  if (!B.live) return;
  __shared__ double red[256], Z[36];
  cta_sum_slots<36>(part_zr, sb[cell] * nsub, se[cell] * nsub, red, Z);
  if (threadIdx.x != 0) return;
  if (!zr_positive(Z, B.mask)) return block_stop(B, stt, cell, CG_BLOCK_FAIL);
  for (int k = 0; k < 36; ++k) B.zr[k] = Z[k];
}

// G = P^T K P, alpha = G^+ Z^T R.  One 256-thread CTA per cell.
__global__ void __launch_bounds__(256) k_bfin_alpha(BlockCG* bst, CGState* stt, const int* sb, const int* se,
                                                    const double* part_g, int ncells, double drop, int nsub) {
  const int cell = blockIdx.x;
  BlockCG& B = bst[cell];
  if (!B.live) return;
  __shared__ double red[256], g[21], G[36], A[36], ZR[36];
  cta_sum_slots<21>(part_g, sb[cell] * nsub, se[cell] * nsub, red, g);
  if (threadIdx.x < 36) ZR[threadIdx.x] = B.zr[threadIdx.x];
  __syncthreads();
  if (threadIdx.x != 0) return;
  expand6(g, true, G);
  if (!chol_solve6(G, ZR, 1.0, A, B.mask, drop)) return block_stop(B, stt, cell, CG_BLOCK_FAIL);
  for (int k = 0; k < 36; ++k) {
    B.alpha[k] = A[k];
    B.g[k] = G[k];
  }
}

// After the update and the preconditioner: convergence of every load case of
// the block, then beta = -G^+ (K P)^T Z.  One 256-thread CTA per cell; the
// Gram partials come in nsub_g sub-slots per slot, the ||r||^2 ones in nsub.
__global__ void __launch_bounds__(256) k_bfin_beta(BlockCG* bst, CGState* stt, const int* sb, const int* se,
                                                   const double* part_upd, const double* part_zr,
                                                   const double* part_qz, int ncells, double drop, int nsub_g,
                                                   int nsub) {
  const int cell = blockIdx.x;
  BlockCG& B = bst[cell];
  if (!B.live) return;
  const int b = sb[cell] * nsub_g, e = se[cell] * nsub_g;
  __shared__ double red[256], Z[36], Q[36], T[36], G[36], rr[kNumRhs];
  cta_sum_slots<36>(part_zr, b, e, red, Z);
  cta_sum_slots<36>(part_qz, b, e, red, Q);
  cta_sum_slots<kNumRhs>(part_upd, sb[cell] * nsub, se[cell] * nsub, red, rr);
  if (threadIdx.x < 36) G[threadIdx.x] = B.g[threadIdx.x];
  __syncthreads();
  if (threadIdx.x != 0) return;
  bool all = true, spent = false, bad = false;
  double worst = 0.0;
  for (int j = 0; j < kNumRhs; ++j) {
    if (!(B.mask >> j & 1)) continue;
    CGState& S = stt[cell * kNumRhs + j];
    S.rr = rr[j];
    S.iters += 1;
    S.rel = sqrt(S.rr / S.bnorm2);
    all = all && S.rel < S.tol;
    spent = spent || S.iters >= S.max_iter;
    bad = bad || !isfinite(S.rel);
    worst = fmax(worst, S.rel);
  }
  if (all) return block_stop(B, stt, cell, CG_CONVERGED);
  if (bad) return block_stop(B, stt, cell, CG_BREAKDOWN);
  if (spent) return block_stop(B, stt, cell, CG_MAXITER);
  if (worst < 0.5 * B.best) {
    B.best = worst;
    B.since = 0;
  } else if (++B.since >= kBlockStallWindow) {
    return block_stop(B, stt, cell, CG_BLOCK_FAIL);
  }
  if (!zr_positive(Z, B.mask) || !chol_solve6(G, Q, -1.0, T, B.mask, drop))
    return block_stop(B, stt, cell, CG_BLOCK_FAIL);
  for (int k = 0; k < 36; ++k) {
    B.beta[k] = T[k];
    B.zr[k] = Z[k];
  }
}

// X += P alpha, R -= Q alpha (Q = K P) for the load cases of each live block,
// with ||r||^2 partials per load case ([sub-slot][6]) and, for the multigrid, the first
// smoothing sweep z0 = omega D^-1 r and the residual copy rm of the V-cycle.
// 256 threads; a node's new residuals wait in shared memory for the 3x3
// node-block sweep (registers kept for three CTAs per SM: four measured slower).
template <typename TV, typename TP, typename TQ, typename TZ>
__global__ void __launch_bounds__(256, 3)
k_bupdate(const CellDesc* cells, const NodeUnit* units, TV* __restrict__ x, TV* __restrict__ r,
          const TP* __restrict__ p, const TQ* __restrict__ q, const float* __restrict__ invd, TZ* __restrict__ z0,
          TZ* __restrict__ rm, double omega, const BlockCG* bst, double* __restrict__ part, long long ntot,
          const float* __restrict__ binv, int nsub) {
  const SubUnit su = sub_unit(units, nsub);
  const CellDesc cd = cells[su.u.cell];
  const int mask = bst[cd.id].live ? bst[cd.id].mask : 0;
  __shared__ double al[36];
  __shared__ double rs[kNumRhs * 3][256];
  if (threadIdx.x < 36) al[threadIdx.x] = bst[cd.id].alpha[threadIdx.x];
  __syncthreads();
  double v[kNumRhs];
#pragma unroll
  for (int j = 0; j < kNumRhs; ++j) v[j] = 0.0;
  if (mask) {
    for (long long n = su.begin + threadIdx.x; n < su.end; n += blockDim.x) {
      const long long g = cd.off + n;
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        double pv[kNumRhs], qv[kNumRhs];
#pragma unroll
        for (int i = 0; i < kNumRhs; ++i) {
          const long long o = ((long long)i * 3 + c) * ntot + g;
          const bool in = mask >> i & 1;
          pv[i] = in ? (double)ld_val(p + o) : 0.0;
          qv[i] = in ? (double)ld_val(q + o) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < kNumRhs; ++j) {
          if (!(mask >> j & 1)) continue;
          double dx = 0.0, dr = 0.0;
#pragma unroll
          for (int i = 0; i < kNumRhs; ++i) {
            dx += al[i * 6 + j] * pv[i];
            dr += al[i * 6 + j] * qv[i];
          }
          const long long o = ((long long)j * 3 + c) * ntot + g;
          const double rj = (n == 0) ? 0.0 : (double)ld_val(r + o) - dr;
          st_val(x + o, (double)ld_val(x + o) + dx);
          st_val(r + o, rj);
          if (rm) st_val(rm + o, rj);
          v[j] += rj * rj;
          rs[j * 3 + c][threadIdx.x] = rj;
        }
      }
      if (z0) {
        const double id = binv ? 0.0 : (double)invd[g];
#pragma unroll 1
        for (int j = 0; j < kNumRhs; ++j) {
          if (!(mask >> j & 1)) continue;
          double d[3] = {rs[j * 3][threadIdx.x], rs[j * 3 + 1][threadIdx.x], rs[j * 3 + 2][threadIdx.x]};
          jacobi_dir<double>(binv, g, id, d);
#pragma unroll
          for (int c = 0; c < 3; ++c) st_val(z0 + ((long long)j * 3 + c) * ntot + g, omega * d[c]);
        }
      }
    }
  }
  __shared__ double red[32 * kNumRhs];
  block_reduce<kNumRhs>(v, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int j = 0; j < kNumRhs; ++j) part[su.sub * kNumRhs + j] = v[j];
}

// P = Z + P beta for the load cases of each live block (first: P = Z).
template <typename TP, typename TZ>
__global__ void __launch_bounds__(256, 4)
k_bdir(const CellDesc* cells, const NodeUnit* units, TP* __restrict__ p, const TZ* __restrict__ z,
       const BlockCG* bst, long long ntot, int first, int nsub) {
  const SubUnit su = sub_unit(units, nsub);
  const CellDesc cd = cells[su.u.cell];
  const int mask = bst[cd.id].live ? bst[cd.id].mask : 0;
  __shared__ double be[36];
  if (threadIdx.x < 36) be[threadIdx.x] = first ? 0.0 : bst[cd.id].beta[threadIdx.x];
  __syncthreads();
  if (!mask) return;
  const bool rd = !first;
  for (long long n = su.begin + threadIdx.x; n < su.end; n += blockDim.x) {
    const long long g = cd.off + n;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double pv[kNumRhs], zv[kNumRhs];
#pragma unroll
      for (int i = 0; i < kNumRhs; ++i) {
        const long long o = ((long long)i * 3 + c) * ntot + g;
        const bool in = mask >> i & 1;
        pv[i] = (rd && in) ? (double)ld_val(p + o) : 0.0;
        zv[i] = in ? (double)ld_val(z + o) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kNumRhs; ++j) {
        if (!(mask >> j & 1)) continue;
        double pj = zv[j];
#pragma unroll
        for (int i = 0; i < kNumRhs; ++i) pj += be[i * 6 + j] * pv[i];
        st_val(p + ((long long)j * 3 + c) * ntot + g, pj);
      }
    }
  }
}

// One warp per (cell, rhs) in the finalisation kernels.
#define FIN_PROLOGUE                                                         \
  const int t = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5); \
  const bool lead = (threadIdx.x & 31) == 0;                                 \
  if (t >= ncells * kNumRhs) return;                                         \
  const int cell = t / kNumRhs, rhs = t % kNumRhs;                           \
  (void)cell;                                                                \
  (void)rhs;

// After k_cg_init: bnorm2, rz (Jacobi) / rr; decide which (cell, rhs) run.
// One thread per (cell, rhs).
// bn2 != nullptr (warm start): ||b||^2 per (cell, rhs), against which the
// residual of the starting x is measured; else the start is x = 0 and r = b.
__global__ void k_fin_init(CGState* stt, const int* slot_begin, const int* slot_end,
                           const double* part, int ncells, int jacobi, const double* bn2) {
  FIN_PROLOGUE
  CGState S = stt[t];
  if (!S.active) return;
  const double rr = sum_slots(part, slot_begin[cell], slot_end[cell], rhs, 2, 0);
  S.bnorm2 = bn2 ? bn2[t] : rr;
  S.rr = rr;
  S.rz = jacobi ? sum_slots(part, slot_begin[cell], slot_end[cell], rhs, 2, 1) : 0.0;
  S.iters = 0;
  S.rel = (S.bnorm2 > 0.0) ? sqrt(rr / S.bnorm2) : 0.0;
  S.best = S.rel;
  S.since = 0;
  if (!(S.bnorm2 > 0.0) || !(rr > 0.0) || S.rel < S.tol) { S.active = 0; S.status = CG_CONVERGED; }
  if (lead) stt[t] = S;
}

// rz for the multigrid preconditioner at start (z . r of the first V-cycle);
// if that is not positive, the pair starts with the Jacobi preconditioner.
// beta = 0 so that the following direction kernel sets p = z.
// part: z.r partials over slot range [zb, ze) of each cell (node units, or the
// stencil units of the sweep that computed them); part_init: the start
// partials over [slot_begin, slot_end).
__global__ void k_fin_rz(CGState* stt, const int* slot_begin, const int* slot_end,
                         const int* zb, const int* ze, const double* part, const double* part_init, int ncells) {
  FIN_PROLOGUE
  CGState S = stt[t];
  if (!S.active) return;
  const double rz_mg = sum_slots(part, zb[cell], ze[cell], rhs, 1, 0);
  const double rz_jac = sum_slots(part_init, slot_begin[cell], slot_end[cell], rhs, 2, 1);
  S.beta = 0.0;
  if (isfinite(rz_mg) && rz_mg > 0.0) {
    S.rz = rz_mg;
  } else {
    S.fallback = 1;
    S.rz = rz_jac;
  }
  if (lead) stt[t] = S;
}

// alpha = rz / (p . K p); breakdown if p.Kp <= 0 or not finite.
__global__ void k_fin_alpha(CGState* stt, const int* slot_begin, const int* slot_end,
                            const double* part, int ncells) {
  FIN_PROLOGUE
  CGState S = stt[t];
  if (!S.active) return;
  const double pq = sum_slots(part, slot_begin[cell], slot_end[cell], rhs, 1, 0);
  S.pq = pq;
  if (!(pq > 0.0) || !isfinite(pq) || !isfinite(S.rz)) {
    S.alpha = 0.0;
    S.active = 0;
    S.status = CG_BREAKDOWN;
  } else {
    S.alpha = S.rz / pq;
  }
  if (lead) stt[t] = S;
}

// After the update (+ preconditioner): convergence test and beta.
// jacobi: rz_new from the update partials; else from the V-cycle partials.
// part_rz: z.r partials over slot range [zb, ze) of each cell.
__global__ void k_fin_beta(CGState* stt, const int* slot_begin, const int* slot_end,
                           const int* zb, const int* ze, const double* part_upd, const double* part_rz,
                           int ncells, int jacobi) {
  FIN_PROLOGUE
  CGState S = stt[t];
  if (!S.active) return;
  const int b = slot_begin[cell], e = slot_end[cell];
  const double rr = sum_slots(part_upd, b, e, rhs, 2, 0);
  const double rz_jac = sum_slots(part_upd, b, e, rhs, 2, 1);
  const double rz_mg = jacobi ? rz_jac : sum_slots(part_rz, zb[cell], ze[cell], rhs, 1, 0);
  const double rzn = (jacobi || S.fallback) ? rz_jac : rz_mg;
  S.rr = rr;
  S.iters += 1;
  S.rel = sqrt(rr / S.bnorm2);
  if (S.rel < S.tol) {
    S.active = 0;
    S.status = CG_CONVERGED;
  } else if (S.iters >= S.max_iter) {
    S.active = 0;
    S.status = CG_MAXITER;
  } else if (S.outer && (S.rel < 0.5 * S.best ? (S.best = S.rel, S.since = 0, false)
                                               : ++S.since >= kInnerStallWindow)) {
    S.active = 0;   // inner solve at its arithmetic's floor: hand back to the outer step
    S.status = CG_MAXITER;
  } else if (!isfinite(rzn) || !(rzn > 0.0)) {
    if (!jacobi && !S.fallback && isfinite(rz_jac) && rz_jac > 0.0) {
      // the V-cycle is not positive definite for this field: restart the
      // search direction with the (always SPD) Jacobi preconditioner
      S.fallback = 1;
      S.beta = 0.0;
      S.rz = rz_jac;
    } else {
      S.active = 0;
      S.status = CG_BREAKDOWN;
    }
  } else {
    S.beta = rzn / S.rz;
    S.rz = rzn;
  }
  if (lead) stt[t] = S;
}

// ---------------------------------------------------------- multigrid ---
// Full-weighting restriction (transpose of trilinear prolongation):
// bc(I) = sum_{d in {-1,0,1}^3} prod_s (1 - |d_s|/2) rf(2I + d); 0 at node 0.
// xc != nullptr: also the coarse level's first damped-Jacobi sweep from a zero
// guess, xc = omega * invdc * bc (as stored), on the coarse cells that are
// smoothed there (child >= 0; the others are solved directly).
template <typename TF, typename TCo>
__global__ void k_restrict(const CellDesc* fine, const CellDesc* coarse, const NodeUnit* units,
                           const TF* __restrict__ rf, TCo* __restrict__ bc, TCo* __restrict__ xc,
                           const float* __restrict__ invdc, double omega, const CGState* stt, long long ntf,
                           long long ntc, const float* __restrict__ binvc) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cc = coarse[u.cell], cf = fine[cc.parent];
  if (stt && !stt[cc.id * kNumRhs + rhs].active) return;
  const bool smooth = xc != nullptr && cc.child >= 0;
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    int i, j, k;
    node_ijk(n, cc.ny, cc.nz, i, j, k);
    double acc[3] = {0, 0, 0};
    if (n != 0) {
      for (int dx = -1; dx <= 1; ++dx) {
        const int fi = wrap(2 * i + dx, cf.nx);
        const double wx = dx ? 0.5 : 1.0;
        for (int dy = -1; dy <= 1; ++dy) {
          const int fj = wrap(2 * j + dy, cf.ny);
          const double wy = wx * (dy ? 0.5 : 1.0);
#pragma unroll
          for (int dz = -1; dz <= 1; ++dz) {
            const int fk = wrap(2 * k + dz, cf.nz);
            const double w = wy * (dz ? 0.5 : 1.0);
            const long long g = cf.off + lin(fi, fj, fk, cf.ny, cf.nz);
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[c] += w * (double)ld_val(rf + ((long long)rhs * 3 + c) * ntf + g);
          }
        }
      }
    }
    const long long g = cc.off + n;
#pragma unroll
    for (int c = 0; c < 3; ++c) st_val(bc + ((long long)rhs * 3 + c) * ntc + g, acc[c]);
    if (smooth) {
      double bs[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) bs[c] = (double)static_cast<TCo>(acc[c]);   // b as stored
      if (binvc) {
        jacobi_dir<double>(binvc, g, 0.0, bs);
      } else {
        const double id = (double)invdc[g];
#pragma unroll
        for (int c = 0; c < 3; ++c) bs[c] *= id;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) st_val(xc + ((long long)rhs * 3 + c) * ntc + g, omega * bs[c]);
    }
  }
}

// Trilinear prolongation and correction: xf(n) += sum_I w(n,I) ec(I).
// Each thread corrects the two fine nodes 2m and 2m+1 of a z row, which share
// the coarse z nodes m and m+1 (fine 2m = coarse m; fine 2m+1 = mean of m, m+1);
// x and y weights are uniform along the row.  The pinned node 0 keeps 0.
// (All multigrid levels have even fine extents, so pairs never straddle rows.)
template <typename TF, typename TCo>
__global__ void k_prolong_add(const CellDesc* __restrict__ fine, const CellDesc* __restrict__ coarse,
                              const NodeUnit* __restrict__ units, TF* __restrict__ xf,
                              const TCo* __restrict__ ec, const CGState* stt, long long ntf, long long ntc) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cf = fine[u.cell], cc = coarse[fine[u.cell].child];
  if (stt && !stt[cf.id * kNumRhs + rhs].active) return;
  const long long pb = (u.begin + 1) >> 1, pe = (u.end + 1) >> 1;   // node pairs of the unit
  for (long long pr = pb + threadIdx.x; pr < pe; pr += blockDim.x) {
    const long long n = 2 * pr;
    int i, j, k;
    node_ijk(n, cf.ny, cf.nz, i, j, k);   // k even
    const int ci0 = i >> 1, cj0 = j >> 1, m = k >> 1;
    const int ci1 = wrap(ci0 + (i & 1), cc.nx), cj1 = wrap(cj0 + (j & 1), cc.ny);
    const int m1 = wrap(m + 1, cc.nz);
    const double wx = (i & 1) ? 0.5 : 1.0, wy = (j & 1) ? 0.5 : 1.0;
    double a0[3] = {0, 0, 0}, a1[3] = {0, 0, 0};   // at fine k = 2m and 2m+1
#pragma unroll
    for (int ax = 0; ax < 2; ++ax) {
      if (ax == 1 && !(i & 1)) break;
      const int ci = ax ? ci1 : ci0;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay) {
        if (ay == 1 && !(j & 1)) break;
        const int cj = ay ? cj1 : cj0;
        const double w = wx * wy;
        const long long g0 = cc.off + lin(ci, cj, m, cc.ny, cc.nz);
        const long long g1 = cc.off + lin(ci, cj, m1, cc.ny, cc.nz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double e0 = (double)ld_val(ec + ((long long)rhs * 3 + c) * ntc + g0);
          const double e1 = (double)ld_val(ec + ((long long)rhs * 3 + c) * ntc + g1);
          a0[c] += w * e0;
          a1[c] += w * 0.5 * (e0 + e1);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      TF* px = xf + ((long long)rhs * 3 + c) * ntf + cf.off + n;
      if (n != 0) st_val(px, (double)ld_val(px) + a0[c]);
      if (n + 1 < u.end) st_val(px + 1, (double)ld_val(px + 1) + a1[c]);
    }
  }
}

// z = omega * invd * b  (first damped-Jacobi sweep from a zero start); with
// bcopy != nullptr also b converted to TX.
template <typename TB, typename TX>
__global__ void k_jacobi0(const CellDesc* cells, const NodeUnit* units, const TB* __restrict__ b, TX* __restrict__ x,
                          TX* __restrict__ bcopy, const float* __restrict__ invd, double omega, const CGState* stt,
                          long long ntot, const float* __restrict__ binv) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  if (stt && !stt[cd.id * kNumRhs + rhs].active) return;
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x) {
    const long long g = cd.off + n;
    double bv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long o = ((long long)rhs * 3 + c) * ntot + g;
      bv[c] = (double)ld_val(b + o);
      if (bcopy) st_val(bcopy + o, bv[c]);
    }
    if (binv) {
      jacobi_dir<double>(binv, g, 0.0, bv);
    } else {
      const double id = (double)invd[g];
#pragma unroll
      for (int c = 0; c < 3; ++c) bv[c] *= id;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) st_val(x + ((long long)rhs * 3 + c) * ntot + g, omega * bv[c]);
  }
}

// Dense coarse operator of one cell (one CTA per cell), FP64: A = sum_e kc_e K0(1)
// scattered to the periodic DOFs; the 3 DOFs of node 0 are replaced by identity
// rows/columns (pinned).  A is m x m, m = 3 * nodes.
template <typename TC>
__global__ void k_coarse_assemble(const CellDesc* cells, const int* list, const TC* kc,
                                  const double* K0, double* A, const long long* aoff) {
  const CellDesc cd = cells[list[blockIdx.x]];
  const long long nn = (long long)cd.nx * cd.ny * cd.nz;
  const int m = (int)(3 * nn);
  double* M = A + aoff[blockIdx.x];
  for (long long t = threadIdx.x; t < (long long)m * m; t += blockDim.x) M[t] = 0.0;
  __syncthreads();
  for (long long e = 0; e < nn; ++e) {
    int i, j, k;
    node_ijk(e, cd.ny, cd.nz, i, j, k);
    const double ke = (double)kc[cd.off + e];
    for (int t = threadIdx.x; t < 576; t += blockDim.x) {
      const int p = t / 24, q = t % 24;
      const int ap = p / 3, cp = p % 3, aq = q / 3, cq = q % 3;
      const long long np = lin(wrap(i + ((ap >> 2) & 1), cd.nx), wrap(j + ((ap >> 1) & 1), cd.ny),
                               wrap(k + (ap & 1), cd.nz), cd.ny, cd.nz);
      const long long nq = lin(wrap(i + ((aq >> 2) & 1), cd.nx), wrap(j + ((aq >> 1) & 1), cd.ny),
                               wrap(k + (aq & 1), cd.nz), cd.ny, cd.nz);
      M[(3 * np + cp) * m + 3 * nq + cq] += ke * K0[t];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < m; t += blockDim.x)
    for (int c = 0; c < 3; ++c) {
      M[(long long)c * m + t] = (t == c) ? 1.0 : 0.0;
      M[(long long)t * m + c] = (t == c) ? 1.0 : 0.0;
    }
}

// In-place Cholesky A = L L^T, then A <- A^{-1} (explicit SPD inverse, FP64),
// one CTA per cell.  work holds m*m doubles per cell.  status[cell] = 0 ok,
// k+1 if pivot k was not positive.
__global__ void k_coarse_factor(const CellDesc* cells, const int* list, double* A, double* work,
                                const long long* aoff, int* status) {
  const CellDesc cd = cells[list[blockIdx.x]];
  const int m = 3 * cd.nx * cd.ny * cd.nz;
  double* L = A + aoff[blockIdx.x];
  double* X = work + aoff[blockIdx.x];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int k = 0; k < m; ++k) {
    if (threadIdx.x == 0) {
      const double d = L[(long long)k * m + k];
      if (!(d > 0.0) && !bad) bad = k + 1;
      L[(long long)k * m + k] = sqrt(fmax(d, 1e-300));
    }
    __syncthreads();
    const double dk = L[(long long)k * m + k];
    for (int i = k + 1 + threadIdx.x; i < m; i += blockDim.x) L[(long long)i * m + k] /= dk;
    __syncthreads();
    for (long long t = threadIdx.x; t < (long long)(m - k - 1) * (m - k - 1); t += blockDim.x) {
      const int i = k + 1 + (int)(t / (m - k - 1)), j = k + 1 + (int)(t % (m - k - 1));
      if (j <= i) L[(long long)i * m + j] -= L[(long long)i * m + k] * L[(long long)j * m + k];
    }
    __syncthreads();
  }
  // X = A^{-1}: solve L L^T X = I column by column (threads over columns)
  for (int col = threadIdx.x; col < m; col += blockDim.x) {
    for (int i = 0; i < m; ++i) {   // forward: L y = e_col
      double s = (i == col) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) s -= L[(long long)i * m + j] * X[(long long)j * m + col];
      X[(long long)i * m + col] = s / L[(long long)i * m + i];
    }
    for (int i = m - 1; i >= 0; --i) {   // backward: L^T x = y
      double s = X[(long long)i * m + col];
      for (int j = i + 1; j < m; ++j) s -= L[(long long)j * m + i] * X[(long long)j * m + col];
      X[(long long)i * m + col] = s / L[(long long)i * m + i];
    }
  }
  __syncthreads();
  for (long long t = threadIdx.x; t < (long long)m * m; t += blockDim.x) L[t] = X[t];
  if (threadIdx.x == 0) status[blockIdx.x] = bad;
}

// The same factorisation and inverse for coarse systems of m <= kCoarseSmemM
// unknowns (3 x 64 nodes): the lower triangle of A packed in shared memory
// (row i at i(i+1)/2), right-looking Cholesky in place (one warp per trailing
// row, lanes over its columns), then A^{-1} column by column, one warp per
// column: forward L y = e_c from row c on (y = 0 above), backward L^T x = y,
// each row's dot product split over the lanes.  Written over A.
constexpr int kCoarseSmemM = 192;
inline size_t coarse_factor_smem_bytes(int m) {
  return sizeof(double) * ((size_t)m * (m + 1) / 2 + 32 * (size_t)m);
}
__global__ void __launch_bounds__(1024) k_coarse_factor_smem(const CellDesc* cells, const int* list, double* A,
                                                             const long long* aoff, int* status) {
  extern __shared__ double csm[];
  const CellDesc cd = cells[list[blockIdx.x]];
  const int m = 3 * cd.nx * cd.ny * cd.nz;
  double* Ag = A + aoff[blockIdx.x];
  double* Lp = csm;                               // packed lower triangle
  double* Yw = csm + (size_t)m * (m + 1) / 2;     // [32 warps][m] column buffers
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  auto P = [](int i, int j) { return i * (i + 1) / 2 + j; };   // j <= i
  __shared__ int bad;
  if (tid == 0) bad = 0;
  for (int i = warp; i < m; i += nw)
    for (int j = lane; j <= i; j += 32) Lp[P(i, j)] = Ag[(long long)i * m + j];
  __syncthreads();
  for (int k = 0; k < m; ++k) {
    if (tid == 0) {
      const double d = Lp[P(k, k)];
      if (!(d > 0.0) && !bad) bad = k + 1;
      Lp[P(k, k)] = sqrt(fmax(d, 1e-300));
    }
    __syncthreads();
    const double dk = Lp[P(k, k)];
    for (int i = k + 1 + tid; i < m; i += nt) Lp[P(i, k)] /= dk;
    __syncthreads();
    for (int i = k + 1 + warp; i < m; i += nw) {
      const double lik = Lp[P(i, k)];
      for (int j = k + 1 + lane; j <= i; j += 32) Lp[P(i, j)] -= lik * Lp[P(j, k)];
    }
    __syncthreads();
  }
  double* y = Yw + (size_t)warp * m;
  for (int c = warp; c < m; c += nw) {
    for (int i = lane; i < c; i += 32) y[i] = 0.0;
    __syncwarp();
    for (int i = c; i < m; ++i) {   // forward: L y = e_c
      double sacc = 0.0;
      for (int j = c + lane; j < i; j += 32) sacc += Lp[P(i, j)] * y[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
      if (lane == 0) y[i] = ((i == c ? 1.0 : 0.0) - sacc) / Lp[P(i, i)];
      __syncwarp();
    }
    for (int i = m - 1; i >= 0; --i) {   // backward: L^T x = y
      double sacc = 0.0;
      for (int j = i + 1 + lane; j < m; j += 32) sacc += Lp[P(j, i)] * y[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
      if (lane == 0) y[i] = (y[i] - sacc) / Lp[P(i, i)];
      __syncwarp();
    }
    for (int i = lane; i < m; i += 32) Ag[(long long)i * m + c] = y[i];
    __syncwarp();
  }
  __syncthreads();
  if (tid == 0) status[blockIdx.x] = bad;
}

// Coarse solve e = A^{-1} b for one (cell, rhs) per CTA (A^{-1} symmetric).
template <typename TB, typename TX>
__global__ void k_coarse_solve(const CellDesc* cells, const int* list, const double* Ainv,
                               const long long* aoff, const TB* b, TX* x, const CGState* stt,
                               long long ntot) {
  const int cell = list[blockIdx.x], rhs = blockIdx.y;
  const CellDesc cd = cells[cell];
  if (stt && !stt[cd.id * kNumRhs + rhs].active) return;
  const int nn = cd.nx * cd.ny * cd.nz, m = 3 * nn;
  extern __shared__ double sb[];
  for (int t = threadIdx.x; t < m; t += blockDim.x) {
    const int n = t / 3, c = t % 3;
    sb[t] = (double)ld_val(b + ((long long)rhs * 3 + c) * ntot + cd.off + n);
  }
  __syncthreads();
  const double* M = Ainv + aoff[blockIdx.x];
  // one warp per row t (A^{-1} is symmetric: row t is read contiguously), the
  // row's dot product split over the lanes and summed by shuffles
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = warp; t < m; t += nw) {
    const double* Mr = M + (long long)t * m;
    double s = 0.0;
    for (int j = lane; j < m; j += 32) s += Mr[j] * sb[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      const int n = t / 3, c = t % 3;
      st_val(x + ((long long)rhs * 3 + c) * ntot + cd.off + n, (n == 0) ? 0.0 : s);
    }
  }
}

// ------------------------------------------------------- energy kernels ---
// Per voxel: u^I = ue0^I(h) + chi^I (6 load cases), uhat = T u, w = Kh uhat;
// s_IJ = uhat^I . w^J = u^I . K0(1) u^J.  Modes:
//   C partials:   sum_e kc_e s_IJ       (-> C^H = sum / (|Y|))     [slot][21]
//   dC/drho:      out[t][e] = c'(rho_e) h s_t / |Y|
//   dL/drho:      out[e] = c'(rho_e) h sum_t W_t s_t / |Y|
enum EnergyMode : int { EN_C = 0, EN_DCDRHO = 1, EN_GRAD = 2 };
struct EnergyArgs {
  const CellDesc* cells;
  const NodeUnit* units;
  const double* chi;      // [6][3][ntot] FP64
  const double* kc64;     // c_e * h
  const double* rho;      // rho actually used (clamped)
  const ElemConst* ec;
  const double* W;        // [cell][21] symmetric weights for EN_GRAD
  double* part;           // EN_C: [slot][21]
  double* out;            // EN_DCDRHO: [21][ntot]; EN_GRAD: [ntot]
  long long ntot;
  HadK k;
  MatLaw law;
};

template <int MODE>
__global__ void __launch_bounds__(128) k_energy(EnergyArgs a) {
  const NodeUnit u = a.units[blockIdx.x];
  const CellDesc cd = a.cells[u.cell];
  const double vol = (double)cd.nx * cd.ny * cd.nz * cd.h * cd.h * cd.h;
  double acc[22];
#pragma unroll
  for (int t = 0; t < 22; ++t) acc[t] = 0.0;
  for (long long e = u.begin + threadIdx.x; e < u.end; e += blockDim.x) {
    int i, j, k;
    node_ijk(e, cd.ny, cd.nz, i, j, k);
    long long nd[8];
#pragma unroll
    for (int a8 = 0; a8 < 8; ++a8)
      nd[a8] = cd.off + lin(wrap(i + ((a8 >> 2) & 1), cd.nx), wrap(j + ((a8 >> 1) & 1), cd.ny),
                            wrap(k + (a8 & 1), cd.nz), cd.ny, cd.nz);
    double uh[kNumRhs][3][8];
#pragma unroll
    for (int I = 0; I < kNumRhs; ++I)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int a8 = 0; a8 < 8; ++a8) uh[I][c][a8] = a.chi[((long long)I * 3 + c) * a.ntot + nd[a8]];
        fwht8_fwd(uh[I][c]);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) uh[I][c][kk] += cd.h * a.ec->uhat0[I][c][kk];
      }
    double s[21];
#pragma unroll
    for (int J = 0; J < kNumRhs; ++J) {
      double w[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) w[c][kk] = uh[J][c][kk];
      had_block(w, a.k, 1.0);
#pragma unroll
      for (int I = J; I < kNumRhs; ++I) {
        double d = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int kk = 1; kk < 8; ++kk) d += uh[I][c][kk] * w[c][kk];
        s[I * (I + 1) / 2 + J] = d;   // u^I.K0 u^J = (T u^I).Kh (T u^J)
      }
    }
    if (MODE == EN_C) {
      const double ke = a.kc64[cd.off + e];
#pragma unroll
      for (int t = 0; t < 21; ++t) acc[t] += ke * s[t];
      acc[21] += a.rho[cd.off + e];
    } else {
      const double dc = law_dcoef(a.law, a.rho[cd.off + e]) * cd.h / vol;
      if (MODE == EN_DCDRHO) {
#pragma unroll
        for (int t = 0; t < 21; ++t) a.out[(long long)t * a.ntot + cd.off + e] = dc * s[t];
      } else {
        double g = 0.0;
#pragma unroll
        for (int t = 0; t < 21; ++t) g += a.W[cd.id * 21 + t] * s[t];
        a.out[cd.off + e] = dc * g;
      }
    }
  }
  if (MODE == EN_C) {
    __shared__ double red[32 * 22];
    block_reduce<22>(acc, red);
    if (threadIdx.x == 0)
#pragma unroll
      for (int t = 0; t < 22; ++t) a.part[(long long)u.slot * 22 + t] = acc[t];
  }
}

// C^H of each cell from its energy partials (fixed order), one thread per (cell, pair).
__global__ void k_energy_fin(const CellDesc* cells, const int* slot_begin, const int* slot_end,
                             const double* part, double* C, double* dens, int ncells) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncells * 22) return;
  const int cell = t / 22, q = t % 22;
  const CellDesc cd = cells[cell];
  const double nvx = (double)cd.nx * cd.ny * cd.nz;
  const double vol = nvx * cd.h * cd.h * cd.h;
  double s = 0.0;
  for (int sl = slot_begin[cell]; sl < slot_end[cell]; ++sl) s += part[(long long)sl * 22 + q];
  if (q == 21) {
    dens[cell] = s / nvx;
    return;
  }
  int I = 0;
  while ((I + 1) * (I + 2) / 2 <= q) ++I;
  const int J = q - I * (I + 1) / 2;
  C[cell * 36 + I * 6 + J] = s / vol;
  C[cell * 36 + J * 6 + I] = s / vol;
}

// ------------------------------------------------------- misc vector ops ---
// dst = src (cast), per load case, over all nodes of the units.
template <typename TD, typename TS>
__global__ void k_copy(const CellDesc* cells, const NodeUnit* units, TD* __restrict__ dst, const TS* __restrict__ src,
                       const CGState* stt, long long ntot) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  if (stt && !stt[cd.id * kNumRhs + rhs].active) return;
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long o = ((long long)rhs * 3 + c) * ntot + cd.off + n;
      st_val(dst + o, (double)ld_val(src + o));
    }
}

// Defect correction: x64 += d / scale (d from the inner solve).
template <typename TD>
__global__ void k_dc_accum(const CellDesc* cells, const NodeUnit* units, double* __restrict__ x64, const TD* __restrict__ d,
                           const CGState* stt, long long ntot) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  const CGState S = stt[cd.id * kNumRhs + rhs];
  if (!S.outer) return;
  const double inv = 1.0 / S.scale;
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long o = ((long long)rhs * 3 + c) * ntot + cd.off + n;
      x64[o] += inv * (double)ld_val(d + o);
    }
}


// Partial a.b per (unit, rhs) into part[slot][6] (stride 1).
template <typename TA, typename TB2>
__global__ void k_dot(const CellDesc* cells, const NodeUnit* units, const TA* __restrict__ a, const TB2* __restrict__ b,
                      const CGState* stt, double* __restrict__ part, long long ntot) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  double acc[1] = {0.0};
  if (!stt || stt[cd.id * kNumRhs + rhs].active) {
    #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const long long o = ((long long)rhs * 3 + c) * ntot + cd.off + n;
        acc[0] += (double)ld_val(a + o) * (double)ld_val(b + o);
      }
  }
  __shared__ double red[32];
  block_reduce<1>(acc, red);
  if (threadIdx.x == 0) part[(long long)u.slot * kNumRhs + rhs] = acc[0];
}

// Partial ||v||^2 per (unit, rhs) into part[slot][6] (stride 1).
template <typename TV>
__global__ void k_norm2(const CellDesc* cells, const NodeUnit* units, const TV* __restrict__ v, double* __restrict__ part,
                        long long ntot) {
  const NodeUnit u = units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = cells[u.cell];
  double acc[1] = {0.0};
  #pragma unroll 4
  for (long long n = u.begin + threadIdx.x; n < u.end; n += blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double x = (double)ld_val(v + ((long long)rhs * 3 + c) * ntot + cd.off + n);
      acc[0] += x * x;
    }
  __shared__ double red[32];
  block_reduce<1>(acc, red);
  if (threadIdx.x == 0) part[(long long)u.slot * kNumRhs + rhs] = acc[0];
}

// Condition of the CUDA-graph WHILE node around the captured CG iterations
// (one CTA): another pass of `chunk` iterations while some listed cell still
// iterates, the iteration budget `limit` is not spent, and -- for a batch --
// more than half of the `listed` cells still iterate (otherwise the host
// compacts the unit lists to the live cells and relaunches).  loop[0] counts
// the iterations run in this solve, so the loop always ends.
__global__ void k_while_cond(cudaGraphConditionalHandle h, const CGState* __restrict__ stt, int ncells,
                             int listed, int* loop, int chunk, int limit) {
  __shared__ int alive;
  if (threadIdx.x == 0) alive = 0;
  __syncthreads();
  int mine = 0;
  for (int c = threadIdx.x; c < ncells; c += blockDim.x) {
    bool a = false;
#pragma unroll
    for (int r = 0; r < kNumRhs; ++r) a = a || stt[c * kNumRhs + r].active != 0;
    mine += a ? 1 : 0;
  }
  if (mine) atomicAdd(&alive, mine);   // integer count: exact in any order
  __syncthreads();
  if (threadIdx.x == 0) {
    const int done = loop[0] + chunk;
    loop[0] = done;
    const bool more = alive > 0 && done <= limit && !(ncells > 1 && 2 * alive <= listed);
    cudaGraphSetConditional(h, more ? 1u : 0u);
  }
}

// Field chain rule of fast_fem FEM3DFun::df (fast_fem/FEM3DFun.cpp:252-266)
// for piecewise-constant fields: every voxel belongs to one field parameter
// with weight 1, so grad[p] = sum over the voxels of p of (dL/drho_e + c).
// One warp per parameter, its voxels in a fixed order (CSR built on the host):
// deterministic, no atomics.
__global__ void k_param_sum(const int* __restrict__ ptr, const int* __restrict__ vox,
                            const double* __restrict__ dLdrho, double c, double* __restrict__ out, int nparam) {
  const int p = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= nparam) return;
  double s = 0.0;
  for (int q = ptr[p] + lane; q < ptr[p + 1]; q += 32) s += dLdrho[vox[q]] + c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[p] = s;
}


__global__ void k_sum_slots(const int* slot_begin, const int* slot_end, const double* part, double* out,
                            int ncells) {
  FIN_PROLOGUE
  const double v = sum_slots(part, slot_begin[cell], slot_end[cell], rhs, 1, 0);
  if (lead) out[t] = v;
}

// Full-cell displacement on (nx+1)(ny+1)(nz+1) nodes for load case I: periodic
// chi plus the macro-strain affine field, the jump eps (X - X0) on the + faces
// included (fast_fem/FEM3DFun.cpp:31-56 copyPeriodicU).  Layout [node][3].
__global__ void k_full_field(const CellDesc* cells, int cell, const double* chi, int I, double* out,
                             long long ntot) {
  const CellDesc cd = cells[cell];
  const int Nx = cd.nx + 1, Ny = cd.ny + 1, Nz = cd.nz + 1;
  const long long total = (long long)Nx * Ny * Nz;
  double eps[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (I < 3) eps[I][I] = 1.0;
  if (I == 3) eps[1][2] = eps[2][1] = 0.5;
  if (I == 4) eps[0][2] = eps[2][0] = 0.5;
  if (I == 5) eps[0][1] = eps[1][0] = 0.5;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(t, Ny, Nz, i, j, k);
    const long long n0 = cd.off + lin(i % cd.nx, j % cd.ny, k % cd.nz, cd.ny, cd.nz);
    const double X[3] = {i * cd.h, j * cd.h, k * cd.h};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double aff = eps[c][0] * X[0] + eps[c][1] * X[1] + eps[c][2] * X[2];
      out[3 * t + c] = chi[((long long)I * 3 + c) * ntot + n0] + aff;
    }
  }
}

}  // namespace femh

namespace femh {
// [6][3][node] (engine) <-> [6][node][3] (reference layout) for one cell.
template <bool TO_AOS>
__global__ void k_layout(const double* src, double* dst, long long off, long long nn, long long ntot) {
  const long long total = nn * 18;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int I = (int)(t / (3 * nn));
    const long long rem = t - (long long)I * 3 * nn;
    const long long n = rem / 3;
    const int c = (int)(rem - n * 3);
    const long long eng = ((long long)I * 3 + c) * ntot + off + n;   // engine index
    const long long ref = t;                                          // [I][n][c] of this cell
    if (TO_AOS) dst[ref] = src[eng];
    else dst[eng] = src[ref];
  }
}
}  // namespace femh
