// stencil.cuh -- matrix-free periodic operator y = K(c) u for one right-hand
// side per CTA, and its fused epilogues (CG apply+dot, damped-Jacobi sweep,
// residual).
//
// Operator (restates the reference's assembled periodic stiffness,
// SamplesGenerator/NumericalCoarsening.cpp:1238-1306 and the topoOptLib
// ElasticHexFEM it replaces): K(c) = sum_e c_e P_e^T K0 P_e over the voxels of
// a periodic grid.  Row n of K is the node-centric 27-neighbour 3x3-block
// stencil sum_d A_{n,n+d} u_{n+d}, A_{n,n+d} = sum_{e contains n, n+d} c_e
// K0[a_n(e), a_{n+d}(e)].  The kernel evaluates exactly that sum, factored per
// voxel: K0 u_e = T^T (Kh (T u_e)) where T is the +-1 Hadamard transform of the
// 2x2x2 node cube (3 butterfly stages per component) and Kh has 45 nonzeros in
// 8 distinct values (HadK).  This costs ~170 flops per voxel and RHS instead of
// 1152 for a dense 24x24 product, and every output node is written by exactly
// one thread (no atomics, deterministic).
//
// Work decomposition: a CTA owns `rows` node rows (y) x `len` node planes (x)
// of one cell and the whole z ring.  Thread (r, z) streams voxel (i, j0-1+r, z)
// along x: per x step it loads one node of the next plane, exchanges node
// values through a shared plane buffer P, transforms its voxel, keeps the
// upper-plane contributions in registers (carry) and publishes the
// lower-plane ones through Q, from which the owner of each node gathers its 4
// in-plane voxels.  Thread row 0 computes the y-halo voxel row only.
#pragma once
#include "femh_common.cuh"

namespace femh {

enum OutMode : int {
  OUT_APPLY = 0,       // out = K u
  OUT_APPLY_DOT = 1,   // out = K u, partial u . K u
  OUT_JACOBI = 2,      // out = u + omega * invd * (b - K u)
  OUT_JACOBI_DOT = 3,  // same, partial out . b
  OUT_RESID = 4,       // out = b - K u (pinned node 0 of each cell set to 0)
};

template <typename TIn, typename TOut, typename TB, typename TC>
struct StencilArgs {
  const CellDesc* cells;
  const StencilUnit* units;
  const TIn* u;
  TOut* out;
  const TB* b;
  const TC* kc;          // per voxel c_e * h (level scale folded in)
  const float* invd;     // per node inverse diagonal (0 at the pinned node)
  double* partials;      // [slot][6]
  const CGState* stt;    // per (cell, rhs) state (skip inactive) or nullptr
  long long ntot;        // nodes of the level over all cells
  HadK k;
  double omega;
};

template <typename T>
__device__ __forceinline__ void fwht8_fwd(T (&v)[8]) {
#pragma unroll
  for (int b = 1; b < 8; b <<= 1)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (!(a & b)) {
        const T lo = v[a], hi = v[a | b];
        v[a] = hi + lo;
        v[a | b] = hi - lo;
      }
}

template <typename T>
__device__ __forceinline__ void fwht8_inv(T (&v)[8]) {
#pragma unroll
  for (int b = 4; b > 0; b >>= 1)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (!(a & b)) {
        const T k0 = v[a], k1 = v[a | b];
        v[a] = k0 - k1;
        v[a | b] = k0 + k1;
      }
}

// In-place Hadamard-domain element operator, scaled by s = c_e * h.
// w[c][k] for k = 1..7 on input (w[c][0] ignored), output overwrites w.
template <typename T>
__device__ __forceinline__ void had_block(T (&w)[3][8], const HadK& K, T s) {
  const T A = s * (T)K.A, Bdo = s * (T)(K.Bd - K.Bo), Bo = s * (T)K.Bo;
  const T D1o = s * (T)(K.D1 - K.O1), O1 = s * (T)K.O1;
  const T D2o = s * (T)(K.D2 - K.O2), O2 = s * (T)K.O2, G = s * (T)K.G;
  // normal triple (4,x),(2,y),(1,z)
  {
    const T n0 = w[0][4], n1 = w[1][2], n2 = w[2][1];
    const T t = Bo * (n0 + n1 + n2);
    w[0][4] = Bdo * n0 + t;
    w[1][2] = Bdo * n1 + t;
    w[2][1] = Bdo * n2 + t;
  }
  // shear pairs
  {
    const T sxz = A * (w[0][1] + w[2][4]);
    const T syz = A * (w[1][1] + w[2][2]);
    const T sxy = A * (w[0][2] + w[1][4]);
    w[0][1] = sxz; w[2][4] = sxz;
    w[1][1] = syz; w[2][2] = syz;
    w[0][2] = sxy; w[1][4] = sxy;
  }
  // mixed triple (3,x),(5,y),(6,z)
  {
    const T t0 = w[0][3], t1 = w[1][5], t2 = w[2][6];
    const T t = O1 * (t0 + t1 + t2);
    w[0][3] = D1o * t0 + t;
    w[1][5] = D1o * t1 + t;
    w[2][6] = D1o * t2 + t;
  }
  // mixed pairs
  {
    const T a = w[1][3], b = w[0][5], t = O2 * (a + b);
    w[1][3] = D2o * a + t; w[0][5] = D2o * b + t;
  }
  {
    const T a = w[2][3], b = w[0][6], t = O2 * (a + b);
    w[2][3] = D2o * a + t; w[0][6] = D2o * b + t;
  }
  {
    const T a = w[2][5], b = w[1][6], t = O2 * (a + b);
    w[2][5] = D2o * a + t; w[1][6] = D2o * b + t;
  }
  w[0][7] *= G; w[1][7] *= G; w[2][7] *= G;
  w[0][0] = (T)0; w[1][0] = (T)0; w[2][0] = (T)0;
}

// NZ > 0: the cell's z extent is a compile-time constant (all index math
// folds into immediates); NZ == 0: runtime nz.
//
// One barrier per x step: P (node plane) and Q (in-plane corner totals) are
// double-buffered; at step s a thread publishes node plane ie+1 into P[s&1],
// transforms voxel ie into Q[s&1], and gathers node plane ie-1 from
// Q[(s-1)&1], which the previous step completed before this step's barrier.
template <typename T, int NT, int OUT, int NZ, typename TIn, typename TOut, typename TB, typename TC>
__global__ void __launch_bounds__(NT, 1)
stencil_kernel(StencilArgs<TIn, TOut, TB, TC> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const StencilUnit un = a.units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = a.cells[un.cell];
  if (a.stt && !a.stt[cd.id * kNumRhs + rhs].active) return;
  const int nx = cd.nx, ny = cd.ny;
  const int nz = NZ > 0 ? NZ : cd.nz;
  const int R = NT / nz;                 // thread rows (row 0 = y halo)
  const int tid = threadIdx.x;
  const int r = tid / nz, z = tid - r * nz;
  const bool live = r < R && r <= un.rows;   // rows beyond the tile idle
  const int zp = (z + 1 == nz) ? 0 : z + 1;
  const int zm = (z == 0) ? nz - 1 : z - 1;
  int jr = un.j0 - 1 + r;                     // voxel row / lower node row
  if (jr < 0) jr += ny;
  while (jr >= ny) jr -= ny;
  const int jr1 = (jr + 1 == ny) ? 0 : jr + 1;
  const bool extra = live && r == un.rows;    // also loads row jr+1
  const bool owner = live && r >= 1;

  const size_t PS = (size_t)(R + 1) * 3 * nz;   // one P buffer
  const size_t QS = (size_t)R * 12 * nz;        // one Q buffer
  T* P = reinterpret_cast<T*>(smem_raw);        // [2][(R+1)][3][nz]
  T* Q = P + 2 * PS;                            // [2][R][12][nz]
  double* red = reinterpret_cast<double*>(smem_raw + ((sizeof(T) * (2 * PS + 2 * QS) + 15) & ~(size_t)15));
  const size_t prow = (size_t)r * 3 * nz, qrow = (size_t)r * 12 * nz;
  const size_t qup = (size_t)(r > 0 ? r - 1 : 0) * 12 * nz;

  const long long st = a.ntot;
  const long long plane = (long long)ny * nz;
  const long long cellsz = (long long)nx * plane;
  const TIn* ub = a.u + (long long)rhs * 3 * st + cd.off;
  const long long col0 = (long long)jr * nz + z, col1 = (long long)jr1 * nz + z;
  const TC* kcb = a.kc + cd.off + col0;
  const TB* bb = (OUT >= OUT_JACOBI) ? a.b + (long long)rhs * 3 * st + cd.off + col0 : nullptr;
  const float* ib = a.invd + cd.off + col0;
  TOut* obase = a.out + (long long)rhs * 3 * st + cd.off + col0;

  T ld0[3] = {0, 0, 0}, ld1[3] = {0, 0, 0};
  T kcv = 0, kc_next = 0;
  T eb[3] = {0, 0, 0};
  T eid = 0;
  T prev[3][4], carry[3][4];
  T own[3] = {0, 0, 0}, unode[3] = {0, 0, 0};   // of the node plane gathered next
  long long pg = 0;                              // offset of that node plane
  double acc = 0.0;

  auto adv = [&](long long& o) { o += plane; if (o >= cellsz) o -= cellsz; };
  auto gather = [&](const T* Qg) {
    T y[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      y[c] = own[c] + Qg[qrow + (c * 4 + 1) * nz + zm] + Qg[qup + (c * 4 + 2) * nz + z] +
             Qg[qup + (c * 4 + 3) * nz + zm];
    TOut* ob = obase + pg;
    if (OUT == OUT_APPLY || OUT == OUT_APPLY_DOT) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        st_val(ob + c * st, y[c]);
        if (OUT == OUT_APPLY_DOT) acc += (double)unode[c] * (double)y[c];
      }
    } else {
      const bool pin = (pg + col0 == 0);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (OUT == OUT_RESID) {
          st_val(ob + c * st, pin ? (T)0 : eb[c] - y[c]);
        } else {
          const T xv = unode[c] + (T)a.omega * eid * (eb[c] - y[c]);
          st_val(ob + c * st, xv);
          if (OUT == OUT_JACOBI_DOT) acc += (double)xv * (double)eb[c];
        }
      }
    }
  };

  // prologue: node plane i0-1 -> prev (through P[1], which step 1 reuses
  // only after two barriers)
  long long pk = (long long)((un.i0 - 1 + nx) % nx) * plane;   // voxel plane of kc_next
  long long pn = pk;                                           // node plane held in ld
  if (live) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ld0[c] = (T)ld_val(ub + c * st + pn + col0);
      if (extra) ld1[c] = (T)ld_val(ub + c * st + pn + col1);
    }
    kc_next = (T)ld_val(kcb + pk);
    T* Pw = P + PS;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Pw[prow + c * nz + z] = ld0[c];
      if (extra) Pw[prow + (3 + c) * nz + z] = ld1[c];
    }
  }
  __syncthreads();
  adv(pn);
  if (live) {
    const T* Pr = P + PS + prow;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      prev[c][0] = Pr[c * nz + z];
      prev[c][1] = Pr[c * nz + zp];
      prev[c][2] = Pr[(3 + c) * nz + z];
      prev[c][3] = Pr[(3 + c) * nz + zp];
      carry[c][0] = carry[c][1] = carry[c][2] = carry[c][3] = (T)0;
      ld0[c] = (T)ld_val(ub + c * st + pn + col0);
      if (extra) ld1[c] = (T)ld_val(ub + c * st + pn + col1);
    }
  }

  for (int s = 0; s <= un.len; ++s) {
    // voxel plane ie = i0-1+s (offset pe); node plane ie+1 (offset pn) is in ld
    const long long pe = pk;
    T* Pb = P + (s & 1) * PS;
    T* Qb = Q + (s & 1) * QS;
    if (live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Pb[prow + c * nz + z] = ld0[c];
        if (extra) Pb[prow + (3 + c) * nz + z] = ld1[c];
      }
      kcv = kc_next;
      if (s < un.len) {   // prefetch node plane ie+2 and voxel plane ie+1
        adv(pn);
        adv(pk);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ld0[c] = (T)ld_val(ub + c * st + pn + col0);
          if (extra) ld1[c] = (T)ld_val(ub + c * st + pn + col1);
        }
        kc_next = (T)ld_val(kcb + pk);
      }
    }
    __syncthreads();   // P[s&1] holds node plane ie+1; Q[(s-1)&1] holds node plane ie-1
    // gather node plane ie-1 (owned planes i0..i0+len-1 -> steps 2..len+1)
    if (s >= 2 && owner) gather(Q + ((s - 1) & 1) * QS);
    if (OUT >= OUT_JACOBI && owner && s >= 1) {
      // epilogue operands of node plane ie, used by the next step's gather:
      // loaded straight into their registers, a whole step ahead of use
#pragma unroll
      for (int c = 0; c < 3; ++c) eb[c] = (T)ld_val(bb + c * st + pe);
      if (OUT != OUT_RESID) eid = (T)ib[pe];
    }
    if (live) {
      T w[3][8];
      const T* Pr = Pb + prow;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T c0 = Pr[c * nz + z];
        const T c1 = Pr[c * nz + zp];
        const T c2 = Pr[(3 + c) * nz + z];
        const T c3 = Pr[(3 + c) * nz + zp];
        w[c][0] = prev[c][0]; w[c][1] = prev[c][1]; w[c][2] = prev[c][2]; w[c][3] = prev[c][3];
        w[c][4] = c0; w[c][5] = c1; w[c][6] = c2; w[c][7] = c3;
        unode[c] = prev[c][0];      // u at node (ie, jr, z), gathered at the next step
        prev[c][0] = c0; prev[c][1] = c1; prev[c][2] = c2; prev[c][3] = c3;
        fwht8_fwd(w[c]);
      }
      had_block(w, a.k, kcv);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        fwht8_inv(w[c]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const T tot = w[c][q] + carry[c][q];
          carry[c][q] = w[c][4 + q];
          if (q == 0) own[c] = tot;
          else if (s > 0) Qb[qrow + (c * 4 + q) * nz + z] = tot;
        }
      }
      pg = pe;
    }
  }
  __syncthreads();   // Q[len&1] holds the last owned node plane
  if (un.len >= 1 && owner) gather(Q + (un.len & 1) * QS);

  if (OUT == OUT_APPLY_DOT || OUT == OUT_JACOBI_DOT) {
    double v[1] = {acc};
    block_reduce<1>(v, red);
    if (tid == 0) a.partials[(long long)un.slot * kNumRhs + rhs] = v[0];
  }
}

// Shared memory bytes of one CTA (both buffers, + reduction scratch).
template <typename T>
inline size_t stencil_smem_bytes(int NT, int nz) {
  const int R = NT / nz;
  return ((sizeof(T) * 2 * ((size_t)(R + 1) * 3 * nz + (size_t)R * 12 * nz) + 15) & ~(size_t)15) +
         32 * sizeof(double);
}

}  // namespace femh

namespace femh {

// Two voxel rows per thread.  Thread (t, z) of a CTA streams voxels
// (i, e0, z) and (i, e0+1, z), e0 = j0-1+2t, along x.  Node rows n0 = e0,
// n1 = e0+1, n2 = e0+2: the y coupling of its two voxels (node row n1) stays in
// registers; it owns node rows n1 and n2 (n2 needs the lower-y corners of the
// next thread row's first voxel).  Owned rows per tile: 2*TR-1 for TR thread
// rows.  Shared memory per step: node plane P (slots 2t, 2t+1, 2t+2 hold rows
// n0, n1, n2 of thread t; slot 0 is the halo row loaded by t = 0) and corner
// totals Q (A: node (n1, z+1); B: (n2, z+1); C: (n0, z); D: (n0, z+1)), both
// double-buffered, one barrier per step.
template <typename T, int NT, int OUT, int NZ, typename TIn, typename TOut, typename TB, typename TC>
__global__ void __launch_bounds__(NT, 1)
stencil2_kernel(StencilArgs<TIn, TOut, TB, TC> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const StencilUnit un = a.units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = a.cells[un.cell];
  if (a.stt && !a.stt[cd.id * kNumRhs + rhs].active) return;
  const int nx = cd.nx, ny = cd.ny;
  const int nz = NZ > 0 ? NZ : cd.nz;
  const int TR = NT / nz;
  const int tid = threadIdx.x;
  const int t = tid / nz, z = tid - t * nz;
  const int rows = un.rows;
  const bool live = t < TR && 2 * t <= rows;
  const bool own1 = live && 2 * t < rows;
  const bool own2 = live && 2 * t + 1 < rows;
  const int zp = (z + 1 == nz) ? 0 : z + 1;
  const int zm = (z == 0) ? nz - 1 : z - 1;
  auto wrapy = [&](int j) { j %= ny; return j < 0 ? j + ny : j; };
  const int n0 = wrapy(un.j0 - 1 + 2 * t), n1 = wrapy(n0 + 1), n2 = wrapy(n0 + 2);

  const size_t PS = (size_t)(2 * TR + 1) * 3 * nz;
  const size_t QS = (size_t)TR * 12 * nz;
  T* P = reinterpret_cast<T*>(smem_raw);   // [2][2TR+1][3][nz]
  T* Q = P + 2 * PS;                       // [2][TR][4][3][nz]
  double* red = reinterpret_cast<double*>(smem_raw + ((sizeof(T) * (2 * PS + 2 * QS) + 15) & ~(size_t)15));
  const size_t s0 = (size_t)(2 * t) * 3 * nz;   // slot of row n0; n1 at +3nz, n2 at +6nz
  const size_t qt = (size_t)t * 12 * nz;
  const size_t qn = (size_t)(t + 1 < TR ? t + 1 : t) * 12 * nz;

  const long long st = a.ntot;
  const long long plane = (long long)ny * nz;
  const long long cellsz = (long long)nx * plane;
  const TIn* ub = a.u + (long long)rhs * 3 * st + cd.off;
  const long long c0 = (long long)n0 * nz + z, c1 = (long long)n1 * nz + z, c2 = (long long)n2 * nz + z;
  const TC* kcb = a.kc + cd.off;
  const TB* bb = (OUT >= OUT_JACOBI) ? a.b + (long long)rhs * 3 * st + cd.off : nullptr;
  const float* ib = a.invd + cd.off;
  TOut* obase = a.out + (long long)rhs * 3 * st + cd.off;

  T l0[3] = {0, 0, 0}, l1[3] = {0, 0, 0}, l2[3] = {0, 0, 0};   // next node plane, rows n0(t=0 only), n1, n2
  T k0v = 0, k1v = 0, k0n = 0, k1n = 0;                        // kc of voxel rows e0, e1
  T prev[3][2][3];          // [row n0..n2][z, z+1][comp], node plane ie
  T carry[3][2][3];         // upper-x contributions of the voxel pair, by node position
  T own1v[3] = {0, 0, 0}, own2v[3] = {0, 0, 0}, u1[3] = {0, 0, 0}, u2[3] = {0, 0, 0};
  T eb1[3] = {0, 0, 0}, eb2[3] = {0, 0, 0};
  T id1 = 0, id2 = 0;
  long long pg = 0;
  double acc = 0.0;

  auto adv = [&](long long& o) { o += plane; if (o >= cellsz) o -= cellsz; };
  auto load_plane = [&](long long po) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (t == 0) l0[c] = (T)ld_val(ub + c * st + po + c0);
      l1[c] = (T)ld_val(ub + c * st + po + c1);
      l2[c] = (T)ld_val(ub + c * st + po + c2);
    }
  };
  auto store_plane = [&](T* Pb) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (t == 0) Pb[s0 + c * nz + z] = l0[c];
      Pb[s0 + (3 + c) * nz + z] = l1[c];
      Pb[s0 + (6 + c) * nz + z] = l2[c];
    }
  };
  auto epilogue = [&](T (&y)[3], const T (&un_)[3], const T (&ebv)[3], T idv, long long node) {
    TOut* ob = obase + node;
    if (OUT == OUT_APPLY || OUT == OUT_APPLY_DOT) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        st_val(ob + c * st, y[c]);
        if (OUT == OUT_APPLY_DOT) acc += (double)un_[c] * (double)y[c];
      }
    } else {
      const bool pin = (node == 0);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (OUT == OUT_RESID) {
          st_val(ob + c * st, pin ? (T)0 : ebv[c] - y[c]);
        } else {
          const T xv = un_[c] + (T)a.omega * idv * (ebv[c] - y[c]);
          st_val(ob + c * st, xv);
          if (OUT == OUT_JACOBI_DOT) acc += (double)xv * (double)ebv[c];
        }
      }
    }
  };
  auto gather = [&](const T* Qg) {
    if (own1) {
      T y[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) y[c] = own1v[c] + Qg[qt + (0 * 3 + c) * nz + zm];
      epilogue(y, u1, eb1, id1, pg + c1);
    }
    if (own2) {
      T y[3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        y[c] = own2v[c] + Qg[qt + (1 * 3 + c) * nz + zm] + Qg[qn + (2 * 3 + c) * nz + z] +
               Qg[qn + (3 * 3 + c) * nz + zm];
      epilogue(y, u2, eb2, id2, pg + c2);
    }
  };

  // prologue: node plane i0-1 -> prev (via P[1])
  long long pk = (long long)((un.i0 - 1 + nx) % nx) * plane;
  long long pn = pk;
  if (live) {
    load_plane(pn);
    k0n = (T)ld_val(kcb + pk + c0);
    k1n = (T)ld_val(kcb + pk + c1);
    store_plane(P + PS);
  }
  __syncthreads();
  adv(pn);
  if (live) {
    const T* Pr = P + PS + s0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        prev[r][0][c] = Pr[(3 * r + c) * nz + z];
        prev[r][1][c] = Pr[(3 * r + c) * nz + zp];
        carry[r][0][c] = carry[r][1][c] = (T)0;
      }
    load_plane(pn);
  }

  for (int s = 0; s <= un.len; ++s) {
    const long long pe = pk;   // voxel plane ie = i0-1+s
    T* Pb = P + (s & 1) * PS;
    T* Qb = Q + (s & 1) * QS;
    if (live) {
      store_plane(Pb);
      k0v = k0n;
      k1v = k1n;
      if (s < un.len) {
        adv(pn);
        adv(pk);
        load_plane(pn);
        k0n = (T)ld_val(kcb + pk + c0);
        k1n = (T)ld_val(kcb + pk + c1);
      }
    }
    __syncthreads();
    if (s >= 2) gather(Q + ((s - 1) & 1) * QS);
    if (OUT >= OUT_JACOBI && s >= 1) {
      if (own1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) eb1[c] = (T)ld_val(bb + c * st + pe + c1);
        if (OUT != OUT_RESID) id1 = (T)ib[pe + c1];
      }
      if (own2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) eb2[c] = (T)ld_val(bb + c * st + pe + c2);
        if (OUT != OUT_RESID) id2 = (T)ib[pe + c2];
      }
    }
    if (live) {
      T cur[3][2][3];
      const T* Pr = Pb + s0;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cur[r][0][c] = Pr[(3 * r + c) * nz + z];
          cur[r][1][c] = Pr[(3 * r + c) * nz + zp];
        }
      T tot[3][2][3], nc[3][2][3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            tot[r][q][c] = carry[r][q][c];
            nc[r][q][c] = (T)0;
          }
#pragma unroll
      for (int e = 0; e < 2; ++e) {   // voxel rows e0 (node rows 0,1) and e1 (rows 1,2)
        T w[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
          for (int ay = 0; ay < 2; ++ay)
#pragma unroll
            for (int az = 0; az < 2; ++az) {
              w[c][2 * ay + az] = prev[e + ay][az][c];
              w[c][4 + 2 * ay + az] = cur[e + ay][az][c];
            }
          fwht8_fwd(w[c]);
        }
        had_block(w, a.k, e == 0 ? k0v : k1v);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          fwht8_inv(w[c]);
#pragma unroll
          for (int ay = 0; ay < 2; ++ay)
#pragma unroll
            for (int az = 0; az < 2; ++az) {
              tot[e + ay][az][c] += w[c][2 * ay + az];
              nc[e + ay][az][c] += w[c][4 + 2 * ay + az];
            }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u1[c] = prev[1][0][c];
        u2[c] = prev[2][0][c];
        own1v[c] = tot[1][0][c];
        own2v[c] = tot[2][0][c];
        if (s > 0) {
          Qb[qt + (0 * 3 + c) * nz + z] = tot[1][1][c];   // A: node (n1, z+1)
          Qb[qt + (1 * 3 + c) * nz + z] = tot[2][1][c];   // B: node (n2, z+1)
          Qb[qt + (2 * 3 + c) * nz + z] = tot[0][0][c];   // C: node (n0, z)
          Qb[qt + (3 * 3 + c) * nz + z] = tot[0][1][c];   // D: node (n0, z+1)
        }
      }
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            carry[r][q][c] = nc[r][q][c];
            prev[r][q][c] = cur[r][q][c];
          }
      pg = pe;
    }
  }
  __syncthreads();
  if (un.len >= 1) gather(Q + (un.len & 1) * QS);

  if (OUT == OUT_APPLY_DOT || OUT == OUT_JACOBI_DOT) {
    double v[1] = {acc};
    block_reduce<1>(v, red);
    if (tid == 0) a.partials[(long long)un.slot * kNumRhs + rhs] = v[0];
  }
}

}  // namespace femh
