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
  OUT_JACOBI = 2,      // out = u + omega * D^-1 (b - K u), D point or node-block diagonal
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
  float2 kp[8];          // FP32 pairs (x = y) of A, Bd-Bo, Bo, D1-O1, O1, D2-O2, O2, G
  int* err;              // set non-zero by a kernel whose bounded wait ran out
  int wait_limit;        // 0: every stage wait gives up at once (tests); else kWaitLimit rounds
  const int* cta_units;  // staged FP32 kernel: CTA b runs units [cta_units[b], cta_units[b+1]); nullptr: unit b
  const float* binv;     // node-block Jacobi sweeps: per node 3x3 inverse diagonal block
                         // [xx, yy, zz, xy, xz, yz]; nullptr: point Jacobi with invd
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
      T dv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) dv[c] = eb[c] - y[c];
      if (OUT == OUT_RESID) {
#pragma unroll
        for (int c = 0; c < 3; ++c) st_val(ob + c * st, pin ? (T)0 : dv[c]);
      } else {
        jacobi_dir<T>(a.binv, cd.off + pg + col0, (T)a.omega * eid, dv);   // point: omega invd folded in
        const T sc = a.binv ? (T)a.omega : (T)1;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T xv = unode[c] + sc * dv[c];
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
      T dv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) dv[c] = ebv[c] - y[c];
      if (OUT == OUT_RESID) {
#pragma unroll
        for (int c = 0; c < 3; ++c) st_val(ob + c * st, pin ? (T)0 : dv[c]);
      } else {
        jacobi_dir<T>(a.binv, cd.off + node, (T)a.omega * idv, dv);   // point: omega invd folded in
        const T sc = a.binv ? (T)a.omega : (T)1;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T xv = un_[c] + sc * dv[c];
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

// ------------------------------------------------------------------ pairs ---
// Two load cases of one node or voxel in the two lanes of a packed FP32x2
// register: sm_100 add/sub/mul/fma.f32x2 process both lanes in one
// instruction, and the two cases share every index, coefficient and shared
// memory access (64-bit).
using f2 = float2;
__device__ __forceinline__ f2 p_add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 p_mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 p_fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 p_sub(f2 a, f2 b) {
  unsigned long long ra, rb, rd;
  memcpy(&ra, &a, 8);
  memcpy(&rb, &b, 8);
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  f2 d;
  memcpy(&d, &rd, 8);
  return d;
}
__device__ __forceinline__ f2 p_bc(float s) { return make_float2(s, s); }

// Node-block Jacobi direction of two nodes in the two lanes: d <- B d with
// lane x the block at b1, lane y the block at b2 (layout of jacobi_dir).
__device__ __forceinline__ void block_dir2(const float* __restrict__ b1, const float* __restrict__ b2, f2 (&d)[3]) {
  // one scalar load per lane and entry, straight into the pair's halves
  const f2 xx = make_float2(b1[0], b2[0]), yy = make_float2(b1[1], b2[1]), zz = make_float2(b1[2], b2[2]);
  const f2 xy = make_float2(b1[3], b2[3]), xz = make_float2(b1[4], b2[4]), yz = make_float2(b1[5], b2[5]);
  const f2 d0 = d[0], d1 = d[1], d2 = d[2];
  d[0] = p_fma(xz, d2, p_fma(xy, d1, p_mul(xx, d0)));
  d[1] = p_fma(yz, d2, p_fma(yy, d1, p_mul(xy, d0)));
  d[2] = p_fma(zz, d2, p_fma(yz, d1, p_mul(xz, d0)));
}

// 2x2 Hadamard transform of a node patch, index 2*ay + az (same stage order
// and signs as fwht8_fwd restricted to bits 1 and 2).
__device__ __forceinline__ void had4_fwd(f2 (&v)[4]) {
  const f2 a0 = p_add(v[1], v[0]), a1 = p_sub(v[1], v[0]);
  const f2 a2 = p_add(v[3], v[2]), a3 = p_sub(v[3], v[2]);
  v[0] = p_add(a2, a0);
  v[2] = p_sub(a2, a0);
  v[1] = p_add(a3, a1);
  v[3] = p_sub(a3, a1);
}
// Inverse stages of fwht8_inv for bits 2 and 1.
__device__ __forceinline__ void had4_inv(f2 (&v)[4]) {
  const f2 a0 = p_sub(v[0], v[2]), a2 = p_add(v[0], v[2]);
  const f2 a1 = p_sub(v[1], v[3]), a3 = p_add(v[1], v[3]);
  v[0] = p_sub(a0, a1);
  v[1] = p_add(a0, a1);
  v[2] = p_sub(a2, a3);
  v[3] = p_add(a2, a3);
}

// had_block on packed pairs; s = c_e * h (one scale for both lanes).
__device__ __forceinline__ void had_block_p(f2 (&w)[3][8], const HadK& K, float s) {
  const f2 A = p_bc(s * (float)K.A), Bdo = p_bc(s * (float)(K.Bd - K.Bo)), Bo = p_bc(s * (float)K.Bo);
  const f2 D1o = p_bc(s * (float)(K.D1 - K.O1)), O1 = p_bc(s * (float)K.O1);
  const f2 D2o = p_bc(s * (float)(K.D2 - K.O2)), O2 = p_bc(s * (float)K.O2), G = p_bc(s * (float)K.G);
  {
    const f2 n0 = w[0][4], n1 = w[1][2], n2 = w[2][1];
    const f2 t = p_mul(Bo, p_add(p_add(n0, n1), n2));
    w[0][4] = p_fma(Bdo, n0, t);
    w[1][2] = p_fma(Bdo, n1, t);
    w[2][1] = p_fma(Bdo, n2, t);
  }
  {
    const f2 sxz = p_mul(A, p_add(w[0][1], w[2][4]));
    const f2 syz = p_mul(A, p_add(w[1][1], w[2][2]));
    const f2 sxy = p_mul(A, p_add(w[0][2], w[1][4]));
    w[0][1] = sxz; w[2][4] = sxz;
    w[1][1] = syz; w[2][2] = syz;
    w[0][2] = sxy; w[1][4] = sxy;
  }
  {
    const f2 t0 = w[0][3], t1 = w[1][5], t2 = w[2][6];
    const f2 t = p_mul(O1, p_add(p_add(t0, t1), t2));
    w[0][3] = p_fma(D1o, t0, t);
    w[1][5] = p_fma(D1o, t1, t);
    w[2][6] = p_fma(D1o, t2, t);
  }
  {
    const f2 a = w[1][3], b = w[0][5], t = p_mul(O2, p_add(a, b));
    w[1][3] = p_fma(D2o, a, t); w[0][5] = p_fma(D2o, b, t);
  }
  {
    const f2 a = w[2][3], b = w[0][6], t = p_mul(O2, p_add(a, b));
    w[2][3] = p_fma(D2o, a, t); w[0][6] = p_fma(D2o, b, t);
  }
  {
    const f2 a = w[2][5], b = w[1][6], t = p_mul(O2, p_add(a, b));
    w[2][5] = p_fma(D2o, a, t); w[1][6] = p_fma(D2o, b, t);
  }
  w[0][7] = p_mul(w[0][7], G); w[1][7] = p_mul(w[1][7], G); w[2][7] = p_mul(w[2][7], G);
}

// One voxel row per thread, two load cases per CTA (blockIdx.y = case pair),
// FP32x2 arithmetic.  Layout and schedule of stencil_kernel, with two changes
// that remove redundant transform work: the lower node plane of each voxel is
// carried from the previous step already transformed in y and z (a voxel's
// upper plane is the next voxel's lower plane), and the upper-plane
// contributions are carried in the same half-transformed basis, so the y/z
// inverse stages run once per node plane on the summed contributions of both
// voxels that share it.  Shared memory: P[2][R+1][3][nz] node planes and
// Q[2][R][3 corners][3][nz] corner totals (pairs, shared between threads), and
// per thread the two carried sets (12 pairs each) as float4 slots
// [6][NT] that only their thread touches (no barrier; registers stay below
// the 128 a 512-thread CTA allows).
template <int NT, int OUT, int NZ, typename TIn, typename TOut, typename TB, typename TC>
__global__ void __launch_bounds__(NT, 1)
stencilp_kernel(StencilArgs<TIn, TOut, TB, TC> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const StencilUnit un = a.units[blockIdx.x];
  const int pr = blockIdx.y;   // load cases 2pr, 2pr+1
  const CellDesc cd = a.cells[un.cell];
  if (a.stt && !a.stt[cd.id * kNumRhs + 2 * pr].active && !a.stt[cd.id * kNumRhs + 2 * pr + 1].active) return;
  const int nx = cd.nx, ny = cd.ny;
  const int nz = NZ > 0 ? NZ : cd.nz;
  const int R = NT / nz;
  const int tid = threadIdx.x;
  const int r = tid / nz, z = tid - r * nz;
  const bool live = r < R && r <= un.rows;
  const int zp = (z + 1 == nz) ? 0 : z + 1;
  const int zm = (z == 0) ? nz - 1 : z - 1;
  int jr = un.j0 - 1 + r;
  if (jr < 0) jr += ny;
  while (jr >= ny) jr -= ny;
  const int jr1 = (jr + 1 == ny) ? 0 : jr + 1;
  const bool extra = live && r == un.rows;
  const bool owner = live && r >= 1;

  // private carries first (16-byte aligned float4 slots), then P, Q, reduction
  float4* CPv = reinterpret_cast<float4*>(smem_raw);   // [6][NT] transformed lower plane
  float4* CCa = CPv + 6 * NT;                           // [6][NT] upper-plane contributions
  const int PS = (R + 1) * 3 * nz;   // pairs in one P buffer
  const int QS = R * 9 * nz;         // pairs in one Q buffer
  f2* P = reinterpret_cast<f2*>(CCa + 6 * NT);
  f2* Q = P + 2 * PS;
  double* red = reinterpret_cast<double*>(Q + 2 * QS);
  const int prow = r * 3 * nz, qrow = r * 9 * nz;
  const int qup = (r > 0 ? r - 1 : 0) * 9 * nz;

  const long long st = a.ntot, st3 = 3 * a.ntot;
  const int plane = ny * nz;
  const int cellsz = nx * plane;
  const int col0 = jr * nz + z, col1 = jr1 * nz + z;
  const TIn* ua = a.u + (long long)(2 * pr) * 3 * st + cd.off;
  const TC* kcb = a.kc + cd.off + col0;
  const TB* ba = (OUT >= OUT_JACOBI) ? a.b + (long long)(2 * pr) * 3 * st + cd.off + col0 : nullptr;
  const float* ib = a.invd + cd.off + col0;
  TOut* oa = a.out + (long long)(2 * pr) * 3 * st + cd.off + col0;

  auto ldp = [&](const TIn* p) { return make_float2((float)ld_val(p), (float)ld_val(p + st3)); };
  auto put = [&](float4* base, const f2 (&h)[3][4]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 2; ++k)
        base[(2 * c + k) * NT + tid] = make_float4(h[c][2 * k].x, h[c][2 * k].y, h[c][2 * k + 1].x, h[c][2 * k + 1].y);
  };
  auto get = [&](const float4* base, f2 (&h)[3][4]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const float4 v = base[(2 * c + k) * NT + tid];
        h[c][2 * k] = make_float2(v.x, v.y);
        h[c][2 * k + 1] = make_float2(v.z, v.w);
      }
  };

  using TBv = decltype(ld_val(a.b));   // raw operand, converted where it is used
  f2 ld0[3], ld1[3];
  TBv ebA[3], ebB[3];
  float kcv = 0.f, kc_next = 0.f, eid = 0.f;
  f2 own[3], unode[3], rawn[3];
  int pg = 0;
  double accA = 0.0, accB = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ld0[c] = ld1[c] = own[c] = unode[c] = rawn[c] = p_bc(0.f);
    ebA[c] = ebB[c] = (TBv)0;
  }

  auto adv = [&](int& o) { o += plane; if (o >= cellsz) o -= cellsz; };
  auto gather = [&](const f2* Qg) {
    f2 y[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      y[c] = p_add(p_add(own[c], Qg[qrow + (0 * 3 + c) * nz + zm]),
                   p_add(Qg[qup + (1 * 3 + c) * nz + z], Qg[qup + (2 * 3 + c) * nz + zm]));
    TOut* ob = oa + pg;
    if (OUT == OUT_APPLY || OUT == OUT_APPLY_DOT) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        st_val(ob + c * st, y[c].x);
        st_val(ob + c * st + st3, y[c].y);
        if (OUT == OUT_APPLY_DOT) {
          accA += (double)unode[c].x * (double)y[c].x;
          accB += (double)unode[c].y * (double)y[c].y;
        }
      }
    } else {
      const bool pin = (pg + col0 == 0);
      const f2 wd = p_bc((float)a.omega * eid);
      f2 bd[3];   // node-block Jacobi: B (b - y), both load cases
      if (OUT != OUT_RESID && a.binv) {
        float dA[3], dB[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          dA[c] = (float)ebA[c] - y[c].x;
          dB[c] = (float)ebB[c] - y[c].y;
        }
        jacobi_dir<float>(a.binv, cd.off + pg + col0, 0.f, dA);
        jacobi_dir<float>(a.binv, cd.off + pg + col0, 0.f, dB);
#pragma unroll
        for (int c = 0; c < 3; ++c) bd[c] = make_float2(dA[c], dB[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const f2 bv = make_float2((float)ebA[c], (float)ebB[c]);
        const f2 d = p_sub(bv, y[c]);
        if (OUT == OUT_RESID) {
          st_val(ob + c * st, pin ? 0.f : d.x);
          st_val(ob + c * st + st3, pin ? 0.f : d.y);
        } else {
          const f2 xv = a.binv ? p_fma(p_bc((float)a.omega), bd[c], unode[c]) : p_fma(wd, d, unode[c]);
          st_val(ob + c * st, xv.x);
          st_val(ob + c * st + st3, xv.y);
          if (OUT == OUT_JACOBI_DOT) {
            accA += (double)xv.x * (double)bv.x;
            accB += (double)xv.y * (double)bv.y;
          }
        }
      }
    }
  };
  // the 2x2 patch of node plane Pb whose lower corner is this thread's node
  // (own value given), transformed in y and z
  auto patch = [&](const f2* Pb, const f2 (&mine)[3], f2 (&h)[3][4]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      h[c][0] = mine[c];
      h[c][1] = Pb[prow + c * nz + zp];
      h[c][2] = Pb[prow + (3 + c) * nz + z];
      h[c][3] = Pb[prow + (3 + c) * nz + zp];
      had4_fwd(h[c]);
    }
  };

  // prologue: node plane i0-1 -> carried lower plane (through P[1])
  int pk = ((un.i0 - 1 + nx) % nx) * plane;
  int pn = pk;
  if (live) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ld0[c] = ldp(ua + c * st + pn + col0);
      if (extra) ld1[c] = ldp(ua + c * st + pn + col1);
    }
    kc_next = (float)ld_val(kcb + pk);
    f2* Pw = P + PS;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Pw[prow + c * nz + z] = ld0[c];
      if (extra) Pw[prow + (3 + c) * nz + z] = ld1[c];
    }
  }
  __syncthreads();
  adv(pn);
  if (live) {
    f2 h[3][4];
    patch(P + PS, ld0, h);
    put(CPv, h);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int q = 0; q < 4; ++q) h[c][q] = p_bc(0.f);
      rawn[c] = ld0[c];
      ld0[c] = ldp(ua + c * st + pn + col0);
      if (extra) ld1[c] = ldp(ua + c * st + pn + col1);
    }
    put(CCa, h);
  }

  for (int s = 0; s <= un.len; ++s) {
    const int pe = pk;   // voxel plane ie = i0-1+s; node plane ie+1 is in ld0/ld1
    f2* Pb = P + (s & 1) * PS;
    f2* Qb = Q + (s & 1) * QS;
    f2 cur0[3];
    if (live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Pb[prow + c * nz + z] = ld0[c];
        if (extra) Pb[prow + (3 + c) * nz + z] = ld1[c];
        cur0[c] = ld0[c];
      }
      kcv = kc_next;
      if (s < un.len) {
        adv(pn);
        adv(pk);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ld0[c] = ldp(ua + c * st + pn + col0);
          if (extra) ld1[c] = ldp(ua + c * st + pn + col1);
        }
        kc_next = (float)ld_val(kcb + pk);
      }
    }
    __syncthreads();   // P[s&1] holds node plane ie+1; Q[(s-1)&1] holds node plane ie-1
    if (s >= 2 && owner) gather(Q + ((s - 1) & 1) * QS);
    if (OUT >= OUT_JACOBI && owner && s >= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ebA[c] = ld_val(ba + c * st + pe);
        ebB[c] = ld_val(ba + c * st + st3 + pe);
      }
      if (OUT != OUT_RESID) eid = ib[pe];
    }
    if (live) {
      f2 w[3][8];
      {
        f2 cur[3][4], prv[3][4];
        patch(Pb, cur0, cur);
        get(CPv, prv);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (q > 0) w[c][q] = p_add(cur[c][q], prv[c][q]);
            w[c][4 + q] = p_sub(cur[c][q], prv[c][q]);
          }
        put(CPv, cur);
      }
      had_block_p(w, a.k, kcv);
      // inverse x stage: lower plane (node plane ie) = w[q] - w[4+q], upper
      // plane = w[q] + w[4+q]; w[0] = 0 (translations carry no energy)
      f2 car[3][4];
      get(CCa, car);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        f2 tot[4];
        tot[0] = p_sub(car[c][0], w[c][4]);
        car[c][0] = w[c][4];
#pragma unroll
        for (int q = 1; q < 4; ++q) {
          tot[q] = p_add(p_sub(w[c][q], w[c][4 + q]), car[c][q]);
          car[c][q] = p_add(w[c][q], w[c][4 + q]);
        }
        had4_inv(tot);
        own[c] = tot[0];
        unode[c] = rawn[c];
        rawn[c] = cur0[c];
        if (s > 0) {
          Qb[qrow + (0 * 3 + c) * nz + z] = tot[1];   // node (jr, z+1)
          Qb[qrow + (1 * 3 + c) * nz + z] = tot[2];   // node (jr+1, z)
          Qb[qrow + (2 * 3 + c) * nz + z] = tot[3];   // node (jr+1, z+1)
        }
      }
      put(CCa, car);
      pg = pe;
    }
  }
  __syncthreads();
  if (un.len >= 1 && owner) gather(Q + (un.len & 1) * QS);

  if (OUT == OUT_APPLY_DOT || OUT == OUT_JACOBI_DOT) {
    double v[2] = {accA, accB};
    block_reduce<2>(v, red);
    if (tid == 0) {
      a.partials[(long long)un.slot * kNumRhs + 2 * pr] = v[0];
      a.partials[(long long)un.slot * kNumRhs + 2 * pr + 1] = v[1];
    }
  }
}

// Two voxel rows per thread with the two voxels in the two lanes of packed
// FP32x2 registers (FP32 operators).  Thread (t, z) streams voxels (i, e0, z)
// (lane x) and (i, e0+1, z) (lane y), e0 = j0-1+2t, along x; node rows
// n0 = e0, n1, n2.  Lane x of a patch pair is row n0 or n1 and lane y the row
// one above, so the pair (n1, n2) of this thread's own nodes is used as
// loaded, and the two stiffness scales (kc of rows e0, e0+1) form a pair.  As
// in stencilp_kernel the lower node plane is carried transformed in y and z
// and the upper-plane contributions are carried half transformed.
// Shared memory (double-buffered): P2[TR][3][nz] pairs (n1, n2) of each
// thread, H0[3][nz] the halo row n0 of thread 0; QAB[TR][3][nz] pairs of
// corner totals (node (n1, z+1), node (n2, z+1)) and QCD[TR][3][nz] pairs
// (node (n0, z), node (n0, z+1)) for the thread below.
template <int NT, int OUT, int NZ, typename TIn, typename TOut, typename TB, typename TC>
__global__ void __launch_bounds__(NT, 1)
stencil2p_kernel(StencilArgs<TIn, TOut, TB, TC> a) {
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

  const int PS = TR * 3 * nz;        // pairs in one P2 / QAB / QCD buffer
  f2* P2 = reinterpret_cast<f2*>(smem_raw);   // [2][TR][3][nz]
  f2* QAB = P2 + 2 * PS;                       // [2][TR][3][nz]
  f2* QCD = QAB + 2 * PS;                      // [2][TR][3][nz]
  float* H0 = reinterpret_cast<float*>(QCD + 2 * PS);   // [2][3][nz]
  double* red = reinterpret_cast<double*>(H0 + ((6 * nz + 1) & ~1));
  const int pt = t * 3 * nz;                   // this thread's slot
  const int pb = (t > 0 ? t - 1 : 0) * 3 * nz; // slot of the thread below (n0 = its n2)
  const int pa = (t + 1 < TR ? t + 1 : t) * 3 * nz;   // slot of the thread above

  const long long st = a.ntot;
  const int plane = ny * nz;
  const int cellsz = nx * plane;
  const int c0 = n0 * nz + z, c1 = n1 * nz + z, c2 = n2 * nz + z;
  const TIn* ub = a.u + (long long)rhs * 3 * st + cd.off;
  const TC* kcb = a.kc + cd.off;
  const TB* bb = (OUT >= OUT_JACOBI) ? a.b + (long long)rhs * 3 * st + cd.off : nullptr;
  const float* ib = a.invd + cd.off;
  TOut* obase = a.out + (long long)rhs * 3 * st + cd.off;

  using TBv = decltype(ld_val(a.b));
  f2 l12[3];                 // node plane being prefetched: rows (n1, n2)
  float l0[3] = {0.f, 0.f, 0.f};   // and row n0 (thread 0: the halo row)
  f2 kn = p_bc(0.f), kv;     // kc of voxel rows (e0, e0+1), next and current
  f2 prv[3][4], car[3][4];
  f2 own[3], u12[3], raw[3];
  TBv eb1[3], eb2[3];
  f2 id12 = p_bc(0.f);
  int pg = 0;
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    l12[c] = own[c] = u12[c] = raw[c] = p_bc(0.f);
    eb1[c] = eb2[c] = (TBv)0;
  }

  auto adv = [&](int& o) { o += plane; if (o >= cellsz) o -= cellsz; };
  auto load_plane = [&](int po) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (t == 0) l0[c] = (float)ld_val(ub + c * st + po + c0);
      l12[c] = make_float2((float)ld_val(ub + c * st + po + c1), (float)ld_val(ub + c * st + po + c2));
    }
  };
  auto load_kc = [&](int pk) { kn = make_float2((float)ld_val(kcb + pk + c0), (float)ld_val(kcb + pk + c1)); };
  auto store_plane = [&](f2* Pb, float* Hb) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Pb[pt + c * nz + z] = l12[c];
      if (t == 0) Hb[c * nz + z] = l0[c];
    }
  };
  // y/z-transformed patches of the node plane in Pb/Hb (own pair given)
  auto patch = [&](const f2* Pb, const float* Hb, const f2 (&mine)[3], f2 (&h)[3][4]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const f2 up = Pb[pt + c * nz + zp];   // (n1, n2) at z+1
      const float b0 = t == 0 ? Hb[c * nz + z] : Pb[pb + c * nz + z].y;
      const float b1 = t == 0 ? Hb[c * nz + zp] : Pb[pb + c * nz + zp].y;
      h[c][0] = make_float2(b0, mine[c].x);
      h[c][1] = make_float2(b1, up.x);
      h[c][2] = mine[c];
      h[c][3] = up;
      had4_fwd(h[c]);
    }
  };
  auto epilogue = [&](const f2 (&y)[3]) {
    TOut* ob = obase + pg;
    if (OUT == OUT_APPLY || OUT == OUT_APPLY_DOT) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (own1) st_val(ob + c * st + c1, y[c].x);
        if (own2) st_val(ob + c * st + c2, y[c].y);
        if (OUT == OUT_APPLY_DOT) {
          if (own1) acc += (double)u12[c].x * (double)y[c].x;
          if (own2) acc += (double)u12[c].y * (double)y[c].y;
        }
      }
    } else {
      const bool pin1 = (pg + c1 == 0), pin2 = (pg + c2 == 0);
      const f2 wd = p_mul(p_bc((float)a.omega), id12);
      f2 bd[3];   // node-block Jacobi: B (b - y) of both nodes
      if (OUT != OUT_RESID && a.binv) {
#pragma unroll
        for (int c = 0; c < 3; ++c) bd[c] = p_sub(make_float2((float)eb1[c], (float)eb2[c]), y[c]);
        block_dir2(a.binv + 6 * (cd.off + pg + c1), a.binv + 6 * (cd.off + pg + c2), bd);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const f2 bv = make_float2((float)eb1[c], (float)eb2[c]);
        const f2 d = p_sub(bv, y[c]);
        if (OUT == OUT_RESID) {
          if (own1) st_val(ob + c * st + c1, pin1 ? 0.f : d.x);
          if (own2) st_val(ob + c * st + c2, pin2 ? 0.f : d.y);
        } else {
          const f2 xv = a.binv ? p_fma(p_bc((float)a.omega), bd[c], u12[c]) : p_fma(wd, d, u12[c]);
          if (own1) st_val(ob + c * st + c1, xv.x);
          if (own2) st_val(ob + c * st + c2, xv.y);
          if (OUT == OUT_JACOBI_DOT) {
            if (own1) acc += (double)xv.x * (double)bv.x;
            if (own2) acc += (double)xv.y * (double)bv.y;
          }
        }
      }
    }
  };
  auto gather = [&](int buf) {
    const f2* Qab = QAB + buf * PS;
    const f2* Qcd = QCD + buf * PS;
    f2 y[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      y[c] = p_add(own[c], Qab[pt + c * nz + zm]);
      y[c].y += Qcd[pa + c * nz + z].x + Qcd[pa + c * nz + zm].y;
    }
    epilogue(y);
  };

  // prologue: node plane i0-1 -> carried transformed patches (through buffer 1)
  int pk = ((un.i0 - 1 + nx) % nx) * plane;
  int pn = pk;
  if (live) {
    load_plane(pn);
    load_kc(pk);
    store_plane(P2 + PS, H0 + 3 * nz);
  }
  __syncthreads();
  adv(pn);
  if (live) {
    patch(P2 + PS, H0 + 3 * nz, l12, prv);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      raw[c] = l12[c];
#pragma unroll
      for (int q = 0; q < 4; ++q) car[c][q] = p_bc(0.f);
    }
    load_plane(pn);
  }

  for (int s = 0; s <= un.len; ++s) {
    const int pe = pk;   // voxel plane ie = i0-1+s; node plane ie+1 is in l12/l0
    const int buf = s & 1;
    f2* Pb = P2 + buf * PS;
    float* Hb = H0 + buf * 3 * nz;
    f2 cur0[3];
    if (live) {
      store_plane(Pb, Hb);
#pragma unroll
      for (int c = 0; c < 3; ++c) cur0[c] = l12[c];
      kv = kn;
      if (s < un.len) {
        adv(pn);
        adv(pk);
        load_plane(pn);
        load_kc(pk);
      }
    }
    __syncthreads();   // buffer buf holds node plane ie+1; Q[buf^1] holds node plane ie-1
    if (s >= 2 && live) gather(buf ^ 1);
    if (OUT >= OUT_JACOBI && s >= 1 && live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        eb1[c] = ld_val(bb + c * st + pe + c1);
        eb2[c] = ld_val(bb + c * st + pe + c2);
      }
      if (OUT != OUT_RESID) id12 = make_float2(ib[pe + c1], ib[pe + c2]);
    }
    if (live) {
      f2 w[3][8];
      {
        f2 cur[3][4];
        patch(Pb, Hb, cur0, cur);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (q > 0) w[c][q] = p_add(cur[c][q], prv[c][q]);
            w[c][4 + q] = p_sub(cur[c][q], prv[c][q]);
            prv[c][q] = cur[c][q];
          }
      }
      {   // Hadamard-domain element operator, scales (kc(e0), kc(e0+1))
        const f2 A = p_mul(kv, a.kp[0]), Bdo = p_mul(kv, a.kp[1]), Bo = p_mul(kv, a.kp[2]);
        const f2 D1o = p_mul(kv, a.kp[3]), O1 = p_mul(kv, a.kp[4]);
        const f2 D2o = p_mul(kv, a.kp[5]), O2 = p_mul(kv, a.kp[6]), G = p_mul(kv, a.kp[7]);
        {
          const f2 m0 = w[0][4], m1 = w[1][2], m2 = w[2][1];
          const f2 tt = p_mul(Bo, p_add(p_add(m0, m1), m2));
          w[0][4] = p_fma(Bdo, m0, tt); w[1][2] = p_fma(Bdo, m1, tt); w[2][1] = p_fma(Bdo, m2, tt);
        }
        {
          const f2 sxz = p_mul(A, p_add(w[0][1], w[2][4]));
          const f2 syz = p_mul(A, p_add(w[1][1], w[2][2]));
          const f2 sxy = p_mul(A, p_add(w[0][2], w[1][4]));
          w[0][1] = sxz; w[2][4] = sxz; w[1][1] = syz; w[2][2] = syz; w[0][2] = sxy; w[1][4] = sxy;
        }
        {
          const f2 m0 = w[0][3], m1 = w[1][5], m2 = w[2][6];
          const f2 tt = p_mul(O1, p_add(p_add(m0, m1), m2));
          w[0][3] = p_fma(D1o, m0, tt); w[1][5] = p_fma(D1o, m1, tt); w[2][6] = p_fma(D1o, m2, tt);
        }
        {
          const f2 x0 = w[1][3], x1 = w[0][5], tt = p_mul(O2, p_add(x0, x1));
          w[1][3] = p_fma(D2o, x0, tt); w[0][5] = p_fma(D2o, x1, tt);
        }
        {
          const f2 x0 = w[2][3], x1 = w[0][6], tt = p_mul(O2, p_add(x0, x1));
          w[2][3] = p_fma(D2o, x0, tt); w[0][6] = p_fma(D2o, x1, tt);
        }
        {
          const f2 x0 = w[2][5], x1 = w[1][6], tt = p_mul(O2, p_add(x0, x1));
          w[2][5] = p_fma(D2o, x0, tt); w[1][6] = p_fma(D2o, x1, tt);
        }
        w[0][7] = p_mul(w[0][7], G); w[1][7] = p_mul(w[1][7], G); w[2][7] = p_mul(w[2][7], G);
      }
      f2* Qab = QAB + buf * PS;
      f2* Qcd = QCD + buf * PS;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        f2 tot[4];
        tot[0] = p_sub(car[c][0], w[c][4]);
        car[c][0] = w[c][4];
#pragma unroll
        for (int q = 1; q < 4; ++q) {
          tot[q] = p_add(p_sub(w[c][q], w[c][4 + q]), car[c][q]);
          car[c][q] = p_add(w[c][q], w[c][4 + q]);
        }
        had4_inv(tot);
        // lane x: rows (n0 | n1), lane y: rows (n1 | n2); index 2*ay + az
        own[c] = make_float2(tot[0].y + tot[2].x, tot[2].y);   // nodes (n1, z), (n2, z)
        u12[c] = raw[c];
        raw[c] = cur0[c];
        if (s > 0) {
          Qab[pt + c * nz + z] = make_float2(tot[1].y + tot[3].x, tot[3].y);   // (n1, z+1), (n2, z+1)
          Qcd[pt + c * nz + z] = make_float2(tot[0].x, tot[1].x);             // (n0, z), (n0, z+1)
        }
      }
      pg = pe;
    }
  }
  __syncthreads();
  if (un.len >= 1 && live) gather(un.len & 1);

  if (OUT == OUT_APPLY_DOT || OUT == OUT_JACOBI_DOT) {
    double v[1] = {acc};
    block_reduce<1>(v, red);
    if (tid == 0) a.partials[(long long)un.slot * kNumRhs + rhs] = v[0];
  }
}

// ------------------------------------------------ bulk-copy staging ---
// mbarrier + cp.async.bulk helpers (PTX; addresses are shared-window offsets).
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for a phase of an mbarrier: false if it did not complete
// within `limit` try_wait rounds (each also suspends for a while).
constexpr int kWaitLimit = 1 << 20;
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int limit = kWaitLimit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Stage wait of the staged kernels: the compile-time bound above, except that
// every wait gives up at once when give_up (FEMH_STAGE_WAIT_LIMIT=0, tests of
// the timeout path) is set.  A flag test rather than a runtime round limit:
// the kernels run at their register cap, and a runtime loop bound made the
// FP64 one spill.
__device__ __forceinline__ bool mbar_wait_stage(unsigned bar, unsigned parity, int give_up) {
  if (give_up) return false;
  return mbar_wait(bar, parity);
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// stencil2p_kernel with its inputs staged by bulk copies (FP32 storage).  A
// stage holds, for step s (voxel plane ie = i0-1+s), node plane ie+1 of u
// (node rows j0-1 .. j0+rows+1), voxel plane ie of kc (voxel rows j0-1 ..
// j0+rows) and, for the gather of node plane ie-1, b and invd of the owned
// node rows j0 .. j0+rows-1.  Rows of the z ring are contiguous in memory, so
// a stage is a handful of row-segment copies (split where y wraps) that the
// lanes of warp 0 issue against one mbarrier.  A ring of kBulkSlots stages
// runs kBulkSlots-1 steps ahead of the one in use; no per-thread loads of
// inputs remain.
// Work of a CTA: one unit (a.cta_units == nullptr), or the run of units
// [cta_units[b], cta_units[b+1]) as a persistent CTA.  Units that continue
// each other along x (same cell and rows, adjacent x ranges) form one stream:
// the carried planes pass from one unit to the next, so only a change of tile
// pays the pipeline's fill (three stages) again.  The dot partial sums stay
// per unit (written when a unit's last node plane is gathered), so results
// are the same bits as one CTA per unit.  Stage g of a stream uses ring slot
// (gbase + g) % kBulkSlots, gbase = stages of the CTA's earlier streams.
// Requirements (checked by the host): nz % 4 == 0 on every cell, 16-byte
// aligned arrays.  A tile has at most ny rows, so an array spans at most three
// row segments: at most 20 copies per stage, one per lane of warp 0.
constexpr int kBulkSlots = 4;

template <int NT, int OUT, int NZ>
__global__ void __launch_bounds__(NT, 1)
stencil2b_kernel(StencilArgs<float, float, float, float> a) {
  static_assert(NZ > 0 && NZ % 4 == 0, "staged rows need a compile-time z extent, multiple of 4");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rhs = blockIdx.y;
  int kb = blockIdx.x, ke = blockIdx.x + 1;   // units of this CTA: [kb, ke)
  if (a.cta_units) {
    kb = a.cta_units[blockIdx.x];
    ke = a.cta_units[blockIdx.x + 1];
  }
  constexpr int nz = NZ;
  constexpr int TR = NT / NZ;
  const int tid = threadIdx.x;
  const int t = tid / nz, z = tid - t * nz;
  const int zp = (z + 1 == nz) ? 0 : z + 1;
  const int zm = (z == 0) ? nz - 1 : z - 1;

  constexpr int RB = 2 * TR - 1, NRU = RB + 3, NRK = RB + 2;
  // stage layout (floats): U[3][NRU][nz], KC[NRK][nz], B[3][RB][nz], I[RB][nz][6]
  // (invd rows, or the node-block inverses [6] of a block sweep)
  constexpr int oK = 3 * NRU * NZ, oB = oK + NRK * NZ, oI = oB + 3 * RB * NZ;
  constexpr int SS = (oI + 6 * RB * NZ + 3) & ~3;
  constexpr int PS = TR * 3 * nz;
  float* stg = reinterpret_cast<float*>(smem_raw);
  f2* QAB = reinterpret_cast<f2*>(stg + kBulkSlots * SS);   // [2][TR][3][nz]
  f2* QCD = QAB + 2 * PS;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(QCD + 2 * PS);
  double* red = reinterpret_cast<double*>(bars + kBulkSlots);
  __shared__ int abort_flag;
  const int pt = t * 3 * nz;
  const int pa = (t + 1 < TR ? t + 1 : t) * 3 * nz;
  const long long st = a.ntot;

  if (tid == 0) {
    for (int k = 0; k < kBulkSlots; ++k) mbar_init(smem_addr(bars + k), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  unsigned gbase = 0;   // stages of the earlier streams (slot and phase of stage g: gbase + g)
  for (int k = kb; k < ke;) {
    const StencilUnit un = a.units[k];
    const CellDesc cd = a.cells[un.cell];
    int k2 = k + 1, len = un.len;
    while (k2 < ke) {
      const StencilUnit v = a.units[k2];
      if (v.cell != un.cell || v.j0 != un.j0 || v.rows != un.rows || v.i0 != un.i0 + len) break;
      len += v.len;
      ++k2;
    }
    if (a.stt && !a.stt[cd.id * kNumRhs + rhs].active) {
      k = k2;
      continue;
    }
    const int nx = cd.nx, ny = cd.ny;
    const int rows = un.rows;
    const bool live = t < TR && 2 * t <= rows;
    const bool own1 = live && 2 * t < rows;
    const bool own2 = live && 2 * t + 1 < rows;
    auto wrapy = [&](int j) { j %= ny; return j < 0 ? j + ny : j; };
    const int n1 = wrapy(un.j0 + 2 * t), n2 = wrapy(un.j0 + 2 * t + 1);
    const int plane = ny * nz;
    const int c1 = n1 * nz + z, c2 = n2 * nz + z;
    float* obase = a.out + (long long)rhs * 3 * st + cd.off;

    const char* src_base = nullptr;
    int plane_lag = 0, src_off = 0, dst_off = 0, bytes = 0, esz = 4;
    unsigned tx_total = 0;
    if (tid < 32) {
      int idx = 0;
      // es: bytes per node of the array (4, or 24 for the node blocks)
      auto seg = [&](const float* base, int lag, int row0, int nrows, int dst, int es = 4) {
        int done = 0;
        while (done < nrows) {
          const int r0 = wrapy(row0 + done);
          const int n = min(nrows - done, ny - r0);
          if (idx == tid) {
            src_base = reinterpret_cast<const char*>(base);
            plane_lag = lag;
            esz = es;
            src_off = r0 * nz;
            dst_off = dst + done * nz * (es / 4);
            bytes = n * nz * es;
          }
          tx_total += (unsigned)(n * nz * es);
          ++idx;
          done += n;
        }
      };
      for (int c = 0; c < 3; ++c)
        seg(a.u + ((long long)rhs * 3 + c) * st + cd.off, 1, un.j0 - 1, rows + 3, c * NRU * nz);
      seg(a.kc + cd.off, 0, un.j0 - 1, rows + 2, oK);
      if (OUT >= OUT_JACOBI) {
        for (int c = 0; c < 3; ++c)
          seg(a.b + ((long long)rhs * 3 + c) * st + cd.off, -1, un.j0, rows, oB + c * RB * nz);
        if (OUT != OUT_RESID) {
          if (a.binv) seg(a.binv + 6 * cd.off, -1, un.j0, rows, oI, 24);
          else seg(a.invd + cd.off, -1, un.j0, rows, oI);
        }
      }
    }
    int pl_next = ((un.i0 - 2 + plane_lag) % nx + nx) % nx;
    int issued = 0;
    auto issue = [&](int g) {
      issued = g + 1;
      const unsigned gg = gbase + (unsigned)g;
      const int slot = (int)(gg % kBulkSlots);
      const unsigned bar = smem_addr(bars + slot);
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, tx_total);
      }
      __syncwarp();
      if (bytes > 0)
        bulk_g2s(smem_addr(stg + slot * SS + dst_off),
                 src_base + (long long)esz * ((long long)pl_next * plane + src_off), (unsigned)bytes, bar);
      if (++pl_next == nx) pl_next = 0;
    };
    const int G = len + 3;
    if (tid < 32)
      for (int g = 0; g < kBulkSlots && g < G; ++g) issue(g);
    int waited = 0;
    auto wait_stage = [&](int g) {
      const unsigned gg = gbase + (unsigned)g;
      if (!mbar_wait_stage(smem_addr(bars + gg % kBulkSlots), (gg / kBulkSlots) & 1u, a.wait_limit == 0)) {
        if (a.err) atomicExch(a.err, 1);
        abort_flag = 1;
      } else if (waited == g) {
        waited = g + 1;
      }
    };

    f2 prv[3][4], car[3][4];
    f2 own[3], u12[3], raw[3];
    int pg = 0;
    double acc = 0.0;
    int ku = k, kend = un.len;   // unit of the gathered planes, and its end (plane index in the stream)
#pragma unroll
    for (int c = 0; c < 3; ++c) own[c] = u12[c] = raw[c] = p_bc(0.f);

    auto patch = [&](const float* U, f2 (&h)[3][4], f2 (&mine)[3]) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* Uc = U + c * NRU * nz;
        const int r0 = (2 * t) * nz;
        mine[c] = make_float2(Uc[r0 + nz + z], Uc[r0 + 2 * nz + z]);
        const f2 up = make_float2(Uc[r0 + nz + zp], Uc[r0 + 2 * nz + zp]);
        h[c][0] = make_float2(Uc[r0 + z], mine[c].x);
        h[c][1] = make_float2(Uc[r0 + zp], up.x);
        h[c][2] = mine[c];
        h[c][3] = up;
        had4_fwd(h[c]);
      }
    };
    auto gather = [&](int buf, const float* S) {
      const f2* Qab = QAB + buf * PS;
      const f2* Qcd = QCD + buf * PS;
      f2 y[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        y[c] = p_add(own[c], Qab[pt + c * nz + zm]);
        y[c].y += Qcd[pa + c * nz + z].x + Qcd[pa + c * nz + zm].y;
      }
      float* ob = obase + pg;
      const int r1 = (2 * t) * nz + z, r2 = r1 + nz;
      if (OUT == OUT_APPLY || OUT == OUT_APPLY_DOT) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (own1) ob[c * st + c1] = y[c].x;
          if (own2) ob[c * st + c2] = y[c].y;
          if (OUT == OUT_APPLY_DOT) {
            if (own1) acc += (double)u12[c].x * (double)y[c].x;
            if (own2) acc += (double)u12[c].y * (double)y[c].y;
          }
        }
      } else {
        const bool pin1 = (pg + c1 == 0), pin2 = (pg + c2 == 0);
        const float* Bs = S + oB;
        // rows beyond the tile read stale stage entries: their lanes are not stored
        f2 bv[3], d[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          bv[c] = make_float2(Bs[c * RB * NZ + r1], Bs[c * RB * NZ + r2]);
          d[c] = p_sub(bv[c], y[c]);
        }
        if (OUT == OUT_RESID) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (own1) ob[c * st + c1] = pin1 ? 0.f : d[c].x;
            if (own2) ob[c * st + c2] = pin2 ? 0.f : d[c].y;
          }
        } else {
          const float* Is = S + oI;
          f2 wd;
          if (a.binv) {   // node-block sweep: d <- B d of both nodes
            block_dir2(Is + 6 * r1, Is + 6 * r2, d);
            wd = p_bc((float)a.omega);
          } else {
            wd = p_mul(p_bc((float)a.omega), make_float2(Is[r1], Is[r2]));
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const f2 xv = p_fma(wd, d[c], u12[c]);
            if (own1) ob[c * st + c1] = xv.x;
            if (own2) ob[c * st + c2] = xv.y;
            if (OUT == OUT_JACOBI_DOT) {
              if (own1) acc += (double)xv.x * (double)bv[c].x;
              if (own2) acc += (double)xv.y * (double)bv[c].y;
            }
          }
        }
      }
    };

    wait_stage(0);
    if (live) {
      f2 mine[3];
      patch(stg + (gbase % kBulkSlots) * SS, prv, mine);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        raw[c] = mine[c];
#pragma unroll
        for (int q = 0; q < 4; ++q) car[c][q] = p_bc(0.f);
      }
    }
    const int cellsz = nx * plane;
    int pe_next = ((un.i0 - 1 + nx) % nx) * plane;
    for (int s = 0; s <= len + 1; ++s) {
      const int g = s + 1;
      wait_stage(g);
      __syncthreads();
      if (abort_flag) break;
      if (tid < 32 && g + kBulkSlots - 1 < G) issue(g + kBulkSlots - 1);
      const float* S = stg + ((gbase + (unsigned)g) % kBulkSlots) * SS;
      const int pe = pe_next;
      pe_next += plane;
      if (pe_next >= cellsz) pe_next -= cellsz;
      if (s >= 2) {
        if (live) gather((s - 1) & 1, S);
        if (OUT == OUT_APPLY_DOT || OUT == OUT_JACOBI_DOT) {
          if (s - 1 == kend) {   // gathered plane s-2 was the last one of unit ku
            double v[1] = {acc};
            block_reduce<1>(v, red);
            if (tid == 0) a.partials[(long long)a.units[ku].slot * kNumRhs + rhs] = v[0];
            acc = 0.0;
            if (++ku < k2) kend += a.units[ku].len;
          }
        }
      }
      if (s > len || !live) continue;
      f2 w[3][8];
      f2 cur0[3];
      {
        f2 cur[3][4];
        patch(S, cur, cur0);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (q > 0) w[c][q] = p_add(cur[c][q], prv[c][q]);
            w[c][4 + q] = p_sub(cur[c][q], prv[c][q]);
            prv[c][q] = cur[c][q];
          }
      }
      {
        const float* K = S + oK + (2 * t) * nz + z;
        const f2 kv = make_float2(K[0], K[nz]);
        const f2 A = p_mul(kv, a.kp[0]), Bdo = p_mul(kv, a.kp[1]), Bo = p_mul(kv, a.kp[2]);
        const f2 D1o = p_mul(kv, a.kp[3]), O1 = p_mul(kv, a.kp[4]);
        const f2 D2o = p_mul(kv, a.kp[5]), O2 = p_mul(kv, a.kp[6]), Gd = p_mul(kv, a.kp[7]);
        {
          const f2 m0 = w[0][4], m1 = w[1][2], m2 = w[2][1];
          const f2 tt = p_mul(Bo, p_add(p_add(m0, m1), m2));
          w[0][4] = p_fma(Bdo, m0, tt); w[1][2] = p_fma(Bdo, m1, tt); w[2][1] = p_fma(Bdo, m2, tt);
        }
        {
          const f2 sxz = p_mul(A, p_add(w[0][1], w[2][4]));
          const f2 syz = p_mul(A, p_add(w[1][1], w[2][2]));
          const f2 sxy = p_mul(A, p_add(w[0][2], w[1][4]));
          w[0][1] = sxz; w[2][4] = sxz; w[1][1] = syz; w[2][2] = syz; w[0][2] = sxy; w[1][4] = sxy;
        }
        {
          const f2 m0 = w[0][3], m1 = w[1][5], m2 = w[2][6];
          const f2 tt = p_mul(O1, p_add(p_add(m0, m1), m2));
          w[0][3] = p_fma(D1o, m0, tt); w[1][5] = p_fma(D1o, m1, tt); w[2][6] = p_fma(D1o, m2, tt);
        }
        {
          const f2 x0 = w[1][3], x1 = w[0][5], tt = p_mul(O2, p_add(x0, x1));
          w[1][3] = p_fma(D2o, x0, tt); w[0][5] = p_fma(D2o, x1, tt);
        }
        {
          const f2 x0 = w[2][3], x1 = w[0][6], tt = p_mul(O2, p_add(x0, x1));
          w[2][3] = p_fma(D2o, x0, tt); w[0][6] = p_fma(D2o, x1, tt);
        }
        {
          const f2 x0 = w[2][5], x1 = w[1][6], tt = p_mul(O2, p_add(x0, x1));
          w[2][5] = p_fma(D2o, x0, tt); w[1][6] = p_fma(D2o, x1, tt);
        }
        w[0][7] = p_mul(w[0][7], Gd); w[1][7] = p_mul(w[1][7], Gd); w[2][7] = p_mul(w[2][7], Gd);
      }
      f2* Qab = QAB + (s & 1) * PS;
      f2* Qcd = QCD + (s & 1) * PS;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        f2 tot[4];
        tot[0] = p_sub(car[c][0], w[c][4]);
        car[c][0] = w[c][4];
#pragma unroll
        for (int q = 1; q < 4; ++q) {
          tot[q] = p_add(p_sub(w[c][q], w[c][4 + q]), car[c][q]);
          car[c][q] = p_add(w[c][q], w[c][4 + q]);
        }
        had4_inv(tot);
        own[c] = make_float2(tot[0].y + tot[2].x, tot[2].y);
        u12[c] = raw[c];
        raw[c] = cur0[c];
        if (s > 0) {
          Qab[pt + c * nz + z] = make_float2(tot[1].y + tot[3].x, tot[3].y);
          Qcd[pt + c * nz + z] = make_float2(tot[0].x, tot[1].x);
        }
      }
      pg = pe;
    }
    if (abort_flag) {   // drain this stream's outstanding stages (bounded) and stop
      if (tid == 0)
        for (int g = waited; g < issued; ++g) {
          const unsigned gg = gbase + (unsigned)g;
          if (!mbar_wait(smem_addr(bars + gg % kBulkSlots), (gg / kBulkSlots) & 1u)) break;
        }
      break;
    }
    gbase += (unsigned)G;
    k = k2;
    __syncthreads();   // every read of this stream's stages and Q buffers is done before the next issues
  }
}

// Scalar 2x2 Hadamard transform of a node patch and its inverse (same stage
// order and signs as had4_fwd / had4_inv).
template <typename T>
__device__ __forceinline__ void had4s_fwd(T (&v)[4]) {
  const T a0 = v[1] + v[0], a1 = v[1] - v[0], a2 = v[3] + v[2], a3 = v[3] - v[2];
  v[0] = a2 + a0; v[2] = a2 - a0; v[1] = a3 + a1; v[3] = a3 - a1;
}
template <typename T>
__device__ __forceinline__ void had4s_inv(T (&v)[4]) {
  const T a0 = v[0] - v[2], a2 = v[0] + v[2], a1 = v[1] - v[3], a3 = v[1] + v[3];
  v[0] = a0 - a1; v[1] = a0 + a1; v[2] = a2 - a3; v[3] = a2 + a3;
}

// FP64 operator, one voxel row per thread, inputs staged by bulk copies.
// Schedule and staging of stencil2b_kernel (stage g = step g-1; u of node
// plane ie+1, kc of voxel plane ie, b / invd of node plane ie-1), the
// carried lower plane transformed in y and z and the upper-plane
// contributions half transformed (as in stencilp_kernel), arithmetic in FP64.
// Thread (r, z) streams voxel (i, j0-1+r, z); row 0 is the y halo.  Stage
// layout: U[3][R+1][nz] (TIn), KC[R][nz], B[3][R-1][nz] (double), ID[R-1][nz]
// (float); Q[2][R][3 corners][3][nz] doubles.
template <int NT, int OUT, int NZ, typename TIn>
__global__ void __launch_bounds__(NT, 1)
stencil1b_kernel(StencilArgs<TIn, double, double, double> a) {
  static_assert(NZ > 0 && NZ % 4 == 0, "staged rows need a compile-time z extent, multiple of 4");
  constexpr int R = NT / NZ, NRU = R + 1, NRK = R, RB = R - 1;
  constexpr int bU = 0, bK = bU + 3 * NRU * NZ * (int)sizeof(TIn), bB = bK + NRK * NZ * 8,
                bI = bB + 3 * RB * NZ * 8;
  constexpr int SSB = (bI + RB * NZ * 4 + 15) & ~15;   // bytes per stage
  constexpr int QS = R * 9 * NZ;                       // doubles per Q buffer
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const StencilUnit un = a.units[blockIdx.x];
  const int rhs = blockIdx.y;
  const CellDesc cd = a.cells[un.cell];
  if (a.stt && !a.stt[cd.id * kNumRhs + rhs].active) return;
  const int nx = cd.nx, ny = cd.ny;
  constexpr int nz = NZ;
  const int tid = threadIdx.x;
  const int r = tid / nz, z = tid - r * nz;
  const int rows = un.rows;
  const bool live = r <= rows;
  const bool owner = live && r >= 1;
  const int zp = (z + 1 == nz) ? 0 : z + 1;
  const int zm = (z == 0) ? nz - 1 : z - 1;
  auto wrapy = [&](int j) { j %= ny; return j < 0 ? j + ny : j; };
  const int jr = wrapy(un.j0 - 1 + r);

  unsigned char* stg = smem_raw;
  double* Q = reinterpret_cast<double*>(stg + kBulkSlots * SSB);   // [2][R][3][3][nz]
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(Q + 2 * QS);
  double* red = reinterpret_cast<double*>(bars + kBulkSlots);
  __shared__ int abort_flag;
  const int qrow = r * 9 * nz, qup = (r > 0 ? r - 1 : 0) * 9 * nz;

  const long long st = a.ntot;
  const int plane = ny * nz;
  const int col = jr * nz + z;
  double* obase = a.out + (long long)rhs * 3 * st + cd.off;

  const char* src_base = nullptr;
  int plane_lag = 0, src_off = 0, dst_off = 0, bytes = 0, esz = 0;
  unsigned tx_total = 0;
  if (tid < 32) {
    int idx = 0;
    auto seg = [&](const void* base, int es, int lag, int row0, int nrows, int dst) {
      int done = 0;
      while (done < nrows) {
        const int r0 = wrapy(row0 + done);
        const int n = min(nrows - done, ny - r0);
        if (idx == tid) {
          src_base = reinterpret_cast<const char*>(base);
          esz = es;
          plane_lag = lag;
          src_off = r0 * nz;
          dst_off = dst + done * nz * es;
          bytes = n * nz * es;
        }
        tx_total += (unsigned)(n * nz * es);
        ++idx;
        done += n;
      }
    };
    for (int c = 0; c < 3; ++c)
      seg(a.u + ((long long)rhs * 3 + c) * st + cd.off, (int)sizeof(TIn), 1, un.j0 - 1, rows + 2,
          bU + c * NRU * nz * (int)sizeof(TIn));
    seg(a.kc + cd.off, 8, 0, un.j0 - 1, rows + 1, bK);
    if (OUT >= OUT_JACOBI) {
      for (int c = 0; c < 3; ++c) seg(a.b + ((long long)rhs * 3 + c) * st + cd.off, 8, -1, un.j0, rows, bB + c * RB * nz * 8);
      if (OUT != OUT_RESID && !a.binv) seg(a.invd + cd.off, 4, -1, un.j0, rows, bI);
    }
  }
  int pl_next = ((un.i0 - 2 + plane_lag) % nx + nx) % nx;
  int issued = 0;
  auto issue = [&](int g) {
    issued = g + 1;
    const int slot = g % kBulkSlots;
    const unsigned bar = smem_addr(bars + slot);
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(bar, tx_total);
    }
    __syncwarp();
    if (bytes > 0)
      bulk_g2s(smem_addr(stg + slot * SSB + dst_off), src_base + (long long)esz * ((long long)pl_next * plane + src_off),
               (unsigned)bytes, bar);
    if (++pl_next == nx) pl_next = 0;
  };
  const int G = un.len + 3;
  if (tid == 0) {
    for (int k = 0; k < kBulkSlots; ++k) mbar_init(smem_addr(bars + k), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid < 32)
    for (int g = 0; g < kBulkSlots && g < G; ++g) issue(g);
  int waited = 0;   // stages 0 .. waited-1 completed for this thread (the exit drain starts there)
  auto wait_stage = [&](int g) {
    if (!mbar_wait_stage(smem_addr(bars + g % kBulkSlots), (unsigned)((g / kBulkSlots) & 1), a.wait_limit == 0)) {
      if (a.err) atomicExch(a.err, 1);
      abort_flag = 1;
    } else if (waited == g) {
      waited = g + 1;   // a stage that timed out stays owed to the drain
    }
  };

  double prv[3][4], car[3][4];
  double own[3] = {0, 0, 0}, unode[3] = {0, 0, 0}, rawn[3] = {0, 0, 0};
  int pg = 0;
  double acc = 0.0;
  auto patch = [&](const unsigned char* S, double (&h)[3][4], double (&mine)[3]) {
    const TIn* U = reinterpret_cast<const TIn*>(S + bU);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const TIn* Uc = U + c * NRU * nz + r * nz;
      mine[c] = (double)Uc[z];
      h[c][0] = mine[c];
      h[c][1] = (double)Uc[zp];
      h[c][2] = (double)Uc[nz + z];
      h[c][3] = (double)Uc[nz + zp];
      had4s_fwd(h[c]);
    }
  };
  auto gather = [&](int buf, const unsigned char* S) {
    const double* Qg = Q + buf * QS;
    double* ob = obase + pg + col;
    const int rb = (r - 1) * nz + z;   // owned row in the b / invd arrays
    const bool pin = (pg + col == 0);
    const double* Bs = reinterpret_cast<const double*>(S + bB);
    double y[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      y[c] = own[c] + Qg[qrow + (0 * 3 + c) * nz + zm] + Qg[qup + (1 * 3 + c) * nz + z] + Qg[qup + (2 * 3 + c) * nz + zm];
    if (OUT == OUT_APPLY || OUT == OUT_APPLY_DOT) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ob[c * st] = y[c];
        if (OUT == OUT_APPLY_DOT) acc += unode[c] * y[c];
      }
    } else if (OUT == OUT_RESID) {
#pragma unroll
      for (int c = 0; c < 3; ++c) ob[c * st] = pin ? 0.0 : Bs[c * RB * nz + rb] - y[c];
    } else {
      const float* Is = reinterpret_cast<const float*>(S + bI);
      double dv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) dv[c] = Bs[c * RB * nz + rb] - y[c];
      if (a.binv) {   // node-block sweep: the node's block inverse, read where the gather needs it
        jacobi_dir<double>(a.binv, cd.off + pg + col, 0.0, dv);
#pragma unroll
        for (int c = 0; c < 3; ++c) dv[c] *= a.omega;
      } else {
        const double idv = a.omega * (double)Is[rb];
#pragma unroll
        for (int c = 0; c < 3; ++c) dv[c] *= idv;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double xv = unode[c] + dv[c];
        ob[c * st] = xv;
        if (OUT == OUT_JACOBI_DOT) acc += xv * Bs[c * RB * nz + rb];
      }
    }
  };

  wait_stage(0);
  if (live) {
    double mine[3];
    patch(stg, prv, mine);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      rawn[c] = mine[c];
#pragma unroll
      for (int q = 0; q < 4; ++q) car[c][q] = 0.0;
    }
  }
  const int cellsz = nx * plane;
  int pe_next = ((un.i0 - 1 + nx) % nx) * plane;
  for (int s = 0; s <= un.len + 1; ++s) {
    const int g = s + 1;
    wait_stage(g);
    __syncthreads();
    if (abort_flag) break;
    if (tid < 32 && g + kBulkSlots - 1 < G) issue(g + kBulkSlots - 1);
    const unsigned char* S = stg + (g % kBulkSlots) * SSB;
    const int pe = pe_next;
    pe_next += plane;
    if (pe_next >= cellsz) pe_next -= cellsz;
    if (s >= 2 && owner) gather((s - 1) & 1, S);
    if (s > un.len || !live) continue;
    double w[3][8];
    double cur0[3];
    {
      double cur[3][4];
      patch(S, cur, cur0);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          w[c][q] = cur[c][q] + prv[c][q];
          w[c][4 + q] = cur[c][q] - prv[c][q];
          prv[c][q] = cur[c][q];
        }
    }
    had_block(w, a.k, reinterpret_cast<const double*>(S + bK)[r * nz + z]);
    double* Qb = Q + (s & 1) * QS;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double tot[4];
      tot[0] = car[c][0] - w[c][4];
      car[c][0] = w[c][4];
#pragma unroll
      for (int q = 1; q < 4; ++q) {
        tot[q] = (w[c][q] - w[c][4 + q]) + car[c][q];
        car[c][q] = w[c][q] + w[c][4 + q];
      }
      had4s_inv(tot);
      own[c] = tot[0];
      unode[c] = rawn[c];
      rawn[c] = cur0[c];
      if (s > 0) {
        Qb[qrow + (0 * 3 + c) * nz + z] = tot[1];   // node (jr, z+1)
        Qb[qrow + (1 * 3 + c) * nz + z] = tot[2];   // node (jr+1, z)
        Qb[qrow + (2 * 3 + c) * nz + z] = tot[3];   // node (jr+1, z+1)
      }
    }
    pg = pe;
  }
  if (tid == 0) {
    for (int g = waited; g < issued; ++g)
      if (!mbar_wait(smem_addr(bars + g % kBulkSlots), (unsigned)((g / kBulkSlots) & 1))) break;
  }
  if (OUT == OUT_APPLY_DOT || OUT == OUT_JACOBI_DOT) {
    double v[1] = {acc};
    block_reduce<1>(v, red);
    if (tid == 0) a.partials[(long long)un.slot * kNumRhs + rhs] = v[0];
  }
}

// Shared memory bytes of one stencil1b_kernel CTA.
inline size_t stencil1b_smem_bytes(int NT, int nz, int in_size) {
  const int R = NT / nz;
  const size_t stage = ((size_t)3 * (R + 1) * nz * in_size + (size_t)R * nz * 8 + (size_t)3 * (R - 1) * nz * 8 +
                        (size_t)(R - 1) * nz * 4 + 15) & ~(size_t)15;
  return kBulkSlots * stage + sizeof(double) * 2 * (size_t)R * 9 * nz + sizeof(unsigned long long) * kBulkSlots +
         64 * sizeof(double);
}

// Shared memory bytes of one stencil2b_kernel CTA (tiles of up to 2*TR-1 rows).
inline size_t stencil2b_smem_bytes(int NT, int nz) {
  const int TR = NT / nz, rows = 2 * TR - 1;
  const size_t SS = ((size_t)(3 * (rows + 3) + (rows + 2) + 9 * rows) * nz + 3) & ~(size_t)3;   // as in the kernel
  return sizeof(float) * kBulkSlots * SS + sizeof(f2) * 4 * (size_t)TR * 3 * nz +
         sizeof(unsigned long long) * kBulkSlots + 64 * sizeof(double);
}

// Shared memory bytes of one stencil2p_kernel CTA.
inline size_t stencil2p_smem_bytes(int NT, int nz) {
  const int TR = NT / nz;
  return sizeof(f2) * 6 * (size_t)TR * 3 * nz + sizeof(float) * ((6 * (size_t)nz + 1) & ~(size_t)1) +
         64 * sizeof(double);
}

// Shared memory bytes of one pair-kernel CTA.
inline size_t stencilp_smem_bytes(int NT, int nz) {
  const int R = NT / nz;
  return sizeof(float4) * 12 * (size_t)NT + sizeof(f2) * 2 * ((size_t)(R + 1) * 3 * nz + (size_t)R * 9 * nz) +
         64 * sizeof(double);
}

}  // namespace femh
