// femh_common.cuh -- shared device-side types of the femh homogenization engine.
//
// Grid conventions (same as the reference, desaic/fem):
//   voxel / node index (i*ny + j)*nz + k, x slowest, z fastest
//   (fast_fem/ArrayUtil.cpp gridToLinearIdx); voxel (i,j,k) has lower corner
//   node (i,j,k); local node a = 4*ax + 2*ay + az (the `oneV` order of
//   fast_fem/FEM3DFun.cpp:58-60); DOF 3*a + c.
// Device vector layout (engine-internal): [rhs][comp][node], the node range of
// every cell of a level packed one after another ("plane stride" = nodes of
// the level over all cells).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace femh {

constexpr int kNumRhs = 6;

// One periodic cell at one multigrid level.
struct CellDesc {
  int nx, ny, nz;
  int id;            // cell index in the batch (indexes per-cell state)
  int parent;        // index of this cell in the next finer level's table (-1 at the finest)
  int child;         // index in the next coarser level's table (-1 at the cell's coarsest level)
  long long off;     // first node (= first voxel) of this cell in the level arrays
  double h;          // voxel edge at this level
};

// One CTA of the stencil kernel: rows [j0, j0+rows) x planes [i0, i0+len) of a cell.
struct StencilUnit {
  int cell;   // index into the level's CellDesc table
  int j0, rows;
  int i0, len;
  int slot;   // partial-sum slot of this unit inside its cell
};

// Node-parallel work of vector kernels: a contiguous node range of one cell.
struct NodeUnit {
  int cell;
  int slot;
  long long begin, end;   // node range relative to the cell
};

// The element stiffness of a unit cube (E = 1, h = 1) in the Hadamard basis of
// the 2x2x2 node cube.  u_hat_c(k) = sum_a chi_k(a) u_{a,c}, chi_k(a) =
// prod_s (2*bit_s(a)-1)^bit_s(k).  K0 = T^T Kh T with T = H8 (x) I3 and Kh
// block-sparse with 45 nonzeros; these eight numbers are its distinct values
// (derived on the host from the Gauss-integrated K0 and checked there).
struct HadK {
  double A;    // shear pairs  (k=1,c=x)-(k=4,c=z), (1,y)-(2,z), (2,x)-(4,y)
  double Bd;   // normal triple diagonal (4,x),(2,y),(1,z)
  double Bo;   // normal triple off-diagonal
  double D1;   // mixed triple diagonal (3,x),(5,y),(6,z)
  double O1;   // mixed triple off-diagonal
  double D2;   // mixed pairs diagonal (3,y)-(5,x), (3,z)-(6,x), (5,z)-(6,y)
  double O2;   // mixed pairs off-diagonal
  double G;    // k=7 (xyz mixed) diagonal
  double diag; // K0 diagonal entry (all 24 equal for the cube)
};

// Per (cell, load case) CG state, kept on the device so that iterations can be
// captured in a CUDA graph without host round trips.
struct CGState {
  double rz, pq, alpha, beta, rr, bnorm2, rel, scale;
  int iters, active, status, max_iter;
  double tol;
  int outer;        // defect correction: this (cell, rhs) takes part in the current outer step
  int fallback;     // 1: the multigrid preconditioner turned indefinite; Jacobi from then on
  double best;      // smallest relative residual so far (inner solves of defect correction)
  int since;        // iterations since it last halved
};
// An inner (FP32) solve of defect correction stops when its residual has not
// halved for this many iterations: it has reached what its arithmetic resolves,
// and the next outer step (FP64 residual) continues from there.
constexpr int kInnerStallWindow = 200;
// CG_BLOCK_FAIL: a block PCG step matrix turned indefinite; the cell's load
// cases are solved again one at a time.
enum CGStatus : int { CG_RUNNING = 0, CG_CONVERGED = 1, CG_MAXITER = 2, CG_BREAKDOWN = 3, CG_BLOCK_FAIL = 4 };

template <typename T> struct VT { using type = T; };

__device__ __forceinline__ double ld_val(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ld_val(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ld_val(const __nv_bfloat16* p) {
  return __bfloat162float(*p);
}
__device__ __forceinline__ void st_val(double* p, double v) { *p = v; }
__device__ __forceinline__ void st_val(float* p, float v) { *p = v; }
__device__ __forceinline__ void st_val(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

// Damped-Jacobi direction at one node: d <- D^-1 d, D the point diagonal
// (inverse id, the same for the 3 components) or, with binv != nullptr, the
// node's 3x3 diagonal block of K (node-block Jacobi; the symmetric inverse
// [xx, yy, zz, xy, xz, yz] stored at binv + 6 g, 8-byte aligned).
template <typename T>
__device__ __forceinline__ void jacobi_dir(const float* __restrict__ binv, long long g, T id, T (&d)[3]) {
  if (binv) {
    const float2 b01 = *reinterpret_cast<const float2*>(binv + 6 * g);
    const float2 b23 = *reinterpret_cast<const float2*>(binv + 6 * g + 2);
    const float2 b45 = *reinterpret_cast<const float2*>(binv + 6 * g + 4);
    const T xx = (T)b01.x, yy = (T)b01.y, zz = (T)b23.x, xy = (T)b23.y, xz = (T)b45.x, yz = (T)b45.y;
    const T d0 = d[0], d1 = d[1], d2 = d[2];
    d[0] = xx * d0 + xy * d1 + xz * d2;
    d[1] = xy * d0 + yy * d1 + yz * d2;
    d[2] = xz * d0 + yz * d1 + zz * d2;
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] *= id;
  }
}

// Warp + block reduction of nv doubles; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* smem /* >= 32*NV */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) smem[warp * NV + q] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = (lane < nwarps) ? smem[lane * NV + q] : 0.0;
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
}

}  // namespace femh
