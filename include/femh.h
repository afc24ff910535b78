/*
 * femh.h -- C ABI of the B200 voxel-FEM homogenization engine (libfemh.so).
 *
 * The engine computes the homogenized 6x6 elasticity tensor C^H of periodic
 * voxel cells (trilinear hex8 elements, one shared element stiffness scaled
 * per voxel), its density gradient, and batches of cells of uneven size, on
 * one NVIDIA B200 (sm_100a).  It replaces the solve + energy reduction behind
 * the reference's homogenization calls (desaic/fem):
 *   - fast_fem FEM3DFun::setParam / f / df           (fast_fem/FEM3DFun.cpp:128-268,
 *     RealFun virtuals fast_fem/RealFun.hpp:29-36), which drive topoOptLib's
 *     Homogenization<3>::Homogenize() (fast_fem/FEM3DFun.cpp:153-154);
 *   - NumericalCoarseningUsingMultigrid::computeCoarsenedElasticityTensorAndParameters3D
 *     (SamplesGenerator/NumericalCoarseningUsingMultigrid.h:27-30,
 *      SamplesGenerator/NumericalCoarseningUsingMultiGrid.cpp:221-345).
 *
 * Conventions
 *   - voxel index (i*ny + j)*nz + k (x slowest, z fastest), the reference's
 *     gridToLinearIdx / getGridToVectorIndex (Utilities/src/cfgMaterialUtilities.cpp:1003-1007);
 *   - Voigt order xx, yy, zz, yz, xz, xy with engineering shear
 *     (MaterialOpt/src/Homogenize3D.cpp:196-201, femlib/src/MeshUtilities.cpp:852-857);
 *   - C_out is row-major 6x6 and symmetric (the reference fills only the
 *     upper triangle of its G, fast_fem/FEM3DFun.cpp:163-178; both halves here);
 *   - lower-triangle order of 21-entry outputs: (0,0),(1,0),(1,1),(2,0),...
 *     (the order NumericalCoarseningUsingMultiGrid.cpp:315-324 appends);
 *   - node 0 of every cell is pinned (removes the 3 translations); C^H does not
 *     depend on that choice.
 * Threading: one handle = one CUDA stream; calls on one handle are serialised
 * by the caller; different handles are independent.
 * Ownership: inputs and outputs belong to the caller; the handle keeps its own
 * copies of the solved fields for the gradient calls.
 * Errors: every function returns a femh_status; femh_last_error() gives text.
 */
#ifndef FEMH_H
#define FEMH_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int femh_status;
enum {
  FEMH_OK = 0,
  FEMH_E_ARG = 1,            /* invalid argument (sizes, pointers, config) */
  FEMH_E_CUDA = 2,           /* CUDA runtime error */
  FEMH_E_OOM = 3,            /* device allocation failed */
  FEMH_E_NOT_CONVERGED = 4,  /* max_iter reached; results written, see info */
  FEMH_E_BREAKDOWN = 5,      /* CG breakdown (p.Kp <= 0 or non-finite) */
  FEMH_E_STATE = 6           /* call order (e.g. gradient before a solve) */
};

/* material law of the per-voxel Young's modulus E(rho); K0 uses nu */
enum { FEMH_INTERP_SIMP = 0,    /* E_min + rho^p (E_s - E_min)   MaterialOpt/src/FEM3DFun.cpp:244-257 */
       FEMH_INTERP_RAMP3 = 1,   /* E_s rho/(3-2rho)  fast_fem/FEM3DFun.cpp:20-27 */
       FEMH_INTERP_BINARY = 2   /* rho>=0.5 ? bin_hi : bin_lo
                                   NumericalCoarseningUsingMultiGrid.cpp:235-241 */ };
enum { FEMH_FP64 = 0,           /* plain method, all FP64 */
       FEMH_MIXED = 1,          /* FP32 inner PCG solves in FP64 defect correction */
       FEMH_MIXED_PC = 2 };     /* FP64 CG + operator, FP32 multigrid preconditioner */
enum { FEMH_JACOBI_PCG = 0, FEMH_GMG_PCG = 1 };

typedef struct {
  int device;             /* CUDA device ordinal */
  int interp;             /* FEMH_INTERP_* */
  double E_s, E_min, penal, nu;
  double bin_hi, bin_lo;
  double rho_min, rho_max; /* clamp applied before the law (fast_fem clamps 1e-3..1); a
                              density that is NaN, infinite or negative is not clamped but
                              rejected: the solve returns FEMH_E_ARG */
  int precision;          /* FEMH_FP64 | FEMH_MIXED | FEMH_MIXED_PC */
  int solver;             /* FEMH_JACOBI_PCG | FEMH_GMG_PCG */
  int pre_smooth, post_smooth; /* damped-Jacobi sweeps per level (GMG); equal counts keep the
                                  V-cycle symmetric, which CG needs */
  double omega;           /* Jacobi damping */
  int coarse_max_nodes;   /* coarsen until a level has <= this many nodes (GMG) */
  double tol;             /* relative residual ||b - K x|| / ||b||, FP64 */
  int max_iter;           /* CG iterations (plain) / inner iterations per outer step (mixed) */
  double inner_tol;       /* mixed: relative reduction asked of each inner solve */
  int max_outer;          /* mixed: defect-correction steps */
  int store_bf16;         /* mixed: bf16 storage of search directions and rho.  Converges on
                             small cells (<= 32^3 tested); on the 128^3 smooth and 256^3
                             binary benchmark cells CG then stalls near 1e-4 (the rounded
                             search directions lose conjugacy): keep 0 there.  FEMH_MIXED_PC
                             with block_cg keeps its search directions in FP64 regardless */
  int graph_chunk;        /* CG iterations per captured CUDA graph (0 = no graphs) */
  int coarse_avg;         /* coarse voxel modulus from its 8 children: 0 arithmetic mean
                             (rediscretisation of the mean), 1 geometric, 2 harmonic */
  int autotune;           /* 1: time the stencil's x-chunk length per level at set-up */
  int stencil_variant;    /* 0: chosen by the autotuner; else forced: 1 one voxel row per
                             thread, 2 two rows per thread, 3 two load cases per thread in
                             packed FP32x2 lanes, 4 two rows per thread in packed FP32x2
                             lanes, 5 as 4 with the inputs staged in shared memory by bulk
                             copies (3-5: FP32 operators; FP64 ones use 1 or 2), 6 one row
                             per thread in FP64 with staged inputs (FP64 operators; FP32
                             ones use 1), 7 as 5 with one persistent CTA per multiprocessor
                             running a balanced run of units (FP32 operators; levels of one
                             z extent).  5-7 need every cell of a level to have a z extent
                             in {16,24,32,48,64,128 (,256 for 6)} (levels of mixed extents
                             launch one kernel per extent; 7 runs as 5 there); elsewhere 4
                             and 1 run */
  int warm_start;         /* 1: a solve on the same cells as the handle's previous solve
                             starts from that solution (chi) instead of zero -- the
                             line-search / descent case of fast_fem/run3d.cpp:238-289;
                             results agree with a cold start within the tolerance */
  double cheb_ratio;      /* 0: every smoothing sweep is damped by omega; > 1: the sweeps
                             of a pass use the reciprocal roots of the Chebyshev
                             polynomial of that degree on [lmax/cheb_ratio, lmax], lmax =
                             the largest eigenvalue of D0^-1 K0 (a bound on the spectrum
                             of D^-1 K for every coefficient field; D0 the element's
                             diagonal, or its 3x3 node blocks with block_jacobi) */
  int block_jacobi;       /* multigrid sweeps: 0 point Jacobi, D = diag(K); 1 node-block
                             Jacobi, D = the 3x3 diagonal blocks of K (the three
                             displacement components of a node solved together; they
                             couple where the coefficients jump) */
  int block_cg;           /* GMG-PCG with FP64 CG (FEMH_FP64, FEMH_MIXED_PC), cold start:
                             1 block conjugate gradients over the six load cases of a cell
                             (one Krylov space, 6x6 step matrices; a cell whose block turns
                             indefinite is solved again case by case), 0 six independent
                             PCG runs */
} femh_config;

typedef struct {
  int status;             /* FEMH_OK / FEMH_E_NOT_CONVERGED / FEMH_E_BREAKDOWN */
  int iterations[6];      /* total inner CG iterations per load case */
  int outer_iterations;   /* defect-correction steps (mixed), 1 for FP64 */
  double rel_residual[6]; /* final FP64 ||b - K x|| / ||b|| per load case */
  double solve_ms;        /* device time of the solve (CUDA events) */
  double density;         /* mean rho used (fast_fem/FEM3DFun.cpp:189-193) */
} femh_solve_info;

typedef struct {
  int nx, ny, nz;         /* voxels per axis (periodic) */
  double h;               /* voxel edge; |Y| = nx*ny*nz*h^3 */
  const double* rho;      /* nx*ny*nz densities (host or device, per call flag) */
} femh_cell;

typedef struct femh_handle femh_handle;

/* Defaults: SIMP E_s=1, E_min=1e-6, p=3, nu=0.3, FP64 GMG-PCG, tol 1e-10, 3 + 3
 * Jacobi sweeps per level with Chebyshev-root weights (cheb_ratio 64). */
femh_status femh_config_default(femh_config* cfg);

/* Create an engine on cfg->device.  Replaces ElasticHexFEM/Homogenization
 * initialisation (fast_fem/run3d.cpp:118-164,
 * NumericalCoarseningUsingMultiGrid.cpp:134-218). */
femh_status femh_create(femh_handle** h, const femh_config* cfg);
femh_status femh_destroy(femh_handle* h);

/* Solve the six periodic load cases of one cell and return C^H (6x6, row
 * major).  rho has nx*ny*nz entries, on the device if rho_on_device.
 * Replaces FEM3DFun::setParam's Homogenize + energy loop
 * (fast_fem/FEM3DFun.cpp:128-196) and
 * NumericalCoarseningUsingMultiGrid.cpp:269-313. */
femh_status femh_homogenize(femh_handle* h, int nx, int ny, int nz, double hvox, const double* rho,
                            int rho_on_device, double C_out[36], femh_solve_info* info);

/* dL/drho_e for a loss with dL/dC = dLdC (6x6 row major) at the last solve:
 * dL/drho_e = c'(rho_e) h/|Y| sum_IJ dLdC_IJ u^I_e.K0(1) u^J_e  (self-adjoint,
 * no second solve).  Replaces FEM3DFun::df (fast_fem/FEM3DFun.cpp:222-268). */
femh_status femh_homogenize_grad(femh_handle* h, const double dLdC[36], double* dLdrho,
                                 int out_on_device);

/* Gradient of a loss with respect to the parameters of a piecewise-constant
 * density field, at the last solve: the field chain rule of FEM3DFun::df
 * (fast_fem/FEM3DFun.cpp:252-266) for the fields whose df(x) is one parameter
 * with weight 1 (PiecewiseConstant3D / Sym3D / Cubic3D,
 * fast_fem/PiecewiseConstant*3D.cpp), on the device:
 *   grad[p] = sum over voxels e with voxel_param[e] == p of (dL/drho_e + dLdrho_add),
 * dL/drho_e as femh_homogenize_grad computes it from dLdC, dLdrho_add a term
 * added to every voxel (FEM3DFun's density penalty, mw/n (density - m0),
 * FEM3DFun.cpp:229-231).  voxel_param: nx*ny*nz host ints in [0, nparam), or
 * -1 for a voxel that belongs to no parameter; grad_out: nparam host doubles.
 * The sums run in a fixed order (bit-reproducible).  The voxel lists are built
 * on the host and kept on the device until the map or the cells change. */
femh_status femh_field_gradient(femh_handle* h, const double dLdC[36], double dLdrho_add, int nparam,
                                const int* voxel_param, double* grad_out);

/* dC^H_IJ/drho_e for the 21 lower-triangle pairs, layout [21][nx*ny*nz]. */
femh_status femh_dCdrho(femh_handle* h, double* out, int out_on_device);

/* femlib's force-driven coarse tensor of every cell of the last solve
 * (femh_homogenize: 1 cell; femh_homogenize_batch: ncell cells), C_out
 * [cell][36] row major.  NumericalCoarsening::computeCoarsenedElasticityTensor-
 * AndParameters3D (SamplesGenerator/NumericalCoarsening.cpp:262-340) solves
 * six face-force load cases with periodic-jump, translation and rotation
 * multipliers (femlib/src/EMeshStiffness.cpp:53-274) and forms
 * C = G^-T (sum_e sum_q w_q Gv^T E Gv / nelem) G^-1 from the coarse and local
 * strains of those fields (femlib/src/MeshUtilities.cpp:960-1060).  Its fields
 * span the same space as the six strain-driven fluctuation fields solved here,
 * and the formula does not depend on the basis, so this evaluates it on those
 * fields: femlib's Voigt columns hold tensor shear strains against the
 * engineering matrix E, hence C = S W' S with S = diag(1,1,1,2,2,2) and W' the
 * energy pairs of the material E with its shear modulus divided by 4.
 * Cubic cells only (FEMH_E_ARG otherwise): on an nx != ny cell femlib's shear
 * loads (f/2 on faces of different areas) are out of moment balance and its
 * rotation multipliers load the interior, so its fields leave that space.
 * femlib additionally scales the diagonal of K by 1 + 1e-5
 * (NumericalCoarsening.cpp:1262-1264); this is the exact (unregularised)
 * value, which femlib's differs from at that 1e-5 level.  Equals C^H only for
 * homogeneous cells.  (E, nu) of the reference's parameters come from the
 * compliance (C^H)^-1 under its unit face loads, see femh_host.hpp. */
femh_status femh_force_tensors(femh_handle* h, double* C_out);

/* Full-cell displacement of load case I on (nx+1)(ny+1)(nz+1) nodes, layout
 * [node][3] with node (i*(ny+1)+j)*(nz+1)+k, including the affine jump on the
 * + faces: fast_fem/FEM3DFun.cpp:31-56 copyPeriodicU. */
femh_status femh_full_field(femh_handle* h, int load_case, double* u_out, int out_on_device);

/* Periodic fluctuation chi of the last solve, layout [6][nx*ny*nz][3]. */
femh_status femh_fluctuation(femh_handle* h, double* chi_out, int out_on_device);

/* Apply the periodic operator: y_I = K(rho) u_I for the 6 fields u, layout
 * [6][nx*ny*nz][3] (the reference's assembled K, e.g.
 * SamplesGenerator/NumericalCoarsening.cpp:1238-1306, matrix-free).  FP64
 * unless the handle's precision is mixed with FP32 storage: then the FP32
 * kernel the multigrid sweeps use (coefficients and u rounded to FP32). */
femh_status femh_apply_operator(femh_handle* h, int nx, int ny, int nz, double hvox,
                                const double* rho, const double* u, double* y, int on_device);

/* Many cells of uneven size in one set of launches (the sample generator's
 * 8-thread loop, SamplesGenerator/SamplesGeneratorImpl.cpp:3703-3736).
 * C_out: 36*ncell.  dLdC (36*ncell) and dLdrho (sum of voxels, cell after cell)
 * are optional (both NULL to skip the gradient).  infos: ncell entries or NULL.
 * All pointers host-side. */
femh_status femh_homogenize_batch(femh_handle* h, int ncell, const femh_cell* cells, double* C_out,
                                  const double* dLdC, double* dLdrho, femh_solve_info* infos);

/* Device memory a femh_homogenize_batch call on these cells needs under the
 * handle's configuration (need_bytes: multigrid levels, coarse matrices and
 * solver vectors; about 0.9 KB per voxel in FEMH_MIXED_PC, 1.1 KB in FEMH_FP64),
 * and what is available to it (avail_bytes: free device memory plus what the
 * handle itself holds, which the call would release first).  Either output may
 * be NULL.  For splitting a cell set that does not fit one call (the sample
 * generator's batches); no counterpart in the reference, whose per-cell
 * PARDISO solves never hold more than one cell. */
femh_status femh_batch_memory(femh_handle* h, int ncell, const femh_cell* cells, double* need_bytes,
                              double* avail_bytes);

/* Copy the last error message (NUL-terminated) into buf. */
femh_status femh_last_error(const femh_handle* h, char* buf, size_t n);

/* Stream used by the handle (cudaStream_t as void*); NULL restores its own. */
femh_status femh_set_stream(femh_handle* h, void* stream);

/* Kernel executions issued by the handle since creation (all are this
 * library's own kernels; CUDA-graph replays count every kernel they run). */
long long femh_kernel_launches(const femh_handle* h);

/* Measurement hooks (no counterpart in the reference, whose only timing is an
 * ad-hoc wall clock, femlib/src/Timer.cpp).  With profiling on, CUDA graphs are
 * not captured and every launch is bracketed by CUDA events on the handle's
 * stream; stats accumulate per kernel class with the algorithmic bytes each
 * launch must move (inputs read once + outputs written once). */
typedef struct {
  char name[64];
  long long launches;
  double total_ms;
  double bytes;
} femh_kernel_stat;
femh_status femh_profile(femh_handle* h, int enable);   /* also clears the stats */
femh_status femh_profile_read(femh_handle* h, femh_kernel_stat* out, int max, int* n);

/* C^H of one cell from a caller-provided density field and periodic
 * fluctuation, allocating nothing.  No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- code whose device memory belongs
 * to another allocator (a host framework's caching allocator that has already
 * reserved the device, an application that must keep its footprint fixed after
 * start-up) and latency-critical loops that cannot afford cudaMalloc/cudaFree's
 * implicit device synchronisation.
 *   cfg  material law (interp, E_s, E_min, penal, nu, bin_hi/lo, rho clamp);
 *        cfg->device must be the calling thread's current device
 *   rho  device pointer, nx*ny*nz densities;   chi  device pointer, the
 *        fluctuation in femh_fluctuation's layout [6][nx*ny*nz][3]
 *   C_out device pointer, 36 doubles (6x6 row major, both triangles written)
 *   stream cudaStream_t as void* (NULL = default stream); the call is
 *        asynchronous on it.
 * Limits: nx*ny*nz <= 256^3 (16,777,216 voxels); larger cells return
 * FEMH_E_ARG before any device work.  Its scratch is a fixed 336 KiB device
 * array (2048 slots x 21 doubles) that every GPU loading this library holds
 * until the process exits; every call overwrites it, so calls that overlap on
 * the GPU (different streams or threads) race -- serialise them.  The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress) and
 * caches it; make that first call before any stream capture. */
femh_status femh_energy_noalloc(const femh_config* cfg, int nx, int ny, int nz, double hvox,
                                const double* rho, const double* chi, double* C_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FEMH_H */
