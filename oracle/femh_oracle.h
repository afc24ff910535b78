/* femh_oracle.h -- CPU FP64 oracle of the periodic voxel homogenization.
 * Test infrastructure only (see femh_oracle.c header). */
#ifndef FEMH_ORACLE_H
#define FEMH_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { FO_INTERP_SIMP = 0, FO_INTERP_RAMP3 = 1, FO_INTERP_BINARY = 2 };

typedef struct {
  int interp;
  double E_s, E_min, penal, nu, bin_hi, bin_lo;
} fo_material;

void fo_k0(double E, double nu, double h, double K[576]);
double fo_coef(const fo_material* m, double rho);
double fo_dcoef(const fo_material* m, double rho);
void fo_affine(double h, double ue0[6][24]);
void fo_apply(int nx, int ny, int nz, const double* K0, const double* coef, const double* u,
              double* y, int nrhs);
void fo_rhs(int nx, int ny, int nz, double h, const double* K0, const double* coef, double* b);
void fo_inv_diag(int nx, int ny, int nz, const double* K0, const double* coef, double* dinv);
int fo_pcg1(int nx, int ny, int nz, const double* K0, const double* coef, const double* dinv,
            const double* b, double* x, double tol, int max_iter, double* rel_out);
void fo_energy(int nx, int ny, int nz, double h, const double* K0, const double* coef,
               const double* chi, double C[36]);
void fo_dCdrho(int nx, int ny, int nz, double h, const double* K0, const fo_material* m,
               const double* rho, const double* chi, double* out);
void fo_grad(int nx, int ny, int nz, double h, const double* K0, const fo_material* m,
             const double* rho, const double* chi, const double dLdC[36], double* dLdrho);
int fo_homogenize(int nx, int ny, int nz, double h, const double* rho, const fo_material* m,
                  double tol, int max_iter, double C[36], double* chi_out, int iters[6],
                  double rel[6]);
int fo_num_threads(void);

/* femh_oracle_mg.c: the same problem solved by geometric-multigrid PCG
 * (returns 0 converged, 1 max_iter reached, 2 breakdown, < 0 set-up error) */
int fo_mg_homogenize(int nx, int ny, int nz, double h, const double* rho, const fo_material* m,
                     double tol, int max_iter, int pre, int post, double cheb_ratio, int coarse_max,
                     double C[36], double* chi_out, int iters[6], double rel[6]);
/* the same with the node-block Jacobi smoother when block != 0 */
int fo_mg_homogenize_b(int nx, int ny, int nz, double h, const double* rho, const fo_material* m,
                       double tol, int max_iter, int pre, int post, double cheb_ratio, int coarse_max,
                       int block, double C[36], double* chi_out, int iters[6], double rel[6]);
void fo_mg_apply(int nx, int ny, int nz, double h, const double* coef, double nu, const double* u,
                 double* y);

#ifdef __cplusplus
}
#endif
#endif
