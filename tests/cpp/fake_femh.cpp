// A stand-in for libfemh's C ABI (test double, no GPU): the ten entry points
// the C++ host layer calls, returning deterministic tensors so that the host
// layer's own logic -- material mapping, repMaterialAssignment, parameter
// formulas, batch bookkeeping, error paths -- can be checked on the CPU.
//
// C^H of a cell is an isotropic tensor of the mean voxel modulus (two-material
// law of the config) with its xx, yy and yz entries raised by 5%, 3% and 2%,
// so that the cell is not cubic and each axis has its own Y and nu.  The
// force-driven tensor is C^H with its shear rows and columns scaled by 0.9;
// like the engine it refuses non-cubic cells.  dL/drho_e = trace(dL/dC).
#include <cstring>
#include <string>
#include <vector>

#include "../../include/femh.h"

struct femh_handle {
  femh_config cfg;
  std::vector<double> C;   // [cell][36] of the last solve
  std::vector<int> cubic;
  std::string err;
  int nvox = 0;
};

int g_batch_calls = 0;        // femh_homogenize_batch calls so far (read by the test driver)
int g_fail_batch_call = -1;   // that call (by count) returns FEMH_E_OOM, as a batch too large would
double g_fake_avail = 1e12;   // device bytes femh_batch_memory reports available

namespace {
void fake_C(const femh_config& c, int nx, int ny, int nz, const double* rho, double C[36]) {
  const long long n = (long long)nx * ny * nz;
  double E = 0.0;
  for (long long i = 0; i < n; ++i) {
    const double r = rho[i] < c.rho_min ? c.rho_min : (rho[i] > c.rho_max ? c.rho_max : rho[i]);
    if (c.interp == FEMH_INTERP_BINARY) E += r >= 0.5 ? c.bin_hi : c.bin_lo;
    else if (c.interp == FEMH_INTERP_RAMP3) E += c.E_s * r / (3.0 - 2.0 * r);
    else E += c.E_min + r * r * r * (c.E_s - c.E_min);
  }
  E /= (double)n;
  const double nu = c.nu, lam = E * nu / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
  std::memset(C, 0, 36 * sizeof(double));
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) C[6 * a + b] = lam + (a == b ? 2 * mu : 0.0);
  for (int a = 3; a < 6; ++a) C[7 * a] = mu;
  C[0] *= 1.05;
  C[7] *= 1.03;
  C[21] *= 1.02;
}
}  // namespace

extern "C" {

femh_status femh_config_default(femh_config* c) {
  if (!c) return FEMH_E_ARG;
  std::memset(c, 0, sizeof(*c));
  c->interp = FEMH_INTERP_SIMP;
  c->E_s = 1.0;
  c->E_min = 1e-6;
  c->penal = 3.0;
  c->nu = 0.3;
  c->bin_hi = 1.0;
  c->bin_lo = 1e-4;
  c->rho_max = 1.0;
  return FEMH_OK;
}

femh_status femh_create(femh_handle** h, const femh_config* cfg) {
  if (!h || !cfg) return FEMH_E_ARG;
  *h = new femh_handle{*cfg, {}, {}, {}, 0};
  return FEMH_OK;
}

femh_status femh_destroy(femh_handle* h) {
  delete h;
  return FEMH_OK;
}

femh_status femh_homogenize(femh_handle* h, int nx, int ny, int nz, double, const double* rho, int,
                            double C_out[36], femh_solve_info* info) {
  if (!h || !rho || !C_out || nx < 1 || ny < 1 || nz < 1) return FEMH_E_ARG;
  fake_C(h->cfg, nx, ny, nz, rho, C_out);
  h->C.assign(C_out, C_out + 36);
  h->cubic.assign(1, nx == ny && ny == nz);
  h->nvox = nx * ny * nz;
  if (info) *info = femh_solve_info{};
  return FEMH_OK;
}

femh_status femh_homogenize_batch(femh_handle* h, int ncell, const femh_cell* cells, double* C_out,
                                  const double*, double*, femh_solve_info* infos) {
  if (!h || ncell < 1 || !cells || !C_out) return FEMH_E_ARG;
  if (++g_batch_calls == g_fail_batch_call) {
    h->err = "out of device memory (test double)";
    return FEMH_E_OOM;
  }
  h->C.clear();
  h->cubic.clear();
  for (int i = 0; i < ncell; ++i) {
    const femh_cell& c = cells[i];
    fake_C(h->cfg, c.nx, c.ny, c.nz, c.rho, C_out + 36 * i);
    h->C.insert(h->C.end(), C_out + 36 * i, C_out + 36 * i + 36);
    h->cubic.push_back(c.nx == c.ny && c.ny == c.nz);
    if (infos) infos[i] = femh_solve_info{};
  }
  h->nvox = 0;
  return FEMH_OK;
}

femh_status femh_force_tensors(femh_handle* h, double* C_out) {
  if (!h || !C_out) return FEMH_E_ARG;
  if (h->C.empty()) return FEMH_E_STATE;
  for (int c : h->cubic)
    if (!c) {
      h->err = "the force-driven tensor needs cubic cells (nx = ny = nz)";
      return FEMH_E_ARG;
    }
  for (size_t i = 0; i < h->C.size(); ++i) {
    const int r = (int)(i % 36) / 6, c = (int)(i % 6);
    C_out[i] = h->C[i] * (r >= 3 ? 0.9 : 1.0) * (c >= 3 ? 0.9 : 1.0);
  }
  return FEMH_OK;
}

femh_status femh_homogenize_grad(femh_handle* h, const double dLdC[36], double* dLdrho, int) {
  if (!h || !dLdC || !dLdrho || h->nvox < 1) return FEMH_E_STATE;
  double t = 0.0;
  for (int a = 0; a < 6; ++a) t += dLdC[7 * a];
  for (int i = 0; i < h->nvox; ++i) dLdrho[i] = t;
  return FEMH_OK;
}

// grad[p] = sum over the voxels of p of (trace(dL/dC) + add)
femh_status femh_field_gradient(femh_handle* h, const double dLdC[36], double add, int nparam, const int* map,
                                double* grad) {
  if (!h || !dLdC || !map || !grad || nparam < 1 || h->nvox < 1) return FEMH_E_STATE;
  double t = 0.0;
  for (int a = 0; a < 6; ++a) t += dLdC[7 * a];
  for (int p = 0; p < nparam; ++p) grad[p] = 0.0;
  for (int e = 0; e < h->nvox; ++e)
    if (map[e] >= 0) grad[map[e]] += t + add;
  return FEMH_OK;
}

// 1000 bytes per voxel; g_fake_avail available
femh_status femh_batch_memory(femh_handle* h, int ncell, const femh_cell* cells, double* need, double* avail) {
  if (!h || ncell < 0 || (ncell > 0 && !cells)) return FEMH_E_ARG;
  double b = 0.0;
  for (int i = 0; i < ncell; ++i) b += 1000.0 * cells[i].nx * cells[i].ny * cells[i].nz;
  if (need) *need = b;
  if (avail) *avail = g_fake_avail;
  return FEMH_OK;
}

femh_status femh_last_error(const femh_handle* h, char* buf, size_t n) {
  if (!buf || n == 0) return FEMH_E_ARG;
  std::strncpy(buf, h ? h->err.c_str() : "", n - 1);
  buf[n - 1] = 0;
  return FEMH_OK;
}

}  // extern "C"
