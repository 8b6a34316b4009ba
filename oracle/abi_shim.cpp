// TEST INFRASTRUCTURE ONLY.  The FP64 CPU oracle (afqmc_oracle.cpp) behind the subset of
// the library's C ABI (include/afqmc_b200.h) that the driver program
// (miniafqmc_b200/app/miniafqmc.cpp) calls, so that the tests can build the driver
// against it and check the driver's call sequence, layouts and input handling on a host
// without a GPU, against the oracle run through the Python driver.  Nothing in the
// product links it.
//
// BLAS/LAPACK: the oracle's Fortran entry points are looked up in the shared library
// named by AFQ_ORACLE_LAPACK (the tests pass scipy's bundled OpenBLAS) under the names
// given by AFQ_ORACLE_LAPACK_PREFIX + {zgemm_, zgemv_, zgetrf_, zgetri_, zgelqf_,
// zunglq_}.  Calls outside the subset are not defined here (the link fails).
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "afqmc_b200.h"

struct orc_handle;
extern "C" {
int orc_set_lapack(void* zgemm, void* zgemv, void* zgetrf, void* zgetri, void* zgelqf,
                   void* zunglq);
orc_handle* orc_create(int nmo, int naea, int nchol, int nwalk, double dt, int order);
void orc_destroy(orc_handle* h);
void orc_set_spvn(orc_handle* h, int nrows, int ncols, const int* ri, const int* c,
                  const double* v);
void orc_set_spvnT(orc_handle* h, int nrows, int ncols, const int* ri, const int* c,
                   const double* v);
void orc_set_vakbl(orc_handle* h, int nrows, int ncols, const int* ri, const int* c,
                   const double* v);
void orc_set_dense(orc_handle* h, const double* P, const double* haj, const double* trial,
                   const double* Lh);
void orc_set_walkers(orc_handle* h, const double* W, const double* Wd);
void orc_get_walkers(const orc_handle* h, double* W, double* Wd);
double orc_get_eshift(const orc_handle* h);
void orc_set_eshift(orc_handle* h, double e);
void orc_mixed_density_matrix(orc_handle* h);
void orc_mixed_density_matrix_full(orc_handle* h);
void orc_vbias(orc_handle* h);
void orc_vbias_full(orc_handle* h);
void orc_overlaps(orc_handle* h, int save_old);
void orc_sigma(orc_handle* h, uint64_t seed, uint64_t step);
void orc_vhs(orc_handle* h);
void orc_propagate(orc_handle* h);
void orc_update_weights(orc_handle* h);
void orc_orthogonalize(orc_handle* h);
double orc_energy_vakbl(orc_handle* h);
double orc_energy_chol(orc_handle* h, double* parts);
void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out);
long long orc_halfrotate(int N, int n, int nchol, const int* ri, const int* ci,
                         const double* vals, const double* trial_a, const double* trial_b,
                         double cutoff, int* out_rowIndex, int* out_cols, double* out_vals);
}

struct afq_handle {
  orc_handle* o = nullptr;
  afq_system_desc d{};
  bool has_vakbl = false, has_lh = false;
  std::string err;
};

namespace {

bool lapack_loaded() {
  static const bool ok = [] {
    const char* path = std::getenv("AFQ_ORACLE_LAPACK");
    const char* pre = std::getenv("AFQ_ORACLE_LAPACK_PREFIX");
    if (!path) return false;
    void* lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!lib) return false;
    const std::string p = pre ? pre : "";
    void* f[6];
    const char* names[6] = {"zgemm_", "zgemv_", "zgetrf_", "zgetri_", "zgelqf_", "zunglq_"};
    for (int i = 0; i < 6; i++) f[i] = dlsym(lib, (p + names[i]).c_str());
    return orc_set_lapack(f[0], f[1], f[2], f[3], f[4], f[5]) == 0;
  }();
  return ok;
}

afq_status fail(afq_handle* h, afq_status s, const char* msg) {
  if (h) h->err = msg;
  return s;
}

}  // namespace

extern "C" {

const char* afq_status_string(afq_status s) {
  switch (s) {
    case AFQ_OK: return "ok";
    case AFQ_ERR_ARG: return "invalid argument";
    case AFQ_ERR_STATE: return "call out of order";
    case AFQ_ERR_CUDA: return "CUDA error";
    case AFQ_ERR_OOM: return "out of device memory";
    case AFQ_ERR_UNSUPPORTED: return "unsupported";
    case AFQ_ERR_SINGULAR: return "singular overlap matrix";
  }
  return "unknown status";
}

const char* afq_last_error(const afq_handle* h) { return h ? h->err.c_str() : ""; }

afq_status afq_halfrotate(int, const afq_csr_z* Spvn, int nmo, int naea, int nchol,
                          const double* trial, double cutoff, double lh_scale, long long* nnz,
                          int32_t* rowIndex, int32_t* cols, double* vals, double* Lhalf) {
  if (!lapack_loaded()) return AFQ_ERR_UNSUPPORTED;
  if (!Spvn || !trial || !nnz || Spvn->nrows != nmo * nmo || Spvn->ncols != nchol)
    return AFQ_ERR_ARG;
  const double* ta = trial;
  const double* tb = trial + 2LL * nmo * naea;
  *nnz = orc_halfrotate(nmo, naea, nchol, Spvn->rowIndex, Spvn->cols, Spvn->vals, ta, tb,
                        cutoff, nullptr, nullptr, nullptr);
  if (rowIndex) {
    std::vector<int> c((size_t)*nnz);
    std::vector<double> v((size_t)2 * *nnz);
    orc_halfrotate(nmo, naea, nchol, Spvn->rowIndex, Spvn->cols, Spvn->vals, ta, tb, cutoff,
                   rowIndex, c.data(), v.data());
    for (long long p = 0; p < *nnz; p++) {
      if (cols) cols[p] = c[p];
      if (vals) {
        vals[2 * p] = v[2 * p];
        vals[2 * p + 1] = v[2 * p + 1];
      }
    }
  }
  if (Lhalf) {   // every entry (cutoff below any magnitude), scaled, into the dense layout
    const long long width = 2LL * naea * nmo;
    std::vector<int> ri((size_t)nchol + 1);
    const long long all = orc_halfrotate(nmo, naea, nchol, Spvn->rowIndex, Spvn->cols,
                                         Spvn->vals, ta, tb, -1.0, nullptr, nullptr, nullptr);
    std::vector<int> c((size_t)all);
    std::vector<double> v((size_t)2 * all);
    orc_halfrotate(nmo, naea, nchol, Spvn->rowIndex, Spvn->cols, Spvn->vals, ta, tb, -1.0,
                   ri.data(), c.data(), v.data());
    for (long long e = 0; e < 2 * nchol * width; e++) Lhalf[e] = 0.0;
    for (int r = 0; r < nchol; r++)
      for (int p = ri[r]; p < ri[r + 1]; p++) {
        Lhalf[2 * (r * width + c[p])] = v[2 * p] * lh_scale;
        Lhalf[2 * (r * width + c[p]) + 1] = v[2 * p + 1] * lh_scale;
      }
  }
  return AFQ_OK;
}

afq_status afq_create(const afq_system_desc* desc, afq_handle** out) {
  if (!desc || !out || desc->nmo <= 0 || desc->naea <= 0 || desc->nchol <= 0 ||
      desc->nwalk <= 0)
    return AFQ_ERR_ARG;
  if (!lapack_loaded()) return AFQ_ERR_UNSUPPORTED;
  afq_handle* h = new afq_handle();
  h->d = *desc;
  h->o = orc_create(desc->nmo, desc->naea, desc->nchol, desc->nwalk, desc->dt,
                    desc->taylor_order);
  *out = h;
  return AFQ_OK;
}

void afq_destroy(afq_handle* h) {
  if (!h) return;
  orc_destroy(h->o);
  delete h;
}

afq_status afq_set_hamiltonian(afq_handle* h, const afq_csr_z* Spvn, const afq_csr_z* SpvnT,
                               const double* Propg1, const double* haj, const double* trial,
                               const afq_csr_z* Vakbl, const double* Lhalf) {
  if (!h || !Spvn || !SpvnT || !Propg1 || !haj || !trial || (!Vakbl && !Lhalf))
    return fail(h, AFQ_ERR_ARG, "null operand");
  orc_set_spvn(h->o, Spvn->nrows, Spvn->ncols, Spvn->rowIndex, Spvn->cols, Spvn->vals);
  orc_set_spvnT(h->o, SpvnT->nrows, SpvnT->ncols, SpvnT->rowIndex, SpvnT->cols, SpvnT->vals);
  if (Vakbl) orc_set_vakbl(h->o, Vakbl->nrows, Vakbl->ncols, Vakbl->rowIndex, Vakbl->cols,
                           Vakbl->vals);
  orc_set_dense(h->o, Propg1, haj, trial, Lhalf);
  h->has_vakbl = Vakbl != nullptr;
  h->has_lh = Lhalf != nullptr;
  return AFQ_OK;
}

afq_status afq_cv_configure(afq_handle* h, int, double, uint64_t, long long, int) {
  return fail(h, AFQ_ERR_UNSUPPORTED, "no control variate in the oracle");
}

afq_status afq_cv_set_base(afq_handle* h, int) {
  return fail(h, AFQ_ERR_UNSUPPORTED, "no control variate in the oracle");
}

afq_status afq_set_walkers(afq_handle* h, const double* W, const double* W_data) {
  if (!h || !W || !W_data) return fail(h, AFQ_ERR_ARG, "null walkers");
  orc_set_walkers(h->o, W, W_data);
  return AFQ_OK;
}

afq_status afq_get_walkers(afq_handle* h, double* W, double* W_data) {
  if (!h) return AFQ_ERR_ARG;
  orc_get_walkers(h->o, W, W_data);
  return AFQ_OK;
}

afq_status afq_set_eshift(afq_handle* h, double eshift) {
  if (!h) return AFQ_ERR_ARG;
  orc_set_eshift(h->o, eshift);
  return AFQ_OK;
}

// The comb of afq_population_control (oracle.comb restated in C++): prefix sums of
// max(Re w, 0) in walker order, copy j = first walker with C_i > (j + u) T / nw, weight
// T / nw; u from Philox4x32-10 at counter (0, 0, step) with key seed ^ 0x9E3779B97F4A7C15.
afq_status afq_population_control(afq_handle* h, uint64_t seed, uint64_t step) {
  if (!h) return AFQ_ERR_ARG;
  const int nw = h->d.nwalk;
  const size_t per = (size_t)2 * h->d.nmo * h->d.naea * 2;   // doubles per walker
  std::vector<double> W(per * nw), Wd((size_t)16 * nw);
  orc_get_walkers(h->o, W.data(), Wd.data());
  std::vector<double> C(nw);
  double T = 0.0;
  int last = -1;
  for (int i = 0; i < nw; i++) {
    const double w = std::max(Wd[(size_t)16 * i + 2], 0.0);
    T += w;
    C[i] = T;
    if (w > 0.0) last = i;
  }
  if (last < 0) return fail(h, AFQ_ERR_STATE, "population control: no walker has positive weight");
  const uint64_t key = seed ^ 0x9E3779B97F4A7C15ull;
  const uint32_t ctr[4] = {0, 0, (uint32_t)step, (uint32_t)(step >> 32)};
  const uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
  uint32_t r[4];
  orc_philox(ctr, k, r);
  const double u =
      (double)((((uint64_t)(r[0] >> 5)) << 26) | (uint64_t)(r[1] >> 6)) * (1.0 / 9007199254740992.0);
  std::vector<double> Wn(per * nw), Wdn((size_t)16 * nw);
  for (int j = 0; j < nw; j++) {
    const double t = ((double)j + u) * T / nw;
    int i = (int)(std::upper_bound(C.begin(), C.end(), t) - C.begin());
    if (i >= nw) i = last;
    std::copy(W.begin() + per * i, W.begin() + per * (i + 1), Wn.begin() + per * j);
    std::copy(Wd.begin() + 16 * (size_t)i, Wd.begin() + 16 * (size_t)(i + 1),
              Wdn.begin() + 16 * (size_t)j);
    Wdn[(size_t)16 * j + 2] = T / nw;
    Wdn[(size_t)16 * j + 3] = 0.0;
  }
  orc_set_walkers(h->o, Wn.data(), Wdn.data());
  return AFQ_OK;
}

afq_status afq_profile(afq_handle* h, int) { return h ? AFQ_OK : AFQ_ERR_ARG; }

afq_status afq_stage_times(afq_handle* h, double* ms, long long* launches, int) {
  if (!h) return AFQ_ERR_ARG;
  for (int s = 0; s < AFQ_NSTAGES; s++) {
    if (ms) ms[s] = 0.0;
    if (launches) launches[s] = 0;
  }
  return AFQ_OK;
}

afq_status afq_mixed_density_matrix(afq_handle* h) {
  orc_mixed_density_matrix(h->o);
  return AFQ_OK;
}
afq_status afq_mixed_density_matrix_full(afq_handle* h) {
  orc_mixed_density_matrix_full(h->o);
  return AFQ_OK;
}
afq_status afq_vbias(afq_handle* h) {
  orc_vbias(h->o);
  return AFQ_OK;
}
afq_status afq_vbias_full(afq_handle* h) {
  orc_vbias_full(h->o);
  return AFQ_OK;
}
afq_status afq_sigma(afq_handle* h, uint64_t seed, uint64_t step) {
  orc_sigma(h->o, seed, step);
  return AFQ_OK;
}
afq_status afq_vhs(afq_handle* h) {
  orc_vhs(h->o);
  return AFQ_OK;
}
afq_status afq_propagate(afq_handle* h) {
  orc_propagate(h->o);
  return AFQ_OK;
}
afq_status afq_overlaps(afq_handle* h, int save_old) {
  orc_overlaps(h->o, save_old);
  return AFQ_OK;
}
afq_status afq_update_weights(afq_handle* h) {
  orc_update_weights(h->o);
  return AFQ_OK;
}
afq_status afq_orthogonalize(afq_handle* h) {
  orc_orthogonalize(h->o);
  return AFQ_OK;
}
afq_status afq_get_eshift(afq_handle* h, double* eshift) {
  if (!h || !eshift) return AFQ_ERR_ARG;
  *eshift = orc_get_eshift(h->o);
  return AFQ_OK;
}
afq_status afq_synchronize(afq_handle* h) { return h ? AFQ_OK : AFQ_ERR_ARG; }

afq_status afq_energy(afq_handle* h, int mode, double* eav) {
  if (!h || !eav) return AFQ_ERR_ARG;
  if (mode == AFQ_ENERGY_VAKBL && h->has_vakbl) *eav = orc_energy_vakbl(h->o);
  else if (mode == AFQ_ENERGY_CHOLESKY && h->has_lh) *eav = orc_energy_chol(h->o, nullptr);
  else return fail(h, AFQ_ERR_UNSUPPORTED, "energy mode not available");
  return AFQ_OK;
}

// the op sequence of one substep (miniafqmc_base.cpp:251-337)
afq_status afq_substep(afq_handle* h, uint64_t seed, uint64_t step_tot, int northo) {
  if (!h || northo <= 0) return AFQ_ERR_ARG;
  orc_mixed_density_matrix(h->o);
  orc_vbias(h->o);
  orc_sigma(h->o, seed, step_tot);
  orc_vhs(h->o);
  orc_propagate(h->o);
  orc_overlaps(h->o, 1);
  orc_update_weights(h->o);
  if (step_tot > 0 && step_tot % (uint64_t)northo == 0) {
    orc_orthogonalize(h->o);
    orc_overlaps(h->o, 0);
  }
  return AFQ_OK;
}

}  // extern "C"
