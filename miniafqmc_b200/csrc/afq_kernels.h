// Launch wrappers of the walker-step kernels (internal to libafqmc_b200).
#pragma once
#include <algorithm>
#include <cstddef>
#include "afq_common.cuh"

namespace afq {

size_t dm_smem_bytes(int n);
cudaError_t launch_dm(const z_t* W, const z_t* tw, int N, int n, int nw, z_t* Gc, z_t* Wd,
                      int* info, int want_gc, int save_old, cudaStream_t st);
cudaError_t launch_sigma(const z_t* vbias, z_t* X, double* xraw, z_t* hybridW, int nchol,
                         int nw, const DevScalars* sc, int use_xraw, cudaStream_t st);
// CSR x walker-fast dense (vHS = Spvn X).  cfg 0 is the built-in CTA shape (16 rows x 64
// walkers), 1..kCsrWalkerCfgs the shapes the set-up tuner times (csr_walker_cfg_name).
constexpr int kCsrWalkerCfgs = 7;
cudaError_t launch_csr_walker(const int* rowIndex, const int* cols, const z_t* zvals,
                              const double* rvals, const z_t* B, int nrows, int nw, z_t* out,
                              long long out_ld, cudaStream_t st, int cfg = 0);
const char* csr_walker_cfg_name(int cfg);
cudaError_t launch_csr_gather(const int* rowIndex, const int* cols, const z_t* vals, const z_t* G,
                              long long ldg, int nrows, int nw, z_t* out, cudaStream_t st);
cudaError_t launch_weights(z_t* Wd, const z_t* hybridW, int nw, double dt, DevScalars* sc,
                           int update_eshift, cudaStream_t st);
cudaError_t launch_set_scalars(DevScalars* sc, unsigned long long seed, unsigned long long step,
                               int set_eshift, double eshift, cudaStream_t st,
                               int walker_offset = 0, long long nwalk_global = 0);
cudaError_t launch_ortho(z_t* W, int N, int n, int nw, cudaStream_t st);
cudaError_t launch_ortho_cholqr(z_t* W, int N, int n, int nw, int* info, cudaStream_t st);
size_t exch_smem_bytes();
cudaError_t launch_exchange(const z_t* Lh, const z_t* Gc, int N, int n, int nchol, int nw,
                            z_t* Kpart, int* nblk_out, cudaStream_t st);
cudaError_t launch_energy_reduce(const z_t* Gc, const z_t* haj, int nak, const z_t* Gcloc,
                                 const z_t* cv, int nchol, const z_t* Kpart, int nblk, int nw,
                                 int mode, z_t* Wd, double* parts, cudaStream_t st);
cudaError_t launch_e4sum_out(const DevScalars* sc, double* out, cudaStream_t st);
cudaError_t launch_eshift_from(DevScalars* sc, const double* total, int nw, cudaStream_t st);
cudaError_t launch_eav(const z_t* Wd, int nw, DevScalars* sc, cudaStream_t st);
// Population control by the comb (popcontrol.cu): u = comb_uniform(seed, step, offset of
// the handle's walker block); C [nw],
// idx [nw], wnew [1] device scratch; Wscr / Wdscr hold the copies before they replace
// W [nw][per] and W_data [nw][8].  Synchronises once to read the total weight (*total);
// with no positive weight nothing is copied.
double comb_uniform(unsigned long long seed, unsigned long long step, int walker_offset);
cudaError_t launch_comb(z_t* W, z_t* Wd, int nw, long long per, double u, double* C, int* idx,
                        double* wnew, z_t* Wscr, z_t* Wdscr, double* total, cudaStream_t st);

}  // namespace afq
