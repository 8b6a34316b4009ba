// Mixed-precision (tensor-core) form of the contraction stages.  FP64 stays in the
// LU/overlaps, QR and weights; these entry points replace vbias, vHS, the propagation
// chain and the Cholesky energy when the handle is created with AFQ_PREC_MIXED.
#pragma once
#include <string>
#include "afq_common.cuh"

namespace afq {

struct MixedState;

// Product sites whose kernel (persistent or per-tile) is chosen at set-up by timing:
// vHS, the propagation chain, the split-K vbias / Coulomb products, the exchange over all
// walkers and over a 1/8 subset, and T1.
enum TuneSite { TS_VHS, TS_PROP, TS_PART, TS_EXF, TS_EXS, TS_T1, TS_N };

struct MixedInit {
  int N, n, nchol, nw, order;
  const z_t* P;             // Propg1 [N][N]
  const z_t* Lh;            // [nchol][2nN] unscaled (may be null)
  const z_t* SpvnT_dense;   // [nchol][2nN] or null
  const int* sp_ri;         // Spvn CSR
  const int* sp_ci;
  const z_t* sp_v;
  const double* sp_rv;
  const z_t* trial;         // [N][2n] (null: the density matrix stays FP64)
};

cudaError_t mixed_create(const MixedInit* init, MixedState** out, std::string* msg,
                         cudaStream_t st);
void mixed_destroy(MixedState* m);
cudaError_t mixed_vbias(MixedState* m, const z_t* Gc, z_t* vbias, cudaStream_t st);
cudaError_t mixed_vhs(MixedState* m, const z_t* X, z_t* vHS, cudaStream_t st);
cudaError_t mixed_propagate(MixedState* m, z_t* W, const z_t* vHS, cudaStream_t st);
cudaError_t mixed_energy_chol(MixedState* m, const z_t* Gc, z_t* cvec, z_t* Kpart, int nblk,
                              cudaStream_t st);
cudaError_t mixed_coulomb(MixedState* m, const z_t* Gc, z_t* cvec, cudaStream_t st);
cudaError_t mixed_exchange(MixedState* m, const z_t* Gc, int nsub, z_t* Kpart, int nblk,
                           cudaStream_t st);
// The exchange partial sums in plain bf16 (hi parts of the split operands, one product):
// the control variate's low-precision base.  cudaErrorNotSupported unless the exchange
// runs on bf16 split operands.
cudaError_t mixed_exchange_lowp(MixedState* m, const z_t* Gc, int nsub, z_t* Kpart, int nblk,
                                cudaStream_t st);
// Mixed density matrix: T1 = W^T tw in split bf16 on tensor cores, FP64 Gauss-Jordan for
// det(T1) (-> W_data overlaps, info) and T1^-1, Gc = T1^-1 W^T on tensor cores.
// want_gc == 0 computes the overlaps (and keeps T1^-1); cached != 0 forms Gc from the
// T1^-1 of an earlier call on the same walkers.
bool mixed_has_dm(const MixedState* m);
cudaError_t mixed_dm(MixedState* m, const z_t* W, z_t* Gc, z_t* Wd, int* info, int want_gc,
                     int save_old, int cached, cudaStream_t st);
// Packed operand forms of the walkers (the T1 and P W operands): the propagation
// leaves them current; mixed_invalidate marks them stale after any other change of W,
// mixed_repack forms them from W, mixed_ensure_packed does so only when they are stale.
void mixed_invalidate(MixedState* m);
cudaError_t mixed_repack(MixedState* m, const z_t* W, cudaStream_t st);
cudaError_t mixed_ensure_packed(MixedState* m, const z_t* W, cudaStream_t st);
int mixed_repack_launches(const MixedState* m);
// Kernels one call of a stage issues (afq_stage numbering), for the launch counters.
int mixed_launches(const MixedState* m, int stage);
// Cholesky-vector blocks of the exchange partial sums (Kpart[nw][2][nblk]).
int mixed_nblk(const MixedState* m);
// Timeout flags raised by the tensor-core kernels (0 when clean).
cudaError_t mixed_error(MixedState* m, int* flags);
// Work-wait bound of this module's tensor-core kernels on the current device (SM clocks;
// <= 0 restores the default of about one second).
cudaError_t mixed_set_wait_clocks(long long clocks);
// Kernel choices: choice[TS_N + 1] (0 built-in rule, 1 persistent, 2 per-tile; the last
// entry is the split-K slice count), ms[TS_N][2] the set-up timings (0 when not timed).
// Walkers per group of the propagation chain picked at set-up (0: all walkers per
// product) and, in ms[6], the timed chain for 0 (all), 32, 48, 64, 96 and 128 walkers.
int mixed_prop_group(const MixedState* m, float* ms);
// Symmetric vHS epilogue picked at set-up (0 row-wise, 1 through the shared-memory tile,
// 2 the same with two CTAs per SM, 3 as 2 with two 64-byte-slab stages per CTA) and, in
// ms[4], the timed product for each (0 when not timed).
int mixed_vhs_epilogue(const MixedState* m, float* ms);
// Walkers per wave of the fused propagation chain (0: eight launches) and, in ms[6], the
// timed chain: eight launches, waves of 16, 24, 32, 48 and 64 walkers (0 when not timed).
int mixed_prop_chain(const MixedState* m, float* ms);
void mixed_tuning(const MixedState* m, int* choice, float* ms);
// Heterogeneous batches: the vHS product and the propagation chain of n systems (n <= 4),
// each product one launch over every system's tiles.  mixed_multi_compatible: the systems
// share the precisions and the Taylor order.  mixed_vhs_pack / mixed_prop_pack
// (on each system's stream, before the joint launches) pack X and, unless current, the
// P W operand; mixed_prop_multi leaves no packed walker forms current.
bool mixed_multi_compatible(MixedState* const* ms, int n);
cudaError_t mixed_vhs_pack(MixedState* m, const z_t* X, cudaStream_t st);
cudaError_t mixed_vhs_multi(MixedState* const* ms, int n, cudaStream_t st);
cudaError_t mixed_prop_pack(MixedState* m, const z_t* W, cudaStream_t st);
int mixed_prop_pack_launches(const MixedState* m);
cudaError_t mixed_prop_multi(MixedState* const* ms, z_t* const* W, int n, cudaStream_t st);
// FP64 copy of the V operand ([nw][N*N]), for copy-out.
cudaError_t mixed_unpack_vhs(MixedState* m, z_t* vHS, cudaStream_t st);

}  // namespace afq
