/* afqmc_b200.h - C ABI of the B200 (sm_100a) walker propagation and measurement path.
 *
 * A drop-in for the operation calls the miniAFQMC driver makes on its walker set
 * (QMCPACK miniAFQMC, src/miniapps/miniafqmc_base.cpp:249-345).  Every entry point
 * takes plain pointers and sizes; complex numbers are interleaved FP64 pairs
 * (std::complex<double> / double _Complex compatible), arrays are row-major with the
 * reference's index orders:
 *
 *   W       [nwalk][2][NMO][NAEA]       walker Slater matrices   (miniafqmc_base.cpp:222)
 *   W_data  [nwalk][8]                  0 eloc, 1 weight, 2/3 overlap alpha/beta,
 *                                       4 hybrid energy, 5 previous 4, 6/7 previous 2/3
 *                                                                  (miniafqmc_base.cpp:223-224)
 *   Gc      [2*NAEA*NMO][nwalk]         compact mixed density matrix (walker fastest)
 *   vbias   [nchol][nwalk], X [nchol][nwalk], vHS [NMO*NMO][nwalk]
 *
 * The handle owns all device memory; walker state stays on the GPU between calls and
 * only the host arrays passed to set/get/copy calls cross PCIe.  A handle is used by one
 * host thread at a time and runs its work on its own CUDA stream.  All calls return an
 * afq_status; none of them aborts the process.
 */
#ifndef AFQMC_B200_H
#define AFQMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AFQ_OK = 0,
  AFQ_ERR_ARG = 1,          /* null pointer, inconsistent or out-of-range size          */
  AFQ_ERR_STATE = 2,        /* call out of order (e.g. no Hamiltonian loaded yet)        */
  AFQ_ERR_CUDA = 3,         /* a CUDA runtime call failed; see afq_last_error            */
  AFQ_ERR_OOM = 4,          /* device allocation failed                                  */
  AFQ_ERR_UNSUPPORTED = 5,  /* size or option not supported by this build                */
  AFQ_ERR_SINGULAR = 6      /* some walker had an exactly singular overlap matrix;
                               its overlap is 0 and its flags are in afq_get_info        */
} afq_status;

typedef enum {
  AFQ_PREC_FP64 = 0,        /* every contraction in FP64 (the plain form)                */
  AFQ_PREC_MIXED = 1        /* tensor-core contractions, FP64 LU/QR/weights              */
} afq_precision;

typedef enum {
  AFQ_ENERGY_VAKBL = 0,     /* eloc = 1/2 Gc.(Vakbl Gc) + Gc.haj (energy.hpp:66-102)     */
  AFQ_ENERGY_CHOLESKY = 1,  /* same energy from the half-rotated Cholesky factors        */
  AFQ_ENERGY_CV = 2         /* Cholesky energy with the exchange term estimated by the
                               learned control variate (afq_cv_configure); unbiased     */
} afq_energy_mode;

typedef enum {
  AFQ_BUF_GC = 0, AFQ_BUF_VBIAS = 1, AFQ_BUF_X = 2, AFQ_BUF_VHS = 3, AFQ_BUF_HYBRIDW = 4,
  AFQ_BUF_XRAW = 5,         /* real normals [nchol][nwalk] (double)                      */
  AFQ_BUF_INFO = 6,         /* int32 [nwalk][2], nonzero = singular overlap matrix      */
  AFQ_BUF_ENERGY_PARTS = 7, /* double [nwalk][3] = (E1, EJ, EK) of the last Cholesky
                               energy evaluation                                         */
  AFQ_BUF_CV_PRED = 8,      /* double [nwalk] surrogate exchange energy of every walker
                               from the last AFQ_ENERGY_CV measurement (0 before the
                               estimator is active)                                      */
  AFQ_BUF_G_FULL = 9        /* [2*NMO*NMO][nwalk] full density matrix of the last
                               afq_mixed_density_matrix_full                            */
} afq_buffer;

typedef struct {
  int nmo;                  /* NMO                                                       */
  int naea, naeb;           /* electrons per spin; the reference requires naea == naeb
                               (initialize_serial.hpp:67-71)                              */
  int nchol;                /* number of Cholesky vectors                                */
  int nwalk;                /* walkers held by this handle                               */
  double dt;                /* time step; Spvn passed in is already scaled by sqrt(dt)   */
  int taylor_order;         /* terms of exp(vHS) (the reference fixes 6, vHS.hpp:65)     */
  int precision;            /* afq_precision                                             */
  int device;               /* CUDA device ordinal                                       */
} afq_system_desc;

/* Zero-based CSR with int32 indices, rows sorted and columns sorted within each row,
 * as SparseMatrix::compress leaves them (src/Matrix/SparseMatrix.hpp:295-319). */
typedef struct {
  int nrows, ncols;
  const int32_t* rowIndex;  /* [nrows+1]                                                 */
  const int32_t* cols;      /* [nnz]                                                     */
  const double* vals;       /* [2*nnz] interleaved complex                               */
} afq_csr_z;

typedef struct afq_handle afq_handle;

/* Set-up: replaces base::afqmc_sys::setup (afqmc_sys.hpp:61-93) and the data
 * afqmc::Initialize + base::halfrotate_cholesky produce (miniafqmc_base.cpp:176-185). */
afq_status afq_create(const afq_system_desc* desc, afq_handle** out);
void afq_destroy(afq_handle* h);
const char* afq_status_string(afq_status s);
const char* afq_last_error(const afq_handle* h);

/* Spvn: [NMO^2 x nchol] scaled by sqrt(dt) (initialize_serial.hpp:221);
 * SpvnT: [nchol x 2*NAEA*NMO] half-rotated (rotate.hpp:69-169);
 * Propg1 [NMO][NMO]; haj [2*NAEA][NMO]; trial [2][NMO][NAEA] = conj(Wavefun)
 * (afqmc_sys.hpp:58-59); Vakbl [2*NAEA*NMO]^2 or NULL; Lhalf [nchol][2][NAEA][NMO]
 * unscaled half-rotated factors without cutoff, or NULL.  At least one of Vakbl and
 * Lhalf is needed for afq_energy. */
afq_status afq_set_hamiltonian(afq_handle* h, const afq_csr_z* Spvn, const afq_csr_z* SpvnT,
                               const double* Propg1, const double* haj, const double* trial,
                               const afq_csr_z* Vakbl, const double* Lhalf);

afq_status afq_set_walkers(afq_handle* h, const double* W, const double* W_data);
/* Copies the walkers and walker data of `src` into `dst` on the device (same NMO,
 * electrons, walker count and device; the two may be of different numerical forms), after
 * the work queued on src's stream.  No reference counterpart: it lets one form measure
 * another form's walkers (for example the mixed form's energy on the FP64 trajectory)
 * without a round trip through host memory.  Synchronous. */
afq_status afq_copy_walkers(afq_handle* dst, afq_handle* src);
afq_status afq_get_walkers(afq_handle* h, double* W, double* W_data);

/* afqmc_sys::calculate_mixed_density_matrix(W, W_data, Gc, compact=true)
 * (afqmc_sys.hpp:98-116): Gc and W_data[:,2..3] on the device. */
afq_status afq_mixed_density_matrix(afq_handle* h);
/* afqmc_sys::calculate_overlaps (afqmc_sys.hpp:136-144).  save_old != 0 first does the
 * driver's W_data[5,6,7] <- W_data[4,2,3] copy (miniafqmc_base.cpp:305-309). */
afq_status afq_overlaps(afq_handle* h, int save_old);
/* base::get_vbias(SpvnT, Gc, vbias, true) (vbias.hpp:49-63). */
afq_status afq_vbias(afq_handle* h);
/* The reference's transposed_Spvn == false path (CLI `-t no`, miniafqmc_base.cpp:265-273;
 * the flag's parsing is broken there, :120,138), in both forms (the mixed form's compact
 * Gc comes from its tensor-core density matrix; the full G and the gather are FP64):
 * afqmc_sys::calculate_mixed_density_matrix(W, W_data, G, compact=false)
 * (afqmc_sys.hpp:98-116, mixed_density_matrix.hpp:96-99) -> the full G [2][NMO][NMO] of
 * every walker (AFQ_BUF_G_FULL) plus the compact Gc and overlaps;
 * base::get_vbias(Spvn, G, vbias, false) (vbias.hpp:66-81) -> vbias = T(Spvn) G_alpha +
 * T(Spvn) G_beta.  Needs about 32 NMO^2 nwalk bytes of device memory, allocated on first
 * use. */
afq_status afq_mixed_density_matrix_full(afq_handle* h);
afq_status afq_vbias_full(afq_handle* h);
/* Driver step 2 (miniafqmc_base.cpp:281-289) with x ~ N(0,1) from Philox4x32-10
 * keyed by seed, counter (pair index, step).  afq_sigma_from takes x from the host. */
afq_status afq_sigma(afq_handle* h, uint64_t seed, uint64_t step);
afq_status afq_sigma_from(afq_handle* h, const double* x);
/* base::get_vHS(Spvn, X, vHS) (vHS.hpp:47-56). */
afq_status afq_vhs(afq_handle* h);
/* afqmc_sys::propagate(W, Propg1, vHS) (afqmc_sys.hpp:150-173), Taylor order from desc. */
afq_status afq_propagate(afq_handle* h);
/* Driver step 6 (miniafqmc_base.cpp:316-327); Eshift lives on the device. */
afq_status afq_update_weights(afq_handle* h);
/* Same weight update with the current Eshift but without replacing it; returns the
 * local sum of Re W_data[:,4] so a walker-sharded caller can all-reduce it and call
 * afq_set_eshift(global_sum / global_nwalk). */
afq_status afq_update_weights_partial(afq_handle* h, double* e4_sum);
afq_status afq_get_eshift(afq_handle* h, double* eshift);
/* Population control by the comb (systematic resampling).  No counterpart in the
 * reference, which leaves branching out (miniafqmc_base.cpp:347).  With weights
 * w_i = max(Re W_data[i][1], 0), total T and prefix sums C_i in walker order, copy j of
 * nwalk takes the first walker with C_i > (j + u) T / nwalk and weight T / nwalk; the
 * other W_data entries come with it.  u is one Philox4x32-10 uniform for (seed, step,
 * walker offset), drawn from a stream apart from the auxiliary fields', so a run restored
 * from saved walkers (afq_set_walkers, afq_set_eshift) at the same seed and step repeats
 * it.  Per handle: the blocks of a sharded ensemble (afq_set_walker_offset) comb their own
 * walkers, each with the u of its offset, and keep their own total weight.  AFQ_ERR_STATE
 * when no walker has positive weight.  Synchronous. */
afq_status afq_population_control(afq_handle* h, uint64_t seed, uint64_t step);
afq_status afq_set_eshift(afq_handle* h, double eshift);
/* Places this handle's walkers at [offset, offset+nwalk) of an ensemble of nwalk_global
 * walkers, so that the Philox stream (indexed by the global walker) gives every shard
 * the auxiliary fields the unsharded ensemble would draw.  No reference counterpart:
 * the reference runs one ensemble in one process (miniafqmc_base.cpp:282). */
afq_status afq_set_walker_offset(afq_handle* h, int offset, int nwalk_global);
/* afqmc_sys::orthogonalize (afqmc_sys.hpp:176-207): zgelqf + zunglq conventions. */
afq_status afq_orthogonalize(afq_handle* h);
/* afqmc_sys::calculate_energy (afqmc_sys.hpp:121-133) on the current Gc:
 * W_data[:,0] = eloc and *eav = sum Re(eloc) Re(w) / sum Re(w). */
afq_status afq_energy(afq_handle* h, int mode, double* eav);
/* As afq_energy, returning the two weighted sums instead of their ratio (for sharded
 * callers): sums[0] = sum Re(eloc) Re(w), sums[1] = sum Re(w). */
afq_status afq_energy_sums(afq_handle* h, int mode, double* sums);

/* One whole substep of the driver loop (miniafqmc_base.cpp:251-337) as one CUDA graph
 * launch: mixed density matrix, vbias, sigma (Philox, counter `step_tot`), vHS,
 * propagation, overlaps, weights, and orthogonalization + overlaps when
 * step_tot > 0 && step_tot % northo == 0.  Asynchronous. */
afq_status afq_substep(afq_handle* h, uint64_t seed, uint64_t step_tot, int northo);
/* The same substep for a walker-sharded ensemble (afq_set_walker_offset), in two CUDA-graph
 * launches around the one coupling of the ranks (miniafqmc_base.cpp:317-327).  No
 * reference counterpart: the reference runs one ensemble in one process.
 * afq_substep_begin runs everything up to the weight update, which uses the current
 * Eshift, and leaves this block's sum of Re W_data[:,4] in a device double owned by the
 * handle, whose address it returns in *e4sum (valid in the handle's stream order).  The
 * caller all-reduces (sums) that double in place across the ranks, ordered on the handle's
 * stream (for example NCCL on afq_get_stream's stream).  afq_substep_end then sets
 * Eshift = that sum / nwalk_global on the device and re-orthogonalises when
 * step_tot > 0 && step_tot % northo == 0.  No host synchronisation; with one rank the
 * result equals afq_substep bit for bit. */
afq_status afq_substep_begin(afq_handle* h, uint64_t seed, uint64_t step_tot, double** e4sum);
afq_status afq_substep_end(afq_handle* h, uint64_t step_tot, int northo);

/* Waits for the handle's work.  AFQ_ERR_CUDA when a tensor-core kernel's pipeline wait
 * timed out since the last call (afq_set_tc_wait_limit); the flags are cleared once
 * reported, so the next calls run normally. */
afq_status afq_synchronize(afq_handle* h);

/* Learned control variate for the exchange energy (no reference counterpart).  A
 * 36 -> hidden -> hidden -> 1 GELU network (BF16 weights, FP32 Adam at rate lr) predicts
 * each walker's exchange energy from the Coulomb vector's fixed random projection (32),
 * E_J, E_1, log|overlap| and its phase.  AFQ_ENERGY_CV evaluates the exact exchange on
 * every walker until train_walker_steps exact samples have been gathered, then on a
 * seeded random 1/subset_den of the walkers per measurement, correcting the surrogate
 * with a Horvitz-Thompson term so the weighted energy stays unbiased; the network keeps
 * training online on the exact samples.  Call after afq_set_hamiltonian with Lhalf. */
afq_status afq_cv_configure(afq_handle* h, int hidden, double lr, uint64_t seed,
                            long long train_walker_steps, int subset_den);
/* Two-level control variate (no reference counterpart): base = 1 makes the surrogate of
 * each walker's exchange energy the exchange from one plain bf16 tensor-core product
 * (the hi parts of the split operands; about a third of the exact product's work) on
 * every walker, plus the network's prediction of the exact-minus-base residual -- the
 * network's last two inputs carry the base in place of the linearised exchange.  The
 * Horvitz-Thompson correction on the exact subset keeps the estimator unbiased either
 * way; the base shrinks the residual the subset must correct, and with it the estimator's
 * sampling noise.  base = 0 (the default): the network on the step's own features.
 * Mixed form only (AFQ_ERR_UNSUPPORTED otherwise); restarts the control variate. */
afq_status afq_cv_set_base(afq_handle* h, int base);
/* stats[8] = exact samples so far, subset size of the last measurement, last training
 * loss (standardised units), estimator active (0/1), measurements, sampling variance
 * (Ha^2) that the subset correction adds to the last weighted mean energy,
 * re-standardisations of the network so far, fallback to exact exchange on every walker
 * after a non-finite training loss (0/1). */
afq_status afq_cv_stats(afq_handle* h, double* stats);

/* The surrogate network on its own (used by the control variate; exposed for testing
 * and for callers that train it offline).  Parameters are one flat fp32 vector:
 * W1[hidden][nin], b1[hidden], W2[hidden][hidden], b2[hidden], w3[hidden], b3.
 * Host arrays: x[B][nin], t[B], y[B]; B <= capacity.  The loss is
 * L = 1/(2B) sum_b (y_b - t_b)^2. */
typedef struct afq_mlp afq_mlp;
afq_status afq_mlp_create(int nin, int hidden, int capacity, uint64_t seed, afq_mlp** out);
void afq_mlp_destroy(afq_mlp* m);
long long afq_mlp_num_params(const afq_mlp* m);
afq_status afq_mlp_set_params(afq_mlp* m, const float* params);
afq_status afq_mlp_get_params(afq_mlp* m, float* params);
afq_status afq_mlp_forward(afq_mlp* m, int B, const float* x, float* y);
afq_status afq_mlp_gradient(afq_mlp* m, int B, const float* x, const float* t, float* grad,
                            float* loss);
afq_status afq_mlp_train(afq_mlp* m, int B, const float* x, const float* t, int iters, float lr,
                         float* loss);

/* Stage timers, the counterpart of the reference's NewTimer stages
 * (miniafqmc_base.cpp:50-77): with profiling on, every op-by-op call records CUDA events
 * on the handle's stream around its kernels (graph substeps are not split). */
typedef enum {
  AFQ_STAGE_DM = 0, AFQ_STAGE_VBIAS = 1, AFQ_STAGE_SIGMA = 2, AFQ_STAGE_VHS = 3,
  AFQ_STAGE_PROPAGATE = 4, AFQ_STAGE_OVERLAP = 5, AFQ_STAGE_WEIGHTS = 6,
  AFQ_STAGE_ORTHO = 7, AFQ_STAGE_ENERGY = 8, AFQ_NSTAGES = 9
} afq_stage;
afq_status afq_profile(afq_handle* h, int enable);
/* Synchronizes, then writes accumulated GPU milliseconds and kernel launches per stage
 * ([AFQ_NSTAGES] each, either may be NULL); reset != 0 clears the accumulators.
 * Launch counts include graph substeps. */
afq_status afq_stage_times(afq_handle* h, double* ms, long long* launches, int reset);
/* Kernel choices made when afq_set_hamiltonian times the candidates on the handle's own
 * shapes.  No counterpart in the reference (its kernels have fixed launch shapes).
 * choice[12]:
 *   [0..5]  mixed form, per tensor-core product site (vHS, propagation chain, split-K
 *           vbias / Coulomb, exchange over all walkers, exchange over a 1/8 subset,
 *           T1 = W^T trial): 0 built-in rule, 1 persistent kernel, 2 per-tile kernel;
 *   [6]     mixed form: split-K slice count;
 *   [7..11] FP64 form: CTA shape of the vHS CSR product, ZGEMM tile shape of the
 *           propagation chain, dense vbias, Coulomb and dense Vakbl products
 *           (0 built-in rule, k > 0 the k-th listed shape).
 * ms[24]: for mixed sites the timed milliseconds of candidates 1 and 2, for FP64 sites
 * those of the chosen shape and of the rule (0 when not timed).  Sites of the other form
 * read 0.  AFQ_TUNE=0 in the environment skips the timing, AFQ_TUNE=1 or 2 forces one
 * tensor-core kernel. */
afq_status afq_get_tuning(afq_handle* h, int* choice, double* ms);
/* FP64 form: which product the set-up tuner measured faster for each sparse operand.
 * The reference multiplies its CSR matrices with one loop (sparse.hpp:166-180, called from
 * vHS.hpp:47-56, vbias.hpp:49-63 and energy.hpp:89-97); here an operand whose density
 * reaches 2% (and whose dense copy fits in 30% of free device memory) is also held as a
 * dense row-major tile operand, both products are timed on the handle's shapes, and the
 * slower operand is freed (Spvn keeps its CSR for the full-G path).  path[3], for Spvn
 * (vHS), SpvnT (vbias) and Vakbl (energy): 1 dense-tile GEMM, 0 CSR, -1 operand absent or
 * mixed form.  ms[6]: the best milliseconds of the CSR product and of the dense product
 * per operand (0 when not timed).  With AFQ_TUNE=0 the rule is dense at >= 25% density. */
afq_status afq_get_sparse_paths(afq_handle* h, int* path, double* ms);
/* Mixed form: launch schedule the set-up tuner picked (no reference counterpart); 0s for
 * the FP64 form.
 * sched[0]: walkers per group of the propagation chain.  The chain's products (P W, the
 *   Taylor terms, P S) run group by group, so one group's Taylor sum, operands and V can
 *   stay in L2 between its products; 0 = every product over all walkers at once.  Timed:
 *   0, 32, 48, 64, 96 and 128 walkers (those below nwalk) -> ms[0..5].  Results do not
 *   depend on it.  AFQ_PROP_GROUP=<walkers> forces one.
 * sched[1]: epilogue of the vHS product over symmetric block pairs: 0 = row-wise (each
 *   lane writes its walker's entries, the mirrored block as 4-byte stores), 1 = through
 *   the fp32 tile in shared memory on the per-tile kernel (direct and mirrored rows as
 *   16-byte stores), 2 = the same with two CTAs per SM (one operand stage each, the tile
 *   staged in two halves), so one CTA's epilogue overlaps the other's main loop; the same
 *   values.  3 = as 2 with two 48 KB stages of 64-byte K slabs (SWIZZLE_64B) per CTA: the
 *   same products in another fp32 summation order (1e-6 relative).  Timed -> ms[6..9].
 *   AFQ_VHS_EPI=0..3 forces one; a forced kernel (AFQ_TUNE=1 or 2) keeps 0.
 * sched[2]: walkers per wave of the fused propagation chain, 0 = eight launches per
 *   substep.  Fused (2n a multiple of 32): the whole chain is ONE cooperative persistent
 *   launch whose tiles run in pairs of walker waves, product by product, a tile starting
 *   once every tile of the previous product of its walker is done, so a wave's V, Taylor
 *   sum and operands stay in L2 across the eight products.  Same values.  Timed -> ms[10]
 *   (eight launches), ms[11..15] (waves of 16, 24, 32, 48, 64).  AFQ_PROP_CHAIN=0 keeps
 *   the eight launches, =<walkers> forces a wave.
 * ms[16] may be NULL; 0 where not timed. */
afq_status afq_get_schedule(afq_handle* h, int* sched, double* ms);
/* The handle's CUDA stream (a cudaStream_t), for callers that order their own work
 * or events against the library's. */
afq_status afq_get_stream(afq_handle* h, void** stream);
/* Copies a device buffer to host memory in the reference layout (see afq_buffer). */
afq_status afq_copy_out(afq_handle* h, int which, void* host);

/* Exchange energy of a batch of walkers without allocating any device memory.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc: work recorded
 * into a CUDA graph under stream capture (an allocation there breaks the capture) and
 * host frameworks that own all device memory through their own pool.
 *   Lh  [nchol][2][naea][nmo] complex, unscaled half-rotated factors (device memory)
 *   Gc  [nwalk][2][naea][nmo] complex, compact density matrices, walker-major (device)
 *   ek  [nwalk] complex output (device): EK_w = 1/2 sum_{s,n} tr(T T), T = Lh_s[n] Gc_s^T
 * Lh, Gc and ek must be 16-byte aligned (the kernels move whole complex values);
 * other pointers are rejected with AFQ_ERR_ARG before any device work.
 * Asynchronous on `stream` (a cudaStream_t, NULL for the default stream).  The partial
 * sums live in one file-scope device array of 2^18 complex values (4 MiB, held by every
 * GPU that loads the library until exit): calls with 2 * nwalk * ceil(nchol / (96 /
 * naea)) above that, or with ceil(nwalk / (96 / naea)) above 65535, are rejected with
 * AFQ_ERR_UNSUPPORTED (split the walkers into batches); naea must be <= 96.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current and keeps it for the life of the process; make that first call before
 * any stream capture, and do not reset the device (cudaDeviceReset) after it, since the
 * kept address would then be stale.  All calls share the array, so calls that overlap on
 * the GPU (on different streams) race; serialise them. */
afq_status afq_exchange_energy_noalloc(const double* Lh, const double* Gc, int nmo, int naea,
                                       int nchol, int nwalk, double* ek, void* stream);

/* Heterogeneous multi-system batch (no reference counterpart; the reference runs one
 * system per process).  A batch groups handles of systems with different NMO, electron
 * count, nchol and walker count (each set up as usual, on one device, with its own
 * walkers, Hamiltonian and control variate).  afq_batch_substep advances every system by
 * one substep (the afq_substep sequence of each) with ONE CUDA-graph launch: the
 * systems' stages are parallel branches of the graph, so small systems share the GPU
 * instead of running one after another.  seeds[i] is the Philox seed of system i;
 * step_tot and northo are common.  Results equal afq_substep on each handle alone.
 * Energy measurements stay per handle (afq_energy).  The handles must not be used from
 * other threads during the call; stage profiling must be off. */
typedef struct afq_batch afq_batch;
afq_status afq_batch_create(afq_handle* const* handles, int count, afq_batch** out);
void afq_batch_destroy(afq_batch* b);
afq_status afq_batch_substep(afq_batch* b, const uint64_t* seeds, uint64_t step_tot,
                             int northo);
/* nsub (1..64) substeps of every system in ONE graph launch: substeps step_tot ..
 * step_tot + nsub - 1, each re-orthogonalising when its step_tot > 0 is a multiple of
 * northo.  The systems join once per launch instead of once per substep (use the
 * substeps between two energy measurements).  Equal to nsub afq_batch_substep calls. */
afq_status afq_batch_substeps(afq_batch* b, const uint64_t* seeds, uint64_t step_tot, int nsub,
                              int northo);
/* Fused batch: the vHS product (fused bit 1) and / or each of the propagation chain's
 * products (P W, the Taylor terms, P S; bit 2) run as ONE launch over the tiles of every
 * system, a work list of (system, walker, M tile, N tile) in one grid, instead of one
 * launch per system; the other stages stay per system on the systems' streams.  Needs
 * every handle in the mixed form with the same precisions and Taylor order, at most 4
 * systems (else AFQ_ERR_UNSUPPORTED; the batch stays as it was).  Every tile runs the
 * MMAs and epilogue arithmetic of the system's own launches, so results equal the
 * unfused batch; the joint chain writes the walkers through the shared-memory tile
 * epilogue and leaves no packed walker forms (the overlap stage packs its operand).
 * Tensor-core timeouts of the joint launches are reported on the first handle.
 * fused = 0 restores the per-system graph branches; fused = 3 joins both. */
afq_status afq_batch_set_fused(afq_batch* b, int fused);
/* Waits for the batch's work and reports any handle's tensor-core timeout flags. */
afq_status afq_batch_synchronize(afq_batch* b);

/* Half-rotation of the Cholesky tensor on the GPU: base::halfrotate_cholesky
 * (rotate.hpp:69-169) computed on `device`.
 *   SpvnT[c][s*naea*nmo + a*nmo + k] = sum_i trial_s(i, a) Spvn[i*nmo + k][c]
 * with entries of |value| <= cutoff dropped (rotate.hpp:119,156), rows and columns in
 * order.  Spvn: [nmo^2 x nchol] CSR (scaled by sqrt(dt)); trial [2][nmo][naea] as for
 * afq_set_hamiltonian.  Writes *nnz; with rowIndex != NULL also rowIndex[nchol+1], and
 * cols[nnz] / vals[2*nnz] when those are not NULL (call once without them to size the
 * buffers).  Lhalf (optional): the dense [nchol][2][naea][nmo] values times lh_scale
 * without the cutoff (lh_scale = 1/sqrt(dt) gives the unscaled factors afq_set_hamiltonian
 * takes).  Allocates and frees device memory; synchronous. */
afq_status afq_halfrotate(int device, const afq_csr_z* Spvn, int nmo, int naea, int nchol,
                          const double* trial, double cutoff, double lh_scale, long long* nnz,
                          int32_t* rowIndex, int32_t* cols, double* vals, double* Lhalf);

/* Self-test of the tensor-core GEMM used by the mixed form (no reference counterpart):
 * C[b][m][n] = sum_k A[b][m][k] B[b][n][k] for host fp32 arrays, computed on the current
 * device with bf16 operands (tf32 == 0, inputs rounded to nearest bf16) or tf32 operands,
 * fp32 accumulation, tile width bn in {64, 128, 192, 256}; K must be a multiple of 8.
 * mode 0 = one CTA per tile, 1 / 2 = persistent kernel with one / two epilogue
 * warpgroups, 3 / 4 = per-tile / persistent kernel with 64-byte K slabs (SWIZZLE_64B
 * operand tiles).  Split modes (bf16 only; hi = A rounded to bf16, lo = A - hi rounded,
 * C = hi*hi + hi*lo + lo*hi): 5 / 6 = per-tile kernel with 128- / 64-byte K slabs,
 * 7 / 8 = persistent kernel (two epilogue warpgroups) with 128- / 64-byte K slabs.
 * *kernel_err receives the kernel's timeout flags (0 when clean). */
afq_status afq_selftest_tc_gemm(int M, int N, int K, int batch, int tf32, int bn, int mode,
                                const float* A, const float* B, float* C, int* kernel_err);
/* Bound, in SM clocks, of the tensor-core kernels' pipeline waits on `device` (no
 * reference counterpart; the reference has no device code).  Each wait of a kernel's TMA
 * producer, MMA issuer and epilogue gives up after this many clocks, sets a timeout flag
 * (reported, then cleared, by afq_synchronize) and ends the kernel's work; the kernel still
 * waits, with the default bound, for the copies and MMAs it has issued before it frees its
 * tensor memory.  clocks <= 0 restores the default (2e9 clocks, about one second).  Meant
 * for tests of the timeout path and for watchdogs; it applies to every handle on the
 * device, so set it while no other work of this library runs there. */
afq_status afq_set_tc_wait_limit(int device, long long clocks);

#ifdef __cplusplus
}
#endif
#endif /* AFQMC_B200_H */
