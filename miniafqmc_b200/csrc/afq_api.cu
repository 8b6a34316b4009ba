// C ABI of libafqmc_b200 (declared in include/afqmc_b200.h): the handle, device buffers,
// one entry point per reference operation, and the CUDA-graph substep.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <algorithm>
#include <functional>
#include <mutex>
#include <map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/afqmc_b200.h"
#include "afq_cv.h"
#include "afq_kernels.h"
#include "afq_mixed.h"
#include "zgemm_fp64.cuh"

using afq::launch_csr_gather;

struct afq_handle {
  afq_system_desc d{};
  int N = 0, n = 0, nc = 0, nw = 0;
  int walker_offset = 0;     // global index of walker 0 (afq_set_walker_offset)
  long long NAK = 0;
  cudaStream_t st = nullptr;
  std::string err;
  bool have_ham = false;
  bool have_walkers = false;
  std::vector<void*> allocs;

  z_t *W = nullptr, *Wd = nullptr, *tw = nullptr, *P = nullptr, *haj = nullptr;
  z_t *Gc = nullptr, *vbias = nullptr, *X = nullptr, *hybridW = nullptr, *vHS = nullptr;
  z_t *S = nullptr, *T1 = nullptr, *T2 = nullptr;
  double* xraw = nullptr;
  int* info = nullptr;
  DevScalars* sc = nullptr;
  DevScalars* h_sc = nullptr;  // pinned mirror

  int *sp_ri = nullptr, *sp_ci = nullptr;
  z_t* sp_v = nullptr;
  double* sp_rv = nullptr;
  z_t* spT_dense = nullptr;
  int *spT_ri = nullptr, *spT_ci = nullptr;
  z_t* spT_v = nullptr;
  z_t* vk_dense = nullptr;
  int *vk_ri = nullptr, *vk_ci = nullptr;
  z_t* vk_v = nullptr;
  bool have_vakbl = false;
  z_t* Lh = nullptr;

  z_t *Gcloc = nullptr, *cvec = nullptr, *Kpart = nullptr;
  int nblk = 0;
  double* parts = nullptr;

  // FP64 form: ZGEMM tile shape per site (propagation, dense vbias, Coulomb, dense Vakbl)
  // and CTA shape of the vHS CSR product, 0 = built-in rule (fp64_tune); timings in ms of
  // the chosen shape and of the rule
  enum { F64_VHS, F64_PROP, F64_VBIAS, F64_COUL, F64_VAKBL, F64_N };
  int f64cfg[F64_N] = {0};
  float f64ms[F64_N][2] = {};
  // FP64 form: sparse operands (Spvn for vHS, SpvnT for vbias, Vakbl for the energy) keep
  // the CSR arrays and, above kDenseCandidate density and within the memory budget, a
  // dense row-major copy as well; the set-up tuner times both products and frees the
  // slower operand.  sp_path: 1 dense-tile GEMM, 0 CSR, -1 operand absent; sp_ms: best
  // milliseconds of the CSR and of the dense product (0 when not timed).
  enum { SP_SPVN, SP_SPVNT, SP_VAKBL, SP_N };
  int sp_path[SP_N] = {-1, -1, -1};
  float sp_ms[SP_N][2] = {};
  double sp_density[SP_N] = {};
  z_t* sp_dense = nullptr;   // dense Spvn [N^2][nchol] (complex values)
  double* sp_dense_r = nullptr;   // the same when every value is real
  int vhsd_cfg = 0;          // ZGEMM tile shape of the dense vHS product

  // full-G path (transposed_Spvn == false): G [nw][2][N][N] walker-major, and T(Spvn) for
  // both spins as one CSR [nchol x 2 N^2] (allocated by the first full-G call)
  z_t* Gf = nullptr;
  int *spf_ri = nullptr, *spf_ci = nullptr;
  z_t* spf_v = nullptr;
  // population control scratch (allocated by the first afq_population_control)
  double *comb_C = nullptr, *comb_w = nullptr;
  int* comb_idx = nullptr;

  afq::MixedState* mixed = nullptr;
  afq::CvState* cv = nullptr;
  afq::CvConfig cv_cfg;

  cudaGraphExec_t g_plain = nullptr, g_ortho = nullptr;
  // sharded substeps: everything up to the weight update (g_begin), the
  // re-orthogonalisation and its overlaps (g_orth); the local sum of Re W_data[:,4] for the
  // caller's all-reduce lives in e4buf
  cudaGraphExec_t g_begin = nullptr, g_orth = nullptr;
  long long g_begin_launches[AFQ_NSTAGES] = {0}, g_orth_launches[AFQ_NSTAGES] = {0};
  double* e4buf = nullptr;
  // mixed form: the T1^-1 of the last overlap / density-matrix call matches the current
  // walkers (cleared by propagate, orthogonalise and set_walkers)
  bool dm_cache = false;
  // mixed form: energies are measured on an FP64 density matrix (dm_kernel) whose
  // overlaps go to scratch, so the walkers' W_data keeps the propagation's values
  z_t* Wd_scr = nullptr;
  int* info_scr = nullptr;
  long long g_plain_launches[AFQ_NSTAGES] = {0}, g_ortho_launches[AFQ_NSTAGES] = {0};
  unsigned long long host_seed = ~0ull, host_step = ~0ull;

  // stage timers
  struct Rec {
    int stage;
    cudaEvent_t a, b;
  };
  bool profiling = false;
  bool capturing = false;
  std::vector<Rec> recs;
  size_t nrec = 0;
  double stage_ms[AFQ_NSTAGES] = {0};
  long long stage_launches[AFQ_NSTAGES] = {0};
  long long* launch_sink = nullptr;   // where launch counts go (capture counts per graph)
};

namespace {

const double kDenseThreshold = 0.25;  // built-in rule: a CSR operand above this density is
                                      // multiplied as a dense tile (the mixed form needs it)
const double kDenseCandidate = 0.02;  // FP64 form: below this density the CSR product wins
                                      // without timing; above it both paths are timed

afq_status fail(afq_handle* h, afq_status s, const std::string& msg) {
  if (h) h->err = msg;
  return s;
}

#define AFQ_CUDA(h, call)                                                               \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(h, e_ == cudaErrorMemoryAllocation ? AFQ_ERR_OOM : AFQ_ERR_CUDA,      \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                 \
  } while (0)

template <class T>
cudaError_t dalloc(afq_handle* h, T** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * (count ? count : 1));
  if (e != cudaSuccess) return e;
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return cudaSuccess;
}

void dfree(afq_handle* h, void* p) {
  if (!p) return;
  for (auto& q : h->allocs)
    if (q == p) {
      cudaFree(q);
      q = nullptr;
    }
}

// Scatters a real CSR into a zeroed dense row-major matrix of doubles.
__global__ void csr_to_dense_real_kernel(const int* ri, const int* ci, const double* rv, int nrows,
                                         long long ncols, double* out) {
  int r = blockIdx.x * blockDim.y + threadIdx.y;
  if (r >= nrows) return;
  for (int p = ri[r] + threadIdx.x; p < ri[r + 1]; p += blockDim.x)
    out[(long long)r * ncols + ci[p]] = rv[p];
}

// Scatters a CSR into a zeroed dense row-major matrix; rv (real values) replaces v when
// non-null.
__global__ void csr_to_dense_kernel(const int* ri, const int* ci, const z_t* v, const double* rv,
                                    int nrows, long long ncols, z_t* out) {
  int r = blockIdx.x * blockDim.y + threadIdx.y;
  if (r >= nrows) return;
  for (int p = ri[r] + threadIdx.x; p < ri[r + 1]; p += blockDim.x)
    out[(long long)r * ncols + ci[p]] = rv ? zmk(rv[p], 0.0) : v[p];
}

// Dense copy of a device CSR (rows x cols) into a new buffer, when the density reaches
// kDenseCandidate and the copy takes at most 30% of the free device memory; else *dense
// stays null.
afq_status densify(afq_handle* h, const int* ri, const int* ci, const z_t* v, const double* rv,
                   int nrows, long long ncols, double density, z_t** dense) {
  *dense = nullptr;
  if (density < kDenseCandidate) return AFQ_OK;
  const size_t cnt = (size_t)nrows * (size_t)ncols;
  size_t free_b = 0, total_b = 0;
  AFQ_CUDA(h, cudaMemGetInfo(&free_b, &total_b));
  if (sizeof(z_t) * cnt > free_b / 10 * 3) return AFQ_OK;
  // the CSR arrays came up by pageable copies whose DMA may still be in flight
  AFQ_CUDA(h, cudaDeviceSynchronize());
  AFQ_CUDA(h, dalloc(h, dense, cnt));
  AFQ_CUDA(h, cudaMemsetAsync(*dense, 0, sizeof(z_t) * cnt, h->st));
  csr_to_dense_kernel<<<(nrows + 7) / 8, dim3(32, 8), 0, h->st>>>(ri, ci, v, rv, nrows, ncols,
                                                                  *dense);
  AFQ_CUDA(h, cudaGetLastError());
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  return AFQ_OK;
}

afq_status check_csr(afq_handle* h, const afq_csr_z* m, int nrows, int ncols, const char* name) {
  if (!m || !m->rowIndex || !m->cols || !m->vals)
    return fail(h, AFQ_ERR_ARG, std::string(name) + ": null CSR");
  if (m->nrows != nrows || m->ncols != ncols)
    return fail(h, AFQ_ERR_ARG, std::string(name) + ": wrong shape");
  if (m->rowIndex[0] != 0) return fail(h, AFQ_ERR_ARG, std::string(name) + ": rowIndex[0] != 0");
  long long nnz = m->rowIndex[nrows];
  for (int r = 0; r < nrows; r++)
    if (m->rowIndex[r + 1] < m->rowIndex[r])
      return fail(h, AFQ_ERR_ARG, std::string(name) + ": rowIndex not monotone");
  for (long long p = 0; p < nnz; p++)
    if (m->cols[p] < 0 || m->cols[p] >= ncols)
      return fail(h, AFQ_ERR_ARG, std::string(name) + ": column index out of range");
  return AFQ_OK;
}

// Uploads a CSR.  keep_both (FP64 form): a dense copy is added next to the CSR arrays
// when densify allows one (the tuner keeps the faster).  Otherwise, when dense_out is
// non-null and the density reaches kDenseThreshold, a dense row-major copy is built on
// the device instead and the CSR arrays are released.
afq_status upload_csr(afq_handle* h, const afq_csr_z* m, int** ri, int** ci, z_t** v,
                      z_t** dense_out, bool allow_dense, bool keep_both = false,
                      double* density = nullptr) {
  long long nnz = m->rowIndex[m->nrows];
  AFQ_CUDA(h, dalloc(h, ri, m->nrows + 1));
  AFQ_CUDA(h, dalloc(h, ci, nnz));
  AFQ_CUDA(h, dalloc(h, v, nnz));
  AFQ_CUDA(h, cudaMemcpy(*ri, m->rowIndex, sizeof(int) * (m->nrows + 1), cudaMemcpyHostToDevice));
  AFQ_CUDA(h, cudaMemcpy(*ci, m->cols, sizeof(int) * nnz, cudaMemcpyHostToDevice));
  AFQ_CUDA(h, cudaMemcpy(*v, m->vals, sizeof(z_t) * nnz, cudaMemcpyHostToDevice));
  double dens = (double)nnz / ((double)m->nrows * (double)m->ncols);
  if (density) *density = dens;
  if (dense_out) *dense_out = nullptr;
  if (keep_both && dense_out)
    return densify(h, *ri, *ci, *v, nullptr, m->nrows, m->ncols, dens, dense_out);
  if (allow_dense && dense_out && dens >= kDenseThreshold) {
    size_t cnt = (size_t)m->nrows * m->ncols;
    AFQ_CUDA(h, cudaDeviceSynchronize());   // pageable uploads above
    AFQ_CUDA(h, dalloc(h, dense_out, cnt));
    AFQ_CUDA(h, cudaMemsetAsync(*dense_out, 0, sizeof(z_t) * cnt, h->st));
    csr_to_dense_kernel<<<(m->nrows + 7) / 8, dim3(32, 8), 0, h->st>>>(*ri, *ci, *v, nullptr,
                                                                       m->nrows, m->ncols,
                                                                       *dense_out);
    AFQ_CUDA(h, cudaGetLastError());
    AFQ_CUDA(h, cudaStreamSynchronize(h->st));
    dfree(h, *ri); dfree(h, *ci); dfree(h, *v);
    *ri = nullptr; *ci = nullptr; *v = nullptr;
  }
  return AFQ_OK;
}

cudaError_t collect_stage_times(afq_handle* h) {
  if (h->nrec == 0) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return e;
  for (size_t i = 0; i < h->nrec; i++) {
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, h->recs[i].a, h->recs[i].b);
    if (e != cudaSuccess) return e;
    h->stage_ms[h->recs[i].stage] += ms;
  }
  h->nrec = 0;
  return cudaSuccess;
}

// Runs one stage body, counting its kernel launches and, with profiling on (and outside
// stream capture), bracketing it with CUDA events on the handle's stream.
// NVTX range per stage call, in the library's own domain "afqmc_b200" (a profiler shows
// the reference's stage names on the timeline; the caller's ranges in the default domain
// keep their own stack).  Host-only and without effect unless a tool is attached.
struct StageRange {
  explicit StageRange(int stage) {
    static nvtxDomainHandle_t dom = nvtxDomainCreateA("afqmc_b200");
    static const char* const names[AFQ_NSTAGES] = {
        "mixed density matrix", "bias potential", "sigma", "H-S potential", "propagation",
        "overlap", "weights", "orthogonalization", "local energy"};
    nvtxEventAttributes_t a{};
    a.version = NVTX_VERSION;
    a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
    a.messageType = NVTX_MESSAGE_TYPE_ASCII;
    a.message.ascii = (stage >= 0 && stage < AFQ_NSTAGES) ? names[stage] : "stage";
    dom_ = dom;
    nvtxDomainRangePushEx(dom_, &a);
  }
  ~StageRange() { nvtxDomainRangePop(dom_); }
  StageRange(const StageRange&) = delete;
  StageRange& operator=(const StageRange&) = delete;

 private:
  nvtxDomainHandle_t dom_;
};

template <class F>
cudaError_t staged(afq_handle* h, int stage, int nlaunch, F&& body) {
  (h->launch_sink ? h->launch_sink : h->stage_launches)[stage] += nlaunch;
  StageRange range(stage);
  if (!h->profiling || h->capturing) return body();
  if (h->nrec == 4096) {
    cudaError_t e = collect_stage_times(h);
    if (e != cudaSuccess) return e;
  }
  if (h->nrec == h->recs.size()) {
    afq_handle::Rec r{};
    cudaError_t e = cudaEventCreate(&r.a);
    if (e == cudaSuccess) e = cudaEventCreate(&r.b);
    if (e != cudaSuccess) return e;
    h->recs.push_back(r);
  }
  afq_handle::Rec& r = h->recs[h->nrec++];
  r.stage = stage;
  cudaError_t e = cudaEventRecord(r.a, h->st);
  if (e != cudaSuccess) return e;
  e = body();
  if (e != cudaSuccess) return e;
  return cudaEventRecord(r.b, h->st);
}

afq_status need_ready(afq_handle* h) {
  if (!h) return AFQ_ERR_ARG;
  if (!h->have_ham) return fail(h, AFQ_ERR_STATE, "Hamiltonian not set");
  if (!h->have_walkers) return fail(h, AFQ_ERR_STATE, "walkers not set");
  return AFQ_OK;
}

// ------------------------------------------------------------ stage bodies (async)
bool mixed_dm_on(const afq_handle* h) { return h->mixed && afq::mixed_has_dm(h->mixed); }

cudaError_t body_dm(afq_handle* h, int want_gc, int save_old) {
  if (mixed_dm_on(h)) {
    cudaError_t e = afq::mixed_dm(h->mixed, h->W, h->Gc, h->Wd, h->info, want_gc, save_old,
                                  h->dm_cache ? 1 : 0, h->st);
    h->dm_cache = e == cudaSuccess;
    return e;
  }
  return afq::launch_dm(h->W, h->tw, h->N, h->n, h->nw, h->Gc, h->Wd, h->info, want_gc, save_old,
                        h->st);
}

cudaError_t body_vbias(afq_handle* h) {
  if (h->mixed) return afq::mixed_vbias(h->mixed, h->Gc, h->vbias, h->st);
  if (h->spT_dense) {
    ZGemmDesc g{h->nc, h->nw, (int)h->NAK, h->spT_dense, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
    EpiStore e{h->vbias, h->nw, 0, zmk(0, 0), 0};
    return zgemm_launch<true, true>(g, 1, e, h->st, h->f64cfg[afq_handle::F64_VBIAS]);
  }
  return launch_csr_gather(h->spT_ri, h->spT_ci, h->spT_v, h->Gc, h->NAK, h->nc, h->nw, h->vbias,
                           h->st);
}

cudaError_t body_sigma(afq_handle* h, int use_xraw) {
  return afq::launch_sigma(h->vbias, h->X, h->xraw, h->hybridW, h->nc, h->nw, h->sc, use_xraw,
                           h->st);
}

// vHS^T [w][ik] = sum_c X[c][w] Spvn[ik][c] with the dense Spvn: one ZGEMM of M = nw,
// N = NMO^2, K = nchol writing each walker's matrix row by row (real x complex
// multiply-adds when Spvn is real).
cudaError_t dense_vhs(afq_handle* h, int cfg) {
  const long long NN = (long long)h->N * h->N;
  ZGemmDesc g{h->nw, (int)NN, h->nc, h->X, h->nw, 0, h->sp_dense, h->nc, 0, zmk(1, 0)};
  EpiStore ep{h->vHS, NN, 0, zmk(0, 0), 0};
  if (h->sp_dense_r) {
    g.Br = h->sp_dense_r;
    return zgemm_launch<false, true, EpiStore, true>(g, 1, ep, h->st, cfg);
  }
  return zgemm_launch<false, true>(g, 1, ep, h->st, cfg);
}

cudaError_t body_vhs(afq_handle* h) {
  if (h->mixed) return afq::mixed_vhs(h->mixed, h->X, h->vHS, h->st);
  if (h->sp_dense || h->sp_dense_r) return dense_vhs(h, h->vhsd_cfg);
  return afq::launch_csr_walker(h->sp_ri, h->sp_ci, h->sp_v, h->sp_rv, h->X, h->N * h->N, h->nw,
                                h->vHS, (long long)h->N * h->N, h->st,
                                h->f64cfg[afq_handle::F64_VHS]);
}

cudaError_t body_propagate(afq_handle* h) {
  h->dm_cache = false;
  if (h->mixed) return afq::mixed_propagate(h->mixed, h->W, h->vHS, h->st);
  const int N = h->N, n2 = 2 * h->n, nw = h->nw;
  const long long sWN = (long long)N * n2, sV = (long long)N * N;
  const int zc = h->f64cfg[afq_handle::F64_PROP];
  cudaError_t e;
  {  // S = P W, T1 = S
    ZGemmDesc g{N, n2, N, h->P, N, 0, h->W, n2, sWN, zmk(1, 0)};
    EpiDual ep{h->T1, h->S, n2, sWN};
    if ((e = zgemm_launch<true, false>(g, nw, ep, h->st, zc)) != cudaSuccess) return e;
  }
  z_t* cur = h->T1;
  z_t* nxt = h->T2;
  for (int k = 1; k <= h->d.taylor_order; k++) {  // T = (i/k) V T; S += T
    ZGemmDesc g{N, n2, N, h->vHS, N, sV, cur, n2, sWN, zmk(0.0, 1.0 / (double)k)};
    EpiTaylor ep{nxt, h->S, n2, sWN};
    if ((e = zgemm_launch<true, false>(g, nw, ep, h->st, zc)) != cudaSuccess) return e;
    std::swap(cur, nxt);
  }
  {  // W = P S
    ZGemmDesc g{N, n2, N, h->P, N, 0, h->S, n2, sWN, zmk(1, 0)};
    EpiStore ep{h->W, n2, sWN, zmk(0, 0), 0};
    if ((e = zgemm_launch<true, false>(g, nw, ep, h->st, zc)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t body_weights(afq_handle* h, int update_eshift) {
  return afq::launch_weights(h->Wd, h->hybridW, h->nw, h->d.dt, h->sc, update_eshift, h->st);
}

// The FP64 form keeps LAPACK's Householder convention (raw overlaps match the
// reference); the mixed form uses CholeskyQR2, equal up to column signs.
cudaError_t body_ortho(afq_handle* h) {
  h->dm_cache = false;
  if (h->mixed) {   // then the packed operand forms of the new walkers
    cudaError_t e = afq::launch_ortho_cholqr(h->W, h->N, h->n, h->nw, h->info, h->st);
    return e == cudaSuccess ? afq::mixed_repack(h->mixed, h->W, h->st) : e;
  }
  return afq::launch_ortho(h->W, h->N, h->n, h->nw, h->st);
}

cudaError_t body_energy(afq_handle* h, int mode) {
  cudaError_t e;
  const int nak = (int)h->NAK;
  if (mode == AFQ_ENERGY_VAKBL) {
    if (h->vk_dense) {
      ZGemmDesc g{nak, h->nw, nak, h->vk_dense, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
      EpiStore ep{h->Gcloc, h->nw, 0, zmk(0, 0), 0};
      if ((e = zgemm_launch<true, true>(g, 1, ep, h->st, h->f64cfg[afq_handle::F64_VAKBL])) !=
          cudaSuccess)
        return e;
    } else {
      if ((e = launch_csr_gather(h->vk_ri, h->vk_ci, h->vk_v, h->Gc, h->NAK, nak, h->nw, h->Gcloc,
                                 h->st)) != cudaSuccess)
        return e;
    }
    if ((e = afq::launch_energy_reduce(h->Gc, h->haj, nak, h->Gcloc, nullptr, 0, nullptr, 0, h->nw,
                                       0, h->Wd, nullptr, h->st)) != cudaSuccess)
      return e;
  } else {
    if (h->mixed) {
      if ((e = afq::mixed_energy_chol(h->mixed, h->Gc, h->cvec, h->Kpart, h->nblk, h->st)) !=
          cudaSuccess)
        return e;
    } else {
      ZGemmDesc g{h->nc, h->nw, nak, h->Lh, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
      EpiStore ep{h->cvec, h->nw, 0, zmk(0, 0), 0};
      if ((e = zgemm_launch<true, true>(g, 1, ep, h->st, h->f64cfg[afq_handle::F64_COUL])) !=
          cudaSuccess)
        return e;
      int nb = 0;
      if ((e = afq::launch_exchange(h->Lh, h->Gc, h->N, h->n, h->nc, h->nw, h->Kpart, &nb,
                                    h->st)) != cudaSuccess)
        return e;
    }
    if ((e = afq::launch_energy_reduce(h->Gc, h->haj, nak, nullptr, h->cvec, h->nc, h->Kpart,
                                       h->nblk, h->nw, 1, h->Wd, h->parts, h->st)) != cudaSuccess)
      return e;
  }
  return afq::launch_eav(h->Wd, h->nw, h->sc, h->st);
}

// Timed / counted stages.  The launch counts are the kernels each body issues.
cudaError_t st_dm(afq_handle* h, int want_gc, int save_old) {
  const int stage = want_gc ? AFQ_STAGE_DM : AFQ_STAGE_OVERLAP;
  const int nl = !mixed_dm_on(h) ? 1 : (want_gc && h->dm_cache) ? 3 : afq::mixed_launches(h->mixed, stage);
  return staged(h, stage, nl, [&] { return body_dm(h, want_gc, save_old); });
}
cudaError_t st_vbias(afq_handle* h) {
  int nl = h->mixed ? afq::mixed_launches(h->mixed, AFQ_STAGE_VBIAS) : 1;
  return staged(h, AFQ_STAGE_VBIAS, nl, [&] { return body_vbias(h); });
}
cudaError_t st_sigma(afq_handle* h, int use_xraw) {
  return staged(h, AFQ_STAGE_SIGMA, 1, [&] { return body_sigma(h, use_xraw); });
}
cudaError_t st_vhs(afq_handle* h) {
  int nl = h->mixed ? afq::mixed_launches(h->mixed, AFQ_STAGE_VHS) : 1;
  return staged(h, AFQ_STAGE_VHS, nl, [&] { return body_vhs(h); });
}
cudaError_t st_propagate(afq_handle* h) {
  int nl = h->mixed ? afq::mixed_launches(h->mixed, AFQ_STAGE_PROPAGATE) : h->d.taylor_order + 2;
  return staged(h, AFQ_STAGE_PROPAGATE, nl, [&] { return body_propagate(h); });
}
cudaError_t st_weights(afq_handle* h, int update_eshift) {
  return staged(h, AFQ_STAGE_WEIGHTS, 1, [&] { return body_weights(h, update_eshift); });
}
cudaError_t st_ortho(afq_handle* h) {
  return staged(h, AFQ_STAGE_ORTHO, 1 + (h->mixed ? afq::mixed_repack_launches(h->mixed) : 0),
                [&] { return body_ortho(h); });
}
cudaError_t st_energy(afq_handle* h, int mode) {
  int nl = mode == AFQ_ENERGY_VAKBL ? 3
           : (h->mixed ? afq::mixed_launches(h->mixed, AFQ_STAGE_ENERGY) + 2 : 5);
  return staged(h, AFQ_STAGE_ENERGY, nl, [&] { return body_energy(h, mode); });
}

// One substep; part 0 = all of it, 1 = up to the weight update without the Eshift update
// (sharded: the caller all-reduces the sum first), 2 = the re-orthogonalisation only.
cudaError_t st_substep(afq_handle* h, bool ortho, int part = 0) {
  cudaError_t e;
  if (part != 2) {
    if ((e = st_dm(h, 1, 0)) != cudaSuccess) return e;
    if ((e = st_vbias(h)) != cudaSuccess) return e;
    if ((e = st_sigma(h, 0)) != cudaSuccess) return e;
    if ((e = st_vhs(h)) != cudaSuccess) return e;
    if ((e = st_propagate(h)) != cudaSuccess) return e;
    if ((e = st_dm(h, 0, 1)) != cudaSuccess) return e;
    if ((e = st_weights(h, part == 1 ? 0 : 1)) != cudaSuccess) return e;
  }
  if (ortho && part != 1) {
    if ((e = st_ortho(h)) != cudaSuccess) return e;
    if ((e = st_dm(h, 0, 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

afq_status set_scalars(afq_handle* h, uint64_t seed, uint64_t step) {
  AFQ_CUDA(h, afq::launch_set_scalars(h->sc, seed, step, 0, 0.0, h->st));
  h->host_seed = seed;
  h->host_step = step;
  return AFQ_OK;
}

// Captures (once) and launches one substep graph: part as for st_substep.
afq_status launch_substep_graph(afq_handle* h, cudaGraphExec_t* slot, long long* counts,
                                bool ortho, int part) {
  if (!*slot) {
    cudaGraph_t g = nullptr;
    AFQ_CUDA(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed));
    h->capturing = true;
    for (int i = 0; i < AFQ_NSTAGES; i++) counts[i] = 0;
    h->launch_sink = counts;
    cudaError_t e = st_substep(h, ortho, part);
    h->launch_sink = nullptr;
    h->capturing = false;
    cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(h, AFQ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    }
    AFQ_CUDA(h, e2);
    e = cudaGraphInstantiate(slot, g, 0);
    cudaGraphDestroy(g);
    AFQ_CUDA(h, e);
  }
  AFQ_CUDA(h, cudaGraphLaunch(*slot, h->st));
  for (int i = 0; i < AFQ_NSTAGES; i++) h->stage_launches[i] += counts[i];
  return AFQ_OK;
}

void drop_graphs(afq_handle* h) {
  for (cudaGraphExec_t* g : {&h->g_plain, &h->g_ortho, &h->g_begin, &h->g_orth}) {
    if (*g) cudaGraphExecDestroy(*g);
    *g = nullptr;
  }
}

// FP64 form: times the tile shapes of its ZGEMM sites and the CTA shapes of the vHS CSR
// product on the handle's shapes (per-step scratch zeroed, products written to scratch)
// and keeps the fastest.  Every shape sums each output in the same order, so results do
// not depend on the choice.  A candidate whose first call takes over 3x the best so far is
// dropped after that call; calls over 20 ms are timed once.  Choices are cached per shape
// for the process.  AFQ_TUNE=0 keeps the built-in rules.
// Keeps one form of each sparse operand of the FP64 form: dense[op] keeps the dense copy
// (and frees the CSR arrays of SpvnT / Vakbl; Spvn's CSR stays for the full-G path),
// otherwise the dense copy is freed.
void keep_paths(afq_handle* h, const int* dense) {
  auto one = [&](int op, z_t** d, int** ri, int** ci, z_t** v, bool free_csr) {
    if (h->sp_path[op] < 0) return;
    if (dense[op] && *d) {
      if (free_csr) {
        dfree(h, *ri); dfree(h, *ci); dfree(h, *v);
        *ri = nullptr; *ci = nullptr; *v = nullptr;
      }
      h->sp_path[op] = 1;
    } else {
      if (*d) dfree(h, *d);
      *d = nullptr;
      h->sp_path[op] = 0;
    }
  };
  int *r0 = nullptr, *c0 = nullptr;
  z_t* v0 = nullptr;
  if (h->sp_dense_r) {   // real dense Spvn: the CSR stays either way
    if (h->sp_path[afq_handle::SP_SPVN] >= 0) {
      if (dense[afq_handle::SP_SPVN]) {
        h->sp_path[afq_handle::SP_SPVN] = 1;
      } else {
        dfree(h, h->sp_dense_r);
        h->sp_dense_r = nullptr;
        h->sp_path[afq_handle::SP_SPVN] = 0;
      }
    }
  } else {
    one(afq_handle::SP_SPVN, &h->sp_dense, &r0, &c0, &v0, false);
  }
  one(afq_handle::SP_SPVNT, &h->spT_dense, &h->spT_ri, &h->spT_ci, &h->spT_v, true);
  one(afq_handle::SP_VAKBL, &h->vk_dense, &h->vk_ri, &h->vk_ci, &h->vk_v, true);
}

// FP64 form, built-in rule for the sparse operands: dense above kDenseThreshold.
void rule_paths(afq_handle* h) {
  int dense[afq_handle::SP_N];
  for (int i = 0; i < afq_handle::SP_N; i++) dense[i] = h->sp_density[i] >= kDenseThreshold;
  keep_paths(h, dense);
}

cudaError_t fp64_tune(afq_handle* h) {
  const char* env = getenv("AFQ_TUNE");
  if (env && atoi(env) == 0) {
    rule_paths(h);
    return cudaSuccess;
  }
  static std::mutex mu;
  static std::map<std::string, std::vector<float>> cache;
  char key[200];
  snprintf(key, sizeof key, "N%d_n%d_nc%d_nw%d_sp%lld_d%d%d%d_l%d_v%d_p%d%d%d", h->N, h->n, h->nc,
           h->nw, h->sp_ri ? 1LL : 0LL, (h->sp_dense || h->sp_dense_r) ? 1 : 0, h->spT_dense ? 1 : 0,
           h->vk_dense ? 1 : 0, h->Lh ? 1 : 0, h->sp_rv ? 1 : 0, h->sp_path[0], h->sp_path[1],
           h->sp_path[2]);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      const std::vector<float>& c = it->second;
      for (int i = 0; i < afq_handle::F64_N; i++) {
        h->f64cfg[i] = (int)c[3 * i];
        h->f64ms[i][0] = c[3 * i + 1];
        h->f64ms[i][1] = c[3 * i + 2];
      }
      const size_t o = 3 * afq_handle::F64_N;
      int dense[afq_handle::SP_N];
      for (int i = 0; i < afq_handle::SP_N; i++) {
        dense[i] = (int)c[o + 3 * i];
        h->sp_ms[i][0] = c[o + 3 * i + 1];
        h->sp_ms[i][1] = c[o + 3 * i + 2];
      }
      h->vhsd_cfg = (int)c[o + 3 * afq_handle::SP_N];
      keep_paths(h, dense);
      return cudaSuccess;
    }
  }
  const int N = h->N, n2 = 2 * h->n, nw = h->nw, nak = (int)h->NAK;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  A(cudaMemsetAsync(h->vHS, 0, sizeof(z_t) * (size_t)nw * N * N, h->st));
  A(cudaMemsetAsync(h->T1, 0, sizeof(z_t) * (size_t)nw * N * n2, h->st));
  A(cudaMemsetAsync(h->X, 0, sizeof(z_t) * (size_t)h->nc * nw, h->st));
  A(cudaMemsetAsync(h->Gc, 0, sizeof(z_t) * (size_t)nw * nak, h->st));
  cudaEvent_t ev[4] = {};
  for (auto& x : ev) A(cudaEventCreate(&x));
  A(cudaStreamSynchronize(h->st));
  // median (or single) time of one call after a warm-up call; < 0 when it fails
  auto timed = [&](const std::function<cudaError_t()>& run, float cap) -> float {
    if (e != cudaSuccess) return -1.0f;
    cudaEventRecord(ev[0], h->st);
    if (run() != cudaSuccess) {
      cudaGetLastError();
      return -1.0f;
    }
    cudaEventRecord(ev[1], h->st);
    float t0 = -1.0f;
    if (cudaEventSynchronize(ev[1]) != cudaSuccess) {
      e = cudaGetLastError();
      return -1.0f;
    }
    cudaEventElapsedTime(&t0, ev[0], ev[1]);
    if (t0 > cap) return t0;        // far slower than the best: not a contender
    if (t0 > 20.0f) {               // long call: time it once more, alone
      cudaEventRecord(ev[0], h->st);
      run();
      cudaEventRecord(ev[1], h->st);
      cudaEventSynchronize(ev[1]);
      cudaEventElapsedTime(&t0, ev[0], ev[1]);
      return t0;
    }
    cudaEventRecord(ev[0], h->st);
    for (int r = 0; r < 3; r++) {
      run();
      cudaEventRecord(ev[r + 1], h->st);
    }
    if (cudaEventSynchronize(ev[3]) != cudaSuccess) {
      e = cudaGetLastError();
      return -1.0f;
    }
    float t[3];
    for (int r = 0; r < 3; r++) cudaEventElapsedTime(&t[r], ev[r], ev[r + 1]);
    std::sort(t, t + 3);
    return t[1];
  };
  struct Best {
    int cfg = 0;
    float ms = -1.0f, rule = -1.0f;
  };
  auto fastest = [&](int ncfg, const std::function<cudaError_t(int)>& run) {
    Best b;
    for (int c = 0; c <= ncfg; c++) {
      const float t = timed([&] { return run(c); }, b.ms > 0.0f ? 3.0f * b.ms : 1e30f);
      if (c == 0) b.rule = t;
      if (t > 0.0f && (b.ms < 0.0f || t < b.ms)) {
        b.ms = t;
        b.cfg = c;
      }
    }
    return b;
  };
  auto pick = [&](int site, int ncfg, const std::function<cudaError_t(int)>& run) {
    const Best b = fastest(ncfg, run);
    h->f64cfg[site] = b.cfg;
    h->f64ms[site][0] = b.ms > 0.0f ? b.ms : 0.0f;
    h->f64ms[site][1] = b.rule > 0.0f ? b.rule : 0.0f;
    return b;
  };
  // dense or CSR for each sparse operand: the faster of the two best shapes
  int dense[afq_handle::SP_N] = {0, 0, 0};
  auto choose = [&](int op, float t_csr, float t_dense) {
    h->sp_ms[op][0] = t_csr > 0.0f ? t_csr : 0.0f;
    h->sp_ms[op][1] = t_dense > 0.0f ? t_dense : 0.0f;
    dense[op] = t_dense > 0.0f && (t_csr <= 0.0f || t_dense < t_csr);
  };
  {
    const Best bc = pick(afq_handle::F64_VHS, afq::kCsrWalkerCfgs, [&](int c) {
      return afq::launch_csr_walker(h->sp_ri, h->sp_ci, h->sp_v, h->sp_rv, h->X, N * N, nw, h->vHS,
                                    (long long)N * N, h->st, c);
    });
    Best bd;
    if (h->sp_dense || h->sp_dense_r) {
      bd = fastest(kZgCfgs, [&](int c) { return dense_vhs(h, c); });
      h->vhsd_cfg = bd.cfg;
    }
    choose(afq_handle::SP_SPVN, bc.ms, bd.ms);
  }
  pick(afq_handle::F64_PROP, kZgCfgs, [&](int c) {   // T2 = (i/k) V T1 of every walker
    ZGemmDesc g{N, n2, N, h->vHS, N, (long long)N * N, h->T1, n2, (long long)N * n2, zmk(0, 1)};
    EpiStore ep{h->T2, n2, (long long)N * n2, zmk(0, 0), 0};
    return zgemm_launch<true, false>(g, nw, ep, h->st, c);
  });
  if (h->sp_path[afq_handle::SP_SPVNT] >= 0) {
    Best bd, bc;
    if (h->spT_dense)
      bd = pick(afq_handle::F64_VBIAS, kZgCfgs, [&](int c) {
        ZGemmDesc g{h->nc, nw, nak, h->spT_dense, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
        EpiStore ep{h->vbias, nw, 0, zmk(0, 0), 0};
        return zgemm_launch<true, true>(g, 1, ep, h->st, c);
      });
    if (h->spT_ri)
      bc = fastest(0, [&](int) {
        return launch_csr_gather(h->spT_ri, h->spT_ci, h->spT_v, h->Gc, h->NAK, h->nc, nw,
                                 h->vbias, h->st);
      });
    choose(afq_handle::SP_SPVNT, bc.ms, bd.ms);
  }
  if (h->Lh && h->cvec)
    pick(afq_handle::F64_COUL, kZgCfgs, [&](int c) {
      ZGemmDesc g{h->nc, nw, nak, h->Lh, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
      EpiStore ep{h->cvec, nw, 0, zmk(0, 0), 0};
      return zgemm_launch<true, true>(g, 1, ep, h->st, c);
    });
  if (h->sp_path[afq_handle::SP_VAKBL] >= 0 && h->Gcloc) {
    Best bd, bc;
    if (h->vk_dense)
      bd = pick(afq_handle::F64_VAKBL, kZgCfgs, [&](int c) {
        ZGemmDesc g{nak, nw, nak, h->vk_dense, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
        EpiStore ep{h->Gcloc, nw, 0, zmk(0, 0), 0};
        return zgemm_launch<true, true>(g, 1, ep, h->st, c);
      });
    if (h->vk_ri)
      bc = fastest(0, [&](int) {
        return launch_csr_gather(h->vk_ri, h->vk_ci, h->vk_v, h->Gc, h->NAK, nak, nw, h->Gcloc,
                                 h->st);
      });
    choose(afq_handle::SP_VAKBL, bc.ms, bd.ms);
  }
  for (auto& x : ev)
    if (x) cudaEventDestroy(x);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) return e;
  if (getenv("AFQ_TUNE_VERBOSE"))
    fprintf(stderr, "afq tune fp64: vhs %s (%.3f, rule %.3f) prop %s (%.3f, %.3f) vbias %s "
            "(%.3f, %.3f) coulomb %s (%.3f, %.3f) vakbl %s (%.3f, %.3f) ms\n",
            afq::csr_walker_cfg_name(h->f64cfg[0]), h->f64ms[0][0], h->f64ms[0][1],
            zgemm_cfg_name(h->f64cfg[1]), h->f64ms[1][0], h->f64ms[1][1],
            zgemm_cfg_name(h->f64cfg[2]), h->f64ms[2][0], h->f64ms[2][1],
            zgemm_cfg_name(h->f64cfg[3]), h->f64ms[3][0], h->f64ms[3][1],
            zgemm_cfg_name(h->f64cfg[4]), h->f64ms[4][0], h->f64ms[4][1]);
  std::vector<float> rec;
  for (int i = 0; i < afq_handle::F64_N; i++) {
    rec.push_back((float)h->f64cfg[i]);
    rec.push_back(h->f64ms[i][0]);
    rec.push_back(h->f64ms[i][1]);
  }
  for (int i = 0; i < afq_handle::SP_N; i++) {
    rec.push_back((float)dense[i]);
    rec.push_back(h->sp_ms[i][0]);
    rec.push_back(h->sp_ms[i][1]);
  }
  rec.push_back((float)h->vhsd_cfg);
  keep_paths(h, dense);
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = rec;
  return cudaSuccess;
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
    case AFQ_ERR_UNSUPPORTED: return "unsupported size or option";
    case AFQ_ERR_SINGULAR: return "singular overlap matrix";
  }
  return "unknown status";
}

const char* afq_last_error(const afq_handle* h) { return h ? h->err.c_str() : ""; }

afq_status afq_create(const afq_system_desc* desc, afq_handle** out) {
  if (!desc || !out) return AFQ_ERR_ARG;
  *out = nullptr;
  if (desc->nmo <= 0 || desc->naea <= 0 || desc->nchol <= 0 || desc->nwalk <= 0 ||
      desc->taylor_order < 0 || !(desc->dt > 0.0))
    return AFQ_ERR_ARG;
  if (desc->naea != desc->naeb) return AFQ_ERR_UNSUPPORTED;   // initialize_serial.hpp:67-71
  if (desc->naea > 64 || desc->naea > desc->nmo) return AFQ_ERR_UNSUPPORTED;
  if (desc->precision != AFQ_PREC_FP64 && desc->precision != AFQ_PREC_MIXED)
    return AFQ_ERR_ARG;
  afq_handle* h = new afq_handle();
  h->d = *desc;
  h->N = desc->nmo; h->n = desc->naea; h->nc = desc->nchol; h->nw = desc->nwalk;
  h->NAK = 2LL * h->n * h->N;
  cudaError_t e = cudaSetDevice(desc->device);
  if (e != cudaSuccess) { delete h; return AFQ_ERR_CUDA; }
  e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete h; return AFQ_ERR_CUDA; }
  const size_t N = h->N, n = h->n, nw = h->nw, nc = h->nc;
  afq_status s = AFQ_OK;
  auto A = [&](cudaError_t r) { if (r != cudaSuccess && s == AFQ_OK) s = (r == cudaErrorMemoryAllocation) ? AFQ_ERR_OOM : AFQ_ERR_CUDA; };
  A(dalloc(h, &h->W, nw * N * 2 * n));
  A(dalloc(h, &h->Wd, nw * 8));
  A(dalloc(h, &h->tw, N * 2 * n));
  A(dalloc(h, &h->P, N * N));
  A(dalloc(h, &h->haj, 2 * n * N));
  A(dalloc(h, &h->Gc, nw * 2 * n * N));
  A(dalloc(h, &h->vbias, nc * nw));
  A(dalloc(h, &h->X, nc * nw));
  A(dalloc(h, &h->xraw, nc * nw));
  A(dalloc(h, &h->hybridW, nw));
  A(dalloc(h, &h->vHS, nw * N * N));
  A(dalloc(h, &h->S, nw * N * 2 * n));
  A(dalloc(h, &h->T1, nw * N * 2 * n));
  A(dalloc(h, &h->T2, nw * N * 2 * n));
  A(dalloc(h, &h->info, nw * 2));
  A(dalloc(h, &h->sc, 1));
  A(dalloc(h, &h->cvec, nc * nw));
  A(dalloc(h, &h->parts, nw * 3));
  if (s == AFQ_OK) {
    int nb = 0;
    afq::launch_exchange(nullptr, nullptr, h->N, h->n, h->nc, h->nw, nullptr, &nb, h->st);
    h->nblk = nb;
    A(dalloc(h, &h->Kpart, nw * 2 * (size_t)nb));
    A(cudaMallocHost(&h->h_sc, sizeof(DevScalars)));
  }
  if (s == AFQ_OK) {
    A(cudaMemsetAsync(h->sc, 0, sizeof(DevScalars), h->st));
    A(cudaMemsetAsync(h->Wd, 0, sizeof(z_t) * nw * 8, h->st));
    A(cudaMemsetAsync(h->parts, 0, sizeof(double) * nw * 3, h->st));
    A(cudaStreamSynchronize(h->st));
  }
  if (s != AFQ_OK) {
    afq_destroy(h);
    return s;
  }
  *out = h;
  return AFQ_OK;
}

void afq_destroy(afq_handle* h) {
  if (!h) return;
  drop_graphs(h);
  for (auto& r : h->recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  if (h->mixed) afq::mixed_destroy(h->mixed);
  if (h->cv) afq::cv_destroy(h->cv);
  if (h->st) cudaStreamSynchronize(h->st);
  for (void* p : h->allocs)
    if (p) cudaFree(p);
  if (h->h_sc) cudaFreeHost(h->h_sc);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

afq_status afq_set_hamiltonian(afq_handle* h, const afq_csr_z* Spvn, const afq_csr_z* SpvnT,
                               const double* Propg1, const double* haj, const double* trial,
                               const afq_csr_z* Vakbl, const double* Lhalf) {
  if (!h) return AFQ_ERR_ARG;
  if (h->have_ham) return fail(h, AFQ_ERR_STATE, "Hamiltonian already set");
  if (!Propg1 || !haj || !trial) return fail(h, AFQ_ERR_ARG, "null dense operand");
  if (!Vakbl && !Lhalf) return fail(h, AFQ_ERR_ARG, "need Vakbl or Lhalf for the energy");
  const int N = h->N, n = h->n, nc = h->nc;
  const int NAK = (int)h->NAK;
  afq_status s;
  if ((s = check_csr(h, Spvn, N * N, nc, "Spvn")) != AFQ_OK) return s;
  if ((s = check_csr(h, SpvnT, nc, NAK, "SpvnT")) != AFQ_OK) return s;
  if (Vakbl && (s = check_csr(h, Vakbl, NAK, NAK, "Vakbl")) != AFQ_OK) return s;
  cudaSetDevice(h->d.device);
  const bool mixed_form = h->d.precision == AFQ_PREC_MIXED;
  // Spvn: keep real values only when every imaginary part is zero
  {
    long long nnz = Spvn->rowIndex[N * N];
    bool real = true;
    for (long long p = 0; p < nnz && real; p++) real = Spvn->vals[2 * p + 1] == 0.0;
    AFQ_CUDA(h, dalloc(h, &h->sp_ri, (size_t)N * N + 1));
    AFQ_CUDA(h, dalloc(h, &h->sp_ci, nnz));
    AFQ_CUDA(h, cudaMemcpy(h->sp_ri, Spvn->rowIndex, sizeof(int) * ((size_t)N * N + 1),
                           cudaMemcpyHostToDevice));
    AFQ_CUDA(h, cudaMemcpy(h->sp_ci, Spvn->cols, sizeof(int) * nnz, cudaMemcpyHostToDevice));
    if (real) {
      std::vector<double> rv(nnz);
      for (long long p = 0; p < nnz; p++) rv[p] = Spvn->vals[2 * p];
      AFQ_CUDA(h, dalloc(h, &h->sp_rv, nnz));
      AFQ_CUDA(h, cudaMemcpy(h->sp_rv, rv.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice));
    } else {
      AFQ_CUDA(h, dalloc(h, &h->sp_v, nnz));
      AFQ_CUDA(h, cudaMemcpy(h->sp_v, Spvn->vals, sizeof(z_t) * nnz, cudaMemcpyHostToDevice));
    }
    if (!mixed_form) {   // the dense-tile candidate of the vHS product
      AFQ_CUDA(h, cudaDeviceSynchronize());
      h->sp_path[afq_handle::SP_SPVN] = 0;
      h->sp_density[afq_handle::SP_SPVN] = (double)nnz / ((double)N * N * nc);
      if (h->sp_rv) {   // real values: a dense operand of doubles (half the bytes)
        size_t free_b = 0, total_b = 0;
        const size_t cnt = (size_t)N * N * nc;
        AFQ_CUDA(h, cudaMemGetInfo(&free_b, &total_b));
        if (h->sp_density[afq_handle::SP_SPVN] >= kDenseCandidate &&
            sizeof(double) * cnt <= free_b / 10 * 3) {
          AFQ_CUDA(h, dalloc(h, &h->sp_dense_r, cnt));
          AFQ_CUDA(h, cudaMemsetAsync(h->sp_dense_r, 0, sizeof(double) * cnt, h->st));
          csr_to_dense_real_kernel<<<(N * N + 7) / 8, dim3(32, 8), 0, h->st>>>(
              h->sp_ri, h->sp_ci, h->sp_rv, N * N, nc, h->sp_dense_r);
          AFQ_CUDA(h, cudaGetLastError());
          AFQ_CUDA(h, cudaStreamSynchronize(h->st));
        }
      } else if ((s = densify(h, h->sp_ri, h->sp_ci, h->sp_v, h->sp_rv, N * N, nc,
                              h->sp_density[afq_handle::SP_SPVN], &h->sp_dense)) != AFQ_OK) {
        return s;
      }
    }
  }
  if ((s = upload_csr(h, SpvnT, &h->spT_ri, &h->spT_ci, &h->spT_v, &h->spT_dense, true,
                      !mixed_form, &h->sp_density[afq_handle::SP_SPVNT])) != AFQ_OK)
    return s;
  if (!mixed_form) h->sp_path[afq_handle::SP_SPVNT] = 0;
  if (Vakbl) {
    if ((s = upload_csr(h, Vakbl, &h->vk_ri, &h->vk_ci, &h->vk_v, &h->vk_dense, true,
                        !mixed_form, &h->sp_density[afq_handle::SP_VAKBL])) != AFQ_OK)
      return s;
    if (!mixed_form) h->sp_path[afq_handle::SP_VAKBL] = 0;
    AFQ_CUDA(h, dalloc(h, &h->Gcloc, (size_t)NAK * h->nw));
    h->have_vakbl = true;
  }
  if (Lhalf) {
    AFQ_CUDA(h, dalloc(h, &h->Lh, (size_t)nc * NAK));
    AFQ_CUDA(h, cudaMemcpy(h->Lh, Lhalf, sizeof(z_t) * (size_t)nc * NAK, cudaMemcpyHostToDevice));
  }
  AFQ_CUDA(h, cudaMemcpy(h->P, Propg1, sizeof(z_t) * (size_t)N * N, cudaMemcpyHostToDevice));
  AFQ_CUDA(h, cudaMemcpy(h->haj, haj, sizeof(z_t) * (size_t)NAK, cudaMemcpyHostToDevice));
  {  // trial [2][N][n] -> [N][2n]
    std::vector<z_t> t((size_t)N * 2 * n);
    const z_t* src = reinterpret_cast<const z_t*>(trial);
    for (int s2 = 0; s2 < 2; s2++)
      for (int i = 0; i < N; i++)
        for (int a = 0; a < n; a++) t[(size_t)i * 2 * n + s2 * n + a] = src[((size_t)s2 * N + i) * n + a];
    AFQ_CUDA(h, cudaMemcpy(h->tw, t.data(), sizeof(z_t) * t.size(), cudaMemcpyHostToDevice));
  }
  // the uploads above are pageable cudaMemcpy calls, which may return before their DMA
  // lands; the handle's stream does not wait for the legacy stream, so finish them here
  AFQ_CUDA(h, cudaDeviceSynchronize());
  if (h->d.precision == AFQ_PREC_MIXED) {
    afq::MixedInit mi{};
    mi.N = N; mi.n = n; mi.nchol = nc; mi.nw = h->nw; mi.order = h->d.taylor_order;
    mi.P = h->P; mi.Lh = h->Lh; mi.SpvnT_dense = h->spT_dense;
    mi.sp_ri = h->sp_ri; mi.sp_ci = h->sp_ci; mi.sp_v = h->sp_v; mi.sp_rv = h->sp_rv;
    mi.trial = getenv("AFQ_MIXED_DM_FP64") ? nullptr : h->tw;
    std::string msg;
    cudaError_t e = afq::mixed_create(&mi, &h->mixed, &msg, h->st);
    if (e != cudaSuccess || !h->mixed)
      return fail(h, e == cudaErrorInvalidValue ? AFQ_ERR_UNSUPPORTED : AFQ_ERR_CUDA,
                  "mixed: " + msg);
    if (h->Lh) {   // the tensor-core exchange uses its own Cholesky blocking
      int nb = afq::mixed_nblk(h->mixed);
      if (nb > h->nblk) AFQ_CUDA(h, dalloc(h, &h->Kpart, (size_t)h->nw * 2 * nb));
      h->nblk = nb;
    }
  }
  if (!h->mixed) AFQ_CUDA(h, fp64_tune(h));
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  h->have_ham = true;
  return AFQ_OK;
}

afq_status afq_set_walkers(afq_handle* h, const double* W, const double* W_data) {
  if (!h || !W || !W_data) return AFQ_ERR_ARG;
  const size_t N = h->N, n = h->n, nw = h->nw;
  std::vector<z_t> t(nw * N * 2 * n);
  const z_t* src = reinterpret_cast<const z_t*>(W);
  for (size_t w = 0; w < nw; w++)
    for (int s = 0; s < 2; s++)
      for (size_t i = 0; i < N; i++)
        for (size_t a = 0; a < n; a++)
          t[(w * N + i) * 2 * n + s * n + a] = src[((w * 2 + s) * N + i) * n + a];
  cudaSetDevice(h->d.device);
  AFQ_CUDA(h, cudaMemcpyAsync(h->W, t.data(), sizeof(z_t) * t.size(), cudaMemcpyHostToDevice, h->st));
  AFQ_CUDA(h, cudaMemcpyAsync(h->Wd, W_data, sizeof(z_t) * nw * 8, cudaMemcpyHostToDevice, h->st));
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  h->have_walkers = true;
  h->dm_cache = false;
  afq::mixed_invalidate(h->mixed);
  return AFQ_OK;
}

afq_status afq_get_walkers(afq_handle* h, double* W, double* W_data) {
  if (!h) return AFQ_ERR_ARG;
  const size_t N = h->N, n = h->n, nw = h->nw;
  cudaSetDevice(h->d.device);
  if (W) {
    std::vector<z_t> t(nw * N * 2 * n);
    AFQ_CUDA(h, cudaMemcpyAsync(t.data(), h->W, sizeof(z_t) * t.size(), cudaMemcpyDeviceToHost, h->st));
    AFQ_CUDA(h, cudaStreamSynchronize(h->st));
    z_t* dst = reinterpret_cast<z_t*>(W);
    for (size_t w = 0; w < nw; w++)
      for (int s = 0; s < 2; s++)
        for (size_t i = 0; i < N; i++)
          for (size_t a = 0; a < n; a++)
            dst[((w * 2 + s) * N + i) * n + a] = t[(w * N + i) * 2 * n + s * n + a];
  }
  if (W_data) {
    AFQ_CUDA(h, cudaMemcpyAsync(W_data, h->Wd, sizeof(z_t) * nw * 8, cudaMemcpyDeviceToHost, h->st));
    AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  }
  return AFQ_OK;
}

afq_status afq_mixed_density_matrix(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_dm(h, 1, 0));
  return AFQ_OK;
}

// The reference's transposed_Spvn == false branch (miniafqmc_base.cpp:265-273): the
// non-compact density matrix G_s = conj(A_s) T1^-1 T(W_s) (mixed_density_matrix.hpp:96-99),
// formed here as trial_s Gc_s by a batched ZGEMM after the compact one (FP64 form).
afq_status afq_mixed_density_matrix_full(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  // mixed form: the compact Gc comes from the tensor-core density matrix (stored in FP64);
  // the full G and the T(Spvn) gather below run in FP64 in both forms
  const int N = h->N, n = h->n, nw = h->nw;
  if (!h->Gf) AFQ_CUDA(h, dalloc(h, &h->Gf, (size_t)nw * 2 * N * N));
  AFQ_CUDA(h, st_dm(h, 1, 0));
  for (int sp = 0; sp < 2; sp++) {   // G_s[i][k] = sum_a trial_s[i][a] Gc_s[a][k]
    ZGemmDesc g{N, N, n, h->tw + sp * n, 2 * n, 0, h->Gc + (size_t)sp * n * N, N, h->NAK,
                zmk(1, 0)};
    EpiStore ep{h->Gf + (size_t)sp * N * N, N, 2LL * N * N, zmk(0, 0), 0};
    AFQ_CUDA(h, (zgemm_launch<true, false>(g, nw, ep, h->st)));
  }
  return AFQ_OK;
}

// base::get_vbias(Spvn, G, vbias, false) (vbias.hpp:66-81): vbias = T(Spvn) G_alpha +
// T(Spvn) G_beta.  T(Spvn) of both spins is one CSR whose row c lists the alpha entries
// (columns ik) then the beta ones (N^2 + ik), each in increasing ik: the gather sums every
// vbias element in the order the reference's two scatter passes add it.
afq_status afq_vbias_full(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (!h->Gf) return fail(h, AFQ_ERR_STATE, "full density matrix not formed");
  const long long N2 = (long long)h->N * h->N;
  if (!h->spf_ri) {   // transpose once on the host from the device copy of Spvn
    std::vector<int> ri(N2 + 1);
    AFQ_CUDA(h, cudaMemcpy(ri.data(), h->sp_ri, sizeof(int) * (N2 + 1), cudaMemcpyDeviceToHost));
    const long long nz = ri[N2];
    std::vector<int> ci(nz);
    std::vector<z_t> v(nz);
    AFQ_CUDA(h, cudaMemcpy(ci.data(), h->sp_ci, sizeof(int) * nz, cudaMemcpyDeviceToHost));
    if (h->sp_rv) {
      std::vector<double> rv(nz);
      AFQ_CUDA(h, cudaMemcpy(rv.data(), h->sp_rv, sizeof(double) * nz, cudaMemcpyDeviceToHost));
      for (long long p = 0; p < nz; p++) v[p] = zmk(rv[p], 0.0);
    } else {
      AFQ_CUDA(h, cudaMemcpy(v.data(), h->sp_v, sizeof(z_t) * nz, cudaMemcpyDeviceToHost));
    }
    const int nc = h->nc;
    std::vector<long long> cnt(nc + 1, 0);
    for (long long p = 0; p < nz; p++) cnt[ci[p] + 1] += 2;
    for (int c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
    if (cnt[nc] > 0x7fffffffLL) return fail(h, AFQ_ERR_UNSUPPORTED, "T(Spvn) exceeds int32");
    std::vector<int> tri(nc + 1), tci(cnt[nc]);
    std::vector<z_t> tv(cnt[nc]);
    std::vector<long long> half(nc), pos(nc);
    for (int c = 0; c < nc; c++) {
      tri[c] = (int)cnt[c];
      half[c] = (cnt[c + 1] - cnt[c]) / 2;
      pos[c] = 0;
    }
    tri[nc] = (int)cnt[nc];
    for (long long r = 0; r < N2; r++)   // rows in order: entries land in increasing ik
      for (int p = ri[r]; p < ri[r + 1]; p++) {
        const int c = ci[p];
        const long long q = cnt[c] + pos[c]++;
        tci[q] = (int)r;
        tv[q] = v[p];
        tci[q + half[c]] = (int)(N2 + r);
        tv[q + half[c]] = v[p];
      }
    AFQ_CUDA(h, dalloc(h, &h->spf_ri, (size_t)nc + 1));
    AFQ_CUDA(h, dalloc(h, &h->spf_ci, (size_t)cnt[nc]));
    AFQ_CUDA(h, dalloc(h, &h->spf_v, (size_t)cnt[nc]));
    // on the handle's (non-blocking) stream, so the gather below is ordered after them
    AFQ_CUDA(h, cudaMemcpyAsync(h->spf_ri, tri.data(), sizeof(int) * (nc + 1),
                                cudaMemcpyHostToDevice, h->st));
    AFQ_CUDA(h, cudaMemcpyAsync(h->spf_ci, tci.data(), sizeof(int) * cnt[nc],
                                cudaMemcpyHostToDevice, h->st));
    AFQ_CUDA(h, cudaMemcpyAsync(h->spf_v, tv.data(), sizeof(z_t) * cnt[nc],
                                cudaMemcpyHostToDevice, h->st));
    AFQ_CUDA(h, cudaStreamSynchronize(h->st));   // before the host vectors go
  }
  AFQ_CUDA(h, launch_csr_gather(h->spf_ri, h->spf_ci, h->spf_v, h->Gf, 2 * N2, h->nc, h->nw,
                                h->vbias, h->st));
  return AFQ_OK;
}

afq_status afq_overlaps(afq_handle* h, int save_old) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_dm(h, 0, save_old ? 1 : 0));
  return AFQ_OK;
}

afq_status afq_vbias(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_vbias(h));
  return AFQ_OK;
}

afq_status afq_sigma(afq_handle* h, uint64_t seed, uint64_t step) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if ((s = set_scalars(h, seed, step)) != AFQ_OK) return s;
  AFQ_CUDA(h, st_sigma(h, 0));
  return AFQ_OK;
}

afq_status afq_sigma_from(afq_handle* h, const double* x) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (!x) return fail(h, AFQ_ERR_ARG, "null x");
  AFQ_CUDA(h, cudaMemcpyAsync(h->xraw, x, sizeof(double) * (size_t)h->nc * h->nw,
                              cudaMemcpyHostToDevice, h->st));
  AFQ_CUDA(h, st_sigma(h, 1));
  return AFQ_OK;
}

afq_status afq_vhs(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_vhs(h));
  return AFQ_OK;
}

afq_status afq_propagate(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_propagate(h));
  return AFQ_OK;
}

afq_status afq_update_weights(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_weights(h, 1));
  h->host_step++;
  return AFQ_OK;
}

afq_status afq_update_weights_partial(afq_handle* h, double* e4_sum) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (!e4_sum) return fail(h, AFQ_ERR_ARG, "null e4_sum");
  AFQ_CUDA(h, st_weights(h, 0));
  h->host_step++;
  AFQ_CUDA(h, cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  *e4_sum = h->h_sc->e4sum;
  return AFQ_OK;
}

afq_status afq_population_control(afq_handle* h, uint64_t seed, uint64_t step) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (h->capturing) return fail(h, AFQ_ERR_STATE, "population control inside a captured step");
  cudaSetDevice(h->d.device);
  if (!h->comb_C) {
    AFQ_CUDA(h, dalloc(h, &h->comb_C, (size_t)h->nw));
    AFQ_CUDA(h, dalloc(h, &h->comb_idx, (size_t)h->nw));
    AFQ_CUDA(h, dalloc(h, &h->comb_w, 1));
  }
  // copies go through T2 (walkers) and T1 (walker data), per-step scratch of the propagation
  double total = 0.0;
  AFQ_CUDA(h, afq::launch_comb(h->W, h->Wd, h->nw, (long long)h->N * 2 * h->n,
                               afq::comb_uniform(seed, step, h->walker_offset), h->comb_C, h->comb_idx,
                               h->comb_w, h->T2, h->T1, &total, h->st));
  if (!(total > 0.0))   // walkers untouched
    return fail(h, AFQ_ERR_STATE, "population control: no walker has positive weight");
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  h->dm_cache = false;   // the walkers changed
  afq::mixed_invalidate(h->mixed);
  return AFQ_OK;
}

afq_status afq_copy_walkers(afq_handle* dst, afq_handle* src) {
  if (!dst || !src || dst == src) return AFQ_ERR_ARG;
  if (dst->N != src->N || dst->n != src->n || dst->nw != src->nw ||
      dst->d.device != src->d.device)
    return fail(dst, AFQ_ERR_ARG, "afq_copy_walkers: handles of different shapes or devices");
  if (!src->have_walkers) return fail(dst, AFQ_ERR_STATE, "source has no walkers");
  cudaSetDevice(dst->d.device);
  // the copy is ordered after the source's work and before the destination's next work
  cudaEvent_t ev = nullptr;
  AFQ_CUDA(dst, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, src->st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(dst->st, ev, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dst->W, src->W, sizeof(z_t) * (size_t)dst->nw * dst->N * 2 * dst->n,
                        cudaMemcpyDeviceToDevice, dst->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dst->Wd, src->Wd, sizeof(z_t) * (size_t)dst->nw * 8,
                        cudaMemcpyDeviceToDevice, dst->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(dst->st);
  cudaEventDestroy(ev);
  AFQ_CUDA(dst, e);
  dst->have_walkers = true;
  dst->dm_cache = false;
  afq::mixed_invalidate(dst->mixed);
  return AFQ_OK;
}

afq_status afq_get_eshift(afq_handle* h, double* eshift) {
  if (!h || !eshift) return AFQ_ERR_ARG;
  AFQ_CUDA(h, cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  *eshift = h->h_sc->eshift;
  return AFQ_OK;
}

afq_status afq_set_eshift(afq_handle* h, double eshift) {
  if (!h) return AFQ_ERR_ARG;
  uint64_t seed = h->host_seed == ~0ull ? 0 : h->host_seed;
  uint64_t step = h->host_step == ~0ull ? 0 : h->host_step;
  AFQ_CUDA(h, afq::launch_set_scalars(h->sc, seed, step, 1, eshift, h->st));
  h->host_seed = seed;
  h->host_step = step;
  return AFQ_OK;
}

afq_status afq_set_walker_offset(afq_handle* h, int offset, int nwalk_global) {
  if (!h || offset < 0 || nwalk_global < offset + h->nw) return AFQ_ERR_ARG;
  uint64_t seed = h->host_seed == ~0ull ? 0 : h->host_seed;
  uint64_t step = h->host_step == ~0ull ? 0 : h->host_step;
  AFQ_CUDA(h, afq::launch_set_scalars(h->sc, seed, step, 0, 0.0, h->st, offset, nwalk_global));
  h->host_seed = seed;
  h->host_step = step;
  h->walker_offset = offset;
  return AFQ_OK;
}

afq_status afq_orthogonalize(afq_handle* h) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  AFQ_CUDA(h, st_ortho(h));
  return AFQ_OK;
}

// Control-variate measurement: exact E_1 and E_J for every walker, surrogate + exact
// exchange on a subset (cv_energy.cu).
afq_status energy_cv(afq_handle* h, double* sums) {
  if (!h->Lh) return fail(h, AFQ_ERR_STATE, "no Lhalf loaded");
  if (!h->cv) {
    cudaError_t e = afq::cv_create(h->cv_cfg, h->nw, h->nc, h->NAK, &h->cv, h->st);
    if (e != cudaSuccess) return fail(h, AFQ_ERR_CUDA, "control variate set-up failed");
  }
  afq::CvInputs in;
  in.Gc = h->Gc;
  in.haj = h->haj;
  in.cvec = h->cvec;
  in.Wd = h->Wd;
  in.Kpart = h->Kpart;
  in.nblk = h->nblk;
  in.Lh = h->Lh;
  in.n = h->n;
  in.N = h->N;
  in.exact_exchange = [h](const z_t* gsub, int m, z_t* kp) -> cudaError_t {
    if (h->mixed) return afq::mixed_exchange(h->mixed, gsub, m, kp, h->nblk, h->st);
    int nb = 0;
    return afq::launch_exchange(h->Lh, gsub, h->N, h->n, h->nc, m, kp, &nb, h->st);
  };
  if (h->mixed && h->cv_cfg.base)
    in.base_exchange = [h](const z_t* g, int m, z_t* kp) -> cudaError_t {
      return afq::mixed_exchange_lowp(h->mixed, g, m, kp, h->nblk, h->st);
    };
  cudaError_t e = staged(h, AFQ_STAGE_ENERGY, 0, [&]() -> cudaError_t {
    cudaError_t r;
    if (h->mixed) {
      r = afq::mixed_coulomb(h->mixed, h->Gc, h->cvec, h->st);
    } else {
      const int nak = (int)h->NAK;
      ZGemmDesc g{h->nc, h->nw, nak, h->Lh, h->NAK, 0, h->Gc, h->NAK, 0, zmk(1, 0)};
      EpiStore ep{h->cvec, h->nw, 0, zmk(0, 0), 0};
      r = zgemm_launch<true, true>(g, 1, ep, h->st);
    }
    if (r != cudaSuccess) return r;
    return afq::cv_energy(h->cv, in, sums, h->st);
  });
  if (e != cudaSuccess) return fail(h, AFQ_ERR_CUDA, std::string("cv energy: ") + cudaGetErrorString(e));
  // coulomb and exact exchange (2-3 launches each) plus the estimator's own kernels
  h->stage_launches[AFQ_STAGE_ENERGY] += 5 + afq::cv_launches(h->cv);
  return AFQ_OK;
}

// The E1 term of the energy is a sum of G over all orbitals: its relative error is that
// of G (a few 1e-6 of E1 with the tensor-core G at 48+48 electrons), so the mixed form
// measures on an FP64 G; the two-body terms keep the tensor-core contractions.
// AFQ_MIXED_ENERGY_G=mixed keeps the tensor-core G.
cudaError_t energy_density_matrix(afq_handle* h) {
  static const bool keep = getenv("AFQ_MIXED_ENERGY_G") &&
                           std::string(getenv("AFQ_MIXED_ENERGY_G")) == "mixed";
  if (!h->mixed || keep) return cudaSuccess;
  cudaError_t e = cudaSuccess;
  if (!h->Wd_scr && (e = cudaMalloc(&h->Wd_scr, sizeof(z_t) * (size_t)h->nw * 8)) == cudaSuccess)
    h->allocs.push_back(h->Wd_scr);
  if (e == cudaSuccess && !h->info_scr &&
      (e = cudaMalloc(&h->info_scr, sizeof(int) * 2 * (size_t)h->nw)) == cudaSuccess)
    h->allocs.push_back(h->info_scr);
  if (e != cudaSuccess) return e;
  return staged(h, AFQ_STAGE_ENERGY, 1, [&] {
    return afq::launch_dm(h->W, h->tw, h->N, h->n, h->nw, h->Gc, h->Wd_scr, h->info_scr, 1, 0,
                          h->st);
  });
}

afq_status afq_energy_sums(afq_handle* h, int mode, double* sums) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (!sums) return fail(h, AFQ_ERR_ARG, "null sums");
  if (mode != AFQ_ENERGY_VAKBL) AFQ_CUDA(h, energy_density_matrix(h));
  if (mode == AFQ_ENERGY_CV) return energy_cv(h, sums);
  if (mode == AFQ_ENERGY_VAKBL && !h->have_vakbl) return fail(h, AFQ_ERR_STATE, "no Vakbl loaded");
  if (mode == AFQ_ENERGY_CHOLESKY && !h->Lh) return fail(h, AFQ_ERR_STATE, "no Lhalf loaded");
  if (mode != AFQ_ENERGY_VAKBL && mode != AFQ_ENERGY_CHOLESKY) return fail(h, AFQ_ERR_ARG, "mode");
  AFQ_CUDA(h, st_energy(h, mode));
  AFQ_CUDA(h, cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  sums[0] = h->h_sc->esum[0];
  sums[1] = h->h_sc->esum[1];
  return AFQ_OK;
}

afq_status afq_energy(afq_handle* h, int mode, double* eav) {
  double sums[2];
  afq_status s = afq_energy_sums(h, mode, sums);
  if (s != AFQ_OK) return s;
  if (eav) *eav = sums[0] / sums[1];
  return AFQ_OK;
}

afq_status afq_substep(afq_handle* h, uint64_t seed, uint64_t step_tot, int northo) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (northo <= 0) return fail(h, AFQ_ERR_ARG, "northo must be positive");
  if (seed != h->host_seed || step_tot != h->host_step)
    if ((s = set_scalars(h, seed, step_tot)) != AFQ_OK) return s;
  const bool ortho = step_tot > 0 && step_tot % (uint64_t)northo == 0;
  // the captured substep starts with a density matrix formed from the cached T1^-1 and the
  // packed operand forms of the walkers (and leaves both valid at its end): refresh them
  // first when they are stale
  if (h->mixed) AFQ_CUDA(h, afq::mixed_ensure_packed(h->mixed, h->W, h->st));
  if (mixed_dm_on(h) && !h->dm_cache) AFQ_CUDA(h, st_dm(h, 0, 0));
  if ((s = launch_substep_graph(h, ortho ? &h->g_ortho : &h->g_plain,
                                 ortho ? h->g_ortho_launches : h->g_plain_launches, ortho, 0)) !=
      AFQ_OK)
    return s;
  h->host_step = step_tot + 1;
  return AFQ_OK;
}

afq_status afq_substep_begin(afq_handle* h, uint64_t seed, uint64_t step_tot, double** e4sum) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (!e4sum) return fail(h, AFQ_ERR_ARG, "null e4sum");
  if (seed != h->host_seed || step_tot != h->host_step)
    if ((s = set_scalars(h, seed, step_tot)) != AFQ_OK) return s;
  if (!h->e4buf) AFQ_CUDA(h, dalloc(h, &h->e4buf, 1));
  if (h->mixed) AFQ_CUDA(h, afq::mixed_ensure_packed(h->mixed, h->W, h->st));
  if (mixed_dm_on(h) && !h->dm_cache) AFQ_CUDA(h, st_dm(h, 0, 0));
  if ((s = launch_substep_graph(h, &h->g_begin, h->g_begin_launches, false, 1)) != AFQ_OK)
    return s;
  AFQ_CUDA(h, afq::launch_e4sum_out(h->sc, h->e4buf, h->st));
  *e4sum = h->e4buf;
  h->host_step = step_tot + 1;
  return AFQ_OK;
}

afq_status afq_substep_end(afq_handle* h, uint64_t step_tot, int northo) {
  afq_status s = need_ready(h);
  if (s != AFQ_OK) return s;
  if (northo <= 0) return fail(h, AFQ_ERR_ARG, "northo must be positive");
  if (!h->e4buf || h->host_step != step_tot + 1)
    return fail(h, AFQ_ERR_STATE, "afq_substep_end without afq_substep_begin of that step");
  AFQ_CUDA(h, afq::launch_eshift_from(h->sc, h->e4buf, h->nw, h->st));
  h->stage_launches[AFQ_STAGE_WEIGHTS] += 1;
  if (step_tot > 0 && step_tot % (uint64_t)northo == 0)
    return launch_substep_graph(h, &h->g_orth, h->g_orth_launches, true, 2);
  return AFQ_OK;
}

}  // extern "C"

// ------------------------------------------------------------ multi-system batch
struct afq_batch {
  std::vector<afq_handle*> hs;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> pre, join;
  // recorded by the graph at the end of each system's branch (external event nodes): a
  // handle's later work waits for its own system only, not for the whole batch
  std::vector<cudaEvent_t> sysdone;
  // fused: the vHS product (bit 1) and / or the propagation chain (bit 2) of every system
  // run as one launch each over all systems' tiles (mixed-form systems of matching
  // precisions); 0 = per-system graph branches
  int fused = 0;
  // one graph per (substeps per launch, which of them re-orthogonalise)
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    std::vector<std::vector<long long>> counts;   // per handle, per stage
  };
  std::map<std::pair<int, uint64_t>, Graph> g;
};

namespace {
void batch_release(afq_batch* b) {
  for (auto& kv : b->g)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  for (cudaEvent_t e : b->pre) cudaEventDestroy(e);
  for (cudaEvent_t e : b->join) cudaEventDestroy(e);
  for (cudaEvent_t e : b->sysdone)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->done) cudaEventDestroy(b->done);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
}

void count_launches(afq_handle* h, int stage, long long k) {
  (h->launch_sink ? h->launch_sink : h->stage_launches)[stage] += k;
}

// One substep of every system of a fused batch.  Each system's stages up to sigma, and
// from the overlaps on, run on its own stream; the vHS product and the eight products of
// the propagation chain are joint launches on the batch stream (counted on the first
// system), with the systems' streams joined before and forked after them.
cudaError_t batch_substep_fused(afq_batch* b, bool ortho) {
  const int n = (int)b->hs.size();
  std::vector<afq::MixedState*> ms(n);
  std::vector<z_t*> W(n);
  for (int i = 0; i < n; i++) {
    ms[i] = b->hs[i]->mixed;
    W[i] = b->hs[i]->W;
  }
  auto join = [&]() {
    for (int i = 0; i < n; i++) {
      cudaError_t r = cudaEventRecord(b->pre[i], b->hs[i]->st);
      if (r == cudaSuccess) r = cudaStreamWaitEvent(b->st, b->pre[i], 0);
      if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
  };
  auto fork = [&]() {
    cudaError_t r = cudaEventRecord(b->fork, b->st);
    for (int i = 0; i < n && r == cudaSuccess; i++)
      r = cudaStreamWaitEvent(b->hs[i]->st, b->fork, 0);
    return r;
  };
  cudaError_t e;
  const bool jv = b->fused & 1, jp = b->fused & 2;
  for (afq_handle* h : b->hs) {
    if ((e = st_dm(h, 1, 0)) != cudaSuccess || (e = st_vbias(h)) != cudaSuccess ||
        (e = st_sigma(h, 0)) != cudaSuccess)
      return e;
    if (!jv) {
      if ((e = st_vhs(h)) != cudaSuccess) return e;
    } else if ((e = staged(h, AFQ_STAGE_VHS, 1, [&] {
                  return afq::mixed_vhs_pack(h->mixed, h->X, h->st);
                })) != cudaSuccess) {
      return e;
    }
  }
  if (jv) {
    if ((e = join()) != cudaSuccess) return e;
    count_launches(b->hs[0], AFQ_STAGE_VHS, 1);
    if ((e = afq::mixed_vhs_multi(ms.data(), n, b->st)) != cudaSuccess) return e;
    if ((e = fork()) != cudaSuccess) return e;
  }
  for (afq_handle* h : b->hs) {
    if (!jp) {
      if ((e = st_propagate(h)) != cudaSuccess) return e;
      continue;
    }
    h->dm_cache = false;
    if ((e = staged(h, AFQ_STAGE_PROPAGATE, afq::mixed_prop_pack_launches(h->mixed),
                    [&] { return afq::mixed_prop_pack(h->mixed, h->W, h->st); })) != cudaSuccess)
      return e;
  }
  if (jp) {
    if ((e = join()) != cudaSuccess) return e;
    count_launches(b->hs[0], AFQ_STAGE_PROPAGATE, b->hs[0]->d.taylor_order + 2);
    if ((e = afq::mixed_prop_multi(ms.data(), W.data(), n, b->st)) != cudaSuccess) return e;
    if ((e = fork()) != cudaSuccess) return e;
  }
  for (afq_handle* h : b->hs) {
    if ((e = st_dm(h, 0, 1)) != cudaSuccess || (e = st_weights(h, 1)) != cudaSuccess) return e;
    if (ortho && ((e = st_ortho(h)) != cudaSuccess || (e = st_dm(h, 0, 0)) != cudaSuccess))
      return e;
  }
  return cudaSuccess;
}

bool batch_fusable(const afq_batch* b) {
  std::vector<afq::MixedState*> ms;
  for (afq_handle* h : b->hs) {
    if (!h->mixed) return false;
    ms.push_back(h->mixed);
  }
  return afq::mixed_multi_compatible(ms.data(), (int)ms.size());
}
}  // namespace

extern "C" {

afq_status afq_batch_create(afq_handle* const* handles, int count, afq_batch** out) {
  if (!handles || count < 1 || !out) return AFQ_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < count; i++) {
    if (!handles[i]) return AFQ_ERR_ARG;
    if (handles[i]->d.device != handles[0]->d.device) return AFQ_ERR_UNSUPPORTED;
    for (int j = 0; j < i; j++)
      if (handles[j] == handles[i]) return AFQ_ERR_ARG;
  }
  afq_batch* b = new afq_batch();
  b->hs.assign(handles, handles + count);
  b->device = handles[0]->d.device;
  cudaSetDevice(b->device);
  bool ok = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
  b->pre.assign(count, nullptr);
  b->join.assign(count, nullptr);
  b->sysdone.assign(count, nullptr);
  for (int i = 0; ok && i < count; i++)
    ok = cudaEventCreateWithFlags(&b->pre[i], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->sysdone[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    batch_release(b);
    return AFQ_ERR_CUDA;
  }
  *out = b;
  return AFQ_OK;
}

void afq_batch_destroy(afq_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->st);
  batch_release(b);
}

afq_status afq_batch_substeps(afq_batch* b, const uint64_t* seeds, uint64_t step_tot, int nsub,
                              int northo) {
  if (!b || !seeds || northo <= 0 || nsub < 1 || nsub > 64) return AFQ_ERR_ARG;
  cudaSetDevice(b->device);
  const int n = (int)b->hs.size();
  uint64_t omask = 0;   // substeps of this launch that re-orthogonalise
  for (int k = 0; k < nsub; k++) {
    const uint64_t t = step_tot + (uint64_t)k;
    if (t > 0 && t % (uint64_t)northo == 0) omask |= 1ull << k;
  }
  // per system: scalars of this step, a fresh T1^-1 for the graph's first density matrix
  for (int i = 0; i < n; i++) {
    afq_handle* h = b->hs[i];
    afq_status s = need_ready(h);
    if (s != AFQ_OK) return s;
    if (h->profiling) return fail(h, AFQ_ERR_STATE, "stage profiling is on");
    if (seeds[i] != h->host_seed || step_tot != h->host_step)
      if ((s = set_scalars(h, seeds[i], step_tot)) != AFQ_OK) return s;
    // the fused chain starts from W itself: every capture and launch of its graph sees
    // no packed forms
    if (h->mixed && b->fused) afq::mixed_invalidate(h->mixed);
    if (h->mixed && !b->fused) AFQ_CUDA(h, afq::mixed_ensure_packed(h->mixed, h->W, h->st));
    if (mixed_dm_on(h) && !h->dm_cache) AFQ_CUDA(h, st_dm(h, 0, 0));
    AFQ_CUDA(h, cudaEventRecord(b->pre[i], h->st));
    if (cudaStreamWaitEvent(b->st, b->pre[i], 0) != cudaSuccess) return AFQ_ERR_CUDA;
  }
  afq_batch::Graph& gr = b->g[{nsub, omask}];
  if (!gr.exec) {
    // one graph: fork from the batch stream into every handle's stream, nsub substeps of
    // each system as its branch, join back
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return AFQ_ERR_CUDA;
    cudaError_t e = cudaEventRecord(b->fork, b->st);
    gr.counts.assign(n, std::vector<long long>(AFQ_NSTAGES, 0));
    if (b->fused) {
      for (int i = 0; i < n && e == cudaSuccess; i++) {
        afq_handle* h = b->hs[i];
        e = cudaStreamWaitEvent(h->st, b->fork, 0);
        h->capturing = true;
        h->launch_sink = gr.counts[i].data();
      }
      for (int k = 0; k < nsub && e == cudaSuccess; k++)
        e = batch_substep_fused(b, (omask >> k) & 1);
      for (int i = 0; i < n; i++) {
        afq_handle* h = b->hs[i];
        h->launch_sink = nullptr;
        h->capturing = false;
        if (e == cudaSuccess)
          e = cudaEventRecordWithFlags(b->sysdone[i], h->st, cudaEventRecordExternal);
        if (e == cudaSuccess) e = cudaEventRecord(b->join[i], h->st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, b->join[i], 0);
      }
    }
    for (int i = 0; i < n && e == cudaSuccess && !b->fused; i++) {
      afq_handle* h = b->hs[i];
      if ((e = cudaStreamWaitEvent(h->st, b->fork, 0)) != cudaSuccess) break;
      h->capturing = true;
      h->launch_sink = gr.counts[i].data();
      for (int k = 0; k < nsub && e == cudaSuccess; k++) e = st_substep(h, (omask >> k) & 1);
      h->launch_sink = nullptr;
      h->capturing = false;
      if (e == cudaSuccess)
        e = cudaEventRecordWithFlags(b->sysdone[i], h->st, cudaEventRecordExternal);
      if (e == cudaSuccess) e = cudaEventRecord(b->join[i], h->st);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, b->join[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->st, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gr.exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      gr.exec = nullptr;
      return fail(b->hs[0], AFQ_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
    }
  }
  if (cudaGraphLaunch(gr.exec, b->st) != cudaSuccess || cudaEventRecord(b->done, b->st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  for (int i = 0; i < n; i++) {   // later work on a handle's own stream follows the step
    afq_handle* h = b->hs[i];
    AFQ_CUDA(h, cudaStreamWaitEvent(h->st, b->sysdone[i], 0));
    for (int k = 0; k < AFQ_NSTAGES; k++) h->stage_launches[k] += gr.counts[i][k];
    h->host_step = step_tot + (uint64_t)nsub;
  }
  return AFQ_OK;
}

afq_status afq_batch_substep(afq_batch* b, const uint64_t* seeds, uint64_t step_tot,
                             int northo) {
  return afq_batch_substeps(b, seeds, step_tot, 1, northo);
}

afq_status afq_batch_set_fused(afq_batch* b, int fused) {
  if (!b || fused < 0 || fused > 3) return AFQ_ERR_ARG;
  if (fused && !batch_fusable(b)) return AFQ_ERR_UNSUPPORTED;
  cudaSetDevice(b->device);
  if (b->fused != fused) {   // graphs of another mode
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return AFQ_ERR_CUDA;
    for (auto& kv : b->g)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    b->g.clear();
    b->fused = fused;
  }
  return AFQ_OK;
}

afq_status afq_batch_synchronize(afq_batch* b) {
  if (!b) return AFQ_ERR_ARG;
  cudaSetDevice(b->device);
  if (cudaStreamSynchronize(b->st) != cudaSuccess) return AFQ_ERR_CUDA;
  for (afq_handle* h : b->hs) {
    afq_status s = afq_synchronize(h);
    if (s != AFQ_OK) return s;
  }
  return AFQ_OK;
}

afq_status afq_cv_configure(afq_handle* h, int hidden, double lr, uint64_t seed,
                            long long train_walker_steps, int subset_den) {
  if (!h || hidden <= 0 || hidden % 32 || hidden > 1024 || !(lr > 0.0) || subset_den < 1 ||
      train_walker_steps < 0)
    return AFQ_ERR_ARG;
  if (h->cv) {
    afq::cv_destroy(h->cv);
    h->cv = nullptr;
  }
  h->cv_cfg.hidden = hidden;
  h->cv_cfg.lr = (float)lr;
  h->cv_cfg.seed = seed;
  h->cv_cfg.train_walker_steps = train_walker_steps;
  h->cv_cfg.subset_den = subset_den;
  return AFQ_OK;
}

afq_status afq_cv_set_base(afq_handle* h, int base) {
  if (!h || base < 0 || base > 1) return AFQ_ERR_ARG;
  if (base && h->d.precision != AFQ_PREC_MIXED)
    return fail(h, AFQ_ERR_UNSUPPORTED, "low-precision base: mixed form only");
  if (h->cv) {
    afq::cv_destroy(h->cv);
    h->cv = nullptr;
  }
  h->cv_cfg.base = base;
  return AFQ_OK;
}

afq_status afq_cv_stats(afq_handle* h, double* stats) {
  if (!h || !stats) return AFQ_ERR_ARG;
  if (!h->cv) {
    for (int i = 0; i < 8; i++) stats[i] = 0.0;
    return AFQ_OK;
  }
  afq::cv_stats(h->cv, stats);
  return AFQ_OK;
}

afq_status afq_get_tuning(afq_handle* h, int* choice, double* ms) {
  if (!h || (!choice && !ms)) return AFQ_ERR_ARG;
  int c[afq::TS_N + 1] = {};
  float t[2 * afq::TS_N] = {};
  if (h->mixed) afq::mixed_tuning(h->mixed, c, t);
  for (int i = 0; i <= afq::TS_N; i++)
    if (choice) choice[i] = c[i];
  for (int i = 0; i < 2 * afq::TS_N; i++)
    if (ms) ms[i] = t[i];
  for (int i = 0; i < afq_handle::F64_N; i++) {   // FP64-form sites follow
    if (choice) choice[afq::TS_N + 1 + i] = h->f64cfg[i];
    if (ms) {
      ms[2 * afq::TS_N + 2 * i] = h->f64ms[i][0];
      ms[2 * afq::TS_N + 2 * i + 1] = h->f64ms[i][1];
    }
  }
  return AFQ_OK;
}

afq_status afq_get_schedule(afq_handle* h, int* sched, double* ms) {
  if (!h || !sched) return AFQ_ERR_ARG;
  float t[16] = {};
  sched[0] = h->mixed ? afq::mixed_prop_group(h->mixed, t) : 0;
  sched[1] = h->mixed ? afq::mixed_vhs_epilogue(h->mixed, t + 6) : 0;
  sched[2] = h->mixed ? afq::mixed_prop_chain(h->mixed, t + 10) : 0;
  if (ms)
    for (int i = 0; i < 16; i++) ms[i] = t[i];
  return AFQ_OK;
}

afq_status afq_get_sparse_paths(afq_handle* h, int* path, double* ms) {
  if (!h || (!path && !ms)) return AFQ_ERR_ARG;
  for (int i = 0; i < afq_handle::SP_N; i++) {
    if (path) path[i] = h->sp_path[i];
    if (ms) {
      ms[2 * i] = h->sp_ms[i][0];
      ms[2 * i + 1] = h->sp_ms[i][1];
    }
  }
  return AFQ_OK;
}

afq_status afq_profile(afq_handle* h, int enable) {
  if (!h) return AFQ_ERR_ARG;
  h->profiling = enable != 0;
  return AFQ_OK;
}

afq_status afq_stage_times(afq_handle* h, double* ms, long long* launches, int reset) {
  if (!h) return AFQ_ERR_ARG;
  AFQ_CUDA(h, collect_stage_times(h));
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  for (int i = 0; i < AFQ_NSTAGES; i++) {
    if (ms) ms[i] = h->stage_ms[i];
    if (launches) launches[i] = h->stage_launches[i];
    if (reset) {
      h->stage_ms[i] = 0.0;
      h->stage_launches[i] = 0;
    }
  }
  return AFQ_OK;
}

afq_status afq_get_stream(afq_handle* h, void** stream) {
  if (!h || !stream) return AFQ_ERR_ARG;
  *stream = (void*)h->st;
  return AFQ_OK;
}

afq_status afq_synchronize(afq_handle* h) {
  if (!h) return AFQ_ERR_ARG;
  AFQ_CUDA(h, cudaStreamSynchronize(h->st));
  if (h->cv) AFQ_CUDA(h, afq::cv_sync(h->cv));   // the estimator's online training
  if (h->mixed) {
    int flags = 0;
    AFQ_CUDA(h, afq::mixed_error(h->mixed, &flags));
    if (flags) return fail(h, AFQ_ERR_CUDA, "tensor-core pipeline wait timed out (flags " +
                                                std::to_string(flags) + ")");
  }
  return AFQ_OK;
}

afq_status afq_copy_out(afq_handle* h, int which, void* host) {
  if (!h || !host) return AFQ_ERR_ARG;
  const size_t N = h->N, nw = h->nw, nc = h->nc, NAK = h->NAK;
  cudaSetDevice(h->d.device);
  auto d2h = [&](void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    return e;
  };
  switch (which) {
    case AFQ_BUF_GC: {
      std::vector<z_t> t(nw * NAK);
      AFQ_CUDA(h, d2h(t.data(), h->Gc, sizeof(z_t) * t.size()));
      z_t* dst = static_cast<z_t*>(host);
      for (size_t w = 0; w < nw; w++)
        for (size_t i = 0; i < NAK; i++) dst[i * nw + w] = t[w * NAK + i];
      break;
    }
    case AFQ_BUF_VHS: {
      if (h->mixed) AFQ_CUDA(h, afq::mixed_unpack_vhs(h->mixed, h->vHS, h->st));
      std::vector<z_t> t(nw * N * N);
      AFQ_CUDA(h, d2h(t.data(), h->vHS, sizeof(z_t) * t.size()));
      z_t* dst = static_cast<z_t*>(host);
      for (size_t w = 0; w < nw; w++)
        for (size_t i = 0; i < N * N; i++) dst[i * nw + w] = t[w * N * N + i];
      break;
    }
    case AFQ_BUF_VBIAS: AFQ_CUDA(h, d2h(host, h->vbias, sizeof(z_t) * nc * nw)); break;
    case AFQ_BUF_X: AFQ_CUDA(h, d2h(host, h->X, sizeof(z_t) * nc * nw)); break;
    case AFQ_BUF_HYBRIDW: AFQ_CUDA(h, d2h(host, h->hybridW, sizeof(z_t) * nw)); break;
    case AFQ_BUF_XRAW: AFQ_CUDA(h, d2h(host, h->xraw, sizeof(double) * nc * nw)); break;
    case AFQ_BUF_INFO: AFQ_CUDA(h, d2h(host, h->info, sizeof(int) * nw * 2)); break;
    case AFQ_BUF_ENERGY_PARTS: AFQ_CUDA(h, d2h(host, h->parts, sizeof(double) * nw * 3)); break;
    case AFQ_BUF_G_FULL: {
      if (!h->Gf) return fail(h, AFQ_ERR_STATE, "full density matrix not formed");
      std::vector<z_t> t(nw * 2 * N * N);
      AFQ_CUDA(h, d2h(t.data(), h->Gf, sizeof(z_t) * t.size()));
      z_t* dst = static_cast<z_t*>(host);
      for (size_t w = 0; w < nw; w++)
        for (size_t i = 0; i < 2 * N * N; i++) dst[i * nw + w] = t[w * 2 * N * N + i];
      break;
    }
    case AFQ_BUF_CV_PRED:
      if (!h->cv) {
        for (size_t w = 0; w < nw; w++) static_cast<double*>(host)[w] = 0.0;
        break;
      }
      AFQ_CUDA(h, afq::cv_predictions(h->cv, static_cast<double*>(host), h->st));
      break;
    default: return fail(h, AFQ_ERR_ARG, "unknown buffer");
  }
  return AFQ_OK;
}

}  // extern "C"
