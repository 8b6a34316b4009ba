// Control-variate energy estimator with the learned exchange surrogate.
//
// Per measurement (after the mixed density matrix):
//   features of every walker from quantities the step already has: a fixed Gaussian
//     projection (32 rows) of the Coulomb vector c_w = Lh Gc_w, E_J = 1/2 c_w.c_w,
//     E_1 = Gc_w.haj, log|ovlp_a ovlp_b| and its phase, and the linearised exchange
//     Q.Gc_w (Re, Im), Q = dE_K/dG at the first measurement's mean G -- or, with the
//     low-precision base (cfg.base), in place of the linearisation the exchange of every
//     walker from one plain bf16 tensor-core product, the network then learning the exact
//     E_K minus that base (a two-level control variate: cheap exchange + learned residual);
//   surrogate f_w = MLP(features) on every walker;
//   exact exchange E_K on a seeded subset S drawn with m = ceil(nw / subset_den) teeth
//     (all walkers until the first train_walker_steps exact samples are in): by default a
//     systematic sample with probability proportional to the walker weight over the
//     walkers ordered by f, so walker w gets m w_w / T teeth on average (T = sum of the
//     weights), and
//       sum_w w_w eloc_w = sum_w w_w (E1 + EJ)_w - [sum_w w_w f_w + (T/m) sum_teeth (EK - f)]
//     (AFQ_CV_SAMPLING=0: a simple random sample of m walkers and the correction
//     (nw/m) sum_{w in S} w_w (EK_w - f_w));  either way unbiased for the exact weighted
//     energy whatever the network predicts (Horvitz-Thompson);
//   W_data[:,0] holds exact energies on S and E1 + EJ - f elsewhere;
//   the exact (features, E_K) pairs of S enter a replay buffer of raw values and the
//     network takes a few Adam steps on it -- after the estimate, so the estimate never
//     sees its own data.
//
// Scales.  Walkers start identical and spread out as the run goes on, so feature and
// target scales come from the whole replay buffer, not one measurement: the network works
// on standardised inputs (x - mu) / sd clipped to +-8 and standardised targets clipped to
// +-16.  When the buffer's statistics drift (a scale off by 1.5x or a mean shifted by half
// a scale) the network is rescaled so it computes the same function of the new
// coordinates (mlp_restandardize) and training continues.  A non-finite training loss
// switches the estimator off for good: exact exchange on every walker, the fallback.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "afq_cv.h"
#include "zgemm_fp64.cuh"

namespace afq {

constexpr int CV_NIN = 38, CV_NPROJ = 32;
constexpr float CV_CLIP_X = 8.0f, CV_CLIP_T = 16.0f;

struct CvState {
  CvConfig cfg;
  int nw = 0, nc = 0;
  long long nak = 0;
  Mlp* mlp = nullptr;
  float *R = nullptr, *feats = nullptr, *featn = nullptr, *fpred = nullptr;
  float *d_mu = nullptr, *d_sd = nullptr, *d_a = nullptr, *d_c = nullptr, *d_stat = nullptr;
  float *raw_x = nullptr, *raw_t = nullptr, *buf_x = nullptr, *buf_t = nullptr;
  double *e1ej = nullptr, *ek_sub = nullptr, *d_sums = nullptr, *h_sums = nullptr;
  int *d_sub = nullptr, *member = nullptr, *h_sub = nullptr;
  // weight-proportional design: per member, its number of teeth and teeth * T / m
  int *d_cnt = nullptr, *h_cnt = nullptr;
  double *d_mult = nullptr, *h_mult = nullptr, *d_wt = nullptr, *h_wt = nullptr;
  float* h_f = nullptr;
  z_t* Gc_sub = nullptr;
  int sub_cap = 0, cap = 0, buf_n = 0, buf_head = 0;
  // standardisation: features (mu, sd); targets E_K = ref + mu_r + sd_r * y
  float mu[CV_NIN] = {}, sd[CV_NIN] = {};
  double ref = 0.0, mu_r = 0.0, sd_r = 1.0;
  bool have_ref = false, trained = false, active = false, failed = false;
  long long seen = 0, meas = 0, restd = 0, launches = 0;
  int last_m = 0;
  float last_loss = 0.0f;
  double ht_var = 0.0;
  z_t* Q = nullptr;      // [2][n][N] linearised exchange dE_K/dG at the mean G Gm
  bool have_q = false;
  long long q_meas = 0;  // measurement of the last Q
  // Q set-up scratch: Gm [2][n][N], Tq [2][nc][n][n], Qpart [nc][n][N]; qoff = Q.Gm / 2
  z_t *Gm = nullptr, *Tq = nullptr, *Qpart = nullptr, *d_qoff = nullptr;
  double lin_ref = 0.0;  // Re of the first linearisation's E_K(Gm)
  double* ek_base = nullptr;   // [nw][2] low-precision exchange of every walker (cfg.base)
  float* fsort = nullptr;      // [nw] surrogate in the order the subset design sorts by
  // online training runs on its own stream after the estimate, overlapping the next
  // substeps; the next measurement (and any use of the network) waits for ev_trained
  cudaStream_t tst = nullptr;
  cudaEvent_t ev_ready = nullptr, ev_trained = nullptr;
  float* h_loss = nullptr;   // pinned: loss of the last training step
  bool pending = false;
  std::vector<void*> allocs;
};

namespace {

template <class T>
cudaError_t cmal(CvState* s, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * (n ? n : 1));
  if (e == cudaSuccess) {
    s->allocs.push_back(q);
    *p = static_cast<T*>(q);
  }
  return e;
}
int gridn(long long n, int t) { return (int)std::min<long long>((n + t - 1) / t, 148LL * 32); }

__global__ void cv_proj_init_kernel(float* R, long long count, int twonc,
                                    unsigned long long seed) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x) {
    double a, b;
    normal_pair(seed ^ 0x9e3779b97f4a7c15ull, 7, (unsigned long long)e, &a, &b);
    R[e] = (float)(a / sqrt((double)twonc));
  }
}

// One CTA (256 threads) per walker.
__global__ void __launch_bounds__(256)
cv_features_kernel(const z_t* __restrict__ Gc, const z_t* __restrict__ haj, long long nak,
                   const z_t* __restrict__ cvec, int nc, int nw, const z_t* __restrict__ Wd,
                   const float* __restrict__ R, const z_t* __restrict__ Q,
                   const z_t* __restrict__ qoff, double lin_ref, float* __restrict__ feats,
                   double* __restrict__ e1ej) {
  __shared__ z_t red[8];
  __shared__ float proj[CV_NPROJ];
  const int w = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  z_t e1 = zmk(0, 0), ej = zmk(0, 0), eq = zmk(0, 0);
  for (long long i = tid; i < nak; i += blockDim.x) {
    const z_t g = Gc[(long long)w * nak + i];
    zfma(e1, g, haj[i]);
    zfma(eq, g, Q[i]);
  }
  eq = block_zsum(eq, red);
  for (int c = tid; c < nc; c += blockDim.x) {
    z_t v = cvec[(long long)c * nw + w];
    zfma(ej, v, v);
  }
  e1 = block_zsum(e1, red);
  ej = block_zsum(ej, red);
  for (int q = warp; q < CV_NPROJ; q += 8) {
    const float* Rq = R + (long long)q * 2 * nc;
    float s = 0.0f;
    for (int c = lane; c < nc; c += 32) {
      z_t v = cvec[(long long)c * nw + w];
      s = fmaf(Rq[c], (float)v.x, s);
      s = fmaf(Rq[nc + c], (float)v.y, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) proj[q] = s;
  }
  __syncthreads();
  if (tid < CV_NPROJ) feats[(long long)w * CV_NIN + tid] = proj[tid];
  if (tid == 0) {
    const z_t ov = zmul(Wd[(long long)w * 8 + 2], Wd[(long long)w * 8 + 3]);
    float* f = feats + (long long)w * CV_NIN;
    f[32] = (float)(0.5 * ej.x);
    f[33] = (float)e1.x;
    f[34] = (float)log(fmax(hypot(ov.x, ov.y), 1e-300));
    f[35] = (float)atan2(ov.y, ov.x);
    // linearised exchange E_K(Gm) + Q.(G_w - Gm) = Q.G_w - Q.Gm / 2 (E_K is quadratic)
    f[36] = (float)(eq.x - qoff->x - lin_ref);
    f[37] = (float)(eq.y - qoff->y);
    double* o = e1ej + (long long)w * 4;
    o[0] = e1.x; o[1] = e1.y; o[2] = 0.5 * ej.x; o[3] = 0.5 * ej.y;
  }
}

// Weighted mean density matrix Gm[q] = sum_w Re(W_data[w][1]) Gc[w][q] / sum_w Re(...).
__global__ void cv_gmean_kernel(const z_t* __restrict__ Gc, long long nak, int nw,
                                const z_t* __restrict__ Wd, z_t* __restrict__ Gm) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nak;
       q += (long long)gridDim.x * blockDim.x) {
    z_t s = zmk(0, 0);
    double wt = 0.0;
    for (int w = 0; w < nw; w++) {
      const double om = Wd[(long long)w * 8 + 1].x;
      s = zadd(s, zscale(Gc[(long long)w * nak + q], om));
      wt += om;
    }
    Gm[q] = zscale(s, wt != 0.0 ? 1.0 / wt : 0.0);
  }
}
// Q[e] = sum over Cholesky vectors c of part[c][e] (fixed order).
__global__ void cv_qsum_kernel(const z_t* __restrict__ part, int nc, long long per,
                               z_t* __restrict__ Q) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < per;
       e += (long long)gridDim.x * blockDim.x) {
    z_t t = zmk(0, 0);
    for (int c = 0; c < nc; c++) t = zadd(t, part[(long long)c * per + e]);
    Q[e] = t;
  }
}
// qoff = Q.Gm / 2 = E_K(Gm) (one CTA, fixed order).
__global__ void __launch_bounds__(256)
cv_qoff_kernel(const z_t* __restrict__ Q, const z_t* __restrict__ Gm, long long nak,
               z_t* __restrict__ qoff) {
  __shared__ z_t red[8];
  z_t s = zmk(0, 0);
  for (long long i = threadIdx.x; i < nak; i += blockDim.x) zfma(s, Q[i], Gm[i]);
  s = block_zsum(s, red);
  if (threadIdx.x == 0) *qoff = zscale(s, 0.5);
}

// Standardised, clipped features: out = clip((f - mu) / sd, +-CV_CLIP_X).
__global__ void cv_normalize_kernel(const float* __restrict__ f, long long count,
                                    const float* __restrict__ mu, const float* __restrict__ sd,
                                    float* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e % CV_NIN);
    out[e] = fminf(fmaxf((f[e] - mu[q]) / sd[q], -CV_CLIP_X), CV_CLIP_X);
  }
}

// Training copy of the replay buffer: standardised features and targets.
__global__ void cv_normalize_buffer_kernel(const float* __restrict__ rx,
                                           const float* __restrict__ rt, int n,
                                           const float* __restrict__ mu,
                                           const float* __restrict__ sd, float mu_r, float sd_r,
                                           int residual, float* __restrict__ bx,
                                           float* __restrict__ bt) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * CV_NIN;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e % CV_NIN);
    bx[e] = fminf(fmaxf((rx[e] - mu[q]) / sd[q], -CV_CLIP_X), CV_CLIP_X);
    if (q == 0) {
      const long long b = e / CV_NIN;
      const float t = rt[b] - (residual ? rx[b * CV_NIN + 36] : 0.0f);
      bt[b] = fminf(fmaxf((t - mu_r) / sd_r, -CV_CLIP_T), CV_CLIP_T);
    }
  }
}

// Column means and standard deviations of the raw buffer (36 features, then the target):
// one CTA per column, two passes in double, fixed reduction order.
__global__ void __launch_bounds__(256)
cv_buffer_stats_kernel(const float* __restrict__ rx, const float* __restrict__ rt, int n,
                       int residual, float* __restrict__ stat) {
  __shared__ z_t red[8];
  const int q = blockIdx.x;
  auto val = [&](int b) -> double {
    if (q < CV_NIN) return (double)rx[(long long)b * CV_NIN + q];
    return (double)rt[b] - (residual ? (double)rx[(long long)b * CV_NIN + 36] : 0.0);
  };
  double s = 0.0;
  for (int b = threadIdx.x; b < n; b += blockDim.x) s += val(b);
  const double mean = block_zsum(zmk(s, 0.0), red).x / n;
  double v = 0.0;
  for (int b = threadIdx.x; b < n; b += blockDim.x) {
    const double d = val(b) - mean;
    v += d * d;
  }
  const double var = block_zsum(zmk(v, 0.0), red).x / n;
  if (threadIdx.x == 0) {
    stat[q] = (float)mean;
    stat[CV_NIN + 1 + q] = (float)sqrt(var);
  }
}

__global__ void cv_gather_kernel(const z_t* __restrict__ Gc, long long nak,
                                 const int* __restrict__ sub, int m, z_t* __restrict__ out) {
  const long long tot = (long long)m * nak;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / nak, q = e % nak;
    out[e] = Gc[(long long)sub[i] * nak + q];
  }
}

__global__ void __launch_bounds__(128)
cv_ek_kernel(const z_t* __restrict__ Kpart, int nblk, double* __restrict__ ek) {
  __shared__ z_t red[4];
  const int i = blockIdx.x;
  z_t s = zmk(0, 0);
  for (int q = threadIdx.x; q < 2 * nblk; q += blockDim.x)
    s = zadd(s, Kpart[(long long)i * 2 * nblk + q]);
  s = block_zsum(s, red);
  if (threadIdx.x == 0) {
    ek[2 * i] = 0.5 * s.x;
    ek[2 * i + 1] = 0.5 * s.y;
  }
}

// Features 36/37 from the low-precision exchange of every walker (relative to ref).
__global__ void cv_base_feature_kernel(const double* __restrict__ ek, int nw, double ref,
                                       float* __restrict__ feats) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    feats[(long long)w * CV_NIN + 36] = (float)(ek[2 * w] - ref);
    feats[(long long)w * CV_NIN + 37] = (float)ek[2 * w + 1];
  }
}

// The surrogate up to a constant: fs * network output (+ feature 36 it was trained on top
// of), the key of the weight-proportional design's ordering.
__global__ void cv_sortkey_kernel(const float* __restrict__ fpred, const float* __restrict__ fbase,
                                  float fs, int nw, float* __restrict__ out) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x)
    out[w] = fs * fpred[w] + (fbase ? fbase[(long long)w * CV_NIN] : 0.0f);
}

__global__ void cv_mark_kernel(const int* __restrict__ sub, int m, int* __restrict__ member) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    member[sub[i]] = i;
}

// Replay buffer append of raw values: features of the subset and E_K - ref.
__global__ void cv_append_kernel(const float* __restrict__ feats, const int* __restrict__ sub,
                                 int m, const double* __restrict__ ek, double ref,
                                 float* __restrict__ rx, float* __restrict__ rt, int head,
                                 int cap) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m * CV_NIN;
       e += gridDim.x * blockDim.x) {
    const int i = e / CV_NIN, q = e % CV_NIN, slot = (head + i) % cap;
    rx[(long long)slot * CV_NIN + q] = feats[(long long)sub[i] * CV_NIN + q];
    if (q == 0) rt[slot] = (float)(ek[2 * i] - ref);
  }
}

// Re W_data[w][1] of every walker (the weights the subset design draws by).
__global__ void cv_weights_kernel(const z_t* __restrict__ Wd, int nw, double* __restrict__ wt) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x)
    wt[w] = Wd[(long long)w * 8 + 1].x;
}

// Assembles W_data[:,0] and the weighted sums of the estimator (one CTA, fixed order).
// Simple random sample (mult == null): sums = [numerator, sum of weights, sum_S x,
// sum_S x^2] with x = w (E_K - f) on the subset (the terms of the Horvitz-Thompson
// correction, for its sampling variance).  Weight-proportional teeth (mult != null,
// member i drawn cnt[i] times, mult[i] = cnt[i] T / m): the correction is
// sum_S mult (E_K - f), and sums[2..3] = sum_S cnt r, sum_S cnt r^2 with r = E_K - f.
__global__ void __launch_bounds__(1024)
cv_assemble_kernel(int nw, int m, int active, const int* __restrict__ member,
                   const double* __restrict__ e1ej, const double* __restrict__ ek,
                   const float* __restrict__ fpred, double f0, double fs,
                   const float* __restrict__ fbase, const int* __restrict__ cnt,
                   const double* __restrict__ mult, z_t* __restrict__ Wd,
                   double* __restrict__ sums) {
  __shared__ z_t red[32];
  double A = 0.0, Bc = 0.0, Wt = 0.0, B2 = 0.0, Wt2 = 0.0;
  for (int w = threadIdx.x; w < nw; w += blockDim.x) {
    const double* p = e1ej + (long long)w * 4;
    const int i = member[w];
    // surrogate E_K: network output (plus the linearisation it was trained on top of)
    const double f = active ? f0 + fs * (double)fpred[w] +
                                  (fbase ? (double)fbase[(long long)w * CV_NIN] : 0.0)
                            : 0.0;
    z_t e;
    if (i >= 0) e = zmk(p[0] + p[2] - ek[2 * i], p[1] + p[3] - ek[2 * i + 1]);
    else e = zmk(p[0] + p[2] - f, p[1] + p[3]);
    Wd[(long long)w * 8] = e;
    const double om = Wd[(long long)w * 8 + 1].x;
    if (active) {
      A += om * (p[0] + p[2] - f);
      if (i >= 0 && mult) {
        const double r = ek[2 * i] - f;
        Bc += mult[i] * r;
        Wt2 += cnt[i] * r;
        B2 += cnt[i] * r * r;
      } else if (i >= 0) {
        const double x = om * (ek[2 * i] - f);
        Bc += x;
        Wt2 += x;
        B2 += x * x;
      }
    } else {
      A += om * e.x;
    }
    Wt += om;
  }
  const z_t ab = block_zsum(zmk(A, Bc), red);
  const z_t wt = block_zsum(zmk(Wt, B2), red);
  const z_t s2 = block_zsum(zmk(Wt2, 0.0), red);
  if (threadIdx.x == 0) {
    sums[0] = !active ? ab.x : mult ? ab.x - ab.y : ab.x - ((double)nw / (double)m) * ab.y;
    sums[1] = wt.x;
    sums[2] = active ? s2.x : 0.0;
    sums[3] = active ? wt.y : 0.0;
  }
}

// Seeded simple random sample of m walkers out of nw (partial Fisher-Yates on Philox).
void sample_subset(unsigned long long seed, long long meas, int nw, int m, int* out) {
  std::vector<int> idx(nw);
  for (int i = 0; i < nw; i++) idx[i] = i;
  for (int i = 0; i < m; i++) {
    uint32_t c[4] = {(uint32_t)i, 0x53554253u, (uint32_t)meas, (uint32_t)(meas >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t r = ((uint64_t)c[0] << 32) | c[1];
    const int j = i + (int)(r % (uint64_t)(nw - i));
    std::swap(idx[i], idx[j]);
  }
  std::sort(idx.begin(), idx.begin() + m);
  for (int i = 0; i < m; i++) out[i] = idx[i];
}

// Systematic sample with probability proportional to weight: the walkers are ordered by
// their surrogate prediction f (ties by index), weights clipped at zero are summed in that
// order (total T), and m teeth at (j + u) T / m pick the walkers whose cumulative weight
// first exceeds them.  Walker w is expected to get m w / T teeth whatever u is, so
// (T / m) sum over teeth of (E_K - f) is unbiased for sum_w w (E_K - f); ordering by f
// stratifies the sample.  Writes the distinct members in increasing walker order with
// their teeth counts and weights cnt T / m; returns how many there are (0: no weight).
int sample_pps(unsigned long long seed, long long meas, int nw, int m, const float* f,
               const double* w, int* out, int* cnt, double* mult, double* total) {
  std::vector<int> order(nw);
  for (int i = 0; i < nw; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return f[a] < f[b]; });
  std::vector<double> C(nw);
  double T = 0.0;
  for (int i = 0; i < nw; i++) {
    T += std::max(w[order[i]], 0.0);
    C[i] = T;
  }
  *total = T;
  if (!(T > 0.0)) return 0;
  uint32_t c[4] = {0u, 0x50505331u, (uint32_t)meas, (uint32_t)(meas >> 32)};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double u = (double)(((uint64_t)(c[0] >> 5) << 26) | (c[1] >> 6)) * (1.0 / 9007199254740992.0);
  std::vector<int> teeth(nw, 0);
  int i = 0;
  for (int j = 0; j < m; j++) {
    const double t = ((double)j + u) * T / m;
    while (i < nw - 1 && !(C[i] > t)) i++;
    teeth[order[i]]++;
  }
  int k = 0;
  for (int v = 0; v < nw; v++)
    if (teeth[v] > 0) {
      out[k] = v;
      cnt[k] = teeth[v];
      mult[k] = teeth[v] * T / m;
      k++;
    }
  return k;
}

// Scale of a column: its standard deviation, floored so constant columns (identical
// walkers at the start of a run) do not divide by zero.
float floor_sd(float sd, float mu) { return std::max(sd, 1e-6f * (fabsf(mu) + 1.0f)); }

// New buffer statistics; (re)standardises the network when they drifted.
cudaError_t cv_restandardize(CvState* s, cudaStream_t st) {
  cudaError_t e;
  cv_buffer_stats_kernel<<<CV_NIN + 1, 256, 0, st>>>(s->raw_x, s->raw_t, s->buf_n,
                                                     s->cfg.residual, s->d_stat);
  s->launches++;
  float hs[2 * (CV_NIN + 1)];
  if ((e = cudaMemcpyAsync(hs, s->d_stat, sizeof(hs), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  float mu[CV_NIN], sd[CV_NIN];
  bool drift = false;
  for (int q = 0; q < CV_NIN; q++) {
    mu[q] = hs[q];
    sd[q] = floor_sd(hs[CV_NIN + 1 + q], mu[q]);
    if (s->trained)
      drift = drift || fabsf(logf(sd[q] / s->sd[q])) > logf(1.5f) ||
              fabsf(mu[q] - s->mu[q]) > 0.5f * s->sd[q];
  }
  const double mu_r = hs[CV_NIN];
  const double sd_r = floor_sd(hs[2 * CV_NIN + 1], (float)mu_r);
  if (s->trained)
    drift = drift || fabs(log(sd_r / s->sd_r)) > log(1.5) || fabs(mu_r - s->mu_r) > 0.5 * s->sd_r;
  if (s->trained && !drift) return cudaSuccess;
  if (s->trained) {
    float a[CV_NIN], c[CV_NIN];
    for (int q = 0; q < CV_NIN; q++) {
      a[q] = sd[q] / s->sd[q];
      c[q] = (mu[q] - s->mu[q]) / s->sd[q];
    }
    if ((e = cudaMemcpyAsync(s->d_a, a, sizeof(a), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(s->d_c, c, sizeof(c), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return e;
    const float alpha = (float)(s->sd_r / sd_r), gamma = (float)((s->mu_r - mu_r) / sd_r);
    if ((e = mlp_restandardize(s->mlp, s->d_a, s->d_c, alpha, gamma, st)) != cudaSuccess) return e;
    s->launches += 2;
    s->restd++;
    // the host arrays a, c must outlive the copies
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  }
  std::copy(mu, mu + CV_NIN, s->mu);
  std::copy(sd, sd + CV_NIN, s->sd);
  s->mu_r = mu_r;
  s->sd_r = sd_r;
  if ((e = cudaMemcpyAsync(s->d_mu, s->mu, sizeof(s->mu), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(s->d_sd, s->sd, sizeof(s->sd), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return e;
  return cudaStreamSynchronize(st);
}

// Q = dE_K/dG at the weighted-mean density matrix Gm, with batched FP64 ZGEMMs over the
// Cholesky vectors c (E_K = 1/2 sum_c tr(T_c T_c), T_c = Lh_c Gm^T per spin):
//   Tq[s][c][a][b] = sum_k Gm[s][a][k] Lh[c][s][b][k]   (= T_c[b][a])
//   Qpart[c][b][k] = sum_a T_c[b][a] Lh[c][s][a][k],  Q[s][b][k] = sum_c Qpart[c][b][k]
// and qoff = Q.Gm / 2 = E_K(Gm).  Scratch is allocated on the first call.
cudaError_t cv_refresh_q(CvState* s, const CvInputs& in, cudaStream_t st) {
  const int n = in.n, N = in.N, nc = s->nc;
  cudaError_t e = cudaSuccess;
  if (!s->Gm) {
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(cmal(s, &s->Gm, (size_t)s->nak));
    A(cmal(s, &s->Tq, (size_t)2 * nc * n * n));
    A(cmal(s, &s->Qpart, (size_t)nc * n * N));
    if (e != cudaSuccess) return e;
  }
  cv_gmean_kernel<<<gridn(s->nak, 256), 256, 0, st>>>(in.Gc, s->nak, s->nw, in.Wd, s->Gm);
  s->launches++;
  for (int sp = 0; sp < 2; sp++) {
    const long long so = (long long)sp * n * N;
    ZGemmDesc g1{n, n, N, s->Gm + so, N, 0, in.Lh + so, N, 2LL * n * N, zmk(1, 0)};
    EpiStore e1{s->Tq + (long long)sp * nc * n * n, n, (long long)n * n, zmk(0, 0), 0};
    if ((e = zgemm_launch<true, true>(g1, nc, e1, st)) != cudaSuccess) return e;
    ZGemmDesc g2{n, N, n, s->Tq + (long long)sp * nc * n * n, n, (long long)n * n, in.Lh + so, N,
                 2LL * n * N, zmk(1, 0)};
    EpiStore e2{s->Qpart, N, (long long)n * N, zmk(0, 0), 0};
    if ((e = zgemm_launch<false, false>(g2, nc, e2, st)) != cudaSuccess) return e;
    cv_qsum_kernel<<<gridn((long long)n * N, 256), 256, 0, st>>>(s->Qpart, nc, (long long)n * N,
                                                                 s->Q + so);
    s->launches += 3;
  }
  cv_qoff_kernel<<<1, 256, 0, st>>>(s->Q, s->Gm, s->nak, s->d_qoff);
  s->launches++;
  return cudaGetLastError();
}

}  // namespace

cudaError_t cv_create(const CvConfig& cfg, int nw, int nchol, long long nak, CvState** out,
                      cudaStream_t st) {
  *out = nullptr;
  if (cfg.subset_den < 1 || cfg.hidden % 32 || cfg.hidden > 1024) return cudaErrorInvalidValue;
  CvState* s = new CvState();
  s->cfg = cfg;
  if (const char* it = getenv("AFQ_CV_ITERS")) s->cfg.iters_online = std::max(1, atoi(it));
  if (const char* sm = getenv("AFQ_CV_SAMPLING")) s->cfg.sampling = atoi(sm) == 0 ? 0 : 1;
  if (const char* qr = getenv("AFQ_CV_QREFRESH")) s->cfg.q_refresh = std::max(0, atoi(qr));
  if (const char* rs = getenv("AFQ_CV_RESIDUAL")) s->cfg.residual = atoi(rs) != 0;
  if (s->cfg.base) s->cfg.residual = 1;
  s->nw = nw; s->nc = nchol; s->nak = nak;
  s->sub_cap = (nw + cfg.subset_den - 1) / cfg.subset_den;
  s->cap = std::max(4096, nw);
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  A(cmal(s, &s->R, (size_t)CV_NPROJ * 2 * nchol));
  A(cmal(s, &s->feats, (size_t)nw * CV_NIN));
  A(cmal(s, &s->featn, (size_t)nw * CV_NIN));
  A(cmal(s, &s->fpred, nw));
  A(cmal(s, &s->d_mu, CV_NIN));
  A(cmal(s, &s->d_sd, CV_NIN));
  A(cmal(s, &s->d_a, CV_NIN));
  A(cmal(s, &s->d_c, CV_NIN));
  A(cmal(s, &s->d_stat, 2 * (CV_NIN + 1)));
  A(cmal(s, &s->raw_x, (size_t)s->cap * CV_NIN));
  A(cmal(s, &s->raw_t, s->cap));
  A(cmal(s, &s->buf_x, (size_t)s->cap * CV_NIN));
  A(cmal(s, &s->buf_t, s->cap));
  A(cmal(s, &s->e1ej, (size_t)nw * 4));
  A(cmal(s, &s->ek_sub, (size_t)nw * 2));
  A(cmal(s, &s->d_sums, 4));
  A(cmal(s, &s->d_sub, nw));
  A(cmal(s, &s->member, nw));
  A(cmal(s, &s->d_cnt, nw));
  A(cmal(s, &s->d_mult, nw));
  A(cmal(s, &s->d_wt, nw));
  A(cmal(s, &s->Gc_sub, (size_t)s->sub_cap * nak));
  A(cmal(s, &s->Q, (size_t)nak));
  A(cmal(s, &s->d_qoff, 1));
  A(cmal(s, &s->ek_base, (size_t)nw * 2));
  A(cmal(s, &s->fsort, nw));
  if (e == cudaSuccess) e = cudaMemsetAsync(s->Q, 0, sizeof(z_t) * nak, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_qoff, 0, sizeof(z_t), st);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_sub, sizeof(int) * nw);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_sums, sizeof(double) * 4);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_cnt, sizeof(int) * nw);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_mult, sizeof(double) * nw);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_wt, sizeof(double) * nw);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_f, sizeof(float) * nw);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_loss, sizeof(float));
  if (e == cudaSuccess) {   // lowest priority: the step's own kernels go first
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    e = cudaStreamCreateWithPriority(&s->tst, cudaStreamNonBlocking, lo);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_trained, cudaEventDisableTiming);
  if (e == cudaSuccess) e = mlp_create(CV_NIN, cfg.hidden, s->cap, cfg.seed, &s->mlp, st);
  if (e == cudaSuccess) {
    cv_proj_init_kernel<<<gridn((long long)CV_NPROJ * 2 * nchol, 256), 256, 0, st>>>(
        s->R, (long long)CV_NPROJ * 2 * nchol, 2 * nchol, cfg.seed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cv_destroy(s);
    return e;
  }
  *out = s;
  return cudaSuccess;
}

void cv_destroy(CvState* s) {
  if (!s) return;
  if (s->tst) cudaStreamSynchronize(s->tst);
  mlp_destroy(s->mlp);
  if (s->h_loss) cudaFreeHost(s->h_loss);
  if (s->ev_ready) cudaEventDestroy(s->ev_ready);
  if (s->ev_trained) cudaEventDestroy(s->ev_trained);
  if (s->tst) cudaStreamDestroy(s->tst);
  if (s->h_sub) cudaFreeHost(s->h_sub);
  if (s->h_sums) cudaFreeHost(s->h_sums);
  if (s->h_cnt) cudaFreeHost(s->h_cnt);
  if (s->h_mult) cudaFreeHost(s->h_mult);
  if (s->h_wt) cudaFreeHost(s->h_wt);
  if (s->h_f) cudaFreeHost(s->h_f);
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

// Takes the loss of a finished online training (blocking: waits for it); a non-finite loss
// switches the estimator off.
static void cv_settle(CvState* s, bool block) {
  if (!s->pending) return;
  if (block) {
    if (cudaEventSynchronize(s->ev_trained) != cudaSuccess) return;
  } else if (cudaEventQuery(s->ev_trained) != cudaSuccess) {
    return;
  }
  s->last_loss = *s->h_loss;
  if (!std::isfinite(s->last_loss)) s->failed = true;
  s->pending = false;
}

cudaError_t cv_sync(CvState* s) {
  if (!s || !s->tst) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(s->tst);
  cv_settle(s, true);
  return e;
}

void cv_stats(CvState* s, double* o) {
  cv_settle(s, false);
  o[0] = (double)s->seen;
  o[1] = (double)s->last_m;
  o[2] = (double)s->last_loss;
  o[3] = s->active ? 1.0 : 0.0;
  o[4] = (double)s->meas;
  o[5] = s->ht_var;
  o[6] = (double)s->restd;
  o[7] = s->failed ? 1.0 : 0.0;
}

long long cv_launches(const CvState* s) { return s->launches; }

cudaError_t cv_predictions(CvState* s, double* host, cudaStream_t st) {
  std::vector<float> f(s->nw, 0.0f), x((size_t)s->nw * CV_NIN, 0.0f);
  if (s->active) {
    cudaError_t e = cudaMemcpyAsync(f.data(), s->fpred, sizeof(float) * s->nw,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(x.data(), s->feats, sizeof(float) * x.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
  }
  for (int w = 0; w < s->nw; w++)
    host[w] = s->active ? s->ref + s->mu_r + s->sd_r * (double)f[w] +
                              (s->cfg.residual ? (double)x[(size_t)w * CV_NIN + 36] : 0.0)
                        : 0.0;
  return cudaSuccess;
}

cudaError_t cv_energy(CvState* s, const CvInputs& in, double* sums, cudaStream_t st) {
  const int nw = s->nw;
  cudaError_t e;
  if (s->pending) {   // the network of the previous online training
    if ((e = cudaStreamWaitEvent(st, s->ev_trained, 0)) != cudaSuccess) return e;
    cv_settle(s, true);
  }
  s->meas++;
  s->launches = 0;
  const bool base = s->cfg.base && in.base_exchange;
  // linearised exchange about the weighted-mean G: at the first measurement, then every
  // q_refresh measurements (not with the low-precision base, which takes its features)
  if (!base && in.Lh &&
      (!s->have_q || (s->cfg.q_refresh > 0 && s->meas - s->q_meas >= s->cfg.q_refresh))) {
    if ((e = cv_refresh_q(s, in, st)) != cudaSuccess) return e;
    if (!s->have_q) {   // the reference of feature 36: E_K at the first mean G
      z_t q0;
      if ((e = cudaMemcpyAsync(&q0, s->d_qoff, sizeof(q0), cudaMemcpyDeviceToHost, st)) !=
              cudaSuccess ||
          (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
      s->lin_ref = q0.x;
    }
    s->have_q = true;
    s->q_meas = s->meas;
  }
  cv_features_kernel<<<nw, 256, 0, st>>>(in.Gc, in.haj, s->nak, in.cvec, s->nc, nw, in.Wd, s->R,
                                         s->Q, s->d_qoff, s->lin_ref, s->feats, s->e1ej);
  s->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (base) {   // low-precision exchange of every walker -> features 36/37
    if ((e = in.base_exchange(in.Gc, nw, in.Kpart)) != cudaSuccess) return e;
    cv_ek_kernel<<<nw, 128, 0, st>>>(in.Kpart, in.nblk, s->ek_base);
    s->launches += 3;
    if (!s->have_q) {   // the reference of feature 36: the first walker's first value
      double b0[2];
      if ((e = cudaMemcpyAsync(b0, s->ek_base, sizeof(b0), cudaMemcpyDeviceToHost, st)) !=
              cudaSuccess ||
          (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
      s->lin_ref = b0[0];
      s->have_q = true;
      s->q_meas = s->meas;
    }
    cv_base_feature_kernel<<<gridn(nw, 256), 256, 0, st>>>(s->ek_base, nw, s->lin_ref, s->feats);
    s->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  s->active = s->trained && !s->failed;
  const int m_design = s->active ? s->sub_cap : nw;   // sample size, or teeth
  if (s->active) {
    cv_normalize_kernel<<<gridn((long long)nw * CV_NIN, 256), 256, 0, st>>>(
        s->feats, (long long)nw * CV_NIN, s->d_mu, s->d_sd, s->featn);
    if ((e = mlp_forward(s->mlp, s->featn, nw, s->fpred, false, st)) != cudaSuccess) return e;
    s->launches += 2;
  }
  bool pps = s->active && s->cfg.sampling == 1;
  double total_w = 0.0;
  int m = m_design;   // distinct walkers evaluated exactly
  if (pps) {   // the design needs the predictions and weights on the host
    cv_weights_kernel<<<gridn(nw, 256), 256, 0, st>>>(in.Wd, nw, s->d_wt);
    cv_sortkey_kernel<<<gridn(nw, 256), 256, 0, st>>>(
        s->fpred, s->cfg.residual ? s->feats + 36 : nullptr, (float)s->sd_r, nw, s->fsort);
    s->launches += 2;
    if ((e = cudaMemcpyAsync(s->h_f, s->fsort, sizeof(float) * nw, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(s->h_wt, s->d_wt, sizeof(double) * nw, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return e;
    m = sample_pps(s->cfg.seed, s->meas, nw, m_design, s->h_f, s->h_wt, s->h_sub, s->h_cnt,
                   s->h_mult, &total_w);
    if (m == 0) pps = false;   // no positive weight: fall back to the simple random sample
  }
  if (pps) {
    if ((e = cudaMemcpyAsync(s->d_cnt, s->h_cnt, sizeof(int) * m, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(s->d_mult, s->h_mult, sizeof(double) * m, cudaMemcpyHostToDevice,
                             st)) != cudaSuccess)
      return e;
  } else if (s->active) {
    m = m_design;
    sample_subset(s->cfg.seed, s->meas, nw, m, s->h_sub);
  } else {
    for (int i = 0; i < nw; i++) s->h_sub[i] = i;
  }
  s->last_m = m;
  if ((e = cudaMemcpyAsync(s->d_sub, s->h_sub, sizeof(int) * m, cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return e;
  // exact exchange on the subset
  const z_t* gsub = in.Gc;
  if (s->active) {
    cv_gather_kernel<<<gridn((long long)m * s->nak, 256), 256, 0, st>>>(in.Gc, s->nak, s->d_sub, m,
                                                                        s->Gc_sub);
    s->launches++;
    gsub = s->Gc_sub;
  }
  if ((e = in.exact_exchange(gsub, m, in.Kpart)) != cudaSuccess) return e;
  cv_ek_kernel<<<m, 128, 0, st>>>(in.Kpart, in.nblk, s->ek_sub);
  if ((e = cudaMemsetAsync(s->member, 0xFF, sizeof(int) * nw, st)) != cudaSuccess) return e;
  cv_mark_kernel<<<gridn(m, 256), 256, 0, st>>>(s->d_sub, m, s->member);
  cv_assemble_kernel<<<1, 1024, 0, st>>>(nw, m, s->active ? 1 : 0, s->member, s->e1ej, s->ek_sub,
                                          s->fpred, s->ref + s->mu_r, s->sd_r,
                                          s->cfg.residual ? s->feats + 36 : nullptr,
                                          pps ? s->d_cnt : nullptr, pps ? s->d_mult : nullptr,
                                          in.Wd, s->d_sums);
  s->launches += 3;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(s->h_sums, s->d_sums, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                           st)) != cudaSuccess)
    return e;
  if (!s->have_ref && s->cfg.residual && s->have_q) {
    // residual learning: targets relative to the first linearisation's E_K(Gm), the same
    // reference feature 36 is relative to
    s->ref = s->lin_ref;
    s->have_ref = true;
  }
  if (!s->have_ref) {
    // offset of the stored targets: the first walker's exact exchange energy
    double ek0[2];
    if ((e = cudaMemcpyAsync(ek0, s->ek_sub, sizeof(ek0), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return e;
    s->ref = ek0[0];
    s->have_ref = true;
  }
  // replay buffer of raw (features, E_K - ref) pairs
  cv_append_kernel<<<gridn((long long)m * CV_NIN, 256), 256, 0, st>>>(
      s->feats, s->d_sub, m, s->ek_sub, s->ref, s->raw_x, s->raw_t, s->buf_head, s->cap);
  s->launches++;
  s->buf_head = (s->buf_head + m) % s->cap;
  s->buf_n = std::min(s->cap, s->buf_n + m);
  s->seen += m;
  if (!s->failed && s->seen >= s->cfg.train_walker_steps) {
    // training on the side stream, after this measurement's work on st
    const cudaStream_t ts = s->tst;
    if ((e = cudaEventRecord(s->ev_ready, st)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(ts, s->ev_ready, 0)) != cudaSuccess)
      return e;
    const bool first = !s->trained;
    if ((e = cv_restandardize(s, ts)) != cudaSuccess) return e;
    s->trained = true;
    cv_normalize_buffer_kernel<<<gridn((long long)s->buf_n * CV_NIN, 256), 256, 0, ts>>>(
        s->raw_x, s->raw_t, s->buf_n, s->d_mu, s->d_sd, (float)s->mu_r, (float)s->sd_r,
        s->cfg.residual, s->buf_x, s->buf_t);
    s->launches++;
    const int iters = first ? s->cfg.iters_warm : s->cfg.iters_online;
    const int bb = s->cfg.batch_online;
    if (first || bb <= 0 || s->buf_n <= bb) {   // full-buffer steps
      if ((e = mlp_train(s->mlp, s->buf_x, s->buf_t, s->buf_n, iters, s->cfg.lr, s->h_loss, ts,
                         false)) != cudaSuccess)
        return e;
    } else {   // online: each step on the next contiguous window of bb buffered samples
      for (int it = 0; it < iters; it++) {
        const long long off = ((s->meas * iters + it) * (long long)bb) % (s->buf_n - bb + 1);
        if ((e = mlp_train(s->mlp, s->buf_x + off * CV_NIN, s->buf_t + off, bb, 1, s->cfg.lr,
                           it == iters - 1 ? s->h_loss : nullptr, ts, false)) != cudaSuccess)
          return e;
      }
    }
    s->launches += 10LL * iters;
    if ((e = cudaEventRecord(s->ev_trained, ts)) != cudaSuccess) return e;
    s->pending = true;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  const double* hs = s->h_sums;
  sums[0] = hs[0];
  sums[1] = hs[1];
  // sampling variance of the weighted mean from the subset correction.  Simple random
  // sample (without replacement): nw^2 (1 - m/nw) S_x^2 / m / (sum w)^2.  Weight-
  // proportional teeth: the with-replacement bound (T / sum w)^2 S_r^2 / m over the m
  // teeth (systematic sampling of an ordered population does at least as well)
  s->ht_var = 0.0;
  if (pps && m_design > 1 && hs[1] != 0.0) {
    const double md = m_design;
    const double S2 = (hs[3] - hs[2] * hs[2] / md) / (md - 1);
    s->ht_var = (total_w / hs[1]) * (total_w / hs[1]) * std::max(S2, 0.0) / md;
  } else if (s->active && m > 1 && hs[1] != 0.0) {
    const double S2 = (hs[3] - hs[2] * hs[2] / m) / (m - 1);
    s->ht_var = (double)nw * nw * (1.0 - (double)m / nw) * std::max(S2, 0.0) / m / (hs[1] * hs[1]);
  }
  return cudaSuccess;
}

}  // namespace afq
