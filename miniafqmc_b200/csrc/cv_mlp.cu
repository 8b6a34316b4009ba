// Exchange-energy surrogate for the control-variate energy estimator: a 36 -> H -> H -> 1
// MLP with GELU activations, BF16 weights in the forward and backward products, FP32
// master weights, FP32 Adam.  No reference counterpart (the reference evaluates the
// exact energy for every walker, energy.hpp:66-102).
//
// Kernels (CUDA cores; the network is ~75k parameters, far below tensor-core sizes):
//   mlp_fwd    MLP_SB samples per CTA, one hidden unit per thread; keeps z1, z2 for backward
//   mlp_bwd_x  per-sample backward through the layers (dz2, dz1)
//   mlp_atb    tiled weight + bias gradients (dz^T [x|1]) over sample chunks, mlp_gsum
//              adds the chunks; fixed order
//   mlp_adam   Adam update of the FP32 master weights and refresh of the BF16 copies
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/afqmc_b200.h"
#include "afq_common.cuh"
#include "afq_cv.h"

namespace afq {

typedef __nv_bfloat16 bf16;

AFQ_D float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
AFQ_D float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * 0.39894228040143268f * expf(-0.5f * x * x);
}

struct MlpLayout {
  int nin, H;
  long long oW1, ob1, oW2, ob2, ow3, ob3, total;
  MlpLayout(int nin_, int H_) : nin(nin_), H(H_) {
    oW1 = 0;
    ob1 = oW1 + (long long)H * nin;
    oW2 = ob1 + H;
    ob2 = oW2 + (long long)H * H;
    ow3 = ob2 + H;
    ob3 = ow3 + H;
    total = ob3 + 1;
  }
};

constexpr int MLP_SB = 2;   // samples per CTA in the per-sample kernels (few: many CTAs per SM)

// y = w3 . gelu(W2 gelu(W1 x + b1) + b2) + b3 for MLP_SB samples per CTA; blockDim = H.
__global__ void mlp_fwd_kernel(const float* __restrict__ x, int B, int nin,
                               const bf16* __restrict__ W1t,   // [nin][H]
                               const float* __restrict__ b1,
                               const bf16* __restrict__ W2t,   // [H][H] transposed (k, j)
                               const float* __restrict__ b2, const bf16* __restrict__ w3,
                               const float* __restrict__ b3, float* __restrict__ z1,
                               float* __restrict__ z2, float* __restrict__ h1,
                               float* __restrict__ h2, float* __restrict__ y) {
  extern __shared__ float fs[];
  const int H = blockDim.x, j = threadIdx.x;
  float* xs = fs;                       // [SB][nin]
  float* h1s = xs + MLP_SB * nin;       // [SB][H]
  float* red = h1s + MLP_SB * H;        // [SB][H/32]
  const int b0 = blockIdx.x * MLP_SB;
  for (int e = j; e < MLP_SB * nin; e += H) {
    int bb = e / nin, i = e % nin;
    xs[e] = (b0 + bb < B) ? x[(long long)(b0 + bb) * nin + i] : 0.0f;
  }
  __syncthreads();
  float acc[MLP_SB];
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) acc[bb] = b1[j];
  for (int i = 0; i < nin; i++) {
    const float w = __bfloat162float(W1t[(long long)i * H + j]);
#pragma unroll
    for (int bb = 0; bb < MLP_SB; bb++) acc[bb] = fmaf(w, xs[bb * nin + i], acc[bb]);
  }
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) {
    const int b = b0 + bb;
    const float g = gelu(acc[bb]);
    h1s[bb * H + j] = g;
    if (b < B) {
      if (z1) z1[(long long)b * H + j] = acc[bb];
      if (h1) h1[(long long)b * H + j] = g;
    }
  }
  __syncthreads();
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) acc[bb] = b2[j];
  for (int k = 0; k < H; k++) {
    const float w = __bfloat162float(W2t[(long long)k * H + j]);
#pragma unroll
    for (int bb = 0; bb < MLP_SB; bb++) acc[bb] = fmaf(w, h1s[bb * H + k], acc[bb]);
  }
  const float w3j = __bfloat162float(w3[j]);
  const int lane = j & 31, warp = j >> 5, nwarp = H >> 5;
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) {
    const int b = b0 + bb;
    const float g = gelu(acc[bb]);
    if (b < B) {
      if (z2) z2[(long long)b * H + j] = acc[bb];
      if (h2) h2[(long long)b * H + j] = g;
    }
    float p = w3j * g;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
    if (lane == 0) red[bb * nwarp + warp] = p;
  }
  __syncthreads();
  if (j < MLP_SB && b0 + j < B) {
    float s = b3[0];
    for (int q = 0; q < nwarp; q++) s += red[j * nwarp + q];
    y[b0 + j] = s;
  }
}

// dy = (y - t) / B; dz2 = dy w3 gelu'(z2); dh1 = W2^T dz2; dz1 = dh1 gelu'(z1).
__global__ void mlp_bwd_x_kernel(const float* __restrict__ y, const float* __restrict__ t, int B,
                                 const bf16* __restrict__ W2,   // [H][H] (j, k)
                                 const bf16* __restrict__ w3, const float* __restrict__ z1,
                                 const float* __restrict__ z2, float* __restrict__ dy,
                                 float* __restrict__ dz1, float* __restrict__ dz2) {
  extern __shared__ float fs[];
  const int H = blockDim.x, j = threadIdx.x;
  float* d2s = fs;   // [SB][H]
  const int b0 = blockIdx.x * MLP_SB;
  const float w3j = __bfloat162float(w3[j]);
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) {
    const int b = b0 + bb;
    float d = 0.0f;
    if (b < B) {
      const float g = (y[b] - t[b]) / (float)B;
      if (j == 0) dy[b] = g;
      d = g * w3j * gelu_d(z2[(long long)b * H + j]);
      dz2[(long long)b * H + j] = d;
    }
    d2s[bb * H + j] = d;
  }
  __syncthreads();
  float acc[MLP_SB];
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) acc[bb] = 0.0f;
  for (int q = 0; q < H; q++) {
    const float w = __bfloat162float(W2[(long long)q * H + j]);   // W2[q][j]
#pragma unroll
    for (int bb = 0; bb < MLP_SB; bb++) acc[bb] = fmaf(w, d2s[bb * H + q], acc[bb]);
  }
#pragma unroll
  for (int bb = 0; bb < MLP_SB; bb++) {
    const int b = b0 + bb;
    if (b < B) dz1[(long long)b * H + j] = acc[bb] * gelu_d(z1[(long long)b * H + j]);
  }
}

// Weight and bias gradients of one layer, C[i][j] = sum_b A[b][i] B[b][j] for j < N and
// C[i][N] = sum_b A[b][i] (B extended by a column of ones): gW1 = dz1^T [x|1],
// gW2 = dz2^T [h1|1], [gw3|gb3] = dy^T [h2|1].  64 x 64 outputs per CTA, 4 x 4 per thread,
// 16-sample slabs in shared memory; grid z splits the samples into chunks whose partial
// sums part[z][M][N+1] are added in fixed order by mlp_gsum_kernel.
constexpr int GW_T = 64, GW_K = 16;
__global__ void __launch_bounds__(256)
mlp_atb_kernel(const float* __restrict__ A, const float* __restrict__ B, int Bn, int M, int N,
               int chunk, float* __restrict__ part) {
  __shared__ float As[GW_K][GW_T], Bs[GW_K][GW_T];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int i0 = blockIdx.y * GW_T, j0 = blockIdx.x * GW_T, N1 = N + 1;
  const int bbeg = blockIdx.z * chunk, bend = min(Bn, bbeg + chunk);
  float acc[4][4] = {};
  for (int b0 = bbeg; b0 < bend; b0 += GW_K) {
    for (int e = threadIdx.x; e < GW_K * GW_T; e += 256) {
      const int kk = e / GW_T, c = e % GW_T, b = b0 + kk, j = j0 + c;
      const bool in = b < bend;
      As[kk][c] = (in && i0 + c < M) ? A[(long long)b * M + i0 + c] : 0.0f;
      Bs[kk][c] = !in ? 0.0f : j < N ? B[(long long)b * N + j] : j == N ? 1.0f : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GW_K; kk++) {
      float a[4], bb[4];
#pragma unroll
      for (int r = 0; r < 4; r++) a[r] = As[kk][ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; c++) bb[c] = Bs[kk][tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = fmaf(a[r], bb[c], acc[r][c]);
    }
    __syncthreads();
  }
  float* P = part + (long long)blockIdx.z * M * N1;
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = i0 + ty + 16 * r, j = j0 + tx + 16 * c;
      if (i < M && j < N1) P[(long long)i * N1 + j] = acc[r][c];
    }
}

// gW[i][j] = sum_z part[z][i][j] (j < N), gb[i] = sum_z part[z][i][N]; fixed order.
__global__ void mlp_gsum_kernel(const float* __restrict__ part, int nz, int M, int N,
                                float* __restrict__ gW, float* __restrict__ gb) {
  const int N1 = N + 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M * N1; e += gridDim.x * blockDim.x) {
    float t = 0.0f;
    for (int z = 0; z < nz; z++) t += part[(long long)z * M * N1 + e];
    const int i = e / N1, j = e % N1;
    if (j < N) gW[(long long)i * N + j] = t;
    else gb[i] = t;
  }
}

// Sample chunking of one layer's gradient: enough CTAs to cover the GPU twice.
struct GradSplit {
  int nz, chunk;
  static int target(int Bn, int M, int N) {
    const int tiles = ((N + 1 + GW_T - 1) / GW_T) * ((M + GW_T - 1) / GW_T);
    return std::min(std::max(1, (Bn + GW_K - 1) / GW_K), std::max(1, (2 * 148 + tiles - 1) / tiles));
  }
  GradSplit(int Bn, int M, int N) {
    const int z = target(Bn, M, N);
    chunk = ((Bn + z - 1) / z + GW_K - 1) / GW_K * GW_K;
    nz = std::max(1, (Bn + chunk - 1) / chunk);   // <= target(cap, M, N) for Bn <= cap
  }
  static long long max_part(int cap, int M, int N) {
    return (long long)target(cap, M, N) * M * (N + 1);
  }
};

// Adam on the FP32 master weights, then BF16 copies: W1t [nin][H], W2 [H][H], W2t, w3.
__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                                float* __restrict__ m, float* __restrict__ v, float lr, float b1p,
                                float b2p, MlpLayout L, bf16* __restrict__ W1t,
                                bf16* __restrict__ W2, bf16* __restrict__ W2t,
                                bf16* __restrict__ w3) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= L.total) return;
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  const float gi = g[e];
  const float mi = beta1 * m[e] + (1.0f - beta1) * gi;
  const float vi = beta2 * v[e] + (1.0f - beta2) * gi * gi;
  m[e] = mi;
  v[e] = vi;
  const float pi = p[e] - lr * (mi / (1.0f - b1p)) / (sqrtf(vi / (1.0f - b2p)) + eps);
  p[e] = pi;
  const bf16 q = __float2bfloat16_rn(pi);
  if (e < L.ob1) {
    const int j = (int)(e / L.nin), i = (int)(e % L.nin);
    W1t[(long long)i * L.H + j] = q;
  } else if (e >= L.oW2 && e < L.ob2) {
    const long long r = e - L.oW2;
    const int j = (int)(r / L.H), k = (int)(r % L.H);
    W2[r] = q;
    W2t[(long long)k * L.H + j] = q;
  } else if (e >= L.ow3 && e < L.ob3) {
    w3[e - L.ow3] = q;
  }
}

// BF16 copies from the FP32 parameters (after set_params or initialisation).
__global__ void mlp_refresh_kernel(const float* __restrict__ p, MlpLayout L, bf16* __restrict__ W1t,
                                   bf16* __restrict__ W2, bf16* __restrict__ W2t,
                                   bf16* __restrict__ w3) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= L.total) return;
  const bf16 q = __float2bfloat16_rn(p[e]);
  if (e < L.ob1) {
    const int j = (int)(e / L.nin), i = (int)(e % L.nin);
    W1t[(long long)i * L.H + j] = q;
  } else if (e >= L.oW2 && e < L.ob2) {
    const long long r = e - L.oW2;
    W2[r] = q;
    W2t[(r % L.H) * L.H + r / L.H] = q;
  } else if (e >= L.ow3 && e < L.ob3) {
    w3[e - L.ow3] = q;
  }
}

__global__ void mlp_loss_kernel(const float* __restrict__ y, const float* __restrict__ t, int B,
                                float* __restrict__ loss) {
  __shared__ z_t red[32];
  double s = 0.0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    double d = (double)y[b] - (double)t[b];
    s += 0.5 * d * d;
  }
  z_t r = block_zsum(zmk(s, 0.0), red);
  if (threadIdx.x == 0) *loss = (float)(r.x / B);
}

struct Mlp {
  MlpLayout L;
  int cap;                    // batch capacity of the activation buffers
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16 *W1t = nullptr, *W2 = nullptr, *W2t = nullptr, *w3 = nullptr;
  float *x = nullptr, *t = nullptr, *y = nullptr, *z1 = nullptr, *z2 = nullptr, *h1 = nullptr,
        *h2 = nullptr, *dy = nullptr, *dz1 = nullptr, *dz2 = nullptr, *loss = nullptr,
        *part = nullptr;   // per-chunk gradient partial sums
  long long step = 0;
  std::vector<void*> allocs;
  Mlp(int nin, int H) : L(nin, H) {}
};

namespace {
template <class T>
cudaError_t mal(Mlp* m, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * (n ? n : 1));
  if (e == cudaSuccess) {
    m->allocs.push_back(q);
    *p = static_cast<T*>(q);
  }
  return e;
}
int nblk(long long n, int t) { return (int)((n + t - 1) / t); }
}  // namespace

cudaError_t mlp_create(int nin, int H, int cap, unsigned long long seed, Mlp** out,
                       cudaStream_t st) {
  *out = nullptr;
  if (H % 32 || H > 1024 || nin <= 0 || cap <= 0) return cudaErrorInvalidValue;
  Mlp* m = new Mlp(nin, H);
  m->cap = cap;
  const long long P = m->L.total;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  A(mal(m, &m->p, P)); A(mal(m, &m->g, P)); A(mal(m, &m->m, P)); A(mal(m, &m->v, P));
  A(mal(m, &m->W1t, (size_t)nin * H)); A(mal(m, &m->W2, (size_t)H * H));
  A(mal(m, &m->W2t, (size_t)H * H)); A(mal(m, &m->w3, H));
  A(mal(m, &m->x, (size_t)cap * nin)); A(mal(m, &m->t, cap)); A(mal(m, &m->y, cap));
  A(mal(m, &m->z1, (size_t)cap * H)); A(mal(m, &m->z2, (size_t)cap * H));
  A(mal(m, &m->h1, (size_t)cap * H)); A(mal(m, &m->h2, (size_t)cap * H));
  A(mal(m, &m->dy, cap)); A(mal(m, &m->dz1, (size_t)cap * H)); A(mal(m, &m->dz2, (size_t)cap * H));
  A(mal(m, &m->loss, 1));
  A(mal(m, &m->part, (size_t)std::max({GradSplit::max_part(cap, H, nin),
                                         GradSplit::max_part(cap, H, H),
                                         GradSplit::max_part(cap, 1, H)})));
  if (e != cudaSuccess) {
    mlp_destroy(m);
    return e;
  }
  // He-style initialisation from a seeded Philox stream (host side, deterministic)
  std::vector<float> hp(P, 0.0f);
  auto normal = [&](unsigned long long idx) {
    uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), 0x4d4c50u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    double u1 = ((double)c[0] + 1.0) / 4294967296.0, u2 = (double)c[1] / 4294967296.0;
    return (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
  };
  const MlpLayout& L = m->L;
  for (long long i = L.oW1; i < L.ob1; i++) hp[i] = normal(i) * sqrtf(2.0f / nin);
  for (long long i = L.oW2; i < L.ob2; i++) hp[i] = normal(i) * sqrtf(2.0f / H);
  for (long long i = L.ow3; i < L.ob3; i++) hp[i] = normal(i) * sqrtf(1.0f / H);
  A(cudaMemcpyAsync(m->p, hp.data(), sizeof(float) * P, cudaMemcpyHostToDevice, st));
  A(cudaMemsetAsync(m->m, 0, sizeof(float) * P, st));
  A(cudaMemsetAsync(m->v, 0, sizeof(float) * P, st));
  mlp_refresh_kernel<<<nblk(P, 256), 256, 0, st>>>(m->p, m->L, m->W1t, m->W2, m->W2t, m->w3);
  A(cudaGetLastError());
  A(cudaStreamSynchronize(st));
  if (e != cudaSuccess) {
    mlp_destroy(m);
    return e;
  }
  *out = m;
  return cudaSuccess;
}

void mlp_destroy(Mlp* m) {
  if (!m) return;
  for (void* q : m->allocs) cudaFree(q);
  delete m;
}

long long mlp_nparams(const Mlp* m) { return m->L.total; }
int mlp_capacity(const Mlp* m) { return m->cap; }
float* mlp_x(Mlp* m) { return m->x; }
float* mlp_t(Mlp* m) { return m->t; }
float* mlp_y(Mlp* m) { return m->y; }

cudaError_t mlp_set_params(Mlp* m, const float* host, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(m->p, host, sizeof(float) * m->L.total, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  mlp_refresh_kernel<<<nblk(m->L.total, 256), 256, 0, st>>>(m->p, m->L, m->W1t, m->W2, m->W2t, m->w3);
  return cudaGetLastError();
}

cudaError_t mlp_get_params(Mlp* m, float* host, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(host, m->p, sizeof(float) * m->L.total, cudaMemcpyDeviceToHost, st);
  return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

// Function-preserving change of the input and output scales: with x_old = a * x_new + c
// and y_new = alpha * y_old + gamma, W1' = W1 diag(a), b1' = b1 + W1 c, w3' = alpha w3,
// b3' = alpha b3 + gamma.  One thread per hidden unit.
__global__ void mlp_restd_kernel(float* __restrict__ p, MlpLayout L, const float* __restrict__ a,
                                 const float* __restrict__ c, float alpha, float gamma) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < L.H) {
    float* w = p + L.oW1 + (long long)j * L.nin;
    float db = 0.0f;
    for (int i = 0; i < L.nin; i++) {
      db = fmaf(w[i], c[i], db);
      w[i] *= a[i];
    }
    p[L.ob1 + j] += db;
    p[L.ow3 + j] *= alpha;
  }
  if (j == 0) p[L.ob3] = alpha * p[L.ob3] + gamma;
}

cudaError_t mlp_restandardize(Mlp* m, const float* a, const float* c, float alpha, float gamma,
                              cudaStream_t st) {
  const long long P = m->L.total;
  mlp_restd_kernel<<<nblk(m->L.H, 128), 128, 0, st>>>(m->p, m->L, a, c, alpha, gamma);
  cudaError_t e = cudaGetLastError();
  // the Adam moments belong to the old coordinates: restart them
  if (e == cudaSuccess) e = cudaMemsetAsync(m->m, 0, sizeof(float) * P, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->v, 0, sizeof(float) * P, st);
  m->step = 0;
  if (e != cudaSuccess) return e;
  mlp_refresh_kernel<<<nblk(P, 256), 256, 0, st>>>(m->p, m->L, m->W1t, m->W2, m->W2t, m->w3);
  return cudaGetLastError();
}

// Forward on device inputs x [B][nin] (normalised features) into y [B].
cudaError_t mlp_forward(Mlp* m, const float* x, int B, float* y, bool keep, cudaStream_t st) {
  if (B <= 0) return cudaSuccess;
  if (keep && B > m->cap) return cudaErrorInvalidValue;
  const int H = m->L.H, nin = m->L.nin;
  const size_t smem = sizeof(float) * (MLP_SB * nin + MLP_SB * H + MLP_SB * (H / 32));
  const MlpLayout& L = m->L;
  mlp_fwd_kernel<<<nblk(B, MLP_SB), H, smem, st>>>(
      x, B, nin, m->W1t, m->p + L.ob1, m->W2t, m->p + L.ob2, m->w3, m->p + L.ob3,
      keep ? m->z1 : nullptr, keep ? m->z2 : nullptr, keep ? m->h1 : nullptr,
      keep ? m->h2 : nullptr, y);
  return cudaGetLastError();
}

// Gradient of L = 1/(2B) sum (y - t)^2 at the current weights into m->g; x, t on device.
cudaError_t mlp_gradient(Mlp* m, const float* x, const float* t, int B, cudaStream_t st) {
  if (B <= 0 || B > m->cap) return cudaErrorInvalidValue;
  const int H = m->L.H;
  cudaError_t e = mlp_forward(m, x, B, m->y, true, st);
  if (e != cudaSuccess) return e;
  mlp_bwd_x_kernel<<<nblk(B, MLP_SB), H, sizeof(float) * MLP_SB * H, st>>>(
      m->y, t, B, m->W2, m->w3, m->z1, m->z2, m->dy, m->dz1, m->dz2);
  const MlpLayout& L = m->L;
  const int nin = L.nin;
  auto layer = [&](const float* A, const float* Bm, int M, int N, float* gW, float* gb) {
    const GradSplit gs(B, M, N);
    mlp_atb_kernel<<<dim3(nblk(N + 1, GW_T), nblk(M, GW_T), gs.nz), 256, 0, st>>>(
        A, Bm, B, M, N, gs.chunk, m->part);
    mlp_gsum_kernel<<<nblk((long long)M * (N + 1), 256), 256, 0, st>>>(m->part, gs.nz, M, N, gW, gb);
  };
  layer(m->dz1, x, H, nin, m->g + L.oW1, m->g + L.ob1);
  layer(m->dz2, m->h1, H, H, m->g + L.oW2, m->g + L.ob2);
  layer(m->dy, m->h2, 1, H, m->g + L.ow3, m->g + L.ob3);
  mlp_loss_kernel<<<1, 256, 0, st>>>(m->y, t, B, m->loss);
  return cudaGetLastError();
}

cudaError_t mlp_train(Mlp* m, const float* x, const float* t, int B, int iters, float lr,
                      float* last_loss, cudaStream_t st, bool sync_loss) {
  cudaError_t e = cudaSuccess;
  for (int it = 0; it < iters && e == cudaSuccess; it++) {
    e = mlp_gradient(m, x, t, B, st);
    if (e != cudaSuccess) break;
    m->step++;
    const float b1p = powf(0.9f, (float)m->step), b2p = powf(0.999f, (float)m->step);
    mlp_adam_kernel<<<nblk(m->L.total, 256), 256, 0, st>>>(m->p, m->g, m->m, m->v, lr, b1p, b2p,
                                                           m->L, m->W1t, m->W2, m->W2t, m->w3);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && last_loss) {
    e = cudaMemcpyAsync(last_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && sync_loss) e = cudaStreamSynchronize(st);
  }
  return e;
}

cudaError_t mlp_copy_grad(Mlp* m, float* host, float* loss, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(host, m->g, sizeof(float) * m->L.total, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && loss)
    e = cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
  return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

}  // namespace afq

// ------------------------------------------------------------------ C ABI
struct afq_mlp {
  afq::Mlp* m = nullptr;
  cudaStream_t st = nullptr;
};

extern "C" {

afq_status afq_mlp_create(int nin, int hidden, int capacity, uint64_t seed, afq_mlp** out) {
  if (!out) return AFQ_ERR_ARG;
  *out = nullptr;
  afq_mlp* h = new afq_mlp();
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return AFQ_ERR_CUDA;
  }
  cudaError_t e = afq::mlp_create(nin, hidden, capacity, seed, &h->m, h->st);
  if (e != cudaSuccess) {
    cudaStreamDestroy(h->st);
    delete h;
    return e == cudaErrorInvalidValue ? AFQ_ERR_ARG : AFQ_ERR_CUDA;
  }
  *out = h;
  return AFQ_OK;
}

void afq_mlp_destroy(afq_mlp* h) {
  if (!h) return;
  afq::mlp_destroy(h->m);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

long long afq_mlp_num_params(const afq_mlp* h) { return h ? afq::mlp_nparams(h->m) : 0; }

afq_status afq_mlp_set_params(afq_mlp* h, const float* params) {
  if (!h || !params) return AFQ_ERR_ARG;
  if (afq::mlp_set_params(h->m, params, h->st) != cudaSuccess) return AFQ_ERR_CUDA;
  return cudaStreamSynchronize(h->st) == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

afq_status afq_mlp_get_params(afq_mlp* h, float* params) {
  if (!h || !params) return AFQ_ERR_ARG;
  return afq::mlp_get_params(h->m, params, h->st) == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

static afq_status upload(afq_mlp* h, const float* x, const float* t, int B) {
  afq::Mlp* m = h->m;
  if (B <= 0 || B > afq::mlp_capacity(m)) return AFQ_ERR_ARG;
  const int nin = m->L.nin;
  if (x && cudaMemcpyAsync(afq::mlp_x(m), x, sizeof(float) * (size_t)B * nin, cudaMemcpyHostToDevice,
                           h->st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  if (t && cudaMemcpyAsync(afq::mlp_t(m), t, sizeof(float) * B, cudaMemcpyHostToDevice, h->st) !=
               cudaSuccess)
    return AFQ_ERR_CUDA;
  return AFQ_OK;
}

afq_status afq_mlp_forward(afq_mlp* h, int B, const float* x, float* y) {
  if (!h || !x || !y) return AFQ_ERR_ARG;
  afq_status s = upload(h, x, nullptr, B);
  if (s != AFQ_OK) return s;
  afq::Mlp* m = h->m;
  if (afq::mlp_forward(m, afq::mlp_x(m), B, afq::mlp_y(m), false, h->st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  if (cudaMemcpyAsync(y, afq::mlp_y(m), sizeof(float) * B, cudaMemcpyDeviceToHost, h->st) !=
      cudaSuccess)
    return AFQ_ERR_CUDA;
  return cudaStreamSynchronize(h->st) == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

afq_status afq_mlp_gradient(afq_mlp* h, int B, const float* x, const float* t, float* grad,
                            float* loss) {
  if (!h || !x || !t || !grad) return AFQ_ERR_ARG;
  afq_status s = upload(h, x, t, B);
  if (s != AFQ_OK) return s;
  afq::Mlp* m = h->m;
  if (afq::mlp_gradient(m, afq::mlp_x(m), afq::mlp_t(m), B, h->st) != cudaSuccess) return AFQ_ERR_CUDA;
  return afq::mlp_copy_grad(m, grad, loss, h->st) == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}

afq_status afq_mlp_train(afq_mlp* h, int B, const float* x, const float* t, int iters, float lr,
                         float* loss) {
  if (!h || !x || !t || iters < 0) return AFQ_ERR_ARG;
  afq_status s = upload(h, x, t, B);
  if (s != AFQ_OK) return s;
  afq::Mlp* m = h->m;
  return afq::mlp_train(m, afq::mlp_x(m), afq::mlp_t(m), B, iters, lr, loss, h->st) == cudaSuccess
             ? AFQ_OK
             : AFQ_ERR_CUDA;
}

}  // extern "C"
