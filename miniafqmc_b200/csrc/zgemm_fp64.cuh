// Batched complex FP64 GEMM on the FP64 FMA pipe, with fused epilogues.
//
// C(b)[m][n] = epilogue( alpha * sum_k A(b)(m,k) * B(b)(k,n) )
//   A_KMAJ: A(m,k) = A[b*sA + m*lda + k]   else A(m,k) = A[b*sA + k*lda + m]
//   B_KMAJ: B(k,n) = B[b*sB + n*ldb + k]   else B(k,n) = B[b*sB + k*ldb + n]
//   B_REAL: B holds real doubles (ZGemmDesc::Br), each multiply-add a real x complex one
//
// sm_100a has no FP64 tensor-core kind for tcgen05 and its FP64 FMA rate equals its
// FP64 MMA rate, so the FP64 form is a register-tiled CUDA-core GEMM: a BM x BN tile per
// CTA, TM x TN complex accumulators per thread, BK-deep k slabs double-buffered in
// shared memory with cp.async.  A and B slabs are stored [k][m] / [k][n] so the inner
// loop reads one A broadcast and TN consecutive B values per k.
#pragma once
#include "afq_common.cuh"

struct ZGemmDesc {
  int M, N, K;
  const z_t* A;
  long long lda, sA;
  const z_t* B;
  long long ldb, sB;
  z_t alpha;
  const double* Br = nullptr;   // real B operand (B_REAL launches; B unused)
};

// ---------------------------------------------------------------- epilogues
// C = alpha*AB + beta*C (beta applied only when beta_nonzero)
struct EpiStore {
  z_t* C;
  long long ldc, sC;
  z_t beta;
  int beta_nonzero;
  AFQ_D void operator()(long long b, int m, int n, z_t v) const {
    z_t* p = C + b * sC + (long long)m * ldc + n;
    if (beta_nonzero) zfma(v, beta, *p);
    *p = v;
  }
};
// T = v and S = v (the first one-body half step: S = Propg1*W, T1 = S)
struct EpiDual {
  z_t* T;
  z_t* S;
  long long ld, s;
  AFQ_D void operator()(long long b, int m, int n, z_t v) const {
    long long o = b * s + (long long)m * ld + n;
    T[o] = v;
    S[o] = v;
  }
};
// Taylor term: T = v, S += v (apply_expM, vHS.hpp:79-89)
struct EpiTaylor {
  z_t* T;
  z_t* S;
  long long ld, s;
  AFQ_D void operator()(long long b, int m, int n, z_t v) const {
    long long o = b * s + (long long)m * ld + n;
    T[o] = v;
    z_t t = S[o];
    S[o] = zadd(t, v);
  }
};

template <int BM, int BN, int BK, int TM, int TN>
struct ZTileCfg {
  static constexpr int NTX = BN / TN, NTY = BM / TM, NT = NTX * NTY;
  static constexpr int LDA_S = BM + 1, LDB_S = BN + 1;
  static constexpr size_t SMEM = sizeof(z_t) * 2 * BK * (LDA_S + LDB_S);
};

template <int BM, int BN, int BK, int TM, int TN, bool A_KMAJ, bool B_KMAJ, class Epi,
          bool B_REAL = false>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
zgemm_kernel(ZGemmDesc d, Epi epi) {
  using Cfg = ZTileCfg<BM, BN, BK, TM, TN>;
  constexpr int NTX = Cfg::NTX, NTY = Cfg::NTY, NT = Cfg::NT;
  constexpr int LDA_S = Cfg::LDA_S, LDB_S = Cfg::LDB_S;
  extern __shared__ __align__(16) unsigned char zg_smem[];
  z_t* As = reinterpret_cast<z_t*>(zg_smem);
  z_t* Bs = As + 2 * BK * LDA_S;
  const int tid = threadIdx.x, tx = tid % NTX, ty = tid / NTX;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const long long b = blockIdx.z;
  const z_t* A = d.A + b * d.sA;
  const z_t* B = B_REAL ? nullptr : d.B + b * d.sB;
  const double* Br = B_REAL ? d.Br + b * d.sB : nullptr;
  double* Bsr = reinterpret_cast<double*>(Bs);   // real B slabs (same row stride)
  const int M = d.M, N = d.N, K = d.K;

  auto load = [&](int stage, int k0) {
    z_t* as = As + stage * BK * LDA_S;
    z_t* bs = Bs + stage * BK * LDB_S;
#pragma unroll 4
    for (int e = tid; e < BM * BK; e += NT) {
      int m, k;
      if (A_KMAJ) { m = e / BK; k = e % BK; } else { k = e / BM; m = e % BM; }
      int gm = m0 + m, gk = k0 + k;
      const z_t* src = A;
      int bytes = 0;
      if (gm < M && gk < K) {
        src = A_KMAJ ? A + (long long)gm * d.lda + gk : A + (long long)gk * d.lda + gm;
        bytes = 16;
      }
      cp_async16(as + k * LDA_S + m, src, bytes);
    }
#pragma unroll 4
    for (int e = tid; e < BN * BK; e += NT) {
      int n, k;
      if (B_KMAJ) { n = e / BK; k = e % BK; } else { k = e / BN; n = e % BN; }
      int gn = n0 + n, gk = k0 + k;
      const bool in = gn < N && gk < K;
      const long long off = B_KMAJ ? (long long)gn * d.ldb + gk : (long long)gk * d.ldb + gn;
      if constexpr (B_REAL) {
        double* bsr = Bsr + stage * BK * LDB_S;
        cp_async8(bsr + k * LDB_S + n, in ? Br + off : Br, in ? 8 : 0);
      } else {
        cp_async16(bs + k * LDB_S + n, in ? B + off : B, in ? 16 : 0);
      }
    }
    cp_async_commit();
  };

  z_t acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = zmk(0, 0);

  const int nk = (K + BK - 1) / BK;
  load(0, 0);
  for (int kt = 0; kt < nk; kt++) {
    if (kt + 1 < nk) {
      load((kt + 1) & 1, (kt + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const z_t* as = As + (kt & 1) * BK * LDA_S;
    const z_t* bs = Bs + (kt & 1) * BK * LDB_S;
    const double* bsr = Bsr + (kt & 1) * BK * LDB_S;
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      z_t a[TM];
#pragma unroll
      for (int i = 0; i < TM; i++) a[i] = as[kk * LDA_S + ty + i * NTY];
      if constexpr (B_REAL) {
        double bb[TN];
#pragma unroll
        for (int j = 0; j < TN; j++) bb[j] = bsr[kk * LDB_S + tx + j * NTX];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int j = 0; j < TN; j++) {
            acc[i][j].x = fma(a[i].x, bb[j], acc[i][j].x);
            acc[i][j].y = fma(a[i].y, bb[j], acc[i][j].y);
          }
      } else {
        z_t bb[TN];
#pragma unroll
        for (int j = 0; j < TN; j++) bb[j] = bs[kk * LDB_S + tx + j * NTX];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int j = 0; j < TN; j++) zfma(acc[i][j], a[i], bb[j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) {
      int m = m0 + ty + i * NTY, n = n0 + tx + j * NTX;
      if (m < M && n < N) epi(b, m, n, zmul(d.alpha, acc[i][j]));
    }
}

// Tile shapes (BM x BN, TM x TN per thread, 256 threads) a launch may use: 0 picks by N,
// 1..kZgCfgs the entries of this list (the set-up tuner times them).  Every shape sums each
// output over K in the same order, so the choice never changes a result.
constexpr int kZgCfgs = 7;
inline const char* zgemm_cfg_name(int cfg) {
  static const char* names[kZgCfgs + 1] = {"rule",     "64x32/4x2", "64x64/4x4", "64x96/4x6",
                                           "32x64/2x4", "32x96/2x6", "128x64/8x4", "32x32/2x2"};
  return cfg >= 0 && cfg <= kZgCfgs ? names[cfg] : "?";
}

// Host-side launcher: tile shape `cfg` (0: picked from N), dynamic shared memory set once
// per instantiation.
template <bool A_KMAJ, bool B_KMAJ, class Epi, bool B_REAL = false>
cudaError_t zgemm_launch(const ZGemmDesc& d, int batch, const Epi& epi, cudaStream_t st,
                         int cfg = 0) {
  if (d.M <= 0 || d.N <= 0 || batch <= 0) return cudaSuccess;
#define AFQ_ZG_CASE(BM_, BN_, TM_, TN_)                                                     \
  {                                                                                        \
    using Cfg = ZTileCfg<BM_, BN_, 16, TM_, TN_>;                                          \
    auto kern = zgemm_kernel<BM_, BN_, 16, TM_, TN_, A_KMAJ, B_KMAJ, Epi, B_REAL>;         \
    static DeviceAttr attr;                                                                \
    const cudaError_t e = attr.ensure(Cfg::SMEM, [kern](size_t b) {                        \
      return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b); \
    });                                                                                    \
    if (e != cudaSuccess) return e;                                                        \
    dim3 grid((d.N + BN_ - 1) / BN_, (d.M + BM_ - 1) / BM_, batch);                        \
    kern<<<grid, Cfg::NT, Cfg::SMEM, st>>>(d, epi);                                        \
    return cudaGetLastError();                                                             \
  }
  switch (cfg) {
    case 1: AFQ_ZG_CASE(64, 32, 4, 2)
    case 2: AFQ_ZG_CASE(64, 64, 4, 4)
    case 3: AFQ_ZG_CASE(64, 96, 4, 6)
    case 4: AFQ_ZG_CASE(32, 64, 2, 4)
    case 5: AFQ_ZG_CASE(32, 96, 2, 6)
    case 6: AFQ_ZG_CASE(128, 64, 8, 4)
    case 7: AFQ_ZG_CASE(32, 32, 2, 2)
    default: break;
  }
  if (d.N <= 32) AFQ_ZG_CASE(64, 32, 4, 2)
  if (d.N <= 64 || (d.N > 96 && d.N <= 128)) AFQ_ZG_CASE(64, 64, 4, 4)
  if (d.N <= 96) AFQ_ZG_CASE(64, 96, 4, 6)
  AFQ_ZG_CASE(64, 64, 4, 4)
#undef AFQ_ZG_CASE
}
