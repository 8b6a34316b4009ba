// Self-test entry of the tcgen05 GEMM: host fp32 operands in, fp32 product out.
// Used by the numerics tests to compare the tensor-core kernel with a plain fp32
// reference of the same operation on bf16- or tf32-representable inputs.
#include <cuda_bf16.h>
#include <vector>

#include "../../include/afqmc_b200.h"
#include "afq_mixed.h"
#include "tc_gemm.cuh"

namespace {

struct EpiStoreF32 {
  static constexpr bool kTile = false, kPair = false;
  float* C;
  int M, N;
  long long sC;
  AFQ_D void operator()(int b, int, int m, int n0, const float* v) const {
    if (m >= M) return;
    float* row = C + (long long)b * sC + (long long)m * N;
#pragma unroll
    for (int i = 0; i < 32; i++)
      if (n0 + i < N) row[n0 + i] = v[i];
  }
};

// Split modes (bf16 hi + lo parts of both operands, hi*hi + hi*lo + lo*hi):
// 5 / 6 = per-tile kernel with 128- / 64-byte K slabs, 7 / 8 = persistent kernel (two
// epilogue warpgroups) with 128- / 64-byte K slabs.
template <int BN>
cudaError_t run_split(const void* dA, const void* dAl, const void* dB, const void* dBl,
                      float* dC, int M, int N, int K, int batch, int mode, int* derr,
                      cudaStream_t st) {
  tc::Maps maps;
  const uint32_t slab = (mode == 6 || mode == 8) ? 64 : 128;
  const uint64_t sa = (uint64_t)M * K, sb = (uint64_t)N * K;
  if (tc::make_kmajor_map(&maps.a, dA, false, K, M, batch, K, sa, 128, slab) != CUDA_SUCCESS ||
      tc::make_kmajor_map(&maps.a_lo, dAl, false, K, M, batch, K, sa, 128, slab) != CUDA_SUCCESS ||
      tc::make_kmajor_map(&maps.b, dB, false, K, N, batch, K, sb, BN, slab) != CUDA_SUCCESS ||
      tc::make_kmajor_map(&maps.b_lo, dBl, false, K, N, batch, K, sb, BN, slab) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  tc::GemmShape g{M, N, K, batch, 128, (M + 127) / 128, true, true, 0};
  EpiStoreF32 epi{dC, M, N, (long long)M * N};
  if (mode == 5) return tc::launch<BN, 2, 1, true, EpiStoreF32>(maps, g, epi, derr, st);
  if (mode == 6) return tc::launch<BN, 4, 1, true, EpiStoreF32, 1, 64>(maps, g, epi, derr, st);
  if (mode == 7) return tc::launch_persistent<BN, 2, 1, true, EpiStoreF32, 2>(maps, g, epi, derr, st);
  return tc::launch_persistent<BN, 4, 1, true, EpiStoreF32, 2, 64>(maps, g, epi, derr, st);
}

template <int BN, bool TF32>
cudaError_t run(const void* dA, const void* dB, float* dC, int M, int N, int K, int batch,
                int mode, int* derr, cudaStream_t st) {
  tc::Maps maps;
  const uint32_t slab = mode >= 3 ? 64 : 128;   // modes 3 / 4: 64-byte K slabs
  if (tc::make_kmajor_map(&maps.a, dA, TF32, K, M, batch, K, (uint64_t)M * K, 128, slab) !=
      CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  if (tc::make_kmajor_map(&maps.b, dB, TF32, K, N, batch, K, (uint64_t)N * K, BN, slab) !=
      CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  maps.a_lo = maps.a;
  maps.b_lo = maps.b;
  tc::GemmShape g{M, N, K, batch, 128, (M + 127) / 128, true, true, 0};
  EpiStoreF32 epi{dC, M, N, (long long)M * N};
  if (mode == 3) return tc::launch<BN, 4, (TF32 ? 2 : 1), false, EpiStoreF32, 1, 64>(maps, g, epi, derr, st);
  if (mode == 4) return tc::launch_persistent<BN, 4, (TF32 ? 2 : 1), false, EpiStoreF32, 1, 64>(maps, g, epi, derr, st);
  if (mode == 1) return tc::launch_persistent<BN, 4, (TF32 ? 2 : 1), false, EpiStoreF32, 1>(maps, g, epi, derr, st);
  if (mode == 2) return tc::launch_persistent<BN, 4, (TF32 ? 2 : 1), false, EpiStoreF32, 2>(maps, g, epi, derr, st);
  return tc::launch<BN, 4, (TF32 ? 2 : 1), false>(maps, g, epi, derr, st);
}

}  // namespace

extern "C" afq_status afq_selftest_tc_gemm(int M, int N, int K, int batch, int tf32, int bn,
                                          int mode, const float* A, const float* B, float* C,
                                          int* kernel_err) {
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0 || !A || !B || !C || mode < 0 || mode > 8)
    return AFQ_ERR_ARG;
  if (bn != 64 && bn != 128 && bn != 192 && bn != 256) return AFQ_ERR_ARG;
  if (K % 8 != 0) return AFQ_ERR_UNSUPPORTED;   // 16-byte row strides for TMA
  const bool split = mode >= 5;
  if (split && tf32) return AFQ_ERR_UNSUPPORTED;
  const size_t na = (size_t)batch * M * K, nb = (size_t)batch * N * K, nc = (size_t)batch * M * N;
  void *dA = nullptr, *dB = nullptr, *dAl = nullptr, *dBl = nullptr;
  float* dC = nullptr;
  int* derr = nullptr;
  cudaStream_t st = nullptr;
  afq_status s = AFQ_OK;
  const size_t esz = tf32 ? 4 : 2;
  if (cudaMalloc(&dA, na * esz) != cudaSuccess || cudaMalloc(&dB, nb * esz) != cudaSuccess ||
      cudaMalloc(&dC, nc * 4) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess ||
      cudaStreamCreate(&st) != cudaSuccess) {
    s = AFQ_ERR_OOM;
  }
  if (s == AFQ_OK && split &&
      (cudaMalloc(&dAl, na * 2) != cudaSuccess || cudaMalloc(&dBl, nb * 2) != cudaSuccess))
    s = AFQ_ERR_OOM;
  if (s == AFQ_OK) {
    if (tf32) {
      cudaMemcpy(dA, A, na * 4, cudaMemcpyHostToDevice);
      cudaMemcpy(dB, B, nb * 4, cudaMemcpyHostToDevice);
    } else {
      // hi = A rounded to bf16; the split modes also take lo = (A - hi) rounded to bf16
      std::vector<__nv_bfloat16> ha(na), hb(nb), la(split ? na : 0), lb(split ? nb : 0);
      for (size_t i = 0; i < na; i++) {
        ha[i] = __float2bfloat16_rn(A[i]);
        if (split) la[i] = __float2bfloat16_rn(A[i] - __bfloat162float(ha[i]));
      }
      for (size_t i = 0; i < nb; i++) {
        hb[i] = __float2bfloat16_rn(B[i]);
        if (split) lb[i] = __float2bfloat16_rn(B[i] - __bfloat162float(hb[i]));
      }
      cudaMemcpy(dA, ha.data(), na * 2, cudaMemcpyHostToDevice);
      cudaMemcpy(dB, hb.data(), nb * 2, cudaMemcpyHostToDevice);
      if (split) {
        cudaMemcpy(dAl, la.data(), na * 2, cudaMemcpyHostToDevice);
        cudaMemcpy(dBl, lb.data(), nb * 2, cudaMemcpyHostToDevice);
      }
    }
    cudaMemset(dC, 0, nc * 4);
    cudaMemset(derr, 0, sizeof(int));
    cudaError_t e;
    if (split) {
      if (bn == 64) e = run_split<64>(dA, dAl, dB, dBl, dC, M, N, K, batch, mode, derr, st);
      else if (bn == 192) e = run_split<192>(dA, dAl, dB, dBl, dC, M, N, K, batch, mode, derr, st);
      else if (bn == 256) e = run_split<256>(dA, dAl, dB, dBl, dC, M, N, K, batch, mode, derr, st);
      else e = run_split<128>(dA, dAl, dB, dBl, dC, M, N, K, batch, mode, derr, st);
    } else if (bn == 256) e = tf32 ? run<256, true>(dA, dB, dC, M, N, K, batch, mode, derr, st)
                                   : run<256, false>(dA, dB, dC, M, N, K, batch, mode, derr, st);
    else if (bn == 64) e = tf32 ? run<64, true>(dA, dB, dC, M, N, K, batch, mode, derr, st)
                           : run<64, false>(dA, dB, dC, M, N, K, batch, mode, derr, st);
    else if (bn == 192) e = tf32 ? run<192, true>(dA, dB, dC, M, N, K, batch, mode, derr, st)
                                 : run<192, false>(dA, dB, dC, M, N, K, batch, mode, derr, st);
    else e = tf32 ? run<128, true>(dA, dB, dC, M, N, K, batch, mode, derr, st)
                  : run<128, false>(dA, dB, dC, M, N, K, batch, mode, derr, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = AFQ_ERR_CUDA;
    cudaMemcpy(C, dC, nc * 4, cudaMemcpyDeviceToHost);
    if (kernel_err) cudaMemcpy(kernel_err, derr, sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (st) cudaStreamDestroy(st);
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dAl);
  cudaFree(dBl);
  cudaFree(dC);
  cudaFree(derr);
  return s;
}

extern "C" afq_status afq_set_tc_wait_limit(int device, long long clocks) {
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess)
    return AFQ_ERR_ARG;
  // every module holding tensor-core kernels keeps its own copy of the bound
  cudaError_t e = tc::set_wait_clocks(clocks);
  if (e == cudaSuccess) e = afq::mixed_set_wait_clocks(clocks);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaSetDevice(prev);
  return e == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}
