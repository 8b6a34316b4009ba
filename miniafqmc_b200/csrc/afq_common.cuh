// Shared device helpers for the sm_100a walker path: complex FP64 arithmetic,
// cp.async staging, block reductions and the Philox4x32-10 normal generator.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstddef>
#include <mutex>

#define AFQ_HD __host__ __device__ __forceinline__
#define AFQ_D __device__ __forceinline__

typedef double2 z_t;

// Host: a kernel's one-time function attributes (dynamic shared memory size, carveout)
// belong to the device current when they are set, and one process may drive handles on
// several devices (afq_system_desc::device) from several threads.  ensure(bytes, set)
// runs set(bytes) the first time a launch on the current device needs `bytes` or more,
// under a lock, so the recorded size (and the attribute) only grows.  A device ordinal
// outside the table runs set(bytes) every time.
struct DeviceAttr {
  static constexpr int kDevices = 64;
  std::atomic<size_t> set_bytes[kDevices] = {};
  std::mutex mu;
  template <class F>
  cudaError_t ensure(size_t bytes, F&& set) {
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kDevices) return set(bytes);
    if (set_bytes[d].load(std::memory_order_acquire) >= bytes) return cudaSuccess;
    std::lock_guard<std::mutex> lock(mu);
    if (set_bytes[d].load(std::memory_order_relaxed) >= bytes) return cudaSuccess;
    const cudaError_t e = set(bytes);
    if (e == cudaSuccess) set_bytes[d].store(bytes, std::memory_order_release);
    return e;
  }
};

AFQ_HD z_t zmk(double r, double i) { return make_double2(r, i); }
AFQ_HD z_t zadd(z_t a, z_t b) { return make_double2(a.x + b.x, a.y + b.y); }
AFQ_HD z_t zsub(z_t a, z_t b) { return make_double2(a.x - b.x, a.y - b.y); }
AFQ_HD z_t zmul(z_t a, z_t b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
AFQ_HD z_t zscale(z_t a, double s) { return make_double2(a.x * s, a.y * s); }
AFQ_HD z_t zconj(z_t a) { return make_double2(a.x, -a.y); }
// acc += a * b
AFQ_HD void zfma(z_t& acc, z_t a, z_t b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
AFQ_HD void zfma_conj(z_t& acc, z_t a, z_t b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
// acc += r * b with r real
AFQ_HD void zfma_r(z_t& acc, double r, z_t b) {
  acc.x = fma(r, b.x, acc.x);
  acc.y = fma(r, b.y, acc.y);
}
// 1 / a with Smith's scaling
AFQ_HD z_t zrecip(z_t a) {
  if (fabs(a.x) >= fabs(a.y)) {
    double r = a.y / a.x, d = a.x + a.y * r;
    return make_double2(1.0 / d, -r / d);
  } else {
    double r = a.x / a.y, d = a.x * r + a.y;
    return make_double2(r / d, -1.0 / d);
  }
}
AFQ_HD z_t zdiv(z_t a, z_t b) { return zmul(a, zrecip(b)); }
AFQ_HD double zabs1(z_t a) { return fabs(a.x) + fabs(a.y); }

// ------------------------------------------------------------------ cp.async
AFQ_D void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
AFQ_D void cp_async8(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
AFQ_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
AFQ_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ------------------------------------------------------------------ reductions
AFQ_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
AFQ_D z_t warp_zsum(z_t v) {
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  return v;
}
// Deterministic block sum (fixed tree); every thread gets the result.  `red` holds
// blockDim.x/32 entries.
AFQ_D z_t block_zsum(z_t v, z_t* red) {
  v = warp_zsum(v);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  z_t t = zmk(0, 0);
  if (wid == 0) {
    t = lane < nwarp ? red[lane] : zmk(0, 0);
    t = warp_zsum(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  t = red[0];
  __syncthreads();
  return t;
}

// ------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
AFQ_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * c[0];
    uint64_t p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += W0; k1 += W1;
  }
}

// N(0,1) pair number j of step `step`: Box-Muller on two 53-bit uniforms.
AFQ_D void normal_pair(uint64_t seed, uint64_t step, uint64_t j, double* x0, double* x1) {
  uint32_t c[4] = {(uint32_t)j, (uint32_t)(j >> 32), (uint32_t)step, (uint32_t)(step >> 32)};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double s53 = 1.0 / 9007199254740992.0;
  double u1 = ((double)(((uint64_t)(c[0] >> 5) << 26) | (c[1] >> 6)) + 1.0) * s53;
  double u2 = (double)(((uint64_t)(c[2] >> 5) << 26) | (c[3] >> 6)) * s53;
  double r = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586 * u2;
  double sn, cs;
  sincos(th, &sn, &cs);
  *x0 = r * cs;
  *x1 = r * sn;
}

// Device-resident scalars of one walker set, read and written by the step kernels so a
// captured CUDA graph can be replayed without host updates.
struct DevScalars {
  unsigned long long seed;
  unsigned long long step;   // Philox step counter, incremented by the weight kernel
  double eshift;             // Eshift (miniafqmc_base.cpp:187,327)
  double e4sum;              // sum of Re W_data[:,4] from the last weight update
  double esum[2];            // sum Re(eloc) Re(w), sum Re(w) from the last energy
  int singular;              // count of singular overlap matrices seen
  int walker_offset;         // global index of this handle's first walker
  long long nwalk_global;    // walkers in the whole (possibly sharded) ensemble
};
