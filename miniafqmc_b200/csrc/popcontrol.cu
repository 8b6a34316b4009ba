// Population control by the comb (systematic resampling).  The reference has none: its
// driver marks the place ("Branching in real code would happen here",
// miniafqmc_base.cpp:347).  With weights w_i = max(Re W_data[i][1], 0), total T and
// inclusive prefix sums C_i (summed in walker order), tooth j = 0..nw-1 sits at
// t_j = (j + u) T / nw for one uniform u in [0, 1) and picks the first walker with
// C_i > t_j; every copy carries weight T / nw, so the total weight is unchanged and a
// walker's expected number of copies is nw w_i / T.  u comes from Philox4x32-10 on the
// counter (walker offset, 0, step) with the key seed ^ kCombKey, a stream apart from the
// auxiliary fields' (counter (pair, step), key seed), so a run resumed from saved walkers
// at the same seed and step draws the same comb.  The walker offset is the global index
// of the handle's first walker (0 unless the ensemble is sharded): the blocks of a
// sharded ensemble comb independently, each with its own u, and keep their own total
// weight (no weight moves between blocks).
#include "afq_kernels.h"

namespace afq {
namespace {

constexpr unsigned long long kCombKey = 0x9E3779B97F4A7C15ull;

// One CTA: thread 0 forms the prefix sums in walker order (nw doubles), then the threads
// place the teeth by binary search.  idx[j] = parent of copy j.
__global__ void __launch_bounds__(1024)
comb_kernel(const z_t* __restrict__ Wd, int nw, double u, double* __restrict__ C,
            int* __restrict__ idx, double* __restrict__ wnew) {
  __shared__ double total;
  __shared__ int last;   // last walker of positive weight (teeth at T round to it)
  if (threadIdx.x == 0) {
    double s = 0.0;
    int lp = -1;
    for (int i = 0; i < nw; i++) {
      const double w = fmax(Wd[(long long)i * 8 + 1].x, 0.0);
      s += w;
      C[i] = s;
      if (w > 0.0) lp = i;
    }
    total = s;
    last = lp;
    *wnew = s / nw;
  }
  __syncthreads();
  const double T = total;
  for (int j = threadIdx.x; j < nw; j += blockDim.x) {
    const double t = ((double)j + u) * T / (double)nw;
    int lo = 0, hi = nw;   // first i with C[i] > t
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (C[mid] > t) hi = mid;
      else lo = mid + 1;
    }
    idx[j] = lo < nw ? lo : (last >= 0 ? last : j);
  }
}

// copy j of the walkers: W rows [N][2n] and W_data[8] of parent idx[j], weight T / nw
__global__ void comb_gather_kernel(const z_t* __restrict__ W, const z_t* __restrict__ Wd,
                                   const int* __restrict__ idx, const double* __restrict__ wnew,
                                   long long per, int nw, z_t* __restrict__ Wo,
                                   z_t* __restrict__ Wdo) {
  const long long tot = per * nw;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long j = e / per, q = e - j * per;
    const int p = min(max(idx[j], 0), nw - 1);
    Wo[e] = W[(long long)p * per + q];
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 8LL * nw;
       e += (long long)gridDim.x * blockDim.x) {
    const long long j = e / 8, q = e % 8;
    const int p = min(max(idx[j], 0), nw - 1);
    Wdo[e] = q == 1 ? zmk(*wnew, 0.0) : Wd[(long long)p * 8 + q];
  }
}

}  // namespace

double comb_uniform(unsigned long long seed, unsigned long long step, int walker_offset) {
  const unsigned long long key = seed ^ kCombKey;
  uint32_t c[4] = {(uint32_t)walker_offset, 0u, (uint32_t)step, (uint32_t)(step >> 32)};
  philox4x32_10(c, (uint32_t)key, (uint32_t)(key >> 32));
  return (double)(((uint64_t)(c[0] >> 5) << 26) | (c[1] >> 6)) * (1.0 / 9007199254740992.0);
}

cudaError_t launch_comb(z_t* W, z_t* Wd, int nw, long long per, double u, double* C, int* idx,
                        double* wnew, z_t* Wscr, z_t* Wdscr, double* total, cudaStream_t st) {
  comb_kernel<<<1, 1024, 0, st>>>(Wd, nw, u, C, idx, wnew);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // no copies at all unless some walker has positive weight
  double w = 0.0;
  if ((e = cudaMemcpyAsync(&w, wnew, sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return e;
  *total = w * nw;
  if (!(w > 0.0)) return cudaSuccess;
  const long long tot = per * nw;
  const int grid = (int)std::min<long long>((tot + 255) / 256, 148LL * 16);
  comb_gather_kernel<<<grid, 256, 0, st>>>(W, Wd, idx, wnew, per, nw, Wscr, Wdscr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(W, Wscr, sizeof(z_t) * tot, cudaMemcpyDeviceToDevice, st)) !=
      cudaSuccess)
    return e;
  return cudaMemcpyAsync(Wd, Wdscr, sizeof(z_t) * 8 * nw, cudaMemcpyDeviceToDevice, st);
}

}  // namespace afq
