// Exchange energy of a walker batch with no device allocation at all.
//
// Some callers cannot call cudaMalloc: code that records its work into a CUDA graph
// under stream capture (an allocation there breaks the capture), and host frameworks
// that hand every byte of device memory to their own pool and forbid allocations after
// start-up.  This entry point serves them: the caller passes device inputs and outputs,
// and the partial sums the exchange kernel needs live in a fixed file-scope device
// array instead of a per-handle buffer.
#include <cstdint>
#include <mutex>

#include "../../include/afqmc_b200.h"
#include "afq_kernels.h"

namespace {

// Partial sums of the exchange contraction: one complex value per (walker, spin,
// Cholesky block); 2^18 of them = 4 MiB, held by every device that loads the library.
constexpr long long kMaxExchangePartials = 1LL << 18;
static __device__ __align__(256) z_t g_exchange_scratch[kMaxExchangePartials];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
z_t* g_scratch_addr[kMaxDevices] = {};

// EK[w] = 1/2 sum over spins and Cholesky blocks of the partials, in a fixed order.
__global__ void __launch_bounds__(128)
exchange_finish_kernel(const z_t* __restrict__ part, int nblk, z_t* __restrict__ ek) {
  __shared__ z_t red[4];
  const int w = blockIdx.x;
  z_t s = zmk(0, 0);
  for (int q = threadIdx.x; q < 2 * nblk; q += blockDim.x)
    s = zadd(s, part[(long long)w * 2 * nblk + q]);
  s = block_zsum(s, red);
  if (threadIdx.x == 0) ek[w] = zscale(s, 0.5);
}

}  // namespace

extern "C" afq_status afq_exchange_energy_noalloc(const double* Lh, const double* Gc, int nmo,
                                                  int naea, int nchol, int nwalk, double* ek,
                                                  void* stream) {
  if (!Lh || !Gc || !ek || nmo <= 0 || naea <= 0 || nchol <= 0 || nwalk <= 0)
    return AFQ_ERR_ARG;
  // the exchange kernel reads Lh and Gc with 16-byte asynchronous copies and the finish
  // kernel stores whole complex values: a buffer that is only 8-byte aligned (a view at an
  // odd double offset) would fault on the device, so it is refused here
  if ((reinterpret_cast<uintptr_t>(Lh) | reinterpret_cast<uintptr_t>(Gc) |
       reinterpret_cast<uintptr_t>(ek)) & 15u)
    return AFQ_ERR_ARG;
  if (naea > 96 || naea > nmo) return AFQ_ERR_UNSUPPORTED;
  int nblk = 0;
  afq::launch_exchange(nullptr, nullptr, nmo, naea, nchol, nwalk, nullptr, &nblk, nullptr);
  const long long used = 2LL * nwalk * nblk;
  if (used > kMaxExchangePartials) return AFQ_ERR_UNSUPPORTED;   // batch too large for scratch
  // one CTA row per group of 96 / naea walkers: the grid's y extent is at most 65535
  if ((nwalk + 96 / naea - 1) / (96 / naea) > 65535) return AFQ_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return AFQ_ERR_CUDA;
  z_t* scratch = nullptr;
  {
    // set-up, once per device with that device current: the host-side symbol is only a
    // stand-in, the kernels need the device address of the array
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_exchange_scratch) != cudaSuccess || !p) return AFQ_ERR_CUDA;
      g_scratch_addr[dev] = static_cast<z_t*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: clear the part this call reads
  if (cudaMemsetAsync(scratch, 0, sizeof(z_t) * used, st) != cudaSuccess) return AFQ_ERR_CUDA;
  int nb = 0;
  if (afq::launch_exchange(reinterpret_cast<const z_t*>(Lh), reinterpret_cast<const z_t*>(Gc), nmo,
                           naea, nchol, nwalk, scratch, &nb, st) != cudaSuccess)
    return AFQ_ERR_CUDA;
  exchange_finish_kernel<<<nwalk, 128, 0, st>>>(scratch, nb, reinterpret_cast<z_t*>(ek));
  return cudaGetLastError() == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}
