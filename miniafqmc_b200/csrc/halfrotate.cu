// Half-rotation of the Cholesky tensor on the GPU: the set-up product that
// base::halfrotate_cholesky (rotate.hpp:69-169) forms per Cholesky vector on the host,
//   SpvnT[c][s n N + a N + k] = sum_i trial_s(i, a) Spvn[i N + k][c],
// kept where |value| > cutoff, rows c in order, columns in order (the reference's count
// and fill passes).  Steps:
//   1. regroup Spvn (rows i N + k, columns c) into B (rows c N + k, entries ordered by i):
//      counts per B row, an exclusive scan, then one CTA per k walks i in order and appends
//      each nonzero to its B row, so every row's entries are in increasing i (same
//      summation order as the reference's dense product, whose skipped terms are zeros);
//   2. one warp per B row (c, k): lanes over a, both spins, D[c][s][a][k] = sum over the
//      row's entries of trial_s(i, a) v;
//   3. per row c: count |D| > cutoff, scan on the host (nchol values), ordered compaction.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/afqmc_b200.h"
#include "afq_common.cuh"

namespace {

__global__ void hr_count_kernel(const int* __restrict__ ri, const int* __restrict__ ci,
                                long long nrows, int N, int* __restrict__ cnt) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrows;
       r += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(r % N);
    for (int p = ri[r]; p < ri[r + 1]; p++) atomicAdd(&cnt[(long long)ci[p] * N + k], 1);
  }
}

// One CTA per orbital k: rows i N + k for i = 0.. N-1 in order; the nonzeros of one Spvn
// row have distinct Cholesky indices, so their B rows (c, k) are distinct.
__global__ void __launch_bounds__(256)
hr_fill_kernel(const int* __restrict__ ri, const int* __restrict__ ci, const z_t* __restrict__ v,
               int N, const long long* __restrict__ off, int* __restrict__ cur,
               int* __restrict__ bi, z_t* __restrict__ bv) {
  const int k = blockIdx.x;
  for (int i = 0; i < N; i++) {
    const long long r = (long long)i * N + k;
    for (int p = ri[r] + threadIdx.x; p < ri[r + 1]; p += blockDim.x) {
      const long long row = (long long)ci[p] * N + k;
      const long long q = off[row] + cur[row]++;
      bi[q] = i;
      bv[q] = v[p];
    }
    __syncthreads();
  }
}

// D[c][s][a][k] = sum_j trial_s(i_j, a) v_j over B row c N + k; warp per row, lanes on a.
__global__ void __launch_bounds__(256)
hr_rotate_kernel(const long long* __restrict__ off, const int* __restrict__ bi,
                 const z_t* __restrict__ bv, const z_t* __restrict__ trial, long long nrows,
                 int N, int n, z_t* __restrict__ D) {
  const int lane = threadIdx.x & 31;
  const long long row = blockIdx.x * 8LL + (threadIdx.x >> 5);
  if (row >= nrows) return;
  const long long c = row / N;
  const int k = (int)(row % N);
  for (int s = 0; s < 2; s++) {
    const z_t* t = trial + (long long)s * N * n;
    for (int a0 = 0; a0 < n; a0 += 32) {
      const int a = a0 + lane;
      z_t acc = zmk(0, 0);
      if (a < n)
        for (long long j = off[row]; j < off[row + 1]; j++) zfma(acc, t[(long long)bi[j] * n + a], bv[j]);
      if (a < n) D[((c * 2 + s) * n + a) * N + k] = acc;
    }
  }
}

__global__ void __launch_bounds__(256)
hr_rowcount_kernel(const z_t* __restrict__ D, long long width, double cutoff,
                   long long* __restrict__ cnt) {
  __shared__ long long red[8];
  const z_t* row = D + blockIdx.x * width;
  long long m = 0;
  for (long long q = threadIdx.x; q < width; q += blockDim.x)
    if (hypot(row[q].x, row[q].y) > cutoff) m++;
  for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < 8; w++) t += red[w];
    cnt[blockIdx.x] = t;
  }
}

// Ordered compaction of row c: chunks of 256 columns, block-wide prefix of the keep flags.
__global__ void __launch_bounds__(256)
hr_compact_kernel(const z_t* __restrict__ D, long long width, double cutoff,
                  const long long* __restrict__ start, int* __restrict__ cols,
                  z_t* __restrict__ vals) {
  __shared__ int wsum[8];
  __shared__ long long base;
  const z_t* row = D + blockIdx.x * width;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) base = start[blockIdx.x];
  __syncthreads();
  for (long long q0 = 0; q0 < width; q0 += blockDim.x) {
    const long long q = q0 + threadIdx.x;
    const bool keep = q < width && hypot(row[q].x, row[q].y) > cutoff;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < 8; w++) {
      if (w < warp) before += wsum[w];
      total += wsum[w];
    }
    if (keep) {
      const long long pos = base + before + __popc(bal & ((1u << lane) - 1u));
      cols[pos] = (int)q;
      vals[pos] = row[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) base += total;
    __syncthreads();
  }
}

__global__ void hr_scale_kernel(z_t* __restrict__ D, long long count, double scale) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x)
    D[e] = zscale(D[e], scale);
}

int grid_of(long long count, int per) {
  return (int)std::max(1LL, std::min((count + per - 1) / per, 148LL * 16));
}

struct Dev {   // device allocations of one call, freed on every exit
  std::vector<void*> p;
  template <class T>
  cudaError_t get(T** out, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(count, 1));
    if (e == cudaSuccess) {
      p.push_back(q);
      *out = static_cast<T*>(q);
    }
    return e;
  }
  ~Dev() {
    for (void* q : p) cudaFree(q);
  }
};

}  // namespace

extern "C" afq_status afq_halfrotate(int device, const afq_csr_z* Spvn, int nmo, int naea,
                                     int nchol, const double* trial, double cutoff,
                                     double lh_scale, long long* nnz, int32_t* rowIndex,
                                     int32_t* cols, double* vals, double* Lhalf) {
  if (!Spvn || !trial || !nnz || nmo <= 0 || naea <= 0 || nchol <= 0 || !(cutoff >= 0.0) ||
      Spvn->nrows != nmo * nmo || Spvn->ncols != nchol || !Spvn->rowIndex ||
      (Spvn->rowIndex[Spvn->nrows] > 0 && (!Spvn->cols || !Spvn->vals)) ||
      ((cols || vals) && !rowIndex))
    return AFQ_ERR_ARG;
  const int N = nmo, n = naea;
  const long long nr = (long long)N * N, nz = Spvn->rowIndex[nr];
  const long long brows = (long long)nchol * N, width = 2LL * n * N;
  if (cudaSetDevice(device) != cudaSuccess) return AFQ_ERR_CUDA;
  Dev d;
  int *ri = nullptr, *ci = nullptr, *cnt = nullptr, *cur = nullptr, *bi = nullptr;
  long long *off = nullptr, *rc = nullptr, *start = nullptr;
  z_t *v = nullptr, *bv = nullptr, *tr = nullptr, *D = nullptr;
  if (d.get(&ri, nr + 1) || d.get(&ci, nz) || d.get(&v, nz) || d.get(&cnt, brows) ||
      d.get(&cur, brows) || d.get(&off, brows + 1) || d.get(&bi, nz) || d.get(&bv, nz) ||
      d.get(&tr, 2LL * N * n) || d.get(&D, nchol * width) || d.get(&rc, nchol) ||
      d.get(&start, nchol))
    return AFQ_ERR_OOM;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  A(cudaMemcpy(ri, Spvn->rowIndex, sizeof(int) * (nr + 1), cudaMemcpyHostToDevice));
  if (nz) {
    A(cudaMemcpy(ci, Spvn->cols, sizeof(int) * nz, cudaMemcpyHostToDevice));
    A(cudaMemcpy(v, Spvn->vals, sizeof(z_t) * nz, cudaMemcpyHostToDevice));
  }
  A(cudaMemcpy(tr, trial, sizeof(z_t) * 2 * N * n, cudaMemcpyHostToDevice));
  A(cudaMemset(cnt, 0, sizeof(int) * brows));
  A(cudaMemset(cur, 0, sizeof(int) * brows));
  if (e != cudaSuccess) return AFQ_ERR_CUDA;
  // row offsets non-decreasing from 0 and Cholesky indices in [0, nchol): checked on the
  // host before any kernel reads them
  if (Spvn->rowIndex[0] != 0) return AFQ_ERR_ARG;
  for (long long r = 0; r < nr; r++)
    if (Spvn->rowIndex[r + 1] < Spvn->rowIndex[r]) return AFQ_ERR_ARG;
  for (long long p = 0; p < nz; p++)
    if (Spvn->cols[p] < 0 || Spvn->cols[p] >= nchol) return AFQ_ERR_ARG;
  hr_count_kernel<<<grid_of(nr, 256), 256>>>(ri, ci, nr, N, cnt);
  std::vector<int> hc(brows);
  std::vector<long long> ho(brows + 1, 0);
  A(cudaGetLastError());
  A(cudaMemcpy(hc.data(), cnt, sizeof(int) * brows, cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) return AFQ_ERR_CUDA;
  for (long long r = 0; r < brows; r++) ho[r + 1] = ho[r] + hc[r];
  A(cudaMemcpy(off, ho.data(), sizeof(long long) * (brows + 1), cudaMemcpyHostToDevice));
  hr_fill_kernel<<<N, 256>>>(ri, ci, v, N, off, cur, bi, bv);
  A(cudaGetLastError());
  hr_rotate_kernel<<<(int)((brows + 7) / 8), 256>>>(off, bi, bv, tr, brows, N, n, D);
  A(cudaGetLastError());
  hr_rowcount_kernel<<<nchol, 256>>>(D, width, cutoff, rc);
  A(cudaGetLastError());
  std::vector<long long> hrc(nchol), hs(nchol + 1, 0);
  A(cudaMemcpy(hrc.data(), rc, sizeof(long long) * nchol, cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) return AFQ_ERR_CUDA;
  for (int c = 0; c < nchol; c++) hs[c + 1] = hs[c] + hrc[c];
  *nnz = hs[nchol];
  if (hs[nchol] > 0x7fffffffLL) return AFQ_ERR_UNSUPPORTED;   // int32 CSR indices
  if (rowIndex) {
    for (int c = 0; c <= nchol; c++) rowIndex[c] = (int32_t)hs[c];
    if (cols || vals) {
      int* oc = nullptr;
      z_t* ov = nullptr;
      if (d.get(&oc, hs[nchol]) || d.get(&ov, hs[nchol])) return AFQ_ERR_OOM;
      A(cudaMemcpy(start, hs.data(), sizeof(long long) * nchol, cudaMemcpyHostToDevice));
      hr_compact_kernel<<<nchol, 256>>>(D, width, cutoff, start, oc, ov);
      A(cudaGetLastError());
      if (cols) A(cudaMemcpy(cols, oc, sizeof(int) * hs[nchol], cudaMemcpyDeviceToHost));
      if (vals) A(cudaMemcpy(vals, ov, sizeof(z_t) * hs[nchol], cudaMemcpyDeviceToHost));
    }
  }
  if (Lhalf) {
    hr_scale_kernel<<<grid_of(nchol * width, 256), 256>>>(D, nchol * width, lh_scale);
    A(cudaGetLastError());
    A(cudaMemcpy(Lhalf, D, sizeof(z_t) * nchol * width, cudaMemcpyDeviceToHost));
  }
  A(cudaDeviceSynchronize());
  return e == cudaSuccess ? AFQ_OK : AFQ_ERR_CUDA;
}
