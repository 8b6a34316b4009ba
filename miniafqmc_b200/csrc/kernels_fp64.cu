// FP64 kernels of the walker step (the plain form): mixed density matrix and overlaps,
// sigma (Philox), CSR SpMM for vHS / vbias / Vakbl, weight update, Householder
// re-orthogonalisation and the local energy.  Internal device layouts:
//   W   [nw][N][2n]   (spin s occupies columns s*n .. s*n+n-1 of each row)
//   tw  [N][2n]       trial, same interleave
//   Gc  [nw][2][n][N] per-walker compact density matrices (linear index s*n*N + a*N + k)
//   vHS [nw][N][N], vbias / X / xraw [nchol][nw] (reference layout)
#include <cstdlib>

#include "afq_kernels.h"
#include "afq_common.cuh"

namespace afq {

// ============================================================ mixed density matrix
// One CTA per (walker, spin).  T1 = W_s^T tw_s (n x n, mixed_density_matrix.hpp:83);
// Gauss-Jordan with partial pivoting (max |re|+|im|, as izamax) gives det(T1) and
// T1^-1 (ma_operations.hpp:244-260); Gc_s = T1^-1 W_s^T (mixed_density_matrix.hpp:91).
// want_gc == 0 runs only the LU elimination for the determinant (Overlap, :124-138).
constexpr int DM_KC = 32;
constexpr int DM_THREADS = 256;

size_t dm_smem_bytes(int n) {
  size_t ldT = n + 1;
  size_t buf = std::max((size_t)2 * DM_KC * n, (size_t)n * 65);   // phase 1 slabs | W^T chunk
  return sizeof(z_t) * (n * ldT + buf + n) + sizeof(int) * n;
}

__global__ void __launch_bounds__(DM_THREADS)
dm_kernel(const z_t* __restrict__ W, const z_t* __restrict__ tw, int N, int n,
          z_t* __restrict__ Gc, z_t* __restrict__ Wd, int* __restrict__ info, int want_gc,
          int save_old) {
  extern __shared__ __align__(16) unsigned char dm_smem[];
  const int w = blockIdx.x >> 1, s = blockIdx.x & 1;
  const int ldT = n + 1;
  z_t* T = reinterpret_cast<z_t*>(dm_smem);
  z_t* buf = T + n * ldT;
  const int bufsz = max(2 * DM_KC * n, n * 65);
  z_t* fcol = buf + bufsz;
  int* perm = reinterpret_cast<int*>(fcol + n);
  __shared__ int s_piv, s_sing;
  const long long ldw = 2 * n;
  const z_t* Ws = W + (long long)w * N * ldw + s * n;
  const z_t* ts = tw + s * n;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nout = n * n;

  // ---- phase 1: T1 = W_s^T tw_s; thread (ta, tb) of a 16 x 16 grid owns rows
  // a = ta + 16i and columns b = tb + 16j (i, j < R = ceil(n/16)), a register block that
  // reuses each shared-memory operand R times
  const int R = (n + 15) / 16;
  const int ta = tid / 16, tb = tid % 16;
  {
    z_t acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = zmk(0, 0);
    for (int k0 = 0; k0 < N; k0 += DM_KC) {
      const int kc = min(DM_KC, N - k0);
      for (int e = tid; e < kc * n; e += nt) {
        int kk = e / n, a = e % n;
        buf[kk * n + a] = Ws[(long long)(k0 + kk) * ldw + a];
        buf[DM_KC * n + kk * n + a] = ts[(long long)(k0 + kk) * ldw + a];
      }
      __syncthreads();
      for (int kk = 0; kk < kc; kk++) {
        z_t av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int a = ta + 16 * i, b = tb + 16 * i;
          av[i] = (i < R && a < n) ? buf[kk * n + a] : zmk(0, 0);
          bv[i] = (i < R && b < n) ? buf[DM_KC * n + kk * n + b] : zmk(0, 0);
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (i < R && j < R) zfma(acc[i][j], av[i], bv[j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int a = ta + 16 * i, b = tb + 16 * j;
        if (i < R && j < R && a < n && b < n) T[a * ldT + b] = acc[i][j];
      }
  }
  if (tid == 0) s_sing = 0;
  __syncthreads();

  // ---- phase 2: pivoted elimination
  z_t det = zmk(1.0, 0.0);
  for (int j = 0; j < n; j++) {
    if (tid < 32) {
      double best = -1.0;
      int bi = n;
      for (int i = j + tid; i < n; i += 32) {
        double v = zabs1(T[i * ldT + j]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (tid == 0) { s_piv = bi; perm[j] = bi; }
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j)
      for (int c = tid; c < n; c += nt) {
        z_t t = T[j * ldT + c];
        T[j * ldT + c] = T[p * ldT + c];
        T[p * ldT + c] = t;
      }
    __syncthreads();
    const z_t pv = T[j * ldT + j];
    if (pv.x == 0.0 && pv.y == 0.0) {  // exactly singular: uniform across the CTA
      if (tid == 0) s_sing = 1;
      break;
    }
    if (tid == 0) {
      det = zmul(det, pv);
      if (p != j) det = zmk(-det.x, -det.y);
    }
    const z_t inv = zrecip(pv);
    if (!want_gc) {
      const int m = n - j - 1;
      for (int e = tid; e < m * m; e += nt) {
        int i = j + 1 + e / m, c = j + 1 + e % m;
        z_t f = zmul(T[i * ldT + j], inv);
        T[i * ldT + c] = zsub(T[i * ldT + c], zmul(f, T[j * ldT + c]));
      }
      __syncthreads();
    } else {
      for (int i = tid; i < n; i += nt) fcol[i] = T[i * ldT + j];
      __syncthreads();
      for (int c = tid; c < n; c += nt)
        T[j * ldT + c] = (c == j) ? inv : zmul(T[j * ldT + c], inv);
      __syncthreads();
      for (int e = tid; e < nout; e += nt) {
        int i = e / n, c = e % n;
        if (i == j) continue;
        z_t base = (c == j) ? zmk(0, 0) : T[i * ldT + c];
        T[i * ldT + c] = zsub(base, zmul(fcol[i], T[j * ldT + c]));
      }
      __syncthreads();
    }
  }
  __syncthreads();
  const int sing = s_sing;
  if (sing) det = zmk(0, 0);

  // ---- phase 3: Gc_s = T1^-1 W_s^T
  if (want_gc) {
    z_t* Gout = Gc + ((long long)w * 2 + s) * n * N;
    if (!sing) {
      for (int j = n - 1; j >= 0; j--) {   // undo the row interchanges on the columns
        int p = perm[j];
        if (p != j)
          for (int r = tid; r < n; r += nt) {
            z_t t = T[r * ldT + j];
            T[r * ldT + j] = T[r * ldT + p];
            T[r * ldT + p] = t;
          }
        __syncthreads();
      }
    }
    // Gc[a][k] = sum_b Tinv[a][b] W[k][b] over 64-row chunks of W: thread (ta, tk) owns
    // rows a = ta + 16i (i < R) and chunk columns k = tk + 16j (j < 4)
    constexpr int KC3 = 64;
    const int tk = tb;
    for (int k0 = 0; k0 < N; k0 += KC3) {
      const int kc = min(KC3, N - k0);
      for (int e = tid; e < kc * n; e += nt) {
        int kk = e / n, b = e % n;
        buf[b * (KC3 + 1) + kk] = Ws[(long long)(k0 + kk) * ldw + b];
      }
      __syncthreads();
      z_t acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = zmk(0, 0);
      if (!sing)
        for (int b = 0; b < n; b++) {
          z_t tv[4], wv[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int a = ta + 16 * i;
            tv[i] = (i < R && a < n) ? T[a * ldT + b] : zmk(0, 0);
            wv[i] = buf[b * (KC3 + 1) + tk + 16 * i];
          }
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
              if (i < R) zfma(acc[i][j], tv[i], wv[j]);
        }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int a = ta + 16 * i, kk = tk + 16 * j;
          if (i < R && a < n && kk < kc) Gout[(long long)a * N + k0 + kk] = acc[i][j];
        }
      __syncthreads();
    }
  }
  if (tid == 0) {
    z_t* d = Wd + (long long)w * 8;
    if (save_old) {
      if (s == 0) d[5] = d[4];
      d[6 + s] = d[2 + s];
    }
    d[2 + s] = det;
    info[w * 2 + s] = sing;
  }
}

cudaError_t launch_dm(const z_t* W, const z_t* tw, int N, int n, int nw, z_t* Gc, z_t* Wd,
                      int* info, int want_gc, int save_old, cudaStream_t st) {
  size_t smem = dm_smem_bytes(n);
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(smem, [](size_t b) {
    cudaError_t r = cudaFuncSetAttribute(dm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)b);
    if (r == cudaSuccess)   // several CTAs per SM need the full shared-memory carveout
      r = cudaFuncSetAttribute(dm_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    return r;
  });
  if (e != cudaSuccess) return e;
  dm_kernel<<<2 * nw, DM_THREADS, smem, st>>>(W, tw, N, n, Gc, Wd, info, want_gc, save_old);
  return cudaGetLastError();
}

// ============================================================ sigma
// X = x + i vbias, hybridW[w] = -sum_c i vb (x + i/2 vb)  (miniafqmc_base.cpp:281-289).
// Block (32 walkers) x (32 groups of Cholesky rows); fixed-order reduction over groups.
__global__ void __launch_bounds__(1024)
sigma_kernel(const z_t* __restrict__ vbias, z_t* __restrict__ X, double* __restrict__ xraw,
             z_t* __restrict__ hybridW, int nchol, int nw, const DevScalars* __restrict__ sc,
             int use_xraw) {
  __shared__ z_t red[32][33];
  const int lane = threadIdx.x, g = threadIdx.y;
  const int w = blockIdx.x * 32 + lane;
  const unsigned long long seed = sc->seed, step = sc->step;
  const long long nwg = sc->nwalk_global > 0 ? sc->nwalk_global : nw;
  const long long woff = sc->walker_offset;
  z_t hw = zmk(0, 0);
  if (w < nw) {
    for (int c = g; c < nchol; c += 32) {
      long long e = (long long)c * nw + w;
      double x;
      if (use_xraw) {
        x = xraw[e];
      } else {
        // the stream is indexed by the global walker so shards reproduce one ensemble
        long long eg = (long long)c * nwg + woff + w;
        double x0, x1;
        normal_pair(seed, step, (unsigned long long)eg >> 1, &x0, &x1);
        x = (eg & 1) ? x1 : x0;
        xraw[e] = x;
      }
      z_t vb = vbias[e];
      z_t ivb = zmk(-vb.y, vb.x);                      // i vb
      z_t t = zmk(x - 0.5 * vb.y, 0.5 * vb.x);         // x + (i/2) vb
      hw = zsub(hw, zmul(ivb, t));
      X[e] = zmk(x - vb.y, vb.x);                      // x + i vb
    }
  }
  red[g][lane] = hw;
  __syncthreads();
  if (g == 0 && w < nw) {
    z_t s = zmk(0, 0);
    for (int q = 0; q < 32; q++) s = zadd(s, red[q][lane]);
    hybridW[w] = s;
  }
}

cudaError_t launch_sigma(const z_t* vbias, z_t* X, double* xraw, z_t* hybridW, int nchol,
                         int nw, const DevScalars* sc, int use_xraw, cudaStream_t st) {
  sigma_kernel<<<(nw + 31) / 32, dim3(32, 32), 0, st>>>(vbias, X, xraw, hybridW, nchol, nw, sc,
                                                         use_xraw);
  return cudaGetLastError();
}

// ============================================================ CSR x dense (walker-fast B)
// out[w][r] = sum_p A[p] B[col(p)][w] for the rows r of a CSR, B [ncols][nw] walker
// fastest (vHS = Spvn X, vHS.hpp:47-56).  A warp owns a row; its lanes own walkers;
// the nonzeros of a row are fetched 32 at a time and broadcast with shuffles.  The CTA
// stages its [rows x walkers] results in shared memory and writes them walker-major.
// ROWS warps (rows) per CTA, WPL walkers per lane (CTA covers 32 WPL walkers); the set-up
// tuner picks the shape (every shape sums each output in CSR order: same results).
template <bool REALV, int ROWS, int WPL>
__global__ void __launch_bounds__(ROWS * 32)
csr_walker_kernel(const int* __restrict__ rowIndex, const int* __restrict__ cols,
                  const z_t* __restrict__ zvals, const double* __restrict__ rvals,
                  const z_t* __restrict__ B, int nrows, int nw, z_t* __restrict__ out,
                  long long out_ld) {
  constexpr int WALK = 32 * WPL;
  __shared__ z_t tile[ROWS][WALK + 1];
  const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
  const int r0 = blockIdx.x * ROWS, r = r0 + wy;
  const int w0 = blockIdx.y * WALK;
  z_t acc[WPL];
#pragma unroll
  for (int j = 0; j < WPL; j++) acc[j] = zmk(0, 0);
  if (r < nrows) {
    const int beg = rowIndex[r], end = rowIndex[r + 1];
    for (int p0 = beg; p0 < end; p0 += 32) {
      const int cnt = min(32, end - p0);
      int myc = 0;
      z_t myv = zmk(0, 0);
      double myr = 0.0;
      if (lane < cnt) {
        myc = cols[p0 + lane];
        if (REALV) myr = rvals[p0 + lane];
        else myv = zvals[p0 + lane];
      }
      for (int q = 0; q < cnt; q++) {
        const int c = __shfl_sync(0xffffffffu, myc, q);
        const z_t* br = B + (long long)c * nw;
        if (REALV) {
          const double v = __shfl_sync(0xffffffffu, myr, q);
#pragma unroll
          for (int j = 0; j < WPL; j++) {
            const int w = w0 + 32 * j + lane;
            if (w < nw) zfma_r(acc[j], v, br[w]);
          }
        } else {
          z_t v;
          v.x = __shfl_sync(0xffffffffu, myv.x, q);
          v.y = __shfl_sync(0xffffffffu, myv.y, q);
#pragma unroll
          for (int j = 0; j < WPL; j++) {
            const int w = w0 + 32 * j + lane;
            if (w < nw) zfma(acc[j], v, br[w]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < WPL; j++) tile[wy][32 * j + lane] = acc[j];
  __syncthreads();
  for (int e = threadIdx.x; e < ROWS * WALK; e += ROWS * 32) {
    const int wl = e / ROWS, rr = e % ROWS;
    const int w = w0 + wl, rw = r0 + rr;
    if (w < nw && rw < nrows) out[(long long)w * out_ld + rw] = tile[rr][wl];
  }
}

template <int ROWS, int WPL>
cudaError_t csr_walker_launch(const int* rowIndex, const int* cols, const z_t* zvals,
                              const double* rvals, const z_t* B, int nrows, int nw, z_t* out,
                              long long out_ld, cudaStream_t st) {
  dim3 grid((nrows + ROWS - 1) / ROWS, (nw + 32 * WPL - 1) / (32 * WPL));
  if (rvals)
    csr_walker_kernel<true, ROWS, WPL><<<grid, ROWS * 32, 0, st>>>(rowIndex, cols, nullptr, rvals,
                                                                   B, nrows, nw, out, out_ld);
  else
    csr_walker_kernel<false, ROWS, WPL><<<grid, ROWS * 32, 0, st>>>(rowIndex, cols, zvals, nullptr,
                                                                    B, nrows, nw, out, out_ld);
  return cudaGetLastError();
}

const char* csr_walker_cfg_name(int cfg) {
  static const char* names[kCsrWalkerCfgs + 1] = {"16x2", "16x2", "8x2", "4x2",
                                                  "16x1", "8x4",  "4x4", "32x1"};
  return cfg >= 0 && cfg <= kCsrWalkerCfgs ? names[cfg] : "?";
}

// cfg: 0 built-in (16 rows x 2 walkers per lane), 1..kCsrWalkerCfgs the shapes above
cudaError_t launch_csr_walker(const int* rowIndex, const int* cols, const z_t* zvals,
                              const double* rvals, const z_t* B, int nrows, int nw, z_t* out,
                              long long out_ld, cudaStream_t st, int cfg) {
  switch (cfg) {
    case 2: return csr_walker_launch<8, 2>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
    case 3: return csr_walker_launch<4, 2>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
    case 4: return csr_walker_launch<16, 1>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
    case 5: return csr_walker_launch<8, 4>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
    case 6: return csr_walker_launch<4, 4>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
    case 7: return csr_walker_launch<32, 1>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
    default: return csr_walker_launch<16, 2>(rowIndex, cols, zvals, rvals, B, nrows, nw, out, out_ld, st);
  }
}

// ============================================================ CSR x walker-major G
// out[r][w] = sum_p A[p] G[w][col(p)] (vbias = SpvnT Gc when SpvnT is sparse,
// vbias.hpp:63; Gcloc = Vakbl Gc, energy.hpp:89).  Warp per row, lanes over walkers.
__global__ void __launch_bounds__(256)
csr_gather_kernel(const int* __restrict__ rowIndex, const int* __restrict__ cols,
                  const z_t* __restrict__ vals, const z_t* __restrict__ G, long long ldg,
                  int nrows, int nw, z_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (r >= nrows) return;
  const int beg = rowIndex[r], end = rowIndex[r + 1];
  for (int w0 = 0; w0 < nw; w0 += 32) {
    const int w = w0 + lane;
    z_t acc = zmk(0, 0);
    for (int p0 = beg; p0 < end; p0 += 32) {
      const int cnt = min(32, end - p0);
      int myc = 0;
      z_t myv = zmk(0, 0);
      if (lane < cnt) { myc = cols[p0 + lane]; myv = vals[p0 + lane]; }
      for (int q = 0; q < cnt; q++) {
        const int c = __shfl_sync(0xffffffffu, myc, q);
        z_t v;
        v.x = __shfl_sync(0xffffffffu, myv.x, q);
        v.y = __shfl_sync(0xffffffffu, myv.y, q);
        if (w < nw) zfma(acc, v, G[(long long)w * ldg + c]);
      }
    }
    if (w < nw) out[(long long)r * nw + w] = acc;
  }
}

cudaError_t launch_csr_gather(const int* rowIndex, const int* cols, const z_t* vals, const z_t* G,
                              long long ldg, int nrows, int nw, z_t* out, cudaStream_t st) {
  csr_gather_kernel<<<(nrows + 7) / 8, 256, 0, st>>>(rowIndex, cols, vals, G, ldg, nrows, nw, out);
  return cudaGetLastError();
}

// ============================================================ weights
// miniafqmc_base.cpp:316-327; one CTA, fixed-order reduction of sum Re e4.
__global__ void __launch_bounds__(1024)
weights_kernel(z_t* __restrict__ Wd, const z_t* __restrict__ hybridW, int nw, double dt,
               DevScalars* __restrict__ sc, int update_eshift) {
  __shared__ z_t red[32];
  const double eshift = sc->eshift;
  double sum = 0.0;
  for (int w = threadIdx.x; w < nw; w += blockDim.x) {
    z_t* d = Wd + (long long)w * 8;
    z_t ratio = zdiv(zmul(d[2], d[3]), zmul(d[6], d[7]));
    double ang = atan2(ratio.y, ratio.x);
    double scale = fmax(0.0, cos(ang));
    z_t lr = zmk(log(hypot(ratio.x, ratio.y)), ang);
    z_t hw = hybridW[w];
    z_t e4 = zmk(-(hw.x + lr.x) / dt, -(hw.y + lr.y) / dt);
    double f = scale * exp(-dt * (0.5 * (e4.x + d[5].x) - eshift));
    d[4] = e4;
    d[1] = zmk(d[1].x * f, d[1].y * f);
    sum += e4.x;
  }
  z_t t = block_zsum(zmk(sum, 0.0), red);
  if (threadIdx.x == 0) {
    sc->e4sum = t.x;
    if (update_eshift) sc->eshift = t.x / nw;
    sc->step += 1;
  }
}

cudaError_t launch_weights(z_t* Wd, const z_t* hybridW, int nw, double dt, DevScalars* sc,
                           int update_eshift, cudaStream_t st) {
  weights_kernel<<<1, 1024, 0, st>>>(Wd, hybridW, nw, dt, sc, update_eshift);
  return cudaGetLastError();
}

// Sharded substeps: the last weight update's local sum of Re W_data[:,4] into a device
// double, and Eshift = (the ensemble's sum, all-reduced in place by the caller) / walkers
// of the whole ensemble (miniafqmc_base.cpp:327).
__global__ void e4sum_out_kernel(const DevScalars* __restrict__ sc, double* __restrict__ out) {
  *out = sc->e4sum;
}
__global__ void eshift_from_kernel(DevScalars* __restrict__ sc, const double* __restrict__ total,
                                   int nw) {
  const long long ng = sc->nwalk_global > 0 ? sc->nwalk_global : nw;
  sc->eshift = *total / (double)ng;
}
cudaError_t launch_e4sum_out(const DevScalars* sc, double* out, cudaStream_t st) {
  e4sum_out_kernel<<<1, 1, 0, st>>>(sc, out);
  return cudaGetLastError();
}
cudaError_t launch_eshift_from(DevScalars* sc, const double* total, int nw, cudaStream_t st) {
  eshift_from_kernel<<<1, 1, 0, st>>>(sc, total, nw);
  return cudaGetLastError();
}

__global__ void set_scalars_kernel(DevScalars* sc, unsigned long long seed,
                                   unsigned long long step, int set_eshift, double eshift,
                                   int walker_offset, long long nwalk_global) {
  sc->seed = seed;
  sc->step = step;
  if (set_eshift) sc->eshift = eshift;
  if (nwalk_global > 0) {
    sc->walker_offset = walker_offset;
    sc->nwalk_global = nwalk_global;
  }
}

cudaError_t launch_set_scalars(DevScalars* sc, unsigned long long seed, unsigned long long step,
                               int set_eshift, double eshift, cudaStream_t st,
                               int walker_offset, long long nwalk_global) {
  set_scalars_kernel<<<1, 1, 0, st>>>(sc, seed, step, set_eshift, eshift, walker_offset,
                                      nwalk_global);
  return cudaGetLastError();
}

// ============================================================ orthogonalisation
// LQ of W_s seen column-major (zgelqf + zunglq, afqmc_sys.hpp:200-204) is the QR of
// B = conj(W_s) (N x n): Householder reflectors with zlarfg's conventions (real beta
// of sign -sign(Re alpha); tau = (beta - alpha)/beta; v = x/(alpha - beta)), each
// H^H = I - conj(tau) v v^H applied from the left (zgeqr2), then Q = H(1)..H(n) formed
// by backward accumulation (zung2r) and W_s = conj(Q).  One CTA per (walker, spin)
// works in place on the walker buffer (L2 resident); threads are laid out as
// (column, row-group) so row segments are read contiguously.
constexpr int QR_THREADS = 256;

__global__ void __launch_bounds__(QR_THREADS)
ortho_kernel(z_t* __restrict__ W, int N, int n) {
  __shared__ z_t tau_s[64];
  __shared__ z_t sdot[4][65];
  __shared__ z_t red[QR_THREADS / 32];
  __shared__ z_t s_ctau, s_scal;
  __shared__ double s_beta;
  __shared__ int s_skip;
  const int w = blockIdx.x >> 1, s = blockIdx.x & 1;
  const long long ld = 2 * n;
  z_t* B = W + (long long)w * N * ld + s * n;
  const int tid = threadIdx.x;
  const int lc = tid % 64, rg = tid / 64;   // column lane, row group (4 groups)

  for (long long e = tid; e < (long long)N * n; e += QR_THREADS) {
    long long i = e / n, c = e % n;
    z_t v = B[i * ld + c];
    B[i * ld + c] = zconj(v);
  }
  __syncthreads();

  for (int j = 0; j < n; j++) {
    // xnorm^2 over rows j+1..N-1 of column j
    double part = 0.0;
    for (int i = j + 1 + tid; i < N; i += QR_THREADS) {
      z_t v = B[(long long)i * ld + j];
      part += v.x * v.x + v.y * v.y;
    }
    z_t tot = block_zsum(zmk(part, 0.0), red);
    if (tid == 0) {
      z_t alpha = B[(long long)j * ld + j];
      double xn2 = tot.x;
      if (xn2 == 0.0 && alpha.y == 0.0) {
        s_skip = 1;
        tau_s[j] = zmk(0, 0);
      } else {
        double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
        double beta = -copysign(nrm, alpha.x);
        z_t tau = zmk((beta - alpha.x) / beta, -alpha.y / beta);
        tau_s[j] = tau;
        s_ctau = zconj(tau);
        s_scal = zrecip(zmk(alpha.x - beta, alpha.y));
        s_beta = beta;
        s_skip = 0;
      }
    }
    __syncthreads();
    if (s_skip) continue;
    const z_t scal = s_scal;
    for (int i = j + 1 + tid; i < N; i += QR_THREADS) {
      long long o = (long long)i * ld + j;
      B[o] = zmul(B[o], scal);
    }
    __syncthreads();
    if (tid == 0) B[(long long)j * ld + j] = zmk(s_beta, 0.0);
    // s_l = v^H B[j:, l] for l > j (v_j = 1)
    const int l = j + 1 + lc;
    z_t acc = zmk(0, 0);
    if (l < n) {
      if (rg == 0) acc = B[(long long)j * ld + l];
      for (int i = j + 1 + rg; i < N; i += 4)
        zfma_conj(acc, B[(long long)i * ld + j], B[(long long)i * ld + l]);
    }
    sdot[rg][lc] = acc;
    __syncthreads();
    if (rg == 0 && l < n)
      sdot[0][lc] = zadd(zadd(sdot[0][lc], sdot[1][lc]), zadd(sdot[2][lc], sdot[3][lc]));
    __syncthreads();
    if (l < n) {
      const z_t f = zmul(s_ctau, sdot[0][lc]);
      if (rg == 0) {
        long long o = (long long)j * ld + l;
        B[o] = zsub(B[o], f);
      }
      for (int i = j + 1 + rg; i < N; i += 4) {
        long long o = (long long)i * ld + l;
        B[o] = zsub(B[o], zmul(B[(long long)i * ld + j], f));
      }
    }
    __syncthreads();
  }

  // Q = H(1) ... H(n) applied to the first n columns of the identity (zung2r)
  for (int i = n - 1; i >= 0; i--) {
    const z_t tau = tau_s[i];
    if (i < n - 1) {
      const int l = i + 1 + lc;
      z_t acc = zmk(0, 0);
      if (l < n) {
        if (rg == 0) acc = B[(long long)i * ld + l];   // v_i = 1
        for (int r = i + 1 + rg; r < N; r += 4)
          zfma_conj(acc, B[(long long)r * ld + i], B[(long long)r * ld + l]);
      }
      sdot[rg][lc] = acc;
      __syncthreads();
      if (rg == 0 && l < n)
        sdot[0][lc] = zadd(zadd(sdot[0][lc], sdot[1][lc]), zadd(sdot[2][lc], sdot[3][lc]));
      __syncthreads();
      if (l < n) {
        const z_t f = zmul(tau, sdot[0][lc]);
        if (rg == 0) {
          long long o = (long long)i * ld + l;
          B[o] = zsub(B[o], f);
        }
        for (int r = i + 1 + rg; r < N; r += 4) {
          long long o = (long long)r * ld + l;
          B[o] = zsub(B[o], zmul(B[(long long)r * ld + i], f));
        }
      }
      __syncthreads();
    }
    const z_t mt = zmk(-tau.x, -tau.y);
    for (int r = i + 1 + tid; r < N; r += QR_THREADS) {
      long long o = (long long)r * ld + i;
      B[o] = zmul(B[o], mt);
    }
    if (tid == 0) B[(long long)i * ld + i] = zmk(1.0 - tau.x, -tau.y);
    for (int r = tid; r < i; r += QR_THREADS) B[(long long)r * ld + i] = zmk(0, 0);
    __syncthreads();
  }

  for (long long e = tid; e < (long long)N * n; e += QR_THREADS) {
    long long i = e / n, c = e % n;
    z_t v = B[i * ld + c];
    B[i * ld + c] = zconj(v);
  }
}

cudaError_t launch_ortho(z_t* W, int N, int n, int nw, cudaStream_t st) {
  ortho_kernel<<<2 * nw, QR_THREADS, 0, st>>>(W, N, n);
  return cudaGetLastError();
}

// CholeskyQR2 re-orthogonalisation (FP64): G = W_s^H W_s, G = R^H R (R upper, positive
// real diagonal), W_s <- W_s R^-1, done twice.  The columns span the same space as the
// Householder result and differ from it by a diagonal of +-1, so G, overlap ratios,
// weights and energies are unchanged; only raw overlaps may change sign.  One CTA per
// (walker, spin); the n x n factors live in shared memory, W streams through it in
// 32-row chunks.  A walker whose Gram matrix is not positive definite is left as is
// and flagged in info.
// One pass leaves W R^-1 orthonormal to about n eps kappa(W)^2; the second pass is
// skipped when kappa_F = |R|_F |R^-1|_F (>= the 2-norm condition number) is at most 4n,
// i.e. orthonormal to ~1e-11 or better.  Walkers re-orthogonalised every few steps meet
// that bound; a run may force both passes with two_pass = 1.
constexpr int CQ_KC = 32;

size_t cholqr_smem_bytes(int n) {
  return sizeof(z_t) * ((size_t)2 * n * (n + 1) + (size_t)CQ_KC * (n + 1));
}

__global__ void __launch_bounds__(256)
ortho_cholqr_kernel(z_t* __restrict__ W, int N, int n, int* __restrict__ info, int two_pass) {
  extern __shared__ __align__(16) unsigned char cq_smem[];
  const int w = blockIdx.x >> 1, s = blockIdx.x & 1;
  const int ld = n + 1;
  z_t* G = reinterpret_cast<z_t*>(cq_smem);     // Gram matrix, then R
  z_t* Ri = G + n * ld;                          // R^-1
  z_t* buf = Ri + n * ld;                        // W chunk [KC][n+1]
  __shared__ int s_bad;
  __shared__ z_t s_red[32];
  const long long ldw = 2 * n;
  z_t* B = W + (long long)w * N * ldw + s * n;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int R = (n + 15) / 16, ta = tid / 16, tb = tid % 16;   // n <= 64, 256 threads
  if (tid == 0) s_bad = 0;
  for (int pass = 0; pass < 2; pass++) {
    // ---- Gram matrix G[a][b] = sum_k conj(B[k][a]) B[k][b]; thread (ta, tb) of a 16 x 16
    // grid owns a = ta + 16i, b = tb + 16j (i, j < R = ceil(n/16)): R^2 products per 2R
    // shared-memory reads
    {
      z_t acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = zmk(0, 0);
      for (int k0 = 0; k0 < N; k0 += CQ_KC) {
        const int kc = min(CQ_KC, N - k0);
        for (int e = tid; e < kc * n; e += nt) {
          int kk = e / n, a = e % n;
          buf[kk * ld + a] = B[(long long)(k0 + kk) * ldw + a];
        }
        __syncthreads();
        for (int kk = 0; kk < kc; kk++) {
          z_t av[4], bv[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int a = ta + 16 * i, b = tb + 16 * i;
            av[i] = (i < R && a < n) ? buf[kk * ld + a] : zmk(0, 0);
            bv[i] = (i < R && b < n) ? buf[kk * ld + b] : zmk(0, 0);
          }
          // blocks i > j hold only a > b: the lower triangle, which nothing reads
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = i; j < 4; j++)
              if (i < R && j < R) zfma_conj(acc[i][j], av[i], bv[j]);
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = i; j < 4; j++) {
          const int a = ta + 16 * i, b = tb + 16 * j;
          if (i < R && j < R && a < n && b < n) G[a * ld + b] = acc[i][j];
        }
    }
    __syncthreads();
    // ---- Cholesky G = R^H R in place (upper triangle)
    for (int j = 0; j < n; j++) {
      const double dj = G[j * ld + j].x;
      if (!(dj > 0.0)) {
        if (tid == 0) s_bad = 1;
        break;
      }
      const double d = sqrt(dj), inv = 1.0 / d;
      __syncthreads();
      for (int l = j + tid; l < n; l += nt)
        G[j * ld + l] = (l == j) ? zmk(d, 0.0) : zscale(G[j * ld + l], inv);
      __syncthreads();
      const int m = n - j - 1;
      for (int e = tid; e < m * m; e += nt) {
        int a = j + 1 + e / m, b = j + 1 + e % m;
        if (b < a) continue;   // upper triangle only
        z_t t = G[a * ld + b];
        zfma(t, zmk(-G[j * ld + a].x, G[j * ld + a].y), G[j * ld + b]);   // -= conj(R_ja) R_jb
        G[a * ld + b] = t;
      }
      __syncthreads();
    }
    __syncthreads();
    if (s_bad) break;
    // ---- R^-1 (upper) by back substitution, one column per thread
    for (int j = tid; j < n; j += nt) {
      for (int i = n - 1; i >= 0; i--) {
        z_t t = (i == j) ? zmk(1.0, 0.0) : zmk(0.0, 0.0);
        if (i <= j) {
          for (int l = i + 1; l <= j; l++) t = zsub(t, zmul(G[i * ld + l], Ri[l * ld + j]));
          t = zscale(t, 1.0 / G[i * ld + i].x);
        }
        Ri[i * ld + j] = t;
      }
    }
    __syncthreads();
    bool last = pass == 1;
    if (pass == 0 && !two_pass) {   // |R|_F^2 and |R^-1|_F^2 over the upper triangles
      double r2 = 0.0, q2 = 0.0;
      for (int e = tid; e < n * n; e += nt) {
        const int a = e / n, b = e % n;
        if (b < a) continue;
        const z_t g = G[a * ld + b], q = Ri[a * ld + b];
        r2 += g.x * g.x + g.y * g.y;
        q2 += q.x * q.x + q.y * q.y;
      }
      const z_t t = block_zsum(zmk(r2, q2), s_red);
      last = t.x * t.y <= 16.0 * n * n;
    }
    // ---- B <- B R^-1 in 32-row chunks: thread (tk, tb) owns rows k = tk + 16i (i < 2)
    // and columns b = tb + 16j (j < R); R^-1 is upper triangular (zeros below)
    for (int k0 = 0; k0 < N; k0 += CQ_KC) {
      const int kc = min(CQ_KC, N - k0);
      for (int e = tid; e < kc * n; e += nt) {
        int kk = e / n, a = e % n;
        buf[kk * ld + a] = B[(long long)(k0 + kk) * ldw + a];
      }
      __syncthreads();
      z_t acc[2][4];
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = zmk(0, 0);
      // R^-1 is upper triangular: rows a in [16r, 16r + 16) reach columns b = tb + 16j
      // only for j >= r
#pragma unroll
      for (int r = 0; r < 4; r++) {
        if (r >= R) break;
        const int a1 = min(16 * r + 16, n);
        for (int a = 16 * r; a < a1; a++) {
          z_t bv[2], rv[4];
#pragma unroll
          for (int i = 0; i < 2; i++) bv[i] = buf[(ta + 16 * i) * ld + a];
#pragma unroll
          for (int j = r; j < 4; j++) {
            const int b = tb + 16 * j;
            rv[j] = (j < R && b < n) ? Ri[a * ld + b] : zmk(0, 0);
          }
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = r; j < 4; j++)
              if (j < R) zfma(acc[i][j], bv[i], rv[j]);
        }
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int kk = ta + 16 * i, b = tb + 16 * j;
          if (j < R && kk < kc && b < n) B[(long long)(k0 + kk) * ldw + b] = acc[i][j];
        }
      __syncthreads();
    }
    if (last) break;
  }
  if (tid == 0) info[w * 2 + s] |= s_bad ? 2 : 0;
}

cudaError_t launch_ortho_cholqr(z_t* W, int N, int n, int nw, int* info, cudaStream_t st) {
  if (n > 64) return cudaErrorInvalidValue;   // the register tiles cover n <= 64
  size_t smem = cholqr_smem_bytes(n);
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(smem, [](size_t b) {
    cudaError_t r = cudaFuncSetAttribute(ortho_cholqr_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
    if (r == cudaSuccess)
      r = cudaFuncSetAttribute(ortho_cholqr_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    return r;
  });
  if (e != cudaSuccess) return e;
  static const int two_pass = [] {
    const char* e = getenv("AFQ_CHOLQR_PASSES");
    return e && atoi(e) == 2 ? 1 : 0;
  }();
  ortho_cholqr_kernel<<<2 * nw, 256, smem, st>>>(W, N, n, info, two_pass);
  return cudaGetLastError();
}

// ============================================================ exchange energy
// K_w = 1/2 sum_{s,c} tr(T T), T = Lh_s[c] Gc_s^T (n x n), for Gn Cholesky vectors x Gw
// walkers per CTA: a (Gn*n) x (Gw*n) complex tile over K = N, then the trace of each
// n x n block squared from shared memory.  Partial sums per (walker, spin, c-block).
constexpr int EX_T = 96, EX_BK = 16, EX_TM = 6, EX_TN = 6, EX_THREADS = 256;

size_t exch_smem_bytes() {
  size_t main = sizeof(z_t) * 2 * EX_BK * 2 * (EX_T + 1);
  size_t epi = sizeof(z_t) * EX_T * (EX_T + 1);
  return std::max(main, epi);
}

__global__ void __launch_bounds__(EX_THREADS)
exchange_kernel(const z_t* __restrict__ Lh, const z_t* __restrict__ Gc, int N, int n, int nchol,
                int nw, int Gn, int Gw, z_t* __restrict__ Kpart, int nblk) {
  extern __shared__ __align__(16) unsigned char ex_smem[];
  z_t* As = reinterpret_cast<z_t*>(ex_smem);          // [2][BK][T+1]
  z_t* Bs = As + 2 * EX_BK * (EX_T + 1);
  const int s = blockIdx.z;
  const int c0 = blockIdx.x * Gn, w0 = blockIdx.y * Gw;
  const long long NAK = 2LL * n * N;
  const int Mr = Gn * n, Nc = Gw * n;
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;

  auto load = [&](int stage, int k0) {
    z_t* as = As + stage * EX_BK * (EX_T + 1);
    z_t* bs = Bs + stage * EX_BK * (EX_T + 1);
    for (int e = tid; e < EX_T * EX_BK; e += EX_THREADS) {
      int m = e / EX_BK, k = e % EX_BK, gk = k0 + k;
      int cv = m / n, a = m % n;
      const z_t* src = Lh;
      int bytes = 0;
      if (m < Mr && c0 + cv < nchol && gk < N) {
        src = Lh + (long long)(c0 + cv) * NAK + (long long)s * n * N + (long long)a * N + gk;
        bytes = 16;
      }
      cp_async16(as + k * (EX_T + 1) + m, src, bytes);
      const z_t* srcb = Gc;
      int bb = 0;
      if (m < Nc && w0 + m / n < nw && gk < N) {
        int wl = m / n, b = m % n;
        srcb = Gc + (long long)(w0 + wl) * NAK + (long long)s * n * N + (long long)b * N + gk;
        bb = 16;
      }
      cp_async16(bs + k * (EX_T + 1) + m, srcb, bb);
    }
    cp_async_commit();
  };

  z_t acc[EX_TM][EX_TN];
#pragma unroll
  for (int i = 0; i < EX_TM; i++)
#pragma unroll
    for (int j = 0; j < EX_TN; j++) acc[i][j] = zmk(0, 0);
  const int nk = (N + EX_BK - 1) / EX_BK;
  load(0, 0);
  for (int kt = 0; kt < nk; kt++) {
    if (kt + 1 < nk) {
      load((kt + 1) & 1, (kt + 1) * EX_BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const z_t* as = As + (kt & 1) * EX_BK * (EX_T + 1);
    const z_t* bs = Bs + (kt & 1) * EX_BK * (EX_T + 1);
#pragma unroll 4
    for (int kk = 0; kk < EX_BK; kk++) {
      z_t a[EX_TM], b[EX_TN];
#pragma unroll
      for (int i = 0; i < EX_TM; i++) a[i] = as[kk * (EX_T + 1) + ty + 16 * i];
#pragma unroll
      for (int j = 0; j < EX_TN; j++) b[j] = bs[kk * (EX_T + 1) + tx + 16 * j];
#pragma unroll
      for (int i = 0; i < EX_TM; i++)
#pragma unroll
        for (int j = 0; j < EX_TN; j++) zfma(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  z_t* Ts = reinterpret_cast<z_t*>(ex_smem);             // [T][T+1], reuses the slabs
#pragma unroll
  for (int i = 0; i < EX_TM; i++)
#pragma unroll
    for (int j = 0; j < EX_TN; j++) Ts[(ty + 16 * i) * (EX_T + 1) + tx + 16 * j] = acc[i][j];
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  for (int wl = warp; wl < Gw; wl += EX_THREADS / 32) {
    z_t sum = zmk(0, 0);
    for (int cv = 0; cv < Gn; cv++)
      for (int t = lane; t < n * n; t += 32) {
        int a = t / n, b = t % n;
        zfma(sum, Ts[(cv * n + a) * (EX_T + 1) + wl * n + b], Ts[(cv * n + b) * (EX_T + 1) + wl * n + a]);
      }
    sum = warp_zsum(sum);
    if (lane == 0 && w0 + wl < nw) Kpart[((long long)(w0 + wl) * 2 + s) * nblk + blockIdx.x] = sum;
  }
}

cudaError_t launch_exchange(const z_t* Lh, const z_t* Gc, int N, int n, int nchol, int nw,
                            z_t* Kpart, int* nblk_out, cudaStream_t st) {
  if (n > EX_T) return cudaErrorInvalidValue;
  const int Gn = EX_T / n, Gw = EX_T / n;
  const int nblk = (nchol + Gn - 1) / Gn;
  *nblk_out = nblk;
  if (!Kpart) return cudaSuccess;
  size_t smem = exch_smem_bytes();
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(smem, [](size_t b) {
    return cudaFuncSetAttribute(exchange_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)b);
  });
  if (e != cudaSuccess) return e;
  dim3 grid(nblk, (nw + Gw - 1) / Gw, 2);
  exchange_kernel<<<grid, EX_THREADS, smem, st>>>(Lh, Gc, N, n, nchol, nw, Gn, Gw, Kpart, nblk);
  return cudaGetLastError();
}

// ============================================================ energy reductions
// Per walker: E1 = sum Gc.haj (energy.hpp:100); mode 0 (Vakbl): E2 = 1/2 sum Gc.Gcloc
// (energy.hpp:93-97); mode 1 (Cholesky): EJ = 1/2 sum_c cv^2, EK = 1/2 sum Kpart.
__global__ void __launch_bounds__(256)
energy_reduce_kernel(const z_t* __restrict__ Gc, const z_t* __restrict__ haj, int nak,
                     const z_t* __restrict__ Gcloc, const z_t* __restrict__ cv, int nchol,
                     const z_t* __restrict__ Kpart, int nblk, int nw, int mode,
                     z_t* __restrict__ Wd, double* __restrict__ parts) {
  __shared__ z_t red[8];
  const int w = blockIdx.x;
  const z_t* g = Gc + (long long)w * nak;
  z_t e1 = zmk(0, 0), e2 = zmk(0, 0);
  for (int i = threadIdx.x; i < nak; i += blockDim.x) {
    z_t gi = g[i];
    zfma(e1, gi, haj[i]);
    if (mode == 0) zfma(e2, gi, Gcloc[(long long)i * nw + w]);
  }
  e1 = block_zsum(e1, red);
  z_t ej = zmk(0, 0), ek = zmk(0, 0);
  if (mode == 0) {
    e2 = block_zsum(e2, red);
  } else {
    for (int c = threadIdx.x; c < nchol; c += blockDim.x) {
      z_t v = cv[(long long)c * nw + w];
      zfma(ej, v, v);
    }
    for (int q = threadIdx.x; q < 2 * nblk; q += blockDim.x)
      ek = zadd(ek, Kpart[(long long)w * 2 * nblk + q]);
    ej = block_zsum(ej, red);
    ek = block_zsum(ek, red);
  }
  if (threadIdx.x == 0) {
    z_t e;
    if (mode == 0) {
      e = zadd(zscale(e2, 0.5), e1);
    } else {
      ej = zscale(ej, 0.5);
      ek = zscale(ek, 0.5);
      e = zsub(zadd(e1, ej), ek);
      if (parts) {
        parts[3 * w] = e1.x; parts[3 * w + 1] = ej.x; parts[3 * w + 2] = ek.x;
      }
    }
    Wd[(long long)w * 8] = e;
  }
}

cudaError_t launch_energy_reduce(const z_t* Gc, const z_t* haj, int nak, const z_t* Gcloc,
                                 const z_t* cv, int nchol, const z_t* Kpart, int nblk, int nw,
                                 int mode, z_t* Wd, double* parts, cudaStream_t st) {
  energy_reduce_kernel<<<nw, 256, 0, st>>>(Gc, haj, nak, Gcloc, cv, nchol, Kpart, nblk, nw, mode,
                                           Wd, parts);
  return cudaGetLastError();
}

// sum Re(eloc) Re(w) and sum Re(w) (afqmc_sys.hpp:127-132), fixed-order reduction.
__global__ void __launch_bounds__(1024)
eav_kernel(const z_t* __restrict__ Wd, int nw, DevScalars* __restrict__ sc) {
  __shared__ z_t red[32];
  double a = 0.0, b = 0.0;
  for (int w = threadIdx.x; w < nw; w += blockDim.x) {
    const z_t* d = Wd + (long long)w * 8;
    a += d[0].x * d[1].x;
    b += d[1].x;
  }
  z_t t = block_zsum(zmk(a, b), red);
  if (threadIdx.x == 0) {
    sc->esum[0] = t.x;
    sc->esum[1] = t.y;
  }
}

cudaError_t launch_eav(const z_t* Wd, int nw, DevScalars* sc, cudaStream_t st) {
  eav_kernel<<<1, 1024, 0, st>>>(Wd, nw, sc);
  return cudaGetLastError();
}

}  // namespace afq
