// FP64 CPU oracle for the miniAFQMC walker hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++, the algorithm of the
// reference miniapp (QMCPACK miniAFQMC) for one walker ensemble, with the reference's
// call granularity: a per-walker loop of small zgemm / zgetrf / zgetri / zgelqf / zunglq
// calls and the serial CSR x dense loop of `mySPBLAS::csrmm`.  The GPU library's tests
// compare against it and the bench times it as the CPU baseline; nothing in the product
// links or calls it.
//
// BLAS/LAPACK are not part of the reference tree (it links any Fortran LAPACK,
// `CMakeLists.txt:432-456`).  The oracle calls the LAPACK routines the reference calls,
// through Fortran-ABI function pointers handed in by the caller (scipy's bundled
// OpenBLAS in the Python wrapper), so pivoting and Householder conventions are
// LAPACK's own.
//
// Layouts are the reference's (miniafqmc_base.cpp:213-224):
//   W[nw][2][N][n], W_data[nw][8], Gc[2][n][N][nw] (walker fastest), vbias[nchol][nw],
//   X[nchol][nw], vHS[N*N][nw], hybridW[nw].
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

extern "C" {
typedef void (*zgemm_t)(const char*, const char*, const int*, const int*, const int*,
                        const cd*, const cd*, const int*, const cd*, const int*,
                        const cd*, cd*, const int*);
typedef void (*zgemv_t)(const char*, const int*, const int*, const cd*, const cd*,
                        const int*, const cd*, const int*, const cd*, cd*, const int*);
typedef void (*zgetrf_t)(const int*, const int*, cd*, const int*, int*, int*);
typedef void (*zgetri_t)(const int*, cd*, const int*, const int*, cd*, const int*, int*);
typedef void (*zgelqf_t)(const int*, const int*, cd*, const int*, cd*, cd*, const int*, int*);
typedef void (*zunglq_t)(const int*, const int*, const int*, cd*, const int*, const cd*,
                         cd*, const int*, int*);
}

namespace {

struct Lapack {
  zgemm_t zgemm = nullptr;
  zgemv_t zgemv = nullptr;
  zgetrf_t zgetrf = nullptr;
  zgetri_t zgetri = nullptr;
  zgelqf_t zgelqf = nullptr;
  zunglq_t zunglq = nullptr;
};
Lapack g_lapack;

struct CSR {
  int nrows = 0, ncols = 0;
  std::vector<int> rowIndex, cols;
  std::vector<cd> vals;
  bool empty() const { return nrows == 0; }
};

// Row-major C[M][Nc] = alpha * op(A) * op(B) + beta * C, expressed the way
// `ma::product` maps row-major arrays onto column-major gemm by swapping operands
// (ma_operations.hpp:101-107 -> ma_blas.hpp:79-121).  opA/opB are 'N' or 'T';
// lda/ldb are the row strides of A and B as stored.
void rm_gemm(char opA, char opB, int M, int Nc, int K, cd alpha, const cd* A, int lda,
             const cd* B, int ldb, cd beta, cd* C, int ldc) {
  g_lapack.zgemm(&opB, &opA, &Nc, &M, &K, &alpha, B, &ldb, A, &lda, &beta, C, &ldc);
}

// Serial CSR x dense product, 'N' branch of mySPBLAS::csrmm (sparse.hpp:166-180):
// C[r][:] = beta*C[r][:] + sum_{nz in row r} alpha*A[nz] * B[col][:].
void csrmm_N(const CSR& A, int ncolsB, cd alpha, const cd* B, int ldb, cd beta, cd* C,
             int ldc) {
  for (int r = 0; r < A.nrows; r++) {
    cd* Cr = C + (size_t)r * ldc;
    for (int i = 0; i < ncolsB; i++) Cr[i] *= beta;
    for (int p = A.rowIndex[r]; p < A.rowIndex[r + 1]; p++) {
      int c = A.cols[p];
      if (c >= A.ncols) continue;
      const cd* Bc = B + (size_t)c * ldb;
      cd Arc = alpha * A.vals[p];
      for (int k = 0; k < ncolsB; k++) Cr[k] += Arc * Bc[k];
    }
  }
}

// Row-parallel variant with the same per-row arithmetic order (each row is owned by one
// thread, so results are identical to csrmm_N for any thread count).
void csrmm_N_par(const CSR& A, int ncolsB, cd alpha, const cd* B, int ldb, cd beta,
                 cd* C, int ldc) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int r = 0; r < A.nrows; r++) {
    cd* Cr = C + (size_t)r * ldc;
    for (int i = 0; i < ncolsB; i++) Cr[i] *= beta;
    for (int p = A.rowIndex[r]; p < A.rowIndex[r + 1]; p++) {
      int c = A.cols[p];
      if (c >= A.ncols) continue;
      const cd* Bc = B + (size_t)c * ldb;
      cd Arc = alpha * A.vals[p];
      for (int k = 0; k < ncolsB; k++) Cr[k] += Arc * Bc[k];
    }
  }
}

// 'T' branch of mySPBLAS::csrmm (sparse.hpp:181-197): C[col][:] += alpha*A[nz]*B[r][:].
void csrmm_T(const CSR& A, int ncolsB, cd alpha, const cd* B, int ldb, cd beta, cd* C,
             int ldc) {
  for (int i = 0; i < A.ncols; i++)
    for (int j = 0; j < ncolsB; j++) C[(size_t)i * ldc + j] *= beta;
  for (int r = 0; r < A.nrows; r++) {
    const cd* Br = B + (size_t)r * ldb;
    for (int p = A.rowIndex[r]; p < A.rowIndex[r + 1]; p++) {
      int c = A.cols[p];
      if (c >= A.ncols) continue;
      cd* Cc = C + (size_t)c * ldc;
      cd Arc = alpha * A.vals[p];
      for (int k = 0; k < ncolsB; k++) Cc[k] += Arc * Br[k];
    }
  }
}

// ---------------------------------------------------------------- Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror and Shaw (SC'11), restated.
inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * ctr[0];
    uint64_t p1 = (uint64_t)M1 * ctr[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ ctr[1] ^ k0, n2 = hi0 ^ ctr[3] ^ k1;
    ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
    k0 += W0; k1 += W1;
  }
}

// Two N(0,1) numbers for pair index j of step `step` (Box-Muller on 53-bit uniforms).
// The same function is implemented on the device; x is real, as the reference's
// BoxMuller2 writes real normals into its complex buffer (RandomGenerator.h:81-95).
inline void normal_pair(uint64_t seed, uint64_t step, uint64_t j, double* x0, double* x1) {
  uint32_t c[4] = {(uint32_t)j, (uint32_t)(j >> 32), (uint32_t)step, (uint32_t)(step >> 32)};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double s53 = 1.0 / 9007199254740992.0;  // 2^-53
  double u1 = ((double)(((uint64_t)(c[0] >> 5) << 26) | (c[1] >> 6)) + 1.0) * s53;  // (0,1]
  double u2 = (double)(((uint64_t)(c[2] >> 5) << 26) | (c[3] >> 6)) * s53;          // [0,1)
  double r = std::sqrt(-2.0 * std::log(u1));
  double th = 6.283185307179586 * u2;
  *x0 = r * std::cos(th);
  *x1 = r * std::sin(th);
}

}  // namespace

struct orc_handle {
  int N = 0, n = 0, nchol = 0, nw = 0, order = 6;
  double dt = 0.01;
  CSR Spvn, SpvnT, Vakbl;
  std::vector<cd> P, haj, trial[2], Lh;
  std::vector<cd> W, Wd, Gc, vbias, X, vHS, hybridW;
  std::vector<cd> G;         // full density matrix [2][N][N][nw] (transposed_Spvn == false)
  std::vector<double> xraw;
  std::vector<int> info;
  double Eshift = 0.0;
  int nthreads = 1;
  int walker_offset = 0;     // global index of walker 0 (sharded ensembles)
  long long nwalk_global = 0;
};

extern "C" {

int orc_set_lapack(void* zgemm, void* zgemv, void* zgetrf, void* zgetri, void* zgelqf,
                   void* zunglq) {
  g_lapack.zgemm = (zgemm_t)zgemm;
  g_lapack.zgemv = (zgemv_t)zgemv;
  g_lapack.zgetrf = (zgetrf_t)zgetrf;
  g_lapack.zgetri = (zgetri_t)zgetri;
  g_lapack.zgelqf = (zgelqf_t)zgelqf;
  g_lapack.zunglq = (zunglq_t)zunglq;
  return (zgemm && zgemv && zgetrf && zgetri && zgelqf && zunglq) ? 0 : 1;
}

orc_handle* orc_create(int nmo, int naea, int nchol, int nwalk, double dt, int order) {
  orc_handle* h = new orc_handle();
  h->N = nmo; h->n = naea; h->nchol = nchol; h->nw = nwalk; h->dt = dt; h->order = order;
  size_t NAK = 2ull * naea * nmo;
  h->W.assign((size_t)nwalk * 2 * nmo * naea, cd(0));
  h->Wd.assign((size_t)nwalk * 8, cd(0));
  h->Gc.assign(NAK * nwalk, cd(0));
  h->vbias.assign((size_t)nchol * nwalk, cd(0));
  h->X.assign((size_t)nchol * nwalk, cd(0));
  h->xraw.assign((size_t)nchol * nwalk, 0.0);
  h->vHS.assign((size_t)nmo * nmo * nwalk, cd(0));
  h->hybridW.assign(nwalk, cd(0));
  h->info.assign((size_t)nwalk * 2, 0);
  return h;
}

void orc_destroy(orc_handle* h) { delete h; }

void orc_set_threads(orc_handle* h, int nthreads) {
  h->nthreads = nthreads < 1 ? 1 : nthreads;
#ifdef _OPENMP
  omp_set_num_threads(h->nthreads);
#endif
}

static void load_csr(CSR& A, int nrows, int ncols, const int* rowIndex, const int* cols,
                     const double* vals) {
  A.nrows = nrows; A.ncols = ncols;
  A.rowIndex.assign(rowIndex, rowIndex + nrows + 1);
  long long nnz = rowIndex[nrows];
  A.cols.assign(cols, cols + nnz);
  A.vals.resize(nnz);
  std::memcpy(A.vals.data(), vals, sizeof(cd) * nnz);
}

void orc_set_spvn(orc_handle* h, int nrows, int ncols, const int* ri, const int* c,
                  const double* v) { load_csr(h->Spvn, nrows, ncols, ri, c, v); }
void orc_set_spvnT(orc_handle* h, int nrows, int ncols, const int* ri, const int* c,
                   const double* v) { load_csr(h->SpvnT, nrows, ncols, ri, c, v); }
void orc_set_vakbl(orc_handle* h, int nrows, int ncols, const int* ri, const int* c,
                   const double* v) { load_csr(h->Vakbl, nrows, ncols, ri, c, v); }

// Propg1[N][N], haj[2n][N], trial[2][N][n] (= conj(Wavefun)), Lh[nchol][2][n][N] or null.
void orc_set_dense(orc_handle* h, const double* P, const double* haj, const double* trial,
                   const double* Lh) {
  size_t N = h->N, n = h->n;
  h->P.assign((const cd*)P, (const cd*)P + N * N);
  h->haj.assign((const cd*)haj, (const cd*)haj + 2 * n * N);
  h->trial[0].assign((const cd*)trial, (const cd*)trial + N * n);
  h->trial[1].assign((const cd*)trial + N * n, (const cd*)trial + 2 * N * n);
  if (Lh) h->Lh.assign((const cd*)Lh, (const cd*)Lh + (size_t)h->nchol * 2 * n * N);
  else h->Lh.clear();
}

void orc_set_walkers(orc_handle* h, const double* W, const double* Wd) {
  std::memcpy(h->W.data(), W, sizeof(cd) * h->W.size());
  std::memcpy(h->Wd.data(), Wd, sizeof(cd) * h->Wd.size());
}
void orc_get_walkers(const orc_handle* h, double* W, double* Wd) {
  if (W) std::memcpy(W, h->W.data(), sizeof(cd) * h->W.size());
  if (Wd) std::memcpy(Wd, h->Wd.data(), sizeof(cd) * h->Wd.size());
}

// which: 0 Gc, 1 vbias, 2 X, 3 vHS, 4 hybridW, 5 xraw (double), 6 info (int)
void orc_copy_out(const orc_handle* h, int which, void* dst) {
  switch (which) {
    case 0: std::memcpy(dst, h->Gc.data(), sizeof(cd) * h->Gc.size()); break;
    case 1: std::memcpy(dst, h->vbias.data(), sizeof(cd) * h->vbias.size()); break;
    case 2: std::memcpy(dst, h->X.data(), sizeof(cd) * h->X.size()); break;
    case 3: std::memcpy(dst, h->vHS.data(), sizeof(cd) * h->vHS.size()); break;
    case 4: std::memcpy(dst, h->hybridW.data(), sizeof(cd) * h->hybridW.size()); break;
    case 5: std::memcpy(dst, h->xraw.data(), sizeof(double) * h->xraw.size()); break;
    case 6: std::memcpy(dst, h->info.data(), sizeof(int) * h->info.size()); break;
    case 7: std::memcpy(dst, h->G.data(), sizeof(cd) * h->G.size()); break;
  }
}

double orc_get_eshift(const orc_handle* h) { return h->Eshift; }
void orc_set_eshift(orc_handle* h, double e) { h->Eshift = e; }

// ma::invert (ma_operations.hpp:244-260): getrf, det from the pivots, getri.
// Returns det; *info != 0 when getrf found an exactly singular pivot.
static cd invert(cd* T1, int n, int* ipiv, cd* work, int lwork, int* info) {
  g_lapack.zgetrf(&n, &n, T1, &n, ipiv, info);
  cd det(1.0);
  for (int i = 0; i < n; i++) det *= (ipiv[i] == i + 1) ? T1[i * n + i] : -T1[i * n + i];
  if (*info == 0) {
    int inf2 = 0;
    g_lapack.zgetri(&n, T1, &n, ipiv, work, &lwork, &inf2);
  }
  return det;
}

// ma::determinant (ma_operations.hpp:276-291).
static cd determinant(cd* T1, int n, int* ipiv, int* info) {
  g_lapack.zgetrf(&n, &n, T1, &n, ipiv, info);
  cd det(1.0);
  for (int i = 0; i < n; i++) det *= (ipiv[i] == i + 1) ? T1[i * n + i] : -T1[i * n + i];
  return det;
}

// afqmc_sys::calculate_mixed_density_matrix (afqmc_sys.hpp:98-116) with compact=true,
// base::MixedDensityMatrix (mixed_density_matrix.hpp:63-104).
void orc_mixed_density_matrix(orc_handle* h) {
  const int N = h->N, n = h->n, nw = h->nw;
#pragma omp parallel
  {
    std::vector<cd> T1((size_t)n * n), DM((size_t)n * N), work((size_t)64 * n);
    std::vector<int> ipiv(n);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nw; w++) {
      for (int s = 0; s < 2; s++) {
        const cd* Ws = h->W.data() + ((size_t)w * 2 + s) * N * n;
        // T1 = T(W) * conj(A)   (mixed_density_matrix.hpp:83)
        rm_gemm('T', 'N', n, n, N, cd(1), Ws, n, h->trial[s].data(), n, cd(0), T1.data(), n);
        int info = 0;
        cd ov = invert(T1.data(), n, ipiv.data(), work.data(), (int)work.size(), &info);
        h->info[(size_t)w * 2 + s] = info;
        // C = T1 * T(W)          (mixed_density_matrix.hpp:91)
        rm_gemm('N', 'T', n, N, n, cd(1), T1.data(), n, Ws, n, cd(0), DM.data(), N);
        h->Wd[(size_t)w * 8 + 2 + s] = ov;
        // G_4D[s][a][k][w] = DM[a][k]   (afqmc_sys.hpp:110,114)
        for (int a = 0; a < n; a++)
          for (int k = 0; k < N; k++)
            h->Gc[(((size_t)s * n + a) * N + k) * nw + w] = DM[(size_t)a * N + k];
      }
    }
  }
}

// afqmc_sys::calculate_mixed_density_matrix with compact=false (afqmc_sys.hpp:98-116),
// the non-compact branch of base::MixedDensityMatrix (mixed_density_matrix.hpp:96-99):
// T2 = T1^-1 T(W), C = conj(A) T2, stored as G_4D[s][i][k][w] with N_ = NMO.
void orc_mixed_density_matrix_full(orc_handle* h) {
  const int N = h->N, n = h->n, nw = h->nw;
  h->G.assign((size_t)2 * N * N * nw, cd(0));
#pragma omp parallel
  {
    std::vector<cd> T1((size_t)n * n), T2((size_t)n * N), DM((size_t)N * N),
        work((size_t)64 * n);
    std::vector<int> ipiv(n);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nw; w++) {
      for (int s = 0; s < 2; s++) {
        const cd* Ws = h->W.data() + ((size_t)w * 2 + s) * N * n;
        rm_gemm('T', 'N', n, n, N, cd(1), Ws, n, h->trial[s].data(), n, cd(0), T1.data(), n);
        int info = 0;
        cd ov = invert(T1.data(), n, ipiv.data(), work.data(), (int)work.size(), &info);
        h->info[(size_t)w * 2 + s] = info;
        rm_gemm('N', 'T', n, N, n, cd(1), T1.data(), n, Ws, n, cd(0), T2.data(), N);
        rm_gemm('N', 'N', N, N, n, cd(1), h->trial[s].data(), n, T2.data(), N, cd(0), DM.data(), N);
        h->Wd[(size_t)w * 8 + 2 + s] = ov;
        for (int i = 0; i < N; i++)
          for (int k = 0; k < N; k++)
            h->G[(((size_t)s * N + i) * N + k) * nw + w] = DM[(size_t)i * N + k];
      }
    }
  }
}

// base::get_vbias(Spvn, G, vbias, false) (vbias.hpp:66-81): vbias = T(Spvn) G_alpha, then
// vbias += T(Spvn) G_beta.
void orc_vbias_full(orc_handle* h) {
  const size_t half = (size_t)h->N * h->N * h->nw;
  csrmm_T(h->Spvn, h->nw, cd(1), h->G.data(), h->nw, cd(0), h->vbias.data(), h->nw);
  csrmm_T(h->Spvn, h->nw, cd(1), h->G.data() + half, h->nw, cd(1), h->vbias.data(), h->nw);
}

// afqmc_sys::calculate_overlaps (afqmc_sys.hpp:136-144), base::Overlap
// (mixed_density_matrix.hpp:124-138).  save_old=1 first performs the driver's
// W_data[5,6,7] <- W_data[4,2,3] shuffle (miniafqmc_base.cpp:305-309).
void orc_overlaps(orc_handle* h, int save_old) {
  const int N = h->N, n = h->n, nw = h->nw;
  if (save_old)
    for (int w = 0; w < nw; w++) {
      cd* d = h->Wd.data() + (size_t)w * 8;
      d[5] = d[4]; d[6] = d[2]; d[7] = d[3];
    }
#pragma omp parallel
  {
    std::vector<cd> T1((size_t)n * n);
    std::vector<int> ipiv(n);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nw; w++)
      for (int s = 0; s < 2; s++) {
        const cd* Ws = h->W.data() + ((size_t)w * 2 + s) * N * n;
        rm_gemm('T', 'N', n, n, N, cd(1), Ws, n, h->trial[s].data(), n, cd(0), T1.data(), n);
        int info = 0;
        h->Wd[(size_t)w * 8 + 2 + s] = determinant(T1.data(), n, ipiv.data(), &info);
        h->info[(size_t)w * 2 + s] = info;
      }
  }
}

// base::get_vbias(SpvnT, Gc, vbias, true) (vbias.hpp:56-63): vbias = SpvnT * Gc.
void orc_vbias(orc_handle* h) {
  if (h->nthreads > 1)
    csrmm_N_par(h->SpvnT, h->nw, cd(1), h->Gc.data(), h->nw, cd(0), h->vbias.data(), h->nw);
  else
    csrmm_N(h->SpvnT, h->nw, cd(1), h->Gc.data(), h->nw, cd(0), h->vbias.data(), h->nw);
}

// Driver step 2 (miniafqmc_base.cpp:281-289): X = x + i vbias, hybridW.
// use_given=1 takes x from xraw (set by orc_set_xraw) instead of the generator.
static void sigma_core(orc_handle* h) {
  const int nc = h->nchol, nw = h->nw;
  const cd im(0.0, 1.0), halfim(0.0, 0.5);
  for (int w = 0; w < nw; w++) h->hybridW[w] = cd(0.);
  for (int c = 0; c < nc; c++)
    for (int w = 0; w < nw; w++) {
      size_t i = (size_t)c * nw + w;
      cd x(h->xraw[i], 0.0);
      cd vb = h->vbias[i];
      h->hybridW[w] -= im * vb * (x + halfim * vb);
      h->X[i] = x + im * vb;
    }
}

// x[c][w] is element c*nwg + woff + w of one stream over the global ensemble, so a
// sharded ensemble draws the same fields as the unsharded one.
void orc_generate_x(orc_handle* h, uint64_t seed, uint64_t step) {
  const long long nwg = h->nwalk_global > 0 ? h->nwalk_global : h->nw;
  for (int c = 0; c < h->nchol; c++)
    for (int w = 0; w < h->nw; w++) {
      long long eg = (long long)c * nwg + h->walker_offset + w;
      double a, b;
      normal_pair(seed, step, (uint64_t)eg >> 1, &a, &b);
      h->xraw[(size_t)c * h->nw + w] = (eg & 1) ? b : a;
    }
}

void orc_set_walker_offset(orc_handle* h, int offset, long long nwalk_global) {
  h->walker_offset = offset;
  h->nwalk_global = nwalk_global;
}

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; i++) out[i] = c[i];
}

void orc_sigma(orc_handle* h, uint64_t seed, uint64_t step) {
  orc_generate_x(h, seed, step);
  sigma_core(h);
}

void orc_sigma_from(orc_handle* h, const double* x) {
  std::memcpy(h->xraw.data(), x, sizeof(double) * h->xraw.size());
  sigma_core(h);
}

// base::get_vHS (vHS.hpp:47-56): vHS = Spvn * X.
void orc_vhs(orc_handle* h) {
  if (h->nthreads > 1)
    csrmm_N_par(h->Spvn, h->nw, cd(1), h->X.data(), h->nw, cd(0), h->vHS.data(), h->nw);
  else
    csrmm_N(h->Spvn, h->nw, cd(1), h->X.data(), h->nw, cd(0), h->vHS.data(), h->nw);
}

// base::apply_expM (vHS.hpp:65-90): S <- sum_{k<=order} (iV)^k/k! S.
static void apply_expM(const cd* V, cd* S, cd* T1, cd* T2, int N, int n, int order) {
  std::memcpy(T1, S, sizeof(cd) * N * n);
  for (int k = 1; k <= order; k++) {
    cd fact = cd(0.0, 1.0) * cd(1.0 / (double)k);
    rm_gemm('N', 'N', N, n, N, fact, V, N, T1, n, cd(0), T2, n);
    for (size_t i = 0; i < (size_t)N * n; i++) S[i] += T2[i];
    std::swap(T1, T2);
  }
}

// afqmc_sys::propagate (afqmc_sys.hpp:150-173).
void orc_propagate(orc_handle* h) {
  const int N = h->N, n = h->n, nw = h->nw;
#pragma omp parallel
  {
    std::vector<cd> MM((size_t)N * N), MN((size_t)N * n), T1((size_t)N * n), T2((size_t)N * n);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nw; w++) {
      for (size_t ik = 0; ik < (size_t)N * N; ik++) MM[ik] = h->vHS[ik * nw + w];
      for (int s = 0; s < 2; s++) {
        cd* Ws = h->W.data() + ((size_t)w * 2 + s) * N * n;
        rm_gemm('N', 'N', N, n, N, cd(1), h->P.data(), N, Ws, n, cd(0), MN.data(), n);
        apply_expM(MM.data(), MN.data(), T1.data(), T2.data(), N, n, h->order);
        rm_gemm('N', 'N', N, n, N, cd(1), h->P.data(), N, MN.data(), n, cd(0), Ws, n);
      }
    }
  }
}

// Driver step 6 (miniafqmc_base.cpp:316-327).
void orc_update_weights(orc_handle* h) {
  double et = 0.0;
  const double dt = h->dt;
  for (int w = 0; w < h->nw; w++) {
    cd* d = h->Wd.data() + (size_t)w * 8;
    cd ratio = d[2] * d[3] / (d[6] * d[7]);
    double scale = std::max(0.0, std::cos(std::arg(ratio)));
    d[4] = -(h->hybridW[w] + std::log(ratio)) / dt;
    d[1] *= cd(scale * std::exp(-dt * (0.5 * (d[4].real() + d[5].real()) - h->Eshift)), 0.0);
    et += d[4].real();
  }
  h->Eshift = et / h->nw;
}

// Partial sum of Re W_data[4] without touching Eshift (used by the sharded driver).
double orc_sum_e4(const orc_handle* h) {
  double et = 0.0;
  for (int w = 0; w < h->nw; w++) et += h->Wd[(size_t)w * 8 + 4].real();
  return et;
}

// afqmc_sys::orthogonalize (afqmc_sys.hpp:176-207): LQ of each W[w][s] viewed
// column-major (zgelqf + zunglq).
void orc_orthogonalize(orc_handle* h) {
  const int N = h->N, n = h->n, nw = h->nw;
#pragma omp parallel
  {
    std::vector<cd> tau(std::max(N, n));
    int lwork = -1, info = 0;
    cd wq;
    int M_ = n, N_ = N, K_ = n, lda = n;
    g_lapack.zgelqf(&M_, &N_, nullptr, &lda, nullptr, &wq, &lwork, &info);
    int lw1 = (int)wq.real();
    g_lapack.zunglq(&M_, &N_, &K_, nullptr, &lda, nullptr, &wq, &lwork, &info);
    int lw2 = (int)wq.real();
    int lw = std::max(std::max(lw1, lw2), std::max(N, n));
    std::vector<cd> work(lw);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nw; w++)
      for (int s = 0; s < 2; s++) {
        cd* Ws = h->W.data() + ((size_t)w * 2 + s) * N * n;
        int inf = 0;
        g_lapack.zgelqf(&M_, &N_, Ws, &lda, tau.data(), work.data(), &lw, &inf);
        g_lapack.zunglq(&M_, &N_, &K_, Ws, &lda, tau.data(), work.data(), &lw, &inf);
      }
  }
}

// afqmc_sys::calculate_energy (afqmc_sys.hpp:121-133) -> base::calculate_energy
// (energy.hpp:66-102) with the two-body matrix Vakbl.  Returns Eav.
double orc_energy_vakbl(orc_handle* h) {
  const int nw = h->nw;
  const int NAK = 2 * h->n * h->N;
  std::vector<cd> Gcloc((size_t)NAK * nw);
  for (int w = 0; w < nw; w++) h->Wd[(size_t)w * 8] = cd(0.);
  if (h->nthreads > 1)
    csrmm_N_par(h->Vakbl, nw, cd(1), h->Gc.data(), nw, cd(0), Gcloc.data(), nw);
  else
    csrmm_N(h->Vakbl, nw, cd(1), h->Gc.data(), nw, cd(0), Gcloc.data(), nw);
  for (int i = 0; i < NAK; i++)
    for (int w = 0; w < nw; w++)
      h->Wd[(size_t)w * 8] += h->Gc[(size_t)i * nw + w] * Gcloc[(size_t)i * nw + w];
  for (int w = 0; w < nw; w++) h->Wd[(size_t)w * 8] *= cd(0.5);
  // one-body: W_data[:,0] += T(Gc) * haj (energy.hpp:100)
  cd one(1.0);
  int inc1 = 1, inc8 = 8;
  g_lapack.zgemv("N", &nw, &NAK, &one, h->Gc.data(), &nw, h->haj.data(), &inc1, &one,
                 h->Wd.data(), &inc8);
  double eav = 0., wgt = 0.;
  for (int w = 0; w < nw; w++) {
    wgt += h->Wd[(size_t)w * 8 + 1].real();
    eav += h->Wd[(size_t)w * 8].real() * h->Wd[(size_t)w * 8 + 1].real();
  }
  return eav / wgt;
}

// Local energy from the unscaled half-rotated Cholesky factors (no reference symbol;
// the identity with energy.hpp:66-102 follows from the Vakbl definition at
// energy.hpp:37-51):  eloc = sum Gc.haj + 1/2 sum_n c_n^2 - 1/2 sum_{s,n} tr(T_sn T_sn),
// c_n = sum_{s,a,k} Lh_s[n][a][k] Gc_s[a][k],  T_sn = Lh_s[n] * Gc_s^T (n x n).
// Also writes the per-walker (E1, EJ, EK) triples into parts[nw][3] when non-null.
double orc_energy_chol(orc_handle* h, double* parts) {
  const int N = h->N, n = h->n, nw = h->nw, nc = h->nchol;
  const size_t NAK = 2ull * n * N;
#pragma omp parallel
  {
    std::vector<cd> G(NAK), T((size_t)n * n), cv(nc);
#pragma omp for schedule(dynamic, 1)
    for (int w = 0; w < nw; w++) {
      for (size_t i = 0; i < NAK; i++) G[i] = h->Gc[i * nw + w];
      cd e1(0.);
      for (size_t i = 0; i < NAK; i++) e1 += G[i] * h->haj[i];
      // c = Lh[nc][NAK] * G
      int one_i = 1, nak = (int)NAK;
      cd one(1.0), zero(0.0);
      g_lapack.zgemv("T", &nak, &nc, &one, h->Lh.data(), &nak, G.data(), &one_i, &zero,
                     cv.data(), &one_i);
      cd ej(0.);
      for (int c = 0; c < nc; c++) ej += cv[c] * cv[c];
      ej *= 0.5;
      cd ek(0.);
      for (int c = 0; c < nc; c++)
        for (int s = 0; s < 2; s++) {
          const cd* L = h->Lh.data() + (size_t)c * NAK + (size_t)s * n * N;
          const cd* Gs = G.data() + (size_t)s * n * N;
          rm_gemm('N', 'T', n, n, N, cd(1), L, N, Gs, N, cd(0), T.data(), n);
          cd tr(0.);
          for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++) tr += T[(size_t)a * n + b] * T[(size_t)b * n + a];
          ek += tr;
        }
      ek *= 0.5;
      h->Wd[(size_t)w * 8] = e1 + ej - ek;
      if (parts) {
        parts[3 * w] = e1.real(); parts[3 * w + 1] = ej.real(); parts[3 * w + 2] = ek.real();
      }
    }
  }
  double eav = 0., wgt = 0.;
  for (int w = 0; w < nw; w++) {
    wgt += h->Wd[(size_t)w * 8 + 1].real();
    eav += h->Wd[(size_t)w * 8].real() * h->Wd[(size_t)w * 8 + 1].real();
  }
  return eav / wgt;
}

// base::halfrotate_cholesky (rotate.hpp:69-169) with the reference's two-pass count and
// fill over Cholesky vectors.  Input: Spvn CSR [N*N x nchol] (already scaled), trial
// alpha/beta [N][n].  Output: CSR [nchol x 2nN] written into caller buffers sized by a
// first call with out_rowIndex == nullptr, which returns nnz.
long long orc_halfrotate(int N, int n, int nchol, const int* ri, const int* ci,
                         const double* vals, const double* trial_a, const double* trial_b,
                         double cutoff, int* out_rowIndex, int* out_cols, double* out_vals) {
  // transpose A (rotate.hpp:92): per Cholesky vector the list of (ik, value)
  std::vector<std::vector<std::pair<int, cd>>> byvec(nchol);
  const cd* v = (const cd*)vals;
  for (int r = 0; r < N * N; r++)
    for (int p = ri[r]; p < ri[r + 1]; p++) byvec[ci[p]].push_back({r, v[p]});
  std::vector<cd> An((size_t)N * N), C((size_t)n * N);
  const cd* tr[2] = {(const cd*)trial_a, (const cd*)trial_b};
  long long nz = 0;
  if (out_rowIndex) out_rowIndex[0] = 0;
  for (int i = 0; i < nchol; i++) {
    if (!byvec[i].empty()) {
      std::fill(An.begin(), An.end(), cd(0));
      for (auto& e : byvec[i]) An[e.first] = e.second;
      for (int s = 0; s < 2; s++) {
        // C = T(trial) * An (rotate.hpp:116,122)
        rm_gemm('T', 'N', n, N, N, cd(1), tr[s], n, An.data(), N, cd(0), C.data(), N);
        for (int a = 0; a < n; a++)
          for (int k = 0; k < N; k++)
            if (std::abs(C[(size_t)a * N + k]) > cutoff) {
              if (out_rowIndex) {
                out_cols[nz] = s * n * N + a * N + k;
                out_vals[2 * nz] = C[(size_t)a * N + k].real();
                out_vals[2 * nz + 1] = C[(size_t)a * N + k].imag();
              }
              nz++;
            }
      }
    }
    if (out_rowIndex) out_rowIndex[i + 1] = (int)nz;
  }
  return nz;
}

// Generic helpers exposed for the known-answer tests of the reference's own self-tests.
void orc_csrmm(char trans, int nrows, int ncols, const int* ri, const int* ci,
               const double* vals, int ncolsB, const double* alpha, const double* B, int ldb,
               const double* beta, double* C, int ldc) {
  CSR A;
  load_csr(A, nrows, ncols, ri, ci, vals);
  cd a(alpha[0], alpha[1]), b(beta[0], beta[1]);
  if (trans == 'N') csrmm_N(A, ncolsB, a, (const cd*)B, ldb, b, (cd*)C, ldc);
  else csrmm_T(A, ncolsB, a, (const cd*)B, ldb, b, (cd*)C, ldc);
}

void orc_rm_gemm(char opA, char opB, int M, int Nc, int K, const double* A, int lda,
                 const double* B, int ldb, double* C, int ldc) {
  rm_gemm(opA, opB, M, Nc, K, cd(1), (const cd*)A, lda, (const cd*)B, ldb, cd(0), (cd*)C, ldc);
}

// Square matrix inversion and determinant as ma::invert performs them.
int orc_invert(int n, double* A, double* det) {
  std::vector<int> ipiv(n);
  std::vector<cd> work(64 * (size_t)n);
  int info = 0;
  cd d = invert((cd*)A, n, ipiv.data(), work.data(), (int)work.size(), &info);
  det[0] = d.real(); det[1] = d.imag();
  return info;
}

void orc_normals(uint64_t seed, uint64_t step, long long count, double* out) {
  for (long long j = 0; 2 * j < count; j++) {
    double a, b;
    normal_pair(seed, step, (uint64_t)j, &a, &b);
    out[2 * j] = a;
    if (2 * j + 1 < count) out[2 * j + 1] = b;
  }
}

}  // extern "C"
