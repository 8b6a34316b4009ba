// Mixed-precision form of the contraction stages on tcgen05 tensor cores.
//
// Complex products C = A B run as real GEMMs D[m][n] = sum_k A'[m][k] B'[n][k] (both
// operands K-major bf16, fp32 accumulation in TMEM):
//   A' rows are A's rows with real and imaginary parts interleaved along K;
//   B' has two rows per column j of B: (Re b, -Im b) interleaved -> D = Re C[:, j],
//                                      (Im b,  Re b) interleaved -> D = Im C[:, j].
// Each operand is stored as bf16 hi and lo parts (x = hi + lo); a stage runs either plain
// bf16 (hi only) or the split form hi*hi + hi*lo + lo*hi (~16 significant bits).
//
//   vHS   : D[(w,re|im)][ik] = sum_c X[c][w] Spvn[ik][c]        -> V_w operand (epilogue)
//   prop  : S = P W; T_k = (i/k) V T_{k-1}, S += T_k; W = P S    (fused Taylor epilogues)
//   vbias : D[c][(w,re|im)] = sum_ak SpvnT[c][ak] Gc_w[ak]       (split K, fixed-order sum)
//   E_J   : same product with the unscaled half-rotated factors
//   E_K   : T_cw = Lh_c Gc_w^T per spin, trace of T^2 from the tile in shared memory
// LU/overlaps, orthogonalisation, weights and the energy assembly stay FP64.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "afq_kernels.h"
#include "afq_mixed.h"
#include "tc_gemm.cuh"

namespace afq {

typedef __nv_bfloat16 bf16;
typedef __nv_bfloat162 bf162;

// PREC_BF16: plain bf16; PREC_SPLIT: bf16 hi + lo (hi*hi + hi*lo + lo*hi, ~16 bits);
// PREC_SPLIT16: fp16 hi + lo of power-of-two scaled values (~22 bits)
enum { PREC_BF16 = 0, PREC_SPLIT = 1, PREC_SPLIT16 = 2 };

// A 2-byte operand in hi (+ lo) parts.  f16: the parts are fp16 and every value is
// multiplied by `scale` (a power of two chosen from the operand's range) when written.
struct Op {
  bf16* hi = nullptr;
  bf16* lo = nullptr;
  int f16 = 0;
  float scale = 1.0f;
};

// bf16 writers (an operand whose consumer runs plain bf16 is passed with lo == nullptr:
// hi only).  The epilogues of the products use these; put2f / put1f below also handle
// fp16 operands and are used by the pack kernels of operands that may be fp16.
AFQ_D void put2(const Op& o, long long idx, float a, float b) {
  bf162 h = __floats2bfloat162_rn(a, b);
  *reinterpret_cast<bf162*>(o.hi + idx) = h;
  if (o.lo) {
    float2 hf = __bfloat1622float2(h);
    *reinterpret_cast<bf162*>(o.lo + idx) = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  }
}
AFQ_D void put1(const Op& o, long long idx, float a) {
  bf16 h = __float2bfloat16_rn(a);
  o.hi[idx] = h;
  if (o.lo) o.lo[idx] = __float2bfloat16_rn(a - __bfloat162float(h));
}
AFQ_D void put2f(const Op& o, long long idx, float a, float b) {
  if (!o.f16) {
    put2(o, idx, a, b);
    return;
  }
  a *= o.scale;
  b *= o.scale;
  const __half2 h = __floats2half2_rn(a, b);
  *reinterpret_cast<__half2*>(o.hi + idx) = h;
  if (o.lo) {
    const float2 hf = __half22float2(h);
    *reinterpret_cast<__half2*>(o.lo + idx) = __floats2half2_rn(a - hf.x, b - hf.y);
  }
}
AFQ_D void put1f(const Op& o, long long idx, float a) {
  if (!o.f16) {
    put1(o, idx, a);
    return;
  }
  a *= o.scale;
  const __half h = __float2half_rn(a);
  reinterpret_cast<__half*>(o.hi)[idx] = h;
  if (o.lo) reinterpret_cast<__half*>(o.lo)[idx] = __float2half_rn(a - __half2float(h));
}
AFQ_D float2 get2(const Op& o, long long idx) {   // bf16 operands
  float2 h = __bfloat1622float2(*reinterpret_cast<const bf162*>(o.hi + idx));
  float2 l = __bfloat1622float2(*reinterpret_cast<const bf162*>(o.lo + idx));
  return make_float2(h.x + l.x, h.y + l.y);
}

struct MixedState {
  MixedInit in{};
  int N = 0, n = 0, nc = 0, nw = 0;
  long long NAK = 0;
  bool s_real = true;
  int Kv = 0;                  // K of the vHS product (nchol, or 2*nchol for complex Spvn)
  int prec_vhs = PREC_SPLIT, prec_p = PREC_SPLIT, prec_v1 = PREC_SPLIT, prec_vk = PREC_BF16;
  // fp16 split (PREC_SPLIT16) measured no better than bf16 split for these products: their
  // error at C4 sizes is set by the fp32 accumulation over long K, not by the operands
  int prec_vbias = PREC_SPLIT, prec_ej = PREC_SPLIT, prec_ek = PREC_SPLIT;
  int bn_prop = 0;             // tile width >= 4n of the propagation products
  Op Sd, Pf, SpT, LhJ, LhX;    // static operands
  Op Xf, Vf, F[2], Gb, Gx;     // per-step operands
  float2* S = nullptr;         // Taylor sum [nw][2n][N]
  float* part = nullptr;       // split-K partial products
  int splits = 1, ksplit = 0;
  // real SpvnT and Lh (real orbitals and Cholesky vectors): A operands hold real values
  // only and the G operands carry Re and Im in separate rows, so K is halved
  bool greal = false;
  bool preal = false;   // real Propg1: P W and P S take K = N with (Re | Im) B rows
  // fp16 split for the G products (vbias, E_J, E_K): static operands scaled by a power of
  // two (sSpT, sLh), the G operands per walker (wscale[w], from the walker's max |G|)
  bool f16g = false;
  float sSpT = 1.0f, sLh = 1.0f;
  float* wscale = nullptr;
  double* dmax = nullptr;
  int* err = nullptr;
  int ex_Gn = 0, ex_Gw = 0, ex_bn = 0, ex_mtiles = 0;
  std::vector<void*> allocs;
  tc::Maps m_vhs, m_pw[2], m_v[2], m_vbias, m_ej, m_ek;
  tc::Maps m_vhs64;   // vHS operands in 64-byte K slabs (SWIZZLE_64B), epilogue choice 3
  // walker width 2n = 80: the promoted exchange on 160-column tiles (two walkers, one
  // epilogue warpgroup), with its own Gx map (160-row boxes)
  tc::Maps m_ek80;
  bool ex80 = false;
  // symmetric Cholesky vectors (L_n(i,k) = L_n(k,i)): the vHS product covers the 16 x 16
  // orbital blocks (ib <= jb) only and the epilogue mirrors them
  bool vsym = false;
  int npairs = 0;
  int* pairs = nullptr;        // [npairs] ib << 16 | jb
  // mixed density matrix: T1 = W^T tw (split bf16) -> FP64 LU / inverse -> Gc = T1^-1 W^T
  Op TwB, Wn, Tinv;            // trial B form, W natural bf16, B form of T1^-1 per spin
  float2* T1 = nullptr;        // [nw][2][n][n]
  int bn_t1 = 0, bn_gc = 0;
  tc::Maps m_t1, m_gc[2];
  // packed forms of the current walkers written by the last propagation product (pair
  // epilogue) or by mixed_repack: F2 = the next P W operand, F[fa_buf] = the T1 operand.
  // `packed` is false after anything else changed W.  (The Gc operand Wn is packed by the
  // density matrix: its row-strided stores cost the epilogue more than the pack kernel.)
  Op F2;
  tc::Maps m_pw2, m_t1_1;
  // symmetric vHS epilogue: 0 row-wise (EpiVhsSym, the tuned kernel), 1 through the
  // shared-memory tile (EpiVhsSymTile, per-tile kernel), 2 the same with two CTAs per SM
  // (one stage each, the tile staged in halves), 3 as 2 with two 64-byte-slab stages per
  // CTA; picked by the set-up tuner
  int vhs_epi = 0;
  float vhs_epi_ms[4] = {};
  bool packed = false;
  int fa_buf = 0;
  // kernel of each product site (0 built-in rule, 1 persistent, 2 per-tile), chosen at
  // set-up by timing the candidates on the real shapes; part_cap = split-K slots allocated
  int tune[TS_N] = {};
  float tune_ms[TS_N][2] = {};
  // propagation chain run walker group by walker group (0: all walkers per product), so a
  // group's Taylor sum, operands and V stay in L2 across its eight products; picked by the
  // set-up tuner (prop_group_ms: the timed chain per candidate, 0 = all walkers first)
  int prop_group = 0;
  float prop_group_ms[6] = {};
  // the propagation chain as one cooperative persistent launch per substep (2n a multiple
  // of 32): per-walker dependency counters, walkers per wave (0: eight launches), timed by
  // the set-up tuner (chain_ms: eight launches, waves of 16, 24 and 32 walkers)
  unsigned* dep = nullptr;
  int chain_wave = 0;
  float chain_ms[6] = {};
  int splits0 = 1, part_cap = 1;
};

namespace {

template <class T>
cudaError_t malloc_track(MixedState* m, T** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * (count ? count : 1));
  if (e == cudaSuccess) {
    m->allocs.push_back(q);
    *p = static_cast<T*>(q);
  }
  return e;
}
cudaError_t alloc_op(MixedState* m, Op& o, size_t count) {
  cudaError_t e = malloc_track(m, &o.hi, count);
  if (e == cudaSuccess) e = malloc_track(m, &o.lo, count);
  return e;
}

// ------------------------------------------------------------ static operand packing
// interleaved complex rows: dst[r][2q + {0,1}] = (Re, Im) src[r][q]
__global__ void pack_complex_kernel(const z_t* __restrict__ src, long long count, Op dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x) {
    z_t v = src[e];
    put2f(dst, 2 * e, (float)v.x, (float)v.y);
  }
}
// max over src of max(|re|, |im|), into *out (double; atomicMax on the bit pattern of a
// non-negative double orders like the value)
__global__ void maxabs_kernel(const z_t* __restrict__ src, long long count,
                              unsigned long long* out) {
  double m = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fmax(fabs(src[e].x), fabs(src[e].y)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
// power-of-two scale that brings a magnitude m to [2^11, 2^12): fp16 keeps 16x headroom
AFQ_HD float pow2_scale(double m) {
  if (!(m > 0.0) || !isfinite(m)) return 1.0f;
  int ex;
  frexp(m, &ex);   // m = f * 2^ex, f in [0.5, 1)
  return (float)ldexp(1.0, 12 - ex);
}
// per-walker scale of the compact density matrices Gc [nw][NAK]
__global__ void __launch_bounds__(256)
gc_scale_kernel(const z_t* __restrict__ Gc, long long nak, float* __restrict__ wscale) {
  __shared__ double red[8];
  const int w = blockIdx.x;
  double m = 0.0;
  for (long long i = threadIdx.x; i < nak; i += blockDim.x) {
    const z_t g = Gc[(long long)w * nak + i];
    m = fmax(m, fmax(fabs(g.x), fabs(g.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = red[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) mm = fmax(mm, red[i]);
    wscale[w] = pow2_scale(mm);
  }
}

// flag = 1 if any imaginary part of src is nonzero
__global__ void check_imag_kernel(const z_t* __restrict__ src, long long count, int* flag) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x)
    if (src[e].y != 0.0) *flag = 1;
}
// real parts: dst[e] = Re src[e]
__global__ void pack_real_kernel(const z_t* __restrict__ src, long long count, Op dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x)
    put1f(dst, e, (float)src[e].x);
}
// Lh [c][s][a][k] -> real LhX [s][c][a][k]
__global__ void pack_lhx_real_kernel(const z_t* __restrict__ Lh, int nc, int n, int N, Op dst) {
  const long long per = (long long)n * N, tot = 2LL * nc * per;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long s = e / (nc * per), r = e % (nc * per), c = r / per, q = r % per;
    put1f(dst, e, (float)Lh[c * 2 * per + s * per + q].x);
  }
}
// Lh [c][s][a][k] -> LhX [s][c][a][2k]
__global__ void pack_lhx_kernel(const z_t* __restrict__ Lh, int nc, int n, int N, Op dst) {
  const long long per = (long long)n * N, tot = 2LL * nc * per;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long s = e / (nc * per), r = e % (nc * per), c = r / per, q = r % per;
    z_t v = Lh[c * 2 * per + s * per + q];
    put2f(dst, 2 * e, (float)v.x, (float)v.y);
  }
}
// dense Spvn from CSR: real values -> [ik][c]; complex -> [ik][2c + {0,1}]
__global__ void pack_spvn_kernel(const int* __restrict__ ri, const int* __restrict__ ci,
                                 const z_t* __restrict__ zv, const double* __restrict__ rv,
                                 int nrows, int Kv, int real, Op dst) {
  int r = blockIdx.x * blockDim.y + threadIdx.y;
  if (r >= nrows) return;
  for (int p = ri[r] + threadIdx.x; p < ri[r + 1]; p += blockDim.x) {
    long long base = (long long)r * Kv;
    if (real) put1(dst, base + ci[p], (float)(rv ? rv[p] : zv[p].x));
    else put2(dst, base + 2LL * ci[p], (float)zv[p].x, (float)zv[p].y);
  }
}

// Symmetry test of the packed Spvn rows ik = i*N + k: flag = 1 if any (i,k) row differs
// from the (k,i) row in either bf16 part.
__global__ void check_sym_kernel(Op Sd, int N, int Kv, int* flag) {
  const long long tot = (long long)N * N * Kv;
  const uint16_t* hi = reinterpret_cast<const uint16_t*>(Sd.hi);
  const uint16_t* lo = reinterpret_cast<const uint16_t*>(Sd.lo);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / Kv, c = e % Kv;
    const int i = (int)(r / N), k = (int)(r % N);
    if (i >= k) continue;
    const long long t = ((long long)k * N + i) * Kv + c;
    if (hi[e] != hi[t] || lo[e] != lo[t]) *flag = 1;
  }
}
// Block-pair rows: dst row p = t*256 + ii*16 + jj <- Sd row (ib*16 + ii)*N + jb*16 + jj
// for the t-th block pair (ib, jb); 16-byte copies (Kv is a multiple of 8).
__global__ void pack_sym_kernel(Op Sd, int N, int Kv, const int* __restrict__ pairs, int npairs,
                                Op dst) {
  const int q = Kv / 8;   // uint4 per row
  const long long tot = (long long)npairs * 256 * q;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / q;
    const int c = (int)(e % q), t = (int)(p >> 8), ii = (int)((p >> 4) & 15), jj = (int)(p & 15);
    const int ib = pairs[t] >> 16, jb = pairs[t] & 0xffff;
    const long long src = ((long long)(ib * 16 + ii) * N + jb * 16 + jj) * q + c;
    reinterpret_cast<uint4*>(dst.hi)[e] = reinterpret_cast<const uint4*>(Sd.hi)[src];
    reinterpret_cast<uint4*>(dst.lo)[e] = reinterpret_cast<const uint4*>(Sd.lo)[src];
  }
}

// ------------------------------------------------------------ per-step operand packing
// X [nc][nw] -> Xf rows (w, re|im): real Spvn: (Re X[:,w]) and (Im X[:,w]);
// complex Spvn: (Re, -Im) and (Im, Re) interleaved along c.
__global__ void pack_x_kernel(const z_t* __restrict__ X, int nc, int nw, int Kv, int real, Op dst) {
  __shared__ z_t t[32][33];
  const int c0 = blockIdx.x * 32, w0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int c = c0 + i, w = w0 + threadIdx.x;
    t[i][threadIdx.x] = (c < nc && w < nw) ? X[(long long)c * nw + w] : zmk(0, 0);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int w = w0 + i, c = c0 + threadIdx.x;
    if (w >= nw || c >= nc) continue;
    z_t v = t[threadIdx.x][i];
    long long r0 = (2LL * w) * Kv, r1 = (2LL * w + 1) * Kv;
    if (real) {
      put1(dst, r0 + c, (float)v.x);
      put1(dst, r1 + c, (float)v.y);
    } else {
      put2(dst, r0 + 2 * c, (float)v.x, (float)-v.y);
      put2(dst, r1 + 2 * c, (float)v.y, (float)v.x);
    }
  }
}
// W [nw][N][2n] -> B form F [nw][4n][2N]: row j: (Re W[:,j], -Im W[:,j]); row 2n+j: (Im, Re)
// both == 2: real-A form instead, row j = Re W[:, j], row n2 + j = Im W[:, j] (K = N).
__global__ void pack_w_kernel(const z_t* __restrict__ W, int N, int n2, Op dst, int both = 1) {
  __shared__ z_t t[32][33];
  const int w = blockIdx.z, k0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const z_t* Ww = W + (long long)w * N * n2;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int k = k0 + i, j = j0 + threadIdx.x;
    t[i][threadIdx.x] = (k < N && j < n2) ? Ww[(long long)k * n2 + j] : zmk(0, 0);
  }
  __syncthreads();
  const long long base = (long long)w * 2 * n2 * 2 * N;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int j = j0 + i, k = k0 + threadIdx.x;
    if (j >= n2 || k >= N) continue;
    z_t v = t[threadIdx.x][i];
    if (both == 2) {
      put1(dst, base + (long long)j * 2 * N + k, (float)v.x);
      put1(dst, base + (long long)(n2 + j) * 2 * N + k, (float)v.y);
      continue;
    }
    put2(dst, base + (long long)j * 2 * N + 2 * k, (float)v.x, (float)-v.y);
    if (both) put2(dst, base + (long long)(n2 + j) * 2 * N + 2 * k, (float)v.y, (float)v.x);
  }
}
// Trial B form of T1: rows 2(s n + b) = (Re tw, Im tw), 2(s n + b) + 1 = (-Im tw, Re tw)
// interleaved along k (the conjugate-trial rows; the product then gives conj(T1)).
__global__ void pack_trial_kernel(const z_t* __restrict__ tw, int N, int n2, Op dst) {
  const long long tot = (long long)N * n2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / n2), j = (int)(e % n2);
    const z_t v = tw[e];
    put2(dst, (2LL * j) * 2 * N + 2 * k, (float)v.x, (float)v.y);
    put2(dst, (2LL * j + 1) * 2 * N + 2 * k, (float)-v.y, (float)v.x);
  }
}
// W [nw][N][n2] -> bf16 hi/lo in the same layout ((re, im) pairs): A operand of Gc.
__global__ void pack_wn_kernel(const z_t* __restrict__ W, long long count, Op dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x) {
    const z_t v = W[e];
    put2(dst, 2 * e, (float)v.x, (float)v.y);
  }
}

// Batched FP64 Gauss-Jordan of the n x n overlap matrices T1, one CTA per walker-spin
// with the matrix in registers: thread (r, q), numbered t = q * GR + r so that a column's
// owners are consecutive lanes, holds the elements (r + GR a, q + GC b).  Pivoting as
// izamax (max |re| + |im| over the rows not yet used, ma_operations.hpp:244-260), without
// moving rows: step j pivots on (p_j, j), scales the pivot row and eliminates column j
// from every other row (in-place exchange form).  Afterwards element (i, c) holds
// T1^-1[invp(i)][p_c] and det(T1) = sign(p) prod pivots.  Writes det (overlap), the
// singular flag and, when want_inv, T1^-1 as the B form of the Gc product:
// rows 2a = (Re y, -Im y), 2a + 1 = (Im y, Re y) along b, y = T1^-1[a][.].
// Per step: the column's owners (GR consecutive lanes) pick the pivot with shuffles, one
// barrier publishes it, a second one publishes the scaled pivot row and the column.
template <int GR, int GC, int RT, int CT>
__global__ void __launch_bounds__(GR * GC)
lu_inv_kernel(const float2* __restrict__ T1, int n, Op Tinv, z_t* __restrict__ Wd,
              int* __restrict__ info, int want_inv, int save_old) {
  static_assert(GR == 8 || GR == 16, "a column's owners fill a half warp or a quarter");
  __shared__ z_t prow[64], pcol[64];
  __shared__ z_t s_pv;
  __shared__ int s_p, pivrow[64], invp[64];
  const int q = blockIdx.x, t = threadIdx.x, cq = t / GR, r = t % GR;
  const float2* src = T1 + (long long)q * n * n;
  z_t M[RT][CT];
#pragma unroll
  for (int a = 0; a < RT; a++)
#pragma unroll
    for (int b = 0; b < CT; b++) {
      const int i = r + GR * a, c = cq + GC * b;
      const float2 v = (i < n && c < n) ? src[i * n + c] : make_float2(0.f, 0.f);
      M[a][b] = zmk(v.x, v.y);
    }
  unsigned used = 0;   // bit a: row r + GR a is a pivot row already
  z_t det = zmk(1.0, 0.0);
  int sing = 0;
  for (int j = 0; j < n; j++) {
    const int jq = j % GC, jb = j / GC;
    if (cq == jq) {   // owners of column j: pivot among their unused rows, then shuffles
      double best = -1.0;
      int bi = n;
      z_t bv = zmk(0, 0);
#pragma unroll
      for (int a = 0; a < RT; a++) {
        const int i = r + GR * a;
        z_t v = zmk(0, 0);
#pragma unroll
        for (int b = 0; b < CT; b++)
          if (b == jb) v = M[a][b];
        if (i < n && !((used >> a) & 1u)) {
          const double m = zabs1(v);
          if (m > best) { best = m; bi = i; bv = v; }
        }
      }
      // the GR owners are consecutive lanes of one warp: shuffle among them only
      const unsigned grp = ((1u << GR) - 1u) << ((t & 31) & ~(GR - 1));
#pragma unroll
      for (int o = GR / 2; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(grp, best, o);
        const int oi = __shfl_xor_sync(grp, bi, o);
        const double ovx = __shfl_xor_sync(grp, bv.x, o);
        const double ovy = __shfl_xor_sync(grp, bv.y, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; bv = zmk(ovx, ovy); }
      }
      if (r == 0) {
        s_p = best > 0.0 ? bi : -1;   // exactly singular: no nonzero candidate
        s_pv = bv;
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) { sing = 1; break; }   // uniform across the CTA
    const z_t pv = s_pv;
    if (t == 0) {
      det = zmul(det, pv);
      pivrow[j] = p;
    }
    const int pr = p % GR, pa = p / GR;
    if (r == pr) {   // pivot-row owners publish the scaled row
      const z_t inv = zrecip(pv);
#pragma unroll
      for (int a = 0; a < RT; a++)
        if (a == pa)
#pragma unroll
          for (int b = 0; b < CT; b++) {
            const int c = cq + GC * b;
            if (c < n) prow[c] = (c == j) ? inv : zmul(M[a][b], inv);
          }
      used |= 1u << pa;
    }
    if (cq == jq) {   // column owners publish column j
#pragma unroll
      for (int a = 0; a < RT; a++) {
        const int i = r + GR * a;
        z_t v = zmk(0, 0);
#pragma unroll
        for (int b = 0; b < CT; b++)
          if (b == jb) v = M[a][b];
        if (i < n) pcol[i] = v;
      }
    }
    __syncthreads();
    z_t rowv[CT];
#pragma unroll
    for (int b = 0; b < CT; b++) {
      const int c = cq + GC * b;
      rowv[b] = c < n ? prow[c] : zmk(0, 0);
    }
#pragma unroll
    for (int a = 0; a < RT; a++) {
      const int i = r + GR * a;
      if (i >= n) continue;
      if (i == p) {
#pragma unroll
        for (int b = 0; b < CT; b++) M[a][b] = rowv[b];
      } else {
        const z_t f = pcol[i];
#pragma unroll
        for (int b = 0; b < CT; b++) {
          const z_t base = (cq + GC * b == j) ? zmk(0, 0) : M[a][b];
          M[a][b] = zsub(base, zmul(f, rowv[b]));
        }
      }
    }
    // prow / pcol are rewritten only after the next step's first barrier, which every
    // thread reaches after finishing this update
  }
  if (sing) det = zmk(0, 0);
  if (t == 0 && !sing) {   // sign of the permutation j -> p_j (inversion count)
    int inv_cnt = 0;
    for (int a = 0; a < n; a++)
      for (int b = a + 1; b < n; b++) inv_cnt += pivrow[a] > pivrow[b];
    if (inv_cnt & 1) det = zmk(-det.x, -det.y);
    for (int a = 0; a < n; a++) invp[pivrow[a]] = a;
  }
  __syncthreads();
  if (want_inv) {
    const long long base = (long long)q * 2 * n * 2 * n;
#pragma unroll
    for (int a = 0; a < RT; a++)
#pragma unroll
      for (int b = 0; b < CT; b++) {
        const int i = r + GR * a, c = cq + GC * b;
        if (i >= n || c >= n) continue;
        const int ra = sing ? i : invp[i], cb = sing ? c : pivrow[c];
        const z_t y = sing ? zmk(0, 0) : M[a][b];
        put2(Tinv, base + (2LL * ra) * 2 * n + 2 * cb, (float)y.x, (float)-y.y);
        put2(Tinv, base + (2LL * ra + 1) * 2 * n + 2 * cb, (float)y.y, (float)y.x);
      }
  }
  if (t == 0) {
    const int w = q >> 1, sp = q & 1;
    z_t* d = Wd + (long long)w * 8;
    if (save_old) {
      if (sp == 0) d[5] = d[4];
      d[6 + sp] = d[2 + sp];
    }
    d[2 + sp] = det;
    info[q] = sing;
  }
}

// The same Gauss-Jordan (in-place exchange form, implicit izamax pivoting) with the matrix
// in shared memory: 128 threads per matrix (warps on rows, lanes on columns), two
// barriers per pivot (the searching warp also scales the pivot row); small register
// footprint, so five matrices share an SM.
constexpr int LUS_THREADS = 128;
size_t lus_smem_bytes(int n) { return sizeof(z_t) * ((size_t)n * (n + 1) + 2 * n); }

__global__ void __launch_bounds__(LUS_THREADS)
lu_smem_kernel(const float2* __restrict__ T1, int n, Op Tinv, z_t* __restrict__ Wd,
               int* __restrict__ info, int want_inv, int save_old) {
  extern __shared__ __align__(16) unsigned char lus_raw[];
  __shared__ int s_p, pivrow[64], invp[64], used[64];
  __shared__ z_t s_pv;
  const int q = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int NWARP = LUS_THREADS / 32;
  const int ld = n + 1, nn = n * n;
  z_t* T = reinterpret_cast<z_t*>(lus_raw);
  z_t* pcol = T + n * ld;
  z_t* prow = pcol + n;
  const float2* src = T1 + (long long)q * nn;
  for (int e = tid; e < nn; e += LUS_THREADS) {
    const float2 v = src[e];
    T[(e / n) * ld + e % n] = zmk(v.x, v.y);
  }
  for (int i = tid; i < 64; i += LUS_THREADS) used[i] = 0;
  __syncthreads();
  z_t det = zmk(1.0, 0.0);
  int sing = 0;
  for (int j = 0; j < n; j++) {
    if (warp == 0) {   // pivot: max |re| + |im| of column j over the unused rows
      double best = -1.0;
      int bi = n;
      for (int i = lane; i < n; i += 32) {
        if (used[i]) continue;
        const double v = zabs1(T[i * ld + j]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) {
        s_p = best > 0.0 ? bi : -1;
        if (bi < n) {
          s_pv = T[bi * ld + j];
          used[bi] = 1;
          pivrow[j] = bi;
        }
      }
    }
    if (warp == 0) {   // the scaled pivot row, prepared by the searching warp
      __syncwarp();
      const int pp = s_p;
      if (pp >= 0) {
        const z_t inv = zrecip(T[pp * ld + j]);
        for (int c = lane; c < n; c += 32) prow[c] = (c == j) ? inv : zmul(T[pp * ld + c], inv);
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) { sing = 1; break; }   // uniform across the CTA
    if (tid == 0) det = zmul(det, s_pv);
    // lanes own columns lane and lane + 32 (n <= 64): the pivot row's values stay in
    // registers across the rows; a row's factor is its own column-j entry, read before
    // any lane of the warp writes the row; four rows per warp in flight
    const bool c0 = lane < n, c1 = lane + 32 < n;
    const z_t pr0 = c0 ? prow[lane] : zmk(0, 0), pr1 = c1 ? prow[lane + 32] : zmk(0, 0);
#pragma unroll 4
    for (int i = warp; i < n; i += NWARP) {
      z_t* Ti = T + i * ld;
      if (i == p) {
        if (c0) Ti[lane] = pr0;
        if (c1) Ti[lane + 32] = pr1;
        continue;
      }
      const z_t f = Ti[j];
      const z_t b0 = (c0 && lane != j) ? Ti[lane] : zmk(0, 0);
      const z_t b1 = (c1 && lane + 32 != j) ? Ti[lane + 32] : zmk(0, 0);
      __syncwarp();
      if (c0)
        Ti[lane] = zmk(fma(-f.x, pr0.x, fma(f.y, pr0.y, b0.x)), fma(-f.x, pr0.y, fma(-f.y, pr0.x, b0.y)));
      if (c1)
        Ti[lane + 32] =
            zmk(fma(-f.x, pr1.x, fma(f.y, pr1.y, b1.x)), fma(-f.x, pr1.y, fma(-f.y, pr1.x, b1.y)));
    }
    __syncthreads();
  }
  if (sing) det = zmk(0, 0);
  if (tid == 0 && !sing) {
    int inv_cnt = 0;
    for (int a = 0; a < n; a++)
      for (int b = a + 1; b < n; b++) inv_cnt += pivrow[a] > pivrow[b];
    if (inv_cnt & 1) det = zmk(-det.x, -det.y);
    for (int a = 0; a < n; a++) invp[pivrow[a]] = a;
  }
  __syncthreads();
  if (want_inv) {
    const long long base = (long long)q * 2 * n * 2 * n;
    for (int e = tid; e < nn; e += LUS_THREADS) {
      const int i = e / n, c = e % n;
      const int ra = sing ? i : invp[i], cb = sing ? c : pivrow[c];
      const z_t y = sing ? zmk(0, 0) : T[i * ld + c];
      put2(Tinv, base + (2LL * ra) * 2 * n + 2 * cb, (float)y.x, (float)-y.y);
      put2(Tinv, base + (2LL * ra + 1) * 2 * n + 2 * cb, (float)y.y, (float)y.x);
    }
  }
  if (tid == 0) {
    const int w = q >> 1, sp = q & 1;
    z_t* d = Wd + (long long)w * 8;
    if (save_old) {
      if (sp == 0) d[5] = d[4];
      d[6 + sp] = d[2 + sp];
    }
    d[2 + sp] = det;
    info[q] = sing;
  }
}

cudaError_t launch_lu(const float2* T1, int n, int nmat, Op Tinv, z_t* Wd, int* info, int want_inv,
                      int save_old, cudaStream_t st) {
  static const bool regs = getenv("AFQ_LU_REGISTERS") != nullptr;
  if (!regs && n <= 64) {   // shared-memory form (default)
    const size_t smem = lus_smem_bytes(n);
    static DeviceAttr attr;   // and the full shared-memory carveout: five matrices per SM
    cudaError_t e = attr.ensure(smem, [](size_t b) {
      cudaError_t r = cudaFuncSetAttribute(lu_smem_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
      if (r == cudaSuccess)
        r = cudaFuncSetAttribute(lu_smem_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
      return r;
    });
    if (e != cudaSuccess) return e;
    lu_smem_kernel<<<nmat, LUS_THREADS, smem, st>>>(T1, n, Tinv, Wd, info, want_inv, save_old);
    return cudaGetLastError();
  }
  // 16 x 16 threads per matrix: few registers per thread, many warps per SM
  if (n <= 16)
    lu_inv_kernel<8, 8, 2, 2><<<nmat, 64, 0, st>>>(T1, n, Tinv, Wd, info, want_inv, save_old);
  else if (n <= 32)
    lu_inv_kernel<16, 16, 2, 2><<<nmat, 256, 0, st>>>(T1, n, Tinv, Wd, info, want_inv, save_old);
  else if (n <= 48)
    lu_inv_kernel<16, 16, 3, 3><<<nmat, 256, 0, st>>>(T1, n, Tinv, Wd, info, want_inv, save_old);
  else if (n <= 64)
    lu_inv_kernel<16, 16, 4, 4><<<nmat, 256, 0, st>>>(T1, n, Tinv, Wd, info, want_inv, save_old);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// Gc [nw][2][n][N] -> Gb [2nw][2*NAK] (vbias / Coulomb B form) and, when Gx.hi is set,
// Gx [2][nwx][2n][2N] (exchange B form, rows (w, re|im, b) per spin; nwx = the walker
// capacity of Gx, which fixes the spin stride the exchange product reads with).
// real == 1 (real A operands): Gb rows w = Re Gc_w, nw + w = Im Gc_w over NAK; Gx rows
// (w, re, b) = Re Gc_w[b][.], (w, im, b) = Im over N.
// wscale (optional): per-walker factor applied before the conversion (fp16 operands).
__global__ void pack_gc_kernel(const z_t* __restrict__ Gc, int nw, int n, int N, Op Gb, Op Gx,
                               int nwx = 0, int real = 0, const float* __restrict__ wscale = nullptr) {
  const long long NAK = 2LL * n * N, tot = (long long)nw * NAK;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long w = e / NAK, q = e % NAK;
    z_t g = Gc[e];
    if (wscale) g = zscale(g, (double)wscale[w]);
    if (real) {
      if (Gb.hi) {
        put1f(Gb, w * NAK + q, (float)g.x);
        put1f(Gb, (nw + w) * NAK + q, (float)g.y);
      }
      if (Gx.hi) {
        const long long s = q / ((long long)n * N), r = q % ((long long)n * N);
        const long long b = r / N, k = r % N;
        const long long row0 = (s * (nwx ? nwx : nw) + w) * 2 * n + b;
        put1f(Gx, row0 * N + k, (float)g.x);
        put1f(Gx, (row0 + n) * N + k, (float)g.y);
      }
      continue;
    }
    if (Gb.hi) {
      put2f(Gb, w * 2 * NAK + 2 * q, (float)g.x, (float)-g.y);
      put2f(Gb, (nw + w) * 2 * NAK + 2 * q, (float)g.y, (float)g.x);
    }
    if (Gx.hi) {
      const long long s = q / ((long long)n * N), r = q % ((long long)n * N);
      const long long b = r / N, k = r % N;
      const long long row0 = (s * (nwx ? nwx : nw) + w) * 2 * n + b, row1 = row0 + n;
      put2f(Gx, row0 * 2 * N + 2 * k, (float)g.x, (float)-g.y);
      put2f(Gx, row1 * 2 * N + 2 * k, (float)g.y, (float)g.x);
    }
  }
}
// sum of split-K partials: out[c][w] = sum_z part[z][c][w] + i part[z][c][nw + w]
// (scaled operands: the sum is divided by ascale * wscale[w])
__global__ void reduce_part_kernel(const float* __restrict__ part, int splits, int M, int nw,
                                   z_t* __restrict__ out, float ascale = 1.0f,
                                   const float* __restrict__ wscale = nullptr) {
  const long long tot = (long long)M * nw, sz = (long long)M * 2 * nw;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const long long c = e / nw, w = e % nw;
    double re = 0.0, im = 0.0;
    for (int z = 0; z < splits; z++) {
      re += part[z * sz + c * 2 * nw + w];
      im += part[z * sz + c * 2 * nw + nw + w];
    }
    const double u = 1.0 / ((double)ascale * (wscale ? (double)wscale[w] : 1.0));
    out[e] = zmk(re * u, im * u);
  }
}
// V operand back to FP64 vHS [nw][N*N] (for copy-out only)
__global__ void unpack_v_kernel(Op V, long long count, z_t* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
       e += (long long)gridDim.x * blockDim.x) {
    float2 v = get2(V, 2 * e);
    out[e] = zmk(v.x, v.y);
  }
}

int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

// ------------------------------------------------------------ epilogues
// vHS: rows (w, re|im) are adjacent lanes; the even lane writes columns 0-15 of the
// chunk, the odd lane columns 16-31, as (re, im) pairs of V_w[ik].
struct EpiVhs {
  static constexpr bool kTile = false, kPair = false;
  static constexpr bool kPerTile = true;
  Op V;
  int nw;
  long long nik;
  AFQ_D void operator()(int, int, int m, int n0, const float* v) const {
    const bool odd = threadIdx.x & 1;
    float o[32];
#pragma unroll
    for (int i = 0; i < 32; i++) o[i] = __shfl_xor_sync(0xffffffffu, v[i], 1);
    const int w = m >> 1;
    if (w >= nw) return;
#pragma unroll
    for (int i = 0; i < 32; i++) {
      if ((i < 16) == odd) continue;
      const long long ik = n0 + i;
      if (ik >= nik) continue;
      const float re = odd ? o[i] : v[i], im = odd ? v[i] : o[i];
      put2(V, ((long long)w * nik + ik) * 2, re, im);
    }
  }
};


// T1 product: rows j = s n + a of the walker (first 2n rows of the tile), columns
// 2(s' n + b) + {re, im} of conj(T1); keeps the s' == s blocks as T1[w][s][a][b].
struct EpiT1 {
  static constexpr bool kTile = false, kPair = false;
  float2* T1;
  int n;
  AFQ_D void operator()(int w, int row, int, int n0, const float* v) const {
    if (row >= 2 * n) return;
    const int s = row / n, a = row % n;
    float2* dst = T1 + (((long long)w * 2 + s) * n + a) * n;
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int col = n0 + 2 * i, sb = col / (2 * n), b = (col % (2 * n)) >> 1;
      if (sb == s) dst[b] = make_float2(v[2 * i], -v[2 * i + 1]);
    }
  }
};

// Gc product of spin s: rows k, columns 2a + {re, im}: Gc[w][s][a][k].
struct EpiGc {
  static constexpr bool kTile = false, kPair = false;
  z_t* Gc;
  int n, N, s;
  AFQ_D void operator()(int w, int, int k, int n0, const float* v) const {
    if (k >= N) return;
    z_t* dst = Gc + ((long long)w * 2 + s) * n * N + k;
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int a = (n0 >> 1) + i;
      if (a < n) dst[(long long)a * N] = zmk(v[2 * i], v[2 * i + 1]);
    }
  }
};

// vHS of symmetric Cholesky vectors: each 256-column tile is one 16 x 16 orbital block
// pair (ib, jb), column q = ii*16 + jj; the value goes to V[i][j] and, off the block
// diagonal, to V[j][i].
struct EpiVhsSym {
  static constexpr bool kTile = false, kPair = false;
  static constexpr bool kPerTile = true;   // measured faster than the persistent kernel
  Op V;
  int nw, N;
  const int* pairs;
  AFQ_D void operator()(int, int, int m, int n0, const float* v) const {
    const bool odd = threadIdx.x & 1;
    float o[32];
#pragma unroll
    for (int c = 0; c < 32; c++) o[c] = __shfl_xor_sync(0xffffffffu, v[c], 1);
    const int w = m >> 1;
    if (w >= nw) return;
    // tile t -> block pair (ib, jb), ib <= jb, in row order (no memory access)
    int t = n0 >> 8, ib = 0;
    const int nb = N >> 4;
    while (t >= nb - ib) { t -= nb - ib; ib++; }
    const int jb = ib + t;
    const int i = ib * 16 + ((n0 & 255) >> 4) + (odd ? 1 : 0);
    const long long vw = (long long)w * N * N;
#pragma unroll
    for (int jj = 0; jj < 16; jj++) {
      const float re = odd ? o[16 + jj] : v[jj], im = odd ? v[16 + jj] : o[jj];
      const int j = jb * 16 + jj;
      put2(V, (vw + (long long)i * N + j) * 2, re, im);
      if (ib != jb) put2(V, (vw + (long long)j * N + i) * 2, re, im);
    }
  }
};

// EpiVhsSym through the fp32 tile in shared memory (per-tile kernel): the same values,
// written as 16-byte vector stores of four complex entries.  Tile row r = 2 wl (Re) /
// 2 wl + 1 (Im) of walker mt * 64 + wl, column q = ii * 16 + jj.  Items (walker, row of
// the 16 x 16 block, quarter): V[i][jb*16 + 4 quarter ..] from row ii of the block and,
// off the block diagonal, V[j][ib*16 + 4 quarter ..] from column jj (the mirror), so both
// halves leave as contiguous 64-byte rows instead of the row-wise functor's
// one-lane-per-walker 4-byte mirror stores.  Needs N % 4 == 0 (16-byte aligned rows).
struct EpiVhsSymTile {
  static constexpr bool kTile = true, kPair = false, kHalfTile = true;
  Op V;
  int nw, N;
  const int* pairs;
  AFQ_D static void put4(const Op& o, long long idx, const float* re, const float* im) {
    bf162 h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      h[e] = __floats2bfloat162_rn(re[e], im[e]);
      const float2 hf = __bfloat1622float2(h[e]);
      l[e] = __floats2bfloat162_rn(re[e] - hf.x, im[e] - hf.y);
    }
    *reinterpret_cast<uint4*>(o.hi + idx) = *reinterpret_cast<const uint4*>(h);
    if (o.lo) *reinterpret_cast<uint4*>(o.lo + idx) = *reinterpret_cast<const uint4*>(l);
  }
  AFQ_D void tile(int b, int mt, int nt, const float* t, int ld, int tid) const {
    tile_part(b, mt, nt, t, ld, tid, 0, 256);
  }
  // the tile's columns [c_first, c_first + c_count) (whole block rows ii; c_count 128 or
  // 256) staged in t: block rows ii of the direct half, quarters of the mirrored half
  AFQ_D void tile_part(int, int mt, int nt, const float* t, int ld, int tid, int c_first,
                       int c_count) const {
    int tt = nt, ib = 0;   // tile -> block pair (ib, jb), ib <= jb, in row order
    const int nb = N >> 4;
    while (tt >= nb - ib) { tt -= nb - ib; ib++; }
    const int jb = ib + tt;
    const int r0 = c_first >> 4, nr = c_count >> 4;   // block rows ii in [r0, r0 + nr)
    const int q0 = r0 >> 2, nq = nr >> 2;            // their quarters of the mirrored rows
    const int per = 64 * nr * 4;                      // items of each half
    const int nitems = ib != jb ? 2 * per : per;
    // items: (walker, block row, quarter) of the direct half, then (walker, column jj,
    // quarter) of the mirrored half; quarter fastest, so four consecutive threads write
    // one 64-byte row
#pragma unroll 1
    for (int it = tid; it < nitems; it += 128) {
      const bool mir = it >= per;
      const int k = mir ? it - per : it;
      int wl, rr, qt;
      if (!mir) {
        qt = k & 3;
        rr = r0 + (k >> 2) % nr;
        wl = (k >> 2) / nr;
      } else {
        qt = q0 + k % nq;
        rr = (k / nq) & 15;
        wl = k / (nq * 16);
      }
      const int w = mt * 64 + wl;
      if (w >= nw) continue;
      const float* tr = t + (2 * wl) * ld;
      const float* ti = tr + ld;
      float re[4], im[4];
      long long row;
      if (!mir) {   // V[ib*16 + rr][jb*16 + 4 qt + e] = tile column rr*16 + 4 qt + e
#pragma unroll
        for (int e = 0; e < 4; e++) {
          re[e] = tr[rr * 16 + 4 * qt + e - c_first];
          im[e] = ti[rr * 16 + 4 * qt + e - c_first];
        }
        row = (long long)w * N * N + (long long)(ib * 16 + rr) * N + jb * 16 + 4 * qt;
      } else {      // V[jb*16 + rr][ib*16 + 4 qt + e] = tile column (4 qt + e)*16 + rr
#pragma unroll
        for (int e = 0; e < 4; e++) {
          re[e] = tr[(4 * qt + e) * 16 + rr - c_first];
          im[e] = ti[(4 * qt + e) * 16 + rr - c_first];
        }
        row = (long long)w * N * N + (long long)(jb * 16 + rr) * N + ib * 16 + 4 * qt;
      }
      put4(V, row * 2, re, im);
    }
  }
};

// split-K partial products part[z][m][n]
struct EpiPart {
  static constexpr bool kTile = false, kPair = false, kF16 = true;
  float* part;
  int M, Ncol;
  long long sz;
  AFQ_D void operator()(int z, int, int m, int n0, const float* v) const {
    if (m >= M) return;
    float* row = part + z * sz + (long long)m * Ncol;
#pragma unroll
    for (int i = 0; i < 32; i++)
      if (n0 + i < Ncol) row[n0 + i] = v[i];
  }
};

// Split-K partials with the accumulator promoted every PKB K slabs (persistent kernel).
template <int PKB>
struct EpiPartPromoted : EpiPart {
  static constexpr int kPromoteKB = PKB;
};

// Propagation products: tile rows i (orbital), columns [Re C | Im C] over the 2n walker
// columns.  mode 0: S = C (P W); mode 1: T = (i/k) C, S += T (Taylor term k; the last
// term forms S); mode 2: W = C (P S).  Modes 0 and 1 write the next B operand.
struct EpiProp {
  static constexpr bool kTile = true, kPair = false;
  int mode, k, last, N, n2;
  float2* S;     // Taylor sum [nw][n2][N] (orbital-major: lanes on consecutive rows)
  z_t* W;
  Op F;          // B form of the next product [nw][2*n2][2N]
  int real_next; // the next product has a real A operand (P S with real P): (Re | Im) rows
  AFQ_D void tile(int w, int mt, int, float* t, int ld, int tid) const {
    const int i0 = mt * 128;
    if (mode == 2) {   // walker layout [N][n2]: lanes on consecutive columns
      for (int e = tid; e < 128 * n2; e += 128) {
        const int r = e / n2, j = e % n2, i = i0 + r;
        if (i < N) W[(long long)w * N * n2 + (long long)i * n2 + j] = zmk(t[r * ld + j], t[r * ld + n2 + j]);
      }
      return;
    }
    const long long base = (long long)w * 2 * n2 * 2 * N;
    const float inv = mode == 1 ? 1.0f / (float)k : 0.0f;
    for (int e = tid; e < 128 * n2; e += 128) {
      const int j = e / 128, r = e % 128, i = i0 + r;
      if (i >= N) continue;
      float vr = t[r * ld + j], vi = t[r * ld + n2 + j];
      const long long o = (long long)w * N * n2 + (long long)j * N + i;
      if (mode == 0) {
        S[o] = make_float2(vr, vi);
      } else {
        const float tr = -vi * inv, ti = vr * inv;
        float2 sv = S[o];
        sv.x += tr;
        sv.y += ti;
        S[o] = sv;
        vr = last ? sv.x : tr;
        vi = last ? sv.y : ti;
      }
      if (real_next) {
        put1(F, base + (long long)j * 2 * N + i, vr);
        put1(F, base + (long long)(n2 + j) * 2 * N + i, vi);
      } else {
        put2(F, base + (long long)j * 2 * N + 2 * i, vr, -vi);
        put2(F, base + (long long)(n2 + j) * 2 * N + 2 * i, vi, vr);
      }
    }
  }
};

// The same propagation epilogue without a shared-memory tile, for 2n a multiple of 32:
// each thread receives Re C and Im C of 32 columns of its row.  S is updated in place
// and the next B operand is written with lanes on consecutive orbitals (coalesced).
struct EpiPropPair {
  static constexpr bool kTile = false, kPair = true;
  int mode, k, last, N, n2;
  float2* S;
  z_t* W;
  Op F;
  int real_next;
  AFQ_D int pair_stride() const { return n2; }
  AFQ_D void pair(int w, int, int i, int j0, const float* cr, const float* ci) const {
    if (i >= N) return;
    const long long row = (long long)w * N * n2 + (long long)i * n2;    // W[w][i][.]
    const long long scol = (long long)w * N * n2 + i;                   // S[w][.][i]
    const long long base = (long long)w * 2 * n2 * 2 * N;
    const float inv = mode == 1 ? 1.0f / (float)k : 0.0f;
    // the 32 loads of S first: stores to S and F below cannot be moved above them
    float2 sv[32];
    if (mode == 1) {
#pragma unroll
      for (int jj = 0; jj < 32; jj++) sv[jj] = S[scol + (long long)(j0 + jj) * N];
    }
#pragma unroll
    for (int jj = 0; jj < 32; jj++) {
      const int j = j0 + jj;
      float vr = cr[jj], vi = ci[jj];
      if (mode == 0) {
        S[scol + (long long)j * N] = make_float2(vr, vi);
      } else if (mode == 1) {
        const float tr = -vi * inv, ti = vr * inv;
        float2 s = sv[jj];
        s.x += tr;
        s.y += ti;
        S[scol + (long long)j * N] = s;
        vr = last ? s.x : tr;
        vi = last ? s.y : ti;
      } else {
        W[row + j] = zmk(vr, vi);
        continue;
      }
      if (real_next) {
        put1(F, base + (long long)j * 2 * N + i, vr);
        put1(F, base + (long long)(n2 + j) * 2 * N + i, vi);
        continue;
      }
      put2(F, base + (long long)j * 2 * N + 2 * i, vr, -vi);
      put2(F, base + (long long)(n2 + j) * 2 * N + 2 * i, vi, vr);
    }
  }
};

// The propagation epilogue of EpiPropPair for any even 2n, through the persistent kernel's
// staged interface: each thread owns one output row (orbital i of walker w) and takes
// Re C (columns j) and Im C (columns n2 + j) 32 j at a time.  TMEM loads stay on 32-column
// boundaries: when n2 is not a multiple of 32, the Im block [n2 + j0, n2 + j0 + 32) is
// gathered from the aligned chunks that cover it through the thread's own shared-memory
// row of 33 floats (written and read by that thread only).  Same arithmetic as
// EpiPropPair, so the same values.  With nwg epilogue warpgroups, warpgroup wg takes the
// 32-column blocks wg, wg + nwg, ... of every row.
struct EpiPropStaged {
  static constexpr bool kTile = false, kPair = false, kStaged = true;
  static constexpr int kScratchBytes = 128 * 33 * 4;
  int mode, k, last, N, n2;
  float2* S;
  z_t* W;
  Op F;
  int real_next;
  int nwg;
  template <class LD>
  AFQ_D void staged(int w, int mt, int, int row, LD& ld, float* scr, int wg) const {
    const int i = mt * 128 + row;
    float* my = scr + row * 33;
    const long long wrow = (long long)w * N * n2 + (long long)i * n2;   // W[w][i][.]
    const long long scol = (long long)w * N * n2 + i;                   // S[w][.][i]
    const long long base = (long long)w * 2 * n2 * 2 * N;
    const float inv = mode == 1 ? 1.0f / (float)k : 0.0f;
#pragma unroll 1
    for (int j0 = 32 * wg; j0 < n2; j0 += 32 * nwg) {
      float cr[32], ci[32];
      ld(j0, cr);
      const int need = min(32, n2 - j0);           // j in [j0, j0 + need)
      const int c = n2 + j0, a0 = c & ~31, off = c - a0;
      if (off == 0) {
        ld(a0, ci);
      } else {
        float t[32];
        ld(a0, t);
#pragma unroll
        for (int q = 0; q < 32; q++) my[q] = t[q];
#pragma unroll
        for (int jj = 0; jj < 32; jj++)
          if (jj < 32 - off) ci[jj] = my[off + jj];
        if (off + need > 32) {   // the block runs into the next aligned chunk
          ld(a0 + 32, t);
#pragma unroll
          for (int q = 0; q < 32; q++) my[q] = t[q];
#pragma unroll
          for (int jj = 0; jj < 32; jj++)
            if (jj >= 32 - off) ci[jj] = my[jj + off - 32];
        }
      }
      if (i >= N) continue;
      float2 sv[32];
      if (mode == 1) {
#pragma unroll
        for (int jj = 0; jj < 32; jj++)
          if (jj < need) sv[jj] = S[scol + (long long)(j0 + jj) * N];
      }
#pragma unroll
      for (int jj = 0; jj < 32; jj++) {
        if (jj >= need) continue;
        const int j = j0 + jj;
        float vr = cr[jj], vi = ci[jj];
        if (mode == 0) {
          S[scol + (long long)j * N] = make_float2(vr, vi);
        } else if (mode == 1) {
          const float tr = -vi * inv, ti = vr * inv;
          float2 s = sv[jj];
          s.x += tr;
          s.y += ti;
          S[scol + (long long)j * N] = s;
          vr = last ? s.x : tr;
          vi = last ? s.y : ti;
        } else {
          W[wrow + j] = zmk(vr, vi);
          continue;
        }
        if (real_next) {
          put1(F, base + (long long)j * 2 * N + i, vr);
          put1(F, base + (long long)(n2 + j) * 2 * N + i, vi);
          continue;
        }
        put2(F, base + (long long)j * 2 * N + 2 * i, vr, -vi);
        put2(F, base + (long long)(n2 + j) * 2 * N + 2 * i, vi, vr);
      }
    }
  }
};

// The last propagation product W = P S, written with the new walkers' packed forms
// (pair layout as EpiPropPair): the layouts their next consumers read, as the pack kernels
// form them from W, bit for bit (a float converted to double and back is unchanged).
// FA = the T1 operand (rows (re, -im)); F2 = the next P W operand ((re | im) rows when
// f2_real, else (re, -im) / (im, re) rows); lanes on consecutive orbitals i (coalesced).
// A functor of its own, so that the seven other products per substep keep their short
// epilogue (a longer one in the shared kernel slowed all of them).
struct EpiPropPack {
  static constexpr bool kTile = false, kPair = true;
  int N, n2;
  z_t* W;
  Op FA, F2;
  int f2_real;
  AFQ_D int pair_stride() const { return n2; }
  AFQ_D void pair(int w, int, int i, int j0, const float* cr, const float* ci) const {
    if (i >= N) return;
    const long long row = (long long)w * N * n2 + (long long)i * n2;    // W[w][i][.]
    const long long base = (long long)w * 2 * n2 * 2 * N;
#pragma unroll
    for (int jj = 0; jj < 32; jj++) {
      const int j = j0 + jj;
      const float vr = cr[jj], vi = ci[jj];
      W[row + j] = zmk(vr, vi);
      put2(FA, base + (long long)j * 2 * N + 2 * i, vr, -vi);
      if (f2_real) {
        put1(F2, base + (long long)j * 2 * N + i, vr);
        put1(F2, base + (long long)(n2 + j) * 2 * N + i, vi);
      } else {
        put2(F2, base + (long long)j * 2 * N + 2 * i, vr, -vi);
        put2(F2, base + (long long)(n2 + j) * 2 * N + 2 * i, vi, vr);
      }
    }
  }
};

// Epilogue of the fused propagation chain: EpiPropPair for P W and the Taylor terms,
// EpiPropPack for the last product; the active functor is copied locally per call so its
// fields stay in registers across the stores.
struct EpiChain {
  static constexpr bool kTile = false, kPair = true;
  int pack;
  EpiPropPair pr;
  EpiPropPack pk;
  AFQ_D int pair_stride() const { return pack ? pk.n2 : pr.n2; }
  AFQ_D void pair(int w, int r, int i, int j0, const float* cr, const float* ci) const {
    if (pack) {
      const EpiPropPack e = pk;
      e.pair(w, r, i, j0, cr, ci);
    } else {
      const EpiPropPair e = pr;
      e.pair(w, r, i, j0, cr, ci);
    }
  }
};

// Exchange: rows (cv, a), columns (wl, re|im, b); per (cv, wl) the trace of T^2 with
// T[a][b] = tile[cv*n + a][wl*2n + b] + i tile[cv*n + a][wl*2n + n + b].
struct EpiExchange {
  static constexpr bool kTile = true, kPair = false, kF16 = true;
  int n, Gn, Gw, nc, nw, nblk;
  z_t* Kpart;
  float ascale;           // scale of the Lh operand (1 for bf16)
  const float* wscale;    // per-walker scale of the G operand (null for bf16)
  AFQ_D void tile(int s, int mt, int nt, float* t, int ld, int tid) const {
    const int lane = tid & 31, warp = tid >> 5;
    for (int wl = warp; wl < Gw; wl += 4) {
      const int w = nt * Gw + wl;
      double sr = 0.0, si = 0.0;
      for (int cv = 0; cv < Gn; cv++) {
        if (mt * Gn + cv >= nc) break;
        const float* rows = t + (long long)cv * n * ld + wl * 2 * n;
        for (int q = lane; q < n * n; q += 32) {
          const int a = q / n, b = q % n;
          const double ar = rows[a * ld + b], ai = rows[a * ld + n + b];
          const double br = rows[b * ld + a], bi = rows[b * ld + n + a];
          sr += ar * br - ai * bi;
          si += ar * bi + ai * br;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
      }
      if (lane == 0 && w < nw) {
        const double u = 1.0 / ((double)ascale * (wscale ? (double)wscale[w] : 1.0));
        Kpart[((long long)w * 2 + s) * nblk + mt] = zmk(sr * u * u, si * u * u);
      }
    }
  }
};

// Exchange from the accumulator with per-walker staging (persistent kernel): for each
// walker of the tile its 2n columns go to shared memory, then all four warps share the
// trace sums of the tile's Cholesky vectors, added in fixed order.
template <int TWO_N>
struct EpiExchangeStaged {
  static constexpr bool kTile = false, kPair = false, kStaged = true, kF16 = true;
  static constexpr int LD = TWO_N + 1;
  static constexpr int kScratchBytes = 128 * LD * 4;
  int n, Gn, Gw, nc, nw, nblk;
  z_t* Kpart;
  float ascale;           // scale of the Lh operand (1 for bf16)
  const float* wscale;    // per-walker scale of the G operand (null for bf16)
  // epilogue warpgroups of the launch: warpgroup wg takes the tile's walkers wg, wg + nwg,
  // ... (with two, each keeps to one half of `red`; consecutive walkers of a warpgroup
  // reuse its half only after the barrier that follows the staging)
  int nwg = 1;
  template <class Ld>
  AFQ_D void staged(int s, int mt, int nt, int row, Ld& ld, float* scr, int wg) const {
    __shared__ double red[2][4][2];
    const int lane = row & 31, warp = row >> 5;
    const int ncv = min(Gn, nc - mt * Gn);
    for (int wl = wg; wl < Gw; wl += nwg) {
      float v[32];
#pragma unroll
      for (int q = 0; q < TWO_N / 32; q++) {
        ld(wl * TWO_N + q * 32, v);
#pragma unroll
        for (int i = 0; i < 32; i++) scr[row * LD + q * 32 + i] = v[i];
      }
      tc::epi_bar_group(wg);
      // thread `row` = (cv, a) sums T[a][b] T[b][a] over b: its own staged row and the
      // column a of the same Cholesky vector (both bank-conflict free, LD = 1 mod 32);
      // fp32 products over n terms, double across threads
      double sr = 0.0, si = 0.0;
      if (row < ncv * n) {
        const int cv = row / n, a = row - cv * n;
        const float* own = scr + row * LD;
        const float* col = scr + cv * n * LD + a;
        float fr = 0.0f, fi = 0.0f;
        for (int b = 0; b < n; b++) {
          const float ar = own[b], ai = own[n + b];
          const float br = col[b * LD], bi = col[b * LD + n];
          fr = fmaf(ar, br, fmaf(-ai, bi, fr));
          fi = fmaf(ar, bi, fmaf(ai, br, fi));
        }
        sr = fr;
        si = fi;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
      }
      if (lane == 0) {
        red[wl & 1][warp][0] = sr;
        red[wl & 1][warp][1] = si;
      }
      tc::epi_bar_group(wg);
      const int w = nt * Gw + wl;
      if (row == 0 && w < nw) {
        const double (*r)[2] = red[wl & 1];
        const double u = 1.0 / ((double)ascale * (wscale ? (double)wscale[w] : 1.0));
        Kpart[((long long)w * 2 + s) * nblk + mt] =
            zmk((((r[0][0] + r[1][0]) + r[2][0]) + r[3][0]) * u * u,
                (((r[0][1] + r[1][1]) + r[2][1]) + r[3][1]) * u * u);
      }
    }
  }
};

// Exchange from register-promoted accumulators (persistent kernel, two epilogue
// warpgroups, each owning BN / 2 columns = whole walkers): the K sum of T is chunked every
// PKB slabs and added in fp32 registers.  Per walker, thread (cv, a) then sums
// T[a][b] T[b][a] over b from its own row (registers) and column a of its Cholesky block,
// which passes through shared memory as the real, then the imaginary parts of half the
// block's rows at a time (scratch of 128 / n blocks x n / 2 rows x (n + 1) floats).
template <int TWO_N, int PKB>
struct EpiExchangePromoted {
  static constexpr bool kTile = false, kPair = false, kF16 = true, kRegs = true;
  static constexpr int kPromoteKB = PKB;
  static constexpr int NH = TWO_N / 2;       // n
  static constexpr int BW = NH / 2;          // rows of a block staged per pass
  static constexpr int GMAX = 128 / NH;      // Cholesky blocks of a tile
  static constexpr int LD = NH + 1;          // conflict-free column reads (LD odd)
  static constexpr int kScratchBytes = GMAX * BW * LD * 4;
  int n, Gn, Gw, nc, nw, nblk;
  z_t* Kpart;
  float ascale;
  const float* wscale;
  template <int CPW>
  AFQ_D void regs(int s, int mt, int nt, int row, const float (&acc)[CPW], float* scr,
                  int wg) const {
    if constexpr (CPW % TWO_N != 0) {
      return;   // not launched: the host requires whole walkers per warpgroup
    } else {
      constexpr int WPG = CPW / TWO_N;
      __shared__ double red[2][2][4][2];
      const int lane = row & 31, warp = row >> 5;
      const int ncv = min(Gn, nc - mt * Gn);
      const bool act = row < ncv * NH;
      const bool slot = row < GMAX * NH;
      const int cv = row / NH, a = row - cv * NH;
      const float* col = scr + cv * BW * LD + a;
#pragma unroll
      for (int q = 0; q < WPG; q++) {
        const float* re = acc + q * TWO_N;
        const float* im = re + NH;
        float fr = 0.0f, fi = 0.0f;
#pragma unroll
        for (int part = 0; part < 2; part++) {   // real, then imaginary rows
          const float* mine = part ? im : re;
#pragma unroll
          for (int rc = 0; rc < 2; rc++) {
            const int b0 = rc * BW;
            if (slot && a >= b0 && a < b0 + BW) {
              float* dst = scr + (cv * BW + a - b0) * LD;
#pragma unroll
              for (int c = 0; c < NH; c++) dst[c] = mine[c];
            }
            tc::epi_bar_group(wg);
            if (act) {
#pragma unroll
              for (int bb = 0; bb < BW; bb++) {
                const float v = col[bb * LD];
                if (part == 0) {
                  fr = fmaf(re[b0 + bb], v, fr);
                  fi = fmaf(im[b0 + bb], v, fi);
                } else {
                  fr = fmaf(-im[b0 + bb], v, fr);
                  fi = fmaf(re[b0 + bb], v, fi);
                }
              }
            }
            tc::epi_bar_group(wg);
          }
        }
        double sr = fr, si = fi;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          sr += __shfl_xor_sync(0xffffffffu, sr, o);
          si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (lane == 0) {
          red[wg][q & 1][warp][0] = sr;
          red[wg][q & 1][warp][1] = si;
        }
        tc::epi_bar_group(wg);
        const int w = nt * Gw + wg * WPG + q;
        if (row == 0 && w < nw) {
          const double (*r)[2] = red[wg][q & 1];
          const double u = 1.0 / ((double)ascale * (wscale ? (double)wscale[w] : 1.0));
          Kpart[((long long)w * 2 + s) * nblk + mt] =
              zmk((((r[0][0] + r[1][0]) + r[2][0]) + r[3][0]) * u * u,
                  (((r[0][1] + r[1][1]) + r[2][1]) + r[3][1]) * u * u);
        }
      }
    }
  }
};

// ------------------------------------------------------------ dispatch helpers
// The persistent kernel (double-buffered accumulator) runs every product whose epilogue
// needs no shared-memory tile; AFQ_TC_PERSISTENT=0 selects the per-tile kernel instead.
bool tc_persistent() {
  static const bool on = [] {   // initialised once, thread-safe
    const char* e = getenv("AFQ_TC_PERSISTENT");
    return !(e && atoi(e) == 0);
  }();
  return on;
}

// K slabs per promoted chunk: AFQ_PROMOTE="part=<k>,ex=<k>" (0 turns promotion off)
enum { PROMOTE_PART, PROMOTE_EXCHANGE };
int promote_kb(int which) {
  struct KB { int v[2]; };
  static const KB kb = [] {   // initialised once, thread-safe
    // C4 (NMO 384, 48+48 electrons, nchol 1536, 1024 walkers), same walkers as the FP64
    // form: E_J error 2e-6 Ha with part=2; E_K -1.4e-5 Ha with ex=1 (5.9 ms per 128-walker
    // subset), -2.7e-5 Ha with ex=2 (4.7 ms), -9.1e-5 Ha without promotion (4.4 ms)
    KB r{{2, 2}};
    if (const char* env = getenv("AFQ_PROMOTE")) {
      const std::string s(env);
      const size_t p = s.find("part="), q = s.find("ex=");
      if (p != std::string::npos) r.v[0] = atoi(s.c_str() + p + 5);
      if (q != std::string::npos) r.v[1] = atoi(s.c_str() + q + 3);
    }
    return r;
  }();
  return kb.v[which];
}

// Functors that may consume fp16 split operands (kF16) get that variant compiled.
template <class E, class = void> struct EpiF16 : std::false_type {};
template <class E>
struct EpiF16<E, std::void_t<decltype(E::kF16)>> : std::integral_constant<bool, E::kF16> {};

// Kernel variant of a product: 0 = the default rule (persistent unless the functor asks
// for the per-tile kernel or AFQ_TC_PERSISTENT=0), 1 = persistent, 2 = per-tile.  The
// set-up autotuner (mixed_tune) picks 1 or 2 per product site by timing both.
template <int BN, int ST, bool SPLIT, class Epi, int MINB = 1, int FMT = 1>
cudaError_t run_gemm(const tc::Maps& mp, const tc::GemmShape& g, const Epi& e, int* err,
                     cudaStream_t st, int variant = 0) {
  if constexpr (!Epi::kTile) {
    constexpr int PST = SPLIT ? 2 : 4;
    constexpr int WG = tc::EpiStaged<Epi>::value ? 1 : 2;
    constexpr bool only_persistent = tc::EpiStaged<Epi>::value || tc::EpiPromote<Epi>::value > 0;
    const bool persist = only_persistent || variant == 1 ||
                         (variant == 0 && tc_persistent() && !tc::EpiPerTile<Epi>::value);
    if (persist) {
      if constexpr (tc::PCfg<BN, PST, FMT, SPLIT, Epi, WG>::kFits)
        return tc::launch_persistent<BN, PST, FMT, SPLIT, Epi, WG>(mp, g, e, err, st);
      else
        return cudaErrorInvalidValue;
    }
  }
  if constexpr (tc::EpiStaged<Epi>::value || tc::EpiPromote<Epi>::value > 0) {
    return cudaErrorInvalidValue;
  } else {
    return tc::launch<BN, ST, FMT, SPLIT, Epi, MINB>(mp, g, e, err, st);
  }
}

// Stage counts: the default ring (4 plain / 2 split stages) keeps one CTA per SM busy;
// the lean ring (2 plain / 1 split) lets two CTAs share an SM so one's epilogue overlaps
// the other's main loop (used when the epilogue needs no shared-memory tile).
template <int BN, bool LEAN, class Epi>
cudaError_t run_prec(int prec, const tc::Maps& mp, const tc::GemmShape& g, const Epi& e, int* err,
                     cudaStream_t st, int variant) {
  if (prec == PREC_SPLIT16) {
    if constexpr (EpiF16<Epi>::value)
      return run_gemm<BN, (LEAN ? 1 : 2), true, Epi, (LEAN ? 2 : 1), 0>(mp, g, e, err, st, variant);
    else
      return cudaErrorInvalidValue;
  }
  if (prec == PREC_SPLIT)
    return run_gemm<BN, (LEAN ? 1 : 2), true, Epi, (LEAN ? 2 : 1)>(mp, g, e, err, st, variant);
  return run_gemm<BN, (LEAN ? 2 : 4), false, Epi, (LEAN ? 2 : 1)>(mp, g, e, err, st, variant);
}

template <bool LEAN = false, class Epi>
cudaError_t run_bn(int bn, int prec, const tc::Maps& mp, const tc::GemmShape& g, const Epi& e,
                   int* err, cudaStream_t st, int variant = 0) {
  switch (bn) {
    case 64: return run_prec<64, LEAN>(prec, mp, g, e, err, st, variant);
    case 128: return run_prec<128, LEAN>(prec, mp, g, e, err, st, variant);
    case 192: return run_prec<192, LEAN>(prec, mp, g, e, err, st, variant);
    case 256: return run_prec<256, LEAN>(prec, mp, g, e, err, st, variant);
  }
  return cudaErrorInvalidValue;
}

// the staged propagation epilogue on the persistent kernel, two epilogue warpgroups
template <int BN>
cudaError_t run_prop_staged(int prec, const tc::Maps& mp, const tc::GemmShape& g,
                            const EpiPropStaged& ep, int* err, cudaStream_t st) {
  if (prec == PREC_SPLIT)
    return tc::launch_persistent<BN, 2, 1, true, EpiPropStaged, 2>(mp, g, ep, err, st);
  if (prec == PREC_BF16)
    return tc::launch_persistent<BN, 4, 1, false, EpiPropStaged, 2>(mp, g, ep, err, st);
  return cudaErrorInvalidValue;
}

// propagation product with the pair epilogue when 2n is a multiple of 32; for any other
// 2n the staged epilogue on the persistent kernel (kernel choice 0 or 1) or the
// shared-memory tile epilogue on the per-tile kernel (choice 2): the same values
cudaError_t run_prop(MixedState* m, int prec, const tc::Maps& mp, const tc::GemmShape& g, int mode,
                     int k, int last, z_t* W, const Op& F, cudaStream_t st, int fa_buf = -1) {
  const int n2 = 2 * m->n;
  if (n2 % 32 == 0) {
    if (mode == 2 && fa_buf >= 0) {   // the new walkers' packed forms as well
      EpiPropPack ep{m->N, n2, W, m->F[fa_buf], m->F2, (m->preal && m->in.order >= 1) ? 1 : 0};
      return run_bn<true>(m->bn_prop, prec, mp, g, ep, m->err, st, m->tune[TS_PROP]);
    }
    EpiPropPair ep{mode, k, last, m->N, n2, m->S, W, F, (last && m->preal) ? 1 : 0};
    return run_bn<true>(m->bn_prop, prec, mp, g, ep, m->err, st, m->tune[TS_PROP]);
  }
  if (m->tune[TS_PROP] != 2 && tc_persistent()) {
    EpiPropStaged ep{mode, k, last, m->N, n2, m->S, W, F, (last && m->preal) ? 1 : 0, 2};
    switch (m->bn_prop) {
      case 64: return run_prop_staged<64>(prec, mp, g, ep, m->err, st);
      case 128: return run_prop_staged<128>(prec, mp, g, ep, m->err, st);
      case 192: return run_prop_staged<192>(prec, mp, g, ep, m->err, st);
      case 256: return run_prop_staged<256>(prec, mp, g, ep, m->err, st);
    }
    return cudaErrorInvalidValue;
  }
  EpiProp ep{mode, k, last, m->N, n2, m->S, W, F, (last && m->preal) ? 1 : 0};
  return run_bn(m->bn_prop, prec, mp, g, ep, m->err, st, m->tune[TS_PROP]);
}

int pick_bn(int cols) {
  if (cols <= 64) return 64;
  if (cols <= 128) return 128;
  if (cols <= 192) return 192;
  if (cols <= 256) return 256;
  return 0;
}

// sp slices of the vbias / Coulomb K (a multiple of 64 each; fewer when K is short)
void set_splits(MixedState* m, int sp) {
  const long long Kq = m->greal ? m->NAK : 2 * m->NAK;
  sp = std::max(1, std::min(32, sp));
  long long ks = (Kq + sp - 1) / sp;
  ks = (ks + 63) / 64 * 64;
  m->splits = (int)((Kq + ks - 1) / ks);
  m->ksplit = (int)ks;
}

bool map2(tc::Maps& mp, const Op& a, uint64_t Ka, uint64_t ra, uint64_t ba, uint64_t lda,
          uint64_t sa, const Op& b, uint64_t Kb, uint64_t rb, uint64_t bb, uint64_t ldb,
          uint64_t sb, uint32_t bn, uint32_t slab = 128) {
  return tc::make_kmajor_map(&mp.a, a.hi, false, Ka, ra, ba, lda, sa, 128, slab) == CUDA_SUCCESS &&
         tc::make_kmajor_map(&mp.a_lo, a.lo, false, Ka, ra, ba, lda, sa, 128, slab) == CUDA_SUCCESS &&
         tc::make_kmajor_map(&mp.b, b.hi, false, Kb, rb, bb, ldb, sb, bn, slab) == CUDA_SUCCESS &&
         tc::make_kmajor_map(&mp.b_lo, b.lo, false, Kb, rb, bb, ldb, sb, bn, slab) == CUDA_SUCCESS;
}

void parse_prec(MixedState* m) {
  // e.g. "vhs=1,p=1,v1=1,vk=0,vbias=2,ej=2,ek=2" (0 plain bf16, 1 bf16 split, 2 fp16 split;
  // fp16 split applies to vbias / ej / ek only)
  const char* env = getenv("AFQ_MIXED_PREC");
  if (!env) return;
  std::string s(env);
  auto get = [&](const char* key, int& dst) {
    std::string k = std::string(key) + "=";
    size_t p = s.find(k);
    if (p != std::string::npos) {
      const int v = atoi(s.c_str() + p + k.size());
      dst = v == 2 ? PREC_SPLIT16 : v ? PREC_SPLIT : PREC_BF16;
    }
  };
  get("vhs", m->prec_vhs); get("p", m->prec_p); get("v1", m->prec_v1); get("vk", m->prec_vk);
  get("vbias", m->prec_vbias); get("ej", m->prec_ej); get("ek", m->prec_ek);
}

}  // namespace

// ------------------------------------------------------------ public entry points
static cudaError_t mixed_tune(MixedState* m, cudaStream_t st);

cudaError_t mixed_create(const MixedInit* init, MixedState** out, std::string* msg,
                         cudaStream_t st) {
  *out = nullptr;
  MixedState* m = new MixedState();
  m->in = *init;
  m->N = init->N; m->n = init->n; m->nc = init->nchol; m->nw = init->nw;
  m->NAK = 2LL * m->n * m->N;
  const int N = m->N, n = m->n, nc = m->nc, nw = m->nw;
  const long long NAK = m->NAK;
  parse_prec(m);
  auto bail = [&](cudaError_t e, const std::string& why) {
    if (msg) *msg = why;
    mixed_destroy(m);
    return e == cudaSuccess ? cudaErrorInvalidValue : e;
  };
  // vbias and E_J share the G operand Gb: one format for both
  if (m->prec_vbias == PREC_SPLIT16 || m->prec_ej == PREC_SPLIT16)
    m->prec_vbias = m->prec_ej = PREC_SPLIT16;
  m->bn_prop = pick_bn(4 * n);
  if (!m->bn_prop) return bail(cudaSuccess, "4*NAEA exceeds 256");
  if (!init->SpvnT_dense) return bail(cudaSuccess, "SpvnT below the dense threshold");
  if ((2 * N) % 8 || (2 * NAK) % 8) return bail(cudaSuccess, "operand rows must be 16-byte multiples");
  m->s_real = init->sp_rv != nullptr;
  m->Kv = m->s_real ? nc : 2 * nc;
  if (m->Kv % 8) return bail(cudaSuccess, "nchol must be a multiple of 8 (4 for complex Spvn)");
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  A(alloc_op(m, m->Sd, (size_t)N * N * m->Kv));
  A(alloc_op(m, m->Pf, (size_t)N * 2 * N));
  A(alloc_op(m, m->SpT, (size_t)nc * 2 * NAK));
  A(alloc_op(m, m->Xf, (size_t)2 * nw * m->Kv));
  A(alloc_op(m, m->Vf, (size_t)nw * N * 2 * N));
  A(alloc_op(m, m->F[0], (size_t)nw * 4 * n * 2 * N));
  A(alloc_op(m, m->F[1], (size_t)nw * 4 * n * 2 * N));
  A(alloc_op(m, m->Gb, (size_t)2 * nw * 2 * NAK));
  A(malloc_track(m, &m->S, (size_t)nw * N * 2 * n));
  A(malloc_track(m, &m->err, 1));
  if ((2 * n) % 32 == 0) A(malloc_track(m, &m->dep, (size_t)nw));   // fused chain counters
  A(malloc_track(m, &m->wscale, nw));
  A(malloc_track(m, &m->dmax, 2));
  A(alloc_op(m, m->F2, (size_t)nw * 4 * n * 2 * N));
  if (init->trial) {
    A(alloc_op(m, m->TwB, (size_t)4 * n * 2 * N));
    A(alloc_op(m, m->Wn, (size_t)nw * N * 4 * n));
    A(alloc_op(m, m->Tinv, (size_t)nw * 2 * 2 * n * 2 * n));
    A(malloc_track(m, &m->T1, (size_t)nw * 2 * n * n));
  }
  if (init->Lh) {
    A(alloc_op(m, m->LhJ, (size_t)nc * 2 * NAK));
    A(alloc_op(m, m->LhX, (size_t)nc * 2 * NAK));
    A(alloc_op(m, m->Gx, (size_t)nw * 2 * NAK * 2));
  }
  // real half-rotated operands?
  if (e == cudaSuccess && !getenv("AFQ_MIXED_COMPLEX")) {
    A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
    check_imag_kernel<<<148 * 8, 256, 0, st>>>(init->SpvnT_dense, (long long)nc * NAK, m->err);
    if (init->Lh) check_imag_kernel<<<148 * 8, 256, 0, st>>>(init->Lh, (long long)nc * NAK, m->err);
    int cplx = 1;
    A(cudaGetLastError());
    A(cudaMemcpyAsync(&cplx, m->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    A(cudaStreamSynchronize(st));
    m->greal = e == cudaSuccess && !cplx;
    A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
    check_imag_kernel<<<148 * 8, 256, 0, st>>>(init->P, (long long)N * N, m->err);
    cplx = 1;
    A(cudaGetLastError());
    A(cudaMemcpyAsync(&cplx, m->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    A(cudaStreamSynchronize(st));
    m->preal = e == cudaSuccess && !cplx && init->order >= 1;
    A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
  }
  // fp16 split G products: power-of-two scales of the static operands from their ranges
  if (e == cudaSuccess) {
    const bool gb16 = m->prec_vbias == PREC_SPLIT16, gx16 = m->prec_ek == PREC_SPLIT16;
    if (gb16 || gx16) {
      A(cudaMemsetAsync(m->dmax, 0, 2 * sizeof(double), st));
      unsigned long long* dm = reinterpret_cast<unsigned long long*>(m->dmax);
      maxabs_kernel<<<148 * 4, 256, 0, st>>>(init->SpvnT_dense, (long long)nc * NAK, dm);
      if (init->Lh) maxabs_kernel<<<148 * 4, 256, 0, st>>>(init->Lh, (long long)nc * NAK, dm + 1);
      double hm[2] = {0.0, 0.0};
      A(cudaGetLastError());
      A(cudaMemcpyAsync(hm, m->dmax, sizeof(hm), cudaMemcpyDeviceToHost, st));
      A(cudaStreamSynchronize(st));
      m->sSpT = pow2_scale(hm[0]);
      m->sLh = pow2_scale(hm[1]);
    }
    m->SpT.f16 = m->Gb.f16 = gb16 ? 1 : 0;
    m->SpT.scale = gb16 ? m->sSpT : 1.0f;
    if (init->Lh) {
      m->LhJ.f16 = gb16 ? 1 : 0;
      m->LhJ.scale = gb16 ? m->sLh : 1.0f;
      m->LhX.f16 = m->Gx.f16 = gx16 ? 1 : 0;
      m->LhX.scale = gx16 ? m->sLh : 1.0f;
    }
  }
  // split K of the vbias / Coulomb products so the grid covers the GPU (about four tiles
  // per SM); the tuner also tries half and twice as many slices
  {
    const int tiles = ((nc + 127) / 128) * ((2 * nw + 127) / 128);
    set_splits(m, std::max(1, std::min(16, (int)((4 * 148 + tiles - 1) / tiles))));
    m->splits0 = m->splits;
    const int ks = m->ksplit;
    const char* fs = getenv("AFQ_SPLITK");   // forced slice count
    set_splits(m, std::max(2 * m->splits0, fs ? atoi(fs) : 0));
    m->part_cap = m->splits;
    m->splits = m->splits0;
    m->ksplit = ks;
    A(malloc_track(m, &m->part, (size_t)m->part_cap * nc * 2 * nw));
  }
  if (e != cudaSuccess) return bail(e, "allocation");
  A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
  A(cudaMemsetAsync(m->Sd.hi, 0, sizeof(bf16) * (size_t)N * N * m->Kv, st));
  A(cudaMemsetAsync(m->Sd.lo, 0, sizeof(bf16) * (size_t)N * N * m->Kv, st));
  pack_spvn_kernel<<<(N * N + 7) / 8, dim3(32, 8), 0, st>>>(init->sp_ri, init->sp_ci, init->sp_v,
                                                            init->sp_rv, N * N, m->Kv, m->s_real,
                                                            m->Sd);
  if (m->preal)
    pack_real_kernel<<<grid_for((long long)N * N), 256, 0, st>>>(init->P, (long long)N * N, m->Pf);
  else
    pack_complex_kernel<<<grid_for((long long)N * N), 256, 0, st>>>(init->P, (long long)N * N, m->Pf);
  if (m->greal)
    pack_real_kernel<<<grid_for((long long)nc * NAK), 256, 0, st>>>(init->SpvnT_dense,
                                                                   (long long)nc * NAK, m->SpT);
  else
    pack_complex_kernel<<<grid_for((long long)nc * NAK), 256, 0, st>>>(init->SpvnT_dense,
                                                                      (long long)nc * NAK, m->SpT);
  for (int i = 0; i < 2; i++) {   // rows the products read past their data stay finite
    A(cudaMemsetAsync(m->F[i].hi, 0, sizeof(bf16) * (size_t)nw * 4 * n * 2 * N, st));
    A(cudaMemsetAsync(m->F[i].lo, 0, sizeof(bf16) * (size_t)nw * 4 * n * 2 * N, st));
  }
  if (init->trial) {
    A(cudaMemsetAsync(m->TwB.hi, 0, sizeof(bf16) * (size_t)4 * n * 2 * N, st));
    A(cudaMemsetAsync(m->TwB.lo, 0, sizeof(bf16) * (size_t)4 * n * 2 * N, st));
    pack_trial_kernel<<<grid_for((long long)N * 2 * n), 256, 0, st>>>(init->trial, N, 2 * n, m->TwB);
  }
  if (init->Lh && m->greal) {
    pack_real_kernel<<<grid_for((long long)nc * NAK), 256, 0, st>>>(init->Lh, (long long)nc * NAK,
                                                                   m->LhJ);
    pack_lhx_real_kernel<<<grid_for((long long)nc * NAK), 256, 0, st>>>(init->Lh, nc, n, N, m->LhX);
  } else if (init->Lh) {
    pack_complex_kernel<<<grid_for((long long)nc * NAK), 256, 0, st>>>(init->Lh, (long long)nc * NAK,
                                                                      m->LhJ);
    pack_lhx_kernel<<<grid_for((long long)nc * NAK), 256, 0, st>>>(init->Lh, nc, n, N, m->LhX);
  }
  A(cudaGetLastError());
  A(cudaStreamSynchronize(st));
  if (e != cudaSuccess) return bail(e, "packing");
  // symmetric Cholesky vectors: keep only the 16 x 16 block pairs ib <= jb
  if (N % 16 == 0 && !getenv("AFQ_VHS_FULL")) {
    A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
    check_sym_kernel<<<148 * 8, 256, 0, st>>>(m->Sd, N, m->Kv, m->err);
    int asym = 1;
    A(cudaGetLastError());
    A(cudaMemcpyAsync(&asym, m->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    A(cudaStreamSynchronize(st));
    A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
    if (e == cudaSuccess && !asym) {
      const int nb = N / 16;
      std::vector<int> hp;
      for (int ib = 0; ib < nb; ib++)
        for (int jb = ib; jb < nb; jb++) hp.push_back(ib << 16 | jb);
      m->npairs = (int)hp.size();
      Op sym;
      A(malloc_track(m, &m->pairs, hp.size()));
      A(alloc_op(m, sym, (size_t)m->npairs * 256 * m->Kv));
      A(cudaMemcpyAsync(m->pairs, hp.data(), sizeof(int) * hp.size(), cudaMemcpyHostToDevice, st));
      if (e == cudaSuccess)
        pack_sym_kernel<<<148 * 8, 256, 0, st>>>(m->Sd, N, m->Kv, m->pairs, m->npairs, sym);
      A(cudaGetLastError());
      A(cudaStreamSynchronize(st));
      if (e != cudaSuccess) return bail(e, "symmetric Spvn packing");
      // the full dense operand was a set-up temporary
      for (void* q : {(void*)m->Sd.hi, (void*)m->Sd.lo}) {
        m->allocs.erase(std::find(m->allocs.begin(), m->allocs.end(), q));
        cudaFree(q);
      }
      m->Sd = sym;
      m->vsym = true;
    }
  }
  // tensor maps
  bool ok = true;
  const int bnv = 256;
  const uint64_t vrows = m->vsym ? (uint64_t)m->npairs * 256 : (uint64_t)N * N;
  ok &= map2(m->m_vhs, m->Xf, m->Kv, 2 * nw, 1, m->Kv, 0, m->Sd, m->Kv, vrows, 1, m->Kv, 0, bnv);
  ok &= map2(m->m_vhs64, m->Xf, m->Kv, 2 * nw, 1, m->Kv, 0, m->Sd, m->Kv, vrows, 1, m->Kv, 0, bnv,
             64);
  const uint64_t fr = 4 * n, fsz = (uint64_t)4 * n * 2 * N;
  {
    const uint64_t Kp = m->preal ? N : 2 * N;
    ok &= map2(m->m_pw2, m->Pf, Kp, N, 1, Kp, 0, m->F2, Kp, fr, nw, 2 * N, fsz, m->bn_prop);
  }
  for (int i = 0; i < 2; i++) {
    const uint64_t Kp = m->preal ? N : 2 * N;
    ok &= map2(m->m_pw[i], m->Pf, Kp, N, 1, Kp, 0, m->F[i], Kp, fr, nw, 2 * N, fsz, m->bn_prop);
    ok &= map2(m->m_v[i], m->Vf, 2 * N, N, nw, 2 * N, (uint64_t)N * 2 * N, m->F[i], 2 * N, fr, nw,
               2 * N, fsz, m->bn_prop);
  }
  const uint64_t Kg = m->greal ? NAK : 2 * NAK;   // K of the vbias / Coulomb products
  const uint64_t Kx = m->greal ? N : 2 * N;       // K of the exchange product
  ok &= map2(m->m_vbias, m->SpT, Kg, nc, 1, Kg, 0, m->Gb, Kg, 2 * nw, 1, Kg, 0,
             128);
  if (init->Lh) {
    ok &= map2(m->m_ej, m->LhJ, Kg, nc, 1, Kg, 0, m->Gb, Kg, 2 * nw, 1, Kg, 0,
               128);
    m->ex_Gn = 128 / n;
    m->ex_Gw = std::max(1, 256 / (2 * n));
    while (m->ex_Gw > 1 && !pick_bn(m->ex_Gw * 2 * n)) m->ex_Gw--;
    m->ex_bn = pick_bn(m->ex_Gw * 2 * n);
    // the tile must hold whole walkers: use the exact width when it is a compiled size
    if (m->ex_bn != m->ex_Gw * 2 * n) {
      int gw = m->ex_Gw;
      while (gw > 1 && pick_bn(gw * 2 * n) != gw * 2 * n) gw--;
      if (pick_bn(gw * 2 * n) == gw * 2 * n) { m->ex_Gw = gw; m->ex_bn = gw * 2 * n; }
    }
    m->ex_mtiles = (nc + m->ex_Gn - 1) / m->ex_Gn;
    ok &= map2(m->m_ek, m->LhX, Kx, (uint64_t)nc * n, 2, Kx, (uint64_t)nc * n * Kx, m->Gx, Kx,
               (uint64_t)nw * 2 * n, 2, Kx, (uint64_t)nw * 2 * n * Kx, m->ex_bn);
    if (2 * n == 80) {
      m->ex80 = map2(m->m_ek80, m->LhX, Kx, (uint64_t)nc * n, 2, Kx, (uint64_t)nc * n * Kx, m->Gx,
                     Kx, (uint64_t)nw * 2 * n, 2, Kx, (uint64_t)nw * 2 * n * Kx, 160);
      ok &= m->ex80;
    }
  }
  if (init->trial && n <= 64) {
    m->bn_t1 = pick_bn(4 * n);
    m->bn_gc = pick_bn(2 * n);
    const uint64_t fr = 4 * n, fsz = (uint64_t)4 * n * 2 * N;
    ok &= map2(m->m_t1, m->F[0], 2 * N, fr, nw, 2 * N, fsz, m->TwB, 2 * N, 4 * n, 1, 2 * N, 0,
               m->bn_t1);
    ok &= map2(m->m_t1_1, m->F[1], 2 * N, fr, nw, 2 * N, fsz, m->TwB, 2 * N, 4 * n, 1, 2 * N, 0,
               m->bn_t1);
    for (int sp = 0; sp < 2; sp++) {
      Op a{m->Wn.hi + 2 * n * sp, m->Wn.lo + 2 * n * sp};
      Op b{m->Tinv.hi + (size_t)sp * 2 * n * 2 * n, m->Tinv.lo + (size_t)sp * 2 * n * 2 * n};
      ok &= map2(m->m_gc[sp], a, 2 * n, N, nw, 4 * n, (uint64_t)N * 4 * n, b, 2 * n, 2 * n, nw,
                 2 * n, (uint64_t)2 * 2 * n * 2 * n, m->bn_gc);
    }
  }
  if (!ok) return bail(cudaSuccess, "tensor map encoding failed");
  if ((e = mixed_tune(m, st)) != cudaSuccess) return bail(e, "kernel tuning");
  *out = m;
  return cudaSuccess;
}

void mixed_destroy(MixedState* m) {
  if (!m) return;
  for (void* p : m->allocs) cudaFree(p);
  delete m;
}

int mixed_nblk(const MixedState* m) { return m ? m->ex_mtiles : 0; }

// Timeout flags of the tensor-core kernels since the last call; reading clears them, so
// one failed call does not condemn the calls after it.
cudaError_t mixed_error(MixedState* m, int* flags) {
  cudaError_t e = cudaMemcpy(flags, m->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && *flags) e = cudaMemset(m->err, 0, sizeof(int));
  return e;
}

cudaError_t mixed_set_wait_clocks(long long clocks) { return tc::set_wait_clocks(clocks); }

int mixed_launches(const MixedState* m, int stage) {
  switch (stage) {
    case 1: return 3;                                  // pack, GEMM, reduce (vbias)
    case 3: return 2;                                  // pack, GEMM (vHS)
    // the walker packs drop out while the packed forms are current (m->packed at the call)
    case 4: {   // [pack], then per walker group P W, terms, P S (one launch when fused)
      if (m->chain_wave > 0) return (m->packed ? 0 : 1) + 1;
      const int G = m->prop_group > 0 && m->prop_group < m->nw ? m->prop_group : m->nw;
      return (m->packed ? 0 : 1) + ((m->nw + G - 1) / G) * (m->in.order + 2);
    }
    case 8: return m->in.Lh ? 4 : 0;                   // pack, E_J GEMM, reduce, E_K GEMM
    case 0: return m->packed ? 5 : 6;                  // [pack], T1, LU, pack, Gc x 2
    case 5: return m->packed ? 2 : 3;                  // [pack], T1, LU (overlaps)
  }
  return 0;
}

// V = X^T Spvn of every walker from the packed fields Xf
static cudaError_t vhs_product(MixedState* m, cudaStream_t st) {
  const int nw = m->nw, N = m->N;
  if (m->vsym) {
    tc::GemmShape g{2 * nw, m->npairs * 256, m->Kv, 1, 128, (2 * nw + 127) / 128, false, false, 0,
                    true};
    if (m->vhs_epi == 1) {
      EpiVhsSymTile epi{m->Vf, nw, N, m->pairs};
      return run_bn(256, m->prec_vhs, m->m_vhs, g, epi, m->err, st, 2);
    }
    if (m->vhs_epi == 2 || m->vhs_epi == 3) {   // two CTAs per SM: one overlaps the other's epilogue
      EpiVhsSymTile epi{m->Vf, nw, N, m->pairs};
      if (m->vhs_epi == 3 && m->prec_vhs == PREC_SPLIT)   // two 48 KB stages of 64-byte slabs
        return tc::launch<256, 2, 1, true, EpiVhsSymTile, 2, 64>(m->m_vhs64, g, epi, m->err, st);
      if (m->vhs_epi == 3) return cudaErrorInvalidValue;
      if (m->prec_vhs == PREC_SPLIT)
        return tc::launch<256, 1, 1, true, EpiVhsSymTile, 2>(m->m_vhs, g, epi, m->err, st);
      if (m->prec_vhs == PREC_BF16)
        return tc::launch<256, 2, 1, false, EpiVhsSymTile, 2>(m->m_vhs, g, epi, m->err, st);
      return cudaErrorInvalidValue;
    }
    EpiVhsSym epi{m->Vf, nw, N, m->pairs};
    return run_bn(256, m->prec_vhs, m->m_vhs, g, epi, m->err, st, m->tune[TS_VHS]);
  }
  tc::GemmShape g{2 * nw, N * N, m->Kv, 1, 128, (2 * nw + 127) / 128, false, false, 0, true};
  EpiVhs epi{m->Vf, nw, (long long)N * N};
  return run_bn(256, m->prec_vhs, m->m_vhs, g, epi, m->err, st, m->tune[TS_VHS]);
}

cudaError_t mixed_vhs_pack(MixedState* m, const z_t* X, cudaStream_t st) {
  const int nc = m->nc, nw = m->nw;
  pack_x_kernel<<<dim3((nc + 31) / 32, (nw + 31) / 32), dim3(32, 8), 0, st>>>(X, nc, nw, m->Kv,
                                                                             m->s_real, m->Xf);
  return cudaGetLastError();
}

cudaError_t mixed_vhs(MixedState* m, const z_t* X, z_t*, cudaStream_t st) {
  cudaError_t e = mixed_vhs_pack(m, X, st);
  if (e != cudaSuccess) return e;
  return vhs_product(m, st);
}

cudaError_t mixed_unpack_vhs(MixedState* m, z_t* vHS, cudaStream_t st) {
  const long long cnt = (long long)m->nw * m->N * m->N;
  unpack_v_kernel<<<grid_for(cnt), 256, 0, st>>>(m->Vf, cnt, vHS);
  return cudaGetLastError();
}

// B operand of the next product: the lo part only when that product runs split
static Op next_op(const Op& F, int prec) { return prec == PREC_SPLIT ? F : Op{F.hi, nullptr}; }

// The whole propagation chain as one cooperative persistent launch (tc::launch_chain):
// P W, the Taylor terms and P S over walker waves of `wave` walkers, a product's tile of
// walker w starting once every tile of the previous product of w has published; the same
// tiles, MMA order and epilogue arithmetic as the eight launches, so the same walkers.
// timing (W unused, may be null): no pack of W, and the last product writes S and an
// operand (as the tuner's eight-launch timing does) instead of the walkers and their
// packed forms.
using ChainJob = tc::PJob<EpiChain, 8>;
static cudaError_t propagate_chain(MixedState* m, z_t* W, int wave, bool timing,
                                   cudaStream_t st) {
  const int N = m->N, n2 = 2 * m->n, nw = m->nw, order = m->in.order;
  if (n2 % 32 || !m->dep || order + 2 > 8 || wave < 1) return cudaErrorInvalidValue;
  for (int p : {m->prec_p, m->prec_v1, m->prec_vk})
    if (p != PREC_SPLIT && p != PREC_BF16) return cudaErrorInvalidValue;
  const bool pr = m->preal && order >= 1;
  const bool from_f2 = !timing && m->packed;   // the P W operand is in F2 already
  if (!timing) m->packed = false;
  cudaError_t e;
  if (!from_f2 && !timing) {
    pack_w_kernel<<<dim3((N + 31) / 32, (n2 + 31) / 32, nw), dim3(32, 8), 0, st>>>(
        W, N, n2, m->F[0], pr ? 2 : 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  ChainJob job{};
  const int mt = (N + 127) / 128, ntl = (2 * n2 + m->bn_prop - 1) / m->bn_prop;
  const int Kp = pr ? N : 2 * N;
  auto add = [&](int p, const tc::Maps& mp, const EpiChain& ep, int K, int a_batched, int prec) {
    job.maps[p] = mp;
    job.epi[p] = ep;
    job.sched[p] = tc::TileSched{mt, ntl, nw, 0, 0};
    job.K[p] = K;
    job.m_step[p] = 128;
    job.n_step[p] = m->bn_prop;
    job.a_batched[p] = a_batched;
    job.b_batched[p] = 1;
    job.k_split[p] = 0;
    job.bn[p] = m->bn_prop;
    job.split[p] = prec == PREC_SPLIT ? 1 : 0;
  };
  add(0, from_f2 ? m->m_pw2 : m->m_pw[0],
      EpiChain{0, EpiPropPair{0, 0, 0, N, n2, m->S, W, next_op(m->F[1], m->prec_v1), 0}, {}}, Kp,
      0, m->prec_p);
  int cur = 1;
  for (int k = 1; k <= order; k++) {  // T_k = (i/k) V T_{k-1}; S += T_k
    const int prec = k == 1 ? m->prec_v1 : m->prec_vk;
    const int nprec = k < order ? m->prec_vk : m->prec_p;
    add(k, m->m_v[cur],
        EpiChain{0, EpiPropPair{1, k, k == order ? 1 : 0, N, n2, m->S, W,
                                next_op(m->F[cur ^ 1], nprec), (k == order && m->preal) ? 1 : 0},
                 {}},
        2 * N, 1, prec);
    cur ^= 1;
  }
  if (timing)
    add(order + 1, m->m_pw[cur],
        EpiChain{0, EpiPropPair{0, 0, 0, N, n2, m->S, W, next_op(m->F[cur ^ 1], m->prec_p), 0}, {}},
        Kp, 0, m->prec_p);
  else   // W = P S with the new walkers' packed forms
    add(order + 1, m->m_pw[cur],
        EpiChain{1, {}, EpiPropPack{N, n2, W, m->F[cur ^ 1], m->F2, pr ? 1 : 0}}, Kp, 0,
        m->prec_p);
  job.np = order + 2;
  job.dep = m->dep;
  job.wave = wave;
  job.nbatch = nw;
  if ((e = cudaMemsetAsync(m->dep, 0, sizeof(unsigned) * nw, st)) != cudaSuccess) return e;
  switch (m->bn_prop) {
    case 64: e = tc::launch_chain<64, 2, 1, EpiChain, 2, 8>(job, m->err, st); break;
    case 128: e = tc::launch_chain<128, 2, 1, EpiChain, 2, 8>(job, m->err, st); break;
    case 192: e = tc::launch_chain<192, 2, 1, EpiChain, 2, 8>(job, m->err, st); break;
    case 256: e = tc::launch_chain<256, 2, 1, EpiChain, 2, 8>(job, m->err, st); break;
    default: e = cudaErrorInvalidValue;
  }
  if (e == cudaSuccess && !timing && m->Wn.hi) {
    m->packed = true;
    m->fa_buf = cur ^ 1;
  }
  return e;
}

cudaError_t mixed_propagate(MixedState* m, z_t* W, const z_t*, cudaStream_t st) {
  if (m->chain_wave > 0) return propagate_chain(m, W, m->chain_wave, false, st);
  const int N = m->N, n2 = 2 * m->n, nw = m->nw;
  const bool pr = m->preal && m->in.order >= 1;
  const bool from_f2 = m->packed;   // the P W operand of these walkers is in F2 already
  m->packed = false;
  cudaError_t e;
  if (!from_f2) {
    pack_w_kernel<<<dim3((N + 31) / 32, (n2 + 31) / 32, nw), dim3(32, 8), 0, st>>>(
        W, N, n2, m->F[0], pr ? 2 : 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  const int mt = (N + 127) / 128;
  const int Kp = pr ? N : 2 * N;   // K of P W and P S
  // walker groups: every product of the chain over one group before the next group (the
  // same tiles and epilogues as one launch over all walkers, in another order)
  const int G = m->prop_group > 0 && m->prop_group < nw ? m->prop_group : nw;
  int cur = 0;
  for (int z0 = 0; z0 < nw; z0 += G) {
    const int gb = std::min(G, nw - z0);
    cur = 0;
    {  // S = P W
      tc::GemmShape g{N, 2 * n2, Kp, gb, 128, mt, false, true, 0};
      g.z0 = z0;
      if ((e = run_prop(m, m->prec_p, from_f2 ? m->m_pw2 : m->m_pw[0], g, 0, 0, 0, nullptr,
                        next_op(m->F[1], m->prec_v1), st)) != cudaSuccess)
        return e;
      cur = 1;
    }
    for (int k = 1; k <= m->in.order; k++) {  // T_k = (i/k) V T_{k-1}; S += T_k
      tc::GemmShape g{N, 2 * n2, 2 * N, gb, 128, mt, true, true, 0};
      g.z0 = z0;
      int prec = k == 1 ? m->prec_v1 : m->prec_vk;
      const int nprec = k < m->in.order ? m->prec_vk : m->prec_p;   // precision of the next product
      if ((e = run_prop(m, prec, m->m_v[cur], g, 1, k, k == m->in.order, nullptr,
                        next_op(m->F[cur ^ 1], nprec),
                        st)) != cudaSuccess)
        return e;
      cur ^= 1;
    }
    {  // W = P S (with order 0 the B operand of S = P W is already in F[cur]); the pair
       // epilogue also writes the new walkers' packed forms (F[cur ^ 1] is free)
      tc::GemmShape g{N, 2 * n2, Kp, gb, 128, mt, false, true, 0};
      g.z0 = z0;
      if ((e = run_prop(m, m->prec_p, m->m_pw[cur], g, 2, 0, 0, W, Op{}, st, cur ^ 1)) !=
          cudaSuccess)
        return e;
    }
  }
  if (n2 % 32 == 0 && m->Wn.hi) {   // pair epilogue, and a trial (the T1 product exists)
    m->packed = true;
    m->fa_buf = cur ^ 1;
  }
  return cudaSuccess;
}

void mixed_invalidate(MixedState* m) {
  if (m) m->packed = false;
}

// ------------------------------------------------------------ heterogeneous batches
// The vHS product and the eight products of the propagation chain of several systems,
// each product one launch over the work list of every system's (walker, M tile, N tile)
// tiles: vHS on per-tile CTAs (tc::launch_multi), the chain on the persistent kernel
// (tc::launch_persistent_multi, two epilogue warpgroups).  The systems share the precisions
// and the Taylor order (the vHS epilogue form is picked per system); the chain runs
// EpiPropStaged for every system and writes no packed walker forms (the overlap stage
// packs its own operand).
namespace {
constexpr int kMultiMax = 4;

template <class Epi>
void multi_add(tc::MultiJob<Epi, kMultiMax>& job, int i, const tc::Maps& mp, const Epi& ep,
               int K, int m_tiles, int n_tiles, int bn, int batch, int a_batched,
               int b_batched, int& t) {
  job.maps[i] = mp;
  job.epi[i] = ep;
  job.K[i] = K;
  job.m_step[i] = 128;
  job.n_step[i] = bn;
  job.bn[i] = bn;
  job.m_tiles[i] = m_tiles;
  job.n_tiles[i] = n_tiles;
  job.a_batched[i] = a_batched;
  job.b_batched[i] = b_batched;
  job.tile0[i] = t;
  t += batch * m_tiles * n_tiles;
}

template <class Epi>
cudaError_t multi_run(int prec, const tc::MultiJob<Epi, kMultiMax>& job, int* err,
                      cudaStream_t st) {
  if (prec == PREC_SPLIT) return tc::launch_multi<256, 2, 1, true, Epi, kMultiMax>(job, err, st);
  if (prec == PREC_BF16) return tc::launch_multi<256, 4, 1, false, Epi, kMultiMax>(job, err, st);
  return cudaErrorInvalidValue;
}

// one propagation product of every system: persistent kernel, two epilogue warpgroups
constexpr int kPropWG = 2;
using PropJob = tc::PJob<EpiPropStaged, kMultiMax>;
void prop_add(PropJob& job, int i, const tc::Maps& mp, const EpiPropStaged& ep, int K,
              const MixedState* m, int a_batched, int& t) {
  job.maps[i] = mp;
  job.epi[i] = ep;
  job.sched[i] = tc::TileSched{(m->N + 127) / 128, (4 * m->n + m->bn_prop - 1) / m->bn_prop,
                               m->nw, 0, 0};
  job.K[i] = K;
  job.m_step[i] = 128;
  job.n_step[i] = m->bn_prop;
  job.a_batched[i] = a_batched;
  job.b_batched[i] = 1;
  job.k_split[i] = 0;
  job.bn[i] = m->bn_prop;
  job.tile0[i] = t;
  t += job.sched[i].total();
}
cudaError_t prop_run(int prec, PropJob& job, int n, int t, int* err, cudaStream_t st) {
  job.tile0[n] = t;
  job.np = n;
  if (prec == PREC_SPLIT)
    return tc::launch_persistent_multi<256, 2, 1, true, EpiPropStaged, kPropWG>(job, err, st);
  if (prec == PREC_BF16)
    return tc::launch_persistent_multi<256, 4, 1, false, EpiPropStaged, kPropWG>(job, err, st);
  return cudaErrorInvalidValue;
}
}  // namespace

bool mixed_multi_compatible(MixedState* const* ms, int n) {
  if (n < 1 || n > kMultiMax) return false;
  for (int i = 0; i < n; i++) {
    const MixedState* m = ms[i];
    const MixedState* a = ms[0];
    if (!m || m->prec_vhs != a->prec_vhs || m->prec_p != a->prec_p || m->prec_v1 != a->prec_v1 ||
        m->prec_vk != a->prec_vk || m->in.order != a->in.order || m->bn_prop < 32 ||
        m->bn_prop > 256 || 4 * m->n > m->bn_prop)
      return false;
    for (int p : {m->prec_vhs, m->prec_p, m->prec_v1, m->prec_vk})
      if (p != PREC_SPLIT && p != PREC_BF16) return false;
  }
  return true;
}

// vHS epilogue of either form (block pairs of symmetric L_n, or the full N^2 columns),
// picked per system of a joint launch
struct EpiVhsAny {
  static constexpr bool kTile = false, kPair = false;
  int sym;
  EpiVhsSym s;
  EpiVhs f;
  AFQ_D void operator()(int b, int r, int m, int n0, const float* v) const {
    if (sym)
      s(b, r, m, n0, v);
    else
      f(b, r, m, n0, v);
  }
};

cudaError_t mixed_vhs_multi(MixedState* const* ms, int n, cudaStream_t st) {
  if (!mixed_multi_compatible(ms, n)) return cudaErrorInvalidValue;
  int t = 0;
  tc::MultiJob<EpiVhsAny, kMultiMax> job{};
  int ord[kMultiMax];   // systems in decreasing K: long tiles first
  for (int i = 0; i < n; i++) ord[i] = i;
  std::sort(ord, ord + n, [&](int a, int b) { return ms[a]->Kv > ms[b]->Kv; });
  for (int i = 0; i < n; i++) {
    MixedState* m = ms[ord[i]];
    const long long NN = (long long)m->N * m->N;
    EpiVhsAny ep{m->vsym ? 1 : 0, EpiVhsSym{m->Vf, m->nw, m->N, m->pairs},
                 EpiVhs{m->Vf, m->nw, NN}};
    const int ntiles = m->vsym ? m->npairs : (int)((NN + 255) / 256);
    multi_add(job, i, m->m_vhs, ep, m->Kv, (2 * m->nw + 127) / 128, ntiles, 256, 1, 0, 0, t);
  }
  job.tile0[n] = t;
  job.np = n;
  return multi_run(ms[0]->prec_vhs, job, ms[0]->err, st);
}

cudaError_t mixed_prop_pack(MixedState* m, const z_t* W, cudaStream_t st) {
  if (m->packed) return cudaSuccess;   // the P W operand is in F2
  const bool pr = m->preal && m->in.order >= 1;
  pack_w_kernel<<<dim3((m->N + 31) / 32, (2 * m->n + 31) / 32, m->nw), dim3(32, 8), 0, st>>>(
      W, m->N, 2 * m->n, m->F[0], pr ? 2 : 1);
  return cudaGetLastError();
}

int mixed_prop_pack_launches(const MixedState* m) { return m->packed ? 0 : 1; }

cudaError_t mixed_prop_multi(MixedState* const* ms, z_t* const* W, int n, cudaStream_t st) {
  if (!mixed_multi_compatible(ms, n)) return cudaErrorInvalidValue;
  const int order = ms[0]->in.order;
  bool from_f2[kMultiMax];
  for (int i = 0; i < n; i++) {
    from_f2[i] = ms[i]->packed;
    ms[i]->packed = false;
  }
  // systems in decreasing K (per-tile work): the persistent CTAs take the long tiles
  // first and the short ones fill the tail
  int ord[kMultiMax];
  for (int i = 0; i < n; i++) ord[i] = i;
  std::sort(ord, ord + n, [&](int a, int b) { return ms[a]->N > ms[b]->N; });
  cudaError_t e;
  {  // S = P W
    PropJob job{};
    int t = 0;
    for (int i = 0; i < n; i++) {
      MixedState* m = ms[ord[i]];
      const bool pr = m->preal && order >= 1;
      EpiPropStaged ep{0, 0, 0, m->N, 2 * m->n, m->S, nullptr, next_op(m->F[1], m->prec_v1), 0,
                       kPropWG};
      prop_add(job, i, from_f2[ord[i]] ? m->m_pw2 : m->m_pw[0], ep, pr ? m->N : 2 * m->N, m, 0,
               t);
    }
    if ((e = prop_run(ms[0]->prec_p, job, n, t, ms[0]->err, st)) != cudaSuccess) return e;
  }
  int cur = 1;
  for (int k = 1; k <= order; k++) {  // T_k = (i/k) V T_{k-1}; S += T_k
    const int prec = k == 1 ? ms[0]->prec_v1 : ms[0]->prec_vk;
    const int nprec = k < order ? ms[0]->prec_vk : ms[0]->prec_p;
    PropJob job{};
    int t = 0;
    for (int i = 0; i < n; i++) {
      MixedState* m = ms[ord[i]];
      EpiPropStaged ep{1, k, k == order ? 1 : 0, m->N, 2 * m->n, m->S, nullptr,
                       next_op(m->F[cur ^ 1], nprec), (k == order && m->preal) ? 1 : 0, kPropWG};
      prop_add(job, i, m->m_v[cur], ep, 2 * m->N, m, 1, t);
    }
    if ((e = prop_run(prec, job, n, t, ms[0]->err, st)) != cudaSuccess) return e;
    cur ^= 1;
  }
  {  // W = P S
    PropJob job{};
    int t = 0;
    for (int i = 0; i < n; i++) {
      MixedState* m = ms[ord[i]];
      const bool pr = m->preal && order >= 1;
      EpiPropStaged ep{2, 0, 0, m->N, 2 * m->n, m->S, W[ord[i]], Op{}, 0, kPropWG};
      prop_add(job, i, m->m_pw[cur], ep, pr ? m->N : 2 * m->N, m, 0, t);
    }
    if ((e = prop_run(ms[0]->prec_p, job, n, t, ms[0]->err, st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The packed forms from W itself (after the orthogonalisation, or before a captured
// substep that expects them): the same layouts the propagation epilogue writes.
cudaError_t mixed_repack(MixedState* m, const z_t* W, cudaStream_t st) {
  if (!m) return cudaSuccess;
  const int N = m->N, n2 = 2 * m->n, nw = m->nw;
  m->packed = false;
  if (n2 % 32 || !m->Wn.hi) return cudaSuccess;   // no fused path: the consumers pack
  const bool pr = m->preal && m->in.order >= 1;
  const dim3 grid((N + 31) / 32, (n2 + 31) / 32, nw), blk(32, 8);
  pack_w_kernel<<<grid, blk, 0, st>>>(W, N, n2, m->F2, pr ? 2 : 1);
  pack_w_kernel<<<grid, blk, 0, st>>>(W, N, n2, m->F[0], 0);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    m->packed = true;
    m->fa_buf = 0;
  }
  return e;
}

int mixed_repack_launches(const MixedState* m) {
  return (m && 2 * m->n % 32 == 0 && m->Wn.hi) ? 2 : 0;
}

cudaError_t mixed_ensure_packed(MixedState* m, const z_t* W, cudaStream_t st) {
  if (!m || m->packed) return cudaSuccess;
  return mixed_repack(m, W, st);
}

static cudaError_t splitk_product(MixedState* m, const tc::Maps& mp, int prec, float ascale,
                                  z_t* out, cudaStream_t st) {
  const int nc = m->nc, nw = m->nw;
  tc::GemmShape g{nc, 2 * nw, (int)(m->greal ? m->NAK : 2 * m->NAK), m->splits, 128,
                  (nc + 127) / 128, false, false, m->ksplit};
  EpiPart ep{m->part, nc, 2 * nw, (long long)nc * 2 * nw};
  cudaError_t e;
  const int pk = promote_kb(PROMOTE_PART);
  if (pk && m->tune[TS_PART] == 2) return cudaErrorInvalidValue;   // promotion: persistent only
  switch (pk) {   // chained K slabs in TMEM (0: whole slice)
    case 1: e = run_bn(128, prec, mp, g, EpiPartPromoted<1>{ep}, m->err, st); break;
    case 2: e = run_bn(128, prec, mp, g, EpiPartPromoted<2>{ep}, m->err, st); break;
    case 4: e = run_bn(128, prec, mp, g, EpiPartPromoted<4>{ep}, m->err, st); break;
    default: e = run_bn(128, prec, mp, g, ep, m->err, st, m->tune[TS_PART]);
  }
  if (e != cudaSuccess) return e;
  const bool f16 = prec == PREC_SPLIT16;
  reduce_part_kernel<<<grid_for((long long)nc * nw), 256, 0, st>>>(
      m->part, m->splits, nc, nw, out, f16 ? ascale : 1.0f, f16 ? m->wscale : nullptr);
  return cudaGetLastError();
}

// Gb of every walker (per-walker scales first when the G products run fp16 split)
static cudaError_t pack_gb(MixedState* m, const z_t* Gc, cudaStream_t st) {
  if (m->Gb.f16) gc_scale_kernel<<<m->nw, 256, 0, st>>>(Gc, m->NAK, m->wscale);
  pack_gc_kernel<<<grid_for((long long)m->nw * m->NAK), 256, 0, st>>>(
      Gc, m->nw, m->n, m->N, m->Gb, Op{}, 0, m->greal, m->Gb.f16 ? m->wscale : nullptr);
  return cudaGetLastError();
}

cudaError_t mixed_vbias(MixedState* m, const z_t* Gc, z_t* vbias, cudaStream_t st) {
  cudaError_t e = pack_gb(m, Gc, st);
  if (e != cudaSuccess) return e;
  return splitk_product(m, m->m_vbias, m->prec_vbias, m->sSpT, vbias, st);
}

// Coulomb vector cvec[c][w] = sum_ak Lh[c][ak] Gc_w[ak] of every walker.
cudaError_t mixed_coulomb(MixedState* m, const z_t* Gc, z_t* cvec, cudaStream_t st) {
  if (!m->in.Lh) return cudaErrorInvalidValue;
  cudaError_t e = pack_gb(m, Gc, st);
  if (e != cudaSuccess) return e;
  return splitk_product(m, m->m_ej, m->prec_ej, m->sLh, cvec, st);
}

// The promoted exchange for 2n = 80: 160-column tiles of two walkers, one epilogue
// warpgroup holding all 160 accumulator columns (5 chunks of 32).
template <int PK>
static cudaError_t exchange80(MixedState* m, const tc::GemmShape& g, int nsub, z_t* Kpart,
                              int nblk, float as, const float* ws, int prec, cudaStream_t st) {
  using E = EpiExchangePromoted<80, PK>;
  const E ep{m->n, m->ex_Gn, 2, m->nc, nsub, nblk, Kpart, as, ws};
  tc::GemmShape g2 = g;
  g2.n_step = 160;
  if (prec == PREC_SPLIT16)
    return tc::launch_persistent<160, 2, 0, true, E, 1>(m->m_ek80, g2, ep, m->err, st);
  if (prec == PREC_SPLIT)
    return tc::launch_persistent<160, 2, 1, true, E, 1>(m->m_ek80, g2, ep, m->err, st);
  return tc::launch_persistent<160, 4, 1, false, E, 1>(m->m_ek80, g2, ep, m->err, st);
}

// Exchange product of the first nsub walkers packed in Gx: the staged persistent kernel
// (per-row traces from TMEM) for the compiled walker widths, else the per-tile kernel.
// prec < 0: the exchange's own operand precision (m->prec_ek); PREC_BF16 with bf16 split
// operands multiplies their hi parts only.  promote = false: no accumulator promotion (the
// staged or per-tile epilogue).
static cudaError_t exchange_product(MixedState* m, int nsub, z_t* Kpart, int nblk,
                                    cudaStream_t st, int prec = -1, bool promote = true) {
  if (prec < 0) prec = m->prec_ek;
  const int n = m->n;
  const bool f16 = m->Gx.f16;
  const float as = f16 ? m->sLh : 1.0f;
  const float* ws = f16 ? m->wscale : nullptr;
  // N tiles step by whole walker groups (Gw walkers of 2n columns): when no compiled tile
  // width is a multiple of 2n the tile's last BN - Gw 2n columns are not used
  tc::GemmShape g{m->nc * n, nsub * 2 * n, m->greal ? m->N : 2 * m->N, 2, m->ex_Gn * n,
                  m->ex_mtiles, true, true, 0, false, m->ex_Gw * 2 * n};
  const int v = m->tune[2 * nsub > m->nw ? TS_EXF : TS_EXS];
  const int pk = promote ? promote_kb(PROMOTE_EXCHANGE) : 0;
  if ((v == 1 || (v == 0 && tc_persistent())) && pk && m->ex80) {
    if (pk == 1) return exchange80<1>(m, g, nsub, Kpart, nblk, as, ws, prec, st);
    if (pk == 2) return exchange80<2>(m, g, nsub, Kpart, nblk, as, ws, prec, st);
  }
  if ((v == 1 || (v == 0 && tc_persistent())) && pk && (m->ex_bn / 2) % (2 * n) == 0) {
    cudaError_t r = cudaErrorInvalidValue;
#define AFQ_EXP(TN, PK)                                                                        \
  case TN * 8 + PK:                                                                            \
    r = run_bn(m->ex_bn, prec, m->m_ek, g,                                               \
               EpiExchangePromoted<TN, PK>{n, m->ex_Gn, m->ex_Gw, m->nc, nsub, nblk, Kpart, as, ws}, \
               m->err, st);                                                                    \
    break;
    switch (2 * n * 8 + pk) {   // promoted exchange for the compiled walker widths
      AFQ_EXP(24, 1) AFQ_EXP(24, 2) AFQ_EXP(32, 1) AFQ_EXP(32, 2) AFQ_EXP(64, 1) AFQ_EXP(64, 2)
      AFQ_EXP(96, 1) AFQ_EXP(96, 2) AFQ_EXP(128, 1) AFQ_EXP(128, 2)
    }
#undef AFQ_EXP
    // invalid value: no such instance, or its shared memory does not fit (nothing launched)
    if (r != cudaErrorInvalidValue) return r;
  }
  if (v == 1 || (v == 0 && tc_persistent())) {
    switch (2 * n) {
      case 32: return run_bn(m->ex_bn, prec, m->m_ek, g,
                             EpiExchangeStaged<32>{n, m->ex_Gn, m->ex_Gw, m->nc, nsub, nblk, Kpart, as, ws},
                             m->err, st);
      case 64: return run_bn(m->ex_bn, prec, m->m_ek, g,
                             EpiExchangeStaged<64>{n, m->ex_Gn, m->ex_Gw, m->nc, nsub, nblk, Kpart, as, ws},
                             m->err, st);
      case 96: return run_bn(m->ex_bn, prec, m->m_ek, g,
                             EpiExchangeStaged<96>{n, m->ex_Gn, m->ex_Gw, m->nc, nsub, nblk, Kpart, as, ws},
                             m->err, st);
    }
    if (v == 1 && promote) return cudaErrorInvalidValue;
  }
  EpiExchange ep{n, m->ex_Gn, m->ex_Gw, m->nc, nsub, nblk, Kpart, as, ws};
  return run_bn(m->ex_bn, prec, m->m_ek, g, ep, m->err, st);
}

// Exchange partial sums Kpart[w][s][block] of the first nsub walkers packed in Gc.
cudaError_t mixed_exchange(MixedState* m, const z_t* Gc, int nsub, z_t* Kpart, int nblk,
                           cudaStream_t st) {
  if (!m->in.Lh || nsub > m->nw) return cudaErrorInvalidValue;
  const bool f16 = m->Gx.f16;
  if (f16) gc_scale_kernel<<<nsub, 256, 0, st>>>(Gc, m->NAK, m->wscale);
  pack_gc_kernel<<<grid_for((long long)nsub * m->NAK), 256, 0, st>>>(
      Gc, nsub, m->n, m->N, Op{}, m->Gx, m->nw, m->greal, f16 ? m->wscale : nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return exchange_product(m, nsub, Kpart, nblk, st);
}

// The low-precision base's product on the staged epilogue with two epilogue warpgroups
// (one walker each at a time) and a 3-stage ring: the single product's main loop is a
// third of the split product's, and one warpgroup's traces would set the pace (ncu at
// C4 with 128 walkers: tensor pipe 27%, L2 32% with one warpgroup).  Walker widths with a
// staged instance whose tiles hold an even number of walkers; invalid value otherwise
// (nothing launched).
template <int TWO_N, int BN>
static cudaError_t exchange_base2(MixedState* m, const tc::GemmShape& g, int nsub, z_t* Kpart,
                                  int nblk, cudaStream_t st) {
  using E = EpiExchangeStaged<TWO_N>;
  using P = tc::PCfg<BN, 3, 1, false, E, 2>;
  if constexpr (P::kFits && BN % (2 * TWO_N) == 0) {
    E ep{m->n, m->ex_Gn, m->ex_Gw, m->nc, nsub, nblk, Kpart, 1.0f, nullptr};
    ep.nwg = 2;
    return tc::launch_persistent<BN, 3, 1, false, E, 2>(m->m_ek, g, ep, m->err, st);
  } else {
    return cudaErrorInvalidValue;
  }
}

// The same exchange partial sums in plain bf16: the hi parts of the split operands, one
// product instead of three (about 8 significant bits per operand).  Unsupported when the
// exchange runs on fp16 split operands.
cudaError_t mixed_exchange_lowp(MixedState* m, const z_t* Gc, int nsub, z_t* Kpart, int nblk,
                                cudaStream_t st) {
  if (!m->in.Lh || nsub > m->nw) return cudaErrorInvalidValue;
  if (m->Gx.f16 || m->prec_ek != PREC_SPLIT) return cudaErrorNotSupported;
  pack_gc_kernel<<<grid_for((long long)nsub * m->NAK), 256, 0, st>>>(
      Gc, nsub, m->n, m->N, Op{}, m->Gx, m->nw, m->greal, nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the base's fp32 sums over K need no promotion next to its bf16 operand rounding; the
  // staged epilogue keeps up with the single product's shorter main loop
  static const bool promote = getenv("AFQ_CV_BASE_PROMOTE") != nullptr;
  static const bool one_wg = getenv("AFQ_CV_BASE_WG1") != nullptr;
  if (!promote && !one_wg && m->ex_bn == m->ex_Gw * 2 * m->n && m->ex_Gw % 2 == 0) {
    const int n = m->n;
    tc::GemmShape g{m->nc * n, nsub * 2 * n, m->greal ? m->N : 2 * m->N, 2, m->ex_Gn * n,
                    m->ex_mtiles, true, true, 0, false, m->ex_Gw * 2 * n};
    cudaError_t r = cudaErrorInvalidValue;
    switch (2 * n * 1000 + m->ex_bn) {
      case 96 * 1000 + 192: r = exchange_base2<96, 192>(m, g, nsub, Kpart, nblk, st); break;
      case 64 * 1000 + 256: r = exchange_base2<64, 256>(m, g, nsub, Kpart, nblk, st); break;
      case 64 * 1000 + 128: r = exchange_base2<64, 128>(m, g, nsub, Kpart, nblk, st); break;
      case 32 * 1000 + 256: r = exchange_base2<32, 256>(m, g, nsub, Kpart, nblk, st); break;
      case 32 * 1000 + 128: r = exchange_base2<32, 128>(m, g, nsub, Kpart, nblk, st); break;
    }
    if (r != cudaErrorInvalidValue) return r;
  }
  return exchange_product(m, nsub, Kpart, nblk, st, PREC_BF16, promote);
}

bool mixed_has_dm(const MixedState* m) { return m && m->T1 && m->bn_t1 && m->bn_gc; }

// Overlaps (want_gc == 0) or the full mixed density matrix of every walker.  Both compute
// T1^-1 (kept in Tinv); cached != 0 reuses the T1^-1 of an earlier call on the same W.
cudaError_t mixed_dm(MixedState* m, const z_t* W, z_t* Gc, z_t* Wd, int* info, int want_gc,
                     int save_old, int cached, cudaStream_t st) {
  if (!mixed_has_dm(m)) return cudaErrorInvalidValue;
  const int N = m->N, n = m->n, n2 = 2 * n, nw = m->nw;
  cudaError_t e;
  if (!(cached && want_gc)) {
    // T1 (conjugated) of both spins: one 128-row tile per walker; its A operand is packed
    // unless the walkers' packed forms are current
    if (!m->packed) {
      pack_w_kernel<<<dim3((N + 31) / 32, (n2 + 31) / 32, nw), dim3(32, 8), 0, st>>>(W, N, n2,
                                                                                   m->F[0], 0);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    const tc::Maps& mt1 = (m->packed && m->fa_buf == 1) ? m->m_t1_1 : m->m_t1;
    tc::GemmShape g{128, 4 * n, 2 * N, nw, 128, 1, true, false, 0};
    if ((e = run_bn(m->bn_t1, PREC_SPLIT, mt1, g, EpiT1{m->T1, n}, m->err, st,
                    m->tune[TS_T1])) != cudaSuccess)
      return e;
    if ((e = launch_lu(m->T1, n, 2 * nw, m->Tinv, Wd, info, 1, save_old, st)) != cudaSuccess ||
        !want_gc)
      return e;
  }
  pack_wn_kernel<<<grid_for((long long)nw * N * n2), 256, 0, st>>>(W, (long long)nw * N * n2, m->Wn);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  for (int sp = 0; sp < 2; sp++) {
    tc::GemmShape g{N, 2 * n, 2 * n, nw, 128, (N + 127) / 128, true, true, 0};
    if ((e = run_bn(m->bn_gc, PREC_SPLIT, m->m_gc[sp], g, EpiGc{Gc, n, N, sp}, m->err, st)) !=
        cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

cudaError_t mixed_energy_chol(MixedState* m, const z_t* Gc, z_t* cvec, z_t* Kpart, int nblk,
                              cudaStream_t st) {
  cudaError_t e = mixed_coulomb(m, Gc, cvec, st);
  if (e != cudaSuccess) return e;
  return mixed_exchange(m, Gc, m->nw, Kpart, nblk, st);
}

// ------------------------------------------------------------ kernel autotuning
// Times the candidate kernels of each product site on the real shapes and keeps the
// fastest: persistent or per-tile for every site, and for the split-K vbias / Coulomb
// products also half, once and twice the default slice count.  The per-step operands are
// zeroed first and every timed product writes scratch only (S, F, Vf, T1, part and the
// temporaries below), so the walkers are untouched.  AFQ_TUNE=0 keeps the built-in rules,
// AFQ_TUNE=1 / 2 (or AFQ_TC_PERSISTENT=0) forces the persistent / per-tile kernel wherever
// it exists, with the default slice count; AFQ_SPLITK=<s> sets the slice count.
// Choices are cached per shape for the process (every handle of one shape computes with
// the same kernels and slice counts, so its results do not depend on timing noise) and,
// with AFQ_TUNE_CACHE=<file>, across processes: the file holds one line per shape and is
// read before timing and appended after it.
namespace {
struct TuneRec {
  int tune[TS_N];
  float ms[TS_N][2];
  float group_ms[6];
  int vhs_epi;
  float vhs_epi_ms[4];
  int chain_wave;
  float chain_ms[6];
  int splits;
  int prop_group;
};
std::mutex tune_mu;
std::map<std::string, TuneRec>& tune_cache() {
  static std::map<std::string, TuneRec> c;
  return c;
}
std::string tune_key(const MixedState* m) {
  char b[256];
  snprintf(b, sizeof b, "N%d_n%d_nc%d_nw%d_o%d_g%d_p%d_s%d_v%d_x%d_t%d_q%d%d%d%d%d%d%d",
           m->N, m->n, m->nc, m->nw, m->in.order, (int)m->greal, (int)m->preal, (int)m->s_real,
           (int)m->vsym, m->in.Lh ? 1 : 0, mixed_has_dm(m) ? 1 : 0, m->prec_vhs, m->prec_p,
           m->prec_v1, m->prec_vk, m->prec_vbias, m->prec_ej, m->prec_ek);
  return b;
}
std::set<std::string>& tune_file_keys() {   // shapes present in the loaded file
  static std::set<std::string> k;
  return k;
}
void tune_load(const char* path) {
  static std::string loaded;
  if (!path || loaded == path) return;
  loaded = path;
  tune_file_keys().clear();
  FILE* f = fopen(path, "r");
  if (!f) return;
  char key[256];
  TuneRec r{};
  while (fscanf(f, "%255s", key) == 1) {
    bool ok = true;
    for (int i = 0; i < TS_N && ok; i++)
      ok = fscanf(f, "%d %f %f", &r.tune[i], &r.ms[i][0], &r.ms[i][1]) == 3;
    for (int i = 0; i < 6 && ok; i++) ok = fscanf(f, "%f", &r.group_ms[i]) == 1;
    if (ok) ok = fscanf(f, "%d", &r.vhs_epi) == 1;
    for (int i = 0; i < 4 && ok; i++) ok = fscanf(f, "%f", &r.vhs_epi_ms[i]) == 1;
    if (ok) ok = fscanf(f, "%d", &r.chain_wave) == 1;
    for (int i = 0; i < 6 && ok; i++) ok = fscanf(f, "%f", &r.chain_ms[i]) == 1;
    if (!ok || fscanf(f, "%d %d", &r.splits, &r.prop_group) != 2) break;
    tune_cache()[key] = r;
    tune_file_keys().insert(key);
  }
  fclose(f);
}
void tune_save(const char* path, const std::string& key, const TuneRec& r) {
  if (!path || !tune_file_keys().insert(key).second) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s", key.c_str());
  for (int i = 0; i < TS_N; i++) fprintf(f, " %d %.5f %.5f", r.tune[i], r.ms[i][0], r.ms[i][1]);
  for (int i = 0; i < 6; i++) fprintf(f, " %.5f", r.group_ms[i]);
  fprintf(f, " %d", r.vhs_epi);
  for (int i = 0; i < 4; i++) fprintf(f, " %.5f", r.vhs_epi_ms[i]);
  fprintf(f, " %d", r.chain_wave);
  for (int i = 0; i < 6; i++) fprintf(f, " %.5f", r.chain_ms[i]);
  fprintf(f, " %d %d\n", r.splits, r.prop_group);
  fclose(f);
}
}  // namespace

static cudaError_t mixed_tune(MixedState* m, cudaStream_t st) {
  const char* env = getenv("AFQ_TUNE");
  int force = env ? atoi(env) : -1;
  if (force == 0) {
    if (const char* fs = getenv("AFQ_SPLITK")) set_splits(m, std::max(1, atoi(fs)));
    return cudaSuccess;
  }
  if (force < 0 && !tc_persistent()) force = 2;   // AFQ_TC_PERSISTENT=0: per-tile kernels
  const char* fsk = getenv("AFQ_SPLITK");
  const char* fpg = getenv("AFQ_PROP_GROUP");
  const char* fve = getenv("AFQ_VHS_EPI");
  const char* fch = getenv("AFQ_PROP_CHAIN");
  const std::string key = tune_key(m) + "_pg" + std::to_string(fpg ? atoi(fpg) : -1) + "_ve" +
                          std::to_string(fve ? atoi(fve) : -1) + "_ch" +
                          std::to_string(fch ? atoi(fch) : -1) + "_f" +
                          std::to_string(force) + "_k" +
                          std::to_string(fsk ? atoi(fsk) : 0) + "_p" +
                          std::to_string(promote_kb(PROMOTE_PART)) +
                          std::to_string(promote_kb(PROMOTE_EXCHANGE));
  const char* cache_path = getenv("AFQ_TUNE_CACHE");
  {
    std::lock_guard<std::mutex> lk(tune_mu);
    tune_load(cache_path);
    auto it = tune_cache().find(key);
    if (it != tune_cache().end()) {
      const TuneRec& r = it->second;
      for (int i = 0; i < TS_N; i++) {
        m->tune[i] = r.tune[i];
        m->tune_ms[i][0] = r.ms[i][0];
        m->tune_ms[i][1] = r.ms[i][1];
      }
      if (r.splits >= 1) {
        set_splits(m, r.splits);
        if (m->splits > m->part_cap) set_splits(m, m->splits0);
      }
      m->prop_group = r.prop_group;
      for (int i = 0; i < 6; i++) m->prop_group_ms[i] = r.group_ms[i];
      m->vhs_epi = r.vhs_epi;
      for (int v = 0; v < 4; v++) m->vhs_epi_ms[v] = r.vhs_epi_ms[v];
      m->chain_wave = m->dep ? r.chain_wave : 0;
      for (int i = 0; i < 6; i++) m->chain_ms[i] = r.chain_ms[i];
      tune_save(cache_path, key, r);   // a shape timed before the file was named
      return cudaSuccess;
    }
  }
  const int N = m->N, n = m->n, nw = m->nw, nc = m->nc;
  const long long NAK = m->NAK;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  auto zero = [&](const Op& o, size_t count) {
    if (o.hi) A(cudaMemsetAsync(o.hi, 0, sizeof(*o.hi) * count, st));
    if (o.lo) A(cudaMemsetAsync(o.lo, 0, sizeof(*o.lo) * count, st));
  };
  zero(m->Xf, (size_t)2 * nw * m->Kv);
  zero(m->Vf, (size_t)nw * N * 2 * N);
  zero(m->F[0], (size_t)nw * 4 * n * 2 * N);
  zero(m->F[1], (size_t)nw * 4 * n * 2 * N);
  zero(m->Gb, (size_t)2 * nw * 2 * NAK);
  if (m->in.Lh) zero(m->Gx, (size_t)nw * 2 * NAK * 2);
  A(cudaMemsetAsync(m->S, 0, sizeof(float2) * (size_t)nw * N * 2 * n, st));
  A(cudaMemsetAsync(m->wscale, 0, sizeof(float) * nw, st));
  z_t* out = nullptr;   // vbias-shaped result of the split-K products
  z_t* kp = nullptr;    // exchange partial sums
  A(cudaMallocAsync(&out, sizeof(z_t) * (size_t)nc * nw, st));
  if (m->in.Lh) A(cudaMallocAsync(&kp, sizeof(z_t) * (size_t)nw * 2 * m->ex_mtiles, st));
  A(cudaStreamSynchronize(st));
  bool fatal = e != cudaSuccess;
  // median time of three calls after a warm-up call; < 0 when the candidate does not
  // launch or a kernel raised a timeout flag (the candidate is then never chosen)
  const bool verbose = getenv("AFQ_TUNE_VERBOSE") != nullptr;
  cudaEvent_t ev[4] = {};
  for (auto& x : ev) A(cudaEventCreate(&x));
  auto timed = [&](const std::function<cudaError_t()>& run) -> float {
    if (fatal) return -1.0f;
    cudaMemsetAsync(m->err, 0, sizeof(int), st);
    if (run() != cudaSuccess) {
      cudaGetLastError();
      return -1.0f;
    }
    cudaEventRecord(ev[0], st);
    for (int r = 0; r < 3; r++) {
      run();
      cudaEventRecord(ev[r + 1], st);
    }
    float t[3] = {-1.0f, -1.0f, -1.0f};
    int flags = 0;
    if (cudaEventSynchronize(ev[3]) != cudaSuccess ||
        cudaMemcpy(&flags, m->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
      fatal = true;
      return -1.0f;
    }
    for (int r = 0; r < 3; r++) cudaEventElapsedTime(&t[r], ev[r], ev[r + 1]);
    if (verbose)
      fprintf(stderr, "afq tune:   %.4f %.4f %.4f ms, flags %d\n", t[0], t[1], t[2], flags);
    if (flags) {
      cudaMemsetAsync(m->err, 0, sizeof(int), st);
      return -1.0f;
    }
    std::sort(t, t + 3);
    return t[1];
  };
  // candidates: both kernels, or (only_persistent) the promoted persistent one, whose
  // accuracy the per-tile kernel does not match
  auto pick = [&](int site, const std::function<cudaError_t()>& run, bool only_persistent = false) {
    int best = 0;
    for (int v = 1; v <= 2; v++) {
      if (force > 0 && v != force) continue;
      if (only_persistent && force <= 0 && v == 2) continue;
      m->tune[site] = v;
      if (verbose) fprintf(stderr, "afq tune: site %d kernel %d slices %d\n", site, v, m->splits);
      const float t = timed(run);
      m->tune_ms[site][v - 1] = t > 0.0f ? t : 0.0f;
      if (t > 0.0f && (!best || t < m->tune_ms[site][best - 1])) best = v;
    }
    m->tune[site] = best;
  };
  pick(TS_VHS, [&] { return vhs_product(m, st); });
  // then the symmetric vHS epilogue: the tuned row-wise one against the shared-memory
  // tile (full tuning only, so forced kernels stay comparable); AFQ_VHS_EPI=0|1 forces
  if (m->vsym && m->tune[TS_VHS] && force < 0) {
    const char* fe = getenv("AFQ_VHS_EPI");
    float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    int bv = 0;
    for (int v = 0; v < 4; v++) {
      if (fe && atoi(fe) != v) continue;
      m->vhs_epi = v;
      const float ms = timed([&] { return vhs_product(m, st); });
      t[v] = ms > 0.0f ? ms : 0.0f;
      if (t[v] > 0.0f && (t[bv] <= 0.0f || t[v] < t[bv])) bv = v;
    }
    m->vhs_epi = bv;
    for (int v = 0; v < 4; v++) m->vhs_epi_ms[v] = t[v];
  }
  {
    const int mt = (N + 127) / 128, n2 = 2 * n;
    const int Kp = m->preal ? N : 2 * N;
    const int order = m->in.order;
    int group = 0;   // walkers per group of the timed chain (0: all)
    auto chain = [&] {   // the chain: two P products and `order` V products per group
      const int G = group > 0 && group < nw ? group : nw;
      cudaError_t r = cudaSuccess;
      for (int z0 = 0; z0 < nw && r == cudaSuccess; z0 += G) {
        const int gb = std::min(G, nw - z0);
        tc::GemmShape gp{N, 2 * n2, Kp, gb, 128, mt, false, true, 0};
        tc::GemmShape gv{N, 2 * n2, 2 * N, gb, 128, mt, true, true, 0};
        gp.z0 = gv.z0 = z0;
        r = run_prop(m, m->prec_p, m->m_pw[0], gp, 0, 0, 0, nullptr,
                     next_op(m->F[1], m->prec_v1), st);
        for (int k = 1; k <= order && r == cudaSuccess; k++)
          r = run_prop(m, k == 1 ? m->prec_v1 : m->prec_vk, m->m_v[0], gv, 1, k, 0, nullptr,
                       next_op(m->F[1], m->prec_vk), st);
        if (r == cudaSuccess)
          r = run_prop(m, m->prec_p, m->m_pw[0], gp, 0, 0, 0, nullptr,
                       next_op(m->F[1], m->prec_p), st);
      }
      return r;
    };
    pick(TS_PROP, chain);
    // then the walker group of the chosen kernel: all walkers, or groups whose Taylor sum,
    // operands and V fit in L2 together; AFQ_PROP_GROUP=<walkers> forces one
    const char* fg = getenv("AFQ_PROP_GROUP");
    const int cand[6] = {0, 32, 48, 64, 96, 128};
    int best = 0;
    float bt = 0.0f;
    for (int c = 0; c < 6 && m->tune[TS_PROP]; c++) {
      if (cand[c] >= nw || (fg && cand[c] != atoi(fg))) continue;
      group = cand[c];
      const float t = timed(chain);
      m->prop_group_ms[c] = t > 0.0f ? t : 0.0f;
      if (t > 0.0f && (bt == 0.0f || t < bt)) {
        bt = t;
        best = group;
      }
    }
    m->prop_group = best;
    // then the whole chain as one cooperative launch (waves of 16, 24, 32, 48 or 64 walkers)
    // against the eight launches of the chosen kernel over all walkers; AFQ_PROP_CHAIN=0
    // keeps the eight launches, =<walkers> forces a wave
    const char* fc = getenv("AFQ_PROP_CHAIN");
    const int fcw = fc ? atoi(fc) : -1;
    if (m->dep && m->prop_group == 0 && m->tune[TS_PROP] && fcw != 0) {
      m->chain_ms[0] = m->prop_group_ms[0];
      const int waves[5] = {16, 24, 32, 48, 64};
      int bw = 0;
      float bwt = m->chain_ms[0] > 0.0f && fcw < 0 ? m->chain_ms[0] : 0.0f;
      for (int c = 0; c < 5; c++) {
        if (fcw > 0 && waves[c] != fcw) continue;
        const float t = timed([&] { return propagate_chain(m, nullptr, waves[c], true, st); });
        m->chain_ms[c + 1] = t > 0.0f ? t : 0.0f;
        if (t > 0.0f && (bwt == 0.0f || t < bwt)) {
          bwt = t;
          bw = waves[c];
        }
      }
      m->chain_wave = bw;
    }
  }
  {  // split-K slices x kernel
    int bs = m->splits0, bv = 0;
    float bt = 0.0f, bms[2] = {0.0f, 0.0f};
    const char* fs = getenv("AFQ_SPLITK");
    const int fsp = fs ? std::max(1, atoi(fs)) : 0;
    const int cand[3] = {fsp ? fsp : m->splits0, std::max(1, m->splits0 / 2), 2 * m->splits0};
    // forced kernels or AFQ_SPLITK: one slice count
    for (int c = 0; c < (force > 0 || fsp ? 1 : 3); c++) {
      set_splits(m, cand[c]);
      if (m->splits > m->part_cap) continue;
      pick(TS_PART, [&] { return splitk_product(m, m->m_vbias, m->prec_vbias, m->sSpT, out, st); });
      const int v = m->tune[TS_PART];
      if (v && (!bv || m->tune_ms[TS_PART][v - 1] < bt)) {
        bv = v;
        bs = m->splits;
        bt = m->tune_ms[TS_PART][v - 1];
        bms[0] = m->tune_ms[TS_PART][0];
        bms[1] = m->tune_ms[TS_PART][1];
      }
    }
    set_splits(m, bs);
    m->tune[TS_PART] = bv;
    m->tune_ms[TS_PART][0] = bms[0];
    m->tune_ms[TS_PART][1] = bms[1];
  }
  if (m->in.Lh) {
    const int nsub = std::max(1, nw / 8);
    // the promoted exchange instances (walker widths 24, 32, 64, 96, 128, and 80 on its
    // own 160-column tiles) run on the persistent kernel only: the tuner may not trade
    // their accuracy for speed
    const int w2 = 2 * n;
    const int pke = promote_kb(PROMOTE_EXCHANGE);
    const bool exp = (pke > 0 && (w2 == 24 || w2 == 32 || w2 == 64 || w2 == 96 || w2 == 128) &&
                      (m->ex_bn / 2) % w2 == 0) ||
                     ((pke == 1 || pke == 2) && m->ex80);
    pick(TS_EXF, [&] { return exchange_product(m, nw, kp, m->ex_mtiles, st); }, exp);
    pick(TS_EXS, [&] { return exchange_product(m, nsub, kp, m->ex_mtiles, st); }, exp);
  }
  if (mixed_has_dm(m)) {
    pick(TS_T1, [&] {
      tc::GemmShape g{128, 4 * n, 2 * N, nw, 128, 1, true, false, 0};
      return run_bn(m->bn_t1, PREC_SPLIT, m->m_t1, g, EpiT1{m->T1, n}, m->err, st, m->tune[TS_T1]);
    });
  }
  for (auto& x : ev)
    if (x) cudaEventDestroy(x);
  if (out) cudaFreeAsync(out, st);
  if (kp) cudaFreeAsync(kp, st);
  A(cudaMemsetAsync(m->err, 0, sizeof(int), st));
  A(cudaStreamSynchronize(st));
  if (fatal && e == cudaSuccess) e = cudaGetLastError();
  if (fatal && e == cudaSuccess) e = cudaErrorUnknown;
  if (e == cudaSuccess) {
    TuneRec r{};
    for (int i = 0; i < TS_N; i++) {
      r.tune[i] = m->tune[i];
      r.ms[i][0] = m->tune_ms[i][0];
      r.ms[i][1] = m->tune_ms[i][1];
    }
    r.splits = m->splits;
    r.prop_group = m->prop_group;
    for (int i = 0; i < 6; i++) r.group_ms[i] = m->prop_group_ms[i];
    r.vhs_epi = m->vhs_epi;
    for (int v = 0; v < 4; v++) r.vhs_epi_ms[v] = m->vhs_epi_ms[v];
    r.chain_wave = m->chain_wave;
    for (int i = 0; i < 6; i++) r.chain_ms[i] = m->chain_ms[i];
    std::lock_guard<std::mutex> lk(tune_mu);
    tune_cache()[key] = r;
    tune_save(cache_path, key, r);
  }
  if (getenv("AFQ_TUNE_VERBOSE"))
    fprintf(stderr, "afq tune: vhs %d (%.3f %.3f) prop %d (%.3f %.3f) part %d x%d (%.3f %.3f) "
            "exf %d (%.3f %.3f) exs %d (%.3f %.3f) t1 %d (%.3f %.3f) ms\n",
            m->tune[TS_VHS], m->tune_ms[TS_VHS][0], m->tune_ms[TS_VHS][1], m->tune[TS_PROP],
            m->tune_ms[TS_PROP][0], m->tune_ms[TS_PROP][1], m->tune[TS_PART], m->splits,
            m->tune_ms[TS_PART][0], m->tune_ms[TS_PART][1], m->tune[TS_EXF],
            m->tune_ms[TS_EXF][0], m->tune_ms[TS_EXF][1], m->tune[TS_EXS],
            m->tune_ms[TS_EXS][0], m->tune_ms[TS_EXS][1], m->tune[TS_T1], m->tune_ms[TS_T1][0],
            m->tune_ms[TS_T1][1]);
  return e;
}

int mixed_prop_chain(const MixedState* m, float* ms) {
  if (ms)
    for (int i = 0; i < 6; i++) ms[i] = m ? m->chain_ms[i] : 0.0f;
  return m ? m->chain_wave : 0;
}

int mixed_vhs_epilogue(const MixedState* m, float* ms) {
  if (ms)
    for (int i = 0; i < 4; i++) ms[i] = m ? m->vhs_epi_ms[i] : 0.0f;
  return m ? m->vhs_epi : 0;
}

int mixed_prop_group(const MixedState* m, float* ms) {
  if (ms)
    for (int i = 0; i < 6; i++) ms[i] = m ? m->prop_group_ms[i] : 0.0f;
  return m ? m->prop_group : 0;
}

void mixed_tuning(const MixedState* m, int* choice, float* ms) {
  for (int i = 0; i < TS_N; i++) {
    if (choice) choice[i] = m ? m->tune[i] : 0;
    if (ms) {
      ms[2 * i] = m ? m->tune_ms[i][0] : 0.0f;
      ms[2 * i + 1] = m ? m->tune_ms[i][1] : 0.0f;
    }
  }
  if (choice) choice[TS_N] = m ? m->splits : 0;
}

}  // namespace afq
