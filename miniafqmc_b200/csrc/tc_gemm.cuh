// tcgen05 (5th-generation tensor core) GEMM for sm_100a with TMA staging.
//
// D[b][m][n] = sum_k A[b][m][k] * B[b][n][k]      (both operands K-major, fp32 accumulate)
//
// One CTA computes a 128 x BN tile: warp 4 issues TMA loads of 128-byte-wide K slabs
// (SWIZZLE_128B) into a STAGES-deep shared-memory ring guarded by mbarriers; one thread
// of warp 5 issues tcgen05.mma (kind::f16 for bf16 operands, kind::tf32 for fp32 operands)
// into a TMEM accumulator and frees each stage with tcgen05.commit; warps 0-3 then read
// the accumulator with tcgen05.ld (one TMEM lane per output row) and hand 32-column
// chunks (or the whole tile, staged in shared memory) to the epilogue functor.
// The split form loads hi and lo parts of both operands per stage and accumulates
// hi*hi + hi*lo + lo*hi: with bf16 parts that carries ~16 significant bits per operand
// (bf16x3), with tf32 parts ~21 bits (3xTF32).
//
// Every mbarrier wait is bounded (about one second of SM clocks); on timeout the CTA
// records an error code in *err and skips its remaining work.  Before it frees its TMEM
// and exits it drains its own asynchronous work -- the TMA fills it issued and the MMAs it
// issued -- with waits that keep the one-second bound whatever the work waits' bound is
// (g_tc_wait_clocks, which a test may lower to make the work waits run out).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <type_traits>
#include "afq_common.cuh"

namespace tc {

enum : int { ERR_TIMEOUT_PRODUCER = 1, ERR_TIMEOUT_MMA = 2, ERR_TIMEOUT_EPILOGUE = 4 };

AFQ_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

AFQ_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
AFQ_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bound of the work waits in SM clocks (default ~1 s at 1.96 GHz); one copy per
// translation unit, set with the module's set_wait_clocks.  The drains use kDrainClocks.
constexpr long long kDrainClocks = 2000000000LL;
static __device__ long long g_tc_wait_clocks = kDrainClocks;

// Waits for the phase with the given parity to complete; false after `limit` clocks.
AFQ_D bool mbar_wait_for(uint64_t* bar, uint32_t parity, long long limit) {
  const uint32_t addr = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}
// A work wait (bounded by g_tc_wait_clocks).
AFQ_D bool mbar_wait(uint64_t* bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, g_tc_wait_clocks);
}
// A drain of the CTA's own asynchronous copies or MMAs before it frees TMEM or exits.
AFQ_D bool mbar_wait_drain(uint64_t* bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, kDrainClocks);
}

// Host side: sets this translation unit's work-wait bound on the current device
// (clocks <= 0 restores the default).
inline cudaError_t set_wait_clocks(long long clocks) {
  const long long v = clocks > 0 ? clocks : kDrainClocks;
  return cudaMemcpyToSymbol(g_tc_wait_clocks, &v, sizeof(v));
}
AFQ_D void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
AFQ_D void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
AFQ_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

AFQ_D void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

AFQ_D void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols));
}
AFQ_D void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
AFQ_D void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
AFQ_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
AFQ_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// FMT: operand format of both A and B: 0 = fp16, 1 = bf16 (kind::f16), 2 = tf32.
template <int FMT>
AFQ_D void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  if (FMT == 2)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
  else
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}
AFQ_D void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 consecutive fp32 columns of this thread's TMEM lane.
AFQ_D void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// acc[i] += column i of 32 consecutive fp32 TMEM columns of this thread's lane.  Load,
// wait and adds sit in one asm block so the 32 loaded values die at once (a promoting
// epilogue holds its whole accumulator in registers next to them).
AFQ_D void tmem_ld32_add(uint32_t taddr, float* acc) {
  asm volatile(
      "{\n .reg .b32 t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, t12, t13, t14, t15, t16, t17, t18, t19, t20, t21, t22, t23, t24, t25, t26, t27, t28, t29, t30, t31;\n"
      " tcgen05.ld.sync.aligned.32x32b.x32.b32 {t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, t12, t13, t14, t15, t16, t17, t18, t19, t20, t21, t22, t23, t24, t25, t26, t27, t28, t29, t30, t31}, [%32];\n"
      " tcgen05.wait::ld.sync.aligned;\n"
      " add.f32 %0, %0, t0;\n"
      " add.f32 %1, %1, t1;\n"
      " add.f32 %2, %2, t2;\n"
      " add.f32 %3, %3, t3;\n"
      " add.f32 %4, %4, t4;\n"
      " add.f32 %5, %5, t5;\n"
      " add.f32 %6, %6, t6;\n"
      " add.f32 %7, %7, t7;\n"
      " add.f32 %8, %8, t8;\n"
      " add.f32 %9, %9, t9;\n"
      " add.f32 %10, %10, t10;\n"
      " add.f32 %11, %11, t11;\n"
      " add.f32 %12, %12, t12;\n"
      " add.f32 %13, %13, t13;\n"
      " add.f32 %14, %14, t14;\n"
      " add.f32 %15, %15, t15;\n"
      " add.f32 %16, %16, t16;\n"
      " add.f32 %17, %17, t17;\n"
      " add.f32 %18, %18, t18;\n"
      " add.f32 %19, %19, t19;\n"
      " add.f32 %20, %20, t20;\n"
      " add.f32 %21, %21, t21;\n"
      " add.f32 %22, %22, t22;\n"
      " add.f32 %23, %23, t23;\n"
      " add.f32 %24, %24, t24;\n"
      " add.f32 %25, %25, t25;\n"
      " add.f32 %26, %26, t26;\n"
      " add.f32 %27, %27, t27;\n"
      " add.f32 %28, %28, t28;\n"
      " add.f32 %29, %29, t29;\n"
      " add.f32 %30, %30, t30;\n"
      " add.f32 %31, %31, t31;\n"
      "}\n"
      : "+f"(acc[0]), "+f"(acc[1]), "+f"(acc[2]), "+f"(acc[3]),
        "+f"(acc[4]), "+f"(acc[5]), "+f"(acc[6]), "+f"(acc[7]),
        "+f"(acc[8]), "+f"(acc[9]), "+f"(acc[10]), "+f"(acc[11]),
        "+f"(acc[12]), "+f"(acc[13]), "+f"(acc[14]), "+f"(acc[15]),
        "+f"(acc[16]), "+f"(acc[17]), "+f"(acc[18]), "+f"(acc[19]),
        "+f"(acc[20]), "+f"(acc[21]), "+f"(acc[22]), "+f"(acc[23]),
        "+f"(acc[24]), "+f"(acc[25]), "+f"(acc[26]), "+f"(acc[27]),
        "+f"(acc[28]), "+f"(acc[29]), "+f"(acc[30]), "+f"(acc[31])
      : "r"(taddr)
      : "memory");
}

// Shared-memory matrix descriptor: K-major operand tile written by TMA with
// SWIZZLE_128B (rows of 128 bytes, 8-row groups 1024 bytes apart) or, for SLAB = 64,
// SWIZZLE_64B (rows of 64 bytes, 8-row groups 512 bytes apart).
template <int SLAB = 128>
AFQ_D uint64_t sdesc_k(uint32_t saddr) {
  static_assert(SLAB == 128 || SLAB == 64, "K slab of 64 or 128 bytes");
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);   // start address
  d |= (uint64_t)1 << 16;                     // leading byte offset (unused when swizzled)
  d |= (uint64_t)(8 * SLAB >> 4) << 32;       // stride byte offset: one 8-row group
  d |= (uint64_t)1 << 46;                     // descriptor version for sm_100
  d |= (uint64_t)(SLAB == 128 ? 2 : 4) << 61; // SWIZZLE_128B / SWIZZLE_64B
  return d;
}
AFQ_D uint64_t sdesc_k128(uint32_t saddr) { return sdesc_k<128>(saddr); }

// Instruction descriptor: fp32 accumulator, A and B of the same format (0 = fp16,
// 1 = bf16 for kind::f16; 2 = tf32 for kind::tf32), both K-major.
constexpr uint32_t idesc(int M, int N, int fmt) {
  return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

template <int BN, int STAGES, int FMT, bool SPLIT, int SLAB = 128>
struct Cfg {
  static constexpr int BM = 128;
  static constexpr int ELEM = FMT == 2 ? 4 : 2;
  static constexpr int BK = SLAB / ELEM;         // elements per K slab (128 or 64 bytes)
  static constexpr int UK = 32 / ELEM;           // K of one tcgen05.mma
  static constexpr uint32_t A_BYTES = BM * SLAB, B_BYTES = BN * SLAB;
  static constexpr int PARTS = SPLIT ? 2 : 1;    // hi (and lo) parts of each operand
  static constexpr uint32_t STAGE_BYTES = PARTS * (A_BYTES + B_BYTES);
  static constexpr uint32_t TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  static constexpr size_t SMEM = 1024 + STAGES * STAGE_BYTES + 8 * (2 * STAGES + 2) + 16;
  static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "UMMA N for M=128");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// Operand tensor maps; the lo parts are used only by the split form.
struct Maps {
  CUtensorMap a, b, a_lo, b_lo;
};

// Named barrier among the 128 epilogue threads (warps 0-3).
AFQ_D void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
// Named barrier of epilogue warpgroup g of the persistent kernel (ids 1, 2).
AFQ_D void epi_bar_group(int g) { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); }

// Optional epilogue traits: kStaged functors get TMEM access and kScratchBytes of shared
// memory per epilogue warpgroup (persistent kernel only).
template <class E, class = void> struct EpiStaged : std::false_type {};
template <class E>
struct EpiStaged<E, std::void_t<decltype(E::kStaged)>> : std::integral_constant<bool, E::kStaged> {};
// kPerTile functors run on the per-tile kernel even when the persistent one is enabled.
template <class E, class = void> struct EpiPerTile : std::false_type {};
template <class E>
struct EpiPerTile<E, std::void_t<decltype(E::kPerTile)>> : std::integral_constant<bool, E::kPerTile> {};
// kPromoteKB functors (persistent kernel only): the MMA restarts the accumulator every
// kPromoteKB K slabs and the epilogue warps add the chunks in registers with
// round-to-nearest fp32 adds.  The tensor pipe rounds its fp32 accumulator toward zero on
// every MMA, which biases long sums of like-signed terms; promotion bounds every chain in
// TMEM to kPromoteKB slabs.  Warpgroup g then owns the contiguous columns
// [g BN / EPI_WG, (g + 1) BN / EPI_WG) and gets them as one register array: row-wise
// functors are called per 32-column chunk, kRegs functors once through
//   epi.regs(batch, m_tile, n_tile, tile_row, acc, scratch, wg).
template <class E, class = void> struct EpiPromote : std::integral_constant<int, 0> {};
template <class E>
struct EpiPromote<E, std::void_t<decltype(E::kPromoteKB)>>
    : std::integral_constant<int, E::kPromoteKB> {};
template <class E, class = void> struct EpiRegs : std::false_type {};
template <class E>
struct EpiRegs<E, std::void_t<decltype(E::kRegs)>> : std::integral_constant<bool, E::kRegs> {};
template <class E, class = void> struct EpiScratch : std::integral_constant<int, 0> {};
template <class E>
struct EpiScratch<E, std::void_t<decltype(E::kScratchBytes)>>
    : std::integral_constant<int, E::kScratchBytes> {};

// Epilogue interface.  Row-wise functors (Epi::kTile == Epi::kPair == false) get
//   epi(batch, tile_row, m, n_first, v[32])
// for each 32-column chunk of each of the 128 rows.  Pair functors (kPair) get chunks
// c0 and c0 + P of a row together, epi.pair(batch, tile_row, m, c0, v[32], u[32]), for
// c0 < P = epi.pair_stride().  Tile functors (kTile) get the whole fp32 tile in shared
// memory (row stride BN + 1) after the epilogue barrier:
//   epi.tile(batch, m_tile, n_tile, tile, ld, tid)  with tid in [0, 128).
//   MINB = CTAs per SM the launch is compiled for (2 caps registers at 170 per thread so a
//   lean ring's CTAs pair up on an SM).
// Whether the fp32 tile of a tile epilogue (128 rows x BN + 1 floats) fits the operand
// ring; kHalfTile functors also run with half the columns staged at a time.
template <int BN, int STAGES, uint32_t STAGE_BYTES>
struct TileInRing
    : std::integral_constant<bool, (size_t)128 * (BN + 1) * 4 <= (size_t)STAGES * STAGE_BYTES> {};
template <class E, class = void> struct EpiHalfTile : std::false_type {};
template <class E>
struct EpiHalfTile<E, std::void_t<decltype(E::kHalfTile)>>
    : std::integral_constant<bool, E::kHalfTile> {};

// The body of the per-tile kernels: one 128 x bn output tile (bn <= BN, a multiple of 32:
// the epilogues take 32-column chunks; the B tensor map's box holds bn rows) of batch
// `batch`, K range [kbase, kbase + klen), operand batches za / zb.  The shared-memory ring
// is laid out for BN.
template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int SLAB>
AFQ_D void gemm_tile(const Maps& maps, int mt, int nt, int m0, int n0, int batch, int za,
                     int zb, int kbase, int klen, int bn, const Epi epi, int* err) {
  using C = Cfg<BN, STAGES, FMT, SPLIT, SLAB>;
  extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  // stage s: [A_hi | B_hi | A_lo | B_lo]
  auto stA = [&](int s, int part) { return smem + s * C::STAGE_BYTES + part * (C::A_BYTES + C::B_BYTES); };
  auto stB = [&](int s, int part) { return stA(s, part) + C::A_BYTES; };
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint64_t* fin = done + 1;          // the issuer's MMAs after it gave up
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (klen + C::BK - 1) / C::BK;
  const uint32_t stage_bytes = C::PARTS * (C::A_BYTES + (uint32_t)bn * SLAB);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    mbar_init(fin, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, C::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4 && lane == 0) {
    // ---- TMA producer
    int issued = 0;
    for (int kb = 0; kb < nk; kb++) {
      const int kx = kbase + kb * C::BK;
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (!mbar_wait(&empty[s], ph ^ 1)) {
        atomicOr(err, ERR_TIMEOUT_PRODUCER);
        break;
      }
      mbar_expect_tx(&full[s], stage_bytes);
      tma_load_3d(stA(s, 0), &maps.a, &full[s], kx, m0, za);
      tma_load_3d(stB(s, 0), &maps.b, &full[s], kx, n0, zb);
      if (SPLIT) {
        tma_load_3d(stA(s, 1), &maps.a_lo, &full[s], kx, m0, za);
        tma_load_3d(stB(s, 1), &maps.b_lo, &full[s], kx, n0, zb);
      }
      issued = kb + 1;
    }
    // the last fills of each stage land before the CTA can exit
    for (int q = max(0, issued - STAGES); q < issued; q++)
      mbar_wait_drain(&full[q % STAGES], (q / STAGES) & 1);
  } else if (warp == 5 && lane == 0) {
    // ---- MMA issuer
    const uint32_t ID = idesc(128, bn, FMT);
    bool ok = true;
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (!mbar_wait(&full[s], ph)) {
        atomicOr(err, ERR_TIMEOUT_MMA);
        ok = false;
        break;
      }
      tc_fence_after();
      const uint64_t ad = sdesc_k<SLAB>(smem_u32(stA(s, 0)));
      const uint64_t bd = sdesc_k<SLAB>(smem_u32(stB(s, 0)));
#pragma unroll
      for (int k = 0; k < C::BK / C::UK; k++)   // advance 32 bytes along K per MMA
        umma<FMT>(tmem, ad + 2 * k, bd + 2 * k, ID, (kb | k) != 0);
      if (SPLIT) {
        const uint64_t al = sdesc_k<SLAB>(smem_u32(stA(s, 1)));
        const uint64_t bl = sdesc_k<SLAB>(smem_u32(stB(s, 1)));
#pragma unroll
        for (int k = 0; k < C::BK / C::UK; k++) {
          umma<FMT>(tmem, ad + 2 * k, bl + 2 * k, ID, 1u);   // hi * lo
          umma<FMT>(tmem, al + 2 * k, bd + 2 * k, ID, 1u);   // lo * hi
        }
      }
      umma_commit(&empty[s]);
    }
    // every MMA issued above completes before the TMEM is freed: `done` releases the
    // epilogue; after a timeout `fin` only drains (the epilogue gives up on its own)
    uint64_t* last = ok ? done : fin;
    umma_commit(last);
    mbar_wait_drain(last, 0);
  }

  if (warp < 4) {
    // ---- epilogue: TMEM lane = tile row
    const bool ok = mbar_wait(done, 0);
    if (!ok) {
      if (lane == 0) atomicOr(err, ERR_TIMEOUT_EPILOGUE);
    } else {
      tc_fence_after();
      const int row = warp * 32 + lane;
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
      float v[32];
      if constexpr (Epi::kPair) {
        // columns [0, P) pair with [P, 2P): chunk c0 and chunk c0 + P reach the functor
        // together (P = epi.pair_stride(), a multiple of 32)
        const int P = epi.pair_stride();
        float u[32];
#pragma unroll 1
        for (int c0 = 0; c0 < P && c0 + P < bn + 1; c0 += 32) {
          tmem_ld32(trow + c0, v);
          tmem_ld32(trow + c0 + P, u);
          epi.pair(batch, row, m0 + row, c0, v, u);
        }
      } else if constexpr (Epi::kTile) {
        // the operand ring is idle once `done` has fired: reuse it for the fp32 tile, or,
        // when the ring cannot hold it (kHalfTile functors), for one half of the columns
        // at a time through epi.tile_part(..., first column, columns)
        float* tile = reinterpret_cast<float*>(smem);
        if constexpr (TileInRing<BN, STAGES, C::STAGE_BYTES>::value) {
#pragma unroll 1
          for (int c0 = 0; c0 < bn; c0 += 32) {
            tmem_ld32(trow + c0, v);
#pragma unroll
            for (int i = 0; i < 32; i++) tile[row * (BN + 1) + c0 + i] = v[i];
          }
          epi_bar();
          epi.tile(batch, mt, nt, tile, BN + 1, threadIdx.x);
        } else {
          constexpr int TC = BN / 2;
#pragma unroll 1
          for (int h = 0; h < 2; h++) {
            if (h) epi_bar();   // every thread is done with the first half
#pragma unroll 1
            for (int c0 = 0; c0 < TC; c0 += 32) {
              tmem_ld32(trow + h * TC + c0, v);
#pragma unroll
              for (int i = 0; i < 32; i++) tile[row * (TC + 1) + c0 + i] = v[i];
            }
            epi_bar();
            epi.tile_part(batch, mt, nt, tile, TC + 1, threadIdx.x, h * TC, TC);
          }
        }
      } else {
#pragma unroll 1
        for (int c0 = 0; c0 < bn; c0 += 32) {
          tmem_ld32(trow + c0, v);
          epi(batch, row, m0 + row, n0 + c0, v);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, C::TMEM_COLS);
}

template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int MINB = 1, int SLAB = 128>
__global__ void __launch_bounds__(192, MINB)
tc_gemm_kernel(const __grid_constant__ Maps maps, int K, int m_step, int n_step, int a_batched,
               int b_batched, int k_split, int m_fast, int z0, Epi epi, int* err) {
  // m_fast: M tiles along grid x, so the CTAs that share a B tile run together
  const int mt = m_fast ? blockIdx.x : blockIdx.y, nt = m_fast ? blockIdx.y : blockIdx.x;
  const int batch = z0 + blockIdx.z;
  // split-K: z selects the K range [z*k_split, (z+1)*k_split) of an unbatched product
  const int kbase = k_split ? batch * k_split : 0;
  const int klen = k_split ? min(k_split, K - kbase) : K;
  const int za = (a_batched && !k_split) ? batch : 0, zb = (b_batched && !k_split) ? batch : 0;
  gemm_tile<BN, STAGES, FMT, SPLIT, Epi, SLAB>(maps, mt, nt, mt * m_step, nt * n_step, batch, za,
                                               zb, kbase, klen, BN, epi, err);
}

// Several independent batched products (one per problem: a system of a heterogeneous
// batch) in one launch over a work list of (problem, batch, M tile, N tile): problem p
// owns the CTAs [tile0[p], tile0[p + 1]) of the 1-D grid, batch-major then M tiles then N
// tiles.  Each problem has its own tensor maps, K, row / column steps, tile width
// bn[p] <= BN and epilogue functor; the template (ring depth, precision, epilogue type) is
// shared.  No split-K.
template <class Epi, int NP>
struct MultiJob {
  Maps maps[NP];
  Epi epi[NP];
  int K[NP], m_step[NP], n_step[NP], bn[NP], m_tiles[NP], n_tiles[NP];
  int a_batched[NP], b_batched[NP];
  int tile0[NP + 1];
  int np;
};

template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int NP, int SLAB = 128>
__global__ void __launch_bounds__(192, 1)
tc_gemm_multi_kernel(const __grid_constant__ MultiJob<Epi, NP> job, int* err) {
  const int t = blockIdx.x;
  int p = 0;
  while (p + 1 < job.np && t >= job.tile0[p + 1]) p++;
  const int local = t - job.tile0[p];
  const int per = job.m_tiles[p] * job.n_tiles[p];
  const int batch = local / per, r = local - batch * per;
  const int nt = r % job.n_tiles[p], mt = r / job.n_tiles[p];
  gemm_tile<BN, STAGES, FMT, SPLIT, Epi, SLAB>(
      job.maps[p], mt, nt, mt * job.m_step[p], nt * job.n_step[p], batch,
      job.a_batched[p] ? batch : 0, job.b_batched[p] ? batch : 0, 0, job.K[p], job.bn[p],
      job.epi[p], err);
}

// ------------------------------------------------------------------ persistent form
// One CTA per SM walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...  The TMA
// producer (one thread) and the MMA issuer (one thread) run ahead across tile boundaries
// through the operand ring; the accumulator is double-buffered in TMEM (2 x TMEM_COLS
// columns), so the epilogue of tile i (EPI_WG warpgroups splitting the 32-column chunks)
// overlaps the main loop of tile i + 1.  Barriers: full/empty per ring stage, acc_full /
// acc_empty per accumulator buffer, fin for the issuer's last MMAs.  Every wait is
// bounded as in the per-tile kernel; a role that times out records the error and stops,
// and the others follow at their next wait.
struct TileSched {
  int m_tiles, n_tiles, nbatch, m_fast;
  int z0 = 0;   // first batch index of the launch (a walker group of a larger batch)
  AFQ_HD int total() const { return m_tiles * n_tiles * nbatch; }
  AFQ_D void decode(int t, int& z, int& mt, int& nt) const {
    const int per = m_tiles * n_tiles;
    const int zl = t / per;   // batch within the launch
    const int r = t - zl * per;
    z = z0 + zl;
    if (m_fast) {
      mt = r % m_tiles;
      nt = r / m_tiles;
    } else {
      nt = r % n_tiles;
      mt = r / n_tiles;
    }
  }
};

template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int EPI_WG, int SLAB = 128>
struct PCfg {
  using C = Cfg<BN, STAGES, FMT, SPLIT, SLAB>;
  static constexpr int NEPI = 128 * EPI_WG, THREADS = NEPI + 64;
  static constexpr uint32_t ACC_COLS = 2 * C::TMEM_COLS;
  static constexpr size_t SCRATCH = (size_t)EpiScratch<Epi>::value * EPI_WG;
  static constexpr size_t BAR = 8 * (2 * STAGES + 5);
  static constexpr size_t SMEM = 1024 + STAGES * C::STAGE_BYTES + SCRATCH + BAR + 16;
  static constexpr bool kFits = SMEM <= 227 * 1024 && ACC_COLS <= 512;
};

// Problems of a persistent launch: one (every single product), or several independent
// batched products (the systems of a heterogeneous batch) walked as one tile list.
// Problem p owns tiles [tile0[p], tile0[p + 1]), decoded by sched[p]; its tensor maps,
// K, row / column steps, split-K extent, tile width bn[p] <= BN (a multiple of 32; BN for
// promoting epilogues) and epilogue functor are its own.
//
// Chain launches (the kernel's CHAIN parameter): the problems are consecutive products of
// one batched chain (problem p + 1 reads what problem p wrote for the same batch), all of
// the same batch count and tiles per batch.  The tile list runs in pairs of walker waves
// of `wave` batches, problems in order within a pair (wave a problem 0, wave b problem 0,
// wave a problem 1, ...), so a wave's operands stay in L2 across its products and one
// wave's tiles fill the wait for the other's.  A tile of problem p > 0 waits until
// dep[z] >= p * dep_per (every tile of problem p - 1 of batch z has published: each
// epilogue warp adds 1 per tile, so dep_per = tiles per batch x epilogue warps).
// split[p] selects split or plain operands per problem within the split-capacity ring: a
// plain tile puts two consecutive K slabs in each stage (parts 0 and 1), so its MMAs run
// in the same K order as the plain ring's.
template <class Epi, int NP>
struct PJob {
  Maps maps[NP];
  Epi epi[NP];
  TileSched sched[NP];
  int K[NP], m_step[NP], n_step[NP], a_batched[NP], b_batched[NP], k_split[NP], bn[NP];
  int tile0[NP + 1];
  int np;
  // chain launches only
  int split[NP];
  unsigned* dep;
  int dep_per, wave, nbatch;
  // tile t -> problem p and its (batch z, M tile, N tile)
  AFQ_D void locate(int t, int& p, int& z, int& mt, int& nt) const {
    p = 0;
    if constexpr (NP > 1) {
      while (p + 1 < np && t >= tile0[p + 1]) p++;
      t -= tile0[p];
    }
    sched[p].decode(t, z, mt, nt);
  }
  // chain order: pairs of waves, problems in order within a pair
  AFQ_D void locate_chain(int t, int& p, int& z, int& mt, int& nt) const {
    const int per = sched[0].m_tiles * sched[0].n_tiles;
    const int nfull = nbatch / wave, rem = nbatch - nfull * wave;
    const int fpairs = nfull / 2;                      // pairs of two full waves
    const int tp = np * 2 * wave * per;                // tiles of a full pair
    int w0, za, zb;                                    // first wave, batches of waves a, b
    if (t < fpairs * tp) {
      const int q = t / tp;
      t -= q * tp;
      w0 = 2 * q;
      za = zb = wave;
    } else {
      t -= fpairs * tp;
      w0 = 2 * fpairs;
      const bool a_full = w0 < nfull;
      za = a_full ? wave : rem;
      zb = a_full ? (w0 + 1 < nfull ? wave : rem) : 0;
    }
    const int pp = (za + zb) * per;                    // tiles of one problem in the pair
    p = t / pp;
    int r = t - p * pp;
    int which = 0;
    if (r >= za * per) {
      r -= za * per;
      which = 1;
    }
    const int zl = r / per, ti = r - zl * per;
    z = (w0 + which) * wave + zl;
    const TileSched& sc = sched[p];
    if (sc.m_fast) {
      mt = ti % sc.m_tiles;
      nt = ti / sc.m_tiles;
    } else {
      nt = ti % sc.n_tiles;
      mt = ti / sc.n_tiles;
    }
  }
};

// Chain dependency counters: the epilogue publishes a finished tile with a release add,
// the waiting producer reads with acquire and then orders its TMA reads (async proxy)
// after the data it now sees (generic proxy).
AFQ_D unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
AFQ_D void red_release_gpu_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
AFQ_D void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int EPI_WG, int SLAB = 128,
          int NP = 1, bool CHAIN = false>
__global__ void __launch_bounds__(128 * EPI_WG + 64, 1)
tc_gemm_persistent_kernel(const __grid_constant__ PJob<Epi, NP> job, int* err) {
  using C = Cfg<BN, STAGES, FMT, SPLIT, SLAB>;
  using P = PCfg<BN, STAGES, FMT, SPLIT, Epi, EPI_WG, SLAB>;
  static_assert(!Epi::kTile, "tile epilogues reuse the operand ring: per-tile kernel only");
  static_assert(!CHAIN || (SPLIT && EpiPromote<Epi>::value == 0),
                "chain launches: split-capacity ring, no promotion");
  extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  auto stA = [&](int s, int part) { return smem + s * C::STAGE_BYTES + part * (C::A_BYTES + C::B_BYTES); };
  auto stB = [&](int s, int part) { return stA(s, part) + C::A_BYTES; };
  float* scratch = reinterpret_cast<float*>(smem + STAGES * C::STAGE_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE_BYTES + P::SCRATCH);
  uint64_t* empty = full + STAGES;
  uint64_t* accf = empty + STAGES;   // [2]
  uint64_t* acce = accf + 2;         // [2]
  uint64_t* fin = acce + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int WPROD = P::NEPI / 32, WMMA = WPROD + 1;
  constexpr int PK = EpiPromote<Epi>::value;
  static_assert(PK == 0 || !(Epi::kPair || EpiStaged<Epi>::value),
                "promotion: row-wise or kRegs functors");
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], P::NEPI);
    }
    mbar_init(fin, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, P::ACC_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int total = job.tile0[job.np];
  auto where = [&](int t, int& p, int& z, int& mt, int& nt) {
    if constexpr (CHAIN)
      job.locate_chain(t, p, z, mt, nt);
    else
      job.locate(t, p, z, mt, nt);
  };
  // split operands for problem p (chain launches choose per problem)
  auto split_of = [&](int p) {
    if constexpr (CHAIN) return job.split[p] != 0;
    else return SPLIT;
  };
  // stage fills of a tile: one K slab per stage, or two when a chain tile is plain
  auto fills = [&](int nk, bool sp) { return (CHAIN && !sp) ? (nk + 1) / 2 : nk; };
  // one problem: the epilogue functor as a local copy, so the compiler knows the
  // epilogue's global stores cannot change it (a reference into the parameter block makes
  // it reload the fields after every store); several problems, and the staged functors
  // (whose copies would spill beside their staging arrays): a reference
  using EpiHold = std::conditional_t<NP == 1 && !EpiStaged<Epi>::value, const Epi, const Epi&>;
  // K slabs of tile t's problem
  auto kslabs = [&](int p, int z, int& kbase) {
    const int ks = job.k_split[p];
    kbase = ks ? z * ks : 0;
    const int klen = ks ? min(ks, job.K[p] - kbase) : job.K[p];
    return (klen + C::BK - 1) / C::BK;
  };

  if (warp == WPROD && lane == 0) {
    // ---- TMA producer
    int g = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
      int p, z, mt, nt, kbase;
      where(t, p, z, mt, nt);
      const int nk = kslabs(p, z, kbase);
      const int za = (job.a_batched[p] && !job.k_split[p]) ? z : 0;
      const int zb = (job.b_batched[p] && !job.k_split[p]) ? z : 0;
      const int m0 = mt * job.m_step[p], n0 = nt * job.n_step[p];
      const Maps& maps = job.maps[p];
      const bool sp = split_of(p);
      const uint32_t part_bytes = C::A_BYTES + (uint32_t)job.bn[p] * SLAB;
      if constexpr (CHAIN) {
        if (p > 0) {   // every tile of problem p - 1 of batch z has published
          const unsigned target = (unsigned)(p * job.dep_per);
          const long long t0 = clock64();
          while (ld_acquire_gpu(job.dep + z) < target) {
            if (clock64() - t0 > g_tc_wait_clocks) {
              ok = false;
              break;
            }
          }
          if (!ok) {
            atomicOr(err, ERR_TIMEOUT_PRODUCER);
            break;
          }
          fence_proxy_async_global();
        }
      }
      const int nf = fills(nk, sp);
      for (int f = 0; f < nf; f++, g++) {
        const int s = g % STAGES;
        if (!mbar_wait(&empty[s], ((g / STAGES) & 1) ^ 1)) {
          atomicOr(err, ERR_TIMEOUT_PRODUCER);
          ok = false;
          break;
        }
        if (CHAIN && !sp) {   // plain chain tile: K slabs 2f and 2f + 1 in parts 0 and 1
          const int kb = 2 * f, two = kb + 1 < nk;
          mbar_expect_tx(&full[s], part_bytes * (two ? 2u : 1u));
          tma_load_3d(stA(s, 0), &maps.a, &full[s], kbase + kb * C::BK, m0, za);
          tma_load_3d(stB(s, 0), &maps.b, &full[s], kbase + kb * C::BK, n0, zb);
          if (two) {
            tma_load_3d(stA(s, 1), &maps.a, &full[s], kbase + (kb + 1) * C::BK, m0, za);
            tma_load_3d(stB(s, 1), &maps.b, &full[s], kbase + (kb + 1) * C::BK, n0, zb);
          }
          continue;
        }
        const int kx = kbase + f * C::BK;
        mbar_expect_tx(&full[s], C::PARTS * part_bytes);
        tma_load_3d(stA(s, 0), &maps.a, &full[s], kx, m0, za);
        tma_load_3d(stB(s, 0), &maps.b, &full[s], kx, n0, zb);
        if (SPLIT) {
          tma_load_3d(stA(s, 1), &maps.a_lo, &full[s], kx, m0, za);
          tma_load_3d(stB(s, 1), &maps.b_lo, &full[s], kx, n0, zb);
        }
      }
    }
    // the last fills of each stage land before the CTA can exit
    for (int q = max(0, g - STAGES); q < g; q++)
      mbar_wait_drain(&full[q % STAGES], (q / STAGES) & 1);
  } else if (warp == WMMA && lane == 0) {
    // ---- MMA issuer: one accumulator buffer per tile, or per K chunk when promoting
    int g = 0, li = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
      int p, z, mt, nt, kbase;
      where(t, p, z, mt, nt);
      const int nk = kslabs(p, z, kbase);
      const uint32_t ID = idesc(128, job.bn[p], FMT);
      const int nch = PK ? (nk + PK - 1) / PK : 1;
      const bool sp = split_of(p);
      if (CHAIN && !sp) {   // plain chain tile: two K slabs per stage, one accumulator
        const int b = li & 1;
        if (!mbar_wait(&acce[b], ((li >> 1) & 1) ^ 1)) {
          atomicOr(err, ERR_TIMEOUT_MMA);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + b * C::TMEM_COLS;
        const int nf = fills(nk, sp);
        for (int f = 0; f < nf; f++, g++) {
          const int s = g % STAGES;
          if (!mbar_wait(&full[s], (g / STAGES) & 1)) {
            atomicOr(err, ERR_TIMEOUT_MMA);
            ok = false;
            break;
          }
          tc_fence_after();
          const int nparts = 2 * f + 1 < nk ? 2 : 1;
          for (int part = 0; part < nparts; part++) {
            const uint64_t ad = sdesc_k<SLAB>(smem_u32(stA(s, part)));
            const uint64_t bd = sdesc_k<SLAB>(smem_u32(stB(s, part)));
#pragma unroll
            for (int k = 0; k < C::BK / C::UK; k++)
              umma<FMT>(d, ad + 2 * k, bd + 2 * k, ID, (f != 0 || part != 0 || k != 0) ? 1u : 0u);
          }
          umma_commit(&empty[s]);
        }
        if (!ok) break;
        umma_commit(&accf[b]);
        li++;
        continue;
      }
      for (int ch = 0; ch < nch && ok; ch++, li++) {
        const int b = li & 1;
        if (!mbar_wait(&acce[b], ((li >> 1) & 1) ^ 1)) {   // the epilogue released buffer b
          atomicOr(err, ERR_TIMEOUT_MMA);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + b * C::TMEM_COLS;
        const int kb0 = PK ? ch * PK : 0, kb1 = PK ? min(nk, kb0 + PK) : nk;
        for (int kb = kb0; kb < kb1; kb++, g++) {
          const int s = g % STAGES;
          if (!mbar_wait(&full[s], (g / STAGES) & 1)) {
            atomicOr(err, ERR_TIMEOUT_MMA);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad = sdesc_k<SLAB>(smem_u32(stA(s, 0)));
          const uint64_t bd = sdesc_k<SLAB>(smem_u32(stB(s, 0)));
#pragma unroll
          for (int k = 0; k < C::BK / C::UK; k++)
            umma<FMT>(d, ad + 2 * k, bd + 2 * k, ID, (kb != kb0 || k != 0) ? 1u : 0u);
          if (SPLIT) {
            const uint64_t al = sdesc_k<SLAB>(smem_u32(stA(s, 1)));
            const uint64_t bl = sdesc_k<SLAB>(smem_u32(stB(s, 1)));
#pragma unroll
            for (int k = 0; k < C::BK / C::UK; k++) {
              umma<FMT>(d, ad + 2 * k, bl + 2 * k, ID, 1u);
              umma<FMT>(d, al + 2 * k, bd + 2 * k, ID, 1u);
            }
          }
          umma_commit(&empty[s]);
        }
        if (!ok) break;
        umma_commit(&accf[b]);
      }
    }
    umma_commit(fin);   // fires once every MMA issued above has completed
    mbar_wait_drain(fin, 0);
  }

  if constexpr (PK > 0) {
    if (warp < WPROD) {
      // ---- promoting epilogue: warpgroup wg sums its columns over the K chunks
      constexpr int CPW = BN / EPI_WG;
      static_assert(CPW % 32 == 0, "promotion: whole 32-column chunks per warpgroup");
      const int wg = warp >> 2, wq = warp & 3;
      const int row = wq * 32 + lane;
      float* scr = scratch + (size_t)wg * (EpiScratch<Epi>::value / 4);
      float acc[CPW];
      int li = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        int p, z, mt, nt, kbase;
        job.locate(t, p, z, mt, nt);
        const int nk = kslabs(p, z, kbase);
        const int nch = (nk + PK - 1) / PK;
        EpiHold epi = job.epi[p];
        for (int ch = 0; ch < nch; ch++, li++) {
          const int b = li & 1;
          if (!mbar_wait(&accf[b], (li >> 1) & 1)) {
            if (lane == 0) atomicOr(err, ERR_TIMEOUT_EPILOGUE);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t trow =
              tmem + b * C::TMEM_COLS + ((uint32_t)(wq * 32) << 16) + (uint32_t)(wg * CPW);
          if (ch == 0) {
#pragma unroll
            for (int j = 0; j < CPW / 32; j++) tmem_ld32(trow + j * 32, acc + j * 32);
          } else {
#pragma unroll
            for (int j = 0; j < CPW / 32; j++) tmem_ld32_add(trow + j * 32, acc + j * 32);
          }
          tc_fence_before();
          mbar_arrive(&acce[b]);
        }
        if (!ok) break;
        if constexpr (EpiRegs<Epi>::value) {
          epi.regs(z, mt, nt, row, acc, scr, wg);
        } else {
          const int m0 = mt * job.m_step[p], n0 = nt * job.n_step[p];
#pragma unroll
          for (int j = 0; j < CPW / 32; j++) epi(z, row, m0 + row, n0 + wg * CPW + j * 32, acc + j * 32);
        }
      }
    }
  } else if (warp < WPROD) {
    // ---- epilogue: warpgroup wg takes chunks wg, wg + EPI_WG, ...; TMEM lane = tile row
    const int wg = warp >> 2, wq = warp & 3;
    const int row = wq * 32 + lane;
    int li = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, li++) {
      int p, z, mt, nt;
      where(t, p, z, mt, nt);
      EpiHold epi = job.epi[p];
      const int bn = job.bn[p];
      const int b = li & 1;
      bool got = mbar_wait(&accf[b], (li >> 1) & 1);
      // chain launches publish per warp: the warp decides as one whether to go on
      if constexpr (CHAIN) got = __all_sync(0xffffffffu, got);
      if (!got) {
        if (lane == 0) atomicOr(err, ERR_TIMEOUT_EPILOGUE);
        break;
      }
      tc_fence_after();
      if constexpr (CHAIN) {   // see what problem p - 1 published before reading its output
        if (p > 0) (void)ld_acquire_gpu(job.dep + z);
      }
      const uint32_t trow = tmem + b * C::TMEM_COLS + ((uint32_t)(wq * 32) << 16);
      const int m0 = mt * job.m_step[p], n0 = nt * job.n_step[p];
      float v[32];
      if constexpr (Epi::kPair) {
        const int Pw = epi.pair_stride();
        float u[32];
#pragma unroll 1
        for (int c0 = wg * 32; c0 < Pw && c0 + Pw < bn + 1; c0 += 32 * EPI_WG) {
          tmem_ld32(trow + c0, v);
          tmem_ld32(trow + c0 + Pw, u);
          epi.pair(z, row, m0 + row, c0, v, u);
        }
      } else if constexpr (EpiStaged<Epi>::value) {
        float* scr = scratch + (size_t)wg * (EpiScratch<Epi>::value / 4);
        auto ld = [&](int col, float* out) { tmem_ld32(trow + col, out); };
        epi.staged(z, mt, nt, row, ld, scr, wg);
      } else {
#pragma unroll 1
        for (int c0 = wg * 32; c0 < bn; c0 += 32 * EPI_WG) {
          tmem_ld32(trow + c0, v);
          epi(z, row, m0 + row, n0 + c0, v);
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[b]);
      if constexpr (CHAIN) {   // publish: this warp's writes of the tile are done
        __threadfence();
        __syncwarp();
        if (lane == 0) red_release_gpu_add(job.dep + z, 1u);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, P::ACC_COLS);
}

// ------------------------------------------------------------------ host side
// Tensor map of a [batch][rows][K] K-major operand (rows strided by ld elements, batches
// by sbatch elements), tiles of box_rows x slab bytes (128: SWIZZLE_128B, 64:
// SWIZZLE_64B), zero fill outside.
inline CUresult make_kmajor_map(CUtensorMap* map, const void* base, bool fp32, uint64_t K,
                                uint64_t rows, uint64_t batch, uint64_t ld, uint64_t sbatch,
                                uint32_t box_rows, uint32_t slab = 128) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&encode, cudaEnableDefault,
                                &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !encode)
      return CUDA_ERROR_NOT_FOUND;
  }
  const uint32_t esz = fp32 ? 4 : 2;
  cuuint64_t dims[3] = {K, rows, batch};
  cuuint64_t strides[2] = {ld * esz, (batch > 1 ? sbatch : rows * ld) * esz};
  cuuint32_t box[3] = {slab / esz, box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return encode(map, fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3,
                const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                slab == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

struct GemmShape {
  int M, N, K, batch;  // batch = number of z slices (batches, or K splits when k_split > 0)
  int m_step;          // rows between consecutive M tiles (128 unless aligned to row groups)
  int m_tiles;         // number of M tiles
  bool a_batched, b_batched;
  int k_split;         // 0, or the K extent of each z slice (a multiple of the K slab)
  bool m_fast = false; // raster M tiles fastest (B tiles reused from L2 across M)
  int n_step = 0;      // columns between consecutive N tiles (0: BN); a smaller step lets a
                       // tile hold whole column groups that do not fill BN
  int z0 = 0;          // first batch of the launch: batches z0 .. z0 + batch - 1 of operands
                       // (and epilogue outputs) that hold more (no split-K)
};

template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int MINB = 1, int SLAB = 128>
cudaError_t launch(const Maps& maps, const GemmShape& g, const Epi& epi, int* err,
                   cudaStream_t st) {
  using C = Cfg<BN, STAGES, FMT, SPLIT, SLAB>;
  static_assert(!Epi::kTile || TileInRing<BN, STAGES, C::STAGE_BYTES>::value ||
                    (EpiHalfTile<Epi>::value && BN % 64 == 0 &&
                     (size_t)128 * (BN / 2 + 1) * 4 <= (size_t)STAGES * C::STAGE_BYTES),
                "tile epilogue needs the operand ring to hold the fp32 tile (or half of it)");
  static_assert(MINB * C::SMEM <= 228 * 1024 && MINB * C::TMEM_COLS <= 512,
                "CTAs per SM exceed shared memory or TMEM");
  auto kern = tc_gemm_kernel<BN, STAGES, FMT, SPLIT, Epi, MINB, SLAB>;
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(C::SMEM, [kern](size_t b) {
    cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
    if (r == cudaSuccess && MINB > 1)
      r = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    return r;
  });
  if (e != cudaSuccess) return e;
  const int ns = g.n_step > 0 ? g.n_step : BN;
  const unsigned ntiles = (g.N + ns - 1) / ns;
  dim3 grid(g.m_fast ? g.m_tiles : ntiles, g.m_fast ? ntiles : g.m_tiles, g.batch);
  kern<<<grid, 192, C::SMEM, st>>>(maps, g.K, g.m_step, ns, g.a_batched, g.b_batched, g.k_split,
                                    g.m_fast ? 1 : 0, g.z0, epi, err);
  return cudaGetLastError();
}

// One launch over the work list of job.np problems (job.tile0 filled by the caller: the
// running sum of batch x m_tiles x n_tiles).  Tile widths must be multiples of 32 within BN.
template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int NP, int SLAB = 128>
cudaError_t launch_multi(const MultiJob<Epi, NP>& job, int* err, cudaStream_t st) {
  using C = Cfg<BN, STAGES, FMT, SPLIT, SLAB>;
  static_assert(!Epi::kTile || TileInRing<BN, STAGES, C::STAGE_BYTES>::value ||
                    (EpiHalfTile<Epi>::value && BN % 64 == 0 &&
                     (size_t)128 * (BN / 2 + 1) * 4 <= (size_t)STAGES * C::STAGE_BYTES),
                "tile epilogue needs the operand ring to hold the fp32 tile (or half of it)");
  static_assert(C::SMEM <= 227 * 1024 && C::TMEM_COLS <= 512, "shared memory or TMEM");
  if (job.np < 1 || job.np > NP || job.tile0[0] != 0) return cudaErrorInvalidValue;
  for (int p = 0; p < job.np; p++) {
    if (job.bn[p] < 32 || job.bn[p] > BN || job.bn[p] % 32 || job.m_tiles[p] < 1 ||
        job.n_tiles[p] < 1 || job.K[p] < 1 || job.tile0[p + 1] < job.tile0[p] ||
        (job.tile0[p + 1] - job.tile0[p]) % (job.m_tiles[p] * job.n_tiles[p]))
      return cudaErrorInvalidValue;
  }
  const int total = job.tile0[job.np];
  if (total <= 0) return cudaSuccess;
  auto kern = tc_gemm_multi_kernel<BN, STAGES, FMT, SPLIT, Epi, NP, SLAB>;
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(C::SMEM, [kern](size_t b) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
  });
  if (e != cudaSuccess) return e;
  kern<<<total, 192, C::SMEM, st>>>(job, err);
  return cudaGetLastError();
}

inline int sm_count() {
  static const int n = [] {   // initialised once, thread-safe (every device is a B200)
    int dev = 0, c = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0)
      c = 148;
    return c;
  }();
  return n;
}

template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int EPI_WG = 1, int SLAB = 128>
cudaError_t launch_persistent(const Maps& maps, const GemmShape& g, const Epi& epi, int* err,
                              cudaStream_t st) {
  using P = PCfg<BN, STAGES, FMT, SPLIT, Epi, EPI_WG, SLAB>;
  static_assert(P::kFits, "persistent configuration exceeds shared memory or TMEM");
  auto kern = tc_gemm_persistent_kernel<BN, STAGES, FMT, SPLIT, Epi, EPI_WG, SLAB>;
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(P::SMEM, [kern](size_t b) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
  });
  if (e != cudaSuccess) return e;
  const int ns = g.n_step > 0 ? g.n_step : BN;
  PJob<Epi, 1> job;
  job.maps[0] = maps;
  job.epi[0] = epi;
  job.sched[0] = TileSched{g.m_tiles, (g.N + ns - 1) / ns, g.batch, g.m_fast ? 1 : 0, g.z0};
  job.K[0] = g.K;
  job.m_step[0] = g.m_step;
  job.n_step[0] = ns;
  job.a_batched[0] = g.a_batched;
  job.b_batched[0] = g.b_batched;
  job.k_split[0] = g.k_split;
  job.bn[0] = BN;
  job.tile0[0] = 0;
  job.tile0[1] = job.sched[0].total();
  job.np = 1;
  const int total = job.tile0[1];
  if (total <= 0) return cudaSuccess;
  const int grid = total < sm_count() ? total : sm_count();
  kern<<<grid, P::THREADS, P::SMEM, st>>>(job, err);
  return cudaGetLastError();
}

// Chain launch: the persistent kernel over a dependency-ordered tile list (PJob chain
// fields).  Its CTAs wait on one another's tiles, so the launch is cooperative: every CTA
// is resident at once (one per SM at most), and no CTA waits on one that has not started.
// Every problem: the same batch count and tiles per batch; job.dep zeroed by the caller
// (nbatch counters) before the launch.
template <int BN, int STAGES, int FMT, class Epi, int EPI_WG, int NP>
cudaError_t launch_chain(PJob<Epi, NP>& job, int* err, cudaStream_t st) {
  using P = PCfg<BN, STAGES, FMT, true, Epi, EPI_WG>;
  static_assert(P::kFits, "persistent configuration exceeds shared memory or TMEM");
  if (job.np < 1 || job.np > NP || job.wave < 1 || job.nbatch < 1 || !job.dep)
    return cudaErrorInvalidValue;
  const int per = job.sched[0].m_tiles * job.sched[0].n_tiles;
  for (int p = 0; p < job.np; p++)
    if (job.bn[p] < 32 || job.bn[p] > BN || job.bn[p] % 32 || job.K[p] < 1 || job.k_split[p] ||
        job.sched[p].m_tiles * job.sched[p].n_tiles != per || job.sched[p].nbatch != job.nbatch ||
        job.sched[p].z0 != 0)
      return cudaErrorInvalidValue;
  job.dep_per = per * 4 * EPI_WG;   // one publish per epilogue warp per tile
  job.tile0[0] = 0;
  job.tile0[job.np] = job.np * job.nbatch * per;
  const int total = job.tile0[job.np];
  auto kern = tc_gemm_persistent_kernel<BN, STAGES, FMT, true, Epi, EPI_WG, 128, NP, true>;
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(P::SMEM, [kern](size_t b) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
  });
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P::THREADS, P::SMEM);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = total < sm_count() ? total : sm_count();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(P::THREADS);
  cfg.dynamicSmemBytes = P::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, (const PJob<Epi, NP>)job, err);
}

// The persistent kernel over job.np <= NP problems (no promoting epilogue): tile0 and the
// schedules filled by the caller; tile widths multiples of 32 within BN.
template <int BN, int STAGES, int FMT, bool SPLIT, class Epi, int EPI_WG, int NP>
cudaError_t launch_persistent_multi(const PJob<Epi, NP>& job, int* err, cudaStream_t st) {
  using P = PCfg<BN, STAGES, FMT, SPLIT, Epi, EPI_WG>;
  static_assert(P::kFits, "persistent configuration exceeds shared memory or TMEM");
  static_assert(EpiPromote<Epi>::value == 0, "promoting epilogues need the full tile width");
  if (job.np < 1 || job.np > NP || job.tile0[0] != 0) return cudaErrorInvalidValue;
  for (int p = 0; p < job.np; p++)
    if (job.bn[p] < 32 || job.bn[p] > BN || job.bn[p] % 32 || job.K[p] < 1 ||
        job.tile0[p + 1] - job.tile0[p] != job.sched[p].total())
      return cudaErrorInvalidValue;
  const int total = job.tile0[job.np];
  if (total <= 0) return cudaSuccess;
  auto kern = tc_gemm_persistent_kernel<BN, STAGES, FMT, SPLIT, Epi, EPI_WG, 128, NP>;
  static DeviceAttr attr;
  cudaError_t e = attr.ensure(P::SMEM, [kern](size_t b) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
  });
  if (e != cudaSuccess) return e;
  const int grid = total < sm_count() ? total : sm_count();
  kern<<<grid, P::THREADS, P::SMEM, st>>>(job, err);
  return cudaGetLastError();
}

}  // namespace tc
