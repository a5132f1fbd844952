// umma.cuh -- the sm_100a tensor-core GEMM engine (tcgen05 + TMA + TMEM).
//
// Computes, for every batch b < nbatch,
//     D_b[p][q] = sum_k X_b[p][k] * Y_b[q][k]          (both operands K-major)
// and hands each 32-column strip of a 128 x BN accumulator tile to an
// epilogue functor.  This is the B200 replacement of the reference's whole
// GEMM machinery: the OpenMP N split and thread-0 packing of
// src/gemm_driver.c:136-188 become a persistent grid over output tiles, the
// packing of src/gemm_copy.c becomes TMA loads into 128B-swizzled shared
// memory, and the 24x8 FMA register tile of src/kernel/gemm_kernel.S becomes
// 128 x BN x 32-byte tcgen05.mma instructions accumulating in TMEM.
//
// Roles (192 threads, one CTA per SM):
//   warp 0      TMA producer: fills a STAGES-deep ring of (X, Y) K-blocks.
//   warp 1      TMEM owner + MMA issuer (one elected lane).
//   warps 2..5  epilogue: tcgen05.ld of their 32-lane quarter of the
//               accumulator, then the functor.
// TMEM holds two accumulators (2 x BN columns) so the epilogue of tile i
// overlaps the MMAs of tile i+1.
//
// Every mbarrier wait is bounded (Problem::wait_ns of wall time from
// %globaltimer, 2 s unless a test shortens it); on expiry the waiter stores
// B2_ERR_TIMEOUT into the error word (device memory, or host memory mapped
// into the device so the host reads it without a copy) and raises a shared
// abort flag, every role leaves its loop, and once all roles have stopped the
// producer waits (again bounded) for the copies still in flight; TMEM is
// freed and the kernel returns.  Nothing traps.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "b2_internal.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace umma {

// KIND_I8: signed 8-bit operands, KIND_U8: unsigned 8-bit (both kind::i8, S32
// accumulators); KIND_BF16: kind::f16 with BF16 operands; KIND_TF32: kind::tf32.
enum Kind { KIND_I8 = 0, KIND_BF16 = 1, KIND_TF32 = 2, KIND_U8 = 3 };

constexpr int BM = 128;            // accumulator lanes (X rows) per tile
constexpr int KBLOCK_BYTES = 128;  // one 128B swizzle atom along K per stage
constexpr int THREADS = 192;
constexpr uint64_t B2_WAIT_NS = 2000000000ull;  // 2 s per wait: far above any legal wait

// Wait limit (ns) given to the next launches and the number of launches that
// withhold their first K-block's TMA loads (a stall made on purpose, used only
// by the failure-detection tests through b2_test_bounded_wait).
extern std::atomic<unsigned long long> g_wait_ns;
extern std::atomic<int> g_withhold;
// Reads the two settings above for one launch (consumes one withheld launch).
inline void launch_wait_settings(uint64_t *wait_ns, int *withhold) {
  *wait_ns = g_wait_ns.load(std::memory_order_relaxed);
  int w = g_withhold.load(std::memory_order_relaxed);
  while (w > 0 && !g_withhold.compare_exchange_weak(w, w - 1)) {
  }
  *withhold = w > 0 ? 1 : 0;
}

__host__ __device__ constexpr bool is_int8(int kind) { return kind == KIND_I8 || kind == KIND_U8; }
__host__ __device__ constexpr int elem_bytes(int kind) { return is_int8(kind) ? 1 : kind == KIND_BF16 ? 2 : 4; }

// Instruction descriptor (PTX ISA tcgen05 "instruction descriptor" for
// .kind::f16 / .kind::tf32 / .kind::i8): D format at [4,6), A/B formats at
// [7,10)/[10,13), K-major A and B (bits 15/16 clear), N>>3 at [17,23),
// M>>4 at [24,29).
__host__ __device__ constexpr uint32_t make_idesc(int kind, int m, int n) {
  const uint32_t dfmt = is_int8(kind) ? 2u : 1u;        // S32 : F32
  const uint32_t abfmt = kind == KIND_U8 ? 0u             // unsigned 8-bit
                         : kind == KIND_I8 ? 1u           // signed 8-bit
                         : kind == KIND_BF16 ? 1u          // BF16
                                             : 2u;         // TF32
  return (dfmt << 4) | (abfmt << 7) | (abfmt << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

// ----------------------------------------------------------- PTX helpers --
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// Completes `bytes` of a phase's expected transaction count without a copy
// (for copies that were never issued, so that the phase can still complete).
__device__ __forceinline__ void mbar_complete_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Records a timeout in the error word.  A plain store (every writer stores
// the same value), so the word may live in mapped host memory.
__device__ __forceinline__ void record_timeout(int *derr) {
  *reinterpret_cast<volatile int *>(derr) = (int)B2_ERR_TIMEOUT;
  __threadfence_system();
}

// Bounded wait.  Returns false if the wait was abandoned (timeout here or an
// abort raised by another role); a timeout records the error.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          int *derr, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0) {
      if (*abort_flag) return false;
      if (gtimer() - t0 > limit_ns) {
        *abort_flag = 1;
        record_timeout(derr);
        return false;
      }
    }
  }
}

// Bounded plain wait (no abort flag, no error): used while draining.
__device__ __forceinline__ void mbar_wait_drain(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = gtimer();
  while (!mbar_try_wait(bar, parity) && gtimer() - t0 < limit_ns) {
  }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

template <int KIND>
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  if constexpr (is_int8(KIND)) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else if constexpr (KIND == KIND_BF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}

// Shared-memory matrix descriptor for a K-major operand tile stored as rows of
// 128 bytes with the 128B swizzle (the layout TMA writes with
// CU_TENSOR_MAP_SWIZZLE_128B): start address >> 4 at [0,14), leading byte
// offset (unused for this layout) = 1 at [16,30), stride byte offset = 1024 B
// (8 rows x 128 B) >> 4 at [32,46), descriptor version 1 at [46,48), base
// offset 0 (tile bases are 1024-B aligned), swizzle mode 2 = 128B at [61,64).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
// Wait for tcgen05.ld; the registers are threaded through so no use of them
// can be scheduled above the wait.
__device__ __forceinline__ void tmem_ld_wait(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                 "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// ---------------------------------------------------------------- kernel --
struct Problem {
  int P, Q;        // rows of X and of Y (output tile space P x Q)
  int kblocks;     // K extent in 128-byte blocks
  int ksplit;      // K ranges per output tile (split-K; 1 = whole K in one accumulator)
  int kb_per_split;  // K blocks per range (every range is non-empty)
  int nbatch;      // independent products (3-D tensor maps, batch = outer coordinate)
  const int *nbatch_dev;  // if set: the batch count actually run (<= nbatch), read on the device
  int tiles_p, tiles_q;
  int group;       // tile rasterisation: GROUP rows of P tiles share a sweep over Q
  int *derr;       // device error word
  // Three-term interleave (0 = off): K' block j is term j % 3 of K block j / 3;
  // the operands store 2 segments of seg_kb K blocks (0 = big, 1 = small) and
  // bit t of seg_x / seg_y names the segment term t reads.  The big part that
  // two terms share is read from DRAM once: its second load follows the first
  // within three K' blocks and is served by L2.
  int seg_kb;
  unsigned seg_x, seg_y;
  uint64_t wait_ns;  // limit of every bounded wait
  int withhold;      // test only: the first fill of each producer posts its
                     // byte count but issues no copy (the wait for it times out)
};

template <int BN, int STAGES>
struct SmemLayout {
  static constexpr int X_BYTES = BM * KBLOCK_BYTES;
  static constexpr int Y_BYTES = BN * KBLOCK_BYTES;
  static constexpr int STAGE_BYTES = X_BYTES + Y_BYTES;
  static constexpr int BAR_OFF = STAGES * STAGE_BYTES;
  // full[S], empty[S], tfull[2], tempty[2], drain, then tmem address (+0),
  // abort flag (+8) and the CTA pair's odd-CTA fill count (+12)
  static constexpr int BAR_BYTES = (2 * STAGES + 5) * 8;
  static constexpr int TOTAL = BAR_OFF + BAR_BYTES + 16 + 1024;  // + alignment slack
};

__device__ __forceinline__ void tile_coords(const Problem &pr, int t, int &b, int &tp, int &tq) {
  const int per_batch = pr.tiles_p * pr.tiles_q;
  b = t / per_batch;
  const int r = t - b * per_batch;
  const int gsz = pr.group * pr.tiles_q;
  const int g = r / gsz;
  const int first_p = g * pr.group;
  const int gp = min(pr.group, pr.tiles_p - first_p);
  const int rr = r - g * gsz;
  tp = first_p + rr % gp;
  tq = rr / gp;
}

// TMEM columns of an allocation: a power of two, at least 32.
__host__ __device__ constexpr int tmem_cols(int need) {
  return need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
}

// NACC = 1: every (batch, tile, K range) is its own work unit.  NACC > 1: a
// work unit is a tile, and the unit multiplies batches 0 .. NACC-1 of the
// operands into NACC accumulators that its epilogue receives together
// (epi(p, q0, v0, v1, v2) for NACC = 3: the three real products of the 3M
// method); no split-K.
template <int KIND, int BN, int STAGES, class Epi, int NACC = 1>
__global__ void __launch_bounds__(THREADS, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmX,
                     const __grid_constant__ CUtensorMap tmY, const Problem pr, const Epi epi) {
  using L = SmemLayout<BN, STAGES>;
  // accumulator sets: two (the epilogue of a unit overlaps the next unit's
  // MMAs) when they fit in TMEM's 512 columns, else one
  constexpr int SETS = 2 * NACC * BN <= 512 ? 2 : 1;
  static_assert(NACC * BN <= 512, "one set of accumulators must fit in TMEM");
  static_assert(NACC == 1 || NACC == 3, "one accumulator, or three for the 3M products");
  static_assert(NACC == 3 || SETS == 2, "the single-accumulator engine double-buffers");
  constexpr int TCOLS = tmem_cols(SETS * NACC * BN);
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *gbase = smem_raw + (base - raw);
  const uint32_t bar0 = base + L::BAR_OFF;
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
  auto tfull_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + a); };
  auto tempty_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + 2 + a); };
  const uint32_t drain_bar = bar0 + 8u * (2 * STAGES + 4);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gbase + L::BAR_OFF + L::BAR_BYTES);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(gbase + L::BAR_OFF + L::BAR_BYTES + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nbatch = pr.nbatch_dev ? min(*pr.nbatch_dev, pr.nbatch) : pr.nbatch;
  const int total_tiles = pr.tiles_p * pr.tiles_q * (NACC == 1 ? nbatch : 1);
  // work units: (tile, K range) pairs, the K range innermost
  const int total_units = total_tiles * pr.ksplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull_bar(a), 1);
      mbar_init(tempty_bar(a), 4);  // one arrival per epilogue warp
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    prefetch_tmap(&tmX);
    prefetch_tmap(&tmY);
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  long issued = 0;  // fills posted by the producer (warp 0, lane 0)
  if (warp == 0) {
    // ------------------------------------------------------ TMA producer
    if (lane == 0) {
      const int kcoord = KBLOCK_BYTES / elem_bytes(KIND);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < total_units && ok; u += gridDim.x) {
        const int t = u / pr.ksplit, ks = u - t * pr.ksplit;
        int b, tp, tq;
        tile_coords(pr, t, b, tp, tq);
        const int kb0 = ks * pr.kb_per_split, kb1 = min(pr.kblocks, kb0 + pr.kb_per_split);
        // NACC > 1: the unit's batches interleaved per K block (the three
        // products of a K block back to back, so the operand panels of all
        // batches stay in L2 together)
        for (int kbb = kb0; kbb < kb0 + NACC * (kb1 - kb0) && ok; ++kbb) {
          if (NACC > 1) b = (kbb - kb0) % NACC;
          const int kb = NACC > 1 ? kb0 + (kbb - kb0) / NACC : kbb;
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag, pr.derr, pr.wait_ns)) {
            ok = false;
            break;
          }
          const uint32_t sx = base + stage * L::STAGE_BYTES;
          const uint32_t sy = sx + L::X_BYTES;
          mbar_expect_tx(full_bar(stage), L::STAGE_BYTES);
          int kx = kb * kcoord, ky = kx;
          if (pr.seg_kb) {
            const int kq = kb / 3, tt = kb - 3 * kq;
            kx = ((int)((pr.seg_x >> tt) & 1u) * pr.seg_kb + kq) * kcoord;
            ky = ((int)((pr.seg_y >> tt) & 1u) * pr.seg_kb + kq) * kcoord;
          }
          if (!(pr.withhold && issued == 0)) {
            tma_load_3d(sx, &tmX, full_bar(stage), kx, tp * BM, b);
            tma_load_3d(sy, &tmY, full_bar(stage), ky, tq * BN, b);
          }
          ++issued;
          if (++stage == STAGES) { stage = 0; phase ^= 1u; }
        }
      }
    }
  } else if (warp == 1) {
    // -------------------------------------------------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = make_idesc(KIND, BM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < total_units && ok; u += gridDim.x, ++it) {
        const int ks = u % pr.ksplit;
        const int kb0 = ks * pr.kb_per_split, kb1 = min(pr.kblocks, kb0 + pr.kb_per_split);
        const int acc = it % SETS;
        const uint32_t acc_phase = (uint32_t)((it / SETS) & 1);
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag, pr.derr, pr.wait_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int kbb = kb0; kbb < kb0 + NACC * (kb1 - kb0); ++kbb) {
          const int bi = NACC > 1 ? (kbb - kb0) % NACC : 0;
          const int kb = NACC > 1 ? kb0 + (kbb - kb0) / NACC : kbb;
          const uint32_t d_tmem = tmem_base + (uint32_t)((acc * NACC + bi) * BN);
          if (!mbar_wait(full_bar(stage), phase, abort_flag, pr.derr, pr.wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sx = base + stage * L::STAGE_BYTES;
          const uint32_t sy = sx + L::X_BYTES;
#pragma unroll
          for (int kk = 0; kk < KBLOCK_BYTES / 32; ++kk) {
            tc_mma<KIND>(d_tmem, sw128_desc(sx + kk * 32), sw128_desc(sy + kk * 32), idesc,
                         (kb != kb0 || kk) ? 1u : 0u);
          }
          tc_commit(empty_bar(stage));  // frees the stage once these MMAs have read it
          if (++stage == STAGES) { stage = 0; phase ^= 1u; }
        }
        if (!ok) break;
        tc_commit(tfull_bar(acc));
      }
      // All MMAs issued so far complete before the drain barrier flips.
      tc_commit(drain_bar);
      mbar_wait_drain(drain_bar, 0, pr.wait_ns);
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int quarter = warp & 3;  // TMEM lanes this warp may access
    int it = 0;
    for (int u = blockIdx.x; u < total_units; u += gridDim.x, ++it) {
      const int t = u / pr.ksplit, ks = u - t * pr.ksplit;
      int b, tp, tq;
      tile_coords(pr, t, b, tp, tq);
      const int acc = it % SETS;
      const bool ok =
          mbar_wait(tfull_bar(acc), (uint32_t)((it / SETS) & 1), abort_flag, pr.derr, pr.wait_ns);
      if (!__all_sync(0xffffffffu, ok)) break;  // keep the warp converged for tcgen05.ld
      tc_fence_after();
      const int p = tp * BM + quarter * 32 + lane;
      const uint32_t taddr =
          tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * NACC * BN);
#pragma unroll 1
      for (int c = 0; c < BN / 32; ++c) {
        if constexpr (NACC == 1) {
          uint32_t v[32];
          tmem_ld32(taddr + (uint32_t)(c * 32), v);
          tmem_ld_wait(v);
          epi(b * pr.ksplit + ks, p, tq * BN + c * 32, v);  // batch x K range
        } else {
          uint32_t v0[32], v1[32], v2[32];
          tmem_ld32(taddr + (uint32_t)(c * 32), v0);
          tmem_ld32(taddr + (uint32_t)(BN + c * 32), v1);
          tmem_ld32(taddr + (uint32_t)(2 * BN + c * 32), v2);
          tmem_ld_wait(v0);
          tmem_ld_wait(v1);
          tmem_ld_wait(v2);
          epi(p, tq * BN + c * 32, v0, v1, v2);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty_bar(acc));
    }
  }

  tc_fence_before();
  __syncthreads();  // every role has left its loop: the abort flag is final
  tc_fence_after();
  if (warp == 0 && lane == 0 && *abort_flag) {
    // Abandoned: wait (bounded) until the copies of the newest fill of every
    // stage have landed (older fills were consumed), so no TMA writes into
    // shared memory after this CTA retires.  A withheld fill never receives
    // its bytes; they are completed here so its phase can still flip.
    const long first = issued - STAGES > 0 ? issued - STAGES : 0;
    for (long i = first; i < issued; ++i) {
      const int s = (int)(i % STAGES);
      if (pr.withhold && i == 0) mbar_complete_tx(full_bar(s), L::STAGE_BYTES);
      mbar_wait_drain(full_bar(s), (uint32_t)((i / STAGES) & 1), pr.wait_ns);
    }
  }
  if (warp == 1) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                 "r"(TCOLS));
  }
}

// ------------------------------------------------- CTA-pair (cta_group::2) --
// The same product (work units of tile x K range, the three-term segment map)
// on a cluster of two CTAs that execute one 256 x BN MMA
// together (tcgen05.mma.cta_group::2): CTA r of the pair stages X rows
// [256 tp + 128 r, +128) and Y rows [BN tq + (BN/2) r, +BN/2) of every
// K-block in its own shared memory, and the even ("leader") CTA issues the
// MMAs, which read both CTAs' tiles and leave rows 128 r.. of the 256 x BN
// accumulator in CTA r's TMEM.  Per MMA each SM loads a third less operand
// data than the single-CTA 128 x 256 tile (32 KB vs 48 KB per K-block), which
// is what keeps the tensor pipe fed from L2.
//
// Protocol (all loads are plain per-CTA TMA loads; none is multicast):
//   full[s]   only the leader's is used: its producer posts expect_tx for both
//             CTAs' bytes, and both CTAs' loads complete_tx on it (the
//             .cta_group::2 load form with the leader's barrier address).
//   empty[s]  one per CTA; the leader's commit arrives on both (commit
//             multicast to the pair).
//   tfull[a]  one per CTA; the leader's commit arrives on both.
//   tempty[a] only the leader's is used: 8 arrivals, the 4 epilogue warps of
//             each CTA (remote arrive from the odd CTA).
// A timeout in either CTA raises the abort flag of both.  The pair meets in a
// cluster barrier before TMEM is freed, so no MMA of the leader can still be
// writing the odd CTA's TMEM, and neither CTA leaves while the other's copies
// may still signal its barriers.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_rank(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void st_cluster_u32(uint32_t cluster_addr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(cluster_addr), "r"(v) : "memory");
}
// Per-CTA load into this CTA's shared memory, completing on a barrier that may
// be the peer's (the pair form of the bulk tensor copy; no multicast).
__device__ __forceinline__ void tma_load_3d_pair(uint32_t dst, const CUtensorMap *map,
                                                 uint32_t bar_cluster, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(bar_cluster), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
// Arrive (once the pair's MMAs issued so far complete) on the barrier at the
// same offset in every CTA named by `mask`.
__device__ __forceinline__ void tc_commit_pair(uint32_t bar, uint16_t mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(bar),
      "h"(mask)
      : "memory");
}
template <int KIND>
__device__ __forceinline__ void tc_mma_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  if constexpr (is_int8(KIND)) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else if constexpr (KIND == KIND_BF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}

// Bounded wait that also raises the peer CTA's abort flag on a timeout.
__device__ __forceinline__ bool mbar_wait_pair(uint32_t bar, uint32_t parity,
                                               volatile int *abort_flag, uint32_t peer_abort,
                                               int *derr, uint64_t limit_ns) {
  if (mbar_wait(bar, parity, abort_flag, derr, limit_ns)) return true;
  st_cluster_u32(peer_abort, 1u);
  return false;
}

constexpr int PAIR_BM = 2 * BM;  // output rows per pair tile

template <int KIND, int BN, int STAGES, class Epi>
__global__ void __launch_bounds__(THREADS, 1)
    umma_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmX,
                          const __grid_constant__ CUtensorMap tmY, const Problem pr,
                          const Epi epi) {
  using L = SmemLayout<BN / 2, STAGES>;  // per CTA: 128 X rows + BN/2 Y rows per stage
  static_assert(BN % 32 == 0 && BN >= 64 && BN <= 256, "pair MMA N in [64, 256]");
  static_assert(2 * BN <= 512, "two accumulators must fit in TMEM");
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *gbase = smem_raw + (base - raw);
  const uint32_t bar0 = base + L::BAR_OFF;
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
  auto tfull_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + a); };
  auto tempty_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + 2 + a); };
  const uint32_t drain_bar = bar0 + 8u * (2 * STAGES + 4);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gbase + L::BAR_OFF + L::BAR_BYTES);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(gbase + L::BAR_OFF + L::BAR_BYTES + 8);
  // the odd CTA's fill count, stored into the leader's copy of this word
  volatile uint32_t *odd_fills =
      reinterpret_cast<volatile uint32_t *>(gbase + L::BAR_OFF + L::BAR_BYTES + 12);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int pair = (int)cluster_id_x(), npairs = (int)cluster_count_x();
  const int nbatch = pr.nbatch_dev ? min(*pr.nbatch_dev, pr.nbatch) : pr.nbatch;
  const int total_tiles = pr.tiles_p * pr.tiles_q * nbatch;
  // work units: (tile, K range) pairs, the K range innermost
  const int total_units = total_tiles * pr.ksplit;
  const uint32_t peer_abort = map_rank(smem_u32((const void *)abort_flag), rank ^ 1u);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull_bar(a), 1);
      mbar_init(tempty_bar(a), 8);  // 4 epilogue warps in each CTA of the pair
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    *odd_fills = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    prefetch_tmap(&tmX);
    prefetch_tmap(&tmY);
  }
  cluster_sync();  // both CTAs' barriers exist before any remote signal
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(2 * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  cluster_sync();  // both CTAs hold the accumulator columns before the first MMA
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  long issued = 0;  // fills this CTA's producer (warp 0, lane 0) took part in
  if (warp == 0) {
    // ------------------------------------------------------ TMA producer
    if (lane == 0) {
      const int kcoord = KBLOCK_BYTES / elem_bytes(KIND);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int u = pair; u < total_units && ok; u += npairs) {
        const int t = u / pr.ksplit, ks = u - t * pr.ksplit;
        int b, tp, tq;
        tile_coords(pr, t, b, tp, tq);
        const int xrow = tp * PAIR_BM + (int)rank * BM;
        const int yrow = tq * BN + (int)rank * (BN / 2);
        const int kb0 = ks * pr.kb_per_split, kb1 = min(pr.kblocks, kb0 + pr.kb_per_split);
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait_pair(empty_bar(stage), phase ^ 1u, abort_flag, peer_abort, pr.derr,
                              pr.wait_ns)) {
            ok = false;
            break;
          }
          const uint32_t sx = base + stage * L::STAGE_BYTES;
          const uint32_t sy = sx + L::X_BYTES;
          const uint32_t fb = map_rank(full_bar(stage), 0);
          if (leader) mbar_expect_tx(full_bar(stage), 2 * L::STAGE_BYTES);
          int kx = kb * kcoord, ky = kx;
          if (pr.seg_kb) {
            const int kq = kb / 3, tt = kb - 3 * kq;
            kx = ((int)((pr.seg_x >> tt) & 1u) * pr.seg_kb + kq) * kcoord;
            ky = ((int)((pr.seg_y >> tt) & 1u) * pr.seg_kb + kq) * kcoord;
          }
          if (!(leader && pr.withhold && issued == 0)) {
            tma_load_3d_pair(sx, &tmX, fb, kx, xrow, b);
            tma_load_3d_pair(sy, &tmY, fb, ky, yrow, b);
          }
          ++issued;
          if (++stage == STAGES) { stage = 0; phase ^= 1u; }
        }
      }
      // The odd CTA's copies complete on the leader's barriers: the leader
      // needs this count to drain them if the pair is abandoned.
      if (!leader) st_cluster_u32(map_rank(smem_u32((const void *)odd_fills), 0), (uint32_t)issued);
    }
  } else if (warp == 1) {
    // ------------------------------------------- MMA issuer (leader only)
    if (leader && lane == 0) {
      constexpr uint32_t idesc = make_idesc(KIND, PAIR_BM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;
      bool ok = true;
      for (int u = pair; u < total_units && ok; u += npairs, ++it) {
        const int ks = u % pr.ksplit;
        const int kb0 = ks * pr.kb_per_split, kb1 = min(pr.kblocks, kb0 + pr.kb_per_split);
        const int acc = it & 1;
        const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
        if (!mbar_wait_pair(tempty_bar(acc), acc_phase ^ 1u, abort_flag, peer_abort, pr.derr,
                            pr.wait_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait_pair(full_bar(stage), phase, abort_flag, peer_abort, pr.derr,
                              pr.wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sx = base + stage * L::STAGE_BYTES;
          const uint32_t sy = sx + L::X_BYTES;
#pragma unroll
          for (int kk = 0; kk < KBLOCK_BYTES / 32; ++kk) {
            tc_mma_pair<KIND>(d_tmem, sw128_desc(sx + kk * 32), sw128_desc(sy + kk * 32), idesc,
                              (kb != kb0 || kk) ? 1u : 0u);
          }
          tc_commit_pair(empty_bar(stage), (uint16_t)3);  // frees the stage in both CTAs
          if (++stage == STAGES) { stage = 0; phase ^= 1u; }
        }
        if (!ok) break;
        tc_commit_pair(tfull_bar(acc), (uint16_t)3);
      }
      tc_commit_pair(drain_bar, (uint16_t)1);
      mbar_wait_drain(drain_bar, 0, pr.wait_ns);
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int quarter = warp & 3;
    int it = 0;
    for (int u = pair; u < total_units; u += npairs, ++it) {
      const int t = u / pr.ksplit, ks = u - t * pr.ksplit;
      int b, tp, tq;
      tile_coords(pr, t, b, tp, tq);
      const int acc = it & 1;
      const bool ok = mbar_wait_pair(tfull_bar(acc), (uint32_t)((it >> 1) & 1), abort_flag,
                                     peer_abort, pr.derr, pr.wait_ns);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
      const int p = tp * PAIR_BM + (int)rank * BM + quarter * 32 + lane;
      const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int c = 0; c < BN / 32; ++c) {
        uint32_t v[32];
        tmem_ld32(taddr + (uint32_t)(c * 32), v);
        tmem_ld_wait(v);
        epi(b * pr.ksplit + ks, p, tq * BN + c * 32, v);  // batch x K range
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_remote(map_rank(tempty_bar(acc), 0));
    }
  }

  tc_fence_before();
  __syncthreads();
  // Both CTAs' roles have left their loops: each abort flag is final (a
  // failed wait in either CTA raised both) and the odd CTA's fill count has
  // been stored into the leader.
  cluster_sync();
  if (leader && warp == 0 && lane == 0 && *abort_flag) {
    // Abandoned: every copy either CTA issued completes on the leader's full
    // barriers.  Wait (bounded) for the newest fill of every stage (older
    // ones were consumed).  A fill posted by only one side gets the other
    // side's share settled here -- bytes the leader expected but nobody will
    // copy are completed, a fill only the odd CTA issued gets its arrival --
    // so every wait below ends as soon as the real copies have landed.
    const long lf = issued, of = (long)*odd_fills;
    const long hi = lf > of ? lf : of;
    const long first = hi - STAGES > 0 ? hi - STAGES : 0;
    for (long i = first; i < hi; ++i) {
      const int s = (int)(i % STAGES);
      if (i >= lf) {
        mbar_expect_tx(full_bar(s), L::STAGE_BYTES);
      } else {
        if (pr.withhold && i == 0) mbar_complete_tx(full_bar(s), L::STAGE_BYTES);
        if (i >= of) mbar_complete_tx(full_bar(s), L::STAGE_BYTES);
      }
      mbar_wait_drain(full_bar(s), (uint32_t)((i / STAGES) & 1), pr.wait_ns);
    }
  }
  cluster_sync();  // no CTA of the pair leaves while the leader drains
  tc_fence_after();
  if (warp == 1) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                 "r"(2 * BN));
  }
}

// ------------------------------------------------------------------ host --
// 3-D tensor map over `nbatch` planes of `rows` x `kelems` K-major elements
// (row pitch `row_bytes`, plane pitch `plane_bytes`, both multiples of 16),
// box = 128 B of K x box_rows rows x 1 plane, 128B swizzle, OOB zero fill.
int make_kmajor_map(CUtensorMap *map, int kind, const void *base, long long kelems, long long rows,
                    long long nbatch, long long row_bytes, long long plane_bytes, int box_rows);

template <int KIND, int BN, int STAGES, class Epi, int NACC = 1>
int launch(const CUtensorMap &tmX, const CUtensorMap &tmY, int P, int Q, long long kelems,
           int nbatch, const Epi &epi, int sm_count, int *derr, cudaStream_t s,
           const char *prof_name, int max_ctas = 0, const int *nbatch_dev = nullptr,
           int ksplit = 1, int seg_kb = 0, unsigned seg_x = 0, unsigned seg_y = 0) {
  if (NACC > 1 && (ksplit > 1 || nbatch != NACC || nbatch_dev)) return B2_ERR_ARG;
  using L = SmemLayout<BN, STAGES>;
  Problem pr;
  pr.P = P;
  pr.Q = Q;
  pr.seg_kb = seg_kb;
  pr.seg_x = seg_x;
  pr.seg_y = seg_y;
  pr.kblocks = (int)((kelems * elem_bytes(KIND) + KBLOCK_BYTES - 1) / KBLOCK_BYTES);
  pr.nbatch = nbatch;
  pr.nbatch_dev = nbatch_dev;
  pr.tiles_p = (P + BM - 1) / BM;
  pr.tiles_q = (Q + BN - 1) / BN;
  pr.group = 8;
  pr.derr = derr;
  launch_wait_settings(&pr.wait_ns, &pr.withhold);
  // split-K: ranges of ceil(kblocks / ksplit) blocks, their count recomputed so
  // that none is empty (an empty range would leave its accumulator unwritten)
  if (ksplit < 1) ksplit = 1;
  if (ksplit > pr.kblocks) ksplit = pr.kblocks > 0 ? pr.kblocks : 1;
  pr.kb_per_split = (pr.kblocks + ksplit - 1) / ksplit;
  pr.ksplit = pr.kb_per_split > 0 ? (pr.kblocks + pr.kb_per_split - 1) / pr.kb_per_split : 1;
  if (pr.ksplit < 1) pr.ksplit = 1;
  const long long total =
      (long long)pr.tiles_p * pr.tiles_q * (NACC == 1 ? nbatch : 1) * pr.ksplit;
  if (total <= 0 || (NACC > 1 && pr.kblocks <= 0)) return B2_OK;
  int grid = (int)(total < sm_count ? total : sm_count);
  if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
  auto kern = umma_gemm_kernel<KIND, BN, STAGES, Epi, NACC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL);
  if (e != cudaSuccess) return cuda_fail(e, "umma smem attribute");
  B2_PROF(prof_name, s);
  kern<<<grid, THREADS, L::TOTAL, s>>>(tmX, tmY, pr, epi);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, prof_name);
  return B2_OK;
}

// Pair launch: clusters of 2 CTAs, one pair per two SMs (as many pairs as can
// be resident at once, queried once per device), tiles of 256 X rows x BN Y
// rows.  tmX must have a 128-row box and tmY a BN/2-row box.
template <int KIND, int BN, int STAGES, class Epi>
int launch_pair(const CUtensorMap &tmX, const CUtensorMap &tmY, int P, int Q, long long kelems,
                int nbatch, const Epi &epi, int device, int *derr, cudaStream_t s,
                const char *prof_name, const int *nbatch_dev = nullptr, int ksplit = 1,
                int seg_kb = 0, unsigned seg_x = 0, unsigned seg_y = 0) {
  using L = SmemLayout<BN / 2, STAGES>;
  Problem pr;
  pr.P = P;
  pr.Q = Q;
  pr.kblocks = (int)((kelems * elem_bytes(KIND) + KBLOCK_BYTES - 1) / KBLOCK_BYTES);
  pr.nbatch = nbatch;
  pr.nbatch_dev = nbatch_dev;
  pr.seg_kb = seg_kb;
  pr.seg_x = seg_x;
  pr.seg_y = seg_y;
  // split-K exactly as in launch(): ranges of ceil(kblocks / ksplit) blocks,
  // their count recomputed so that none is empty
  if (ksplit < 1) ksplit = 1;
  if (ksplit > pr.kblocks) ksplit = pr.kblocks > 0 ? pr.kblocks : 1;
  pr.kb_per_split = (pr.kblocks + ksplit - 1) / ksplit;
  pr.ksplit = pr.kb_per_split > 0 ? (pr.kblocks + pr.kb_per_split - 1) / pr.kb_per_split : 1;
  if (pr.ksplit < 1) pr.ksplit = 1;
  pr.tiles_p = (P + PAIR_BM - 1) / PAIR_BM;
  pr.tiles_q = (Q + BN - 1) / BN;
  pr.group = 8;
  pr.derr = derr;
  launch_wait_settings(&pr.wait_ns, &pr.withhold);
  const long long total = (long long)pr.tiles_p * pr.tiles_q * nbatch * pr.ksplit;
  if (total <= 0) return B2_OK;
  auto kern = umma_gemm_pair_kernel<KIND, BN, STAGES, Epi>;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = L::TOTAL;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  static std::atomic<int> resident_pairs[64];  // per device, filled on first use (0 = unknown)
  const int dslot = device >= 0 && device < 64 ? device : 0;
  if (resident_pairs[dslot].load() == 0) {
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL);
    if (e != cudaSuccess) return cuda_fail(e, "umma pair smem attribute");
    cfg.gridDim = dim3(2);
    int nc = 0;
    e = cudaOccupancyMaxActiveClusters(&nc, kern, &cfg);
    if (e != cudaSuccess || nc < 1) {
      (void)cudaGetLastError();
      return e != cudaSuccess ? cuda_fail(e, "umma pair occupancy") : (int)B2_ERR_UNSUPPORTED;
    }
    resident_pairs[dslot].store(nc);
  } else {
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL);
    if (e != cudaSuccess) return cuda_fail(e, "umma pair smem attribute");
  }
  const int resident = resident_pairs[dslot].load();
  const int pairs = (int)(total < resident ? total : resident);
  cfg.gridDim = dim3(2 * pairs);
  B2_PROF(prof_name, s);
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, tmX, tmY, pr, epi);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, prof_name);
  return B2_OK;
}

}  // namespace umma
}  // namespace b2
