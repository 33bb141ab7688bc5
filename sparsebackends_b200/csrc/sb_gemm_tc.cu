// Grouped block GEMM on the fifth-generation tensor cores (tcgen05): the
// 3xTF32 split form and single-pass TF32, with FP32 operands and an FP32 or
// FP64 result.
//
// Same plan as the FP64 DMMA kernels (GemmCBlock / GemmPair: for every C block
// C_c = sum over its pairs of X_p * Y_p).  Every operand value (FP64 or FP32)
// is rounded to FP32 and split  x = hi + lo  with  hi = tf32(x) and
// lo = tf32(x - hi),  and each product is  a_hi*b_lo + a_lo*b_hi + a_hi*b_hi
// (the lo*lo term is below FP32 rounding); single-pass TF32 keeps hi*hi.
//
// Two kernels.  k_tc_pack converts every operand tile once: for each k-tile
// (32 deep) of each 128-row tile of an A-side block and of each nbs-row tile
// of a B-side block it writes the hi and lo planes in the exact layout the
// tensor core reads from shared memory (K-major, 128-byte swizzle: row r of an
// 8-row group at r*128 bytes, 16-byte chunk c at position c ^ r), so a tile
// that several output tiles share is split once.  k_gemm_tc then moves those
// images into shared memory with bulk asynchronous copies (cp.async.bulk
// completing on an mbarrier, no thread work), which leaves the tensor core as
// the only busy unit of the main loop.
//
// Roles.  tcgen05.mma computes D[m, n] = sum_k A[m, k] * B[n, k] with M = 128
// rows of A (TMEM lanes) and N <= 256 rows of B (TMEM columns): the widest
// single-CTA form, which the tensor core runs at 1.4x the rate per flop of
// N = 128 (measured on B200: 1.10 against 0.79 PFLOP/s of TF32 products).  A
// tile is (C block, 128 rows on the A side, nb rows on the B side).  Without
// SWAP the A side is X (rows i of C) and the B side is Y^T (columns j of C);
// with SWAP the roles exchange.  Warp 0 (one thread) issues the copies of a
// k-tile into one of two stages and arms the stage's "full" barrier with their
// byte count; warp 1 (one thread) waits for it, issues the k-tile's MMAs into
// the accumulator of the current chunk and commits them to the stage's
// "empty" barrier (and, at a chunk's end, to the accumulator's "full"
// barrier); warps 2-9 drain (warp w reads TMEM lane quarter w % 4, the rows of
// the A side, and one half of the columns): they add a finished chunk to
// their register sums, arrive on the accumulator's "empty" barrier and, after
// an item's last chunk, write it.  The three roles walk the same sequence of
// items, k-tiles and chunks.
//
// Accumulation.  The tensor core accumulates in FP32 and its error grows with
// the number of accumulation steps (measured: ~9e-5 relative over 17 000
// terms).  The k-tiles of a tile are therefore cut into chunks of kc k-tiles;
// each chunk accumulates from zero in one of two TMEM accumulators (the next
// chunk runs in the other one), and the drain adds the chunks in FP32 with
// round-to-nearest adds (a compensated sum measured the same error: the
// chunks' own accumulation dominates).
//
// Every mbarrier wait is bounded (about two seconds of %globaltimer); a wait
// that runs out sets *status = 1, and the CTA stops issuing MMAs and waiting,
// so the kernel always returns and the host reports SB_ERR_TIMEOUT.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "sb_kernels.hpp"

namespace sb {
namespace {

constexpr int kTcBK = 32;                 // k-tile: 32 TF32 values = one 128-byte swizzle row
constexpr int kTcStages = 2;
constexpr int kTcImg = 128 * 128;                  // bytes of one A plane (128 rows x 128 B)
constexpr int kTcBPlane = kTcMaxN * 128;           // bytes reserved for one B plane (up to 256 rows)
constexpr int kTcStageBytes = 2 * kTcImg + 2 * kTcBPlane;  // A hi, A lo, B hi, B lo
constexpr int kTcDrainWarps = 8;
constexpr int kTcEpiBytes = kTcDrainWarps * 32 * 32 * 4;  // per-warp 32 x 32 FP32 transpose buffers
constexpr int kTcSmemBytes = kTcStages * kTcStageBytes + kTcEpiBytes + 1024 /*alignment*/ + 256 /*barriers*/;
constexpr int kTcTmemCols = 512;                   // two accumulators of up to 256 columns
constexpr int kTcReduceSlices = kTcMaxN / 32;      // 32-column slices of a split tile
constexpr unsigned long long kWaitNs = 2000000000ull;  // bound of every mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the completion of phase `parity` of the mbarrier.  Returns
// false (and records the failure) when the bound runs out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* status) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > kWaitNs) {
      atomicExch(status, 1);
      return false;
    }
  }
}

// The same wait for roles that sit out most of a k-tile (the drain warps):
// between polls the warp sleeps, leaving its issue slots to the producers.
__device__ __forceinline__ bool mbar_wait_idle(uint32_t bar, uint32_t parity, int* status) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    __nanosleep(256);
    if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > kWaitNs) {
      atomicExch(status, 1);
      return false;
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major SWIZZLE_128B operand image:
// start address >> 4, leading-byte offset 16 (unused by swizzled K-major
// layouts), stride-byte offset 1024 (8 rows of 128 bytes), descriptor version
// 1, layout type 2 (128-byte swizzle).  Advancing along K inside the 128-byte
// row adds the byte offset to the start address.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return static_cast<uint64_t>((addr & 0x3FFFFu) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
         (2ull << 61);
}

// Instruction descriptor of kind::tf32, FP32 accumulator, both operands
// K-major, M = 128, N = n (multiple of 16, 16..256).
__device__ __forceinline__ uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15, %16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])));
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  tmem_ld16(taddr, *reinterpret_cast<float(*)[16]>(&v[0]));
  tmem_ld16(taddr + 16, *reinterpret_cast<float(*)[16]>(&v[16]));
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
  tmem_st16(taddr, *reinterpret_cast<const float(*)[16]>(&v[0]));
  tmem_st16(taddr + 16, *reinterpret_cast<const float(*)[16]>(&v[16]));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// x = hi + lo with both parts exactly representable in TF32 (low 13 mantissa
// bits zero).
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - __uint_as_float(h)));
  hi = h;
  lo = l;
}

// Byte offset of the 16-byte chunk c (k = 4c..4c+3) of row r in a K-major
// SWIZZLE_128B image.
__device__ __forceinline__ uint32_t img_off(int r, int c) {
  return static_cast<uint32_t>((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

// 16-byte global store (packed images).
__device__ __forceinline__ void st_global_v4(void* p, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.global.v4.b32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bulk asynchronous copy global -> this CTA's shared memory, completing
// `bytes` of transaction count on the mbarrier (16-byte aligned addresses,
// size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// One packed k-tile image: rows [0, rows) x k [0, kv) of the operand tile at
// src (element (r, k) at src + r*ld + k when kc, else src + r + k*ld), the rest
// zero; hi plane at dst, lo plane at dst + plane (plane = image rows x 128 B).
template <bool F64>
__global__ void __launch_bounds__(256)
    k_tc_pack(const void* __restrict__ srcv, const TcImage* __restrict__ imgs, int64_t nimg,
              unsigned char* __restrict__ dst, int32_t passes) {
  const int tid = static_cast<int>(threadIdx.x);
  for (int64_t i = blockIdx.x; i < nimg; i += gridDim.x) {
    const TcImage im = imgs[i];
    const int rows_img = im.plane >> 7;
    const int nchunks = rows_img * 8;
    unsigned char* const d = dst + im.dst;
    for (int ch = tid; ch < nchunks; ch += 256) {
      // k-contiguous sources: consecutive threads take the chunks of one row;
      // row-contiguous sources: consecutive rows of one chunk
      const int r = im.kc ? ch >> 3 : ch % rows_img, c = im.kc ? ch & 7 : ch / rows_img;
      uint32_t h[4], l[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = 4 * c + j;
        float x = 0.0f;
        if (r < im.rows && k < im.kv) {
          const int64_t e = im.src + (im.kc ? static_cast<int64_t>(r) * im.ld + k : r + static_cast<int64_t>(k) * im.ld);
          x = F64 ? __double2float_rn(static_cast<const double*>(srcv)[e]) : static_cast<const float*>(srcv)[e];
        }
        split_tf32(x, h[j], l[j]);
      }
      const uint32_t off = img_off(r, c);
      st_global_v4(d + off, h[0], h[1], h[2], h[3]);
      if (passes == 3) st_global_v4(d + im.plane + off, l[0], l[1], l[2], l[3]);
    }
  }
}

// Position of a k-tile: work item t (into the tile list), pair p of its C
// block, k offset k0 inside the pair, k-tile index kt inside the item.
struct Cursor {
  int t, p, k0, kt;
};

constexpr int kTcMmaWarp = 1;
constexpr int kTcEpiWarp0 = 2;  // warps 2-9
constexpr int kTcAllThreads = (2 + kTcDrainWarps) * 32;
static_assert(kTcSmemBytes <= 227 * 1024, "shared memory of the tensor-core GEMM");

template <bool SWAP, bool OUT64>
__global__ void __launch_bounds__(kTcAllThreads, 1)
    k_gemm_tc(const unsigned char* __restrict__ pack_a, const unsigned char* __restrict__ pack_b,
              void* __restrict__ Cv, const GemmCBlock* __restrict__ cblocks, const GemmPair* __restrict__ pairs,
              const TcPack* __restrict__ packs, const TcTile* __restrict__ tiles, int32_t ntiles, int32_t nz_begin,
              int32_t passes, int32_t kc, int32_t fold, double* __restrict__ partial, int* __restrict__ status) {
  extern __shared__ unsigned char smem_raw[];
  const int tid = static_cast<int>(threadIdx.x);
  const int warp = tid >> 5, lane = tid & 31;
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;  // 1024-aligned swizzle atoms
  const uint32_t epi_addr = base + kTcStages * kTcStageBytes;
  const uint32_t bars = epi_addr + kTcEpiBytes;
  const uint32_t bar_full0 = bars;                // kTcStages barriers, 8 bytes apart
  const uint32_t bar_empty0 = bars + 32;          // kTcStages
  const uint32_t bar_accf0 = bars + 64;           // 2 (accumulators 0 and 1)
  const uint32_t bar_acce0 = bars + 80;           // 2
  const uint32_t tmem_slot = bars + 96;
  unsigned char* const tmem_slot_ptr = smem_raw + (tmem_slot - raw);
  const bool split = passes == 3;
  const int grid = static_cast<int>(gridDim.x);

  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(bar_full0 + 8 * s, 1);  // the producer's arrive + the copies' bytes
      mbar_init(bar_empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_accf0 + 8 * b, 1);
      mbar_init(bar_acce0 + 8 * b, kTcDrainWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tmem_slot),
                 "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot_ptr);

  if (warp == 0) {
    // ── producer (one thread): bulk copies of the packed images ───────────
    if (lane == 0) {
      bool failed = false;
      auto first_of = [&](int t) -> Cursor {
        if (t >= nz_begin) return Cursor{t, 0, 0, 0};
        const TcTile tl = tiles[t];
        return Cursor{t, tl.p0, tl.k0, 0};
      };
      auto advance = [&](Cursor c) -> Cursor {
        if (c.kt + 1 >= tiles[c.t].nkt) return first_of(c.t + grid);
        if (c.k0 + kTcBK < pairs[c.p].K) return Cursor{c.t, c.p, c.k0 + kTcBK, c.kt + 1};
        return Cursor{c.t, c.p + 1, 0, c.kt + 1};
      };
      uint32_t g = 0;
      for (Cursor c = first_of(static_cast<int>(blockIdx.x)); c.t < nz_begin && !failed; c = advance(c), ++g) {
        const int s = static_cast<int>(g % kTcStages);
        if (g >= kTcStages) failed = !mbar_wait(bar_empty0 + 8 * s, ((g / kTcStages) - 1) & 1, status);
        if (failed) break;
        const TcTile tl = tiles[c.t];
        const TcPack pk = packs[c.p];
        const int j = c.k0 / kTcBK;  // k-tile of the pair
        const unsigned char* ga =
            pack_a + pk.a_base + (static_cast<int64_t>(tl.a0 >> 7) * pk.nkt + j) * (2 * kTcImg);
        const int64_t bimg = 2LL * pk.nbs * 128;
        const unsigned char* gb = pack_b + pk.b_base + (static_cast<int64_t>(tl.b0 / pk.nbs) * pk.nkt + j) * bimg;
        const uint32_t bplane = static_cast<uint32_t>(tl.nb) * 128u;
        const uint32_t sa = base + s * kTcStageBytes, sbh = sa + 2 * kTcImg;
        const uint32_t full = bar_full0 + 8 * s;
        mbar_expect_tx(full, split ? 2u * kTcImg + 2u * bplane : static_cast<uint32_t>(kTcImg) + bplane);
        bulk_g2s(sa, ga, kTcImg, full);
        bulk_g2s(sbh, gb, bplane, full);
        if (split) {
          bulk_g2s(sa + kTcImg, ga + kTcImg, kTcImg, full);
          bulk_g2s(sbh + kTcBPlane, gb + pk.nbs * 128, bplane, full);
        }
      }
      // copies still in flight land before the CTA exits: wait (bounded) for
      // the last stages issued; consumed stages have completed already
      for (uint32_t q = g > kTcStages ? g - kTcStages : 0; q < g; ++q)
        mbar_wait(bar_full0 + 8 * (q % kTcStages), (q / kTcStages) & 1, status);
    }
  } else if (warp == kTcMmaWarp) {
    // ── MMA issue (one thread) ────────────────────────────────────────────
    if (lane == 0) {
      bool failed = false;
      uint32_t g = 0, cg = 0;
      for (int t = static_cast<int>(blockIdx.x); t < nz_begin && !failed; t += grid) {
        const TcTile tl = tiles[t];
        const uint32_t idesc = idesc_tf32(tl.nb);
        for (int kt = 0; kt < tl.nkt && !failed; ++kt) {
          const bool chunk_first = kt % kc == 0;
          const bool chunk_last = kt + 1 == tl.nkt || (kt + 1) % kc == 0;
          // fold: one accumulator, freed by the drain after every chunk;
          // otherwise two, alternating per chunk
          const uint32_t b = fold ? 0u : (cg & 1);
          if (chunk_first && fold && cg >= 1) failed = !mbar_wait(bar_acce0, (cg - 1) & 1, status);
          if (chunk_first && !fold && cg >= 2) failed = !mbar_wait(bar_acce0 + 8 * b, ((cg >> 1) - 1) & 1, status);
          const int s = static_cast<int>(g % kTcStages);
          if (!failed) failed = !mbar_wait(bar_full0 + 8 * s, (g / kTcStages) & 1, status);
          if (failed) break;
          tc_fence_after();
          const uint32_t acc = tmem + 256 * b;
          const uint32_t sa_hi = base + s * kTcStageBytes, sa_lo = sa_hi + kTcImg;  // planes: A hi, A lo, B hi, B lo
          const uint32_t sb_hi = sa_hi + 2 * kTcImg, sb_lo = sb_hi + kTcBPlane;
#pragma unroll
          for (int kk = 0; kk < kTcBK / 8; ++kk) {
            const uint64_t ah = smem_desc(sa_hi + 32 * kk), bh = smem_desc(sb_hi + 32 * kk);
            bool accum = !(chunk_first && kk == 0);
            if (split) {
              mma_tf32(acc, ah, smem_desc(sb_lo + 32 * kk), idesc, accum);
              mma_tf32(acc, smem_desc(sa_lo + 32 * kk), bh, idesc, true);
              accum = true;
            }
            mma_tf32(acc, ah, bh, idesc, accum);
          }
          mma_commit(bar_empty0 + 8 * s);
          if (chunk_last) {
            mma_commit(bar_accf0 + 8 * b);
            ++cg;
          }
          ++g;
        }
      }
    }
  } else {
    // ── drain: warps 2-9; warp w reads TMEM lane quarter w % 4 (32 rows of
    // the A side) and column half h = (w - 2) / 4 ([128h, 128h + 128)).  With
    // fold the chunks of an item are added into a sum kept in TMEM columns
    // [256, 512) (FP32, round to nearest); otherwise items have one chunk. ──
    bool failed = false;
    const int dw = warp - kTcEpiWarp0;
    const int q = warp & 3, h = dw >> 2;
    const uint32_t lanes = static_cast<uint32_t>(32 * q) << 16;
    float* const epi = reinterpret_cast<float*>(smem_raw + (epi_addr - raw)) + dw * 1024;
    uint32_t cg = 0;
    for (int t = static_cast<int>(blockIdx.x); t < nz_begin; t += grid) {
      const TcTile tl = tiles[t];
      const GemmCBlock cb = cblocks[tl.cb];
      const int ma = SWAP ? cb.N : cb.M, nbv = SWAP ? cb.M : cb.N;
      const int arow0 = tl.a0 + 32 * q;         // first A-side row of this warp
      const int arow = arow0 + lane;            // A-side row of this thread
      const int rows_ok = min(32, ma - arow0);  // valid rows of this warp (may be <= 0)
      const int c_lo = 128 * h;                 // this warp's columns [c_lo, c_hi) of the item
      const int c_hi = min(tl.nb, c_lo + 128);
      const int nch = (tl.nkt + kc - 1) / kc;
      for (int ch = 0; ch < nch; ++ch, ++cg) {
        const bool first = ch == 0, last = ch + 1 == nch;
        const uint32_t b = fold ? 0u : (cg & 1);
        const uint32_t parity = fold ? (cg & 1) : ((cg >> 1) & 1);
        if (!failed) failed = !mbar_wait_idle(bar_accf0 + 8 * b, parity, status);
        tc_fence_after();
        const uint32_t acc = tmem + 256 * b + static_cast<uint32_t>(c_lo) + lanes;
        const uint32_t tsum = tmem + 256 + static_cast<uint32_t>(c_lo) + lanes;
        for (int gp = 0; gp < 4; ++gp) {  // 32 columns per TMEM wait
          const int c0 = c_lo + 32 * gp;  // item column of v[0]
          if (c0 >= c_hi) break;
          float v[32], sm[32];
          tmem_ld32(acc + 32 * gp, v);
          if (fold && !first) tmem_ld32(tsum + 32 * gp, sm);
          tmem_wait_ld();
          if (fold && !first)
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] += sm[j];
          if (!last) {
            tmem_st32(tsum + 32 * gp, v);
            continue;
          }
          if (failed || rows_ok <= 0) continue;
          if (tl.part >= 0) {
            // partial tile (column-major 128 x 256): lanes write consecutive rows
            double* pt = partial + static_cast<int64_t>(tl.part) * kTcPartElems + 32 * q + lane;
            if (lane < rows_ok)
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (c0 + j < c_hi) pt[(c0 + j) * 128] = static_cast<double>(v[j]);
            continue;
          }
          if constexpr (!SWAP) {
            // C(i = arow, j = bcol) at arow + bcol * ldc: lanes write consecutive rows
            if (lane < rows_ok)
#pragma unroll
              for (int j = 0; j < 32; ++j) {
                const int bcol = tl.b0 + c0 + j;
                if (c0 + j >= c_hi || bcol >= nbv) break;
                const int64_t off = cb.c_off + arow + static_cast<int64_t>(bcol) * cb.ldc;
                if (OUT64) static_cast<double*>(Cv)[off] = static_cast<double>(v[j]);
                else static_cast<float*>(Cv)[off] = v[j];
              }
          } else {
            // SWAP: stage 32 rows x 32 columns in the warp's shared buffer
            // (XOR-swizzled: no bank conflicts either way), then lanes write
            // consecutive columns of one row: C(i = bcol, j = arow) at bcol + arow * ldc
#pragma unroll
            for (int j = 0; j < 32; ++j) epi[lane * 32 + (j ^ lane)] = v[j];
            __syncwarp();
            const int bcol = tl.b0 + c0 + lane;
            const bool col_ok = bcol < nbv && c0 + lane < c_hi;
            for (int r = 0; r < rows_ok; ++r) {
              const float val = epi[r * 32 + (lane ^ r)];
              if (!col_ok) continue;
              const int64_t off = cb.c_off + bcol + static_cast<int64_t>(arow0 + r) * cb.ldc;
              if (OUT64) static_cast<double*>(Cv)[off] = static_cast<double>(val);
              else static_cast<float*>(Cv)[off] = val;
            }
            __syncwarp();
          }
        }
        if (!last) tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_acce0 + 8 * b);
      }
    }
    // C blocks without pairs (items [nz_begin, ntiles)): zeros
    const int et = tid - kTcEpiWarp0 * 32;
    for (int t = nz_begin + static_cast<int>(blockIdx.x); t < ntiles; t += grid) {
      const TcTile tl = tiles[t];
      const GemmCBlock cb = cblocks[tl.cb];
      const int ma = SWAP ? cb.N : cb.M, nbv = SWAP ? cb.M : cb.N;
      const int rows = min(128, ma - tl.a0), cols = min(tl.nb, nbv - tl.b0);
      for (int e = et; e < rows * cols; e += 32 * kTcDrainWarps) {
        const int r = tl.a0 + e % rows, c = tl.b0 + e / rows;
        const int64_t off =
            cb.c_off + (SWAP ? c + static_cast<int64_t>(r) * cb.ldc : r + static_cast<int64_t>(c) * cb.ldc);
        if (OUT64) static_cast<double*>(Cv)[off] = 0.0;
        else static_cast<float*>(Cv)[off] = 0.0f;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
  }
}

template <bool SWAP, bool OUT64>
cudaError_t launch_tc_t(const unsigned char* pa, const unsigned char* pb, void* C, const GemmCBlock* cb,
                        const GemmPair* pr, const TcPack* packs, const TcTile* tiles, int32_t ntiles,
                        int32_t nz_begin, int passes, int kc, bool fold, double* partial, int* status,
                        cudaStream_t s) {
  auto kern = k_gemm_tc<SWAP, OUT64>;
  static std::atomic<int> grid_of[64] = {};  // one CTA per SM, per device ordinal
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int grid = grid_of[dev & 63].load();
  if (grid == 0) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemBytes);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&grid, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    grid_of[dev & 63].store(grid);
  }
  const unsigned g = static_cast<unsigned>(std::min<int64_t>(ntiles, grid));
  kern<<<g, kTcAllThreads, kTcSmemBytes, s>>>(pa, pb, C, cb, pr, packs, tiles, ntiles, nz_begin, passes, kc,
                                               fold ? 1 : 0, partial, status);
  return cudaGetLastError();
}

// Sum of the k-segment partial tiles of split tiles, in segment order (FP64,
// deterministic), into C.  Element (r, c) of the column-major partial tile is
// (A-side row r, B-side row c).
template <bool SWAP, bool OUT64>
__global__ void __launch_bounds__(256) k_tc_reduce(const double* __restrict__ partial, void* __restrict__ Cv,
                                                   const GemmCBlock* __restrict__ cblocks,
                                                   const TcSplit* __restrict__ splits) {
  // block = (split tile, 32-column slice): partials read along rows, summed in
  // segment order, staged, and written along C's contiguous direction
  __shared__ double S[32][129];
  const TcSplit sp = splits[blockIdx.x / kTcReduceSlices];
  const int c0 = 32 * static_cast<int>(blockIdx.x % kTcReduceSlices);
  const GemmCBlock cb = cblocks[sp.cb];
  const int ma = SWAP ? cb.N : cb.M, nbv = SWAP ? cb.M : cb.N;
  const int rows = min(128, ma - sp.a0), cols = min(sp.nb, nbv - sp.b0) - c0;
  if (cols <= 0) return;
  const int tid = static_cast<int>(threadIdx.x);
  for (int e = tid; e < 128 * 32; e += 256) {
    const int r = e & 127, c = e >> 7;
    double acc = 0.0;
    if (r < rows && c < cols)
      for (int q = 0; q < sp.nparts; ++q)
        acc += partial[static_cast<int64_t>(sp.part0 + q) * kTcPartElems + r + (c0 + c) * 128];
    S[c][r] = acc;
  }
  __syncthreads();
  for (int e = tid; e < 128 * 32; e += 256) {
    // SWAP: consecutive threads take consecutive B-side rows (contiguous in C)
    const int r = SWAP ? e >> 5 : e & 127, c = SWAP ? e & 31 : e >> 7;
    if (r >= rows || c >= cols) continue;
    const int arow = sp.a0 + r, bcol = sp.b0 + c0 + c;
    const int64_t off = cb.c_off + (SWAP ? bcol + static_cast<int64_t>(arow) * cb.ldc
                                         : arow + static_cast<int64_t>(bcol) * cb.ldc);
    if (OUT64) static_cast<double*>(Cv)[off] = S[c][r];
    else static_cast<float*>(Cv)[off] = static_cast<float>(S[c][r]);
  }
}

}  // namespace

cudaError_t launch_tc_pack(const void* src, bool src_f64, const TcImage* d_imgs, int64_t nimg, void* dst, int passes,
                           cudaStream_t s) {
  if (nimg <= 0) return cudaSuccess;
  if (passes != 1 && passes != 3) return cudaErrorInvalidValue;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned g = static_cast<unsigned>(std::min<int64_t>(nimg, 8LL * sms));
  if (src_f64)
    k_tc_pack<true><<<g, 256, 0, s>>>(src, d_imgs, nimg, static_cast<unsigned char*>(dst), passes);
  else
    k_tc_pack<false><<<g, 256, 0, s>>>(src, d_imgs, nimg, static_cast<unsigned char*>(dst), passes);
  return cudaGetLastError();
}

cudaError_t launch_gemm_tc(const void* pack_a, const void* pack_b, void* C, bool c_f64, const GemmCBlock* d_cblocks,
                           const GemmPair* d_pairs, const TcPack* d_packs, const TcTile* d_tiles, int32_t ntiles,
                           int32_t nz_begin, bool swap, int passes, int kc, bool fold, double* d_partial,
                           const TcSplit* d_splits, int32_t nsplits, int* d_status, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  if ((passes != 1 && passes != 3) || kc < 1 || (nsplits > 0 && (!d_partial || !d_splits)))
    return cudaErrorInvalidValue;
  const auto* pa = static_cast<const unsigned char*>(pack_a);
  const auto* pb = static_cast<const unsigned char*>(pack_b);
  cudaError_t e;
  if (swap)
    e = c_f64 ? launch_tc_t<true, true>(pa, pb, C, d_cblocks, d_pairs, d_packs, d_tiles, ntiles, nz_begin, passes, kc,
                                        fold, d_partial, d_status, s)
              : launch_tc_t<true, false>(pa, pb, C, d_cblocks, d_pairs, d_packs, d_tiles, ntiles, nz_begin, passes,
                                         kc, fold, d_partial, d_status, s);
  else
    e = c_f64 ? launch_tc_t<false, true>(pa, pb, C, d_cblocks, d_pairs, d_packs, d_tiles, ntiles, nz_begin, passes,
                                         kc, fold, d_partial, d_status, s)
              : launch_tc_t<false, false>(pa, pb, C, d_cblocks, d_pairs, d_packs, d_tiles, ntiles, nz_begin, passes,
                                          kc, fold, d_partial, d_status, s);
  if (e != cudaSuccess || nsplits <= 0) return e;
  if (swap) {
    if (c_f64) k_tc_reduce<true, true><<<nsplits * kTcReduceSlices, 256, 0, s>>>(d_partial, C, d_cblocks, d_splits);
    else k_tc_reduce<true, false><<<nsplits * kTcReduceSlices, 256, 0, s>>>(d_partial, C, d_cblocks, d_splits);
  } else {
    if (c_f64) k_tc_reduce<false, true><<<nsplits * kTcReduceSlices, 256, 0, s>>>(d_partial, C, d_cblocks, d_splits);
    else k_tc_reduce<false, false><<<nsplits * kTcReduceSlices, 256, 0, s>>>(d_partial, C, d_cblocks, d_splits);
  }
  return cudaGetLastError();
}

}  // namespace sb
