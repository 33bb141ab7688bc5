// Grouped FP64 block GEMM for sm_100a with segmented (atomics-free) accumulation.
//
// Blackwell's tcgen05.mma has no f64 kind, so the FP64 tensor-core path is the
// warp-level DMMA instruction (mma.sync.aligned.m8n8k4 .f64).  Tiles of X and
// Y are staged into shared memory by a 3-stage cp.async pipeline that runs
// straight across the pairs of one C block (the K loops of all pairs feeding a
// C tile are concatenated), so one CTA owns one C tile and writes it once.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "../../include/sparseb.h"
#include "sb_kernels.hpp"

namespace sb {
namespace {

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int bytes = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem, bool valid) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int bytes = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

constexpr int kBK = 16;       // default k-tile
constexpr int kStages = 3;    // default pipeline depth

// Shared-memory layout of one operand tile (BK-deep, ST pipeline stages): the
// dimension that is contiguous in global memory stays contiguous in shared
// memory (conflict-free cp.async writes); the padding (rows of BM+4 or BK+4
// doubles) makes the DMMA fragment reads conflict-free within each half-warp.
template <int BM, int BN, bool XT, bool YT, int BK = kBK, int ST = kStages>
struct TileLayout {
  static constexpr int KP = BK + 4;  // padded k-run length of k-contiguous tiles
  static constexpr int XSZ = XT ? BM * KP : BK * (BM + 4);  // X: [i][k] if XT else [k][i]
  static constexpr int YSZ = YT ? BK * (BN + 4) : BN * KP;  // Y: [k][j] if YT else [j][k]
  static constexpr int bytes() { return ST * (XSZ + YSZ) * 8; }
  __device__ static int xidx(int i, int k) { return XT ? i * KP + k : k * (BM + 4) + i; }
  __device__ static int yidx(int k, int j) { return YT ? k * (BN + 4) + j : j * KP + k; }
};

// C block of tile `bid`: the last c with tile_begin <= bid.
__device__ __forceinline__ int tile_cblock(const GemmCBlock* __restrict__ cblocks, int32_t ncb, int bid) {
  int lo = 0, hi = ncb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cblocks[mid].tile_begin <= bid) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The same lookup by a full warp (every lane gets the result): each round
// tests 32 evenly spaced candidates at once, so 120 blocks take two dependent
// loads and 30000 take three, against 7 and 15 for a bisection.  The answer
// stays in [lo, hi] with tile_begin[lo] <= bid; the lanes whose candidate
// still starts at or before bid form a prefix, so their count narrows the
// range to one step.
__device__ __forceinline__ int tile_cblock_warp(const GemmCBlock* __restrict__ cblocks, int32_t ncb, int bid) {
  const int lane = static_cast<int>(threadIdx.x & 31);
  int lo = 0, hi = ncb - 1;
  while (lo < hi) {
    const int step = (hi - lo + 32) / 32;
    const int idx = lo + (lane + 1) * step;
    const bool le = idx <= hi && cblocks[idx].tile_begin <= bid;
    const int k = __popc(__ballot_sync(0xffffffffu, le));
    lo += k * step;
    hi = min(hi, lo + step - 1);
  }
  return lo;
}

// One CTA of the tiled GEMM: tile lt of C block cb, k-segment seg of splitk;
// with splitk > 1 the BMC x BNC tile goes to pt (column-major) instead of C.
// BM x BN is the staged (shared-memory) tile; the C tile BMC x BNC may be
// narrower (48 of 64 rows or columns: the operand copies past BMC / BNC are
// zero-filled without reading memory, and no warp multiplies them).
template <int BM, int BN, int WM, int WN, bool XT, bool YT, int BK, int ST, int BMC = BM, int BNC = BN>
__device__ __forceinline__ void gemm_cta(const double* __restrict__ X, const double* __restrict__ Y,
                                         double* __restrict__ C, const GemmCBlock& cb,
                                         const GemmPair* __restrict__ pairs, int lt, int seg, int32_t splitk,
                                         double* __restrict__ pt, double* smem) {
  constexpr int kBK = BK;
  constexpr int kStages = ST;
  using TL = TileLayout<BM, BN, XT, YT, BK, ST>;
  static_assert(BMC <= BM && BNC <= BN && BMC % WM == 0 && BNC % WN == 0, "compute tile must tile the warps");
  constexpr int NWM = BMC / WM;
  constexpr int NWN = BNC / WN;
  constexpr int NT = NWM * NWN * 32;
  constexpr int MT = WM / 8;
  constexpr int NTL = WN / 8;
  constexpr int XLOADS = BM * kBK / NT;
  constexpr int YLOADS = BN * kBK / NT;
  static_assert(BM * kBK % NT == 0 && BN * kBK % NT == 0, "tile/threads mismatch");

  double* Xs = smem;                    // kStages tiles of TL::XSZ
  double* Ys = smem + kStages * TL::XSZ;  // kStages tiles of TL::YSZ

  const int M = cb.M, N = cb.N;
  const int m0 = (lt % cb.mtiles) * BMC, n0 = (lt / cb.mtiles) * BNC;
  const int tid = threadIdx.x;

  // k-tiles of all pairs: the lanes of each warp sum a stride of the pairs
  int ktot = 0;
  for (int p = cb.pair_begin + static_cast<int>(threadIdx.x & 31); p < cb.pair_end; p += 32)
    ktot += (pairs[p].K + kBK - 1) / kBK;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ktot += __shfl_xor_sync(0xffffffffu, ktot, o);
  // this segment's range of the concatenated k-tiles
  const int kb = static_cast<int>(static_cast<int64_t>(ktot) * seg / splitk);
  const int ke = static_cast<int>(static_cast<int64_t>(ktot) * (seg + 1) / splitk);
  const int total = ke - kb;

  int lp = cb.pair_begin;  // load cursor: pair index and k-tile within it
  int lkt = kb;
  while (lp < cb.pair_end && lkt >= (pairs[lp].K + kBK - 1) / kBK) {
    lkt -= (pairs[lp].K + kBK - 1) / kBK;
    ++lp;
  }
  // Load geometry of this thread (fixed for the CTA): NT is a multiple of the
  // tile's contiguous extent, so all elements a thread stages share one index
  // (x_fix / y_fix) and step the other by a constant per unroll step r.
  static_assert(NT % kBK == 0 && NT % BM == 0 && NT % BN == 0, "thread count must tile the operand rows");
  constexpr int XR = XT ? NT / kBK : NT / BM;  // step of the varying index (XT: row i, else k)
  constexpr int YR = YT ? NT / BN : NT / kBK;  // (YT: k, else column j)
  const int x_fix = XT ? tid % kBK : tid % BM;
  const int x_var = XT ? tid / kBK : tid / BM;
  const int y_fix = YT ? tid % BN : tid % kBK;
  const int y_var = YT ? tid / BN : tid / kBK;
  const int sx0 = XT ? x_var * TL::KP + x_fix : x_var * (BM + 4) + x_fix;  // shared offsets at r = 0
  const int sy0 = YT ? y_var * (BN + 4) + y_fix : y_var * TL::KP + y_fix;
  constexpr int SXR = XT ? XR * TL::KP : XR * (BM + 4);
  constexpr int SYR = YT ? YR * (BN + 4) : YR * TL::KP;
  const int mleft = min(M - m0, BMC), nleft = min(N - n0, BNC);

  // descriptor of the pair being loaded and this thread's global addresses in
  // it, kept in registers; the next pair is fetched when the cursor moves on,
  // a k-tile before it is needed
  GemmPair pr{};
  const double *xg = X, *yg = Y;
  int64_t xstep = 0, ystep = 0;
  auto set_pair = [&]() {
    if (XT) {
      xg = X + pr.x_off + static_cast<int64_t>(m0 + x_var) * pr.ldx + x_fix;
    } else {
      xg = X + pr.x_off + (m0 + x_fix) + static_cast<int64_t>(x_var) * pr.ldx;
    }
    xstep = static_cast<int64_t>(XR) * pr.ldx;
    if (YT) {
      yg = Y + pr.y_off + (n0 + y_fix) + static_cast<int64_t>(y_var) * pr.ldy;
    } else {
      yg = Y + pr.y_off + y_fix + static_cast<int64_t>(n0 + y_var) * pr.ldy;
    }
    ystep = static_cast<int64_t>(YR) * pr.ldy;
  };
  if (lp < cb.pair_end) {
    pr = pairs[lp];
    set_pair();
  }

  // Staging of one k-tile, in kParts slices so that the copies of the next
  // stage interleave with the DMMAs of the current one.
  constexpr int kParts = kBK / 4;
  static_assert(XLOADS % kParts == 0 && YLOADS % kParts == 0, "loads must split evenly over the k4 steps");
  int kleft = 0;
  const double *xp = X, *yp = Y;
  double *xs_st = Xs, *ys_st = Ys;
  auto begin_load = [&](int stage) {
    const int k0 = lkt * kBK;
    kleft = pr.K - k0;  // valid k entries of this k-tile
    xp = xg + (XT ? static_cast<int64_t>(k0) : static_cast<int64_t>(k0) * pr.ldx);
    yp = yg + (YT ? static_cast<int64_t>(k0) * pr.ldy : static_cast<int64_t>(k0));
    xs_st = Xs + stage * TL::XSZ + sx0;
    ys_st = Ys + stage * TL::YSZ + sy0;
  };
  auto load_part = [&](int part) {
#pragma unroll
    for (int q = 0; q < XLOADS / kParts; ++q) {
      const int r = part * (XLOADS / kParts) + q;
      const int var = x_var + r * XR;
      const bool v = XT ? (var < mleft && x_fix < kleft) : (x_fix < mleft && var < kleft);
      cp_async8(xs_st + r * SXR, v ? xp + r * xstep : X, v);
    }
#pragma unroll
    for (int q = 0; q < YLOADS / kParts; ++q) {
      const int r = part * (YLOADS / kParts) + q;
      const int var = y_var + r * YR;
      const bool v = YT ? (y_fix < nleft && var < kleft) : (var < nleft && y_fix < kleft);
      cp_async8(ys_st + r * SYR, v ? yp + r * ystep : Y, v);
    }
  };
  auto end_load = [&]() {
    if (++lkt * kBK >= pr.K) {
      lkt = 0;
      if (++lp < cb.pair_end) {
        pr = pairs[lp];
        set_pair();
      }
    }
  };
  auto issue_load = [&](int stage) {
    begin_load(stage);
#pragma unroll
    for (int part = 0; part < kParts; ++part) load_part(part);
    end_load();
  };

  const int warp = tid >> 5, lane = tid & 31;
  const int wm = warp % NWM, wn = warp / NWM;
  const int g = lane >> 2, t = lane & 3;

  double acc[MT][NTL][2];
#pragma unroll
  for (int a = 0; a < MT; ++a)
#pragma unroll
    for (int b = 0; b < NTL; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < total) issue_load(s);
    cp_async_commit();
  }

  for (int it = 0; it < total; ++it) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    const bool more = it + kStages - 1 < total;
    if (more) begin_load((it + kStages - 1) % kStages);
    const double* xs = Xs + (it % kStages) * TL::XSZ;
    const double* ys = Ys + (it % kStages) * TL::YSZ;
#pragma unroll
    for (int k4 = 0; k4 < kBK; k4 += 4) {
      if (more) load_part(k4 / 4);
      double af[MT], bf[NTL];
#pragma unroll
      for (int a = 0; a < MT; ++a) af[a] = xs[TL::xidx(wm * WM + a * 8 + g, k4 + t)];
#pragma unroll
      for (int b = 0; b < NTL; ++b) bf[b] = ys[TL::yidx(k4 + t, wn * WN + b * 8 + g)];
#pragma unroll
      for (int a = 0; a < MT; ++a)
#pragma unroll
        for (int b = 0; b < NTL; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
    if (more) end_load();
    cp_async_commit();
  }
  cp_async_wait<0>();

  if (splitk > 1) {
    // partial tile, column-major BMC x BNC, reduced by k_splitk_reduce
#pragma unroll
    for (int a = 0; a < MT; ++a) {
      const int rl = wm * WM + a * 8 + g;
#pragma unroll
      for (int b = 0; b < NTL; ++b) {
        const int cl = wn * WN + b * 8 + 2 * t;
        pt[rl + cl * BMC] = acc[a][b][0];
        pt[rl + (cl + 1) * BMC] = acc[a][b][1];
      }
    }
    return;
  }
  double* cbase = C + cb.c_off;
#pragma unroll
  for (int a = 0; a < MT; ++a) {
    const int row = m0 + wm * WM + a * 8 + g;
    if (row >= M) continue;
#pragma unroll
    for (int b = 0; b < NTL; ++b) {
      const int col = n0 + wn * WN + b * 8 + 2 * t;
      if (col < N) cbase[row + (int64_t)col * cb.ldc] = acc[a][b][0];
      if (col + 1 < N) cbase[row + (int64_t)(col + 1) * cb.ldc] = acc[a][b][1];
    }
  }
}

// Split-K: CTA = (segment, tile), segments outermost so that concurrently
// running CTAs work on the same K range of neighbouring tiles.
template <int BM, int BN, int WM, int WN, bool XT, bool YT, int BK = kBK, int ST = kStages>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32, 512 / ((BM / WM) * (BN / WN) * 32))
    k_gemm_f64(const double* __restrict__ X, const double* __restrict__ Y, double* __restrict__ C,
               const GemmCBlock* __restrict__ cblocks, int32_t ncb, const GemmPair* __restrict__ pairs,
               int32_t splitk, int32_t ntiles, double* __restrict__ partial) {
  extern __shared__ double smem[];
  const int seg = static_cast<int>(blockIdx.x) / ntiles;
  const int bid = static_cast<int>(blockIdx.x) % ntiles;
  const GemmCBlock cb = cblocks[tile_cblock_warp(cblocks, ncb, bid)];
  double* pt = splitk > 1 ? partial + (static_cast<int64_t>(seg) * ntiles + bid) * (BM * BN) : nullptr;
  gemm_cta<BM, BN, WM, WN, XT, YT, BK, ST>(X, Y, C, cb, pairs, bid - cb.tile_begin, seg, splitk, pt, smem);
}

// Five tile shapes in one launch (launch_gemm_f64_edges): the tiles of every
// C sub-block are numbered consecutively through tile_begin as usual, and the
// sub-block's tshape picks the CTA's tile: 0 = 64x64 (32x32 warp tiles),
// 1 = 64x32 (32x16), 2 = 32x64 (16x32), 3 = 64x48 (32x24), 4 = 48x64 (24x32),
// all four warps and 3 stages (the 48-wide ones stage 64x64 operand tiles).
// Partial tiles of split-K are kEdgePart doubles apart whatever their shape.
constexpr int kEdgeThreads = 128;
constexpr int kEdgePart = 64 * 64;
template <bool XT, bool YT>
__global__ void __launch_bounds__(kEdgeThreads, 4)
    k_gemm_f64_edges(const double* __restrict__ X, const double* __restrict__ Y, double* __restrict__ C,
                     const GemmCBlock* __restrict__ cblocks, int32_t ncb, const GemmPair* __restrict__ pairs,
                     int32_t splitk, int32_t ntiles, double* __restrict__ partial) {
  extern __shared__ double smem[];
  const int seg = static_cast<int>(blockIdx.x) / ntiles;
  const int bid = static_cast<int>(blockIdx.x) % ntiles;
  const GemmCBlock cb = cblocks[tile_cblock_warp(cblocks, ncb, bid)];
  double* pt = splitk > 1 ? partial + (static_cast<int64_t>(seg) * ntiles + bid) * kEdgePart : nullptr;
  const int lt = bid - cb.tile_begin;
  if (cb.tshape == 0)
    gemm_cta<64, 64, 32, 32, XT, YT, kBK, kStages>(X, Y, C, cb, pairs, lt, seg, splitk, pt, smem);
  else if (cb.tshape == 1)
    gemm_cta<64, 32, 32, 16, XT, YT, kBK, kStages>(X, Y, C, cb, pairs, lt, seg, splitk, pt, smem);
  else if (cb.tshape == 2)
    gemm_cta<32, 64, 16, 32, XT, YT, kBK, kStages>(X, Y, C, cb, pairs, lt, seg, splitk, pt, smem);
  else if (cb.tshape == 3)
    gemm_cta<64, 64, 32, 24, XT, YT, kBK, kStages, 64, 48>(X, Y, C, cb, pairs, lt, seg, splitk, pt, smem);
  else
    gemm_cta<64, 64, 24, 32, XT, YT, kBK, kStages, 48, 64>(X, Y, C, cb, pairs, lt, seg, splitk, pt, smem);
}

// Deterministic split-K reduction: C tile = sum over segments in order.
// Element e: tile e / stride, offset e % stride in the column-major BM x BN
// partial tile.
__device__ __forceinline__ void splitk_reduce_elem(double* __restrict__ C, const GemmCBlock& cb, int bm, int bn,
                                                   int lt, int w, int32_t splitk, int64_t seg_stride,
                                                   const double* __restrict__ pt) {
  if (w >= bm * bn) return;
  const int rl = w % bm, cl = w / bm;
  const int row = (lt % cb.mtiles) * bm + rl, col = (lt / cb.mtiles) * bn + cl;
  if (row >= cb.M || col >= cb.N) return;
  double acc = 0.0;
  for (int sg = 0; sg < splitk; ++sg) acc += pt[sg * seg_stride + w];
  C[cb.c_off + row + static_cast<int64_t>(col) * cb.ldc] = acc;
}

template <int BM, int BN>
__global__ void k_splitk_reduce(double* __restrict__ C, const GemmCBlock* __restrict__ cblocks, int32_t ncb,
                                int32_t splitk, int32_t ntiles, const double* __restrict__ partial) {
  const int64_t total = static_cast<int64_t>(ntiles) * BM * BN;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int bid = static_cast<int>(e / (BM * BN)), w = static_cast<int>(e % (BM * BN));
    const GemmCBlock cb = cblocks[tile_cblock(cblocks, ncb, bid)];
    splitk_reduce_elem(C, cb, BM, BN, bid - cb.tile_begin, w, splitk, static_cast<int64_t>(ntiles) * BM * BN,
                       partial + static_cast<int64_t>(bid) * BM * BN);
  }
}

__global__ void k_splitk_reduce_edges(double* __restrict__ C, const GemmCBlock* __restrict__ cblocks, int32_t ncb,
                                      int32_t splitk, int32_t ntiles, const double* __restrict__ partial) {
  const int64_t total = static_cast<int64_t>(ntiles) * kEdgePart;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int bid = static_cast<int>(e / kEdgePart), w = static_cast<int>(e % kEdgePart);
    const GemmCBlock cb = cblocks[tile_cblock(cblocks, ncb, bid)];
    const int bm = cb.tshape == 2 ? 32 : cb.tshape == 4 ? 48 : 64;
    const int bn = cb.tshape == 1 ? 32 : cb.tshape == 3 ? 48 : 64;
    splitk_reduce_elem(C, cb, bm, bn, bid - cb.tile_begin, w, splitk, static_cast<int64_t>(ntiles) * kEdgePart,
                       partial + static_cast<int64_t>(bid) * kEdgePart);
  }
}

template <int BM, int BN, int WM, int WN, bool XT, bool YT, int BK = kBK, int ST = kStages>
cudaError_t launch_t(const double* X, const double* Y, double* C, const GemmCBlock* cb, int32_t ncb,
                     const GemmPair* pr, int64_t ntiles, int splitk, double* partial, cudaStream_t s) {
  constexpr int threads = (BM / WM) * (BN / WN) * 32;
  constexpr int smem = TileLayout<BM, BN, XT, YT, BK, ST>::bytes();
  auto kern = k_gemm_f64<BM, BN, WM, WN, XT, YT, BK, ST>;
  static std::atomic<unsigned long long> configured{0};  // one bit per device ordinal (host threads may race)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(configured & bit)) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit);
  }
  if (ntiles <= 0) return cudaSuccess;
  if (splitk < 1 || ntiles * splitk > 0x7fffffffLL || (splitk > 1 && !partial)) return cudaErrorInvalidValue;
  kern<<<static_cast<unsigned>(ntiles * splitk), threads, smem, s>>>(X, Y, C, cb, ncb, pr, splitk,
                                                                     static_cast<int32_t>(ntiles), partial);
  e = cudaGetLastError();
  if (e != cudaSuccess || splitk == 1) return e;
  const int64_t elems = ntiles * BM * BN;
  const unsigned g = static_cast<unsigned>(std::min<int64_t>((elems + 255) / 256, 148LL * 64));
  k_splitk_reduce<BM, BN><<<g, 256, 0, s>>>(C, cb, ncb, splitk, static_cast<int32_t>(ntiles), partial);
  return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, int BK = kBK, int ST = kStages>
cudaError_t dispatch_t(bool xT, bool yT, const double* X, const double* Y, double* C,
                       const GemmCBlock* cb, int32_t ncb, const GemmPair* pr, int64_t nt, int sk, double* part,
                       cudaStream_t s) {
  if (!xT && !yT) return launch_t<BM, BN, WM, WN, false, false, BK, ST>(X, Y, C, cb, ncb, pr, nt, sk, part, s);
  if (!xT && yT) return launch_t<BM, BN, WM, WN, false, true, BK, ST>(X, Y, C, cb, ncb, pr, nt, sk, part, s);
  if (xT && !yT) return launch_t<BM, BN, WM, WN, true, false, BK, ST>(X, Y, C, cb, ncb, pr, nt, sk, part, s);
  return launch_t<BM, BN, WM, WN, true, true, BK, ST>(X, Y, C, cb, ncb, pr, nt, sk, part, s);
}

// ── thin GEMM (K <= 16, one of M/N <= 16, the other long) ─────────────────
// One CTA covers kThinBig elements of the long dimension of one C block; the
// long operand tile (kThinBig x 16) and the small one (16 x 16) of each pair
// are staged by cp.async with the next pair prefetched while DMMA runs on the
// current one; the C tile goes through shared memory so that its stores are
// fully coalesced (C columns of the long side, or the contiguous run of short
// columns).
constexpr int kThinBig = 128;
constexpr int kThinThreads = 128;
constexpr int kThinKP = 20;            // padded k-run / small-side stride
constexpr int kThinBP = kThinBig + 4;  // padded long-side stride

template <bool SR, bool XT, bool YT>
struct ThinLayout {
  // long operand: X when !SR (rows), Y when SR (columns); small operand the other.
  static constexpr bool LONG_KCONTIG = SR ? !YT : XT;  // long tile stored [l][k] when k is contiguous
  static constexpr int LSZ = LONG_KCONTIG ? kThinBig * kThinKP : 16 * kThinBP;
  // small operand: Y when !SR, X when SR; stored [s][k] when k is contiguous
  // in global memory, else [k][s], so that consecutive threads load
  // consecutive global addresses into consecutive shared addresses
  static constexpr bool SMALL_KCONTIG = SR ? XT : !YT;
  static constexpr int SSZ = 16 * kThinKP;
  __device__ static int lidx(int l, int k) { return LONG_KCONTIG ? l * kThinKP + k : k * kThinBP + l; }
  __device__ static int sidx(int k, int s) { return SMALL_KCONTIG ? s * kThinKP + k : k * kThinKP + s; }
};

template <bool SR, bool XT, bool YT>
__global__ void __launch_bounds__(kThinThreads, 5)
    k_gemm_thin(const double* __restrict__ X, const double* __restrict__ Y, double* __restrict__ C,
                const GemmCBlock* __restrict__ cblocks, int32_t ncb, const GemmPair* __restrict__ pairs) {
  using TL = ThinLayout<SR, XT, YT>;
  static_assert(2 * TL::LSZ >= kThinBig * 17, "C staging must fit in the long-operand buffers");
  __shared__ double Ls[2][TL::LSZ];
  __shared__ double Ss[2][TL::SSZ];
  double* Cs = &Ls[0][0];  // reused for the C tile after the last pair
  int lo = 0, hi = ncb - 1;
  const int bid = static_cast<int>(blockIdx.x);
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cblocks[mid].tile_begin <= bid) lo = mid; else hi = mid - 1;
  }
  // a group of S = mtiles blocks ending at lo numbers its strips in turn
  const int grp = cblocks[lo].mtiles, rel = bid - cblocks[lo].tile_begin;
  const GemmCBlock cb = cblocks[lo - (grp - 1) + rel % grp];
  const int M = cb.M, N = cb.N;
  const int L = SR ? N : M;   // long extent
  const int ns = SR ? M : N;  // short extent (<= 16)
  const int l0 = (rel / grp) * kThinBig;
  const int tid = threadIdx.x;

  // Load geometry: the long tile's elements of this thread share their k
  // (k-contiguous layout) or their l (l-contiguous layout) and step the other
  // index by a constant; the small tile's by 8 rows.
  const int lleft = L - l0;
  const int tq = tid & 15, tr = tid >> 4;
  auto load = [&](int stage, const GemmPair& pr) {
    const int K = pr.K;
    const double* lbase = SR ? Y + pr.y_off : X + pr.x_off;
    const double* sbase = SR ? X + pr.x_off : Y + pr.y_off;
    const int64_t lld = SR ? pr.ldy : pr.ldx;
    const int64_t sld = SR ? pr.ldx : pr.ldy;
    // long tile: kThinBig x 16
    constexpr int LR = kThinBig * 16 / kThinThreads;
    if (TL::LONG_KCONTIG) {
      // element (l = tr + 8 r, k = tq) at lbase + k + (l0 + l) * lld
      const double* lp = lbase + tq + static_cast<int64_t>(l0 + tr) * lld;
      double* dst = &Ls[stage][tr * kThinKP + tq];
#pragma unroll
      for (int r = 0; r < LR; ++r) {
        const bool v = tr + 8 * r < lleft && tq < K;
        cp_async8(dst + r * 8 * kThinKP, v ? lp + static_cast<int64_t>(8 * r) * lld : lbase, v);
      }
    } else {
      // element (l = tid, k = r) at lbase + (l0 + l) + k * lld
      const double* lp = lbase + l0 + tid;
      double* dst = &Ls[stage][tid];
#pragma unroll
      for (int r = 0; r < LR; ++r) {
        const bool v = tid < lleft && r < K;
        cp_async8(dst + r * kThinBP, v ? lp + static_cast<int64_t>(r) * lld : lbase, v);
      }
    }
    // small tile: 16 x 16; the global-contiguous index (k or s) is tq, the
    // other one tr + 8 r
    const double* sp = sbase + tq + static_cast<int64_t>(tr) * sld;
    double* sdst = &Ss[stage][tr * kThinKP + tq];
#pragma unroll
    for (int r = 0; r < 256 / kThinThreads; ++r) {
      const int o = tr + 8 * r;
      const bool v = TL::SMALL_KCONTIG ? (o < ns && tq < K) : (tq < ns && o < K);
      cp_async8(sdst + r * 8 * kThinKP, v ? sp + static_cast<int64_t>(8 * r) * sld : sbase, v);
    }
  };

  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  // !SR: warp owns long rows [warp*32, +32) x 16 short columns: 4 x 2 m8n8 tiles
  //  SR: warp owns long columns [warp*32, +32) x 16 short rows: 2 x 4 tiles
  double acc[8][2];
#pragma unroll
  for (int a = 0; a < 8; ++a) acc[a][0] = acc[a][1] = 0.0;

  const int p0 = cb.pair_begin, p1 = cb.pair_end;
  // pair descriptors are read one pair ahead of their copies
  GemmPair pnext{};
  if (p0 < p1) load(0, pairs[p0]);
  if (p0 + 1 < p1) pnext = pairs[p0 + 1];
  cp_async_commit();
  for (int p = p0; p < p1; ++p) {
    const int st = (p - p0) & 1;
    if (p + 1 < p1) {
      load(st ^ 1, pnext);
      if (p + 2 < p1) pnext = pairs[p + 2];
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double* ls = Ls[st];
    const double* ss = Ss[st];
#pragma unroll
    for (int k4 = 0; k4 < 16; k4 += 4) {
      if (!SR) {
        double af[4], bf[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) af[a] = ls[TL::lidx(warp * 32 + a * 8 + g, k4 + t)];
#pragma unroll
        for (int b = 0; b < 2; ++b) bf[b] = ss[TL::sidx(k4 + t, b * 8 + g)];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b) dmma_8x8x4(acc[a * 2 + b][0], acc[a * 2 + b][1], af[a], bf[b]);
      } else {
        double af[2], bf[4];
#pragma unroll
        for (int a = 0; a < 2; ++a) af[a] = ss[TL::sidx(k4 + t, a * 8 + g)];
#pragma unroll
        for (int b = 0; b < 4; ++b) bf[b] = ls[TL::lidx(warp * 32 + b * 8 + g, k4 + t)];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a * 4 + b][0], acc[a * 4 + b][1], af[a], bf[b]);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  __syncthreads();
  // stage C tile as Cs[l * 17 + s] (long index l, short index s)
  if (!SR) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int l = warp * 32 + a * 8 + g, s0 = b * 8 + 2 * t;
        Cs[l * 17 + s0] = acc[a * 2 + b][0];
        Cs[l * 17 + s0 + 1] = acc[a * 2 + b][1];
      }
  } else {
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int s = a * 8 + g, l0c = warp * 32 + b * 8 + 2 * t;
        Cs[l0c * 17 + s] = acc[a * 4 + b][0];
        Cs[(l0c + 1) * 17 + s] = acc[a * 4 + b][1];
      }
  }
  __syncthreads();
  double* cbase = C + cb.c_off;
  const int nl = min(kThinBig, L - l0);
  if (!SR) {
    // C(i = l0 + l, j = s) at i + j*ldc: coalesced along l for each s
    for (int e = tid; e < nl * ns; e += kThinThreads) {
      const int l = e % nl, s = e / nl;
      cbase[(l0 + l) + (int64_t)s * cb.ldc] = Cs[l * 17 + s];
    }
  } else {
    // C(i = s, j = l0 + l) at s + (l0 + l)*M with M = ns: one contiguous run
    double* run = cbase + (int64_t)l0 * M;
    for (int e = tid; e < nl * ns; e += kThinThreads) run[e] = Cs[(e / ns) * 17 + (e % ns)];
  }
}

// Persistent variant of k_gemm_thin: a fixed grid of CTAs walks the 128-long
// strips (tiles) with stride gridDim.x, and the double-buffered copy pipeline
// runs across tile boundaries, so the first pair of the next strip is in
// flight while the current one finishes; C is stored straight from the DMMA
// fragments (runs of 8 consecutive doubles per column).
// LF: the long operand and C hold FP32 values (staged as FP32, widened to FP64
// when read into the DMMA fragments; C rounded to FP32 when stored).
template <bool SR, bool XT, bool YT, bool LF = false>
__global__ void __launch_bounds__(kThinThreads, 5)
    k_gemm_thin_p(const double* __restrict__ X, const double* __restrict__ Y, double* __restrict__ C,
                  const GemmCBlock* __restrict__ cblocks, int32_t ncb, const GemmPair* __restrict__ pairs,
                  int32_t ntiles) {
  using TL = ThinLayout<SR, XT, YT>;
  __shared__ double Ls[2][TL::LSZ];  // FP32 long tiles use the first half of each stage
  __shared__ double Ss[2][TL::SSZ];
  const int tid = threadIdx.x;
  const int tq = tid & 15, tr = tid >> 4;

  // C block of a strip: the last c with tile_begin <= tile.  A CTA visits its
  // strips in increasing order, so the search gallops forward from the block
  // of the previous strip and then bisects; with blocks of many strips it is
  // one probe, where a bisection over all blocks is a chain of ~log2(ncb)
  // dependent global loads on the loop's critical path.
  int cur = 0;
  auto find = [&](int tile, GemmCBlock& cb, int& l0) {
    int lo = cur, step = 1;
    while (lo + step < ncb && cblocks[lo + step].tile_begin <= tile) {
      lo += step;
      step <<= 1;
    }
    int hi = min(lo + step, ncb) - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cblocks[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    cur = lo;
    // a group of S = mtiles blocks ending at lo numbers its strips in turn
    const int grp = cblocks[lo].mtiles, rel = tile - cblocks[lo].tile_begin;
    cb = cblocks[lo - (grp - 1) + rel % grp];
    l0 = (rel / grp) * kThinBig;
  };
  auto load = [&](int stage, const GemmPair& pr, const GemmCBlock& cb, int l0) {
    const int K = pr.K;
    const int L = SR ? cb.N : cb.M, ns = SR ? cb.M : cb.N;
    const int lleft = L - l0;
    const double* sbase = SR ? X + pr.x_off : Y + pr.y_off;
    const int64_t lld = SR ? pr.ldy : pr.ldx;
    const int64_t sld = SR ? pr.ldx : pr.ldy;
    constexpr int LR = kThinBig * 16 / kThinThreads;
    if (LF) {
      const float* lbase = reinterpret_cast<const float*>(SR ? Y : X) + (SR ? pr.y_off : pr.x_off);
      float* lsf = reinterpret_cast<float*>(&Ls[stage][0]);
      if (TL::LONG_KCONTIG) {
        const float* lp = lbase + tq + static_cast<int64_t>(l0 + tr) * lld;
        float* dst = lsf + tr * kThinKP + tq;
#pragma unroll
        for (int r = 0; r < LR; ++r) {
          const bool v = tr + 8 * r < lleft && tq < K;
          cp_async4(dst + r * 8 * kThinKP, v ? lp + static_cast<int64_t>(8 * r) * lld : lbase, v);
        }
      } else {
        const float* lp = lbase + l0 + tid;
        float* dst = lsf + tid;
#pragma unroll
        for (int r = 0; r < LR; ++r) {
          const bool v = tid < lleft && r < K;
          cp_async4(dst + r * kThinBP, v ? lp + static_cast<int64_t>(r) * lld : lbase, v);
        }
      }
    } else {
      const double* lbase = SR ? Y + pr.y_off : X + pr.x_off;
      if (TL::LONG_KCONTIG) {
        const double* lp = lbase + tq + static_cast<int64_t>(l0 + tr) * lld;
        double* dst = &Ls[stage][tr * kThinKP + tq];
#pragma unroll
        for (int r = 0; r < LR; ++r) {
          const bool v = tr + 8 * r < lleft && tq < K;
          cp_async8(dst + r * 8 * kThinKP, v ? lp + static_cast<int64_t>(8 * r) * lld : lbase, v);
        }
      } else {
        const double* lp = lbase + l0 + tid;
        double* dst = &Ls[stage][tid];
#pragma unroll
        for (int r = 0; r < LR; ++r) {
          const bool v = tid < lleft && r < K;
          cp_async8(dst + r * kThinBP, v ? lp + static_cast<int64_t>(r) * lld : lbase, v);
        }
      }
    }
    const double* sp = sbase + tq + static_cast<int64_t>(tr) * sld;
    double* sdst = &Ss[stage][tr * kThinKP + tq];
#pragma unroll
    for (int r = 0; r < 256 / kThinThreads; ++r) {
      const int o = tr + 8 * r;
      const bool v = TL::SMALL_KCONTIG ? (o < ns && tq < K) : (tq < ns && o < K);
      cp_async8(sdst + r * 8 * kThinKP, v ? sp + static_cast<int64_t>(8 * r) * sld : sbase, v);
    }
  };

  int ltile = blockIdx.x;
  if (ltile >= ntiles) return;
  GemmCBlock lcb, ccb;
  int ll0, cl0;
  find(ltile, lcb, ll0);
  int lp = lcb.pair_begin;
  load(0, pairs[lp], lcb, ll0);
  cp_async_commit();
  ccb = lcb;
  cl0 = ll0;
  int cpair = lp;
  auto advance = [&]() {
    if (++lp >= lcb.pair_end) {
      ltile += gridDim.x;
      if (ltile < ntiles) {
        find(ltile, lcb, ll0);
        lp = lcb.pair_begin;
      }
    }
  };
  advance();

  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  auto lval = [&](const double* ls, int idx) -> double {
    if (LF) return static_cast<double>(reinterpret_cast<const float*>(ls)[idx]);
    return ls[idx];
  };
  double acc[8][2];
#pragma unroll
  for (int a = 0; a < 8; ++a) acc[a][0] = acc[a][1] = 0.0;
  int st = 0;
  while (true) {
    const bool more = ltile < ntiles;
    if (more) load(st ^ 1, pairs[lp], lcb, ll0);
    cp_async_commit();
    // the pair just issued becomes current next iteration; look up the one
    // after it now, while this stage's copies are still in flight
    const GemmCBlock icb = lcb;
    const int il0 = ll0, ipair = lp;
    if (more) advance();
    cp_async_wait<1>();
    __syncthreads();
    const double* ls = Ls[st];
    const double* ss = Ss[st];
#pragma unroll
    for (int k4 = 0; k4 < 16; k4 += 4) {
      if (!SR) {
        double af[4], bf[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) af[a] = lval(ls, TL::lidx(warp * 32 + a * 8 + g, k4 + t));
#pragma unroll
        for (int b = 0; b < 2; ++b) bf[b] = ss[TL::sidx(k4 + t, b * 8 + g)];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b) dmma_8x8x4(acc[a * 2 + b][0], acc[a * 2 + b][1], af[a], bf[b]);
      } else {
        double af[2], bf[4];
#pragma unroll
        for (int a = 0; a < 2; ++a) af[a] = ss[TL::sidx(k4 + t, a * 8 + g)];
#pragma unroll
        for (int b = 0; b < 4; ++b) bf[b] = lval(ls, TL::lidx(warp * 32 + b * 8 + g, k4 + t));
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a * 4 + b][0], acc[a * 4 + b][1], af[a], bf[b]);
      }
    }
    __syncthreads();  // stage st is free for the next copy
    if (cpair + 1 == ccb.pair_end) {
      // last pair of this strip: store it from the fragments and start over
      const int M = ccb.M;
      const int64_t ldc = ccb.ldc;
      auto cstore = [&](int64_t off, double v) {
        if (LF) reinterpret_cast<float*>(C)[ccb.c_off + off] = static_cast<float>(v);
        else C[ccb.c_off + off] = v;
      };
      if (!SR) {
        const int L = M, ns = ccb.N;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const int l = cl0 + warp * 32 + a * 8 + g;
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const int s0 = b * 8 + 2 * t;
            if (l < L && s0 < ns) cstore(l + s0 * ldc, acc[a * 2 + b][0]);
            if (l < L && s0 + 1 < ns) cstore(l + (s0 + 1) * ldc, acc[a * 2 + b][1]);
          }
        }
      } else {
        const int L = ccb.N, ns = M;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          const int sI = a * 8 + g;
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int l = cl0 + warp * 32 + b * 8 + 2 * t;
            if (sI < ns && l < L) cstore(sI + l * ldc, acc[a * 4 + b][0]);
            if (sI < ns && l + 1 < L) cstore(sI + (l + 1) * ldc, acc[a * 4 + b][1]);
          }
        }
      }
#pragma unroll
      for (int a = 0; a < 8; ++a) acc[a][0] = acc[a][1] = 0.0;
    }
    if (!more) break;
    ccb = icb;
    cl0 = il0;
    cpair = ipair;
    st ^= 1;
  }
  cp_async_wait<0>();
}

// The persistent grid: every SM's resident CTAs of this instantiation (5 for
// the 38 KB shared-memory layouts, 4 for the 45 KB ones), queried once per
// device.
template <bool SR, bool XT, bool YT, bool LF = false>
cudaError_t launch_thin_p(const double* X, const double* Y, double* C, const GemmCBlock* cb, int32_t ncb,
                          const GemmPair* pr, int64_t nctas, cudaStream_t s) {
  static std::atomic<int> grid_of[64] = {};  // host threads may race on the first call
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int grid = grid_of[dev & 63].load();
  if (grid == 0) {
    int sms = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gemm_thin_p<SR, XT, YT, LF>, kThinThreads, 0);
    if (e != cudaSuccess) return e;
    grid = sms * std::max(per_sm, 1);
    grid_of[dev & 63].store(grid);
  }
  const unsigned g = static_cast<unsigned>(std::min<int64_t>(nctas, grid));
  k_gemm_thin_p<SR, XT, YT, LF><<<g, kThinThreads, 0, s>>>(X, Y, C, cb, ncb, pr, static_cast<int32_t>(nctas));
  return cudaGetLastError();
}

template <bool SR>
cudaError_t thin_t(bool xT, bool yT, const double* X, const double* Y, double* C, const GemmCBlock* cb, int32_t ncb,
                   const GemmPair* pr, int64_t nctas, bool persistent, cudaStream_t s, bool lf) {
  if (lf) {
    if (!persistent) return cudaErrorInvalidValue;
    if (!xT && !yT) return launch_thin_p<SR, false, false, true>(X, Y, C, cb, ncb, pr, nctas, s);
    if (!xT && yT) return launch_thin_p<SR, false, true, true>(X, Y, C, cb, ncb, pr, nctas, s);
    if (xT && !yT) return launch_thin_p<SR, true, false, true>(X, Y, C, cb, ncb, pr, nctas, s);
    return launch_thin_p<SR, true, true, true>(X, Y, C, cb, ncb, pr, nctas, s);
  }
  if (persistent) {
    if (!xT && !yT) return launch_thin_p<SR, false, false>(X, Y, C, cb, ncb, pr, nctas, s);
    if (!xT && yT) return launch_thin_p<SR, false, true>(X, Y, C, cb, ncb, pr, nctas, s);
    if (xT && !yT) return launch_thin_p<SR, true, false>(X, Y, C, cb, ncb, pr, nctas, s);
    return launch_thin_p<SR, true, true>(X, Y, C, cb, ncb, pr, nctas, s);
  }
  const unsigned g = static_cast<unsigned>(nctas);
  if (!xT && !yT) k_gemm_thin<SR, false, false><<<g, kThinThreads, 0, s>>>(X, Y, C, cb, ncb, pr);
  else if (!xT && yT) k_gemm_thin<SR, false, true><<<g, kThinThreads, 0, s>>>(X, Y, C, cb, ncb, pr);
  else if (xT && !yT) k_gemm_thin<SR, true, false><<<g, kThinThreads, 0, s>>>(X, Y, C, cb, ncb, pr);
  else k_gemm_thin<SR, true, true><<<g, kThinThreads, 0, s>>>(X, Y, C, cb, ncb, pr);
  return cudaGetLastError();
}

}  // namespace

void gemm_tile_dims(GemmShape shape, int* bm, int* bn) {
  switch (shape) {
    case GemmShape::T128x32: *bm = 128; *bn = 32; break;
    case GemmShape::T32x128: *bm = 32; *bn = 128; break;
    case GemmShape::T128x64: *bm = 128; *bn = 64; break;
    case GemmShape::T64x128: *bm = 64; *bn = 128; break;
    case GemmShape::T64x32: *bm = 64; *bn = 32; break;
    default: *bm = 64; *bn = 64; break;
  }
}

cudaError_t launch_gemm_f64_skinny(const double* X, const double* Y, double* C, const GemmCBlock* d_cblocks,
                                   int32_t ncb, const GemmPair* d_pairs, int64_t nctas, bool xT, bool yT,
                                   bool small_rows, int small_max, int k_max, cudaStream_t s, bool persistent,
                                   bool long_f32) {
  if (nctas <= 0) return cudaSuccess;
  if (nctas > 0x7fffffffLL || small_max > 16 || k_max > 16) return cudaErrorInvalidValue;
  return small_rows ? thin_t<true>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, nctas, persistent, s, long_f32)
                    : thin_t<false>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, nctas, persistent, s, long_f32);
}

template <bool XT, bool YT>
cudaError_t launch_edges_t(const double* X, const double* Y, double* C, const GemmCBlock* cb, int32_t ncb,
                           const GemmPair* pr, int64_t ntiles, int splitk, double* partial, cudaStream_t s) {
  constexpr int smem = std::max(std::max(TileLayout<64, 64, XT, YT>::bytes(), TileLayout<64, 32, XT, YT>::bytes()),
                                TileLayout<32, 64, XT, YT>::bytes());
  auto kern = k_gemm_f64_edges<XT, YT>;
  static std::atomic<unsigned long long> configured{0};  // one bit per device ordinal (host threads may race)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(configured & bit)) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit);
  }
  kern<<<static_cast<unsigned>(ntiles * splitk), kEdgeThreads, smem, s>>>(X, Y, C, cb, ncb, pr, splitk,
                                                                          static_cast<int32_t>(ntiles), partial);
  e = cudaGetLastError();
  if (e != cudaSuccess || splitk == 1) return e;
  const int64_t elems = ntiles * kEdgePart;
  const unsigned g = static_cast<unsigned>(std::min<int64_t>((elems + 255) / 256, 148LL * 64));
  k_splitk_reduce_edges<<<g, 256, 0, s>>>(C, cb, ncb, splitk, static_cast<int32_t>(ntiles), partial);
  return cudaGetLastError();
}

cudaError_t launch_gemm_f64_edges(const double* X, const double* Y, double* C, const GemmCBlock* d_cblocks,
                                  int32_t ncb, const GemmPair* d_pairs, int64_t ntiles, bool xT, bool yT,
                                  cudaStream_t s, int splitk, double* partial) {
  if (ntiles <= 0) return cudaSuccess;
  if (splitk < 1 || ntiles * splitk > 0x7fffffffLL || (splitk > 1 && !partial)) return cudaErrorInvalidValue;
  if (!xT && !yT) return launch_edges_t<false, false>(X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
  if (!xT && yT) return launch_edges_t<false, true>(X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
  if (xT && !yT) return launch_edges_t<true, false>(X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
  return launch_edges_t<true, true>(X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
}

cudaError_t launch_gemm_f64(const double* X, const double* Y, double* C,
                            const GemmCBlock* d_cblocks, int32_t ncb, const GemmPair* d_pairs,
                            int64_t ntiles, bool xT, bool yT, GemmShape shape, cudaStream_t s,
                            int splitk, double* partial) {
  switch (shape) {
    case GemmShape::T128x32:
      return dispatch_t<128, 32, 32, 32>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
    case GemmShape::T32x128:
      return dispatch_t<32, 128, 32, 32>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
    case GemmShape::T128x64:
      return dispatch_t<128, 64, 32, 32>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
    case GemmShape::T64x128:
      return dispatch_t<64, 128, 32, 32>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
    case GemmShape::T64x32:
      return dispatch_t<64, 32, 32, 16, 16, 4>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
    default:
      return dispatch_t<64, 64, 32, 32>(xT, yT, X, Y, C, d_cblocks, ncb, d_pairs, ntiles, splitk, partial, s);
  }
}

}  // namespace sb

// ── allocation-free grouped GEMM (sb_block_gemm_f64_noalloc) ───────────────
//
// For callers that cannot allocate device memory themselves or let a library
// do it: code running under a strict memory budget or a pre-sized pool, or
// hosts (e.g. a Julia CUDA.jl or embedded runtime) that forbid cudaMalloc
// during a solve.  The plan descriptors that sb_contract keeps in allocated
// device buffers live instead in this file-scope device array, which every GPU
// that loads the library holds until process exit.  Limits: at most
// kNoAllocMaxCBlocks output blocks and kNoAllocMaxPairs block pairs per call
// (672 KiB of scratch).
namespace {

constexpr int kNoAllocMaxCBlocks = 4096;
constexpr int kNoAllocMaxPairs = 16384;
constexpr size_t kNoAllocScratchBytes =
    kNoAllocMaxCBlocks * sizeof(sb::GemmCBlock) + kNoAllocMaxPairs * sizeof(sb::GemmPair);

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device ordinal, resolved once per
// device (with that device current) by cudaGetSymbolAddress.
constexpr int kMaxDevices = 64;
std::atomic<void*> g_scratch_addr[kMaxDevices] = {};

// Host staging of the plan; per thread so concurrent host threads do not share it.
thread_local sb::GemmCBlock t_cblocks[kNoAllocMaxCBlocks];
thread_local sb::GemmPair t_pairs[kNoAllocMaxPairs];
thread_local char* t_err = nullptr;
thread_local int32_t t_err_len = 0;

sb_status noalloc_fail(sb_status code, const char* msg) {
  if (t_err && t_err_len > 0) std::snprintf(t_err, static_cast<size_t>(t_err_len), "sb_block_gemm_f64_noalloc: %s", msg);
  return code;
}

}  // namespace

extern "C" SB_API sb_status sb_block_gemm_f64_noalloc(void* stream, const double* d_X, const double* d_Y, double* d_C,
                                                      int32_t n_cblocks, const int64_t* c_off, const int32_t* c_rows,
                                                      const int32_t* c_cols, const int32_t* c_pair_begin,
                                                      const int64_t* x_off, const int64_t* y_off, const int32_t* K,
                                                      const int32_t* ldx, const int32_t* ldy, int x_trans,
                                                      int y_trans, char* err, int32_t err_len) {
  t_err = err;
  t_err_len = err_len;
  if (err && err_len > 0) err[0] = '\0';
  if (n_cblocks < 0) return noalloc_fail(SB_ERR_INVALID_ARG, "n_cblocks < 0");
  if (n_cblocks == 0) return SB_OK;
  if (!d_X || !d_Y || !d_C || !c_off || !c_rows || !c_cols || !c_pair_begin)
    return noalloc_fail(SB_ERR_INVALID_ARG, "NULL pointer argument");
  if (n_cblocks > kNoAllocMaxCBlocks) {
    char m[160];
    std::snprintf(m, sizeof(m), "%d output blocks exceed the static scratch limit of %d", n_cblocks, kNoAllocMaxCBlocks);
    return noalloc_fail(SB_ERR_INVALID_ARG, m);
  }
  const int32_t n_pairs = c_pair_begin[n_cblocks];
  if (c_pair_begin[0] != 0 || n_pairs < 0) return noalloc_fail(SB_ERR_INVALID_ARG, "c_pair_begin must start at 0");
  if (n_pairs > kNoAllocMaxPairs) {
    char m[160];
    std::snprintf(m, sizeof(m), "%d block pairs exceed the static scratch limit of %d", n_pairs, kNoAllocMaxPairs);
    return noalloc_fail(SB_ERR_INVALID_ARG, m);
  }
  if (n_pairs > 0 && (!x_off || !y_off || !K || !ldx || !ldy))
    return noalloc_fail(SB_ERR_INVALID_ARG, "NULL pair array");

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(SB_ERR_CUDA, "no usable current CUDA device");
  // One-time set-up on this device (the first call on a device must not be
  // inside a stream capture).
  void* scratch = g_scratch_addr[dev].load();
  if (!scratch) {
    const cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess || !scratch) return noalloc_fail(SB_ERR_CUDA, cudaGetErrorString(e));
    g_scratch_addr[dev].store(scratch);  // every thread resolves the same address
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The plan is copied from host arrays at call time, which a captured graph
  // could not repeat: calls on a capturing stream are rejected.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return noalloc_fail(SB_ERR_INVALID_ARG, "the stream is capturing (or cannot be queried); the plan copy reads "
                                            "host memory at call time");
  auto* d_cb = static_cast<sb::GemmCBlock*>(scratch);
  auto* d_pr = reinterpret_cast<sb::GemmPair*>(static_cast<unsigned char*>(scratch) +
                                               kNoAllocMaxCBlocks * sizeof(sb::GemmCBlock));

  // Tile shape: same rule as the library's allocating path.
  int32_t Mx = 0, Nx = 0;
  for (int32_t c = 0; c < n_cblocks; ++c) {
    if (c_rows[c] < 1 || c_cols[c] < 1) return noalloc_fail(SB_ERR_INVALID_ARG, "C block extents must be >= 1");
    if (c_pair_begin[c + 1] < c_pair_begin[c]) return noalloc_fail(SB_ERR_INVALID_ARG, "c_pair_begin not monotone");
    Mx = c_rows[c] > Mx ? c_rows[c] : Mx;
    Nx = c_cols[c] > Nx ? c_cols[c] : Nx;
  }
  sb::GemmShape shape = sb::GemmShape::T64x64;
  if (Nx <= 32 && Mx >= 128) shape = sb::GemmShape::T128x32;
  else if (Mx <= 32 && Nx >= 128) shape = sb::GemmShape::T32x128;
  else if (Mx >= 256 && Nx >= 128) shape = Mx >= Nx ? sb::GemmShape::T128x64 : sb::GemmShape::T64x128;
  int bm = 64, bn = 64;
  sb::gemm_tile_dims(shape, &bm, &bn);

  int64_t ntiles = 0;
  for (int32_t c = 0; c < n_cblocks; ++c) {
    const int64_t mt = (c_rows[c] + bm - 1) / bm, nt = (c_cols[c] + bn - 1) / bn;
    if (ntiles + mt * nt >= (1LL << 31)) return noalloc_fail(SB_ERR_INVALID_ARG, "too many GEMM tiles");
    t_cblocks[c] = sb::GemmCBlock{c_off[c], c_rows[c], c_cols[c], c_pair_begin[c], c_pair_begin[c + 1],
                                  static_cast<int32_t>(ntiles), static_cast<int32_t>(mt), c_rows[c], 0};
    ntiles += mt * nt;
  }
  for (int32_t c = 0; c < n_cblocks; ++c) {
    if (c_off[c] < 0) return noalloc_fail(SB_ERR_INVALID_ARG, "negative c_off");
    for (int32_t p = c_pair_begin[c]; p < c_pair_begin[c + 1]; ++p) {
      if (K[p] < 1) return noalloc_fail(SB_ERR_INVALID_ARG, "pair K must be >= 1");
      if (x_off[p] < 0 || y_off[p] < 0) return noalloc_fail(SB_ERR_INVALID_ARG, "negative x_off or y_off");
      // leading dimensions at least the contiguous extent of each operand block
      if (ldx[p] < (x_trans ? K[p] : c_rows[c]) || ldy[p] < (y_trans ? c_cols[c] : K[p]))
        return noalloc_fail(SB_ERR_INVALID_ARG, "ldx or ldy below the block's leading extent");
      t_pairs[p] = sb::GemmPair{x_off[p], y_off[p], K[p], ldx[p], ldy[p], 0};
    }
  }
  // Every call rewrites the descriptors it uses; nothing in the scratch has to
  // start at zero.  Copies from pageable host memory return once the data is
  // staged, so the thread-local host arrays may be reused on the next call.
  cudaError_t e = cudaMemcpyAsync(d_cb, t_cblocks, n_cblocks * sizeof(sb::GemmCBlock), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n_pairs)
    e = cudaMemcpyAsync(d_pr, t_pairs, n_pairs * sizeof(sb::GemmPair), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = sb::launch_gemm_f64(d_X, d_Y, d_C, d_cb, n_cblocks, d_pr, ntiles, x_trans != 0, y_trans != 0, shape, s);
  if (e != cudaSuccess) return noalloc_fail(SB_ERR_CUDA, cudaGetErrorString(e));
  return SB_OK;
}
