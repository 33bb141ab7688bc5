// Bandwidth-bound kernels of the block-sparse contraction engine (sm_100a):
// tail permutes (tiled shared-memory transposes), outer-product and scaled
// segmented accumulation with the reference's rounding, structure flags,
// gathers/scatters and the scalar programs of the aliased format.
#include <algorithm>
#include <atomic>

#include "sb_kernels.hpp"

namespace sb {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n, int per_block = kThreads) {
  int64_t g = (n + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > 148LL * 32) g = 148LL * 32;  // grid-stride loops beyond this
  return static_cast<unsigned>(g);
}

// ── outer-product accumulation ────────────────────────────────────────────
__global__ void k_outer_acc(const double* __restrict__ A, const double* __restrict__ B,
                            double* __restrict__ C, const OuterCBlock* __restrict__ cbs,
                            int64_t ncb, const OuterPair* __restrict__ pairs, bool kahan) {
  for (int64_t c = blockIdx.y; c < ncb; c += gridDim.y) {
    const OuterCBlock cb = cbs[c];
    const int64_t n = (int64_t)cb.M * cb.N;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
      const int64_t i = e % cb.M, j = e / cb.M;
      double acc = 0.0, comp = 0.0;
      if (kahan) {
        for (int p = cb.pair_begin; p < cb.pair_end; ++p) {
          const double prod = __dmul_rn(A[pairs[p].a_off + i], B[pairs[p].b_off + j]);
          const double y = __dsub_rn(prod, comp);
          const double t = __dadd_rn(acc, y);
          comp = __dsub_rn(__dsub_rn(t, acc), y);
          acc = t;
        }
      } else {
        for (int p = cb.pair_begin; p < cb.pair_end; ++p)
          acc = __dadd_rn(acc, __dmul_rn(A[pairs[p].a_off + i], B[pairs[p].b_off + j]));
      }
      C[cb.c_off + e] = acc;
    }
  }
}

// ── segmented scaled accumulation ─────────────────────────────────────────
__global__ void k_axpy_seg(const double* __restrict__ src, const double* __restrict__ alpha,
                           double* __restrict__ C, const AxpySeg* __restrict__ segs, int64_t nsegs,
                           const AxpyEntry* __restrict__ ents) {
  for (int64_t g = blockIdx.y; g < nsegs; g += gridDim.y) {
    const AxpySeg sg = segs[g];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < sg.len;
         t += (int64_t)gridDim.x * blockDim.x) {
      double acc = 0.0;
      for (int e = sg.e_begin; e < sg.e_end; ++e) {
        const AxpyEntry en = ents[e];
        const double a = en.alpha_idx >= 0 ? alpha[en.alpha_idx] : 1.0;
        acc = __dadd_rn(acc, __dmul_rn(a, src[en.src_off + t]));
      }
      C[sg.c_off + t] = acc;
    }
  }
}

// ── permutes ──────────────────────────────────────────────────────────────
// General gather: consecutive threads write consecutive output elements.
__global__ void k_permute_general(const double* __restrict__ src, double* __restrict__ dst,
                                  const int64_t* __restrict__ src_off, int64_t nblocks, int64_t blk,
                                  PermDesc d) {
  const int64_t total = nblocks * blk;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = idx / blk;
    int64_t e = idx - b * blk;
    int64_t so = 0;
    for (int r = 0; r < d.rank; ++r) {
      const int64_t c = e % d.out_dims[r];
      e /= d.out_dims[r];
      so += c * d.in_strides[r];
    }
    dst[idx] = src[src_off[b] + so];
  }
}

// Contiguous runs: output axis 0 has unit source stride too, so every run of
// the leading output axes that are contiguous in both layouts (len doubles) is
// a straight copy.  One warp per run: the source offset of a run is computed
// once, then the lanes copy it with coalesced accesses, four loads in flight
// per lane.
__global__ void k_permute_runs(const double* __restrict__ src, double* __restrict__ dst,
                               const int64_t* __restrict__ src_off, int64_t blk, int64_t len, int64_t runs_per_block,
                               int64_t total_runs, PermDesc d, int first_outer) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t run = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; run < total_runs;
       run += warps) {
    const int64_t b = run / runs_per_block;
    int64_t rr = run - b * runs_per_block;
    const double* s = src + src_off[b];
    double* o = dst + b * blk + rr * len;
    for (int r = first_outer; r < d.rank; ++r) {
      const int64_t c = rr % d.out_dims[r];
      rr /= d.out_dims[r];
      s += c * d.in_strides[r];
    }
#pragma unroll 4
    for (int64_t e = lane; e < len; e += 32) o[e] = s[e];
  }
}

// Transposes: output axis q is the first with unit source stride; the output
// axes before it, flattened, are the row axis v (contiguous in the output,
// extent dv, each row's source offset decomposed from its index), output
// axis q is u (extent du, output stride dv), and the axes after it are a
// batch.  A tile is read coalesced along u and written coalesced along v.
struct TileDesc {
  int64_t dv, du;        // extents of the row axis (output axes before q) and of output axis q
  int nv;                // number of output axes before q
  int64_t vdims[kMaxRank];
  int64_t vsrc[kMaxRank];  // their source strides
  int64_t ou;            // output stride of output axis q
  int nb;                // number of batch axes
  int64_t bdims[kMaxRank];
  int64_t bsrc[kMaxRank];
  int64_t bdst[kMaxRank];
  int64_t nbatch, tiles_u, tiles_v;
};

// Source offset of row v (relative to the tile's batch base).
__device__ __forceinline__ int64_t row_src(const TileDesc& d, int64_t v) {
  int64_t off = 0;
  for (int r = 0; r < d.nv - 1; ++r) {
    const int64_t c = v % d.vdims[r];
    v /= d.vdims[r];
    off += c * d.vsrc[r];
  }
  return off + v * d.vsrc[d.nv - 1];
}
constexpr int kTileU = 64;   // tile extent along output axis q (unit source stride)
constexpr int kTileV = 64;   // tile extent along output axis 0
constexpr int kNarrowSmem = 64 * 1024;  // narrow transpose: shared memory of a tile (bytes)

// Source and destination bases of tile `cta` (tiles_u x tiles_v x batch x block).
__device__ __forceinline__ void tile_bases(const TileDesc& d, const int64_t* __restrict__ src_off, int64_t blk,
                                           int64_t cta, int64_t& tu, int64_t& tv, int64_t& sb, int64_t& db) {
  int64_t t = cta;
  tu = t % d.tiles_u; t /= d.tiles_u;
  tv = t % d.tiles_v; t /= d.tiles_v;
  int64_t bt = t % d.nbatch;
  const int64_t b = t / d.nbatch;
  sb = src_off[b];
  db = b * blk;
  for (int r = 0; r < d.nb; ++r) {
    const int64_t c = bt % d.bdims[r];
    bt /= d.bdims[r];
    sb += c * d.bsrc[r];
    db += c * d.bdst[r];
  }
}

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Persistent: each CTA walks its tiles with stride gridDim.x through two
// shared-memory buffers; the copies of the next tile (cp.async, no registers)
// are in flight while the current one is stored.
constexpr int kTilePitch = kTileV + 1;
constexpr int kTileElems = kTileU * kTilePitch;
__global__ void __launch_bounds__(256) k_permute_tiled(const double* __restrict__ src, double* __restrict__ dst,
                                                      const int64_t* __restrict__ src_off, int64_t blk, TileDesc d,
                                                      int64_t total_ctas) {
  extern __shared__ double ttile[];
  auto issue = [&](int64_t cta, double* buf) {
    int64_t tu, tv, sb, db;
    tile_bases(d, src_off, blk, cta, tu, tv, sb, db);
    const int64_t u0 = tu * kTileU, v0 = tv * kTileV;
#pragma unroll
    for (int j = 0; j < kTileV / 8; ++j) {
      const int yy = threadIdx.y + 8 * j;
      const int64_t v = v0 + yy;
      if (v >= d.dv) continue;
      const double* row = src + sb + row_src(d, v);
#pragma unroll
      for (int h = 0; h < kTileU / 32; ++h) {
        const int64_t u = u0 + h * 32 + threadIdx.x;
        if (u < d.du) cp_async8(&buf[(h * 32 + threadIdx.x) * kTilePitch + yy], row + u);
      }
    }
  };
  int64_t cta = blockIdx.x;
  if (cta >= total_ctas) return;
  issue(cta, ttile);
  cp_async_commit();
  int b = 0;
  for (; cta < total_ctas; cta += gridDim.x) {
    const int64_t next = cta + gridDim.x;
    if (next < total_ctas) issue(next, ttile + (b ^ 1) * kTileElems);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const double* tile = ttile + b * kTileElems;
    int64_t tu, tv, sb, db;
    tile_bases(d, src_off, blk, cta, tu, tv, sb, db);
    const int64_t u0 = tu * kTileU, v0 = tv * kTileV;
    // store: threadIdx.x runs along v (unit output stride)
#pragma unroll
    for (int h = 0; h < kTileV / 32; ++h)
#pragma unroll
      for (int uu = threadIdx.y; uu < kTileU; uu += 8) {
        const int64_t u = u0 + uu, v = v0 + h * 32 + threadIdx.x;
        if (v < d.dv && u < d.du) dst[db + v + u * d.ou] = tile[uu * kTilePitch + h * 32 + threadIdx.x];
      }
    __syncthreads();  // buffer b is refilled by the next iteration's copies
    b ^= 1;
  }
}

// Narrow transpose: the row axis is short (dv <= 32), so the output of a tile
// (all rows x tu of axis q) is one contiguous run.  A tile spans all of axis 1 when it fits in shared memory
// (then its source rows are one contiguous slab too): rows are loaded by
// warps, coalesced along axis 1 (unit source stride), and the run is stored
// with consecutive threads on consecutive addresses.  The row pitch in shared
// memory is odd, so both phases are free of bank conflicts.
__global__ void k_permute_narrow(const double* __restrict__ src, double* __restrict__ dst,
                                 const int64_t* __restrict__ src_off, int64_t blk, TileDesc d, int tu,
                                 int64_t total_ctas) {
  extern __shared__ double ntile[];
  const int dv = static_cast<int>(d.dv);
  const int pitch = dv | 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // this thread's first output element of a run and the step per pass, as
  // (u, v) = divmod(i, dv), advanced without dividing again
  const int su = static_cast<int>(blockDim.x) / dv, sv = static_cast<int>(blockDim.x) % dv;
  const int iu = static_cast<int>(threadIdx.x) / dv, iv = static_cast<int>(threadIdx.x) % dv;
  for (int64_t cta = blockIdx.x; cta < total_ctas; cta += gridDim.x) {
    int64_t tiu, tiv, sb, db;
    tile_bases(d, src_off, blk, cta, tiu, tiv, sb, db);
    const int64_t u0 = tiu * tu;
    const int nu = static_cast<int>(d.du - u0 < tu ? d.du - u0 : tu);
    const double* sp = src + sb + u0;
    for (int v = warp; v < dv; v += nwarps) {
      const double* row = sp + row_src(d, v);
#pragma unroll 4
      for (int u = lane; u < nu; u += 32) ntile[u * pitch + v] = row[u];
    }
    __syncthreads();
    double* o = dst + db + u0 * dv;
    const int n = nu * dv;
    int u = iu, v = iv;
#pragma unroll 4
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      o[i] = ntile[u * pitch + v];
      u += su;
      v += sv;
      if (v >= dv) {
        v -= dv;
        ++u;
      }
    }
    __syncthreads();
  }
}

// ── variable-size block copies / permutes ─────────────────────────────────
__global__ void k_copy_blocks(const double* __restrict__ src, double* __restrict__ dst,
                              const BlockCopy* __restrict__ items, int64_t n) {
  for (int64_t b = blockIdx.y; b < n; b += gridDim.y) {
    const BlockCopy it = items[b];
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < it.len; e += (int64_t)gridDim.x * blockDim.x)
      dst[it.dst_off + e] = src[it.src_off + e];
  }
}

__global__ void k_perm_blocks(const double* __restrict__ src, double* __restrict__ dst,
                              const BlockPerm* __restrict__ items, int64_t n) {
  for (int64_t b = blockIdx.y; b < n; b += gridDim.y) {
    const BlockPerm& it = items[b];
    if (it.len < (int64_t{1} << 31)) {
      // a block below 2^31 elements: 32-bit index arithmetic (every extent and
      // coordinate of it fits), several times cheaper than 64-bit division
      for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e0 < it.len;
           e0 += (int64_t)gridDim.x * blockDim.x) {
        uint32_t e = static_cast<uint32_t>(e0);
        int64_t so = 0;
        bool in = true;
        for (int r = 0; r < it.rank; ++r) {
          const uint32_t d = static_cast<uint32_t>(it.out_dims[r]);
          const uint32_t c = e % d;
          e /= d;
          in = in && c < it.in_lim[r];
          so += static_cast<int64_t>(c) * it.in_strides[r];
        }
        dst[it.dst_off + e0] = in ? src[it.src_off + so] : 0.0;
      }
      continue;
    }
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e0 < it.len;
         e0 += (int64_t)gridDim.x * blockDim.x) {
      int64_t e = e0, so = 0;
      bool in = true;
      for (int r = 0; r < it.rank; ++r) {
        const int64_t c = e % it.out_dims[r];
        e /= it.out_dims[r];
        in = in && c < it.in_lim[r];
        so += c * it.in_strides[r];
      }
      dst[it.dst_off + e0] = in ? src[it.src_off + so] : 0.0;
    }
  }
}

// Rows of per-block permutes whose output axis 0 keeps unit source stride
// (zero padding, cropping, permutes of the outer axes): one warp per row of
// out_dims[0] elements, its source offset computed once; entries past the
// source limits are written as zeros.
__global__ void k_perm_block_rows(const double* __restrict__ src, double* __restrict__ dst,
                                  const BlockPerm* __restrict__ items, int64_t n) {
  const int lane = threadIdx.x & 31;
  const int64_t wpc = blockDim.x >> 5;
  for (int64_t b = blockIdx.y; b < n; b += gridDim.y) {
    const BlockPerm& it = items[b];
    const int64_t d0 = it.out_dims[0];
    const int64_t rows = it.len / d0;
    const int64_t lim0 = it.in_lim[0] < d0 ? it.in_lim[0] : d0;
    for (int64_t row = static_cast<int64_t>(blockIdx.x) * wpc + (threadIdx.x >> 5); row < rows;
         row += static_cast<int64_t>(gridDim.x) * wpc) {
      int64_t rr = row, so = 0;
      bool in = true;
      for (int r = 1; r < it.rank; ++r) {
        const int64_t c = rr % it.out_dims[r];
        rr /= it.out_dims[r];
        in = in && c < it.in_lim[r];
        so += c * it.in_strides[r];
      }
      const double* sp = src + it.src_off + so;
      double* o = dst + it.dst_off + row * d0;
      const int64_t lim = in ? lim0 : 0;
#pragma unroll 4
      for (int64_t e = lane; e < d0; e += 32) o[e] = e < lim ? sp[e] : 0.0;
    }
  }
}

__global__ void k_outside_nonzero(const double* __restrict__ src, const BlockPerm* __restrict__ items, int64_t n,
                                  uint8_t* __restrict__ flags) {
  for (int64_t b = blockIdx.x; b < n; b += gridDim.x) {
    const BlockPerm& it = items[b];
    int any = 0;
    for (int64_t e0 = threadIdx.x; e0 < it.len && !any; e0 += blockDim.x) {
      int64_t e = e0;
      bool in = true;
      for (int r = 0; r < it.rank; ++r) {
        const int64_t c = e % it.out_dims[r];
        e /= it.out_dims[r];
        in = in && c < it.in_lim[r];
      }
      any = !in && src[it.src_off + e0] != 0.0;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) flags[b] = any ? 1 : 0;
  }
}

// ── structure flags ───────────────────────────────────────────────────────
__global__ void k_slice_nonzero(const double* __restrict__ src, const int64_t* __restrict__ off,
                                int64_t nslices, int64_t chunk, uint8_t* __restrict__ flags,
                                int64_t nseg) {
  for (int64_t sgi = blockIdx.x; sgi < nseg; sgi += gridDim.x) {
    const int64_t b = sgi / nslices, s = sgi % nslices;
    const double* p = src + off[b] + s * chunk;
    int any = 0;
    for (int64_t t = threadIdx.x; t < chunk && !any; t += blockDim.x) any = (p[t] != 0.0);
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) flags[sgi] = any ? 1 : 0;
  }
}

__global__ void k_scaled_slice_nonzero(const double* __restrict__ src, const double* __restrict__ alpha,
                                       const int64_t* __restrict__ off, const int64_t* __restrict__ ai,
                                       int64_t n, int64_t chunk, uint8_t* __restrict__ flags) {
  for (int64_t q = blockIdx.x; q < n; q += gridDim.x) {
    const double a = alpha[ai[q]];
    const double* p = src + off[q];
    int any = 0;
    for (int64_t t = threadIdx.x; t < chunk && !any; t += blockDim.x) any = (__dmul_rn(a, p[t]) != 0.0);
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) flags[q] = any ? 1 : 0;
  }
}

__global__ void k_block_max_gt(const double* __restrict__ src, int64_t nblocks, int64_t blk, double tol,
                               uint8_t* __restrict__ flags) {
  __shared__ double red[kThreads];
  for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
    double m = 0.0;
    for (int64_t t = threadIdx.x; t < blk; t += blockDim.x) {
      const double a = fabs(src[b * blk + t]);
      if (a > m) m = a;  // NaN never compares greater, as in the reference loop
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s && red[threadIdx.x + s] > red[threadIdx.x]) red[threadIdx.x] = red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) flags[b] = red[0] > tol ? 1 : 0;
    __syncthreads();
  }
}

__global__ void k_elem_keep(const double* __restrict__ src, int64_t n, double atol, double rtol,
                            uint8_t* __restrict__ flags) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = fabs(src[i]);
    flags[i] = (a > atol + rtol * a) ? 1 : 0;
  }
}

__global__ void k_maxabs(const double* __restrict__ src, int64_t n, double* __restrict__ out) {
  __shared__ double red[kThreads];
  double m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(src[i]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// ── gathers / scatters ────────────────────────────────────────────────────
__global__ void k_gather(const double* __restrict__ src, const int64_t* __restrict__ idx, int64_t n,
                         double* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}
__global__ void k_scatter(const double* __restrict__ src, const int64_t* __restrict__ idx, int64_t n,
                          double* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[idx[i]] = src[i];
}
__global__ void k_scale_blocks(const double* __restrict__ src, const int64_t* __restrict__ toff,
                               const double* __restrict__ scal, int64_t nblocks, int64_t blk,
                               double* __restrict__ dst) {
  const int64_t total = nblocks * blk;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / blk, t = i - b * blk;
    dst[i] = __dmul_rn(scal[b], src[toff[b] + t]);
  }
}
__global__ void k_blocks_to_strided(const double* __restrict__ data, const int64_t* __restrict__ lin,
                                    int64_t nblocks, int64_t blk, int64_t stride, double* __restrict__ dense) {
  const int64_t total = nblocks * blk;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / blk, t = i - b * blk;
    dense[lin[b] + stride * t] = data[i];
  }
}

// ── scalar programs ───────────────────────────────────────────────────────
__global__ void k_scalar_prog(const double* __restrict__ sa, const double* __restrict__ sb,
                              const ScalarTerm* __restrict__ terms, const int32_t* __restrict__ seg,
                              int64_t nsegs, double* __restrict__ out) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < nsegs; g += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    bool first = true;
    for (int e = seg[g]; e < seg[g + 1]; ++e) {
      const ScalarTerm tm = terms[e];
      const double v = tm.ib >= 0 ? __dmul_rn(sa[tm.ia], sb[tm.ib]) : sa[tm.ia];
      acc = first ? v : __dadd_rn(acc, v);
      first = false;
    }
    out[g] = acc;
  }
}

}  // namespace

cudaError_t launch_outer_acc(const double* A, const double* B, double* C, const OuterCBlock* d_cb,
                             int64_t ncb, const OuterPair* d_pairs, int64_t max_elems, bool kahan,
                             cudaStream_t s) {
  if (ncb <= 0 || max_elems <= 0) return cudaSuccess;
  dim3 grid(grid_for(max_elems), static_cast<unsigned>(ncb < 65535 ? ncb : 65535));
  if ((int64_t)grid.x * grid.y > 148LL * 64) grid.x = static_cast<unsigned>(std::max<int64_t>(1, 148LL * 64 / grid.y));
  k_outer_acc<<<grid, kThreads, 0, s>>>(A, B, C, d_cb, ncb, d_pairs, kahan);
  return cudaGetLastError();
}

cudaError_t launch_axpy_seg(const double* src, const double* d_alpha, double* C, const AxpySeg* d_segs,
                            int64_t nsegs, const AxpyEntry* d_entries, int64_t max_len, cudaStream_t s) {
  if (nsegs <= 0 || max_len <= 0) return cudaSuccess;
  dim3 grid(grid_for(max_len), static_cast<unsigned>(nsegs < 65535 ? nsegs : 65535));
  if ((int64_t)grid.x * grid.y > 148LL * 64) grid.x = static_cast<unsigned>(std::max<int64_t>(1, 148LL * 64 / grid.y));
  k_axpy_seg<<<grid, kThreads, 0, s>>>(src, d_alpha, C, d_segs, nsegs, d_entries);
  return cudaGetLastError();
}

cudaError_t launch_permute_blocks(const double* src, double* dst, const int64_t* d_src_off, int64_t nblocks,
                                  int64_t blk, const PermDesc& desc, cudaStream_t s) {
  if (nblocks <= 0 || blk <= 0) return cudaSuccess;
  // Find the output axis with unit source stride (q) and decide the kernel.
  int q = -1;
  for (int r = 0; r < desc.rank; ++r)
    if (desc.in_strides[r] == 1 && desc.out_dims[r] > 1) { q = r; break; }
  const bool first_unit = desc.rank == 0 || desc.in_strides[0] == 1 || desc.out_dims[0] == 1;
  if (desc.rank > 0 && desc.in_strides[0] == 1) {
    // leading output axes contiguous in the source as well: one run
    int j = 1;
    int64_t len = desc.out_dims[0];
    while (j < desc.rank && desc.in_strides[j] == len) len *= desc.out_dims[j++];
    if (len >= 32) {
      const int64_t runs = blk / len, total = nblocks * runs;
      const int64_t ctas = std::min<int64_t>((total + 7) / 8, 148LL * 8);
      k_permute_runs<<<static_cast<unsigned>(std::max<int64_t>(ctas, 1)), kThreads, 0, s>>>(
          src, dst, d_src_off, blk, len, runs, total, desc, j);
      return cudaGetLastError();
    }
  }
  if (first_unit || q <= 0 || desc.out_dims[q] < 4) {
    k_permute_general<<<grid_for(nblocks * blk), kThreads, 0, s>>>(src, dst, d_src_off, nblocks, blk, desc);
    return cudaGetLastError();
  }
  TileDesc td{};
  td.du = desc.out_dims[q];
  td.nv = q;
  td.dv = 1;
  for (int r = 0; r < q; ++r) {
    td.vdims[r] = desc.out_dims[r];
    td.vsrc[r] = desc.in_strides[r];
    td.dv *= desc.out_dims[r];
  }
  td.ou = td.dv;
  int64_t ostride = td.dv * td.du;
  int nb = 0;
  for (int r = q + 1; r < desc.rank; ++r) {
    td.bdims[nb] = desc.out_dims[r];
    td.bsrc[nb] = desc.in_strides[r];
    td.bdst[nb] = ostride;
    ++nb;
    ostride *= desc.out_dims[r];
  }
  td.nb = nb;
  td.nbatch = 1;
  for (int r = 0; r < nb; ++r) td.nbatch *= td.bdims[r];
  if (td.dv <= 32) {
    // the widest tile (a multiple of 32 along axis q, or all of it) that fits
    const int pitch = static_cast<int>(td.dv) | 1;
    int64_t tu = kNarrowSmem / 8 / pitch;
    tu = td.du <= tu ? td.du : tu / 32 * 32;
    static std::atomic<bool> configured[64] = {};  // host threads may race on the first call
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!configured[dev & 63].load()) {
      e = cudaFuncSetAttribute(k_permute_narrow, cudaFuncAttributeMaxDynamicSharedMemorySize, kNarrowSmem);
      if (e != cudaSuccess) return e;
      configured[dev & 63].store(true);
    }
    td.tiles_u = (td.du + tu - 1) / tu;
    td.tiles_v = 1;
    const int64_t total = nblocks * td.nbatch * td.tiles_u;
    const unsigned g = static_cast<unsigned>(total < 148LL * 8 ? total : 148LL * 8);
    const size_t smem = static_cast<size_t>(tu) * pitch * sizeof(double);
    k_permute_narrow<<<g, kThreads, smem, s>>>(src, dst, d_src_off, blk, td, static_cast<int>(tu), total);
    return cudaGetLastError();
  }
  td.tiles_u = (td.du + kTileU - 1) / kTileU;
  td.tiles_v = (td.dv + kTileV - 1) / kTileV;
  const int64_t total = nblocks * td.nbatch * td.tiles_u * td.tiles_v;
  constexpr int smem = 2 * kTileElems * static_cast<int>(sizeof(double));
  static std::atomic<int> grid_of[64] = {};  // host threads may race on the first call
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int grid = grid_of[dev & 63].load();
  if (grid == 0) {
    e = cudaFuncSetAttribute(k_permute_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int sms = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_permute_tiled, 256, smem);
    if (e != cudaSuccess) return e;
    grid = sms * std::max(per_sm, 1);
    grid_of[dev & 63].store(grid);
  }
  const unsigned g = static_cast<unsigned>(total < grid ? total : grid);
  k_permute_tiled<<<g, dim3(32, 8), smem, s>>>(src, dst, d_src_off, blk, td, total);
  return cudaGetLastError();
}

cudaError_t launch_copy_blocks(const double* src, double* dst, const BlockCopy* d_items, int64_t n, int64_t max_len,
                               cudaStream_t s) {
  if (n <= 0 || max_len <= 0) return cudaSuccess;
  dim3 grid(grid_for(max_len), static_cast<unsigned>(n < 65535 ? n : 65535));
  if ((int64_t)grid.x * grid.y > 148LL * 64) grid.x = static_cast<unsigned>(std::max<int64_t>(1, 148LL * 64 / grid.y));
  k_copy_blocks<<<grid, kThreads, 0, s>>>(src, dst, d_items, n);
  return cudaGetLastError();
}

cudaError_t launch_perm_block_rows(const double* src, double* dst, const BlockPerm* d_items, int64_t n,
                                   int64_t max_rows, cudaStream_t s) {
  if (n <= 0 || max_rows <= 0) return cudaSuccess;
  const int64_t gy = n < 65535 ? n : 65535;
  int64_t gx = (max_rows + 7) / 8;  // eight warps per CTA
  gx = std::max<int64_t>(1, std::min<int64_t>(gx, 148LL * 16 / gy));
  k_perm_block_rows<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy)), kThreads, 0, s>>>(src, dst,
                                                                                                    d_items, n);
  return cudaGetLastError();
}

cudaError_t launch_perm_blocks(const double* src, double* dst, const BlockPerm* d_items, int64_t n, int64_t max_len,
                               cudaStream_t s) {
  if (n <= 0 || max_len <= 0) return cudaSuccess;
  dim3 grid(grid_for(max_len), static_cast<unsigned>(n < 65535 ? n : 65535));
  if ((int64_t)grid.x * grid.y > 148LL * 64) grid.x = static_cast<unsigned>(std::max<int64_t>(1, 148LL * 64 / grid.y));
  k_perm_blocks<<<grid, kThreads, 0, s>>>(src, dst, d_items, n);
  return cudaGetLastError();
}

// Smallest tail extents of every block that keep all its nonzero entries:
// ext[b*n2 + r] = 1 + the largest axis-r coordinate of a nonzero element
// (ext holds 1s on entry).  A block is a column-major matrix of d0 rows
// (axis 0) and cols columns (the other axes, flattened).  Work comes in warp
// tasks, task_begin[b] .. task_begin[b+1] for block b, in one of three forms
// fixed by (d0, cols) alone (ext_task_shape): rows of one column split into
// 8192-long segments (cols == 1); a run of columns, one at a time by the whole
// warp (d0 >= 32); 2048 columns, one lane per column (d0 < 32).  A column with
// a nonzero entry has its other coordinates decomposed once; the maxima go to
// ext with one atomicMax per axis and task.
__host__ __device__ inline int64_t ext_task_cols(int64_t d0, int64_t cols) {
  if (cols == 1) return 1;
  if (d0 < 32) return 2048;
  const int64_t per = 8192 / d0;
  return per < 1 ? 1 : per > 32 ? 32 : per;
}
__host__ __device__ inline int64_t ext_tasks(int64_t d0, int64_t cols) {
  if (d0 == 0 || cols == 0) return 0;
  if (cols == 1) return (d0 + 8191) / 8192;
  const int64_t per = ext_task_cols(d0, cols);
  return (cols + per - 1) / per;
}

__global__ void k_block_extents(const double* __restrict__ src, const int64_t* __restrict__ off,
                                const int64_t* __restrict__ dims, const int64_t* __restrict__ task_begin,
                                int64_t nblocks, int n2, int* __restrict__ ext) {
  const int lane = threadIdx.x & 31;
  const int64_t ntasks = task_begin[nblocks];
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < ntasks; w += warps) {
    int64_t lo = 0, hi = nblocks - 1;  // the last block with task_begin <= w
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (task_begin[mid] <= w) lo = mid; else hi = mid - 1;
    }
    const int64_t b = lo, t = w - task_begin[b];
    const int64_t* bd = dims + b * n2;
    const int64_t d0 = bd[0];
    int64_t cols = 1;
    for (int r = 1; r < n2; ++r) cols *= bd[r];
    const double* base = src + off[b];
    int64_t mrow = 0;
    int64_t mc[kMaxRank];
    for (int r = 1; r < n2; ++r) mc[r] = 0;
    auto note_col = [&](int64_t c) {
      int64_t q = c;
      for (int r = 1; r < n2; ++r) {
        const int64_t x = q % bd[r] + 1;
        q /= bd[r];
        mc[r] = x > mc[r] ? x : mc[r];
      }
    };
    if (cols == 1 || d0 >= 32) {
      const int64_t per = ext_task_cols(d0, cols);
      const int64_t c0 = cols == 1 ? 0 : t * per, c1 = cols == 1 ? 1 : (c0 + per < cols ? c0 + per : cols);
      const int64_t r0 = cols == 1 ? t * 8192 : 0, r1 = cols == 1 ? (r0 + 8192 < d0 ? r0 + 8192 : d0) : d0;
      for (int64_t c = c0; c < c1; ++c) {
        const double* col = base + c * d0;
        int64_t m = 0;
#pragma unroll 4
        for (int64_t r = r0 + lane; r < r1; r += 32)
          if (col[r] != 0.0) m = r + 1;
        if (__any_sync(0xffffffffu, m > 0)) {
          mrow = m > mrow ? m : mrow;
          note_col(c);
        }
      }
    } else {
      // one lane per column; the warp's 32 columns are one contiguous run
      const int64_t c0 = t * 2048, c1 = c0 + 2048 < cols ? c0 + 2048 : cols;
      for (int64_t c = c0 + lane; c < c1; c += 32) {
        const double* col = base + c * d0;
        int64_t m = 0;
        for (int64_t r = 0; r < d0; ++r)
          if (col[r] != 0.0) m = r + 1;
        if (m > 0) {
          mrow = m > mrow ? m : mrow;
          note_col(c);
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int64_t y = __shfl_xor_sync(0xffffffffu, mrow, o);
      mrow = y > mrow ? y : mrow;
      for (int r = 1; r < n2; ++r) {
        const int64_t z = __shfl_xor_sync(0xffffffffu, mc[r], o);
        mc[r] = z > mc[r] ? z : mc[r];
      }
    }
    if (lane == 0 && mrow > 0) {
      atomicMax(&ext[b * n2], static_cast<int>(mrow));
      for (int r = 1; r < n2; ++r) atomicMax(&ext[b * n2 + r], static_cast<int>(mc[r]));
    }
  }
}

int64_t block_extent_tasks(int64_t d0, int64_t cols) { return ext_tasks(d0, cols); }

cudaError_t launch_block_extents(const double* src, const int64_t* d_off, const int64_t* d_dims,
                                 const int64_t* d_task_begin, int64_t nblocks, int64_t ntasks, int n2, int* d_ext,
                                 cudaStream_t s) {
  if (ntasks <= 0 || nblocks <= 0) return cudaSuccess;
  if (n2 < 1 || n2 > kMaxRank) return cudaErrorInvalidValue;
  const int64_t ctas = std::min<int64_t>((ntasks + 7) / 8, 148LL * 8);
  k_block_extents<<<static_cast<unsigned>(ctas), kThreads, 0, s>>>(src, d_off, d_dims, d_task_begin, nblocks, n2,
                                                                    d_ext);
  return cudaGetLastError();
}

cudaError_t launch_outside_nonzero(const double* src, const BlockPerm* d_items, int64_t n, int64_t max_len,
                                   uint8_t* flags, cudaStream_t s) {
  (void)max_len;
  if (n <= 0) return cudaSuccess;
  const unsigned g = static_cast<unsigned>(n < 148LL * 32 ? n : 148LL * 32);
  k_outside_nonzero<<<g, 128, 0, s>>>(src, d_items, n, flags);
  return cudaGetLastError();
}

cudaError_t launch_slice_nonzero(const double* src, const int64_t* d_off, int64_t nblocks, int64_t nslices,
                                 int64_t chunk, uint8_t* flags, cudaStream_t s) {
  const int64_t nseg = nblocks * nslices;
  if (nseg <= 0) return cudaSuccess;
  const unsigned g = static_cast<unsigned>(nseg < 148LL * 32 ? nseg : 148LL * 32);
  k_slice_nonzero<<<g, 128, 0, s>>>(src, d_off, nslices, chunk, flags, nseg);
  return cudaGetLastError();
}

cudaError_t launch_scaled_slice_nonzero(const double* src, const double* alpha, const int64_t* d_off,
                                        const int64_t* d_ai, int64_t n, int64_t chunk, uint8_t* flags,
                                        cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const unsigned g = static_cast<unsigned>(n < 148LL * 32 ? n : 148LL * 32);
  k_scaled_slice_nonzero<<<g, 128, 0, s>>>(src, alpha, d_off, d_ai, n, chunk, flags);
  return cudaGetLastError();
}

cudaError_t launch_block_max_gt(const double* src, int64_t nblocks, int64_t blk, double tol, uint8_t* flags,
                                cudaStream_t s) {
  if (nblocks <= 0) return cudaSuccess;
  const unsigned g = static_cast<unsigned>(nblocks < 148LL * 32 ? nblocks : 148LL * 32);
  k_block_max_gt<<<g, kThreads, 0, s>>>(src, nblocks, blk, tol, flags);
  return cudaGetLastError();
}

cudaError_t launch_elem_keep(const double* src, int64_t n, double atol, double rtol, uint8_t* flags,
                             cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_elem_keep<<<grid_for(n), kThreads, 0, s>>>(src, n, atol, rtol, flags);
  return cudaGetLastError();
}

cudaError_t launch_maxabs(const double* src, int64_t n, double* d_out, cudaStream_t s) {
  k_maxabs<<<1, kThreads, 0, s>>>(src, n, d_out);
  return cudaGetLastError();
}

cudaError_t launch_gather(const double* src, const int64_t* d_idx, int64_t n, double* dst, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_gather<<<grid_for(n), kThreads, 0, s>>>(src, d_idx, n, dst);
  return cudaGetLastError();
}

cudaError_t launch_scatter(const double* src, const int64_t* d_idx, int64_t n, double* dst, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_scatter<<<grid_for(n), kThreads, 0, s>>>(src, d_idx, n, dst);
  return cudaGetLastError();
}

cudaError_t launch_scale_blocks(const double* src, const int64_t* d_tmpl_off, const double* d_scal,
                                int64_t nblocks, int64_t blk, double* dst, cudaStream_t s) {
  if (nblocks <= 0 || blk <= 0) return cudaSuccess;
  k_scale_blocks<<<grid_for(nblocks * blk), kThreads, 0, s>>>(src, d_tmpl_off, d_scal, nblocks, blk, dst);
  return cudaGetLastError();
}

cudaError_t launch_blocks_to_strided(const double* data, const int64_t* d_lin, int64_t nblocks, int64_t blk,
                                     int64_t stride, double* dense, cudaStream_t s) {
  if (nblocks <= 0 || blk <= 0) return cudaSuccess;
  k_blocks_to_strided<<<grid_for(nblocks * blk), kThreads, 0, s>>>(data, d_lin, nblocks, blk, stride, dense);
  return cudaGetLastError();
}

cudaError_t launch_scalar_prog(const double* sa, const double* sb, const ScalarTerm* d_terms,
                               const int32_t* d_seg_begin, int64_t nsegs, double* out, cudaStream_t s) {
  if (nsegs <= 0) return cudaSuccess;
  k_scalar_prog<<<grid_for(nsegs), kThreads, 0, s>>>(sa, sb, d_terms, d_seg_begin, nsegs, out);
  return cudaGetLastError();
}

}  // namespace sb
