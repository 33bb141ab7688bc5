// Device kernel launchers for the block-sparse contraction engine (sm_100a).
//
// Every launcher enqueues work on the given stream and returns immediately.
// Offsets are in elements (doubles) relative to the base pointers passed.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sb {

// ── grouped FP64 GEMM with segmented accumulation ──────────────────────────
//
// For every C block c:  C_c = sum_{p in [pair_begin_c, pair_end_c)} X_p * Y_p
// where X_p is M_c x K_p and Y_p is K_p x N_c, C_c is column-major M_c x N_c
// (leading dimension M_c).  X is read "N" (element (i,k) at x + i + k*ldx) or
// "T" (element (i,k) at x + k + i*ldx); Y likewise ((k,j) at y + k + j*ldy or
// y + j + k*ldy).  Each C tile is produced by exactly one CTA: no atomics, C
// is written once (no zero-init needed), accumulation order over pairs is the
// pair order.
// Tiles of C block c are CTAs [tile_begin, tile_begin + mtiles*ntiles); the
// kernel finds its C block by binary search over tile_begin, so no per-tile
// descriptor list is built or uploaded.
// ldc: column stride of the C block in C.  It equals M except for the edge
// sub-blocks of launch_gemm_f64_edges (a row range of a larger block); the
// thin kernels with small rows (small_rows) require ldc == M.  tshape: tile shape of the block in
// launch_gemm_f64_edges (0 = 64x64, 1 = 64x32, 2 = 32x64, 3 = 64x48,
// 4 = 48x64), else 0.
struct GemmCBlock {
  int64_t c_off;
  int32_t M, N;
  int32_t pair_begin, pair_end;
  int32_t tile_begin, mtiles;
  int32_t ldc, tshape;
};
struct GemmPair {
  int64_t x_off, y_off;
  int32_t K, ldx, ldy, pad;
};

// CTA tile shapes with 32x32 warp tiles, k-tile 16, 3 stages, plus T64x32.
// Measured on the H_eff steps (chi = 2048): 32x64 / 64x32 warp tiles need
// 190-250 registers, halve the resident CTAs and run 4-16% slower; 4 stages,
// k-tile 32 and eight 32x16 warps run 0-18% slower on the psi*L step.
// T64x32: four 32x16 warps, 4 stages, used for the few-tile, long-K launches
// that otherwise go to split-K (H_eff R*T3: 2.17 against 2.26 ms).
enum class GemmShape : int { T64x64 = 0, T128x32 = 1, T32x128 = 2, T128x64 = 3, T64x128 = 4, T64x32 = 5 };

// splitk > 1: the concatenated K range of every C tile is cut into splitk
// segments computed by separate CTAs into partial (splitk * ntiles * BM*BN
// doubles), then summed in segment order by a second kernel (deterministic).
cudaError_t launch_gemm_f64(const double* X, const double* Y, double* C,
                            const GemmCBlock* d_cblocks, int32_t ncblocks, const GemmPair* d_pairs,
                            int64_t ntiles, bool xT, bool yT, GemmShape shape, cudaStream_t s,
                            int splitk = 1, double* partial = nullptr);

// Tiled GEMM over C sub-blocks of five tile shapes in one launch: each
// GemmCBlock's tshape gives its tile (0 = 64x64; 1 = 64x32 and 3 = 64x48 for
// column edges of width <= 32 and <= 48; 2 = 32x64 and 4 = 48x64 for row
// edges of height <= 32 and <= 48); tiles are
// numbered through tile_begin / mtiles of that shape.  Sub-blocks carry their
// own ldc and pairs whose offsets start at the sub-block's first row and
// column.  splitk > 1: partial holds splitk * ntiles * 4096 doubles.
cudaError_t launch_gemm_f64_edges(const double* X, const double* Y, double* C, const GemmCBlock* d_cblocks,
                                  int32_t ncblocks, const GemmPair* d_pairs, int64_t ntiles, bool xT, bool yT,
                                  cudaStream_t s, int splitk = 1, double* partial = nullptr);

// Thin variant for launches whose every pair has K <= 16 and whose C blocks
// have min(M, N) <= 16 (HBM-bound): DMMA on 128 x 16 strips of the long side,
// cp.async double buffering across pairs.  Strips of C block c:
// [tile_begin, tile_begin + ceil(long/128)) when mtiles == 1; a group of S
// consecutive blocks with equal long extent, each carrying the group's
// tile_begin and mtiles = S, takes strips in turn (strip s of member j is
// tile_begin + s*S + j).  persistent: a
// grid of 5 CTAs per SM walks the strips with the copy pipeline running
// across strip boundaries and stores C from the fragments (needs >= 1 pair
// per C block); otherwise one CTA per strip with shared-memory staged stores.
// long_f32: the long operand (Y when small_rows, else X) and C hold FP32
// values (the intermediates of the tensor-core H_eff chain); the small
// operand stays FP64 and the arithmetic FP64.  Persistent kernel only.
cudaError_t launch_gemm_f64_skinny(const double* X, const double* Y, double* C,
                                   const GemmCBlock* d_cblocks, int32_t ncblocks, const GemmPair* d_pairs,
                                   int64_t nctas, bool xT, bool yT, bool small_rows, int small_max,
                                   int k_max, cudaStream_t s, bool persistent = false, bool long_f32 = false);

// Number of tiles of a (M, N) C block for the given tile shape.
void gemm_tile_dims(GemmShape shape, int* bm, int* bn);

// ── the same grouped GEMM on the tcgen05 tensor cores (sb_gemm_tc.cu) ─────
//
// FP32 operands (X, Y: element offsets as in GemmPair), arithmetic in TF32
// with FP32 accumulation, result FP64 (c_f64) or FP32.  passes = 3 splits
// every operand into TF32 hi + lo parts and sums a_hi*b_lo + a_lo*b_hi +
// a_hi*b_hi (about 22 significant bits per operand), passes = 1 multiplies
// the TF32-rounded operands once.
// Work items are listed explicitly: item i covers rows [a0, a0 + 128) of the
// A side and [b0, b0 + nb) of the B side of C block cb (nb a multiple of 16
// in 16..256), and nkt k-tiles (32 deep) of its C block's concatenated pair
// K ranges starting at pair p0, offset k0 (a multiple of 32).  Without swap
// the A side is X (rows of C) and the B side Y (columns of C); with swap the
// other way round.  An item with part < 0 covers the whole K range and
// writes C; part >= 0 marks a k-segment of a split tile, written in FP64 to
// partial tile `part` (column-major 128 x 256 doubles) and summed in segment
// order into C by the reduction that follows (one TcSplit per split tile:
// its geometry and its parts [part0, part0 + nparts)).  Items [nz_begin,
// ntiles) belong to C blocks without pairs and are written as zeros.  Within
// an item the k-tiles accumulate in FP32 chunks of kc k-tiles (the tensor
// core's accumulation error grows with the chunk length) whose sum is formed
// in FP32 with round-to-nearest adds.  fold must be set when an item has
// more than kc k-tiles (one accumulator and the running sum in TMEM; without
// it two accumulators alternate and every item is one chunk).  A persistent grid of one CTA per SM walks the list
// with stride gridDim.x, so the list order (the host sorts by work) balances
// the load.  *d_status is set to 1 if a bounded wait on the tensor core ran
// out (the results are then invalid).
struct TcTile {
  int32_t cb, a0, b0, nb;
  int32_t p0, k0, nkt, part;
};
struct TcSplit {
  int32_t cb, a0, b0, nb;
  int32_t part0, nparts, pad0, pad1;
};
constexpr int kTcMaxN = 256;
constexpr int64_t kTcPartElems = 128 * kTcMaxN;  // doubles of one partial tile
// Operands arrive packed (launch_tc_pack): per pair p, packs[p] locates the
// images of its A-side block (a_base: 128-row tiles, nkt k-tiles each, 32 KB
// per k-tile: hi plane then lo plane) and of its B-side block (b_base: tiles
// of nbs rows, 2*nbs*128 bytes per k-tile); item rows a0 and b0 select the
// tile (a0 / 128, b0 / nbs).
struct TcPack {
  int64_t a_base, b_base;
  int32_t nkt, nbs;
};
cudaError_t launch_gemm_tc(const void* pack_a, const void* pack_b, void* C, bool c_f64, const GemmCBlock* d_cblocks,
                           const GemmPair* d_pairs, const TcPack* d_packs, const TcTile* d_tiles, int32_t ntiles,
                           int32_t nz_begin, bool swap, int passes, int kc, bool fold, double* d_partial,
                           const TcSplit* d_splits, int32_t nsplits, int* d_status, cudaStream_t s);
// One packed k-tile image of one operand tile: rows [0, rows) x k [0, kv)
// (element (r, k) at src + r*ld + k when kc, else src + r + k*ld; elements of
// the FP64 or FP32 operand array), zero elsewhere, written at byte dst as the
// hi plane and (passes = 3) the lo plane plane bytes further; plane = image
// rows x 128 bytes in the K-major 128-byte-swizzled layout the tensor core
// reads.
struct TcImage {
  int64_t src, ld, dst;
  int32_t rows, kv, plane, kc;
};
cudaError_t launch_tc_pack(const void* src, bool src_f64, const TcImage* d_imgs, int64_t nimg, void* dst, int passes,
                           cudaStream_t s);

// ── outer-product accumulation (K = 1 pairs) on CUDA cores ─────────────────
//
// For every C block c: C_c[i + j*M] = sum_p a_p[i] * b_p[j] in pair order, with
// the reference's rounding (c = c + a*b, no fusion) or Kahan compensation.
struct OuterCBlock {
  int64_t c_off;
  int32_t M, N;
  int32_t pair_begin, pair_end;
};
struct OuterPair {
  int64_t a_off, b_off;
};
cudaError_t launch_outer_acc(const double* Abase, const double* Bbase, double* C,
                             const OuterCBlock* d_cblocks, int64_t ncblocks,
                             const OuterPair* d_pairs, int64_t max_elems, bool kahan,
                             cudaStream_t s);

// ── segmented scaled accumulation (axpy) ───────────────────────────────────
//
// For every segment g: C[c_off_g + t] = sum_{e in seg g} alpha_e * src[src_off_e + t]
// for t < len_g, rounding as c = c + alpha*src (alpha from d_alpha[alpha_idx_e],
// or 1.0 when alpha_idx_e < 0).
struct AxpySeg {
  int64_t c_off;
  int64_t len;
  int32_t e_begin, e_end;
};
struct AxpyEntry {
  int64_t src_off;
  int64_t alpha_idx;
};
cudaError_t launch_axpy_seg(const double* src, const double* d_alpha, double* C,
                            const AxpySeg* d_segs, int64_t nsegs, const AxpyEntry* d_entries,
                            int64_t max_len, cudaStream_t s);

// ── permutes ───────────────────────────────────────────────────────────────
//
// dst block b (packed at b*blk) = tail-permute of src block at src_off[b].
// out_dims[r]: output tail dims (fastest first); in_strides[r]: stride in the
// source block of output axis r.
constexpr int kMaxRank = 12;
struct PermDesc {
  int rank;
  int64_t out_dims[kMaxRank];
  int64_t in_strides[kMaxRank];
};
cudaError_t launch_permute_blocks(const double* src, double* dst, const int64_t* d_src_off,
                                  int64_t nblocks, int64_t blk, const PermDesc& desc,
                                  cudaStream_t s);

// Variable-size block copy: dst[dst_off[i] + e] = src[src_off[i] + e] for e < len[i].
struct BlockCopy {
  int64_t src_off, dst_off, len;
};
cudaError_t launch_copy_blocks(const double* src, double* dst, const BlockCopy* d_items, int64_t n,
                               int64_t max_len, cudaStream_t s);
// Per-block tail permute / pad / crop: output block i (dst_off, out_dims) element
// e reads src[src_off + sum_r c_r * in_strides[r]] when every coordinate c_r is
// below in_lim[r], and writes 0 otherwise (zero padding).
struct BlockPerm {
  int64_t src_off, dst_off, len;
  int rank;
  int64_t out_dims[kMaxRank];
  int64_t in_strides[kMaxRank];
  int64_t in_lim[kMaxRank];
};
cudaError_t launch_perm_blocks(const double* src, double* dst, const BlockPerm* d_items, int64_t n,
                               int64_t max_len, cudaStream_t s);
// The same for items whose out_dims[0] has in_strides[0] == 1 (one warp per
// row of out_dims[0]); max_rows = the largest len / out_dims[0].
cudaError_t launch_perm_block_rows(const double* src, double* dst, const BlockPerm* d_items, int64_t n,
                                   int64_t max_rows, cudaStream_t s);
// ext[b*n2 + r] = smallest axis-r extent of block b (payload at d_off[b],
// extents d_dims[b*n2 ..]) that keeps all its nonzero entries (>= 1; d_ext
// holds 1s on entry).  The scan runs in warp tasks: block b has
// block_extent_tasks(d0, cols) of them (d0 = its first extent, cols = the
// product of the others), starting at d_task_begin[b]; d_task_begin has
// nblocks + 1 entries, the last = ntasks.
int64_t block_extent_tasks(int64_t d0, int64_t cols);
cudaError_t launch_block_extents(const double* src, const int64_t* d_off, const int64_t* d_dims,
                                 const int64_t* d_task_begin, int64_t nblocks, int64_t ntasks, int n2, int* d_ext,
                                 cudaStream_t s);
// flags[i] = 1 if block i of src holds a nonzero outside its box in_lim
// (used to check that cropping a padded block loses nothing).
cudaError_t launch_outside_nonzero(const double* src, const BlockPerm* d_items, int64_t n, int64_t max_len,
                                   uint8_t* flags, cudaStream_t s);

// ── value-dependent structure helpers ──────────────────────────────────────
// flags[b*nslices + s] = any(src[off_b + s*chunk + t] != 0, t < chunk)
cudaError_t launch_slice_nonzero(const double* src, const int64_t* d_off, int64_t nblocks,
                                 int64_t nslices, int64_t chunk, uint8_t* flags, cudaStream_t s);
// flags[q] = any(alpha[ai_q] * src[off_q + t] != 0, t < chunk)
cudaError_t launch_scaled_slice_nonzero(const double* src, const double* alpha,
                                        const int64_t* d_off, const int64_t* d_ai, int64_t n,
                                        int64_t chunk, uint8_t* flags, cudaStream_t s);
// flags[b] = max_t |src[b*blk + t]| > tol
cudaError_t launch_block_max_gt(const double* src, int64_t nblocks, int64_t blk, double tol,
                                uint8_t* flags, cudaStream_t s);
// flags[i] = |src[i]| > atol + rtol*|src[i]|
cudaError_t launch_elem_keep(const double* src, int64_t n, double atol, double rtol,
                             uint8_t* flags, cudaStream_t s);
// max |src[i]| into *d_out (single value)
cudaError_t launch_maxabs(const double* src, int64_t n, double* d_out, cudaStream_t s);

// ── gathers / scatters ─────────────────────────────────────────────────────
cudaError_t launch_gather(const double* src, const int64_t* d_idx, int64_t n, double* dst,
                          cudaStream_t s);
cudaError_t launch_scatter(const double* src, const int64_t* d_idx, int64_t n, double* dst,
                           cudaStream_t s);
// dst[b*blk + t] = scal[b] * src[tmpl_off[b] + t]
cudaError_t launch_scale_blocks(const double* src, const int64_t* d_tmpl_off,
                                const double* d_scal, int64_t nblocks, int64_t blk,
                                double* dst, cudaStream_t s);
// dense[lin_b + stride*t] = data[b*blk + t]
cudaError_t launch_blocks_to_strided(const double* data, const int64_t* d_lin, int64_t nblocks,
                                     int64_t blk, int64_t stride, double* dense, cudaStream_t s);

// ── vector-space operations (Krylov solvers) ───────────────────────────────
// Dot product over chunks of at most kDotChunk elements: *d_out = sum over
// chunks of sum_t (s*X[x_off+t]) * (s*Y[y_off+t]) with s = S[s_idx] (s = 1
// when s_idx < 0); d_partial holds nchunks doubles.  Fixed reduction order:
// identical bits on every call.
constexpr int kDotChunk = 1024;  // 4 elements per thread of a 256-thread CTA
struct DotChunk {
  int64_t x_off, y_off;
  int64_t s_idx;
  int32_t len, pad;
};
cudaError_t launch_dot_chunks(const double* X, const double* Y, const double* S, const DotChunk* d_chunks,
                              int64_t nchunks, double* d_partial, double* d_out, cudaStream_t s);
// Elementwise R[i] = f(R[i], A[i]) for i < n.
enum MapOp : int { kMapAxpy = 0, kMapAxpby = 1, kMapCopy = 2, kMapMul = 3, kMapScale = 4, kMapFill = 5 };
cudaError_t launch_map(double* R, const double* A, int64_t n, int op, double alpha, double beta, cudaStream_t s);
// Key-union add: C[c_off + e] = A-block, 0 + B-block, or A-block + B-block
// (a_off / b_off < 0 marks a missing operand block).
struct AddBlock {
  int64_t a_off, b_off, c_off, len;
};
cudaError_t launch_add_blocks(const double* A, const double* B, double* C, const AddBlock* d_items, int64_t n,
                              int64_t max_len, cudaStream_t s);

// ── block factorisations (QR, SVD truncation) ──────────────────────────────
// In-place Householder QR of the column-major m x n matrix M (LAPACK dlarfg
// convention): R in the upper triangle, reflector j below the diagonal of
// column j with scale tau[j]; *launches counts the kernels issued.
cudaError_t launch_householder_qr(double* M, int64_t m, int64_t n, double* tau, cudaStream_t s, int64_t* launches);
// Thin Q (m x k, column-major) from the reflectors in M.
cudaError_t launch_householder_form_q(const double* M, int64_t m, int64_t k, const double* tau, double* Q,
                                      cudaStream_t s, int64_t* launches);
// R (k x n, column-major) = upper triangle of the first k rows of M.
cudaError_t launch_upper(const double* M, int64_t m, int64_t k, int64_t n, double* R, cudaStream_t s);
// Strided 2-D copies: dst[dst_off + r*dst_rs + c*dst_cs] = src[src_off + r*src_rs + c*src_cs]
// (times scale[s_idx] when s_idx >= 0) for r < rows, c < cols.
struct Gather2D {
  int64_t src_off, dst_off, rows, cols, src_rs, src_cs, dst_rs, dst_cs, s_idx;
};
cudaError_t launch_gather_2d(const double* src, double* dst, const double* scale, const Gather2D* d_items, int64_t n,
                             int64_t max_elems, cudaStream_t s);
// One-sided Jacobi SVD of row-major m x n matrices (m <= kSvdMaxRows) at
// A + a_off: on return Vt + a_off holds the right singular vectors as rows,
// U + u_off the left ones (column-major m x m) and S + s_off the m singular
// values, all sorted by decreasing singular value.  A is overwritten.
// *d_status is set to 1 when some matrix has not converged in max_sweeps.
constexpr int kSvdMaxRows = 32;
struct SvdGroup {
  int64_t a_off;
  int64_t n;
  int64_t u_off, s_off;
  int32_t m, pad;
};
cudaError_t launch_svd_rows(double* A, double* Vt, double* U, double* S, const SvdGroup* d_groups, int64_t ngroups,
                            int max_sweeps, int* d_status, cudaStream_t s);

// ── scalar programs (aliased bookkeeping) ──────────────────────────────────
// out[g] = sum_{e in seg g} (sa[ia_e] * (ib_e >= 0 ? sb[ib_e] : 1)), left to right.
struct ScalarTerm {
  int64_t ia, ib;
};
cudaError_t launch_scalar_prog(const double* sa, const double* sb, const ScalarTerm* d_terms,
                               const int32_t* d_seg_begin, int64_t nsegs, double* out,
                               cudaStream_t s);

}  // namespace sb
