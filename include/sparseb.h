/*
 * sparseb.h — C ABI of the B200 block-sparse contraction library (libsparseb.so).
 *
 * Drop-in for SparseBackends' tensor-algebra entry point
 *     SparseBackends.contract!(C, labelsC, A, labelsA, B, labelsB)
 *     (SparseBackends/src/tensoralgebra/contract.jl:37-104)
 * and the storage/conversion functions it relies on.  A Julia `ccall` shim
 * replaces the Julia kernels with these calls; Python reaches the same
 * symbols through ctypes (package sparsebackends_b200).
 *
 * Conventions (identical to the reference):
 *  - all tensors are FP64; dense payloads are column-major;
 *  - keys are 1-based integer tuples, one row of P (block-sparse/aliased) or N
 *    (COO) int64 values per entry;
 *  - block-sparse and aliased keys are kept sorted by the column-major linear
 *    index of the prefix; COO keys keep the order given (dirty flag as in the
 *    reference, sorted by sb_coo_sort);
 *  - a label is two uint64 values (Index id, prime level), so a label vector
 *    of rank n is 2*n uint64 values;
 *  - sb_contract overwrites C (keys, payload) exactly like the reference kernels.
 *
 * Threading: one sb_ctx per host thread.  Every call enqueues device work on
 * the context's stream; calls that must read device-computed structure flags
 * (value-dependent block creation) synchronise that stream internally.
 * No function allocates pinned host memory or blocks on other streams.
 */
#ifndef SPARSEB_H
#define SPARSEB_H

#include <stdint.h>

#if defined(__GNUC__)
#define SB_API __attribute__((visibility("default")))
#else
#define SB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sb_status {
  SB_OK = 0,
  SB_ERR_INVALID_ARG = 1,        /* bad pointer, rank, size or enum value                  */
  SB_ERR_DIM_MISMATCH = 2,       /* shared-label extents or block sizes disagree            */
  SB_ERR_LABEL = 3,              /* label missing / must be reduced / crosses prefix-tail   */
  SB_ERR_UNSUPPORTED_LAYOUT = 4, /* C dense tail interleaves A and B kept axes              */
  SB_ERR_UNSUPPORTED_TYPES = 5,  /* no kernel for this (C, A, B) storage combination        */
  SB_ERR_OOM = 6,                /* device allocation failed                                */
  SB_ERR_TIMEOUT = 7,            /* reserved: a bounded device wait gave up                 */
  SB_ERR_CUDA = 8,               /* CUDA runtime error (message in sb_last_error)           */
  SB_ERR_ASSERTION = 9           /* a precondition the reference asserts was violated      */
} sb_status;

typedef enum sb_kind {
  SB_KIND_DENSE = 0,
  SB_KIND_COO = 1,         /* COOTensor            (src/coo/storage.jl:1-6)              */
  SB_KIND_BLOCKSPARSE = 2, /* NewBlockSparseSorted (src/blocksparse/storage.jl:3-9)      */
  SB_KIND_ALIASED = 3      /* AliasedBlockSparse   (src/aliased/storage.jl:46-54)        */
} sb_kind;

typedef struct sb_ctx sb_ctx;
typedef struct sb_tensor sb_tensor;

/* ── context ─────────────────────────────────────────────────────────────── */
/* Creates a context on `device` with its own non-blocking stream.  Tensors
 * keep their context alive: destroying a context that still owns tensors
 * is deferred until the last of them is freed.                              */
SB_API sb_status sb_ctx_create(int device, unsigned flags, sb_ctx** out);
SB_API sb_status sb_ctx_destroy(sb_ctx* ctx);
/* Message of the last failing call on this context ("" if none).            */
SB_API const char* sb_last_error(const sb_ctx* ctx);
/* Use an external cudaStream_t (e.g. a Julia/torch stream) for all work.      */
SB_API sb_status sb_ctx_set_stream(sb_ctx* ctx, void* cuda_stream);
SB_API void* sb_ctx_get_stream(const sb_ctx* ctx);
SB_API sb_status sb_ctx_synchronize(sb_ctx* ctx);
/* Number of kernels this context has launched so far.                        */
SB_API int64_t sb_ctx_launch_count(const sb_ctx* ctx);
/* Arithmetic of the block GEMMs inside sb_contract (the per-pair mul! of
 * ta/contract_bs_bs.jl:716-723 and ta/contract_bs_dense.jl:576-611, which the
 * reference runs in FP64).  Tensors stay FP64 unless created with
 * sb_tensor_create_bs_f32.
 *   SB_PRECISION_F64    FP64 tensor-core (DMMA) GEMMs, the drop-in (default);
 *   SB_PRECISION_TF32X3 tcgen05 tensor cores: every operand value rounded
 *                       to FP32 and split into TF32 hi + lo, the three
 *                       significant products accumulated in FP32 chunks of
 *                       kc k-tiles that are then added in FP32 (a few 1e-7 to
 *                       a few 1e-6 relative per block);
 *   SB_PRECISION_TF32   tcgen05, one TF32 product (about 3e-4 relative).
 * Only the tiled GEMMs change; the K <= 16 (MPO) steps, outer products,
 * Kahan sums and axpys compute in FP64.  Operands must lie in FP32's range.
 * The split operand images of a contraction are kept with its plan and
 * remade after the library writes the operand tensor or hands out its device
 * pointer (sb_tensor_device_data); inside a captured graph they are remade on
 * every replay.  Not while a capture is open.  A bounded wait of the tensor-core
 * kernel that runs out is reported by the next sb_ctx_synchronize as
 * SB_ERR_TIMEOUT.                                                           */
typedef enum sb_precision {
  SB_PRECISION_F64 = 0,
  SB_PRECISION_TF32X3 = 1,
  SB_PRECISION_TF32 = 2
} sb_precision;
SB_API sb_status sb_ctx_set_precision(sb_ctx* ctx, int precision);
SB_API int sb_ctx_get_precision(const sb_ctx* ctx);
/* Per-launch kernel timing (CUDA events on the context stream), the
 * replacement of the reference's SB_TRACE stage timers
 * (ta/contract_bs_dense.jl:46-202).  Enabling clears earlier records.       */
SB_API sb_status sb_ctx_set_profiling(sb_ctx* ctx, int enable);
/* Totals for one kernel class since profiling was enabled:
 * kind 0 = tiled block GEMM (with its split-K reduction), 1 = permute,
 * 2 = outer-product accumulation, 3 = segmented axpy, 4 = other (QR/SVD,
 * gathers), 5 = vector-space operations, 6 = thin block GEMM (K <= 16),
 * 7 = tensor-core (tcgen05) block GEMM, 8 = packing of its operands (TF32
 * hi/lo split into the tensor core's shared-memory image layout).
 * Synchronises the context stream.                                           */
SB_API sb_status sb_ctx_profile_summary(sb_ctx* ctx, int kind, int64_t* launches, double* total_ms,
                                        double* flops, double* bytes);

/* ── tensor creation (host arrays are copied to the device) ──────────────── */
/* Dense tensor; data may be NULL (zeros).  Replaces the Array operands of
 * contract! (e.g. ta/contract_bs_dense.jl:411, B::AbstractArray).            */
SB_API sb_status sb_tensor_create_dense(sb_ctx* ctx, int nd, const int64_t* dims, const double* data,
                                 sb_tensor** out);
/* Same, from a device pointer (copied device-to-device).                     */
SB_API sb_status sb_tensor_create_dense_device(sb_ctx* ctx, int nd, const int64_t* dims,
                                        const double* d_data, sb_tensor** out);
/* NewBlockSparseSorted{T,N,N2}(dims, blksize, keys, ids, data)
 * (src/blocksparse/storage.jl:3-13).  keys: nblocks x P (row per block,
 * 1-based), need not be sorted but must be unique; ids: 1-based slot of each
 * key's payload in data (NULL means 1..nblocks); data: nblocks*blksize.
 * nblocks = 0 gives the empty tensor of NewBlockSparseSorted{T,N,N2}(dims)
 * (storage.jl:86-93).                                                        */
SB_API sb_status sb_tensor_create_bs(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail, int64_t nblocks,
                              const int64_t* keys, const int64_t* ids, const double* data,
                              sb_tensor** out);
/* Ragged block-sparse tensor: the reference's NewBlockSparseSorted
 * (src/blocksparse/storage.jl:3-9) extended with per-block tail extents, for
 * U(1)-graded links whose sectors differ in size (the reference pads every
 * block to the largest sector).  block_dims: nblocks x n_tail extents, each
 * in 1:dims of its tail axis; data: the blocks in the order of keys, each
 * column-major over its own extents.  Logically equal to the uniform tensor
 * obtained by zero padding (sb_tensor_to_uniform).                           */
SB_API sb_status sb_tensor_create_bs_ragged(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail,
                                            int64_t nblocks, const int64_t* keys, const int64_t* block_dims,
                                            const double* data, sb_tensor** out);
/* Empty block-sparse tensor with FP32 storage, to receive the result of
 * sb_contract in a tensor-core precision (SB_PRECISION_TF32X3 / _TF32): the
 * intermediates of a two-site H_eff chain (psi*L, *W1, *W2) kept in FP32 halve
 * the bytes of the memory-bound MPO steps.  Such tensors may be the output or
 * an operand of a multi-label block-sparse contraction (contract_shared!,
 * ta/contract_bs_bs.jl:572-730) only: as the long operand and result of a
 * K <= 16 step, or as either operand or result of a tensor-core GEMM step;
 * every other kernel rejects them with SB_ERR_UNSUPPORTED_TYPES.
 * sb_tensor_export_bs widens their values to FP64.  No counterpart in the
 * reference (FP64 throughout).                                              */
SB_API sb_status sb_tensor_create_bs_f32(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail, sb_tensor** out);
/* *f32 = 1 for FP32 storage (sb_tensor_create_bs_f32), else 0.              */
SB_API sb_status sb_tensor_storage_f32(const sb_tensor* t, int* f32);
/* *dense = 1 when every combination of the prefix axes has a block (a dense
 * tensor, or a block-sparse one with no prefix), else 0: `is_dense`
 * (src/blocksparse/storage.jl:413-425), which the wrappers use to return a plain
 * dense ITensor (src/tensor_wrappers.jl:389-427).  COO and aliased tensors:
 * SB_ERR_UNSUPPORTED_TYPES (the reference defines it for NewBlockSparseSorted). */
SB_API sb_status sb_tensor_is_dense(const sb_tensor* t, int* dense);
/* COOTensor{T,N}(dims, keys, vals, dirty) (src/coo/storage.jl:1-15).        */
SB_API sb_status sb_tensor_create_coo(sb_ctx* ctx, int nd, const int64_t* dims, int64_t nnz,
                               const int64_t* keys, const double* vals, int dirty, sb_tensor** out);
/* AliasedBlockSparse{T,N,N2,P}(dims, blksize, templates, n_templates, keys,
 * alias_ids, scalars) (src/aliased/storage.jl:46-59).                        */
SB_API sb_status sb_tensor_create_aliased(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail,
                                   int64_t n_templates, const double* templates, int64_t nblocks,
                                   const int64_t* keys, const int64_t* alias_ids,
                                   const double* scalars, sb_tensor** out);
SB_API sb_status sb_tensor_free(sb_tensor* t);

/* ── queries and export ──────────────────────────────────────────────────── */
/* dims must hold nd values (call with dims=NULL first to learn nd).          */
SB_API sb_status sb_tensor_info(const sb_tensor* t, int* kind, int* nd, int64_t* dims, int* n_tail,
                         int64_t* nkeys, int64_t* blksize, int64_t* n_templates, int* dirty);
/* Block-sparse export in the reference layout: keys sorted column-major,
 * ids = 1:n in that order, data packed accordingly.  Any pointer may be NULL. */
SB_API sb_status sb_tensor_export_bs(sb_ctx* ctx, const sb_tensor* t, int64_t* keys, int64_t* ids,
                              double* data);
/* sb_tensor_export_bs without the final synchronisation: keys and ids are
 * written at once, the payload copy is enqueued on the context stream and is
 * complete only after that stream reaches this point (sb_ctx_synchronize, or an
 * event the caller records).  With pinned `data` the copy overlaps work on
 * other streams, e.g. the next request of a serving loop.  No counterpart in
 * the reference (its export is a plain array read).                          */
SB_API sb_status sb_tensor_export_bs_async(sb_ctx* ctx, const sb_tensor* t, int64_t* keys, int64_t* ids, double* data);
SB_API sb_status sb_tensor_export_coo(sb_ctx* ctx, const sb_tensor* t, int64_t* keys, double* vals);
SB_API sb_status sb_tensor_export_aliased(sb_ctx* ctx, const sb_tensor* t, double* templates,
                                   int64_t* keys, int64_t* alias_ids, double* scalars);
SB_API sb_status sb_tensor_export_dense(sb_ctx* ctx, const sb_tensor* t, double* data);
/* Block layout: ragged flag, per-block tail extents (nkeys x n_tail, in key
 * order) and payload length in doubles.  Any pointer may be NULL.           */
SB_API sb_status sb_tensor_block_dims(const sb_tensor* t, int* ragged, int64_t* block_dims,
                                      int64_t* payload_len);
/* Ragged -> uniform by zero padding (the reference layout, for a Julia
 * caller), and uniform -> ragged by cropping each block to block_dims; with
 * check_zero, cropping a nonzero entry is an SB_ERR_ASSERTION.              */
SB_API sb_status sb_tensor_to_uniform(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out);
SB_API sb_status sb_tensor_to_ragged(sb_ctx* ctx, const sb_tensor* A, const int64_t* block_dims,
                                     int check_zero, sb_tensor** out);
/* Zero padding removed from the values: the ragged tensor whose blocks are
 * A's blocks cropped, axis by axis, to the smallest extents that keep every
 * nonzero entry (an all-zero block keeps extent 1).  For operands in the
 * reference's layout (src/blocksparse/storage.jl:3-9), where every U(1)
 * sector is zero-padded to the largest one, this recovers the sector extents
 * without the caller knowing them; contractions on the result equal those
 * of A up to rounding (sb_tensor_to_uniform pads a result back).  No
 * counterpart in the reference.  One device scan and one read-back.          */
SB_API sb_status sb_tensor_crop_padding(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out);
/* Device pointer and length (doubles) of the payload (dense data, block data,
 * COO values or aliased templates), for zero-copy interop.                   */
SB_API sb_status sb_tensor_device_data(const sb_tensor* t, double** d_ptr, int64_t* len);

/* ── operations ──────────────────────────────────────────────────────────── */
/* contract!(C, labelsC, A, labelsA, B, labelsB) (ta/contract.jl:37-104) with the
 * type-dispatched kernels of ta/contract_{coo,coo_dense,coo_bs,bs_bs,bs_dense}.jl
 * and ta/contract_aliased*.jl.  Supported (C, A, B) kinds:
 *   (COO, COO, COO)              contract_coo.jl:93-170          one label
 *   (BS, COO, DENSE)             contract_coo_dense.jl:48-125    one label
 *   (BS, COO, BS)                contract_coo_bs.jl:14-241       one label
 *   (BS, BS, BS)                 contract_bs_bs.jl:126-730       one or more labels
 *   (BS, BS, DENSE)              contract_bs_dense.jl:34-619     one or more labels
 *   (ALIASED, COO, DENSE)        contract_aliased_coo_dense.jl:34-164
 *   (ALIASED, ALIASED, DENSE)    contract_aliased.jl, contract_aliased_shared.jl
 *   (ALIASED, ALIASED, ALIASED)  contract_aliased.jl, contract_aliased_shared.jl
 *   (DENSE, BS, BS)              contract_bs_bs_to_dense! (contract_bs_bs.jl:736-754)
 * C must already have the output dims (and tail count); it is overwritten.   */
SB_API sb_status sb_contract(sb_ctx* ctx, sb_tensor* C, const uint64_t* labelsC, int nC,
                      const sb_tensor* A, const uint64_t* labelsA, int nA, const sb_tensor* B,
                      const uint64_t* labelsB, int nB);
/* permutedims for every kind (storage.jl:188-264, coo/storage.jl:153-166,
 * aliased/storage.jl:172-236); perm is 1-based.  Block-sparse/aliased perms
 * may not cross the prefix/tail boundary (storage.jl:126-132).               */
SB_API sb_status sb_permutedims(sb_ctx* ctx, const sb_tensor* A, const int* perm, sb_tensor** out);
/* sort_coo! (coo/storage.jl:182-189): column-major order, clears dirty.      */
SB_API sb_status sb_coo_sort(sb_ctx* ctx, sb_tensor* A);
/* blocksparse_from_dense(A, Val(N2); atol, rtol, dropzeros)
 * (src/blocksparse/conversions.jl:21-75).                                    */
SB_API sb_status sb_blocksparse_from_dense(sb_ctx* ctx, const sb_tensor* dense, int n_tail, double atol,
                                    double rtol, int dropzeros, sb_tensor** out);
/* coo_from_dense(A; atol, rtol) (src/coo/conversions.jl:13-26).              */
SB_API sb_status sb_coo_from_dense(sb_ctx* ctx, const sb_tensor* dense, double atol, double rtol,
                            sb_tensor** out);
/* to_dense for COO / block-sparse / aliased (coo/conversions.jl:4-10,
 * blocksparse/conversions.jl:83-187, aliased/conversions.jl:45-62).          */
SB_API sb_status sb_to_dense(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out);
/* to_blocksparse(::AliasedBlockSparse) (aliased/conversions.jl:18-32).       */
SB_API sb_status sb_aliased_to_blocksparse(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out);

/* ── CUDA graph capture of a sequence of calls ───────────────────────────────
 * No counterpart in the reference (its calls are Julia function calls).  For
 * repeated contractions with fixed block structure, e.g. the H_eff matvec of
 * every Lanczos step, the host planning and the launches of a sequence of
 * calls are captured once and replayed as one CUDA graph on the context
 * stream.  Rules:
 *  - run the sequence once before capturing, so every output tensor already
 *    has its storage (a capture that would leave new device buffers alive
 *    fails with SB_ERR_INVALID_ARG);
 *  - calls whose output structure depends on values read back from the GPU
 *    (dense_bb, dense_bd, dense_index, COO x COO, *_from_dense) and host
 *    readbacks (exports, norm, dot) cannot be captured: they fail and the
 *    capture is abandoned;
 *  - a replay recomputes the values of the captured outputs from the current
 *    contents of the captured inputs' device storage (same tensors, same
 *    structure); the host-side structure of the outputs is the one at capture.
 * Plan arrays the graph reads are device buffers owned by the graph.         */
typedef struct sb_graph sb_graph;
SB_API sb_status sb_ctx_capture_begin(sb_ctx* ctx);
SB_API sb_status sb_ctx_capture_end(sb_ctx* ctx, sb_graph** out);
SB_API sb_status sb_graph_launch(sb_ctx* ctx, const sb_graph* g);
SB_API sb_status sb_graph_free(sb_graph* g);

/* ── vector-space operations (Krylov solvers) ────────────────────────────────
 * The hooks KrylovKit's Lanczos needs from stored tensors
 * (SparseBackends/src/tensor_wrappers.jl:793-923; aliased variants
 * src/tensor_wrappers_aliased.jl:524-551).  All values stay on the device;
 * sb_tensor_dot and sb_tensor_norm synchronise the context stream to return
 * their scalar.  Reductions run in a fixed order (identical bits run to run). */

/* Elementwise ops of map!(f, R, R, A): R[i] = f(R[i], A[i]) over the stored
 * values by position (tensor_wrappers.jl:854-868), rounded as written.       */
typedef enum {
  SB_MAP_AXPY = 0,  /* r = r + alpha*a            */
  SB_MAP_AXPBY = 1, /* r = beta*r + alpha*a       */
  SB_MAP_COPY = 2,  /* r = a                      */
  SB_MAP_MUL = 3    /* r = r*a                    */
} sb_map_op;

/* LinearAlgebra.norm(w) (tensor_wrappers.jl:796-799): 2-norm of the stored
 * values; aliased: sqrt(sum_i sum_j (scalars[i]*template[alias_i][j])^2)
 * (tensor_wrappers_aliased.jl:524-536).                                      */
SB_API sb_status sb_tensor_norm(sb_ctx* ctx, const sb_tensor* A, double* out);
/* dot(x, y) = (dag(x) * y)[]: the full contraction of contract_bs_bs_to_dense!
 * with every label shared (ta/contract_bs_bs.jl:736-754) = sum over keys in
 * both operands of the block dot products.  Block-sparse x block-sparse
 * (uniform or ragged; equal extents per shared key) or dense x dense.        */
SB_API sb_status sb_tensor_dot(sb_ctx* ctx, const sb_tensor* A, const sb_tensor* B, double* out);
/* copy(w) (tensor_wrappers.jl:816-822): deep copy, any kind.                 */
SB_API sb_status sb_tensor_copy(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out);
/* similar(w) (tensor_wrappers.jl:897-918): same structure, zero values.      */
SB_API sb_status sb_tensor_similar(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out);
/* In-place scale, the value part of alpha * w (tensor_wrappers.jl:803-810):
 * stored values (aliased: the per-block scalars) multiplied by alpha.        */
SB_API sb_status sb_tensor_scale(sb_ctx* ctx, sb_tensor* A, double alpha);
/* fill!(w, x) (tensor_wrappers.jl:848-851): every stored value set to x
 * (block-sparse, COO, dense).                                                */
SB_API sb_status sb_tensor_fill(sb_ctx* ctx, sb_tensor* A, double x);
/* map!(f, R, R, A) for f in sb_map_op (tensor_wrappers.jl:854-868,
 * tensor_wrappers_aliased.jl:538-551 on the scalars).  Same kind and the same
 * number of stored values, else SB_ERR_DIM_MISMATCH ("Mismatched sparsity
 * patterns").                                                                */
SB_API sb_status sb_tensor_map(sb_ctx* ctx, sb_tensor* R, const sb_tensor* A, int op, double alpha, double beta);
/* x + y (tensor_wrappers.jl:825-838): union of block keys; a key in both gets
 * a + b.  Block-sparse + block-sparse (uniform or ragged) or dense + dense.  */
SB_API sb_status sb_tensor_add(sb_ctx* ctx, const sb_tensor* A, const sb_tensor* B, sb_tensor** out);

/* Axis fusion, axes 1-based.  Block-sparse: fuse_two_axes!
 * (src/blocksparse/conversions.jl:228-314): two prefix axes a1 < a2 fold into
 * a1 with key (k[a2]-1)*d[a1] + k[a1] (keys re-sorted); two tail axes fold
 * after moving the later one next to the earlier one (uniform tensors only);
 * mixed prefix/tail is SB_ERR_INVALID_ARG.  COO: fuse_axes_coo
 * (src/coo/conversions.jl:174-222): adjacent axes only (else
 * SB_ERR_ASSERTION), ax1 kept as the fast index, result sorted.              */
SB_API sb_status sb_fuse_axes(sb_ctx* ctx, const sb_tensor* A, int ax1, int ax2, sb_tensor** out);

/* ── block factorisations (src/ops_factorize.jl) ─────────────────────────────
 * Values on the device (Householder QR; batched one-sided Jacobi SVD); index
 * bookkeeping and the truncation decision on the host, as in the reference.  */

/* blocksparse_left_qr(A) (ops_factorize.jl:8-43) for A with prefix (l, r) and
 * dense tail (s) (N = 3, n_tail = 1, uniform).  M[(li-1)*d_s + s, ri] =
 * A[l_vals[li], r_vals[ri]][s] over the sorted distinct l and r values of the
 * keys; thin QR M = Q R, k = min(n_l*d_s, n_r), Householder reflectors with
 * LAPACK's sign convention.  *Q: block-sparse, dims (dims[0], d_s, k), prefix
 * (l), one block per l value (d_s x k); *R: dense k x n_r.  l_vals (capacity
 * dims[0]) and r_vals (capacity dims[1]) receive the distinct values when not
 * NULL; their counts go to *n_l and *n_r.                                    */
SB_API sb_status sb_blocksparse_left_qr(sb_ctx* ctx, const sb_tensor* A, sb_tensor** Q, sb_tensor** R,
                                        int64_t* l_vals, int64_t* n_l, int64_t* r_vals, int64_t* n_r);
/* blocksparse_svd(A; ortho, maxdim, mindim, cutoff) (ops_factorize.jl:50-148)
 * for A with prefix (L, R) and dense tail (s1, s2) (N = 4, n_tail = 2,
 * uniform, s1 <= 32).  One SVD per L group of d_s1 x (n_R(L)*d_s2), global
 * truncation: keep min(maxdim, total), then drop the smallest while the count
 * is above mindim and sv < cutoff * max sv.  *U: dims (dims[0], new_bond,
 * d_s1), prefix (L, b); *SV: dims (new_bond, dims[1], d_s2), prefix (b, R);
 * the singular values go to U when ortho_right, to SV otherwise.  svs gets
 * the kept singular values in bond order (min(capacity, *n_kept) of them;
 * dims[0]*d_s1 always suffices); *truncerr = sum of the dropped sv^2 (the
 * Spectrum of the reference is (svs.^2, truncerr)).                          */
SB_API sb_status sb_blocksparse_svd(sb_ctx* ctx, const sb_tensor* A, int ortho_right, int64_t maxdim,
                                    int64_t mindim, double cutoff, sb_tensor** U, sb_tensor** SV, double* svs,
                                    int64_t svs_capacity, int64_t* n_kept, double* truncerr);

/* ── allocation-free grouped block GEMM ──────────────────────────────────────
 * No counterpart in the reference: an extra entry point of this library.
 *
 * For callers that cannot allocate device memory during a solve (a fixed
 * memory budget or pre-sized pool, or a host runtime that forbids cudaMalloc
 * while it owns the device): runs the block GEMM that sb_contract uses,
 *     C[c_off[c] + i + j*c_rows[c]] = sum_{p in [c_pair_begin[c], c_pair_begin[c+1])} X_p(i,:) . Y_p(:,j)
 * with X_p at d_X + x_off[p] (element (i,k) at i + k*ldx[p], or k + i*ldx[p]
 * when x_trans) and Y_p at d_Y + y_off[p] (element (k,j) at k + j*ldy[p], or
 * j + k*ldy[p] when y_trans), K[p] the reduced extent.  Every C block is
 * written exactly once (no accumulation into prior C contents).
 * The caller passes device pointers for inputs and outputs and the plan in
 * host arrays; the function calls no cudaMalloc/cudaFree or any allocating
 * routine: the plan is copied into a static device array of 672 KiB that
 * every GPU loading the library holds until exit.
 * Limits: n_cblocks <= 4096 and c_pair_begin[n_cblocks] <= 16384; larger
 * plans are rejected with SB_ERR_INVALID_ARG and a message in err (if given).
 * The first call on a device resolves the array's device address (set-up).
 * A call on a stream that is capturing is rejected (SB_ERR_INVALID_ARG): the
 * plan is copied from host memory at call time.  Negative offsets and
 * leading dimensions below a block's contiguous extent are rejected too.
 * All calls share the array: calls that overlap on the GPU (e.g. on
 * different streams) race.                                                   */
SB_API sb_status sb_block_gemm_f64_noalloc(void* stream, const double* d_X, const double* d_Y, double* d_C,
                                           int32_t n_cblocks, const int64_t* c_off, const int32_t* c_rows,
                                           const int32_t* c_cols, const int32_t* c_pair_begin,
                                           const int64_t* x_off, const int64_t* y_off, const int32_t* K,
                                           const int32_t* ldx, const int32_t* ldy, int x_trans, int y_trans,
                                           char* err, int32_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* SPARSEB_H */
