// Host-side data structures of libsparseb: context, device buffers, tensors.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <unordered_map>
#include <vector>

#include "../../include/sparseb.h"
#include "sb_kernels.hpp"

namespace sb {

struct Error : std::runtime_error {
  sb_status code;
  Error(sb_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(sb_status c, const std::string& m) { throw Error(c, m); }
inline void require(bool cond, sb_status c, const std::string& m) {
  if (!cond) fail(c, m);
}
void check_cuda(cudaError_t e, const char* what);
#define SB_CK(x) ::sb::check_cuda((x), #x)

struct Ctx;

// Stream-ordered device buffer of doubles (or raw bytes), freed on the
// owning context's stream.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(Ctx* ctx, size_t bytes);
  ~DevBuf();
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept;
  void reset();
  void* raw() const { return p_; }
  double* d() const { return static_cast<double*>(p_); }
  template <class T>
  T* as() const { return static_cast<T*>(p_); }
  size_t bytes() const { return n_; }

 private:
  Ctx* ctx_ = nullptr;
  void* p_ = nullptr;
  size_t n_ = 0;
  bool plain_ = false;  // cudaMalloc'd (allocated while a capture was open) instead of stream-ordered
};

// Kernel classes reported by the in-library profiler.
enum ProfKind : int {
  PROF_GEMM = 0, PROF_PERMUTE = 1, PROF_OUTER = 2, PROF_AXPY = 3, PROF_OTHER = 4, PROF_VECTOR = 5,
  PROF_GEMM_THIN = 6, PROF_GEMM_TC = 7, PROF_TC_PACK = 8, PROF_NKINDS = 9
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  int64_t launches = 0;
  // Optional per-launch timing: a pair of CUDA events on the context stream
  // around every kernel, with the launch's algorithmic FLOPs and bytes.
  struct ProfRec {
    int kind;
    cudaEvent_t a, b;
    double flops, bytes;
  };
  bool profiling = false;
  std::vector<ProfRec> prof;
  // SPARSEB_TRACE=1 (read once at context creation): one line per contract!
  // call on stderr with the kernel chosen, block counts and host time.
  bool trace = false;
  const char* kernel_name = "";
  // The last GEMM variant a contraction launched (e.g. "tiled 64x64 sk1"), for the trace line.
  char gemm_desc[96] = "";
  // SPARSEB_GEMM_TILE=<BM>x<BN> forces one GEMM tile shape (tuning); -1 = auto.
  int gemm_tile = -1;
  // SPARSEB_GEMM_SPLITK=<n> forces the split-K factor (tuning); 0 = auto.
  int gemm_splitk = 0;
  // SPARSEB_GEMM_THIN=0 keeps K<=16 launches on the tiled kernel, =1 uses the
  // one-CTA-per-strip thin kernel (tuning); -1 = auto: the persistent thin
  // kernel for every launch it can serve.
  int gemm_thin = -1;
  // SPARSEB_GEMM_EDGES=0 keeps 64x64-tile launches in one tile shape (tuning);
  // -1 = auto: column / row edges of <= 32 go to 64x32 / 32x64 tiles.
  int gemm_edges = -1;
  // SPARSEB_AUTOTUNE=1: the first FP64 tiled block GEMM of a block-shape
  // histogram times the candidate tile shapes on its own operands and keeps the
  // fastest; later launches with the same histogram take it without timing
  // (histogram key -> (gemm_tile, gemm_edges)).  Off by default: the choice
  // depends on measured times, so two processes may pick differently.
  bool autotune = false;
  std::unordered_map<uint64_t, std::pair<int, int>> tune_table;
  // Arithmetic of the tiled block GEMMs (sb_ctx_set_precision): SB_PRECISION_F64
  // (DMMA, the drop-in), SB_PRECISION_TF32X3 or SB_PRECISION_TF32 (tcgen05).
  // The thin K <= 16 launches compute in FP64 in every mode (they are
  // HBM-bound); they read and write FP32-stored intermediates as FP32.
  int precision = SB_PRECISION_F64;
  // k-tiles (32 deep) per FP32 accumulation chunk of the tensor-core GEMM
  // (SPARSEB_TC_KC); chunks are summed with Kahan compensation.
  int tc_kc = 8;
  // SPARSEB_POISON_OUTPUT=1: contract! outputs are filled with NaN before the
  // kernels write them (a test aid that exposes unwritten elements).
  bool poison_output = false;
  // Device status word of the tensor-core GEMM (set to 1 when one of its
  // bounded waits ran out); allocated when a tensor-core precision is chosen
  // and read by sb_ctx_synchronize.
  DevBuf tc_status;
  bool tc_launched = false;  // a tensor-core GEMM ran since the status was last read
  // Plan cache of the BS x BS contract_shared! path (sb_contract.cpp): the
  // output block structure and the prepared block GEMM of recent
  // contractions, reused when the same labels meet operands of the same block
  // structure.  SPARSEB_PLAN_CACHE=0 turns it off.  Opaque here.
  bool plan_cache_on = true;
  bool plan_cache_hit = false;  // the last contraction reused a cached plan (trace line)
  // Zero padding cropped inside contract_shared! (BS x BS) on uniform
  // operands: SPARSEB_AUTO_CROP=0 off, 1 (default) for compute-heavy
  // contractions that the scan shows to be padded, 2 whenever the cropped
  // work is smaller (tests).
  int auto_crop = 1;
  bool auto_cropped = false;  // the last contraction ran cropped (trace line)
  // Device buffers of the cropped operands and result, kept per output tensor
  // between calls (sb_contract.cpp), so that repeated contractions of one
  // structure allocate nothing.  Opaque here.
  std::shared_ptr<void> crop_scratch;
  std::shared_ptr<void> plan_cache;
  // Pinned staging ring for host-to-device plan uploads: a copy from pinned
  // memory does not synchronise the stream, so host planning of the next
  // contraction overlaps the device work of the current one.  A slot is
  // reused once the event recorded after its copy has completed.
  struct Slot {
    void* host = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
  };
  std::vector<Slot> slots;
  size_t next_slot = 0;
  void stage_copy(void* dst, const void* src, size_t bytes);
  void release_staging();
  // Tensors keep their context alive: sb_ctx_destroy with live tensors only
  // marks the context, and the last sb_tensor_free destroys it.
  int64_t live_tensors = 0;  // tensors and graphs that still reference this context
  bool destroy_pending = false;
  // Stream capture into a CUDA graph (sb_ctx_capture_begin/end).  While a
  // capture is open, new device buffers are plain cudaMalloc allocations
  // (plan arrays are filled by synchronous copies outside the captured
  // stream), and every buffer released is handed to the graph instead of
  // being freed: the captured kernels may read it on every replay, so it lives
  // until sb_graph_free.
  bool capturing = false;
  std::vector<void*> capture_keep;        // plain buffers, cudaFree at graph free
  std::vector<void*> capture_keep_async;  // stream-ordered buffers, cudaFreeAsync at graph free
  void note_launch(int64_t n = 1) { launches += n; }
  void sync();
  void clear_profile();
};

// Records events around one kernel launch when the context is profiling.
class ProfScope {
 public:
  ProfScope(Ctx* c, int kind, double flops, double bytes);
  ~ProfScope();

 private:
  Ctx* c_;
  int kind_;
  double flops_, bytes_;
  cudaEvent_t a_ = nullptr;
};

// Upload a host vector to a new device buffer (stream-ordered).
template <class T>
DevBuf upload(Ctx* ctx, const std::vector<T>& v) {
  DevBuf b(ctx, v.size() * sizeof(T));
  if (ctx->capturing) {
    // outside the captured stream: the plan is on the device before any replay
    if (!v.empty()) check_cuda(cudaMemcpy(b.raw(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice),
                               "capture plan copy");
    return b;
  }
  if (!v.empty()) ctx->stage_copy(b.raw(), v.data(), v.size() * sizeof(T));
  return b;
}
template <class T>
std::vector<T> download(Ctx* ctx, const void* dptr, size_t n) {
  std::vector<T> v(n);
  if (n) {
    check_cuda(cudaMemcpyAsync(v.data(), dptr, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream), "download");
    check_cuda(cudaStreamSynchronize(ctx->stream), "download sync");
  }
  return v;
}

enum Kind : int { DENSE = SB_KIND_DENSE, COO = SB_KIND_COO, BS = SB_KIND_BLOCKSPARSE, ALIASED = SB_KIND_ALIASED };

// A fresh payload version, unique across all tensors of the process.
uint64_t next_version();

struct Tensor {
  Ctx* ctx = nullptr;
  Kind kind = DENSE;
  std::vector<int64_t> dims;
  int n2 = 0;                 // tail count (BS / aliased); dense: nd; COO: 0
  std::vector<int64_t> keys;  // row-major: nkeys x P (BS/aliased) or nkeys x N (COO); 1-based
  int64_t nkeys = 0;
  DevBuf data;                // dense values | BS blocks (packed, key order) | COO vals | aliased templates
  // aliased only
  int64_t n_templates = 0;
  std::vector<int64_t> alias_ids;  // 1-based, per key
  DevBuf scalars;                  // per key
  // COO only
  bool dirty = false;
  // Ragged block-sparse (extension of the reference format): every block has
  // its own tail extents (bdims, nkeys x n2) and offset (boff, nkeys + 1);
  // block i is column-major over bdims[i].  A uniform tensor is the special
  // case bdims[i] = dims[P:], boff[i] = i * blksize (left implicit).
  bool ragged = false;
  std::vector<int64_t> bdims;
  std::vector<int64_t> boff;
  // Key-reordering view of another tensor's payload (the operands of
  // contract_shared! whose permutation moves prefix axes only): vdata is the
  // other tensor's payload and voff[i] the offset of block i in it; data
  // stays empty.  Only the contraction that made the view reads it.
  const double* vdata = nullptr;
  std::vector<int64_t> voff;
  const struct Tensor* vsrc = nullptr;  // the tensor whose payload a view points into
  // FP32 storage (block-sparse only): the payload holds floats, one per
  // element, at the same element offsets.  Only the tensor-core contraction
  // path reads or writes such tensors (the intermediates of a TF32 H_eff
  // chain); every other kernel rejects them.
  bool f32 = false;
  // Renewed (next_version) by every library call that writes the payload
  // (contract! output, vector-space updates, a device pointer handed out);
  // unique across tensors, so (payload, version) names the values.  The
  // packed tensor-core images of an operand are kept while it matches.
  uint64_t version = next_version();

  int N() const { return static_cast<int>(dims.size()); }
  int P() const { return N() - n2; }
  int64_t blksize() const {
    int64_t b = 1;
    for (int i = P(); i < N(); ++i) b *= dims[i];
    return b;
  }
  int64_t numel() const {
    int64_t b = 1;
    for (auto d : dims) b *= d;
    return b;
  }
  const int64_t* key(int64_t i) const { return keys.data() + i * (kind == COO ? N() : P()); }
  int64_t key_len() const { return kind == COO ? N() : P(); }
  // Per-block layout, valid for uniform and ragged tensors.
  int64_t block_off(int64_t i) const { return !voff.empty() ? voff[i] : ragged ? boff[i] : i * blksize(); }
  const double* payload() const { return vdata ? vdata : data.d(); }
  // Tensor that owns the payload (itself unless a key-reordering view).
  const Tensor& owner() const { return vsrc ? *vsrc : *this; }
  int64_t block_len(int64_t i) const { return ragged ? boff[i + 1] - boff[i] : blksize(); }
  int64_t block_dim(int64_t i, int t) const { return ragged ? bdims[i * n2 + t] : dims[P() + t]; }
  int64_t payload_len() const {
    switch (kind) {
      case DENSE: return numel();
      case BS: return ragged ? (nkeys ? boff[nkeys] : 0) : nkeys * blksize();
      case COO: return nkeys;
      default: return n_templates * blksize();
    }
  }
};

using TensorPtr = std::unique_ptr<Tensor>;

// Column-major 0-based linear index of a 1-based key over dims[0..len).
inline int64_t lin0(const int64_t* k, const int64_t* dims, int len) {
  int64_t idx = 0, stride = 1;
  for (int d = 0; d < len; ++d) {
    idx += (k[d] - 1) * stride;
    stride *= dims[d];
  }
  return idx;
}

// ── tensor utilities (sb_tensor.cpp) ─────────────────────────────────────
TensorPtr make_tensor(Ctx* ctx, Kind kind, const std::vector<int64_t>& dims, int n2);
void sort_bs_keys_in_place(Tensor& t);  // keys must already be sorted-able; used at creation
TensorPtr bs_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm1);  // 1-based perm
TensorPtr aliased_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm1);
TensorPtr dense_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm1);
TensorPtr coo_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm1);  // dirty, unsorted
void coo_sort(Ctx* ctx, Tensor& A);
TensorPtr copy_tensor(Ctx* ctx, const Tensor& A);
TensorPtr bs_from_dense(Ctx* ctx, const Tensor& D, int n2, double atol, double rtol, bool dropzeros);
TensorPtr coo_from_dense(Ctx* ctx, const Tensor& D, double atol, double rtol);
TensorPtr to_dense(Ctx* ctx, const Tensor& A);
TensorPtr aliased_to_bs(Ctx* ctx, const Tensor& A);
// Ragged <-> uniform adapters (zero padding / cropping).
TensorPtr bs_to_uniform(Ctx* ctx, const Tensor& A);
// reuse: a buffer to hold the payload when its size is exactly the one needed
// (moved into the result; a new one is allocated otherwise).
TensorPtr bs_to_ragged(Ctx* ctx, const Tensor& A, const std::vector<int64_t>& bdims, bool check_zero,
                       DevBuf* reuse = nullptr);
TensorPtr bs_crop_padding(Ctx* ctx, const Tensor& A);
std::vector<std::vector<int64_t>> bs_nonzero_extents(Ctx* ctx, const std::vector<const Tensor*>& ts);
void bs_pad_into(Ctx* ctx, const Tensor& A, double* dst);
// Copies variable-size blocks: dst[dst_off[i] + e] = src[src_off[i] + e], e < len[i].
void copy_blocks(Ctx* ctx, const double* src, double* dst, const std::vector<int64_t>& src_off,
                 const std::vector<int64_t>& dst_off, const std::vector<int64_t>& len);
void require_uniform(const Tensor& t, const char* what);
// Rejects FP32-stored tensors on paths that only handle FP64 payloads.
void require_f64(const Tensor& t, const char* what);
void check_no_cross_perm(const std::vector<int>& perm1, int N, int P);
bool is_identity(const std::vector<int>& perm1);

// ── vector-space operations (sb_vector.cpp) ──────────────────────────────
double tensor_dot(Ctx* ctx, const Tensor& A, const Tensor& B);
double tensor_norm(Ctx* ctx, const Tensor& A);
void tensor_scale(Ctx* ctx, Tensor& A, double alpha);
void tensor_fill(Ctx* ctx, Tensor& A, double x);
void tensor_map(Ctx* ctx, Tensor& R, const Tensor& A, int op, double alpha, double beta);
TensorPtr tensor_similar(Ctx* ctx, const Tensor& A);
TensorPtr tensor_add(Ctx* ctx, const Tensor& A, const Tensor& B);

// ── axis fusion (sb_fuse.cpp); axes 1-based ──────────────────────────────
TensorPtr bs_fuse_axes(Ctx* ctx, const Tensor& A, int ax1, int ax2);
TensorPtr coo_fuse_axes(Ctx* ctx, const Tensor& A, int ax1, int ax2);

// ── block factorisations (sb_factorize.cpp) ──────────────────────────────
struct QrResult {
  TensorPtr Q, R;
  std::vector<int64_t> l_vals, r_vals;
};
struct SvdResult {
  TensorPtr U, SV;
  std::vector<double> svs;
  double truncerr = 0.0;
};
QrResult blocksparse_left_qr(Ctx* ctx, const Tensor& A);
SvdResult blocksparse_svd(Ctx* ctx, const Tensor& A, bool ortho_right, int64_t maxdim, int64_t mindim,
                          double cutoff);

// ── contraction (sb_contract.cpp) ────────────────────────────────────────
struct Label {
  uint64_t id, plev;
  bool operator==(const Label& o) const { return id == o.id && plev == o.plev; }
  bool operator!=(const Label& o) const { return !(*this == o); }
};
using Labels = std::vector<Label>;
void contract(Ctx* ctx, Tensor& C, const Labels& lC, const Tensor& A, const Labels& lA, const Tensor& B,
              const Labels& lB);

}  // namespace sb

struct sb_ctx {
  sb::Ctx impl;
};
struct sb_graph {
  sb_ctx* owner = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<void*> keep, keep_async;  // buffers the captured kernels may read
};
struct sb_tensor {
  sb::TensorPtr impl;
  sb_ctx* owner = nullptr;
};
