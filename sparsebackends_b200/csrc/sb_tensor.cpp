// Tensor storage on the device: creation helpers, permutes and conversions.
//
// Reference: SparseBackends/src/blocksparse/{storage,conversions}.jl,
// src/coo/{storage,conversions}.jl, src/aliased/{storage,conversions}.jl.
// Keys (integer metadata) live on the host; every payload value lives on and
// is produced by the device.
#include <atomic>
#include <algorithm>
#include <cstring>
#include <numeric>

#include "sb_internal.hpp"

namespace sb {

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    fail(SB_ERR_OOM, std::string("device allocation failed: ") + what);
  }
  fail(SB_ERR_CUDA, std::string(cudaGetErrorString(e)) + " at " + what);
}

void Ctx::sync() { SB_CK(cudaStreamSynchronize(stream)); }

void Ctx::stage_copy(void* dst, const void* src, size_t bytes) {
  if (slots.empty()) slots.resize(32);
  Slot& s = slots[next_slot];
  next_slot = (next_slot + 1) % slots.size();
  if (s.pending) {
    SB_CK(cudaEventSynchronize(s.ev));
    s.pending = false;
  }
  if (!s.ev) SB_CK(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  if (s.cap < bytes) {
    if (s.host) SB_CK(cudaFreeHost(s.host));
    s.host = nullptr;
    s.cap = 0;
    const size_t cap = std::max<size_t>(bytes, std::max<size_t>(64 << 10, 2 * s.cap));
    SB_CK(cudaHostAlloc(&s.host, cap, cudaHostAllocDefault));
    s.cap = cap;
  }
  std::memcpy(s.host, src, bytes);
  SB_CK(cudaMemcpyAsync(dst, s.host, bytes, cudaMemcpyHostToDevice, stream));
  SB_CK(cudaEventRecord(s.ev, stream));
  s.pending = true;
}

void Ctx::release_staging() {
  for (auto& s : slots) {
    if (s.ev) {
      cudaEventSynchronize(s.ev);
      cudaEventDestroy(s.ev);
    }
    if (s.host) cudaFreeHost(s.host);
  }
  slots.clear();
  next_slot = 0;
}

void Ctx::clear_profile() {
  for (auto& r : prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  prof.clear();
}

ProfScope::ProfScope(Ctx* c, int kind, double flops, double bytes) : c_(c), kind_(kind), flops_(flops), bytes_(bytes) {
  if (!c_->profiling || c_->capturing) return;
  SB_CK(cudaEventCreate(&a_));
  SB_CK(cudaEventRecord(a_, c_->stream));
}
ProfScope::~ProfScope() {
  if (!a_) return;
  cudaEvent_t b = nullptr;
  if (cudaEventCreate(&b) != cudaSuccess || cudaEventRecord(b, c_->stream) != cudaSuccess) {
    cudaEventDestroy(a_);
    if (b) cudaEventDestroy(b);
    return;
  }
  c_->prof.push_back(Ctx::ProfRec{kind_, a_, b, flops_, bytes_});
}

DevBuf::DevBuf(Ctx* ctx, size_t bytes) : ctx_(ctx), n_(bytes) {
  if (!bytes) return;
  if (ctx->capturing) {
    SB_CK(cudaMalloc(&p_, bytes));
    plain_ = true;
  } else {
    SB_CK(cudaMallocAsync(&p_, bytes, ctx->stream));
  }
}
DevBuf::~DevBuf() { reset(); }
void DevBuf::reset() {
  if (p_) {
    if (ctx_->capturing) {
      (plain_ ? ctx_->capture_keep : ctx_->capture_keep_async).push_back(p_);
    } else if (plain_) {
      cudaFree(p_);
    } else {
      cudaFreeAsync(p_, ctx_->stream);
    }
  }
  p_ = nullptr;
  n_ = 0;
  plain_ = false;
}
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    reset();
    ctx_ = o.ctx_;
    p_ = o.p_;
    n_ = o.n_;
    plain_ = o.plain_;
    o.p_ = nullptr;
    o.n_ = 0;
    o.plain_ = false;
  }
  return *this;
}

TensorPtr make_tensor(Ctx* ctx, Kind kind, const std::vector<int64_t>& dims, int n2) {
  auto t = std::make_unique<Tensor>();
  t->ctx = ctx;
  t->kind = kind;
  t->dims = dims;
  t->n2 = n2;
  return t;
}

bool is_identity(const std::vector<int>& p) {
  for (size_t i = 0; i < p.size(); ++i)
    if (p[i] != static_cast<int>(i) + 1) return false;
  return true;
}

void check_no_cross_perm(const std::vector<int>& perm, int N, int P) {
  require(static_cast<int>(perm.size()) == N, SB_ERR_ASSERTION, "perm length must equal rank");
  std::vector<int> s(perm);
  std::sort(s.begin(), s.end());
  for (int i = 0; i < N; ++i) require(s[i] == i + 1, SB_ERR_ASSERTION, "perm must be a permutation of 1:N");
  for (int i = 0; i < P; ++i)
    require(perm[i] <= P, SB_ERR_ASSERTION, "No-cross reorder violated: output prefix axis uses old block axis");
  for (int i = P; i < N; ++i)
    require(perm[i] > P, SB_ERR_ASSERTION, "No-cross reorder violated: output block axis uses old prefix axis");
}

// Column-major strides of dims[lo..hi).
static std::vector<int64_t> cm_strides(const std::vector<int64_t>& dims, int lo, int hi) {
  std::vector<int64_t> s(hi - lo);
  int64_t acc = 1;
  for (int i = lo; i < hi; ++i) {
    s[i - lo] = acc;
    acc *= dims[i];
  }
  return s;
}

// dst block b = tail permutation of src block at src_off[b].
static void permute_blocks(Ctx* ctx, const double* src, double* dst, const std::vector<int64_t>& src_off,
                           int64_t blk, const std::vector<int64_t>& out_dims, const std::vector<int64_t>& in_strides) {
  if (src_off.empty() || blk == 0) return;
  require(out_dims.size() <= static_cast<size_t>(kMaxRank), SB_ERR_INVALID_ARG, "tail rank too large");
  PermDesc d{};
  // Drop unit axes; they do not move data.
  int r = 0;
  for (size_t i = 0; i < out_dims.size(); ++i) {
    if (out_dims[i] == 1) continue;
    d.out_dims[r] = out_dims[i];
    d.in_strides[r] = in_strides[i];
    ++r;
  }
  d.rank = r;
  DevBuf doff = upload(ctx, src_off);
  {
    ProfScope ps(ctx, PROF_PERMUTE, 0.0, 16.0 * static_cast<double>(src_off.size()) * static_cast<double>(blk));
    SB_CK(launch_permute_blocks(src, dst, doff.as<int64_t>(), static_cast<int64_t>(src_off.size()), blk, d, ctx->stream));
  }
  ctx->note_launch();
}

void sort_bs_keys_in_place(Tensor& t) {
  (void)t;  // keys are kept sorted by construction
}

void require_uniform(const Tensor& t, const char* what) {
  if (t.ragged)
    fail(SB_ERR_UNSUPPORTED_LAYOUT,
         std::string(what) + ": ragged block-sparse operands are supported by contract_shared! (BS x BS), "
                             "permutedims and the uniform/ragged adapters; convert with sb_tensor_to_uniform");
}

void require_f64(const Tensor& t, const char* what) {
  if (t.f32)
    fail(SB_ERR_UNSUPPORTED_TYPES,
         std::string(what) + ": FP32-stored tensors (tensor-core chain intermediates) are supported by "
                             "contract_shared! (BS x BS) and the exports only");
}

uint64_t next_version() {
  static std::atomic<uint64_t> counter{0};
  return counter.fetch_add(1, std::memory_order_relaxed) + 1;
}

void copy_blocks(Ctx* ctx, const double* src, double* dst, const std::vector<int64_t>& src_off,
                 const std::vector<int64_t>& dst_off, const std::vector<int64_t>& len) {
  if (src_off.empty()) return;
  std::vector<BlockCopy> items(src_off.size());
  int64_t mx = 0;
  double bytes = 0.0;
  for (size_t i = 0; i < items.size(); ++i) {
    items[i] = BlockCopy{src_off[i], dst_off[i], len[i]};
    mx = std::max(mx, len[i]);
    bytes += 16.0 * len[i];
  }
  DevBuf d = upload(ctx, items);
  ProfScope ps(ctx, PROF_PERMUTE, 0.0, bytes);
  SB_CK(launch_copy_blocks(src, dst, d.as<BlockCopy>(), static_cast<int64_t>(items.size()), mx, ctx->stream));
  ctx->note_launch();
}

// Per-block permute/pad/crop through BlockPerm descriptors.
static void perm_blocks(Ctx* ctx, const double* src, double* dst, std::vector<BlockPerm>& items) {
  if (items.empty()) return;
  int64_t mx = 0, mx_rows = 0;
  double bytes = 0.0;
  // rows of unit-stride runs (padding, cropping, outer-axis permutes) when
  // every item has them and they are at least 16 long on average
  bool rows = true;
  int64_t elems = 0, nrows = 0;
  for (auto& it : items) {
    mx = std::max(mx, it.len);
    bytes += 16.0 * it.len;
    rows = rows && it.rank >= 1 && it.in_strides[0] == 1 && it.out_dims[0] >= 1;
    if (rows) {
      mx_rows = std::max(mx_rows, it.len / it.out_dims[0]);
      elems += it.len;
      nrows += it.len / it.out_dims[0];
    }
  }
  rows = rows && elems >= 16 * nrows;
  DevBuf d = upload(ctx, items);
  ProfScope ps(ctx, PROF_PERMUTE, 0.0, bytes);
  if (rows)
    SB_CK(launch_perm_block_rows(src, dst, d.as<BlockPerm>(), static_cast<int64_t>(items.size()), mx_rows,
                                 ctx->stream));
  else
    SB_CK(launch_perm_blocks(src, dst, d.as<BlockPerm>(), static_cast<int64_t>(items.size()), mx, ctx->stream));
  ctx->note_launch();
}

static BlockPerm make_block_perm(int64_t src_off, int64_t dst_off, const std::vector<int64_t>& out_dims,
                                 const std::vector<int64_t>& in_strides, const std::vector<int64_t>& in_lim) {
  require(out_dims.size() <= static_cast<size_t>(kMaxRank), SB_ERR_INVALID_ARG, "tail rank too large");
  BlockPerm b{};
  b.src_off = src_off;
  b.dst_off = dst_off;
  b.len = 1;
  b.rank = static_cast<int>(out_dims.size());
  for (size_t r = 0; r < out_dims.size(); ++r) {
    b.out_dims[r] = out_dims[r];
    b.in_strides[r] = in_strides[r];
    b.in_lim[r] = in_lim[r];
    b.len *= out_dims[r];
  }
  return b;
}

// The uniform (zero-padded) blocks of A, in key order, written to dst
// (nkeys x blksize doubles).
void bs_pad_into(Ctx* ctx, const Tensor& A, double* dst) {
  const int64_t blk = A.blksize();
  if (!A.ragged) {
    if (A.nkeys)
      SB_CK(cudaMemcpyAsync(dst, A.payload(), A.nkeys * blk * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    return;
  }
  const int P = A.P();
  std::vector<int64_t> od(A.dims.begin() + P, A.dims.end());
  std::vector<BlockPerm> items;
  for (int64_t i = 0; i < A.nkeys; ++i) {
    std::vector<int64_t> st(A.n2), lim(A.n2);
    int64_t acc = 1;
    for (int t = 0; t < A.n2; ++t) {
      st[t] = acc;
      lim[t] = A.block_dim(i, t);
      acc *= lim[t];
    }
    items.push_back(make_block_perm(A.block_off(i), i * blk, od, st, lim));
  }
  perm_blocks(ctx, A.payload(), dst, items);
}

TensorPtr bs_to_uniform(Ctx* ctx, const Tensor& A) {
  require(A.kind == BS, SB_ERR_INVALID_ARG, "to_uniform needs a block-sparse tensor");
  auto out = make_tensor(ctx, BS, A.dims, A.n2);
  out->keys = A.keys;
  out->nkeys = A.nkeys;
  out->data = DevBuf(ctx, A.nkeys * A.blksize() * sizeof(double));
  bs_pad_into(ctx, A, out->data.d());
  return out;
}

// Per block (key order) and tail axis: 1 + the largest coordinate of a
// nonzero entry (1 for an all-zero block), for each of the tensors: one device
// scan each, one read-back for all of them.
std::vector<std::vector<int64_t>> bs_nonzero_extents(Ctx* ctx, const std::vector<const Tensor*>& ts) {
  std::vector<std::vector<int64_t>> out(ts.size());
  std::vector<int64_t> base(ts.size() + 1, 0);
  for (size_t k = 0; k < ts.size(); ++k) base[k + 1] = base[k] + ts[k]->nkeys * ts[k]->n2;
  if (base.back() == 0) {
    for (size_t k = 0; k < ts.size(); ++k) out[k].assign(ts[k]->nkeys * ts[k]->n2, 1);
    return out;
  }
  DevBuf dext = upload(ctx, std::vector<int>(base.back(), 1));
  std::vector<DevBuf> keep;
  for (size_t k = 0; k < ts.size(); ++k) {
    const Tensor& A = *ts[k];
    const int64_t n = A.nkeys;
    if (n == 0 || A.n2 == 0) continue;
    std::vector<int64_t> off(n), dims(n * A.n2), tb(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
      off[i] = A.block_off(i);
      int64_t cols = 1;
      for (int t = 0; t < A.n2; ++t) {
        dims[i * A.n2 + t] = A.block_dim(i, t);
        if (t > 0) cols *= dims[i * A.n2 + t];
      }
      tb[i + 1] = tb[i] + block_extent_tasks(dims[i * A.n2], cols);
    }
    keep.push_back(upload(ctx, off));
    keep.push_back(upload(ctx, dims));
    keep.push_back(upload(ctx, tb));
    const size_t m = keep.size();
    SB_CK(launch_block_extents(A.payload(), keep[m - 3].as<int64_t>(), keep[m - 2].as<int64_t>(),
                               keep[m - 1].as<int64_t>(), n, tb[n], A.n2, dext.as<int>() + base[k], ctx->stream));
    ctx->note_launch();
  }
  const auto e = download<int>(ctx, dext.raw(), base.back());
  for (size_t k = 0; k < ts.size(); ++k) out[k].assign(e.begin() + base[k], e.begin() + base[k + 1]);
  return out;
}

// The ragged tensor whose blocks are A's blocks cropped to the smallest tail
// extents that keep their nonzero entries: the reference layout's zero
// padding (every U(1) sector padded to the largest) found from the values.
TensorPtr bs_crop_padding(Ctx* ctx, const Tensor& A) {
  require(A.kind == BS, SB_ERR_INVALID_ARG, "crop_padding needs a block-sparse tensor");
  return bs_to_ragged(ctx, A, bs_nonzero_extents(ctx, {&A})[0], false);
}

TensorPtr bs_to_ragged(Ctx* ctx, const Tensor& A, const std::vector<int64_t>& bd, bool check_zero, DevBuf* reuse) {
  require(A.kind == BS, SB_ERR_INVALID_ARG, "to_ragged needs a block-sparse tensor");
  require(static_cast<int64_t>(bd.size()) == A.nkeys * A.n2, SB_ERR_INVALID_ARG, "block_dims must be nkeys x n_tail");
  const int P = A.P();
  auto out = make_tensor(ctx, BS, A.dims, A.n2);
  out->keys = A.keys;
  out->nkeys = A.nkeys;
  out->ragged = true;
  out->bdims = bd;
  out->boff.assign(A.nkeys + 1, 0);
  for (int64_t i = 0; i < A.nkeys; ++i) {
    int64_t len = 1;
    for (int t = 0; t < A.n2; ++t) {
      const int64_t e = bd[i * A.n2 + t];
      require(e >= 1 && e <= A.block_dim(i, t), SB_ERR_ASSERTION, "block extent out of range");
      len *= e;
    }
    out->boff[i + 1] = out->boff[i] + len;
  }
  const size_t need = out->boff[A.nkeys] * sizeof(double);
  if (reuse && reuse->bytes() == need) out->data = std::move(*reuse);
  else out->data = DevBuf(ctx, need);
  std::vector<BlockPerm> items, checks;
  for (int64_t i = 0; i < A.nkeys; ++i) {
    std::vector<int64_t> od(A.n2), st(A.n2), full(A.n2);
    int64_t acc = 1;
    for (int t = 0; t < A.n2; ++t) {
      od[t] = bd[i * A.n2 + t];
      full[t] = A.block_dim(i, t);
      st[t] = acc;
      acc *= full[t];
    }
    items.push_back(make_block_perm(A.block_off(i), out->boff[i], od, st, od));
    if (check_zero) checks.push_back(make_block_perm(A.block_off(i), 0, full, st, od));
  }
  if (check_zero && !checks.empty()) {
    int64_t mx = 0;
    for (auto& c : checks) mx = std::max(mx, c.len);
    DevBuf dc = upload(ctx, checks);
    DevBuf fl(ctx, checks.size());
    SB_CK(launch_outside_nonzero(A.payload(), dc.as<BlockPerm>(), static_cast<int64_t>(checks.size()), mx,
                                 fl.as<uint8_t>(), ctx->stream));
    ctx->note_launch();
    auto f = download<uint8_t>(ctx, fl.raw(), checks.size());
    for (size_t i = 0; i < f.size(); ++i)
      require(!f[i], SB_ERR_ASSERTION, "cropping would drop nonzero entries of block " + std::to_string(i + 1));
  }
  perm_blocks(ctx, A.payload(), out->data.d(), items);
  return out;
}

TensorPtr bs_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm) {
  const int N = A.N(), P = A.P();
  check_no_cross_perm(perm, N, P);
  std::vector<int64_t> dimsB(N);
  for (int j = 0; j < N; ++j) dimsB[j] = A.dims[perm[j] - 1];
  auto out = make_tensor(ctx, BS, dimsB, A.n2);
  const int64_t n = A.nkeys, blk = A.blksize();
  std::vector<int64_t> nk(n * P);
  std::vector<int64_t> lin(n);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t* k = A.key(i);
    for (int j = 0; j < P; ++j) nk[i * P + j] = k[perm[j] - 1];
    lin[i] = lin0(&nk[i * P], dimsB.data(), P);
  }
  std::vector<int64_t> p(n);
  std::iota(p.begin(), p.end(), 0);
  std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
  out->keys.resize(n * P);
  for (int64_t i = 0; i < n; ++i)
    std::copy(&nk[p[i] * P], &nk[p[i] * P] + P, &out->keys[i * P]);
  out->nkeys = n;
  bool tail_identity = true;
  for (int r = 0; r < A.n2; ++r) tail_identity = tail_identity && perm[P + r] == P + r + 1;
  if (A.ragged) {
    // per-block extents travel with their blocks, permuted like the tail axes
    out->ragged = true;
    out->bdims.resize(n * A.n2);
    out->boff.assign(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
      for (int r = 0; r < A.n2; ++r) out->bdims[i * A.n2 + r] = A.block_dim(p[i], perm[P + r] - 1 - P);
      out->boff[i + 1] = out->boff[i] + A.block_len(p[i]);
    }
    out->data = DevBuf(ctx, out->boff[n] * sizeof(double));
    if (tail_identity) {
      std::vector<int64_t> so(n), dof(n), len(n);
      for (int64_t i = 0; i < n; ++i) {
        so[i] = A.block_off(p[i]);
        dof[i] = out->boff[i];
        len[i] = A.block_len(p[i]);
      }
      copy_blocks(ctx, A.payload(), out->data.d(), so, dof, len);
    } else {
      std::vector<BlockPerm> items;
      for (int64_t i = 0; i < n; ++i) {
        std::vector<int64_t> sst(A.n2), od(A.n2), is(A.n2);
        int64_t acc = 1;
        for (int t = 0; t < A.n2; ++t) {
          sst[t] = acc;
          acc *= A.block_dim(p[i], t);
        }
        for (int r = 0; r < A.n2; ++r) {
          od[r] = out->bdims[i * A.n2 + r];
          is[r] = sst[perm[P + r] - 1 - P];
        }
        items.push_back(make_block_perm(A.block_off(p[i]), out->boff[i], od, is, od));
      }
      perm_blocks(ctx, A.payload(), out->data.d(), items);
    }
    return out;
  }
  out->data = DevBuf(ctx, n * blk * sizeof(double));
  std::vector<int64_t> soff(n);
  for (int64_t i = 0; i < n; ++i) soff[i] = A.block_off(p[i]);
  auto so = cm_strides(A.dims, P, N);
  std::vector<int64_t> od(A.n2), is(A.n2);
  for (int r = 0; r < A.n2; ++r) {
    od[r] = dimsB[P + r];
    is[r] = so[perm[P + r] - 1 - P];
  }
  permute_blocks(ctx, A.payload(), out->data.d(), soff, blk, od, is);
  return out;
}

TensorPtr aliased_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm) {
  const int N = A.N(), P = A.P();
  check_no_cross_perm(perm, N, P);
  std::vector<int64_t> dimsB(N);
  for (int j = 0; j < N; ++j) dimsB[j] = A.dims[perm[j] - 1];
  auto out = make_tensor(ctx, ALIASED, dimsB, A.n2);
  const int64_t blk = A.blksize();
  out->n_templates = A.n_templates;
  out->data = DevBuf(ctx, A.n_templates * blk * sizeof(double));
  std::vector<int64_t> soff(A.n_templates);
  for (int64_t t = 0; t < A.n_templates; ++t) soff[t] = t * blk;
  auto so = cm_strides(A.dims, P, N);
  std::vector<int64_t> od(A.n2), is(A.n2);
  for (int r = 0; r < A.n2; ++r) {
    od[r] = dimsB[P + r];
    is[r] = so[perm[P + r] - 1 - P];
  }
  permute_blocks(ctx, A.data.d(), out->data.d(), soff, blk, od, is);
  const int64_t n = A.nkeys;
  std::vector<int64_t> nk(n * P), lin(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int j = 0; j < P; ++j) nk[i * P + j] = A.key(i)[perm[j] - 1];
    lin[i] = lin0(&nk[i * P], dimsB.data(), P);
  }
  std::vector<int64_t> p(n);
  std::iota(p.begin(), p.end(), 0);
  std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
  out->keys.resize(n * P);
  out->alias_ids.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    std::copy(&nk[p[i] * P], &nk[p[i] * P] + P, &out->keys[i * P]);
    out->alias_ids[i] = A.alias_ids[p[i]];
  }
  out->nkeys = n;
  out->scalars = DevBuf(ctx, n * sizeof(double));
  if (n) {
    DevBuf dp = upload(ctx, p);
    SB_CK(launch_gather(A.scalars.d(), dp.as<int64_t>(), n, out->scalars.d(), ctx->stream));
    ctx->note_launch();
  }
  return out;
}

TensorPtr dense_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm) {
  const int N = A.N();
  require(static_cast<int>(perm.size()) == N, SB_ERR_ASSERTION, "perm length must equal rank");
  std::vector<int64_t> dimsB(N);
  for (int j = 0; j < N; ++j) dimsB[j] = A.dims[perm[j] - 1];
  auto out = make_tensor(ctx, DENSE, dimsB, N);
  const int64_t n = A.numel();
  out->data = DevBuf(ctx, n * sizeof(double));
  auto so = cm_strides(A.dims, 0, N);
  std::vector<int64_t> is(N);
  for (int r = 0; r < N; ++r) is[r] = so[perm[r] - 1];
  permute_blocks(ctx, A.data.d(), out->data.d(), {0}, n, dimsB, is);
  return out;
}

TensorPtr copy_tensor(Ctx* ctx, const Tensor& A) {
  auto out = make_tensor(ctx, A.kind, A.dims, A.n2);
  out->keys = A.keys;
  out->nkeys = A.nkeys;
  out->n_templates = A.n_templates;
  out->alias_ids = A.alias_ids;
  out->dirty = A.dirty;
  out->ragged = A.ragged;
  out->bdims = A.bdims;
  out->boff = A.boff;
  const int64_t len = A.payload_len();
  out->data = DevBuf(ctx, len * sizeof(double));
  if (len) SB_CK(cudaMemcpyAsync(out->data.raw(), A.data.raw(), len * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (A.kind == ALIASED) {
    out->scalars = DevBuf(ctx, A.nkeys * sizeof(double));
    if (A.nkeys)
      SB_CK(cudaMemcpyAsync(out->scalars.raw(), A.scalars.raw(), A.nkeys * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return out;
}

TensorPtr coo_permute(Ctx* ctx, const Tensor& A, const std::vector<int>& perm) {
  const int N = A.N();
  require(static_cast<int>(perm.size()) == N, SB_ERR_ASSERTION, "perm length must equal rank");
  std::vector<int> s(perm);
  std::sort(s.begin(), s.end());
  for (int i = 0; i < N; ++i) require(s[i] == i + 1, SB_ERR_INVALID_ARG, "perm must be a permutation of 1:N");
  auto out = copy_tensor(ctx, A);
  for (int j = 0; j < N; ++j) out->dims[j] = A.dims[perm[j] - 1];
  for (int64_t i = 0; i < A.nkeys; ++i)
    for (int j = 0; j < N; ++j) out->keys[i * N + j] = A.keys[i * N + perm[j] - 1];
  out->dirty = true;
  return out;
}

void coo_sort(Ctx* ctx, Tensor& A) {
  if (!A.dirty) return;
  const int N = A.N();
  const int64_t n = A.nkeys;
  std::vector<int64_t> p(n);
  std::iota(p.begin(), p.end(), 0);
  // sortperm(keys; by = reverse): lexicographic on the reversed tuple.
  std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) {
    for (int d = N - 1; d >= 0; --d) {
      const int64_t x = A.keys[a * N + d], y = A.keys[b * N + d];
      if (x != y) return x < y;
    }
    return false;
  });
  std::vector<int64_t> nk(n * N);
  for (int64_t i = 0; i < n; ++i) std::copy(&A.keys[p[i] * N], &A.keys[p[i] * N] + N, &nk[i * N]);
  A.keys.swap(nk);
  if (n) {
    DevBuf nv(ctx, n * sizeof(double));
    DevBuf dp = upload(ctx, p);
    SB_CK(launch_gather(A.data.d(), dp.as<int64_t>(), n, nv.d(), ctx->stream));
    ctx->note_launch();
    A.data = std::move(nv);
  }
  A.dirty = false;
}

TensorPtr bs_from_dense(Ctx* ctx, const Tensor& D, int n2, double atol, double rtol, bool dropzeros) {
  require(D.kind == DENSE, SB_ERR_INVALID_ARG, "blocksparse_from_dense needs a dense tensor");
  const int N = D.N();
  require(n2 >= 0 && n2 <= N, SB_ERR_ASSERTION, "0 <= N2 <= N required");
  const int P = N - n2;
  int64_t Ptot = 1, blk = 1;
  for (int i = 0; i < P; ++i) Ptot *= D.dims[i];
  for (int i = P; i < N; ++i) blk *= D.dims[i];
  auto out = make_tensor(ctx, BS, D.dims, n2);
  // Block-major copy: blocks[p*blk + t] = dense[p + Ptot*t].
  DevBuf blocks(ctx, Ptot * blk * sizeof(double));
  permute_blocks(ctx, D.data.d(), blocks.d(), {0}, Ptot * blk, {blk, Ptot}, {Ptot, 1});
  double gmax = 0.0;
  if (rtol != 0.0 && Ptot * blk > 0) {
    DevBuf dm(ctx, sizeof(double));
    SB_CK(launch_maxabs(D.data.d(), Ptot * blk, dm.d(), ctx->stream));
    ctx->note_launch();
    gmax = download<double>(ctx, dm.raw(), 1)[0];
  }
  const double tol = std::max(atol, rtol * gmax);
  std::vector<uint8_t> keep(Ptot, 1);
  if (dropzeros && Ptot > 0) {
    DevBuf fl(ctx, Ptot);
    SB_CK(launch_block_max_gt(blocks.d(), Ptot, blk, tol, fl.as<uint8_t>(), ctx->stream));
    ctx->note_launch();
    keep = download<uint8_t>(ctx, fl.raw(), Ptot);
  }
  std::vector<int64_t> soff;
  for (int64_t p = 0; p < Ptot; ++p) {
    if (!keep[p]) continue;
    soff.push_back(p * blk);
    int64_t r = p;
    for (int d = 0; d < P; ++d) {
      out->keys.push_back(r % D.dims[d] + 1);
      r /= D.dims[d];
    }
  }
  out->nkeys = static_cast<int64_t>(soff.size());
  out->data = DevBuf(ctx, out->nkeys * blk * sizeof(double));
  permute_blocks(ctx, blocks.d(), out->data.d(), soff, blk, {blk}, {1});
  return out;
}

TensorPtr coo_from_dense(Ctx* ctx, const Tensor& D, double atol, double rtol) {
  require(D.kind == DENSE, SB_ERR_INVALID_ARG, "coo_from_dense needs a dense tensor");
  const int N = D.N();
  const int64_t n = D.numel();
  auto out = make_tensor(ctx, COO, D.dims, 0);
  std::vector<uint8_t> keep;
  if (n) {
    DevBuf fl(ctx, n);
    SB_CK(launch_elem_keep(D.data.d(), n, atol, rtol, fl.as<uint8_t>(), ctx->stream));
    ctx->note_launch();
    keep = download<uint8_t>(ctx, fl.raw(), n);
  }
  std::vector<int64_t> idx;
  for (int64_t i = 0; i < n; ++i) {
    if (!keep[i]) continue;
    idx.push_back(i);
    int64_t r = i;
    for (int d = 0; d < N; ++d) {
      out->keys.push_back(r % D.dims[d] + 1);
      r /= D.dims[d];
    }
  }
  out->nkeys = static_cast<int64_t>(idx.size());
  out->data = DevBuf(ctx, out->nkeys * sizeof(double));
  if (out->nkeys) {
    DevBuf di = upload(ctx, idx);
    SB_CK(launch_gather(D.data.d(), di.as<int64_t>(), out->nkeys, out->data.d(), ctx->stream));
    ctx->note_launch();
  }
  out->dirty = false;
  return out;
}

TensorPtr aliased_to_bs(Ctx* ctx, const Tensor& A) {
  require(A.kind == ALIASED, SB_ERR_INVALID_ARG, "to_blocksparse needs an aliased tensor");
  auto out = make_tensor(ctx, BS, A.dims, A.n2);
  out->keys = A.keys;
  out->nkeys = A.nkeys;
  const int64_t blk = A.blksize();
  out->data = DevBuf(ctx, A.nkeys * blk * sizeof(double));
  if (A.nkeys) {
    std::vector<int64_t> toff(A.nkeys);
    for (int64_t i = 0; i < A.nkeys; ++i) toff[i] = (A.alias_ids[i] - 1) * blk;
    DevBuf dt = upload(ctx, toff);
    SB_CK(launch_scale_blocks(A.data.d(), dt.as<int64_t>(), A.scalars.d(), A.nkeys, blk, out->data.d(), ctx->stream));
    ctx->note_launch();
  }
  return out;
}

TensorPtr to_dense(Ctx* ctx, const Tensor& A) {
  if (A.kind == DENSE) return copy_tensor(ctx, A);
  if (A.kind == BS && A.ragged) {
    auto u = bs_to_uniform(ctx, A);
    return to_dense(ctx, *u);
  }
  if (A.kind == ALIASED) {
    auto b = aliased_to_bs(ctx, A);
    return to_dense(ctx, *b);
  }
  const int N = A.N();
  auto out = make_tensor(ctx, DENSE, A.dims, N);
  const int64_t n = A.numel();
  out->data = DevBuf(ctx, n * sizeof(double));
  if (n) SB_CK(cudaMemsetAsync(out->data.raw(), 0, n * sizeof(double), ctx->stream));
  if (A.kind == BS) {
    const int P = A.P();
    int64_t Ptot = 1;
    for (int i = 0; i < P; ++i) Ptot *= A.dims[i];
    std::vector<int64_t> lin(A.nkeys);
    for (int64_t i = 0; i < A.nkeys; ++i) lin[i] = lin0(A.key(i), A.dims.data(), P);
    if (A.nkeys) {
      DevBuf dl = upload(ctx, lin);
      SB_CK(launch_blocks_to_strided(A.data.d(), dl.as<int64_t>(), A.nkeys, A.blksize(), Ptot, out->data.d(), ctx->stream));
      ctx->note_launch();
    }
  } else {  // COO: later duplicates overwrite earlier ones, as `out[coord...] = v` in order
    std::vector<int64_t> lin(A.nkeys);
    for (int64_t i = 0; i < A.nkeys; ++i) lin[i] = lin0(A.key(i), A.dims.data(), N);
    std::vector<int64_t> last_src, dst;
    std::vector<int64_t> order(A.nkeys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
    for (size_t j = 0; j < order.size(); ++j) {
      if (j + 1 < order.size() && lin[order[j + 1]] == lin[order[j]]) continue;
      last_src.push_back(order[j]);
      dst.push_back(lin[order[j]]);
    }
    if (!dst.empty()) {
      DevBuf ds = upload(ctx, last_src), dd = upload(ctx, dst);
      DevBuf tmp(ctx, dst.size() * sizeof(double));
      SB_CK(launch_gather(A.data.d(), ds.as<int64_t>(), static_cast<int64_t>(dst.size()), tmp.d(), ctx->stream));
      SB_CK(launch_scatter(tmp.d(), dd.as<int64_t>(), static_cast<int64_t>(dst.size()), out->data.d(), ctx->stream));
      ctx->note_launch(2);
    }
  }
  return out;
}

}  // namespace sb
