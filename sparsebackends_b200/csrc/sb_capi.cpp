// extern "C" entry points of libsparseb (declared in include/sparseb.h).
// No C++ exception crosses this boundary: every failure becomes an
// sb_status and a message retrievable with sb_last_error().
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "sb_internal.hpp"

using namespace sb;

namespace {

thread_local std::string g_noctx_error;

template <class F>
sb_status guard(sb_ctx* ctx, F&& f) {
  try {
    f();
    if (ctx) ctx->impl.last_error.clear();
    return SB_OK;
  } catch (const Error& e) {
    (ctx ? ctx->impl.last_error : g_noctx_error) = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    (ctx ? ctx->impl.last_error : g_noctx_error) = "host allocation failed";
    return SB_ERR_OOM;
  } catch (const std::exception& e) {
    (ctx ? ctx->impl.last_error : g_noctx_error) = e.what();
    return SB_ERR_INVALID_ARG;
  }
}

std::vector<int64_t> read_dims(int nd, const int64_t* dims) {
  require(nd >= 0 && nd <= 64, SB_ERR_INVALID_ARG, "rank out of range");
  require(nd == 0 || dims != nullptr, SB_ERR_INVALID_ARG, "dims is NULL");
  std::vector<int64_t> d(dims, dims + nd);
  for (auto x : d) require(x >= 1, SB_ERR_ASSERTION, "all dims must be >= 1");
  return d;
}

Labels read_labels(const uint64_t* p, int n) {
  require(n >= 0 && (n == 0 || p != nullptr), SB_ERR_INVALID_ARG, "label array is NULL");
  Labels l(n);
  for (int i = 0; i < n; ++i) l[i] = Label{p[2 * i], p[2 * i + 1]};
  return l;
}

sb_tensor* wrap(sb_ctx* ctx, TensorPtr t) {
  auto* h = new sb_tensor;
  h->impl = std::move(t);
  h->owner = ctx;
  if (ctx) ++ctx->impl.live_tensors;
  return h;
}

void destroy_ctx_now(sb_ctx* ctx) {
  cudaSetDevice(ctx->impl.device);
  cudaStreamSynchronize(ctx->impl.stream);
  ctx->impl.clear_profile();
  ctx->impl.plan_cache.reset();  // its device buffers are released on the stream
  ctx->impl.crop_scratch.reset();
  ctx->impl.tc_status.reset();
  cudaStreamSynchronize(ctx->impl.stream);
  ctx->impl.release_staging();
  if (ctx->impl.own_stream) cudaStreamDestroy(ctx->impl.stream);
  delete ctx;
}

void check_keys_in_range(const std::vector<int64_t>& keys, int64_t n, int klen, const std::vector<int64_t>& dims) {
  for (int64_t i = 0; i < n; ++i)
    for (int j = 0; j < klen; ++j) {
      const int64_t v = keys[i * klen + j];
      require(v >= 1 && v <= dims[j], SB_ERR_ASSERTION, "key coordinate out of bounds");
    }
}

void check_ctx(sb_ctx* ctx) { require(ctx != nullptr, SB_ERR_INVALID_ARG, "context is NULL"); }

// After a synchronisation: a tensor-core GEMM whose bounded wait ran out
// left 1 in the context's status word (its results are invalid).
void check_tc_status(sb_ctx* ctx) {
  if (!ctx->impl.tc_launched || !ctx->impl.tc_status.raw()) return;
  int st = 0;
  SB_CK(cudaMemcpy(&st, ctx->impl.tc_status.raw(), sizeof(int), cudaMemcpyDeviceToHost));
  ctx->impl.tc_launched = false;
  if (st != 0) {
    SB_CK(cudaMemset(ctx->impl.tc_status.raw(), 0, sizeof(int)));
    sb::fail(SB_ERR_TIMEOUT, "tensor-core block GEMM: a bounded wait on the tensor core ran out; results are invalid");
  }
}
void check_t(const sb_tensor* t) { require(t != nullptr && t->impl, SB_ERR_INVALID_ARG, "tensor is NULL"); }

}  // namespace

extern "C" {

sb_status sb_ctx_create(int device, unsigned flags, sb_ctx** out) {
  (void)flags;
  return guard(nullptr, [&] {
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(device));
    auto* c = new sb_ctx;
    c->impl.device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->impl.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete c;
      check_cuda(e, "cudaStreamCreateWithFlags");
    }
    c->impl.own_stream = true;
    const char* tr = std::getenv("SPARSEB_TRACE");
    c->impl.trace = tr && tr[0] && tr[0] != '0';
    if (const char* gt = std::getenv("SPARSEB_GEMM_TILE")) {
      const std::string v(gt);
      if (v == "64x64") c->impl.gemm_tile = 0;
      else if (v == "128x32") c->impl.gemm_tile = 1;
      else if (v == "32x128") c->impl.gemm_tile = 2;
      else if (v == "128x64") c->impl.gemm_tile = 3;
      else if (v == "64x128") c->impl.gemm_tile = 4;
      else if (v == "64x32") c->impl.gemm_tile = 5;
    }
    if (const char* th = std::getenv("SPARSEB_GEMM_THIN")) c->impl.gemm_thin = std::atoi(th);
    if (const char* ge = std::getenv("SPARSEB_GEMM_EDGES")) c->impl.gemm_edges = std::atoi(ge);
    if (const char* pc = std::getenv("SPARSEB_PLAN_CACHE")) c->impl.plan_cache_on = std::atoi(pc) != 0;
    if (const char* ac = std::getenv("SPARSEB_AUTO_CROP")) c->impl.auto_crop = std::atoi(ac);
    if (const char* sk = std::getenv("SPARSEB_GEMM_SPLITK")) c->impl.gemm_splitk = std::max(0, std::atoi(sk));
    if (const char* kc = std::getenv("SPARSEB_TC_KC")) c->impl.tc_kc = std::max(1, std::atoi(kc));
    if (const char* po = std::getenv("SPARSEB_POISON_OUTPUT")) c->impl.poison_output = std::atoi(po) != 0;
    if (const char* at = std::getenv("SPARSEB_AUTOTUNE")) c->impl.autotune = std::atoi(at) != 0;
    // Keep freed device memory cached in the stream-ordered pool.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = c;
  });
}

sb_status sb_ctx_destroy(sb_ctx* ctx) {
  if (!ctx) return SB_OK;
  if (ctx->impl.live_tensors > 0) {
    ctx->impl.destroy_pending = true;  // the last sb_tensor_free finishes the job
    return SB_OK;
  }
  destroy_ctx_now(ctx);
  return SB_OK;
}

const char* sb_last_error(const sb_ctx* ctx) { return ctx ? ctx->impl.last_error.c_str() : g_noctx_error.c_str(); }

sb_status sb_ctx_set_stream(sb_ctx* ctx, void* stream) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    SB_CK(cudaSetDevice(ctx->impl.device));
    SB_CK(cudaStreamSynchronize(ctx->impl.stream));
    ctx->impl.release_staging();
    if (ctx->impl.own_stream) cudaStreamDestroy(ctx->impl.stream);
    ctx->impl.stream = static_cast<cudaStream_t>(stream);
    ctx->impl.own_stream = false;
  });
}

void* sb_ctx_get_stream(const sb_ctx* ctx) { return ctx ? static_cast<void*>(ctx->impl.stream) : nullptr; }

sb_status sb_ctx_synchronize(sb_ctx* ctx) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    ctx->impl.sync();
    check_tc_status(ctx);
  });
}

sb_status sb_ctx_set_precision(sb_ctx* ctx, int precision) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(precision == SB_PRECISION_F64 || precision == SB_PRECISION_TF32X3 || precision == SB_PRECISION_TF32,
            SB_ERR_INVALID_ARG, "unknown precision");
    require(!ctx->impl.capturing, SB_ERR_INVALID_ARG, "precision cannot change while a capture is open");
    SB_CK(cudaSetDevice(ctx->impl.device));
    if (precision != SB_PRECISION_F64 && !ctx->impl.tc_status.raw()) {
      ctx->impl.tc_status = sb::DevBuf(&ctx->impl, sizeof(int));
      SB_CK(cudaMemsetAsync(ctx->impl.tc_status.raw(), 0, sizeof(int), ctx->impl.stream));
    }
    ctx->impl.precision = precision;
  });
}

int sb_ctx_get_precision(const sb_ctx* ctx) { return ctx ? ctx->impl.precision : -1; }

int64_t sb_ctx_launch_count(const sb_ctx* ctx) { return ctx ? ctx->impl.launches : 0; }

sb_status sb_ctx_set_profiling(sb_ctx* ctx, int enable) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    SB_CK(cudaSetDevice(ctx->impl.device));
    ctx->impl.sync();
    ctx->impl.clear_profile();
    ctx->impl.profiling = enable != 0;
  });
}

sb_status sb_ctx_profile_summary(sb_ctx* ctx, int kind, int64_t* launches, double* total_ms, double* flops,
                                 double* bytes) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(kind >= 0 && kind < PROF_NKINDS, SB_ERR_INVALID_ARG, "unknown kernel class");
    SB_CK(cudaSetDevice(ctx->impl.device));
    ctx->impl.sync();
    int64_t n = 0;
    double ms = 0.0, f = 0.0, b = 0.0;
    for (auto& r : ctx->impl.prof) {
      if (r.kind != kind) continue;
      float e = 0.f;
      SB_CK(cudaEventElapsedTime(&e, r.a, r.b));
      ++n;
      ms += e;
      f += r.flops;
      b += r.bytes;
    }
    if (launches) *launches = n;
    if (total_ms) *total_ms = ms;
    if (flops) *flops = f;
    if (bytes) *bytes = b;
  });
}

sb_status sb_tensor_create_dense(sb_ctx* ctx, int nd, const int64_t* dims, const double* data, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto t = make_tensor(&ctx->impl, DENSE, read_dims(nd, dims), nd);
    const int64_t n = t->numel();
    t->data = DevBuf(&ctx->impl, n * sizeof(double));
    if (data) SB_CK(cudaMemcpyAsync(t->data.raw(), data, n * sizeof(double), cudaMemcpyHostToDevice, ctx->impl.stream));
    else SB_CK(cudaMemsetAsync(t->data.raw(), 0, n * sizeof(double), ctx->impl.stream));
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_create_dense_device(sb_ctx* ctx, int nd, const int64_t* dims, const double* d_data, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr && d_data != nullptr, SB_ERR_INVALID_ARG, "out or d_data is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto t = make_tensor(&ctx->impl, DENSE, read_dims(nd, dims), nd);
    const int64_t n = t->numel();
    t->data = DevBuf(&ctx->impl, n * sizeof(double));
    SB_CK(cudaMemcpyAsync(t->data.raw(), d_data, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->impl.stream));
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_create_bs(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail, int64_t nblocks, const int64_t* keys,
                              const int64_t* ids, const double* data, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto d = read_dims(nd, dims);
    require((nd == 0 && n_tail == 0) || (n_tail > 0 && n_tail <= nd), SB_ERR_ASSERTION, "0 < N2 <= N required");
    require(nblocks >= 0, SB_ERR_INVALID_ARG, "nblocks < 0");
    require(nblocks == 0 || (keys && data) || (nd - n_tail == 0 && data), SB_ERR_INVALID_ARG, "keys/data NULL");
    Ctx* c = &ctx->impl;
    auto t = make_tensor(c, BS, d, n_tail);
    const int P = t->P();
    const int64_t blk = t->blksize();
    std::vector<int64_t> k(nblocks * P);
    if (P) std::copy(keys, keys + nblocks * P, k.begin());
    check_keys_in_range(k, nblocks, P, d);
    std::vector<int64_t> lin(nblocks), p(nblocks);
    for (int64_t i = 0; i < nblocks; ++i) lin[i] = lin0(&k[i * P], d.data(), P);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
    for (int64_t i = 1; i < nblocks; ++i) require(lin[p[i]] != lin[p[i - 1]], SB_ERR_ASSERTION, "duplicate block key");
    std::vector<int64_t> src_off(nblocks);
    for (int64_t i = 0; i < nblocks; ++i) {
      const int64_t id = ids ? ids[p[i]] : p[i] + 1;
      require(id >= 1 && id <= nblocks, SB_ERR_ASSERTION, "block id out of range");
      src_off[i] = (id - 1) * blk;
    }
    t->keys.resize(nblocks * P);
    for (int64_t i = 0; i < nblocks; ++i) std::copy(&k[p[i] * P], &k[p[i] * P] + P, &t->keys[i * P]);
    t->nkeys = nblocks;
    t->data = DevBuf(c, nblocks * blk * sizeof(double));
    if (nblocks) {
      DevBuf raw(c, nblocks * blk * sizeof(double));
      SB_CK(cudaMemcpyAsync(raw.raw(), data, nblocks * blk * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      bool packed = true;
      for (int64_t i = 0; i < nblocks; ++i) packed = packed && src_off[i] == i * blk;
      if (packed) {
        t->data = std::move(raw);
      } else {
        std::vector<int64_t> dof(nblocks), len(nblocks, blk);
        for (int64_t i = 0; i < nblocks; ++i) dof[i] = i * blk;
        copy_blocks(c, raw.d(), t->data.d(), src_off, dof, len);
      }
    }
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_create_bs_ragged(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail, int64_t nblocks,
                                     const int64_t* keys, const int64_t* block_dims, const double* data,
                                     sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto d = read_dims(nd, dims);
    require(n_tail > 0 && n_tail <= nd, SB_ERR_ASSERTION, "0 < N2 <= N required");
    require(nblocks >= 0, SB_ERR_INVALID_ARG, "nblocks < 0");
    require(nblocks == 0 || (block_dims && data && (keys || nd == n_tail)), SB_ERR_INVALID_ARG,
            "keys/block_dims/data NULL");
    Ctx* c = &ctx->impl;
    auto t = make_tensor(c, BS, d, n_tail);
    const int P = t->P();
    std::vector<int64_t> k(nblocks * P);
    if (P) std::copy(keys, keys + nblocks * P, k.begin());
    check_keys_in_range(k, nblocks, P, d);
    std::vector<int64_t> lin(nblocks), p(nblocks), in_off(nblocks + 1, 0);
    for (int64_t i = 0; i < nblocks; ++i) {
      lin[i] = lin0(&k[i * P], d.data(), P);
      int64_t len = 1;
      for (int r = 0; r < n_tail; ++r) {
        const int64_t e = block_dims[i * n_tail + r];
        require(e >= 1 && e <= d[P + r], SB_ERR_ASSERTION, "block extent must be in 1:dims of its tail axis");
        len *= e;
      }
      in_off[i + 1] = in_off[i] + len;
    }
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
    for (int64_t i = 1; i < nblocks; ++i) require(lin[p[i]] != lin[p[i - 1]], SB_ERR_ASSERTION, "duplicate block key");
    t->ragged = true;
    t->keys.resize(nblocks * P);
    t->bdims.resize(nblocks * n_tail);
    t->boff.assign(nblocks + 1, 0);
    std::vector<int64_t> so(nblocks), dof(nblocks), len(nblocks);
    for (int64_t i = 0; i < nblocks; ++i) {
      std::copy(&k[p[i] * P], &k[p[i] * P] + P, &t->keys[i * P]);
      std::copy(block_dims + p[i] * n_tail, block_dims + (p[i] + 1) * n_tail, &t->bdims[i * n_tail]);
      len[i] = in_off[p[i] + 1] - in_off[p[i]];
      so[i] = in_off[p[i]];
      t->boff[i + 1] = t->boff[i] + len[i];
      dof[i] = t->boff[i];
    }
    t->nkeys = nblocks;
    const int64_t total = in_off[nblocks];
    if (total) {
      DevBuf raw(c, total * sizeof(double));
      SB_CK(cudaMemcpyAsync(raw.raw(), data, total * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      bool sorted = true;
      for (int64_t i = 0; i < nblocks; ++i) sorted = sorted && p[i] == i;
      if (sorted) {
        t->data = std::move(raw);
      } else {
        t->data = DevBuf(c, total * sizeof(double));
        copy_blocks(c, raw.d(), t->data.d(), so, dof, len);
      }
    }
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_block_dims(const sb_tensor* t, int* ragged, int64_t* block_dims, int64_t* payload_len) {
  return guard(t ? t->owner : nullptr, [&] {
    check_t(t);
    const Tensor& x = *t->impl;
    if (ragged) *ragged = x.ragged ? 1 : 0;
    if (payload_len) *payload_len = x.payload_len();
    if (block_dims && x.kind == BS)
      for (int64_t i = 0; i < x.nkeys; ++i)
        for (int r = 0; r < x.n2; ++r) block_dims[i * x.n2 + r] = x.block_dim(i, r);
  });
}

sb_status sb_tensor_to_uniform(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, bs_to_uniform(&ctx->impl, *A->impl));
  });
}

sb_status sb_tensor_to_ragged(sb_ctx* ctx, const sb_tensor* A, const int64_t* block_dims, int check_zero, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr && (block_dims || A->impl->nkeys == 0), SB_ERR_INVALID_ARG, "out/block_dims NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    const Tensor& x = *A->impl;
    std::vector<int64_t> bd(block_dims, block_dims + x.nkeys * x.n2);
    *out = wrap(ctx, bs_to_ragged(&ctx->impl, x, bd, check_zero != 0));
  });
}

sb_status sb_tensor_crop_padding(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, bs_crop_padding(&ctx->impl, *A->impl));
  });
}

sb_status sb_tensor_create_coo(sb_ctx* ctx, int nd, const int64_t* dims, int64_t nnz, const int64_t* keys,
                               const double* vals, int dirty, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto d = read_dims(nd, dims);
    require(nnz >= 0 && (nnz == 0 || (keys && vals)), SB_ERR_INVALID_ARG, "keys/vals NULL");
    auto t = make_tensor(&ctx->impl, COO, d, 0);
    t->keys.assign(keys, keys + nnz * nd);
    check_keys_in_range(t->keys, nnz, nd, d);
    t->nkeys = nnz;
    t->dirty = dirty != 0;
    t->data = DevBuf(&ctx->impl, nnz * sizeof(double));
    if (nnz) SB_CK(cudaMemcpyAsync(t->data.raw(), vals, nnz * sizeof(double), cudaMemcpyHostToDevice, ctx->impl.stream));
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_create_aliased(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail, int64_t n_templates,
                                   const double* templates, int64_t nblocks, const int64_t* keys,
                                   const int64_t* alias_ids, const double* scalars, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto d = read_dims(nd, dims);
    require(n_tail > 0 && n_tail <= nd, SB_ERR_ASSERTION, "0 < N2 <= N required");
    require(n_templates >= 0 && nblocks >= 0, SB_ERR_INVALID_ARG, "negative count");
    require(n_templates == 0 || templates, SB_ERR_INVALID_ARG, "templates NULL");
    require(nblocks == 0 || (keys && alias_ids && scalars), SB_ERR_INVALID_ARG, "keys/alias_ids/scalars NULL");
    Ctx* c = &ctx->impl;
    auto t = make_tensor(c, ALIASED, d, n_tail);
    const int P = t->P();
    const int64_t blk = t->blksize();
    std::vector<int64_t> k(keys, keys + nblocks * P);
    check_keys_in_range(k, nblocks, P, d);
    std::vector<int64_t> lin(nblocks), p(nblocks);
    for (int64_t i = 0; i < nblocks; ++i) lin[i] = lin0(&k[i * P], d.data(), P);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
    for (int64_t i = 1; i < nblocks; ++i) require(lin[p[i]] != lin[p[i - 1]], SB_ERR_ASSERTION, "duplicate block key");
    std::vector<double> sc(nblocks);
    t->keys.resize(nblocks * P);
    t->alias_ids.resize(nblocks);
    for (int64_t i = 0; i < nblocks; ++i) {
      std::copy(&k[p[i] * P], &k[p[i] * P] + P, &t->keys[i * P]);
      t->alias_ids[i] = alias_ids[p[i]];
      require(t->alias_ids[i] >= 1 && t->alias_ids[i] <= n_templates, SB_ERR_ASSERTION, "alias id out of range");
      sc[i] = scalars[p[i]];
    }
    t->nkeys = nblocks;
    t->n_templates = n_templates;
    t->data = DevBuf(c, n_templates * blk * sizeof(double));
    if (n_templates)
      SB_CK(cudaMemcpyAsync(t->data.raw(), templates, n_templates * blk * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    t->scalars = upload(c, sc);
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_free(sb_tensor* t) {
  if (!t) return SB_OK;
  sb_ctx* ctx = t->owner;
  const sb_status st = guard(ctx, [&] {
    if (ctx) SB_CK(cudaSetDevice(ctx->impl.device));
    delete t;
  });
  if (ctx && --ctx->impl.live_tensors == 0 && ctx->impl.destroy_pending) destroy_ctx_now(ctx);
  return st;
}

sb_status sb_tensor_info(const sb_tensor* t, int* kind, int* nd, int64_t* dims, int* n_tail, int64_t* nkeys,
                         int64_t* blksize, int64_t* n_templates, int* dirty) {
  return guard(t ? t->owner : nullptr, [&] {
    check_t(t);
    const Tensor& x = *t->impl;
    if (kind) *kind = x.kind;
    if (nd) *nd = x.N();
    if (dims) std::copy(x.dims.begin(), x.dims.end(), dims);
    if (n_tail) *n_tail = x.n2;
    if (nkeys) *nkeys = x.nkeys;
    if (blksize) *blksize = (x.kind == BS || x.kind == ALIASED) ? x.blksize() : 0;
    if (n_templates) *n_templates = x.n_templates;
    if (dirty) *dirty = x.dirty ? 1 : 0;
  });
}

sb_status sb_tensor_export_bs(sb_ctx* ctx, const sb_tensor* t, int64_t* keys, int64_t* ids, double* data) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(t);
    const Tensor& x = *t->impl;
    require(x.kind == BS, SB_ERR_INVALID_ARG, "not a block-sparse tensor");
    SB_CK(cudaSetDevice(ctx->impl.device));
    if (keys) std::copy(x.keys.begin(), x.keys.end(), keys);
    if (ids)
      for (int64_t i = 0; i < x.nkeys; ++i) ids[i] = i + 1;
    if (data && x.nkeys) {
      if (x.f32) {  // FP32 storage: widened on the host
        std::vector<float> tmp(static_cast<size_t>(x.payload_len()));
        SB_CK(cudaMemcpyAsync(tmp.data(), x.data.raw(), tmp.size() * sizeof(float), cudaMemcpyDeviceToHost,
                              ctx->impl.stream));
        ctx->impl.sync();
        std::copy(tmp.begin(), tmp.end(), data);
      } else {
        SB_CK(cudaMemcpyAsync(data, x.data.raw(), x.payload_len() * sizeof(double), cudaMemcpyDeviceToHost,
                              ctx->impl.stream));
        ctx->impl.sync();
      }
    }
  });
}

sb_status sb_tensor_export_bs_async(sb_ctx* ctx, const sb_tensor* t, int64_t* keys, int64_t* ids, double* data) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(t);
    const Tensor& x = *t->impl;
    require(x.kind == BS, SB_ERR_INVALID_ARG, "not a block-sparse tensor");
    SB_CK(cudaSetDevice(ctx->impl.device));
    if (keys) std::copy(x.keys.begin(), x.keys.end(), keys);
    if (ids)
      for (int64_t i = 0; i < x.nkeys; ++i) ids[i] = i + 1;
    require_f64(x, "sb_tensor_export_bs_async");
    if (data && x.nkeys)
      SB_CK(cudaMemcpyAsync(data, x.data.raw(), x.payload_len() * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->impl.stream));
  });
}

sb_status sb_tensor_create_bs_f32(sb_ctx* ctx, int nd, const int64_t* dims, int n_tail, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    auto d = read_dims(nd, dims);
    require(n_tail > 0 && n_tail <= nd, SB_ERR_ASSERTION, "0 < N2 <= N required");
    auto t = make_tensor(&ctx->impl, BS, d, n_tail);
    t->f32 = true;
    *out = wrap(ctx, std::move(t));
  });
}

sb_status sb_tensor_storage_f32(const sb_tensor* t, int* f32) {
  return guard(t ? t->owner : nullptr, [&] {
    check_t(t);
    if (f32) *f32 = t->impl->f32 ? 1 : 0;
  });
}

// is_dense (src/blocksparse/storage.jl:413-425): every prefix combination has a
// block (no prefix: the one whole-tensor block, at most one key).
sb_status sb_tensor_is_dense(const sb_tensor* t, int* dense) {
  return guard(t ? t->owner : nullptr, [&] {
    check_t(t);
    require(dense != nullptr, SB_ERR_INVALID_ARG, "dense is NULL");
    const Tensor& A = *t->impl;
    if (A.kind == DENSE) {
      *dense = 1;
      return;
    }
    require(A.kind == BS, SB_ERR_UNSUPPORTED_TYPES, "is_dense: block-sparse or dense tensors only");
    if (A.P() == 0) {
      require(A.nkeys <= 1, SB_ERR_ASSERTION, "P=0 means no prefix, so at most one block (the whole tensor) is allowed");
      *dense = 1;
      return;
    }
    int64_t combos = 1;
    for (int i = 0; i < A.P(); ++i) combos *= A.dims[i];
    *dense = A.nkeys == combos ? 1 : 0;
  });
}

sb_status sb_tensor_export_coo(sb_ctx* ctx, const sb_tensor* t, int64_t* keys, double* vals) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(t);
    const Tensor& x = *t->impl;
    require(x.kind == COO, SB_ERR_INVALID_ARG, "not a COO tensor");
    SB_CK(cudaSetDevice(ctx->impl.device));
    if (keys) std::copy(x.keys.begin(), x.keys.end(), keys);
    if (vals && x.nkeys) {
      SB_CK(cudaMemcpyAsync(vals, x.data.raw(), x.nkeys * sizeof(double), cudaMemcpyDeviceToHost, ctx->impl.stream));
      ctx->impl.sync();
    }
  });
}

sb_status sb_tensor_export_aliased(sb_ctx* ctx, const sb_tensor* t, double* templates, int64_t* keys, int64_t* alias_ids,
                                   double* scalars) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(t);
    const Tensor& x = *t->impl;
    require(x.kind == ALIASED, SB_ERR_INVALID_ARG, "not an aliased tensor");
    SB_CK(cudaSetDevice(ctx->impl.device));
    if (keys) std::copy(x.keys.begin(), x.keys.end(), keys);
    if (alias_ids) std::copy(x.alias_ids.begin(), x.alias_ids.end(), alias_ids);
    if (templates && x.n_templates)
      SB_CK(cudaMemcpyAsync(templates, x.data.raw(), x.n_templates * x.blksize() * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->impl.stream));
    if (scalars && x.nkeys)
      SB_CK(cudaMemcpyAsync(scalars, x.scalars.raw(), x.nkeys * sizeof(double), cudaMemcpyDeviceToHost, ctx->impl.stream));
    ctx->impl.sync();
  });
}

sb_status sb_tensor_export_dense(sb_ctx* ctx, const sb_tensor* t, double* data) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(t);
    const Tensor& x = *t->impl;
    require(x.kind == DENSE, SB_ERR_INVALID_ARG, "not a dense tensor");
    require(data != nullptr, SB_ERR_INVALID_ARG, "data is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    SB_CK(cudaMemcpyAsync(data, x.data.raw(), x.numel() * sizeof(double), cudaMemcpyDeviceToHost, ctx->impl.stream));
    ctx->impl.sync();
  });
}

sb_status sb_tensor_device_data(const sb_tensor* t, double** d_ptr, int64_t* len) {
  return guard(t ? t->owner : nullptr, [&] {
    check_t(t);
    t->impl->version = next_version();  // the caller may write through the pointer
    if (d_ptr) *d_ptr = t->impl->data.d();
    if (len) *len = t->impl->payload_len();
  });
}

sb_status sb_contract(sb_ctx* ctx, sb_tensor* C, const uint64_t* labelsC, int nC, const sb_tensor* A,
                      const uint64_t* labelsA, int nA, const sb_tensor* B, const uint64_t* labelsB, int nB) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(C);
    check_t(A);
    check_t(B);
    SB_CK(cudaSetDevice(ctx->impl.device));
    const auto t0 = std::chrono::steady_clock::now();
    ctx->impl.gemm_desc[0] = '\0';
    ctx->impl.plan_cache_hit = false;
    ctx->impl.auto_cropped = false;
    contract(&ctx->impl, *C->impl, read_labels(labelsC, nC), *A->impl, read_labels(labelsA, nA), *B->impl,
             read_labels(labelsB, nB));
    if (ctx->impl.trace) {
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      std::fprintf(stderr,
                   "[sparseb] %s  A(kind=%d, keys=%lld) x B(kind=%d, keys=%lld) -> C(keys=%lld)  host %.3f ms%s%s%s%s\n",
                   ctx->impl.kernel_name, A->impl->kind, static_cast<long long>(A->impl->nkeys), B->impl->kind,
                   static_cast<long long>(B->impl->nkeys), static_cast<long long>(C->impl->nkeys), ms,
                   ctx->impl.gemm_desc[0] ? "  gemm: " : "", ctx->impl.gemm_desc,
                   ctx->impl.plan_cache_hit ? "  (cached plan)" : "",
                   ctx->impl.auto_cropped ? "  (zero padding cropped)" : "");
    }
  });
}

sb_status sb_permutedims(sb_ctx* ctx, const sb_tensor* A, const int* perm, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr && (perm != nullptr || A->impl->N() == 0), SB_ERR_INVALID_ARG, "perm/out NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    const Tensor& x = *A->impl;
    std::vector<int> p(perm, perm + x.N());
    TensorPtr r;
    switch (x.kind) {
      case BS: r = bs_permute(&ctx->impl, x, p); break;
      case ALIASED: r = aliased_permute(&ctx->impl, x, p); break;
      case COO: r = coo_permute(&ctx->impl, x, p); break;
      default: {
        std::vector<int> s(p);
        std::sort(s.begin(), s.end());
        for (int i = 0; i < x.N(); ++i) require(s[i] == i + 1, SB_ERR_INVALID_ARG, "perm must be a permutation of 1:N");
        r = dense_permute(&ctx->impl, x, p);
      }
    }
    *out = wrap(ctx, std::move(r));
  });
}

sb_status sb_coo_sort(sb_ctx* ctx, sb_tensor* A) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(A->impl->kind == COO, SB_ERR_INVALID_ARG, "not a COO tensor");
    SB_CK(cudaSetDevice(ctx->impl.device));
    coo_sort(&ctx->impl, *A->impl);
  });
}

sb_status sb_blocksparse_from_dense(sb_ctx* ctx, const sb_tensor* dense, int n_tail, double atol, double rtol, int dropzeros,
                                    sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(dense);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, bs_from_dense(&ctx->impl, *dense->impl, n_tail, atol, rtol, dropzeros != 0));
  });
}

sb_status sb_coo_from_dense(sb_ctx* ctx, const sb_tensor* dense, double atol, double rtol, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(dense);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, coo_from_dense(&ctx->impl, *dense->impl, atol, rtol));
  });
}

sb_status sb_to_dense(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, to_dense(&ctx->impl, *A->impl));
  });
}

sb_status sb_aliased_to_blocksparse(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, aliased_to_bs(&ctx->impl, *A->impl));
  });
}

// ── vector-space operations ────────────────────────────────────────────────

sb_status sb_tensor_norm(sb_ctx* ctx, const sb_tensor* A, double* out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = tensor_norm(&ctx->impl, *A->impl);
  });
}

sb_status sb_tensor_dot(sb_ctx* ctx, const sb_tensor* A, const sb_tensor* B, double* out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    check_t(B);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = tensor_dot(&ctx->impl, *A->impl, *B->impl);
  });
}

sb_status sb_tensor_copy(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, copy_tensor(&ctx->impl, *A->impl));
  });
}

sb_status sb_tensor_similar(sb_ctx* ctx, const sb_tensor* A, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, tensor_similar(&ctx->impl, *A->impl));
  });
}

sb_status sb_tensor_scale(sb_ctx* ctx, sb_tensor* A, double alpha) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    SB_CK(cudaSetDevice(ctx->impl.device));
    A->impl->version = next_version();
    tensor_scale(&ctx->impl, *A->impl, alpha);
  });
}

sb_status sb_tensor_fill(sb_ctx* ctx, sb_tensor* A, double x) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    SB_CK(cudaSetDevice(ctx->impl.device));
    A->impl->version = next_version();
    tensor_fill(&ctx->impl, *A->impl, x);
  });
}

sb_status sb_tensor_map(sb_ctx* ctx, sb_tensor* R, const sb_tensor* A, int op, double alpha, double beta) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(R);
    check_t(A);
    SB_CK(cudaSetDevice(ctx->impl.device));
    R->impl->version = next_version();
    tensor_map(&ctx->impl, *R->impl, *A->impl, op, alpha, beta);
  });
}

sb_status sb_tensor_add(sb_ctx* ctx, const sb_tensor* A, const sb_tensor* B, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    check_t(B);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    *out = wrap(ctx, tensor_add(&ctx->impl, *A->impl, *B->impl));
  });
}

// ── block factorisations ───────────────────────────────────────────────────

sb_status sb_blocksparse_left_qr(sb_ctx* ctx, const sb_tensor* A, sb_tensor** Q, sb_tensor** R, int64_t* l_vals,
                                 int64_t* n_l, int64_t* r_vals, int64_t* n_r) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(Q != nullptr && R != nullptr, SB_ERR_INVALID_ARG, "Q/R out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    QrResult r = blocksparse_left_qr(&ctx->impl, *A->impl);
    if (l_vals) std::copy(r.l_vals.begin(), r.l_vals.end(), l_vals);
    if (r_vals) std::copy(r.r_vals.begin(), r.r_vals.end(), r_vals);
    if (n_l) *n_l = static_cast<int64_t>(r.l_vals.size());
    if (n_r) *n_r = static_cast<int64_t>(r.r_vals.size());
    *Q = wrap(ctx, std::move(r.Q));
    *R = wrap(ctx, std::move(r.R));
  });
}

sb_status sb_blocksparse_svd(sb_ctx* ctx, const sb_tensor* A, int ortho_right, int64_t maxdim, int64_t mindim,
                             double cutoff, sb_tensor** U, sb_tensor** SV, double* svs, int64_t svs_capacity,
                             int64_t* n_kept, double* truncerr) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(U != nullptr && SV != nullptr, SB_ERR_INVALID_ARG, "U/SV out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    SvdResult r = blocksparse_svd(&ctx->impl, *A->impl, ortho_right != 0, maxdim, mindim, cutoff);
    const int64_t nk = static_cast<int64_t>(r.svs.size());
    if (svs) std::copy(r.svs.begin(), r.svs.begin() + std::min(nk, std::max<int64_t>(svs_capacity, 0)), svs);
    if (n_kept) *n_kept = nk;
    if (truncerr) *truncerr = r.truncerr;
    *U = wrap(ctx, std::move(r.U));
    *SV = wrap(ctx, std::move(r.SV));
  });
}

sb_status sb_fuse_axes(sb_ctx* ctx, const sb_tensor* A, int ax1, int ax2, sb_tensor** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    check_t(A);
    require(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
    SB_CK(cudaSetDevice(ctx->impl.device));
    const Tensor& x = *A->impl;
    require(x.kind == BS || x.kind == COO, SB_ERR_UNSUPPORTED_TYPES, "fuse: block-sparse or COO tensor expected");
    *out = wrap(ctx, x.kind == BS ? bs_fuse_axes(&ctx->impl, x, ax1, ax2) : coo_fuse_axes(&ctx->impl, x, ax1, ax2));
  });
}

// ── CUDA graph capture ─────────────────────────────────────────────────────

sb_status sb_ctx_capture_begin(sb_ctx* ctx) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    Ctx& c = ctx->impl;
    require(!c.capturing, SB_ERR_INVALID_ARG, "a capture is already open on this context");
    require(!c.profiling, SB_ERR_INVALID_ARG, "switch profiling off before capturing");
    SB_CK(cudaSetDevice(c.device));
    c.sync();  // staged plan uploads of earlier calls are complete
    SB_CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
    c.capturing = true;
    c.capture_keep.clear();
    c.capture_keep_async.clear();
  });
}

sb_status sb_ctx_capture_end(sb_ctx* ctx, sb_graph** out) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    Ctx& c = ctx->impl;
    require(c.capturing, SB_ERR_INVALID_ARG, "no capture is open on this context");
    SB_CK(cudaSetDevice(c.device));
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c.stream, &graph);
    c.capturing = false;
    (void)cudaGetLastError();  // an abandoned capture leaves its error as the last error: clear it
    std::vector<void*> keep, keep_async;
    keep.swap(c.capture_keep);
    keep_async.swap(c.capture_keep_async);
    // buffers released during the capture are freed only now that no graph
    // will read them (the stream is idle: nothing captured ever ran)
    auto drop = [&] {
      if (graph) cudaGraphDestroy(graph);
      for (void* p : keep) cudaFree(p);
      for (void* p : keep_async) cudaFreeAsync(p, c.stream);
    };
    if (e != cudaSuccess || !graph) {
      drop();
      check_cuda(e != cudaSuccess ? e : cudaErrorStreamCaptureInvalidated, "cudaStreamEndCapture");
    }
    if (out == nullptr) {
      drop();
      fail(SB_ERR_INVALID_ARG, "out is NULL");
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    if (ei != cudaSuccess) {
      drop();
      check_cuda(ei, "cudaGraphInstantiate");
    }
    auto* g = new sb_graph;
    g->owner = ctx;
    g->graph = graph;
    g->exec = exec;
    g->keep = std::move(keep);
    g->keep_async = std::move(keep_async);
    ++c.live_tensors;
    *out = g;
  });
}

sb_status sb_graph_launch(sb_ctx* ctx, const sb_graph* g) {
  return guard(ctx, [&] {
    check_ctx(ctx);
    require(g != nullptr && g->exec, SB_ERR_INVALID_ARG, "graph is NULL");
    require(g->owner == ctx, SB_ERR_INVALID_ARG, "graph belongs to another context");
    require(!ctx->impl.capturing, SB_ERR_INVALID_ARG, "cannot launch a graph while capturing");
    SB_CK(cudaSetDevice(ctx->impl.device));
    SB_CK(cudaGraphLaunch(g->exec, ctx->impl.stream));
    ctx->impl.note_launch();
  });
}

sb_status sb_graph_free(sb_graph* g) {
  if (!g) return SB_OK;
  sb_ctx* ctx = g->owner;
  if (ctx) {
    cudaSetDevice(ctx->impl.device);
    cudaStreamSynchronize(ctx->impl.stream);
  }
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (void* p : g->keep) cudaFree(p);
  if (ctx)
    for (void* p : g->keep_async) cudaFreeAsync(p, ctx->impl.stream);
  delete g;
  if (ctx && --ctx->impl.live_tensors == 0 && ctx->impl.destroy_pending) destroy_ctx_now(ctx);
  return SB_OK;
}

}  // extern "C"
