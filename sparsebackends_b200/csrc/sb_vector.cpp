// Vector-space operations on stored tensors: the hooks a Krylov eigensolver
// (KrylovKit's Lanczos, through ITensors) needs from SparseBackends tensors.
//
// Reference: SparseBackends/src/tensor_wrappers.jl:793-923
//   norm        :796-799   norm of the stored values
//   alpha * x   :803-810   new tensor, same keys, values scaled
//   copy        :816-822   deep copy
//   x + y       :825-838   union of block keys, c = copy(x); c[key] += y[key]
//   fill!       :848-851   every stored value set to x
//   map!        :854-868   R[i] = f(R[i], A[i]) over the stored values by
//                          position; lengths must agree
//   similar     :897-918   zeros with the same structure
// and the aliased variants, SparseBackends/src/tensor_wrappers_aliased.jl:
//   norm        :524-536   sqrt(sum_i sum_j (scalars[i] * template[alias_i][j])^2)
//   map!        :538-551   f applied to the per-block scalars
// The inner product is ITensors' dot(x, y) = (dag(x) * y)[], a full
// contraction over all labels, i.e. contract_bs_bs_to_dense!
// (ta/contract_bs_bs.jl:736-754) with P_C = 0: sum over keys present in both
// operands of the block dot products.  Here it is a key merge-join on the host
// and one chunked reduction kernel on the device.
#include <algorithm>
#include <cmath>

#include "sb_internal.hpp"
#include "sb_kernels.hpp"

namespace sb {
namespace {

struct Seg {
  int64_t x_off, y_off, len, s_idx;
};

// Merge contiguous segments, cut into chunks, reduce on the device.
double run_dot(Ctx* ctx, const double* X, const double* Y, const double* S, std::vector<Seg> segs) {
  std::vector<Seg> merged;
  merged.reserve(segs.size());
  for (const Seg& s : segs) {
    if (s.len <= 0) continue;
    if (!merged.empty()) {
      Seg& m = merged.back();
      if (m.s_idx < 0 && s.s_idx < 0 && m.x_off + m.len == s.x_off && m.y_off + m.len == s.y_off) {
        m.len += s.len;
        continue;
      }
    }
    merged.push_back(s);
  }
  std::vector<DotChunk> chunks;
  int64_t total = 0;
  for (const Seg& s : merged) {
    total += s.len;
    for (int64_t b = 0; b < s.len; b += kDotChunk)
      chunks.push_back(DotChunk{s.x_off + b, s.y_off + b, s.s_idx,
                                static_cast<int32_t>(std::min<int64_t>(kDotChunk, s.len - b)), 0});
  }
  DevBuf dc = upload(ctx, chunks);
  DevBuf part(ctx, std::max<size_t>(chunks.size(), 1) * sizeof(double));
  DevBuf out(ctx, sizeof(double));
  {
    ProfScope ps(ctx, PROF_VECTOR, 2.0 * total, 16.0 * total);
    SB_CK(launch_dot_chunks(X, Y, S, dc.as<DotChunk>(), static_cast<int64_t>(chunks.size()), part.d(), out.d(),
                            ctx->stream));
  }
  ctx->note_launch(chunks.empty() ? 0 : 2);
  return download<double>(ctx, out.raw(), 1)[0];
}

void map_values(Ctx* ctx, double* R, const double* A, int64_t n, int op, double alpha, double beta) {
  if (n <= 0) return;
  ProfScope ps(ctx, PROF_VECTOR, 2.0 * n, (A ? 24.0 : 16.0) * n);
  SB_CK(launch_map(R, A, n, op, alpha, beta, ctx->stream));
  ctx->note_launch();
}

// The array that holds a tensor's stored values for map!/fill!/scale, and its length.
std::pair<double*, int64_t> value_array(Tensor& t) {
  if (t.kind == ALIASED) return {t.scalars.d(), t.nkeys};
  return {t.data.d(), t.payload_len()};
}

std::vector<int64_t> key_lins(const Tensor& t) {
  std::vector<int64_t> lin(t.nkeys);
  for (int64_t i = 0; i < t.nkeys; ++i) lin[i] = lin0(t.key(i), t.dims.data(), t.P());
  return lin;
}

void require_same_blocks(const Tensor& A, int64_t ia, const Tensor& B, int64_t ib) {
  for (int t = 0; t < A.n2; ++t)
    require(A.block_dim(ia, t) == B.block_dim(ib, t), SB_ERR_DIM_MISMATCH,
            "blocks with the same key have different extents");
}

}  // namespace

double tensor_dot(Ctx* ctx, const Tensor& A, const Tensor& B) {
  require(A.dims == B.dims, SB_ERR_DIM_MISMATCH, "dot: dims differ");
  if (A.kind == DENSE && B.kind == DENSE)
    return run_dot(ctx, A.data.d(), B.data.d(), nullptr, {Seg{0, 0, A.numel(), -1}});
  require(A.kind == BS && B.kind == BS, SB_ERR_UNSUPPORTED_TYPES,
          "dot: supported for block-sparse x block-sparse and dense x dense");
  require(A.n2 == B.n2, SB_ERR_DIM_MISMATCH, "dot: tail counts differ");
  const auto la = key_lins(A), lb = key_lins(B);
  std::vector<Seg> segs;
  int64_t i = 0, j = 0;
  while (i < A.nkeys && j < B.nkeys) {
    if (la[i] < lb[j]) { ++i; continue; }
    if (lb[j] < la[i]) { ++j; continue; }
    require_same_blocks(A, i, B, j);
    segs.push_back(Seg{A.block_off(i), B.block_off(j), A.block_len(i), -1});
    ++i;
    ++j;
  }
  return run_dot(ctx, A.data.d(), B.data.d(), nullptr, std::move(segs));
}

double tensor_norm(Ctx* ctx, const Tensor& A) {
  if (A.kind == ALIASED) {
    const int64_t blk = A.blksize();
    std::vector<Seg> segs;
    segs.reserve(A.nkeys);
    for (int64_t i = 0; i < A.nkeys; ++i) {
      const int64_t off = (A.alias_ids[i] - 1) * blk;
      segs.push_back(Seg{off, off, blk, i});
    }
    return std::sqrt(run_dot(ctx, A.data.d(), A.data.d(), A.scalars.d(), std::move(segs)));
  }
  const int64_t n = A.payload_len();
  return std::sqrt(run_dot(ctx, A.data.d(), A.data.d(), nullptr, {Seg{0, 0, n, -1}}));
}

void tensor_scale(Ctx* ctx, Tensor& A, double alpha) {
  auto [p, n] = value_array(A);
  map_values(ctx, p, nullptr, n, kMapScale, alpha, 0.0);
}

void tensor_fill(Ctx* ctx, Tensor& A, double x) {
  require(A.kind != ALIASED, SB_ERR_UNSUPPORTED_TYPES, "fill!: not defined for aliased tensors");
  auto [p, n] = value_array(A);
  map_values(ctx, p, nullptr, n, kMapFill, x, 0.0);
}

void tensor_map(Ctx* ctx, Tensor& R, const Tensor& A, int op, double alpha, double beta) {
  require(op == kMapAxpy || op == kMapAxpby || op == kMapCopy || op == kMapMul, SB_ERR_INVALID_ARG,
          "map!: unknown op");
  require(R.kind == A.kind, SB_ERR_UNSUPPORTED_TYPES, "map!: operands of different storage kinds");
  auto [pr, nr] = value_array(R);
  auto [pa, na] = value_array(const_cast<Tensor&>(A));
  require(nr == na, SB_ERR_DIM_MISMATCH, "Mismatched sparsity patterns in map!");
  map_values(ctx, pr, pa, nr, op, alpha, beta);
}

TensorPtr tensor_similar(Ctx* ctx, const Tensor& A) {
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
  if (len) SB_CK(cudaMemsetAsync(out->data.raw(), 0, len * sizeof(double), ctx->stream));
  if (A.kind == ALIASED) {
    out->scalars = DevBuf(ctx, A.nkeys * sizeof(double));
    if (A.nkeys) SB_CK(cudaMemsetAsync(out->scalars.raw(), 0, A.nkeys * sizeof(double), ctx->stream));
  }
  return out;
}

TensorPtr tensor_add(Ctx* ctx, const Tensor& A, const Tensor& B) {
  require(A.dims == B.dims, SB_ERR_DIM_MISMATCH, "+: dims differ");
  if (A.kind == DENSE && B.kind == DENSE) {
    auto out = copy_tensor(ctx, A);
    map_values(ctx, out->data.d(), B.data.d(), A.numel(), kMapAxpy, 1.0, 0.0);
    return out;
  }
  require(A.kind == BS && B.kind == BS, SB_ERR_UNSUPPORTED_TYPES,
          "+: supported for block-sparse + block-sparse and dense + dense");
  require(A.n2 == B.n2, SB_ERR_DIM_MISMATCH, "+: tail counts differ");
  const int P = A.P();
  const auto la = key_lins(A), lb = key_lins(B);
  auto out = make_tensor(ctx, BS, A.dims, A.n2);
  const bool ragged = A.ragged || B.ragged;
  out->ragged = ragged;
  std::vector<AddBlock> items;
  int64_t i = 0, j = 0, off = 0, max_len = 0;
  if (ragged) out->boff.push_back(0);
  auto emit = [&](const Tensor& src, int64_t k, int64_t a_off, int64_t b_off, int64_t len) {
    out->keys.insert(out->keys.end(), src.key(k), src.key(k) + P);
    if (ragged) {
      for (int t = 0; t < src.n2; ++t) out->bdims.push_back(src.block_dim(k, t));
      out->boff.push_back(off + len);
    }
    items.push_back(AddBlock{a_off, b_off, off, len});
    off += len;
    max_len = std::max(max_len, len);
  };
  while (i < A.nkeys || j < B.nkeys) {
    if (j >= B.nkeys || (i < A.nkeys && la[i] < lb[j])) {
      emit(A, i, A.block_off(i), -1, A.block_len(i));
      ++i;
    } else if (i >= A.nkeys || lb[j] < la[i]) {
      emit(B, j, -1, B.block_off(j), B.block_len(j));
      ++j;
    } else {
      require_same_blocks(A, i, B, j);
      emit(A, i, A.block_off(i), B.block_off(j), A.block_len(i));
      ++i;
      ++j;
    }
  }
  out->nkeys = static_cast<int64_t>(items.size());
  out->data = DevBuf(ctx, off * sizeof(double));
  if (!items.empty()) {
    DevBuf di = upload(ctx, items);
    ProfScope ps(ctx, PROF_VECTOR, static_cast<double>(off), 24.0 * off);
    SB_CK(launch_add_blocks(A.data.d(), B.data.d(), out->data.d(), di.as<AddBlock>(),
                            static_cast<int64_t>(items.size()), max_len, ctx->stream));
    ctx->note_launch();
  }
  return out;
}

}  // namespace sb
