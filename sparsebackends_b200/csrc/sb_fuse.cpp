// Axis fusion (link fusion after MPO x MPO contractions).
//
// fuse_two_axes! (src/blocksparse/conversions.jl:228-314):
//   * two prefix axes a1 < a2 (fuse_sparse_axes, :228-262): the fused key is
//     (k[a2] - 1) * d1 + k[a1] at position a1 (a1 the fast index), axis a2
//     dropped; blocks unchanged.  The reference keeps the old key order, which
//     is the sorted order only when a2 = a1 + 1; here the keys are re-sorted
//     (blocks follow) so the sorted-key invariant always holds.
//   * two tail axes (fuse_dense_axes!, :264-296): if they are not adjacent,
//     the tail is permuted first so that the later one directly follows the
//     earlier one (stable move, _move_to_after!); the two adjacent axes then
//     fold into one (the block memory is unchanged, column-major).
//   * one prefix and one tail axis: ArgumentError.
// fuse_axes_coo (src/coo/conversions.jl:174-222): adjacent axes only; the
//   kept axis ax1 is the fast index: fused = (c[ax2] - 1) * d[ax1] + c[ax1] at
//   position ax1 - (ax2 < ax1); the result is sorted (sort!, column-major).
#include <algorithm>
#include <numeric>

#include "sb_internal.hpp"
#include "sb_kernels.hpp"

namespace sb {

TensorPtr bs_fuse_axes(Ctx* ctx, const Tensor& A, int ax1, int ax2) {
  const int N = A.N(), P = A.P();
  require(ax1 >= 1 && ax1 <= N && ax2 >= 1 && ax2 <= N, SB_ERR_INVALID_ARG, "axes must be in 1:N");
  require(ax1 != ax2, SB_ERR_INVALID_ARG, "axes must be distinct");
  const bool s1 = ax1 <= P, s2 = ax2 <= P;
  require(s1 == s2, SB_ERR_INVALID_ARG, "Cannot fuse across sparse-head and dense-tail axes");
  const int a1 = std::min(ax1, ax2), a2 = std::max(ax1, ax2);
  if (s1) {
    const int64_t d1 = A.dims[a1 - 1], d2 = A.dims[a2 - 1];
    std::vector<int64_t> nd;
    for (int i = 1; i <= N; ++i) {
      if (i == a2) continue;
      nd.push_back(i == a1 ? d1 * d2 : A.dims[i - 1]);
    }
    const int Pn = P - 1;
    auto out = make_tensor(ctx, BS, nd, A.n2);
    const int64_t n = A.nkeys;
    std::vector<int64_t> nk(n * Pn), lin(n);
    for (int64_t i = 0; i < n; ++i) {
      const int64_t* k = A.key(i);
      int t = 0;
      for (int j = 1; j <= P; ++j) {
        if (j == a2) continue;
        nk[i * Pn + t++] = j == a1 ? (k[a2 - 1] - 1) * d1 + k[a1 - 1] : k[j - 1];
      }
      lin[i] = lin0(&nk[i * Pn], nd.data(), Pn);
    }
    std::vector<int64_t> p(n);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int64_t x, int64_t y) { return lin[x] < lin[y]; });
    out->nkeys = n;
    out->keys.resize(n * Pn);
    out->ragged = A.ragged;
    if (A.ragged) out->boff.assign(n + 1, 0);
    std::vector<int64_t> so(n), dof(n), ln(n);
    int64_t off = 0;
    for (int64_t i = 0; i < n; ++i) {
      std::copy(&nk[p[i] * Pn], &nk[p[i] * Pn] + Pn, &out->keys[i * Pn]);
      if (A.ragged) {
        for (int r = 0; r < A.n2; ++r) out->bdims.push_back(A.block_dim(p[i], r));
        out->boff[i + 1] = out->boff[i] + A.block_len(p[i]);
      }
      so[i] = A.block_off(p[i]);
      dof[i] = off;
      ln[i] = A.block_len(p[i]);
      off += ln[i];
    }
    out->data = DevBuf(ctx, std::max<int64_t>(off, 1) * sizeof(double));
    copy_blocks(ctx, A.data.d(), out->data.d(), so, dof, ln);
    return out;
  }
  require_uniform(A, "fuse_two_axes! (tail axes)");
  const int N2 = A.n2;
  const int p1 = a1 - P, p2 = a2 - P;  // 1-based tail positions
  TensorPtr B;
  if (p2 != p1 + 1) {
    std::vector<int> pb(N2);
    std::iota(pb.begin(), pb.end(), 1);
    const int x = pb[p2 - 1];  // move the element at p2 to position p1 + 1 (stable)
    pb.erase(pb.begin() + (p2 - 1));
    pb.insert(pb.begin() + p1, x);
    std::vector<int> perm(N);
    std::iota(perm.begin(), perm.end(), 1);
    for (int i = 0; i < N2; ++i) perm[P + i] = P + pb[i];
    B = bs_permute(ctx, A, perm);
  } else {
    B = copy_tensor(ctx, A);
  }
  std::vector<int64_t> nd;
  for (int i = 1; i <= N; ++i) {
    if (i == a1 + 1) continue;
    nd.push_back(i == a1 ? B->dims[a1 - 1] * B->dims[a1] : B->dims[i - 1]);
  }
  B->dims = nd;
  B->n2 = N2 - 1;
  return B;
}

TensorPtr coo_fuse_axes(Ctx* ctx, const Tensor& A, int ax1, int ax2) {
  const int N = A.N();
  require(ax1 != ax2, SB_ERR_INVALID_ARG, "ax1 and ax2 must be distinct");
  require(ax1 >= 1 && ax1 <= N && ax2 >= 1 && ax2 <= N, SB_ERR_INVALID_ARG, "axis out of bounds");
  require(std::abs(ax1 - ax2) == 1, SB_ERR_ASSERTION, "Currently only adjacent axes can be fused");
  const int64_t dkeep = A.dims[ax1 - 1];
  const int ax1_out = ax1 - (ax2 < ax1 ? 1 : 0);
  auto old_axis = [&](int j) { return j < ax2 ? j : j + 1; };
  std::vector<int64_t> nd(N - 1);
  for (int j = 1; j <= N - 1; ++j) nd[j - 1] = j == ax1_out ? dkeep * A.dims[ax2 - 1] : A.dims[old_axis(j) - 1];
  auto out = copy_tensor(ctx, A);
  out->dims = nd;
  out->keys.assign(A.nkeys * (N - 1), 0);
  for (int64_t i = 0; i < A.nkeys; ++i) {
    const int64_t* c = A.key(i);
    for (int j = 1; j <= N - 1; ++j)
      out->keys[i * (N - 1) + j - 1] = j == ax1_out ? (c[ax2 - 1] - 1) * dkeep + c[ax1 - 1] : c[old_axis(j) - 1];
  }
  out->dirty = true;
  coo_sort(ctx, *out);
  return out;
}

}  // namespace sb
