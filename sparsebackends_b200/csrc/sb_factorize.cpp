// Block factorisations of SparseBackends (src/ops_factorize.jl) on the device.
//
// blocksparse_left_qr (ops_factorize.jl:8-43): A[(l, r) | s] -> M with
//   M[(li-1)*d_s + s, ri] = A[l_vals[li], r_vals[ri]][s] over the sorted distinct
//   l and r values of the keys, thin QR M = Q R (k = min(rows, cols)), and
//   Q as a block-sparse tensor (l | s, b) with one block for every l value
//   (setindex! creates it, storage.jl:114-124).  Householder QR on the device.
// blocksparse_svd (ops_factorize.jl:50-148): A[(L, R) | s1, s2] grouped by L;
//   per group M_L = [A[L, R_1] ... A[L, R_n]] as d_s1 x (n * d_s2), SVD of every
//   group (batched one-sided Jacobi, one CTA per group), then the global
//   truncation: singular values sorted decreasing (stable), keep
//   min(maxdim, total), then drop while count > mindim and sv < cutoff*max_sv,
//   truncerr = sum of the dropped sv^2; per group the first k_kept columns,
//   new bond indices contiguous per group in L order; U blocks (L, nb) =
//   U_L[:, col] (times sv when ortho = right), SV blocks (nb, R_j) =
//   Vt_L[col, R_j part] (times sv when ortho = left).
// The index bookkeeping (distinct values, groups, the sort of the singular
// values and the keep counts) is host work, as in the reference; every value
// is computed on the device.
#include <algorithm>
#include <map>
#include <numeric>

#include "sb_internal.hpp"
#include "sb_kernels.hpp"

namespace sb {

namespace {

void gather(Ctx* ctx, const double* src, double* dst, const double* scale, const std::vector<Gather2D>& items) {
  if (items.empty()) return;
  int64_t mx = 0;
  for (const auto& it : items) mx = std::max(mx, it.rows * it.cols);
  DevBuf d = upload(ctx, items);
  ProfScope ps(ctx, PROF_OTHER, 0.0, 0.0);
  SB_CK(launch_gather_2d(src, dst, scale, d.as<Gather2D>(), static_cast<int64_t>(items.size()), mx, ctx->stream));
  ctx->note_launch();
}

}  // namespace

QrResult blocksparse_left_qr(Ctx* ctx, const Tensor& A) {
  require(A.kind == BS, SB_ERR_UNSUPPORTED_TYPES, "blocksparse_left_qr: block-sparse tensor expected");
  require(A.N() == 3 && A.n2 == 1, SB_ERR_UNSUPPORTED_LAYOUT,
          "blocksparse_left_qr: expects N = 3 with prefix (l, r) and dense tail (s)");
  require_uniform(A, "blocksparse_left_qr");
  require(A.nkeys > 0, SB_ERR_INVALID_ARG, "blocksparse_left_qr: tensor has no blocks");
  QrResult out;
  for (int64_t i = 0; i < A.nkeys; ++i) {
    out.l_vals.push_back(A.key(i)[0]);
    out.r_vals.push_back(A.key(i)[1]);
  }
  for (auto* v : {&out.l_vals, &out.r_vals}) {
    std::sort(v->begin(), v->end());
    v->erase(std::unique(v->begin(), v->end()), v->end());
  }
  const int64_t ds = A.dims[2];
  const int64_t nl = static_cast<int64_t>(out.l_vals.size()), nr = static_cast<int64_t>(out.r_vals.size());
  const int64_t m = nl * ds, n = nr, k = std::min(m, n);
  auto pos = [](const std::vector<int64_t>& v, int64_t x) {
    return static_cast<int64_t>(std::lower_bound(v.begin(), v.end(), x) - v.begin());
  };
  // dense M (column-major m x n)
  DevBuf M(ctx, std::max<int64_t>(m * n, 1) * sizeof(double));
  if (m * n) SB_CK(cudaMemsetAsync(M.raw(), 0, m * n * sizeof(double), ctx->stream));
  std::vector<int64_t> so, dof, ln;
  for (int64_t i = 0; i < A.nkeys; ++i) {
    const int64_t li = pos(out.l_vals, A.key(i)[0]), ri = pos(out.r_vals, A.key(i)[1]);
    so.push_back(A.block_off(i));
    dof.push_back(li * ds + ri * m);
    ln.push_back(ds);
  }
  copy_blocks(ctx, A.data.d(), M.d(), so, dof, ln);
  DevBuf tau(ctx, std::max<int64_t>(k, 1) * sizeof(double));
  DevBuf Q(ctx, std::max<int64_t>(m * k, 1) * sizeof(double));
  if (k > 0) {
    ProfScope ps(ctx, PROF_OTHER, 4.0 * m * n * k, 8.0 * m * n);
    int64_t launches = 0;
    SB_CK(launch_householder_qr(M.d(), m, n, tau.d(), ctx->stream, &launches));
    SB_CK(launch_householder_form_q(M.d(), m, k, tau.d(), Q.d(), ctx->stream, &launches));
    ctx->note_launch(launches);
  }
  // R (k x n) dense
  out.R = make_tensor(ctx, DENSE, {k, n}, 2);
  out.R->data = DevBuf(ctx, std::max<int64_t>(k * n, 1) * sizeof(double));
  if (k * n) {
    SB_CK(launch_upper(M.d(), m, k, n, out.R->data.d(), ctx->stream));
    ctx->note_launch();
  }
  // Q as block-sparse (l | s, b): one block per l value, ds x k each
  out.Q = make_tensor(ctx, BS, {A.dims[0], ds, k}, 2);
  std::vector<Gather2D> items;
  for (int64_t li = 0; li < nl && k > 0; ++li) {
    out.Q->keys.push_back(out.l_vals[li]);
    items.push_back(Gather2D{li * ds, li * ds * k, ds, k, 1, m, 1, ds, -1});
  }
  out.Q->nkeys = static_cast<int64_t>(items.size());
  out.Q->data = DevBuf(ctx, std::max<int64_t>(out.Q->nkeys * ds * k, 1) * sizeof(double));
  gather(ctx, Q.d(), out.Q->data.d(), nullptr, items);
  return out;
}

SvdResult blocksparse_svd(Ctx* ctx, const Tensor& A, bool ortho_right, int64_t maxdim, int64_t mindim,
                          double cutoff) {
  require(A.kind == BS, SB_ERR_UNSUPPORTED_TYPES, "blocksparse_svd: block-sparse tensor expected");
  require(A.N() == 4 && A.n2 == 2, SB_ERR_UNSUPPORTED_LAYOUT,
          "blocksparse_svd: expects N = 4 with prefix (L, R) and dense tail (s1, s2)");
  require_uniform(A, "blocksparse_svd");
  const int64_t nL = A.dims[0], nR = A.dims[1], d1 = A.dims[2], d2 = A.dims[3];
  require(d1 <= kSvdMaxRows, SB_ERR_UNSUPPORTED_LAYOUT, "blocksparse_svd: first dense dim exceeds 32");
  require(A.nkeys > 0, SB_ERR_INVALID_ARG, "blocksparse_svd: tensor has no blocks");
  require(maxdim >= 1 && mindim >= 0 && cutoff >= 0.0, SB_ERR_INVALID_ARG,
          "blocksparse_svd: maxdim >= 1, mindim >= 0, cutoff >= 0 required");
  // group keys by L (keys are sorted by L + nL*R, so R ascends within a group)
  std::map<int64_t, std::vector<std::pair<int64_t, int64_t>>> groups;  // L -> [(R, key index)]
  for (int64_t i = 0; i < A.nkeys; ++i) groups[A.key(i)[0]].push_back({A.key(i)[1], i});
  struct G {
    int64_t L, n, a_off, u_off, s_off, k;
    std::vector<int64_t> rlist;
  };
  std::vector<G> gs;
  int64_t aw = 0, uw = 0, sw = 0;
  std::vector<Gather2D> items;
  for (auto& [L, lst] : groups) {
    std::sort(lst.begin(), lst.end());
    G g{L, static_cast<int64_t>(lst.size()) * d2, aw, uw, sw, 0, {}};
    g.k = std::min(d1, g.n);
    for (size_t j = 0; j < lst.size(); ++j) {
      g.rlist.push_back(lst[j].first);
      // M_L[s1, j*d2 + s2] (row-major, row length n) = A block [s1 + s2*d1]
      items.push_back(Gather2D{A.block_off(lst[j].second), g.a_off + static_cast<int64_t>(j) * d2, d1, d2, 1, d1,
                               g.n, 1, -1});
    }
    aw += d1 * g.n;
    uw += d1 * d1;
    sw += d1;
    gs.push_back(std::move(g));
  }
  SvdResult out;
  DevBuf W(ctx, std::max<int64_t>(aw, 1) * sizeof(double)), Vt(ctx, std::max<int64_t>(aw, 1) * sizeof(double));
  DevBuf U(ctx, std::max<int64_t>(uw, 1) * sizeof(double)), S(ctx, std::max<int64_t>(sw, 1) * sizeof(double));
  gather(ctx, A.data.d(), W.d(), nullptr, items);
  std::vector<double> sv(sw);
  if (!gs.empty()) {
    std::vector<SvdGroup> sg;
    for (const G& g : gs) sg.push_back(SvdGroup{g.a_off, g.n, g.u_off, g.s_off, static_cast<int32_t>(d1), 0});
    DevBuf dg = upload(ctx, sg);
    DevBuf st(ctx, sizeof(int));
    SB_CK(cudaMemsetAsync(st.raw(), 0, sizeof(int), ctx->stream));
    {
      ProfScope ps(ctx, PROF_OTHER, 0.0, 16.0 * aw);
      SB_CK(launch_svd_rows(W.d(), Vt.d(), U.d(), S.d(), dg.as<SvdGroup>(), static_cast<int64_t>(sg.size()), 64,
                            st.as<int>(), ctx->stream));
    }
    ctx->note_launch();
    require(download<int>(ctx, st.raw(), 1)[0] == 0, SB_ERR_ASSERTION,
            "blocksparse_svd: Jacobi SVD did not converge in 64 sweeps");
    sv = download<double>(ctx, S.raw(), sw);
  }
  // global truncation (host bookkeeping on the singular values)
  struct SvRef {
    double sv;
    int64_t g, col;
  };
  std::vector<SvRef> all;
  for (size_t gi = 0; gi < gs.size(); ++gi)
    for (int64_t c = 0; c < gs[gi].k; ++c) all.push_back(SvRef{sv[gs[gi].s_off + c], static_cast<int64_t>(gi), c});
  std::stable_sort(all.begin(), all.end(), [](const SvRef& a, const SvRef& b) { return a.sv > b.sv; });
  const double max_sv = all.empty() ? 1.0 : all[0].sv;
  int64_t keep = std::min<int64_t>(maxdim, static_cast<int64_t>(all.size()));
  while (keep > mindim && all[keep - 1].sv < cutoff * max_sv) --keep;
  out.truncerr = 0.0;
  for (size_t i = static_cast<size_t>(keep); i < all.size(); ++i) out.truncerr += all[i].sv * all[i].sv;
  std::vector<int64_t> kk(gs.size(), 0), off(gs.size(), 0);
  for (int64_t i = 0; i < keep; ++i) ++kk[all[i].g];
  int64_t nb = 0;
  for (size_t gi = 0; gi < gs.size(); ++gi) {
    off[gi] = nb;
    nb += kk[gi];
  }
  out.svs.assign(nb, 0.0);
  // U: dims (nL, nb, d1), prefix (L, b), dense s1; keys in nb order are sorted
  out.U = make_tensor(ctx, BS, {nL, nb, d1}, 1);
  out.SV = make_tensor(ctx, BS, {nb, nR, d2}, 1);
  std::vector<Gather2D> ui;
  struct SvItem {
    int64_t lin, b, r;
    Gather2D g;
  };
  std::vector<SvItem> vi;
  for (size_t gi = 0; gi < gs.size(); ++gi) {
    const G& g = gs[gi];
    for (int64_t c = 0; c < kk[gi]; ++c) {
      const int64_t b = off[gi] + c;
      out.svs[b] = sv[g.s_off + c];
      out.U->keys.push_back(g.L);
      out.U->keys.push_back(b + 1);
      ui.push_back(Gather2D{g.u_off + c * d1, b * d1, d1, 1, 1, 0, 1, 0, ortho_right ? g.s_off + c : -1});
      for (size_t j = 0; j < g.rlist.size(); ++j)
        vi.push_back(SvItem{b + nb * (g.rlist[j] - 1), b + 1, g.rlist[j],
                            Gather2D{g.a_off + c * g.n + static_cast<int64_t>(j) * d2, 0, d2, 1, 1, 0, 1, 0,
                                     ortho_right ? -1 : g.s_off + c}});
    }
  }
  out.U->nkeys = nb;
  out.U->data = DevBuf(ctx, std::max<int64_t>(nb * d1, 1) * sizeof(double));
  gather(ctx, U.d(), out.U->data.d(), S.d(), ui);
  std::stable_sort(vi.begin(), vi.end(), [](const SvItem& a, const SvItem& b) { return a.lin < b.lin; });
  std::vector<Gather2D> vg;
  for (size_t i = 0; i < vi.size(); ++i) {
    out.SV->keys.push_back(vi[i].b);
    out.SV->keys.push_back(vi[i].r);
    Gather2D g = vi[i].g;
    g.dst_off = static_cast<int64_t>(i) * d2;
    vg.push_back(g);
  }
  out.SV->nkeys = static_cast<int64_t>(vi.size());
  out.SV->data = DevBuf(ctx, std::max<int64_t>(out.SV->nkeys * d2, 1) * sizeof(double));
  gather(ctx, Vt.d(), out.SV->data.d(), S.d(), vg);
  return out;
}

}  // namespace sb
