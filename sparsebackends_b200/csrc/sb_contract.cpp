// contract!(C, labelsC, A, labelsA, B, labelsB) on the device.
//
// Host side: label analysis, operand permutation plans, merge-join of the
// sorted integer keys into block-pair lists, output key lists (the reference's
// block-creation rules, including the value-dependent ones, whose flags are
// computed on the device).  Device side: every floating-point value.
//
// Function-by-function correspondence (SparseBackends/src/tensoralgebra/):
//   contract()                 contract.jl:37-104
//   prefix_outer_bb()          contract_bs_bs.jl:173-263
//   dense_bb()                 contract_bs_bs.jl:288-423
//   shared_bb()                contract_bs_bs.jl:572-730
//   prefix_outer_bd()          contract_bs_dense.jl:34-204 (Kahan)
//   dense_bd()                 contract_bs_dense.jl:248-392
//   shared_bd()                contract_bs_dense.jl:411-619
//   coo_coo()                  contract_coo.jl:48-170
//   coo_dense()                contract_coo_dense.jl:4-125
//   coo_bs_prefix()            contract_coo_bs.jl:51-124
//   coo_bs_dense_index()       contract_coo_bs.jl:140-241
//   aliased_*()                contract_aliased_coo_dense.jl, contract_aliased.jl,
//                              contract_aliased_shared.jl
//   bs_bs_to_dense()           contract_bs_bs.jl:736-754
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <numeric>
#include <unordered_map>

#include "sb_internal.hpp"

namespace sb {
namespace {

int find(const Labels& l, const Label& x) {
  for (size_t i = 0; i < l.size(); ++i)
    if (l[i] == x) return static_cast<int>(i);
  return -1;
}
bool has(const Labels& l, const Label& x) { return find(l, x) >= 0; }
std::string lab_str(const Label& l) { return "(" + std::to_string(l.id) + "," + std::to_string(l.plev) + ")"; }

int64_t prod(const std::vector<int64_t>& d, int lo, int hi) {
  int64_t p = 1;
  for (int i = lo; i < hi; ++i) p *= d[i];
  return p;
}

// An operand after an optional permutation (owned copy) with its labels.
struct Op {
  const Tensor* t = nullptr;
  TensorPtr owned;
  Labels labels;
  const Tensor& operator*() const { return *t; }
  const Tensor* operator->() const { return t; }
};

Op view(const Tensor& t, const Labels& l) {
  Op o;
  o.t = &t;
  o.labels = l;
  return o;
}

Op permuted(Ctx* ctx, const Op& in, const std::vector<int>& perm) {
  if (is_identity(perm)) {
    Op o;
    o.t = in.t;
    o.labels = in.labels;
    return o;
  }
  Op o;
  switch (in.t->kind) {
    case BS: o.owned = bs_permute(ctx, *in.t, perm); break;
    case ALIASED: o.owned = aliased_permute(ctx, *in.t, perm); break;
    case DENSE: o.owned = dense_permute(ctx, *in.t, perm); break;
    default: o.owned = coo_permute(ctx, *in.t, perm); break;
  }
  o.t = o.owned.get();
  for (int p : perm) o.labels.push_back(in.labels[p - 1]);
  return o;
}

// A block-sparse operand whose permutation moves prefix axes only keeps
// every block's payload as it is: the permuted tensor re-sorts the keys and
// points each block at its payload in the original tensor (no copy, no
// launch).  Other permutations copy as `permuted` does.
Op permuted_keys_only(Ctx* ctx, const Op& in, const std::vector<int>& perm) {
  const Tensor& A = *in.t;
  if (is_identity(perm) || A.kind != BS) return permuted(ctx, in, perm);
  const int N = A.N(), P = A.P();
  for (int r = 0; r < A.n2; ++r)
    if (perm[P + r] != P + r + 1) return permuted(ctx, in, perm);
  check_no_cross_perm(perm, N, P);
  std::vector<int64_t> dims(N);
  for (int j = 0; j < N; ++j) dims[j] = A.dims[perm[j] - 1];
  auto v = make_tensor(ctx, BS, dims, A.n2);
  const int64_t n = A.nkeys;
  std::vector<int64_t> nk(n * P), lin(n), ord(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int j = 0; j < P; ++j) nk[i * P + j] = A.key(i)[perm[j] - 1];
    lin[i] = lin0(&nk[i * P], dims.data(), P);
  }
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
  v->keys.resize(n * P);
  v->voff.resize(n);
  v->nkeys = n;
  v->ragged = A.ragged;
  if (A.ragged) {
    v->bdims.resize(n * A.n2);
    v->boff.assign(n + 1, 0);
  }
  for (int64_t i = 0; i < n; ++i) {
    const int64_t o = ord[i];
    std::copy(&nk[o * P], &nk[o * P] + P, &v->keys[i * P]);
    v->voff[i] = A.block_off(o);
    if (A.ragged) {
      for (int r = 0; r < A.n2; ++r) v->bdims[i * A.n2 + r] = A.block_dim(o, r);
      v->boff[i + 1] = v->boff[i] + A.block_len(o);
    }
  }
  v->vdata = A.payload();
  v->vsrc = &A.owner();
  v->f32 = A.f32;
  Op out;
  out.owned = std::move(v);
  out.t = out.owned.get();
  for (int p : perm) out.labels.push_back(in.labels[p - 1]);
  return out;
}

// _find_permutation_for_tensor (contract_bs_bs.jl:33-45); axisr is 1-based.
std::vector<int> perm_r_last(int P, int N, int axisr) {
  std::vector<int> perm;
  if (axisr <= P) {
    for (int a = 1; a <= P; ++a)
      if (a != axisr) perm.push_back(a);
    perm.push_back(axisr);
    for (int a = P + 1; a <= N; ++a) perm.push_back(a);
  } else {
    for (int a = 1; a <= P; ++a) perm.push_back(a);
    for (int a = P + 1; a <= N; ++a)
      if (a != axisr) perm.push_back(a);
    perm.push_back(axisr);
  }
  return perm;
}

// _permute_r_to_last_prefix (contract_bs_bs.jl:77-95)
Op r_to_last_prefix(Ctx* ctx, const Op& in, const Label& r) {
  const int ax = find(in.labels, r) + 1;
  require(ax >= 1 && ax <= in->P(), SB_ERR_LABEL, "rlab must be in prefix to use prefix kernel");
  if (ax == in->P()) return view(*in.t, in.labels);
  return permuted(ctx, in, perm_r_last(in->P(), in->N(), ax));
}

enum class Mode { AthenB, BthenA, Interleaved };

// _cdense_grouping_and_orders (contract_bs_bs.jl:470-505)
Mode cdense_grouping(const Labels& Cdense, const Labels& keepA, const Labels& keepB, Labels* dkA, Labels* dkB) {
  std::vector<int> origin;
  for (auto& l : Cdense) {
    if (has(keepA, l)) origin.push_back(1);
    else if (has(keepB, l)) origin.push_back(0);
    else fail(SB_ERR_LABEL, "Cdense label " + lab_str(l) + " not found in keepA/keepB");
  }
  int firstA = -1, lastA = -1, firstB = -1, lastB = -1;
  for (int i = 0; i < static_cast<int>(origin.size()); ++i) {
    if (origin[i]) { if (firstA < 0) firstA = i; lastA = i; }
    else { if (firstB < 0) firstB = i; lastB = i; }
  }
  dkA->clear();
  dkB->clear();
  for (auto& l : Cdense) (has(keepA, l) ? dkA : dkB)->push_back(l);
  if (firstB < 0 || firstA < 0) return Mode::AthenB;
  if (lastA < firstB) return Mode::AthenB;
  if (lastB < firstA) return Mode::BthenA;
  return Mode::Interleaved;
}

bool same_set(const Labels& a, const Labels& b) {
  if (a.size() != b.size()) return false;
  for (auto& x : a)
    if (!has(b, x)) return false;
  return true;
}

// Output key collector: contributions arrive in the reference's iteration
// order; C blocks end up sorted by column-major prefix index (the order that
// _ensure_block!'s sorted insertion produces) with per-block contribution
// lists kept in arrival order.
struct CKeys {
  int PC;
  std::vector<int64_t> cdims;
  std::unordered_map<int64_t, int> index;
  std::vector<std::vector<int64_t>> keys;
  std::vector<int64_t> lins;
  std::vector<std::vector<int>> contribs;
  int ncontrib = 0;

  CKeys(const Tensor& C) : PC(C.P()), cdims(C.dims) {}

  int touch(const std::vector<int64_t>& k) {
    const int64_t l = lin0(k.data(), cdims.data(), PC);
    auto it = index.find(l);
    int id;
    if (it == index.end()) {
      id = static_cast<int>(keys.size());
      index.emplace(l, id);
      keys.push_back(k);
      lins.push_back(l);
      contribs.emplace_back();
    } else {
      id = it->second;
    }
    contribs[id].push_back(ncontrib++);
    return id;
  }
  // Sorted order of local ids.
  std::vector<int> order() const {
    std::vector<int> o(keys.size());
    std::iota(o.begin(), o.end(), 0);
    std::sort(o.begin(), o.end(), [&](int a, int b) { return lins[a] < lins[b]; });
    return o;
  }
  // Write sorted keys into C.
  void commit_keys(Tensor& C, const std::vector<int>& ord) const {
    C.keys.clear();
    for (int id : ord) C.keys.insert(C.keys.end(), keys[id].begin(), keys[id].end());
    C.nkeys = static_cast<int64_t>(ord.size());
  }
};

// Overwrite semantics of contract! (every kernel empties C first).  The
// payload buffer is kept when its size does not change: every element of it
// is rewritten by the kernel that follows.
void reset_output(Ctx* ctx, Tensor& C, int64_t nkeys, int64_t payload) {
  C.version = next_version();
  C.keys.clear();
  C.alias_ids.clear();
  C.nkeys = nkeys;
  C.n_templates = 0;
  const size_t esz = C.f32 ? sizeof(float) : sizeof(double);
  if (C.data.bytes() != static_cast<size_t>(payload) * esz) C.data = DevBuf(ctx, payload * esz);
  // SPARSEB_POISON_OUTPUT=1 (tests): every output payload starts as NaN, so
  // an element that no kernel writes cannot pass for a computed value
  if (ctx->poison_output && payload > 0)
    SB_CK(cudaMemsetAsync(C.data.raw(), 0xFF, static_cast<size_t>(payload) * esz, ctx->stream));
  C.scalars.reset();
  C.ragged = false;
  C.bdims.clear();
  C.boff.clear();
}

// ── launch helpers ────────────────────────────────────────────────────────
// A prepared block GEMM: the plan arrays on the device and the launch
// parameters, so that a contraction with an unchanged block structure can be
// launched again without planning or uploads (the plan cache of shared_bb).
struct GemmLaunch {
  enum Kind { NONE, THIN, TILED, EDGES, TC } kind = NONE;
  DevBuf dc, dp, dt, dsplit;
  int32_t ncb = 0;
  int64_t n = 0;  // strips (thin) or tiles
  bool xT = false, yT = false, small_rows = false, persistent = false;
  int small_max = 0, k_max = 0, splitk = 1, bm = 64, bn = 64;
  GemmShape shape = GemmShape::T64x64;
  // tensor-core launches: explicit tile list, tiles [nz_begin, n) are the
  // pair-less C blocks; swap puts Y on the 128-row side; passes 3 or 1
  int32_t nz_begin = 0, nsplits = 0, nparts = 0;
  bool swap = false, fold = false;
  int passes = 3, kc = 16;
  // packed operand images (launch_tc_pack): descriptors of the A side (the
  // 128-row side: Y with swap, else X) and of the B side, per-pair locations,
  // image bytes, and the elements the packing reads
  DevBuf dpk, dimg_a, dimg_b;
  int64_t nimg_a = 0, nimg_b = 0, pack_a_bytes = 0, pack_b_bytes = 0, pack_a_elems = 0, pack_b_elems = 0;
  // the images of the last call, reused while the operand's payload and
  // version are unchanged (an environment across the matvecs of a solve);
  // never inside a graph capture
  mutable DevBuf pk_a, pk_b;
  mutable const void* pk_a_src = nullptr;
  mutable const void* pk_b_src = nullptr;
  mutable uint64_t pk_a_ver = 0, pk_b_ver = 0;
  double flops = 0.0, bytes = 0.0;
  char desc[sizeof(Ctx::gemm_desc)] = "";
  // Tensor-core launch: X and Y FP64 or FP32 arrays (versions 0 = unknown,
  // packed every call), C FP64 or FP32.
  void run_tc(Ctx* ctx, const void* X, bool x64, uint64_t xver, const void* Y, bool y64, uint64_t yver, void* C,
              bool c_f64) const {
    require(ctx->tc_status.raw() != nullptr, SB_ERR_INVALID_ARG, "tensor-core GEMM without a status word");
    std::memcpy(ctx->gemm_desc, desc, sizeof(desc));
    const void* A = swap ? Y : X;
    const void* B = swap ? X : Y;
    const bool a64 = swap ? y64 : x64, b64 = swap ? x64 : y64;
    const uint64_t aver = swap ? yver : xver, bver = swap ? xver : yver;
    DevBuf sa, sb;  // scratch images inside a capture
    auto images = [&](DevBuf& cache, const void*& key, uint64_t& kver, DevBuf& scratch, const void* src, bool f64,
                      uint64_t ver, const DevBuf& imgs, int64_t nimg, int64_t bytes, int64_t elems) -> const void* {
      if (bytes == 0) return nullptr;
      DevBuf* buf = &cache;
      if (ctx->capturing) {
        scratch = DevBuf(ctx, bytes);
        buf = &scratch;
      } else if (ver != 0 && key == src && kver == ver && cache.bytes() == static_cast<size_t>(bytes)) {
        return cache.raw();
      }
      if (!ctx->capturing && cache.bytes() != static_cast<size_t>(bytes)) cache = DevBuf(ctx, bytes);
      {
        ProfScope ps(ctx, PROF_TC_PACK, 0.0,
                     static_cast<double>(elems) * (f64 ? 8 : 4) + static_cast<double>(bytes) / (passes == 3 ? 1 : 2));
        SB_CK(launch_tc_pack(src, f64, imgs.as<TcImage>(), nimg, buf->raw(), passes, ctx->stream));
      }
      ctx->note_launch();
      if (!ctx->capturing) {
        key = src;
        kver = ver;
      }
      return buf->raw();
    };
    const void* pa = images(pk_a, pk_a_src, pk_a_ver, sa, A, a64, aver, dimg_a, nimg_a, pack_a_bytes, pack_a_elems);
    const void* pb = images(pk_b, pk_b_src, pk_b_ver, sb, B, b64, bver, dimg_b, nimg_b, pack_b_bytes, pack_b_elems);
    DevBuf part;  // k-segment partial tiles of split tiles (stream-ordered scratch)
    if (nparts > 0) part = DevBuf(ctx, static_cast<size_t>(nparts) * kTcPartElems * sizeof(double));
    {
      ProfScope ps(ctx, PROF_GEMM_TC, flops, bytes);
      SB_CK(launch_gemm_tc(pa, pb, C, c_f64, dc.as<GemmCBlock>(), dp.as<GemmPair>(), dpk.as<TcPack>(),
                           dt.as<TcTile>(), static_cast<int32_t>(n), nz_begin, swap, passes, kc, fold, part.d(),
                           dsplit.as<TcSplit>(), nsplits, ctx->tc_status.as<int>(), ctx->stream));
    }
    ctx->tc_launched = true;
    ctx->note_launch(nsplits > 0 ? 2 : 1);
  }
  // Operands and result as tensors: FP32-stored tensors (the intermediates of
  // a tensor-core H_eff chain) go to the launches that read or write them;
  // a tensor-core launch packs FP64 and FP32 operands alike.
  void run_io(Ctx* ctx, const Tensor& Xt, const Tensor& Yt, Tensor& Ct) const {
    if (kind == NONE) return;
    if (kind == TC) {
      run_tc(ctx, Xt.payload(), !Xt.f32, Xt.owner().version, Yt.payload(), !Yt.f32, Yt.owner().version,
             Ct.data.raw(), !Ct.f32);
      return;
    }
    if (kind == THIN) {
      const Tensor& lt = small_rows ? Yt : Xt;
      const Tensor& st = small_rows ? Xt : Yt;
      require(lt.f32 == Ct.f32 && !st.f32, SB_ERR_UNSUPPORTED_TYPES,
              "K <= 16 contraction with FP32 storage: the long operand and the result must both be FP32 and "
              "the short operand FP64");
      run(ctx, Xt.payload(), Yt.payload(), Ct.data.d(), lt.f32);
      return;
    }
    require(!Xt.f32 && !Yt.f32 && !Ct.f32, SB_ERR_UNSUPPORTED_TYPES,
            "FP32-stored tensors need a tensor-core precision (sb_ctx_set_precision)");
    run(ctx, Xt.payload(), Yt.payload(), Ct.data.d());
  }
  void run(Ctx* ctx, const double* X, const double* Y, double* C, bool long_f32 = false) const {
    if (kind == NONE) return;
    if (kind == TC) {
      run_tc(ctx, X, true, 0, Y, true, 0, C, true);  // no tensors: packed every call
      return;
    }
    std::memcpy(ctx->gemm_desc, desc, sizeof(desc));
    if (kind == THIN) {
      {
        ProfScope ps(ctx, PROF_GEMM_THIN, flops, bytes);
        SB_CK(launch_gemm_f64_skinny(X, Y, C, dc.as<GemmCBlock>(), ncb, dp.as<GemmPair>(), n, xT, yT, small_rows,
                                     small_max, k_max, ctx->stream, persistent, long_f32));
      }
      ctx->note_launch();
      return;
    }
    DevBuf part;
    const int64_t tile = kind == EDGES ? 64 * 64 : static_cast<int64_t>(bm) * bn;
    if (splitk > 1) part = DevBuf(ctx, static_cast<size_t>(splitk) * n * tile * sizeof(double));
    {
      ProfScope ps(ctx, PROF_GEMM, flops, bytes);
      if (kind == EDGES)
        SB_CK(launch_gemm_f64_edges(X, Y, C, dc.as<GemmCBlock>(), ncb, dp.as<GemmPair>(), n, xT, yT, ctx->stream,
                                    splitk, part.d()));
      else
        SB_CK(launch_gemm_f64(X, Y, C, dc.as<GemmCBlock>(), ncb, dp.as<GemmPair>(), n, xT, yT, shape, ctx->stream,
                              splitk, part.d()));
    }
    ctx->note_launch(splitk > 1 ? 2 : 1);
  }
};

struct GemmPlan {
  std::vector<GemmCBlock> cbs;
  std::vector<GemmPair> pairs;
  int cur = -1;
  void add_cblock(int64_t c_off, int64_t M, int64_t N) {
    require(M < (1LL << 31) && N < (1LL << 31), SB_ERR_INVALID_ARG, "block matrix extent exceeds 2^31");
    cbs.push_back(GemmCBlock{c_off, static_cast<int32_t>(M), static_cast<int32_t>(N),
                             static_cast<int32_t>(pairs.size()), static_cast<int32_t>(pairs.size()), 0, 1,
                             static_cast<int32_t>(M), 0});
  }
  void add_pair(int64_t x_off, int64_t y_off, int64_t K, int64_t ldx, int64_t ldy) {
    require(K < (1LL << 31) && ldx < (1LL << 31) && ldy < (1LL << 31), SB_ERR_INVALID_ARG,
            "block matrix extent exceeds 2^31");
    pairs.push_back(GemmPair{x_off, y_off, static_cast<int32_t>(K), static_cast<int32_t>(ldx),
                             static_cast<int32_t>(ldy), 0});
    cbs.back().pair_end = static_cast<int32_t>(pairs.size());
  }
  void launch(Ctx* ctx, const double* X, const double* Y, double* C, bool xT, bool yT) {
    prepare(ctx, xT, yT).run(ctx, X, Y, C);
  }
  // f32mask: bit 0 = X, bit 1 = Y, bit 2 = C hold FP32 values (FP32-stored
  // tensors); the thin kernel takes them only as its long operand and result.
  GemmLaunch prepare(Ctx* ctx, bool xT, bool yT, int f32mask = 0) {
    GemmLaunch g;
    g.xT = xT;
    g.yT = yT;
    if (cbs.empty()) return g;
    int64_t M = 0, N = 0, Kmax = 0;
    double flops = 0.0, bytes = 0.0;
    for (auto& c : cbs) {
      M = std::max<int64_t>(M, c.M);
      N = std::max<int64_t>(N, c.N);
      bytes += 8.0 * c.M * c.N;
      for (int p = c.pair_begin; p < c.pair_end; ++p) {
        Kmax = std::max<int64_t>(Kmax, pairs[p].K);
        flops += 2.0 * c.M * c.N * pairs[p].K;
        bytes += 8.0 * (static_cast<double>(c.M) + c.N) * pairs[p].K;
      }
    }
    // Thin kernel: every pair K <= 16 and one side <= 16 in every C block
    // (HBM-bound outer-product-like GEMMs, e.g. the MPO steps of H_eff).  It
    // beats the tiled kernel also when some blocks have a short long side
    // (ragged chi=1024 H_eff: 0.11 ms against 0.20 ms per MPO step).
    const bool skinny_n = Kmax <= 16 && N <= 16;
    const bool skinny_m = Kmax <= 16 && M <= 16;
    bool thin_types = true;
    if (f32mask != 0) {  // FP32 values: persistent thin kernel only (it needs a pair in every C block)
      for (auto& c : cbs) thin_types = thin_types && c.pair_end > c.pair_begin;
      const bool long_f32 = (f32mask >> (skinny_m ? 1 : 0)) & 1, short_f32 = (f32mask >> (skinny_m ? 0 : 1)) & 1;
      thin_types = thin_types && long_f32 == ((f32mask >> 2) & 1) && !short_f32 && ctx->gemm_thin != 1;
    }
    if ((skinny_n || skinny_m) && ctx->gemm_tile < 0 && ctx->gemm_thin != 0 && thin_types) {
      const bool small_rows = skinny_m;
      std::vector<int> group;
      const bool interleaved = group_shared_long(small_rows, group);
      bool every_block_has_pairs = true;
      for (auto& c : cbs) every_block_has_pairs = every_block_has_pairs && c.pair_end > c.pair_begin;
      // strips of a group of S blocks: strip s of member j is the group's
      // strip s*S + j; every member carries the group's tile_begin and S in
      // mtiles (the thin kernels find the group's last block and step back)
      int64_t nctas = 0;
      for (size_t i = 0; i < cbs.size();) {
        const int S = group[i];
        const int64_t bigx = small_rows ? cbs[i].N : cbs[i].M;
        for (int j = 0; j < S; ++j) {
          cbs[i + j].tile_begin = static_cast<int32_t>(nctas);
          cbs[i + j].mtiles = S;
        }
        nctas += S * ((bigx + 127) / 128);
        require(nctas < (1LL << 31), SB_ERR_INVALID_ARG, "too many GEMM strips in one launch");
        i += S;
      }
      g.persistent = ctx->gemm_thin != 1 && every_block_has_pairs;
      std::snprintf(g.desc, sizeof(g.desc), "thin%s %s%s", g.persistent ? " persistent" : "",
                    small_rows ? "rows<=16" : "cols<=16", interleaved ? " interleaved" : "");
      g.kind = GemmLaunch::THIN;
      g.dc = upload(ctx, cbs);
      g.dp = upload(ctx, pairs);
      g.ncb = static_cast<int32_t>(cbs.size());
      g.n = nctas;
      g.small_rows = small_rows;
      g.small_max = static_cast<int>(small_rows ? M : N);
      g.k_max = static_cast<int>(Kmax);
      g.flops = flops;
      g.bytes = bytes;
      return g;
    }
    if (ctx->precision != SB_PRECISION_F64) {
      prepare_tc(ctx, g, flops, bytes);
      return g;
    }
    // Tile shape from the FLOP-weighted block shape (ragged launches mix
    // large and small blocks; the heavy ones decide).
    double wm = 0.0, wn = 0.0, wsum = 0.0;
    for (auto& c : cbs) {
      double w = 0.0;
      for (int p = c.pair_begin; p < c.pair_end; ++p) w += static_cast<double>(pairs[p].K);
      w *= static_cast<double>(c.M) * c.N;
      wm += w * c.M;
      wn += w * c.N;
      wsum += w;
    }
    const double am = wsum > 0 ? wm / wsum : static_cast<double>(M), an = wsum > 0 ? wn / wsum : static_cast<double>(N);
    GemmShape shape = GemmShape::T64x64;
    if (an <= 32 && am >= 128) shape = GemmShape::T128x32;
    else if (am <= 32 && an >= 128) shape = GemmShape::T32x128;
    else if (am >= 1024 && an >= 512) shape = am >= an ? GemmShape::T128x64 : GemmShape::T64x128;
    if (shape == GemmShape::T64x64 && ctx->gemm_tile < 0 && ctx->gemm_edges != 0 && prepare_edges(ctx, g, flops, bytes))
      return g;
    if (shape == GemmShape::T64x64) {
      // few 64x64 tiles with long K (the split-K regime): smaller tiles with a
      // deeper pipeline keep more CTAs busy
      int64_t t64 = 0, kt = 0;
      for (auto& c : cbs) {
        const int64_t nt = ((c.M + 63) / 64) * ((c.N + 63) / 64);
        t64 += nt;
        for (int p = c.pair_begin; p < c.pair_end; ++p) kt += nt * ((pairs[p].K + 15) / 16);
      }
      if (t64 < 3 * 148 * 4 && t64 > 0 && kt / t64 >= 64) shape = GemmShape::T64x32;
    }
    if (ctx->gemm_tile >= 0) shape = static_cast<GemmShape>(ctx->gemm_tile);
    int bm, bn;
    gemm_tile_dims(shape, &bm, &bn);
    int64_t ntiles = 0;
    for (auto& c : cbs) {
      const int64_t mt = (c.M + bm - 1) / bm, nt = (c.N + bn - 1) / bn;
      require(ntiles + mt * nt < (1LL << 31), SB_ERR_INVALID_ARG, "too many GEMM tiles in one launch");
      c.tile_begin = static_cast<int32_t>(ntiles);
      c.mtiles = static_cast<int32_t>(mt);
      ntiles += mt * nt;
    }
    // Split-K when the tiles fill few waves of the 148 SMs and each tile has a
    // long K loop (choose_splitk).
    int64_t kt_avg = 0;
    for (auto& c : cbs) {
      int64_t kt = 0;
      for (int p = c.pair_begin; p < c.pair_end; ++p) kt += (pairs[p].K + 15) / 16;
      kt_avg += kt * ((c.M + bm - 1) / bm) * ((c.N + bn - 1) / bn);
    }
    kt_avg = ntiles ? kt_avg / ntiles : 0;
    const int splitk = choose_splitk(ctx, ntiles, kt_avg);
    std::snprintf(g.desc, sizeof(g.desc), "tiled %dx%d sk%d", bm, bn, splitk);
    g.kind = GemmLaunch::TILED;
    g.dc = upload(ctx, cbs);
    g.dp = upload(ctx, pairs);
    g.ncb = static_cast<int32_t>(cbs.size());
    g.n = ntiles;
    g.shape = shape;
    g.bm = bm;
    g.bn = bn;
    g.splitk = splitk;
    g.flops = flops;
    g.bytes = bytes;
    return g;
  }

  // Tensor-core launch (launch_gemm_tc).  Orientation: the side of C that
  // goes to the 128-row tiles pads to a multiple of 128, the other side to a
  // multiple of 16, so the launch takes the orientation with less padded work
  // (ragged H_eff psi*L: the long side N = chi_l' * w to the 128-row tiles).
  // Each C block is cut into 128-row A-side tiles and as few B-side tiles of
  // at most 128 rows as cover it, of equal width rounded up to 16.  When the
  // tiles are too few to keep every SM busy for a balanced share (fewer than
  // four per SM; H_eff R*T3 with its long concatenated K), tiles whose k-tile
  // count exceeds the segment length are cut into k-segments that write FP64
  // partial tiles, summed in order by a reduction launch.  The work items are
  // sorted by work (k-tiles times width), largest first, so that the
  // persistent grid's stride walk gives every SM a similar share.
  void prepare_tc(Ctx* ctx, GemmLaunch& g, double flops, double bytes) {
    auto up = [](int64_t v, int64_t m) { return (v + m - 1) / m * m; };
    double w_keep = 0.0, w_swap = 0.0;
    std::vector<int64_t> kt_of(cbs.size(), 0);  // k-tiles of each C block (its pairs' K ranges concatenated)
    for (size_t c = 0; c < cbs.size(); ++c) {
      for (int p = cbs[c].pair_begin; p < cbs[c].pair_end; ++p) kt_of[c] += (pairs[p].K + 31) / 32;
      w_keep += static_cast<double>(up(cbs[c].M, 128)) * up(cbs[c].N, 16) * kt_of[c];
      w_swap += static_cast<double>(up(cbs[c].N, 128)) * up(cbs[c].M, 16) * kt_of[c];
    }
    const bool swap = w_swap < w_keep;
    struct Geo { int32_t c, a0, b0, nb; };
    std::vector<Geo> geo, zero;
    int64_t total_kt = 0;
    for (size_t c = 0; c < cbs.size(); ++c) {
      const int64_t ma = swap ? cbs[c].N : cbs[c].M, nbx = swap ? cbs[c].M : cbs[c].N;
      const int64_t nbt = (nbx + kTcMaxN - 1) / kTcMaxN, nbs = up((nbx + nbt - 1) / nbt, 16);
      for (int64_t a0 = 0; a0 < ma; a0 += 128)
        for (int64_t j = 0; j < nbt; ++j) {
          const int64_t b0 = j * nbs;
          if (b0 >= nbx) break;
          const Geo t{static_cast<int32_t>(c), static_cast<int32_t>(a0), static_cast<int32_t>(b0),
                      static_cast<int32_t>(std::min(nbs, up(nbx - b0, 16)))};
          (kt_of[c] > 0 ? geo : zero).push_back(t);
          total_kt += kt_of[c];
        }
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const int64_t target = 4LL * sms;
    // segment length in k-tiles; 0 = no splitting (enough tiles already)
    int64_t seg = 0;
    if (static_cast<int64_t>(geo.size()) < target && total_kt > 0)
      seg = std::max<int64_t>(ctx->tc_kc, (total_kt + target - 1) / target);
    // group = (C block, k-segment): its items read the same operand images
    // (A rows for every b0, B rows for every a0) and are kept adjacent, so
    // that consecutive CTAs run them together and the images come from L2
    struct W { TcTile t; int64_t work; int64_t group; };
    std::vector<W> items;
    std::vector<TcSplit> splits;
    int32_t nparts = 0;
    for (const Geo& t : geo) {
      const int64_t kt = kt_of[t.c];
      const int64_t nseg = (seg > 0 && 4 * kt > 5 * seg) ? (kt + seg - 1) / seg : 1;
      int p = cbs[t.c].pair_begin, k0 = 0;  // walk the k-tiles of the C block's pairs
      if (nseg > 1) splits.push_back(TcSplit{t.c, t.a0, t.b0, t.nb, nparts, static_cast<int32_t>(nseg), 0, 0});
      for (int64_t q = 0; q < nseg; ++q) {
        const int64_t kb = kt * q / nseg, ke = kt * (q + 1) / nseg;
        items.push_back(W{TcTile{t.c, t.a0, t.b0, t.nb, p, k0, static_cast<int32_t>(ke - kb),
                                 nseg > 1 ? nparts + static_cast<int32_t>(q) : -1},
                          (ke - kb) * t.nb, (static_cast<int64_t>(t.c) << 32) | q});
        for (int64_t i = kb; i < ke; ++i) {  // advance to k-tile ke
          k0 += 32;
          if (k0 >= pairs[p].K) {
            ++p;
            k0 = 0;
          }
        }
      }
      if (nseg > 1) nparts += static_cast<int32_t>(nseg);
    }
    // heaviest groups first (load balance of the persistent grid), a group's
    // items together
    std::unordered_map<int64_t, int64_t> gwork;
    for (const W& w : items) gwork[w.group] += w.work;
    std::stable_sort(items.begin(), items.end(), [&](const W& a, const W& b) {
      const int64_t wa = gwork[a.group], wb = gwork[b.group];
      return wa != wb ? wa > wb : a.group < b.group;
    });
    std::vector<TcTile> tiles;
    tiles.reserve(items.size() + zero.size());
    for (auto& w : items) tiles.push_back(w.t);
    for (auto& t : zero) tiles.push_back(TcTile{t.c, t.a0, t.b0, t.nb, 0, 0, 0, -1});
    require(tiles.size() < (1ULL << 31), SB_ERR_INVALID_ARG, "too many GEMM tiles in one launch");
    g.kind = GemmLaunch::TC;
    g.dc = upload(ctx, cbs);
    g.dp = upload(ctx, pairs);
    g.dt = upload(ctx, tiles);
    g.dsplit = upload(ctx, splits);
    g.nsplits = static_cast<int32_t>(splits.size());
    g.nparts = nparts;
    g.ncb = static_cast<int32_t>(cbs.size());
    g.n = static_cast<int64_t>(tiles.size());
    g.nz_begin = static_cast<int32_t>(items.size());
    g.swap = swap;
    g.passes = ctx->precision == SB_PRECISION_TF32 ? 1 : 3;
    // chunks: items of at most 2*kc k-tiles run as one chunk each (two
    // accumulators alternate, no running sum); longer items fold chunks of kc
    // k-tiles into a sum kept in TMEM (one accumulator)
    int64_t max_nkt = 1;
    for (const W& w : items) max_nkt = std::max<int64_t>(max_nkt, w.t.nkt);
    g.fold = max_nkt > 2LL * ctx->tc_kc;
    g.kc = g.fold ? ctx->tc_kc : static_cast<int>(max_nkt);
    // packed images: one set per distinct A-side block (128-row tiles) and per
    // distinct B-side block (nbs-row tiles, nbs as in the item geometry), each
    // with the block's k-tiles; a block that several C blocks read is packed once
    {
      const bool akc = swap ? !g.yT : g.xT;  // A side K-contiguous
      const bool bkc = swap ? g.xT : !g.yT;
      std::vector<TcPack> pk(pairs.size(), TcPack{0, 0, 0, 0});
      std::vector<TcImage> ia, ib;
      struct Seen { int64_t base, K, ld; };
      std::unordered_map<int64_t, Seen> sa, sb;
      auto add = [&](std::unordered_map<int64_t, Seen>& seen, std::vector<TcImage>& out, int64_t& total,
                     int64_t& elems, int64_t off, int64_t ld, int64_t K, int64_t rows, int64_t tile, bool kc) -> int64_t {
        auto it = seen.find(off);
        if (it != seen.end()) {
          require(it->second.K == K && it->second.ld == ld, SB_ERR_ASSERTION, "operand block packed twice differently");
          return it->second.base;
        }
        const int64_t base = total, nkt = (K + 31) / 32, plane = tile * 128;
        for (int64_t r0 = 0; r0 < rows; r0 += tile)
          for (int64_t j = 0; j < nkt; ++j) {
            const int64_t k0 = 32 * j;
            out.push_back(TcImage{off + (kc ? r0 * ld + k0 : r0 + k0 * ld), ld, total,
                                  static_cast<int32_t>(std::min(tile, rows - r0)),
                                  static_cast<int32_t>(std::min<int64_t>(32, K - k0)), static_cast<int32_t>(plane),
                                  kc ? 1 : 0});
            elems += std::min(tile, rows - r0) * std::min<int64_t>(32, K - k0);
            total += 2 * plane;
          }
        seen.emplace(off, Seen{base, K, ld});
        return base;
      };
      for (size_t c = 0; c < cbs.size(); ++c) {
        const int64_t ma = swap ? cbs[c].N : cbs[c].M, nbx = swap ? cbs[c].M : cbs[c].N;
        const int64_t nbt = (nbx + kTcMaxN - 1) / kTcMaxN, nbs = up((nbx + nbt - 1) / nbt, 16);
        for (int p = cbs[c].pair_begin; p < cbs[c].pair_end; ++p) {
          const GemmPair& q = pairs[p];
          const int64_t ab = add(sa, ia, g.pack_a_bytes, g.pack_a_elems, swap ? q.y_off : q.x_off,
                                 swap ? q.ldy : q.ldx, q.K, ma, 128, akc);
          const int64_t bb = add(sb, ib, g.pack_b_bytes, g.pack_b_elems, swap ? q.x_off : q.y_off,
                                 swap ? q.ldx : q.ldy, q.K, nbx, nbs, bkc);
          pk[p] = TcPack{ab, bb, static_cast<int32_t>((q.K + 31) / 32), static_cast<int32_t>(nbs)};
        }
      }
      g.dpk = upload(ctx, pk);
      g.dimg_a = upload(ctx, ia);
      g.dimg_b = upload(ctx, ib);
      g.nimg_a = static_cast<int64_t>(ia.size());
      g.nimg_b = static_cast<int64_t>(ib.size());
    }
    g.flops = flops;
    g.bytes = bytes;
    std::snprintf(g.desc, sizeof(g.desc), "tcgen05 %s 128xN%s items:%lld split:%d chunk:%d%s",
                  g.passes == 3 ? "3xtf32" : "tf32", swap ? " swapped" : "", static_cast<long long>(g.n), g.nsplits,
                  g.kc, g.fold ? " fold" : "");
  }

  // Thin launches (K <= 16): output blocks whose pairs read the same block of
  // the long operand (the MPO steps of H_eff, where one T1 block feeds up to
  // two output blocks) are made adjacent in cbs as one group per shared
  // operand set and long extent, and their strips are numbered in turn (strip
  // s of every member, then strip s + 1), so that the reads of one long-operand
  // strip by the group's members follow each other and all but the first hit
  // L2 instead of DRAM.  group[i] = size of the group of cbs[i] (1 when
  // alone).  Returns whether any group has two or more members.
  bool group_shared_long(bool small_rows, std::vector<int>& group) {
    const int n = static_cast<int>(cbs.size());
    std::vector<int> parent(n);
    std::iota(parent.begin(), parent.end(), 0);
    auto root = [&](int c) {
      while (parent[c] != c) c = parent[c] = parent[parent[c]];
      return c;
    };
    std::unordered_map<int64_t, int> user;  // long-operand block offset -> first C block reading it
    bool shared = false;
    for (int c = 0; c < n; ++c)
      for (int p = cbs[c].pair_begin; p < cbs[c].pair_end; ++p) {
        const int64_t off = small_rows ? pairs[p].y_off : pairs[p].x_off;
        auto it = user.emplace(off, c);
        if (it.second) continue;
        const int a = root(c), b = root(it.first->second);
        if (a != b) {
          parent[std::max(a, b)] = std::min(a, b);
          shared = true;
        }
      }
    group.assign(n, 1);
    if (!shared) return false;
    // components in order of their first block; inside one, members of equal
    // long extent form a group (blocks that share operand rows have the same
    // extent, so this splits nothing in practice)
    std::vector<std::vector<int>> comps;
    std::vector<int> comp_of(n, -1);
    for (int c = 0; c < n; ++c) {
      const int r = root(c);
      if (comp_of[r] < 0) {
        comp_of[r] = static_cast<int>(comps.size());
        comps.emplace_back();
      }
      comps[comp_of[r]].push_back(c);
    }
    std::vector<GemmCBlock> nc;
    nc.reserve(cbs.size());
    bool any = false;
    for (auto& comp : comps) {
      auto len = [&](int c) { return small_rows ? cbs[c].N : cbs[c].M; };
      std::stable_sort(comp.begin(), comp.end(), [&](int a, int b) { return len(a) < len(b); });
      for (size_t a = 0; a < comp.size();) {
        size_t b = a;
        while (b < comp.size() && len(comp[b]) == len(comp[a])) ++b;
        for (size_t k = a; k < b; ++k) {
          nc.push_back(cbs[comp[k]]);
          group[nc.size() - 1] = static_cast<int>(b - a);
        }
        any = any || b - a > 1;
        a = b;
      }
    }
    cbs.swap(nc);
    return any;
  }

  // Split-K factor for ntiles tiles averaging kt_avg k-tiles: split while the
  // tiles fill less than ~6 waves of 148 SMs x 4 CTAs and every segment keeps
  // >= 32 k-tiles (6 waves against 3: R*T3 at chi=2048 2.02 -> 1.98 ms ragged,
  // 8.04 -> 7.89 ms zero-padded; the shorter CTAs balance the uneven K loops).
  static int choose_splitk(Ctx* ctx, int64_t ntiles, int64_t kt_avg) {
    int splitk = 1;
    const int64_t wave = 148 * 4;
    while (splitk < 16 && ntiles * splitk < 6 * wave && kt_avg / (2 * splitk) >= 32) splitk *= 2;
    if (ctx->gemm_splitk > 0) splitk = ctx->gemm_splitk;
    return splitk;
  }
  // 64x64 tiles with the edges cut off: a column remainder N mod 64 of <= 32
  // or <= 48 (the whole block when N is that small) goes to 64x32 or 64x48
  // tiles, a row remainder likewise to 32x64 or 48x64 tiles, one launch for
  // all five shapes (ragged sector extents at chi=2048: executed/algorithmic
  // FLOPs 1.109 -> 1.047 on L*psi, 1.165 -> 1.050 on R*T3).  Returns false,
  // launching nothing, when that saves < 3% of the padded 64x64 work.
  static int edge_rows(int shape) { return shape == 2 ? 32 : shape == 4 ? 48 : 64; }
  static int edge_cols(int shape) { return shape == 1 ? 32 : shape == 3 ? 48 : 64; }
  bool prepare_edges(Ctx* ctx, GemmLaunch& g, double flops, double bytes) {
    const bool xT = g.xT, yT = g.yT;
    auto up = [](int64_t v, int64_t t) { return (v + t - 1) / t * t; };
    auto body64 = [](int64_t v) { const int64_t e = v % 64; return e > 0 && e <= 48 ? v - e : v; };
    auto edge = [](int64_t e) -> int64_t { return e <= 32 ? 32 : 48; };
    double w64 = 0.0, wseg = 0.0;
    for (auto& c : cbs) {
      int64_t kt = 0;
      for (int p = c.pair_begin; p < c.pair_end; ++p) kt += (pairs[p].K + 15) / 16;
      kt = std::max<int64_t>(kt, 1);
      const int64_t mm = body64(c.M), nm = body64(c.N);
      w64 += static_cast<double>(up(c.M, 64) * up(c.N, 64)) * kt;
      wseg += static_cast<double>(up(mm, 64) * up(nm, 64) +
                                  (nm < c.N ? up(c.M, 64) * up(c.N - nm, edge(c.N - nm)) : 0) +
                                  (mm < c.M && nm > 0 ? up(c.M - mm, edge(c.M - mm)) * up(nm, 64) : 0)) * kt;
    }
    if (!(wseg < 0.97 * w64)) return false;
    // Sub-blocks of one C block stay adjacent (its tiles run together and
    // share the operand panels in L2: ragged chi=2048 L*psi reads 405 MB
    // instead of 657 MB): body, column edge, row edge.
    std::vector<GemmCBlock> sc;
    std::vector<GemmPair> ep(pairs);
    sc.reserve(cbs.size() * 3);
    int64_t ntiles = 0, kts = 0;
    for (auto& c : cbs) {
      int64_t kt = 0;
      for (int p = c.pair_begin; p < c.pair_end; ++p) kt += (pairs[p].K + 15) / 16;
      const int32_t mm = static_cast<int32_t>(body64(c.M)), nm = static_cast<int32_t>(body64(c.N));
      auto sub = [&](int32_t shape, int32_t r0, int32_t c0, int32_t rows, int32_t cols) {
        const int bm = edge_rows(shape), bn = edge_cols(shape);
        GemmCBlock s{c.c_off + r0 + static_cast<int64_t>(c0) * c.ldc, rows, cols, c.pair_begin, c.pair_end, 0, 0,
                     c.ldc, shape};
        if (r0 != 0 || c0 != 0) {
          s.pair_begin = static_cast<int32_t>(ep.size());
          for (int p = c.pair_begin; p < c.pair_end; ++p) {
            GemmPair q = pairs[p];
            q.x_off += xT ? static_cast<int64_t>(r0) * q.ldx : r0;
            q.y_off += yT ? c0 : static_cast<int64_t>(c0) * q.ldy;
            ep.push_back(q);
          }
          s.pair_end = static_cast<int32_t>(ep.size());
        }
        const int64_t mt = (rows + bm - 1) / bm, ntl = (cols + bn - 1) / bn;
        require(ntiles + mt * ntl < (1LL << 31), SB_ERR_INVALID_ARG, "too many GEMM tiles in one launch");
        s.tile_begin = static_cast<int32_t>(ntiles);
        s.mtiles = static_cast<int32_t>(mt);
        ntiles += mt * ntl;
        kts += mt * ntl * kt;
        sc.push_back(s);
      };
      if (mm > 0 && nm > 0) sub(0, 0, 0, mm, nm);
      if (nm < c.N) sub(c.N - nm <= 32 ? 1 : 3, 0, nm, c.M, c.N - nm);
      if (mm < c.M && nm > 0) sub(c.M - mm <= 32 ? 2 : 4, mm, 0, c.M - mm, nm);
    }
    require(ep.size() < (1ULL << 31), SB_ERR_INVALID_ARG, "too many GEMM block pairs in one launch");
    const int64_t kt_avg = ntiles ? kts / ntiles : 0;
    if (kt_avg >= 64) {
      // Long K loops: the tiles that share an operand panel stream it in
      // step only when they advance at one speed, so tiles of one shape run
      // together: all bodies, then the edges shape by shape (zero-padded
      // chi=2048 R*T3: 8.5 against 14.7 GB read, 7.98 against 8.48 ms).
      std::stable_sort(sc.begin(), sc.end(),
                       [](const GemmCBlock& a, const GemmCBlock& b) { return a.tshape < b.tshape; });
      ntiles = 0;
      for (auto& b : sc) {
        const int64_t bn = edge_cols(b.tshape);
        b.tile_begin = static_cast<int32_t>(ntiles);
        ntiles += static_cast<int64_t>(b.mtiles) * ((b.N + bn - 1) / bn);
      }
    }
    const int splitk = choose_splitk(ctx, ntiles, kt_avg);
    long long nshape[5] = {0, 0, 0, 0, 0};
    for (auto& b : sc) nshape[b.tshape] += static_cast<long long>(b.mtiles) * ((b.N + edge_cols(b.tshape) - 1) /
                                                                                edge_cols(b.tshape));
    std::snprintf(g.desc, sizeof(g.desc), "edges 64x64:%lld 64x32:%lld 32x64:%lld 64x48:%lld 48x64:%lld sk%d",
                  nshape[0], nshape[1], nshape[2], nshape[3], nshape[4], splitk);
    g.kind = GemmLaunch::EDGES;
    g.dc = upload(ctx, sc);
    g.dp = upload(ctx, ep);
    g.ncb = static_cast<int32_t>(sc.size());
    g.n = ntiles;
    g.splitk = splitk;
    g.flops = flops;
    g.bytes = bytes;
    return true;
  }
};

struct OuterPlan {
  std::vector<OuterCBlock> cbs;
  std::vector<OuterPair> pairs;
  int64_t max_elems = 0;
  void add_cblock(int64_t c_off, int64_t M, int64_t N) {
    cbs.push_back(OuterCBlock{c_off, static_cast<int32_t>(M), static_cast<int32_t>(N),
                              static_cast<int32_t>(pairs.size()), static_cast<int32_t>(pairs.size())});
    max_elems = std::max(max_elems, M * N);
  }
  void add_pair(int64_t a_off, int64_t b_off) {
    pairs.push_back(OuterPair{a_off, b_off});
    cbs.back().pair_end = static_cast<int32_t>(pairs.size());
  }
  void launch(Ctx* ctx, const double* A, const double* B, double* C, bool kahan) {
    if (cbs.empty()) return;
    DevBuf dc = upload(ctx, cbs), dp = upload(ctx, pairs);
    double flops = 0.0, bytes = 0.0;
    for (auto& c : cbs) {
      const double np = c.pair_end - c.pair_begin;
      flops += 2.0 * c.M * c.N * np;
      bytes += 8.0 * (static_cast<double>(c.M) * c.N + np * (c.M + c.N));
    }
    {
      ProfScope ps(ctx, PROF_OUTER, flops, bytes);
      SB_CK(launch_outer_acc(A, B, C, dc.as<OuterCBlock>(), static_cast<int64_t>(cbs.size()), dp.as<OuterPair>(),
                             max_elems, kahan, ctx->stream));
    }
    ctx->note_launch();
  }
};

struct AxpyPlan {
  std::vector<AxpySeg> segs;
  std::vector<AxpyEntry> ents;
  int64_t max_len = 0;
  void add_seg(int64_t c_off, int64_t len) {
    segs.push_back(AxpySeg{c_off, len, static_cast<int32_t>(ents.size()), static_cast<int32_t>(ents.size())});
    max_len = std::max(max_len, len);
  }
  void add(int64_t src_off, int64_t alpha_idx) {
    ents.push_back(AxpyEntry{src_off, alpha_idx});
    segs.back().e_end = static_cast<int32_t>(ents.size());
  }
  void launch(Ctx* ctx, const double* src, const double* alpha, double* C) {
    if (segs.empty()) return;
    DevBuf ds = upload(ctx, segs), de = upload(ctx, ents);
    double flops = 0.0, bytes = 0.0;
    for (auto& g : segs) {
      const double ne = g.e_end - g.e_begin;
      flops += 2.0 * g.len * ne;
      bytes += 8.0 * g.len * (1.0 + ne);
    }
    {
      ProfScope ps(ctx, PROF_AXPY, flops, bytes);
      SB_CK(launch_axpy_seg(src, alpha, C, ds.as<AxpySeg>(), static_cast<int64_t>(segs.size()), de.as<AxpyEntry>(),
                            max_len, ctx->stream));
    }
    ctx->note_launch();
  }
};

// Per-(block, slice) nonzero flags of a block-sparse tensor whose reduced
// axis is the last tail axis (_slice_any_nonzero, contract_bs_bs.jl:280-285).
std::vector<uint8_t> slice_flags(Ctx* ctx, const double* data, const std::vector<int64_t>& offs, int64_t R,
                                 int64_t chunk) {
  const int64_t nb = static_cast<int64_t>(offs.size());
  if (nb == 0 || R == 0) return {};
  DevBuf doff = upload(ctx, offs);
  DevBuf fl(ctx, nb * R);
  SB_CK(launch_slice_nonzero(data, doff.as<int64_t>(), nb, R, chunk, fl.as<uint8_t>(), ctx->stream));
  ctx->note_launch();
  return download<uint8_t>(ctx, fl.raw(), nb * R);
}

void check_c_dims(const Tensor& C, const Labels& lC, const Op& A, const Op& B) {
  for (size_t j = 0; j < lC.size(); ++j) {
    int ia = find(A.labels, lC[j]), ib = find(B.labels, lC[j]);
    int64_t d = ia >= 0 ? A->dims[ia] : (ib >= 0 ? B->dims[ib] : -1);
    require(d >= 0, SB_ERR_LABEL, "C label " + lab_str(lC[j]) + " not found in A or B");
    require(d == C.dims[j], SB_ERR_DIM_MISMATCH, "C dim of label " + lab_str(lC[j]) + " does not match the operand");
  }
}

// ══════════════════════════ BS × BS ══════════════════════════════════════

void prefix_outer_bb(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A, const Op& B, const Label& r) {
  ctx->kernel_name = "contract_prefix_outer_bb!";
  const int PA = A->P(), PB = B->P(), PC = C.P();
  Labels Ad(A.labels.begin() + PA, A.labels.end()), Bd(B.labels.begin() + PB, B.labels.end()),
      Cd(lC.begin() + PC, lC.end());
  for (auto& l : Ad) require(!has(Bd, l), SB_ERR_ASSERTION, "outer kernel assumes disjoint dense labels");
  Labels AB(Ad), BA(Bd);
  AB.insert(AB.end(), Bd.begin(), Bd.end());
  BA.insert(BA.end(), Ad.begin(), Ad.end());
  int order;
  if (Cd == AB) order = 1;
  else if (Cd == BA) order = 2;
  else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense must be [A_dense...,B_dense...] or [B_dense..., A_dense...]");
  require(C.blksize() == A->blksize() * B->blksize(), SB_ERR_DIM_MISMATCH, "C.blksize must equal A.blksize * B.blksize");
  std::vector<int> src;
  for (int j = 0; j < PC; ++j) {
    int ia = find(A.labels, lC[j]), ib = find(B.labels, lC[j]);
    if (ia >= 0) src.push_back(ia + 1);
    else { require(ib >= 0, SB_ERR_LABEL, "Label not found in A or B"); src.push_back(-(ib + 1)); }
  }
  CKeys ck(C);
  std::vector<std::pair<int64_t, int64_t>> pr;  // (a block, b block) per contribution
  const int64_t nA = A->nkeys, nB = B->nkeys;
  int64_t iA = 0, iB = 0;
  std::vector<int64_t> k(PC);
  while (iA < nA && iB < nB) {
    const int64_t rvA = A->key(iA)[PA - 1], rvB = B->key(iB)[PB - 1];
    if (rvA < rvB) { while (iA < nA && A->key(iA)[PA - 1] == rvA) ++iA; continue; }
    if (rvB < rvA) { while (iB < nB && B->key(iB)[PB - 1] == rvB) ++iB; continue; }
    const int64_t blo = iB;
    while (iB < nB && B->key(iB)[PB - 1] == rvA) ++iB;
    for (; iA < nA && A->key(iA)[PA - 1] == rvA; ++iA)
      for (int64_t j = blo; j < iB; ++j) {
        for (int q = 0; q < PC; ++q) k[q] = src[q] > 0 ? A->key(iA)[src[q] - 1] : B->key(j)[-src[q] - 1];
        ck.touch(k);
        pr.emplace_back(iA, j);
      }
  }
  auto ord = ck.order();
  const int64_t blkA = A->blksize(), blkB = B->blksize(), blkC = C.blksize();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * blkC);
  ck.commit_keys(C, ord);
  OuterPlan op;
  for (size_t c = 0; c < ord.size(); ++c) {
    if (order == 1) op.add_cblock(static_cast<int64_t>(c) * blkC, blkA, blkB);
    else op.add_cblock(static_cast<int64_t>(c) * blkC, blkB, blkA);
    for (int ci : ck.contribs[ord[c]]) {
      if (order == 1) op.add_pair(pr[ci].first * blkA, pr[ci].second * blkB);
      else op.add_pair(pr[ci].second * blkB, pr[ci].first * blkA);
    }
  }
  if (order == 1) op.launch(ctx, A->data.d(), B->data.d(), C.data.d(), false);
  else op.launch(ctx, B->data.d(), A->data.d(), C.data.d(), false);
}

void dense_bb(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_dense_bb!";
  const int PA = A0->P(), PB = B0->P(), PC = C.P();
  const int axA = find(A0.labels, r) + 1, axB = find(B0.labels, r) + 1;
  require(axA > PA, SB_ERR_LABEL, "rlab must be in A dense tail");
  require(axB > PB, SB_ERR_LABEL, "rlab must be in B dense tail");
  Op A = axA != A0->N() ? permuted(ctx, A0, perm_r_last(PA, A0->N(), axA)) : view(*A0.t, A0.labels);
  Op B = axB != B0->N() ? permuted(ctx, B0, perm_r_last(PB, B0->N(), axB)) : view(*B0.t, B0.labels);
  const int64_t R = A->dims.back();
  require(B->dims.back() == R, SB_ERR_DIM_MISMATCH, "reduction extents differ");
  const int64_t chunkA = A->blksize() / R, chunkB = B->blksize() / R;
  require(C.n2 == (A->n2 - 1) + (B->n2 - 1), SB_ERR_ASSERTION, "N2C must equal (N2A-1)+(N2B-1)");
  require(C.blksize() == chunkA * chunkB, SB_ERR_DIM_MISMATCH, "C.blksize must equal chunkA*chunkB");
  Labels Awo(A.labels.begin() + PA, A.labels.end() - 1), Bwo(B.labels.begin() + PB, B.labels.end() - 1),
      Cd(lC.begin() + PC, lC.end());
  Labels AB(Awo), BA(Bwo);
  AB.insert(AB.end(), Bwo.begin(), Bwo.end());
  BA.insert(BA.end(), Awo.begin(), Awo.end());
  bool ab;
  if (Cd == AB) ab = true;
  else if (Cd == BA) ab = false;
  else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense tail must be [A_dense..., B_dense...] or [B_dense..., A_dense...]");
  std::vector<int> srcA(PC, 0), srcB(PC, 0);
  for (int j = 0; j < PC; ++j) {
    int ia = find(A.labels, lC[j]);
    if (ia >= 0) { require(ia < PA, SB_ERR_LABEL, "C prefix label must come from A prefix"); srcA[j] = ia + 1; }
    else { int ib = find(B.labels, lC[j]); require(ib >= 0 && ib < PB, SB_ERR_LABEL, "C prefix label must come from B prefix"); srcB[j] = ib + 1; }
  }
  const int64_t nA = A->nkeys, nB = B->nkeys, blkA = A->blksize(), blkB = B->blksize();
  std::vector<int64_t> offA(nA), offB(nB);
  for (int64_t i = 0; i < nA; ++i) offA[i] = i * blkA;
  for (int64_t i = 0; i < nB; ++i) offB[i] = i * blkB;
  auto fA = slice_flags(ctx, A->data.d(), offA, R, chunkA);
  auto fB = slice_flags(ctx, B->data.d(), offB, R, chunkB);
  CKeys ck(C);
  std::vector<std::pair<int64_t, int64_t>> pr;
  std::vector<int64_t> k(PC);
  for (int64_t a = 0; a < nA; ++a)
    for (int64_t b = 0; b < nB; ++b) {
      bool any = false;
      for (int64_t s = 0; s < R && !any; ++s) any = fA[a * R + s] && fB[b * R + s];
      if (!any) continue;  // block created only if some r-slice of both is nonzero
      for (int q = 0; q < PC; ++q) k[q] = srcA[q] ? A->key(a)[srcA[q] - 1] : B->key(b)[srcB[q] - 1];
      ck.touch(k);
      pr.emplace_back(a, b);
    }
  auto ord = ck.order();
  const int64_t blkC = C.blksize();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * blkC);
  ck.commit_keys(C, ord);
  GemmPlan gp;
  for (size_t c = 0; c < ord.size(); ++c) {
    if (ab) gp.add_cblock(static_cast<int64_t>(c) * blkC, chunkA, chunkB);
    else gp.add_cblock(static_cast<int64_t>(c) * blkC, chunkB, chunkA);
    for (int ci : ck.contribs[ord[c]]) {
      // AB: C(chunkA x chunkB) = A(chunkA x R) * B(chunkB x R)^T
      if (ab) gp.add_pair(pr[ci].first * blkA, pr[ci].second * blkB, R, chunkA, chunkB);
      else gp.add_pair(pr[ci].second * blkB, pr[ci].first * blkA, R, chunkB, chunkA);
    }
  }
  if (ab) gp.launch(ctx, A->data.d(), B->data.d(), C.data.d(), false, true);
  else gp.launch(ctx, B->data.d(), A->data.d(), C.data.d(), false, true);
}

// Shared-label classification and permutation plan common to the BS and
// aliased multi-label kernels (contract_bs_bs.jl:584-667).
struct SharedPlan {
  Labels shared_prefix, red_dense, dkA, dkB;
  Mode mode;
  std::vector<int> permA, permB;
};

std::vector<int> perm_A_join_dense(const Labels& lA, int PA, const Labels& sp, const Labels& dkA, const Labels& red) {
  std::vector<int> spax, perm;
  for (auto& l : sp) spax.push_back(find(lA, l) + 1);
  for (int a = 1; a <= PA; ++a)
    if (std::find(spax.begin(), spax.end(), a) == spax.end()) perm.push_back(a);
  perm.insert(perm.end(), spax.begin(), spax.end());
  for (auto& l : dkA) perm.push_back(find(lA, l) + 1);
  for (auto& l : red) perm.push_back(find(lA, l) + 1);
  require(static_cast<int>(perm.size()) == static_cast<int>(lA.size()), SB_ERR_ASSERTION, "A perm length mismatch");
  return perm;
}
std::vector<int> perm_B_join_redfirst(const Labels& lB, int PB, const Labels& sp, const Labels& red, const Labels& dkB) {
  std::vector<int> spax, perm;
  for (auto& l : sp) spax.push_back(find(lB, l) + 1);
  for (int a = 1; a <= PB; ++a)
    if (std::find(spax.begin(), spax.end(), a) == spax.end()) perm.push_back(a);
  perm.insert(perm.end(), spax.begin(), spax.end());
  for (auto& l : red) perm.push_back(find(lB, l) + 1);
  for (auto& l : dkB) perm.push_back(find(lB, l) + 1);
  require(static_cast<int>(perm.size()) == static_cast<int>(lB.size()), SB_ERR_ASSERTION, "B perm length mismatch");
  return perm;
}

SharedPlan plan_shared(const Labels& lC, int PC, const Op& A, const Op& B, const Labels& shared, bool B_dense) {
  SharedPlan sp;
  for (auto& l : shared)
    require(!has(lC, l), SB_ERR_LABEL, "shared label " + lab_str(l) + " must be reduced (must not appear in labelsC)");
  const int PA = A->P(), PB = B_dense ? 0 : B->P();
  Labels shared_dense;
  for (auto& l : shared) {
    const int ia = find(A.labels, l), ib = find(B.labels, l);
    require(ia >= 0 && ib >= 0, SB_ERR_LABEL, "shared label must exist in both A and B");
    const bool ap = ia < PA;
    if (B_dense) {
      (ap ? sp.shared_prefix : shared_dense).push_back(l);
    } else {
      const bool bp = ib < PB;
      if (ap && bp) sp.shared_prefix.push_back(l);
      else if (!ap && !bp) shared_dense.push_back(l);
      else fail(SB_ERR_LABEL, "shared label " + lab_str(l) + " crosses prefix/dense; not supported");
    }
  }
  Labels keepA0, keepB0;
  for (int i = PA; i < A->N(); ++i) {
    if (has(shared_dense, A.labels[i])) sp.red_dense.push_back(A.labels[i]);
    else keepA0.push_back(A.labels[i]);
  }
  for (int i = PB; i < B->N(); ++i)
    if (B_dense ? !has(shared, B.labels[i]) : !has(shared_dense, B.labels[i])) keepB0.push_back(B.labels[i]);
  Labels Cd(lC.begin() + PC, lC.end());
  sp.mode = cdense_grouping(Cd, keepA0, keepB0, &sp.dkA, &sp.dkB);
  if (sp.mode == Mode::Interleaved)
    fail(SB_ERR_UNSUPPORTED_LAYOUT, "Cdense interleaves A/B kept dims; would require permuting C (unsupported; sort/fallback)");
  require(same_set(sp.dkA, keepA0) && same_set(sp.dkB, keepB0), SB_ERR_LABEL,
          "C dense labels must be exactly the kept dense labels of A and B");
  sp.permA = perm_A_join_dense(A.labels, PA, sp.shared_prefix, sp.dkA, sp.red_dense);
  if (!B_dense) sp.permB = perm_B_join_redfirst(B.labels, PB, sp.shared_prefix, sp.red_dense, sp.dkB);
  return sp;
}

// Order of two keys on their join tuples.  The operands are permuted so that
// the join axes are the last prefix axes, and keys are sorted column-major,
// so the LAST join axis is the most significant: compare from it down.  (The
// reference's _cmp_join_tuple, contract_bs_bs.jl:430-442, compares the first
// join axis first; with two or more join axes whose value sets differ between
// A and B its merge loses matched pairs.  Where it loses none, both orders
// visit the same runs in the same order.)
int cmp_join(const int64_t* a, const int64_t* b, const std::vector<int>& pa, const std::vector<int>& pb) {
  for (size_t t = pa.size(); t-- > 0;) {
    const int64_t x = a[pa[t] - 1], y = b[pb[t] - 1];
    if (x < y) return -1;
    if (x > y) return 1;
  }
  return 0;
}
int64_t advance_run(const Tensor& T, int64_t i0, const std::vector<int>& pos) {
  const int64_t n = T.nkeys;
  if (pos.empty()) return n;
  int64_t i = i0 + 1;
  while (i < n) {
    bool eq = true;
    for (int p : pos) eq = eq && T.key(i0)[p - 1] == T.key(i)[p - 1];
    if (!eq) break;
    ++i;
  }
  return i;
}

// Merge-join of two key-sorted operands on join positions; calls f(ia, ib)
// for every matched pair in the reference's order (contract_bs_bs.jl:684-728).
template <class F>
void merge_join(const Tensor& A, const std::vector<int>& jA, const Tensor& B, const std::vector<int>& jB, F f) {
  int64_t iA = 0, iB = 0;
  while (iA < A.nkeys && iB < B.nkeys) {
    const int c = cmp_join(A.key(iA), B.key(iB), jA, jB);
    if (c < 0) { iA = advance_run(A, iA, jA); continue; }
    if (c > 0) { iB = advance_run(B, iB, jB); continue; }
    const int64_t iA2 = advance_run(A, iA, jA), iB2 = advance_run(B, iB, jB);
    for (int64_t a = iA; a < iA2; ++a)
      for (int64_t b = iB; b < iB2; ++b) f(a, b);
    iA = iA2;
    iB = iB2;
  }
}

std::vector<int> csrc_AB(const Labels& lC, int PC, const Op& A, const Op& B, bool b_has_prefix) {
  std::vector<int> src;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    const int ib = find(B.labels, lC[j]);
    if (ia >= 0 && ia < A->P()) src.push_back(ia + 1);
    else if (b_has_prefix && ib >= 0 && ib < B->P()) src.push_back(-(ib + 1));
    else fail(SB_ERR_LABEL, "C prefix label " + lab_str(lC[j]) + " must come from A/B prefix");
  }
  return src;
}

// Plan cache of contract_shared! (BS x BS).  An entry holds what a call
// derives from block structure alone: the output keys and layout, and the
// prepared GEMM (plan arrays already on the device).  It is used when the
// labels and both operands' structure (dims, tail count, keys, block extents)
// equal the entry's exactly, as in the H_eff contractions of every Lanczos
// step; nothing in it depends on values.  Not used while a capture is open
// (a graph keeps the buffers allocated during its capture, the cache keeps
// its own).  The 32 most recent structures are kept.
struct SharedPlanEntry {
  std::vector<uint64_t> sig;  // labels of C, A, B; dims and tail counts; flags
  std::vector<int64_t> akeys, abd, bkeys, bbd;
  int64_t c_nkeys = 0, c_payload = 0;
  std::vector<int64_t> c_keys, c_bdims, c_boff;
  bool c_ragged = false;
  GemmLaunch gemm;
};
struct SharedPlanCache {
  std::vector<std::unique_ptr<SharedPlanEntry>> entries;  // most recent last
  static constexpr size_t kMax = 32;
};

std::vector<uint64_t> shared_signature(const Tensor& C, const Labels& lC, const Op& A0, const Op& B0) {
  std::vector<uint64_t> sig;
  auto labels = [&](const Labels& l) {
    sig.push_back(l.size());
    for (auto& x : l) {
      sig.push_back(x.id);
      sig.push_back(x.plev);
    }
  };
  // C contributes only its shape (it is overwritten); the operands also their
  // layout flag and block count (their keys and extents are compared apart)
  auto shape = [&](const Tensor& t, bool operand) {
    sig.push_back(static_cast<uint64_t>(t.kind));
    sig.push_back(t.dims.size());
    for (auto d : t.dims) sig.push_back(static_cast<uint64_t>(d));
    sig.push_back(static_cast<uint64_t>(t.n2));
    if (!operand) return;
    sig.push_back(t.ragged ? 1 : 0);
    sig.push_back(static_cast<uint64_t>(t.nkeys));
  };
  labels(lC);
  labels(A0.labels);
  labels(B0.labels);
  shape(C, false);
  shape(*A0, true);
  shape(*B0, true);
  return sig;
}

// Autotuner of the FP64 tiled block GEMM (SPARSEB_AUTOTUNE=1).  Key: the
// histogram of the pairs' (M, N, K) by powers of two (and the count of pairs
// per bin, also by powers of two) plus the operand order; the same key on a
// later plan reuses the choice.  Candidates: the heuristic's own choice (edge
// tiles included) and every tile shape forced; each runs twice on this call's
// operands (the first run warms it) and the second run is timed with events on
// the context stream.  The chosen launch then writes C once more, so C is what
// that launch computes.
uint64_t histogram_key(const GemmPlan& gp, bool athenb) {
  auto lg = [](int64_t v) { int b = 0; while ((1LL << b) < v) ++b; return b; };
  std::map<std::tuple<int, int, int>, int64_t> h;
  for (const auto& c : gp.cbs)
    for (int p = c.pair_begin; p < c.pair_end; ++p) ++h[{lg(c.M), lg(c.N), lg(gp.pairs[p].K)}];
  uint64_t x = 1469598103934665603ull ^ (athenb ? 1 : 2);
  auto mix = [&](uint64_t v) { x = (x ^ v) * 1099511628211ull; };
  for (const auto& [k, n] : h) {
    mix(static_cast<uint64_t>(std::get<0>(k)));
    mix(static_cast<uint64_t>(std::get<1>(k)));
    mix(static_cast<uint64_t>(std::get<2>(k)));
    mix(static_cast<uint64_t>(lg(n)));
  }
  return x;
}

template <class Run>
GemmLaunch autotune_gemm(Ctx* ctx, const GemmPlan& gp, bool athenb, GemmLaunch g0, Run run_g) {
  const uint64_t key = histogram_key(gp, athenb);
  const int tile0 = ctx->gemm_tile, edges0 = ctx->gemm_edges;
  auto with = [&](int tile, int edges) {
    ctx->gemm_tile = tile;
    ctx->gemm_edges = edges;
    GemmPlan gc = gp;
    GemmLaunch gl = athenb ? gc.prepare(ctx, false, false, 0) : gc.prepare(ctx, true, true, 0);
    ctx->gemm_tile = tile0;
    ctx->gemm_edges = edges0;
    return gl;
  };
  auto it = ctx->tune_table.find(key);
  if (it != ctx->tune_table.end()) {
    if (it->second.first == -2) return g0;  // the heuristic's choice won
    return with(it->second.first, it->second.second);
  }
  cudaEvent_t e0, e1;
  SB_CK(cudaEventCreate(&e0));
  SB_CK(cudaEventCreate(&e1));
  auto time_ms = [&](const GemmLaunch& gl) {
    run_g(gl);
    SB_CK(cudaEventRecord(e0, ctx->stream));
    run_g(gl);
    SB_CK(cudaEventRecord(e1, ctx->stream));
    SB_CK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    SB_CK(cudaEventElapsedTime(&ms, e0, e1));
    return ms;
  };
  float best = time_ms(g0);
  std::pair<int, int> choice{-2, 0};
  GemmLaunch best_g = std::move(g0);
  for (int tile = 0; tile <= 5; ++tile) {  // every shape forced (no edge tiles)
    GemmLaunch gl = with(tile, 0);
    if (gl.kind != GemmLaunch::TILED && gl.kind != GemmLaunch::EDGES) continue;
    const float ms = time_ms(gl);
    if (ms < best) {
      best = ms;
      best_g = std::move(gl);
      choice = {tile, 0};
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->tune_table[key] = choice;
  return best_g;
}

void shared_bb(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Labels& shared);

struct CropScratch {
  DevBuf a, b, c;
};
struct CropScratchMap {
  static constexpr size_t kMax = 8;  // output tensors whose buffers are kept
  std::unordered_map<const Tensor*, CropScratch> m;
};

// Zero padding cropped from uniform operands (the reference layout pads
// every U(1) sector block to the largest sector).  The operands' nonzero
// extents are scanned on the device and made consistent over the block
// pairs: the reduced axes of a matched pair, and each kept axis over all the
// pairs that feed one output block, take one extent, the largest scanned in
// their class (a union-find over (block, axis)).  The operands are cropped to
// these extents, the contraction runs on the ragged blocks and its result is
// padded back into C.  No nonzero entry is cropped, so C equals the uniform
// contraction up to the order in which zero products are (not) added.  Runs
// for compute-heavy contractions only (every GEMM extent >= 32, >= 1e8 padded
// FLOPs) when the cropped work is at most 0.8 of the padded work; never while
// a capture is open (the scan reads extents back to the host).
bool shared_bb_cropped(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Labels& shared) {
  if (ctx->auto_crop <= 0 || ctx->capturing || C.f32 || A0->f32 || B0->f32) return false;
  const Tensor& TA = *A0;
  const Tensor& TB = *B0;
  if (TA.ragged || TB.ragged || C.kind != BS || TA.nkeys == 0 || TB.nkeys == 0 || TA.n2 == 0 || TB.n2 == 0 ||
      C.n2 == 0 || !TA.voff.empty() || !TB.voff.empty())
    return false;
  const int PC = C.P();
  SharedPlan sp = plan_shared(lC, PC, A0, B0, shared, false);
  auto tail_kept = [](const std::vector<int>& perm, const Tensor& T) {
    for (int r = 0; r < T.n2; ++r)
      if (perm[T.P() + r] != T.P() + r + 1) return false;
    return true;
  };
  if (!tail_kept(sp.permA, TA) || !tail_kept(sp.permB, TB)) return false;
  const int nkA = static_cast<int>(sp.dkA.size()), nkB = static_cast<int>(sp.dkB.size()),
            nred = static_cast<int>(sp.red_dense.size());
  const int PA = TA.P(), PB = TB.P();
  const int64_t M = prod(TA.dims, PA, PA + nkA), K = prod(TA.dims, PA + nkA, TA.N()), N = prod(TB.dims, PB + nred, TB.N());
  if (ctx->auto_crop < 2 && (M < 32 || N < 32 || K < 32)) return false;
  // the join (key-sorted views of the operands, as shared_bb makes them)
  Op A = permuted_keys_only(ctx, A0, sp.permA);
  Op B = permuted_keys_only(ctx, B0, sp.permB);
  auto orig = [](const Op& V, const Tensor& T0, int64_t i) { return V.t == &T0 ? i : V->voff[i] / T0.blksize(); };
  auto src = csrc_AB(lC, PC, A, B, true);
  std::vector<int> jA, jB;
  for (auto& l : sp.shared_prefix) { jA.push_back(find(A.labels, l) + 1); jB.push_back(find(B.labels, l) + 1); }
  CKeys ck(C);
  std::vector<std::pair<int64_t, int64_t>> pr;
  std::vector<int64_t> k(PC);
  merge_join(*A, jA, *B, jB, [&](int64_t a, int64_t b) {
    for (int q = 0; q < PC; ++q) k[q] = src[q] > 0 ? A->key(a)[src[q] - 1] : B->key(b)[-src[q] - 1];
    ck.touch(k);
    pr.emplace_back(orig(A, TA, a), orig(B, TB, b));
  });
  const double padded = 2.0 * static_cast<double>(M) * static_cast<double>(K) * static_cast<double>(N) *
                        static_cast<double>(pr.size());
  if (pr.empty() || (ctx->auto_crop < 2 && padded < 1e8)) return false;
  // scanned extents, harmonised
  const auto scans = bs_nonzero_extents(ctx, {&TA, &TB});
  const std::vector<int64_t>& sA = scans[0];
  const std::vector<int64_t>& sB = scans[1];
  const int64_t nvA = TA.nkeys * TA.n2, nv = nvA + TB.nkeys * TB.n2;
  std::vector<int64_t> parent(nv);
  std::iota(parent.begin(), parent.end(), 0);
  auto root = [&](int64_t v) {
    while (parent[v] != v) v = parent[v] = parent[parent[v]];
    return v;
  };
  auto unite = [&](int64_t a, int64_t b) {
    a = root(a);
    b = root(b);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  };
  auto vA = [&](int64_t o, int t) { return o * TA.n2 + t; };
  auto vB = [&](int64_t o, int t) { return nvA + o * TB.n2 + t; };
  for (auto& p : pr)
    for (int t = 0; t < nred; ++t) unite(vA(p.first, nkA + t), vB(p.second, t));
  for (auto& cs : ck.contribs)
    for (size_t i = 1; i < cs.size(); ++i) {
      const auto& p0 = pr[cs[0]];
      const auto& p = pr[cs[i]];
      for (int t = 0; t < nkA; ++t) unite(vA(p.first, t), vA(p0.first, t));
      for (int t = 0; t < nkB; ++t) unite(vB(p.second, nred + t), vB(p0.second, nred + t));
    }
  std::vector<int64_t> mx(nv, 1);
  for (int64_t v = 0; v < nv; ++v) {
    const int64_t r = root(v);
    mx[r] = std::max(mx[r], v < nvA ? sA[v] : sB[v - nvA]);
  }
  std::vector<int64_t> eA(nvA), eB(nv - nvA);
  for (int64_t v = 0; v < nv; ++v) (v < nvA ? eA[v] : eB[v - nvA]) = mx[root(v)];
  double cropped = 0.0;
  for (auto& p : pr) {
    double m = 1, kk = 1, n = 1;
    for (int t = 0; t < nkA; ++t) m *= static_cast<double>(eA[vA(p.first, t)]);
    for (int t = 0; t < nred; ++t) kk *= static_cast<double>(eA[vA(p.first, nkA + t)]);
    for (int t = 0; t < nkB; ++t) n *= static_cast<double>(eB[vB(p.second, nred + t) - nvA]);
    cropped += 2.0 * m * kk * n;
  }
  if (!(cropped <= (ctx->auto_crop < 2 ? 0.8 : 1.0) * padded) || (ctx->auto_crop >= 2 && cropped >= padded))
    return false;
  // the cropped operands and the ragged result live in buffers kept for this
  // output tensor: a contraction repeated on one structure (every Lanczos
  // step) allocates nothing
  if (!ctx->crop_scratch) ctx->crop_scratch = std::make_shared<CropScratchMap>();
  auto& scm = static_cast<CropScratchMap*>(ctx->crop_scratch.get())->m;
  if (scm.size() >= CropScratchMap::kMax && !scm.count(&C)) scm.clear();
  CropScratch& sc = scm[&C];
  TensorPtr Ar = bs_to_ragged(ctx, TA, eA, false, &sc.a);
  TensorPtr Br = bs_to_ragged(ctx, TB, eB, false, &sc.b);
  auto Cr = make_tensor(ctx, BS, C.dims, C.n2);
  Cr->data = std::move(sc.c);
  shared_bb(ctx, *Cr, lC, view(*Ar, A0.labels), view(*Br, B0.labels), shared);
  reset_output(ctx, C, Cr->nkeys, Cr->nkeys * C.blksize());
  C.keys = Cr->keys;
  bs_pad_into(ctx, *Cr, C.data.d());
  sc.a = std::move(Ar->data);
  sc.b = std::move(Br->data);
  sc.c = std::move(Cr->data);
  ctx->auto_cropped = true;
  return true;
}

void shared_bb(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Labels& shared) {
  if (shared_bb_cropped(ctx, C, lC, A0, B0, shared)) return;
  ctx->kernel_name = "contract_shared! (BS x BS)";
  const int PC = C.P();
  SharedPlan sp = plan_shared(lC, PC, A0, B0, shared, false);
  const bool cacheable = ctx->plan_cache_on && !ctx->capturing;
  std::vector<uint64_t> sig;
  SharedPlanCache* cache = nullptr;
  if (cacheable) {
    if (!ctx->plan_cache) ctx->plan_cache = std::make_shared<SharedPlanCache>();
    cache = static_cast<SharedPlanCache*>(ctx->plan_cache.get());
    sig = shared_signature(C, lC, A0, B0);
    sig.push_back(static_cast<uint64_t>(ctx->precision));
    sig.push_back((C.f32 ? 1u : 0u) | (A0->f32 ? 2u : 0u) | (B0->f32 ? 4u : 0u));
    for (auto it = cache->entries.rbegin(); it != cache->entries.rend(); ++it) {
      const SharedPlanEntry& e = **it;
      if (e.sig != sig || e.akeys != A0->keys || e.bkeys != B0->keys || e.abd != A0->bdims || e.bbd != B0->bdims)
        continue;
      Op A = permuted_keys_only(ctx, A0, sp.permA);
      Op B = permuted_keys_only(ctx, B0, sp.permB);
      reset_output(ctx, C, e.c_nkeys, e.c_payload);
      C.keys = e.c_keys;
      if (e.c_ragged) {
        C.ragged = true;
        C.bdims = e.c_bdims;
        C.boff = e.c_boff;
      }
      if (sp.mode == Mode::AthenB) e.gemm.run_io(ctx, *A, *B, C);
      else e.gemm.run_io(ctx, *B, *A, C);
      ctx->plan_cache_hit = true;
      return;
    }
  }
  Op A = permuted_keys_only(ctx, A0, sp.permA);
  Op B = permuted_keys_only(ctx, B0, sp.permB);
  const int PA = A->P(), PB = B->P();
  const int nkA = static_cast<int>(sp.dkA.size()), nkB = static_cast<int>(sp.dkB.size()),
            nred = static_cast<int>(sp.red_dense.size());
  const int64_t M = prod(A->dims, PA, PA + nkA), K = prod(A->dims, PA + nkA, A->N()), N = prod(B->dims, PB + nred, B->N());
  require(K == prod(B->dims, PB, PB + nred), SB_ERR_DIM_MISMATCH, "Reduced dense extents mismatch between A and B");
  require(C.blksize() == M * N, SB_ERR_DIM_MISMATCH, "C.blksize must equal M*N");
  auto src = csrc_AB(lC, PC, A, B, true);
  std::vector<int> jA, jB;
  for (auto& l : sp.shared_prefix) { jA.push_back(find(A.labels, l) + 1); jB.push_back(find(B.labels, l) + 1); }
  CKeys ck(C);
  std::vector<std::pair<int64_t, int64_t>> pr;
  std::vector<int64_t> k(PC);
  merge_join(*A, jA, *B, jB, [&](int64_t a, int64_t b) {
    for (int q = 0; q < PC; ++q) k[q] = src[q] > 0 ? A->key(a)[src[q] - 1] : B->key(b)[-src[q] - 1];
    ck.touch(k);
    pr.emplace_back(a, b);
  });
  auto ord = ck.order();
  const bool athenb = sp.mode == Mode::AthenB;
  const bool ragged = A->ragged || B->ragged;
  const int n2C = C.n2;
  // Per-pair GEMM extents from the blocks' own tail extents (uniform tensors:
  // the full dims).  Ragged operands must agree on every reduced extent, and
  // all pairs feeding one C block must agree on its extents.
  struct PairDims { int64_t m, k, n; };
  std::vector<PairDims> pd(pr.size());
  std::vector<int64_t> cbd(ragged ? ord.size() * n2C : 0);
  for (size_t c = 0; c < ord.size(); ++c) {
    bool first = true;
    for (int ci : ck.contribs[ord[c]]) {
      const int64_t a = pr[ci].first, b = pr[ci].second;
      int64_t m = 1, kk = 1, n = 1;
      for (int t = 0; t < nkA; ++t) m *= A->block_dim(a, t);
      for (int t = 0; t < nred; ++t) {
        const int64_t ea = A->block_dim(a, nkA + t), eb = B->block_dim(b, t);
        require(ea == eb, SB_ERR_DIM_MISMATCH, "ragged reduced extents differ within a matched block pair");
        kk *= ea;
      }
      for (int t = 0; t < nkB; ++t) n *= B->block_dim(b, nred + t);
      pd[ci] = PairDims{m, kk, n};
      if (ragged) {
        std::vector<int64_t> e;
        if (athenb) {
          for (int t = 0; t < nkA; ++t) e.push_back(A->block_dim(a, t));
          for (int t = 0; t < nkB; ++t) e.push_back(B->block_dim(b, nred + t));
        } else {
          for (int t = 0; t < nkB; ++t) e.push_back(B->block_dim(b, nred + t));
          for (int t = 0; t < nkA; ++t) e.push_back(A->block_dim(a, t));
        }
        if (first) std::copy(e.begin(), e.end(), cbd.begin() + c * n2C);
        else
          require(std::equal(e.begin(), e.end(), cbd.begin() + c * n2C), SB_ERR_DIM_MISMATCH,
                  "ragged extents of one output block differ between contributing pairs");
      }
      first = false;
    }
  }
  const int64_t blkC = C.blksize();
  std::vector<int64_t> cboff(ord.size() + 1, 0);
  for (size_t c = 0; c < ord.size(); ++c) {
    int64_t len = blkC;
    if (ragged) {
      len = 1;
      for (int t = 0; t < n2C; ++t) len *= cbd[c * n2C + t];
    }
    cboff[c + 1] = cboff[c] + len;
  }
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), cboff.back());
  ck.commit_keys(C, ord);
  if (ragged) {
    C.ragged = true;
    C.bdims = std::move(cbd);
    C.boff = cboff;
  }
  GemmPlan gp;
  for (size_t c = 0; c < ord.size(); ++c) {
    const auto& c0 = pd[ck.contribs[ord[c]][0]];
    if (athenb) gp.add_cblock(cboff[c], c0.m, c0.n);
    else gp.add_cblock(cboff[c], c0.n, c0.m);
    for (int ci : ck.contribs[ord[c]]) {
      const int64_t xa = A->block_off(pr[ci].first), yb = B->block_off(pr[ci].second);
      const auto& d = pd[ci];
      // AthenB: C(MxN) = A(MxK) B(KxN); BthenA: C(NxM) = B^T A^T
      if (athenb) gp.add_pair(xa, yb, d.k, d.m, d.k);
      else gp.add_pair(yb, xa, d.k, d.k, d.m);
    }
  }
  const int f32mask = athenb ? (A->f32 ? 1 : 0) | (B->f32 ? 2 : 0) | (C.f32 ? 4 : 0)
                              : (B->f32 ? 1 : 0) | (A->f32 ? 2 : 0) | (C.f32 ? 4 : 0);
  auto run_g = [&](const GemmLaunch& gl) {
    if (athenb) gl.run_io(ctx, *A, *B, C);
    else gl.run_io(ctx, *B, *A, C);
  };
  GemmLaunch g = athenb ? gp.prepare(ctx, false, false, f32mask) : gp.prepare(ctx, true, true, f32mask);
  if (ctx->autotune && !ctx->capturing && f32mask == 0 && ctx->precision == SB_PRECISION_F64 &&
      (g.kind == GemmLaunch::TILED || g.kind == GemmLaunch::EDGES))
    g = autotune_gemm(ctx, gp, athenb, std::move(g), run_g);
  run_g(g);
  if (cache) {
    auto e = std::make_unique<SharedPlanEntry>();
    e->sig = std::move(sig);
    e->akeys = A0->keys;
    e->abd = A0->bdims;
    e->bkeys = B0->keys;
    e->bbd = B0->bdims;
    e->c_nkeys = C.nkeys;
    e->c_payload = C.payload_len();
    e->c_keys = C.keys;
    e->c_ragged = C.ragged;
    e->c_bdims = C.bdims;
    e->c_boff = C.boff;
    e->gemm = std::move(g);
    if (cache->entries.size() >= SharedPlanCache::kMax) cache->entries.erase(cache->entries.begin());
    cache->entries.push_back(std::move(e));
  }
}

// ══════════════════════════ BS × Dense ═══════════════════════════════════

std::vector<int> move_axis_last(int N, int ax) {
  std::vector<int> p;
  for (int d = 1; d <= N; ++d)
    if (d != ax) p.push_back(d);
  p.push_back(ax);
  return p;
}

void prefix_outer_bd(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_prefix_outer_bd!";
  const int PC = C.P();
  Op A = r_to_last_prefix(ctx, A0, r);
  const int PA = A->P();
  const int NB = B0->N();
  const int axB = find(B0.labels, r) + 1;
  require(axB >= 1, SB_ERR_LABEL, "rlab must be a dim of dense B");
  const int64_t R = B0->dims[axB - 1];
  Op B = axB == NB ? view(*B0.t, B0.labels) : permuted(ctx, B0, move_axis_last(NB, axB));
  const int64_t chunkB = B->numel() / R;
  Labels Ad(A.labels.begin() + PA, A.labels.end()), Bwo(B.labels.begin(), B.labels.end() - 1),
      Cd(lC.begin() + PC, lC.end());
  Labels AB(Ad), BA(Bwo);
  AB.insert(AB.end(), Bwo.begin(), Bwo.end());
  BA.insert(BA.end(), Ad.begin(), Ad.end());
  bool ab;
  if (Cd == AB) ab = true;
  else if (Cd == BA) ab = false;
  else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense tail must be [A_dense..., B_wo_r...] or [B_wo_r..., A_dense...]");
  const int64_t chunkA = A->blksize();
  require(C.blksize() == chunkA * chunkB, SB_ERR_DIM_MISMATCH, "C.blksize must equal A.blksize * (prod(B dims without r))");
  std::vector<int> src;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    require(ia >= 0, SB_ERR_LABEL, "C prefix label not in A");
    require(ia < PA && !(lC[j] == r), SB_ERR_LABEL, "C prefix must be from A prefix excluding rlab");
    src.push_back(ia + 1);
  }
  const int64_t nA = A->nkeys;
  std::vector<std::vector<int64_t>> ck(nA, std::vector<int64_t>(PC));
  for (int64_t i = 0; i < nA; ++i)
    for (int q = 0; q < PC; ++q) ck[i][q] = A->key(i)[src[q] - 1];
  std::vector<int64_t> perm(nA);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return ck[a] < ck[b]; });  // sortperm(ckeys)
  CKeys keys(C);
  std::vector<int64_t> contrib_a;
  for (int64_t i = 0; i < nA; ++i) {
    keys.touch(ck[perm[i]]);
    contrib_a.push_back(perm[i]);
    const int64_t rv = A->key(perm[i])[PA - 1];
    require(rv >= 1 && rv <= R, SB_ERR_ASSERTION, "A block key r out of bounds for dense B");
  }
  auto ord = keys.order();
  const int64_t blkC = C.blksize();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * blkC);
  keys.commit_keys(C, ord);
  OuterPlan op;
  for (size_t c = 0; c < ord.size(); ++c) {
    op.add_cblock(static_cast<int64_t>(c) * blkC, ab ? chunkA : chunkB, ab ? chunkB : chunkA);
    for (int ci : keys.contribs[ord[c]]) {
      const int64_t a = contrib_a[ci];
      const int64_t rv = A->key(a)[PA - 1];
      if (ab) op.add_pair(a * chunkA, (rv - 1) * chunkB);
      else op.add_pair((rv - 1) * chunkB, a * chunkA);
    }
  }
  if (ab) op.launch(ctx, A->data.d(), B->data.d(), C.data.d(), true);
  else op.launch(ctx, B->data.d(), A->data.d(), C.data.d(), true);
}

void dense_bd(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_dense_bd!";
  const int PA = A0->P(), PC = C.P();
  const int axA = find(A0.labels, r) + 1, axB = find(B0.labels, r) + 1;
  require(axA > PA, SB_ERR_LABEL, "rlab must be in A dense tail");
  require(axB >= 1, SB_ERR_LABEL, "rlab must be an axis of B");
  Op A = axA != A0->N() ? permuted(ctx, A0, perm_r_last(PA, A0->N(), axA)) : view(*A0.t, A0.labels);
  const int NB = B0->N();
  Op B = axB != NB ? permuted(ctx, B0, move_axis_last(NB, axB)) : view(*B0.t, B0.labels);
  const int64_t R = A->dims.back();
  require(B->dims.back() == R, SB_ERR_DIM_MISMATCH, "reduction extents differ");
  const int64_t chunkA = A->blksize() / R, chunkB = B->numel() / R;
  require(C.n2 == (A->n2 - 1) + (NB - 1), SB_ERR_ASSERTION, "N2C must equal (N2A-1)+(NB-1)");
  require(C.blksize() == chunkA * chunkB, SB_ERR_DIM_MISMATCH, "C.blksize must equal chunkA*chunkB");
  Labels Awo(A.labels.begin() + PA, A.labels.end() - 1), Bwo(B.labels.begin(), B.labels.end() - 1),
      Cd(lC.begin() + PC, lC.end());
  Labels AB(Awo), BA(Bwo);
  AB.insert(AB.end(), Bwo.begin(), Bwo.end());
  BA.insert(BA.end(), Awo.begin(), Awo.end());
  bool ab;
  if (Cd == AB) ab = true;
  else if (Cd == BA) ab = false;
  else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense tail must be [A_dense..., B_dense...] or [B_dense..., A_dense...]");
  std::vector<int> srcA;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    require(ia >= 0 && ia < PA, SB_ERR_LABEL, "C sparse prefix label must come from A sparse head");
    srcA.push_back(ia + 1);
  }
  const int64_t nA = A->nkeys, blkA = A->blksize();
  std::vector<int64_t> offA(nA);
  for (int64_t i = 0; i < nA; ++i) offA[i] = i * blkA;
  auto fA = slice_flags(ctx, A->data.d(), offA, R, chunkA);
  auto fB = slice_flags(ctx, B->data.d(), {0}, R, chunkB);
  CKeys ck(C);
  std::vector<int64_t> contrib_a;
  std::vector<int64_t> k(PC);
  for (int64_t a = 0; a < nA; ++a) {
    bool any = false;
    for (int64_t s = 0; s < R && !any; ++s) any = fA[a * R + s] && fB[s];
    if (!any) continue;
    for (int q = 0; q < PC; ++q) k[q] = A->key(a)[srcA[q] - 1];
    ck.touch(k);
    contrib_a.push_back(a);
  }
  auto ord = ck.order();
  const int64_t blkC = C.blksize();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * blkC);
  ck.commit_keys(C, ord);
  GemmPlan gp;
  for (size_t c = 0; c < ord.size(); ++c) {
    gp.add_cblock(static_cast<int64_t>(c) * blkC, ab ? chunkA : chunkB, ab ? chunkB : chunkA);
    for (int ci : ck.contribs[ord[c]]) {
      const int64_t a = contrib_a[ci];
      if (ab) gp.add_pair(a * blkA, 0, R, chunkA, chunkB);
      else gp.add_pair(0, a * blkA, R, chunkB, chunkA);
    }
  }
  if (ab) gp.launch(ctx, A->data.d(), B->data.d(), C.data.d(), false, true);
  else gp.launch(ctx, B->data.d(), A->data.d(), C.data.d(), false, true);
}

// Dense B permuted to [red..., keepB..., shared_prefix...] so that every slice
// Bp[:, :, sp_vals] is one contiguous K x N column-major matrix (the values of
// the reference's Bp[sp_vals..., :, ...] view, contract_bs_dense.jl:589-592).
struct DenseSlices {
  Op Bp;
  int64_t K = 1, N = 1, slab = 0;
  std::vector<int64_t> sp_dims;
};
DenseSlices dense_slices(Ctx* ctx, const Op& B0, const Labels& sp, const Labels& red, const Labels& dkB) {
  std::vector<int> perm;
  for (auto& l : red) perm.push_back(find(B0.labels, l) + 1);
  for (auto& l : dkB) perm.push_back(find(B0.labels, l) + 1);
  for (auto& l : sp) perm.push_back(find(B0.labels, l) + 1);
  require(static_cast<int>(perm.size()) == B0->N(), SB_ERR_ASSERTION, "B perm length mismatch; labelsB must match B ndims");
  DenseSlices ds;
  ds.Bp = permuted(ctx, B0, perm);
  const int nr = static_cast<int>(red.size()), nk = static_cast<int>(dkB.size());
  ds.K = prod(ds.Bp->dims, 0, nr);
  ds.N = prod(ds.Bp->dims, nr, nr + nk);
  ds.slab = ds.K * ds.N;
  ds.sp_dims.assign(ds.Bp->dims.begin() + nr + nk, ds.Bp->dims.end());
  return ds;
}

void shared_bd(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Labels& shared) {
  ctx->kernel_name = "contract_shared! (BS x Dense)";
  const int PC = C.P();
  SharedPlan sp = plan_shared(lC, PC, A0, B0, shared, true);
  Op A = permuted(ctx, A0, sp.permA);
  const int PA = A->P();
  const int nkA = static_cast<int>(sp.dkA.size());
  DenseSlices ds = dense_slices(ctx, B0, sp.shared_prefix, sp.red_dense, sp.dkB);
  const int64_t M = prod(A->dims, PA, PA + nkA), K = prod(A->dims, PA + nkA, A->N()), N = ds.N;
  require(K == ds.K, SB_ERR_DIM_MISMATCH, "Reduced dense extents mismatch between A and B");
  require(C.blksize() == M * N, SB_ERR_DIM_MISMATCH, "C.blksize must equal M*N");
  std::vector<int> csrc;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    require(ia >= 0, SB_ERR_LABEL, "C prefix label must exist in A");
    require(ia < PA && !has(sp.shared_prefix, lC[j]), SB_ERR_LABEL, "C prefix label must come from A prefix");
    csrc.push_back(ia + 1);
  }
  std::vector<int> jA;
  for (auto& l : sp.shared_prefix) jA.push_back(find(A.labels, l) + 1);
  CKeys ck(C);
  std::vector<std::pair<int64_t, int64_t>> pr;  // (a block, B slab offset)
  std::vector<int64_t> k(PC);
  for (int64_t iA = 0; iA < A->nkeys;) {
    const int64_t iA2 = advance_run(*A, iA, jA);
    int64_t slab = 0, stride = 1;
    for (size_t t = 0; t < jA.size(); ++t) {
      slab += (A->key(iA)[jA[t] - 1] - 1) * stride;
      stride *= ds.sp_dims[t];
    }
    for (int64_t a = iA; a < iA2; ++a) {
      for (int q = 0; q < PC; ++q) k[q] = A->key(a)[csrc[q] - 1];
      ck.touch(k);
      pr.emplace_back(a, slab * ds.slab);
    }
    iA = iA2;
  }
  auto ord = ck.order();
  const int64_t blkA = A->blksize(), blkC = C.blksize();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * blkC);
  ck.commit_keys(C, ord);
  GemmPlan gp;
  const bool athenb = sp.mode == Mode::AthenB;
  for (size_t c = 0; c < ord.size(); ++c) {
    if (athenb) gp.add_cblock(static_cast<int64_t>(c) * blkC, M, N);
    else gp.add_cblock(static_cast<int64_t>(c) * blkC, N, M);
    for (int ci : ck.contribs[ord[c]]) {
      if (athenb) gp.add_pair(pr[ci].first * blkA, pr[ci].second, K, M, K);
      else gp.add_pair(pr[ci].second, pr[ci].first * blkA, K, K, M);
    }
  }
  if (athenb) gp.launch(ctx, A->data.d(), ds.Bp->data.d(), C.data.d(), false, false);
  else gp.launch(ctx, ds.Bp->data.d(), A->data.d(), C.data.d(), true, true);
}

// ══════════════════════════ COO kernels ══════════════════════════════════

// ensure_rlab_last_and_sorted (contract_coo.jl:48-82)
Op coo_r_last_sorted(Ctx* ctx, const Op& A, const Label& r) {
  if (A.labels.back() == r) return view(*A.t, A.labels);
  std::vector<int> perm;
  for (int i = 0; i < A->N(); ++i)
    if (!(A.labels[i] == r)) perm.push_back(i + 1);
  perm.push_back(find(A.labels, r) + 1);
  Op o = permuted(ctx, A, perm);
  o.owned->dirty = true;
  coo_sort(ctx, *o.owned);
  return o;
}

void coo_coo(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract! (COO x COO)";
  Op A = coo_r_last_sorted(ctx, A0, r), B = coo_r_last_sorted(ctx, B0, r);
  const int NC = C.N(), NA = A->N(), NB = B->N();
  std::vector<std::pair<int, int>> src;
  for (int t = 0; t < NC; ++t) {
    const int ia = find(A.labels, lC[t]);
    if (ia >= 0) src.emplace_back(1, ia);
    else { const int ib = find(B.labels, lC[t]); require(ib >= 0, SB_ERR_LABEL, "C label not in A or B"); src.emplace_back(2, ib); }
  }
  std::vector<int64_t> ia_list, ib_list;
  int64_t i = 0, j = 0;
  while (i < A->nkeys && j < B->nkeys) {
    const int64_t ra = A->key(i)[NA - 1], rb = B->key(j)[NB - 1];
    if (ra < rb) ++i;
    else if (rb < ra) ++j;
    else {
      const int64_t jlo = j;
      while (j < B->nkeys && B->key(j)[NB - 1] == rb) ++j;
      for (; i < A->nkeys && A->key(i)[NA - 1] == ra; ++i)
        for (int64_t jj = jlo; jj < j; ++jj) { ia_list.push_back(i); ib_list.push_back(jj); }
    }
  }
  const int64_t n = static_cast<int64_t>(ia_list.size());
  // products on the device; exact zeros are dropped (_push_term!, contract_coo.jl:84-91)
  std::vector<ScalarTerm> terms(n);
  std::vector<int32_t> seg(n + 1);
  for (int64_t q = 0; q < n; ++q) { terms[q] = ScalarTerm{ia_list[q], ib_list[q]}; seg[q] = static_cast<int32_t>(q); }
  seg[n] = static_cast<int32_t>(n);
  DevBuf prod_buf(ctx, n * sizeof(double));
  std::vector<uint8_t> nz;
  if (n) {
    DevBuf dt = upload(ctx, terms), dsg = upload(ctx, seg);
    SB_CK(launch_scalar_prog(A->data.d(), B->data.d(), dt.as<ScalarTerm>(), dsg.as<int32_t>(), n, prod_buf.d(), ctx->stream));
    DevBuf fl(ctx, n);
    std::vector<int64_t> offs(n);
    std::iota(offs.begin(), offs.end(), 0);
    DevBuf doff = upload(ctx, offs);
    SB_CK(launch_slice_nonzero(prod_buf.d(), doff.as<int64_t>(), n, 1, 1, fl.as<uint8_t>(), ctx->stream));
    ctx->note_launch(2);
    nz = download<uint8_t>(ctx, fl.raw(), n);
  }
  std::vector<int64_t> keep;
  C.keys.clear();
  for (int64_t q = 0; q < n; ++q) {
    if (!nz[q]) continue;
    keep.push_back(q);
    for (int t = 0; t < NC; ++t)
      C.keys.push_back(src[t].first == 1 ? A->key(ia_list[q])[src[t].second] : B->key(ib_list[q])[src[t].second]);
  }
  C.nkeys = static_cast<int64_t>(keep.size());
  C.dirty = true;
  C.data = DevBuf(ctx, C.nkeys * sizeof(double));
  if (C.nkeys) {
    DevBuf dk = upload(ctx, keep);
    SB_CK(launch_gather(prod_buf.d(), dk.as<int64_t>(), C.nkeys, C.data.d(), ctx->stream));
    ctx->note_launch();
  }
}

// aligned_A_to_Cprefix (contract_coo_dense.jl:4-18)
Op coo_align_to_cprefix(Ctx* ctx, const Op& A, const Labels& lC, int PC, const Label& r) {
  std::vector<int> perm;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    require(ia >= 0, SB_ERR_LABEL, "C prefix label not in A");
    perm.push_back(ia + 1);
  }
  const int ir = find(A.labels, r);
  require(ir >= 0, SB_ERR_LABEL, "rlab not in A");
  perm.push_back(ir + 1);
  require(static_cast<int>(perm.size()) == A->N(), SB_ERR_ASSERTION, "PC mismatch: C prefix must be A labels without r");
  Op o;
  o.owned = coo_permute(ctx, *A.t, perm);
  coo_sort(ctx, *o.owned);
  o.t = o.owned.get();
  for (int p : perm) o.labels.push_back(A.labels[p - 1]);
  return o;
}

Op dense_c_tail_r_last(Ctx* ctx, const Op& B, const Labels& lC, int PC, const Label& r) {
  std::vector<int> perm;
  for (size_t j = PC; j < lC.size(); ++j) {
    const int ib = find(B.labels, lC[j]);
    require(ib >= 0, SB_ERR_LABEL, "label not found in labelsB");
    perm.push_back(ib + 1);
  }
  const int ir = find(B.labels, r);
  require(ir >= 0, SB_ERR_LABEL, "rlab not found in labelsB");
  perm.push_back(ir + 1);
  require(static_cast<int>(perm.size()) == B->N(), SB_ERR_ASSERTION, "N2 mismatch: C dense labels must be B labels without r");
  return permuted(ctx, B, perm);
}

void coo_dense(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract! (COO x Dense)";
  const int PC = C.P();
  require(!has(lC, r), SB_ERR_LABEL, "rlab must be reduced (not in labelsC)");
  Op A = coo_align_to_cprefix(ctx, A0, lC, PC, r);
  Op B = dense_c_tail_r_last(ctx, B0, lC, PC, r);
  require(C.n2 == B->N() - 1, SB_ERR_ASSERTION, "N2 mismatch");
  const int64_t R = B->dims.back(), chunk = B->numel() / R;
  require(C.blksize() == chunk, SB_ERR_DIM_MISMATCH, "C.blksize must equal prod(B dims without r)");
  CKeys ck(C);
  std::vector<int64_t> ca;
  const int NA = A->N();
  for (int64_t i = 0; i < A->nkeys; ++i) {
    const int64_t rv = A->key(i)[NA - 1];
    if (rv < 1 || rv > R) continue;
    ck.touch(std::vector<int64_t>(A->key(i), A->key(i) + PC));
    ca.push_back(i);
  }
  auto ord = ck.order();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * chunk);
  ck.commit_keys(C, ord);
  AxpyPlan ap;
  for (size_t c = 0; c < ord.size(); ++c) {
    ap.add_seg(static_cast<int64_t>(c) * chunk, chunk);
    for (int ci : ck.contribs[ord[c]]) {
      const int64_t a = ca[ci];
      ap.add((A->key(a)[NA - 1] - 1) * chunk, a);
    }
  }
  ap.launch(ctx, B->data.d(), A->data.d(), C.data.d());
}

void coo_bs_prefix(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A, const Op& B, const Label& r) {
  ctx->kernel_name = "contract_prefix! (COO x BS)";
  const int PB = B->P(), PC = C.P(), NA = A->N();
  require(PC == NA + PB - 2, SB_ERR_ASSERTION, "PC must equal NA + PB - 2");
  require(C.n2 == B->n2, SB_ERR_ASSERTION, "C tail must equal B tail");
  const int aR = find(A.labels, r), bR = find(B.labels, r);
  std::vector<int> src;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    if (ia >= 0) src.push_back(ia + 1);
    else { const int ib = find(B.labels, lC[j]); require(ib >= 0 && ib < PB, SB_ERR_LABEL, "C prefix label must come from A or B prefix"); src.push_back(-(ib + 1)); }
  }
  CKeys ck(C);
  std::vector<std::pair<int64_t, int64_t>> pr;
  std::vector<int64_t> k(PC);
  int64_t iA = 0, iB = 0;
  while (iA < A->nkeys && iB < B->nkeys) {
    const int64_t rA = A->key(iA)[aR], rB = B->key(iB)[bR];
    if (rA < rB) { while (iA < A->nkeys && A->key(iA)[aR] == rA) ++iA; }
    else if (rB < rA) { while (iB < B->nkeys && B->key(iB)[bR] == rB) ++iB; }
    else {
      const int64_t blo = iB;
      while (iB < B->nkeys && B->key(iB)[bR] == rA) ++iB;
      for (; iA < A->nkeys && A->key(iA)[aR] == rA; ++iA)
        for (int64_t b = blo; b < iB; ++b) {
          for (int q = 0; q < PC; ++q) k[q] = src[q] > 0 ? A->key(iA)[src[q] - 1] : B->key(b)[-src[q] - 1];
          ck.touch(k);
          pr.emplace_back(iA, b);
        }
    }
  }
  auto ord = ck.order();
  const int64_t blk = C.blksize();
  require(blk == B->blksize(), SB_ERR_DIM_MISMATCH, "C.blksize must equal B.blksize");
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * blk);
  ck.commit_keys(C, ord);
  AxpyPlan ap;
  for (size_t c = 0; c < ord.size(); ++c) {
    ap.add_seg(static_cast<int64_t>(c) * blk, blk);
    for (int ci : ck.contribs[ord[c]]) ap.add(pr[ci].second * blk, pr[ci].first);
  }
  ap.launch(ctx, B->data.d(), A->data.d(), C.data.d());
}

void coo_bs_dense_index(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_dense_index! (COO x BS)";
  const int PB = B0->P(), PC = C.P(), NA = A->N();
  require(!has(lC, r), SB_ERR_LABEL, "rlab must be reduced (not in labelsC)");
  require(C.n2 == B0->n2 - 1, SB_ERR_ASSERTION, "N2C must equal N2B - 1");
  const int axB = find(B0.labels, r) + 1;
  require(axB > PB, SB_ERR_LABEL, "rlab must be in B dense tail");
  require(find(A.labels, r) + 1 == NA, SB_ERR_ASSERTION, "Expected A to have rlab as last axis");
  Op B = axB != B0->N() ? permuted(ctx, B0, perm_r_last(PB, B0->N(), axB)) : view(*B0.t, B0.labels);
  const int64_t dim_r = B->dims.back(), chunk = B->blksize() / dim_r;
  Labels exp(B.labels.begin() + PB, B.labels.end() - 1), Cd(lC.begin() + PC, lC.end());
  require(Cd == exp, SB_ERR_LABEL, "C dense tail must be B dense tail without r");
  require(C.blksize() == chunk, SB_ERR_DIM_MISMATCH, "C.blksize must equal chunk");
  std::vector<int> srcA(PC, 0), srcB(PC, 0);
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    if (ia >= 0) srcA[j] = ia + 1;
    else { const int ib = find(B.labels, lC[j]); require(ib >= 0 && ib < PB, SB_ERR_LABEL, "Label in C prefix must come from B prefix"); srcB[j] = ib + 1; }
  }
  // candidate (nnz, block) pairs; value-dependent skip of all-zero α·slice
  const int64_t nA = A->nkeys, nB = B->nkeys, blkB = B->blksize();
  std::vector<int64_t> offs, ai;
  offs.reserve(nA * nB);
  for (int64_t a = 0; a < nA; ++a) {
    const int64_t rv = A->key(a)[NA - 1];
    require(rv >= 1 && rv <= dim_r, SB_ERR_ASSERTION, "Reduction index out of bounds");
    for (int64_t b = 0; b < nB; ++b) { offs.push_back(b * blkB + (rv - 1) * chunk); ai.push_back(a); }
  }
  std::vector<uint8_t> nz;
  const int64_t ncand = static_cast<int64_t>(offs.size());
  if (ncand) {
    DevBuf doff = upload(ctx, offs), dai = upload(ctx, ai);
    DevBuf fl(ctx, ncand);
    SB_CK(launch_scaled_slice_nonzero(B->data.d(), A->data.d(), doff.as<int64_t>(), dai.as<int64_t>(), ncand, chunk,
                                      fl.as<uint8_t>(), ctx->stream));
    ctx->note_launch();
    nz = download<uint8_t>(ctx, fl.raw(), ncand);
  }
  CKeys ck(C);
  std::vector<int64_t> cq;
  std::vector<int64_t> k(PC);
  for (int64_t q = 0; q < ncand; ++q) {
    if (!nz[q]) continue;
    const int64_t a = q / nB, b = q % nB;
    for (int t = 0; t < PC; ++t) k[t] = srcA[t] ? A->key(a)[srcA[t] - 1] : B->key(b)[srcB[t] - 1];
    ck.touch(k);
    cq.push_back(q);
  }
  auto ord = ck.order();
  reset_output(ctx, C, static_cast<int64_t>(ord.size()), static_cast<int64_t>(ord.size()) * chunk);
  ck.commit_keys(C, ord);
  AxpyPlan ap;
  for (size_t c = 0; c < ord.size(); ++c) {
    ap.add_seg(static_cast<int64_t>(c) * chunk, chunk);
    for (int ci : ck.contribs[ord[c]]) ap.add(offs[cq[ci]], ai[cq[ci]]);
  }
  ap.launch(ctx, B->data.d(), A->data.d(), C.data.d());
}

// ══════════════════════════ aliased kernels ══════════════════════════════
//
// Template bookkeeping of _aliased_contribute! / _commit_aliased_dicts!
// (contract_aliased.jl:75-146) decided on template ids (structure); scalar
// sums, template products and demoted accumulators computed on the device.

struct AliasBook {
  struct Contrib {
    int tid;        // 1-based combined template id
    ScalarTerm sc;  // scalar = sa[ia] * sb[ib] (ib < 0: sa[ia])
  };
  std::vector<std::vector<int64_t>> keys;
  std::vector<int64_t> lins;
  std::unordered_map<int64_t, int> index;
  std::vector<std::vector<Contrib>> contribs;
  int PC;
  std::vector<int64_t> cdims;
  AliasBook(const Tensor& C) : PC(C.P()), cdims(C.dims) {}
  void contribute(const std::vector<int64_t>& k, int tid, ScalarTerm sc) {
    const int64_t l = lin0(k.data(), cdims.data(), PC);
    auto it = index.find(l);
    int id;
    if (it == index.end()) {
      id = static_cast<int>(keys.size());
      index.emplace(l, id);
      keys.push_back(k);
      lins.push_back(l);
      contribs.emplace_back();
    } else {
      id = it->second;
    }
    contribs[id].push_back(Contrib{tid, sc});
  }
  // templates: device buffer holding n_combined templates; produces C.
  void commit(Ctx* ctx, Tensor& C, DevBuf&& templates, int64_t n_combined, const double* sa, const double* sb) {
    const int64_t blk = C.blksize();
    const int nk = static_cast<int>(keys.size());
    // Replay the alias/accum state machine on template ids.
    std::vector<char> demoted(nk, 0);
    std::vector<int> alias_tid(nk, 0);
    std::vector<ScalarTerm> terms;
    std::vector<int32_t> seg{0};
    std::vector<int64_t> alias_seg(nk, -1);  // scalar segment of an aliased key
    struct AccEntry { int tid; int64_t seg; };
    std::vector<std::vector<AccEntry>> acc(nk);
    for (int id = 0; id < nk; ++id) {
      const auto& cs = contribs[id];
      size_t q = 0;
      const int t0 = cs[0].tid;
      while (q < cs.size() && cs[q].tid == t0) terms.push_back(cs[q++].sc);
      seg.push_back(static_cast<int32_t>(terms.size()));
      const int64_t first_seg = static_cast<int64_t>(seg.size()) - 2;
      if (q == cs.size()) {
        alias_tid[id] = t0;
        alias_seg[id] = first_seg;
        continue;
      }
      demoted[id] = 1;
      acc[id].push_back(AccEntry{t0, first_seg});
      for (; q < cs.size(); ++q) {
        terms.push_back(cs[q].sc);
        seg.push_back(static_cast<int32_t>(terms.size()));
        acc[id].push_back(AccEntry{cs[q].tid, static_cast<int64_t>(seg.size()) - 2});
      }
    }
    const int64_t nseg = static_cast<int64_t>(seg.size()) - 1;
    DevBuf sv(ctx, nseg * sizeof(double));
    if (nseg) {
      DevBuf dt = upload(ctx, terms), ds = upload(ctx, seg);
      SB_CK(launch_scalar_prog(sa, sb, dt.as<ScalarTerm>(), ds.as<int32_t>(), nseg, sv.d(), ctx->stream));
      ctx->note_launch();
    }
    // Commit: aliased keys keep (tid, scalar); demoted keys get new templates.
    std::vector<int> order_alias, order_acc;
    for (int id = 0; id < nk; ++id) (demoted[id] ? order_acc : order_alias).push_back(id);
    const int64_t n_acc = static_cast<int64_t>(order_acc.size());
    const int64_t ntot = n_combined + n_acc;
    DevBuf all(ctx, ntot * blk * sizeof(double));
    if (n_combined)
      SB_CK(cudaMemcpyAsync(all.raw(), templates.raw(), n_combined * blk * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    AxpyPlan ap;
    for (int64_t j = 0; j < n_acc; ++j) {
      ap.add_seg((n_combined + j) * blk, blk);
      for (auto& e : acc[order_acc[j]]) ap.add((e.tid - 1) * blk, e.seg);
    }
    ap.launch(ctx, templates.d(), sv.d(), all.d());
    // per-key (tid, scalar-segment) in commit order, then sorted by lin
    std::vector<int> commit_ids(order_alias);
    commit_ids.insert(commit_ids.end(), order_acc.begin(), order_acc.end());
    std::vector<int64_t> tids(nk), segidx(nk);
    for (size_t j = 0; j < order_alias.size(); ++j) {
      tids[j] = alias_tid[order_alias[j]];
      segidx[j] = alias_seg[order_alias[j]];
    }
    for (int64_t j = 0; j < n_acc; ++j) {
      tids[order_alias.size() + j] = n_combined + j + 1;
      segidx[order_alias.size() + j] = -1;  // scalar 1
    }
    std::vector<int> p(nk);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int a, int b) { return lins[commit_ids[a]] < lins[commit_ids[b]]; });
    C.keys.clear();
    C.alias_ids.assign(nk, 0);
    std::vector<int64_t> sidx(nk);
    for (int i = 0; i < nk; ++i) {
      const int src = p[i];
      const auto& k = keys[commit_ids[src]];
      C.keys.insert(C.keys.end(), k.begin(), k.end());
      C.alias_ids[i] = tids[src];
      sidx[i] = segidx[src];
    }
    C.nkeys = nk;
    C.n_templates = ntot;
    C.data = std::move(all);
    // scalars: segment sums for aliased keys, 1.0 for demoted keys
    C.scalars = DevBuf(ctx, nk * sizeof(double));
    std::vector<int64_t> gidx, gdst;
    for (int i = 0; i < nk; ++i)
      if (sidx[i] >= 0) { gidx.push_back(sidx[i]); gdst.push_back(i); }
    if (nk) {
      std::vector<double> host_ones(nk, 1.0);
      SB_CK(cudaMemcpyAsync(C.scalars.raw(), host_ones.data(), nk * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      if (!gidx.empty()) {
        DevBuf dg = upload(ctx, gidx), dd = upload(ctx, gdst);
        DevBuf tmp(ctx, gidx.size() * sizeof(double));
        SB_CK(launch_gather(sv.d(), dg.as<int64_t>(), static_cast<int64_t>(gidx.size()), tmp.d(), ctx->stream));
        SB_CK(launch_scatter(tmp.d(), dd.as<int64_t>(), static_cast<int64_t>(gidx.size()), C.scalars.d(), ctx->stream));
        ctx->note_launch(2);
      }
    }
  }
};

void reset_aliased(Ctx* ctx, Tensor& C) {
  C.keys.clear();
  C.alias_ids.clear();
  C.nkeys = 0;
  C.n_templates = 0;
  C.data = DevBuf();
  C.scalars = DevBuf();
  (void)ctx;
}

void aliased_coo_dense(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_aliased! (COO x Dense)";
  const int PC = C.P();
  Op A = coo_align_to_cprefix(ctx, A0, lC, PC, r);
  Op B = dense_c_tail_r_last(ctx, B0, lC, PC, r);
  const int64_t R = B->dims.back(), chunk = B->numel() / R;
  require(C.blksize() == chunk, SB_ERR_DIM_MISMATCH, "C.blksize must equal prod(B dims without r)");
  reset_aliased(ctx, C);
  AliasBook book(C);
  std::unordered_map<int64_t, int> rv_tid;
  std::vector<int64_t> tmpl_src;  // B column offsets of the templates
  const int NA = A->N();
  for (int64_t i = 0; i < A->nkeys; ++i) {
    const int64_t rv = A->key(i)[NA - 1];
    if (rv < 1 || rv > R) continue;
    auto it = rv_tid.find(rv);
    int tid;
    if (it == rv_tid.end()) {
      tmpl_src.push_back((rv - 1) * chunk);
      tid = static_cast<int>(tmpl_src.size());
      rv_tid.emplace(rv, tid);
    } else {
      tid = it->second;
    }
    book.contribute(std::vector<int64_t>(A->key(i), A->key(i) + PC), tid, ScalarTerm{i, -1});
  }
  const int64_t nt = static_cast<int64_t>(tmpl_src.size());
  DevBuf tmpl(ctx, nt * chunk * sizeof(double));
  if (nt) {
    std::vector<int64_t> idx(nt * chunk);
    for (int64_t t = 0; t < nt; ++t)
      for (int64_t e = 0; e < chunk; ++e) idx[t * chunk + e] = tmpl_src[t] + e;
    DevBuf di = upload(ctx, idx);
    SB_CK(launch_gather(B->data.d(), di.as<int64_t>(), nt * chunk, tmpl.d(), ctx->stream));
    ctx->note_launch();
  }
  book.commit(ctx, C, std::move(tmpl), nt, A->data.d(), nullptr);
}

Op aliased_r_last_prefix(Ctx* ctx, const Op& A, const Label& r) {
  const int ax = find(A.labels, r) + 1;
  require(ax >= 1 && ax <= A->P(), SB_ERR_LABEL, "rlab must be in sparse prefix");
  if (ax == A->P()) return view(*A.t, A.labels);
  return permuted(ctx, A, perm_r_last(A->P(), A->N(), ax));
}
Op aliased_r_last_dense(Ctx* ctx, const Op& A, const Label& r) {
  const int ax = find(A.labels, r) + 1;
  require(ax > A->P(), SB_ERR_LABEL, "rlab must be in dense tail");
  if (ax == A->N()) return view(*A.t, A.labels);
  return permuted(ctx, A, perm_r_last(A->P(), A->N(), ax));
}

void aliased_ad(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_aliased! (Aliased x Dense)";
  require(!has(lC, r), SB_ERR_LABEL, "rlab must be reduced");
  const int PC = C.P();
  const int NB = B0->N();
  const int axB = find(B0.labels, r) + 1;
  require(axB >= 1, SB_ERR_LABEL, "rlab must be an axis of B");
  Op B = axB == NB ? view(*B0.t, B0.labels) : permuted(ctx, B0, move_axis_last(NB, axB));
  const int64_t R = B->dims.back(), chunkB = B->numel() / R;
  Labels Bwo(B.labels.begin(), B.labels.end() - 1), Cd(lC.begin() + PC, lC.end());
  const bool r_prefix = find(A0.labels, r) < A0->P();
  if (r_prefix) {  // _contract_aliased_prefix_outer_ad! (contract_aliased.jl:154-237)
    Op A = aliased_r_last_prefix(ctx, A0, r);
    const int PA = A->P();
    Labels Ad(A.labels.begin() + PA, A.labels.end());
    Labels AB(Ad), BA(Bwo);
    AB.insert(AB.end(), Bwo.begin(), Bwo.end());
    BA.insert(BA.end(), Ad.begin(), Ad.end());
    bool ab;
    if (Cd == AB) ab = true;
    else if (Cd == BA) ab = false;
    else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense tail must be [A_dense...,B_wo_r...] or [B_wo_r...,A_dense...]");
    const int64_t blkA = A->blksize();
    require(C.blksize() == blkA * chunkB, SB_ERR_DIM_MISMATCH, "C.blksize must equal A.blksize * chunkB");
    std::vector<int> src;
    for (int j = 0; j < PC; ++j) {
      const int ia = find(A.labels, lC[j]);
      require(ia >= 0 && ia < PA && !(lC[j] == r), SB_ERR_LABEL, "C prefix label must come from A sparse prefix excluding rlab");
      src.push_back(ia + 1);
    }
    reset_aliased(ctx, C);
    AliasBook book(C);
    std::map<std::pair<int64_t, int64_t>, int> ctm;
    std::vector<std::pair<int64_t, int64_t>> jobs;  // (tidA, rv)
    std::vector<int64_t> k(PC);
    for (int64_t i = 0; i < A->nkeys; ++i) {
      const int64_t rv = A->key(i)[PA - 1];
      if (rv < 1 || rv > R) continue;
      const int64_t tA = A->alias_ids[i];
      auto key = std::make_pair(tA, rv);
      auto it = ctm.find(key);
      int ct;
      if (it == ctm.end()) { jobs.push_back(key); ct = static_cast<int>(jobs.size()); ctm.emplace(key, ct); }
      else ct = it->second;
      for (int q = 0; q < PC; ++q) k[q] = A->key(i)[src[q] - 1];
      book.contribute(k, ct, ScalarTerm{i, -1});
    }
    const int64_t blkC = C.blksize(), nt = static_cast<int64_t>(jobs.size());
    DevBuf tmpl(ctx, nt * blkC * sizeof(double));
    OuterPlan op;
    for (int64_t t = 0; t < nt; ++t) {
      op.add_cblock(t * blkC, ab ? blkA : chunkB, ab ? chunkB : blkA);
      if (ab) op.add_pair((jobs[t].first - 1) * blkA, (jobs[t].second - 1) * chunkB);
      else op.add_pair((jobs[t].second - 1) * chunkB, (jobs[t].first - 1) * blkA);
    }
    if (ab) op.launch(ctx, A->data.d(), B->data.d(), tmpl.d(), false);
    else op.launch(ctx, B->data.d(), A->data.d(), tmpl.d(), false);
    book.commit(ctx, C, std::move(tmpl), nt, A->scalars.d(), nullptr);
    return;
  }
  // _contract_aliased_dense_ad! (contract_aliased.jl:244-365)
  Op A = aliased_r_last_dense(ctx, A0, r);
  const int PA = A->P();
  require(PC == PA, SB_ERR_ASSERTION, "C sparse prefix must equal A sparse prefix for dense-tail reduction");
  require(A->dims.back() == R, SB_ERR_DIM_MISMATCH, "Reduction size R mismatch between A dense tail and B");
  const int64_t chunkA = A->blksize() / R;
  require(C.blksize() == chunkA * chunkB, SB_ERR_DIM_MISMATCH, "C.blksize must equal chunkA*chunkB");
  Labels Awo(A.labels.begin() + PA, A.labels.end() - 1);
  Labels AB(Awo), BA(Bwo);
  AB.insert(AB.end(), Bwo.begin(), Bwo.end());
  BA.insert(BA.end(), Awo.begin(), Awo.end());
  bool ab;
  if (Cd == AB) ab = true;
  else if (Cd == BA) ab = false;
  else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense tail must be [A_dense_wo_r...,B_wo_r...] or [B_wo_r...,A_dense_wo_r...]");
  std::vector<int> src;
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    require(ia >= 0 && ia < PA, SB_ERR_LABEL, "C prefix label must come from A sparse prefix");
    src.push_back(ia + 1);
  }
  const int64_t nt = A->n_templates, blkA = A->blksize(), blkC = C.blksize();
  reset_aliased(ctx, C);
  C.data = DevBuf(ctx, nt * blkC * sizeof(double));
  GemmPlan gp;
  for (int64_t t = 0; t < nt; ++t) {
    gp.add_cblock(t * blkC, ab ? chunkA : chunkB, ab ? chunkB : chunkA);
    if (ab) gp.add_pair(t * blkA, 0, R, chunkA, chunkB);
    else gp.add_pair(0, t * blkA, R, chunkB, chunkA);
  }
  if (ab) gp.launch(ctx, A->data.d(), B->data.d(), C.data.d(), false, true);
  else gp.launch(ctx, B->data.d(), A->data.d(), C.data.d(), false, true);
  C.n_templates = nt;
  const int64_t n = A->nkeys;
  std::vector<std::vector<int64_t>> keys(n, std::vector<int64_t>(PC));
  std::vector<int64_t> lins(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int q = 0; q < PC; ++q) keys[i][q] = A->key(i)[src[q] - 1];
    lins[i] = lin0(keys[i].data(), C.dims.data(), PC);
  }
  std::vector<int64_t> p(n);
  std::iota(p.begin(), p.end(), 0);
  std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return lins[a] < lins[b]; });
  C.keys.clear();
  C.alias_ids.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    C.keys.insert(C.keys.end(), keys[p[i]].begin(), keys[p[i]].end());
    C.alias_ids[i] = A->alias_ids[p[i]];
  }
  C.nkeys = n;
  C.scalars = DevBuf(ctx, n * sizeof(double));
  if (n) {
    DevBuf dp = upload(ctx, p);
    SB_CK(launch_gather(A->scalars.d(), dp.as<int64_t>(), n, C.scalars.d(), ctx->stream));
    ctx->note_launch();
  }
}

void aliased_aa(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Label& r) {
  ctx->kernel_name = "contract_aliased! (Aliased x Aliased)";
  require(!has(lC, r), SB_ERR_LABEL, "rlab must be reduced");
  const int PC = C.P();
  const bool r_prefix = find(B0.labels, r) < B0->P();
  AliasBook book(C);
  reset_aliased(ctx, C);
  std::map<std::pair<int64_t, int64_t>, int> ctm;
  std::vector<std::pair<int64_t, int64_t>> jobs;
  std::vector<int64_t> k(PC);
  if (r_prefix) {  // _contract_aliased_prefix_outer_aa! (contract_aliased.jl:417-520)
    Op A = aliased_r_last_prefix(ctx, A0, r), B = aliased_r_last_prefix(ctx, B0, r);
    const int PA = A->P(), PB = B->P();
    require(C.blksize() == A->blksize() * B->blksize(), SB_ERR_DIM_MISMATCH, "C.blksize must equal A.blksize*B.blksize");
    Labels Ad(A.labels.begin() + PA, A.labels.end()), Bd(B.labels.begin() + PB, B.labels.end()), Cd(lC.begin() + PC, lC.end());
    Labels AB(Ad), BA(Bd);
    AB.insert(AB.end(), Bd.begin(), Bd.end());
    BA.insert(BA.end(), Ad.begin(), Ad.end());
    int order;
    if (Cd == AB) order = 1;
    else if (Cd == BA) order = 2;
    else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense must be [A_dense...,B_dense...] or [B_dense...,A_dense...]");
    std::vector<int> src;
    for (int j = 0; j < PC; ++j) {
      const int ia = find(A.labels, lC[j]);
      if (ia >= 0 && ia != PA - 1) src.push_back(ia + 1);
      else { const int ib = find(B.labels, lC[j]); require(ib >= 0 && ib < PB && !(lC[j] == r), SB_ERR_LABEL, "C prefix label not found in A or B"); src.push_back(-(ib + 1)); }
    }
    std::vector<int> jA{PA}, jB{PB};
    merge_join(*A, jA, *B, jB, [&](int64_t a, int64_t b) {
      auto key = std::make_pair(A->alias_ids[a], B->alias_ids[b]);
      auto it = ctm.find(key);
      int ct;
      if (it == ctm.end()) { jobs.push_back(key); ct = static_cast<int>(jobs.size()); ctm.emplace(key, ct); }
      else ct = it->second;
      for (int q = 0; q < PC; ++q) k[q] = src[q] > 0 ? A->key(a)[src[q] - 1] : B->key(b)[-src[q] - 1];
      book.contribute(k, ct, ScalarTerm{a, b});
    });
    const int64_t blkA = A->blksize(), blkB = B->blksize(), blkC = C.blksize(), nt = static_cast<int64_t>(jobs.size());
    DevBuf tmpl(ctx, nt * blkC * sizeof(double));
    OuterPlan op;
    for (int64_t t = 0; t < nt; ++t) {
      op.add_cblock(t * blkC, order == 1 ? blkA : blkB, order == 1 ? blkB : blkA);
      if (order == 1) op.add_pair((jobs[t].first - 1) * blkA, (jobs[t].second - 1) * blkB);
      else op.add_pair((jobs[t].second - 1) * blkB, (jobs[t].first - 1) * blkA);
    }
    if (order == 1) op.launch(ctx, A->data.d(), B->data.d(), tmpl.d(), false);
    else op.launch(ctx, B->data.d(), A->data.d(), tmpl.d(), false);
    book.commit(ctx, C, std::move(tmpl), nt, A->scalars.d(), B->scalars.d());
    return;
  }
  // _contract_aliased_dense_aa! (contract_aliased.jl:527-643)
  require(find(A0.labels, r) >= A0->P(), SB_ERR_LABEL, "rlab must be in A dense tail when it is in B dense tail");
  Op A = aliased_r_last_dense(ctx, A0, r), B = aliased_r_last_dense(ctx, B0, r);
  const int PA = A->P(), PB = B->P();
  const int64_t R = A->dims.back();
  require(B->dims.back() == R, SB_ERR_DIM_MISMATCH, "Reduction size mismatch");
  const int64_t chunkA = A->blksize() / R, chunkB = B->blksize() / R;
  require(C.blksize() == chunkA * chunkB, SB_ERR_DIM_MISMATCH, "C.blksize must equal chunkA*chunkB");
  Labels Awo(A.labels.begin() + PA, A.labels.end() - 1), Bwo(B.labels.begin() + PB, B.labels.end() - 1),
      Cd(lC.begin() + PC, lC.end());
  Labels AB(Awo), BA(Bwo);
  AB.insert(AB.end(), Bwo.begin(), Bwo.end());
  BA.insert(BA.end(), Awo.begin(), Awo.end());
  bool ab;
  if (Cd == AB) ab = true;
  else if (Cd == BA) ab = false;
  else fail(SB_ERR_UNSUPPORTED_LAYOUT, "C dense tail must be [A_dense_wo_r...,B_dense_wo_r...] or swapped");
  std::vector<int> srcA(PC, 0), srcB(PC, 0);
  for (int j = 0; j < PC; ++j) {
    const int ia = find(A.labels, lC[j]);
    if (ia >= 0) { require(ia < PA, SB_ERR_LABEL, "C prefix label must be in A prefix"); srcA[j] = ia + 1; }
    else { const int ib = find(B.labels, lC[j]); require(ib >= 0 && ib < PB, SB_ERR_LABEL, "C prefix label must be in B prefix"); srcB[j] = ib + 1; }
  }
  for (int64_t a = 0; a < A->nkeys; ++a)
    for (int64_t b = 0; b < B->nkeys; ++b) {
      auto key = std::make_pair(A->alias_ids[a], B->alias_ids[b]);
      auto it = ctm.find(key);
      int ct;
      if (it == ctm.end()) { jobs.push_back(key); ct = static_cast<int>(jobs.size()); ctm.emplace(key, ct); }
      else ct = it->second;
      for (int q = 0; q < PC; ++q) k[q] = srcA[q] ? A->key(a)[srcA[q] - 1] : B->key(b)[srcB[q] - 1];
      book.contribute(k, ct, ScalarTerm{a, b});
    }
  const int64_t blkA = A->blksize(), blkB = B->blksize(), blkC = C.blksize(), nt = static_cast<int64_t>(jobs.size());
  DevBuf tmpl(ctx, nt * blkC * sizeof(double));
  GemmPlan gp;
  for (int64_t t = 0; t < nt; ++t) {
    gp.add_cblock(t * blkC, ab ? chunkA : chunkB, ab ? chunkB : chunkA);
    if (ab) gp.add_pair((jobs[t].first - 1) * blkA, (jobs[t].second - 1) * blkB, R, chunkA, chunkB);
    else gp.add_pair((jobs[t].second - 1) * blkB, (jobs[t].first - 1) * blkA, R, chunkB, chunkA);
  }
  if (ab) gp.launch(ctx, A->data.d(), B->data.d(), tmpl.d(), false, true);
  else gp.launch(ctx, B->data.d(), A->data.d(), tmpl.d(), false, true);
  book.commit(ctx, C, std::move(tmpl), nt, A->scalars.d(), B->scalars.d());
}

void shared_aliased(Ctx* ctx, Tensor& C, const Labels& lC, const Op& A0, const Op& B0, const Labels& shared) {
  ctx->kernel_name = "contract_shared! (Aliased)";
  const int PC = C.P();
  const bool B_dense = B0->kind == DENSE;
  SharedPlan sp = plan_shared(lC, PC, A0, B0, shared, B_dense);
  Op A = permuted(ctx, A0, sp.permA);
  const int PA = A->P();
  const int nkA = static_cast<int>(sp.dkA.size());
  const int64_t M = prod(A->dims, PA, PA + nkA), K = prod(A->dims, PA + nkA, A->N());
  reset_aliased(ctx, C);
  AliasBook book(C);
  std::map<std::pair<int64_t, int64_t>, int> ctm;
  std::vector<std::pair<int64_t, int64_t>> jobs;
  std::vector<int64_t> k(PC);
  const bool athenb = sp.mode == Mode::AthenB;
  if (B_dense) {  // contract_aliased_shared.jl:103-302
    DenseSlices ds = dense_slices(ctx, B0, sp.shared_prefix, sp.red_dense, sp.dkB);
    const int64_t N = ds.N;
    require(K == ds.K, SB_ERR_DIM_MISMATCH, "Reduction extent mismatch between A dense tail and B");
    require(C.blksize() == M * N, SB_ERR_DIM_MISMATCH, "C.blksize must equal M*N");
    std::vector<int> csrc;
    for (int j = 0; j < PC; ++j) {
      const int ia = find(A.labels, lC[j]);
      require(ia >= 0 && ia < PA && !has(sp.shared_prefix, lC[j]), SB_ERR_LABEL, "C prefix label must come from A sparse prefix");
      csrc.push_back(ia + 1);
    }
    std::vector<int> jA;
    for (auto& l : sp.shared_prefix) jA.push_back(find(A.labels, l) + 1);
    for (int64_t iA = 0; iA < A->nkeys;) {
      const int64_t iA2 = advance_run(*A, iA, jA);
      int64_t slab = 0, stride = 1;
      for (size_t t = 0; t < jA.size(); ++t) {
        slab += (A->key(iA)[jA[t] - 1] - 1) * stride;
        stride *= ds.sp_dims[t];
      }
      for (int64_t a = iA; a < iA2; ++a) {
        auto key = std::make_pair(A->alias_ids[a], slab);
        auto it = ctm.find(key);
        int ct;
        if (it == ctm.end()) { jobs.push_back(key); ct = static_cast<int>(jobs.size()); ctm.emplace(key, ct); }
        else ct = it->second;
        for (int q = 0; q < PC; ++q) k[q] = A->key(a)[csrc[q] - 1];
        book.contribute(k, ct, ScalarTerm{a, -1});
      }
      iA = iA2;
    }
    const int64_t blkA = A->blksize(), blkC = C.blksize(), nt = static_cast<int64_t>(jobs.size());
    DevBuf tmpl(ctx, nt * blkC * sizeof(double));
    GemmPlan gp;
    for (int64_t t = 0; t < nt; ++t) {
      const int64_t ao = (jobs[t].first - 1) * blkA, bo = jobs[t].second * ds.slab;
      if (athenb) { gp.add_cblock(t * blkC, M, N); gp.add_pair(ao, bo, K, M, K); }
      else { gp.add_cblock(t * blkC, N, M); gp.add_pair(bo, ao, K, K, M); }
    }
    if (athenb) gp.launch(ctx, A->data.d(), ds.Bp->data.d(), tmpl.d(), false, false);
    else gp.launch(ctx, ds.Bp->data.d(), A->data.d(), tmpl.d(), true, true);
    book.commit(ctx, C, std::move(tmpl), nt, A->scalars.d(), nullptr);
    return;
  }
  // contract_aliased_shared.jl:325-523
  Op B = permuted(ctx, B0, sp.permB);
  const int PB = B->P();
  const int nred = static_cast<int>(sp.red_dense.size());
  const int64_t N = prod(B->dims, PB + nred, B->N());
  require(K == prod(B->dims, PB, PB + nred), SB_ERR_DIM_MISMATCH, "Reduction extent mismatch between A and B dense tails");
  require(C.blksize() == M * N, SB_ERR_DIM_MISMATCH, "C.blksize must equal M*N");
  auto src = csrc_AB(lC, PC, A, B, true);
  std::vector<int> jA, jB;
  for (auto& l : sp.shared_prefix) { jA.push_back(find(A.labels, l) + 1); jB.push_back(find(B.labels, l) + 1); }
  merge_join(*A, jA, *B, jB, [&](int64_t a, int64_t b) {
    auto key = std::make_pair(A->alias_ids[a], B->alias_ids[b]);
    auto it = ctm.find(key);
    int ct;
    if (it == ctm.end()) { jobs.push_back(key); ct = static_cast<int>(jobs.size()); ctm.emplace(key, ct); }
    else ct = it->second;
    for (int q = 0; q < PC; ++q) k[q] = src[q] > 0 ? A->key(a)[src[q] - 1] : B->key(b)[-src[q] - 1];
    book.contribute(k, ct, ScalarTerm{a, b});
  });
  const int64_t blkA = A->blksize(), blkB = B->blksize(), blkC = C.blksize(), nt = static_cast<int64_t>(jobs.size());
  DevBuf tmpl(ctx, nt * blkC * sizeof(double));
  GemmPlan gp;
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t ao = (jobs[t].first - 1) * blkA, bo = (jobs[t].second - 1) * blkB;
    if (athenb) { gp.add_cblock(t * blkC, M, N); gp.add_pair(ao, bo, K, M, K); }
    else { gp.add_cblock(t * blkC, N, M); gp.add_pair(bo, ao, K, K, M); }
  }
  if (athenb) gp.launch(ctx, A->data.d(), B->data.d(), tmpl.d(), false, false);
  else gp.launch(ctx, B->data.d(), A->data.d(), tmpl.d(), true, true);
  book.commit(ctx, C, std::move(tmpl), nt, A->scalars.d(), B->scalars.d());
}

}  // namespace

// ══════════════════════════ dispatch ═════════════════════════════════════

void contract(Ctx* ctx, Tensor& C, const Labels& lC, const Tensor& A, const Labels& lA, const Tensor& B,
              const Labels& lB) {
  require(static_cast<int>(lA.size()) == A.N(), SB_ERR_ASSERTION, "labelsA length must match A rank");
  require(static_cast<int>(lB.size()) == B.N(), SB_ERR_ASSERTION, "labelsB length must match B rank");
  require(static_cast<int>(lC.size()) == C.N(), SB_ERR_ASSERTION, "labelsC length must match C rank");
  Op oA = view(A, lA), oB = view(B, lB);
  if (C.kind == DENSE) {
    // contract_bs_bs_to_dense! (contract_bs_bs.jl:736-754): P_C = 0 sink.
    require_f64(A, "contract_bs_bs_to_dense!");
    require_f64(B, "contract_bs_bs_to_dense!");
    require(A.kind == BS && B.kind == BS, SB_ERR_UNSUPPORTED_TYPES, "dense C needs block-sparse A and B");
    require_uniform(A.ragged ? A : B, "contract_bs_bs_to_dense!");
    auto sink = make_tensor(ctx, BS, C.dims, C.N());
    contract(ctx, *sink, lC, A, lA, B, lB);
    const int64_t n = C.numel();
    C.data = DevBuf(ctx, n * sizeof(double));
    if (sink->nkeys) SB_CK(cudaMemcpyAsync(C.data.raw(), sink->data.raw(), n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    else SB_CK(cudaMemsetAsync(C.data.raw(), 0, n * sizeof(double), ctx->stream));
    return;
  }
  check_c_dims(C, lC, oA, oB);
  const bool ragged_in = (A.kind == BS && A.ragged) || (B.kind == BS && B.ragged);
  Labels shared, reduced;
  for (auto& l : lA)
    if (has(lB, l)) shared.push_back(l);
  for (auto& l : shared)
    if (!has(lC, l)) reduced.push_back(l);
  if (reduced.size() == 1) {
    require_f64(C, "single-label contract!");
    require_f64(A, "single-label contract!");
    require_f64(B, "single-label contract!");
    require(shared.size() == 1, SB_ERR_ASSERTION, "Expected exactly 1 shared label");
    const Label r = reduced[0];
    require(A.dims[find(lA, r)] == B.dims[find(lB, r)], SB_ERR_DIM_MISMATCH, "Dim mismatch on shared label " + lab_str(r));
    if (ragged_in) require_uniform(A.ragged ? A : B, "single-label contract!");
    const Kind c = C.kind, a = A.kind, b = B.kind;
    if (c == COO && a == COO && b == COO) return coo_coo(ctx, C, lC, oA, oB, r);
    if (c == BS && a == BS && b == BS) {
      if (find(lB, r) < B.P()) {
        Op A2 = r_to_last_prefix(ctx, oA, r), B2 = r_to_last_prefix(ctx, oB, r);
        return prefix_outer_bb(ctx, C, lC, A2, B2, r);
      }
      return dense_bb(ctx, C, lC, oA, oB, r);
    }
    if (c == BS && a == COO && b == BS) {
      Op A2 = coo_r_last_sorted(ctx, oA, r);
      if (find(lB, r) < B.P()) {
        Op B2 = r_to_last_prefix(ctx, oB, r);
        return coo_bs_prefix(ctx, C, lC, A2, B2, r);
      }
      return coo_bs_dense_index(ctx, C, lC, A2, oB, r);
    }
    if (c == BS && a == COO && b == DENSE) return coo_dense(ctx, C, lC, oA, oB, r);
    if (c == BS && a == BS && b == DENSE) {
      if (find(lA, r) < A.P()) return prefix_outer_bd(ctx, C, lC, oA, oB, r);
      return dense_bd(ctx, C, lC, oA, oB, r);
    }
    if (c == ALIASED && a == ALIASED && b == DENSE) return aliased_ad(ctx, C, lC, oA, oB, r);
    if (c == ALIASED && a == ALIASED && b == ALIASED) return aliased_aa(ctx, C, lC, oA, oB, r);
    if (c == ALIASED && a == COO && b == DENSE) return aliased_coo_dense(ctx, C, lC, oA, oB, r);
    fail(SB_ERR_UNSUPPORTED_TYPES, "no contract! kernel for this (C, A, B) storage combination");
  }
  const Kind c = C.kind, a = A.kind, b = B.kind;
  if (c == BS && a == BS && b == BS) return shared_bb(ctx, C, lC, oA, oB, shared);
  require_f64(C, "contract_shared!");
  require_f64(A, "contract_shared!");
  require_f64(B, "contract_shared!");
  if (ragged_in) require_uniform(A.ragged ? A : B, "contract_shared!");
  if (c == BS && a == BS && b == DENSE) return shared_bd(ctx, C, lC, oA, oB, shared);
  if (c == ALIASED && a == ALIASED && (b == DENSE || b == ALIASED)) return shared_aliased(ctx, C, lC, oA, oB, shared);
  fail(SB_ERR_UNSUPPORTED_TYPES, "no contract_shared! kernel for this (C, A, B) storage combination");
}

}  // namespace sb
