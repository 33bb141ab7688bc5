// C++ restatement of SparseBackends' multi-label block-sparse contraction on the
// CPU, linked at run time to OpenBLAS.
//
// THIS FILE IS TEST INFRASTRUCTURE (the CPU baseline of the benchmark and a
// second oracle for the tests); the product path never calls it.
//
// It restates, for the uniform reference layout:
//   * NewBlockSparseSorted (src/blocksparse/storage.jl:3-9): keys sorted by the
//     1-based column-major prefix index (_prefix_lin, :16-18), one flat
//     column-major block of blksize values per key;
//   * Base.permutedims (storage.jl:188-264): remapped keys re-sorted, every
//     block gathered through the tail permutation (map_old, :220-261);
//   * contract_shared! BS x BS (ta/contract_bs_bs.jl:572-730): shared labels
//     split into shared-prefix and reduced-dense labels, the C dense tail's
//     grouping (_cdense_grouping_and_orders, :470-505), the operand
//     permutations (:513-567), the merge-join over the shared-prefix tuple
//     (_cmp_join_tuple / _advance_run, :430-464) and one
//     mul!(C, A, B, 1, 1) per matched pair (:700-726), a dgemm with beta = 1.
//
// The join compares the shared-prefix tuple from its last axis down, the order
// the keys are sorted in (the reference compares from the first axis; the two
// agree wherever the reference's merge finds every match).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using i64 = int64_t;

// cblas_dgemm of OpenBLAS with 64-bit integers (column-major = 102,
// no-transpose = 111, transpose = 112).
using dgemm_fn = void (*)(int, int, int, i64, i64, i64, double, const double*, i64, const double*, i64, double,
                          double*, i64);
dgemm_fn g_dgemm = nullptr;

struct T {
  std::vector<i64> dims;
  int n2 = 0;
  std::vector<i64> keys;    // nkeys x P, 1-based, sorted by prefix_lin
  std::vector<double> data;  // nkeys x blk, key order
  int N() const { return static_cast<int>(dims.size()); }
  int P() const { return N() - n2; }
  i64 blk() const {
    i64 b = 1;
    for (int i = P(); i < N(); ++i) b *= dims[i];
    return b;
  }
  i64 nkeys() const { return P() ? static_cast<i64>(keys.size()) / P() : (data.empty() ? 0 : 1); }
  const i64* key(i64 i) const { return keys.data() + i * P(); }
  const double* block(i64 i) const { return data.data() + i * blk(); }
};

void require(bool c, const char* msg) {
  if (!c) throw std::runtime_error(msg);
}

i64 prefix_lin(const i64* k, const std::vector<i64>& dims, int P) {
  i64 idx = 0, stride = 1;
  for (int d = 0; d < P; ++d) {
    idx += (k[d] - 1) * stride;
    stride *= dims[d];
  }
  return idx;
}

// Sort keys (and their blocks) by prefix_lin, stably.
void sort_keys(T& t) {
  const i64 n = t.nkeys(), P = t.P(), b = t.blk();
  if (P == 0 || n < 2) return;
  std::vector<i64> lin(n), p(n);
  for (i64 i = 0; i < n; ++i) lin[i] = prefix_lin(t.key(i), t.dims, static_cast<int>(P));
  std::iota(p.begin(), p.end(), 0);
  std::stable_sort(p.begin(), p.end(), [&](i64 a, i64 c) { return lin[a] < lin[c]; });
  std::vector<i64> k2(t.keys.size());
  std::vector<double> d2(t.data.size());
  for (i64 i = 0; i < n; ++i) {
    std::copy(t.key(p[i]), t.key(p[i]) + P, k2.begin() + i * P);
    std::copy(t.block(p[i]), t.block(p[i]) + b, d2.begin() + i * b);
  }
  t.keys.swap(k2);
  t.data.swap(d2);
}

// Base.permutedims (storage.jl:188-264); perm is 1-based, no prefix/tail crossing.
T permute(const T& A, const std::vector<int>& perm) {
  const int N = A.N(), P = A.P();
  require(static_cast<int>(perm.size()) == N, "perm length must equal N");
  for (int j = 0; j < P; ++j) require(perm[j] >= 1 && perm[j] <= P, "No-cross reorder violated (prefix)");
  for (int j = P; j < N; ++j) require(perm[j] > P && perm[j] <= N, "No-cross reorder violated (tail)");
  T B;
  B.n2 = A.n2;
  B.dims.resize(N);
  for (int j = 0; j < N; ++j) B.dims[j] = A.dims[perm[j] - 1];
  const i64 n = A.nkeys(), blk = A.blk();
  B.keys.resize(n * P);
  for (i64 i = 0; i < n; ++i)
    for (int j = 0; j < P; ++j) B.keys[i * P + j] = A.key(i)[perm[j] - 1];
  // tail gather: out index (col-major over new tail dims) -> old offset
  const int n2 = A.n2;
  std::vector<i64> ostride(n2), newdims(n2), src_stride(n2);
  {
    i64 s = 1;
    for (int t = 0; t < n2; ++t) {
      ostride[t] = s;
      s *= A.dims[P + t];
    }
    for (int t = 0; t < n2; ++t) {
      newdims[t] = B.dims[P + t];
      src_stride[t] = ostride[perm[P + t] - 1 - P];
    }
  }
  B.data.resize(A.data.size());
  std::vector<i64> idx(n2);
  for (i64 i = 0; i < n; ++i) {
    const double* src = A.block(i);
    double* dst = B.data.data() + i * blk;
    std::fill(idx.begin(), idx.end(), 0);
    i64 off = 0;
    for (i64 e = 0; e < blk; ++e) {
      dst[e] = src[off];
      for (int t = 0; t < n2; ++t) {  // odometer over the new tail, first axis fastest
        if (++idx[t] < newdims[t]) {
          off += src_stride[t];
          break;
        }
        off -= (newdims[t] - 1) * src_stride[t];
        idx[t] = 0;
      }
    }
  }
  sort_keys(B);
  return B;
}

int find(const std::vector<i64>& l, i64 x) {
  for (size_t i = 0; i < l.size(); ++i)
    if (l[i] == x) return static_cast<int>(i);
  return -1;
}

// _advance_run (contract_bs_bs.jl:455-464): end of the run of keys whose join
// tuple equals key i0's.
i64 advance_run(const T& X, i64 i0, const std::vector<int>& pos) {
  const i64 n = X.nkeys();
  if (pos.empty()) return n;
  i64 i = i0 + 1;
  for (; i < n; ++i) {
    bool same = true;
    for (int p : pos) same = same && X.key(i)[p] == X.key(i0)[p];
    if (!same) break;
  }
  return i;
}

int cmp_join(const i64* a, const i64* b, const std::vector<int>& pa, const std::vector<int>& pb) {
  for (int t = static_cast<int>(pa.size()) - 1; t >= 0; --t) {
    if (a[pa[t]] < b[pb[t]]) return -1;
    if (a[pa[t]] > b[pb[t]]) return 1;
  }
  return 0;
}

// contract_shared! BS x BS (contract_bs_bs.jl:572-730).
T contract_shared(const std::vector<i64>& dimsC, int n2C, const std::vector<i64>& lC, const T& A0,
                  const std::vector<i64>& lA0, const T& B0, const std::vector<i64>& lB0) {
  require(g_dgemm != nullptr, "dgemm not set (oref_set_dgemm)");
  const int PA0 = A0.P(), PB0 = B0.P(), NC = static_cast<int>(dimsC.size()), PC = NC - n2C;
  require(static_cast<int>(lA0.size()) == A0.N() && static_cast<int>(lB0.size()) == B0.N() &&
              static_cast<int>(lC.size()) == NC, "label counts must match ranks");
  std::vector<i64> shared;
  for (i64 l : lA0)
    if (find(lB0, l) >= 0) shared.push_back(l);
  std::vector<i64> sp, sd;
  for (i64 l : shared) {
    require(find(lC, l) < 0, "shared labels must be reduced");
    const bool ap = find(lA0, l) < PA0, bp = find(lB0, l) < PB0;
    require(ap == bp, "shared label crosses prefix/dense; not supported");
    (ap ? sp : sd).push_back(l);
  }
  std::vector<i64> red, keepA0, keepB0;
  for (int j = PA0; j < A0.N(); ++j) (find(sd, lA0[j]) >= 0 ? red : keepA0).push_back(lA0[j]);
  for (int j = PB0; j < B0.N(); ++j)
    if (find(sd, lB0[j]) < 0) keepB0.push_back(lB0[j]);
  // _cdense_grouping_and_orders (:470-505)
  std::vector<int> origin;  // 1 = from A, 0 = from B
  std::vector<i64> dkA, dkB;
  for (int j = PC; j < NC; ++j) {
    if (find(keepA0, lC[j]) >= 0) { origin.push_back(1); dkA.push_back(lC[j]); }
    else if (find(keepB0, lC[j]) >= 0) { origin.push_back(0); dkB.push_back(lC[j]); }
    else throw std::runtime_error("C dense label not found in the kept labels of A or B");
  }
  int firstA = -1, lastA = -1, firstB = -1, lastB = -1;
  for (int i = 0; i < static_cast<int>(origin.size()); ++i) {
    if (origin[i]) { if (firstA < 0) firstA = i; lastA = i; }
    else { if (firstB < 0) firstB = i; lastB = i; }
  }
  bool athenb;
  if (firstA < 0 || firstB < 0 || lastA < firstB) athenb = true;
  else if (lastB < firstA) athenb = false;
  else throw std::runtime_error("C dense tail interleaves A and B kept labels");
  require(dkA.size() == keepA0.size() && dkB.size() == keepB0.size(), "C dense tail must hold every kept label");
  // permutations (:513-567): [kept prefix, shared prefix | kept dense, reduced] and
  // [kept prefix, shared prefix | reduced, kept dense]
  std::vector<int> pA, pB;
  for (int j = 0; j < PA0; ++j)
    if (find(sp, lA0[j]) < 0) pA.push_back(j + 1);
  for (i64 l : sp) pA.push_back(find(lA0, l) + 1);
  for (i64 l : dkA) pA.push_back(find(lA0, l) + 1);
  for (i64 l : red) pA.push_back(find(lA0, l) + 1);
  for (int j = 0; j < PB0; ++j)
    if (find(sp, lB0[j]) < 0) pB.push_back(j + 1);
  for (i64 l : sp) pB.push_back(find(lB0, l) + 1);
  for (i64 l : red) pB.push_back(find(lB0, l) + 1);
  for (i64 l : dkB) pB.push_back(find(lB0, l) + 1);
  // operands whose permutation is the identity are used in place
  auto is_ident = [](const std::vector<int>& p) {
    for (size_t j = 0; j < p.size(); ++j)
      if (p[j] != static_cast<int>(j) + 1) return false;
    return true;
  };
  T Ap, Bp;
  if (!is_ident(pA)) Ap = permute(A0, pA);
  if (!is_ident(pB)) Bp = permute(B0, pB);
  const T& A = is_ident(pA) ? A0 : Ap;
  const T& B = is_ident(pB) ? B0 : Bp;
  std::vector<i64> lA, lB;
  for (int p : pA) lA.push_back(lA0[p - 1]);
  for (int p : pB) lB.push_back(lB0[p - 1]);
  const int PA = A.P(), PB = B.P();
  const int nkA = static_cast<int>(dkA.size()), nred = static_cast<int>(red.size());
  i64 M = 1, K = 1, N = 1, K2 = 1;
  for (int t = 0; t < nkA; ++t) M *= A.dims[PA + t];
  for (int t = nkA; t < A.n2; ++t) K *= A.dims[PA + t];
  for (int t = 0; t < nred; ++t) K2 *= B.dims[PB + t];
  for (int t = nred; t < B.n2; ++t) N *= B.dims[PB + t];
  require(K == K2, "Reduced dense extents mismatch between A and B");
  T C;
  C.dims = dimsC;
  C.n2 = n2C;
  require(C.blk() == M * N, "C.blksize must equal M*N");
  std::vector<int> src;  // >0: A prefix position + 1, <0: -(B prefix position + 1)
  for (int j = 0; j < PC; ++j) {
    const int ia = find(lA, lC[j]), ib = find(lB, lC[j]);
    if (ia >= 0 && ia < PA) src.push_back(ia + 1);
    else if (ib >= 0 && ib < PB) src.push_back(-(ib + 1));
    else throw std::runtime_error("C prefix label must come from A or B prefix");
  }
  std::vector<int> jA, jB;
  for (i64 l : sp) {
    jA.push_back(find(lA, l));
    jB.push_back(find(lB, l));
  }
  std::map<i64, std::pair<std::vector<i64>, i64>> cmap;  // prefix_lin -> (key, slot)
  std::vector<std::vector<double>> slots;
  std::vector<i64> ck(PC);
  const i64 nA = A.nkeys(), nB = B.nkeys();
  i64 iA = 0, iB = 0;
  while (iA < nA && iB < nB) {
    const int c = cmp_join(A.key(iA), B.key(iB), jA, jB);
    if (c < 0) { iA = advance_run(A, iA, jA); continue; }
    if (c > 0) { iB = advance_run(B, iB, jB); continue; }
    const i64 iA2 = advance_run(A, iA, jA), iB2 = advance_run(B, iB, jB);
    for (i64 a = iA; a < iA2; ++a)
      for (i64 b = iB; b < iB2; ++b) {
        for (int q = 0; q < PC; ++q) ck[q] = src[q] > 0 ? A.key(a)[src[q] - 1] : B.key(b)[-src[q] - 1];
        const i64 lin = prefix_lin(ck.data(), C.dims, PC);
        auto it = cmap.find(lin);
        if (it == cmap.end()) {  // _ensure_block!: a zero block
          slots.emplace_back(M * N, 0.0);
          it = cmap.emplace(lin, std::make_pair(ck, static_cast<i64>(slots.size()) - 1)).first;
        }
        double* Cm = slots[it->second.second].data();
        if (athenb)  // mul!(Cmat(M,N), Amat(M,K), Bmat(K,N), 1, 1)
          g_dgemm(102, 111, 111, M, N, K, 1.0, A.block(a), M, B.block(b), K, 1.0, Cm, M);
        else  // mul!(Cmat(N,M), transpose(Bmat), transpose(Amat), 1, 1)
          g_dgemm(102, 112, 112, N, M, K, 1.0, B.block(b), K, A.block(a), M, 1.0, Cm, N);
      }
    iA = iA2;
    iB = iB2;
  }
  C.keys.reserve(cmap.size() * PC);
  C.data.reserve(cmap.size() * M * N);
  for (auto& kv : cmap) {
    C.keys.insert(C.keys.end(), kv.second.first.begin(), kv.second.first.end());
    const auto& s = slots[kv.second.second];
    C.data.insert(C.data.end(), s.begin(), s.end());
  }
  return C;
}

// fuse_two_axes! for two prefix axes (blocksparse/conversions.jl:228-262):
// the fused key (k[a2] - 1) * d[a1] + k[a1] sits at a1, axis a2 is dropped,
// the blocks are unchanged; the keys are kept sorted.
T fuse_prefix(const T& A, int ax1, int ax2) {
  const int N = A.N(), P = A.P();
  const int a1 = std::min(ax1, ax2), a2 = std::max(ax1, ax2);
  require(a1 >= 1 && a2 <= P && a1 != a2, "prefix axes must be distinct and in 1:P");
  T B;
  B.n2 = A.n2;
  for (int i = 1; i <= N; ++i)
    if (i != a2) B.dims.push_back(i == a1 ? A.dims[a1 - 1] * A.dims[a2 - 1] : A.dims[i - 1]);
  const i64 n = A.nkeys();
  for (i64 r = 0; r < n; ++r) {
    const i64* k = A.key(r);
    for (int j = 1; j <= P; ++j) {
      if (j == a2) continue;
      B.keys.push_back(j == a1 ? (k[a2 - 1] - 1) * A.dims[a1 - 1] + k[a1 - 1] : k[j - 1]);
    }
  }
  B.data = A.data;
  sort_keys(B);
  return B;
}

struct Coo {
  std::vector<i64> dims;
  std::vector<i64> keys;  // nnz x N, 1-based
  std::vector<double> vals;
  int N() const { return static_cast<int>(dims.size()); }
  i64 nnz() const { return static_cast<i64>(vals.size()); }
  const i64* key(i64 i) const { return keys.data() + i * N(); }
};

// contract_prefix! COO x BS (contract_coo_bs.jl:51-124) for one reduced label r
// in B's prefix: A's keys with r last, sorted column-major
// (ensure_rlab_last_and_sorted, contract_coo.jl:48-82), B with r as its last
// prefix axis; for every A entry and B block with equal r,
// C[key] += a * B_block (_scale_add_block!, :4-10).
T contract_coo_prefix(const std::vector<i64>& dimsC, int n2C, const std::vector<i64>& lC, const Coo& A0,
                      const std::vector<i64>& lA0, const T& B0, const std::vector<i64>& lB0) {
  std::vector<i64> shared;
  for (i64 l : lA0)
    if (find(lB0, l) >= 0) shared.push_back(l);
  require(shared.size() == 1 && find(lC, shared[0]) < 0, "contract_prefix! reduces exactly one label");
  const i64 r = shared[0];
  const int NA = A0.N(), PB0 = B0.P(), NC = static_cast<int>(dimsC.size()), PC = NC - n2C;
  require(find(lB0, r) < PB0, "the reduced label must be in B's prefix");
  require(PC == NA + PB0 - 2, "PC must equal NA + PB - 2");
  // A: r last, keys sorted column-major (last axis slowest)
  std::vector<int> pa;
  for (int j = 0; j < NA; ++j)
    if (lA0[j] != r) pa.push_back(j);
  pa.push_back(find(lA0, r));
  Coo A;
  std::vector<i64> lA;
  for (int j : pa) {
    A.dims.push_back(A0.dims[j]);
    lA.push_back(lA0[j]);
  }
  std::vector<i64> order(A0.nnz());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](i64 x, i64 y) {
    for (int t = NA - 1; t >= 0; --t) {
      const i64 a = A0.key(x)[pa[t]], b = A0.key(y)[pa[t]];
      if (a != b) return a < b;
    }
    return false;
  });
  for (i64 e : order) {
    for (int j : pa) A.keys.push_back(A0.key(e)[j]);
    A.vals.push_back(A0.vals[e]);
  }
  // B: r to the last prefix position (r_to_last_prefix)
  std::vector<int> pb;
  const int br = find(lB0, r);
  for (int j = 0; j < PB0; ++j)
    if (j != br) pb.push_back(j + 1);
  pb.push_back(br + 1);
  for (int j = PB0; j < B0.N(); ++j) pb.push_back(j + 1);
  bool ident = true;
  for (size_t j = 0; j < pb.size(); ++j) ident = ident && pb[j] == static_cast<int>(j) + 1;
  T Bp;
  if (!ident) Bp = permute(B0, pb);
  const T& B = ident ? B0 : Bp;
  std::vector<i64> lB;
  for (int p : pb) lB.push_back(lB0[p - 1]);
  T C;
  C.dims = dimsC;
  C.n2 = n2C;
  require(C.blk() == B.blk(), "C.blksize must equal B.blksize");
  std::vector<int> src;  // >0: A position + 1, <0: -(B prefix position + 1)
  for (int j = 0; j < PC; ++j) {
    const int ia = find(lA, lC[j]), ib = find(lB, lC[j]);
    if (ia >= 0) src.push_back(ia + 1);
    else if (ib >= 0 && ib < B.P()) src.push_back(-(ib + 1));
    else throw std::runtime_error("C prefix label must come from A or B prefix");
  }
  const int aR = NA - 1, bR = B.P() - 1;
  const i64 blk = B.blk();
  std::map<i64, std::pair<std::vector<i64>, i64>> cmap;
  std::vector<std::vector<double>> slots;
  std::vector<i64> ck(PC);
  i64 iA = 0, iB = 0;
  const i64 nA = A.nnz(), nB = B.nkeys();
  while (iA < nA && iB < nB) {
    const i64 rA = A.key(iA)[aR], rB = B.key(iB)[bR];
    if (rA < rB) { while (iA < nA && A.key(iA)[aR] == rA) ++iA; continue; }
    if (rB < rA) { while (iB < nB && B.key(iB)[bR] == rB) ++iB; continue; }
    const i64 blo = iB;
    while (iB < nB && B.key(iB)[bR] == rA) ++iB;
    for (; iA < nA && A.key(iA)[aR] == rA; ++iA)
      for (i64 b = blo; b < iB; ++b) {
        for (int q = 0; q < PC; ++q) ck[q] = src[q] > 0 ? A.key(iA)[src[q] - 1] : B.key(b)[-src[q] - 1];
        const i64 lin = prefix_lin(ck.data(), C.dims, PC);
        auto it = cmap.find(lin);
        if (it == cmap.end()) {
          slots.emplace_back(blk, 0.0);
          it = cmap.emplace(lin, std::make_pair(ck, static_cast<i64>(slots.size()) - 1)).first;
        }
        double* c = slots[it->second.second].data();
        const double a = A.vals[iA];
        const double* x = B.block(b);
        for (i64 e = 0; e < blk; ++e) c[e] += a * x[e];
      }
  }
  for (auto& kv : cmap) {
    C.keys.insert(C.keys.end(), kv.second.first.begin(), kv.second.first.end());
    const auto& sl = slots[kv.second.second];
    C.data.insert(C.data.end(), sl.begin(), sl.end());
  }
  return C;
}

thread_local std::string g_err;

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

}  // namespace

extern "C" {

void oref_set_dgemm(void* fn) { g_dgemm = reinterpret_cast<dgemm_fn>(fn); }

const char* oref_last_error() { return g_err.c_str(); }

// A block-sparse tensor from (dims, n2, keys nkeys x P row-major 1-based, data
// nkeys x blksize in the order of keys); the keys are sorted here.
int oref_new(int nd, const int64_t* dims, int n2, int64_t nkeys, const int64_t* keys, const double* data,
             void** out) {
  return guard([&] {
    require(out != nullptr && nd >= 0 && n2 >= 0 && n2 <= nd && nkeys >= 0, "bad arguments");
    auto* t = new T;
    t->dims.assign(dims, dims + nd);
    t->n2 = n2;
    const int P = nd - n2;
    t->keys.assign(keys, keys + nkeys * P);
    t->data.assign(data, data + nkeys * t->blk());
    sort_keys(*t);
    *out = t;
  });
}

void oref_free(void* t) { delete static_cast<T*>(t); }

int oref_info(void* t, int64_t* nkeys, int64_t* blksize) {
  return guard([&] {
    const T& x = *static_cast<T*>(t);
    *nkeys = x.nkeys();
    *blksize = x.blk();
  });
}

int oref_export(void* t, int64_t* keys, double* data) {
  return guard([&] {
    const T& x = *static_cast<T*>(t);
    if (keys) std::copy(x.keys.begin(), x.keys.end(), keys);
    if (data) std::copy(x.data.begin(), x.data.end(), data);
  });
}

// contract! for three block-sparse tensors with two or more shared labels
// (contract_shared!); labels are int64 ids.  *out receives a new C.
int oref_contract_shared(int ndC, const int64_t* dimsC, int n2C, const int64_t* lC, void* A, const int64_t* lA,
                         void* B, const int64_t* lB, void** out) {
  return guard([&] {
    const T& a = *static_cast<T*>(A);
    const T& b = *static_cast<T*>(B);
    std::vector<i64> dc(dimsC, dimsC + ndC), lc(lC, lC + ndC), la(lA, lA + a.N()), lb(lB, lB + b.N());
    *out = new T(contract_shared(dc, n2C, lc, a, la, b, lb));
  });
}

// fuse_two_axes! of two prefix axes (1-based); *out receives a new tensor.
int oref_fuse_prefix(void* A, int ax1, int ax2, void** out) {
  return guard([&] { *out = new T(fuse_prefix(*static_cast<T*>(A), ax1, ax2)); });
}

// contract_prefix! (COO x block-sparse, one reduced label in B's prefix); the
// COO operand as (nd, dims, nnz, keys nnz x nd row-major 1-based, vals).
int oref_contract_coo_prefix(int ndC, const int64_t* dimsC, int n2C, const int64_t* lC, int ndA, const int64_t* dimsA,
                             int64_t nnz, const int64_t* keysA, const double* valsA, const int64_t* lA, void* B,
                             const int64_t* lB, void** out) {
  return guard([&] {
    Coo a;
    a.dims.assign(dimsA, dimsA + ndA);
    a.keys.assign(keysA, keysA + nnz * ndA);
    a.vals.assign(valsA, valsA + nnz);
    const T& b = *static_cast<T*>(B);
    std::vector<i64> dc(dimsC, dimsC + ndC), lc(lC, lC + ndC), la(lA, lA + ndA), lb(lB, lB + b.N());
    *out = new T(contract_coo_prefix(dc, n2C, lc, a, la, b, lb));
  });
}

}  // extern "C"
