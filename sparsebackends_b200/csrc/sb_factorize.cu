// Device kernels of the block factorisations (QR and SVD truncation).
//
// * Householder QR of a column-major m x n matrix, one reflector at a time:
//   k_house_gen forms reflector j with LAPACK's dlarfg convention
//   (beta = -sign(alpha) * ||x||, tau = (beta - alpha) / beta, v = x / (alpha - beta),
//   H = I when the sub-column is zero), so Q and R agree with LAPACK
//   geqrf/orgqr up to rounding; k_house_apply applies H_j to a range of
//   columns, one CTA per column.
// * One-sided (Hestenes) Jacobi SVD of many small row-major matrices, one CTA
//   per matrix: rows are rotated pairwise until orthogonal, U accumulates the
//   rotations; singular values are the final row norms (high relative
//   accuracy, which the relative cutoff of the truncation needs).
// Every loop is bounded; a Jacobi solve that has not converged after
// max_sweeps sweeps raises a status flag the host reads.
#include <algorithm>

#include "sb_kernels.hpp"

namespace sb {
namespace {

constexpr int kFacThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
  // fixed-order tree reduction over kFacThreads threads; result broadcast
  red[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = kFacThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kFacThreads)
    k_house_gen(double* __restrict__ M, int64_t ld, int64_t m, int64_t j, double* __restrict__ tau) {
  __shared__ double red[kFacThreads];
  __shared__ double scal;
  double* col = M + j * ld;
  double acc = 0.0;
  for (int64_t i = j + 1 + threadIdx.x; i < m; i += kFacThreads) acc = __fma_rn(col[i], col[i], acc);
  const double xn2 = block_sum(acc, red);
  if (threadIdx.x == 0) {
    const double alpha = col[j];
    if (xn2 == 0.0) {
      tau[j] = 0.0;
      scal = 0.0;
    } else {
      const double nrm = sqrt(__fma_rn(alpha, alpha, xn2));
      const double beta = alpha >= 0.0 ? -nrm : nrm;
      tau[j] = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
      col[j] = beta;
    }
  }
  __syncthreads();
  const double s = scal;
  if (s != 0.0)
    for (int64_t i = j + 1 + threadIdx.x; i < m; i += kFacThreads) col[i] = __dmul_rn(col[i], s);
}

// T[:, c] = (I - tau_j v v^T) T[:, c] for c in [c0, c0 + gridDim.x); v_j = 1,
// v_i = V[i + j*ldv] for i > j; rows below j only.
__global__ void __launch_bounds__(kFacThreads)
    k_house_apply(const double* __restrict__ V, int64_t ldv, double* __restrict__ T, int64_t ldt, int64_t m,
                  int64_t j, int64_t c0, const double* __restrict__ tau) {
  __shared__ double red[kFacThreads];
  const double t = tau[j];
  if (t == 0.0) return;
  const double* v = V + j * ldv;
  double* col = T + (c0 + blockIdx.x) * ldt;
  double acc = 0.0;
  for (int64_t i = j + 1 + threadIdx.x; i < m; i += kFacThreads) acc = __fma_rn(v[i], col[i], acc);
  const double s = block_sum(acc, red);
  const double w = __dmul_rn(t, __dadd_rn(col[j], s));
  if (threadIdx.x == 0) col[j] = __dsub_rn(col[j], w);
  for (int64_t i = j + 1 + threadIdx.x; i < m; i += kFacThreads) col[i] = __fma_rn(-v[i], w, col[i]);
}

__global__ void k_identity_cols(double* __restrict__ Q, int64_t m, int64_t k) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < m * k;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    Q[e] = (e % m == e / m) ? 1.0 : 0.0;
}

__global__ void k_upper(const double* __restrict__ M, int64_t m, int64_t k, int64_t n, double* __restrict__ R) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < k * n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e % k, c = e / k;
    R[e] = r <= c ? M[r + c * m] : 0.0;
  }
}

__global__ void k_gather_2d(const double* __restrict__ src, double* __restrict__ dst, const double* __restrict__ scale,
                            const Gather2D* __restrict__ items) {
  const Gather2D it = items[blockIdx.y];
  const int64_t n = it.rows * it.cols;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e % it.rows, c = e / it.rows;
    const double v = src[it.src_off + r * it.src_rs + c * it.src_cs];
    dst[it.dst_off + r * it.dst_rs + c * it.dst_cs] = it.s_idx >= 0 ? __dmul_rn(v, scale[it.s_idx]) : v;
  }
}

__global__ void __launch_bounds__(kFacThreads)
    k_svd_rows(double* __restrict__ A, double* __restrict__ Vt, double* __restrict__ U, double* __restrict__ S,
               const SvdGroup* __restrict__ groups, int max_sweeps, int* __restrict__ status) {
  __shared__ double red[kFacThreads];
  __shared__ double Us[kSvdMaxRows * kSvdMaxRows];
  __shared__ double nrm[kSvdMaxRows];
  __shared__ int perm[kSvdMaxRows];
  const SvdGroup g = groups[blockIdx.x];
  const int m = g.m;
  const int64_t n = g.n;
  double* a = A + g.a_off;
  for (int e = threadIdx.x; e < m * m; e += kFacThreads) Us[e] = (e % m == e / m) ? 1.0 : 0.0;
  __syncthreads();
  // Rotation threshold |gamma| > tol * sqrt(alpha * beta) with tol = n * eps,
  // the rounding bound of the length-n dot products: below it the rows are
  // orthogonal to working accuracy.  (A tighter threshold makes rank-deficient
  // groups rotate rounding-level rows forever.)
  const double eps = 2.220446049250313e-16;
  const double tol = eps * static_cast<double>(n > 1 ? n : 1);
  // Rows with norm below eps * ||A||_F are rounding noise: they take part in
  // no rotation (rotating them against each other never settles).
  double fro = 0.0;
  for (int64_t i = threadIdx.x; i < static_cast<int64_t>(m) * n; i += kFacThreads) fro = __fma_rn(a[i], a[i], fro);
  const double tiny = eps * eps * block_sum(fro, red);
  bool rotated = true;
  int sweep = 0;
  for (; sweep < max_sweeps && rotated; ++sweep) {
    rotated = false;
    for (int p = 0; p < m - 1; ++p) {
      for (int q = p + 1; q < m; ++q) {
        double* rp = a + static_cast<int64_t>(p) * n;
        double* rq = a + static_cast<int64_t>(q) * n;
        double sa = 0.0, sb2 = 0.0, sc = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += kFacThreads) {
          const double x = rp[i], y = rq[i];
          sa = __fma_rn(x, x, sa);
          sb2 = __fma_rn(y, y, sb2);
          sc = __fma_rn(x, y, sc);
        }
        const double alpha = block_sum(sa, red);
        const double beta = block_sum(sb2, red);
        const double gamma = block_sum(sc, red);
        // uniform across the CTA (reduced values)
        if (alpha <= tiny || beta <= tiny || gamma == 0.0 || fabs(gamma) <= tol * sqrt(alpha) * sqrt(beta)) continue;
        rotated = true;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + hypot(1.0, zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t);
        const double sn = cs * t;
        for (int64_t i = threadIdx.x; i < n; i += kFacThreads) {
          const double x = rp[i], y = rq[i];
          rp[i] = cs * x - sn * y;
          rq[i] = sn * x + cs * y;
        }
        if (threadIdx.x < m) {
          const double x = Us[threadIdx.x + p * m], y = Us[threadIdx.x + q * m];
          Us[threadIdx.x + p * m] = cs * x - sn * y;
          Us[threadIdx.x + q * m] = sn * x + cs * y;
        }
        __syncthreads();
      }
    }
  }
  if (rotated && threadIdx.x == 0) atomicExch(status, 1);  // not converged within max_sweeps
  // singular values = row norms, sorted descending (stable in row index)
  for (int p = 0; p < m; ++p) {
    const double* rp = a + static_cast<int64_t>(p) * n;
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += kFacThreads) s = __fma_rn(rp[i], rp[i], s);
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) nrm[p] = sqrt(t);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int p = 0; p < m; ++p) perm[p] = p;
    for (int p = 1; p < m; ++p) {
      const int x = perm[p];
      int q = p - 1;
      while (q >= 0 && nrm[perm[q]] < nrm[x]) {
        perm[q + 1] = perm[q];
        --q;
      }
      perm[q + 1] = x;
    }
  }
  __syncthreads();
  for (int r = 0; r < m; ++r) {
    const int p = perm[r];
    const double s = nrm[p];
    const double inv = s > 0.0 ? 1.0 / s : 0.0;
    const double* rp = a + static_cast<int64_t>(p) * n;
    double* out = Vt + g.a_off + static_cast<int64_t>(r) * n;
    for (int64_t i = threadIdx.x; i < n; i += kFacThreads) out[i] = s > 0.0 ? rp[i] * inv : 0.0;
    if (threadIdx.x < m) U[g.u_off + threadIdx.x + static_cast<int64_t>(r) * m] = Us[threadIdx.x + p * m];
    if (threadIdx.x == 0) S[g.s_off + r] = s;
  }
}

unsigned grid_1d(int64_t n) {
  const int64_t g = (n + 255) / 256;
  return static_cast<unsigned>(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace

cudaError_t launch_householder_qr(double* M, int64_t m, int64_t n, double* tau, cudaStream_t s, int64_t* launches) {
  const int64_t k = std::min(m, n);
  for (int64_t j = 0; j < k; ++j) {
    k_house_gen<<<1, kFacThreads, 0, s>>>(M, m, m, j, tau);
    ++*launches;
    const int64_t nc = n - j - 1;
    for (int64_t c = 0; c < nc; c += 65535) {
      const unsigned g = static_cast<unsigned>(std::min<int64_t>(65535, nc - c));
      k_house_apply<<<g, kFacThreads, 0, s>>>(M, m, M, m, m, j, j + 1 + c, tau);
      ++*launches;
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_householder_form_q(const double* M, int64_t m, int64_t k, const double* tau, double* Q,
                                      cudaStream_t s, int64_t* launches) {
  if (m <= 0 || k <= 0) return cudaSuccess;
  k_identity_cols<<<grid_1d(m * k), 256, 0, s>>>(Q, m, k);
  ++*launches;
  for (int64_t j = k - 1; j >= 0; --j) {
    const int64_t nc = k - j;
    for (int64_t c = 0; c < nc; c += 65535) {
      const unsigned g = static_cast<unsigned>(std::min<int64_t>(65535, nc - c));
      k_house_apply<<<g, kFacThreads, 0, s>>>(M, m, Q, m, m, j, j + c, tau);
      ++*launches;
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_upper(const double* M, int64_t m, int64_t k, int64_t n, double* R, cudaStream_t s) {
  if (k <= 0 || n <= 0) return cudaSuccess;
  k_upper<<<grid_1d(k * n), 256, 0, s>>>(M, m, k, n, R);
  return cudaGetLastError();
}

cudaError_t launch_gather_2d(const double* src, double* dst, const double* scale, const Gather2D* d_items, int64_t n,
                             int64_t max_elems, cudaStream_t s) {
  if (n <= 0 || max_elems <= 0) return cudaSuccess;
  for (int64_t b = 0; b < n; b += 65535) {
    const unsigned gy = static_cast<unsigned>(std::min<int64_t>(65535, n - b));
    const unsigned gx = static_cast<unsigned>(std::min<int64_t>((max_elems + 255) / 256, 64));
    k_gather_2d<<<dim3(gx, gy), 256, 0, s>>>(src, dst, scale, d_items + b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_svd_rows(double* A, double* Vt, double* U, double* S, const SvdGroup* d_groups, int64_t ngroups,
                            int max_sweeps, int* d_status, cudaStream_t s) {
  if (ngroups <= 0) return cudaSuccess;
  if (ngroups > 0x7fffffffLL) return cudaErrorInvalidValue;
  k_svd_rows<<<static_cast<unsigned>(ngroups), kFacThreads, 0, s>>>(A, Vt, U, S, d_groups, max_sweeps, d_status);
  return cudaGetLastError();
}

}  // namespace sb
