// Vector-space kernels for Krylov solvers: chunked deterministic dot products,
// elementwise maps (axpy / axpby / copy / multiply), scale, fill and the
// key-union block add.  All HBM-bound; every floating-point step is an
// explicitly rounded double operation so results do not depend on contraction
// choices of the compiler, and reductions run in a fixed order so repeated
// calls give identical bits.
#include <algorithm>

#include "sb_kernels.hpp"

namespace sb {
namespace {

constexpr int kDotThreads = 256;

// One CTA per chunk: partial[c] = sum_t (s*x[t]) * (s*y[t]) in a fixed
// thread-stride-then-tree order.
__global__ void __launch_bounds__(kDotThreads)
    k_dot_chunks(const double* __restrict__ X, const double* __restrict__ Y, const double* __restrict__ S,
                 const DotChunk* __restrict__ chunks, double* __restrict__ partial) {
  __shared__ double red[kDotThreads];
  const DotChunk c = chunks[blockIdx.x];
  const double* x = X + c.x_off;
  const double* y = Y + c.y_off;
  // a chunk is at most kDotChunk = 4 * kDotThreads elements: every thread
  // issues its (up to) four loads of each operand before the first FMA
  constexpr int kPer = kDotChunk / kDotThreads;
  double xv[kPer], yv[kPer];
#pragma unroll
  for (int r = 0; r < kPer; ++r) {
    const int t = threadIdx.x + r * kDotThreads;
    xv[r] = t < c.len ? x[t] : 0.0;
    yv[r] = t < c.len ? y[t] : 0.0;
  }
  const double sc = c.s_idx < 0 ? 1.0 : S[c.s_idx];
  double acc = 0.0;
#pragma unroll
  for (int r = 0; r < kPer; ++r)
    acc = c.s_idx < 0 ? __fma_rn(xv[r], yv[r], acc) : __fma_rn(__dmul_rn(sc, xv[r]), __dmul_rn(sc, yv[r]), acc);
  red[threadIdx.x] = acc;
  __syncthreads();
#pragma unroll
  for (int s = kDotThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// out[0] = sum of partial[0..n) in a fixed order (one CTA).
__global__ void __launch_bounds__(1024) k_sum_ordered(const double* __restrict__ partial, int64_t n,
                                                      double* __restrict__ out) {
  __shared__ double red[1024];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 1024) acc = __dadd_rn(acc, partial[i]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

__global__ void k_map(double* __restrict__ R, const double* __restrict__ A, int64_t n, int op, double alpha,
                      double beta) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double r = R[i];
    const double a = A ? A[i] : 0.0;
    double v;
    switch (op) {
      case kMapAxpy: v = __dadd_rn(r, __dmul_rn(alpha, a)); break;
      case kMapAxpby: v = __dadd_rn(__dmul_rn(beta, r), __dmul_rn(alpha, a)); break;
      case kMapCopy: v = a; break;
      case kMapMul: v = __dmul_rn(r, a); break;
      case kMapScale: v = __dmul_rn(alpha, r); break;
      default: v = alpha; break;  // kMapFill
    }
    R[i] = v;
  }
}

// C block = A block (A only), 0 + B block (B only) or A + B (both): the
// rounding of copy(A) followed by `c += b` over a zero-initialised new block.
__global__ void k_add_blocks(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C,
                             const AddBlock* __restrict__ items) {
  const AddBlock it = items[blockIdx.y];
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < it.len;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double v;
    if (it.b_off < 0) v = A[it.a_off + e];
    else v = __dadd_rn(it.a_off >= 0 ? A[it.a_off + e] : 0.0, B[it.b_off + e]);
    C[it.c_off + e] = v;
  }
}

unsigned grid_1d(int64_t n, int threads) {
  const int64_t g = (n + threads - 1) / threads;
  return static_cast<unsigned>(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace

cudaError_t launch_dot_chunks(const double* X, const double* Y, const double* S, const DotChunk* d_chunks,
                              int64_t nchunks, double* d_partial, double* d_out, cudaStream_t s) {
  if (nchunks <= 0) return cudaMemsetAsync(d_out, 0, sizeof(double), s);
  if (nchunks > 0x7fffffffLL) return cudaErrorInvalidValue;
  k_dot_chunks<<<static_cast<unsigned>(nchunks), kDotThreads, 0, s>>>(X, Y, S, d_chunks, d_partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_ordered<<<1, 1024, 0, s>>>(d_partial, nchunks, d_out);
  return cudaGetLastError();
}

cudaError_t launch_map(double* R, const double* A, int64_t n, int op, double alpha, double beta, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_map<<<grid_1d(n, 256), 256, 0, s>>>(R, A, n, op, alpha, beta);
  return cudaGetLastError();
}

cudaError_t launch_add_blocks(const double* A, const double* B, double* C, const AddBlock* d_items, int64_t n,
                              int64_t max_len, cudaStream_t s) {
  if (n <= 0 || max_len <= 0) return cudaSuccess;
  if (n > 65535) {
    // grid.y is limited to 65535: launch in slices of items
    for (int64_t b = 0; b < n; b += 65535) {
      const cudaError_t e = launch_add_blocks(A, B, C, d_items + b, std::min<int64_t>(65535, n - b), max_len, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  const unsigned gx = static_cast<unsigned>(std::min<int64_t>((max_len + 255) / 256, 64));
  k_add_blocks<<<dim3(gx, static_cast<unsigned>(n)), 256, 0, s>>>(A, B, C, d_items);
  return cudaGetLastError();
}

}  // namespace sb
