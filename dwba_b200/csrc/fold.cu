// Operand folds: a = T (f .* g) with T diagonal (weights), tridiagonal (outer
// CC fold) or pentadiagonal (exchange inner CC fold).
//
// These replace the density products of dwba_matrix_elements.py:1028-1046
// (rho = chi_f*chi_i, u_f*u_i, u_f*chi_i, chi_f*u_i, optionally times the
// Simpson weights) combined with the node-set operators built in nodes.cu.
#include "common.cuh"

namespace {

template <int H>
__device__ __forceinline__ double fold_row(const dwba_fold_t& f, int i) {
  double acc = 0.0;
  const double* __restrict__ op = f.op_dev + (int64_t)(2 * H + 1) * i;
#pragma unroll
  for (int d = -H; d <= H; ++d) {
    const int k = i + d;
    if (k >= 0 && k < f.n_src) acc += op[d + H] * (f.f_dev[k] * f.g_dev[k]);
  }
  return acc;
}

__global__ void fold_kernel(const dwba_fold_t* __restrict__ folds) {
  const dwba_fold_t f = folds[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n_clear; i += gridDim.x * blockDim.x) {
    double v = 0.0;
    if (i < f.n_out) {
      if (f.half_band == 0) v = fold_row<0>(f, i);
      else if (f.half_band == 1) v = fold_row<1>(f, i);
      else v = fold_row<2>(f, i);
    }
    f.out_dev[i] = v;
  }
}

// One output row of a multi-fold, a factor at a time. (Measured slower on the 64-energy sweep:
// issuing the loads of two or more factors before their products, 8.3 ms and up; the factors
// spread over the warps of a CTA, 10.0 ms; against 7.3 ms for this form.)
template <int H>
__device__ __forceinline__ void fold_multi_row(const dwba_fold_multi_t& m, int n_f, int n_src, int i) {
  double tap[2 * H + 1], gv[2 * H + 1];
  const double* __restrict__ op = m.op_dev + (int64_t)(2 * H + 1) * i;
  const double* __restrict__ g = m.g_dev;
#pragma unroll
  for (int d = -H; d <= H; ++d) {
    const int k = i + d;
    const bool in = k >= 0 && k < n_src;
    tap[d + H] = in ? op[d + H] : 0.0;
    gv[d + H] = in ? g[k] : 0.0;
  }
  for (int t = 0; t < n_f; ++t) {
    const double* __restrict__ f = m.f_dev[t];
    double acc = 0.0;
#pragma unroll
    for (int d = -H; d <= H; ++d) {
      const int k = i + d;
      if (k >= 0 && k < n_src) acc += tap[d + H] * (f[k] * gv[d + H]);
    }
    m.out_dev[t][i] = acc;
  }
}

__global__ void fold_multi_kernel(const dwba_fold_multi_t* __restrict__ folds) {
  // this CTA's descriptor in shared memory: every row reads its factor and output addresses
  // (7.4-7.7 ms against 8.2 ms for the folds of the 64-energy sweep when read from global memory)
  __shared__ dwba_fold_multi_t m;
  {
    constexpr int W = (int)(sizeof(dwba_fold_multi_t) / sizeof(unsigned long long));
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(folds + blockIdx.y);
    for (int w = threadIdx.x; w < W; w += blockDim.x) reinterpret_cast<unsigned long long*>(&m)[w] = src[w];
  }
  __syncthreads();
  const int n_f = m.n_f, H = m.half_band, n_out = m.n_out, n_src = m.n_src, n_clear = m.n_clear;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_clear; i += gridDim.x * blockDim.x) {
    if (i < n_out) {
      if (H == 0) fold_multi_row<0>(m, n_f, n_src, i);
      else if (H == 1) fold_multi_row<1>(m, n_f, n_src, i);
      else fold_multi_row<2>(m, n_f, n_src, i);
    } else {
      for (int t = 0; t < n_f; ++t) m.out_dev[t][i] = 0.0;
    }
  }
}

#ifndef DWBA_FOLD_THREADS
#define DWBA_FOLD_THREADS 128
#endif
#ifndef DWBA_FOLD_FILL
#define DWBA_FOLD_FILL 512 // CTAs per SM the launch aims for
#endif
// Row blocks per fold: enough CTAs in total to fill the GPU (DWBA_FOLD_FILL per SM),
// never more than the longest fold needs. The kernels stride over the rows of their fold, so a
// batch of folds of very different lengths launches no CTAs that find no rows.
int fold_grid_x(int max_rows, int n_folds) {
  const int need = (max_rows + DWBA_FOLD_THREADS - 1) / DWBA_FOLD_THREADS;
  const int fill = (int)(((int64_t)148 * DWBA_FOLD_FILL + n_folds - 1) / n_folds);
  return need < fill ? (need > 0 ? need : 1) : (fill > 0 ? fill : 1);
}

}  // namespace

extern "C" int dwba_fold_multi(const dwba_fold_multi_t* folds_dev, int n_folds, int max_rows, dwba_stream_t stream) {
  if (n_folds <= 0) return DWBA_OK;
  if (!folds_dev || max_rows < 0 || n_folds > 65535) return DWBA_ERR_INVALID_ARG;
  dim3 grid(fold_grid_x(max_rows, n_folds), n_folds);
  fold_multi_kernel<<<grid, DWBA_FOLD_THREADS, 0, (cudaStream_t)stream>>>(folds_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

extern "C" int dwba_fold(const dwba_fold_t* folds_dev, int n_folds, int max_rows, dwba_stream_t stream) {
  if (n_folds <= 0) return DWBA_OK;
  if (!folds_dev || max_rows < 0 || n_folds > 65535) return DWBA_ERR_INVALID_ARG;
  dim3 grid(fold_grid_x(max_rows, n_folds), n_folds);
  fold_kernel<<<grid, DWBA_FOLD_THREADS, 0, (cudaStream_t)stream>>>(folds_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
