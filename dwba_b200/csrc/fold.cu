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

}  // namespace

extern "C" int dwba_fold(const dwba_fold_t* folds_dev, int n_folds, int max_rows, dwba_stream_t stream) {
  if (n_folds <= 0) return DWBA_OK;
  if (!folds_dev || max_rows < 0 || n_folds > 65535) return DWBA_ERR_INVALID_ARG;
  dim3 grid(dwba_grid_1d(max_rows, 256, 1024), n_folds);
  fold_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(folds_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
