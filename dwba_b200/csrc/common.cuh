// Shared helpers for the dwba_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/dwba_b200.h"

#define DWBA_CHECK_LAUNCH()                          \
  do {                                               \
    cudaError_t e_ = cudaGetLastError();             \
    if (e_ != cudaSuccess) return DWBA_ERR_CUDA;     \
  } while (0)

static inline int dwba_grid_1d(int64_t n, int threads, int cap = 1 << 30) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

// IEEE arithmetic without contraction, where a value must match the
// reference's NumPy expression to the last bit.
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }

// Largest j in [0, n) with r[j] <= x (requires r[0] <= x), i.e. upper_bound - 1.
__device__ __forceinline__ int dwba_floor_index(const double* __restrict__ r, int n, double x) {
  int lo = 0, hi = n;  // invariant: r[lo] <= x < r[hi] (r[n] = +inf)
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (r[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// First k in [0, n] with r[k] >= x (numpy searchsorted side='left').
__device__ __forceinline__ int dwba_lower_bound(const double* __restrict__ r, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (r[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// First index c in [0, n] with key[c] >= v for a non-decreasing int array.
__device__ __forceinline__ int dwba_lower_bound_i(const int32_t* __restrict__ key, int n, int v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (key[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}
