// Phase-interval helpers shared by the node-set kernels (nodes.cu, cupy_nodes.cu): the breakpoints
// of generate_phase_nodes (oscillatory_integrals.py:1625-1713) -- numpy.linspace arithmetic when no
// breakpoint list is given -- and the search for the interval containing a radius.
#pragma once
#include "common.cuh"

namespace dwba_nodes {

constexpr int MAX_CC = 15;

struct SetView {
  const double* r;
  const double* lr;
  const double* br;  // breakpoints or nullptr (linspace)
  int n_grid, n1, n_int, log1, log2;
  double start, stop, step;
};

__device__ __forceinline__ void interval(const SetView& s, int m, double& a, double& b) {
  if (s.br != nullptr) {
    a = s.br[m];
    b = s.br[m + 1];
  } else {  // numpy.linspace: y[i] = i*step + start, y[num-1] = stop
    a = rn_add(rn_mul((double)m, s.step), s.start);
    b = (m + 1 == s.n_int) ? s.stop : rn_add(rn_mul((double)(m + 1), s.step), s.start);
  }
}

// last interval m whose left end a_m <= x (0 if none)
__device__ __forceinline__ int interval_floor(const SetView& s, double x) {
  if (s.br != nullptr) {
    int lo = 0, hi = s.n_int;  // a_lo <= x < a_hi
    if (!(s.br[0] <= x)) return 0;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s.br[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
  }
  double q = floor((x - s.start) / s.step);
  int m = q < 0.0 ? 0 : (q > (double)(s.n_int - 1) ? s.n_int - 1 : (int)q);
  // the closed form can be one off after rounding: correct against the exact interval ends
  double a, b;
  interval(s, m, a, b);
  while (m > 0 && a > x) { --m; interval(s, m, a, b); }
  while (m + 1 < s.n_int) {
    double a2, b2;
    interval(s, m + 1, a2, b2);
    if (a2 <= x) { ++m; } else break;
  }
  return m;
}

// log(1 + u) for 0 <= u <= 1/64 by its Taylor series: 6 terms for u <= 2^-9, else 12 (the
// truncation stays below 1e-17 relative either way)
__device__ __forceinline__ double log1p_small(double u) {
  if (u <= 0.001953125) {
    double q = -1.0 / 6.0;
    q = fma(q, u, 1.0 / 5.0);
    q = fma(q, u, -1.0 / 4.0);
    q = fma(q, u, 1.0 / 3.0);
    q = fma(q, u, -0.5);
    q = fma(q, u, 1.0);
    return q * u;
  }
  double p = -1.0 / 12.0;
  p = fma(p, u, 1.0 / 11.0);
  p = fma(p, u, -1.0 / 10.0);
  p = fma(p, u, 1.0 / 9.0);
  p = fma(p, u, -1.0 / 8.0);
  p = fma(p, u, 1.0 / 7.0);
  p = fma(p, u, -1.0 / 6.0);
  p = fma(p, u, 1.0 / 5.0);
  p = fma(p, u, -1.0 / 4.0);
  p = fma(p, u, 1.0 / 3.0);
  p = fma(p, u, -0.5);
  p = fma(p, u, 1.0);
  return p * u;
}

}  // namespace dwba_nodes
