// Node-set operators: the phase-split Clenshaw-Curtis quadrature of the
// reference folded into banded matrices on the radial grid.
//
// Reference semantics (oscillatory_integrals.py):
//   * breakpoints: generate_phase_nodes (:1625-1713) -- linspace for eta == 0
//     (rebuilt here on the device with numpy's linspace arithmetic), host list otherwise;
//   * CC nodes of interval [a, b]: x = hw*(x_ref+1) + a, W = w_ref*hw, hw = 0.5*(b-a),
//     intervals with b - a <= 1e-12 skipped (:2578-2601, :2701-2712);
//   * outer interpolation P1: _interp_on_radial_grid on r[:n1] (:279-302);
//   * exchange: rho2 interpolated by P2 on the full grid, kernel columns by
//     linear-in-r weights Q with idx_right = clip(searchsorted(r, x), 1, N-1) (:2714-2742).
// With these, the reference's outer sum sum_c W_c (P1 rho1)_c (P1 v)_c equals
// rho1^T T v, T = P1^T diag(W) P1 (tridiagonal), and the exchange inner sum
// sum_c K(r_i, x_c) W_c (P2 rho2)_c equals sum_k K_ik (B rho2)_k with
// B = Q^T diag(W) P2 (band of half-width 2).
//
// One thread per grid row k gathers the nodes that touch row k: a node with
// interpolation interval j feeds rows j and j+1, so row k needs exactly the
// nodes in [r_{k-1}, r_{k+1}]. The thread enumerates the phase intervals that
// overlap that window, recomputes their nodes with the reference's arithmetic,
// and sums the contributions in ascending node order (deterministic, no scratch
// memory, no atomics).
#include "common.cuh"

namespace {

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

// One warp per CTA: 32 consecutive rows do similar work (their windows hold similar node counts),
// and the small CTAs keep the SMs evenly loaded although the work per row grows with r.
constexpr int ROWS_CTA = 32;
__global__ void __launch_bounds__(ROWS_CTA, 24) nodeset_rows_kernel(const dwba_nodeset_t* __restrict__ sets, const double* __restrict__ ccx_g,
                                    const double* __restrict__ ccw_g, int n_cc, int* status) {
  __shared__ double ccx[MAX_CC], ccw[MAX_CC], ccx1[MAX_CC];
  if (threadIdx.x < n_cc) {
    ccx[threadIdx.x] = ccx_g[threadIdx.x];
    ccw[threadIdx.x] = ccw_g[threadIdx.x];
    ccx1[threadIdx.x] = rn_add(ccx_g[threadIdx.x], 1.0);
  }
  __syncthreads();
  const dwba_nodeset_t d = sets[blockIdx.y];
  SetView s;
  s.r = d.r_dev;
  s.lr = d.logr_dev;
  s.br = d.breaks_dev;
  s.n_grid = d.n_grid;
  s.n1 = d.n1;
  s.n_int = d.n_breaks - 1;
  s.log1 = d.log1;
  s.log2 = d.log2;
  s.start = s.r[0];
  s.stop = s.r[s.n1 - 1];
  s.step = rn_sub(s.stop, s.start) / (double)s.n_int;
  const int N = s.n_grid, n1 = s.n1;
  const double* __restrict__ r = s.r;

  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    const double wlo = k >= 1 ? r[k - 1] : -1.0e308;
    const double whi = k + 1 <= N - 1 ? r[k + 1] : 1.0e308;
    double t_lo = 0.0, t_di = 0.0, t_up = 0.0;
    double band0 = 0.0, band1 = 0.0, band2 = 0.0, band3 = 0.0, band4 = 0.0;
    bool bad = false;
    // the interpolation intervals a node of this row can use are j in {k-1, k, k+1}: their
    // reciprocal widths (log r or r) and the reciprocal kernel-column spacings, once per row
    auto recip = [&](int j, bool lg) -> double {
      if (j < 0 || j + 1 > N - 1) return 0.0;
      return lg ? 1.0 / (s.lr[j + 1] - s.lr[j]) : 1.0 / (r[j + 1] - r[j]);
    };
    const double iT0 = recip(k - 1, s.log1), iT1 = recip(k, s.log1);
    const double iB0 = recip(k - 1, s.log2), iB1 = recip(k, s.log2), iB2 = recip(k + 1, s.log2);
    const double iW0 = k >= 1 ? 1.0 / (r[k] - r[k - 1] + 1e-30) : 0.0;          // il = k-1
    const double iW1 = k + 1 <= N - 1 ? 1.0 / (r[k + 1] - r[k] + 1e-30) : 0.0;  // il = k
    // grid values the nodes of this row can touch, held in registers
    const double rk = r[k], rkm = k >= 1 ? r[k - 1] : 0.0, rkp = k + 1 <= N - 1 ? r[k + 1] : 0.0;
    const double lk = s.lr[k], lkm = k >= 1 ? s.lr[k - 1] : 0.0, lkp = k + 1 <= N - 1 ? s.lr[k + 1] : 0.0;
    const double r_first = r[0], r_lim = r[n1 - 1], r_last = r[N - 1];
    // nodes never leave [r0, r[n1-1]]; rows past n1+1 have none
    if (k <= n1 + 1) {
      // one interval earlier too: its top node can coincide with the window's lower end
      const int m0 = max(0, interval_floor(s, wlo) - 1);
      for (int m = m0; m < s.n_int; ++m) {
        double a, b;
        interval(s, m, a, b);
        if (a > whi) break;
        const double width = rn_sub(b, a);
        if (!(width > 1e-12)) continue;
        const double hw = rn_mul(0.5, width);
        for (int sl = n_cc - 1; sl >= 0; --sl) {  // ascending positions within the interval
          double x = rn_add(rn_mul(hw, ccx1[sl]), a);
          x = fmin(fmax(x, a), b);  // the top node can round one ulp past b
          if (x < wlo || x > whi) continue;
          // kernel columns: searchsorted(r, x, 'left') within the window, clipped to [1, N-1]
          int ir;
          if (k >= 1 && x <= rkm) ir = k - 1;
          else if (x <= rk) ir = k;
          else ir = k + 1;
          ir = ir < 1 ? 1 : (ir > N - 1 ? N - 1 : ir);
          const int il = ir - 1;
          const bool b_row = il == k || il == k - 1;
          if (k >= n1 && !b_row) continue;  // reaches neither a T nor a B entry of this row
          const double w = rn_mul(ccw[sl], hw);
          // interpolation interval on r[:n] (np.interp after clipping; x is inside [r_{k-1}, r_{k+1}])
          const double lx = (s.log1 || s.log2) ? log(x) : 0.0;
          int jf;  // floor index in the full grid
          if (k + 1 <= N - 1 && x >= rkp) jf = k + 1;
          else if (x >= rk) jf = k;
          else jf = k - 1;
          // --- T rows: nodes with j1 in {k-1, k}
          if (k < n1) {
            int j1;
            double t1;
            if (x <= r_first) { j1 = 0; t1 = 0.0; }
            else if (x >= r_lim) { j1 = n1 - 2; t1 = 1.0; }
            else {
              j1 = jf > n1 - 2 ? n1 - 2 : jf;
              if (j1 == k || j1 == k - 1) {
                const double inv = j1 == k ? iT1 : iT0;
                t1 = s.log1 ? (lx - (j1 == k ? lk : lkm)) * inv : (x - (j1 == k ? rk : rkm)) * inv;
              } else {
                t1 = 0.0;  // reaches no T entry of this row
              }
            }
            if (j1 == k) {
              t_di += w * (1.0 - t1) * (1.0 - t1);
              t_up += w * (1.0 - t1) * t1;
            } else if (j1 == k - 1) {
              t_di += w * t1 * t1;
              t_lo += w * t1 * (1.0 - t1);
            }
          }
          // --- B rows: nodes with il in {k-1, k}
          if (!b_row) continue;
          int j2;
          double t2;
          if (x <= r_first) { j2 = 0; t2 = 0.0; }
          else if (x >= r_last) { j2 = N - 2; t2 = 1.0; }
          else {
            j2 = jf > N - 2 ? N - 2 : jf;
            const int dj = j2 - k;  // -1, 0 or 1 inside the window
            const double inv = dj < 0 ? iB0 : (dj == 0 ? iB1 : iB2);
            t2 = s.log2 ? (lx - (dj < 0 ? lkm : (dj == 0 ? lk : lkp))) * inv
                        : (x - (dj < 0 ? rkm : (dj == 0 ? rk : rkp))) * inv;
          }
          const double wr = (x - (il == k ? rk : rkm)) * (il == k ? iW1 : iW0);
          const double q = il == k ? 1.0 - wr : wr;
          const int d0 = j2 - k;
          if (d0 < -2 || d0 + 1 > 2) { bad = true; continue; }
          const double v0 = q * w * (1.0 - t2), v1 = q * w * t2;
          // taps d0, d0+1 of the row's band (registers: no dynamic indexing)
          if (d0 == -2) { band0 += v0; band1 += v1; }
          else if (d0 == -1) { band1 += v0; band2 += v1; }
          else if (d0 == 0) { band2 += v0; band3 += v1; }
          else { band3 += v0; band4 += v1; }
        }
      }
    }
    if (k < n1) {
      d.ta_dev[3 * k + 0] = t_lo;
      d.ta_dev[3 * k + 1] = t_di;
      d.ta_dev[3 * k + 2] = t_up;
    }
    double* bx = d.bx_dev + 5 * (int64_t)k;
    bx[0] = band0;
    bx[1] = band1;
    bx[2] = band2;
    bx[3] = band3;
    bx[4] = band4;
    if (bad) atomicExch(status, 1);
  }
}

}  // namespace

extern "C" int dwba_build_nodesets(const dwba_nodeset_t* sets_dev, int n_sets, int max_grid, const double* cc_x_dev,
                                   const double* cc_w_dev, int n_cc, int* status_dev, dwba_stream_t stream) {
  if (n_sets <= 0) return DWBA_OK;
  if (!sets_dev || !cc_x_dev || !cc_w_dev || !status_dev || n_cc < 2 || n_cc > MAX_CC || max_grid < 2 ||
      n_sets > 65535)
    return DWBA_ERR_INVALID_ARG;
  dim3 grid(dwba_grid_1d(max_grid, ROWS_CTA), n_sets);
  nodeset_rows_kernel<<<grid, ROWS_CTA, 0, (cudaStream_t)stream>>>(sets_dev, cc_x_dev, cc_w_dev, n_cc, status_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
