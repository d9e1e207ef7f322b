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
// Every CC node lies in one grid interval (r_g, r_{g+1}] and feeds only rows g,
// g+1 and g+2, so one thread per grid interval evaluates the nodes it owns once
// (enumerating the phase intervals that overlap its grid interval and recomputing
// their nodes with the reference's arithmetic), sums their contributions per
// target row in ascending node order, and each row adds the sums of its three
// owners through warp shuffles (deterministic, no scratch memory, no atomics).
#include "phase_nodes.cuh"

namespace {

using namespace dwba_nodes;

// reciprocal width of interpolation interval j (log r or r), zero past the grid
__device__ __forceinline__ double recip_width(const SetView& s, int j, bool lg) {
  if (j < 0 || j + 1 > s.n_grid - 1) return 0.0;
  return lg ? 1.0 / (s.lr[j + 1] - s.lr[j]) : 1.0 / (s.r[j + 1] - s.r[j]);
}

// log(1 + u) for 0 <= u <= 1/64 by its Taylor series in Estrin form (shorter dependency chains
// than Horner): 6 terms for u <= 2^-9, 12 terms up to 1/64 (truncation below 1e-17 relative).
__device__ __forceinline__ double log1p_series6(double u) {
  const double u2 = u * u;
  const double e0 = fma(-0.5, u, 1.0), e1 = fma(-0.25, u, 1.0 / 3.0), e2 = fma(-1.0 / 6.0, u, 0.2);
  return u * fma(fma(e2, u2, e1), u2, e0);
}
__device__ __forceinline__ double log1p_series12(double u) {
  const double u2 = u * u, u4 = u2 * u2;
  const double e0 = fma(-0.5, u, 1.0), e1 = fma(-0.25, u, 1.0 / 3.0), e2 = fma(-1.0 / 6.0, u, 0.2);
  const double e3 = fma(-0.125, u, 1.0 / 7.0), e4 = fma(-0.1, u, 1.0 / 9.0), e5 = fma(-1.0 / 12.0, u, 1.0 / 11.0);
  const double lo = fma(fma(e2, u2, e1), u2, e0);
  const double hi = fma(fma(e5, u2, e4), u2, e3);
  return u * fma(hi, u4 * u2, lo);
}

// One warp per CTA covers OWN_ROWS consecutive grid rows. Lane j owns grid interval
// g = k0 - 2 + j: the CC nodes whose kernel-column interval (searchsorted left, clipped) is
// il = g, i.e. x in (r_g, r_{g+1}] (g = 0: [r_0, r_1]). Each node is evaluated once, by its
// owner, and reaches rows g, g+1 (T and B) and g+2 (T, a node exactly at r_{g+1}); the owner
// sums them per target row in ascending node order, and row k adds the sums of lanes k-2,
// k-1 and k in that order through warp shuffles. Lanes 0 and 1 are the halo of the first two
// rows (their own rows are written by the previous CTA).
//
// Per node, a node strictly inside its interval (and inside r[:n1], with a log step below 1/64)
// takes the fast path: both interpolations use interval g, so with t the (log-)interpolation
// weight, wr the linear column weight and w the CC weight,
//   T: row g += w(1-t)^2 (diagonal), w(1-t)t (upper); row g+1 += wt^2 (diagonal), wt(1-t) (lower)
//   B: row g += (1-wr) w(1-t2), (1-wr) w t2 (taps 0, 1); row g+1 += wr w(1-t2), wr w t2 (taps -1, 0)
// from the shared products w(1-t) and wt. Nodes on a grid point or outside those bounds take the
// general path, which handles every case the reference's clipping and searchsorted produce.
constexpr int OWN_ROWS = 30;
#ifndef DWBA_NODESET_FILL
#define DWBA_NODESET_FILL 32 // resident-CTA waves the launch aims for
#endif
// resident CTAs per SM the register budget is set for: 24 (80 registers) for the stored-operator
// kernel; 32 (64 registers, a few spills) for the one applied at once to the folds, where the
// extra warps hide more of the fold loads' latency than the spills cost (2.49 ms against 2.60 ms
// on the 2048-set batch, bit-identical; 2 or 4 warps per CTA at 48-56 registers spill too much)
#ifndef DWBA_NODESET_MIN_BLOCKS
#define DWBA_NODESET_MIN_BLOCKS 24
#endif
#ifndef DWBA_NODESET_FOLD_MIN_BLOCKS
#define DWBA_NODESET_FOLD_MIN_BLOCKS 32
#endif
#ifndef DWBA_NODESET_FC
#define DWBA_NODESET_FC 1  // factors per chunk of the fold loads (1: 2.39 ms, 2: 2.47 ms, 4: 2.49 ms, 8 spills: 3.32 ms)
#endif
#ifndef DWBA_NODESET_WARPS
#define DWBA_NODESET_WARPS 1  // warps per CTA, each on its own row blocks of the CTA's set
#endif
constexpr int NS_WARPS = DWBA_NODESET_WARPS;
// FOLD = true: the operators are not stored; each row applies them at once to the two multi-folds
// of its set (folds[2 set] with the tridiagonal T, folds[2 set + 1] with the band B), with the
// arithmetic of fold_multi_kernel, and writes the folded operands instead.
template <int H>
__device__ __forceinline__ void fold_row_from_taps(const dwba_fold_multi_t& m, int i, const double* tap) {
  if (i >= m.n_clear) return;
  const int n_f = m.n_f, n_src = m.n_src;
  if (i >= m.n_out) {
    for (int t = 0; t < n_f; ++t) m.out_dev[t][i] = 0.0;
    return;
  }
  const double* __restrict__ g = m.g_dev;
  double tp[2 * H + 1], gv[2 * H + 1];
  bool in[2 * H + 1];
#pragma unroll
  for (int d = -H; d <= H; ++d) {
    const int k = i + d;
    in[d + H] = k >= 0 && k < n_src;
    tp[d + H] = in[d + H] ? tap[d + H] : 0.0;
    gv[d + H] = in[d + H] ? g[k] : 0.0;
  }
  // factors in chunks of FC: every tap load of a chunk is issued before its products, so the loads
  // are in flight together instead of one factor's after the previous factor's store (the stores
  // could alias the next factor's array for all the compiler knows)
  constexpr int FC = DWBA_NODESET_FC;
  for (int t0 = 0; t0 < n_f; t0 += FC) {
    double fv[FC][2 * H + 1];
#pragma unroll
    for (int c = 0; c < FC; ++c) {
      const bool live = t0 + c < n_f;
      const double* __restrict__ f = live ? m.f_dev[t0 + c] : g;
#pragma unroll
      for (int d = -H; d <= H; ++d) fv[c][d + H] = (live && in[d + H]) ? f[i + d] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < FC; ++c) {
      if (t0 + c < n_f) {
        double acc = 0.0;
#pragma unroll
        for (int d = -H; d <= H; ++d)
          if (in[d + H]) acc += tp[d + H] * (fv[c][d + H] * gv[d + H]);
        __stcs(m.out_dev[t0 + c] + i, acc);  // streaming store: the folded operands are read by the next kernels from DRAM
      }
    }
  }
}

template <int NCC, bool FOLD>  // NCC: CC nodes per interval known at compile time (0: n_cc at run time)
__global__ void __launch_bounds__(32 * NS_WARPS, FOLD ? DWBA_NODESET_FOLD_MIN_BLOCKS : DWBA_NODESET_MIN_BLOCKS)
    nodeset_rows_kernel(const dwba_nodeset_t* __restrict__ sets,
                                                              const double* __restrict__ ccx_g,
                                                              const double* __restrict__ ccw_g, int n_cc_rt,
                                                              int* status,
                                                              const dwba_fold_multi_t* __restrict__ folds) {
  __shared__ double ccw[MAX_CC], ccx1[MAX_CC];
  // the set's two multi-fold descriptors (T, then B), read by every row of the CTA
  __shared__ dwba_fold_multi_t fm[FOLD ? 2 : 1];
  const int n_cc = NCC > 0 ? NCC : n_cc_rt;
  if (threadIdx.x < n_cc) {
    ccw[threadIdx.x] = ccw_g[threadIdx.x];
    ccx1[threadIdx.x] = rn_add(ccx_g[threadIdx.x], 1.0);
  }
  if (FOLD) {
    constexpr int W = (int)(2 * sizeof(dwba_fold_multi_t) / sizeof(unsigned long long));
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(folds + 2 * (int64_t)blockIdx.y);
    for (int w = threadIdx.x; w < W; w += blockDim.x) reinterpret_cast<unsigned long long*>(fm)[w] = src[w];
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
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double r_first = r[0], r_lim = r[n1 - 1], r_last = r[N - 1];
  // with n1 == N and one spacing test for both, the B taps of a node are its T taps
  const bool shared = s.log1 == s.log2 && n1 == N;
  const bool any_log = s.log1 || s.log2;

  for (int k0 = (blockIdx.x * NS_WARPS + warp) * OWN_ROWS; k0 < N; k0 += gridDim.x * NS_WARPS * OWN_ROWS) {
    const int g = k0 - 2 + lane;
    // sums for row g (o_*), row g+1 (x_*) and row g+2 (n_*)
    double o_di = 0.0, o_up = 0.0, o_b2 = 0.0, o_b3 = 0.0, o_b4 = 0.0;
    double x_lo = 0.0, x_di = 0.0, x_up = 0.0, x_b1 = 0.0, x_b2 = 0.0, x_b3 = 0.0;
    double n_lo = 0.0, n_di = 0.0;
    bool bad = false;
    // nodes lie in [r_0, r_{n1-1}], so owners stop at g = n1 - 2
    if (g >= 0 && g <= n1 - 2) {
      const double rg = r[g], rg1 = r[g + 1];
      const double lo = g == 0 ? -1.0e308 : rg;  // exclusive lower end of the owned interval
      bool first = true, done = false, short6 = true;
      double iT0 = 0.0, iT1 = 0.0, iB0 = 0.0, iB1 = 0.0, iW = 0.0, lg = 0.0, lg1 = 0.0, irg = 0.0;
      for (int m = interval_floor(s, rg); m < s.n_int && !done; ++m) {
        double a, b;
        interval(s, m, a, b);
        if (a > rg1) break;
        const double width = rn_sub(b, a);
        if (!(width > 1e-12)) continue;
        const double hw = rn_mul(0.5, width);
        // an interval strictly inside the owned grid interval (and not at r_0), on a grid whose
        // step here keeps every node on the fast path: its nodes need none of the per-node range
        // tests. Same nodes, order and arithmetic as the loop below.
        if (NCC > 0 && a > lo && b < rg1 && (g >= 1 || a > r_first)) {
          if (first) {
            iT0 = recip_width(s, g, s.log1);
            iT1 = recip_width(s, g + 1, s.log1);
            iB0 = recip_width(s, g, s.log2);
            iB1 = recip_width(s, g + 1, s.log2);
            iW = 1.0 / (rg1 - rg + 1e-30);
            lg = s.lr[g];
            lg1 = s.lr[g + 1];
            irg = 1.0 / rg;
            short6 = (rg1 - rg) * irg <= 0.001953125;
            first = false;
          }
          if (!any_log || (rg1 - rg) * irg <= 0.015625) {
            // rolled, like the general loop: unrolled it spills (measured 1.94 ms unrolled, 1.80 ms
            // rolled, 1.88 ms without this block on the 2048-set batch)
#pragma unroll 1
            for (int q = 0; q < (NCC > 0 ? NCC : 1); ++q) {
              const int sl = n_cc - 1 - q;
              double x = rn_add(rn_mul(hw, ccx1[sl]), a);
              x = fmin(fmax(x, a), b);
              const double w = rn_mul(ccw[sl], hw);
              const double dx = x - rg;
              const double u = dx * irg;
              double dl = 0.0;
              if (any_log) dl = short6 ? log1p_series6(u) : log1p_series12(u);
              const double t = s.log1 ? dl * iT0 : dx * iT0;
              const double omt = 1.0 - t;
              double wo = w * omt, wt = w * t;
              o_di = fma(wo, omt, o_di);
              o_up = fma(wo, t, o_up);
              x_di = fma(wt, t, x_di);
              x_lo = fma(wt, omt, x_lo);
              if (!shared) {
                const double t2 = s.log2 ? dl * iB0 : dx * iB0;
                wo = w * (1.0 - t2);
                wt = w * t2;
              }
              const double q1 = dx * iW, q0 = 1.0 - q1;
              o_b2 = fma(q0, wo, o_b2);
              o_b3 = fma(q0, wt, o_b3);
              x_b1 = fma(q1, wo, x_b1);
              x_b2 = fma(q1, wt, x_b2);
            }
            continue;
          }
        }
        // kept rolled: unrolling the node loop spills at this register budget (measured 2.46 ms
        // unrolled against 1.89 ms rolled on the 2048-set batch)
#pragma unroll 1
        for (int q = 0; q < (NCC > 0 ? NCC : MAX_CC); ++q) {  // ascending positions within the interval
          if (NCC == 0 && q >= n_cc) break;
          const int sl = n_cc - 1 - q;
          double x = rn_add(rn_mul(hw, ccx1[sl]), a);
          x = fmin(fmax(x, a), b);  // the top node can round one ulp past b
          if (!(x > lo)) continue;
          if (x > rg1) {
            done = true;
            break;
          }
          if (first) {  // reciprocal widths of the intervals j in {g, g+1} a node of this owner uses
            iT0 = recip_width(s, g, s.log1);
            iT1 = recip_width(s, g + 1, s.log1);
            iB0 = recip_width(s, g, s.log2);
            iB1 = recip_width(s, g + 1, s.log2);
            iW = 1.0 / (rg1 - rg + 1e-30);
            lg = s.lr[g];
            lg1 = s.lr[g + 1];
            irg = 1.0 / rg;
            short6 = (rg1 - rg) * irg <= 0.001953125;
            first = false;
          }
          const double w = rn_mul(ccw[sl], hw);
          const double dx = x - rg;
          const double u = dx * irg;
          if (x < rg1 && x > r_first && x < r_lim && (shared || x < r_last) && (!any_log || u <= 0.015625)) {
            // fast path: j1 = j2 = g
            double dl = 0.0;
            if (any_log) dl = short6 ? log1p_series6(u) : log1p_series12(u);
            const double t = s.log1 ? dl * iT0 : dx * iT0;
            const double omt = 1.0 - t;
            double wo = w * omt, wt = w * t;
            o_di = fma(wo, omt, o_di);
            o_up = fma(wo, t, o_up);
            x_di = fma(wt, t, x_di);
            x_lo = fma(wt, omt, x_lo);
            if (!shared) {
              const double t2 = s.log2 ? dl * iB0 : dx * iB0;
              wo = w * (1.0 - t2);
              wt = w * t2;
            }
            const double q1 = dx * iW, q0 = 1.0 - q1;
            o_b2 = fma(q0, wo, o_b2);
            o_b3 = fma(q0, wt, o_b3);
            x_b1 = fma(q1, wo, x_b1);
            x_b2 = fma(q1, wt, x_b2);
            continue;
          }
          // general path
          const bool at_top = x >= rg1;  // floor index in the full grid: g + 1 at r_{g+1}, else g
          // log x - log r_g: from the series of log(1 + (x - r_g)/r_g) when the grid step is small
          // (it then equals the difference of the two logs to a few ulps of that difference), else
          // as the difference; log x - log r_{g+1} only for a node exactly at r_{g+1}
          double dl = 0.0, dl_up = 0.0;
          if (any_log) {
            dl = u <= 0.015625 ? log1p_small(u) : log(x) - lg;
            if (at_top) dl_up = log(x) - lg1;
          }
          // --- T: rows j1 and j1 + 1, j1 in {g, g+1}
          int j1;
          double t1;
          {
            if (x <= r_first) { j1 = 0; t1 = 0.0; }
            else if (x >= r_lim) { j1 = n1 - 2; t1 = 1.0; }
            else {
              j1 = (at_top && g + 1 <= n1 - 2) ? g + 1 : g;
              const bool up = j1 != g;
              const double inv = up ? iT1 : iT0;
              t1 = s.log1 ? (up ? dl_up : dl) * inv : (x - (up ? rg1 : rg)) * inv;
            }
            const double v_di0 = w * (1.0 - t1) * (1.0 - t1), v_up0 = w * (1.0 - t1) * t1;
            const double v_di1 = w * t1 * t1, v_lo1 = w * t1 * (1.0 - t1);
            if (j1 == g) {
              o_di += v_di0; o_up += v_up0;
              x_di += v_di1; x_lo += v_lo1;
            } else if (j1 == g + 1) {
              x_di += v_di0; x_up += v_up0;
              n_di += v_di1; n_lo += v_lo1;
            } else {
              bad = true;
            }
          }
          // --- B: rows il = g (weight 1 - wr) and g + 1 (weight wr), taps d0, d0 + 1
          {
            int j2;
            double t2;
            if (shared) { j2 = j1; t2 = t1; }
            else if (x <= r_first) { j2 = 0; t2 = 0.0; }
            else if (x >= r_last) { j2 = N - 2; t2 = 1.0; }
            else {
              j2 = (at_top && g + 1 <= N - 2) ? g + 1 : g;
              const bool up = j2 != g;
              const double inv = up ? iB1 : iB0;
              t2 = s.log2 ? (up ? dl_up : dl) * inv : (x - (up ? rg1 : rg)) * inv;
            }
            const double wr = dx * iW;
            const double q0 = 1.0 - wr, q1 = wr;
            if (j2 == g) {  // row g: taps 0, 1 (band 2, 3); row g+1: taps -1, 0 (band 1, 2)
              o_b2 += q0 * w * (1.0 - t2); o_b3 += q0 * w * t2;
              x_b1 += q1 * w * (1.0 - t2); x_b2 += q1 * w * t2;
            } else if (j2 == g + 1) {  // row g: taps 1, 2 (band 3, 4); row g+1: taps 0, 1 (band 2, 3)
              o_b3 += q0 * w * (1.0 - t2); o_b4 += q0 * w * t2;
              x_b2 += q1 * w * (1.0 - t2); x_b3 += q1 * w * t2;
            } else {
              bad = true;
            }
          }
        }
      }
    }
    // row g = sums of lane - 2 (its row g+2), lane - 1 (its row g+1) and this lane, in that order
    const double p_lo = __shfl_up_sync(0xffffffffu, n_lo, 2), p_di = __shfl_up_sync(0xffffffffu, n_di, 2);
    const double q_lo = __shfl_up_sync(0xffffffffu, x_lo, 1), q_di = __shfl_up_sync(0xffffffffu, x_di, 1);
    const double q_up = __shfl_up_sync(0xffffffffu, x_up, 1);
    const double q_b1 = __shfl_up_sync(0xffffffffu, x_b1, 1), q_b2 = __shfl_up_sync(0xffffffffu, x_b2, 1);
    const double q_b3 = __shfl_up_sync(0xffffffffu, x_b3, 1);
    if (lane >= 2 && g < N) {
      const double t0 = p_lo + q_lo;  // from nodes below r_g only
      const double t1 = (p_di + q_di) + o_di;
      const double t2 = q_up + o_up;
      const double b1 = q_b1, b2 = q_b2 + o_b2, b3 = q_b3 + o_b3, b4 = o_b4;
      if (FOLD) {
        if (g < n1) {
          const double tt[3] = {t0, t1, t2};
          fold_row_from_taps<1>(fm[0], g, tt);
        }
        const double bb[5] = {0.0, b1, b2, b3, b4};
        fold_row_from_taps<2>(fm[FOLD ? 1 : 0], g, bb);
      } else {
        if (g < n1) {
          d.ta_dev[3 * g + 0] = t0;
          d.ta_dev[3 * g + 1] = t1;
          d.ta_dev[3 * g + 2] = t2;
        }
        double* bx = d.bx_dev + 5 * (int64_t)g;
        bx[0] = 0.0;
        bx[1] = b1;
        bx[2] = b2;
        bx[3] = b3;
        bx[4] = b4;
      }
    }
    if (bad) atomicExch(status, 1);
  }
}

// row groups per set: enough warps in total to fill the GPU several times over, never more than
// the largest set needs (each warp strides over its set's row blocks)
dim3 nodeset_grid(int max_grid, int n_sets) {
  const int need = (max_grid + OWN_ROWS * NS_WARPS - 1) / (OWN_ROWS * NS_WARPS);
  const int fill = (int)(((int64_t)148 * 24 * DWBA_NODESET_FILL + (int64_t)n_sets * NS_WARPS - 1) /
                         ((int64_t)n_sets * NS_WARPS));
  return dim3(need < fill ? need : fill, n_sets);
}

}  // namespace

extern "C" int dwba_build_nodesets(const dwba_nodeset_t* sets_dev, int n_sets, int max_grid, const double* cc_x_dev,
                                   const double* cc_w_dev, int n_cc, int* status_dev, dwba_stream_t stream) {
  if (n_sets <= 0) return DWBA_OK;
  if (!sets_dev || !cc_x_dev || !cc_w_dev || !status_dev || n_cc < 2 || n_cc > MAX_CC || max_grid < 2 ||
      n_sets > 65535)
    return DWBA_ERR_INVALID_ARG;
  const dim3 grid = nodeset_grid(max_grid, n_sets);
  if (n_cc == 5)
    nodeset_rows_kernel<5, false><<<grid, 32 * NS_WARPS, 0, (cudaStream_t)stream>>>(sets_dev, cc_x_dev, cc_w_dev, n_cc,
                                                                         status_dev, nullptr);
  else
    nodeset_rows_kernel<0, false><<<grid, 32 * NS_WARPS, 0, (cudaStream_t)stream>>>(sets_dev, cc_x_dev, cc_w_dev, n_cc,
                                                                         status_dev, nullptr);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

extern "C" int dwba_build_nodesets_folded(const dwba_nodeset_t* sets_dev, const dwba_fold_multi_t* folds_dev,
                                          int n_sets, int max_grid, const double* cc_x_dev, const double* cc_w_dev,
                                          int n_cc, int* status_dev, dwba_stream_t stream) {
  if (n_sets <= 0) return DWBA_OK;
  if (!sets_dev || !folds_dev || !cc_x_dev || !cc_w_dev || !status_dev || n_cc < 2 || n_cc > MAX_CC ||
      max_grid < 2 || n_sets > 65535)
    return DWBA_ERR_INVALID_ARG;
  const dim3 grid = nodeset_grid(max_grid, n_sets);
  if (n_cc == 5)
    nodeset_rows_kernel<5, true><<<grid, 32 * NS_WARPS, 0, (cudaStream_t)stream>>>(sets_dev, cc_x_dev, cc_w_dev, n_cc,
                                                                        status_dev, folds_dev);
  else
    nodeset_rows_kernel<0, true><<<grid, 32 * NS_WARPS, 0, (cudaStream_t)stream>>>(sets_dev, cc_x_dev, cc_w_dev, n_cc,
                                                                        status_dev, folds_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
