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
//     linear-in-r weights Q (:2714-2742).
// With these, the reference's outer sum sum_c W_c (P1 rho1)_c (P1 v)_c equals
// rho1^T T v, T = P1^T diag(W) P1 (tridiagonal), and the exchange inner sum
// sum_c K(r_i, x_c) W_c (P2 rho2)_c equals sum_k K_ik (B rho2)_k with
// B = Q^T diag(W) P2 (band of half-width 2).
#include "common.cuh"

namespace {

struct NodeGeom {
  double x, w;
};

// Position and weight of node c (ascending order) of one node set.
__device__ __forceinline__ NodeGeom node_geom(const dwba_nodeset_t& s, const double* __restrict__ ccx,
                                              const double* __restrict__ ccw, int n_cc, int c) {
  const int m = c / n_cc;
  const int slot = n_cc - 1 - (c - m * n_cc);  // reference order runs x_ref from +1 down to -1
  double a, b;
  if (s.breaks_dev != nullptr) {
    a = s.breaks_dev[m];
    b = s.breaks_dev[m + 1];
  } else {
    // numpy.linspace(start, stop, num): y[i] = i*step + start, y[num-1] = stop
    const double start = s.r_dev[0];
    const double stop = s.r_dev[s.n1 - 1];
    const int div = s.n_breaks - 1;
    const double step = rn_sub(stop, start) / (double)div;
    a = rn_add(rn_mul((double)m, step), start);
    b = (m + 1 == div) ? stop : rn_add(rn_mul((double)(m + 1), step), start);
  }
  NodeGeom g;
  const double hw = rn_mul(0.5, rn_sub(b, a));
  g.x = rn_add(rn_mul(hw, rn_add(ccx[slot], 1.0)), a);
  // Keep the node inside [a, b]: the top node hw*2 + a can round one ulp past b,
  // and a sorted node list is what the row gathers below rely on.
  g.x = fmin(fmax(g.x, a), b);
  g.w = rn_sub(b, a) > 1e-12 ? rn_mul(ccw[slot], hw) : 0.0;
  return g;
}

// Interpolation interval and weight on r[:n] for np.interp semantics after
// clipping into [r0, r[n-1]] (log-r when log_grid): value = (1-t) y[j] + t y[j+1].
__device__ __forceinline__ void interp_op(const double* __restrict__ r, const double* __restrict__ lr, int n,
                                          int log_grid, double x, int& j, double& t) {
  if (x <= r[0]) { j = 0; t = 0.0; return; }
  if (x >= r[n - 1]) { j = n - 2; t = 1.0; return; }
  j = dwba_floor_index(r, n, x);
  if (j > n - 2) j = n - 2;
  if (log_grid) {
    t = (log(x) - lr[j]) / (lr[j + 1] - lr[j]);
  } else {
    t = (x - r[j]) / (r[j + 1] - r[j]);
  }
}

__global__ void nodes_kernel(const dwba_nodeset_t* __restrict__ sets, const double* __restrict__ ccx,
                             const double* __restrict__ ccw, int n_cc) {
  const dwba_nodeset_t s = sets[blockIdx.y];
  const int n_nodes = (s.n_breaks - 1) * n_cc;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_nodes; c += gridDim.x * blockDim.x) {
    const NodeGeom g = node_geom(s, ccx, ccw, n_cc, c);
    int j1, j2;
    double t1, t2;
    interp_op(s.r_dev, s.logr_dev, s.n1, s.log1, g.x, j1, t1);
    interp_op(s.r_dev, s.logr_dev, s.n_grid, s.log2, g.x, j2, t2);
    // kernel-column weights: idx_right = clip(searchsorted(r, x), 1, N-1)
    int ir = dwba_lower_bound(s.r_dev, s.n_grid, g.x);
    ir = ir < 1 ? 1 : (ir > s.n_grid - 1 ? s.n_grid - 1 : ir);
    const int il = ir - 1;
    const double wr = (g.x - s.r_dev[il]) / (s.r_dev[ir] - s.r_dev[il] + 1e-30);
    s.node_w_dev[c] = g.w;
    s.node_t1_dev[c] = t1;
    s.node_t2_dev[c] = t2;
    s.node_wr_dev[c] = wr;
    s.node_j1_dev[c] = j1;
    s.node_j2_dev[c] = j2;
    s.node_il_dev[c] = il;
  }
}

// Row gathers (deterministic: each output row sums its nodes in ascending order).
__global__ void bands_kernel(const dwba_nodeset_t* __restrict__ sets, int n_cc, int* status) {
  const dwba_nodeset_t s = sets[blockIdx.y];
  const int n_nodes = (s.n_breaks - 1) * n_cc;
  const int n_rows = s.n_grid;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_rows; k += gridDim.x * blockDim.x) {
    // --- T = P1^T diag(W) P1, rows k < n1 -------------------------------------------
    if (k < s.n1) {
      double lo = 0.0, di = 0.0, up = 0.0;
      // nodes with j1 == k-1 contribute through their right tap (weight t)
      if (k >= 1) {
        int c0 = dwba_lower_bound_i(s.node_j1_dev, n_nodes, k - 1);
        for (int c = c0; c < n_nodes && s.node_j1_dev[c] == k - 1; ++c) {
          const double w = s.node_w_dev[c], t = s.node_t1_dev[c];
          di += w * t * t;
          lo += w * t * (1.0 - t);
        }
      }
      int c0 = dwba_lower_bound_i(s.node_j1_dev, n_nodes, k);
      for (int c = c0; c < n_nodes && s.node_j1_dev[c] == k; ++c) {
        const double w = s.node_w_dev[c], t = s.node_t1_dev[c];
        di += w * (1.0 - t) * (1.0 - t);
        up += w * (1.0 - t) * t;
      }
      s.ta_dev[3 * k + 0] = lo;
      s.ta_dev[3 * k + 1] = di;
      s.ta_dev[3 * k + 2] = up;
    }
    // --- B = Q^T diag(W) P2, all rows ----------------------------------------------
    double band[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    bool bad = false;
    for (int side = 0; side < 2; ++side) {
      // side 0: nodes with il == k (left column, weight 1-wr); side 1: il == k-1 (right column, wr)
      const int key = k - side;
      if (key < 0) continue;
      int c0 = dwba_lower_bound_i(s.node_il_dev, n_nodes, key);
      for (int c = c0; c < n_nodes && s.node_il_dev[c] == key; ++c) {
        const double wr = s.node_wr_dev[c];
        const double q = side == 0 ? 1.0 - wr : wr;
        const double w = s.node_w_dev[c], t = s.node_t2_dev[c];
        const int j = s.node_j2_dev[c];
        const int d0 = j - k, d1 = j + 1 - k;
        if (d0 < -2 || d1 > 2) { bad = true; continue; }
        band[d0 + 2] += q * w * (1.0 - t);
        band[d1 + 2] += q * w * t;
      }
    }
    if (bad) atomicExch(status, 1);
#pragma unroll
    for (int d = 0; d < 5; ++d) s.bx_dev[5 * k + d] = band[d];
  }
}

}  // namespace

extern "C" int dwba_build_nodesets(const dwba_nodeset_t* sets_dev, int n_sets, int max_nodes, int max_grid,
                                   const double* cc_x_dev, const double* cc_w_dev, int n_cc, int* status_dev,
                                   dwba_stream_t stream) {
  if (n_sets <= 0) return DWBA_OK;
  if (!sets_dev || !cc_x_dev || !cc_w_dev || !status_dev || n_cc < 2 || n_cc > 15 || max_nodes < 0 ||
      max_grid < 2 || n_sets > 65535)
    return DWBA_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  dim3 g1(dwba_grid_1d(max_nodes, 256, 4096), n_sets);
  nodes_kernel<<<g1, 256, 0, st>>>(sets_dev, cc_x_dev, cc_w_dev, n_cc);
  DWBA_CHECK_LAUNCH();
  dim3 g2(dwba_grid_1d(max_grid, 256, 4096), n_sets);
  bands_kernel<<<g2, 256, 0, st>>>(sets_dev, n_cc, status_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
