// Exchange integrals with the quadrature of the reference's CuPy path.
//
// radial_ME_all_L_gpu (dwba_matrix_elements.py:1563-2549) evaluates the exchange inner integral over
// the Clenshaw-Curtis nodes of r[:n1] with the kernel at a node x in (r_j, r_{j+1}] formed from the
// linearly interpolated 1/r_> and log-ratio of the grid columns j and j+1 (:2072-2091,
// _gpu_filon_exchange :1469-1560):
//     K~(r_i, x) = [wL/max(r_i, r_j) + wR/max(r_i, r_{j+1})]
//                  exp(L [wL log(min/max)(r_i, r_j) + wR log(min/max)(r_i, r_{j+1})]),
// wR = (x - r_j)/(r_{j+1} - r_j + 1e-30), wL = 1 - wR. For a grid row i this factorises exactly:
//     i >= j+1:  K~ = r_i^-(L+1) G^L,          i <= j:  K~ = h r_i^L G^-L,
// with G = exp(wL log r_j + wR log r_{j+1}) (the geometric interpolation of the interval ends) and
// h = wL/r_j + wR/r_{j+1}. With rho2 interpolated linearly on r[:n1] (cp.interp; weight t),
//     inner_i = r_i^-(L+1) sum_{j<i} [alpha_L(j) rho2_j + beta_L(j) rho2_{j+1}]
//             + r_i^L      sum_{j>=i} [gamma_L(j) rho2_j + delta_L(j) rho2_{j+1}],
//     alpha = sum_c W G^L (1-t), beta = sum_c W G^L t, gamma = sum_c W h G^-L (1-t), delta = sum_c W h G^-L t
// over the nodes c of interval j. The outer sum is the CC fold a = T rho1 of the same node set
// (linear interpolation), so I_L = sum_{i<n1} a_i inner_i: O(n1 L) per form, the interval
// coefficients computed once per node set.
#include "phase_nodes.cuh"

namespace {

using namespace dwba_nodes;

constexpr int OPS_THREADS = 128;
constexpr int OPS_NL = 8;  // multipoles per pass of the coefficient kernel

// One thread per grid interval j < n1 - 1: the nodes x it owns (x in (r_j, r_{j+1}], j = 0 also r_0,
// the intervals searchsorted-left and the clip to [1, n1-1] assign) and their coefficients for the
// multipoles L0 .. L0+NL-1, written to ops[((L * n1) + j) * 4 + {0: alpha, 1: beta, 2: gamma, 3: delta}].
template <int NL>
__global__ void __launch_bounds__(OPS_THREADS)
cupy_ops_kernel(const dwba_cupy_set_t* __restrict__ sets, const double* __restrict__ ccx_g,
                const double* __restrict__ ccw_g, int n_cc, int L0) {
  __shared__ double ccw[MAX_CC], ccx1[MAX_CC];
  if (threadIdx.x < n_cc) {
    ccw[threadIdx.x] = ccw_g[threadIdx.x];
    ccx1[threadIdx.x] = rn_add(ccx_g[threadIdx.x], 1.0);
  }
  __syncthreads();
  const dwba_cupy_set_t d = sets[blockIdx.y];
  SetView s;
  s.r = d.r_dev;
  s.lr = d.logr_dev;
  s.br = nullptr;  // the CuPy path's phase intervals are always a linspace
  s.n_grid = d.n1;
  s.n1 = d.n1;
  s.n_int = d.n_breaks - 1;
  s.log1 = s.log2 = 0;
  s.start = s.r[0];
  s.stop = s.r[s.n1 - 1];
  s.step = rn_sub(s.stop, s.start) / (double)s.n_int;
  const int n1 = d.n1;
  const double* __restrict__ r = s.r;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n1; j += gridDim.x * blockDim.x) {
    double al[NL], be[NL], ga[NL], de[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) al[l] = be[l] = ga[l] = de[l] = 0.0;
    if (j <= n1 - 2) {
      const double rj = r[j], rj1 = r[j + 1];
      const double lj = s.lr[j], lj1 = s.lr[j + 1];
      const double lo = j == 0 ? -1.0e308 : rj;
      const double iw = 1.0 / (rj1 - rj + 1e-30), it = 1.0 / (rj1 - rj);
      bool done = false;
      for (int m = interval_floor(s, rj); m < s.n_int && !done; ++m) {
        double a, b;
        interval(s, m, a, b);
        if (a > rj1) break;
        const double width = rn_sub(b, a);
        if (!(width > 1e-12)) continue;
        const double hw = rn_mul(0.5, width);
        for (int sl = n_cc - 1; sl >= 0; --sl) {
          double x = rn_add(rn_mul(hw, ccx1[sl]), a);
          x = fmin(fmax(x, a), b);
          if (!(x > lo)) continue;
          if (x > rj1) {
            done = true;
            break;
          }
          const double W = rn_mul(ccw[sl], hw);
          const double wR = (x - rj) * iw, wL = 1.0 - wR;
          const double t = (x - rj) * it;
          const double G = exp(wL * lj + wR * lj1);
          const double iG = 1.0 / G;
          const double h = wL / rj + wR / rj1;
          double p = L0 > 0 ? pow(G, (double)L0) : 1.0;
          double q = h * (L0 > 0 ? pow(iG, (double)L0) : 1.0);
          const double w0 = W * (1.0 - t), w1 = W * t;
#pragma unroll
          for (int l = 0; l < NL; ++l) {
            al[l] = fma(p, w0, al[l]);
            be[l] = fma(p, w1, be[l]);
            ga[l] = fma(q, w0, ga[l]);
            de[l] = fma(q, w1, de[l]);
            p *= G;
            q *= iG;
          }
        }
      }
    }
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (L0 + l > d.L_max) break;
      double* o = d.ops_dev + ((int64_t)(L0 + l) * n1 + j) * 4;
      o[0] = al[l];
      o[1] = be[l];
      o[2] = ga[l];
      o[3] = de[l];
    }
  }
}

template <int NL>
int launch_ops(const dwba_cupy_set_t* sets, int n_sets, int max_n1, const double* ccx, const double* ccw, int n_cc,
               int L0, cudaStream_t st) {
  dim3 grid(dwba_grid_1d(max_n1, OPS_THREADS, 4096), n_sets);
  cupy_ops_kernel<NL><<<grid, OPS_THREADS, 0, st>>>(sets, ccx, ccw, n_cc, L0);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

// ---- forms ------------------------------------------------------------------------------------
constexpr int FT = 128;
constexpr int F_NL = 8;

__device__ __forceinline__ double ipow(double x, int e) {
  double r = 1.0;
  while (e > 0) {
    if (e & 1) r *= x;
    x *= x;
    e >>= 1;
  }
  return r;
}

// I_L = sum_{i<n1} a_i [r_i^-(L+1) sum_{j<i} A_L(j) + r_i^L sum_{j>=i} B_L(j)], A_L(j) = alpha rho2_j +
// beta rho2_{j+1}, B_L(j) = gamma rho2_j + delta rho2_{j+1} (rho2 = f g), by segments per thread:
// segment totals, an exclusive prefix of A and suffix of B over segments, then a forward sweep with the
// running prefix and a backward sweep with the running suffix.
template <int NL>
__global__ void __launch_bounds__(FT)
cupy_forms_kernel(const dwba_cupy_form_t* __restrict__ forms, int L0) {
  __shared__ double scan[2 * NL][FT + 1];
  __shared__ double red[FT / 32][NL];
  const dwba_cupy_form_t F = forms[blockIdx.x];
  const int n1 = F.n1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int seg = (n1 + FT - 1) / FT;
  const int p0 = tid * seg, p1 = min(n1, p0 + seg);
  auto rho = [&](int j) { return j < n1 ? F.f_dev[j] * F.g_dev[j] : 0.0; };
  auto cols = [&](int j, int l, double& A, double& B) {
    if (j > n1 - 2) {
      A = B = 0.0;
      return;
    }
    const double* o = F.ops_dev + ((int64_t)(L0 + l) * n1 + j) * 4;
    const double x0 = rho(j), x1 = rho(j + 1);
    A = fma(o[0], x0, o[1] * x1);
    B = fma(o[2], x0, o[3] * x1);
  };
  double tA[NL], tB[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) tA[l] = tB[l] = 0.0;
  for (int j = p0; j < p1; ++j) {
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (L0 + l > F.L_max) break;
      double A, B;
      cols(j, l, A, B);
      tA[l] += A;
      tB[l] += B;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    scan[l][tid] = tA[l];
    scan[NL + l][tid + 1] = tB[l];
  }
  __syncthreads();
  if (tid < NL) {
    double s = 0.0;
    for (int k = 0; k < FT; ++k) {
      const double v = scan[tid][k];
      scan[tid][k] = s;
      s += v;
    }
  } else if (tid < 2 * NL) {
    double s = 0.0;
    for (int k = FT - 1; k >= 0; --k) {
      const double v = scan[tid][k + 1];
      scan[tid][k + 1] = s;
      s += v;
    }
  }
  __syncthreads();
  double acc[NL], P[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    acc[l] = 0.0;
    P[l] = scan[l][tid];
  }
  for (int i = p0; i < p1; ++i) {  // forward: the intervals below row i
    const double ai = F.a_dev[i], ri = F.r_dev[i], inv = 1.0 / ri;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (L0 + l > F.L_max) break;
      acc[l] = fma(ai * ip, P[l], acc[l]);
      double A, B;
      cols(i, l, A, B);
      P[l] += A;
      ip *= inv;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) P[l] = scan[NL + l][tid + 1];
  for (int i = p1 - 1; i >= p0; --i) {  // backward: the intervals j >= i
    const double ai = F.a_dev[i], ri = F.r_dev[i];
    double pw = L0 > 0 ? ipow(ri, L0) : 1.0;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (L0 + l > F.L_max) break;
      double A, B;
      cols(i, l, A, B);
      P[l] += B;
      acc[l] = fma(ai * pw, P[l], acc[l]);
      pw *= ri;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double v = acc[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][l] = v;
  }
  __syncthreads();
  if (tid < NL && L0 + tid <= F.L_max) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < FT / 32; ++w) v += red[w][tid];
    F.out_dev[L0 + tid] = v;
  }
}

template <int NL>
int launch_forms(const dwba_cupy_form_t* forms, int n, int L0, cudaStream_t st) {
  cupy_forms_kernel<NL><<<n, FT, 0, st>>>(forms, L0);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

}  // namespace

extern "C" int dwba_cupy_exchange_ops(const dwba_cupy_set_t* sets_dev, int n_sets, int max_n1, int L_max,
                                      const double* cc_x_dev, const double* cc_w_dev, int n_cc, dwba_stream_t stream) {
  if (n_sets <= 0) return DWBA_OK;
  if (!sets_dev || !cc_x_dev || !cc_w_dev || n_cc < 2 || n_cc > MAX_CC || max_n1 < 2 || n_sets > 65535 ||
      L_max < 0 || L_max > DWBA_MAX_L)
    return DWBA_ERR_INVALID_ARG;
  for (int L0 = 0; L0 <= L_max; L0 += OPS_NL) {
    const int rc = launch_ops<OPS_NL>(sets_dev, n_sets, max_n1, cc_x_dev, cc_w_dev, n_cc, L0, (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}

extern "C" int dwba_cupy_exchange_forms(const dwba_cupy_form_t* forms_dev, int n, int L_max, double r_min_all,
                                        double r_max_all, dwba_stream_t stream) {
  if (n <= 0) return DWBA_OK;
  if (!forms_dev || L_max < 0 || L_max > DWBA_MAX_L || !(r_min_all > 0.0) || !(r_max_all >= r_min_all))
    return DWBA_ERR_INVALID_ARG;
  const double lmin = log10(r_min_all), lmax = log10(r_max_all);
  if (fmax(fabs(lmin), fabs(lmax)) * (L_max + 1) > 280.0) return DWBA_ERR_UNSUPPORTED;
  for (int L0 = 0; L0 <= L_max; L0 += F_NL) {
    const int rc = launch_forms<F_NL>(forms_dev, n, L0, (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}
