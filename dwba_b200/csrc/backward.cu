// Backward of the bilinear forms and of the operand folds (FP64, exact).
//
// The forward computes I_L = a^T K_L b (semisep_fp64.cu). K_L is symmetric, so for upstream
// gradients g_L = dLoss/dI_L the operand gradients are
//   dLoss/da = K_g b,   dLoss/db = K_g a,   K_g = sum_L g_L K_L,
// and with the semiseparable structure K_L(p, q) = r_q^L / r_p^(L+1) (q < p), its transpose
// above the diagonal and (1-1e-12)^L / r_p on it:
//   (K_g y)_p = sum_L g_L [ r_p^-(L+1) sum_{q<p} y_q r_q^L + r_p^L sum_{q>p} y_q r_q^-(L+1)
//                           + d_L y_p / r_p ].
// The prefix sums run forward and the suffix sums backward (each is accumulated from its own
// end, so no sum is formed as a difference of totals). One CTA per form, segments per thread
// as in the forward kernel.
//
// The folds a = Op (f .* g) (fold.cu) are linear in the product, so dLoss/d(f .* g) = Op^T y
// for y = dLoss/da; the caller multiplies by g and f.
#include "common.cuh"

namespace {

constexpr int THREADS = 128;
constexpr int NL_MAX = 8;  // 4 scanned series x 8 multipoles x 129 doubles = 33 KB of shared memory

struct DiagScale {
  double v[DWBA_MAX_L + 1];
};

__device__ __forceinline__ double ipow(double x, int e) {
  double r = 1.0;
  while (e > 0) {
    if (e & 1) r *= x;
    x *= x;
    e >>= 1;
  }
  return r;
}

template <int NL>
__global__ void __launch_bounds__(THREADS)
semisep_backward_kernel(const dwba_form_grad_t* __restrict__ forms, const double* __restrict__ grad, int L0,
                        int n_ltot, DiagScale ds, int accumulate) {
  __shared__ double scan[4 * NL][THREADS + 1];
  const dwba_form_grad_t F = forms[blockIdx.x];
  const int M = F.n_rows > F.n_cols ? F.n_rows : F.n_cols;
  const int tid = threadIdx.x;
  const int seg = (M + THREADS - 1) / THREADS;
  const int p0 = tid * seg;
  const int p1 = min(M, p0 + seg);
  double g[NL];
  double gd = 0.0;  // sum_L g_L d_L over this chunk of multipoles
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    g[l] = grad[(int64_t)blockIdx.x * n_ltot + L0 + l];
    gd += g[l] * ds.v[L0 + l];
  }

  // pass 1: segment totals of a r^L, b r^L (prefix series) and a r^-(L+1), b r^-(L+1) (suffix series)
  double ta[NL], tb[NL], sa[NL], sb[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) ta[l] = tb[l] = sa[l] = sb[l] = 0.0;
  for (int p = p0; p < p1; ++p) {
    const double X = p < F.n_rows ? F.a_dev[p] : 0.0;
    const double Y = p < F.n_cols ? F.b_dev[p] : 0.0;
    const double r = F.r_dev[p], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      ta[l] += X * pw;
      tb[l] += Y * pw;
      sa[l] += X * ip;
      sb[l] += Y * ip;
      pw *= r;
      ip *= inv;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    scan[l][tid] = ta[l];
    scan[NL + l][tid] = tb[l];
    scan[2 * NL + l][tid + 1] = sa[l];
    scan[3 * NL + l][tid + 1] = sb[l];
  }
  __syncthreads();
  if (tid < 2 * NL) {  // exclusive prefix over segments: entry k = sum of segments < k
    double s = 0.0;
    for (int k = 0; k < THREADS; ++k) {
      const double v = scan[tid][k];
      scan[tid][k] = s;
      s += v;
    }
  } else if (tid < 4 * NL) {  // exclusive suffix over segments: entry k+1 = sum of segments > k
    double s = 0.0;
    for (int k = THREADS - 1; k >= 0; --k) {
      const double v = scan[tid][k + 1];
      scan[tid][k + 1] = s;
      s += v;
    }
  }
  __syncthreads();

  // pass 2: forward sweep with running prefixes (and the diagonal term)
  double PA[NL], PB[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    PA[l] = scan[l][tid];
    PB[l] = scan[NL + l][tid];
  }
  for (int p = p0; p < p1; ++p) {
    const double X = p < F.n_rows ? F.a_dev[p] : 0.0;
    const double Y = p < F.n_cols ? F.b_dev[p] : 0.0;
    const double r = F.r_dev[p], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
    double u = gd * Y * inv, v = gd * X * inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      u += g[l] * ip * PB[l];
      v += g[l] * ip * PA[l];
      PA[l] += X * pw;
      PB[l] += Y * pw;
      pw *= r;
      ip *= inv;
    }
    if (p < F.n_rows) F.ga_dev[p] = accumulate ? F.ga_dev[p] + u : u;
    if (p < F.n_cols) F.gb_dev[p] = accumulate ? F.gb_dev[p] + v : v;
  }
  // pass 3: backward sweep with running suffixes (same thread, same elements: no barrier needed)
  double SA[NL], SB[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    SA[l] = scan[2 * NL + l][tid + 1];
    SB[l] = scan[3 * NL + l][tid + 1];
  }
  for (int p = p1 - 1; p >= p0; --p) {
    const double X = p < F.n_rows ? F.a_dev[p] : 0.0;
    const double Y = p < F.n_cols ? F.b_dev[p] : 0.0;
    const double r = F.r_dev[p], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
    double u = 0.0, v = 0.0;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      u += g[l] * pw * SB[l];
      v += g[l] * pw * SA[l];
      SA[l] += X * ip;
      SB[l] += Y * ip;
      pw *= r;
      ip *= inv;
    }
    if (p < F.n_rows) F.ga_dev[p] += u;
    if (p < F.n_cols) F.gb_dev[p] += v;
  }
}

template <int NL>
int launch(const dwba_form_grad_t* forms, int n, const double* grad, int L0, int n_ltot, const DiagScale& ds,
           int acc, cudaStream_t st) {
  semisep_backward_kernel<NL><<<n, THREADS, 0, st>>>(forms, grad, L0, n_ltot, ds, acc);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

int launch_nl(int nl, const dwba_form_grad_t* forms, int n, const double* grad, int L0, int n_ltot,
              const DiagScale& ds, int acc, cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch<N>(forms, n, grad, L0, n_ltot, ds, acc, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

// z = Op^T y for one fold; Op row i holds the taps of columns i-H..i+H
__global__ void fold_adjoint_kernel(const dwba_fold_adj_t* __restrict__ adj) {
  const dwba_fold_adj_t A = adj[blockIdx.y];
  const int H = A.half_band, W = 2 * H + 1;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < A.n_src; k += gridDim.x * blockDim.x) {
    double z = 0.0;
    for (int d = -H; d <= H; ++d) {
      const int i = k - d;  // row whose tap d reaches column k
      if (i >= 0 && i < A.n_out) z += A.op_dev[(int64_t)W * i + (d + H)] * A.y_dev[i];
    }
    A.z_dev[k] = z;
  }
}

}  // namespace

extern "C" int dwba_bilinear_semisep_backward_fp64(const dwba_form_grad_t* forms_dev, int n_forms, int L_max,
                                                   const double* diag_scale_host, const double* grad_dev,
                                                   double r_min_all, double r_max_all, dwba_stream_t stream) {
  if (n_forms <= 0) return DWBA_OK;
  if (!forms_dev || !diag_scale_host || !grad_dev || L_max < 0 || L_max > DWBA_MAX_L || !(r_min_all > 0.0) ||
      !(r_max_all >= r_min_all) || n_forms > 0x7fffffff)
    return DWBA_ERR_INVALID_ARG;
  const double lmin = log10(r_min_all), lmax = log10(r_max_all);
  const double worst = fmax(fabs(lmin) * (L_max + 1), fabs(lmax) * (L_max + 1));
  if (worst > 280.0) return DWBA_ERR_UNSUPPORTED;
  DiagScale ds;
  for (int l = 0; l <= DWBA_MAX_L; ++l) ds.v[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  const int n_ltot = L_max + 1;
  for (int L0 = 0; L0 < n_ltot; L0 += NL_MAX) {
    const int nl = (n_ltot - L0) < NL_MAX ? (n_ltot - L0) : NL_MAX;
    const int rc = launch_nl(nl, forms_dev, n_forms, grad_dev, L0, n_ltot, ds, L0 > 0 ? 1 : 0,
                             (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}

extern "C" int dwba_fold_adjoint(const dwba_fold_adj_t* adj_dev, int n, int max_len, dwba_stream_t stream) {
  if (n <= 0) return DWBA_OK;
  if (!adj_dev || max_len < 0 || n > 65535) return DWBA_ERR_INVALID_ARG;
  dim3 grid(dwba_grid_1d(max_len, 256, 1024), n);
  fold_adjoint_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(adj_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
