// Exact O(n L) evaluation of the bilinear forms a^T K_L b in FP64.
//
// The multipole kernel of dwba_matrix_elements.py:1057-1116 is semiseparable:
// K_L(r_p, r_q) = r_q^L / r_p^(L+1) for q < p. With X = a, Y = b (zero past their
// lengths) and exclusive prefix sums A_L(p) = sum_{q<p} X_q r_q^L,
// B_L(p) = sum_{q<p} Y_q r_q^L:
//   I_L = sum_p r_p^-(L+1) (X_p B_L(p) + Y_p A_L(p)) + sum_p X_p Y_p (1-1e-12)^L / r_p,
// the same identity the reference uses for Hartree potentials
// (distorting_potential.py:235-251). One CTA per form: each thread owns a
// contiguous segment, segment totals are scanned in shared memory, then every
// thread sweeps its segment again with its running prefix.
#include "common.cuh"

namespace {

constexpr int THREADS = 128;  // 2*16*(128+1) doubles of scan storage stay under 48 KB
constexpr int NL_MAX = 16;

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
semisep_kernel(const dwba_form_t* __restrict__ forms, int L0, int n_ltot, DiagScale ds, double* __restrict__ out) {
  __shared__ double scan[2 * NL][THREADS + 1];
  __shared__ double red[THREADS / 32][NL];
  const dwba_form_t F = forms[blockIdx.x];
  const int M = F.n_rows > F.n_cols ? F.n_rows : F.n_cols;
  const int tid = threadIdx.x;
  const int seg = (M + THREADS - 1) / THREADS;
  const int p0 = tid * seg;
  const int p1 = min(M, p0 + seg);

  // pass 1: segment totals of X r^L and Y r^L
  double sa[NL], sb[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) sa[l] = sb[l] = 0.0;
  for (int p = p0; p < p1; ++p) {
    const double X = p < F.n_rows ? F.a_dev[p] : 0.0;
    const double Y = p < F.n_cols ? F.b_dev[p] : 0.0;
    const double r = F.r_dev[p];
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      sa[l] += X * pw;
      sb[l] += Y * pw;
      pw *= r;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    scan[l][tid + 1] = sa[l];
    scan[NL + l][tid + 1] = sb[l];
  }
  __syncthreads();
  if (tid < 2 * NL) {  // exclusive scan over the segments, one thread per series
    double s = 0.0;
    scan[tid][0] = 0.0;
    for (int k = 1; k <= THREADS; ++k) {
      s += scan[tid][k];
      scan[tid][k] = s;
    }
  }
  __syncthreads();
  double A[NL], B[NL], acc[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    A[l] = scan[l][tid];
    B[l] = scan[NL + l][tid];
    acc[l] = 0.0;
  }
  // pass 2: sweep with running prefixes; two elements per iteration so their power chains
  // overlap. The diagonal term sum_p X_p Y_p / r_p is collected once and scaled per L at the end.
  double dsum = 0.0;
  int p = p0;
  for (; p + 1 < p1; p += 2) {
    const double X0 = p < F.n_rows ? F.a_dev[p] : 0.0, X1 = p + 1 < F.n_rows ? F.a_dev[p + 1] : 0.0;
    const double Y0 = p < F.n_cols ? F.b_dev[p] : 0.0, Y1 = p + 1 < F.n_cols ? F.b_dev[p + 1] : 0.0;
    const double r0 = F.r_dev[p], r1 = F.r_dev[p + 1];
    const double i0 = 1.0 / r0, i1 = 1.0 / r1;
    double pw0 = L0 > 0 ? ipow(r0, L0) : 1.0, pw1 = L0 > 0 ? ipow(r1, L0) : 1.0;
    double ip0 = L0 > 0 ? ipow(i0, L0 + 1) : i0, ip1 = L0 > 0 ? ipow(i1, L0 + 1) : i1;
    dsum += X0 * Y0 * i0;
    dsum += X1 * Y1 * i1;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      acc[l] += ip0 * fma(X0, B[l], Y0 * A[l]);
      A[l] += X0 * pw0;
      B[l] += Y0 * pw0;
      acc[l] += ip1 * fma(X1, B[l], Y1 * A[l]);
      A[l] += X1 * pw1;
      B[l] += Y1 * pw1;
      pw0 *= r0;
      pw1 *= r1;
      ip0 *= i0;
      ip1 *= i1;
    }
  }
  for (; p < p1; ++p) {
    const double X = p < F.n_rows ? F.a_dev[p] : 0.0;
    const double Y = p < F.n_cols ? F.b_dev[p] : 0.0;
    const double r = F.r_dev[p];
    const double inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ipw = L0 > 0 ? ipow(inv, L0 + 1) : inv;
    dsum += X * Y * inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      acc[l] += ipw * fma(X, B[l], Y * A[l]);
      A[l] += X * pw;
      B[l] += Y * pw;
      pw *= r;
      ipw *= inv;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) acc[l] += dsum * ds.v[L0 + l];
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double v = acc[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][l] = v;
  }
  __syncthreads();
  if (tid < NL) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < THREADS / 32; ++w) s += red[w][tid];
    out[(int64_t)blockIdx.x * n_ltot + L0 + tid] = s;
  }
}

template <int NL>
int launch(const dwba_form_t* forms, int n_forms, int L0, int n_ltot, const DiagScale& ds, double* out,
           cudaStream_t st) {
  semisep_kernel<NL><<<n_forms, THREADS, 0, st>>>(forms, L0, n_ltot, ds, out);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

int launch_nl(int nl, const dwba_form_t* forms, int n_forms, int L0, int n_ltot, const DiagScale& ds, double* out,
              cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch<N>(forms, n_forms, L0, n_ltot, ds, out, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
    DWBA_CASE(9) DWBA_CASE(10) DWBA_CASE(11) DWBA_CASE(12) DWBA_CASE(13) DWBA_CASE(14) DWBA_CASE(15)
    DWBA_CASE(16)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

}  // namespace

extern "C" int dwba_bilinear_semisep_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max,
                                          const double* diag_scale_host, double r_min_all, double r_max_all,
                                          double* out_dev, dwba_stream_t stream) {
  if (n_forms <= 0) return DWBA_OK;
  if (!forms_dev || !diag_scale_host || !out_dev || L_max < 0 || L_max > DWBA_MAX_L || !(r_min_all > 0.0) ||
      !(r_max_all >= r_min_all) || n_forms > 0x7fffffff)
    return DWBA_ERR_INVALID_ARG;
  // r^L and r^-(L+1) must stay finite and normal in FP64
  const double lmin = log10(r_min_all), lmax = log10(r_max_all);
  const double worst = fmax(fabs(lmin) * (L_max + 1), fabs(lmax) * (L_max + 1));
  if (worst > 280.0) return DWBA_ERR_UNSUPPORTED;
  DiagScale ds;
  for (int l = 0; l <= DWBA_MAX_L; ++l) ds.v[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  const int n_ltot = L_max + 1;
  for (int L0 = 0; L0 < n_ltot; L0 += NL_MAX) {
    const int nl = (n_ltot - L0) < NL_MAX ? (n_ltot - L0) : NL_MAX;
    int rc = launch_nl(nl, forms_dev, n_forms, L0, n_ltot, ds, out_dev, (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}
