// Exact O(n L) evaluation of the bilinear forms a^T K_L b in FP64.
//
// The multipole kernel of dwba_matrix_elements.py:1057-1116 is semiseparable:
// K_L(r_p, r_q) = r_q^L / r_p^(L+1) for q < p. With X = a, Y = b (zero past their
// lengths) and exclusive prefix sums A_L(p) = sum_{q<p} X_q r_q^L,
// B_L(p) = sum_{q<p} Y_q r_q^L:
//   I_L = sum_p r_p^-(L+1) (X_p B_L(p) + Y_p A_L(p)) + sum_p X_p Y_p (1-1e-12)^L / r_p,
// the same identity the reference uses for Hartree potentials
// (distorting_potential.py:235-251). One CTA per form and one pass over the operands:
// each thread owns a contiguous segment (see semisep_kernel).
#include "common.cuh"

namespace {

constexpr int THREADS = 128;
constexpr int NL_MAX = 9;  // multipoles per launch (5 accumulators each per thread)

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

// Single pass over the operands. Thread s owns a contiguous segment and accumulates, per L,
//   TA = sum X r^L, TB = sum Y r^L          (segment totals)
//   SX = sum X r^-(L+1), SY = sum Y r^-(L+1)
//   LOC = sum r_p^-(L+1) (X_p B_loc(p) + Y_p A_loc(p))   (prefixes local to the segment)
// and with the exclusive prefixes A0, B0 of TA, TB over the segments before it,
//   I_L = sum_s [LOC_s + A0_s SY_s + B0_s SX_s] + sum_p X_p Y_p d_L / r_p.
// The prefixes over segments come from warp shuffles and a per-warp table in shared memory.
// ABS = true evaluates |a|^T K_L |b| (the cancellation scale S_L of the form) instead.
template <int NL, bool ABS = false>
__global__ void __launch_bounds__(THREADS, 4)
semisep_kernel(const dwba_form_t* __restrict__ forms, int L0, int n_ltot, DiagScale ds, double* __restrict__ out) {
  constexpr int NW = THREADS / 32;
  __shared__ double wtot[2 * NL][NW];
  __shared__ double red[NW][NL];
  const dwba_form_t F = forms[blockIdx.x];
  const int M = F.n_rows > F.n_cols ? F.n_rows : F.n_cols;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int seg = (M + THREADS - 1) / THREADS;
  const int p0 = tid * seg;
  const int p1 = min(M, p0 + seg);

  double A[NL], B[NL], SX[NL], SY[NL], LOC[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) A[l] = B[l] = SX[l] = SY[l] = LOC[l] = 0.0;
  double dsum = 0.0;
  // the operands of point p+1 are loaded while point p is accumulated (one point of lead hides
  // the load latency of the thread's strided walk; 128 registers keep four CTAs per SM)
  auto ldx = [&](int p) { return p < F.n_rows ? (ABS ? fabs(__ldg(F.a_dev + p)) : __ldg(F.a_dev + p)) : 0.0; };
  auto ldy = [&](int p) { return p < F.n_cols ? (ABS ? fabs(__ldg(F.b_dev + p)) : __ldg(F.b_dev + p)) : 0.0; };
  double Xn = p0 < p1 ? ldx(p0) : 0.0, Yn = p0 < p1 ? ldy(p0) : 0.0, rn = p0 < p1 ? __ldg(F.r_dev + p0) : 1.0;
  for (int p = p0; p < p1; ++p) {
    const double X = Xn, Y = Yn, r = rn;
    if (p + 1 < p1) {
      Xn = ldx(p + 1);
      Yn = ldy(p + 1);
      rn = __ldg(F.r_dev + p + 1);
    }
    const double inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
    dsum += X * Y * inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      LOC[l] += ip * fma(X, B[l], Y * A[l]);
      SX[l] += ip * X;
      SY[l] += ip * Y;
      A[l] += X * pw;
      B[l] += Y * pw;
      pw *= r;
      ip *= inv;
    }
  }
  // exclusive prefix over segments of A and B (warp scan, then warp totals)
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double va = A[l], vb = B[l];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double ta = __shfl_up_sync(0xffffffffu, va, off), tb = __shfl_up_sync(0xffffffffu, vb, off);
      if (lane >= off) {
        va += ta;
        vb += tb;
      }
    }
    if (lane == 31) {
      wtot[l][warp] = va;
      wtot[NL + l][warp] = vb;
    }
    A[l] = va - A[l];  // exclusive within the warp
    B[l] = vb - B[l];
  }
  __syncthreads();
  double acc[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double oa = 0.0, ob = 0.0;
    for (int w = 0; w < warp; ++w) {
      oa += wtot[l][w];
      ob += wtot[NL + l][w];
    }
    acc[l] = LOC[l] + (A[l] + oa) * SY[l] + (B[l] + ob) * SX[l] + dsum * ds.v[L0 + l];
  }
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
    for (int w = 0; w < NW; ++w) s += red[w][tid];
    out[(int64_t)blockIdx.x * n_ltot + L0 + tid] = s;
  }
}

template <int NL, bool ABS>
int launch(const dwba_form_t* forms, int n_forms, int L0, int n_ltot, const DiagScale& ds, double* out,
           cudaStream_t st) {
  semisep_kernel<NL, ABS><<<n_forms, THREADS, 0, st>>>(forms, L0, n_ltot, ds, out);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

template <bool ABS>
int launch_nl(int nl, const dwba_form_t* forms, int n_forms, int L0, int n_ltot, const DiagScale& ds, double* out,
              cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch<N, ABS>(forms, n_forms, L0, n_ltot, ds, out, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
    DWBA_CASE(9)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

}  // namespace

template <bool ABS>
static int semisep_entry(const dwba_form_t* forms_dev, int n_forms, int L_max, const double* diag_scale_host,
                  double r_min_all, double r_max_all, double* out_dev, dwba_stream_t stream) {
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
    int rc = launch_nl<ABS>(nl, forms_dev, n_forms, L0, n_ltot, ds, out_dev, (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}

extern "C" int dwba_bilinear_semisep_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max,
                                          const double* diag_scale_host, double r_min_all, double r_max_all,
                                          double* out_dev, dwba_stream_t stream) {
  return semisep_entry<false>(forms_dev, n_forms, L_max, diag_scale_host, r_min_all, r_max_all, out_dev, stream);
}

extern "C" int dwba_bilinear_semisep_abs_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max,
                                              const double* diag_scale_host, double r_min_all, double r_max_all,
                                              double* out_dev, dwba_stream_t stream) {
  return semisep_entry<true>(forms_dev, n_forms, L_max, diag_scale_host, r_min_all, r_max_all, out_dev, stream);
}
