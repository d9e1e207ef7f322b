// Direct integrals through the multipole potential of the bound density.
//
// In the reference's Filon direct term (oscillatory_integrals.py:2555-2651) the inner integral
//     int_r2(r_p) = sum_q K_L(r_p, r_q) rho2(r_q) w_q         (:2571, rho2 = u_f u_i)
// depends on the bound states only, so every (l_i, l_f) pair of a transition shares it, and the
// outer sum is a plain weighted dot product with the pair's folded density a (the CC fold of
// chi_f chi_i). Here the inner integral of every multipole is one potential per transition,
//     phi_L(p) = r_p^-(L+1) sum_{q<p} b_q r_q^L + r_p^L sum_{q>p} b_q r_q^-(L+1) + d_L b_p / r_p,
// (K_L is semiseparable; d_L = (1-1e-12)^L is the reference's clamp of the diagonal ratio), built
// exactly in O(N L) with forward prefix and backward suffix sums, and each direct integral is
// I_L = sum_{i<n1} a_i phi_L(i): O(n1 L) per pair instead of an O(n1 L) semiseparable form with
// nine accumulator updates per point and multipole.
#include "common.cuh"

namespace {

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

// ---- potentials -------------------------------------------------------------------------------
constexpr int PT = 128;     // threads per potential (one contiguous segment each)
constexpr int P_NL = 8;     // multipoles per launch (2 scanned series x 8 x 129 doubles of shared memory)

template <int NL>
__global__ void __launch_bounds__(PT)
potential_kernel(const dwba_potential_t* __restrict__ pots, int L0, DiagScale ds) {
  __shared__ double scan[2 * NL][PT + 1];
  const dwba_potential_t D = pots[blockIdx.x];
  const int M = D.n_rows > D.n_cols ? D.n_rows : D.n_cols;
  const int tid = threadIdx.x;
  const int seg = (M + PT - 1) / PT;
  const int p0 = tid * seg;
  const int p1 = min(M, p0 + seg);
  // pass 1: segment totals of b r^L (prefix series) and b r^-(L+1) (suffix series)
  double tb[NL], sb[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) tb[l] = sb[l] = 0.0;
  for (int p = p0; p < p1; ++p) {
    const double Y = p < D.n_cols ? D.b_dev[p] : 0.0;
    const double r = D.r_dev[p], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      tb[l] += Y * pw;
      sb[l] += Y * ip;
      pw *= r;
      ip *= inv;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    scan[l][tid] = tb[l];
    scan[NL + l][tid + 1] = sb[l];
  }
  __syncthreads();
  if (tid < NL) {  // exclusive prefix over segments: entry k = sum of segments < k
    double s = 0.0;
    for (int k = 0; k < PT; ++k) {
      const double v = scan[tid][k];
      scan[tid][k] = s;
      s += v;
    }
  } else if (tid < 2 * NL) {  // exclusive suffix over segments: entry k+1 = sum of segments > k
    double s = 0.0;
    for (int k = PT - 1; k >= 0; --k) {
      const double v = scan[tid][k + 1];
      scan[tid][k + 1] = s;
      s += v;
    }
  }
  __syncthreads();
  const int pe = min(p1, D.n_rows);  // rows written
  // pass 2: forward sweep with the running prefix, plus the diagonal
  double PB[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) PB[l] = scan[l][tid];
  for (int p = p0; p < p1; ++p) {
    const double Y = p < D.n_cols ? D.b_dev[p] : 0.0;
    const double r = D.r_dev[p], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
    const double yd = Y * inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (p < pe) D.phi_dev[(int64_t)(L0 + l) * D.stride + p] = ip * PB[l] + yd * ds.v[L0 + l];
      PB[l] += Y * pw;
      pw *= r;
      ip *= inv;
    }
  }
  // pass 3: backward sweep with the running suffix (the thread's own elements: no barrier)
  double SB[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) SB[l] = scan[NL + l][tid + 1];
  for (int p = p1 - 1; p >= p0; --p) {
    const double Y = p < D.n_cols ? D.b_dev[p] : 0.0;
    const double r = D.r_dev[p], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (p < pe) D.phi_dev[(int64_t)(L0 + l) * D.stride + p] += pw * SB[l];
      SB[l] += Y * ip;
      pw *= r;
      ip *= inv;
    }
  }
}

template <int NL>
int launch_pot(const dwba_potential_t* pots, int n, int L0, const DiagScale& ds, cudaStream_t st) {
  potential_kernel<NL><<<n, PT, 0, st>>>(pots, L0, ds);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

int launch_pot_nl(int nl, const dwba_potential_t* pots, int n, int L0, const DiagScale& ds, cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch_pot<N>(pots, n, L0, ds, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

// ---- dot forms --------------------------------------------------------------------------------
// A CTA takes DOT_PER_CTA consecutive descriptors that share one potential (the caller groups
// them and pads a group with empty descriptors, n_rows = 0). Tiles of the potential's rows
// (NL multipoles x DOT_TILE points) are staged in shared memory once for all of them; warp w
// accumulates descriptors 2w and 2w+1 (each staged value serves two pairs), lanes stride over the
// tile's points, and the lanes' sums are added by shuffles in a fixed order.
constexpr int DOT_THREADS = 256;
constexpr int DOT_PER_CTA = 16;
constexpr int DOT_TILE = 128;
constexpr int DOT_NL = 16;

template <int NL>
__global__ void __launch_bounds__(DOT_THREADS)
dot_kernel(const dwba_dot_t* __restrict__ dots, int n, int L0, int n_ltot) {
  __shared__ double sphi[NL][DOT_TILE];
  __shared__ int s_rows;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int d0 = blockIdx.x * DOT_PER_CTA;
  const int da = d0 + 2 * warp, db = da + 1;
  const dwba_dot_t A = da < n ? dots[da] : dwba_dot_t{nullptr, nullptr, nullptr, 0, 0};
  const dwba_dot_t B = db < n ? dots[db] : dwba_dot_t{nullptr, nullptr, nullptr, 0, 0};
  if (tid == 0) s_rows = 0;
  __syncthreads();
  if (lane == 0) atomicMax(&s_rows, max(A.n_rows, B.n_rows));
  __syncthreads();
  const int rows = s_rows;
  // the group's potential: the first descriptor's (every non-empty one of the group shares it)
  const dwba_dot_t G = dots[d0];
  double acc_a[NL], acc_b[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) acc_a[l] = acc_b[l] = 0.0;
  for (int i0 = 0; i0 < rows; i0 += DOT_TILE) {
    for (int k = tid; k < NL * DOT_TILE; k += DOT_THREADS) {
      const int l = k / DOT_TILE, i = i0 + (k - l * DOT_TILE);
      sphi[l][k - l * DOT_TILE] = i < rows ? G.phi_dev[(int64_t)(L0 + l) * G.stride + i] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < DOT_TILE / 32; ++q) {
      const int ii = q * 32 + lane, i = i0 + ii;
      const double xa = i < A.n_rows ? A.a_dev[i] : 0.0;
      const double xb = i < B.n_rows ? B.a_dev[i] : 0.0;
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        const double ph = sphi[l][ii];
        acc_a[l] = fma(xa, ph, acc_a[l]);
        acc_b[l] = fma(xb, ph, acc_b[l]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double va = acc_a[l], vb = acc_b[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      va += __shfl_down_sync(0xffffffffu, va, off);
      vb += __shfl_down_sync(0xffffffffu, vb, off);
    }
    if (lane == 0) {
      if (A.out_dev != nullptr) A.out_dev[L0 + l] = va;
      if (B.out_dev != nullptr) B.out_dev[L0 + l] = vb;
    }
  }
}

template <int NL>
int launch_dot(const dwba_dot_t* dots, int n, int L0, int n_ltot, cudaStream_t st) {
  const int grid = (n + DOT_PER_CTA - 1) / DOT_PER_CTA;
  dot_kernel<NL><<<grid, DOT_THREADS, 0, st>>>(dots, n, L0, n_ltot);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

int launch_dot_nl(int nl, const dwba_dot_t* dots, int n, int L0, int n_ltot, cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch_dot<N>(dots, n, L0, n_ltot, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
    DWBA_CASE(9) DWBA_CASE(10) DWBA_CASE(11) DWBA_CASE(12) DWBA_CASE(13) DWBA_CASE(14) DWBA_CASE(15)
    DWBA_CASE(16)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

}  // namespace

extern "C" int dwba_multipole_potentials(const dwba_potential_t* pots_dev, int n, int L_max,
                                         const double* diag_scale_host, double r_min_all, double r_max_all,
                                         dwba_stream_t stream) {
  if (n <= 0) return DWBA_OK;
  if (!pots_dev || !diag_scale_host || L_max < 0 || L_max > DWBA_MAX_L || !(r_min_all > 0.0) ||
      !(r_max_all >= r_min_all) || n > 0x7fffffff)
    return DWBA_ERR_INVALID_ARG;
  // r^L and r^-(L+1) must stay finite and normal in FP64
  const double lmin = log10(r_min_all), lmax = log10(r_max_all);
  if (fmax(fabs(lmin), fabs(lmax)) * (L_max + 1) > 280.0) return DWBA_ERR_UNSUPPORTED;
  DiagScale ds;
  for (int l = 0; l <= DWBA_MAX_L; ++l) ds.v[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  const int n_ltot = L_max + 1;
  for (int L0 = 0; L0 < n_ltot; L0 += P_NL) {
    const int nl = (n_ltot - L0) < P_NL ? (n_ltot - L0) : P_NL;
    const int rc = launch_pot_nl(nl, pots_dev, n, L0, ds, (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}

extern "C" int dwba_dot_forms(const dwba_dot_t* dots_dev, int n, int L_max, dwba_stream_t stream) {
  if (n <= 0) return DWBA_OK;
  if (!dots_dev || L_max < 0 || L_max > DWBA_MAX_L) return DWBA_ERR_INVALID_ARG;
  const int n_ltot = L_max + 1;
  for (int L0 = 0; L0 < n_ltot; L0 += DOT_NL) {
    const int nl = (n_ltot - L0) < DOT_NL ? (n_ltot - L0) : DOT_NL;
    const int rc = launch_dot_nl(nl, dots_dev, n, L0, n_ltot, (cudaStream_t)stream);
    if (rc != DWBA_OK) return rc;
  }
  return DWBA_OK;
}
