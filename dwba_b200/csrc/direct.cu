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
// CTAs stride over chunks of PCH rows of one potential (grid.y = potential; grid.x sized so that
// even a handful of potentials fill the GPU). For each chunk a CTA first sums the prefix series b r^L over the columns before its
// chunk and the suffix series b r^-(L+1) over the columns after it (every CTA re-reads the
// potential's columns from L2: O(M) loads per CTA, no scratch and no inter-CTA waits), then scans
// its own chunk: each thread holds PPT consecutive points, the threads' sums are combined by warp
// scans and a scan of the warp totals, and every row gets
//     phi_L(p) = r_p^-(L+1) (prefix before p) + r_p^L (suffix after p) + d_L b_p / r_p.
constexpr int PT = 256;            // threads per CTA
constexpr int PPT = 4;             // consecutive points per thread
constexpr int PCH = PT * PPT;      // rows per CTA
constexpr int P_NL = 12;           // multipoles per launch

__device__ __forceinline__ double load_or_zero(const double* p, int i, int n) { return i < n ? p[i] : 0.0; }

template <int NL>
__global__ void __launch_bounds__(PT)
potential_kernel(const dwba_potential_t* __restrict__ pots, int L0, DiagScale ds) {
  __shared__ double wsum[2][PT / 32][NL];
  __shared__ double outer[2][NL];
  const dwba_potential_t D = pots[blockIdx.y];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ncol = D.n_cols;
  for (int c0 = blockIdx.x * PCH; c0 < D.n_rows; c0 += gridDim.x * PCH) {  // uniform over the CTA
  const int c1 = min(D.n_rows, c0 + PCH);
  __syncthreads();  // wsum / outer of the previous chunk are consumed
  // 1. the series over the columns outside the chunk: prefix over [0, c0), suffix over [c1, ncol)
  double pre[NL], suf[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) pre[l] = suf[l] = 0.0;
  const int c0c = min(c0, ncol);
  for (int q = tid; q < c0c; q += PT) {
    const double Y = D.b_dev[q], r = D.r_dev[q];
    double pw = Y * (L0 > 0 ? ipow(r, L0) : 1.0);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      pre[l] += pw;
      pw *= r;
    }
  }
  for (int q = c1 + tid; q < ncol; q += PT) {
    const double Y = D.b_dev[q], inv = 1.0 / D.r_dev[q];
    double ip = Y * (L0 > 0 ? ipow(inv, L0 + 1) : inv);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      suf[l] += ip;
      ip *= inv;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double a = pre[l], b = suf[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, off);
      b += __shfl_down_sync(0xffffffffu, b, off);
    }
    if (lane == 0) {
      wsum[0][warp][l] = a;
      wsum[1][warp][l] = b;
    }
  }
  __syncthreads();
  if (tid < 2 * NL) {
    const int k = tid / NL, l = tid - k * NL;
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < PT / 32; ++w) v += wsum[k][w][l];
    outer[k][l] = v;
  }
  __syncthreads();
  // 2. the chunk: this thread's points p0 .. p0+PPT-1
  const int p0 = c0 + tid * PPT;
  double Yv[PPT], rv[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = p0 + k;
    Yv[k] = p < c1 ? load_or_zero(D.b_dev, p, ncol) : 0.0;
    rv[k] = p < c1 ? D.r_dev[p] : 1.0;
  }
  double tp[NL], ts[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) tp[l] = ts[l] = 0.0;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const double r = rv[k], inv = 1.0 / r;
    double pw = Yv[k] * (L0 > 0 ? ipow(r, L0) : 1.0);
    double ip = Yv[k] * (L0 > 0 ? ipow(inv, L0 + 1) : inv);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      tp[l] += pw;
      ts[l] += ip;
      pw *= r;
      ip *= inv;
    }
  }
  // exclusive prefix of tp over the threads before this one, exclusive suffix of ts over the threads after
  __syncthreads();  // wsum is reused
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double a = tp[l], b = ts[l];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double ua = __shfl_up_sync(0xffffffffu, a, off);
      const double db = __shfl_down_sync(0xffffffffu, b, off);
      if (lane >= off) a += ua;
      if (lane + off < 32) b += db;
    }
    if (lane == 31) wsum[0][warp][l] = a;  // warp totals
    if (lane == 0) wsum[1][warp][l] = b;
    tp[l] = a - tp[l];  // exclusive within the warp
    ts[l] = b - ts[l];
  }
  __syncthreads();
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double a = outer[0][l], b = outer[1][l];
    for (int w = 0; w < warp; ++w) a += wsum[0][w][l];
    for (int w = warp + 1; w < PT / 32; ++w) b += wsum[1][w][l];
    tp[l] += a;
    ts[l] += b;
  }
  // 3. rows: forward over the thread's points for the prefix part and the diagonal, then backward
  // for the suffix part (each thread writes only its own rows)
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = p0 + k;
    const double r = rv[k], inv = 1.0 / r;
    double pw = Yv[k] * (L0 > 0 ? ipow(r, L0) : 1.0);
    double ip = L0 > 0 ? ipow(inv, L0 + 1) : inv;
    const double yd = Yv[k] * inv;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (p < c1) D.phi_dev[(int64_t)(L0 + l) * D.stride + p] = ip * tp[l] + yd * ds.v[L0 + l];
      tp[l] += pw;
      pw *= r;
      ip *= inv;
    }
  }
#pragma unroll
  for (int k = PPT - 1; k >= 0; --k) {
    const int p = p0 + k;
    const double r = rv[k], inv = 1.0 / r;
    double pw = L0 > 0 ? ipow(r, L0) : 1.0;
    double ip = Yv[k] * (L0 > 0 ? ipow(inv, L0 + 1) : inv);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      if (p < c1) D.phi_dev[(int64_t)(L0 + l) * D.stride + p] += pw * ts[l];
      ts[l] += ip;
      pw *= r;
      ip *= inv;
    }
  }
  }
}

template <int NL>
int launch_pot(const dwba_potential_t* pots, int n, int L0, const DiagScale& ds, cudaStream_t st) {
  // about eight CTAs per SM over all potentials; each CTA loops over its potential's chunks.
  // grid.y (one potential each) is limited to 65535: larger batches go in several launches
  for (int s0 = 0; s0 < n; s0 += 65535) {
    const int m = (n - s0) < 65535 ? (n - s0) : 65535;
    const int per = (8 * 148 + m - 1) / m;
    dim3 grid(per < 1 ? 1 : (per > 64 ? 64 : per), m);
    potential_kernel<NL><<<grid, PT, 0, st>>>(pots + s0, L0, ds);
    DWBA_CHECK_LAUNCH();
  }
  return DWBA_OK;
}

int launch_pot_nl(int nl, const dwba_potential_t* pots, int n, int L0, const DiagScale& ds, cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch_pot<N>(pots, n, L0, ds, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
    DWBA_CASE(9) DWBA_CASE(10) DWBA_CASE(11) DWBA_CASE(12)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

// ---- dot forms --------------------------------------------------------------------------------
// A CTA takes DOT_PER_CTA consecutive descriptors that share one potential (the caller groups
// them and pads a group with empty descriptors, n_rows = 0). Tiles of the potential's rows
// (NL multipoles x DOT_TILE points) are staged in shared memory once for all of them, in two
// buffers: the loads of tile t+1 (potential and the descriptors' rows) are issued into registers
// before tile t is accumulated, so each tile costs one barrier and no exposed load latency. Warp
// w accumulates descriptors 2w and 2w+1 (each staged value serves two pairs), lanes stride over
// the tile's points, and the lanes' sums are added by shuffles in a fixed order.
constexpr int DOT_THREADS = 256;
constexpr int DOT_PER_CTA = 16;
constexpr int DOT_TILE = 128;
constexpr int DOT_NL = 16;
constexpr int DOT_RPL = DOT_TILE / 32;  // rows per lane and tile

template <int NL>
__global__ void __launch_bounds__(DOT_THREADS)
dot_kernel(const dwba_dot_t* __restrict__ dots, int n, int L0, int n_ltot) {
  constexpr int PER = (NL * DOT_TILE + DOT_THREADS - 1) / DOT_THREADS;  // staged values per thread
  __shared__ double sphi[2][NL * DOT_TILE];
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
  const int n_tiles = (rows + DOT_TILE - 1) / DOT_TILE;
  // the group's potential: the first descriptor's (every non-empty one of the group shares it)
  const dwba_dot_t G = dots[d0];
  double pf[PER], xa[DOT_RPL], xb[DOT_RPL];
  auto load_tile = [&](int i0) {
#pragma unroll
    for (int m = 0; m < PER; ++m) {
      const int k = tid + m * DOT_THREADS;
      const int l = k / DOT_TILE, i = i0 + (k - l * DOT_TILE);
      pf[m] = (k < NL * DOT_TILE && i < rows) ? G.phi_dev[(int64_t)(L0 + l) * G.stride + i] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < DOT_RPL; ++q) {
      const int i = i0 + q * 32 + lane;
      xa[q] = i < A.n_rows ? A.a_dev[i] : 0.0;
      xb[q] = i < B.n_rows ? B.a_dev[i] : 0.0;
    }
  };
  double acc_a[NL], acc_b[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) acc_a[l] = acc_b[l] = 0.0;
  if (n_tiles > 0) load_tile(0);
  for (int t = 0; t < n_tiles; ++t) {
    double* buf = sphi[t & 1];
#pragma unroll
    for (int m = 0; m < PER; ++m) {
      const int k = tid + m * DOT_THREADS;
      if (k < NL * DOT_TILE) buf[k] = pf[m];
    }
    double ca[DOT_RPL], cb[DOT_RPL];
#pragma unroll
    for (int q = 0; q < DOT_RPL; ++q) {
      ca[q] = xa[q];
      cb[q] = xb[q];
    }
    // one barrier per tile: it publishes this buffer, and every thread passed the previous one
    // only after accumulating the tile that last used this buffer
    __syncthreads();
    if (t + 1 < n_tiles) load_tile((t + 1) * DOT_TILE);  // in flight during the accumulation
#pragma unroll
    for (int q = 0; q < DOT_RPL; ++q) {
      const int ii = q * 32 + lane;
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        const double ph = buf[l * DOT_TILE + ii];
        acc_a[l] = fma(ca[q], ph, acc_a[l]);
        acc_b[l] = fma(cb[q], ph, acc_b[l]);
      }
    }
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
