// Plain FP64 bilinear forms  I_L = a^T K_L b  with every kernel element
// generated in registers.
//
// Reference: the dense kernels K_L = (1/r_>) exp(L log(min(r_</r_>, 1-1e-12)))
// of dwba_matrix_elements.py:1057-1116 (CPU) and :1963-2002, :2324-2409 (CuPy),
// contracted by the gemv/dot pairs of oscillatory_integrals.py:2571, :2644,
// :2745-2770 and dwba_matrix_elements.py:1242-1245, :2350, :2474-2477.
//
// On a strictly increasing grid K_L is symmetric with K_L(p,q) = r_q^L / r_p^(L+1)
// for q < p, so with X = a (zero past n_rows), Y = b (zero past n_cols):
//   I_L = sum_{q<p} (X_p Y_q + X_q Y_p) r_q^L / r_p^(L+1) + sum_p X_p Y_p (1-1e-12)^L / r_p.
// Each element of the strict lower triangle is generated once:
//   t_0 = (X_p/r_p) Y_q + (Y_p/r_p) X_q,   t_L = t_{L-1} * (r_q / r_p).
// Work is tiled in 128x128 (p, q) tiles; a CTA owns row tiles P and T-1-P of one
// form (equal work per CTA), stages the q operands in shared memory, and reduces
// its per-thread sums with warp shuffles into one partial per (form, chunk, L);
// a second kernel adds the partials of each form in a fixed order.
#include "common.cuh"

namespace {

constexpr int TP = 128;       // tile edge (rows p and columns q)
constexpr int THREADS = 256;  // 64 row slots x 4 column groups
constexpr int NL_MAX = 16;    // multipoles per pass

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
__global__ void __launch_bounds__(THREADS, 2)
dense_tri_kernel(const dwba_form_t* __restrict__ forms, const int64_t* __restrict__ chunk_prefix, int n_forms,
                 int L0, int n_ltot, DiagScale ds, double* __restrict__ partials) {
  __shared__ double sx[TP], sy[TP], sr[TP];
  __shared__ double red[THREADS / 32][NL];

  // locate (form, chunk)
  const int64_t cta = blockIdx.x;
  int lo = 0, hi = n_forms;  // chunk_prefix[lo] <= cta < chunk_prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (chunk_prefix[mid] <= cta) lo = mid; else hi = mid;
  }
  const int fi = lo;
  const int chunk = (int)(cta - chunk_prefix[fi]);
  const dwba_form_t F = forms[fi];
  const int M = F.n_rows > F.n_cols ? F.n_rows : F.n_cols;
  const int T = (M + TP - 1) / TP;

  const int tid = threadIdx.x;
  const int rs = tid & 63;
  const int cg = tid >> 6;

  double tot[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) tot[l] = 0.0;

  for (int pass = 0; pass < 2; ++pass) {
    const int P = pass == 0 ? chunk : T - 1 - chunk;
    if (pass == 1 && P == chunk) break;
    // this thread's two rows
    double xi[2], yi[2], inv[2];
    int prow[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = P * TP + rs + 64 * h;
      prow[h] = p;
      const double X = (p < F.n_rows) ? F.a_dev[p] : 0.0;
      const double Y = (p < F.n_cols) ? F.b_dev[p] : 0.0;
      const double iv = (p < M) ? 1.0 / F.r_dev[p] : 0.0;
      xi[h] = X * iv;
      yi[h] = Y * iv;
      inv[h] = iv;
    }
    for (int Q = 0; Q <= P; ++Q) {
      __syncthreads();
      if (tid < TP) {
        const int q = Q * TP + tid;
        sx[tid] = (q < F.n_rows) ? F.a_dev[q] : 0.0;
        sy[tid] = (q < F.n_cols) ? F.b_dev[q] : 0.0;
        sr[tid] = (q < M) ? F.r_dev[q] : 0.0;
      }
      __syncthreads();
      double acc[NL];
#pragma unroll
      for (int l = 0; l < NL; ++l) acc[l] = 0.0;
      if (Q < P) {
#pragma unroll 2
        for (int k = cg; k < TP; k += 4) {
          const double xq = sx[k], yq = sy[k], rq = sr[k];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const double ratio = rq * inv[h];
            double t = fma(xi[h], yq, yi[h] * xq);
            if (L0 > 0) t *= ipow(ratio, L0);
            acc[0] += t;
#pragma unroll
            for (int l = 1; l < NL; ++l) {
              t *= ratio;
              acc[l] += t;
            }
          }
        }
      } else {
        for (int k = cg; k < TP; k += 4) {
          const double xq = sx[k], yq = sy[k], rq = sr[k];
          const int q = Q * TP + k;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            if (q < prow[h]) {
              const double ratio = rq * inv[h];
              double t = fma(xi[h], yq, yi[h] * xq);
              if (L0 > 0) t *= ipow(ratio, L0);
              acc[0] += t;
#pragma unroll
              for (int l = 1; l < NL; ++l) {
                t *= ratio;
                acc[l] += t;
              }
            }
          }
        }
        if (cg == 0) {  // diagonal elements, (1-1e-12)^L / r_p as the reference's clamp gives
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const double d = (prow[h] < M) ? xi[h] * yi[h] / inv[h] : 0.0;  // X Y / r
#pragma unroll
            for (int l = 0; l < NL; ++l) acc[l] += d * ds.v[L0 + l];
          }
        }
      }
#pragma unroll
      for (int l = 0; l < NL; ++l) tot[l] += acc[l];
    }
  }
  // CTA reduction: shuffles within warps, then across the 8 warps in a fixed order
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    double v = tot[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][l] = v;
  }
  __syncthreads();
  if (tid < NL) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < THREADS / 32; ++w) s += red[w][tid];
    partials[cta * n_ltot + L0 + tid] = s;
  }
}

__global__ void reduce_partials_kernel(const int64_t* __restrict__ chunk_prefix, int n_forms, int n_ltot,
                                       const double* __restrict__ partials, double* __restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_forms * n_ltot) return;
  const int f = (int)(idx / n_ltot), l = (int)(idx - (int64_t)f * n_ltot);
  double s = 0.0;
  for (int64_t c = chunk_prefix[f]; c < chunk_prefix[f + 1]; ++c) s += partials[c * n_ltot + l];
  out[idx] = s;
}

template <int NL>
int launch_dense(const dwba_form_t* forms, const int64_t* prefix, int n_forms, int L0, int n_ltot,
                 const DiagScale& ds, double* partials, int64_t n_cta, cudaStream_t st) {
  dense_tri_kernel<NL><<<(unsigned)n_cta, THREADS, 0, st>>>(forms, prefix, n_forms, L0, n_ltot, ds, partials);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

int launch_dense_nl(int nl, const dwba_form_t* forms, const int64_t* prefix, int n_forms, int L0, int n_ltot,
                    const DiagScale& ds, double* partials, int64_t n_cta, cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch_dense<N>(forms, prefix, n_forms, L0, n_ltot, ds, partials, n_cta, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
    DWBA_CASE(9) DWBA_CASE(10) DWBA_CASE(11) DWBA_CASE(12) DWBA_CASE(13) DWBA_CASE(14) DWBA_CASE(15)
    DWBA_CASE(16)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

}  // namespace

static inline int64_t dense_chunks(int m) {
  const int64_t T = (m + TP - 1) / TP;
  return (T + 1) / 2;
}

extern "C" int64_t dwba_dense_chunk_prefix(const int32_t* m_host, int n_forms, int64_t* prefix_host) {
  if (!m_host || !prefix_host || n_forms < 0) return -1;
  prefix_host[0] = 0;
  for (int f = 0; f < n_forms; ++f) {
    if (m_host[f] < 1) return -1;
    prefix_host[f + 1] = prefix_host[f] + dense_chunks(m_host[f]);
  }
  return prefix_host[n_forms];
}

extern "C" int dwba_bilinear_dense_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max,
                                        const double* diag_scale_host, const int64_t* chunk_prefix_dev,
                                        int64_t n_cta, double* partial_dev, int64_t partial_cap, double* out_dev,
                                        dwba_stream_t stream) {
  if (n_forms <= 0) return DWBA_OK;
  if (!forms_dev || !diag_scale_host || !chunk_prefix_dev || !partial_dev || !out_dev || L_max < 0 ||
      L_max > DWBA_MAX_L || n_cta < 1 || n_cta > 0x7fffffffLL)
    return DWBA_ERR_INVALID_ARG;
  const int n_ltot = L_max + 1;
  if (n_cta * n_ltot > partial_cap) return DWBA_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  DiagScale ds;
  for (int l = 0; l <= DWBA_MAX_L; ++l) ds.v[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  for (int L0 = 0; L0 < n_ltot; L0 += NL_MAX) {
    const int nl = (n_ltot - L0) < NL_MAX ? (n_ltot - L0) : NL_MAX;
    int rc = launch_dense_nl(nl, forms_dev, chunk_prefix_dev, n_forms, L0, n_ltot, ds, partial_dev, n_cta, st);
    if (rc != DWBA_OK) return rc;
  }
  const int64_t n_out = (int64_t)n_forms * n_ltot;
  reduce_partials_kernel<<<dwba_grid_1d(n_out, 256), 256, 0, st>>>(chunk_prefix_dev, n_forms, n_ltot, partial_dev,
                                                                  out_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
