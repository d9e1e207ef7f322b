// Allocation-free variant of the dense FP64 bilinear forms.
//
// Some callers cannot hand this library a scratch buffer: their device memory
// belongs to another allocator (a framework's caching pool or a pool sized once
// at start-up), or their inner loop must not call cudaMalloc/cudaFree, which
// synchronise the device. dwba_bilinear_dense_fp64_noalloc serves them: it
// computes the same forms as dwba_bilinear_dense_fp64 with the same tiling and
// summation order, but keeps its per-chunk partial sums in a fixed array that
// lives in this library's device memory for the life of the process. The caller
// passes only the inputs (descriptors, grids, operands) and the output.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int TP = 128;
constexpr int THREADS = 256;
constexpr int NL_MAX = 16;

// Shared scratch: 2^20 doubles (8 MiB) of partial sums, held by every GPU that
// loads the library until the process exits. Every call overwrites the part it
// uses before reading it, so nothing needs clearing; two calls that overlap on
// the GPU (different streams, no ordering between them) race on this array.
static __device__ __align__(256) double g_noalloc_partials[DWBA_NOALLOC_SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
double* g_scratch[MAX_DEVICES] = {nullptr};
void* g_scratch_ctx[MAX_DEVICES] = {nullptr};

// The calling thread's current driver context (through the runtime's driver entry point, so
// the library needs no link against the driver library); nullptr if it cannot be read.
void* current_context() {
  using ctx_fn = int (*)(void**);
  static ctx_fn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<ctx_fn>(p);
    tried = true;
  }
  void* ctx = nullptr;
  if (fn == nullptr || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array on the current device, looked up once per device and
// context: a device reset (cudaDeviceReset) ends the context and reloads this module, so the
// address is looked up again in the new context.
int scratch_ptr(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return DWBA_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mutex);
  void* ctx = current_context();
  if (g_scratch[dev] == nullptr || ctx == nullptr || ctx != g_scratch_ctx[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return DWBA_ERR_CUDA;
    }
    g_scratch[dev] = static_cast<double*>(p);
    g_scratch_ctx[dev] = current_context();
  }
  *out = g_scratch[dev];
  return DWBA_OK;
}

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

__device__ __forceinline__ int chunks_of(int m) {
  const int T = (m + TP - 1) / TP;
  return (T + 1) / 2;
}

// Same tile walk as dense_tri_kernel (dense_fp64.cu); the (form, chunk) pair comes
// from a 2-D grid instead of a prefix search, and partials go to the fixed array.
template <int NL>
__global__ void __launch_bounds__(THREADS, 2)
noalloc_tri_kernel(const dwba_form_t* __restrict__ forms, int max_chunks, int L0, int n_ltot, DiagScale ds,
                   double* __restrict__ partials) {
  __shared__ double sx[TP], sy[TP], sr[TP];
  __shared__ double red[THREADS / 32][NL];
  const int fi = blockIdx.y;
  const int chunk = blockIdx.x;
  const dwba_form_t F = forms[fi];
  const int M = F.n_rows > F.n_cols ? F.n_rows : F.n_cols;
  if (M < 1 || chunk >= chunks_of(M) || chunk >= max_chunks) return;
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
        if (cg == 0) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const double d = (prow[h] < M) ? xi[h] * yi[h] / inv[h] : 0.0;
#pragma unroll
            for (int l = 0; l < NL; ++l) acc[l] += d * ds.v[L0 + l];
          }
        }
      }
#pragma unroll
      for (int l = 0; l < NL; ++l) tot[l] += acc[l];
    }
  }
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
    partials[((int64_t)fi * max_chunks + chunk) * n_ltot + L0 + tid] = s;
  }
}

// Adds each form's partials in chunk order; a form larger than max_m gets NaN, an empty form
// (no rows and no columns) the empty sum 0.
__global__ void noalloc_reduce_kernel(const dwba_form_t* __restrict__ forms, int n_forms, int max_chunks, int n_ltot,
                                      const double* __restrict__ partials, double* __restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_forms * n_ltot) return;
  const int f = (int)(idx / n_ltot), l = (int)(idx - (int64_t)f * n_ltot);
  const dwba_form_t F = forms[f];
  const int M = F.n_rows > F.n_cols ? F.n_rows : F.n_cols;
  if (M < 1) {
    out[idx] = 0.0;
    return;
  }
  const int nc = chunks_of(M);
  if (nc > max_chunks) {
    out[idx] = __longlong_as_double(0x7ff8000000000000LL);
    return;
  }
  double s = 0.0;
  for (int c = 0; c < nc; ++c) s += partials[((int64_t)f * max_chunks + c) * n_ltot + l];
  out[idx] = s;
}

template <int NL>
int launch_nl_t(const dwba_form_t* forms, int n_forms, int max_chunks, int L0, int n_ltot, const DiagScale& ds,
                double* partials, cudaStream_t st) {
  dim3 grid(max_chunks, n_forms);
  noalloc_tri_kernel<NL><<<grid, THREADS, 0, st>>>(forms, max_chunks, L0, n_ltot, ds, partials);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

int launch_nl(int nl, const dwba_form_t* forms, int n_forms, int max_chunks, int L0, int n_ltot, const DiagScale& ds,
              double* partials, cudaStream_t st) {
  switch (nl) {
#define DWBA_CASE(N) \
  case N: return launch_nl_t<N>(forms, n_forms, max_chunks, L0, n_ltot, ds, partials, st);
    DWBA_CASE(1) DWBA_CASE(2) DWBA_CASE(3) DWBA_CASE(4) DWBA_CASE(5) DWBA_CASE(6) DWBA_CASE(7) DWBA_CASE(8)
    DWBA_CASE(9) DWBA_CASE(10) DWBA_CASE(11) DWBA_CASE(12) DWBA_CASE(13) DWBA_CASE(14) DWBA_CASE(15)
    DWBA_CASE(16)
#undef DWBA_CASE
    default: return DWBA_ERR_INVALID_ARG;
  }
}

}  // namespace

extern "C" int dwba_bilinear_dense_fp64_noalloc(const dwba_form_t* forms_dev, int n_forms, int max_m, int L_max,
                                                const double* diag_scale_host, double* out_dev,
                                                dwba_stream_t stream) {
  if (n_forms <= 0) return DWBA_OK;
  if (!forms_dev || !diag_scale_host || !out_dev || L_max < 0 || L_max > DWBA_MAX_L || max_m < 1 ||
      n_forms > 65535)
    return DWBA_ERR_INVALID_ARG;
  const int n_ltot = L_max + 1;
  const int max_chunks = ((max_m + TP - 1) / TP + 1) / 2;
  if ((int64_t)n_forms * max_chunks * n_ltot > (int64_t)DWBA_NOALLOC_SCRATCH_DOUBLES) return DWBA_ERR_WORKSPACE;
  double* partials = nullptr;
  int rc = scratch_ptr(&partials);
  if (rc != DWBA_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  DiagScale ds;
  for (int l = 0; l <= DWBA_MAX_L; ++l) ds.v[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  for (int L0 = 0; L0 < n_ltot; L0 += NL_MAX) {
    const int nl = (n_ltot - L0) < NL_MAX ? (n_ltot - L0) : NL_MAX;
    rc = launch_nl(nl, forms_dev, n_forms, max_chunks, L0, n_ltot, ds, partials, st);
    if (rc != DWBA_OK) return rc;
  }
  const int64_t n_out = (int64_t)n_forms * n_ltot;
  noalloc_reduce_kernel<<<dwba_grid_1d(n_out, 256), 256, 0, st>>>(forms_dev, n_forms, max_chunks, n_ltot, partials,
                                                                  out_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
