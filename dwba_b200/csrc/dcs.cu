// Amplitudes, DCS and TCS from the radial integrals of many partial-wave channels.
//
// Per target sublevel pair a and channel p the amplitudes are linear in the integrals with one
// spherical harmonic of l_f as angular factor (dwba_coupling.py:285-505):
//   f_a(theta) = sum_p yd[a][p](theta) sum_L cf[a][p][L] I_dir[p][L]
//   g_a(theta) = sum_p ye[a][p](theta) sum_L cg[a][p][L] I_exc[p][L]
// and DCS(theta) = pref sum_a [1/4 |f_a + g_a|^2 + 3/4 |f_a - g_a|^2], clipped at 0
// (sigma_total.py:147-177); TCS = 2 pi trapz(sin(theta) DCS, theta) (sigma_total.py:179-217).
// One thread per angle; the channel sums run in ascending p, the trapezoid in a fixed tree.
#include "common.cuh"

namespace {

__global__ void dcs_kernel(const double2* __restrict__ cf, const double2* __restrict__ cg,
                           const double* __restrict__ yd, const double* __restrict__ ye,
                           const double* __restrict__ I_dir, const double* __restrict__ I_exc, int n_M, int P,
                           int nl, int n_theta, double pref, double* __restrict__ dcs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_theta) return;
  double acc = 0.0;
  for (int a = 0; a < n_M; ++a) {
    double fr = 0.0, fi = 0.0, gr = 0.0, gi = 0.0;
    for (int p = 0; p < P; ++p) {
      const double2* c1 = cf + ((int64_t)a * P + p) * nl;
      const double2* c2 = cg + ((int64_t)a * P + p) * nl;
      const double* d = I_dir + (int64_t)p * nl;
      const double* e = I_exc + (int64_t)p * nl;
      double sdr = 0.0, sdi = 0.0, ser = 0.0, sei = 0.0;
      for (int L = 0; L < nl; ++L) {
        sdr += c1[L].x * d[L];
        sdi += c1[L].y * d[L];
        ser += c2[L].x * e[L];
        sei += c2[L].y * e[L];
      }
      const double y1 = yd[((int64_t)a * P + p) * n_theta + t];
      const double y2 = ye[((int64_t)a * P + p) * n_theta + t];
      fr += y1 * sdr;
      fi += y1 * sdi;
      gr += y2 * ser;
      gi += y2 * sei;
    }
    const double sr = fr + gr, si = fi + gi, dr = fr - gr, di = fi - gi;
    acc += pref * (0.25 * (sr * sr + si * si) + 0.75 * (dr * dr + di * di));
  }
  dcs[t] = acc > 0.0 ? acc : 0.0;
}

// 2 pi sum of trapezoids of sin(theta) DCS, one block, fixed reduction tree
__global__ void tcs_kernel(const double* __restrict__ theta, const double* __restrict__ dcs, int n, double* tcs) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i + 1 < n; i += blockDim.x)
    s += 0.5 * (theta[i + 1] - theta[i]) * (sin(theta[i]) * dcs[i] + sin(theta[i + 1]) * dcs[i + 1]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *tcs = 2.0 * M_PI * red[0];
}

}  // namespace

extern "C" int dwba_cross_sections(const double* cf_dev, const double* cg_dev, const double* yd_dev,
                                   const double* ye_dev, const double* I_dir_dev, const double* I_exc_dev,
                                   const double* theta_dev, int n_M, int P, int nl, int n_theta, double pref,
                                   double* dcs_dev, double* tcs_dev, dwba_stream_t stream) {
  if (n_theta <= 0) return DWBA_OK;
  if (!cf_dev || !cg_dev || !yd_dev || !ye_dev || !I_dir_dev || !I_exc_dev || !theta_dev || !dcs_dev || n_M < 1 ||
      P < 0 || nl < 1 || nl > DWBA_MAX_L + 1)
    return DWBA_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  dcs_kernel<<<dwba_grid_1d(n_theta, 128), 128, 0, st>>>((const double2*)cf_dev, (const double2*)cg_dev, yd_dev,
                                                         ye_dev, I_dir_dev, I_exc_dev, n_M, P, nl, n_theta, pref,
                                                         dcs_dev);
  DWBA_CHECK_LAUNCH();
  if (tcs_dev) {
    tcs_kernel<<<1, 256, 0, st>>>(theta_dev, dcs_dev, n_theta, tcs_dev);
    DWBA_CHECK_LAUNCH();
  }
  return DWBA_OK;
}
