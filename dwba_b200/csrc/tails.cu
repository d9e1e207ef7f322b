// Outer tails of the direct integral on the GPU: one warp per (pair, L), lanes over segments.
//
// Same quantity and formulas as the host path (host.cpp, dwba_outer_tails), which follows
// oscillatory_integrals.py: dwba_outer_integral_1d (:459-535) with
// compute_outer_integral_oscillatory (:1361-1451: Filon when |Phi''| h^2 < 0.1, else Levin),
// _filon_segment_complex (:1165-1277), _levin_segment_complex (:1024-1095) and
// _analytical_multipole_tail (:2064-2184). The reference sums segment contributions with
// math.fsum; here each lane keeps a compensated sum and the warp adds the 32 partials.
// Pairs whose mid-interval frequency is below 1e-10 (the reference's adaptive-quadrature
// branch) are left to the host path: the caller routes them there.
#include "common.cuh"

namespace {

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx cscale(double s, cplx a) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ cplx cexpi(double phi) {
  double s, c;
  sincos(phi, &s, &c);
  return {c, s};
}

struct WaveD {
  double k, delta, eta, sigma;
  int l;
};

struct PhaseD {
  WaveD a, b;
  int sgn;
  double kk, cc;
  __device__ PhaseD(const WaveD& wa, const WaveD& wb, int s) : a(wa), b(wb), sgn(s) {
    const double ca = -a.l * M_PI / 2 + a.sigma + a.delta;
    const double cb = -b.l * M_PI / 2 + b.sigma + b.delta;
    kk = s < 0 ? a.k - b.k : a.k + b.k;
    cc = s < 0 ? ca - cb : ca + cb;
  }
  __device__ double phi(double r) const {
    double v = kk * r + cc;
    if (fabs(a.eta) > 1e-15) v += a.eta * log(2 * a.k * r + 1e-30);
    if (fabs(b.eta) > 1e-15) {
      const double t = b.eta * log(2 * b.k * r + 1e-30);
      v = sgn < 0 ? v - t : v + t;
    }
    if (a.l > 0) v -= (a.l * (a.l + 1)) / (2.0 * a.k * r);
    if (b.l > 0) {
      const double t = (b.l * (b.l + 1)) / (2.0 * b.k * r);
      v = sgn < 0 ? v + t : v - t;
    }
    return v;
  }
  __device__ double d1(double r) const {
    double v = kk;
    if (fabs(a.eta) > 1e-15) v += a.eta / r;
    if (fabs(b.eta) > 1e-15) v = sgn < 0 ? v - b.eta / r : v + b.eta / r;
    if (a.l > 0) v += (a.l * (a.l + 1)) / (2.0 * a.k * (r * r));
    if (b.l > 0) {
      const double t = (b.l * (b.l + 1)) / (2.0 * b.k * (r * r));
      v = sgn < 0 ? v - t : v + t;
    }
    return v;
  }
  __device__ double d2(double r) const {
    double v = 0.0;
    if (fabs(a.eta) > 1e-15) v -= a.eta / (r * r);
    if (fabs(b.eta) > 1e-15) v = sgn < 0 ? v + b.eta / (r * r) : v - b.eta / (r * r);
    if (a.l > 0) v -= (a.l * (a.l + 1)) / (a.k * pow(r, 3.0));
    if (b.l > 0) {
      const double t = (b.l * (b.l + 1)) / (b.k * pow(r, 3.0));
      v = sgn < 0 ? v + t : v - t;
    }
    return v;
  }
};

__device__ __forceinline__ double envelope(double m, int L, double r) { return r > 1e-6 ? m / pow(r, (double)(L + 1)) : 0.0; }

// numpy.linspace(a, b, n)[i]
__device__ __forceinline__ double lin(double a, double b, int n, int i) {
  if (i == n - 1) return b;
  return (double)i * ((b - a) / (double)(n - 1)) + a;
}

// compensated lane sum
struct KSum {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
};

// Filon on one segment with nn equally spaced nodes (nn odd), _filon_segment_complex
__device__ cplx filon_segment(double m, int L, double a, double b, int nn, double omega, double off) {
  cplx res = {0.0, 0.0};
  if (!(b - a >= 1e-15)) return res;
  double xs[15], fs[15];
  for (int i = 0; i < nn; ++i) {
    xs[i] = lin(a, b, nn, i);
    fs[i] = envelope(m, L, xs[i]);
  }
  if (fabs(omega * (b - a)) < 1e-3) {  // scipy simpson with possibly unequal spacing
    double acc = 0.0;
    for (int i = 0; i + 2 < nn; i += 2) {
      const double h0 = xs[i + 1] - xs[i], h1 = xs[i + 2] - xs[i + 1];
      const double hs = h0 + h1, hp = h0 * h1, q = h0 / h1;
      acc += hs / 6.0 * (fs[i] * (2.0 - 1.0 / q) + fs[i + 1] * (hs * (hs / hp)) + fs[i + 2] * (2.0 - q));
    }
    return cscale(acc, cexpi(omega * (a + b) / 2 + off));
  }
  for (int i = 0; i + 2 < nn; i += 2) {
    const double x0 = xs[i], x1 = xs[i + 1], x2 = xs[i + 2];
    const double h = x2 - x0;
    if (h < 1e-15) continue;
    if (fabs(omega * h) < 1e-3) {  // the 3-node panel itself is non-oscillatory: Simpson times the mid phase
      const double h0 = x1 - x0, h1 = x2 - x1;
      const double hs = h0 + h1, hp = h0 * h1, q = h0 / h1;
      const double v = hs / 6.0 * (fs[i] * (2.0 - 1.0 / q) + fs[i + 1] * (hs * (hs / hp)) + fs[i + 2] * (2.0 - q));
      res = cadd(res, cscale(v, cexpi(omega * (x0 + x2) / 2 + off)));
      continue;
    }
    const double th = omega * h / 2;
    double st, ct;
    sincos(th, &st, &ct);
    double al, be, ga;
    if (fabs(th) < 0.3) {
      const double t2 = th * th, t3 = pow(th, 3.0);
      al = 2 * t3 / 45 * (1 - t2 / 7 + (t2 * t2) / 189);
      be = 2.0 / 3 + 2 * t2 / 15 - 4 * (t2 * t2) / 105 + 2 * pow(t2, 3.0) / 567;
      ga = 4.0 / 3 - 2 * t2 / 15 + 1 * (t2 * t2) / 210 - pow(t2, 3.0) / 11340;
    } else {
      const double t2 = th * th, t3 = pow(th, 3.0);
      double s2, c2;
      sincos(2 * th, &s2, &c2);
      al = (t2 + th * s2 / 2 - 2 * (st * st)) / t3;
      be = 2 * (th * (1 + c2) - s2) / t3;
      ga = 4 * (st - th * ct) / t3;
    }
    const cplx e0 = cexpi(omega * x0 + off), e1 = cexpi(omega * x1 + off), e2 = cexpi(omega * x2 + off);
    const cplx mi = {0.0, -1.0 / omega};
    const cplx d02 = csub(cscale(fs[i + 2], e2), cscale(fs[i], e0));
    const cplx s02 = cadd(cscale(fs[i], e0), cscale(fs[i + 2], e2));
    cplx t = cadd(cmul(cscale(al, mi), d02), cadd(cscale(be, s02), cscale(ga * fs[i + 1], e1)));
    res = cadd(res, cscale(h / 2, t));
  }
  return res;
}

struct LevinD {
  double D[8][8];  // Chebyshev differentiation matrix of descending Lobatto points (reference convention)
  double xr[8];    // ascending reference nodes in [-1, 1]
};

// Levin collocation on one segment, _levin_segment_complex (8 nodes)
__device__ cplx levin_segment(double m, int L, const PhaseD& ph, double a, double b, const LevinD& lv) {
  cplx A[8][8], u[8];
  double x[8];
  for (int k = 0; k < 8; ++k) x[k] = 0.5 * (b - a) * (lv.xr[k] + 1) + a;
  const double h = x[7] - x[0];
  if (h < 1e-15) return {0.0, 0.0};
  const double sc = 2.0 / h;
  for (int i = 0; i < 8; ++i) {
    for (int j = 0; j < 8; ++j) A[i][j] = {lv.D[i][j] * sc, 0.0};
    A[i][i].im += ph.d1(x[i]);
    u[i] = {envelope(m, L, x[i]), 0.0};
  }
  for (int k = 0; k < 8; ++k) {  // partial pivoting by |re| + |im|
    int piv = k;
    double best = -1.0;
    for (int i = k; i < 8; ++i) {
      const double mm = fabs(A[i][k].re) + fabs(A[i][k].im);
      if (mm > best) { best = mm; piv = i; }
    }
    if (best == 0.0) return {0.0, 0.0};
    if (piv != k) {
      for (int j = 0; j < 8; ++j) { cplx t = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = t; }
      cplx t = u[k]; u[k] = u[piv]; u[piv] = t;
    }
    const cplx inv = cdiv({1.0, 0.0}, A[k][k]);
    for (int i = k + 1; i < 8; ++i) {
      const cplx l = cmul(A[i][k], inv);
      for (int j = k + 1; j < 8; ++j) A[i][j] = csub(A[i][j], cmul(l, A[k][j]));
      u[i] = csub(u[i], cmul(l, u[k]));
    }
  }
  for (int i = 7; i >= 0; --i) {
    cplx s = u[i];
    for (int j = i + 1; j < 8; ++j) s = csub(s, cmul(A[i][j], u[j]));
    u[i] = cdiv(s, A[i][i]);
  }
  return csub(cmul(u[7], cexpi(ph.phi(x[7]))), cmul(u[0], cexpi(ph.phi(x[0]))));
}

__device__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return __shfl_sync(0xffffffffu, v, 0);
}

// one branch (cos(Phi_a -/+ Phi_b)) of the outer integral; Re part, summed over the warp
__device__ double outer_branch(double m, int L, const PhaseD& ph, double rm, double rmax, int max_seg,
                               double max_dphi, const LevinD& lv, int lane) {
  const double delta_phi = M_PI / 4;
  const double om = fabs(ph.d1((rm + rmax) / 2));
  const double h = delta_phi / om;
  const double lin_t = fabs(ph.d2((rm + rmax) / 2)) * h * h;
  KSum re;
  if (lin_t < 0.1) {
    const double off = ph.phi(rm) - om * rm;
    const double dr = delta_phi / om;
    const long long nraw = max(1LL, (long long)ceil((rmax - rm) / dr));
    const int nseg = (int)min(nraw, (long long)max_seg);
    const double eff = om * (rmax - rm) / max(1, nseg);
    int nn = 5;
    if (eff > max_dphi) {
      const int scl = (int)ceil(eff / max_dphi);
      nn = min(15, max(5, 5 + 2 * (scl - 1)));
    }
    for (int s = lane; s < nseg; s += 32) {
      const double a = lin(rm, rmax, nseg + 1, s), b = lin(rm, rmax, nseg + 1, s + 1);
      re.add(filon_segment(m, L, a, b, nn, om, off).re);
    }
  } else {
    const int nseg = (int)max(1.0, ceil((rmax - rm) / h));
    for (int s = lane; s < nseg; s += 32) {
      const double a = lin(rm, rmax, nseg + 1, s), b = lin(rm, rmax, nseg + 1, s + 1);
      re.add(levin_segment(m, L, ph, a, b, lv).re);
    }
  }
  return warp_sum(re.s + re.c);
}

__device__ double analytical_tail(double r_m, const WaveD& wi, const WaveD& wf, int L, double overlap) {
  if (r_m < 1e-3 || fabs(overlap) < 1e-12) return 0.0;
  const double lti = fabs(wi.eta) > 1e-10 ? wi.eta * log(2 * wi.k * r_m + 1e-30) : 0.0;
  const double ltf = fabs(wf.eta) > 1e-10 ? wf.eta * log(2 * wf.k * r_m + 1e-30) : 0.0;
  const double ci = -wi.l * M_PI / 2 + wi.sigma + wi.delta + lti;
  const double cf = -wf.l * M_PI / 2 + wf.sigma + wf.delta + ltf;
  const double kd = wi.k - wf.k, ks = wi.k + wf.k;
  const int n = L + 1;
  double t = 0.0;
  const double pd = kd * r_m + ci - cf;
  if (fabs(kd) > 1e-6) {
    t += 0.5 * (sin(pd) / (kd * pow(r_m, (double)n)) + n * cos(pd) / ((kd * kd) * pow(r_m, (double)(n + 1))));
  } else if (n > 1) {
    t += 0.5 * cos(pd) / ((n - 1) * pow(r_m, (double)(n - 1)));
  }
  const double ps = ks * r_m + ci + cf;
  if (ks > 1e-6) t -= 0.5 * (sin(ps) / (ks * pow(r_m, (double)n)) + n * cos(ps) / ((ks * ks) * pow(r_m, (double)(n + 1))));
  if (!isfinite(t)) return 0.0;
  return t * overlap;
}

__global__ void tails_kernel(const dwba_tail_t* __restrict__ recs, int n, int L_max, int max_seg, double max_dphi,
                             LevinD lv) {
  const int lane = threadIdx.x & 31;
  const int64_t warp_g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t n_items = (int64_t)n * L_max;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t it = warp_g; it < n_items; it += stride) {
    const int rec = (int)(it / L_max);
    const int L = (int)(it - (int64_t)rec * L_max) + 1;
    const dwba_tail_t R = recs[rec];
    const WaveD wi = {R.wave[0], R.wave[2], R.wave[3], R.wave[4], (int)R.wave[1]};
    const WaveD wf = {R.wave[5], R.wave[7], R.wave[8], R.wave[9], (int)R.wave[6]};
    const double m = R.moments_dev[L];
    double t = 0.0;
    if (fabs(m) > 1e-12) {
      if (R.mode == 1) {
        t = analytical_tail(R.r_m, wi, wf, L, m);
      } else {
        if (!(R.r_max <= R.r_m + 1e-10)) {
          const double im = outer_branch(m, L, PhaseD(wi, wf, -1), R.r_m, R.r_max, max_seg, max_dphi, lv, lane);
          const double ip = outer_branch(m, L, PhaseD(wi, wf, +1), R.r_m, R.r_max, max_seg, max_dphi, lv, lane);
          t = 0.5 * (im - ip);
        }
        t += analytical_tail(R.r_max, wi, wf, L, m);
      }
    }
    if (lane == 0) {
      R.out_dev[L] = t;
      if (L == 1) R.out_dev[0] = 0.0;
    }
  }
}

}  // namespace

extern "C" int dwba_outer_tails_batch(const dwba_tail_t* tails_dev, int n, int L_max, int max_filon_segments,
                                      double max_effective_dphi, dwba_stream_t stream) {
  if (n <= 0 || L_max < 1) return DWBA_OK;
  if (!tails_dev || L_max > DWBA_MAX_L || max_filon_segments < 1 || !(max_effective_dphi > 0.0))
    return DWBA_ERR_INVALID_ARG;
  // Chebyshev differentiation matrix (descending Lobatto points) and ascending nodes, n = 8
  LevinD lv;
  double x[8], c[8];
  for (int i = 0; i < 8; ++i) {
    x[i] = cos(M_PI * i / 7);
    c[i] = (i == 0 || i == 7) ? 2.0 : 1.0;
  }
  for (int i = 0; i < 8; ++i) {
    double rs = 0.0;
    for (int j = 0; j < 8; ++j) {
      if (i == j) continue;
      const double sgn = ((i + j) % 2 == 0) ? 1.0 : -1.0;
      lv.D[i][j] = (c[i] / c[j]) * sgn / (x[i] - x[j]);
      rs += lv.D[i][j];
    }
    lv.D[i][i] = -rs;
  }
  for (int k = 0; k < 8; ++k) lv.xr[k] = cos(M_PI * (7 - k) / 7);
  const int64_t warps = (int64_t)n * L_max;
  const int blocks = dwba_grid_1d(warps * 32, 128, 65535);
  tails_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>(tails_dev, n, L_max, max_filon_segments, max_effective_dphi,
                                                         lv);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
