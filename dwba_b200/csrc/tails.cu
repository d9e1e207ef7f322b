// Outer tails of the direct integral on the GPU: one warp per (pair, chunk of up to 8 multipoles),
// lanes over segments; each node's phase factor, each Filon panel's weights and each Levin
// segment's factorised collocation system serve every multipole of the chunk.
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

struct LevinD {
  double D[8][8];  // Chebyshev differentiation matrix of descending Lobatto points (reference convention)
  double xr[8];    // ascending reference nodes in [-1, 1]
};

__shared__ LevinD s_lv;  // the launch's Levin tables, staged once per block

__device__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return __shfl_sync(0xffffffffu, v, 0);
}

constexpr int LC = 8;  // multipoles evaluated together (one accumulator each per lane)

// b^e for e >= 0 by repeated squaring
__device__ __forceinline__ double ipow(double b, int e) {
  double r = 1.0;
  while (e) {
    if (e & 1) r *= b;
    b *= b;
    e >>= 1;
  }
  return r;
}

// x^-(L0+1) for the envelopes f_L(x) = m_L x^-(L+1) of a chunk (0 where x <= 1e-6): the envelope of
// multipole L0 + q is m[q] p with p advanced by 1/x per multipole
struct EnvPow {
  double p0, inv;
  __device__ __forceinline__ EnvPow(double x, int L0) {
    const bool in = x > 1e-6;
    inv = in ? 1.0 / x : 0.0;
    p0 = in ? ipow(inv, L0 + 1) : 0.0;
  }
};

// Filon constants shared by every panel of one phase branch: the segments are equal (linspace) and
// so are their panels, so alpha, beta, gamma of the panel angle theta = omega h / 2 and the phase
// step between nodes, E = exp(i omega h / 2), are evaluated once per branch instead of per panel.
struct FilonConst {
  double al, be, ga;
  cplx E;
};

__device__ __forceinline__ FilonConst filon_const(double omega, double seg_w, int nn) {
  FilonConst c;
  const double h = 2.0 * seg_w / (nn - 1);  // panel width (two node spacings)
  const double th = omega * h / 2;
  double st, ct;
  sincos(th, &st, &ct);
  c.E = {ct, st};
  if (fabs(th) < 0.3) {
    const double t2 = th * th, t3 = t2 * th, t6 = t2 * t2 * t2;
    c.al = 2 * t3 / 45 * (1 - t2 / 7 + (t2 * t2) / 189);
    c.be = 2.0 / 3 + 2 * t2 / 15 - 4 * (t2 * t2) / 105 + 2 * t6 / 567;
    c.ga = 4.0 / 3 - 2 * t2 / 15 + 1 * (t2 * t2) / 210 - t6 / 11340;
  } else {
    const double t2 = th * th, t3 = t2 * th;
    double s2, c2;
    sincos(2 * th, &s2, &c2);
    c.al = (t2 + th * s2 / 2 - 2 * (st * st)) / t3;
    c.be = 2 * (th * (1 + c2) - s2) / t3;
    c.ga = 4 * (st - th * ct) / t3;
  }
  return c;
}

// Re of the Filon integral over one segment (nn equally spaced nodes, nn odd) for every multipole
// of the chunk: _filon_segment_complex with the node phases and the panel weights shared by all L.
// The first node's phase factor is evaluated directly, the next ones by the recurrence
// e_{j+1} = e_j E (nn - 1 <= 14 steps: a few ulps), and the panels use the branch's FilonConst.
// Envelope values are formed inside the multipole loops from one running power per node, so no
// per-node arrays of envelopes are kept.
__device__ __forceinline__ void filon_segment_all(const double* m, int L0, int nl, double a, double b, int nn, double omega,
                                  double off, const FilonConst& fc, KSum* acc) {
  if (!(b - a >= 1e-15)) return;
  if (fabs(omega * (b - a)) < 1e-3) {  // scipy simpson with possibly unequal spacing, times the mid phase
    const double ce = cexpi(omega * (a + b) / 2 + off).re;
    double part[LC];
#pragma unroll
    for (int q = 0; q < LC; ++q) part[q] = 0.0;
    for (int i = 0; i + 2 < nn; i += 2) {
      const double x0 = lin(a, b, nn, i), x1 = lin(a, b, nn, i + 1), x2 = lin(a, b, nn, i + 2);
      const double h0 = x1 - x0, h1 = x2 - x1;
      const double hs = h0 + h1, hp = h0 * h1, qq = h0 / h1;
      const EnvPow e0(x0, L0), e1(x1, L0), e2(x2, L0);
      double p0 = e0.p0, p1 = e1.p0, p2 = e2.p0;
#pragma unroll
      for (int q = 0; q < LC; ++q) {
        const double mq = q < nl ? m[q] : 0.0;
        part[q] += hs / 6.0 * ((mq * p0) * (2.0 - 1.0 / qq) + (mq * p1) * (hs * (hs / hp)) + (mq * p2) * (2.0 - qq));
        p0 *= e0.inv;
        p1 *= e1.inv;
        p2 *= e2.inv;
      }
    }
#pragma unroll
    for (int q = 0; q < LC; ++q) acc[q].add(part[q] * ce);
    return;
  }
  double seg[LC];
#pragma unroll
  for (int q = 0; q < LC; ++q) seg[q] = 0.0;
  double x0 = a;
  cplx e0 = cexpi(omega * x0 + off);
  EnvPow v0(x0, L0);
  const cplx mi = {0.0, -1.0 / omega};
  const cplx am = cscale(fc.al, mi);
  const cplx wl = csub(cplx{fc.be, 0.0}, am), wr = cadd(cplx{fc.be, 0.0}, am);
  for (int i = 0; i + 2 < nn; i += 2) {
    const double x1 = lin(a, b, nn, i + 1), x2 = lin(a, b, nn, i + 2);
    const double h = x2 - x0;
    const cplx e1 = cmul(e0, fc.E), e2 = cmul(e1, fc.E);
    const EnvPow v1(x1, L0), v2(x2, L0);
    if (h >= 1e-15) {
      double w0, w1, w2;
      if (fabs(omega * h) < 1e-3) {  // the 3-node panel itself is non-oscillatory: Simpson times the mid phase
        const double h0 = x1 - x0, h1 = x2 - x1;
        const double hs = h0 + h1, hp = h0 * h1, qq = h0 / h1;
        const double ce = cexpi(omega * (x0 + x2) / 2 + off).re;
        w0 = ce * (hs / 6.0) * (2.0 - 1.0 / qq);
        w1 = ce * (hs / 6.0) * (hs * (hs / hp));
        w2 = ce * (hs / 6.0) * (2.0 - qq);
      } else {
        // (h/2) [alpha (-i/omega) (f2 e2 - f0 e0) + beta (f0 e0 + f2 e2) + gamma f1 e1], real part,
        // as weights of f0, f1, f2 that every multipole shares
        w0 = (h / 2) * cmul(wl, e0).re;
        w1 = (h / 2) * (fc.ga * e1.re);
        w2 = (h / 2) * cmul(wr, e2).re;
      }
      double p0 = v0.p0, p1 = v1.p0, p2 = v2.p0;
#pragma unroll
      for (int q = 0; q < LC; ++q) {
        const double mq = q < nl ? m[q] : 0.0;
        seg[q] += w0 * (mq * p0) + w1 * (mq * p1) + w2 * (mq * p2);
        p0 *= v0.inv;
        p1 *= v1.inv;
        p2 *= v2.inv;
      }
    }
    x0 = x2;
    e0 = e2;
    v0 = v2;
  }
#pragma unroll
  for (int q = 0; q < LC; ++q) acc[q].add(seg[q]);
}

// Levin collocation on one segment (8 nodes) for every multipole of the chunk, solved by a group
// of 8 lanes: lane `row` of the group holds row `row` of the 8x8 complex collocation system in
// registers (compile-time column indices only, so nothing goes to local memory). The system does
// not depend on L: it is factorised once by Gaussian elimination with partial pivoting (largest
// |re| + |im| of the column among the rows not yet used; the pivot order is kept instead of
// swapping rows, and the pivot row is broadcast by shuffles) and solved for each envelope.
// All 32 lanes call it together (shuffles over groups of 8); `valid` = the group has a segment.
// res[q]: the segment's contribution to multipole L0 + q, the same on every lane of the group
// (zero for an invalid group or a singular system).
__device__ __noinline__ void levin_segment_group(const double* m, int L0, int nl, const PhaseD& ph, double a, double b,
                                                 bool valid, double* res) {
  const int row = threadIdx.x & 7;
  const LevinD& lv = s_lv;
  const double hw = 0.5 * (b - a);
  const double xi = hw * (lv.xr[row] + 1) + a;
  const double x0 = hw * (lv.xr[0] + 1) + a, x7 = hw * (lv.xr[7] + 1) + a;
  const double h = x7 - x0;
  bool ok = valid && !(h < 1e-15);
  const double sc = ok ? 2.0 / h : 0.0;
  const double d1 = ph.d1(xi);
  cplx A[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) A[j] = {lv.D[row][j] * sc, j == row ? d1 : 0.0};
  int step_of = 8;  // elimination step at which this row became the pivot
  int pv[8];        // pivot row of each step
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double mag = step_of < 8 ? -1.0 : fabs(A[k].re) + fabs(A[k].im);
    int who = row;
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) {  // group argmax, ties to the lower row
      const double om = __shfl_xor_sync(0xffffffffu, mag, off, 8);
      const int ow = __shfl_xor_sync(0xffffffffu, who, off, 8);
      if (om > mag || (om == mag && ow < who)) {
        mag = om;
        who = ow;
      }
    }
    pv[k] = who;
    if (!(mag > 0.0)) ok = false;  // singular (or an invalid group): the result is dropped
    cplx P[8];
#pragma unroll
    for (int j = k; j < 8; ++j) {
      P[j].re = __shfl_sync(0xffffffffu, A[j].re, who, 8);
      P[j].im = __shfl_sync(0xffffffffu, A[j].im, who, 8);
    }
    if (row == who) {
      step_of = k;
    } else if (step_of == 8) {
      const cplx inv = cdiv({1.0, 0.0}, P[k]);
      const cplx l = cmul(A[k], inv);
      A[k] = l;
#pragma unroll
      for (int j = k + 1; j < 8; ++j) A[j] = csub(A[j], cmul(l, P[j]));
    }
  }
  const cplx e7 = cexpi(ph.phi(x7)), e0 = cexpi(ph.phi(x0));
  const double inv_x = xi > 1e-6 ? 1.0 / xi : 0.0;
  double pw = xi > 1e-6 ? ipow(inv_x, L0 + 1) : 0.0;
#pragma unroll 1
  for (int q = 0; q < LC; ++q) {
    res[q] = 0.0;
    if (q >= nl) continue;  // warp-uniform
    cplx u = {m[q] * pw, 0.0};
    pw *= inv_x;
    // forward: rows that became pivots after step k take their multiplier of step k
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      cplx y;
      y.re = __shfl_sync(0xffffffffu, u.re, pv[k], 8);
      y.im = __shfl_sync(0xffffffffu, u.im, pv[k], 8);
      if (step_of > k) u = csub(u, cmul(A[k], y));
    }
    // backward: the pivot row of step k gives unknown k (node k); every lane keeps all unknowns
    cplx z[8];
#pragma unroll
    for (int k = 7; k >= 0; --k) {
      cplx t = u;
#pragma unroll
      for (int j = k + 1; j < 8; ++j) t = csub(t, cmul(A[j], z[j]));
      const cplx zk = cdiv(t, A[k]);
      z[k].re = __shfl_sync(0xffffffffu, zk.re, pv[k], 8);
      z[k].im = __shfl_sync(0xffffffffu, zk.im, pv[k], 8);
    }
    res[q] = ok ? csub(cmul(z[7], e7), cmul(z[0], e0)).re : 0.0;
  }
}

// one phase branch (cos(Phi_a -/+ Phi_b)) of the outer integral for a chunk of multipoles: Re part
// per multipole, summed over the warp into res[q]
__device__ __noinline__ void outer_branch_all(const double* m, int L0, int nl, const PhaseD& ph, double rm, double rmax,
                                 int max_seg, double max_dphi, int lane, double* res) {
  const double delta_phi = M_PI / 4;
  const double om = fabs(ph.d1((rm + rmax) / 2));
  const double h = delta_phi / om;
  const double lin_t = fabs(ph.d2((rm + rmax) / 2)) * h * h;
  KSum acc[LC];
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
    const FilonConst fc = filon_const(om, (rmax - rm) / nseg, nn);
    for (int s = lane; s < nseg; s += 32) {
      const double a = lin(rm, rmax, nseg + 1, s), b = lin(rm, rmax, nseg + 1, s + 1);
      filon_segment_all(m, L0, nl, a, b, nn, om, off, fc, acc);
    }
  } else {
    // four segments per warp pass, one per group of 8 lanes; lane 0 of a group accumulates it
    const int nseg = (int)max(1.0, ceil((rmax - rm) / h));
    const int grp = lane >> 3;
    for (int s0 = 0; s0 < nseg; s0 += 4) {  // warp-uniform
      const int s = s0 + grp;
      const bool valid = s < nseg;
      const double a = valid ? lin(rm, rmax, nseg + 1, s) : rm;
      const double b = valid ? lin(rm, rmax, nseg + 1, s + 1) : rm;
      double res[LC];
      levin_segment_group(m, L0, nl, ph, a, b, valid, res);
      if (valid && (lane & 7) == 0) {
#pragma unroll
        for (int q = 0; q < LC; ++q)
          if (q < nl) acc[q].add(res[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < LC; ++q) res[q] = warp_sum(acc[q].s + acc[q].c);
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

// one warp per (record, chunk of up to LC multipoles): the Filon / Levin segments of both phase
// branches over the lanes, every node's phase factor and every panel's weights shared by the chunk
#ifndef DWBA_TAILS_MIN_BLOCKS
// three CTAs per SM (168 registers): measured 5.87 ms on the 64-energy sweep's 106,293 records,
// against 6.31 ms at four (128 registers, spills)
#define DWBA_TAILS_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(128, DWBA_TAILS_MIN_BLOCKS) tails_kernel(const dwba_tail_t* __restrict__ recs, int n, int L_max, int max_seg, double max_dphi,
                             LevinD lv) {
  for (int i = threadIdx.x; i < 72; i += blockDim.x)
    (&s_lv.D[0][0])[i] = i < 64 ? lv.D[i / 8][i % 8] : lv.xr[i - 64];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int n_chunk = (L_max + LC - 1) / LC;
  const int64_t warp_g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t n_items = (int64_t)n * n_chunk;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t it = warp_g; it < n_items; it += stride) {
    const int rec = (int)(it / n_chunk);
    const int L0 = 1 + (int)(it - (int64_t)rec * n_chunk) * LC;  // multipoles L0 .. L0+nl-1
    const int nl = min(LC, L_max + 1 - L0);
    const dwba_tail_t* R = recs + rec;
    const WaveD wi = {R->wave[0], R->wave[2], R->wave[3], R->wave[4], (int)R->wave[1]};
    const WaveD wf = {R->wave[5], R->wave[7], R->wave[8], R->wave[9], (int)R->wave[6]};
    const double r_m = R->r_m, r_max = R->r_max;
    double m[LC];
    bool any = false;
#pragma unroll
    for (int q = 0; q < LC; ++q) {
      const double v = q < nl ? R->moments_dev[L0 + q] : 0.0;
      m[q] = fabs(v) > 1e-12 ? v : 0.0;  // moments at or below the cut-off give a zero tail
      any = any || m[q] != 0.0;
    }
    double t[LC];
#pragma unroll
    for (int q = 0; q < LC; ++q) t[q] = 0.0;
    if (any && R->mode != 1 && !(r_max <= r_m + 1e-10)) {
      double im[LC], ip[LC];
      outer_branch_all(m, L0, nl, PhaseD(wi, wf, -1), r_m, r_max, max_seg, max_dphi, lane, im);
      outer_branch_all(m, L0, nl, PhaseD(wi, wf, +1), r_m, r_max, max_seg, max_dphi, lane, ip);
#pragma unroll
      for (int q = 0; q < LC; ++q) t[q] = 0.5 * (im[q] - ip[q]);
    }
    if (lane == 0) {
      for (int q = 0; q < nl; ++q) {
        double v = 0.0;
        if (m[q] != 0.0) {
          v = R->mode == 1 ? analytical_tail(r_m, wi, wf, L0 + q, m[q])
                           : t[q] + analytical_tail(r_max, wi, wf, L0 + q, m[q]);
        }
        R->out_dev[L0 + q] = v;
      }
      if (L0 == 1) R->out_dev[0] = 0.0;
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
  const int64_t warps = (int64_t)n * ((L_max + LC - 1) / LC);
  const int blocks = dwba_grid_1d(warps * 32, 128, 65535);
  tails_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>(tails_dev, n, L_max, max_filon_segments, max_effective_dphi,
                                                         lv);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}
