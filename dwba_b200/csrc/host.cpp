// Host-side helpers of the C ABI: status strings, device probe, Coulomb phase
// breakpoints and the outer-tail integrals of the direct term.
//
// Compiled with -ffp-contract=off: the breakpoint recursion and the phase
// arithmetic must round exactly like the reference's NumPy/Python scalar code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "../../include/dwba_b200.h"

typedef std::complex<double> cplx;

extern "C" int dwba_abi_version(void) { return DWBA_ABI_VERSION; }

extern "C" const char* dwba_status_string(int status) {
  switch (status) {
    case DWBA_OK: return "ok";
    case DWBA_ERR_INVALID_ARG: return "invalid argument";
    case DWBA_ERR_CUDA: return "CUDA launch or runtime failure";
    case DWBA_ERR_NO_DEVICE: return "no usable sm_100 GPU";
    case DWBA_ERR_WORKSPACE: return "workspace too small";
    case DWBA_ERR_UNSUPPORTED: return "request outside the kernel's numeric range";
    case DWBA_ERR_RANGE: return "device-side consistency check failed";
    default: return "unknown status";
  }
}

extern "C" int dwba_device_probe(int* n_devices, int* cc_major, int* cc_minor) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    if (n_devices) *n_devices = 0;
    return DWBA_ERR_NO_DEVICE;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return DWBA_ERR_NO_DEVICE;
  if (n_devices) *n_devices = n;
  if (cc_major) *cc_major = prop.major;
  if (cc_minor) *cc_minor = prop.minor;
  return prop.major == 10 ? DWBA_OK : DWBA_ERR_NO_DEVICE;
}

// oscillatory_integrals.py:1677-1710 (generate_phase_nodes, eta != 0), same
// operation order so every breakpoint is bit-identical to the Python loop.
extern "C" int dwba_phase_breaks_coulomb(double r_start, double r_end, double k_total, double dphi,
                                         double eta_total, double* out_host, int cap, int* n_out) {
  if (!out_host || !n_out || cap < 2) return DWBA_ERR_INVALID_ARG;
  int n = 0;
  out_host[n++] = r_start;
  double r = r_start;
  const double span10 = (r_end - r_start) / 10;
  while (r < r_end) {
    const double phi_prime = k_total + eta_total / std::max(r, 1e-10);
    double dr = dphi / std::fabs(phi_prime);
    dr = std::min(dr, span10);
    dr = std::max(dr, 1e-6);
    double rn = r + dr;
    if (rn >= r_end) rn = r_end;
    if (n >= cap) return DWBA_ERR_WORKSPACE;
    out_host[n++] = rn;
    r = rn;
    if (n > 10000) break;
  }
  *n_out = n;
  return DWBA_OK;
}

// ---------------------------------------------------------------------------
// Outer tails (oscillatory_integrals.py)
// ---------------------------------------------------------------------------
namespace {

struct Wave {
  double k, delta, eta, sigma;
  int l;
};

// Phase of cos(Phi_a -/+ Phi_b) with its derivatives, :312-456.
struct Phase {
  Wave a, b;
  int sgn;  // -1: difference, +1: sum
  double kk, cc;
  Phase(const Wave& wa, const Wave& wb, int s) : a(wa), b(wb), sgn(s) {
    const double ca = -a.l * M_PI / 2 + a.sigma + a.delta;
    const double cb = -b.l * M_PI / 2 + b.sigma + b.delta;
    kk = s < 0 ? a.k - b.k : a.k + b.k;
    cc = s < 0 ? ca - cb : ca + cb;
  }
  double phi(double r) const {
    double v = kk * r + cc;
    if (std::fabs(a.eta) > 1e-15) v += a.eta * std::log(2 * a.k * r + 1e-30);
    if (std::fabs(b.eta) > 1e-15) {
      const double t = b.eta * std::log(2 * b.k * r + 1e-30);
      v = sgn < 0 ? v - t : v + t;
    }
    if (a.l > 0) v -= (a.l * (a.l + 1)) / (2.0 * a.k * r);
    if (b.l > 0) {
      const double t = (b.l * (b.l + 1)) / (2.0 * b.k * r);
      v = sgn < 0 ? v + t : v - t;
    }
    return v;
  }
  double d1(double r) const {
    double v = kk;
    if (std::fabs(a.eta) > 1e-15) v += a.eta / r;
    if (std::fabs(b.eta) > 1e-15) v = sgn < 0 ? v - b.eta / r : v + b.eta / r;
    if (a.l > 0) v += (a.l * (a.l + 1)) / (2.0 * a.k * std::pow(r, 2.0));
    if (b.l > 0) {
      const double t = (b.l * (b.l + 1)) / (2.0 * b.k * std::pow(r, 2.0));
      v = sgn < 0 ? v - t : v + t;
    }
    return v;
  }
  double d2(double r) const {
    double v = 0.0;
    if (std::fabs(a.eta) > 1e-15) v -= a.eta / (r * r);
    if (std::fabs(b.eta) > 1e-15) v = sgn < 0 ? v + b.eta / (r * r) : v - b.eta / (r * r);
    if (a.l > 0) v -= (a.l * (a.l + 1)) / (a.k * std::pow(r, 3.0));
    if (b.l > 0) {
      const double t = (b.l * (b.l + 1)) / (b.k * std::pow(r, 3.0));
      v = sgn < 0 ? v + t : v - t;
    }
    return v;
  }
};

// Envelope M_L / r^(L+1) (zero for r <= 1e-6), dwba_matrix_elements.py:1223-1224.
struct Envelope {
  double m;
  int L;
  double operator()(double r) const { return r > 1e-6 ? m / std::pow(r, (double)(L + 1)) : 0.0; }
};

// numpy.linspace arithmetic
static void linspace(double a, double b, int n, std::vector<double>& out) {
  out.resize(n);
  if (n == 1) { out[0] = a; return; }
  const double step = (b - a) / (double)(n - 1);
  for (int i = 0; i < n; ++i) out[i] = (double)i * step + a;
  out[n - 1] = b;
}

// exactly-rounded style summation (Neumaier) standing in for math.fsum
struct CompSum {
  double s = 0.0, c = 0.0;
  void add(double x) {
    const double t = s + x;
    if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};

// scipy.integrate.simpson for an odd number of points with possibly unequal spacing
static double simpson_odd(const double* y, const double* x, int n) {
  double acc = 0.0;
  for (int i = 0; i + 2 < n; i += 2) {
    const double h0 = x[i + 1] - x[i], h1 = x[i + 2] - x[i + 1];
    const double hs = h0 + h1, hp = h0 * h1, q = h0 / h1;
    acc += hs / 6.0 * (y[i] * (2.0 - 1.0 / q) + y[i + 1] * (hs * (hs / hp)) + y[i + 2] * (2.0 - q));
  }
  return acc;
}

static cplx cexpi(double phi) { return cplx(std::cos(phi), std::sin(phi)); }

// _filon_segment_complex, :1165-1277
static cplx filon_segment(const double* f, const double* x, int n, double omega, double off) {
  if (n < 2) return cplx(0, 0);
  const double a = x[0], b = x[n - 1], h = b - a;
  if (h < 1e-15) return cplx(0, 0);
  if (std::fabs(omega * h) < 1e-3) {
    const double mid = omega * (a + b) / 2 + off;
    return simpson_odd(f, x, n) * cexpi(mid);
  }
  if (n == 3) {
    const double th = omega * h / 2;
    const double st = std::sin(th), ct = std::cos(th);
    double al, be, ga;
    if (std::fabs(th) < 0.3) {
      const double t2 = std::pow(th, 2.0), t3 = std::pow(th, 3.0);
      al = 2 * t3 / 45 * (1 - t2 / 7 + std::pow(t2, 2.0) / 189);
      be = 2.0 / 3 + 2 * t2 / 15 - 4 * std::pow(t2, 2.0) / 105 + 2 * std::pow(t2, 3.0) / 567;
      ga = 4.0 / 3 - 2 * t2 / 15 + 1 * std::pow(t2, 2.0) / 210 - std::pow(t2, 3.0) / 11340;
    } else {
      const double t2 = std::pow(th, 2.0);
      const double s2 = std::sin(2 * th), c2 = std::cos(2 * th), t3 = std::pow(th, 3.0);
      al = (t2 + th * s2 / 2 - 2 * std::pow(st, 2.0)) / t3;
      be = 2 * (th * (1 + c2) - s2) / t3;
      ga = 4 * (st - th * ct) / t3;
    }
    const cplx e0 = cexpi(omega * x[0] + off), e1 = cexpi(omega * x[1] + off), e2 = cexpi(omega * x[2] + off);
    const cplx mi = cplx(0.0, -1.0) / omega;
    return (h / 2) * (al * mi * (f[2] * e2 - f[0] * e0) + be * (f[0] * e0 + f[2] * e2) + ga * f[1] * e1);
  }
  cplx res(0, 0);
  for (int i = 0; i + 2 < n; i += 2) res += filon_segment(f + i, x + i, 3, omega, off);
  if (n > 2 && (n - 1) % 2 == 1) {
    const double p0 = omega * x[n - 2] + off, p1 = omega * x[n - 1] + off;
    res += 0.5 * (x[n - 1] - x[n - 2]) * (f[n - 2] * cexpi(p0) + f[n - 1] * cexpi(p1));
  }
  return res;
}

// Gauss-Kronrod 21-point rule (QUADPACK qk21 nodes/weights) with bisection on the
// largest error, standing in for scipy.integrate.quad on the smooth envelopes.
template <class F>
static double gk21(const F& f, double a, double b, double* err) {
  static const double xgk[11] = {0.995657163025808080735527280689003, 0.973906528517171720077964012084452,
                                 0.930157491355708226001207180059508, 0.865063366688984510732096688423493,
                                 0.780817726586416897063717578345042, 0.679409568299024406234327365114874,
                                 0.562757134668604683339000099272694, 0.433395394129247190799265943165784,
                                 0.294392862701460198131126603103866, 0.148874338981631210884826001129720,
                                 0.000000000000000000000000000000000};
  static const double wgk[11] = {0.011694638867371874278064396062192, 0.032558162307964727478818972459390,
                                 0.054755896574351996031381300244580, 0.075039674810919952767043140916190,
                                 0.093125454583697605535065465083366, 0.109387158802297641899210590325805,
                                 0.123491976262065851077600525430180, 0.134709217311473325928054001771707,
                                 0.142775938577060080797094273138717, 0.147739104901338491374841515972068,
                                 0.149445554002916905664936468389821};
  static const double wg[5] = {0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
                               0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
                               0.295524224714752870173892994651338};
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  const double fc = f(c);
  double rk = fc * wgk[10], rg = 0.0;
  for (int j = 0; j < 10; ++j) {
    const double dx = h * xgk[j];
    const double s = f(c - dx) + f(c + dx);
    rk += wgk[j] * s;
    if (j % 2 == 1) rg += wg[j / 2] * s;
  }
  *err = std::fabs((rk - rg) * h);
  return rk * h;
}

template <class F>
static double adaptive_quad(const F& f, double a, double b) {
  struct Seg {
    double a, b, v, e;
  };
  std::vector<Seg> segs;
  double e;
  double v = gk21(f, a, b, &e);
  segs.push_back({a, b, v, e});
  for (int it = 0; it < 50; ++it) {
    double tv = 0.0, te = 0.0;
    size_t worst = 0;
    for (size_t i = 0; i < segs.size(); ++i) {
      tv += segs[i].v;
      te += segs[i].e;
      if (segs[i].e > segs[worst].e) worst = i;
    }
    if (te <= std::max(1.49e-8, 1.49e-8 * std::fabs(tv))) return tv;
    Seg s = segs[worst];
    const double m = 0.5 * (s.a + s.b);
    double e1, e2;
    const double v1 = gk21(f, s.a, m, &e1), v2 = gk21(f, m, s.b, &e2);
    segs[worst] = {s.a, m, v1, e1};
    segs.push_back({m, s.b, v2, e2});
  }
  double tv = 0.0;
  for (auto& s : segs) tv += s.v;
  return tv;
}

// filon_oscillatory_integral, :1280-1358
static cplx filon_integral(const Envelope& env, double omega, double off, double r0, double r1, double dphi,
                           int max_seg, double max_dphi) {
  const int nseg_nodes = 5;
  const double dr = dphi / std::fabs(omega);
  const long nraw = std::max(1L, (long)std::ceil((r1 - r0) / dr));
  const int nseg = (int)std::min<long>(nraw, max_seg);
  const double eff = std::fabs(omega) * (r1 - r0) / std::max(1, nseg);
  int nn = nseg_nodes;
  if (eff > max_dphi) {
    const int sc = (int)std::ceil(eff / max_dphi);
    nn = std::min(15, std::max(nseg_nodes, nseg_nodes + 2 * (sc - 1)));
  }
  std::vector<double> bnd, x, fv(nn);
  linspace(r0, r1, nseg + 1, bnd);
  CompSum re, im;
  for (int i = 0; i < nseg; ++i) {
    linspace(bnd[i], bnd[i + 1], nn, x);
    for (int j = 0; j < nn; ++j) fv[j] = env(x[j]);
    const cplx c = filon_segment(fv.data(), x.data(), nn, omega, off);
    re.add(c.real());
    im.add(c.imag());
  }
  return cplx(re.value(), im.value());
}

// _chebyshev_differentiation_matrix, :970-1021 (Chebyshev-Lobatto points descending)
static void cheb_D(int n, std::vector<double>& D) {
  D.assign((size_t)n * n, 0.0);
  std::vector<double> x(n), c(n, 1.0);
  for (int i = 0; i < n; ++i) x[i] = std::cos(M_PI * i / (n - 1));
  c[0] = c[n - 1] = 2.0;
  for (int i = 0; i < n; ++i) {
    double rs = 0.0;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      const double sgn = ((i + j) % 2 == 0) ? 1.0 : -1.0;
      const double v = (c[i] / c[j]) * sgn / (x[i] - x[j]);
      D[(size_t)i * n + j] = v;
      rs += v;
    }
    D[(size_t)i * n + i] = -rs;
  }
}

// complex LU with partial pivoting (pivot by |re|+|im| as LAPACK's izamax)
static bool csolve(std::vector<cplx>& A, std::vector<cplx>& b, int n) {
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = -1.0;
    for (int i = k; i < n; ++i) {
      const cplx v = A[(size_t)i * n + k];
      const double m = std::fabs(v.real()) + std::fabs(v.imag());
      if (m > best) { best = m; piv = i; }
    }
    if (best == 0.0) return false;
    if (piv != k) {
      for (int j = 0; j < n; ++j) std::swap(A[(size_t)k * n + j], A[(size_t)piv * n + j]);
      std::swap(b[k], b[piv]);
    }
    const cplx inv = 1.0 / A[(size_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      const cplx l = A[(size_t)i * n + k] * inv;
      if (l == cplx(0, 0)) continue;
      for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    cplx s = b[i];
    for (int j = i + 1; j < n; ++j) s -= A[(size_t)i * n + j] * b[j];
    b[i] = s / A[(size_t)i * n + i];
  }
  return true;
}

// levin_oscillatory_integral + _levin_segment_complex, :1024-1162
static cplx levin_integral(const Envelope& env, const Phase& ph, double r0, double r1, int n, int nseg) {
  std::vector<double> bnd, Dref;
  linspace(r0, r1, std::max(1, nseg) + 1, bnd);
  cheb_D(n, Dref);
  std::vector<double> xr(n), x(n);
  for (int k = 0; k < n; ++k) xr[k] = std::cos(M_PI * (n - 1 - k) / (n - 1));  // ascending (reversed) nodes
  CompSum re, im;
  std::vector<cplx> A((size_t)n * n), u(n);
  for (int s = 0; s < std::max(1, nseg); ++s) {
    const double a = bnd[s], b = bnd[s + 1];
    for (int k = 0; k < n; ++k) x[k] = 0.5 * (b - a) * (xr[k] + 1) + a;
    const double h = x[n - 1] - x[0];
    if (h < 1e-15) continue;
    const double sc = 2.0 / h;
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = cplx(Dref[(size_t)i * n + j] * sc, 0.0);
      A[(size_t)i * n + i] += cplx(0.0, ph.d1(x[i]));
      u[i] = cplx(env(x[i]), 0.0);
    }
    if (!csolve(A, u, n)) continue;  // the reference falls back to lstsq; a singular system does not occur here
    const cplx c = u[n - 1] * cexpi(ph.phi(x[n - 1])) - u[0] * cexpi(ph.phi(x[0]));
    re.add(c.real());
    im.add(c.imag());
  }
  return cplx(re.value(), im.value());
}

// compute_outer_integral_oscillatory, :1361-1451
static cplx outer_osc(const Envelope& env, const Phase& ph, double rm, double rmax, int max_seg, double max_dphi) {
  const double delta_phi = M_PI / 4;
  if (rmax <= rm + 1e-10) return cplx(0, 0);
  const double om = std::fabs(ph.d1((rm + rmax) / 2));
  if (om < 1e-10) {
    const double re = adaptive_quad([&](double r) { return env(r) * std::cos(ph.phi(r)); }, rm, rmax);
    const double im = adaptive_quad([&](double r) { return env(r) * std::sin(ph.phi(r)); }, rm, rmax);
    return cplx(re, im);
  }
  const double h = delta_phi / om;
  const double lin = std::fabs(ph.d2((rm + rmax) / 2)) * h * h;
  if (lin < 0.1) return filon_integral(env, om, ph.phi(rm) - om * rm, rm, rmax, delta_phi, max_seg, max_dphi);
  const int nseg = (int)std::max(1.0, std::ceil((rmax - rm) / h));
  return levin_integral(env, ph, rm, rmax, 8, nseg);
}

// _analytical_multipole_tail, :2064-2184
static double analytical_tail(double r_m, const Wave& wi, const Wave& wf, int L, double overlap) {
  if (r_m < 1e-3 || std::fabs(overlap) < 1e-12) return 0.0;
  const double lti = std::fabs(wi.eta) > 1e-10 ? wi.eta * std::log(2 * wi.k * r_m + 1e-30) : 0.0;
  const double ltf = std::fabs(wf.eta) > 1e-10 ? wf.eta * std::log(2 * wf.k * r_m + 1e-30) : 0.0;
  const double ci = -wi.l * M_PI / 2 + wi.sigma + wi.delta + lti;
  const double cf = -wf.l * M_PI / 2 + wf.sigma + wf.delta + ltf;
  const double kd = wi.k - wf.k, ks = wi.k + wf.k;
  const int n = L + 1;
  double t = 0.0;
  const double pd = kd * r_m + ci - cf;
  if (std::fabs(kd) > 1e-6) {
    const double lead = std::sin(pd) / (kd * std::pow(r_m, (double)n));
    const double corr = n * std::cos(pd) / (std::pow(kd, 2.0) * std::pow(r_m, (double)(n + 1)));
    t += 0.5 * (lead + corr);
  } else if (n > 1) {
    t += 0.5 * std::cos(pd) / ((n - 1) * std::pow(r_m, (double)(n - 1)));
  }
  const double ps = ks * r_m + ci + cf;
  if (ks > 1e-6) {
    const double lead = std::sin(ps) / (ks * std::pow(r_m, (double)n));
    const double corr = n * std::cos(ps) / (std::pow(ks, 2.0) * std::pow(r_m, (double)(n + 1)));
    t -= 0.5 * (lead + corr);
  }
  if (!std::isfinite(t)) return 0.0;
  return t * overlap;
}

}  // namespace

extern "C" int dwba_outer_tails(const double* wave_host, double r_m, double r_max, int L_max,
                                const double* moments_host, int mode, int max_filon_segments,
                                double max_effective_dphi, double* tail_host) {
  if (!wave_host || !moments_host || !tail_host || L_max < 0 || L_max > DWBA_MAX_L || (mode != 0 && mode != 1) ||
      max_filon_segments < 1 || !(max_effective_dphi > 0.0))
    return DWBA_ERR_INVALID_ARG;
  const Wave wi = {wave_host[0], wave_host[2], wave_host[3], wave_host[4], (int)wave_host[1]};
  const Wave wf = {wave_host[5], wave_host[7], wave_host[8], wave_host[9], (int)wave_host[6]};
  tail_host[0] = 0.0;
  for (int L = 1; L <= L_max; ++L) {
    const double m = moments_host[L];
    tail_host[L] = 0.0;
    if (!(std::fabs(m) > 1e-12)) continue;
    if (mode == 1) {  // legacy: analytical tail from the match point
      tail_host[L] = analytical_tail(r_m, wi, wf, L, m);
      continue;
    }
    double t = 0.0;
    if (!(r_max <= r_m + 1e-10)) {
      const Envelope env{m, L};
      const cplx im = outer_osc(env, Phase(wi, wf, -1), r_m, r_max, max_filon_segments, max_effective_dphi);
      const cplx ip = outer_osc(env, Phase(wi, wf, +1), r_m, r_max, max_filon_segments, max_effective_dphi);
      t = 0.5 * (im.real() - ip.real());
    }
    tail_host[L] = t + analytical_tail(r_max, wi, wf, L, m);
  }
  return DWBA_OK;
}

// Sizes of the descriptor structs, so a binding can verify its layout.
extern "C" int dwba_struct_sizes(int64_t* sizes, int n) {
  if (!sizes || n < 3) return DWBA_ERR_INVALID_ARG;
  sizes[0] = (int64_t)sizeof(dwba_nodeset_t);
  sizes[1] = (int64_t)sizeof(dwba_fold_t);
  sizes[2] = (int64_t)sizeof(dwba_form_t);
  if (n >= 4) sizes[3] = (int64_t)sizeof(dwba_tail_t);
  if (n >= 5) sizes[4] = (int64_t)sizeof(dwba_form_grad_t);
  if (n >= 6) sizes[5] = (int64_t)sizeof(dwba_fold_adj_t);
  if (n >= 7) sizes[6] = (int64_t)sizeof(dwba_fold_multi_t);
  if (n >= 8) sizes[7] = (int64_t)sizeof(dwba_potential_t);
  if (n >= 9) sizes[8] = (int64_t)sizeof(dwba_dot_t);
  if (n >= 10) sizes[9] = (int64_t)sizeof(dwba_cupy_set_t);
  if (n >= 11) sizes[10] = (int64_t)sizeof(dwba_cupy_form_t);
  if (n >= 12) sizes[11] = (int64_t)sizeof(dwba_tc_segment_t);
  if (n >= 13) sizes[12] = (int64_t)sizeof(dwba_tc_tile_t);
  return DWBA_OK;
}

// 1 when both phase branches of a pair take the Filon/Levin path (the device kernel's domain),
// 0 when one of them falls into the adaptive-quadrature branch (mid-interval frequency < 1e-10).
extern "C" int dwba_outer_tail_on_device(const double* wave_host, double r_m, double r_max) {
  if (!wave_host) return 0;
  const Wave wi = {wave_host[0], wave_host[2], wave_host[3], wave_host[4], (int)wave_host[1]};
  const Wave wf = {wave_host[5], wave_host[7], wave_host[8], wave_host[9], (int)wave_host[6]};
  const double mid = (r_m + r_max) / 2;
  for (int sgn = -1; sgn <= 1; sgn += 2)
    if (std::fabs(Phase(wi, wf, sgn).d1(mid)) < 1e-10) return 0;
  return 1;
}
