// Exchange-correlation functionals on the device.
//
// The reference evaluates its functionals with libxc on the host
// (xc_lda_exc_vxc / xc_gga_exc_vxc, nukexc/xc_integrals.hpp:113, :203, :471,
// :617), copying rho/sigma device->host and the potentials back.  Here they
// are restated from the published definitions and evaluated on the device:
//   1   LDA_X       Dirac/Slater exchange
//   7   LDA_C_VWN   Vosko-Wilk-Nusair 1980, parametrisation V (VWN5)
//   101 GGA_X_PBE   Perdew-Burke-Ernzerhof 1996 exchange (kappa 0.804,
//                   mu = beta pi^2 / 3)
//   130 GGA_C_PBE   PBE correlation on Perdew-Wang 1992 LDA correlation
// f(ra, rb, saa, sab, sbb) is the energy per unit volume; the potentials are
// its exact partial derivatives, taken by forward-mode dual numbers.
#pragma once

#include "common.cuh"

namespace nkx {

template <int N>
struct Dual {
  double v;
  double d[N];
};

template <int N>
NKX_HD inline Dual<N> dconst(double c) {
  Dual<N> r;
  r.v = c;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = 0.0;
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  const double ib = 1.0 / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator+(const Dual<N> &a, double c) {
  Dual<N> r = a;
  r.v += c;
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator+(double c, const Dual<N> &a) {
  return a + c;
}
template <int N>
NKX_HD inline Dual<N> operator-(const Dual<N> &a, double c) {
  Dual<N> r = a;
  r.v -= c;
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator-(double c, const Dual<N> &a) {
  Dual<N> r;
  r.v = c - a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator-(const Dual<N> &a) {
  return 0.0 - a;
}
template <int N>
NKX_HD inline Dual<N> operator*(const Dual<N> &a, double c) {
  Dual<N> r;
  r.v = a.v * c;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * c;
  return r;
}
template <int N>
NKX_HD inline Dual<N> operator*(double c, const Dual<N> &a) {
  return a * c;
}
template <int N>
NKX_HD inline Dual<N> operator/(const Dual<N> &a, double c) {
  return a * (1.0 / c);
}
template <int N>
NKX_HD inline Dual<N> operator/(double c, const Dual<N> &a) {
  return dconst<N>(c) / a;
}
template <int N>
NKX_HD inline Dual<N> chain(const Dual<N> &a, double v, double dv) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = dv * a.d[i];
  return r;
}
template <int N>
NKX_HD inline Dual<N> dpow(const Dual<N> &a, double p) {
  const double v = pow(a.v, p);
  return chain(a, v, p * v / a.v);
}
template <int N>
NKX_HD inline Dual<N> dexp(const Dual<N> &a) {
  const double v = exp(a.v);
  return chain(a, v, v);
}
template <int N>
NKX_HD inline Dual<N> dexpm1(const Dual<N> &a) {
  return chain(a, expm1(a.v), exp(a.v));
}
template <int N>
NKX_HD inline Dual<N> dlog(const Dual<N> &a) {
  return chain(a, log(a.v), 1.0 / a.v);
}
template <int N>
NKX_HD inline Dual<N> dsqrt(const Dual<N> &a) {
  const double v = sqrt(a.v);
  return chain(a, v, 0.5 / v);
}
template <int N>
NKX_HD inline Dual<N> datan(const Dual<N> &a) {
  return chain(a, atan(a.v), 1.0 / (1.0 + a.v * a.v));
}

// ------------------------------------------------------------ formulas ----
// f(zeta) of the spin interpolation, from 1 + zeta = 2 ra / rho and
// 1 - zeta = 2 rb / rho (no cancellation at zeta -> +-1)
template <class T>
NKX_HD inline T fzeta(const T &opz, const T &omz) {
  return (dpow(opz, 4.0 / 3.0) + dpow(omz, 4.0 / 3.0) - 2.0) / (pow(2.0, 4.0 / 3.0) - 2.0);
}

template <class T>
NKX_HD inline T f_lda_x(const T &ra, const T &rb) {
  const double c = -0.75 * cbrt(6.0 / kPi);
  return c * (dpow(ra, 4.0 / 3.0) + dpow(rb, 4.0 / 3.0));
}

template <class T>
NKX_HD inline T vwn_g(const T &x, double A, double b, double c, double x0) {
  const double Q = sqrt(4.0 * c - b * b);
  const T X = x * x + b * x + c;
  const double X0 = x0 * x0 + b * x0 + c;
  const T at = datan(Q / (2.0 * x + b));
  return A * (dlog(x * x / X) + (2.0 * b / Q) * at -
              (b * x0 / X0) * (dlog((x - x0) * (x - x0) / X) + (2.0 * (b + 2.0 * x0) / Q) * at));
}

template <class T>
NKX_HD inline T f_vwn5(const T &ra, const T &rb) {
  const T rho = ra + rb;
  const T rs = dpow(3.0 / (4.0 * kPi * rho), 1.0 / 3.0);
  const T x = dsqrt(rs);
  const T zeta = (ra - rb) / rho;
  const T opz = 2.0 * ra / rho, omz = 2.0 * rb / rho;
  const T eP = vwn_g(x, 0.0310907, 3.72744, 12.9352, -0.10498);
  const T eF = vwn_g(x, 0.01554535, 7.06042, 18.0578, -0.32500);
  const T eA = vwn_g(x, -1.0 / (6.0 * kPi * kPi), 1.13107, 13.0045, -0.0047584);
  const double fpp0 = 4.0 / (9.0 * (cbrt(2.0) - 1.0));
  const T fz = fzeta(opz, omz);
  const T z2 = zeta * zeta;
  const T z4 = z2 * z2;
  return rho * (eP + eA * fz * (1.0 / fpp0) * (1.0 - z4) + (eF - eP) * fz * z4);
}

template <class T>
NKX_HD inline T pw92_g(const T &rs, double A, double a1, double b1, double b2, double b3, double b4) {
  const T srs = dsqrt(rs);
  const T den = 2.0 * A * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
  return -2.0 * A * (1.0 + a1 * rs) * dlog(1.0 + 1.0 / den);
}

// Perdew-Wang 92 correlation energy per particle (Phys. Rev. B 45, 13244).
// mod = false: the published constants (A = 0.031091, 0.015545, 0.016887,
// f''(0) = 1.709921; libxc's LDA_C_PW); mod = true: the constants carried to
// more digits that PBE correlation uses (libxc's LDA_C_PW_MOD).
template <class T>
NKX_HD inline T eps_pw92(const T &rs, const T &zeta, const T &opz, const T &omz, bool mod = true) {
  const T gP = pw92_g(rs, mod ? 0.0310907 : 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294);
  const T gF = pw92_g(rs, mod ? 0.01554535 : 0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517);
  const T gA = pw92_g(rs, mod ? 0.0168869 : 0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671);
  const double fz20 = mod ? 1.709920934161365617563962776245 : 1.709921;
  const T fz = fzeta(opz, omz);
  const T z2 = zeta * zeta;
  const T z4 = z2 * z2;
  return gP - gA * fz * (1.0 / fz20) * (1.0 - z4) + (gF - gP) * fz * z4;
}

template <class T>
NKX_HD inline T f_pw92(const T &ra, const T &rb, bool mod) {
  const T rho = ra + rb;
  const T rs = dpow(3.0 / (4.0 * kPi * rho), 1.0 / 3.0);
  return rho * eps_pw92(rs, (ra - rb) / rho, 2.0 * ra / rho, 2.0 * rb / rho, mod);
}

template <class T>
NKX_HD inline T f_pbe_x_unpol(const T &n, const T &s2n) {
  const double kappa = 0.8040, mu = 0.2195149727645171;
  const T ex = (-0.75 * cbrt(3.0 / kPi)) * dpow(n, 4.0 / 3.0);
  const T s2 = s2n / ((4.0 * pow(3.0 * kPi * kPi, 2.0 / 3.0)) * dpow(n, 8.0 / 3.0));
  const T Fx = (1.0 + kappa) - kappa / (1.0 + (mu / kappa) * s2);
  return ex * Fx;
}

template <class T>
NKX_HD inline T f_pbe_x(const T &ra, const T &rb, const T &saa, const T &sbb) {
  return 0.5 * f_pbe_x_unpol(2.0 * ra, 4.0 * saa) + 0.5 * f_pbe_x_unpol(2.0 * rb, 4.0 * sbb);
}

template <class T>
NKX_HD inline T f_pbe_c(const T &ra, const T &rb, const T &sigma) {
  const double beta = 0.06672455060314922;
  const double gamma = (1.0 - log(2.0)) / (kPi * kPi);
  const T rho = ra + rb;
  const T zeta = (ra - rb) / rho;
  const T opz = 2.0 * ra / rho, omz = 2.0 * rb / rho;
  const T rs = dpow(3.0 / (4.0 * kPi * rho), 1.0 / 3.0);
  const T ec = eps_pw92(rs, zeta, opz, omz);
  const T phi = 0.5 * (dpow(opz, 2.0 / 3.0) + dpow(omz, 2.0 / 3.0));
  const T kF = dpow(3.0 * kPi * kPi * rho, 1.0 / 3.0);
  const T ks2 = 4.0 * kF / kPi;
  const T t2 = sigma / (4.0 * phi * phi * ks2 * rho * rho);
  const T phi3 = phi * phi * phi;
  const T A = (beta / gamma) / dexpm1(-ec / (gamma * phi3));
  const T At2 = A * t2;
  const T H = gamma * phi3 * dlog(1.0 + (beta / gamma) * t2 * (1.0 + At2) / (1.0 + At2 + At2 * At2));
  return rho * (ec + H);
}

NKX_HD inline bool func_is_gga(int id) { return id == NKX_XC_GGA_X_PBE || id == NKX_XC_GGA_C_PBE; }
NKX_HD inline bool func_supported(int id) {
  return id == NKX_XC_LDA_X || id == NKX_XC_LDA_C_VWN || id == NKX_XC_LDA_C_PW || id == NKX_XC_LDA_C_PW_MOD ||
         id == NKX_XC_GGA_X_PBE || id == NKX_XC_GGA_C_PBE;
}

template <int N>
NKX_HD inline Dual<N> f_total(int id, const Dual<N> &ra, const Dual<N> &rb, const Dual<N> &saa,
                              const Dual<N> &sab, const Dual<N> &sbb) {
  switch (id) {
    case NKX_XC_LDA_X: return f_lda_x(ra, rb);
    case NKX_XC_LDA_C_VWN: return f_vwn5(ra, rb);
    case NKX_XC_LDA_C_PW: return f_pw92(ra, rb, false);
    case NKX_XC_LDA_C_PW_MOD: return f_pw92(ra, rb, true);
    case NKX_XC_GGA_X_PBE: return f_pbe_x(ra, rb, saa, sbb);
    case NKX_XC_GGA_C_PBE: return f_pbe_c(ra, rb, saa + 2.0 * sab + sbb);
    default: return dconst<N>(0.0);
  }
}

// Functional list evaluated at one point.
struct XcSpec {
  int nfunc;
  int ids[4];
  double thr;
};

// Closed shell: f(rho, sigma) summed over the list, with d f / d rho and
// d f / d sigma.  Evaluated as the spin-polarised formula at
// ra = rb = rho/2, saa = sab = sbb = sigma/4 (the libxc convention).
NKX_HD inline void xc_unpol(const XcSpec &s, double rho, double sigma, double &f, double &vrho,
                            double &vsigma) {
  f = vrho = vsigma = 0.0;
  if (!(rho >= s.thr)) return;
  Dual<2> ra, sg;
  ra.v = fmax(0.5 * rho, 1e-30);
  ra.d[0] = 0.5;
  ra.d[1] = 0.0;
  sg.v = fmax(0.25 * sigma, 1e-40);
  sg.d[0] = 0.0;
  sg.d[1] = 0.25;
  for (int i = 0; i < s.nfunc; ++i) {
    const Dual<2> r = f_total<2>(s.ids[i], ra, ra, sg, sg, sg);
    f += r.v;
    vrho += r.d[0];
    vsigma += r.d[1];
  }
}

// Open shell: f(ra, rb, saa, sab, sbb) and its five partial derivatives.
NKX_HD inline void xc_pol(const XcSpec &s, double ra_, double rb_, double saa_, double sab_, double sbb_,
                          double &f, double d[5]) {
  f = 0.0;
  for (int i = 0; i < 5; ++i) d[i] = 0.0;
  if (!(ra_ + rb_ >= s.thr)) return;
  Dual<5> in[5];
  const double base[5] = {fmax(ra_, 1e-30), fmax(rb_, 1e-30), fmax(saa_, 1e-40), sab_, fmax(sbb_, 1e-40)};
  for (int k = 0; k < 5; ++k) {
    in[k].v = base[k];
    for (int j = 0; j < 5; ++j) in[k].d[j] = (j == k) ? 1.0 : 0.0;
  }
  for (int i = 0; i < s.nfunc; ++i) {
    const Dual<5> r = f_total<5>(s.ids[i], in[0], in[1], in[2], in[3], in[4]);
    f += r.v;
    for (int j = 0; j < 5; ++j) d[j] += r.d[j];
  }
}

}  // namespace nkx
