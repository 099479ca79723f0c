// Electrostatic potential of an STO auxiliary function on the device
// (nukexc/stopotential.hpp:45-100, incomplete gamma functions
// nukexc/nukexc_utils.hpp:152-196):
//   V_a(r) = C S_lm(r-A) [gamma(n+l+2, zeta r) / (zeta^(n+l+2) r^(2l+1))
//                         + Gamma(n-l+1, zeta r) / zeta^(n-l+1)]
//   C = 4 pi (2 zeta)^(n+1/2) / (sqrt((2n)!) (2l+1)).
// Beyond zeta r > xfar (chosen per function on the host so that
// e^-x x^(a-1)/(a-1)! < 1e-18) the exponential terms are below rounding and
// the potential is the exact multipole C S_lm (n+l+1)! / (zeta^(n+l+2) r^(2l+1)).
#pragma once

#include "sto.cuh"

namespace nkx {

struct AuxFunc {
  double cx, cy, cz;
  double zeta;
  double C;        // 4 pi N / (2l+1)
  double ga_full;  // (a-1)! / zeta^a, a = n+l+2  (the r -> infinity limit of gamma(a,.)/zeta^a)
  double zb;       // 1 / zeta^b, b = n-l+1
  double xfar;     // far-field switch on zeta r
  int a, b, l, m;
};

NKX_HD inline double fact_d(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

// Gamma(n, x) for integer n >= 1: (n-1)! e^-x sum_{k<n} x^k/k!
NKX_HD inline double upper_gamma_int(int n, double x) {
  double sum = 1.0, term = 1.0;
  for (int k = 1; k < n; ++k) {
    term *= x / k;
    sum += term;
  }
  return fact_d(n - 1) * exp(-x) * sum;
}

// gamma(n, x) for integer n >= 1: ascending series for x < n, else
// (n-1)! - Gamma(n, x) (nukexc_utils.hpp:169-196)
NKX_HD inline double lower_gamma_int(int n, double x) {
  if (x < n) {
    double sum = 1.0 / n, term = 1.0 / n;
    for (int k = 1; k < 1000; ++k) {
      term *= x / (n + k);
      sum += term;
      if (term < 1e-16 * sum) break;
    }
    return exp(n * log(x) - x) * sum;
  }
  return fact_d(n - 1) - upper_gamma_int(n, x);
}

// radial factor I(r) of V_a = C S_lm I(r); shared by the 2l+1 functions of a shell
NKX_HD inline double aux_radial(const AuxFunc &f, double r) {
  if (r < 1e-12) return fact_d(f.b - 1) * f.zb;
  const double zr = f.zeta * r;
  const double r2l1 = ipow(r, 2 * f.l + 1);
  if (zr > f.xfar) return f.ga_full / r2l1;
  return lower_gamma_int(f.a, zr) * (f.ga_full / fact_d(f.a - 1)) / r2l1 + upper_gamma_int(f.b, zr) * f.zb;
}

NKX_HD inline double aux_potential(const AuxFunc &f, double px, double py, double pz) {
  const double dx = px - f.cx, dy = py - f.cy, dz = pz - f.cz;
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  return f.C * solid_harmonic(f.l, f.m, dx, dy, dz) * aux_radial(f, r);
}

// Consecutive aux functions with one centre, zeta, n and l and m running
// m0, m0+1, ... : the radial factor is evaluated once for all of them.
struct AuxShell {
  AuxFunc f;  // the shell's first function (its m is m0)
  int first;  // index of the first function
  int nm;     // number of functions (<= 2l+1)
};

}  // namespace nkx
