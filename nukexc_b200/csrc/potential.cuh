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
  double za;       // 1 / zeta^a
  double ub;       // (b-1)! / zeta^b, b = n-l+1 (the r -> 0 limit of Gamma(b,.)/zeta^b)
  double xfar;     // far-field switch on zeta r
  int a, b, l, m;
};

#ifdef __CUDACC__
__constant__ const double kInvIntDev[65] = {
    0.0,        1.0 / 1,  1.0 / 2,  1.0 / 3,  1.0 / 4,  1.0 / 5,  1.0 / 6,  1.0 / 7,  1.0 / 8,  1.0 / 9,  1.0 / 10,
    1.0 / 11,   1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20, 1.0 / 21,
    1.0 / 22,   1.0 / 23, 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30, 1.0 / 31, 1.0 / 32,
    1.0 / 33,   1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39, 1.0 / 40, 1.0 / 41, 1.0 / 42, 1.0 / 43,
    1.0 / 44,   1.0 / 45, 1.0 / 46, 1.0 / 47, 1.0 / 48, 1.0 / 49, 1.0 / 50, 1.0 / 51, 1.0 / 52, 1.0 / 53, 1.0 / 54,
    1.0 / 55,   1.0 / 56, 1.0 / 57, 1.0 / 58, 1.0 / 59, 1.0 / 60, 1.0 / 61, 1.0 / 62, 1.0 / 63, 1.0 / 64};
#endif

NKX_HD inline double fact_d(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

// 1/k for k = 0..64 (entry 0 unused): the series below multiply by these
// instead of dividing
NKX_HD inline double inv_int(int k) {
#ifdef __CUDA_ARCH__
  return kInvIntDev[k];
#else
  return 1.0 / k;
#endif
}

// radial factor I(r) of V_a = C S_lm I(r); shared by the 2l+1 functions of a
// shell.  One exp(-x) serves both incomplete gammas: Gamma(b, x) =
// (b-1)! e^-x sum_(k<b) x^k/k!, and gamma(a, x) by its ascending series
// x^a e^-x sum_k x^k / (a (a+1) ... (a+k)) for x < a/2 (ratio below 1/2, so
// a few tens of terms) or as (a-1)! - Gamma(a, x) above, where
// P(a, x) >= P(a, a/2) keeps the subtraction's relative error near 1e-15.
// x^N for a compile-time N
template <int N>
NKX_HD inline double ipow_c(double x) {
  double v = 1.0;
#pragma unroll
  for (int i = 0; i < N; ++i) v *= x;
  return v;
}

// with r^-(2l+1) given, so the shells of one (centre, l) group share it
NKX_HD inline double aux_radial_r(const AuxFunc &f, double r, double r2l1inv) {
  if (r < 1e-12) return f.ub;
  const double x = f.zeta * r;
  if (x > f.xfar) return f.ga_full * r2l1inv;
  const double ex = exp(-x);
  double su = 1.0, t = 1.0;
  for (int k = 1; k < f.b; ++k) {
    t *= x * inv_int(k);
    su += t;
  }
  const double upper = f.ub * ex * su;
  double lower;
  const int a = f.a;
  if (2.0 * x < a) {
    double sum = a <= 64 ? inv_int(a) : 1.0 / a, term = sum;
    for (int k = 1; k < 200; ++k) {
      term *= x * (a + k <= 64 ? inv_int(a + k) : 1.0 / (a + k));
      sum += term;
      if (term < 1e-17 * sum) break;
    }
    lower = ipow(x, a) * ex * sum * f.za;
  } else {
    double sl = 1.0, tl = 1.0;
    for (int k = 1; k < a; ++k) {
      tl *= x * (k <= 64 ? inv_int(k) : 1.0 / k);
      sl += tl;
    }
    lower = f.ga_full * (1.0 - ex * sl);
  }
  return lower * r2l1inv + upper;
}

NKX_HD inline double aux_radial(const AuxFunc &f, double r) {
  return aux_radial_r(f, r, r < 1e-12 ? 0.0 : 1.0 / ipow(r, 2 * f.l + 1));
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

// Complete shells (m = -l..l) of one centre and one l <= 3, consecutive in
// the shell list: the solid harmonics of a point are evaluated once for the
// group.  Groups hold at most kAuxGroupMax(l) shells.
struct AuxGroup {
  double cx, cy, cz;
  int l;
  int first;  // first shell
  int n;      // shells in the group
};
NKX_HD constexpr int aux_group_max(int l) { return (32 / (2 * l + 1)) < 16 ? (32 / (2 * l + 1)) : 16; }

// the 2L+1 real solid harmonics of degree L at (x, y, z), m = -L..L
template <int L>
NKX_HD inline void solid_harmonics_all(double x, double y, double z, double S[2 * L + 1]) {
#pragma unroll
  for (int m = -L; m <= L; ++m) S[m + L] = solid_harmonic(L, m, x, y, z);
}

}  // namespace nkx
