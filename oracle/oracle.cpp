// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++/OpenMP FP64 CPU restatement of the NuKEXC grid-integration
// Fock-build algorithms (Kokkos reference, not compilable here: Kokkos,
// KokkosKernels, libxc, IntegratorXX and ArborX are absent).  Only the tests,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this
// library, and only as the checker / the timed CPU baseline.  The product
// (nukexc_b200) never calls it.
//
// Every function cites the reference file:line it restates (paths relative to
// the NuKEXC project root).  Third-party arithmetic the reference delegates
// (IntegratorXX radial/Lebedev grids, libxc functionals, BLAS/LAPACK) is
// restated from the published definitions; see the comments at each site.
//
// Parity pins: the golden values of tests/test_density.cxx,
// tests/test_hydrogen.cxx, tests/test_helium.cxx and tests/test_partition.cxx
// (checked by tests/test_oracle_golden.py).  Correlation functionals
// (VWN5, PBE-C) are not pinned by any reference test.
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../nukexc_b200/csrc/lebedev_orbits.inc"

#define ORC_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Small math helpers (nukexc/nukexc_utils.hpp:49-150)
// ---------------------------------------------------------------------------
double factorial(int n) {  // nukexc_utils.hpp:79-90
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}
double binom(int n, int k) { return factorial(n) / (factorial(k) * factorial(n - k)); }
double int_pow(double r, int k) {  // nukexc_utils.hpp:116-150
  double v = 1.0;
  for (int i = 0; i < k; ++i) v *= r;
  return v;
}

// ---------------------------------------------------------------------------
// Real solid harmonics, generic form (nukexc/spherical_harmonics.hpp:50-102,
// :213-232, gradient :235-347).  S_lm = N_lm * Pi_l^|m|(z, r^2) * A_m or B_|m|
// with A_m + i B_m = (x + i y)^m and
//   Pi = 2^-l sum_k (-1)^k C(l,k) C(2l-2k,l) (l-2k)!/(l-2k-m)! z^(l-2k-m) r^(2k).
// ---------------------------------------------------------------------------
struct Harm {
  double v, gx, gy, gz;
};
Harm solid_harmonic(int l, int m, double x, double y, double z) {
  const int am = std::abs(m);
  const double s = x * x + y * y + z * z;
  double P = 0.0, Ps = 0.0, Pz = 0.0;  // Pi, dPi/ds (s = r^2), dPi/dz
  for (int k = 0; 2 * k <= l - am; ++k) {
    const int p = l - 2 * k - am;
    const double c = ((k % 2) ? -1.0 : 1.0) * std::ldexp(1.0, -l) * binom(l, k) *
                     binom(2 * l - 2 * k, l) * factorial(l - 2 * k) / factorial(l - 2 * k - am);
    P += c * int_pow(z, p) * int_pow(s, k);
    if (k > 0) Ps += c * k * int_pow(z, p) * int_pow(s, k - 1);
    if (p > 0) Pz += c * p * int_pow(z, p - 1) * int_pow(s, k);
  }
  // (x + i y)^am and (x + i y)^(am-1)
  std::complex<double> w(1.0, 0.0), wm1(0.0, 0.0);
  for (int i = 0; i < am; ++i) {
    wm1 = w;
    w *= std::complex<double>(x, y);
  }
  double A, Ax, Ay;
  if (m >= 0) {
    A = w.real();
    Ax = am * wm1.real();
    Ay = -am * wm1.imag();
  } else {
    A = w.imag();
    Ax = am * wm1.imag();
    Ay = am * wm1.real();
  }
  if (m == 0) {
    Ax = Ay = 0.0;
  }
  const double N = (m == 0) ? std::sqrt((2.0 * l + 1.0) / (4.0 * kPi))
                            : std::sqrt((2.0 * l + 1.0) / (2.0 * kPi) * factorial(l - am) / factorial(l + am));
  Harm h;
  h.v = N * P * A;
  h.gx = N * (2.0 * x * Ps * A + P * Ax);
  h.gy = N * (2.0 * y * Ps * A + P * Ay);
  h.gz = N * (2.0 * z * Ps + Pz) * A;
  return h;
}

// ---------------------------------------------------------------------------
// STO basis (nukexc/stobasis.hpp)
// ---------------------------------------------------------------------------
struct Basis {
  int nbf;
  const int *n, *l, *m;
  const double *zeta, *center;  // center: 3*nbf
};
double sto_norm(int n, double zeta) {  // stobasis.hpp:198-201
  return std::pow(2.0 * zeta, n + 0.5) / std::sqrt(factorial(2 * n));
}
// phi and its gradient at (x,y,z) (stobasis.hpp:494-584, :599-638)
void basis_vg(const Basis &b, int mu, double px, double py, double pz, double out[4]) {
  const double dx = px - b.center[3 * mu], dy = py - b.center[3 * mu + 1], dz = pz - b.center[3 * mu + 2];
  const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
  const int k = b.n[mu] - b.l[mu] - 1;
  const double R = sto_norm(b.n[mu], b.zeta[mu]) * int_pow(r, k) * std::exp(-b.zeta[mu] * r);
  const Harm h = solid_harmonic(b.l[mu], b.m[mu], dx, dy, dz);
  out[0] = R * h.v;
  if (r > 0.0) {
    const double cR = (k / r - b.zeta[mu]) * R / r;  // (dR/dr)/r
    out[1] = R * h.gx + h.v * dx * cR;
    out[2] = R * h.gy + h.v * dy * cR;
    out[3] = R * h.gz + h.v * dz * cR;
  } else {
    out[1] = R * h.gx;
    out[2] = R * h.gy;
    out[3] = R * h.gz;
  }
}

// ---------------------------------------------------------------------------
// Exchange-correlation functionals (libxc call sites
// nukexc/xc_integrals.hpp:113, :203, :471, :617).  libxc is absent; the
// energy densities are restated from the published functionals and the
// potentials are obtained by complex-step differentiation (exact to
// rounding for these analytic formulas).
//   1   LDA_X       Dirac/Slater exchange
//   7   LDA_C_VWN   Vosko-Wilk-Nusair 1980, parametrisation V (VWN5)
//   101 GGA_X_PBE   Perdew-Burke-Ernzerhof 1996 exchange
//   130 GGA_C_PBE   PBE correlation on Perdew-Wang 1992 LDA correlation
// f(...) below is the energy per unit volume; exc = f / rho.
// ---------------------------------------------------------------------------
using cplx = std::complex<double>;

cplx cbrt_c(cplx x) { return std::pow(x, 1.0 / 3.0); }

// exp(z) - 1 without cancellation for the complex-step argument a + i b
cplx expm1_c(cplx z) {
  const double a = z.real(), b = z.imag();
  return cplx(std::expm1(a) * std::cos(b) - 2.0 * std::sin(0.5 * b) * std::sin(0.5 * b), std::exp(a) * std::sin(b));
}

// spin-polarised Slater exchange per volume
cplx f_lda_x(cplx ra, cplx rb) {
  const double c = -0.75 * std::cbrt(6.0 / kPi);
  cplx v = 0.0;
  if (ra.real() > 0) v += c * std::pow(ra, 4.0 / 3.0);
  if (rb.real() > 0) v += c * std::pow(rb, 4.0 / 3.0);
  return v;
}

cplx vwn_g(cplx x, double A, double b, double c, double x0) {
  const double Q = std::sqrt(4.0 * c - b * b);
  const cplx X = x * x + b * x + c;
  const double X0 = x0 * x0 + b * x0 + c;
  const cplx at = std::atan(Q / (2.0 * x + b));
  return A * (std::log(x * x / X) + 2.0 * b / Q * at -
              b * x0 / X0 * (std::log((x - x0) * (x - x0) / X) + 2.0 * (b + 2.0 * x0) / Q * at));
}
// f(zeta) from 1 + zeta = 2 ra / rho, 1 - zeta = 2 rb / rho (exact at zeta -> +-1)
cplx fzeta(cplx opz, cplx omz) {
  return (std::pow(opz, 4.0 / 3.0) + std::pow(omz, 4.0 / 3.0) - 2.0) / (std::pow(2.0, 4.0 / 3.0) - 2.0);
}
cplx f_vwn5(cplx ra, cplx rb) {
  const cplx rho = ra + rb;
  const cplx rs = cbrt_c(3.0 / (4.0 * kPi * rho));
  const cplx x = std::sqrt(rs);
  const cplx zeta = (ra - rb) / rho;
  const cplx opz = 2.0 * ra / rho, omz = 2.0 * rb / rho;
  const cplx eP = vwn_g(x, 0.0310907, 3.72744, 12.9352, -0.10498);
  const cplx eF = vwn_g(x, 0.01554535, 7.06042, 18.0578, -0.32500);
  const cplx eA = vwn_g(x, -1.0 / (6.0 * kPi * kPi), 1.13107, 13.0045, -0.0047584);
  const double fpp0 = 4.0 / (9.0 * (std::cbrt(2.0) - 1.0));
  const cplx fz = fzeta(opz, omz);
  const cplx z4 = zeta * zeta * zeta * zeta;
  return rho * (eP + eA * fz / fpp0 * (1.0 - z4) + (eF - eP) * fz * z4);
}

// Perdew-Wang 92 correlation energy per particle (Phys. Rev. B 45, 13244
// (1992), eqs. 8-10 and Table I); mod: the more precise constants of
// libxc's LDA_C_PW_MOD, used inside PBE correlation; otherwise the published
// ones (libxc's LDA_C_PW, the reference driver's default correlation
// lda_c_pw, tests/standalone.cxx:88, standalone_helpers.hpp:191-192)
cplx pw92_g(cplx rs, double A, double a1, double b1, double b2, double b3, double b4) {
  const cplx srs = std::sqrt(rs);
  const cplx den = 2.0 * A * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
  return -2.0 * A * (1.0 + a1 * rs) * std::log(1.0 + 1.0 / den);
}
cplx eps_pw92(cplx rs, cplx zeta, cplx opz, cplx omz, bool mod = true) {
  const cplx gP = pw92_g(rs, mod ? 0.0310907 : 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294);
  const cplx gF = pw92_g(rs, mod ? 0.01554535 : 0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517);
  const cplx gA = pw92_g(rs, mod ? 0.0168869 : 0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671);
  const double fz20 = mod ? 1.709920934161365617563962776245 : 1.709921;
  const cplx fz = fzeta(opz, omz);
  const cplx z4 = zeta * zeta * zeta * zeta;
  return gP - gA * fz / fz20 * (1.0 - z4) + (gF - gP) * fz * z4;
}

cplx f_pw92(cplx ra, cplx rb, bool mod) {
  const cplx rho = ra + rb;
  const cplx rs = cbrt_c(3.0 / (4.0 * kPi * rho));
  return rho * eps_pw92(rs, (ra - rb) / rho, 2.0 * ra / rho, 2.0 * rb / rho, mod);
}

// PBE exchange, unpolarised form per volume of a closed-shell density n
cplx f_pbe_x_unpol(cplx n, cplx s2n) {
  const double kappa = 0.8040, mu = 0.2195149727645171;
  const cplx ex = -0.75 * std::cbrt(3.0 / kPi) * std::pow(n, 4.0 / 3.0);
  const cplx s2 = s2n / (4.0 * std::pow(3.0 * kPi * kPi, 2.0 / 3.0) * std::pow(n, 8.0 / 3.0));
  const cplx Fx = 1.0 + kappa - kappa / (1.0 + mu * s2 / kappa);
  return ex * Fx;
}
cplx f_pbe_x(cplx ra, cplx rb, cplx saa, cplx sbb) {
  cplx v = 0.0;  // spin scaling: Ex[a,b] = (Ex[2a] + Ex[2b]) / 2
  if (ra.real() > 0) v += 0.5 * f_pbe_x_unpol(2.0 * ra, 4.0 * saa);
  if (rb.real() > 0) v += 0.5 * f_pbe_x_unpol(2.0 * rb, 4.0 * sbb);
  return v;
}
cplx f_pbe_c(cplx ra, cplx rb, cplx sigma) {
  const double beta = 0.06672455060314922;
  const double gamma = (1.0 - std::log(2.0)) / (kPi * kPi);
  const cplx rho = ra + rb;
  const cplx zeta = (ra - rb) / rho;
  const cplx opz = 2.0 * ra / rho, omz = 2.0 * rb / rho;
  const cplx rs = cbrt_c(3.0 / (4.0 * kPi * rho));
  const cplx ec = eps_pw92(rs, zeta, opz, omz);
  const cplx phi = 0.5 * (std::pow(opz, 2.0 / 3.0) + std::pow(omz, 2.0 / 3.0));
  const cplx kF = cbrt_c(3.0 * kPi * kPi * rho);
  const cplx ks = std::sqrt(4.0 * kF / kPi);
  const cplx t2 = sigma / (4.0 * phi * phi * ks * ks * rho * rho);
  const cplx phi3 = phi * phi * phi;
  const cplx A = beta / gamma / expm1_c(-ec / (gamma * phi3));
  const cplx At2 = A * t2;
  const cplx H = gamma * phi3 * std::log(1.0 + beta / gamma * t2 * (1.0 + At2) / (1.0 + At2 + At2 * At2));
  return rho * (ec + H);
}

// Total functional value per volume; inputs (ra, rb, saa, sab, sbb).
cplx f_total(int id, const cplx in[5]) {
  switch (id) {
    case 1: return f_lda_x(in[0], in[1]);
    case 7: return f_vwn5(in[0], in[1]);
    case 12: return f_pw92(in[0], in[1], false);
    case 13: return f_pw92(in[0], in[1], true);
    case 101: return f_pbe_x(in[0], in[1], in[2], in[4]);
    case 130: return f_pbe_c(in[0], in[1], in[2] + 2.0 * in[3] + in[4]);
    default: throw std::runtime_error("oracle: unsupported functional id");
  }
}
bool is_gga(int id) { return id == 101 || id == 130; }

// Evaluate one point, polarised layout.  Returns f and the partial
// derivatives d f / d(ra, rb, saa, sab, sbb) by complex step.
void xc_point_pol(int id, double ra, double rb, double saa, double sab, double sbb, double thr, double &f,
                  double d[5]) {
  for (int i = 0; i < 5; ++i) d[i] = 0.0;
  f = 0.0;
  if (ra + rb < thr) return;
  // density floors so spin-resolved formulas stay finite (libxc-like)
  const double zthr = 1e-30;
  ra = std::max(ra, zthr);
  rb = std::max(rb, zthr);
  const double sthr = 1e-40;
  saa = std::max(saa, sthr);
  sbb = std::max(sbb, sthr);
  const double base[5] = {ra, rb, saa, sab, sbb};
  cplx in[5];
  for (int i = 0; i < 5; ++i) in[i] = base[i];
  f = f_total(id, in).real();
  const int nd = is_gga(id) ? 5 : 2;
  for (int i = 0; i < nd; ++i) {
    const double h = 1e-20 * std::max(std::fabs(base[i]), 1e-280);
    for (int j = 0; j < 5; ++j) in[j] = base[j];
    in[i] = cplx(base[i], h);
    d[i] = f_total(id, in).imag() / h;
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

// Number of points of the Lebedev rule of algebraic order >= order
// (IntegratorXX next_algebraic_order / npts_by_algebraic_order, grid.hpp:186-187).
ORC_API int orc_lebedev_npts(int order) {
  for (int i = 0; i < kLebedevNumRules; ++i)
    if (kLebedevIndex[i].order >= order) return kLebedevIndex[i].npts;
  return -1;
}

// Expand the Lebedev rule of order >= `order` into xyz[3*npts], w[npts]
// (weights sum to 4*pi).  Orbit expansion: all signed permutations of the
// representative, deduplicated.
ORC_API int orc_lebedev(int order, double *xyz, double *w) {
  int ri = -1;
  for (int i = 0; i < kLebedevNumRules; ++i)
    if (kLebedevIndex[i].order >= order) {
      ri = i;
      break;
    }
  if (ri < 0) return -1;
  const auto &R = kLebedevIndex[ri];
  int cnt = 0;
  static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (int o = 0; o < R.norbits; ++o) {
    const double *rep = kLebedevOrbits[R.first_orbit + o];
    std::vector<std::array<double, 3>> pts;
    for (auto &p : perms)
      for (int s = 0; s < 8; ++s) {
        std::array<double, 3> q = {rep[p[0]] * ((s & 1) ? -1 : 1), rep[p[1]] * ((s & 2) ? -1 : 1),
                                   rep[p[2]] * ((s & 4) ? -1 : 1)};
        for (auto &c : q)
          if (c == 0.0) c = 0.0;  // fold -0.0
        if (std::find(pts.begin(), pts.end(), q) == pts.end()) pts.push_back(q);
      }
    for (auto &q : pts) {
      xyz[3 * cnt] = q[0];
      xyz[3 * cnt + 1] = q[1];
      xyz[3 * cnt + 2] = q[2];
      w[cnt] = 4.0 * kPi * rep[3];
      ++cnt;
    }
  }
  return cnt;
}

// Radial grids on Chebyshev second-kind nodes x_i = cos(i pi/(n+1)), i=1..n:
//  scheme 0: Becke 1988 mapping r = R (1+x)/(1-x)            (IntegratorXX Becke)
//  scheme 1: Treutler-Ahlrichs r = R/ln2 (1+x)^a ln(2/(1-x)) (grid.hpp:104-108)
// Weights include the r^2 Jacobian: w_i = pi/(n+1) sin(t_i) r'(x_i) r_i^2.
ORC_API void orc_radial(int scheme, int n, double R, double alpha, double *r, double *w) {
  for (int i = 1; i <= n; ++i) {
    const double t = i * kPi / (n + 1);
    const double x = std::cos(t);
    double ri, dr;
    if (scheme == 0) {
      ri = R * (1.0 + x) / (1.0 - x);
      dr = 2.0 * R / ((1.0 - x) * (1.0 - x));
    } else {
      const double c = R / std::log(2.0);
      const double pa = std::pow(1.0 + x, alpha);
      const double lg = std::log(2.0 / (1.0 - x));
      ri = c * pa * lg;
      dr = c * (alpha * std::pow(1.0 + x, alpha - 1.0) * lg + pa / (1.0 - x));
    }
    r[i - 1] = ri;
    w[i - 1] = kPi / (n + 1) * std::sin(t) * dr * ri * ri;
  }
}

// Becke fuzzy-cell weights, Laqua-clamped team variant
// (nukexc/partitioning.hpp:44-55, :126-213): R_ij = min(|A_i-A_j|, 5 bohr),
// mu = clamp((r_i - r_j)/R_ij), P_i = prod_{j!=i} s(p(p(p(mu)))),
// w_g *= P_owner / sum_i P_i.  clamp_R <= 0 selects the unclamped original
// (partitioning.hpp:63-120).
ORC_API void orc_becke(int natoms, const double *centers, int npts, const double *pts, const int *owner,
                       double *weights, double clamp_R) {
  std::vector<double> Rij((size_t)natoms * natoms);
  for (int i = 0; i < natoms; ++i)
    for (int j = 0; j < natoms; ++j) {
      const double dx = centers[3 * i] - centers[3 * j], dy = centers[3 * i + 1] - centers[3 * j + 1],
                   dz = centers[3 * i + 2] - centers[3 * j + 2];
      const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
      Rij[(size_t)i * natoms + j] = clamp_R > 0 ? std::min(d, clamp_R) : d;
    }
#pragma omp parallel
  {
    std::vector<double> r(natoms);
#pragma omp for schedule(static)
    for (int g = 0; g < npts; ++g) {
      for (int i = 0; i < natoms; ++i) {
        const double dx = pts[3 * g] - centers[3 * i], dy = pts[3 * g + 1] - centers[3 * i + 1],
                     dz = pts[3 * g + 2] - centers[3 * i + 2];
        r[i] = std::sqrt(dx * dx + dy * dy + dz * dz);
      }
      double norm = 0.0, wown = 0.0;
      for (int i = 0; i < natoms; ++i) {
        double P = 1.0;
        for (int j = 0; j < natoms; ++j) {
          if (i == j) continue;
          double mu = (r[i] - r[j]) / Rij[(size_t)i * natoms + j];
          mu = mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
          double p = 1.5 * mu - 0.5 * mu * mu * mu;
          p = 1.5 * p - 0.5 * p * p * p;
          p = 1.5 * p - 0.5 * p * p * p;
          P *= 0.5 * (1.0 - p);
        }
        if (i == owner[g]) wown = P;
        norm += P;
      }
      weights[g] *= wown / norm;
    }
  }
}

// Unpartitioned atom-centred grid of make_flat_grid (grid.hpp:172-287):
// radial-outer / angular-inner per atom, translated to the atom, weight =
// radial weight * angular weight.  R_atom is the per-atom radial scale.
// Returns the total point count (query with pts == nullptr).
ORC_API long orc_atom_grids(int natoms, const double *centers, const int *nrad, const double *R_atom,
                            int scheme, double alpha, int ang_order, double *pts, double *w, int *owner) {
  const int nang = orc_lebedev_npts(ang_order);
  if (nang < 0) return -1;
  long total = 0;
  for (int a = 0; a < natoms; ++a) total += (long)nrad[a] * nang;
  if (!pts) return total;
  std::vector<double> axyz(3 * nang), aw(nang);
  orc_lebedev(ang_order, axyz.data(), aw.data());
  long g = 0;
  for (int a = 0; a < natoms; ++a) {
    std::vector<double> r(nrad[a]), rw(nrad[a]);
    orc_radial(scheme, nrad[a], R_atom[a], alpha, r.data(), rw.data());
    for (int i = 0; i < nrad[a]; ++i)
      for (int j = 0; j < nang; ++j, ++g) {
        pts[3 * g] = centers[3 * a] + r[i] * axyz[3 * j];
        pts[3 * g + 1] = centers[3 * a + 1] + r[i] * axyz[3 * j + 1];
        pts[3 * g + 2] = centers[3 * a + 2] + r[i] * axyz[3 * j + 2];
        w[g] = rw[i] * aw[j];
        owner[g] = a;
      }
  }
  return total;
}

// STO cutoff radius: root of ln N + (n-1) ln r - zeta r = ln tol beyond the
// peak, safeguarded Newton (nukexc/stobasis.hpp:90-173).
ORC_API double orc_cutoff(int n, double zeta, double tol) {
  const double norm = sto_norm(n, zeta);
  if (norm <= tol) return 0.0;
  const double lt = std::log(tol), ln = std::log(norm);
  const double peak = n > 1 ? (n - 1) / zeta : 0.0;
  double r = std::max(peak + (ln - lt) / zeta, peak + 1e-6);
  double lo = peak + 1e-10, hi = r;
  for (int k = 0; k < 64; ++k) {
    if (ln + (n - 1) * std::log(hi) - zeta * hi - lt <= 0.0) break;
    hi *= 2.0;
  }
  r = hi;
  for (int k = 0; k < 50; ++k) {
    const double g = ln + (n - 1) * std::log(r) - zeta * r - lt;
    if (g > 0.0)
      lo = r;
    else
      hi = r;
    const double gp = (n - 1) / r - zeta;
    double nx;
    if (gp >= 0.0)
      nx = 0.5 * (lo + hi);
    else {
      nx = r - g / gp;
      if (nx <= lo || nx >= hi) nx = 0.5 * (lo + hi);
    }
    const double d = std::fabs(nx - r);
    r = nx;
    if (d < 1e-10 * r) break;
  }
  return r;
}

ORC_API double orc_sto_norm(int n, double zeta) { return sto_norm(n, zeta); }

ORC_API void orc_solid_harmonic(int l, int m, double x, double y, double z, double *out4) {
  Harm h = solid_harmonic(l, m, x, y, z);
  out4[0] = h.v;
  out4[1] = h.gx;
  out4[2] = h.gy;
  out4[3] = h.gz;
}

// Dense collocation Phi (nbf x npts, column-major like LayoutLeft) and its
// gradient (fill_collocation / fill_grad_collocation, stobasis.hpp:494-584).
// grad may be null.
ORC_API void orc_collocation(int nbf, const int *n, const int *l, const int *m, const double *zeta,
                             const double *center, int npts, const double *pts, double *phi, double *gx,
                             double *gy, double *gz) {
  Basis b{nbf, n, l, m, zeta, center};
#pragma omp parallel for schedule(static)
  for (int g = 0; g < npts; ++g)
    for (int mu = 0; mu < nbf; ++mu) {
      double v[4];
      basis_vg(b, mu, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], v);
      const size_t idx = (size_t)mu + (size_t)g * nbf;
      phi[idx] = v[0];
      if (gx) {
        gx[idx] = v[1];
        gy[idx] = v[2];
        gz[idx] = v[3];
      }
    }
}

// Functional evaluation with libxc's array layouts (xc_lda_exc_vxc /
// xc_gga_exc_vxc): nspin 1: rho[np], sigma[np]; nspin 2: rho[2np] (a,b
// interleaved), sigma[3np] (aa,ab,bb).  exc per particle.
ORC_API void orc_xc_eval(int id, int nspin, int np, const double *rho, const double *sigma, double thr,
                         double *exc, double *vrho, double *vsigma) {
#pragma omp parallel for schedule(static)
  for (int g = 0; g < np; ++g) {
    double f, d[5];
    if (nspin == 1) {
      const double r = rho[g];
      const double s = sigma ? sigma[g] : 0.0;
      // closed shell: ra = rb = r/2, saa = sab = sbb = s/4
      xc_point_pol(id, 0.5 * r, 0.5 * r, 0.25 * s, 0.25 * s, 0.25 * s, thr, f, d);
      exc[g] = r > 0 && f != 0.0 ? f / r : 0.0;
      vrho[g] = 0.5 * (d[0] + d[1]);
      if (vsigma) vsigma[g] = 0.25 * (d[2] + d[3] + d[4]);
    } else {
      const double ra = rho[2 * g], rb = rho[2 * g + 1];
      xc_point_pol(id, ra, rb, sigma ? sigma[3 * g] : 0.0, sigma ? sigma[3 * g + 1] : 0.0,
                   sigma ? sigma[3 * g + 2] : 0.0, thr, f, d);
      exc[g] = (ra + rb) > 0 && f != 0.0 ? f / (ra + rb) : 0.0;
      vrho[2 * g] = d[0];
      vrho[2 * g + 1] = d[1];
      if (vsigma) {
        vsigma[3 * g] = d[2];
        vsigma[3 * g + 1] = d[3];
        vsigma[3 * g + 2] = d[4];
      }
    }
  }
}

// Dense XC build restating compute_lda / compute_gga / compute_lsda /
// compute_gga_lsda (nukexc/xc_integrals.hpp:73-166, :168-261, :424-541,
// :543-726) on explicit points, with a list of functional ids whose outputs
// are summed (the driver calls X and C separately and adds them,
// tests/standalone.cxx:705-720).
//   C: nbf x nocc column-major per spin; occ: nocc per spin.
//   nspin 1: V[nbf*nbf]; nspin 2: V[2*nbf*nbf] (alpha then beta).
// Returns E_xc.  rho_out (npts*nspin) optional.
ORC_API double orc_xc_build(int nbf, const int *n, const int *l, const int *m, const double *zeta,
                            const double *center, int npts, const double *pts, const double *wts, int nfunc,
                            const int *func_ids, int nspin, int nocc, const double *C, const double *occ,
                            double thr, double *V, double *rho_out) {
  Basis b{nbf, n, l, m, zeta, center};
  bool gga = false;
  for (int f = 0; f < nfunc; ++f) gga = gga || is_gga(func_ids[f]);
  const size_t nn = (size_t)nbf * nbf;
  std::fill(V, V + nn * nspin, 0.0);
  double E = 0.0;
  const int BLK = 64;
#pragma omp parallel reduction(+ : E)
  {
    std::vector<double> Vloc(nn * nspin, 0.0);
    std::vector<double> phi((size_t)4 * nbf * BLK), Z((size_t)nspin * nbf * BLK);
#pragma omp for schedule(dynamic, 1)
    for (int g0 = 0; g0 < npts; g0 += BLK) {
      const int gn = std::min(BLK, npts - g0);
      for (int gi = 0; gi < gn; ++gi) {
        const int g = g0 + gi;
        double *ph = &phi[(size_t)4 * nbf * gi];
        for (int mu = 0; mu < nbf; ++mu) {
          double v[4];
          basis_vg(b, mu, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], v);
          ph[mu] = v[0];
          ph[nbf + mu] = v[1];
          ph[2 * nbf + mu] = v[2];
          ph[3 * nbf + mu] = v[3];
        }
        // density and gradient per spin (density.hpp:188-255)
        double rs[2] = {0, 0}, grs[2][3] = {{0, 0, 0}, {0, 0, 0}};
        for (int s = 0; s < nspin; ++s) {
          const double *Cs = C + (size_t)s * nbf * nocc;
          const double *os = occ + (size_t)s * nocc;
          double r = 0, gxs = 0, gys = 0, gzs = 0;
          for (int i = 0; i < nocc; ++i) {
            double t = 0, tx = 0, ty = 0, tz = 0;
            const double *ci = Cs + (size_t)i * nbf;
            for (int mu = 0; mu < nbf; ++mu) {
              t += ci[mu] * ph[mu];
              tx += ci[mu] * ph[nbf + mu];
              ty += ci[mu] * ph[2 * nbf + mu];
              tz += ci[mu] * ph[3 * nbf + mu];
            }
            r += os[i] * t * t;
            gxs += os[i] * tx * t;
            gys += os[i] * ty * t;
            gzs += os[i] * tz * t;
          }
          rs[s] = r;
          grs[s][0] = 2 * gxs;
          grs[s][1] = 2 * gys;
          grs[s][2] = 2 * gzs;
          if (rho_out) rho_out[(size_t)g * nspin + s] = r;
        }
        // functional
        double ra, rb, saa, sab, sbb;
        if (nspin == 1) {
          ra = rb = 0.5 * rs[0];
          const double s = grs[0][0] * grs[0][0] + grs[0][1] * grs[0][1] + grs[0][2] * grs[0][2];
          saa = sab = sbb = 0.25 * s;
        } else {
          ra = rs[0];
          rb = rs[1];
          saa = grs[0][0] * grs[0][0] + grs[0][1] * grs[0][1] + grs[0][2] * grs[0][2];
          sab = grs[0][0] * grs[1][0] + grs[0][1] * grs[1][1] + grs[0][2] * grs[1][2];
          sbb = grs[1][0] * grs[1][0] + grs[1][1] * grs[1][1] + grs[1][2] * grs[1][2];
        }
        double fsum = 0, dsum[5] = {0, 0, 0, 0, 0};
        for (int f = 0; f < nfunc; ++f) {
          double fv, d[5];
          xc_point_pol(func_ids[f], ra, rb, saa, sab, sbb, thr, fv, d);
          fsum += fv;
          for (int k = 0; k < 5; ++k) dsum[k] += d[k];
        }
        E += wts[g] * fsum;
        const double w = wts[g];
        for (int s = 0; s < nspin; ++s) {
          double vr, vec[3] = {0, 0, 0};
          if (nspin == 1) {
            vr = 0.5 * (dsum[0] + dsum[1]);
            const double vs = 0.25 * (dsum[2] + dsum[3] + dsum[4]);
            for (int k = 0; k < 3; ++k) vec[k] = 2.0 * vs * grs[0][k];  // xc_integrals.hpp:506-514
          } else {
            vr = dsum[s];
            const double vss = dsum[s == 0 ? 2 : 4], vab = dsum[3];
            for (int k = 0; k < 3; ++k) vec[k] = 2.0 * vss * grs[s][k] + vab * grs[1 - s][k];  // :655-664
          }
          double *Zs = &Z[(size_t)(s * BLK + gi) * nbf];
          for (int mu = 0; mu < nbf; ++mu) {
            double z = 0.5 * ph[mu] * vr;
            if (gga) z += vec[0] * ph[nbf + mu] + vec[1] * ph[2 * nbf + mu] + vec[2] * ph[3 * nbf + mu];
            Zs[mu] = w * z;
          }
        }
      }
      // V_bar(mu,nu) += sum_g phi(mu,g) Z(nu,g)  (xc_integrals.hpp:145, :520, :700)
      for (int s = 0; s < nspin; ++s) {
        double *Vs = &Vloc[s * nn];
        for (int gi = 0; gi < gn; ++gi) {
          const double *ph = &phi[(size_t)4 * nbf * gi];
          const double *Zs = &Z[(size_t)(s * BLK + gi) * nbf];
          for (int nu = 0; nu < nbf; ++nu) {
            const double z = Zs[nu];
            double *col = Vs + (size_t)nu * nbf;
            for (int mu = 0; mu < nbf; ++mu) col[mu] += ph[mu] * z;
          }
        }
      }
    }
#pragma omp critical
    for (size_t k = 0; k < nn * nspin; ++k) V[k] += Vloc[k];
  }
  // symmetrise V = V_bar + V_bar^T (xc_integrals.hpp:148-153)
  for (int s = 0; s < nspin; ++s) {
    double *Vs = V + s * nn;
    for (int i = 0; i < nbf; ++i)
      for (int j = i; j < nbf; ++j) {
        const double v = Vs[(size_t)i + (size_t)j * nbf] + Vs[(size_t)j + (size_t)i * nbf];
        Vs[(size_t)i + (size_t)j * nbf] = v;
        Vs[(size_t)j + (size_t)i * nbf] = v;
      }
  }
  return E;
}

// ---------------------------------------------------------------------------
// STO potential (nukexc/stopotential.hpp:45-124, gamma functions
// nukexc_utils.hpp:152-196).
// ---------------------------------------------------------------------------
namespace {
double upper_gamma(int n, double x) {  // Gamma(n, x), integer n
  if (n <= 0) return 0.0;
  double sum = 1.0, term = 1.0;
  for (int k = 1; k < n; ++k) {
    term *= x / k;
    sum += term;
  }
  return factorial(n - 1) * std::exp(-x) * sum;
}
double lower_gamma(int n, double x) {  // gamma(n, x), integer n
  if (n <= 0) return 0.0;
  if (x < n) {
    double sum = 1.0 / n, term = 1.0 / n;
    for (int k = 1; k < 1000; ++k) {
      term *= x / (n + k);
      sum += term;
      if (term < 1e-16 * sum) break;
    }
    return std::exp(n * std::log(x) - x) * sum;
  }
  return factorial(n - 1) - upper_gamma(n, x);
}
double I_tilde(int n, int l, double r, double zeta) {
  const int a = n + l + 2, b = n - l + 1;
  if (r < 1e-12) return factorial(b - 1) / std::pow(zeta, b);
  const double zr = zeta * r;
  return lower_gamma(a, zr) / (std::pow(zeta, a) * std::pow(r, 2 * l + 1)) + upper_gamma(b, zr) / std::pow(zeta, b);
}
double sto_potential(int n, int l, int m, double x, double y, double z, double zeta) {
  const double r = std::sqrt(x * x + y * y + z * z);
  const double C = 4.0 * kPi * std::pow(2.0 * zeta, n + 0.5) / (std::sqrt(factorial(2 * n)) * (2 * l + 1));
  return C * solid_harmonic(l, m, x, y, z).v * I_tilde(n, l, r, zeta);
}
}  // namespace

ORC_API double orc_sto_potential(int n, int l, int m, double x, double y, double z, double zeta) {
  return sto_potential(n, l, m, x, y, z, zeta);
}

// Weighted potential collocation Vw(alpha, g) = V_alpha(r_g) w_g, column-major
// naux x npts (sto_potential_collocation_scaled, stopotential.hpp:101-124).
ORC_API void orc_potential_collocation(int naux, const int *n, const int *l, const int *m, const double *zeta,
                                       const double *center, int npts, const double *pts, const double *wts,
                                       double *Vw) {
#pragma omp parallel for schedule(static)
  for (int g = 0; g < npts; ++g)
    for (int a = 0; a < naux; ++a)
      Vw[(size_t)a + (size_t)g * naux] =
          sto_potential(n[a], l[a], m[a], pts[3 * g] - center[3 * a], pts[3 * g + 1] - center[3 * a + 1],
                        pts[3 * g + 2] - center[3 * a + 2], zeta[a]) *
          wts[g];
}

// ---------------------------------------------------------------------------
// Dense linear algebra for the DF metric.
// ---------------------------------------------------------------------------
namespace {
// Cyclic Jacobi eigen-decomposition of a symmetric matrix (column-major).
void jacobi_eigen(int N, std::vector<double> &A, std::vector<double> &lam, std::vector<double> &U) {
  U.assign((size_t)N * N, 0.0);
  for (int i = 0; i < N; ++i) U[(size_t)i * N + i] = 1.0;
  auto a = [&](int i, int j) -> double & { return A[(size_t)i + (size_t)j * N]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        tot += a(i, j) * a(i, j);
        if (i != j) off += a(i, j) * a(i, j);
      }
    if (off <= 1e-30 * tot) break;
    for (int p = 0; p < N - 1; ++p)
      for (int q = p + 1; q < N; ++q) {
        const double apq = a(p, q);
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < N; ++k) {
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < N; ++k) {
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < N; ++k) {
          const double ukp = U[(size_t)k + (size_t)p * N], ukq = U[(size_t)k + (size_t)q * N];
          U[(size_t)k + (size_t)p * N] = c * ukp - s * ukq;
          U[(size_t)k + (size_t)q * N] = s * ukp + c * ukq;
        }
      }
  }
  lam.resize(N);
  for (int i = 0; i < N; ++i) lam[i] = a(i, i);
}
}  // namespace

// Preconditioned half inverse (nukexc/nukexc_utils.hpp:198-270):
// D = sqrt(diag S), A = D^-1 S D^-1, A = U s U^T, keep s > thr,
// X = U_kept s^-1/2 / D.  For a symmetric matrix the SVD's singular values
// are |eigenvalues| with U the eigenvectors; that is used here.  Returns K.
ORC_API int orc_half_inverse(int N, const double *S, double thr, double *X) {
  std::vector<double> D(N), A((size_t)N * N), lam, U;
  for (int i = 0; i < N; ++i) D[i] = std::sqrt(S[(size_t)i * N + i]);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) A[(size_t)i + (size_t)j * N] = S[(size_t)i + (size_t)j * N] / (D[i] * D[j]);
  jacobi_eigen(N, A, lam, U);
  std::vector<int> order(N);
  for (int i = 0; i < N; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return std::fabs(lam[a]) > std::fabs(lam[b]); });
  int K = 0;
  for (int oi = 0; oi < N; ++oi) {
    const int k = order[oi];
    const double s = std::fabs(lam[k]);
    if (s > thr) {
      for (int i = 0; i < N; ++i) X[(size_t)i + (size_t)K * N] = U[(size_t)i + (size_t)k * N] / std::sqrt(s) / D[i];
      ++K;
    }
  }
  return K;
}

// Cholesky solve S c = y (S symmetric positive definite, column-major).
// Returns 0 on success, -1 if not positive definite.
ORC_API int orc_cholesky_solve(int N, const double *S, const double *y, double *c) {
  std::vector<double> L((size_t)N * N, 0.0);
  for (int j = 0; j < N; ++j) {
    double d = S[(size_t)j + (size_t)j * N];
    for (int k = 0; k < j; ++k) d -= L[(size_t)j + (size_t)k * N] * L[(size_t)j + (size_t)k * N];
    if (d <= 0) return -1;
    d = std::sqrt(d);
    L[(size_t)j + (size_t)j * N] = d;
    for (int i = j + 1; i < N; ++i) {
      double s = S[(size_t)i + (size_t)j * N];
      for (int k = 0; k < j; ++k) s -= L[(size_t)i + (size_t)k * N] * L[(size_t)j + (size_t)k * N];
      L[(size_t)i + (size_t)j * N] = s / d;
    }
  }
  std::vector<double> t(N);
  for (int i = 0; i < N; ++i) {
    double s = y[i];
    for (int k = 0; k < i; ++k) s -= L[(size_t)i + (size_t)k * N] * t[k];
    t[i] = s / L[(size_t)i + (size_t)i * N];
  }
  for (int i = N - 1; i >= 0; --i) {
    double s = t[i];
    for (int k = i + 1; k < N; ++k) s -= L[(size_t)k + (size_t)i * N] * c[k];
    c[i] = s / L[(size_t)i + (size_t)i * N];
  }
  return 0;
}

// Aux Coulomb metric (A|B) = 1/2 (Phi_aux Vw^T + transpose) on explicit
// points (tests/test_hydrogen.cxx:604-618, standalone.cxx:452-460).
ORC_API void orc_aux_metric(int naux, const int *n, const int *l, const int *m, const double *zeta,
                            const double *center, int npts, const double *pts, const double *wts, double *S) {
  std::fill(S, S + (size_t)naux * naux, 0.0);
  Basis b{naux, n, l, m, zeta, center};
#pragma omp parallel
  {
    std::vector<double> Sl((size_t)naux * naux, 0.0), ph(naux), vw(naux);
#pragma omp for schedule(static)
    for (int g = 0; g < npts; ++g) {
      for (int a = 0; a < naux; ++a) {
        double v[4];
        basis_vg(b, a, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], v);
        ph[a] = v[0];
        vw[a] = sto_potential(n[a], l[a], m[a], pts[3 * g] - center[3 * a], pts[3 * g + 1] - center[3 * a + 1],
                              pts[3 * g + 2] - center[3 * a + 2], zeta[a]) *
                wts[g];
      }
      for (int j = 0; j < naux; ++j)
        for (int i = 0; i < naux; ++i) Sl[(size_t)i + (size_t)j * naux] += ph[i] * vw[j];
    }
#pragma omp critical
    for (size_t k = 0; k < (size_t)naux * naux; ++k) S[k] += Sl[k];
  }
  for (int i = 0; i < naux; ++i)
    for (int j = i; j < naux; ++j) {
      const double v = 0.5 * (S[(size_t)i + (size_t)j * naux] + S[(size_t)j + (size_t)i * naux]);
      S[(size_t)i + (size_t)j * naux] = S[(size_t)j + (size_t)i * naux] = v;
    }
}

// Dense grid-integrated RI-J (nukexc/coulomb.hpp:56-115):
// rho = density; y = Vw rho; c = X X^T y (X: naux x K) or, when X is null,
// c = S^-1 y by Cholesky of the metric S; v = Vw^T c; J = Phi diag(v) Phi^T.
// C: nbf x nocc, occ[nocc].  Writes J (nbf x nbf) and optionally c[naux].
ORC_API int orc_coulomb(int nbf, const int *n, const int *l, const int *m, const double *zeta, const double *center,
                        int naux, const int *an, const int *al, const int *am, const double *azeta,
                        const double *acenter, int npts, const double *pts, const double *wts, int nocc,
                        const double *C, const double *occ, const double *X, int K, const double *S, double *J,
                        double *c_out) {
  Basis b{nbf, n, l, m, zeta, center};
  std::vector<double> rho(npts), y(naux, 0.0), c(naux, 0.0);
#pragma omp parallel for schedule(static)
  for (int g = 0; g < npts; ++g) {
    std::vector<double> ph(nbf);
    for (int mu = 0; mu < nbf; ++mu) {
      double v[4];
      basis_vg(b, mu, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], v);
      ph[mu] = v[0];
    }
    double r = 0;
    for (int i = 0; i < nocc; ++i) {
      double t = 0;
      for (int mu = 0; mu < nbf; ++mu) t += C[(size_t)i * nbf + mu] * ph[mu];
      r += occ[i] * t * t;
    }
    rho[g] = r;
  }
  auto vpot = [&](int a, int g) {
    return sto_potential(an[a], al[a], am[a], pts[3 * g] - acenter[3 * a], pts[3 * g + 1] - acenter[3 * a + 1],
                         pts[3 * g + 2] - acenter[3 * a + 2], azeta[a]) *
           wts[g];
  };
#pragma omp parallel for schedule(static)
  for (int a = 0; a < naux; ++a) {
    double s = 0;
    for (int g = 0; g < npts; ++g) s += vpot(a, g) * rho[g];
    y[a] = s;
  }
  if (X) {
    std::vector<double> t(K, 0.0);
    for (int k = 0; k < K; ++k)
      for (int a = 0; a < naux; ++a) t[k] += X[(size_t)a + (size_t)k * naux] * y[a];
    for (int a = 0; a < naux; ++a)
      for (int k = 0; k < K; ++k) c[a] += X[(size_t)a + (size_t)k * naux] * t[k];
  } else {
    if (orc_cholesky_solve(naux, S, y.data(), c.data()) != 0) return -1;
  }
  if (c_out)
    for (int a = 0; a < naux; ++a) c_out[a] = c[a];
  std::vector<double> v(npts, 0.0);
#pragma omp parallel for schedule(static)
  for (int g = 0; g < npts; ++g) {
    double s = 0;
    for (int a = 0; a < naux; ++a) s += vpot(a, g) * c[a];
    v[g] = s;
  }
  std::fill(J, J + (size_t)nbf * nbf, 0.0);
#pragma omp parallel
  {
    std::vector<double> Jl((size_t)nbf * nbf, 0.0), ph(nbf);
#pragma omp for schedule(static)
    for (int g = 0; g < npts; ++g) {
      for (int mu = 0; mu < nbf; ++mu) {
        double vv[4];
        basis_vg(b, mu, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], vv);
        ph[mu] = vv[0];
      }
      for (int j = 0; j < nbf; ++j) {
        const double z = ph[j] * v[g];
        for (int i = 0; i < nbf; ++i) Jl[(size_t)i + (size_t)j * nbf] += ph[i] * z;
      }
    }
#pragma omp critical
    for (size_t k = 0; k < (size_t)nbf * nbf; ++k) J[k] += Jl[k];
  }
  return 0;
}
