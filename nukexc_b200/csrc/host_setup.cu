// Host-side set-up: basis tables, cutoff radii, Lebedev expansion and
// radial rules (the host half of make_flat_grid, nukexc/grid.hpp:172-287,
// and of make_manual_basis, nukexc/stobasis.hpp:90-225).
#include "host_setup.hpp"

#include <algorithm>
#include <array>

namespace nkx {

#include "lebedev_orbits.inc"

// Radius beyond which N r^(n-1) e^(-zeta r) < tol: root of
// ln N + (n-1) ln r - zeta r - ln tol on the decreasing side of the peak,
// Newton with a bisection safeguard (compute_cutoff, stobasis.hpp:90-173).
double sto_cutoff(int n, double zeta, double tol) {
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
    (g > 0.0 ? lo : hi) = r;
    const double gp = (n - 1) / r - zeta;
    double nx = (gp >= 0.0) ? 0.5 * (lo + hi) : r - g / gp;
    if (nx <= lo || nx >= hi) nx = 0.5 * (lo + hi);
    const double d = std::fabs(nx - r);
    r = nx;
    if (d < 1e-10 * r) break;
  }
  return r;
}

std::vector<StoFunc> make_sto_table(const nkx_basis &b) {
  std::vector<StoFunc> t(b.nbf);
  for (int i = 0; i < b.nbf; ++i) {
    StoFunc &f = t[i];
    f.cx = b.center[3 * i];
    f.cy = b.center[3 * i + 1];
    f.cz = b.center[3 * i + 2];
    f.zeta = b.zeta[i];
    f.norm = sto_norm(b.n[i], b.zeta[i]);
    f.k = b.n[i] - b.l[i] - 1;
    f.l = b.l[i];
    f.m = b.m[i];
    f.pad = 0;
  }
  return t;
}

std::vector<double> make_cutoffs(const nkx_basis &b, double tol) {
  std::vector<double> c(b.nbf);
  for (int i = 0; i < b.nbf; ++i) c[i] = sto_cutoff(b.n[i], b.zeta[i], tol);
  return c;
}

std::vector<AuxFunc> make_aux_table(const nkx_basis &b) {
  std::vector<AuxFunc> t(b.nbf);
  for (int i = 0; i < b.nbf; ++i) {
    AuxFunc &f = t[i];
    const int n = b.n[i], l = b.l[i];
    f.cx = b.center[3 * i];
    f.cy = b.center[3 * i + 1];
    f.cz = b.center[3 * i + 2];
    f.zeta = b.zeta[i];
    f.C = 4.0 * kPi * std::pow(2.0 * f.zeta, n + 0.5) / (std::sqrt(fact_d(2 * n)) * (2 * l + 1));
    f.a = n + l + 2;
    f.b = n - l + 1;
    f.ga_full = fact_d(f.a - 1) / std::pow(f.zeta, f.a);
    f.za = 1.0 / std::pow(f.zeta, f.a);
    f.ub = fact_d(f.b - 1) / std::pow(f.zeta, f.b);
    f.l = l;
    f.m = b.m[i];
    // smallest x with e^-x x^(a-1)/(a-1)! < 1e-18 beyond the peak at a-1
    double x = std::max(1.0, (double)(f.a - 1));
    for (int k = 0; k < 10000; ++k) {
      const double lg = -x + (f.a - 1) * std::log(x) - std::lgamma((double)f.a);
      if (lg < std::log(1e-18)) break;
      x += 0.25;
    }
    f.xfar = x;
  }
  return t;
}

std::vector<AuxShell> make_aux_shells(const std::vector<AuxFunc> &t) {
  std::vector<AuxShell> sh;
  for (int i = 0; i < (int)t.size(); ++i) {
    if (!sh.empty()) {
      AuxShell &s = sh.back();
      const AuxFunc &f = s.f, &g = t[i];
      if (g.cx == f.cx && g.cy == f.cy && g.cz == f.cz && g.zeta == f.zeta && g.a == f.a && g.l == f.l &&
          g.m == f.m + s.nm && g.m <= g.l && s.first + s.nm == i) {
        ++s.nm;
        continue;
      }
    }
    sh.push_back(AuxShell{t[i], i, 1});
  }
  return sh;
}

std::vector<AuxGroup> make_aux_groups(const std::vector<AuxShell> &sh, std::vector<int> &loose) {
  std::vector<AuxGroup> g;
  loose.clear();
  for (int i = 0; i < (int)sh.size(); ++i) {
    const AuxFunc &f = sh[i].f;
    const bool complete = f.l <= 3 && sh[i].nm == 2 * f.l + 1 && f.m == -f.l;
    if (!complete) {
      loose.push_back(i);
      continue;
    }
    if (!g.empty()) {
      AuxGroup &G = g.back();
      if (G.first + G.n == i && G.l == f.l && G.cx == f.cx && G.cy == f.cy && G.cz == f.cz &&
          G.n < aux_group_max(f.l)) {
        ++G.n;
        continue;
      }
    }
    g.push_back(AuxGroup{f.cx, f.cy, f.cz, f.l, i, 1});
  }
  std::stable_sort(g.begin(), g.end(), [](const AuxGroup &a, const AuxGroup &b) { return a.l < b.l; });
  return g;
}

bool lebedev_rule(int order, std::vector<double> &xyz, std::vector<double> &w) {
  int ri = -1;
  for (int i = 0; i < kLebedevNumRules; ++i)
    if (kLebedevIndex[i].order >= order) {
      ri = i;
      break;
    }
  if (ri < 0) return false;
  const LebedevRuleIndex &R = kLebedevIndex[ri];
  xyz.clear();
  w.clear();
  static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (int o = 0; o < R.norbits; ++o) {
    const double *rep = kLebedevOrbits[R.first_orbit + o];
    std::vector<std::array<double, 3>> pts;
    for (const auto &p : perms)
      for (int s = 0; s < 8; ++s) {
        std::array<double, 3> q = {rep[p[0]] * ((s & 1) ? -1.0 : 1.0), rep[p[1]] * ((s & 2) ? -1.0 : 1.0),
                                   rep[p[2]] * ((s & 4) ? -1.0 : 1.0)};
        for (double &c : q)
          if (c == 0.0) c = 0.0;
        if (std::find(pts.begin(), pts.end(), q) == pts.end()) pts.push_back(q);
      }
    for (const auto &q : pts) {
      xyz.insert(xyz.end(), q.begin(), q.end());
      w.push_back(4.0 * kPi * rep[3]);
    }
  }
  return (int)w.size() == R.npts;
}

// scheme 0 (Becke): r = R (1+x)/(1-x); scheme 1 (Treutler-Ahlrichs):
// r = R/ln2 (1+x)^alpha ln(2/(1-x)) (grid.hpp:104-108); nodes
// x_i = cos(i pi/(n+1)); w_i = pi/(n+1) sin(t_i) r'(x_i) r_i^2.
void radial_rule(int scheme, int n, double R, double alpha, std::vector<double> &r, std::vector<double> &w) {
  r.resize(n);
  w.resize(n);
  for (int i = 1; i <= n; ++i) {
    const double t = i * kPi / (n + 1);
    const double x = std::cos(t);
    double ri, dr;
    if (scheme == NKX_RADIAL_BECKE) {
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

}  // namespace nkx
