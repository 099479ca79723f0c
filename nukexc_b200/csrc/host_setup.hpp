// Host-side set-up shared by the C-ABI entry points: basis tables, the
// atom-centred grid generator and the per-element radial data.
#pragma once

#include <cmath>
#include <vector>

#include "potential.cuh"

namespace nkx {

// Treutler-Ahlrichs radial scale xi per element, Z <= 36 (JCP 102, 346
// (1995), Table 1; the reference's TA_XI, nukexc/grid.hpp:98-102).
inline double ta_xi(int Z) {
  static const double t[] = {0.00, 0.8, 0.9, 1.8, 1.4, 1.3, 1.1, 0.9, 0.9, 0.9, 0.9, 1.4, 1.3,
                             1.3,  1.2, 1.1, 1.0, 1.0, 1.0, 1.5, 1.4, 1.3, 1.2, 1.2, 1.2,
                             1.2,  1.2, 1.2, 1.1, 1.1, 1.1, 1.1, 1.0, 0.9, 0.9, 0.9, 0.9};
  return (Z >= 0 && Z < (int)(sizeof(t) / sizeof(t[0]))) ? t[Z] : 1.0;
}

// Bragg-Slater radii in Angstrom (H as modified by Becke, JCP 88, 2547
// (1988); the reference's BECKE_SLATER_RADII, nukexc/grid.hpp:71-96), Z <= 36.
inline double bragg_slater(int Z) {
  static const double t[] = {0.00, 0.35, 0.35, 1.45, 1.05, 0.85, 0.70, 0.65, 0.60, 0.50, 0.35, 1.80, 1.50,
                             1.25, 1.10, 1.00, 1.00, 1.00, 0.70, 2.20, 1.80, 1.60, 1.45, 1.40, 1.35, 1.40,
                             1.35, 1.35, 1.35, 1.35, 1.35, 1.30, 1.25, 1.15, 1.10, 1.00, 0.90};
  return (Z >= 0 && Z < (int)(sizeof(t) / sizeof(t[0]))) ? t[Z] : -1.0;
}

constexpr double kAngToBohr = 1.8897259885681697;  // nukexc/atomic_properties.hpp:49

inline int periodic_row(int Z) {
  if (Z <= 2) return 1;
  if (Z <= 10) return 2;
  if (Z <= 18) return 3;
  if (Z <= 36) return 4;
  if (Z <= 54) return 5;
  if (Z <= 86) return 6;
  return 7;
}

// STO normalisation N = (2 zeta)^(n+1/2) / sqrt((2n)!) (stobasis.hpp:198-201)
inline double sto_norm(int n, double zeta) { return std::pow(2.0 * zeta, n + 0.5) / std::sqrt(fact_d(2 * n)); }

double sto_cutoff(int n, double zeta, double tol);

std::vector<StoFunc> make_sto_table(const nkx_basis &b);
std::vector<AuxFunc> make_aux_table(const nkx_basis &b);
// shells of consecutive functions sharing centre, zeta, n and l with m rising by 1
std::vector<AuxShell> make_aux_shells(const std::vector<AuxFunc> &t);
// groups of complete shells (l <= 3) sharing a centre and l, sorted by l
// (stable); loose receives the indices of the remaining shells
std::vector<AuxGroup> make_aux_groups(const std::vector<AuxShell> &sh, std::vector<int> &loose);
std::vector<double> make_cutoffs(const nkx_basis &b, double tol);

// Lebedev rule of algebraic order >= order: unit vectors (xyz) and weights
// summing to 4 pi.  Returns false if no such rule.
bool lebedev_rule(int order, std::vector<double> &xyz, std::vector<double> &w);

// Radial rule on Chebyshev second-kind nodes with r^2 in the weights.
void radial_rule(int scheme, int n, double R, double alpha, std::vector<double> &r, std::vector<double> &w);

}  // namespace nkx
