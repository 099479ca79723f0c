// Device evaluation of Slater-type orbitals and their derivatives.
//
// phi(r) = N |r-O|^(n-l-1) exp(-zeta |r-O|) S_lm(r-O)   (nukexc/stobasis.hpp:379-408)
// grad phi = R grad S + S (dR/dr) (r-O)/|r-O|,  dR/dr = ((n-l-1)/r - zeta) R
// (basis_eval_with_grad, nukexc/stobasis.hpp:599-638).  At r = 0 the radial
// derivative term is dropped (the cusp has no gradient; grid points never
// sit on a nucleus).
#pragma once

#include "common.cuh"

namespace nkx {

#include "solid_harmonics.inc"

struct StoFunc {
  double cx, cy, cz;  // centre
  double zeta, norm;
  int k;              // n - l - 1
  int l, m;
  int pad;
};

NKX_HD inline double ipow(double r, int k) {
  double v = 1.0;
  for (int i = 0; i < k; ++i) v *= r;
  return v;
}

NKX_HD inline double sto_value(const StoFunc &f, double px, double py, double pz) {
  const double dx = px - f.cx, dy = py - f.cy, dz = pz - f.cz;
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double R = f.norm * ipow(r, f.k) * exp(-f.zeta * r);
  return R * solid_harmonic(f.l, f.m, dx, dy, dz);
}

NKX_HD inline void sto_value_grad(const StoFunc &f, double px, double py, double pz, double &v, double &gx,
                                  double &gy, double &gz) {
  const double dx = px - f.cx, dy = py - f.cy, dz = pz - f.cz;
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double R = f.norm * ipow(r, f.k) * exp(-f.zeta * r);
  double s, sx, sy, sz;
  solid_harmonic_grad(f.l, f.m, dx, dy, dz, s, sx, sy, sz);
  v = R * s;
  const double cR = r > 0.0 ? (f.k / r - f.zeta) * R / r : 0.0;
  gx = R * sx + s * dx * cR;
  gy = R * sy + s * dy * cR;
  gz = R * sz + s * dz * cR;
}

}  // namespace nkx
