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

// value, gradient and Hessian (h = xx, xy, xz, yy, yz, zz):
// with R(r) = N r^k e^(-zeta r), R' = (k/r - zeta) R, R'' = ((k/r - zeta)^2 - k/r^2) R,
// d_j R = (R'/r) d_j and d_j d_k R = (R'/r) delta_jk + (R'' - R'/r) d_j d_k / r^2;
// phi = R S gives d_j d_k phi = d_j d_k R S + d_j R d_k S + d_k R d_j S + R d_j d_k S.
// The radial derivative terms are dropped at r = 0 (as in sto_value_grad).
NKX_HD inline void sto_value_grad_hess(const StoFunc &f, double px, double py, double pz, double &v, double g[3],
                                       double h[6]) {
  const double d[3] = {px - f.cx, py - f.cy, pz - f.cz};
  const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double R = f.norm * ipow(r, f.k) * exp(-f.zeta * r);
  double s, sg[3], sh[6];
  solid_harmonic_grad(f.l, f.m, d[0], d[1], d[2], s, sg[0], sg[1], sg[2]);
  solid_harmonic_hess(f.l, f.m, d[0], d[1], d[2], sh[0], sh[1], sh[2], sh[3], sh[4], sh[5]);
  double cR = 0.0, dd = 0.0;
  if (r > 0.0) {
    const double a = f.k / r - f.zeta;
    cR = a * R / r;
    dd = ((a * a - f.k / (r * r)) * R - cR) / (r * r);
  }
  v = R * s;
  double dR[3];
  for (int j = 0; j < 3; ++j) {
    dR[j] = cR * d[j];
    g[j] = dR[j] * s + R * sg[j];
  }
  const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  for (int e = 0; e < 6; ++e) {
    const int j = ij[e][0], k = ij[e][1];
    const double d2R = (j == k ? cR : 0.0) + dd * d[j] * d[k];
    h[e] = d2R * s + dR[j] * sg[k] + dR[k] * sg[j] + R * sh[e];
  }
}

// Radial factor cache for consecutive functions of one lane: functions of a
// shell (same centre, zeta and n - l - 1) share r, R(r) and dR/dr / r.
struct RadialCache {
  double cx = 1e300, cy = 0, cz = 0, zeta = -1;
  int k = -1;
  double r, R, cR;
};

// value + gradient reusing the radial factor of the previous call when the
// function shares centre, zeta and k with it (same results as sto_value_grad)
NKX_HD inline void sto_value_grad_cached(const StoFunc &f, double px, double py, double pz, RadialCache &rc,
                                         double &v, double &gx, double &gy, double &gz) {
  const double dx = px - f.cx, dy = py - f.cy, dz = pz - f.cz;
  if (!(f.cx == rc.cx && f.cy == rc.cy && f.cz == rc.cz && f.zeta == rc.zeta && f.k == rc.k)) {
    rc.cx = f.cx;
    rc.cy = f.cy;
    rc.cz = f.cz;
    rc.zeta = f.zeta;
    rc.k = f.k;
    rc.r = sqrt(dx * dx + dy * dy + dz * dz);
    rc.R = ipow(rc.r, f.k) * exp(-f.zeta * rc.r);
    rc.cR = rc.r > 0.0 ? (f.k / rc.r - f.zeta) / rc.r : 0.0;
  }
  const double R = f.norm * rc.R;
  double s, sx, sy, sz;
  solid_harmonic_grad(f.l, f.m, dx, dy, dz, s, sx, sy, sz);
  v = R * s;
  const double cR = rc.cR * R;
  gx = R * sx + s * dx * cR;
  gy = R * sy + s * dy * cR;
  gz = R * sz + s * dz * cR;
}

NKX_HD inline double sto_value_cached(const StoFunc &f, double px, double py, double pz, RadialCache &rc) {
  const double dx = px - f.cx, dy = py - f.cy, dz = pz - f.cz;
  if (!(f.cx == rc.cx && f.cy == rc.cy && f.cz == rc.cz && f.zeta == rc.zeta && f.k == rc.k)) {
    rc.cx = f.cx;
    rc.cy = f.cy;
    rc.cz = f.cz;
    rc.zeta = f.zeta;
    rc.k = f.k;
    rc.r = sqrt(dx * dx + dy * dy + dz * dz);
    rc.R = ipow(rc.r, f.k) * exp(-f.zeta * rc.r);
    rc.cR = 0.0;
  }
  return f.norm * rc.R * solid_harmonic(f.l, f.m, dx, dy, dz);
}

// A radial shell of a function block: the functions sharing centre, zeta and
// n - l - 1 share r^(n-l-1) e^(-zeta r) and its derivative.
struct StoShell {
  double cx, cy, cz, zeta;
  int k, pad;
};

#ifdef __CUDACC__
// One 128-function block in shared memory, laid out for kernels in which lane
// l of a warp evaluates functions 4l .. 4l+3: field[c][l] holds function
// 4l + c, so the 32 reads of one field by a warp are consecutive; sh[c][l]
// is the function's radial shell.  Per point, the lanes of a warp first
// evaluate the radial factor of each of the block's nshell shells once
// (block_radials), then each function combines its shell's factor with its
// solid harmonic (block_funcs_eval4).
struct BlockFuncs {
  double norm[4][32];
  int l[4][32], m[4][32], sh[4][32];
  double scx[128], scy[128], scz[128], szeta[128];
  int sk[128];
  int nshell;
};

// fill B for block I from the plan's tables; the caller synchronises
__device__ inline void load_block_funcs(BlockFuncs &B, const StoFunc *__restrict__ sto,
                                        const int *__restrict__ fshell, const StoShell *__restrict__ bshell,
                                        const int *__restrict__ bnshell, int I, int tid, int nthr) {
  for (int t = tid; t < 128; t += nthr) {
    const int lane = t >> 2, c = t & 3;
    const StoFunc &f = sto[I * 128 + t];
    B.norm[c][lane] = f.norm;
    B.l[c][lane] = f.l;
    B.m[c][lane] = f.m;
    B.sh[c][lane] = fshell[I * 128 + t];
    const StoShell &h = bshell[I * 128 + t];
    B.scx[t] = h.cx;
    B.scy[t] = h.cy;
    B.scz[t] = h.cz;
    B.szeta[t] = h.zeta;
    B.sk[t] = h.k;
  }
  if (tid == 0) B.nshell = bnshell[I];
}

// e^x for -700 <= x <= 0 (0 below) to about 1e-14 relative, for the
// mixed-precision collocation, whose values are rounded to 31 bits anyway:
// Cody-Waite reduction x = n ln2 + t, |t| <= ln2 / 2, with ln 2 split into
// a double and its remainder (the FMAs form x - n ln2 without cancellation
// error), e^t by its Taylor polynomial of degree 11 (truncation below
// (ln2/2)^12 / 12! < 1e-14) and 2^n from the exponent bits.
__device__ __forceinline__ double exp_neg(double x) {
  if (x < -700.0) return 0.0;
  const double n = rint(x * 1.4426950408889634);
  double t = fma(-n, 0x1.62e42fefa39efp-1, x);
  t = fma(-n, 0x1.abc9e3b39803fp-56, t);
  double p = 0x1.ae64567f544e4p-26;  // 1/11!
  p = fma(p, t, 0x1.27e4fb7789f5cp-22);
  p = fma(p, t, 0x1.71de3a556c734p-19);
  p = fma(p, t, 0x1.a01a01a01a01ap-16);
  p = fma(p, t, 0x1.a01a01a01a01ap-13);
  p = fma(p, t, 0x1.6c16c16c16c17p-10);
  p = fma(p, t, 0x1.1111111111111p-7);
  p = fma(p, t, 0x1.5555555555555p-5);
  p = fma(p, t, 0x1.5555555555555p-3);
  p = fma(p, t, 0.5);
  p = fma(p, t, 1.0);
  p = fma(p, t, 1.0);
  return p * __hiloint2double(((int)n + 1023) << 20, 0);
}

// Radial factor cache of sto_value_grad_hess for consecutive functions of
// one thread at one point: functions of a shell share r, 1/r, r^k e^(-zeta r)
// and k/r - zeta (the function's norm scales them).
struct HessRadialCache {
  double cx = 1e300, cy = 0, cz = 0, zeta = -1;
  int k = -1;
  double r = 0, ir = 0, Rn = 0, a = 0;
};

// sto_value_grad_hess with the radial factor shared over a shell's functions
// (rc) and, with FAST, e^x by exp_neg (about 1e-14 relative; the
// mixed-precision gradient); the same formulas, so the results differ from
// sto_value_grad_hess by rounding only.
template <bool FAST>
__device__ __forceinline__ void sto_value_grad_hess_cached(const StoFunc &f, double px, double py, double pz,
                                                           HessRadialCache &rc, double &v, double g[3],
                                                           double h[6]) {
  const double d[3] = {px - f.cx, py - f.cy, pz - f.cz};
  if (!(f.cx == rc.cx && f.cy == rc.cy && f.cz == rc.cz && f.zeta == rc.zeta && f.k == rc.k)) {
    rc.cx = f.cx;
    rc.cy = f.cy;
    rc.cz = f.cz;
    rc.zeta = f.zeta;
    rc.k = f.k;
    rc.r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    rc.ir = rc.r > 0.0 ? 1.0 / rc.r : 0.0;
    rc.Rn = ipow(rc.r, f.k) * (FAST ? exp_neg(-f.zeta * rc.r) : exp(-f.zeta * rc.r));
    rc.a = f.k * rc.ir - f.zeta;
  }
  const double R = f.norm * rc.Rn;
  double s, sg[3], sh[6];
  solid_harmonic_grad(f.l, f.m, d[0], d[1], d[2], s, sg[0], sg[1], sg[2]);
  solid_harmonic_hess(f.l, f.m, d[0], d[1], d[2], sh[0], sh[1], sh[2], sh[3], sh[4], sh[5]);
  double cR = 0.0, dd = 0.0;
  if (rc.r > 0.0) {
    cR = rc.a * R * rc.ir;
    dd = ((rc.a * rc.a - f.k * rc.ir * rc.ir) * R - cR) * (rc.ir * rc.ir);
  }
  v = R * s;
  double dR[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    dR[j] = cR * d[j];
    g[j] = dR[j] * s + R * sg[j];
  }
  const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const int j = ij[e][0], k = ij[e][1];
    const double d2R = (j == k ? cR : 0.0) + dd * d[j] * d[k];
    h[e] = d2R * s + dR[j] * sg[k] + dR[k] * sg[j] + R * sh[e];
  }
}

// radial factors of every shell of the block at one point, shared by the
// warp: R[s] = r^k e^(-zeta r) and, with GRAD, C[s] = (k/r - zeta)/r (0 at r = 0),
// from 1/r = rsqrt(r^2) (1 ulp) and exp_neg
template <bool GRAD>
__device__ __forceinline__ void block_radials(const BlockFuncs &B, int lane, double x, double y, double z,
                                              double *__restrict__ R, double *__restrict__ C) {
  for (int s = lane; s < B.nshell; s += 32) {
    const double dx = x - B.scx[s], dy = y - B.scy[s], dz = z - B.scz[s];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double ri = r2 > 0.0 ? rsqrt(r2) : 0.0;
    const double r = r2 * ri;
    const int k = B.sk[s];
    R[s] = ipow(r, k) * exp_neg(-B.szeta[s] * r);
    if (GRAD) C[s] = (k * ri - B.szeta[s]) * ri;
  }
}

// the four functions of one lane at one point from the warp's radial
// factors: values v[c] and, with GRAD, gradients gx/gy/gz[c]; same arithmetic
// as sto_value(_grad)
template <bool GRAD>
__device__ __forceinline__ void block_funcs_eval4(const BlockFuncs &B, int lane, double x, double y, double z,
                                                  const double *__restrict__ Rs, const double *__restrict__ Cs,
                                                  double v[4], double gx[4], double gy[4], double gz[4]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int s = B.sh[c][lane];
    const double dx = x - B.scx[s], dy = y - B.scy[s], dz = z - B.scz[s];
    const double R = B.norm[c][lane] * Rs[s];
    if (GRAD) {
      double S, sx, sy, sz;
      solid_harmonic_grad(B.l[c][lane], B.m[c][lane], dx, dy, dz, S, sx, sy, sz);
      v[c] = R * S;
      const double cR = Cs[s] * R;
      gx[c] = R * sx + S * dx * cR;
      gy[c] = R * sy + S * dy * cR;
      gz[c] = R * sz + S * dz * cR;
    } else {
      v[c] = R * solid_harmonic(B.l[c][lane], B.m[c][lane], dx, dy, dz);
    }
  }
}
#endif

}  // namespace nkx
