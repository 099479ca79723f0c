// Drop-in replacement of the collocation part of nukexc/stobasis.hpp:
// STOFunc (:85-89), STOBasisSet (:54-64), make_manual_basis (:175-225),
// fill_collocation (:494-533) and fill_grad_collocation (:535-584), over
// nkx_fill_collocation.  The basis arrays live on the device like the
// reference's views; the normalisation and cutoff radii are computed by the
// library.
#pragma once

#include <cmath>
#include <vector>

#include "nukexc_config.hpp"

namespace Nukexc {

struct STOFunc {
  int n, l, m;
  double zeta;
  double ox, oy, oz;
};

struct STOBasisSet {
  DeviceArray<int> n, l, m;
  DeviceArray<double> norm, zeta;
  DeviceArray<Point> O;
  DeviceArray<double> cutoff_radii;
  double cutoff_tol = 1e-10;

  size_t nbf() const { return O.extent(0); }
};

namespace shim_detail {
// (2 zeta)^(n + 1/2) / sqrt((2n)!)  (stobasis.hpp:200-201)
inline double sto_norm(int n, double zeta) {
  return std::exp((n + 0.5) * std::log(2.0 * zeta) - 0.5 * std::lgamma(2.0 * n + 1.0));
}

// host SoA copy of a basis, in the form nkx_basis points into
struct HostBasis {
  std::vector<int> n, l, m;
  std::vector<double> zeta, center;
  nkx_basis c{};
  explicit HostBasis(const STOBasisSet &b) {
    const size_t N = b.nbf();
    n = nkx_shim::to_host(b.n.data(), N);
    l = nkx_shim::to_host(b.l.data(), N);
    m = nkx_shim::to_host(b.m.data(), N);
    zeta = nkx_shim::to_host(b.zeta.data(), N);
    std::vector<Point> O = nkx_shim::to_host(b.O.data(), N);
    center.resize(3 * N);
    for (size_t i = 0; i < N; ++i)
      for (int d = 0; d < 3; ++d) center[3 * i + d] = O[i][d];
    c.nbf = (int)N;
    c.n = n.data();
    c.l = l.data();
    c.m = m.data();
    c.zeta = zeta.data();
    c.center = center.data();
    c.cutoff_tol = b.cutoff_tol;
  }
};
}  // namespace shim_detail

inline STOBasisSet make_manual_basis(const std::vector<STOFunc> &funcs, double cutoff_tol = 1e-10) {
  const size_t N = funcs.size();
  STOBasisSet b;
  b.n = DeviceArray<int>("n", N);
  b.l = DeviceArray<int>("l", N);
  b.m = DeviceArray<int>("m", N);
  b.zeta = DeviceArray<double>("zeta", N);
  b.norm = DeviceArray<double>("coeff", N);
  b.O = DeviceArray<Point>(" centers ", N);
  b.cutoff_radii = DeviceArray<double>("cutoff radii", N);
  b.cutoff_tol = cutoff_tol;
  std::vector<int> n(N), l(N), m(N);
  std::vector<double> z(N), nm(N), rc(N);
  std::vector<Point> O(N);
  for (size_t i = 0; i < N; ++i) {
    const STOFunc &f = funcs[i];
    if (f.n < 1 || f.l < 0 || f.l >= f.n || f.m < -f.l || f.m > f.l || !(f.zeta > 0.0))
      throw std::runtime_error("make_manual_basis: invalid STO function");
    n[i] = f.n;
    l[i] = f.l;
    m[i] = f.m;
    z[i] = f.zeta;
    nm[i] = shim_detail::sto_norm(f.n, f.zeta);
    O[i][0] = f.ox;
    O[i][1] = f.oy;
    O[i][2] = f.oz;
    // cutoff radius: largest r with N r^(n-1) e^(-zeta r) >= tol (bisection on
    // the decreasing tail beyond the maximum at r = (n-1)/zeta)
    double lo = (f.n - 1) / f.zeta, hi = lo + 1.0;
    auto g = [&](double r) { return std::log(nm[i]) + (f.n - 1) * std::log(std::max(r, 1e-300)) - f.zeta * r; };
    while (g(hi) > std::log(cutoff_tol)) hi *= 2.0;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      (g(mid) > std::log(cutoff_tol) ? lo : hi) = mid;
    }
    rc[i] = hi;
  }
  auto up = [](void *d, const void *h, size_t bytes) {
    nkx_shim::check_cuda(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
  };
  up(b.n.data(), n.data(), N * sizeof(int));
  up(b.l.data(), l.data(), N * sizeof(int));
  up(b.m.data(), m.data(), N * sizeof(int));
  up(b.zeta.data(), z.data(), N * sizeof(double));
  up(b.norm.data(), nm.data(), N * sizeof(double));
  up(b.O.data(), O.data(), N * sizeof(Point));
  up(b.cutoff_radii.data(), rc.data(), N * sizeof(double));
  return b;
}

// values (nbf x npts, column-major) at the points of a Point view
template <class Space, class PointsView, class ValuesView>
void fill_collocation(Space &space, const STOBasisSet &basis, PointsView collocation_points,
                      ValuesView collocation_values) {
  shim_detail::HostBasis hb(basis);
  nkx_shim::check(nkx_fill_collocation(&hb.c, reinterpret_cast<const double *>(collocation_points.data()),
                                       (long)collocation_points.extent(0), collocation_values.data(), nullptr,
                                       nullptr, nullptr, stream_of(space)),
                  "fill_collocation");
}

template <class Space, class PointsView, class ValuesView>
void fill_grad_collocation(Space &space, const STOBasisSet &basis_set, PointsView &collocation_points,
                           ValuesView &collocation_gx, ValuesView &collocation_gy, ValuesView &collocation_gz) {
  shim_detail::HostBasis hb(basis_set);
  const long G = (long)collocation_points.extent(0);
  // the C ABI fills values and gradients together; the values go to scratch
  ValuesView vals("collocation values (scratch)", hb.c.nbf, G);
  nkx_shim::check(nkx_fill_collocation(&hb.c, reinterpret_cast<const double *>(collocation_points.data()), G,
                                       vals.data(), collocation_gx.data(), collocation_gy.data(),
                                       collocation_gz.data(), stream_of(space)),
                  "fill_grad_collocation");
}

}  // namespace Nukexc
