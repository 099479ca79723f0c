// Drop-in replacement of nukexc/grid.hpp for the grid-integration path:
// FlatGrid (:150-160) and make_flat_grid<radial, angular> (:172-348) over
// nkx_make_flat_grid.  The reference's template arguments are IntegratorXX
// quadrature types; here they are the tag types below (same roles: radial
// Treutler-Ahlrichs M4 or Becke, Lebedev angular).
#pragma once

#include <vector>

#include "molecule.hpp"

namespace Nukexc {

struct FlatGrid {
  DeviceArray<Point> quad_points;
  DeviceArray<double> weights;
  DeviceArray<Point> atom_centers;
  DeviceArray<unsigned> Z;
  DeviceArray<int> point_owner;  // owning atom of each point
};

// radial / angular quadrature tags (IntegratorXX::TreutlerAhlrichs,
// IntegratorXX::Becke, IntegratorXX::LebedevLaikov in the reference)
struct TreutlerAhlrichs {
  static constexpr int scheme = NKX_RADIAL_TA;
};
struct BeckeRadial {
  static constexpr int scheme = NKX_RADIAL_BECKE;
};
struct LebedevLaikov {};

constexpr double TA_M4 = 0.6;

enum class RadialSizing { Uniform = NKX_SIZING_UNIFORM, PySCF = NKX_SIZING_PYSCF };

template <typename radial_type, typename angular_type = LebedevLaikov>
FlatGrid make_flat_grid(const Molecule &mol, const size_t nrad = 50, const size_t nang_order = 30,
                        const double weight_threshold = 1e-30, const double ta_alpha = TA_M4,
                        const RadialSizing radial_sizing = RadialSizing::Uniform, double becke_clamp = 5.0) {
  const int na = (int)mol.natoms;
  std::vector<Point> c = nkx_shim::to_host(mol.atom_centers.data(), na);
  std::vector<unsigned> Zu = nkx_shim::to_host(mol.Z.data(), na);
  std::vector<double> xyz(3 * na);
  std::vector<int> Z(na);
  for (int i = 0; i < na; ++i) {
    for (int d = 0; d < 3; ++d) xyz[3 * i + d] = c[i][d];
    Z[i] = (int)Zu[i];
  }
  nkx_molecule m{na, xyz.data(), Z.data()};
  nkx_grid_spec spec{radial_type::scheme, (int)nrad,          (int)nang_order, weight_threshold,
                     ta_alpha,            (int)radial_sizing, becke_clamp};
  long np = 0;
  nkx_shim::check(nkx_make_flat_grid(&m, &spec, &np, nullptr, nullptr, nullptr), "make_flat_grid");
  std::vector<double> pts(3 * (size_t)np), w(np);
  std::vector<int> owner(np);
  nkx_shim::check(nkx_make_flat_grid(&m, &spec, &np, pts.data(), w.data(), owner.data()), "make_flat_grid");
  FlatGrid g;
  g.quad_points = DeviceArray<Point>("quad points", np);
  g.weights = DeviceArray<double>("weights", np);
  g.point_owner = DeviceArray<int>("point owner", np);
  g.atom_centers = mol.atom_centers;
  g.Z = mol.Z;
  auto up = [](void *d, const void *h, size_t bytes) {
    nkx_shim::check_cuda(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
  };
  up(g.quad_points.data(), pts.data(), pts.size() * sizeof(double));
  up(g.weights.data(), w.data(), w.size() * sizeof(double));
  up(g.point_owner.data(), owner.data(), owner.size() * sizeof(int));
  return g;
}

}  // namespace Nukexc
