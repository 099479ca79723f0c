// The reference's hydrogen/helium known answers through the drop-in headers
// include/nukexc/*.hpp (no Kokkos): written the way the reference's own tests
// call its functions (tests/test_hydrogen.cxx, tests/test_density.cxx), so
// the same call sites compile against libnkx.so.  Prints one JSON object.
#include <cmath>
#include <cstdio>
#include <vector>

#include "nukexc/coulomb.hpp"
#include "nukexc/density.hpp"
#include "nukexc/grid.hpp"
#include "nukexc/nukexc_utils.hpp"
#include "nukexc/partitioning.hpp"
#include "nukexc/stobasis.hpp"
#include "nukexc/stopotential.hpp"
#include "nukexc/xc_integrals.hpp"

using namespace Nukexc;

// stands in for libxc's xc_func_type: the shims read info->number
struct XcInfo {
  int number;
};
struct XcFunc {
  const XcInfo *info;
};

static double dot_w(const DeviceView1D &a, const DeviceView1D &w) {
  auto ha = nkx_shim::copy_to_host(a), hw = nkx_shim::copy_to_host(w);
  double s = 0.0;
  for (size_t i = 0; i < ha.size(); ++i) s += ha[i] * hw[i];
  return s;
}

int main() {
  ExecSpace space;
  Molecule mol({{0.0, 0.0, 0.0}}, {1u});
  auto basis = make_manual_basis({{1, 0, 0, 1.0, 0.0, 0.0, 0.0}});
  DeviceView2DLeft C("mo", 1, 1);
  DeviceView1D occ("occ", 1);
  nkx_shim::copy_from_host(C, std::vector<double>{1.0});
  nkx_shim::copy_from_host(occ, std::vector<double>{1.0});

  // density: tests/test_density.cxx:109-142 (Becke 100 x L40)
  FlatGrid g40 = make_flat_grid<BeckeRadial>(mol, 100, 40);
  const size_t G40 = g40.weights.extent(0);
  DeviceView2DLeft phi40("phi", 1, G40);
  fill_collocation(space, basis, g40.quad_points, phi40);
  DeviceView1D rho40 = compute_density(phi40, C, occ);
  const double int_rho = dot_w(rho40, g40.weights);

  // XC: tests/test_hydrogen.cxx:815-912 (Becke 100 x L20)
  FlatGrid g = make_flat_grid<BeckeRadial>(mol, 100, 20);
  const size_t G = g.weights.extent(0);
  DeviceView2DLeft phi("phi", 1, G), gx("gx", 1, G), gy("gy", 1, G), gz("gz", 1, G);
  fill_collocation(space, basis, g.quad_points, phi);
  fill_grad_collocation(space, basis, g.quad_points, gx, gy, gz);
  const XcInfo lda_x{1}, pbe_x{101};
  XC_result lda = compute_lda(phi, g.weights, C, occ, XcFunc{&lda_x});
  XC_result pbe = compute_gga(phi, gx, gy, gz, g.weights, C, occ, XcFunc{&pbe_x});
  const double pbe_v00 = nkx_shim::copy_to_host(pbe.potential)[0];

  // open shell: all of the density in the alpha channel
  DeviceView1D occ0("occ beta", 1);
  XC_result_polarized pol = compute_gga_lsda(phi, gx, gy, gz, g.weights, C, occ, C, occ0, XcFunc{&pbe_x});

  // density and sigma: tests/test_density.cxx:252-307 (Becke 200 x L20)
  FlatGrid g2 = make_flat_grid<BeckeRadial>(mol, 200, 20);
  const size_t G2 = g2.weights.extent(0);
  DeviceView2DLeft p2("phi", 1, G2), x2("gx", 1, G2), y2("gy", 1, G2), z2("gz", 1, G2);
  fill_collocation(space, basis, g2.quad_points, p2);
  fill_grad_collocation(space, basis, g2.quad_points, x2, y2, z2);
  DeviceView1D r2("rho", G2), dx("gx", G2), dy("gy", G2), dz("gz", G2), sg("sigma", G2);
  compute_density_and_sigma(p2, x2, y2, z2, C, occ, r2, dx, dy, dz, sg);
  const double int_sigma = dot_w(sg, g2.weights);

  // J: tests/test_hydrogen.cxx:562-631 (5 s-type aux, half inverse thr 1e-4)
  std::vector<STOFunc> auxf;
  for (double z : {0.5, 1.0, 2.0, 3.0, 4.0}) auxf.push_back({1, 0, 0, z, 0.0, 0.0, 0.0});
  auto aux = make_manual_basis(auxf);
  const int NA = (int)auxf.size();
  DeviceView2DLeft phi_aux("phi aux", NA, G), Vw("Vw", NA, G);
  fill_collocation(space, aux, g.quad_points, phi_aux);
  sto_potential_collocation_scaled(space, aux, g, Vw);
  auto hA = nkx_shim::copy_to_host(phi_aux), hV = nkx_shim::copy_to_host(Vw);
  std::vector<double> S((size_t)NA * NA, 0.0);
  for (int a = 0; a < NA; ++a)
    for (int b = 0; b < NA; ++b) {
      double s = 0.0;
      for (size_t k = 0; k < G; ++k) s += hA[a + k * NA] * hV[b + k * NA] + hV[a + k * NA] * hA[b + k * NA];
      S[a + b * NA] = 0.5 * s;
    }
  DeviceView2DLeft Sd("metric", NA, NA);
  nkx_shim::copy_from_host(Sd, S);
  DeviceView2DLeft X = compute_half_inverse(Sd, 1e-4);
  DeviceView2DLeft J = compute_coulomb(space, C, occ, phi, phi_aux, Vw, X);
  const double j00 = nkx_shim::copy_to_host(J)[0];

  // Becke partition of unity on the grid's own points (tests/test_partition.cxx:197-257)
  DeviceView1D ones("ones", G);
  nkx_shim::copy_from_host(ones, std::vector<double>(G, 1.0));
  partition_becke_team(g.atom_centers, g.quad_points, g.point_owner, ones);
  const double w_single = nkx_shim::copy_to_host(ones)[G / 2];

  std::printf(
      "{\"int_rho\": %.17g, \"E_lda_x\": %.17g, \"E_pbe_x\": %.17g, \"V00_pbe_x\": %.17g, \"E_pbe_x_pol\": %.17g, "
      "\"int_sigma\": %.17g, \"J00\": %.17g, \"K\": %d, \"becke_single_atom\": %.17g}\n",
      int_rho, lda.energy, pbe.energy, pbe_v00, pol.energy, int_sigma, j00, (int)X.extent(1), w_single);
  return 0;
}
