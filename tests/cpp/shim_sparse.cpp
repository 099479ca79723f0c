// The reference's sparse / tiled path through the drop-in headers
// include/nukexc/*.hpp, called the way its tests call it
// (tests/test_hydrogen.cxx:633-686, :914-952, :994-1073): bounding boxes,
// neighbour lists, the sparse Coulomb metric, half inverse, sparse and tiled
// J; plus sparse density and polarised XC against the dense functions on the
// same (Morton-sorted) grid.  Prints one JSON object.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "nukexc/core_hamiltonian.hpp"
#include "nukexc/coulomb.hpp"
#include "nukexc/density.hpp"
#include "nukexc/exact_exchange.hpp"
#include "nukexc/grid.hpp"
#include "nukexc/nukexc_utils.hpp"
#include "nukexc/octree.hpp"
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

static double max_abs_diff(const std::vector<double> &a, const std::vector<double> &b) {
  double m = 0.0;
  for (size_t i = 0; i < a.size(); ++i) m = std::max(m, std::fabs(a[i] - b[i]));
  return m;
}
static double max_abs(const std::vector<double> &a) {
  double m = 0.0;
  for (double v : a) m = std::max(m, std::fabs(v));
  return m;
}
static DeviceView2DLeft matrix(size_t r, size_t c, const std::vector<double> &colmajor) {
  DeviceView2DLeft m("m", r, c);
  nkx_shim::copy_from_host(m, colmajor);
  return m;
}
static DeviceView1D vec(const std::vector<double> &h) {
  DeviceView1D v("v", h.size());
  nkx_shim::copy_from_host(v, h);
  return v;
}

int main() {
  ExecSpace space;
  const int max_points_per_box = 32;

  // ---- hydrogen 1s self-repulsion, sparse and tiled (test_hydrogen.cxx:633-686, :914-952)
  double J_sparse_h1s = 0.0, J_tiled_h1s = 0.0, K_dense_h1s = 0.0, K_sparse_h1s = 0.0, K_tiled_h1s = 0.0;
  double S00 = 0.0, T00 = 0.0, V00 = 0.0, H00 = 0.0, coreH_screened_diff = 0.0;
  {
    Molecule mol({{0.0, 0.0, 0.0}}, {1u});
    FlatGrid grid = make_flat_grid<BeckeRadial>(mol, 100, 20);
    auto basis = make_manual_basis({{1, 0, 0, 1.0, 0.0, 0.0, 0.0}});
    auto basis_aux = make_manual_basis({{1, 0, 0, 0.5, 0.0, 0.0, 0.0},
                                        {1, 0, 0, 1.0, 0.0, 0.0, 0.0},
                                        {1, 0, 0, 2.0, 0.0, 0.0, 0.0},
                                        {1, 0, 0, 3.0, 0.0, 0.0, 0.0},
                                        {1, 0, 0, 4.0, 0.0, 0.0, 0.0}});
    DeviceView2DLeft mo = matrix(1, 1, {1.0});
    DeviceView1D occ = vec({1.0});
    auto bb = create_bounding_boxes(grid, max_points_per_box);
    NeighborList nl, nl_aux;
    build_neighbor_list(basis, bb, max_points_per_box, (int)grid.quad_points.extent(0), nl);
    build_neighbor_list(basis_aux, bb, max_points_per_box, (int)grid.quad_points.extent(0), nl_aux);
    DeviceView2DLeft S = coulomb_overlap_integral_sparse(space, basis_aux, grid, nl_aux);
    DeviceView2DLeft X = compute_half_inverse(S, 1e-4);
    J_sparse_h1s = nkx_shim::copy_to_host(compute_coulomb_sparse(space, mo, occ, basis, basis_aux, grid, nl, X))[0];
    J_tiled_h1s = nkx_shim::copy_to_host(compute_coulomb_tiled(space, mo, occ, basis, basis_aux, grid, nl, X))[0];
    // self-exchange (test_hydrogen.cxx:688-758, :760-822, :954-992)
    K_sparse_h1s =
        nkx_shim::copy_to_host(compute_exact_exchange_sparse(space, mo, occ, basis, basis_aux, grid, nl, X))[0];
    K_tiled_h1s =
        nkx_shim::copy_to_host(compute_exact_exchange_tiled(space, mo, occ, basis, basis_aux, grid, nl, X))[0];
    const size_t G = grid.weights.extent(0);
    DeviceView2DLeft phi("phi", 1, G), phi_aux("phi aux", 5, G), vw("Vw", 5, G);
    fill_collocation(space, basis, grid.quad_points, phi);
    fill_collocation(space, basis_aux, grid.quad_points, phi_aux);
    sto_potential_collocation_scaled(space, basis_aux, grid, vw);
    K_dense_h1s = nkx_shim::copy_to_host(compute_exact_exchange(space, mo, occ, phi, phi_aux, vw, X))[0];
    // core Hamiltonian of H 1s by quadrature: S = 1, T = 1/2, V = -1
    CoreHamiltonianResult h = compute_core_hamiltonian(basis, grid);
    S00 = nkx_shim::copy_to_host(h.overlap)[0];
    T00 = nkx_shim::copy_to_host(h.kinetic)[0];
    V00 = nkx_shim::copy_to_host(h.nuclear)[0];
    H00 = nkx_shim::copy_to_host(h.hamiltonian)[0];
    const CoreHamiltonianResult hs[4] = {compute_core_hamiltonian_screened(basis, grid, nl),
                                         compute_core_hamiltonian_screened_scratch(basis, grid, nl),
                                         compute_core_hamiltonian_screened_tiled(basis, grid, nl),
                                         compute_core_hamiltonian_screened_sparse(basis, grid, nl)};
    for (const CoreHamiltonianResult &x : hs)
      coreH_screened_diff = std::max(coreH_screened_diff, std::fabs(nkx_shim::copy_to_host(x.hamiltonian)[0] - H00));
  }

  // ---- H2, two s-STOs per atom (test_hydrogen.cxx:994-1073) plus p functions
  Molecule mol({{0.0, 0.0, 0.0}, {0.0, 0.0, 1.4}}, {1u, 1u});
  FlatGrid grid = make_flat_grid<BeckeRadial>(mol, 60, 14);
  const size_t G0 = grid.weights.extent(0);
  const std::vector<double> w_before = nkx_shim::copy_to_host(grid.weights);
  auto basis = make_manual_basis({{1, 0, 0, 1.0, 0.0, 0.0, 0.0},
                                  {1, 0, 0, 1.6, 0.0, 0.0, 0.0},
                                  {2, 1, 0, 1.2, 0.0, 0.0, 0.0},
                                  {1, 0, 0, 1.0, 0.0, 0.0, 1.4},
                                  {1, 0, 0, 1.6, 0.0, 0.0, 1.4},
                                  {2, 1, 1, 1.2, 0.0, 0.0, 1.4}});
  auto basis_aux = make_manual_basis({{1, 0, 0, 0.7, 0.0, 0.0, 0.0},
                                      {1, 0, 0, 2.0, 0.0, 0.0, 0.0},
                                      {1, 0, 0, 0.7, 0.0, 0.0, 1.4},
                                      {1, 0, 0, 2.0, 0.0, 0.0, 1.4}});
  const size_t N = basis.nbf();
  auto bb = create_bounding_boxes(grid, max_points_per_box);
  NeighborList nl, nl_aux;
  build_neighbor_list(basis, bb, max_points_per_box, (int)G0, nl);
  build_neighbor_list(basis_aux, bb, max_points_per_box, (int)G0, nl_aux);

  // boxes hold their points; the weights are a permutation of the old ones
  const std::vector<Point> pts = nkx_shim::copy_to_host(grid.quad_points);
  const std::vector<Box> boxes = nkx_shim::copy_to_host(bb);
  int boxes_ok = boxes.size() == (G0 + max_points_per_box - 1) / max_points_per_box;
  for (size_t g = 0; g < G0 && boxes_ok; ++g) {
    const Box &b = boxes[g / max_points_per_box];
    for (int d = 0; d < 3; ++d)
      if (pts[g][d] < b.min_corner[d] || pts[g][d] > b.max_corner[d]) boxes_ok = 0;
  }
  std::vector<double> w_after = nkx_shim::copy_to_host(grid.weights), wb = w_before;
  std::sort(wb.begin(), wb.end());
  std::sort(w_after.begin(), w_after.end());
  const int weights_permuted = wb == w_after;

  // neighbour list = brute-force sphere-box test, ascending per box
  const std::vector<int> off = nkx_shim::copy_to_host(nl.offsets), nb = nkx_shim::copy_to_host(nl.neighbors);
  const std::vector<Point> O = nkx_shim::copy_to_host(basis.O);
  const std::vector<double> rc = nkx_shim::copy_to_host(basis.cutoff_radii);
  int nl_ok = off.size() == boxes.size() + 1;
  for (size_t b = 0; b < boxes.size() && nl_ok; ++b) {
    std::vector<int> want;
    for (size_t f = 0; f < N; ++f) {
      double d2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double e = std::max({boxes[b].min_corner[d] - O[f][d], 0.0, O[f][d] - boxes[b].max_corner[d]});
        d2 += e * e;
      }
      if (d2 <= rc[f] * rc[f]) want.push_back((int)f);
    }
    const std::vector<int> got(nb.begin() + off[b], nb.begin() + off[b + 1]);
    if (got != want) nl_ok = 0;
  }

  // (A|B) sparse vs tiled(tile=1) and J sparse vs tiled(tile=1), element-wise
  DeviceView2DLeft S = coulomb_overlap_integral_sparse(space, basis_aux, grid, nl_aux);
  DeviceView2DLeft St = coulomb_overlap_integral_tiled(space, basis_aux, grid, nl_aux, 1);
  DeviceView2DLeft X = compute_half_inverse(S, 1e-6);
  DeviceView2DLeft mo = matrix(N, 2, {0.6, 0.3, 0.1, 0.6, 0.3, -0.1, 0.2, -0.1, 0.5, -0.2, 0.1, 0.4});
  DeviceView1D occ = vec({1.0, 0.5});
  DeviceView2DLeft Js = compute_coulomb_sparse(space, mo, occ, basis, basis_aux, grid, nl, X);
  DeviceView2DLeft Jt = compute_coulomb_tiled(space, mo, occ, basis, basis_aux, grid, nl, X, 1);
  const double metric_tiled_vs_sparse = max_abs_diff(nkx_shim::copy_to_host(S), nkx_shim::copy_to_host(St));
  const double J_tiled_vs_sparse = max_abs_diff(nkx_shim::copy_to_host(Js), nkx_shim::copy_to_host(Jt));

  // dense collocations on the same (sorted) grid
  DeviceView2DLeft phi("phi", N, G0), gx("gx", N, G0), gy("gy", N, G0), gz("gz", N, G0);
  fill_collocation(space, basis, grid.quad_points, phi);
  fill_grad_collocation(space, basis, grid.quad_points, gx, gy, gz);
  const size_t NA = basis_aux.nbf();
  DeviceView2DLeft phi_aux("phi aux", NA, G0), vw("Vw", NA, G0);
  fill_collocation(space, basis_aux, grid.quad_points, phi_aux);
  sto_potential_collocation_scaled(space, basis_aux, grid, vw);
  DeviceView2DLeft Jd = compute_coulomb(space, mo, occ, phi, phi_aux, vw, X);
  const double J_sparse_vs_dense = max_abs_diff(nkx_shim::copy_to_host(Js), nkx_shim::copy_to_host(Jd));
  const double J_scale = max_abs(nkx_shim::copy_to_host(Jd));
  // exchange: tiled(tile=1) vs sparse element-wise (test_hydrogen.cxx:994-1073), sparse vs dense
  DeviceView2DLeft Ks = compute_exact_exchange_sparse(space, mo, occ, basis, basis_aux, grid, nl, X);
  DeviceView2DLeft Kt = compute_exact_exchange_tiled(space, mo, occ, basis, basis_aux, grid, nl, X, 1);
  DeviceView2DLeft Kd = compute_exact_exchange(space, mo, occ, phi, phi_aux, vw, X);
  const double K_tiled_vs_sparse = max_abs_diff(nkx_shim::copy_to_host(Ks), nkx_shim::copy_to_host(Kt));
  const double K_sparse_vs_dense = max_abs_diff(nkx_shim::copy_to_host(Ks), nkx_shim::copy_to_host(Kd));
  const double K_scale = max_abs(nkx_shim::copy_to_host(Kd));

  // density: sparse vs dense
  DeviceView1D rho_s = compute_density_sparse(basis, grid, nl, mo, occ);
  DeviceView1D rho_d = compute_density(phi, mo, occ);
  const double rho_sparse_vs_dense = std::max(
      max_abs_diff(nkx_shim::copy_to_host(rho_s), nkx_shim::copy_to_host(rho_d)),
      max_abs_diff(nkx_shim::copy_to_host(compute_density(basis, grid, mo, occ)), nkx_shim::copy_to_host(rho_d)));
  DeviceView1D r2("rho", G0), ax("gx", G0), ay("gy", G0), az("gz", G0), sg("sigma", G0);
  compute_density_and_sigma_sparse(basis, grid, nl, mo, occ, r2, ax, ay, az, sg);
  DeviceView1D r3("rho", G0), bx("gx", G0), by("gy", G0), bz("gz", G0), sd("sigma", G0);
  compute_density_and_sigma(phi, gx, gy, gz, mo, occ, r3, bx, by, bz, sd);
  const double sigma_sparse_vs_dense = max_abs_diff(nkx_shim::copy_to_host(sg), nkx_shim::copy_to_host(sd));
  const double grad_sparse_vs_dense = std::max({max_abs_diff(nkx_shim::copy_to_host(ax), nkx_shim::copy_to_host(bx)),
                                                max_abs_diff(nkx_shim::copy_to_host(ay), nkx_shim::copy_to_host(by)),
                                                max_abs_diff(nkx_shim::copy_to_host(az), nkx_shim::copy_to_host(bz))});
  // accumulation contract: a second call adds the same density again
  compute_density_and_sigma_sparse(basis, grid, nl, mo, occ, r2, ax, ay, az, sg);
  std::vector<double> twice = nkx_shim::copy_to_host(r3);
  for (double &v : twice) v *= 2.0;
  const double rho_accumulated = max_abs_diff(nkx_shim::copy_to_host(r2), twice);
  const double sigma_scale = max_abs(nkx_shim::copy_to_host(sd));

  // polarised XC: sparse vs dense, alpha 2 orbitals, beta 1
  DeviceView2DLeft mo_b = matrix(N, 1, {0.5, 0.2, 0.0, 0.5, 0.2, 0.0});
  DeviceView1D occ_b = vec({1.0});
  DeviceView1D occ_a = vec({1.0, 1.0});
  const XcInfo lda_x{1}, vwn{7}, pbe_x{101}, pbe_c{130};
  const XcInfo *ids[4] = {&lda_x, &vwn, &pbe_x, &pbe_c};
  double xc_dE = 0.0, xc_dV = 0.0, xc_E[4], mixed_dE = 0.0, mixed_dV = 0.0;
  for (int k = 0; k < 4; ++k) {
    XcFunc f{ids[k]};
    XC_result_polarized s, d, m;
    if (k < 2) {
      s = compute_lsda_sparse(basis, grid, nl, mo, occ_a, mo_b, occ_b, f);
      d = compute_lsda(phi, grid.weights, mo, occ_a, mo_b, occ_b, f);
      set_precision(NKX_PREC_MIXED);
      m = compute_lsda_sparse(basis, grid, nl, mo, occ_a, mo_b, occ_b, f);
    } else {
      s = compute_gga_lsda_sparse(basis, grid, nl, mo, occ_a, mo_b, occ_b, f);
      d = compute_gga_lsda(phi, gx, gy, gz, grid.weights, mo, occ_a, mo_b, occ_b, f);
      set_precision(NKX_PREC_MIXED);
      m = compute_gga_lsda_sparse(basis, grid, nl, mo, occ_a, mo_b, occ_b, f);
    }
    set_precision(NKX_PREC_FP64);
    // the tensor-core path selected by set_precision, against the FP64 sparse result
    mixed_dE = std::max(mixed_dE, std::fabs(m.energy - s.energy));
    mixed_dV = std::max({mixed_dV,
                         max_abs_diff(nkx_shim::copy_to_host(m.potential_alpha), nkx_shim::copy_to_host(s.potential_alpha)),
                         max_abs_diff(nkx_shim::copy_to_host(m.potential_beta), nkx_shim::copy_to_host(s.potential_beta))});
    xc_E[k] = s.energy;
    xc_dE = std::max(xc_dE, std::fabs(s.energy - d.energy));
    xc_dV = std::max({xc_dV,
                      max_abs_diff(nkx_shim::copy_to_host(s.potential_alpha), nkx_shim::copy_to_host(d.potential_alpha)),
                      max_abs_diff(nkx_shim::copy_to_host(s.potential_beta), nkx_shim::copy_to_host(d.potential_beta))});
  }
  set_precision(NKX_PREC_MIXED);
  DeviceView2DLeft Jm = compute_coulomb_sparse(space, mo, occ, basis, basis_aux, grid, nl, X);
  set_precision(NKX_PREC_FP64);
  const double J_mixed_vs_fp64 = max_abs_diff(nkx_shim::copy_to_host(Jm), nkx_shim::copy_to_host(Js));
  int family_checked = 0;
  try {
    XcFunc f{&pbe_x};
    compute_lsda_sparse(basis, grid, nl, mo, occ_a, mo_b, occ_b, f);
  } catch (const std::runtime_error &) {
    family_checked = 1;
  }

  std::printf(
      "{\"J_sparse_h1s\": %.17g, \"J_tiled_h1s\": %.17g, \"boxes_ok\": %d, \"weights_permuted\": %d, "
      "\"neighbor_list_ok\": %d, \"nnz\": %zu, \"metric_tiled_vs_sparse\": %.3e, \"J_tiled_vs_sparse\": %.3e, "
      "\"J_sparse_vs_dense\": %.3e, \"J_scale\": %.6g, \"rho_sparse_vs_dense\": %.3e, "
      "\"grad_sparse_vs_dense\": %.3e, \"sigma_sparse_vs_dense\": %.3e, \"sigma_scale\": %.6g, "
      "\"rho_accumulated\": %.3e, \"xc_dE\": %.3e, \"xc_dV\": %.3e, \"E_lda_x\": %.12g, \"E_vwn\": %.12g, "
      "\"E_pbe_x\": %.12g, \"E_pbe_c\": %.12g, \"family_checked\": %d, \"K_dense_h1s\": %.17g, "
      "\"K_sparse_h1s\": %.17g, \"K_tiled_h1s\": %.17g, \"K_tiled_vs_sparse\": %.3e, \"K_sparse_vs_dense\": %.3e, "
      "\"K_scale\": %.6g, \"S00\": %.17g, \"T00\": %.17g, \"V00\": %.17g, \"H00\": %.17g, "
      "\"coreH_screened_diff\": %.3e, \"mixed_dE\": %.3e, \"mixed_dV\": %.3e, \"J_mixed_vs_fp64\": %.3e}\n",
      J_sparse_h1s, J_tiled_h1s, boxes_ok, weights_permuted, nl_ok, nb.size(), metric_tiled_vs_sparse,
      J_tiled_vs_sparse, J_sparse_vs_dense, J_scale, rho_sparse_vs_dense, grad_sparse_vs_dense, sigma_sparse_vs_dense,
      sigma_scale, rho_accumulated, xc_dE, xc_dV, xc_E[0], xc_E[1], xc_E[2], xc_E[3], family_checked, K_dense_h1s,
      K_sparse_h1s, K_tiled_h1s, K_tiled_vs_sparse, K_sparse_vs_dense, K_scale, S00, T00, V00, H00,
      coreH_screened_diff, mixed_dE, mixed_dV, J_mixed_vs_fp64);
  return 0;
}
