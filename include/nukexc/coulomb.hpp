// Drop-in replacement of nukexc/coulomb.hpp: compute_coulomb (:56-115) over
// nkx_coulomb_dense, J = Phi diag(v) Phi^T with v = Vw^T X X^T Vw rho
// (basis_aux_collocation is used, as in the reference, only for N_aux); the
// sparse and tiled variants compute_coulomb_sparse (:117-368) and
// compute_coulomb_tiled (:383-689) over the neighbour list's plan with the
// caller's half inverse X (nkx_plan_set_half_inverse + nkx_fock_build, in
// the precision chosen by set_precision / NKX_PRECISION, FP64 by default);
// and the grid Coulomb metric coulomb_overlap_integral_sparse (:691-813) /
// _tiled (:827-958) over nkx_aux_metric.  The tile size of the tiled
// variants is a performance parameter of the reference's kernels; here it is
// validated and has no other effect.
#pragma once

#include "nukexc_config.hpp"
#include "octree.hpp"

namespace Nukexc {

template <class Space>
DeviceView2DLeft compute_coulomb(const Space space, const DeviceView2DLeft mo_orbitals, const DeviceView1D mo_coeff,
                                 const DeviceView2DLeft basis_collocation,
                                 const DeviceView2DLeft basis_aux_collocation,
                                 const DeviceView2DLeft potential_collocation_scaled,
                                 const DeviceView2DLeft half_inverse_X) {
  const int nbf = (int)basis_collocation.extent(0);
  const int naux = (int)basis_aux_collocation.extent(0);
  DeviceView2DLeft J("Coulomb matrix", nbf, nbf);
  nkx_shim::check(nkx_coulomb_dense(nbf, naux, (long)basis_collocation.extent(1), basis_collocation.data(),
                                    potential_collocation_scaled.data(), half_inverse_X.data(),
                                    (int)half_inverse_X.extent(1), (int)mo_orbitals.extent(1), mo_orbitals.data(),
                                    mo_coeff.data(), J.data(), stream_of(space)),
                  "compute_coulomb");
  return J;
}

namespace shim_detail {
template <class Space>
DeviceView2DLeft coulomb_plan(const Space &space, const DeviceView2DLeft &mo_orbitals, const DeviceView1D &mo_coeff,
                              const STOBasisSet &basis, const STOBasisSet &basis_aux, const FlatGrid &grid,
                              const NeighborList &nl, const DeviceView2DLeft &half_inverse_X, const char *where) {
  const size_t nbf = basis.nbf();
  if (half_inverse_X.extent(0) != basis_aux.nbf()) throw std::runtime_error(std::string(where) + ": X is not N_aux x K");
  nkx_plan *p = nl.plans->get(basis, &basis_aux, grid);
  nkx_shim::check(nkx_plan_set_half_inverse(p, (int)half_inverse_X.extent(1), half_inverse_X.data(), NKX_MEM_DEVICE),
                  where);
  DeviceView2DLeft J("Coulomb matrix", nbf, nbf);
  double E = 0.0;
  nkx_shim::check(nkx_fock_build(p, precision(), 1, (int)mo_orbitals.extent(1), mo_orbitals.data(), mo_coeff.data(),
                                 NKX_MEM_DEVICE, 0, &E, nullptr, J.data(), stream_of(space)),
                  where);
  return J;
}

template <class Space>
DeviceView2DLeft aux_metric(const Space &space, const STOBasisSet &basis_aux, const FlatGrid &grid, const char *where) {
  const size_t naux = basis_aux.nbf();
  HostBasis ha(basis_aux);
  DeviceView2DLeft S("Overlap matrix Symmetrized", naux, naux);
  nkx_shim::check(nkx_aux_metric(&ha.c, (long)grid.weights.extent(0),
                                 reinterpret_cast<const double *>(grid.quad_points.data()), grid.weights.data(),
                                 S.data(), stream_of(space)),
                  where);
  return S;
}
}  // namespace shim_detail

template <class Space>
DeviceView2DLeft compute_coulomb_sparse(const Space space, const DeviceView2DLeft mo_orbitals,
                                        const DeviceView1D mo_coeff, const STOBasisSet basis,
                                        const STOBasisSet basis_aux, const FlatGrid grid, const NeighborList nl,
                                        const DeviceView2DLeft half_inverse_X) {
  return shim_detail::coulomb_plan(space, mo_orbitals, mo_coeff, basis, basis_aux, grid, nl, half_inverse_X,
                                   "compute_coulomb_sparse");
}

template <class Space>
DeviceView2DLeft compute_coulomb_tiled(const Space space, const DeviceView2DLeft mo_orbitals,
                                       const DeviceView1D mo_coeff, const STOBasisSet basis,
                                       const STOBasisSet basis_aux, const FlatGrid grid, const NeighborList nl,
                                       const DeviceView2DLeft half_inverse_X, const int tile_size = 32) {
  if (tile_size < 1) throw std::runtime_error("compute_coulomb_tiled: tile_size must be positive");
  return shim_detail::coulomb_plan(space, mo_orbitals, mo_coeff, basis, basis_aux, grid, nl, half_inverse_X,
                                   "compute_coulomb_tiled");
}

template <class Space>
DeviceView2DLeft coulomb_overlap_integral_sparse(const Space space, const STOBasisSet &basis_aux,
                                                 const FlatGrid &grid, const NeighborList nl) {
  (void)nl;
  return shim_detail::aux_metric(space, basis_aux, grid, "coulomb_overlap_integral_sparse");
}

template <class Space>
DeviceView2DLeft coulomb_overlap_integral_tiled(const Space space, const STOBasisSet &basis_aux,
                                                const FlatGrid &grid, const NeighborList nl,
                                                const int tile_size = 32) {
  (void)nl;
  if (tile_size < 1) throw std::runtime_error("coulomb_overlap_integral_tiled: tile_size must be positive");
  return shim_detail::aux_metric(space, basis_aux, grid, "coulomb_overlap_integral_tiled");
}

}  // namespace Nukexc
