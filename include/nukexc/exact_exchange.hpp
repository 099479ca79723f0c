// Drop-in replacement of nukexc/exact_exchange.hpp: the grid RI-K
// compute_exact_exchange (:57-119) over nkx_exchange_dense, and its sparse
// (:121-279) and tiled (:281-442) variants, which here form the dense
// collocation of the basis and the weighted aux potentials on the grid
// (fill_collocation, sto_potential_collocation_scaled) and take the same
// dense path, so they suit the small systems the reference's tests use.  As
// in the reference, the occupied orbitals are counted by mo_coeff and the
// tile size only tunes the reference's kernels (validated, no other effect).
#pragma once

#include <string>

#include "octree.hpp"
#include "stopotential.hpp"

namespace Nukexc {

template <class Space>
DeviceView2DLeft compute_exact_exchange(const Space space, const DeviceView2DLeft mo_orbitals,
                                        const DeviceView1D mo_coeff, const DeviceView2DLeft basis_collocation,
                                        const DeviceView2DLeft basis_aux_collocation,
                                        const DeviceView2DLeft potential_collocation_scaled,
                                        const DeviceView2DLeft half_inverse_X) {
  const int nbf = (int)basis_collocation.extent(0);
  const int naux = (int)basis_aux_collocation.extent(0);
  DeviceView2DLeft K("Exchange matrix", nbf, nbf);
  nkx_shim::check(nkx_exchange_dense(nbf, naux, (long)basis_collocation.extent(1), basis_collocation.data(),
                                     potential_collocation_scaled.data(), half_inverse_X.data(),
                                     (int)half_inverse_X.extent(1), (int)mo_coeff.extent(0), mo_orbitals.data(),
                                     mo_coeff.data(), K.data(), stream_of(space)),
                  "compute_exact_exchange");
  return K;
}

namespace shim_detail {
template <class Space>
DeviceView2DLeft exchange_on_grid(const Space &space, const DeviceView2DLeft &mo_orbitals,
                                  const DeviceView1D &mo_coeff, const STOBasisSet &basis,
                                  const STOBasisSet &basis_aux, const FlatGrid &grid,
                                  const DeviceView2DLeft &half_inverse_X) {
  const size_t G = grid.weights.extent(0);
  DeviceView2DLeft phi("Basis collocation", basis.nbf(), G), phi_aux("Aux collocation", basis_aux.nbf(), G),
      vw("Potential collocation", basis_aux.nbf(), G);
  Space sp = space;
  fill_collocation(sp, basis, grid.quad_points, phi);
  sto_potential_collocation_scaled(space, basis_aux, grid, vw);
  return compute_exact_exchange(space, mo_orbitals, mo_coeff, phi, phi_aux, vw, half_inverse_X);
}
}  // namespace shim_detail

template <class Space>
DeviceView2DLeft compute_exact_exchange_sparse(const Space space, const DeviceView2DLeft mo_orbitals,
                                               const DeviceView1D mo_coeff, const STOBasisSet basis,
                                               const STOBasisSet basis_aux, const FlatGrid grid,
                                               const NeighborList nl, const DeviceView2DLeft half_inverse_X) {
  (void)nl;
  return shim_detail::exchange_on_grid(space, mo_orbitals, mo_coeff, basis, basis_aux, grid, half_inverse_X);
}

template <class Space>
DeviceView2DLeft compute_exact_exchange_tiled(const Space space, const DeviceView2DLeft mo_orbitals,
                                              const DeviceView1D mo_coeff, const STOBasisSet basis,
                                              const STOBasisSet basis_aux, const FlatGrid grid,
                                              const NeighborList nl, const DeviceView2DLeft half_inverse_X,
                                              const int tile_size = 32) {
  (void)nl;
  if (tile_size < 1) throw std::runtime_error("compute_exact_exchange_tiled: tile_size must be positive");
  return shim_detail::exchange_on_grid(space, mo_orbitals, mo_coeff, basis, basis_aux, grid, half_inverse_X);
}

}  // namespace Nukexc
