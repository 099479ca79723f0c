// Drop-in replacement of compute_coulomb (nukexc/coulomb.hpp:56-115) over
// nkx_coulomb_dense: J = Phi diag(v) Phi^T with v = Vw^T X X^T Vw rho.
// basis_aux_collocation is used, as in the reference, only for N_aux.
#pragma once

#include "nukexc_config.hpp"

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

}  // namespace Nukexc
