// Drop-in replacement of sto_potential_collocation_scaled
// (nukexc/stopotential.hpp:101-124) over nkx_potential_collocation:
// potential_collocation(alpha, g) = V_alpha(r_g) w_g, N_aux x N_g column-major.
#pragma once

#include "grid.hpp"
#include "stobasis.hpp"

namespace Nukexc {

template <class Space>
void sto_potential_collocation_scaled(const Space space, const STOBasisSet basis, const FlatGrid grid,
                                      DeviceView2DLeft potential_collocation) {
  shim_detail::HostBasis hb(basis);
  nkx_shim::check(nkx_potential_collocation(&hb.c, reinterpret_cast<const double *>(grid.quad_points.data()),
                                            grid.weights.data(), (long)grid.weights.extent(0),
                                            potential_collocation.data(), stream_of(space)),
                  "sto_potential_collocation_scaled");
}

}  // namespace Nukexc
