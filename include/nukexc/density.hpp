// Drop-in replacement of the dense part of nukexc/density.hpp:
// compute_density (:150-186) and compute_density_and_sigma (:188-255) over
// nkx_density_dense.  Collocation (nbf x npts) and orbitals (nbf x nocc) are
// column-major device matrices, mo_coeff the occupations.
#pragma once

#include "nukexc_config.hpp"

namespace Nukexc {

template <class V2, class V1>
V1 compute_density_t(const V2 collocation_values, const V2 mo_orbitals, const V1 mo_coeff) {
  const long G = (long)collocation_values.extent(1);
  V1 rho("density", G);
  nkx_shim::check(nkx_density_dense((int)collocation_values.extent(0), G, collocation_values.data(), nullptr,
                                    nullptr, nullptr, (int)mo_orbitals.extent(1), mo_orbitals.data(),
                                    mo_coeff.data(), rho.data(), nullptr, nullptr, nullptr),
                  "compute_density");
  return rho;
}

inline DeviceView1D compute_density(const DeviceView2DLeft collocation_values, const DeviceView2DLeft mo_orbitals,
                                    const DeviceView1D mo_coeff) {
  return compute_density_t<DeviceView2DLeft, DeviceView1D>(collocation_values, mo_orbitals, mo_coeff);
}

// rho, the three gradient components and sigma = |grad rho|^2, written into
// the caller's views
inline void compute_density_and_sigma(const DeviceView2DLeft collocation_values,
                                      const DeviceView2DLeft collocation_gx, const DeviceView2DLeft collocation_gy,
                                      const DeviceView2DLeft collocation_gz, const DeviceView2DLeft mo_orbitals,
                                      const DeviceView1D mo_coeff, DeviceView1D rho, DeviceView1D gx_rho,
                                      DeviceView1D gy_rho, DeviceView1D gz_rho, DeviceView1D sigma) {
  const long G = (long)collocation_values.extent(1);
  DeviceView1D grad("grad rho", 3 * G);
  nkx_shim::check(nkx_density_dense((int)collocation_values.extent(0), G, collocation_values.data(),
                                    collocation_gx.data(), collocation_gy.data(), collocation_gz.data(),
                                    (int)mo_orbitals.extent(1), mo_orbitals.data(), mo_coeff.data(), rho.data(),
                                    grad.data(), sigma.data(), nullptr),
                  "compute_density_and_sigma");
  nkx_shim::check_cuda(cudaMemcpy(gx_rho.data(), grad.data(), G * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  nkx_shim::check_cuda(cudaMemcpy(gy_rho.data(), grad.data() + G, G * sizeof(double), cudaMemcpyDeviceToDevice),
                       "copy");
  nkx_shim::check_cuda(cudaMemcpy(gz_rho.data(), grad.data() + 2 * G, G * sizeof(double), cudaMemcpyDeviceToDevice),
                       "copy");
}

}  // namespace Nukexc
