// Drop-in replacement of nukexc/density.hpp: compute_density (:150-186, and the
// (basis, grid) overload :55-95) and
// compute_density_and_sigma (:188-255) over nkx_density_dense, and their
// sparse variants compute_density_sparse (:97-148) and
// compute_density_and_sigma_sparse (:261-328) over the neighbour list's plan
// (nkx_plan_density, FP64).  Collocation (nbf x npts) and orbitals
// (nbf x nocc) are column-major device matrices, mo_coeff the occupations.
#pragma once

#include "nukexc_config.hpp"
#include "octree.hpp"

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

// rho on the grid from the basis (density.hpp:55-95): the collocation is
// formed on the grid's points first
inline DeviceView1D compute_density(const STOBasisSet basis, const FlatGrid grid, const DeviceView2DLeft mo_orbitals,
                                    const DeviceView1D mo_coeff) {
  ExecSpace space;
  DeviceView2DLeft phi("collocation", basis.nbf(), grid.weights.extent(0));
  fill_collocation(space, basis, grid.quad_points, phi);
  return compute_density(phi, mo_orbitals, mo_coeff);
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

// rho on the grid (in its current, Morton, order) from the orbitals
inline DeviceView1D compute_density_sparse(const STOBasisSet basis, const FlatGrid grid, const NeighborList nl,
                                           const DeviceView2DLeft mo_orbitals, const DeviceView1D mo_coeff) {
  nkx_plan *p = nl.plans->get(basis, nullptr, grid);
  DeviceView1D rho("density", grid.weights.extent(0));
  nkx_shim::check(nkx_plan_density(p, 1, (int)mo_orbitals.extent(1), mo_orbitals.data(), mo_coeff.data(),
                                   NKX_MEM_DEVICE, 0, rho.data(), nullptr, nullptr, nullptr),
                  "compute_density_sparse");
  return rho;
}

// rho, gx_rho, gy_rho and gz_rho are accumulated into (zero them first, as in
// the reference); sigma is overwritten with |grad rho|^2 of the sums
inline void compute_density_and_sigma_sparse(const STOBasisSet basis, const FlatGrid grid, const NeighborList nl,
                                             const DeviceView2DLeft mo_orbitals, const DeviceView1D mo_coeff,
                                             DeviceView1D rho, DeviceView1D gx_rho, DeviceView1D gy_rho,
                                             DeviceView1D gz_rho, DeviceView1D sigma) {
  nkx_plan *p = nl.plans->get(basis, nullptr, grid);
  const size_t G = grid.weights.extent(0);
  DeviceView1D grad("grad rho", 3 * G);
  const DeviceView1D planes[3] = {gx_rho, gy_rho, gz_rho};
  for (int d = 0; d < 3; ++d)
    nkx_shim::check_cuda(cudaMemcpy(grad.data() + d * G, planes[d].data(), G * sizeof(double),
                                    cudaMemcpyDeviceToDevice),
                         "copy");
  nkx_shim::check(nkx_plan_density(p, 1, (int)mo_orbitals.extent(1), mo_orbitals.data(), mo_coeff.data(),
                                   NKX_MEM_DEVICE, 1, rho.data(), grad.data(), sigma.data(), nullptr),
                  "compute_density_and_sigma_sparse");
  for (int d = 0; d < 3; ++d)
    nkx_shim::check_cuda(cudaMemcpy(planes[d].data(), grad.data() + d * G, G * sizeof(double),
                                    cudaMemcpyDeviceToDevice),
                         "copy");
}

}  // namespace Nukexc
