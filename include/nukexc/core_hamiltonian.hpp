// Drop-in replacement of nukexc/core_hamiltonian.hpp for the quadrature
// core Hamiltonian: CoreHamiltonianResult (:121-126), compute_core_hamiltonian
// (:133-289) over nkx_core_hamiltonian_dense, and the screened variants
// compute_core_hamiltonian_screened (:320-438), _screened_scratch (:440-601),
// _screened_tiled (:603-958) and _screened_sparse (:960-1155) over the
// neighbour list's plan (nkx_plan_core_hamiltonian: only the significant
// (batch, function block) pairs are integrated; the reference checks its
// screened variants against the unscreened result at 1e-6,
// tests/test_integration.cxx:83-311).  S = sum_g w phi phi^T,
// T = 1/2 sum_g w grad phi . grad phi^T, V = -sum_g w sum_A Z_A /
// (|r - R_A| + 1e-30) phi phi^T, H = T + V.  The SAP nuclear term (use_SAP,
// tabulated screened potentials read from files) is not provided.
#pragma once

#include <string>
#include <vector>

#include "octree.hpp"

namespace Nukexc {

struct CoreHamiltonianResult {
  DeviceView2DLeft overlap;
  DeviceView2DLeft kinetic;
  DeviceView2DLeft nuclear;
  DeviceView2DLeft hamiltonian;  // T + V_n
};

inline CoreHamiltonianResult compute_core_hamiltonian(const STOBasisSet &basis, const FlatGrid &grid,
                                                      const bool use_SAP = false, const std::string &sap_dir = "") {
  (void)sap_dir;
  if (use_SAP) throw std::runtime_error("compute_core_hamiltonian: the SAP nuclear potential is not provided");
  const size_t N = basis.nbf(), na = grid.atom_centers.extent(0);
  shim_detail::HostBasis hb(basis);
  const std::vector<Point> c = nkx_shim::to_host(grid.atom_centers.data(), na);
  const std::vector<unsigned> Zu = nkx_shim::to_host(grid.Z.data(), na);
  std::vector<double> xyz(3 * na);
  std::vector<int> Z(na);
  for (size_t a = 0; a < na; ++a) {
    for (int d = 0; d < 3; ++d) xyz[3 * a + d] = c[a][d];
    Z[a] = (int)Zu[a];
  }
  const nkx_molecule mol{(int)na, xyz.data(), Z.data()};
  CoreHamiltonianResult r;
  r.overlap = DeviceView2DLeft("Overlap", N, N);
  r.kinetic = DeviceView2DLeft("Kinetic", N, N);
  r.nuclear = DeviceView2DLeft("Nuclear", N, N);
  r.hamiltonian = DeviceView2DLeft("Core Hamiltonian", N, N);
  nkx_shim::check(nkx_core_hamiltonian_dense(&hb.c, &mol, reinterpret_cast<const double *>(grid.quad_points.data()),
                                             grid.weights.data(), (long)grid.weights.extent(0), r.overlap.data(),
                                             r.kinetic.data(), r.nuclear.data(), nullptr),
                  "compute_core_hamiltonian");
  const std::vector<double> T = nkx_shim::to_host(r.kinetic.data(), N * N), V = nkx_shim::to_host(r.nuclear.data(), N * N);
  std::vector<double> H(N * N);
  for (size_t e = 0; e < N * N; ++e) H[e] = T[e] + V[e];
  nkx_shim::check_cuda(cudaMemcpy(r.hamiltonian.data(), H.data(), N * N * sizeof(double), cudaMemcpyHostToDevice),
                       "cudaMemcpy");
  return r;
}

namespace shim_detail {
// the screened quadrature over the neighbour list's plan (nkx_plan_core_hamiltonian)
inline CoreHamiltonianResult core_hamiltonian_plan(const STOBasisSet &basis, const FlatGrid &grid,
                                                   const NeighborList &nl, const char *where) {
  const size_t N = basis.nbf(), na = grid.atom_centers.extent(0);
  const std::vector<Point> c = nkx_shim::to_host(grid.atom_centers.data(), na);
  const std::vector<unsigned> Zu = nkx_shim::to_host(grid.Z.data(), na);
  std::vector<double> xyz(3 * na);
  std::vector<int> Z(na);
  for (size_t a = 0; a < na; ++a) {
    for (int d = 0; d < 3; ++d) xyz[3 * a + d] = c[a][d];
    Z[a] = (int)Zu[a];
  }
  const nkx_molecule mol{(int)na, xyz.data(), Z.data()};
  nkx_plan *p = nl.plans->get(basis, nullptr, grid);
  CoreHamiltonianResult r;
  r.overlap = DeviceView2DLeft("Overlap", N, N);
  r.kinetic = DeviceView2DLeft("Kinetic", N, N);
  r.nuclear = DeviceView2DLeft("Nuclear", N, N);
  r.hamiltonian = DeviceView2DLeft("Core Hamiltonian", N, N);
  nkx_shim::check(nkx_plan_core_hamiltonian(p, &mol, r.overlap.data(), r.kinetic.data(), r.nuclear.data(),
                                            NKX_MEM_DEVICE, nullptr),
                  where);
  const std::vector<double> T = nkx_shim::to_host(r.kinetic.data(), N * N), V = nkx_shim::to_host(r.nuclear.data(), N * N);
  std::vector<double> H(N * N);
  for (size_t e = 0; e < N * N; ++e) H[e] = T[e] + V[e];
  nkx_shim::check_cuda(cudaMemcpy(r.hamiltonian.data(), H.data(), N * N * sizeof(double), cudaMemcpyHostToDevice),
                       "cudaMemcpy");
  return r;
}
}  // namespace shim_detail

inline CoreHamiltonianResult compute_core_hamiltonian_screened(const STOBasisSet &basis, const FlatGrid &grid,
                                                               const NeighborList &nl) {
  return shim_detail::core_hamiltonian_plan(basis, grid, nl, "compute_core_hamiltonian_screened");
}

inline CoreHamiltonianResult compute_core_hamiltonian_screened_scratch(const STOBasisSet &basis,
                                                                       const FlatGrid &grid, const NeighborList &nl) {
  return shim_detail::core_hamiltonian_plan(basis, grid, nl, "compute_core_hamiltonian_screened_scratch");
}

template <int MAX_NEIGHBORS_TILE = 8, int MAX_POINTS_PER_TILE = 8>
CoreHamiltonianResult compute_core_hamiltonian_screened_tiled(const STOBasisSet &basis, const FlatGrid &grid,
                                                              const NeighborList &nl) {
  return shim_detail::core_hamiltonian_plan(basis, grid, nl, "compute_core_hamiltonian_screened_tiled");
}

inline CoreHamiltonianResult compute_core_hamiltonian_screened_sparse(const STOBasisSet &basis,
                                                                      const FlatGrid &grid, const NeighborList &nl) {
  return shim_detail::core_hamiltonian_plan(basis, grid, nl, "compute_core_hamiltonian_screened_sparse");
}

}  // namespace Nukexc
