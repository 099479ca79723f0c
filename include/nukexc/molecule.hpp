// Drop-in replacement of nukexc/molecule.hpp (Molecule, :50-92) for the
// grid-integration path: centres (bohr) and atomic numbers on the device.
#pragma once

#include <set>
#include <vector>

#include "nukexc_config.hpp"

namespace Nukexc {

struct Molecule {
  DeviceArray<Point> atom_centers;  // bohr
  DeviceArray<unsigned> Z;
  unsigned natoms = 0;
  std::set<unsigned> element_list;
  unsigned Z_total = 0;

  Molecule() = default;
  Molecule(const std::vector<std::vector<double>> &atom_centers_v, const std::vector<unsigned> &Z_v)
      : atom_centers("Atom centers", Z_v.size()), Z("Atomic numbers", Z_v.size()), natoms((unsigned)Z_v.size()),
        element_list(Z_v.begin(), Z_v.end()) {
    std::vector<Point> c(natoms);
    for (unsigned i = 0; i < natoms; ++i) {
      for (int d = 0; d < 3; ++d) c[i][d] = atom_centers_v.at(i).at(d);
      Z_total += Z_v[i];
    }
    nkx_shim::check_cuda(cudaMemcpy(atom_centers.data(), c.data(), sizeof(Point) * natoms, cudaMemcpyHostToDevice),
                         "cudaMemcpy");
    nkx_shim::check_cuda(cudaMemcpy(Z.data(), Z_v.data(), sizeof(unsigned) * natoms, cudaMemcpyHostToDevice),
                         "cudaMemcpy");
  }
};

}  // namespace Nukexc
