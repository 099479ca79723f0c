// Drop-in replacement of nukexc/partitioning.hpp: partition_becke_team
// (:126-213, Laqua clamp R_ij = min(|A_i - A_j|, 5)) and partition_becke
// (:63-120, original Becke) over nkx_becke_partition; weights are scaled in
// place by P_owner / sum_i P_i, as in the reference.
#pragma once

#include "nukexc_config.hpp"

namespace Nukexc {

template <class PointView, class IntView, class WeightView>
void partition_becke_team(const PointView &atom_centers, const PointView &quadrature_points,
                          const IntView &point_owner, WeightView &weights) {
  nkx_shim::check(nkx_becke_partition(reinterpret_cast<const double *>(atom_centers.data()),
                                      (int)atom_centers.extent(0),
                                      reinterpret_cast<const double *>(quadrature_points.data()),
                                      point_owner.data(), (long)quadrature_points.extent(0), weights.data(), 5.0,
                                      nullptr),
                  "partition_becke_team");
}

template <class PointView, class IntView, class WeightView>
void partition_becke(const PointView &atom_centers, const PointView &quadrature_points, const IntView &point_owner,
                     WeightView &weights) {
  nkx_shim::check(nkx_becke_partition(reinterpret_cast<const double *>(atom_centers.data()),
                                      (int)atom_centers.extent(0),
                                      reinterpret_cast<const double *>(quadrature_points.data()),
                                      point_owner.data(), (long)quadrature_points.extent(0), weights.data(), 0.0,
                                      nullptr),
                  "partition_becke");
}

}  // namespace Nukexc
