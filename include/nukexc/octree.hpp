// Drop-in replacement of nukexc/octree.hpp, the set-up of the reference's
// sparse / tiled path: Box (ArborX::Box<3, double>), create_bounding_boxes
// (:70-144), NeighborList (:279-285), print_neighbor_list_histogram
// (:289-306) and build_neighbor_list (:317-390), over nkx_morton_order and
// nkx_neighbor_list.
//
// As in the reference, create_bounding_boxes permutes grid.quad_points,
// grid.weights and grid.point_owner in place into Morton order (data derived
// from the old point order becomes invalid), and a NeighborList is the CSR of
// the basis functions whose cutoff sphere meets each box, ascending per box.
//
// The sparse functions that take a NeighborList (compute_density_sparse,
// compute_lsda_sparse, compute_coulomb_sparse, ...) run the library's batched
// plan on the same grid: the list carries, besides the reference's fields, the
// plans built for it on first use, one per (basis, aux basis, grid) it is
// used with; copies of the list share them.  The plan screens the basis per
// 256-point batch and 128-function block with the same cutoff radii, so the
// results equal the neighbour-list sums up to the contributions the cutoff
// drops (below the basis cutoff tolerance).
#pragma once

#include <algorithm>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "grid.hpp"
#include "stobasis.hpp"

namespace Nukexc {

// ArborX::Box<3, double> layout: minimum corner, then maximum corner
struct Box {
  Point min_corner, max_corner;
  Point &minCorner() { return min_corner; }
  Point &maxCorner() { return max_corner; }
  const Point &minCorner() const { return min_corner; }
  const Point &maxCorner() const { return max_corner; }
};
static_assert(sizeof(Box) == 6 * sizeof(double), "Box must be six packed doubles");

namespace shim_detail {
// Library plans of one neighbour list, keyed by the device arrays of the
// primary basis, the aux basis (none for XC and density) and the grid.
class SparsePlans {
 public:
  SparsePlans() = default;
  SparsePlans(const SparsePlans &) = delete;
  SparsePlans &operator=(const SparsePlans &) = delete;
  ~SparsePlans() {
    for (Entry &e : entries_) nkx_plan_destroy(e.plan);
  }

  nkx_plan *get(const STOBasisSet &basis, const STOBasisSet *aux, const FlatGrid &grid) {
    const Entry key{basis.zeta.data(), aux ? aux->zeta.data() : nullptr, grid.quad_points.data(),
                    grid.weights.data(), (long)grid.weights.extent(0), nullptr};
    for (const Entry &e : entries_)
      if (e.basis == key.basis && e.aux == key.aux && e.points == key.points && e.weights == key.weights &&
          e.npts == key.npts)
        return e.plan;
    HostBasis hb(basis);
    std::unique_ptr<HostBasis> ha(aux ? new HostBasis(*aux) : nullptr);
    const size_t G = grid.weights.extent(0);
    const std::vector<Point> pts = nkx_shim::to_host(grid.quad_points.data(), G);
    const std::vector<double> w = nkx_shim::to_host(grid.weights.data(), G);
    nkx_plan_options o{};
    o.batch_points = 256;
    o.screen_tol = basis.cutoff_tol;
    o.nfunc = 1;
    o.func_ids[0] = NKX_XC_LDA_X;  // replaced per call (nkx_plan_set_functional)
    o.dens_threshold = 1e-15;
    nkx_plan *p = nullptr;
    nkx_shim::check(nkx_plan_create(nullptr, &hb.c, ha ? &ha->c : nullptr, (long)G,
                                    reinterpret_cast<const double *>(pts.data()), w.data(), nullptr, &o, &p),
                    "sparse plan");
    Entry e = key;
    e.plan = p;
    entries_.push_back(e);
    return p;
  }

 private:
  struct Entry {
    const void *basis, *aux, *points, *weights;
    long npts;
    nkx_plan *plan;
  };
  std::vector<Entry> entries_;
};
}  // namespace shim_detail

// Data structure that will later be used to compute batched Dgemm and scalings
struct NeighborList {
  DeviceArray<int> neighbors;  // flat list of basis function indices
  DeviceArray<int> offsets;    // offsets(i)..offsets(i+1) gives neighbors of box i
  int max_points_per_box = 0;
  int total_points = 0;
  std::shared_ptr<shim_detail::SparsePlans> plans = std::make_shared<shim_detail::SparsePlans>();
};

// Morton-sorts the grid in place and returns the axis-aligned bounds of each
// run of max_points_per_bb consecutive points (the last run may be shorter).
inline DeviceArray<Box> create_bounding_boxes(FlatGrid &grid, const int max_points_per_bb) {
  if (max_points_per_bb <= 0) throw std::runtime_error("create_bounding_boxes: max_points_per_bb must be positive");
  const size_t G = grid.quad_points.extent(0);
  if (G == 0) return DeviceArray<Box>("bounding_boxes", 0);
  std::vector<Point> pts = nkx_shim::to_host(grid.quad_points.data(), G);
  std::vector<long> perm(G);
  nkx_shim::check(nkx_morton_order((long)G, reinterpret_cast<const double *>(pts.data()), perm.data()),
                  "create_bounding_boxes");
  auto permute = [&](auto *d, size_t n) {
    if (!d || n != G) return;
    auto h = nkx_shim::to_host(d, n);
    decltype(h) out(n);
    for (size_t k = 0; k < n; ++k) out[k] = h[perm[k]];
    nkx_shim::check_cuda(cudaMemcpy(d, out.data(), n * sizeof(out[0]), cudaMemcpyHostToDevice), "cudaMemcpy");
  };
  permute(grid.quad_points.data(), G);
  permute(grid.weights.data(), grid.weights.extent(0));
  permute(grid.point_owner.data(), grid.point_owner.extent(0));
  std::vector<Point> sorted(G);
  for (size_t k = 0; k < G; ++k) sorted[k] = pts[perm[k]];
  const size_t nb = (G + max_points_per_bb - 1) / max_points_per_bb;
  std::vector<Box> h(nb);
  for (size_t b = 0; b < nb; ++b) {
    const size_t g0 = b * max_points_per_bb, g1 = std::min(G, g0 + max_points_per_bb);
    Box bx{sorted[g0], sorted[g0]};
    for (size_t g = g0 + 1; g < g1; ++g)
      for (int d = 0; d < 3; ++d) {
        bx.min_corner[d] = std::min(bx.min_corner[d], sorted[g][d]);
        bx.max_corner[d] = std::max(bx.max_corner[d], sorted[g][d]);
      }
    h[b] = bx;
  }
  DeviceArray<Box> boxes("bounding_boxes", nb);
  nkx_shim::check_cuda(cudaMemcpy(boxes.data(), h.data(), nb * sizeof(Box), cudaMemcpyHostToDevice), "cudaMemcpy");
  return boxes;
}

// Histogram of the per-box neighbour counts as a percentage of the basis
// size, printed to stdout (the reference also writes pgfplots files named
// after output_stem; this replacement prints only).
inline void print_neighbor_list_histogram(const NeighborList &neighbor_list, const int num_basis_functions,
                                          const int num_bins = 50,
                                          const std::string &output_stem = "neighbor_histogram") {
  (void)output_stem;
  const std::vector<int> off = nkx_shim::to_host(neighbor_list.offsets.data(), neighbor_list.offsets.extent(0));
  const int num_boxes = (int)off.size() - 1;
  if (num_boxes <= 0 || num_basis_functions <= 0 || num_bins <= 0) return;
  std::vector<long> bins(num_bins, 0);
  for (int b = 0; b < num_boxes; ++b) {
    const double pct = (off[b + 1] - off[b]) * 100.0 / num_basis_functions;
    bins[std::min(num_bins - 1, std::max(0, (int)(pct / 100.0 * num_bins)))]++;
  }
  const long mx = *std::max_element(bins.begin(), bins.end());
  for (int i = 0; i < num_bins; ++i) {
    std::printf("%6.1f-%6.1f%% | %8ld ", 100.0 * i / num_bins, 100.0 * (i + 1) / num_bins, bins[i]);
    const int bar = mx ? (int)(60 * bins[i] / mx) : 0;
    for (int k = 0; k < bar; ++k) std::putchar('#');
    std::putchar('\n');
  }
}

inline void build_neighbor_list(const STOBasisSet basis, const DeviceArray<Box> &bounding_boxes,
                                const int max_points_per_box, const int total_points, NeighborList &neighbor_list,
                                const bool print_histogram = false,
                                const std::string &histogram_stem = "neighbor_histogram") {
  const int N = (int)basis.nbf();
  const long nb = (long)bounding_boxes.extent(0);
  DeviceArray<int> offsets("offsets", nb + 1), neighbors;
  long nnz = 0;
  if (N > 0 && nb > 0) {
    const double *O = reinterpret_cast<const double *>(basis.O.data());
    const double *B = reinterpret_cast<const double *>(bounding_boxes.data());
    nkx_shim::check(nkx_neighbor_list(N, O, basis.cutoff_radii.data(), nb, B, offsets.data(), nullptr, &nnz, nullptr),
                    "build_neighbor_list");
    neighbors = DeviceArray<int>("neighbors", (size_t)nnz);
    if (nnz > 0)
      nkx_shim::check(
          nkx_neighbor_list(N, O, basis.cutoff_radii.data(), nb, B, offsets.data(), neighbors.data(), &nnz, nullptr),
          "build_neighbor_list");
  }
  neighbor_list.neighbors = neighbors;
  neighbor_list.offsets = offsets;
  neighbor_list.max_points_per_box = max_points_per_box;
  neighbor_list.total_points = total_points;
  neighbor_list.plans = std::make_shared<shim_detail::SparsePlans>();
  if (print_histogram) print_neighbor_list_histogram(neighbor_list, N, 50, histogram_stem);
}

}  // namespace Nukexc
