// Box neighbour lists of the reference's sparse path (build_neighbor_list,
// nukexc/octree.hpp:317-390): for every box of consecutive grid points, the
// ascending indices of the basis functions whose cutoff sphere
// (centre O_mu, radius r_mu) meets the box's axis-aligned bounds.  The
// reference queries an ArborX BVH and sorts each list; here one warp scans
// the functions of one box in index order, 32 at a time, so the list comes
// out sorted by construction: a ballot of the 32 sphere-box tests gives each
// hit its slot (popc of the lower lanes).  Two passes: counts, then (after
// the CSR offsets) the indices.
#include <cuda_runtime.h>

#include <functional>
#include <vector>

#include "common.cuh"

namespace nkx {

nkx_status run_guarded(const char *where, const std::function<void()> &fn);

// sphere-box test of ArborX::intersects(Sphere, Box): the squared distance
// from the centre to the box (0 inside) is at most r^2
__device__ __forceinline__ bool sphere_meets_box(const double *__restrict__ c, double r,
                                                 const double *__restrict__ box) {
  double d2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = box[d], hi = box[3 + d];
    const double e = c[d] < lo ? lo - c[d] : (c[d] > hi ? c[d] - hi : 0.0);
    d2 += e * e;
  }
  return d2 <= r * r;
}

// one warp per box; with out == NULL the hit count goes to count[b],
// otherwise the hits are written from out + offsets[b]
__global__ void neighbor_kernel(int nfunc, const double *__restrict__ centers, const double *__restrict__ radii,
                                long nboxes, const double *__restrict__ boxes, const int *__restrict__ offsets,
                                int *__restrict__ count, int *__restrict__ out) {
  const long b = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= nboxes) return;
  double box[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) box[k] = boxes[6 * b + k];
  int n = 0;
  int *dst = out ? out + offsets[b] : nullptr;
  for (int f0 = 0; f0 < nfunc; f0 += 32) {
    const int f = f0 + lane;
    const bool hit = f < nfunc && sphere_meets_box(centers + 3 * (size_t)f, radii[f], box);
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (dst && hit) dst[n + __popc(m & ((1u << lane) - 1u))] = f;
    n += __popc(m);
  }
  if (!out && lane == 0) count[b] = n;
}

}  // namespace nkx

using namespace nkx;

extern "C" NKX_API nkx_status nkx_neighbor_list(int nfunc, const double *d_centers, const double *d_radii,
                                                long nboxes, const double *d_boxes, int *d_offsets, int *d_neighbors,
                                                long *nnz, void *stream) {
  return run_guarded("nkx_neighbor_list", [&] {
    NKX_REQUIRE(nfunc > 0 && nboxes > 0 && d_centers && d_radii && d_boxes && d_offsets && nnz, NKX_ERR_ARG,
                "invalid arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = (unsigned)((nboxes * 32 + 255) / 256);
    int *cnt = nullptr;
    NKX_CUDA(cudaMalloc(&cnt, sizeof(int) * nboxes));
    std::vector<int> h(nboxes);
    cudaError_t e = cudaSuccess;
    neighbor_kernel<<<grid, 256, 0, s>>>(nfunc, d_centers, d_radii, nboxes, d_boxes, nullptr, cnt, nullptr);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), cnt, sizeof(int) * nboxes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(cnt);
    NKX_CUDA(e);
    // CSR offsets (int, as NeighborList::offsets)
    std::vector<int> off(nboxes + 1, 0);
    long total = 0;
    for (long b = 0; b < nboxes; ++b) {
      off[b] = (int)total;
      total += h[b];
      NKX_REQUIRE(total <= 0x7fffffffL, NKX_ERR_UNSUPPORTED, "neighbour list longer than 2^31 - 1 entries");
    }
    off[nboxes] = (int)total;
    if (d_neighbors) NKX_REQUIRE(total <= *nnz, NKX_ERR_ARG, "neighbors buffer smaller than the list (*nnz)");
    NKX_CUDA(cudaMemcpyAsync(d_offsets, off.data(), sizeof(int) * (nboxes + 1), cudaMemcpyHostToDevice, s));
    if (d_neighbors && total > 0) {
      neighbor_kernel<<<grid, 256, 0, s>>>(nfunc, d_centers, d_radii, nboxes, d_boxes, d_offsets, nullptr,
                                           d_neighbors);
      NKX_LAUNCH_CHECK();
    }
    NKX_CUDA(cudaStreamSynchronize(s));
    *nnz = total;
  });
}
