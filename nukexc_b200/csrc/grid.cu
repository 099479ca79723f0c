// Grid construction on the device: atom grids, Becke partition and the
// compaction of make_flat_grid.
#include <functional>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "host_setup.hpp"

namespace nkx {

void set_error(const std::string &msg);
nkx_status run_guarded(const char *where, const std::function<void()> &fn);

// Becke cell function step s(p(p(p(mu)))) (partitioning.hpp:44-55)
__device__ __forceinline__ double becke_s(double mu) {
  mu = mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
  double p = 1.5 * mu - 0.5 * mu * mu * mu;
  p = 1.5 * p - 0.5 * p * p * p;
  p = 1.5 * p - 0.5 * p * p * p;
  return 0.5 * (1.0 - p);
}

__device__ __forceinline__ double dist3(const double *a, const double *b) {
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

constexpr int kBeckeList = 128;

// One thread per point.  With the Laqua clamp R_ij = min(|A_i-A_j|, Rc)
// (partitioning.hpp:134-148) the cell functions are exactly 0 or 1 far from
// the point: every atom with r_i >= r_min + Rc has P_i = 0 (its factor
// against the nearest atom is s(1) = 0), and in P_i of the others every atom
// with r_j >= r_i + Rc contributes s(-1) = 1.  Only atoms with
// r_j < r_min + 2 Rc are therefore visited, in index order, which gives the
// same products and sums as the full O(N_atoms^2) loop of
// partition_becke_team (partitioning.hpp:166-212).  Rc <= 0 selects the
// unclamped original (partition_becke, partitioning.hpp:63-120) without
// screening.
__global__ void becke_kernel(const double *__restrict__ centers, int natoms, const double *__restrict__ pts,
                             const int *__restrict__ owner, long npts, double *__restrict__ w, double Rc) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= npts) return;
  const double *p = pts + 3 * g;
  const bool clamp = Rc > 0.0;
  double rmin = 1e300;
  for (int i = 0; i < natoms; ++i) rmin = fmin(rmin, dist3(p, centers + 3 * i));
  int list[kBeckeList];
  int nl = 0;
  bool full = !clamp;
  if (clamp) {
    const double lim = rmin + 2.0 * Rc;
    for (int j = 0; j < natoms; ++j) {
      if (dist3(p, centers + 3 * j) < lim) {
        if (nl == kBeckeList) {
          full = true;
          break;
        }
        list[nl++] = j;
      }
    }
  }
  const int own = owner[g];
  double norm = 0.0, pown = 0.0;
  if (full) {
    // with the clamp, factors of atoms j with r_j >= r_i + Rc are 1 (mu <= -1
    // is clamped) and cells with r_i >= r_min + Rc are 0 (the nearest atom
    // gives mu >= 1): skipping them is the full loop without its trivial terms
    for (int i = 0; i < natoms; ++i) {
      const double ri = dist3(p, centers + 3 * i);
      if (clamp && ri >= rmin + Rc) continue;
      double P = 1.0;
      for (int j = 0; j < natoms; ++j) {
        if (j == i) continue;
        const double rj = dist3(p, centers + 3 * j);
        if (clamp && rj >= ri + Rc) continue;
        double Rij = dist3(centers + 3 * i, centers + 3 * j);
        if (clamp) Rij = fmin(Rij, Rc);
        P *= becke_s((ri - rj) / Rij);
      }
      if (i == own) pown = P;
      norm += P;
    }
  } else {
    for (int a = 0; a < nl; ++a) {
      const int i = list[a];
      const double ri = dist3(p, centers + 3 * i);
      if (ri >= rmin + Rc) continue;  // P_i == 0 exactly
      double P = 1.0;
      for (int c = 0; c < nl; ++c) {
        const int j = list[c];
        if (j == i) continue;
        const double Rij = fmin(dist3(centers + 3 * i, centers + 3 * j), Rc);
        P *= becke_s((ri - dist3(p, centers + 3 * j)) / Rij);
      }
      if (i == own) pown = P;
      norm += P;
    }
  }
  w[g] *= pown / norm;
}

void launch_becke(const double *d_centers, int natoms, const double *d_pts, const int *d_owner, long npts,
                  double *d_w, double clamp, cudaStream_t s) {
  if (npts <= 0) return;
  const int T = 128;
  becke_kernel<<<(unsigned)((npts + T - 1) / T), T, 0, s>>>(d_centers, natoms, d_pts, d_owner, npts, d_w, clamp);
  NKX_LAUNCH_CHECK();
}

// ------------------------------------------------ grid on the device ----
// The unpartitioned atom grids, radial-outer and angular-inner per atom
// (grid.hpp:214-287), built on the device.
// Point g of atom a (g - off[a] = i nang + j) is radial node i and angular
// node j: xyz = A + r_i (x_j, y_j, z_j), w = w_i^rad w_j^ang, the same
// products and sums as the host construction (no fused multiply-add, so the
// coordinates are bit-identical to it).
__global__ void atom_grid_kernel(const double *__restrict__ centers, const long *__restrict__ off, int natoms,
                                 const long *__restrict__ roff, const double *__restrict__ rad,
                                 const double *__restrict__ ang, int nang, long n, double *__restrict__ xyz,
                                 double *__restrict__ w, int *__restrict__ owner) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= n) return;
  int lo = 0, hi = natoms - 1;  // the atom a with off[a] <= g < off[a + 1]
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= g) lo = mid; else hi = mid - 1;
  }
  const long l = g - off[lo];
  const long i = l / nang;
  const int j = (int)(l - i * nang);
  const double r = rad[2 * (roff[lo] + i)], rw = rad[2 * (roff[lo] + i) + 1];
#pragma unroll
  for (int k = 0; k < 3; ++k) xyz[3 * g + k] = __dadd_rn(centers[3 * lo + k], __dmul_rn(r, ang[4 * j + k]));
  w[g] = __dmul_rn(rw, ang[4 * j + 3]);
  owner[g] = lo;
}

constexpr int kCompactBlock = 1024;

// points with w > threshold in each block of kCompactBlock points
__global__ void __launch_bounds__(kCompactBlock) compact_count_kernel(const double *__restrict__ w, long n, double thr,
                                                                      int *__restrict__ cnt) {
  const long g = blockIdx.x * (long)kCompactBlock + threadIdx.x;
  const bool keep = g < n && w[g] > thr;
  const int c = __syncthreads_count(keep);
  if (threadIdx.x == 0) cnt[blockIdx.x] = c;
}

// stable compaction: block b writes its kept points from out_off[b] on, in
// point order (warp ballots and a scan of the 32 warp counts)
__global__ void __launch_bounds__(kCompactBlock) compact_scatter_kernel(
    const double *__restrict__ xyz, const double *__restrict__ w, const int *__restrict__ owner, long n, double thr,
    const long *__restrict__ out_off, double *__restrict__ oxyz, double *__restrict__ ow, int *__restrict__ oown) {
  __shared__ int wsum[kCompactBlock / 32];
  const long g = blockIdx.x * (long)kCompactBlock + threadIdx.x;
  const bool keep = g < n && w[g] > thr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) wsum[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    int v = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    wsum[lane] = v - wsum[lane];  // exclusive
  }
  __syncthreads();
  if (keep) {
    const long d = out_off[blockIdx.x] + wsum[warp] + __popc(m & ((1u << lane) - 1u));
    oxyz[3 * d] = xyz[3 * g];
    oxyz[3 * d + 1] = xyz[3 * g + 1];
    oxyz[3 * d + 2] = xyz[3 * g + 2];
    ow[d] = w[g];
    oown[d] = owner[g];
  }
}

// The last grid built by nkx_make_flat_grid, on the device, keyed by the
// call's inputs: the counting call builds it and the filling call with the
// same inputs copies it out (and frees it) instead of building it again.
struct GridCache {
  std::vector<unsigned char> key;
  long n = 0;
  double *xyz = nullptr, *w = nullptr;
  int *owner = nullptr;
  void clear() {
    cudaFree(xyz);
    cudaFree(w);
    cudaFree(owner);
    xyz = w = nullptr;
    owner = nullptr;
    key.clear();
    n = 0;
  }
};
static GridCache g_grid;
static std::mutex g_grid_mu;

// the call's inputs as bytes (the spec field by field: no padding bytes)
static std::vector<unsigned char> grid_key(const nkx_molecule &mol, const nkx_grid_spec &spec) {
  std::vector<unsigned char> k;
  auto put = [&](const void *q, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(q);
    k.insert(k.end(), b, b + n);
  };
  put(&mol.natoms, sizeof(int));
  put(&spec.radial_scheme, sizeof(int));
  put(&spec.nrad, sizeof(int));
  put(&spec.nang_order, sizeof(int));
  put(&spec.weight_threshold, sizeof(double));
  put(&spec.ta_alpha, sizeof(double));
  put(&spec.sizing, sizeof(int));
  put(&spec.becke_clamp, sizeof(double));
  put(mol.xyz, sizeof(double) * 3 * mol.natoms);
  put(mol.Z, sizeof(int) * mol.natoms);
  return k;
}

template <class T>
static T *dev_alloc(size_t n) {
  T *p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(1, n)) != cudaSuccess) {
    cudaGetLastError();
    throw Error{NKX_ERR_ALLOC, "grid construction: device allocation of " + std::to_string(sizeof(T) * n) + " bytes failed"};
  }
  return p;
}

// Builds the compacted grid on the device into g_grid (the caller holds the
// lock): radial and Lebedev rules on the host (small tables), points,
// weights and owners by atom_grid_kernel, the Becke partition, then the
// stable compaction of w > threshold (grid.hpp:307-338, order kept).
static void build_grid_device(const nkx_molecule &mol, const nkx_grid_spec &spec) {
  std::vector<double> axyz, aw;
  NKX_REQUIRE(lebedev_rule(spec.nang_order, axyz, aw), NKX_ERR_UNSUPPORTED, "no Lebedev rule of the requested order");
  const int nang = (int)aw.size();
  std::vector<double> ang(4 * (size_t)nang), rad;
  bool ang_pos = false, ang_neg = false;
  for (int j = 0; j < nang; ++j) {
    for (int k = 0; k < 3; ++k) ang[4 * j + k] = axyz[3 * j + k];
    ang[4 * j + 3] = aw[j];
    ang_pos |= aw[j] > 0.0;
    ang_neg |= aw[j] < 0.0;
  }
  std::vector<long> off(mol.natoms + 1, 0), roff(mol.natoms + 1, 0);
  for (int a = 0; a < mol.natoms; ++a) {
    const int Z = mol.Z[a];
    double R = 1.0;
    if (spec.radial_scheme == NKX_RADIAL_TA) {
      R = ta_xi(Z);
    } else {
      const double bs = bragg_slater(Z);
      if (bs > 0) R = 0.5 * bs * kAngToBohr;
    }
    static const double ratio[7] = {1.0, 1.5, 1.6, 1.8, 1.9, 2.0, 2.1};  // grid.hpp:142
    const int nr = spec.sizing == NKX_SIZING_PYSCF ? (int)(spec.nrad * ratio[periodic_row(Z) - 1] + 0.5) : spec.nrad;
    std::vector<double> r, rw;
    radial_rule(spec.radial_scheme, nr, R, spec.ta_alpha, r, rw);
    for (int i = 0; i < nr; ++i) {
      // every product w_i^rad w_j^ang must be non-negative (grid.hpp:284-286)
      NKX_REQUIRE(!((rw[i] > 0.0 && ang_neg) || (rw[i] < 0.0 && ang_pos)), NKX_ERR_NUMERIC,
                  "Detected negative weights aborting");
      rad.push_back(r[i]);
      rad.push_back(rw[i]);
    }
    roff[a + 1] = roff[a] + nr;
    off[a + 1] = off[a] + (long)nr * nang;
  }
  const long n = off[mol.natoms];
  g_grid.clear();
  double *dc = nullptr, *drad = nullptr, *dang = nullptr, *dp = nullptr, *dw = nullptr;
  long *doff = nullptr, *droff = nullptr, *dout = nullptr;
  int *dow = nullptr, *dcnt = nullptr;
  auto release = [&] {
    for (void *q : {(void *)dc, (void *)drad, (void *)dang, (void *)dp, (void *)dw, (void *)doff, (void *)droff,
                    (void *)dout, (void *)dow, (void *)dcnt})
      cudaFree(q);
  };
  try {
    dc = dev_alloc<double>(3 * (size_t)mol.natoms);
    doff = dev_alloc<long>(mol.natoms + 1);
    droff = dev_alloc<long>(mol.natoms + 1);
    drad = dev_alloc<double>(rad.size());
    dang = dev_alloc<double>(ang.size());
    dp = dev_alloc<double>(3 * (size_t)n);
    dw = dev_alloc<double>(n);
    dow = dev_alloc<int>(n);
    NKX_CUDA(cudaMemcpy(dc, mol.xyz, sizeof(double) * 3 * mol.natoms, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(doff, off.data(), sizeof(long) * off.size(), cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(droff, roff.data(), sizeof(long) * roff.size(), cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(drad, rad.data(), sizeof(double) * rad.size(), cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(dang, ang.data(), sizeof(double) * ang.size(), cudaMemcpyHostToDevice));
    if (n > 0) {
      atom_grid_kernel<<<(unsigned)((n + 255) / 256), 256>>>(dc, doff, mol.natoms, droff, drad, dang, nang, n, dp, dw,
                                                             dow);
      NKX_LAUNCH_CHECK();
    }
    launch_becke(dc, mol.natoms, dp, dow, n, dw, spec.becke_clamp, 0);
    const long nblk = std::max<long>(1, (n + kCompactBlock - 1) / kCompactBlock);
    dcnt = dev_alloc<int>(nblk);
    dout = dev_alloc<long>(nblk);
    if (n > 0) {
      compact_count_kernel<<<(unsigned)nblk, kCompactBlock>>>(dw, n, spec.weight_threshold, dcnt);
      NKX_LAUNCH_CHECK();
    }
    std::vector<int> cnt(nblk, 0);
    std::vector<long> bo(nblk, 0);
    if (n > 0) NKX_CUDA(cudaMemcpy(cnt.data(), dcnt, sizeof(int) * nblk, cudaMemcpyDeviceToHost));
    long tot = 0;
    for (long b = 0; b < nblk; ++b) {
      bo[b] = tot;
      tot += cnt[b];
    }
    NKX_CUDA(cudaMemcpy(dout, bo.data(), sizeof(long) * nblk, cudaMemcpyHostToDevice));
    g_grid.xyz = dev_alloc<double>(3 * (size_t)tot);
    g_grid.w = dev_alloc<double>(tot);
    g_grid.owner = dev_alloc<int>(tot);
    if (n > 0) {
      compact_scatter_kernel<<<(unsigned)nblk, kCompactBlock>>>(dp, dw, dow, n, spec.weight_threshold, dout,
                                                                g_grid.xyz, g_grid.w, g_grid.owner);
      NKX_LAUNCH_CHECK();
    }
    NKX_CUDA(cudaDeviceSynchronize());
    g_grid.n = tot;
    g_grid.key = grid_key(mol, spec);
  } catch (...) {
    release();
    g_grid.clear();
    throw;
  }
  release();
}

}  // namespace nkx

using namespace nkx;

extern "C" nkx_status nkx_becke_partition(const double *d_centers, int natoms, const double *d_points,
                                          const int *d_owner, long npts, double *d_weights, double clamp,
                                          void *stream) {
  return run_guarded("nkx_becke_partition", [&] {
    NKX_REQUIRE(natoms > 0 && npts >= 0 && d_centers && (npts == 0 || (d_points && d_owner && d_weights)),
                NKX_ERR_ARG, "invalid arguments");
    launch_becke(d_centers, natoms, d_points, d_owner, npts, d_weights, clamp, (cudaStream_t)stream);
  });
}

extern "C" nkx_status nkx_make_flat_grid(const nkx_molecule *mol, const nkx_grid_spec *spec, long *npoints,
                                         double *xyz, double *w, int *owner) {
  return run_guarded("nkx_make_flat_grid", [&] {
    NKX_REQUIRE(mol && spec && npoints && mol->natoms > 0 && spec->nrad > 0, NKX_ERR_ARG, "invalid arguments");
    NKX_REQUIRE(!xyz || (w && owner), NKX_ERR_ARG, "xyz, w and owner are given together");
    std::lock_guard<std::mutex> lock(g_grid_mu);
    if (g_grid.key.empty() || g_grid.key != grid_key(*mol, *spec)) build_grid_device(*mol, *spec);
    *npoints = g_grid.n;
    if (xyz) {
      NKX_CUDA(cudaMemcpy(xyz, g_grid.xyz, sizeof(double) * 3 * g_grid.n, cudaMemcpyDeviceToHost));
      NKX_CUDA(cudaMemcpy(w, g_grid.w, sizeof(double) * g_grid.n, cudaMemcpyDeviceToHost));
      NKX_CUDA(cudaMemcpy(owner, g_grid.owner, sizeof(int) * g_grid.n, cudaMemcpyDeviceToHost));
      g_grid.clear();  // the pair of calls is complete
    }
  });
}
