// Grid construction: Becke partition on the device and make_flat_grid.
#include <functional>
#include <algorithm>
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

// Host assembly of the unpartitioned atom grids: radial-outer,
// angular-inner per atom (grid.hpp:214-287).
void atom_grids(const nkx_molecule &mol, const nkx_grid_spec &spec, std::vector<double> &xyz,
                std::vector<double> &w, std::vector<int> &owner) {
  std::vector<double> axyz, aw;
  NKX_REQUIRE(lebedev_rule(spec.nang_order, axyz, aw), NKX_ERR_UNSUPPORTED,
              "no Lebedev rule of the requested order");
  const int nang = (int)aw.size();
  xyz.clear();
  w.clear();
  owner.clear();
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
    const int nr = spec.sizing == NKX_SIZING_PYSCF ? (int)(spec.nrad * ratio[periodic_row(Z) - 1] + 0.5)
                                                   : spec.nrad;
    std::vector<double> r, rw;
    radial_rule(spec.radial_scheme, nr, R, spec.ta_alpha, r, rw);
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nang; ++j) {
        xyz.push_back(mol.xyz[3 * a] + r[i] * axyz[3 * j]);
        xyz.push_back(mol.xyz[3 * a + 1] + r[i] * axyz[3 * j + 1]);
        xyz.push_back(mol.xyz[3 * a + 2] + r[i] * axyz[3 * j + 2]);
        NKX_REQUIRE(rw[i] * aw[j] >= 0.0, NKX_ERR_NUMERIC, "Detected negative weights aborting");
        w.push_back(rw[i] * aw[j]);
        owner.push_back(a);
      }
  }
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
    std::vector<double> hx, hw;
    std::vector<int> ho;
    atom_grids(*mol, *spec, hx, hw, ho);
    const long n = (long)hw.size();
    double *dc = nullptr, *dp = nullptr, *dw = nullptr;
    int *dow = nullptr;
    NKX_CUDA(cudaMalloc(&dc, sizeof(double) * 3 * mol->natoms));
    NKX_CUDA(cudaMalloc(&dp, sizeof(double) * 3 * n));
    NKX_CUDA(cudaMalloc(&dw, sizeof(double) * n));
    NKX_CUDA(cudaMalloc(&dow, sizeof(int) * n));
    NKX_CUDA(cudaMemcpy(dc, mol->xyz, sizeof(double) * 3 * mol->natoms, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(dp, hx.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(dw, hw.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(dow, ho.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    launch_becke(dc, mol->natoms, dp, dow, n, dw, spec->becke_clamp, 0);
    NKX_CUDA(cudaMemcpy(hw.data(), dw, sizeof(double) * n, cudaMemcpyDeviceToHost));
    cudaFree(dc);
    cudaFree(dp);
    cudaFree(dw);
    cudaFree(dow);
    // stable compaction of w > threshold (grid.hpp:307-338, order kept)
    long cnt = 0;
    for (long g = 0; g < n; ++g)
      if (hw[g] > spec->weight_threshold) {
        if (xyz) {
          xyz[3 * cnt] = hx[3 * g];
          xyz[3 * cnt + 1] = hx[3 * g + 1];
          xyz[3 * cnt + 2] = hx[3 * g + 2];
          w[cnt] = hw[g];
          owner[cnt] = ho[g];
        }
        ++cnt;
      }
    *npoints = cnt;
  });
}
