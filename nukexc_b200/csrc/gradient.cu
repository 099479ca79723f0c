// XC nuclear gradient at fixed orbitals (FP64).  No counterpart in the
// reference; it differentiates exactly what nkx_fock_build integrates:
//
//   E_xc(R) = sum_g w_g(R) f(rho(r_g), grad rho(r_g)),
//   r_g = R_owner(g) + fixed offset,   w_g = a_g P_owner(r_g) / sum_i P_i(r_g)
//
// (grid points move with their owner atom; a_g, the radial x angular weight,
// does not depend on the geometry; P_i are Becke cell functions with the
// Laqua clamp R_ij = min(|R_i - R_j|, clamp), partitioning.hpp:126-213).
//
// dE/dR_A = sum_g w_g sum_s sum_mu t_(s,mu,g) (delta_(owner(g),A) - delta_(atom(mu),A))
//         + sum_g f_g a_g dQ_g/dR_A,
//
// with X^s_mu(g) = sum_nu P^s_mu,nu phi_nu(g) = sum_i C^s_mu,i occ_i T^s_i(g)
// (T = C^T Phi, the orbital values) and, per spin,
//   t_j = 4 c0 d_j phi X + 2 sum_k c_k (d_j d_k phi X + d_j phi d_k X),
// c0 = w v_rho / 2 and c_k = w df/d(d_k rho_s) being the Z coefficients of the
// Fock build (xc_integrals.hpp:506-514, :655-664).  The first sum holds the
// basis-centre and the point-motion terms, the second the Becke-weight term.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <string>
#include <vector>

#include "common.cuh"
#include "nkx.h"
#include "plan.cuh"
#include "sto.cuh"

namespace nkx {

nkx_status run_guarded(const char *where, const std::function<void()> &fn);

static inline unsigned gblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

// T[(bl, spin, comp)][i][g] = sum_f Phi_comp(g, f) C(i, f) over the batch's
// significant blocks: one 64-point x 64-orbital tile per thread block,
// thread (ty, tx) owning points ty + 16a and orbitals tx + 16j.
template <bool GRAD>
__global__ void __launch_bounds__(256) orbital_values_kernel(const double *__restrict__ phiT,
                                                             const double *__restrict__ Ct, int nocc, int nocc_pad,
                                                             int nbf_pad, const int *__restrict__ pair_off,
                                                             const int *__restrict__ pair_blk, long sb0, long p0,
                                                             int nspin, double *__restrict__ T) {
  constexpr int NC = GRAD ? 4 : 1;
  constexpr int KS = 16;
  __shared__ double Ps[NC][KS][64 + 1];
  __shared__ double Cs[KS][64 + 1];
  const int spin = blockIdx.y;
  const long bl = blockIdx.x / 4, b = sb0 + bl;
  const int g0 = (blockIdx.x % 4) * 64, i0 = blockIdx.z * 64;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const double *C = Ct + (size_t)spin * nocc * nbf_pad;
  const size_t tile = (size_t)kBatch * kBlockF;
  double acc[NC][4][4];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[c][a][j] = 0.0;
  for (int q = pair_off[b]; q < pair_off[b + 1]; ++q) {
    const int I = pair_blk[q];
    const double *P = phiT + (size_t)(q - p0) * NC * tile;
    for (int f0 = 0; f0 < kBlockF; f0 += KS) {
      for (int e = threadIdx.x; e < NC * 64 * KS; e += 256) {
        const int c = e / (64 * KS), r = (e / KS) % 64, k = e % KS;
        Ps[c][k][r] = P[c * tile + (size_t)(g0 + r) * kBlockF + f0 + k];
      }
      for (int e = threadIdx.x; e < 64 * KS; e += 256) {
        const int r = e / KS, k = e % KS, i = i0 + r;
        Cs[k][r] = i < nocc ? C[(size_t)i * nbf_pad + I * kBlockF + f0 + k] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < KS; ++k) {
        double bv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) bv[j] = Cs[k][tx + 16 * j];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const double av = Ps[c][k][ty + 16 * a];
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[c][a][j] += av * bv[j];
          }
      }
      __syncthreads();
    }
  }
  double *Tb = T + ((size_t)(bl * nspin + spin) * NC) * nocc_pad * kBatch;
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        Tb[((size_t)c * nocc_pad + i0 + tx + 16 * j) * kBatch + g0 + ty + 16 * a] = acc[c][a][j];
}

// Basis-centre and point-motion terms of one (batch, block) pair.  Thread
// (ty, tx) owns functions 4 ty .. 4 ty + 3 of the block and, per 16-point
// subtile, points 2 tx, 2 tx + 1.  X and grad X come from a small FP64 GEMM
// of C (block rows) with occ * T staged in shared memory, or (XIN) are read
// from X[pair][spin][comp][g][mu] made by the tensor cores.  Contributions
// are summed per owner atom (points) and per function atom in shared memory
// and leave the block as a few global atomics.
template <bool GRAD, bool XIN = false>
__global__ void __launch_bounds__(256) grad_pair_kernel(
    const StoFunc *__restrict__ sto, const int *__restrict__ fatom, const double *__restrict__ px,
    const double *__restrict__ py, const double *__restrict__ pz, const int *__restrict__ owner,
    const int *__restrict__ pair_batch, const int *__restrict__ pair_blk, long pstart, long sb0,
    const double *__restrict__ Ct, const double *__restrict__ occ, int nocc, int nocc_pad, int nbf_pad, int nspin,
    const double *__restrict__ T, const double *__restrict__ coef, long npad, double *__restrict__ F,
    const double *__restrict__ Xin = nullptr) {
  constexpr int NC = GRAD ? 4 : 1;
  __shared__ double Cs[16][kBlockF];
  __shared__ double Ts[16][NC][16];
  __shared__ StoFunc sfn[kBlockF];
  __shared__ int s_owner[kBatch], rep_pt[kBatch], s_fatom[kBlockF], rep_f[kBlockF];
  __shared__ double tp[kBatch][3], tfs[kBlockF][3];
  const long p = pstart + blockIdx.x;
  const int b = pair_batch[p], I = pair_blk[p];
  const long bl = b - sb0;
  const int tid = threadIdx.x, ty = tid >> 3, tx = tid & 7;
  {
    const int g = tid;
    s_owner[g] = owner[(long)b * kBatch + g];
    tp[g][0] = tp[g][1] = tp[g][2] = 0.0;
    if (tid < kBlockF) {
      s_fatom[tid] = fatom[I * kBlockF + tid];
      sfn[tid] = sto[I * kBlockF + tid];
      tfs[tid][0] = tfs[tid][1] = tfs[tid][2] = 0.0;
    }
  }
  __syncthreads();
  {
    const int g = tid;
    int r = g;
    for (int h = 0; h < g; ++h)
      if (s_owner[h] == s_owner[g]) {
        r = h;
        break;
      }
    rep_pt[g] = r;
    if (tid < kBlockF) {
      int rf = tid;
      for (int h = 0; h < tid; ++h)
        if (s_fatom[h] == s_fatom[tid]) {
          rf = h;
          break;
        }
      rep_f[tid] = rf;
    }
  }
  __syncthreads();
  double tf[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a) tf[a][0] = tf[a][1] = tf[a][2] = 0.0;
  for (int s = 0; s < nspin; ++s) {
    const double *C = Ct + (size_t)s * nocc * nbf_pad;
    const double *oc = occ + (size_t)s * nocc;
    const double *Tb = T + ((size_t)(bl * nspin + s) * NC) * nocc_pad * kBatch;
    const double *cs = coef + (size_t)s * 4 * npad;
    for (int st = 0; st < kBatch / 16; ++st) {
      double acc[4][2][NC];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[a][q][c] = 0.0;
      if (XIN) {
        const double *Xs = Xin + ((size_t)blockIdx.x * nspin + s) * NC * kBatch * kBlockF;
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const double2 *xp =
                reinterpret_cast<const double2 *>(Xs + ((size_t)c * kBatch + st * 16 + 2 * tx + q) * kBlockF + 4 * ty);
            const double2 u = xp[0], v = xp[1];
            acc[0][q][c] = u.x;
            acc[1][q][c] = u.y;
            acc[2][q][c] = v.x;
            acc[3][q][c] = v.y;
          }
      }
      for (int i0 = 0; !XIN && i0 < nocc; i0 += 16) {
        for (int e = tid; e < 16 * kBlockF; e += 256) {
          const int k = e >> 7, m = e & 127, i = i0 + k;
          Cs[k][m] = i < nocc ? C[(size_t)i * nbf_pad + I * kBlockF + m] : 0.0;
        }
        for (int e = tid; e < 16 * NC * 16; e += 256) {
          const int k = e / (NC * 16), c = (e / 16) % NC, gl = e & 15, i = i0 + k;
          Ts[k][c][gl] = i < nocc ? oc[i] * Tb[((size_t)c * nocc_pad + i) * kBatch + st * 16 + gl] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
          double cv[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) cv[a] = Cs[k][4 * ty + a];
#pragma unroll
          for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              const double tv = Ts[k][c][2 * tx + q];
#pragma unroll
              for (int a = 0; a < 4; ++a) acc[a][q][c] += cv[a] * tv;
            }
        }
        __syncthreads();
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int g = st * 16 + 2 * tx + q;
        const long gg = (long)b * kBatch + g;
        const double x = px[gg], y = py[gg], z = pz[gg];
        const double c0 = cs[gg];
        double ck[3] = {0.0, 0.0, 0.0};
        if (GRAD) {
          ck[0] = cs[npad + gg];
          ck[1] = cs[2 * npad + gg];
          ck[2] = cs[3 * npad + gg];
        }
        double tq[3] = {0.0, 0.0, 0.0};
        HessRadialCache rc;  // the thread's four functions at this point
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const StoFunc &fn = sfn[4 * ty + a];
          const double X = acc[a][q][0];
          double t[3];
          if (GRAD) {
            double v, gr[3], h[6];
            // the mixed gradient (XIN) takes e^x from exp_neg
            sto_value_grad_hess_cached<XIN>(fn, x, y, z, rc, v, gr, h);
            const double H[3][3] = {{h[0], h[1], h[2]}, {h[1], h[3], h[4]}, {h[2], h[4], h[5]}};
            const double dX[3] = {acc[a][q][NC > 1 ? 1 : 0], acc[a][q][NC > 2 ? 2 : 0], acc[a][q][NC > 3 ? 3 : 0]};
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              double u = 0.0;
#pragma unroll
              for (int k = 0; k < 3; ++k) u += ck[k] * (H[j][k] * X + gr[j] * dX[k]);
              t[j] = 4.0 * c0 * gr[j] * X + 2.0 * u;
            }
          } else {
            double v, gr[3];
            sto_value_grad(fn, x, y, z, v, gr[0], gr[1], gr[2]);
#pragma unroll
            for (int j = 0; j < 3; ++j) t[j] = 4.0 * c0 * gr[j] * X;
          }
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            tf[a][j] += t[j];
            tq[j] += t[j];
          }
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) atomicAdd(&tp[rep_pt[g]][j], tq[j]);
      }
    }
  }
  // the eight tx lanes of a ty hold the same functions: reduce, then one add
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double v = tf[a][j];
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      if (tx == 0) atomicAdd(&tfs[rep_f[4 * ty + a]][j], v);
    }
  __syncthreads();
  {
    const int g = tid;
    if (rep_pt[g] == g)
      for (int j = 0; j < 3; ++j)
        if (tp[g][j] != 0.0) atomicAdd(&F[3 * s_owner[g] + j], tp[g][j]);
    if (tid < kBlockF && rep_f[tid] == tid)
      for (int j = 0; j < 3; ++j)
        if (tfs[tid][j] != 0.0) atomicAdd(&F[3 * s_fatom[tid] + j], -tfs[tid][j]);
  }
}

// Becke-weight term: for point g with owner o, Q = P_o / Z, Z = sum_i P_i,
// dQ = sum_i kappa_i sum_(j != i) s'(mu_ij)/s(mu_ij) dmu_ij with
// kappa_i = Q (delta_io - P_i / Z), and
// dmu_ij/dR_A = [u_i (d_oA - d_iA) - u_j (d_oA - d_jA)] / R_ij
//             - mu_ij (e_ij (d_iA - d_jA)) / R_ij   (last term only where
// R_ij = |R_i - R_j| is below the clamp), u_i = (r - R_i)/|r - R_i|,
// e_ij = (R_i - R_j)/|R_i - R_j|.  One thread per point; the gradient is
// accumulated in shared memory (3 natoms doubles) when it fits, else in
// global memory directly.
__device__ __forceinline__ void becke_s_ds(double mu, double &s, double &ds) {
  const double p1 = 1.5 * mu - 0.5 * mu * mu * mu;
  const double p2 = 1.5 * p1 - 0.5 * p1 * p1 * p1;
  const double p3 = 1.5 * p2 - 0.5 * p2 * p2 * p2;
  s = 0.5 * (1.0 - p3);
  ds = -0.5 * (1.5 - 1.5 * p2 * p2) * (1.5 - 1.5 * p1 * p1) * (1.5 - 1.5 * mu * mu);
}

// Atoms that can contribute at a point: with the Laqua clamp Rc, a cell i
// with r_i >= r_min + Rc has P_i = 0 exactly (the nearest atom gives
// mu >= 1), and a factor j with r_j >= r_i + Rc is exactly 1 with s' = 0
// (mu <= -1), so every non-trivial cell, factor and derivative term involves
// only atoms with r < r_min + 2 Rc -- the same exact screening as
// becke_kernel.  Without the clamp, or when more than kGradList atoms are that
// close, the loops run over all atoms.
constexpr int kGradList = 192;

// The Becke-weight term of one point over its candidate list (n <= kGradList
// atoms): the distances to the listed atoms once, every cell function once,
// then the pair terms.  Of the three atoms a pair term (i, j) moves, the
// owner's and i's shares are summed in registers and added once per point
// and per i; only j's share goes to shared memory per pair.
__device__ void becke_grad_listed(const double *__restrict__ C, const double r[3], int o, const int *list, int n,
                                  double rmin, double clamp, double wg, double eg, double *Fa) {
  double rd[kGradList], Pl[kGradList];
  for (int k = 0; k < n; ++k) {
    const int a = list[k];
    const double dx = r[0] - C[3 * a], dy = r[1] - C[3 * a + 1], dz = r[2] - C[3 * a + 2];
    rd[k] = sqrt(dx * dx + dy * dy + dz * dz);
  }
  double Z = 0.0, Po = 0.0;
  for (int k = 0; k < n; ++k) {
    const int i = list[k];
    double P = 0.0;
    if (rd[k] < rmin + clamp) {  // else P_i = 0 exactly (Laqua clamp)
      P = 1.0;
      for (int c = 0; c < n && P != 0.0; ++c) {
        if (c == k) continue;
        const int j = list[c];
        const double dx = C[3 * i] - C[3 * j], dy = C[3 * i + 1] - C[3 * j + 1], dz = C[3 * i + 2] - C[3 * j + 2];
        const double Rij = fmin(sqrt(dx * dx + dy * dy + dz * dz), clamp);
        double mu = (rd[k] - rd[c]) / Rij;
        mu = mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
        double sv, dsv;
        becke_s_ds(mu, sv, dsv);
        P *= sv;
      }
    }
    Pl[k] = P;
    Z += P;
    if (i == o) Po = P;
  }
  if (!(Po > 0.0 && Z > 0.0)) return;
  const double Q = Po / Z, fa = eg * (wg / Q);
  double Fo[3] = {0.0, 0.0, 0.0};
  for (int ci = 0; ci < n; ++ci) {
    const int i = list[ci];
    const double kappa = Q * ((i == o ? 1.0 : 0.0) - Pl[ci] / Z);
    if (kappa == 0.0 || !(rd[ci] > 0.0)) continue;
    const double ri = rd[ci];
    const double ui[3] = {(r[0] - C[3 * i]) / ri, (r[1] - C[3 * i + 1]) / ri, (r[2] - C[3 * i + 2]) / ri};
    double Fi[3] = {0.0, 0.0, 0.0};
    for (int cj = 0; cj < n; ++cj) {
      if (cj == ci) continue;
      const int j = list[cj];
      const double rj = rd[cj];
      if (!(rj > 0.0)) continue;
      const double e[3] = {C[3 * i] - C[3 * j], C[3 * i + 1] - C[3 * j + 1], C[3 * i + 2] - C[3 * j + 2]};
      const double dij = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
      const bool clamped = dij >= clamp;
      const double Rij = clamped ? clamp : dij;
      const double mu = (ri - rj) / Rij;
      if (!(mu > -1.0 && mu < 1.0)) continue;  // clamped: s' = 0
      double sv, ds;
      becke_s_ds(mu, sv, ds);
      if (!(sv > 0.0)) continue;
      const double lam = fa * kappa * ds / sv / Rij;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double uj = (r[k] - C[3 * j + k]) / rj;
        const double ek = clamped ? 0.0 : mu * e[k] / dij;
        Fo[k] += lam * (ui[k] - uj);
        Fi[k] -= lam * (ui[k] + ek);
        atomicAdd(&Fa[3 * j + k], lam * (uj + ek));
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (Fi[k] != 0.0) atomicAdd(&Fa[3 * i + k], Fi[k]);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (Fo[k] != 0.0) atomicAdd(&Fa[3 * o + k], Fo[k]);
}

__global__ void becke_grad_kernel(const double *__restrict__ C, int natoms, const double *__restrict__ px,
                                  const double *__restrict__ py, const double *__restrict__ pz,
                                  const double *__restrict__ w, const int *__restrict__ owner,
                                  const double *__restrict__ edens, long npad, double clamp, bool smem,
                                  double *__restrict__ F) {
  extern __shared__ double Fs[];
  double *Fa = smem ? Fs : F;
  if (smem) {
    for (int e = threadIdx.x; e < 3 * natoms; e += blockDim.x) Fs[e] = 0.0;
    __syncthreads();
  }
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g < npad && w[g] != 0.0 && edens[g] != 0.0) {
    const double r[3] = {px[g], py[g], pz[g]};
    const int o = owner[g];
    auto dist = [&](int a) {
      const double dx = r[0] - C[3 * a], dy = r[1] - C[3 * a + 1], dz = r[2] - C[3 * a + 2];
      return sqrt(dx * dx + dy * dy + dz * dz);
    };
    int list[kGradList];
    int nl = 0;
    bool full = !(clamp > 0.0);
    double rmin = 1e300;
    if (!full) {
      for (int a = 0; a < natoms; ++a) rmin = fmin(rmin, dist(a));
      for (int a = 0; a < natoms; ++a)
        if (dist(a) < rmin + 2.0 * clamp) {
          if (nl == kGradList) {
            full = true;
            break;
          }
          list[nl++] = a;
        }
    }
    if (!full) {
      becke_grad_listed(C, r, o, list, nl, rmin, clamp, w[g], edens[g], Fa);
    } else {
      // without the clamp, or with more than kGradList candidates: every atom
      const int n = natoms;
      auto atom = [&](int k) { return k; };
      // P_i over the candidate set (factors of the other atoms are exactly 1)
      auto cellP = [&](int i) {
        const double ri = dist(i);
        if (!full && ri >= rmin + clamp) return 0.0;
        double P = 1.0;
        for (int c = 0; c < n && P != 0.0; ++c) {
          const int j = atom(c);
          if (j == i) continue;
          const double dx = C[3 * i] - C[3 * j], dy = C[3 * i + 1] - C[3 * j + 1], dz = C[3 * i + 2] - C[3 * j + 2];
          double Rij = sqrt(dx * dx + dy * dy + dz * dz);
          if (clamp > 0.0) Rij = fmin(Rij, clamp);
          double mu = (ri - dist(j)) / Rij;
          mu = mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
          double sv, dsv;
          becke_s_ds(mu, sv, dsv);
          P *= sv;
        }
        return P;
      };
      double Z = 0.0, Po = 0.0;
      for (int c = 0; c < n; ++c) {
        const int i = atom(c);
        const double P = cellP(i);
        Z += P;
        if (i == o) Po = P;
      }
      if (Po > 0.0 && Z > 0.0) {
        const double Q = Po / Z, a = w[g] / Q, fa = edens[g] * a;
        for (int ci = 0; ci < n; ++ci) {
          const int i = atom(ci);
          const double Pi = (i == o) ? Po : cellP(i);
          const double kappa = Q * ((i == o ? 1.0 : 0.0) - Pi / Z);
          if (kappa == 0.0) continue;
          double ui[3] = {r[0] - C[3 * i], r[1] - C[3 * i + 1], r[2] - C[3 * i + 2]};
          const double ri = sqrt(ui[0] * ui[0] + ui[1] * ui[1] + ui[2] * ui[2]);
          if (!(ri > 0.0)) continue;
          for (int k = 0; k < 3; ++k) ui[k] /= ri;
          for (int cj = 0; cj < n; ++cj) {
            const int j = atom(cj);
            if (j == i) continue;
            double e[3] = {C[3 * i] - C[3 * j], C[3 * i + 1] - C[3 * j + 1], C[3 * i + 2] - C[3 * j + 2]};
            const double dij = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            const bool clamped = clamp > 0.0 && dij >= clamp;
            const double Rij = clamped ? clamp : dij;
            double uj[3] = {r[0] - C[3 * j], r[1] - C[3 * j + 1], r[2] - C[3 * j + 2]};
            const double rj = sqrt(uj[0] * uj[0] + uj[1] * uj[1] + uj[2] * uj[2]);
            if (!(rj > 0.0)) continue;
            const double mu = (ri - rj) / Rij;
            if (!(mu > -1.0 && mu < 1.0)) continue;  // clamped: s' = 0
            double sv, ds;
            becke_s_ds(mu, sv, ds);
            if (!(sv > 0.0)) continue;
            const double lam = fa * kappa * ds / sv / Rij;
            for (int k = 0; k < 3; ++k) {
              uj[k] /= rj;
              const double ek = clamped ? 0.0 : mu * e[k] / dij;
              atomicAdd(&Fa[3 * o + k], lam * (ui[k] - uj[k]));
              atomicAdd(&Fa[3 * i + k], -lam * (ui[k] + ek));
              atomicAdd(&Fa[3 * j + k], lam * (uj[k] + ek));
            }
          }
        }
      }
    }  // every atom
  }
  if (smem) {
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * natoms; e += blockDim.x)
      if (Fs[e] != 0.0) atomicAdd(&F[e], Fs[e]);
  }
}

struct GradState {
  double *T = nullptr, *edens = nullptr, *F = nullptr;
  long cap_batches = 0;
  int nocc_pad = 0, nspin = 0;
  std::vector<void *> bufs;
  ~GradState() {
    for (void *p : bufs) cudaFree(p);
  }
  double *alloc(size_t n) {
    double *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      throw Error{NKX_ERR_ALLOC, "gradient workspace allocation of " + std::to_string(n * 8) + " bytes failed"};
    }
    bufs.push_back(p);
    return p;
  }
};

void destroy_grad_state(void *p) { delete static_cast<GradState *>(p); }

// orbital-value tiles of at most this many bytes per sub-range of batches
constexpr size_t kGradTBytes = (size_t)2 << 30;

static GradState &grad_state(Plan &P, int nspin, int nocc, bool need_T) {
  if (!P.grad_state) {
    GradState *G = new GradState();
    P.grad_state = G;
    G->edens = G->alloc(P.npad);
    G->F = G->alloc(3 * (size_t)P.natoms);
  }
  GradState &G = *static_cast<GradState *>(P.grad_state);
  if (!need_T) return G;
  const int NC = P.gga ? 4 : 1;
  const int nocc_pad = ((nocc + 63) / 64) * 64;
  long maxb = 1;
  for (const Chunk &c : P.chunks) maxb = std::max(maxb, c.b1 - c.b0);
  const size_t per_batch = (size_t)nspin * NC * nocc_pad * kBatch * sizeof(double);
  const long cap = std::max<long>(1, std::min<long>(maxb, (long)(kGradTBytes / per_batch)));
  if (nocc_pad != G.nocc_pad || nspin != G.nspin || cap > G.cap_batches) {
    G.nocc_pad = nocc_pad;
    G.nspin = nspin;
    G.cap_batches = cap;
    G.T = G.alloc((size_t)cap * per_batch / sizeof(double));
  }
  return G;
}

// FP64 part of the gradient: the density of the FP64 build, the functional,
// then per chunk the FP64 collocation, the orbital values T and the pair terms.
static void fp64_gradient_chunks(Plan &P, GradState &G, int nspin, int nocc, cudaStream_t s, StageTimer &Tm) {
  fp64_density_pass(P, nspin, nocc, s, Tm);
  functional_kernel<<<gblk(P.npad, 256), 256, 0, s>>>(P.xc, P.gga, nspin, P.npad, P.npad, P.d_w, P.d_rho, P.d_grad, nullptr,
                                                     P.d_coef, P.d_E, G.edens);
  NKX_LAUNCH_CHECK();
  ++P.launches;
  for (const Chunk &c : P.chunks) {
    if (c.p1 <= c.p0) continue;
    launch_colloc(P, c, s);
    for (long sb0 = c.b0; sb0 < c.b1; sb0 += G.cap_batches) {
      const long sb1 = std::min(c.b1, sb0 + G.cap_batches);
      const long q0 = P.h_pair_off[sb0], q1 = P.h_pair_off[sb1];
      if (q1 <= q0) continue;
      const dim3 og((unsigned)((sb1 - sb0) * 4), nspin, G.nocc_pad / 64);
      if (P.gga)
        orbital_values_kernel<true><<<og, 256, 0, s>>>(P.ws_phi, P.d_Ct, nocc, G.nocc_pad, P.nbf_pad, P.d_pair_off,
                                                       P.d_pair_blk, sb0, c.p0, nspin, G.T);
      else
        orbital_values_kernel<false><<<og, 256, 0, s>>>(P.ws_phi, P.d_Ct, nocc, G.nocc_pad, P.nbf_pad, P.d_pair_off,
                                                        P.d_pair_blk, sb0, c.p0, nspin, G.T);
      NKX_LAUNCH_CHECK();
      if (P.gga)
        grad_pair_kernel<true><<<(unsigned)(q1 - q0), 256, 0, s>>>(
            P.d_sto, P.d_fatom, P.d_px, P.d_py, P.d_pz, P.d_owner, P.d_pair_batch, P.d_pair_blk, q0, sb0, P.d_Ct,
            P.d_occ, nocc, G.nocc_pad, P.nbf_pad, nspin, G.T, P.d_coef, P.npad, G.F);
      else
        grad_pair_kernel<false><<<(unsigned)(q1 - q0), 256, 0, s>>>(
            P.d_sto, P.d_fatom, P.d_px, P.d_py, P.d_pz, P.d_owner, P.d_pair_batch, P.d_pair_blk, q0, sb0, P.d_Ct,
            P.d_occ, nocc, G.nocc_pad, P.nbf_pad, nspin, G.T, P.d_coef, P.npad, G.F);
      NKX_LAUNCH_CHECK();
      P.launches += 2;
    }
  }
}

static void xc_gradient(Plan &P, int precision, int nspin, int nocc, const double *C, const double *occ, int mem,
                        double clamp, double *grad, cudaStream_t s) {
  NKX_REQUIRE(precision == NKX_PREC_FP64 || precision == NKX_PREC_MIXED, NKX_ERR_ARG,
              "precision must be NKX_PREC_FP64 or NKX_PREC_MIXED");
  NKX_REQUIRE(precision == NKX_PREC_FP64 || mixed_available(P), NKX_ERR_UNSUPPORTED,
              "the mixed-precision gradient needs an sm_100 device");
  NKX_REQUIRE(nspin == 1 || nspin == 2, NKX_ERR_ARG, "nspin must be 1 or 2");
  NKX_REQUIRE(nocc > 0 && C && occ && grad, NKX_ERR_ARG, "invalid arguments");
  NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
  NKX_REQUIRE(P.natoms > 0 && P.d_owner, NKX_ERR_ARG, "the gradient needs a plan created with atoms and point owners");
  NKX_REQUIRE(P.all_funcs_on_atoms, NKX_ERR_ARG, "the gradient needs every basis function centred on an atom");
  P.launches = 0;
  StageTimer Tm;
  NKX_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int) * 2, s));
  upload_orbitals(P, nspin, nocc, C, occ, mem, s);
  const bool mixed = precision == NKX_PREC_MIXED;
  GradState &G = grad_state(P, nspin, nocc, !mixed);
  NKX_CUDA(cudaMemsetAsync(P.d_E, 0, sizeof(double), s));
  NKX_CUDA(cudaMemsetAsync(G.F, 0, sizeof(double) * 3 * P.natoms, s));
  if (mixed) {
    // Mixed precision: per chunk, the orbital values T_c come from the int8
    // digit contraction on the tensor cores, which also gives rho, grad rho
    // and the functional of the chunk's points, and so do X = C (occ T) and
    // its gradient; the pair terms with the STO Hessians and the Becke term
    // are FP64.
    mixed_gradient_begin(P, nspin, nocc, s);
    for (const Chunk &c : P.chunks) {
      int npadT = 0;
      const double *X = nullptr;
      const double *T = mixed_gradient_chunk(P, c, nspin, nocc, G.edens, s, &npadT, &X);
      const long q0 = c.p0, q1 = c.p1;
      if (q1 <= q0) continue;
      if (P.gga)
        grad_pair_kernel<true, true><<<(unsigned)(q1 - q0), 256, 0, s>>>(
            P.d_sto, P.d_fatom, P.d_px, P.d_py, P.d_pz, P.d_owner, P.d_pair_batch, P.d_pair_blk, q0, c.b0, P.d_Ct,
            P.d_occ, nocc, npadT, P.nbf_pad, nspin, T, P.d_coef, P.npad, G.F, X);
      else
        grad_pair_kernel<false, true><<<(unsigned)(q1 - q0), 256, 0, s>>>(
            P.d_sto, P.d_fatom, P.d_px, P.d_py, P.d_pz, P.d_owner, P.d_pair_batch, P.d_pair_blk, q0, c.b0, P.d_Ct,
            P.d_occ, nocc, npadT, P.nbf_pad, nspin, T, P.d_coef, P.npad, G.F, X);
      NKX_LAUNCH_CHECK();
      ++P.launches;
    }
  } else {
    fp64_gradient_chunks(P, G, nspin, nocc, s, Tm);
  }
  const size_t fs_bytes = sizeof(double) * 3 * (size_t)P.natoms;
  const bool smem = fs_bytes <= 48 * 1024;
  becke_grad_kernel<<<gblk(P.npad, 128), 128, smem ? fs_bytes : 0, s>>>(P.d_centers, P.natoms, P.d_px, P.d_py,
                                                                         P.d_pz, P.d_w, P.d_owner, G.edens, P.npad,
                                                                         clamp, smem, G.F);
  NKX_LAUNCH_CHECK();
  P.launches += 2;
  NKX_CUDA(cudaMemcpyAsync(grad, G.F, fs_bytes, cudaMemcpyDeviceToHost, s));
  int status[2] = {0, 0};
  NKX_CUDA(cudaMemcpyAsync(status, P.d_status, sizeof(status), cudaMemcpyDeviceToHost, s));
  NKX_CUDA(cudaStreamSynchronize(s));
  NKX_REQUIRE(status[0] == 0, NKX_ERR_TIMEOUT, "a tensor-core kernel wait gave up; the gradient is invalid");
  NKX_REQUIRE(status[1] == 0, NKX_ERR_NUMERIC, "non-finite value in the orbitals or occupations");
}

}  // namespace nkx

extern "C" NKX_API nkx_status nkx_xc_gradient(nkx_plan *plan, int precision, int nspin, int nocc, const double *C,
                                               const double *occ, int mem, double becke_clamp, double *grad,
                                               void *stream) {
  return nkx::run_guarded("nkx_xc_gradient", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    nkx::Plan &P = *reinterpret_cast<nkx::Plan *>(plan);
    nkx::xc_gradient(P, precision, nspin, nocc, C, occ, mem, becke_clamp, grad,
                     stream ? (cudaStream_t)stream : P.stream);
  });
}
