// The batched, screened grid-integration Fock build (the hot path).
//
// Once per geometry (nkx_plan_create): the grid is sorted into Morton order
// and cut into 256-point batches (create_bounding_boxes,
// nukexc/octree.hpp:70-141); basis functions are grouped into blocks of 128
// in basis order and a block is significant for a batch when the cutoff
// sphere of any of its functions meets the batch's bounding box
// (build_neighbor_list, nukexc/octree.hpp:317-390); the aux Coulomb metric is
// integrated on the grid and Cholesky-factorised in FP64.
//
// Per SCF iteration (nkx_fock_build), streamed over chunks of batches that
// fit the workspace:
//   pass A  collocation  PhiT[pair][g][f] (value + gradient)       colloc_*
//           density      T = PhiT C, rho = sum occ T^2, grad rho    density_*
//   J       y = (Vw rho), c = (A|B)^-1 y, v_g = sum c_a V_a(g) w_g  aux_*
//   XC      functional on every point, E_xc, Z coefficients         functional_kernel
//   pass B  Z^T[pair][g][f] = a_g phi + b_g . grad phi              zbuild_*
//           Vbar(I,J) += sum_b PhiT_bI^T Z_bJ  per function-block tile
//   end     V = Vbar + Vbar^T, unpadded to nbf x nbf
// (compute_gga / compute_gga_lsda, nukexc/xc_integrals.hpp:424-726, and
// compute_coulomb, nukexc/coulomb.hpp:56-115, reorganised into batches).
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <parallel/algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <vector>

#include "functionals.cuh"
#include "host_setup.hpp"
#include "plan.cuh"

namespace nkx {

// ------------------------------------------------------------- errors ----
static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

nkx_status run_guarded(const char *where, const std::function<void()> &fn) {
  try {
    fn();
    return NKX_OK;
  } catch (const Error &e) {
    set_error(std::string(where) + ": " + e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    set_error(std::string(where) + ": host allocation failed");
    return NKX_ERR_ALLOC;
  } catch (const std::exception &e) {
    set_error(std::string(where) + ": " + e.what());
    return NKX_ERR_ARG;
  }
}

XcSpec make_spec(const nkx_plan_options *o);
bool spec_is_gga(const XcSpec &s);

template <class T>
static T *dalloc(size_t n) {
  T *p = nullptr;
  if (n == 0) return nullptr;
  const cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error{NKX_ERR_ALLOC, "cudaMalloc of " + std::to_string(n * sizeof(T)) + " bytes failed"};
  }
  return p;
}

static unsigned nblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

// ========================================================== kernels ======

// Collocation of one (batch, function block) pair per CTA.  Lane l of a warp
// owns the four consecutive functions f = 4l .. 4l+3 of the block (so the
// functions of a shell share one radial factor, RadialCache); warp w owns
// points g = w + 8j.  Output PhiT[pair][comp][g][f], comp 0 = value,
// 1..3 = gradient (GRAD only); each warp store covers 32 x 4 consecutive f.
template <bool GRAD>
__global__ void __launch_bounds__(256) colloc_fp64_kernel(const StoFunc *__restrict__ sto, const double *__restrict__ px,
                                                          const double *__restrict__ py, const double *__restrict__ pz,
                                                          const int *__restrict__ pair_batch,
                                                          const int *__restrict__ pair_blk, long p0,
                                                          double *__restrict__ out) {
  const long p = p0 + blockIdx.x;
  const int b = pair_batch[p], I = pair_blk[p];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ double sx[kBatch], sy[kBatch], sz[kBatch];
  for (int g = threadIdx.x; g < kBatch; g += blockDim.x) {
    sx[g] = px[(long)b * kBatch + g];
    sy[g] = py[(long)b * kBatch + g];
    sz[g] = pz[(long)b * kBatch + g];
  }
  __syncthreads();
  StoFunc f[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) f[c] = sto[I * kBlockF + 4 * lane + c];
  const size_t tile = (size_t)kBatch * kBlockF;
  double *o = out + (size_t)blockIdx.x * (GRAD ? 4 : 1) * tile;
  for (int g = warp; g < kBatch; g += 8) {
    const double x = sx[g], y = sy[g], z = sz[g];
    RadialCache rc;
    double v[4][4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (GRAD)
        sto_value_grad_cached(f[c], x, y, z, rc, v[0][c], v[1][c], v[2][c], v[3][c]);
      else
        v[0][c] = sto_value_cached(f[c], x, y, z, rc);
    }
    const size_t idx = (size_t)g * kBlockF + 4 * lane;
#pragma unroll
    for (int k = 0; k < (GRAD ? 4 : 1); ++k) {
      double2 *dst = reinterpret_cast<double2 *>(o + k * tile + idx);
      dst[0] = make_double2(v[k][0], v[k][1]);
      dst[1] = make_double2(v[k][2], v[k][3]);
    }
  }
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Density of one 64-point tile of one batch for one spin, FP64.
// T(g,i) = sum_f PhiT(g,f) C(f,i) over the batch's significant blocks (and
// the three gradient components), then rho = sum_i occ_i T^2 and
// grad rho = 2 sum_i occ_i T grad T (density.hpp:188-255).  Thread (ty, tx)
// owns points g = ty + 16a (a < 4) and orbitals i = tx + 16c (c < 4) of the
// CTA's 64-orbital tile.  The orbital tile is the fastest index of the grid,
// so the CTAs of one 64-point slab run together and its PhiT rows come from
// L2 after the first (at 2850 orbitals a slab serves 45 tiles); each CTA adds
// its tile's share of rho and grad rho atomically (they are zeroed by the
// caller).  A K step is 16 functions of one block: the
// PhiT rows (16 contiguous functions per component and point) and the rows
// of the function-major orbitals Cf (64 contiguous orbitals per function)
// stream into shared memory with 16-byte cp.async copies through a ring of
// kDStages stages while the previous steps are multiplied.
constexpr int kDKs = 16, kDStages = 3;
template <bool GRAD>
constexpr int kDStageDoubles = (GRAD ? 4 : 1) * 64 * kDKs + kDKs * 64;
template <bool GRAD>
constexpr int kDSmemBytes = kDStages * kDStageDoubles<GRAD> * 8;

template <bool GRAD>
__global__ void __launch_bounds__(256) density_fp64_kernel(const double *__restrict__ phiT, const double *__restrict__ Cf,
                                                           const double *__restrict__ occ, int nocc, int nocc_pad,
                                                           int nbf_pad, const int *__restrict__ pair_off,
                                                           const int *__restrict__ pair_blk, long b0, long p0,
                                                           double *__restrict__ rho, double *__restrict__ grad,
                                                           long npad) {
  constexpr int NC = GRAD ? 4 : 1;
  constexpr int SD = kDStageDoubles<GRAD>;
  extern __shared__ __align__(16) double dsm[];  // [stage][Ps: NC x 64 points x 16 | Cs: 16 x 64 orbitals]
  const int spin = blockIdx.y;
  const int ntile = nocc_pad / 64;
  const int i0 = (blockIdx.x % ntile) * 64;
  const long bq = blockIdx.x / ntile;
  const long b = b0 + bq / 4;
  const int g0 = (int)(bq % 4) * 64;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const double *C = Cf + (size_t)spin * nbf_pad * nocc_pad;
  const double *oc = occ + (size_t)spin * nocc;
  const int q0 = pair_off[b], q1 = pair_off[b + 1];
  const size_t tile = (size_t)kBatch * kBlockF;
  const int total = (q1 - q0) * (kBlockF / kDKs);  // K steps of the orbital tile
  if (total == 0) return;  // no significant function: nothing to add
  auto issue = [&](int t, int st) {
    if (t < total) {
      const int r = t;
      const int q = q0 + r / (kBlockF / kDKs), f0 = (r % (kBlockF / kDKs)) * kDKs;
      const double *P = phiT + (size_t)(q - p0) * NC * tile + (size_t)g0 * kBlockF + f0;
      double *Ps = dsm + st * SD, *Cs = Ps + NC * 64 * kDKs;
      for (int e = threadIdx.x; e < NC * 64 * (kDKs / 2); e += 256) {
        const int row = e / (kDKs / 2), part = e % (kDKs / 2);  // row = (comp, point)
        cp_async16(Ps + row * kDKs + 2 * part, P + (size_t)(row / 64) * tile + (size_t)(row % 64) * kBlockF + 2 * part);
      }
      const double *Cr = C + (size_t)(pair_blk[q] * kBlockF + f0) * nocc_pad + i0;
      for (int e = threadIdx.x; e < kDKs * 32; e += 256) {
        const int k = e / 32, part = e % 32;
        cp_async16(Cs + k * 64 + 2 * part, Cr + (size_t)k * nocc_pad + 2 * part);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int st = 0; st < kDStages - 1; ++st) issue(st, st);
  double acc[NC][4][4];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[c][a][j] = 0.0;
  for (int t = 0; t < total; ++t) {
    cp_async_wait<kDStages - 2>();
    __syncthreads();  // step t is visible; the stage refilled below was read in step t - 1
    issue(t + kDStages - 1, (t + kDStages - 1) % kDStages);
    const double *Ps = dsm + (t % kDStages) * SD, *Cs = Ps + NC * 64 * kDKs;
#pragma unroll
    for (int k = 0; k < kDKs; ++k) {
      double bv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Cs[k * 64 + tx + 16 * j];
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const double av = Ps[(c * 64 + ty + 16 * a) * kDKs + k];
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[c][a][j] = fma(av, bv[j], acc[c][a][j]);
        }
    }
    if (t == total - 1) {
      // contract over this orbital tile
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        double sm[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int i = i0 + tx + 16 * j;
          const double o = i < nocc ? oc[i] : 0.0;
          const double tv = acc[0][a][j];
          sm[0] += o * tv * tv;
          if (GRAD) {
            sm[1] += o * tv * acc[NC > 1 ? 1 : 0][a][j];
            sm[2] += o * tv * acc[NC > 2 ? 2 : 0][a][j];
            sm[3] += o * tv * acc[NC > 3 ? 3 : 0][a][j];
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (int off = 8; off; off >>= 1) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], off);
        if (tx == 0) {
          const long g = b * kBatch + g0 + ty + 16 * a;
          atomicAdd(&rho[(size_t)spin * npad + g], sm[0]);
          if (GRAD) {
            atomicAdd(&grad[((size_t)spin * 3 + 0) * npad + g], 2.0 * sm[1]);
            atomicAdd(&grad[((size_t)spin * 3 + 1) * npad + g], 2.0 * sm[2]);
            atomicAdd(&grad[((size_t)spin * 3 + 2) * npad + g], 2.0 * sm[3]);
          }
        }
      }
    }
  }
  cp_async_wait<0>();
}

// Orbitals in function-major order for density_fp64_kernel:
// Cf[spin][f][i] = Ct[spin][i][f], orbitals padded to nocc_pad with zeros.
__global__ void transpose_orbitals_kernel(const double *__restrict__ Ct, int nocc, int nocc_pad, int nbf_pad,
                                          double *__restrict__ Cf) {
  __shared__ double t[32][33];
  const int spin = blockIdx.z;
  const int f0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r;
    t[r][threadIdx.x] = i < nocc ? Ct[((size_t)spin * nocc + i) * nbf_pad + f0 + threadIdx.x] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y)
    Cf[((size_t)spin * nbf_pad + f0 + r) * nocc_pad + i0 + threadIdx.x] = t[threadIdx.x][r];
}

// Functional on points [0, n) of the arrays given (plane stride npad; callers
// offset the pointers to work on a range): E_xc, and the Z coefficients
// coef[spin][0][g] = w (1/2 vrho + 1/2 vJ), coef[spin][1..3][g] = w vec
// (xc_integrals.hpp:506-514 closed shell, :655-664 open shell).  vj (may be
// null) is the weighted fitted Coulomb potential folded into both spins.
__global__ void functional_kernel(XcSpec s, bool gga, int nspin, long npad, long n, const double *__restrict__ w,
                                  const double *__restrict__ rho, const double *__restrict__ grad,
                                  const double *__restrict__ vj, double *__restrict__ coef, double *Eacc,
                                  double *__restrict__ edens) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double e = 0.0, fdens = 0.0;
  if (g < n) {
    const double wg = w[g];
    double vr[2] = {0, 0}, vec[2][3] = {{0, 0, 0}, {0, 0, 0}}, gr[2][3] = {{0, 0, 0}, {0, 0, 0}};
    if (gga)
      for (int sp = 0; sp < nspin; ++sp)
        for (int k = 0; k < 3; ++k) gr[sp][k] = grad[((size_t)sp * 3 + k) * npad + g];
    if (wg != 0.0) {
      if (nspin == 1) {
        const double sg = gr[0][0] * gr[0][0] + gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2];
        double f, vrho, vs;
        xc_unpol(s, rho[g], sg, f, vrho, vs);
        fdens = f;
        e = wg * f;
        vr[0] = vrho;
        for (int k = 0; k < 3; ++k) vec[0][k] = 2.0 * vs * gr[0][k];
      } else {
        const double saa = gr[0][0] * gr[0][0] + gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2];
        const double sab = gr[0][0] * gr[1][0] + gr[0][1] * gr[1][1] + gr[0][2] * gr[1][2];
        const double sbb = gr[1][0] * gr[1][0] + gr[1][1] * gr[1][1] + gr[1][2] * gr[1][2];
        double f, d[5];
        xc_pol(s, rho[g], rho[npad + g], saa, sab, sbb, f, d);
        fdens = f;
        e = wg * f;
        vr[0] = d[0];
        vr[1] = d[1];
        for (int k = 0; k < 3; ++k) {
          vec[0][k] = 2.0 * d[2] * gr[0][k] + d[3] * gr[1][k];
          vec[1][k] = 2.0 * d[4] * gr[1][k] + d[3] * gr[0][k];
        }
      }
    }
    if (edens) edens[g] = fdens;
    const double vjg = vj ? vj[g] : 0.0;
    for (int sp = 0; sp < nspin; ++sp) {
      coef[((size_t)sp * 4 + 0) * npad + g] = wg * 0.5 * vr[sp] + 0.5 * vjg;
      coef[((size_t)sp * 4 + 1) * npad + g] = wg * vec[sp][0];
      coef[((size_t)sp * 4 + 2) * npad + g] = wg * vec[sp][1];
      coef[((size_t)sp * 4 + 3) * npad + g] = wg * vec[sp][2];
    }
  }
  __shared__ double red[32];
  for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    e = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (threadIdx.x == 0) atomicAdd(Eacc, e);
  }
}

// Z^T[pair][spin][g][f] = coef0 phi + coef1 dphi/dx + coef2 dphi/dy + coef3 dphi/dz.
// Spin index nspin (when jonly) builds Z_J = 1/2 vJ phi for a separate J.
template <bool GRAD>
__global__ void zbuild_fp64_kernel(const double *__restrict__ phiT, const double *__restrict__ coef,
                                   const double *__restrict__ vj, const int *__restrict__ pair_batch, long p0,
                                   int nz, int nspin, long npad, double *__restrict__ zT) {
  constexpr int NC = GRAD ? 4 : 1;
  const long q = blockIdx.x;
  const int b = pair_batch[p0 + q];
  const size_t tile = (size_t)kBatch * kBlockF;
  const double *P = phiT + q * NC * tile;
  for (int e = threadIdx.x; e < kBatch * kBlockF; e += blockDim.x) {
    const int g = e / kBlockF;
    const long gg = (long)b * kBatch + g;
    const double v = P[e];
    double dx = 0, dy = 0, dz = 0;
    if (GRAD) {
      dx = P[tile + e];
      dy = P[2 * tile + e];
      dz = P[3 * tile + e];
    }
    for (int s = 0; s < nz; ++s) {
      double z;
      if (s < nspin) {
        const double *c = coef + (size_t)s * 4 * npad;
        z = c[gg] * v;
        if (GRAD) z += c[npad + gg] * dx + c[2 * npad + gg] * dy + c[3 * npad + gg] * dz;
      } else {
        z = 0.5 * vj[gg] * v;
      }
      zT[(q * nz + s) * tile + e] = z;
    }
  }
}

__device__ __forceinline__ int block_pos(const uint32_t *m, int I) {
  int pos = 0;
  for (int w = 0; w < (I >> 5); ++w) pos += __popc(m[w]);
  return pos + __popc(m[I >> 5] & ((1u << (I & 31)) - 1u));
}
__device__ __forceinline__ bool block_has(const uint32_t *m, int I) { return (m[I >> 5] >> (I & 31)) & 1u; }

// V contraction of the FP64 build: Vbar(I, J) += sum_b PhiT_b,I^T Z_b,J over
// the chunk's batches b where blocks I and J are both significant
// (xc_integrals.hpp:677-706), one 128 x 128 output tile per CTA (8 x 8 per
// thread).  The operand rows of a pair, PhiT[g][f] and Z^T[g][f], are 1 KB
// rows of 128 functions per point, so each 16-point K step of both operands
// (32 KB) streams into shared memory with 16-byte cp.async copies through a
// ring of kVStages stages while the previous steps are multiplied.
constexpr int kVKs = 16, kVStages = 4;
constexpr int kVStageDoubles = 2 * kVKs * kBlockF;
constexpr int kVSmemBytes = kVStages * kVStageDoubles * 8;

// next K step of a V unit: step k of batch b, batches without both blocks skipped
__device__ __forceinline__ void vstep_next(const uint32_t *__restrict__ mask, int mask_words, long b1, int I, int J,
                                           long &b, int &k) {
  if (++k < kBatch / kVKs) return;
  k = 0;
  for (++b; b < b1; ++b) {
    const uint32_t *m = mask + b * mask_words;
    if (block_has(m, I) && block_has(m, J)) return;
  }
}

__global__ void __launch_bounds__(256) vgemm_fp64_kernel(const double *__restrict__ phiT, const double *__restrict__ zT,
                                                         int phi_stride_tiles, int z_stride, const int *__restrict__ pair_off,
                                                         const uint32_t *__restrict__ mask, int mask_words, long b0,
                                                         long b1, long p0, int nbf_pad, double *__restrict__ V) {
  extern __shared__ __align__(16) double vsm[];  // [stage][A | B][kVKs][128]
  const int J = blockIdx.x, I = blockIdx.y, zi = blockIdx.z;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const size_t tile = (size_t)kBatch * kBlockF;
  // first step: the first batch with both blocks significant
  long lb = b0 - 1;
  int lk = kBatch / kVKs - 1;
  vstep_next(mask, mask_words, b1, I, J, lb, lk);
  if (lb >= b1) return;
  long cb = lb;
  int ck = lk;
  // issue the copies of step (lb, lk) into stage st; returns false past the end
  auto issue = [&](int st) {
    if (lb < b1) {
      const uint32_t *m = mask + lb * mask_words;
      const long qb = pair_off[lb] - p0;
      const double *A = phiT + (size_t)(qb + block_pos(m, I)) * phi_stride_tiles * tile + (size_t)lk * kVKs * kBlockF;
      const double *B = zT + ((size_t)(qb + block_pos(m, J)) * z_stride + zi) * tile + (size_t)lk * kVKs * kBlockF;
      double *dA = vsm + st * kVStageDoubles, *dB = dA + kVKs * kBlockF;
#pragma unroll
      for (int r = 0; r < (kVKs * kBlockF / 2) / 256; ++r) {
        const int e = 2 * (threadIdx.x + 256 * r);
        cp_async16(dA + e, A + e);
        cp_async16(dB + e, B + e);
      }
      vstep_next(mask, mask_words, b1, I, J, lb, lk);
    }
    cp_async_commit();  // an empty group past the end keeps the group count uniform
  };
#pragma unroll
  for (int st = 0; st < kVStages - 1; ++st) issue(st);
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  for (int it = 0; cb < b1; ++it) {
    cp_async_wait<kVStages - 2>();
    __syncthreads();  // step it is visible; the stage refilled below was read in step it - 1
    issue((it + kVStages - 1) % kVStages);
    const double *As = vsm + (it % kVStages) * kVStageDoubles, *Bs = As + kVKs * kBlockF;
#pragma unroll
    for (int k = 0; k < kVKs; ++k) {
      double a[8], bb[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[k * kBlockF + ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; ++j) bb[j] = Bs[k * kBlockF + tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
    vstep_next(mask, mask_words, b1, I, J, cb, ck);
  }
  cp_async_wait<0>();
  double *Vz = V + (size_t)zi * nbf_pad * nbf_pad;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const size_t r = (size_t)I * 128 + ty + 16 * i, c = (size_t)J * 128 + tx + 16 * j;
      Vz[r + c * nbf_pad] += acc[i][j];
    }
}

// out(i, j) = Vp(pi, pj) + Vp(pj, pi), p = finv[.] the plan position of
// caller function i (symmetrise, unpad and undo the plan order)
// Plan-order density of one spin (blockIdx.y) -> caller order: rho and the
// gradient are written, or added to the output with accumulate (the
// "accumulated into" contract of compute_density_and_sigma_sparse,
// nukexc/density.hpp:257-260); sigma = |grad rho|^2 of the resulting
// gradient.  Output planes are npts long: rho[s], grad[3 s + d], sigma[s].
__global__ void density_out_kernel(long npts, long npad, const long *__restrict__ perm, const double *__restrict__ rho,
                                   const double *__restrict__ grad, int accumulate, double *__restrict__ orho,
                                   double *__restrict__ ograd, double *__restrict__ osigma) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (p >= npts) return;
  const long g = perm[p];
  if (orho) {
    const double v = rho[(size_t)s * npad + p];
    orho[(size_t)s * npts + g] = accumulate ? orho[(size_t)s * npts + g] + v : v;
  }
  if (ograd || osigma) {
    double sg = 0.0;
    for (int d = 0; d < 3; ++d) {
      double v = grad[((size_t)s * 3 + d) * npad + p];
      if (ograd) {
        const size_t o = ((size_t)s * 3 + d) * npts + g;
        if (accumulate) v += ograd[o];
        ograd[o] = v;
      }
      sg += v * v;
    }
    if (osigma) osigma[(size_t)s * npts + g] = sg;
  }
}

__global__ void symmetrize_unpad_kernel(int n, int npad, const int *__restrict__ finv, const double *__restrict__ Vp,
                                        double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < n && j < n) {
    const size_t pi = finv[i], pj = finv[j];
    out[(size_t)i + (size_t)j * n] = Vp[pi + pj * npad] + Vp[pj + pi * npad];
  }
}

// C (nbf x nocc column-major, per spin) -> Ct[spin][i][p] = C(fperm[p], i)
// in plan order, zero at padding positions (fperm < 0)
// Orbitals into plan order; a non-finite coefficient or occupation raises
// nonfinite[0] (the build then returns NKX_ERR_NUMERIC).
__global__ void pack_orbitals_kernel(const double *__restrict__ C, const double *__restrict__ occ,
                                     const int *__restrict__ fperm, int nbf, int nocc, int nspin, int nbf_pad,
                                     double *__restrict__ Ct, int *nonfinite) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long tot = (long)nspin * nocc * nbf_pad;
  if (e >= tot) return;
  const int f = fperm[e % nbf_pad];
  const long si = e / nbf_pad;
  const double c = f >= 0 ? C[si * nbf + f] : 0.0;
  Ct[e] = c;
  bool bad = !isfinite(c);
  if (e < (long)nspin * nocc) bad = bad || !isfinite(occ[e]);
  if (bad) atomicOr(nonfinite, 1);
}

// y_a += sum over a slice of points of w_g rho_g V_a(g) for the functions of
// one aux shell: the radial factor once per point, then C S_lm per m
// (coulomb.hpp:84-85).  Every thread of a block works on the same shell, so
// the solid-harmonic branch is uniform.
__global__ void aux_y_shell_kernel(const AuxShell *__restrict__ shells, const int *__restrict__ list,
                                   const double *__restrict__ px, const double *__restrict__ py,
                                   const double *__restrict__ pz, const double *__restrict__ w,
                                   const double *__restrict__ rho, int nspin, long npad, long slice,
                                   const float *__restrict__ rtab, double *__restrict__ y) {
  const int shell = list[blockIdx.x];
  const AuxShell sh = shells[shell];
  const AuxFunc &f = sh.f;
  const long g0 = blockIdx.y * slice, g1 = min(npad, g0 + slice);
  double acc[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) acc[k] = 0.0;
  for (long g = g0 + threadIdx.x; g < g1; g += blockDim.x) {
    double r = rho[g];
    if (nspin == 2) r += rho[npad + g];
    const double wr = w[g] * r;
    if (wr == 0.0) continue;
    const double dx = px[g] - f.cx, dy = py[g] - f.cy, dz = pz[g] - f.cz;
    const double wI =
        wr * (rtab ? (double)rtab[(size_t)shell * npad + g] : f.C * aux_radial(f, sqrt(dx * dx + dy * dy + dz * dz)));
#pragma unroll
    for (int k = 0; k < 15; ++k)
      if (k < sh.nm) acc[k] += wI * solid_harmonic(f.l, f.m + k, dx, dy, dz);
  }
  __shared__ double red[32];
  for (int k = 0; k < sh.nm; ++k) {
    double s = acc[0];
#pragma unroll
    for (int q = 1; q < 15; ++q)
      if (q == k) s = acc[q];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
      for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) atomicAdd(y + sh.first + k, s);
    }
  }
}

// y over the functions of one (centre, l) group of complete shells: per
// point one distance, one set of 2L+1 solid harmonics, then the radial factor
// of each shell (coulomb.hpp:84-85).
// FP32 table of the aux shells' scaled radial factors C R(shell, g), with
// R = I(|r_g - A|) the factor aux_radial evaluates (V_a = C S_lm R), one row
// of npad points per shell.  It depends on the geometry only, so the mixed-precision build
// computes it once per plan and both J passes read it instead of
// re-evaluating the incomplete gamma functions: the grid RI-J's 3-index
// contractions in mixed precision (FP32 operands, FP64 accumulation).
__global__ void aux_rtab_kernel(const AuxShell *__restrict__ shells, int nshell, const double *__restrict__ px,
                                const double *__restrict__ py, const double *__restrict__ pz, long npad,
                                float *__restrict__ rtab) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int sh = blockIdx.y;
  if (g >= npad || sh >= nshell) return;
  const AuxFunc &f = shells[sh].f;
  const double dx = px[g] - f.cx, dy = py[g] - f.cy, dz = pz[g] - f.cz;
  rtab[(size_t)sh * npad + g] = (float)(f.C * aux_radial(f, sqrt(dx * dx + dy * dy + dz * dz)));
}

// TAB: C R from the mixed build's table (no distance powers or radial
// factors evaluated here)
template <int L, bool TAB>
__global__ void __launch_bounds__(256, TAB ? 2 : 1) aux_y_group_kernel(const AuxGroup *__restrict__ groups, const AuxShell *__restrict__ shells,
                                   const double *__restrict__ px, const double *__restrict__ py,
                                   const double *__restrict__ pz, const double *__restrict__ w,
                                   const double *__restrict__ rho, int nspin, long npad, long slice,
                                   const float *__restrict__ rtab, double *__restrict__ y) {
  constexpr int NM = 2 * L + 1, QM = aux_group_max(L);
  const AuxGroup G = groups[blockIdx.x];
  const long g0 = blockIdx.y * slice, g1 = min(npad, g0 + slice);
  double acc[QM][NM];
#pragma unroll
  for (int q = 0; q < QM; ++q)
#pragma unroll
    for (int m = 0; m < NM; ++m) acc[q][m] = 0.0;
  if constexpr (TAB) {
    // two points per thread and iteration, every table load of both issued
    // before use (fixed-count shell loop, loads predicated on the group's
    // size): the loop is load-latency bound otherwise
    const float *tab = rtab + (size_t)G.first * npad;
    for (long ga = g0 + threadIdx.x; ga < g1; ga += 2 * blockDim.x) {
      const long gb = ga + blockDim.x;
      const bool hb = gb < g1;
      double wr[2], S[2][NM];
      float t[2][QM];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const long g = k ? (hb ? gb : ga) : ga;
        double r = rho[g];
        if (nspin == 2) r += rho[npad + g];
        wr[k] = (k == 0 || hb) ? w[g] * r : 0.0;
#pragma unroll
        for (int q = 0; q < QM; ++q) t[k][q] = q < G.n ? tab[(size_t)q * npad + g] : 0.0f;
        solid_harmonics_all<L>(px[g] - G.cx, py[g] - G.cy, pz[g] - G.cz, S[k]);
      }
#pragma unroll
      for (int q = 0; q < QM; ++q) {
        const double wa = wr[0] * (double)t[0][q], wb = wr[1] * (double)t[1][q];
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[q][m] = fma(wb, S[1][m], fma(wa, S[0][m], acc[q][m]));
      }
    }
  } else {
  for (long g = g0 + threadIdx.x; g < g1; g += blockDim.x) {
    double r = rho[g];
    if (nspin == 2) r += rho[npad + g];
    const double wr = w[g] * r;
    if (wr == 0.0) continue;
    const double dx = px[g] - G.cx, dy = py[g] - G.cy, dz = pz[g] - G.cz;
    double S[NM];
    solid_harmonics_all<L>(dx, dy, dz, S);
    {
      const double rr = sqrt(dx * dx + dy * dy + dz * dz);
      const double r2l1inv = rr < 1e-12 ? 0.0 : ipow_c<2 * L + 1>(1.0 / rr);
#pragma unroll
      for (int q = 0; q < QM; ++q) {
        if (q >= G.n) break;
        const AuxFunc &f = shells[G.first + q].f;
        const double wI = wr * (f.C * aux_radial_r(f, rr, r2l1inv));
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[q][m] = fma(wI, S[m], acc[q][m]);
      }
    }
  }
  }
  __shared__ double red[32];
#pragma unroll
  for (int q = 0; q < QM; ++q) {
    if (q >= G.n) break;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      double s = acc[q][m];
      for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      __syncthreads();
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(y + shells[G.first + q].first + m, s);
      }
    }
  }
}

template <int L, bool TAB>
__device__ __forceinline__ double aux_group_v(const AuxGroup &G, const AuxShell *__restrict__ shells,
                                              const double *__restrict__ c, double x, double y, double z,
                                              const float *__restrict__ rtab, long npad, long g) {
  constexpr int NM = 2 * L + 1;
  const double dx = x - G.cx, dy = y - G.cy, dz = z - G.cz;
  double S[NM];
  solid_harmonics_all<L>(dx, dy, dz, S);
  double s = 0.0;
  if constexpr (TAB) {
    for (int q = 0; q < G.n; ++q) {
      const int f0 = shells[G.first + q].first;
      double a = 0.0;
#pragma unroll
      for (int m = 0; m < NM; ++m) a = fma(c[f0 + m], S[m], a);
      s = fma(a, (double)rtab[(size_t)(G.first + q) * npad + g], s);
    }
  } else {
    const double rr = sqrt(dx * dx + dy * dy + dz * dz);
    const double r2l1inv = rr < 1e-12 ? 0.0 : ipow_c<2 * L + 1>(1.0 / rr);
    for (int q = 0; q < G.n; ++q) {
      const AuxShell &sh = shells[G.first + q];
      double a = 0.0;
#pragma unroll
      for (int m = 0; m < NM; ++m) a += c[sh.first + m] * (sh.f.C * S[m]);
      if (a != 0.0) s += a * aux_radial_r(sh.f, rr, r2l1inv);
    }
  }
  return s;
}

// v_g = w_g sum_a c_a V_a(g) over the groups, then the loose shells
// (coulomb.hpp:90-95)
// v of two points (ga, gb) from one group with the C R table: the group's
// data and the fit coefficients are loaded once for both
template <int L>
__device__ __forceinline__ void aux_group_v2_tab(const AuxGroup &G, const AuxShell *__restrict__ shells,
                                                 const double *__restrict__ c, const double (&x)[2],
                                                 const double (&y)[2], const double (&z)[2],
                                                 const float *__restrict__ rtab, long npad, long ga, long gb,
                                                 double (&s)[2]) {
  constexpr int NM = 2 * L + 1;
  double S[2][NM];
  solid_harmonics_all<L>(x[0] - G.cx, y[0] - G.cy, z[0] - G.cz, S[0]);
  solid_harmonics_all<L>(x[1] - G.cx, y[1] - G.cy, z[1] - G.cz, S[1]);
  for (int q = 0; q < G.n; ++q) {
    const int f0 = shells[G.first + q].first;
    const float *row = rtab + (size_t)(G.first + q) * npad;
    const double ra = (double)row[ga], rb = (double)row[gb];
    double a0 = 0.0, a1 = 0.0;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      const double cm = c[f0 + m];
      a0 = fma(cm, S[0][m], a0);
      a1 = fma(cm, S[1][m], a1);
    }
    s[0] = fma(a0, ra, s[0]);
    s[1] = fma(a1, rb, s[1]);
  }
}

// the table form of aux_v_group_kernel: two points per thread
__global__ void aux_v_group_tab_kernel(const AuxGroup *__restrict__ groups, int4 goff,
                                       const AuxShell *__restrict__ shells, const int *__restrict__ loose, int nloose,
                                       const double *__restrict__ c, const double *__restrict__ px,
                                       const double *__restrict__ py, const double *__restrict__ pz,
                                       const double *__restrict__ w, long npad, const float *__restrict__ rtab,
                                       double *__restrict__ v) {
  const long ga = blockIdx.x * 2L * blockDim.x + threadIdx.x;
  if (ga >= npad) return;
  const long gb = min(ga + (long)blockDim.x, npad - 1);  // a duplicate of the last point when past the end
  const double x[2] = {px[ga], px[gb]}, y[2] = {py[ga], py[gb]}, z[2] = {pz[ga], pz[gb]};
  double s[2] = {0.0, 0.0};
  for (int k = 0; k < goff.x; ++k) aux_group_v2_tab<0>(groups[k], shells, c, x, y, z, rtab, npad, ga, gb, s);
  for (int k = goff.x; k < goff.y; ++k) aux_group_v2_tab<1>(groups[k], shells, c, x, y, z, rtab, npad, ga, gb, s);
  for (int k = goff.y; k < goff.z; ++k) aux_group_v2_tab<2>(groups[k], shells, c, x, y, z, rtab, npad, ga, gb, s);
  for (int k = goff.z; k < goff.w; ++k) aux_group_v2_tab<3>(groups[k], shells, c, x, y, z, rtab, npad, ga, gb, s);
  for (int k = 0; k < nloose; ++k) {
    const AuxShell &sh = shells[loose[k]];
    const AuxFunc &f = sh.f;
    const float *row = rtab + (size_t)loose[k] * npad;
    for (int e = 0; e < 2; ++e) {
      double a = 0.0;
      for (int m = 0; m < sh.nm; ++m)
        a += c[sh.first + m] * solid_harmonic(f.l, f.m + m, x[e] - f.cx, y[e] - f.cy, z[e] - f.cz);
      s[e] += a * (double)row[e ? gb : ga];
    }
  }
  v[ga] = s[0] * w[ga];
  if (ga + (long)blockDim.x < npad) v[gb] = s[1] * w[gb];
}

template <bool TAB>
__global__ void aux_v_group_kernel(const AuxGroup *__restrict__ groups, int4 goff,
                                   const AuxShell *__restrict__ shells, const int *__restrict__ loose, int nloose,
                                   const double *__restrict__ c, const double *__restrict__ px,
                                   const double *__restrict__ py, const double *__restrict__ pz,
                                   const double *__restrict__ w, long npad, const float *__restrict__ rtab,
                                   double *__restrict__ v) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= npad) return;
  if (w[g] == 0.0) {
    v[g] = 0.0;
    return;
  }
  const double x = px[g], y = py[g], z = pz[g];
  double s = 0.0;
  // groups sorted by l: [0, goff.x) l = 0, [goff.x, goff.y) l = 1, ...
  for (int k = 0; k < goff.x; ++k) s += aux_group_v<0, TAB>(groups[k], shells, c, x, y, z, rtab, npad, g);
  for (int k = goff.x; k < goff.y; ++k) s += aux_group_v<1, TAB>(groups[k], shells, c, x, y, z, rtab, npad, g);
  for (int k = goff.y; k < goff.z; ++k) s += aux_group_v<2, TAB>(groups[k], shells, c, x, y, z, rtab, npad, g);
  for (int k = goff.z; k < goff.w; ++k) s += aux_group_v<3, TAB>(groups[k], shells, c, x, y, z, rtab, npad, g);
  for (int k = 0; k < nloose; ++k) {
    const AuxShell &sh = shells[loose[k]];
    const AuxFunc &f = sh.f;
    const double dx = x - f.cx, dy = y - f.cy, dz = z - f.cz;
    double a = 0.0;
    for (int m = 0; m < sh.nm; ++m) a += c[sh.first + m] * solid_harmonic(f.l, f.m + m, dx, dy, dz);
    if (a != 0.0)
      s += a * (TAB ? (double)rtab[(size_t)loose[k] * npad + g] : f.C * aux_radial(f, sqrt(dx * dx + dy * dy + dz * dz)));
  }
  v[g] = s * w[g];
}

// Aux collocation phi_A(g) and weighted potential Vw_B(g) of a slice of
// points, column-major naux x np (metric (A|B) set-up, standalone.cxx:443-461)
__global__ void aux_tables_kernel(const StoFunc *__restrict__ sto, const AuxFunc *__restrict__ aux, int naux,
                                  const double *__restrict__ px, const double *__restrict__ py,
                                  const double *__restrict__ pz, const double *__restrict__ w, long g0, long np,
                                  double *__restrict__ phi, double *__restrict__ vw) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= (long)naux * np) return;
  const int a = (int)(e % naux);
  const long g = g0 + e / naux;
  phi[e] = sto_value(sto[a], px[g], py[g], pz[g]);
  vw[e] = aux_potential(aux[a], px[g], py[g], pz[g]) * w[g];
}

// interleaved points xyz[3n] -> planes x[n], y[n], z[n]
__global__ void split_points_kernel(long n, const double *__restrict__ xyz, double *__restrict__ soa) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= n) return;
  for (int d = 0; d < 3; ++d) soa[(size_t)d * n + g] = xyz[3 * g + d];
}

__global__ void gather_kernel(int K, const int *__restrict__ piv, const double *__restrict__ y, double *__restrict__ t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < K) t[i] = y[piv[i]];
}
__global__ void scatter_kernel(int K, const int *__restrict__ piv, const double *__restrict__ t, double *__restrict__ c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < K) c[piv[i]] = t[i];
}

__global__ void sym_half_kernel(int n, double *S) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && j < n && i < j) {
    const double v = 0.5 * (S[(size_t)i + (size_t)j * n] + S[(size_t)j + (size_t)i * n]);
    S[(size_t)i + (size_t)j * n] = v;
    S[(size_t)j + (size_t)i * n] = v;
  }
}

// (A|B) = (M + M^T) / 2 with M_AB = sum_g phi_A(g) w_g V_B(g): the grid
// Coulomb metric of coulomb_overlap_integral(_sparse/_tiled)
// (nukexc/coulomb.hpp:691-813, :827-958), FP64 GEMMs over point slices of at
// most 256 MB of tables; S is naux x naux, column-major, on the device.
static void grid_metric(const StoFunc *d_asto, const AuxFunc *d_aux, int naux, const double *px, const double *py,
                        const double *pz, const double *w, long n, cublasHandle_t hb, cudaStream_t s, double *S) {
  const size_t NA = naux;
  const long slice = std::max<long>(kBatch, std::min<long>(n, (long)((size_t)1 << 28) / (16 * NA)));
  double *sphi = dalloc<double>(NA * slice), *svw = dalloc<double>(NA * slice);
  NKX_CUDA(cudaMemsetAsync(S, 0, sizeof(double) * NA * NA, s));
  for (long g0 = 0; g0 < n; g0 += slice) {
    const long np = std::min(slice, n - g0);
    aux_tables_kernel<<<nblk(NA * np, 128), 128, 0, s>>>(d_asto, d_aux, naux, px, py, pz, w, g0, np, sphi, svw);
    NKX_LAUNCH_CHECK();
    const double one = 1.0;
    NKX_REQUIRE(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, naux, naux, (int)np, &one, sphi, naux, svw, naux, &one, S,
                            naux) == CUBLAS_STATUS_SUCCESS,
                NKX_ERR_CUDA, "cublasDgemm failed");
  }
  dim3 tb(16, 16), gb(nblk(naux, 16), nblk(naux, 16));
  sym_half_kernel<<<gb, tb, 0, s>>>(naux, S);
  NKX_LAUNCH_CHECK();
  NKX_CUDA(cudaStreamSynchronize(s));
  cudaFree(sphi);
  cudaFree(svw);
}

// ========================================================= plan set-up ==

static uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

// Morton (Z-order) permutation of n points xyz[3n]: 21-bit codes per axis
// over the points' bounding box, ties kept in input order.  perm[k] is the
// input index of the k-th point in the order (the space-filling-curve
// permutation of create_bounding_boxes, nukexc/octree.hpp:85-104).
static void morton_order(long n, const double *xyz, std::vector<long> &perm) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (long g = 0; g < n; ++g)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], xyz[3 * g + d]);
      hi[d] = std::max(hi[d], xyz[3 * g + d]);
    }
  // (code, index) pairs sorted lexicographically: the stable Morton order
  std::vector<std::pair<uint64_t, long>> key(n);
#pragma omp parallel for schedule(static)
  for (long g = 0; g < n; ++g) {
    uint64_t c = 0;
    for (int d = 0; d < 3; ++d) {
      const double span = hi[d] > lo[d] ? hi[d] - lo[d] : 1.0;
      const double u = (xyz[3 * g + d] - lo[d]) / span;
      c |= spread3((uint64_t)std::min(2097151.0, std::max(0.0, u * 2097151.0))) << d;
    }
    key[g] = {c, g};
  }
  __gnu_parallel::sort(key.begin(), key.end());
  perm.resize(n);
  for (long g = 0; g < n; ++g) perm[g] = key[g].second;
}

void destroy_mixed_state(void *p);

Plan::~Plan() {
  for (BuildGraph &g : graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (mx_state) destroy_mixed_state(mx_state);
  if (grad_state) destroy_grad_state(grad_state);
  for (void *p : allocs) cudaFree(p);
  if (cublas) cublasDestroy((cublasHandle_t)cublas);
  if (cusolver) cusolverDnDestroy((cusolverDnHandle_t)cusolver);
  for (auto &e : ev) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

template <class T>
T *Plan::alloc(size_t n) {
  T *p = dalloc<T>(n);
  if (p) allocs.push_back(p);
  return p;
}

// Factor of the Coulomb metric held in P.h_metric (naux x naux, column-major,
// symmetrised): the reference's preconditioned half inverse when the plan
// was created with metric_svd_thr > 0, else a pivoted Cholesky of the
// Jacobi-preconditioned metric.  Used at plan creation and by
// nkx_plan_set_metric (the full-grid metric of a grid sharded over ranks).
static void factor_metric(Plan &P) {
  const size_t NA = P.naux;
  NKX_CUDA(cudaMemcpy(P.d_L, P.h_metric.data(), sizeof(double) * NA * NA, cudaMemcpyHostToDevice));
  if (P.svd_mode) {
    // the reference's preconditioned half inverse: c = X X^T y
    int K = 0;
    NKX_REQUIRE(nkx_half_inverse(P.naux, P.d_L, P.metric_svd_thr, P.d_X, &K, P.stream) == NKX_OK,
                NKX_ERR_NUMERIC, "half inverse of the metric failed");
    P.K = K;
    P.metric_min_diag = 0.0;
  } else {
    // Pivoted Cholesky of the Jacobi-preconditioned metric A = D^-1 S D^-1:
    // the grid-integrated (A|B) of an even-tempered aux set is indefinite
    // at the 1e-4 level (diffuse functions reach past the grid), so aux
    // functions whose remaining diagonal falls below kMetricTol are
    // dropped (their fit coefficient is 0) and the kept block is factorised.
    const double kMetricTol = 1e-5;
    std::vector<double> D(NA), A(NA * NA);
    for (size_t i = 0; i < NA; ++i) D[i] = std::sqrt(P.h_metric[i + i * NA]);
    for (size_t j = 0; j < NA; ++j)
      for (size_t i = 0; i < NA; ++i) A[i * NA + j] = P.h_metric[i + j * NA] / (D[i] * D[j]);
    std::vector<double> Lr(NA * NA, 0.0), d(NA);  // row-major rows of L
    std::vector<char> used(NA, 0);
    for (size_t i = 0; i < NA; ++i) d[i] = A[i * NA + i];
    std::vector<int> piv;
    for (size_t k = 0; k < NA; ++k) {
      long p = -1;
      double best = kMetricTol;
      for (size_t i = 0; i < NA; ++i)
        if (!used[i] && d[i] >= best) {
          best = d[i];
          p = (long)i;
        }
      if (p < 0) break;
      used[p] = 1;
      piv.push_back((int)p);
      const double sq = std::sqrt(d[p]);
      const double *lp = &Lr[(size_t)p * NA];
#pragma omp parallel for schedule(static)
      for (long i = 0; i < (long)NA; ++i) {
        if (used[i] && i != p) continue;
        const double *li = &Lr[(size_t)i * NA];
        double acc = A[(size_t)i * NA + p];
        for (size_t c = 0; c < k; ++c) acc -= li[c] * lp[c];
        const double v = acc / sq;
        Lr[(size_t)i * NA + k] = v;
        if (i != p) d[i] -= v * v;
      }
    }
    const int K = (int)piv.size();
    NKX_REQUIRE(K > 0, NKX_ERR_NUMERIC, "aux metric (A|B) has no positive pivot");
    // F = D_sel L_sel, lower triangular K x K in pivot order, column-major
    std::vector<double> F((size_t)K * K, 0.0);
    double mn = 1e300;
    for (int a = 0; a < K; ++a)
      for (int c = 0; c <= a; ++c) F[a + (size_t)c * K] = D[piv[a]] * Lr[(size_t)piv[a] * NA + c];
    for (int a = 0; a < K; ++a) mn = std::min(mn, F[a + (size_t)a * K] / D[piv[a]]);
    P.K = K;
    P.h_piv = piv;
    NKX_CUDA(cudaMemcpy(P.d_L, F.data(), sizeof(double) * K * K, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(P.d_piv, piv.data(), sizeof(int) * K, cudaMemcpyHostToDevice));
    P.metric_min_diag = mn;
  }
}

void Plan::release(void *p) {
  if (!p) return;
  cudaFree(p);
  allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
}

// Device bytes a chunk needs per (batch, block) pair: the FP64 staging of
// four 256 x 128 planes (1 MB) plus the mixed build's int8 digits (1 MB), or
// the FP64 build's three Z planes (0.75 MB).  The default workspace is
// kDefaultWorkspace or a third of the free memory, whichever is smaller.
constexpr size_t kPairBytes = (size_t)2 << 20;
constexpr size_t kDefaultWorkspace = (size_t)24 << 30;

// Chunks of consecutive batches holding at most maxp (batch, block) pairs,
// and the chunk-sized staging: the FP64 planes now; the FP64 build's Z
// planes and the mixed build's digits when a build first needs them.
void plan_chunks(Plan &P, long maxp) {
  P.drop_graphs();
  P.chunks.clear();
  P.max_chunk_pairs = 0;
  long b = 0;
  while (b < P.nbatch) {
    Chunk c;
    c.b0 = b;
    c.p0 = P.h_pair_off[b];
    while (b < P.nbatch && (P.h_pair_off[b + 1] - c.p0 <= maxp || b == c.b0)) ++b;
    c.b1 = b;
    c.p1 = P.h_pair_off[b];
    P.max_chunk_pairs = std::max(P.max_chunk_pairs, c.p1 - c.p0);
    P.chunks.push_back(c);
  }
  P.chunk_pair_limit = maxp;
  // V output tiles of each chunk.  A unit of the V contraction is one
  // (I, J) tile walking the chunk's batches where both blocks are
  // significant; tiles with no such batch get no unit, and the rest are
  // ordered heaviest first (round-robin over the SMs then spreads the heavy
  // tiles evenly).  Ties keep a square-patch order (row blocks in super-rows
  // of about sqrt(SMs)), so that the units running at once share their phi
  // and Z tiles in L2; on a dense problem every tile costs the same and the
  // whole order is the patch order.
  {
    int nsm = 148;
    NKX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P.device));
    const int nb = P.nblk, vrow = std::max(1, std::min(nb, (int)std::lround(std::sqrt((double)nsm))));
    NKX_REQUIRE(nb < (1 << 15), NKX_ERR_UNSUPPORTED, "more than 32767 function blocks");
    std::vector<int> patch;
    patch.reserve((size_t)nb * nb);
    for (int r0 = 0; r0 < nb; r0 += vrow)
      for (int J = 0; J < nb; ++J)
        for (int I = r0; I < std::min(nb, r0 + vrow); ++I) patch.push_back(I * nb + J);
    // pair tiles (R, J) of the CTA-pair V contraction: row blocks 2R and
    // 2R + 1 together, costed by the batches where J and either row block
    // are significant, in the same patch order over about sqrt(SMs / 2) row
    // pairs
    const int nr = (nb + 1) / 2, vrow2 = std::max(1, std::min(nr, (int)std::lround(std::sqrt(nsm / 2.0))));
    std::vector<int> patch2;
    patch2.reserve((size_t)nr * nb);
    for (int r0 = 0; r0 < nr; r0 += vrow2)
      for (int J = 0; J < nb; ++J)
        for (int R = r0; R < std::min(nr, r0 + vrow2); ++R) patch2.push_back(R * nb + J);
    std::vector<int> cnt((size_t)nb * nb), cnt2((size_t)nr * nb), blk, rows, tiles, all, all2;
    for (Chunk &c : P.chunks) {
      std::fill(cnt.begin(), cnt.end(), 0);
      std::fill(cnt2.begin(), cnt2.end(), 0);
      for (long b = c.b0; b < c.b1; ++b) {
        blk.clear();
        rows.clear();
        for (int w = 0; w < P.mask_words; ++w)
          for (uint32_t m = P.h_mask[b * P.mask_words + w]; m; m &= m - 1) blk.push_back(32 * w + __builtin_ctz(m));
        for (int I : blk)
          if (rows.empty() || rows.back() != I / 2) rows.push_back(I / 2);  // blk is ascending
        for (int I : blk)
          for (int J : blk) ++cnt[(size_t)I * nb + J];
        for (int R : rows)
          for (int J : blk) ++cnt2[(size_t)R * nb + J];
      }
      tiles.clear();
      for (int t : patch)
        if (cnt[t]) tiles.push_back(t);
      std::stable_sort(tiles.begin(), tiles.end(), [&](int x, int y) { return cnt[x] > cnt[y]; });
      c.t0 = (long)all.size();
      for (int t : tiles) all.push_back(((t / nb) << 16) | (t % nb));
      c.t1 = (long)all.size();
      tiles.clear();
      for (int t : patch2)
        if (cnt2[t]) tiles.push_back(t);
      std::stable_sort(tiles.begin(), tiles.end(), [&](int x, int y) { return cnt2[x] > cnt2[y]; });
      c.u0 = (long)all2.size();
      for (int t : tiles) all2.push_back(((t / nb) << 16) | (t % nb));
      c.u1 = (long)all2.size();
    }
    P.release(P.d_vtiles);
    P.d_vtiles = P.alloc<int>(std::max<size_t>(1, all.size()));
    if (!all.empty())
      NKX_CUDA(cudaMemcpy(P.d_vtiles, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice));
    P.release(P.d_vtiles2);
    P.d_vtiles2 = P.alloc<int>(std::max<size_t>(1, all2.size()));
    if (!all2.empty())
      NKX_CUDA(cudaMemcpy(P.d_vtiles2, all2.data(), sizeof(int) * all2.size(), cudaMemcpyHostToDevice));
  }
  const size_t tile = (size_t)kBatch * kBlockF;
  P.release(P.ws_phi);
  P.release(P.ws_z);
  P.ws_z = nullptr;
  if (P.mx_state) {
    destroy_mixed_state(P.mx_state);
    P.mx_state = nullptr;
  }
  P.ws_phi = P.alloc<double>(std::max<long>(1, P.max_chunk_pairs) * 4 * tile);
}

static void build_plan(Plan &P, const nkx_molecule *mol, const nkx_basis *prim, const nkx_basis *aux, long npoints,
                       const double *xyz, const double *w, const int *owner, const nkx_plan_options *opts) {
  NKX_REQUIRE(prim && prim->nbf > 0 && npoints > 0 && xyz && w && opts, NKX_ERR_ARG, "invalid arguments");
  NKX_REQUIRE(opts->batch_points == 0 || opts->batch_points == kBatch, NKX_ERR_UNSUPPORTED,
              "batch_points must be 256");
  for (int i = 0; i < prim->nbf; ++i)
    NKX_REQUIRE(prim->l[i] >= 0 && prim->l[i] <= 7 && prim->n[i] > prim->l[i] && abs(prim->m[i]) <= prim->l[i] &&
                    prim->zeta[i] > 0,
                NKX_ERR_UNSUPPORTED, "basis function outside n > l, |m| <= l <= 7, zeta > 0");
  P.xc = make_spec(opts);
  P.gga = spec_is_gga(P.xc);
  NKX_CUDA(cudaGetDevice(&P.device));
  NKX_CUDA(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
  for (auto &e : P.ev) NKX_CUDA(cudaEventCreate(&e));
  P.nbf = prim->nbf;
  P.nblk = (P.nbf + kBlockF - 1) / kBlockF;
  P.nbf_pad = P.nblk * kBlockF;
  P.mask_words = (P.nblk + 31) / 32;
  P.npts = npoints;
  P.nbatch = (npoints + kBatch - 1) / kBatch;
  P.npad = P.nbatch * kBatch;

  // --- Morton order of the points (create_bounding_boxes, octree.hpp:70-110)
  morton_order(npoints, xyz, P.perm);
  std::vector<double> hx(P.npad), hy(P.npad), hz(P.npad), hw(P.npad, 0.0);
  for (long p = 0; p < P.npad; ++p) {
    const long g = P.perm[std::min(p, npoints - 1)];
    hx[p] = xyz[3 * g];
    hy[p] = xyz[3 * g + 1];
    hz[p] = xyz[3 * g + 2];
    if (p < npoints) hw[p] = w[g];
  }

  // --- basis table in plan order (padded positions have norm 0).  Within
  // each 128-function block, position p = 4 lane + c holds the block's
  // function of rank 32 c + lane, ranks sorted by (l, m): the collocation
  // kernels give lane l of a warp positions 4l .. 4l+3, so the 32 lanes
  // evaluating slot c take the same solid-harmonic branch.  Blocks keep
  // their function sets.
  auto tab0 = make_sto_table(*prim);
  // Before that, the functions are grouped by centre (runs of one centre in
  // the caller's order) and the centres put in Morton order of position, so
  // the 128-function blocks are compact in space and screening keeps few
  // blocks per batch even when the caller lists atoms in random order.
  std::vector<int> order(P.nbf);
  {
    struct Run {
      int first, n;
      uint64_t code;
    };
    std::vector<Run> runs;
    auto same_centre = [&](int f, int g) {
      return prim->center[3 * f] == prim->center[3 * g] && prim->center[3 * f + 1] == prim->center[3 * g + 1] &&
             prim->center[3 * f + 2] == prim->center[3 * g + 2];
    };
    for (int f = 0; f < P.nbf; ++f) {
      if (!runs.empty() && same_centre(runs.back().first, f)) {
        ++runs.back().n;
        continue;
      }
      runs.push_back(Run{f, 1, 0});
    }
    double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
    for (const Run &r : runs)
      for (int d = 0; d < 3; ++d) {
        clo[d] = std::min(clo[d], prim->center[3 * r.first + d]);
        chi[d] = std::max(chi[d], prim->center[3 * r.first + d]);
      }
    for (Run &r : runs) {
      uint64_t c = 0;
      for (int d = 0; d < 3; ++d) {
        const double span = chi[d] > clo[d] ? chi[d] - clo[d] : 1.0;
        const double u = (prim->center[3 * r.first + d] - clo[d]) / span;
        c |= spread3((uint64_t)std::min(2097151.0, std::max(0.0, u * 2097151.0))) << d;
      }
      r.code = c;
    }
    std::stable_sort(runs.begin(), runs.end(), [](const Run &a, const Run &b) { return a.code < b.code; });
    int k = 0;
    for (const Run &r : runs)
      for (int i = 0; i < r.n; ++i) order[k++] = r.first + i;
  }
  std::vector<StoFunc> tab(P.nbf_pad);
  P.h_fperm.assign(P.nbf_pad, -1);
  std::vector<int> finv(std::max(1, P.nbf), 0);
  for (int I = 0; I < P.nblk; ++I) {
    std::vector<int> fs;
    for (int q = I * kBlockF; q < std::min(P.nbf, (I + 1) * kBlockF); ++q) fs.push_back(order[q]);
    std::stable_sort(fs.begin(), fs.end(), [&](int x, int y) {
      return tab0[x].l != tab0[y].l ? tab0[x].l < tab0[y].l : tab0[x].m < tab0[y].m;
    });
    for (int k = 0; k < (int)fs.size(); ++k) {
      const int pos = I * kBlockF + 4 * (k % 32) + k / 32;
      P.h_fperm[pos] = fs[k];
      finv[fs[k]] = pos;
    }
  }
  for (int p = 0; p < P.nbf_pad; ++p) {
    if (P.h_fperm[p] >= 0) {
      tab[p] = tab0[P.h_fperm[p]];
    } else {
      tab[p] = tab0[0];
      tab[p].norm = 0.0;
    }
  }
  // --- atoms, point owners (plan order) and the atom of every function, for
  // the nuclear gradient; functions whose centre is on no atom get -1
  if (mol && mol->natoms > 0 && mol->xyz) {
    P.natoms = mol->natoms;
    P.h_centers.assign(mol->xyz, mol->xyz + 3 * (size_t)mol->natoms);
    P.d_centers = P.alloc<double>(3 * (size_t)P.natoms);
    NKX_CUDA(cudaMemcpy(P.d_centers, P.h_centers.data(), sizeof(double) * 3 * P.natoms, cudaMemcpyHostToDevice));

    std::vector<int> fatom(P.nbf_pad, 0);
    P.all_funcs_on_atoms = true;
    for (int q = 0; q < P.nbf_pad; ++q) {
      const int f = P.h_fperm[q];
      if (f < 0) continue;
      int best = -1;
      for (int a = 0; a < P.natoms; ++a) {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          const double e = prim->center[3 * f + d] - mol->xyz[3 * a + d];
          d2 += e * e;
        }
        if (d2 < 1e-20) best = a;
      }
      if (best < 0) P.all_funcs_on_atoms = false;
      fatom[q] = std::max(best, 0);
    }
    P.d_fatom = P.alloc<int>(P.nbf_pad);
    NKX_CUDA(cudaMemcpy(P.d_fatom, fatom.data(), sizeof(int) * P.nbf_pad, cudaMemcpyHostToDevice));
    if (owner) {
      std::vector<int> ho(P.npad, 0);
      for (long p = 0; p < npoints; ++p) {
        const int o = owner[P.perm[p]];
        NKX_REQUIRE(o >= 0 && o < P.natoms, NKX_ERR_ARG, "point owner outside [0, natoms)");
        ho[p] = o;
      }
      P.d_owner = P.alloc<int>(P.npad);
      NKX_CUDA(cudaMemcpy(P.d_owner, ho.data(), sizeof(int) * P.npad, cudaMemcpyHostToDevice));
    }
  }
  // radial shells of every block (functions sharing centre, zeta and
  // n - l - 1), for the collocation kernels' shared radial factors; padding
  // positions (norm 0) point at shell 0
  {
    std::vector<StoShell> hsh((size_t)P.nblk * kBlockF);
    std::vector<int> hns(P.nblk, 0), hfs(P.nbf_pad, 0);
    for (int I = 0; I < P.nblk; ++I) {
      int n = 0;
      StoShell *S = hsh.data() + (size_t)I * kBlockF;
      for (int q = I * kBlockF; q < (I + 1) * kBlockF; ++q) {
        if (P.h_fperm[q] < 0) continue;
        const StoFunc &f = tab[q];
        int s = 0;
        while (s < n && !(S[s].cx == f.cx && S[s].cy == f.cy && S[s].cz == f.cz && S[s].zeta == f.zeta &&
                          S[s].k == f.k))
          ++s;
        if (s == n) S[n++] = StoShell{f.cx, f.cy, f.cz, f.zeta, f.k, 0};
        hfs[q] = s;
      }
      if (n == 0) S[n++] = StoShell{tab[I * kBlockF].cx, tab[I * kBlockF].cy, tab[I * kBlockF].cz, 1.0, 0, 0};
      hns[I] = n;
    }
    P.d_bshell = P.alloc<StoShell>(hsh.size());
    NKX_CUDA(cudaMemcpy(P.d_bshell, hsh.data(), sizeof(StoShell) * hsh.size(), cudaMemcpyHostToDevice));
    P.d_bnshell = P.alloc<int>(P.nblk);
    NKX_CUDA(cudaMemcpy(P.d_bnshell, hns.data(), sizeof(int) * P.nblk, cudaMemcpyHostToDevice));
    P.d_fshell = P.alloc<int>(P.nbf_pad);
    NKX_CUDA(cudaMemcpy(P.d_fshell, hfs.data(), sizeof(int) * P.nbf_pad, cudaMemcpyHostToDevice));
  }
  P.d_fperm = P.alloc<int>(P.nbf_pad);
  NKX_CUDA(cudaMemcpy(P.d_fperm, P.h_fperm.data(), sizeof(int) * P.nbf_pad, cudaMemcpyHostToDevice));
  P.d_finv = P.alloc<int>(finv.size());
  NKX_CUDA(cudaMemcpy(P.d_finv, finv.data(), sizeof(int) * finv.size(), cudaMemcpyHostToDevice));
  const double tol = opts->screen_tol > 0 ? opts->screen_tol : 1e-10;
  auto cut = make_cutoffs(*prim, tol);

  // --- screening: block I is significant for batch b if any function's
  // cutoff sphere meets the batch bounding box (octree.hpp:331-366)
  P.h_mask.assign((size_t)P.nbatch * P.mask_words, 0u);
  P.h_pair_off.assign(P.nbatch + 1, 0);
  // per block, the box holding every function's cutoff sphere: a block whose
  // box misses the batch box has no significant function there
  std::vector<double> blo(3 * (size_t)P.nblk, 1e300), bhi(3 * (size_t)P.nblk, -1e300);
  for (int q = 0; q < P.nbf_pad; ++q) {
    const int f = P.h_fperm[q], I = q / kBlockF;
    if (f < 0) continue;
    for (int d = 0; d < 3; ++d) {
      blo[3 * I + d] = std::min(blo[3 * I + d], prim->center[3 * f + d] - cut[f]);
      bhi[3 * I + d] = std::max(bhi[3 * I + d], prim->center[3 * f + d] + cut[f]);
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (long b = 0; b < P.nbatch; ++b) {
    double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
    for (int g = 0; g < kBatch; ++g) {
      const long p = b * kBatch + g;
      const double v[3] = {hx[p], hy[p], hz[p]};
      for (int d = 0; d < 3; ++d) {
        bl[d] = std::min(bl[d], v[d]);
        bh[d] = std::max(bh[d], v[d]);
      }
    }
    for (int I = 0; I < P.nblk; ++I) {
      bool near = true;
      for (int d = 0; d < 3; ++d) near = near && blo[3 * I + d] <= bh[d] && bhi[3 * I + d] >= bl[d];
      if (!near) continue;
      bool sig = false;
      for (int q = I * kBlockF; q < (I + 1) * kBlockF && !sig; ++q) {
        const int f = P.h_fperm[q];
        if (f < 0) continue;
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          const double c = prim->center[3 * f + d];
          const double e = c < bl[d] ? bl[d] - c : (c > bh[d] ? c - bh[d] : 0.0);
          d2 += e * e;
        }
        sig = d2 <= cut[f] * cut[f];
      }
      if (sig) P.h_mask[b * P.mask_words + I / 32] |= 1u << (I % 32);
    }
  }
  std::vector<int> pblk, pbatch;
  for (long b = 0; b < P.nbatch; ++b) {
    for (int I = 0; I < P.nblk; ++I)
      if ((P.h_mask[b * P.mask_words + I / 32] >> (I % 32)) & 1u) {
        pblk.push_back(I);
        pbatch.push_back((int)b);
      }
    P.h_pair_off[b + 1] = (int)pblk.size();
  }
  P.npairs = (long)pblk.size();

  // --- device copies
  P.d_px = P.alloc<double>(P.npad);
  P.d_py = P.alloc<double>(P.npad);
  P.d_pz = P.alloc<double>(P.npad);
  P.d_w = P.alloc<double>(P.npad);
  NKX_CUDA(cudaMemcpy(P.d_px, hx.data(), sizeof(double) * P.npad, cudaMemcpyHostToDevice));
  NKX_CUDA(cudaMemcpy(P.d_py, hy.data(), sizeof(double) * P.npad, cudaMemcpyHostToDevice));
  NKX_CUDA(cudaMemcpy(P.d_pz, hz.data(), sizeof(double) * P.npad, cudaMemcpyHostToDevice));
  NKX_CUDA(cudaMemcpy(P.d_w, hw.data(), sizeof(double) * P.npad, cudaMemcpyHostToDevice));
  P.d_sto = P.alloc<StoFunc>(P.nbf_pad);
  NKX_CUDA(cudaMemcpy(P.d_sto, tab.data(), sizeof(StoFunc) * P.nbf_pad, cudaMemcpyHostToDevice));
  P.d_mask = P.alloc<uint32_t>(P.h_mask.size());
  NKX_CUDA(cudaMemcpy(P.d_mask, P.h_mask.data(), sizeof(uint32_t) * P.h_mask.size(), cudaMemcpyHostToDevice));
  P.d_pair_off = P.alloc<int>(P.nbatch + 1);
  NKX_CUDA(cudaMemcpy(P.d_pair_off, P.h_pair_off.data(), sizeof(int) * (P.nbatch + 1), cudaMemcpyHostToDevice));
  P.d_pair_blk = P.alloc<int>(std::max<long>(1, P.npairs));
  P.d_pair_batch = P.alloc<int>(std::max<long>(1, P.npairs));
  if (P.npairs) {
    NKX_CUDA(cudaMemcpy(P.d_pair_blk, pblk.data(), sizeof(int) * P.npairs, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(P.d_pair_batch, pbatch.data(), sizeof(int) * P.npairs, cudaMemcpyHostToDevice));
  }

  // --- chunks of batches sized by the workspace
  size_t ws = opts->workspace_bytes;
  if (ws == 0) {
    size_t fr = 0, tot = 0;
    NKX_CUDA(cudaMemGetInfo(&fr, &tot));
    ws = std::min<size_t>(kDefaultWorkspace, fr / 3);
  }
  plan_chunks(P, std::max<long>(1, (long)(ws / kPairBytes)));

  // per-point arrays (two spins)
  P.d_rho = P.alloc<double>(2 * P.npad);
  P.d_grad = P.alloc<double>(6 * P.npad);
  P.d_coef = P.alloc<double>(8 * P.npad);
  P.d_vj = P.alloc<double>(P.npad);
  P.d_V = P.alloc<double>(3 * (size_t)P.nbf_pad * P.nbf_pad);
  P.d_E = P.alloc<double>(1);
  P.d_status = P.alloc<int>(2);
  NKX_CUDA(cudaMemset(P.d_status, 0, sizeof(int) * 2));
  NKX_CUDA(cudaMemset(P.d_rho, 0, sizeof(double) * 2 * P.npad));
  NKX_CUDA(cudaMemset(P.d_grad, 0, sizeof(double) * 6 * P.npad));

  // --- aux metric and its factor
  if (aux && aux->nbf > 0) {
    for (int i = 0; i < aux->nbf; ++i)
      NKX_REQUIRE(aux->l[i] >= 0 && aux->l[i] <= 7 && aux->n[i] > aux->l[i] && abs(aux->m[i]) <= aux->l[i] &&
                      aux->zeta[i] > 0,
                  NKX_ERR_UNSUPPORTED, "aux function outside n > l, |m| <= l <= 7, zeta > 0");
    P.naux = aux->nbf;
    auto atab = make_aux_table(*aux);
    auto astab = make_sto_table(*aux);
    P.d_aux = P.alloc<AuxFunc>(P.naux);
    NKX_CUDA(cudaMemcpy(P.d_aux, atab.data(), sizeof(AuxFunc) * P.naux, cudaMemcpyHostToDevice));
    const auto ash = make_aux_shells(atab);
    P.nashell = (int)ash.size();
    P.d_ashell = P.alloc<AuxShell>(ash.size());
    NKX_CUDA(cudaMemcpy(P.d_ashell, ash.data(), sizeof(AuxShell) * ash.size(), cudaMemcpyHostToDevice));
    std::vector<int> loose;
    const auto grp = make_aux_groups(ash, loose);
    P.nagroup = (int)grp.size();
    P.nloose = (int)loose.size();
    P.h_group_off.assign(5, 0);
    for (const AuxGroup &G : grp) ++P.h_group_off[G.l + 1];
    for (int L = 0; L < 4; ++L) P.h_group_off[L + 1] += P.h_group_off[L];
    P.d_agroup = P.alloc<AuxGroup>(std::max<size_t>(1, grp.size()));
    if (!grp.empty())
      NKX_CUDA(cudaMemcpy(P.d_agroup, grp.data(), sizeof(AuxGroup) * grp.size(), cudaMemcpyHostToDevice));
    P.d_loose = P.alloc<int>(std::max<size_t>(1, loose.size()));
    if (!loose.empty())
      NKX_CUDA(cudaMemcpy(P.d_loose, loose.data(), sizeof(int) * loose.size(), cudaMemcpyHostToDevice));
    StoFunc *d_asto = dalloc<StoFunc>(P.naux);
    NKX_CUDA(cudaMemcpy(d_asto, astab.data(), sizeof(StoFunc) * P.naux, cudaMemcpyHostToDevice));
    const size_t NA = P.naux;
    P.d_L = P.alloc<double>(NA * NA);
    P.d_y = P.alloc<double>(NA);
    P.d_c = P.alloc<double>(NA);
    P.d_info = P.alloc<int>(1);
    cublasHandle_t hb;
    NKX_REQUIRE(cublasCreate(&hb) == CUBLAS_STATUS_SUCCESS, NKX_ERR_CUDA, "cublasCreate failed");
    P.cublas = hb;
    cublasSetStream(hb, P.stream);
    grid_metric(d_asto, P.d_aux, P.naux, P.d_px, P.d_py, P.d_pz, P.d_w, P.npad, hb, P.stream, P.d_L);
    cudaFree(d_asto);
    P.h_metric.resize(NA * NA);
    NKX_CUDA(cudaMemcpy(P.h_metric.data(), P.d_L, sizeof(double) * NA * NA, cudaMemcpyDeviceToHost));
    cusolverDnHandle_t hs;
    NKX_REQUIRE(cusolverDnCreate(&hs) == CUSOLVER_STATUS_SUCCESS, NKX_ERR_CUDA, "cusolverDnCreate failed");
    P.cusolver = hs;
    cusolverDnSetStream(hs, P.stream);
    P.svd_mode = opts->metric_svd_thr > 0;
    P.metric_svd_thr = opts->metric_svd_thr;
    P.d_X = P.svd_mode ? P.alloc<double>(NA * NA) : nullptr;
    P.d_t = P.alloc<double>(NA);
    P.d_piv = P.alloc<int>(NA);
    factor_metric(P);
  }
  NKX_CUDA(cudaStreamSynchronize(P.stream));
}

// ------------------------------------------------- core Hamiltonian ----
// w_g v_n(g) = w_g sum_A Z_A / (|r_g - R_A| + 1e-30), the nuclear attraction
// weight of core_hamiltonian.hpp:133-289 (V_n = -sum_g w v_n phi phi^T)
__global__ void core_vne_kernel(const double *__restrict__ px, const double *__restrict__ py,
                                const double *__restrict__ pz, const double *__restrict__ w, long npad,
                                const double *__restrict__ centers, const double *__restrict__ charges, int natoms,
                                double *__restrict__ wv) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= npad) return;
  double v = 0.0;
  if (w[g] != 0.0)
    for (int a = 0; a < natoms; ++a) {
      const double dx = px[g] - centers[3 * a], dy = py[g] - centers[3 * a + 1], dz = pz[g] - centers[3 * a + 2];
      v += charges[a] / (sqrt(dx * dx + dy * dy + dz * dz) + 1e-30);
    }
  wv[g] = w[g] * v;
}

// Z planes of the core Hamiltonian for the pairs of one chunk, Z^T[pair][3][g][f]
// from PhiT[pair][4][g][f]: pass 0: plane 0 = 1/2 w phi (S), plane 1 =
// -1/2 w v_n phi (V_n); pass 1: plane k = 1/4 w d_k phi (T, k = x, y, z), so
// that Vbar + Vbar^T of each contraction is the matrix itself.
__global__ void core_z_kernel(const double *__restrict__ phiT, const double *__restrict__ w,
                              const double *__restrict__ wv, const int *__restrict__ pair_batch, long p0, int pass,
                              double *__restrict__ zT) {
  const size_t tile = (size_t)kBatch * kBlockF;
  const long q = blockIdx.x;
  const long b = pair_batch[p0 + q];
  const double *P = phiT + (size_t)q * 4 * tile;
  double *Z = zT + (size_t)q * 3 * tile;
  for (int e = threadIdx.x; e < (int)tile; e += blockDim.x) {
    const long g = b * kBatch + e / kBlockF;
    if (pass == 0) {
      Z[e] = 0.5 * w[g] * P[e];
      Z[tile + e] = -0.5 * wv[g] * P[e];
    } else {
      const double h = 0.25 * w[g];
      Z[e] = h * P[tile + e];
      Z[2 * tile + e] = h * P[3 * tile + e];
      Z[tile + e] = h * P[2 * tile + e];
    }
  }
}

// ========================================================= Fock build ===

void launch_colloc(Plan &P, const Chunk &c, cudaStream_t s) {
  const long np = c.p1 - c.p0;
  if (np <= 0) return;
  if (P.gga)
    colloc_fp64_kernel<true><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_px, P.d_py, P.d_pz, P.d_pair_batch,
                                                          P.d_pair_blk, c.p0, P.ws_phi);
  else
    colloc_fp64_kernel<false><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_px, P.d_py, P.d_pz, P.d_pair_batch,
                                                           P.d_pair_blk, c.p0, P.ws_phi);
  NKX_LAUNCH_CHECK();
  ++P.launches;
}

// The grid RI-J fit (coulomb.hpp:84-95) in two steps, so that a grid
// sharded over ranks can sum y between them: coulomb_y forms this plan's
// y = Vw rho_total over its points; coulomb_solve solves c = (A|B)^-1 y
// (pivoted Cholesky or half inverse) and forms v_g = w_g sum_a c_a V_a(g).
// The FP64 build evaluates the potentials' radial factors; the mixed build
// reads them from the plan's FP32 table when it fits (coulomb_table).
// The FP32 radial-factor table of the mixed build (aux_rtab_kernel), made on
// first use when it fits in a quarter of the free device memory (and
// kRtabMaxBytes); otherwise the J passes evaluate the factors as FP64 does.
constexpr size_t kRtabMaxBytes = (size_t)32 << 30;
static const float *coulomb_table(Plan &P, bool mixed, cudaStream_t s) {
  if (!mixed || P.rtab_failed) return nullptr;
  if (!P.d_rtab) {
    const size_t bytes = (size_t)P.nashell * P.npad * sizeof(float);
    size_t fr = 0, tot = 0;
    NKX_CUDA(cudaMemGetInfo(&fr, &tot));
    if (bytes > kRtabMaxBytes || bytes > fr / 4 || cudaMalloc(&P.d_rtab, bytes) != cudaSuccess) {
      cudaGetLastError();
      P.d_rtab = nullptr;
      P.rtab_failed = true;
      return nullptr;
    }
    P.allocs.push_back(P.d_rtab);
    aux_rtab_kernel<<<dim3(nblk(P.npad, 256), (unsigned)P.nashell), 256, 0, s>>>(P.d_ashell, P.nashell, P.d_px, P.d_py,
                                                                                P.d_pz, P.npad, P.d_rtab);
    NKX_LAUNCH_CHECK();
    ++P.launches;
  }
  return P.d_rtab;
}

void coulomb_y(Plan &P, int nspin, cudaStream_t s, bool mixed) {
    const float *rtab = coulomb_table(P, mixed, s);
    NKX_CUDA(cudaMemsetAsync(P.d_y, 0, sizeof(double) * P.naux, s));
    const long nsl = std::max<long>(1, std::min<long>(64, (P.npad + 4095) / 4096));
    const long slice = (P.npad + nsl - 1) / nsl;
    for (int L = 0; L <= 3; ++L) {
      const int n = P.h_group_off[L + 1] - P.h_group_off[L];
      if (n == 0) continue;
      const AuxGroup *gp = P.d_agroup + P.h_group_off[L];
      const dim3 gy((unsigned)n, (unsigned)nsl);
      switch (L) {
        case 0:
          if (rtab)
            aux_y_group_kernel<0, true><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          else
            aux_y_group_kernel<0, false><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          break;
        case 1:
          if (rtab)
            aux_y_group_kernel<1, true><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          else
            aux_y_group_kernel<1, false><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          break;
        case 2:
          if (rtab)
            aux_y_group_kernel<2, true><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          else
            aux_y_group_kernel<2, false><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          break;
        default:
          if (rtab)
            aux_y_group_kernel<3, true><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          else
            aux_y_group_kernel<3, false><<<gy, 256, 0, s>>>(gp, P.d_ashell, P.d_px, P.d_py, P.d_pz, P.d_w, P.d_rho, nspin, P.npad, slice, rtab, P.d_y);
          break;
      }
      NKX_LAUNCH_CHECK();
      ++P.launches;
    }
    if (P.nloose > 0) {
      aux_y_shell_kernel<<<dim3(P.nloose, (unsigned)nsl), 256, 0, s>>>(P.d_ashell, P.d_loose, P.d_px, P.d_py, P.d_pz,
                                                                      P.d_w, P.d_rho, nspin, P.npad, slice, rtab,
                                                                      P.d_y);
      NKX_LAUNCH_CHECK();
      ++P.launches;
    }
}

void coulomb_solve(Plan &P, cudaStream_t s, bool mixed) {
    const float *rtab = coulomb_table(P, mixed, s);
    if (P.svd_mode) {
      const double one = 1.0, zero = 0.0;
      cublasHandle_t hb = (cublasHandle_t)P.cublas;
      cublasSetStream(hb, s);
      NKX_REQUIRE(cublasDgemv(hb, CUBLAS_OP_T, P.naux, P.K, &one, P.d_X, P.naux, P.d_y, 1, &zero, P.d_t, 1) ==
                          CUBLAS_STATUS_SUCCESS &&
                      cublasDgemv(hb, CUBLAS_OP_N, P.naux, P.K, &one, P.d_X, P.naux, P.d_t, 1, &zero, P.d_c, 1) ==
                          CUBLAS_STATUS_SUCCESS,
                  NKX_ERR_CUDA, "cublasDgemv failed");
    } else {
      gather_kernel<<<nblk(P.K, 128), 128, 0, s>>>(P.K, P.d_piv, P.d_y, P.d_t);
      cusolverDnHandle_t hs = (cusolverDnHandle_t)P.cusolver;
      cusolverDnSetStream(hs, s);
      NKX_REQUIRE(cusolverDnDpotrs(hs, CUBLAS_FILL_MODE_LOWER, P.K, 1, P.d_L, P.K, P.d_t, P.K, P.d_info) ==
                      CUSOLVER_STATUS_SUCCESS,
                  NKX_ERR_CUDA, "cusolverDnDpotrs failed");
      NKX_CUDA(cudaMemsetAsync(P.d_c, 0, sizeof(double) * P.naux, s));
      scatter_kernel<<<nblk(P.K, 128), 128, 0, s>>>(P.K, P.d_piv, P.d_t, P.d_c);
      NKX_LAUNCH_CHECK();
      P.launches += 2;
    }
    const int4 goff = make_int4(P.h_group_off[1], P.h_group_off[2], P.h_group_off[3], P.h_group_off[4]);
    if (rtab)
      aux_v_group_tab_kernel<<<nblk(P.npad, 256), 128, 0, s>>>(P.d_agroup, goff, P.d_ashell, P.d_loose, P.nloose,
                                                               P.d_c, P.d_px, P.d_py, P.d_pz, P.d_w, P.npad, rtab,
                                                               P.d_vj);
    else
      aux_v_group_kernel<false><<<nblk(P.npad, 128), 128, 0, s>>>(P.d_agroup, goff, P.d_ashell, P.d_loose, P.nloose,
                                                                  P.d_c, P.d_px, P.d_py, P.d_pz, P.d_w, P.npad, rtab,
                                                                  P.d_vj);
    NKX_LAUNCH_CHECK();
    ++P.launches;
}

// FP64 pass A: collocation + density of every chunk into d_rho / d_grad
void fp64_density_pass(Plan &P, int nspin, int nocc, cudaStream_t s, StageTimer &T) {
  const int nocc_pad = (nocc + 63) / 64 * 64;
  if ((size_t)nocc_pad * P.nbf_pad * 2 > P.cf_cap) {
    P.cf_cap = (size_t)nocc_pad * P.nbf_pad * 2;
    P.d_Cf = P.alloc<double>(P.cf_cap);
  }
  transpose_orbitals_kernel<<<dim3(P.nbf_pad / 32, nocc_pad / 32, nspin), dim3(32, 8), 0, s>>>(P.d_Ct, nocc, nocc_pad,
                                                                                             P.nbf_pad, P.d_Cf);
  NKX_LAUNCH_CHECK();
  ++P.launches;
  NKX_CUDA(cudaFuncSetAttribute(density_fp64_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kDSmemBytes<true>));
  NKX_CUDA(cudaFuncSetAttribute(density_fp64_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kDSmemBytes<false>));
  // the density kernels add their orbital tiles' shares
  NKX_CUDA(cudaMemsetAsync(P.d_rho, 0, sizeof(double) * nspin * P.npad, s));
  if (P.gga) NKX_CUDA(cudaMemsetAsync(P.d_grad, 0, sizeof(double) * 3 * nspin * P.npad, s));
  for (const Chunk &c : P.chunks) {
    const long nb = c.b1 - c.b0;
    if (c.p1 - c.p0 > 0) {
      T.begin(ST_COLLOC, s);
      launch_colloc(P, c, s);
      T.end(s);
    }
    T.begin(ST_DENSITY, s);
    dim3 grid((unsigned)(nb * 4 * (nocc_pad / 64)), nspin);
    if (P.gga)
      density_fp64_kernel<true><<<grid, 256, kDSmemBytes<true>, s>>>(P.ws_phi, P.d_Cf, P.d_occ, nocc, nocc_pad, P.nbf_pad, P.d_pair_off,
                                                     P.d_pair_blk, c.b0, c.p0, P.d_rho, P.d_grad, P.npad);
    else
      density_fp64_kernel<false><<<grid, 256, kDSmemBytes<false>, s>>>(P.ws_phi, P.d_Cf, P.d_occ, nocc, nocc_pad, P.nbf_pad, P.d_pair_off,
                                                      P.d_pair_blk, c.b0, c.p0, P.d_rho, P.d_grad, P.npad);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    T.end(s);
  }
}

void fock_build_fp64(Plan &P, int nspin, int nocc, bool needJ, bool fuse, bool separateJ, cudaStream_t s,
                     StageTimer &T, int phase) {
  const bool multi = P.chunks.size() > 1;
  const int nzs = nspin + (separateJ ? 1 : 0);
  if (!P.ws_z) P.ws_z = P.alloc<double>(std::max<long>(1, P.max_chunk_pairs) * 3 * (size_t)kBatch * kBlockF);
  NKX_CUDA(cudaFuncSetAttribute(vgemm_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kVSmemBytes));
  if (phase != 2) {
    // ---- pass A: collocation + density, and this plan's share of the J fit vector
    fp64_density_pass(P, nspin, nocc, s, T);
    if (needJ) {
      T.begin(ST_COULOMB, s);
      coulomb_y(P, nspin, s, false);
      T.end(s);
    }
    if (phase == 1) return;
  }
  // ---- J: fit coefficients and fitted potential
  if (needJ) {
    T.begin(ST_COULOMB, s);
    coulomb_solve(P, s, false);
    T.end(s);
  }
  // ---- functional
  T.begin(ST_FUNC, s);
  NKX_CUDA(cudaMemsetAsync(P.d_E, 0, sizeof(double), s));
  functional_kernel<<<nblk(P.npad, 256), 256, 0, s>>>(P.xc, P.gga, nspin, P.npad, P.npad, P.d_w, P.d_rho, P.d_grad,
                                                      (needJ && fuse) ? P.d_vj : nullptr, P.d_coef, P.d_E,
                                                      nullptr);
  NKX_LAUNCH_CHECK();
  ++P.launches;
  T.end(s);
  // ---- pass B: Z and the V contraction
  const size_t tile = (size_t)kBatch * kBlockF;
  NKX_CUDA(cudaMemsetAsync(P.d_V, 0, sizeof(double) * nzs * P.nbf_pad * P.nbf_pad, s));
  for (const Chunk &c : P.chunks) {
    const long np = c.p1 - c.p0;
    if (np <= 0) continue;
    if (multi) {
      T.begin(ST_COLLOC, s);
      launch_colloc(P, c, s);
      T.end(s);
    }
    T.begin(ST_ZBUILD, s);
    if (P.gga)
      zbuild_fp64_kernel<true><<<(unsigned)np, 256, 0, s>>>(P.ws_phi, P.d_coef, P.d_vj, P.d_pair_batch, c.p0, nzs,
                                                            nspin, P.npad, P.ws_z);
    else
      zbuild_fp64_kernel<false><<<(unsigned)np, 256, 0, s>>>(P.ws_phi, P.d_coef, P.d_vj, P.d_pair_batch, c.p0, nzs,
                                                             nspin, P.npad, P.ws_z);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    T.end(s);
    T.begin(ST_VGEMM, s);
    vgemm_fp64_kernel<<<dim3(P.nblk, P.nblk, nzs), 256, kVSmemBytes, s>>>(P.ws_phi, P.ws_z, P.gga ? 4 : 1, nzs, P.d_pair_off,
                                                                P.d_mask, P.mask_words, c.b0, c.b1, c.p0, P.nbf_pad,
                                                                P.d_V);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    T.end(s);
  }
  (void)tile;
}

// orbitals -> Ct[spin][i][p] in plan order (host or device C / occ)
void upload_orbitals(Plan &P, int nspin, int nocc, const double *C, const double *occ, int mem, cudaStream_t s) {
  if (nocc > P.nocc_cap) {
    P.nocc_cap = nocc;
    P.d_Ct = P.alloc<double>((size_t)2 * nocc * P.nbf_pad);
    P.d_occ = P.alloc<double>((size_t)2 * nocc);
    P.d_Cin = P.alloc<double>((size_t)2 * nocc * P.nbf);
  }
  const double *Cd = C;
  if (mem == NKX_MEM_HOST) {
    NKX_CUDA(cudaMemcpyAsync(P.d_Cin, C, sizeof(double) * nspin * nocc * P.nbf, cudaMemcpyHostToDevice, s));
    NKX_CUDA(cudaMemcpyAsync(P.d_occ, occ, sizeof(double) * nspin * nocc, cudaMemcpyHostToDevice, s));
    Cd = P.d_Cin;
  } else {
    NKX_CUDA(cudaMemcpyAsync(P.d_occ, occ, sizeof(double) * nspin * nocc, cudaMemcpyDeviceToDevice, s));
  }
  pack_orbitals_kernel<<<nblk((long)nspin * nocc * P.nbf_pad, 256), 256, 0, s>>>(
      Cd, P.d_occ, P.d_fperm, P.nbf, nocc, nspin, P.nbf_pad, P.d_Ct, P.d_status + 1);
  NKX_LAUNCH_CHECK();
  ++P.launches;
}

// One Fock build (phase 0), or one half of a build whose grid is sharded
// over ranks: phase 1 uploads the orbitals, runs the density pass and writes
// this plan's share of the J fit vector y to `y` (naux doubles, host or
// device by `mem`); the caller sums y over the ranks; phase 2 takes the
// summed y (same memory kind) and finishes the build (fit, functional, V and
// J on this plan's points).  Phase 2 needs a phase 1 of the same
// precision, spin count and orbitals on this plan immediately before it.
// One build on the stream.  capture_only (device buffers, phase 0): only the
// device work is issued -- no events, host copies, synchronisation or status
// check -- so that it can be recorded into a CUDA graph.
static void fock_build_once(Plan &P, int precision, int nspin, int nocc, const double *C, const double *occ, int mem,
                            int fuse_j, double *E, double *V, double *J, cudaStream_t user, int phase, double *y,
                            bool capture_only) {
  if (phase == 2) {
    NKX_REQUIRE(P.phase1_done, NKX_ERR_ARG, "phase 2 of a sharded build needs phase 1 on this plan first");
    precision = P.phase1_precision;
    nspin = P.phase1_nspin;
    nocc = P.phase1_nocc;
  }
  NKX_REQUIRE(nspin == 1 || nspin == 2, NKX_ERR_ARG, "nspin must be 1 or 2");
  NKX_REQUIRE(phase == 2 || (nocc > 0 && C && occ), NKX_ERR_ARG, "invalid orbitals");
  NKX_REQUIRE(phase == 1 || (E && (V || J)), NKX_ERR_ARG, "invalid outputs");
  NKX_REQUIRE(phase == 0 || (y && P.naux > 0), NKX_ERR_ARG, "a sharded build needs y and a plan with an aux basis");
  NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
  NKX_REQUIRE(precision == NKX_PREC_FP64 || precision == NKX_PREC_MIXED, NKX_ERR_ARG, "unknown precision");
  const bool needJ = P.naux > 0 && (J != nullptr || fuse_j || phase != 0);
  NKX_REQUIRE(!(fuse_j && P.naux == 0), NKX_ERR_ARG, "fuse_j needs a plan with an aux basis");
  // V may be NULL only when J alone is asked for (the exchange-correlation
  // terms are then formed and dropped)
  NKX_REQUIRE(phase == 1 || V != nullptr || (J != nullptr && !fuse_j && P.naux > 0), NKX_ERR_ARG,
              "V must be given unless J alone is requested from a plan with an aux basis");
  const bool separateJ = needJ && !fuse_j && J;
  cudaStream_t s = user ? user : P.stream;
  P.launches = 0;
  StageTimer T;
  T.on = !capture_only;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (!capture_only) {
    NKX_CUDA(cudaEventCreate(&t0));
    NKX_CUDA(cudaEventCreate(&t1));
    NKX_CUDA(cudaEventRecord(t0, s));
  }
  P.phase1_done = false;
  if (phase == 2) {
    NKX_CUDA(cudaMemcpyAsync(P.d_y, y, sizeof(double) * P.naux,
                             mem == NKX_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  } else {
    NKX_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int) * 2, s));
    upload_orbitals(P, nspin, nocc, C, occ, mem, s);
  }

  const bool mixed = precision == NKX_PREC_MIXED && mixed_available(P);
  NKX_REQUIRE(mixed || precision == NKX_PREC_FP64, NKX_ERR_UNSUPPORTED, "mixed precision path unavailable");
  if (mixed)
    fock_build_mixed(P, nspin, nocc, needJ, fuse_j != 0, separateJ, s, T, phase);
  else
    fock_build_fp64(P, nspin, nocc, needJ, fuse_j != 0, separateJ, s, T, phase);

  if (phase == 1) {
    NKX_CUDA(cudaMemcpyAsync(y, P.d_y, sizeof(double) * P.naux,
                             mem == NKX_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    int status[2] = {0, 0};
    NKX_CUDA(cudaMemcpyAsync(status, P.d_status, sizeof(status), cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaEventRecord(t1, s));
    NKX_CUDA(cudaStreamSynchronize(s));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    NKX_REQUIRE(status[0] == 0, NKX_ERR_TIMEOUT, "a tensor-core kernel wait gave up in phase 1");
    NKX_REQUIRE(status[1] == 0, NKX_ERR_NUMERIC, "non-finite value in the orbitals, occupations or an operand");
    P.phase1_done = true;
    P.phase1_precision = precision;
    P.phase1_nspin = nspin;
    P.phase1_nocc = nocc;
    return;
  }

  // symmetrise + unpad into the output (device) or a staging buffer (host)
  const size_t nn = (size_t)P.nbf * P.nbf;
  const int nout = nspin + (separateJ ? 1 : 0);
  double *dst = nullptr;
  if (mem == NKX_MEM_DEVICE) {
    dst = V;
  } else {
    if (!P.d_out) P.d_out = P.alloc<double>(3 * nn);
    dst = P.d_out;
  }
  dim3 tb(16, 16), gb(nblk(P.nbf, 16), nblk(P.nbf, 16));
  for (int z = 0; z < nout; ++z) {
    if (z < nspin && !V) continue;
    double *o = (z < nspin) ? dst + z * nn : (mem == NKX_MEM_DEVICE ? J : dst + nspin * nn);
    symmetrize_unpad_kernel<<<gb, tb, 0, s>>>(P.nbf, P.nbf_pad, P.d_finv, P.d_V + (size_t)z * P.nbf_pad * P.nbf_pad,
                                              o);
    ++P.launches;
  }
  NKX_LAUNCH_CHECK();
  if (capture_only) return;
  if (mem == NKX_MEM_HOST) {
    if (V) NKX_CUDA(cudaMemcpyAsync(V, dst, sizeof(double) * nspin * nn, cudaMemcpyDeviceToHost, s));
    if (separateJ) NKX_CUDA(cudaMemcpyAsync(J, dst + nspin * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
  }
  NKX_CUDA(cudaMemcpyAsync(E, P.d_E, sizeof(double), cudaMemcpyDeviceToHost, s));
  int status[2] = {0, 0};
  NKX_CUDA(cudaMemcpyAsync(status, P.d_status, sizeof(status), cudaMemcpyDeviceToHost, s));
  NKX_CUDA(cudaEventRecord(t1, s));
  NKX_CUDA(cudaStreamSynchronize(s));
  float st[6];
  T.collect(st);
  P.last.colloc_ms = st[ST_COLLOC];
  P.last.density_ms = st[ST_DENSITY];
  P.last.functional_ms = st[ST_FUNC];
  P.last.coulomb_ms = st[ST_COULOMB];
  P.last.zbuild_ms = st[ST_ZBUILD];
  P.last.vgemm_ms = st[ST_VGEMM];
  cudaEventElapsedTime(&P.last.total_ms, t0, t1);
  P.last.launches = P.launches;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  P.last_nspin = nspin;
  NKX_REQUIRE(status[0] == 0, NKX_ERR_TIMEOUT,
              "a tensor-core kernel wait gave up (wait code " + std::to_string(status[0]) + "); outputs are invalid");
  NKX_REQUIRE(status[1] == 0 && std::isfinite(*E), NKX_ERR_NUMERIC,
              "non-finite value in the orbitals, occupations, grid or an operand of the build; outputs are invalid");
}

void Plan::drop_graphs() {
  for (BuildGraph &g : graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    release(g.C);
    release(g.occ);
    release(g.V);
    release(g.J);
  }
  graphs.clear();
}

// A build replayed from a CUDA graph (graph mode, device buffers, phase 0).
// The second build of a kind (precision, spins, orbitals, outputs) records the
// device work of a build that reads the orbitals from, and writes V and J to,
// buffers of the graph's own; every build of that kind then copies the
// caller's orbitals in, launches the graph and copies the results out.  A
// build of another kind, or any change of the plan, drops the graphs first
// (their launch arguments and buffers are baked in).  If recording fails the
// kind keeps running ordinary builds.
static void fock_build_graph(Plan &P, int precision, int nspin, int nocc, const double *C, const double *occ,
                             int fuse_j, double *E, double *V, double *J, cudaStream_t user) {
  BuildGraph *g = nullptr;
  for (BuildGraph &x : P.graphs)
    if (x.precision == precision && x.nspin == nspin && x.nocc == nocc && x.fuse == fuse_j && x.hasV == (V != nullptr) &&
        x.hasJ == (J != nullptr))
      g = &x;
  if (!g || g->failed || !g->exec) {
    const bool record = g && !g->failed;
    if (!record) {
      // first build of this kind: an ordinary build (it may grow buffers the
      // recorded builds of other kinds use), then remember the kind
      P.drop_graphs();
      fock_build_once(P, precision, nspin, nocc, C, occ, NKX_MEM_DEVICE, fuse_j, E, V, J, user, 0, nullptr, false);
      BuildGraph n;
      n.precision = precision;
      n.nspin = nspin;
      n.nocc = nocc;
      n.fuse = fuse_j;
      n.hasV = V != nullptr;
      n.hasJ = J != nullptr;
      if (!g) P.graphs.push_back(n);
      return;
    }
    // second build of this kind: record it
    const size_t nn = (size_t)P.nbf * P.nbf;
    g->C = P.alloc<double>((size_t)nspin * nocc * P.nbf);
    g->occ = P.alloc<double>((size_t)nspin * nocc);
    g->V = V ? P.alloc<double>(nspin * nn) : nullptr;
    g->J = J ? P.alloc<double>(nn) : nullptr;
    cudaStream_t s = user ? user : P.stream;
    cudaGraph_t graph = nullptr;
    double e_unused = 0.0;
    NKX_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      fock_build_once(P, precision, nspin, nocc, g->C, g->occ, NKX_MEM_DEVICE, fuse_j, &e_unused, g->V, g->J, s, 0,
                      nullptr, true);
    } catch (...) {
      cudaStreamEndCapture(s, &graph);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      g->failed = true;
      fock_build_once(P, precision, nspin, nocc, C, occ, NKX_MEM_DEVICE, fuse_j, E, V, J, user, 0, nullptr, false);
      return;
    }
    NKX_CUDA(cudaStreamEndCapture(s, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      cudaGetLastError();
      g->exec = nullptr;
      g->failed = true;
      fock_build_once(P, precision, nspin, nocc, C, occ, NKX_MEM_DEVICE, fuse_j, E, V, J, user, 0, nullptr, false);
      return;
    }
    g->launches = P.launches;
  }
  // replay
  cudaStream_t s = user ? user : P.stream;
  const size_t nn = (size_t)P.nbf * P.nbf;
  cudaEvent_t t0, t1;
  NKX_CUDA(cudaEventCreate(&t0));
  NKX_CUDA(cudaEventCreate(&t1));
  NKX_CUDA(cudaEventRecord(t0, s));
  NKX_CUDA(cudaMemcpyAsync(g->C, C, sizeof(double) * nspin * nocc * P.nbf, cudaMemcpyDeviceToDevice, s));
  NKX_CUDA(cudaMemcpyAsync(g->occ, occ, sizeof(double) * nspin * nocc, cudaMemcpyDeviceToDevice, s));
  NKX_CUDA(cudaGraphLaunch(g->exec, s));
  if (V) NKX_CUDA(cudaMemcpyAsync(V, g->V, sizeof(double) * nspin * nn, cudaMemcpyDeviceToDevice, s));
  if (J) NKX_CUDA(cudaMemcpyAsync(J, g->J, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
  NKX_CUDA(cudaMemcpyAsync(E, P.d_E, sizeof(double), cudaMemcpyDeviceToHost, s));
  int status[2] = {0, 0};
  NKX_CUDA(cudaMemcpyAsync(status, P.d_status, sizeof(status), cudaMemcpyDeviceToHost, s));
  NKX_CUDA(cudaEventRecord(t1, s));
  NKX_CUDA(cudaStreamSynchronize(s));
  P.last = nkx_build_timing{};
  cudaEventElapsedTime(&P.last.total_ms, t0, t1);
  P.last.launches = g->launches;
  P.last_nspin = nspin;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  ++P.graph_replays;
  NKX_REQUIRE(status[0] == 0, NKX_ERR_TIMEOUT, "a tensor-core kernel wait gave up; outputs are invalid");
  NKX_REQUIRE(status[1] == 0 && std::isfinite(*E), NKX_ERR_NUMERIC,
              "non-finite value in the orbitals, occupations, grid or an operand of the build; outputs are invalid");
}

void fock_build(Plan &P, int precision, int nspin, int nocc, const double *C, const double *occ, int mem, int fuse_j,
                double *E, double *V, double *J, cudaStream_t user, int phase, double *y) {
  if (P.graph_mode && phase == 0 && mem == NKX_MEM_DEVICE) {
    NKX_REQUIRE(nspin == 1 || nspin == 2, NKX_ERR_ARG, "nspin must be 1 or 2");
    NKX_REQUIRE(nocc > 0 && C && occ && E && (V || J), NKX_ERR_ARG, "invalid arguments");
    fock_build_graph(P, precision, nspin, nocc, C, occ, fuse_j, E, V, J, user);
    return;
  }
  if (!P.graphs.empty()) P.drop_graphs();  // an ordinary build may grow buffers a graph uses
  fock_build_once(P, precision, nspin, nocc, C, occ, mem, fuse_j, E, V, J, user, phase, y, false);
}

}  // namespace nkx

using namespace nkx;

extern "C" {

NKX_API const char *nkx_last_error(void) { return g_last_error.c_str(); }

NKX_API nkx_status nkx_plan_create(const nkx_molecule *mol, const nkx_basis *prim, const nkx_basis *aux, long npoints,
                                   const double *xyz, const double *w, const int *owner, const nkx_plan_options *opts,
                                   nkx_plan **plan) {
  return run_guarded("nkx_plan_create", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan pointer is NULL");
    *plan = nullptr;
    auto P = std::make_unique<Plan>();
    build_plan(*P, mol, prim, aux, npoints, xyz, w, owner, opts);
    *plan = reinterpret_cast<nkx_plan *>(P.release());
  });
}

NKX_API nkx_status nkx_plan_get_info(const nkx_plan *plan, nkx_plan_info *info) {
  return run_guarded("nkx_plan_get_info", [&] {
    NKX_REQUIRE(plan && info, NKX_ERR_ARG, "invalid arguments");
    const Plan &P = *reinterpret_cast<const Plan *>(plan);
    info->npoints = P.npts;
    info->nbatches = P.nbatch;
    info->nbf = P.nbf;
    info->naux = P.naux;
    info->nblocks = P.nblk;
    info->npairs = P.npairs;
    info->nchunks = (int)P.chunks.size();
    info->metric_min_diag = P.metric_min_diag;
    info->graph_replays = P.graph_replays;
  });
}

NKX_API nkx_status nkx_fock_build(nkx_plan *plan, int precision, int nspin, int nocc, const double *C,
                                  const double *occ, int mem, int fuse_j, double *E, double *V, double *J,
                                  void *stream) {
  return run_guarded("nkx_fock_build", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    fock_build(P, precision, nspin, nocc, C, occ, mem, fuse_j, E, V, J, (cudaStream_t)stream);
  });
}

NKX_API nkx_status nkx_fock_build_phase1(nkx_plan *plan, int precision, int nspin, int nocc, const double *C,
                                         const double *occ, int mem, double *y, void *stream) {
  return run_guarded("nkx_fock_build_phase1", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    fock_build(P, precision, nspin, nocc, C, occ, mem, 0, nullptr, nullptr, nullptr, (cudaStream_t)stream, 1, y);
  });
}

NKX_API nkx_status nkx_fock_build_phase2(nkx_plan *plan, const double *y, int mem, int fuse_j, double *E, double *V,
                                         double *J, void *stream) {
  return run_guarded("nkx_fock_build_phase2", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    fock_build(P, 0, 0, 0, nullptr, nullptr, mem, fuse_j, E, V, J, (cudaStream_t)stream, 2, const_cast<double *>(y));
  });
}

NKX_API nkx_status nkx_plan_set_metric(nkx_plan *plan, const double *S, int mem) {
  return run_guarded("nkx_plan_set_metric", [&] {
    NKX_REQUIRE(plan && S, NKX_ERR_ARG, "invalid arguments");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    P.drop_graphs();
    NKX_REQUIRE(P.naux > 0, NKX_ERR_ARG, "the plan has no aux basis");
    NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
    const size_t NA = P.naux;
    P.h_metric.resize(NA * NA);
    NKX_CUDA(cudaMemcpy(P.h_metric.data(), S, sizeof(double) * NA * NA,
                        mem == NKX_MEM_HOST ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < NA; ++i)
      NKX_REQUIRE(std::isfinite(P.h_metric[i + i * NA]) && P.h_metric[i + i * NA] > 0, NKX_ERR_NUMERIC,
                  "metric diagonal must be positive and finite");
    // the mode chosen at plan creation (a caller's half inverse is replaced)
    P.svd_mode = P.metric_svd_thr > 0;
    if (P.svd_mode && !P.d_X) P.d_X = P.alloc<double>(NA * NA);
    factor_metric(P);
    NKX_CUDA(cudaStreamSynchronize(P.stream));
  });
}

NKX_API nkx_status nkx_get_last_timing(const nkx_plan *plan, nkx_build_timing *t) {
  return run_guarded("nkx_get_last_timing", [&] {
    NKX_REQUIRE(plan && t, NKX_ERR_ARG, "invalid arguments");
    *t = reinterpret_cast<const Plan *>(plan)->last;
  });
}

NKX_API nkx_status nkx_plan_last_density(const nkx_plan *plan, double *rho, long *perm) {
  return run_guarded("nkx_plan_last_density", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    const Plan &P = *reinterpret_cast<const Plan *>(plan);
    if (rho) {
      std::vector<double> h(2 * P.npad);
      NKX_CUDA(cudaMemcpy(h.data(), P.d_rho, sizeof(double) * 2 * P.npad, cudaMemcpyDeviceToHost));
      const int ns = std::max(1, P.last_nspin);
      for (long p = 0; p < P.npts; ++p)
        for (int s = 0; s < ns; ++s) rho[p * ns + s] = h[(size_t)s * P.npad + p];
    }
    if (perm)
      for (long p = 0; p < P.npts; ++p) perm[p] = P.perm[p];
  });
}

NKX_API nkx_status nkx_plan_batch_blocks(const nkx_plan *plan, int *counts) {
  return run_guarded("nkx_plan_batch_blocks", [&] {
    NKX_REQUIRE(plan && counts, NKX_ERR_ARG, "invalid arguments");
    const Plan &P = *reinterpret_cast<const Plan *>(plan);
    for (long b = 0; b < P.nbatch; ++b) counts[b] = P.h_pair_off[b + 1] - P.h_pair_off[b];
  });
}

NKX_API nkx_status nkx_plan_set_functional(nkx_plan *plan, int nfunc, const int *func_ids, double dens_threshold) {
  return run_guarded("nkx_plan_set_functional", [&] {
    NKX_REQUIRE(plan && func_ids, NKX_ERR_ARG, "invalid arguments");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    P.drop_graphs();
    nkx_plan_options o{};
    o.nfunc = nfunc;
    for (int i = 0; i < 4 && i < nfunc; ++i) o.func_ids[i] = func_ids[i];
    o.dens_threshold = dens_threshold;
    const XcSpec x = make_spec(&o);  // validates nfunc and the ids
    P.xc = x;
    P.gga = spec_is_gga(x);
  });
}

NKX_API nkx_status nkx_plan_set_half_inverse(nkx_plan *plan, int K, const double *X, int mem) {
  return run_guarded("nkx_plan_set_half_inverse", [&] {
    NKX_REQUIRE(plan && X, NKX_ERR_ARG, "invalid arguments");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    P.drop_graphs();
    NKX_REQUIRE(P.naux > 0, NKX_ERR_ARG, "the plan has no aux basis");
    NKX_REQUIRE(K >= 1 && K <= P.naux, NKX_ERR_ARG, "K must be in [1, naux]");
    NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
    const size_t NA = P.naux;
    if (!P.d_X) P.d_X = P.alloc<double>(NA * NA);
    if (!P.d_t) P.d_t = P.alloc<double>(NA);
    NKX_CUDA(cudaMemcpy(P.d_X, X, sizeof(double) * NA * K,
                        mem == NKX_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice));
    P.K = K;
    P.svd_mode = true;
  });
}

NKX_API nkx_status nkx_plan_set_wait_limit(nkx_plan *plan, unsigned long long ns, int stall) {
  return run_guarded("nkx_plan_set_wait_limit", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    P.drop_graphs();
    P.wait_ns = ns ? ns : 2000000000ull;
    P.stall_test = stall != 0;
  });
}

NKX_API nkx_status nkx_plan_set_graph(nkx_plan *plan, int enable) {
  return run_guarded("nkx_plan_set_graph", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    P.drop_graphs();
    P.graph_mode = enable != 0;
  });
}

NKX_API nkx_status nkx_plan_aux_metric(const nkx_plan *plan, double *S, int mem) {
  return run_guarded("nkx_plan_aux_metric", [&] {
    NKX_REQUIRE(plan && S, NKX_ERR_ARG, "invalid arguments");
    const Plan &P = *reinterpret_cast<const Plan *>(plan);
    NKX_REQUIRE(P.naux > 0, NKX_ERR_ARG, "the plan has no aux basis");
    NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
    const size_t bytes = sizeof(double) * P.naux * P.naux;
    if (mem == NKX_MEM_HOST)
      std::memcpy(S, P.h_metric.data(), bytes);
    else
      NKX_CUDA(cudaMemcpy(S, P.h_metric.data(), bytes, cudaMemcpyHostToDevice));
  });
}

NKX_API nkx_status nkx_plan_density(nkx_plan *plan, int nspin, int nocc, const double *C, const double *occ, int mem,
                                    int accumulate, double *rho, double *grad, double *sigma, void *stream) {
  return run_guarded("nkx_plan_density", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    NKX_REQUIRE(nspin == 1 || nspin == 2, NKX_ERR_ARG, "nspin must be 1 or 2");
    NKX_REQUIRE(nocc > 0 && C && occ && (rho || grad || sigma), NKX_ERR_ARG, "invalid arguments");
    NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
    cudaStream_t s = stream ? (cudaStream_t)stream : P.stream;
    const size_t n = (size_t)P.npts;
    if (!P.d_perm) {
      P.d_perm = P.alloc<long>(n);
      NKX_CUDA(cudaMemcpy(P.d_perm, P.perm.data(), sizeof(long) * n, cudaMemcpyHostToDevice));
    }
    NKX_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int) * 2, s));
    upload_orbitals(P, nspin, nocc, C, occ, mem, s);
    // the gradient needs the gradient collocation whatever the functional
    const bool gga = P.gga;
    P.gga = grad || sigma;
    StageTimer T;
    try {
      fp64_density_pass(P, nspin, nocc, s, T);
    } catch (...) {
      P.gga = gga;
      throw;
    }
    P.gga = gga;
    // outputs: the caller's device buffers, or device staging for host ones
    double *orho = rho, *ograd = grad, *osig = sigma;
    if (mem == NKX_MEM_HOST) {
      if (!P.d_dens_out) P.d_dens_out = P.alloc<double>(2 * 5 * n);
      orho = rho ? P.d_dens_out : nullptr;
      ograd = grad ? P.d_dens_out + 2 * n : nullptr;
      osig = sigma ? P.d_dens_out + 8 * n : nullptr;
      if (accumulate && rho)
        NKX_CUDA(cudaMemcpyAsync(orho, rho, sizeof(double) * nspin * n, cudaMemcpyHostToDevice, s));
      if (accumulate && grad)
        NKX_CUDA(cudaMemcpyAsync(ograd, grad, sizeof(double) * 3 * nspin * n, cudaMemcpyHostToDevice, s));
    }
    density_out_kernel<<<dim3(nblk((long)n, 256), nspin), 256, 0, s>>>((long)n, P.npad, P.d_perm, P.d_rho, P.d_grad,
                                                                        accumulate != 0, orho, ograd, osig);
    NKX_LAUNCH_CHECK();
    if (mem == NKX_MEM_HOST) {
      if (rho) NKX_CUDA(cudaMemcpyAsync(rho, orho, sizeof(double) * nspin * n, cudaMemcpyDeviceToHost, s));
      if (grad) NKX_CUDA(cudaMemcpyAsync(grad, ograd, sizeof(double) * 3 * nspin * n, cudaMemcpyDeviceToHost, s));
      if (sigma) NKX_CUDA(cudaMemcpyAsync(sigma, osig, sizeof(double) * nspin * n, cudaMemcpyDeviceToHost, s));
    }
    int status[2] = {0, 0};
    NKX_CUDA(cudaMemcpyAsync(status, P.d_status, sizeof(status), cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaStreamSynchronize(s));
    P.last_nspin = nspin;
    NKX_REQUIRE(status[1] == 0, NKX_ERR_NUMERIC, "non-finite value in the orbitals or occupations");
  });
}

NKX_API nkx_status nkx_plan_core_hamiltonian(nkx_plan *plan, const nkx_molecule *mol, double *S, double *T,
                                             double *V, int mem, void *stream) {
  return run_guarded("nkx_plan_core_hamiltonian", [&] {
    NKX_REQUIRE(plan && mol && mol->natoms > 0 && mol->xyz && mol->Z && S && T && V, NKX_ERR_ARG,
                "invalid arguments");
    NKX_REQUIRE(mem == NKX_MEM_DEVICE || mem == NKX_MEM_HOST, NKX_ERR_ARG, "mem must be NKX_MEM_DEVICE or NKX_MEM_HOST");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    cudaStream_t s = stream ? (cudaStream_t)stream : P.stream;
    const size_t tile = (size_t)kBatch * kBlockF, nn = (size_t)P.nbf_pad * P.nbf_pad;
    std::vector<double> zc(mol->natoms);
    for (int a = 0; a < mol->natoms; ++a) zc[a] = mol->Z[a];
    double *dc = P.alloc<double>(3 * (size_t)mol->natoms), *dz = P.alloc<double>(mol->natoms);
    NKX_CUDA(cudaMemcpyAsync(dc, mol->xyz, sizeof(double) * 3 * mol->natoms, cudaMemcpyHostToDevice, s));
    NKX_CUDA(cudaMemcpyAsync(dz, zc.data(), sizeof(double) * mol->natoms, cudaMemcpyHostToDevice, s));
    if (!P.ws_z) P.ws_z = P.alloc<double>(std::max<long>(1, P.max_chunk_pairs) * 3 * tile);
    NKX_CUDA(cudaFuncSetAttribute(vgemm_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kVSmemBytes));
    core_vne_kernel<<<nblk(P.npad, 256), 256, 0, s>>>(P.d_px, P.d_py, P.d_pz, P.d_w, P.npad, dc, dz, mol->natoms,
                                                     P.d_vj);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaMemsetAsync(P.d_V, 0, sizeof(double) * 3 * nn, s));
    // the collocation with gradients whatever the plan's functional
    const bool gga = P.gga;
    P.gga = true;
    try {
      for (const Chunk &c : P.chunks) {
        const long np = c.p1 - c.p0;
        if (np <= 0) continue;
        launch_colloc(P, c, s);
        // S (plane 0) and V_n (plane 1)
        core_z_kernel<<<(unsigned)np, 256, 0, s>>>(P.ws_phi, P.d_w, P.d_vj, P.d_pair_batch, c.p0, 0, P.ws_z);
        vgemm_fp64_kernel<<<dim3(P.nblk, P.nblk, 2), 256, kVSmemBytes, s>>>(
            P.ws_phi, P.ws_z, 4, 3, P.d_pair_off, P.d_mask, P.mask_words, c.b0, c.b1, c.p0, P.nbf_pad, P.d_V);
        // T (plane 2): the three gradient components into one output
        core_z_kernel<<<(unsigned)np, 256, 0, s>>>(P.ws_phi, P.d_w, P.d_vj, P.d_pair_batch, c.p0, 1, P.ws_z);
        for (int k = 0; k < 3; ++k)
          vgemm_fp64_kernel<<<dim3(P.nblk, P.nblk, 1), 256, kVSmemBytes, s>>>(
              P.ws_phi + (size_t)(k + 1) * tile, P.ws_z + (size_t)k * tile, 4, 3, P.d_pair_off, P.d_mask,
              P.mask_words, c.b0, c.b1, c.p0, P.nbf_pad, P.d_V + 2 * nn);
        NKX_LAUNCH_CHECK();
      }
    } catch (...) {
      P.gga = gga;
      throw;
    }
    P.gga = gga;
    const size_t nb = (size_t)P.nbf * P.nbf;
    double *out = nullptr;
    if (mem == NKX_MEM_HOST) {
      if (!P.d_out) P.d_out = P.alloc<double>(3 * nb);
      out = P.d_out;
    }
    double *dst[3] = {mem == NKX_MEM_HOST ? out : S, mem == NKX_MEM_HOST ? out + nb : V,
                      mem == NKX_MEM_HOST ? out + 2 * nb : T};
    dim3 tb(16, 16), gb(nblk(P.nbf, 16), nblk(P.nbf, 16));
    for (int z = 0; z < 3; ++z)
      symmetrize_unpad_kernel<<<gb, tb, 0, s>>>(P.nbf, P.nbf_pad, P.d_finv, P.d_V + z * nn, dst[z]);
    NKX_LAUNCH_CHECK();
    if (mem == NKX_MEM_HOST) {
      NKX_CUDA(cudaMemcpyAsync(S, dst[0], sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
      NKX_CUDA(cudaMemcpyAsync(V, dst[1], sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
      NKX_CUDA(cudaMemcpyAsync(T, dst[2], sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
    }
    NKX_CUDA(cudaStreamSynchronize(s));
    P.release(dc);
    P.release(dz);
  });
}

NKX_API nkx_status nkx_morton_order(long npoints, const double *xyz, long *perm) {
  return run_guarded("nkx_morton_order", [&] {
    NKX_REQUIRE(npoints > 0 && xyz && perm, NKX_ERR_ARG, "invalid arguments");
    std::vector<long> p;
    morton_order(npoints, xyz, p);
    std::copy(p.begin(), p.end(), perm);
  });
}

NKX_API nkx_status nkx_aux_metric(const nkx_basis *aux, long npoints, const double *d_xyz, const double *d_w,
                                  double *d_S, void *stream) {
  return run_guarded("nkx_aux_metric", [&] {
    NKX_REQUIRE(aux && aux->nbf > 0 && npoints > 0 && d_xyz && d_w && d_S, NKX_ERR_ARG, "invalid arguments");
    for (int i = 0; i < aux->nbf; ++i)
      NKX_REQUIRE(aux->l[i] >= 0 && aux->l[i] <= 7 && aux->n[i] > aux->l[i] && abs(aux->m[i]) <= aux->l[i] &&
                      aux->zeta[i] > 0,
                  NKX_ERR_UNSUPPORTED, "aux function outside n > l, |m| <= l <= 7, zeta > 0");
    cudaStream_t s = (cudaStream_t)stream;
    const auto atab = make_aux_table(*aux);
    const auto astab = make_sto_table(*aux);
    auto del = [](void *q) { cudaFree(q); };
    std::unique_ptr<void, decltype(del)> a1(dalloc<AuxFunc>(aux->nbf), del), a2(dalloc<StoFunc>(aux->nbf), del),
        a3(dalloc<double>(3 * (size_t)npoints), del);
    AuxFunc *d_aux = static_cast<AuxFunc *>(a1.get());
    StoFunc *d_asto = static_cast<StoFunc *>(a2.get());
    double *soa = static_cast<double *>(a3.get());
    NKX_CUDA(cudaMemcpy(d_aux, atab.data(), sizeof(AuxFunc) * aux->nbf, cudaMemcpyHostToDevice));
    NKX_CUDA(cudaMemcpy(d_asto, astab.data(), sizeof(StoFunc) * aux->nbf, cudaMemcpyHostToDevice));
    split_points_kernel<<<nblk(npoints, 256), 256, 0, s>>>(npoints, d_xyz, soa);
    NKX_LAUNCH_CHECK();
    cublasHandle_t hb;
    NKX_REQUIRE(cublasCreate(&hb) == CUBLAS_STATUS_SUCCESS, NKX_ERR_CUDA, "cublasCreate failed");
    std::unique_ptr<cublasContext, decltype(&cublasDestroy)> hguard(hb, &cublasDestroy);
    cublasSetStream(hb, s);
    grid_metric(d_asto, d_aux, aux->nbf, soa, soa + npoints, soa + 2 * npoints, d_w, npoints, hb, s, d_S);
  });
}

NKX_API nkx_status nkx_plan_destroy(nkx_plan *plan) {
  return run_guarded("nkx_plan_destroy", [&] { delete reinterpret_cast<Plan *>(plan); });
}

}  // extern "C"
