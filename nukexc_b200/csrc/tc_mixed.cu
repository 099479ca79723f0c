// Mixed-precision Fock build on the 5th-generation tensor cores (sm_100a).
//
// Both dense contractions of the Fock build run as one warp-specialised
// tcgen05 kernel (tc_gemm_kernel):
//   density  T_c(g, i) = sum_f PhiT_c(g, f) Ct(i, f)      c = value, d/dx, d/dy, d/dz
//   V        Vbar(mu, nu) += sum_g Phi(mu, g) Z(nu, g)    per (batch, block) pair
// Operands are stored pre-split as TF32 pairs x = hi + lo and each product is
// hi*hi + hi*lo + lo*hi (three kind::tf32 MMAs into one FP32 TMEM
// accumulator).  The V contraction flushes the FP32 accumulator after every
// 256-point batch into FP64 registers; the density accumulates the whole
// function range of a batch in FP32 and is contracted to rho and grad rho in
// FP64 (density.hpp:188-255, xc_integrals.hpp:424-726).
//
// Roles (320 threads): warp 0 lane 0 issues TMA tile loads into a 3-stage
// ring of 64 KB stages (A_hi, A_lo, B_hi, B_lo tiles of 128 x 32 FP32,
// 128-byte swizzle); warp 1 lane 0 issues the MMAs (M = N = 128, K = 8) and
// owns the TMEM allocation (2 x 128 columns, double-buffered accumulator);
// warps 2..9 are the epilogue (warp w reads TMEM lanes 32 (w % 4) .. + 31,
// columns 64 ((w - 2) / 4) .. + 63).  All waits are bounded (tc_ptx.cuh).
#include <cuda.h>

#include <algorithm>
#include <vector>

#include "plan.cuh"
#include "tc_ptx.cuh"

namespace nkx {

using namespace tc;

constexpr int kStages = 3;
constexpr int kTileBytes = 128 * 128;  // 128 rows x 128 B
constexpr int kStageBytes = 4 * kTileBytes;
constexpr int kGemmThreads = 320;
constexpr uint32_t kIdesc = idesc_tf32(128, 128);

enum { TC_MODE_V = 0, TC_MODE_DENSITY = 1 };

struct TcArgs {
  int mode;
  long b0, b1, p0;
  const int *pair_off, *pair_blk;
  const uint32_t *mask;
  int mask_words;
  // V mode
  int nblk, nz, nbf_pad;
  double *V;
  // density mode
  int nspin, ncomp, ntile_i, nocc_pad;
  float *T;
  long nunits;
  int *err;
};

// Iterates the accumulation groups and K steps of one work unit; the three
// roles run the same iteration so their barrier phases stay in step.
struct UnitIter {
  const TcArgs &a;
  long u;
  // decoded unit
  int I = 0, J = 0, zi = 0;               // V
  long bl = 0;                            // density: batch within chunk
  int h = 0, c = 0, s = 0, t = 0;         // density: point half, comp, spin, orbital tile
  __device__ UnitIter(const TcArgs &args, long unit) : a(args), u(unit) {
    if (a.mode == TC_MODE_V) {
      const long n2 = (long)a.nblk * a.nblk;
      zi = (int)(u / n2);
      I = (int)((u % n2) / a.nblk);
      J = (int)(u % a.nblk);
    } else {
      long r = u;
      t = (int)(r % a.ntile_i);
      r /= a.ntile_i;
      c = (int)(r % a.ncomp);
      r /= a.ncomp;
      h = (int)(r % 2);
      r /= 2;
      s = (int)(r % a.nspin);
      bl = r / a.nspin;
    }
  }
};

__device__ __forceinline__ int blk_pos(const uint32_t *m, int I) {
  int pos = 0;
  for (int w = 0; w < (I >> 5); ++w) pos += __popc(m[w]);
  return pos + __popc(m[I >> 5] & ((1u << (I & 31)) - 1u));
}
__device__ __forceinline__ bool blk_has(const uint32_t *m, int I) { return (m[I >> 5] >> (I & 31)) & 1u; }

// Calls fn(group_index_within_unit, nsteps, coords_fn) for each group.
// For the V mode a group is one batch with both blocks significant (8 K
// steps of 32 points); for the density mode the single group runs over all
// significant blocks of the batch (4 K steps of 32 functions per block).
template <class GroupFn>
__device__ __forceinline__ void for_each_group(const TcArgs &a, const UnitIter &it, GroupFn &&fn) {
  if (a.mode == TC_MODE_V) {
    for (long b = a.b0; b < a.b1; ++b) {
      const uint32_t *m = a.mask + b * a.mask_words;
      if (!blk_has(m, it.I) || !blk_has(m, it.J)) continue;
      const long qb = a.pair_off[b] - a.p0;
      const int ya = (int)((qb + blk_pos(m, it.I)) * 128);
      const int yb = (int)(((qb + blk_pos(m, it.J)) * a.nz + it.zi) * 128);
      fn(8, [=](int k, int &xa, int &yA, int &xb, int &yB) {
        xa = 32 * k;
        yA = ya;
        xb = 32 * k;
        yB = yb;
      });
    }
  } else {
    const long b = a.b0 + it.bl;
    const int q0 = a.pair_off[b], q1 = a.pair_off[b + 1];
    const int ncomp = a.ncomp;
    const long p0 = a.p0;
    const int *pb = a.pair_blk;
    const int rowB = it.s * a.nocc_pad + it.t * 128;
    const int c = it.c, h = it.h;
    fn(4 * (q1 - q0), [=](int k, int &xa, int &yA, int &xb, int &yB) {
      const int q = q0 + k / 4, sub = k % 4;
      xa = 32 * sub;
      yA = (int)((((long)(q - p0) * ncomp + c) * 256) + 128 * h);
      xb = pb[q] * 128 + 32 * sub;
      yB = rowB;
    });
  }
}

__global__ void __launch_bounds__(kGemmThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap mapA_hi, const __grid_constant__ CUtensorMap mapA_lo,
                   const __grid_constant__ CUtensorMap mapB_hi, const __grid_constant__ CUtensorMap mapB_lo,
                   TcArgs a) {
  extern __shared__ __align__(1024) uint8_t dsmem[];
  __shared__ uint64_t full_bar[kStages], empty_bar[kStages], tfull_bar[2], tempty_bar[2], drain_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_flag;
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dsmem) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull_bar[i], 1);
      mbar_init(&tempty_bar[i], 256);
    }
    mbar_init(&drain_bar, 1);
    fence_mbar_init();
    prefetch_tmap(&mapA_hi);
    prefetch_tmap(&mapA_lo);
    prefetch_tmap(&mapB_hi);
    prefetch_tmap(&mapB_lo);
  }
  if (warp == 1) {
    tmem_alloc(&tmem_base_sh, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp == 0) {
    // ------------------------------------------------------ TMA producer
    if (lane == 0) {
      uint32_t step = 0;
      for (long u = blockIdx.x; u < a.nunits && !abort_flag; u += gridDim.x) {
        UnitIter it(a, u);
        for_each_group(a, it, [&](int nsteps, auto coords) {
          for (int k = 0; k < nsteps && !abort_flag; ++k, ++step) {
            const int st = step % kStages;
            if (!mbar_wait(&empty_bar[st], ((step / kStages) & 1) ^ 1, a.err, 1, &abort_flag)) return;
            int xa, ya, xb, yb;
            coords(k, xa, ya, xb, yb);
            uint8_t *base = smem + st * kStageBytes;
            mbar_arrive_expect_tx(&full_bar[st], kStageBytes);
            tma_load_2d(base, &mapA_hi, xa, ya, &full_bar[st]);
            tma_load_2d(base + kTileBytes, &mapA_lo, xa, ya, &full_bar[st]);
            tma_load_2d(base + 2 * kTileBytes, &mapB_hi, xb, yb, &full_bar[st]);
            tma_load_2d(base + 3 * kTileBytes, &mapB_lo, xb, yb, &full_bar[st]);
          }
        });
      }
      // drain: every issued stage has been consumed (or, after an abort,
      // its copy has landed) before the CTA may exit
      volatile int keep_waiting = 0;
      for (uint32_t k = (step > kStages ? step - kStages : 0); k < step; ++k)
        mbar_wait(&full_bar[k % kStages], (k / kStages) & 1, a.err, 2, &keep_waiting);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t step = 0, grp = 0;
      for (long u = blockIdx.x; u < a.nunits && !abort_flag; u += gridDim.x) {
        UnitIter it(a, u);
        for_each_group(a, it, [&](int nsteps, auto) {
          if (abort_flag) return;
          const uint32_t buf = grp & 1, use = grp >> 1;
          if (!mbar_wait(&tempty_bar[buf], (use & 1) ^ 1, a.err, 3, &abort_flag)) return;
          tc_fence_after();
          const uint32_t d = tmem + buf * 128;
          for (int k = 0; k < nsteps; ++k, ++step) {
            const int st = step % kStages;
            if (!mbar_wait(&full_bar[st], (step / kStages) & 1, a.err, 4, &abort_flag)) return;
            tc_fence_after();
            const uint32_t base = smem_u32(smem + st * kStageBytes);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const uint64_t ah = smem_desc_k128(base + kk * 32);
              const uint64_t al = smem_desc_k128(base + kTileBytes + kk * 32);
              const uint64_t bh = smem_desc_k128(base + 2 * kTileBytes + kk * 32);
              const uint64_t bo = smem_desc_k128(base + 3 * kTileBytes + kk * 32);
              mma_tf32(d, ah, bh, kIdesc, (k > 0 || kk > 0) ? 1u : 0u);
              mma_tf32(d, ah, bo, kIdesc, 1u);
              mma_tf32(d, al, bh, kIdesc, 1u);
            }
            mma_commit(&empty_bar[st]);
          }
          mma_commit(&tfull_bar[buf]);
          ++grp;
        });
      }
      // all MMAs done before TMEM is released
      volatile int keep_waiting = 0;
      mma_commit(&drain_bar);
      mbar_wait(&drain_bar, 0, a.err, 5, &keep_waiting);
    }
  } else {
    // ------------------------------------------------------ epilogue
    const int q = warp & 3, half = (warp - 2) >> 2;
    const int row = 32 * q + lane;
    const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
    uint32_t grp = 0;
    for (long u = blockIdx.x; u < a.nunits && !abort_flag; u += gridDim.x) {
      UnitIter it(a, u);
      double acc[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) acc[j] = 0.0;
      bool any = false;
      for_each_group(a, it, [&](int nsteps, auto) {
        if (abort_flag) return;
        const uint32_t buf = grp & 1, use = grp >> 1;
        if (!mbar_wait(&tfull_bar[buf], use & 1, a.err, 6, &abort_flag)) return;
        tc_fence_after();
        any = true;
        __syncwarp();
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          float v[32];
          tmem_ld32(tmem + lane_addr + buf * 128 + 64 * half + 32 * part, v);
          if (a.mode == TC_MODE_V) {
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[32 * part + j] += (double)v[j];
          } else {
            // T[bl][s][c][i][g]: lanes write consecutive g
            const long plane = ((it.bl * a.nspin + it.s) * a.ncomp + it.c);
            float *Tp = a.T + plane * (long)a.nocc_pad * 256 + 128 * it.h + row;
            const int i0 = it.t * 128 + 64 * half + 32 * part;
#pragma unroll
            for (int j = 0; j < 32; ++j) Tp[(long)(i0 + j) * 256] = nsteps > 0 ? v[j] : 0.0f;
          }
        }
        tc_fence_before();
        mbar_arrive(&tempty_bar[buf]);
        ++grp;
      });
      if (a.mode == TC_MODE_V && any) {
        double *Vz = a.V + (size_t)it.zi * a.nbf_pad * a.nbf_pad;
        const size_t r = (size_t)it.I * 128 + row;
#pragma unroll
        for (int j = 0; j < 64; ++j) {
          const size_t col = (size_t)it.J * 128 + 64 * half + j;
          Vz[r + col * a.nbf_pad] += acc[j];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}


// ------------------------------------------------------ data kernels ----

// Collocation of one (batch, block) pair per CTA as TF32 pairs:
// out_hi/out_lo[pair][comp][g][f] (layout of colloc_fp64_kernel).
template <bool GRAD>
__global__ void __launch_bounds__(256) colloc_split_kernel(const StoFunc *__restrict__ sto, const double *__restrict__ px,
                                                           const double *__restrict__ py, const double *__restrict__ pz,
                                                           const int *__restrict__ pair_batch,
                                                           const int *__restrict__ pair_blk, long p0,
                                                           float *__restrict__ out_hi, float *__restrict__ out_lo) {
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
  for (int c = 0; c < 4; ++c) f[c] = sto[I * kBlockF + lane + 32 * c];
  const size_t tile = (size_t)kBatch * kBlockF;
  const size_t off = (size_t)blockIdx.x * (GRAD ? 4 : 1) * tile;
  float *oh = out_hi + off, *ol = out_lo + off;
  for (int g = warp; g < kBatch; g += 8) {
    const double x = sx[g], y = sy[g], z = sz[g];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const size_t idx = (size_t)g * kBlockF + lane + 32 * c;
      double v[4];
      if (GRAD)
        sto_value_grad(f[c], x, y, z, v[0], v[1], v[2], v[3]);
      else
        v[0] = sto_value(f[c], x, y, z);
#pragma unroll
      for (int k = 0; k < (GRAD ? 4 : 1); ++k) {
        float hi, lo;
        split_tf32(v[k], hi, lo);
        oh[k * tile + idx] = hi;
        ol[k * tile + idx] = lo;
      }
    }
  }
}

// Orbitals Ct[spin][i][f] (FP64, f padded) -> TF32 pairs with orbital rows
// padded to nocc_pad (zeros).
__global__ void split_orbitals_kernel(const double *__restrict__ Ct, int nocc, int nocc_pad, int nspin, int nbf_pad,
                                      float *__restrict__ hi, float *__restrict__ lo) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long tot = (long)nspin * nocc_pad * nbf_pad;
  if (e >= tot) return;
  const int f = (int)(e % nbf_pad);
  const long si = e / nbf_pad;
  const int s = (int)(si / nocc_pad), i = (int)(si % nocc_pad);
  const double v = i < nocc ? Ct[((size_t)s * nocc + i) * nbf_pad + f] : 0.0;
  float h, l;
  split_tf32(v, h, l);
  hi[e] = h;
  lo[e] = l;
}

// rho(g) = sum_i occ_i T0(g,i)^2, grad rho = 2 sum_i occ_i T0 Tc in FP64 from
// the FP32 tensor-core products T[bl][s][c][i][g] (density.hpp:188-255).
template <bool GRAD>
__global__ void density_contract_kernel(const float *__restrict__ T, const double *__restrict__ occ, int nocc,
                                        int nocc_pad, int nspin, long b0, double *__restrict__ rho,
                                        double *__restrict__ grad, long npad) {
  constexpr int NC = GRAD ? 4 : 1;
  const long bl = blockIdx.x;
  const int s = blockIdx.y, g = threadIdx.x;
  const float *Tp = T + ((bl * nspin + s) * NC) * (size_t)nocc_pad * 256 + g;
  const size_t plane = (size_t)nocc_pad * 256;
  double r = 0, gx = 0, gy = 0, gz = 0;
  for (int i = 0; i < nocc; ++i) {
    const double o = occ[(size_t)s * nocc + i];
    const double t = Tp[(size_t)i * 256];
    r += o * t * t;
    if (GRAD) {
      gx += o * t * (double)Tp[plane + (size_t)i * 256];
      gy += o * t * (double)Tp[2 * plane + (size_t)i * 256];
      gz += o * t * (double)Tp[3 * plane + (size_t)i * 256];
    }
  }
  const long gg = (b0 + bl) * kBatch + g;
  rho[(size_t)s * npad + gg] = r;
  if (GRAD) {
    grad[((size_t)s * 3 + 0) * npad + gg] = 2 * gx;
    grad[((size_t)s * 3 + 1) * npad + gg] = 2 * gy;
    grad[((size_t)s * 3 + 2) * npad + gg] = 2 * gz;
  }
}

// Z build for the tensor-core V contraction: from PhiT (TF32 pairs,
// [pair][comp][g][f]) and the per-point coefficients, write Phi[pair][f][g]
// and Z[pair][z][f][g] as TF32 pairs (transposed through shared memory in
// slabs of 32 points).  z < nspin: Z_s = c0 phi + c . grad phi; z == nspin
// (separate J): Z_J = 1/2 vJ phi.
template <bool GRAD>
__global__ void __launch_bounds__(256) zbuild_split_kernel(const float *__restrict__ ph_hi, const float *__restrict__ ph_lo,
                                                           const double *__restrict__ coef, const double *__restrict__ vj,
                                                           const int *__restrict__ pair_batch, long p0, int nz, int nspin,
                                                           long npad, float *__restrict__ phi_hi, float *__restrict__ phi_lo,
                                                           float *__restrict__ z_hi, float *__restrict__ z_lo) {
  constexpr int NC = GRAD ? 4 : 1;
  __shared__ float tile[128][33];
  const long q = blockIdx.x;
  const int b = pair_batch[p0 + q];
  const size_t T = (size_t)kBatch * kBlockF;
  const float *H = ph_hi + q * NC * T, *L = ph_lo + q * NC * T;
  const int f = threadIdx.x & 127, gsub = threadIdx.x >> 7;  // 2 point rows per pass
  for (int g0 = 0; g0 < kBatch; g0 += 32) {
    double val[16], zv[3][16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int g = g0 + gsub + 2 * k;
      const size_t e = (size_t)g * kBlockF + f;
      const double v = (double)H[e] + (double)L[e];
      double dx = 0, dy = 0, dz = 0;
      if (GRAD) {
        dx = (double)H[T + e] + (double)L[T + e];
        dy = (double)H[2 * T + e] + (double)L[2 * T + e];
        dz = (double)H[3 * T + e] + (double)L[3 * T + e];
      }
      val[k] = v;
      const long gg = (long)b * kBatch + g;
      for (int z = 0; z < 3; ++z) {
        double r = 0.0;
        if (z < nspin) {
          const double *c = coef + (size_t)z * 4 * npad;
          r = c[gg] * v;
          if (GRAD) r += c[npad + gg] * dx + c[2 * npad + gg] * dy + c[3 * npad + gg] * dz;
        } else if (z < nz) {
          r = 0.5 * vj[gg] * v;
        }
        zv[z][k] = r;
      }
    }
    // planes: phi hi, phi lo, then (z hi, z lo) for z < nz
    for (int pl = 0; pl < 2 + 2 * nz; ++pl) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const double x = pl < 2 ? val[k] : zv[(pl - 2) / 2][k];
        float hi, lo;
        split_tf32(x, hi, lo);
        tile[f][gsub + 2 * k] = (pl & 1) ? lo : hi;
      }
      __syncthreads();
      float *dst;
      if (pl < 2)
        dst = (pl == 0 ? phi_hi : phi_lo) + q * T;
      else
        dst = ((pl & 1) ? z_lo : z_hi) + (q * nz + (pl - 2) / 2) * T;
      // 128 rows (f) x 32 points; each thread writes 16 consecutive points
      const int rf = threadIdx.x >> 1, part = threadIdx.x & 1;
#pragma unroll
      for (int k = 0; k < 16; ++k) dst[(size_t)rf * kBatch + g0 + 16 * part + k] = tile[rf][16 * part + k];
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------- host ----

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    NKX_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    NKX_REQUIRE(p && q == cudaDriverEntryPointSuccess, NKX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D FP32 tensor map over a row-major [rows][cols] array, box 32 x 128,
// 128-byte swizzle.  cols * 4 must be a multiple of 16 and >= 32 elements.
static CUtensorMap make_map(const float *base, long rows, long cols) {
  NKX_REQUIRE(cols % 32 == 0 && rows >= 128 && ((uintptr_t)base % 16) == 0, NKX_ERR_ARG, "bad tensor map shape");
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(float)};
  const cuuint32_t box[2] = {32, 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  NKX_REQUIRE(r == CUDA_SUCCESS, NKX_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

struct MixedState {
  long cap_pairs = 0;
  int nocc_pad = 0, nspin = 0, nbatch_chunk = 0;
  float *phT_hi = nullptr, *phT_lo = nullptr;  // [pair][4][256][128]
  float *ph_hi = nullptr, *ph_lo = nullptr;    // [pair][128][256]
  float *z_hi = nullptr, *z_lo = nullptr;      // [pair][3][128][256]
  float *ct_hi = nullptr, *ct_lo = nullptr;    // [2][nocc_pad][nbf_pad]
  float *T = nullptr;                          // [batch][spin][4][nocc_pad][256]
  int *err = nullptr;
  CUtensorMap m_phT_hi, m_phT_lo, m_ph_hi, m_ph_lo, m_z_hi, m_z_lo, m_ct_hi, m_ct_lo;
  std::vector<void *> bufs;
  int nsm = 148;
  ~MixedState() {
    for (void *p : bufs) cudaFree(p);
  }
  template <class T>
  T *alloc(size_t n) {
    T *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      throw Error{NKX_ERR_ALLOC, "mixed workspace allocation of " + std::to_string(n * sizeof(T)) + " bytes failed"};
    }
    bufs.push_back(p);
    return p;
  }
};

bool mixed_available(const Plan &) {
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  return major == 10 && minor == 0;
}

static MixedState &mixed_state(Plan &P, int nspin, int nocc) {
  if (!P.mx_state) P.mx_state = new MixedState();
  MixedState &M = *static_cast<MixedState *>(P.mx_state);
  const size_t T = (size_t)kBatch * kBlockF;
  if (!M.phT_hi) {
    M.cap_pairs = std::max<long>(1, P.max_chunk_pairs);
    long nb = 1;
    for (const Chunk &c : P.chunks) nb = std::max(nb, c.b1 - c.b0);
    M.nbatch_chunk = (int)nb;
    M.phT_hi = M.alloc<float>(M.cap_pairs * 4 * T);
    M.phT_lo = M.alloc<float>(M.cap_pairs * 4 * T);
    M.ph_hi = M.alloc<float>(M.cap_pairs * T);
    M.ph_lo = M.alloc<float>(M.cap_pairs * T);
    M.z_hi = M.alloc<float>(M.cap_pairs * 3 * T);
    M.z_lo = M.alloc<float>(M.cap_pairs * 3 * T);
    M.err = M.alloc<int>(1);
    NKX_CUDA(cudaMemset(M.err, 0, sizeof(int)));
    M.m_phT_hi = make_map(M.phT_hi, M.cap_pairs * 4 * 256, 128);
    M.m_phT_lo = make_map(M.phT_lo, M.cap_pairs * 4 * 256, 128);
    M.m_ph_hi = make_map(M.ph_hi, M.cap_pairs * 128, 256);
    M.m_ph_lo = make_map(M.ph_lo, M.cap_pairs * 128, 256);
    M.m_z_hi = make_map(M.z_hi, M.cap_pairs * 3 * 128, 256);
    M.m_z_lo = make_map(M.z_lo, M.cap_pairs * 3 * 128, 256);
    int dev = 0;
    NKX_CUDA(cudaGetDevice(&dev));
    NKX_CUDA(cudaDeviceGetAttribute(&M.nsm, cudaDevAttrMultiProcessorCount, dev));
    NKX_CUDA(cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kStages * kStageBytes + 1024));
  }
  const int nocc_pad = ((nocc + 127) / 128) * 128;
  if (nocc_pad > M.nocc_pad || nspin > M.nspin) {
    M.nocc_pad = std::max(nocc_pad, M.nocc_pad);
    M.nspin = std::max(nspin, M.nspin);
    M.ct_hi = M.alloc<float>((size_t)2 * M.nocc_pad * P.nbf_pad);
    M.ct_lo = M.alloc<float>((size_t)2 * M.nocc_pad * P.nbf_pad);
    M.m_ct_hi = make_map(M.ct_hi, (long)2 * M.nocc_pad, P.nbf_pad);
    M.m_ct_lo = make_map(M.ct_lo, (long)2 * M.nocc_pad, P.nbf_pad);
    M.T = M.alloc<float>((size_t)M.nbatch_chunk * 2 * 4 * M.nocc_pad * 256);
  }
  return M;
}

static void launch_gemm(MixedState &M, const CUtensorMap &ah, const CUtensorMap &al, const CUtensorMap &bh,
                        const CUtensorMap &bl, const TcArgs &a, cudaStream_t s) {
  if (a.nunits <= 0) return;
  const unsigned grid = (unsigned)std::min<long>(a.nunits, M.nsm);
  tc_gemm_kernel<<<grid, kGemmThreads, kStages * kStageBytes + 1024, s>>>(ah, al, bh, bl, a);
  NKX_LAUNCH_CHECK();
}

__global__ void functional_kernel(XcSpec s, bool gga, int nspin, long npad, const double *__restrict__ w,
                                  const double *__restrict__ rho, const double *__restrict__ grad,
                                  const double *__restrict__ vj, double *__restrict__ coef, double *Eacc);
void coulomb_fit(Plan &P, int nspin, cudaStream_t s);

void fock_build_mixed(Plan &P, int nspin, int nocc, bool needJ, bool fuse, bool separateJ, cudaStream_t s,
                      StageTimer &Tm) {
  MixedState &M = mixed_state(P, nspin, nocc);
  const int ncomp = P.gga ? 4 : 1;
  const int nzs = nspin + (separateJ ? 1 : 0);
  NKX_REQUIRE(nzs <= 3, NKX_ERR_ARG, "too many Z planes");
  const bool multi = P.chunks.size() > 1;
  NKX_CUDA(cudaMemsetAsync(M.err, 0, sizeof(int), s));
  {
    const long tot = (long)nspin * M.nocc_pad * P.nbf_pad;
    split_orbitals_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(P.d_Ct, nocc, M.nocc_pad, nspin, P.nbf_pad,
                                                                          M.ct_hi, M.ct_lo);
    NKX_LAUNCH_CHECK();
    ++P.launches;
  }
  auto colloc = [&](const Chunk &c) {
    const long np = c.p1 - c.p0;
    if (np <= 0) return;
    Tm.begin(ST_COLLOC, s);
    if (P.gga)
      colloc_split_kernel<true><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_px, P.d_py, P.d_pz, P.d_pair_batch,
                                                             P.d_pair_blk, c.p0, M.phT_hi, M.phT_lo);
    else
      colloc_split_kernel<false><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_px, P.d_py, P.d_pz, P.d_pair_batch,
                                                              P.d_pair_blk, c.p0, M.phT_hi, M.phT_lo);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    Tm.end(s);
  };
  // ---- pass A: collocation, density GEMM, contraction
  for (const Chunk &c : P.chunks) {
    colloc(c);
    const long nb = c.b1 - c.b0;
    Tm.begin(ST_DENSITY, s);
    TcArgs a{};
    a.mode = TC_MODE_DENSITY;
    a.b0 = c.b0;
    a.b1 = c.b1;
    a.p0 = c.p0;
    a.pair_off = P.d_pair_off;
    a.pair_blk = P.d_pair_blk;
    a.mask = P.d_mask;
    a.mask_words = P.mask_words;
    a.nspin = nspin;
    a.ncomp = ncomp;
    a.ntile_i = M.nocc_pad / 128;
    a.nocc_pad = M.nocc_pad;
    a.T = M.T;
    a.err = M.err;
    a.nunits = nb * nspin * 2 * ncomp * a.ntile_i;
    launch_gemm(M, M.m_phT_hi, M.m_phT_lo, M.m_ct_hi, M.m_ct_lo, a, s);
    ++P.launches;
    if (P.gga)
      density_contract_kernel<true><<<dim3((unsigned)nb, nspin), 256, 0, s>>>(M.T, P.d_occ, nocc, M.nocc_pad, nspin,
                                                                              c.b0, P.d_rho, P.d_grad, P.npad);
    else
      density_contract_kernel<false><<<dim3((unsigned)nb, nspin), 256, 0, s>>>(M.T, P.d_occ, nocc, M.nocc_pad, nspin,
                                                                               c.b0, P.d_rho, P.d_grad, P.npad);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    Tm.end(s);
  }
  // ---- J fit and the functional, in FP64
  if (needJ) {
    Tm.begin(ST_COULOMB, s);
    coulomb_fit(P, nspin, s);
    Tm.end(s);
  }
  Tm.begin(ST_FUNC, s);
  NKX_CUDA(cudaMemsetAsync(P.d_E, 0, sizeof(double), s));
  functional_kernel<<<(unsigned)((P.npad + 255) / 256), 256, 0, s>>>(P.xc, P.gga, nspin, P.npad, P.d_w, P.d_rho,
                                                                      P.d_grad, (needJ && fuse) ? P.d_vj : nullptr,
                                                                      P.d_coef, P.d_E);
  NKX_LAUNCH_CHECK();
  ++P.launches;
  Tm.end(s);
  // ---- pass B: Z and the V contraction
  NKX_CUDA(cudaMemsetAsync(P.d_V, 0, sizeof(double) * nzs * P.nbf_pad * P.nbf_pad, s));
  for (const Chunk &c : P.chunks) {
    const long np = c.p1 - c.p0;
    if (np <= 0) continue;
    if (multi) colloc(c);
    Tm.begin(ST_ZBUILD, s);
    if (P.gga)
      zbuild_split_kernel<true><<<(unsigned)np, 256, 0, s>>>(M.phT_hi, M.phT_lo, P.d_coef, P.d_vj, P.d_pair_batch,
                                                             c.p0, nzs, nspin, P.npad, M.ph_hi, M.ph_lo, M.z_hi,
                                                             M.z_lo);
    else
      zbuild_split_kernel<false><<<(unsigned)np, 256, 0, s>>>(M.phT_hi, M.phT_lo, P.d_coef, P.d_vj, P.d_pair_batch,
                                                              c.p0, nzs, nspin, P.npad, M.ph_hi, M.ph_lo, M.z_hi,
                                                              M.z_lo);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    Tm.end(s);
    Tm.begin(ST_VGEMM, s);
    TcArgs a{};
    a.mode = TC_MODE_V;
    a.b0 = c.b0;
    a.b1 = c.b1;
    a.p0 = c.p0;
    a.pair_off = P.d_pair_off;
    a.pair_blk = P.d_pair_blk;
    a.mask = P.d_mask;
    a.mask_words = P.mask_words;
    a.nblk = P.nblk;
    a.nz = nzs;
    a.nbf_pad = P.nbf_pad;
    a.V = P.d_V;
    a.err = M.err;
    a.nunits = (long)P.nblk * P.nblk * nzs;
    launch_gemm(M, M.m_ph_hi, M.m_ph_lo, M.m_z_hi, M.m_z_lo, a, s);
    ++P.launches;
    Tm.end(s);
  }
  int herr = 0;
  NKX_CUDA(cudaMemcpyAsync(&herr, M.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  NKX_CUDA(cudaStreamSynchronize(s));
  NKX_REQUIRE(herr == 0, NKX_ERR_TIMEOUT, "tensor-core kernel wait timed out (code " + std::to_string(herr) + ")");
}

void destroy_mixed_state(void *p) { delete static_cast<MixedState *>(p); }

}  // namespace nkx
