// Mixed-precision Fock build on the 5th-generation tensor cores (sm_100a):
// error-free int8 digit contractions with exact int32 accumulation.
//
// The dense contractions of the Fock build,
//   density  T_c(g, i) = sum_f PhiT_c(g, f) Ct(i, f)      c = value, d/dx, d/dy, d/dz
//   V        Vbar(mu, nu) += sum_g Phi(mu, g) Z(nu, g)    per (batch, block) pair
// (density.hpp:188-255, xc_integrals.hpp:424-726) and, for GGA from 256
// orbitals on, Y(g, mu) = sum_i T_0(g, i) C(mu, i) occ_i in place of the three
// gradient components of T (grad rho = 2 sum_mu grad phi_mu Y_mu), run on one
// warp-specialised tcgen05 kernel of kind::i8.  Every operand row r of a
// tile is scaled by a power of two s_r >= max|row| and rounded to a 31-bit
// integer written as four balanced base-256 digits (digits_word, tc_ptx.cuh).
// A contraction over K is then
//   sum_k a_k b_k = s_a s_b 2^-60 sum_{L=0..3} 2^(8(6-L)) Acc_L,
//   Acc_L = sum_k sum_{i+j=L} d_i(a_k) d_j(b_k)            (int32, exact)
// i.e. ten int8 MMAs per K step into four int32 TMEM accumulators, combined
// in FP64 after every accumulation group (one 256-point batch for V, one
// 128-function block for the density).  Products with i + j >= 4 (at most
// 2^-30 s_a s_b each) are dropped; everything kept is exact, so unlike FP32
// tensor-core accumulation the result carries no rounding bias.
//
// Roles: warp 0 lane 0 issues 3-D TMA loads of the four digit planes of A
// (128 rows) and B (N rows), 64 K-bytes per stage, into a ring of stages
// (64-byte swizzle); warp 1 lane 0 issues the MMAs (M = 128, N, K = 32) and
// owns TMEM (all 512 columns: NBUF buffers x 4 levels x N); warps 2.. are
// the epilogue (warp w reads TMEM lanes 32 (w % 4) .. + 31, columns
// 32 ((w - 2) / 4) .. + 31 of each level, in slices) with FP64 accumulators
// in registers.  The V contraction uses N = 128 (576 threads, one TMEM
// buffer): M = 128 x N = 64 int8 MMAs are limited by shared-memory operand
// bandwidth to about two thirds of the tensor rate.  The density
// contractions (T0 and the Y pass) run N = 64 (320 threads, two TMEM
// buffers; their groups are short, so overlapping the epilogue matters) or,
// from 1024 orbitals on, N = 128.  All waits are bounded (tc_ptx.cuh).
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "plan.cuh"
#include "tc_ptx.cuh"

namespace nkx {

using namespace tc;

constexpr int kABytes = 4 * 128 * 64;  // four digit planes, 128 rows x 64 B
constexpr double kTwoM36 = 0x1p-36;

// TC_MODE_GRAD: Y(g, mu) = sum_i T0(g, i) (C occ)(mu, i) over the orbitals
// (grad rho = 2 sum_mu grad phi_mu Y_mu, summed in the Y pass's epilogue)
// TC_MODE_X (mixed XC gradient): X_c(g, mu) = sum_i T_c(g, i) (C occ)(mu, i)
// for the value and the three gradient components, written in FP64
enum { TC_MODE_V = 0, TC_MODE_DENSITY = 1, TC_MODE_GRAD = 2, TC_MODE_X = 3 };

// Shape by the MMA width N.  N = 128: one TMEM buffer of 4 levels x 128
// columns, 16 epilogue warps, 3 stages of 64 KB.  N = 64: two buffers of
// 4 levels x 64 columns, so the epilogue of one group overlaps the MMAs of
// the next, 8 epilogue warps, 4 stages of 48 KB.  Any contraction can run
// either shape (the V unit then covers a 128 x N part of its output tile,
// the density unit an N-orbital tile, the Y-pass unit N functions).  The
// plan's tuning (nkx_plan_autotune) picks the shape per contraction; the
// defaults are N = 128 for V and, for T0 and the Y pass, N = 64 below 1024
// orbitals and N = 128 from there on.
//
// EW epilogue warps (default N / 8): warp w reads TMEM lanes 32 (w % 4) ..,
// and CW = 4 N / EW columns of each level.  The V contraction can also run
// N = 128 with 8 epilogue warps of 64 columns each (320 threads, 200
// registers a thread: the FP64 accumulators of 64 columns fit without
// spilling), chosen by the tuning.
template <int N_, int EW_ = N_ / 8>
struct TcShape {
  static constexpr int N = N_;
  static constexpr int EW = EW_;
  static constexpr int CW = 4 * N / EW;  // columns of an epilogue warp
  static constexpr int NBUF = N == 128 ? 1 : 2;
  static constexpr int kStages = N == 128 ? 3 : 4;
  static constexpr int kBBytes = 4 * N * 64;
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kEpiThreads = 32 * EW;
  static constexpr int kThreads = 64 + kEpiThreads;
  static constexpr uint32_t kIdesc = idesc_i8(128, N);
  static constexpr int kSmem = kStages * kStageBytes + 1024;
};

struct TcArgs {
  int mode;
  long b0, b1, p0;
  const int *pair_off, *pair_blk;
  const uint32_t *mask;
  int mask_words, nblk;
  // V mode; nsplit > 1 splits each output tile's batches over that many
  // units (interleaved), which then add their tiles atomically
  int nz, nbf_pad, nsplit;
  const double *sA, *sB;  // row scales: V: sph[q][128], sz[q*nz+z][128]
  double *V;
  // density mode: sA = sphT[q][ncs][256], sB = sct[s][i][blk]; ncomp
  // components are contracted, ncs are stored per pair in qphT / sphT
  int nspin, ncomp, ncs, ntile_i, nocc_pad;
  double *T;
  // grad mode: sA = st0[(bl, s, h)][128] (T0 row scales), sB = sco[s][mu]
  // (C occ row scales); grad phi from the pass-A digits qphT[pair][comp][digit][g][f]
  // and scales sphT[pair][comp][g] (ncs components); output the partial sums
  // Gp[pair][spin][t][cq][c][256] of 2 grad phi_c . Y over 32 functions
  const int *pair_batch;
  const uint8_t *qphT;
  const double *sphT;
  double *Gp;
  // X mode (same operands as grad mode, ncomp components of T): output
  // X[pair][spin][comp][g][mu] in FP64
  double *X;
  long nunits;
  // err[0]: code of the first wait that gave up (0: none); waits that can
  // be abandoned give up after wait_ns, the drain waits after kDrainLimitNs
  int *err;
  unsigned long long wait_ns;
  // stall != 0 (tests of the error path): the MMA issuer first waits on a
  // barrier that nothing completes, so the kernel gives up after wait_ns
  int stall;
  int nt;  // MMA width N of the launched kernel (V: 128 / nt units per output tile)
  int ew;  // epilogue warps of the launched kernel (N = 128 V: 16 or 8)
  const int *vtiles;  // V: the chunk's output tiles (I << 16 | J), ntiles of them
  long ntiles;
};

// S = 2^24 L0 + 2^16 L1 + 2^8 L2 + L3 of four int32 accumulator levels,
// exact: the integer sum (|S| < 2^49) is formed in int64 and converted by
// adding the bit pattern of 1.5 2^52 (the sum is then the FP64 number
// 1.5 2^52 + S, exact below 2^51) and subtracting 1.5 2^52 in FP64.  Measured
// on B200: 16.7 values per clock and SM against 11.8 for an int64 -> FP64
// conversion instruction and 14.8 for four int32 conversions and FMAs.
__device__ __forceinline__ double level_sum(uint32_t l0, uint32_t l1, uint32_t l2, uint32_t l3) {
  const long long S = (long long)(int)l0 * (1LL << 24) + (long long)(int)l1 * (1LL << 16) +
                      (long long)(int)l2 * (1LL << 8) + (long long)(int)l3;
  return __longlong_as_double(S + 0x4338000000000000LL) - 0x1.8p52;
}

struct UnitIter {
  int I = 0, J = 0, zi = 0, sp = 0, hc = 0;  // V: row block, column block, Z plane, batch split, column part
  long bl = 0;                     // density: batch within chunk
  long q = 0;                      // grad: chunk-relative pair
  int h = 0, c = 0, s = 0, t = 0;  // density: point half, comp, spin, 128-orbital tile
  // nh: column parts of a 128-function block in a V unit (128 / N, a
  // compile-time constant at the kernel's call sites); MODE = a.mode, so
  // each kernel carries only its own mode's decoding
  template <int MODE>
  __device__ UnitIter(std::integral_constant<int, MODE>, const TcArgs &a, long u, int nh) {
    if constexpr (MODE == TC_MODE_V) {
      const long n2 = a.ntiles * nh, n3 = n2 * a.nz;
      sp = (int)(u / n3);
      u %= n3;
      zi = (int)(u / n2);
      u %= n2;
      hc = (int)(u % nh);
      const int t = a.vtiles[u / nh];
      I = t >> 16;
      J = t & 0xffff;
    } else if constexpr (MODE == TC_MODE_GRAD || MODE == TC_MODE_X) {
      const int nt = 128 / a.nt;  // column parts of the block (N = 64: two halves)
      t = (int)(u % nt);
      h = (int)((u / nt) % 2);
      const int nc = MODE == TC_MODE_X ? a.ncomp : 1;
      c = (int)((u / (2 * nt)) % nc);
      s = (int)((u / (2 * nt * nc)) % a.nspin);
      q = u / (2 * nt * nc * a.nspin);
      bl = a.pair_batch[a.p0 + q] - a.b0;
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

struct Group {
  int nsteps;   // K steps of 64 bytes
  long qa, qb;  // V: chunk-relative pairs of the row / column blocks
  int blk;      // density: function block (-1: empty batch)
};

__device__ __forceinline__ int blk_pos(const uint32_t *m, int I) {
  int pos = 0;
  for (int w = 0; w < (I >> 5); ++w) pos += __popc(m[w]);
  return pos + __popc(m[I >> 5] & ((1u << (I & 31)) - 1u));
}
__device__ __forceinline__ bool blk_has(const uint32_t *m, int I) { return (m[I >> 5] >> (I & 31)) & 1u; }

// Calls fn(group, coords) for each accumulation group of a unit; the three
// roles run the same iteration so their barrier phases stay in step.
// coords(k, xa, ya, za, xb, yb, zb) gives the 3-D TMA box origins of step k.
template <int MODE, class Fn>
__device__ __forceinline__ void for_each_group(const TcArgs &a, const UnitIter &it, Fn &&fn) {
  if constexpr (MODE == TC_MODE_V) {
    const int Jb = it.J;
    for (long b = a.b0 + it.sp; b < a.b1; b += a.nsplit) {
      const uint32_t *m = a.mask + b * a.mask_words;
      if (!blk_has(m, it.I) || !blk_has(m, Jb)) continue;
      const long qb0 = a.pair_off[b] - a.p0;
      Group g;
      g.nsteps = 4;
      g.qa = qb0 + blk_pos(m, it.I);
      g.qb = qb0 + blk_pos(m, Jb);
      g.blk = 0;
      const int za = (int)(g.qa * 4), zb = (int)((g.qb * a.nz + it.zi) * 4), yb = a.nt * it.hc;
      fn(g, [=](int k, int &xa, int &ya, int &zA, int &xb, int &yB, int &zB) {
        xa = 64 * k;
        ya = 0;
        zA = za;
        xb = 64 * k;
        yB = yb;
        zB = zb;
      });
    }
  } else if constexpr (MODE == TC_MODE_GRAD || MODE == TC_MODE_X) {
    // one run over all orbitals: A = T_c digits of (batch, spin, comp, half)
    // (the Y pass: c = 0 only), B = (C occ) digits of the pair's block
    Group g;
    g.nsteps = a.nocc_pad / 64;
    g.qa = it.q;
    g.qb = 0;
    g.blk = a.pair_blk[a.p0 + it.q];
    const int nc = MODE == TC_MODE_X ? a.ncomp : 1;
    const int za = (int)((((it.bl * a.nspin + it.s) * nc + it.c) * 2 + it.h) * 4), yb = 128 * g.blk + a.nt * it.t,
              zb = it.s * 4;
    fn(g, [=](int k, int &xa, int &ya, int &zA, int &xb, int &yB, int &zB) {
      xa = 64 * k;
      ya = 0;
      zA = za;
      xb = 64 * k;
      yB = yb;
      zB = zb;
    });
  } else {
    const long b = a.b0 + it.bl;
    const int q0 = a.pair_off[b], q1 = a.pair_off[b + 1];
    for (int q = q0; q < q1; ++q) {
      Group g;
      g.nsteps = 2;
      g.qa = q - a.p0;
      g.qb = 0;
      g.blk = a.pair_blk[q];
      const int za = (int)((g.qa * a.ncs + it.c) * 4), ya = 128 * it.h;
      const int xb0 = g.blk * 128, yb = a.nt * it.t, zb = it.s * 4;
      fn(g, [=](int k, int &xa, int &yA, int &zA, int &xb, int &yB, int &zB) {
        xa = 64 * k;
        yA = ya;
        zA = za;
        xb = xb0 + 64 * k;
        yB = yb;
        zB = zb;
      });
    }
    if (q1 == q0) {  // batch without significant functions: one empty group
      Group g;
      g.nsteps = 0;
      g.qa = g.qb = 0;
      g.blk = -1;
      fn(g, [=](int, int &, int &, int &, int &, int &, int &) {});
    }
  }
}

template <int MODE, int NW, int EW = NW / 8>
__global__ void __launch_bounds__(TcShape<NW, EW>::kThreads, 1)
    tc_i8_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcArgs a) {
  using Sh = TcShape<NW, EW>;
  constexpr int N = Sh::N, NBUF = Sh::NBUF, kStages = Sh::kStages, kStageBytes = Sh::kStageBytes, CW = Sh::CW;
  static_assert(MODE == TC_MODE_V || CW == 32, "the density, Y and X epilogues take 32 columns a warp");
  extern __shared__ __align__(1024) uint8_t dsmem[];
  __shared__ uint64_t full_bar[kStages], empty_bar[kStages], tfull_bar[NBUF], tempty_bar[NBUF], drain_bar, stall_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_flag;
  // V and density: the column scales of each epilogue warp's current group
  __shared__ __align__(16) double colscale[MODE == TC_MODE_V || MODE == TC_MODE_DENSITY ? Sh::EW * CW : 2];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dsmem) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < NBUF; ++i) {
      mbar_init(&tfull_bar[i], 1);
      mbar_init(&tempty_bar[i], Sh::kEpiThreads);
    }
    mbar_init(&drain_bar, 1);
    mbar_init(&stall_bar, 1);
    fence_mbar_init();
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
  }
  if (warp == 1) {
    tmem_alloc(&tmem_base_sh, 512);
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
        const UnitIter it(std::integral_constant<int, MODE>{}, a, u, kBlockF / N);
        for_each_group<MODE>(a, it, [&](const Group &g, auto coords) {
          for (int k = 0; k < g.nsteps && !abort_flag; ++k, ++step) {
            const int st = step % kStages;
            if (!mbar_wait(&empty_bar[st], ((step / kStages) & 1) ^ 1, a.err, 1, &abort_flag, a.wait_ns)) return;
            int xa, ya, za, xb, yb, zb;
            coords(k, xa, ya, za, xb, yb, zb);
            uint8_t *base = smem + st * kStageBytes;
            mbar_arrive_expect_tx(&full_bar[st], kStageBytes);
            tma_load_3d(base, &mapA, xa, ya, za, &full_bar[st]);
            tma_load_3d(base + kABytes, &mapB, xb, yb, zb, &full_bar[st]);
          }
        });
      }
      volatile int keep_waiting = 0;
      for (uint32_t k = (step > kStages ? step - kStages : 0); k < step; ++k)
        mbar_wait(&full_bar[k % kStages], (k / kStages) & 1, a.err, 2, &keep_waiting, kDrainLimitNs);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t step = 0, grp = 0;
      if (a.stall) mbar_wait(&stall_bar, 0, a.err, 7, &abort_flag, a.wait_ns);
      for (long u = blockIdx.x; u < a.nunits && !abort_flag; u += gridDim.x) {
        const UnitIter it(std::integral_constant<int, MODE>{}, a, u, kBlockF / N);
        for_each_group<MODE>(a, it, [&](const Group &g, auto) {
          if (abort_flag) return;
          // TMEM buffer grp % NBUF: wait until the epilogue has read the group
          // that used it last
          const uint32_t buf = grp % NBUF, use = grp / NBUF;
          if (!mbar_wait(&tempty_bar[buf], (use & 1) ^ 1, a.err, 3, &abort_flag, a.wait_ns)) return;
          tc_fence_after();
          const uint32_t d = tmem + buf * 4 * N;
          for (int k = 0; k < g.nsteps; ++k, ++step) {
            const int st = step % kStages;
            if (!mbar_wait(&full_bar[st], (step / kStages) & 1, a.err, 4, &abort_flag, a.wait_ns)) return;
            tc_fence_after();
            const uint32_t base = smem_u32(smem + st * kStageBytes);
            // products of A digit plane i with B planes j = 0 .. 3-i into
            // level L = i + j; the A plane stays in the collector buffer for
            // its run, so shared memory feeds 4 A tiles per 32-byte K slice
            // instead of 10
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                const uint64_t ad = smem_desc_k64(base + i * (128 * 64) + kk * 32);
#pragma unroll
                for (int j = 0; j <= 3 - i; ++j) {
                  const uint64_t bd = smem_desc_k64(base + kABytes + j * (N * 64) + kk * 32);
                  const uint32_t dt = d + (i + j) * N;
                  const uint32_t acc = (k == 0 && kk == 0 && i == 0) ? 0u : 1u;
                  if (i == 3)
                    mma_i8_a<CollectorDiscard>(dt, ad, bd, Sh::kIdesc, acc);
                  else if (j == 0)
                    mma_i8_a<CollectorFill>(dt, ad, bd, Sh::kIdesc, acc);
                  else if (j == 3 - i)
                    mma_i8_a<CollectorLastUse>(dt, ad, bd, Sh::kIdesc, acc);
                  else
                    mma_i8_a<CollectorUse>(dt, ad, bd, Sh::kIdesc, acc);
                }
              }
            mma_commit(&empty_bar[st]);
          }
          mma_commit(&tfull_bar[buf]);
          ++grp;
        });
      }
      volatile int keep_waiting = 0;
      mma_commit(&drain_bar);
      mbar_wait(&drain_bar, 0, a.err, 5, &keep_waiting, kDrainLimitNs);
    }
  } else {
    // ------------------------------------------------------ epilogue
    const int q = warp & 3, cq = (warp - 2) >> 2;
    const int row = 32 * q + lane;
    const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
    uint32_t grp = 0;
    for (long u = blockIdx.x; u < a.nunits && !abort_flag; u += gridDim.x) {
      const UnitIter it(std::integral_constant<int, MODE>{}, a, u, kBlockF / N);
      double acc[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) acc[j] = 0.0;
      bool any = false;
      for_each_group<MODE>(a, it, [&](const Group &g, auto) {
        if (abort_flag) return;
        const uint32_t buf = grp % NBUF, use = grp / NBUF;
        if constexpr (MODE == TC_MODE_X) {
          // X_c(g, mu) of the thread's point and 32 functions, written in
          // FP64 slice by slice (8 consecutive doubles a slice)
          const int gpt = 128 * it.h + row;
          const double sa =
              a.sA[((((it.bl * a.nspin + it.s) * a.ncomp + it.c) * 2 + it.h)) * 128 + row] * kTwoM36;
          const double sbl = a.sB[(size_t)it.s * a.nbf_pad + 128 * g.blk + 64 * it.t + 32 * cq + lane];
          if (!mbar_wait(&tfull_bar[buf], use & 1, a.err, 6, &abort_flag, a.wait_ns)) return;
          tc_fence_after();
          __syncwarp();
          double *Xp = a.X + ((((size_t)it.q * a.nspin + it.s) * a.ncomp + it.c) * kBatch + gpt) * kBlockF +
                       64 * it.t + 32 * cq;
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            uint32_t v0[8], v1[8], v2[8], v3[8];
            const uint32_t ta = tmem + lane_addr + buf * 4 * N + 32 * cq + 8 * h;
            tmem_ld8u_async(ta, v0);
            tmem_ld8u_async(ta + N, v1);
            tmem_ld8u_async(ta + 2 * N, v2);
            tmem_ld8u_async(ta + 3 * N, v3);
            tmem_wait8(v0);
            tmem_wait8(v1);
            tmem_wait8(v2);
            tmem_wait8(v3);
            if (h == 3) {
              tc_fence_before();
              mbar_arrive(&tempty_bar[buf]);
            }
            double x[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
              x[j] = level_sum(v0[j], v1[j], v2[j], v3[j]) * (sa * __shfl_sync(0xffffffffu, sbl, 8 * h + j));
#pragma unroll
            for (int j = 0; j < 8; j += 2) reinterpret_cast<double2 *>(Xp + 8 * h + j)[0] = make_double2(x[j], x[j + 1]);
          }
          ++grp;
          return;
        }
        if constexpr (MODE == TC_MODE_GRAD) {
          // Y(g, mu) of the thread's point and 32 functions stays in
          // registers: the thread adds grad phi_c(g, mu) Y(g, mu) over them
          // (c = x, y, z), grad phi from the pass-A digits, and writes three
          // partial sums that ygrad_sum_kernel adds up per point.  The 32
          // columns go in NH parts (two of 16 in the 96-register N = 128
          // shape); each digit plane of a component and part is one load per
          // thread (the part's function bytes of its point), and the loads of
          // the next (part, component) are in flight while the current one is
          // combined, those of the first before the wait for the accumulators.
          constexpr int NH = N == 128 ? 2 : 1, CWH = 32 / NH, WPP = CWH / 4;
          const int gpt = 128 * it.h + row;
          const int f0 = N * it.t + 32 * cq;  // the warp's first function in the block
          constexpr size_t kPlane = (size_t)kBatch * kBlockF;  // one digit plane of a pair, bytes
          const uint8_t *dg = a.qphT + ((size_t)it.q * a.ncs + 1) * 4 * kPlane + (size_t)gpt * kBlockF + f0;
          uint32_t w0[4][WPP], w1[4][WPP];
          auto load = [&](int idx, uint32_t(&w)[4][WPP]) {  // idx = 3 part + component
            const int hf = idx / 3, c = idx % 3;
#pragma unroll
            for (int d = 0; d < 4; ++d) {
              const uint8_t *p = dg + (4 * c + d) * kPlane + CWH * hf;
              if constexpr (WPP == 8)
                ldg256(p, w[d]);
              else
                ldg128(p, w[d]);
            }
          };
          load(0, w0);
          const double sa = a.sA[((it.bl * a.nspin + it.s) * 2 + it.h) * 128 + row] * kTwoM36;
          const double sbl = a.sB[(size_t)it.s * a.nbf_pad + 128 * g.blk + f0 + lane];
          if (!mbar_wait(&tfull_bar[buf], use & 1, a.err, 6, &abort_flag, a.wait_ns)) return;
          tc_fence_after();
          __syncwarp();
          double gs[3] = {0.0, 0.0, 0.0};
          // word k of plane d holds digit d of functions 4k .. 4k + 3 of the part
          auto combine = [&](const uint32_t(&w)[4][WPP], const double(&y)[CWH]) {
            double gsum = 0.0;
#pragma unroll
            for (int k = 0; k < WPP; ++k) {
              const uint32_t wd[4] = {w[3][k], w[2][k], w[1][k], w[0][k]};
              uint32_t bw[4];
              transpose4(wd, bw);
#pragma unroll
              for (int e = 0; e < 4; ++e) gsum = fma(int_to_double(digits_value(bw[e])), y[4 * k + e], gsum);
            }
            return gsum;
          };
#pragma unroll
          for (int hf = 0; hf < NH; ++hf) {
            double y[CWH];
            // slices of SLW columns (4 in the 96-register shape)
            constexpr int SLW = NH == 2 ? 4 : 8;
#pragma unroll
            for (int h = 0; h < CWH / SLW; ++h) {
              uint32_t v0[SLW], v1[SLW], v2[SLW], v3[SLW];
              const uint32_t ta = tmem + lane_addr + buf * 4 * N + 32 * cq + CWH * hf + SLW * h;
              if constexpr (SLW == 8) {
                tmem_ld8u_async(ta, v0);
                tmem_ld8u_async(ta + N, v1);
                tmem_ld8u_async(ta + 2 * N, v2);
                tmem_ld8u_async(ta + 3 * N, v3);
                tmem_wait8(v0);
                tmem_wait8(v1);
                tmem_wait8(v2);
                tmem_wait8(v3);
              } else {
                tmem_ld4u_async(ta, v0);
                tmem_ld4u_async(ta + N, v1);
                tmem_ld4u_async(ta + 2 * N, v2);
                tmem_ld4u_async(ta + 3 * N, v3);
                tmem_wait4x4(v0, v1, v2, v3);
              }
              if (hf == NH - 1 && h == CWH / SLW - 1) {
                tc_fence_before();
                mbar_arrive(&tempty_bar[buf]);
              }
#pragma unroll
              for (int j = 0; j < SLW; ++j)
                y[SLW * h + j] = level_sum(v0[j], v1[j], v2[j], v3[j]) *
                                 (sa * __shfl_sync(0xffffffffu, sbl, CWH * hf + SLW * h + j));
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const int idx = 3 * hf + c;
              if ((idx & 1) == 0) {
                if (idx + 1 < 3 * NH) load(idx + 1, w1);
                gs[c] += combine(w0, y);
              } else {
                if (idx + 1 < 3 * NH) load(idx + 1, w0);
                gs[c] += combine(w1, y);
              }
            }
          }
          // partial sum p = (column part, warp column group) of 4 per (pair, spin)
          const int p = it.t * (N / 32) + cq;
          double *out = a.Gp + (((size_t)it.q * a.nspin + it.s) * 4 + p) * 3 * kBatch + gpt;
#pragma unroll
          for (int c = 0; c < 3; ++c)
            out[c * kBatch] = gs[c] * (a.sphT[((size_t)it.q * a.ncs + 1 + c) * kBatch + gpt] * 0x1p-29);
          ++grp;
          return;
        }
        const bool live = g.nsteps > 0;
        // the group's row and column scales are loaded before the wait for
        // its accumulators, so their latency hides behind the MMAs
        double sa_g = 0.0, sb_g[MODE == TC_MODE_V ? CW / 32 : 1];
        if (live) {
          if constexpr (MODE == TC_MODE_V) {
            sa_g = a.sA[g.qa * 128 + row];
            const double *sbp = a.sB + (g.qb * a.nz + it.zi) * 128 + N * it.hc + CW * cq;
#pragma unroll
            for (int k = 0; k < CW / 32; ++k) sb_g[k] = sbp[32 * k + lane];
          } else {
            sa_g = a.sA[(g.qa * a.ncs + it.c) * 256 + 128 * it.h + row];
            sb_g[0] = a.sB[((size_t)it.s * a.nocc_pad + N * it.t + 32 * cq + lane) * a.nblk + g.blk];
          }
        }
        if (!mbar_wait(&tfull_bar[buf], use & 1, a.err, 6, &abort_flag, a.wait_ns)) return;
        tc_fence_after();
        __syncwarp();
        // exact combine of the four levels, S = sum_L 2^(8 (3 - L)) Acc_L:
        // |Acc_L| < 2^24 for K <= 256, so |S| < 2^49 (level_sum); the product
        // is s_a s_b 2^-36 S (one rounding per group and element)
        if constexpr (MODE == TC_MODE_V || MODE == TC_MODE_DENSITY) {
          // s_a is the thread's row scale; the warp's CW column scales are
          // staged in shared memory once per group and read back as
          // broadcasts, two per 16-byte load (instead of two shuffles per
          // element).  Slices of four columns are software-pipelined: the
          // loads of slice h + 1 are in flight while slice h is combined, and
          // TMEM is released as soon as the last slice has arrived in
          // registers.
          if (live) {
            const double sa = sa_g * kTwoM36;
            double *cs = colscale + (warp - 2) * CW;
#pragma unroll
            for (int k = 0; k < CW / 32; ++k) cs[32 * k + lane] = sb_g[k];
            __syncwarp();
            const uint32_t tb = tmem + lane_addr + buf * 4 * N + CW * cq;
            constexpr int NS = CW / 4;
            uint32_t p0[4], p1[4], p2[4], p3[4], r0[4], r1[4], r2[4], r3[4];
            auto issue = [&](int h, uint32_t(&x0)[4], uint32_t(&x1)[4], uint32_t(&x2)[4], uint32_t(&x3)[4]) {
              const uint32_t ta = tb + 4 * h;
              tmem_ld4u_async(ta, x0);
              tmem_ld4u_async(ta + N, x1);
              tmem_ld4u_async(ta + 2 * N, x2);
              tmem_ld4u_async(ta + 3 * N, x3);
            };
            auto combine = [&](int h, const uint32_t(&x0)[4], const uint32_t(&x1)[4], const uint32_t(&x2)[4],
                               const uint32_t(&x3)[4]) {
              const double2 c01 = *reinterpret_cast<const double2 *>(cs + 4 * h);
              const double2 c23 = *reinterpret_cast<const double2 *>(cs + 4 * h + 2);
              const double sc[4] = {c01.x, c01.y, c23.x, c23.y};
#pragma unroll
              for (int j = 0; j < 4; ++j)
                acc[4 * h + j] = fma(level_sum(x0[j], x1[j], x2[j], x3[j]), sa * sc[j], acc[4 * h + j]);
            };
            issue(0, p0, p1, p2, p3);
#pragma unroll
            for (int h = 0; h < NS; ++h) {
              if ((h & 1) == 0) {
                tmem_wait4x4(p0, p1, p2, p3);
                if (h + 1 < NS) issue(h + 1, r0, r1, r2, r3);
              } else {
                tmem_wait4x4(r0, r1, r2, r3);
                if (h + 1 < NS) issue(h + 1, p0, p1, p2, p3);
              }
              if (h + 1 == NS) {
                tc_fence_before();
                mbar_arrive(&tempty_bar[buf]);
              }
              if ((h & 1) == 0)
                combine(h, p0, p1, p2, p3);
              else
                combine(h, r0, r1, r2, r3);
            }
          } else {
            tc_fence_before();
            mbar_arrive(&tempty_bar[buf]);
          }
          ++grp;
          any = any || live;
          return;
        }
      });
      if constexpr (MODE == TC_MODE_V) {
        if (any) {
          double *Vz = a.V + (size_t)it.zi * a.nbf_pad * a.nbf_pad;
          const size_t r = (size_t)it.I * 128 + row;
          const size_t c0 = (size_t)it.J * 128 + N * it.hc + CW * cq;
          if (a.nsplit > 1) {
#pragma unroll
            for (int j = 0; j < CW; ++j) atomicAdd(&Vz[r + (c0 + j) * a.nbf_pad], acc[j]);
          } else {
#pragma unroll
            for (int j = 0; j < CW; ++j) Vz[r + (c0 + j) * a.nbf_pad] += acc[j];
          }
        }
      } else if constexpr (MODE == TC_MODE_GRAD || MODE == TC_MODE_X) {
        // the partial sums (grad) or X (x) are written per group above
      } else {
        const long plane = (it.bl * a.nspin + it.s) * a.ncomp + it.c;
        double *Tp = a.T + plane * (long)a.nocc_pad * 256 + 128 * it.h + row;
#pragma unroll
        for (int j = 0; j < 32; ++j) Tp[(size_t)(N * it.t + 32 * cq + j) * 256] = acc[j];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ------------------------------------------------ V on CTA pairs ----
//
// The V contraction on clusters of two CTAs (tcgen05 cta_group::2): one
// M = 256 x N = 64 MMA covers the rows of two function blocks (I0 = 2R on
// rank 0, I1 = 2R + 1 on rank 1) against 64 columns of block J.  Per K step
// each CTA stages its own block's Phi digits (4 planes x 128 rows) and half
// of the 64 Z columns (4 planes x 32 rows), 40 KB, in a 5-stage ring.
// Rank 0 issues the MMAs; its full barriers count the bytes of both CTAs'
// loads, and its commits arrive on the empty and TMEM-full barriers of both
// CTAs.  Four int32 levels of N = 64 fill half of TMEM, so the accumulators
// are double-buffered: the epilogue of one batch (each CTA reads its own
// 128 rows) overlaps the MMAs of the next, and both CTAs' epilogue warps
// report a drained buffer on rank 0's TMEM-empty barrier.  A batch where
// only one of the two row blocks is significant still runs the pair's MMAs:
// the CTA without its block loads the other block's digits and discards
// its accumulators.  Per SM an MMA reads 4 KB of A (kept in the collector
// across its run of B planes) and 1 KB of B from shared memory for
// 128 x 64 x 32 products, so the tensor pipe, not shared memory, bounds it.
constexpr int kPairStages = 5;
constexpr int kPairABytes = 4 * 128 * 64;  // four digit planes, 128 rows x 64 B
constexpr int kPairBBytes = 4 * 32 * 64;   // four digit planes, 32 rows x 64 B
constexpr int kPairStageBytes = kPairABytes + kPairBBytes;
constexpr int kPairSmem = kPairStages * kPairStageBytes + 1024;
constexpr uint32_t kPairIdesc = idesc_i8(256, 64);

struct PairGroup {
  long qa;    // chunk-relative pair whose Phi digits this CTA loads
  long qb;    // chunk-relative pair of block J
  bool live;  // this CTA's row block is significant in the batch
};

// The batches of a pair unit (row blocks 2R, 2R + 1, column block J): those
// where J and at least one of the row blocks are significant.
template <class Fn>
__device__ __forceinline__ void for_each_pair_group(const TcArgs &a, int R, int J, int sp, uint32_t rank, Fn &&fn) {
  const int I0 = 2 * R, I1 = 2 * R + 1;
  for (long b = a.b0 + sp; b < a.b1; b += a.nsplit) {
    const uint32_t *m = a.mask + b * a.mask_words;
    if (!blk_has(m, J)) continue;
    const bool h0 = blk_has(m, I0), h1 = I1 < a.nblk && blk_has(m, I1);
    if (!h0 && !h1) continue;
    const bool own = rank == 0 ? h0 : h1;
    const int Ia = (rank == 0) == own ? I0 : I1;
    const long qb0 = a.pair_off[b] - a.p0;
    PairGroup g;
    g.qa = qb0 + blk_pos(m, Ia);
    g.qb = qb0 + blk_pos(m, J);
    g.live = own;
    fn(g);
  }
}

// EW epilogue warps a CTA (8: 32 columns each, 16: 16 columns each)
template <int EW>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(64 + 32 * EW, 1)
    tc_v_pair_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcArgs a) {
  constexpr int N = 64, CW = 4 * N / EW, S = kPairStages;
  static_assert(CW == 16 || CW == 32, "16 or 32 columns an epilogue warp");
  extern __shared__ __align__(1024) uint8_t dsmem[];
  __shared__ uint64_t full_bar[S], empty_bar[S], tfull_bar[2], tempty_bar[2], drain_bar, stall_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_flag;
  __shared__ __align__(16) double colscale[EW * CW];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dsmem) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int i = 0; i < S; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull_bar[i], 1);
      mbar_init(&tempty_bar[i], 2 * EW);  // one arrival per epilogue warp of either CTA
    }
    mbar_init(&drain_bar, 1);
    mbar_init(&stall_bar, 1);
    fence_mbar_init();
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
  }
  if (warp == 1) {
    tmem_alloc_pair(&tmem_base_sh, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync();  // both CTAs' barriers initialised before any remote arrival
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  // a wait that gave up stops the other CTA of the pair as well
  const uint32_t peer_abort = map_to_rank((const void *)&abort_flag, rank ^ 1u);
  auto give_up = [&]() { st_cluster_u32(peer_abort, 1u); };
  const long cid = cluster_id_x(), ncl = cluster_count_x();
  auto unit = [&](long u, int &R, int &J, int &zi, int &hc, int &sp) {
    const long n2 = a.ntiles * 2, n3 = n2 * a.nz;
    sp = (int)(u / n3);
    u %= n3;
    zi = (int)(u / n2);
    u %= n2;
    hc = (int)(u % 2);
    const int t = a.vtiles[u / 2];
    R = t >> 16;
    J = t & 0xffff;
  };

  if (warp == 0) {
    // ------------------------------------------------------ TMA producer
    if (lane == 0) {
      uint32_t step = 0;
      for (long u = cid; u < a.nunits && !abort_flag; u += ncl) {
        int R, J, zi, hc, sp;
        unit(u, R, J, zi, hc, sp);
        for_each_pair_group(a, R, J, sp, rank, [&](const PairGroup &g) {
          const int za = (int)(g.qa * 4), zb = (int)((g.qb * a.nz + zi) * 4), yb = 64 * hc + 32 * (int)rank;
          for (int k = 0; k < 4 && !abort_flag; ++k, ++step) {
            const int st = step % S;
            if (!mbar_wait(&empty_bar[st], ((step / S) & 1) ^ 1, a.err, 1, &abort_flag, a.wait_ns)) {
              give_up();
              return;
            }
            uint8_t *base = smem + st * kPairStageBytes;
            if (rank == 0) mbar_arrive_expect_tx(&full_bar[st], 2 * kPairStageBytes);
            const uint32_t fb = map_to_rank(&full_bar[st], 0);
            tma_load_3d_pair(base, &mapA, 64 * k, 0, za, fb);
            tma_load_3d_pair(base + kPairABytes, &mapB, 64 * k, yb, zb, fb);
          }
        });
      }
      if (rank == 0) {
        // the last stages' loads of both CTAs have landed
        volatile int keep_waiting = 0;
        for (uint32_t k = (step > S ? step - S : 0); k < step; ++k)
          mbar_wait(&full_bar[k % S], (k / S) & 1, a.err, 2, &keep_waiting, kDrainLimitNs);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------ MMA issuer (rank 0)
    if (lane == 0 && rank == 0) {
      uint32_t step = 0, grp = 0;
      if (a.stall && !mbar_wait(&stall_bar, 0, a.err, 7, &abort_flag, a.wait_ns)) give_up();
      for (long u = cid; u < a.nunits && !abort_flag; u += ncl) {
        int R, J, zi, hc, sp;
        unit(u, R, J, zi, hc, sp);
        for_each_pair_group(a, R, J, sp, rank, [&](const PairGroup &) {
          if (abort_flag) return;
          const uint32_t buf = grp & 1, use = grp >> 1;
          if (!mbar_wait(&tempty_bar[buf], (use & 1) ^ 1, a.err, 3, &abort_flag, a.wait_ns)) {
            give_up();
            return;
          }
          tc_fence_after();
          const uint32_t d = tmem + buf * 4 * N;
          for (int k = 0; k < 4; ++k, ++step) {
            const int st = step % S;
            if (!mbar_wait(&full_bar[st], (step / S) & 1, a.err, 4, &abort_flag, a.wait_ns)) {
              give_up();
              return;
            }
            tc_fence_after();
            const uint32_t base = smem_u32(smem + st * kPairStageBytes);
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                const uint64_t ad = smem_desc_k64(base + i * (128 * 64) + kk * 32);
#pragma unroll
                for (int j = 0; j <= 3 - i; ++j) {
                  const uint64_t bd = smem_desc_k64(base + kPairABytes + j * (32 * 64) + kk * 32);
                  const uint32_t dt = d + (i + j) * N;
                  const uint32_t acc = (k == 0 && kk == 0 && i == 0) ? 0u : 1u;
                  if (i == 3)
                    mma_i8_pair<CollectorDiscard>(dt, ad, bd, kPairIdesc, acc);
                  else if (j == 0)
                    mma_i8_pair<CollectorFill>(dt, ad, bd, kPairIdesc, acc);
                  else if (j == 3 - i)
                    mma_i8_pair<CollectorLastUse>(dt, ad, bd, kPairIdesc, acc);
                  else
                    mma_i8_pair<CollectorUse>(dt, ad, bd, kPairIdesc, acc);
                }
              }
            mma_commit_pair(&empty_bar[st], 3);
          }
          mma_commit_pair(&tfull_bar[buf], 3);
          ++grp;
        });
      }
      volatile int keep_waiting = 0;
      mma_commit_pair(&drain_bar, 1);
      mbar_wait(&drain_bar, 0, a.err, 5, &keep_waiting, kDrainLimitNs);
    }
  } else {
    // ------------------------------------------------------ epilogue
    const int q = warp & 3, cq = (warp - 2) >> 2;
    const int row = 32 * q + lane;
    const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
    const uint32_t tempty_r0[2] = {map_to_rank(&tempty_bar[0], 0), map_to_rank(&tempty_bar[1], 0)};
    double *cs = colscale + (warp - 2) * CW;
    uint32_t grp = 0;
    for (long u = cid; u < a.nunits && !abort_flag; u += ncl) {
      int R, J, zi, hc, sp;
      unit(u, R, J, zi, hc, sp);
      double acc[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) acc[j] = 0.0;
      bool any = false;
      for_each_pair_group(a, R, J, sp, rank, [&](const PairGroup &g) {
        if (abort_flag) return;
        const uint32_t buf = grp & 1, use = grp >> 1;
        auto release = [&]() {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_cluster(tempty_r0[buf]);
        };
        double sa = 0.0, sb = 0.0;
        if (g.live) {
          sa = a.sA[g.qa * 128 + row] * kTwoM36;
          if (lane < CW) sb = a.sB[(g.qb * a.nz + zi) * 128 + 64 * hc + CW * cq + lane];
        }
        if (!mbar_wait(&tfull_bar[buf], use & 1, a.err, 6, &abort_flag, a.wait_ns)) {
          give_up();
          return;
        }
        tc_fence_after();
        __syncwarp();
        if (g.live) {
          if (lane < CW) cs[lane] = sb;
          __syncwarp();
          const uint32_t tb = tmem + lane_addr + buf * 4 * N + CW * cq;
          constexpr int NS = CW / 4;
          uint32_t p0[4], p1[4], p2[4], p3[4], r0[4], r1[4], r2[4], r3[4];
          auto issue = [&](int h, uint32_t(&x0)[4], uint32_t(&x1)[4], uint32_t(&x2)[4], uint32_t(&x3)[4]) {
            const uint32_t ta = tb + 4 * h;
            tmem_ld4u_async(ta, x0);
            tmem_ld4u_async(ta + N, x1);
            tmem_ld4u_async(ta + 2 * N, x2);
            tmem_ld4u_async(ta + 3 * N, x3);
          };
          auto combine = [&](int h, const uint32_t(&x0)[4], const uint32_t(&x1)[4], const uint32_t(&x2)[4],
                             const uint32_t(&x3)[4]) {
            const double2 c01 = *reinterpret_cast<const double2 *>(cs + 4 * h);
            const double2 c23 = *reinterpret_cast<const double2 *>(cs + 4 * h + 2);
            const double sc[4] = {c01.x, c01.y, c23.x, c23.y};
#pragma unroll
            for (int j = 0; j < 4; ++j)
              acc[4 * h + j] = fma(level_sum(x0[j], x1[j], x2[j], x3[j]), sa * sc[j], acc[4 * h + j]);
          };
          issue(0, p0, p1, p2, p3);
#pragma unroll
          for (int h = 0; h < NS; ++h) {
            if ((h & 1) == 0) {
              tmem_wait4x4(p0, p1, p2, p3);
              if (h + 1 < NS) issue(h + 1, r0, r1, r2, r3);
            } else {
              tmem_wait4x4(r0, r1, r2, r3);
              if (h + 1 < NS) issue(h + 1, p0, p1, p2, p3);
            }
            if (h + 1 == NS) release();
            if ((h & 1) == 0)
              combine(h, p0, p1, p2, p3);
            else
              combine(h, r0, r1, r2, r3);
          }
          __syncwarp();  // the column scales are read before the next group overwrites them
        } else {
          release();
        }
        ++grp;
        any = any || g.live;
      });
      const int I = 2 * R + (int)rank;
      if (any && I < a.nblk) {
        double *Vz = a.V + (size_t)zi * a.nbf_pad * a.nbf_pad;
        const size_t r = (size_t)I * 128 + row;
        const size_t c0 = (size_t)J * 128 + 64 * hc + CW * cq;
        if (a.nsplit > 1) {
#pragma unroll
          for (int j = 0; j < CW; ++j) atomicAdd(&Vz[r + (c0 + j) * a.nbf_pad], acc[j]);
        } else {
#pragma unroll
          for (int j = 0; j < CW; ++j) Vz[r + (c0 + j) * a.nbf_pad] += acc[j];
        }
      }
    }
  }
  tc_fence_before();
  cluster_sync();  // neither CTA leaves while the other's MMAs or loads may touch its memory
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc_pair(tmem, 512);
  }
}

// ----------------------------------------------------- quantisation ----

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// A non-finite operand value (exponent field 0x7ff) would still become
// finite digits and a silently wrong product, so every quantiser reports one
// in *flag (the plan's numeric status word) and the build returns
// NKX_ERR_NUMERIC.  Called by all lanes of a warp.
__device__ __forceinline__ void report_nonfinite(bool bad, int *flag) {
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// four consecutive values -> four digit planes (one packed word per plane:
// w[p] byte k = digit p of value k, p = 0 the leading digit)
__device__ __forceinline__ void quant4(const double v[4], double inv, uint32_t w[4]) {
  const double s30 = inv * 0x1p30;
  uint32_t b[4], t[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) b[k] = digits_word(v[k], s30);
  transpose4(b, t);
#pragma unroll
  for (int p = 0; p < 4; ++p) w[p] = t[3 - p];
}

// Density operand B: orbital rows (spin, i) over each 128-function block.
// qct[spin][digit][i][f], sct[spin][i][blk]; rows i >= nocc are zero.
__global__ void quant_ct_kernel(const double *__restrict__ Ct, int nocc, int nocc_pad, int nspin, int nbf_pad,
                                int nblk, uint8_t *__restrict__ q, double *__restrict__ sc, int *nonfinite) {
  const long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= (long)nspin * nocc_pad * nblk) return;
  const int blk = (int)(r % nblk);
  const long si = r / nblk;
  const int s = (int)(si / nocc_pad), i = (int)(si % nocc_pad);
  const int f0 = blk * 128 + 4 * lane;
  double v[4] = {0, 0, 0, 0};
  if (i < nocc)
    for (int k = 0; k < 4; ++k) v[k] = Ct[((size_t)s * nocc + i) * nbf_pad + f0 + k];
  report_nonfinite(max(max(exp_field(v[0]), exp_field(v[1])), max(exp_field(v[2]), exp_field(v[3]))) == 0x7ffu,
                   nonfinite);
  const double m = warp_max(fmax(fmax(fabs(v[0]), fabs(v[1])), fmax(fabs(v[2]), fabs(v[3]))));
  double scl;
  const double inv = inv_pow2_scale(m, scl);
  uint32_t w[4];
  quant4(v, inv, w);
#pragma unroll
  for (int p = 0; p < 4; ++p)
    *reinterpret_cast<uint32_t *>(q + (((size_t)s * 4 + p) * nocc_pad + i) * nbf_pad + f0) = w[p];
  if (lane == 0) sc[((size_t)s * nocc_pad + i) * nblk + blk] = scl;
}

// 128 operand rows r with K values each, x(r, k) = src[k * kstride + r]
// (times kmul[k] when given; k >= K read as 0), into four digit planes
// out[d][r][k] (row stride Kpad bytes, plane stride plane_stride) with one
// power-of-two scale per row over all K, scale_out[r].  One thread per row;
// 64 values at a time go through a shared tile so the rows leave as 64-byte
// segments.
__device__ __forceinline__ void quant_rows_128(const double *__restrict__ src, long kstride,
                                               const double *__restrict__ kmul, int K, int Kpad,
                                               uint8_t *__restrict__ out, size_t plane_stride,
                                               double *__restrict__ scale_out) {
  __shared__ uint32_t tile[4][128][17];
  const int r = threadIdx.x;
  double m = 0.0;
  for (int k = 0; k < K; ++k) m = fmax(m, fabs(src[(size_t)k * kstride + r] * (kmul ? kmul[k] : 1.0)));
  double sc;
  const double s30 = inv_pow2_scale(m, sc) * 0x1p30;
  scale_out[r] = sc;
  for (int k0 = 0; k0 < Kpad; k0 += 64) {
#pragma unroll 4
    for (int w = 0; w < 16; ++w) {
      uint32_t b[4], t[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + 4 * w + j;
        const double v = k < K ? src[(size_t)k * kstride + r] * (kmul ? kmul[k] : 1.0) : 0.0;
        b[j] = digits_word(v, s30);
      }
      transpose4(b, t);
#pragma unroll
      for (int d = 0; d < 4; ++d) tile[d][r][w] = t[3 - d];
    }
    __syncthreads();
    for (int e = r; e < 4 * 128 * 16; e += 128) {
      const int d = e >> 11, rr = (e >> 4) & 127, w = e & 15;
      *reinterpret_cast<uint32_t *>(out + d * plane_stride + (size_t)rr * Kpad + k0 + 4 * w) = tile[d][rr][w];
    }
    __syncthreads();
  }
}

// Grad-mode operand A: T0(g, i) of every (batch, spin, half) of the chunk as
// rows g over the orbitals, qt0[(bl, s, h)][digit][g][i], st0[(bl, s, h)][g].
__global__ void __launch_bounds__(128) quant_t0_kernel(const double *__restrict__ T, int nocc, int nocc_pad,
                                                        uint8_t *__restrict__ q, double *__restrict__ sc) {
  const long base = blockIdx.x;  // ((bl * nspin + s) * 2 + h)
  const long plane = base >> 1;
  const int h = (int)(base & 1);
  quant_rows_128(T + plane * (long)nocc_pad * 256 + 128 * h, 256, nullptr, nocc, nocc_pad,
                 q + base * 4 * 128 * (size_t)nocc_pad, (size_t)128 * nocc_pad, sc + base * 128);
}

// Grad-mode operand B: (C occ)(mu, i) as rows mu over the orbitals,
// qco[s][digit][mu][i], sco[s][mu]; block y = spin, x = 128-function block.
__global__ void __launch_bounds__(128) quant_cocc_kernel(const double *__restrict__ Ct, const double *__restrict__ occ,
                                                          int nocc, int nocc_pad, int nbf_pad,
                                                          uint8_t *__restrict__ q, double *__restrict__ sc) {
  const int s = blockIdx.y, I = blockIdx.x;
  quant_rows_128(Ct + (size_t)s * nocc * nbf_pad + 128 * I, nbf_pad, occ + (size_t)s * nocc, nocc, nocc_pad,
                 q + ((size_t)s * 4 * nbf_pad + 128 * I) * nocc_pad, (size_t)nbf_pad * nocc_pad,
                 sc + (size_t)s * nbf_pad + 128 * I);
}

// grad rho(g) of one batch (block x of the chunk) and spin (block y), one
// thread per point: the sum over the batch's pairs, function halves and
// column groups of the partial sums 2 sum_mu grad phi_c(g, mu) Y(g, mu) that
// the fused Y pass wrote, Gp[pair][spin][t][cq][c][g] (a fixed order, so the
// result does not depend on scheduling).
__global__ void __launch_bounds__(256) ygrad_sum_kernel(const double *__restrict__ Gp, const int *__restrict__ pair_off,
                                                        long b0, long p0, int nspin, long npad,
                                                        double *__restrict__ grad) {
  const long b = b0 + blockIdx.x;
  const int s = blockIdx.y, g = threadIdx.x;
  const int q0 = pair_off[b], q1 = pair_off[b + 1];
  double gs[3] = {0.0, 0.0, 0.0};
  for (int q = q0; q < q1; ++q) {
    const double *p = Gp + ((size_t)(q - p0) * nspin + s) * 12 * kBatch + g;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) gs[c] += p[(3 * k + c) * kBatch];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) grad[((size_t)s * 3 + c) * npad + b * kBatch + g] = gs[c];
}

// Pass A, fused: collocation of one (batch, block) pair straight into the
// density operand digits.  Lane l owns functions f = 4l .. 4l+3, warp w the
// points g = w + 8j; the row scale of (comp, g) over the 128 functions of
// the block is a warp maximum.  qphT[pair][comp][digit][g][f],
// sphT[pair][comp][g].
template <bool GRAD>
__global__ void __launch_bounds__(256) colloc_quantT_kernel(const StoFunc *__restrict__ sto,
                                                            const int *__restrict__ fshell,
                                                            const StoShell *__restrict__ bshell,
                                                            const int *__restrict__ bnshell,
                                                            const double *__restrict__ px,
                                                            const double *__restrict__ py, const double *__restrict__ pz,
                                                            const int *__restrict__ pair_batch,
                                                            const int *__restrict__ pair_blk, long p0,
                                                            uint8_t *__restrict__ q, double *__restrict__ sc,
                                                            int *nonfinite) {
  constexpr int NC = GRAD ? 4 : 1;
  const long p = p0 + blockIdx.x;
  const int b = pair_batch[p], I = pair_blk[p];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ double sx[kBatch], sy[kBatch], sz[kBatch];
  __shared__ BlockFuncs B;
  __shared__ double wR[8][128], wC[8][128];
  for (int g = threadIdx.x; g < kBatch; g += blockDim.x) {
    sx[g] = px[(long)b * kBatch + g];
    sy[g] = py[(long)b * kBatch + g];
    sz[g] = pz[(long)b * kBatch + g];
  }
  load_block_funcs(B, sto, fshell, bshell, bnshell, I, threadIdx.x, blockDim.x);
  __syncthreads();
  const long qrel = blockIdx.x;
  for (int g = warp; g < kBatch; g += 8) {
    double v[4][4];
    __syncwarp();
    block_radials<GRAD>(B, lane, sx[g], sy[g], sz[g], wR[warp], wC[warp]);
    __syncwarp();
    block_funcs_eval4<GRAD>(B, lane, sx[g], sy[g], sz[g], wR[warp], wC[warp], v[0], v[1], v[2], v[3]);
#pragma unroll
    for (int k = 0; k < NC; ++k) {
      const unsigned el = max(max(exp_field(v[k][0]), exp_field(v[k][1])), max(exp_field(v[k][2]), exp_field(v[k][3])));
      report_nonfinite(el == 0x7ffu, nonfinite);
      double s;
      const double inv = warp_inv_pow2_scale(
          el, fmax(fmax(fabs(v[k][0]), fabs(v[k][1])), fmax(fabs(v[k][2]), fabs(v[k][3]))), s);
      uint32_t w[4];
      quant4(v[k], inv, w);
      const long pc = qrel * NC + k;
#pragma unroll
      for (int d = 0; d < 4; ++d) reinterpret_cast<uint32_t *>(q + ((pc * 4 + d) * 256 + g) * 128)[lane] = w[d];
      if (lane == 0) sc[pc * 256 + g] = s;
    }
  }
}

// Row scales of a pair's V operands from the per-warp maxima red[w][o][f]
// (256-thread blocks, o = 0 phi, o >= 1 the Z planes): one power-of-two scale
// per function row, sph[pair][f] and szs[pair][z][f].  (One scale for a whole
// Z block would let the V epilogue skip the per-column scales, but rows far
// below the block maximum then lose digits: max|dV| grew from about 1e-9 to
// 1.3e-7 on an open-shell water cluster, over the 1e-7 target.)
__device__ void store_operand_scales(double (*red)[4][128], int nop, int nz, long qrel, double *sph, double *szs) {
  for (int e = threadIdx.x; e < nop * 128; e += blockDim.x) {
    const int o = e / 128, ff = e % 128;
    double mm = 0.0;
    for (int w = 0; w < 8; ++w) mm = fmax(mm, red[w][o][ff]);
    double sc;
    inv_pow2_scale(mm, sc);
    if (o == 0)
      sph[qrel * 128 + ff] = sc;
    else
      szs[(qrel * nz + (o - 1)) * 128 + ff] = sc;
  }
}

// Pass B, part 1: collocation of one (batch, block) pair and the operand
// values of the V contraction, o = 0: phi, o = 1 + z: Z_z (z < nspin:
// c0 phi + c . grad phi with the functional's per-point coefficients;
// z == nspin for a separate J: 1/2 vJ phi), written as FP64 ws[pair][o][g][f]
// (lane l owns f = 4l .. 4l+3, warp w the points g = w + 8j), together with
// the row scale of every (o, f) over the 256 points: sph[pair][f],
// sz[pair][z][f].
template <bool GRAD, int NZ>
__global__ void __launch_bounds__(256, 2) colloc_z_kernel(const StoFunc *__restrict__ sto,
                                                         const int *__restrict__ fshell,
                                                         const StoShell *__restrict__ bshell,
                                                         const int *__restrict__ bnshell,
                                                         const double *__restrict__ px,
                                                         const double *__restrict__ py, const double *__restrict__ pz,
                                                         const int *__restrict__ pair_batch,
                                                         const int *__restrict__ pair_blk, long p0,
                                                         const double *__restrict__ coef, const double *__restrict__ vj,
                                                         int nspin, long npad, double *__restrict__ ws,
                                                         double *__restrict__ sph, double *__restrict__ szs,
                                                         int *nonfinite) {
  __shared__ double red[8][4][128];
  const long p = p0 + blockIdx.x, qrel = blockIdx.x;
  const int b = pair_batch[p], I = pair_blk[p];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nz = NZ, nop = 1 + NZ;
  const size_t T = (size_t)kBatch * kBlockF;
  __shared__ BlockFuncs B;
  // during the point loop red[w][0] and red[w][1] hold warp w's radial factors
  double *wR = red[warp][0], *wC = red[warp][1];
  load_block_funcs(B, sto, fshell, bshell, bnshell, I, threadIdx.x, blockDim.x);
  __syncthreads();
  double m[nop][4];
#pragma unroll
  for (int o = 0; o < nop; ++o)
#pragma unroll
    for (int c = 0; c < 4; ++c) m[o][c] = 0.0;
  double *out = ws + qrel * 4 * T;
  unsigned efield = 0;  // largest exponent field of the operand values (0x7ff: non-finite)
  for (int g = warp; g < kBatch; g += 8) {
    const long gg = (long)b * kBatch + g;
    const double x = px[gg], y = py[gg], z = pz[gg];
    double cf[NZ][4];
#pragma unroll
    for (int s = 0; s < NZ; ++s) {
      cf[s][0] = cf[s][1] = cf[s][2] = cf[s][3] = 0.0;
      if (s < nspin) {
        const double *cs = coef + (size_t)s * 4 * npad;
        cf[s][0] = cs[gg];
        if (GRAD) {
          cf[s][1] = cs[npad + gg];
          cf[s][2] = cs[2 * npad + gg];
          cf[s][3] = cs[3 * npad + gg];
        }
      } else {
        cf[s][0] = 0.5 * vj[gg];
      }
    }
    double v[nop][4], gx[4], gy[4], gz[4];
    __syncwarp();
    block_radials<GRAD>(B, lane, x, y, z, wR, wC);
    __syncwarp();
    block_funcs_eval4<GRAD>(B, lane, x, y, z, wR, wC, v[0], gx, gy, gz);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double val = v[0][c];
#pragma unroll
      for (int s = 0; s < NZ; ++s) {
        v[1 + s][c] = cf[s][0] * val;
        if (GRAD) v[1 + s][c] += cf[s][1] * gx[c] + cf[s][2] * gy[c] + cf[s][3] * gz[c];
      }
    }
#pragma unroll
    for (int o = 0; o < nop; ++o) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        m[o][c] = fmax(m[o][c], fabs(v[o][c]));
        efield = max(efield, exp_field(v[o][c]));
      }
      double2 *dst = reinterpret_cast<double2 *>(out + o * T + (size_t)g * kBlockF + 4 * lane);
      dst[0] = make_double2(v[o][0], v[o][1]);
      dst[1] = make_double2(v[o][2], v[o][3]);
    }
  }
  report_nonfinite(efield == 0x7ffu, nonfinite);
  __syncwarp();
#pragma unroll
  for (int o = 0; o < nop; ++o)
#pragma unroll
    for (int c = 0; c < 4; ++c) red[warp][o][4 * lane + c] = m[o][c];
  __syncthreads();
  store_operand_scales(red, nop, nz, qrel, sph, szs);
}

// Pass B of a build without J in one kernel: the V operands of one
// (batch, block) pair on a cluster of four CTAs, 64 points each.  Phi and
// grad Phi come back exactly from the pair's pass-A digits; the Z planes
// (Z_s = c0 phi + c . grad phi, s < nz) go to shared memory in FP64, phi as
// its packed pass-A digits and point scales, and each (plane, function)
// row's largest exponent field is reduced over the CTA's warps and then,
// pushed into every CTA's shared memory, over the four CTAs: the row scale is
// 2^(E - 1022) for the largest field E, the power-of-two scale of the row
// maximum.  Each CTA then writes the digits of its 64 points from shared
// memory as 16-byte pieces of the rows of qph[pair][digit][f][g] and
// qz[pair][z][digit][f][g]; rank 0 writes the scales sph[pair][f] and
// szs[pair][z][f].  Against the staging of Z in HBM by a separate kernel
// this moves about half the bytes (the pass-A digits in, the V digits
// out).  (Clusters of eight CTAs of 32 points, phi staged in FP64, ran
// 111 ms per (H2O)64 build against 97.)  Planes s >= nspin (a J build's
// separate Coulomb plane) are Z = 1/2 vJ phi.  A row field of 0x7fd or more
// (values of 2^1022 and up, Inf, NaN) is reported in *nonfinite.
constexpr int kZdRanks = 4;
constexpr size_t zdigits_smem(int nz) {
  return ((size_t)nz * 8 + 4) * (kBatch / kZdRanks) * kBlockF + 8 * (kBatch / kZdRanks);
}
template <bool GRAD, int NZ>
__global__ void __cluster_dims__(kZdRanks, 1, 1) __launch_bounds__(256, 2)
    zdigits_kernel(const uint8_t *__restrict__ qphT, const double *__restrict__ sphT,
                   const int *__restrict__ pair_batch, long p0, const double *__restrict__ coef,
                   const double *__restrict__ vj, int nspin, long npad, uint8_t *__restrict__ qph,
                   double *__restrict__ sph, uint8_t *__restrict__ qz, double *__restrict__ szs, int *nonfinite) {
  constexpr int NC = GRAD ? 4 : 1, nop = 1 + NZ, kPts = kBatch / kZdRanks;
  constexpr size_t kPlane = (size_t)kBatch * kBlockF;  // one digit plane of a pair, bytes
  // dynamic shared memory: Z_s [NZ][kPts][128] FP64, then phi as packed
  // pass-A digits [kPts][128] and its point scales s_g 2^-30 [kPts]
  extern __shared__ __align__(16) double zst[];
  uint32_t(*phid)[128] = reinterpret_cast<uint32_t(*)[128]>(zst + (size_t)NZ * kPts * kBlockF);
  double *phis = reinterpret_cast<double *>(phid + kPts);
  __shared__ uint32_t red[8][nop][128];
  __shared__ uint32_t part[kZdRanks][nop][128];  // every CTA's row fields, pushed by their owners
  __shared__ double inv_s[nop][128];
  const uint32_t rank = cluster_rank();
  const long q = cluster_id_x();
  const int b = pair_batch[p0 + q];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gbase = kPts * (int)rank;
  // first half of a barrier whose wait, before the first store into another
  // CTA's shared memory, shows that every CTA of the cluster has started
  cluster_arrive_relaxed();
  const int ncs = NC;
  uint32_t e[nop][8];
#pragma unroll
  for (int o = 0; o < nop; ++o)
#pragma unroll
    for (int k = 0; k < 8; ++k) e[o][k] = 0u;
  // ---- phase 1: lanes 16 h .. 16 h + 15 of warp w take point
  // gl = 2 (w + 8 j) + h, lane l functions 8 (l % 16) .. + 7 (one 8-byte
  // load per digit plane and component)
  const int hp = lane >> 4, f8 = 8 * (lane & 15);
#pragma unroll 2
  for (int j = 0; j < kPts / 16; ++j) {
    const int gl = 2 * (warp + 8 * j) + hp, g = gbase + gl;
    const long gg = (long)b * kBatch + g;
    double z[NZ][8], t[NZ][8];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long pc = q * ncs + c;
      const double sc = sphT[pc * kBatch + g] * 0x1p-30;
      uint2 wv[4];
#pragma unroll
      for (int d = 0; d < 4; ++d)
        wv[d] = *reinterpret_cast<const uint2 *>(qphT + (pc * 4 + d) * kPlane + (size_t)g * kBlockF + f8);
      uint32_t bw[8];
      {
        const uint32_t lo[4] = {wv[3].x, wv[2].x, wv[1].x, wv[0].x}, hi[4] = {wv[3].y, wv[2].y, wv[1].y, wv[0].y};
        transpose4(lo, bw);
        transpose4(hi, bw + 4);
      }
      double v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = int_to_double(digits_value(bw[k])) * sc;
      if (c == 0) {
        uint4 *pd = reinterpret_cast<uint4 *>(&phid[gl][f8]);
        pd[0] = make_uint4(bw[0], bw[1], bw[2], bw[3]);
        pd[1] = make_uint4(bw[4], bw[5], bw[6], bw[7]);
        if ((lane & 15) == 0) phis[gl] = sc;
#pragma unroll
        for (int k = 0; k < 8; ++k) e[0][k] = max(e[0][k], exp_field(v[k]));
      }
#pragma unroll
      for (int s = 0; s < NZ; ++s) {
        const double cc = s < nspin ? coef[((size_t)s * 4 + c) * npad + gg] : (c == 0 ? 0.5 * vj[gg] : 0.0);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          // Z = c0 phi + ((c1 dx phi + c2 dy phi) + c3 dz phi)
          if (c == 0)
            z[s][k] = cc * v[k];
          else if (c == 1)
            t[s][k] = cc * v[k];
          else
            t[s][k] += cc * v[k];
        }
      }
    }
#pragma unroll
    for (int s = 0; s < NZ; ++s) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (GRAD) z[s][k] += t[s][k];
        e[1 + s][k] = max(e[1 + s][k], exp_field(z[s][k]));
      }
      double2 *dst = reinterpret_cast<double2 *>(zst + ((size_t)s * kPts + gl) * kBlockF + f8);
#pragma unroll
      for (int k = 0; k < 8; k += 2) dst[k / 2] = make_double2(z[s][k], z[s][k + 1]);
    }
  }
  unsigned ez = 0;
#pragma unroll
  for (int o = 1; o < nop; ++o)
#pragma unroll
    for (int k = 0; k < 8; ++k) ez = max(ez, e[o][k]);
  report_nonfinite(ez >= 0x7fdu, nonfinite);
  // the two points of a warp step, then the warps
#pragma unroll
  for (int o = 0; o < nop; ++o)
#pragma unroll
    for (int k = 0; k < 8; ++k) e[o][k] = max(e[o][k], __shfl_xor_sync(0xffffffffu, e[o][k], 16));
  if (hp == 0) {
#pragma unroll
    for (int o = 0; o < nop; ++o)
#pragma unroll
      for (int k = 0; k < 8; ++k) red[warp][o][f8 + k] = e[o][k];
  }
  __syncthreads();
  cluster_wait();
  // this CTA's row fields go to slot `rank` of every CTA's part[]: every
  // access to another CTA's shared memory comes before the cluster barrier
  // below, so none can meet a CTA that has finished
  for (int t = threadIdx.x; t < nop * 128; t += blockDim.x) {
    uint32_t m = 0u;
#pragma unroll
    for (int w = 0; w < 8; ++w) m = max(m, red[w][t / 128][t % 128]);
#pragma unroll
    for (uint32_t rr = 0; rr < kZdRanks; ++rr) st_cluster_u32(map_to_rank(&part[rank][t / 128][t % 128], rr), m);
  }
  cluster_sync();  // every CTA's row fields are in place in every CTA
  for (int t = threadIdx.x; t < nop * 128; t += blockDim.x) {
    const int o = t / 128, f = t % 128;
    uint32_t E = 0u;
#pragma unroll
    for (int rr = 0; rr < kZdRanks; ++rr) E = max(E, part[rr][o][f]);
    double sc = 1.0, inv = 1.0;  // an all-zero row keeps scale 1
    if (E > 0u && E < 0x7fdu) {
      sc = __hiloint2double((int)((E + 1u) << 20), 0);
      inv = __hiloint2double((int)((2045u - E) << 20), 0);
    }
    inv_s[o][f] = inv;
    if (rank == 0) {
      if (o == 0)
        sph[q * 128 + f] = sc;
      else
        szs[(q * NZ + (o - 1)) * 128 + f] = sc;
    }
  }
  __syncthreads();
  // ---- phase 2: thread (f, gh) writes points gbase + 32 gh .. + 31 of row f
  static_assert(kPts == 64, "two threads a row, 32 points each");
  {
    const int f = threadIdx.x & 127, gh = threadIdx.x >> 7;
#pragma unroll
    for (int o = 0; o < nop; ++o) {
      const double inv = inv_s[o][f];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t w[4][4];  // [digit plane][group of four points]
#pragma unroll
        for (int k4 = 0; k4 < 4; ++k4) {
          const int gl = 32 * gh + 16 * h + 4 * k4;
          double v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i)
            v[i] = (o == 0) ? int_to_double(digits_value(phid[gl + i][f])) * phis[gl + i]
                            : zst[((size_t)(o - 1) * kPts + gl + i) * kBlockF + f];
          uint32_t ww[4];
          quant4(v, inv, ww);
#pragma unroll
          for (int d = 0; d < 4; ++d) w[d][k4] = ww[d];
        }
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          uint8_t *row = (o == 0) ? qph + ((q * 4 + d) * 128 + f) * (size_t)kBatch
                                  : qz + (((q * NZ + (o - 1)) * 4 + d) * 128 + f) * (size_t)kBatch;
          *reinterpret_cast<uint4 *>(row + gbase + 32 * gh + 16 * h) =
              make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
        }
      }
    }
  }
}

// Pass B, part 2: digits of the V operands, transposed to
// qph[pair][digit][f][g] and qz[pair][z][digit][f][g] through a shared
// tile in slabs of 32 points (rows padded to 36 bytes: conflict-free; 37 KB
// for one Z plane, so four blocks share an SM).
__global__ void __launch_bounds__(256) zquant_kernel(const double *__restrict__ ws, const double *__restrict__ sph,
                                                     const double *__restrict__ szs, int nz, uint8_t *__restrict__ qph,
                                                     uint8_t *__restrict__ qz) {
  extern __shared__ __align__(16) uint8_t tile[];  // [(1 + nz)][4][128][36]
  const long q = blockIdx.x;
  const size_t T = (size_t)kBatch * kBlockF;
  const int f = threadIdx.x & 127, gs = threadIdx.x >> 7;
  const int nop = 1 + nz;
  double inv[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    if (o >= nop) break;
    const double s = (o == 0) ? sph[q * 128 + f] : szs[(q * nz + (o - 1)) * 128 + f];
    inv[o] = 1.0 / s;  // exact: s is a power of two
  }
  const double *src = ws + q * 4 * T;
  for (int g0 = 0; g0 < kBatch; g0 += 32) {
    // thread (f, gs) quantises points 4 gq .. 4 gq + 3 of the slab, gq = gs + 2 kq:
    // all loads of a step are issued before use, and the four digit bytes of
    // four consecutive points go to shared memory as one word
    for (int kq = 0; kq < 4; ++kq) {
      const int gq = gs + 2 * kq;
      double v[4][4];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if (o >= nop) break;
#pragma unroll
        for (int r = 0; r < 4; ++r) v[o][r] = src[o * T + (size_t)(g0 + 4 * gq + r) * kBlockF + f];
      }
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if (o >= nop) break;
        uint32_t w[4];
        quant4(v[o], inv[o], w);
        uint32_t *t = reinterpret_cast<uint32_t *>(tile + ((size_t)o * 4 * 128 + f) * 36) + gq;
#pragma unroll
        for (int dd = 0; dd < 4; ++dd) t[dd * 128 * 9] = w[dd];
      }
    }
    __syncthreads();
    const int nrow = nop * 4 * 128;
    for (int e = threadIdx.x; e < nrow * 8; e += 256) {
      const int rw = e >> 3, part = e & 7;
      const int o = rw / 512, d = (rw / 128) & 3, ff = rw & 127;
      const uint32_t val = *reinterpret_cast<const uint32_t *>(tile + (size_t)rw * 36 + 4 * part);
      uint8_t *dst = (o == 0) ? qph + ((q * 4 + d) * 128 + ff) * 256
                              : qz + (((q * nz + (o - 1)) * 4 + d) * 128 + ff) * 256;
      *reinterpret_cast<uint32_t *>(dst + g0 + 4 * part) = val;
    }
    __syncthreads();
  }
}

// rho(g) = sum_i occ_i T0(g,i)^2, grad rho = 2 sum_i occ_i T0 Tc from the
// FP64 products T[bl][s][c][i][g] (density.hpp:188-255).
template <bool GRAD>
__global__ void density_contract_kernel(const double *__restrict__ T, const double *__restrict__ occ, int nocc,
                                        int nocc_pad, int nspin, long b0, double *__restrict__ rho,
                                        double *__restrict__ grad, long npad) {
  constexpr int NC = GRAD ? 4 : 1;
  const long bl = blockIdx.x;
  const int s = blockIdx.y, g = threadIdx.x;
  const size_t plane = (size_t)nocc_pad * 256;
  const double *Tp = T + ((bl * nspin + s) * NC) * plane + g;
  double r = 0, gx = 0, gy = 0, gz = 0;
  for (int i = 0; i < nocc; ++i) {
    const double o = occ[(size_t)s * nocc + i];
    const double t = Tp[(size_t)i * 256];
    r += o * t * t;
    if (GRAD) {
      gx += o * t * Tp[plane + (size_t)i * 256];
      gy += o * t * Tp[2 * plane + (size_t)i * 256];
      gz += o * t * Tp[3 * plane + (size_t)i * 256];
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

// ------------------------------------------------------------- host ----

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    NKX_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr));
    NKX_REQUIRE(p && qr == cudaDriverEntryPointSuccess, NKX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 3-D byte tensor [planes][rows][cols] (cols contiguous), box
// {64 bytes, box_rows, 4 planes}, 64-byte swizzle.
static CUtensorMap make_map3(const uint8_t *base, long cols, long rows, long planes, int box_rows) {
  NKX_REQUIRE(cols % 64 == 0 && rows % box_rows == 0 && planes % 4 == 0 && ((uintptr_t)base % 16) == 0,
              NKX_ERR_ARG, "bad tensor map shape");
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)cols, (cuuint64_t)cols * rows};
  const cuuint32_t box[3] = {64, (cuuint32_t)box_rows, 4};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t *>(base), dims, strides,
                                 box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  NKX_REQUIRE(r == CUDA_SUCCESS, NKX_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

struct MixedState {
  long cap = 0;  // pairs per chunk
  int nocc_pad = 0, nbatch_chunk = 0, nsm = 148;
  uint8_t *qphT = nullptr, *qph = nullptr, *qz = nullptr, *qct = nullptr;
  double *sphT = nullptr, *sph = nullptr, *sz = nullptr, *sct = nullptr, *T = nullptr;
  // grad mode: T0 and (C occ) digits with their row scales
  uint8_t *qt0 = nullptr, *qco = nullptr;
  double *st0 = nullptr, *sco = nullptr;
  // B operand maps by box width: Z with 128- and 64-row boxes (V at N = 128 / 64),
  // Ct with 64- and 128-row boxes (density at N = 64 / 128); Z with 32-row
  // boxes for the CTA-pair V contraction (each CTA's half of 64 columns)
  CUtensorMap m_phT, m_ph, m_z, m_z64, m_z32, m_ct, m_ct128, m_t0, m_co, m_co128;
  int pair_clusters = 0;  // CTA pairs of the V contraction that fit on the device at once
  std::vector<void *> bufs;
  size_t T_cap = 0, qt0_cap = 0;  // doubles of T, bytes of qt0 (grown on demand)
  ~MixedState() {
    for (void *p : bufs) cudaFree(p);
    cudaFree(T);
    cudaFree(qt0);
    cudaFree(X);
    cudaFree(qphT_res);
    cudaFree(sphT_res);
  }
  // J builds: every chunk's pass-A digits and scales, kept until pass B when
  // they fit in half of the free device memory (qphT / sphT / m_phT then
  // address the current chunk's slice of them; the chunk buffers are
  // restored after the build)
  uint8_t *qphT_res = nullptr, *qphT_chunk = nullptr;
  double *sphT_res = nullptr, *sphT_chunk = nullptr;
  CUtensorMap m_phT_chunk;
  long res_pairs = 0;
  bool ensure_resident(long npairs) {
    const size_t tile = (size_t)kBatch * kBlockF;
    if (qphT_res && res_pairs >= npairs) return true;
    cudaFree(qphT_res);
    cudaFree(sphT_res);
    qphT_res = nullptr;
    sphT_res = nullptr;
    res_pairs = 0;
    const size_t bytes = (size_t)npairs * 4 * 4 * tile, sbytes = (size_t)npairs * 4 * 256 * sizeof(double);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess || bytes + sbytes > fr / 2) {
      cudaGetLastError();
      return false;
    }
    if (cudaMalloc(&qphT_res, bytes) != cudaSuccess || cudaMalloc(&sphT_res, sbytes) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(qphT_res);
      cudaFree(sphT_res);
      qphT_res = nullptr;
      sphT_res = nullptr;
      return false;
    }
    res_pairs = npairs;
    return true;
  }
  void use_resident_slice(const Chunk &c) {
    const size_t tile = (size_t)kBatch * kBlockF;
    qphT = qphT_res + (size_t)c.p0 * 4 * 4 * tile;
    sphT = sphT_res + (size_t)c.p0 * 4 * 256;
    m_phT = make_map3(qphT, 128, 256, std::max<long>(1, c.p1 - c.p0) * 4 * 4, 128);
  }
  void use_chunk_buffers() {
    qphT = qphT_chunk;
    sphT = sphT_chunk;
    m_phT = m_phT_chunk;
  }
  double *X = nullptr;  // the mixed gradient's X[pair][spin][comp][g][mu]
  size_t X_cap = 0;
  void ensure_X(size_t doubles) {
    if (doubles <= X_cap) return;
    cudaFree(X);
    X = nullptr;
    X_cap = 0;
    if (cudaMalloc(&X, doubles * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      throw Error{NKX_ERR_ALLOC, "gradient X allocation of " + std::to_string(doubles * 8) + " bytes failed"};
    }
    X_cap = doubles;
  }
  // T: the chunk's FP64 density tiles, nbatch x nspin x ncomp planes of
  // nocc_pad x 256 (one component on the Y path); qt0: their T0 digits
  void ensure_T(size_t doubles) {
    if (doubles <= T_cap) return;
    cudaFree(T);
    T = nullptr;
    T_cap = 0;
    if (cudaMalloc(&T, doubles * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      throw Error{NKX_ERR_ALLOC, "density tile allocation of " + std::to_string(doubles * 8) + " bytes failed"};
    }
    T_cap = doubles;
  }
  void ensure_qt0(size_t bytes, long rows_planes, int nocc_pad_) {
    if (bytes <= qt0_cap) return;
    cudaFree(qt0);
    qt0 = nullptr;
    qt0_cap = 0;
    if (cudaMalloc(&qt0, bytes) != cudaSuccess) {
      cudaGetLastError();
      throw Error{NKX_ERR_ALLOC, "T0 digit allocation of " + std::to_string(bytes) + " bytes failed"};
    }
    qt0_cap = bytes;
    m_t0 = make_map3(qt0, nocc_pad_, 128, rows_planes, 128);
  }
  template <class X>
  X *alloc(size_t n) {
    X *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(X)) != cudaSuccess) {
      cudaGetLastError();
      throw Error{NKX_ERR_ALLOC, "mixed workspace allocation of " + std::to_string(n * sizeof(X)) + " bytes failed"};
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

static MixedState &mixed_state(Plan &P, int nocc) {
  if (!P.mx_state) {
    MixedState *M = new MixedState();
    P.mx_state = M;
    M->cap = std::max<long>(1, P.max_chunk_pairs);
    long nb = 1;
    for (const Chunk &c : P.chunks) nb = std::max(nb, c.b1 - c.b0);
    M->nbatch_chunk = (int)nb;
    const size_t tile = (size_t)kBatch * kBlockF;
    M->qphT = M->alloc<uint8_t>(M->cap * 4 * 4 * tile);
    M->sphT = M->alloc<double>(M->cap * 4 * 256);
    M->qph = M->alloc<uint8_t>(M->cap * 4 * tile);
    M->sph = M->alloc<double>(M->cap * 128);
    M->qz = M->alloc<uint8_t>(M->cap * 3 * 4 * tile);
    M->sz = M->alloc<double>(M->cap * 3 * 128);
    M->m_phT = make_map3(M->qphT, 128, 256, M->cap * 4 * 4, 128);
    M->qphT_chunk = M->qphT;
    M->sphT_chunk = M->sphT;
    M->m_phT_chunk = M->m_phT;
    M->m_ph = make_map3(M->qph, 256, 128, M->cap * 4, 128);
    M->m_z = make_map3(M->qz, 256, 128, M->cap * 3 * 4, 128);
    M->m_z64 = make_map3(M->qz, 256, 128, M->cap * 3 * 4, 64);
    M->m_z32 = make_map3(M->qz, 256, 128, M->cap * 3 * 4, 32);
    int dev = 0;
    NKX_CUDA(cudaGetDevice(&dev));
    NKX_CUDA(cudaDeviceGetAttribute(&M->nsm, cudaDevAttrMultiProcessorCount, dev));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_V, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<128>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_v_pair_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_v_pair_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairSmem));
    {
      // clusters of two that are resident at once (the persistent grid)
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(2 * M->nsm);
      cfg.blockDim = dim3(64 + 32 * 8);
      cfg.dynamicSmemBytes = kPairSmem;
      int ncl = 0;
      NKX_CUDA(cudaOccupancyMaxActiveClusters(&ncl, tc_v_pair_kernel<8>, &cfg));
      M->pair_clusters = std::max(1, ncl);
    }
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_V, 128, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<128, 8>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_V, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<64>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_DENSITY, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<64>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_DENSITY, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<128>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_GRAD, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<64>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_X, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<64>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(tc_i8_kernel<TC_MODE_GRAD, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TcShape<128>::kSmem));
    NKX_CUDA(cudaFuncSetAttribute(zquant_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * 4 * 128 * 36));
    NKX_CUDA(cudaFuncSetAttribute(zdigits_kernel<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zdigits_smem(1)));
    NKX_CUDA(cudaFuncSetAttribute(zdigits_kernel<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zdigits_smem(2)));
    NKX_CUDA(cudaFuncSetAttribute(zdigits_kernel<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zdigits_smem(1)));
    NKX_CUDA(cudaFuncSetAttribute(zdigits_kernel<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zdigits_smem(2)));
  }
  MixedState &M = *static_cast<MixedState *>(P.mx_state);
  // orbitals pad to 128 so that either density tile width divides them
  const int nocc_pad = ((nocc + 127) / 128) * 128;
  if (nocc_pad > M.nocc_pad) {
    M.nocc_pad = nocc_pad;
    M.qct = M.alloc<uint8_t>((size_t)2 * 4 * nocc_pad * P.nbf_pad);
    M.sct = M.alloc<double>((size_t)2 * nocc_pad * P.nblk);
    M.T_cap = M.qt0_cap = 0;  // regrown for the new orbital padding
    M.m_ct = make_map3(M.qct, P.nbf_pad, nocc_pad, 8, 64);
    M.m_ct128 = make_map3(M.qct, P.nbf_pad, nocc_pad, 8, 128);
    M.st0 = M.alloc<double>((size_t)M.nbatch_chunk * 2 * 4 * 2 * 128);  // up to 2 spins x 4 comps x 2 halves
    M.qco = M.alloc<uint8_t>((size_t)2 * 4 * P.nbf_pad * nocc_pad);
    M.sco = M.alloc<double>((size_t)2 * P.nbf_pad);
    M.m_co = make_map3(M.qco, nocc_pad, P.nbf_pad, 2 * 4, 64);
    M.m_co128 = make_map3(M.qco, nocc_pad, P.nbf_pad, 2 * 4, 128);
  }
  return M;
}

template <int MODE, int NW, int EW = NW / 8>
static void launch_i8_shape(const CUtensorMap &mA, const CUtensorMap &mB, const TcArgs &a, unsigned grid,
                            cudaStream_t s) {
  tc_i8_kernel<MODE, NW, EW><<<grid, TcShape<NW, EW>::kThreads, TcShape<NW, EW>::kSmem, s>>>(mA, mB, a);
}

// The CTA-pair V contraction: one persistent cluster of two per pair of
// SMs that fits at once (or per unit when there are fewer).
static void launch_v_pair(MixedState &M, const TcArgs &a, int ew, cudaStream_t s) {
  if (a.nunits <= 0) return;
  const unsigned grid = 2u * (unsigned)std::min<long>(a.nunits, M.pair_clusters);
  NKX_REQUIRE(ew == 8 || ew == 16, NKX_ERR_ARG, "CTA-pair V epilogue warps must be 8 or 16");
  if (ew == 8)
    tc_v_pair_kernel<8><<<grid, 64 + 32 * 8, kPairSmem, s>>>(M.m_ph, M.m_z32, a);
  else
    tc_v_pair_kernel<16><<<grid, 64 + 32 * 16, kPairSmem, s>>>(M.m_ph, M.m_z32, a);
  NKX_LAUNCH_CHECK();
}

// one persistent CTA per SM (or per unit when there are fewer)
static void launch_i8(MixedState &M, const CUtensorMap &mA, const CUtensorMap &mB, const TcArgs &a, cudaStream_t s) {
  if (a.nunits <= 0) return;
  const unsigned grid = (unsigned)std::min<long>(a.nunits, M.nsm);
  NKX_REQUIRE(a.nt == 64 || a.nt == 128, NKX_ERR_ARG, "tensor-core width must be 64 or 128");
  NKX_REQUIRE(a.mode != TC_MODE_X || a.nt == 64, NKX_ERR_ARG, "the X pass runs N = 64");
  NKX_REQUIRE(a.ew == a.nt / 8 || (a.mode == TC_MODE_V && a.nt == 128 && a.ew == 8), NKX_ERR_ARG,
              "epilogue warps: N / 8, or 8 for the N = 128 V contraction");
  if (a.mode == TC_MODE_V) {
    if (a.nt == 64)
      launch_i8_shape<TC_MODE_V, 64>(mA, mB, a, grid, s);
    else if (a.ew == 8)
      launch_i8_shape<TC_MODE_V, 128, 8>(mA, mB, a, grid, s);
    else
      launch_i8_shape<TC_MODE_V, 128>(mA, mB, a, grid, s);
  }
  else if (a.mode == TC_MODE_GRAD)
    a.nt == 128 ? launch_i8_shape<TC_MODE_GRAD, 128>(mA, mB, a, grid, s)
                : launch_i8_shape<TC_MODE_GRAD, 64>(mA, mB, a, grid, s);
  else if (a.mode == TC_MODE_X)
    launch_i8_shape<TC_MODE_X, 64>(mA, mB, a, grid, s);
  else
    a.nt == 128 ? launch_i8_shape<TC_MODE_DENSITY, 128>(mA, mB, a, grid, s)
                : launch_i8_shape<TC_MODE_DENSITY, 64>(mA, mB, a, grid, s);
  NKX_LAUNCH_CHECK();
}


template <bool GRAD>
static void launch_colloc_z_g(Plan &P, MixedState &M, const Chunk &c, int nzs, int nspin, cudaStream_t s) {
  const unsigned np = (unsigned)(c.p1 - c.p0);
#define NKX_CZ(NZ)                                                                                                   \
  colloc_z_kernel<GRAD, NZ><<<np, 256, 0, s>>>(P.d_sto, P.d_fshell, P.d_bshell, P.d_bnshell, P.d_px, P.d_py, P.d_pz, P.d_pair_batch, P.d_pair_blk, c.p0, \
                                               P.d_coef, P.d_vj, nspin, P.npad, P.ws_phi, M.sph, M.sz, P.d_status + 1)
  if (nzs == 1)
    NKX_CZ(1);
  else if (nzs == 2)
    NKX_CZ(2);
  else
    NKX_CZ(3);
#undef NKX_CZ
}

static void launch_colloc_z(Plan &P, MixedState &M, const Chunk &c, int nzs, int nspin, cudaStream_t s) {
  if (P.gga)
    launch_colloc_z_g<true>(P, M, c, nzs, nspin, s);
  else
    launch_colloc_z_g<false>(P, M, c, nzs, nspin, s);
}

// The mixed-precision XC gradient's per-build set-up: the orbital digits.
void mixed_gradient_begin(Plan &P, int nspin, int nocc, cudaStream_t s) {
  MixedState &M = mixed_state(P, nocc);
  const int nc = P.gga ? 4 : 1;
  M.ensure_T((size_t)M.nbatch_chunk * nspin * nc * M.nocc_pad * 256);
  M.ensure_qt0((size_t)M.nbatch_chunk * nspin * nc * 2 * 4 * 128 * M.nocc_pad,
               (long)M.nbatch_chunk * nspin * nc * 2 * 4, M.nocc_pad);
  M.ensure_X((size_t)M.cap * nspin * nc * kBatch * kBlockF);
  const long rows = (long)nspin * M.nocc_pad * P.nblk;
  quant_ct_kernel<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, s>>>(P.d_Ct, nocc, M.nocc_pad, nspin, P.nbf_pad,
                                                                       P.nblk, M.qct, M.sct, P.d_status + 1);
  NKX_LAUNCH_CHECK();
  quant_cocc_kernel<<<dim3((unsigned)P.nblk, nspin), 128, 0, s>>>(P.d_Ct, P.d_occ, nocc, M.nocc_pad, P.nbf_pad,
                                                                  M.qco, M.sco);
  NKX_LAUNCH_CHECK();
  P.launches += 2;
}

// One chunk of the mixed-precision XC gradient: pass-A digits of the chunk's
// pairs, the orbital values T_c(g, i) = sum_f Phi_c(g, f) C(f, i) for the
// value and (GGA) the three gradient components on the tensor cores (the
// density contraction with all components), rho and grad rho of the chunk's
// points from them, and the functional there (Z coefficients, energy, energy
// density edens).  Returns T[(bl, s, c)][i][g] (bl from the chunk's first
// batch, i padded to *nocc_pad), resident until the next chunk.
const double *mixed_gradient_chunk(Plan &P, const Chunk &c, int nspin, int nocc, double *edens, cudaStream_t s,
                                   int *nocc_pad, const double **X) {
  MixedState &M = mixed_state(P, nocc);
  const int nc = P.gga ? 4 : 1;
  const long np = c.p1 - c.p0, nb = c.b1 - c.b0;
  if (np > 0) {
    if (P.gga)
      colloc_quantT_kernel<true><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_fshell, P.d_bshell, P.d_bnshell, P.d_px,
                                                              P.d_py, P.d_pz, P.d_pair_batch, P.d_pair_blk, c.p0,
                                                              M.qphT, M.sphT, P.d_status + 1);
    else
      colloc_quantT_kernel<false><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_fshell, P.d_bshell, P.d_bnshell, P.d_px,
                                                               P.d_py, P.d_pz, P.d_pair_batch, P.d_pair_blk, c.p0,
                                                               M.qphT, M.sphT, P.d_status + 1);
    NKX_LAUNCH_CHECK();
    ++P.launches;
  }
  TcArgs a{};
  a.mode = TC_MODE_DENSITY;
  a.b0 = c.b0;
  a.b1 = c.b1;
  a.p0 = c.p0;
  a.pair_off = P.d_pair_off;
  a.pair_blk = P.d_pair_blk;
  a.mask = P.d_mask;
  a.mask_words = P.mask_words;
  a.nblk = P.nblk;
  a.sA = M.sphT;
  a.sB = M.sct;
  a.nspin = nspin;
  a.ncs = nc;
  a.ncomp = nc;
  a.nt = density_width(P, nocc);
  a.ew = a.nt / 8;
  a.ntile_i = (nocc + a.nt - 1) / a.nt;
  a.nocc_pad = M.nocc_pad;
  a.T = M.T;
  a.err = P.d_status;
  a.wait_ns = P.wait_ns;
  a.stall = P.stall_test;
  a.nunits = nb * nspin * 2 * a.ncomp * a.ntile_i;
  launch_i8(M, M.m_phT, a.nt == 128 ? M.m_ct128 : M.m_ct, a, s);
  ++P.launches;
  if (P.gga)
    density_contract_kernel<true><<<dim3((unsigned)nb, nspin), 256, 0, s>>>(M.T, P.d_occ, nocc, M.nocc_pad, nspin,
                                                                            c.b0, P.d_rho, P.d_grad, P.npad);
  else
    density_contract_kernel<false><<<dim3((unsigned)nb, nspin), 256, 0, s>>>(M.T, P.d_occ, nocc, M.nocc_pad, nspin,
                                                                             c.b0, P.d_rho, P.d_grad, P.npad);
  NKX_LAUNCH_CHECK();
  ++P.launches;
  const long g0 = c.b0 * kBatch, n = nb * kBatch;
  functional_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P.xc, P.gga, nspin, P.npad, n, P.d_w + g0,
                                                                P.d_rho + g0, P.d_grad + g0, nullptr, P.d_coef + g0,
                                                                P.d_E, edens + g0);
  NKX_LAUNCH_CHECK();
  ++P.launches;
  // X_c(g, mu) = sum_i T_c(g, i) occ_i C(mu, i) of every pair on the tensor
  // cores: T_c as digit rows over the orbitals, then the Y-pass contraction
  // with all components, written in FP64
  if (np > 0) {
    quant_t0_kernel<<<(unsigned)(nb * nspin * nc * 2), 128, 0, s>>>(M.T, nocc, M.nocc_pad, M.qt0, M.st0);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    TcArgs x{};
    x.mode = TC_MODE_X;
    x.b0 = c.b0;
    x.b1 = c.b1;
    x.p0 = c.p0;
    x.pair_blk = P.d_pair_blk;
    x.pair_batch = P.d_pair_batch;
    x.nblk = P.nblk;
    x.nbf_pad = P.nbf_pad;
    x.sA = M.st0;
    x.sB = M.sco;
    x.nspin = nspin;
    x.ncs = nc;
    x.ncomp = nc;
    x.nocc_pad = M.nocc_pad;
    x.X = M.X;
    x.err = P.d_status;
    x.wait_ns = P.wait_ns;
    x.stall = P.stall_test;
    x.nunits = np * nspin * nc * 4;
    x.nt = 64;
    x.ew = 8;
    launch_i8(M, M.m_t0, M.m_co, x, s);
    ++P.launches;
  }
  *nocc_pad = M.nocc_pad;
  *X = M.X;
  return M.T;
}

void fock_build_mixed(Plan &P, int nspin, int nocc, bool needJ, bool fuse, bool separateJ, cudaStream_t s,
                      StageTimer &Tm, int phase) {
  MixedState &M = mixed_state(P, nocc);
  const int nc = P.gga ? 4 : 1;
  const int nzs = nspin + (separateJ ? 1 : 0);
  NKX_REQUIRE(nzs <= 3, NKX_ERR_ARG, "too many Z planes");
  NKX_REQUIRE(phase == 0 || needJ, NKX_ERR_ARG, "a sharded (two-phase) build needs J");
  // Y path for the GGA density gradient (see below): the plan's tuning, or
  // by default from 256 orbitals on
  const bool y_ok = P.gga && M.nocc_pad <= 8192;
  const bool grad_mode = y_ok && (P.tune.ypath >= 0 ? P.tune.ypath != 0 : M.nocc_pad >= 256);
  if (phase != 2) {
    M.ensure_T((size_t)M.nbatch_chunk * nspin * (grad_mode ? 1 : nc) * M.nocc_pad * 256);
    if (grad_mode)
      M.ensure_qt0((size_t)M.nbatch_chunk * nspin * 2 * 4 * 128 * M.nocc_pad, (long)M.nbatch_chunk * nspin * 2 * 4,
                   M.nocc_pad);
  }
  if (phase != 2) {
    const long rows = (long)nspin * M.nocc_pad * P.nblk;
    quant_ct_kernel<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, s>>>(P.d_Ct, nocc, M.nocc_pad, nspin, P.nbf_pad,
                                                                         P.nblk, M.qct, M.sct, P.d_status + 1);
    NKX_LAUNCH_CHECK();
    ++P.launches;
  }
  // GGA density gradient through Y = T0 (C occ)^T: grad rho = 2 sum_mu
  // grad phi_mu Y_mu needs one orbital contraction (T0) and one more over
  // the orbitals (Y) instead of the three gradient components of T.  It pays
  // from about 256 orbitals on ((H2O)64, 320 orbitals: 226 vs 232 ms; the
  // 1500-atom aggregate, 2850: 12.2 vs 24.8 s); with fewer the per-pair Y
  // traffic dominates.  Above 8192 orbitals the int32 levels could overflow.
  if (grad_mode && phase != 2) {
    quant_cocc_kernel<<<dim3((unsigned)P.nblk, nspin), 128, 0, s>>>(P.d_Ct, P.d_occ, nocc, M.nocc_pad, P.nbf_pad,
                                                                    M.qco, M.sco);
    NKX_LAUNCH_CHECK();
    ++P.launches;
  }
  // pass A of one chunk: collocation -> digits, int8 density contraction,
  // FP64 rho / grad rho of the chunk's batches
  auto pass_a = [&](const Chunk &c) {
    const long np = c.p1 - c.p0, nb = c.b1 - c.b0;
    if (np > 0) {
      Tm.begin(ST_COLLOC, s);
      if (P.gga)
        colloc_quantT_kernel<true><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_fshell, P.d_bshell, P.d_bnshell, P.d_px, P.d_py, P.d_pz, P.d_pair_batch,
                                                                P.d_pair_blk, c.p0, M.qphT, M.sphT, P.d_status + 1);
      else
        colloc_quantT_kernel<false><<<(unsigned)np, 256, 0, s>>>(P.d_sto, P.d_fshell, P.d_bshell, P.d_bnshell, P.d_px, P.d_py, P.d_pz, P.d_pair_batch,
                                                                 P.d_pair_blk, c.p0, M.qphT, M.sphT, P.d_status + 1);
      NKX_LAUNCH_CHECK();
      ++P.launches;
      Tm.end(s);
    }
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
    a.nblk = P.nblk;
    a.sA = M.sphT;
    a.sB = M.sct;
    a.nspin = nspin;
    a.ncs = nc;
    a.ncomp = grad_mode ? 1 : nc;
    a.nt = density_width(P, nocc);
    a.ew = a.nt / 8;
    a.ntile_i = (nocc + a.nt - 1) / a.nt;
    a.nocc_pad = M.nocc_pad;
    a.T = M.T;
    a.err = P.d_status;
    a.wait_ns = P.wait_ns;
    a.stall = P.stall_test;
    a.nunits = nb * nspin * 2 * a.ncomp * a.ntile_i;
    launch_i8(M, M.m_phT, a.nt == 128 ? M.m_ct128 : M.m_ct, a, s);
    ++P.launches;
    if (P.gga && !grad_mode)
      density_contract_kernel<true><<<dim3((unsigned)nb, nspin), 256, 0, s>>>(M.T, P.d_occ, nocc, M.nocc_pad, nspin,
                                                                              c.b0, P.d_rho, P.d_grad, P.npad);
    else
      density_contract_kernel<false><<<dim3((unsigned)nb, nspin), 256, 0, s>>>(M.T, P.d_occ, nocc, M.nocc_pad, nspin,
                                                                               c.b0, P.d_rho, P.d_grad, P.npad);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    if (grad_mode && np > 0) {
      quant_t0_kernel<<<(unsigned)(nb * nspin * 2), 128, 0, s>>>(M.T, nocc, M.nocc_pad, M.qt0, M.st0);
      NKX_LAUNCH_CHECK();
      ++P.launches;
      TcArgs g{};
      g.mode = TC_MODE_GRAD;
      g.b0 = c.b0;
      g.b1 = c.b1;
      g.p0 = c.p0;
      g.pair_blk = P.d_pair_blk;
      g.pair_batch = P.d_pair_batch;
      g.nblk = P.nblk;
      g.nbf_pad = P.nbf_pad;
      g.sA = M.st0;
      g.sB = M.sco;
      g.nspin = nspin;
      g.ncs = nc;
      g.nocc_pad = M.nocc_pad;
      g.qphT = M.qphT;
      g.sphT = M.sphT;
      g.Gp = P.ws_phi;  // free during pass A: the FP64 staging of pass B
      g.err = P.d_status;
      g.wait_ns = P.wait_ns;
      g.stall = P.stall_test;
      // the density contractions' MMA width: N = 128 covers a whole block
      // per unit (shared-memory operand traffic per MMA halved), N = 64 a
      // half with two TMEM buffers (read-back overlapped; better for short
      // orbital runs)
      g.nt = density_width(P, nocc);
      g.ew = g.nt / 8;
      g.nunits = np * nspin * 2 * (128 / g.nt);
      launch_i8(M, M.m_t0, g.nt == 128 ? M.m_co128 : M.m_co, g, s);
      ++P.launches;
      ygrad_sum_kernel<<<dim3((unsigned)nb, nspin), 256, 0, s>>>(P.ws_phi, P.d_pair_off, c.b0, c.p0, nspin, P.npad,
                                                                P.d_grad);
      NKX_LAUNCH_CHECK();
      ++P.launches;
    }
    Tm.end(s);
  };
  // pass B of one chunk: the digits of the V operands from their FP64
  // staging (quantise; the streamed build writes them directly), int8 V
  auto pass_b = [&](const Chunk &c, bool quantise) {
    const long np = c.p1 - c.p0;
    if (quantise) {
      Tm.begin(ST_ZBUILD, s);
      zquant_kernel<<<(unsigned)np, 256, (size_t)(1 + nzs) * 4 * 128 * 36, s>>>(P.ws_phi, M.sph, M.sz, nzs, M.qph,
                                                                                M.qz);
      NKX_LAUNCH_CHECK();
      ++P.launches;
      Tm.end(s);
    }
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
    a.sA = M.sph;
    a.sB = M.sz;
    a.V = P.d_V;
    a.err = P.d_status;
    a.wait_ns = P.wait_ns;
    a.stall = P.stall_test;
    // the chunk's nonempty output tiles, heaviest first; too few units for
    // the SMs: split the chunk's batches
    if (P.tune.v_pair) {
      // pair tiles (row blocks 2R, 2R + 1; column block J) in two column
      // halves; too few units for the CTA pairs: split the chunk's batches
      a.vtiles = P.d_vtiles2 + c.u0;
      a.ntiles = c.u1 - c.u0;
      a.nt = 64;
      const long parts = (long)nzs * a.ntiles * 2;
      a.nsplit = (parts == 0 || parts >= M.pair_clusters)
                     ? 1
                     : (int)std::min<long>({(M.pair_clusters + parts - 1) / parts, c.b1 - c.b0, 16L});
      a.nsplit = std::max(1, a.nsplit);
      a.nunits = parts * a.nsplit;
      launch_v_pair(M, a, P.tune.v_warps, s);
      ++P.launches;
      Tm.end(s);
      return;
    }
    a.vtiles = P.d_vtiles + c.t0;
    a.ntiles = c.t1 - c.t0;
    const long tiles = (long)nzs * a.ntiles;
    a.nt = P.tune.v_n;
    a.ew = a.nt == 128 ? P.tune.v_warps : 8;
    const long parts = tiles * (kBlockF / a.nt);
    a.nsplit = (parts == 0 || parts >= M.nsm) ? 1 : (int)std::min<long>({(M.nsm + parts - 1) / parts, c.b1 - c.b0, 16L});
    a.nsplit = std::max(1, a.nsplit);
    a.nunits = parts * a.nsplit;
    launch_i8(M, M.m_ph, a.nt == 128 ? M.m_z : M.m_z64, a, s);
    ++P.launches;
    Tm.end(s);
  };
  // the V operands' digits of one chunk straight from its pass-A digits
  // (one cluster of four CTAs per pair); nzs <= 2
  auto launch_zdigits = [&](const Chunk &c) {
    const long np = c.p1 - c.p0;
#define NKX_ZD(G, NZ)                                                                                            \
  zdigits_kernel<G, NZ><<<(unsigned)np * kZdRanks, 256, zdigits_smem(NZ), s>>>(                               \
      M.qphT, M.sphT, P.d_pair_batch, c.p0, P.d_coef, P.d_vj, nspin, P.npad, M.qph, M.sph, M.qz, M.sz,         \
      P.d_status + 1)
    if (P.gga) {
      if (nzs == 1)
        NKX_ZD(true, 1);
      else
        NKX_ZD(true, 2);
    } else {
      if (nzs == 1)
        NKX_ZD(false, 1);
      else
        NKX_ZD(false, 2);
    }
#undef NKX_ZD
    NKX_LAUNCH_CHECK();
    ++P.launches;
  };
  NKX_CUDA(cudaMemsetAsync(P.d_E, 0, sizeof(double), s));
  NKX_CUDA(cudaMemsetAsync(P.d_V, 0, sizeof(double) * nzs * P.nbf_pad * P.nbf_pad, s));
  if (!needJ) {
    // Without J every point's functional needs only its own batch, so each
    // chunk goes through both passes while its pass-A digits are resident,
    // and pass B recovers Phi and grad Phi from them instead of evaluating
    // the STOs again.
    for (const Chunk &c : P.chunks) {
      pass_a(c);
      const long g0 = c.b0 * kBatch, n = (c.b1 - c.b0) * kBatch;
      Tm.begin(ST_FUNC, s);
      functional_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P.xc, P.gga, nspin, P.npad, n, P.d_w + g0,
                                                                    P.d_rho + g0, P.d_grad + g0, nullptr,
                                                                    P.d_coef + g0, P.d_E, nullptr);
      NKX_LAUNCH_CHECK();
      ++P.launches;
      Tm.end(s);
      const long np = c.p1 - c.p0;
      if (np <= 0) continue;
      Tm.begin(ST_ZBUILD, s);
      // the V operands' digits straight from the pass-A digits (one cluster
      // of four CTAs per pair)
      launch_zdigits(c);
      Tm.end(s);
      pass_b(c, false);
    }
  } else {
    // J needs every point's density before any Z.  When every chunk's pass-A
    // digits fit in half of the free device memory (at (H2O)32, 47 GB) they
    // stay there until pass B, which takes Phi and grad Phi back from them
    // (zdigits_kernel); otherwise pass B evaluates the STOs again
    // (colloc_z_kernel) and quantises their FP64 staging.  Only whole builds
    // (a two-phase build may run other builds between its phases).
    const bool resident = phase == 0 && nzs <= 2 && M.ensure_resident(P.npairs);
    struct Restore {
      MixedState &M;
      ~Restore() { M.use_chunk_buffers(); }
    } restore{M};
    if (phase != 2) {
      for (const Chunk &c : P.chunks) {
        if (resident) M.use_resident_slice(c);
        pass_a(c);
      }
      // this plan's share of the J fit vector
      Tm.begin(ST_COULOMB, s);
      coulomb_y(P, nspin, s, true);
      Tm.end(s);
      if (phase == 1) return;
    }
    // ---- J fit and the functional, in FP64
    Tm.begin(ST_COULOMB, s);
    coulomb_solve(P, s, true);
    Tm.end(s);
    Tm.begin(ST_FUNC, s);
    functional_kernel<<<(unsigned)((P.npad + 255) / 256), 256, 0, s>>>(P.xc, P.gga, nspin, P.npad, P.npad, P.d_w,
                                                                        P.d_rho, P.d_grad, fuse ? P.d_vj : nullptr,
                                                                        P.d_coef, P.d_E, nullptr);
    NKX_LAUNCH_CHECK();
    ++P.launches;
    Tm.end(s);
    // ---- pass B: Phi and Z from the resident pass-A digits or from a second
    // collocation, digits, int8 V contraction
    for (const Chunk &c : P.chunks) {
      if (c.p1 - c.p0 <= 0) continue;
      if (resident) {
        M.use_resident_slice(c);
        Tm.begin(ST_ZBUILD, s);
        launch_zdigits(c);
        Tm.end(s);
        pass_b(c, false);
        continue;
      }
      Tm.begin(ST_COLLOC, s);
      launch_colloc_z(P, M, c, nzs, nspin, s);
      NKX_LAUNCH_CHECK();
      ++P.launches;
      Tm.end(s);
      pass_b(c, true);
    }
  }
}

void destroy_mixed_state(void *p) { delete static_cast<MixedState *>(p); }

}  // namespace nkx
