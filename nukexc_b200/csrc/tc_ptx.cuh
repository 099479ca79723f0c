// Thin inline-PTX layer for the sm_100a tensor-core kernels: mbarriers,
// TMA tile loads into the CTA's own shared memory (never multicast), tcgen05
// MMA / TMEM, on one CTA or a cluster of two (cta_group::2).  Every wait is
// bounded: after its limit of global time it raises an error flag and
// returns false, so no kernel can spin forever.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace nkx {
namespace tc {

// Default limit of the waits that can be abandoned (a plan may shorten it),
// and the fixed limit of the drain waits at the end of a kernel, which only
// wait for TMA copies and MMAs that were already issued.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;   // 2 s
constexpr unsigned long long kDrainLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.  On timeout
// (limit_ns of global time) records `code` in *err, raises *abort_flag and
// returns false; it also returns false once another thread raised the flag.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          volatile int *abort_flag, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0) {
      if (*abort_flag) return false;
      if (globaltimer() - t0 > limit_ns) {
        atomicCAS(err, 0, code);
        *abort_flag = 1;
        return false;
      }
    }
  }
}

// 3-D TMA box load (x innermost), completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---------------------------------------------------------------- TMEM --
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major tile with 64-byte swizzle (rows of 64 B, 8-row atoms of 512 B):
// LBO field 1, SBO 512 B, version 1, layout type SWIZZLE_64B (4).
__device__ __forceinline__ uint64_t smem_desc_k64(uint32_t saddr) {
  const uint64_t lo = (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16);
  const uint64_t hi = (uint64_t)(512u >> 4) | ((uint64_t)1u << 14) | ((uint64_t)4u << 29);
  return lo | (hi << 32);
}

// Instruction descriptor of kind::i8: signed int8 A and B, S32 accumulator,
// both operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// kind::i8 MMA that keeps its A operand in the tensor core's collector
// buffer: consecutive MMAs on the same A tile read shared memory once
// (CollectorFill on the first, CollectorUse in between, CollectorLastUse on
// the last); CollectorDiscard is the plain form.
enum CollectorUsage { CollectorDiscard = 0, CollectorFill = 1, CollectorUse = 2, CollectorLastUse = 3 };

template <int U>
__device__ __forceinline__ void mma_i8_a(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
#define NKX_MMA_I8(Q)                                                                                      \
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"                                          \
               "tcgen05.mma.cta_group::1.kind::i8" Q " [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem), "l"(a_desc), \
               "l"(b_desc), "r"(idesc), "r"(accumulate)                                                    \
               : "memory")
  if constexpr (U == CollectorFill)
    NKX_MMA_I8(".collector::a::fill");
  else if constexpr (U == CollectorUse)
    NKX_MMA_I8(".collector::a::use");
  else if constexpr (U == CollectorLastUse)
    NKX_MMA_I8(".collector::a::lastuse");
  else
    NKX_MMA_I8("");
#undef NKX_MMA_I8
}

// Arrive on `bar` once all previously issued MMAs of this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 lanes x 4 columns of 32-bit words from TMEM, without waiting; the
// registers are valid only after tmem_wait4 on the same array
__device__ __forceinline__ void tmem_ld4u_async(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait4(uint32_t (&r)[4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])
               :
               : "memory");
}

// waits for every TMEM load of the thread; the four arrays (one slice of the
// four accumulator levels) are valid afterwards
__device__ __forceinline__ void tmem_wait4x4(uint32_t (&a)[4], uint32_t (&b)[4], uint32_t (&c)[4], uint32_t (&d)[4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]),
                 "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3]), "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
               :
               : "memory");
}

// ------------------------------------------------------ CTA pairs --
// A cluster of two CTAs on two SMs runs one M = 256 MMA (cta_group::2): each
// CTA holds half of A (128 rows) and half of B (N / 2 rows) in its own
// shared memory at the same offsets and receives its 128 rows x N of D in
// its own TMEM.  Rank 0 issues the MMAs.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// shared::cluster address of the same shared-memory location in CTA `rank`
__device__ __forceinline__ uint32_t map_to_rank(const void *p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
// all threads of both CTAs (the non-.aligned form: callers may come from
// diverged warps)
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
// the two halves of a cluster barrier: arrive early, wait later (every
// thread, in this order)
__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ uint32_t ld_cluster_u32(uint32_t cluster_addr) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(cluster_addr) : "memory");
  return v;
}
__device__ __forceinline__ void st_cluster_u32(uint32_t cluster_addr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(cluster_addr), "r"(v) : "memory");
}
// 3-D TMA box load into this CTA's shared memory whose completion is
// counted on an mbarrier of either CTA of the pair (a shared::cluster
// address); no multicast
__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map, int x, int y, int z,
                                                 uint32_t bar_cluster_addr) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
      "%4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar_cluster_addr)
      : "memory");
}
// TMEM of a CTA pair: the same warp of both CTAs allocates (and frees) the
// same columns in both SMs
__device__ __forceinline__ void tmem_alloc_pair(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish_pair() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
// M = 256 kind::i8 MMA of the pair (collector usage as mma_i8_a)
template <int U>
__device__ __forceinline__ void mma_i8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
#define NKX_MMA_I8_PAIR(Q)                                                                                 \
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"                                          \
               "tcgen05.mma.cta_group::2.kind::i8" Q " [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem), "l"(a_desc), \
               "l"(b_desc), "r"(idesc), "r"(accumulate)                                                    \
               : "memory")
  if constexpr (U == CollectorFill)
    NKX_MMA_I8_PAIR(".collector::a::fill");
  else if constexpr (U == CollectorUse)
    NKX_MMA_I8_PAIR(".collector::a::use");
  else if constexpr (U == CollectorLastUse)
    NKX_MMA_I8_PAIR(".collector::a::lastuse");
  else
    NKX_MMA_I8_PAIR("");
#undef NKX_MMA_I8_PAIR
}
// Arrive once on the mbarrier at `bar`'s offset in every CTA of cta_mask
// when all earlier MMAs of this thread complete
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar, uint16_t cta_mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"(cta_mask)
      : "memory");
}

// 16 bytes from global memory in one read-only load (16-byte aligned address)
__device__ __forceinline__ void ldg128(const void *p, uint32_t (&r)[4]) {
  asm volatile("ld.global.nc.v4.b32 {%0, %1, %2, %3}, [%4];" : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "l"(p));
}

// 32 bytes from global memory in one read-only load (32-byte aligned address)
__device__ __forceinline__ void ldg256(const void *p, uint32_t (&r)[8]) {
  asm volatile("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "l"(p));
}

// 32 lanes x 8 columns of 32-bit words from TMEM, without waiting; the
// registers are valid only after tmem_wait8 on the same array
__device__ __forceinline__ void tmem_ld8u_async(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait8(uint32_t (&r)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
               :
               : "memory");
}

// Digits of X = rint(x * 2^30 / s) (|X| <= 2^30, s the row's power-of-two
// scale; s30 = 2^30 / s) as four balanced base-256 digits d0..d3,
// X = d0 2^24 + d1 2^16 + d2 2^8 + d3 with d1..d3 in [-128, 127] and d0 in
// [-64, 64], packed in one
// word with byte 0 = d3 .. byte 3 = d0.  The rounding is the FP64
// round-to-nearest-even of x s30 + 1.5 2^52, whose low word is X; the lower
// three bytes of Y = X + 0x808080 are the digits plus 128 and its top byte is
// d0, so the packed digits are Y ^ 0x808080.
__device__ __forceinline__ uint32_t digits_word(double x, double s30) {
  const int X = __double2loint(fma(x, s30, 0x1.8p52));
  return (uint32_t)(X + 0x00808080) ^ 0x00808080u;
}
// X back from its packed digits
__device__ __forceinline__ int digits_value(uint32_t w) { return (int)(w ^ 0x00808080u) - 0x00808080; }
// exact int32 -> FP64 through the FP64 adder: the low word of 2^52 + 2^31 + X
__device__ __forceinline__ double int_to_double(int X) {
  return __hiloint2double(0x43300000, X ^ (int)0x80000000) - 0x1.00000800000p52;
}
// 4 x 4 byte transpose: t[i] byte j = a[j] byte i
__device__ __forceinline__ void transpose4(const uint32_t a[4], uint32_t t[4]) {
  const uint32_t lo01 = __byte_perm(a[0], a[1], 0x5140), hi01 = __byte_perm(a[0], a[1], 0x7362);
  const uint32_t lo23 = __byte_perm(a[2], a[3], 0x5140), hi23 = __byte_perm(a[2], a[3], 0x7362);
  t[0] = __byte_perm(lo01, lo23, 0x5410);
  t[1] = __byte_perm(lo01, lo23, 0x7632);
  t[2] = __byte_perm(hi01, hi23, 0x5410);
  t[3] = __byte_perm(hi01, hi23, 0x7632);
}

// power-of-two scale 2^E >= m (E from frexp; 1 for m == 0), as its inverse
__device__ __forceinline__ double inv_pow2_scale(double m, double &scale) {
  if (!(m > 0.0)) {
    scale = 1.0;
    return 1.0;
  }
  int e;
  frexp(m, &e);
  scale = ldexp(1.0, e);
  return ldexp(1.0, -e);
}

// The same scale for the largest |v| of a warp, from the biased exponents
// alone: a normal m with exponent field E has frexp exponent E - 1022, so
// scale = 2^(E - 1022) and its inverse are built from their bits.  Each lane
// passes the largest exponent field of its values; all-zero or subnormal
// (E = 0) and huge (E >= 2045) rows take the general path through `m`.
__device__ __forceinline__ double warp_inv_pow2_scale(unsigned e_lane, double m_lane, double &scale) {
  const unsigned e = __reduce_max_sync(0xffffffffu, e_lane);
  if (e == 0u || e >= 2045u) {
    double m = m_lane;
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    return inv_pow2_scale(m, scale);
  }
  scale = __hiloint2double((int)((e + 1u) << 20), 0);
  return __hiloint2double((int)((2045u - e) << 20), 0);
}
// exponent field of x (sign ignored)
__device__ __forceinline__ unsigned exp_field(double x) { return ((unsigned)__double2hiint(x) >> 20) & 0x7ffu; }

}  // namespace tc
}  // namespace nkx
