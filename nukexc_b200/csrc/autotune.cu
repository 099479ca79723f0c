// Autotuner of the mixed-precision Fock build (nkx_plan_autotune): it times
// whole builds on the caller's orbitals and keeps, one knob at a time, the
// fastest of
//   the Y path of the GGA density gradient (off / on),
//   the tcgen05 MMA width of the density contraction (N = 64 / 128; by
//   default 128 from 1024 orbitals on),
//   the V contraction's shape: CTA pairs (M = 256 x N = 64, double-buffered
//   accumulators) or one CTA per tile, and then its MMA width (N = 128 / 64)
//   and its epilogue warps (16 / 8; CTA pairs, or one CTA at N = 128),
//   the chunk size (x1, x2, x4 of the current pair limit, memory permitting),
// each knob tried with the others at their best so far.  Every new
// configuration gets one untimed build first (allocations, first touch), then
// one timed build (CUDA events around the whole build).  Results can be kept
// in a text cache file, one line per problem:
//   <device name>|<SMs>|nbf|nblk|npairs|npts|nocc|nspin|gga|v2  v_n dens_n ypath v_warps v_pair chunk_pairs best_ms
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <functional>
#include <sstream>
#include <string>
#include <vector>

#include "plan.cuh"

namespace nkx {

nkx_status run_guarded(const char *where, const std::function<void()> &fn);

namespace {

std::string signature(const Plan &P, int nspin, int nocc) {
  cudaDeviceProp prop{};
  NKX_CUDA(cudaGetDeviceProperties(&prop, P.device));
  std::string name = prop.name;
  std::replace(name.begin(), name.end(), ' ', '_');
  std::ostringstream o;
  o << name << "|" << prop.multiProcessorCount << "|" << P.nbf << "|" << P.nblk << "|" << P.npairs << "|" << P.npts
    << "|" << nocc << "|" << nspin << "|" << (P.gga ? 1 : 0) << "|v2";
  return o.str();
}

bool cache_lookup(const char *path, const std::string &sig, nkx_tuning &t) {
  if (!path) return false;
  std::ifstream f(path);
  std::string line;
  bool hit = false;
  while (std::getline(f, line)) {  // the last line of a signature wins
    std::istringstream in(line);
    std::string key;
    nkx_tuning r{};
    if (in >> key >> r.v_n >> r.dens_n >> r.ypath >> r.v_warps >> r.v_pair >> r.chunk_pairs >> r.best_ms &&
        key == sig) {
      t = r;
      hit = true;
    }
  }
  return hit;
}

void cache_store(const char *path, const std::string &sig, const nkx_tuning &t) {
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  NKX_REQUIRE(f.good(), NKX_ERR_ARG, std::string("cannot append to the tuning cache ") + path);
  f << sig << " " << t.v_n << " " << t.dens_n << " " << t.ypath << " " << t.v_warps << " " << t.v_pair << " "
    << t.chunk_pairs << " " << t.best_ms << "\n";
}

void apply(Plan &P, const nkx_tuning &t) {
  NKX_REQUIRE((t.v_n == 64 || t.v_n == 128) && (t.dens_n == 0 || t.dens_n == 64 || t.dens_n == 128) && t.ypath >= -1 &&
                  t.ypath <= 1 && (t.v_warps == 8 || t.v_warps == 16) && (t.v_pair == 0 || t.v_pair == 1),
              NKX_ERR_ARG,
              "tuning: v_n must be 64 or 128, dens_n 0, 64 or 128, ypath -1, 0 or 1, v_warps 8 or 16, v_pair 0 or 1");
  P.drop_graphs();
  P.tune.v_n = t.v_n;
  P.tune.dens_n = t.dens_n;
  P.tune.ypath = t.ypath;
  P.tune.v_warps = t.v_warps;
  P.tune.v_pair = t.v_pair;
  if (t.chunk_pairs > 0 && t.chunk_pairs != P.chunk_pair_limit) plan_chunks(P, t.chunk_pairs);
}

nkx_tuning current(const Plan &P) {
  nkx_tuning t{};
  t.v_n = P.tune.v_n;
  t.dens_n = P.tune.dens_n;
  t.ypath = P.tune.ypath;
  t.v_warps = P.tune.v_warps;
  t.v_pair = P.tune.v_pair;
  t.chunk_pairs = P.chunk_pair_limit;
  return t;
}

}  // namespace

static void autotune(Plan &P, int nspin, int nocc, const double *C, const double *occ, int mem, const char *cache,
                     nkx_tuning *out, cudaStream_t s) {
  NKX_REQUIRE(nspin == 1 || nspin == 2, NKX_ERR_ARG, "nspin must be 1 or 2");
  NKX_REQUIRE(nocc > 0 && C && occ, NKX_ERR_ARG, "invalid orbitals");
  NKX_REQUIRE(mixed_available(P), NKX_ERR_UNSUPPORTED, "the mixed-precision build needs an sm_100 device");
  const std::string sig = signature(P, nspin, nocc);
  nkx_tuning best = current(P);
  if (cache_lookup(cache, sig, best)) {
    apply(P, best);
    best.from_cache = 1;
    if (out) *out = best;
    return;
  }
  if (best.dens_n == 0) best.dens_n = density_width(P, nocc);  // the width the default picks
  const size_t nn = (size_t)P.nbf * P.nbf;
  double *V = nullptr;
  NKX_CUDA(cudaMalloc(&V, sizeof(double) * nspin * nn));
  int trials = 0;
  auto time_build = [&](const nkx_tuning &t) -> float {
    apply(P, t);
    double E = 0.0;
    fock_build(P, NKX_PREC_MIXED, nspin, nocc, C, occ, mem, 0, &E, V, nullptr, s);  // untimed: allocations
    fock_build(P, NKX_PREC_MIXED, nspin, nocc, C, occ, mem, 0, &E, V, nullptr, s);
    ++trials;
    return P.last.total_ms;
  };
  try {
    const long base_chunk = P.chunk_pair_limit;
    best.default_ms = time_build(best);
    best.best_ms = best.default_ms;
    auto consider = [&](nkx_tuning cand) {
      float ms = 0.f;
      try {
        ms = time_build(cand);
      } catch (const Error &e) {
        if (e.code != NKX_ERR_ALLOC) throw;  // a candidate that does not fit is skipped
        cudaGetLastError();
        apply(P, best);
        return;
      }
      if (ms < best.best_ms) {
        const float d = best.default_ms;
        best = cand;
        best.best_ms = ms;
        best.default_ms = d;
      }
    };
    if (P.gga) {
      nkx_tuning c = best;
      c.ypath = (best.ypath == 1) ? 0 : 1;
      if (best.ypath == -1) c.ypath = ((nocc + 127) / 128 * 128 >= 256) ? 0 : 1;  // the non-default side
      consider(c);
    }
    {
      nkx_tuning c = best;
      c.dens_n = best.dens_n == 64 ? 128 : 64;
      consider(c);
    }
    {
      nkx_tuning c = best;
      c.v_pair = 1 - best.v_pair;
      consider(c);
    }
    if (!best.v_pair) {
      nkx_tuning c = best;
      c.v_n = best.v_n == 128 ? 64 : 128;
      consider(c);
    }
    if (best.v_pair || best.v_n == 128) {
      nkx_tuning c = best;
      c.v_warps = best.v_warps == 16 ? 8 : 16;
      consider(c);
    }
    for (int mult : {2, 4}) {
      if (base_chunk * mult > P.npairs * 2) break;  // already one chunk
      size_t fr = 0, tot = 0;
      NKX_CUDA(cudaMemGetInfo(&fr, &tot));
      const double extra = (double)(base_chunk * mult - best.chunk_pairs) * (4 << 20);  // generous per-pair bytes
      if (extra > 0.8 * (double)fr) break;
      nkx_tuning c = best;
      c.chunk_pairs = base_chunk * mult;
      consider(c);
    }
  } catch (...) {
    cudaFree(V);
    throw;
  }
  cudaFree(V);
  apply(P, best);
  best.trials = trials;
  best.from_cache = 0;
  cache_store(cache, sig, best);
  if (out) *out = best;
}

}  // namespace nkx

using namespace nkx;

extern "C" {

NKX_API nkx_status nkx_plan_autotune(nkx_plan *plan, int nspin, int nocc, const double *C, const double *occ, int mem,
                                     const char *cache_path, nkx_tuning *out, void *stream) {
  return run_guarded("nkx_plan_autotune", [&] {
    NKX_REQUIRE(plan, NKX_ERR_ARG, "plan is NULL");
    Plan &P = *reinterpret_cast<Plan *>(plan);
    autotune(P, nspin, nocc, C, occ, mem, cache_path, out, stream ? (cudaStream_t)stream : P.stream);
  });
}

NKX_API nkx_status nkx_plan_get_tuning(const nkx_plan *plan, nkx_tuning *out) {
  return run_guarded("nkx_plan_get_tuning", [&] {
    NKX_REQUIRE(plan && out, NKX_ERR_ARG, "invalid arguments");
    *out = current(*reinterpret_cast<const Plan *>(plan));
  });
}

NKX_API nkx_status nkx_plan_set_tuning(nkx_plan *plan, const nkx_tuning *t) {
  return run_guarded("nkx_plan_set_tuning", [&] {
    NKX_REQUIRE(plan && t, NKX_ERR_ARG, "invalid arguments");
    apply(*reinterpret_cast<Plan *>(plan), *t);
  });
}

}  // extern "C"
