// Mixed-precision (tcgen05 tensor-core) Fock build path.
#include "plan.cuh"

namespace nkx {

bool mixed_available(const Plan &) { return false; }

void fock_build_mixed(Plan &, int, int, bool, bool, bool, cudaStream_t, StageTimer &) {
  throw Error{NKX_ERR_UNSUPPORTED, "mixed precision path unavailable"};
}

}  // namespace nkx
