// Shared definitions of the nkx CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/nkx.h"

#define NKX_HD __host__ __device__

namespace nkx {

constexpr double kPi = 3.14159265358979323846;
constexpr int kBatch = 256;      // grid points per batch
constexpr int kBlockF = 128;     // basis functions per function block

void set_error(const std::string &msg);

struct Error {
  nkx_status code;
  std::string msg;
};

}  // namespace nkx

// Throw-free status plumbing: inside the library every failing CUDA call is
// converted into a C++ exception that the C-ABI wrappers catch.
#define NKX_CUDA(call)                                                                            \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      throw nkx::Error{NKX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + \
                                         __FILE__ + ":" + std::to_string(__LINE__)};              \
  } while (0)

#define NKX_REQUIRE(cond, code, msg)                  \
  do {                                                \
    if (!(cond)) throw nkx::Error{(code), (msg)};     \
  } while (0)

#define NKX_LAUNCH_CHECK() NKX_CUDA(cudaGetLastError())
