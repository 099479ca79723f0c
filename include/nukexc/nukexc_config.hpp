// Drop-in replacement of nukexc/nukexc_config.hpp for the grid-integration
// Fock-build path: the view aliases, Point and ExecSpace that the reference's
// hot-path headers use (nukexc/nukexc_config.hpp:90-115), over libnkx.so.
//
// Two modes:
//  * NKX_WITH_KOKKOS defined: the aliases are the reference's Kokkos views
//    (device memory, LayoutLeft); the shim functions read view.data() and
//    view.extent(i) and call the C ABI of include/nkx.h.
//  * otherwise: a minimal reference-counted device array (nkx_shim::View)
//    stands in for Kokkos::View, so code written against the reference's
//    functions compiles and runs without Kokkos.
// Errors of the C ABI become std::runtime_error (the reference's error
// convention), with the message of nkx_last_error().
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../nkx.h"

#ifdef NKX_WITH_KOKKOS
#include <Kokkos_Core.hpp>
#endif

namespace nkx_shim {

inline void check(nkx_status st, const char *where) {
  if (st != NKX_OK) throw std::runtime_error(std::string(where) + ": " + nkx_last_error());
}
inline void check_cuda(cudaError_t e, const char *where) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

#ifndef NKX_WITH_KOKKOS
// Device array standing in for Kokkos::View<T*> / Kokkos::View<T**, LayoutLeft>:
// shallow copies share the allocation (like views), element (i, j) of a
// rank-2 array is at data()[i + j * extent(0)], new arrays are zeroed.
template <class T>
class View {
 public:
  View() = default;
  explicit View(const std::string &label, size_t n0 = 0, size_t n1 = 1) : label_(label), n0_(n0), n1_(n1) {
    const size_t n = n0 * n1;
    if (n) {
      T *p = nullptr;
      check_cuda(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
      check_cuda(cudaMemset(p, 0, n * sizeof(T)), "cudaMemset");
      p_ = std::shared_ptr<T>(p, [](T *q) { cudaFree(q); });
    }
  }
  T *data() const { return p_.get(); }
  size_t extent(int r) const { return r == 0 ? n0_ : (r == 1 ? n1_ : 1); }
  size_t size() const { return n0_ * n1_; }
  bool span_is_contiguous() const { return true; }
  const std::string &label() const { return label_; }

 private:
  std::string label_;
  size_t n0_ = 0, n1_ = 1;
  std::shared_ptr<T> p_;
};

template <class T>
void copy_from_host(View<T> &v, const std::vector<T> &h) {
  if (h.size() != v.size()) throw std::runtime_error("copy_from_host: size mismatch");
  check_cuda(cudaMemcpy(v.data(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
}
template <class T>
std::vector<T> copy_to_host(const View<T> &v) {
  std::vector<T> h(v.size());
  check_cuda(cudaMemcpy(h.data(), v.data(), h.size() * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy");
  return h;
}
#endif

// host copy of a device buffer of n elements
template <class T>
std::vector<T> to_host(const T *d, size_t n) {
  std::vector<T> h(n);
  if (n) check_cuda(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy");
  return h;
}

}  // namespace nkx_shim

namespace Nukexc {

// ArborX::Point<3, double> layout: three contiguous doubles
struct Point {
  double coords[3];
  double &operator[](int i) { return coords[i]; }
  const double &operator[](int i) const { return coords[i]; }
};
static_assert(sizeof(Point) == 3 * sizeof(double), "Point must be three packed doubles");

#ifdef NKX_WITH_KOKKOS
using ExecSpace = Kokkos::DefaultExecutionSpace;
using DeviceView2DLeft = Kokkos::View<double **, Kokkos::LayoutLeft, ExecSpace>;
using DeviceView2D = Kokkos::View<double **, ExecSpace>;
using DeviceView1D = Kokkos::View<double *, ExecSpace>;
using DeviceView1DLeft = Kokkos::View<double *, Kokkos::LayoutLeft, ExecSpace>;
template <class T>
using DeviceArray = Kokkos::View<T *, ExecSpace>;
inline cudaStream_t stream_of(const ExecSpace &s) { return s.cuda_stream(); }
#else
// the default stream stands in for a Kokkos execution-space instance
struct ExecSpace {
  cudaStream_t stream = nullptr;
};
using DeviceView2DLeft = nkx_shim::View<double>;
using DeviceView2D = nkx_shim::View<double>;
using DeviceView1D = nkx_shim::View<double>;
using DeviceView1DLeft = nkx_shim::View<double>;
template <class T>
using DeviceArray = nkx_shim::View<T>;
inline cudaStream_t stream_of(const ExecSpace &s) { return s.stream; }
#endif

// Precision of the plan-based drop-ins (the *_sparse / *_tiled XC and J
// functions, which run the batched Fock build of nkx_fock_build).
// NKX_PREC_FP64 (the default) computes like the reference; NKX_PREC_MIXED
// runs the contractions on the B200 tensor cores as exact int8-digit
// products (about 1e-9 relative to the operands' row maxima; within
// |dE_xc| <= 1e-6 Eh and max|dV_xc| <= 1e-7 of FP64).  The first use reads
// the environment variable NKX_PRECISION ("mixed" or "fp64"), so an
// unmodified driver compiled against these headers can switch without a code
// change; set_precision() overrides it.  The dense functions (compute_lda ...
// on collocation matrices) are always FP64.
namespace shim_detail {
inline int &precision_slot() {
  static int p = [] {
    const char *e = std::getenv("NKX_PRECISION");
    return (e && (std::string(e) == "mixed" || std::string(e) == "MIXED")) ? (int)NKX_PREC_MIXED
                                                                            : (int)NKX_PREC_FP64;
  }();
  return p;
}
}  // namespace shim_detail
inline void set_precision(int precision) {
  if (precision != NKX_PREC_FP64 && precision != NKX_PREC_MIXED)
    throw std::runtime_error("set_precision: NKX_PREC_FP64 or NKX_PREC_MIXED expected");
  shim_detail::precision_slot() = precision;
}
inline int precision() { return shim_detail::precision_slot(); }

// libxc's xc_func_type identifies the functional by info->number; any type
// with that member works here (the ids LDA_X 1, LDA_C_VWN 7, LDA_C_PW 12,
// LDA_C_PW_MOD 13, GGA_X_PBE 101, GGA_C_PBE 130 are supported)
template <class F>
int functional_id(const F &func) {
  return func.info->number;
}

}  // namespace Nukexc
