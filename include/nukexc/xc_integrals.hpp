// Drop-in replacement of the dense functions of nukexc/xc_integrals.hpp:
// XC_result / XC_result_polarized (:60-71), compute_lda (:73-166),
// compute_lsda (:168-261), compute_gga (:424-541) and compute_gga_lsda
// (:543-726) over nkx_xc_dense.  As in the reference, one call evaluates one
// functional (`func`, identified by libxc's info->number); the returned
// potential is the full symmetrised N_bf x N_bf matrix and the energy is
// sum_g w_g rho_g exc_g.  Functional families are checked like the reference
// checks libxc's family and spin.
#pragma once

#include "nukexc_config.hpp"

namespace Nukexc {

struct XC_result {
  double energy;
  DeviceView2DLeft potential;
};

struct XC_result_polarized {
  double energy;
  DeviceView2DLeft potential_alpha;
  DeviceView2DLeft potential_beta;
};

namespace shim_detail {
inline bool is_gga(int id) { return id == NKX_XC_GGA_X_PBE || id == NKX_XC_GGA_C_PBE; }

inline nkx_plan_options xc_options(int id) {
  nkx_plan_options o{};
  o.batch_points = 256;
  o.screen_tol = 1e-10;
  o.nfunc = 1;
  o.func_ids[0] = id;
  o.dens_threshold = 1e-15;
  return o;
}

// nspin = 1: one block; nspin = 2: alpha and beta stacked into scratch
inline double xc_dense(const DeviceView2DLeft &phi, const double *gx, const double *gy, const double *gz,
                       const DeviceView1D &w, int nspin, int nocc, const double *C, const double *occ, int id,
                       double *V) {
  nkx_plan_options o = xc_options(id);
  double E = 0.0;
  nkx_shim::check(nkx_xc_dense((int)phi.extent(0), (long)phi.extent(1), phi.data(), gx, gy, gz, w.data(), nspin,
                               nocc, C, occ, &o, &E, V, nullptr),
                  "compute_xc");
  return E;
}

inline void stack2(const DeviceView2DLeft &a, const DeviceView2DLeft &b, DeviceView1D &out, size_t n) {
  nkx_shim::check_cuda(cudaMemcpy(out.data(), a.data(), n * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  nkx_shim::check_cuda(cudaMemcpy(out.data() + n, b.data(), n * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
}
}  // namespace shim_detail

template <class F>
XC_result compute_lda(const DeviceView2DLeft collocation_values, const DeviceView1D weights,
                      const DeviceView2DLeft mo_orbitals, const DeviceView1D mo_coeff, const F &func) {
  const int id = functional_id(func);
  if (shim_detail::is_gga(id)) throw std::runtime_error("compute_lda: functional is not an LDA");
  const size_t nbf = collocation_values.extent(0);
  DeviceView2DLeft V("XC potential", nbf, nbf);
  const double E = shim_detail::xc_dense(collocation_values, nullptr, nullptr, nullptr, weights, 1,
                                         (int)mo_orbitals.extent(1), mo_orbitals.data(), mo_coeff.data(), id,
                                         V.data());
  return XC_result{E, V};
}

template <class F>
XC_result compute_gga(const DeviceView2DLeft collocation_values, const DeviceView2DLeft collocation_gx,
                      const DeviceView2DLeft collocation_gy, const DeviceView2DLeft collocation_gz,
                      const DeviceView1D weights, const DeviceView2DLeft mo_orbitals, const DeviceView1D mo_coeff,
                      const F &func) {
  const int id = functional_id(func);
  if (!shim_detail::is_gga(id)) throw std::runtime_error("compute_gga: functional is not a GGA");
  const size_t nbf = collocation_values.extent(0);
  DeviceView2DLeft V("XC potential", nbf, nbf);
  const double E = shim_detail::xc_dense(collocation_values, collocation_gx.data(), collocation_gy.data(),
                                         collocation_gz.data(), weights, 1, (int)mo_orbitals.extent(1),
                                         mo_orbitals.data(), mo_coeff.data(), id, V.data());
  return XC_result{E, V};
}

namespace shim_detail {
inline XC_result_polarized polarized(const DeviceView2DLeft &phi, const double *gx, const double *gy,
                                     const double *gz, const DeviceView1D &w, const DeviceView2DLeft &Ca,
                                     const DeviceView1D &oa, const DeviceView2DLeft &Cb, const DeviceView1D &ob,
                                     int id) {
  const size_t nbf = phi.extent(0), nocc = Ca.extent(1);
  if (Cb.extent(1) != nocc || Cb.extent(0) != nbf)
    throw std::runtime_error("compute_lsda: alpha and beta orbital blocks must have the same shape");
  DeviceView1D C("stacked orbitals", 2 * nbf * nocc), occ("stacked occupations", 2 * nocc),
      V("stacked potentials", 2 * nbf * nbf);
  stack2(Ca, Cb, C, nbf * nocc);
  nkx_shim::check_cuda(cudaMemcpy(occ.data(), oa.data(), nocc * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  nkx_shim::check_cuda(cudaMemcpy(occ.data() + nocc, ob.data(), nocc * sizeof(double), cudaMemcpyDeviceToDevice),
                       "copy");
  const double E = xc_dense(phi, gx, gy, gz, w, 2, (int)nocc, C.data(), occ.data(), id, V.data());
  DeviceView2DLeft Va("XC potential alpha", nbf, nbf), Vb("XC potential beta", nbf, nbf);
  nkx_shim::check_cuda(cudaMemcpy(Va.data(), V.data(), nbf * nbf * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  nkx_shim::check_cuda(
      cudaMemcpy(Vb.data(), V.data() + nbf * nbf, nbf * nbf * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  return XC_result_polarized{E, Va, Vb};
}
}  // namespace shim_detail

template <class F>
XC_result_polarized compute_lsda(const DeviceView2DLeft collocation_values, const DeviceView1D weights,
                                 const DeviceView2DLeft mo_alpha, const DeviceView1D occ_alpha,
                                 const DeviceView2DLeft mo_beta, const DeviceView1D occ_beta, const F &func) {
  const int id = functional_id(func);
  if (shim_detail::is_gga(id)) throw std::runtime_error("compute_lsda: functional is not an LDA");
  return shim_detail::polarized(collocation_values, nullptr, nullptr, nullptr, weights, mo_alpha, occ_alpha, mo_beta,
                                occ_beta, id);
}

template <class F>
XC_result_polarized compute_gga_lsda(const DeviceView2DLeft collocation_values,
                                     const DeviceView2DLeft collocation_gx, const DeviceView2DLeft collocation_gy,
                                     const DeviceView2DLeft collocation_gz, const DeviceView1D weights,
                                     const DeviceView2DLeft mo_alpha, const DeviceView1D occ_alpha,
                                     const DeviceView2DLeft mo_beta, const DeviceView1D occ_beta, const F &func) {
  const int id = functional_id(func);
  if (!shim_detail::is_gga(id)) throw std::runtime_error("compute_gga_lsda: functional is not a GGA");
  return shim_detail::polarized(collocation_values, collocation_gx.data(), collocation_gy.data(),
                                collocation_gz.data(), weights, mo_alpha, occ_alpha, mo_beta, occ_beta, id);
}

}  // namespace Nukexc
