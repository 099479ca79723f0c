// Drop-in replacement of the functions of nukexc/xc_integrals.hpp:
// XC_result / XC_result_polarized (:60-71), compute_lda (:73-166),
// compute_lsda (:168-261), compute_gga (:424-541) and compute_gga_lsda
// (:543-726) over nkx_xc_dense, and the sparse variants compute_lsda_sparse
// (:263-422) and compute_gga_lsda_sparse (:728-977) over the neighbour list's
// plan (nkx_plan_set_functional + nkx_fock_build, in the precision chosen by
// set_precision / NKX_PRECISION, FP64 by default).  As in the
// reference, one call evaluates one functional (`func`, identified by libxc's
// info->number); the returned potential is the full symmetrised
// N_bf x N_bf matrix and the energy is sum_g w_g rho_g exc_g.  Functional
// families are checked like the reference checks libxc's family and spin.
// Alpha and beta may have different numbers of orbitals.
#pragma once

#include "nukexc_config.hpp"
#include "octree.hpp"

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

// alpha and beta orbitals / occupations stacked into 2 blocks of
// nocc = max(nocc_a, nocc_b) columns (missing columns zero, occupation 0)
struct SpinStack {
  size_t nocc;
  DeviceView1D C, occ;
  SpinStack(const DeviceView2DLeft &Ca, const DeviceView1D &oa, const DeviceView2DLeft &Cb, const DeviceView1D &ob)
      : nocc(std::max<size_t>(1, std::max(Ca.extent(1), Cb.extent(1)))),
        C("stacked orbitals", 2 * Ca.extent(0) * nocc),
        occ("stacked occupations", 2 * nocc) {
    const size_t nbf = Ca.extent(0);
    if (Cb.extent(0) != nbf) throw std::runtime_error("alpha and beta orbitals must have the same number of rows");
    const DeviceView2DLeft *Cs[2] = {&Ca, &Cb};
    const DeviceView1D *os[2] = {&oa, &ob};
    for (int s = 0; s < 2; ++s) {
      const size_t n = Cs[s]->extent(1);
      if (os[s]->extent(0) < n) throw std::runtime_error("fewer occupations than orbitals");
      if (n == 0) continue;
      nkx_shim::check_cuda(cudaMemcpy(C.data() + s * nbf * nocc, Cs[s]->data(), nbf * n * sizeof(double),
                                      cudaMemcpyDeviceToDevice),
                           "copy");
      nkx_shim::check_cuda(
          cudaMemcpy(occ.data() + s * nocc, os[s]->data(), n * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
    }
  }
};

inline XC_result_polarized split_potential(double E, const DeviceView1D &V, size_t nbf) {
  DeviceView2DLeft Va("XC potential alpha", nbf, nbf), Vb("XC potential beta", nbf, nbf);
  nkx_shim::check_cuda(cudaMemcpy(Va.data(), V.data(), nbf * nbf * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  nkx_shim::check_cuda(
      cudaMemcpy(Vb.data(), V.data() + nbf * nbf, nbf * nbf * sizeof(double), cudaMemcpyDeviceToDevice), "copy");
  return XC_result_polarized{E, Va, Vb};
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
  const size_t nbf = phi.extent(0);
  if (Ca.extent(0) != nbf) throw std::runtime_error("compute_lsda: orbitals and collocation differ in N_bf");
  SpinStack st(Ca, oa, Cb, ob);
  DeviceView1D V("stacked potentials", 2 * nbf * nbf);
  const double E = xc_dense(phi, gx, gy, gz, w, 2, (int)st.nocc, st.C.data(), st.occ.data(), id, V.data());
  return split_potential(E, V, nbf);
}

// polarised XC through the neighbour list's plan (precision())
inline XC_result_polarized polarized_sparse(const STOBasisSet &basis, const FlatGrid &grid, const NeighborList &nl,
                                            const DeviceView2DLeft &Ca, const DeviceView1D &oa,
                                            const DeviceView2DLeft &Cb, const DeviceView1D &ob, int id) {
  const size_t nbf = basis.nbf();
  if (Ca.extent(0) != nbf) throw std::runtime_error("compute_lsda_sparse: orbitals and basis differ in N_bf");
  nkx_plan *p = nl.plans->get(basis, nullptr, grid);
  nkx_shim::check(nkx_plan_set_functional(p, 1, &id, xc_options(id).dens_threshold), "compute_lsda_sparse");
  SpinStack st(Ca, oa, Cb, ob);
  DeviceView1D V("stacked potentials", 2 * nbf * nbf);
  double E = 0.0;
  nkx_shim::check(nkx_fock_build(p, precision(), 2, (int)st.nocc, st.C.data(), st.occ.data(), NKX_MEM_DEVICE, 0,
                                 &E, V.data(), nullptr, nullptr),
                  "compute_xc_sparse");
  return split_potential(E, V, nbf);
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

template <class F>
XC_result_polarized compute_lsda_sparse(const STOBasisSet basis, const FlatGrid grid, const NeighborList nl,
                                        const DeviceView2DLeft mo_alpha, const DeviceView1D occ_alpha,
                                        const DeviceView2DLeft mo_beta, const DeviceView1D occ_beta, const F &func) {
  const int id = functional_id(func);
  if (shim_detail::is_gga(id)) throw std::runtime_error("compute_lsda_sparse: functional is not an LDA");
  return shim_detail::polarized_sparse(basis, grid, nl, mo_alpha, occ_alpha, mo_beta, occ_beta, id);
}

template <class F>
XC_result_polarized compute_gga_lsda_sparse(const STOBasisSet basis, const FlatGrid grid, const NeighborList nl,
                                            const DeviceView2DLeft mo_alpha, const DeviceView1D occ_alpha,
                                            const DeviceView2DLeft mo_beta, const DeviceView1D occ_beta,
                                            const F &func) {
  const int id = functional_id(func);
  if (!shim_detail::is_gga(id)) throw std::runtime_error("compute_gga_lsda_sparse: functional is not a GGA");
  return shim_detail::polarized_sparse(basis, grid, nl, mo_alpha, occ_alpha, mo_beta, occ_beta, id);
}

}  // namespace Nukexc
