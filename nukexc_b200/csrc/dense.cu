// Dense-matrix entry points with the shapes of the reference's dense
// algorithm (fill_collocation, compute_density_and_sigma, compute_gga ...,
// sto_potential_collocation_scaled, compute_half_inverse).  They operate on
// caller-owned device buffers.  The batched, screened Fock build of plan.cu
// is the hot path; these exist so the reference's dense call sequence can be
// replaced one function at a time.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <functional>
#include <vector>

#include "functionals.cuh"
#include "host_setup.hpp"

namespace nkx {

nkx_status run_guarded(const char *where, const std::function<void()> &fn);

template <class T>
struct DevBuf {
  T *p = nullptr;
  explicit DevBuf(size_t n) {
    if (n) NKX_CUDA(cudaMalloc(&p, n * sizeof(T)));
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

__global__ void colloc_dense_kernel(const StoFunc *__restrict__ f, int nbf, const double *__restrict__ pts,
                                    long npts, double *phi, double *gx, double *gy, double *gz) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)nbf * npts) return;
  const int mu = (int)(idx % nbf);
  const long g = idx / nbf;
  const double px = pts[3 * g], py = pts[3 * g + 1], pz = pts[3 * g + 2];
  if (gx) {
    double v, a, b, c;
    sto_value_grad(f[mu], px, py, pz, v, a, b, c);
    phi[idx] = v;
    gx[idx] = a;
    gy[idx] = b;
    gz[idx] = c;
  } else {
    phi[idx] = sto_value(f[mu], px, py, pz);
  }
}

// One warp per point: T_i = sum_mu C(mu,i) phi(mu,g); rho = sum occ_i T_i^2,
// grad rho = 2 sum occ_i T_i grad T_i (density.hpp:188-255).
__global__ void density_dense_kernel(int nbf, long npts, const double *__restrict__ phi,
                                     const double *__restrict__ gx, const double *__restrict__ gy,
                                     const double *__restrict__ gz, int nocc, const double *__restrict__ C,
                                     const double *__restrict__ occ, double *rho, double *grad, double *sigma) {
  const long g = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= npts) return;
  const double *ph = phi + g * (long)nbf;
  double r = 0, sx = 0, sy = 0, sz = 0;
  for (int i = 0; i < nocc; ++i) {
    const double *ci = C + (long)i * nbf;
    double t = 0, tx = 0, ty = 0, tz = 0;
    for (int mu = lane; mu < nbf; mu += 32) {
      t += ci[mu] * ph[mu];
      if (gx) {
        tx += ci[mu] * gx[g * (long)nbf + mu];
        ty += ci[mu] * gy[g * (long)nbf + mu];
        tz += ci[mu] * gz[g * (long)nbf + mu];
      }
    }
    for (int o = 16; o; o >>= 1) {
      t += __shfl_xor_sync(0xffffffffu, t, o);
      tx += __shfl_xor_sync(0xffffffffu, tx, o);
      ty += __shfl_xor_sync(0xffffffffu, ty, o);
      tz += __shfl_xor_sync(0xffffffffu, tz, o);
    }
    r += occ[i] * t * t;
    sx += occ[i] * tx * t;
    sy += occ[i] * ty * t;
    sz += occ[i] * tz * t;
  }
  if (lane == 0) {
    rho[g] = r;
    if (grad) {
      grad[g] = 2 * sx;
      grad[npts + g] = 2 * sy;
      grad[2 * npts + g] = 2 * sz;
    }
    if (sigma) sigma[g] = 4.0 * (sx * sx + sy * sy + sz * sz);
  }
}

// libxc-layout functional evaluation (thread per point)
__global__ void xc_eval_kernel(XcSpec s, int nspin, long n, const double *rho, const double *sigma, double *exc,
                               double *vrho, double *vsigma) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= n) return;
  if (nspin == 1) {
    double f, vr, vs;
    const double r = rho[g];
    xc_unpol(s, r, sigma ? sigma[g] : 0.0, f, vr, vs);
    exc[g] = (r > 0 && f != 0.0) ? f / r : 0.0;
    vrho[g] = vr;
    if (vsigma) vsigma[g] = vs;
  } else {
    double f, d[5];
    const double ra = rho[2 * g], rb = rho[2 * g + 1];
    xc_pol(s, ra, rb, sigma ? sigma[3 * g] : 0.0, sigma ? sigma[3 * g + 1] : 0.0, sigma ? sigma[3 * g + 2] : 0.0,
           f, d);
    exc[g] = (ra + rb > 0 && f != 0.0) ? f / (ra + rb) : 0.0;
    vrho[2 * g] = d[0];
    vrho[2 * g + 1] = d[1];
    if (vsigma) {
      vsigma[3 * g] = d[2];
      vsigma[3 * g + 1] = d[3];
      vsigma[3 * g + 2] = d[4];
    }
  }
}

// Per point: functional of the (spin) densities, energy, and the Z matrix
// Z(mu, g) = w (1/2 phi vrho + vec . grad phi) (xc_integrals.hpp:486-515,
// :655-697).  Z holds nspin blocks of nbf x npts.
__global__ void xc_z_dense_kernel(XcSpec s, bool gga, int nbf, long npts, int nspin, const double *phi,
                                  const double *gx, const double *gy, const double *gz, const double *w,
                                  const double *rho, const double *grad, double *Z, double *Eacc) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double e = 0.0;
  if (g < npts) {
    double vr[2] = {0, 0}, vec[2][3] = {{0, 0, 0}, {0, 0, 0}};
    double gr[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int sp = 0; sp < nspin; ++sp)
      if (gga)
        for (int k = 0; k < 3; ++k) gr[sp][k] = grad[(size_t)sp * 3 * npts + k * npts + g];
    if (nspin == 1) {
      const double r = rho[g];
      const double sg = gr[0][0] * gr[0][0] + gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2];
      double f, vrho, vs;
      xc_unpol(s, r, sg, f, vrho, vs);
      e = w[g] * f;
      vr[0] = vrho;
      for (int k = 0; k < 3; ++k) vec[0][k] = 2.0 * vs * gr[0][k];
    } else {
      const double ra = rho[g], rb = rho[npts + g];
      const double saa = gr[0][0] * gr[0][0] + gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2];
      const double sab = gr[0][0] * gr[1][0] + gr[0][1] * gr[1][1] + gr[0][2] * gr[1][2];
      const double sbb = gr[1][0] * gr[1][0] + gr[1][1] * gr[1][1] + gr[1][2] * gr[1][2];
      double f, d[5];
      xc_pol(s, ra, rb, saa, sab, sbb, f, d);
      e = w[g] * f;
      vr[0] = d[0];
      vr[1] = d[1];
      for (int k = 0; k < 3; ++k) {
        vec[0][k] = 2.0 * d[2] * gr[0][k] + d[3] * gr[1][k];
        vec[1][k] = 2.0 * d[4] * gr[1][k] + d[3] * gr[0][k];
      }
    }
    for (int sp = 0; sp < nspin; ++sp) {
      double *Zs = Z + (size_t)sp * nbf * npts;
      for (int mu = 0; mu < nbf; ++mu) {
        const size_t i = (size_t)mu + (size_t)g * nbf;
        double z = 0.5 * phi[i] * vr[sp];
        if (gga) z += vec[sp][0] * gx[i] + vec[sp][1] * gy[i] + vec[sp][2] * gz[i];
        Zs[i] = w[g] * z;
      }
    }
  }
  for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(Eacc, e);
}

// V += Vbar + Vbar^T with Vbar(i,j) = sum_g A(i,g) B(j,g); A, B column-major
// n x npts (xc_integrals.hpp:148-153 forms Vbar by DGEMM and then adds its
// transpose).  n is small (the basis) and npts large, so the point range is
// split over blockIdx.z: each block forms a 64 x 64 tile over its slice of
// points in registers (4 x 4 per thread, 16-point steps through shared
// memory) and adds it to V(i,j) and V(j,i) atomically.  V must be zero on
// entry.
constexpr int kGemmTile = 64, kGemmK = 16;
__global__ void __launch_bounds__(256) nt_gemm_sym_kernel(int n, long npts, long kslice, const double *__restrict__ A,
                                                          const double *__restrict__ B, double *V) {
  __shared__ double As[kGemmK][kGemmTile + 1], Bs[kGemmK][kGemmTile + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.y * kGemmTile, j0 = blockIdx.x * kGemmTile;
  const long g_lo = blockIdx.z * kslice, g_hi = min(npts, g_lo + kslice);
  double acc[4][4] = {};
  for (long g0 = g_lo; g0 < g_hi; g0 += kGemmK) {
    // 64 rows x 16 points of A and of B: thread t loads rows t % 64, points
    // t / 64 + 4 e (coalesced along the rows)
    for (int e = 0; e < 4; ++e) {
      const int r = threadIdx.x & 63, k = (threadIdx.x >> 6) + 4 * e;
      const long g = g0 + k;
      const bool gin = g < g_hi;
      As[k][r] = (gin && i0 + r < n) ? A[(size_t)(i0 + r) + (size_t)g * n] : 0.0;
      Bs[k][r] = (gin && j0 + r < n) ? B[(size_t)(j0 + r) + (size_t)g * n] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kGemmK; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        a[r] = As[k][tx + 16 * r];
        b[r] = Bs[k][ty + 16 * r];
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * c;
      if (i < n && j < n) {
        atomicAdd(&V[(size_t)i + (size_t)j * n], acc[r][c]);
        atomicAdd(&V[(size_t)j + (size_t)i * n], acc[r][c]);
      }
    }
}

// Launch of nt_gemm_sym_kernel for one n x n output (zeroed here): enough
// point slices to give every SM a couple of blocks.
static void launch_nt_gemm_sym(int n, long npts, const double *A, const double *B, double *V, cudaStream_t s) {
  NKX_CUDA(cudaMemsetAsync(V, 0, sizeof(double) * n * n, s));
  const int nt = (n + kGemmTile - 1) / kGemmTile;
  const long want = std::max<long>(1, (2L * 148 + (long)nt * nt - 1) / ((long)nt * nt));
  const long nsl = std::max<long>(1, std::min<long>(want, (npts + 255) / 256));
  const long kslice = ((npts + nsl - 1) / nsl + kGemmK - 1) / kGemmK * kGemmK;
  const long nz = (npts + kslice - 1) / kslice;
  nt_gemm_sym_kernel<<<dim3(nt, nt, (unsigned)nz), 256, 0, s>>>(n, npts, kslice, A, B, V);
}

__global__ void potential_dense_kernel(const AuxFunc *__restrict__ f, int naux, const double *__restrict__ pts,
                                       const double *__restrict__ w, long npts, double *Vw) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)naux * npts) return;
  const int a = (int)(idx % naux);
  const long g = idx / naux;
  Vw[idx] = aux_potential(f[a], pts[3 * g], pts[3 * g + 1], pts[3 * g + 2]) * w[g];
}

__global__ void precondition_kernel(int N, const double *S, double *A, double *D) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N && j < N) A[(size_t)i + (size_t)j * N] = S[(size_t)i + (size_t)j * N] /
                                                      sqrt(S[(size_t)i + (size_t)i * N] * S[(size_t)j + (size_t)j * N]);
  if (j == 0 && i < N) D[i] = sqrt(S[(size_t)i + (size_t)i * N]);
}

XcSpec make_spec(const nkx_plan_options *o) {
  XcSpec s;
  NKX_REQUIRE(o && o->nfunc >= 1 && o->nfunc <= 4, NKX_ERR_ARG, "opts.nfunc must be 1..4");
  s.nfunc = o->nfunc;
  for (int i = 0; i < 4; ++i) s.ids[i] = i < o->nfunc ? o->func_ids[i] : 0;
  for (int i = 0; i < o->nfunc; ++i)
    NKX_REQUIRE(func_supported(o->func_ids[i]), NKX_ERR_UNSUPPORTED, "unsupported functional id");
  s.thr = o->dens_threshold > 0 ? o->dens_threshold : 1e-15;
  return s;
}

bool spec_is_gga(const XcSpec &s) {
  for (int i = 0; i < s.nfunc; ++i)
    if (func_is_gga(s.ids[i])) return true;
  return false;
}

}  // namespace nkx

using namespace nkx;

static unsigned nblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

extern "C" nkx_status nkx_fill_collocation(const nkx_basis *basis, const double *d_points, long npts, double *d_phi,
                                           double *d_gx, double *d_gy, double *d_gz, void *stream) {
  return run_guarded("nkx_fill_collocation", [&] {
    NKX_REQUIRE(basis && basis->nbf > 0 && npts >= 0 && d_points && d_phi, NKX_ERR_ARG, "invalid arguments");
    NKX_REQUIRE(!d_gx || (d_gy && d_gz), NKX_ERR_ARG, "gradient buffers must be given together");
    for (int i = 0; i < basis->nbf; ++i)
      NKX_REQUIRE(basis->l[i] >= 0 && basis->l[i] <= 7 && basis->n[i] > basis->l[i] &&
                      abs(basis->m[i]) <= basis->l[i] && basis->zeta[i] > 0,
                  NKX_ERR_UNSUPPORTED, "basis function outside n > l, |m| <= l <= 7, zeta > 0");
    auto tab = make_sto_table(*basis);
    DevBuf<StoFunc> df(tab.size());
    cudaStream_t s = (cudaStream_t)stream;
    NKX_CUDA(cudaMemcpyAsync(df.p, tab.data(), tab.size() * sizeof(StoFunc), cudaMemcpyHostToDevice, s));
    const long tot = (long)basis->nbf * npts;
    if (tot > 0) colloc_dense_kernel<<<nblk(tot, 128), 128, 0, s>>>(df.p, basis->nbf, d_points, npts, d_phi, d_gx, d_gy, d_gz);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaStreamSynchronize(s));
  });
}

extern "C" nkx_status nkx_density_dense(int nbf, long npts, const double *d_phi, const double *d_gx,
                                        const double *d_gy, const double *d_gz, int nocc, const double *d_C,
                                        const double *d_occ, double *d_rho, double *d_grad, double *d_sigma,
                                        void *stream) {
  return run_guarded("nkx_density_dense", [&] {
    NKX_REQUIRE(nbf > 0 && npts >= 0 && nocc > 0 && d_phi && d_C && d_occ && d_rho, NKX_ERR_ARG,
                "invalid arguments");
    NKX_REQUIRE(!(d_grad || d_sigma) || (d_gx && d_gy && d_gz), NKX_ERR_ARG, "gradient output needs grad inputs");
    cudaStream_t s = (cudaStream_t)stream;
    if (npts > 0)
      density_dense_kernel<<<nblk(npts * 32, 256), 256, 0, s>>>(nbf, npts, d_phi, (d_grad || d_sigma) ? d_gx : nullptr,
                                                                d_gy, d_gz, nocc, d_C, d_occ, d_rho, d_grad, d_sigma);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaStreamSynchronize(s));
  });
}

extern "C" nkx_status nkx_xc_eval(int func_id, int nspin, long n, const double *d_rho, const double *d_sigma,
                                  double dens_threshold, double *d_exc, double *d_vrho, double *d_vsigma,
                                  void *stream) {
  return run_guarded("nkx_xc_eval", [&] {
    NKX_REQUIRE((nspin == 1 || nspin == 2) && n >= 0 && d_rho && d_exc && d_vrho, NKX_ERR_ARG, "invalid arguments");
    NKX_REQUIRE(func_supported(func_id), NKX_ERR_UNSUPPORTED, "unsupported functional id");
    NKX_REQUIRE(!func_is_gga(func_id) || (d_sigma && d_vsigma), NKX_ERR_ARG, "GGA needs sigma and vsigma");
    XcSpec sp;
    sp.nfunc = 1;
    sp.ids[0] = func_id;
    sp.ids[1] = sp.ids[2] = sp.ids[3] = 0;
    sp.thr = dens_threshold > 0 ? dens_threshold : 1e-15;
    cudaStream_t s = (cudaStream_t)stream;
    if (n > 0) xc_eval_kernel<<<nblk(n, 128), 128, 0, s>>>(sp, nspin, n, d_rho, d_sigma, d_exc, d_vrho, d_vsigma);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaStreamSynchronize(s));
  });
}

extern "C" nkx_status nkx_xc_dense(int nbf, long npts, const double *d_phi, const double *d_gx, const double *d_gy,
                                   const double *d_gz, const double *d_w, int nspin, int nocc, const double *d_C,
                                   const double *d_occ, const nkx_plan_options *opts, double *E, double *d_V,
                                   void *stream) {
  return run_guarded("nkx_xc_dense", [&] {
    NKX_REQUIRE(nbf > 0 && npts > 0 && (nspin == 1 || nspin == 2) && nocc > 0 && d_phi && d_w && d_C && d_occ &&
                    E && d_V,
                NKX_ERR_ARG, "invalid arguments");
    const XcSpec sp = make_spec(opts);
    const bool gga = spec_is_gga(sp);
    NKX_REQUIRE(!gga || (d_gx && d_gy && d_gz), NKX_ERR_ARG, "GGA needs collocation gradients");
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf<double> rho((size_t)nspin * npts), grad((size_t)nspin * 3 * npts), Z((size_t)nspin * nbf * npts), Ed(1);
    for (int sp_i = 0; sp_i < nspin; ++sp_i)
      density_dense_kernel<<<nblk(npts * 32, 256), 256, 0, s>>>(
          nbf, npts, d_phi, gga ? d_gx : nullptr, d_gy, d_gz, nocc, d_C + (size_t)sp_i * nbf * nocc,
          d_occ + (size_t)sp_i * nocc, rho.p + (size_t)sp_i * npts, gga ? grad.p + (size_t)sp_i * 3 * npts : nullptr,
          nullptr);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaMemsetAsync(Ed.p, 0, sizeof(double), s));
    xc_z_dense_kernel<<<nblk(npts, 128), 128, 0, s>>>(sp, gga, nbf, npts, nspin, d_phi, d_gx, d_gy, d_gz, d_w,
                                                     rho.p, grad.p, Z.p, Ed.p);
    NKX_LAUNCH_CHECK();
    for (int sp_i = 0; sp_i < nspin; ++sp_i)
      launch_nt_gemm_sym(nbf, npts, d_phi, Z.p + (size_t)sp_i * nbf * npts, d_V + (size_t)sp_i * nbf * nbf, s);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaMemcpyAsync(E, Ed.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaStreamSynchronize(s));
  });
}

extern "C" nkx_status nkx_potential_collocation(const nkx_basis *aux, const double *d_points, const double *d_w,
                                                long npts, double *d_Vw, void *stream) {
  return run_guarded("nkx_potential_collocation", [&] {
    NKX_REQUIRE(aux && aux->nbf > 0 && npts >= 0 && d_points && d_w && d_Vw, NKX_ERR_ARG, "invalid arguments");
    auto tab = make_aux_table(*aux);
    DevBuf<AuxFunc> df(tab.size());
    cudaStream_t s = (cudaStream_t)stream;
    NKX_CUDA(cudaMemcpyAsync(df.p, tab.data(), tab.size() * sizeof(AuxFunc), cudaMemcpyHostToDevice, s));
    const long tot = (long)aux->nbf * npts;
    if (tot > 0) potential_dense_kernel<<<nblk(tot, 128), 128, 0, s>>>(df.p, aux->nbf, d_points, d_w, npts, d_Vw);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaStreamSynchronize(s));
  });
}

// S(f, g) = Phi(f, g) v(g)
__global__ void scale_columns_kernel(int nbf, long npts, const double *__restrict__ phi, const double *__restrict__ v,
                                     double *__restrict__ S) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e < (long)nbf * npts) S[e] = phi[e] * v[e / nbf];
}

extern "C" nkx_status nkx_coulomb_dense(int nbf, int naux, long npts, const double *d_phi, const double *d_Vw,
                                        const double *d_X, int K, int nocc, const double *d_C, const double *d_occ,
                                        double *d_J, void *stream) {
  return run_guarded("nkx_coulomb_dense", [&] {
    NKX_REQUIRE(nbf > 0 && naux > 0 && npts > 0 && K > 0 && K <= naux && nocc > 0 && d_phi && d_Vw && d_X && d_C &&
                    d_occ && d_J,
                NKX_ERR_ARG, "invalid arguments");
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf<double> rho(npts), y(naux), t(K), c(naux), v(npts), S((size_t)nbf * npts);
    density_dense_kernel<<<nblk(npts * 32, 256), 256, 0, s>>>(nbf, npts, d_phi, nullptr, nullptr, nullptr, nocc, d_C,
                                                              d_occ, rho.p, nullptr, nullptr);
    NKX_LAUNCH_CHECK();
    cublasHandle_t h;
    NKX_REQUIRE(cublasCreate(&h) == CUBLAS_STATUS_SUCCESS, NKX_ERR_CUDA, "cublasCreate failed");
    cublasSetStream(h, s);
    const double one = 1.0, zero = 0.0;
    bool ok = cublasDgemv(h, CUBLAS_OP_N, naux, (int)npts, &one, d_Vw, naux, rho.p, 1, &zero, y.p, 1) ==
              CUBLAS_STATUS_SUCCESS;
    ok = ok && cublasDgemv(h, CUBLAS_OP_T, naux, K, &one, d_X, naux, y.p, 1, &zero, t.p, 1) == CUBLAS_STATUS_SUCCESS;
    ok = ok && cublasDgemv(h, CUBLAS_OP_N, naux, K, &one, d_X, naux, t.p, 1, &zero, c.p, 1) == CUBLAS_STATUS_SUCCESS;
    ok = ok && cublasDgemv(h, CUBLAS_OP_T, naux, (int)npts, &one, d_Vw, naux, c.p, 1, &zero, v.p, 1) ==
                   CUBLAS_STATUS_SUCCESS;
    if (ok) {
      scale_columns_kernel<<<nblk((long)nbf * npts, 256), 256, 0, s>>>(nbf, npts, d_phi, v.p, S.p);
      ok = cudaGetLastError() == cudaSuccess;
    }
    ok = ok && cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, (int)npts, &one, d_phi, nbf, S.p, nbf, &zero, d_J,
                           nbf) == CUBLAS_STATUS_SUCCESS;
    NKX_CUDA(cudaStreamSynchronize(s));
    cublasDestroy(h);
    NKX_REQUIRE(ok, NKX_ERR_CUDA, "cuBLAS call in nkx_coulomb_dense failed");
  });
}

// compute_exact_exchange (nukexc/exact_exchange.hpp:57-119), the reference's
// dense grid RI-K: T = Phi^T C (npts x nocc), then per orbital i
//   B = Phi o T_i (columns scaled), (P|mu i) = Vw B^T (naux x nbf),
//   Y = (P|mu i)^T X (nbf x K),  K += occ_i Y Y^T,
// FP64 cuBLAS GEMMs.  The work is nocc * naux * nbf * npts: small systems.
extern "C" nkx_status nkx_exchange_dense(int nbf, int naux, long npts, const double *d_phi, const double *d_Vw,
                                         const double *d_X, int K, int nocc, const double *d_C, const double *d_occ,
                                         double *d_K, void *stream) {
  return run_guarded("nkx_exchange_dense", [&] {
    NKX_REQUIRE(nbf > 0 && naux > 0 && npts > 0 && K > 0 && K <= naux && nocc > 0 && d_phi && d_Vw && d_X && d_C &&
                    d_occ && d_K,
                NKX_ERR_ARG, "invalid arguments");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<double> occ(nocc);
    NKX_CUDA(cudaMemcpyAsync(occ.data(), d_occ, sizeof(double) * nocc, cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaStreamSynchronize(s));
    DevBuf<double> T((size_t)npts * nocc), B((size_t)nbf * npts), P3((size_t)naux * nbf), Y((size_t)nbf * K);
    cublasHandle_t h;
    NKX_REQUIRE(cublasCreate(&h) == CUBLAS_STATUS_SUCCESS, NKX_ERR_CUDA, "cublasCreate failed");
    cublasSetStream(h, s);
    const double one = 1.0, zero = 0.0;
    bool ok = cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)npts, nocc, nbf, &one, d_phi, nbf, d_C, nbf, &zero, T.p,
                          (int)npts) == CUBLAS_STATUS_SUCCESS;
    ok = ok && cudaMemsetAsync(d_K, 0, sizeof(double) * nbf * nbf, s) == cudaSuccess;
    for (int i = 0; i < nocc && ok; ++i) {
      scale_columns_kernel<<<nblk((long)nbf * npts, 256), 256, 0, s>>>(nbf, npts, d_phi, T.p + (size_t)i * npts,
                                                                        B.p);
      ok = cudaGetLastError() == cudaSuccess;
      ok = ok && cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, naux, nbf, (int)npts, &one, d_Vw, naux, B.p, nbf, &zero,
                             P3.p, naux) == CUBLAS_STATUS_SUCCESS;
      ok = ok && cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nbf, K, naux, &one, P3.p, naux, d_X, naux, &zero, Y.p,
                             nbf) == CUBLAS_STATUS_SUCCESS;
      const double oi = occ[i];
      ok = ok && cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, K, &oi, Y.p, nbf, Y.p, nbf, &one, d_K, nbf) ==
                     CUBLAS_STATUS_SUCCESS;
    }
    NKX_CUDA(cudaStreamSynchronize(s));
    cublasDestroy(h);
    NKX_REQUIRE(ok, NKX_ERR_CUDA, "cuBLAS call in nkx_exchange_dense failed");
  });
}

// per chunk point g: ws[g] = w_g, wv[g] = w_g sum_A Z_A / (|r_g - R_A| + 1e-30)
// (core_hamiltonian.hpp:226-236)
__global__ void core_weights_kernel(const double *__restrict__ pts, const double *__restrict__ w, long n,
                                    const double *__restrict__ centers, const double *__restrict__ Zc, int natoms,
                                    double *__restrict__ wv) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= n) return;
  double v = 0.0;
  for (int a = 0; a < natoms; ++a) {
    const double dx = pts[3 * g] - centers[3 * a], dy = pts[3 * g + 1] - centers[3 * a + 1],
                 dz = pts[3 * g + 2] - centers[3 * a + 2];
    v += Zc[a] / (sqrt(dx * dx + dy * dy + dz * dz) + 1e-30);
  }
  wv[g] = w[g] * v;
}
// out(mu, g) = in(mu, g) * s[g]
__global__ void scale_cols_kernel(int nbf, long n, const double *__restrict__ in, const double *__restrict__ s,
                                  double *__restrict__ out) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e < (long)nbf * n) out[e] = in[e] * s[e / nbf];
}

extern "C" nkx_status nkx_core_hamiltonian_dense(const nkx_basis *basis, const nkx_molecule *mol,
                                                 const double *d_points, const double *d_w, long npts, double *d_S,
                                                 double *d_T, double *d_V, void *stream) {
  return run_guarded("nkx_core_hamiltonian_dense", [&] {
    NKX_REQUIRE(basis && basis->nbf > 0 && mol && mol->natoms > 0 && d_points && d_w && npts > 0 && d_S && d_T && d_V,
                NKX_ERR_ARG, "invalid arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const int nbf = basis->nbf;
    auto tab = make_sto_table(*basis);
    DevBuf<StoFunc> df(tab.size());
    NKX_CUDA(cudaMemcpyAsync(df.p, tab.data(), sizeof(StoFunc) * tab.size(), cudaMemcpyHostToDevice, s));
    std::vector<double> zc(mol->natoms);
    for (int a = 0; a < mol->natoms; ++a) zc[a] = mol->Z[a];
    DevBuf<double> dc(3 * (size_t)mol->natoms), dz(mol->natoms);
    NKX_CUDA(cudaMemcpyAsync(dc.p, mol->xyz, sizeof(double) * 3 * mol->natoms, cudaMemcpyHostToDevice, s));
    NKX_CUDA(cudaMemcpyAsync(dz.p, zc.data(), sizeof(double) * mol->natoms, cudaMemcpyHostToDevice, s));
    // points in chunks holding 6 nbf x chunk matrices in about 1 GiB
    const long chunk = std::max<long>(256, std::min<long>(npts, ((long)1 << 27) / (6L * nbf)));
    DevBuf<double> phi((size_t)nbf * chunk), gx((size_t)nbf * chunk), gy((size_t)nbf * chunk),
        gz((size_t)nbf * chunk), sc((size_t)nbf * chunk), wv(chunk);
    NKX_CUDA(cudaMemsetAsync(d_S, 0, sizeof(double) * nbf * nbf, s));
    NKX_CUDA(cudaMemsetAsync(d_T, 0, sizeof(double) * nbf * nbf, s));
    NKX_CUDA(cudaMemsetAsync(d_V, 0, sizeof(double) * nbf * nbf, s));
    cublasHandle_t h;
    NKX_REQUIRE(cublasCreate(&h) == CUBLAS_STATUS_SUCCESS, NKX_ERR_CUDA, "cublasCreate failed");
    cublasSetStream(h, s);
    bool ok = true;
    const double one = 1.0, half = 0.5, mone = -1.0;
    for (long g0 = 0; g0 < npts && ok; g0 += chunk) {
      const long n = std::min(chunk, npts - g0);
      const long tot = (long)nbf * n;
      colloc_dense_kernel<<<nblk(tot, 128), 128, 0, s>>>(df.p, nbf, d_points + 3 * g0, n, phi.p, gx.p, gy.p, gz.p);
      core_weights_kernel<<<nblk(n, 128), 128, 0, s>>>(d_points + 3 * g0, d_w + g0, n, dc.p, dz.p, mol->natoms, wv.p);
      // S += phi (w phi)^T
      scale_cols_kernel<<<nblk(tot, 256), 256, 0, s>>>(nbf, n, phi.p, d_w + g0, sc.p);
      ok = ok && cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, (int)n, &one, phi.p, nbf, sc.p, nbf, &one, d_S,
                             nbf) == CUBLAS_STATUS_SUCCESS;
      // V -= phi (w v phi)^T
      scale_cols_kernel<<<nblk(tot, 256), 256, 0, s>>>(nbf, n, phi.p, wv.p, sc.p);
      ok = ok && cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, (int)n, &mone, phi.p, nbf, sc.p, nbf, &one, d_V,
                             nbf) == CUBLAS_STATUS_SUCCESS;
      // T += 1/2 sum_k g_k (w g_k)^T
      for (double *gk : {gx.p, gy.p, gz.p}) {
        scale_cols_kernel<<<nblk(tot, 256), 256, 0, s>>>(nbf, n, gk, d_w + g0, sc.p);
        ok = ok && cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, nbf, nbf, (int)n, &half, gk, nbf, sc.p, nbf, &one, d_T,
                               nbf) == CUBLAS_STATUS_SUCCESS;
      }
      ok = ok && cudaGetLastError() == cudaSuccess;
    }
    NKX_CUDA(cudaStreamSynchronize(s));
    cublasDestroy(h);
    NKX_REQUIRE(ok, NKX_ERR_CUDA, "kernel or cuBLAS failure in nkx_core_hamiltonian_dense");
  });
}

extern "C" nkx_status nkx_half_inverse(int N, const double *d_S, double thr, double *d_X, int *K, void *stream) {
  return run_guarded("nkx_half_inverse", [&] {
    NKX_REQUIRE(N > 0 && d_S && d_X && K, NKX_ERR_ARG, "invalid arguments");
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf<double> A((size_t)N * N), D(N), lam(N);
    DevBuf<int> info(1);
    dim3 tb(16, 16), gb(nblk(N, 16), nblk(N, 16));
    precondition_kernel<<<gb, tb, 0, s>>>(N, d_S, A.p, D.p);
    NKX_LAUNCH_CHECK();
    cusolverDnHandle_t h;
    NKX_REQUIRE(cusolverDnCreate(&h) == CUSOLVER_STATUS_SUCCESS, NKX_ERR_CUDA, "cusolverDnCreate failed");
    cusolverDnSetStream(h, s);
    int lwork = 0;
    cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, N, A.p, N, lam.p, &lwork);
    DevBuf<double> work(lwork > 0 ? lwork : 1);
    const cusolverStatus_t st =
        cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, N, A.p, N, lam.p, work.p, lwork, info.p);
    cusolverDnDestroy(h);
    NKX_REQUIRE(st == CUSOLVER_STATUS_SUCCESS, NKX_ERR_CUDA, "cusolverDnDsyevd failed");
    std::vector<double> hl(N), hU((size_t)N * N), hD(N);
    NKX_CUDA(cudaMemcpyAsync(hl.data(), lam.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaMemcpyAsync(hU.data(), A.p, sizeof(double) * N * N, cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaMemcpyAsync(hD.data(), D.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaStreamSynchronize(s));
    // singular values of a symmetric matrix are |eigenvalues|; keep s > thr,
    // largest first (the reference's SVD ordering)
    std::vector<int> order(N);
    for (int i = 0; i < N; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return fabs(hl[a]) > fabs(hl[b]); });
    std::vector<double> hX((size_t)N * N, 0.0);
    int k = 0;
    for (int oi = 0; oi < N; ++oi) {
      const int e = order[oi];
      const double sv = fabs(hl[e]);
      if (!(sv > thr)) continue;
      for (int i = 0; i < N; ++i) hX[(size_t)i + (size_t)k * N] = hU[(size_t)i + (size_t)e * N] / sqrt(sv) / hD[i];
      ++k;
    }
    NKX_CUDA(cudaMemcpyAsync(d_X, hX.data(), sizeof(double) * N * N, cudaMemcpyHostToDevice, s));
    NKX_CUDA(cudaStreamSynchronize(s));
    *K = k;
  });
}

// ---------------------------------------------------------------------------
// nkx_xc_dense_noalloc: the dense XC build of nkx_xc_dense for callers that
// must not allocate device memory.  Some host programs hand (almost) all of
// the GPU's memory to their own pool allocator when they start, so a
// cudaMalloc from a library would fail or fragment that pool; others run the
// Fock build inside a latency-critical loop where cudaMalloc / cudaFree,
// which synchronise the whole device, are not acceptable.  This entry point
// keeps its scratch (energy accumulator, per-point density and gradient, the
// Z matrix) in one file-scope __device__ array of kNoAllocScratchDoubles
// doubles (32 MiB), which every GPU that loads the library holds until the
// process exits, and it calls no cudaMalloc, cudaFree or allocating library
// routine.
//
// In host code the array's name is only a host-side stand-in, never a device
// address, so the first call made on a device (with that device current)
// looks the address up with cudaGetSymbolAddress and remembers it for that
// device; that first call should come before any stream capture.  The
// remembered address belongs to the device's current context: the library
// must not be used across a cudaDeviceReset.  Every call shares the array and
// finds the previous call's contents there, so everything that must start at
// zero is cleared by the call itself; calls whose work overlaps on the GPU
// (other streams, other host threads) race on the array and must be
// serialised by the caller.  Problems that need more scratch than the array
// holds are rejected with NKX_ERR_ARG before anything is launched.
// ---------------------------------------------------------------------------
#include <mutex>

namespace nkx {

constexpr size_t kNoAllocScratchDoubles = (size_t)4 << 20;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

static double *noalloc_scratch_address() {
  static std::mutex mu;
  static double *addr[128] = {nullptr};
  int dev = 0;
  NKX_CUDA(cudaGetDevice(&dev));
  NKX_REQUIRE(dev >= 0 && dev < 128, NKX_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    NKX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    addr[dev] = static_cast<double *>(p);
  }
  return addr[dev];
}

}  // namespace nkx

extern "C" nkx_status nkx_xc_dense_noalloc(int nbf, long npts, const double *d_phi, const double *d_gx,
                                           const double *d_gy, const double *d_gz, const double *d_w, int nspin,
                                           int nocc, const double *d_C, const double *d_occ,
                                           const nkx_plan_options *opts, double *E, double *d_V, void *stream) {
  return run_guarded("nkx_xc_dense_noalloc", [&] {
    NKX_REQUIRE(nbf > 0 && npts > 0 && (nspin == 1 || nspin == 2) && nocc > 0 && d_phi && d_w && d_C && d_occ &&
                    E && d_V,
                NKX_ERR_ARG, "invalid arguments");
    const XcSpec sp = make_spec(opts);
    const bool gga = spec_is_gga(sp);
    NKX_REQUIRE(!gga || (d_gx && d_gy && d_gz), NKX_ERR_ARG, "GGA needs collocation gradients");
    // layout in doubles, each piece 256-byte aligned: E | rho | grad | Z.
    // npts is bounded first, so the products below cannot wrap around.
    const size_t per_point = (size_t)nspin * ((size_t)nbf + 4);
    const std::string too_large =
        "problem too large for the fixed 32 MiB scratch: needs about nspin*npts*(nbf+4) doubles <= 4194304";
    NKX_REQUIRE((size_t)npts <= kNoAllocScratchDoubles / per_point, NKX_ERR_ARG,
                too_large + " (nspin " + std::to_string(nspin) + ", npts " + std::to_string(npts) + ", nbf " +
                    std::to_string(nbf) + ")");
    auto up = [](size_t n) { return (n + 31) & ~(size_t)31; };
    const size_t nE = 32, nrho = up((size_t)nspin * npts), ngrad = up((size_t)nspin * 3 * npts);
    const size_t nZ = up((size_t)nspin * nbf * npts);
    const size_t need = nE + nrho + ngrad + nZ;
    NKX_REQUIRE(need <= kNoAllocScratchDoubles, NKX_ERR_ARG, too_large + " (" + std::to_string(need) + " requested)");
    double *base = noalloc_scratch_address();
    double *Ed = base, *rho = base + nE, *grad = rho + nrho, *Z = grad + ngrad;
    cudaStream_t s = (cudaStream_t)stream;
    for (int sp_i = 0; sp_i < nspin; ++sp_i)
      density_dense_kernel<<<nblk(npts * 32, 256), 256, 0, s>>>(
          nbf, npts, d_phi, gga ? d_gx : nullptr, d_gy, d_gz, nocc, d_C + (size_t)sp_i * nbf * nocc,
          d_occ + (size_t)sp_i * nocc, rho + (size_t)sp_i * npts, gga ? grad + (size_t)sp_i * 3 * npts : nullptr,
          nullptr);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaMemsetAsync(Ed, 0, sizeof(double), s));  // the array keeps the previous call's sum
    xc_z_dense_kernel<<<nblk(npts, 128), 128, 0, s>>>(sp, gga, nbf, npts, nspin, d_phi, d_gx, d_gy, d_gz, d_w,
                                                     rho, grad, Z, Ed);
    NKX_LAUNCH_CHECK();
    for (int sp_i = 0; sp_i < nspin; ++sp_i)
      launch_nt_gemm_sym(nbf, npts, d_phi, Z + (size_t)sp_i * nbf * npts, d_V + (size_t)sp_i * nbf * nbf, s);
    NKX_LAUNCH_CHECK();
    NKX_CUDA(cudaMemcpyAsync(E, Ed, sizeof(double), cudaMemcpyDeviceToHost, s));
    NKX_CUDA(cudaStreamSynchronize(s));
  });
}
