/*
 * nkx.h -- C ABI of the B200-native grid-integration Fock build.
 *
 * Plain pointers and sizes only.  Every function returns an nkx_status and
 * never throws across the boundary.  "Device" pointers are CUDA device
 * pointers of the current device; "stream" is a cudaStream_t passed as
 * void* (NULL = legacy default stream).  Matrices are column-major
 * (Kokkos LayoutLeft in the reference): element (i, j) of an R x C matrix
 * is at i + j*R.
 *
 * Each entry point names the NuKEXC interface it replaces (paths relative
 * to the NuKEXC project root).
 */
#ifndef NKX_H
#define NKX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define NKX_API __declspec(dllexport)
#else
#define NKX_API __attribute__((visibility("default")))
#endif

typedef int nkx_status;
enum {
  NKX_OK = 0,
  NKX_ERR_ARG = 1,         /* invalid argument (reference: std::runtime_error) */
  NKX_ERR_ALLOC = 2,       /* device or host allocation failed */
  NKX_ERR_CUDA = 3,        /* a CUDA runtime / library call failed */
  NKX_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
  NKX_ERR_NUMERIC = 5,     /* non-positive metric, negative grid weight, NaN */
  NKX_ERR_UNSUPPORTED = 6  /* functional id, angular momentum or size not supported */
};

/* Precision of the dense contractions (the density and the V = Phi Z^T
 * contraction).  FP64: plain FP64 kernels.  MIXED: every operand row is
 * scaled by a power of two and rounded to a 31-bit integer held as four
 * int8 digits; the products run as tcgen05 kind::i8 tensor-core MMAs with
 * exact int32 accumulation per grid batch, combined in FP64 across batches
 * (relative error about 1e-9 of the row maxima). */
enum { NKX_PREC_FP64 = 0, NKX_PREC_MIXED = 1 };

/* Radial quadratures (IntegratorXX Becke / TreutlerAhlrichs, nukexc/grid.hpp:172-305) */
enum { NKX_RADIAL_BECKE = 0, NKX_RADIAL_TA = 1 };
/* Per-element radial sizing (nukexc/grid.hpp:129-148) */
enum { NKX_SIZING_UNIFORM = 0, NKX_SIZING_PYSCF = 1 };

/* libxc functional ids supported on the device (libxc numbering) */
enum {
  NKX_XC_LDA_X = 1,
  NKX_XC_LDA_C_VWN = 7, /* VWN5 */
  NKX_XC_LDA_C_PW = 12,     /* Perdew-Wang 92, published constants */
  NKX_XC_LDA_C_PW_MOD = 13, /* Perdew-Wang 92, constants as used inside PBE correlation */
  NKX_XC_GGA_X_PBE = 101,
  NKX_XC_GGA_C_PBE = 130
};

/* Memory space of the caller's buffers for nkx_fock_build */
enum { NKX_MEM_DEVICE = 0, NKX_MEM_HOST = 1 };

/* Molecule (nukexc/molecule.hpp:50-93): natoms centres in bohr, xyz[3*natoms] */
typedef struct {
  int natoms;
  const double *xyz;
  const int *Z;
} nkx_molecule;

/* STO basis in SoA form (STOBasisSet, nukexc/stobasis.hpp:54-64): one entry
 * per function; center[3*nbf] in bohr.  The normalisation
 * N = (2 zeta)^(n+1/2) / sqrt((2n)!) and the cutoff radius at cutoff_tol
 * are computed by the library (make_manual_basis, stobasis.hpp:175-225). */
typedef struct {
  int nbf;
  const int *n, *l, *m;
  const double *zeta;
  const double *center;
  double cutoff_tol; /* reference default 1e-10 */
} nkx_basis;

/* make_flat_grid parameters (nukexc/grid.hpp:172-181) */
typedef struct {
  int radial_scheme;       /* NKX_RADIAL_* */
  int nrad;                /* radial points (H/He count for PySCF sizing) */
  int nang_order;          /* Lebedev algebraic order requested (next available is used) */
  double weight_threshold; /* drop points with w <= threshold after Becke */
  double ta_alpha;         /* Treutler-Ahlrichs exponent (0.6 = M4) */
  int sizing;              /* NKX_SIZING_* */
  double becke_clamp;      /* Laqua clamp of R_ij in bohr (5.0); <= 0: original Becke */
} nkx_grid_spec;

/* Plan options */
typedef struct {
  int batch_points;        /* points per grid batch; 256 */
  double screen_tol;       /* basis cutoff tolerance for batch screening (1e-10) */
  int nfunc;               /* number of functional ids summed (1..4) */
  int func_ids[4];         /* NKX_XC_* */
  double dens_threshold;   /* points with rho < threshold give no XC contribution */
  size_t workspace_bytes;  /* device workspace for streamed batch chunks; 0 = auto */
  double metric_svd_thr;   /* 0: FP64 Cholesky of (A|B); > 0: the reference's preconditioned
                              half inverse keeping singular values > thr (nukexc_utils.hpp:198-270) */
} nkx_plan_options;

typedef struct nkx_plan nkx_plan;

typedef struct {
  long npoints;            /* grid points after compaction */
  long nbatches;
  int nbf, naux, nblocks;  /* nblocks = ceil(nbf / 128) function blocks */
  long npairs;             /* significant (batch, function block) pairs */
  int nchunks;             /* batch chunks streamed per pass */
  double metric_min_diag;  /* smallest diagonal of the Cholesky factor of (A|B) */
  long graph_replays;      /* builds replayed from a CUDA graph so far (nkx_plan_set_graph) */
} nkx_plan_info;

/* Timing of the last nkx_fock_build, per stage, in milliseconds (CUDA events). */
typedef struct {
  float colloc_ms, density_ms, functional_ms, coulomb_ms, zbuild_ms, vgemm_ms, total_ms;
  int launches;            /* kernels launched by the build */
} nkx_build_timing;

/* ---------------------------------------------------------------- grid -- */

/* make_flat_grid (nukexc/grid.hpp:172-348): per-atom radial x Lebedev
 * grids, Becke partition on the device (partition_becke_team,
 * nukexc/partitioning.hpp:126-213), compaction of w <= threshold keeping the
 * original order.  Two-call pattern: pass xyz == NULL to get *npoints, then
 * host buffers xyz[3*npoints], w[npoints], owner[npoints]. */
NKX_API nkx_status nkx_make_flat_grid(const nkx_molecule *mol, const nkx_grid_spec *spec, long *npoints,
                                      double *xyz, double *w, int *owner);

/* partition_becke_team / partition_becke (nukexc/partitioning.hpp:63-213)
 * on device buffers: weights[g] *= P_owner(g) / sum_i P_i.  clamp > 0 is the
 * Laqua-clamped team variant (R_ij = min(|A_i - A_j|, clamp)), clamp <= 0 the
 * original Becke.  centers[3*natoms], points[3*npts] (AoS, like
 * Kokkos::View<Point*>). */
NKX_API nkx_status nkx_becke_partition(const double *d_centers, int natoms, const double *d_points,
                                       const int *d_owner, long npts, double *d_weights, double clamp,
                                       void *stream);

/* ----------------------------------------------------- dense reference API */

/* fill_collocation / fill_grad_collocation (nukexc/stobasis.hpp:494-584):
 * Phi (nbf x npts column-major) and optionally its gradient (d_gx == NULL
 * skips it) at device points[3*npts]. */
NKX_API nkx_status nkx_fill_collocation(const nkx_basis *basis, const double *d_points, long npts,
                                        double *d_phi, double *d_gx, double *d_gy, double *d_gz,
                                        void *stream);

/* compute_density_and_sigma (nukexc/density.hpp:188-255) and
 * compute_density (:150-186) on dense collocation matrices.  C is
 * nbf x nocc column-major, occ[nocc].  rho[npts]; d_grad (3*npts, x|y|z
 * planes) and d_sigma may be NULL (then the gradient inputs may be NULL). */
NKX_API nkx_status nkx_density_dense(int nbf, long npts, const double *d_phi, const double *d_gx,
                                     const double *d_gy, const double *d_gz, int nocc, const double *d_C,
                                     const double *d_occ, double *d_rho, double *d_grad, double *d_sigma,
                                     void *stream);

/* compute_lda / compute_gga (nspin 1) and compute_lsda / compute_gga_lsda
 * (nspin 2) (nukexc/xc_integrals.hpp:73-726) on dense collocation: C and occ
 * hold nspin blocks (nbf x nocc, nocc).  The functional ids of `opts` are
 * summed.  E_xc is written to *E (host).  d_V receives nspin symmetric
 * nbf x nbf matrices. */
NKX_API nkx_status nkx_xc_dense(int nbf, long npts, const double *d_phi, const double *d_gx,
                                const double *d_gy, const double *d_gz, const double *d_w, int nspin,
                                int nocc, const double *d_C, const double *d_occ, const nkx_plan_options *opts,
                                double *E, double *d_V, void *stream);

/* The dense XC build of nkx_xc_dense for callers that must not allocate
 * device memory: host programs that give (almost) all GPU memory to their
 * own pool allocator at start-up, where a library cudaMalloc would fail or
 * fragment the pool, and latency-critical loops that cannot take the
 * device-wide synchronisation of cudaMalloc / cudaFree.  No counterpart in
 * the reference.  Same arguments and results as nkx_xc_dense; it calls no
 * cudaMalloc, cudaFree or allocating library routine.  Its scratch is one
 * fixed array of NKX_NOALLOC_SCRATCH_DOUBLES doubles (32 MiB) in the
 * library's device memory, held by every GPU that loads the library until
 * the process exits; problems with
 * 32 + pad(nspin*npts) + pad(3*nspin*npts) + pad(nspin*nbf*npts) > that
 * (pad = round up to 32; about nspin*npts*(nbf+4)) are rejected with
 * NKX_ERR_ARG before any work is launched.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) and should come before
 * any stream capture; the library must not be used across a
 * cudaDeviceReset.  All calls share the array and each clears what must
 * start at zero: calls that overlap on the GPU race on it and must be
 * serialised by the caller. */
#define NKX_NOALLOC_SCRATCH_DOUBLES (4u << 20)
NKX_API nkx_status nkx_xc_dense_noalloc(int nbf, long npts, const double *d_phi, const double *d_gx,
                                        const double *d_gy, const double *d_gz, const double *d_w, int nspin,
                                        int nocc, const double *d_C, const double *d_occ,
                                        const nkx_plan_options *opts, double *E, double *d_V, void *stream);

/* Functional evaluation with libxc's array layouts (xc_lda_exc_vxc /
 * xc_gga_exc_vxc, the host calls of nukexc/xc_integrals.hpp:113-617), on the
 * device: nspin 1: rho[n], sigma[n]; nspin 2: rho[2n], sigma[3n]
 * interleaved.  exc per particle.  sigma/vsigma may be NULL for LDA. */
NKX_API nkx_status nkx_xc_eval(int func_id, int nspin, long n, const double *d_rho, const double *d_sigma,
                               double dens_threshold, double *d_exc, double *d_vrho, double *d_vsigma,
                               void *stream);

/* sto_potential_collocation_scaled (nukexc/stopotential.hpp:101-124):
 * Vw(alpha, g) = V_alpha(r_g) w_g, naux x npts column-major. */
NKX_API nkx_status nkx_potential_collocation(const nkx_basis *aux, const double *d_points, const double *d_w,
                                             long npts, double *d_Vw, void *stream);

/* compute_coulomb (nukexc/coulomb.hpp:56-115) on dense matrices: rho from
 * Phi (nbf x npts) and C (nbf x nocc), y = Vw rho (Vw naux x npts), c = X X^T y
 * (X naux x K), v = Vw^T c, J = Phi diag(v) Phi^T (nbf x nbf column-major).
 * All pointers are device buffers. */
NKX_API nkx_status nkx_coulomb_dense(int nbf, int naux, long npts, const double *d_phi, const double *d_Vw,
                                     const double *d_X, int K, int nocc, const double *d_C, const double *d_occ,
                                     double *d_J, void *stream);

/* compute_exact_exchange (nukexc/exact_exchange.hpp:57-119), the grid RI-K
 * of the reference's dense path: T = Phi^T C, and per occupied orbital i
 * (P|mu i) = sum_g Vw(P, g) phi_mu(g) T_i(g), Y_i = (P|mu i)^T X,
 * K = sum_i occ_i Y_i Y_i^T.  Same operands as nkx_coulomb_dense (column-major
 * device arrays; d_K nbf x nbf).  FP64 cuBLAS; nocc * naux * nbf * npts work. */
NKX_API nkx_status nkx_exchange_dense(int nbf, int naux, long npts, const double *d_phi, const double *d_Vw,
                                      const double *d_X, int K, int nocc, const double *d_C, const double *d_occ,
                                      double *d_K, void *stream);

/* compute_core_hamiltonian (nukexc/core_hamiltonian.hpp:133-289) by
 * quadrature on device points/weights: S = sum_g w phi phi^T,
 * T = 1/2 sum_g w grad phi . grad phi^T, V = -sum_g w (sum_A Z_A / |r - R_A|) phi phi^T
 * (nbf x nbf column-major device outputs; mol holds host centres and charges). */
NKX_API nkx_status nkx_core_hamiltonian_dense(const nkx_basis *basis, const nkx_molecule *mol,
                                              const double *d_points, const double *d_w, long npts, double *d_S,
                                              double *d_T, double *d_V, void *stream);

/* The quadrature core Hamiltonian of nkx_core_hamiltonian_dense over a plan's
 * screened batches: only (batch, 128-function block) pairs with the block
 * significant are integrated, as the reference's screened variants do
 * (compute_core_hamiltonian_screened / _scratch / _tiled / _sparse,
 * nukexc/core_hamiltonian.hpp:320-1155).  FP64.  S, T, V (nbf x nbf,
 * column-major; mem: host or device buffers); mol holds host centres and
 * charges. */
NKX_API nkx_status nkx_plan_core_hamiltonian(nkx_plan *plan, const nkx_molecule *mol, double *S, double *T, double *V,
                                             int mem, void *stream);

/* compute_half_inverse (nukexc/nukexc_utils.hpp:198-270): X = U s^-1/2 / D
 * of the preconditioned metric, keeping s > thr (symmetric
 * eigendecomposition on the device).  d_X must hold N*N; *K receives the
 * kept column count. */
NKX_API nkx_status nkx_half_inverse(int N, const double *d_S, double thr, double *d_X, int *K, void *stream);

/* ---------------------------------------------------------------- plan -- */

/* Once per geometry: Morton-ordered 256-point batches of the given grid
 * (create_bounding_boxes, nukexc/octree.hpp:70-141), screening of basis
 * function blocks per batch (build_neighbor_list, :317-390), the aux metric
 * (A|B) on the grid and its FP64 Cholesky factor (replaces the SVD half
 * inverse of nukexc/nukexc_utils.hpp:198-270; aux may be NULL for XC only).
 * The caller's grid arrays (host) are copied, never permuted. */
NKX_API nkx_status nkx_plan_create(const nkx_molecule *mol, const nkx_basis *prim, const nkx_basis *aux,
                                   long npoints, const double *xyz, const double *w, const int *owner,
                                   const nkx_plan_options *opts, nkx_plan **plan);

NKX_API nkx_status nkx_plan_get_info(const nkx_plan *plan, nkx_plan_info *info);

/* One Fock build (the per-SCF-iteration work of tests/standalone.cxx:572-846):
 * E_xc and V_xc (compute_gga / compute_gga_lsda ...) and, when the plan
 * has an aux basis and J != NULL, the grid-integrated RI-J
 * (compute_coulomb, nukexc/coulomb.hpp:56-115).
 *   nspin 1: C = nbf x nocc, occ[nocc]; V = nbf x nbf.
 *   nspin 2: C = 2 blocks (alpha, beta), occ = 2 blocks; V = 2 matrices;
 *            J is built from the total density.
 * mem selects whether C/occ/V/J are host or device buffers (host buffers
 * are copied inside the call).  With fuse_j != 0 (and nspin 1), J is folded
 * into the XC contraction and V receives V_xc + J (J may then be NULL).
 * V may be NULL when J is given and fuse_j == 0: J alone is returned
 * (compute_coulomb and its sparse / tiled variants).
 * E_xc is written to host *E.  The call is synchronous on return. */
NKX_API nkx_status nkx_fock_build(nkx_plan *plan, int precision, int nspin, int nocc, const double *C,
                                  const double *occ, int mem, int fuse_j, double *E, double *V, double *J,
                                  void *stream);

/* Two-phase Fock build for a grid sharded over ranks (one process per GPU,
 * one plan per rank made from the points that rank integrates).  The grid
 * RI-J fit (nukexc/coulomb.hpp:84-95) needs the whole grid's fit vector
 * y = Vw rho before any potential, so the build is split around that
 * exchange, which the caller performs (e.g. ncclAllReduce on `stream`):
 *   phase 1: C and occ in (as nkx_fock_build), the density pass, and this
 *            rank's share of y (naux doubles) written to y;
 *   caller:  y_total = sum of y over the ranks;
 *   phase 2: y_total in; c = (A|B)^-1 y_total with the plan's metric (set it
 *            to the all-reduced full-grid metric with nkx_plan_set_metric),
 *            the functional, V and J on this rank's points.  E, V, J as in
 *            nkx_fock_build are this rank's partial sums, to be all-reduced.
 * Phase 2 must follow phase 1 on the same plan; it reuses phase 1's
 * precision, spin count and orbitals.  y and the outputs follow `mem`.
 * No counterpart in the reference (a single device). */
NKX_API nkx_status nkx_fock_build_phase1(nkx_plan *plan, int precision, int nspin, int nocc, const double *C,
                                         const double *occ, int mem, double *y, void *stream);
NKX_API nkx_status nkx_fock_build_phase2(nkx_plan *plan, const double *y, int mem, int fuse_j, double *E, double *V,
                                         double *J, void *stream);

/* Replace the plan's Coulomb metric (A|B) (naux x naux, symmetric,
 * column-major; mem: host or device) and factor it again the way the plan
 * was created (pivoted Cholesky, or the half inverse when metric_svd_thr > 0;
 * a half inverse set with nkx_plan_set_half_inverse is dropped).  For a
 * sharded grid this is the sum over ranks of nkx_plan_aux_metric. */
NKX_API nkx_status nkx_plan_set_metric(nkx_plan *plan, const double *S, int mem);

/* Choices of the mixed-precision build that nkx_plan_autotune measures. */
typedef struct {
  int v_n;            /* tcgen05 MMA width N of the V contraction: 128 or 64 */
  int dens_n;         /* MMA width of the density contractions (T0 and the GGA Y pass): 64, 128, or 0 (128 from 1024 orbitals on) */
  int ypath;          /* GGA density gradient through Y = T0 (C occ)^T: -1 auto (from 256 orbitals), 0, 1 */
  int v_warps;        /* epilogue warps a CTA of the V contraction: 16 or 8 (N = 128 on one CTA: 32 or 64 columns
                         each; CTA pairs: 16 or 32) */
  int v_pair;         /* 1: V on clusters of two CTAs (tcgen05 cta_group::2, M = 256 x N = 64, double-buffered
                         accumulators; v_n unused), 0: one CTA per output tile */
  long chunk_pairs;   /* (batch, block) pairs per streamed chunk */
  int from_cache;     /* out: 1 when the choices came from the cache file */
  int trials;         /* out: builds timed */
  float default_ms;   /* out: build time with the choices the plan had before */
  float best_ms;      /* out: build time with the chosen ones */
} nkx_tuning;

/* Autotuner of the mixed-precision build (no counterpart in the reference:
 * its kernels take fixed launch shapes).  With the caller's orbitals (as
 * nkx_fock_build, XC only), it times whole builds (CUDA events) and keeps, one
 * knob at a time with the others at their best so far: the Y path (GGA), the
 * density MMA width, the V MMA width and epilogue warps, and the chunk size (x1, x2, x4 of the
 * current one while device memory allows).  With cache_path != NULL a file of
 * earlier results keyed by the device and the problem's shape (functions,
 * blocks, pairs, points, orbitals, spins, GGA) is read first -- a hit applies
 * its choices without timing -- and the new result is appended.  *out (may be
 * NULL) receives the choices and timings.  The plan keeps the choices for
 * all later mixed builds. */
NKX_API nkx_status nkx_plan_autotune(nkx_plan *plan, int nspin, int nocc, const double *C, const double *occ, int mem,
                                     const char *cache_path, nkx_tuning *out, void *stream);
NKX_API nkx_status nkx_plan_get_tuning(const nkx_plan *plan, nkx_tuning *out);
/* Apply choices (for example a stored autotune result); chunk_pairs <= 0 keeps the chunking. */
NKX_API nkx_status nkx_plan_set_tuning(nkx_plan *plan, const nkx_tuning *t);

/* XC nuclear gradient at fixed orbitals (no counterpart in the reference):
 * grad[3*natoms] (host, Eh/bohr) = dE_xc/dR of
 * E_xc = sum_g w_g f(rho(r_g)) with every grid point moving with its owner
 * atom and the Becke weights differentiated (becke_clamp as in
 * nkx_becke_partition; the plan's weights must be radial x angular weights
 * times that Becke partition).  The plan must have been created with the
 * molecule and the point owners, with every basis function centred on an
 * atom.  C / occ as in nkx_fock_build (mem selects host or device).
 * precision: NKX_PREC_FP64 (everything in FP64), or NKX_PREC_MIXED (B200:
 * the orbital values T = C^T Phi and grad Phi, and with them the density,
 * come from the int8-digit tensor-core contraction of the mixed Fock build;
 * the pair terms, STO Hessians and the Becke term stay FP64). */
NKX_API nkx_status nkx_xc_gradient(nkx_plan *plan, int precision, int nspin, int nocc, const double *C,
                                   const double *occ, int mem, double becke_clamp, double *grad, void *stream);

NKX_API nkx_status nkx_get_last_timing(const nkx_plan *plan, nkx_build_timing *t);

/* Per-point density of the last build (rho[npoints*nspin], plan point order
 * = Morton order) and the plan's permutation perm[npoints] (plan point p is
 * caller point perm[p]); host buffers. */
NKX_API nkx_status nkx_plan_last_density(const nkx_plan *plan, double *rho, long *perm);

/* Number of significant 128-function blocks of every batch (counts[nbatches]). */
NKX_API nkx_status nkx_plan_batch_blocks(const nkx_plan *plan, int *counts);

/* Replace the plan's functional (the ids and density threshold of
 * nkx_plan_options) for the following builds: the reference evaluates one
 * libxc functional per call (compute_lsda_sparse / compute_gga_lsda_sparse,
 * nukexc/xc_integrals.hpp:263-264, :728-729). */
NKX_API nkx_status nkx_plan_set_functional(nkx_plan *plan, int nfunc, const int *func_ids, double dens_threshold);

/* Use the caller's half inverse X (naux x K, column-major; mem selects host
 * or device) for the J fit c = X X^T y of the following builds, as
 * compute_coulomb_sparse / _tiled take half_inverse_X
 * (nukexc/coulomb.hpp:117-121, :383-387). */
NKX_API nkx_status nkx_plan_set_half_inverse(nkx_plan *plan, int K, const double *X, int mem);

/* CUDA-graph replay of the Fock build (no counterpart in the reference; the
 * reference's driver launches every kernel of every build from the host).
 * With enable != 0, builds with device buffers (NKX_MEM_DEVICE, phase 0) of
 * one kind -- precision, spin count, orbital count, J mode -- are recorded
 * into a CUDA graph on their second call and replayed from then on: the
 * orbitals are copied into the graph's own buffers and V / J out of them
 * around one graph launch, so the caller may pass other buffers each time,
 * as an SCF loop on the device does.  Any other build, or any change of the
 * plan (functional, metric, half inverse, wait limit, tuning, chunking),
 * drops the graphs; a kind that cannot be recorded keeps running ordinary
 * builds.  Replays record no stage times (nkx_get_last_timing gives the
 * total); nkx_plan_info.graph_replays counts them. */
NKX_API nkx_status nkx_plan_set_graph(nkx_plan *plan, int enable);

/* Limit, in nanoseconds, of the device-side waits of the plan's tensor-core
 * kernels that may be abandoned (0 restores the default of 2 s).  When such a
 * wait runs out, the kernel stops issuing work, waits for the copies and MMAs
 * it has already issued (those drain waits keep a fixed 2 s limit), frees its
 * tensor memory and returns; the build then fails with NKX_ERR_TIMEOUT and
 * the plan stays usable for the next build.  stall != 0 exists to test that
 * path: each tensor-core kernel of the following mixed builds first waits on
 * a barrier that nothing completes, so it gives up after `ns`; stall = 0
 * restores normal builds.  No counterpart in the reference (its kernels have
 * no device waits). */
NKX_API nkx_status nkx_plan_set_wait_limit(nkx_plan *plan, unsigned long long ns, int stall);

/* The plan's grid Coulomb metric (A|B) (naux x naux, symmetrised),
 * coulomb_overlap_integral_sparse (nukexc/coulomb.hpp:691-813); mem selects
 * host or device output. */
NKX_API nkx_status nkx_plan_aux_metric(const nkx_plan *plan, double *S, int mem);

/* Density on the plan's grid in the caller's point order, FP64
 * (compute_density_sparse, nukexc/density.hpp:97-148, and
 * compute_density_and_sigma_sparse, :261-328): rho[nspin][npoints],
 * grad[nspin][3][npoints], sigma[nspin][npoints] = |grad rho_s|^2; any of the
 * three may be NULL.  With accumulate != 0, rho and grad are added to the
 * buffers' contents (the reference's contract) and sigma is formed from the
 * summed gradient.  C / occ / outputs as in nkx_fock_build (mem). */
NKX_API nkx_status nkx_plan_density(nkx_plan *plan, int nspin, int nocc, const double *C, const double *occ, int mem,
                                    int accumulate, double *rho, double *grad, double *sigma, void *stream);

/* ------------------------------------------------------ sparse set-up -- */

/* Morton (Z-order) permutation of npoints host points xyz[3*npoints]:
 * perm[k] = input index of the k-th point (create_bounding_boxes,
 * nukexc/octree.hpp:70-110; the order the plans use). */
NKX_API nkx_status nkx_morton_order(long npoints, const double *xyz, long *perm);

/* build_neighbor_list (nukexc/octree.hpp:317-390) on the device: box b is
 * boxes[6b .. 6b+5] = (min x, y, z, max x, y, z); function f is the sphere
 * (centers[3f..3f+2], radii[f]).  offsets[nboxes+1] and neighbors[] are the
 * CSR of the functions meeting each box, ascending within a box.  Two-call
 * pattern: with neighbors == NULL the offsets are written and *nnz = list
 * length; then call again with a neighbors buffer of *nnz entries. */
NKX_API nkx_status nkx_neighbor_list(int nfunc, const double *d_centers, const double *d_radii, long nboxes,
                                     const double *d_boxes, int *d_offsets, int *d_neighbors, long *nnz,
                                     void *stream);

/* Grid Coulomb metric (A|B) = (M + M^T)/2, M_AB = sum_g phi_A(g) w_g V_B(g),
 * of an aux basis on npoints device points d_xyz[3*npoints] with weights
 * d_w, into d_S (naux x naux, device), FP64
 * (coulomb_overlap_integral_sparse / _tiled, nukexc/coulomb.hpp:691-958). */
NKX_API nkx_status nkx_aux_metric(const nkx_basis *aux, long npoints, const double *d_xyz, const double *d_w,
                                  double *d_S, void *stream);

NKX_API nkx_status nkx_plan_destroy(nkx_plan *plan);

/* Message of the last failed call on this thread (static storage). */
NKX_API const char *nkx_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* NKX_H */
