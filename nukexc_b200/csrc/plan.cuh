// The plan object behind nkx_plan (internal).
#pragma once

#include <cstdint>
#include <vector>

#include "functionals.cuh"
#include "potential.cuh"

namespace nkx {

struct Chunk {
  long b0 = 0, b1 = 0;  // batch range
  long p0 = 0, p1 = 0;  // (batch, block) pair range
  long t0 = 0, t1 = 0;  // range of the chunk's V output tiles in d_vtiles
  long u0 = 0, u1 = 0;  // range of its V pair tiles (row blocks 2R, 2R + 1) in d_vtiles2
};

// Choices of the mixed-precision build that the autotuner (nkx_plan_autotune)
// measures; the defaults are what it found best on (H2O)_64.
struct Tuning {
  int v_n = 128;   // tcgen05 MMA width N of the V contraction (128 or 64)
  int dens_n = 0;  // MMA width of the density contraction (64, 128, or 0: by orbital count, density_width)
  int ypath = -1;  // GGA density gradient through Y = T0 (C occ)^T: -1 from 256 orbitals, 0 off, 1 on
  int v_warps = 16; // epilogue warps of the N = 128 V contraction (16 of 32 columns, or 8 of 64)
  // V on CTA pairs (M = 256 x N = 64, double-buffered TMEM, v_warps
  // epilogue warps a CTA) instead of one CTA per tile
  int v_pair = 0;
};

// A Fock build recorded into a CUDA graph (graph mode) with the buffers it
// reads its orbitals from and writes its results to.
struct BuildGraph {
  int precision = 0, nspin = 0, nocc = 0, fuse = 0;
  bool hasV = false, hasJ = false, failed = false;
  cudaGraphExec_t exec = nullptr;
  double *C = nullptr, *occ = nullptr, *V = nullptr, *J = nullptr;
  int launches = 0;
};

struct Plan {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  std::vector<void *> allocs;
  void *cublas = nullptr, *cusolver = nullptr;

  XcSpec xc{};
  bool gga = false;

  int nbf = 0, nbf_pad = 0, nblk = 0, mask_words = 0, naux = 0;
  long npts = 0, nbatch = 0, npad = 0, npairs = 0;
  std::vector<long> perm;  // plan point p <- caller point perm[p]

  // grid (Morton order, padded to nbatch * 256; padded points have w = 0)
  double *d_px = nullptr, *d_py = nullptr, *d_pz = nullptr, *d_w = nullptr;
  StoFunc *d_sto = nullptr;  // basis in plan order (see build_plan)
  std::vector<int> h_fperm;  // plan position -> caller function (-1: padding)
  int *d_fperm = nullptr, *d_finv = nullptr;
  StoShell *d_bshell = nullptr;  // radial shells per block [nblk][128]
  int *d_bnshell = nullptr, *d_fshell = nullptr;
  // atoms (for the nuclear gradient)
  int natoms = 0;
  std::vector<double> h_centers;
  double *d_centers = nullptr;
  int *d_fatom = nullptr;  // atom of each function, plan order
  int *d_owner = nullptr;  // owner atom of each point, plan order (null if not given)
  bool all_funcs_on_atoms = false;
  void *grad_state = nullptr;
  AuxFunc *d_aux = nullptr;
  AuxShell *d_ashell = nullptr;
  int nashell = 0;
  AuxGroup *d_agroup = nullptr;  // (centre, l) groups, sorted by l
  int nagroup = 0, nloose = 0;
  std::vector<int> h_group_off;  // groups of l = L at [off[L], off[L+1])
  int *d_loose = nullptr;        // shells outside the groups
  float *d_rtab = nullptr;       // FP32 radial factors [shell][point] of the mixed build's J
  bool rtab_failed = false;      // the table did not fit: the mixed J evaluates the factors

  // screening: pairs of (batch, significant function block), CSR by batch
  std::vector<int> h_pair_off;
  std::vector<uint32_t> h_mask;
  int *d_pair_off = nullptr, *d_pair_blk = nullptr, *d_pair_batch = nullptr;
  uint32_t *d_mask = nullptr;

  std::vector<Chunk> chunks;
  long max_chunk_pairs = 0, chunk_pair_limit = 0;
  // V output tiles (I << 16 | J) of each chunk that have at least one batch
  // with both blocks significant, heaviest first (plan_chunks)
  int *d_vtiles = nullptr;
  int *d_vtiles2 = nullptr;  // V pair tiles (R << 16 | J), by chunk
  Tuning tune;
  double *ws_phi = nullptr;  // PhiT tiles of a chunk: [pair][comp][g][f]
  double *ws_z = nullptr;    // Z^T tiles of a chunk:  [pair][z][g][f]

  // per point (two spins)
  double *d_rho = nullptr, *d_grad = nullptr, *d_coef = nullptr, *d_vj = nullptr;
  // orbitals
  int nocc_cap = 0;
  double *d_Ct = nullptr, *d_occ = nullptr, *d_Cin = nullptr;
  double *d_Cf = nullptr;  // function-major orbitals of the FP64 density pass
  size_t cf_cap = 0;
  // accumulators / outputs
  double *d_V = nullptr, *d_E = nullptr, *d_out = nullptr;
  // caller-order density outputs (nkx_plan_density)
  long *d_perm = nullptr;
  double *d_dens_out = nullptr;

  // Coulomb metric
  bool svd_mode = false;
  double metric_svd_thr = 0.0;
  int K = 0, lwork = 0;
  double *d_L = nullptr, *d_X = nullptr, *d_t = nullptr, *d_y = nullptr, *d_c = nullptr, *d_work = nullptr;
  int *d_info = nullptr, *d_piv = nullptr;
  std::vector<int> h_piv;
  double metric_min_diag = 0.0;
  std::vector<double> h_metric;

  // mixed-precision workspaces (tensor-core path)
  float *mx_phi = nullptr, *mx_a = nullptr, *mx_b = nullptr, *mx_c = nullptr;
  void *mx_state = nullptr;

  // build status words, zeroed by every build: [0] code of the first
  // tensor-core wait that gave up, [1] non-finite input or operand seen
  int *d_status = nullptr;
  // limit of the device waits that may be abandoned (nkx_plan_set_wait_limit)
  unsigned long long wait_ns = 2000000000ull;
  int stall_test = 0;  // tests of the error path: tensor-core kernels wait on a barrier nothing completes
  // state kept between the two phases of a sharded build
  bool phase1_done = false;
  int phase1_precision = 0, phase1_nspin = 1, phase1_nocc = 0;

  // CUDA-graph replay of builds with device buffers (nkx_plan_set_graph)
  bool graph_mode = false;
  std::vector<BuildGraph> graphs;
  long graph_replays = 0;
  void drop_graphs();

  nkx_build_timing last{};
  int launches = 0;
  int last_nspin = 1;

  ~Plan();
  template <class T>
  T *alloc(size_t n);
  void release(void *p);  // frees one allocation made with alloc
};

void plan_chunks(Plan &P, long max_pairs);
// one Fock build, or phase 1 / 2 of a build on a sharded grid (plan.cu)
void fock_build(Plan &P, int precision, int nspin, int nocc, const double *C, const double *occ, int mem, int fuse_j,
                double *E, double *V, double *J, cudaStream_t user, int phase = 0, double *y = nullptr);
void destroy_mixed_state(void *p);

// Accumulates CUDA-event time per build stage.
struct StageTimer {
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  cudaEvent_t begin_ev = nullptr;
  int cur = -1;
  bool on = true;  // off while a build is recorded into a CUDA graph
  ~StageTimer() {
    for (auto &m : marks) {
      cudaEventDestroy(m.second.first);
      cudaEventDestroy(m.second.second);
    }
  }
  void begin(int stage, cudaStream_t s) {
    if (!on) return;
    cudaEvent_t e;
    NKX_CUDA(cudaEventCreate(&e));
    NKX_CUDA(cudaEventRecord(e, s));
    begin_ev = e;
    cur = stage;
  }
  void end(cudaStream_t s) {
    if (!on) return;
    cudaEvent_t e;
    NKX_CUDA(cudaEventCreate(&e));
    NKX_CUDA(cudaEventRecord(e, s));
    marks.push_back({cur, {begin_ev, e}});
  }
  void collect(float out[6]) {
    for (int i = 0; i < 6; ++i) out[i] = 0.f;
    for (auto &m : marks) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, m.second.first, m.second.second);
      out[m.first] += ms;
    }
  }
};

enum { ST_COLLOC = 0, ST_DENSITY = 1, ST_FUNC = 2, ST_COULOMB = 3, ST_ZBUILD = 4, ST_VGEMM = 5 };

bool mixed_available(const Plan &P);
void upload_orbitals(Plan &P, int nspin, int nocc, const double *C, const double *occ, int mem, cudaStream_t s);
void fp64_density_pass(Plan &P, int nspin, int nocc, cudaStream_t s, StageTimer &T);
void launch_colloc(Plan &P, const Chunk &c, cudaStream_t s);
void destroy_grad_state(void *p);
__global__ void functional_kernel(XcSpec s, bool gga, int nspin, long npad, long n, const double *__restrict__ w,
                                  const double *__restrict__ rho, const double *__restrict__ grad,
                                  const double *__restrict__ vj, double *__restrict__ coef, double *Eacc,
                                  double *__restrict__ edens);
// MMA width of the density contraction: the tuning's, or by default 128 from
// 1024 (padded) orbitals on -- half as many orbital tiles re-read each
// Phi tile (1500-atom aggregate, 2850 orbitals: 11.0 vs 12.0 s) -- else 64
// (two TMEM buffers; ahead for short orbital ranges)
inline int density_width(const Plan &P, int nocc) {
  if (P.tune.dens_n) return P.tune.dens_n;
  return ((nocc + 127) / 128) * 128 >= 1024 ? 128 : 64;
}
void mixed_gradient_begin(Plan &P, int nspin, int nocc, cudaStream_t s);
const double *mixed_gradient_chunk(Plan &P, const Chunk &c, int nspin, int nocc, double *edens, cudaStream_t s,
                                   int *nocc_pad, const double **X);
void fock_build_mixed(Plan &P, int nspin, int nocc, bool needJ, bool fuse, bool separateJ, cudaStream_t s,
                      StageTimer &T, int phase);
// mixed: read the aux radial factors from the plan's FP32 table (made on first use)
void coulomb_y(Plan &P, int nspin, cudaStream_t s, bool mixed);
void coulomb_solve(Plan &P, cudaStream_t s, bool mixed);

}  // namespace nkx
