// The library context (cfdv_ctx of include/cfdv_gpu.h) and the internal helpers that the
// translation units of the C ABI share.  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/cfdv_gpu.h"
#include "cfdv_types.h"

struct cfdv_ctx {
  int dev = 0;
  int ndim = 0, nnod = 0, neqn = 0, nbnod = 0, nface = 0, n_nodes = 0, n_elements = 0, n_dof = 0, Ke = 0;
  cfdv::GasParams gas{};
  int phys3d = 0;
  cudaStream_t st = nullptr;
  // mesh
  double* d_x = nullptr;
  int* d_conn = nullptr;
  int* d_bc = nullptr;
  uint64_t* d_mask = nullptr;
  int* d_hnm_idx = nullptr;   // [E] row of d_hnm for an adaptive element, -1 otherwise (null: none)
  double* d_hnm = nullptr;    // [n_adaptive][nnod*nnod] Hnm(N, M) at N + nnod*M
  int n_adaptive = 0;
  double* d_cleng = nullptr;
  int* d_csr_ptr = nullptr;
  int* d_csr_idx = nullptr;
  // state
  double* d_U = nullptr;
  double* d_U0 = nullptr;
  double* d_du = nullptr;
  // element data
  double* d_R64 = nullptr;
  float* d_R32 = nullptr;
  double* d_rhs = nullptr;
  double* d_s = nullptr;
  unsigned char* d_marks = nullptr;  // [E] refinement marks (cfdv_refine_marks)
  double* d_Y64 = nullptr;
  float* d_Y32 = nullptr;
  bool formed = false, have32 = false;
  bool du_valid = false;  // d_du holds a finite solution of an earlier solve
  double dt_formed = 0;
  // krylov
  int m_cap = 0;
  double* d_V = nullptr;
  double* d_W = nullptr;
  double* d_b = nullptr;
  double* d_pa = nullptr;
  double* d_pb = nullptr;
  double* d_H = nullptr;   // Hessenberg (m+1) x m column-major + scalars
  double* d_sc = nullptr;  // scalars: [0] g0/beta, [1] ||b||, [2] dt
  double* d_y = nullptr;
  double* d_rms = nullptr;
  int* d_status = nullptr;
  unsigned int* d_cfl_count = nullptr;  // blocks of the CFL kernel done (the last one resets it)
  double* h_pin = nullptr;  // pinned host staging
  double* h_hist = nullptr;  // pinned: the Givens estimates and final |g| of a persistent solve
  size_t h_hist_cap = 0;
  double* d_pers = nullptr;  // persistent-solve scratch
  size_t pers_cap = 0;
  int* d_pers_int = nullptr;
  double* d_Dinv = nullptr;  // node-block Jacobi inverse [Nn][neqn][neqn]
  double* d_Z = nullptr;     // preconditioned Krylov vector
  double* d_pm = nullptr;    // (D)CGS2 multi-dot partials, two buffers [128][kRedBlocks]
  int* d_nbr_ptr = nullptr;  // neighbour sets of the persistent solve (2D), CSR over its blocks
  int* d_nbr_idx = nullptr;
  int nbr_blocks = 0;        // grid size they were built for (0: none)
  int max_valence = 0;       // most (element, local node) entries of a node
  // adjoint and tangent runs (adjoint.cu)
  std::vector<double> h_records;   // node records of cfdv_load_node_records: the initial state
  double* d_adj_e = nullptr;       // [E][Ke + 3] per-element gradient rows, d/ddt, d/dMach
  double* d_adj_v = nullptr;       // 4 DOF vectors
  double* d_adj_states = nullptr;  // checkpoints and one segment of states
  size_t adj_state_cap = 0;
  // element-matrix sets of a segment's recomputed steps, kept for their reverse steps
  std::vector<double*> adj_pool64;
  std::vector<float*> adj_pool32;
  int* d_wall_elems = nullptr;     // elements with a face of the wall code
  double* d_wall_buf = nullptr;
  int n_wall_elems = 0, wall_bc_cached = -1 << 30;
  // profiling
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_form;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_solve;
  long mv_launches = 0;
  long launches = 0;    // kernels launched since the last cfdv_profile()
  double mv_bytes = 0;  // algorithmic bytes of the timed element passes
  double mv_full_bytes = 0;  // ... and of the whole products (element + node pass)
  double solve_bytes = 0;  // algorithmic bytes of the timed single-launch solves
  std::string err;
};

namespace cfdv {
namespace ctxi {

inline int fail(cfdv_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(c, CFDV_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
inline int dalloc(cfdv_ctx* c, T** p, size_t n) {
  if (*p) { cudaFree(*p); *p = nullptr; }
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(c, CFDV_ERR_ALLOC, std::string("cudaMalloc of ") + std::to_string(n * sizeof(T)) + " bytes: " +
                                       cudaGetErrorString(e));
  }
  return CFDV_OK;
}

template <typename T>
inline void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// internal steps of the solver (cfdv_abi.cu)
// Restarted GMRES(m) in CORRECT mode as one persistent launch; the right-hand side is the
// assembled element rhs (rhs_vec == nullptr) or the device vector rhs_vec; transpose = 1
// solves A^T x = rhs and restores the element blocks afterwards, kTransposeKeep solves
// A^T x = rhs and leaves them transposed (the caller re-forms before the next use).  The
// iteration starts from the device vector x0 (zero when null): every restart cycle, the first
// included, starts from r = b - A x.  The solution is left in c->d_du.
constexpr int kTransposeKeep = 2;
int solve_device(cfdv_ctx* c, const cfdv_gmres_opts* o, cfdv_gmres_report* rep, const double* rhs_vec,
                 int transpose, const double* x0 = nullptr);

// solve_device in two halves: solve_launch enqueues the persistent launch and the read-back
// of its results into c->h_pin + kPinSolve without waiting; solve_finish waits for the
// stream and fills the report.
constexpr int kPinSolve = 4000;  // 4 doubles of int flags, 8 results
constexpr int kPinStep = 4016;   // dt, formation status of a step
struct SolveLaunch {
  double* est;
  double* gfinal;
  const double* h_est;  // pinned copies of est and gfinal, filled by the stream
  const double* h_gfinal;
  int est_cap, gf_cap;
  int* err;   // device error flags of the launch (bit 0 barrier timeout, bit 1 non-finite)
  int fp32;
};
int solve_launch(cfdv_ctx* c, const cfdv_gmres_opts* o, const double* rhs_vec, int transpose, SolveLaunch* L,
                 const double* x0 = nullptr);
int solve_finish(cfdv_ctx* c, const SolveLaunch& L, cfdv_gmres_report* rep);

}  // namespace ctxi
}  // namespace cfdv
