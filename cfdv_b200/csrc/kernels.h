// Kernel launchers and device helpers shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "cfdv_types.h"

namespace cfdv {

// bits of the device status word
enum : int {
  STATUS_NONFINITE_MATRIX = 1,  // a non-finite entry in an element matrix or rhs
  STATUS_NONFINITE_VECTOR = 2,  // a non-finite Krylov scalar
  STATUS_SINGULAR_BLOCK = 4,    // a node block of the preconditioner is singular (identity used)
};

constexpr int kRedBlocks = 4 * 148;  // fixed partial count: reductions are deterministic
constexpr int kRedThreads = 256;

#if defined(__CUDACC__)
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
// fixed-shape tree: the same inputs always give the same bits; result valid in thread 0
__device__ __forceinline__ double block_reduce_sum(double v) {
  __shared__ double ws[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? ws[threadIdx.x] : 0.0;
  if (wid == 0) v = warp_sum(v);
  return v;
}
__device__ __forceinline__ double block_reduce_min(double v) {
  __shared__ double wm[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_min(v);
  __syncthreads();
  if (lane == 0) wm[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? wm[threadIdx.x] : 1e300;
  if (wid == 0) v = warp_min(v);
  return v;
}
// every block sums the same partials in the same order -> identical value everywhere
__device__ __forceinline__ double reduce_partials(const double* __restrict__ p, int n) {
  __shared__ double bc;
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
  v = block_reduce_sum(v);
  if (threadIdx.x == 0) bc = v;
  __syncthreads();
  const double r = bc;
  __syncthreads();
  return r;
}
#endif

// ---- launchers ---------------------------------------------------------------
struct FormArgs;
cudaError_t launch_form(int ndim, const FormArgs& a, cudaStream_t st);
// FDVParam's s1 > threshold per element from the node states U (refinement marks, 1 byte each)
cudaError_t launch_refine_marks(int ndim, const double* U, const double* x, const int* conn, int E, const GasParams& g,
                                double threshold, unsigned char* marks, cudaStream_t st);
cudaError_t launch_cfl(int ndim, const double* U, const int* conn, const double* cleng, int E, const GasParams& g,
                       double cfl, double* partial, unsigned int* count, int nb, double* dt_out, cudaStream_t st);

// EBE product y = sum_e P_e^T R_e P_e x (optionally transposed), element pass + node pass.
struct EbeArgs {
  int ndim, nnod, neqn, n_elements, n_dof;
  const int* conn;       // [E][nnod]
  const int* csr_ptr;    // [Nn+1] node -> (element, local node) list
  const int* csr_idx;    // e * nnod + local
  const double* R64;     // [E][Ke*Ke] column-major
  const float* R32;
  double* Y64;           // [E][Ke] element products (scratch)
  float* Y32;
};
// mode: 0 out = A x ; 1 out = b - A x.  dot_with: null -> no partial, == out -> ||out||^2
// ev[0..2] (may be null): recorded before the element pass, between the passes, after the node pass
cudaError_t launch_ebe(const EbeArgs& a, int use_fp32, int transpose, const double* x, double* out, int mode,
                       const double* b, const double* dot_with, double* partial, cudaStream_t st,
                       cudaEvent_t* ev = nullptr);
// b = sum_e scatter(rhs_e) with the partial of ||b||^2
cudaError_t launch_compose_rhs(const EbeArgs& a, const double* rhs, double* b, double* partial, cudaStream_t st);

// Krylov vector kernels (FP64).  Scalars come from partial sums reduced on device.
cudaError_t launch_dot(const double* a, const double* b, int n, double* partial, cudaStream_t st);
// h = sum(pin); *hout = h; w -= h v; pout = partial dot(w, next) (next == null -> dot(w, w))
cudaError_t launch_mgs(double* w, const double* v, int n, const double* pin, double* hout, const double* next,
                       double* pout, cudaStream_t st);
// nrm = sqrt(sum(pin)); *hout = nrm; vout = w / nrm
cudaError_t launch_normalize(const double* w, int n, const double* pin, double* hout, double* vout,
                             cudaStream_t st);
// *out = sum(pin) (single value, for host read-back)
cudaError_t launch_reduce(const double* pin, double* out, int do_sqrt, cudaStream_t st);
// x += sum_i y_i V_i  (V column-major, ld = n), summed in i order per entry
cudaError_t launch_combine(double* x, const double* V, int n, const double* y, int m, cudaStream_t st);
// out[i] = (float) in[i]
cudaError_t launch_to_float(const double* in, float* out, size_t n, cudaStream_t st);
// transpose every element block of R64 and R32 (either may be null) in place; ke = 16 or 40
cudaError_t launch_transpose_blocks(int ke, double* R64, float* R32, int E, cudaStream_t st);
// node-block Jacobi: Dinv_n = (sum of the node's diagonal element blocks)^-1, FP64
cudaError_t launch_block_jacobi(int ndim, const int* ptr, const int* idx, const double* R, int n_nodes, double* Dinv,
                                int* status, const double* rhs, double* b, cudaStream_t st);
// z = Dinv v
cudaError_t launch_block_apply(int ndim, const double* Dinv, const double* v, double* z, int n_nodes, cudaStream_t st);
// du += Dinv (V y)
cudaError_t launch_combine_precond(int ndim, double* du, const double* V, size_t ld, const double* y, int m,
                                   const double* Dinv, int n_nodes, cudaStream_t st);
// U0 = U ; U += du
cudaError_t launch_state_update(double* U, double* U0, const double* du, int n, cudaStream_t st);
// the update, skipped on the device when *err != 0, the formation status flags a non-finite
// entry, or *dt is not finite and positive
cudaError_t launch_state_update_guarded(double* U, double* U0, const double* du, int n, const int* err,
                                        const int* status, const double* dt, cudaStream_t st);
// per-field sums of U^2 and U0^2 -> partial[blk][2*neqn]
cudaError_t launch_rms_partial(const double* U, const double* U0, int n_nodes, int neqn, double* partial,
                               cudaStream_t st);

}  // namespace cfdv
