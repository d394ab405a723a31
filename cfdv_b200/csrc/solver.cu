// Element-by-element product and Krylov vector kernels of the GMRES solve.
//
// The EBE product y = sum_e P_e^T R_e P_e x (MPI_GMRES::sum_Av / sum_Ax,
// Utility/Solvers/MPI_GMRES.h:442-693) runs as two deterministic passes:
//   element pass  Y_e = R_e x_e, x_e gathered through the connectivity; R_e streamed
//                 once, element-major, rows read coalesced (column-major storage)
//   node pass     y_n = sum over the node's (element, local node) list of Y_e; the list
//                 is a CSR built once per mesh, so the scatter needs no atomics and no
//                 colouring, and sums always run in the same order.
// Krylov dots/norms reduce to a fixed set of block partials; every consumer block
// re-reduces them in the same order, so all scalars are bitwise reproducible.
#include <cuda_runtime.h>

#include "kernels.h"

namespace cfdv {

template <int KE, int NEQ, int NNOD, int EPB, typename TR, typename TY, bool TRANS>
__global__ void __launch_bounds__(KE* EPB) ebe_elem_kernel(const TR* __restrict__ R, const int* __restrict__ conn,
                                                            const double* __restrict__ x, TY* __restrict__ Y,
                                                            int E) {
  __shared__ TR xs[EPB][KE];
  const int le = threadIdx.x / KE, i = threadIdx.x % KE;
  const int e = blockIdx.x * EPB + le;
  if (e < E) xs[le][i] = (TR)x[(size_t)conn[(size_t)e * NNOD + i / NEQ] * NEQ + i % NEQ];
  __syncthreads();
  if (e >= E) return;
  const TR* __restrict__ Re = R + (size_t)e * KE * KE;
  TR acc = 0;
  if (!TRANS) {
#pragma unroll 8
    for (int j = 0; j < KE; j++) acc += __ldg(Re + j * KE + i) * xs[le][j];
  } else {
#pragma unroll 8
    for (int j = 0; j < KE; j++) acc += __ldg(Re + i * KE + j) * xs[le][j];
  }
  Y[(size_t)e * KE + i] = (TY)acc;
}

template <int NEQ, int NNOD, typename TY>
__global__ void __launch_bounds__(kRedThreads) ebe_node_kernel(const int* __restrict__ ptr,
                                                               const int* __restrict__ idx,
                                                               const TY* __restrict__ Y, int ndof, int mode,
                                                               const double* __restrict__ b, double* out,
                                                               const double* dotv, double* partial) {
  constexpr int KE = NEQ * NNOD;
  double part = 0.0;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < ndof; d += gridDim.x * blockDim.x) {
    const int n = d / NEQ, k = d % NEQ;
    double s = 0.0;
    const int p1 = ptr[n + 1];
    for (int p = ptr[n]; p < p1; p++) {
      const int v = idx[p];
      const int e = v / NNOD, l = v % NNOD;
      s += (double)Y[(size_t)e * KE + l * NEQ + k];
    }
    const double val = mode ? b[d] - s : s;
    out[d] = val;
    if (dotv) part += val * ((dotv == out) ? val : dotv[d]);
  }
  if (partial) {
    part = block_reduce_sum(part);
    if (threadIdx.x == 0) partial[blockIdx.x] = part;
  }
}

template <int NEQ, int NNOD>
static cudaError_t ebe_dispatch(const EbeArgs& a, int use_fp32, int transpose, const double* x, double* out,
                                int mode, const double* b, const double* dot_with, double* partial,
                                cudaStream_t st, cudaEvent_t* ev) {
  constexpr int KE = NEQ * NNOD;
  constexpr int EPB = (KE == 16) ? 16 : 8;
  const int grid = (a.n_elements + EPB - 1) / EPB;
  if (ev) cudaEventRecord(ev[0], st);
  if (grid > 0) {
    if (use_fp32) {
      if (transpose) ebe_elem_kernel<KE, NEQ, NNOD, EPB, float, float, true><<<grid, KE * EPB, 0, st>>>(a.R32, a.conn, x, a.Y32, a.n_elements);
      else ebe_elem_kernel<KE, NEQ, NNOD, EPB, float, float, false><<<grid, KE * EPB, 0, st>>>(a.R32, a.conn, x, a.Y32, a.n_elements);
    } else {
      if (transpose) ebe_elem_kernel<KE, NEQ, NNOD, EPB, double, double, true><<<grid, KE * EPB, 0, st>>>(a.R64, a.conn, x, a.Y64, a.n_elements);
      else ebe_elem_kernel<KE, NEQ, NNOD, EPB, double, double, false><<<grid, KE * EPB, 0, st>>>(a.R64, a.conn, x, a.Y64, a.n_elements);
    }
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (use_fp32)
    ebe_node_kernel<NEQ, NNOD, float><<<kRedBlocks, kRedThreads, 0, st>>>(a.csr_ptr, a.csr_idx, a.Y32, a.n_dof, mode, b, out, dot_with, partial);
  else
    ebe_node_kernel<NEQ, NNOD, double><<<kRedBlocks, kRedThreads, 0, st>>>(a.csr_ptr, a.csr_idx, a.Y64, a.n_dof, mode, b, out, dot_with, partial);
  if (ev) cudaEventRecord(ev[2], st);
  return cudaGetLastError();
}

cudaError_t launch_ebe(const EbeArgs& a, int use_fp32, int transpose, const double* x, double* out, int mode,
                       const double* b, const double* dot_with, double* partial, cudaStream_t st, cudaEvent_t* ev) {
  if (a.ndim == 2) return ebe_dispatch<4, 4>(a, use_fp32, transpose, x, out, mode, b, dot_with, partial, st, ev);
  return ebe_dispatch<5, 8>(a, use_fp32, transpose, x, out, mode, b, dot_with, partial, st, ev);
}

cudaError_t launch_compose_rhs(const EbeArgs& a, const double* rhs, double* b, double* partial, cudaStream_t st) {
  if (a.ndim == 2)
    ebe_node_kernel<4, 4, double><<<kRedBlocks, kRedThreads, 0, st>>>(a.csr_ptr, a.csr_idx, rhs, a.n_dof, 0, nullptr, b, b, partial);
  else
    ebe_node_kernel<5, 8, double><<<kRedBlocks, kRedThreads, 0, st>>>(a.csr_ptr, a.csr_idx, rhs, a.n_dof, 0, nullptr, b, b, partial);
  return cudaGetLastError();
}

// ---- Krylov vector kernels ---------------------------------------------------
__global__ void __launch_bounds__(kRedThreads) dot_kernel(const double* __restrict__ a,
                                                          const double* __restrict__ b, int n, double* partial) {
  double part = 0.0;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) part += a[d] * b[d];
  part = block_reduce_sum(part);
  if (threadIdx.x == 0) partial[blockIdx.x] = part;
}

__global__ void __launch_bounds__(kRedThreads) mgs_kernel(double* w, const double* __restrict__ v, int n,
                                                          const double* __restrict__ pin, double* hout,
                                                          const double* next, double* pout) {
  const double h = reduce_partials(pin, kRedBlocks);
  if (blockIdx.x == 0 && threadIdx.x == 0) *hout = h;
  double part = 0.0;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
    const double wn = w[d] - h * v[d];
    w[d] = wn;
    part += wn * (next ? next[d] : wn);
  }
  part = block_reduce_sum(part);
  if (threadIdx.x == 0) pout[blockIdx.x] = part;
}

__global__ void __launch_bounds__(kRedThreads) normalize_kernel(const double* w, int n,
                                                                const double* __restrict__ pin, double* hout,
                                                                double* vout) {
  const double nrm = sqrt(reduce_partials(pin, kRedBlocks));
  if (blockIdx.x == 0 && threadIdx.x == 0) *hout = nrm;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) vout[d] = w[d] / nrm;
}

__global__ void reduce_kernel(const double* __restrict__ pin, double* out, int do_sqrt) {
  const double s = reduce_partials(pin, kRedBlocks);
  if (threadIdx.x == 0) out[0] = do_sqrt ? sqrt(s) : s;
}

__global__ void __launch_bounds__(kRedThreads) combine_kernel(double* x, const double* __restrict__ V, int n,
                                                              const double* __restrict__ y, int m) {
  __shared__ double ys[256];
  for (int i = threadIdx.x; i < m; i += blockDim.x) ys[i] = y[i];
  __syncthreads();
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
    double z = 0.0;
    for (int i = 0; i < m; i++) z += ys[i] * V[(size_t)i * n + d];
    x[d] += z;
  }
}

__global__ void state_update_kernel(double* U, double* U0, const double* __restrict__ du, int n) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
    const double u = U[d];
    U0[d] = u;
    U[d] = u + du[d];
  }
}

// the same update, skipped when the solve (err), the formation (status) or the time step failed
__global__ void state_update_guarded_kernel(double* U, double* U0, const double* __restrict__ du, int n,
                                            const int* err, const int* status, const double* dt) {
  const double d = *dt;
  if (*err != 0 || (*status & STATUS_NONFINITE_MATRIX) || !(d > 0.0) || !isfinite(d)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double u = U[i];
    U0[i] = u;
    U[i] = u + du[i];
  }
}

__global__ void __launch_bounds__(kRedThreads) rms_partial_kernel(const double* __restrict__ U,
                                                                  const double* __restrict__ U0, int n_nodes,
                                                                  int neqn, double* partial) {
  double s[10];
  for (int k = 0; k < 10; k++) s[k] = 0.0;
  for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < n_nodes; nd += gridDim.x * blockDim.x)
    for (int k = 0; k < neqn; k++) {
      const double u = U[(size_t)nd * neqn + k], u0 = U0[(size_t)nd * neqn + k];
      s[k] += u * u;
      s[5 + k] += u0 * u0;
    }
  for (int k = 0; k < 10; k++) {
    const double t = block_reduce_sum(s[k]);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * 10 + k] = t;
  }
}

// In-place transpose of every element's Ke x Ke block (entry (r, c) at c*Ke + r becomes
// entry (c, r)): the adjoint solve then streams R_e^T with the same coalesced row loads as the
// forward solve.  One block per element at a time; the block is staged in shared memory with
// a padded row stride.
template <int KE, typename T>
__global__ void __launch_bounds__(256) transpose_blocks_kernel(T* R, int E) {
  __shared__ T tile[KE * (KE + 1)];
  for (int e = blockIdx.x; e < E; e += gridDim.x) {
    T* M = R + (size_t)e * KE * KE;
    for (int k = threadIdx.x; k < KE * KE; k += blockDim.x) tile[(k / KE) * (KE + 1) + k % KE] = M[k];
    __syncthreads();
    for (int k = threadIdx.x; k < KE * KE; k += blockDim.x) M[k] = tile[(k % KE) * (KE + 1) + k / KE];
    __syncthreads();
  }
}

cudaError_t launch_transpose_blocks(int ke, double* R64, float* R32, int E, cudaStream_t st) {
  const int grid = E < 16 * kRedBlocks ? E : 16 * kRedBlocks;
  if (E <= 0) return cudaSuccess;
  if (ke == 16) {
    if (R64) transpose_blocks_kernel<16, double><<<grid, 256, 0, st>>>(R64, E);
    if (R32) transpose_blocks_kernel<16, float><<<grid, 256, 0, st>>>(R32, E);
  } else if (ke == 40) {
    if (R64) transpose_blocks_kernel<40, double><<<grid, 256, 0, st>>>(R64, E);
    if (R32) transpose_blocks_kernel<40, float><<<grid, 256, 0, st>>>(R32, E);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

cudaError_t launch_to_float(const double* in, float* out, size_t n, cudaStream_t st) {
  to_float_kernel<<<4 * 148, 256, 0, st>>>(in, out, n);
  return cudaGetLastError();
}

cudaError_t launch_dot(const double* a, const double* b, int n, double* partial, cudaStream_t st) {
  dot_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, b, n, partial);
  return cudaGetLastError();
}
cudaError_t launch_mgs(double* w, const double* v, int n, const double* pin, double* hout, const double* next,
                       double* pout, cudaStream_t st) {
  mgs_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, v, n, pin, hout, next, pout);
  return cudaGetLastError();
}
cudaError_t launch_normalize(const double* w, int n, const double* pin, double* hout, double* vout,
                             cudaStream_t st) {
  normalize_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, n, pin, hout, vout);
  return cudaGetLastError();
}
cudaError_t launch_reduce(const double* pin, double* out, int do_sqrt, cudaStream_t st) {
  reduce_kernel<<<1, kRedThreads, 0, st>>>(pin, out, do_sqrt);
  return cudaGetLastError();
}
cudaError_t launch_combine(double* x, const double* V, int n, const double* y, int m, cudaStream_t st) {
  if (m > 256) return cudaErrorInvalidValue;
  combine_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(x, V, n, y, m);
  return cudaGetLastError();
}
cudaError_t launch_state_update(double* U, double* U0, const double* du, int n, cudaStream_t st) {
  state_update_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(U, U0, du, n);
  return cudaGetLastError();
}
cudaError_t launch_state_update_guarded(double* U, double* U0, const double* du, int n, const int* err,
                                        const int* status, const double* dt, cudaStream_t st) {
  state_update_guarded_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(U, U0, du, n, err, status, dt);
  return cudaGetLastError();
}
cudaError_t launch_rms_partial(const double* U, const double* U0, int n_nodes, int neqn, double* partial,
                               cudaStream_t st) {
  rms_partial_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(U, U0, n_nodes, neqn, partial);
  return cudaGetLastError();
}

}  // namespace cfdv

// ---- node-block Jacobi preconditioner (textbook mode) -------------------------
// D_n = sum over the node's (element, local node) list of the element matrix's diagonal
// neqn x neqn block at that local node; Dinv_n by Gauss-Jordan with partial pivoting in FP64.
namespace cfdv {

// With rhs, the node also assembles b = gather(rhs) over the same list, in the list's order as
// the node pass does (so the same bits), saving that pass its own launch.
template <int NEQ, int NNOD>
__global__ void block_jacobi_kernel(const int* __restrict__ ptr, const int* __restrict__ idx,
                                    const double* __restrict__ R, int n_nodes, double* Dinv, int* status,
                                    const double* __restrict__ rhs, double* b) {
  constexpr int KE = NEQ * NNOD;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
    if (rhs)
      for (int k = 0; k < NEQ; k++) {
        double s = 0.0;
        for (int p = ptr[n]; p < ptr[n + 1]; p++) {
          const int v = idx[p];
          s += rhs[(size_t)(v / NNOD) * KE + (v % NNOD) * NEQ + k];
        }
        b[(size_t)n * NEQ + k] = s;
      }
    double A[NEQ][2 * NEQ];
#pragma unroll
    for (int r = 0; r < NEQ; r++)
#pragma unroll
      for (int s = 0; s < 2 * NEQ; s++) A[r][s] = (s - NEQ == r) ? 1.0 : 0.0;
    for (int p = ptr[n]; p < ptr[n + 1]; p++) {
      const int v = idx[p];
      const int e = v / NNOD, l = v % NNOD;
      const double* Re = R + (size_t)e * KE * KE;
#pragma unroll
      for (int s = 0; s < NEQ; s++)
#pragma unroll
        for (int r = 0; r < NEQ; r++) A[r][s] += Re[(l * NEQ + s) * KE + l * NEQ + r];
    }
    bool ok = true;
#pragma unroll
    for (int c = 0; c < NEQ; c++) {
      int piv = c;
      double best = fabs(A[c][c]);
#pragma unroll
      for (int r = c + 1; r < NEQ; r++)
        if (fabs(A[r][c]) > best) { best = fabs(A[r][c]); piv = r; }
      if (!(best > 0.0)) { ok = false; break; }
      if (piv != c)
#pragma unroll
        for (int s = 0; s < 2 * NEQ; s++) { const double t = A[c][s]; A[c][s] = A[piv][s]; A[piv][s] = t; }
      const double inv = 1.0 / A[c][c];
#pragma unroll
      for (int s = 0; s < 2 * NEQ; s++) A[c][s] *= inv;
#pragma unroll
      for (int r = 0; r < NEQ; r++) {
        if (r == c) continue;
        const double f = A[r][c];
#pragma unroll
        for (int s = 0; s < 2 * NEQ; s++) A[r][s] -= f * A[c][s];
      }
    }
    double* D = Dinv + (size_t)n * NEQ * NEQ;
#pragma unroll
    for (int r = 0; r < NEQ; r++)
#pragma unroll
      for (int s = 0; s < NEQ; s++) D[r * NEQ + s] = ok ? A[r][NEQ + s] : (r == s ? 1.0 : 0.0);
    if (!ok) atomicOr(status, STATUS_SINGULAR_BLOCK);
  }
}

// z = Dinv v node by node (v may be scaled by 1/nrm on the fly: z = Dinv (w / nrm))
template <int NEQ>
__global__ void block_apply_kernel(const double* __restrict__ Dinv, const double* __restrict__ v, double* z,
                                   int n_nodes) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
    double x[NEQ];
#pragma unroll
    for (int s = 0; s < NEQ; s++) x[s] = v[(size_t)n * NEQ + s];
    const double* D = Dinv + (size_t)n * NEQ * NEQ;
#pragma unroll
    for (int r = 0; r < NEQ; r++) {
      double t = 0.0;
#pragma unroll
      for (int s = 0; s < NEQ; s++) t += D[r * NEQ + s] * x[s];
      z[(size_t)n * NEQ + r] = t;
    }
  }
}

// du += Dinv (sum_i y_i V_i) node by node
template <int NEQ>
__global__ void combine_precond_kernel(double* du, const double* __restrict__ V, size_t ld, const double* __restrict__ y,
                                       int m, const double* __restrict__ Dinv, int n_nodes) {
  __shared__ double ys[256];
  for (int i = threadIdx.x; i < m; i += blockDim.x) ys[i] = y[i];
  __syncthreads();
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
    double t[NEQ];
#pragma unroll
    for (int s = 0; s < NEQ; s++) {
      double acc = 0.0;
      for (int i = 0; i < m; i++) acc += ys[i] * V[(size_t)i * ld + (size_t)n * NEQ + s];
      t[s] = acc;
    }
    const double* D = Dinv + (size_t)n * NEQ * NEQ;
#pragma unroll
    for (int r = 0; r < NEQ; r++) {
      double acc = 0.0;
#pragma unroll
      for (int s = 0; s < NEQ; s++) acc += D[r * NEQ + s] * t[s];
      du[(size_t)n * NEQ + r] += acc;
    }
  }
}

cudaError_t launch_block_jacobi(int ndim, const int* ptr, const int* idx, const double* R, int n_nodes, double* Dinv,
                                int* status, const double* rhs, double* b, cudaStream_t st) {
  if (ndim == 2) block_jacobi_kernel<4, 4><<<kRedBlocks, 128, 0, st>>>(ptr, idx, R, n_nodes, Dinv, status, rhs, b);
  else block_jacobi_kernel<5, 8><<<kRedBlocks, 128, 0, st>>>(ptr, idx, R, n_nodes, Dinv, status, rhs, b);
  return cudaGetLastError();
}

cudaError_t launch_block_apply(int ndim, const double* Dinv, const double* v, double* z, int n_nodes, cudaStream_t st) {
  if (ndim == 2) block_apply_kernel<4><<<kRedBlocks, kRedThreads, 0, st>>>(Dinv, v, z, n_nodes);
  else block_apply_kernel<5><<<kRedBlocks, kRedThreads, 0, st>>>(Dinv, v, z, n_nodes);
  return cudaGetLastError();
}

cudaError_t launch_combine_precond(int ndim, double* du, const double* V, size_t ld, const double* y, int m,
                                   const double* Dinv, int n_nodes, cudaStream_t st) {
  if (m > 256) return cudaErrorInvalidValue;
  if (ndim == 2) combine_precond_kernel<4><<<kRedBlocks, kRedThreads, 0, st>>>(du, V, ld, y, m, Dinv, n_nodes);
  else combine_precond_kernel<5><<<kRedBlocks, kRedThreads, 0, st>>>(du, V, ld, y, m, Dinv, n_nodes);
  return cudaGetLastError();
}

}  // namespace cfdv
