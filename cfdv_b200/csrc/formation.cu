// CUDA kernels for the per-step FDV set-up: element formation (+ ApplyBC) and the
// CFL time step.  Formation is one thread block per element running the phases of
// formation.cuh; the CFL step is a per-element minimum with a deterministic
// two-level reduction.
#include <cuda_runtime.h>

#include "formation.cuh"
#include "kernels.h"

namespace cfdv {

template <int NDIM>
__global__ void __launch_bounds__(FormTraits<NDIM>::THREADS, FormTraits<NDIM>::MIN_BLOCKS)
    fdv_form_kernel(FormArgs a) {
  __shared__ FormShared<NDIM> sh;
  __shared__ int bad;
  const int tid = threadIdx.x;
  if (tid == 0) bad = 0;
  for (int e = blockIdx.x; e < a.n_elements; e += gridDim.x) {
    form_step<NDIM>(0, a, sh, e, tid, &bad);
    __syncthreads();
    const int n = form_nsteps<NDIM>(sh);
    for (int k = 1; k < n; k++) {
      form_step<NDIM>(k, a, sh, e, tid, &bad);
      __syncthreads();
    }
  }
  if (tid == 0 && bad) atomicOr(a.status, STATUS_NONFINITE_MATRIX);
}

cudaError_t launch_form(int ndim, const FormArgs& a, cudaStream_t st) {
  if (a.n_elements <= 0) return cudaSuccess;
  const int grid = a.n_elements;
  if (ndim == 2) fdv_form_kernel<2><<<grid, FormTraits<2>::THREADS, 0, st>>>(a);
  else fdv_form_kernel<3><<<grid, FormTraits<3>::THREADS, 0, st>>>(a);
  return cudaGetLastError();
}

// ---- CFL (MPI_CFL.h:124-171): dt = cfl * min_e min_nodes cleng_e / (|v| + sqrt(1.4 cgas T))
template <int NDIM>
__global__ void cfl_partial_kernel(const double* __restrict__ U, const int* __restrict__ conn,
                                   const double* __restrict__ cleng, int E, GasParams g, double* partial) {
  constexpr int NNOD = (NDIM == 2) ? 4 : 8, NEQ = NDIM + 2;
  double best = 1000.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    double dxele = 1000.0;
    for (int i = 0; i < NNOD; i++) {
      const double* u = U + (size_t)conn[(size_t)e * NNOD + i] * NEQ;
      double dxn;
      if (cfl_node_len<NDIM>(u, cleng[e], g, &dxn) && dxn < dxele) dxele = dxn;
    }
    best = fmin(best, dxele);
  }
  best = block_reduce_min(best);
  if (threadIdx.x == 0) partial[blockIdx.x] = best;
}

// final min over the block partials and dt = cfl * min (dt stays unset when no element
// has a finite signal speed, as in the reference where dx_dv starts at 1000)
__global__ void cfl_final_kernel(const double* partial, int nb, double cfl, double* dt_out) {
  double best = 1000.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) best = fmin(best, partial[i]);
  best = block_reduce_min(best);
  if (threadIdx.x == 0) dt_out[0] = (best < 1000.0) ? cfl * best : 0.0;
}

cudaError_t launch_cfl(int ndim, const double* U, const int* conn, const double* cleng, int E, const GasParams& g,
                       double cfl, double* partial, int nb, double* dt_out, cudaStream_t st) {
  if (ndim == 2) cfl_partial_kernel<2><<<nb, 256, 0, st>>>(U, conn, cleng, E, g, partial);
  else cfl_partial_kernel<3><<<nb, 256, 0, st>>>(U, conn, cleng, E, g, partial);
  cfl_final_kernel<<<1, 256, 0, st>>>(partial, nb, cfl, dt_out);
  return cudaGetLastError();
}

}  // namespace cfdv
