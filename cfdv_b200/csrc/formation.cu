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

// ---- refinement marks (RefineListAdaptive.h:25-36): FDVParam's s1 from the element's node
// Mach numbers, by the same node unpack and s1 arithmetic as the formation's FDV parameters
template <int NDIM>
__global__ void refine_mark_kernel(const double* __restrict__ U, const double* __restrict__ x,
                                   const int* __restrict__ conn, int E, GasParams g, double threshold,
                                   unsigned char* marks) {
  constexpr int NNOD = (NDIM == 2) ? 4 : 8, NEQ = NDIM + 2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    double Mn[NNOD], Ren[NNOD], s[2];
    for (int i = 0; i < NNOD; i++) {
      const int n = conn[(size_t)e * NNOD + i];
      NodePrim nd;
      node_unpack<NDIM>(g, U + (size_t)n * NEQ, x + (size_t)n * NDIM, nd);
      node_mach_re<NDIM>(g, nd, &Mn[i], &Ren[i]);
    }
    fdv_pair<NNOD>(Mn, 0, s);
    marks[e] = s[0] > threshold ? 1 : 0;
  }
}

cudaError_t launch_refine_marks(int ndim, const double* U, const double* x, const int* conn, int E, const GasParams& g,
                                double threshold, unsigned char* marks, cudaStream_t st) {
  if (E <= 0) return cudaSuccess;
  const int grid = (E + 255) / 256;
  if (ndim == 2) refine_mark_kernel<2><<<grid, 256, 0, st>>>(U, x, conn, E, g, threshold, marks);
  else refine_mark_kernel<3><<<grid, 256, 0, st>>>(U, x, conn, E, g, threshold, marks);
  return cudaGetLastError();
}

// ---- CFL (MPI_CFL.h:7-56): dt = cfl * min_e min_nodes cleng_e / (|v| + sqrt(1.4 cgas T))
template <int NDIM>
__global__ void cfl_partial_kernel(const double* __restrict__ U, const int* __restrict__ conn,
                                   const double* __restrict__ cleng, int E, GasParams g, double* partial,
                                   unsigned int* count, double cfl, double* dt_out) {
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
  // the last block to finish takes the min over the block partials: dt = cfl * min (dt stays
  // unset when no element has a finite signal speed, as in the reference where dx_dv starts
  // at 1000); a min does not depend on the order, and the last block resets the count
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = best;
    __threadfence();
    last = atomicAdd(count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double all = 1000.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) all = fmin(all, __ldcg(partial + i));
  all = block_reduce_min(all);
  if (threadIdx.x == 0) {
    dt_out[0] = (all < 1000.0) ? cfl * all : 0.0;
    *count = 0u;
  }
}

cudaError_t launch_cfl(int ndim, const double* U, const int* conn, const double* cleng, int E, const GasParams& g,
                       double cfl, double* partial, unsigned int* count, int nb, double* dt_out, cudaStream_t st) {
  if (ndim == 2) cfl_partial_kernel<2><<<nb, 256, 0, st>>>(U, conn, cleng, E, g, partial, count, cfl, dt_out);
  else cfl_partial_kernel<3><<<nb, 256, 0, st>>>(U, conn, cleng, E, g, partial, count, cfl, dt_out);
  return cudaGetLastError();
}

}  // namespace cfdv
