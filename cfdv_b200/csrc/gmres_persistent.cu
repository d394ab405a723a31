// Restarted GMRES(m) to a relative tolerance as ONE persistent cooperative kernel.
//
// Launching one kernel per MGS pass and reading every Hessenberg column back to the
// host costs more than the arithmetic on the 2D cases (they fit in L2), and on the 3D
// cases the host round trips still idle the GPU between passes.  This kernel keeps the
// whole solve on the device: every restart recomputes r = b - A du with the FP64
// matrices, then runs the Arnoldi cycle (dots reduced from fixed block partials, so every
// block derives the same scalars), block 0 applies the Givens rotations and tests
// |g_{j+1}| < rtol ||b|| (the stopping rule of the textbook solver), back-substitutes the
// small triangular system and all blocks add V y to du.  Products use the FP64 matrices,
// or the FP32 matrices with FP32 accumulation for the mixed form (the restart residual
// stays FP64: GMRES-based iterative refinement).  With `transpose` every product is A^T x
// (the adjoint system) and the node-block preconditioner is applied transposed.
//
// Orthogonalisation: classical Gram-Schmidt applied twice (CGS2, the default) or modified
// Gram-Schmidt (MGS), both with FP64 dots and norms.  MGS reduces one projection at a time:
// j+3 grid barriers for Arnoldi step j.  CGS2 reduces the j+1 projections of a pass at once
// and repeats the pass once ("twice is enough": orthogonality to working precision, as with
// MGS): 4 grid barriers per step.  On the L2-resident 2D cases the solve is bound by that
// chain of barriers.
//
// Shape: 512-thread blocks, two per SM, so that the element pass keeps as many matrix
// loads in flight as the stand-alone element kernel (each thread owns one row of one
// element and issues its Ke loads back to back).
//
// Phases are separated by a grid barrier.  Its spin is bounded: a block that waits
// longer than the limit sets an error flag and every block returns at the next
// barrier, so a broken launch ends instead of hanging.  The launch is cooperative,
// which guarantees that all blocks are resident.  Data written by other blocks in the
// same launch is read through L2 (__ldcg): L1 is not coherent across SMs.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "gmres_persistent.h"
#include "kernels.h"

namespace cfdv {

namespace {

constexpr long long kSpinLimit = 1ll << 27;  // ~ seconds of polling: far above any barrier
constexpr int kThreads = 512;
constexpr int kBlocksPerSm = 2;

struct Barrier {
  unsigned int* count;
  unsigned int* gen;
  int* err;
};

// sense-counting barrier over all blocks; returns false if this or another block failed
__device__ __forceinline__ bool grid_sync(const Barrier& b, unsigned int nblocks) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    const unsigned int g = *(volatile unsigned int*)b.gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(b.count, 1u) + 1u;
    if (arrived == nblocks) {
      *(volatile unsigned int*)b.count = 0u;
      __threadfence();
      atomicAdd(b.gen, 1u);
    } else {
      long long spins = 0;
      while (*(volatile unsigned int*)b.gen == g) {
        if (++spins > kSpinLimit) {
          atomicOr(b.err, 1);
          break;
        }
        __nanosleep(20);
      }
    }
    __threadfence();
    if (*(volatile int*)b.err) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  __shared__ double res;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = (lane < nw) ? ws[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) res = v;
  }
  __syncthreads();
  return res;
}

// the same partials summed in the same order by every block
__device__ __forceinline__ double sum_partials(const double* p, int n) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += __ldcg(p + i);
  return block_sum(v);
}

// z_d = sum_s P[r][s] * (w[n*NEQ + s] / scale), d = n*NEQ + r, P = Dinv (or Dinv^T), with
// the same division as the stored v so that z = P v exactly
template <int NEQ>
__device__ __forceinline__ double precond_at(const double* Dinv, const double* w, int d, double scale, bool trans) {
  const int n = d / NEQ, r = d % NEQ;
  const double* D = Dinv + (size_t)n * NEQ * NEQ;
  double t = 0.0;
#pragma unroll
  for (int s = 0; s < NEQ; s++)
    t += D[trans ? s * NEQ + r : r * NEQ + s] * (__ldcg(w + (size_t)n * NEQ + s) / scale);
  return t;
}

// Element pass Y_e = R_e x_e (TRANS: R_e^T x_e) over the grid: thread (le, i) owns row i of
// element le of each block iteration; x_e is gathered into a double-buffered shared tile.
template <int KE, int NEQ, int NNOD, typename TM, bool TRANS>
__device__ __forceinline__ void elem_pass(const TM* __restrict__ R, const int* __restrict__ conn, const double* x,
                                          TM* Y, int E, TM (*xs)[kThreads / KE][KE]) {
  constexpr int EPB = kThreads / KE;
  const int le = threadIdx.x / KE, i = threadIdx.x % KE;
  int buf = 0;
  for (int e0 = blockIdx.x * EPB; e0 < E; e0 += gridDim.x * EPB) {
    const int e = e0 + le;
    const bool act = le < EPB && e < E;
    if (act) xs[buf][le][i] = (TM)__ldcg(x + (size_t)__ldg(conn + (size_t)e * NNOD + i / NEQ) * NEQ + i % NEQ);
    __syncthreads();  // the other buffer was last read before the previous barrier
    if (act) {
      const TM* Re = R + (size_t)e * KE * KE;
      TM acc = 0;
      if constexpr (!TRANS) {
#pragma unroll
        for (int j = 0; j < KE; j++) acc += __ldg(Re + j * KE + i) * xs[buf][le][j];
      } else {  // row i of R_e^T is R_e's contiguous column i (served by L1 across j)
#pragma unroll
        for (int j = 0; j < KE; j++) acc += __ldg(Re + i * KE + j) * xs[buf][le][j];
      }
      Y[(size_t)e * KE + i] = acc;
    }
    buf ^= 1;
  }
}

constexpr int kWarps = kThreads / 32;
constexpr int kMaxBasis = 64;  // CGS2 runs for m + 1 <= 64; larger m falls back to MGS

// part[bid * ld + i] = this block's share of <V_i, w>, i < nv: a warp sum per i into
// red[warp][i], then one sum over the warps per i (fixed order)
__device__ __forceinline__ void multi_dot_partials(const double* V, const double* w, int n, int nv, double* part,
                                                   int ld, double (*red)[kMaxBasis]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int gtid = blockIdx.x * kThreads + threadIdx.x, gstride = gridDim.x * kThreads;
  // four projections at a time: their loads and butterfly sums overlap
  for (int i0 = 0; i0 < nv; i0 += 4) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int d = gtid; d < n; d += gstride) {
      const double wd = __ldcg(w + d);
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (i0 + q < nv) acc[q] += __ldcg(V + (size_t)(i0 + q) * n + d) * wd;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (i0 + q < nv) red[wid][i0 + q] = acc[q];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nv; i += kThreads) {
    double t = 0.0;
    for (int k = 0; k < kWarps; k++) t += red[k][i];
    part[(size_t)blockIdx.x * ld + i] = t;
  }
}

// hs[i] = sum over the nb blocks of part[b * ld + i], i < nv, the same bits in every block:
// the threads split the blocks into `slices` fixed ranges per i, and the slice sums are
// added in slice order.  stage holds kThreads doubles.
__device__ __forceinline__ void reduce_multi(const double* part, int ld, int nv, int nb, double* hs, double* stage) {
  const int slices = kThreads / nv;
  const int t = threadIdx.x, i = t % nv, sl = t / nv;
  double acc = 0.0;
  if (sl < slices) {
    const int per = (nb + slices - 1) / slices;
    const int b1 = min(nb, (sl + 1) * per);
    for (int b = sl * per; b < b1; b++) acc += __ldcg(part + (size_t)b * ld + i);
  }
  stage[t] = acc;
  __syncthreads();
  if (t < nv) {
    double s = 0.0;
    for (int k = 0; k < slices; k++) s += stage[k * nv + t];
    hs[t] = s;
  }
  __syncthreads();
}

}  // namespace

template <int KE, int NEQ, int NNOD, typename TR, bool TRANS>
__global__ void __launch_bounds__(kThreads, kBlocksPerSm) gmres_persistent_kernel(PersistentArgs a) {
  const unsigned int nb = gridDim.x;
  const int tid = threadIdx.x, bid = blockIdx.x;
  const int gtid = bid * kThreads + tid, gstride = nb * kThreads;
  const int n = a.n_dof;
  constexpr bool tr = TRANS;
  Barrier bar{a.bar_count, a.bar_gen, a.err};
  constexpr int EPB = kThreads / KE;
  __shared__ double xs64[2][EPB][KE];
  __shared__ TR xs[2][EPB][KE];
  double* V = a.V;
  double* W = a.W;
  double* pa = a.part0;
  double* pb = a.part1;
  const bool cgs = a.orth == 0 && a.m + 1 <= kMaxBasis && a.partm != nullptr;
  __shared__ double red[kWarps][kMaxBasis];  // CGS2: per-warp dot partials
  __shared__ double hs1[kMaxBasis], hs2[kMaxBasis], stage[kThreads];

  auto elem_pass64 = [&](const double* x) {
    elem_pass<KE, NEQ, NNOD, double, TRANS>(a.R64, a.conn, x, a.Y64, a.n_elements, xs64);
  };
  // FP64 matrices, or FP32 matrices with FP32 accumulation
  auto elem_pass_op = [&](const double* x) {
    if (sizeof(TR) == 8) elem_pass64(x);
    else elem_pass<KE, NEQ, NNOD, TR, TRANS>((const TR*)a.R32, a.conn, x, (TR*)a.Y32, a.n_elements, xs);
  };
  // node pass: out = gather(Y) (mode 0) or b - gather(Y) (mode 1); partial of out . dotv
  auto node_pass = [&](bool fp32, int mode, double* out, const double* dotv, double* part) {
    double acc = 0.0;
    for (int d = gtid; d < n; d += gstride) {
      const int nd = d / NEQ, k = d % NEQ;
      double s = 0.0;
      const int p1 = __ldg(a.csr_ptr + nd + 1);
      for (int p = __ldg(a.csr_ptr + nd); p < p1; p++) {
        const int v = __ldg(a.csr_idx + p);
        const size_t yi = (size_t)(v / NNOD) * KE + (v % NNOD) * NEQ + k;
        s += fp32 ? (double)__ldcg(a.Y32 + yi) : __ldcg(a.Y64 + yi);
      }
      const double val = mode ? a.b[d] - s : s;
      out[d] = val;
      acc += val * (dotv ? __ldcg(dotv + d) : val);
    }
    acc = block_sum(acc);
    if (tid == 0) part[bid] = acc;
  };

  const int m = a.m;
  double* H = a.H;  // (m+1) x m column-major, rotated in place by block 0
  int total_est = 0, mv = 0, mv64 = 0;
  long passes = 0;  // algorithmic DOF-vector passes of the orthogonalisation and combination
  bool converged = false;
  double beta = 0.0;
  for (int cycle = 0; cycle < a.max_restarts; cycle++) {
    // r = b - A64 du, beta = ||r||
    elem_pass64(a.du);
    if (!grid_sync(bar, nb)) return;
    node_pass(false, 1, W, nullptr, pa);
    mv++;
    mv64++;
    if (!grid_sync(bar, nb)) return;
    beta = sqrt(sum_partials(pa, nb));
    if (!(beta == beta)) {
      if (bid == 0 && tid == 0) atomicOr(a.err, 2);
      return;
    }
    if (beta < a.atol) {
      converged = true;
      break;
    }
    for (int d = gtid; d < n; d += gstride) {
      V[d] = __ldcg(W + d) / beta;
      if (a.Dinv) a.Z[d] = precond_at<NEQ>(a.Dinv, W, d, beta, tr);
    }
    if (bid == 0 && tid == 0) {
      for (int i = 0; i <= m; i++) a.g[i] = 0.0;
      a.g[0] = beta;
    }
    if (!grid_sync(bar, nb)) return;
    int k = 0;
    for (int j = 0; j < m; j++) {
      const double* xj = a.Dinv ? a.Z : V + (size_t)j * n;  // right preconditioning: A P v_j
      elem_pass_op(xj);
      if (!grid_sync(bar, nb)) return;
      double* Hj = H + (size_t)j * (m + 1);
      if (cgs) {
        // CGS2.  Every thread owns the same unknowns d = gtid + k*gstride in all passes, so
        // the node pass's w feeds this thread's first dots without a grid barrier.
        const int nv = j + 1, ld = m + 1;
        node_pass(sizeof(TR) == 4, 0, W, nullptr, pa);
        mv++;
        multi_dot_partials(V, W, n, nv, a.partm, ld, red);  // h1 = V^T w
        if (!grid_sync(bar, nb)) return;
        reduce_multi(a.partm, ld, nv, nb, hs1, stage);
        for (int d = gtid; d < n; d += gstride) {  // w -= V h1
          double w = __ldcg(W + d);
#pragma unroll 8
          for (int i = 0; i < nv; i++) w -= hs1[i] * __ldcg(V + (size_t)i * n + d);
          W[d] = w;
        }
        multi_dot_partials(V, W, n, nv, a.partm, ld, red);  // h2 = V^T w (the second pass)
        if (!grid_sync(bar, nb)) return;
        reduce_multi(a.partm, ld, nv, nb, hs2, stage);
        if (bid == 0)
          for (int i = tid; i < nv; i += kThreads) Hj[i] = hs1[i] + hs2[i];
        double acc = 0.0;
        for (int d = gtid; d < n; d += gstride) {  // w -= V h2, ||w||^2
          double w = __ldcg(W + d);
#pragma unroll 8
          for (int i = 0; i < nv; i++) w -= hs2[i] * __ldcg(V + (size_t)i * n + d);
          W[d] = w;
          acc += w * w;
        }
        acc = block_sum(acc);
        if (tid == 0) pa[bid] = acc;
        if (!grid_sync(bar, nb)) return;
      } else {
      node_pass(sizeof(TR) == 4, 0, W, V, pa);
      mv++;
      if (!grid_sync(bar, nb)) return;
      for (int i = 0; i <= j; i++) {
        // MGS step i: h = <w, v_i> (reduced from the partials of the previous pass),
        // w -= h v_i, and the partial of the next dot <w, v_{i+1}> (or ||w||^2)
        const double h = sum_partials(pa, nb);
        if (bid == 0 && tid == 0) Hj[i] = h;
        const double* vi = V + (size_t)i * n;
        const double* nx = (i < j) ? V + (size_t)(i + 1) * n : nullptr;
        double acc = 0.0;
#pragma unroll 4
        for (int d = gtid; d < n; d += gstride) {
          const double wn = __ldcg(W + d) - h * __ldcg(vi + d);
          W[d] = wn;
          acc += wn * (nx ? __ldcg(nx + d) : wn);
        }
        acc = block_sum(acc);
        if (tid == 0) pb[bid] = acc;
        double* t = pa; pa = pb; pb = t;
        if (!grid_sync(bar, nb)) return;
      }
      }
      const double nrm = sqrt(sum_partials(pa, nb));
      double* vn = V + (size_t)(j + 1) * n;
      for (int d = gtid; d < n; d += gstride) {
        vn[d] = __ldcg(W + d) / nrm;
        if (a.Dinv) a.Z[d] = precond_at<NEQ>(a.Dinv, W, d, nrm, tr);
      }
      if (bid == 0 && tid == 0) {
        // Givens QR of column j (rotations of earlier columns are stored in cs/sn)
        Hj[j + 1] = nrm;
        for (int i = 0; i < j; i++) {
          const double t0 = a.cs[i] * Hj[i] + a.sn[i] * Hj[i + 1];
          Hj[i + 1] = -a.sn[i] * Hj[i] + a.cs[i] * Hj[i + 1];
          Hj[i] = t0;
        }
        const double den = hypot(Hj[j], Hj[j + 1]);
        const double c = den > 0 ? Hj[j] / den : 1.0, s = den > 0 ? Hj[j + 1] / den : 0.0;
        a.cs[j] = c;
        a.sn[j] = s;
        Hj[j] = den;
        Hj[j + 1] = 0.0;
        a.g[j + 1] = -s * a.g[j];
        a.g[j] = c * a.g[j];
        if (total_est < a.est_capacity) a.est[total_est] = a.g[j + 1];
        *a.stop = (fabs(a.g[j + 1]) < a.atol || nrm == 0.0 || !(nrm == nrm)) ? 1 : 0;
      }
      total_est++;
      passes += j + 2;  // v_0 .. v_j read once, v_{j+1} written
      k = j + 1;
      if (!grid_sync(bar, nb)) return;
      if (*(volatile int*)a.stop) break;
    }
    // y from the upper-triangular system, du += P V y
    if (bid == 0 && tid == 0) {
      for (int i = k - 1; i >= 0; i--) {
        double s = a.g[i];
        for (int jj = i + 1; jj < k; jj++) s -= H[(size_t)jj * (m + 1) + i] * a.y[jj];
        a.y[i] = s / H[(size_t)i * (m + 1) + i];
      }
      if (cycle < a.gfinal_capacity) a.gfinal[cycle] = a.g[k];
    }
    if (!grid_sync(bar, nb)) return;
    for (int d = gtid; d < n; d += gstride) {
      if (a.Dinv) {  // du += P (V y), P = Dinv or Dinv^T
        const int nd = d / NEQ, r = d % NEQ;
        double acc = 0.0;
#pragma unroll
        for (int s2 = 0; s2 < NEQ; s2++) {
          double t = 0.0;
          for (int i = 0; i < k; i++) t += __ldcg(a.y + i) * __ldcg(V + (size_t)i * n + (size_t)nd * NEQ + s2);
          acc += a.Dinv[(size_t)nd * NEQ * NEQ + (tr ? s2 * NEQ + r : r * NEQ + s2)] * t;
        }
        a.du[d] += acc;
      } else {
        double z = 0.0;
        for (int i = 0; i < k; i++) z += __ldcg(a.y + i) * __ldcg(V + (size_t)i * n + d);
        a.du[d] += z;
      }
    }
    if (!grid_sync(bar, nb)) return;
    passes += k + 2;  // du += V y: k basis vectors read, du read and written
    if (bid == 0 && tid == 0) a.out[0] = cycle + 1;
  }
  if (!converged) {  // residual after the last cycle
    elem_pass64(a.du);
    if (!grid_sync(bar, nb)) return;
    node_pass(false, 1, W, nullptr, pa);
    mv++;
    mv64++;
    if (!grid_sync(bar, nb)) return;
    beta = sqrt(sum_partials(pa, nb));
  }
  if (bid == 0 && tid == 0) {
    a.result[0] = beta;
    a.result[1] = converged ? 1.0 : 0.0;
    a.result[2] = (double)total_est;
    a.result[3] = (double)mv;
    a.result[4] = (double)mv64;
    a.result[5] = (double)passes;
  }
}

template <int KE, int NEQ, int NNOD, typename TR, bool TRANS>
static cudaError_t launch_one(const PersistentArgs& a, cudaStream_t st) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gmres_persistent_kernel<KE, NEQ, NNOD, TR, TRANS>,
                                                                kThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidConfiguration;
  // every co-resident block: on the 2D plate (81k unknowns, L2-resident) and the 3D ramp
  // (1.4M unknowns) alike, fewer blocks made each barrier cheaper but every pass slower
  int blocks = sms * (per_sm < kBlocksPerSm ? per_sm : kBlocksPerSm);
  if (blocks > a.max_blocks) blocks = a.max_blocks;
  PersistentArgs args = a;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel((void*)gmres_persistent_kernel<KE, NEQ, NNOD, TR, TRANS>, dim3(blocks), dim3(kThreads),
                                     params, 0, st);
}

template <bool TRANS>
static cudaError_t launch_dim(int ndim, int fp32, const PersistentArgs& a, cudaStream_t st) {
  if (ndim == 2) return fp32 ? launch_one<16, 4, 4, float, TRANS>(a, st) : launch_one<16, 4, 4, double, TRANS>(a, st);
  return fp32 ? launch_one<40, 5, 8, float, TRANS>(a, st) : launch_one<40, 5, 8, double, TRANS>(a, st);
}

cudaError_t launch_gmres_persistent(int ndim, int fp32, const PersistentArgs& a, cudaStream_t st) {
  return a.transpose ? launch_dim<true>(ndim, fp32, a, st) : launch_dim<false>(ndim, fp32, a, st);
}

int persistent_max_blocks() { return kRedBlocks; }

}  // namespace cfdv
