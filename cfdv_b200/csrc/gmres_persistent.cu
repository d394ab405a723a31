// Restarted GMRES(m) to a relative tolerance as ONE persistent cooperative kernel.
//
// Launching one kernel per MGS pass and reading every Hessenberg column back to the
// host costs more than the arithmetic on the 2D cases (they fit in L2), and on the 3D
// cases the host round trips still idle the GPU between passes.  This kernel keeps the
// whole solve on the device: every restart recomputes r = b - A du with the FP64
// matrices, then runs the Arnoldi cycle, applies the Givens rotations, tests
// |g_{j+1}| < rtol ||b|| (the stopping rule of the textbook solver), back-substitutes the
// small triangular system and adds P V y to du.  Products use the FP64 matrices, or the
// FP32 matrices with FP32 accumulation for the mixed form (the restart residual stays
// FP64: GMRES-based iterative refinement).  The adjoint system A^T x = b runs through the same
// kernel: the host transposes every element block in place around the launch.
//
// Ownership.  One 1024-thread block per SM.  Block b owns a contiguous range of whole
// nodes; every Krylov vector entry, w, z = P v and du of those unknowns is written only by
// b, so the orthogonalisation, normalisation and update passes need no grid barrier of
// their own.  Only the element pass (it gathers x at the nodes of its elements) and the
// node pass (it gathers the element products of the node's elements) read other blocks'
// data.  When the block's share of the basis fits in shared memory (the 2D cases) it is
// kept there as well ("resident"), and the Gram-Schmidt passes run out of shared memory.
//
// Scalars.  Dot products are reduced from per-block partials in a fixed order, so every
// block derives the same bits; every block then applies the Givens rotations, keeps the
// triangular factor and back-substitutes on its own (redundantly, in shared memory), so
// no block waits for another to publish those scalars.  Block 0 alone records H, the
// residual estimates and the counters.
//
// Orthogonalisation: classical Gram-Schmidt applied twice (CGS2, the default) or modified
// Gram-Schmidt (MGS), both with FP64 dots and norms.  CGS2 reduces the j+1 projections of
// a pass at once and repeats the pass once ("twice is enough": orthogonality to working
// precision, as with MGS).  The norm of the new vector comes from the second pass's
// partials, ||w2||^2 = ||w1||^2 - ||h2||^2 (w2 = w1 - V h2 with V orthonormal); when that
// difference loses more than four digits to cancellation it is recomputed directly, with
// one more grid barrier.  That gives 4 grid barriers per Arnoldi step (MGS: j+3).
//
// Grid barrier: one arrival counter per launch; barrier k completes when the count reaches
// k * blocks.  Its wait is bounded in time: a block that waits longer than the limit sets
// the failure bit and every block returns at its next barrier, so a broken launch ends
// instead of hanging.  The launch is cooperative, which guarantees that all blocks are
// resident.  Data written by other blocks in the same launch is read through L2 (__ldcg):
// L1 is not coherent across SMs.
#include <cuda_runtime.h>

#include <algorithm>

#include "gmres_persistent.h"
#include "kernels.h"

namespace cfdv {

namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxBasis = 64;         // CGS2 / DCGS2: m + 2 <= kMaxBasis
constexpr int kMaxValence = 8;        // node-pass offsets cached for nodes with at most 8 entries
constexpr int kSlots = 128;           // partial slots of one reduction (DCGS2: 2j + 3)
constexpr int kPartLd = kRedBlocks;   // partm[i * kPartLd + block]
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s: far above any barrier wait
constexpr double kPythMin = 1e-4;     // ||w2||^2 / ||w1||^2 below this: recompute the norm

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct Barrier {
  unsigned int* count;  // arrivals since the launch (zero before it); bit 31: failure
  int* err;
  unsigned int target;
};

// every block: returns false if this or another block gave up waiting
__device__ __forceinline__ bool grid_sync(Barrier& b) {
  __shared__ int ok;
  __syncthreads();
  b.target += gridDim.x;
  if (threadIdx.x == 0) {
    unsigned int v;
    // release: this block's writes (ordered before by the block barrier) precede the arrival
    asm volatile("atom.release.gpu.global.add.u32 %0, [%1], 1;" : "=r"(v) : "l"(b.count) : "memory");
    v += 1u;
    if ((v & 0x7fffffffu) < b.target && !(v & 0x80000000u)) {
      const unsigned long long t0 = now_ns();
      unsigned int polls = 0;
      do {  // one poll in flight per block; a back-off sleep measured 1% slower on the plate solve
        ++polls;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(b.count) : "memory");
        if ((polls & 255u) == 0 && now_ns() - t0 > kWaitNs) {
          atomicOr(b.count, 0x80000000u);
          atomicOr(b.err, 1);
          v = 0x80000000u;
        }
      } while ((v & 0x7fffffffu) < b.target && !(v & 0x80000000u));
    }
    ok = (v & 0x80000000u) ? 0 : 1;
  }
  __syncthreads();
  return ok != 0;
}

constexpr int kFlagStride = 32;  // neighbour-sync flags one 128-byte line apart

// Neighbour sync: publish this block's writes (the k-th neighbour sync of the launch sets its
// flag to k), then wait until every block of its set has reached the same sync.  Lane i of
// warp 0 polls block nbrs[i] (shared memory, -1: none; sets have at most 32 blocks).  Every
// block takes the same sequence of syncs, so equal counts mean the same point of the solve.
// Returns false if a block gave up waiting, here or at a grid barrier (bit 31 of its count).
__device__ __forceinline__ bool local_sync(Barrier& b, unsigned int* flag, const int* nbrs, unsigned int& phase) {
  __shared__ int ok;
  __syncthreads();
  ++phase;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x, o = nbrs[lane];
    if (lane == 0)  // release: the block's writes (ordered before by the block barrier) precede it
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(flag + blockIdx.x * kFlagStride), "r"(phase) : "memory");
    bool good = true;
    if (o >= 0) {
      unsigned int v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag + o * kFlagStride) : "memory");
      if (v < phase) {
        const unsigned long long t0 = now_ns();
        unsigned int polls = 0;
        do {
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag + o * kFlagStride) : "memory");
          if ((++polls & 255u) == 0) {
            unsigned int cnt;
            asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(cnt) : "l"(b.count) : "memory");
            if (cnt & 0x80000000u) { good = false; break; }
            if (now_ns() - t0 > kWaitNs) {
              atomicOr(b.count, 0x80000000u);
              atomicOr(b.err, 1);
              good = false;
              break;
            }
          }
        } while (v < phase);
      }
    }
    good = __all_sync(0xffffffffu, good);
    if (lane == 0) ok = good ? 1 : 0;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ double xor_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[kWarps];
  __shared__ double res;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = xor_sum(v);
  __syncthreads();
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = xor_sum(ws[lane]);
    if (lane == 0) res = v;
  }
  __syncthreads();
  return res;
}

// the same partials summed in the same order by every block
__device__ __forceinline__ double sum_partials(const double* p, int n) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) v += __ldcg(p + i);
  return block_sum(v);
}

// ---- 3D element pass through a shared-memory ring ---------------------------------------
// The element matrices are one contiguous stream per block (its elements form one range), so a
// ring of kRingStages stages in shared memory is filled by bulk copies (cp.async.bulk, no
// tensor map, this GPU's memory only) that one producer thread issues, each completing on the
// stage's `full` mbarrier.  The other warps form kRingStages groups; group g consumes the stages
// of slot g: a warp takes whole elements (lane l owns rows l and l + 32), gathers x_e while the
// stage's copy is in flight, waits for `full`, forms its rows from shared memory and stores
// them, and arrives on the slot's `empty` mbarrier, which the producer waits for before
// refilling the slot.  No block barrier stands between stages.  Each row sums over j in
// increasing order, as the direct pass does, so the products are bitwise the same.
constexpr int kRingStages = 3;

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// wait for the phase of `parity` to complete, at most kWaitNs, and give up early when another
// block has set the launch's failure bit; false: the launch is failing (bit set here if not yet)
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, const Barrier& b) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  for (unsigned polls = 1;; polls++) {
    if (mbar_test(bar, parity)) return true;
    if ((polls & 63u) == 0) {
      unsigned cnt;
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(cnt) : "l"(b.count) : "memory");
      if (cnt & 0x80000000u) return false;
      if (now_ns() - t0 > kWaitNs) {
        atomicOr(b.count, 0x80000000u);
        atomicOr(b.err, 1);
        return false;
      }
    }
  }
}
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, unsigned bytes, unsigned long long* bar,
                                               unsigned long long policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// consumer warps (all but warp 0) of slot g
__host__ __device__ constexpr int ring_members(int g) { return (kWarps - 1 - g + kRingStages - 1) / kRingStages; }

// dynamic shared memory of the ring: the stages, then per-warp x_e buffers (KE doubles a warp),
// then the 2 kRingStages mbarriers
constexpr size_t ring_xbuf_offset(size_t stage_bytes) { return (size_t)kRingStages * stage_bytes; }
constexpr size_t ring_bar_offset(size_t stage_bytes) { return ring_xbuf_offset(stage_bytes) + (size_t)kWarps * 40 * 8; }
constexpr size_t ring_total_bytes(size_t stage_bytes) { return ring_bar_offset(stage_bytes) + 64; }

// the ring's pieces in dynamic shared memory (stage_bytes: the launch's stage size)
struct RingView {
  unsigned char* buf;
  unsigned long long* full;
  unsigned long long* empty;
  __device__ __forceinline__ explicit RingView(unsigned stage_bytes) {
    extern __shared__ __align__(16) double dyn[];
    buf = reinterpret_cast<unsigned char*>(dyn);
    full = reinterpret_cast<unsigned long long*>(buf + ring_bar_offset(stage_bytes));
    empty = full + kRingStages;
  }
};

// one thread: barriers of every slot (full: the producer's arrival + the copy's bytes; empty:
// one arrival per consumer warp of the slot), made visible to the bulk-copy unit
__device__ __forceinline__ void ring_init(unsigned stage_bytes) {
  if (threadIdx.x == 0) {
    const RingView rv(stage_bytes);
    for (int sl = 0; sl < kRingStages; sl++) {
      mbar_init(rv.full + sl, 1);
      mbar_init(rv.empty + sl, ring_members(sl));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
}

// ring_t: stages of this launch so far (every thread keeps the same count)
template <int KE, int NEQ, int NNOD, typename TM>
__device__ __noinline__ void elem_pass_ring(const TM* __restrict__ R, const int* __restrict__ conn, const double* x,
                                               TM* Y, int E, unsigned stage_bytes, unsigned& ring_t,
                                               const Barrier& bar) {
  constexpr unsigned EB = KE * KE * sizeof(TM);
  const RingView rv(stage_bytes);
  const int per = (E + gridDim.x - 1) / gridDim.x;
  const int e0 = min(E, (int)blockIdx.x * per), e1 = min(E, e0 + per);
  const int SE = (int)(stage_bytes / EB);
  const int T = (e1 - e0 + SE - 1) / SE;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (wid == 0) {
    if (lane == 0) {
      unsigned long long policy;  // L2 evict-first for the streamed matrices
      asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
      int issued = 0;
      for (int t = 0; t < T; t++) {
        const unsigned tt = ring_t + t, sl = tt % kRingStages, k = tt / kRingStages;
        if (k >= 1 && !mbar_wait(rv.empty + sl, (k - 1) & 1u, bar)) break;
        const int es = e0 + t * SE, ne = min(SE, e1 - es);
        const unsigned bytes = (unsigned)ne * EB;
        mbar_expect_tx(rv.full + sl, bytes);
        bulk_to_shared(rv.buf + (size_t)sl * stage_bytes, R + (size_t)es * KE * KE, bytes, rv.full + sl, policy);
        issued = t + 1;
      }
      // copies still in flight land before the pass ends (the consumers wait for them too;
      // this covers a pass that is being abandoned)
      for (int t = max(0, issued - kRingStages); t < issued; t++) {
        const unsigned tt = ring_t + t;
        mbar_wait(rv.full + tt % kRingStages, (tt / kRingStages) & 1u, bar);
      }
    }
  } else {
    const int c = wid - 1, g = c % kRingStages, q = c / kRingStages, members = ring_members(g);
    TM* xw = reinterpret_cast<TM*>(rv.buf + ring_xbuf_offset(stage_bytes)) + wid * KE;  // this warp's x_e
    for (int t = 0; t < T; t++) {
      const unsigned tt = ring_t + t, sl = tt % kRingStages, k = tt / kRingStages;
      if ((int)sl != g) continue;
      const int es = e0 + t * SE, ne = min(SE, e1 - es);
      bool first = true;
      for (int le = q; le < ne; le += members) {
        const int e = es + le;
        // x_e: rows lane and lane + 32
        const TM xa = (TM)__ldcg(x + (size_t)__ldg(conn + (size_t)e * NNOD + lane / NEQ) * NEQ + lane % NEQ);
        TM xb = 0;
        if (lane + 32 < KE)
          xb = (TM)__ldcg(x + (size_t)__ldg(conn + (size_t)e * NNOD + (lane + 32) / NEQ) * NEQ + (lane + 32) % NEQ);
        xw[lane] = xa;
        if (lane + 32 < KE) xw[lane + 32] = xb;
        __syncwarp();
        if (first) {
          if (!mbar_wait(rv.full + sl, k & 1u, bar)) return;
          first = false;
        }
        const TM* Rs = reinterpret_cast<const TM*>(rv.buf + (size_t)sl * stage_bytes) + (size_t)le * KE * KE;
        TM acc0 = 0, acc1 = 0;
#pragma unroll 8
        for (int j = 0; j < KE; j++) {
          const TM xj = xw[j];
          acc0 += Rs[j * KE + lane] * xj;
          if (lane + 32 < KE) acc1 += Rs[j * KE + lane + 32] * xj;
        }
        Y[(size_t)e * KE + lane] = acc0;
        if (lane + 32 < KE) Y[(size_t)e * KE + lane + 32] = acc1;
        __syncwarp();  // xw is rewritten for the next element
      }
      if (first && !mbar_wait(rv.full + sl, k & 1u, bar)) return;  // no element of this stage: keep phases in step
      __syncwarp();
      if (lane == 0) mbar_arrive(rv.empty + sl);
    }
  }
  ring_t += T;
}

// Element pass Y_e = R_e x_e, thread (le, i) owning row i of element le.
// 2D (L2-resident, latency-bound): the block's warps form groups of G = lcm(Ke, 32) / 32
// warps (one warp, two elements) that each take U = 3 waves of their elements at once from
// the block's contiguous range (the block's whole share in one chunk), synchronising only
// within the group.  3D (streamed from HBM): waves of kThreads / Ke elements interleaved over
// the grid with a block barrier per wave; this kept more of the HBM bandwidth than
// independent groups or bulk L2 prefetches of the next waves did.  x_e of a wave is gathered
// into a shared tile; the gather offsets of the first chunk are kept from launch start
// (`first`, shared memory).
template <int KE>
struct ElemGroups {
  static constexpr int L = KE % 32 == 0 ? KE : (KE == 16 ? 32 : (KE == 40 ? 160 : 32 * KE));  // lcm(KE, 32)
  static constexpr int G = L / 32;            // warps per group
  static constexpr int EPG = L / KE;          // elements per wave of a group
  static constexpr int NG = kWarps / G;       // groups per block
  static constexpr int U = KE <= 16 ? 3 : 1;  // waves per chunk
  static constexpr int CH = U * EPG;          // elements per chunk of a group
  static constexpr int TILE = 2 * U * EPG * KE;  // tile entries per group (double-buffered)
  static constexpr int EPW = kThreads / KE;      // 3D: elements per block wave
  static constexpr int TILES = (U > 1 ? NG * TILE : 2 * EPW * KE);  // tile entries of the block
  static_assert(L % KE == 0 && L % 32 == 0 && NG >= 1 && (G == 1 || NG <= 15), "element groups");  // named barriers 1..15
};

// chunk k of group g of this block covers elements [first_e + k * stride, + CH), elements < end
template <int KE>
struct ElemChunks {
  int first_e, stride, end;
  __device__ __forceinline__ ElemChunks(int E, int g) {
    using EG = ElemGroups<KE>;
    if constexpr (EG::U > 1) {
      const int per = (E + gridDim.x - 1) / gridDim.x;
      const int e0 = min(E, (int)blockIdx.x * per);
      end = min(E, e0 + per);
      first_e = e0 + g * EG::CH;
      stride = EG::NG * EG::CH;
    } else {
      end = E;
      first_e = ((int)blockIdx.x * EG::NG + g) * EG::CH;
      stride = gridDim.x * EG::NG * EG::CH;
    }
  }
};

__device__ __forceinline__ void group_sync(int g, int nthreads) {
  if (nthreads == 32) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(nthreads) : "memory");
}

template <int KE, int NEQ, int NNOD>
__device__ __forceinline__ void elem_first(const int* __restrict__ conn, int E, int (*first)[kThreads]) {
  using EG = ElemGroups<KE>;
  if constexpr (EG::U == 1) {
    const int le = threadIdx.x / KE, i = threadIdx.x % KE, e = blockIdx.x * EG::EPW + le;
    first[0][threadIdx.x] = (le < EG::EPW && e < E) ? __ldg(conn + (size_t)e * NNOD + i / NEQ) * NEQ + i % NEQ : -1;
    return;
  }
  const int g = threadIdx.x / (32 * EG::G), t = threadIdx.x % (32 * EG::G), le = t / KE, i = t % KE;
  const ElemChunks<KE> ch(E, g);
#pragma unroll
  for (int u = 0; u < EG::U; u++) {
    const int e = ch.first_e + u * EG::EPG + le;
    first[u][threadIdx.x] =
        (g < EG::NG && e < ch.end) ? __ldg(conn + (size_t)e * NNOD + i / NEQ) * NEQ + i % NEQ : -1;
  }
}

template <int KE, int NEQ, int NNOD, typename TM>
__device__ __forceinline__ void elem_pass(const TM* __restrict__ R, const int* __restrict__ conn, const double* x,
                                          TM* Y, int E, const int (*first)[kThreads], TM* tiles) {
  using EG = ElemGroups<KE>;
  constexpr int U = EG::U, EPG = EG::EPG;
  if constexpr (U == 1) {
    constexpr int EPW = EG::EPW;
    const int le = threadIdx.x / KE, i = threadIdx.x % KE;
    const bool lact = le < EPW;
    int buf = 0;
    for (int e0 = blockIdx.x * EPW; e0 < E; e0 += gridDim.x * EPW) {
      const int e = e0 + le;
      const bool act = lact && e < E;
      TM* tb = tiles + (size_t)buf * EPW * KE;
      if (act) {
        const int f = e0 == (int)blockIdx.x * EPW ? first[0][threadIdx.x]
                                                  : __ldg(conn + (size_t)e * NNOD + i / NEQ) * NEQ + i % NEQ;
        tb[le * KE + i] = (TM)__ldcg(x + f);
      }
      __syncthreads();  // the other buffer was last read before the previous barrier
      if (act) {
        const TM* Re = R + (size_t)e * KE * KE;
        TM acc = 0;
#pragma unroll
        for (int j = 0; j < KE; j++)
          acc += __ldg(Re + j * KE + i) * tb[le * KE + j];
        Y[(size_t)e * KE + i] = acc;
      }
      buf ^= 1;
    }
    return;
  }
  const int g = threadIdx.x / (32 * EG::G), t = threadIdx.x % (32 * EG::G), le = t / KE, i = t % KE;
  if (g >= EG::NG) return;  // warps left over by the grouping
  const ElemChunks<KE> ch(E, g);
  const int e1 = ch.end;
  TM* tile = tiles + (size_t)g * EG::TILE;  // [2][U][EPG][KE]
  TM nx[U];
#pragma unroll
  for (int u = 0; u < U; u++) {
    const int f = first[u][threadIdx.x];
    nx[u] = f >= 0 ? (TM)__ldcg(x + f) : TM(0);
  }
  int buf = 0;
  for (int c0 = ch.first_e; c0 < e1; c0 += ch.stride) {
    TM* tb = tile + (size_t)buf * U * EPG * KE;
    if (c0 != ch.first_e)
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int e = c0 + u * EPG + le;
        nx[u] = e < e1 ? (TM)__ldcg(x + (size_t)__ldg(conn + (size_t)e * NNOD + i / NEQ) * NEQ + i % NEQ) : TM(0);
      }
#pragma unroll
    for (int u = 0; u < U; u++) tb[(u * EPG + le) * KE + i] = nx[u];
    group_sync(g, 32 * EG::G);  // the other buffer was last read before the previous chunk's barrier
    const TM* Ru[U];
    TM acc[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      Ru[u] = R + (size_t)min(c0 + u * EPG + le, e1 - 1) * KE * KE;  // clamped: rows past the range are not stored
      acc[u] = 0;
    }
#pragma unroll
    for (int j = 0; j < KE; j++)
#pragma unroll
      for (int u = 0; u < U; u++) {
        const TM rv = __ldg(Ru[u] + j * KE + i);
        acc[u] += rv * tb[(u * EPG + le) * KE + j];
      }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int e = c0 + u * EPG + le;
      if (e < e1) Y[(size_t)e * KE + i] = acc[u];
    }
    buf ^= 1;
  }
}

}  // namespace

// Element tiles of all groups (in doubles, enough for FP64) and first-chunk gather offsets
template <int KE>
constexpr size_t tile_doubles() {
  return (size_t)ElemGroups<KE>::TILES + (size_t)ElemGroups<KE>::U * kThreads / 2;
}

// Dynamic shared memory in doubles (the host sizes the launch with it): the element tile and
// gather offsets, g (m+1), cs (m), sn (m), col (m+1), y (m), the packed triangular factor
// m(m+1)/2, the unrotated Hessenberg matrix (m+1) m and a pending column (m+1) of DCGS2,
// then either the resident basis and w ((m+1)*S + S, S = unknowns per block) or the
// per-warp dot partials of the streaming passes (kWarps * kSlots).
template <int KE>
size_t persistent_dyn_doubles(int m, int S, bool resident, size_t ring_stage_bytes = 0) {
  const size_t front = ring_stage_bytes ? ring_total_bytes(ring_stage_bytes) / sizeof(double) : tile_doubles<KE>();
  const size_t base = front + (size_t)5 * m + 2 + (size_t)m * (m + 1) / 2 + (size_t)(m + 1) * (m + 1);
  return base + (resident ? (size_t)(m + 2) * S : (size_t)kWarps * kSlots);
}

template <int KE, int NEQ, int NNOD, typename TR, bool RES>
__global__ void __launch_bounds__(kThreads, 1) gmres_persistent_kernel(PersistentArgs a) {
  extern __shared__ __align__(16) double dyn[];
  const int nb = gridDim.x, tid = threadIdx.x, bid = blockIdx.x, lane = tid & 31, wid = tid >> 5;
  const int n = a.n_dof, m = a.m;
  // own unknowns [lo, lo + ns): whole nodes, S per block
  const int pn = (n / NEQ + nb - 1) / nb, S = pn * NEQ;
  const int lo = min(n, bid * S), ns = min(n, lo + S) - lo;
  Barrier bar{a.bar_count, a.err, 0u};
  // one tile area for both products (FP64 restart residual, TR Arnoldi products)
  double* tile64 = dyn;
  TR* tileR = reinterpret_cast<TR*>(dyn);
  auto* first = reinterpret_cast<int (*)[kThreads]>(dyn + (size_t)ElemGroups<KE>::TILES);
  // 3D with FP32 products (the mixed form): every element pass of the launch, the FP64 restart
  // residuals included, streams its matrices through the shared-memory ring.  The FP64 form keeps
  // the direct pass: measured, the ring made its whole solve slower (see the element pass notes).
  const bool use_ring = KE == 40 && !RES && sizeof(TR) == 4 && a.ring_stage_bytes > 0;
  unsigned ring_t = 0;
  if (use_ring) ring_init(a.ring_stage_bytes);  // visible after the first grid barrier
  else elem_first<KE, NEQ, NNOD>(a.conn, a.n_elements, first);  // each thread reads its own entries
  __shared__ double hs1[kSlots], hs2[kMaxBasis], sc[4];
  __shared__ int s_stop;
  double* g = dyn + (use_ring ? ring_total_bytes(a.ring_stage_bytes) / sizeof(double) : tile_doubles<KE>());  // Givens right-hand side
  double* cs = g + (m + 1);    // rotations
  double* sn = cs + m;
  double* col = sn + m;        // Hessenberg column being rotated
  double* y = col + (m + 1);   // least-squares solution
  double* tri = y + m;         // R column j at tri[j (j+1) / 2 + i], i <= j
  double* Hf = tri + (size_t)m * (m + 1) / 2;  // DCGS2: unrotated column j at Hf[j (m+1) + i]
  double* pend = Hf + (size_t)(m + 1) * m;      // DCGS2: pending column (m+1)
  double* rest = pend + (m + 1);
  double* sV = rest;                          // resident: (m+1) x S own-slice basis
  double* sW = rest + (size_t)(m + 1) * S;    // resident: own slice of w
  // resident, with room: per own node its entry count and the offsets (into Y) of its entries
  int* ncnt = reinterpret_cast<int*>(rest + (size_t)(m + 2) * S);
  int* noff = ncnt + pn;
  double (*red)[kSlots] = reinterpret_cast<double (*)[kSlots]>(rest);  // streaming: per-warp dots
  double* V = a.V;
  double* W = a.W;
  const bool cgs = a.orth == 0 && m + 2 <= kMaxBasis && a.partm != nullptr;
  const bool dcgs = (a.orth == 2 || a.orth == 3) && m + 2 <= kMaxBasis && a.partm != nullptr;
  // DCGS2 step: neighbour syncs where only neighbours' data is read (the gathers of the element
  // and node passes); the one reduction per step stays a grid barrier
  const bool local = a.orth == 2 && a.nbr_ptr != nullptr && a.nbr_blocks == nb;
  __shared__ int s_nbr[2][32];  // this block's two neighbour sets, one block per lane (-1: none)
  if (local && tid < 64) {
    const int row = (tid >> 5) * (nb + 1) + bid, p0 = __ldg(a.nbr_ptr + row) + lane;
    s_nbr[tid >> 5][lane] = p0 < __ldg(a.nbr_ptr + row + 1) ? __ldg(a.nbr_idx + p0) : -1;
  }  // visible after the first grid barrier
  unsigned int lphase = 0;
  auto sync_x = [&]() -> bool {  // x of the next element pass written by the blocks owning its nodes
    return local ? local_sync(bar, a.nbr_flag, s_nbr[0], lphase) : grid_sync(bar);
  };
  auto sync_y = [&]() -> bool {  // element products at this block's nodes written by their owners
    return local ? local_sync(bar, a.nbr_flag, s_nbr[1], lphase) : grid_sync(bar);
  };
  // dot partials: DCGS2 alternates two buffers by step parity, so a block running ahead writes
  // step j+1's partials while others still read step j's (the grid barrier of step j+1 bounds it)
  double* pm = a.partm;

  // own-slice accessors: basis entry i, w
  auto vld = [&](int i, int dl) -> double {
    if constexpr (RES) return sV[(size_t)i * S + dl];
    else return __ldcg(V + (size_t)i * n + lo + dl);
  };
  auto wld = [&](int dl) -> double {
    if constexpr (RES) return sW[dl];
    else return W[lo + dl];  // written by this block only
  };
  auto wst = [&](int dl, double v) {
    if constexpr (RES) sW[dl] = v;
    else W[lo + dl] = v;
  };
  auto vst = [&](int i, int dl, double v) {
    V[(size_t)i * n + lo + dl] = v;  // the element pass gathers it when there is no preconditioner
    if constexpr (RES) sV[(size_t)i * S + dl] = v;
  };

  auto elem_pass64 = [&](const double* x) {
    if (use_ring) elem_pass_ring<KE, NEQ, NNOD, double>(a.R64, a.conn, x, a.Y64, a.n_elements, a.ring_stage_bytes, ring_t, bar);
    else elem_pass<KE, NEQ, NNOD, double>(a.R64, a.conn, x, a.Y64, a.n_elements, first, tile64);
  };
  // FP64 matrices, or FP32 matrices with FP32 accumulation
  auto elem_pass_op = [&](const double* x) {
    if (sizeof(TR) == 8) elem_pass64(x);
    else if (use_ring)
      elem_pass_ring<KE, NEQ, NNOD, TR>((const TR*)a.R32, a.conn, x, (TR*)a.Y32, a.n_elements, a.ring_stage_bytes,
                                        ring_t, bar);
    else elem_pass<KE, NEQ, NNOD, TR>((const TR*)a.R32, a.conn, x, (TR*)a.Y32, a.n_elements, first, tileR);
  };
  // node pass over the own unknowns: w = gather(Y) (mode 0) or b - gather(Y) (mode 1);
  // returns this thread's share of <w, dotv> (dotv null: ||w||^2)
  auto node_pass = [&](bool fp32, int mode, const double* dotv) -> double {
    double acc = 0.0;
    for (int dl = tid; dl < ns; dl += kThreads) {
      const int d = lo + dl, nd = d / NEQ, k = d % NEQ;
      double s = 0.0;
      if (RES && a.node_cache) {  // the same entries in the same order, offsets from shared memory
        const int il = dl / NEQ, cnt = ncnt[il];
        for (int q = 0; q < cnt; q++) {
          const size_t yi = (size_t)noff[il * kMaxValence + q] + k;
          s += fp32 ? (double)__ldcg(a.Y32 + yi) : __ldcg(a.Y64 + yi);
        }
      } else {
        const int p1 = __ldg(a.csr_ptr + nd + 1);
        for (int p = __ldg(a.csr_ptr + nd); p < p1; p++) {
          const int v = __ldg(a.csr_idx + p);
          const size_t yi = (size_t)(v / NNOD) * KE + (v % NNOD) * NEQ + k;
          s += fp32 ? (double)__ldcg(a.Y32 + yi) : __ldcg(a.Y64 + yi);
        }
      }
      const double val = mode ? a.b[d] - s : s;
      wst(dl, val);
      acc += val * (dotv ? __ldcg(dotv + d) : val);
    }
    return acc;
  };
  // z = P v on the own nodes from the stored v_i (P = Dinv, or Dinv^T for the adjoint)
  auto precond_slice = [&](int i) {
    __syncthreads();  // v_i of the whole node is written
    for (int dl = tid; dl < ns; dl += kThreads) {
      const int d = lo + dl, nd = d / NEQ, r = d % NEQ, base = dl - r;
      const double* D = a.Dinv + (size_t)nd * NEQ * NEQ;
      double t = 0.0;
#pragma unroll
      for (int s = 0; s < NEQ; s++) t += D[r * NEQ + s] * vld(i, base + s);
      a.Z[d] = t;
    }
  };
  // the same by the first nthr threads (a multiple of 32), synchronised by named barrier 15
  auto precond_slice_part = [&](int i, int nthr) {
    asm volatile("bar.sync 15, %0;" ::"r"(nthr) : "memory");  // v_i of the whole node is written
    for (int dl = tid; dl < ns; dl += nthr) {
      const int d = lo + dl, nd = d / NEQ, r = d % NEQ, base = dl - r;
      const double* D = a.Dinv + (size_t)nd * NEQ * NEQ;
      double t = 0.0;
#pragma unroll
      for (int s = 0; s < NEQ; s++) t += D[r * NEQ + s] * vld(i, base + s);
      a.Z[d] = t;
    }
  };
  // partm[i][bid] = <v_i, w> over the own unknowns, i < nv; with `norm` also ||w||^2 at i = nv
  auto dots = [&](int nv, bool norm) {
    const int nt = nv + (norm ? 1 : 0);
    if constexpr (RES) {  // warp per projection, out of shared memory
      __syncthreads();    // w written by other threads
      for (int i = wid; i < nt; i += kWarps) {
        const double* vi = i < nv ? sV + (size_t)i * S : sW;
        double acc = 0.0;
        for (int dl = lane; dl < ns; dl += 32) acc += vi[dl] * sW[dl];
        acc = xor_sum(acc);
        if (lane == 0) pm[(size_t)i * kPartLd + bid] = acc;
      }
    } else {  // streaming: each thread its own unknowns, four projections per load batch
      for (int i0 = 0; i0 < nt; i0 += 4) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int dl = tid; dl < ns; dl += kThreads) {
          const double wd = wld(dl);
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (i0 + q < nt) acc[q] += (i0 + q < nv ? vld(i0 + q, dl) : wd) * wd;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q] = xor_sum(acc[q]);
        if (lane == 0)
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (i0 + q < nt) red[wid][i0 + q] = acc[q];
      }
      __syncthreads();
      for (int i = tid; i < nt; i += kThreads) {
        double t = 0.0;
        for (int k = 0; k < kWarps; k++) t += red[k][i];
        pm[(size_t)i * kPartLd + bid] = t;
      }
    }
  };
  // hs[i] = sum over the blocks of partm[i][b], i < nt, in the same order in every block
  // (two slots per warp at once, so up to 64 slots cost one round trip to L2)
  auto reduce_parts = [&](int nt, double* hs) {
    for (int i = wid; i < nt; i += 2 * kWarps) {
      const int i2 = i + kWarps;
      double acc = 0.0, acc2 = 0.0;
#pragma unroll 4
      for (int b = lane; b < nb; b += 32) {
        acc += __ldcg(pm + (size_t)i * kPartLd + b);
        if (i2 < nt) acc2 += __ldcg(pm + (size_t)i2 * kPartLd + b);
      }
      acc = xor_sum(acc);
      acc2 = xor_sum(acc2);
      if (lane == 0) {
        hs[i] = acc;
        if (i2 < nt) hs[i2] = acc2;
      }
    }
    __syncthreads();
  };
  // w -= V h over the own unknowns; returns this thread's share of ||w||^2, and with `scale`
  // (nrm > 0) stores v_{j+1} = w / nrm instead of w
  auto update = [&](int nv, const double* h, int jn, double nrm) -> double {
    double acc = 0.0;
    for (int dl = tid; dl < ns; dl += kThreads) {
      double w = wld(dl);
#pragma unroll 8
      for (int i = 0; i < nv; i++) w -= h[i] * vld(i, dl);
      if (jn >= 0) vst(jn, dl, w / nrm);
      else wst(dl, w);
      acc += w * w;
    }
    return acc;
  };
  // DCGS2 pass A: partm[s][bid] over the own unknowns of, with u~ = slot j of V,
  //   s < j: <q_s, u~>;  with w: j <= s < 2j: <q_{s-j}, w>, 2j: <u~, u~>, 2j+1: <u~, w>,
  //   2j+2: <w, w>;  without w: j: <u~, u~>
  auto dots_d = [&](int j, bool with_w) {
    const int nt = with_w ? 2 * j + 3 : j + 1, s0 = with_w ? 2 * j : j;
    if constexpr (RES) {
      __syncthreads();  // w and u~ written by other threads
      const double* sU = sV + (size_t)j * S;
      for (int sl = wid; sl < nt; sl += kWarps) {
        const double *x, *yv;
        if (sl < j) { x = sV + (size_t)sl * S; yv = sU; }
        else if (sl < s0) { x = sV + (size_t)(sl - j) * S; yv = sW; }
        else { const int r = sl - s0; x = r == 2 ? sW : sU; yv = r == 0 ? sU : sW; }
        double acc = 0.0;
        for (int dl = lane; dl < ns; dl += 32) acc += x[dl] * yv[dl];
        acc = xor_sum(acc);
        if (lane == 0) pm[(size_t)sl * kPartLd + bid] = acc;
      }
    } else {  // streaming: each thread its own unknowns, four basis vectors per load batch
      for (int i0 = 0; i0 < j; i0 += 4) {
        double au[4] = {0.0, 0.0, 0.0, 0.0}, aw[4] = {0.0, 0.0, 0.0, 0.0};
        for (int dl = tid; dl < ns; dl += kThreads) {
          const double u = vld(j, dl), w = with_w ? wld(dl) : 0.0;
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (i0 + q < j) {
              const double v = vld(i0 + q, dl);
              au[q] += v * u;
              aw[q] += v * w;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          au[q] = xor_sum(au[q]);
          aw[q] = xor_sum(aw[q]);
        }
        if (lane == 0)
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (i0 + q < j) {
              red[wid][i0 + q] = au[q];
              if (with_w) red[wid][j + i0 + q] = aw[q];
            }
      }
      double uu = 0.0, uw = 0.0, ww = 0.0;
      for (int dl = tid; dl < ns; dl += kThreads) {
        const double u = vld(j, dl);
        uu += u * u;
        if (with_w) {
          const double w = wld(dl);
          uw += u * w;
          ww += w * w;
        }
      }
      uu = xor_sum(uu);
      uw = xor_sum(uw);
      ww = xor_sum(ww);
      if (lane == 0) {
        red[wid][s0] = uu;
        if (with_w) {
          red[wid][s0 + 1] = uw;
          red[wid][s0 + 2] = ww;
        }
      }
      __syncthreads();
      for (int sl = tid; sl < nt; sl += kThreads) {
        double t = 0.0;
        for (int k = 0; k < kWarps; k++) t += red[k][sl];
        pm[(size_t)sl * kPartLd + bid] = t;
      }
    }
  };
  // DCGS2 pass B over the own unknowns, with c = hs1[0..j), p = hs1[j..2j) ++ pj:
  //   q_j = (u~_j - Q_j c) / nu  (final, into slot j),  u = w - Q_j p[0..j) - pj q_j,
  //   slot j+1 = u / sigma (sigma > 0), or u kept in w (sigma = 0); returns the share of ||u||^2
  // pass B by the first nthr threads of the block (the resident path's overlapped step)
  auto pass_b_part = [&](int j, double nu, double pj, double sigma, int nthr) {
    for (int dl = tid; dl < ns; dl += nthr) {
      double su = 0.0, sw = 0.0;
#pragma unroll 4
      for (int i = 0; i < j; i++) {
        const double q = vld(i, dl);
        su += hs1[i] * q;
        sw += hs1[j + i] * q;
      }
      const double qj = (vld(j, dl) - su) / nu;
      const double u = wld(dl) - sw - pj * qj;
      vst(j, dl, qj);
      vst(j + 1, dl, u / sigma);
    }
  };
  auto pass_b = [&](int j, double nu, double pj, double sigma) -> double {
    double acc = 0.0;
    for (int dl = tid; dl < ns; dl += kThreads) {
      double su = 0.0, sw = 0.0;
#pragma unroll 4
      for (int i = 0; i < j; i++) {
        const double q = vld(i, dl);
        su += hs1[i] * q;
        sw += hs1[j + i] * q;
      }
      const double qj = (vld(j, dl) - su) / nu;
      const double u = wld(dl) - sw - pj * qj;
      vst(j, dl, qj);
      if (sigma > 0.0) vst(j + 1, dl, u / sigma);
      else wst(dl, u);
      acc += u * u;
    }
    return acc;
  };
  // DCGS2 scalars from the reduced slots (warp 0, the same order in every block):
  // sc[0] = nu = sqrt(<u~,u~> - |c|^2), sc[1] = pj = (<u~,w> - c.p) / nu, sc[2] = <w,w> - |p|^2
  auto dcgs_scalars = [&](int j, bool with_w) {
    if (wid == 0) {
      double cc = 0.0, cp = 0.0, pp = 0.0;
      for (int i = lane; i < j; i += 32) {
        const double c = hs1[i];
        cc += c * c;
        if (with_w) {
          const double p = hs1[j + i];
          cp += c * p;
          pp += p * p;
        }
      }
      cc = xor_sum(cc);
      cp = xor_sum(cp);
      pp = xor_sum(pp);
      if (lane == 0) {
        const int s0 = with_w ? 2 * j : j;
        const double nu = sqrt(hs1[s0] - cc);
        sc[0] = nu;
        if (with_w) {
          const double pj = (hs1[s0 + 1] - cp) / nu;
          sc[1] = pj;
          sc[2] = hs1[s0 + 2] - (pp + pj * pj);
          sc[3] = hs1[s0 + 2];
        }
      }
    }
    __syncthreads();
  };
  if (RES && a.node_cache)  // visible after the first grid barrier
    for (int il = tid; il < ns / NEQ; il += kThreads) {
      const int nd = lo / NEQ + il, p0 = __ldg(a.csr_ptr + nd), cnt = __ldg(a.csr_ptr + nd + 1) - p0;
      ncnt[il] = cnt;
      for (int q = 0; q < cnt; q++) {
        const int v = __ldg(a.csr_idx + p0 + q);
        noff[il * kMaxValence + q] = (v / NNOD) * KE + (v % NNOD) * NEQ;
      }
    }
  // ||b|| over the own unknowns, then the stopping threshold rtol ||b|| (the same bits in
  // every block)
  {
    double acc = 0.0;
    for (int dl = tid; dl < ns; dl += kThreads) {
      const double v = a.b[lo + dl];
      acc += v * v;
    }
    acc = block_sum(acc);
    if (tid == 0) a.part1[bid] = acc;
  }
  if (!grid_sync(bar)) return;
  const double bnorm = sqrt(sum_partials(a.part1, nb));
  const double atol = a.rtol * bnorm;
  if (!(bnorm == bnorm)) {
    if (bid == 0 && tid == 0) atomicOr(a.err, 2);
    return;
  }
  // Givens QR of Hessenberg column j (col[0..j], subdiagonal nrm) with the stored rotations,
  // by one thread of every block; sets s_stop
  int total_est = 0;
  auto givens = [&](int j, double nrm) {
    if (tid == kThreads - 1) {
      double* Rj = tri + (size_t)j * (j + 1) / 2;
      double hi = col[0];
      for (int i = 0; i < j; i++) {
        const double h1 = col[i + 1];
        Rj[i] = cs[i] * hi + sn[i] * h1;
        hi = -sn[i] * hi + cs[i] * h1;
      }
      const double den = hypot(hi, nrm);
      const double c = den > 0 ? hi / den : 1.0, s = den > 0 ? nrm / den : 0.0;
      cs[j] = c;
      sn[j] = s;
      Rj[j] = den;
      g[j + 1] = -s * g[j];
      g[j] = c * g[j];
      const int stop = (fabs(g[j + 1]) < atol || nrm == 0.0 || !(nrm == nrm)) ? 1 : 0;
      s_stop = stop;
      if (bid == 0) {
        double* Hj = a.H + (size_t)j * (m + 1);
        for (int i = 0; i <= j; i++) Hj[i] = Rj[i];
        Hj[j + 1] = 0.0;
        if (total_est < a.est_capacity) a.est[total_est] = g[j + 1];
        *a.stop = stop;
      }
    }
  };

  int mv = 0, mv64 = 0;
  long passes = 0;  // algorithmic DOF-vector passes of the orthogonalisation and combination
  bool converged = bnorm == 0.0;  // b = 0: du = 0 is the solution
  double beta = 0.0;
  for (int cycle = 0; cycle < a.max_restarts && !converged; cycle++) {
    // r = b - A64 du, beta = ||r||
    elem_pass64(a.du);
    if (!grid_sync(bar)) return;
    {
      const double acc = block_sum(node_pass(false, 1, nullptr));
      if (tid == 0) a.part0[bid] = acc;
    }
    mv++;
    mv64++;
    if (!grid_sync(bar)) return;
    beta = sqrt(sum_partials(a.part0, nb));
    if (!(beta == beta)) {
      if (bid == 0 && tid == 0) atomicOr(a.err, 2);
      return;
    }
    if (beta < atol) {
      converged = true;
      break;
    }
    for (int dl = tid; dl < ns; dl += kThreads) vst(0, dl, wld(dl) / beta);
    if (a.Dinv) precond_slice(0);
    for (int i = tid; i <= m; i += kThreads) g[i] = i == 0 ? beta : 0.0;
    if (!grid_sync(bar)) return;
    int k = 0;
    if (dcgs) {
      // DCGS2 (delayed CGS2, one reduction per step): slot j of V holds the candidate u~_j,
      // projected once and normalised; its second projection happens in step j's pass B, with
      // the coefficients of that step's single reduction, and column j-1 of H is completed
      // then: A P q_{j-1} = Q_j (a + t c) + t nu q_j with the pending (a, t) of step j-1.
      double tpend = 0.0;
      bool done = false;
      for (int j = 0; j < m && !done; j++) {
        pm = a.partm + (size_t)(j & 1) * kSlots * kPartLd;
        elem_pass_op(a.Dinv ? a.Z : V + (size_t)j * n);  // A P u~_j
        if (!sync_y()) return;
        node_pass(sizeof(TR) == 4, 0, nullptr);
        mv++;
        dots_d(j, true);
        if (!grid_sync(bar)) return;
        reduce_parts(2 * j + 3, hs1);
        dcgs_scalars(j, true);
        const double nu = sc[0], pj = sc[1], s2 = sc[2], w2 = sc[3];
        if (RES && s2 > kPythMin * w2) {  // the same decision in every block; then sigma > 0
          // Resident basis (latency-bound): the last warp completes column j-1, rotates it (the
          // stopping test) and forms the pending column j, while the other warps run pass B and
          // the preconditioner; the two parts share no data.  When the test stops the cycle,
          // pass B has written slots j and j+1 only, which the update (slots < j) does not read.
          const double sigma = sqrt(s2);
          if (wid == kWarps - 1) {
            if (j == 0) {
              if (lane == 0) g[0] = beta * nu;  // r = beta u~_0 = beta nu q_0
            } else {
              for (int r = lane; r <= j; r += 32) {
                const double h = r < j ? pend[r] + tpend * hs1[r] : tpend * nu;
                col[r] = h;
                Hf[(size_t)(j - 1) * (m + 1) + r] = h;
              }
              __syncwarp();
              givens(j - 1, tpend * nu);
              __syncwarp();
            }
            for (int r = lane; r <= j; r += 32) {
              double hc = 0.0;
              for (int cj = r > 0 ? r - 1 : 0; cj < j; cj++) hc += Hf[(size_t)cj * (m + 1) + r] * hs1[cj];
              pend[r] = ((r < j ? hs1[j + r] : pj) - hc) / nu;
            }
          } else {
            pass_b_part(j, nu, pj, sigma, kThreads - 32);
            if (a.Dinv) precond_slice_part(j + 1, kThreads - 32);
          }
          __syncthreads();
          if (j > 0) {
            total_est++;
            if (s_stop) {
              k = j;
              break;
            }
          }
          passes += j + 2;
          tpend = sigma / nu;
          k = j + 1;
          if (!sync_x()) return;
          continue;
        }
        if (j == 0) {
          if (tid == 0) g[0] = beta * nu;  // r = beta u~_0 = beta nu q_0
        } else {  // complete column j-1 and rotate it
          for (int r = tid; r <= j; r += kThreads) {
            const double h = r < j ? pend[r] + tpend * hs1[r] : tpend * nu;
            col[r] = h;
            Hf[(size_t)(j - 1) * (m + 1) + r] = h;
          }
          __syncthreads();
          givens(j - 1, tpend * nu);
          total_est++;
          __syncthreads();
          if (s_stop) {
            k = j;
            break;
          }
        }
        // pending column j: a = (p - H_j c) / nu (rows 0..j), t = sigma / nu
        for (int r = tid; r <= j; r += kThreads) {
          double hc = 0.0;
          for (int cj = r > 0 ? r - 1 : 0; cj < j; cj++) hc += Hf[(size_t)cj * (m + 1) + r] * hs1[cj];
          pend[r] = ((r < j ? hs1[j + r] : pj) - hc) / nu;
        }
        double sigma;
        if (s2 > kPythMin * w2) {  // the same decision in every block
          sigma = sqrt(s2);
          pass_b(j, nu, pj, sigma);
        } else {  // cancellation: the norm of the projected w directly
          const double acc = block_sum(pass_b(j, nu, pj, 0.0));
          if (tid == 0) a.part0[bid] = acc;
          if (!grid_sync(bar)) return;
          sigma = sqrt(sum_partials(a.part0, nb));
          if (sigma > 0.0)
            for (int dl = tid; dl < ns; dl += kThreads) vst(j + 1, dl, wld(dl) / sigma);
        }
        passes += j + 2;
        if (!(sigma > 0.0)) {  // invariant subspace (or a non-finite norm): column j is final
          __syncthreads();
          for (int r = tid; r <= j; r += kThreads) col[r] = pend[r];
          __syncthreads();
          givens(j, 0.0);
          total_est++;
          k = j + 1;
          done = true;
          if (!grid_sync(bar)) return;
          break;
        }
        tpend = sigma / nu;
        if (a.Dinv) precond_slice(j + 1);
        k = j + 1;
        if (!sync_x()) return;
      }
      if (!done && k == m) {
        // the cycle ran to m: complete the last column from u~_m's coefficients
        pm = a.partm + (size_t)(m & 1) * kSlots * kPartLd;
        dots_d(m, false);
        if (!grid_sync(bar)) return;
        reduce_parts(m + 1, hs1);
        dcgs_scalars(m, false);
        const double nu = sc[0];
        for (int r = tid; r < m; r += kThreads) col[r] = pend[r] + tpend * hs1[r];
        __syncthreads();
        givens(m - 1, tpend * nu);
        total_est++;
        __syncthreads();
      }
    }
    for (int j = 0; j < m && !dcgs; j++) {
      const double* xj = a.Dinv ? a.Z : V + (size_t)j * n;  // right preconditioning: A P v_j
      elem_pass_op(xj);
      if (!grid_sync(bar)) return;
      const int nv = j + 1;
      double nrm;
      if (cgs) {
        // CGS2: h1 = V^T w, w1 = w - V h1, h2 = V^T w1, w2 = w1 - V h2, H(:, j) = h1 + h2
        node_pass(sizeof(TR) == 4, 0, nullptr);
        mv++;
        dots(nv, false);
        if (!grid_sync(bar)) return;
        reduce_parts(nv, hs1);
        update(nv, hs1, -1, 0.0);
        dots(nv, true);
        if (!grid_sync(bar)) return;
        reduce_parts(nv + 1, hs2);
        double hh = 0.0;
        for (int i = 0; i < nv; i++) hh += hs2[i] * hs2[i];
        const double w1n2 = hs2[nv], n2 = w1n2 - hh;
        for (int i = tid; i < nv; i += kThreads) col[i] = hs1[i] + hs2[i];
        if (n2 > kPythMin * w1n2) {  // the same decision in every block
          nrm = sqrt(n2);
          update(nv, hs2, j + 1, nrm);
        } else {
          const double acc = block_sum(update(nv, hs2, -1, 0.0));
          if (tid == 0) a.part0[bid] = acc;
          if (!grid_sync(bar)) return;
          nrm = sqrt(sum_partials(a.part0, nb));
          for (int dl = tid; dl < ns; dl += kThreads) vst(j + 1, dl, wld(dl) / nrm);
        }
      } else {
        // MGS: h_i = <w, v_i> reduced from the partials of the previous pass, w -= h_i v_i
        double* pa = a.part0;
        double* pb = a.part1;
        {
          const double acc = block_sum(node_pass(sizeof(TR) == 4, 0, V));
          if (tid == 0) pa[bid] = acc;
        }
        mv++;
        if (!grid_sync(bar)) return;
        for (int i = 0; i <= j; i++) {
          const double h = sum_partials(pa, nb);
          if (tid == 0) col[i] = h;
          const double* nx = (i < j) ? V + (size_t)(i + 1) * n : nullptr;
          double acc = 0.0;
          for (int dl = tid; dl < ns; dl += kThreads) {
            const double wn = wld(dl) - h * vld(i, dl);
            wst(dl, wn);
            acc += wn * (nx ? __ldcg(nx + lo + dl) : wn);
          }
          acc = block_sum(acc);
          if (tid == 0) pb[bid] = acc;
          double* t = pa; pa = pb; pb = t;
          if (!grid_sync(bar)) return;
        }
        nrm = sqrt(sum_partials(pa, nb));
        for (int dl = tid; dl < ns; dl += kThreads) vst(j + 1, dl, wld(dl) / nrm);
      }
      if (a.Dinv) precond_slice(j + 1);
      __syncthreads();  // col complete
      givens(j, nrm);
      total_est++;
      passes += j + 2;  // v_0 .. v_j read once, v_{j+1} written
      k = j + 1;
      if (!grid_sync(bar)) return;
      if (s_stop) break;
    }
    // y from R y = g (column-oriented back substitution by one warp of every block)
    if (wid == 0) {
      for (int i = k - 1; i >= 0; i--) {
        const double* Ri = tri + (size_t)i * (i + 1) / 2;
        const double yi = g[i] / Ri[i];
        __syncwarp();
        for (int r = lane; r < i; r += 32) g[r] -= Ri[r] * yi;
        if (lane == 0) y[i] = yi;
        __syncwarp();
      }
    }
    if (bid == 0 && tid == 0 && cycle < a.gfinal_capacity) a.gfinal[cycle] = g[k];
    __syncthreads();
    // du += P V y over the own unknowns
    for (int dl = tid; dl < ns; dl += kThreads) {
      const int d = lo + dl;
      if (a.Dinv) {
        const int nd = d / NEQ, r = d % NEQ, base = dl - r;
        double acc = 0.0;
#pragma unroll
        for (int s2 = 0; s2 < NEQ; s2++) {
          double t = 0.0;
          for (int i = 0; i < k; i++) t += y[i] * vld(i, base + s2);
          acc += a.Dinv[(size_t)nd * NEQ * NEQ + r * NEQ + s2] * t;
        }
        a.du[d] += acc;
      } else {
        double z = 0.0;
        for (int i = 0; i < k; i++) z += y[i] * vld(i, dl);
        a.du[d] += z;
      }
    }
    if (!grid_sync(bar)) return;
    passes += k + 2;  // du += V y: k basis vectors read, du read and written
    if (bid == 0 && tid == 0) a.out[0] = cycle + 1;
  }
  if (!converged) {  // residual after the last cycle
    elem_pass64(a.du);
    if (!grid_sync(bar)) return;
    const double acc = block_sum(node_pass(false, 1, nullptr));
    if (tid == 0) a.part0[bid] = acc;
    mv++;
    mv64++;
    if (!grid_sync(bar)) return;
    beta = sqrt(sum_partials(a.part0, nb));
  }
  if (bid == 0 && tid == 0) {
    a.result[0] = beta;
    a.result[1] = converged ? 1.0 : 0.0;
    a.result[2] = (double)total_est;
    a.result[3] = (double)mv;
    a.result[4] = (double)mv64;
    a.result[5] = (double)passes;
    a.result[6] = bnorm;
    a.result[7] = atol;
  }
}

namespace {

template <int KE, int NEQ, int NNOD, typename TR, bool RES>
cudaError_t launch_cfg(const PersistentArgs& a, int blocks, size_t dyn_bytes, int node_cache, cudaStream_t st) {
  auto* k = gmres_persistent_kernel<KE, NEQ, NNOD, TR, RES>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, dyn_bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  PersistentArgs args = a;
  args.node_cache = node_cache;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel((void*)k, dim3(blocks), dim3(kThreads), params, dyn_bytes, st);
}

// resident basis when the block's share of it fits next to the static arrays
template <int KE, int NEQ, int NNOD, typename TR>
cudaError_t launch_one(const PersistentArgs& a, cudaStream_t st) {
  int dev = 0, sms = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int blocks = sms < a.max_blocks ? sms : a.max_blocks;
  const int pn = (a.n_dof / NEQ + blocks - 1) / blocks, S = pn * NEQ;
  const bool cgs = (a.orth == 0 || a.orth == 2 || a.orth == 3) && a.m + 2 <= kMaxBasis && a.partm != nullptr;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, gmres_persistent_kernel<KE, NEQ, NNOD, TR, true>);
  if (e != cudaSuccess) return e;
  const size_t res_bytes = sizeof(double) * persistent_dyn_doubles<KE>(a.m, S, true);
  // the node pass's offsets: an entry count and kMaxValence offsets per own node
  const size_t cache_bytes = (sizeof(int) * (size_t)pn * (kMaxValence + 1) + 7) / 8 * 8;
  if (cgs && a.max_valence <= kMaxValence && fa.sharedSizeBytes + res_bytes + cache_bytes <= (size_t)optin)
    return launch_cfg<KE, NEQ, NNOD, TR, true>(a, blocks, res_bytes + cache_bytes, 1, st);
  if (cgs && fa.sharedSizeBytes + res_bytes <= (size_t)optin)
    return launch_cfg<KE, NEQ, NNOD, TR, true>(a, blocks, res_bytes, 0, st);
  e = cudaFuncGetAttributes(&fa, gmres_persistent_kernel<KE, NEQ, NNOD, TR, false>);
  if (e != cudaSuccess) return e;
  if (KE == 40 && a.ring && sizeof(TR) == 4) {
    // 3D: the largest ring stage (a multiple of one FP64 element matrix, at most 4 of them) that
    // fits beside the rest; stages hold 4 FP64 or 8 FP32 element matrices at m <= 50
    constexpr size_t kElem64 = (size_t)KE * KE * sizeof(double);
    for (size_t se = 4; se >= 1; se--) {
      const size_t ring_bytes = sizeof(double) * persistent_dyn_doubles<KE>(a.m, S, false, se * kElem64);
      if (fa.sharedSizeBytes + ring_bytes <= (size_t)optin) {
        PersistentArgs ar = a;
        ar.ring_stage_bytes = (int)(se * kElem64);
        return launch_cfg<KE, NEQ, NNOD, TR, false>(ar, blocks, ring_bytes, 0, st);
      }
    }
  }
  const size_t str_bytes = sizeof(double) * persistent_dyn_doubles<KE>(a.m, S, false);
  if (fa.sharedSizeBytes + str_bytes > (size_t)optin) return cudaErrorInvalidValue;  // m too large
  PersistentArgs ad = a;
  ad.ring_stage_bytes = 0;
  return launch_cfg<KE, NEQ, NNOD, TR, false>(ad, blocks, str_bytes, 0, st);
}

cudaError_t launch_dim(int ndim, int fp32, const PersistentArgs& a, cudaStream_t st) {
  if (ndim == 2) return fp32 ? launch_one<16, 4, 4, float>(a, st) : launch_one<16, 4, 4, double>(a, st);
  return fp32 ? launch_one<40, 5, 8, float>(a, st) : launch_one<40, 5, 8, double>(a, st);
}

}  // namespace

cudaError_t launch_gmres_persistent(int ndim, int fp32, const PersistentArgs& a, cudaStream_t st) {
  return launch_dim(ndim, fp32, a, st);
}

int persistent_max_blocks() { return kRedBlocks; }

int persistent_blocks() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  return sms < kRedBlocks ? sms : kRedBlocks;
}


}  // namespace cfdv
