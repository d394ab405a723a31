// Arguments of the single-launch restarted GMRES solve (gmres_persistent.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "neighbour_sets.h"

namespace cfdv {

struct PersistentArgs {
  int n_dof, n_elements, m, max_restarts, max_blocks;
  int orth;                    // 0: CGS2, 1: MGS, 2: delayed CGS2, 3: delayed CGS2 with grid barriers only
  double* partm;               // CGS2 multi-dot partials [gridDim.x][m+1]
  double rtol;                 // stop when ||b - A du|| < rtol ||b|| (true residual, FP64 matrices)
  const int* conn;
  const int* csr_ptr;
  const int* csr_idx;
  const double* R64;
  const float* R32;
  double* Y64;
  float* Y32;
  const double* b;
  double* du;                  // solution, starts at zero
  double* V;                   // (m+1) Krylov vectors
  double* W;
  const double* Dinv;          // node-block Jacobi inverse (right preconditioning) or null
  double* Z;                   // preconditioned vector z_j = Dinv v_j
  double* part0;               // block partials (>= gridDim.x each)
  double* part1;
  double* H;                   // (m+1) x m, column-major
  double* g;                   // m+1
  double* cs;                  // m
  double* sn;                  // m
  double* y;                   // m
  double* est;                 // Givens residual estimate per inner step
  int est_capacity;
  double* gfinal;              // |g_k| at the end of each cycle
  int gfinal_capacity;
  int* stop;
  int* out;                    // [0] cycles run
  double* result;              // [0] final ||r||, [1] converged, [2] estimates, [3] products,
                               // [4] FP64 products, [5] algorithmic vector passes, [6] ||b||,
                               // [7] the stopping threshold rtol ||b||
  unsigned int* bar_count;     // grid barrier arrivals, zero before launch
  int* err;                    // bit 0: barrier timeout, bit 1: non-finite residual
  // Neighbour sets of the delayed-CGS2 step (2D, orth 2), CSR over the blocks: rows [0, nb] list
  // the blocks owning nodes of a block's elements, rows [nb + 1, 2 nb + 1] the blocks owning
  // elements at a block's nodes.  Null, or built for another grid size: grid barriers only.
  const int* nbr_ptr;
  const int* nbr_idx;
  int nbr_blocks;
  unsigned int* nbr_flag;      // per block (32 apart): neighbour syncs passed, zero before launch
  int max_valence;             // most (element, local node) entries of a node in the CSR
  int node_cache;              // set at launch: the node pass's gather offsets kept in shared memory
  int ring;                    // 3D: 1 = stream the element matrices through the shared-memory ring
                               // (bulk copies under mbarriers), 0 = direct loads in waves
  int ring_stage_bytes;        // set at launch: bytes of one ring stage (0: direct loads)
};

int persistent_blocks();

cudaError_t launch_gmres_persistent(int ndim, int fp32, const PersistentArgs& a, cudaStream_t st);
int persistent_max_blocks();

}  // namespace cfdv
