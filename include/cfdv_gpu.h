/* cfdv_gpu.h -- C ABI of the B200 FDV step library (libcfdv_gpu.so).
 *
 * Drop-in boundary for the per-step path of the CFDV driver (src/main.cpp:169-198):
 *
 *   reference call (CFDV src/)                           replaced by
 *   ---------------------------------------------------  ----------------------------------
 *   LoadBinaryData::read_nodes/read_elements             cfdv_create / cfdv_upload_mesh
 *     (Utility/IO/ASCIItoBinary/LoadBinary.h:116-246)      + cfdv_load_node_records
 *   LoadBinaryData::adap (LoadBinary.h:247-261; the      cfdv_set_adaptive
 *     hanging-node Hnm of refined elements)
 *   CalcLength (FDV/Function/CalcLength.h:34-66)         inside cfdv_create
 *   ClearElement + NodeUnpack (main.cpp:169-171)         fused into cfdv_cfl / cfdv_form
 *   CFL (FDV/Function/MPI_CFL.h:7-56, main.cpp:179)   cfdv_cfl
 *   FDVGalerkin over elements (main.cpp:185-186,         cfdv_form
 *     FDV/FDVGalerkin.h:121-154) + ApplyBC (main.cpp:194,
 *     FDV/Function/ApplyBC.h:14-133)
 *   GMRESbase::iterate (Utility/Solvers/GMRESbase.h:16,  cfdv_gmres
 *     MPI_GMRES.h:125-220)
 *   GMRESbase::update (GMRESbase.h:21, MPI_GMRES.h:224)  cfdv_update
 *   RMSErr (MPIBinaryConfiguration.h:138-142,            cfdv_rms
 *     FDV/Function/MPI_RMSError.h:21-75)
 *   MPI_TecplotOut s1..s4 (Utility/IO/MPI_TecplotOut.h)  cfdv_get_fdv_params + cfdv_get_state
 *
 * Conventions: every call returns 0 on success or a cfdv_status code; the message of
 * the last failure is cfdv_last_error(ctx).  No exception crosses the boundary.  A
 * context belongs to one host thread and one CUDA device (the current device at
 * cfdv_create); all work is ordered on the context's stream and the library
 * synchronises only where a result comes back to the host.  Layouts: U is node-major
 * [n_nodes][neqn] (the reference's global DOF order neqn*node + eq); element
 * matrices are column-major per element, R_e(i,j) at R[e*Ke*Ke + j*Ke + i]
 * (Utility/Tensor.h:89-92), with Ke = nnod*neqn.
 */
#ifndef CFDV_GPU_H
#define CFDV_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfdv_ctx cfdv_ctx;

typedef enum {
  CFDV_OK = 0,
  CFDV_ERR_ARG = 1,        /* bad argument or size */
  CFDV_ERR_CUDA = 2,       /* a CUDA runtime call failed */
  CFDV_ERR_MESH = 3,       /* degenerate or inverted element / face */
  CFDV_ERR_NONFINITE = 4,  /* NaN/Inf in an element matrix, rhs or Krylov scalar */
  CFDV_ERR_ALLOC = 5,      /* device allocation failed */
  CFDV_ERR_STATE = 6,      /* call out of order (e.g. cfdv_gmres before cfdv_form) */
  CFDV_ERR_NOT_CONVERGED = 7
} cfdv_status;

/* Mesh as the reference loads it (LoadBinary.h:156-246): 0-based node ids, the
 * element's nnod node ids in reference order, and nface boundary codes per element
 * (0 = interior face).  2D: nnod 4, nface 4; 3D: nnod 8, nface 6. */
typedef struct {
  int ndim;        /* 2 or 3 */
  int n_nodes;
  int n_elements;
  const double* x; /* [n_nodes][ndim] */
  const int* conn; /* [n_elements][nnod] */
  const int* bc;   /* [n_elements][nface] */
} cfdv_mesh;

/* aero + control parameters (MPIBinaryConfiguration.h:29-69, Thermo.h:22-33) */
typedef struct {
  double gamma, mach, reynolds, prandtl, tinf, twall;
  int adiabatic;
  int physical_3d_flux; /* 0: as the reference (3D convective flux F = 0); 1: F evaluated */
} cfdv_params;

typedef enum { CFDV_PREC_FP64 = 0, CFDV_PREC_MIXED = 1 } cfdv_precision;
typedef enum { CFDV_GMRES_REFERENCE = 0, CFDV_GMRES_CORRECT = 1 } cfdv_gmres_mode;

typedef struct {
  int mode;       /* cfdv_gmres_mode: REFERENCE reproduces MPI_GMRES::iterate (restart count,
                     tol = ||b||*1e-9 inner break, rotate_and_check, back substitution);
                     CORRECT is restarted GMRES(m) to rtol with Givens QR and textbook back
                     substitution; its Gram-Schmidt is `orth` below with engine 0 (the host
                     driver and the Python binding pass 2, delayed CGS2), MGS with engine 1 */
  int m;          /* Krylov dimension (control "gmresiter") */
  int restarts;   /* REFERENCE: restart count (control "gmresrestart"); CORRECT: maximum */
  double rtol;    /* CORRECT: stop when ||b - A du|| / ||b|| < rtol */
  int precision;  /* cfdv_precision: MIXED = FP32 element matrices and matvec inside
                     FP64 iterative refinement (CORRECT mode only) */
  int true_residual; /* 1: report ||b - A du||/||b|| with an extra FP64 product */
  int engine;        /* CORRECT mode: 0 = the whole solve as one persistent cooperative kernel
                        (no host round trip per Arnoldi step), 1 = host-driven (one kernel per
                        pass, Hessenberg column read back every step) */
  int precond;       /* CORRECT mode: 1 = right node-block Jacobi preconditioning (the inverse of
                        each node's assembled neqn x neqn diagonal block); the stopping test
                        stays the true residual of the unpreconditioned system.  0 = none */
  int orth;          /* CORRECT mode, engine 0: 0 = classical Gram-Schmidt applied twice (4 grid
                        barriers per Arnoldi step; m <= 62), 1 = modified Gram-Schmidt as the
                        reference's Arnoldi (MPI_GMRES.h:164-181; j+3 barriers per step j),
                        2 = delayed CGS2: the second projection of a step's vector is taken in
                        the next step's single reduction (two passes over the basis and 3
                        synchronisations per step; m <= 62; in 2D the two around the product
                        wait only for the blocks owning neighbouring nodes and elements),
                        3 = delayed CGS2 with grid barriers at all 3 (bitwise equal to 2) */
  int warm_start;    /* CORRECT mode, engine 0: 1 = start from the context's last solution
                        (the previous step's dU) instead of zero; the stopping test stays
                        ||b - A du|| / ||b|| < rtol.  0 = from zero, as the reference does */
} cfdv_gmres_opts;

typedef struct {
  double tol;          /* REFERENCE: ||b||*1e-9 ; CORRECT: rtol*||b|| */
  double bnorm;
  int n_est;           /* inner-iteration Givens residual estimates written to est */
  int est_capacity;    /* caller buffer sizes */
  double* est;
  int gfinal_capacity;
  double* gfinal;      /* g(m) after each restart's rotation (MPI_GMRES.h:202-203) */
  int n_restarts;
  int n_matvec;        /* EBE products issued */
  double true_rel_res; /* when requested */
} cfdv_gmres_report;

/* ---- lifetime --------------------------------------------------------------- */
/* Create a context on the current CUDA device; uploads the mesh, builds the Dirichlet
 * row masks of ApplyBC (flags per LoadBinary.h:264-318), the node->element CSR used by
 * the scatter, and element lengths (CalcLength.h:34-66). */
int cfdv_create(const cfdv_mesh* mesh, const cfdv_params* params, cfdv_ctx** out);
/* Replace the mesh (e.g. after host-side refinement); state and matrices are reset. */
int cfdv_upload_mesh(cfdv_ctx* ctx, const cfdv_mesh* mesh);
/* Adaptive (hanging-node) elements after a host refinement, replacing the reference's
 * "adap" file load (LoadBinary.h:247-261 into Element::adap / Element::Hnm, Element.h:39-40):
 * elements[k] carries hnm[k*nnod*nnod ...], Hnm(N, M) at N + nnod*M (the reference Tensor's
 * storage).  Formation then transforms the element's shape functions (MeshRefine2D.h:877-952,
 * FDVGalerkin.h:183-201, 488-497; calc_TF_norm3D.h:25-66).  n = 0 clears the set;
 * cfdv_upload_mesh clears it too.  Element ids must be distinct and in range. */
int cfdv_set_adaptive(cfdv_ctx* ctx, int n, const int* elements, const double* hnm);
void cfdv_destroy(cfdv_ctx* ctx);
const char* cfdv_last_error(const cfdv_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for event timing by the caller. */
int cfdv_get_stream(cfdv_ctx* ctx, void** stream);

/* ---- state ------------------------------------------------------------------ */
/* Upload conserved U [n_nodes*neqn] from host memory. */
int cfdv_set_state(cfdv_ctx* ctx, const double* U, size_t n);
/* Set U from binary node records {x[ndim], rho, v[ndim], T} (LoadBinary.h:156-205). */
int cfdv_load_node_records(cfdv_ctx* ctx, const double* records, size_t n_nodes);
/* Read U and U0 (state before the last update); either pointer may be NULL. */
int cfdv_get_state(cfdv_ctx* ctx, double* U, double* U0, size_t n);
/* Device pointer of U (resident state; valid until the context is destroyed). */
int cfdv_state_device_ptr(cfdv_ctx* ctx, double** U);

/* ---- the step --------------------------------------------------------------- */
/* dt = cfl * min_e min_nodes cleng/(|v| + sqrt(1.4 cgas T)) (MPI_CFL.h:7-56). */
int cfdv_cfl(cfdv_ctx* ctx, double cfl, double* dt);
/* Element LHS/RHS at time step dt with ApplyBC; precision MIXED also keeps FP32
 * copies of the matrices for the FP32 products. */
int cfdv_form(cfdv_ctx* ctx, double dt, int precision);
/* Element matrices formed elsewhere (e.g. by the reference's FDVGalerkin on the CPU):
 * R [E][Ke*Ke] column-major per element, rhs [E][Ke], ApplyBC already applied.  Lets
 * the GPU solver plug in at GMRESbase alone (GMRESbase.h:8-23). */
int cfdv_set_element_matrices(cfdv_ctx* ctx, const double* R, const double* rhs, int precision);
/* Solve for dU from the formed matrices (GMRESbase::iterate). */
int cfdv_gmres(cfdv_ctx* ctx, const cfdv_gmres_opts* opts, cfdv_gmres_report* report);
/* U0 = U; U += dU (GMRESbase::update). */
int cfdv_update(cfdv_ctx* ctx);
/* Per-field RMS change sqrt(sum U^2 / sum U0^2) - 1 (MPI_RMSError.h:46-52), rms[neqn]. */
int cfdv_rms(cfdv_ctx* ctx, double* rms);
/* cfdv_cfl + cfdv_form + cfdv_gmres + cfdv_update in the driver's order (main.cpp:179-197). */
int cfdv_step(cfdv_ctx* ctx, double cfl, const cfdv_gmres_opts* opts, cfdv_gmres_report* report, double* dt);
/* cfdv_step with the state in host memory: U_in [n_nodes*neqn] (null: keep the device state) is
 * copied in before the step and the state after it (unchanged when the step failed) is copied to
 * U_out (null: none), all on the context's stream with the step's single wait.  The same as
 * cfdv_set_state + cfdv_step + cfdv_get_state, one host synchronisation instead of three: a
 * driver that keeps its nodes' state on the host, as main.cpp:169-198 does, calls this. */
int cfdv_step_host(cfdv_ctx* ctx, double cfl, const cfdv_gmres_opts* opts, cfdv_gmres_report* report, double* dt,
                   const double* U_in, double* U_out);

/* ---- inspection (tests, output) --------------------------------------------- */
/* s1..s4 per element [n_elements][4] from the last cfdv_form (Tecplot cell data). */
int cfdv_get_fdv_params(cfdv_ctx* ctx, double* s);
/* Element matrices [E][Ke*Ke] (FP64) and rhs [E][Ke] from the last cfdv_form. */
int cfdv_get_element_matrices(cfdv_ctx* ctx, double* R, double* rhs);
/* The elements the reference's adaptive refinement marks at the current state: FDVParam's s1
 * of the element above `threshold` (0.8 in the reference, RefineListAdaptive.h:25-36),
 * computed on the device from U; ascending element ids, min(*n, capacity) of them written to
 * elements, *n = how many.  The dependency closure and the refinement itself stay on the host
 * (AdaptiveRefineList, MeshRefine2D); the refined mesh comes back through cfdv_upload_mesh,
 * cfdv_load_node_records (or cfdv_set_state) and cfdv_set_adaptive. */
int cfdv_refine_marks(cfdv_ctx* ctx, double threshold, int* elements, int capacity, int* n);
/* The same for the n elements ids[0..n): R [n][Ke*Ke], rhs [n][Ke] and s1..s4 [n][4] (any
 * may be NULL), without copying the whole mesh's matrices -- the reference's elements[e]->R,
 * ->rhs and FDVParam (Element.h:33-34, FDVParam.h:15-111) for a sample of e. */
int cfdv_get_element_subset(cfdv_ctx* ctx, int n, const int* ids, double* R, double* rhs, double* s);
/* Assembled rhs b [n_nodes*neqn] (MPI_GMRES::compose_rhs, MPI_GMRES.h:369-438). */
int cfdv_get_rhs_vector(cfdv_ctx* ctx, double* b);
/* dU of the last solve [n_nodes*neqn]. */
int cfdv_get_du(cfdv_ctx* ctx, double* du);
/* y = A x (transpose = 1: A^T x) with the formed matrices, host vectors. */
int cfdv_matvec(cfdv_ctx* ctx, const double* x, double* y, int precision, int transpose);

/* ---- measurement -------------------------------------------------------------- */
typedef struct {
  long launches;      /* element-pass launches of the EBE product while profiling */
  double total_ms;    /* their summed device time (CUDA events on the context stream) */
  double bytes;       /* algorithmic bytes of those launches: E*Ke^2*s_R + DOF*8 + E*Ke*s_R each */
  long form_launches;
  double form_ms;
  long kernel_launches; /* every kernel this context launched since cfdv_profile() */
  long solves;          /* single-launch GMRES solves (engine 0) and their device time */
  double solve_ms;
  double solve_bytes;   /* algorithmic bytes of those solves: per product E*Ke^2*s_R + 2*DOF*8,
                           per Arnoldi step (j+2) DOF vectors, per cycle (k+2) DOF vectors */
  double matvec_ms;     /* the whole EBE products of the `launches` above (element pass and node
                           pass, gather-multiply-scatter), summed device time */
  double matvec_bytes;  /* their algorithmic bytes: E*Ke^2*s_R + DOF*(8 + 8) each (matrices once,
                           x read, y written) */
} cfdv_kernel_stats;
int cfdv_profile(cfdv_ctx* ctx, int enable);
int cfdv_profile_read(cfdv_ctx* ctx, cfdv_kernel_stats* out);

/* ---- discrete adjoint and tangent of the step ------------------------------------- */
/* The reference has no adjoint; these entry points differentiate the CORRECT-mode step
 * (dt = CFL(U), A(U,dt) dU = b(U,dt), U += dU) exactly, through the same physics as
 * cfdv_form, by forward-mode dual numbers per element.  The element residual is
 * r_e = rhs_e - R_e dU_e with dU fixed; Dirichlet rows (ApplyBC) are constant.
 *
 * Objective: the wall x-force F_x = sum over element faces with boundary code wall_bc of
 * the face integral of p n_x - (1/Re) tau_xj n_j (2-point Gauss per face direction; n the
 * outward normal of the fluid element, p and T interpolated from the nodes, tau from the
 * element's velocity gradient at the face point), and J = (1/N) sum_{n=1..N} F_x(U_n) over
 * an N-step run from the loaded node records.  Parameters: the Mach number (gas constants
 * Cv, cgas, cmach and the initial rho E through Cv) and the initial temperature of each
 * wall node (the nodes of the wall_bc faces; an isothermal wall keeps it through the
 * Dirichlet energy row). */
typedef struct {
  int n_steps;          /* N steps from the records of cfdv_load_node_records */
  int checkpoint_every; /* k: the forward run keeps U every k steps; the backward sweep
                           recomputes each segment's states from its checkpoint.  The
                           element matrices of the recomputed steps, and of each segment's
                           last step from the forward run, stay on the device for their
                           reverse steps, as many sets as fit beside a reserve of free
                           memory (recomputed steps first); the other reverse steps form
                           theirs again */
  double cfl;
  int m, restarts;      /* GMRES(m), at most `restarts` cycles, CORRECT mode, node-block */
  double rtol;          /* Jacobi; forward, tangent and adjoint solves to this rtol */
  int precision;        /* cfdv_precision of every solve (MIXED: FP32 inner products) */
  int wall_bc;          /* boundary code of the wall faces */
  int max_kept_sets;    /* element-matrix sets kept on the device for the reverse steps (see
                           checkpoint_every): 0 = as many as fit, n > 0 = at most n, -1 = none
                           (every reverse step forms its matrices again) */
} cfdv_adjoint_opts;

typedef struct {
  double J;             /* (1/N) sum_{n=1..N} F_x(U_n) */
  double dJ_dmach;
  double dJ_dtwall;     /* all wall-node temperatures moved together */
  int n_wall_nodes;     /* written: number of wall nodes */
  int wall_capacity;    /* size of the two caller buffers below (may be 0) */
  int* wall_nodes;      /* node ids of the wall nodes, ascending */
  double* dJ_dtnode;    /* dJ / d T0 of each wall node */
  double forward_ms;    /* device time of the forward run */
  double backward_ms;   /* device time of the backward sweep, recomputation included */
  int forward_matvecs;  /* EBE products of all forward solves (recomputation included) */
  int adjoint_matvecs;  /* EBE products of the transposed solves */
  int kept_matrix_sets; /* element-matrix sets kept: recomputed steps', then segment ends' */
  int reverse_forms;    /* formations run by reverse steps (the others reused kept sets) */
} cfdv_adjoint_result;

/* Vector-Jacobian product of the element residuals at the current U and the dt of the
 * last cfdv_form: gU = sum_e P_e^T (d r_e / d U_e)^T mu_e (host vectors [n_nodes*neqn]),
 * g_dt = mu^T dr/ddt, g_mach = mu^T dr/dMach, for the step solution du. */
int cfdv_vjp(cfdv_ctx* ctx, const double* mu, const double* du, double* gU, double* g_dt, double* g_mach);
/* Jacobian-vector product: dr = (dr/dU) tU + (dr/ddt) t_dt + (dr/dMach) t_mach, assembled. */
int cfdv_jvp(cfdv_ctx* ctx, const double* du, const double* tU, double t_dt, double t_mach, double* dr);
/* L_e = sum over unmasked rows of mu_e (rhs_e - R_e du_e) per element [n_elements] (checks). */
int cfdv_element_functional(cfdv_ctx* ctx, const double* mu, const double* du, double* L);
/* F_x at the current U; dF_dU [n_nodes*neqn] and dF_dmach may be NULL. */
int cfdv_wall_force(cfdv_ctx* ctx, int wall_bc, double* F, double* dF_dU, double* dF_dmach);
/* The wall nodes of wall_bc (ascending ids, up to capacity) and their number. */
int cfdv_wall_nodes(cfdv_ctx* ctx, int wall_bc, int* ids, int capacity, int* n);
/* Forward run with checkpoints, then the reverse sweep: lambda_N = (1/N) dF/dU(U_N),
 * mu_n = A_n^-T lambda_{n+1}, lambda_n = lambda_{n+1} + (dr_n/dU)^T mu_n
 * + (mu_n^T dr_n/ddt) d dt_n/dU + [n >= 1] (1/N) dF/dU(U_n); gradients from lambda_0.
 * Each transposed solve starts from the previous reverse step's mu.  The context's state is
 * U_N afterwards, with no element matrices formed (the transposed solves leave them
 * transposed): cfdv_form before the next solve. */
int cfdv_adjoint(cfdv_ctx* ctx, const cfdv_adjoint_opts* opts, cfdv_adjoint_result* res);
/* FP64 tangent-linear run along (dmach, dT_wall[n_wall_nodes], NULL = 0): J and dJ. */
int cfdv_tangent(cfdv_ctx* ctx, const cfdv_adjoint_opts* opts, double dmach, const double* dT_wall, double* J,
                 double* dJ);

/* ---- EBE product without device allocation ------------------------------------ */
/* No counterpart in the reference; it exists for callers of this library that may not
 * allocate device memory.  Examples: a solver plug-in that runs inside an application
 * whose own memory pool has already claimed the GPU's free memory, so a cudaMalloc from
 * the library would fail; or code running between other streams' work, where cudaFree
 * (and often cudaMalloc) would synchronise the whole device.  A context (cfdv_create)
 * allocates its buffers, so such callers use this call instead.
 *
 * y = A x (transpose = 1: A^T x) for element matrices R [n_elements][Ke*Ke] (column-
 * major per element, as above), computed by the same element and node passes as
 * cfdv_matvec.  Every pointer is memory of the CURRENT device (cudaMalloc'd or from the
 * caller's pool) or managed memory, owned by the caller; host memory (pageable or pinned)
 * and another GPU's memory are rejected with CFDV_ERR_ARG before any GPU work:
 *   conn     [n_elements][nnod] node ids (nnod 4 in 2D, 8 in 3D), as in cfdv_mesh
 *   node_ptr [n_nodes+1], node_idx [n_elements*nnod]: for node n, the entries
 *            node_idx[node_ptr[n] .. node_ptr[n+1]) are e*nnod + l for every element e
 *            and local node l with conn[e*nnod + l] == n, in increasing order
 *   x, y     [n_nodes*neqn], neqn = ndim + 2; y is overwritten, x and y must not overlap
 * The element products go to one scratch array compiled into the library, a static
 * device array of CFDV_STATIC_SCRATCH_DOUBLES doubles (16 MiB) that every GPU which loads
 * the library keeps until the process exits.  So n_elements * Ke must not exceed
 * CFDV_STATIC_SCRATCH_DOUBLES (2D quads: 131072 elements, 3D hexes: 52428); a larger
 * mesh returns CFDV_ERR_TOO_LARGE before any GPU work.  The call allocates nothing.
 * The first call on a device looks up the array's device address (with that device
 * current) and keeps it; make that first call before any stream capture begins.  After a
 * cudaDeviceReset the kept address no longer names device memory, and the next call looks
 * it up again: that call, too, belongs outside a capture.  The
 * work is queued on `stream` (a cudaStream_t; NULL = the default stream) and the call
 * returns without waiting for it.  All calls share the one array, which keeps the last
 * call's contents: calls whose work overlaps on a GPU (different streams, or different
 * host threads, without ordering between them) race on it and give wrong results. */
#define CFDV_STATIC_SCRATCH_DOUBLES 2097152
#define CFDV_ERR_TOO_LARGE 8
int cfdv_ebe_matvec_static(int ndim, int n_nodes, int n_elements, const int* conn, const int* node_ptr,
                           const int* node_idx, const double* R, const double* x, double* y, int transpose,
                           void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CFDV_GPU_H */
