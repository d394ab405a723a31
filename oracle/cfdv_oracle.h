/* CPU restatement of the CFDV per-step FDV path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker the parity tests (tests/), __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg compare the CUDA path against.  It is never
 * linked into, loaded by, or called from the product library (libcfdv_gpu.so).
 * Every function cites the reference file:line it restates; it is pinned against
 * the reference itself (oracle/_ref/cfdv_ref, built from the unmodified sources)
 * by tests/test_oracle_pin.py.
 *
 * Layouts: U is node-major [Nn][neqn]; x is [Nn][ndim]; conn is [E][nnod];
 * bc is [E][nface]; element matrices are column-major per element,
 * R_e(i,j) at R[e*Ke*Ke + j*Ke + i] (the reference Tensor layout, Tensor.h:89-92).
 */
#ifndef CFDV_ORACLE_H
#define CFDV_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int ndim, nnod, neqn, nbnod, nface;
  int n_nodes, n_elements;
  const double* x;   /* [Nn][ndim] */
  const int* conn;   /* [E][nnod]  */
  const int* bc;     /* [E][nface] */
  /* adaptive (hanging-node) elements (Element.h:39-40, LoadBinary.h:247-261): hnm_idx[e] is
   * the row of hnm that applies to element e, -1 for a plain element (both may be null);
   * hnm[k] holds Hnm(N, M) at N + nnod*M */
  const int* hnm_idx;
  const double* hnm;
} oracle_mesh;

typedef struct {
  double gamma, mach, reynolds, prandtl, tinf, twall;
  int adiabatic;
} oracle_aero;

/* node Dirichlet flags per DOF, set by the faces (LoadBinary.h:264-318) */
void oracle_dirichlet(const oracle_mesh* m, const oracle_aero* a, uint8_t* dir /*[Nn*neqn]*/);
/* per-element Dirichlet row mask after ApplyBC (ApplyBC.h:14-133); bit i = local DOF i */
void oracle_bc_rowmask(const oracle_mesh* m, const oracle_aero* a, const uint8_t* dir, uint64_t* mask /*[E]*/);
/* conserved U from the binary node records {x, rho, v, T} (LoadBinary.h:179-196) */
void oracle_init_U(const oracle_mesh* m, const oracle_aero* a, const double* prim, double* U);
/* element characteristic length (CalcLength.h:34-110) */
void oracle_cleng(const oracle_mesh* m, double* cleng);
/* dt from the CFL condition (MPI_CFL.h:7-56); returns dt */
double oracle_cfl(const oracle_mesh* m, const oracle_aero* a, const double* cleng, const double* U, double cfl);
/* FDV parameters s1..s4 per element (FDVParam.h:15-111), [E][4] */
void oracle_fdvparam(const oracle_mesh* m, const oracle_aero* a, const double* U, double* s);
/* element LHS/RHS (FDVGalerkin.h:121-811), optionally followed by ApplyBC.
 * physical_3d_flux = 1 evaluates the 3D convective flux F that the reference drops
 * (NavierStokes3D.h:10 hides NavierStokes.h:6); 0 reproduces the reference. */
void oracle_form(const oracle_mesh* m, const oracle_aero* a, const double* U, double dt, int apply_bc,
                 int physical_3d_flux, double* R, double* rhs);

/* GMRES report: the quantities the reference prints (MPI_GMRES.h:141, 728, 203) */
typedef struct {
  double tol;            /* ||b|| * 1e-9 */
  double bnorm;
  int n_est;             /* number of inner-iteration estimates written */
  double* est;           /* caller buffer, capacity restart*m */
  double* gfinal;        /* caller buffer, capacity restart: g(m) after rotate() */
  int n_restarts_run;
  double true_rel_res;   /* ||b - A du|| / ||b|| after the solve */
} oracle_gmres_report;

/* b = sum_e scatter(rhs_e) (MPI_GMRES.h:369-389) */
void oracle_compose_rhs(const oracle_mesh* m, const double* rhs, double* b);
/* y = sum_e P_e^T R_e P_e x (MPI_GMRES.h:570-640 loop order) */
void oracle_ebe_matvec(const oracle_mesh* m, const double* R, const double* x, double* y);
/* y = sum_e P_e^T R_e^T P_e x (transposed EBE product) */
void oracle_ebe_matvec_t(const oracle_mesh* m, const double* R, const double* x, double* y);
/* the reference's restarted GMRES, quirks included (MPI_GMRES.h:125-220, 696-780) */
int oracle_gmres_ref(const oracle_mesh* m, const double* R, const double* rhs, int mdim, int restart,
                     double* du, oracle_gmres_report* rep);
/* textbook restarted GMRES(m) with MGS + Givens to ||b-A du||/||b|| < rtol */
int oracle_gmres_correct(const oracle_mesh* m, const double* R, const double* rhs, int mdim, int max_restart,
                         double rtol, double* du, oracle_gmres_report* rep);

/* one full FDV step of the reference driver (main.cpp:169-198) on U in place.
 * mode 0 = reference GMRES, 1 = textbook GMRES to rtol.  U0 receives U before the update.
 * Returns dt in *dt_out and the per-field RMS line (MPI_RMSError.h:46-52) in rms[neqn]. */
int oracle_step(const oracle_mesh* m, const oracle_aero* a, const double* cleng, double cfl, int mdim,
                int restart, int mode, double rtol, int physical_3d_flux, double* U, double* U0,
                double* dt_out, double* rms, oracle_gmres_report* rep);

/* Gauss-Legendre points/weights of GaussQuad::get_gauss (GaussQuad.h:116-159) */
void oracle_gauss(int n, double* zeta, double* w);

#ifdef __cplusplus
}
#endif
#endif
