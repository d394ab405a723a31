// FDV element formation as the phases of one thread block ("CTA") per element.
//
// Per element the CTA computes what the reference builds in FDVGalerkin::operator()
// (FDV/FDVGalerkin.h:121-154) followed by ApplyBC (FDV/Function/ApplyBC.h:14-133):
//   load      node unpack (NodeUnpack.h:9-29), boundary face list
//   domain    one thread per Gauss point: FDVParam (FDVParam.h:15-111), shape functions,
//             Gauss-point state, stress, SUPG/discontinuity-capturing test function
//             (FDVGalerkin.h:225-387), flux Jacobians and the rhs flux terms
//   hmat      all threads: h_ij = -dt s3 c_ij + dt^2/2 (a_i+b_i)(s2 a_j + s4 b_j)
//             (FDVGalerkin.h:611-628; for a face m_ij = -h_ij, :698-715)
//   contract  R(N r, M s) += sum_k B_k(N,M) C_k(r,s) with
//             B = wJ Phi_N Phi_M (C = I), wJ(Psi_N sum_j dPhi_Mj - dPhi_Ni Phi_M) (C = X_i),
//             wJ dPhi_Ni dPhi_Mj (C = h_ij); X_i = dt (s1 a_i + s3 b_i) = -g_i = nd_i
//             (FDVGalerkin.h:405-451)
//   faces     same three phases per boundary face with 0 != bc < 100
//             (FDVGalerkin.h:455-533, 643-756; TFNorm2D TestFunctions1D.h:73-82,
//             TFNorm3D calc_TF_norm3D.h:9-167, eval1dboundary.h, eval2dboundary.h)
//   write     ApplyBC through the precomputed Dirichlet row mask, then a coalesced
//             store of R (column-major, FP64 or FP32) and rhs.
// Every phase is a host/device function of (block state, thread id) so that the
// same code runs in the CUDA kernel (phases separated by __syncthreads()).
#pragma once
#include "fdv_physics.cuh"

namespace cfdv {

#ifndef CFDV_FORM3D_BLOCKS
#define CFDV_FORM3D_BLOCKS 5  // 3D formation blocks per SM the register allocation is sized for
#endif

template <int NDIM>
struct FormTraits {
  static constexpr int NNOD = (NDIM == 2) ? 4 : 8;
  static constexpr int NEQ = NDIM + 2;
  static constexpr int KE = NNOD * NEQ;
  static constexpr int Q = (NDIM == 2) ? 4 : 8;      // domain Gauss points
  static constexpr int NBN = (NDIM == 2) ? 2 : 4;    // nodes per face
  static constexpr int QF = (NDIM == 2) ? 2 : 4;     // Gauss points per face
  static constexpr int NFACE = (NDIM == 2) ? 4 : 6;
  static constexpr int THREADS = (NDIM == 2) ? 64 : 128;
  static constexpr int RS = NEQ * NEQ;
  // contraction: thread `tid` owns the (node N, equation pair r,s) pairs p = tid + k*THREADS,
  // p = (r*NEQ + s)*NNOD + N, with one accumulator per column node M
  static constexpr int NPAIR = NNOD * RS;
  static constexpr int PAIRS = (NPAIR + THREADS - 1) / THREADS;
  // coefficient rows per Gauss point for the column node M: Phi_M, dPhi_M,j (j < NDIM) and,
  // in 2D, S_M = sum_j dPhi_M,j for the upwind term
  static constexpr int NCOEF = 1 + NDIM + (NDIM == 2 ? 1 : 0);
  static constexpr int MIN_BLOCKS = (NDIM == 2) ? 12 : CFDV_FORM3D_BLOCKS;  // resident blocks per SM (register cap)
};

// hex8 faces (FiniteElement/get_face.h:106-164), quad4 edges (get_face.h:80-89)
// hex8 face f lists nodes {3,2,1,0}, {0,1,5,4}, {1,2,6,5}, {2,3,7,6}, {3,0,4,7}, {6,7,4,5},
// packed four bits per node so that the lookup needs no memory
CFDV_HD CFDV_INLINE int face_node(int ndim, int f, int i) {
  if (ndim == 2) return (f + i) & 3;
  const unsigned long long lo = 0x6732562145100123ull, hi = 0x54767403ull;  // faces 0-3, 4-5
  const unsigned long long w = (f < 4) ? (lo >> (16 * f)) : (hi >> (16 * (f - 4)));
  return (int)((w >> (4 * i)) & 15ull);
}

// ---- adaptive (hanging-node) elements ---------------------------------------------------
// An adaptive element carries Hnm (nnod x nnod, Hnm(N, M) at H[N + nnod*M], the reference
// Tensor's storage).  Its domain shape functions become Phi_M <- sum_N Phi_N Hnm(N, M) and
// dPxi(M, j) likewise (MeshRefine2D.h:877-900, applied at FDVGalerkin.h:183-186, 198-201)
// before the Jacobian; the 2D streamline-upwind term keeps the Jacobian of the untransformed
// shape functions (FDVGalerkin.h:237-240).  A 3D boundary face takes its geometry from the
// rows of Hnm x at its nodes (calc_TF_norm3D.h:25-66) and transforms its face shape
// functions with the face's block of Hnm (MeshRefine2D.h:904-951 via FDVGalerkin.h:489-497;
// the face derivatives stay as computed).  2D faces are unchanged (FDVGalerkin.h:481-484).
template <int NDIM>
CFDV_HD CFDV_INLINE void hnm_shape(const double* H, double* Phi, double (*dPxi)[3]) {
  constexpr int NNOD = (NDIM == 2) ? 4 : 8;
  double P[NNOD], D[NNOD][3];
  for (int M = 0; M < NNOD; M++) {
    P[M] = 0.0;
    for (int j = 0; j < NDIM; j++) D[M][j] = 0.0;
  }
  for (int N = 0; N < NNOD; N++)
    for (int M = 0; M < NNOD; M++) {
      const double h = H[N + NNOD * M];
      P[M] = RN_ADD(P[M], RN_MUL(Phi[N], h));
      for (int j = 0; j < NDIM; j++) D[M][j] = RN_ADD(D[M][j], RN_MUL(dPxi[N][j], h));
    }
  for (int M = 0; M < NNOD; M++) {
    Phi[M] = P[M];
    for (int j = 0; j < NDIM; j++) dPxi[M][j] = D[M][j];
  }
}

// the 2D isoparametric Jacobian of the untransformed shape functions at z (x4: node x)
CFDV_HD CFDV_INLINE void plain_jac_2d(const double* z, const double* const* x4, double (*jac)[3]) {
  double ph[4], dpx[4][3];
  shape_fn<2>(z, ph, dpx);
  for (int i = 0; i < 2; i++)
    for (int k = 0; k < 2; k++) {
      double j = 0.0;
      for (int N = 0; N < 4; N++) j = RN_ADD(j, RN_MUL(dpx[N][k], x4[N][i]));
      jac[i][k] = j;
    }
}

// 3D face f of an adaptive element: the face nodes' positions sum_M Hnm(N, M) x_M (xe: the
// element's node coordinates), face order
CFDV_HD CFDV_INLINE void hnm_face_nodes_3d(const double* H, const double* const* xe, int f, double (*xl)[3]) {
  for (int j = 0; j < 4; j++) {
    const int N = face_node(3, f, j);
    for (int k = 0; k < 3; k++) {
      double s = 0.0;
      for (int M = 0; M < 8; M++) s = RN_ADD(s, RN_MUL(H[N + 8 * M], xe[M][k]));
      xl[j][k] = s;
    }
  }
}

// 3D face f of an adaptive element: phib_M <- sum_N phib_N Hnm(n_N, n_M) over the face nodes
CFDV_HD CFDV_INLINE void hnm_face_phi_3d(const double* H, int f, double* phib) {
  double pt[4] = {0.0, 0.0, 0.0, 0.0};
  for (int N = 0; N < 4; N++)
    for (int M = 0; M < 4; M++) pt[M] = RN_ADD(pt[M], RN_MUL(phib[N], H[face_node(3, f, N) + 8 * face_node(3, f, M)]));
  for (int M = 0; M < 4; M++) phib[M] = pt[M];
}

// one Gauss point's worth of coefficients
template <int NDIM>
struct GpGeom {  // isoparametric map at the Gauss point (dead once the flow state exists)
  double jac[3][3];  // dx_i / dxi_k
  double inv[3][3];  // adjugate (3D)
  double iJ;         // 1 / det
  double dPxi[FormTraits<NDIM>::NNOD][3];
  double pjac[NDIM == 2 ? 3 : 1][3];  // 2D adaptive element: Jacobian of the plain shape functions
};

template <int NDIM>
struct GpSlot {
  static constexpr int NNOD = FormTraits<NDIM>::NNOD;
  alignas(16) double cM[FormTraits<NDIM>::NCOEF][NNOD];  // contraction coefficients, row-major
  double wJ;
  double Phi[NNOD];
  double dPhi[NNOD][3];
  double Psi[NNOD];
  double en[3];
  double H[9][25];     // c, then h (domain) or m (face)
  double P[NDIM][5];   // rhs coefficient per direction and equation
  union {
    GpState st;          // flow state (until the Jacobians are formed)
    double X[NDIM][25];  // dt (s1 a + s3 b)
  };
  union {
    GpGeom<NDIM> g;
    double F[NDIM + 1][5];  // Fbar(i, r) for i < NDIM, div F(r) in row NDIM
  };
};

template <int NDIM>
struct FormShared {
  using T = FormTraits<NDIM>;
  NodePrim nd[T::NNOD];
  int faces[T::NFACE];
  int codes[T::NFACE];
  int nfaces;
  int hnm;  // row of a.hnm for an adaptive element, -1 otherwise
  uint64_t mask;
  double Mn[T::NNOD], Ren[T::NNOD];  // node Mach and Reynolds numbers
  double s[4];                        // s1..s4 of the element
  double dt, dtsq_2;                  // time step of the formation and dt^2 / 2
  double rhs[T::KE];
  GpSlot<NDIM> slot[T::Q];
  union {
    // A(q, i) = a + b and D(q, i) = s2 a + s4 b of the domain Gauss points (a, b until step 7)
    double AD[T::Q][2][NDIM][25];
    // the element matrix, column-major, accumulated from the domain contraction on
    double Rt[T::KE * T::KE];
  };
};

// A and D of a Gauss point: the domain points keep them beside the element matrix; a face
// point, evaluated after the domain contraction, borrows the h storage of domain slot QF + q
template <int NDIM>
CFDV_HD CFDV_INLINE double (*gp_A(FormShared<NDIM>& sh, int q, bool face))[25] {
  return face ? sh.slot[FormTraits<NDIM>::QF + q].H : sh.AD[q][0];
}
template <int NDIM>
CFDV_HD CFDV_INLINE double (*gp_D(FormShared<NDIM>& sh, int q, bool face))[25] {
  return face ? sh.slot[FormTraits<NDIM>::QF + q].H + NDIM : sh.AD[q][1];
}

// The Gauss points of a pass: the element's Q domain points over its NNOD nodes, or the
// QF points of one boundary face over the face's NBN nodes (face-local node numbering)
template <int NDIM, bool FACE>
struct Pass {
  using T = FormTraits<NDIM>;
  static constexpr int NQ = FACE ? T::QF : T::Q;
  static constexpr int NN = FACE ? T::NBN : T::NNOD;
};
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE const NodePrim& pass_node(const FormShared<NDIM>& sh, int f, int N) {
  return sh.nd[FACE ? face_node(NDIM, f, N) : N];
}



// FDVParam.h:15-111, per node: Mach and Reynolds numbers
template <int NDIM, class S>
CFDV_HD CFDV_INLINE void node_mach_re(const GasT<S>& g, const NodePrimT<S>& n, S* M, S* Re) {
  S vv = 0;
  for (int i = 0; i < NDIM; i++) vv = RN_ADD(vv, RN_MUL(n.v[i], n.v[i]));
  const S V = sqrt(vv);
  S Tn = n.T;
  if (Tn < 1.0E-12) Tn = 0;
  const S snd = sqrt(RN_MUL(RN_MUL(g.gamma, g.cgas), Tn));
  *M = (snd < 1.0E-12) ? S(0) : RN_DIV(V, snd);
  *Re = RN_DIV(RN_MUL(n.rho, V), gas_mu(g, Tn));
}

// FDVParam.h:15-111 over the element's nodes: which = 0 gives s1 and s2 from the Mach
// numbers, which = 1 gives s3 and s4 from the Reynolds numbers, into s[2*which], s[2*which+1]
template <int NNOD, class S>
CFDV_HD CFDV_INLINE void fdv_pair(const S* val, int which, S* s) {
  S vmin = val[0], vmax = val[0];
  for (int b = 1; b < NNOD; b++) {
    vmax = fmax(vmax, val[b]);
    vmin = fmin(vmin, val[b]);
  }
  const double eps = 0.0000001;
  // the spread stays in FP64: max ~ min cancels
  const S r = RN_DIV(sqrt(RN_SUB(RN_MUL(vmax, vmax), RN_MUL(vmin, vmin))), RN_ADD(vmin, eps));
  S sv = 0.0;  // r == 0.01 exactly: the reference keeps the previous element's value
  if (r > 0.01) sv = fmin(r, S(1.0));
  else if (r < 0.01 && vmin >= 10E-10) sv = 0.0;
  else if (which == 0 ? (vmin < 10E-10) : (vmin <= 10E-10)) sv = 1.0;
  s[2 * which] = sv;
  s[2 * which + 1] = 0.5 * (1 + pow(sv, 0.2));
}

// ---- domain steps ------------------------------------------------------------
// The domain part of an element runs as block-wide steps separated by barriers.  Each
// step hands independent values (one Jacobian entry, one state sum, one flux column,
// one h entry ...) to separate threads; every value is computed by the same expression,
// in the same order, as a single thread would compute it for the whole Gauss point.

// Gauss point q: natural coordinates, returns the weight (GaussQuad.h:69-112 loop order:
// q = (i*2 + j)*2 + k)
template <int NDIM>
CFDV_HD CFDV_INLINE double gp_point(const FormArgs& a, int q, double* z) {
  double w = 1.0;
  for (int d = 0; d < NDIM; d++) {
    const int bit = (q >> (NDIM - 1 - d)) & 1;
    z[d] = a.gz[bit];
    w *= a.gw[bit];
  }
  return w;
}

// step 0: node unpack (NodeUnpack.h:9-29) with the node's Mach and Reynolds numbers,
// boundary face list, shape functions
template <int NDIM>
CFDV_HD CFDV_INLINE void step_load(const FormArgs& a, FormShared<NDIM>& sh, int e, int tid) {
  using T = FormTraits<NDIM>;
  if (tid < T::NNOD) {
    const int n = a.conn[(size_t)e * T::NNOD + tid];
    node_unpack<NDIM>(a.gas, a.U + (size_t)n * T::NEQ, a.x + (size_t)n * NDIM, sh.nd[tid]);
    node_mach_re<NDIM>(a.gas, sh.nd[tid], &sh.Mn[tid], &sh.Ren[tid]);
  }
  if (tid == 32 % T::THREADS) {
    int nf = 0;
    for (int f = 0; f < T::NFACE; f++) {
      const int c = a.bc[(size_t)e * T::NFACE + f];
      if (c != 0 && c < 100) {  // FDVGalerkin.h:460
        sh.faces[nf] = f;
        sh.codes[nf] = c;
        nf++;
      }
    }
    sh.nfaces = nf;
    sh.hnm = a.hnm_idx ? a.hnm_idx[e] : -1;
    sh.mask = a.rowmask ? a.rowmask[e] : 0ull;
    sh.dt = a.dt_dev ? *a.dt_dev : a.dt;
    sh.dtsq_2 = a.dt_dev ? sh.dt * sh.dt / 2.0 : a.dtsq_2;
  }
  const int q = tid - (T::THREADS - T::Q);
  if (q >= 0) {
    double z[3];
    gp_point<NDIM>(a, q, z);
    shape_fn<NDIM>(z, sh.slot[q].Phi, sh.slot[q].g.dPxi);
    const int hi = a.hnm_idx ? a.hnm_idx[e] : -1;
    if (hi >= 0) hnm_shape<NDIM>(a.hnm + (size_t)hi * T::NNOD * T::NNOD, sh.slot[q].Phi, sh.slot[q].g.dPxi);
  }
}

// step 1: isoparametric Jacobian entries (q, i, k); FDV parameters of the element (two threads)
template <int NDIM>
CFDV_HD CFDV_INLINE void step_geom_jac(const FormArgs& a, FormShared<NDIM>& sh, int tid) {
  using T = FormTraits<NDIM>;
  if (tid < T::Q * NDIM * NDIM) {
    const int q = tid / (NDIM * NDIM), i = (tid / NDIM) % NDIM, k = tid % NDIM;
    GpSlot<NDIM>& sl = sh.slot[q];
    sl.g.jac[i][k] = geom_jac_entry<T::NNOD>(sl.g.dPxi, sh.nd, i, k);
    if (NDIM == 2 && sh.hnm >= 0 && i == 0 && k == 0) {
      double z[3];
      gp_point<NDIM>(a, q, z);
      const double* x4[4] = {sh.nd[0].x, sh.nd[1].x, sh.nd[2].x, sh.nd[3 % T::NNOD].x};
      plain_jac_2d(z, x4, sl.g.pjac);
    }
  }
  if (tid >= T::THREADS - 2) {
    const int which = tid - (T::THREADS - 2);
    fdv_pair<T::NNOD>(which ? sh.Ren : sh.Mn, which, sh.s);
  }
}

// step 2: determinant, adjugate, integration weight (one thread per Gauss point)
template <int NDIM>
CFDV_HD CFDV_INLINE void step_geom_det(const FormArgs& a, FormShared<NDIM>& sh, int tid) {
  if (tid < FormTraits<NDIM>::Q) {
    GpSlot<NDIM>& sl = sh.slot[tid];
    double z[3];
    const double w = gp_point<NDIM>(a, tid, z);
    const double J = geom_det<NDIM>(sl.g.jac, sl.g.inv);
    sl.g.iJ = RN_DIV(1.0, J);
    sl.wJ = w * J;
  }
}

// step 3: physical shape-function derivatives (q, N)
template <int NDIM>
CFDV_HD CFDV_INLINE void step_dphi(FormShared<NDIM>& sh, int tid) {
  using T = FormTraits<NDIM>;
  if (tid < T::Q * T::NNOD) {
    GpSlot<NDIM>& sl = sh.slot[tid / T::NNOD];
    const int N = tid % T::NNOD;
    geom_dphi<NDIM>(sl.g.dPxi[N], sl.g.jac, sl.g.inv, sl.g.iJ, sl.dPhi[N]);
    sl.cM[0][N] = sl.Phi[N];
    double sd = 0.0;
    for (int j = 0; j < NDIM; j++) {
      sl.cM[1 + j][N] = sl.dPhi[N][j];
      sd += sl.dPhi[N][j];
    }
    if (NDIM == 2) sl.cM[T::NCOEF - 1][N] = sd;
  }
}

// Gauss-point state sums (FDVGalerkin.h:761-797): value v of the state at slot sl is
// sum_N coef_N * field_N, coef = Phi_N or dPhi_N,c
template <int NDIM>
struct StateSums {
  static constexpr int NEQ = NDIM + 2;
  static constexpr int COUNT = 2 + NEQ + NEQ * NDIM + NDIM + NDIM + NDIM * NDIM;
};

template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void state_sum(const FormShared<NDIM>& sh, int fc, GpSlot<NDIM>& sl, int v) {
  constexpr int NEQ = NDIM + 2, NN = Pass<NDIM, FACE>::NN;
  GpState& f = sl.st;
  double* dst;
  int c = -1, kind, idx = 0;  // kind: 0 E, 1 T, 2 U[idx], 3 v[idx]
  if (v == 0) { dst = &f.E; kind = 0; }
  else if (v == 1) { dst = &f.T; kind = 1; }
  else if ((v -= 2) < NEQ) { dst = &f.U[v]; kind = 2; idx = v; }
  else if ((v -= NEQ) < NEQ * NDIM) { idx = v / NDIM; c = v % NDIM; dst = &f.dU[idx][c]; kind = 2; }
  else if ((v -= NEQ * NDIM) < NDIM) { dst = &f.v[v]; kind = 3; idx = v; }
  else if ((v -= NDIM) < NDIM) { dst = &f.dT[v]; kind = 1; c = v; }
  else { v -= NDIM; idx = v / NDIM; c = v % NDIM; dst = &f.dV[idx][c]; kind = 3; }
  double acc = 0;
  for (int N = 0; N < NN; N++) {
    const NodePrim& n = pass_node<NDIM, FACE>(sh, fc, N);
    const double coef = (c < 0) ? sl.Phi[N] : sl.dPhi[N][c];
    const double val = (kind == 0) ? n.E : (kind == 1) ? n.T : (kind == 2) ? n.U[idx] : n.v[idx];
    acc = RN_ADD(acc, RN_MUL(coef, val));
  }
  *dst = acc;
}

// step 4 (and face step 1): the state sums (q, value)
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void step_state(FormShared<NDIM>& sh, int lf, int tid) {
  using T = FormTraits<NDIM>;
  constexpr int NV = StateSums<NDIM>::COUNT, NQ = Pass<NDIM, FACE>::NQ;
  const int fc = FACE ? sh.faces[lf] : 0;
  for (int t = tid; t < NQ * NV; t += T::THREADS) state_sum<NDIM, FACE>(sh, fc, sh.slot[t / NV], t % NV);
}

// SUPG coefficient alpha(R) = coth(R/2) - 2/R with coth = cosh/sinh, in the reference's
// operation order (FDVGalerkin.h:46-50, 308-319); alpha = 0 at R == 0.
CFDV_HD CFDV_INLINE double supg_alpha(double R) {
  return (R == 0) ? 0.0 : RN_SUB(RN_DIV(cosh(R / 2.), sinh(R / 2.)), RN_DIV(2., R));
}
// The dual form keeps that value; its derivative uses d alpha / dR = 2/R^2 - 1/(2 sinh^2(R/2)),
// which for |R| < 0.1 is evaluated from its series 1/6 - R^2/120 + R^4/3024 - R^6/86400:
// the two terms of the closed form cancel to ~R^2 of their size, so at small cell Reynolds
// numbers their rounding would swamp the derivative.
CFDV_HD CFDV_INLINE Dual supg_alpha(const Dual& R) {
  const double r = R.v;
  double da;
  if (fabs(r) < 0.1) {
    const double r2 = r * r;
    da = 1.0 / 6.0 - r2 / 120.0 + r2 * r2 / 3024.0 - r2 * r2 * r2 / 86400.0;
  } else {
    const double sh = sinh(r / 2.);
    da = 2.0 / (r * r) - 1.0 / (2.0 * sh * sh);
  }
  return Dual(supg_alpha(r), (r == 0) ? 0.0 : R.d * da);
}

// 2D streamline-upwind test function Psi (FDVGalerkin.h:225-332) with discontinuity
// capturing (FDVGalerkin.h:336-387), evaluated in the reference's operation order without
// contraction (RN_*), because its exact-zero tests decide whether a term is present at all.
// jac: isoparametric Jacobian at the point, x4: the element's node coordinates.
template <class S>
CFDV_HD CFDV_INLINE void psi_2d(const double (*jac)[3], const double* const* x4, const GpStateT<S>& f,
                                const double (*dPhi)[3], S* Psi) {
  const double J_xi = RN_ADD(RN_MUL(jac[0][0], jac[0][0]), RN_MUL(jac[1][0], jac[1][0]));
  const double J_eta = RN_ADD(RN_MUL(jac[0][1], jac[0][1]), RN_MUL(jac[1][1], jac[1][1]));
  const double ixi = RN_DIV(1., sqrt(J_xi)), ieta = RN_DIV(1., sqrt(J_eta));
  const S v_xi = RN_ADD(RN_MUL(f.v[0], RN_MUL(ixi, jac[0][0])), RN_MUL(f.v[1], RN_MUL(ixi, jac[1][0])));
  const S v_eta = RN_ADD(RN_MUL(f.v[0], RN_MUL(ieta, jac[0][1])), RN_MUL(f.v[1], RN_MUL(ieta, jac[1][1])));
  const S S2 = RN_ADD(RN_MUL(f.v[0], f.v[0]), RN_MUL(f.v[1], f.v[1]));
  // element extents between opposite edge midpoints, accumulated node by node with the
  // edge-midpoint interpolants (the eta extent is taken bottom minus top)
  const double h_xi =
      RN_SUB(RN_ADD(RN_ADD(-RN_MUL(0.5, x4[0][0]), RN_MUL(0.5, x4[1][0])), RN_MUL(0.5, x4[2][0])),
             RN_MUL(0.5, x4[3][0]));
  const double h_eta =
      RN_SUB(RN_SUB(RN_ADD(RN_MUL(0.5, x4[0][1]), RN_MUL(0.5, x4[1][1])), RN_MUL(0.5, x4[2][1])),
             RN_MUL(0.5, x4[3][1]));
  const S R_xi = RN_DIV(RN_MUL(RN_MUL(f.U[0], v_xi), h_xi), f.mu);
  const S R_eta = RN_DIV(RN_MUL(RN_MUL(f.U[0], v_eta), h_eta), f.mu);
  const S al_xi = supg_alpha(R_xi);
  const S al_eta = supg_alpha(R_eta);
  const S tau = (S2 == 0) ? S(0.0)
                          : RN_DIV(RN_MUL(0.25, RN_ADD(RN_MUL(RN_MUL(al_xi, h_xi), v_xi),
                                                        RN_MUL(RN_MUL(al_eta, h_eta), v_eta))),
                                   S2);
  for (int N = 0; N < 4; N++)
    Psi[N] = RN_ADD(RN_MUL(RN_MUL(tau, f.v[0]), dPhi[N][0]), RN_MUL(RN_MUL(tau, f.v[1]), dPhi[N][1]));
  S A[2] = {0, 0};
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++) A[j] = RN_ADD(A[j], RN_MUL(f.dV[j][k], f.v[k]));
  const S gam = RN_MUL(sqrt(RN_ADD(RN_MUL(f.v[0], f.v[0]), RN_MUL(f.v[1], f.v[1]))),
                       sqrt(RN_ADD(RN_MUL(A[0], A[0]), RN_MUL(A[1], A[1]))));
  S tau_b = 0.0;
  if (gam != 0) {
    tau_b = RN_ADD(RN_DIV(RN_MUL(RN_MUL(tau, f.v[0]), A[0]), gam), RN_DIV(RN_MUL(RN_MUL(tau, f.v[1]), A[1]), gam));
    if (RN_SUB(tau_b, tau) < 0) tau_b = tau;
  }
  for (int N = 0; N < 4; N++)
    Psi[N] = RN_ADD(RN_ADD(Psi[N], RN_MUL(RN_MUL(tau_b, f.v[0]), dPhi[N][0])), RN_MUL(RN_MUL(tau_b, f.v[1]), dPhi[N][1]));
}

CFDV_HD CFDV_INLINE void supg_psi_2d(const FormShared<2>& sh, GpSlot<2>& sl) {
  const double* x4[4] = {sh.nd[0].x, sh.nd[1].x, sh.nd[2].x, sh.nd[3].x};
  psi_2d<double>(sh.hnm >= 0 ? sl.g.pjac : sl.g.jac, x4, sl.st, sl.dPhi, sl.Psi);
}

// step 5: viscosity, conductivity, stress; the 2D test function (one thread per Gauss point)
template <int NDIM>
CFDV_HD CFDV_INLINE void step_stress(const FormArgs& a, FormShared<NDIM>& sh, int tid) {
  using T = FormTraits<NDIM>;
  if (tid < T::Q) {
    GpSlot<NDIM>& sl = sh.slot[tid];
    sl.st.mu = gas_mu(a.gas, sl.st.T);
    sl.st.k = gas_k(a.gas, sl.st.mu);
    viscous_stress<NDIM>(sl.st);
    for (int N = 0; N < T::NNOD; N++) sl.Psi[N] = 0.0;  // 3D: tau = 0, no upwinding
    if constexpr (NDIM == 2) supg_psi_2d(sh, sl);
  }
}

// rhs flux sums for equation r at one Gauss point (FDVGalerkin.h:549-609, 410-427):
// Fbar(i,r) = sum_b Phi_b FG_b(i,r), divF(r) = sum_b sum_i dPhi_b,i FG_b(i,r)
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void flux_sums(const FormArgs& a, const FormShared<NDIM>& sh, int fc, GpSlot<NDIM>& sl, int r) {
  constexpr int NN = Pass<NDIM, FACE>::NN;
  double Fbar[NDIM], divF = 0.0;
  for (int i = 0; i < NDIM; i++) Fbar[i] = 0.0;
  const bool withF = (NDIM == 2) || a.physical_3d_flux;
  for (int b = 0; b < NN; b++) {
    const NodePrim& nb = pass_node<NDIM, FACE>(sh, fc, b);
    for (int i = 0; i < NDIM; i++) {
      const double fg = node_flux_entry<NDIM>(sl.st, nb, a.gas.creyn, withF, i, r);
      Fbar[i] += sl.Phi[b] * fg;
      divF += sl.dPhi[b][i] * fg;
    }
  }
  for (int i = 0; i < NDIM; i++) sl.F[i][r] = Fbar[i];
  sl.F[NDIM][r] = divF;
}

// step 6: flux Jacobians a, b, c (FDV/NavierStokes2D.h, NavierStokes3D.h) and the rhs flux
// sums; b and c are formed one direction i at a time, and each kind of task fills whole
// warps where the block has them
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void step_jacobians(const FormArgs& a, FormShared<NDIM>& sh, int lf, int tid) {
  using T = FormTraits<NDIM>;
  constexpr int Q = Pass<NDIM, FACE>::NQ, NEQ = T::NEQ;
  constexpr int C0 = 0, CN = Q * NDIM;                     // c: (q, i)
  constexpr int B0 = 32, BN = Q * NDIM;                    // b: (q, i)
  constexpr int A0 = (NDIM == 3) ? 104 : 8;                // a: q
  constexpr int F0 = (NDIM == 3) ? 64 : 40, FN = Q * NEQ;  // flux sums: (q, r)
  static_assert(CN <= B0 && B0 + BN <= F0 && F0 + FN <= T::THREADS && A0 + Q <= T::THREADS &&
                    (NDIM == 2 ? (CN <= A0 && A0 + Q <= B0) : (F0 + FN <= A0)),
                "task ranges overlap");
  if (tid >= C0 && tid < C0 + CN) {
    GpSlot<NDIM>& sl = sh.slot[(tid - C0) / NDIM];
    const int i = (tid - C0) % NDIM;
    jac_c_rows<NDIM>(a.gas, sl.st, i, &sl.H[i * 3][0]);
  } else if (tid >= B0 && tid < B0 + BN) {
    const int q = (tid - B0) / NDIM, i = (tid - B0) % NDIM;
    jac_b_rows<NDIM>(a.gas, sh.slot[q].st, i, &gp_D<NDIM>(sh, q, FACE)[i][0]);
  } else if (tid >= A0 && tid < A0 + Q) {
    jac_a<NDIM>(a.gas, sh.slot[tid - A0].st, &gp_A<NDIM>(sh, tid - A0, FACE)[0][0]);
  } else if (tid >= F0 && tid < F0 + FN) {
    flux_sums<NDIM, FACE>(a, sh, FACE ? sh.faces[lf] : 0, sh.slot[(tid - F0) / NEQ], (tid - F0) % NEQ);
  }
}

// step 7: X = dt (s1 a + s3 b), A = a + b, D = s2 a + s4 b, entry by entry (q, i, r, s)
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void step_coeffs(const FormArgs& a, FormShared<NDIM>& sh, int tid) {
  using T = FormTraits<NDIM>;
  constexpr int NEQ = T::NEQ, PER = NDIM * NEQ * NEQ;
  const double* s = sh.s;
  for (int t = tid; t < Pass<NDIM, FACE>::NQ * PER; t += T::THREADS) {
    const int q = t / PER, rem = t % PER, i = rem / (NEQ * NEQ), r = (rem / NEQ) % NEQ, c = rem % NEQ;
    const int k = r * 5 + c;
    double* A = &gp_A<NDIM>(sh, q, FACE)[i][k];
    double* D = &gp_D<NDIM>(sh, q, FACE)[i][k];
    const double av = *A, bv = *D;
    sh.slot[q].X[i][k] = sh.dt * (s[0] * av + s[2] * bv);
    *A = av + bv;
    *D = s[1] * av + s[3] * bv;
  }
}

// one entry of h (sign = +1, domain) or m (sign = -1, face):
// h_ij(r,s) = -dt s3 c_ij(r,s) + dt^2/2 sum_k A_i(r,k) D_j(k,s)  (FDVGalerkin.h:611-628, 698-715)
template <int NDIM>
CFDV_HD CFDV_INLINE void hmat_entry(const FormArgs& a, FormShared<NDIM>& sh, int it, double sign, bool face) {
  constexpr int NEQ = NDIM + 2;
  constexpr int PER = NDIM * NDIM * NEQ * NEQ;
  const double s3_dt = sh.dt * sh.s[2];
  const int q = it / PER;
  int rem = it % PER;
  const int ij = rem / (NEQ * NEQ);
  rem %= NEQ * NEQ;
  const int r = rem / NEQ, s = rem % NEQ;
  const int i = ij / NDIM, j = ij % NDIM;
  GpSlot<NDIM>& sl = sh.slot[q];
  const double(*A)[25] = gp_A<NDIM>(sh, q, face);
  const double(*D)[25] = gp_D<NDIM>(sh, q, face);
  double t = 0.0;
  for (int k = 0; k < NEQ; k++) t += A[i][r * 5 + k] * D[j][k * 5 + s];
  const double c = sl.H[i * 3 + j][r * 5 + s];
  sl.H[i * 3 + j][r * 5 + s] = sign * (-s3_dt * c + sh.dtsq_2 * t);
}

// step 8: h entries and the rhs coefficient P(i,r) = dt Fbar(i,r) - dt^2/2 sum_s A_i(r,s) divF(s);
// face step 5: m = -h and P with the opposite signs (FDVGalerkin.h:643-680, 698-738)
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void step_hmat_rhs(const FormArgs& a, FormShared<NDIM>& sh, int tid) {
  using T = FormTraits<NDIM>;
  constexpr int NEQ = T::NEQ, NQ = Pass<NDIM, FACE>::NQ;
  constexpr int NH = NQ * NDIM * NDIM * NEQ * NEQ, NP = NQ * NDIM * NEQ;
  for (int t = tid; t < NH + NP; t += T::THREADS) {
    if (t < NH) {
      hmat_entry<NDIM>(a, sh, t, FACE ? -1.0 : 1.0, FACE);
    } else {
      const int p = t - NH, q = p / (NDIM * NEQ), i = (p / NEQ) % NDIM, r = p % NEQ;
      GpSlot<NDIM>& sl = sh.slot[q];
      const double(*A)[25] = gp_A<NDIM>(sh, q, FACE);
      double u = 0.0;
      for (int q2 = 0; q2 < NEQ; q2++) u += A[i][r * 5 + q2] * sl.F[NDIM][q2];
      if (FACE) sl.P[i][r] = -sh.dt * sl.F[i][r] + sh.dtsq_2 * u;
      else sl.P[i][r] = sh.dt * sl.F[i][r] - sh.dtsq_2 * u;
    }
  }
}
// Domain contraction, factored through the row node N:
//   R(N r, M s) = sum_q [ Phi_M G0 + sum_j dPhi_M,j G1j (+ S_M G2 in 2D) ]  with
//   G0  = wJ (Phi_N delta_rs - sum_i dPhi_N,i X_i(r,s)),
//   G1j = wJ sum_i dPhi_N,i h_ij(r,s),   G2 = wJ Psi_N sum_i X_i(r,s),
// which is sum_k B_k(N,M) C_k(r,s) of FDVGalerkin.h:405-451 regrouped (S_M = sum_j dPhi_M,j).
template <int NDIM>
CFDV_HD CFDV_INLINE void phase_contract_domain(FormShared<NDIM>& sh, int tid) {
  using T = FormTraits<NDIM>;
  constexpr int NEQ = T::NEQ, NNOD = T::NNOD, NC = T::NCOEF;
  const int N = tid % NNOD;  // THREADS is a multiple of NNOD: every pair of this thread has row node N
  for (int k = 0; k < T::PAIRS; k++) {
    const int p = tid + k * T::THREADS;
    if (p >= T::NPAIR) break;
    const int rs = p / NNOD, r = rs / NEQ, s = rs % NEQ, idx = r * 5 + s;
    double acc[NNOD];
    for (int M = 0; M < NNOD; M++) acc[M] = 0.0;
    for (int q = 0; q < T::Q; q++) {
      const GpSlot<NDIM>& sl = sh.slot[q];
      const double wJ = sl.wJ;
      double G[NC];
      double x = 0.0;
      for (int i = 0; i < NDIM; i++) x += sl.dPhi[N][i] * sl.X[i][idx];
      G[0] = wJ * (((r == s) ? sl.Phi[N] : 0.0) - x);
      for (int j = 0; j < NDIM; j++) {
        double h = 0.0;
        for (int i = 0; i < NDIM; i++) h += sl.dPhi[N][i] * sl.H[i * 3 + j][idx];
        G[1 + j] = wJ * h;
      }
      if (NDIM == 2) {
        double sx = 0.0;
        for (int i = 0; i < NDIM; i++) sx += sl.X[i][idx];
        G[NC - 1] = wJ * sl.Psi[N] * sx;
      }
      for (int M = 0; M < NNOD; M++) {
        double t = acc[M];
        for (int c = 0; c < NC; c++) t += sl.cM[c][M] * G[c];
        acc[M] = t;
      }
    }
    // the tile aliases A and D, which every thread has finished reading at the last barrier
    for (int M = 0; M < NNOD; M++) sh.Rt[(M * NEQ + s) * T::KE + N * NEQ + r] = acc[M];
  }
  // rhs(N r) = sum_q wJ sum_i dPhi_Ni P_q(i, r)
  if (tid < T::KE) {
    const int Nn = tid / NEQ, r = tid % NEQ;
    double rhs = 0.0;
    for (int q = 0; q < T::Q; q++) {
      const GpSlot<NDIM>& sl = sh.slot[q];
      double t = 0.0;
      for (int i = 0; i < NDIM; i++) t += sl.dPhi[Nn][i] * sl.P[i][r];
      rhs += sl.wJ * t;
    }
    sh.rhs[tid] = rhs;
  }
}

// 3D boundary-state edits (eval2dboundary.h:14-371); tau enters as zero
template <class S>
CFDV_HD CFDV_INLINE void edit_face_state_3d(int code, GpStateT<S>& f, const double* en, int adiabatic) {
  switch (code) {
    case 2:
    case 12:
      for (int i = 0; i < 3; i++) f.dV[i][2] = 0;
      f.dT[2] = 0;
      break;
    case 22:
      for (int i = 0; i < 3; i++) f.dV[i][1] = 0;
      f.dT[1] = 0;
      viscous_stress<3>(f);
      f.tau[0][1] = 0.0; f.tau[1][1] = 0.0; f.tau[2][1] = 0.0; f.tau[1][0] = 0.0; f.tau[1][2] = 0.0;
      break;
    case 1:
    case 51:
      if (adiabatic) f.dT[2] = 0.0;
      viscous_stress<3>(f);
      break;
    case 21:
    case 31:
      if (adiabatic) f.dT[1] = 0.0;
      viscous_stress<3>(f);
      break;
    case 11:
      if (adiabatic) f.dT[0] = 0.0;
      viscous_stress<3>(f);
      break;
    case -1:
      break;
    case 6:
      f.dT[0] = 0.0;
      viscous_stress<3>(f);
      for (int i = 0; i < 3; i++) f.tau[i][0] = 0;
      break;
    case 7:  // falls through into 77/32 in the reference (eval2dboundary.h:113-145)
      f.dT[2] = 0.0;
      f.dT[1] = 0.0;
      viscous_stress<3>(f);
      for (int i = 0; i < 3; i++) { f.tau[i][2] = 0; f.tau[i][1] = 0; }
      break;
    case 77:
    case 32:
      f.dT[1] = 0.0;
      viscous_stress<3>(f);
      for (int i = 0; i < 3; i++) f.tau[i][1] = 0;
      break;
    case 4: {
      f.v[0] = 0; f.v[1] = 0; f.v[2] = 0;
      const double* n = en;  // the weighted normal, not a unit vector
      const S dud = f.dV[0][0] * n[0] + f.dV[0][1] * n[1] + f.dV[0][2] * n[2];
      const S dvd = f.dV[1][0] * n[0] + f.dV[1][1] * n[1] + f.dV[1][2] * n[2];
      const S dtd = f.dT[0] * n[0] + f.dT[1] * n[1] + f.dT[2] * n[2];
      for (int j = 0; j < 3; j++) { f.dV[0][j] -= dud * n[j]; f.dV[1][j] -= dvd * n[j]; f.dT[j] -= dtd * n[j]; }
      S dUd[3];
      for (int i = 0; i < 3; i++) dUd[i] = f.dU[i][0] * n[0] + f.dU[i][1] * n[1] + f.dU[i][2] * n[2];
      for (int i = 0; i < 3; i++)  // only the first three equations (loop bound dU.jmax() = 3)
        for (int j = 0; j < 3; j++) f.dU[i][j] -= dUd[i] * n[j];
    } break;
    case 8:
      viscous_stress<3>(f);
      break;
    case -12:
      f.dV[0][2] = 0.0; f.dV[1][2] = 0.0; f.dV[2][2] = 0.0;
      f.dT[2] = 0.0;
      f.v[2] = 0.0;
      break;
    default:
      break;
  }
}

// 2D boundary-state edits (eval1dboundary.h:9-251); x0, x1: the edge's node coordinates
template <class S>
CFDV_HD CFDV_INLINE void edit_face_state_2d(int code, GpStateT<S>& f, const double* x0, const double* x1,
                                            const double* en) {
  const double len = sqrt(en[0] * en[0] + en[1] * en[1]);
  const double n[2] = {en[0] / len, en[1] / len};
  switch (code) {
    case 2:
    case 12: {
      S d = f.v[0] * n[0] + f.v[1] * n[1];
      f.v[0] -= d * n[0];
      d = f.v[0] * n[0] + f.v[1] * n[1];  // re-evaluated after the first component
      f.v[1] -= d * n[1];
      d = f.dT[0] * n[0] + f.dT[1] * n[1];
      f.dT[0] -= d * n[0];
      d = f.dT[0] * n[0] + f.dT[1] * n[1];
      f.dT[1] -= d * n[1];
    } break;
    case 1:
    case 51: {
      S d = f.dT[0] * n[0] + f.dT[1] * n[1];
      f.dT[0] -= d * n[0];
      d = f.dT[0] * n[0] + f.dT[1] * n[1];
      f.dT[1] -= d * n[1];
    } break;
    case -1:
      f.dV[0][0] = 0.0; f.dV[1][0] = 0.0; f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[0] = 0.0;
      break;
    case 6:
      f.dV[0][0] = 0.0; f.dV[1][0] = 0.0; f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[0] = 0.0;
      for (int i = 0; i < 4; i++) f.dU[i][0] = 0.0;
      break;
    case -2:
    case 7:
      f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[1] = 0.0;
      for (int i = 0; i < 4; i++) f.dU[i][1] = 0.0;
      break;
    case 4:
    case 8: {
      double nn[2];
      if (code == 4) {
        f.v[0] = 0; f.v[1] = 0;
        nn[0] = en[0]; nn[1] = en[1];
      } else {  // fixed 10 degree ramp direction scaled by the edge height
        const double alpha = 10 * (3.14159 / 180.0);
        const double dl = fabs(x1[1] - x0[1]);
        nn[0] = cos(alpha) * dl;
        nn[1] = sin(alpha) * dl;
      }
      const S dud = f.dV[0][0] * nn[0] + f.dV[0][1] * nn[1];
      const S dvd = f.dV[1][0] * nn[0] + f.dV[1][1] * nn[1];
      const S dtd = f.dT[0] * nn[0] + f.dT[1] * nn[1];
      f.dV[0][0] -= dud * nn[0]; f.dV[0][1] -= dud * nn[1];
      f.dV[1][0] -= dvd * nn[0]; f.dV[1][1] -= dvd * nn[1];
      f.dT[0] -= dtd * nn[0]; f.dT[1] -= dtd * nn[1];
      S dUd[4];
      for (int i = 0; i < 4; i++) dUd[i] = f.dU[i][0] * nn[0] + f.dU[i][1] * nn[1];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 2; j++) f.dU[i][j] -= dUd[i] * nn[j];
    } break;
    case -12:
      f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[1] = 0.0;
      f.v[1] = 0.0;
      for (int i = 0; i < 4; i++) f.dU[i][1] = 0.0;
      break;
    case 11:
    case 21:
      f.v[0] = 0; f.v[1] = 0;
      f.dV[0][0] = 0.0; f.dV[1][0] = 0.0;
      f.dT[1] = 0.0;
      for (int i = 0; i < 4; i++) f.dU[i][1] = 0.0;
      break;
    default:
      break;
  }
  viscous_stress<2>(f);
  if (code == 2 || code == 12 || code == 7) { f.tau[0][1] = 0.0; f.tau[1][0] = 0.0; }
  if (code == 6) { f.tau[0][0] = 0.; f.tau[1][0] = 0.; }
}

// Face shape functions phib, derivatives along the face dpidx and the weighted normal en
// at face Gauss point qf (2D TestFunctions1D.h:7-82, 3D calc_TF_norm3D.h:9-167); xf
// holds the coordinates of the face's NBN nodes in face order.
template <int NDIM>
CFDV_HD CFDV_INLINE void face_point_geom(const double* gz, const double* gw, const double* const* xf, int qf,
                                         double* phib, double (*dpidx)[3], double* en) {
  constexpr int NBN = FormTraits<NDIM>::NBN;
  for (int i = 0; i < NBN; i++)
    for (int j = 0; j < 3; j++) dpidx[i][j] = 0.0;
  en[2] = 0.0;
  if (NDIM == 2) {  // TestFunctions1D.h:7-82
    const double z = gz[qf], w = gw[qf];
    phib[0] = 0.5 * (1 - z);
    phib[1] = 0.5 * (1 + z);
    const double dxds = -0.5 * xf[0][0] + 0.5 * xf[1][0];
    const double dyds = -0.5 * xf[0][1] + 0.5 * xf[1][1];
    en[0] = dyds * w;
    en[1] = -dxds * w;
    const double delx = xf[1][0] - xf[0][0], dely = xf[1][1] - xf[0][1];
    if (!(fabs(delx) < 1.0E-12)) { dpidx[0][0] = -1.0 / delx; dpidx[1][0] = 1.0 / delx; }
    if (!(fabs(dely) < 1.0E-12)) { dpidx[0][1] = -1.0 / dely; dpidx[1][1] = 1.0 / dely; }
  } else {  // calc_TF_norm3D.h:9-167
    const double z[2] = {gz[qf >> 1], gz[qf & 1]};
    const double w0 = gw[qf >> 1], w1 = gw[qf & 1];
    double ph[4], dpxi[4][3];
    shape_fn<2>(z, ph, dpxi);
    for (int i = 0; i < 4; i++) phib[i] = ph[i];
    double L[3], Mu[3];
    for (int i = 0; i < 3; i++) { L[i] = xf[1][i] - xf[0][i]; Mu[i] = xf[3][i] - xf[0][i]; }
    for (int j = 0; j < 3; j++) {  // magnitude re-evaluated after each component
      L[j] /= sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
      Mu[j] /= sqrt(Mu[0] * Mu[0] + Mu[1] * Mu[1] + Mu[2] * Mu[2]);
    }
    double nrm[3], gm[3];
    nrm[0] = L[1] * Mu[2] - L[2] * Mu[1];
    nrm[1] = L[2] * Mu[0] - L[0] * Mu[2];
    nrm[2] = L[0] * Mu[1] - L[1] * Mu[0];
    gm[0] = nrm[1] * L[2] - nrm[2] * L[1];
    gm[1] = nrm[2] * L[0] - nrm[0] * L[2];
    gm[2] = nrm[0] * L[1] - nrm[1] * L[0];
    double dxd[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int N = 0; N < 4; N++)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 2; j++) dxd[i][j] += dpxi[N][j] * xf[N][i];
    double tr[2][2];
    for (int j = 0; j < 2; j++) {
      tr[0][j] = L[0] * dxd[0][j] + L[1] * dxd[1][j] + L[2] * dxd[2][j];
      tr[1][j] = gm[0] * dxd[0][j] + gm[1] * dxd[1][j] + gm[2] * dxd[2][j];
    }
    const double det = tr[0][0] * tr[1][1] - tr[1][0] * tr[0][1];
    const double idet = 1. / det;
    for (int N = 0; N < 4; N++) {
      const double p0 = (tr[1][1] * dpxi[N][0] - tr[1][0] * dpxi[N][1]) * idet;
      const double p1 = (-tr[0][1] * dpxi[N][0] + tr[0][0] * dpxi[N][1]) * idet;
      for (int i = 0; i < 3; i++) dpidx[N][i] = L[i] * p0 + gm[i] * p1;
    }
    for (int i = 0; i < 3; i++) en[i] = nrm[i] * w0 * w1 * det;
  }
}

// face step 0: the face geometry of Gauss point qf (one thread per face Gauss point) and
// the face-local coefficient rows of the contraction
template <int NDIM>
CFDV_HD CFDV_INLINE void step_face_geom(const FormArgs& a, FormShared<NDIM>& sh, int lf, int qf) {
  using T = FormTraits<NDIM>;
  constexpr int NBN = T::NBN;
  if (qf >= T::QF) return;
  GpSlot<NDIM>& sl = sh.slot[qf];
  const int f = sh.faces[lf];
  const double* xf[NBN];
  for (int i = 0; i < NBN; i++) xf[i] = sh.nd[face_node(NDIM, f, i)].x;
  double xl[4][3];
  const double* H = (NDIM == 3 && sh.hnm >= 0) ? a.hnm + (size_t)sh.hnm * 64 : nullptr;
  if (H) {
    const double* xe[8];
    for (int M = 0; M < 8; M++) xe[M] = sh.nd[M % T::NNOD].x;
    hnm_face_nodes_3d(H, xe, f, xl);
    for (int i = 0; i < NBN; i++) xf[i] = xl[i % 4];
  }
  face_point_geom<NDIM>(a.gz, a.gw, xf, qf, sl.Phi, sl.dPhi, sl.en);
  if constexpr (NDIM == 3)
    if (H) hnm_face_phi_3d(H, f, sl.Phi);
  for (int m = 0; m < NBN; m++) {
    sl.cM[0][m] = sl.Phi[m];
    for (int j = 0; j < NDIM; j++) sl.cM[1 + j][m] = sl.dPhi[m][j];
  }
}

// face step 2: viscosity and conductivity at the face point, stress zero, then the
// boundary-condition edits of the state (eval1dboundary.h, eval2dboundary.h)
template <int NDIM>
CFDV_HD CFDV_INLINE void step_face_edit(const FormArgs& a, FormShared<NDIM>& sh, int lf, int qf) {
  using T = FormTraits<NDIM>;
  if (qf >= T::QF) return;
  GpSlot<NDIM>& sl = sh.slot[qf];
  GpState& fs = sl.st;
  const int f = sh.faces[lf], code = sh.codes[lf];
  fs.mu = gas_mu(a.gas, fs.T);
  fs.k = gas_k(a.gas, fs.mu);
  for (int i = 0; i < NDIM; i++)
    for (int j = 0; j < NDIM; j++) fs.tau[i][j] = 0;
  if (NDIM == 2) edit_face_state_2d(code, fs, sh.nd[face_node(NDIM, f, 0)].x, sh.nd[face_node(NDIM, f, 1)].x, sl.en);
  else edit_face_state_3d(code, fs, sl.en, a.gas.adiabatic);
}

template <int NDIM>
CFDV_HD CFDV_INLINE int face_pos(int f, int node) {
  for (int i = 0; i < FormTraits<NDIM>::NBN; i++)
    if (face_node(NDIM, f, i) == node) return i;
  return -1;
}

// Face contraction, factored the same way over the face's nodes (local numbering m):
//   R(N r, M s) += sum_qf Phi_N [ Phi_M sum_i en_i X_i(r,s) + sum_j dPhi_M,j sum_i en_i m_ij(r,s) ]
// (FDVGalerkin.h:455-533, 643-756)
template <int NDIM>
CFDV_HD CFDV_INLINE void phase_contract_face(FormShared<NDIM>& sh, int lf, int tid) {
  using T = FormTraits<NDIM>;
  constexpr int NEQ = T::NEQ, NNOD = T::NNOD;
  const int f = sh.faces[lf];
  const int N = tid % NNOD;
  const int fN = face_pos<NDIM>(f, N);
  if (fN >= 0) {
    int fM[NNOD];
    for (int M = 0; M < NNOD; M++) fM[M] = face_pos<NDIM>(f, M);
    for (int q = 0; q < T::QF; q++) {
      const GpSlot<NDIM>& sl = sh.slot[q];
      const double PhiN = sl.Phi[fN];
      for (int k = 0; k < T::PAIRS; k++) {
        const int p = tid + k * T::THREADS;
        if (p < T::NPAIR) {
          const int rs = p / NNOD, idx = (rs / NEQ) * 5 + rs % NEQ;
          double G[1 + NDIM];
          double x = 0.0;
          for (int i = 0; i < NDIM; i++) x += sl.en[i] * sl.X[i][idx];
          G[0] = PhiN * x;
          for (int j = 0; j < NDIM; j++) {
            double h = 0.0;
            for (int i = 0; i < NDIM; i++) h += sl.en[i] * sl.H[i * 3 + j][idx];
            G[1 + j] = PhiN * h;
          }
          const int r = rs / NEQ, s = rs % NEQ;
          for (int M = 0; M < NNOD; M++) {
            if (fM[M] >= 0) {  // each (pair, M) entry of the tile belongs to this thread alone
              double& t = sh.Rt[(M * NEQ + s) * T::KE + N * NEQ + r];
              double v = t;
              for (int c = 0; c <= NDIM; c++) v += sl.cM[c][fM[M]] * G[c];
              t = v;
            }
          }
        }
      }
    }
  }
  if (tid < T::KE) {
    const int Nn = tid / NEQ, r = tid % NEQ;
    const int fp = face_pos<NDIM>(f, Nn);
    if (fp >= 0) {
      double rhs = sh.rhs[tid];
      for (int q = 0; q < T::QF; q++) {
        const GpSlot<NDIM>& sl = sh.slot[q];
        double t = 0.0;
        for (int i = 0; i < NDIM; i++) t += sl.en[i] * sl.P[i][r];
        rhs += sl.Phi[fp] * t;
      }
      sh.rhs[tid] = rhs;
    }
  }
}

// ApplyBC (rows of Dirichlet DOFs: zero, diagonal 0.5, rhs 0) and the coalesced store
template <int NDIM>
CFDV_HD CFDV_INLINE void phase_write(const FormArgs& a, FormShared<NDIM>& sh, int e, int tid, int* bad) {
  using T = FormTraits<NDIM>;
  constexpr int KE = T::KE;
  const uint64_t mk = sh.mask;
  const size_t base = (size_t)e * KE * KE;
  for (int k = tid; k < KE * KE; k += T::THREADS) {
    const int I = k % KE, J = k / KE;
    double v = sh.Rt[k];
    if ((mk >> I) & 1ull) v = (I == J) ? 0.5 : 0.0;
    if (!(v == v) || v - v != 0.0) *bad = 1;
    if (a.R64) a.R64[base + k] = v;
    if (a.R32) a.R32[base + k] = (float)v;
  }
  if (tid < KE) {
    double v = ((mk >> tid) & 1ull) ? 0.0 : sh.rhs[tid];
    if (!(v == v) || v - v != 0.0) *bad = 1;
    a.rhs[(size_t)e * KE + tid] = v;
  }
  if (tid == 0 && a.s_out)
    for (int i = 0; i < 4; i++) a.s_out[(size_t)e * 4 + i] = sh.s[i];
}

// ---- the element as a sequence of block-wide steps --------------------------------
// Steps 0-9 form the domain integrals (step 9 leaves the element matrix in the shared
// tile), then seven steps per boundary face (geometry, state sums, boundary edits,
// Jacobians and flux sums, coefficients, m and rhs, contraction into the tile), then
// ApplyBC and the store.  Every step is followed by a block barrier; the CPU emulation
// runs the same steps thread by thread.
constexpr int kDomainSteps = 10;
constexpr int kFaceSteps = 7;

template <int NDIM>
CFDV_HD CFDV_INLINE int form_nsteps(const FormShared<NDIM>& sh) {
  return kDomainSteps + kFaceSteps * sh.nfaces + 1;
}

template <int NDIM>
CFDV_HD CFDV_INLINE void form_step(int k, const FormArgs& a, FormShared<NDIM>& sh, int e, int tid, int* bad) {
  switch (k) {
    case 0: step_load<NDIM>(a, sh, e, tid); return;
    case 1: step_geom_jac<NDIM>(a, sh, tid); return;
    case 2: step_geom_det<NDIM>(a, sh, tid); return;
    case 3: step_dphi<NDIM>(sh, tid); return;
    case 4: step_state<NDIM, false>(sh, 0, tid); return;
    case 5: step_stress<NDIM>(a, sh, tid); return;
    case 6: step_jacobians<NDIM, false>(a, sh, 0, tid); return;
    case 7: step_coeffs<NDIM, false>(a, sh, tid); return;
    case 8: step_hmat_rhs<NDIM, false>(a, sh, tid); return;
    case 9: phase_contract_domain<NDIM>(sh, tid); return;
    default: break;
  }
  const int f = k - kDomainSteps, nf = sh.nfaces;
  if (f < kFaceSteps * nf) {
    const int lf = f / kFaceSteps;
    switch (f % kFaceSteps) {
      case 0: step_face_geom<NDIM>(a, sh, lf, tid); return;
      case 1: step_state<NDIM, true>(sh, lf, tid); return;
      case 2: step_face_edit<NDIM>(a, sh, lf, tid); return;
      case 3: step_jacobians<NDIM, true>(a, sh, lf, tid); return;
      case 4: step_coeffs<NDIM, true>(a, sh, tid); return;
      case 5: step_hmat_rhs<NDIM, true>(a, sh, tid); return;
      default: phase_contract_face<NDIM>(sh, lf, tid); return;
    }
  }
  phase_write<NDIM>(a, sh, e, tid, bad);
}

}  // namespace cfdv
