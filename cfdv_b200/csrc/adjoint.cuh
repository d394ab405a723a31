// Element functionals of the discrete adjoint and tangent of the FDV step (kernels and
// host driver in adjoint.cu).  Host/device code, so that a CPU build can check it
// against the oracle.
//
// One step of the textbook path is  dt = CFL(U),  A(U, dt) dU = b(U, dt),  U' = U + dU,
// with A, b the assembled element matrices and rhs after ApplyBC (FDVGalerkin.h:121-154,
// ApplyBC.h:14-133).  With dU held fixed, the element residual r_e = rhs_e - R_e dU_e
// carries every dependence of the step on U, dt and the Mach number; its derivatives are
// evaluated here by forward-mode dual numbers through the same templated physics the
// formation kernel runs (fdv_physics.cuh, formation.cuh), so they are the derivatives of
// the same floating-point program.
//
// Element functional.  For weights w (one per element row) the kernels evaluate
//   L_e = sum over unmasked rows (N r) of w(N r) [rhs_e - R_e dU_e](N r)
// without forming R_e: with the factorisation of the formation kernel,
//   R(N r, M s) = sum_q [Phi_M G0 + sum_j dPhi_M,j G1j + S_M G2] (+ face terms),
// L_e collapses per Gauss point to a few neqn-vectors (m1_i = sum_N dPhi_N,i w_N,
// u0 = sum_M Phi_M dU_M, u1_j = sum_M dPhi_M,j dU_M, ...) contracted with the flux
// Jacobians a_i, b_i, c_ij entry by entry.  A thread evaluates L_e for one element and
// one seed direction (the GPU runs the JVP this way; the VJP runs as the reverse sweep of
// adjoint_warp.cuh, which the CPU build checks against these VJP seeds):
//   VJP  (adjoint):  w = mu_e (the adjoint solution), seed = one of the element's Ke
//                    unknowns, dt, or the Mach number -> one gradient entry per thread;
//   JVP  (tangent):  w = a unit row, seed = the tangent (dU, ddt, dMach) -> one entry of
//                    the residual's directional derivative per thread.
// ApplyBC rows (the Dirichlet row mask) are constant (0.5 on the diagonal, rhs 0): their
// weights are zero.
//
// Objective: the wall x-force F_x = sum over faces with the wall code of the integral of
// p n_x - (1/Re) tau_xj n_j (n outward from the fluid, i.e. into the body), with p and T
// interpolated from the nodes and tau from the element's velocity gradient at the face
// Gauss points.  The reference integrates no force; this functional is defined here.
#pragma once
#include "dual.cuh"
#include "formation.cuh"
#include "jac_adjoint.cuh"

namespace cfdv {

struct FunctionalArgs {
  GasParams gas;
  double dt;
  double gz[2], gw[2];
  int n_elements, physical_3d_flux;
  int mode;                 // 0: VJP seeds (Ke unknowns, dt, Mach; forward mode, the CPU build's check of
                            // the reverse sweep), 1: JVP (the GPU's functional_kernel)
  const double* U;          // [Nn][neqn]
  const double* x;          // [Nn][ndim]
  const int* conn;          // [E][nnod]
  const int* bc;            // [E][nface]
  const uint64_t* rowmask;  // [E]
  const int* hnm_idx;       // [E] adaptive elements (as in FormArgs), or null
  const double* hnm;
  const double* dU;         // the step's solution [Nn][neqn]
  const double* w;          // VJP: adjoint weights [Nn][neqn]
  const double* tU;         // JVP: tangent of U [Nn][neqn]
  double t_dt, t_mach;      // JVP: tangents of dt and of the Mach number
  double* out;              // VJP: [E][Ke] d L_e / d U_e ; JVP: [E][Ke] d r_e
  double* out_dt;           // VJP: [E] d L_e / d dt
  double* out_mach;         // VJP: [E] d L_e / d Mach
  double* out_val;          // VJP: [E] L_e (value, for checks) or null
};

struct ForceArgs {
  GasParams gas;
  double gz[2], gw[2];
  int n_list, wall_bc;
  const int* elems;         // [n_list] elements with a wall face
  const double* U;
  const double* x;
  const int* conn;
  const int* bc;
  const int* hnm_idx;       // [E] adaptive elements (as in FormArgs), or null
  const double* hnm;
  double* out;              // [n_list][Ke] d F / d U_e
  double* out_mach;         // [n_list] d F / d Mach
  double* out_val;          // [n_list] F of the element's wall faces
};

// Mach-number derivative of the gas constants: Cv = 1/(gamma (gamma-1) M^2), cgas = 1/(gamma M^2)
CFDV_HD CFDV_INLINE GasT<Dual> dual_gas(const GasParams& g, double dM) {
  GasT<Dual> d;
  d.gamma = g.gamma; d.gamm1 = g.gamm1; d.gm1d2 = g.gm1d2; d.gamm3 = g.gamm3; d.gm3d2 = g.gm3d2;
  d.Pr = g.Pr; d.csuth = g.csuth; d.creyn = g.creyn; d.Twall = g.Twall; d.adiabatic = g.adiabatic;
  d.Cv = Dual(g.Cv, -2.0 * g.Cv / g.cmach * dM);
  d.cgas = Dual(g.cgas, -2.0 * g.cgas / g.cmach * dM);
  d.cmach = Dual(g.cmach, dM);
  return d;
}

// Gauss-point state sums (FDVGalerkin.h:761-797) over the NN nodes of a pass, in the order
// of the formation kernel's state_sum: acc += coef_N * field_N, N ascending
template <int NDIM, int NN, class S>
CFDV_HD CFDV_INLINE void gp_state_sums(const NodePrimT<S>* const* nd, const double* Phi, const double (*dPhi)[3],
                                       GpStateT<S>& f) {
  constexpr int NEQ = NDIM + 2;
  f.E = 0.0;
  f.T = 0.0;
  for (int N = 0; N < NN; N++) {
    f.E = RN_ADD(f.E, RN_MUL(Phi[N], nd[N]->E));
    f.T = RN_ADD(f.T, RN_MUL(Phi[N], nd[N]->T));
  }
  for (int q = 0; q < NEQ; q++) {
    S u = 0.0;
    for (int N = 0; N < NN; N++) u = RN_ADD(u, RN_MUL(Phi[N], nd[N]->U[q]));
    f.U[q] = u;
    for (int c = 0; c < NDIM; c++) {
      S d = 0.0;
      for (int N = 0; N < NN; N++) d = RN_ADD(d, RN_MUL(dPhi[N][c], nd[N]->U[q]));
      f.dU[q][c] = d;
    }
  }
  for (int i = 0; i < NDIM; i++) {
    S v = 0.0;
    for (int N = 0; N < NN; N++) v = RN_ADD(v, RN_MUL(Phi[N], nd[N]->v[i]));
    f.v[i] = v;
  }
  for (int c = 0; c < NDIM; c++) {
    S t = 0.0;
    for (int N = 0; N < NN; N++) t = RN_ADD(t, RN_MUL(dPhi[N][c], nd[N]->T));
    f.dT[c] = t;
  }
  for (int i = 0; i < NDIM; i++)
    for (int c = 0; c < NDIM; c++) {
      S t = 0.0;
      for (int N = 0; N < NN; N++) t = RN_ADD(t, RN_MUL(dPhi[N][c], nd[N]->v[i]));
      f.dV[i][c] = t;
    }
}

// Weighted contraction of one Gauss point of a pass (domain: sgn = +1, face: sgn = -1):
//   sgn (dt Fterm - dt^2/2 abar.divF) - mterm + sgn dt (s1 Sa + s3 Sb)
//   - sgn (-dt s3 Gam + dt^2/2 abar.beta) - psi
// with wi(r) the row weights of direction i, u0 / u1 the interpolated dU and its
// gradient, abar = sum_i wi^T (a_i + b_i), beta = sum_j (s2 a_j + s4 b_j) u1_j,
// Sa = sum_i wi^T a_i u0, Sb = sum_i wi^T b_i u0, Gam = sum_ij wi^T c_ij u1_j,
// Fterm = sum_b Phi_b sum_i wi . FG_b(i), divF = sum_b sum_i dPhi_b,i FG_b(i), and in the
// 2D domain psi = dt mPsi . (s1 sum_i a_i uS + s3 sum_i b_i uS) (FDVGalerkin.h:405-451,
// 536-641, 643-756 regrouped; h_ij and m_ij = -h_ij, FDVGalerkin.h:611-628, 698-715).
template <int NDIM, int NN>
CFDV_HD CFDV_INLINE Dual pass_terms(const GasT<Dual>& g, const GpStateT<Dual>& f, const NodePrimT<Dual>* const* nd,
                                    const double* Phi, const double (*dPhi)[3], const Dual& dt, const Dual& dtsq_2,
                                    const Dual* s, const double (*wi)[5], const double* u0, const double (*u1)[5],
                                    const double* uS, const Dual* mPsi, bool with_psi, bool withF, double sgn,
                                    double mterm) {
  constexpr int NEQ = NDIM + 2;
  Dual abar[5], va1[5], vb1[5], vaS[5], vbS[5];
  Dual Sa = 0.0, Sb = 0.0, Gam = 0.0;
  Dual J[NDIM * 25];
  jac_a<NDIM>(g, f, J);
  // a: abar, va1, Sa, vaS
  for (int i = 0; i < NDIM; i++)
    for (int r = 0; r < NEQ; r++)
      for (int c = 0; c < NEQ; c++) {
        const Dual& av = J[i * 25 + r * 5 + c];
        abar[c] += wi[i][r] * av;
        va1[r] += av * u1[i][c];
        Sa += wi[i][r] * (av * u0[c]);
        if (with_psi) vaS[r] += av * uS[c];
      }
  // b, one direction at a time into the same buffer
  for (int i = 0; i < NDIM; i++) {
    jac_b_rows<NDIM>(g, f, i, J);
    for (int r = 0; r < NEQ; r++)
      for (int c = 0; c < NEQ; c++) {
        const Dual& bv = J[r * 5 + c];
        abar[c] += wi[i][r] * bv;
        vb1[r] += bv * u1[i][c];
        Sb += wi[i][r] * (bv * u0[c]);
        if (with_psi) vbS[r] += bv * uS[c];
      }
  }
  // c: the bilinear form, one direction i at a time
  {
    Dual C[75];
    for (int i = 0; i < NDIM; i++) {
      jac_c_rows<NDIM>(g, f, i, C);
      for (int j = 0; j < NDIM; j++)
        for (int r = 0; r < NEQ; r++) {
          Dual t = 0.0;
          for (int c = 0; c < NEQ; c++) t += C[j * 25 + r * 5 + c] * u1[j][c];
          Gam += wi[i][r] * t;
        }
    }
  }
  // fluxes of the pass nodes
  Dual Fterm = 0.0, divF[5];
  for (int b = 0; b < NN; b++)
    for (int i = 0; i < NDIM; i++)
      for (int r = 0; r < NEQ; r++) {
        const Dual fg = node_flux_entry<NDIM>(f, *nd[b], g.creyn, withF, i, r);
        Fterm += (Phi[b] * wi[i][r]) * fg;
        divF[r] += dPhi[b][i] * fg;
      }
  Dual ad = 0.0, ab = 0.0;
  for (int r = 0; r < NEQ; r++) {
    ad += abar[r] * divF[r];
    ab += abar[r] * (s[1] * va1[r] + s[3] * vb1[r]);
  }
  Dual t = sgn * (dt * Fterm - dtsq_2 * ad) - mterm + sgn * dt * (s[0] * Sa + s[2] * Sb) -
           sgn * (-(dt * s[2]) * Gam + dtsq_2 * ab);
  if (with_psi) {
    Dual p = 0.0;
    for (int r = 0; r < NEQ; r++) p += mPsi[r] * (s[0] * vaS[r] + s[2] * vbS[r]);
    t -= dt * p;
  }
  return t;
}

// L_e for element e and thread slot k (VJP: seed direction k of Ke + 2; JVP: row k)
template <int NDIM>
CFDV_HD Dual element_functional(const FunctionalArgs& a, int e, int k) {
  using T = FormTraits<NDIM>;
  constexpr int NNOD = T::NNOD, NEQ = T::NEQ, KE = T::KE, NFACE = T::NFACE, NBN = T::NBN;
  const double* Hn = (a.hnm_idx && a.hnm_idx[e] >= 0) ? a.hnm + (size_t)a.hnm_idx[e] * NNOD * NNOD : nullptr;
  const bool vjp = a.mode != 1;
  const uint64_t mask = a.rowmask ? a.rowmask[e] : 0ull;
  if (!vjp && ((mask >> k) & 1ull)) return Dual(0.0);
  double dM = 0.0, ddt = 0.0;
  if (vjp) {
    if (k == KE) ddt = 1.0;
    else if (k == KE + 1) dM = 1.0;
  } else {
    ddt = a.t_dt;
    dM = a.t_mach;
  }
  const GasT<Dual> g = dual_gas(a.gas, dM);
  const Dual dt(a.dt, ddt);
  const Dual dtsq_2 = dt * dt / 2.0;
  NodePrimT<Dual> nd[NNOD];
  double wgt[KE], du[KE];
  Dual Mn[NNOD], Ren[NNOD], s[4];
  for (int N = 0; N < NNOD; N++) {
    const int n = a.conn[(size_t)e * NNOD + N];
    Dual u[NEQ];
    for (int c = 0; c < NEQ; c++) {
      const size_t gi = (size_t)n * NEQ + c;
      const double seed = vjp ? ((k == N * NEQ + c) ? 1.0 : 0.0) : a.tU[gi];
      u[c] = Dual(a.U[gi], seed);
      const int row = N * NEQ + c;
      wgt[row] = vjp ? (((mask >> row) & 1ull) ? 0.0 : a.w[gi]) : (row == k ? 1.0 : 0.0);
      du[row] = a.dU[gi];
    }
    node_unpack<NDIM>(g, u, a.x + (size_t)n * NDIM, nd[N]);
    node_mach_re<NDIM>(g, nd[N], &Mn[N], &Ren[N]);
  }
  fdv_pair<NNOD>(Mn, 0, s);
  fdv_pair<NNOD>(Ren, 1, s);
  const bool withF = (NDIM == 2) || a.physical_3d_flux;
  const NodePrimT<Dual>* all[NNOD];
  for (int N = 0; N < NNOD; N++) all[N] = &nd[N];
  Dual L = 0.0;
  // ---- domain Gauss points ----
  for (int q = 0; q < T::Q; q++) {
    double z[3], Phi[NNOD], dPxi[NNOD][3], dPhi[NNOD][3], jac[3][3];
    double w = 1.0;
    for (int d = 0; d < NDIM; d++) {
      const int bit = (q >> (NDIM - 1 - d)) & 1;
      z[d] = a.gz[bit];
      w *= a.gw[bit];
    }
    shape_fn<NDIM>(z, Phi, dPxi);
    if (Hn) hnm_shape<NDIM>(Hn, Phi, dPxi);
    const double J = phys_deriv<NDIM>(dPxi, nd, dPhi, jac);
    const double wJ = w * J;
    GpStateT<Dual> f;
    gp_state_sums<NDIM, NNOD>(all, Phi, dPhi, f);
    f.mu = gas_mu(g, f.T);
    f.k = gas_k(g, f.mu);
    viscous_stress<NDIM>(f);
    Dual Psi[NNOD];
    if constexpr (NDIM == 2) {
      const double* x4[4] = {nd[0].x, nd[1].x, nd[2].x, nd[3].x};
      double pj[3][3];  // the upwind term's Jacobian: of the untransformed shape functions
      if (Hn) plain_jac_2d(z, x4, pj);
      psi_2d<Dual>(Hn ? pj : jac, x4, f, dPhi, Psi);
    }
    double wi[3][5], u0[5], u1[3][5], uS[5], m0[5];
    Dual mPsi[5];
    for (int r = 0; r < NEQ; r++) {
      double a0 = 0.0, b0 = 0.0, bs = 0.0;
      Dual ps = 0.0;
      double a1[3] = {0, 0, 0}, b1[3] = {0, 0, 0};
      for (int N = 0; N < NNOD; N++) {
        const double wv = wgt[N * NEQ + r], dv = du[N * NEQ + r];
        double sd = 0.0;
        for (int j = 0; j < NDIM; j++) sd += dPhi[N][j];
        a0 += Phi[N] * wv;
        b0 += Phi[N] * dv;
        bs += sd * dv;
        if (NDIM == 2) ps += Psi[N] * wv;
        for (int i = 0; i < NDIM; i++) {
          a1[i] += dPhi[N][i] * wv;
          b1[i] += dPhi[N][i] * dv;
        }
      }
      m0[r] = a0;
      u0[r] = b0;
      uS[r] = bs;
      mPsi[r] = ps;
      for (int i = 0; i < NDIM; i++) {
        wi[i][r] = a1[i];
        u1[i][r] = b1[i];
      }
    }
    double mterm = 0.0;
    for (int r = 0; r < NEQ; r++) mterm += m0[r] * u0[r];
    L += wJ * pass_terms<NDIM, NNOD>(g, f, all, Phi, dPhi, dt, dtsq_2, s, wi, u0, u1, uS, mPsi, NDIM == 2, withF,
                                     1.0, mterm);
  }
  // ---- boundary faces with 0 != bc < 100 (FDVGalerkin.h:455-533) ----
  for (int fc = 0; fc < NFACE; fc++) {
    const int code = a.bc[(size_t)e * NFACE + fc];
    if (code == 0 || code >= 100) continue;
    const NodePrimT<Dual>* fn[NBN];
    const double* xf[NBN];
    int ln[NBN];
    for (int i = 0; i < NBN; i++) {
      ln[i] = face_node(NDIM, fc, i);
      fn[i] = &nd[ln[i]];
      xf[i] = nd[ln[i]].x;
    }
    double xl[4][3];
    if (NDIM == 3 && Hn) {  // adaptive element: face geometry from Hnm x
      const double* xe[8];
      for (int M = 0; M < 8; M++) xe[M] = nd[M % NNOD].x;
      hnm_face_nodes_3d(Hn, xe, fc, xl);
      for (int i = 0; i < NBN; i++) xf[i] = xl[i % 4];
    }
    for (int qf = 0; qf < T::QF; qf++) {
      double phib[NBN], dpidx[NBN][3], en[3];
      face_point_geom<NDIM>(a.gz, a.gw, xf, qf, phib, dpidx, en);
      if constexpr (NDIM == 3)
        if (Hn) hnm_face_phi_3d(Hn, fc, phib);
      GpStateT<Dual> f;
      gp_state_sums<NDIM, NBN>(fn, phib, dpidx, f);
      f.mu = gas_mu(g, f.T);
      f.k = gas_k(g, f.mu);
      for (int i = 0; i < NDIM; i++)
        for (int j = 0; j < NDIM; j++) f.tau[i][j] = 0.0;
      if constexpr (NDIM == 2) edit_face_state_2d(code, f, xf[0], xf[1], en);
      else edit_face_state_3d(code, f, en, a.gas.adiabatic);
      double wi[3][5], u0[5], u1[3][5];
      for (int r = 0; r < NEQ; r++) {
        double m0 = 0.0, b0 = 0.0, b1[3] = {0, 0, 0};
        for (int m = 0; m < NBN; m++) {
          const double wv = wgt[ln[m] * NEQ + r], dv = du[ln[m] * NEQ + r];
          m0 += phib[m] * wv;
          b0 += phib[m] * dv;
          for (int j = 0; j < NDIM; j++) b1[j] += dpidx[m][j] * dv;
        }
        u0[r] = b0;
        for (int i = 0; i < NDIM; i++) {
          wi[i][r] = en[i] * m0;
          u1[i][r] = b1[i];
        }
      }
      L += pass_terms<NDIM, NBN>(g, f, fn, phib, dpidx, dt, dtsq_2, s, wi, u0, u1, nullptr, nullptr, false, withF,
                                 -1.0, 0.0);
    }
  }
  return L;
}

// Wall x-force of element e's faces with the wall code, seeded along direction k (k < Ke:
// the element's unknown k; k == Ke: the Mach number)
template <int NDIM>
CFDV_HD Dual wall_force_element(const ForceArgs& a, int e, int k) {
  using T = FormTraits<NDIM>;
  constexpr int NNOD = T::NNOD, NEQ = T::NEQ, KE = T::KE, NFACE = T::NFACE;
  const double* Hn = (a.hnm_idx && a.hnm_idx[e] >= 0) ? a.hnm + (size_t)a.hnm_idx[e] * NNOD * NNOD : nullptr;
  const GasT<Dual> g = dual_gas(a.gas, k == KE ? 1.0 : 0.0);
  NodePrimT<Dual> nd[NNOD];
  for (int N = 0; N < NNOD; N++) {
    const int n = a.conn[(size_t)e * NNOD + N];
    Dual u[NEQ];
    for (int c = 0; c < NEQ; c++) u[c] = Dual(a.U[(size_t)n * NEQ + c], (k == N * NEQ + c) ? 1.0 : 0.0);
    node_unpack<NDIM>(g, u, a.x + (size_t)n * NDIM, nd[N]);
  }
  Dual F = 0.0;
  for (int fc = 0; fc < NFACE; fc++) {
    if (a.bc[(size_t)e * NFACE + fc] != a.wall_bc) continue;
    // the face lies on xi_d = sgn in natural coordinates (face tables of get_face.h)
    int d, sgn;
    if (NDIM == 2) {
      d = (fc & 1) ? 0 : 1;
      sgn = (fc == 0 || fc == 3) ? -1 : 1;
    } else {
      const int dd[6] = {2, 1, 0, 1, 0, 2}, ss[6] = {-1, -1, 1, 1, -1, 1};
      d = dd[fc];
      sgn = ss[fc];
    }
    const int nq = (NDIM == 2) ? 2 : 4;
    for (int q = 0; q < nq; q++) {
      double z[3], w = 1.0;
      int free = 0;
      for (int c = 0; c < NDIM; c++) {
        if (c == d) {
          z[c] = sgn;
        } else {
          const int bit = (q >> free) & 1;
          z[c] = a.gz[bit];
          w *= a.gw[bit];
          free++;
        }
      }
      double Phi[NNOD], dPxi[NNOD][3], dPhi[NNOD][3], jac[3][3];
      shape_fn<NDIM>(z, Phi, dPxi);
      if (Hn) hnm_shape<NDIM>(Hn, Phi, dPxi);
      phys_deriv<NDIM>(dPxi, nd, dPhi, jac);
      double n[3] = {0, 0, 0};  // outward normal times the surface element and the weight
      if (NDIM == 2) {
        const int c1 = 1 - d;
        const double tx = jac[0][c1], ty = jac[1][c1];
        n[0] = (d == 0 ? ty : -ty) * sgn * w;
        n[1] = (d == 0 ? -tx : tx) * sgn * w;
      } else {
        const int c1 = (d + 1) % 3, c2 = (d + 2) % 3;
        const double t1[3] = {jac[0][c1], jac[1][c1], jac[2][c1]}, t2[3] = {jac[0][c2], jac[1][c2], jac[2][c2]};
        n[0] = (t1[1] * t2[2] - t1[2] * t2[1]) * sgn * w;
        n[1] = (t1[2] * t2[0] - t1[0] * t2[2]) * sgn * w;
        n[2] = (t1[0] * t2[1] - t1[1] * t2[0]) * sgn * w;
      }
      GpStateT<Dual> f;
      Dual p = 0.0, Tq = 0.0;
      for (int N = 0; N < NNOD; N++) {
        p += Phi[N] * nd[N].p;
        Tq += Phi[N] * nd[N].T;
      }
      for (int i = 0; i < NDIM; i++)
        for (int c = 0; c < NDIM; c++) {
          Dual t = 0.0;
          for (int N = 0; N < NNOD; N++) t += dPhi[N][c] * nd[N].v[i];
          f.dV[i][c] = t;
        }
      f.mu = gas_mu(g, Tq);
      viscous_stress<NDIM>(f);
      Dual tn = 0.0;
      for (int j = 0; j < NDIM; j++) tn += f.tau[0][j] * n[j];
      F += p * n[0] - tn / a.gas.creyn;
    }
  }
  return F;
}


// ==== pieces of the reverse sweep (adjoint_warp.cuh) ====================================
// The forward-mode functional above costs one evaluation per seed.  The reverse sweep
// evaluates L_e once in FP64 and sweeps back through it: the flux Jacobians by the
// generated reverse code (jac_adjoint.cuh), the rest by hand, and four small pieces (the
// SUPG test function, the boundary-state edits, the FDV parameters, node unpack) by dual
// numbers over their few inputs.

// adjoint of a node's primitives (fields of NodePrim)
struct PrimAdj {
  double U[5], v[3], rho, E, T, p;
};

// tau = mu (dV + dV^T) - 2/3 mu div v I: adjoint into mu and dV
template <int NDIM>
CFDV_HD CFDV_INLINE void stress_adj(const GpState& f, GpState& g) {
  double vkk = 0.0, tkk = 0.0;
  for (int k = 0; k < NDIM; k++) {
    vkk += f.dV[k][k];
    tkk += g.tau[k][k];
  }
  for (int i = 0; i < NDIM; i++)
    for (int j = 0; j < NDIM; j++) {
      const double tb = g.tau[i][j];
      g.mu += tb * (f.dV[i][j] + f.dV[j][i] - (i == j ? 2.0 / 3.0 * vkk : 0.0));
      g.dV[i][j] += f.mu * tb;
      g.dV[j][i] += f.mu * tb;
    }
  for (int k = 0; k < NDIM; k++) g.dV[k][k] -= 2.0 / 3.0 * f.mu * tkk;
}

// k = k(mu), mu = mu(T) (Thermo.h:53-75): adjoints into mu, then T
CFDV_HD CFDV_INLINE void gas_adj(const GasParams& gp, const GpState& f, GpState& g) {
  g.mu += g.k / ((gp.gamma - 1.0) * (gp.cmach * gp.cmach) * gp.Pr);
  if (!(f.T < 1.0E-12)) g.T += g.mu * f.mu * (1.5 / f.T - 1.0 / (f.T + gp.csuth));
}

CFDV_HD CFDV_INLINE void gp_zero(GpState& g) {
  g.E = g.T = g.mu = g.k = 0.0;
  for (int q = 0; q < 5; q++) {
    g.U[q] = 0.0;
    for (int c = 0; c < 3; c++) g.dU[q][c] = 0.0;
  }
  for (int i = 0; i < 3; i++) {
    g.v[i] = g.dT[i] = 0.0;
    for (int j = 0; j < 3; j++) g.dV[i][j] = g.tau[i][j] = 0.0;
  }
}

template <int NDIM, class WA>
CFDV_HD CFDV_INLINE void jac_a_adj(const GasParams& th, const GpState& f, const WA& W, GpState& g, double& gCv) {
  if constexpr (NDIM == 2) jac_a_adj_2d(th, f, W, g, gCv);
  else jac_a_adj_3d(th, f, W, g, gCv);
}
template <int NDIM, class WA>
CFDV_HD CFDV_INLINE void jac_b_rows_adj(const GasParams& th, const GpState& f, int i, const WA& W, GpState& g,
                                        double& gCv) {
  if constexpr (NDIM == 2) jac_b_rows_adj_2d(th, f, i, W, g, gCv);
  else jac_b_rows_adj_3d(th, f, i, W, g, gCv);
}
template <int NDIM, class WA>
CFDV_HD CFDV_INLINE void jac_c_rows_adj(const GasParams& th, const GpState& f, int i, const WA& W, GpState& g,
                                        double& gCv) {
  if constexpr (NDIM == 2) jac_c_rows_adj_2d(th, f, i, W, g, gCv);
  else jac_c_rows_adj_3d(th, f, i, W, g, gCv);
}

// the 2D test function's adjoint into the state (dual numbers over v, dV, rho, mu)
CFDV_HD CFDV_INLINE void psi_2d_adj(const double (*jac)[3], const double* const* x4, const GpState& f,
                                    const double (*dPhi)[3], const double* psibar, GpState& g) {
  for (int q = 0; q < 8; q++) {
    GpStateT<Dual> fd;
    fd.U[0] = Dual(f.U[0], q == 6 ? 1.0 : 0.0);
    fd.mu = Dual(f.mu, q == 7 ? 1.0 : 0.0);
    for (int i = 0; i < 2; i++) {
      fd.v[i] = Dual(f.v[i], q == i ? 1.0 : 0.0);
      for (int j = 0; j < 2; j++) fd.dV[i][j] = Dual(f.dV[i][j], q == 2 + 2 * i + j ? 1.0 : 0.0);
    }
    Dual Psi[4];
    psi_2d<Dual>(jac, x4, fd, dPhi, Psi);
    double d = 0.0;
    for (int N = 0; N < 4; N++) d += psibar[N] * Psi[N].d;
    if (q < 2) g.v[q] += d;
    else if (q < 6) g.dV[(q - 2) / 2][(q - 2) % 2] += d;
    else if (q == 6) g.U[0] += d;
    else g.mu += d;
  }
}

// the boundary-state edits' adjoint: g (of the edited state) -> graw (of the sums), dual
// numbers over the fields an edit reads (v, dV, dT, dU, mu); E, T, U, k pass through
template <int NDIM>
CFDV_HD void face_edit_adj(int code, const GpState& fraw, const double* x0, const double* x1, const double* en,
                           int adiabatic, const GpState& g, GpState& graw) {
  constexpr int NEQ = NDIM + 2;
  graw.E += g.E;
  graw.T += g.T;
  graw.k += g.k;
  for (int q = 0; q < NEQ; q++) graw.U[q] += g.U[q];
  constexpr int K = NDIM + NDIM * NDIM + NDIM + NEQ * NDIM + 1;
  for (int q = 0; q < K; q++) {
    GpStateT<Dual> fd;
    fd.E = fraw.E; fd.T = fraw.T; fd.k = fraw.k;
    for (int c = 0; c < 5; c++) {
      fd.U[c] = fraw.U[c];
      for (int d = 0; d < 3; d++) fd.dU[c][d] = fraw.dU[c][d];
    }
    for (int i = 0; i < 3; i++) {
      fd.v[i] = fraw.v[i];
      fd.dT[i] = fraw.dT[i];
      for (int j = 0; j < 3; j++) {
        fd.dV[i][j] = fraw.dV[i][j];
        fd.tau[i][j] = 0.0;
      }
    }
    fd.mu = fraw.mu;
    int o = q;
    if (o < NDIM) fd.v[o].d = 1.0;
    else if ((o -= NDIM) < NDIM * NDIM) fd.dV[o / NDIM][o % NDIM].d = 1.0;
    else if ((o -= NDIM * NDIM) < NDIM) fd.dT[o].d = 1.0;
    else if ((o -= NDIM) < NEQ * NDIM) fd.dU[o / NDIM][o % NDIM].d = 1.0;
    else fd.mu.d = 1.0;
    if constexpr (NDIM == 2) edit_face_state_2d(code, fd, x0, x1, en);
    else edit_face_state_3d(code, fd, en, adiabatic);
    double d = g.mu * fd.mu.d;
    for (int i = 0; i < NDIM; i++) {
      d += g.v[i] * fd.v[i].d + g.dT[i] * fd.dT[i].d;
      for (int j = 0; j < NDIM; j++) d += g.dV[i][j] * fd.dV[i][j].d + g.tau[i][j] * fd.tau[i][j].d;
    }
    for (int c = 0; c < NEQ; c++)
      for (int j = 0; j < NDIM; j++) d += g.dU[c][j] * fd.dU[c][j].d;
    o = q;
    if (o < NDIM) graw.v[o] += d;
    else if ((o -= NDIM) < NDIM * NDIM) graw.dV[o / NDIM][o % NDIM] += d;
    else if ((o -= NDIM * NDIM) < NDIM) graw.dT[o] += d;
    else if ((o -= NDIM) < NEQ * NDIM) graw.dU[o / NDIM][o % NDIM] += d;
    else graw.mu += d;
  }
}

}  // namespace cfdv
