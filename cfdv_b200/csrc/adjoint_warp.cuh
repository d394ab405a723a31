// Reverse sweep of the element functional, one lane per Gauss point (the kernel is in
// adjoint.cu; tests/emu/adj_emu.cpp runs the same code on the CPU with one fiber per lane).
//
// A sweep of a whole element by one thread would keep the element's tape in that thread's
// local memory.  Here a warp takes EPW = 32 / Q elements (4 hex8, 8 quad4) and each lane one
// Gauss point of one element:
//   lane = j * Q + q: element slot j of the warp, Gauss point q (and node q: Q == NNOD).
// Every lane runs the same code on its own point, so the warp never diverges on the
// Jacobian kind or direction.  Per pass (the domain points, then each boundary face's points)
// a lane
//   1. forms the flux Jacobians a, b, c of its point and contracts them with the row
//      weights as it goes (nothing of size 25 or 75 is kept), and the flux sums;
//   2. forms the scalar adjoints of the contraction;
//   3. reverses the flux sums and the Jacobians (the generated reverse code, with the entry
//      weights formed where that code reads them) into the state adjoint g, then the stress,
//      gas law and (2D) upwind test function, or on a face the boundary edits;
//   4. scatters g to the pass nodes: for each node the element's lanes sum their shares with
//      shuffles, and the lane whose index is the node's adds them to the node's adjoint.
// A lane's point (state, shape functions, row weights) sits in its own shared-memory slot,
// the element's nodes and node adjoints in shared memory beside them.  The lanes then reverse the FDV
// parameters and the node unpack (lane q for node q).  The same sweep gives d L_e / d dt and
// d L_e / d Mach: dt enters only the contraction; the Mach number enters through Cv, cgas and
// cmach (node unpack, node Mach and Reynolds numbers, k(mu) at the points, Cv in the b and c
// Jacobians).
//
// Lanes is the warp's collectives, called by every lane at the same points: sync() (a barrier
// with shared-memory ordering), sum(v, m) = v + the value of lane (lane ^ m) for m < Q (the
// element's lanes), any(p) (p of some lane of the warp), and task_sync() at each Jacobian
// task of the domain pass, where every warp of the block meets (a barrier of the block, or
// nothing), so that the block's warps run one task's code at a time.
#pragma once
#include "adjoint.cuh"

namespace cfdv {

template <int NDIM>
struct WarpVjp {
  using T = FormTraits<NDIM>;
  static constexpr int Q = T::Q, QF = T::QF, NNOD = T::NNOD, NBN = T::NBN, NEQ = T::NEQ, KE = T::KE,
                       NFACE = T::NFACE;
  static constexpr int EPW = 32 / Q;  // elements per warp
  static constexpr int NSUM = StateSums<NDIM>::COUNT;
  static_assert(Q == NNOD, "lane q owns Gauss point q and node q");
};

// the upwind test function of a 2D domain point (nothing in 3D)
template <int NDIM>
struct WarpVjpSupg {
  double uS[5], mPsi[5], Psi[4];
  double sj[3][3];  // the upwind term's Jacobian
};
template <>
struct WarpVjpSupg<3> {};

// 3D: the scalar adjoints that weight the a and b entries (abar_b, va1_b, vb1_b of the pass),
// kept here rather than in registers through the Jacobians' reverse (2D: in registers)
template <int NDIM>
struct WarpVjpEntryAdj {
  double xb[5], va[5], vb[5];
};
template <>
struct WarpVjpEntryAdj<2> {};

// one lane's Gauss point
template <int NDIM>
struct WarpVjpPointData : WarpVjpSupg<NDIM>, WarpVjpEntryAdj<NDIM> {
  static constexpr int NNOD = FormTraits<NDIM>::NNOD;
  GpState f;  // state at the point (edited on a face)
  double Phi[NNOD], dPhi[NNOD][3];
  double wi[NDIM][5], u0[5], u1[NDIM][5];  // row weights and interpolated dU
  double mterm;                            // sum_r m0(r) u0(r): the mass term of L_e
  double en[3];                            // face: weighted normal
  double omega;                            // w J (domain) or 1 (face)
};
// padded to an odd number of doubles, so that the 32 lanes reading one field of their own
// slots hit distinct banks
template <int NDIM>
struct WarpVjpPoint : WarpVjpPointData<NDIM> {
  double pad[(sizeof(WarpVjpPointData<NDIM>) / 8) % 2 == 0 ? 1 : 2];
};

template <int NDIM>
struct WarpVjpElem {
  using T = FormTraits<NDIM>;
  NodePrim nd[T::NNOD];
  PrimAdj na[T::NNOD];  // node adjoints: lane q alone writes na[q]
  double wgt[T::KE], du[T::KE];
  double Mn[T::NNOD], Ren[T::NNOD];
  double s[4];  // s1..s4
};

template <int NDIM>
struct WarpVjpShared {
  WarpVjpElem<NDIM> el[WarpVjp<NDIM>::EPW];
  WarpVjpPoint<NDIM> pt[32];
};

// a lane's running sums over its element (summed over the element's lanes at the end)
struct WarpVjpAcc {
  double sbar[4];  // adjoints of s1..s4
  double ddt, dmach, val;
};

// ---- the Jacobians of a point, contracted with the row weights as they are formed ---------
template <int NDIM, int I, bool PSI>
CFDV_HD CFDV_INLINE void fwd_b_rows(const GasParams& gp, const WarpVjpPoint<NDIM>& P, double* abar, double* vb1,
                                    double& Sb, double* vbS) {
  constexpr int NEQ = NDIM + 2;
  double J[25];
  jac_b_rows<NDIM>(gp, P.f, I, J);
#pragma unroll
  for (int r = 0; r < NEQ; r++)
#pragma unroll
    for (int c = 0; c < NEQ; c++) {
      const double bv = J[r * 5 + c];
      abar[c] += P.wi[I][r] * bv;
      vb1[r] += bv * P.u1[I][c];
      Sb += P.wi[I][r] * (bv * P.u0[c]);
      if constexpr (PSI) vbS[r] += bv * P.uS[c];
    }
}

template <int NDIM, int I>
CFDV_HD CFDV_INLINE double fwd_c_rows(const GasParams& gp, const WarpVjpPoint<NDIM>& P) {
  constexpr int NEQ = NDIM + 2;
  double C[75];
  jac_c_rows<NDIM>(gp, P.f, I, C);
  double Gam = 0.0;
#pragma unroll
  for (int j = 0; j < NDIM; j++)
#pragma unroll
    for (int r = 0; r < NEQ; r++) {
      double t = 0.0;
#pragma unroll
      for (int c = 0; c < NEQ; c++) t += C[j * 25 + r * 5 + c] * P.u1[j][c];
      Gam += P.wi[I][r] * t;
    }
  return Gam;
}

template <int NDIM, bool PSI>
CFDV_HD CFDV_INLINE void fwd_a(const GasParams& gp, const WarpVjpPoint<NDIM>& P, double* abar, double* va1,
                               double& Sa, double* vaS) {
  constexpr int NEQ = NDIM + 2;
  double J[NDIM * 25];
  jac_a<NDIM>(gp, P.f, J);
#pragma unroll
  for (int i = 0; i < NDIM; i++)
#pragma unroll
    for (int r = 0; r < NEQ; r++)
#pragma unroll
      for (int c = 0; c < NEQ; c++) {
        const double av = J[i * 25 + r * 5 + c];
        abar[c] += P.wi[i][r] * av;
        va1[r] += av * P.u1[i][c];
        Sa += P.wi[i][r] * (av * P.u0[c]);
        if constexpr (PSI) vaS[r] += av * P.uS[c];
      }
}

// ---- entry weights of the Jacobian reverse, formed where the generated code reads them ----
// a (I0 = 0, idx = i*25 + r*5 + c) and the b rows of direction I0 (idx = r*5 + c):
//   W = wi(i,r) xbar_b(c) + v1_b(r) u1(i,c) + S_b wi(i,r) u0(c) [+ vS_b(r) uS(c)]
template <int NDIM, bool PSI, int I0>
struct WeightsAB {
  const WarpVjpPoint<NDIM>& P;
  const double* xbar_b;
  const double* v1_b;
  const double* vS_b;
  double S_b;
  CFDV_HD CFDV_INLINE double operator[](int idx) const {
    const int i = I0 + idx / 25, r = (idx / 5) % 5, c = idx % 5;
    double w = P.wi[i][r] * xbar_b[c] + v1_b[r] * P.u1[i][c] + S_b * P.wi[i][r] * P.u0[c];
    if constexpr (PSI) w += vS_b[r] * P.uS[c];
    return w;
  }
};
// c rows of direction I (idx = j*25 + r*5 + c): W = Gam_b wi(I,r) u1(j,c)
template <int NDIM, int I>
struct WeightsC {
  const WarpVjpPoint<NDIM>& P;
  double Gam_b;
  CFDV_HD CFDV_INLINE double operator[](int idx) const {
    const int j = idx / 25, r = (idx / 5) % 5, c = idx % 5;
    return Gam_b * P.wi[I][r] * P.u1[j][c];
  }
};

// Reverse of the convective part F(i, r) of node_flux_entry with respect to the node's U and
// p: nU += fb dF/dU, np += fb dF/dp (the same formulas, differentiated by hand)
template <int NDIM>
CFDV_HD CFDV_INLINE void conv_flux_adj(const NodePrim& n, int i, int r, double fb, double* nU, double& np) {
  const double rho = n.U[0], irho = 1.0 / rho;
  if constexpr (NDIM == 2) {
    const double l = n.U[1], m = n.U[2], e = n.U[3], p = n.p;
    const double li = (i == 0) ? l : m;
    if (r == 0) {
      nU[1 + i] += fb;
    } else if (r == 1 || r == 2) {
      if (r == 1 + i) {  // p + li^2 / rho
        np += fb;
        nU[1 + i] += fb * 2.0 * li * irho;
        nU[0] -= fb * li * li * irho * irho;
      } else {  // l m / rho
        nU[1] += fb * m * irho;
        nU[2] += fb * l * irho;
        nU[0] -= fb * l * m * irho * irho;
      }
    } else {  // (p + e) li / rho
      np += fb * li * irho;
      nU[3] += fb * li * irho;
      nU[1 + i] += fb * (p + e) * irho;
      nU[0] -= fb * (p + e) * li * irho * irho;
    }
  } else {
    const double vi = n.U[1 + i] * irho;
    if (r == 0) {  // rho vi, rho = U0: d/dU0 = vi - vi
      nU[1 + i] += fb;
    } else if (r <= 3) {  // rho vi vj (+ p)
      const double vj = n.U[r] * irho;
      nU[0] -= fb * vi * vj;
      nU[1 + i] += fb * vj;
      nU[r] += fb * vi;
      if (i == r - 1) np += fb;
    } else {  // (rho E + p) vi, E = U4 / U0
      const double h = n.U[4] + n.p;
      nU[0] -= fb * h * vi * irho;
      nU[1 + i] += fb * h * irho;
      nU[4] += fb * vi;
      np += fb * vi;
    }
  }
}

// Reverse of the 3D boundary edits that only zero entries and recompute the stress
// (edit_face_state_3d, formation.cuh): g (of the edited state f) -> graw (of the raw sums),
// for the fields the edits read (v, dV, dT, dU, mu); E, T, U, k pass through in face_edit_adj
// and here alike.  Returns false for the codes left to the dual-number face_edit_adj.
CFDV_HD CFDV_INLINE bool face_edit_adj_3d_direct(int code, const GpState& f, int adiabatic, GpState& g,
                                                 GpState& graw) {
  int zero_dV = -1, zero_dT = -1;  // column of dV / entry of dT the edit zeroes (-1: none)
  bool stress = false;
  switch (code) {
    case 2:
    case 12: zero_dV = 2; zero_dT = 2; break;
    case -1: break;
    case 1:
    case 51: stress = true; zero_dT = adiabatic ? 2 : -1; break;
    case 21:
    case 31: stress = true; zero_dT = adiabatic ? 1 : -1; break;
    case 11: stress = true; zero_dT = adiabatic ? 0 : -1; break;
    case 8: stress = true; break;
    case 6:  // dT[0] = 0, stress, tau[i][0] = 0
      stress = true;
      zero_dT = 0;
      for (int i = 0; i < 3; i++) g.tau[i][0] = 0.0;
      break;
    case 22:  // dV[:,1] = 0, dT[1] = 0, stress, five entries of tau zeroed
      stress = true;
      zero_dV = 1;
      zero_dT = 1;
      g.tau[0][1] = g.tau[1][1] = g.tau[2][1] = g.tau[1][0] = g.tau[1][2] = 0.0;
      break;
    default: return false;
  }
  if (stress) stress_adj<3>(f, g);  // f: the state the stress was formed from (edited dV)
  if (zero_dV >= 0)
    for (int i = 0; i < 3; i++) g.dV[i][zero_dV] = 0.0;
  if (zero_dT >= 0) g.dT[zero_dT] = 0.0;
  graw.E += g.E;
  graw.T += g.T;
  graw.k += g.k;
  graw.mu += g.mu;
  for (int q = 0; q < 5; q++) {
    graw.U[q] += g.U[q];
    for (int c = 0; c < 3; c++) graw.dU[q][c] += g.dU[q][c];
  }
  for (int i = 0; i < 3; i++) {
    graw.v[i] += g.v[i];
    graw.dT[i] += g.dT[i];
    for (int j = 0; j < 3; j++) graw.dV[i][j] += g.dV[i][j];
  }
  return true;
}

// element node of pass node b (face-local numbering on a face)
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE int pass_elem_node(int fc, int b) {
  return FACE ? face_node(NDIM, fc, b) : b;
}

// sum over the element's lanes (masks 1 .. Q/2)
template <int Q, class Lanes>
CFDV_HD CFDV_INLINE double elem_sum(Lanes& L, double v) {
#pragma unroll
  for (int m = 1; m < Q; m <<= 1) v = L.sum(v, m);
  return v;
}

// Gauss-point state sum v of point P over the pass nodes (the order of gp_state_sums)
template <int NDIM, bool FACE>
CFDV_HD CFDV_INLINE void warp_state_sum(const WarpVjpElem<NDIM>& El, int fc, WarpVjpPoint<NDIM>& P, int v) {
  constexpr int NEQ = NDIM + 2, NN = FACE ? FormTraits<NDIM>::NBN : FormTraits<NDIM>::NNOD;
  GpState& f = P.f;
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
    const NodePrim& n = El.nd[pass_elem_node<NDIM, FACE>(fc, N)];
    const double coef = (c < 0) ? P.Phi[N] : P.dPhi[N][c];
    const double val = (kind == 0) ? n.E : (kind == 1) ? n.T : (kind == 2) ? n.U[idx] : n.v[idx];
    acc = RN_ADD(acc, RN_MUL(coef, val));
  }
  *dst = acc;
}

// sums over the pass nodes of the point's shape functions, weighted by the node velocity:
// SP = sum_b Phi_b, SD_i = sum_b dPhi_b,i, PV_j = sum_b Phi_b v_b,j, DV_ij = sum_b dPhi_b,i v_b,j
template <int NDIM>
CFDV_HD CFDV_INLINE void pass_node_sums(const WarpVjpElem<NDIM>& El, const WarpVjpPoint<NDIM>& P, bool face, int fc,
                                        double& SP, double* SD, double* PV, double (*DV)[NDIM]) {
  const int NN = face ? FormTraits<NDIM>::NBN : FormTraits<NDIM>::NNOD;
  SP = 0.0;
#pragma unroll
  for (int i = 0; i < NDIM; i++) {
    SD[i] = PV[i] = 0.0;
#pragma unroll
    for (int j = 0; j < NDIM; j++) DV[i][j] = 0.0;
  }
  for (int b = 0; b < NN; b++) {
    const NodePrim& nb = El.nd[face ? face_node(NDIM, fc, b) : b];
    const double ph = P.Phi[b];
    SP += ph;
#pragma unroll
    for (int j = 0; j < NDIM; j++) PV[j] += ph * nb.v[j];
#pragma unroll
    for (int i = 0; i < NDIM; i++) {
      const double d = P.dPhi[b][i];
      SD[i] += d;
#pragma unroll
      for (int j = 0; j < NDIM; j++) DV[i][j] += d * nb.v[j];
    }
  }
}

// ---- one pass: the domain points, or the points of boundary face fc ----------------------
// On entry the lane's point (P; on a face also the state before the edits, fr) is formed
// when `on` (the lane has a point in this pass); `pass` tells whether the lane's element
// takes part (it then owns node q in the scatter).  The pass's node adjoints are added into
// na, the adjoint of the lane's node q.  Domain and face passes run the same code (one copy
// of the Jacobians' reverse in the kernel); a 2D face point has uS = mPsi = 0, which drops
// the upwind terms.
template <int NDIM, class Lanes>
CFDV_HD CFDV_INLINE void warp_vjp_pass(const FunctionalArgs& a, const WarpVjpElem<NDIM>& El, WarpVjpPoint<NDIM>& P,
                                       const GpState& fr, const double* s, bool face, bool on, bool pass, int q,
                                       int fc, int code, Lanes& L, WarpVjpAcc& acc, PrimAdj& na) {
  using V = WarpVjp<NDIM>;
  constexpr int NEQ = V::NEQ;
  constexpr bool PSI = NDIM == 2;
  const int NN = face ? V::NBN : V::NNOD;
  const GasParams& gp = a.gas;
  const bool withF = (NDIM == 2) || a.physical_3d_flux;
  const double dt = a.dt, dtsq_2 = dt * dt / 2.0, sgn = face ? -1.0 : 1.0;
  const double reinv = 1.0 / gp.creyn;

  // 1. forward: the Jacobians contracted with the row weights, the flux sums
  double abar[5] = {0, 0, 0, 0, 0}, va1[5] = {0, 0, 0, 0, 0}, vb1[5] = {0, 0, 0, 0, 0};
  double vaS[5] = {0, 0, 0, 0, 0}, vbS[5] = {0, 0, 0, 0, 0}, divF[5] = {0, 0, 0, 0, 0};
  double Sa = 0.0, Sb = 0.0, Gam = 0.0, Fterm = 0.0;
  // one Jacobian at a time, the same task in every lane (and, through task_sync in the
  // domain pass, in every warp of the block): one Jacobian's code and temporaries at once
#pragma unroll 1
  for (int t = 0; t < 1 + 2 * NDIM; t++) {
    if (!face) L.task_sync();
    if (on) {
      switch (t) {
        case 0: fwd_a<NDIM, PSI>(gp, P, abar, va1, Sa, vaS); break;
        case 1: fwd_b_rows<NDIM, 0, PSI>(gp, P, abar, vb1, Sb, vbS); break;
        case 2: fwd_b_rows<NDIM, 1, PSI>(gp, P, abar, vb1, Sb, vbS); break;
        case 3: Gam += fwd_c_rows<NDIM, 0>(gp, P); break;
        case 4: Gam += fwd_c_rows<NDIM, 1>(gp, P); break;
        case 5:
          if constexpr (NDIM == 3) fwd_b_rows<NDIM, 2, PSI>(gp, P, abar, vb1, Sb, vbS);
          break;
        default:
          if constexpr (NDIM == 3) Gam += fwd_c_rows<NDIM, 2>(gp, P);
          break;
      }
    }
  }
  if (on) {
    // the viscous flux G(i, r) is the same at every pass node for r = 1..ndim and linear in the
    // node velocity for the energy row, so its sums over the nodes need only
    // SP = sum_b Phi_b, SD_i = sum_b dPhi_b,i, PV_j = sum_b Phi_b v_b,j, DV_ij = sum_b dPhi_b,i v_b,j
    double SP, SD[NDIM], PV[NDIM], DV[NDIM][NDIM];
    pass_node_sums<NDIM>(El, P, face, fc, SP, SD, PV, DV);
#pragma unroll
    for (int i = 0; i < NDIM; i++) {
#pragma unroll
      for (int r = 1; r <= NDIM; r++) {
        const double G = -P.f.tau[i][r - 1] * reinv;
        Fterm += (SP * P.wi[i][r]) * G;
        divF[r] += SD[i] * G;
      }
      double tp = 0.0, td = 0.0;
#pragma unroll
      for (int j = 0; j < NDIM; j++) {
        tp -= P.f.tau[i][j] * PV[j];
        td -= P.f.tau[i][j] * DV[i][j];
      }
      Fterm += P.wi[i][NDIM + 1] * ((tp - P.f.k * P.f.dT[i] * SP) * reinv);
      divF[NDIM + 1] += (td - P.f.k * P.f.dT[i] * SD[i]) * reinv;
    }
    if (withF) {  // the nodes' convective fluxes
      for (int b = 0; b < NN; b++) {
        const NodePrim& nb = El.nd[face ? face_node(NDIM, fc, b) : b];
#pragma unroll
        for (int i = 0; i < NDIM; i++)
#pragma unroll
          for (int r = 0; r < NEQ; r++) {
            const double F = node_conv_flux_entry<NDIM>(nb, i, r);
            Fterm += (P.Phi[b] * P.wi[i][r]) * F;
            divF[r] += P.dPhi[b][i] * F;
          }
      }
    }
  }
  // 2. scalar adjoints
  const double om = on ? P.omega : 0.0;
  double abar_b[5], divF_b[5], va1_b[5], vb1_b[5], vaS_b[5], vbS_b[5];
  double ad = 0.0, ab = 0.0, ava = 0.0, avb = 0.0, pa = 0.0, pb = 0.0;
#pragma unroll
  for (int r = 0; r < 5; r++) abar_b[r] = divF_b[r] = va1_b[r] = vb1_b[r] = vaS_b[r] = vbS_b[r] = 0.0;
#pragma unroll
  for (int r = 0; r < NEQ; r++) {
    const double beta = s[1] * va1[r] + s[3] * vb1[r];
    abar_b[r] = -om * sgn * dtsq_2 * (divF[r] + beta);
    divF_b[r] = -om * sgn * dtsq_2 * abar[r];  // also the adjoint of beta
    va1_b[r] = divF_b[r] * s[1];
    vb1_b[r] = divF_b[r] * s[3];
    if constexpr (PSI) {
      const double mp = on ? P.mPsi[r] : 0.0;
      vaS_b[r] = -om * dt * mp * s[0];
      vbS_b[r] = -om * dt * mp * s[2];
      pa += mp * vaS[r];
      pb += mp * vbS[r];
    }
    ad += abar[r] * divF[r];
    ab += abar[r] * beta;
    ava += abar[r] * va1[r];
    avb += abar[r] * vb1[r];
  }
  const double Sa_b = om * sgn * dt * s[0], Sb_b = om * sgn * dt * s[2], Gam_b = om * sgn * dt * s[2];
  const double Fterm_b = om * sgn * dt;
  if (on) {
    const double pterm = PSI ? s[0] * pa + s[2] * pb : 0.0;
    acc.sbar[0] += om * (sgn * dt * Sa - (PSI ? dt * pa : 0.0));
    acc.sbar[1] += -om * sgn * dtsq_2 * ava;
    acc.sbar[2] += om * (sgn * dt * Sb + sgn * dt * Gam - (PSI ? dt * pb : 0.0));
    acc.sbar[3] += -om * sgn * dtsq_2 * avb;
    acc.ddt += om * (sgn * (Fterm - dt * ad) + sgn * (s[0] * Sa + s[2] * Sb) + sgn * s[2] * Gam - sgn * dt * ab - pterm);
    const double mterm = face ? 0.0 : P.mterm;
    acc.val += om * (sgn * (dt * Fterm - dtsq_2 * ad) - mterm + sgn * dt * (s[0] * Sa + s[2] * Sb) -
                     sgn * (-(dt * s[2]) * Gam + dtsq_2 * ab) - dt * pterm);
  }

  // 3. reverse into the state adjoint g
  GpState g;
  gp_zero(g);
  if (on) {
    // flux sums: the Gauss-point part (the node part is scattered below), over the same sums
    double SP, SD[NDIM], PV[NDIM], DV[NDIM][NDIM];
    pass_node_sums<NDIM>(El, P, face, fc, SP, SD, PV, DV);
#pragma unroll
    for (int i = 0; i < NDIM; i++) {
#pragma unroll
      for (int r = 1; r <= NDIM; r++) g.tau[i][r - 1] -= (Fterm_b * P.wi[i][r] * SP + divF_b[r] * SD[i]) * reinv;
      const double aw = Fterm_b * P.wi[i][NDIM + 1], ad_ = divF_b[NDIM + 1];
#pragma unroll
      for (int j = 0; j < NDIM; j++) g.tau[i][j] -= (aw * PV[j] + ad_ * DV[i][j]) * reinv;
      const double fbs = aw * SP + ad_ * SD[i];
      g.k -= fbs * P.f.dT[i] * reinv;
      g.dT[i] -= fbs * P.f.k * reinv;
    }
  }
  // the Jacobians
  const double *XB = abar_b, *VA = va1_b, *VB = vb1_b;
  if constexpr (NDIM == 3) {  // the entry weights read them from the lane's slot
    if (on)
#pragma unroll
      for (int r = 0; r < 5; r++) {
        P.xb[r] = abar_b[r];
        P.va[r] = va1_b[r];
        P.vb[r] = vb1_b[r];
      }
    XB = P.xb;
    VA = P.va;
    VB = P.vb;
  }
  double gCv = 0.0;
#pragma unroll 1
  for (int t = 0; t < 1 + 2 * NDIM; t++) {
    if (!face) L.task_sync();
    if (on) {
      switch (t) {
        case 0: jac_a_adj<NDIM>(gp, P.f, WeightsAB<NDIM, PSI, 0>{P, XB, VA, vaS_b, Sa_b}, g, gCv); break;
        case 1:
          jac_b_rows_adj<NDIM>(gp, P.f, 0, WeightsAB<NDIM, PSI, 0>{P, XB, VB, vbS_b, Sb_b}, g, gCv);
          break;
        case 2:
          jac_b_rows_adj<NDIM>(gp, P.f, 1, WeightsAB<NDIM, PSI, 1>{P, XB, VB, vbS_b, Sb_b}, g, gCv);
          break;
        case 3: jac_c_rows_adj<NDIM>(gp, P.f, 0, WeightsC<NDIM, 0>{P, Gam_b}, g, gCv); break;
        case 4: jac_c_rows_adj<NDIM>(gp, P.f, 1, WeightsC<NDIM, 1>{P, Gam_b}, g, gCv); break;
        case 5:
          if constexpr (NDIM == 3)
            jac_b_rows_adj<NDIM>(gp, P.f, 2, WeightsAB<NDIM, PSI, 2>{P, XB, VB, vbS_b, Sb_b}, g, gCv);
          break;
        default:
          if constexpr (NDIM == 3) jac_c_rows_adj<NDIM>(gp, P.f, 2, WeightsC<NDIM, 2>{P, Gam_b}, g, gCv);
          break;
      }
    }
  }
  if (on) {
    acc.dmach += gCv * (-2.0 * gp.Cv / gp.cmach);  // d Cv / d M = -2 Cv / M
    // stress, gas law, test function; or the boundary edits
    if (!face) {
      if constexpr (NDIM == 2) {
        double psibar[4];
        for (int N = 0; N < 4; N++) {
          double t = 0.0;
          for (int r = 0; r < NEQ; r++) t += (-om * dt * (s[0] * vaS[r] + s[2] * vbS[r])) * El.wgt[N * NEQ + r];
          psibar[N] = t;
        }
        const double* x4[4] = {El.nd[0].x, El.nd[1].x, El.nd[2].x, El.nd[3 % V::NNOD].x};
        psi_2d_adj(P.sj, x4, P.f, P.dPhi, psibar, g);
      }
      stress_adj<NDIM>(P.f, g);
      acc.dmach += g.k * P.f.k * (-2.0 / gp.cmach);  // k = mu / ((gamma-1) M^2 Pr)
      gas_adj(gp, P.f, g);
    } else {
      GpState graw;
      gp_zero(graw);
      bool direct = false;  // the zeroing-and-stress edits of 3D faces, reversed directly
      if constexpr (NDIM == 3) direct = face_edit_adj_3d_direct(code, P.f, gp.adiabatic, g, graw);
      if (!direct)
        face_edit_adj<NDIM>(code, fr, El.nd[face_node(NDIM, fc, 0)].x, El.nd[face_node(NDIM, fc, 1)].x, P.en,
                            gp.adiabatic, g, graw);
      acc.dmach += graw.k * fr.k * (-2.0 / gp.cmach);
      gas_adj(gp, fr, graw);
      g = graw;
    }
  }
  // 4. scatter to the pass nodes: state sums and the node part of the flux sums
  for (int b = 0; b < NN; b++) {
    const int node = face ? face_node(NDIM, fc, b) : b;
    double cE = 0.0, cT = 0.0, cU[5] = {0, 0, 0, 0, 0}, cv[3] = {0, 0, 0}, cp = 0.0;
    if (on) {
      const double Phi = P.Phi[b];
      cE = Phi * g.E;
      double t = Phi * g.T;
#pragma unroll
      for (int c = 0; c < NDIM; c++) t += P.dPhi[b][c] * g.dT[c];
      cT = t;
#pragma unroll
      for (int qq = 0; qq < NEQ; qq++) {
        double u = Phi * g.U[qq];
#pragma unroll
        for (int c = 0; c < NDIM; c++) u += P.dPhi[b][c] * g.dU[qq][c];
        cU[qq] = u;
      }
#pragma unroll
      for (int i = 0; i < NDIM; i++) {
        double v = Phi * g.v[i];
#pragma unroll
        for (int c = 0; c < NDIM; c++) v += P.dPhi[b][c] * g.dV[i][c];
        cv[i] = v;
      }
      const NodePrim& nb = El.nd[node];
#pragma unroll
      for (int i = 0; i < NDIM; i++) {
        const double fb = Fterm_b * P.Phi[b] * P.wi[i][NDIM + 1] + divF_b[NDIM + 1] * P.dPhi[b][i];
#pragma unroll
        for (int j = 0; j < NDIM; j++) cv[j] -= fb * P.f.tau[i][j] * reinv;
      }
      if (withF) {
#pragma unroll
        for (int i = 0; i < NDIM; i++)
#pragma unroll
          for (int r = 0; r < NEQ; r++) {
            const double fb = Fterm_b * P.Phi[b] * P.wi[i][r] + divF_b[r] * P.dPhi[b][i];
            conv_flux_adj<NDIM>(nb, i, r, fb, cU, cp);
          }
      }
    }
    cE = elem_sum<V::Q>(L, cE);
    cT = elem_sum<V::Q>(L, cT);
#pragma unroll
    for (int qq = 0; qq < NEQ; qq++) cU[qq] = elem_sum<V::Q>(L, cU[qq]);
#pragma unroll
    for (int i = 0; i < NDIM; i++) cv[i] = elem_sum<V::Q>(L, cv[i]);
    if (withF) cp = elem_sum<V::Q>(L, cp);
    if (pass && q == node) {
      na.E += cE;
      na.T += cT;
#pragma unroll
      for (int qq = 0; qq < NEQ; qq++) na.U[qq] += cU[qq];
#pragma unroll
      for (int i = 0; i < NDIM; i++) na.v[i] += cv[i];
      na.p += cp;
    }
  }
}

// The elements e0 .. e0 + EPW - 1 (those below n_elements): d L_e / d U_e into a.out, and
// d L_e / d dt, d L_e / d Mach, L_e into a.out_dt, a.out_mach, a.out_val when set.  Every
// lane of the warp calls it; the functional is that of element_functional (adjoint.cuh).
template <int NDIM, class Lanes>
CFDV_HD CFDV_INLINE void warp_vjp(const FunctionalArgs& a, WarpVjpShared<NDIM>& sh, int e0, int lane, Lanes& L) {
  using V = WarpVjp<NDIM>;
  constexpr int NNOD = V::NNOD, NEQ = V::NEQ, KE = V::KE, Q = V::Q, QF = V::QF, NBN = V::NBN;
  const GasParams& gp = a.gas;
  const int j = lane / Q, q = lane % Q, e = e0 + j;
  const bool valid = e < a.n_elements;
  WarpVjpElem<NDIM>& El = sh.el[j];
  WarpVjpPoint<NDIM>& P = sh.pt[lane];
  // ---- the element's nodes (lane q: node q) and rows ----
  if (valid) {
    const int n = a.conn[(size_t)e * NNOD + q];
    node_unpack<NDIM>(gp, a.U + (size_t)n * NEQ, a.x + (size_t)n * NDIM, El.nd[q]);
    node_mach_re<NDIM>(gp, El.nd[q], &El.Mn[q], &El.Ren[q]);
    PrimAdj& z = El.na[q];
    z.rho = z.E = z.T = z.p = 0.0;
    for (int c = 0; c < 5; c++) z.U[c] = 0.0;
    for (int c = 0; c < 3; c++) z.v[c] = 0.0;
    const uint64_t mask = a.rowmask ? a.rowmask[e] : 0ull;
    for (int t = q; t < KE; t += Q) {
      const size_t gi = (size_t)a.conn[(size_t)e * NNOD + t / NEQ] * NEQ + t % NEQ;
      El.wgt[t] = ((mask >> t) & 1ull) ? 0.0 : a.w[gi];
      El.du[t] = a.dU[gi];
    }
  }
  L.sync();
  const int hi = (valid && a.hnm_idx) ? a.hnm_idx[e] : -1;
  const double* Hn = (hi >= 0) ? a.hnm + (size_t)hi * NNOD * NNOD : nullptr;
  if (valid && q < 2) fdv_pair<NNOD>(q ? El.Ren : El.Mn, q, El.s);  // s1, s2 | s3, s4
  if (valid) {
    // ---- domain point q: geometry, state, row weights, stress (2D: the test function) ----
    double z[3], dPxi[NNOD][3], jac[3][3];
    double w = 1.0;
    for (int d = 0; d < NDIM; d++) {
      const int bit = (q >> (NDIM - 1 - d)) & 1;
      z[d] = a.gz[bit];
      w *= a.gw[bit];
    }
    shape_fn<NDIM>(z, P.Phi, dPxi);
    if (Hn) hnm_shape<NDIM>(Hn, P.Phi, dPxi);
    const double J = phys_deriv<NDIM>(dPxi, El.nd, P.dPhi, jac);
    P.omega = w * J;
    for (int v = 0; v < V::NSUM; v++) warp_state_sum<NDIM, false>(El, 0, P, v);
    double mterm = 0.0;
    for (int r = 0; r < NEQ; r++) {
      double a0 = 0.0, b0 = 0.0, bs = 0.0, a1[3] = {0, 0, 0}, b1[3] = {0, 0, 0};
      for (int N = 0; N < NNOD; N++) {
        const double wv = El.wgt[N * NEQ + r], dv = El.du[N * NEQ + r];
        double sd = 0.0;
#pragma unroll
        for (int jj = 0; jj < NDIM; jj++) sd += P.dPhi[N][jj];
        a0 += P.Phi[N] * wv;
        b0 += P.Phi[N] * dv;
        bs += sd * dv;
#pragma unroll
        for (int i = 0; i < NDIM; i++) {
          a1[i] += P.dPhi[N][i] * wv;
          b1[i] += P.dPhi[N][i] * dv;
        }
      }
      mterm += a0 * b0;
      P.u0[r] = b0;
      if constexpr (NDIM == 2) P.uS[r] = bs;
#pragma unroll
      for (int i = 0; i < NDIM; i++) {
        P.wi[i][r] = a1[i];
        P.u1[i][r] = b1[i];
      }
    }
    P.mterm = mterm;
    P.f.mu = gas_mu(gp, P.f.T);
    P.f.k = gas_k(gp, P.f.mu);
    viscous_stress<NDIM>(P.f);
    if constexpr (NDIM == 2) {
      const double* x4[4] = {El.nd[0].x, El.nd[1].x, El.nd[2].x, El.nd[3].x};
      if (Hn) {
        plain_jac_2d(z, x4, P.sj);  // the upwind term's Jacobian: of the untransformed shape functions
      } else {
        for (int i = 0; i < 3; i++)
          for (int k = 0; k < 3; k++) P.sj[i][k] = jac[i][k];
      }
      psi_2d<double>(P.sj, x4, P.f, P.dPhi, P.Psi);
      for (int r = 0; r < NEQ; r++) {
        double ps = 0.0;
        for (int N = 0; N < NNOD; N++) ps += P.Psi[N] * El.wgt[N * NEQ + r];
        P.mPsi[r] = ps;
      }
    }
  }
  WarpVjpAcc acc;
  for (int i = 0; i < 4; i++) acc.sbar[i] = 0.0;
  acc.ddt = acc.dmach = acc.val = 0.0;
  PrimAdj& na = El.na[q];  // adjoint of node q's primitives
  const double* s = El.s;
  L.sync();  // s1..s4 of every element
  // ---- the passes: the domain (pass -1), then each boundary face with 0 != bc < 100
  //      (FDVGalerkin.h:455-533); one call site, so the kernel holds one copy of the pass ----
  for (int fc = -1; fc < V::NFACE; fc++) {
    const bool face = fc >= 0;
    const int code = (face && valid) ? a.bc[(size_t)e * V::NFACE + fc] : 0;
    const bool pass = face ? (code != 0 && code < 100) : valid;
    if (face && !L.any(pass)) continue;
    const bool on = pass && (!face || q < QF);
    GpState& fr = sh.pt[lane + (q < QF ? QF : 0)].f;  // face: the slot of an idle point of the element
    if (face && on) {
      const double* xf[NBN];
      for (int i = 0; i < NBN; i++) xf[i] = El.nd[face_node(NDIM, fc, i)].x;
      double xl[4][3];
      if (NDIM == 3 && Hn) {  // adaptive element: face geometry from Hnm x
        const double* xe[8];
        for (int M = 0; M < 8; M++) xe[M] = El.nd[M % NNOD].x;
        hnm_face_nodes_3d(Hn, xe, fc, xl);
        for (int i = 0; i < NBN; i++) xf[i] = xl[i % 4];
      }
      face_point_geom<NDIM>(a.gz, a.gw, xf, q, P.Phi, P.dPhi, P.en);
      if constexpr (NDIM == 3) {
        if (Hn) hnm_face_phi_3d(Hn, fc, P.Phi);
      } else {
        for (int r = 0; r < 5; r++) P.uS[r] = P.mPsi[r] = 0.0;  // no upwind term on a face
      }
      P.omega = 1.0;
      for (int v = 0; v < V::NSUM; v++) warp_state_sum<NDIM, true>(El, fc, P, v);
      for (int r = 0; r < NEQ; r++) {
        double m0 = 0.0, b0 = 0.0, b1[3] = {0, 0, 0};
        for (int m = 0; m < NBN; m++) {
          const int row = face_node(NDIM, fc, m) * NEQ + r;
          const double wv = El.wgt[row], dv = El.du[row];
          m0 += P.Phi[m] * wv;
          b0 += P.Phi[m] * dv;
#pragma unroll
          for (int jj = 0; jj < NDIM; jj++) b1[jj] += P.dPhi[m][jj] * dv;
        }
        P.u0[r] = b0;
#pragma unroll
        for (int i = 0; i < NDIM; i++) {
          P.wi[i][r] = P.en[i] * m0;
          P.u1[i][r] = b1[i];
        }
      }
      // the state before and after the boundary edits
      P.f.mu = gas_mu(gp, P.f.T);
      P.f.k = gas_k(gp, P.f.mu);
      for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) P.f.tau[i][k] = 0.0;
      fr = P.f;
      if constexpr (NDIM == 2)
        edit_face_state_2d(code, P.f, El.nd[face_node(NDIM, fc, 0)].x, El.nd[face_node(NDIM, fc, 1)].x, P.en);
      else
        edit_face_state_3d(code, P.f, P.en, gp.adiabatic);
    }
    warp_vjp_pass<NDIM>(a, El, P, face ? fr : P.f, s, face, on, pass, q, face ? fc : 0, code, L, acc, na);
  }
  // ---- FDV parameters: s1..s4 from the nodes' Mach and Reynolds numbers ----
#pragma unroll
  for (int i = 0; i < 4; i++) acc.sbar[i] = elem_sum<Q>(L, acc.sbar[i]);
  if (valid) {
    Dual vm[NNOD], vr[NNOD], sd[4];
    for (int k = 0; k < NNOD; k++) {
      vm[k] = Dual(El.Mn[k], k == q ? 1.0 : 0.0);
      vr[k] = Dual(El.Ren[k], k == q ? 1.0 : 0.0);
    }
    fdv_pair<NNOD>(vm, 0, sd);
    fdv_pair<NNOD>(vr, 1, sd);
    const double Mb = acc.sbar[0] * sd[0].d + acc.sbar[1] * sd[1].d;
    const double Rb = acc.sbar[2] * sd[2].d + acc.sbar[3] * sd[3].d;
    // ---- node q's primitives -> its U (node unpack, Mach and Reynolds numbers), and the
    //      same chain along the Mach number ----
    const NodePrim& nd = El.nd[q];
    for (int c = 0; c <= NEQ; c++) {
      const GasT<Dual> gd = dual_gas(gp, c == NEQ ? 1.0 : 0.0);
      Dual u[NEQ];
      for (int k = 0; k < NEQ; k++) u[k] = Dual(nd.U[k], k == c ? 1.0 : 0.0);
      NodePrimT<Dual> p;
      node_unpack<NDIM>(gd, u, nd.x, p);
      Dual M, R;
      node_mach_re<NDIM>(gd, p, &M, &R);
      double d = na.rho * p.rho.d + na.E * p.E.d + na.T * p.T.d + na.p * p.p.d + Mb * M.d + Rb * R.d;
      for (int k = 0; k < NEQ; k++) d += na.U[k] * p.U[k].d;
      for (int k = 0; k < NDIM; k++) d += na.v[k] * p.v[k].d;
      if (c < NEQ) a.out[(size_t)e * KE + q * NEQ + c] = d;
      else acc.dmach += d;
    }
  }
  acc.ddt = elem_sum<Q>(L, acc.ddt);
  acc.dmach = elem_sum<Q>(L, acc.dmach);
  acc.val = elem_sum<Q>(L, acc.val);
  if (valid && q == 0) {
    if (a.out_dt) a.out_dt[e] = acc.ddt;
    if (a.out_mach) a.out_mach[e] = acc.dmach;
    if (a.out_val) a.out_val[e] = acc.val;
  }
  L.sync();  // the next elements may overwrite the shared state
}

}  // namespace cfdv
