// Device-side FDV physics for one Gauss point: gas model, shape functions,
// Gauss-point flow state, viscous stress, flux Jacobians and fluxes.
//
// Formulas follow the CFDV reference (paths relative to its src/):
//   gas model            FDV/Thermo.h:8-86
//   shape functions      FiniteElement/TestFunctions2D.h:7-102, TestFunctions3D.h:7-123
//   Gauss-point state    FDV/FDVGalerkin.h:761-797, FDV/tau.h:14-42
//   a = dF/dU            FDV/NavierStokes2D.h:59-97,  FDV/NavierStokes3D.h:74-189
//   b = dG/dU            FDV/NavierStokes2D.h:100-158, FDV/NavierStokes3D.h:193-343
//   c = dG/dU_,j         FDV/NavierStokes2D.h:163-222, FDV/NavierStokes3D.h:347-477
//   F, G                 FDV/NavierStokes2D.h:11-47,  FDV/NavierStokes3D.h:10-64
// Jacobian tensors are written to shared memory with a fixed 5-equation stride:
//   a(i,r,s) -> a[(i*5+r)*5+s],  c(i,j,r,s) -> c[((i*3+j)*5+r)*5+s].
#pragma once
#include "cfdv_types.h"
#include "dual.cuh"

namespace cfdv {

// Round-to-nearest arithmetic that the compiler may not contract into FMA.  The
// Gauss-point state feeds exact-zero tests of the reference (gamma == 0, R == 0,
// S == 0 in FDVGalerkin.h:308-379); evaluating it with the reference's operation
// order and without contraction makes those decisions agree with the reference.
// rn_* (dual.cuh) are the intrinsics for doubles and carry a derivative for duals.
#define RN_MUL(a, b) ::cfdv::rn_mul((a), (b))
#define RN_ADD(a, b) ::cfdv::rn_add((a), (b))
#define RN_SUB(a, b) ::cfdv::rn_sub((a), (b))
#define RN_DIV(a, b) ::cfdv::rn_div((a), (b))

#define JA(t, i, r, s) (t)[((i)*5 + (r)) * 5 + (s)]
#define JC(t, i, j, r, s) (t)[(((i)*3 + (j)) * 5 + (r)) * 5 + (s)]

template <class S>
CFDV_HD CFDV_INLINE S gas_mu(const GasT<S>& g, S T) {
  if (T < 1.0E-12) return S(1.0);
  return RN_MUL(RN_MUL(RN_DIV(1 + g.csuth, RN_ADD(T, g.csuth)), T), sqrt(T));
}
template <class S>
CFDV_HD CFDV_INLINE S gas_k(const GasT<S>& g, S mu) {
  return mu / ((g.gamma - 1.0) * (g.cmach * g.cmach) * g.Pr);
}

// primitive state of a node (NodeUnpack.h:9-29); coordinates are plain doubles
template <class S>
struct NodePrimT {
  S U[5];
  double x[3];
  S v[3];
  S rho, E, T, p;
};
using NodePrim = NodePrimT<double>;

template <int NDIM, class S>
CFDV_HD CFDV_INLINE void node_unpack(const GasT<S>& g, const S* U, const double* x, NodePrimT<S>& n) {
#pragma unroll
  for (int k = 0; k < NDIM + 2; k++) n.U[k] = U[k];
#pragma unroll
  for (int k = 0; k < NDIM; k++) n.x[k] = x[k];
  n.rho = U[0];
  S vsqr = 0;
#pragma unroll
  for (int i = 0; i < NDIM; i++) {
    n.v[i] = RN_DIV(U[1 + i], U[0]);
    vsqr = RN_ADD(vsqr, RN_MUL(n.v[i], n.v[i]));
  }
  n.E = RN_DIV(U[NDIM + 1], U[0]);
  S e = RN_SUB(n.E, RN_MUL(0.5, vsqr));
  n.T = RN_DIV(e, g.Cv);
  n.p = RN_MUL(RN_MUL(n.rho, g.gamma - 1.0), e);
}

// CFL length of one node of an element (MPI_CFL.h:7-56): cleng / (|v| + sqrt(1.4 cgas T))
// with T from NodeUnpack (NodeUnpack.h:24-28) clipped at 1e-9; the reference uses 1.4, not
// gamma.  Returns false (no candidate) where the signal speed is not above 1e-9.
template <int NDIM, class S>
CFDV_HD CFDV_INLINE bool cfl_node_len(const S* u, double cleng, const GasT<S>& g, S* dxn) {
  S vv = 0.0;
  for (int k = 0; k < NDIM; k++) {
    const S v = RN_DIV(u[1 + k], u[0]);
    vv = RN_ADD(vv, RN_MUL(v, v));
  }
  const S Tn = RN_DIV(RN_SUB(RN_DIV(u[NDIM + 1], u[0]), RN_MUL(0.5, vv)), g.Cv);
  const S Temp = (Tn > 10E-10) ? Tn : S(0.0);
  const S sv = sqrt(vv), snd = sqrt(RN_MUL(RN_MUL(1.4, g.cgas), Temp));
  if (!(RN_ADD(sv, snd) > 10E-10)) return false;
  *dxn = RN_DIV(S(cleng), RN_ADD(sv, snd));
  return true;
}

// shape functions and natural-coordinate derivatives
template <int NDIM>
CFDV_HD CFDV_INLINE void shape_fn(const double* z, double* Phi, double (*dPxi)[3]);

template <>
CFDV_HD CFDV_INLINE void shape_fn<2>(const double* z, double* Phi, double (*dPxi)[3]) {
  const double a0 = 1 - z[0], b0 = 1 + z[0], a1 = 1 - z[1], b1 = 1 + z[1];
  Phi[0] = 0.25 * a0 * a1;
  Phi[1] = 0.25 * b0 * a1;
  Phi[2] = 0.25 * b0 * b1;
  Phi[3] = 0.25 * a0 * b1;
  dPxi[0][0] = -0.25 * a1; dPxi[1][0] = 0.25 * a1; dPxi[2][0] = 0.25 * b1; dPxi[3][0] = -0.25 * b1;
  dPxi[0][1] = -0.25 * a0; dPxi[1][1] = -0.25 * b0; dPxi[2][1] = 0.25 * b0; dPxi[3][1] = 0.25 * a0;
}

template <>
CFDV_HD CFDV_INLINE void shape_fn<3>(const double* z, double* Phi, double (*dPxi)[3]) {
  const double m[3] = {1 - z[0], 1 - z[1], 1 - z[2]};
  const double p[3] = {1 + z[0], 1 + z[1], 1 + z[2]};
  // hex8 corner signs: node N sits at (sx, sy, sz)
#pragma unroll
  for (int N = 0; N < 8; N++) {
    const int sx = ((N & 1) ^ ((N >> 1) & 1)) ? 1 : -1;  // 0:-,1:+,2:+,3:-
    const int sy = ((N >> 1) & 1) ? 1 : -1;              // 0,1:- 2,3:+
    const int sz = (N >> 2) ? 1 : -1;
    const double fx = sx > 0 ? p[0] : m[0], fy = sy > 0 ? p[1] : m[1], fz = sz > 0 ? p[2] : m[2];
    Phi[N] = 0.125 * fx * fy * fz;
    dPxi[N][0] = (sx * 0.125) * fy * fz;
    dPxi[N][1] = (sy * 0.125) * fx * fz;
    dPxi[N][2] = (sz * 0.125) * fx * fy;
  }
}

// Isoparametric map, split into the pieces a thread block evaluates in parallel:
//   jac[i][k] = dx_i/dxi_k = sum_N dPxi_N,k x_N,i      (geom_jac_entry, one entry)
//   det J and, in 3D, the adjugate inv                 (geom_det)
//   dPhi_N,i from dPxi_N, jac/inv and 1/det            (geom_dphi, one shape function)
// phys_deriv runs them in sequence for one Gauss point.
template <int NNOD, class NP>
CFDV_HD CFDV_INLINE double geom_jac_entry(const double (*dPxi)[3], const NP* nd, int i, int k) {
  double j = 0;
#pragma unroll
  for (int N = 0; N < NNOD; N++) j = RN_ADD(j, RN_MUL(dPxi[N][k], nd[N].x[i]));
  return j;
}

template <int NDIM>
CFDV_HD CFDV_INLINE double geom_det(const double (*j)[3], double (*inv)[3]);

template <>
CFDV_HD CFDV_INLINE double geom_det<2>(const double (*j)[3], double (*inv)[3]) {
  (void)inv;
  return RN_SUB(RN_MUL(j[0][0], j[1][1]), RN_MUL(j[1][0], j[0][1]));
}

template <>
CFDV_HD CFDV_INLINE double geom_det<3>(const double (*j)[3], double (*inv)[3]) {
#define M3(a, b, c) RN_MUL(RN_MUL(a, b), c)
  const double J = RN_SUB(RN_SUB(RN_SUB(RN_ADD(RN_ADD(M3(j[0][0], j[1][1], j[2][2]), M3(j[0][1], j[1][2], j[2][0])),
                                               M3(j[0][2], j[1][0], j[2][1])),
                                        M3(j[0][2], j[1][1], j[2][0])),
                                 M3(j[0][1], j[1][0], j[2][2])),
                          M3(j[0][0], j[1][2], j[2][1]));
#undef M3
#define D2(a, b, c, d) RN_SUB(RN_MUL(a, b), RN_MUL(c, d))
  inv[0][0] = D2(j[1][1], j[2][2], j[1][2], j[2][1]);
  inv[0][1] = -D2(j[1][0], j[2][2], j[1][2], j[2][0]);
  inv[0][2] = D2(j[1][0], j[2][1], j[1][1], j[2][0]);
  inv[1][0] = -D2(j[0][1], j[2][2], j[0][2], j[2][1]);
  inv[1][1] = D2(j[0][0], j[2][2], j[0][2], j[2][0]);
  inv[1][2] = -D2(j[0][0], j[2][1], j[0][1], j[2][0]);
  inv[2][0] = D2(j[0][1], j[1][2], j[0][2], j[1][1]);
  inv[2][1] = -D2(j[0][0], j[1][2], j[0][2], j[1][0]);
  inv[2][2] = D2(j[0][0], j[1][1], j[0][1], j[1][0]);
#undef D2
  return J;
}

template <int NDIM>
CFDV_HD CFDV_INLINE void geom_dphi(const double* dPxi, const double (*j)[3], const double (*inv)[3], double iJ,
                                   double* dPhi);

template <>
CFDV_HD CFDV_INLINE void geom_dphi<2>(const double* dPxi, const double (*j)[3], const double (*inv)[3], double iJ,
                                      double* dPhi) {
  (void)inv;
  dPhi[0] = RN_MUL(iJ, RN_SUB(RN_MUL(dPxi[0], j[1][1]), RN_MUL(j[1][0], dPxi[1])));
  dPhi[1] = RN_MUL(iJ, RN_SUB(RN_MUL(j[0][0], dPxi[1]), RN_MUL(dPxi[0], j[0][1])));
}

template <>
CFDV_HD CFDV_INLINE void geom_dphi<3>(const double* dPxi, const double (*j)[3], const double (*inv)[3], double iJ,
                                      double* dPhi) {
  (void)j;
#pragma unroll
  for (int i = 0; i < 3; i++)
    dPhi[i] = RN_ADD(RN_ADD(RN_MUL(iJ, RN_MUL(inv[i][0], dPxi[0])), RN_MUL(iJ, RN_MUL(inv[i][1], dPxi[1]))),
                     RN_MUL(iJ, RN_MUL(inv[i][2], dPxi[2])));
}

// isoparametric Jacobian, physical derivatives dPhi, returns det J; jac[i][j] = dx_i/dxi_j
template <int NDIM, class NP>
CFDV_HD CFDV_INLINE double phys_deriv(const double (*dPxi)[3], const NP* nd, double (*dPhi)[3],
                                      double (*jac)[3]) {
  constexpr int NNOD = (NDIM == 2) ? 4 : 8;
#pragma unroll
  for (int i = 0; i < NDIM; i++)
#pragma unroll
    for (int k = 0; k < NDIM; k++) jac[i][k] = geom_jac_entry<NNOD>(dPxi, nd, i, k);
  double inv[3][3];
  const double J = geom_det<NDIM>(jac, inv);
  const double iJ = RN_DIV(1.0, J);
#pragma unroll
  for (int N = 0; N < NNOD; N++) geom_dphi<NDIM>(dPxi[N], jac, inv, iJ, dPhi[N]);
  return J;
}

// Gauss-point flow state
template <class S>
struct GpStateT {
  S E, T, U[5], dU[5][3], v[3], dV[3][3], dT[3], mu, k, tau[3][3];
};
using GpState = GpStateT<double>;

template <int NDIM, class S>
CFDV_HD CFDV_INLINE void viscous_stress(GpStateT<S>& f) {
  S vkk = 0;
#pragma unroll
  for (int k = 0; k < NDIM; k++) vkk = RN_ADD(vkk, f.dV[k][k]);
#pragma unroll
  for (int i = 0; i < NDIM; i++)
#pragma unroll
    for (int j = 0; j < NDIM; j++) {
      S t = RN_MUL(f.mu, RN_ADD(f.dV[i][j], f.dV[j][i]));
      if (i == j) t = RN_SUB(t, RN_MUL(RN_MUL(2.0 / 3.0, f.mu), vkk));
      f.tau[i][j] = t;
    }
}

// ---- flux Jacobians ---------------------------------------------------------
// jac_a<NDIM>: a(i, ., .) for all i at m[i*25 + r*5 + s]; jac_b_rows<NDIM>: b(i, ., .) for
// one i at m[r*5 + s]; jac_c_rows<NDIM>: c(i, j, ., .) for one i at m[j*25 + r*5 + s].  Each
// has a 2D and a 3D form below, templated on the scalar.

template <class S>
CFDV_HD CFDV_INLINE void jac_a_2d(const GasT<S>& th, const GpStateT<S>& f, S* m) {
  #pragma unroll
  for (int i = 0; i < 2 * 25; i++) m[i] = 0.0;
  const S u = f.v[0], v = f.v[1], uu = u * u, uv = u * v, vv = v * v, E = f.E;
  JA(m, 0, 0, 1) = 1.0;
  JA(m, 0, 1, 0) = th.gm3d2 * uu + th.gm1d2 * vv;
  JA(m, 0, 1, 1) = -th.gamm3 * u;
  JA(m, 0, 1, 2) = -th.gamm1 * v;
  JA(m, 0, 1, 3) = th.gamm1;
  JA(m, 0, 2, 0) = -uv;
  JA(m, 0, 2, 1) = v;
  JA(m, 0, 2, 2) = u;
  JA(m, 0, 3, 0) = -th.gamma * E * u + th.gamm1 * u * (uu + vv);
  JA(m, 0, 3, 1) = th.gamma * E - th.gm1d2 * (3. * uu + vv);
  JA(m, 0, 3, 2) = -th.gamm1 * uv;
  JA(m, 0, 3, 3) = th.gamma * u;
  JA(m, 1, 0, 2) = 1.0;
  JA(m, 1, 1, 0) = -uv;
  JA(m, 1, 1, 1) = v;
  JA(m, 1, 1, 2) = u;
  JA(m, 1, 2, 0) = th.gm1d2 * uu + th.gm3d2 * vv;
  JA(m, 1, 2, 1) = -th.gamm1 * u;
  JA(m, 1, 2, 2) = -th.gamm3 * v;
  JA(m, 1, 2, 3) = th.gamm1;
  JA(m, 1, 3, 0) = -th.gamma * E * v + th.gamm1 * v * (uu + vv);
  JA(m, 1, 3, 1) = -th.gamm1 * uv;
  JA(m, 1, 3, 2) = th.gamma * E - th.gm1d2 * (uu + 3. * vv);
  JA(m, 1, 3, 3) = th.gamma * v;
}

template <class S>
CFDV_HD CFDV_INLINE void jac_b_rows_2d(const GasT<S>& th, const GpStateT<S>& f, int i, S* m) {
  S* blk = m;
  #pragma unroll
  for (int k = 0; k < 25; k++) blk[k] = 0.0;
  const S reinv = 1.0 / th.creyn, mu = f.mu, E = f.E;
  const S lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  const S rho = f.U[0], DENOM = 1. / (rho * rho), TERM1 = f.k * DENOM / th.Cv;
  const S u = f.v[0], v = f.v[1], uu = u * u, vv = v * v;
  const S drdx = f.dU[0][0], dldx = f.dU[1][0], dmdx = f.dU[2][0], dedx = f.dU[3][0];
  const S drdy = f.dU[0][1], dldy = f.dU[1][1], dmdy = f.dU[2][1], dedy = f.dU[3][1];
  const S t00 = f.tau[0][0], t01 = f.tau[0][1], t10 = f.tau[1][0], t11 = f.tau[1][1];
  const S b010 = (DENOM * (mu_R * dldx + lambda * dmdy - 2. * (mu_R * u * drdx + lambda * v * drdy))) * reinv;
  const S b011 = mu_R * drdx * DENOM * reinv, b012 = lambda * drdy * DENOM * reinv;
  const S b020 = (mu * DENOM * (dldy + dmdx - 2. * (u * drdy + v * drdx))) * reinv;
  const S b021 = mu * drdy * DENOM * reinv, b022 = mu * drdx * DENOM * reinv;
  const S b120 = (DENOM * (lambda * (dldx + 4. * v * drdy) + mu_R * (u * drdx + dmdy))) * reinv;
  const S b121 = lambda * drdx * DENOM * reinv, b122 = mu_R * drdy * DENOM * reinv;
  if (i == 0) {
    JA(blk, 0, 1, 0) = b010;
    JA(blk, 0, 1, 1) = b011;
    JA(blk, 0, 1, 2) = b012;
    JA(blk, 0, 2, 0) = b020;
    JA(blk, 0, 2, 1) = b021;
    JA(blk, 0, 2, 2) = b022;
    JA(blk, 0, 3, 0) = u * b010 + v * b020 +
        ((u * t00 + v * t10) / rho -
        TERM1 * (-dedx + (2. * E - 3. * uu - 3. * vv) * drdx + 2. * u * dldx + 2. * v * dmdx)) * reinv;
    JA(blk, 0, 3, 1) = u * b011 + v * b021 + (-t00 / rho - TERM1 * (2. * u * drdx - dldx)) * reinv;
    JA(blk, 0, 3, 2) = u * b012 + v * b022 + (-t10 / rho - TERM1 * (-dmdx + 2. * v * drdx)) * reinv;
    JA(blk, 0, 3, 3) = TERM1 * drdx * reinv;
  } else {
    JA(blk, 0, 1, 0) = b020;
    JA(blk, 0, 1, 1) = b021;
    JA(blk, 0, 1, 2) = b022;
    JA(blk, 0, 2, 0) = b120;
    JA(blk, 0, 2, 1) = b121;
    JA(blk, 0, 2, 2) = b122;
    JA(blk, 0, 3, 0) = u * b020 + v * b120 +
        ((u * t01 + v * t11) / rho -
        TERM1 * (-dedy + (2. * E - 3. * uu - 3. * vv) * drdy + 2. * u * dldy + 2. * v * dmdy)) * reinv;
    JA(blk, 0, 3, 1) = u * b021 + v * b121 + (-t10 / rho - TERM1 * (-dldy + 2. * u * drdy)) * reinv;
    JA(blk, 0, 3, 2) = u * b022 + v * b122 + (-t11 / rho - TERM1 * (2. * v * drdy - dmdy)) * reinv;
    JA(blk, 0, 3, 3) = TERM1 * drdy * reinv;
  }
}

template <class S>
CFDV_HD CFDV_INLINE void jac_c_rows_2d(const GasT<S>& th, const GpStateT<S>& f, int i, S* m) {
  S* blk = m;
  #pragma unroll
  for (int k = 0; k < 75; k++) blk[k] = 0.0;
  const S reinv = 1.0 / th.creyn, mu = f.mu;
  const S lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  const S rho = f.U[0], denom = 1. / (rho * rho), denom2 = denom / rho;
  const S l = f.U[1], mv = f.U[2], re = f.U[3];
  const S ll = l * l, lm = l * mv, mm = mv * mv, rv = ll + mm, hkocv = f.k / th.Cv;
  if (i == 0) {
    JC(blk, 0, 0, 1, 0) = mu_R * l * denom * reinv;
    JC(blk, 0, 0, 1, 1) = -mu_R / rho * reinv;
    JC(blk, 0, 0, 2, 0) = mu * mv * denom * reinv;
    JC(blk, 0, 0, 2, 2) = -mu / rho * reinv;
    JC(blk, 0, 0, 3, 0) = ((mu_R * ll * denom2 + mu * mm * denom2) - hkocv * (-re * denom + rv * denom2)) * reinv;
    JC(blk, 0, 0, 3, 1) = (-mu_R + hkocv) * l * denom * reinv;
    JC(blk, 0, 0, 3, 2) = (-mu + hkocv) * mv * denom * reinv;
    JC(blk, 0, 0, 3, 3) = -hkocv / rho * reinv;
    JC(blk, 0, 1, 1, 0) = lambda * mv * denom * reinv;
    JC(blk, 0, 1, 1, 2) = -lambda / rho * reinv;
    JC(blk, 0, 1, 2, 0) = mu * l * denom * reinv;
    JC(blk, 0, 1, 2, 1) = -mu / rho * reinv;
    JC(blk, 0, 1, 3, 0) = (lambda + mu) * lm * denom2 * reinv;
    JC(blk, 0, 1, 3, 1) = -mu * mv * denom * reinv;
    JC(blk, 0, 1, 3, 2) = -lambda * l * denom * reinv;
  } else {
    JC(blk, 0, 0, 1, 0) = mu * mv * denom * reinv;
    JC(blk, 0, 0, 1, 2) = -mu / rho * reinv;
    JC(blk, 0, 0, 2, 0) = lambda * l * denom * reinv;
    JC(blk, 0, 0, 2, 1) = -lambda / rho * reinv;
    JC(blk, 0, 0, 3, 0) = (mu + lambda) * lm * denom2 * reinv;
    JC(blk, 0, 0, 3, 1) = -lambda * mv * denom * reinv;
    JC(blk, 0, 0, 3, 2) = -mu * l * denom * reinv;
    JC(blk, 0, 1, 1, 0) = mu * l * denom * reinv;
    JC(blk, 0, 1, 1, 1) = -mu / rho * reinv;
    JC(blk, 0, 1, 2, 0) = mu_R * mv * denom * reinv;
    JC(blk, 0, 1, 2, 2) = -mu_R / rho * reinv;
    JC(blk, 0, 1, 3, 0) = ((mu * ll * denom2 + mu_R * mm * denom2) - hkocv * (-re * denom + rv * denom2)) * reinv;
    JC(blk, 0, 1, 3, 1) = (-mu + hkocv) * l * denom * reinv;
    JC(blk, 0, 1, 3, 2) = (-mu_R + hkocv) * mv * denom * reinv;
    JC(blk, 0, 1, 3, 3) = -hkocv / rho * reinv;
  }
}

template <class S>
CFDV_HD CFDV_INLINE void jac_a_3d(const GasT<S>& th, const GpStateT<S>& f, S* m) {
  #pragma unroll
  for (int i = 0; i < 3 * 25; i++) m[i] = 0.0;
  const S gamma = th.gamma, g1 = th.gamm1, g3 = th.gamm3, gm3d2 = th.gm3d2, gm1d2 = th.gm1d2;
  const S u = f.v[0], v = f.v[1], w = f.v[2];
  const S uu = u * u, uv = u * v, vv = v * v, ww = w * w, uw = u * w, vw = v * w, E = f.E;
  const S q2 = uu + vv + ww;
  JA(m, 0, 0, 1) = 1.0;
  JA(m, 0, 1, 0) = gm3d2 * uu + gm1d2 * (vv + ww);
  JA(m, 0, 1, 1) = -g3 * u; JA(m, 0, 1, 2) = -g1 * v; JA(m, 0, 1, 3) = -g1 * w; JA(m, 0, 1, 4) = g1;
  JA(m, 0, 2, 0) = -uv; JA(m, 0, 2, 1) = v; JA(m, 0, 2, 2) = u;
  JA(m, 0, 3, 0) = -uw; JA(m, 0, 3, 1) = w; JA(m, 0, 3, 3) = u;
  JA(m, 0, 4, 0) = -gamma * E * u + g1 * u * q2;
  JA(m, 0, 4, 1) = gamma * E - gm1d2 * (3. * uu + (vv + ww));
  JA(m, 0, 4, 2) = -g1 * uv; JA(m, 0, 4, 3) = -g1 * uw; JA(m, 0, 4, 4) = gamma * u;
  JA(m, 1, 0, 2) = 1.0;
  JA(m, 1, 1, 0) = -uv; JA(m, 1, 1, 1) = v; JA(m, 1, 1, 2) = u;
  JA(m, 1, 2, 0) = gm1d2 * (uu + ww) + gm3d2 * vv;
  JA(m, 1, 2, 1) = -g1 * u; JA(m, 1, 2, 2) = -g3 * v; JA(m, 1, 2, 3) = -g1 * w; JA(m, 1, 2, 4) = g1;
  JA(m, 1, 3, 0) = -vw; JA(m, 1, 3, 2) = w; JA(m, 1, 3, 3) = v;
  JA(m, 1, 4, 0) = -gamma * E * v + g1 * v * q2;
  JA(m, 1, 4, 1) = -g1 * uv;
  JA(m, 1, 4, 2) = gamma * E - gm1d2 * ((uu + ww) + 3. * vv);
  JA(m, 1, 4, 3) = -g1 * vw; JA(m, 1, 4, 4) = gamma * v;
  JA(m, 2, 0, 3) = 1.0;
  JA(m, 2, 1, 0) = -uw; JA(m, 2, 1, 1) = w; JA(m, 2, 1, 3) = u;
  JA(m, 2, 2, 0) = -vw; JA(m, 2, 2, 2) = w; JA(m, 2, 2, 3) = v;
  JA(m, 2, 3, 0) = gm1d2 * (uu + vv) + gm3d2 * ww;
  JA(m, 2, 3, 1) = -g1 * u; JA(m, 2, 3, 2) = -g1 * v; JA(m, 2, 3, 3) = -g3 * w; JA(m, 2, 3, 4) = g1;
  JA(m, 2, 4, 0) = -gamma * E * w + g1 * w * q2;
  JA(m, 2, 4, 1) = -g1 * uw; JA(m, 2, 4, 2) = -g1 * vw;
  JA(m, 2, 4, 3) = gamma * E - gm1d2 * ((uu + vv) + 3. * ww);
  JA(m, 2, 4, 4) = gamma * w;
}

template <class S>
CFDV_HD CFDV_INLINE void jac_b_rows_3d(const GasT<S>& th, const GpStateT<S>& f, int i, S* m) {
  S* blk = m;
  #pragma unroll
  for (int k = 0; k < 25; k++) blk[k] = 0.0;
  const S mu = f.mu, E = f.E;
  const S lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  const S rho = f.U[0], denom = 1. / (rho * rho), TERM1 = f.k * denom / th.Cv;
  const S irho = 1. / rho;  // one division: the entries below multiply by it
  const S u = f.v[0], v = f.v[1], w = f.v[2], uu = u * u, vv = v * v, ww = w * w, q2 = uu + vv + ww;
  const S drdx = f.dU[0][0], dldx = f.dU[1][0], dmdx = f.dU[2][0], dndx = f.dU[3][0], dedx = f.dU[4][0];
  const S drdy = f.dU[0][1], dldy = f.dU[1][1], dmdy = f.dU[2][1], dndy = f.dU[3][1], dedy = f.dU[4][1];
  const S drdz = f.dU[0][2], dldz = f.dU[1][2], dmdz = f.dU[2][2], dndz = f.dU[3][2], dedz = f.dU[4][2];
  const S l = f.U[1], mv = f.U[2], n = f.U[3];
  const auto& t = f.tau;
  // built unscaled, then multiplied by 1/Re (NavierStokes3D.h:331-342)
  const S b010 = (denom * (mu_R * dldx + lambda * (dmdy + dndz) + mu_R * (-2. * u * drdx + v * drdy + w * drdz)));
  const S b011 = mu_R * drdx * denom, b012 = lambda * drdy * denom, b013 = lambda * drdz * denom;
  const S b020 = (mu * denom * (dldy + dmdx - 2. * (u * drdy + v * drdx)));
  const S b021 = mu * drdy * denom, b022 = mu * drdx * denom;
  const S b030 = (mu * denom * (dldz + dndx - 2. * (u * drdz + w * drdx)));
  const S b031 = mu * drdz * denom, b033 = mu * drdx * denom;
  const S b120 = (denom * (lambda * (dldx + dndz) + mu_R * (dmdy + u * drdx - 2. * v * drdy + w * drdz)));
  const S b121 = lambda * drdx * denom, b122 = mu_R * drdy * denom, b123 = lambda * drdz * denom;
  const S b130 = (mu * denom * (dmdz + dndy - 2. * (v * drdz + w * drdy)));
  const S b132 = mu * denom * drdz, b133 = mu * denom * drdy;
  const S b230 = (denom * (mu_R * (dndz + u * drdx + v * drdy - 2. * w * drdz) + lambda * (dldx + dmdy)));
  const S b231 = lambda * drdx * denom, b232 = lambda * drdy * denom, b233 = mu_R * drdz * denom;
  if (i == 0) {
    JA(blk, 0, 1, 0) = b010;
    JA(blk, 0, 1, 1) = b011;
    JA(blk, 0, 1, 2) = b012;
    JA(blk, 0, 1, 3) = b013;
    JA(blk, 0, 2, 0) = b020;
    JA(blk, 0, 2, 1) = b021;
    JA(blk, 0, 2, 2) = b022;
    JA(blk, 0, 3, 0) = b030;
    JA(blk, 0, 3, 1) = b031;
    JA(blk, 0, 3, 3) = b033;
    JA(blk, 0, 4, 0) = u * b010 + v * b020 + w * b030 +
        (denom * (l * t[0][0] + mv * t[0][1] + n * t[0][2]) -
        TERM1 * (-dedx + (2. * E - 3. * q2) * drdx + 2. * (u * dldx + v * dmdx + w * dndx)));
    JA(blk, 0, 4, 1) = u * b011 + v * b021 + w * b031 + (-t[0][0] * irho - TERM1 * (2. * u * drdx - dldx));
    JA(blk, 0, 4, 2) = u * b012 + v * b022 + w * 0.0 + (-t[0][1] * irho - TERM1 * (-dmdx + 2. * v * drdx));
    JA(blk, 0, 4, 3) = u * b013 + v * 0.0 + w * b033 + (-t[0][2] * irho - TERM1 * (2 * w * drdx - dndx));
    JA(blk, 0, 4, 4) = TERM1 * drdx;
  } else if (i == 1) {
    JA(blk, 0, 1, 0) = b020;
    JA(blk, 0, 1, 1) = b021;
    JA(blk, 0, 1, 2) = b022;
    JA(blk, 0, 2, 0) = b120;
    JA(blk, 0, 2, 1) = b121;
    JA(blk, 0, 2, 2) = b122;
    JA(blk, 0, 2, 3) = b123;
    JA(blk, 0, 3, 0) = b130;
    JA(blk, 0, 3, 2) = b132;
    JA(blk, 0, 3, 3) = b133;
    JA(blk, 0, 4, 0) = u * b020 + v * b120 + w * b130 +
        (denom * (l * t[1][0] + mv * t[1][1] + n * t[1][2]) -
        TERM1 * (-dedy + (2. * E - 3. * q2) * drdy + 2. * (u * dldy + v * dmdy + w * dndy)));
    JA(blk, 0, 4, 1) = u * b021 + v * b121 + w * 0.0 + (-t[1][0] * irho - TERM1 * (-dldy + 2. * u * drdy));
    JA(blk, 0, 4, 2) = u * b022 + v * b122 + w * b132 + (-t[1][1] * irho - TERM1 * (2. * v * drdy - dmdy));
    JA(blk, 0, 4, 3) = u * 0.0 + v * b123 + w * b133 + (-t[1][2] * irho - TERM1 * (2. * w * drdy - dndy));
    JA(blk, 0, 4, 4) = TERM1 * drdy;
  } else {
    JA(blk, 0, 1, 0) = b030;
    JA(blk, 0, 1, 1) = b031;
    JA(blk, 0, 1, 3) = b033;
    JA(blk, 0, 2, 0) = b130;
    JA(blk, 0, 2, 2) = b132;
    JA(blk, 0, 2, 3) = b133;
    JA(blk, 0, 3, 0) = b230;
    JA(blk, 0, 3, 1) = b231;
    JA(blk, 0, 3, 2) = b232;
    JA(blk, 0, 3, 3) = b233;
    JA(blk, 0, 4, 0) = u * b030 + v * b130 + w * b230 +
        (denom * (l * t[2][0] + mv * t[2][1] + n * t[2][2]) -
        TERM1 * (-dedz + (2. * E - 3. * q2) * drdz + 2. * (u * dldz + v * dmdz + w * dndz)));
    JA(blk, 0, 4, 1) = u * b031 + v * 0.0 + w * b231 + (-t[2][0] * irho - TERM1 * (2. * u * drdz - dldz));
    JA(blk, 0, 4, 2) = u * 0.0 + v * b132 + w * b232 + (-t[2][1] * irho - TERM1 * (2. * v * drdz - dmdz));
    JA(blk, 0, 4, 3) = u * b033 + v * b133 + w * b233 + (-t[2][2] * irho - TERM1 * (2. * w * drdz - dndz));
    JA(blk, 0, 4, 4) = TERM1 * drdz;
  }
  const S reinv = 1.0 / th.creyn;
  #pragma unroll
  for (int k = 0; k < 25; k++) blk[k] *= reinv;
}

template <class S>
CFDV_HD CFDV_INLINE void jac_c_rows_3d(const GasT<S>& th, const GpStateT<S>& f, int i, S* m) {
  S* blk = m;
  #pragma unroll
  for (int k = 0; k < 75; k++) blk[k] = 0.0;
  const S mu = f.mu, lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  const S rho = f.U[0], denom = 1. / (rho * rho);
  const S irho = 1. / rho;  // one division: the entries below multiply by it
  const S l = f.U[1], mv = f.U[2], n = f.U[3], re = f.U[4];
  const S ll = l * l, mm = mv * mv, nn = n * n, hkocv = f.k / th.Cv, TERM1 = f.k / th.Cv * denom;
  const S q = (-re + (ll + mm + nn) * irho);
  if (i == 0) {
    const S d10[3] = {mu_R * l * denom, mu * mv * denom, mu * n * denom};    // JC(0,0,1..3,0)
    JC(blk, 0, 0, 1, 0) = mu_R * l * denom;
    JC(blk, 0, 0, 1, 1) = (-mu_R * irho);
    JC(blk, 0, 0, 2, 0) = mu * mv * denom;
    JC(blk, 0, 0, 2, 2) = (-mu * irho);
    JC(blk, 0, 0, 3, 0) = mu * n * denom;
    JC(blk, 0, 0, 3, 3) = (-mu * irho);
    JC(blk, 0, 0, 4, 0) = (l * d10[0] + mv * d10[1] + n * d10[2]) * irho - TERM1 * q;
    JC(blk, 0, 0, 4, 1) = (l * irho) * (-mu_R * irho) + TERM1 * l;
    JC(blk, 0, 0, 4, 2) = (mv * irho) * (-mu * irho) + TERM1 * mv;
    JC(blk, 0, 0, 4, 3) = (n * irho) * (-mu * irho) + TERM1 * n;
    JC(blk, 0, 0, 4, 4) = (-hkocv * irho);
    JC(blk, 0, 1, 1, 0) = lambda * mv * denom;
    JC(blk, 0, 1, 1, 2) = (-lambda * irho);
    JC(blk, 0, 1, 2, 0) = mu * l * denom;
    JC(blk, 0, 1, 2, 1) = (-mu * irho);
    JC(blk, 0, 1, 4, 0) = (l * irho) * (lambda * mv * denom) + (mv * irho) * (mu * l * denom);
    JC(blk, 0, 1, 4, 1) = (mv * irho) * (-mu * irho);
    JC(blk, 0, 1, 4, 2) = (l * irho) * (-lambda * irho);
    JC(blk, 0, 2, 1, 0) = lambda * n * denom;
    JC(blk, 0, 2, 1, 3) = (-lambda * irho);
    JC(blk, 0, 2, 3, 0) = mu * l * denom;
    JC(blk, 0, 2, 3, 1) = (-mu * irho);
    JC(blk, 0, 2, 4, 0) = (l * irho) * (lambda * n * denom) + (n * irho) * (mu * l * denom);
    JC(blk, 0, 2, 4, 1) = (n * irho) * (-mu * irho);
    JC(blk, 0, 2, 4, 3) = (l * irho) * (-lambda * irho);
  } else if (i == 1) {
    const S e10 = mu * l * denom, e20 = mu_R * mv * denom, e30 = mu * n * denom;  // JC(1,1,1..3,0)
    JC(blk, 0, 1, 1, 0) = e10;
    JC(blk, 0, 1, 1, 1) = (-mu * irho);
    JC(blk, 0, 1, 2, 0) = e20;
    JC(blk, 0, 1, 2, 2) = (-mu_R * irho);
    JC(blk, 0, 1, 3, 0) = e30;
    JC(blk, 0, 1, 3, 3) = (-mu * irho);
    JC(blk, 0, 1, 4, 0) = (l * e10 + mv * e20 + n * e30) * irho - TERM1 * q;
    JC(blk, 0, 1, 4, 1) = (l * irho) * (-mu * irho) + TERM1 * l;
    JC(blk, 0, 1, 4, 2) = (mv * irho) * (-mu_R * irho) + TERM1 * mv;
    JC(blk, 0, 1, 4, 3) = (n * irho) * (-mu * irho) + TERM1 * n;
    JC(blk, 0, 1, 4, 4) = (-hkocv * irho);
    JC(blk, 0, 0, 1, 0) = mu * mv * denom;
    JC(blk, 0, 0, 1, 2) = (-mu * irho);
    JC(blk, 0, 0, 2, 0) = lambda * l * denom;
    JC(blk, 0, 0, 2, 1) = (-lambda * irho);
    JC(blk, 0, 0, 4, 0) = (l * irho) * (mu * mv * denom) + (mv * irho) * (lambda * l * denom);
    JC(blk, 0, 0, 4, 1) = (mv * irho) * (-lambda * irho);
    JC(blk, 0, 0, 4, 2) = (l * irho) * (-mu * irho);
    JC(blk, 0, 2, 2, 0) = lambda * n * denom;
    JC(blk, 0, 2, 2, 3) = (-lambda * irho);
    JC(blk, 0, 2, 3, 0) = mu * mv * denom;
    JC(blk, 0, 2, 3, 2) = (-mu * irho);
    JC(blk, 0, 2, 4, 0) = (mv * irho) * (lambda * n * denom) + (n * irho) * (mu * mv * denom);
    JC(blk, 0, 2, 4, 2) = (n * irho) * (-mu * irho);
    JC(blk, 0, 2, 4, 3) = (mv * irho) * (-lambda * irho);
  } else {
    const S f10 = mu * l * denom, f20 = mu * mv * denom, f30 = mu_R * n * denom;  // JC(2,2,1..3,0)
    JC(blk, 0, 2, 1, 0) = f10;
    JC(blk, 0, 2, 1, 1) = (-mu * irho);
    JC(blk, 0, 2, 2, 0) = f20;
    JC(blk, 0, 2, 2, 2) = (-mu * irho);
    JC(blk, 0, 2, 3, 0) = f30;
    JC(blk, 0, 2, 3, 3) = (-mu_R * irho);
    JC(blk, 0, 2, 4, 0) = (l * f10 + mv * f20 + n * f30) * irho - TERM1 * q;
    JC(blk, 0, 2, 4, 1) = (l * irho) * (-mu * irho) + TERM1 * l;
    JC(blk, 0, 2, 4, 2) = (mv * irho) * (-mu * irho) + TERM1 * mv;
    JC(blk, 0, 2, 4, 3) = (n * irho) * (-mu_R * irho) + TERM1 * n;
    JC(blk, 0, 2, 4, 4) = (-hkocv * irho);
    JC(blk, 0, 0, 1, 0) = mu * n * denom;
    JC(blk, 0, 0, 1, 3) = (-mu * irho);
    JC(blk, 0, 0, 3, 0) = lambda * l * denom;
    JC(blk, 0, 0, 3, 1) = (-lambda * irho);
    JC(blk, 0, 0, 4, 0) = (l * irho) * (mu * n * denom) + (n * irho) * (lambda * l * denom);
    JC(blk, 0, 0, 4, 1) = (n * irho) * (-lambda * irho);
    JC(blk, 0, 0, 4, 3) = (l * irho) * (-mu * irho);
    JC(blk, 0, 1, 2, 0) = mu * n * denom;
    JC(blk, 0, 1, 2, 3) = (-mu * irho);
    JC(blk, 0, 1, 3, 0) = lambda * mv * denom;
    JC(blk, 0, 1, 3, 2) = (-lambda * irho);
    JC(blk, 0, 1, 4, 0) = (mv * irho) * (mu * n * denom) + (n * irho) * (lambda * mv * denom);
    JC(blk, 0, 1, 4, 2) = (n * irho) * (-lambda * irho);
    JC(blk, 0, 1, 4, 3) = (mv * irho) * (-mu * irho);
  }
  const S reinv = 1.0 / th.creyn;
  #pragma unroll
  for (int k = 0; k < 75; k++) blk[k] *= reinv;
}

template <int NDIM, class S>
CFDV_HD CFDV_INLINE void jac_a(const GasT<S>& th, const GpStateT<S>& f, S* m) {
  if constexpr (NDIM == 2) jac_a_2d(th, f, m);
  else jac_a_3d(th, f, m);
}
template <int NDIM, class S>
CFDV_HD CFDV_INLINE void jac_b_rows(const GasT<S>& th, const GpStateT<S>& f, int i, S* m) {
  if constexpr (NDIM == 2) jac_b_rows_2d(th, f, i, m);
  else jac_b_rows_3d(th, f, i, m);
}
template <int NDIM, class S>
CFDV_HD CFDV_INLINE void jac_c_rows(const GasT<S>& th, const GpStateT<S>& f, int i, S* m) {
  if constexpr (NDIM == 2) jac_c_rows_2d(th, f, i, m);
  else jac_c_rows_3d(th, f, i, m);
}

// Convective flux of one node, entry (i, r): F(i,r) from the node's U and p alone.
template <int NDIM, class S>
CFDV_HD CFDV_INLINE S node_conv_flux_entry(const NodePrimT<S>& n, int i, int r) {
  S F = 0.0;
  if (NDIM == 2) {
    const S rho = n.U[0], l = n.U[1], m = n.U[2], e = n.U[3], p = n.p;
    const S li = (i == 0) ? l : m;
    if (r == 0) F = li;
    else if (r == 1) F = (i == 0) ? p + l * l / rho : (l * m) / rho;
    else if (r == 2) F = (i == 0) ? (l * m) / rho : p + m * m / rho;
    else F = (p + e) * (li / rho);
  } else {
    const S rho = n.U[0], p = n.p;
    const S vi = n.U[1 + i] / n.U[0];
    if (r == 0) {
      F = rho * vi;
    } else if (r <= 3) {
      const S vj = n.U[r] / n.U[0];
      F = rho * vi * vj + (i == r - 1 ? p : 0.0);
    } else {
      const S E = n.U[4] / n.U[0];
      F = (rho * E + p) * vi;
    }
  }
  return F;
}

// Convective + viscous flux of one node, entry (i, r): F(i,r) + G(i,r).  F is the node's own
// flux; G uses the Gauss-point stress, dT and k with the node velocity.  with_F = 0 drops F
// (the 3D reference evaluates the empty base-class flux).  r may be a run-time index:
// nothing here is an array in registers or local memory.
template <int NDIM, class S>
CFDV_HD CFDV_INLINE S node_flux_entry(const GpStateT<S>& f, const NodePrimT<S>& n, double Re, bool with_F, int i,
                                      int r) {
  const S reinv = 1.0 / Re;
  S G = 0.0;
  if (r >= 1 && r <= NDIM) {
    G = -f.tau[i][r - 1] * reinv;
  } else if (r == NDIM + 1) {
    S s = -f.tau[i][0] * n.v[0];
#pragma unroll
    for (int j = 1; j < NDIM; j++) s = s - f.tau[i][j] * n.v[j];
    G = (s - f.k * f.dT[i]) * reinv;
  }
  const S F = with_F ? node_conv_flux_entry<NDIM>(n, i, r) : S(0.0);
  return F + G;
}

}  // namespace cfdv
