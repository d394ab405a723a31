// CPU restatement of the CFDV per-step FDV path -- TEST INFRASTRUCTURE ONLY.
//
// The parity tests, smoke() and the CPU-baseline leg of bench.py use this as the
// checker for the CUDA path; the product library never links or loads it.  Each
// routine restates the reference routine named beside it (paths relative to the
// CFDV source tree) and keeps the reference's accumulation order, so that on the
// same inputs it agrees with the reference build (oracle/_ref) to rounding.
#include "cfdv_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

// Thermo.h:8-86 (nondimensional gas model)
struct Gas {
  double gamma, gamm1, gm1d2, gamm3, gm3d2, Pr, csuth, Cv, cgas, cmach, creyn, Twall;
  bool adiabatic;
  explicit Gas(const oracle_aero* a) {
    gamma = a->gamma;
    gamm1 = gamma - 1.0;
    gm1d2 = (gamma - 1.0) / 2.0;
    gamm3 = gamma - 3.0;
    gm3d2 = (gamma - 3.0) / 2.0;
    Pr = a->prandtl;
    csuth = 110.0 / a->tinf;
    cmach = a->mach;
    Cv = 1. / gamma / (gamma - 1.0) / std::pow(a->mach, 2);
    cgas = 1.0 / gamma / std::pow(a->mach, 2);
    creyn = a->reynolds;
    Twall = a->twall;
    adiabatic = a->adiabatic != 0;
  }
  double mu(double T) const {  // Thermo.h:53-70
    if (T < 1.0E-12) return 1.0;
    return ((1 + csuth) / (T + csuth)) * T * std::sqrt(T);
  }
  double k(double mu) const { return mu / ((gamma - 1.0) * (cmach * cmach) * Pr); }  // Thermo.h:72-75
};

// NodeUnpack.h:9-29: primitives from the conserved vector
struct NodeState {
  double x[3], U[5], v[3];
  double rho, E, e, T, p;
};

void unpack(const Gas& g, int ndim, const double* U, const double* x, NodeState& n) {
  for (int k = 0; k < ndim + 2; k++) n.U[k] = U[k];
  for (int k = 0; k < ndim; k++) n.x[k] = x[k];
  n.rho = U[0];
  double vsqr = 0;
  for (int i = 0; i < ndim; i++) {
    n.v[i] = U[1 + i] / U[0];
    vsqr += n.v[i] * n.v[i];
  }
  n.E = U[ndim + 1] / U[0];
  n.e = n.E - 0.5 * vsqr;
  n.T = n.e / g.Cv;
  n.p = n.rho * (g.gamma - 1.0) * n.e;
}

// GaussQuad.h:116-159: Newton iteration on the Legendre polynomial
void gauss(int N, double* zeta, double* w) {
  const double x1 = -1.0, x2 = 1.0, eps = 3.E-14;
  double m = (N + 1) / 2;
  double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
  double p[4] = {0, 0, 0, 0};
  for (int i = 1; i <= m; i++) {
    double z = std::cos(3.141592654 * (i - 0.25) / (N + 0.5));
    double z1 = z + 10;
    p[0] = 0;
    while (std::abs(z - z1) > eps) {
      p[1] = 1.0;
      p[2] = 0.0;
      for (int j = 1; j <= N; j++) {
        p[3] = p[2];
        p[2] = p[1];
        p[1] = ((2.0 * j - 1.0) * z * p[2] - (j - 1.) * p[3]) / j;
      }
      p[0] = N * (z * p[1] - p[2]) / (z * z - 1.0);
      z1 = z;
      z = z1 - p[1] / p[0];
    }
    zeta[i - 1] = xm - xl * z;
    zeta[N - i] = xm + xl * z;
    w[i - 1] = 2.0 * xl / ((1.0 - z * z) * p[0] * p[0]);
    w[N - i] = w[i - 1];
  }
  for (int i = 0; i < N; i++) {
    if (std::abs(zeta[i]) < eps) zeta[i] = 0.0;
    if (std::abs(w[i]) < eps) w[i] = 0.0;
  }
}

// ---- shape functions ------------------------------------------------------
// TestFunctions2D.h:7-43
void shape2(const double* z, double* Phi, double dPxi[][3]) {
  Phi[0] = 0.25 * (1 - z[0]) * (1 - z[1]);
  Phi[1] = 0.25 * (1 + z[0]) * (1 - z[1]);
  Phi[2] = 0.25 * (1 + z[0]) * (1 + z[1]);
  Phi[3] = 0.25 * (1 - z[0]) * (1 + z[1]);
  dPxi[0][0] = -0.25 * (1 - z[1]);
  dPxi[1][0] = 0.25 * (1 - z[1]);
  dPxi[2][0] = 0.25 * (1 + z[1]);
  dPxi[3][0] = -0.25 * (1 + z[1]);
  dPxi[0][1] = -0.25 * (1 - z[0]);
  dPxi[1][1] = -0.25 * (1 + z[0]);
  dPxi[2][1] = 0.25 * (1 + z[0]);
  dPxi[3][1] = 0.25 * (1 - z[0]);
}

// TestFunctions3D.h:7-56
void shape3(const double* z, double* Phi, double dPxi[][3]) {
  const double a0 = 1 - z[0], b0 = 1 + z[0], a1 = 1 - z[1], b1 = 1 + z[1], a2 = 1 - z[2], b2 = 1 + z[2];
  Phi[0] = 0.125 * a0 * a1 * a2;
  Phi[1] = 0.125 * b0 * a1 * a2;
  Phi[2] = 0.125 * b0 * b1 * a2;
  Phi[3] = 0.125 * a0 * b1 * a2;
  Phi[4] = 0.125 * a0 * a1 * b2;
  Phi[5] = 0.125 * b0 * a1 * b2;
  Phi[6] = 0.125 * b0 * b1 * b2;
  Phi[7] = 0.125 * a0 * b1 * b2;
  const double s0[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  const double s1[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  const double s2[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int N = 0; N < 8; N++) {
    double f0 = s1[N] < 0 ? a1 : b1, g0 = s2[N] < 0 ? a2 : b2;
    double f1 = s0[N] < 0 ? a0 : b0;
    dPxi[N][0] = s0[N] * 0.125 * f0 * g0;
    dPxi[N][1] = s1[N] * 0.125 * f1 * g0;
    dPxi[N][2] = s2[N] * 0.125 * f1 * f0;
  }
}

// TestFunctions2D.h:46-90 (jacobian, dtestfunctiondx)
double jac2(const double dPxi[][3], NodeState* const* nd, double jac[3][3], double dPhi[][3]) {
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) jac[i][j] = 0;
  for (int N = 0; N < 4; N++)
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) jac[i][j] += dPxi[N][j] * nd[N]->x[i];
  double J = (jac[0][0] * jac[1][1] - jac[1][0] * jac[0][1]);
  double dxdxi = jac[0][0], dxdeta = jac[0][1], dydeta = jac[1][1], dydxi = jac[1][0];
  for (int N = 0; N < 4; N++) {
    dPhi[N][0] = (1.0 / J) * (dPxi[N][0] * dydeta - dydxi * dPxi[N][1]);
    dPhi[N][1] = (1.0 / J) * (dxdxi * dPxi[N][1] - dPxi[N][0] * dxdeta);
  }
  return J;
}

// TestFunctions3D.h:58-123 (jacobian3d, dtestfunctiondx3d)
double jac3(const double dPxi[][3], NodeState* const* nd, double dPhi[][3]) {
  double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int N = 0; N < 8; N++)
    for (int i = 0; i < 3; i++)
      for (int k = 0; k < 3; k++) j[i][k] += dPxi[N][k] * nd[N]->x[i];
  double J = j[0][0] * j[1][1] * j[2][2] + j[0][1] * j[1][2] * j[2][0] + j[0][2] * j[1][0] * j[2][1] -
             j[0][2] * j[1][1] * j[2][0] - j[0][1] * j[1][0] * j[2][2] - j[0][0] * j[1][2] * j[2][1];
  double inv[3][3];
  inv[0][0] = j[1][1] * j[2][2] - j[1][2] * j[2][1];
  inv[0][1] = -(j[1][0] * j[2][2] - j[1][2] * j[2][0]);
  inv[0][2] = j[1][0] * j[2][1] - j[1][1] * j[2][0];
  inv[1][0] = -(j[0][1] * j[2][2] - j[0][2] * j[2][1]);
  inv[1][1] = j[0][0] * j[2][2] - j[0][2] * j[2][0];
  inv[1][2] = -(j[0][0] * j[2][1] - j[0][1] * j[2][0]);
  inv[2][0] = j[0][1] * j[1][2] - j[0][2] * j[1][1];
  inv[2][1] = -(j[0][0] * j[1][2] - j[0][2] * j[1][0]);
  inv[2][2] = j[0][0] * j[1][1] - j[0][1] * j[1][0];
  for (int N = 0; N < 8; N++)
    for (int i = 0; i < 3; i++) dPhi[N][i] = 0;
  for (int i = 0; i < 3; i++)
    for (int N = 0; N < 8; N++)
      for (int k = 0; k < 3; k++) dPhi[N][i] += (1.0 / J) * (inv[i][k] * dPxi[N][k]);
  return J;
}

// ---- Gauss-point flow state (Flow.h, FDVGalerkin.h:761-797, tau.h:14-42) ---
struct FlowPt {
  double E, T, v[3], x[3], U[5], dU[5][3], dV[3][3], dT[3], k, mu, tau[3][3];
};

void gp_sum(const Gas& g, int ndim, int neqn, int nn, NodeState* const* nd, const double* Phi,
            const double dPhi[][3], FlowPt& f) {
  std::memset(&f, 0, sizeof(f));
  for (int N = 0; N < nn; N++) {
    f.E += Phi[N] * nd[N]->E;
    f.T += Phi[N] * nd[N]->T;
    for (int i = 0; i < neqn; i++) {
      f.U[i] += Phi[N] * nd[N]->U[i];
      for (int j = 0; j < ndim; j++) f.dU[i][j] += dPhi[N][j] * nd[N]->U[i];
    }
    for (int i = 0; i < ndim; i++) {
      f.x[i] += Phi[N] * nd[N]->x[i];
      f.v[i] += Phi[N] * nd[N]->v[i];
      f.dT[i] += dPhi[N][i] * nd[N]->T;
      for (int d = 0; d < ndim; d++) f.dV[i][d] += dPhi[N][d] * nd[N]->v[i];
    }
  }
  f.mu = g.mu(f.T);
  f.k = g.k(f.mu);
}

void tau_calc(int ndim, FlowPt& f) {  // tau.h:14-42
  double vkk = 0;
  for (int k = 0; k < ndim; k++) vkk += f.dV[k][k];
  for (int i = 0; i < ndim; i++)
    for (int j = 0; j < ndim; j++) {
      f.tau[i][j] = f.mu * (f.dV[i][j] + f.dV[j][i]);
      if (i == j) f.tau[i][j] -= (2.0 / 3.0) * f.mu * vkk;
    }
}

// ---- flux Jacobians: a = dF/dU, b = dG/dU, c = dG/dU_,j -------------------
// Index helpers: A(i,r,s) -> a[(i*5+r)*5+s]; C(i,j,r,s) -> c[((i*3+j)*5+r)*5+s]
#define A3(t, i, r, s) t[((i)*5 + (r)) * 5 + (s)]
#define C4(t, i, j, r, s) t[(((i)*3 + (j)) * 5 + (r)) * 5 + (s)]

void calc_a2(const Gas& th, const FlowPt& f, double* m) {  // NavierStokes2D.h:59-97
  std::fill(m, m + 75, 0.0);
  double u = f.v[0], v = f.v[1], uu = u * u, uv = u * v, vv = v * v, E = f.E;
  A3(m, 0, 0, 1) = 1.0;
  A3(m, 0, 1, 0) = th.gm3d2 * uu + th.gm1d2 * vv;
  A3(m, 0, 1, 1) = -th.gamm3 * u;
  A3(m, 0, 1, 2) = -th.gamm1 * v;
  A3(m, 0, 1, 3) = th.gamm1;
  A3(m, 0, 2, 0) = -uv;
  A3(m, 0, 2, 1) = v;
  A3(m, 0, 2, 2) = u;
  A3(m, 0, 3, 0) = -th.gamma * E * u + th.gamm1 * u * (uu + vv);
  A3(m, 0, 3, 1) = th.gamma * E - th.gm1d2 * (3. * uu + vv);
  A3(m, 0, 3, 2) = -th.gamm1 * uv;
  A3(m, 0, 3, 3) = th.gamma * u;
  A3(m, 1, 0, 2) = 1.0;
  A3(m, 1, 1, 0) = -uv;
  A3(m, 1, 1, 1) = v;
  A3(m, 1, 1, 2) = u;
  A3(m, 1, 2, 0) = th.gm1d2 * uu + th.gm3d2 * vv;
  A3(m, 1, 2, 1) = -th.gamm1 * u;
  A3(m, 1, 2, 2) = -th.gamm3 * v;
  A3(m, 1, 2, 3) = th.gamm1;
  A3(m, 1, 3, 0) = -th.gamma * E * v + th.gamm1 * v * (uu + vv);
  A3(m, 1, 3, 1) = -th.gamm1 * uv;
  A3(m, 1, 3, 2) = th.gamma * E - th.gm1d2 * (uu + 3. * vv);
  A3(m, 1, 3, 3) = th.gamma * v;
}

void calc_b2(const Gas& th, const FlowPt& f, double* m) {  // NavierStokes2D.h:100-158
  std::fill(m, m + 75, 0.0);
  double reinv = 1.0 / th.creyn, mu = f.mu, E = f.E;
  double lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  double DENOM = 1. / std::pow(f.U[0], 2), TERM1 = f.k * DENOM / th.Cv;
  double rho = f.U[0], u = f.v[0], v = f.v[1], uu = u * u, vv = v * v;
  double drdx = f.dU[0][0], dldx = f.dU[1][0], dmdx = f.dU[2][0], dedx = f.dU[3][0];
  double drdy = f.dU[0][1], dldy = f.dU[1][1], dmdy = f.dU[2][1], dedy = f.dU[3][1];
  auto& t = f.tau;
  A3(m, 0, 1, 0) = (DENOM * (mu_R * dldx + lambda * dmdy - 2. * (mu_R * u * drdx + lambda * v * drdy))) * reinv;
  A3(m, 0, 1, 1) = mu_R * drdx * DENOM * reinv;
  A3(m, 0, 1, 2) = lambda * drdy * DENOM * reinv;
  A3(m, 0, 2, 0) = (mu * DENOM * (dldy + dmdx - 2. * (u * drdy + v * drdx))) * reinv;
  A3(m, 0, 2, 1) = mu * drdy * DENOM * reinv;
  A3(m, 0, 2, 2) = mu * drdx * DENOM * reinv;
  A3(m, 0, 3, 0) = u * A3(m, 0, 1, 0) + v * A3(m, 0, 2, 0) +
                   ((u * t[0][0] + v * t[1][0]) / rho -
                    TERM1 * (-dedx + (2. * E - 3. * uu - 3. * vv) * drdx + 2. * u * dldx + 2. * v * dmdx)) * reinv;
  A3(m, 0, 3, 1) = u * A3(m, 0, 1, 1) + v * A3(m, 0, 2, 1) + (-t[0][0] / rho - TERM1 * (2. * u * drdx - dldx)) * reinv;
  A3(m, 0, 3, 2) = u * A3(m, 0, 1, 2) + v * A3(m, 0, 2, 2) + (-t[1][0] / rho - TERM1 * (-dmdx + 2. * v * drdx)) * reinv;
  A3(m, 0, 3, 3) = TERM1 * drdx * reinv;
  A3(m, 1, 1, 0) = A3(m, 0, 2, 0);
  A3(m, 1, 1, 1) = A3(m, 0, 2, 1);
  A3(m, 1, 1, 2) = A3(m, 0, 2, 2);
  A3(m, 1, 2, 0) = (DENOM * (lambda * (dldx + 4. * v * drdy) + mu_R * (u * drdx + dmdy))) * reinv;
  A3(m, 1, 2, 1) = lambda * drdx * DENOM * reinv;
  A3(m, 1, 2, 2) = mu_R * drdy * DENOM * reinv;
  A3(m, 1, 3, 0) = u * A3(m, 1, 1, 0) + v * A3(m, 1, 2, 0) +
                   ((u * t[0][1] + v * t[1][1]) / rho -
                    TERM1 * (-dedy + (2. * E - 3. * uu - 3. * vv) * drdy + 2. * u * dldy + 2. * v * dmdy)) * reinv;
  A3(m, 1, 3, 1) = u * A3(m, 1, 1, 1) + v * A3(m, 1, 2, 1) + (-t[1][0] / rho - TERM1 * (-dldy + 2. * u * drdy)) * reinv;
  A3(m, 1, 3, 2) = u * A3(m, 1, 1, 2) + v * A3(m, 1, 2, 2) + (-t[1][1] / rho - TERM1 * (2. * v * drdy - dmdy)) * reinv;
  A3(m, 1, 3, 3) = TERM1 * drdy * reinv;
}

void calc_c2(const Gas& th, const FlowPt& f, double* m) {  // NavierStokes2D.h:163-222
  std::fill(m, m + 225, 0.0);
  double reinv = 1.0 / th.creyn, mu = f.mu;
  double lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  double rho = f.U[0], denom = 1. / std::pow(rho, 2), denom2 = denom / rho;
  double l = f.U[1], mm_ = f.U[2], re = f.U[3];
  double ll = l * l, lm = l * mm_, mm = mm_ * mm_, rv11p22 = ll + mm, hkocv = f.k / th.Cv;
  C4(m, 0, 0, 1, 0) = mu_R * l * denom * reinv;
  C4(m, 0, 0, 1, 1) = -mu_R / rho * reinv;
  C4(m, 0, 0, 2, 0) = mu * mm_ * denom * reinv;
  C4(m, 0, 0, 2, 2) = -mu / rho * reinv;
  C4(m, 0, 0, 3, 0) = ((mu_R * ll * denom2 + mu * mm * denom2) - hkocv * (-re * denom + (rv11p22)*denom2)) * reinv;
  C4(m, 0, 0, 3, 1) = (-mu_R + hkocv) * l * denom * reinv;
  C4(m, 0, 0, 3, 2) = (-mu + hkocv) * mm_ * denom * reinv;
  C4(m, 0, 0, 3, 3) = -hkocv / rho * reinv;
  C4(m, 0, 1, 1, 0) = lambda * mm_ * denom * reinv;
  C4(m, 0, 1, 1, 2) = -lambda / rho * reinv;
  C4(m, 0, 1, 2, 0) = mu * l * denom * reinv;
  C4(m, 0, 1, 2, 1) = -mu / rho * reinv;
  C4(m, 0, 1, 3, 0) = (lambda + mu) * lm * denom2 * reinv;
  C4(m, 0, 1, 3, 1) = -mu * mm_ * denom * reinv;
  C4(m, 0, 1, 3, 2) = -lambda * l * denom * reinv;
  C4(m, 1, 0, 1, 0) = mu * mm_ * denom * reinv;
  C4(m, 1, 0, 1, 2) = -mu / rho * reinv;
  C4(m, 1, 0, 2, 0) = lambda * l * denom * reinv;
  C4(m, 1, 0, 2, 1) = -lambda / rho * reinv;
  C4(m, 1, 0, 3, 0) = (mu + lambda) * lm * denom2 * reinv;
  C4(m, 1, 0, 3, 1) = -lambda * mm_ * denom * reinv;
  C4(m, 1, 0, 3, 2) = -mu * l * denom * reinv;
  C4(m, 1, 1, 1, 0) = mu * l * denom * reinv;
  C4(m, 1, 1, 1, 1) = -mu / rho * reinv;
  C4(m, 1, 1, 2, 0) = mu_R * mm_ * denom * reinv;
  C4(m, 1, 1, 2, 2) = -mu_R / rho * reinv;
  C4(m, 1, 1, 3, 0) = ((mu * ll * denom2 + mu_R * mm * denom2) - hkocv * (-re * denom + rv11p22 * denom2)) * reinv;
  C4(m, 1, 1, 3, 1) = (-mu + hkocv) * l * denom * reinv;
  C4(m, 1, 1, 3, 2) = (-mu_R + hkocv) * mm_ * denom * reinv;
  C4(m, 1, 1, 3, 3) = -hkocv / rho * reinv;
}

void calc_a3(const Gas& th, const FlowPt& f, double* m) {  // NavierStokes3D.h:74-189
  std::fill(m, m + 75, 0.0);
  double gamma = th.gamma, g1 = th.gamm1, g3 = th.gamm3, gm3d2 = th.gm3d2, gm1d2 = th.gm1d2;
  double u = f.v[0], v = f.v[1], w = f.v[2];
  double uu = u * u, uv = u * v, vv = v * v, ww = w * w, uw = u * w, vw = v * w, E = f.E;
  A3(m, 0, 0, 1) = 1.0;
  A3(m, 0, 1, 0) = gm3d2 * uu + gm1d2 * (vv + ww);
  A3(m, 0, 1, 1) = -g3 * u;
  A3(m, 0, 1, 2) = -g1 * v;
  A3(m, 0, 1, 3) = -g1 * w;
  A3(m, 0, 1, 4) = g1;
  A3(m, 0, 2, 0) = -uv;
  A3(m, 0, 2, 1) = v;
  A3(m, 0, 2, 2) = u;
  A3(m, 0, 3, 0) = -uw;
  A3(m, 0, 3, 1) = w;
  A3(m, 0, 3, 3) = u;
  A3(m, 0, 4, 0) = -gamma * E * u + g1 * u * (uu + vv + ww);
  A3(m, 0, 4, 1) = gamma * E - gm1d2 * (3. * uu + (vv + ww));
  A3(m, 0, 4, 2) = -g1 * uv;
  A3(m, 0, 4, 3) = -g1 * uw;
  A3(m, 0, 4, 4) = gamma * u;
  A3(m, 1, 0, 2) = 1.0;
  A3(m, 1, 1, 0) = -uv;
  A3(m, 1, 1, 1) = v;
  A3(m, 1, 1, 2) = u;
  A3(m, 1, 2, 0) = gm1d2 * (uu + ww) + gm3d2 * vv;
  A3(m, 1, 2, 1) = -g1 * u;
  A3(m, 1, 2, 2) = -g3 * v;
  A3(m, 1, 2, 3) = -g1 * w;
  A3(m, 1, 2, 4) = g1;
  A3(m, 1, 3, 0) = -vw;
  A3(m, 1, 3, 2) = w;
  A3(m, 1, 3, 3) = v;
  A3(m, 1, 4, 0) = -gamma * E * v + g1 * v * (uu + vv + ww);
  A3(m, 1, 4, 1) = -g1 * uv;
  A3(m, 1, 4, 2) = gamma * E - gm1d2 * ((uu + ww) + 3. * vv);
  A3(m, 1, 4, 3) = -g1 * vw;
  A3(m, 1, 4, 4) = gamma * v;
  A3(m, 2, 0, 3) = 1.0;
  A3(m, 2, 1, 0) = -uw;
  A3(m, 2, 1, 1) = w;
  A3(m, 2, 1, 3) = u;
  A3(m, 2, 2, 0) = -vw;
  A3(m, 2, 2, 2) = w;
  A3(m, 2, 2, 3) = v;
  A3(m, 2, 3, 0) = gm1d2 * (uu + vv) + gm3d2 * ww;
  A3(m, 2, 3, 1) = -g1 * u;
  A3(m, 2, 3, 2) = -g1 * v;
  A3(m, 2, 3, 3) = -g3 * w;
  A3(m, 2, 3, 4) = g1;
  A3(m, 2, 4, 0) = -gamma * E * w + g1 * w * (uu + vv + ww);
  A3(m, 2, 4, 1) = -g1 * uw;
  A3(m, 2, 4, 2) = -g1 * vw;
  A3(m, 2, 4, 3) = gamma * E - gm1d2 * ((uu + vv) + 3. * ww);
  A3(m, 2, 4, 4) = gamma * w;
}

void calc_b3(const Gas& th, const FlowPt& f, double* m) {  // NavierStokes3D.h:193-343
  std::fill(m, m + 75, 0.0);
  double mu = f.mu, E = f.E;
  auto& t = f.tau;
  double lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  double denom = 1. / std::pow(f.U[0], 2), TERM1 = f.k * denom / th.Cv;
  double rho = f.U[0], u = f.v[0], v = f.v[1], w = f.v[2], uu = u * u, vv = v * v, ww = w * w;
  double drdx = f.dU[0][0], dldx = f.dU[1][0], dmdx = f.dU[2][0], dndx = f.dU[3][0], dedx = f.dU[4][0];
  double drdy = f.dU[0][1], dldy = f.dU[1][1], dmdy = f.dU[2][1], dndy = f.dU[3][1], dedy = f.dU[4][1];
  double drdz = f.dU[0][2], dldz = f.dU[1][2], dmdz = f.dU[2][2], dndz = f.dU[3][2], dedz = f.dU[4][2];
  double l = f.U[1], mm = f.U[2], n = f.U[3];
  // the reference builds these with reinv = 1 and scales by 1/Re at the end
  A3(m, 0, 1, 0) = (denom * (mu_R * dldx + lambda * (dmdy + dndz) + mu_R * (-2. * u * drdx + v * drdy + w * drdz)));
  A3(m, 0, 1, 1) = mu_R * drdx * denom;
  A3(m, 0, 1, 2) = lambda * drdy * denom;
  A3(m, 0, 1, 3) = lambda * drdz * denom;
  A3(m, 0, 2, 0) = (mu * denom * (dldy + dmdx - 2. * (u * drdy + v * drdx)));
  A3(m, 0, 2, 1) = mu * drdy * denom;
  A3(m, 0, 2, 2) = mu * drdx * denom;
  A3(m, 0, 3, 0) = (mu * denom * (dldz + dndx - 2. * (u * drdz + w * drdx)));
  A3(m, 0, 3, 1) = mu * drdz * denom;
  A3(m, 0, 3, 3) = mu * drdx * denom;
  A3(m, 0, 4, 0) = u * A3(m, 0, 1, 0) + v * A3(m, 0, 2, 0) + w * A3(m, 0, 3, 0) +
                   (denom * (l * t[0][0] + mm * t[0][1] + n * t[0][2]) -
                    TERM1 * (-dedx + (2. * E - 3. * (uu + vv + ww)) * drdx + 2. * (u * dldx + v * dmdx + w * dndx)));
  A3(m, 0, 4, 1) = u * A3(m, 0, 1, 1) + v * A3(m, 0, 2, 1) + w * A3(m, 0, 3, 1) + (-t[0][0] / rho - TERM1 * (2. * u * drdx - dldx));
  A3(m, 0, 4, 2) = u * A3(m, 0, 1, 2) + v * A3(m, 0, 2, 2) + w * A3(m, 0, 3, 2) + (-t[0][1] / rho - TERM1 * (-dmdx + 2. * v * drdx));
  A3(m, 0, 4, 3) = u * A3(m, 0, 1, 3) + v * A3(m, 0, 2, 3) + w * A3(m, 0, 3, 3) + (-t[0][2] / rho - TERM1 * (2 * w * drdx - dndx));
  A3(m, 0, 4, 4) = TERM1 * drdx;
  A3(m, 1, 1, 0) = A3(m, 0, 2, 0);
  A3(m, 1, 1, 1) = A3(m, 0, 2, 1);
  A3(m, 1, 1, 2) = A3(m, 0, 2, 2);
  A3(m, 1, 2, 0) = (denom * (lambda * (dldx + dndz) + mu_R * (dmdy + u * drdx - 2. * v * drdy + w * drdz)));
  A3(m, 1, 2, 1) = lambda * drdx * denom;
  A3(m, 1, 2, 2) = mu_R * drdy * denom;
  A3(m, 1, 2, 3) = lambda * drdz * denom;
  A3(m, 1, 3, 0) = (mu * denom * (dmdz + dndy - 2. * (v * drdz + w * drdy)));
  A3(m, 1, 3, 2) = mu * denom * drdz;
  A3(m, 1, 3, 3) = mu * denom * drdy;
  A3(m, 1, 4, 0) = u * A3(m, 1, 1, 0) + v * A3(m, 1, 2, 0) + w * A3(m, 1, 3, 0) +
                   (denom * (l * t[1][0] + mm * t[1][1] + n * t[1][2]) -
                    TERM1 * (-dedy + (2. * E - 3. * (uu + vv + ww)) * drdy + 2. * (u * dldy + v * dmdy + w * dndy)));
  A3(m, 1, 4, 1) = u * A3(m, 1, 1, 1) + v * A3(m, 1, 2, 1) + w * A3(m, 1, 3, 1) + (-t[1][0] / rho - TERM1 * (-dldy + 2. * u * drdy));
  A3(m, 1, 4, 2) = u * A3(m, 1, 1, 2) + v * A3(m, 1, 2, 2) + w * A3(m, 1, 3, 2) + (-t[1][1] / rho - TERM1 * (2. * v * drdy - dmdy));
  A3(m, 1, 4, 3) = u * A3(m, 1, 1, 3) + v * A3(m, 1, 2, 3) + w * A3(m, 1, 3, 3) + (-t[1][2] / rho - TERM1 * (2. * w * drdy - dndy));
  A3(m, 1, 4, 4) = TERM1 * drdy;
  A3(m, 2, 1, 0) = A3(m, 0, 3, 0);
  A3(m, 2, 1, 1) = A3(m, 0, 3, 1);
  A3(m, 2, 1, 3) = A3(m, 0, 3, 3);
  A3(m, 2, 2, 0) = A3(m, 1, 3, 0);
  A3(m, 2, 2, 2) = A3(m, 1, 3, 2);
  A3(m, 2, 2, 3) = A3(m, 1, 3, 3);
  A3(m, 2, 3, 0) = (denom * (mu_R * (dndz + u * drdx + v * drdy - 2. * w * drdz) + lambda * (dldx + dmdy)));
  A3(m, 2, 3, 1) = lambda * drdx * denom;
  A3(m, 2, 3, 2) = lambda * drdy * denom;
  A3(m, 2, 3, 3) = mu_R * drdz * denom;
  A3(m, 2, 4, 0) = u * A3(m, 2, 1, 0) + v * A3(m, 2, 2, 0) + w * A3(m, 2, 3, 0) +
                   (denom * (l * t[2][0] + mm * t[2][1] + n * t[2][2]) -
                    TERM1 * (-dedz + (2. * E - 3. * (uu + vv + ww)) * drdz + 2. * (u * dldz + v * dmdz + w * dndz)));
  A3(m, 2, 4, 1) = u * A3(m, 2, 1, 1) + v * A3(m, 2, 2, 1) + w * A3(m, 2, 3, 1) + (-t[2][0] / rho - TERM1 * (2. * u * drdz - dldz));
  A3(m, 2, 4, 2) = u * A3(m, 2, 1, 2) + v * A3(m, 2, 2, 2) + w * A3(m, 2, 3, 2) + (-t[2][1] / rho - TERM1 * (2. * v * drdz - dmdz));
  A3(m, 2, 4, 3) = u * A3(m, 2, 1, 3) + v * A3(m, 2, 2, 3) + w * A3(m, 2, 3, 3) + (-t[2][2] / rho - TERM1 * (2. * w * drdz - dndz));
  A3(m, 2, 4, 4) = TERM1 * drdz;
  double reinv = 1.0 / th.creyn;
  for (int i = 0; i < 75; i++) m[i] *= reinv;
}

void calc_c3(const Gas& th, const FlowPt& f, double* m) {  // NavierStokes3D.h:347-477
  std::fill(m, m + 225, 0.0);
  double mu = f.mu, lambda = -2. * mu / 3., mu_R = 2. * mu + lambda;
  double rho = f.U[0], denom = 1. / std::pow(rho, 2);
  double l = f.U[1], mm = f.U[2], n = f.U[3], re = f.U[4];
  double ll = l * l, mm2 = mm * mm, nn = n * n, hkocv = f.k / th.Cv, TERM1 = f.k / th.Cv * denom;
  // built with reinv = 1, scaled by 1/Re at the end (NavierStokes3D.h:462-476)
  C4(m, 0, 0, 1, 0) = mu_R * l * denom;
  C4(m, 0, 0, 1, 1) = (-mu_R / rho);
  C4(m, 0, 0, 2, 0) = mu * mm * denom;
  C4(m, 0, 0, 2, 2) = (-mu / rho);
  C4(m, 0, 0, 3, 0) = mu * n * denom;
  C4(m, 0, 0, 3, 3) = (-mu / rho);
  C4(m, 0, 0, 4, 0) = (l * C4(m, 0, 0, 1, 0) + mm * C4(m, 0, 0, 2, 0) + n * C4(m, 0, 0, 3, 0)) / rho -
                      TERM1 * (-re + (ll + mm2 + nn) / rho);
  C4(m, 0, 0, 4, 1) = (l / rho) * C4(m, 0, 0, 1, 1) + TERM1 * l;
  C4(m, 0, 0, 4, 2) = (mm / rho) * C4(m, 0, 0, 2, 2) + TERM1 * mm;
  C4(m, 0, 0, 4, 3) = (n / rho) * C4(m, 0, 0, 3, 3) + TERM1 * n;
  C4(m, 0, 0, 4, 4) = (-hkocv / rho);
  C4(m, 0, 1, 1, 0) = lambda * mm * denom;
  C4(m, 0, 1, 1, 2) = (-lambda / rho);
  C4(m, 0, 1, 2, 0) = mu * l * denom;
  C4(m, 0, 1, 2, 1) = (-mu / rho);
  C4(m, 0, 1, 4, 0) = (l / rho) * C4(m, 0, 1, 1, 0) + (mm / rho) * C4(m, 0, 1, 2, 0);
  C4(m, 0, 1, 4, 1) = (mm / rho) * C4(m, 0, 1, 2, 1);
  C4(m, 0, 1, 4, 2) = (l / rho) * C4(m, 0, 1, 1, 2);
  C4(m, 0, 2, 1, 0) = lambda * n * denom;
  C4(m, 0, 2, 1, 3) = (-lambda / rho);
  C4(m, 0, 2, 3, 0) = mu * l * denom;
  C4(m, 0, 2, 3, 1) = (-mu / rho);
  C4(m, 0, 2, 4, 0) = (l / rho) * C4(m, 0, 2, 1, 0) + (n / rho) * C4(m, 0, 2, 3, 0);
  C4(m, 0, 2, 4, 1) = (n / rho) * C4(m, 0, 2, 3, 1);
  C4(m, 0, 2, 4, 3) = (l / rho) * C4(m, 0, 2, 1, 3);
  C4(m, 1, 0, 1, 0) = C4(m, 0, 0, 2, 0);
  C4(m, 1, 0, 1, 2) = C4(m, 0, 0, 2, 2);
  C4(m, 1, 0, 2, 0) = lambda * l * denom;
  C4(m, 1, 0, 2, 1) = (-lambda / rho);
  C4(m, 1, 0, 4, 0) = (l / rho) * C4(m, 1, 0, 1, 0) + (mm / rho) * C4(m, 1, 0, 2, 0);
  C4(m, 1, 0, 4, 1) = (mm / rho) * C4(m, 1, 0, 2, 1);
  C4(m, 1, 0, 4, 2) = (l / rho) * C4(m, 1, 0, 1, 2);
  C4(m, 1, 1, 1, 0) = C4(m, 0, 1, 2, 0);
  C4(m, 1, 1, 1, 1) = C4(m, 0, 1, 2, 1);
  C4(m, 1, 1, 2, 0) = mu_R * mm * denom;
  C4(m, 1, 1, 2, 2) = (-mu_R / rho);
  C4(m, 1, 1, 3, 0) = mu * n * denom;
  C4(m, 1, 1, 3, 3) = (-mu / rho);
  C4(m, 1, 1, 4, 0) = (l * C4(m, 1, 1, 1, 0) + mm * C4(m, 1, 1, 2, 0) + n * C4(m, 1, 1, 3, 0)) / rho -
                      TERM1 * (-re + (ll + mm2 + nn) / rho);
  C4(m, 1, 1, 4, 1) = (l / rho) * C4(m, 1, 1, 1, 1) + TERM1 * l;
  C4(m, 1, 1, 4, 2) = (mm / rho) * C4(m, 1, 1, 2, 2) + TERM1 * mm;
  C4(m, 1, 1, 4, 3) = (n / rho) * C4(m, 1, 1, 3, 3) + TERM1 * n;
  C4(m, 1, 1, 4, 4) = (-hkocv / rho);
  C4(m, 1, 2, 2, 0) = lambda * n * denom;
  C4(m, 1, 2, 2, 3) = (-lambda / rho);
  C4(m, 1, 2, 3, 0) = mu * mm * denom;
  C4(m, 1, 2, 3, 2) = (-mu / rho);
  C4(m, 1, 2, 4, 0) = (mm / rho) * C4(m, 1, 2, 2, 0) + (n / rho) * C4(m, 1, 2, 3, 0);
  C4(m, 1, 2, 4, 2) = (n / rho) * C4(m, 1, 2, 3, 2);
  C4(m, 1, 2, 4, 3) = (mm / rho) * C4(m, 1, 2, 2, 3);
  C4(m, 2, 0, 1, 0) = C4(m, 0, 0, 3, 0);
  C4(m, 2, 0, 1, 3) = C4(m, 0, 0, 3, 3);
  C4(m, 2, 0, 3, 0) = lambda * l * denom;
  C4(m, 2, 0, 3, 1) = (-lambda / rho);
  C4(m, 2, 0, 4, 0) = (l / rho) * C4(m, 2, 0, 1, 0) + (n / rho) * C4(m, 2, 0, 3, 0);
  C4(m, 2, 0, 4, 1) = (n / rho) * C4(m, 2, 0, 3, 1);
  C4(m, 2, 0, 4, 3) = (l / rho) * C4(m, 2, 0, 1, 3);
  C4(m, 2, 1, 2, 0) = C4(m, 1, 1, 3, 0);
  C4(m, 2, 1, 2, 3) = C4(m, 1, 1, 3, 3);
  C4(m, 2, 1, 3, 0) = lambda * mm * denom;
  C4(m, 2, 1, 3, 2) = (-lambda / rho);
  C4(m, 2, 1, 4, 0) = (mm / rho) * C4(m, 2, 1, 2, 0) + (n / rho) * C4(m, 2, 1, 3, 0);
  C4(m, 2, 1, 4, 2) = (n / rho) * C4(m, 2, 1, 3, 2);
  C4(m, 2, 1, 4, 3) = (mm / rho) * C4(m, 2, 1, 2, 3);
  C4(m, 2, 2, 1, 0) = C4(m, 0, 2, 3, 0);
  C4(m, 2, 2, 1, 1) = C4(m, 0, 2, 3, 1);
  C4(m, 2, 2, 2, 0) = C4(m, 1, 2, 3, 0);
  C4(m, 2, 2, 2, 2) = C4(m, 1, 2, 3, 2);
  C4(m, 2, 2, 3, 0) = mu_R * n * denom;
  C4(m, 2, 2, 3, 3) = (-mu_R / rho);
  C4(m, 2, 2, 4, 0) = (l * C4(m, 2, 2, 1, 0) + mm * C4(m, 2, 2, 2, 0) + n * C4(m, 2, 2, 3, 0)) / rho -
                      TERM1 * (-re + (ll + mm2 + nn) / rho);
  C4(m, 2, 2, 4, 1) = (l / rho) * C4(m, 2, 2, 1, 1) + TERM1 * l;
  C4(m, 2, 2, 4, 2) = (mm / rho) * C4(m, 2, 2, 2, 2) + TERM1 * mm;
  C4(m, 2, 2, 4, 3) = (n / rho) * C4(m, 2, 2, 3, 3) + TERM1 * n;
  C4(m, 2, 2, 4, 4) = (-hkocv / rho);
  double reinv = 1.0 / th.creyn;
  for (int i = 0; i < 225; i++) m[i] *= reinv;
}

// convective flux F (NavierStokes2D.h:11-29, NavierStokes3D.h:10-37) and viscous flux G
// (NavierStokes2D.h:32-47, NavierStokes3D.h:41-64); F/G stored [i][r] -> [i*5+r]
void calc_F(int ndim, const NodeState& n, double* F) {
  std::fill(F, F + 15, 0.0);
  if (ndim == 2) {
    double rho = n.U[0], l = n.U[1], m = n.U[2], e = n.U[3], p = n.p;
    F[0 * 5 + 0] = l;
    F[0 * 5 + 1] = p + std::pow(l, 2) / rho;
    F[0 * 5 + 2] = (l * m) / rho;
    F[0 * 5 + 3] = (p + e) * (l / rho);
    F[1 * 5 + 0] = m;
    F[1 * 5 + 1] = (l * m) / rho;
    F[1 * 5 + 2] = p + std::pow(m, 2) / rho;
    F[1 * 5 + 3] = (p + e) * (m / rho);
  } else {
    double rho = n.U[0], u = n.U[1] / n.U[0], v = n.U[2] / n.U[0], w = n.U[3] / n.U[0], E = n.U[4] / n.U[0], p = n.p;
    double vel[3] = {u, v, w};
    for (int i = 0; i < 3; i++) {
      F[i * 5 + 0] = rho * vel[i];
      F[i * 5 + 4] = (rho * E + p) * vel[i];
    }
    F[0 * 5 + 1] = rho * u * u + p;
    F[0 * 5 + 2] = rho * u * v;
    F[0 * 5 + 3] = rho * u * w;
    F[1 * 5 + 1] = rho * u * v;
    F[1 * 5 + 2] = rho * v * v + p;
    F[1 * 5 + 3] = rho * v * w;
    F[2 * 5 + 1] = rho * u * w;
    F[2 * 5 + 2] = rho * v * w;
    F[2 * 5 + 3] = rho * w * w + p;
  }
}

void calc_G(int ndim, const FlowPt& f, const double* v, double Re, double* G) {
  std::fill(G, G + 15, 0.0);
  double reinv = 1.0 / Re;
  for (int i = 0; i < ndim; i++) {
    G[i * 5 + 0] = 0.0;
    for (int j = 0; j < ndim; j++) G[i * 5 + 1 + j] = -f.tau[i][j] * reinv;
    double s = -f.tau[i][0] * v[0];
    for (int j = 1; j < ndim; j++) s = s - f.tau[i][j] * v[j];
    G[i * 5 + ndim + 1] = (s - f.k * f.dT[i]) * reinv;
  }
}

// ---- one element ----------------------------------------------------------
struct ElemCtx {
  const Gas* g;
  int ndim, nnod, neqn, nbnod, Ke;
  double dt, dtsq_2, s1, s2, s3, s4;
  int phys3d;
  NodeState* nd[8];
  const double* H;  // Hnm of an adaptive element (Hnm(N, M) at N + nnod*M) or null
  double* R;    // column-major Ke x Ke
  double* rhs;
  double gz[2], gw[2];
  double& Rm(int i, int j) { return R[(size_t)j * Ke + i]; }
};

void jacobians(const ElemCtx& c, const FlowPt& f, double* a, double* b, double* cc) {
  if (c.ndim == 2) {
    calc_a2(*c.g, f, a);
    calc_b2(*c.g, f, b);
    calc_c2(*c.g, f, cc);
  } else {
    calc_a3(*c.g, f, a);
    calc_b3(*c.g, f, b);
    calc_c3(*c.g, f, cc);
  }
}

void node_flux(const ElemCtx& c, const FlowPt& f, NodeState* const* nd, int nn, double F[][15], double G[][15]) {
  for (int N = 0; N < nn; N++) {
    if (c.ndim == 2 || c.phys3d) calc_F(c.ndim, *nd[N], F[N]);
    else std::fill(F[N], F[N] + 15, 0.0);  // NavierStokes.h:6 base body runs in 3D
    calc_G(c.ndim, f, nd[N]->v, c.g->creyn, G[N]);
  }
}

// MeshRefine2D.h:877-900 (adap): Phi_M <- sum_N Phi_N Hnm(N, M), dPxi(M, j) likewise, for
// the shape functions of an adaptive element before its Jacobian
void hnm_transform(const double* H, int nnod, int ndim, double* Phi, double dPxi[][3]) {
  double P[8] = {0, 0, 0, 0, 0, 0, 0, 0}, D[8][3] = {};
  for (int N = 0; N < nnod; N++)
    for (int M = 0; M < nnod; M++) {
      P[M] += Phi[N] * H[N + nnod * M];
      for (int j = 0; j < ndim; j++) D[M][j] += dPxi[N][j] * H[N + nnod * M];
    }
  for (int M = 0; M < nnod; M++) {
    Phi[M] = P[M];
    for (int j = 0; j < ndim; j++) dPxi[M][j] = D[M][j];
  }
}

// FDVGalerkin.h:157-451 (domain integral at one Gauss point)
void domain(ElemCtx& c, const double* w, const double* zeta) {
  const int ndim = c.ndim, nnod = c.nnod, neqn = c.neqn;
  double Phi[8], dPxi[8][3], dPhi[8][3], J, jac[3][3];
  if (ndim == 2) shape2(zeta, Phi, dPxi);
  else shape3(zeta, Phi, dPxi);
  if (c.H) hnm_transform(c.H, nnod, ndim, Phi, dPxi);  // FDVGalerkin.h:183-186, 198-201
  if (ndim == 2) J = jac2(dPxi, c.nd, jac, dPhi);
  else J = jac3(dPxi, c.nd, dPhi);
  FlowPt f;
  gp_sum(*c.g, ndim, neqn, nnod, c.nd, Phi, dPhi, f);
  tau_calc(ndim, f);

  double Psi[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double tau = 0;
  if (ndim == 2) {  // FDVGalerkin.h:225-332 streamline-upwind diffusion (2D only)
    // its Jacobian comes from the untransformed shape functions (FDVGalerkin.h:237-240), which
    // differs from jac for an adaptive element
    double (*sj)[3] = jac, jp[3][3];
    if (c.H) {
      double pph[8], pdx[8][3], pdp[8][3];
      shape2(zeta, pph, pdx);
      jac2(pdx, c.nd, jp, pdp);
      sj = jp;
    }
    double J_xi = std::pow(sj[0][0], 2) + std::pow(sj[1][0], 2);
    double J_eta = std::pow(sj[0][1], 2) + std::pow(sj[1][1], 2);
    double e_xi[2], e_eta[2];
    for (int i = 0; i < 2; i++) {
      e_xi[i] = 1. / std::pow(J_xi, 0.5) * sj[i][0];
      e_eta[i] = 1. / std::pow(J_eta, 0.5) * sj[i][1];
    }
    double v_xi = 0, v_eta = 0, S = 0;
    for (int i = 0; i < 2; i++) v_xi += f.v[i] * e_xi[i];
    for (int i = 0; i < 2; i++) v_eta += f.v[i] * e_eta[i];
    for (int i = 0; i < 2; i++) S += f.v[i] * f.v[i];
    // edge-midpoint interpolants: xi=-1, xi=+1, eta=-1, eta=+1
    const double xleft[4] = {0.5, 0.0, 0.0, 0.5}, xright[4] = {0.0, 0.5, 0.5, 0.0};
    const double xtop[4] = {0.5, 0.5, 0.0, 0.0}, xbottom[4] = {0.0, 0.0, 0.5, 0.5};
    double h_xi = 0.0, h_eta = 0.0;
    for (int N = 0; N < nnod; N++) {
      h_xi += xright[N] * c.nd[N]->x[0] - xleft[N] * c.nd[N]->x[0];
      h_eta += xtop[N] * c.nd[N]->x[1] - xbottom[N] * c.nd[N]->x[1];
    }
    double R_xi = f.U[0] * v_xi * h_xi / f.mu;
    double R_eta = f.U[0] * v_eta * h_eta / f.mu;
    double alpha_xi = (R_xi == 0) ? 0 : std::cosh(R_xi / 2.) / std::sinh(R_xi / 2.) - 2. / R_xi;
    double alpha_eta = (R_eta == 0) ? 0 : std::cosh(R_eta / 2.) / std::sinh(R_eta / 2.) - 2. / R_eta;
    tau = (S == 0) ? 0 : (1. / 4.) * (alpha_xi * h_xi * v_xi + alpha_eta * h_eta * v_eta) / S;
    for (int N = 0; N < nnod; N++)
      for (int i = 0; i < ndim; i++) Psi[N] += tau * f.v[i] * dPhi[N][i];
  }
  {  // FDVGalerkin.h:336-387 discontinuity capturing
    double A[3] = {0, 0, 0};
    for (int k = 0; k < ndim; k++)
      for (int j = 0; j < ndim; j++) A[j] += f.dV[j][k] * f.v[k];
    double vv = 0, AA = 0;
    for (int i = 0; i < ndim; i++) vv += f.v[i] * f.v[i];
    for (int i = 0; i < ndim; i++) AA += A[i] * A[i];
    double gamma = std::sqrt(vv) * std::sqrt(AA);
    double tau_b = 0;
    for (int j = 0; j < ndim; j++) tau_b += tau * f.v[j] * A[j] / gamma;
    if ((tau_b - tau) < 0) tau_b = tau;
    if (gamma == 0) tau_b = 0;
    for (int N = 0; N < nnod; N++)
      for (int i = 0; i < ndim; i++) Psi[N] += tau_b * f.v[i] * dPhi[N][i];
  }

  double a[75], b[75], cc[225];
  jacobians(c, f, a, b, cc);
  double F[8][15], G[8][15];
  node_flux(c, f, c.nd, nnod, F, G);

  // FDVGalerkin.h:536-641 (d = 0, B = 0, s5 = s6 = 0: eta = identity and the d/B terms vanish)
  const double dt = c.dt, dtsq_2 = c.dtsq_2;
  double p[8][3][5], q[8][3][3][5], gq[3][5][5], nd[3][5][5], h[3][3][5][5];
  for (int be = 0; be < nnod; be++)
    for (int i = 0; i < ndim; i++)
      for (int r = 0; r < neqn; r++) p[be][i][r] = 0 + dt * (F[be][i * 5 + r] + G[be][i * 5 + r]);
  for (int i = 0; i < ndim; i++)
    for (int r = 0; r < neqn; r++)
      for (int s = 0; s < neqn; s++) {
        double X = dt * (c.s1 * A3(a, i, r, s) + c.s3 * A3(b, i, r, s));
        gq[i][r][s] = 0 - X;
        nd[i][r][s] = 0 + X;
      }
  for (int be = 0; be < nnod; be++)
    for (int i = 0; i < ndim; i++)
      for (int j = 0; j < ndim; j++)
        for (int r = 0; r < neqn; r++) {
          double acc = 0;
          for (int s = 0; s < neqn; s++)
            acc -= dtsq_2 * (A3(a, i, r, s) + A3(b, i, r, s)) * (F[be][j * 5 + s] + G[be][j * 5 + s]);
          q[be][i][j][r] = acc;
        }
  for (int i = 0; i < ndim; i++)
    for (int j = 0; j < ndim; j++)
      for (int r = 0; r < neqn; r++)
        for (int s = 0; s < neqn; s++) {
          double acc = 0;
          acc -= (dt * c.s3 * C4(cc, i, j, r, s));
          for (int t = 0; t < neqn; t++)
            acc -= (-dtsq_2 * (c.s2 * (A3(a, i, r, t) * A3(a, j, t, s) + A3(b, i, r, t) * A3(a, j, t, s)) +
                               c.s4 * ((A3(a, i, r, t) * A3(b, j, t, s) + A3(b, i, r, t) * A3(b, j, t, s)))));
          h[i][j][r][s] = acc;
        }

  // FDVGalerkin.h:405-451
  double w_i = 1.0;
  for (int d = 0; d < ndim; d++) w_i *= w[d];
  for (int N = 0; N < nnod; N++)
    for (int ir = 0; ir < neqn; ir++) {
      int I = neqn * N + ir;
      for (int i = 0; i < ndim; i++) {
        for (int be = 0; be < nnod; be++) c.rhs[I] += w_i * p[be][i][ir] * dPhi[N][i] * Phi[be] * J;
        for (int j = 0; j < ndim; j++)
          for (int be = 0; be < nnod; be++) c.rhs[I] += w_i * q[be][i][j][ir] * dPhi[N][i] * dPhi[be][j] * J;
      }
      for (int M = 0; M < nnod; M++)
        for (int is = 0; is < neqn; is++) {
          int Jx = neqn * M + is;
          double& Rij = c.Rm(I, Jx);
          Rij += w_i * (ir == is ? 1.0 : 0.0) * Phi[N] * Phi[M] * J;
          for (int i = 0; i < ndim; i++) {
            Rij += w_i * gq[i][ir][is] * dPhi[N][i] * Phi[M] * J;
            for (int j = 0; j < ndim; j++) {
              Rij += w_i * h[i][j][ir][is] * dPhi[N][i] * dPhi[M][j] * J;
              Rij += w_i * nd[i][ir][is] * Psi[N] * dPhi[M][j] * J;
            }
          }
        }
    }
}

// 2D boundary treatment of the Gauss-point state (eval1dboundary.h:9-251)
void bc_1d(int code, FlowPt& f, NodeState* const* nd, const double* en, int neqn) {
  double len = std::sqrt(en[0] * en[0] + en[1] * en[1]);
  double n[2] = {en[0] / len, en[1] / len};
  auto dot2 = [](const double* a, const double* b) { return 0 + a[0] * b[0] + a[1] * b[1]; };
  switch (code) {
    case 2:
    case 12:
      f.v[0] -= dot2(f.v, n) * n[0];
      f.v[1] -= dot2(f.v, n) * n[1];
      f.dT[0] -= dot2(f.dT, n) * n[0];
      f.dT[1] -= dot2(f.dT, n) * n[1];
      break;
    case 1:
    case 51:
      f.dT[0] -= dot2(f.dT, n) * n[0];
      f.dT[1] -= dot2(f.dT, n) * n[1];
      break;
    case -1:
      f.dV[0][0] = 0.0; f.dV[1][0] = 0.0; f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[0] = 0.0;
      break;
    case 6:
      f.dV[0][0] = 0.0; f.dV[1][0] = 0.0; f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[0] = 0.0;
      for (int i = 0; i < neqn; i++) f.dU[i][0] = 0.0;
      break;
    case -2:
    case 7:
      f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[1] = 0.0;
      for (int i = 0; i < neqn; i++) f.dU[i][1] = 0.0;
      break;
    case 4:
    case 8: {
      double nn[2];
      if (code == 4) {
        f.v[0] = 0; f.v[1] = 0;
        nn[0] = en[0]; nn[1] = en[1];
      } else {
        double alpha = 10 * (3.14159 / 180.0);
        double dl = std::abs(nd[1]->x[1] - nd[0]->x[1]);
        nn[0] = std::cos(alpha) * dl;
        nn[1] = std::sin(alpha) * dl;
      }
      double dudot = (f.dV[0][0] * nn[0] + f.dV[0][1] * nn[1]);
      double dvdot = (f.dV[1][0] * nn[0] + f.dV[1][1] * nn[1]);
      double dtdot = (f.dT[0] * nn[0] + f.dT[1] * nn[1]);
      f.dV[0][0] -= dudot * nn[0]; f.dV[0][1] -= dudot * nn[1];
      f.dV[1][0] -= dvdot * nn[0]; f.dV[1][1] -= dvdot * nn[1];
      f.dT[0] -= dtdot * nn[0]; f.dT[1] -= dtdot * nn[1];
      double dUdot[5];
      for (int i = 0; i < neqn; i++) dUdot[i] = f.dU[i][0] * nn[0] + f.dU[i][1] * nn[1];
      for (int i = 0; i < neqn; i++)
        for (int j = 0; j < 2; j++) f.dU[i][j] -= dUdot[i] * nn[j];
    } break;
    case -12:
      f.dV[0][1] = 0.0; f.dV[1][1] = 0.0;
      f.dT[1] = 0.0;
      f.v[1] = 0.0;
      for (int i = 0; i < neqn; i++) f.dU[i][1] = 0.0;
      break;
    case 11:
    case 21:
      f.v[0] = 0; f.v[1] = 0;
      f.dV[0][0] = 0.0; f.dV[1][0] = 0.0;
      f.dT[1] = 0.0;
      for (int i = 0; i < neqn; i++) f.dU[i][1] = 0.0;
      break;
    default:
      break;  // codes without a handler leave the state untouched (the reference stops at cin.get())
  }
  tau_calc(2, f);
  if (code == 2 || code == 12 || code == 7) { f.tau[0][1] = 0.0; f.tau[1][0] = 0.0; }
  if (code == 6) { f.tau[0][0] = 0.; f.tau[1][0] = 0.; }
}

// 3D boundary treatment (eval2dboundary.h:14-371); tau is zero on entry (Flow::clear)
void bc_2d(int code, FlowPt& f, const double* en, bool adiabatic) {
  switch (code) {
    case 2:
    case 12:
      for (int i = 0; i < 3; i++) f.dV[i][2] = 0;
      f.dT[2] = 0;
      break;
    case 22:
      for (int i = 0; i < 3; i++) f.dV[i][1] = 0;
      f.dT[1] = 0;
      tau_calc(3, f);
      f.tau[0][1] = 0.0; f.tau[1][1] = 0.0; f.tau[2][1] = 0.0;
      f.tau[1][0] = 0.0; f.tau[1][2] = 0.0;
      break;
    case 1:
    case 51:
      if (adiabatic) f.dT[2] = 0.0;
      tau_calc(3, f);
      break;
    case 21:
    case 31:
      if (adiabatic) f.dT[1] = 0.0;
      tau_calc(3, f);
      break;
    case 11:
      if (adiabatic) f.dT[0] = 0.0;
      tau_calc(3, f);
      break;
    case -1:
      return;
    case 6:
      f.dT[0] = 0.0;
      tau_calc(3, f);
      for (int i = 0; i < 3; i++) f.tau[i][0] = 0;
      break;
    case 7:
      f.dT[2] = 0.0;
      tau_calc(3, f);
      for (int i = 0; i < 3; i++) f.tau[i][2] = 0;
      // falls through into 77/32 (eval2dboundary.h:113-145)
      f.dT[1] = 0.0;
      tau_calc(3, f);
      for (int i = 0; i < 3; i++) f.tau[i][1] = 0;
      break;
    case 77:
    case 32:
      f.dT[1] = 0.0;
      tau_calc(3, f);
      for (int i = 0; i < 3; i++) f.tau[i][1] = 0;
      break;
    case 4: {
      f.v[0] = 0; f.v[1] = 0; f.v[2] = 0;
      double n[3] = {en[0], en[1], en[2]};
      double dudot = (f.dV[0][0] * n[0] + f.dV[0][1] * n[1] + f.dV[0][2] * n[2]);
      double dvdot = (f.dV[1][0] * n[0] + f.dV[1][1] * n[1] + f.dV[1][2] * n[2]);
      double dtdot = (f.dT[0] * n[0] + f.dT[1] * n[1] + f.dT[2] * n[2]);
      for (int j = 0; j < 3; j++) f.dV[0][j] -= dudot * n[j];
      for (int j = 0; j < 3; j++) f.dV[1][j] -= dvdot * n[j];
      for (int j = 0; j < 3; j++) f.dT[j] -= dtdot * n[j];
      double dUdot[5];
      for (int i = 0; i < 5; i++) dUdot[i] = f.dU[i][0] * n[0] + f.dU[i][1] * n[1] + f.dU[i][2] * n[2];
      for (int i = 0; i < 3; i++)  // loop bound is dU.jmax() = 3 in the reference
        for (int j = 0; j < 3; j++) f.dU[i][j] -= dUdot[i] * n[j];
    } break;
    case 8:
      tau_calc(3, f);
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

// face-local node lists (get_face.h:80-89, 106-164)
const int kFace2[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
const int kFace3[6][4] = {{3, 2, 1, 0}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}, {6, 7, 4, 5}};

// FDVGalerkin.h:467-533 + TFNorm2D/3D + sumBoundaryTerms/sumBoundaryMatrix (:643-756)
void boundary_face(ElemCtx& c, const double* w, const double* zeta, int code, const int* fn) {
  const int ndim = c.ndim, neqn = c.neqn, nb = c.nbnod;
  NodeState* nd[4];
  for (int i = 0; i < nb; i++) nd[i] = c.nd[fn[i]];
  double phib[4], en[3], dpidx[4][3];
  std::memset(dpidx, 0, sizeof(dpidx));
  if (ndim == 2) {  // TestFunctions1D.h:7-82
    phib[0] = 0.5 * (1 - zeta[0]);
    phib[1] = 0.5 * (1 + zeta[0]);
    double dxds = 0, dyds = 0;
    const double dp[2] = {-0.5, 0.5};
    for (int i = 0; i < 2; i++) {
      dxds += dp[i] * nd[i]->x[0];
      dyds += dp[i] * nd[i]->x[1];
    }
    en[0] = dyds * w[0];
    en[1] = -dxds * w[0];
    double delx = nd[1]->x[0] - nd[0]->x[0], dely = nd[1]->x[1] - nd[0]->x[1];
    double dpdx[2] = {0, 0}, dpdy[2] = {0, 0};
    if (!(std::abs(delx) < 1.0E-12)) { dpdx[0] = -1.0 / delx; dpdx[1] = 1.0 / delx; }
    if (!(std::abs(dely) < 1.0E-12)) { dpdy[0] = -1.0 / dely; dpdy[1] = 1.0 / dely; }
    for (int i = 0; i < 2; i++) { dpidx[i][0] = dpdx[i]; dpidx[i][1] = dpdy[i]; }
  } else {  // calc_TF_norm3D.h:9-167
    phib[0] = 0.25 * (1 - zeta[0]) * (1 - zeta[1]);
    phib[1] = 0.25 * (1 + zeta[0]) * (1 - zeta[1]);
    phib[2] = 0.25 * (1 + zeta[0]) * (1 + zeta[1]);
    phib[3] = 0.25 * (1 - zeta[0]) * (1 + zeta[1]);
    // face node positions; for an adaptive element the rows of Hnm x of the face's nodes
    // (calc_TF_norm3D.h:25-66: allnode(N) = sum_M Hnm(N, M) x_M)
    double nodeloc[4][3];
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 3; k++) nodeloc[j][k] = nd[j]->x[k];
    if (c.H) {
      for (int j = 0; j < 4; j++) {
        double an[3] = {0, 0, 0};
        for (int M = 0; M < c.nnod; M++)
          for (int k = 0; k < 3; k++) an[k] += c.H[fn[j] + c.nnod * M] * c.nd[M]->x[k];
        for (int k = 0; k < 3; k++) nodeloc[j][k] = an[k];
      }
    }
    double Lam[3], Mu[3];
    for (int i = 0; i < 3; i++) {
      Lam[i] = nodeloc[1][i] - nodeloc[0][i];
      Mu[i] = nodeloc[3][i] - nodeloc[0][i];
    }
    for (int j = 0; j < 3; j++) {  // magnitude recomputed after each component
      Lam[j] /= std::sqrt(0 + Lam[0] * Lam[0] + Lam[1] * Lam[1] + Lam[2] * Lam[2]);
      Mu[j] /= std::sqrt(0 + Mu[0] * Mu[0] + Mu[1] * Mu[1] + Mu[2] * Mu[2]);
    }
    double enorm[3], gama[3];
    enorm[0] = (Lam[1] * Mu[2] - Lam[2] * Mu[1]);
    enorm[1] = (Lam[2] * Mu[0] - Lam[0] * Mu[2]);
    enorm[2] = (Lam[0] * Mu[1] - Lam[1] * Mu[0]);
    gama[0] = (enorm[1] * Lam[2] - enorm[2] * Lam[1]);
    gama[1] = (enorm[2] * Lam[0] - enorm[0] * Lam[2]);
    gama[2] = (enorm[0] * Lam[1] - enorm[1] * Lam[0]);
    double T[3][3];
    for (int i = 0; i < 3; i++) { T[0][i] = Lam[i]; T[1][i] = gama[i]; T[2][i] = enorm[i]; }
    double ph[4], dpxi[4][3];
    shape2(zeta, ph, dpxi);
    double dxdxi[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int N = 0; N < 4; N++)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 2; j++) dxdxi[i][j] += dpxi[N][j] * nodeloc[N][i];
    double tr[2][2] = {{0, 0}, {0, 0}};
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++)
        for (int k = 0; k < 3; k++) tr[i][j] += T[i][k] * dxdxi[k][j];
    double detjac = tr[0][0] * tr[1][1] - tr[1][0] * tr[0][1];
    double djacinv = 1. / detjac;
    double dpdx[4][2];
    for (int N = 0; N < 4; N++) {
      dpdx[N][0] = (tr[1][1] * dpxi[N][0] - tr[1][0] * dpxi[N][1]) * djacinv;
      dpdx[N][1] = (-tr[0][1] * dpxi[N][0] + tr[0][0] * dpxi[N][1]) * djacinv;
    }
    for (int i = 0; i < 3; i++) {
      for (int N = 0; N < 4; N++)
        for (int j = 0; j < 2; j++) dpidx[N][i] += T[j][i] * dpdx[N][j];
      en[i] = enorm[i] * w[0] * w[1] * detjac;
    }
    if (c.H) {  // FDVGalerkin.h:489-497, MeshRefine2D.h:904-951 (adap_face): phib only
      double pt[4] = {0, 0, 0, 0};
      for (int N = 0; N < 4; N++)
        for (int M = 0; M < 4; M++) pt[M] += phib[N] * c.H[fn[N] + c.nnod * fn[M]];
      for (int M = 0; M < 4; M++) phib[M] = pt[M];
    }
  }
  FlowPt f;
  gp_sum(*c.g, ndim, neqn, nb, nd, phib, dpidx, f);
  if (ndim == 2) bc_1d(code, f, nd, en, neqn);
  else bc_2d(code, f, en, c.g->adiabatic);

  double a[75], b[75], cc[225];
  jacobians(c, f, a, b, cc);
  double F[4][15], G[4][15];
  node_flux(c, f, nd, nb, F, G);

  const double dt = c.dt, dtsq_2 = c.dtsq_2;
  double t[4][3][5], u[4][3][5][3], k[3][5][5], m[3][3][5][5];
  for (int be = 0; be < nb; be++)
    for (int i = 0; i < ndim; i++)
      for (int r = 0; r < neqn; r++) t[be][i][r] = -dt * (F[be][i * 5 + r] + G[be][i * 5 + r]);
  for (int be = 0; be < nb; be++)
    for (int j = 0; j < ndim; j++)
      for (int r = 0; r < neqn; r++)
        for (int i = 0; i < ndim; i++) {
          double acc = 0;
          for (int s = 0; s < neqn; s++)
            acc += dtsq_2 * (A3(a, i, r, s) + A3(b, i, r, s)) * (F[be][j * 5 + s] + G[be][j * 5 + s]);
          u[be][j][r][i] = acc;
        }
  for (int i = 0; i < ndim; i++)
    for (int r = 0; r < neqn; r++)
      for (int s = 0; s < neqn; s++) k[i][r][s] = dt * (c.s1 * A3(a, i, r, s) + c.s3 * A3(b, i, r, s));
  for (int i = 0; i < ndim; i++)
    for (int j = 0; j < ndim; j++)
      for (int r = 0; r < neqn; r++)
        for (int s = 0; s < neqn; s++) {
          double acc = 0;
          acc += (dt * c.s3 * C4(cc, i, j, r, s));
          for (int tt = 0; tt < neqn; tt++)
            acc -= dtsq_2 * (c.s2 * (A3(a, i, r, tt) * A3(a, j, tt, s) + A3(b, i, r, tt) * A3(a, j, tt, s)) +
                             c.s4 * ((A3(a, i, r, tt) * A3(b, j, tt, s)) + (A3(b, i, r, tt) * A3(b, j, tt, s))));
          m[i][j][r][s] = acc;
        }
  for (int N = 0; N < nb; N++)
    for (int ir = 0; ir < neqn; ir++) {
      int I = neqn * fn[N] + ir;
      for (int i = 0; i < ndim; i++) {
        for (int be = 0; be < nb; be++) c.rhs[I] += t[be][i][ir] * en[i] * phib[N] * phib[be];
        for (int j = 0; j < ndim; j++)
          for (int be = 0; be < nb; be++) c.rhs[I] += u[be][j][ir][i] * en[i] * phib[N] * dpidx[be][j];
      }
      for (int M = 0; M < nb; M++)
        for (int is = 0; is < neqn; is++) {
          double& Rij = c.Rm(I, neqn * fn[M] + is);
          for (int i = 0; i < ndim; i++) {
            Rij += k[i][ir][is] * phib[N] * phib[M] * en[i];
            for (int j = 0; j < ndim; j++) Rij += m[i][j][ir][is] * dpidx[M][j] * phib[N] * en[i];
          }
        }
    }
}

// FDVParam.h:15-111 ; s_prev carries the previous element's values (kept when no branch fires)
void fdvparam(const Gas& g, NodeState* const* nd, int nnod, int ndim, double* s) {
  double M_min = 0, M_max = 0, Re_min = 0, Re_max = 0;
  for (int be = 0; be < nnod; be++) {
    double vv = 0;
    for (int i = 0; i < ndim; i++) vv += nd[be]->v[i] * nd[be]->v[i];
    double V = std::sqrt(vv);
    double T = nd[be]->T;
    if (T < 1.0E-12) T = 0;
    double a = std::sqrt(g.gamma * g.cgas * T);
    double M = (a < 1.0E-12) ? 0 : V / a;
    double mu = g.mu(T);
    double Re = (nd[be]->rho * V) / mu;
    if (be == 0) { M_max = M; M_min = M; Re_max = Re; Re_min = Re; }
    M_max = std::max(M_max, M);
    M_min = std::min(M_min, M);
    Re_max = std::max(Re_max, Re);
    Re_min = std::min(Re_min, Re);
  }
  const double eps = 0.0000001;
  double r = std::sqrt(std::pow(M_max, 2) - std::pow(M_min, 2)) / (M_min + eps);
  if (r > 0.01) s[0] = std::min(r, 1.0);
  else if (r < 0.01 && M_min >= 10E-10) s[0] = 0;
  else if (M_min < 10E-10) s[0] = 1.0;
  s[1] = 0.5 * (1 + std::pow(s[0], 0.2));
  r = std::sqrt(std::pow(Re_max, 2) - std::pow(Re_min, 2)) / (Re_min + eps);
  if (r > 0.01) s[2] = std::min(r, 1.0);
  else if (r < 0.01 && Re_min >= 10E-10) s[2] = 0.0;
  else if (Re_min <= 10E-10) s[2] = 1.0;
  s[3] = 0.5 * (1 + std::pow(s[2], 0.2));
}

std::vector<NodeState> unpack_all(const oracle_mesh* m, const Gas& g, const double* U) {
  std::vector<NodeState> ns(m->n_nodes);
  for (int n = 0; n < m->n_nodes; n++)
    unpack(g, m->ndim, U + (size_t)n * m->neqn, m->x + (size_t)n * m->ndim, ns[n]);
  return ns;
}

double dotv(const std::vector<double>& a, const double* b) {
  double r = 0;
  for (size_t i = 0; i < a.size(); i++) r += a[i] * b[i];
  return r;
}

}  // namespace

extern "C" {

void oracle_gauss(int n, double* zeta, double* w) { gauss(n, zeta, w); }

void oracle_dirichlet(const oracle_mesh* m, const oracle_aero* a, uint8_t* dir) {
  const int ndim = m->ndim, neqn = m->neqn;
  std::memset(dir, 0, (size_t)m->n_nodes * neqn);
  for (int e = 0; e < m->n_elements; e++)
    for (int f = 0; f < m->nface; f++) {
      int bc = m->bc[(size_t)e * m->nface + f];
      if (bc == 0) continue;
      for (int i = 0; i < m->nbnod; i++) {
        int ln = (ndim == 2) ? kFace2[f][i] : kFace3[f][i];
        uint8_t* d = dir + (size_t)m->conn[(size_t)e * m->nnod + ln] * neqn;
        if (bc == -1 || bc == -12) {
          for (int j = 0; j < neqn; j++) d[j] = 1;
        } else if (bc == 2 || bc == 9) {
          d[ndim] = 1;
        } else if (bc == 22) {
          d[2] = 1;
        } else if (bc == 1 || bc == 11 || bc == 21 || bc == 31 || bc == 41 || bc == 4) {
          for (int j = 0; j < ndim; j++) d[1 + j] = 1;
          if (!a->adiabatic) d[1 + ndim] = 1;
        }
      }
    }
}

void oracle_bc_rowmask(const oracle_mesh* m, const oracle_aero* a, const uint8_t* dir, uint64_t* mask) {
  const int ndim = m->ndim, neqn = m->neqn;
  for (int e = 0; e < m->n_elements; e++) {
    uint64_t mk = 0;
    for (int f = 0; f < m->nface; f++) {
      int bc = m->bc[(size_t)e * m->nface + f];
      if (bc == 0) continue;
      for (int jn = 0; jn < m->nbnod; jn++) {
        int ja = (ndim == 2) ? kFace2[f][jn] : kFace3[f][jn];
        const uint8_t* d = dir + (size_t)m->conn[(size_t)e * m->nnod + ja] * neqn;
        for (int je = 0; je < neqn; je++) {
          if (!d[je]) continue;
          if (bc == 1 && je == neqn - 1 && !a->adiabatic) continue;  // ApplyBC.h:41-63 (the isothermal-wall branch is commented out)
          mk |= 1ull << (neqn * ja + je);
        }
      }
    }
    mask[e] = mk;
  }
}

void oracle_init_U(const oracle_mesh* m, const oracle_aero* a, const double* prim, double* U) {
  Gas g(a);
  const int ndim = m->ndim, neqn = m->neqn, rs = 2 * ndim + 2;
  for (int n = 0; n < m->n_nodes; n++) {
    const double* p = prim + (size_t)n * rs;
    double* u = U + (size_t)n * neqn;
    u[0] = p[ndim];
    for (int j = 0; j < ndim; j++) u[j + 1] = p[ndim + 1 + j];
    u[ndim + 1] = p[2 * ndim + 1] * g.Cv;
    double v = 0;
    for (int j = 0; j < ndim; j++) {
      v += u[j + 1] * u[j + 1];
      u[j + 1] *= u[0];
    }
    u[ndim + 1] += 0.5 * v;
    u[ndim + 1] *= u[0];
  }
}

void oracle_cleng(const oracle_mesh* m, double* cleng) {
  double z[2], w[2];
  gauss(2, z, w);
  oracle_aero dummy = {1.4, 1, 1, 1, 1, 1, 1};
  Gas g(&dummy);
  for (int e = 0; e < m->n_elements; e++) {
    NodeState ns[8];
    NodeState* nd[8];
    for (int N = 0; N < m->nnod; N++) {
      int gi = m->conn[(size_t)e * m->nnod + N];
      for (int k = 0; k < m->ndim; k++) ns[N].x[k] = m->x[(size_t)gi * m->ndim + k];
      nd[N] = &ns[N];
    }
    double area = 0;
    double Phi[8], dPxi[8][3], dPhi[8][3], jac[3][3];
    if (m->ndim == 2) {
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          double zz[2] = {z[i], z[j]};
          shape2(zz, Phi, dPxi);
          double J = jac2(dPxi, nd, jac, dPhi);
          area += w[i] * w[j] * J;
        }
    } else {
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
          for (int k = 0; k < 2; k++) {
            double zz[3] = {z[i], z[j], z[k]};
            shape3(zz, Phi, dPxi);
            double J = jac3(dPxi, nd, dPhi);
            area += w[i] * w[j] * w[k] * J;
          }
    }
    cleng[e] = std::pow(area, 1.0 / (double)m->ndim);
  }
}

double oracle_cfl(const oracle_mesh* m, const oracle_aero* a, const double* cleng, const double* U, double cfl) {
  Gas g(a);
  auto ns = unpack_all(m, g, U);
  double dx_dv = 1000, dt = 0;
  for (int e = 0; e < m->n_elements; e++) {
    double dxele = 1000;
    for (int i = 0; i < m->nnod; i++) {
      const NodeState& n = ns[m->conn[(size_t)e * m->nnod + i]];
      double Temp = 0;
      if (n.T > 10E-10) Temp = n.T;
      double vv = 0;
      for (int k = 0; k < m->ndim; k++) vv += n.v[k] * n.v[k];
      double v = std::sqrt(vv);
      double a_ = std::sqrt(1.4 * g.cgas * Temp);
      if (v + a_ > 10E-10) {
        double dxnode = cleng[e] / (v + a_);
        if (dxnode < dxele) dxele = dxnode;
      }
    }
    if (dxele < dx_dv) {
      dx_dv = dxele;
      dt = cfl * dx_dv;
    }
  }
  return dt;
}

void oracle_fdvparam(const oracle_mesh* m, const oracle_aero* a, const double* U, double* s) {
  Gas g(a);
  auto ns = unpack_all(m, g, U);
  double prev[4] = {0, 0, 0, 0};
  for (int e = 0; e < m->n_elements; e++) {
    NodeState* nd[8];
    for (int N = 0; N < m->nnod; N++) nd[N] = &ns[m->conn[(size_t)e * m->nnod + N]];
    fdvparam(g, nd, m->nnod, m->ndim, prev);
    for (int k = 0; k < 4; k++) s[4 * e + k] = prev[k];
  }
}

void oracle_form(const oracle_mesh* m, const oracle_aero* a, const double* U, double dt, int apply_bc,
                 int physical_3d_flux, double* R, double* rhs) {
  Gas g(a);
  auto ns = unpack_all(m, g, U);
  const int ndim = m->ndim, nnod = m->nnod, neqn = m->neqn, Ke = nnod * neqn;
  std::vector<uint8_t> dir;
  std::vector<uint64_t> mask;
  if (apply_bc) {
    dir.resize((size_t)m->n_nodes * neqn);
    mask.resize(m->n_elements);
    oracle_dirichlet(m, a, dir.data());
    oracle_bc_rowmask(m, a, dir.data(), mask.data());
  }
  ElemCtx c;
  c.g = &g;
  c.ndim = ndim; c.nnod = nnod; c.neqn = neqn; c.nbnod = m->nbnod; c.Ke = Ke;
  c.dt = dt;
  c.dtsq_2 = std::pow(dt, 2.0) / 2.0;
  c.phys3d = physical_3d_flux;
  gauss(2, c.gz, c.gw);
  double sv[4] = {0, 0, 0, 0};
  for (int e = 0; e < m->n_elements; e++) {
    for (int N = 0; N < nnod; N++) c.nd[N] = &ns[m->conn[(size_t)e * nnod + N]];
    const int hi = m->hnm_idx ? m->hnm_idx[e] : -1;
    c.H = (hi >= 0 && m->hnm) ? m->hnm + (size_t)hi * nnod * nnod : nullptr;
    c.R = R + (size_t)e * Ke * Ke;
    c.rhs = rhs + (size_t)e * Ke;
    std::fill(c.R, c.R + (size_t)Ke * Ke, 0.0);
    std::fill(c.rhs, c.rhs + Ke, 0.0);
    fdvparam(g, c.nd, nnod, ndim, sv);
    c.s1 = sv[0]; c.s2 = sv[1]; c.s3 = sv[2]; c.s4 = sv[3];
    const int* bc = m->bc + (size_t)e * m->nface;
    if (ndim == 2) {  // GaussQuad.h:69-86 then :55-66
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          double w[2] = {c.gw[i], c.gw[j]}, z[2] = {c.gz[i], c.gz[j]};
          domain(c, w, z);
        }
      for (int i = 0; i < 2; i++) {
        double w[1] = {c.gw[i]}, z[1] = {c.gz[i]};
        for (int f = 0; f < 4; f++)
          if (bc[f] != 0 && bc[f] < 100) boundary_face(c, w, z, bc[f], kFace2[f]);
      }
    } else {  // GaussQuad.h:89-112 then :69-86
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
          for (int k = 0; k < 2; k++) {
            double w[3] = {c.gw[i], c.gw[j], c.gw[k]}, z[3] = {c.gz[i], c.gz[j], c.gz[k]};
            domain(c, w, z);
          }
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          double w[2] = {c.gw[i], c.gw[j]}, z[2] = {c.gz[i], c.gz[j]};
          for (int f = 0; f < 6; f++)
            if (bc[f] != 0 && bc[f] < 100) boundary_face(c, w, z, bc[f], kFace3[f]);
        }
    }
    if (apply_bc) {  // ApplyBC.h:14-133: Dirichlet rows zeroed, diagonal 0.5, rhs 0
      uint64_t mk = mask[e];
      for (int I = 0; I < Ke; I++) {
        if (!((mk >> I) & 1ull)) continue;
        for (int k = 0; k < Ke; k++) c.Rm(I, k) = 0.;
        c.Rm(I, I) = 0.5;
        c.rhs[I] = 0.;
      }
    }
  }
}

void oracle_compose_rhs(const oracle_mesh* m, const double* rhs, double* b) {
  const int neqn = m->neqn, nnod = m->nnod, Ke = nnod * neqn;
  std::fill(b, b + (size_t)m->n_nodes * neqn, 0.0);
  for (int e = 0; e < m->n_elements; e++)
    for (int i = 0; i < nnod; i++) {
      int gi = m->conn[(size_t)e * nnod + i];
      for (int k = 0; k < neqn; k++) b[(size_t)neqn * gi + k] += rhs[(size_t)e * Ke + neqn * i + k];
    }
}

void oracle_ebe_matvec(const oracle_mesh* m, const double* R, const double* x, double* y) {
  const int neqn = m->neqn, nnod = m->nnod, Ke = nnod * neqn;
  std::fill(y, y + (size_t)m->n_nodes * neqn, 0.0);
  for (int e = 0; e < m->n_elements; e++) {
    const double* Re = R + (size_t)e * Ke * Ke;
    const int* cn = m->conn + (size_t)e * nnod;
    for (int yn = 0; yn < nnod; yn++) {
      int gy = cn[yn];
      for (int xn = 0; xn < nnod; xn++) {
        int gx = cn[xn];
        for (int xx = 0; xx < neqn; xx++)
          for (int yy = 0; yy < neqn; yy++)
            y[(size_t)gx * neqn + xx] += Re[(size_t)(yn * neqn + yy) * Ke + xn * neqn + xx] * x[(size_t)gy * neqn + yy];
      }
    }
  }
}

void oracle_ebe_matvec_t(const oracle_mesh* m, const double* R, const double* x, double* y) {
  const int neqn = m->neqn, nnod = m->nnod, Ke = nnod * neqn;
  std::fill(y, y + (size_t)m->n_nodes * neqn, 0.0);
  for (int e = 0; e < m->n_elements; e++) {
    const double* Re = R + (size_t)e * Ke * Ke;
    const int* cn = m->conn + (size_t)e * nnod;
    for (int j = 0; j < Ke; j++) {
      double acc = 0;
      for (int i = 0; i < Ke; i++) acc += Re[(size_t)j * Ke + i] * x[(size_t)cn[i / neqn] * neqn + i % neqn];
      y[(size_t)cn[j / neqn] * neqn + j % neqn] += acc;
    }
  }
}

int oracle_gmres_ref(const oracle_mesh* m, const double* R, const double* rhs, int mdim, int restart, double* du,
                     oracle_gmres_report* rep) {
  const size_t n = (size_t)m->n_nodes * m->neqn;
  std::vector<double> b(n), Ax(n), r(n), z(n), V(n * (mdim + 1)), Vt(n * (mdim + 1));
  std::vector<double> h((size_t)(mdim + 1) * mdim), gv(mdim + 1), y(mdim);
  auto H = [&](int i, int j) -> double& { return h[(size_t)j * (mdim + 1) + i]; };
  std::fill(du, du + n, 0.0);  // MPI_GMRES.h:136
  oracle_compose_rhs(m, rhs, b.data());
  double bn = std::sqrt(dotv(b, b.data()));
  double tol = bn * 1.0E-9;  // MPI_GMRES.h:140
  if (rep) { rep->tol = tol; rep->bnorm = bn; rep->n_est = 0; rep->n_restarts_run = 0; }
  int mm = mdim;
  for (int gloop = 0; gloop < restart; gloop++) {
    std::fill(V.begin(), V.end(), 0.0);
    std::fill(Vt.begin(), Vt.end(), 0.0);
    std::fill(h.begin(), h.end(), 0.0);
    std::fill(gv.begin(), gv.end(), 0.0);
    std::fill(y.begin(), y.end(), 0.0);
    std::fill(z.begin(), z.end(), 0.0);
    oracle_ebe_matvec(m, R, du, Ax.data());
    for (size_t i = 0; i < n; i++) r[i] = b[i] - Ax[i];
    double mag_r = std::sqrt(dotv(r, r.data()));
    gv[0] = mag_r;
    for (size_t i = 0; i < n; i++) V[i] = r[i] / mag_r;
    for (int j = 0; j < mm; j++) {
      double* vt = Vt.data() + (size_t)(j + 1) * n;
      oracle_ebe_matvec(m, R, V.data() + (size_t)j * n, vt);
      for (int i = 0; i <= j; i++) {  // modified Gram-Schmidt (MPI_GMRES.h:166-174)
        double hij = 0;
        const double* vi = V.data() + (size_t)i * n;
        for (size_t k = 0; k < n; k++) hij += vt[k] * vi[k];
        H(i, j) = hij;
        for (size_t k = 0; k < n; k++) vt[k] -= hij * vi[k];
      }
      double hn = 0;
      for (size_t k = 0; k < n; k++) hn += vt[k] * vt[k];
      H(j + 1, j) = std::sqrt(hn);
      double* vn = V.data() + (size_t)(j + 1) * n;
      for (size_t k = 0; k < n; k++) vn[k] = vt[k] / H(j + 1, j);
      // rotate_and_check(j+1) (MPI_GMRES.h:696-730): c,s from the unrotated h
      int nn = j + 1;
      std::vector<double> hh((size_t)(nn + 1) * nn), gg(nn + 1, 0.0);
      auto HH = [&](int i, int jj) -> double& { return hh[(size_t)jj * (nn + 1) + i]; };
      gg[0] = gv[0];
      for (int i = 0; i < nn + 1; i++)
        for (int jj = 0; jj < nn; jj++) HH(i, jj) = H(i, jj);
      for (int i = 0; i < nn; i++) {
        double mag = std::sqrt(std::pow(H(i, i), 2) + std::pow(H(i + 1, i), 2));
        double c = H(i, i) / mag, s = H(i + 1, i) / mag;
        for (int jj = 0; jj < nn; jj++) {
          double h0 = HH(i, jj), h1 = HH(i + 1, jj);
          HH(i, jj) = c * h0 + s * h1;
          HH(i + 1, jj) = -s * h0 + c * h1;
        }
        gg[i + 1] = -s * gg[i];
        gg[i] = c * gg[i];
      }
      double est = std::abs(gg[nn]);
      if (rep && rep->est) rep->est[rep->n_est] = gg[nn];
      if (rep) rep->n_est++;
      if (est < tol) { mm = j + 1; break; }
    }
    // rotate() (MPI_GMRES.h:733-752)
    for (int i = 0; i < mm; i++) {
      double mag = std::sqrt(std::pow(H(i, i), 2) + std::pow(H(i + 1, i), 2));
      double c = H(i, i) / mag, s = H(i + 1, i) / mag;
      for (int jj = 0; jj < mm; jj++) {
        double h0 = H(i, jj), h1 = H(i + 1, jj);
        H(i, jj) = c * h0 + s * h1;
        H(i + 1, jj) = -s * h0 + c * h1;
      }
      gv[i + 1] = -s * gv[i];
      gv[i] = c * gv[i];
    }
    if (rep && rep->gfinal) rep->gfinal[gloop] = gv[mm];
    // solve() (MPI_GMRES.h:756-780), back substitution as the reference writes it
    for (int j = mm - 1; j >= 0; j--) {
      y[j] = gv[j];
      for (int i = mm - 1; i >= 0; i--)
        if (i != j) y[j] -= H(i, j) * y[i];
      y[j] /= H(j, j);
    }
    for (size_t k = 0; k < n; k++)
      for (int i = 0; i < mm; i++) z[k] += y[i] * V[(size_t)i * n + k];
    for (size_t k = 0; k < n; k++) du[k] += z[k];
    mm = mdim;
    if (rep) rep->n_restarts_run++;
  }
  if (rep) {
    oracle_ebe_matvec(m, R, du, Ax.data());
    double rn = 0;
    for (size_t i = 0; i < n; i++) rn += (b[i] - Ax[i]) * (b[i] - Ax[i]);
    rep->true_rel_res = bn > 0 ? std::sqrt(rn) / bn : 0.0;
  }
  return 0;
}

int oracle_gmres_correct(const oracle_mesh* m, const double* R, const double* rhs, int mdim, int max_restart,
                         double rtol, double* du, oracle_gmres_report* rep) {
  const size_t n = (size_t)m->n_nodes * m->neqn;
  std::vector<double> b(n), Ax(n), r(n), V(n * (mdim + 1)), w(n);
  std::vector<double> h((size_t)(mdim + 1) * mdim), gv(mdim + 1), cs(mdim), sn(mdim), y(mdim);
  auto H = [&](int i, int j) -> double& { return h[(size_t)j * (mdim + 1) + i]; };
  std::fill(du, du + n, 0.0);
  oracle_compose_rhs(m, rhs, b.data());
  double bn = std::sqrt(dotv(b, b.data()));
  if (rep) { rep->tol = bn * rtol; rep->bnorm = bn; rep->n_est = 0; rep->n_restarts_run = 0; }
  if (bn == 0) { if (rep) rep->true_rel_res = 0; return 0; }
  double rel = 1.0;
  for (int gloop = 0; gloop < max_restart; gloop++) {
    oracle_ebe_matvec(m, R, du, Ax.data());
    for (size_t i = 0; i < n; i++) r[i] = b[i] - Ax[i];
    double beta = std::sqrt(dotv(r, r.data()));
    rel = beta / bn;
    if (rel < rtol) break;
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    for (size_t i = 0; i < n; i++) V[i] = r[i] / beta;
    int k_used = 0;
    for (int j = 0; j < mdim; j++) {
      oracle_ebe_matvec(m, R, V.data() + (size_t)j * n, w.data());
      for (int i = 0; i <= j; i++) {
        const double* vi = V.data() + (size_t)i * n;
        double hij = 0;
        for (size_t k = 0; k < n; k++) hij += w[k] * vi[k];
        H(i, j) = hij;
        for (size_t k = 0; k < n; k++) w[k] -= hij * vi[k];
      }
      double hn = std::sqrt(dotv(w, w.data()));
      H(j + 1, j) = hn;
      double* vn = V.data() + (size_t)(j + 1) * n;
      for (size_t k = 0; k < n; k++) vn[k] = (hn > 0) ? w[k] / hn : 0.0;
      for (int i = 0; i < j; i++) {  // apply previous rotations to the new column
        double t0 = cs[i] * H(i, j) + sn[i] * H(i + 1, j);
        H(i + 1, j) = -sn[i] * H(i, j) + cs[i] * H(i + 1, j);
        H(i, j) = t0;
      }
      double den = std::hypot(H(j, j), H(j + 1, j));
      cs[j] = den > 0 ? H(j, j) / den : 1.0;
      sn[j] = den > 0 ? H(j + 1, j) / den : 0.0;
      H(j, j) = den;
      H(j + 1, j) = 0.0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      k_used = j + 1;
      if (rep && rep->est && rep->n_est < max_restart * mdim) rep->est[rep->n_est] = gv[j + 1];
      if (rep) rep->n_est++;
      if (std::abs(gv[j + 1]) < rtol * bn || hn == 0) break;
    }
    for (int i = k_used - 1; i >= 0; i--) {  // textbook back substitution
      double s = gv[i];
      for (int k = i + 1; k < k_used; k++) s -= H(i, k) * y[k];
      y[i] = s / H(i, i);
    }
    for (int i = 0; i < k_used; i++)
      for (size_t k = 0; k < n; k++) du[k] += y[i] * V[(size_t)i * n + k];
    if (rep && rep->gfinal) rep->gfinal[gloop] = gv[k_used];
    if (rep) rep->n_restarts_run++;
  }
  oracle_ebe_matvec(m, R, du, Ax.data());
  double rn = 0;
  for (size_t i = 0; i < n; i++) rn += (b[i] - Ax[i]) * (b[i] - Ax[i]);
  if (rep) rep->true_rel_res = std::sqrt(rn) / bn;
  return 0;
}

int oracle_step(const oracle_mesh* m, const oracle_aero* a, const double* cleng, double cfl, int mdim, int restart,
                int mode, double rtol, int physical_3d_flux, double* U, double* U0, double* dt_out, double* rms,
                oracle_gmres_report* rep) {
  const int neqn = m->neqn, Ke = m->nnod * neqn;
  const size_t n = (size_t)m->n_nodes * neqn;
  double dt = oracle_cfl(m, a, cleng, U, cfl);
  std::vector<double> R((size_t)m->n_elements * Ke * Ke), rhs((size_t)m->n_elements * Ke), du(n);
  oracle_form(m, a, U, dt, 1, physical_3d_flux, R.data(), rhs.data());
  if (mode == 0) oracle_gmres_ref(m, R.data(), rhs.data(), mdim, restart, du.data(), rep);
  else oracle_gmres_correct(m, R.data(), rhs.data(), mdim, restart, rtol, du.data(), rep);
  for (size_t i = 0; i < n; i++) { U0[i] = U[i]; U[i] += du[i]; }  // MPI_GMRES.h:248-252
  for (int k = 0; k < neqn; k++) {  // MPI_RMSError.h:21-52
    double s = 0, s0 = 0;
    for (int nd = 0; nd < m->n_nodes; nd++) {
      s += U[(size_t)nd * neqn + k] * U[(size_t)nd * neqn + k];
      s0 += U0[(size_t)nd * neqn + k] * U0[(size_t)nd * neqn + k];
    }
    rms[k] = (s0 == 0) ? 1 : std::sqrt(s / s0) - 1.0;
  }
  *dt_out = dt;
  return 0;
}

}  // extern "C"
