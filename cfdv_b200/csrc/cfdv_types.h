// Shared parameter structs for the FDV kernels (device code and host set-up).
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define CFDV_HD __host__ __device__
#define CFDV_INLINE __forceinline__
#else
#define CFDV_HD
#define CFDV_INLINE inline
#endif

namespace cfdv {

// Nondimensional gas model of the reference (Thermo::set, FDV/Thermo.h:22-33).  The
// Mach-number-dependent constants Cv, cgas and cmach have the scalar type S, so that the
// adjoint kernels can differentiate through them (GasT<Dual>); the step uses GasT<double>.
template <class S>
struct GasT {
  double gamma, gamm1, gm1d2, gamm3, gm3d2;
  double Pr, csuth;
  S Cv, cgas, cmach;
  double creyn, Twall;
  int adiabatic;
};
using GasParams = GasT<double>;

inline GasParams make_gas(double gamma, double M, double Re, double Pr, double Tinf, double Tw, int adiabatic) {
  GasParams g;
  g.gamma = gamma;
  g.gamm1 = gamma - 1.0;
  g.gm1d2 = (gamma - 1.0) / 2.0;
  g.gamm3 = gamma - 3.0;
  g.gm3d2 = (gamma - 3.0) / 2.0;
  g.Pr = Pr;
  g.csuth = 110.0 / Tinf;
  g.cmach = M;
  g.Cv = 1. / gamma / (gamma - 1.0) / (M * M);
  g.cgas = 1.0 / gamma / (M * M);
  g.creyn = Re;
  g.Twall = Tw;
  g.adiabatic = adiabatic;
  return g;
}

// Gauss-Legendre points and weights by Newton iteration on P_n, as the reference's
// GaussQuad::get_gauss does (FiniteElement/GaussQuad.h:116-159), so the quadrature
// points carry the reference's last-bit values.
inline void gauss_legendre(int N, double* zeta, double* w) {
  const double eps = 3.E-14;
  const int m = (N + 1) / 2;
  for (int i = 1; i <= m; i++) {
    double z = std::cos(3.141592654 * (i - 0.25) / (N + 0.5));
    double z1 = z + 10, p0 = 0, p1 = 0, p2 = 0, p3 = 0;
    while (std::fabs(z - z1) > eps) {
      p1 = 1.0;
      p2 = 0.0;
      for (int j = 1; j <= N; j++) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.) * p3) / j;
      }
      p0 = N * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / p0;
    }
    zeta[i - 1] = -z;
    zeta[N - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * p0 * p0);
    w[N - i] = w[i - 1];
  }
  for (int i = 0; i < N; i++) {
    if (std::fabs(zeta[i]) < eps) zeta[i] = 0.0;
    if (std::fabs(w[i]) < eps) w[i] = 0.0;
  }
}

// Everything the element-formation kernel reads.
struct FormArgs {
  GasParams gas;
  double dt, dtsq_2;
  const double* dt_dev;      // when set, dt is read from device memory (dtsq_2 = dt^2 / 2)
  double gz[2], gw[2];       // 2-point Gauss-Legendre points and weights
  int n_elements;
  int physical_3d_flux;      // 1: evaluate the 3D convective flux the reference drops
  const double* U;           // [Nn][neqn] conserved state
  const double* x;           // [Nn][ndim]
  const int* conn;           // [E][nnod]
  const int* bc;             // [E][nface]
  const uint64_t* rowmask;   // [E] Dirichlet rows after ApplyBC
  const int* hnm_idx;        // [E] row of hnm for an adaptive element, -1 otherwise (or null)
  const double* hnm;         // [n_adaptive][nnod*nnod] Hnm(N, M) at N + nnod*M
  double* R64;               // [E][Ke*Ke] column-major per element (FP64 output) or null
  float* R32;                // [E][Ke*Ke] (FP32 output) or null
  double* rhs;               // [E][Ke]
  double* s_out;             // [E][4] FDV parameters s1..s4 (may be null)
  int* status;               // error flags (non-finite element matrix -> bit 0)
};

}  // namespace cfdv
