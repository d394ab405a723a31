// Test-only CPU emulation of the element-formation thread block.
//
// Runs the host/device phase functions of cfdv_b200/csrc/formation.cuh thread by
// thread, with each __syncthreads() of the CUDA kernel becoming a phase boundary,
// so the kernel's index arithmetic and algebra can be checked against the oracle
// without a GPU.  Used only by tests/test_form_emulated.py; the product library
// never contains or calls it.
#include <cstring>
#include <vector>

#include "../../cfdv_b200/csrc/formation.cuh"

using namespace cfdv;

template <int NDIM>
static int run(const FormArgs& a) {
  using T = FormTraits<NDIM>;
  int bad = 0;
  FormShared<NDIM>* sh = new FormShared<NDIM>;
  for (int e = 0; e < a.n_elements; e++) {
    std::memset(sh, 0xff, sizeof(*sh));  // garbage in shared memory, as on the device
    for (int t = 0; t < T::THREADS; t++) form_step<NDIM>(0, a, *sh, e, t, &bad);
    const int n = form_nsteps<NDIM>(*sh);
    for (int k = 1; k < n; k++)
      for (int t = 0; t < T::THREADS; t++) form_step<NDIM>(k, a, *sh, e, t, &bad);
  }
  delete sh;
  return bad;
}

// adaptive elements for the following emu_form calls (FormArgs::hnm_idx / hnm), or null
static const int* g_hnm_idx = nullptr;
static const double* g_hnm = nullptr;
extern "C" void emu_set_adaptive(const int* hnm_idx, const double* hnm) {
  g_hnm_idx = hnm_idx;
  g_hnm = hnm;
}

extern "C" int emu_form(int ndim, int n_elements, const double* U, const double* x, const int* conn, const int* bc,
                        const uint64_t* rowmask, double gamma, double M, double Re, double Pr, double Tinf,
                        double Tw, int adiabatic, double dt, int physical_3d_flux, double* R64, float* R32,
                        double* rhs, double* s_out) {
  FormArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = make_gas(gamma, M, Re, Pr, Tinf, Tw, adiabatic);
  a.dt = dt;
  a.dtsq_2 = dt * dt / 2.0;
  gauss_legendre(2, a.gz, a.gw);
  a.n_elements = n_elements;
  a.physical_3d_flux = physical_3d_flux;
  a.U = U; a.x = x; a.conn = conn; a.bc = bc; a.rowmask = rowmask;
  a.hnm_idx = g_hnm_idx; a.hnm = g_hnm;
  a.R64 = R64; a.R32 = R32; a.rhs = rhs; a.s_out = s_out;
  return ndim == 2 ? run<2>(a) : run<3>(a);
}
