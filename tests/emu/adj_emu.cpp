// Test-only CPU build of the adjoint element functionals (cfdv_b200/csrc/adjoint.cuh).
//
// Evaluates, on the host, exactly the per-thread functions the adjoint kernels run on the
// device: the weighted element residual L_e with its dual-number derivative along one seed
// direction, the wall x-force of an element, and the warp reverse sweep (adjoint_warp.cuh,
// one lane per Gauss point) with one fiber per lane.  Used only by tests/test_adjoint_emulated.py
// to check the functionals against the oracle's formation and against finite differences.
#include <ucontext.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../cfdv_b200/csrc/adjoint_warp.cuh"

using namespace cfdv;

// mode 0: out[e*(Ke+2)+k] = d L_e / d(direction k) (k < Ke unknowns, Ke: dt, Ke+1: Mach),
//         val[e] = L_e;   mode 1: out[e*Ke + row] = d r_e(row) along (tU, t_dt, t_mach)
// adaptive elements for the following calls (hnm_idx / hnm of the argument structs), or null
static const int* g_hnm_idx = nullptr;
static const double* g_hnm = nullptr;
extern "C" void emu_set_adaptive(const int* hnm_idx, const double* hnm) {
  g_hnm_idx = hnm_idx;
  g_hnm = hnm;
}
// elements emu_functional evaluates (mask[e] != 0), or null for all; the others get zeros
static const unsigned char* g_elem_mask = nullptr;
extern "C" void emu_set_element_mask(const unsigned char* mask) { g_elem_mask = mask; }

extern "C" void emu_functional(int ndim, int n_elements, const double* U, const double* x, const int* conn,
                               const int* bc, const uint64_t* rowmask, double gamma, double M, double Re, double Pr,
                               double Tinf, double Tw, int adiabatic, double dt, int physical_3d_flux, int mode,
                               const double* dU, const double* w, const double* tU, double t_dt, double t_mach,
                               double* out, double* val) {
  FunctionalArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = make_gas(gamma, M, Re, Pr, Tinf, Tw, adiabatic);
  a.dt = dt;
  gauss_legendre(2, a.gz, a.gw);
  a.n_elements = n_elements;
  a.physical_3d_flux = physical_3d_flux;
  a.mode = mode;
  a.U = U; a.x = x; a.conn = conn; a.bc = bc; a.rowmask = rowmask;
  a.hnm_idx = g_hnm_idx; a.hnm = g_hnm;
  a.dU = dU; a.w = w; a.tU = tU; a.t_dt = t_dt; a.t_mach = t_mach;
  const int Ke = (ndim == 2) ? 16 : 40;
  const int nd = mode == 0 ? Ke + 2 : Ke;
  for (int e = 0; e < n_elements; e++)
    for (int k = 0; k < nd; k++) {
      if (g_elem_mask && !g_elem_mask[e]) {
        out[(size_t)e * nd + k] = 0.0;
        if (k == 0 && val) val[e] = 0.0;
        continue;
      }
      const Dual L = (ndim == 2) ? element_functional<2>(a, e, k) : element_functional<3>(a, e, k);
      out[(size_t)e * nd + k] = L.d;
      if (k == 0 && val) val[e] = L.v;
    }
}

// F_x of each element's wall faces and its gradient: out[e*(Ke+1) + k], k == Ke: Mach
extern "C" void emu_wall_force(int ndim, int n_elements, const double* U, const double* x, const int* conn,
                               const int* bc, double gamma, double M, double Re, double Pr, double Tinf, double Tw,
                               int adiabatic, int wall_bc, double* out, double* val) {
  ForceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = make_gas(gamma, M, Re, Pr, Tinf, Tw, adiabatic);
  gauss_legendre(2, a.gz, a.gw);
  a.wall_bc = wall_bc;
  a.U = U; a.x = x; a.conn = conn; a.bc = bc;
  a.hnm_idx = g_hnm_idx; a.hnm = g_hnm;
  const int Ke = (ndim == 2) ? 16 : 40;
  for (int e = 0; e < n_elements; e++)
    for (int k = 0; k <= Ke; k++) {
      const Dual F = (ndim == 2) ? wall_force_element<2>(a, e, k) : wall_force_element<3>(a, e, k);
      out[(size_t)e * (Ke + 1) + k] = F.d;
      if (k == 0) val[e] = F.v;
    }
}

// ---- the warp reverse sweep (one lane per Gauss point), one fiber per lane --------------------------------
// The 32 lanes run as fibers (ucontext) on the calling thread.  At a collective each lane
// switches to the next one; lane 31 switches back to lane 0, by which time every lane has
// reached the collective.  Each lane counts its collectives, and a lane that reaches the
// end of a round at another count than lane 0 aborts the run (lanes that diverged).
namespace {
struct FiberWarp {
  ucontext_t main_ctx, ctx[32];
  std::vector<char> stack[32];
  long count[32];
  double xch[32];
  void next(int lane) {
    count[lane]++;
    if (lane == 31)
      for (int l = 0; l < 32; l++)
        if (count[l] != count[0]) {
          std::fprintf(stderr, "emu_vjp_warp: lanes diverged at a collective\n");
          std::abort();
        }
    swapcontext(&ctx[lane], &ctx[(lane + 1) % 32]);
  }
};
struct EmuLanes {
  int lane;
  FiberWarp* w;
  void sync() { w->next(lane); }
  double sum(double v, int m) {
    w->xch[lane] = v;
    w->next(lane);
    const double o = w->xch[lane ^ m];
    w->next(lane);
    return v + o;
  }
  void task_sync() {}  // one warp: nothing to meet
  bool any(bool p) {
    w->xch[lane] = p ? 1.0 : 0.0;
    w->next(lane);
    bool r = false;
    for (int l = 0; l < 32; l++) r = r || w->xch[l] != 0.0;
    w->next(lane);
    return r;
  }
};

FiberWarp* g_warp;
const FunctionalArgs* g_args;
int g_ndim;

template <int NDIM>
WarpVjpShared<NDIM>& warp_shared() {
  static WarpVjpShared<NDIM> sh;
  return sh;
}

void lane_main(int lane) {
  EmuLanes L{lane, g_warp};
  const int epw = (g_ndim == 2) ? WarpVjp<2>::EPW : WarpVjp<3>::EPW;
  for (int e0 = 0; e0 < g_args->n_elements; e0 += epw) {
    if (g_ndim == 2) warp_vjp<2>(*g_args, warp_shared<2>(), e0, lane, L);
    else warp_vjp<3>(*g_args, warp_shared<3>(), e0, lane, L);
  }
  // lanes finish in order 0..31; the last returns to the caller
  if (lane < 31) setcontext(&g_warp->ctx[lane + 1]);
  setcontext(&g_warp->main_ctx);
}

void run_warp(const FunctionalArgs& a, int ndim) {
  FiberWarp w;
  g_warp = &w;
  g_args = &a;
  g_ndim = ndim;
  for (int l = 0; l < 32; l++) {
    w.count[l] = 0;
    w.stack[l].resize(1 << 20);
    getcontext(&w.ctx[l]);
    w.ctx[l].uc_stack.ss_sp = w.stack[l].data();
    w.ctx[l].uc_stack.ss_size = w.stack[l].size();
    w.ctx[l].uc_link = nullptr;
    makecontext(&w.ctx[l], (void (*)())lane_main, 1, l);
  }
  swapcontext(&w.main_ctx, &w.ctx[0]);
}
}  // namespace

// out[e*Ke + k] = d L_e / d U_e[k]; out_dt[e], out_mach[e]: d L_e / d dt, d Mach; val[e] = L_e
extern "C" void emu_vjp_warp(int ndim, int n_elements, const double* U, const double* x, const int* conn,
                             const int* bc, const uint64_t* rowmask, double gamma, double M, double Re, double Pr,
                             double Tinf, double Tw, int adiabatic, double dt, int physical_3d_flux, const double* dU,
                             const double* w, double* out, double* out_dt, double* out_mach, double* val) {
  FunctionalArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = make_gas(gamma, M, Re, Pr, Tinf, Tw, adiabatic);
  a.dt = dt;
  gauss_legendre(2, a.gz, a.gw);
  a.n_elements = n_elements;
  a.physical_3d_flux = physical_3d_flux;
  a.U = U; a.x = x; a.conn = conn; a.bc = bc; a.rowmask = rowmask;
  a.hnm_idx = g_hnm_idx; a.hnm = g_hnm;
  a.dU = dU; a.w = w;
  a.out = out; a.out_dt = out_dt; a.out_mach = out_mach; a.out_val = val;
  run_warp(a, ndim);
}
