// Discrete adjoint and tangent of the FDV step: kernels over the element functionals of
// adjoint.cuh and the host driver of cfdv_vjp, cfdv_jvp, cfdv_element_functional,
// cfdv_wall_force, cfdv_wall_nodes, cfdv_adjoint and cfdv_tangent (include/cfdv_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"
#include "adjoint.cuh"
#include "adjoint_warp.cuh"
#include "kernels.h"

using namespace cfdv;
using cfdv::ctxi::dalloc;
using cfdv::ctxi::dfree;
using cfdv::ctxi::fail;

namespace cfdv {

// forward mode (the JVP, a.mode 1): one thread per (element, row), the row's derivative along
// the tangent (tU, t_dt, t_mach)
template <int NDIM>
__global__ void __launch_bounds__(128) functional_kernel(FunctionalArgs a) {
  constexpr int KE = FormTraits<NDIM>::KE;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = (int)(t / KE), k = (int)(t % KE);
  if (e >= a.n_elements) return;
  a.out[(size_t)e * KE + k] = element_functional<NDIM>(a, e, k).d;
}

// the collectives of warp_vjp: the warp's lanes; task_sync is the block's barrier
struct WarpLanes {
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  __device__ __forceinline__ double sum(double v, int m) const { return v + __shfl_xor_sync(0xffffffffu, v, m); }
  __device__ __forceinline__ bool any(bool p) const { return __any_sync(0xffffffffu, p) != 0; }
  __device__ __forceinline__ void task_sync() const { __syncthreads(); }
};

// reverse mode, one lane per Gauss point: d L_e / d U_e, d dt, d Mach (and L_e); each of the
// block's kVjpWarps warps takes 4 (hex8) or 8 (quad4) elements, its shared state in dynamic
// shared memory
constexpr int kVjpWarps = 5;
template <int NDIM>
__global__ void __launch_bounds__(32 * kVjpWarps, 1) vjp_warp_kernel(FunctionalArgs a) {
  extern __shared__ __align__(16) unsigned char vjp_smem[];
  const int w = (int)threadIdx.x / 32;
  WarpVjpShared<NDIM>& sh = reinterpret_cast<WarpVjpShared<NDIM>*>(vjp_smem)[w];
  WarpLanes L;
  warp_vjp<NDIM>(a, sh, ((int)blockIdx.x * kVjpWarps + w) * WarpVjp<NDIM>::EPW, (int)threadIdx.x % 32, L);
}

template <int NDIM>
cudaError_t launch_vjp_warp(const FunctionalArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(WarpVjpShared<NDIM>) * kVjpWarps;
  static const cudaError_t attr =
      cudaFuncSetAttribute(vjp_warp_kernel<NDIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (attr != cudaSuccess) return attr;
  const int per_block = WarpVjp<NDIM>::EPW * kVjpWarps;
  vjp_warp_kernel<NDIM><<<(unsigned)((a.n_elements + per_block - 1) / per_block), 32 * kVjpWarps, smem, st>>>(a);
  return cudaGetLastError();
}

template <int NDIM>
__global__ void __launch_bounds__(128) force_kernel(ForceArgs a) {
  constexpr int KE = FormTraits<NDIM>::KE;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t / (KE + 1)), k = (int)(t % (KE + 1));
  if (i >= a.n_list) return;
  const Dual F = wall_force_element<NDIM>(a, a.elems[i], k);
  if (k < KE) a.out[(size_t)i * KE + k] = F.d;
  else a.out_mach[i] = F.d;
  if (k == 0) a.out_val[i] = F.v;
}

// scatter the per-list-entry rows of out[n_list][Ke] into the element-major buffer
__global__ void list_to_elements_kernel(const int* elems, int n_list, int ke, const double* in, double* out) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)n_list * ke; t += (long)gridDim.x * blockDim.x)
    out[(size_t)elems[t / ke] * ke + t % ke] = in[t];
}

// block partials of sum(v[0..n)) (fixed order) into partial[blockIdx.x]
__global__ void __launch_bounds__(kRedThreads) sum_kernel(const double* __restrict__ v, int n, double* partial) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += v[i];
  s = block_reduce_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// y += alpha x  and  y += x
__global__ void axpy_kernel(double* y, const double* __restrict__ x, double alpha, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += alpha * x[i];
}
__global__ void sub_kernel(double* out, const double* __restrict__ a, const double* __restrict__ b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] - b[i];
}

// first element-node pair (in flat order e*nnod + i) whose CFL length equals the minimum
template <int NDIM>
__global__ void cfl_argmin_kernel(const double* __restrict__ U, const int* __restrict__ conn,
                                  const double* __restrict__ cleng, int E, GasParams g, double target, int* best) {
  constexpr int NNOD = (NDIM == 2) ? 4 : 8, NEQ = NDIM + 2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
    for (int i = 0; i < NNOD; i++) {
      double dxn;
      if (cfl_node_len<NDIM>(U + (size_t)conn[(size_t)e * NNOD + i] * NEQ, cleng[e], g, &dxn) && dxn == target)
        atomicMin(best, e * NNOD + i);
    }
}

}  // namespace cfdv

// ---------------------------------------------------------------------------------
// host side
namespace {

constexpr int kThreadsFn = 128;

double host_sum(cfdv_ctx* c, const double* d_v, int n, int* rc) {
  sum_kernel<<<kRedBlocks, kRedThreads, 0, c->st>>>(d_v, n, c->d_pa);
  launch_reduce(c->d_pa, c->d_sc + 4, 0, c->st);
  c->launches += 2;
  double v = 0.0;
  cudaError_t e = cudaMemcpyAsync(c->h_pin, c->d_sc + 4, sizeof(double), cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) *rc = fail(c, CFDV_ERR_CUDA, std::string("reduction: ") + cudaGetErrorString(e));
  v = c->h_pin[0];
  return v;
}

EbeArgs ebe_of(cfdv_ctx* c) {
  EbeArgs a;
  a.ndim = c->ndim; a.nnod = c->nnod; a.neqn = c->neqn; a.n_elements = c->n_elements; a.n_dof = c->n_dof;
  a.conn = c->d_conn; a.csr_ptr = c->d_csr_ptr; a.csr_idx = c->d_csr_idx;
  a.R64 = c->d_R64; a.R32 = c->d_R32; a.Y64 = c->d_Y64; a.Y32 = c->d_Y32;
  return a;
}

int ensure_adjoint_buffers(cfdv_ctx* c) {
  int rc;
  const size_t E = c->n_elements, Ke = c->Ke, n = c->n_dof;
  if (!c->d_adj_e && (rc = dalloc(c, &c->d_adj_e, E * (Ke + 3)))) return rc;
  if (!c->d_adj_v && (rc = dalloc(c, &c->d_adj_v, 5 * n))) return rc;
  return CFDV_OK;
}

FunctionalArgs functional_args(cfdv_ctx* c, double dt) {
  FunctionalArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = c->gas;
  a.dt = dt;
  gauss_legendre(2, a.gz, a.gw);
  a.n_elements = c->n_elements;
  a.physical_3d_flux = c->phys3d;
  a.U = c->d_U; a.x = c->d_x; a.conn = c->d_conn; a.bc = c->d_bc; a.rowmask = c->d_mask;
  a.hnm_idx = c->d_hnm_idx; a.hnm = c->d_hnm;
  return a;
}

cudaError_t launch_functional(cfdv_ctx* c, const FunctionalArgs& a) {
  if (a.mode != 1) return cudaErrorInvalidValue;  // the VJP runs through vjp_warp_kernel
  const long threads = (long)c->n_elements * c->Ke;
  const int grid = (int)((threads + kThreadsFn - 1) / kThreadsFn);
  if (c->ndim == 2) functional_kernel<2><<<grid, kThreadsFn, 0, c->st>>>(a);
  else functional_kernel<3><<<grid, kThreadsFn, 0, c->st>>>(a);
  c->launches++;
  return cudaGetLastError();
}

// g = (dr/dU)^T w as a node vector (gather of the element rows), g_dt, g_mach; U, dt current
int vjp_device(cfdv_ctx* c, double dt, const double* d_w, const double* d_du, double* d_g, double* g_dt,
               double* g_mach, double* d_val) {
  int rc = ensure_adjoint_buffers(c);
  if (rc) return rc;
  const size_t E = c->n_elements, Ke = c->Ke;
  FunctionalArgs a = functional_args(c, dt);
  a.dU = d_du;
  a.w = d_w;
  a.out = c->d_adj_e;
  a.out_dt = c->d_adj_e + E * Ke;
  a.out_mach = c->d_adj_e + E * (Ke + 1);
  a.out_val = d_val;
  // reverse mode, one lane per Gauss point: the element's unknowns, dt and the Mach number
  CK(c->ndim == 2 ? launch_vjp_warp<2>(a, c->st) : launch_vjp_warp<3>(a, c->st));
  c->launches++;
  CK(launch_compose_rhs(ebe_of(c), a.out, d_g, c->d_pa, c->st));
  c->launches++;
  rc = CFDV_OK;
  *g_dt = host_sum(c, a.out_dt, (int)E, &rc);
  if (rc) return rc;
  *g_mach = host_sum(c, a.out_mach, (int)E, &rc);
  return rc;
}

// dr = (dr/dU) tU + (dr/ddt) t_dt + (dr/dMach) t_mach as a node vector
int jvp_device(cfdv_ctx* c, double dt, const double* d_du, const double* d_tU, double t_dt, double t_mach,
               double* d_dr) {
  int rc = ensure_adjoint_buffers(c);
  if (rc) return rc;
  FunctionalArgs a = functional_args(c, dt);
  a.mode = 1;
  a.dU = d_du;
  a.tU = d_tU;
  a.t_dt = t_dt;
  a.t_mach = t_mach;
  a.out = c->d_adj_e;
  CK(launch_functional(c, a));
  CK(launch_compose_rhs(ebe_of(c), a.out, d_dr, c->d_pa, c->st));
  c->launches++;
  return CFDV_OK;
}

// elements with a face of the wall code (host list, uploaded on first use per code)
int wall_list(cfdv_ctx* c, int wall_bc) {
  if (c->wall_bc_cached == wall_bc && c->d_wall_elems) return CFDV_OK;
  std::vector<int> bc((size_t)c->n_elements * c->nface);
  CK(cudaMemcpy(bc.data(), c->d_bc, sizeof(int) * bc.size(), cudaMemcpyDeviceToHost));
  std::vector<int> el;
  for (int e = 0; e < c->n_elements; e++)
    for (int f = 0; f < c->nface; f++)
      if (bc[(size_t)e * c->nface + f] == wall_bc) {
        el.push_back(e);
        break;
      }
  int rc;
  if ((rc = dalloc(c, &c->d_wall_elems, el.size()))) return rc;
  if ((rc = dalloc(c, &c->d_wall_buf, std::max<size_t>(1, el.size()) * (c->Ke + 2)))) return rc;
  if (!el.empty()) CK(cudaMemcpy(c->d_wall_elems, el.data(), sizeof(int) * el.size(), cudaMemcpyHostToDevice));
  c->n_wall_elems = (int)el.size();
  c->wall_bc_cached = wall_bc;
  return CFDV_OK;
}

// F_x at the current U; optionally dF/dU as a node vector and dF/dMach
int wall_force_device(cfdv_ctx* c, int wall_bc, double* F, double* d_gradU, double* dF_dmach) {
  int rc = wall_list(c, wall_bc);
  if (rc) return rc;
  if (!c->d_adj_e && (rc = ensure_adjoint_buffers(c))) return rc;
  const int nl = c->n_wall_elems, Ke = c->Ke;
  *F = 0.0;
  if (dF_dmach) *dF_dmach = 0.0;
  if (d_gradU) CK(cudaMemsetAsync(d_gradU, 0, sizeof(double) * c->n_dof, c->st));
  if (nl == 0) return CFDV_OK;
  ForceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = c->gas;
  gauss_legendre(2, a.gz, a.gw);
  a.n_list = nl;
  a.wall_bc = wall_bc;
  a.elems = c->d_wall_elems;
  a.U = c->d_U; a.x = c->d_x; a.conn = c->d_conn; a.bc = c->d_bc;
  a.hnm_idx = c->d_hnm_idx; a.hnm = c->d_hnm;
  a.out = c->d_wall_buf;
  a.out_mach = c->d_wall_buf + (size_t)nl * Ke;
  a.out_val = c->d_wall_buf + (size_t)nl * (Ke + 1);
  const long threads = (long)nl * (Ke + 1);
  const int grid = (int)((threads + kThreadsFn - 1) / kThreadsFn);
  if (c->ndim == 2) force_kernel<2><<<grid, kThreadsFn, 0, c->st>>>(a);
  else force_kernel<3><<<grid, kThreadsFn, 0, c->st>>>(a);
  c->launches++;
  CK(cudaGetLastError());
  *F = host_sum(c, a.out_val, nl, &rc);
  if (rc) return rc;
  if (dF_dmach) {
    *dF_dmach = host_sum(c, a.out_mach, nl, &rc);
    if (rc) return rc;
  }
  if (d_gradU) {
    double* eb = c->d_adj_e;  // element-major rows, zero outside the wall elements
    CK(cudaMemsetAsync(eb, 0, sizeof(double) * c->n_elements * Ke, c->st));
    list_to_elements_kernel<<<kRedBlocks, 256, 0, c->st>>>(c->d_wall_elems, nl, Ke, a.out, eb);
    CK(launch_compose_rhs(ebe_of(c), eb, d_gradU, c->d_pa, c->st));
    c->launches += 2;
  }
  return CFDV_OK;
}

// dt = cfl * CFL length at the arg-min node: the node and d dt / d U there, d dt / d Mach
int cfl_sensitivity(cfdv_ctx* c, double cfl, double dt, int* node, double* ddt_dU, double* ddt_dmach) {
  const double target = dt / cfl;
  int* d_best = (int*)(c->d_sc + 8);
  const int big = 0x7fffffff;
  CK(cudaMemcpyAsync(d_best, &big, sizeof(int), cudaMemcpyHostToDevice, c->st));
  if (c->ndim == 2)
    cfl_argmin_kernel<2><<<kRedBlocks, 256, 0, c->st>>>(c->d_U, c->d_conn, c->d_cleng, c->n_elements, c->gas, target,
                                                       d_best);
  else
    cfl_argmin_kernel<3><<<kRedBlocks, 256, 0, c->st>>>(c->d_U, c->d_conn, c->d_cleng, c->n_elements, c->gas, target,
                                                       d_best);
  c->launches++;
  int best = big;
  CK(cudaMemcpyAsync(&best, d_best, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *node = -1;
  for (int k = 0; k < c->neqn; k++) ddt_dU[k] = 0.0;
  *ddt_dmach = 0.0;
  if (best == big) return CFDV_OK;  // (dt / cfl is attained: cannot happen for a finite dt)
  const int e = best / c->nnod, i = best % c->nnod;
  int n = 0;
  double cl = 0.0, u[5];
  CK(cudaMemcpy(&n, c->d_conn + (size_t)e * c->nnod + i, sizeof(int), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&cl, c->d_cleng + e, sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(u, c->d_U + (size_t)n * c->neqn, sizeof(double) * c->neqn, cudaMemcpyDeviceToHost));
  *node = n;
  for (int dir = 0; dir <= c->neqn; dir++) {
    const GasT<Dual> g = dual_gas(c->gas, dir == c->neqn ? 1.0 : 0.0);
    Dual ud[5], dxn;
    for (int k = 0; k < c->neqn; k++) ud[k] = Dual(u[k], k == dir ? 1.0 : 0.0);
    const bool ok = (c->ndim == 2) ? cfl_node_len<2>(ud, cl, g, &dxn) : cfl_node_len<3>(ud, cl, g, &dxn);
    if (!ok) continue;
    if (dir < c->neqn) ddt_dU[dir] = cfl * dxn.d;
    else *ddt_dmach = cfl * dxn.d;
  }
  return CFDV_OK;
}

int check_opts(cfdv_ctx* c, const cfdv_adjoint_opts* o) {
  if (!o || o->n_steps <= 0 || o->checkpoint_every <= 0 || !(o->cfl > 0) || o->m <= 0 || o->restarts <= 0 ||
      !(o->rtol > 0))
    return fail(c, CFDV_ERR_ARG, "adjoint options: n_steps, checkpoint_every, cfl, m, restarts, rtol must be > 0");
  if (c->h_records.empty()) return fail(c, CFDV_ERR_STATE, "adjoint/tangent runs start from cfdv_load_node_records");
  return CFDV_OK;
}

cfdv_gmres_opts solve_opts(const cfdv_adjoint_opts* o) {
  cfdv_gmres_opts g;
  std::memset(&g, 0, sizeof(g));
  g.mode = CFDV_GMRES_CORRECT;
  g.m = o->m;
  g.restarts = o->restarts;
  g.rtol = o->rtol;
  g.precision = o->precision;
  g.engine = 0;
  g.precond = 1;
  g.orth = 2;  // delayed CGS2
  return g;
}

int reload_initial_state(cfdv_ctx* c) {
  return cfdv_load_node_records(c, c->h_records.data(), (size_t)c->n_nodes);
}

// wall nodes: nodes of faces with the wall code, ascending
std::vector<int> wall_node_ids(cfdv_ctx* c, int wall_bc, int* rc) {
  std::vector<int> bc((size_t)c->n_elements * c->nface), conn((size_t)c->n_elements * c->nnod);
  cudaError_t e1 = cudaMemcpy(bc.data(), c->d_bc, sizeof(int) * bc.size(), cudaMemcpyDeviceToHost);
  cudaError_t e2 = cudaMemcpy(conn.data(), c->d_conn, sizeof(int) * conn.size(), cudaMemcpyDeviceToHost);
  std::vector<int> ids;
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    *rc = fail(c, CFDV_ERR_CUDA, "wall nodes: copy of the mesh failed");
    return ids;
  }
  std::vector<char> on(c->n_nodes, 0);
  for (int e = 0; e < c->n_elements; e++)
    for (int f = 0; f < c->nface; f++)
      if (bc[(size_t)e * c->nface + f] == wall_bc)
        for (int i = 0; i < c->nbnod; i++) on[conn[(size_t)e * c->nnod + face_node(c->ndim, f, i)]] = 1;
  for (int n = 0; n < c->n_nodes; n++)
    if (on[n]) ids.push_back(n);
  *rc = CFDV_OK;
  return ids;
}

// d U0 / d p for the initial state of the node records: rho E = rho (Cv T + |v|^2 / 2)
// (LoadBinary.h:179-196), Cv = 1/(gamma (gamma-1) M^2)
void initial_state_tangent(cfdv_ctx* c, double dmach, const std::vector<int>& wall, const double* dT,
                           std::vector<double>& dU0) {
  const int nd = c->ndim, rs = 2 * nd + 2, ne = c->neqn;
  dU0.assign((size_t)c->n_dof, 0.0);
  const double dCv = -2.0 * c->gas.Cv / c->gas.cmach;
  for (int n = 0; n < c->n_nodes; n++) {
    const double* p = c->h_records.data() + (size_t)n * rs;
    dU0[(size_t)n * ne + ne - 1] = p[nd] * p[2 * nd + 1] * dCv * dmach;
  }
  if (dT)
    for (size_t k = 0; k < wall.size(); k++) {
      const double* p = c->h_records.data() + (size_t)wall[k] * rs;
      dU0[(size_t)wall[k] * ne + ne - 1] += p[nd] * c->gas.Cv * dT[k];
    }
}

}  // namespace

extern "C" {

int cfdv_vjp(cfdv_ctx* c, const double* mu, const double* du, double* gU, double* g_dt, double* g_mach) {
  if (!c || !mu || !du || !gU || !g_dt || !g_mach) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "vjp needs the step's dt: call cfdv_form first");
  cudaSetDevice(c->dev);
  int rc = ensure_adjoint_buffers(c);
  if (rc) return rc;
  const size_t n = c->n_dof;
  double* w = c->d_adj_v;
  double* d = c->d_adj_v + n;
  double* g = c->d_adj_v + 2 * n;
  CK(cudaMemcpyAsync(w, mu, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d, du, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  if ((rc = vjp_device(c, c->dt_formed, w, d, g, g_dt, g_mach, nullptr))) return rc;
  CK(cudaMemcpyAsync(gU, g, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_element_functional(cfdv_ctx* c, const double* mu, const double* du, double* L) {
  if (!c || !mu || !du || !L) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "element functional needs the step's dt: call cfdv_form first");
  cudaSetDevice(c->dev);
  int rc = ensure_adjoint_buffers(c);
  if (rc) return rc;
  const size_t n = c->n_dof;
  double* w = c->d_adj_v;
  double* d = c->d_adj_v + n;
  double* g = c->d_adj_v + 2 * n;
  double* val = c->d_adj_v + 3 * n;  // n_dof >= n_elements for every mesh of quads / hexes
  CK(cudaMemcpyAsync(w, mu, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d, du, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  double gd, gm;
  if ((rc = vjp_device(c, c->dt_formed, w, d, g, &gd, &gm, val))) return rc;
  CK(cudaMemcpyAsync(L, val, sizeof(double) * c->n_elements, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_jvp(cfdv_ctx* c, const double* du, const double* tU, double t_dt, double t_mach, double* dr) {
  if (!c || !du || !tU || !dr) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "jvp needs the step's dt: call cfdv_form first");
  cudaSetDevice(c->dev);
  int rc = ensure_adjoint_buffers(c);
  if (rc) return rc;
  const size_t n = c->n_dof;
  double* d = c->d_adj_v;
  double* t = c->d_adj_v + n;
  double* out = c->d_adj_v + 2 * n;
  CK(cudaMemcpyAsync(d, du, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(t, tU, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  if ((rc = jvp_device(c, c->dt_formed, d, t, t_dt, t_mach, out))) return rc;
  CK(cudaMemcpyAsync(dr, out, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_wall_force(cfdv_ctx* c, int wall_bc, double* F, double* dF_dU, double* dF_dmach) {
  if (!c || !F) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  int rc = ensure_adjoint_buffers(c);
  if (rc) return rc;
  double* g = dF_dU ? c->d_adj_v : nullptr;
  if ((rc = wall_force_device(c, wall_bc, F, g, dF_dmach))) return rc;
  if (dF_dU) CK(cudaMemcpyAsync(dF_dU, g, sizeof(double) * c->n_dof, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_wall_nodes(cfdv_ctx* c, int wall_bc, int* ids, int capacity, int* n) {
  if (!c || !n) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  int rc;
  const std::vector<int> w = wall_node_ids(c, wall_bc, &rc);
  if (rc) return rc;
  *n = (int)w.size();
  if (ids)
    for (int k = 0; k < std::min(capacity, *n); k++) ids[k] = w[k];
  return CFDV_OK;
}

int cfdv_tangent(cfdv_ctx* c, const cfdv_adjoint_opts* o, double dmach, const double* dT_wall, double* J,
                 double* dJ) {
  if (!c || !J || !dJ) return CFDV_ERR_ARG;
  int rc = check_opts(c, o);
  if (rc) return rc;
  cudaSetDevice(c->dev);
  if ((rc = ensure_adjoint_buffers(c))) return rc;
  const std::vector<int> wall = wall_node_ids(c, o->wall_bc, &rc);
  if (rc) return rc;
  const size_t n = c->n_dof;
  double* tU = c->d_adj_v;           // tangent of U
  double* dr = c->d_adj_v + n;       // residual tangent
  double* gF = c->d_adj_v + 2 * n;   // dF/dU
  double* du = c->d_adj_v + 3 * n;   // the step's dU
  std::vector<double> h0;
  initial_state_tangent(c, dmach, wall, dT_wall, h0);
  if ((rc = reload_initial_state(c))) return rc;
  CK(cudaMemcpyAsync(tU, h0.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  const cfdv_gmres_opts so = solve_opts(o);
  std::vector<double> hv(n), hg(n);
  double Jsum = 0.0, dJsum = 0.0;
  for (int step = 0; step < o->n_steps; step++) {
    double dt;
    if ((rc = cfdv_cfl(c, o->cfl, &dt))) return rc;
    int node;
    double ddU[5], ddM;
    if ((rc = cfl_sensitivity(c, o->cfl, dt, &node, ddU, &ddM))) return rc;
    double tdt = ddM * dmach;
    if (node >= 0) {
      CK(cudaMemcpy(hv.data(), tU + (size_t)node * c->neqn, sizeof(double) * c->neqn, cudaMemcpyDeviceToHost));
      for (int k = 0; k < c->neqn; k++) tdt += ddU[k] * hv[k];
    }
    if ((rc = cfdv_form(c, dt, o->precision))) return rc;
    if ((rc = cfdv::ctxi::solve_device(c, &so, nullptr, nullptr, 0))) return rc;
    CK(cudaMemcpyAsync(du, c->d_du, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    if ((rc = jvp_device(c, dt, du, tU, tdt, dmach, dr))) return rc;
    if ((rc = cfdv::ctxi::solve_device(c, &so, nullptr, dr, 0))) return rc;  // d(dU) = A^-1 dr
    axpy_kernel<<<kRedBlocks, 256, 0, c->st>>>(tU, c->d_du, 1.0, (int)n);
    CK(cudaMemcpyAsync(c->d_du, du, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    if ((rc = cfdv_update(c))) return rc;
    double F, dFm;
    if ((rc = wall_force_device(c, o->wall_bc, &F, gF, &dFm))) return rc;
    CK(launch_dot(gF, tU, (int)n, c->d_pa, c->st));
    CK(launch_reduce(c->d_pa, c->d_sc + 5, 0, c->st));
    c->launches += 3;
    double gdot = 0.0;
    CK(cudaMemcpyAsync(&gdot, c->d_sc + 5, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    Jsum += F;
    dJsum += gdot + dFm * dmach;
  }
  *J = Jsum / o->n_steps;
  *dJ = dJsum / o->n_steps;
  return CFDV_OK;
}

// Fit the context's pool of element-matrix sets (FP64, and FP32 for the mixed form) to `want`
// usable sets, while a set fits beside a reserve of free device memory (2 GiB or 5% of the
// device, the larger).  A set is usable when it has the parts the form needs.  Parts a run
// does not use are freed first (sets beyond `want`, FP32 parts in FP64 runs), and in a mixed
// run trailing sets are freed to complete earlier ones.  Returns the number of usable sets.
static int grow_matrix_pool(cfdv_ctx* c, int want, bool mixed) {
  const size_t mat = (size_t)c->n_elements * c->Ke * c->Ke;
  auto drop_last = [&]() {
    dfree(c->adj_pool64.back());
    c->adj_pool64.pop_back();
    if (c->adj_pool32.size() > c->adj_pool64.size()) {
      dfree(c->adj_pool32.back());
      c->adj_pool32.pop_back();
    }
  };
  while ((int)c->adj_pool64.size() > want) drop_last();
  if (!mixed)
    for (auto& p : c->adj_pool32) dfree(p);
  if (!mixed) c->adj_pool32.clear();
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
  const size_t reserve = std::max((size_t)2 << 30, total_b / 20);
  int usable = 0;
  for (int i = 0; i < want; i++) {
    const bool have64 = i < (int)c->adj_pool64.size();
    const bool have32 = !mixed || (i < (int)c->adj_pool32.size() && c->adj_pool32[i]);
    const size_t need = (have64 ? 0 : sizeof(double) * mat) + (have32 ? 0 : sizeof(float) * mat);
    if (need) {
      while (free_b < need + reserve && (int)c->adj_pool64.size() > i + 1) {  // complete set i first
        drop_last();
        cudaMemGetInfo(&free_b, &total_b);
      }
      if (free_b < need + reserve) break;
      if (!have64) {
        double* p = nullptr;
        if (cudaMalloc(&p, sizeof(double) * mat) != cudaSuccess) break;
        c->adj_pool64.push_back(p);
      }
      if (!have32) {
        float* p = nullptr;
        if (cudaMalloc(&p, sizeof(float) * mat) != cudaSuccess) break;
        if (i >= (int)c->adj_pool32.size()) c->adj_pool32.resize(i + 1, nullptr);
        c->adj_pool32[i] = p;
      }
      free_b -= need;
    }
    usable++;
  }
  cudaGetLastError();  // a refused allocation only ends the growth
  return usable;
}

int cfdv_adjoint(cfdv_ctx* c, const cfdv_adjoint_opts* o, cfdv_adjoint_result* res) {
  if (!c || !res) return CFDV_ERR_ARG;
  int rc = check_opts(c, o);
  if (rc) return rc;
  cudaSetDevice(c->dev);
  if ((rc = ensure_adjoint_buffers(c))) return rc;
  const std::vector<int> wall = wall_node_ids(c, o->wall_bc, &rc);
  if (rc) return rc;
  const size_t n = c->n_dof;
  const int N = o->n_steps, k = o->checkpoint_every;
  const int nseg = (N + k - 1) / k;
  // states: nseg checkpoints, the k+1 states of one segment, U_N
  const size_t need = (size_t)(nseg + k + 2) * n;
  if (need > c->adj_state_cap) {
    if ((rc = dalloc(c, &c->d_adj_states, need))) return rc;
    c->adj_state_cap = need;
  }
  double* ckpt = c->d_adj_states;
  double* seg = ckpt + (size_t)nseg * n;
  double* UN = seg + (size_t)(k + 1) * n;
  double* lam = c->d_adj_v;
  double* g = c->d_adj_v + n;
  double* gF = c->d_adj_v + 2 * n;
  double* du = c->d_adj_v + 3 * n;
  double* mu_prev = c->d_adj_v + 4 * n;  // the last reverse step's mu: the next solve's start
  bool have_mu = false;
  const cfdv_gmres_opts so = solve_opts(o);
  // Kept sets of the pool: the last P_rec recomputed steps of a segment form into sets
  // 0 .. P_rec-1 (reused by every segment); the forward run's last step of segment s < P_end
  // forms into set P_rec + s (the recomputation does not reach that step).  Their reverse
  // steps solve with those matrices instead of forming again.  Recompute sets come first when
  // memory is short.  The context's own buffers are restored on every exit.
  const bool mixed = o->precision == CFDV_PREC_MIXED;
  if (mixed && !c->d_R32 && (rc = dalloc(c, &c->d_R32, (size_t)c->n_elements * c->Ke * c->Ke))) return rc;
  int want = std::min(k, N) - 1 + nseg;
  if (o->max_kept_sets < 0) want = 0;
  else if (o->max_kept_sets > 0) want = std::min(want, o->max_kept_sets);
  const int P = grow_matrix_pool(c, want, mixed);
  const int P_rec = std::min(P, std::min(k, N) - 1), P_end = P - P_rec;
  struct OwnMatrices {
    cfdv_ctx* c;
    double* r64;
    float* r32;
    void use(int slot, bool mixed) {
      c->d_R64 = c->adj_pool64[slot];
      c->d_R32 = mixed ? c->adj_pool32[slot] : r32;
    }
    void restore() {
      c->d_R64 = r64;
      c->d_R32 = r32;
    }
    ~OwnMatrices() { restore(); }
  } own{c, c->d_R64, c->d_R32};
  int reverse_forms = 0;
  cudaEvent_t ev[3];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  struct Guard {
    cudaEvent_t* e;
    ~Guard() { for (int i = 0; i < 3; i++) cudaEventDestroy(e[i]); }
  } guard{ev};
  cfdv_gmres_report rep;
  std::memset(&rep, 0, sizeof(rep));
  int fwd_mv = 0, adj_mv = 0;
  // ---- forward run, checkpoints every k steps ----
  if ((rc = reload_initial_state(c))) return rc;
  CK(cudaEventRecord(ev[0], c->st));
  double Jsum = 0.0;
  for (int step = 0; step < N; step++) {
    if (step % k == 0)
      CK(cudaMemcpyAsync(ckpt + (size_t)(step / k) * n, c->d_U, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    rep.n_matvec = 0;
    const int seg = step / k;
    const bool keep_end = seg < P_end && step == std::min((seg + 1) * k, N) - 1;  // segment's last step
    if (keep_end) own.use(P_rec + seg, mixed);
    rc = cfdv_step(c, o->cfl, &so, &rep, nullptr);
    own.restore();
    if (rc) return rc;
    fwd_mv += rep.n_matvec;
    double F;
    if ((rc = wall_force_device(c, o->wall_bc, &F, nullptr, nullptr))) return rc;
    Jsum += F;
  }
  CK(cudaMemcpyAsync(UN, c->d_U, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaEventRecord(ev[1], c->st));
  // ---- backward sweep ----
  double gM = 0.0;
  {
    double F, dFm;
    if ((rc = wall_force_device(c, o->wall_bc, &F, lam, &dFm))) return rc;  // lambda_N = (1/N) dF/dU(U_N)
    CK(cudaMemsetAsync(g, 0, sizeof(double) * n, c->st));
    axpy_kernel<<<kRedBlocks, 256, 0, c->st>>>(g, lam, 1.0 / N, (int)n);
    CK(cudaMemcpyAsync(lam, g, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    gM += dFm / N;
  }
  for (int s = nseg - 1; s >= 0; s--) {
    const int n0 = s * k, n1 = std::min(n0 + k, N);
    // recompute U_{n0} .. U_{n1-1} from the checkpoint; U_{n1} is the next checkpoint or U_N
    CK(cudaMemcpyAsync(c->d_U, ckpt + (size_t)s * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(seg, c->d_U, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    const int first_kept = n1 - 1 - P_rec;  // recomputed steps from here on keep their matrices
    for (int step = n0; step < n1 - 1; step++) {
      rep.n_matvec = 0;
      if (step >= first_kept) own.use(step - first_kept, mixed);
      rc = cfdv_step(c, o->cfl, &so, &rep, nullptr);
      own.restore();
      if (rc) return rc;
      fwd_mv += rep.n_matvec;
      CK(cudaMemcpyAsync(seg + (size_t)(step - n0 + 1) * n, c->d_U, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                         c->st));
    }
    const double* Uend = (s + 1 < nseg) ? ckpt + (size_t)(s + 1) * n : UN;
    CK(cudaMemcpyAsync(seg + (size_t)(n1 - n0) * n, Uend, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
    for (int step = n1 - 1; step >= n0; step--) {
      const double* Un = seg + (size_t)(step - n0) * n;
      CK(cudaMemcpyAsync(c->d_U, Un, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
      sub_kernel<<<kRedBlocks, 256, 0, c->st>>>(du, seg + (size_t)(step - n0 + 1) * n, Un, (int)n);
      c->launches++;
      double dt;
      if ((rc = cfdv_cfl(c, o->cfl, &dt))) return rc;
      const bool kept_rec = step < n1 - 1 && step >= first_kept;  // formed by the recompute
      const bool kept_end = step == n1 - 1 && s < P_end;          // formed by the forward run
      if (kept_rec || kept_end) {
        own.use(kept_rec ? step - first_kept : P_rec + s, mixed);
        c->formed = true;
        c->have32 = mixed;
        c->dt_formed = dt;
      } else {
        if ((rc = cfdv_form(c, dt, o->precision))) return rc;
        reverse_forms++;
      }
      // mu = A^-T lambda, started from the previous reverse step's mu (the GMRES stopping test
      // is relative to ||lambda||, so a close start saves products); no later step reads
      // these matrices, so their blocks stay transposed
      rep.n_matvec = 0;
      rc = cfdv::ctxi::solve_device(c, &so, &rep, lam, cfdv::ctxi::kTransposeKeep, have_mu ? mu_prev : nullptr);
      c->formed = false;  // the context's own buffers hold transposed or older matrices
      own.restore();
      if (rc) return rc;
      CK(cudaMemcpyAsync(mu_prev, c->d_du, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
      have_mu = true;
      adj_mv += rep.n_matvec;
      double g_dt, g_m;
      if ((rc = vjp_device(c, dt, c->d_du, du, g, &g_dt, &g_m, nullptr))) return rc;
      axpy_kernel<<<kRedBlocks, 256, 0, c->st>>>(lam, g, 1.0, (int)n);
      c->launches++;
      int node;
      double ddU[5], ddM;
      if ((rc = cfl_sensitivity(c, o->cfl, dt, &node, ddU, &ddM))) return rc;
      if (node >= 0) {
        double h[5];
        CK(cudaMemcpy(h, lam + (size_t)node * c->neqn, sizeof(double) * c->neqn, cudaMemcpyDeviceToHost));
        for (int q = 0; q < c->neqn; q++) h[q] += g_dt * ddU[q];
        CK(cudaMemcpy(lam + (size_t)node * c->neqn, h, sizeof(double) * c->neqn, cudaMemcpyHostToDevice));
      }
      gM += g_m + g_dt * ddM;
      if (step >= 1) {  // J averages F over U_1 .. U_N
        double F, dFm;
        if ((rc = wall_force_device(c, o->wall_bc, &F, gF, &dFm))) return rc;
        axpy_kernel<<<kRedBlocks, 256, 0, c->st>>>(lam, gF, 1.0 / N, (int)n);
        c->launches++;
        gM += dFm / N;
      }
    }
  }
  CK(cudaEventRecord(ev[2], c->st));
  // ---- parameters of the initial state ----
  std::vector<double> hl(n);
  CK(cudaMemcpyAsync(hl.data(), lam, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  std::vector<double> dU0;
  initial_state_tangent(c, 1.0, wall, nullptr, dU0);
  double dM0 = 0.0;
  for (size_t i = 0; i < n; i++) dM0 += hl[i] * dU0[i];
  res->J = Jsum / N;
  res->dJ_dmach = gM + dM0;
  const int nd = c->ndim, rs = 2 * nd + 2, ne = c->neqn;
  double tw = 0.0;
  res->n_wall_nodes = (int)wall.size();
  for (size_t q = 0; q < wall.size(); q++) {
    const double rho = c->h_records[(size_t)wall[q] * rs + nd];
    const double gT = hl[(size_t)wall[q] * ne + ne - 1] * rho * c->gas.Cv;
    tw += gT;
    if ((int)q < res->wall_capacity) {
      if (res->wall_nodes) res->wall_nodes[q] = wall[q];
      if (res->dJ_dtnode) res->dJ_dtnode[q] = gT;
    }
  }
  res->dJ_dtwall = tw;
  float ms1 = 0, ms2 = 0;
  CK(cudaEventElapsedTime(&ms1, ev[0], ev[1]));
  CK(cudaEventElapsedTime(&ms2, ev[1], ev[2]));
  res->forward_ms = ms1;
  res->backward_ms = ms2;
  res->forward_matvecs = fwd_mv;
  res->adjoint_matvecs = adj_mv;
  res->kept_matrix_sets = P;
  res->reverse_forms = reverse_forms;
  // leave the context at the end of the forward run
  CK(cudaMemcpyAsync(c->d_U, UN, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

}  // extern "C"
