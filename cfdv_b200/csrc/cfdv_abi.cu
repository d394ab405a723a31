// C ABI of libcfdv_gpu.so: context, mesh preprocessing and the per-step drivers.
// Declarations and the reference interfaces they replace: include/cfdv_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "context.h"
#include "formation.cuh"
#include "gmres_persistent.h"
#include "kernels.h"

using namespace cfdv;
using cfdv::ctxi::dalloc;
using cfdv::ctxi::dfree;
using cfdv::ctxi::fail;

namespace {

void free_all(cfdv_ctx* c) {
  dfree(c->d_x); dfree(c->d_conn); dfree(c->d_bc); dfree(c->d_mask); dfree(c->d_cleng);
  dfree(c->d_csr_ptr); dfree(c->d_csr_idx);
  dfree(c->d_U); dfree(c->d_U0); dfree(c->d_du);
  dfree(c->d_R64); dfree(c->d_R32); dfree(c->d_rhs); dfree(c->d_s); dfree(c->d_Y64); dfree(c->d_Y32);
  dfree(c->d_marks);
  dfree(c->d_V); dfree(c->d_W); dfree(c->d_b); dfree(c->d_pa); dfree(c->d_pb); dfree(c->d_H); dfree(c->d_sc);
  dfree(c->d_y); dfree(c->d_rms); dfree(c->d_status); dfree(c->d_pers); dfree(c->d_pers_int); dfree(c->d_Dinv); dfree(c->d_Z);
  dfree(c->d_pm); dfree(c->d_cfl_count); dfree(c->d_nbr_ptr); dfree(c->d_nbr_idx); c->nbr_blocks = 0;
  dfree(c->d_hnm_idx); dfree(c->d_hnm); c->n_adaptive = 0;
  dfree(c->d_adj_e); dfree(c->d_adj_v); dfree(c->d_adj_states); dfree(c->d_wall_elems); dfree(c->d_wall_buf);
  c->adj_state_cap = 0;
  for (auto& p : c->adj_pool64) dfree(p);
  for (auto& p : c->adj_pool32) dfree(p);
  c->adj_pool64.clear();
  c->adj_pool32.clear();
  c->n_wall_elems = 0;
  c->wall_bc_cached = -1 << 30;
  c->pers_cap = 0;
  if (c->h_pin) cudaFreeHost(c->h_pin);
  c->h_pin = nullptr;
  if (c->h_hist) cudaFreeHost(c->h_hist);
  c->h_hist = nullptr;
  c->h_hist_cap = 0;
  c->m_cap = 0;
  c->formed = false;
  c->have32 = false;
  c->du_valid = false;
}

// Dirichlet flags per DOF from the faces (LoadBinary.h:264-318) and the per-element
// row mask that ApplyBC (ApplyBC.h:14-133) zeroes: rows of face nodes whose DOF is
// flagged, except energy on bc 1 faces of an isothermal wall (its handler is empty).
void build_bc_masks(const cfdv_mesh* m, int adiabatic, std::vector<uint64_t>& mask) {
  const int ndim = m->ndim, nnod = ndim == 2 ? 4 : 8, neqn = ndim + 2, nface = ndim == 2 ? 4 : 6;
  const int nbnod = ndim == 2 ? 2 : 4;
  std::vector<uint8_t> dir((size_t)m->n_nodes * neqn, 0);
  for (int e = 0; e < m->n_elements; e++)
    for (int f = 0; f < nface; f++) {
      const int bc = m->bc[(size_t)e * nface + f];
      if (bc == 0) continue;
      for (int i = 0; i < nbnod; i++) {
        uint8_t* d = dir.data() + (size_t)m->conn[(size_t)e * nnod + face_node(ndim, f, i)] * neqn;
        if (bc == -1 || bc == -12) {
          for (int j = 0; j < neqn; j++) d[j] = 1;
        } else if (bc == 2 || bc == 9) {
          d[ndim] = 1;
        } else if (bc == 22) {
          d[2] = 1;
        } else if (bc == 1 || bc == 11 || bc == 21 || bc == 31 || bc == 41 || bc == 4) {
          for (int j = 0; j < ndim; j++) d[1 + j] = 1;
          if (!adiabatic) d[1 + ndim] = 1;
        }
      }
    }
  mask.assign(m->n_elements, 0ull);
  for (int e = 0; e < m->n_elements; e++) {
    uint64_t mk = 0;
    for (int f = 0; f < nface; f++) {
      const int bc = m->bc[(size_t)e * nface + f];
      if (bc == 0) continue;
      for (int jn = 0; jn < nbnod; jn++) {
        const int ja = face_node(ndim, f, jn);
        const uint8_t* d = dir.data() + (size_t)m->conn[(size_t)e * nnod + ja] * neqn;
        for (int je = 0; je < neqn; je++) {
          if (!d[je]) continue;
          if (bc == 1 && je == neqn - 1 && !adiabatic) continue;
          mk |= 1ull << (neqn * ja + je);
        }
      }
    }
    mask[e] = mk;
  }
}

// element length (CalcLength.h:34-110) and geometry checks: element Jacobian volume
// must be positive (CalcLength.h:61-65) and boundary-face surface Jacobians >= 1e-12
// (calc_TF_norm3D.h:137-144); the reference stops at cin.get() on either.
template <int NDIM>
int element_geometry(cfdv_ctx* c, const cfdv_mesh* m, std::vector<double>& cleng) {
  using T = FormTraits<NDIM>;
  double gz[2], gw[2];
  gauss_legendre(2, gz, gw);
  cleng.resize(m->n_elements);
  for (int e = 0; e < m->n_elements; e++) {
    NodePrim nd[T::NNOD];
    for (int N = 0; N < T::NNOD; N++) {
      const int g = m->conn[(size_t)e * T::NNOD + N];
      if (g < 0 || g >= m->n_nodes)
        return fail(c, CFDV_ERR_MESH, "element " + std::to_string(e) + " references node " + std::to_string(g));
      for (int k = 0; k < NDIM; k++) nd[N].x[k] = m->x[(size_t)g * NDIM + k];
    }
    double area = 0;
    for (int q = 0; q < T::Q; q++) {
      double z[3], w = 1.0, Phi[8], dPxi[8][3], dPhi[8][3], jac[3][3];
      for (int d = 0; d < NDIM; d++) {
        const int bit = (q >> (NDIM - 1 - d)) & 1;
        z[d] = gz[bit];
        w *= gw[bit];
      }
      shape_fn<NDIM>(z, Phi, dPxi);
      const double J = phys_deriv<NDIM>(dPxi, nd, dPhi, jac);
      area += w * J;
    }
    if (!(area > 0))
      return fail(c, CFDV_ERR_MESH, "element " + std::to_string(e) + " has non-positive area/volume " +
                                        std::to_string(area));
    cleng[e] = std::pow(area, 1.0 / (double)NDIM);
    if (NDIM == 3) {
      for (int f = 0; f < 6; f++) {
        const int bc = m->bc[(size_t)e * 6 + f];
        if (bc == 0 || bc >= 100) continue;
        const NodePrim* fn[4];
        for (int i = 0; i < 4; i++) fn[i] = &nd[face_node(3, f, i)];
        double L[3], Mu[3];
        for (int i = 0; i < 3; i++) { L[i] = fn[1]->x[i] - fn[0]->x[i]; Mu[i] = fn[3]->x[i] - fn[0]->x[i]; }
        for (int j = 0; j < 3; j++) {
          L[j] /= std::sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
          Mu[j] /= std::sqrt(Mu[0] * Mu[0] + Mu[1] * Mu[1] + Mu[2] * Mu[2]);
        }
        const double nr[3] = {L[1] * Mu[2] - L[2] * Mu[1], L[2] * Mu[0] - L[0] * Mu[2], L[0] * Mu[1] - L[1] * Mu[0]};
        const double gm[3] = {nr[1] * L[2] - nr[2] * L[1], nr[2] * L[0] - nr[0] * L[2], nr[0] * L[1] - nr[1] * L[0]};
        for (int q = 0; q < 4; q++) {
          const double z[2] = {gz[q >> 1], gz[q & 1]};
          double ph[4], dp[4][3];
          shape_fn<2>(z, ph, dp);
          double dxd[3][2] = {{0, 0}, {0, 0}, {0, 0}};
          for (int N = 0; N < 4; N++)
            for (int i = 0; i < 3; i++)
              for (int j = 0; j < 2; j++) dxd[i][j] += dp[N][j] * fn[N]->x[i];
          double tr[2][2];
          for (int j = 0; j < 2; j++) {
            tr[0][j] = L[0] * dxd[0][j] + L[1] * dxd[1][j] + L[2] * dxd[2][j];
            tr[1][j] = gm[0] * dxd[0][j] + gm[1] * dxd[1][j] + gm[2] * dxd[2][j];
          }
          const double det = tr[0][0] * tr[1][1] - tr[1][0] * tr[0][1];
          if (!(det >= 1.0E-12))
            return fail(c, CFDV_ERR_MESH, "element " + std::to_string(e) + " face " + std::to_string(f) +
                                              " has surface Jacobian " + std::to_string(det));
        }
      }
    }
  }
  return CFDV_OK;
}

int setup_mesh(cfdv_ctx* c, const cfdv_mesh* m) {
  if (!m || (m->ndim != 2 && m->ndim != 3) || m->n_nodes <= 0 || m->n_elements <= 0 || !m->x || !m->conn || !m->bc)
    return fail(c, CFDV_ERR_ARG, "mesh: ndim must be 2 or 3 with nodes, elements and arrays");
  free_all(c);
  c->ndim = m->ndim;
  c->nnod = m->ndim == 2 ? 4 : 8;
  c->neqn = m->ndim + 2;
  c->nbnod = m->ndim == 2 ? 2 : 4;
  c->nface = m->ndim == 2 ? 4 : 6;
  c->n_nodes = m->n_nodes;
  c->n_elements = m->n_elements;
  c->n_dof = m->n_nodes * c->neqn;
  c->Ke = c->nnod * c->neqn;
  std::vector<double> cleng;
  int rc = (m->ndim == 2) ? element_geometry<2>(c, m, cleng) : element_geometry<3>(c, m, cleng);
  if (rc) return rc;
  std::vector<uint64_t> mask;
  build_bc_masks(m, c->gas.adiabatic, mask);
  // node -> (element, local node) CSR, entries in element order
  std::vector<int> ptr(c->n_nodes + 1, 0), idx((size_t)c->n_elements * c->nnod);
  for (size_t k = 0; k < idx.size(); k++) ptr[m->conn[k] + 1]++;
  c->max_valence = 0;
  for (int n = 0; n < c->n_nodes; n++) c->max_valence = std::max(c->max_valence, ptr[n + 1]);
  for (int n = 0; n < c->n_nodes; n++) ptr[n + 1] += ptr[n];
  {
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int e = 0; e < c->n_elements; e++)
      for (int l = 0; l < c->nnod; l++) idx[fill[m->conn[(size_t)e * c->nnod + l]]++] = e * c->nnod + l;
  }
  // neighbour sets of the persistent solve's delayed-CGS2 step (2D; none: grid barriers)
  std::vector<int> nptr, nidx;
  const int nblk = persistent_blocks();
  const bool nbr = persistent_neighbour_sets(c->ndim, c->n_nodes, c->n_elements, m->conn, ptr.data(), idx.data(),
                                             nblk, nptr, nidx);
  const size_t E = c->n_elements, Ke = c->Ke;
  if (nbr && ((rc = dalloc(c, &c->d_nbr_ptr, nptr.size())) || (rc = dalloc(c, &c->d_nbr_idx, nidx.size()))))
    return rc;
  if ((rc = dalloc(c, &c->d_x, (size_t)c->n_nodes * c->ndim)) || (rc = dalloc(c, &c->d_conn, E * c->nnod)) ||
      (rc = dalloc(c, &c->d_bc, E * c->nface)) || (rc = dalloc(c, &c->d_mask, E)) ||
      (rc = dalloc(c, &c->d_cleng, E)) || (rc = dalloc(c, &c->d_csr_ptr, (size_t)c->n_nodes + 1)) ||
      (rc = dalloc(c, &c->d_csr_idx, idx.size())) || (rc = dalloc(c, &c->d_U, (size_t)c->n_dof)) ||
      (rc = dalloc(c, &c->d_U0, (size_t)c->n_dof)) || (rc = dalloc(c, &c->d_du, (size_t)c->n_dof)) ||
      (rc = dalloc(c, &c->d_R64, E * Ke * Ke)) || (rc = dalloc(c, &c->d_rhs, E * Ke)) ||
      (rc = dalloc(c, &c->d_s, E * 4)) || (rc = dalloc(c, &c->d_Y64, E * Ke)) ||
      (rc = dalloc(c, &c->d_Y32, E * Ke)) || (rc = dalloc(c, &c->d_W, (size_t)c->n_dof)) ||
      (rc = dalloc(c, &c->d_b, (size_t)c->n_dof)) || (rc = dalloc(c, &c->d_pa, (size_t)kRedBlocks * 10)) ||
      (rc = dalloc(c, &c->d_pb, (size_t)kRedBlocks * 10)) || (rc = dalloc(c, &c->d_sc, 16)) ||
      (rc = dalloc(c, &c->d_status, 1)) || (rc = dalloc(c, &c->d_rms, 16)) || (rc = dalloc(c, &c->d_cfl_count, 1)))
    return rc;
  CK(cudaMallocHost((void**)&c->h_pin, 4096 * sizeof(double)));
  CK(cudaMemcpyAsync(c->d_x, m->x, sizeof(double) * c->n_nodes * c->ndim, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_conn, m->conn, sizeof(int) * E * c->nnod, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_bc, m->bc, sizeof(int) * E * c->nface, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_mask, mask.data(), sizeof(uint64_t) * E, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_cleng, cleng.data(), sizeof(double) * E, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_csr_ptr, ptr.data(), sizeof(int) * ptr.size(), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_csr_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, c->st));
  if (nbr) {
    CK(cudaMemcpyAsync(c->d_nbr_ptr, nptr.data(), sizeof(int) * nptr.size(), cudaMemcpyHostToDevice, c->st));
    if (!nidx.empty())
      CK(cudaMemcpyAsync(c->d_nbr_idx, nidx.data(), sizeof(int) * nidx.size(), cudaMemcpyHostToDevice, c->st));
    c->nbr_blocks = nblk;
  }
  CK(cudaMemsetAsync(c->d_U, 0, sizeof(double) * c->n_dof, c->st));
  CK(cudaMemsetAsync(c->d_U0, 0, sizeof(double) * c->n_dof, c->st));
  CK(cudaMemsetAsync(c->d_du, 0, sizeof(double) * c->n_dof, c->st));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->st));
  CK(cudaMemsetAsync(c->d_cfl_count, 0, sizeof(unsigned int), c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int ensure_krylov(cfdv_ctx* c, int m) {
  if (m <= 0 || m > 255) return fail(c, CFDV_ERR_ARG, "gmres: m must be in [1, 255]");
  if (m <= c->m_cap) return CFDV_OK;
  int rc;
  if ((rc = dalloc(c, &c->d_V, (size_t)(m + 1) * c->n_dof)) || (rc = dalloc(c, &c->d_H, (size_t)(m + 1) * m + 8)) ||
      (rc = dalloc(c, &c->d_y, (size_t)m + 1)))
    return rc;
  c->m_cap = m;
  return CFDV_OK;
}

EbeArgs ebe_args(cfdv_ctx* c) {
  EbeArgs a;
  a.ndim = c->ndim; a.nnod = c->nnod; a.neqn = c->neqn; a.n_elements = c->n_elements; a.n_dof = c->n_dof;
  a.conn = c->d_conn; a.csr_ptr = c->d_csr_ptr; a.csr_idx = c->d_csr_idx;
  a.R64 = c->d_R64; a.R32 = c->d_R32; a.Y64 = c->d_Y64; a.Y32 = c->d_Y32;
  return a;
}

cudaEvent_t* next_events(cfdv_ctx* c) {
  if (!c->prof) return nullptr;
  if (c->ev_used + 3 > c->ev_pool.size()) return nullptr;
  cudaEvent_t* e = &c->ev_pool[c->ev_used];
  c->ev_used += 3;
  return e;
}

// one EBE product; counts and (when profiling) times it
int matvec(cfdv_ctx* c, int fp32, const double* x, double* out, int mode, const double* b, const double* dotw,
           double* partial, cfdv_gmres_report* rep) {
  cudaEvent_t* ev = next_events(c);
  CK(launch_ebe(ebe_args(c), fp32, 0, x, out, mode, b, dotw, partial, c->st, ev));
  c->launches += 2;
  c->mv_launches++;
  if (ev) {  // element pass: stream R once, gather x (once per DOF at best), write Y
    const double sr = fp32 ? 4.0 : 8.0;
    c->mv_bytes += (double)c->n_elements * c->Ke * c->Ke * sr + (double)c->n_dof * 8.0 +
                   (double)c->n_elements * c->Ke * sr;
    c->mv_full_bytes += (double)c->n_elements * c->Ke * c->Ke * sr + (double)c->n_dof * 16.0;
  }
  if (rep) rep->n_matvec++;
  return CFDV_OK;
}

int read_status(cfdv_ctx* c) {
  int s = 0;
  CK(cudaMemcpyAsync(&s, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (s & STATUS_NONFINITE_MATRIX) return fail(c, CFDV_ERR_NONFINITE, "non-finite entry in an element matrix or rhs");
  return CFDV_OK;
}

// One Arnoldi step j: V_{j+1} from A V_j by modified Gram-Schmidt (MPI_GMRES.h:164-181).
// Leaves h(0..j+1, j) in d_H and copies them to hcol.
int arnoldi_step(cfdv_ctx* c, int fp32, int m, int j, double* hcol, cfdv_gmres_report* rep, bool pc = false) {
  const size_t n = c->n_dof;
  double* V = c->d_V;
  double* pa = c->d_pa;
  double* pb = c->d_pb;
  // right preconditioning: the product acts on z_j = Dinv v_j (written with v_j)
  const double* x = pc ? c->d_Z : V + (size_t)j * n;
  int rc = matvec(c, fp32, x, c->d_W, 0, nullptr, V, pa, rep);  // partial <W, v_0>
  if (rc) return rc;
  double* H = c->d_H + (size_t)j * (m + 1);
  for (int i = 0; i <= j; i++) {
    const double* next = (i < j) ? V + (size_t)(i + 1) * n : nullptr;
    CK(launch_mgs(c->d_W, V + (size_t)i * n, (int)n, pa, H + i, next, pb, c->st));
    c->launches++;
    std::swap(pa, pb);
  }
  CK(launch_normalize(c->d_W, (int)n, pa, H + j + 1, V + (size_t)(j + 1) * n, c->st));
  c->launches++;
  if (pc) {
    CK(launch_block_apply(c->ndim, c->d_Dinv, V + (size_t)(j + 1) * n, c->d_Z, c->n_nodes, c->st));
    c->launches++;
  }
  CK(cudaMemcpyAsync(c->h_pin, H, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int i = 0; i < j + 2; i++) hcol[i] = c->h_pin[i];
  for (int i = 0; i < j + 2; i++)
    if (!std::isfinite(hcol[i])) return fail(c, CFDV_ERR_NONFINITE, "non-finite Hessenberg entry in GMRES");
  return CFDV_OK;
}

// r = b - A x into W with ||r|| (host), v_0 = r / ||r||
int restart_residual(cfdv_ctx* c, int fp32, const double* x, double* beta, cfdv_gmres_report* rep, bool pc = false) {
  int rc = matvec(c, fp32, x, c->d_W, 1, c->d_b, c->d_W, c->d_pa, rep);
  if (rc) return rc;
  CK(launch_normalize(c->d_W, c->n_dof, c->d_pa, c->d_sc + 0, c->d_V, c->st));
  c->launches++;
  if (pc) {
    CK(launch_block_apply(c->ndim, c->d_Dinv, c->d_V, c->d_Z, c->n_nodes, c->st));
    c->launches++;
  }
  CK(cudaMemcpyAsync(c->h_pin, c->d_sc, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *beta = c->h_pin[0];
  return CFDV_OK;
}

int compose_b(cfdv_ctx* c, double* bnorm) {
  CK(launch_compose_rhs(ebe_args(c), c->d_rhs, c->d_b, c->d_pa, c->st));
  CK(launch_reduce(c->d_pa, c->d_sc + 1, 1, c->st));
  c->launches += 2;
  CK(cudaMemcpyAsync(c->h_pin, c->d_sc + 1, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *bnorm = c->h_pin[0];
  return CFDV_OK;
}

int add_combination(cfdv_ctx* c, const std::vector<double>& y, int mm, bool pc = false) {
  for (int i = 0; i < mm; i++) c->h_pin[i] = y[i];
  CK(cudaMemcpyAsync(c->d_y, c->h_pin, sizeof(double) * mm, cudaMemcpyHostToDevice, c->st));
  if (pc) CK(launch_combine_precond(c->ndim, c->d_du, c->d_V, c->n_dof, c->d_y, mm, c->d_Dinv, c->n_nodes, c->st));
  else CK(launch_combine(c->d_du, c->d_V, c->n_dof, c->d_y, mm, c->st));
  c->launches++;
  CK(cudaStreamSynchronize(c->st));  // h_pin is reused by the next read-back
  return CFDV_OK;
}

void push_est(cfdv_gmres_report* rep, double v) {
  if (!rep) return;
  if (rep->est && rep->n_est < rep->est_capacity) rep->est[rep->n_est] = v;
  rep->n_est++;
}

// The reference's GMRES (MPI_GMRES::iterate, MPI_GMRES.h:125-220) with its
// estimate (rotate_and_check :696-730), rotation (:733-752) and back substitution
// (:756-780) carried out on the host in the same arithmetic order.
int gmres_reference(cfdv_ctx* c, const cfdv_gmres_opts* o, cfdv_gmres_report* rep) {
  const int m = o->m;
  int rc = ensure_krylov(c, m);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->d_du, 0, sizeof(double) * c->n_dof, c->st));
  double bnorm;
  if ((rc = compose_b(c, &bnorm))) return rc;
  const double tol = bnorm * 1.0E-9;
  if (rep) { rep->tol = tol; rep->bnorm = bnorm; }
  std::vector<double> h((size_t)(m + 1) * m), g(m + 1), y(m), hcol(m + 2);
  auto H = [&](int i, int j) -> double& { return h[(size_t)j * (m + 1) + i]; };
  for (int gloop = 0; gloop < o->restarts; gloop++) {
    std::fill(h.begin(), h.end(), 0.0);
    std::fill(g.begin(), g.end(), 0.0);
    std::fill(y.begin(), y.end(), 0.0);
    double mag_r;
    if ((rc = restart_residual(c, 0, c->d_du, &mag_r, rep))) return rc;
    g[0] = mag_r;
    int mm = m;
    for (int j = 0; j < m; j++) {
      if ((rc = arnoldi_step(c, 0, m, j, hcol.data(), rep))) return rc;
      for (int i = 0; i < j + 2; i++) H(i, j) = hcol[i];
      // rotate_and_check(j+1): c, s from the unrotated h applied to a rotated copy
      const int nn = j + 1;
      std::vector<double> hh((size_t)(nn + 1) * nn), gg(nn + 1, 0.0);
      auto HH = [&](int i, int jj) -> double& { return hh[(size_t)jj * (nn + 1) + i]; };
      gg[0] = g[0];
      for (int i = 0; i < nn + 1; i++)
        for (int jj = 0; jj < nn; jj++) HH(i, jj) = H(i, jj);
      for (int i = 0; i < nn; i++) {
        const double mag = std::sqrt(std::pow(H(i, i), 2) + std::pow(H(i + 1, i), 2));
        const double cs = H(i, i) / mag, sn = H(i + 1, i) / mag;
        for (int jj = 0; jj < nn; jj++) {
          const double h0 = HH(i, jj), h1 = HH(i + 1, jj);
          HH(i, jj) = cs * h0 + sn * h1;
          HH(i + 1, jj) = -sn * h0 + cs * h1;
        }
        gg[i + 1] = -sn * gg[i];
        gg[i] = cs * gg[i];
      }
      push_est(rep, gg[nn]);
      if (std::abs(gg[nn]) < tol) { mm = j + 1; break; }
    }
    for (int i = 0; i < mm; i++) {  // rotate()
      const double mag = std::sqrt(std::pow(H(i, i), 2) + std::pow(H(i + 1, i), 2));
      const double cs = H(i, i) / mag, sn = H(i + 1, i) / mag;
      for (int jj = 0; jj < mm; jj++) {
        const double h0 = H(i, jj), h1 = H(i + 1, jj);
        H(i, jj) = cs * h0 + sn * h1;
        H(i + 1, jj) = -sn * h0 + cs * h1;
      }
      g[i + 1] = -sn * g[i];
      g[i] = cs * g[i];
    }
    if (rep && rep->gfinal && gloop < rep->gfinal_capacity) rep->gfinal[gloop] = g[mm];
    for (int j = mm - 1; j >= 0; j--) {  // solve(), back substitution as the reference writes it
      y[j] = g[j];
      for (int i = mm - 1; i >= 0; i--)
        if (i != j) y[j] -= H(i, j) * y[i];
      y[j] /= H(j, j);
    }
    if ((rc = add_combination(c, y, mm))) return rc;
    if (rep) rep->n_restarts = gloop + 1;
  }
  return CFDV_OK;
}

// node-block Jacobi inverse from the FP64 element matrices (one pass over them)
// (with rhs: b = gather(rhs) assembled by the same launch)
int build_block_jacobi(cfdv_ctx* c, const double* rhs = nullptr, double* b = nullptr) {
  int rc;
  if (!c->d_Dinv && (rc = dalloc(c, &c->d_Dinv, (size_t)c->n_nodes * c->neqn * c->neqn))) return rc;
  if (!c->d_Z && (rc = dalloc(c, &c->d_Z, (size_t)c->n_dof))) return rc;
  CK(launch_block_jacobi(c->ndim, c->d_csr_ptr, c->d_csr_idx, c->d_R64, c->n_nodes, c->d_Dinv, c->d_status, rhs, b,
                         c->st));
  c->launches++;
  return CFDV_OK;
}

// Restarted GMRES(m) to ||b - A du|| < rtol ||b||: MGS Arnoldi, Givens QR updated per
// column, upper-triangular back substitution.  With MIXED precision the Krylov cycles
// use the FP32 matrices while every restart residual is recomputed with the FP64
// matrices (GMRES-based iterative refinement).
int gmres_correct(cfdv_ctx* c, const cfdv_gmres_opts* o, cfdv_gmres_report* rep) {
  const int m = o->m;
  const int fp32 = (o->precision == CFDV_PREC_MIXED);
  if (fp32 && !c->have32) return fail(c, CFDV_ERR_STATE, "mixed precision needs cfdv_form(..., CFDV_PREC_MIXED)");
  int rc = ensure_krylov(c, m);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->d_du, 0, sizeof(double) * c->n_dof, c->st));
  double bnorm;
  if ((rc = compose_b(c, &bnorm))) return rc;
  const double atol = o->rtol * bnorm;
  if (rep) { rep->tol = atol; rep->bnorm = bnorm; }
  if (bnorm == 0.0) { if (rep) rep->true_rel_res = 0.0; return CFDV_OK; }
  const bool pc = o->precond != 0;
  if (pc && (rc = build_block_jacobi(c))) return rc;
  std::vector<double> h((size_t)(m + 1) * m), g(m + 1), y(m), cs(m), sn(m), hcol(m + 2);
  auto H = [&](int i, int j) -> double& { return h[(size_t)j * (m + 1) + i]; };
  double beta = bnorm;
  bool converged = false;
  for (int gloop = 0; gloop < o->restarts; gloop++) {
    if ((rc = restart_residual(c, 0, c->d_du, &beta, rep, pc))) return rc;  // FP64 residual
    if (!std::isfinite(beta)) return fail(c, CFDV_ERR_NONFINITE, "non-finite GMRES residual");
    if (beta < atol) { converged = true; break; }
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int k = 0;
    for (int j = 0; j < m; j++) {
      if ((rc = arnoldi_step(c, fp32, m, j, hcol.data(), rep, pc))) return rc;
      for (int i = 0; i < j + 2; i++) H(i, j) = hcol[i];
      for (int i = 0; i < j; i++) {
        const double t = cs[i] * H(i, j) + sn[i] * H(i + 1, j);
        H(i + 1, j) = -sn[i] * H(i, j) + cs[i] * H(i + 1, j);
        H(i, j) = t;
      }
      const double den = std::hypot(H(j, j), H(j + 1, j));
      cs[j] = den > 0 ? H(j, j) / den : 1.0;
      sn[j] = den > 0 ? H(j + 1, j) / den : 0.0;
      H(j, j) = den;
      H(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      k = j + 1;
      push_est(rep, g[j + 1]);
      if (std::abs(g[j + 1]) < atol || hcol[j + 1] == 0.0) break;
    }
    for (int i = k - 1; i >= 0; i--) {
      double s = g[i];
      for (int jj = i + 1; jj < k; jj++) s -= H(i, jj) * y[jj];
      y[i] = s / H(i, i);
    }
    if ((rc = add_combination(c, y, k, pc))) return rc;
    if (rep && rep->gfinal && gloop < rep->gfinal_capacity) rep->gfinal[gloop] = g[k];
    if (rep) rep->n_restarts = gloop + 1;
  }
  if (!converged && o->restarts > 0) {
    // residual after the last cycle
    if ((rc = restart_residual(c, 0, c->d_du, &beta, rep))) return rc;
    converged = beta < atol;
  }
  if (rep) rep->true_rel_res = beta / bnorm;
  return CFDV_OK;
}

}  // namespace

// The same textbook solve as gmres_correct, run as one persistent cooperative kernel
// (gmres_persistent.cu): one launch per solve.  solve_launch enqueues the launch and the
// read-back of its results into pinned memory without waiting; solve_finish waits and
// fills the report, so a caller can enqueue more work (the state update of a step) in
// between.  The kernel computes ||b|| itself.
int cfdv::ctxi::solve_launch(cfdv_ctx* c, const cfdv_gmres_opts* o, const double* rhs_vec, int transpose,
                             SolveLaunch* L, const double* x0) {
  const int m = o->m;
  const int fp32 = (o->precision == CFDV_PREC_MIXED);
  if (fp32 && !c->have32) return fail(c, CFDV_ERR_STATE, "mixed precision needs cfdv_form(..., CFDV_PREC_MIXED)");
  int rc = ensure_krylov(c, m);
  if (rc) return rc;
  const int est_cap = std::max(1, m * std::max(o->restarts, 1));
  const int gf_cap = std::max(1, o->restarts);
  // scratch: g, cs, sn, y (m+1 each) | est | gfinal | result(8)
  const size_t need = 4 * (size_t)(m + 1) + est_cap + gf_cap + 8;
  if (need > c->pers_cap) {
    if ((rc = dalloc(c, &c->d_pers, need))) return rc;
    c->pers_cap = need;
  }
  // stop, cycles, err, barrier count | a neighbour-sync flag per block, 32 apart
  const size_t n_int = 32 + 32 * (size_t)persistent_max_blocks();
  if (!c->d_pers_int && (rc = dalloc(c, &c->d_pers_int, n_int))) return rc;
  if (!x0) CK(cudaMemsetAsync(c->d_du, 0, sizeof(double) * c->n_dof, c->st));
  else if (x0 != c->d_du)
    CK(cudaMemcpyAsync(c->d_du, x0, sizeof(double) * c->n_dof, cudaMemcpyDeviceToDevice, c->st));
  // b from the element rhs: assembled by the block-Jacobi launch when there is one
  const bool fuse_b = !rhs_vec && !transpose && o->precond;
  if (rhs_vec) {
    if (rhs_vec != c->d_b)
      CK(cudaMemcpyAsync(c->d_b, rhs_vec, sizeof(double) * c->n_dof, cudaMemcpyDeviceToDevice, c->st));
  } else if (!fuse_b) {
    CK(launch_compose_rhs(ebe_args(c), c->d_rhs, c->d_b, c->d_pa, c->st));
    c->launches++;
  }
  CK(cudaMemsetAsync(c->d_pers_int, 0, sizeof(int) * n_int, c->st));
  PersistentArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n_dof = c->n_dof; a.n_elements = c->n_elements; a.m = m; a.max_restarts = o->restarts;
  a.max_blocks = persistent_max_blocks();
  a.orth = o->orth;
  if (o->orth == 0 || o->orth == 2 || o->orth == 3) {  // two buffers of 128 partial slots
    if (!c->d_pm && (rc = dalloc(c, &c->d_pm, (size_t)persistent_max_blocks() * 256))) return rc;
    a.partm = c->d_pm;
  }
  a.rtol = o->rtol;
  a.conn = c->d_conn; a.csr_ptr = c->d_csr_ptr; a.csr_idx = c->d_csr_idx;
  a.R64 = c->d_R64; a.R32 = c->d_R32; a.Y64 = c->d_Y64; a.Y32 = c->d_Y32;
  a.b = c->d_b; a.du = c->d_du; a.V = c->d_V; a.W = c->d_W; a.part0 = c->d_pa; a.part1 = c->d_pb;
  // A^T: transpose every element block in place (restored after the launch), so the kernel's
  // coalesced row loads stream R_e^T and the block Jacobi inverse is that of A^T
  float* r32 = c->have32 ? c->d_R32 : nullptr;
  if (transpose) {
    CK(launch_transpose_blocks(c->Ke, c->d_R64, r32, c->n_elements, c->st));
    c->launches += r32 ? 2 : 1;
  }
  if (o->precond) {
    if ((rc = fuse_b ? build_block_jacobi(c, c->d_rhs, c->d_b) : build_block_jacobi(c))) {
      if (transpose == 1) launch_transpose_blocks(c->Ke, c->d_R64, r32, c->n_elements, c->st);
      return rc;
    }
    a.Dinv = c->d_Dinv;
    a.Z = c->d_Z;
  }
  a.H = c->d_H;
  double* p = c->d_pers;
  a.g = p; a.cs = p + (m + 1); a.sn = p + 2 * (m + 1); a.y = p + 3 * (m + 1);
  a.est = p + 4 * (m + 1); a.est_capacity = est_cap;
  a.gfinal = a.est + est_cap; a.gfinal_capacity = gf_cap;
  a.result = a.gfinal + gf_cap;
  int* pi = c->d_pers_int;
  a.stop = pi; a.out = pi + 1; a.err = pi + 2;
  a.bar_count = (unsigned int*)(pi + 3);
  a.nbr_ptr = c->d_nbr_ptr; a.nbr_idx = c->d_nbr_idx; a.nbr_blocks = c->nbr_blocks;
  a.nbr_flag = (unsigned int*)(pi + 32);
  a.max_valence = c->max_valence;
  // 3D element pass through the shared-memory ring (default); CFDV_ELEM_RING=0 selects the
  // direct-load pass (same products bit for bit), for comparison
  static const int ring_env = [] {
    const char* v = std::getenv("CFDV_ELEM_RING");
    return (v && v[0] == '0') ? 0 : 1;
  }();
  a.ring = ring_env;
  std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
  if (c->prof) {
    cudaEventCreate(&ev.first);
    cudaEventCreate(&ev.second);
    cudaEventRecord(ev.first, c->st);
  }
  CK(launch_gmres_persistent(c->ndim, fp32, a, c->st));
  if (c->prof) {
    cudaEventRecord(ev.second, c->st);
    c->ev_solve.push_back(ev);
  }
  c->launches++;
  if (transpose == 1) {  // restore the blocks (kTransposeKeep leaves them transposed)
    CK(launch_transpose_blocks(c->Ke, c->d_R64, r32, c->n_elements, c->st));
    c->launches += r32 ? 2 : 1;
  }
  double* hp = c->h_pin + cfdv::ctxi::kPinSolve;
  CK(cudaMemcpyAsync(hp, pi, sizeof(int) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(hp + 4, a.result, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->st));
  // the residual history comes back with the results (est and gfinal are contiguous), so the
  // report needs no copy after the wait
  const size_t nh = (size_t)est_cap + gf_cap;
  if (nh > c->h_hist_cap) {
    if (c->h_hist) cudaFreeHost(c->h_hist);
    c->h_hist = nullptr;
    c->h_hist_cap = 0;
    CK(cudaMallocHost((void**)&c->h_hist, sizeof(double) * nh));
    c->h_hist_cap = nh;
  }
  CK(cudaMemcpyAsync(c->h_hist, a.est, sizeof(double) * nh, cudaMemcpyDeviceToHost, c->st));
  L->h_est = c->h_hist;
  L->h_gfinal = c->h_hist + est_cap;
  L->est = a.est; L->gfinal = a.gfinal; L->est_cap = est_cap; L->gf_cap = gf_cap;
  L->err = a.err; L->fp32 = fp32;
  return CFDV_OK;
}

int cfdv::ctxi::solve_finish(cfdv_ctx* c, const SolveLaunch& L, cfdv_gmres_report* rep) {
  CK(cudaStreamSynchronize(c->st));
  const double* hp = c->h_pin + kPinSolve;
  int hi[8];
  double res[8];
  std::memcpy(hi, hp, sizeof(hi));
  std::memcpy(res, hp + 4, sizeof(res));
  if (hi[2] & 1) return fail(c, CFDV_ERR_CUDA, "persistent GMRES: grid barrier timed out");
  if (hi[2] & 2) return fail(c, CFDV_ERR_NONFINITE, "persistent GMRES: non-finite residual");
  const double bnorm = res[6];
  if (rep) {
    const int nest = (int)res[2];
    rep->tol = res[7];
    rep->bnorm = bnorm;
    rep->n_est = nest;
    rep->n_restarts = hi[1];
    rep->n_matvec += (int)res[3];
    rep->true_rel_res = bnorm > 0.0 ? res[0] / bnorm : 0.0;
    if (rep->est && rep->est_capacity > 0) {
      const int k = std::min(std::min(nest, rep->est_capacity), L.est_cap);
      if (k > 0) std::memcpy(rep->est, L.h_est, sizeof(double) * k);
    }
    if (rep->gfinal && rep->gfinal_capacity > 0) {
      const int k = std::min(std::min(hi[1], rep->gfinal_capacity), L.gf_cap);
      if (k > 0) std::memcpy(rep->gfinal, L.h_gfinal, sizeof(double) * k);
    }
  }
  c->mv_launches += (long)res[3];
  if (c->prof) {  // algorithmic bytes: each product streams the matrices once, reads x, writes y
    const double sr = L.fp32 ? 4.0 : 8.0, E = c->n_elements, K2 = (double)c->Ke * c->Ke, n8 = 8.0 * c->n_dof;
    c->solve_bytes += res[4] * (E * K2 * 8.0 + 2 * n8) + (res[3] - res[4]) * (E * K2 * sr + 2 * n8) + res[5] * n8;
  }
  c->du_valid = true;  // a finite solution: a start for a warm-started solve
  return CFDV_OK;
}

int cfdv::ctxi::solve_device(cfdv_ctx* c, const cfdv_gmres_opts* o, cfdv_gmres_report* rep, const double* rhs_vec,
                             int transpose, const double* x0) {
  SolveLaunch L;
  const int rc = solve_launch(c, o, rhs_vec, transpose, &L, x0);
  return rc ? rc : solve_finish(c, L, rep);
}

namespace {

int true_residual(cfdv_ctx* c, cfdv_gmres_report* rep) {
  double beta;
  int rc = matvec(c, 0, c->d_du, c->d_W, 1, c->d_b, c->d_W, c->d_pa, nullptr);
  if (rc) return rc;
  CK(launch_reduce(c->d_pa, c->d_sc + 3, 1, c->st));
  c->launches++;
  CK(cudaMemcpyAsync(c->h_pin, c->d_sc + 3, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  beta = c->h_pin[0];
  if (rep) rep->true_rel_res = rep->bnorm > 0 ? beta / rep->bnorm : 0.0;
  return CFDV_OK;
}

}  // namespace

extern "C" {

int cfdv_create(const cfdv_mesh* mesh, const cfdv_params* p, cfdv_ctx** out) {
  if (!out || !p) return CFDV_ERR_ARG;
  *out = nullptr;
  cfdv_ctx* c = new (std::nothrow) cfdv_ctx();
  if (!c) return CFDV_ERR_ALLOC;
  if (cudaGetDevice(&c->dev) != cudaSuccess) {
    delete c;
    return CFDV_ERR_CUDA;
  }
  if (!(p->gamma > 1.0) || p->mach <= 0 || p->reynolds <= 0 || p->prandtl <= 0 || p->tinf <= 0) {
    delete c;
    return CFDV_ERR_ARG;
  }
  c->gas = make_gas(p->gamma, p->mach, p->reynolds, p->prandtl, p->tinf, p->twall, p->adiabatic);
  c->phys3d = p->physical_3d_flux;
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return CFDV_ERR_CUDA;
  }
  int rc = setup_mesh(c, mesh);
  if (rc) {
    *out = c;  // keep the context so the caller can read cfdv_last_error
    return rc;
  }
  *out = c;
  return CFDV_OK;
}

int cfdv_upload_mesh(cfdv_ctx* c, const cfdv_mesh* mesh) {
  if (!c) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  return setup_mesh(c, mesh);
}

int cfdv_set_adaptive(cfdv_ctx* c, int n, const int* elements, const double* hnm) {
  if (!c || n < 0 || (n > 0 && (!elements || !hnm))) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  dfree(c->d_hnm_idx);
  dfree(c->d_hnm);
  c->n_adaptive = 0;
  if (n == 0) return CFDV_OK;
  const size_t nn = (size_t)c->nnod * c->nnod;
  std::vector<int> idx((size_t)c->n_elements, -1);
  for (int k = 0; k < n; k++) {
    const int e = elements[k];
    if (e < 0 || e >= c->n_elements) return fail(c, CFDV_ERR_ARG, "set_adaptive: element id out of range");
    if (idx[e] >= 0) return fail(c, CFDV_ERR_ARG, "set_adaptive: element listed twice");
    idx[e] = k;
    for (size_t i = 0; i < nn; i++)
      if (!std::isfinite(hnm[(size_t)k * nn + i])) return fail(c, CFDV_ERR_ARG, "set_adaptive: non-finite Hnm entry");
  }
  int rc;
  if ((rc = dalloc(c, &c->d_hnm_idx, idx.size())) || (rc = dalloc(c, &c->d_hnm, (size_t)n * nn))) return rc;
  CK(cudaMemcpyAsync(c->d_hnm_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_hnm, hnm, sizeof(double) * n * nn, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->n_adaptive = n;
  return CFDV_OK;
}

void cfdv_destroy(cfdv_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  for (auto& e : c->ev_form) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  for (auto& e : c->ev_solve) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  free_all(c);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

const char* cfdv_last_error(const cfdv_ctx* c) { return c ? c->err.c_str() : "null context"; }

int cfdv_get_stream(cfdv_ctx* c, void** s) {
  if (!c || !s) return CFDV_ERR_ARG;
  *s = (void*)c->st;
  return CFDV_OK;
}

int cfdv_set_state(cfdv_ctx* c, const double* U, size_t n) {
  if (!c || !U || n != (size_t)c->n_dof) return fail(c, CFDV_ERR_ARG, "set_state: size must be n_nodes*neqn");
  cudaSetDevice(c->dev);
  CK(cudaMemcpyAsync(c->d_U, U, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_load_node_records(cfdv_ctx* c, const double* rec, size_t n_nodes) {
  if (!c || !rec || n_nodes != (size_t)c->n_nodes) return fail(c, CFDV_ERR_ARG, "load_node_records: size");
  const int nd = c->ndim, rs = 2 * nd + 2, ne = c->neqn;
  std::vector<double> U((size_t)c->n_dof);
  for (size_t n = 0; n < n_nodes; n++) {  // LoadBinary.h:179-196
    const double* p = rec + n * rs;
    double* u = U.data() + n * ne;
    u[0] = p[nd];
    for (int j = 0; j < nd; j++) u[j + 1] = p[nd + 1 + j];
    u[nd + 1] = p[2 * nd + 1] * c->gas.Cv;
    double v = 0;
    for (int j = 0; j < nd; j++) {
      v += u[j + 1] * u[j + 1];
      u[j + 1] *= u[0];
    }
    u[nd + 1] += 0.5 * v;
    u[nd + 1] *= u[0];
  }
  if (c->h_records.data() != rec) c->h_records.assign(rec, rec + n_nodes * rs);
  return cfdv_set_state(c, U.data(), U.size());
}

int cfdv_get_state(cfdv_ctx* c, double* U, double* U0, size_t n) {
  if (!c || n != (size_t)c->n_dof) return fail(c, CFDV_ERR_ARG, "get_state: size must be n_nodes*neqn");
  cudaSetDevice(c->dev);
  if (U) CK(cudaMemcpyAsync(U, c->d_U, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  if (U0) CK(cudaMemcpyAsync(U0, c->d_U0, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_state_device_ptr(cfdv_ctx* c, double** U) {
  if (!c || !U) return CFDV_ERR_ARG;
  *U = c->d_U;
  return CFDV_OK;
}

int cfdv_cfl(cfdv_ctx* c, double cfl, double* dt) {
  if (!c || !dt) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(launch_cfl(c->ndim, c->d_U, c->d_conn, c->d_cleng, c->n_elements, c->gas, cfl, c->d_pa, c->d_cfl_count,
                kRedBlocks, c->d_sc + 2, c->st));
  c->launches++;
  CK(cudaMemcpyAsync(c->h_pin, c->d_sc + 2, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *dt = c->h_pin[0];
  if (!(*dt > 0) || !std::isfinite(*dt)) return fail(c, CFDV_ERR_NONFINITE, "CFL: no finite positive time step");
  return CFDV_OK;
}

}  // extern "C"

namespace {

// formation launch without the status read-back; dt_dev (device) overrides dt when set
int form_enqueue(cfdv_ctx* c, double dt, const double* dt_dev, int precision) {
  if (precision == CFDV_PREC_MIXED && !c->d_R32) {
    int rc = dalloc(c, &c->d_R32, (size_t)c->n_elements * c->Ke * c->Ke);
    if (rc) return rc;
  }
  FormArgs a;
  std::memset(&a, 0, sizeof(a));
  a.gas = c->gas;
  a.dt = dt;
  a.dtsq_2 = std::pow(dt, 2.0) / 2.0;
  a.dt_dev = dt_dev;
  gauss_legendre(2, a.gz, a.gw);
  a.n_elements = c->n_elements;
  a.physical_3d_flux = c->phys3d;
  a.U = c->d_U; a.x = c->d_x; a.conn = c->d_conn; a.bc = c->d_bc; a.rowmask = c->d_mask;
  a.hnm_idx = c->d_hnm_idx; a.hnm = c->d_hnm;
  a.R64 = c->d_R64;
  a.R32 = (precision == CFDV_PREC_MIXED) ? c->d_R32 : nullptr;
  a.rhs = c->d_rhs; a.s_out = c->d_s; a.status = c->d_status;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->st));
  std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
  if (c->prof) {
    cudaEventCreate(&ev.first);
    cudaEventCreate(&ev.second);
    cudaEventRecord(ev.first, c->st);
  }
  CK(launch_form(c->ndim, a, c->st));
  c->launches++;
  if (c->prof) {
    cudaEventRecord(ev.second, c->st);
    c->ev_form.push_back(ev);
  }
  c->formed = true;
  c->have32 = (precision == CFDV_PREC_MIXED);
  c->dt_formed = dt;
  return CFDV_OK;
}

}  // namespace

extern "C" {

int cfdv_form(cfdv_ctx* c, double dt, int precision) {
  if (!c) return CFDV_ERR_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return fail(c, CFDV_ERR_ARG, "form: dt must be positive and finite");
  cudaSetDevice(c->dev);
  const int rc = form_enqueue(c, dt, nullptr, precision);
  return rc ? rc : read_status(c);
}

int cfdv_set_element_matrices(cfdv_ctx* c, const double* R, const double* rhs, int precision) {
  if (!c || !R || !rhs) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  const size_t E = c->n_elements, Ke = c->Ke;
  CK(cudaMemcpyAsync(c->d_R64, R, sizeof(double) * E * Ke * Ke, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_rhs, rhs, sizeof(double) * E * Ke, cudaMemcpyHostToDevice, c->st));
  if (precision == CFDV_PREC_MIXED) {
    if (!c->d_R32) {
      int rc = dalloc(c, &c->d_R32, E * Ke * Ke);
      if (rc) return rc;
    }
    CK(launch_to_float(c->d_R64, c->d_R32, E * Ke * Ke, c->st));
    c->launches++;
  }
  CK(cudaStreamSynchronize(c->st));
  c->formed = true;
  c->have32 = (precision == CFDV_PREC_MIXED);
  return CFDV_OK;
}

int cfdv_gmres(cfdv_ctx* c, const cfdv_gmres_opts* o, cfdv_gmres_report* rep) {
  if (!c || !o) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "gmres before form");
  if (o->m <= 0 || o->restarts < 0) return fail(c, CFDV_ERR_ARG, "gmres: m > 0, restarts >= 0");
  cudaSetDevice(c->dev);
  if (rep) { rep->n_est = 0; rep->n_restarts = 0; rep->n_matvec = 0; rep->true_rel_res = -1.0; }
  int rc;
  if (o->mode == CFDV_GMRES_REFERENCE) {
    if (o->precision != CFDV_PREC_FP64) return fail(c, CFDV_ERR_ARG, "reference GMRES runs in FP64 only");
    rc = gmres_reference(c, o, rep);
  } else if (o->engine == 1) {
    rc = gmres_correct(c, o, rep);
  } else {
    rc = cfdv::ctxi::solve_device(c, o, rep, nullptr, 0, (o->warm_start && c->du_valid) ? c->d_du : nullptr);
  }
  if (rc) return rc;
  if (o->true_residual && rep && o->mode == CFDV_GMRES_REFERENCE) rc = true_residual(c, rep);
  return rc;
}

int cfdv_update(cfdv_ctx* c) {
  if (!c) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(launch_state_update(c->d_U, c->d_U0, c->d_du, c->n_dof, c->st));
  c->launches++;
  return CFDV_OK;
}

int cfdv_rms(cfdv_ctx* c, double* rms) {
  if (!c || !rms) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(launch_rms_partial(c->d_U, c->d_U0, c->n_nodes, c->neqn, c->d_pa, c->st));
  c->launches++;
  std::vector<double> part((size_t)kRedBlocks * 10);
  CK(cudaMemcpyAsync(part.data(), c->d_pa, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int k = 0; k < c->neqn; k++) {
    double s = 0, s0 = 0;
    for (int b = 0; b < kRedBlocks; b++) { s += part[(size_t)b * 10 + k]; s0 += part[(size_t)b * 10 + 5 + k]; }
    rms[k] = (s0 == 0) ? 1.0 : std::sqrt(s / s0) - 1.0;
  }
  return CFDV_OK;
}

int cfdv_step(cfdv_ctx* c, double cfl, const cfdv_gmres_opts* o, cfdv_gmres_report* rep, double* dt) {
  return cfdv_step_host(c, cfl, o, rep, dt, nullptr, nullptr);
}

int cfdv_step_host(cfdv_ctx* c, double cfl, const cfdv_gmres_opts* o, cfdv_gmres_report* rep, double* dt,
                   const double* U_in, double* U_out) {
  if (!c || !o) return CFDV_ERR_ARG;
  int rc;
  if (o->mode == CFDV_GMRES_REFERENCE || o->engine == 1) {  // host-driven solvers
    if (U_in && (rc = cfdv_set_state(c, U_in, (size_t)c->n_dof))) return rc;
    double d;
    rc = cfdv_cfl(c, cfl, &d);
    if (!rc) rc = cfdv_form(c, d, o->precision);
    if (!rc) rc = cfdv_gmres(c, o, rep);
    if (!rc) rc = cfdv_update(c);
    if (U_out) {
      const int rc2 = cfdv_get_state(c, U_out, nullptr, (size_t)c->n_dof);
      if (!rc) rc = rc2;
    }
    if (rc) return rc;
    if (dt) *dt = d;
    return CFDV_OK;
  }
  // persistent solve: CFL, formation (dt read on the device), solve and state update are
  // enqueued back to back and the host waits once; the update skips itself on the device
  // when dt, the formation or the solve failed, and the errors are reported in that order
  if (o->m <= 0 || o->restarts < 0) return fail(c, CFDV_ERR_ARG, "gmres: m > 0, restarts >= 0");
  cudaSetDevice(c->dev);
  if (rep) { rep->n_est = 0; rep->n_restarts = 0; rep->n_matvec = 0; rep->true_rel_res = -1.0; }
  if (U_in) CK(cudaMemcpyAsync(c->d_U, U_in, sizeof(double) * c->n_dof, cudaMemcpyHostToDevice, c->st));
  double* d_dt = c->d_sc + 2;
  CK(launch_cfl(c->ndim, c->d_U, c->d_conn, c->d_cleng, c->n_elements, c->gas, cfl, c->d_pa, c->d_cfl_count,
                kRedBlocks, d_dt, c->st));
  c->launches++;
  // a failure before the update is enqueued leaves the state as it was: hand it back in U_out
  // as the host-driven branch does
  auto unchanged_out = [&](int code) {
    if (U_out) {
      if (cudaMemcpyAsync(U_out, c->d_U, sizeof(double) * c->n_dof, cudaMemcpyDeviceToHost, c->st) == cudaSuccess)
        cudaStreamSynchronize(c->st);
      cudaGetLastError();
    }
    return code;
  };
  if ((rc = form_enqueue(c, 0.0, d_dt, o->precision))) return unchanged_out(rc);
  cfdv::ctxi::SolveLaunch L;
  if ((rc = cfdv::ctxi::solve_launch(c, o, nullptr, 0, &L, (o->warm_start && c->du_valid) ? c->d_du : nullptr)))
    return unchanged_out(rc);
  CK(launch_state_update_guarded(c->d_U, c->d_U0, c->d_du, c->n_dof, L.err, c->d_status, d_dt, c->st));
  c->launches++;
  double* hs = c->h_pin + cfdv::ctxi::kPinStep;
  CK(cudaMemcpyAsync(hs, d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(hs + 1, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  if (U_out) CK(cudaMemcpyAsync(U_out, c->d_U, sizeof(double) * c->n_dof, cudaMemcpyDeviceToHost, c->st));
  rc = cfdv::ctxi::solve_finish(c, L, rep);  // waits for the stream
  const double d = hs[0];
  int status;
  std::memcpy(&status, hs + 1, sizeof(int));
  if (!(d > 0) || !std::isfinite(d)) return fail(c, CFDV_ERR_NONFINITE, "CFL: no finite positive time step");
  c->dt_formed = d;
  if (status & STATUS_NONFINITE_MATRIX) return fail(c, CFDV_ERR_NONFINITE, "non-finite entry in an element matrix or rhs");
  if (rc) return rc;
  if (dt) *dt = d;
  return CFDV_OK;
}

int cfdv_get_fdv_params(cfdv_ctx* c, double* s) {
  if (!c || !s) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "fdv params before form");
  cudaSetDevice(c->dev);
  CK(cudaMemcpyAsync(s, c->d_s, sizeof(double) * 4 * c->n_elements, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_get_element_matrices(cfdv_ctx* c, double* R, double* rhs) {
  if (!c) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "element matrices before form");
  cudaSetDevice(c->dev);
  const size_t E = c->n_elements, Ke = c->Ke;
  if (R) CK(cudaMemcpyAsync(R, c->d_R64, sizeof(double) * E * Ke * Ke, cudaMemcpyDeviceToHost, c->st));
  if (rhs) CK(cudaMemcpyAsync(rhs, c->d_rhs, sizeof(double) * E * Ke, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_refine_marks(cfdv_ctx* c, double threshold, int* elements, int capacity, int* n) {
  if (!c || !n || capacity < 0 || (capacity > 0 && !elements)) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  int rc;
  if (!c->d_marks && (rc = dalloc(c, &c->d_marks, (size_t)c->n_elements))) return rc;
  CK(launch_refine_marks(c->ndim, c->d_U, c->d_x, c->d_conn, c->n_elements, c->gas, threshold, c->d_marks, c->st));
  c->launches++;
  std::vector<unsigned char> flags((size_t)c->n_elements);
  CK(cudaMemcpyAsync(flags.data(), c->d_marks, flags.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  int k = 0;
  for (int e = 0; e < c->n_elements; e++)
    if (flags[(size_t)e]) {
      if (k < capacity) elements[k] = e;
      k++;
    }
  *n = k;
  return CFDV_OK;
}

int cfdv_get_element_subset(cfdv_ctx* c, int n, const int* ids, double* R, double* rhs, double* s) {
  if (!c || n < 0 || (n > 0 && !ids)) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "element matrices before form");
  for (int k = 0; k < n; k++)
    if (ids[k] < 0 || ids[k] >= c->n_elements) return fail(c, CFDV_ERR_ARG, "element subset: id out of range");
  cudaSetDevice(c->dev);
  const size_t Ke = c->Ke;
  // one copy per element and array: meant for a few hundred elements at most
  for (int k = 0; k < n; k++) {
    const size_t e = (size_t)ids[k];
    if (R) CK(cudaMemcpyAsync(R + k * Ke * Ke, c->d_R64 + e * Ke * Ke, sizeof(double) * Ke * Ke,
                              cudaMemcpyDeviceToHost, c->st));
    if (rhs) CK(cudaMemcpyAsync(rhs + k * Ke, c->d_rhs + e * Ke, sizeof(double) * Ke, cudaMemcpyDeviceToHost, c->st));
    if (s) CK(cudaMemcpyAsync(s + 4 * k, c->d_s + 4 * e, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_get_rhs_vector(cfdv_ctx* c, double* b) {
  if (!c || !b) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "rhs before form");
  cudaSetDevice(c->dev);
  CK(launch_compose_rhs(ebe_args(c), c->d_rhs, c->d_b, c->d_pa, c->st));
  CK(cudaMemcpyAsync(b, c->d_b, sizeof(double) * c->n_dof, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_get_du(cfdv_ctx* c, double* du) {
  if (!c || !du) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(cudaMemcpyAsync(du, c->d_du, sizeof(double) * c->n_dof, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_matvec(cfdv_ctx* c, const double* x, double* y, int precision, int transpose) {
  if (!c || !x || !y) return CFDV_ERR_ARG;
  if (!c->formed) return fail(c, CFDV_ERR_STATE, "matvec before form");
  const int fp32 = (precision == CFDV_PREC_MIXED);
  if (fp32 && !c->have32) return fail(c, CFDV_ERR_STATE, "FP32 matvec needs a MIXED form");
  cudaSetDevice(c->dev);
  CK(cudaMemcpyAsync(c->d_W, x, sizeof(double) * c->n_dof, cudaMemcpyHostToDevice, c->st));
  CK(launch_ebe(ebe_args(c), fp32, transpose, c->d_W, c->d_b, 0, nullptr, nullptr, nullptr, c->st));
  CK(cudaMemcpyAsync(y, c->d_b, sizeof(double) * c->n_dof, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CFDV_OK;
}

int cfdv_profile(cfdv_ctx* c, int enable) {
  if (!c) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  if (enable && c->ev_pool.empty()) {
    c->ev_pool.resize(3 * 8192);
    for (auto& e : c->ev_pool) CK(cudaEventCreate(&e));
  }
  for (auto& e : c->ev_form) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  c->ev_form.clear();
  for (auto& e : c->ev_solve) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  c->ev_solve.clear();
  c->ev_used = 0;
  c->mv_launches = 0;
  c->mv_bytes = 0;
  c->mv_full_bytes = 0;
  c->solve_bytes = 0;
  c->launches = 0;
  c->prof = enable != 0;
  return CFDV_OK;
}

int cfdv_profile_read(cfdv_ctx* c, cfdv_kernel_stats* out) {
  if (!c || !out) return CFDV_ERR_ARG;
  cudaSetDevice(c->dev);
  CK(cudaStreamSynchronize(c->st));
  std::memset(out, 0, sizeof(*out));
  for (size_t i = 0; i + 3 <= c->ev_used; i += 3) {
    float ms = 0, ms_all = 0;
    CK(cudaEventElapsedTime(&ms, c->ev_pool[i], c->ev_pool[i + 1]));
    CK(cudaEventElapsedTime(&ms_all, c->ev_pool[i], c->ev_pool[i + 2]));
    out->total_ms += ms;
    out->matvec_ms += ms_all;
    out->launches++;
  }
  for (auto& e : c->ev_form) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e.first, e.second));
    out->form_ms += ms;
    out->form_launches++;
  }
  for (auto& e : c->ev_solve) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e.first, e.second));
    out->solve_ms += ms;
    out->solves++;
  }
  out->bytes = c->mv_bytes;
  out->matvec_bytes = c->mv_full_bytes;
  out->solve_bytes = c->solve_bytes;
  out->kernel_launches = c->launches;
  return CFDV_OK;
}

}  // extern "C"
