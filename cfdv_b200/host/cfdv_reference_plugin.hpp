// cfdv_reference_plugin.hpp -- the B200 step as plug-ins of the CFDV reference's own classes.
//
// A header for the reference's build: include it after the reference's FDV/Element.h,
// FDV/Node.h and Utility/Solvers/GMRESbase.h (CFDV src/), and link libcfdv_gpu.so.  Two
// plug-ins share one GPU context built from the reference's element and node vectors:
//
//   CudaGMRES : GMRESbase  the reference's solver plug-in point (GMRESbase.h:8-23, whose
//                          header already lists a CUDA solver).  MPIBinaryConfiguration
//                          creates it where it creates MPI_GMRES
//                          (MPIBinaryConfiguration.h:123, 135); main.cpp's
//                          gmres->iterate(elements) / gmres->update(nodes) (main.cpp:196-197)
//                          then run on the GPU.  iterate() takes R and rhs from the elements
//                          (after FDVGalerkin and ApplyBC) unless GpuFormation formed them on
//                          the device for this step; update() applies U0 = U, U += dU to the
//                          nodes, as MPI_GMRES::update does (MPI_GMRES.h:224-301).  It prints
//                          the same tolerance / estimate / g(m) lines as MPI_GMRES
//                          (MPI_GMRES.h:140-142, 185-187, 202-203, 728).
//   GpuFormation           replaces `FDVGalerkin fdv(...); for_each(elements, fdv)` and the
//                          ApplyBC for_each (main.cpp:185-194): it uploads the nodes' U and
//                          forms every element's R and rhs on the device at the host's dt.
//                          With CudaGMRES the matrices stay on the device; otherwise (or on
//                          request) they are copied back into elements[e]->R / ->rhs.
//
// Errors: the reference has no error convention (messages and cin.get()); these classes throw
// std::runtime_error with the library's message.  The C ABI underneath never throws.
#ifndef CFDV_REFERENCE_PLUGIN_HPP
#define CFDV_REFERENCE_PLUGIN_HPP

#include <cmath>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfdv_gpu.h"

namespace cfdv_plugin {

// One GPU context over the reference's mesh objects (one rank: node ids are positions).
class Context {
 public:
  Context(std::vector<Element*>& elements, std::vector<Node*>& nodes, int ndim, int nnod, int neqn,
          const cfdv_params& params)
      : ndim_(ndim), nnod_(nnod), neqn_(neqn), Ke_(nnod * neqn),
        n_nodes_((int)nodes.size()), n_elements_((int)elements.size()) {
    const int nface = ndim == 2 ? 4 : 6;
    std::vector<double> x((size_t)n_nodes_ * ndim);
    for (Node* n : nodes)
      for (int i = 0; i < ndim; i++) x[(size_t)n->number * ndim + i] = n->x(i);
    std::vector<int> conn((size_t)n_elements_ * nnod), bc((size_t)n_elements_ * nface, 0);
    for (int e = 0; e < n_elements_; e++) {
      for (int k = 0; k < nnod; k++) conn[(size_t)e * nnod + k] = (int)elements[e]->node[k]->number;
      // Element::face lists only the faces loaded with a boundary code (LoadBinary.h:264-275)
      for (Face* f : elements[e]->face) bc[(size_t)e * nface + f->face] = f->bc;
    }
    cfdv_mesh m{ndim, n_nodes_, n_elements_, x.data(), conn.data(), bc.data()};
    check(cfdv_create(&m, &params, &ctx_), "cfdv_create");
    // hanging-node elements (Element::adap / Hnm, Element.h:39-40)
    std::vector<int> adap;
    std::vector<double> hnm;
    for (int e = 0; e < n_elements_; e++) {
      if (!elements[e]->adap) continue;
      adap.push_back(e);
      for (int M = 0; M < nnod; M++)
        for (int N = 0; N < nnod; N++) hnm.push_back(elements[e]->Hnm(N, M));  // Hnm(N, M) at N + nnod*M
    }
    if (!adap.empty()) check(cfdv_set_adaptive(ctx_, (int)adap.size(), adap.data(), hnm.data()), "cfdv_set_adaptive");
    U_.resize((size_t)n_nodes_ * neqn);
    du_.resize(U_.size());
  }
  ~Context() { cfdv_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;

  void check(int rc, const char* what) const {
    if (rc) throw std::runtime_error(std::string(what) + ": " + (ctx_ ? cfdv_last_error(ctx_) : "failed"));
  }
  cfdv_ctx* ctx() const { return ctx_; }
  int ndim() const { return ndim_; }
  int nnod() const { return nnod_; }
  int neqn() const { return neqn_; }
  int Ke() const { return Ke_; }
  int n_nodes() const { return n_nodes_; }
  int n_elements() const { return n_elements_; }

  // the nodes' conserved state to the device
  void upload_state(std::vector<Node*>& nodes) {
    for (Node* n : nodes)
      for (int k = 0; k < neqn_; k++) U_[(size_t)n->number * neqn_ + k] = n->U(k);
    check(cfdv_set_state(ctx_, U_.data(), U_.size()), "cfdv_set_state");
  }
  std::vector<double>& du() { return du_; }

  bool formed_on_device = false;  // set by GpuFormation, consumed by CudaGMRES::iterate

 private:
  cfdv_ctx* ctx_ = nullptr;
  int ndim_, nnod_, neqn_, Ke_, n_nodes_, n_elements_;
  std::vector<double> U_, du_;
};

// Replaces the FDVGalerkin and ApplyBC passes of a step (main.cpp:185-194).
class GpuFormation {
 public:
  GpuFormation(Context& c, int precision = CFDV_PREC_FP64) : c_(c), precision_(precision) {}
  // Form at the host's dt (CFL, main.cpp:179).  copy_back writes R and rhs into the elements,
  // for a solver that reads them there (MPI_GMRES) or for output.
  void operator()(std::vector<Element*>& elements, std::vector<Node*>& nodes, double dt, bool copy_back = false) {
    c_.upload_state(nodes);
    c_.check(cfdv_form(c_.ctx(), dt, precision_), "cfdv_form");
    c_.formed_on_device = true;
    if (!copy_back) return;
    const size_t Ke = c_.Ke();
    R_.resize((size_t)c_.n_elements() * Ke * Ke);
    rhs_.resize((size_t)c_.n_elements() * Ke);
    c_.check(cfdv_get_element_matrices(c_.ctx(), R_.data(), rhs_.data()), "cfdv_get_element_matrices");
    for (size_t e = 0; e < elements.size(); e++) {
      for (size_t j = 0; j < Ke; j++)
        for (size_t i = 0; i < Ke; i++) elements[e]->R((int)i, (int)j) = R_[e * Ke * Ke + j * Ke + i];
      for (size_t i = 0; i < Ke; i++) elements[e]->rhs((int)i) = rhs_[e * Ke + i];
    }
  }

 private:
  Context& c_;
  int precision_;
  std::vector<double> R_, rhs_;
};

}  // namespace cfdv_plugin

// The solver plug-in (GMRESbase.h:8-23).  Default: the reference's own GMRES (restart count,
// ||b|| 1e-9 inner break, its back substitution), on the GPU; mode CFDV_GMRES_CORRECT solves to
// rtol instead.
struct CudaGMRES : public GMRESbase {
  CudaGMRES(cfdv_plugin::Context& c, int restart, int m, int mode = CFDV_GMRES_REFERENCE, double rtol = 1e-8,
            int precision = CFDV_PREC_FP64)
      : c_(c) {
    opts_.mode = mode;
    opts_.m = m;
    opts_.restarts = restart;
    opts_.rtol = rtol;
    opts_.precision = precision;
    opts_.true_residual = 0;
    opts_.engine = 0;
    opts_.precond = 1;
    opts_.orth = 2;
    est_.resize((size_t)m * (restart > 0 ? restart : 1));
    gfinal_.resize(restart > 0 ? restart : 1);
  }

  void iterate(std::vector<Element*>& elements) {
    if (!c_.formed_on_device) {  // matrices formed on the host by FDVGalerkin + ApplyBC
      const size_t Ke = c_.Ke();
      R_.resize((size_t)c_.n_elements() * Ke * Ke);
      rhs_.resize((size_t)c_.n_elements() * Ke);
      for (size_t e = 0; e < elements.size(); e++) {
        for (size_t j = 0; j < Ke; j++)
          for (size_t i = 0; i < Ke; i++) R_[e * Ke * Ke + j * Ke + i] = elements[e]->R((int)i, (int)j);
        for (size_t i = 0; i < Ke; i++) rhs_[e * Ke + i] = elements[e]->rhs((int)i);
      }
      c_.check(cfdv_set_element_matrices(c_.ctx(), R_.data(), rhs_.data(), opts_.precision),
               "cfdv_set_element_matrices");
    }
    c_.formed_on_device = false;
    cfdv_gmres_report rep{};
    rep.est_capacity = (int)est_.size();
    rep.est = est_.data();
    rep.gfinal_capacity = (int)gfinal_.size();
    rep.gfinal = gfinal_.data();
    c_.check(cfdv_gmres(c_.ctx(), &opts_, &rep), "cfdv_gmres");
    print_like_reference(rep);
  }

  void update(std::vector<Node*>& nodes) {
    std::vector<double>& du = c_.du();
    c_.check(cfdv_get_du(c_.ctx(), du.data()), "cfdv_get_du");
    const int neqn = c_.neqn();
    for (Node* n : nodes)
      for (int k = 0; k < neqn; k++) {
        n->U0(k) = n->U(k);
        n->U(k) += du[(size_t)n->number * neqn + k];
      }
  }

 private:
  // The lines MPI_GMRES::iterate writes (tolerance, one estimate per Arnoldi step, the break
  // message, g(m) per restart), in its order: a restart ends after m estimates or at the
  // first estimate below the tolerance.
  void print_like_reference(const cfdv_gmres_report& rep) const {
    std::cout << " tolerence: " << rep.tol << std::endl;
    if (opts_.mode != CFDV_GMRES_REFERENCE) return;
    int k = 0;
    for (int r = 0; r < rep.n_restarts; r++) {
      for (int j = 0; j < opts_.m && k < rep.n_est; j++, k++) {
        std::cout << "residual: " << rep.est[k] << std::endl;
        if (std::fabs(rep.est[k]) < rep.tol) {
          std::cout << "mag < tol, breaking..." << std::endl;
          std::cout << "tolerence met msg received in rank " << 0 << std::endl;
          k++;
          break;
        }
      }
      if (r < rep.gfinal_capacity) std::cout << "\tResidual: " << rep.gfinal[r] << std::endl;
    }
  }

  cfdv_plugin::Context& c_;
  cfdv_gmres_opts opts_{};
  std::vector<double> est_, gfinal_, R_, rhs_;
};

#endif  // CFDV_REFERENCE_PLUGIN_HPP
