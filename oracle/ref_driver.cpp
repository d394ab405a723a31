// Oracle driver around the UNMODIFIED CFDV reference sources.
//
// Test infrastructure only: this file is compiled (oracle/Makefile) together with
// the reference's own headers under <reference>/src and the single-rank MPI /
// Boost stand-ins in oracle/shim, into oracle/_ref/cfdv_ref.  It replays the
// per-step sequence of the reference driver (src/main.cpp:169-198) on one rank:
//
//   ClearElement (main.cpp:169) -> NodeUnpack (:171) -> CFL (:179)
//   -> FDVGalerkin over all elements (:185-186) -> ApplyBC (:194)
//   -> gmres->iterate (:196) -> gmres->update (:197) -> RMSErr (:198)
//
// and writes what it computed into a record file (format below) that the tests
// and the fixture generator read with numpy.  Startup follows
// src/MPIBinaryConfiguration.h:22-124 (Thermo::set, LoadBinaryData, MPI_GMRES)
// and src/main.cpp:120-121 (CalcLength); control/aero are parsed here because
// the reference's Boost.ProgramOptions parser is not available.
//
// Record file: a sequence of records
//   u32 name_len, name bytes, u8 type ('d' f64 | 'i' i32), u64 count, payload
//
// Usage: cfdv_ref <case_dir> <out_file> [--steps N] [--dump-step K]
//                 [--gmresiter M] [--restart R] [--quiet] [--tecplot]
//                 [--elements FILE] [--form-subset]
// --elements FILE (int32 element ids) limits the step-K dumps of R and rhs to those
// elements, in the file's order; with --form-subset, step K forms (FDVGalerkin, ApplyBC)
// only those elements, writes the dumps and stops before the solve: on a mesh of 10^5-10^6
// hex8 elements this samples the reference's formation without forming every element.
// The element functor depends only on the element and its nodes, so a subset's matrices
// are those a full pass would give.
// Built with -DCFDV_GPU_PLUGIN (oracle/Makefile target ref-gpu, _ref/cfdv_ref_gpu, linked
// against libcfdv_gpu.so) the same loop can run the B200 plug-ins of
// cfdv_b200/host/cfdv_reference_plugin.hpp in place of the reference's classes:
//   --gpu-solver   CudaGMRES : GMRESbase instead of MPI_GMRES (main.cpp:196-197)
//   --gpu-form     GpuFormation instead of the FDVGalerkin and ApplyBC passes (main.cpp:185-194)
// so that everything else -- load, CalcLength, ClearElement, NodeUnpack, CFL, RMS, the record
// file -- is the reference's own code path.
// --refine runs, after the steps, the reference's mesh-refinement branch (main.cpp:139-148:
// NodeUnpack, NodeCheck, AdaptiveRefineList -- elements with FDVParam s1 > 0.8
// (RefineListAdaptive.h:25-36) and their dependencies -- then MeshRefine2D) and records the
// marked elements and the refined case as Save would write it: node records {x, rho, v, T},
// element node ids and face codes, and the adaptive elements with refine level and Hnm.
// --tecplot writes the reference's outputs into the working directory: tecplot_<iter>.plt
// (MPI_TecplotOut.h) at every iteration divisible by 100, as main.cpp:183 does, and the
// RMSError.txt line of every step (MPI_RMSError.h), as main.cpp:198 does.
#include "mpi.h"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "FDV/Element.h"
#include "FDV/Node.h"
#include "FDV/FDVGalerkin.h"
#include "FDV/Function/ApplyBC.h"
#include "FDV/Function/CalcLength.h"
#include "FDV/Function/ClearElement.h"
#include "FDV/Function/NodeUnpack.h"
#include "FDV/Function/MPI_CFL.h"
#include "FDV/Function/FDVParam.h"
#include "FDV/Function/MPI_RMSError.h"
#include "Utility/Solvers/MPI_GMRES.h"
#include "Utility/IO/ASCIItoBinary/LoadBinary.h"
#include "Utility/IO/MPI_TecplotOut.h"
#include "FDV/Function/NodeCheck.h"
#include "adap/RefineListAdaptive.h"
#include "adap/MeshRefine2D.h"
#ifdef CFDV_GPU_PLUGIN
#include <memory>

#include "cfdv_reference_plugin.hpp"
#endif

namespace {

struct RecordFile {
  FILE* f = nullptr;
  void put(const std::string& name, char type, const void* data, uint64_t count) {
    uint32_t n = (uint32_t)name.size();
    fwrite(&n, 4, 1, f);
    fwrite(name.data(), 1, n, f);
    fwrite(&type, 1, 1, f);
    fwrite(&count, 8, 1, f);
    size_t es = (type == 'd') ? 8 : 4;
    if (count) fwrite(data, es, count, f);
  }
  void putd(const std::string& name, const std::vector<double>& v) { put(name, 'd', v.data(), v.size()); }
  void puti(const std::string& name, const std::vector<int>& v) { put(name, 'i', v.data(), v.size()); }
};

// key = value parser for the reference's control/aero files
// (the keys registered at src/MPIBinaryConfiguration.h:29-63).
std::map<std::string, std::string> parse_kv(const std::string& path) {
  std::map<std::string, std::string> kv;
  std::ifstream in(path.c_str());
  std::string line;
  while (std::getline(in, line)) {
    size_t c = line.find_first_of("!#");
    if (c != std::string::npos) line = line.substr(0, c);
    size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    auto trim = [](std::string s) {
      size_t a = s.find_first_not_of(" \t\r\n");
      size_t b = s.find_last_not_of(" \t\r\n");
      return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    };
    kv[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
  }
  return kv;
}

double getd(std::map<std::string, std::string>& kv, const char* k, double dflt) {
  auto it = kv.find(k);
  return it == kv.end() ? dflt : atof(it->second.c_str());
}
int geti(std::map<std::string, std::string>& kv, const char* k, int dflt) {
  auto it = kv.find(k);
  return it == kv.end() ? dflt : atoi(it->second.c_str());
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s <case_dir> <out_file> [--steps N] [--dump-step K] [--gmresiter M] [--restart R]\n", argv[0]);
    return 2;
  }
  std::string path = argv[1];
  std::string out = argv[2];
  int nsteps = 1, dump_step = -1, m_override = -1, r_override = -1;
  bool quiet = false, tecplot = false, form_subset = false, gpu_solver = false, gpu_form = false, refine = false;
  std::string elements_file;
  for (int i = 3; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--steps" && i + 1 < argc) nsteps = atoi(argv[++i]);
    else if (a == "--dump-step" && i + 1 < argc) dump_step = atoi(argv[++i]);
    else if (a == "--gmresiter" && i + 1 < argc) m_override = atoi(argv[++i]);
    else if (a == "--restart" && i + 1 < argc) r_override = atoi(argv[++i]);
    else if (a == "--quiet") quiet = true;
    else if (a == "--tecplot") tecplot = true;
    else if (a == "--elements" && i + 1 < argc) elements_file = argv[++i];
    else if (a == "--form-subset") form_subset = true;
    else if (a == "--gpu-solver") gpu_solver = true;
    else if (a == "--gpu-form") gpu_form = true;
    else if (a == "--refine") refine = true;
  }
#ifndef CFDV_GPU_PLUGIN
  if (gpu_solver || gpu_form) {
    fprintf(stderr, "--gpu-solver / --gpu-form need the build with CFDV_GPU_PLUGIN (cfdv_ref_gpu)\n");
    return 2;
  }
#endif

  auto cm = parse_kv(path + "/control");
  auto am = parse_kv(path + "/aero");
  const int ndim = geti(cm, "ndim", 2), nnod = geti(cm, "nnod", 4), neqn = geti(cm, "neqn", 4);
  const int nbnod = geti(cm, "nbnod", 2);
  const int Nn = geti(cm, "nodes", 0), E = geti(cm, "elements", 0);
  const double cfl = getd(cm, "cfl", 1.0);
  const int m = m_override > 0 ? m_override : geti(cm, "gmresiter", 20);
  const int restart = r_override > 0 ? r_override : geti(cm, "gmresrestart", 1);

  // MPIBinaryConfiguration.h:90-100
  Thermo::Instance().set(getd(am, "gamma", 1.4), getd(am, "M", 1.0), getd(am, "Re", 1.0), getd(am, "Pr", 0.72),
                         getd(am, "Tinf", 216.6666), getd(am, "Twall", 1.0), geti(am, "Adiabatic", 1) != 0);

  std::vector<Node*> nodes;
  std::vector<Element*> elements;
  // the loader prints per-face diagnostics (LoadBinary.h:305-307); keep them off stdout
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  LoadBinaryData load(elements, nodes, path, nnod, neqn, ndim, nbnod);
  load.read_nodes(0, Nn - 1);
  load.read_elements(0, E);
  if (geti(cm, "adap", 0)) load.read_adap();  // MPIBinaryConfiguration.h:110-113: hanging-node Hnm
  CalcLength<Element*> cl(ndim, nnod);  // main.cpp:120-121
  for_each(elements.begin(), elements.end(), std::ref(cl));
  NavierStokes* NS = (ndim == 2) ? (NavierStokes*)new NavierStokes2D : (NavierStokes*)new NavierStokes3D;
  MPI_GMRES gmres(restart, m, Nn * neqn, neqn, nnod, ndim, 1, 0, 0);  // MPIBinaryConfiguration.h:123
  std::cout.rdbuf(saved);
  GMRESbase* solver = &gmres;
#ifdef CFDV_GPU_PLUGIN
  std::unique_ptr<cfdv_plugin::Context> gctx;
  std::unique_ptr<CudaGMRES> cuda_gmres;
  std::unique_ptr<cfdv_plugin::GpuFormation> gpu_formation;
  if (gpu_solver || gpu_form) {
    cfdv_params gp{getd(am, "gamma", 1.4), getd(am, "M", 1.0),        getd(am, "Re", 1.0),
                   getd(am, "Pr", 0.72),   getd(am, "Tinf", 216.6666), getd(am, "Twall", 1.0),
                   geti(am, "Adiabatic", 1) != 0 ? 1 : 0, 0};
    gctx.reset(new cfdv_plugin::Context(elements, nodes, ndim, nnod, neqn, gp));
    if (gpu_solver) {
      cuda_gmres.reset(new CudaGMRES(*gctx, restart, m));
      solver = cuda_gmres.get();
    }
    if (gpu_form) gpu_formation.reset(new cfdv_plugin::GpuFormation(*gctx));
  }
#endif

  RecordFile rf;
  rf.f = fopen(out.c_str(), "wb");
  if (!rf.f) { perror("open out"); return 1; }
  rf.puti("meta", {ndim, nnod, neqn, Nn, E, nsteps, m, restart});
  {
    std::vector<double> cleng(E), Uinit;
    for (int e = 0; e < E; e++) cleng[e] = elements[e]->cleng;
    for (auto* n : nodes)
      for (int k = 0; k < neqn; k++) Uinit.push_back(n->U(k));
    rf.putd("cleng", cleng);
    rf.putd("U_init", Uinit);
    std::vector<int> dir;
    for (auto* n : nodes)
      for (int k = 0; k < neqn; k++) dir.push_back(n->dirichlet(k) ? 1 : 0);
    rf.puti("dirichlet", dir);
  }

  // the elements whose matrices a dump writes (all, or the --elements list)
  std::vector<int> dump_el;
  if (!elements_file.empty()) {
    FILE* ef = fopen(elements_file.c_str(), "rb");
    if (!ef) { perror("open elements"); return 1; }
    int id;
    while (fread(&id, 4, 1, ef) == 1) {
      if (id < 0 || id >= E) { fprintf(stderr, "element id %d out of range\n", id); return 1; }
      dump_el.push_back(id);
    }
    fclose(ef);
  } else {
    for (int e = 0; e < E; e++) dump_el.push_back(e);
  }
  if (form_subset && elements_file.empty()) { fprintf(stderr, "--form-subset needs --elements\n"); return 2; }
  rf.puti("dump_elements", dump_el);
  std::vector<Element*> subset;
  for (int e : dump_el) subset.push_back(elements[e]);

  const int Ke = nnod * neqn;
  double t = 0, dt = 0, t_form = 0, t_gmres = 0;
  std::cout.precision(17);
  for (int iter = 0; iter < nsteps; iter++) {
    auto t_step0 = std::chrono::steady_clock::now();
    for_each(elements.begin(), elements.end(), ClearElement<Element*>());  // main.cpp:169
    for_each(nodes.begin(), nodes.end(), NodeUnpack<Node*>());             // main.cpp:171
    double cfl_v = cfl;
    CFL<Element*>(elements, cfl_v, dt);  // main.cpp:179
    if (tecplot && iter % 100 == 0) {  // main.cpp:183, after NodeUnpack and CFL
      std::cout.rdbuf(sink.rdbuf());
      MPI_TecplotOut(elements, nodes, iter, ndim, t, true, 0, 0, 1, 0, nnod, neqn);
      std::cout.rdbuf(saved);
    }
    auto t0 = std::chrono::steady_clock::now();
    const bool sub_only = form_subset && iter == dump_step;
    std::vector<Element*>& formed = sub_only ? subset : elements;
    const size_t D = dump_el.size();
#ifdef CFDV_GPU_PLUGIN
    if (gpu_formation) {
      // the device forms and applies the Dirichlet rows in one pass: R and rhs come back to the
      // elements only when the host needs them (a dump, or the reference's own solver)
      (*gpu_formation)(elements, nodes, dt, iter == dump_step || !cuda_gmres);
    } else
#endif
    {
    FDVGalerkin<Element*> fdv(nnod, neqn, ndim, nbnod, dt, NS);  // main.cpp:185-186
    for_each(formed.begin(), formed.end(), std::ref(fdv));
    if (iter == dump_step) {
      std::vector<double> R(D * Ke * Ke), rhs(D * Ke), s(4 * D);
      for (size_t k = 0; k < D; k++) {
        Element* el = elements[dump_el[k]];
        for (int j = 0; j < Ke; j++)
          for (int i = 0; i < Ke; i++) R[k * Ke * Ke + (size_t)j * Ke + i] = el->R(i, j);
        for (int i = 0; i < Ke; i++) rhs[k * Ke + i] = el->rhs(i);
        FDVParam<Element*> fp;
        fp(el, s[4 * k + 0], s[4 * k + 1], s[4 * k + 2], s[4 * k + 3]);
      }
      rf.putd("R_form", R);  // column-major per element: R(i,j) at j*Ke+i
      rf.putd("rhs_form", rhs);
      rf.putd("s1234", s);
    }
    for_each(formed.begin(), formed.end(), ApplyBC<Element*>(neqn, nnod, ndim, nbnod));  // main.cpp:194
    }
    auto t1 = std::chrono::steady_clock::now();
    if (iter == dump_step) {
      std::vector<double> R(D * Ke * Ke), rhs(D * Ke);
      for (size_t k = 0; k < D; k++) {
        Element* el = elements[dump_el[k]];
        for (int j = 0; j < Ke; j++)
          for (int i = 0; i < Ke; i++) R[k * Ke * Ke + (size_t)j * Ke + i] = el->R(i, j);
        for (int i = 0; i < Ke; i++) rhs[k * Ke + i] = el->rhs(i);
      }
      rf.putd("R_bc", R);
      rf.putd("rhs_bc", rhs);
      std::vector<double> Ucur;
      for (auto* n : nodes)
        for (int k = 0; k < neqn; k++) Ucur.push_back(n->U(k));
      rf.putd("U_dump", Ucur);
      rf.putd("dt_dump", {dt});
      if (sub_only) {
        rf.putd("form_time", {std::chrono::duration<double>(t1 - t0).count()});
        break;
      }
    }

    // GMRES prints its tolerance, per-iteration Givens estimates and g(m) on
    // stdout (MPI_GMRES.h:141-142, 728, 202-203); capture them at 17 digits.
    std::ostringstream cap;
    cap.precision(17);
    std::cout.rdbuf(cap.rdbuf());
    solver->iterate(elements);  // main.cpp:196
    solver->update(nodes);      // main.cpp:197
    std::cout.rdbuf(saved);
    auto t2 = std::chrono::steady_clock::now();
    t_form += std::chrono::duration<double>(t1 - t0).count();
    t_gmres += std::chrono::duration<double>(t2 - t1).count();

    std::vector<double> est, fin, tol;
    std::istringstream ls(cap.str());
    std::string line;
    while (std::getline(ls, line)) {
      if (line.rfind("residual: ", 0) == 0) est.push_back(strtod(line.c_str() + 10, nullptr));
      else if (line.rfind("\tResidual: ", 0) == 0) fin.push_back(strtod(line.c_str() + 11, nullptr));
      else if (line.rfind(" tolerence: ", 0) == 0) tol.push_back(strtod(line.c_str() + 12, nullptr));
    }
    std::vector<double> U, U0;
    for (auto* n : nodes)
      for (int k = 0; k < neqn; k++) { U.push_back(n->U(k)); U0.push_back(n->U0(k)); }
    std::string sfx = "@" + std::to_string(iter);
    rf.putd("dt" + sfx, {dt});
    rf.putd("tol" + sfx, tol);
    rf.putd("est" + sfx, est);
    rf.putd("gfinal" + sfx, fin);
    rf.putd("U" + sfx, U);
    // RMSError.txt line (MPI_RMSError.h:21-51)
    std::vector<double> rms(neqn);
    for (int k = 0; k < neqn; k++) {
      double a = 0, b = 0;
      for (auto* n : nodes) { a += n->U(k) * n->U(k); b += n->U0(k) * n->U0(k); }
      rms[k] = (b == 0) ? 1.0 : std::sqrt(a / b) - 1.0;
    }
    rf.putd("rms" + sfx, rms);
    if (tecplot) {  // the reference's RMSError.txt line (MPIBinaryConfiguration.h:138-142)
      std::cout.rdbuf(sink.rdbuf());
      {
        MPI_RMSError<Node*> rmserr("RMSError.txt", t, iter, neqn);
        for_each(nodes.begin(), nodes.end(), std::ref(rmserr));
      }
      std::cout.rdbuf(saved);
    }
    // wall time of the step's path: CFL, formation, ApplyBC, GMRES, update
    rf.putd("steptime" + sfx, {std::chrono::duration<double>(t2 - t_step0).count()});
    t += dt;
    if (!quiet) fprintf(stderr, "step %d dt %.6e gfinal %.3e\n", iter, dt, fin.empty() ? -1.0 : fin.back());
  }
  if (refine) {  // main.cpp:139-148 (the refinement prints its progress: kept off stdout)
    const int nface = geti(cm, "nface", ndim == 2 ? 4 : 6);
    std::cout.rdbuf(sink.rdbuf());
    for_each(nodes.begin(), nodes.end(), NodeUnpack<Node*>());
    for_each(nodes.begin(), nodes.end(), NodeCheck<Node*>());
    std::vector<int> marks;  // the criterion of RefineListAdaptive.h:25-36 before its dependency closure
    {
      FDVParam<Element*> fp;
      double s1, s2, s3, s4;
      for (size_t e = 0; e < elements.size(); e++) {
        fp(elements[e], s1, s2, s3, s4);
        if (s1 > 0.8) marks.push_back((int)e);
      }
    }
    std::vector<int> elelist, refine_level;
    AdaptiveRefineList<Element, Node>(elelist, refine_level, elements, nodes, nnod, nface);
    MeshRefine2D<Element, Node>(elements, nodes, elelist, refine_level, ndim, neqn, nnod, nsteps, nface);
    for_each(nodes.begin(), nodes.end(), NodeUnpack<Node*>());
    for_each(nodes.begin(), nodes.end(), NodeCheck<Node*>());
    std::cout.rdbuf(saved);
    rf.puti("refine_marks", marks);
    rf.puti("refine_elelist", elelist);
    std::vector<double> rec;
    std::vector<int> num;
    for (Node* n : nodes) {  // the binarynodes record (LoadBinary.h:156-205)
      for (int i = 0; i < ndim; i++) rec.push_back(n->x(i));
      rec.push_back(n->rho);
      for (int i = 0; i < ndim; i++) rec.push_back(n->v(i));
      rec.push_back(n->T);
      num.push_back((int)n->number);
    }
    rf.putd("refined_nodes", rec);
    rf.puti("refined_node_numbers", num);
    std::vector<int> conn, bcs, adap, level;
    std::vector<double> hnm;
    for (size_t e = 0; e < elements.size(); e++) {
      Element* el = elements[e];
      for (int k = 0; k < nnod; k++) conn.push_back((int)el->node[k]->number);
      std::vector<int> b(nface, 0);
      for (Face* f : el->face) b[f->face] = f->bc;
      bcs.insert(bcs.end(), b.begin(), b.end());
      if (el->adap) {
        adap.push_back((int)e);
        level.push_back(el->refine_level);
        for (int M = 0; M < nnod; M++)
          for (int N = 0; N < nnod; N++) hnm.push_back(el->Hnm(N, M));  // Hnm(N, M) at N + nnod*M
      }
    }
    rf.puti("refined_conn", conn);
    rf.puti("refined_bc", bcs);
    rf.puti("refined_adap", adap);
    rf.puti("refined_levels", level);
    rf.putd("refined_hnm", hnm);
  }
  rf.putd("timing", {t_form / std::max(nsteps, 1), t_gmres / std::max(nsteps, 1)});
  fclose(rf.f);
  delete NS;
  return 0;
}
