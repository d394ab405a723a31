// cfdv_gpu: the CFDV time loop (src/main.cpp:162-206) with the per-step path on a B200.
//
//   cfdv_gpu <case_dir> [--steps N] [--mode reference|correct] [--precision fp64|mixed]
//            [--rtol R] [--restarts K] [--warm-start] [--physical-3d-flux] [--out DIR] [--save-every K]
//            [--ensight DIR]
//
// Reads the reference case directory (control, aero, binarynodes, binaryelements) and
// runs, per iteration, the reference's call order: CFL (main.cpp:179), Tecplot output
// every 100 iterations (:183), element formation + ApplyBC (:185-194), GMRES iterate and
// update (:196-197), RMSErr (:198).  Output files are the reference's: tecplot_<iter>.plt
// and RMSError.txt, written to --out (default: the working directory), and the checkpoint
// case directories <out>/<iter>/ every --save-every iterations (default 1000, main.cpp:177)
// and after the last one (main.cpp:208); running the driver on such a directory resumes
// the run at its iteration.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cfdv_host.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr,
                 "usage: %s <case_dir> [--steps N] [--mode reference|correct] [--precision fp64|mixed] "
                 "[--rtol R] [--restarts K] [--warm-start] [--physical-3d-flux] [--out DIR] [--save-every K] "
                 "[--ensight DIR]\n",
                 argv[0]);
    return 2;
  }
  std::string dir = argv[1], out = ".", ensight_dir;
  int steps = -1, restarts = -1, phys = 0, save_every = 1000, warm = 0;
  int mode = CFDV_GMRES_REFERENCE, precision = CFDV_PREC_FP64;
  double rtol = 1e-8;
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--steps" && i + 1 < argc) steps = std::atoi(argv[++i]);
    else if (a == "--mode" && i + 1 < argc) mode = std::string(argv[++i]) == "correct" ? CFDV_GMRES_CORRECT : CFDV_GMRES_REFERENCE;
    else if (a == "--precision" && i + 1 < argc) precision = std::string(argv[++i]) == "mixed" ? CFDV_PREC_MIXED : CFDV_PREC_FP64;
    else if (a == "--rtol" && i + 1 < argc) rtol = std::atof(argv[++i]);
    else if (a == "--restarts" && i + 1 < argc) restarts = std::atoi(argv[++i]);
    else if (a == "--physical-3d-flux") phys = 1;
    else if (a == "--warm-start") warm = 1;
    else if (a == "--out" && i + 1 < argc) out = argv[++i];
    else if (a == "--save-every" && i + 1 < argc) save_every = std::atoi(argv[++i]);
    else if (a == "--ensight" && i + 1 < argc) ensight_dir = argv[++i];
  }
  try {
    cfdv_host::CaseConfig cfg(dir);
    cfdv_host::BinaryCase c(dir, cfg);
    const cfdv_params p = cfg.params(phys);
    cfdv_host::GpuFDV fdv(c, p);
    const int iter0 = cfg.ci("iter", 0);
    const int itermax = steps >= 0 ? iter0 + steps : cfg.ci("itermax", 1);
    const double cfl = cfg.cd("cfl", 1.0);
    cfdv_gmres_opts o;
    o.mode = mode;
    o.m = cfg.ci("gmresiter", 20);
    o.restarts = restarts > 0 ? restarts : (mode == CFDV_GMRES_REFERENCE ? cfg.ci("gmresrestart", 1) : 100);
    o.rtol = rtol;
    o.precision = precision;
    o.true_residual = 0;
    o.engine = 0;
    o.precond = 1;
    o.orth = 2;  // delayed CGS2 (one reduction per Arnoldi step)
    o.warm_start = warm;  // correct mode: start each solve from the previous step's dU
    std::vector<double> est((size_t)o.m * o.restarts), gfin(o.restarts);
    cfdv_gmres_report rep;
    std::memset(&rep, 0, sizeof(rep));
    rep.est = est.data();
    rep.est_capacity = (int)est.size();
    rep.gfinal = gfin.data();
    rep.gfinal_capacity = (int)gfin.size();
    double t = 0;
    std::unique_ptr<cfdv_host::EnsightSeries> ensight;
    if (!ensight_dir.empty()) ensight.reset(new cfdv_host::EnsightSeries(ensight_dir, c));
    auto t0 = std::chrono::steady_clock::now();
    for (int iter = iter0; iter < itermax; iter++) {
      if (save_every > 0 && iter % save_every == 0) cfdv_host::save_case(out, iter, c, cfg, p, fdv.state());
      const double dt = fdv.cfl(cfl);
      fdv.form(dt, precision);
      if (iter % 100 == 0) {  // written from this step's state, before the solve
        std::vector<double> U = fdv.state(), s = fdv.fdv_params();
        cfdv_host::tecplot_write(out + "/" + cfdv_host::tecplot_name(iter), c, p, U, &s, t);
        if (ensight) ensight->write(t, p, U, &s);
      }
      fdv.iterate(o, &rep);
      fdv.update();
      cfdv_host::rms_append(out + "/RMSError.txt", iter, fdv.rms());
      t += dt;
      std::printf("iter %d dt %.6e restarts %d matvecs %d\n", iter, dt, rep.n_restarts, rep.n_matvec);
    }
    if (save_every > 0) cfdv_host::save_case(out, itermax, c, cfg, p, fdv.state());
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("%d steps in %.3f s (%.2f steps/s)\n", itermax - iter0, secs, (itermax - iter0) / secs);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cfdv_gpu: %s\n", e.what());
    return 1;
  }
  return 0;
}
