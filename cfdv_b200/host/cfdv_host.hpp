// Host side of the B200 FDV path, in C++ over the C ABI (include/cfdv_gpu.h).
//
// These classes stand where the reference driver's objects stand:
//   CaseConfig   control/aero files      (MPIBinaryConfiguration.h:29-69)
//   BinaryCase   binarynodes/elements    (Utility/IO/ASCIItoBinary/LoadBinary.h:116-246)
//   GpuFDV       element formation + GMRES on the device: the FDVGalerkin/ApplyBC loop
//                (main.cpp:185-194) and the GMRESbase plug-in point
//                (Utility/Solvers/GMRESbase.h:8-23: iterate(), update())
//   TecplotOut   tecplot_<iter>.plt      (Utility/IO/MPI_TecplotOut.h:186-373)
//   RmsLog       RMSError.txt            (FDV/Function/MPI_RMSError.h:56-75)
//   save_case    <iter>/ checkpoints     (MPIBinaryConfiguration.h:148-161, SaveBinary.h)
//   EnsightSeries EnSight Gold output    (new: the reference's EnsightOut.h:9-13 is a stub)
//   convert_ascii ASCII case -> binary   (ConvertMain.cpp, AsciiLoad.h: the CONVERT tool)
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cfdv_gpu.h"

namespace cfdv_host {

struct CaseConfig {
  std::map<std::string, std::string> control, aero;
  static std::map<std::string, std::string> parse(const std::string& path) {
    std::map<std::string, std::string> kv;
    std::ifstream in(path.c_str());
    if (!in) throw std::runtime_error("cannot open " + path);
    std::string line;
    while (std::getline(in, line)) {
      size_t c = line.find_first_of("!#");
      if (c != std::string::npos) line = line.substr(0, c);
      size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      auto trim = [](const std::string& s) {
        size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
        return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
      };
      kv[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    return kv;
  }
  explicit CaseConfig(const std::string& dir) : control(parse(dir + "/control")), aero(parse(dir + "/aero")) {}
  int ci(const char* k, int d) const { auto it = control.find(k); return it == control.end() ? d : std::stoi(it->second); }
  double cd(const char* k, double d) const { auto it = control.find(k); return it == control.end() ? d : std::stod(it->second); }
  double ad(const char* k, double d) const { auto it = aero.find(k); return it == aero.end() ? d : std::stod(it->second); }
  cfdv_params params(int physical_3d_flux = 0) const {
    cfdv_params p;
    p.gamma = ad("gamma", 1.4);
    p.mach = ad("M", 1.0);
    p.reynolds = ad("Re", 1.0);
    p.prandtl = ad("Pr", 0.72);
    p.tinf = ad("Tinf", 216.6666);
    p.twall = ad("Twall", 1.0);
    auto it = aero.find("Adiabatic");
    p.adiabatic = (it == aero.end()) ? 1 : (std::stod(it->second) != 0);
    p.physical_3d_flux = physical_3d_flux;
    return p;
  }
};

// Binary node and element records, whole-file single-rank read (LoadBinary.h:156-246).
struct BinaryCase {
  int ndim = 0, nnod = 0, nface = 0, n_nodes = 0, n_elements = 0;
  std::vector<double> records;  // [Nn][2*ndim+2]
  std::vector<double> x;        // [Nn][ndim]
  std::vector<int> conn, bc;
  // adaptive elements from the "adap" file when control adap is set (LoadBinary.h:247-261):
  // ids, refine levels, and Hnm(N, M) at [k][N + nnod*M] (the Tensor storage, as written)
  std::vector<int> adap_el, adap_level;
  std::vector<double> adap_hnm;

  BinaryCase() = default;
  BinaryCase(const std::string& dir, const CaseConfig& cfg) {
    ndim = cfg.ci("ndim", 2);
    nnod = cfg.ci("nnod", ndim == 2 ? 4 : 8);
    nface = ndim == 2 ? 4 : 6;
    n_nodes = cfg.ci("nodes", 0);
    n_elements = cfg.ci("elements", 0);
    const int rs = 2 * ndim + 2;
    records.resize((size_t)n_nodes * rs);
    read_all(dir + "/binarynodes", records.data(), records.size() * sizeof(double));
    std::vector<int> el((size_t)n_elements * (nnod + nface));
    read_all(dir + "/binaryelements", el.data(), el.size() * sizeof(int));
    x.resize((size_t)n_nodes * ndim);
    for (int n = 0; n < n_nodes; n++)
      for (int k = 0; k < ndim; k++) x[(size_t)n * ndim + k] = records[(size_t)n * rs + k];
    conn.resize((size_t)n_elements * nnod);
    bc.resize((size_t)n_elements * nface);
    for (int e = 0; e < n_elements; e++) {
      for (int k = 0; k < nnod; k++) conn[(size_t)e * nnod + k] = el[(size_t)e * (nnod + nface) + k];
      for (int k = 0; k < nface; k++) bc[(size_t)e * nface + k] = el[(size_t)e * (nnod + nface) + nnod + k];
    }
    if (cfg.ci("adap", 0)) read_adap(dir + "/adap");
  }
  // "elno adap refine_level" then the Tensor serialisation: type, ndim, extents, data
  // (TensorStream.h:95-145); records with adap = 0 are skipped
  void read_adap(const std::string& path) {
    std::ifstream in(path.c_str());
    if (!in) throw std::runtime_error("cannot open " + path);
    int e, flag, level, nd;
    std::string type;
    while (in >> e >> flag >> level >> type >> nd) {
      int ext[2] = {1, 1};
      for (int k = 0; k < nd && k < 2; k++) in >> ext[k];
      if (nd != 2 || ext[0] != nnod || ext[1] != nnod || e < 0 || e >= n_elements)
        throw std::runtime_error("adap: bad record for element " + std::to_string(e));
      std::vector<double> h((size_t)nnod * nnod);
      for (double& v : h) in >> v;
      if (!in) throw std::runtime_error("adap: short record for element " + std::to_string(e));
      if (!flag) continue;
      adap_el.push_back(e);
      adap_level.push_back(level);
      adap_hnm.insert(adap_hnm.end(), h.begin(), h.end());
    }
  }
  static void read_all(const std::string& p, void* dst, size_t bytes) {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + p);
    size_t got = std::fread(dst, 1, bytes, f);
    std::fclose(f);
    if (got != bytes) throw std::runtime_error("short read of " + p);
  }
  cfdv_mesh mesh() const {
    cfdv_mesh m;
    m.ndim = ndim;
    m.n_nodes = n_nodes;
    m.n_elements = n_elements;
    m.x = x.data();
    m.conn = conn.data();
    m.bc = bc.data();
    return m;
  }
};

inline void check(cfdv_ctx* ctx, int rc, const char* what) {
  if (rc) throw std::runtime_error(std::string(what) + ": " + (ctx ? cfdv_last_error(ctx) : "") + " (status " +
                                   std::to_string(rc) + ")");
}

// Device-resident FDV step: formation, GMRES solve and update behind the reference's
// GMRESbase interface shape (iterate / update).
class GpuFDV {
 public:
  GpuFDV(const BinaryCase& c, const cfdv_params& p) : ndim_(c.ndim), n_nodes_(c.n_nodes), n_el_(c.n_elements) {
    cfdv_mesh m = c.mesh();
    int rc = cfdv_create(&m, &p, &ctx_);
    if (rc) {
      std::string msg = ctx_ ? cfdv_last_error(ctx_) : "";
      if (ctx_) cfdv_destroy(ctx_);
      throw std::runtime_error("cfdv_create: " + msg);
    }
    check(ctx_, cfdv_load_node_records(ctx_, c.records.data(), c.n_nodes), "load_node_records");
    if (!c.adap_el.empty())
      check(ctx_, cfdv_set_adaptive(ctx_, (int)c.adap_el.size(), c.adap_el.data(), c.adap_hnm.data()), "set_adaptive");
  }
  ~GpuFDV() { cfdv_destroy(ctx_); }
  GpuFDV(const GpuFDV&) = delete;
  GpuFDV& operator=(const GpuFDV&) = delete;

  double cfl(double cfl) { double dt; check(ctx_, cfdv_cfl(ctx_, cfl, &dt), "cfl"); return dt; }
  void form(double dt, int precision) { check(ctx_, cfdv_form(ctx_, dt, precision), "form"); }
  void iterate(const cfdv_gmres_opts& o, cfdv_gmres_report* rep) { check(ctx_, cfdv_gmres(ctx_, &o, rep), "gmres"); }
  void update() { check(ctx_, cfdv_update(ctx_), "update"); }
  std::vector<double> rms() {
    std::vector<double> r(ndim_ + 2);
    check(ctx_, cfdv_rms(ctx_, r.data()), "rms");
    return r;
  }
  std::vector<double> state() {
    std::vector<double> U((size_t)n_nodes_ * (ndim_ + 2));
    check(ctx_, cfdv_get_state(ctx_, U.data(), nullptr, U.size()), "get_state");
    return U;
  }
  // s1..s4 of the current state: formation at any dt gives them (they depend on U only)
  std::vector<double> fdv_params() {
    std::vector<double> s((size_t)n_el_ * 4);
    check(ctx_, cfdv_get_fdv_params(ctx_, s.data()), "fdv_params");
    return s;
  }
  cfdv_ctx* ctx() { return ctx_; }

 private:
  int ndim_, n_nodes_, n_el_;
  cfdv_ctx* ctx_ = nullptr;
};

// "tecplot_<iter>.plt" in the reference's FE block layout and number format
// (MPI_TecplotOut.h:189-371): primitives from NodeUnpack of U, cell-centred s1..s4.
inline std::string tecplot_name(int iter) {
  std::ostringstream s;
  s << (double)iter;  // to_string<double>(iter): 1000000 prints as 1e+06
  return "tecplot_" + s.str() + ".plt";
}

inline void tecplot_write(const std::string& path, const BinaryCase& c, const cfdv_params& p,
                          const std::vector<double>& U, const std::vector<double>* s, double time) {
  const int nd = c.ndim, ne = nd + 2, Nn = c.n_nodes;
  const double Cv = 1. / p.gamma / (p.gamma - 1.0) / (p.mach * p.mach);
  std::vector<double> rho(Nn), T(Nn), pr(Nn), v((size_t)Nn * nd);
  for (int n = 0; n < Nn; n++) {  // NodeUnpack.h:9-29
    const double* u = &U[(size_t)n * ne];
    rho[n] = u[0];
    double vsqr = 0;
    for (int i = 0; i < nd; i++) {
      v[(size_t)n * nd + i] = u[1 + i] / u[0];
      vsqr += v[(size_t)n * nd + i] * v[(size_t)n * nd + i];
    }
    const double E = u[nd + 1] / u[0], e = E - 0.5 * vsqr;
    T[n] = e / Cv;
    pr[n] = rho[n] * (p.gamma - 1.0) * e;
  }
  std::ofstream t(path.c_str());
  const bool ele = (s != nullptr);
  t << "title = \"Output at time = " << time << " \"" << std::endl;
  t << "variables = \"x\", \"y\",";
  if (nd == 3) t << " \"z\",";
  t << "\"rho\", \"u\", \"v\",";
  if (nd == 3) t << " \"w\",";
  t << "\"T\", \"p\",";
  if (ele) t << "\"s1\", \"s2\", \"s3\", \"s4\", ";
  t << std::endl;
  t << "zone E=" << c.n_elements << ", N=" << Nn;
  t << ", DATAPACKING=BLOCK, ZONETYPE=FEQUADRILATERAL";  // nnod != 3
  if (nd == 3) t << ", DATAPACKING=BLOCK, ZONETYPE=FEBRICK";
  t << std::endl;
  if (ele) t << (nd == 2 ? "VARLOCATION=([8,9,10,11]=CellCentered)" : "VARLOCATION=([10,11,12,13]=CellCentered)")
             << std::endl;
  t << std::endl;
  t << std::scientific << std::endl;
  t << std::setprecision(7) << std::endl;
  auto block = [&](auto get, const char* sep) {
    for (int n = 0; n < Nn; n++) {
      t << get(n) << sep;
      if (n % 100 == 0 && n != 0) t << std::endl;
    }
    t << std::endl;
  };
  for (int k = 0; k < nd; k++) block([&](int n) { return c.x[(size_t)n * nd + k]; }, " ");
  block([&](int n) { return rho[n]; }, " ");
  for (int k = 0; k < nd; k++) block([&](int n) { return v[(size_t)n * nd + k]; }, " ");
  block([&](int n) { return T[n]; }, " ");
  block([&](int n) { return pr[n]; }, "\t");
  if (ele)
    for (int k = 0; k < 4; k++)
      for (int e = 0; e < c.n_elements; e++) {
        t << (*s)[(size_t)e * 4 + k] << "\t";
        if (e % 100 == 0 && e != 0) t << std::endl;
      }
  for (int e = 0; e < c.n_elements; e++) {
    for (int k = 0; k < c.nnod; k++) t << c.conn[(size_t)e * c.nnod + k] + 1 << " ";
    t << std::endl;
  }
}

// Checkpoint of the state (MPIBinaryConfiguration.h:148-161, SaveBinary.h:34-150): the case
// directory <dir>/<iter>/ with binarynodes {x[ndim], rho, v[ndim], T} from NodeUnpack of U,
// binaryelements {node[nnod], bc[nface]}, the aero file, a single-rank MPIBreakdown, and the
// control file with iter = <iter>, so that the run resumes from it (main.cpp:177, control
// "iter").  The reference writes its 3D records with the 2D struct (SaveBinary.h:48-52,
// 110-116); here both layouts are the ones LoadBinary reads (LoadBinary.h:20-48).
inline void write_case_dir(const std::string& out, const BinaryCase& c, const std::map<std::string, std::string>& control,
                           const std::map<std::string, std::string>& aero, const cfdv_params& p,
                           const std::vector<double>& U);

inline void save_case(const std::string& dir, int iter, const BinaryCase& c, const CaseConfig& cfg,
                      const cfdv_params& p, const std::vector<double>& U) {
  const std::string out = dir + "/" + std::to_string(iter);
  std::map<std::string, std::string> ctl = cfg.control;
  ctl["iter"] = std::to_string(iter);
  write_case_dir(out, c, ctl, cfg.aero, p, U);
}

// the case directory `out` (created if needed) of mesh c and conserved state U
inline void write_case_dir(const std::string& out, const BinaryCase& c, const std::map<std::string, std::string>& control,
                           const std::map<std::string, std::string>& aero, const cfdv_params& p,
                           const std::vector<double>& U) {
  if (std::system(("mkdir -p '" + out + "'").c_str()) != 0) throw std::runtime_error("cannot create " + out);
  const int nd = c.ndim, ne = nd + 2, rs = 2 * nd + 2;
  const double Cv = 1. / p.gamma / (p.gamma - 1.0) / (p.mach * p.mach);
  std::vector<double> rec((size_t)c.n_nodes * rs);
  for (int n = 0; n < c.n_nodes; n++) {  // NodeUnpack.h:9-29
    const double* u = &U[(size_t)n * ne];
    double* r = &rec[(size_t)n * rs];
    for (int k = 0; k < nd; k++) r[k] = c.x[(size_t)n * nd + k];
    r[nd] = u[0];
    double vsqr = 0;
    for (int k = 0; k < nd; k++) {
      r[nd + 1 + k] = u[1 + k] / u[0];
      vsqr += r[nd + 1 + k] * r[nd + 1 + k];
    }
    r[2 * nd + 1] = (u[nd + 1] / u[0] - 0.5 * vsqr) / Cv;
  }
  std::vector<int> el((size_t)c.n_elements * (c.nnod + c.nface));
  for (int e = 0; e < c.n_elements; e++) {
    for (int k = 0; k < c.nnod; k++) el[(size_t)e * (c.nnod + c.nface) + k] = c.conn[(size_t)e * c.nnod + k];
    for (int k = 0; k < c.nface; k++) el[(size_t)e * (c.nnod + c.nface) + c.nnod + k] = c.bc[(size_t)e * c.nface + k];
  }
  auto write = [&](const std::string& name, const void* data, size_t bytes) {
    FILE* f = std::fopen((out + "/" + name).c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + out + "/" + name);
    const size_t put = std::fwrite(data, 1, bytes, f);
    std::fclose(f);
    if (put != bytes) throw std::runtime_error("short write of " + out + "/" + name);
  };
  write("binarynodes", rec.data(), rec.size() * sizeof(double));
  write("binaryelements", el.data(), el.size() * sizeof(int));
  if (!c.adap_el.empty()) {  // SaveBinary.h:153-168 (write_adap), at full precision
    std::ofstream a((out + "/adap").c_str());
    a << std::setprecision(17);
    const size_t nn = (size_t)c.nnod * c.nnod;
    for (size_t k = 0; k < c.adap_el.size(); k++) {
      a << c.adap_el[k] << " 1 " << c.adap_level[k] << " double 2 " << c.nnod << " " << c.nnod;
      for (size_t i = 0; i < nn; i++) a << " " << c.adap_hnm[k * nn + i];
      a << "\n";
    }
  }
  auto kv = [&](const std::string& name, std::map<std::string, std::string> m) {
    std::ofstream f((out + "/" + name).c_str());
    for (const auto& it : m) f << it.first << " = " << it.second << "\n";
  };
  kv("control", control);
  kv("aero", aero);
  std::ofstream b((out + "/MPIBreakdown").c_str());  // one rank (MPI_Breakdown.h:23-70)
  b << "1\n";
  b << "elemin, elemax, nodemin, nodemax, nedgenode_l, nedgenode_r, NodeIteratorMin, NodeIteratorMax\n";
  b << "0 " << c.n_elements << " 0 " << c.n_nodes - 1 << " 0 0 0 " << c.n_nodes - 1 << "\n";
}

// ASCII case directory -> binary case directory: the reference's CONVERT (ConvertMain.cpp:20-66:
// AsciiLoad.h:27-340, then NodeUnpack and SaveBinary's write_nodes / write_elements /
// write_adap, with a one-rank MPIBreakdown).  src holds control and aero ("key = value"),
// nodes ("number x[ndim] U[ndim+2]": conserved variables, 1-based numbers), elements
// ("number node[nnod]", 1-based), faces ("element face bc node[nbnod]": 0-based element, the
// bc goes to the element's slot `face`, a later line for the same slot wins) and, with
// control adap, adap (the format LoadBinary reads).  Lines with fewer numbers than their
// record are skipped, as AsciiLoad does; a node or element that no line defines is an error.
// Differences from the reference, on purpose: the 3D records are written in LoadBinary's
// layout (SaveBinary uses the 2D struct for them), and Hnm keeps full precision (AsciiLoad's
// add_adap re-prints it through to_string).
inline std::vector<std::vector<double>> read_number_lines(const std::string& path, bool required) {
  std::vector<std::vector<double>> rows;
  std::ifstream in(path.c_str());
  if (!in) {
    if (required) throw std::runtime_error("cannot open " + path);
    return rows;
  }
  std::string line;
  while (std::getline(in, line)) {
    std::vector<double> r;
    const char* p = line.c_str();
    char* end;
    for (;;) {
      while (*p == ' ' || *p == '\t' || *p == '\r') p++;
      if (!*p) break;
      const double v = std::strtod(p, &end);
      if (end == p) {  // a word (the Tensor type name in adap lines): kept as 0
        while (*p && *p != ' ' && *p != '\t') p++;
        r.push_back(0.0);
        continue;
      }
      r.push_back(v);
      p = end;
    }
    if (!r.empty()) rows.push_back(r);
  }
  return rows;
}

inline void convert_ascii(const std::string& src, const std::string& dst) {
  CaseConfig cfg(src);
  const cfdv_params p = cfg.params();
  BinaryCase c;
  c.ndim = cfg.ci("ndim", 2);
  c.nnod = cfg.ci("nnod", c.ndim == 2 ? 4 : 8);
  c.nface = c.ndim == 2 ? 4 : 6;
  c.n_nodes = cfg.ci("nodes", 0);
  c.n_elements = cfg.ci("elements", 0);
  const int nd = c.ndim, ne = nd + 2, nn = c.nnod, nbnod = cfg.ci("nbnod", nd == 2 ? 2 : 4);
  if (c.n_nodes <= 0 || c.n_elements <= 0) throw std::runtime_error("convert: control needs nodes and elements");
  c.x.assign((size_t)c.n_nodes * nd, 0.0);
  std::vector<double> U((size_t)c.n_nodes * ne, 0.0);
  std::vector<char> seen(c.n_nodes, 0), eseen(c.n_elements, 0);
  for (const auto& r : read_number_lines(src + "/nodes", true)) {  // AsciiLoad.h:188-236
    if ((int)r.size() < 2 * nd + 3) continue;
    const int i = (int)r[0] - 1;
    if (i < 0 || i >= c.n_nodes) throw std::runtime_error("convert: node number out of range");
    for (int j = 0; j < nd; j++) c.x[(size_t)i * nd + j] = r[1 + j];
    for (int j = 0; j < ne; j++) U[(size_t)i * ne + j] = r[1 + nd + j];
    seen[i] = 1;
  }
  c.conn.assign((size_t)c.n_elements * nn, 0);
  c.bc.assign((size_t)c.n_elements * c.nface, 0);
  for (const auto& r : read_number_lines(src + "/elements", true)) {  // AsciiLoad.h:239-253
    if ((int)r.size() < nn + 1) continue;
    const int i = (int)r[0] - 1;
    if (i < 0 || i >= c.n_elements) throw std::runtime_error("convert: element number out of range");
    for (int j = 0; j < nn; j++) {
      const int n = (int)r[1 + j] - 1;
      if (n < 0 || n >= c.n_nodes) throw std::runtime_error("convert: element node out of range");
      c.conn[(size_t)i * nn + j] = n;
    }
    eseen[i] = 1;
  }
  for (int i = 0; i < c.n_nodes; i++)
    if (!seen[i]) throw std::runtime_error("convert: node " + std::to_string(i + 1) + " is not defined");
  for (int i = 0; i < c.n_elements; i++)
    if (!eseen[i]) throw std::runtime_error("convert: element " + std::to_string(i + 1) + " is not defined");
  for (const auto& r : read_number_lines(src + "/faces", true)) {  // AsciiLoad.h:256-313, SaveBinary.h:68-71
    if ((int)r.size() < 3 + nbnod) continue;
    const int e = (int)r[0], f = (int)r[1];
    if (e < 0 || e >= c.n_elements || f < 0 || f >= c.nface) throw std::runtime_error("convert: bad face line");
    c.bc[(size_t)e * c.nface + f] = (int)r[2];
  }
  if (cfg.ci("adap", 0))  // AsciiLoad.h:116-158
    for (const auto& r : read_number_lines(src + "/adap", true)) {
      if ((int)r.size() < 7 + nn * nn || !(int)r[1]) continue;
      const int e = (int)r[0];
      if (e < 0 || e >= c.n_elements) throw std::runtime_error("convert: adap element out of range");
      c.adap_el.push_back(e);
      c.adap_level.push_back((int)r[2]);
      c.adap_hnm.insert(c.adap_hnm.end(), r.begin() + 7, r.begin() + 7 + nn * nn);
    }
  c.records.clear();
  write_case_dir(dst, c, cfg.control, cfg.aero, p, U);
}

// EnSight Gold ASCII time series (the reference's EnsightOut.h:9-13 is an empty stub): one
// geometry file (one part, quad4 or hexa8, z = 0 in 2D), per output step the node
// variables rho, velocity (3 components), T and p from NodeUnpack of U and the element
// variables s1..s4, and a case file listing every step written so far.
//   <dir>/cfdv.case, <dir>/cfdv.geo, <dir>/cfdv.<var>.<00000..>
class EnsightSeries {
 public:
  EnsightSeries(const std::string& dir, const BinaryCase& c) : dir_(dir), c_(c) {
    if (std::system(("mkdir -p '" + dir_ + "'").c_str()) != 0) throw std::runtime_error("cannot create " + dir_);
    std::ofstream g((dir_ + "/cfdv.geo").c_str());
    if (!g) throw std::runtime_error("cannot write " + dir_ + "/cfdv.geo");
    g << "CFDV FDV solution\n" << c.ndim << "D unstructured mesh\n";
    g << "node id off\nelement id off\n";
    g << "part\n" << std::setw(10) << 1 << "\nflow field\ncoordinates\n" << std::setw(10) << c.n_nodes << "\n";
    g << std::scientific << std::setprecision(5);
    for (int k = 0; k < 3; k++)
      for (int n = 0; n < c.n_nodes; n++) g << std::setw(12) << (k < c.ndim ? c.x[(size_t)n * c.ndim + k] : 0.0) << "\n";
    g << element_type() << "\n" << std::setw(10) << c.n_elements << "\n";
    for (int e = 0; e < c.n_elements; e++) {
      for (int k = 0; k < c.nnod; k++) g << std::setw(10) << c.conn[(size_t)e * c.nnod + k] + 1;
      g << "\n";
    }
  }

  void write(double time, const cfdv_params& p, const std::vector<double>& U, const std::vector<double>* s) {
    const int nd = c_.ndim, ne = nd + 2, Nn = c_.n_nodes, step = (int)times_.size();
    const double Cv = 1. / p.gamma / (p.gamma - 1.0) / (p.mach * p.mach);
    std::vector<double> rho(Nn), T(Nn), pr(Nn), v((size_t)Nn * 3, 0.0);
    for (int n = 0; n < Nn; n++) {  // NodeUnpack.h:9-29
      const double* u = &U[(size_t)n * ne];
      rho[n] = u[0];
      double vsqr = 0;
      for (int i = 0; i < nd; i++) {
        v[(size_t)i * Nn + n] = u[1 + i] / u[0];
        vsqr += v[(size_t)i * Nn + n] * v[(size_t)i * Nn + n];
      }
      const double e = u[nd + 1] / u[0] - 0.5 * vsqr;
      T[n] = e / Cv;
      pr[n] = rho[n] * (p.gamma - 1.0) * e;
    }
    node_var("rho", step, rho);
    node_var("velocity", step, v);
    node_var("T", step, T);
    node_var("p", step, pr);
    if (s) {
      has_s_ = true;
      for (int k = 0; k < 4; k++) {
        std::vector<double> sk(c_.n_elements);
        for (int e = 0; e < c_.n_elements; e++) sk[e] = (*s)[(size_t)e * 4 + k];
        element_var("s" + std::to_string(k + 1), step, sk);
      }
    }
    times_.push_back(time);
    write_case();
  }

  static std::string var_file(const std::string& var, int step) {
    std::ostringstream f;
    f << "cfdv." << var << "." << std::setw(5) << std::setfill('0') << step;
    return f.str();
  }

 private:
  const char* element_type() const { return c_.ndim == 2 ? "quad4" : "hexa8"; }

  // scalar (values.size() == n_nodes) or 3-component vector (component-major)
  void node_var(const std::string& var, int step, const std::vector<double>& values) {
    std::ofstream f((dir_ + "/" + var_file(var, step)).c_str());
    if (!f) throw std::runtime_error("cannot write " + dir_ + "/" + var_file(var, step));
    f << var << " at step " << step << "\npart\n" << std::setw(10) << 1 << "\ncoordinates\n";
    f << std::scientific << std::setprecision(5);
    for (double x : values) f << std::setw(12) << x << "\n";
  }

  void element_var(const std::string& var, int step, const std::vector<double>& values) {
    std::ofstream f((dir_ + "/" + var_file(var, step)).c_str());
    if (!f) throw std::runtime_error("cannot write " + dir_ + "/" + var_file(var, step));
    f << var << " at step " << step << "\npart\n" << std::setw(10) << 1 << "\n" << element_type() << "\n";
    f << std::scientific << std::setprecision(5);
    for (double x : values) f << std::setw(12) << x << "\n";
  }

  void write_case() const {
    std::ofstream f((dir_ + "/cfdv.case").c_str());
    f << "FORMAT\ntype: ensight gold\n\nGEOMETRY\nmodel: cfdv.geo\n\nVARIABLE\n";
    f << "scalar per node: 1 rho cfdv.rho.*****\n";
    f << "vector per node: 1 velocity cfdv.velocity.*****\n";
    f << "scalar per node: 1 T cfdv.T.*****\n";
    f << "scalar per node: 1 p cfdv.p.*****\n";
    if (has_s_)
      for (int k = 1; k <= 4; k++) f << "scalar per element: 1 s" << k << " cfdv.s" << k << ".*****\n";
    f << "\nTIME\ntime set: 1\nnumber of steps: " << times_.size() << "\nfilename start number: 0\n";
    f << "filename increment: 1\ntime values:\n";
    f << std::scientific << std::setprecision(9);
    for (double t : times_) f << t << "\n";
  }

  std::string dir_;
  const BinaryCase& c_;
  std::vector<double> times_;
  bool has_s_ = false;
};

// one "iter\t(rms) " line per step (MPI_RMSError.h:56-69)
inline void rms_append(const std::string& path, int iter, const std::vector<double>& rms) {
  std::ofstream f(path.c_str(), std::ios::app);
  f << iter << "\t";
  for (double r : rms) f << r << " ";
  f << std::endl;
}

}  // namespace cfdv_host
