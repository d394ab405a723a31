// Test harness: writes tecplot_<iter>.plt with the host writer of the C++ host layer
// (cfdv_b200/host/cfdv_host.hpp) from a state U and s1..s4 given as raw float64 files,
// so the writer can be compared byte-for-byte with the reference's MPI_TecplotOut
// without a GPU; with a trailing "save" it writes the checkpoint directory
// <out_dir>/<iter>/ of save_case instead, and with "ensight" an EnSight Gold series of two
// steps (times <time> and 2 <time>) of the same state into <out_dir>.
// Usage: tecplot_emit <case_dir> <U.bin> <s.bin> <iter> <time> <out_dir> [save|ensight]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../cfdv_b200/host/cfdv_host.hpp"

int main(int argc, char** argv) {
  if (argc < 7) return 2;
  cfdv_host::CaseConfig cfg(argv[1]);
  cfdv_host::BinaryCase c(argv[1], cfg);
  std::vector<double> U((size_t)c.n_nodes * (c.ndim + 2)), s((size_t)c.n_elements * 4);
  cfdv_host::BinaryCase::read_all(argv[2], U.data(), U.size() * sizeof(double));
  cfdv_host::BinaryCase::read_all(argv[3], s.data(), s.size() * sizeof(double));
  const int iter = std::atoi(argv[4]);
  if (argc > 7 && std::string(argv[7]) == "save") {
    cfdv_host::save_case(argv[6], iter, c, cfg, cfg.params(), U);
    return 0;
  }
  if (argc > 7 && std::string(argv[7]) == "ensight") {
    cfdv_host::EnsightSeries es(argv[6], c);
    es.write(std::atof(argv[5]), cfg.params(), U, &s);
    es.write(2.0 * std::atof(argv[5]), cfg.params(), U, &s);
    return 0;
  }
  cfdv_host::tecplot_write(std::string(argv[6]) + "/" + cfdv_host::tecplot_name(iter), c, cfg.params(), U, &s,
                           std::atof(argv[5]));
  return 0;
}
