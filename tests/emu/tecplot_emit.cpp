// Test harness: writes tecplot_<iter>.plt with the host writer of the C++ host layer
// (cfdv_b200/host/cfdv_host.hpp) from a state U and s1..s4 given as raw float64 files,
// so the writer can be compared byte-for-byte with the reference's MPI_TecplotOut
// without a GPU.  Usage: tecplot_emit <case_dir> <U.bin> <s.bin> <iter> <time> <out_dir>
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
  cfdv_host::tecplot_write(std::string(argv[6]) + "/" + cfdv_host::tecplot_name(iter), c, cfg.params(), U, &s,
                           std::atof(argv[5]));
  return 0;
}
