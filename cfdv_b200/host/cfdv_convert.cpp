// cfdv_convert: an ASCII case directory (control, aero, nodes, elements, faces[, adap]) to the
// binary case directory the solver reads, as the reference's CONVERT program does
// (ConvertMain.cpp).  The conversion is cfdv_host::convert_ascii (cfdv_host.hpp).
//   cfdv_convert <ascii_dir> <binary_dir>
#include <cstdio>
#include <exception>

#include "cfdv_host.hpp"

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <ascii_dir> <binary_dir>\n", argv[0]);
    return 2;
  }
  try {
    cfdv_host::convert_ascii(argv[1], argv[2]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cfdv_convert: %s\n", e.what());
    return 1;
  }
  return 0;
}
