// The persistent solve's neighbour sets (cfdv_b200/csrc/neighbour_sets.h) behind a C entry point,
// so the CPU tests can check them against the ownership they are derived from.
#include <cstring>

#include "../../cfdv_b200/csrc/neighbour_sets.h"

extern "C" int emu_neighbour_sets(int ndim, int n_nodes, int n_elements, const int* conn, const int* csr_ptr,
                                  const int* csr_idx, int blocks, int* out_ptr, int* out_idx, int idx_cap) {
  std::vector<int> ptr, idx;
  if (!cfdv::persistent_neighbour_sets(ndim, n_nodes, n_elements, conn, csr_ptr, csr_idx, blocks, ptr, idx))
    return -1;
  if ((int)idx.size() > idx_cap) return -2;
  std::memcpy(out_ptr, ptr.data(), sizeof(int) * ptr.size());
  std::memcpy(out_idx, idx.data(), sizeof(int) * idx.size());
  return (int)idx.size();
}
