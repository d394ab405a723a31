// Neighbour sets of the persistent GMRES solve's delayed-CGS2 step (gmres_persistent.cu), host
// only.  Block b of the solve owns nodes [b pn, (b+1) pn), pn = ceil(n_nodes / nb), and in 2D
// elements [b per, (b+1) per), per = ceil(E / nb).  Its element pass reads x at the nodes of its
// elements and its node pass reads the products of the elements at its nodes, so before each
// it waits for the blocks that write those.
#pragma once

#include <algorithm>
#include <vector>

namespace cfdv {

// CSR over the blocks: rows [0, nb] list the blocks owning nodes of a block's elements, rows
// [nb + 1, 2 nb + 1] the blocks owning elements at a block's nodes (a block itself excluded).
// False when the sets do not apply (3D, whose element waves interleave over the grid) or when
// a set has more than 32 blocks (one polling lane each).
inline bool persistent_neighbour_sets(int ndim, int n_nodes, int n_elements, const int* conn, const int* csr_ptr,
                                      const int* csr_idx, int blocks, std::vector<int>& ptr, std::vector<int>& idx) {
  constexpr int kMaxSet = 32;  // one polling lane each
  if (ndim != 2 || blocks <= 0 || n_nodes <= 0 || n_elements <= 0) return false;
  constexpr int nnod = 4;
  const int nb = blocks, pn = (n_nodes + nb - 1) / nb, per = (n_elements + nb - 1) / nb;
  ptr.assign(2 * (nb + 1), 0);
  idx.clear();
  std::vector<int> seen(nb, -1);
  auto add = [&](int b, int o) {
    if (o != b && seen[o] != b) {
      seen[o] = b;
      idx.push_back(o);
    }
  };
  for (int b = 0; b < nb; b++) {  // blocks owning the nodes of b's elements
    ptr[b] = (int)idx.size();
    const int e0 = std::min(n_elements, b * per), e1 = std::min(n_elements, e0 + per);
    for (int e = e0; e < e1; e++)
      for (int l = 0; l < nnod; l++) add(b, conn[(size_t)e * nnod + l] / pn);
    if ((int)idx.size() - ptr[b] > kMaxSet) return false;
  }
  ptr[nb] = (int)idx.size();
  std::fill(seen.begin(), seen.end(), -1);
  for (int b = 0; b < nb; b++) {  // blocks owning the elements at b's nodes
    ptr[nb + 1 + b] = (int)idx.size();
    const int n0 = std::min(n_nodes, b * pn), n1 = std::min(n_nodes, n0 + pn);
    for (int nd = n0; nd < n1; nd++)
      for (int p = csr_ptr[nd]; p < csr_ptr[nd + 1]; p++) add(b, (csr_idx[p] / nnod) / per);
    if ((int)idx.size() - ptr[nb + 1 + b] > kMaxSet) return false;
  }
  ptr[2 * nb + 1] = (int)idx.size();
  return true;
}

}  // namespace cfdv
