// special_bonds.h -- special-bond rows from the topology (special_bonds.cpp).
#pragma once
#include <cstdint>
#include <vector>

namespace rbx_host {

struct SpecialRows {
  int maxspecial = 0;
  std::vector<std::vector<int>> part;  // partner atom indices per atom, 1-2 first
  std::vector<std::vector<int>> band;  // 0: 1-2, 1: 1-3, 2: 1-4
};
// Atom indices 0..n-1 in bonds [nb][2], angles [na][3], dihedrals [nd][4].
SpecialRows build_special(int n, int nb, const int64_t* bonds, int na, const int64_t* angles,
                          int nd, const int64_t* dihedrals);
// nspecial [n][3] cumulative counts, special [n][maxspecial] (zero padded).
void fill_special(const SpecialRows& r, int* nspecial, int* special);

}  // namespace rbx_host
