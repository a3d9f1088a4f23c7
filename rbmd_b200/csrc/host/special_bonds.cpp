// special_bonds.cpp -- per-atom special-bond rows from the topology, the way
// LammpsFullReader builds them (lammps_full_reader.cpp:2101-2230): bonds give
// 1-2 pairs, angles their end atoms (1-3), dihedrals their end atoms (1-4);
// a pair already present keeps its first band (1-2 over 1-3 over 1-4), each
// pair goes into both atoms' rows in that order, and nspecial holds the
// cumulative counts (n12, n12 + n13, n12 + n13 + n14).
#include <cstdint>
#include <set>
#include <utility>
#include <vector>

#include "rbx.h"
#include "special_bonds.h"

namespace rbx {
void set_error(const char* fmt, ...);
}

namespace rbx_host {

SpecialRows build_special(int n, int nb, const int64_t* bonds, int na, const int64_t* angles,
                          int nd, const int64_t* dihedrals) {
  SpecialRows r;
  r.part.assign(n, {});
  r.band.assign(n, {});
  std::set<std::pair<int64_t, int64_t>> seen;
  auto add = [&](int64_t a, int64_t b, int band) {
    if (a < 0 || b < 0 || a == b || a >= n || b >= n) return;
    if (!seen.insert(a < b ? std::make_pair(a, b) : std::make_pair(b, a)).second) return;
    r.part[a].push_back((int)b);
    r.band[a].push_back(band);
    r.part[b].push_back((int)a);
    r.band[b].push_back(band);
  };
  for (int k = 0; k < nb; ++k) add(bonds[2 * k], bonds[2 * k + 1], 0);
  for (int k = 0; k < na; ++k) add(angles[3 * k], angles[3 * k + 2], 1);
  for (int k = 0; k < nd; ++k) add(dihedrals[4 * k], dihedrals[4 * k + 3], 2);
  for (int i = 0; i < n; ++i) r.maxspecial = std::max(r.maxspecial, (int)r.part[i].size());
  return r;
}

void fill_special(const SpecialRows& r, int* nspecial, int* special) {
  const int n = (int)r.part.size();
  for (int i = 0; i < n; ++i) {
    int c[3] = {0, 0, 0};
    for (size_t k = 0; k < r.part[i].size(); ++k) {
      special[(size_t)i * r.maxspecial + k] = r.part[i][k];
      ++c[r.band[i][k]];
    }
    for (size_t k = r.part[i].size(); k < (size_t)r.maxspecial; ++k)
      special[(size_t)i * r.maxspecial + k] = 0;
    nspecial[3 * i] = c[0];
    nspecial[3 * i + 1] = c[0] + c[1];
    nspecial[3 * i + 2] = c[0] + c[1] + c[2];
  }
}

}  // namespace rbx_host

extern "C" int rbx_special_build(int n, int nbonds, const int64_t* bonds, int nangles,
                                 const int64_t* angles, int ndihedrals, const int64_t* dihedrals,
                                 int* maxspecial, int* nspecial, int* special) {
  if (n < 0 || !maxspecial || (nbonds > 0 && !bonds) || (nangles > 0 && !angles) ||
      (ndihedrals > 0 && !dihedrals)) {
    rbx::set_error("rbx_special_build: invalid arguments");
    return RBX_ERR_INVALID;
  }
  const auto r = rbx_host::build_special(n, nbonds, bonds, nangles, angles, ndihedrals, dihedrals);
  *maxspecial = r.maxspecial;
  if (nspecial && special) rbx_host::fill_special(r, nspecial, special);
  return RBX_OK;
}
