// lammps_data.cpp -- LAMMPS data file reader and charge-style writer.
#include "lammps_data.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <unordered_map>

#include "units.h"

namespace rbx_host {
namespace {

enum class Section {
  Header, Masses, PairCoeffs, OtherCoeffs, Atoms, Velocities, Bonds, Angles, Dihedrals, Impropers
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) --b;
  return s.substr(a, b - a);
}

std::string strip_comment(const std::string& s) {
  const size_t h = s.find('#');
  return trim(h == std::string::npos ? s : s.substr(0, h));
}

bool starts(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }

bool ends(const std::string& s, const char* p) {
  const size_t n = strlen(p);
  return s.size() >= n && s.compare(s.size() - n, n, p) == 0;
}

// Section keyword at the start of a trimmed line (DetectSection).
bool detect(const std::string& t, Section* sec) {
  struct K {
    const char* key;
    Section sec;
  };
  static const K keys[] = {{"Masses", Section::Masses},
                           {"Pair Coeffs", Section::PairCoeffs},
                           {"PairIJ Coeffs", Section::PairCoeffs},
                           {"Bond Coeffs", Section::OtherCoeffs},
                           {"Angle Coeffs", Section::OtherCoeffs},
                           {"Dihedral Coeffs", Section::OtherCoeffs},
                           {"Improper Coeffs", Section::OtherCoeffs},
                           {"Atoms", Section::Atoms},
                           {"Velocities", Section::Velocities},
                           {"Bonds", Section::Bonds},
                           {"Angles", Section::Angles},
                           {"Dihedrals", Section::Dihedrals},
                           {"Impropers", Section::Impropers}};
  for (const K& k : keys)
    if (starts(t, k.key)) {
      *sec = k.sec;
      return true;
    }
  return false;
}

// Whitespace-separated numbers of a line, parsed in order.
struct Fields {
  const char* p;
  bool ok = true;
  explicit Fields(const std::string& s) : p(s.c_str()) {}
  double real() {
    char* end = nullptr;
    errno = 0;
    const double v = strtod(p, &end);
    if (end == p || errno == ERANGE) ok = false;
    p = end;
    return v;
  }
  int64_t integer() {
    char* end = nullptr;
    errno = 0;
    const long long v = strtoll(p, &end, 10);
    if (end == p || errno == ERANGE) ok = false;
    // an integer field written as a real ("3.0") is accepted like istream >> double
    if (ok && *end == '.') {
      p = end;
      const double f = real();
      if (f != 0.0) ok = false;
      return v;
    }
    p = end;
    return v;
  }
  bool more() {
    while (*p == ' ' || *p == '\t') ++p;
    return *p != '\0';
  }
};

}  // namespace

std::string LammpsData::read(const std::string& path, const std::string& style_in) {
  std::ifstream in(path);
  if (!in) return "cannot open " + path;
  std::string style = style_in;
  Section sec = Section::Header;
  std::unordered_map<int64_t, size_t> index_of;
  char buf[256];
  std::string line;
  bool first = true;
  int64_t lineno = 0;
  auto fail = [&](const char* what) {
    snprintf(buf, sizeof buf, "%s:%lld: %s", path.c_str(), (long long)lineno, what);
    return std::string(buf);
  };
  while (std::getline(in, line)) {
    ++lineno;
    if (first) {  // the title line
      first = false;
      continue;
    }
    const std::string t = trim(line);
    if (t.empty()) continue;
    Section next;
    if (detect(t, &next)) {
      sec = next;
      if (sec == Section::Atoms && style.empty()) {
        const size_t h = t.find('#');
        if (h != std::string::npos) style = trim(t.substr(h + 1));
      }
      if (sec == Section::Atoms) {
        if (style != "atomic" && style != "charge" && style != "full")
          return fail("unknown or missing atom style (atomic, charge or full)");
        atom_style = style;
      }
      if (sec == Section::Masses || sec == Section::PairCoeffs) {
        if (n_atom_types <= 0) return fail("section before the atom type count");
        mass.resize(n_atom_types, 0.0);
        pair_eps.resize(n_atom_types, 0.0);
        pair_sigma.resize(n_atom_types, 0.0);
      }
      continue;
    }
    const std::string c = strip_comment(t);
    if (c.empty()) continue;
    Fields f(c);
    switch (sec) {
      case Section::Header: {
        if (ends(c, "atom types")) n_atom_types = (int)f.integer();
        else if (ends(c, "bond types")) n_bond_types = (int)f.integer();
        else if (ends(c, "angle types")) n_angle_types = (int)f.integer();
        else if (ends(c, "dihedral types")) n_dihedral_types = (int)f.integer();
        else if (ends(c, "improper types")) n_improper_types = (int)f.integer();
        else if (ends(c, "atoms")) n_atoms = f.integer();
        else if (ends(c, "bonds")) n_bonds = f.integer();
        else if (ends(c, "angles")) n_angles = f.integer();
        else if (ends(c, "dihedrals")) n_dihedrals = f.integer();
        else if (ends(c, "impropers")) n_impropers = f.integer();
        else if (c.find("xlo") != std::string::npos && c.find("xhi") != std::string::npos) {
          lo[0] = f.real();
          hi[0] = f.real();
        } else if (c.find("ylo") != std::string::npos && c.find("yhi") != std::string::npos) {
          lo[1] = f.real();
          hi[1] = f.real();
        } else if (c.find("zlo") != std::string::npos && c.find("zhi") != std::string::npos) {
          lo[2] = f.real();
          hi[2] = f.real();
        } else if (c.find("xy") != std::string::npos && c.find("xz") != std::string::npos &&
                   c.find("yz") != std::string::npos) {
          return fail("triclinic boxes are not supported (orthogonal boxes only)");
        }
        if (!f.ok) return fail("malformed header line");
        if (n_atoms > 0 && id.capacity() == 0) {
          id.reserve(n_atoms);
        }
        break;
      }
      case Section::Masses: {
        const int64_t ty = f.integer();
        const double m = f.real();
        if (!f.ok || ty < 1 || ty > n_atom_types) return fail("bad Masses line");
        mass[ty - 1] = m;
        has_masses = true;
        break;
      }
      case Section::PairCoeffs: {
        const int64_t ty = f.integer();
        const double e = f.real();
        const double s = f.real();
        if (!f.ok || ty < 1 || ty > n_atom_types) return fail("bad Pair Coeffs line");
        pair_eps[ty - 1] = e;
        pair_sigma[ty - 1] = s;
        has_pair_coeffs = true;
        break;
      }
      case Section::OtherCoeffs:
        break;  // bonded force fields are not on this path
      case Section::Atoms: {
        int64_t aid = 0, mol = 0, ty = 0;
        double aq = 0.0;
        aid = f.integer();
        if (atom_style == "full") mol = f.integer();
        ty = f.integer();
        if (atom_style != "atomic") aq = f.real();
        const double ax = f.real(), ay = f.real(), az = f.real();
        if (!f.ok) return fail("bad Atoms line");
        int im[3] = {0, 0, 0};
        if (f.more()) {
          for (int d = 0; d < 3; ++d) im[d] = (int)f.integer();
          if (!f.ok) return fail("bad image flags");
          has_images = true;
        }
        if (aid <= 0 || ty <= 0 || ty > n_atom_types) return fail("atom id or type out of range");
        if ((int64_t)id.size() >= n_atoms) return fail("more atoms than the header declares");
        if (!index_of.emplace(aid - 1, id.size()).second) return fail("duplicate atom id");
        id.push_back(aid - 1);
        type.push_back((int)(ty - 1));
        molecule.push_back(atom_style == "full" ? (mol > 0 ? (int)(mol - 1) : -1) : -1);
        q.push_back(aq);
        x.push_back(ax);
        y.push_back(ay);
        z.push_back(az);
        vx.push_back(0.0);
        vy.push_back(0.0);
        vz.push_back(0.0);
        image.insert(image.end(), im, im + 3);
        break;
      }
      case Section::Velocities: {
        const int64_t vid = f.integer();
        const double a = f.real(), b = f.real(), d = f.real();
        if (!f.ok || vid <= 0) return fail("bad Velocities line");
        const auto it = index_of.find(vid - 1);
        if (it == index_of.end()) return fail("velocity of an unknown atom");
        vx[it->second] = a;
        vy[it->second] = b;
        vz[it->second] = d;
        has_velocities = true;
        break;
      }
      default: {  // Bonds, Angles, Dihedrals, Impropers: id type atom...
        const int k = sec == Section::Bonds ? 2 : (sec == Section::Angles ? 3 : 4);
        std::vector<int>& tv = sec == Section::Bonds ? bond_type
                               : sec == Section::Angles ? angle_type
                               : sec == Section::Dihedrals ? dihedral_type
                                                           : improper_type;
        std::vector<int64_t>& av = sec == Section::Bonds ? bond_atoms
                                   : sec == Section::Angles ? angle_atoms
                                   : sec == Section::Dihedrals ? dihedral_atoms
                                                               : improper_atoms;
        f.integer();  // entry id
        const int64_t ty = f.integer();
        int64_t a[4] = {0, 0, 0, 0};
        for (int t2 = 0; t2 < k; ++t2) a[t2] = f.integer();
        if (!f.ok || ty <= 0) return fail("bad topology line");
        tv.push_back((int)(ty - 1));
        for (int t2 = 0; t2 < k; ++t2) {
          if (a[t2] <= 0) return fail("topology atom id out of range");
          av.push_back(a[t2] - 1);
        }
        break;
      }
    }
  }
  if ((int64_t)id.size() != n_atoms) {
    snprintf(buf, sizeof buf, "%s: %lld atoms declared, %lld read", path.c_str(),
             (long long)n_atoms, (long long)id.size());
    return buf;
  }
  const struct {
    const char* name;
    int64_t want;
    size_t got;
  } tops[] = {{"bonds", n_bonds, bond_type.size()},
              {"angles", n_angles, angle_type.size()},
              {"dihedrals", n_dihedrals, dihedral_type.size()},
              {"impropers", n_impropers, improper_type.size()}};
  for (const auto& t : tops)
    if ((int64_t)t.got != t.want) {
      snprintf(buf, sizeof buf, "%s: %lld %s declared, %lld read", path.c_str(),
               (long long)t.want, t.name, (long long)t.got);
      return buf;
    }
  for (int d = 0; d < 3; ++d)
    if (!(hi[d] > lo[d])) return path + ": missing or empty box bounds";
  return "";
}

std::string LammpsData::replicate(int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return "replicate values must be positive";
  if (nx == 1 && ny == 1 && nz == 1) return "";
  const int64_t base = (int64_t)id.size();
  int64_t id_span = 0, mol_span = 0;
  for (int64_t i = 0; i < base; ++i) {
    id_span = std::max(id_span, id[i] + 1);
    if (molecule[i] >= 0) mol_span = std::max(mol_span, (int64_t)molecule[i] + 1);
  }
  const double L[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const int rep[3] = {nx, ny, nz};
  double nhi[3];
  for (int d = 0; d < 3; ++d) nhi[d] = lo[d] + rep[d] * L[d];
  const LammpsData seed = *this;
  id.clear(); type.clear(); molecule.clear(); image.clear();
  q.clear(); x.clear(); y.clear(); z.clear(); vx.clear(); vy.clear(); vz.clear();
  bond_type.clear(); angle_type.clear(); dihedral_type.clear(); improper_type.clear();
  bond_atoms.clear(); angle_atoms.clear(); dihedral_atoms.clear(); improper_atoms.clear();
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const int64_t r = ((int64_t)iz * ny + iy) * nx + ix;
        const double shift[3] = {ix * L[0], iy * L[1], iz * L[2]};
        for (int64_t i = 0; i < base; ++i) {
          id.push_back(seed.id[i] + r * id_span);
          type.push_back(seed.type[i]);
          molecule.push_back(seed.molecule[i] >= 0 ? (int)(seed.molecule[i] + r * mol_span) : -1);
          q.push_back(seed.q[i]);
          vx.push_back(seed.vx[i]);
          vy.push_back(seed.vy[i]);
          vz.push_back(seed.vz[i]);
          const double p0[3] = {seed.x[i], seed.y[i], seed.z[i]};
          double p[3];
          for (int d = 0; d < 3; ++d) {
            const double u = p0[d] + seed.image[3 * i + d] * L[d] + shift[d];
            const double W = nhi[d] - lo[d];
            double img = floor((u - lo[d]) / W);
            double v = u - img * W;
            if (v >= nhi[d]) {  // rounding at the upper face
              v -= W;
              img += 1;
            }
            p[d] = v;
            image.push_back((int)img);
          }
          x.push_back(p[0]);
          y.push_back(p[1]);
          z.push_back(p[2]);
        }
        auto copy_top = [&](const std::vector<int>& st, const std::vector<int64_t>& sa, int k,
                            std::vector<int>& dt, std::vector<int64_t>& da) {
          dt.insert(dt.end(), st.begin(), st.end());
          for (int64_t a : sa) da.push_back(a + r * id_span);
          (void)k;
        };
        copy_top(seed.bond_type, seed.bond_atoms, 2, bond_type, bond_atoms);
        copy_top(seed.angle_type, seed.angle_atoms, 3, angle_type, angle_atoms);
        copy_top(seed.dihedral_type, seed.dihedral_atoms, 4, dihedral_type, dihedral_atoms);
        copy_top(seed.improper_type, seed.improper_atoms, 4, improper_type, improper_atoms);
      }
  for (int d = 0; d < 3; ++d) hi[d] = nhi[d];
  const int64_t nrep = (int64_t)nx * ny * nz;
  n_atoms *= nrep;
  n_bonds *= nrep;
  n_angles *= nrep;
  n_dihedrals *= nrep;
  n_impropers *= nrep;
  has_images = true;
  return "";
}

namespace {
// Seed of one atom's generator: the seed and atom id combined and passed
// through the SplitMix64 finaliser (MixVelocitySeed, lammps_full_reader.cpp:134-143).
uint64_t velocity_seed(uint64_t seed, uint64_t atom_id) {
  uint64_t v = seed + 0x9e3779b97f4a7c15ULL + (atom_id << 6) + (atom_id >> 2);
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
  return v ^ (v >> 31);
}
}  // namespace

std::string LammpsData::gauss_velocities(double temperature, const std::string& unit, int seed) {
  if (!std::isfinite(temperature) || temperature <= 0)
    return "velocity_type GAUSS requires execution.temperature[0] > 0";
  if (seed <= 0) return "velocity_type GAUSS requires a positive seed";
  UnitFactors u;
  try {
    u = UnitsOf(unit);
  } catch (const std::exception& ex) {
    return ex.what();
  }
  const size_t n = id.size();
  if (n == 0) return "";
  std::vector<double> m(n);
  for (size_t i = 0; i < n; ++i) {
    const double mi = has_masses ? mass[type[i]] : 0.0;
    if (!std::isfinite(mi) || mi <= 0)
      return "velocity_type GAUSS requires positive mass for every atom type";
    m[i] = mi;
  }
  double mtot = 0, p[3] = {0, 0, 0};
  std::vector<double>* v[3] = {&vx, &vy, &vz};
  for (size_t i = 0; i < n; ++i) {
    std::mt19937_64 rng(velocity_seed((uint64_t)seed, (uint64_t)(id[i] + 1)));
    std::normal_distribution<double> normal(0.0, 1.0);
    const double f = 1.0 / std::sqrt(m[i]);
    for (int d = 0; d < 3; ++d) {
      (*v[d])[i] = normal(rng) * f;
      p[d] += m[i] * (*v[d])[i];
    }
    mtot += m[i];
  }
  double twice_ke = 0;
  for (size_t i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) (*v[d])[i] -= p[d] / mtot;
    twice_ke += m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
  }
  twice_ke *= u.mvv2e;
  if (!(twice_ke > 0) || !std::isfinite(twice_ke))
    return "velocity_type GAUSS failed to create finite kinetic energy";
  const long long dof = 3LL * (long long)n - 3;
  if (dof <= 0) return "velocity_type GAUSS computed non-positive temperature DOF";
  const double scale = std::sqrt(temperature * (double)dof * u.kb / twice_ke);
  for (size_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) (*v[d])[i] *= scale;
  has_velocities = true;
  return "";
}

std::string write_lammps_charge(const std::string& path, const double lo[3], const double hi[3],
                                int n, int ntypes, const double* mass, const double* eps,
                                const double* sigma, const int64_t* id, const int* type,
                                const double* q, const double* x, const double* y,
                                const double* z, const double* vx, const double* vy,
                                const double* vz) {
  FILE* fp = fopen(path.c_str(), "w");
  if (!fp) return "cannot write " + path;
  fprintf(fp, "LAMMPS data file (atom_style charge)\n\n%d atoms\n%d atom types\n\n", n, ntypes);
  const char* ax[3] = {"x", "y", "z"};
  for (int d = 0; d < 3; ++d)
    fprintf(fp, "%.17g %.17g %slo %shi\n", lo[d], hi[d], ax[d], ax[d]);
  fprintf(fp, "\nMasses\n\n");
  for (int t = 0; t < ntypes; ++t) fprintf(fp, "%d %.17g\n", t + 1, mass[t]);
  fprintf(fp, "\nPair Coeffs # lj/cut/coul/long\n\n");
  for (int t = 0; t < ntypes; ++t) fprintf(fp, "%d %.17g %.17g\n", t + 1, eps[t], sigma[t]);
  fprintf(fp, "\nAtoms # charge\n\n");
  for (int i = 0; i < n; ++i)
    fprintf(fp, "%lld %d %.17g %.17g %.17g %.17g\n", (long long)id[i] + 1, type[i] + 1, q[i],
            x[i], y[i], z[i]);
  if (vx) {
    fprintf(fp, "\nVelocities\n\n");
    for (int i = 0; i < n; ++i)
      fprintf(fp, "%lld %.17g %.17g %.17g\n", (long long)id[i] + 1, vx[i], vy[i], vz[i]);
  }
  const bool ok = fclose(fp) == 0;
  return ok ? "" : "write error on " + path;
}

}  // namespace rbx_host

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#include "rbx.h"

namespace rbx {
void set_error(const char* fmt, ...);
}

struct rbx_lammps_data {
  rbx_host::LammpsData d;
};

extern "C" {

rbx_lammps_data* rbx_lammps_read(const char* path, const char* atom_style,
                                 const int* replicate) {
  if (!path) {
    rbx::set_error("rbx_lammps_read: null path");
    return nullptr;
  }
  auto* h = new rbx_lammps_data();
  std::string err = h->d.read(path, atom_style ? atom_style : "");
  if (err.empty() && replicate) err = h->d.replicate(replicate[0], replicate[1], replicate[2]);
  if (!err.empty()) {
    rbx::set_error("%s", err.c_str());
    delete h;
    return nullptr;
  }
  return h;
}

void rbx_lammps_free(rbx_lammps_data* h) { delete h; }

int rbx_lammps_gauss_velocities(rbx_lammps_data* h, double temperature, const char* unit,
                                int seed) {
  if (!h || !unit) {
    rbx::set_error("rbx_lammps_gauss_velocities: null argument");
    return RBX_ERR_INVALID;
  }
  const std::string err = h->d.gauss_velocities(temperature, unit, seed);
  if (!err.empty()) {
    rbx::set_error("%s", err.c_str());
    return RBX_ERR_INVALID;
  }
  return RBX_OK;
}

int rbx_lammps_get_info(const rbx_lammps_data* h, rbx_lammps_info* out) {
  if (!h || !out) return RBX_ERR_INVALID;
  const auto& d = h->d;
  out->n_atoms = d.n_atoms;
  out->n_bonds = d.n_bonds;
  out->n_angles = d.n_angles;
  out->n_dihedrals = d.n_dihedrals;
  out->n_impropers = d.n_impropers;
  out->n_atom_types = d.n_atom_types;
  out->n_bond_types = d.n_bond_types;
  out->n_angle_types = d.n_angle_types;
  out->n_dihedral_types = d.n_dihedral_types;
  out->n_improper_types = d.n_improper_types;
  out->atom_style = d.atom_style == "atomic" ? 0 : (d.atom_style == "charge" ? 1 : 2);
  out->has_masses = d.has_masses;
  out->has_pair_coeffs = d.has_pair_coeffs;
  out->has_velocities = d.has_velocities;
  out->has_images = d.has_images;
  for (int k = 0; k < 3; ++k) {
    out->box.lo[k] = d.lo[k];
    out->box.hi[k] = d.hi[k];
  }
  return RBX_OK;
}

int rbx_lammps_get_atoms(const rbx_lammps_data* h, int64_t* id, int* type, int* molecule,
                         double* charge, double* x, double* y, double* z, double* vx,
                         double* vy, double* vz, int* image) {
  if (!h) return RBX_ERR_INVALID;
  const auto& d = h->d;
  const size_t n = d.id.size();
  for (size_t i = 0; i < n; ++i) {
    if (id) id[i] = d.id[i];
    if (type) type[i] = d.type[i];
    if (molecule) molecule[i] = d.molecule[i];
    if (charge) charge[i] = d.q[i];
    if (x) x[i] = d.x[i];
    if (y) y[i] = d.y[i];
    if (z) z[i] = d.z[i];
    if (vx) vx[i] = d.vx[i];
    if (vy) vy[i] = d.vy[i];
    if (vz) vz[i] = d.vz[i];
  }
  if (image) std::copy(d.image.begin(), d.image.end(), image);
  return RBX_OK;
}

int rbx_lammps_get_types(const rbx_lammps_data* h, double* mass, double* eps, double* sigma) {
  if (!h) return RBX_ERR_INVALID;
  const auto& d = h->d;
  for (int t = 0; t < d.n_atom_types; ++t) {
    if (mass) mass[t] = d.mass.empty() ? 0.0 : d.mass[t];
    if (eps) eps[t] = d.pair_eps.empty() ? 0.0 : d.pair_eps[t];
    if (sigma) sigma[t] = d.pair_sigma.empty() ? 0.0 : d.pair_sigma[t];
  }
  return RBX_OK;
}

int rbx_lammps_get_topology(const rbx_lammps_data* h, int kind, int* type, int64_t* atoms) {
  if (!h || kind < 2 || kind > 5) {
    rbx::set_error("rbx_lammps_get_topology: kind is 2 bonds, 3 angles, 4 dihedrals, 5 impropers");
    return RBX_ERR_INVALID;
  }
  const auto& d = h->d;
  const std::vector<int>& t = kind == 2 ? d.bond_type
                              : kind == 3 ? d.angle_type
                              : kind == 4 ? d.dihedral_type
                                          : d.improper_type;
  const std::vector<int64_t>& a = kind == 2 ? d.bond_atoms
                                  : kind == 3 ? d.angle_atoms
                                  : kind == 4 ? d.dihedral_atoms
                                              : d.improper_atoms;
  if (type) std::copy(t.begin(), t.end(), type);
  if (atoms) std::copy(a.begin(), a.end(), atoms);
  return RBX_OK;
}

int rbx_lammps_write_charge(const char* path, const rbx_box* box, int n, int ntypes,
                            const double* mass, const double* eps, const double* sigma,
                            const int64_t* id, const int* type, const double* charge,
                            const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz) {
  if (!path || !box || n < 0 || ntypes <= 0 || !mass || !eps || !sigma || !id || !type ||
      !charge || !x || !y || !z) {
    rbx::set_error("rbx_lammps_write_charge: invalid arguments");
    return RBX_ERR_INVALID;
  }
  const std::string err = rbx_host::write_lammps_charge(path, box->lo, box->hi, n, ntypes, mass,
                                                        eps, sigma, id, type, charge, x, y, z,
                                                        vx, vy, vz);
  if (!err.empty()) {
    rbx::set_error("%s", err.c_str());
    return RBX_ERR_INVALID;
  }
  return RBX_OK;
}

}  // extern "C"
