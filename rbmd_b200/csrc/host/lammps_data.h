// lammps_data.h -- LAMMPS data files: the reader behind rbx_lammps_read and
// the writer behind rbx_lammps_write_charge.
//
// Follows RBMD's LammpsFullReader (src/reader/src/format/lammps/
// lammps_full_reader.cpp): header counts and box (ParseHeader, :1228-1357),
// sections found by their leading keyword (DetectSection, :1715-1760), '#'
// comments, Masses / Pair Coeffs (:1359-1410), Atoms in the atomic, charge or
// full style with optional image flags (ParseAtom, :1496-1564), Velocities
// (:1566-1595), Bonds / Angles / Dihedrals / Impropers (:1597-1713).  Ids,
// types and molecules become 0-based as there; atoms stay in file order.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rbx_host {

struct LammpsData {
  std::string atom_style;  // "atomic", "charge" or "full"
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int64_t n_atoms = 0, n_bonds = 0, n_angles = 0, n_dihedrals = 0, n_impropers = 0;
  int n_atom_types = 0, n_bond_types = 0, n_angle_types = 0, n_dihedral_types = 0,
      n_improper_types = 0;
  std::vector<double> mass, pair_eps, pair_sigma;  // per atom type (0 where absent)
  bool has_masses = false, has_pair_coeffs = false, has_velocities = false, has_images = false;
  // atoms, file order
  std::vector<int64_t> id;
  std::vector<int> type, molecule, image;  // image: 3 per atom
  std::vector<double> q, x, y, z, vx, vy, vz;
  // topology: type and 0-based atom ids, 2 / 3 / 4 / 4 per entry
  std::vector<int> bond_type, angle_type, dihedral_type, improper_type;
  std::vector<int64_t> bond_atoms, angle_atoms, dihedral_atoms, improper_atoms;

  // style: "" = from the "Atoms # <style>" comment.  Returns "" or an error.
  std::string read(const std::string& path, const std::string& style);
  // Tile the box nx x ny x nz times (LammpsFullReader::ApplyReplicate,
  // :899-1052, bonds within a replica): replica r = (iz ny + iy) nx + ix gets
  // ids id + r (max id + 1) and molecules + r (max molecule + 1); positions are
  // unwrapped by their image flags, shifted and wrapped into the new box.
  std::string replicate(int nx, int ny, int nz);
  // velocity_type GAUSS (LammpsFullReader::ApplyGaussianVelocitiesIfRequested,
  // :710-864): per atom an std::mt19937_64 seeded by a SplitMix64-style mix of
  // (seed, file id) draws three std::normal_distribution<double> values scaled
  // by 1/sqrt(mass); the centre-of-mass velocity is removed and all velocities
  // scaled to temperature with 3N - 3 degrees of freedom.  Needs Masses.
  std::string gauss_velocities(double temperature, const std::string& unit, int seed);
};

// Writes an atom_style charge data file (Masses, Pair Coeffs, Atoms,
// Velocities) with ids id[i] + 1 and types type[i] + 1, so a reader that makes
// them 0-based sees id[i] and type[i].  Returns "" or an error.
std::string write_lammps_charge(const std::string& path, const double lo[3], const double hi[3],
                                int n, int ntypes, const double* mass, const double* eps,
                                const double* sigma, const int64_t* id, const int* type,
                                const double* q, const double* x, const double* y,
                                const double* z, const double* vx, const double* vy,
                                const double* vz);

}  // namespace rbx_host
