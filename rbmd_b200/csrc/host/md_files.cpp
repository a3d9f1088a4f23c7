// md_files.cpp -- an engine straight from RBMD's input files: the JSON config
// and the LAMMPS data file it names, read the way MDApplication::ReadMDData
// (src/application/md_application.cpp:175-195) and LammpsFullReader::Load
// (src/reader/src/format/lammps/lammps_full_reader.cpp:455-632) do, then the
// LJ/CUT/COUL/LONG plugin built from the same JSON.
#include <cmath>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "config_data.h"
#include "lammps_data.h"
#include "lj_cut_coul_kspace.h"
#include "rbx.h"
#include "special_bonds.h"
#include "units.h"

namespace rbx {
void set_error(const char* fmt, ...);
}

namespace rbx_host {

namespace {

std::string read_text(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("failed to open config file: " + path);
  std::ostringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

// ConfigData::ResolvePath (src/data_manager/include/config_data.h:174-197):
// absolute as given; else next to the config file if it exists there; else
// from the working directory.
std::string resolve(const std::string& path, const std::filesystem::path& config_dir) {
  namespace fs = std::filesystem;
  const fs::path p(path);
  if (p.is_absolute()) return p.lexically_normal().string();
  const fs::path beside = config_dir / p;
  if (fs::exists(beside)) return beside.lexically_normal().string();
  return (fs::current_path() / p).lexically_normal().string();
}

// LoadReplicateFactors (lammps_full_reader.cpp:650-680): "replicate" or
// "replicate_dims", three positive integers.
void replicate_factors(const ConfigData& cfg, int out[3]) {
  out[0] = out[1] = out[2] = 1;
  const bool a = cfg.PathExists({"init_configuration", "read_data", "replicate"});
  const bool b = cfg.PathExists({"init_configuration", "read_data", "replicate_dims"});
  if (!a && !b) return;
  const auto v = cfg.GetArray<int>(a ? "replicate" : "replicate_dims", "init_configuration",
                                   "read_data");
  if (v.size() != 3)
    throw std::runtime_error("init_configuration.read_data.replicate must contain exactly 3 integers");
  for (int d = 0; d < 3; ++d) {
    if (v[d] <= 0)
      throw std::runtime_error("init_configuration.read_data.replicate values must be positive");
    out[d] = v[d];
  }
}

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

rbx_engine* create_from_files(const std::string& json_path, int precision, int device) {
  const std::string text = read_text(json_path);
  const ConfigData cfg(text);
  const auto dir = std::filesystem::absolute(json_path).parent_path();
  const std::string file =
      resolve(cfg.Get<std::string>("file", "init_configuration", "read_data"), dir);
  const std::string style = cfg.Get<std::string>("atom_style", "init_configuration", "read_data");
  const std::string unit = cfg.PathExists({"init_configuration", "read_data", "unit"})
                               ? cfg.Get<std::string>("unit", "init_configuration", "read_data")
                               : std::string("LJ");
  LammpsData d;
  std::string err = d.read(file, style);
  if (!err.empty()) throw std::runtime_error(err);
  int rep[3];
  replicate_factors(cfg, rep);
  err = d.replicate(rep[0], rep[1], rep[2]);
  if (!err.empty()) throw std::runtime_error(err);

  // ApplyGaussianVelocitiesIfRequested (:710-864): only when the file has no
  // Velocities section.
  if (cfg.PathExists({"init_configuration", "read_data", "velocity_type"}) && !d.has_velocities) {
    const std::string vt =
        upper(cfg.Get<std::string>("velocity_type", "init_configuration", "read_data"));
    if (!vt.empty() && vt != "NONE") {
      if (vt != "GAUSS" && vt != "GAUSSIAN")
        throw std::runtime_error("Unsupported velocity_type: " + vt);
      const auto temp = cfg.PathExists({"execution", "temperature"})
                            ? cfg.GetArray<double>("temperature", "execution")
                            : std::vector<double>{};
      int seed = 12345;
      if (cfg.PathExists({"init_configuration", "read_data", "velocity_seed"}))
        seed = cfg.Get<int>("velocity_seed", "init_configuration", "read_data");
      else if (cfg.PathExists({"init_configuration", "read_data", "seed"}))
        seed = cfg.Get<int>("seed", "init_configuration", "read_data");
      err = d.gauss_velocities(temp.empty() ? 0.0 : temp[0], unit, seed);
      if (!err.empty()) throw std::runtime_error(err);
    }
  }

  const int n = (int)d.id.size();
  const int nt = d.n_atom_types;
  if (n <= 0) throw std::runtime_error(file + ": no atoms");
  if (!d.has_masses) throw std::runtime_error(file + ": no Masses section");
  if (!d.has_pair_coeffs)
    throw std::runtime_error(file + ": no Pair Coeffs section (LJ/CUT/COUL/LONG takes eps and "
                                    "sigma per atom type from it)");
  std::vector<int> gid(n), type(d.type), image(3 * (size_t)n, 0);
  for (int i = 0; i < n; ++i) {
    if (d.id[i] < 0 || d.id[i] > INT32_MAX) throw std::runtime_error("atom id beyond 2^31");
    gid[i] = (int)d.id[i];
  }
  std::vector<double> q = d.q;
  if (q.size() != (size_t)n) q.assign(n, 0.0);
  // positions into [lo, hi), the wraps counted in the image flags
  rbx_box box{};
  std::vector<double> pos[3] = {d.x, d.y, d.z};
  for (int k = 0; k < 3; ++k) {
    box.lo[k] = d.lo[k];
    box.hi[k] = d.hi[k];
    const double L = d.hi[k] - d.lo[k];
    for (int i = 0; i < n; ++i) {
      double& x = pos[k][i];
      int w = 0;
      if (x < d.lo[k] || x >= d.hi[k]) {
        w = (int)std::floor((x - d.lo[k]) / L);
        x -= w * L;
        if (x >= d.hi[k]) x -= L, ++w;
        if (x < d.lo[k]) x = d.lo[k];
      }
      image[3 * (size_t)i + k] = (d.has_images ? d.image[3 * (size_t)i + k] : 0) + w;
    }
  }
  std::vector<double> vel[3] = {d.vx, d.vy, d.vz};
  for (auto& v : vel)
    if (v.size() != (size_t)n) v.assign(n, 0.0);

  // execution.ensemble: NVE, or NVT with the Nose-Hoover chain
  // (NVTensemble, nvt_ensemble.cpp; NoseHooverController::Init reads
  // execution.temperature = [start, stop, damp] and num_steps for a ramp).
  const std::string ensemble = cfg.PathExists({"execution", "ensemble"})
                                   ? upper(cfg.Get<std::string>("ensemble", "execution"))
                                   : std::string("NVE");
  std::vector<double> nh;
  long long num_steps = 0;
  if (ensemble == "NVT") {
    const std::string tc = cfg.PathExists({"execution", "temp_ctrl_type"})
                               ? upper(cfg.Get<std::string>("temp_ctrl_type", "execution"))
                               : std::string("NOSE_HOOVER");
    if (tc != "NOSE_HOOVER")
      throw std::runtime_error("execution.temp_ctrl_type " + tc +
                               " is not provided by this engine (NOSE_HOOVER)");
    nh = cfg.GetArray<double>("temperature", "execution");
    if (nh.size() < 3)
      throw std::runtime_error("execution.temperature must be [t_start, t_stop, t_damp]");
    if (cfg.PathExists({"execution", "num_steps"}))
      num_steps = cfg.Get<long long>("num_steps", "execution");
  } else if (ensemble != "NVE") {
    throw std::runtime_error("execution.ensemble " + ensemble +
                             " is not provided by this engine (NVE, NVT)");
  }

  // hyper_parameters.extend: fix_shake (every angle a rigid cluster, the
  // reference's serial ShakeA) and special_bonds (CVFF; read_special_bond_weights,
  // cvff.cpp:309-330, default 1 1 1)
  const bool shake = cfg.PathExists({"hyper_parameters", "extend", "fix_shake"}) &&
                     cfg.Get<bool>("fix_shake", "hyper_parameters", "extend");
  const std::string ff = cfg.PathExists({"hyper_parameters", "force_field", "type"})
                             ? cfg.Get<std::string>("type", "hyper_parameters", "force_field")
                             : std::string("LJ/CUT/COUL/LONG");
  double w[3] = {1.0, 1.0, 1.0};
  if (ff == "CVFF" && cfg.PathExists({"hyper_parameters", "extend", "special_bonds"})) {
    const auto v = cfg.GetArray<double>("special_bonds", "hyper_parameters", "extend");
    for (size_t k = 0; k < v.size() && k < 3; ++k) w[k] = v[k];
  }
  // topology by host index (file order) instead of atom id
  std::unordered_map<int64_t, int> host_of_id;
  for (int i = 0; i < n; ++i) host_of_id[d.id[i]] = i;
  auto to_host = [&](const std::vector<int64_t>& ids) {
    std::vector<int64_t> h(ids.size());
    for (size_t k = 0; k < ids.size(); ++k) {
      const auto it = host_of_id.find(ids[k]);
      if (it == host_of_id.end())
        throw std::runtime_error("topology names atom id " + std::to_string(ids[k] + 1) +
                                 " that is not in Atoms");
      h[k] = it->second;
    }
    return h;
  };
  std::vector<int> clusters;
  if (shake) {
    for (int64_t h : to_host(d.angle_atoms)) clusters.push_back((int)h);
    if (clusters.empty()) throw std::runtime_error("fix_shake needs Angles (rigid clusters)");
  }
  std::vector<int> nspecial, special;
  int maxspecial = 0;
  if (ff == "CVFF" && (w[0] != 1.0 || w[1] != 1.0 || w[2] != 1.0)) {
    const auto hb = to_host(d.bond_atoms), ha = to_host(d.angle_atoms),
               hd = to_host(d.dihedral_atoms);
    const auto rows = build_special(n, (int)d.bond_type.size(), hb.data(),
                                    (int)d.angle_type.size(), ha.data(),
                                    (int)d.dihedral_type.size(), hd.data());
    maxspecial = rows.maxspecial;
    nspecial.resize(3 * (size_t)n);
    special.resize((size_t)n * std::max(maxspecial, 1));
    fill_special(rows, nspecial.data(), special.data());
  }

  LJCutCoulKspace plugin(text, box, n, nt, d.pair_sigma.data(), d.pair_eps.data(), d.mass.data(),
                         q.data(), precision, device);
  plugin.Init();
  rbx_engine* e = plugin.Release();
  const UnitFactors u = UnitsOf(unit);
  if (rbx_engine_set_state(e, gid.data(), type.data(), q.data(), pos[0].data(), pos[1].data(),
                           pos[2].data(), vel[0].data(), vel[1].data(), vel[2].data()) != RBX_OK ||
      rbx_engine_set_images(e, image.data()) != RBX_OK ||
      (shake && rbx_engine_set_shake(e, (int)clusters.size() / 3, clusters.data(), 1.0,
                                     109.47) != RBX_OK) ||
      (maxspecial > 0 && rbx_engine_set_special(e, maxspecial, nspecial.data(), special.data(),
                                                w[0], w[1], w[2]) != RBX_OK) ||
      (!nh.empty() &&
       rbx_engine_set_nose_hoover(e, nh[0], nh[1], nh[2], num_steps, u.kb, u.mvv2e,
                                  shake ? 3.0 * n - 3.0 - n : 0.0) != RBX_OK)) {
    const std::string msg = rbx_last_error();
    rbx_engine_destroy(e);
    throw std::runtime_error(msg);
  }
  return e;
}

}  // namespace
}  // namespace rbx_host

extern "C" rbx_engine* rbx_engine_create_from_files(const char* json_path, int precision,
                                                    int device) {
  if (!json_path) {
    rbx::set_error("rbx_engine_create_from_files: null path");
    return nullptr;
  }
  try {
    return rbx_host::create_from_files(json_path, precision, device);
  } catch (const std::exception& ex) {
    rbx::set_error("%s", ex.what());
    return nullptr;
  }
}
