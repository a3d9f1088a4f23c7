// lj_cut_coul_kspace.cpp -- see lj_cut_coul_kspace.h.
#include "lj_cut_coul_kspace.h"
#include "units.h"

#include <cmath>
#include <stdexcept>

namespace rbx_host {

// UnitFactor<...>::_qqr2e (src/common/unit_factor.cpp): LJ 1, REAL 332.06371,
// METAL 14.399645.
double QqrdFromUnit(const std::string& unit) { return UnitsOf(unit).qqr2e; }

// SetAlphaFromManual (kspace_calculator.cpp:105-118): JSON alpha is g_ewald^2.
void KSpaceCalculator::SetAlphaFromManual(double alpha) {
  if (alpha <= 0.0)
    throw std::runtime_error("Coulomb alpha override must be > 0. Current value: " +
                             std::to_string(alpha));
  _manual_alpha = true;
  _alpha = alpha;
  _g_ewald = std::sqrt(alpha);
  _accuracy = 0.0;
}

// DeriveAlphaFromAccuracy (kspace_calculator.cpp:120-157).
void KSpaceCalculator::DeriveAlphaFromAccuracy(double relative_accuracy, double qqr2e,
                                               double cut_off, const rbx_box& box,
                                               int num_atoms) {
  _manual_alpha = false;
  _accuracy = relative_accuracy * qqr2e;
  if (_accuracy <= 0.0)
    throw std::runtime_error("Coulomb accuracy must be > 0. Current value: " +
                             std::to_string(relative_accuracy));
  if (_q2 <= 0.0)
    throw std::runtime_error("Automatic alpha derivation requires a charged system (q2 > 0).");
  const double V = (box.hi[0] - box.lo[0]) * (box.hi[1] - box.lo[1]) * (box.hi[2] - box.lo[2]);
  _g_ewald = _accuracy * std::sqrt((double)num_atoms * cut_off * V) / (2.0 * _q2);
  if (_g_ewald >= 1.0)
    _g_ewald = (1.35 - 0.15 * std::log(_accuracy)) / cut_off;
  else
    _g_ewald = std::sqrt(-std::log(_g_ewald)) / cut_off;
  _alpha = _g_ewald * _g_ewald;
}

// ComputeRMS (kspace_calculator.cpp:909-918).
double KSpaceCalculator::ComputeRMS(int kmax, double L, int num_atoms) const {
  return 2.0 * _q2 * _g_ewald / L * std::sqrt(1.0 / (M_PI * kmax * num_atoms)) *
         std::exp(-M_PI * M_PI * kmax * kmax / (_g_ewald * _g_ewald * L * L));
}

// SetKspacePara (kspace_calculator.cpp:920-986): smallest kmax per dimension
// whose rms estimate is within the accuracy.
void KSpaceCalculator::SetKspacePara(const rbx_box& box, int num_atoms) {
  for (int d = 0; d < 3; ++d) {
    const double L = box.hi[d] - box.lo[d];
    int k = 1;
    while (ComputeRMS(k, L, num_atoms) > _accuracy) {
      ++k;
      if (k > 512) throw std::runtime_error("automatic kmax exceeds 512; set coulomb.kmax");
    }
    _kmax[d] = k;
  }
}

void KSpaceCalculator::Init(const ConfigData& cfg, double qqr2e, double cut_off,
                            const rbx_box& box, int num_atoms,
                            const std::vector<double>& charges) {
  if (!cfg.PathExists({"hyper_parameters", "coulomb"})) {
    _coulomb_type = "NULL";
    return;
  }
  double qsq = 0.0;
  for (double q : charges) qsq += q * q;
  _q2 = qqr2e * qsq;  // ComputeQsqSum (kspace_calculator.cpp:717-759)
  _coulomb_type = cfg.Get<std::string>("type", "hyper_parameters", "coulomb");
  auto derive_alpha = [&]() {
    if (cfg.PathExists({"hyper_parameters", "coulomb", "alpha"})) {
      SetAlphaFromManual(cfg.Get<double>("alpha", "hyper_parameters", "coulomb"));
    } else {
      if (!cfg.PathExists({"hyper_parameters", "coulomb", "accuracy"}))
        throw std::runtime_error(
            "Coulomb accuracy must be defined under hyper_parameters.coulomb.accuracy when "
            "automatic alpha derivation is enabled.");
      if (charges.empty())
        throw std::runtime_error("alpha derivation from accuracy needs the atom charges");
      DeriveAlphaFromAccuracy(cfg.Get<double>("accuracy", "hyper_parameters", "coulomb"), qqr2e,
                              cut_off, box, num_atoms);
    }
  };
  auto set_kmax = [&]() {
    if (cfg.PathExists({"hyper_parameters", "coulomb", "kmax"})) {
      auto k = cfg.GetArray<int>("kmax", "hyper_parameters", "coulomb");
      if (k.size() != 3)
        throw std::runtime_error(
            "When using Coulomb kmax override, 'kmax' must contain exactly 3 integers.");
      for (int d = 0; d < 3; ++d) _kmax[d] = k[d];
    } else {
      SetKspacePara(box, num_atoms);
    }
  };
  if (_coulomb_type == "RBE") {
    derive_alpha();
    _rbe_p = cfg.Get<int>("coulomb_sample_num", "hyper_parameters", "coulomb");
    if (!cfg.PathExists({"hyper_parameters", "coulomb", "energy_rbe_flag"}))
      throw std::runtime_error(
          "When using RBE for the coulomb type, the key 'energy_rbe_flag' must be defined.");
    _energy_rbe_flag = cfg.Get<std::string>("energy_rbe_flag", "hyper_parameters", "coulomb");
    if (_energy_rbe_flag == "yes") set_kmax();
  } else if (_coulomb_type == "EWALD") {
    derive_alpha();
    set_kmax();
  } else if (_coulomb_type == "RBSOG") {
    // KSpaceCalculator::Init RBSOG branch (kspace_calculator.cpp:253-330)
    if (!cfg.PathExists({"hyper_parameters", "coulomb", "rbsog_level"}))
      throw std::runtime_error("RBSOG requires hyper_parameters.coulomb.rbsog_level.");
    for (const char* legacy : {"accuracy", "rbsog_b", "rbsog_sigma", "rbsog_Mmax", "rbsog_Kcut"})
      if (cfg.PathExists({"hyper_parameters", "coulomb", legacy}))
        throw std::runtime_error(std::string("Legacy RBSOG config key '") + legacy +
                                 "' is not supported. Use hyper_parameters.coulomb.rbsog_level "
                                 "instead.");
    _rbsog_level = cfg.Get<int>("rbsog_level", "hyper_parameters", "coulomb");
    if (_rbsog_level < 0 || _rbsog_level > 4)
      throw std::runtime_error("RBSOG rbsog_level must be in [0, 4]. Current value: " +
                               std::to_string(_rbsog_level));
    _rbe_p = cfg.Get<int>("coulomb_sample_num", "hyper_parameters", "coulomb");
    if (cfg.PathExists({"hyper_parameters", "coulomb", "alpha"})) {
      SetAlphaFromManual(cfg.Get<double>("alpha", "hyper_parameters", "coulomb"));
    } else {
      static const double kTargetAccuracy[5] = {2.289e-3, 1.158e-4, 1.142e-5, 5.583e-8,
                                                3.389e-11};
      if (charges.empty())
        throw std::runtime_error("alpha derivation from accuracy needs the atom charges");
      DeriveAlphaFromAccuracy(kTargetAccuracy[_rbsog_level], qqr2e, cut_off, box, num_atoms);
    }
    _rbe_p = ((_rbe_p + 15) / 16) * 16;
  } else {
    throw std::runtime_error("Unsupported coulomb type: " + _coulomb_type);
  }
}

LJCutCoulKspace::LJCutCoulKspace(const std::string& json_text, const rbx_box& box, int num_atoms,
                                 int ntypes, const double* sigma, const double* eps,
                                 const double* mass, const double* charges, int precision,
                                 int device)
    : _cfg(json_text), _box(box), _n(num_atoms), _ntypes(ntypes), _precision(precision),
      _device(device) {
  _sigma.assign(sigma, sigma + ntypes);
  _eps.assign(eps, eps + ntypes);
  _mass.assign(mass, mass + ntypes);
  if (charges) _charges.assign(charges, charges + num_atoms);
}

LJCutCoulKspace::~LJCutCoulKspace() { rbx_engine_destroy(_engine); }

// LJCutCoulKspace::Init (src/force/src/lj_cut_coul_kspace.cpp:424-462).
void LJCutCoulKspace::Init() {
  const std::string ff =
      _cfg.PathExists({"hyper_parameters", "force_field", "type"})
          ? _cfg.Get<std::string>("type", "hyper_parameters", "force_field")
          : std::string("LJ/CUT/COUL/LONG");
  // CVFF (src/force/src/cvff.cpp) runs the same RBL / RBE force with
  // special-bond weights on the pair term; its bonded terms are not part of
  // this engine (rigid water under SHAKE does not feel them).
  if (ff != "LJ/CUT/COUL/LONG" && ff != "CVFF")
    throw std::runtime_error("force_field.type " + ff + " is not LJ/CUT/COUL/LONG or CVFF");
  const std::string unit = _cfg.PathExists({"init_configuration", "read_data", "unit"})
                               ? _cfg.Get<std::string>("unit", "init_configuration", "read_data")
                               : std::string("LJ");
  const double qqr2e = QqrdFromUnit(unit);
  _lj_units = unit == "LJ";
  const double cut_off = _cfg.Get<double>("cut_off", "hyper_parameters", "neighbor");
  _neighbor_type = _cfg.Get<std::string>("type", "hyper_parameters", "neighbor");
  rbx_params p{};
  p.cut_off = cut_off;
  p.skin = _cfg.PathExists({"hyper_parameters", "neighbor", "skin"})
               ? _cfg.Get<double>("skin", "hyper_parameters", "neighbor")
               : 0.0;
  if (_neighbor_type == "RBL") {
    if (!_cfg.PathExists({"hyper_parameters", "neighbor", "energy_rbl_flag"}))
      throw std::runtime_error(
          "When using RBL for the neighbor type, the key 'energy_rbl_flag' must be defined.");
    _energy_rbl_flag = _cfg.Get<std::string>("energy_rbl_flag", "hyper_parameters", "neighbor");
    p.neighbor_type = RBX_NEIGHBOR_RBL;
    p.r_core = _cfg.Get<double>("r_core", "hyper_parameters", "neighbor");
    p.neighbor_sample_num = _cfg.Get<int>("neighbor_sample_num", "hyper_parameters", "neighbor");
    if (p.neighbor_sample_num <= 0)
      throw std::runtime_error("Error neighbor_sample_num must be large than 0.");
  } else if (_neighbor_type == "Verlet-List" || _neighbor_type == "VERLET") {
    p.neighbor_type = RBX_NEIGHBOR_VERLET;
  } else if (_neighbor_type == "VERLET-SOG") {
    // LJCutCoulKspace::LJCoulSOGInit (lj_cut_coul_kspace.cpp:651-667) reads the level
    p.neighbor_type = RBX_NEIGHBOR_VERLET_SOG;
    p.rbsog_level = _cfg.Get<int>("rbsog_level", "hyper_parameters", "coulomb");
    if (p.rbsog_level < 0 || p.rbsog_level > 4)
      throw std::runtime_error("RBSOG rbsog_level must be in [0, 4]. Current value: " +
                               std::to_string(p.rbsog_level));
  } else {
    throw std::runtime_error("neighbor.type " + _neighbor_type +
                             " is not provided by this engine (RBL, Verlet-List, VERLET-SOG)");
  }
  _kspace.Init(_cfg, qqr2e, cut_off, _box, _n, _charges);
  if (_kspace.type() == "RBE") {
    p.coulomb_type = RBX_COULOMB_RBE;
    p.coulomb_sample_num = _kspace.sample_num();
  } else if (_kspace.type() == "RBSOG") {
    p.coulomb_type = RBX_COULOMB_RBSOG;
    p.coulomb_sample_num = _kspace.sample_num();
    p.rbsog_level = _kspace.rbsog_level();
  } else if (_kspace.type() == "EWALD") {
    throw std::runtime_error("coulomb.type EWALD runs through rbx_ewald_force, not the engine");
  } else {
    p.coulomb_type = RBX_COULOMB_NONE;
  }
  p.alpha = _kspace.alpha();
  for (int d = 0; d < 3; ++d) p.kmax[d] = _kspace.kmax()[d];
  p.random_seed = _cfg.PathExists({"hyper_parameters", "coulomb", "random_seed"})
                      ? (uint64_t)_cfg.Get<long long>("random_seed", "hyper_parameters", "coulomb")
                      : 0x5EEDULL;
  p.qqr2e = qqr2e;
  p.fmt2v = UnitsOf(unit).fmt2v;
  p.dt = _cfg.PathExists({"execution", "timestep"}) ? _cfg.Get<double>("timestep", "execution")
                                                     : 0.001;
  p.precision = _precision;
  p.ntypes = _ntypes;
  p.sigma = _sigma.data();
  p.eps = _eps.data();
  p.mass = _mass.data();
  _engine = rbx_engine_create(&p, &_box, _n, _device);
  if (!_engine) throw std::runtime_error(rbx_last_error());
}

void LJCutCoulKspace::Execute() {
  if (rbx_engine_compute_forces(_engine, epoch) != RBX_OK)
    throw std::runtime_error(rbx_last_error());
  EvaluatePotentialEnergy();
}

// EvaluatePotentialEnergy (lj_cut_coul_kspace.cpp:867-878): k-space energy
// (KSpaceCalculator::EvaluatePotentialEnergy, kspace_calculator.cpp:375-385;
// for RBE with energy_rbe_flag "yes" on a thermo step the exact Ewald energy
// plus the self energy, :630-645), pair energies where RBMD computes them
// (ComputeLJVerlet every step, ComputeLJCoulEnergy after the RBL force when
// energy_rbl_flag is "yes", :570-572, :821-865), each divided by the atom
// count in LJ units.
void LJCutCoulKspace::EvaluatePotentialEnergy() {
  const double per = _lj_units ? 1.0 / (double)_n : 1.0;
  rbx_stats s;
  if (rbx_engine_get_stats(_engine, &s) != RBX_OK) throw std::runtime_error(rbx_last_error());
  double ek = s.e_kspace;
  if (_kspace.type() == "RBE" && _kspace.energy_rbe_flag() == "yes" && thermo_step)
    if (rbx_engine_kspace_energy_exact(_engine, _kspace.kmax(), &ek) != RBX_OK)
      throw std::runtime_error(rbx_last_error());
  _e_kspace = ek * per;
  const bool verlet = _neighbor_type == "Verlet-List" || _neighbor_type == "VERLET";
  if (verlet || (_neighbor_type == "RBL" && _energy_rbl_flag == "yes")) {
    double ev = 0.0, ec = 0.0;
    if (rbx_engine_pair_energy(_engine, &ev, &ec, nullptr) != RBX_OK)
      throw std::runtime_error(rbx_last_error());
    _e_vdwl = ev * per;
    _e_coul = ec * per;
  }
  _e_pe = _e_vdwl + _e_coul + _e_kspace;
}

}  // namespace rbx_host

using rbx_host::LJCutCoulKspace;

namespace rbx {
void set_error(const char* fmt, ...);
}

// The plugin itself behind the C ABI (Force::Init / Execute /
// EvaluatePotentialEnergy, src/force/include/force.h:10-48).
struct rbx_force : LJCutCoulKspace {
  using LJCutCoulKspace::LJCutCoulKspace;
};

extern "C" rbx_force* rbx_force_create_json(const char* json_text, const rbx_box* box,
                                            int num_atoms, int ntypes, const double* sigma,
                                            const double* eps, const double* mass,
                                            const double* charges, int precision, int device) {
  if (!json_text || !box || num_atoms <= 0 || ntypes <= 0 || !sigma || !eps || !mass) {
    rbx::set_error("rbx_force_create_json: null argument or empty system");
    return nullptr;
  }
  try {
    auto* f = new rbx_force(json_text, *box, num_atoms, ntypes, sigma, eps, mass, charges,
                            precision, device);
    try {
      f->Init();
    } catch (...) {
      delete f;
      throw;
    }
    return f;
  } catch (const std::exception& ex) {
    rbx::set_error("%s", ex.what());
    return nullptr;
  }
}

extern "C" void rbx_force_destroy(rbx_force* f) { delete f; }

extern "C" rbx_engine* rbx_force_engine(rbx_force* f) { return f ? f->engine() : nullptr; }

extern "C" int rbx_force_execute(rbx_force* f, int epoch, int thermo_step) {
  if (!f) return RBX_ERR_INVALID;
  try {
    f->epoch = epoch;
    f->thermo_step = thermo_step != 0;
    f->Execute();
    return RBX_OK;
  } catch (const std::exception& ex) {
    rbx::set_error("%s", ex.what());
    return RBX_ERR_INVALID;
  }
}

extern "C" int rbx_force_energies(rbx_force* f, double out[4]) {
  if (!f || !out) return RBX_ERR_INVALID;
  out[0] = f->e_vdwl();
  out[1] = f->e_coul();
  out[2] = f->e_kspace();
  out[3] = f->e_pe();
  return RBX_OK;
}

extern "C" rbx_engine* rbx_engine_create_json(const char* json_text, const rbx_box* box,
                                              int num_atoms, int ntypes, const double* sigma,
                                              const double* eps, const double* mass,
                                              const double* charges, int precision, int device) {
  if (!json_text || !box || num_atoms <= 0 || ntypes <= 0 || !sigma || !eps || !mass) {
    rbx::set_error("rbx_engine_create_json: null argument or empty system");
    return nullptr;
  }
  try {
    LJCutCoulKspace plugin(json_text, *box, num_atoms, ntypes, sigma, eps, mass, charges,
                           precision, device);
    plugin.Init();
    return plugin.Release();
  } catch (const std::exception& ex) {
    rbx::set_error("%s", ex.what());
    return nullptr;
  }
}
