// lj_cut_coul_kspace.h -- the "LJ/CUT/COUL/LONG" force plugin on top of the
// B200 engine.  Mirrors LJCutCoulKspace (src/force/include/lj_cut_coul_kspace.h)
// and the parameter logic of KSpaceCalculator::Init
// (src/force/src/kspace_calculator.cpp:159-355): same JSON keys, same
// required-key errors, alpha either manual (JSON alpha = g_ewald^2) or derived
// from coulomb.accuracy, kmax manual or from the rms estimate.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "config_data.h"
#include "force.h"
#include "rbx.h"

namespace rbx_host {

// KSpaceCalculator parameter derivation (no device work).
class KSpaceCalculator {
 public:
  // charges may be empty when alpha is given explicitly.
  void Init(const ConfigData& cfg, double qqr2e, double cut_off, const rbx_box& box,
            int num_atoms, const std::vector<double>& charges);
  std::string type() const { return _coulomb_type; }
  double alpha() const { return _alpha; }
  double g_ewald() const { return _g_ewald; }
  int sample_num() const { return _rbe_p; }
  const int* kmax() const { return _kmax; }
  bool manual_alpha() const { return _manual_alpha; }
  std::string energy_rbe_flag() const { return _energy_rbe_flag; }
  int rbsog_level() const { return _rbsog_level; }

 private:
  void SetAlphaFromManual(double alpha);
  void DeriveAlphaFromAccuracy(double relative_accuracy, double qqr2e, double cut_off,
                               const rbx_box& box, int num_atoms);
  void SetKspacePara(const rbx_box& box, int num_atoms);
  double ComputeRMS(int kmax, double box_length, int num_atoms) const;

  std::string _coulomb_type = "NULL";
  std::string _energy_rbe_flag = "no";
  double _alpha = 0.0, _g_ewald = 0.0, _accuracy = 0.0, _q2 = 0.0;
  bool _manual_alpha = false;
  int _rbe_p = 0;
  int _rbsog_level = 0;
  int _kmax[3] = {0, 0, 0};
};

double QqrdFromUnit(const std::string& unit);

class LJCutCoulKspace : public Force {
 public:
  LJCutCoulKspace(const std::string& json_text, const rbx_box& box, int num_atoms, int ntypes,
                  const double* sigma, const double* eps, const double* mass,
                  const double* charges, int precision, int device);
  ~LJCutCoulKspace() override;

  void Init() override;
  void Execute() override;  // one force evaluation at the current epoch
  void EvaluatePotentialEnergy() override;

  rbx_engine* engine() const { return _engine; }
  rbx_engine* Release() {
    rbx_engine* e = _engine;
    _engine = nullptr;
    return e;
  }
  int epoch = 0;
  // ThermoStats::ShouldOutput() of the host's pipeline for the next Execute:
  // with energy_rbe_flag "yes" the RBE k-space energy of a thermo step is the
  // exact Ewald energy over kmax plus the self energy (kspace_calculator.cpp:630-645)
  bool thermo_step = true;
  // energies of the last evaluation, per atom in LJ units (totals otherwise);
  // the pair energies only for a Verlet list or RBL with energy_rbl_flag "yes"
  double e_kspace() const { return _e_kspace; }
  double e_vdwl() const { return _e_vdwl; }
  double e_coul() const { return _e_coul; }
  double e_pe() const { return _e_pe; }

 private:
  ConfigData _cfg;
  rbx_box _box;
  int _n, _ntypes, _precision, _device;
  std::vector<double> _sigma, _eps, _mass, _charges;
  std::string _neighbor_type, _energy_rbl_flag = "yes";
  KSpaceCalculator _kspace;
  rbx_engine* _engine = nullptr;
  bool _lj_units = true;
  double _e_kspace = 0.0, _e_vdwl = 0.0, _e_coul = 0.0, _e_pe = 0.0;
};

}  // namespace rbx_host
