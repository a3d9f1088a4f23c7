// units.h -- the unit-style constants of RBMD's UnitFactor (src/common/
// unit_factor.cpp:28-50), written with the same expressions so the doubles
// are the same: Boltzmann constant kb, mvv2e (m v^2 -> energy), fmt2v
// (force / mass * time -> velocity) and qqr2e (Coulomb constant).
#pragma once
#include <cmath>
#include <stdexcept>
#include <string>

namespace rbx_host {

struct UnitFactors {
  double kb, mvv2e, fmt2v, qqr2e;
};

inline UnitFactors UnitsOf(const std::string& unit) {
  if (unit == "LJ") return {1.0, 1.0, 1.0, 1.0};
  if (unit == "REAL")
    return {1.9872067 * std::pow(10.0, -3.0), 1.0 / (4.186 * std::pow(10.0, -4.0)),
            4.186 * std::pow(10.0, -4.0), 332.06371};
  if (unit == "METAL") return {8.617343e-5, 1.0364269e-4, 1.0 / 1.0364269e-4, 14.399645};
  throw std::runtime_error("unsupported init_configuration.read_data.unit: " + unit);
}

}  // namespace rbx_host
