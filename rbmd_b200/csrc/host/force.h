// force.h -- the force-plugin interface of RBMD (src/force/include/force.h:10-48):
// Init(), Execute() once per MD step, EvaluatePotentialEnergy().
#pragma once

namespace rbx_host {

class Force {
 public:
  virtual ~Force() = default;
  virtual void Init() {}
  virtual void Execute() = 0;
  virtual void EvaluatePotentialEnergy() {}
};

}  // namespace rbx_host
