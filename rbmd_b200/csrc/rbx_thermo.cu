// rbx_thermo.cu -- Nose-Hoover chain thermostat (NVT) on the device.
//
// Follows NoseHooverController (src/simulate_pipeline/src/controller/
// pressure_controller/nose_hoover_controller.cpp): chain of 3, one
// sub-cycle, eta masses refreshed every call (SetUp :415-471,
// ComputeTempTarget :473-497, NHCTempIntegrate :732-840), temperature from
// ComputeTemperature (update_temperature_op.hip.cu:7-29) as
// 0.5 * sum(mvv2e m v^2) / (tdof kB / 2).  The reference runs the chain on
// the host after a device reduction and a copy back; here the reduction is
// a fixed-order two-level sum and the chain one thread of a kernel, so the
// whole thermostat stays inside the CUDA-graph step with no host round trip.
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"

namespace rbx {

namespace {
constexpr int KE_BLOCK = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0;
  if (w == 0) {
    s = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  __syncthreads();
  return s;  // valid in thread 0
}

// Per-block partial sums of mvv2e m v^2 over a fixed grid (grid-stride), so
// the sum order does not depend on timing.
__global__ void __launch_bounds__(KE_BLOCK) k_ke_partials(int n, const int* __restrict__ type,
                                                          const double* __restrict__ mass,
                                                          const double* __restrict__ vx,
                                                          const double* __restrict__ vy,
                                                          const double* __restrict__ vz,
                                                          double mvv2e, double* part) {
  __shared__ double sh[32];
  double s = 0;
  for (int i = blockIdx.x * KE_BLOCK + threadIdx.x; i < n; i += gridDim.x * KE_BLOCK)
    s += mvv2e * mass[type[i]] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__device__ void temp_target(const NHParams& p, double* st, long long step) {
  double t = p.t_start;
  if (p.t_stop != p.t_start) {
    double delta = (double)step;
    if (delta != 0.0) delta = delta / (double)p.num_steps;
    t = p.t_start + delta * (p.t_stop - p.t_start);
  }
  st[NH_T_TARGET] = t;
  st[NH_KE_TARGET] = p.tdof * p.kb * t;
}

// NHCTempIntegrate with nc_tchain = 1, drag 0: the chain's half-step update
// and the velocity scale factor (applied by k_scale_v); the temperature is
// rescaled by factor^2 as the reference does instead of being measured again.
__device__ void chain_integrate(const NHParams& p, double* st) {
  double* eta = st + NH_ETA;
  double* eta_dot = st + NH_ETA_DOT;  // NH_CHAIN + 1 entries, the last stays 0
  double* eta_dotdot = st + NH_ETA_DOTDOT;
  double* eta_mass = st + NH_ETA_MASS;
  const double t_target = st[NH_T_TARGET], ke_target = st[NH_KE_TARGET];
  const double tf2 = p.t_freq * p.t_freq;
  const double dt8 = 0.125 * p.dt, dt4 = 0.25 * p.dt, dthalf = 0.5 * p.dt;
  double ke = p.tdof * p.kb * st[NH_TEMP];
  eta_mass[0] = p.tdof * p.kb * t_target / tf2;
  for (int c = 1; c < NH_CHAIN; ++c) eta_mass[c] = p.kb * t_target / tf2;
  eta_dotdot[0] = eta_mass[0] > 0.0 ? (ke - ke_target) / eta_mass[0] : 0.0;
  for (int c = NH_CHAIN - 1; c > 0; --c) {
    const double e = exp(-dt8 * eta_dot[c + 1]);
    eta_dot[c] *= e;
    eta_dot[c] += eta_dotdot[c] * dt4;
    eta_dot[c] *= e;
  }
  const double e1 = exp(-dt8 * eta_dot[1]);
  eta_dot[0] *= e1;
  eta_dot[0] += eta_dotdot[0] * dt4;
  eta_dot[0] *= e1;
  const double f = exp(-dthalf * eta_dot[0]);
  st[NH_FACTOR] = f;
  st[NH_TEMP] = st[NH_TEMP] * f * f;
  ke = p.tdof * p.kb * st[NH_TEMP];
  eta_dotdot[0] = eta_mass[0] > 0.0 ? (ke - ke_target) / eta_mass[0] : 0.0;
  for (int c = 0; c < NH_CHAIN; ++c) eta[c] += dthalf * eta_dot[c];
  eta_dot[0] *= e1;
  eta_dot[0] += eta_dotdot[0] * dt4;
  eta_dot[0] *= e1;
  for (int c = 1; c < NH_CHAIN; ++c) {
    const double e = exp(-dt8 * eta_dot[c + 1]);
    eta_dot[c] *= e;
    eta_dotdot[c] = (eta_mass[c - 1] * eta_dot[c - 1] * eta_dot[c - 1] - p.kb * t_target) /
                    eta_mass[c];
    eta_dot[c] += eta_dotdot[c] * dt4;
    eta_dot[c] *= e;
  }
}

// mode 0: SetUp (temperature from the partials, target at step 0, masses,
// chain forces); 1: InitialIntegrate's target + chain half step at step
// (*step_dev or 0) + step_add; 2: FinalIntegratePostShake's temperature +
// chain half step.  One block; thread 0 runs the chain.
__global__ void __launch_bounds__(KE_BLOCK) k_nh_chain(NHParams p, double* st,
                                                       const double* __restrict__ part,
                                                       int nparts, const int* step_dev,
                                                       long long step_add, int mode) {
  __shared__ double sh[32];
  if (mode != 1) {
    double s = 0;
    for (int b = threadIdx.x; b < nparts; b += KE_BLOCK) s += part[b];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) st[NH_TEMP] = 0.5 * s / (p.tdof * p.kb / 2.0);
  }
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    temp_target(p, st, 0);
    const double tf2 = p.t_freq * p.t_freq;
    st[NH_ETA_MASS] = p.tdof * p.kb * st[NH_T_TARGET] / tf2;
    for (int c = 1; c < NH_CHAIN; ++c) st[NH_ETA_MASS + c] = p.kb * st[NH_T_TARGET] / tf2;
    for (int c = 1; c < NH_CHAIN; ++c)
      st[NH_ETA_DOTDOT + c] = (st[NH_ETA_MASS + c - 1] * st[NH_ETA_DOT + c - 1] *
                                   st[NH_ETA_DOT + c - 1] -
                               p.kb * st[NH_T_TARGET]) /
                              st[NH_ETA_MASS + c];
    st[NH_FACTOR] = 1.0;
    return;
  }
  if (mode == 1) temp_target(p, st, (step_dev ? (long long)*step_dev : 0) + step_add);
  chain_integrate(p, st);
}

__global__ void k_scale_v(int n, const double* __restrict__ st, double* vx, double* vy,
                          double* vz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double f = st[NH_FACTOR];
  vx[i] *= f;
  vy[i] *= f;
  vz[i] *= f;
}
}  // namespace

int launch_ke_partials(int n, const int* type, const double* mass, const double* vx,
                       const double* vy, const double* vz, double mvv2e, double* part,
                       cudaStream_t st) {
  k_ke_partials<<<KE_PARTS, KE_BLOCK, 0, st>>>(n, type, mass, vx, vy, vz, mvv2e, part);
  count_launch();
  return check_launch("ke_partials");
}

int launch_nh_chain(const NHParams& p, double* state, const double* part, const int* step_dev,
                    long long step_add, int mode, cudaStream_t st) {
  k_nh_chain<<<1, KE_BLOCK, 0, st>>>(p, state, part, KE_PARTS, step_dev, step_add, mode);
  count_launch();
  return check_launch("nh_chain");
}

int launch_scale_v(int n, const double* state, double* vx, double* vy, double* vz,
                   cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_scale_v<<<(n + 255) / 256, 256, 0, st>>>(n, state, vx, vy, vz);
  count_launch();
  return check_launch("scale_v");
}

}  // namespace rbx
