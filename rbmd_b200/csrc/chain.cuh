// chain.cuh -- scalar thermostat and barostat updates shared by the step kernels: temperature,
// Nose-Hoover chain halves, the pressure scalar, and the pieces of the isotropic MTK barostat.
// Each runs on one thread per system (the last block of a reduction, or a per-system kernel).
#pragma once

#include "kernels.h"

namespace rbmd {

// ------------------------------------------------------------------ scalar thermostat pieces
__device__ inline void compute_tempe(const SysDev& s, SysState* st, double sum) {
  // ExecutionNVT::ComputeTempe, ExecutionNVT.cpp:736-773
  st->tempT_sum = sum;
  const double n = s.n, kB = s.kB;
  if (s.inbuild) st->temperature = 0.5 * sum / (3 * n / 2.0);
  else if (s.fix_shake == RBMD_SHAKE_NULL) st->temperature = 0.5 * sum / ((3 * n - 3) * kB / 2.0);
  else if (s.fix_shake == RBMD_SHAKE_TRUE) st->temperature = 0.5 * sum / ((3 * n - n - 3) * kB / 2.0);
  else st->temperature = 0.5 * sum / ((3 * n) * kB / 2.0);
}

__device__ inline void compute_temp_target(const SysDev& s, SysState* st) {
  // ExecutionNVT::ComputeTempTarget, ExecutionNVT.cpp:1124-1147
  if (s.t_stop == s.t_start) {
    st->t_target = s.t_start;
  } else {
    double delta = (double)st->step;
    if (delta != 0.0) delta = delta / (double)s.num_steps;
    st->t_target = s.t_start + delta * (s.t_stop - s.t_start);
  }
  st->ke_target = st->tdof * s.boltz * st->t_target;
}

// One half of ExecutionNVT::NHCTempIntegrate (ExecutionNVT.cpp:1172-1256); returns the velocity
// factor and rescales the stored temperature as the reference does.
__device__ inline double nhc_half(const SysDev& s, SysState* st) {
  const int mtchain = 3;
  const double dt = s.dt, dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  const double boltz = s.boltz, tf = st->t_freq;
  double kecurrent = st->tdof * boltz * st->temperature;
  st->eta_mass[0] = st->tdof * boltz * st->t_target / (tf * tf);
  for (int ich = 1; ich < mtchain; ich++) st->eta_mass[ich] = boltz * st->t_target / (tf * tf);
  if (st->eta_mass[0] > 0.0) st->eta_dotdot[0] = (kecurrent - st->ke_target) / st->eta_mass[0];
  else st->eta_dotdot[0] = 0.0;
  const double ncfac = 1.0;
  double expfac;
  for (int ich = mtchain - 1; ich > 0; ich--) {
    expfac = exp(-ncfac * dt8 * st->eta_dot[ich + 1]);
    st->eta_dot[ich] *= expfac;
    st->eta_dot[ich] += st->eta_dotdot[ich] * ncfac * dt4;
    st->eta_dot[ich] *= st->tdrag;
    st->eta_dot[ich] *= expfac;
  }
  expfac = exp(-ncfac * dt8 * st->eta_dot[1]);
  st->eta_dot[0] *= expfac;
  st->eta_dot[0] += st->eta_dotdot[0] * ncfac * dt4;
  st->eta_dot[0] *= st->tdrag;
  st->eta_dot[0] *= expfac;
  const double factor = exp(-ncfac * dthalf * st->eta_dot[0]);
  st->temperature = st->temperature * factor * factor;
  kecurrent = st->tdof * boltz * st->temperature;
  if (st->eta_mass[0] > 0.0) st->eta_dotdot[0] = (kecurrent - st->ke_target) / st->eta_mass[0];
  else st->eta_dotdot[0] = 0.0;
  for (int ich = 0; ich < mtchain; ich++) st->eta[ich] += ncfac * dthalf * st->eta_dot[ich];
  st->eta_dot[0] *= expfac;
  st->eta_dot[0] += st->eta_dotdot[0] * ncfac * dt4;
  st->eta_dot[0] *= expfac;
  for (int ich = 1; ich < mtchain; ich++) {
    expfac = exp(-ncfac * dt8 * st->eta_dot[ich + 1]);
    st->eta_dot[ich] *= expfac;
    st->eta_dotdot[ich] = (st->eta_mass[ich - 1] * st->eta_dot[ich - 1] * st->eta_dot[ich - 1] -
                           boltz * st->t_target) / st->eta_mass[ich];
    st->eta_dot[ich] += st->eta_dotdot[ich] * ncfac * dt4;
    st->eta_dot[ich] *= expfac;
  }
  return factor;
}

// ------------------------------------------------------------------ pressure
// Compute_Pressure_Scalar (ExecutionNPT.cpp:1429-1447) with ExecutionMD::ComputeVirial's sum
// (ExecutionMD.cpp:1263-1370): virial of the last force evaluation plus the SHAKE virial, none
// for EAM; the temperature is the stored PARA_TEMPT.  Writes the virial used to vir.
__device__ inline double pressure_scalar(const SysDev& s, const SysState* st, double vir[6]) {
  for (int k = 0; k < 6; ++k) {
    vir[k] = st->virial[k];
    if (s.fix_shake == RBMD_SHAKE_TRUE) vir[k] = __dadd_rn(vir[k], st->shake_virial[k]);
    if (s.ff == RBMD_FF_EAM) vir[k] = 0.0;
  }
  const double kin = __dmul_rn(__dmul_rn(st->tdof, s.boltz), st->temperature);
  const double sum = __dadd_rn(__dadd_rn(__dadd_rn(kin, vir[0]), vir[1]), vir[2]);
  return __dmul_rn(__dmul_rn(sum / 3.0, 1.0 / s.volume), s.nktv2p);
}

// ------------------------------------------------------------------ MTK barostat (iso, pdim 3)
// ExecutionNPT with temp_ctrl_type and press_ctrl_type NOSE_HOOVER (ExecutionNPT.cpp:1545-2066).

// SetUp, barostat part (ExecutionNPT.cpp:1573-1602), at t_target of step 0.
__device__ inline void mtk_setup(const SysDev& s, SysState* st) {
  const double p_freq = 1 / s.p_damp, p_freq_max = p_freq;
  const double kt = s.boltz * st->t_target;
  const double nkt = (s.n + 1) * kt;
  for (int i = 0; i < 3; ++i) st->omega_mass[i] = nkt / (p_freq * p_freq);
  for (int ich = 0; ich < 3; ich++) st->etap_mass[ich] = s.boltz * st->t_target / (p_freq_max * p_freq_max);
  for (int ich = 1; ich < 3; ich++)
    st->etap_dotdot[ich] = (st->etap_mass[ich - 1] * st->etap_dot[ich - 1] * st->etap_dot[ich - 1] -
                            s.boltz * st->t_target) / st->etap_mass[ich];
}

// NHCPressIntegrate (ExecutionNPT.cpp:1831-1915): chain of length 3 on the barostat velocity.
__device__ inline void nhc_press_half(const SysDev& s, SysState* st) {
  const int mpchain = 3;
  const double dt = s.dt, dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  const double kt = s.boltz * st->t_target;
  double kecurrent = 0.0;
  for (int i = 0; i < 3; ++i) kecurrent += st->omega_mass[i] * st->omega_dot[i] * st->omega_dot[i];
  const double lkt_press = kt;
  st->etap_dotdot[0] = (kecurrent - lkt_press) / st->etap_mass[0];
  const double ncfac = 1.0;
  double expfac;
  for (int ich = mpchain - 1; ich > 0; ich--) {
    expfac = exp(-ncfac * dt8 * st->etap_dot[ich + 1]);
    st->etap_dot[ich] *= expfac;
    st->etap_dot[ich] += st->etap_dotdot[ich] * ncfac * dt4;
    st->etap_dot[ich] *= expfac;
  }
  expfac = exp(-ncfac * dt8 * st->etap_dot[1]);
  st->etap_dot[0] *= expfac;
  st->etap_dot[0] += st->etap_dotdot[0] * ncfac * dt4;
  st->etap_dot[0] *= expfac;
  for (int ich = 0; ich < mpchain; ich++) st->etap[ich] += ncfac * dthalf * st->etap_dot[ich];
  const double factor_etap = exp(-ncfac * dthalf * st->etap_dot[0]);
  for (int i = 0; i < 3; ++i) st->omega_dot[i] *= factor_etap;
  kecurrent = 0.0;
  for (int i = 0; i < 3; ++i) kecurrent += st->omega_mass[i] * st->omega_dot[i] * st->omega_dot[i];
  st->etap_dotdot[0] = (kecurrent - lkt_press) / st->etap_mass[0];
  st->etap_dot[0] *= expfac;
  st->etap_dot[0] += st->etap_dotdot[0] * ncfac * dt4;
  st->etap_dot[0] *= expfac;
  for (int ich = 1; ich < mpchain; ich++) {
    expfac = exp(-ncfac * dt8 * st->etap_dot[ich + 1]);
    st->etap_dot[ich] *= expfac;
    st->etap_dotdot[ich] = (st->etap_mass[ich - 1] * st->etap_dot[ich - 1] * st->etap_dot[ich - 1] -
                            s.boltz * st->t_target) / st->etap_mass[ich];
    st->etap_dot[ich] += st->etap_dotdot[ich] * ncfac * dt4;
    st->etap_dot[ich] *= expfac;
  }
}

// ComputePressTarget (ExecutionNPT.cpp:1631-1669); the division by pdim sits inside the loop
// there, so p_hydro = ((P/3 + P)/3 + P)/3 for an isotropic target P.
__device__ inline void press_target(const SysDev& s, SysState* st) {
  st->p_hydro = 0.0;
  for (int i = 0; i < 3; ++i) {
    double pt;
    if (s.p_stop == s.p_start) {
      pt = s.p_start;
    } else {
      double delta = (double)st->step;
      if (delta != 0.0) delta = delta / (double)s.num_steps;
      pt = s.p_start + delta * (s.p_stop - s.p_start);
    }
    st->p_hydro += pt;
    st->p_hydro /= 3;
  }
}

// NHOmegaDot (ExecutionNPT.cpp:1942-1986), then the NH_V_Press factors (:1988-1997) that the next
// half kick applies twice.
__device__ inline void omega_dot_half(const SysDev& s, SysState* st) {
  const double dthalf = 0.5 * s.dt, dt4 = 0.25 * s.dt;
  const double volume = s.L[0] * s.L[1] * s.L[2];
  st->mtk_term1 = st->tdof * s.boltz * st->temperature;
  st->mtk_term1 /= 3 * s.n;
  for (int i = 0; i < 3; ++i) {
    const double f_omega = (st->p_current - st->p_hydro) * volume / (st->omega_mass[i] * s.nktv2p) +
                           st->mtk_term1 / st->omega_mass[i];
    st->omega_dot[i] += f_omega * dthalf;
  }
  st->mtk_term2 = 0.0;
  for (int i = 0; i < 3; ++i) st->mtk_term2 += st->omega_dot[i];
  st->mtk_term2 /= 3 * s.n;
  for (int k = 0; k < 3; ++k) st->f_press[k] = exp(-dt4 * (st->omega_dot[k] + st->mtk_term2));
}

}  // namespace rbmd
