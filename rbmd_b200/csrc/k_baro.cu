// k_baro.cu -- NPT barostats: the new box with every table that follows from it, and the remap
// of the atoms.
//
//   ExecutionNPT::fix_press_berendsen / Compute_Pressure_Scalar / remap   ExecutionNPT.cpp:1334-1368,
//                                                                        1429-1447, 1506-1538
//   ExecutionNPT::InitialIntegrate / NHCPressIntegrate / NHOmegaDot /    ExecutionNPT.cpp:1631-2066
//                 NH_V_Press / ReMap (MTK)
//   ExecutionMD::ComputeVirial / ApplyPbc                                ExecutionMD.cpp:1239-1370
//   X2LamdaWorklet / Lamda2XWorklet / ApplyPbcFlagWorklet                RunWorklet.cpp:2602-2703
//   ContPointLocator::SetRange (cell dims of the new range)             locator/ContPointLocator.h:44-52
//
// The reference rescales its range on the host and keeps the force function's volume and box
// from Init.  Here one block per NPT system rewrites the system record on the device -- range,
// edges, cell dims, volume, the RBE sigma, S and proposal tables, the Ewald k lists -- and the
// atoms are carried along in reduced coordinates (a per-atom kernel for Berendsen; inside the
// kick-drift kernel for MTK, whose two half-step remaps bracket the drift).  All of it belongs to
// the fixed step sequence, so NPT steps replay from one CUDA graph like the NVT ones.  A scaling
// that would take an edge outside [kBoxShrink, kBoxGrow] x its initial length (the range the cell
// tables were sized for) or below num_cycles cells is refused: the status word gets kErrBoxRange
// and that remap leaves the box as it is.
#include "chain.cuh"

namespace rbmd {

namespace {
// Products and sums rounded one at a time (no contraction into FMA), as the CPU evaluates them.
__device__ inline double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double add(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double sub(double a, double b) { return __dsub_rn(a, b); }

// (a, b, c) of entry l of a k list built as a = -ka..ka, b = -kb..kb, c = -kc..kc (c fastest)
// with the zero vector, the middle entry of the full grid, left out.
__device__ inline void k_index(int l, const int km[3], double m[3]) {
  const int nb = 2 * km[1] + 1, nc = 2 * km[2] + 1;
  const int full = (2 * km[0] + 1) * nb * nc;
  const int f = l < (full - 1) / 2 ? l : l + 1;
  m[0] = (double)(f / (nb * nc) - km[0]);
  m[1] = (double)((f / nc) % nb - km[1]);
  m[2] = (double)(f % nc - km[2]);
}

// A range scaled by mu[k] about its centre (remap / ReMap), with the cell dims of the result.
struct BoxProp {
  double lo[3], hi[3], L[3];
  int dims[3], ncell;
  bool ok;
};

__device__ inline BoxProp propose(const SysDev& s, const double lo[3], const double hi[3], const double mu[3]) {
  BoxProp b;
  b.ncell = 1;
  b.ok = true;
  for (int k = 0; k < 3; ++k) {
    const bool fin = isfinite(mu[k]) && mu[k] > 0.0;
    const double ctr = mul(0.5, add(lo[k], hi[k]));
    b.lo[k] = add(mul(sub(lo[k], ctr), mu[k]), ctr);
    b.hi[k] = add(mul(sub(hi[k], ctr), mu[k]), ctr);
    b.L[k] = sub(b.hi[k], b.lo[k]);
    b.dims[k] = fin ? max(1, (int)(b.L[k] / (s.rc / s.nc))) : 1;
    b.ncell *= b.dims[k];
    if (!fin || !(b.L[k] >= mul(kBoxShrink, s.L0[k]) && b.L[k] <= mul(kBoxGrow, s.L0[k])) || b.dims[k] < s.nc)
      b.ok = false;
  }
  if (b.ncell > s.ncell_cap) b.ok = false;
  return b;
}

// Thread 0: writes an accepted box into the record with the scalars that follow from it; returns
// the H sums of S = H_x H_y H_z - 1 (ExecForceFunction.h:771-797) for the proposal tables.
__device__ inline void commit_box(SysDev& s, const BoxProp& b, double H[3]) {
  for (int k = 0; k < 3; ++k) {
    s.lo[k] = b.lo[k];
    s.hi[k] = b.hi[k];
    s.L[k] = b.L[k];
    s.dims[k] = b.dims[k];
    s.d[k] = b.L[k] / b.dims[k];
  }
  s.ncell = b.ncell;
  s.volume = mul(mul(b.L[0], b.L[1]), b.L[2]);
  if (s.coul != RBMD_COUL_NONE) {
    for (int k = 0; k < 3; ++k) {
      const double factor = -mul(mul(s.alpha, b.L[k]), b.L[k]);
      double h = 0.0;
      for (int m = -10; m <= 10; ++m) h = add(h, exp(mul((double)(m * m), factor)));
      H[k] = mul(h, sqrt(-factor / kPi));
      s.rbe_sigma[k] = mul(sqrt(s.alpha / 2.0), b.L[k]) / kPi;
    }
    s.S = sub(mul(mul(H[0], H[1]), H[2]), 1.0);
  }
}

// All threads of the block: RBE proposal tables P(m), q(m) (RBEPSample.h:85-113) and the Ewald
// force and energy k lists for edges L and volume vol.
__device__ inline void rebuild_tables(SysDev& s, const double L[3], double vol, const double H[3]) {
  const double alpha = s.alpha;
  if (s.coul == RBMD_COUL_RBE) {
    const int mmax = s.rbe_mmax, tw = 2 * mmax + 1;
    for (int e = threadIdx.x; e < 3 * tw; e += blockDim.x) {
      const int k = e / tw, m = e % tw - mmax;
      const double Lk = L[k], xm = (double)m;
      const double sc = sqrt(mul(alpha, pow(Lk, 2.0)) / pow(kPi, 2.0));
      const double P_m = exp(-pow(mul(2 * kPi, xm) / Lk, 2.0) / mul(4.0, alpha)) / H[k];
      double q_m;
      if (m == 0) q_m = erf((1.0 / 2) / sc);
      else q_m = sub(erf(add(1.0 / 2, fabs(xm)) / sc), erf(sub(fabs(xm), 1.0 / 2) / sc)) / 2;
      s.rbe_tab[(size_t)k * tw * 2 + (m + mmax)] = P_m;
      s.rbe_tab[(size_t)k * tw * 2 + tw + (m + mmax)] = q_m;
    }
  }
  if (s.coul != RBMD_COUL_NONE) {
    const int nk = max(s.nk_e, s.coul == RBMD_COUL_EWALD ? s.nk_ewald : 0);
    for (int l = threadIdx.x; l < nk; l += blockDim.x) {
      double m[3];
      k_index(l, s.kmax, m);
      const double kx = mul(2 * kPi, m[0]) / L[0], ky = mul(2 * kPi, m[1]) / L[1], kz = mul(2 * kPi, m[2]) / L[2];
      const double k2 = add(add(mul(kx, kx), mul(ky, ky)), mul(kz, kz));
      if (l < s.nk_e) {
        const double rk = sqrt(k2);
        const double r2 = mul(rk, rk);
        s.kv_e[l] = make_double4(kx, ky, kz, exp(-r2 / mul(4.0, alpha)) / r2);
      }
      if (s.coul == RBMD_COUL_EWALD && l < s.nk_ewald)
        s.kv[l] = make_double4(kx, ky, kz, mul((-4 * kPi) / mul(vol, k2), exp(-k2 / mul(4.0, alpha))));
    }
  }
}
}  // namespace

// ---------------------------------------------------------------- Berendsen (npt 1)
// End of the step: pressure of the step, one dilation mu = (1 - dt/P_damp (P_target - P)/B)^(1/3)
// for all edges, the new box and its tables.  k_baro_remap then moves the atoms.
__global__ void __launch_bounds__(256) k_baro_box(SysDev* __restrict__ S, const int* __restrict__ slots) {
  SysDev& s = S[slots[blockIdx.x]];
  if (s.npt != 1) return;
  SysState* st = s.st;
  __shared__ int s_ok;
  __shared__ double s_L[3], s_H[3], s_vol;
  if (threadIdx.x == 0) {
    double vir[6];
    const double press = pressure_scalar(s, st, vir);
    st->baro_pressure = press;
    for (int k = 0; k < 6; ++k) st->baro_virial[k] = vir[k];
    double delta = (double)st->step;
    if (delta != 0.0) delta = delta / (double)s.num_steps;
    const double dt_over_period = s.dt / s.p_damp;
    const double bulk_inv = 1.0 / s.bulk;
    const double target = add(s.p_start, mul(delta, sub(s.p_stop, s.p_start)));
    const double dil = pow(sub(1.0, mul(mul(dt_over_period, sub(target, press)), bulk_inv)), 1.0 / 3.0);
    const double mu[3] = {dil, dil, dil};
    const BoxProp b = propose(s, s.lo, s.hi, mu);
    if (b.ok) {
      for (int k = 0; k < 3; ++k) {
        st->baro_lo_old[k] = s.lo[k];
        st->baro_hinv_old[k] = 1.0 / s.L[k];  // set_global_box h_inv of the old box
        s_L[k] = b.L[k];
      }
      double H[3] = {0, 0, 0};
      commit_box(s, b, H);
      for (int k = 0; k < 3; ++k) s_H[k] = H[k];
      s_vol = s.volume;
    } else {
      atomicOr(&st->status, kErrBoxRange);
    }
    st->baro_apply = b.ok ? 1 : 0;
    s_ok = b.ok ? 1 : 0;
  }
  __syncthreads();
  if (s_ok) rebuild_tables(s, s_L, s_vol, s_H);
}

// remap (x2lamda with the old box, lamda2x with the new one) and ApplyPbcFlag on the new range.
__global__ void k_baro_remap(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int i = wk.y + threadIdx.x;
  if (s.npt != 1 || i >= s.n) return;
  const SysState* st = s.st;
  if (!st->baro_apply) return;
  double4 x = s.x[i];
  double p[3] = {x.x, x.y, x.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double lamda = mul(st->baro_hinv_old[k], sub(p[k], st->baro_lo_old[k]));
    p[k] = add(mul(s.L[k], lamda), s.lo[k]);
    if (p[k] < s.lo[k]) {
      p[k] = add(p[k], s.L[k]);
      s.image[3 * i + k] -= 1;
    } else if (p[k] >= s.hi[k]) {
      p[k] = sub(p[k], s.L[k]);
      s.image[3 * i + k] += 1;
    }
  }
  s.x[i] = make_double4(p[0], p[1], p[2], x.w);
}

// ---------------------------------------------------------------- MTK (npt 2)
// Step start, the scalar half of InitialIntegrate (ExecutionNPT.cpp:1671-1711): barostat chain
// half, thermostat chain half (velocity factor vscale_a), pressure with the previous step's virial,
// p_hydro, the barostat velocity half step and the NH_V_Press factors, then both half-step remaps
// by exp(dt/2 omega_dot) about the range centre.  The record ends at the box after the second
// remap; the first box and both maps stay in SysState for the kick-drift kernel.
__global__ void __launch_bounds__(256) k_mtk_begin(SysDev* __restrict__ S, const int* __restrict__ slots) {
  SysDev& s = S[slots[blockIdx.x]];
  if (s.npt != 2) return;
  SysState* st = s.st;
  __shared__ int s_changed;
  __shared__ double s_L[3], s_H[3], s_vol;
  if (threadIdx.x == 0) {
    st->step += 1;
    nhc_press_half(s, st);
    compute_temp_target(s, st);
    st->vscale_a = nhc_half(s, st);
    double vir[6];
    st->p_current = pressure_scalar(s, st, vir);
    press_target(s, st);
    omega_dot_half(s, st);
    double mu[3];
    for (int k = 0; k < 3; ++k) mu[k] = exp(0.5 * s.dt * st->omega_dot[k]);  // dto = dt / 2
    double lo0[3], hi0[3];
    for (int k = 0; k < 3; ++k) {
      lo0[k] = s.lo[k];
      hi0[k] = s.hi[k];
    }
    const BoxProp b1 = propose(s, lo0, hi0, mu);
    for (int k = 0; k < 3; ++k) {
      st->mtk_lo0[k] = lo0[k];
      st->mtk_hinv0[k] = 1.0 / s.L[k];
      st->mtk_lo1[k] = b1.ok ? b1.lo[k] : lo0[k];
      st->mtk_hi1[k] = b1.ok ? b1.hi[k] : hi0[k];
      st->mtk_L1[k] = b1.ok ? b1.L[k] : s.L[k];
      st->mtk_hinv1[k] = 1.0 / st->mtk_L1[k];
    }
    const BoxProp b2 = propose(s, st->mtk_lo1, st->mtk_hi1, mu);
    st->mtk_ok[0] = b1.ok ? 1 : 0;
    st->mtk_ok[1] = b2.ok ? 1 : 0;
    if (!b1.ok || !b2.ok) atomicOr(&st->status, kErrBoxRange);
    s_changed = (b1.ok || b2.ok) ? 1 : 0;
    if (s_changed) {
      double H[3] = {0, 0, 0};
      commit_box(s, b2.ok ? b2 : b1, H);
      for (int k = 0; k < 3; ++k) {
        s_H[k] = H[k];
        s_L[k] = s.L[k];
      }
      s_vol = s.volume;
    }
    // this step's force evaluation accumulates a fresh virial
    for (int c = 0; c < 6; ++c) st->virial[c] = 0.0;
  }
  __syncthreads();
  if (s_changed) rebuild_tables(s, s_L, s_vol, s_H);
}

void launch_barostat(const Batch& b, cudaStream_t st) {
  if (b.npt != 1) return;
  k_baro_box<<<b.nsys, 256, 0, st>>>(b.sys, b.d_slots);
  k_baro_remap<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  note_launch(2);
}

void launch_mtk_begin(const Batch& b, cudaStream_t st) {
  k_mtk_begin<<<b.nsys, 256, 0, st>>>(b.sys, b.d_slots);
  note_launch();
}

}  // namespace rbmd
