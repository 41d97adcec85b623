// k_baro.cu -- NPT Berendsen barostat: the pressure of the step, the isotropic dilation, the new
// box with every table that follows from it, and the remap of the atoms.
//
//   ExecutionNPT::fix_press_berendsen / Compute_Pressure_Scalar / remap   ExecutionNPT.cpp:1334-1368,
//                                                                        1429-1447, 1506-1538
//   ExecutionMD::ComputeVirial / ApplyPbc                                ExecutionMD.cpp:1239-1370
//   X2LamdaWorklet / Lamda2XWorklet / ApplyPbcFlagWorklet                RunWorklet.cpp:2602-2703
//   ContPointLocator::SetRange (cell dims of the new range)             locator/ContPointLocator.h:44-52
//
// The reference rescales its range on the host and keeps the force function's volume and box
// from Init.  Here one block per NPT system rewrites the system record on the device -- range,
// edges, cell dims, volume, the RBE sigma, S and proposal tables, the Ewald k lists -- and a
// per-atom kernel carries the atoms along in reduced coordinates.  Both kernels belong to the
// fixed step sequence, so NPT steps replay from one CUDA graph like the NVT ones.  A dilation that
// would take an edge outside [kBoxShrink, kBoxGrow] x its initial length (the range the cell
// tables were sized for) or below num_cycles cells is refused: the status word gets
// kErrBoxRange and the box stays put.
#include "kernels.h"

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
}  // namespace

__global__ void __launch_bounds__(256) k_baro_box(SysDev* __restrict__ S, const int* __restrict__ slots) {
  SysDev& s = S[slots[blockIdx.x]];
  if (!s.npt) return;
  SysState* st = s.st;
  __shared__ int s_ok;
  __shared__ double s_L[3], s_H[3], s_vol;
  if (threadIdx.x == 0) {
    // Compute_Pressure_Scalar: virial of the step's force evaluation plus the SHAKE virial
    // (ComputeVirial; EAM contributes none), temperature as ComputeTempe left it
    double vir[6];
    for (int k = 0; k < 6; ++k) {
      vir[k] = st->virial[k];
      if (s.fix_shake == RBMD_SHAKE_TRUE) vir[k] = add(vir[k], st->shake_virial[k]);
      if (s.ff == RBMD_FF_EAM) vir[k] = 0.0;
      st->baro_virial[k] = vir[k];
    }
    const double kin = mul(mul(st->tdof, s.boltz), st->temperature);
    const double press = mul(mul(add(add(add(kin, vir[0]), vir[1]), vir[2]) / 3.0, 1.0 / s.volume), s.nktv2p);
    st->baro_pressure = press;
    // fix_press_berendsen: target ramped over the run, one dilation for all three edges
    double delta = (double)st->step;
    if (delta != 0.0) delta = delta / (double)s.num_steps;
    const double dt_over_period = s.dt / s.p_damp;
    const double bulk_inv = 1.0 / s.bulk;
    const double target = add(s.p_start, mul(delta, sub(s.p_stop, s.p_start)));
    const double dil = pow(sub(1.0, mul(mul(dt_over_period, sub(target, press)), bulk_inv)), 1.0 / 3.0);
    // remap: scale the range about its centre
    double nlo[3], nhi[3], nL[3];
    int dims[3], ncell = 1;
    bool ok = isfinite(dil) && dil > 0.0;
    for (int k = 0; k < 3; ++k) {
      const double ctr = mul(0.5, add(s.lo[k], s.hi[k]));
      nlo[k] = add(mul(sub(s.lo[k], ctr), dil), ctr);
      nhi[k] = add(mul(sub(s.hi[k], ctr), dil), ctr);
      nL[k] = sub(nhi[k], nlo[k]);
      dims[k] = ok ? max(1, (int)(nL[k] / (s.rc / s.nc))) : 1;
      ncell *= dims[k];
      if (!(nL[k] >= mul(kBoxShrink, s.L0[k]) && nL[k] <= mul(kBoxGrow, s.L0[k])) || dims[k] < s.nc) ok = false;
    }
    if (ncell > s.ncell_cap) ok = false;
    if (ok) {
      for (int k = 0; k < 3; ++k) {
        st->baro_lo_old[k] = s.lo[k];
        st->baro_hinv_old[k] = 1.0 / s.L[k];  // set_global_box h_inv of the old box
        s.lo[k] = nlo[k];
        s.hi[k] = nhi[k];
        s.L[k] = nL[k];
        s.dims[k] = dims[k];
        s.d[k] = nL[k] / dims[k];
        s_L[k] = nL[k];
      }
      s.ncell = ncell;
      s.volume = mul(mul(nL[0], nL[1]), nL[2]);
      s_vol = s.volume;
      if (s.coul != RBMD_COUL_NONE) {
        // S = H_x H_y H_z - 1 (ExecForceFunction.h:771-797)
        for (int k = 0; k < 3; ++k) {
          const double factor = -mul(mul(s.alpha, nL[k]), nL[k]);
          double H = 0.0;
          for (int m = -10; m <= 10; ++m) H = add(H, exp(mul((double)(m * m), factor)));
          s_H[k] = mul(H, sqrt(-factor / kPi));
          s.rbe_sigma[k] = mul(sqrt(s.alpha / 2.0), nL[k]) / kPi;
        }
        s.S = sub(mul(mul(s_H[0], s_H[1]), s_H[2]), 1.0);
      }
    } else {
      atomicOr(&st->status, kErrBoxRange);
    }
    st->baro_apply = ok ? 1 : 0;
    s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  if (!s_ok) return;
  const double alpha = s.alpha;
  // RBE proposal tables P(m), q(m) of the new edges (RBEPSample.h:85-113)
  if (s.coul == RBMD_COUL_RBE) {
    const int mmax = s.rbe_mmax, tw = 2 * mmax + 1;
    for (int e = threadIdx.x; e < 3 * tw; e += blockDim.x) {
      const int k = e / tw, m = e % tw - mmax;
      const double Lk = s_L[k], xm = (double)m;
      const double sc = sqrt(mul(alpha, pow(Lk, 2.0)) / pow(kPi, 2.0));
      const double P_m = exp(-pow(mul(2 * kPi, xm) / Lk, 2.0) / mul(4.0, alpha)) / s_H[k];
      double q_m;
      if (m == 0) q_m = erf((1.0 / 2) / sc);
      else q_m = sub(erf(add(1.0 / 2, fabs(xm)) / sc), erf(sub(fabs(xm), 1.0 / 2) / sc)) / 2;
      s.rbe_tab[(size_t)k * tw * 2 + (m + mmax)] = P_m;
      s.rbe_tab[(size_t)k * tw * 2 + tw + (m + mmax)] = q_m;
    }
  }
  // Ewald force k list and the energy k list of the new edges
  if (s.coul != RBMD_COUL_NONE) {
    const int nk = max(s.nk_e, s.coul == RBMD_COUL_EWALD ? s.nk_ewald : 0);
    for (int l = threadIdx.x; l < nk; l += blockDim.x) {
      double m[3];
      k_index(l, s.kmax, m);
      const double kx = mul(2 * kPi, m[0]) / s_L[0], ky = mul(2 * kPi, m[1]) / s_L[1],
                   kz = mul(2 * kPi, m[2]) / s_L[2];
      const double k2 = add(add(mul(kx, kx), mul(ky, ky)), mul(kz, kz));
      if (l < s.nk_e) {
        const double rk = sqrt(k2);
        const double r2 = mul(rk, rk);
        s.kv_e[l] = make_double4(kx, ky, kz, exp(-r2 / mul(4.0, alpha)) / r2);
      }
      if (s.coul == RBMD_COUL_EWALD && l < s.nk_ewald)
        s.kv[l] = make_double4(kx, ky, kz, mul((-4 * kPi) / mul(s_vol, k2), exp(-k2 / mul(4.0, alpha))));
    }
  }
}

// remap (x2lamda with the old box, lamda2x with the new one) and ApplyPbcFlag on the new range.
__global__ void k_baro_remap(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int i = wk.y + threadIdx.x;
  if (!s.npt || i >= s.n) return;
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

void launch_barostat(const Batch& b, cudaStream_t st) {
  if (!b.npt) return;
  k_baro_box<<<b.nsys, 256, 0, st>>>(b.sys, b.d_slots);
  k_baro_remap<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  note_launch(2);
}

}  // namespace rbmd
