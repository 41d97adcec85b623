// k_kspace.cu -- random batch Ewald: k-vector sampling, structure factor, and the Ewald energy sum.
//
//   RBEPSAMPLE::Fetch_P_Sample / MH_Algorithm   framework/model/RBEPSample.h:64-177  (host in the
//                                                reference, reseeded mt19937 per draw)
//   ComputePnumberChargeStructureFactorWorklet + ReduceByKey  RunWorklet.cpp:2209-2270,
//                                                framework/run/ExecutionMD.cpp:469-501
//   ComputeEwaldEnergy                           framework/run/ExecutionMD.cpp:405-443
//
// Sampling runs on the device so a step never returns to the host: one block per system draws
// every Metropolis proposal and acceptance uniform in parallel from Philox (they do not depend on
// the chain state), then three lanes run the x, y, z chains in lock step, rejecting all-zero
// vectors together as the reference does.  Proposal probabilities come from per-system tables of
// P(m) and q(m) built on the host with the reference's formulas, so the chain makes the same
// accept/reject decisions as the CPU oracle on the same stream.
#include "kernels.h"

namespace rbmd {

constexpr int kMaxRbeSlots = 1024;  // proposal slots held in shared memory per system

// Box-Muller proposal of slot t, dimension d (FetchSample_1D, RBEPSample.h:115-145).
__device__ inline double rbe_gauss(const SysDev& s, uint32_t step, uint32_t t, int d) {
  double U1 = 0.5, U2 = 0.5;
  if (s.random_mode != RBMD_RANDOM_TEST) {
    for (uint32_t attempt = 0; attempt < 64; ++attempt) {  // P(U1 < 1e-6)^64 is nil
      uint32_t o[4];
      philox4x32_10(t, (uint32_t)d | (attempt << 2), step, kTagRbeGauss, s.seed_lo, s.seed_hi, o);
      U1 = u01(o[0], o[1]);
      U2 = u01(o[2], o[3]);
      if (!(U1 < 1e-6)) break;
    }
  }
  return s.rbe_sigma[d] * sqrt(-2.0 * log(U1)) * cos(2 * kPi * U2) + 0.0;
}

__device__ inline double rbe_accept(const SysDev& s, uint32_t step, uint32_t t, int d) {
  if (s.random_mode == RBMD_RANDOM_TEST) return 0.5;
  uint32_t o[4];
  philox4x32_10(t, (uint32_t)d, step, kTagRbeAccept, s.seed_lo, s.seed_hi, o);
  return u01(o[0], o[1]);
}

__global__ void __launch_bounds__(256) k_rbe_sample(const SysDev* __restrict__ S,
                                                    const int* __restrict__ slots) {
  const SysDev& s = S[slots[blockIdx.x]];
  if (s.coul != RBMD_COUL_RBE) return;
  __shared__ double s_m[kMaxRbeSlots * 3];
  __shared__ double s_u[kMaxRbeSlots * 3];
  const uint32_t step = (uint32_t)s.st->step;
  const int nslots = min(s.rbe_slots, kMaxRbeSlots);
  for (int k = threadIdx.x; k < nslots * 3; k += blockDim.x) {
    const int t = k / 3, d = k % 3;
    s_m[k] = round(rbe_gauss(s, step, (uint32_t)t, d));
    s_u[k] = rbe_accept(s, step, (uint32_t)t, d);
  }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const int d = lane < 3 ? lane : 0;
  const int mmax = s.rbe_mmax, tw = 2 * mmax + 1;
  const double* tabP = s.rbe_tab + (size_t)d * tw * 2;
  const double* tabQ = tabP + tw;
  const double eps = 1e-6;
  auto prop = [&](int t) -> double {
    return t < nslots ? s_m[t * 3 + d] : round(rbe_gauss(s, step, (uint32_t)t, d));
  };
  auto acc = [&](int t) -> double { return t < nslots ? s_u[t * 3 + d] : rbe_accept(s, step, (uint32_t)t, d); };
  // The reference loops until it finds non-zero vectors; bound the slots so that a degenerate
  // distribution (all proposals rounding to 0) ends with an error word instead of spinning.
  const int tmax = 4096 + 64 * s.P;
  int t = 0;
  bool exhausted = false;
  double X0;
  for (;;) {
    X0 = prop(t);
    ++t;
    const bool z = fabs(X0) < eps;
    const bool zx = __shfl_sync(0xffffffffu, z, 0), zy = __shfl_sync(0xffffffffu, z, 1),
               zz = __shfl_sync(0xffffffffu, z, 2);
    if (!(zx && zy && zz)) break;
    if (t >= tmax) {
      exhausted = true;
      X0 = (d == 0) ? 1.0 : 0.0;
      break;
    }
  }
  if (lane < 3) s.km[d] = (int)X0;
  for (int i = 1; i < s.P; ++i) {
    if (t >= tmax) {  // fill the rest with the last vector and flag the system
      exhausted = true;
      if (lane < 3) s.km[3 * i + d] = (int)X0;
      continue;
    }
    // MH_Algorithm, RBEPSample.h:64-83
    const double mw = prop(t);
    const double u = acc(t);
    ++t;
    double X1 = X0;
    const int im = (int)X0 + mmax, iw = (int)mw + mmax;
    double Prob = 0.0;
    if (iw >= 0 && iw < tw && im >= 0 && im < tw)
      Prob = (tabP[iw] / tabP[im]) * (tabQ[im] / tabQ[iw]);
    Prob = fmin(Prob, 1.0);
    if (u <= Prob) X1 = mw;
    if (lane < 3) s.km[3 * i + d] = (int)X1;
    X0 = X1;
    const bool z = fabs(X1) < eps;
    const bool zx = __shfl_sync(0xffffffffu, z, 0), zy = __shfl_sync(0xffffffffu, z, 1),
               zz = __shfl_sync(0xffffffffu, z, 2);
    if (zx && zy && zz) i = i - 1;
  }
  __syncwarp();
  // k vectors and force coefficients: k_l = 2 pi m_l / L, coef = -4 pi / (V |k_l|^2)
  for (int l = lane; l < s.P; l += 32) {
    const double kx = 2 * kPi * s.km[3 * l] / s.L[0];
    const double ky = 2 * kPi * s.km[3 * l + 1] / s.L[1];
    const double kz = 2 * kPi * s.km[3 * l + 2] / s.L[2];
    const double k2 = kx * kx + ky * ky + kz * kz;
    s.kv[l] = make_double4(kx, ky, kz, -4 * kPi / (s.volume * k2));
  }
  if (lane == 0 && exhausted) atomicOr(&s.st->status, kErrRbeSlots);
}

// Structure factor over a chunk of kRhoChunk atoms per block, every thread owning k indices; the
// last block of the system sums the chunk partials in chunk order (deterministic, FP64).
template <bool MIXED, bool ENERGY>
__global__ void __launch_bounds__(256) k_rho(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int nk = ENERGY ? s.nk_e : (s.coul == RBMD_COUL_RBE ? s.P : s.nk_ewald);
  const double4* kv = ENERGY ? s.kv_e : s.kv;
  __shared__ double4 s_x[kRhoChunk];
  __shared__ float4 s_u[kRhoChunk];
  const int a0 = wk.y;
  const int na = min(kRhoChunk, s.n - a0);
  for (int k = threadIdx.x; k < na; k += blockDim.x) {
    const double4 p = s.x[a0 + k];
    s_x[k] = p;
    if (MIXED)
      s_u[k] = make_float4((float)(p.x / s.L[0]), (float)(p.y / s.L[1]), (float)(p.z / s.L[2]), (float)p.w);
  }
  __syncthreads();
  const int blk = a0 / kRhoChunk;
  double* part = s.rho_part + (size_t)blk * 2 * nk;
  for (int l = threadIdx.x; l < nk; l += blockDim.x) {
    const double4 k = kv[l];
    double re = 0.0, im = 0.0;
    if (MIXED && !ENERGY) {
      // phase in turns m . (r / L), reduced to [-1/2, 1/2] before the FP32 sine and cosine (the
      // SFU approximations, absolute error about 4e-7 on [-pi, pi])
      const float mxr = (float)s.km[3 * l], myr = (float)s.km[3 * l + 1], mzr = (float)s.km[3 * l + 2];
      // FP32 partial sums over 32 atoms, added in FP64 (the SFU, which also converts FP32 to
      // FP64, is this loop's bottleneck); the nearest integer of the phase by the 1.5 * 2^23
      // addition (round to nearest even, |ph| < 2^22), on the FMA pipe
      for (int j0 = 0; j0 < na; j0 += 32) {
        const int j1 = min(na, j0 + 32);
        float pr = 0.0f, pm = 0.0f;
        for (int j = j0; j < j1; ++j) {
          const float4 u = s_u[j];
          float ph = mxr * u.x + myr * u.y + mzr * u.z;
          ph -= __fsub_rn(__fadd_rn(ph, 12582912.0f), 12582912.0f);
          float sn, cs;
          __sincosf(6.28318531f * ph, &sn, &cs);  // hardware sin / cos: |2 pi ph| <= pi
          pr += u.w * cs;
          pm += u.w * sn;
        }
        re += (double)pr;
        im += (double)pm;
      }
    } else {
      for (int j = 0; j < na; ++j) {
        const double4 p = s_x[j];
        const double dot = k.x * p.x + k.y * p.y + k.z * p.z;
        double sn, cs;
        sincos(dot, &sn, &cs);
        re += p.w * cs;
        im += p.w * sn;
      }
    }
    part[2 * l] = re;
    part[2 * l + 1] = im;
  }
  if (arrive_last(&s.st->counter[ENERGY ? 4 : 1], (unsigned)s.blocks_rho)) {
    double* out = ENERGY ? s.rhok_e : s.rhok;
    double esum = 0.0;
    for (int l = threadIdx.x; l < nk; l += blockDim.x) {
      double re = 0.0, im = 0.0;
      for (int b = 0; b < s.blocks_rho; ++b) {
        re += __ldcg(&s.rho_part[(size_t)b * 2 * nk + 2 * l]);
        im += __ldcg(&s.rho_part[(size_t)b * 2 * nk + 2 * l + 1]);
      }
      out[2 * l] = re;
      out[2 * l + 1] = im;
      if (ENERGY) esum += kv[l].w * (re * re + im * im);
    }
    if (ENERGY) {
      // fixed-order block reduction of the energy terms
      __shared__ double s_e[256];
      s_e[threadIdx.x] = esum;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)blockDim.x; ++k) t += s_e[k];
        s.st->energy[6] = t;
      }
    }
  }
}

void launch_rbe_sample(const Batch& b, cudaStream_t st) {
  k_rbe_sample<<<b.nsys, 256, 0, st>>>(b.sys, b.d_slots);
  note_launch();
}

void launch_rho(const Batch& b, cudaStream_t st, int ewald) {
  (void)ewald;
  if (b.prec == RBMD_PREC_MIXED && b.coul == RBMD_COUL_RBE)
    k_rho<true, false><<<b.rho.n, 256, 0, st>>>(b.sys, b.rho.d);
  else
    k_rho<false, false><<<b.rho.n, 256, 0, st>>>(b.sys, b.rho.d);
  note_launch();
}

void launch_ewald_energy(const Batch& b, cudaStream_t st) {
  k_rho<false, true><<<b.rho.n, 256, 0, st>>>(b.sys, b.rho.d);
  note_launch();
}

}  // namespace rbmd
