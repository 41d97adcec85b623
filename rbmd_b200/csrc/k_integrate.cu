// k_integrate.cu -- velocity Verlet, Nose-Hoover chain, Berendsen / rescale, SHAKE / RATTLE,
// harmonic bonded terms, and the final per-atom kernel that assembles the force.
//
//   UpdateVelocityWorklet / UpdatePositionFlagWorklet / ApplyPbcFlagWorklet  RunWorklet.cpp:2357-2636
//   ExecutionNVT::{InitialIntegrate, FinalIntegrate, NHCTempIntegrate, ComputeTempe, SetUp,
//                  ComputeTempTarget, UpdateVelocityByTempConType}  ExecutionNVT.cpp:270-291,736-773,
//                                                                   1106-1256
//   ComputeNewRBEForceWorklet / ComputeNewFarElectrostaticsWorklet   RunWorklet.cpp:2086-2141,2492-2540
//   SumRBLCorrForce (mean subtraction), SumFarNearForce, AddForceWorklet, UnitRescaleWorklet
//   ComputeSpecialCoulGeneralWorklet                                 RunWorklet.cpp:2012-2084
//   ComputeBondHarmonicWorklet / ComputeAngleHarmonicWorklet        MolecularWorklet.h:58-397
//   NewConstraintA/BWaterBondAngleWorklet                            MolecularWorklet.h:2367-2832
//
// The scalar thermostat work runs on the device in the last block of each system (last-block
// reduction of the kinetic-energy partials), so a whole step is a fixed kernel sequence with no
// host round trip and can be captured in a CUDA graph.
#include "chain.cuh"

namespace rbmd {

// Step start: Executioner::TakeStep increments the step; InitialIntegrate runs the first chain half.
__global__ void k_nhc_a(const SysDev* __restrict__ S, const int* __restrict__ slots, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const SysDev& s = S[slots[k]];
  SysState* st = s.st;
  st->step += 1;
  // NPT Berendsen: the step's force evaluation accumulates the virial the barostat reads (the RBL
  // pair kernels add nothing to it, so it starts from zero here)
  if (s.npt)
    for (int c = 0; c < 6; ++c) st->virial[c] = 0.0;
  if (s.temp_ctrl == RBMD_TC_NOSE_HOOVER) {
    compute_temp_target(s, st);
    st->vscale_a = nhc_half(s, st);
  } else {
    st->vscale_a = 1.0;
  }
}

// v = v * pending * a; v += F/m dt/2; x += v dt; periodic wrap with image flags.  MTK systems
// (npt 2) also take the NH_V_Press factors twice before the kick and are remapped to the first
// half-step box before the drift and to the second after it (InitialIntegrate,
// ExecutionNPT.cpp:1671-1711); the wrap uses the first box and the second remap does not wrap.
__global__ void k_kick_drift(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int i = wk.y + threadIdx.x;
  if (i >= s.n) return;
  const SysState* st = s.st;
  const int flags = s.meta[i].z;
  const double pend = (flags & 1) ? st->vscale_pending_c : st->vscale_pending;
  const double fa = st->vscale_a;
  double4 v = s.v[i];
  const double4 F = s.f[i];
  double vx = v.x * pend, vy = v.y * pend, vz = v.z * pend;
  vx = fa * vx;
  vy = fa * vy;
  vz = fa * vz;
  const bool mtk = s.npt == 2;
  if (mtk)
    for (int r = 0; r < 2; ++r) {
      vx = st->f_press[0] * vx;
      vy = st->f_press[1] * vy;
      vz = st->f_press[2] * vz;
    }
  if (s.has_triples) s.vold[i] = make_double4(vx, vy, vz, v.w);
  const double m = v.w, dt = s.dt, c = s.fmt2v;
  vx += 0.5 * F.x / m * dt * c;
  vy += 0.5 * F.y / m * dt * c;
  vz += 0.5 * F.z / m * dt * c;
  s.v[i] = make_double4(vx, vy, vz, m);
  double4 x = s.x[i];
  if (mtk && st->mtk_ok[0]) {
    x.x = __dadd_rn(__dmul_rn(st->mtk_L1[0], __dmul_rn(st->mtk_hinv0[0], __dsub_rn(x.x, st->mtk_lo0[0]))), st->mtk_lo1[0]);
    x.y = __dadd_rn(__dmul_rn(st->mtk_L1[1], __dmul_rn(st->mtk_hinv0[1], __dsub_rn(x.y, st->mtk_lo0[1]))), st->mtk_lo1[1]);
    x.z = __dadd_rn(__dmul_rn(st->mtk_L1[2], __dmul_rn(st->mtk_hinv0[2], __dsub_rn(x.z, st->mtk_lo0[2]))), st->mtk_lo1[2]);
  }
  if (s.has_triples) s.xold[i] = x;
  double p[3] = {x.x + vx * dt, x.y + vy * dt, x.z + vz * dt};
  const double* blo = mtk ? st->mtk_lo1 : s.lo;
  const double* bhi = mtk ? st->mtk_hi1 : s.hi;
  const double* bL = mtk ? st->mtk_L1 : s.L;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (p[k] < blo[k]) {
      p[k] += bL[k];
      s.image[3 * i + k] -= 1;
    } else if (p[k] >= bhi[k]) {
      p[k] -= bL[k];
      s.image[3 * i + k] += 1;
    }
  }
  if (mtk && st->mtk_ok[1]) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      p[k] = __dadd_rn(__dmul_rn(s.L[k], __dmul_rn(st->mtk_hinv1[k], __dsub_rn(p[k], st->mtk_lo1[k]))), s.lo[k]);
  }
  s.x[i] = make_double4(p[0], p[1], p[2], x.w);
}

// Applies the pending end-of-step velocity factor (between rbmd_step calls the stored velocities
// are always final).
__global__ void k_flush_vscale(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int i = wk.y + threadIdx.x;
  SysState* st = s.st;
  if (i < s.n) {
    const int flags = s.meta[i].z;
    const double pend = (flags & 1) ? st->vscale_pending_c : st->vscale_pending;
    double4 v = s.v[i];
    v.x *= pend;
    v.y *= pend;
    v.z *= pend;
    s.v[i] = v;
  }
  if (arrive_last(&st->counter[6], (unsigned)s.blocks_atom)) {
    if (threadIdx.x == 0) {
      st->vscale_pending = 1.0;
      st->vscale_pending_c = 1.0;
    }
  }
}

// ------------------------------------------------------------------ bonded terms
__global__ void k_bonded(const SysDev* __restrict__ S, const int2* __restrict__ work, int virial) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int t = wk.y + threadIdx.x;
  if (t >= s.n_bonds + s.n_angles + s.n_dihedrals) return;
  if (t >= s.n_bonds + s.n_angles) {
    // ComputeDihedralHarmonicWorklet, MolecularWorklet.h:669-973: E = K [1 + d cos(n phi)]
    const int q = t - s.n_bonds - s.n_angles;
    const int i1 = s.dih_atoms[4 * q], i2 = s.dih_atoms[4 * q + 1], i3 = s.dih_atoms[4 * q + 2],
              i4 = s.dih_atoms[4 * q + 3];
    const int ty = s.dih_type[q];
    const double K = s.dih_k[ty];
    const int m = s.dih_mult[ty];
    const double cos_shift = s.dih_sign[ty] == 1 ? 1.0 : -1.0, sin_shift = 0.0;
    const double4 p1 = s.x[i1], p2 = s.x[i2], p3 = s.x[i3], p4 = s.x[i4];
    double vb1[3] = {p1.x - p2.x, p1.y - p2.y, p1.z - p2.z};
    double vb2[3] = {p3.x - p2.x, p3.y - p2.y, p3.z - p2.z};
    double vb3[3] = {p4.x - p3.x, p4.y - p3.y, p4.z - p3.z};
    min_image(vb1[0], vb1[1], vb1[2], s.L[0], s.L[1], s.L[2]);
    min_image(vb2[0], vb2[1], vb2[2], s.L[0], s.L[1], s.L[2]);
    min_image(vb3[0], vb3[1], vb3[2], s.L[0], s.L[1], s.L[2]);
    const double vb2m[3] = {-vb2[0], -vb2[1], -vb2[2]};
    const double ax = vb1[1] * vb2m[2] - vb1[2] * vb2m[1];
    const double ay = vb1[2] * vb2m[0] - vb1[0] * vb2m[2];
    const double az = vb1[0] * vb2m[1] - vb1[1] * vb2m[0];
    const double bx = vb3[1] * vb2m[2] - vb3[2] * vb2m[1];
    const double by = vb3[2] * vb2m[0] - vb3[0] * vb2m[2];
    const double bz = vb3[0] * vb2m[1] - vb3[1] * vb2m[0];
    const double rasq = ax * ax + ay * ay + az * az;
    const double rbsq = bx * bx + by * by + bz * bz;
    const double rg = sqrt(vb2m[0] * vb2m[0] + vb2m[1] * vb2m[1] + vb2m[2] * vb2m[2]);
    const double rginv = rg > 0 ? 1.0 / rg : 0.0, ra2inv = rasq > 0 ? 1.0 / rasq : 0.0;
    const double rb2inv = rbsq > 0 ? 1.0 / rbsq : 0.0;
    const double rabinv = sqrt(ra2inv * rb2inv);
    double c = (ax * bx + ay * by + az * bz) * rabinv;
    const double sn = rg * rabinv * (ax * vb3[0] + ay * vb3[1] + az * vb3[2]);
    c = fmin(fmax(c, -1.0), 1.0);
    double pp = 1.0, ddf1 = 0.0, df1 = 0.0;
    for (int r = 0; r < m; r++) {  // cos(n phi), sin(n phi) by the angle-addition recurrence
      ddf1 = pp * c - df1 * sn;
      df1 = pp * sn + df1 * c;
      pp = ddf1;
    }
    pp = pp * cos_shift + df1 * sin_shift;
    df1 = df1 * cos_shift - ddf1 * sin_shift;
    df1 *= -m;
    pp += 1.0;
    if (m == 0) {
      pp = 1.0 + cos_shift;
      df1 = 0.0;
    }
    s.term_energy[t] = K * pp;
    const double fg = vb1[0] * vb2m[0] + vb1[1] * vb2m[1] + vb1[2] * vb2m[2];
    const double hg = vb3[0] * vb2m[0] + vb3[1] * vb2m[1] + vb3[2] * vb2m[2];
    const double fga = fg * ra2inv * rginv, hgb = hg * rb2inv * rginv;
    const double gaa = -ra2inv * rg, gbb = rb2inv * rg;
    const double df = -K * df1;
    const double a3[3] = {ax, ay, az}, b3[3] = {bx, by, bz};
    double f1[3], f3[3], f4[3], f2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double s2 = df * (fga * a3[k] - hgb * b3[k]);
      f1[k] = df * (gaa * a3[k]);
      f2[k] = s2 - f1[k];
      f4[k] = df * (gbb * b3[k]);
      f3[k] = -s2 - f4[k];
    }
    const int base = 2 * s.n_bonds + 3 * s.n_angles + 4 * q;
    s.term_force[base] = make_double4(f1[0], f1[1], f1[2], 0.0);
    s.term_force[base + 1] = make_double4(f2[0], f2[1], f2[2], 0.0);
    s.term_force[base + 2] = make_double4(f3[0], f3[1], f3[2], 0.0);
    s.term_force[base + 3] = make_double4(f4[0], f4[1], f4[2], 0.0);
    if (virial) {
      double* v = s.term_vir + 6 * (size_t)t;
      v[0] = vb1[0] * f1[0] + vb2[0] * f3[0] + (vb3[0] + vb2[0]) * f4[0];
      v[1] = vb1[1] * f1[1] + vb2[1] * f3[1] + (vb3[1] + vb2[1]) * f4[1];
      v[2] = vb1[2] * f1[2] + vb2[2] * f3[2] + (vb3[2] + vb2[2]) * f4[2];
      v[3] = vb1[0] * f1[1] + vb2[0] * f3[1] + (vb3[0] + vb2[0]) * f4[1];
      v[4] = vb1[0] * f1[2] + vb2[0] * f3[2] + (vb3[0] + vb2[0]) * f4[2];
      v[5] = vb1[1] * f1[2] + vb2[1] * f3[2] + (vb3[1] + vb2[1]) * f4[2];
    }
    return;
  }
  if (t < s.n_bonds) {
    // ComputeBondHarmonicWorklet, MolecularWorklet.h:58-199
    const int i = s.bond_atoms[2 * t], j = s.bond_atoms[2 * t + 1];
    const double kk = s.bond_k[s.bond_type[t]], r0 = s.bond_r0[s.bond_type[t]];
    const double4 pi = s.x[i], pj = s.x[j];
    double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
    min_image(rx, ry, rz, s.L[0], s.L[1], s.L[2]);
    const double dis = sqrt(rx * rx + ry * ry + rz * rz);
    const double dr = dis - r0, rk = kk * dr;
    const double fb = dis > 0.01 ? -2.0 * rk / dis : 0.0;
    const double fx = rx * fb, fy = ry * fb, fz = rz * fb;
    s.term_force[2 * t] = make_double4(fx, fy, fz, 0.0);
    s.term_force[2 * t + 1] = make_double4(-fx, -fy, -fz, 0.0);
    s.term_energy[t] = rk * dr;
    if (virial) {
      double* v = s.term_vir + 6 * (size_t)t;
      v[0] = rx * fx; v[1] = ry * fy; v[2] = rz * fz; v[3] = rx * fy; v[4] = rx * fz; v[5] = ry * fz;
    }
  } else {
    // ComputeAngleHarmonicWorklet, MolecularWorklet.h:231-397
    const int a = t - s.n_bonds;
    const int i = s.angle_atoms[3 * a], j = s.angle_atoms[3 * a + 1], k = s.angle_atoms[3 * a + 2];
    const double kk = s.angle_k[s.angle_type[a]], th0 = s.angle_t0[s.angle_type[a]];
    const double4 pi = s.x[i], pj = s.x[j], pk = s.x[k];
    double ax = pi.x - pj.x, ay = pi.y - pj.y, az = pi.z - pj.z;
    double bx = pk.x - pj.x, by = pk.y - pj.y, bz = pk.z - pj.z;
    min_image(ax, ay, az, s.L[0], s.L[1], s.L[2]);
    min_image(bx, by, bz, s.L[0], s.L[1], s.L[2]);
    const double d1s = ax * ax + ay * ay + az * az, d1 = sqrt(d1s);
    const double d2s = bx * bx + by * by + bz * bz, d2 = sqrt(d2s);
    double c = (ax * bx + ay * by + az * bz) / (d1 * d2);
    c = fmin(fmax(c, -1.0), 1.0);
    double sn = sqrt(1.0 - c * c);
    if (sn < 0.001) sn = 0.001;
    sn = 1.0 / sn;
    const double dth = acos(c) - (th0 * kPif) / 180;
    const double tk = kk * dth;
    const double aa = -2.0 * tk * sn;
    const double a11 = aa * c / d1s, a12 = -aa / (d1 * d2), a22 = aa * c / d2s;
    const double fix = a11 * ax + a12 * bx, fiy = a11 * ay + a12 * by, fiz = a11 * az + a12 * bz;
    const double fkx = a22 * bx + a12 * ax, fky = a22 * by + a12 * ay, fkz = a22 * bz + a12 * az;
    const int base = 2 * s.n_bonds + 3 * a;
    s.term_force[base] = make_double4(fix, fiy, fiz, 0.0);
    s.term_force[base + 1] = make_double4(-fix - fkx, -fiy - fky, -fiz - fkz, 0.0);
    s.term_force[base + 2] = make_double4(fkx, fky, fkz, 0.0);
    s.term_energy[t] = tk * dth;
    if (virial) {
      double* v = s.term_vir + 6 * (size_t)t;
      v[0] = ax * fix + bx * fkx; v[1] = ay * fiy + by * fky; v[2] = az * fiz + bz * fkz;
      v[3] = ax * fiy + bx * fky; v[4] = ax * fiz + bx * fkz; v[5] = ay * fiz + by * fkz;
    }
  }
}

// ------------------------------------------------------------------ final force + kick
template <bool MIXED, bool VIRIAL>
__global__ void __launch_bounds__(kAtomBlock, 4)
k_final(const SysDev* __restrict__ S, const int2* __restrict__ work, int mode) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int i = wk.y + threadIdx.x;
  const bool act = i < s.n;
  SysState* st = s.st;
  __shared__ double4 s_k[256];
  __shared__ double2 s_r[256];
  __shared__ float4 s_kf[256];
  __shared__ float2 s_rf[256];
  float4* s_kk = reinterpret_cast<float4*>(s_k);  // mixed precision: FP32 k vectors (s_k unused)
  __shared__ double s_part[kAtomBlock / 32][8];

  double4 xi = act ? s.x[i] : make_double4(0, 0, 0, 0);
  double F[3] = {0, 0, 0};
  if (act) {
    const double4 fn = s.f[i];
    F[0] = fn.x;
    F[1] = fn.y;
    F[2] = fn.z;
  }
  if (s.neigh == RBMD_NEIGH_RBL) {
    // SumRBLCorrForce: near_i - mean(near), ExecutionMD.cpp:663-667, 820-826, 1097-1099
    F[0] -= st->fmean[0];
    F[1] -= st->fmean[1];
    F[2] -= st->fmean[2];
  }
  double vir[6] = {0, 0, 0, 0, 0, 0};
  // ---- far field
  const bool far = (s.ff == RBMD_FF_LJ_CUT_COUL_LONG || s.ff == RBMD_FF_CVFF) && s.coul != RBMD_COUL_NONE;
  if (far) {
    const int nk = s.coul == RBMD_COUL_RBE ? s.P : s.nk_ewald;
    double fx = 0, fy = 0, fz = 0;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    const float ux = (float)(xi.x / s.L[0]), uy = (float)(xi.y / s.L[1]), uz = (float)(xi.z / s.L[2]);
    for (int k0 = 0; k0 < nk; k0 += 256) {
      const int nch = min(256, nk - k0);
      __syncthreads();
      for (int k = threadIdx.x; k < nch; k += blockDim.x) {
        const double4 kv = s.kv[k0 + k];
        const double re = s.rhok[2 * (k0 + k)], im = s.rhok[2 * (k0 + k) + 1];
        if (MIXED) {
          const int l = k0 + k;
          s_kf[k] = make_float4((float)s.km[3 * l], (float)s.km[3 * l + 1], (float)s.km[3 * l + 2], (float)kv.w);
          s_rf[k] = make_float2((float)re, (float)im);
          s_kk[k] = make_float4((float)kv.x, (float)kv.y, (float)kv.z, 0.0f);
        } else {
          s_k[k] = kv;
          s_r[k] = make_double2(re, im);
        }
      }
      __syncthreads();
      if (act) {
        if (MIXED) {
          const float q = (float)xi.w;
          for (int k = 0; k < nch; ++k) {
            const float4 m = s_kf[k];
            float ph = m.x * ux + m.y * uy + m.z * uz;
            ph -= __fsub_rn(__fadd_rn(ph, 12582912.0f), 12582912.0f);  // rint on the FMA pipe, |ph| < 2^22
            float sn, cs;
            __sincosf(6.28318531f * ph, &sn, &cs);  // hardware sin / cos: |2 pi ph| <= pi
            const float2 r = s_rf[k];
            const float Fs = m.w * q * (cs * r.y - sn * r.x);
            const float4 kf = s_kk[k];
            gx += Fs * kf.x;
            gy += Fs * kf.y;
            gz += Fs * kf.z;
          }
        } else {
          for (int k = 0; k < nch; ++k) {
            const double4 kv = s_k[k];
            const double2 r = s_r[k];
            const double dot = kv.x * xi.x + kv.y * xi.y + kv.z * xi.z;
            double sn, cs;
            sincos(dot, &sn, &cs);
            const double Fs = kv.w * xi.w * (cs * r.y - sn * r.x);
            fx += Fs * kv.x;
            fy += Fs * kv.y;
            fz += Fs * kv.z;
            if (VIRIAL) {  // ComputeKspaceVirial, ExecForceFunction.h:397-410
              vir[0] += (xi.x * kv.x + xi.x * kv.x) * Fs;
              vir[1] += (xi.y * kv.y + xi.y * kv.y) * Fs;
              vir[2] += (xi.z * kv.z + xi.z * kv.z) * Fs;
              vir[3] += (xi.x * kv.y + xi.y * kv.x) * Fs;
              vir[4] += (xi.x * kv.z + xi.z * kv.x) * Fs;
              vir[5] += (xi.y * kv.z + xi.z * kv.y) * Fs;
            }
          }
        }
      }
    }
    if (MIXED) {
      fx = gx;
      fy = gy;
      fz = gz;
    }
    const double sc = (s.coul == RBMD_COUL_RBE ? s.S / s.P : 1.0) * s.qqr2e;
    F[0] = fx * sc + F[0];
    F[1] = fy * sc + F[1];
    F[2] = fz * sc + F[2];
    if (VIRIAL)
      for (int k = 0; k < 6; ++k) vir[k] *= sc;
  }
  if (act) {
    // ---- intramolecular Coulomb exclusion (CVFF + RBL + special bonds)
    if (s.ff == RBMD_FF_CVFF && s.neigh == RBMD_NEIGH_RBL && s.special) {
      const int4 mi = s.meta[i];
      const int b = s.mol_off[mi.y], e = s.mol_off[mi.y + 1];
      if (e - b >= 3) {
        const int sb = s.sp_off[i], se = s.sp_off[i + 1];
        for (int k = b; k < e; ++k) {
          const int j = s.mol_atoms[k];
          if (j == i) continue;
          const double4 xj = s.x[j];
          double rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
          min_image(rx, ry, rz, s.L[0], s.L[1], s.L[2]);
          const double dis = sqrt(rx * rx + ry * ry + rz * rz);
          const double fc = -332.06371 * xi.w * xj.w / (dis * dis * dis);
          double w = 1.0;
          for (int q = sb; q < se; ++q)
            if (s.sp_ids[q] == j) w = s.sp_w[q];
          const double cx = (1.0 - w) * fc * rx, cy = (1.0 - w) * fc * ry, cz = (1.0 - w) * fc * rz;
          F[0] += cx;
          F[1] += cy;
          F[2] += cz;
          if (VIRIAL) {
            vir[0] += rx * 0.5 * cx; vir[1] += ry * 0.5 * cy; vir[2] += rz * 0.5 * cz;
            vir[3] += rx * 0.5 * cy; vir[4] += rx * 0.5 * cz; vir[5] += ry * 0.5 * cz;
          }
        }
      }
    }
    // ---- bonded terms (per-term forces gathered per atom)
    if (s.n_bonds + s.n_angles + s.n_dihedrals > 0) {
      for (int k = s.aterm_off[i]; k < s.aterm_off[i + 1]; ++k) {
        const double4 tf = s.term_force[s.aterm[k]];
        F[0] += tf.x;
        F[1] += tf.y;
        F[2] += tf.z;
      }
    }
    s.f[i] = make_double4(F[0], F[1], F[2], 0.0);
    if (!(isfinite(F[0]) && isfinite(F[1]) && isfinite(F[2]))) atomicOr(&st->status, kErrNonFinite);
  }
  // ---- half kick and kinetic energy
  double ke = 0.0;
  if (act && mode != kFinalForceOnly) {
    double4 v = s.v[i];
    if (mode == kFinalKick) {
      if (s.has_triples) s.vold2[i] = v;
      const double m = v.w, dt = s.dt, c = s.fmt2v;
      v.x += 0.5 * F[0] / m * dt * c;
      v.y += 0.5 * F[1] / m * dt * c;
      v.z += 0.5 * F[2] / m * dt * c;
      if (s.npt == 2)  // FinalIntegrate: NH_V_Press after the kick (ExecutionNPT.cpp:1713-1720)
        for (int r = 0; r < 2; ++r) {
          v.x = st->f_press[0] * v.x;
          v.y = st->f_press[1] * v.y;
          v.z = st->f_press[2] * v.z;
        }
      s.v[i] = v;
    }
    ke = (v.w * (v.x * v.x + v.y * v.y + v.z * v.z)) * s.mvv2e;
  }
  // ---- block partials and the system epilogue
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double r8[8];
  r8[0] = warp_sum(ke);
#pragma unroll
  for (int k = 0; k < 6; ++k) r8[1 + k] = VIRIAL ? warp_sum(vir[k]) : 0.0;
  r8[7] = 0.0;
  if (lane == 0)
    for (int k = 0; k < 8; ++k) s_part[wid][k] = r8[k];
  __syncthreads();
  const int blk = wk.y / kAtomBlock;
  if (threadIdx.x < 8) {
    double t = 0.0;
    for (int w = 0; w < kAtomBlock / 32; ++w) t += s_part[w][threadIdx.x];
    s.atom_part[(size_t)blk * 8 + threadIdx.x] = t;
  }
  if (arrive_last(&st->counter[2], (unsigned)s.blocks_atom)) {
    __shared__ double s_tot[8];
    if (threadIdx.x < 8) {
      double t = 0.0;
      for (int b = 0; b < s.blocks_atom; ++b) t += __ldcg(&s.atom_part[(size_t)b * 8 + threadIdx.x]);
      s_tot[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (VIRIAL) {
        double tv[6] = {0, 0, 0, 0, 0, 0};
        if (s.term_vir)
          for (int t = 0; t < s.n_bonds + s.n_angles + s.n_dihedrals; ++t)
            for (int k = 0; k < 6; ++k) tv[k] += s.term_vir[6 * (size_t)t + k];
        for (int k = 0; k < 6; ++k) st->virial[k] = st->virial[k] + s_tot[1 + k] + tv[k];
      }
      if (mode == kFinalInit) {
        // ExecutionNVT::InitialCondition + SetUp (ExecutionNVT.cpp:139-187, 1106-1122)
        compute_tempe(s, st, s_tot[0]);
        compute_temp_target(s, st);
        const double tf = st->t_freq;
        st->eta_mass[0] = st->tdof * s.boltz * st->t_target / (tf * tf);
        for (int ich = 1; ich < 3; ich++) st->eta_mass[ich] = s.boltz * st->t_target / (tf * tf);
        for (int ich = 1; ich < 3; ich++)
          st->eta_dotdot[ich] = (st->eta_mass[ich - 1] * st->eta_dot[ich - 1] * st->eta_dot[ich - 1] -
                                 s.boltz * st->t_target) / st->eta_mass[ich];
        if (s.npt == 2) mtk_setup(s, st);
      } else if (mode == kFinalKick) {
        const bool shk_thermo = s.has_triples && s.temp_ctrl != RBMD_TC_NOSE_HOOVER;
        if (!shk_thermo) {
          compute_tempe(s, st, s_tot[0]);
          if (s.temp_ctrl == RBMD_TC_NOSE_HOOVER) {
            if (s.npt == 2) {
              // FinalIntegrate: pressure of this step's forces, barostat velocity half step
              double vir[6];
              st->p_current = pressure_scalar(s, st, vir);
              st->baro_pressure = st->p_current;
              for (int k = 0; k < 6; ++k) st->baro_virial[k] = vir[k];
              omega_dot_half(s, st);
            }
            const double fb = nhc_half(s, st);
            if (s.npt == 2) nhc_press_half(s, st);
            st->vscale_pending = fb;
            st->vscale_pending_c = s.has_triples ? 1.0 : fb;  // RATTLE rebuilds triples from pre-kick v
          } else if (s.temp_ctrl == RBMD_TC_RESCALE) {
            const double c = sqrt(s.t_start / st->temperature);
            st->vscale_pending = st->vscale_pending_c = c;
          } else if (s.temp_ctrl == RBMD_TC_BERENDSEN) {
            const double c = sqrt(1.0 + s.dt / s.t_damp * (s.t_start / st->temperature - 1.0));
            st->vscale_pending = st->vscale_pending_c = c;
          }
        }
      }
    }
  }
}

// Kinetic energy after RATTLE for the rescaling thermostats (the reference computes the
// temperature after ConstraintB there, ExecutionNVT.cpp:92-115).
__global__ void __launch_bounds__(kAtomBlock) k_ke_thermostat(const SysDev* __restrict__ S,
                                                              const int2* __restrict__ work) {
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int i = wk.y + threadIdx.x;
  SysState* st = s.st;
  double ke = 0.0;
  if (i < s.n) {
    const double4 v = s.v[i];
    ke = (v.w * (v.x * v.x + v.y * v.y + v.z * v.z)) * s.mvv2e;
  }
  __shared__ double s_w[kAtomBlock / 32];
  const double w = warp_sum(ke);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = w;
  __syncthreads();
  const int blk = wk.y / kAtomBlock;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kAtomBlock / 32; ++k) t += s_w[k];
    s.atom_part[(size_t)blk * 8] = t;
  }
  if (arrive_last(&st->counter[5], (unsigned)s.blocks_atom)) {
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int b = 0; b < s.blocks_atom; ++b) t += __ldcg(&s.atom_part[(size_t)b * 8]);
      compute_tempe(s, st, t);
      double c = 1.0;
      if (s.temp_ctrl == RBMD_TC_RESCALE) c = sqrt(s.t_start / st->temperature);
      else if (s.temp_ctrl == RBMD_TC_BERENDSEN)
        c = sqrt(1.0 + s.dt / s.t_damp * (s.t_start / st->temperature - 1.0));
      st->vscale_pending = st->vscale_pending_c = c;
    }
  }
}

// ------------------------------------------------------------------ SHAKE / RATTLE
__device__ inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// One thread per triple.  The kernel waits on memory, not on arithmetic, so every load it needs
// (old state, charge, image counters, cell rank) is issued up front, in one round, and only the
// values the update needs after the multiplier iteration are kept (the unconstrained position and
// the half-kicked velocity, formed as the update forms them); the arithmetic and its order are the
// reference's.
__global__ void __launch_bounds__(128, 3) k_shake(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  // NewConstraintAWaterBondAngleWorklet, framework/run/worklet/MolecularWorklet.h:2367-2645
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int a = wk.y + threadIdx.x;
  SysState* st = s.st;
  double sv[6] = {0, 0, 0, 0, 0, 0};
  if (a < s.n_triples) {
    const int id[3] = {s.angle_atoms[3 * a], s.angle_atoms[3 * a + 1], s.angle_atoms[3 * a + 2]};
    const double dt = s.dt, fm = s.fmt2v;
    // every load of the triple in one round
    double4 xo[3], vo[3], fo4[3];
    double qa[3];
    int img[3][3], rk[3];
    for (int t = 0; t < 3; ++t) {
      xo[t] = s.xold[id[t]];
      vo[t] = s.vold[id[t]];
      fo4[t] = s.f[id[t]];
      qa[t] = s.x[id[t]].w;
      rk[t] = s.rank[id[t]];
      for (int k = 0; k < 3; ++k) img[t][k] = s.image[3 * id[t] + k];
    }
    // old position, velocity, force and mass of atom t, and its unconstrained update
    auto load = [&](int t, double* ox, double* ov, double* fo, double& m, double* sp) {
      const double4 x = xo[t], v = vo[t], f = fo4[t];
      ox[0] = x.x; ox[1] = x.y; ox[2] = x.z;
      ov[0] = v.x; ov[1] = v.y; ov[2] = v.z;
      fo[0] = f.x; fo[1] = f.y; fo[2] = f.z;
      m = v.w;
      for (int k = 0; k < 3; ++k) sp[k] = ox[k] + ov[k] * dt + 0.5 * dt * dt * fo[k] / m * fm;
    };
    const double bond1 = 1.0, bond2 = 1.0;
    const double bond12 = sqrt(bond1 * bond1 + bond2 * bond2 - 2.0 * bond1 * bond2 * cos((109.4700 / 180.0) * kPif));
    auto mdv = [&](const double* p, const double* q, double* o) {
      o[0] = p[0] - q[0]; o[1] = p[1] - q[1]; o[2] = p[2] - q[2];
      min_image(o[0], o[1], o[2], s.L[0], s.L[1], s.L[2]);
    };
    double ms[3], r01[3], r12[3], r20[3], spk[3][3], vh[3][3];
    double a11i, a12i, a13i, a21i, a22i, a23i, a31i, a32i, a33i, s01sq, s02sq, s12sq;
    double q1_0101, q1_1212, q1_2020, q1_0120, q1_0112, q1_2012;
    double q2_0101, q2_1212, q2_2020, q2_0120, q2_0112, q2_2012;
    double q3_0101, q3_1212, q3_2020, q3_0120, q3_0112, q3_2012;
    int err = 0;
    {
      double ox[3][3], ov[3][3], fo[3][3], sp[3][3];
      for (int t = 0; t < 3; ++t) {
        load(t, ox[t], ov[t], fo[t], ms[t], sp[t]);
        for (int k = 0; k < 3; ++k) {
          spk[t][k] = sp[t][k];
          vh[t][k] = ov[t][k] + 0.5 * dt * fo[t][k] / ms[t] * fm;  // the update's velocity before the correction
        }
      }
      double s10[3], s21[3], s02[3];
      mdv(ox[1], ox[0], r01);
      mdv(ox[2], ox[1], r12);
      mdv(ox[0], ox[2], r20);
      mdv(sp[0], sp[1], s10);
      mdv(sp[1], sp[2], s21);
      mdv(sp[2], sp[0], s02);
      const double r01sq = dot3(r01, r01), r02sq = dot3(r20, r20), r12sq = dot3(r12, r12);
      s01sq = dot3(s10, s10);
      s02sq = dot3(s02, s02);
      s12sq = dot3(s21, s21);
      const double im0 = 1.0 / ms[0], im1 = 1.0 / ms[1], im2 = 1.0 / ms[2];
      const double a11 = 2.0 * (im0 + im1) * dot3(s10, r01), a12 = -2.0 * im1 * dot3(s10, r12),
                   a13 = -2.0 * im0 * dot3(s10, r20), a21 = -2.0 * im1 * dot3(s21, r01),
                   a22 = 2.0 * (im1 + im2) * dot3(s21, r12), a23 = -2.0 * im2 * dot3(s21, r20),
                   a31 = -2.0 * im0 * dot3(s02, r01), a32 = -2.0 * im2 * dot3(s02, r12),
                   a33 = 2.0 * (im0 + im2) * (dot3(s02, r20));
      const double determ = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a11 * a23 * a32 -
                            a12 * a21 * a33 - a13 * a22 * a31;
      if (fabs(determ) < 0.0001) err |= kErrShakeSingular;
      const double di = 1.0 / determ;
      a11i = di * (a22 * a33 - a23 * a32);
      a12i = -di * (a12 * a33 - a13 * a32);
      a13i = di * (a12 * a23 - a13 * a22);
      a21i = -di * (a21 * a33 - a23 * a31);
      a22i = di * (a11 * a33 - a13 * a31);
      a23i = -di * (a11 * a23 - a13 * a21);
      a31i = di * (a21 * a32 - a22 * a31);
      a32i = -di * (a11 * a32 - a12 * a31);
      a33i = di * (a11 * a22 - a12 * a21);
      const double r0120 = dot3(r01, r20), r0112 = dot3(r01, r12), r2012 = dot3(r20, r12);
      q1_0101 = (im0 + im1) * (im0 + im1) * r01sq;
      q1_1212 = im1 * im1 * r12sq;
      q1_2020 = im0 * im0 * r02sq;
      q1_0120 = -2.0 * (im0 + im1) * im0 * r0120;
      q1_0112 = -2.0 * (im0 + im1) * im1 * r0112;
      q1_2012 = 2.0 * im0 * im1 * r2012;
      q2_0101 = im1 * im1 * r01sq;
      q2_1212 = (im1 + im2) * (im1 + im2) * r12sq;
      q2_2020 = im2 * im2 * r02sq;
      q2_0120 = 2.0 * im1 * im2 * r0120;
      q2_0112 = -2.0 * (im1 + im2) * im1 * r0112;
      q2_2012 = -2.0 * (im1 + im2) * im2 * r2012;
      q3_0101 = im0 * im0 * r01sq;
      q3_1212 = im2 * im2 * r12sq;
      q3_2020 = (im0 + im2) * (im0 + im2) * r02sq;
      q3_0120 = -2.0 * (im0 + im2) * im0 * r0120;
      q3_0112 = 2.0 * im0 * im2 * r0112;
      q3_2012 = -2.0 * (im0 + im2) * im2 * r2012;
    }
    double l01 = 0.0, l20 = 0.0, l12 = 0.0;
    int niter = 0, done = 0;
    while (!done && niter < 5000) {  // bounded like the reference (max_iter 5000)
      const double quad1 = q1_0101 * l01 * l01 + q1_2020 * l20 * l20 + q1_1212 * l12 * l12 +
                           q1_0120 * l01 * l20 + q1_0112 * l01 * l12 + q1_2012 * l20 * l12;
      const double quad2 = q2_0101 * l01 * l01 + q2_2020 * l20 * l20 + q2_1212 * l12 * l12 +
                           q2_0120 * l01 * l20 + q2_0112 * l01 * l12 + q2_2012 * l20 * l12;
      const double quad3 = q3_0101 * l01 * l01 + q3_2020 * l20 * l20 + q3_1212 * l12 * l12 +
                           q3_0120 * l01 * l20 + q3_0112 * l01 * l12 + q3_2012 * l20 * l12;
      const double b1 = bond1 * bond1 - s01sq - quad1;
      const double b2 = bond2 * bond2 - s12sq - quad2;
      const double b3 = bond12 * bond12 - s02sq - quad3;
      const double l01n = a11i * b1 + a12i * b2 + a13i * b3;
      const double l12n = a21i * b1 + a22i * b2 + a23i * b3;
      const double l20n = a31i * b1 + a32i * b2 + a33i * b3;
      done = 1;
      if (fabs(l01n - l01) > 0.00001) done = 0;
      if (fabs(l20n - l20) > 0.00001) done = 0;
      if (fabs(l12n - l12) > 0.00001) done = 0;
      l01 = l01n;
      l20 = l20n;
      l12 = l12n;
      if (isnan(l01) || isnan(l20) || isnan(l12) || fabs(l01) > 1e20 || fabs(l20) > 1e20 || fabs(l12) > 1e20) {
        done = 1;
        err |= kErrShakeOverflow;
      }
      niter++;
    }
    if (!done) err |= kErrShakeNoConverge;
    const double im0 = 1.0 / ms[0], im1 = 1.0 / ms[1], im2 = 1.0 / ms[2];
    double pc[3][3];
    for (int k = 0; k < 3; ++k) {
      pc[0][k] = l01 * r01[k] * im0 - l20 * r20[k] * im0;
      pc[1][k] = l12 * r12[k] * im1 - l01 * r01[k] * im1;
      pc[2][k] = l20 * r20[k] * im2 - l12 * r12[k] * im2;
    }
    float disp_max = 0.0f;  // largest displacement of the triple's atoms since the cell list
    for (int t = 0; t < 3; ++t) {
      const int ii = id[t];
      const double m = ms[t];
      double nv[3], nx[3];
      const double4 xb = s.x[ii];  // the position the cell list was built from
      double disp2 = 0.0;
      bool crossed = false;  // wrapped across the box relative to that position
      for (int k = 0; k < 3; ++k) {
        nv[k] = vh[t][k] + pc[t][k] / dt;
        double xx = spk[t][k] + pc[t][k];
        int im = img[t][k];
        if (xx < s.lo[k]) {
          xx += (s.hi[k] - s.lo[k]);
          im -= 1;
        }
        if (xx > s.hi[k]) {
          xx -= (s.hi[k] - s.lo[k]);
          im += 1;
        }
        nx[k] = xx;
        s.image[3 * ii + k] = im;
        const double L = s.hi[k] - s.lo[k], dk = xx - (&xb.x)[k];
        const double dm = fabs(dk) > 0.5 * L ? fabs(dk) - L : dk;  // nearest image
        crossed |= fabs(dk) > 0.5 * L;
        disp2 += dm * dm;
      }
      disp_max = fmaxf(disp_max, (float)(sqrt(disp2) * (1.0 + 1e-6)));
      if (crossed) {
        const int slot = atomicAdd(&s.st->mig_n, 1);
        if (slot < kMaxMigrated) s.st->mig_cell[slot] = s.cell_of_atom[ii];
      }
      s.v[ii] = make_double4(nv[0], nv[1], nv[2], m);
      const double q = qa[t];
      s.x[ii] = make_double4(nx[0], nx[1], nx[2], q);
      // the cell list was built before the constraint (as the reference's locator is); refresh
      // the cell-ordered copies the pair kernel streams
      const int k = rk[t];
      s.sx[k] = make_double4(nx[0], nx[1], nx[2], q);
      s.sxf[k] = make_float4((float)nx[0], (float)nx[1], (float)nx[2], (float)q);
    }
    {  // one atomic per converged group of lanes (a block's triples belong to one system)
      const unsigned am = __activemask();
      const unsigned mx = __reduce_max_sync(am, __float_as_uint(disp_max));  // non-negative: bits order as values
      if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1)) atomicMax(&s.st->shake_disp_bits, mx);
    }
    const double dtfsq = 0.5 * dt * dt * fm;
    l01 = l01 / dtfsq;
    l20 = l20 / dtfsq;
    l12 = l12 / dtfsq;
    sv[0] = l01 * r01[0] * r01[0] + l20 * r20[0] * r20[0] + l12 * r12[0] * r12[0];
    sv[1] = l01 * r01[1] * r01[1] + l20 * r20[1] * r20[1] + l12 * r12[1] * r12[1];
    sv[2] = l01 * r01[2] * r01[2] + l20 * r20[2] * r20[2] + l12 * r12[2] * r12[2];
    sv[3] = l01 * r01[0] * r01[1] + l20 * r20[0] * r20[1] + l12 * r12[0] * r12[1];
    sv[4] = l01 * r01[0] * r01[2] + l20 * r20[0] * r20[2] + l12 * r12[0] * r12[2];
    sv[5] = l01 * r01[1] * r01[2] + l20 * r20[1] * r20[2] + l12 * r12[1] * r12[2];
    if (err) atomicOr(&st->status, err);
  }
  // SHAKE virial partials (used by the pressure)
  __shared__ double s_w[4][6];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < 6; ++k) {
    const double w = warp_sum(sv[k]);
    if (lane == 0) s_w[wid][k] = w;
  }
  __syncthreads();
  const int blk = wk.y / 128;
  if (threadIdx.x < 6) {
    double t = 0;
    for (int w = 0; w < 4; ++w) t += s_w[w][threadIdx.x];
    s.tri_part[(size_t)blk * 6 + threadIdx.x] = t;
  }
  if (arrive_last(&st->counter[3], (unsigned)s.blocks_tri)) {
    if (threadIdx.x < 6) {
      double t = 0;
      for (int b = 0; b < s.blocks_tri; ++b) t += __ldcg(&s.tri_part[(size_t)b * 6 + threadIdx.x]);
      st->shake_virial[threadIdx.x] = t;
    }
  }
}

__global__ void k_rattle(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  // NewConstraintBWaterBondAngleWorklet, framework/run/worklet/MolecularWorklet.h:2647-2832
  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int a = wk.y + threadIdx.x;
  if (a >= s.n_triples) return;
  const int id[3] = {s.angle_atoms[3 * a], s.angle_atoms[3 * a + 1], s.angle_atoms[3 * a + 2]};
  const double dt = s.dt, fm = s.fmt2v;
  double xs[3][3], sv[3][3], ms[3];
  for (int t = 0; t < 3; ++t) {
    const double4 x = s.x[id[t]], v = s.vold2[id[t]], f = s.f[id[t]];
    xs[t][0] = x.x; xs[t][1] = x.y; xs[t][2] = x.z;
    ms[t] = v.w;
    sv[t][0] = v.x + 0.5 * dt * f.x / v.w * fm;
    sv[t][1] = v.y + 0.5 * dt * f.y / v.w * fm;
    sv[t][2] = v.z + 0.5 * dt * f.z / v.w * fm;
  }
  auto mdv = [&](const double* p, const double* q, double* o) {
    o[0] = p[0] - q[0]; o[1] = p[1] - q[1]; o[2] = p[2] - q[2];
    min_image(o[0], o[1], o[2], s.L[0], s.L[1], s.L[2]);
  };
  double r01[3], r12[3], r20[3];
  mdv(xs[1], xs[0], r01);
  mdv(xs[2], xs[1], r12);
  mdv(xs[0], xs[2], r20);
  double sv10[3], sv21[3], sv02[3];
  for (int k = 0; k < 3; ++k) {
    sv10[k] = sv[0][k] - sv[1][k];
    sv21[k] = sv[1][k] - sv[2][k];
    sv02[k] = sv[2][k] - sv[0][k];
  }
  const double im0 = 1.0 / ms[0], im1 = 1.0 / ms[1], im2 = 1.0 / ms[2];
  double A[3][3];
  A[0][0] = (im1 + im0) * dot3(r01, r01);
  A[0][1] = -im1 * dot3(r01, r12);
  A[0][2] = (-im0) * dot3(r01, r20);
  A[1][0] = A[0][1];
  A[1][1] = (im1 + im2) * dot3(r12, r12);
  A[1][2] = -(im2)*dot3(r20, r12);
  A[2][0] = A[0][2];
  A[2][1] = A[1][2];
  A[2][2] = (im0 + im2) * dot3(r20, r20);
  const double c[3] = {-dot3(sv10, r01), -dot3(sv21, r12), -dot3(sv02, r20)};
  const double determ = A[0][0] * A[1][1] * A[2][2] + A[0][1] * A[1][2] * A[2][0] +
                        A[0][2] * A[1][0] * A[2][1] - A[0][0] * A[1][2] * A[2][1] -
                        A[0][1] * A[1][0] * A[2][2] - A[0][2] * A[1][1] * A[2][0];
  if (fabs(determ) < 0.0001) atomicOr(&s.st->status, kErrRattleSingular);
  const double di = 1.0 / determ;
  double ai[3][3];
  ai[0][0] = di * (A[1][1] * A[2][2] - A[1][2] * A[2][1]);
  ai[0][1] = -di * (A[0][1] * A[2][2] - A[0][2] * A[2][1]);
  ai[0][2] = di * (A[0][1] * A[1][2] - A[0][2] * A[1][1]);
  ai[1][0] = -di * (A[1][0] * A[2][2] - A[1][2] * A[2][0]);
  ai[1][1] = di * (A[0][0] * A[2][2] - A[0][2] * A[2][0]);
  ai[1][2] = -di * (A[0][0] * A[1][2] - A[0][2] * A[1][0]);
  ai[2][0] = di * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  ai[2][1] = -di * (A[0][0] * A[2][1] - A[0][1] * A[2][0]);
  ai[2][2] = di * (A[0][0] * A[1][1] - A[0][1] * A[1][0]);
  double l[3];
  for (int ii = 0; ii < 3; ii++) {
    l[ii] = 0;
    for (int jj = 0; jj < 3; jj++) l[ii] += ai[ii][jj] * c[jj];
  }
  double nv[3][3];
  for (int k = 0; k < 3; ++k) {
    nv[0][k] = sv[0][k] + (l[0] * r01[k] * im0 - l[2] * r20[k] * im0);
    nv[1][k] = sv[1][k] + (l[1] * r12[k] * im1 - l[0] * r01[k] * im1);
    nv[2][k] = sv[2][k] + (l[2] * r20[k] * im2 - l[1] * r12[k] * im2);
  }
  for (int t = 0; t < 3; ++t) s.v[id[t]] = make_double4(nv[t][0], nv[t][1], nv[t][2], ms[t]);
}

// ------------------------------------------------------------------ launchers
void launch_nhc_a(const Batch& b, cudaStream_t st) {
  k_nhc_a<<<(b.nsys + 127) / 128, 128, 0, st>>>(b.sys, b.d_slots, b.nsys);
  note_launch();
}

void launch_kick_drift(const Batch& b, cudaStream_t st) {
  k_kick_drift<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  note_launch();
}

void launch_flush_vscale(const Batch& b, cudaStream_t st) {
  k_flush_vscale<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  note_launch();
}

void launch_bonded(const Batch& b, cudaStream_t st, int virial) {
  if (!b.has_bonded) return;
  k_bonded<<<b.term.n, 128, 0, st>>>(b.sys, b.term.d, virial);
  note_launch();
}

void launch_final(const Batch& b, cudaStream_t st, FinalMode mode, int virial) {
  if (virial) {
    k_final<false, true><<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d, (int)mode);
  } else if (b.prec == RBMD_PREC_MIXED && b.coul == RBMD_COUL_RBE) {
    k_final<true, false><<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d, (int)mode);
  } else {
    k_final<false, false><<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d, (int)mode);
  }
  note_launch();
}

void launch_ke_thermostat(const Batch& b, cudaStream_t st) {
  k_ke_thermostat<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  note_launch();
}

void launch_shake(const Batch& b, cudaStream_t st) {
  if (!b.has_shake) return;
  k_shake<<<b.tri.n, 128, 0, st>>>(b.sys, b.tri.d);
  note_launch();
}

void launch_rattle(const Batch& b, cudaStream_t st) {
  if (!b.has_shake) return;
  k_rattle<<<b.tri.n, 128, 0, st>>>(b.sys, b.tri.d);
  note_launch();
}

}  // namespace rbmd
