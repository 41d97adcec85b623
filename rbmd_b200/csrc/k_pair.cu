// k_pair.cu -- fused cell traversal + random-batch-list selection + short-range pair forces.
//
// Replaces, in one kernel per force evaluation and without materialising any list:
//   ComputeRBLNeighboursOnceWorklet   framework/run/worklet/RunWorklet.cpp:906-980   (list build)
//   ComputeLJForceRBLWorklet           RunWorklet.cpp:1817-1909                       (LJ/CUT, RBL)
//   ComputeNearForceRBLERF[SpecialBonds]Worklet RunWorklet.cpp:982-1266              (LJ + erfc)
//   ComputeNeighboursWorklet + *VerletWorklet   RunWorklet.cpp:296-355, 498-575, 2767-2985
//   ComputeEAMfp_Worklet / ComputeEAMRBLWorklet  RunWorklet.cpp:1651-1815             (EAM passes)
//   LJ / Coulomb / EAM energy worklets           RunWorklet.cpp:2987-3221, ThermoOutput.cpp:293-356
//
// One warp per atom i, atoms taken in cell order so the warps of a block walk overlapping cells.
// The (2 nc + 1)^3 neighbour cells are visited in the reference order (x offset outermost,
// z innermost, ascending atom id inside a cell): 32 cells at a time, one per lane, their atom
// counts prefix-summed so each lane then takes one candidate of the flattened sequence.  The
// shell rank of every candidate is its warp-ballot prefix plus the running shell count, which
// reproduces the reference's sequential "every pice-th shell atom" pick exactly.  Selected pairs
// are compacted through a per-warp shared-memory queue and evaluated 32 at a time, so the force
// arithmetic runs with full warps.  FP64 classification uses explicitly rounded products and
// sums so that it makes the same decisions as the CPU oracle on the same positions.
#include "kernels.h"

namespace rbmd {

enum PairMode {
  kLJ_RBL = 0, kCOUL_RBL = 1, kLJ_VERLET = 2, kCOUL_VERLET = 3,
  kEAM_RHO = 4, kEAM_FORCE = 5, kENERGY = 6, kEAM_ENERGY = 7, kLIST = 8
};

template <typename R> struct Vec4;
template <> struct Vec4<double> { using T = double4; };
template <> struct Vec4<float> { using T = float4; };

__device__ inline double4 ldg4(const double4* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

template <typename R> __device__ inline typename Vec4<R>::T load_sorted(const SysDev& s, int k);
template <> __device__ inline double4 load_sorted<double>(const SysDev& s, int k) { return ldg4(&s.sx[k]); }
template <> __device__ inline float4 load_sorted<float>(const SysDev& s, int k) { return __ldg(&s.sxf[k]); }

__device__ inline double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ inline float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ inline float add_rn(float a, float b) { return __fadd_rn(a, b); }

__device__ inline double r_sqrt(double x) { return sqrt(x); }
__device__ inline float r_sqrt(float x) { return sqrtf(x); }
__device__ inline double r_exp(double x) { return exp(x); }
__device__ inline float r_exp(float x) { return __expf(x); }
__device__ inline double r_erfc(double x) { return erfc(x); }
__device__ inline float r_erfc(float x) { return erfcf(x); }

// EAM spline row evaluation (ExecForceFunction::ComputeEAMrho / ComputeEAMforce)
__device__ inline void eam_row(const double* tab, double r, double rdr, int nr, int& m, double& p) {
  p = r * rdr + 1.0;
  m = (int)p;
  m = min(m, nr - 1);
  p -= m;
  p = fmin(p, 1.0);
}

struct PairAcc {
  double f[3];
  double g[3];    // Coulomb part before qqr2e (RBL Coulomb modes)
  double rho;     // EAM density / energy scalar
  double e0, e1;  // energies
  double vir[6];
};

template <typename R, int MODE, bool SPECIAL, bool VIRIAL>
__device__ inline void eval_pair(const SysDev& s, int i, int ti, int moli, double qi, double fpi,
                                 int js, bool core, R rx, R ry, R rz, const int* spi, const double* spw,
                                 int nsp, R pice, PairAcc& a) {
  const int4 mj = __ldg(&s.smeta[js]);  // atom id, type, molecule
  const R Lx = (R)s.L[0], Ly = (R)s.L[1], Lz = (R)s.L[2];
  if (MODE == kEAM_RHO || MODE == kEAM_FORCE || MODE == kEAM_ENERGY) {
    rx = -rx; ry = -ry; rz = -rz;  // MinDistanceVec(p_i, p_j)
  }
  min_image(rx, ry, rz, Lx, Ly, Lz);
  const R d2 = rx * rx + ry * ry + rz * rz;
  const R rc2 = (R)s.rc2, rs2 = (R)s.rs2;

  if (MODE == kEAM_RHO || MODE == kEAM_FORCE || MODE == kEAM_ENERGY) {
    const double rsq = (double)d2;
    const double cut = (MODE == kEAM_ENERGY) ? s.eam_cut : s.rc;
    bool ok = core ? (rsq < cut * cut && rsq > 0.01) : (rsq < s.rc * s.rc && rsq > s.rs2);
    if (!ok) return;
    const double rr = sqrt(rsq);
    int m;
    double p;
    eam_row(s.rhor_s, rr, 1.0 / s.eam_dr, s.eam_nr, m, p);
    const double scale = core ? 1.0 : (double)pice;
    if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) {
      const double* c = s.rhor_s + 7 * m;
      a.rho += scale * (((__ldg(c + 3) * p + __ldg(c + 4)) * p + __ldg(c + 5)) * p + __ldg(c + 6));
      if (MODE == kEAM_ENERGY) {
        const double* z = s.z2r_s + 7 * m;
        double z2 = ((__ldg(z + 3) * p + __ldg(z + 4)) * p + __ldg(z + 5)) * p + __ldg(z + 6);
        a.e1 += 0.5 * (z2 * (1.0 / rr));
      }
    } else {
      const double* ci = s.rhor_s + 7 * m;
      const double rhoip = (__ldg(ci) * p + __ldg(ci + 1)) * p + __ldg(ci + 2);
      const double* cz = s.z2r_s + 7 * m;
      const double z2p = (__ldg(cz) * p + __ldg(cz + 1)) * p + __ldg(cz + 2);
      const double z2 = ((__ldg(cz + 3) * p + __ldg(cz + 4)) * p + __ldg(cz + 5)) * p + __ldg(cz + 6);
      const double recip = 1.0 / rr;
      const double phi = z2 * recip;
      const double phip = z2p * recip - phi * recip;
      const double psip = fpi * rhoip + __ldg(&s.eam_fp[mj.x]) * rhoip + phip;
      const double fpair = -psip * recip;
      a.f[0] += scale * ((double)rx * fpair);
      a.f[1] += scale * ((double)ry * fpair);
      a.f[2] += scale * ((double)rz * fpair);
    }
    return;
  }

  if (MODE == kLJ_RBL && moli == mj.z) return;  // same-molecule skip, RunWorklet.cpp:1874-1876
  const int tj = mj.y;
  const R eps_i = (R)__ldg(&s.eps[ti]), eps_j = (R)__ldg(&s.eps[tj]);
  const R sig_ij = ((R)__ldg(&s.sig[ti]) + (R)__ldg(&s.sig[tj])) / R(2);
  R w = R(1);
  if (SPECIAL) {
    for (int k = 0; k < nsp; ++k)
      if (spi[k] == mj.x) w = (R)spw[k];
  }
  const R s6 = sig_ij * sig_ij * sig_ij * sig_ij * sig_ij * sig_ij;
  auto lj = [&](R cut2lo, R cut2hi) -> R {  // force / r_vector factor (0 outside the window)
    if (d2 < cut2hi && d2 > cut2lo) {
      const R dis6 = d2 * d2 * d2;
      const R sd6 = s6 / dis6;
      return R(-24) * r_sqrt(eps_i * eps_j) * ((R(2) * sd6 - R(1)) * sd6) / d2;
    }
    return R(0);
  };

  if (MODE == kLJ_RBL) {
    const R fs = core ? lj(R(0.0001), rc2) : pice * lj(rs2, rc2);
    a.f[0] += (double)(fs * rx);
    a.f[1] += (double)(fs * ry);
    a.f[2] += (double)(fs * rz);
    return;
  }
  if (MODE == kLIST) return;

  const R qj = (R)__ldg(reinterpret_cast<const double*>(&s.sx[js]) + 3);
  const R alpha = (R)s.alpha;
  if (MODE == kCOUL_RBL) {
    const R fl = core ? w * lj(R(0.0001), rs2) : w * (pice * lj(rs2, rc2));
    a.f[0] += (double)(fl * rx);
    a.f[1] += (double)(fl * ry);
    a.f[2] += (double)(fl * rz);
    const bool in = core ? (d2 < rc2 && d2 > R(0.0001))
                         : (SPECIAL ? (d2 < rc2 && d2 > rs2) : (d2 < rc2 && d2 > R(0.0001)));
    if (in) {
      const R dis = r_sqrt(d2);
      const R sa = r_sqrt(alpha);
      const R g = r_erfc(sa * dis) / d2 + R(2) * sa * r_exp(-alpha * d2) / ((R)sqrt(kPif) * dis);
      R fc = -(R)qi * qj * g / dis;
      if (!core) fc *= pice;
      a.g[0] += (double)(fc * rx);
      a.g[1] += (double)(fc * ry);
      a.g[2] += (double)(fc * rz);
    }
    return;
  }

  // full-list modes
  const R flj = lj(R(0.0001), rc2);
  if (MODE == kLJ_VERLET) {
    a.f[0] += (double)(flj * rx);
    a.f[1] += (double)(flj * ry);
    a.f[2] += (double)(flj * rz);
    if (VIRIAL) {
      const double h[3] = {0.5 * (double)(flj * rx), 0.5 * (double)(flj * ry), 0.5 * (double)(flj * rz)};
      a.vir[0] += (double)rx * h[0]; a.vir[1] += (double)ry * h[1]; a.vir[2] += (double)rz * h[2];
      a.vir[3] += (double)rx * h[1]; a.vir[4] += (double)rx * h[2]; a.vir[5] += (double)ry * h[2];
    }
    return;
  }
  R fcs = R(0), fbs = R(0);
  R dis = r_sqrt(d2);
  if (d2 < rc2 && d2 > R(0.0001)) {
    const R sa = r_sqrt(alpha);
    const R g = r_erfc(sa * dis) / d2 + R(2) * sa * r_exp(-alpha * d2) / ((R)sqrt(kPif) * dis);
    fcs = -(R)qi * qj * g / dis;
    fbs = -(R)qi * qj / (dis * dis * dis);
  }
  if (MODE == kCOUL_VERLET) {
    const R qq = (R)s.qqr2e;
    const R fp = SPECIAL ? qq * (fcs - (R(1) - w) * fbs) + w * flj : qq * fcs + flj;
    a.f[0] += (double)(fp * rx);
    a.f[1] += (double)(fp * ry);
    a.f[2] += (double)(fp * rz);
    if (VIRIAL) {
      const double sc = SPECIAL ? -0.5 : 0.5;  // ComputePairVirial vs ComputePairVirial_fix
      const double h[3] = {sc * (double)(fp * rx), sc * (double)(fp * ry), sc * (double)(fp * rz)};
      a.vir[0] += (double)rx * h[0]; a.vir[1] += (double)ry * h[1]; a.vir[2] += (double)rz * h[2];
      a.vir[3] += (double)rx * h[1]; a.vir[4] += (double)rx * h[2]; a.vir[5] += (double)ry * h[2];
    }
    return;
  }
  if (MODE == kENERGY) {
    // ComputePotentialEn_fix / ComputeNearEleEnergy_fix / ComputeCoulFactor_fix (FP64 always)
    const double dd2 = (double)d2;
    if (dd2 < s.rc2 && dd2 > 0.0001) {
      const double sg = ((double)s.sig[ti] + (double)s.sig[tj]) / 2;
      const double s6d = sg * sg * sg * sg * sg * sg;
      const double dis6 = dd2 * dd2 * dd2;
      const double eij = sqrt((double)s.eps[ti] * (double)s.eps[tj]);
      const double el = 0.5 * (4 * eij * (s6d / dis6 - 1) * (s6d / dis6));
      a.e0 += (double)w * el;
      if (s.ff != RBMD_FF_LJ_CUT) {
        const double dd = sqrt(dd2);
        const double ec = 0.5 * qi * (double)qj * erfc(sqrt(s.alpha) * dd) / dd;
        const double ef = 0.5 * qi * (double)qj / dd;
        a.e1 += s.qqr2e * (ec - (SPECIAL ? (1.0 - (double)w) * ef : 0.0));
      }
    }
  }
}

template <typename R, int MODE, bool SPECIAL, bool VIRIAL>
__global__ void __launch_bounds__(kPairWarps * 32)
k_pair(const SysDev* __restrict__ S, const int2* __restrict__ work, int cap, int* out_nc,
       int* out_ns, int* out_core, int* out_shell) {
  __shared__ int s_qj[kPairWarps][kQueue];
  __shared__ R s_qr[kPairWarps][3][kQueue];
  __shared__ int s_clo[kPairWarps][32];
  __shared__ int s_cex[kPairWarps][32];
  __shared__ R s_coff[kPairWarps][3][32];
  __shared__ int s_sp[kPairWarps][16];
  __shared__ double s_spw[kPairWarps][16];
  __shared__ double s_red[kPairWarps][9];

  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sidx = wk.y + wid;
  const unsigned FULL = 0xffffffffu;
  PairAcc a;
#pragma unroll
  for (int k = 0; k < 3; ++k) a.f[k] = a.g[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) a.vir[k] = 0.0;
  a.rho = a.e0 = a.e1 = 0.0;
  int i = -1;
  int n_core = 0, n_shell = 0;

  if (sidx < s.n) {
    const int4 mi = __ldg(&s.smeta[sidx]);
    i = mi.x;
    const int ti = mi.y, moli = mi.z;
    const double4 xi = ldg4(&s.sx[sidx]);
    const typename Vec4<R>::T pi4 = load_sorted<R>(s, sidx);
    const R pix = pi4.x, piy = pi4.y, piz = pi4.z;
    int c0 = (int)((xi.x - s.lo[0]) / s.d[0]);
    int c1 = (int)((xi.y - s.lo[1]) / s.d[1]);
    int c2 = (int)((xi.z - s.lo[2]) / s.d[2]);
    const double fpi = (MODE == kEAM_FORCE) ? s.eam_fp[i] : 0.0;
    // special list of i (first 16 entries in shared memory)
    int nsp = 0;
    const int* spi = nullptr;
    const double* spw = nullptr;
    if (SPECIAL) {
      const int b = s.sp_off[i], e = s.sp_off[i + 1];
      nsp = e - b;
      if (nsp <= 16) {
        if (lane < nsp) {
          s_sp[wid][lane] = s.sp_ids[b + lane];
          s_spw[wid][lane] = s.sp_w[b + lane];
        }
        __syncwarp();
        spi = s_sp[wid];
        spw = s_spw[wid];
      } else {
        spi = s.sp_ids + b;
        spw = s.sp_w + b;
      }
    }
    const bool rbl = (MODE == kLJ_RBL || MODE == kCOUL_RBL || MODE == kLIST ||
                      ((MODE == kEAM_RHO || MODE == kEAM_FORCE) && s.neigh == RBMD_NEIGH_RBL));
    const int pice = rbl ? s.pice : 1;
    int nsh = 0;  // running shell index (index_shell of the reference)
    if (rbl && s.rbl_mode == RBMD_RBL_PHILOX && pice > 1) {
      uint32_t o[4];
      philox4x32_10((uint32_t)i, 0u, (uint32_t)s.st->step, kTagRblOffset, s.seed_lo, s.seed_hi, o);
      nsh = (int)(o[0] % (uint32_t)pice);
    }
    const R rc2 = (R)s.rc2, rs2 = (R)s.rs2;
    const int nc = s.nc, side = 2 * nc + 1, ntrav = side * side * side;
    int qn = 0;

    auto flush = [&](int cnt) {
      if (lane < cnt) {
        int js = s_qj[wid][lane];
        const bool core = js >= 0;
        if (!core) js = ~js;
        const R rx = s_qr[wid][0][lane], ry = s_qr[wid][1][lane], rz = s_qr[wid][2][lane];
        eval_pair<R, MODE, SPECIAL, VIRIAL>(s, i, ti, moli, xi.w, fpi, js, core, rx, ry, rz, spi, spw,
                                            nsp, (R)pice, a);
      }
      if (MODE == kLIST) {
        int js = (lane < cnt) ? s_qj[wid][lane] : 0;
        const bool core = (lane < cnt) && js >= 0;
        const bool shell = (lane < cnt) && js < 0;
        const unsigned cm = __ballot_sync(FULL, core), sm = __ballot_sync(FULL, shell);
        if (core) {
          const int pos = n_core + __popc(cm & lanemask_lt(lane));
          if (pos < cap) out_core[(size_t)i * cap + pos] = __ldg(&s.smeta[js]).x;
        }
        if (shell) {
          const int pos = n_shell + __popc(sm & lanemask_lt(lane));
          if (pos < cap) out_shell[(size_t)i * cap + pos] = __ldg(&s.smeta[~js]).x;
        }
        n_core += __popc(cm);
        n_shell += __popc(sm);
      }
    };

    for (int t0 = 0; t0 < ntrav; t0 += 32) {
      const int t = t0 + lane;
      int cnt = 0, clo = 0;
      R ox = R(0), oy = R(0), oz = R(0);
      if (t < ntrav) {
        const int da = t / (side * side) - nc, db = (t / side) % side - nc, de = t % side - nc;
        const int n0 = c0 + da, n1 = c1 + db, n2 = c2 + de;
        // PeriodicIndexOffset: (n + dims) % dims; taken as a true modulo so that a position far
        // outside the box cannot produce a negative cell index
        const int w0 = ((n0 % s.dims[0]) + s.dims[0]) % s.dims[0];
        const int w1 = ((n1 % s.dims[1]) + s.dims[1]) % s.dims[1];
        const int w2 = ((n2 % s.dims[2]) + s.dims[2]) % s.dims[2];
        ox = (R)(s.d[0] * (double)(w0 - n0));
        oy = (R)(s.d[1] * (double)(w1 - n1));
        oz = (R)(s.d[2] * (double)(w2 - n2));
        const int cell = w0 + w1 * s.dims[0] + w2 * s.dims[0] * s.dims[1];
        clo = __ldg(&s.cell_start[cell]);
        cnt = __ldg(&s.cell_start[cell + 1]) - clo;
      }
      const int incl = warp_incl_scan(cnt, lane);
      const int total = __shfl_sync(FULL, incl, 31);
      s_clo[wid][lane] = clo;
      s_cex[wid][lane] = incl - cnt;
      s_coff[wid][0][lane] = ox;
      s_coff[wid][1][lane] = oy;
      s_coff[wid][2][lane] = oz;
      __syncwarp();
      for (int base = 0; base < total; base += 32) {
        const int p = base + lane;
        const bool valid = p < total;
        bool core = false, shell = false;
        R rx = R(0), ry = R(0), rz = R(0);
        int js = 0;
        if (valid) {
          int lo = 0, hi = 31;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_cex[wid][mid] <= p) lo = mid;
            else hi = mid - 1;
          }
          js = s_clo[wid][lo] + (p - s_cex[wid][lo]);
          const typename Vec4<R>::T pj = load_sorted<R>(s, js);
          rx = (pj.x - s_coff[wid][0][lo]) - pix;
          ry = (pj.y - s_coff[wid][1][lo]) - piy;
          rz = (pj.z - s_coff[wid][2][lo]) - piz;
          const R d2 = add_rn(add_rn(mul_rn(rx, rx), mul_rn(ry, ry)), mul_rn(rz, rz));
          if (rbl) {
            shell = (rc2 - d2 > R(0.0001) && d2 - rs2 > R(0.0001));
            core = !shell && (rs2 - d2 > R(0.0001) && d2 > R(0.0001));
          } else {
            core = (rc2 - d2 > R(0.0001) && d2 > R(0.0001));
          }
        }
        bool sel = core;
        if (rbl) {
          if (pice == 1) {
            sel = core || shell;
          } else {
            const unsigned sm = __ballot_sync(FULL, shell);
            const int rank = nsh + __popc(sm & lanemask_lt(lane));
            sel = core || (shell && (rank % pice) == 0);
            nsh += __popc(sm);
          }
        }
        const unsigned selm = __ballot_sync(FULL, sel);
        if (sel) {
          const int pos = qn + __popc(selm & lanemask_lt(lane));
          s_qj[wid][pos] = core ? js : ~js;
          s_qr[wid][0][pos] = rx;
          s_qr[wid][1][pos] = ry;
          s_qr[wid][2][pos] = rz;
        }
        qn += __popc(selm);
        __syncwarp();
        if (qn >= 32) {
          flush(32);
          __syncwarp();
          const int rest = qn - 32;
          int tj = 0;
          R tr0 = R(0), tr1 = R(0), tr2 = R(0);
          if (lane < rest) {
            tj = s_qj[wid][32 + lane];
            tr0 = s_qr[wid][0][32 + lane];
            tr1 = s_qr[wid][1][32 + lane];
            tr2 = s_qr[wid][2][32 + lane];
          }
          __syncwarp();
          if (lane < rest) {
            s_qj[wid][lane] = tj;
            s_qr[wid][0][lane] = tr0;
            s_qr[wid][1][lane] = tr1;
            s_qr[wid][2][lane] = tr2;
          }
          qn = rest;
          __syncwarp();
        }
      }
      __syncwarp();
    }
    if (qn > 0) flush(qn);
    __syncwarp();
  }

  // warp reduction of the per-lane accumulators
  double r9[9];
  r9[0] = warp_sum(a.f[0]);
  r9[1] = warp_sum(a.f[1]);
  r9[2] = warp_sum(a.f[2]);
  if (MODE == kCOUL_RBL) {
    const double q0 = warp_sum(a.g[0]), q1 = warp_sum(a.g[1]), q2 = warp_sum(a.g[2]);
    r9[0] = r9[0] + s.qqr2e * q0;
    r9[1] = r9[1] + s.qqr2e * q1;
    r9[2] = r9[2] + s.qqr2e * q2;
  }
  if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) r9[0] = warp_sum(a.rho);
  if (MODE == kEAM_ENERGY) r9[1] = warp_sum(a.e1);
  if (MODE == kENERGY) {
    r9[0] = warp_sum(a.e0);
    r9[1] = warp_sum(a.e1);
  }
  if (VIRIAL) {
#pragma unroll
    for (int k = 0; k < 6; ++k) r9[3 + k] = warp_sum(a.vir[k]);
  } else {
#pragma unroll
    for (int k = 3; k < 9; ++k) r9[k] = 0.0;
  }
  if (MODE == kLIST) {
    if (lane == 0 && i >= 0) {
      out_nc[i] = n_core;
      out_ns[i] = n_shell;
    }
    return;
  }

  if (lane == 0 && i >= 0) {
    if (MODE == kEAM_RHO) {
      // ComputeEAMfp (ExecForceFunction.h:946-962)
      const double rho = r9[0];
      double p = rho * (1.0 / s.eam_drho) + 1.0;
      int m = (int)p;
      m = max(1, min(m, s.eam_nrho - 1));
      p -= m;
      p = fmin(p, 1.0);
      const double* c = s.frho_s + 7 * m;
      s.eam_fp[i] = (c[0] * p + c[1]) * p + c[2];
    } else if (MODE == kEAM_ENERGY) {
      const double rho = r9[0];
      double p = rho * (1.0 / s.eam_drho) + 1.0;
      int m = (int)p;
      m = max(1, min(m, s.eam_nrho - 1));
      p -= m;
      p = fmin(p, 1.0);
      const double* c = s.frho_s + 7 * m;
      const double fpv = (c[0] * p + c[1]) * p + c[2];
      double phi = ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
      if (rho > s.eam_rhomax) phi += fpv * (rho - s.eam_rhomax);
      r9[0] = phi;
    } else if (MODE != kENERGY) {
      s.f[i] = make_double4(r9[0], r9[1], r9[2], 0.0);
    }
  }
  // per-block partial sums (RBL mean force, virial, energies) and the system epilogue
  const bool need_red = (MODE == kLJ_RBL || MODE == kCOUL_RBL || MODE == kENERGY ||
                         MODE == kEAM_ENERGY || VIRIAL ||
                         (MODE == kEAM_FORCE && s.neigh == RBMD_NEIGH_RBL));
  if (!need_red) return;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 9; ++k) s_red[wid][k] = (i >= 0) ? r9[k] : 0.0;
  }
  __syncthreads();
  const int blk = wk.y / kPairWarps;
  if (threadIdx.x < 9) {
    double t = 0.0;
    for (int w = 0; w < kPairWarps; ++w) t += s_red[w][threadIdx.x];
    s.vir_part[(size_t)blk * 9 + threadIdx.x] = t;
  }
  if (arrive_last(&s.st->counter[0], (unsigned)s.blocks_pair)) {
    if (threadIdx.x < 9) {
      double t = 0.0;
      for (int b = 0; b < s.blocks_pair; ++b) t += __ldcg(&s.vir_part[(size_t)b * 9 + threadIdx.x]);
      const int k = threadIdx.x;
      if (MODE == kENERGY) {
        if (k < 2) s.st->energy[k] = t;
      } else if (MODE == kEAM_ENERGY) {
        if (k < 2) s.st->energy[2 + k] = t;
      } else {
        if (k < 3 && MODE != kEAM_RHO) s.st->fmean[k] = (MODE == kLJ_VERLET || MODE == kCOUL_VERLET) ? 0.0 : t / s.n;
        if (k >= 3 && VIRIAL) s.st->virial[k - 3] = t;
      }
    }
  }
}

template <typename R, int MODE, bool SPECIAL, bool VIRIAL>
static void go(const Batch& b, cudaStream_t st) {
  k_pair<R, MODE, SPECIAL, VIRIAL><<<b.pair.n, kPairWarps * 32, 0, st>>>(b.sys, b.pair.d, 0, nullptr,
                                                                        nullptr, nullptr, nullptr);
  note_launch();
}

template <typename R, bool VIRIAL>
static void dispatch(const Batch& b, cudaStream_t st) {
  if (b.ff == RBMD_FF_EAM) {
    go<R, kEAM_RHO, false, false>(b, st);
    go<R, kEAM_FORCE, false, false>(b, st);
    return;
  }
  const bool coul = b.ff != RBMD_FF_LJ_CUT;
  if (b.neigh == RBMD_NEIGH_RBL) {
    if (!coul) go<R, kLJ_RBL, false, false>(b, st);
    else if (b.special) go<R, kCOUL_RBL, true, false>(b, st);
    else go<R, kCOUL_RBL, false, false>(b, st);
  } else {
    if (!coul) go<R, kLJ_VERLET, false, VIRIAL>(b, st);
    else if (b.special) go<R, kCOUL_VERLET, true, VIRIAL>(b, st);
    else go<R, kCOUL_VERLET, false, VIRIAL>(b, st);
  }
}

void launch_pair(const Batch& b, cudaStream_t st, int virial) {
  if (b.prec == RBMD_PREC_MIXED) {
    if (virial) dispatch<float, true>(b, st);
    else dispatch<float, false>(b, st);
  } else {
    if (virial) dispatch<double, true>(b, st);
    else dispatch<double, false>(b, st);
  }
}

void launch_energy(const Batch& b, cudaStream_t st) {
  if (b.ff == RBMD_FF_EAM) {
    go<double, kEAM_ENERGY, false, false>(b, st);
  } else if (b.special && b.ff != RBMD_FF_LJ_CUT) {
    go<double, kENERGY, true, false>(b, st);
  } else {
    go<double, kENERGY, false, false>(b, st);
  }
}

void launch_rbl_lists(const SysDev* sys, int slot, int n, int cap, int* n_core, int* n_shell,
                      int* ids, cudaStream_t st) {
  // ids holds 2 * n * cap ints: core rows then shell rows
  int nb = (n + kPairWarps - 1) / kPairWarps;
  int2* d_work = nullptr;
  cudaMallocAsync(&d_work, sizeof(int2) * nb, st);
  int2* h = new int2[nb];
  for (int k = 0; k < nb; ++k) h[k] = make_int2(slot, k * kPairWarps);
  cudaMemcpyAsync(d_work, h, sizeof(int2) * nb, cudaMemcpyHostToDevice, st);
  k_pair<double, kLIST, false, false><<<nb, kPairWarps * 32, 0, st>>>(sys, d_work, cap, n_core, n_shell,
                                                                     ids, ids + (size_t)n * cap);
  note_launch();
  cudaStreamSynchronize(st);
  delete[] h;
  cudaFreeAsync(d_work, st);
}

}  // namespace rbmd
