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
// Three traversals share the selection rule and the pair arithmetic:
//   k_pair       one warp per atom, any box (cells may repeat in the stencil of a small box);
//   k_pair2      one warp per atom with per-atom segment tables (every dimension holds 2 nc + 1
//                cells), cells beyond rc of the atom culled;
//   k_pair_tile  one warp per home cell: the cell's atoms share each batch of 32 candidates, the
//                default for mixed precision once cells hold a few atoms.
// All visit the (2 nc + 1)^3 neighbour cells in the reference order (x offset outermost, z
// innermost, ascending atom id inside a cell).  The shell rank of every candidate is its position
// among the shells of that order, which reproduces the reference's sequential "every pice-th shell
// atom" pick exactly.  Selected pairs are queued in shared memory and evaluated with full warps.
// FP64 classification uses explicitly rounded products and sums (or, in the tile kernel, exact
// threshold equivalents of the reference's window tests) so that it makes the same decisions as
// the CPU oracle on the same positions.
#include <algorithm>
#include <mutex>

#include "kernels.h"

#include <type_traits>

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

// Mixed precision: an FP32 squared distance carries the rounding of the FP32 positions and image
// shifts.  A pair whose FP32 value lies within that error band of a classification threshold
// (centres amb_c, half-widths amb_w, set on the host from a bound on the error) is classified
// again from the FP64 positions with the FP64 kernels' arithmetic and thresholds, so that core /
// shell membership, and with it the RBL picks, are exactly those of the FP64 path.  m is the
// candidate's image offset in cells (wrapped - unwrapped cell index) per dimension.
__device__ __forceinline__ bool f32_banded(const SysDev& s, float dd) {
  return (dd >= s.band[0] && dd <= s.band[1]) || (dd >= s.band[2] && dd <= s.band[3]);
}
__device__ __forceinline__ void classify_fp64(const SysDev& s, double pix, double piy, double piz, int js, int mx, int my,
                                           int mz, bool rbl, bool& core, bool& shell) {
  const double4 pj = ldg4(&s.sx[js]);
  const double rx = (pj.x - s.d[0] * (double)mx) - pix;
  const double ry = (pj.y - s.d[1] * (double)my) - piy;
  const double rz = (pj.z - s.d[2] * (double)mz) - piz;
  const double dd = add_rn(add_rn(mul_rn(rx, rx), mul_rn(ry, ry)), mul_rn(rz, rz));
  shell = rbl && dd >= s.cls_d[1] && dd <= s.cls_d[0];
  core = rbl ? (dd <= s.cls_d[2] && dd > 0.0001) : (dd <= s.cls_d[0] && dd > 0.0001);
}

__device__ inline double r_sqrt(double x) { return sqrt(x); }
__device__ inline float r_sqrt(float x) { return sqrtf(x); }
__device__ inline double r_exp(double x) { return exp(x); }
__device__ inline float r_exp(float x) { return __expf(x); }
__device__ inline double r_erfc(double x) { return erfc(x); }
__device__ inline float r_erfc(float x) { return erfcf(x); }

// The reference's near-Coulomb table (ExecStaticTable::Extract + TableGnearValue,
// staticTable/ExecStaticTable.h:96-135): G at the key of the FP32 distance, bits 15-25 of its
// pattern; closer than 0.1, before the reference's first entry, the entry of r = 0.1 (key 921).
__device__ __forceinline__ float near_table_g(const float* __restrict__ tab, float dis) {
  const unsigned k = dis < 0.1f ? 921u : ((__float_as_uint(dis) & 0x03FF8000u) >> 15);
  return __ldg(&tab[k]);
}

// EAM spline row evaluation (ExecForceFunction::ComputeEAMrho / ComputeEAMforce)
__device__ inline void eam_row(const double* tab, double r, double rdr, int nr, int& m, double& p) {
  p = r * rdr + 1.0;
  m = (int)p;
  m = min(m, nr - 1);
  p -= m;
  p = fmin(p, 1.0);
}

// EAM tables of a type and of a type pair: one table of each kind for every type (funcfl, the
// reference's EAM), or per type (setfl): frho / rhor by type, z2r by pair i >= j at i (i+1)/2 + j
// (LAMMPS pair eam/alloy's type2frho, type2rhor, type2z2r).
__device__ inline const double* eam_frho(const SysDev& s, int t) {
  return s.eam_per_type ? s.frho_s + (size_t)t * 7 * (s.eam_nrho + 1) : s.frho_s;
}
__device__ inline const double* eam_rhor(const SysDev& s, int t) {
  return s.eam_per_type ? s.rhor_s + (size_t)t * 7 * (s.eam_nr + 1) : s.rhor_s;
}
__device__ inline const double* eam_z2r(const SysDev& s, int a, int b) {
  if (!s.eam_per_type) return s.z2r_s;
  const int hi = max(a, b), lo = min(a, b);
  return s.z2r_s + (size_t)(hi * (hi + 1) / 2 + lo) * 7 * (s.eam_nr + 1);
}

struct PairAcc {
  double f[3];
  double g[3];    // Coulomb part before qqr2e (RBL Coulomb modes)
  double rho;     // EAM density / energy scalar
  double e0, e1;  // energies
  double vir[6];
};

template <typename R, int MODE, bool SPECIAL, bool VIRIAL, bool NEAR = false>
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
    const int tj = mj.y;
    if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) {
      const double* c = eam_rhor(s, tj) + 7 * m;  // the density the neighbour's type contributes
      a.rho += scale * (((__ldg(c + 3) * p + __ldg(c + 4)) * p + __ldg(c + 5)) * p + __ldg(c + 6));
      if (MODE == kEAM_ENERGY) {
        const double* z = eam_z2r(s, ti, tj) + 7 * m;
        double z2 = ((__ldg(z + 3) * p + __ldg(z + 4)) * p + __ldg(z + 5)) * p + __ldg(z + 6);
        a.e1 += 0.5 * (z2 * (1.0 / rr));
      }
    } else {
      const double* ci = eam_rhor(s, ti) + 7 * m;
      const double rhoip = (__ldg(ci) * p + __ldg(ci + 1)) * p + __ldg(ci + 2);
      const double* cj = eam_rhor(s, tj) + 7 * m;
      const double rhojp = (__ldg(cj) * p + __ldg(cj + 1)) * p + __ldg(cj + 2);
      const double* cz = eam_z2r(s, ti, tj) + 7 * m;
      const double z2p = (__ldg(cz) * p + __ldg(cz + 1)) * p + __ldg(cz + 2);
      const double z2 = ((__ldg(cz + 3) * p + __ldg(cz + 4)) * p + __ldg(cz + 5)) * p + __ldg(cz + 6);
      const double recip = 1.0 / rr;
      const double phi = z2 * recip;
      const double phip = z2p * recip - phi * recip;
      const double psip = fpi * rhojp + __ldg(&s.eam_fp[mj.x]) * rhoip + phip;
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
      R g;
      if constexpr (NEAR) {  // RBMD_NEAR_TABLE
        g = (R)near_table_g(s.near_tab, (float)dis);
      } else {
        const R sa = r_sqrt(alpha);
        g = r_erfc(sa * dis) / d2 + R(2) * sa * r_exp(-alpha * d2) / ((R)sqrt(kPif) * dis);
      }
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

template <typename R, int MODE, bool SPECIAL, bool VIRIAL, bool NEAR = false>
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
        eval_pair<R, MODE, SPECIAL, VIRIAL, NEAR>(s, i, ti, moli, xi.w, fpi, js, core, rx, ry, rz, spi, spw,
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
        const int cell = w2 + s.dims[2] * (w1 + s.dims[1] * w0);
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
          if constexpr (sizeof(R) == 4) {
            if (f32_banded(s, (float)d2))
              classify_fp64(s, xi.x, xi.y, xi.z, js, (int)rintf((float)(s_coff[wid][0][lo] / s.d[0])),
                            (int)rintf((float)(s_coff[wid][1][lo] / s.d[1])),
                            (int)rintf((float)(s_coff[wid][2][lo] / s.d[2])), rbl, core, shell);
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
      const double* c = eam_frho(s, s.meta[i].x) + 7 * m;
      s.eam_fp[i] = (c[0] * p + c[1]) * p + c[2];
    } else if (MODE == kEAM_ENERGY) {
      const double rho = r9[0];
      double p = rho * (1.0 / s.eam_drho) + 1.0;
      int m = (int)p;
      m = max(1, min(m, s.eam_nrho - 1));
      p -= m;
      p = fmin(p, 1.0);
      const double* c = eam_frho(s, s.meta[i].x) + 7 * m;
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

// ------------------------------------------------------------------------------------------------
// Lean warp-per-atom traversal (boxes with at least 2 nc + 1 cells per dimension).  Per atom i the
// warp first builds a segment table: every traversal row (fixed x and y cell offsets) is one or two
// contiguous ranges of the cell-ordered arrays (z-fastest cell numbering; the split is the
// periodic wrap), trimmed to the cells that can hold an atom within rc of i (cells entirely beyond
// rc can never hold a core or shell atom, so dropping them keeps every shell rank unchanged).
// Lanes then walk the flattened candidate sequence with a per-lane segment cursor; the stride pick
// uses a precomputed bit mask instead of a modulo per candidate; selected pairs go through a
// 64-entry ring queue and are evaluated 32 at a time.

// Abramowitz & Stegun 7.1.26: erfc(x) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2),
// t = 1 / (1 + p x), |error| <= 1.5e-7; used by the FP32 path only, sharing the exponential with
// the second term of the real-space Coulomb kernel.  The reciprocal is the hardware approximation
// (a few ulp), well inside the formula's own error.
__device__ inline float erfc_as_times(float x, float e) {
  const float t = __fdividef(1.0f, 1.0f + 0.3275911f * x);
  return t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f)))) * e;
}

// FP32 pair arithmetic of the RBL modes on preloaded data of j (type tj, molecule molj, charge qj)
// and the special-bond weight w of the pair.  IMG applies the minimum image; callers whose
// displacement is already the nearest image (|r| < rc < L / 2) skip it.
template <int MODE, bool IMG = true, bool NEAR = false>
__device__ inline void eval_pair_f32_pre(int moli, float qi, bool core, float rx, float ry, float rz, int ti, int tj,
                                         int molj, float qj, float w, float pice, float rc2, float rs2, float sa,
                                         float alpha, const float* tab, int ntypes, float Lx, float Ly, float Lz,
                                         float& fx, float& fy, float& fz, float& gx, float& gy, float& gz,
                                         bool special, const float* ntab) {
  if (MODE == kLJ_RBL && moli == molj) return;
  if (IMG) min_image(rx, ry, rz, Lx, Ly, Lz);
  const float d2 = rx * rx + ry * ry + rz * rz;
  const int tp = ti * ntypes + tj;
  const float clj = tab[2 * tp], s6 = tab[2 * tp + 1];
  const float inv_r = rsqrtf(d2);
  const float inv_d2 = inv_r * inv_r;
  const float sd6 = s6 * inv_d2 * inv_d2 * inv_d2;
  const float ljf = clj * (2.0f * sd6 - 1.0f) * sd6 * inv_d2;  // force / r_vector
  float fl = 0.0f;
  if (MODE == kLJ_RBL) {
    if (core) fl = (d2 < rc2 && d2 > 0.0001f) ? ljf : 0.0f;
    else fl = (d2 < rc2 && d2 > rs2) ? pice * ljf : 0.0f;
  } else {
    if (core) fl = (d2 < rs2 && d2 > 0.0001f) ? w * ljf : 0.0f;
    else fl = (d2 < rc2 && d2 > rs2) ? w * (pice * ljf) : 0.0f;
  }
  fx += fl * rx;
  fy += fl * ry;
  fz += fl * rz;
  if (MODE == kCOUL_RBL) {
    const bool in = core ? (d2 < rc2 && d2 > 0.0001f)
                         : (special ? (d2 < rc2 && d2 > rs2) : (d2 < rc2 && d2 > 0.0001f));
    if (in) {
      float g;
      if constexpr (NEAR) {  // RBMD_NEAR_TABLE
        g = near_table_g(ntab, __fsqrt_rn(d2));
      } else {
        const float r = d2 * inv_r;
        const float x = sa * r;
        const float e = __expf(-alpha * d2);
        g = erfc_as_times(x, e) * inv_d2 + 1.1283791671f * sa * e * inv_r;  // 2/sqrt(pi)
      }
      float fc = -qi * qj * g * inv_r;
      if (!core) fc *= pice;
      gx += fc * rx;
      gy += fc * ry;
      gz += fc * rz;
    }
  }
}

template <int MODE, bool SPECIAL, bool NEAR = false>
__device__ inline void eval_pair_f32(const SysDev& s, int moli, float qi, int js, bool core, float rx, float ry,
                                     float rz, int ti, const int* spi, const double* spw, int nsp, float pice,
                                     float rc2, float rs2, float sa, float alpha, const float* tab, int ntypes,
                                     float Lx, float Ly, float Lz, float& fx, float& fy, float& fz, float& gx,
                                     float& gy, float& gz) {
  const int4 mj = __ldg(&s.smeta[js]);
  if (MODE == kLJ_RBL && moli == mj.z) return;
  float w = 1.0f;
  if (SPECIAL)
    for (int k = 0; k < nsp; ++k)
      if (spi[k] == mj.x) w = (float)spw[k];
  const float qj = (MODE == kCOUL_RBL) ? __ldg(&s.sxf[js].w) : 0.0f;
  eval_pair_f32_pre<MODE, true, NEAR>(moli, qi, core, rx, ry, rz, ti, mj.y, mj.z, qj, w, pice, rc2, rs2, sa, alpha, tab,
                                      ntypes, Lx, Ly, Lz, fx, fy, fz, gx, gy, gz, SPECIAL, s.near_tab);
}

template <typename R, int MODE, bool SPECIAL, bool VIRIAL, bool NEAR = false>
__global__ void __launch_bounds__(kPairWarps * 32, 3)
k_pair2(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  using R4 = typename Vec4<R>::T;
  constexpr bool F32 = sizeof(R) == 4 && (MODE == kLJ_RBL || MODE == kCOUL_RBL);
  __shared__ int s_qj[kPairWarps][64];
  __shared__ R s_qr[kPairWarps][3][64];
  __shared__ int s_sa[kPairWarps][64];   // segment first sorted index
  __shared__ int s_sb[kPairWarps][64];   // segment begin in the flattened sequence
  __shared__ int s_se[kPairWarps][64];   // segment end in the flattened sequence
  __shared__ R s_so[kPairWarps][3][64];  // segment coordinate offsets
  __shared__ float s_tab[2 * kMaxF32Types * kMaxF32Types];  // FP32 LJ table: -24 sqrt(eps eps), sigma^6
  __shared__ double s_red[kPairWarps][9];

  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  const int n = s.n, ntypes = s.ntypes;
  if (F32) {
    for (int t = threadIdx.x; t < ntypes * ntypes && t < kMaxF32Types * kMaxF32Types; t += blockDim.x) {
      const int a = t / ntypes, b = t % ntypes;
      const double sg = (s.sig[a] + s.sig[b]) / 2;
      s_tab[2 * t] = (float)(-24.0 * sqrt(s.eps[a] * s.eps[b]));
      s_tab[2 * t + 1] = (float)(sg * sg * sg * sg * sg * sg);
    }
    __syncthreads();
  }
  const int sidx = wk.y + wid;
  PairAcc a;
#pragma unroll
  for (int k = 0; k < 3; ++k) a.f[k] = a.g[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) a.vir[k] = 0.0;
  a.rho = a.e0 = a.e1 = 0.0;
  float ffx = 0.f, ffy = 0.f, ffz = 0.f, fgx = 0.f, fgy = 0.f, fgz = 0.f;
  int i = -1;

  if (sidx < n) {
    const int dx = s.dims[0], dy = s.dims[1], dz = s.dims[2];
    const double d0 = s.d[0], d1 = s.d[1], d2c = s.d[2];
    const int4 mi = __ldg(&s.smeta[sidx]);
    i = mi.x;
    const int ti = mi.y, moli = mi.z;
    const double4 xi = ldg4(&s.sx[sidx]);
    const R4 pi4 = load_sorted<R>(s, sidx);
    const R pix = pi4.x, piy = pi4.y, piz = pi4.z;
    // home cell by truncation and NOT clamped (InWhichCell, ExecPointLocator.h:271-274): an atom
    // that a step left outside the box walks the neighbourhood of its unclamped cell, every
    // neighbour cell wrapped by a true modulo below
    const int c0 = (int)((xi.x - s.lo[0]) / d0);
    const int c1 = (int)((xi.y - s.lo[1]) / d1);
    const int c2 = (int)((xi.z - s.lo[2]) / d2c);
    const double fpi = (MODE == kEAM_FORCE) ? s.eam_fp[i] : 0.0;
    int nsp = 0;
    const int* spi = nullptr;
    const double* spw = nullptr;
    if (SPECIAL) {
      const int b = s.sp_off[i];
      nsp = s.sp_off[i + 1] - b;
      spi = s.sp_ids + b;
      spw = s.sp_w + b;
    }
    const bool rbl = (MODE == kLJ_RBL || MODE == kCOUL_RBL ||
                      ((MODE == kEAM_RHO || MODE == kEAM_FORCE) && s.neigh == RBMD_NEIGH_RBL));
    const int pice = rbl ? s.pice : 1;
    int nsh_mod = 0;  // running shell index modulo pice
    if (rbl && s.rbl_mode == RBMD_RBL_PHILOX && pice > 1) {
      uint32_t o[4];
      philox4x32_10((uint32_t)i, 0u, (uint32_t)s.st->step, kTagRblOffset, s.seed_lo, s.seed_hi, o);
      nsh_mod = (int)(o[0] % (uint32_t)pice);
    }
    uint32_t base_mask = 0;  // bits 0, pice, 2 pice, ... below 32
    for (int k = 0; k < 32; k += pice) base_mask |= (1u << k);
    const R rc2 = (R)s.rc2, rs2 = (R)s.rs2;
    const int nc = s.nc, side = 2 * nc + 1, nrows = side * side;
    // conservative culling radius: cells farther than rc from i (with a margin for atoms outside
    // their cell: at least the farthest an atom lay outside its binned cell plus the largest SHAKE
    // displacement since the cell list was built) cannot hold a core or shell atom; cells of atoms
    // SHAKE wrapped across the box (they sit on the far side of it) are never culled, and beyond
    // kMaxMigrated of them nothing is
    const double margin =
        fmax(0.1 * fmin(d0, fmin(d1, d2c)), 1.001 * ((double)__uint_as_float(s.st->shake_disp_bits) +
                                                     (double)__uint_as_float(s.st->out_bits)));
    const int mig_n = s.st->mig_n;
    const double cut2 = s.rc2;
    const double lo0 = s.lo[0], lo1 = s.lo[1], lo2 = s.lo[2];
    const float spice = (float)pice;
    const float fsa = (float)sqrt(s.alpha), falpha = (float)s.alpha;
    const float fLx = (float)s.L[0], fLy = (float)s.L[1], fLz = (float)s.L[2];
    const float frc2 = (float)s.rc2, frs2 = (float)s.rs2;
    int head = 0, qn = 0;

    auto flush = [&](int cnt) {
      if (lane < cnt) {
        const int slot = (head + lane) & 63;
        int js = s_qj[wid][slot];
        const bool core = js >= 0;
        if (!core) js = ~js;
        if (F32) {
          eval_pair_f32<MODE, SPECIAL, NEAR>(s, moli, (float)xi.w, js, core, (float)s_qr[wid][0][slot],
                                       (float)s_qr[wid][1][slot], (float)s_qr[wid][2][slot], ti, spi, spw, nsp,
                                       spice, frc2, frs2, fsa, falpha, s_tab, ntypes, fLx, fLy, fLz, ffx, ffy, ffz,
                                       fgx, fgy, fgz);
        } else {
          eval_pair<R, MODE, SPECIAL, VIRIAL, NEAR>(s, i, ti, moli, xi.w, fpi, js, core, s_qr[wid][0][slot],
                                              s_qr[wid][1][slot], s_qr[wid][2][slot], spi, spw, nsp, (R)pice, a);
        }
      }
      head = (head + cnt) & 63;
      qn -= cnt;
    };

    // rows per segment table: 32 of at most two ranges each, or 21 of at most three when the box
    // holds fewer than 2 nc + 1 cells in z (the table holds 64)
    const int group = dz >= side ? 32 : 21;
    for (int r0 = 0; r0 < nrows; r0 += group) {
      // ---- segment table of rows r0 .. r0 + group - 1 (one row per lane)
      const int r = r0 + lane;
      int nseg = 0, cnt = 0;
      int sa0 = 0, sa1 = 0, sa2 = 0, n0c = 0, n1c = 0, n2c = 0;
      R oxv = R(0), oyv = R(0), oz0 = R(0), oz1 = R(0), oz2 = R(0);
      if (lane < group && r < nrows) {
        const int da = r / side - nc, db = r % side - nc;
        int n0 = c0 + da, n1 = c1 + db;
        int w0 = ((n0 % dx) + dx) % dx;
        int w1 = ((n1 % dy) + dy) % dy;
        const double ox = d0 * (double)(w0 - n0), oy = d1 * (double)(w1 - n1);
        oxv = (R)ox;
        oyv = (R)oy;
        // squared gap between i and the column of cells (unwrapped frame), shrunk by the margin
        const double bx0 = lo0 + n0 * d0 - margin, bx1 = lo0 + (n0 + 1) * d0 + margin;
        const double by0 = lo1 + n1 * d1 - margin, by1 = lo1 + (n1 + 1) * d1 + margin;
        const double gx = fmax(0.0, fmax(bx0 - xi.x, xi.x - bx1));
        const double gy = fmax(0.0, fmax(by0 - xi.y, xi.y - by1));
        const double gxy = gx * gx + gy * gy;
        int elo = nc + 1, ehi = -nc - 1;
        if (gxy < cut2) {
          for (int de = -nc; de <= nc; ++de) {
            const int n2 = c2 + de;
            const double bz0 = lo2 + n2 * d2c - margin, bz1 = lo2 + (n2 + 1) * d2c + margin;
            const double gz = fmax(0.0, fmax(bz0 - xi.z, xi.z - bz1));
            if (gxy + gz * gz < cut2) {
              elo = min(elo, de);
              ehi = max(ehi, de);
            }
          }
        }
        if (mig_n > kMaxMigrated) {
          elo = -nc;
          ehi = nc;
        } else {
          for (int m = 0; m < mig_n; ++m) {
            const int cm = __ldg(&s.st->mig_cell[m]) - dz * (w1 + dy * w0);
            if (cm < 0 || cm >= dz) continue;  // not in this row's column
            for (int de = -nc; de <= nc; ++de)
              if ((((c2 + de) % dz) + dz) % dz == cm) {
                elo = min(elo, de);
                ehi = max(ehi, de);
              }
          }
        }
        {
          if (elo <= ehi) {
            // unwrapped z cells [z0, z1] (len <= 2 nc + 1 <= 2 dz - 1 of them) start in the
            // periodic copy q = floor(z0 / dz); they map to wrapped cells [zw, zw + len) when that
            // stays below dz, else to [zw, dz), then [0, rest) of the next copy, or [0, dz) and
            // [0, rest - dz) of the two next when the stencil is longer than the box.  The shift of
            // a cell is d * (wrapped - unwrapped) = -d dz q, -d dz (q + 1), -d dz (q + 2).
            const int base = dz * (w1 + dy * w0);
            const int z0 = c2 + elo, len = ehi - elo + 1;
            const int zw = ((z0 % dz) + dz) % dz;
            const int q = (z0 - zw) / dz;
            sa0 = __ldg(&s.cell_start[base + zw]);
            oz0 = (R)(-d2c * (double)dz * (double)q);
            if (zw + len <= dz) {
              n0c = __ldg(&s.cell_start[base + zw + len]) - sa0;
              nseg = 1;
            } else {
              n0c = __ldg(&s.cell_start[base + dz]) - sa0;
              const int rest = zw + len - dz;
              sa1 = __ldg(&s.cell_start[base]);
              oz1 = (R)(-d2c * (double)dz * (double)(q + 1));
              if (rest <= dz) {
                n1c = __ldg(&s.cell_start[base + rest]) - sa1;
                nseg = 2;
              } else {
                n1c = __ldg(&s.cell_start[base + dz]) - sa1;
                sa2 = sa1;
                n2c = __ldg(&s.cell_start[base + rest - dz]) - sa2;
                oz2 = (R)(-d2c * (double)dz * (double)(q + 2));
                nseg = 3;
              }
            }
            cnt = n0c + n1c + n2c;
          }
        }
      }
      const int seg_incl = warp_incl_scan(nseg, lane);
      const int cnt_incl = warp_incl_scan(cnt, lane);
      const int nsegs = __shfl_sync(FULL, seg_incl, 31);
      const int total = __shfl_sync(FULL, cnt_incl, 31);
      {
        int slot = seg_incl - nseg, beg = cnt_incl - cnt;
        if (nseg >= 1) {
          s_sa[wid][slot] = sa0;
          s_sb[wid][slot] = beg;
          s_se[wid][slot] = beg + n0c;
          s_so[wid][0][slot] = oxv;
          s_so[wid][1][slot] = oyv;
          s_so[wid][2][slot] = oz0;
        }
        if (nseg >= 2) {
          s_sa[wid][slot + 1] = sa1;
          s_sb[wid][slot + 1] = beg + n0c;
          s_se[wid][slot + 1] = beg + n0c + n1c;
          s_so[wid][0][slot + 1] = oxv;
          s_so[wid][1][slot + 1] = oyv;
          s_so[wid][2][slot + 1] = oz1;
        }
        if (nseg == 3) {
          s_sa[wid][slot + 2] = sa2;
          s_sb[wid][slot + 2] = beg + n0c + n1c;
          s_se[wid][slot + 2] = beg + n0c + n1c + n2c;
          s_so[wid][0][slot + 2] = oxv;
          s_so[wid][1][slot + 2] = oyv;
          s_so[wid][2][slot + 2] = oz2;
        }
      }
      __syncwarp();
      // ---- candidates of the flattened sequence, 32 per iteration
      int seg = 0;
      for (int base = 0; base < total; base += 32) {
        const int p = base + lane;
        const bool valid = p < total;
        bool core = false, shell = false;
        R rx = R(0), ry = R(0), rz = R(0);
        int js = 0;
        if (valid) {
          while (p >= s_se[wid][seg]) ++seg;
          js = s_sa[wid][seg] + (p - s_sb[wid][seg]);
          const R4 pj = load_sorted<R>(s, js);
          rx = (pj.x - s_so[wid][0][seg]) - pix;
          ry = (pj.y - s_so[wid][1][seg]) - piy;
          rz = (pj.z - s_so[wid][2][seg]) - piz;
          const R dd = add_rn(add_rn(mul_rn(rx, rx), mul_rn(ry, ry)), mul_rn(rz, rz));
          if (rbl) {
            shell = (rc2 - dd > R(0.0001) && dd - rs2 > R(0.0001));
            core = !shell && (rs2 - dd > R(0.0001) && dd > R(0.0001));
          } else {
            core = (rc2 - dd > R(0.0001) && dd > R(0.0001));
          }
          if constexpr (sizeof(R) == 4) {
            if (f32_banded(s, (float)dd))
              classify_fp64(s, xi.x, xi.y, xi.z, js, (int)rintf((float)(s_so[wid][0][seg] / d0)),
                            (int)rintf((float)(s_so[wid][1][seg] / d1)), (int)rintf((float)(s_so[wid][2][seg] / d2c)),
                            rbl, core, shell);
          }
        }
        bool sel = core;
        if (rbl) {
          if (pice == 1) {
            sel = core || shell;
          } else {
            const unsigned sm = __ballot_sync(FULL, shell);
            const int phase = nsh_mod == 0 ? 0 : pice - nsh_mod;
            const uint32_t mask = phase < 32 ? (base_mask << phase) : 0u;
            const int pre = __popc(sm & lanemask_lt(lane));
            sel = core || (shell && ((mask >> pre) & 1u));
            nsh_mod += __popc(sm);
            nsh_mod -= pice * (int)((unsigned)nsh_mod / (unsigned)pice);
          }
        }
        const unsigned selm = __ballot_sync(FULL, sel);
        if (sel) {
          const int slot = (head + qn + __popc(selm & lanemask_lt(lane))) & 63;
          s_qj[wid][slot] = core ? js : ~js;
          s_qr[wid][0][slot] = rx;
          s_qr[wid][1][slot] = ry;
          s_qr[wid][2][slot] = rz;
        }
        qn += __popc(selm);
        __syncwarp();
        if (qn >= 32) {
          flush(32);
          __syncwarp();
        }
      }
      __syncwarp();
    }
    if (qn > 0) flush(qn);
    __syncwarp();
  }

  double r9[9];
  if (F32) {
    r9[0] = warp_sum((double)ffx);
    r9[1] = warp_sum((double)ffy);
    r9[2] = warp_sum((double)ffz);
    if (MODE == kCOUL_RBL) {
      const double q0 = warp_sum((double)fgx), q1 = warp_sum((double)fgy), q2 = warp_sum((double)fgz);
      r9[0] = r9[0] + s.qqr2e * q0;
      r9[1] = r9[1] + s.qqr2e * q1;
      r9[2] = r9[2] + s.qqr2e * q2;
    }
  } else {
    r9[0] = warp_sum(a.f[0]);
    r9[1] = warp_sum(a.f[1]);
    r9[2] = warp_sum(a.f[2]);
    if (MODE == kCOUL_RBL) {
      const double q0 = warp_sum(a.g[0]), q1 = warp_sum(a.g[1]), q2 = warp_sum(a.g[2]);
      r9[0] = r9[0] + s.qqr2e * q0;
      r9[1] = r9[1] + s.qqr2e * q1;
      r9[2] = r9[2] + s.qqr2e * q2;
    }
  }
  if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) r9[0] = warp_sum(a.rho);
  if (MODE == kEAM_ENERGY) r9[1] = warp_sum(a.e1);
  if (MODE == kENERGY) {
    r9[0] = warp_sum(a.e0);
    r9[1] = warp_sum(a.e1);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) r9[3 + k] = VIRIAL ? warp_sum(a.vir[k]) : 0.0;

  if (lane == 0 && i >= 0) {
    if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) {
      const double rho = r9[0];
      double p = rho * (1.0 / s.eam_drho) + 1.0;
      int m = (int)p;
      m = max(1, min(m, s.eam_nrho - 1));
      p -= m;
      p = fmin(p, 1.0);
      const double* c = eam_frho(s, s.meta[i].x) + 7 * m;
      if (MODE == kEAM_RHO) {
        s.eam_fp[i] = (c[0] * p + c[1]) * p + c[2];
      } else {
        const double fpv = (c[0] * p + c[1]) * p + c[2];
        double phi = ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
        if (rho > s.eam_rhomax) phi += fpv * (rho - s.eam_rhomax);
        r9[0] = phi;
      }
    } else if (MODE != kENERGY) {
      s.f[i] = make_double4(r9[0], r9[1], r9[2], 0.0);
    }
  }
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
        if (k < 3) s.st->fmean[k] = (MODE == kLJ_VERLET || MODE == kCOUL_VERLET) ? 0.0 : t / s.n;
        if (k >= 3 && VIRIAL) s.st->virial[k - 3] = t;
      }
    }
  }
}

// Hardware approximations (flush-to-zero) for the FP32 tile evaluation; every argument there is
// a normal number (d2 > 1e-4, exponents in [-alpha rc2 log2 e, 0]).
__device__ inline float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ inline float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ inline float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// FP32 force of one RBL pair as a single vector factor: LJ (cutoff rs for core pairs of the
// Coulomb modes, rc for LJ/CUT, shell pairs x pice) plus qqr2e times the real-space Coulomb term
// (erfc by Abramowitz & Stegun 7.1.26, |error| <= 1.5e-7), the same windows as eval_pair_f32_pre.
// alpha_l2 = alpha log2(e), so exp(-alpha d2) = 2^(-alpha_l2 d2); clj = -24 sqrt(eps_i eps_j) and
// s6 = sigma_ij^6 are the type pair's FP32 LJ factors.
// The pair's class is exact (the FP64 decision, with the reference's 1e-4 margins around rs^2
// and rc^2), and it implies every cutoff test of the reference's force functions (core: d2 < rs^2
// and > 1e-4; shell: rs^2 < d2 < rc^2), so none is repeated here on the FP32 d2.
template <int MODE, bool NEAR>
__device__ inline float tile_pair_f32_lj(bool core, float d2, float qi, float qj, float clj, float s6, float w,
                                         float pice, float sa, float alpha_l2, float qq, const float* ntab) {
  const float inv_r = rsqrt_approx(d2);
  const float inv_d2 = inv_r * inv_r;
  const float sd6 = s6 * inv_d2 * inv_d2 * inv_d2;
  const float ljf = clj * (2.0f * sd6 - 1.0f) * sd6 * inv_d2;
  if (MODE == kLJ_RBL) return core ? ljf : pice * ljf;
  const float fl = core ? w * ljf : w * (pice * ljf);
  float g;
  if constexpr (NEAR) {  // RBMD_NEAR_TABLE
    g = near_table_g(ntab, __fsqrt_rn(d2));
  } else {
    const float x = sa * (d2 * inv_r);
    const float e = ex2_approx(-alpha_l2 * d2);
    const float t = rcp_approx(1.0f + 0.3275911f * x);
    const float erfc = t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f)))) * e;
    g = erfc * inv_d2 + 1.1283791671f * sa * e * inv_r;  // 2/sqrt(pi)
  }
  float fc = -qi * qj * g * inv_r;
  if (!core) fc *= pice;
  return fl + qq * fc;
}

// ------------------------------------------------------------------------------------------------
// Tile variant (dense systems: many atoms per cell).  One warp per home cell.  Every atom of a
// home cell walks the same candidate sequence -- the (2 nc + 1)^2 traversal rows of the home cell,
// each one or two contiguous ranges of the cell-ordered arrays -- so the warp streams that
// sequence once, 32 candidates per batch (one per lane), and classifies each batch against every
// atom of the cell in turn: two ballots (core, shell) per (atom, batch), the window tests done as
// single compares against exact thresholds.  In FP32 the compares are against the edges of the
// FP32 rounding bands around rs^2 and rc^2; the few pairs inside a band are classified again from
// the FP64 positions, so the classes -- and the RBL picks that count them -- are exactly the FP64
// path's.  The lane that owns an atom then turns its masks into
// picks -- every pice-th shell atom in traversal order, located with __fns from a running skip
// count -- and queues the selected pairs as packed ints.  When any queue is nearly full the warp
// evaluates all queues in lock step; with 16 or fewer atoms in the cell each queue is shared by
// 2, 4, ... lanes whose partial sums are then added in a fixed order.  An atom outside the box
// (its unclamped cell is not the home cell it is binned into) walks its own neighbourhood with
// the whole warp before the cell's batches, as the reference's locator does.
constexpr int kCellWarps = 4;    // home cells per block (kCellWarpsHost on the host side)
// resident blocks per SM the tile kernel is compiled for (bounds its registers per thread)
#ifndef RBMD_TILE_MIN_BLOCKS
#define RBMD_TILE_MIN_BLOCKS 5
#endif
constexpr int kTileQ = 48;       // queued pairs per atom between evaluations (a batch adds <= 32)
constexpr int kJsBits = 25;      // queue entry: sorted index | shift code << 25 | shell << 31
constexpr int kJsMask = (1 << kJsBits) - 1;
constexpr int kTileSp = 2;       // special partners per atom cached in shared memory (water: 2)
constexpr int kTileHist = 6;     // batches of candidates kept for the queued pairs

template <typename R> __device__ inline R cls_thr(const SysDev& s, int k);
template <> __device__ inline double cls_thr<double>(const SysDev& s, int k) { return s.cls_d[k]; }
template <> __device__ inline float cls_thr<float>(const SysDev& s, int k) { return s.cls_f[k]; }

// Squared distance of the tile kernel: FP64 with every product and sum rounded separately (the
// oracle's order); FP32 as two fused multiply-adds, the same expression in classification and
// evaluation so that both see the same value.
__device__ inline double tile_d2(double x, double y, double z) { return add_rn(add_rn(mul_rn(x, x), mul_rn(y, y)), mul_rn(z, z)); }
__device__ inline float tile_d2(float x, float y, float z) { return __fmaf_rn(z, z, __fmaf_rn(y, y, __fmul_rn(x, x))); }

// FP32 RBL classification against the band edges (SysDev::band), as two flags whose ballots
// carry three outcomes out of the hot loop: x alone = core, y alone = shell, both = banded (to be
// classified in FP64), neither = out (or the pair of an atom with itself).  Outside the bands the
// outcome equals the FP64 classification.  Each flag is one chain of compares (one predicate).
__device__ __forceinline__ void band_classify(float dd, float b0, float b1, float b2, float b3, bool& x, bool& y) {
  x = ((dd <= b1) | (dd >= b2)) & (dd <= b3) & (dd > 0.0001f);
  y = (dd >= b0) & (dd <= b3);
}

// Tile layout, FP32 RBL: the banded pairs of this lane's home atom (bits of amb, candidate lanes
// of the batch) classified from the FP64 positions; returns the corrected (core, shell) words.
// The candidates are identified from the batch's history row: queue entries (hist: sorted index |
// shift code) where the kernel keeps them, else atom ids with the shifted FP32 positions (hid, hp),
// from which the sorted index (rank) and the image of each dimension follow.  Runs for about one
// batch in fifty.
__device__ __forceinline__ uint2 tile_fix_banded(const SysDev& s, const int* hist, const int* hid, const float4* hp4,
                                              int si, unsigned amb, unsigned my_cm, unsigned my_sm) {
  if (amb) {
    const double4 hp = ldg4(&s.sx[si]);
    while (amb) {
      const int b = __ffs(amb) - 1;
      amb &= amb - 1;
      int js, m[3];
      if (hist) {
        const int ent = hist[b];
        js = ent & kJsMask;
        for (int k = 0; k < 3; ++k) m[k] = (((ent >> (kJsBits + 2 * k)) & 3) - 1) * s.dims[k];
      } else {
        js = __ldg(&s.rank[hid[b] & kJsMask]);
        const double4 pj = ldg4(&s.sx[js]);
        const float4 c = hp4[b];  // pj - shift, rounded to FP32
        const double sh[3] = {pj.x - (double)c.x, pj.y - (double)c.y, pj.z - (double)c.z};
        for (int k = 0; k < 3; ++k) m[k] = (int)rint(sh[k] / (s.d[k] * (double)s.dims[k])) * s.dims[k];
      }
      bool core, shell;
      classify_fp64(s, hp.x, hp.y, hp.z, js, m[0], m[1], m[2], true, core, shell);
      const unsigned bit = 1u << b;
      my_cm = core ? (my_cm | bit) : (my_cm & ~bit);
      my_sm = shell ? (my_sm | bit) : (my_sm & ~bit);
    }
  }
  return make_uint2(my_cm, my_sm);
}

// Picked shells of one batch: the set bits of sm at ranks r, r + pice, ... where r is the number
// of shells still to skip; r leaves as the skip count for the next batch.
__device__ inline unsigned pick_shells(unsigned sm, int pice, int& r) {
  if (pice == 1) return sm;
  const int ns = __popc(sm);
  unsigned pk = 0u;
  while (r < ns) {
    pk |= 1u << __fns(sm, 0u, r + 1);
    r += pice;
  }
  r -= ns;
  return pk;
}

// The same picks for pice = 2^lg without a loop: bit k of each shell's rank (the shells before it
// in the mask) is the exclusive prefix parity of the shells whose rank has bits 0..k-1 all set, so
// the shells of rank r = c (mod pice) are an AND of lg such parities; c becomes (c - shells) mod
// pice.  Every lane runs the same lg steps.
__device__ __forceinline__ unsigned prefix_parity_excl(unsigned m) {
  unsigned x = m << 1;
  x ^= x << 1;
  x ^= x << 2;
  x ^= x << 4;
  x ^= x << 8;
  x ^= x << 16;
  return x;
}
__device__ __forceinline__ unsigned pick_shells_pow2(unsigned sm, int lg, int& c) {
  unsigned pm = sm, carry = sm;
  for (int k = 0; k < lg; ++k) {
    const unsigned bit_k = prefix_parity_excl(carry);
    pm &= ((c >> k) & 1) ? bit_k : ~bit_k;
    carry &= bit_k;
  }
  c = (c - __popc(sm)) & ((1 << lg) - 1);
  return pm;
}

// Per-atom result of a pair pass: forces written (or the EAM embedding derivative); r9 leaves as
// the atom's nine reduction values.
template <int MODE>
__device__ inline void finish_atom(const SysDev& s, int i, double (&r9)[9]) {
  if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) {
    const double rho = r9[0];
    double p = rho * (1.0 / s.eam_drho) + 1.0;
    int m = (int)p;
    m = max(1, min(m, s.eam_nrho - 1));
    p -= m;
    p = fmin(p, 1.0);
    const double* c = eam_frho(s, s.meta[i].x) + 7 * m;
    if (MODE == kEAM_RHO) {
      s.eam_fp[i] = (c[0] * p + c[1]) * p + c[2];
    } else {
      const double fpv = (c[0] * p + c[1]) * p + c[2];
      double phi = ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
      if (rho > s.eam_rhomax) phi += fpv * (rho - s.eam_rhomax);
      r9[0] = phi;
    }
  } else if (MODE != kENERGY && MODE != kLIST) {
    s.f[i] = make_double4(r9[0], r9[1], r9[2], 0.0);
  }
}

// The nine per-atom values from the accumulators.
template <int MODE, bool F32, bool VIRIAL>
__device__ inline void acc_to_r9(const SysDev& s, const double (&c)[6], const PairAcc& a, double (&r9)[9]) {
#pragma unroll
  for (int k = 0; k < 9; ++k) r9[k] = 0.0;
  if (F32) {
    r9[0] = c[0];
    r9[1] = c[1];
    r9[2] = c[2];
    if (MODE == kCOUL_RBL) {
      r9[0] = r9[0] + s.qqr2e * c[3];
      r9[1] = r9[1] + s.qqr2e * c[4];
      r9[2] = r9[2] + s.qqr2e * c[5];
    }
    return;
  }
  r9[0] = a.f[0];
  r9[1] = a.f[1];
  r9[2] = a.f[2];
  if (MODE == kCOUL_RBL) {
    r9[0] = r9[0] + s.qqr2e * a.g[0];
    r9[1] = r9[1] + s.qqr2e * a.g[1];
    r9[2] = r9[2] + s.qqr2e * a.g[2];
  }
  if (VIRIAL) {
#pragma unroll
    for (int k = 0; k < 6; ++k) r9[3 + k] = a.vir[k];
  }
  if (MODE == kEAM_RHO || MODE == kEAM_ENERGY) r9[0] = a.rho;
  if (MODE == kEAM_ENERGY) r9[1] = a.e1;
  if (MODE == kENERGY) {
    r9[0] = a.e0;
    r9[1] = a.e1;
  }
}

__device__ inline void acc_zero(float (&ff)[6], PairAcc& a) {
#pragma unroll
  for (int k = 0; k < 6; ++k) ff[k] = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) a.f[k] = a.g[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) a.vir[k] = 0.0;
  a.rho = a.e0 = a.e1 = 0.0;
}

// Adds the accumulators of lanes (a, m), m = 0 .. k - 1 (lane = a + m nat), into lane (a, 0), in a
// fixed tree order.  The FP32 partials are widened to FP64 first.
template <bool F32>
__device__ inline void acc_combine(float (&ff)[6], PairAcc& a, double (&c)[6], int k, int nat) {
  const unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int j = 0; j < 6; ++j) c[j] = (double)ff[j];
  for (int off = k >> 1; off >= 1; off >>= 1) {
    const int d = off * nat;
    if (F32) {
#pragma unroll
      for (int j = 0; j < 6; ++j) c[j] += __shfl_down_sync(FULL, c[j], d);
    } else {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        a.f[j] += __shfl_down_sync(FULL, a.f[j], d);
        a.g[j] += __shfl_down_sync(FULL, a.g[j], d);
      }
#pragma unroll
      for (int j = 0; j < 6; ++j) a.vir[j] += __shfl_down_sync(FULL, a.vir[j], d);
      a.rho += __shfl_down_sync(FULL, a.rho, d);
      a.e0 += __shfl_down_sync(FULL, a.e0, d);
      a.e1 += __shfl_down_sync(FULL, a.e1, d);
    }
  }
}

// Sum over all 32 lanes (every lane gets the total), same fields as acc_combine.
template <bool F32>
__device__ inline void acc_warp_total(float (&ff)[6], PairAcc& a, double (&c)[6]) {
#pragma unroll
  for (int j = 0; j < 6; ++j) c[j] = warp_sum((double)ff[j]);
  if (!F32) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      a.f[j] = warp_sum(a.f[j]);
      a.g[j] = warp_sum(a.g[j]);
    }
#pragma unroll
    for (int j = 0; j < 6; ++j) a.vir[j] = warp_sum(a.vir[j]);
    a.rho = warp_sum(a.rho);
    a.e0 = warp_sum(a.e0);
    a.e1 = warp_sum(a.e1);
  }
}

// One atom whose position lies outside the box, walked by the whole warp over the (2 nc + 1)^3
// cells around its unclamped cell, each wrapped by a true modulo (ExecPointLocator::InWhichCell
// and PeriodicIndexOffset), candidates 32 at a time.  Selected pairs are evaluated in place into
// the lanes' accumulators (zero on entry); list mode writes the rows directly.
template <typename R, int MODE, bool SPECIAL, bool VIRIAL, bool NEAR = false>
__device__ void tile_stray(const SysDev& s, int si, int skip, int pice, bool rbl, const float* s_tab, int cap,
                           int* out_nc, int* out_ns, int* out_core, int* out_shell, float (&ff)[6],
                           PairAcc& acc) {
  using R4 = typename Vec4<R>::T;
  constexpr bool F32 = sizeof(R) == 4 && (MODE == kLJ_RBL || MODE == kCOUL_RBL);
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  const int4 mi = __ldg(&s.smeta[si]);
  const int i = mi.x, ti = mi.y, moli = mi.z;
  const double4 xd = ldg4(&s.sx[si]);
  const R4 p4 = load_sorted<R>(s, si);
  const double fpi = (MODE == kEAM_FORCE) ? s.eam_fp[i] : 0.0;
  int nsp = 0;
  const int* spi = nullptr;
  const double* spw = nullptr;
  if (SPECIAL) {
    const int b = s.sp_off[i];
    nsp = s.sp_off[i + 1] - b;
    spi = s.sp_ids + b;
    spw = s.sp_w + b;
  }
  const R t_rc = cls_thr<R>(s, 0), t_rs_hi = cls_thr<R>(s, 1), t_rs_lo = cls_thr<R>(s, 2);
  const R far = R(1e30);
  const float spice = (float)pice, fsa = (float)sqrt(s.alpha), falpha = (float)s.alpha;
  const int dx = s.dims[0], dy = s.dims[1], dz = s.dims[2];
  const int u0 = (int)((xd.x - s.lo[0]) / s.d[0]), u1 = (int)((xd.y - s.lo[1]) / s.d[1]);
  const int u2 = (int)((xd.z - s.lo[2]) / s.d[2]);
  const int nc = s.nc;
  int n_core = 0, n_shell = 0;
  for (int da = -nc; da <= nc; ++da)
    for (int db = -nc; db <= nc; ++db)
      for (int de = -nc; de <= nc; ++de) {
        const int n0 = u0 + da, n1 = u1 + db, n2 = u2 + de;
        const int w0 = ((n0 % dx) + dx) % dx, w1 = ((n1 % dy) + dy) % dy, w2 = ((n2 % dz) + dz) % dz;
        const R ox = (R)(s.d[0] * (double)(w0 - n0)), oy = (R)(s.d[1] * (double)(w1 - n1));
        const R oz = (R)(s.d[2] * (double)(w2 - n2));
        const int cell = w2 + dz * (w1 + dy * w0);
        const int cs = __ldg(&s.cell_start[cell]), ce = __ldg(&s.cell_start[cell + 1]);
        for (int k0 = cs; k0 < ce; k0 += 32) {
          const int kk = k0 + lane;
          R rx = far, ry = far, rz = far;
          if (kk < ce) {
            const R4 pj = load_sorted<R>(s, kk);
            rx = (pj.x - ox) - p4.x;
            ry = (pj.y - oy) - p4.y;
            rz = (pj.z - oz) - p4.z;
          }
          const R dd = tile_d2(rx, ry, rz);
          bool shell = rbl && dd >= t_rs_hi && dd <= t_rc;
          bool core = rbl ? (dd <= t_rs_lo && dd > R(0.0001)) : (dd <= t_rc && dd > R(0.0001));
          if constexpr (sizeof(R) == 4) {
            if (kk < ce && f32_banded(s, (float)dd))
              classify_fp64(s, xd.x, xd.y, xd.z, kk, w0 - n0, w1 - n1, w2 - n2, rbl, core, shell);
          }
          const unsigned cm = __ballot_sync(FULL, core), sm = __ballot_sync(FULL, shell);
          const unsigned pk = rbl ? pick_shells(sm, pice, skip) : 0u;
          const bool sel = ((cm | pk) >> lane) & 1u;
          if (MODE == kLIST) {
            if (sel) {
              const int id = __ldg(&s.smeta[kk]).x;
              if (core) {
                const int pos = n_core + __popc(cm & lanemask_lt(lane));
                if (pos < cap) out_core[(size_t)i * cap + pos] = id;
              } else {
                const int pos = n_shell + __popc(pk & lanemask_lt(lane));
                if (pos < cap) out_shell[(size_t)i * cap + pos] = id;
              }
            }
            n_core += __popc(cm);
            n_shell += __popc(pk);
          } else if (sel) {
            if (F32)
              eval_pair_f32<MODE, SPECIAL, NEAR>(s, moli, (float)xd.w, kk, core, (float)rx, (float)ry, (float)rz, ti, spi,
                                           spw, nsp, spice, (float)s.rc2, (float)s.rs2, fsa, falpha, s_tab,
                                           s.ntypes, (float)s.L[0], (float)s.L[1], (float)s.L[2], ff[0], ff[1],
                                           ff[2], ff[3], ff[4], ff[5]);
            else
              eval_pair<R, MODE, SPECIAL, VIRIAL, NEAR>(s, i, ti, moli, xd.w, fpi, kk, core, rx, ry, rz, spi, spw, nsp,
                                                  (R)pice, acc);
          }
        }
      }
  if (MODE == kLIST && lane == 0) {
    out_nc[i] = n_core;
    out_ns[i] = n_shell;
  }
}

template <typename R, int MODE, bool SPECIAL, bool VIRIAL, bool NEAR = false>
__global__ void __launch_bounds__(kCellWarps * 32, RBMD_TILE_MIN_BLOCKS)
k_pair_tile(const SysDev* __restrict__ S, const int2* __restrict__ work, int cap, int* out_nc, int* out_ns,
            int* out_core, int* out_shell, float4 band) {
  using R4 = typename Vec4<R>::T;
  constexpr bool F32 = sizeof(R) == 4 && (MODE == kLJ_RBL || MODE == kCOUL_RBL);
  constexpr bool QUEUE = MODE != kLIST;
  // per-atom pair queues (column = atom of the chunk); an entry is (history slot << 5 | lane) with
  // bit 15 set for a shell pair
  __shared__ unsigned short s_q[kCellWarps][kTileQ][32];
  __shared__ R4 s_pi[kCellWarps][32];          // chunk atom positions (far away for box-outside atoms)
  // FP32 path: per chunk atom its type, molecule, special count and first special slot; the
  // concatenated-queue offsets; and its force accumulator
  __shared__ int4 s_ainfo[kCellWarps][32];
  __shared__ int s_off[kCellWarps][33];
  __shared__ float s_acc[kCellWarps][32][3];
  __shared__ int s_hist[kCellWarps][kTileHist][32];  // packed candidates of the batches since the
                                                     // last evaluation; queue entries index it
  // FP32 path: the same candidates' shifted positions, charges and (atom id | type << 25), so
  // that the evaluation reads shared memory only
  __shared__ float4 s_hp[kCellWarps][kTileHist][32];
  __shared__ int s_hid[kCellWarps][kTileHist][32];
  __shared__ int s_sa[kCellWarps][64];         // segment first sorted index
  __shared__ int s_sb[kCellWarps][64];         // segment begin in the flattened sequence
  __shared__ int s_se[kCellWarps][64];         // segment end in the flattened sequence
  __shared__ int s_code[kCellWarps][64];       // segment shift code (<< kJsBits)
  __shared__ R s_shift[3][3];                  // per dimension: d (w - n) for w - n = -dims, 0, +dims
  __shared__ float s_tab[2 * kMaxF32Types * kMaxF32Types];
  __shared__ double s_red[kCellWarps][9];
  __shared__ int s_spi[kCellWarps][kTileSp][32];  // first special partners of each chunk atom
  __shared__ float s_spw[kCellWarps][kTileSp][32];

  const int2 wk = work[blockIdx.x];
  const SysDev& s = S[wk.x];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  const int dx = s.dims[0], dy = s.dims[1], dz = s.dims[2];
  const int ntypes = s.ntypes;
  if (threadIdx.x < 9) {
    const int dim = threadIdx.x / 3, t = threadIdx.x % 3;
    s_shift[dim][t] = (R)(s.d[dim] * (double)((t - 1) * s.dims[dim]));
  }
  if (F32) {
    for (int t = threadIdx.x; t < ntypes * ntypes && t < kMaxF32Types * kMaxF32Types; t += blockDim.x) {
      const int a = t / ntypes, b = t % ntypes;
      const double sg = (s.sig[a] + s.sig[b]) / 2;
      s_tab[2 * t] = (float)(-24.0 * sqrt(s.eps[a] * s.eps[b]));
      s_tab[2 * t + 1] = (float)(sg * sg * sg * sg * sg * sg);
    }
  }
  __syncthreads();

  const bool rbl = (MODE == kLJ_RBL || MODE == kCOUL_RBL || MODE == kLIST ||
                    ((MODE == kEAM_RHO || MODE == kEAM_FORCE) && s.neigh == RBMD_NEIGH_RBL));
  const int pice = rbl ? s.pice : 1;
  const R t_rc = cls_thr<R>(s, 0), t_rs_hi = cls_thr<R>(s, 1), t_rs_lo = cls_thr<R>(s, 2);
  // FP32 band edges: one set for the whole launch, the union of its systems' bands (a batch's
  // systems share rc and rs)
  const float b0 = band.x, b1 = band.y, b2 = band.z, b3 = band.w;
  const float spice = (float)pice, fsa = s.fsa, falpha_l2 = s.falpha_l2, fqq = s.fqq;
  const float* const ntab = s.near_tab;  // RBMD_NEAR_TABLE: the reference's G table
  const R far = R(1e30);
  const int nc = s.nc, side = 2 * nc + 1, nrows = side * side;
  if (lane < 9) s_red[wid][lane] = 0.0;  // per-warp reduction values, added in a fixed order
  // lane 0 adds the warp total of v (owner lanes' values, in lane order) to s_red[wid][k]
  auto add_red = [&](const double (&v)[9], bool take) {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double w = warp_sum(take ? v[k] : 0.0);
      if (lane == 0) s_red[wid][k] += w;
    }
  };

  const int hc = wk.y + wid;
  if (hc < s.ncell) {
    const int hx = hc / (dz * dy), hy = (hc / dz) % dy, hz = hc % dz;
    const int hs = __ldg(&s.cell_start[hc]), he = __ldg(&s.cell_start[hc + 1]);
    for (int g0 = hs; g0 < he; g0 += 32) {
      const int nat = min(32, he - g0);
      int k = 1;
      while (2 * k * nat <= 32) k *= 2;
      const int a = lane % nat, m = lane / nat;
      const bool member = m < k;  // lane (a, m) helps evaluate the queue of atom a
      const bool owner = lane < nat;
      const int si = g0 + a;
      const int4 mi = __ldg(&s.smeta[si]);
      const int i = mi.x, ti = mi.y, moli = mi.z;
      const R4 p4 = load_sorted<R>(s, si);
      const R pix = p4.x, piy = p4.y, piz = p4.z;
      const double4 xd = ldg4(&s.sx[si]);
      const double qi = xd.w;
      const bool stray = (int)((xd.x - s.lo[0]) / s.d[0]) != hx || (int)((xd.y - s.lo[1]) / s.d[1]) != hy ||
                         (int)((xd.z - s.lo[2]) / s.d[2]) != hz;
      const double fpi = (MODE == kEAM_FORCE) ? s.eam_fp[i] : 0.0;
      int nsp = 0;
      const int* spi = nullptr;
      const double* spw = nullptr;
      if (SPECIAL) {
        const int b = s.sp_off[i];
        nsp = s.sp_off[i + 1] - b;
        spi = s.sp_ids + b;
        spw = s.sp_w + b;
      }
      int skip = 0;  // shells still to skip before the next pick (owner lanes)
      if (rbl && s.rbl_mode == RBMD_RBL_PHILOX && pice > 1) {
        uint32_t o[4];
        philox4x32_10((uint32_t)i, 0u, (uint32_t)s.st->step, kTagRblOffset, s.seed_lo, s.seed_hi, o);
        const int nm = (int)(o[0] % (uint32_t)pice);
        skip = nm == 0 ? 0 : pice - nm;
      }
      __syncwarp();  // the previous chunk has finished with s_pi
      if (owner) {
        R4 q = p4;
        if (stray) q.x = q.y = q.z = far;
        s_pi[wid][lane] = q;
        if constexpr (F32) {
          s_ainfo[wid][lane] = make_int4(ti, moli, nsp, SPECIAL ? s.sp_off[i] : 0);
          s_acc[wid][lane][0] = s_acc[wid][lane][1] = s_acc[wid][lane][2] = 0.0f;
        }
        if (SPECIAL && nsp <= kTileSp)
          for (int t = 0; t < nsp; ++t) {
            s_spi[wid][t][lane] = spi[t];
            s_spw[wid][t][lane] = (float)spw[t];
          }
      }
      float ff[6];
      PairAcc acc;
      acc_zero(ff, acc);
      double cmb[6];
      int qc = 0, n_core = 0, n_shell = 0;
      int nh = 0;  // batches in the history ring since the last evaluation (warp-uniform)

      // ---- atoms outside the box: the whole warp walks each one's own neighbourhood
      unsigned strays = __ballot_sync(FULL, owner && stray);
      while (strays) {
        const int as = __ffs(strays) - 1;
        strays &= strays - 1;
        const int sk = __shfl_sync(FULL, skip, as);
        tile_stray<R, MODE, SPECIAL, VIRIAL, NEAR>(s, g0 + as, sk, pice, rbl, s_tab, cap, out_nc, out_ns, out_core,
                                             out_shell, ff, acc);
        if (MODE != kLIST) {
          acc_warp_total<F32>(ff, acc, cmb);
          double r9[9];
          acc_to_r9<MODE, F32, VIRIAL>(s, cmb, acc, r9);
          if (lane == as) finish_atom<MODE>(s, i, r9);
          if (lane == 0) {  // r9 is the same in every lane (a warp total)
#pragma unroll
            for (int q = 0; q < 9; ++q) s_red[wid][q] += r9[q];
          }
          acc_zero(ff, acc);
        }
      }

      auto flush = [&]() {
        const int qa = __shfl_sync(FULL, qc, a);
        const int maxq = __reduce_max_sync(FULL, member ? qa : 0);
        const int rounds = (maxq + k - 1) / k;
        if constexpr (F32) {
          // all queues concatenated (atom a's entries at [s_off[a], s_off[a + 1])) and evaluated 32
          // at a time with every lane busy; each round's per-atom runs are summed by a segmented
          // warp scan and added to the atoms' accumulators by the runs' last lanes, so every
          // atom's sum is formed in a fixed order
          const int incl = warp_incl_scan(owner ? qc : 0, lane);
          if (lane < nat) s_off[wid][lane + 1] = incl;
          if (lane == 0) s_off[wid][0] = 0;
          const int total = __shfl_sync(FULL, incl, 31);
          __syncwarp();
          int ca = 0;  // this lane's atom cursor (monotone over the rounds)
          for (int e0 = 0; e0 < total; e0 += 32) {
            const int e = e0 + lane;
            const bool v = e < total;
            float fx = 0.0f, fy = 0.0f, fz = 0.0f;
            int key = 32 + lane;  // never equal to an atom index
            if (v) {
              while (e >= s_off[wid][ca + 1]) ++ca;
              key = ca;
              const unsigned h = s_q[wid][e - s_off[wid][ca]][ca];
              const float4 pj = s_hp[wid][(h >> 5) & 0x3ff][h & 31];
              const int idt = s_hid[wid][(h >> 5) & 0x3ff][h & 31];
              const float4 pa = s_pi[wid][ca];
              const int4 ai = s_ainfo[wid][ca];
              const float rx = pj.x - pa.x, ry = pj.y - pa.y, rz = pj.z - pa.z;
              const int idj = idt & kJsMask, tj = idt >> kJsBits;
              float w = 1.0f;
              if (SPECIAL) {
                if (ai.z <= kTileSp) {
                  for (int t2 = 0; t2 < ai.z; ++t2)
                    if (s_spi[wid][t2][ca] == idj) w = s_spw[wid][t2][ca];
                } else {
                  for (int t2 = 0; t2 < ai.z; ++t2)
                    if (__ldg(&s.sp_ids[ai.w + t2]) == idj) w = (float)__ldg(&s.sp_w[ai.w + t2]);
                }
              }
              bool skip_pair = false;
              if constexpr (MODE == kLJ_RBL) {
                const int ej = s_hist[wid][(h >> 5) & 0x3ff][h & 31];
                skip_pair = ai.y == __ldg(&s.smeta[ej & kJsMask]).z;  // same molecule
              }
              if (!skip_pair) {
                const float d2 = tile_d2(rx, ry, rz);
                const int tp = ai.x * ntypes + tj;
                const float f = tile_pair_f32_lj<MODE, NEAR>((h & 0x8000u) == 0u, d2, pa.w, pj.w, s_tab[2 * tp],
                                                             s_tab[2 * tp + 1], w, spice, fsa, falpha_l2, fqq, ntab);
                fx = f * rx;
                fy = f * ry;
                fz = f * rz;
              }
            }
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
              const float tx = __shfl_up_sync(FULL, fx, d), ty = __shfl_up_sync(FULL, fy, d);
              const float tz = __shfl_up_sync(FULL, fz, d);
              const int tk = __shfl_up_sync(FULL, key, d);
              if (lane >= d && tk == key) {
                fx += tx;
                fy += ty;
                fz += tz;
              }
            }
            const int nk = __shfl_down_sync(FULL, key, 1);
            if (v && (lane == 31 || nk != key)) {
              s_acc[wid][key][0] += fx;
              s_acc[wid][key][1] += fy;
              s_acc[wid][key][2] += fz;
            }
          }
        } else {
          for (int t = 0; t < rounds; ++t) {
            const int q = t * k + m;
            if (member && q < qa) {
              const int h = s_q[wid][q][a];
              const int e = s_hist[wid][(h >> 5) & 0x3ff][h & 31] | (int)((unsigned)(h & 0x8000) << 16);
              const int js = e & kJsMask;
              const bool core = e >= 0;
              const R4 pj = load_sorted<R>(s, js);
              const R rx = (pj.x - s_shift[0][(e >> kJsBits) & 3]) - pix;
              const R ry = (pj.y - s_shift[1][(e >> (kJsBits + 2)) & 3]) - piy;
              const R rz = (pj.z - s_shift[2][(e >> (kJsBits + 4)) & 3]) - piz;
              eval_pair<R, MODE, SPECIAL, VIRIAL, NEAR>(s, i, ti, moli, qi, fpi, js, core, rx, ry, rz, spi, spw, nsp,
                                                  (R)pice, acc);
            }
          }
        }
        qc = 0;
        nh = 0;
        __syncwarp();
      };

      // ---- the home cell's candidate sequence, traversal rows in groups (one per lane).  A row's
      // unwrapped z cells hz - nc .. hz + nc form one range, two around the periodic wrap, or, when
      // the box holds fewer than 2 nc + 1 cells in z (but more than nc), three: below the box
      // (image -L), inside, above (image +L); the segment table holds 64, so groups are 32 rows,
      // or 21 rows when a row can have three ranges.
      const int group = dz >= side ? 32 : 21;
      for (int r0 = 0; r0 < nrows; r0 += group) {
        const int r = r0 + lane;
        int nseg = 0, cnt = 0, sa0 = 0, sa1 = 0, sa2 = 0, n0c = 0, n1c = 0, n2c = 0, cxy = 0;
        bool below = false, above = false;
        if (lane < group && r < nrows) {
          const int da = r / side - nc, db = r % side - nc;
          const int n0 = hx + da, n1 = hy + db;  // the home cell is inside the grid and nc < dims
          const int w0 = n0 < 0 ? n0 + dx : (n0 >= dx ? n0 - dx : n0);
          const int w1 = n1 < 0 ? n1 + dy : (n1 >= dy ? n1 - dy : n1);
          const int t0 = n0 < 0 ? 2 : (n0 >= dx ? 0 : 1), t1 = n1 < 0 ? 2 : (n1 >= dy ? 0 : 1);
          cxy = (t0 << kJsBits) | (t1 << (kJsBits + 2));
          const int base = dz * (w1 + dy * w0);
          const int z0 = hz - nc, z1 = hz + nc;  // -dz < z0 <= hz <= z1 < 2 dz
          below = z0 < 0;
          above = z1 >= dz;
          if (below) {  // cells z0 + dz .. dz - 1
            sa0 = __ldg(&s.cell_start[base + z0 + dz]);
            n0c = __ldg(&s.cell_start[base + dz]) - sa0;
          }
          {  // cells max(z0, 0) .. min(z1, dz - 1)
            const int za = below ? 0 : z0, zb = above ? dz - 1 : z1;
            sa1 = __ldg(&s.cell_start[base + za]);
            n1c = __ldg(&s.cell_start[base + zb + 1]) - sa1;
          }
          if (above) {  // cells 0 .. z1 - dz
            sa2 = __ldg(&s.cell_start[base]);
            n2c = __ldg(&s.cell_start[base + z1 - dz + 1]) - sa2;
          }
          nseg = 1 + (below ? 1 : 0) + (above ? 1 : 0);
          cnt = n0c + n1c + n2c;
        }
        const int seg_incl = warp_incl_scan(nseg, lane);
        const int cnt_incl = warp_incl_scan(cnt, lane);
        const int total = __shfl_sync(FULL, cnt_incl, 31);
        if (nseg) {
          int slot = seg_incl - nseg;
          const int beg = cnt_incl - cnt;
          if (below) {
            s_sa[wid][slot] = sa0;
            s_sb[wid][slot] = beg;
            s_se[wid][slot] = beg + n0c;
            s_code[wid][slot] = cxy | (2 << (kJsBits + 4));
            ++slot;
          }
          s_sa[wid][slot] = sa1;
          s_sb[wid][slot] = beg + n0c;
          s_se[wid][slot] = beg + n0c + n1c;
          s_code[wid][slot] = cxy | (1 << (kJsBits + 4));
          ++slot;
          if (above) {
            s_sa[wid][slot] = sa2;
            s_sb[wid][slot] = beg + n0c + n1c;
            s_se[wid][slot] = beg + n0c + n1c + n2c;
            s_code[wid][slot] = cxy | (0 << (kJsBits + 4));
          }
        }
        __syncwarp();
        // candidate p of the flattened sequence: the load of batch b + 1 is issued before batch b
        // is classified
        int seg = 0, ent_n = 0, idt_n = 0;
        bool val_n = false;
        R4 pj_n;
        pj_n.x = pj_n.y = pj_n.z = pj_n.w = R(0);
        auto fetch = [&](int p) {
          val_n = p < total;
          if (val_n) {
            while (p >= s_se[wid][seg]) ++seg;
            const int js = s_sa[wid][seg] + (p - s_sb[wid][seg]);
            ent_n = js | s_code[wid][seg];
            pj_n = load_sorted<R>(s, js);
            if (F32) {
              const int4 mj = __ldg(&s.smeta[js]);
              idt_n = mj.x | (mj.y << kJsBits);
            }
          }
        };
        fetch(lane);
        for (int base = 0; base < total; base += 32) {
          const R4 pj = pj_n;
          const int ent = ent_n, idt = idt_n;
          const bool val = val_n;
          // FP32: the next batch is fetched after the classification loop, which then runs with
          // fewer live registers; FP64 fetches it here
          if (!F32 && base + 32 < total) fetch(base + 32 + lane);
          R cx = far, cy = far, cz = far;
          if (val) {
            cx = pj.x - s_shift[0][(ent >> kJsBits) & 3];
            cy = pj.y - s_shift[1][(ent >> (kJsBits + 2)) & 3];
            cz = pj.z - s_shift[2][(ent >> (kJsBits + 4)) & 3];
          }
          if constexpr (!F32 || MODE == kLJ_RBL) s_hist[wid][nh][lane] = val ? ent : 0;
          if (F32) {
            s_hp[wid][nh][lane] = make_float4((float)cx, (float)cy, (float)cz, (float)pj.w);
            s_hid[wid][nh][lane] = idt;
          }
          // every atom of the chunk against the batch: two ballots each, kept by the atom's lane
          unsigned my_cm = 0u, my_sm = 0u;
          // FP32 RBL (the LJ / Coulomb modes, where rbl is known at compile time, and EAM over RBL):
          // the band edges are the thresholds; banded pairs come out with both bits set and are
          // classified again from the FP64 positions (rare)
          constexpr bool kBandOnly = F32;  // no other classification compiled in
          if (kBandOnly || (sizeof(R) == 4 && rbl)) {
            for (int ii = 0; ii < nat; ++ii) {
              const R4 q = s_pi[wid][ii];
              const float dd = tile_d2((float)cx - (float)q.x, (float)cy - (float)q.y, (float)cz - (float)q.z);
              bool core, shell;
              band_classify(dd, b0, b1, b2, b3, core, shell);
              const unsigned cm = __ballot_sync(FULL, core);
              const unsigned sm = __ballot_sync(FULL, shell);
              if (lane == ii) {
                my_cm = cm;
                my_sm = sm;
              }
            }
            const unsigned amb = my_cm & my_sm;  // banded candidates of this lane's home atom
            my_cm &= ~amb;
            my_sm &= ~amb;
            if (__any_sync(FULL, amb != 0u)) {
              const uint2 r = (F32 && MODE != kLJ_RBL)
                                  ? tile_fix_banded(s, nullptr, &s_hid[wid][nh][0], &s_hp[wid][nh][0], g0 + lane, amb,
                                                    my_cm, my_sm)
                                  : tile_fix_banded(s, &s_hist[wid][nh][0], nullptr, nullptr, g0 + lane, amb, my_cm, my_sm);
              my_cm = r.x;
              my_sm = r.y;
            }
          }
          if constexpr (!kBandOnly) if (!(sizeof(R) == 4 && rbl)) {
            for (int ii = 0; ii < nat; ++ii) {
              const R4 q = s_pi[wid][ii];
              const R rx = cx - q.x, ry = cy - q.y, rz = cz - q.z;
              const R dd = tile_d2(rx, ry, rz);
              const bool shell = rbl && dd >= t_rs_hi && dd <= t_rc;
              const bool core = rbl ? (dd <= t_rs_lo && dd > R(0.0001)) : (dd <= t_rc && dd > R(0.0001));
              const unsigned cm = __ballot_sync(FULL, core);
              const unsigned sm = rbl ? __ballot_sync(FULL, shell) : 0u;
              if (lane == ii) {
                my_cm = cm;
                my_sm = sm;
              }
            }
          }
          if (F32 && base + 32 < total) fetch(base + 32 + lane);
          if (!owner || stray) my_cm = my_sm = 0u;
          // picks among this atom's shells (every pice-th in traversal order, after `skip` more),
          // by a predicated walk over the set bits: no data-dependent branches
          unsigned pk = my_sm;
          if (rbl && pice > 1) {
            unsigned x = my_sm;
            int c = skip;
            pk = 0u;
            const int steps = __reduce_max_sync(FULL, __popc(x));
            for (int t = 0; t < steps; ++t) {
              const unsigned low = x & (0u - x);
              pk |= (c == 0) ? low : 0u;
              c = (low == 0u) ? c : (c == 0 ? pice - 1 : c - 1);
              x ^= low;
            }
            skip = c;
          }
          // the selected pairs, in traversal order, into the atom's queue
          unsigned sel = my_cm | pk;
          const int steps2 = __reduce_max_sync(FULL, __popc(sel));
          for (int t = 0; t < steps2; ++t) {
            const unsigned low = sel & (0u - sel);
            sel ^= low;
            if (low) {
              const int b = 31 - __clz(low);
              const bool sh = (pk & low) != 0u;
              if constexpr (MODE == kLIST) {
                const int id = __ldg(&s.smeta[s_hist[wid][nh][b] & kJsMask]).x;
                if (!sh) {
                  if (n_core < cap) out_core[(size_t)i * cap + n_core] = id;
                  ++n_core;
                } else {
                  if (n_shell < cap) out_shell[(size_t)i * cap + n_shell] = id;
                  ++n_shell;
                }
              } else {
                s_q[wid][qc][lane] = (unsigned short)(((nh << 5) | b) | (sh ? 0x8000 : 0));
                ++qc;
              }
            }
          }
          __syncwarp();  // the history and the queues are read before they are written again
          ++nh;
          if (QUEUE) {
            if (__any_sync(FULL, qc > kTileQ - 32) || nh == kTileHist) flush();
          } else if (nh == kTileHist) {
            nh = 0;
          }
        }
        __syncwarp();  // segment table reused by the next row group
      }

      if (MODE == kLIST) {
        if (owner && !stray) {
          out_nc[i] = n_core;
          out_ns[i] = n_shell;
        }
        continue;
      }
      flush();
      double r9[9];
      if constexpr (F32) {
#pragma unroll
        for (int q = 0; q < 9; ++q) r9[q] = 0.0;
        if (owner) {  // Coulomb already scaled by qqr2e inside the pair factor
          r9[0] = (double)s_acc[wid][lane][0];
          r9[1] = (double)s_acc[wid][lane][1];
          r9[2] = (double)s_acc[wid][lane][2];
        }
      } else {
        acc_combine<F32>(ff, acc, cmb, k, nat);
        acc_to_r9<MODE, F32, VIRIAL>(s, cmb, acc, r9);
      }
      if (owner && !stray) finish_atom<MODE>(s, i, r9);
      add_red(r9, owner && !stray);
    }
  }
  if (MODE == kLIST || MODE == kEAM_RHO) return;
  const bool need_red = (MODE == kLJ_RBL || MODE == kCOUL_RBL || MODE == kENERGY ||
                         MODE == kEAM_ENERGY || VIRIAL ||
                         (MODE == kEAM_FORCE && s.neigh == RBMD_NEIGH_RBL));
  if (!need_red) return;
  __syncthreads();
  const int blk = wk.y / kCellWarps;
  if (threadIdx.x < 9) {
    double t = 0.0;
    for (int w = 0; w < kCellWarps; ++w) t += s_red[w][threadIdx.x];
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
        if (k < 3) s.st->fmean[k] = (MODE == kLJ_VERLET || MODE == kCOUL_VERLET) ? 0.0 : t / s.n;
        if (k >= 3 && VIRIAL) s.st->virial[k - 3] = t;
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Column variant (mixed-precision RBL forces: LJ/CUT and LJ + real-space Coulomb).  One warp per
// column of home cells -- fixed x and y cell, all z -- whose atoms are contiguous in the cell-ordered
// arrays (cells are numbered z fastest), taken 32 at a time: one lane per home atom.  The chunk's
// atoms sit in a few consecutive z cells, so for a traversal row (x and y cell offset) their
// candidate windows -- the row's z cells from the atom's own cell - nc to + nc -- are overlapping
// sub-ranges of one contiguous union, which the warp stages once in shared memory, shifted into
// the home frame.  Each lane then walks its own window in lock step with the others (step t: every
// lane reads entry t of its own window), in blocks of 32 steps: a step is one shared load, the FP32
// squared distance and the band compares of the exact classification, setting bit t of a core and
// a shell mask -- no ballots, no cross-lane traffic and no bookkeeping.  Once per block the masks
// are cut to the lane's own window (the lanes step together), the banded candidates (both bits)
// are classified again in FP64, and the RBL picks -- every pice-th shell in traversal order -- are
// taken from the shell mask.  A lane's window is trimmed to the z cells that can hold an atom
// within rc of it (an x/y gap to the row's column of g leaves a z half-width sqrt(rc^2 - g^2));
// cells dropped that way hold no core or shell atom, so the shell ranks, and the RBL picks, stay
// exactly those of the full traversal.  The selected candidates of up to kColQ steps are evaluated
// by their own lane from the masks, in traversal order, so an atom's force is summed in a fixed
// order by one lane.  An atom outside its binned cell (SHAKE moves atoms after binning, and atoms
// may lie outside the box) walks its own neighbourhood with the whole warp (tile_stray, as in the
// tile kernel), in a pass of its own before the column kernel (k_pair_col_strays): its force is
// written there, and the column kernel only reads it back for the RBL mean, so that the stray
// walk's code does not share the instruction cache with the walk and the evaluation.
// The kernel is persistent: one grid of resident blocks, each warp taking the batch's columns one at
// a time from a work counter, longest columns first, so no warp waits for another and the launch's
// tail is short columns.  The RBL mean force is summed per column and the system's last column
// adds the partials in column order: the result does not depend on which warp took which column.
constexpr int kColWarps = 4;     // warps per block
constexpr int kColStage = 256;   // staged candidates per warp
constexpr int kColQ = kColStage;  // the most steps between evaluations: a staged tile
constexpr int kColQW = kColQ / 32;  // 32-step blocks between evaluations
constexpr float kColFar = 1e30f;
// resident blocks per SM: 4 (128 registers per thread) ran the saline stream's column launch in
// 34.2 ms against 36.1 ms at 5 (96 registers, twice the local-memory traffic of spills)
#ifndef RBMD_COL_MIN_BLOCKS
#define RBMD_COL_MIN_BLOCKS 4
#endif

// Rare paths of the column kernel, kept out of line so that their registers do not weigh on the
// walk: the FP64 classification of a banded pair (bit 0 core, bit 1 shell) ...
__device__ __noinline__ unsigned col_classify_fp64(const SysDev* __restrict__ sp, int si, int js, int mx, int my,
                                                   int mz) {
  const SysDev& s = *sp;
  const double4 xd = ldg4(&s.sx[si]);
  bool core, shell;
  classify_fp64(s, xd.x, xd.y, xd.z, js, mx, my, mz, true, core, shell);
  return (core ? 1u : 0u) | (shell ? 2u : 0u);
}

// Whether the atom at sorted index si, binned into home column (hx, hy) at z cell zl, lies outside
// that cell: the unclamped cell of its FP64 position (ExecPointLocator::InWhichCell) is another.
__device__ inline bool col_is_stray(const SysDev& s, int si, int hx, int hy, int zl) {
  const double4 xd = ldg4(&s.sx[si]);
  return (int)((xd.x - s.lo[0]) / s.d[0]) != hx || (int)((xd.y - s.lo[1]) / s.d[1]) != hy ||
         (int)((xd.z - s.lo[2]) / s.d[2]) != zl;
}

// The first shell rank to pick of atom i (RBL Philox offset mode; 0 in stride mode): the count of
// shells still to skip before its first pick.
__device__ inline int col_first_skip(const SysDev& s, int i, int pice) {
  if (s.rbl_mode != RBMD_RBL_PHILOX || pice <= 1) return 0;
  uint32_t o[4];
  philox4x32_10((uint32_t)i, 0u, (uint32_t)s.st->step, kTagRblOffset, s.seed_lo, s.seed_hi, o);
  const int nm = (int)(o[0] % (uint32_t)pice);
  return nm == 0 ? 0 : pice - nm;
}

// The stray atoms of the batch's columns, before the column kernel: each is walked by the whole
// warp over its own neighbourhood and its force written (finish_atom), where the column kernel
// reads it back.  Warps take columns from a work counter (ctr[0]; ctr[1] counts finished warps, and
// the last one resets both), as the column kernel does.
// resident blocks per SM the stray pass is compiled for: its walks wait on dependent loads, so it
// runs more warps per SM than the column kernel, at the price of a few spilled registers (on the
// saline stream 25.79 ms for both pair launches of a step, against 25.83 ms at the column kernel's
// 4 blocks and 25.76 ms at 8)
#ifndef RBMD_STRAY_MIN_BLOCKS
#define RBMD_STRAY_MIN_BLOCKS 6
#endif

template <int MODE, bool SPECIAL, bool NEAR>
__global__ void __launch_bounds__(kColWarps * 32, RBMD_STRAY_MIN_BLOCKS)
k_pair_col_strays(const SysDev* __restrict__ S, const int2* __restrict__ work, int nwork, unsigned* __restrict__ ctr) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  for (;;) {
    int wi = 0;
    if (lane == 0) wi = (int)atomicAdd(&ctr[0], 1u);
    wi = __shfl_sync(FULL, wi, 0);
    if (wi >= nwork) break;
    const int2 wk = __ldg(&work[wi]);
    const SysDev& s = S[wk.x];
    const int dy = s.dims[1], dz = s.dims[2];
    const int hx = wk.y / dy, hy = wk.y % dy;
    const int cbase = dz * (hy + dy * hx);
    const int a0 = __ldg(&s.cell_start[cbase]), a1 = __ldg(&s.cell_start[cbase + dz]);
    for (int g0 = a0; g0 < a1; g0 += 32) {
      const int si = g0 + lane;
      int i = 0, c = 0;
      bool stray = false;
      if (si < a1) {
        i = __ldg(&s.smeta[si]).x;
        stray = col_is_stray(s, si, hx, hy, __ldg(&s.cell_of_atom[i]) - cbase);
        if (stray) c = col_first_skip(s, i, s.pice);
      }
      for (unsigned m = __ballot_sync(FULL, stray); m; m &= m - 1) {
        const int as = __ffs(m) - 1;
        const int sk = __shfl_sync(FULL, c, as);
        float ff[6];
        PairAcc acc;
        acc_zero(ff, acc);
        tile_stray<float, MODE, SPECIAL, false, NEAR>(s, g0 + as, sk, s.pice, true, (const float*)s.ljf, 0, nullptr,
                                                      nullptr, nullptr, nullptr, ff, acc);
        double cmb[6], r9[9];
        acc_warp_total<true>(ff, acc, cmb);
        acc_to_r9<MODE, true, false>(s, cmb, acc, r9);
        if (lane == as) finish_atom<MODE>(s, i, r9);
      }
    }
  }
  if (lane == 0 && atomicAdd(&ctr[1], 1u) == gridDim.x * (unsigned)kColWarps - 1u) {
    ctr[0] = 0u;
    ctr[1] = 0u;
  }
}

template <int MODE, bool SPECIAL, bool NEAR>
__global__ void __launch_bounds__(kColWarps * 32, RBMD_COL_MIN_BLOCKS)
k_pair_col(const SysDev* __restrict__ S, const int2* __restrict__ work, int nwork, unsigned* __restrict__ ctr,
           float4 band) {
  static_assert(MODE == kLJ_RBL || MODE == kCOUL_RBL, "column layout: FP32 RBL forces only");
  static_assert(!NEAR || MODE == kCOUL_RBL, "the near-Coulomb table applies to the Coulomb mode");
  static_assert(kColQ % 32 == 0 && kColStage % 32 == 0, "the walk runs in blocks of 32 steps");
  __shared__ float4 s_c[kColWarps][kColStage];      // candidate position - image shift, charge
  __shared__ int s_id[kColWarps][kColStage];        // atom id (LJ/CUT: molecule) | type << kJsBits
  // per lane and 32-step block since the last evaluation, bit t for step t: the selected candidates
  // (core, or a picked shell) and the picked shells among them
  __shared__ unsigned s_sel[kColWarps][kColQW][32];
  __shared__ unsigned s_pk[kColWarps][kColQW][32];
  // per lane (home atom): what the evaluation needs, kept out of registers during the walk
  __shared__ int4 s_ai[kColWarps][32];    // type, molecule, special partners, first special slot
  __shared__ int2 s_sp[kColWarps][32];    // first two special partners
  __shared__ float2 s_sw[kColWarps][32];  // and their weights
  __shared__ float4 s_f[kColWarps][32];   // force accumulated so far (x, y, z), charge in w
  __shared__ float s_shift[kColWarps][3][3];  // per dimension: d (w - n) for w - n = -dims, 0, +dims

  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  // FP32 band edges of the launch (the union of its systems' bands; a batch shares rc and rs)
  const float b0 = band.x, b1 = band.y, b2 = band.z, b3 = band.w;
  int cur = -1;  // slot of the system whose image shifts s_shift holds
  for (;;) {
    int wi = 0;
    if (lane == 0) wi = (int)atomicAdd(&ctr[0], 1u);
    wi = __shfl_sync(FULL, wi, 0);
    if (wi >= nwork) break;
    const int2 wk = __ldg(&work[wi]);
    const SysDev& s = S[wk.x];
    const int dx = s.dims[0], dy = s.dims[1], dz = s.dims[2];
    const int ntypes = s.ntypes;
    if (wk.x != cur) {
      cur = wk.x;
      __syncwarp();  // the previous column's reads are done
      if (lane < 9) {
        const int dim = lane / 3, t = lane % 3;
        s_shift[wid][dim][t] = (float)(s.d[dim] * (double)((t - 1) * s.dims[dim]));
      }
      __syncwarp();
    }
    const int pice = s.pice;
    const int lgp = (pice & (pice - 1)) == 0 ? __ffs(pice) - 1 : -1;  // log2 pice, -1 if not a power of 2
    const int nc = s.nc, side = 2 * nc + 1, nrows = side * side;
    const float fdx = (float)s.d[0], fdy = (float)s.d[1], fdz = (float)s.d[2];
    const float frc2 = (float)s.rc2;
    // trimming margins: 1e-3 of a cell (far above the FP32 rounding of the coordinates involved) plus
    // the farthest an atom lay outside its binned cell (atoms given outside the box) and the largest
    // distance SHAKE moved an atom since the cell list was built; cells of atoms it wrapped across
    // the box are never trimmed, and beyond kMaxMigrated of them nothing is
    const float mdisp = __uint_as_float(s.st->shake_disp_bits) + __uint_as_float(s.st->out_bits);
    const int mig_n = s.st->mig_n;
    const float mgx = 1e-3f * fdx + mdisp, mgy = 1e-3f * fdy + mdisp, mgz = 1e-3f * fdz + mdisp;
    double red0 = 0.0, red1 = 0.0, red2 = 0.0;  // this lane's atoms' forces (the RBL mean)

    const int col = wk.y;
    {
      const int hx = col / dy, hy = col % dy;
      const int cbase = dz * (hy + dy * hx);
      const int a0 = __ldg(&s.cell_start[cbase]), a1 = __ldg(&s.cell_start[cbase + dz]);
      for (int g0 = a0; g0 < a1; g0 += 32) {
        const int si = g0 + lane;
        const bool valid = si < a1;
        int i = 0, zl = 0;
        float4 p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        bool stray = false;
        int c = 0;  // shells still to skip before the next pick
        __syncwarp();  // the previous chunk's evaluation has read the per-lane records
        if (valid) {
          const int4 mi = __ldg(&s.smeta[si]);
          i = mi.x;
          p4 = __ldg(&s.sxf[si]);
          zl = __ldg(&s.cell_of_atom[i]) - cbase;  // internal cell id iz + dz (iy + dy ix), this column
          stray = col_is_stray(s, si, hx, hy, zl);
          c = col_first_skip(s, i, pice);
          int nsp = 0, spb = 0, sp0 = -1, sp1 = -1;
          float w0 = 1.0f, w1 = 1.0f;
          if (SPECIAL) {  // special partners: the first two cached, the rest read from the CSR lists
            spb = __ldg(&s.sp_off[i]);
            nsp = __ldg(&s.sp_off[i + 1]) - spb;
            if (nsp > 0) {
              sp0 = __ldg(&s.sp_ids[spb]);
              w0 = (float)__ldg(&s.sp_w[spb]);
            }
            if (nsp > 1) {
              sp1 = __ldg(&s.sp_ids[spb + 1]);
              w1 = (float)__ldg(&s.sp_w[spb + 1]);
            }
          }
          s_ai[wid][lane] = make_int4(mi.y, mi.z, nsp, spb);
          s_sp[wid][lane] = make_int2(sp0, sp1);
          s_sw[wid][lane] = make_float2(w0, w1);
        } else {  // a lane without an atom still runs the evaluation rounds (adding nothing): its
                  // record must hold valid indices (type 0, no special partners)
          s_ai[wid][lane] = make_int4(0, -1, 0, 0);
          s_sp[wid][lane] = make_int2(-1, -1);
          s_sw[wid][lane] = make_float2(1.0f, 1.0f);
        }
        s_f[wid][lane] = make_float4(0.0f, 0.0f, 0.0f, p4.w);

        // ---- an atom outside its cell: walked by k_pair_col_strays before this launch, which wrote
        // its force
        if (valid && stray) {
          const double4 fs = s.f[i];
          red0 += fs.x;
          red1 += fs.y;
          red2 += fs.z;
        }

        // ---- the chunk's own atoms, row by row
        const bool act = valid && !stray;
        const int zmin = __reduce_min_sync(FULL, act ? zl : 0x7fffffff);
        const int zmax = __reduce_max_sync(FULL, act ? zl : -1);
        const float pix = p4.x, piy = p4.y, piz = p4.z;
        // evaluates this lane's selected candidates of the last nblk blocks, whose first step read
        // stage entry `base` (the candidates are still in the stage)
        auto flush = [&](int nblk, int base) {
          int qn = 0;
          for (int bk = 0; bk < nblk; ++bk) qn += __popc(s_sel[wid][bk][lane]);
          const int rounds = __reduce_max_sync(FULL, qn);
          if (rounds == 0) return;
          const int4 ai = s_ai[wid][lane];
          const int2 sp = s_sp[wid][lane];
          const float2 sw = s_sw[wid][lane];
          float4 fa = s_f[wid][lane];
          const float spice = (float)pice, fsa = s.fsa, falpha_l2 = s.falpha_l2, fqq = s.fqq;
          const float* const ntab = s.near_tab;  // RBMD_NEAR_TABLE: the reference's G table
          int wc = 0;  // block of the next selected candidate, its remaining bits and its picks
          unsigned mc = s_sel[wid][0][lane], pc = s_pk[wid][0][lane];
          // two rounds per iteration: independent pairs for the scheduler to interleave
#pragma unroll 2
          for (int k = 0; k < rounds; ++k) {
            if (k < qn) {
              while (mc == 0u) {
                ++wc;
                mc = s_sel[wid][wc][lane];
                pc = s_pk[wid][wc][lane];
              }
              const int b = __ffs(mc) - 1;
              mc &= mc - 1u;
              const int e = base + 32 * wc + b;
              const bool core = ((pc >> b) & 1u) == 0u;
              const float4 pj = s_c[wid][e];
              const float rx = pj.x - pix, ry = pj.y - piy, rz = pj.z - piz;
              const float d2 = tile_d2(rx, ry, rz);
              const int idt = s_id[wid][e];
              const int idj = idt & kJsMask, tj = idt >> kJsBits;
              float w = 1.0f;
              if (SPECIAL) {
                if (ai.z <= 2) {
                  w = (idj == sp.x) ? sw.x : w;
                  w = (idj == sp.y) ? sw.y : w;
                } else {
                  for (int t2 = 0; t2 < ai.z; ++t2)
                    if (__ldg(&s.sp_ids[ai.w + t2]) == idj) w = (float)__ldg(&s.sp_w[ai.w + t2]);
                }
              }
              const float2 lj = __ldg(&s.ljf[ai.x * ntypes + tj]);
              float f = tile_pair_f32_lj<MODE, NEAR>(core, d2, fa.w, pj.w, lj.x, lj.y, w, spice, fsa, falpha_l2,
                                                     fqq, ntab);
              // without a branch: the pair of an atom with itself (selected as core, d2 = 0, f not
              // finite) and, for LJ/CUT, pairs of one molecule (its staged id is the molecule) are
              // dropped by the select
              f = ((d2 > 0.0001f) & (MODE != kLJ_RBL || idj != ai.y)) ? f : 0.0f;
              fa.x += f * rx;
              fa.y += f * ry;
              fa.z += f * rz;
            }
          }
          s_f[wid][lane] = fa;
        };

        if (zmax >= 0) {
          const float xr = pix - (float)s.lo[0], yr = piy - (float)s.lo[1], zr = piz - (float)s.lo[2];
          const int u0 = zmin - nc, u1 = zmax + nc;  // the chunk's z cells, unwrapped, -dz < u0, u1 < 2 dz
          for (int r = 0; r < nrows; ++r) {
            const int da = r / side - nc, db = r % side - nc;
            const int n0 = hx + da, n1 = hy + db;  // unwrapped column of the row (nc < dims)
            const int w0c = n0 < 0 ? n0 + dx : (n0 >= dx ? n0 - dx : n0);
            const int w1c = n1 < 0 ? n1 + dy : (n1 >= dy ? n1 - dy : n1);
            const int t0c = n0 < 0 ? 2 : (n0 >= dx ? 0 : 1), t1c = n1 < 0 ? 2 : (n1 >= dy ? 0 : 1);
            const int base = dz * (w1c + dy * w0c);
            // the row's union: unwrapped z cells u0 .. u1 in up to three segments (images -1, 0, +1:
            // below the box, inside, above), segment k holding sorted indices sa_k .., union entries ob_k ..
            int sa0 = 0, sa1, sa2 = 0, ob1, ob2, len = 0;
            if (u0 < 0) {  // below the box: cells u0 + dz .. dz - 1
              sa0 = __ldg(&s.cell_start[base + u0 + dz]);
              len = __ldg(&s.cell_start[base + dz]) - sa0;
            }
            ob1 = len;
            {  // inside: cells max(u0, 0) .. min(u1, dz - 1)
              sa1 = __ldg(&s.cell_start[base + max(u0, 0)]);
              len += __ldg(&s.cell_start[base + min(u1, dz - 1) + 1]) - sa1;
            }
            ob2 = len;
            if (u1 >= dz) {  // above the box: cells 0 .. u1 - dz
              sa2 = __ldg(&s.cell_start[base]);
              len += __ldg(&s.cell_start[base + u1 - dz + 1]) - sa2;
            }
            // union entries before unwrapped cell u (u0 <= u <= u1 + 1)
            auto ucount = [&](int u) -> int {
              if (u > u1) return len;
              if (u < 0) return __ldg(&s.cell_start[base + u + dz]) - sa0;
              if (u < dz) return ob1 + __ldg(&s.cell_start[base + u]) - sa1;
              return ob2 + __ldg(&s.cell_start[base + u - dz]) - sa2;
            };
            // this lane's window, trimmed to the z cells that can hold an atom within rc: the x / y
            // gaps to the row's column (shrunk by the margin) leave a z half-width sqrt(rc^2 - g^2)
            // (grown by it)
            int wb = 0, wl = 0;
            if (act) {
              int zlo = zl + nc + 1, zhi = zl - nc - 1;  // empty
              const float gx = fmaxf(0.0f, fmaxf((float)n0 * fdx - xr, xr - (float)(n0 + 1) * fdx) - mgx);
              const float gy = fmaxf(0.0f, fmaxf((float)n1 * fdy - yr, yr - (float)(n1 + 1) * fdy) - mgy);
              const float g2 = __fmaf_rn(gx, gx, gy * gy);
              if (g2 < frc2) {
                const float h = sqrtf(frc2 - g2) + mgz;
                zlo = max((int)floorf((zr - h) / fdz), zl - nc);
                zhi = min((int)floorf((zr + h) / fdz), zl + nc);
              }
              if (mig_n > kMaxMigrated) {
                zlo = zl - nc;
                zhi = zl + nc;
              } else {
                for (int m = 0; m < mig_n; ++m) {  // the stencil's visits of a recorded cell stay in
                  const int zm = __ldg(&s.st->mig_cell[m]) - base;
                  if (zm < 0 || zm >= dz) continue;  // not in this row's column
                  for (int u = zm - dz; u <= zm + dz; u += dz)
                    if (u >= zl - nc && u <= zl + nc) {
                      zlo = min(zlo, u);
                      zhi = max(zhi, u);
                    }
                }
              }
              if (zlo <= zhi) {
                wb = ucount(zlo);
                wl = ucount(zhi + 1) - wb;
              }
            }
            if (__reduce_max_sync(FULL, wl) == 0) continue;
            // walks the windows of the lanes `in`; their starts lie within kColStage - 32 entries of
            // each other, so every staged tile covers at least one block of 32 steps
            auto walk = [&](bool in) {
              const int ml = __reduce_max_sync(FULL, in ? wl : 0);
              if (ml == 0) return;
              const int gbb = __reduce_min_sync(FULL, in ? wb : 0x7fffffff);
              const int spr = __reduce_max_sync(FULL, in ? wb : gbb) - gbb;
              const int T = (kColStage - spr) & ~31;  // steps per staged tile, whole blocks
              const float shx = s_shift[wid][0][t0c], shy = s_shift[wid][1][t1c];
              // lanes not walking step through the stage too, from a position that matches nothing
              const float wpx = in ? pix : -kColFar, wpy = in ? piy : -kColFar, wpz = in ? piz : -kColFar;
              const int i0 = in ? wb - gbb : 0;
              const int wlen = in ? wl : 0;  // steps of this lane's own window
              for (int t0 = 0; t0 < ml; t0 += T) {
                const int tl = min(T, ml - t0);
                const int nb = (tl + 31) >> 5;  // blocks of this tile
                const int need = spr + tl;      // entries of the tile's windows; up to spr + 32 nb (<=
                                                // kColStage) are read, the rest staged as far away
                const int ub = gbb + t0;        // union index of stage entry 0
                for (int e = lane; e < spr + 32 * nb; e += 32) {
                  const int g = ub + e;
                  float4 cv = make_float4(kColFar, kColFar, kColFar, 0.0f);
                  int idt = 0;
                  if (g < len && e < need) {
                    const int zc = g < ob1 ? 2 : (g < ob2 ? 1 : 0);  // z shift code: below 2, inside 1, above 0
                    const int js = g < ob1 ? sa0 + g : (g < ob2 ? sa1 + (g - ob1) : sa2 + (g - ob2));
                    const float4 pj = __ldg(&s.sxf[js]);
                    const int4 mj = __ldg(&s.smeta[js]);
                    cv = make_float4(pj.x - shx, pj.y - shy, pj.z - s_shift[wid][2][zc], pj.w);
                    idt = (MODE == kLJ_RBL ? mj.z : mj.x) | (mj.y << kJsBits);
                  }
                  s_c[wid][e] = cv;
                  s_id[wid][e] = idt;
                }
                __syncwarp();
                // the walk: blocks of 32 steps, each step a compare into two bit masks, the picks
                // and the FP64 re-classification once per block
                for (int q0 = 0; q0 < nb; q0 += kColQW) {  // at most kColQ steps between evaluations
                  const int nblk = min(kColQW, nb - q0);
                  for (int bk = 0; bk < nblk; ++bk) {
                    const int ib = i0 + 32 * (q0 + bk);  // this lane's stage entry at the block's first step
                    unsigned cm = 0u, sm = 0u;
                    auto step = [&](int st) {
                      const float4 cj = s_c[wid][ib + st];
                      const float ex = cj.x - wpx, ey = cj.y - wpy, ez = cj.z - wpz;
                      const float dd = tile_d2(ex, ey, ez);
                      // x alone: core (or the atom itself, dropped at evaluation); y alone: shell;
                      // both: within a rounding band of rs^2 or rc^2, classified again in FP64
                      const bool x = ((dd <= b1) | (dd >= b2)) & (dd <= b3);
                      const bool y = (dd >= b0) & (dd <= b3);
                      cm |= x ? (1u << st) : 0u;
                      sm |= y ? (1u << st) : 0u;
                    };
                    const int rem = tl - 32 * (q0 + bk);  // steps of the block: 32 but in the tile's last
                    if (rem >= 32) {
#pragma unroll
                      for (int st = 0; st < 32; ++st) step(st);
                    } else {
#pragma unroll 4
                      for (int st = 0; st < rem; ++st) step(st);
                    }
                    // only this lane's own window counts: past its end (the lanes step together) lie
                    // cells beyond rc or outside the stencil
                    const int left = wlen - (t0 + 32 * (q0 + bk));
                    const unsigned vm = left >= 32 ? 0xffffffffu : (left > 0 ? (1u << left) - 1u : 0u);
                    cm &= vm;
                    sm &= vm;
                    for (unsigned bm = cm & sm; bm != 0u; bm &= bm - 1u) {
                      // a banded candidate from its stage slot: union index, segment, sorted index, image
                      const int st = __ffs(bm) - 1;
                      const int g = ub + ib + st;
                      const int zc = g < ob1 ? 2 : (g < ob2 ? 1 : 0);
                      const int js = g < ob1 ? sa0 + g : (g < ob2 ? sa1 + (g - ob1) : sa2 + (g - ob2));
                      const unsigned cs2 = col_classify_fp64(&s, si, js, (t0c - 1) * dx, (t1c - 1) * dy, (zc - 1) * dz);
                      const unsigned bit = 1u << st;
                      cm = (cs2 & 1u) ? (cm | bit) : (cm & ~bit);
                      sm = (cs2 & 2u) ? (sm | bit) : (sm & ~bit);
                    }
                    // every pice-th shell in traversal order, c shells still to skip before the next
                    const unsigned pm = lgp >= 0 ? pick_shells_pow2(sm, lgp, c) : pick_shells(sm, pice, c);
                    s_sel[wid][bk][lane] = cm | pm;
                    s_pk[wid][bk][lane] = pm;
                  }
                  flush(nblk, i0 + 32 * q0);
                }
                __syncwarp();  // the stage is rewritten by the next tile or row
              }
            };
            const int gmin = __reduce_min_sync(FULL, wl > 0 ? wb : 0x7fffffff);
            const int gmax = __reduce_max_sync(FULL, wl > 0 ? wb : -1);
            if (gmax - gmin <= kColStage - 32) {
              walk(wl > 0);
            } else {
              // windows far apart (a sparse home column next to dense ones): the chunk's home cells
              // take turns, and single lanes where one cell's trimmed windows are still too far apart
              for (int zg = zmin; zg <= zmax; ++zg) {
                const bool in = wl > 0 && zl == zg;
                const int lo = __reduce_min_sync(FULL, in ? wb : 0x7fffffff);
                const int hi = __reduce_max_sync(FULL, in ? wb : -1);
                if (hi < 0) continue;
                if (hi - lo <= kColStage - 32) {
                  walk(in);
                } else {
                  for (unsigned m = __ballot_sync(FULL, in); m; m &= m - 1) walk(in && lane == __ffs(m) - 1);
                }
              }
            }
          }
        }
        if (act) {
          const float4 fa = s_f[wid][lane];  // Coulomb already scaled by qqr2e inside the pair factor
          double r9[9];
  #pragma unroll
          for (int q = 0; q < 9; ++q) r9[q] = 0.0;
          r9[0] = (double)fa.x;
          r9[1] = (double)fa.y;
          r9[2] = (double)fa.z;
          finish_atom<MODE>(s, i, r9);
          red0 += r9[0];
          red1 += r9[1];
          red2 += r9[2];
        }
      }
    }
    // RBL mean force: a partial per column; the column of the system that completes last adds them
    // in column order (lane k takes columns k, k + 32, ..., then the fixed butterfly)
    red0 = warp_sum(red0);
    red1 = warp_sum(red1);
    red2 = warp_sum(red2);
    const int ncols = dx * dy;
    int last = 0;
    if (lane == 0) {
      s.vir_part[(size_t)col * 3 + 0] = red0;
      s.vir_part[(size_t)col * 3 + 1] = red1;
      s.vir_part[(size_t)col * 3 + 2] = red2;
      __threadfence();
      last = atomicAdd(&s.st->counter[0], 1u) == (unsigned)(ncols - 1);
      if (last) s.st->counter[0] = 0u;
    }
    if (__shfl_sync(FULL, last, 0)) {
      __threadfence();
      double t0 = 0.0, t1 = 0.0, t2 = 0.0;
      for (int c = lane; c < ncols; c += 32) {
        t0 += __ldcg(&s.vir_part[(size_t)c * 3 + 0]);
        t1 += __ldcg(&s.vir_part[(size_t)c * 3 + 1]);
        t2 += __ldcg(&s.vir_part[(size_t)c * 3 + 2]);
      }
      t0 = warp_sum(t0);
      t1 = warp_sum(t1);
      t2 = warp_sum(t2);
      if (lane == 0) {
        s.st->fmean[0] = t0 / s.n;
        s.st->fmean[1] = t1 / s.n;
        s.st->fmean[2] = t2 / s.n;
      }
    }
  }  // next column
  // the last warp of the launch to finish resets the work counters for the next launch
  if (lane == 0 && atomicAdd(&ctr[1], 1u) == gridDim.x * (unsigned)kColWarps - 1u) {
    ctr[0] = 0u;
    ctr[1] = 0u;
  }
}

// NEAR: RBL Coulomb with the reference's near-Coulomb table (a batch never mixes it with the
// analytic form); a compile-time switch, so that the analytic kernels carry none of its code.
template <typename R, int MODE, bool SPECIAL, bool VIRIAL, bool NEAR>
static void go_near(const Batch& b, cudaStream_t st) {
  static_assert(!NEAR || MODE == kCOUL_RBL, "the near-Coulomb table applies to the RBL Coulomb mode");
  constexpr bool kColumn = sizeof(R) == 4 && (MODE == kLJ_RBL || MODE == kCOUL_RBL) && !VIRIAL;
  const float4 band = make_float4(b.band[0], b.band[1], b.band[2], b.band[3]);
  if constexpr (kColumn) {
    if (b.dense == 2) {
      if (b.pair.n > 0) {
        k_pair_col_strays<MODE, SPECIAL, NEAR><<<b.stray_grid, kColWarps * 32, 0, st>>>(b.sys, b.pair.d, b.pair.n,
                                                                                        b.col_ctr + 2);
        note_launch();
        k_pair_col<MODE, SPECIAL, NEAR><<<b.col_grid, kColWarps * 32, 0, st>>>(b.sys, b.pair.d, b.pair.n, b.col_ctr,
                                                                               band);
        note_launch();
      }
      return;
    }
  }
  if (b.dense)  // the column layout keeps the tile kernel's cell table for every other pass
    k_pair_tile<R, MODE, SPECIAL, VIRIAL, NEAR><<<b.dense == 2 ? b.pair_cells.n : b.pair.n, kCellWarps * 32, 0, st>>>(
        b.sys, b.dense == 2 ? b.pair_cells.d : b.pair.d, 0, nullptr, nullptr, nullptr, nullptr, band);
  else if (b.lean)
    k_pair2<R, MODE, SPECIAL, VIRIAL, NEAR><<<b.pair.n, kPairWarps * 32, 0, st>>>(b.sys, b.pair.d);
  else
    k_pair<R, MODE, SPECIAL, VIRIAL, NEAR><<<b.pair.n, kPairWarps * 32, 0, st>>>(b.sys, b.pair.d, 0, nullptr,
                                                                                nullptr, nullptr, nullptr);
  note_launch();
}

template <typename R, int MODE, bool SPECIAL, bool VIRIAL>
static void go(const Batch& b, cudaStream_t st) {
  if constexpr (MODE == kCOUL_RBL) {
    if (b.near) {
      go_near<R, MODE, SPECIAL, VIRIAL, true>(b, st);
      return;
    }
  }
  go_near<R, MODE, SPECIAL, VIRIAL, false>(b, st);
}

int pair_col_grid(int ncols, int ff, int special, int near, bool strays) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const void* fn;
  if (strays)
    fn = ff == RBMD_FF_LJ_CUT ? (const void*)k_pair_col_strays<kLJ_RBL, false, false>
         : special ? (near ? (const void*)k_pair_col_strays<kCOUL_RBL, true, true>
                           : (const void*)k_pair_col_strays<kCOUL_RBL, true, false>)
                   : (near ? (const void*)k_pair_col_strays<kCOUL_RBL, false, true>
                           : (const void*)k_pair_col_strays<kCOUL_RBL, false, false>);
  else
    fn = ff == RBMD_FF_LJ_CUT ? (const void*)k_pair_col<kLJ_RBL, false, false>
         : special ? (near ? (const void*)k_pair_col<kCOUL_RBL, true, true>
                           : (const void*)k_pair_col<kCOUL_RBL, true, false>)
                   : (near ? (const void*)k_pair_col<kCOUL_RBL, false, true>
                           : (const void*)k_pair_col<kCOUL_RBL, false, false>);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kColWarps * 32, 0);
  const int need = (ncols + kColWarps - 1) / kColWarps;
  return std::max(1, std::min(need, std::max(1, sms) * std::max(1, per_sm)));
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

void launch_rbl_lists(const SysDev* sys, int slot, int n, int ncell, int dense, int cap, int* n_core,
                      int* n_shell, int* ids, cudaStream_t st) {
  // ids holds 2 * n * cap ints: core rows then shell rows
  const int per = dense ? kCellWarps : kPairWarps;
  const int nb = ((dense ? ncell : n) + per - 1) / per;
  int2* d_work = nullptr;
  if (cudaMallocAsync(&d_work, sizeof(int2) * nb, st) != cudaSuccess || !d_work) {
    cudaGetLastError();
    return;  // the caller's sync reports the missing lists
  }
  int2* h = new int2[nb];
  for (int k = 0; k < nb; ++k) h[k] = make_int2(slot, k * per);
  cudaMemcpyAsync(d_work, h, sizeof(int2) * nb, cudaMemcpyHostToDevice, st);
  if (dense)
    k_pair_tile<double, kLIST, false, false><<<nb, kCellWarps * 32, 0, st>>>(sys, d_work, cap, n_core, n_shell,
                                                                             ids, ids + (size_t)n * cap, float4{});
  else
    k_pair<double, kLIST, false, false><<<nb, kPairWarps * 32, 0, st>>>(sys, d_work, cap, n_core, n_shell,
                                                                       ids, ids + (size_t)n * cap);
  note_launch();
  cudaStreamSynchronize(st);
  delete[] h;
  cudaFreeAsync(d_work, st);
}


// ---------------------------------------------------------------- allocation-free RBL lists
// Every temporary of rbmd_get_rbl_lists_static lives in this one file-scope array: the work
// tables of the binning and list kernels, the per-atom counts and the core and shell rows.  Each
// GPU that loads the library holds its copy (kStaticListInts ints = 8 MiB) until the process
// exits.  Host code must not pass the array's name to a kernel (on the host it is a stand-in, not
// a device address): static_list_scratch() gives the device address.
static __device__ __align__(256) int g_list_scratch[kStaticListInts];

namespace {
std::mutex g_scratch_mu;
int* g_scratch_addr[64] = {};

constexpr long long round64(long long v) { return (v + 63) / 64 * 64; }

__global__ void k_static_work(int slot, int per, int2* atom, int na, int2* cell, int nc, int2* pair, int np,
                              int* slot_flag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < na) atom[t] = make_int2(slot, t * kAtomBlock);
  if (t < nc) cell[t] = make_int2(slot, t * kCellBlock);
  if (t < np) pair[t] = make_int2(slot, t * per);
  if (t == 0) {
    slot_flag[0] = slot;
    slot_flag[1] = 0;  // overflow flag: the array keeps the last call's contents, so clear it
  }
}

// warp per atom: shell ids moved behind the core ids of the same row, the rest of the row -1
__global__ void k_static_pack(int n, int cap, const int* __restrict__ n_core, const int* __restrict__ n_shell,
                              int* core_rows, const int* __restrict__ shell_rows, int* flag) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  const int a = n_core[i], b = n_shell[i];
  if (a + b > cap) {
    if (lane == 0) atomicOr(flag, 1);
    return;
  }
  int* row = core_rows + (size_t)i * cap;
  const int* sh = shell_rows + (size_t)i * cap;
  for (int k = lane; k < b; k += 32) row[a + k] = sh[k];
  for (int k = a + b + lane; k < cap; k += 32) row[k] = -1;
}
}  // namespace

int static_list_scratch(int** out) {
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= 64) return (int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_list_scratch);  // with `dev` current
    if (e != cudaSuccess) {
      cudaGetLastError();
      return (int)e;
    }
    g_scratch_addr[dev] = (int*)ptr;
  }
  *out = g_scratch_addr[dev];
  return 0;
}

long long static_list_ints(int n, int ncell, int dense, int cap) {
  const int per = dense ? kCellWarps : kPairWarps;
  const long long na = (n + kAtomBlock - 1) / kAtomBlock, nc = (ncell + kCellBlock - 1) / kCellBlock;
  const long long np = ((dense ? ncell : (long long)n) + per - 1) / per;
  return round64(2 * na) + round64(2 * nc) + round64(2 * np) + 64 + round64(n) + round64(n) +
         round64((long long)n * cap) + round64((long long)n * cap);
}

int launch_rbl_lists_static(const SysDev* sys, int slot, int n, int ncell, int dense, int cap, int* scratch,
                            cudaStream_t st, StaticLists* out) {
  if (!scratch || static_list_ints(n, ncell, dense, cap) > kStaticListInts) return 1;
  const int per = dense ? kCellWarps : kPairWarps;
  const int na = (n + kAtomBlock - 1) / kAtomBlock, nc = (ncell + kCellBlock - 1) / kCellBlock;
  const int np = ((dense ? ncell : n) + per - 1) / per;
  int* p = scratch;
  int2* w_atom = (int2*)p;
  p += round64(2LL * na);
  int2* w_cell = (int2*)p;
  p += round64(2LL * nc);
  int2* w_pair = (int2*)p;
  p += round64(2LL * np);
  int* slot_flag = p;
  p += 64;
  out->n_core = p;
  p += round64(n);
  out->n_shell = p;
  p += round64(n);
  out->rows = p;
  p += round64((long long)n * cap);
  int* shell_rows = p;
  out->flag = slot_flag + 1;

  const int mx = std::max(na, std::max(nc, np));
  k_static_work<<<(mx + 255) / 256, 256, 0, st>>>(slot, per, w_atom, na, w_cell, nc, w_pair, np, slot_flag);
  note_launch();
  Batch b;
  b.sys = const_cast<SysDev*>(sys);
  b.d_slots = slot_flag;
  b.nsys = 1;
  b.atom.d = w_atom;
  b.atom.n = na;
  b.cell.d = w_cell;
  b.cell.n = nc;
  launch_cells(b, st);
  if (dense)
    k_pair_tile<double, kLIST, false, false><<<np, kCellWarps * 32, 0, st>>>(sys, w_pair, cap, out->n_core,
                                                                             out->n_shell, out->rows, shell_rows,
                                                                             float4{});
  else
    k_pair<double, kLIST, false, false><<<np, kPairWarps * 32, 0, st>>>(sys, w_pair, cap, out->n_core,
                                                                       out->n_shell, out->rows, shell_rows);
  note_launch();
  k_static_pack<<<(n + 7) / 8, 256, 0, st>>>(n, cap, out->n_core, out->n_shell, out->rows, shell_rows,
                                             out->flag);
  note_launch();
  return 0;
}

}  // namespace rbmd
