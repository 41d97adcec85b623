// oracle_step.cpp -- pair forces, bonded terms, integrator, thermostats, SHAKE/RATTLE, energies and
// EAM input of the FP64 oracle.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <algorithm>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

#include "oracle.hpp"

namespace oracle {

namespace {

// ExecForceFunction::ComputeLJForce, framework/forceFunction/ExecForceFunction.h:412-437
inline void lj_force(const double r[3], double dis_2, double eps_i, double eps_j, double sig_i,
                     double sig_j, double cut_off, double out[3]) {
  out[0] = out[1] = out[2] = 0;
  const double cut_off_2 = cut_off * cut_off;
  if (dis_2 < cut_off_2 && dis_2 > 0.0001) {
    double sigma_ij = (sig_i + sig_j) / 2;
    double s6 = sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij;
    double dis_6 = dis_2 * dis_2 * dis_2;
    double sd6 = s6 / dis_6;
    double fs = -24 * std::sqrt(eps_i * eps_j) * ((2 * sd6 - 1) * sd6) / dis_2;
    for (int k = 0; k < 3; ++k) out[k] = fs * r[k];
  }
}

// ExecForceFunction::ComputeLJForceRcs, ExecForceFunction.h:439-462
inline void lj_force_rcs(const double r[3], double dis_2, double eps_i, double eps_j, double sig_i,
                         double sig_j, double rc, double rs, double out[3]) {
  out[0] = out[1] = out[2] = 0;
  if (dis_2 < rc * rc && dis_2 > rs * rs) {
    double sigma_ij = (sig_i + sig_j) / 2;
    double s6 = sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij;
    double dis_6 = dis_2 * dis_2 * dis_2;
    double sd6 = s6 / dis_6;
    double fs = -24 * std::sqrt(eps_i * eps_j) * ((2 * sd6 - 1) * sd6) / dis_2;
    for (int k = 0; k < 3; ++k) out[k] = fs * r[k];
  }
}

// ExecForceFunction::Gnear, ExecForceFunction.h:682-689 (analytic form)
inline double gnear(double alpha, double dis) {
  double erfcx = std::sqrt(alpha) * dis;
  double expx = -alpha * dis * dis;
  return (1.0 - std::erf(erfcx)) / (dis * dis) +
         2 * std::sqrt(alpha) * std::exp(expx) / (std::sqrt(kPif) * dis);
}

// ComputePotentialEn_fix, ExecForceFunction.h:818-841
inline double lj_energy(double dis_2, double eps_i, double eps_j, double sig_i, double sig_j,
                        double cut_off) {
  if (dis_2 < cut_off * cut_off && dis_2 > 0.0001) {
    double sigma_ij = (sig_i + sig_j) / 2;
    double s6 = sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij;
    double dis_6 = dis_2 * dis_2 * dis_2;
    double eps_ij = std::sqrt(eps_i * eps_j);
    return 0.5 * (4 * eps_ij * (s6 / dis_6 - 1) * (s6 / dis_6));
  }
  return 0.0;
}

inline void add_virial(double v[6], const double r[3], const double F[3], double scale) {
  // ComputePairVirial (scale -0.5) / ComputePairVirial_fix (scale +0.5), ExecForceFunction.h:304-331
  double h[3] = {scale * F[0], scale * F[1], scale * F[2]};
  v[0] += r[0] * h[0];
  v[1] += r[1] * h[1];
  v[2] += r[2] * h[2];
  v[3] += r[0] * h[1];
  v[4] += r[0] * h[2];
  v[5] += r[1] * h[2];
}

// EAM spline evaluations, ExecForceFunction.h:896-1096
inline double eam_rho(const double* sp, double r, double rdr, int nr) {
  double pp = r * rdr + 1.0;
  int mm = (int)pp;
  mm = std::min(mm, nr - 1);
  pp -= mm;
  pp = std::min(pp, 1.0);
  const double* c = &sp[7 * mm];
  return ((c[3] * pp + c[4]) * pp + c[5]) * pp + c[6];
}

}  // namespace

double special_weight(const System& s, int i, int j) {
  // weight lookup loop of ComputeNearForceRBLERFSpecialBondsWorklet, RunWorklet.cpp:1163-1170
  double w = 1.0;
  for (int k = s.special_offsets[i]; k < s.special_offsets[i + 1]; ++k)
    if (s.special_ids[k] == j) w = s.special_weights[k];
  return w;
}

// ------------------------------------------------------------------ a5 / a7 / a8 / a15
void System::near_force(std::vector<double>& F) {
  F.assign(3 * N, 0.0);
  const double rc = p.cut_off, rs = p.r_core;
  const double rc_2 = rc * rc, rs_2 = rs * rs;
  const int pice = dv.pice_num;
  const bool special = !special_offsets.empty();
  for (int k = 0; k < 6; ++k) virial[k] = 0;

  if (p.force_field == RBMD_FF_EAM) {
    // ComputeRBLEAMForce (ExecutionMD.cpp:1013-1100) / ComputeVerletlistEAMForce (:1102-1160):
    // EAMfp pass then force pass; RBL subtracts the mean force.
    const double rdr = 1.0 / eam_dr, rdrho = 1.0 / eam_drho;
    std::vector<double> fp(N, 0.0);
    const bool rbl = (p.neighbor == RBMD_NEIGH_RBL);
    par_for((long)(N), [&](long i_l) {
      const int i = (int)i_l;
      double rho = 0.0;
      int index_shell = rbl_offset(i);
      traverse(i, [&](int j, const double*, const double* r0, double d2) {
        bool core, shell = false;
        if (rbl) {
          shell = (rc_2 - d2 > 0.0001 && d2 - rs_2 > 0.0001);
          core = !shell && (rs_2 - d2 > 0.0001 && d2 > 0.0001);
          if (shell) {
            bool pick = (index_shell % pice == 0);
            index_shell++;
            if (!pick) return;
          }
        } else {
          core = (rc_2 - d2 > 0.0001 && d2 > 0.0001);
        }
        if (!core && !shell) return;
        double r[3] = {-r0[0], -r0[1], -r0[2]};  // MinDistanceVec(p_i, p_j)
        min_image(r);
        double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        // the density of the neighbour's type (LAMMPS eam/alloy type2rhor[jtype][itype])
        if (core) {
          if (rsq < rc * rc && rsq > 0.01) rho += eam_rho(rhor_of(type[j]), std::sqrt(rsq), rdr, eam_nr);
        } else {
          if (rsq < rc * rc && rsq > rs_2) rho += pice * eam_rho(rhor_of(type[j]), std::sqrt(rsq), rdr, eam_nr);
        }
      });
      // ComputeEAMfp, ExecForceFunction.h:946-962
      double pp = rho * rdrho + 1.0;
      int mm = (int)pp;
      mm = std::max(1, std::min(mm, eam_nrho - 1));
      pp -= mm;
      pp = std::min(pp, 1.0);
      const double* c = frho_of(type[i]) + 7 * mm;
      fp[i] = (c[0] * pp + c[1]) * pp + c[2];
    });
    par_for((long)(N), [&](long i_l) {
      const int i = (int)i_l;
      double fc[3] = {0, 0, 0}, fs[3] = {0, 0, 0};
      int index_shell = rbl_offset(i);
      traverse(i, [&](int j, const double*, const double* r0, double d2) {
        bool core, shell = false;
        if (rbl) {
          shell = (rc_2 - d2 > 0.0001 && d2 - rs_2 > 0.0001);
          core = !shell && (rs_2 - d2 > 0.0001 && d2 > 0.0001);
          if (shell) {
            bool pick = (index_shell % pice == 0);
            index_shell++;
            if (!pick) return;
          }
        } else {
          core = (rc_2 - d2 > 0.0001 && d2 > 0.0001);
        }
        if (!core && !shell) return;
        double r[3] = {-r0[0], -r0[1], -r0[2]};
        min_image(r);
        double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        bool ok = core ? (rsq < rc * rc && rsq > 0.01) : (rsq < rc * rc && rsq > rs_2);
        if (!ok) return;
        // ComputeEAMforce / ComputeEAMforceRBL, ExecForceFunction.h:980-1090
        double rr = std::sqrt(rsq);
        double pp = rr * rdr + 1.0;
        int mm = (int)pp;
        mm = std::min(mm, eam_nr - 1);
        pp -= mm;
        pp = std::min(pp, 1.0);
        const double* ci = rhor_of(type[i]) + 7 * mm;
        double rhoip = (ci[0] * pp + ci[1]) * pp + ci[2];
        const double* cj = rhor_of(type[j]) + 7 * mm;
        double rhojp = (cj[0] * pp + cj[1]) * pp + cj[2];
        const double* cz = z2r_of(type[i], type[j]) + 7 * mm;
        double z2p = (cz[0] * pp + cz[1]) * pp + cz[2];
        double z2 = ((cz[3] * pp + cz[4]) * pp + cz[5]) * pp + cz[6];
        double recip = 1.0 / rr;
        double phi = z2 * recip;
        double phip = z2p * recip - phi * recip;
        double psip = fp[i] * rhojp + fp[j] * rhoip + phip;
        double fpair = -psip * recip;
        double* acc = core ? fc : fs;
        double scale = core ? 1.0 : (double)pice;
        for (int k = 0; k < 3; ++k) acc[k] += scale * (r[k] * fpair);
      });
      for (int k = 0; k < 3; ++k) F[3 * i + k] = fc[k] + fs[k];
    });
    if (rbl) {
      double mean[3] = {0, 0, 0};
      for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) mean[k] += F[3 * i + k];
      for (int k = 0; k < 3; ++k) mean[k] /= N;
      for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) F[3 * i + k] -= mean[k];
    }
    return;
  }

  const bool coul = (p.force_field != RBMD_FF_LJ_CUT);
  if (p.neighbor == RBMD_NEIGH_RBL) {
    // LJ/CUT: ComputeLJForceRBLWorklet (RunWorklet.cpp:1817-1909), same-molecule pairs skipped.
    // Coulomb force fields: ComputeNearForceRBLERFWorklet (RunWorklet.cpp:982-1093) and its
    // special-bond variant (RunWorklet.cpp:1095-1266); core LJ uses cutoff rs there.
    par_for((long)(N), [&](long i_l) {
      const int i = (int)i_l;
      double lj_c[3] = {0, 0, 0}, lj_s[3] = {0, 0, 0}, el_c[3] = {0, 0, 0}, el_s[3] = {0, 0, 0};
      const int ti = type[i];
      int index_shell = rbl_offset(i);
      traverse(i, [&](int j, const double*, const double* r0, double d2) {
        bool shell = (rc_2 - d2 > 0.0001 && d2 - rs_2 > 0.0001);
        bool core = !shell && (rs_2 - d2 > 0.0001 && d2 > 0.0001);
        if (shell) {
          bool pick = (index_shell % pice == 0);
          index_shell++;
          if (!pick) return;
        }
        if (!core && !shell) return;
        if (!coul && mol[i] == mol[j]) return;
        double r[3] = {r0[0], r0[1], r0[2]};
        min_image(r);
        double dis_2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const int tj = type[j];
        double w = special ? special_weight(*this, i, j) : 1.0;
        double t[3];
        if (core) {
          lj_force(r, dis_2, eps[ti], eps[tj], sig[ti], sig[tj], coul ? rs : rc, t);
          for (int k = 0; k < 3; ++k) lj_c[k] += w * t[k];
        } else {
          lj_force_rcs(r, dis_2, eps[ti], eps[tj], sig[ti], sig[tj], rc, rs, t);
          for (int k = 0; k < 3; ++k) lj_s[k] += w * (pice * t[k]);
        }
        if (coul) {
          double dis = std::sqrt(dis_2);
          bool in = core ? (dis_2 < rc_2 && dis_2 > 0.0001)
                         : (special ? (dis_2 < rc_2 && dis_2 > rs_2) : (dis_2 < rc_2 && dis_2 > 0.0001));
          if (in) {
            double g = near_tab.empty() ? gnear(p.alpha, dis) : near_g(dis);
            double fs_ = -q[i] * q[j] * g;
            for (int k = 0; k < 3; ++k) {
              double val = fs_ * r[k] / dis;
              if (core) el_c[k] += val;
              else el_s[k] += pice * val;
            }
          }
        }
      });
      for (int k = 0; k < 3; ++k)
        F[3 * i + k] = (lj_c[k] + lj_s[k]) + u.qqr2e * (el_c[k] + el_s[k]);
    });
    // SumRBLCorrForce with the mean, ExecutionMD.cpp:663-667 / 820-826
    double mean[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i)
      for (int k = 0; k < 3; ++k) mean[k] += F[3 * i + k];
    for (int k = 0; k < 3; ++k) mean[k] /= N;
    for (int i = 0; i < N; ++i)
      for (int k = 0; k < 3; ++k) F[3 * i + k] -= mean[k];
    // The per-atom RBL virials are mean-subtracted too (RunWorklet.cpp:1930-1947), so their sum,
    // which is all ComputeVirial uses, is zero.
    return;
  }

  // VERLETLIST: LJForceVerlet (RunWorklet.cpp:498-575), NearForceVerletVirial (:2890-2985),
  // NearForceVerletWeightVirial (:2767-2888).  Per-atom virials, summed in atom order afterwards.
  std::vector<double> vir_atom(6 * (size_t)N, 0.0);
  par_for((long)(N), [&](long i_l) {
    const int i = (int)i_l;
    double fi[3] = {0, 0, 0};
    double* virial = &vir_atom[6 * (size_t)i];
    const int ti = type[i];
    traverse(i, [&](int j, const double*, const double* r0, double d2) {
      if (!(rc_2 - d2 > 0.0001 && d2 > 0.0001)) return;
      double r[3] = {r0[0], r0[1], r0[2]};
      min_image(r);
      double dis_2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      const int tj = type[j];
      double flj[3];
      lj_force(r, dis_2, eps[ti], eps[tj], sig[ti], sig[tj], rc, flj);
      double fpair[3] = {flj[0], flj[1], flj[2]};
      double vscale = 0.5;
      if (coul) {
        double dis = std::sqrt(dis_2);
        double fc[3] = {0, 0, 0}, fb[3] = {0, 0, 0};
        if (dis_2 < rc_2 && dis_2 > 0.0001) {
          double g = gnear(p.alpha, dis);
          for (int k = 0; k < 3; ++k) {
            fc[k] = -q[i] * q[j] * g * r[k] / dis;
            fb[k] = -q[i] * q[j] * r[k] / (dis * dis * dis);
          }
        }
        if (special) {
          double w = special_weight(*this, i, j);
          for (int k = 0; k < 3; ++k) fpair[k] = u.qqr2e * (fc[k] - (1 - w) * fb[k]) + w * flj[k];
          vscale = -0.5;
        } else {
          for (int k = 0; k < 3; ++k) fpair[k] = u.qqr2e * fc[k] + flj[k];
        }
      }
      for (int k = 0; k < 3; ++k) fi[k] += fpair[k];
      add_virial(virial, r, fpair, vscale);
    });
    for (int k = 0; k < 3; ++k) F[3 * i + k] = fi[k];
  });
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 6; ++k) virial[k] += vir_atom[6 * (size_t)i + k];
}

// ------------------------------------------------------------------ a9 / a19
void System::bonded_force(std::vector<double>& F) {
  F.assign(3 * N, 0.0);
  double vir[6] = {0, 0, 0, 0, 0, 0};
  // ComputeSpecialCoulGeneralWorklet (RunWorklet.cpp:2012-2084), RBL only (ExecutionNVT.cpp:216-219)
  if (p.neighbor == RBMD_NEIGH_RBL && !special_offsets.empty()) {
    for (int i = 0; i < N; ++i) {
      int a0 = mol_offsets[mol[i]], a1 = mol_offsets[mol[i] + 1];
      if (a1 - a0 < 3) continue;
      for (int s = a0; s < a1; ++s) {
        int j = mol_atoms[s];
        if (j == i) continue;
        double r[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
        min_image(r);
        double dis = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        double dis3 = std::pow(dis, 3);
        double fcomp = -332.06371 * q[i] * q[j] / dis3;
        double w = special_weight(*this, i, j);
        double cp[3];
        for (int k = 0; k < 3; ++k) {
          cp[k] = (1.0 - w) * fcomp * r[k];
          F[3 * i + k] += cp[k];
        }
        add_virial(vir, r, cp, 0.5);
      }
    }
  }
  // ComputeBondHarmonicWorklet, MolecularWorklet.h:58-199
  double e_bond = 0;
  int nb = (int)bond_type.size();
  for (int b = 0; b < nb; ++b) {
    int i = bond_atoms[2 * b], j = bond_atoms[2 * b + 1];
    double kk = bond_k[bond_type[b]], r0 = bond_r0[bond_type[b]];
    double r[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
    min_image(r);
    double dis_2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    double disij = std::sqrt(dis_2);
    double dr = disij - r0;
    double rk = kk * dr;
    double fb = disij > 0.01 ? -2.0 * rk / disij : 0.0;
    double fv[3] = {r[0] * fb, r[1] * fb, r[2] * fb};
    for (int k = 0; k < 3; ++k) {
      F[3 * i + k] += fv[k];
      F[3 * j + k] -= fv[k];
    }
    e_bond += rk * dr;
    add_virial(vir, r, fv, 1.0);
  }
  e_bond_avg = nb > 0 ? e_bond / nb : 0.0;
  // ComputeAngleHarmonicWorklet, MolecularWorklet.h:231-397
  double e_angle = 0;
  int na = (int)angle_type.size();
  for (int a = 0; a < na; ++a) {
    int i = angle_atoms[3 * a], j = angle_atoms[3 * a + 1], kx = angle_atoms[3 * a + 2];
    double kk = angle_k[angle_type[a]], th0 = angle_theta0[angle_type[a]];
    double rij[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
    double rkj[3] = {x[3 * kx] - x[3 * j], x[3 * kx + 1] - x[3 * j + 1], x[3 * kx + 2] - x[3 * j + 2]};
    min_image(rij);
    min_image(rkj);
    double dij2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
    double dij = std::sqrt(dij2);
    double dkj2 = rkj[0] * rkj[0] + rkj[1] * rkj[1] + rkj[2] * rkj[2];
    double dkj = std::sqrt(dkj2);
    double c = rij[0] * rkj[0] + rij[1] * rkj[1] + rij[2] * rkj[2];
    c /= dij * dkj;
    if (c > 1.0) c = 1.0;
    if (c < -1.0) c = -1.0;
    double s = std::sqrt(1.0 - c * c);
    if (s < 0.001) s = 0.001;
    s = 1.0 / s;
    double dtheta = std::acos(c) - (th0 * kPif) / 180;
    double tk = kk * dtheta;
    e_angle += tk * dtheta;
    double aa = -2.0 * tk * s;
    double a11 = aa * c / dij2;
    double a12 = -aa / (dij * dkj);
    double a22 = aa * c / dkj2;
    double fi[3], fk[3];
    for (int k = 0; k < 3; ++k) {
      fi[k] = a11 * rij[k] + a12 * rkj[k];
      fk[k] = a22 * rkj[k] + a12 * rij[k];
      F[3 * i + k] += fi[k];
      F[3 * j + k] += -fi[k] - fk[k];
      F[3 * kx + k] += fk[k];
    }
    vir[0] += rij[0] * fi[0] + rkj[0] * fk[0];
    vir[1] += rij[1] * fi[1] + rkj[1] * fk[1];
    vir[2] += rij[2] * fi[2] + rkj[2] * fk[2];
    vir[3] += rij[0] * fi[1] + rkj[0] * fk[1];
    vir[4] += rij[0] * fi[2] + rkj[0] * fk[2];
    vir[5] += rij[1] * fi[2] + rkj[1] * fk[2];
  }
  e_angle_avg = na > 0 ? e_angle / na : 0.0;
  // ComputeDihedralHarmonicWorklet, MolecularWorklet.h:669-973: E = K [1 + d cos(n phi)], forces
  // reduced per atom id, energy averaged over dihedrals (ExecutionNVT.cpp:585-658)
  double e_dih = 0;
  const int nd = (int)dihedral_type.size();
  for (int t = 0; t < nd; ++t) {
    const int i1 = dihedral_atoms[4 * t], i2 = dihedral_atoms[4 * t + 1], i3 = dihedral_atoms[4 * t + 2],
              i4 = dihedral_atoms[4 * t + 3];
    const int ty = dihedral_type[t];
    const double K = dihedral_k[ty];
    const int m = dihedral_mult[ty];
    const double cos_shift = dihedral_sign[ty] == 1 ? 1.0 : -1.0, sin_shift = 0.0;
    double vb1[3], vb2[3], vb2m[3], vb3[3];
    for (int k = 0; k < 3; ++k) {
      vb1[k] = x[3 * i1 + k] - x[3 * i2 + k];
      vb2[k] = x[3 * i3 + k] - x[3 * i2 + k];
      vb3[k] = x[3 * i4 + k] - x[3 * i3 + k];
    }
    min_image(vb1);
    min_image(vb2);
    min_image(vb3);
    for (int k = 0; k < 3; ++k) vb2m[k] = -vb2[k];
    const double ax = vb1[1] * vb2m[2] - vb1[2] * vb2m[1];
    const double ay = vb1[2] * vb2m[0] - vb1[0] * vb2m[2];
    const double az = vb1[0] * vb2m[1] - vb1[1] * vb2m[0];
    const double bx = vb3[1] * vb2m[2] - vb3[2] * vb2m[1];
    const double by = vb3[2] * vb2m[0] - vb3[0] * vb2m[2];
    const double bz = vb3[0] * vb2m[1] - vb3[1] * vb2m[0];
    const double rasq = ax * ax + ay * ay + az * az;
    const double rbsq = bx * bx + by * by + bz * bz;
    const double rgsq = vb2m[0] * vb2m[0] + vb2m[1] * vb2m[1] + vb2m[2] * vb2m[2];
    const double rg = std::sqrt(rgsq);
    double rginv = 0.0, ra2inv = 0.0, rb2inv = 0.0;
    if (rg > 0) rginv = 1.0 / rg;
    if (rasq > 0) ra2inv = 1.0 / rasq;
    if (rbsq > 0) rb2inv = 1.0 / rbsq;
    const double rabinv = std::sqrt(ra2inv * rb2inv);
    double c = (ax * bx + ay * by + az * bz) * rabinv;
    const double s = rg * rabinv * (ax * vb3[0] + ay * vb3[1] + az * vb3[2]);
    if (c > 1.0) c = 1.0;
    if (c < -1.0) c = -1.0;
    double pp = 1.0, ddf1 = 0.0, df1 = 0.0;
    for (int q = 0; q < m; q++) {
      ddf1 = pp * c - df1 * s;
      df1 = pp * s + df1 * c;
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
    e_dih += K * pp;
    const double fg = vb1[0] * vb2m[0] + vb1[1] * vb2m[1] + vb1[2] * vb2m[2];
    const double hg = vb3[0] * vb2m[0] + vb3[1] * vb2m[1] + vb3[2] * vb2m[2];
    const double fga = fg * ra2inv * rginv;
    const double hgb = hg * rb2inv * rginv;
    const double gaa = -ra2inv * rg;
    const double gbb = rb2inv * rg;
    const double dtf[3] = {gaa * ax, gaa * ay, gaa * az};
    const double dtg[3] = {fga * ax - hgb * bx, fga * ay - hgb * by, fga * az - hgb * bz};
    const double dth[3] = {gbb * bx, gbb * by, gbb * bz};
    const double df = -K * df1;
    double f1[3], f2[3], f3[3], f4[3];
    for (int k = 0; k < 3; ++k) {
      const double s2 = df * dtg[k];
      f1[k] = df * dtf[k];
      f2[k] = s2 - f1[k];
      f4[k] = df * dth[k];
      f3[k] = -s2 - f4[k];
      F[3 * i1 + k] += f1[k];
      F[3 * i2 + k] += f2[k];
      F[3 * i3 + k] += f3[k];
      F[3 * i4 + k] += f4[k];
    }
    vir[0] += vb1[0] * f1[0] + vb2[0] * f3[0] + (vb3[0] + vb2[0]) * f4[0];
    vir[1] += vb1[1] * f1[1] + vb2[1] * f3[1] + (vb3[1] + vb2[1]) * f4[1];
    vir[2] += vb1[2] * f1[2] + vb2[2] * f3[2] + (vb3[2] + vb2[2]) * f4[2];
    vir[3] += vb1[0] * f1[1] + vb2[0] * f3[1] + (vb3[0] + vb2[0]) * f4[1];
    vir[4] += vb1[0] * f1[2] + vb2[0] * f3[2] + (vb3[0] + vb2[0]) * f4[2];
    vir[5] += vb1[1] * f1[2] + vb2[1] * f3[2] + (vb3[1] + vb2[1]) * f4[2];
  }
  e_dihedral_avg = nd > 0 ? e_dih / nd : 0.0;
  for (int k = 0; k < 6; ++k) virial[k] += vir[k];
}

// ------------------------------------------------------------------ a20: ComputeForce
void System::compute_force() {
  // ExecutionNVT::ComputeAllForce, framework/run/ExecutionNVT.cpp:195-235
  near_force(f_near);
  double vir_far[6] = {0, 0, 0, 0, 0, 0};
  f_far.assign(3 * N, 0.0);
  if (p.force_field == RBMD_FF_LJ_CUT_COUL_LONG || p.force_field == RBMD_FF_CVFF) {
    if (p.coulomb == RBMD_COUL_RBE) {
      structure_factor();
      rbe_force(f_far, vir_far);
    } else if (p.coulomb == RBMD_COUL_EWALD) {
      ewald_force(f_far, vir_far);
    }
    for (auto& val : f_far) val *= u.qqr2e;  // UnitRescaleWorklet, ExecutionNVT.cpp:718
    for (int k = 0; k < 6; ++k) virial[k] += vir_far[k] * u.qqr2e;
  }
  f_bonded.assign(3 * N, 0.0);
  if (p.force_field == RBMD_FF_CVFF) bonded_force(f_bonded);
  for (int i = 0; i < 3 * N; ++i) f[i] = f_far[i] + f_near[i] + f_bonded[i];
}

// ------------------------------------------------------------------ a16: integrator
void System::update_velocity(std::vector<double>* old_v) {
  // ExecutionNVT::UpdateVelocity + UpdateVelocityWorklet, ExecutionNVT.cpp:237-249,
  // RunWorklet.cpp:2357-2375: v += 0.5 F / m dt fmt2v
  if (old_v) *old_v = v;
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) v[3 * i + k] += 0.5 * f[3 * i + k] / m[i] * p.timestep * u.fmt2v;
}

void System::update_position(std::vector<double>* old_x) {
  // ExecutionNVT::UpdatePosition (ExecutionNVT.cpp:251-268), UpdatePositionFlagWorklet and
  // ApplyPbcFlagWorklet (RunWorklet.cpp:2467-2490, 2602-2636), then the locator rebuild.
  if (old_x) *old_x = x;
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) {
      double& xx = x[3 * i + k];
      xx += v[3 * i + k] * p.timestep;
      if (xx < lo[k]) {
        xx += L[k];
        image[3 * i + k] -= 1;
      } else if (xx >= hi[k]) {
        xx -= L[k];
        image[3 * i + k] += 1;
      }
    }
  build_cells();
}

// ------------------------------------------------------------------ a17: thermostats
void System::compute_tempe() {
  // ExecutionNVT::ComputeTempe, framework/run/ExecutionNVT.cpp:736-773
  double sum = 0.0;
  for (int i = 0; i < N; ++i) {
    double vv = v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2];
    sum += (m[i] * vv) * u.mvv2e;
  }
  th.tempT_sum = sum;
  const double n = N;
  const double kB = u.kB;
  if (p.init_inbuild) th.temperature = 0.5 * sum / (3 * n / 2.0);
  else if (p.fix_shake == RBMD_SHAKE_NULL) th.temperature = 0.5 * sum / ((3 * n - 3) * kB / 2.0);
  else if (p.fix_shake == RBMD_SHAKE_TRUE) th.temperature = 0.5 * sum / ((3 * n - n - 3) * kB / 2.0);
  else th.temperature = 0.5 * sum / ((3 * n) * kB / 2.0);
}

void System::compute_temp_target() {
  // ExecutionNVT::ComputeTempTarget, ExecutionNVT.cpp:1124-1147
  const double t_start = p.temperature[0], t_stop = p.temperature[1];
  if (t_stop == t_start) {
    th.t_target = t_start;
  } else {
    double delta = (double)step;
    if (delta != 0.0) delta = delta / (double)p.num_steps;
    th.t_target = t_start + delta * (t_stop - t_start);
  }
  th.ke_target = th.tdof * u.boltz * th.t_target;
}

void System::nhc_integrate() {
  // ExecutionNVT::NHCTempIntegrate, ExecutionNVT.cpp:1172-1256 (mtchain 3, nc_tchain 1)
  const int mtchain = 3;
  const double dt = p.timestep;
  const double dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  double kecurrent = th.tdof * u.boltz * th.temperature;
  th.eta_mass[0] = th.tdof * u.boltz * th.t_target / (th.t_freq * th.t_freq);
  for (int ich = 1; ich < mtchain; ich++) th.eta_mass[ich] = u.boltz * th.t_target / (th.t_freq * th.t_freq);
  if (th.eta_mass[0] > 0.0) th.eta_dotdot[0] = (kecurrent - th.ke_target) / th.eta_mass[0];
  else th.eta_dotdot[0] = 0.0;
  const double ncfac = 1.0;
  double expfac;
  for (int ich = mtchain - 1; ich > 0; ich--) {
    expfac = std::exp(-ncfac * dt8 * th.eta_dot[ich + 1]);
    th.eta_dot[ich] *= expfac;
    th.eta_dot[ich] += th.eta_dotdot[ich] * ncfac * dt4;
    th.eta_dot[ich] *= th.tdrag_factor;
    th.eta_dot[ich] *= expfac;
  }
  expfac = std::exp(-ncfac * dt8 * th.eta_dot[1]);
  th.eta_dot[0] *= expfac;
  th.eta_dot[0] += th.eta_dotdot[0] * ncfac * dt4;
  th.eta_dot[0] *= th.tdrag_factor;
  th.eta_dot[0] *= expfac;
  double factor_eta = std::exp(-ncfac * dthalf * th.eta_dot[0]);
  for (auto& vv : v) vv = factor_eta * vv;
  th.temperature = th.temperature * factor_eta * factor_eta;
  kecurrent = th.tdof * u.boltz * th.temperature;
  if (th.eta_mass[0] > 0.0) th.eta_dotdot[0] = (kecurrent - th.ke_target) / th.eta_mass[0];
  else th.eta_dotdot[0] = 0.0;
  for (int ich = 0; ich < mtchain; ich++) th.eta[ich] += ncfac * dthalf * th.eta_dot[ich];
  th.eta_dot[0] *= expfac;
  th.eta_dot[0] += th.eta_dotdot[0] * ncfac * dt4;
  th.eta_dot[0] *= expfac;
  for (int ich = 1; ich < mtchain; ich++) {
    expfac = std::exp(-ncfac * dt8 * th.eta_dot[ich + 1]);
    th.eta_dot[ich] *= expfac;
    th.eta_dotdot[ich] = (th.eta_mass[ich - 1] * th.eta_dot[ich - 1] * th.eta_dot[ich - 1] -
                          u.boltz * th.t_target) / th.eta_mass[ich];
    th.eta_dot[ich] += th.eta_dotdot[ich] * ncfac * dt4;
    th.eta_dot[ich] *= expfac;
  }
}

// ------------------------------------------------------------------ a18: SHAKE / RATTLE
void System::shake(const std::vector<double>& old_x, const std::vector<double>& old_v) {
  // NewConstraintAWaterBondAngleWorklet, framework/run/worklet/MolecularWorklet.h:2367-2645.
  // Unconstrained update from the pre-step state, then three Lagrange multipliers by fixed-point
  // iteration; bond 1.0 and 109.47 degrees are hard-coded there (:2418-2421).
  const int na = (int)angle_atoms.size() / 3;
  const double dt = p.timestep, fmt2v = u.fmt2v;
  shake_virial_atom.assign(6 * na, 0.0);
  const double bond1 = 1.0, bond2 = 1.0;
  const double bond12 = std::sqrt(bond1 * bond1 + bond2 * bond2 -
                                  2.0 * bond1 * bond2 * std::cos((109.4700 / 180.0) * kPif));
  for (int a = 0; a < na; ++a) {
    int id[3] = {angle_atoms[3 * a], angle_atoms[3 * a + 1], angle_atoms[3 * a + 2]};
    double sp[3][3];
    for (int t = 0; t < 3; ++t)
      for (int k = 0; k < 3; ++k) {
        int i = id[t];
        sp[t][k] = old_x[3 * i + k] + old_v[3 * i + k] * dt + 0.5 * dt * dt * f[3 * i + k] / m[i] * fmt2v;
      }
    auto mdv = [&](const double* a_, const double* b_, double out[3]) {
      for (int k = 0; k < 3; ++k) out[k] = a_[k] - b_[k];
      min_image(out);
    };
    double r01[3], r12[3], r20[3], s10[3], s21[3], s02[3];
    mdv(&old_x[3 * id[1]], &old_x[3 * id[0]], r01);
    mdv(&old_x[3 * id[2]], &old_x[3 * id[1]], r12);
    mdv(&old_x[3 * id[0]], &old_x[3 * id[2]], r20);
    mdv(sp[0], sp[1], s10);
    mdv(sp[1], sp[2], s21);
    mdv(sp[2], sp[0], s02);
    auto dot = [](const double* a_, const double* b_) { return a_[0] * b_[0] + a_[1] * b_[1] + a_[2] * b_[2]; };
    double r01sq = dot(r01, r01), r02sq = dot(r20, r20), r12sq = dot(r12, r12);
    double s01sq = dot(s10, s10), s02sq = dot(s02, s02), s12sq = dot(s21, s21);
    double im0 = 1.0 / m[id[0]], im1 = 1.0 / m[id[1]], im2 = 1.0 / m[id[2]];
    double a11 = 2.0 * (im0 + im1) * dot(s10, r01);
    double a12 = -2.0 * im1 * dot(s10, r12);
    double a13 = -2.0 * im0 * dot(s10, r20);
    double a21 = -2.0 * im1 * dot(s21, r01);
    double a22 = 2.0 * (im1 + im2) * dot(s21, r12);
    double a23 = -2.0 * im2 * dot(s21, r20);
    double a31 = -2.0 * im0 * dot(s02, r01);
    double a32 = -2.0 * im2 * dot(s02, r12);
    double a33 = 2.0 * (im0 + im2) * (dot(s02, r20));
    double determ = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a11 * a23 * a32 -
                    a12 * a21 * a33 - a13 * a22 * a31;
    if (std::fabs(determ) < 0.0001) status |= 2;  // reference prints "Shake determinant = 0.0"
    double di = 1.0 / determ;
    double a11i = di * (a22 * a33 - a23 * a32);
    double a12i = -di * (a12 * a33 - a13 * a32);
    double a13i = di * (a12 * a23 - a13 * a22);
    double a21i = -di * (a21 * a33 - a23 * a31);
    double a22i = di * (a11 * a33 - a13 * a31);
    double a23i = -di * (a11 * a23 - a13 * a21);
    double a31i = di * (a21 * a32 - a22 * a31);
    double a32i = -di * (a11 * a32 - a12 * a31);
    double a33i = di * (a11 * a22 - a12 * a21);
    double r0120 = dot(r01, r20), r0112 = dot(r01, r12), r2012 = dot(r20, r12);
    double q1_0101 = (im0 + im1) * (im0 + im1) * r01sq, q1_1212 = im1 * im1 * r12sq,
           q1_2020 = im0 * im0 * r02sq, q1_0120 = -2.0 * (im0 + im1) * im0 * r0120,
           q1_0112 = -2.0 * (im0 + im1) * im1 * r0112, q1_2012 = 2.0 * im0 * im1 * r2012;
    double q2_0101 = im1 * im1 * r01sq, q2_1212 = (im1 + im2) * (im1 + im2) * r12sq,
           q2_2020 = im2 * im2 * r02sq, q2_0120 = 2.0 * im1 * im2 * r0120,
           q2_0112 = -2.0 * (im1 + im2) * im1 * r0112, q2_2012 = -2.0 * (im1 + im2) * im2 * r2012;
    double q3_0101 = im0 * im0 * r01sq, q3_1212 = im2 * im2 * r12sq,
           q3_2020 = (im0 + im2) * (im0 + im2) * r02sq, q3_0120 = -2.0 * (im0 + im2) * im0 * r0120,
           q3_0112 = 2.0 * im0 * im2 * r0112, q3_2012 = -2.0 * (im0 + im2) * im2 * r2012;
    const double tolerance = 0.00001;
    const int max_iter = 5000;
    double l01 = 0.0, l20 = 0.0, l12 = 0.0;
    int niter = 0, done = 0;
    while (!done && niter < max_iter) {
      double quad1 = q1_0101 * l01 * l01 + q1_2020 * l20 * l20 + q1_1212 * l12 * l12 +
                     q1_0120 * l01 * l20 + q1_0112 * l01 * l12 + q1_2012 * l20 * l12;
      double quad2 = q2_0101 * l01 * l01 + q2_2020 * l20 * l20 + q2_1212 * l12 * l12 +
                     q2_0120 * l01 * l20 + q2_0112 * l01 * l12 + q2_2012 * l20 * l12;
      double quad3 = q3_0101 * l01 * l01 + q3_2020 * l20 * l20 + q3_1212 * l12 * l12 +
                     q3_0120 * l01 * l20 + q3_0112 * l01 * l12 + q3_2012 * l20 * l12;
      double b1 = bond1 * bond1 - s01sq - quad1;
      double b2 = bond2 * bond2 - s12sq - quad2;
      double b3 = bond12 * bond12 - s02sq - quad3;
      double l01n = a11i * b1 + a12i * b2 + a13i * b3;
      double l12n = a21i * b1 + a22i * b2 + a23i * b3;
      double l20n = a31i * b1 + a32i * b2 + a33i * b3;
      done = 1;
      if (std::fabs(l01n - l01) > tolerance) done = 0;
      if (std::fabs(l20n - l20) > tolerance) done = 0;
      if (std::fabs(l12n - l12) > tolerance) done = 0;
      l01 = l01n;
      l20 = l20n;
      l12 = l12n;
      if (std::isnan(l01) || std::isnan(l20) || std::isnan(l12) || std::fabs(l01) > 1e20 ||
          std::fabs(l20) > 1e20 || std::fabs(l12) > 1e20) {
        done = 1;
        status |= 1;
      }
      niter++;
    }
    if (!done) status |= 4;
    double pc[3][3];
    for (int k = 0; k < 3; ++k) {
      pc[0][k] = l01 * r01[k] * im0 - l20 * r20[k] * im0;
      pc[1][k] = l12 * r12[k] * im1 - l01 * r01[k] * im1;
      pc[2][k] = l20 * r20[k] * im2 - l12 * r12[k] * im2;
    }
    for (int t = 0; t < 3; ++t) {
      int i = id[t];
      for (int k = 0; k < 3; ++k) {
        double sv = old_v[3 * i + k] + 0.5 * dt * f[3 * i + k] / m[i] * fmt2v;
        v[3 * i + k] = sv + pc[t][k] / dt;
        double xx = sp[t][k] + pc[t][k];
        int img = image[3 * i + k];
        // wrap rule of the constraint worklet (MolecularWorklet.h:2580-2600): strict > on top
        if (xx < lo[k]) {
          xx += (hi[k] - lo[k]);
          img -= 1;
        }
        if (xx > hi[k]) {
          xx -= (hi[k] - lo[k]);
          img += 1;
        }
        x[3 * i + k] = xx;
        image[3 * i + k] = img;
      }
    }
    double dtfsq = 0.5 * dt * dt * fmt2v;
    l01 = l01 / dtfsq;
    l20 = l20 / dtfsq;
    l12 = l12 / dtfsq;
    double* sv = &shake_virial_atom[6 * a];
    sv[0] = l01 * r01[0] * r01[0] + l20 * r20[0] * r20[0] + l12 * r12[0] * r12[0];
    sv[1] = l01 * r01[1] * r01[1] + l20 * r20[1] * r20[1] + l12 * r12[1] * r12[1];
    sv[2] = l01 * r01[2] * r01[2] + l20 * r20[2] * r20[2] + l12 * r12[2] * r12[2];
    sv[3] = l01 * r01[0] * r01[1] + l20 * r20[0] * r20[1] + l12 * r12[0] * r12[1];
    sv[4] = l01 * r01[0] * r01[2] + l20 * r20[0] * r20[2] + l12 * r12[0] * r12[2];
    sv[5] = l01 * r01[1] * r01[2] + l20 * r20[1] * r20[2] + l12 * r12[1] * r12[2];
  }
}

void System::rattle(const std::vector<double>& old_v) {
  // NewConstraintBWaterBondAngleWorklet, framework/run/worklet/MolecularWorklet.h:2647-2832
  const int na = (int)angle_atoms.size() / 3;
  const double dt = p.timestep, fmt2v = u.fmt2v;
  for (int a = 0; a < na; ++a) {
    int id[3] = {angle_atoms[3 * a], angle_atoms[3 * a + 1], angle_atoms[3 * a + 2]};
    double sv[3][3];
    for (int t = 0; t < 3; ++t)
      for (int k = 0; k < 3; ++k) {
        int i = id[t];
        sv[t][k] = old_v[3 * i + k] + 0.5 * dt * f[3 * i + k] / m[i] * fmt2v;
      }
    auto mdv = [&](const double* a_, const double* b_, double out[3]) {
      for (int k = 0; k < 3; ++k) out[k] = a_[k] - b_[k];
      min_image(out);
    };
    auto dot = [](const double* a_, const double* b_) { return a_[0] * b_[0] + a_[1] * b_[1] + a_[2] * b_[2]; };
    double r01[3], r12[3], r20[3];
    mdv(&x[3 * id[1]], &x[3 * id[0]], r01);
    mdv(&x[3 * id[2]], &x[3 * id[1]], r12);
    mdv(&x[3 * id[0]], &x[3 * id[2]], r20);
    double sv10[3], sv21[3], sv02[3];
    for (int k = 0; k < 3; ++k) {
      sv10[k] = sv[0][k] - sv[1][k];
      sv21[k] = sv[1][k] - sv[2][k];
      sv02[k] = sv[2][k] - sv[0][k];
    }
    double im0 = 1.0 / m[id[0]], im1 = 1.0 / m[id[1]], im2 = 1.0 / m[id[2]];
    double A[3][3];
    A[0][0] = (im1 + im0) * dot(r01, r01);
    A[0][1] = -im1 * dot(r01, r12);
    A[0][2] = (-im0) * dot(r01, r20);
    A[1][0] = A[0][1];
    A[1][1] = (im1 + im2) * dot(r12, r12);
    A[1][2] = -(im2)*dot(r20, r12);
    A[2][0] = A[0][2];
    A[2][1] = A[1][2];
    A[2][2] = (im0 + im2) * dot(r20, r20);
    double c[3] = {-dot(sv10, r01), -dot(sv21, r12), -dot(sv02, r20)};
    double determ = A[0][0] * A[1][1] * A[2][2] + A[0][1] * A[1][2] * A[2][0] +
                    A[0][2] * A[1][0] * A[2][1] - A[0][0] * A[1][2] * A[2][1] -
                    A[0][1] * A[1][0] * A[2][2] - A[0][2] * A[1][1] * A[2][0];
    if (std::fabs(determ) < 0.0001) status |= 8;
    double di = 1.0 / determ;
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
    for (int i = 0; i < 3; i++) {
      l[i] = 0;
      for (int j = 0; j < 3; j++) l[i] += ai[i][j] * c[j];
    }
    for (int k = 0; k < 3; ++k) {
      v[3 * id[0] + k] = sv[0][k] + (l[0] * r01[k] * im0 - l[2] * r20[k] * im0);
      v[3 * id[1] + k] = sv[1][k] + (l[1] * r12[k] * im1 - l[0] * r01[k] * im1);
      v[3 * id[2] + k] = sv[2][k] + (l[2] * r20[k] * im2 - l[1] * r12[k] * im2);
    }
  }
}

// ------------------------------------------------------------------ Init / step
void System::init() {
  // ExecutionNVT::Init (ExecutionNVT.cpp:60-74): locator, InitialCondition (PreForce, dof, chain
  // set-up, :139-187 + SetUp :1106-1122), first ComputeForce.
  step = 0;
  build_cells();
  if (p.coulomb == RBMD_COUL_RBE) sample_k();
  // Computedof, ExecutionMD.cpp:1251-1261
  th.tdof = 3.0 * N - 3;
  if (p.fix_shake == RBMD_SHAKE_TRUE) th.tdof = th.tdof - N;
  th.t_freq = 1 / p.temperature[2];
  th.tdrag_factor = 1.0 - (p.timestep * th.t_freq * 0.0 / 1);
  for (int k = 0; k < 3; ++k) th.eta[k] = th.eta_dot[k] = th.eta_dotdot[k] = 0.0;
  th.eta_dot[3] = 0;
  compute_tempe();
  compute_temp_target();
  th.eta_mass[0] = th.tdof * u.boltz * th.t_target / (th.t_freq * th.t_freq);
  for (int ich = 1; ich < 3; ich++) th.eta_mass[ich] = u.boltz * th.t_target / (th.t_freq * th.t_freq);
  for (int ich = 1; ich < 3; ich++)
    th.eta_dotdot[ich] = (th.eta_mass[ich - 1] * th.eta_dot[ich - 1] * th.eta_dot[ich - 1] -
                          u.boltz * th.t_target) / th.eta_mass[ich];
  if (mtk()) mtk_setup();
  compute_force();
}

void System::step_once() {
  // Executioner::TakeStep (framework/executioner/Executioner.cpp:112-117) -> ExecutionNVT
  // PreSolve/Solve (framework/run/ExecutionNVT.cpp:76-135)
  if (mtk()) {
    step_mtk();
    return;
  }
  step += 1;
  if (p.coulomb == RBMD_COUL_RBE) sample_k();
  const bool shk = (p.fix_shake == RBMD_SHAKE_TRUE) && !angle_atoms.empty();
  std::vector<double> old_x, old_v, old_v2;
  if (p.temp_ctrl == RBMD_TC_NOSE_HOOVER) {
    compute_temp_target();  // InitialIntegrate, ExecutionNVT.cpp:1149-1158
    nhc_integrate();
    update_velocity(&old_v);
    update_position(&old_x);
    if (shk) shake(old_x, old_v);
    compute_force();
    update_velocity(&old_v2);  // FinalIntegrate, ExecutionNVT.cpp:1160-1170
    compute_tempe();
    nhc_integrate();
    if (shk) rattle(old_v2);
  } else {
    update_velocity(&old_v);
    update_position(&old_x);
    if (shk) shake(old_x, old_v);
    compute_force();
    update_velocity(&old_v2);
    if (shk) rattle(old_v2);
    compute_tempe();
    if (p.temp_ctrl == RBMD_TC_RESCALE) {  // UpdateVelocityByTempConType, ExecutionNVT.cpp:270-291
      double coeff = std::sqrt(p.temperature[0] / th.temperature);
      for (auto& vv : v) vv = coeff * vv;
    } else if (p.temp_ctrl == RBMD_TC_BERENDSEN) {
      double dtt = p.timestep / p.temperature[2];
      double coeff = std::sqrt(1.0 + dtt * (p.temperature[0] / th.temperature - 1.0));
      for (auto& vv : v) vv = coeff * vv;
    }
    // ExecutionNPT::Solve (ExecutionNPT.cpp:90-122): the same sequence, then the barostat
    if (p.ensemble == RBMD_ENS_NPT) barostat_berendsen();
  }
}

// ------------------------------------------------------------------ NPT Berendsen barostat
void System::pressure_scalar(double vir[6], double& press) const {
  // ExecutionMD::ComputeVirial (ExecutionMD.cpp:1263-1370) and Compute_Pressure_Scalar
  // (ExecutionNPT.cpp:1429-1447, ExecutionNVT.cpp:1258-1276).  The temperature is PARA_TEMPT as
  // ComputeTempe left it, before the end-of-step velocity rescale.
  for (int k = 0; k < 6; ++k) vir[k] = virial[k];
  if (p.fix_shake == RBMD_SHAKE_TRUE)
    for (size_t a = 0; a < shake_virial_atom.size() / 6; ++a)
      for (int k = 0; k < 6; ++k) vir[k] += shake_virial_atom[6 * a + k];
  if (p.force_field == RBMD_FF_EAM)
    for (int k = 0; k < 6; ++k) vir[k] = 0;
  press = (th.tdof * u.boltz * th.temperature + vir[0] + vir[1] + vir[2]) / 3.0 * (1.0 / dv.volume) * u.nktv2p;
}

void System::barostat_berendsen() {
  // ExecutionNPT::fix_press_berendsen (ExecutionNPT.cpp:1334-1368): isotropic dilation
  // mu = (1 - dt / P_damp (P_target - P) / B)^(1/3), P_target ramped from P_start to P_stop over the
  // run; remap (:1506-1538) scales the range about its centre and carries every atom along in
  // reduced coordinates (X2Lamda / Lamda2X worklets, RunWorklet.cpp:2638-2703); ApplyPbc
  // (ExecutionMD.cpp:1239-1249) wraps with the new range; the locator is rebuilt.
  double vir[6], press;
  pressure_scalar(vir, press);
  baro_pressure = press;
  for (int k = 0; k < 6; ++k) baro_virial[k] = vir[k];
  double delta = (double)step;  // currentstep - beginstep, beginstep = 0
  if (delta != 0.0) delta = delta / (double)p.num_steps;
  const double dt_over_period = p.timestep / p.pressure[2];
  const double bulkmodulus_inv = 1.0 / p.bulk_modulus;
  const double p_target = p.pressure[0] + delta * (p.pressure[1] - p.pressure[0]);
  const double dilation = std::pow(1.0 - dt_over_period * (p_target - press) * bulkmodulus_inv, 1.0 / 3.0);
  double nlo[3], nhi[3];
  bool ok = std::isfinite(dilation) && dilation > 0.0;
  const double rc = p.cut_off;
  int ncell = 1;
  for (int k = 0; k < 3 && ok; ++k) {
    const double ctr = 0.5 * (lo[k] + hi[k]);
    nlo[k] = (lo[k] - ctr) * dilation + ctr;
    nhi[k] = (hi[k] - ctr) * dilation + ctr;
    const double nL = nhi[k] - nlo[k];
    const int dims = std::max(1, (int)(nL / (rc / dv.num_cycles)));
    ncell *= dims;
    if (!(nL >= kBoxShrink * L0[k] && nL <= kBoxGrow * L0[k]) || dims < dv.num_cycles) ok = false;
  }
  if (!ok || ncell > ncell_cap) {
    status |= RBMD_STATUS_BOX_RANGE;
    return;
  }
  const double olo[3] = {lo[0], lo[1], lo[2]};
  const double hinv[3] = {1.0 / L[0], 1.0 / L[1], 1.0 / L[2]};  // set_global_box h_inv of the old box
  set_box(nlo, nhi);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) {
      double& xx = x[3 * i + k];
      const double lamda = hinv[k] * (xx - olo[k]);
      xx = L[k] * lamda + lo[k];
      if (xx < lo[k]) {
        xx += L[k];
        image[3 * i + k] -= 1;
      } else if (xx >= hi[k]) {
        xx -= L[k];
        image[3 * i + k] += 1;
      }
    }
  build_cells();
}

// ------------------------------------------------------------------ NPT MTK barostat
// ExecutionNPT with temp_ctrl_type and press_ctrl_type NOSE_HOOVER: an isotropic
// Martyna-Tobias-Klein barostat (p_flag 1 1 1, pdim 3) with a 3-link chain on the barostat
// velocity, integrated around velocity Verlet (ExecutionNPT.cpp:145-232, 1545-2066).
void System::mtk_setup() {
  // SetUp, barostat part (ExecutionNPT.cpp:1573-1602); t_target of step 0
  const double p_freq = 1 / p.pressure[2], p_freq_max = p_freq;
  const double kt = u.boltz * th.t_target;
  const double nkt = (N + 1) * kt;
  for (int i = 0; i < 3; ++i) bs.omega_mass[i] = nkt / (p_freq * p_freq);
  bs.etap_mass[0] = u.boltz * th.t_target / (p_freq_max * p_freq_max);
  for (int ich = 1; ich < 3; ich++) bs.etap_mass[ich] = u.boltz * th.t_target / (p_freq_max * p_freq_max);
  for (int ich = 1; ich < 3; ich++)
    bs.etap_dotdot[ich] = (bs.etap_mass[ich - 1] * bs.etap_dot[ich - 1] * bs.etap_dot[ich - 1] -
                           u.boltz * th.t_target) / bs.etap_mass[ich];
}

void System::nhc_press_integrate() {
  // NHCPressIntegrate, ExecutionNPT.cpp:1831-1915 (mpchain 3, nc_pchain 1, no drag)
  const int mpchain = 3;
  const double dt = p.timestep, dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  const double kt = u.boltz * th.t_target;
  const double pdrag_factor = 1.0;
  double kecurrent = 0.0;
  for (int i = 0; i < 3; ++i) kecurrent += bs.omega_mass[i] * bs.omega_dot[i] * bs.omega_dot[i];
  const double lkt_press = kt;
  bs.etap_dotdot[0] = (kecurrent - lkt_press) / bs.etap_mass[0];
  const double ncfac = 1.0;
  double expfac;
  for (int ich = mpchain - 1; ich > 0; ich--) {
    expfac = std::exp(-ncfac * dt8 * bs.etap_dot[ich + 1]);
    bs.etap_dot[ich] *= expfac;
    bs.etap_dot[ich] += bs.etap_dotdot[ich] * ncfac * dt4;
    bs.etap_dot[ich] *= pdrag_factor;
    bs.etap_dot[ich] *= expfac;
  }
  expfac = std::exp(-ncfac * dt8 * bs.etap_dot[1]);
  bs.etap_dot[0] *= expfac;
  bs.etap_dot[0] += bs.etap_dotdot[0] * ncfac * dt4;
  bs.etap_dot[0] *= pdrag_factor;
  bs.etap_dot[0] *= expfac;
  for (int ich = 0; ich < mpchain; ich++) bs.etap[ich] += ncfac * dthalf * bs.etap_dot[ich];
  const double factor_etap = std::exp(-ncfac * dthalf * bs.etap_dot[0]);
  for (int i = 0; i < 3; ++i) bs.omega_dot[i] *= factor_etap;
  kecurrent = 0.0;
  for (int i = 0; i < 3; ++i) kecurrent += bs.omega_mass[i] * bs.omega_dot[i] * bs.omega_dot[i];
  bs.etap_dotdot[0] = (kecurrent - lkt_press) / bs.etap_mass[0];
  bs.etap_dot[0] *= expfac;
  bs.etap_dot[0] += bs.etap_dotdot[0] * ncfac * dt4;
  bs.etap_dot[0] *= expfac;
  for (int ich = 1; ich < mpchain; ich++) {
    expfac = std::exp(-ncfac * dt8 * bs.etap_dot[ich + 1]);
    bs.etap_dot[ich] *= expfac;
    bs.etap_dotdot[ich] = (bs.etap_mass[ich - 1] * bs.etap_dot[ich - 1] * bs.etap_dot[ich - 1] -
                           u.boltz * th.t_target) / bs.etap_mass[ich];
    bs.etap_dot[ich] += bs.etap_dotdot[ich] * ncfac * dt4;
    bs.etap_dot[ich] *= expfac;
  }
}

void System::compute_press_target() {
  // ComputePressTarget, ExecutionNPT.cpp:1631-1669.  The division by pdim sits inside the loop
  // there, so p_hydro = ((P/3 + P)/3 + P)/3 for an isotropic target P; kept as written.
  bs.p_hydro = 0.0;
  for (int i = 0; i < 3; ++i) {
    double pt;
    if (p.pressure[1] == p.pressure[0]) {
      pt = p.pressure[0];
    } else {
      double delta = (double)step;
      if (delta != 0.0) delta = delta / (double)p.num_steps;
      pt = p.pressure[0] + delta * (p.pressure[1] - p.pressure[0]);
    }
    bs.p_hydro += pt;
    bs.p_hydro /= 3;
  }
}

void System::nh_omega_dot() {
  // NHOmegaDot, ExecutionNPT.cpp:1942-1986 (mtk_flag 1, no drag); volume from PARA_BOX
  const double dthalf = 0.5 * p.timestep;
  const double volume = L[0] * L[1] * L[2];
  bs.mtk_term1 = th.tdof * u.boltz * th.temperature;
  bs.mtk_term1 /= 3 * N;
  for (int i = 0; i < 3; ++i) {
    const double f_omega = (bs.p_current - bs.p_hydro) * volume / (bs.omega_mass[i] * u.nktv2p) +
                           bs.mtk_term1 / bs.omega_mass[i];
    bs.omega_dot[i] += f_omega * dthalf;
  }
  bs.mtk_term2 = 0.0;
  for (int i = 0; i < 3; ++i) bs.mtk_term2 += bs.omega_dot[i];
  bs.mtk_term2 /= 3 * N;
}

void System::nh_v_press() {
  // NH_V_Press, ExecutionNPT.cpp:1988-1997: the per-dimension factor is applied twice
  const double dt4 = 0.25 * p.timestep;
  double fac[3];
  for (int k = 0; k < 3; ++k) fac[k] = std::exp(-dt4 * (bs.omega_dot[k] + bs.mtk_term2));
  for (int rep = 0; rep < 2; ++rep)
    for (int i = 0; i < N; ++i)
      for (int k = 0; k < 3; ++k) v[3 * i + k] = fac[k] * v[3 * i + k];
}

void System::mtk_remap() {
  // ReMap, ExecutionNPT.cpp:1999-2066: the range scaled by exp(dto omega_dot) about the fixed point
  // (the range centre set_global_box stored), atoms carried along in reduced coordinates, no wrap.
  const double dto = 0.5 * p.timestep;
  const double rc = p.cut_off;
  double nlo[3], nhi[3];
  bool ok = true;
  int ncell = 1;
  for (int k = 0; k < 3; ++k) {
    const double fixedpoint = 0.5 * (lo[k] + hi[k]);
    const double expfac = std::exp(dto * bs.omega_dot[k]);
    nlo[k] = (lo[k] - fixedpoint) * expfac + fixedpoint;
    nhi[k] = (hi[k] - fixedpoint) * expfac + fixedpoint;
    const double nL = nhi[k] - nlo[k];
    const int dims = (std::isfinite(nL) && nL > 0) ? std::max(1, (int)(nL / (rc / dv.num_cycles))) : 0;
    ncell *= std::max(dims, 1);
    if (!(nL >= kBoxShrink * L0[k] && nL <= kBoxGrow * L0[k]) || dims < dv.num_cycles) ok = false;
  }
  if (!ok || ncell > ncell_cap) {
    status |= RBMD_STATUS_BOX_RANGE;
    return;
  }
  const double olo[3] = {lo[0], lo[1], lo[2]};
  const double hinv[3] = {1.0 / L[0], 1.0 / L[1], 1.0 / L[2]};
  set_box(nlo, nhi);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) {
      double& xx = x[3 * i + k];
      const double lamda = hinv[k] * (xx - olo[k]);
      xx = L[k] * lamda + lo[k];
    }
  build_cells();
}

void System::step_mtk() {
  // ExecutionNPT::Solve, NOSE_HOOVER branch (ExecutionNPT.cpp:123-141): InitialIntegrate
  // (:1671-1711), ConstraintA, ComputeForce, FinalIntegrate (:1713-1741), ConstraintB.  RBE
  // samples are drawn after the two half-step remaps, for the box the force is evaluated in.
  step += 1;
  const bool shk = (p.fix_shake == RBMD_SHAKE_TRUE) && !angle_atoms.empty();
  std::vector<double> old_x, old_v, old_v2;
  double vir[6], press;
  nhc_press_integrate();
  compute_temp_target();
  nhc_integrate();
  pressure_scalar(vir, press);
  bs.p_current = press;
  compute_press_target();
  nh_omega_dot();
  nh_v_press();
  update_velocity(&old_v);
  mtk_remap();
  update_position(&old_x);
  mtk_remap();
  if (shk) shake(old_x, old_v);
  if (p.coulomb == RBMD_COUL_RBE) sample_k();
  compute_force();
  update_velocity(&old_v2);
  nh_v_press();
  compute_tempe();
  pressure_scalar(vir, press);
  bs.p_current = press;
  baro_pressure = press;
  for (int k = 0; k < 6; ++k) baro_virial[k] = vir[k];
  nh_omega_dot();
  nhc_integrate();
  nhc_press_integrate();
  if (shk) rattle(old_v2);
}

// ------------------------------------------------------------------ a6 / a8 / a13 / a15 energies
void System::energies(double& e_lj, double& e_coul, double& e_eam) const {
  // LJEnergyVerlet / LJCoulEnergyVerletVirial / SpecialLJCoulEnergyVerletWeightVirial
  // (RunWorklet.cpp:2987-3221) on the full list, and ThermoOutput::ComputeEAMPotentialEnergy
  // (framework/output/ThermoOutput.cpp:293-356).
  e_lj = e_coul = e_eam = 0;
  const double rc = p.cut_off, rc_2 = rc * rc;
  const bool special = !special_offsets.empty();
  if (p.force_field == RBMD_FF_EAM) {
    const double cut = eam_cut, rdr = 1.0 / eam_dr, rdrho = 1.0 / eam_drho;
    std::vector<double> emb_i(N, 0.0), pair_i(N, 0.0);
    par_for((long)(N), [&](long i_l) {
      const int i = (int)i_l;
      double rho = 0;
      double& pair = pair_i[i];
      traverse(i, [&](int j, const double*, const double* r0, double d2) {
        if (!(rc_2 - d2 > 0.0001 && d2 > 0.0001)) return;
        double r[3] = {-r0[0], -r0[1], -r0[2]};
        min_image(r);
        double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        if (rsq < cut * cut && rsq > 0.01) {
          double rr = std::sqrt(rsq);
          rho += eam_rho(rhor_of(type[j]), rr, rdr, eam_nr);
          double pp = rr * rdr + 1.0;
          int mm = std::min((int)pp, eam_nr - 1);
          pp -= mm;
          pp = std::min(pp, 1.0);
          const double* c = z2r_of(type[i], type[j]) + 7 * mm;
          double z2 = ((c[3] * pp + c[4]) * pp + c[5]) * pp + c[6];
          pair += 0.5 * (z2 * (1.0 / rr));
        }
      });
      double pp = rho * rdrho + 1.0;
      int mm = std::max(1, std::min((int)pp, eam_nrho - 1));
      pp -= mm;
      pp = std::min(pp, 1.0);
      const double* c = frho_of(type[i]) + 7 * mm;
      double fpv = (c[0] * pp + c[1]) * pp + c[2];
      double phi = ((c[3] * pp + c[4]) * pp + c[5]) * pp + c[6];
      if (rho > eam_rhomax) phi += fpv * (rho - eam_rhomax);
      emb_i[i] = phi;
    });
    double emb = 0, pair = 0;
    for (int i = 0; i < N; ++i) {
      emb += emb_i[i];
      pair += pair_i[i];
    }
    e_eam = (emb + pair) / N;
    return;
  }
  const bool coul = (p.force_field != RBMD_FF_LJ_CUT);
  std::vector<double> el(N, 0.0), ecl(N, 0.0);
  par_for((long)(N), [&](long i_l) {
    const int i = (int)i_l;
    const int ti = type[i];
    double& sl = el[i];
    double& sc = ecl[i];
    traverse(i, [&](int j, const double*, const double* r0, double d2) {
      if (!(rc_2 - d2 > 0.0001 && d2 > 0.0001)) return;
      double r[3] = {r0[0], r0[1], r0[2]};
      min_image(r);
      double dis_2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      const int tj = type[j];
      double w = (special && coul) ? special_weight(*this, i, j) : 1.0;
      sl += w * lj_energy(dis_2, eps[ti], eps[tj], sig[ti], sig[tj], rc);
      if (coul && dis_2 < rc_2 && dis_2 > 0.0001) {
        double dis = std::sqrt(dis_2);
        double ec = 0.5 * q[i] * q[j] * (1.0 - std::erf(std::sqrt(p.alpha) * dis)) / dis;
        double ef = 0.5 * q[i] * q[j] / dis;
        sc += u.qqr2e * (ec - (special ? (1 - w) * ef : 0.0));
      }
    });
  });
  double sl = 0, sc = 0;
  for (int i = 0; i < N; ++i) {
    sl += el[i];
    sc += ecl[i];
  }
  e_lj = sl / N;
  e_coul = sc / N;
}

void System::thermo(rbmd_thermo* out) {
  // ThermoOutput::ComputePotentialEnergy (ThermoOutput.cpp:144-186) and Compute_Pressure_Scalar
  // (ExecutionNVT.cpp:1258-1276)
  std::memset(out, 0, sizeof(*out));
  out->step = step;
  out->temperature = th.temperature;
  out->tempT_sum = th.tempT_sum;
  out->kinetic_energy = th.tempT_sum / N * 0.5;
  double e_lj, e_coul, e_eam;
  energies(e_lj, e_coul, e_eam);
  out->e_lj = e_lj;
  out->e_coul_near = e_coul;
  out->e_eam = e_eam;
  out->e_bond = e_bond_avg;
  out->e_angle = e_angle_avg;
  out->e_dihedral = e_dihedral_avg;
  if (p.coulomb != RBMD_COUL_NONE && p.force_field != RBMD_FF_LJ_CUT && p.force_field != RBMD_FF_EAM) {
    double sq = 0;
    for (int i = 0; i < N; ++i) sq += q[i] * q[i];
    double self = -std::sqrt(p.alpha / kPi) * sq / N * u.qqr2e;
    double ew = ewald_energy_total(p.kmax);
    out->e_coul_far = u.qqr2e * ew * ((2 * kPi / dv.volume)) / N + self;
  }
  if (p.force_field == RBMD_FF_LJ_CUT) out->potential_energy = e_lj;
  else if (p.force_field == RBMD_FF_LJ_CUT_COUL_LONG) out->potential_energy = e_lj + out->e_coul_far + e_coul;
  else if (p.force_field == RBMD_FF_CVFF)
    out->potential_energy = e_lj + out->e_coul_far + e_coul + e_bond_avg + e_angle_avg + e_dihedral_avg;
  else out->potential_energy = e_eam;
  out->total_energy = out->potential_energy + out->kinetic_energy;
  double vir[6], press;
  pressure_scalar(vir, press);
  if (p.ensemble == RBMD_ENS_NPT && step > 0) {
    // NPT: the pressure of the step is the one the barostat used (PARA_PRESSURE,
    // ExecutionNPT.cpp:1446), taken before the remap
    press = baro_pressure;
    for (int k = 0; k < 6; ++k) vir[k] = baro_virial[k];
  }
  for (int k = 0; k < 6; ++k) out->virial[k] = vir[k];
  out->volume = dv.volume;
  out->pressure = press;
  for (int k = 0; k < 3; ++k) {
    out->nhc_eta[k] = th.eta[k];
    out->box_lo[k] = lo[k];
    out->box_hi[k] = hi[k];
  }
  for (int k = 0; k < 4; ++k) out->nhc_eta_dot[k] = th.eta_dot[k];
  out->status = status;
}

// ------------------------------------------------------------------ EAM input
bool read_funcfl(const std::string& path, EamFile& out) {
  // ExecutionNVT::ReadPotentialFile, framework/run/ExecutionNVT.cpp:899-931
  std::ifstream in(path);
  if (!in.is_open()) return false;
  for (int i = 0; i < 2; ++i) in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  in >> out.nrho >> out.drho >> out.nr >> out.dr >> out.cut;
  if (!in || out.nrho < 5 || out.nr < 5) return false;
  out.frho.assign(out.nrho + 1, 0.0);
  out.zr.assign(out.nr + 1, 0.0);
  out.rhor.assign(out.nr + 1, 0.0);
  for (int i = 0; i < out.nrho; ++i) in >> out.frho[i];
  for (int i = 0; i < out.nr; ++i) in >> out.zr[i];
  for (int i = 0; i < out.nr; ++i) in >> out.rhor[i];
  return (bool)in;
}

static void interpolate(int n, double delta, const std::vector<double>& f, std::vector<double>& s) {
  // ExecutionNVT::interpolate, framework/run/ExecutionNVT.cpp:1033-1068
  auto S = [&](int mm, int c) -> double& { return s[7 * mm + c]; };
  for (int mm = 1; mm <= n; mm++) S(mm, 6) = f[mm];
  S(1, 5) = S(2, 6) - S(1, 6);
  S(2, 5) = 0.5 * (S(3, 6) - S(1, 6));
  S(n - 1, 5) = 0.5 * (S(n, 6) - S(n - 2, 6));
  S(n, 5) = S(n, 6) - S(n - 1, 6);
  for (int mm = 3; mm <= n - 2; mm++)
    S(mm, 5) = ((S(mm - 2, 6) - S(mm + 2, 6)) + 8.0 * (S(mm + 1, 6) - S(mm - 1, 6))) / 12.0;
  for (int mm = 1; mm <= n - 1; mm++) {
    S(mm, 4) = 3.0 * (S(mm + 1, 6) - S(mm, 6)) - 2.0 * S(mm, 5) - S(mm + 1, 5);
    S(mm, 3) = S(mm, 5) + S(mm + 1, 5) - 2.0 * (S(mm + 1, 6) - S(mm, 6));
  }
  S(n, 4) = 0.0;
  S(n, 3) = 0.0;
  for (int mm = 1; mm <= n; mm++) {
    S(mm, 2) = S(mm, 5) / delta;
    S(mm, 1) = 2.0 * S(mm, 4) / delta;
    S(mm, 0) = 3.0 * S(mm, 3) / delta;
  }
}

void build_setfl_splines(int ne, int nrho, double drho, int nr, double dr, const double* frho, const double* rhor,
                         const double* z2r, const int* type_element, int n_types, std::vector<double>& frho_s,
                         std::vector<double>& rhor_s, std::vector<double>& z2r_s, double& rhomax) {
  (void)ne;
  const size_t rf = 7 * (size_t)(nrho + 1), rr = 7 * (size_t)(nr + 1);
  frho_s.assign(rf * n_types, 0.0);
  rhor_s.assign(rr * n_types, 0.0);
  z2r_s.assign(rr * n_types * (n_types + 1) / 2, 0.0);
  // one table: copy the values into rows 1..n and spline them in place of the output slice
  auto table = [&](const double* src, int n, double delta, std::vector<double>& dst, size_t at) {
    std::vector<double> f(n + 1, 0.0), sp(7 * (size_t)(n + 1), 0.0);
    for (int mm = 1; mm <= n; ++mm) f[mm] = src[mm - 1];
    interpolate(n, delta, f, sp);
    std::copy(sp.begin(), sp.end(), dst.begin() + at);
  };
  for (int t = 0; t < n_types; ++t) {
    const int e = type_element[t];
    table(frho + (size_t)e * nrho, nrho, drho, frho_s, t * rf);
    table(rhor + (size_t)e * nr, nr, dr, rhor_s, t * rr);
  }
  for (int i = 0; i < n_types; ++i)
    for (int j = 0; j <= i; ++j) {
      const int a = std::max(type_element[i], type_element[j]), b = std::min(type_element[i], type_element[j]);
      table(z2r + (size_t)(a * (a + 1) / 2 + b) * nr, nr, dr, z2r_s, (size_t)(i * (i + 1) / 2 + j) * rr);
    }
  rhomax = (nrho - 1) * drho;
}

void build_splines(const EamFile& in, std::vector<double>& frho_s, std::vector<double>& rhor_s,
                   std::vector<double>& z2r_s, int& nrho, double& drho, int& nr, double& dr,
                   double& rhomax) {
  // ExecutionNVT::file2array + array2spline, framework/run/ExecutionNVT.cpp:933-1079.  rhor is
  // sized and resampled over nr points here (the reference sizes it by nrho, :979-995).
  const double sixth = 1.0 / 6.0;
  double rmax = 0;
  dr = drho = rmax = rhomax = 0.0;
  dr = std::max(dr, in.dr);
  drho = std::max(drho, in.drho);
  rmax = std::max(rmax, (in.nr - 1) * in.dr);
  rhomax = std::max(rhomax, (in.nrho - 1) * in.drho);
  nr = (int)(rmax / dr + 0.5);
  nrho = (int)(rhomax / drho + 0.5);
  auto lag = [&](const std::vector<double>& src, int nsrc, double h, double r) {
    double pp = r / h + 1.0;
    int k = (int)pp;
    k = std::min(k, nsrc - 2);
    k = std::max(k, 2);
    pp -= k;
    pp = std::min(pp, 2.0);
    double c1 = -sixth * pp * (pp - 1.0) * (pp - 2.0);
    double c2 = 0.5 * (pp * pp - 1.0) * (pp - 2.0);
    double c3 = -0.5 * pp * (pp + 1.0) * (pp - 2.0);
    double c4 = sixth * pp * (pp * pp - 1.0);
    return c1 * src[k - 1] + c2 * src[k] + c3 * src[k + 1] + c4 * src[k + 2];
  };
  std::vector<double> frho(nrho + 1, 0.0), rhor(nr + 1, 0.0), z2r(nr + 1, 0.0);
  for (int mm = 1; mm <= nrho; mm++) frho[mm] = lag(in.frho, in.nrho, in.drho, (mm - 1) * drho);
  for (int mm = 1; mm <= nr; mm++) rhor[mm] = lag(in.rhor, in.nr, in.dr, (mm - 1) * dr);
  for (int mm = 1; mm <= nr; mm++) {
    double zri = lag(in.zr, in.nr, in.dr, (mm - 1) * dr);
    z2r[mm] = 27.2 * 0.529 * zri * zri;
  }
  frho_s.assign(7 * (nrho + 1), 0.0);
  rhor_s.assign(7 * (nr + 1), 0.0);
  z2r_s.assign(7 * (nr + 1), 0.0);
  interpolate(nrho, drho, frho, frho_s);
  interpolate(nr, dr, rhor, rhor_s);
  interpolate(nr, dr, z2r, z2r_s);
}

}  // namespace oracle
