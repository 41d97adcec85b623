// oracle_core.cpp -- set-up, random streams, cell list, RBL traversal and the k-space parts of the
// FP64 oracle.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).  Every function cites the reference file
// and lines it restates; paths are relative to the reference root.
#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "oracle.hpp"

namespace oracle {

Units make_units(int units) {
  // framework/run/ExecutionMD.cpp:329-360 (same expressions, so the doubles match)
  Units u{};
  if (units == RBMD_UNITS_REAL) {
    u.kB = 1.9872067 * std::pow(10.0, -3);
    u.fmt2v = 4.186 * std::pow(10.0, -4);
    u.mvv2e = 1.0 / (4.186 * std::pow(10.0, -4));
    u.qqr2e = 332.06371;
    u.boltz = 0.0019872067;
    u.nktv2p = 68568.415;
  } else if (units == RBMD_UNITS_METAL) {
    u.kB = 8.617343e-5;
    u.fmt2v = 1.0 / 1.0364269e-4;
    u.mvv2e = 1.0364269e-4;
    u.qqr2e = 14.399645;
    u.boltz = 8.617343e-5;
    u.nktv2p = 1.6021765e6;
  } else {
    u.kB = u.fmt2v = u.mvv2e = u.qqr2e = u.boltz = u.nktv2p = 1.0;
  }
  return u;
}

// ------------------------------------------------------------------ Philox4x32-10
void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double u01(uint32_t hi, uint32_t lo) {
  uint64_t bits = ((uint64_t)(hi >> 5) << 26) | (uint64_t)(lo >> 6);
  return (double)bits * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------------ set-up
// ExecStaticTable::Extract (staticTable/ExecStaticTable.h:125-133): (bits & MASK) >> (23 - 8) with
// MASK = 2^26 - 2^15 (:38-39), i.e. the exponent's low three bits over the mantissa's top eight.
int near_key(float r) {
  uint32_t bits;
  std::memcpy(&bits, &r, 4);
  return (int)((bits & (67108864u - 32768u)) >> 15);
}

// G(r) = erfc(sqrt(a) r) / r^2 + 2 sqrt(a) exp(-a r^2) / (sqrt(pi) r), a = 0.1 (the Gnear form,
// ExecForceFunction.h:682-689).  The tabulated points are, for each key, the first point of the
// walk r = 0.1, 0.1001, ... (below 2) or r = 2, 2.001, ... (below 12) with that key (column 2 of the
// table files); keys no walk reaches hold G at the smallest distance with that key.
void near_table(float* out) {
  const double a = 0.1;
  auto G = [a](double r) {
    return std::erfc(std::sqrt(a) * r) / (r * r) + 2 * std::sqrt(a) * std::exp(-a * r * r) / (std::sqrt(kPi) * r);
  };
  for (int k = 0; k < 2048; ++k) {
    // exponent bits 0-2 -> 2^1..2^3 (distances 2..16), bits 3-7 -> 2^-4..2^0 (1/16..2)
    const int low3 = k / 256;
    const double base = low3 < 3 ? std::pow(2.0, 1 + low3) : std::pow(2.0, low3 - 7);
    out[k] = (float)G(base * (1.0 + (k % 256) / 256.0));
  }
  std::vector<bool> done(2048, false);
  const double start[2] = {0.1, 2.0}, stride[2] = {1e-4, 1e-3}, stop[2] = {2.0, 12.0};
  for (int w = 0; w < 2; ++w)
    for (long m = 0; start[w] + (double)m * stride[w] < stop[w]; ++m) {
      const double r = start[w] + (double)m * stride[w];
      const int k = near_key((float)r);
      if (done[k]) continue;
      done[k] = true;
      out[k] = (float)G(r);
    }
}

// TableGnearValue (ExecStaticTable.h:96-123): the entry at the key, no interpolation.  The
// reference indexes before its table for r < 0.1; the entry of r = 0.1 stands in there.
double System::near_g(double dis) const {
  const float d = (float)dis;
  return (double)near_tab[d < 0.1f ? 921 : near_key(d)];
}

System::System(const rbmd_system_desc& d, const rbmd_params& prm) : p(prm) {
  N = d.n_atoms;
  ntypes = d.n_types;
  if (N <= 0 || ntypes <= 0 || !d.position || !d.mass || !d.type || !d.epsilon || !d.sigma)
    throw std::invalid_argument("oracle: incomplete system description");
  u = make_units(p.units);
  for (int k = 0; k < 3; ++k) {
    lo[k] = d.box_lo[k];
    hi[k] = d.box_hi[k];
    L[k] = hi[k] - lo[k];  // PARA_BOX, ModelFileInitCondition.cpp:204
  }
  x.assign(d.position, d.position + 3 * N);
  v.assign(3 * N, 0.0);
  if (d.velocity) v.assign(d.velocity, d.velocity + 3 * N);
  f.assign(3 * N, 0.0);
  image.assign(3 * N, 0);
  if (d.image) image.assign(d.image, d.image + 3 * N);
  q.assign(N, 0.0);
  // EAM systems carry zero charge (ExecutionMD::InitialCondition, ExecutionMD.cpp:168-174)
  if (d.charge && p.force_field != RBMD_FF_EAM) q.assign(d.charge, d.charge + N);
  m.assign(d.mass, d.mass + N);
  type.assign(d.type, d.type + N);
  mol.resize(N);
  for (int i = 0; i < N; ++i) mol[i] = d.molecule ? d.molecule[i] : i;
  eps.assign(d.epsilon, d.epsilon + ntypes);
  sig.assign(d.sigma, d.sigma + ntypes);
  if (p.near_table == RBMD_NEAR_TABLE) {
    near_tab.resize(2048);
    if (d.near_table_values) near_tab.assign(d.near_table_values, d.near_table_values + 2048);
    else near_table(near_tab.data());
  }
  if (d.n_bonds > 0) {
    bond_atoms.assign(d.bond_atoms, d.bond_atoms + 2 * d.n_bonds);
    bond_type.assign(d.bond_type, d.bond_type + d.n_bonds);
    bond_k.assign(d.bond_k, d.bond_k + d.n_bond_types);
    bond_r0.assign(d.bond_r0, d.bond_r0 + d.n_bond_types);
  }
  if (d.n_angles > 0) {
    angle_atoms.assign(d.angle_atoms, d.angle_atoms + 3 * d.n_angles);
    if (d.angle_type) {
      angle_type.assign(d.angle_type, d.angle_type + d.n_angles);
      angle_k.assign(d.angle_k, d.angle_k + d.n_angle_types);
      angle_theta0.assign(d.angle_theta0, d.angle_theta0 + d.n_angle_types);
    }
  }
  if (d.n_dihedrals > 0 && p.force_field == RBMD_FF_CVFF) {
    dihedral_atoms.assign(d.dihedral_atoms, d.dihedral_atoms + 4 * d.n_dihedrals);
    dihedral_type.assign(d.dihedral_type, d.dihedral_type + d.n_dihedrals);
    dihedral_k.assign(d.dihedral_k, d.dihedral_k + d.n_dihedral_types);
    dihedral_sign.assign(d.dihedral_sign, d.dihedral_sign + d.n_dihedral_types);
    dihedral_mult.assign(d.dihedral_multiplicity, d.dihedral_multiplicity + d.n_dihedral_types);
  }
  if (d.special_offsets) {
    special_offsets.assign(d.special_offsets, d.special_offsets + N + 1);
    int ns = special_offsets[N];
    special_ids.assign(d.special_ids, d.special_ids + ns);
    special_weights.assign(d.special_weights, d.special_weights + ns);
  }
  // molecule member lists, ascending atom id (ContTopology source/offsets)
  {
    int maxmol = 0;
    for (int i = 0; i < N; ++i) maxmol = std::max(maxmol, mol[i]);
    std::vector<int> cnt(maxmol + 2, 0);
    for (int i = 0; i < N; ++i) cnt[mol[i] + 1]++;
    for (int k = 1; k < (int)cnt.size(); ++k) cnt[k] += cnt[k - 1];
    mol_offsets = cnt;
    mol_atoms.assign(N, 0);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < N; ++i) mol_atoms[fill[mol[i]]++] = i;
  }
  if (p.force_field == RBMD_FF_EAM) {
    eam_nrho = d.eam_nrho;
    eam_nr = d.eam_nr;
    eam_drho = d.eam_drho;
    eam_dr = d.eam_dr;
    eam_rhomax = d.eam_rhomax;
    eam_cut = d.eam_cut;
    eam_per_type = d.eam_per_type;
    const size_t t = eam_per_type ? (size_t)d.n_types : 1, pairs = eam_per_type ? t * (t + 1) / 2 : 1;
    frho_spline.assign(d.eam_frho_spline, d.eam_frho_spline + 7 * (eam_nrho + 1) * t);
    rhor_spline.assign(d.eam_rhor_spline, d.eam_rhor_spline + 7 * (eam_nr + 1) * t);
    z2r_spline.assign(d.eam_z2r_spline, d.eam_z2r_spline + 7 * (eam_nr + 1) * pairs);
  }

  // ---- derived parameters
  double rc = p.cut_off;
  double rs = (p.neighbor == RBMD_NEIGH_RBL) ? p.r_core : p.cut_off;  // Neighbor.cpp:39-47
  dv.num_cycles = (int)std::ceil(rc / rs);
  {
    const double lo0[3] = {lo[0], lo[1], lo[2]}, hi0[3] = {hi[0], hi[1], hi[2]};
    set_box(lo0, hi0);
  }
  for (int k = 0; k < 3; ++k) L0[k] = L[k];
  if (p.ensemble == RBMD_ENS_NPT) {
    // cell capacity of the largest box the barostat accepts (kBoxGrow x the initial edge)
    ncell_cap = 1;
    for (int k = 0; k < 3; ++k) ncell_cap *= std::max(1, (int)((kBoxGrow * L0[k]) / (rc / dv.num_cycles)));
  }
  dv.rho = N / dv.volume;  // PARA_RHO, ModelFileInitCondition.cpp:207
  // RBL capacity arithmetic: ExecutionMD.cpp:582-592 (near), 772-783 (LJ), 1033-1040 (EAM)
  if (p.neighbor == RBMD_NEIGH_RBL) {
    double coeff = 1.0;
    if (p.force_field != RBMD_FF_EAM) {
      double coeff_rcs = 1.0 + (0.05 / dv.rho - 0.05);
      coeff = (double)(long)std::round(coeff_rcs);
    }
    dv.rs_num = (int)(coeff * dv.rho * std::ceil(4.0 / 3.0 * kPif * rs * rs * rs) + 1);
    dv.rc_num = (int)(coeff * dv.rho * std::ceil(4.0 / 3.0 * kPif * rc * rc * rc) + 1);
    int rcs_num = dv.rc_num - dv.rs_num;
    double random_num = p.neighbor_sample_num;
    double random_rate = random_num / rcs_num;
    dv.pice_num = (int)std::ceil(1.0 / random_rate);
    if (rcs_num <= 0 || dv.pice_num < 1) dv.pice_num = 1;
  } else {
    dv.rs_num = dv.rc_num = 0;
    dv.pice_num = 1;
  }
  f_near.assign(3 * N, 0.0);
  f_far.assign(3 * N, 0.0);
  f_bonded.assign(3 * N, 0.0);
}

void System::set_box(const double nlo[3], const double nhi[3]) {
  // Everything that follows from the box: PARA_RANGE / PARA_BOX / volume, the locator's dims
  // (ContPointLocator::SetRange, locator/ContPointLocator.h:44-73) and the RBE normalisation
  // S = H_x H_y H_z - 1 (ExecForceFunction.h:771-797, RBEPSample.h:40-63).  Called at set-up and
  // by the barostat after each accepted remap.
  const double rc = p.cut_off;
  for (int k = 0; k < 3; ++k) {
    lo[k] = nlo[k];
    hi[k] = nhi[k];
    L[k] = hi[k] - lo[k];
  }
  dv.volume = L[0] * L[1] * L[2];
  dv.ncell = 1;
  for (int k = 0; k < 3; ++k) {
    dv.dims[k] = (int)(L[k] / (rc / dv.num_cycles));
    if (dv.dims[k] < 1) dv.dims[k] = 1;
    dv.d[k] = L[k] / dv.dims[k];
    dv.ncell *= dv.dims[k];
  }
  if (p.coulomb != RBMD_COUL_NONE) {
    double H[3];
    for (int k = 0; k < 3; ++k) {
      const double factor = -(p.alpha * L[k] * L[k]);
      H[k] = 0.0;
      for (int mm = -10; mm <= 10; ++mm) H[k] += std::exp(mm * mm * factor);
      H[k] *= std::sqrt(-(factor) / kPi);
    }
    dv.S = H[0] * H[1] * H[2] - 1;
  }
  for (int k = 0; k < 3; ++k) {
    cells.dims[k] = dv.dims[k];
    cells.d[k] = dv.d[k];
  }
}

void System::min_image(double r[3]) const {
  // ExecPointLocator::MinDistanceVec, framework/locator/ExecPointLocator.h:200-231
  for (int k = 0; k < 3; ++k)
    if (std::fabs(r[k]) > L[k] * 0.5) r[k] -= (r[k] > 0 ? L[k] : -L[k]);
}

// ------------------------------------------------------------------ a1: cell list
void System::build_cells() {
  // BinPointsWorklet + SortByKey + Upper/LowerBounds, framework/locator/ContPointLocator.cxx:38-92.
  // Within a cell the order is ascending atom id (a stable sort of fresh 0..N-1 point ids).
  const int* dims = cells.dims;
  int ncell = dims[0] * dims[1] * dims[2];
  cells.cell_of_atom.assign(N, 0);
  for (int i = 0; i < N; ++i) {
    int ijk[3];
    for (int k = 0; k < 3; ++k) {
      long c = (long)((x[3 * i + k] - lo[k]) / cells.d[k]);
      if (c < 0) c = 0;
      if (c > dims[k] - 1) c = dims[k] - 1;
      ijk[k] = (int)c;
    }
    cells.cell_of_atom[i] = ijk[0] + ijk[1] * dims[0] + ijk[2] * dims[0] * dims[1];
  }
  std::vector<int> count(ncell + 1, 0);
  for (int i = 0; i < N; ++i) count[cells.cell_of_atom[i] + 1]++;
  for (int c = 0; c < ncell; ++c) count[c + 1] += count[c];
  cells.lower.assign(ncell, 0);
  cells.upper.assign(ncell, 0);
  for (int c = 0; c < ncell; ++c) {
    cells.lower[c] = count[c];
    cells.upper[c] = count[c + 1];
  }
  cells.sorted.assign(N, 0);
  std::vector<int> fill(count.begin(), count.end() - 1);
  for (int i = 0; i < N; ++i) cells.sorted[fill[cells.cell_of_atom[i]]++] = i;
}

int System::rbl_offset(int atom) const {
  if (p.rbl_mode != RBMD_RBL_PHILOX || dv.pice_num <= 1) return 0;
  uint32_t ctr[4] = {(uint32_t)atom, 0u, (uint32_t)step, kTagRblOffset};
  uint32_t key[2] = {(uint32_t)p.seed, (uint32_t)(p.seed >> 32)};
  uint32_t out[4];
  philox4x32_10(ctr, key, out);
  return (int)(out[0] % (uint32_t)dv.pice_num);
}

// ------------------------------------------------------------------ a3: RBL lists
void System::rbl_lists(std::vector<int>& ncore, std::vector<int>& nshell,
                       std::vector<std::vector<int>>& ids,
                       std::vector<std::vector<std::array<double, 3>>>* offs) const {
  // ComputeRBLNeighboursOnceWorklet, framework/run/worklet/RunWorklet.cpp:906-980: shell atoms
  // (rs < r < rc) are taken every pice_num-th in traversal order, core atoms (r < rs) all.
  const double rc = p.cut_off, rs = p.r_core;
  const double rc_2 = rc * rc, rs_2 = rs * rs;
  const int pice = dv.pice_num;
  ncore.assign(N, 0);
  nshell.assign(N, 0);
  ids.assign(N, {});
  if (offs) offs->assign(N, {});
  for (int i = 0; i < N; ++i) {
    std::vector<int> core, shell;
    std::vector<std::array<double, 3>> core_off, shell_off;
    int index_shell = rbl_offset(i);
    traverse(i, [&](int j, const double* off, const double*, double dis_2) {
      if (rc_2 - dis_2 > 0.0001 && dis_2 - rs_2 > 0.0001) {
        if (index_shell % pice == 0) {
          shell.push_back(j);
          shell_off.push_back({off[0], off[1], off[2]});
        }
        index_shell++;
      } else if (rs_2 - dis_2 > 0.0001 && dis_2 > 0.0001) {
        core.push_back(j);
        core_off.push_back({off[0], off[1], off[2]});
      }
    });
    ncore[i] = (int)core.size();
    nshell[i] = (int)shell.size();
    ids[i] = core;
    ids[i].insert(ids[i].end(), shell.begin(), shell.end());
    if (offs) {
      (*offs)[i] = core_off;
      (*offs)[i].insert((*offs)[i].end(), shell_off.begin(), shell_off.end());
    }
  }
}

// ------------------------------------------------------------------ a4: full list
void System::verlet_lists(std::vector<std::vector<int>>& ids,
                          std::vector<std::vector<std::array<double, 3>>>& offs) const {
  // ComputeNeighboursWorklet, framework/run/worklet/RunWorklet.cpp:296-355
  const double rc_2 = p.cut_off * p.cut_off;
  ids.assign(N, {});
  offs.assign(N, {});
  for (int i = 0; i < N; ++i) {
    traverse(i, [&](int j, const double* off, const double*, double dis_2) {
      if (rc_2 - dis_2 > 0.0001 && dis_2 > 0.0001) {
        ids[i].push_back(j);
        offs[i].push_back({off[0], off[1], off[2]});
      }
    });
  }
}

// ------------------------------------------------------------------ a10: RBE sampler
namespace {
struct RbeDraws {
  const System* s;
  double alpha;
  double sigma[3];
  double H[3];
  uint32_t key[2];
  bool test;

  // FetchSample_1D, framework/model/RBEPSample.h:115-145 (uniforms from Philox slot t, dim d)
  double gaussian(uint32_t t, int d) const {
    double U1, U2;
    if (test) {
      U1 = 0.5;
      U2 = 0.5;
    } else {
      uint32_t attempt = 0;
      for (; attempt < 64; ) {  // same cap as the CUDA path
        uint32_t ctr[4] = {t, (uint32_t)d | (attempt << 2), (uint32_t)s->step, kTagRbeGauss};
        uint32_t o[4];
        philox4x32_10(ctr, key, o);
        U1 = u01(o[0], o[1]);
        U2 = u01(o[2], o[3]);
        if (!(U1 < 1e-6)) break;
        ++attempt;
      }
    }
    return sigma[d] * std::sqrt(-2.0 * std::log(U1)) * std::cos(2 * kPi * U2) + 0.0;
  }
  double accept_u(uint32_t t, int d) const {
    if (test) return 0.5;
    uint32_t ctr[4] = {t, (uint32_t)d, (uint32_t)s->step, kTagRbeAccept};
    uint32_t o[4];
    philox4x32_10(ctr, key, o);
    return u01(o[0], o[1]);
  }
  // Distribution_P / Distribution_q, RBEPSample.h:85-113
  double dist_P(double xm, int d) const {
    double P_m = std::exp(-std::pow(2 * kPi * xm / s->L[d], 2) / (4 * alpha));
    return P_m / H[d];
  }
  double dist_q(double xm, int d) const {
    double sc = std::sqrt(alpha * std::pow(s->L[d], 2) / std::pow(kPi, 2));
    if (xm == 0) return std::erf((1.0 / 2) / sc);
    return (std::erf(((1.0 / 2) + std::fabs(xm)) / sc) - std::erf((std::fabs(xm) - (1.0 / 2)) / sc)) / 2;
  }
  // MH_Algorithm, RBEPSample.h:64-83
  double mh(double m, uint32_t t, int d) const {
    double x_wait = gaussian(t, d);
    double m_wait = std::round(x_wait);
    double Prob = (dist_P(m_wait, d) / dist_P(m, d)) * (dist_q(m, d) / dist_q(m_wait, d));
    Prob = std::min(Prob, 1.0);
    double uu = accept_u(t, d);
    if (uu <= Prob) m = m_wait;
    return m;
  }
};
}  // namespace

void System::sample_k() {
  // ExecutionNVT::PreForce (framework/run/ExecutionNVT.cpp:332-354) and
  // RBEPSAMPLE::Fetch_P_Sample (framework/model/RBEPSample.h:147-177).  Philox slot t supplies
  // the three per-dimension draws of one chain step; a rejected all-zero vector consumes a slot.
  const int P = p.coulomb_sample_num;
  RbeDraws dr;
  dr.s = this;
  dr.alpha = p.alpha;
  dr.test = (p.random_mode == RBMD_RANDOM_TEST);
  dr.key[0] = (uint32_t)p.seed;
  dr.key[1] = (uint32_t)(p.seed >> 32);
  for (int d = 0; d < 3; ++d) {
    dr.sigma[d] = std::sqrt(p.alpha / 2.0) * L[d] / kPi;
    const double factor = -(p.alpha * L[d] * L[d]);
    dr.H[d] = 0.0;
    for (int mm = -10; mm <= 10; ++mm) dr.H[d] += std::exp(mm * mm * factor);
    dr.H[d] *= std::sqrt(-(factor) / kPi);
  }
  const double eps = 1e-6;
  kspace_m.assign(3 * P, 0);
  // Bounded: a degenerate distribution ends with the error word 32 instead of looping forever.
  const uint32_t tmax = 4096 + 64 * (uint32_t)P;
  uint32_t t = 0;
  double X0[3];
  for (;;) {
    for (int d = 0; d < 3; ++d) X0[d] = std::round(dr.gaussian(t, d));
    ++t;
    if (!(std::fabs(X0[0]) < eps && std::fabs(X0[1]) < eps && std::fabs(X0[2]) < eps)) break;
    if (t >= tmax) {
      status |= 32;
      X0[0] = 1.0;
      X0[1] = X0[2] = 0.0;
      break;
    }
  }
  for (int d = 0; d < 3; ++d) kspace_m[d] = (int)X0[d];
  for (int i = 1; i < P; ++i) {
    if (t >= tmax) {
      status |= 32;
      for (int d = 0; d < 3; ++d) kspace_m[3 * i + d] = (int)X0[d];
      continue;
    }
    double X1[3];
    for (int d = 0; d < 3; ++d) X1[d] = dr.mh(X0[d], t, d);
    ++t;
    for (int d = 0; d < 3; ++d) {
      kspace_m[3 * i + d] = (int)X1[d];
      X0[d] = X1[d];
    }
    if (std::fabs(X1[0]) < eps && std::fabs(X1[1]) < eps && std::fabs(X1[2]) < eps) {
      i = i - 1;
      continue;
    }
  }
}

// ------------------------------------------------------------------ a11: rho(k)
void System::structure_factor() {
  // ComputePnumberChargeStructureFactorWorklet (RunWorklet.cpp:2209-2270) + ReduceByKey
  // (framework/run/ExecutionMD.cpp:469-501): rho_l = sum_j q_j (cos, sin)(k_l . r_j)
  const int P = p.coulomb_sample_num;
  rhok.assign(2 * P, 0.0);
  par_for((long)(P), [&](long l_l) {
    const int l = (int)l_l;
    double kl[3];
    for (int d = 0; d < 3; ++d) kl[d] = 2 * kPi * kspace_m[3 * l + d] / L[d];
    double re = 0, im = 0;
    for (int j = 0; j < N; ++j) {
      double dot = kl[0] * x[3 * j] + kl[1] * x[3 * j + 1] + kl[2] * x[3 * j + 2];
      re += q[j] * std::cos(dot);
      im += q[j] * std::sin(dot);
    }
    rhok[2 * l] = re;
    rhok[2 * l + 1] = im;
  });
}

static void kspace_virial(const double K[3], const double r[3], double F, double v[6]) {
  // ExecForceFunction::ComputeKspaceVirial, framework/forceFunction/ExecForceFunction.h:397-410
  v[0] += (r[0] * K[0] + r[0] * K[0]) * F;
  v[1] += (r[1] * K[1] + r[1] * K[1]) * F;
  v[2] += (r[2] * K[2] + r[2] * K[2]) * F;
  v[3] += (r[0] * K[1] + r[1] * K[0]) * F;
  v[4] += (r[0] * K[2] + r[2] * K[0]) * F;
  v[5] += (r[1] * K[2] + r[2] * K[1]) * F;
}

// ------------------------------------------------------------------ a12: RBE force
void System::rbe_force(std::vector<double>& F, double vir[6]) const {
  // ComputeNewRBEForceWorklet (RunWorklet.cpp:2086-2141), ComputeRBEForceSum_fix and
  // ComputeRBEForce (ExecForceFunction.h:748-769); result is later scaled by qqr2e.
  const int P = p.coulomb_sample_num;
  F.assign(3 * N, 0.0);
  for (int k = 0; k < 6; ++k) vir[k] = 0;
  std::vector<double> vir_atom(6 * (size_t)N, 0.0);
  par_for((long)(N), [&](long i_l) {
    const int i = (int)i_l;
    const double* ri = &x[3 * i];
    double fi[3] = {0, 0, 0}, vi[6] = {0, 0, 0, 0, 0, 0};
    for (int l = 0; l < P; ++l) {
      double kl[3];
      for (int d = 0; d < 3; ++d) kl[d] = 2 * kPi * kspace_m[3 * l + d] / L[d];
      double k2 = kl[0] * kl[0] + kl[1] * kl[1] + kl[2] * kl[2];
      double dot = kl[0] * ri[0] + kl[1] * ri[1] + kl[2] * ri[2];
      double fa = -4 * kPi * q[i];
      double fb = std::cos(dot) * rhok[2 * l + 1];
      double fc = std::sin(dot) * rhok[2 * l];
      double Fs = (fa / (dv.volume * k2)) * (fb - fc);
      for (int d = 0; d < 3; ++d) fi[d] += Fs * kl[d];
      kspace_virial(kl, ri, Fs, vi);
    }
    for (int d = 0; d < 3; ++d) F[3 * i + d] = fi[d] * dv.S / P;
    for (int k = 0; k < 6; ++k) vir_atom[6 * (size_t)i + k] = vi[k] * dv.S / P;
  });
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 6; ++k) vir[k] += vir_atom[6 * (size_t)i + k];
}

// ------------------------------------------------------------------ a14: full Ewald
void System::ewald_force(std::vector<double>& F, double vir[6]) const {
  // ComputeChargeStructureFactorEwald (framework/run/ExecutionMD.cpp:362-403) and
  // ComputeNewFarElectrostaticsWorklet + Computekspace_fix (RunWorklet.cpp:2492-2540,
  // ExecForceFunction.h:712-727); k order i, j, k nested, origin skipped.
  const int* km = p.kmax;
  std::vector<double> K;
  for (int a = -km[0]; a <= km[0]; ++a)
    for (int b = -km[1]; b <= km[1]; ++b)
      for (int c = -km[2]; c <= km[2]; ++c) {
        if (a == 0 && b == 0 && c == 0) continue;
        double kv[3] = {2 * kPi * a / L[0], 2 * kPi * b / L[1], 2 * kPi * c / L[2]};
        K.insert(K.end(), kv, kv + 3);
      }
  const size_t nk = K.size() / 3;
  std::vector<double> rk(2 * nk, 0.0);
  par_for((long)((long)nk), [&](long l_l) {
    const long l = (long)l_l;
    const double* kv = &K[3 * l];
    double re = 0, im = 0;
    for (int j = 0; j < N; ++j) {
      double dot = kv[0] * x[3 * j] + kv[1] * x[3 * j + 1] + kv[2] * x[3 * j + 2];
      re += q[j] * std::cos(dot);
      im += q[j] * std::sin(dot);
    }
    rk[2 * l] = re;
    rk[2 * l + 1] = im;
  });
  F.assign(3 * N, 0.0);
  for (int k = 0; k < 6; ++k) vir[k] = 0;
  std::vector<double> vir_atom(6 * (size_t)N, 0.0);
  par_for((long)(N), [&](long i_l) {
    const int i = (int)i_l;
    const double* ri = &x[3 * i];
    double fi[3] = {0, 0, 0}, vi[6] = {0, 0, 0, 0, 0, 0};
    for (size_t l = 0; l < nk; ++l) {
      const double* kv = &K[3 * l];
      double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      double dot = kv[0] * ri[0] + kv[1] * ri[1] + kv[2] * ri[2];
      double fa = -4 * kPi * q[i];
      double fb = std::exp(-k2 / (4 * p.alpha));
      double Fs = fa / (dv.volume * k2) * fb * (std::cos(dot) * rk[2 * l + 1] - std::sin(dot) * rk[2 * l]);
      for (int d = 0; d < 3; ++d) fi[d] += Fs * kv[d];
      kspace_virial(kv, ri, Fs, vi);
    }
    for (int d = 0; d < 3; ++d) F[3 * i + d] = fi[d];
    for (int k = 0; k < 6; ++k) vir_atom[6 * (size_t)i + k] = vi[k];
  });
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 6; ++k) vir[k] += vir_atom[6 * (size_t)i + k];
}

double System::ewald_energy_total(const int kmax[3]) const {
  // ExecutionMD::ComputeEwaldEnergy, framework/run/ExecutionMD.cpp:405-443
  std::vector<std::array<int, 3>> ks;
  for (int a = -kmax[0]; a <= kmax[0]; ++a)
    for (int b = -kmax[1]; b <= kmax[1]; ++b)
      for (int c = -kmax[2]; c <= kmax[2]; ++c)
        if (!(a == 0 && b == 0 && c == 0)) ks.push_back({a, b, c});
  std::vector<double> terms(ks.size(), 0.0);
  par_for((long)((long)ks.size()), [&](long t_l) {
    const long t = (long)t_l;
        const int a = ks[t][0], b = ks[t][1], c = ks[t][2];
        double kv[3] = {2 * kPi * a / L[0], 2 * kPi * b / L[1], 2 * kPi * c / L[2]};
        double Range_K = std::sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
        double re = 0, im = 0;
        for (int j = 0; j < N; ++j) {
          double dot = kv[0] * x[3 * j] + kv[1] * x[3 * j + 1] + kv[2] * x[3 * j + 2];
          re += q[j] * std::cos(dot);
          im += q[j] * std::sin(dot);
        }
        double rd2 = re * re + im * im;
        terms[t] = std::exp(-Range_K * Range_K / (4 * p.alpha)) * rd2 / (Range_K * Range_K);
  });
  double total = 0.0;
  for (double v : terms) total += v;
  return total;
}

}  // namespace oracle
