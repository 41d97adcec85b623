// engine.cu -- context, system upload, work tables, step orchestration and the C ABI.
//
// Host side of the drop-in boundary: it plays the role of ExecutionMD::Init / ExecutionNVT::Init
// (framework/run/ExecutionMD.cpp:117-134, framework/run/ExecutionNVT.cpp:60-74) and of the
// PreSolve / Solve sequence (ExecutionNVT.cpp:76-135), enqueuing the sm_100a kernels instead of
// VTK-m worklets.  A step is a fixed kernel sequence with no host synchronisation, so the steps of
// a fixed set of systems can be captured once as a CUDA graph and replayed.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <cstdlib>
#include <cstring>

#include "engine.h"

namespace rbmd {

static std::atomic<long long> g_launches{0};
long long launches_issued() { return g_launches.load(); }
void note_launch(int k) { g_launches += k; }

Units make_units(int units) {
  // ExecutionMD::InitParameters, framework/run/ExecutionMD.cpp:329-360
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

// Derived quantities: ContPointLocator::SetRange/SetCutOff/SetRs (locator/ContPointLocator.h:44-73),
// RBL capacity arithmetic (ExecutionMD.cpp:582-592, 772-783, 1033-1040), RBE normalisation S
// (ExecForceFunction.h:771-797).
static void derive(const rbmd_system_desc& d, const rbmd_params& p, rbmd_derived& dv) {
  std::memset(&dv, 0, sizeof(dv));
  double L[3];
  for (int k = 0; k < 3; ++k) L[k] = d.box_hi[k] - d.box_lo[k];
  dv.volume = L[0] * L[1] * L[2];
  dv.rho_system = d.n_atoms / dv.volume;
  const double rc = p.cut_off;
  const double rs = (p.neighbor == RBMD_NEIGH_RBL) ? p.r_core : p.cut_off;
  dv.num_cycles = (int)std::ceil(rc / rs);
  dv.n_cells = 1;
  for (int k = 0; k < 3; ++k) {
    dv.dims[k] = (int)(L[k] / (rc / dv.num_cycles));
    if (dv.dims[k] < 1) dv.dims[k] = 1;
    dv.cell_width[k] = L[k] / dv.dims[k];
    dv.n_cells *= dv.dims[k];
  }
  if (p.neighbor == RBMD_NEIGH_RBL) {
    double coeff = 1.0;
    if (p.force_field != RBMD_FF_EAM) {
      const double coeff_rcs = 1.0 + (0.05 / dv.rho_system - 0.05);
      coeff = (double)(long)std::round(coeff_rcs);
    }
    dv.rs_num = (int)(coeff * dv.rho_system * std::ceil(4.0 / 3.0 * kPif * rs * rs * rs) + 1);
    dv.rc_num = (int)(coeff * dv.rho_system * std::ceil(4.0 / 3.0 * kPif * rc * rc * rc) + 1);
    const int rcs_num = dv.rc_num - dv.rs_num;
    const double random_rate = (double)p.neighbor_sample_num / rcs_num;
    dv.pice_num = (int)std::ceil(1.0 / random_rate);
    if (rcs_num <= 0 || dv.pice_num < 1) dv.pice_num = 1;
  } else {
    dv.pice_num = 1;
  }
  if (p.coulomb != RBMD_COUL_NONE) {
    double H[3];
    for (int k = 0; k < 3; ++k) {
      const double factor = -(p.alpha * L[k] * L[k]);
      H[k] = 0.0;
      for (int m = -10; m <= 10; ++m) H[k] += std::exp(m * m * factor);
      H[k] *= std::sqrt(-(factor) / kPi);
    }
    dv.S_rbe = H[0] * H[1] * H[2] - 1;
  }
}

// ------------------------------------------------------------------------------ context
namespace {
// Profiler record of a batch's pair launch, by traversal layout.
const char* pair_name(const Batch& b) {
  return b.dense == 2 ? "pair_col" : (b.dense ? "pair_tile" : (b.lean ? "pair_lean" : "pair_atom"));
}

// Exact thresholds for the reference's window tests.  fl(c - x) is non-increasing in x, so
// {x : fl(c - x) > e} is a down-set of the floats and thr_below returns its largest element;
// likewise {x : fl(x - c) > e} is an up-set and thr_above returns its smallest element.
template <class T>
T thr_below(T c, T e) {
  const T inf = std::numeric_limits<T>::infinity();
  T x = c - e;
  while (!(c - x > e)) x = std::nextafter(x, -inf);
  while (c - std::nextafter(x, inf) > e) x = std::nextafter(x, inf);
  return x;
}
template <class T>
T thr_above(T c, T e) {
  const T inf = std::numeric_limits<T>::infinity();
  T x = c + e;
  while (!(x - c > e)) x = std::nextafter(x, inf);
  while (std::nextafter(x, -inf) - c > e) x = std::nextafter(x, -inf);
  return x;
}
}  // namespace

Context::Context(const rbmd_device_cfg& c) : cfg(c) {
  cudaSetDevice(cfg.device);
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = cfg.device;
  if (cudaMemPoolCreate(&pool_, &props) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;  // never hand freed memory back at synchronisation points
    cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep);
  } else {
    pool_ = nullptr;
    cudaGetLastError();
  }
}

void* Context::dmalloc(size_t bytes) {
  if (bytes == 0) bytes = 16;
  void* p = nullptr;
  const cudaError_t e = pool_ ? cudaMallocFromPoolAsync(&p, bytes, pool_, stream) : cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void Context::dfree(void* p) {
  if (!p) return;
  if (pool_) cudaFreeAsync(p, stream);
  else cudaFree(p);
}

Context::~Context() {
  cudaStreamSynchronize(stream);
  snapshots_release();
  for (auto& kv : batch_cache_) {
    if (kv.second->graph) cudaGraphExecDestroy(kv.second->graph);
    for (void* p : kv.second->allocs) dfree(p);
    delete kv.second;
  }
  for (System* s : systems_) {
    if (!s) continue;
    for (void* p : s->allocs) dfree(p);
    delete s;
  }
  if (d_sys_) cudaFree(d_sys_);
  cudaStreamSynchronize(stream);
  if (pool_) cudaMemPoolDestroy(pool_);
  for (auto& r : prof.recs)
    for (auto& e : r.second.ev) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  cudaStreamDestroy(stream);
}

int Context::fail(int code, const std::string& msg) {
  last_error = msg;
  return code;
}

int Context::check_cuda(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(RBMD_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  return RBMD_OK;
}

System* Context::find(int id) {
  for (System* s : systems_)
    if (s && s->id == id) return s;
  return nullptr;
}

int Context::ensure_slots(int need) {
  if (need <= slot_cap_) return RBMD_OK;
  int cap = std::max(need, std::max(16, slot_cap_ * 2));
  SysDev* nd = nullptr;
  if (cudaMalloc(&nd, sizeof(SysDev) * cap) != cudaSuccess) return fail(RBMD_ERR_OOM, "system table");
  cudaMemsetAsync(nd, 0, sizeof(SysDev) * cap, stream);
  if (d_sys_) {
    cudaMemcpyAsync(nd, d_sys_, sizeof(SysDev) * slot_cap_, cudaMemcpyDeviceToDevice, stream);
    cudaStreamSynchronize(stream);
    cudaFree(d_sys_);
  }
  d_sys_ = nd;
  slot_cap_ = cap;
  // every cached batch points at the old table
  for (auto& kv : batch_cache_) {
    kv.second->b.sys = d_sys_;
    if (kv.second->graph) {
      cudaGraphExecDestroy(kv.second->graph);
      kv.second->graph = nullptr;
    }
  }
  return RBMD_OK;
}

int Context::upload_record(System* s) {
  cudaMemcpyAsync(d_sys_ + s->slot, &s->dev, sizeof(SysDev), cudaMemcpyHostToDevice, stream);
  return RBMD_OK;
}

// NPT systems change their box on the device every step: bring the host mirror of the record, and
// the derived quantities the getters report, up to date.
int Context::refresh(System* s) {
  if (!s->dev.npt) return RBMD_OK;
  cudaMemcpyAsync(&s->dev, d_sys_ + s->slot, sizeof(SysDev), cudaMemcpyDeviceToHost, stream);
  const int rc = sync();
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) {
    s->dv.dims[k] = s->dev.dims[k];
    s->dv.cell_width[k] = s->dev.d[k];
  }
  s->dv.n_cells = s->dev.ncell;
  s->dv.volume = s->dev.volume;
  s->dv.S_rbe = s->dev.S;
  return RBMD_OK;
}

int64_t Context::estimate_bytes(const rbmd_system_desc& d, const rbmd_params& p) {
  rbmd_derived dv;
  derive(d, p, dv);
  const int64_t n = d.n_atoms;
  int64_t b = n * (32 * 3 + 16 + 12 + 4 * 2 + 32 + 16 + 16 + 8);  // x v f meta image cells sorted sx sxf smeta fp
  if (p.fix_shake == RBMD_SHAKE_TRUE && d.n_angles > 0) b += n * 32 * 3;
  b += (int64_t)dv.n_cells * 16 * (p.ensemble == RBMD_ENS_NPT ? 2 : 1);  // NPT: room for kBoxGrow^3
  const int P = p.coulomb == RBMD_COUL_RBE ? p.coulomb_sample_num : 0;
  int64_t nk = P;
  if (p.coulomb == RBMD_COUL_EWALD)
    nk = (int64_t)(2 * p.kmax[0] + 1) * (2 * p.kmax[1] + 1) * (2 * p.kmax[2] + 1);
  const int64_t nke = p.coulomb != RBMD_COUL_NONE
                          ? (int64_t)(2 * p.kmax[0] + 1) * (2 * p.kmax[1] + 1) * (2 * p.kmax[2] + 1)
                          : 0;
  const int64_t brho = (n + kRhoChunk - 1) / kRhoChunk;
  b += nk * 48 + nke * 48 + brho * 16 * std::max(nk, nke);
  b += (int64_t)(d.n_bonds * 2 + d.n_angles * 3 + d.n_dihedrals * 4) * 48 +
       (int64_t)(d.n_bonds + d.n_angles + d.n_dihedrals) * 76;
  if (d.special_offsets) b += (int64_t)d.special_offsets[n] * 12 + 4 * (n + 1);
  if (p.force_field == RBMD_FF_EAM) {
    size_t nf, nr, nz;
    eam_table_sizes(d, &nf, &nr, &nz);
    b += (int64_t)(nf + nr + nz) * 8;
  }
  if (p.precision == RBMD_PREC_MIXED) b += (int64_t)d.n_types * d.n_types * 8;  // FP32 LJ factors
  if (p.near_table == RBMD_NEAR_TABLE) b += (int64_t)kNearKeys * 4;
  b += ((n + kPairWarps - 1) / kPairWarps) * 72 + ((n + kAtomBlock - 1) / kAtomBlock) * 64 + 4096;
  return b;
}

// ------------------------------------------------------------------------------ add / remove
int Context::add_system(const rbmd_system_desc& d, const rbmd_params& p, int32_t* out_id) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  if (d.n_atoms <= 0 || d.n_types <= 0 || !d.position || !d.mass || !d.type || !d.epsilon || !d.sigma)
    return fail(RBMD_ERR_ARG, "system description: n_atoms, n_types, position, mass, type, epsilon and sigma are required");
  if (p.force_field < 0 || p.force_field > 3 || p.neighbor < 0 || p.neighbor > 1 || p.coulomb < 0 ||
      p.coulomb > 2 || p.precision < 0 || p.precision > 1 || p.temp_ctrl < 0 || p.temp_ctrl > 3)
    return fail(RBMD_ERR_ARG, "unknown enum value in rbmd_params");
  if (!(p.cut_off > 0) || (p.neighbor == RBMD_NEIGH_RBL && !(p.r_core > 0 && p.r_core <= p.cut_off)))
    return fail(RBMD_ERR_ARG, "cut_off must be > 0 and 0 < r_core <= cut_off");
  if (!(p.timestep > 0)) return fail(RBMD_ERR_ARG, "timestep must be > 0");
  if (p.ensemble < 0 || p.ensemble > 2) return fail(RBMD_ERR_ARG, "unknown ensemble");
  if (p.ensemble == RBMD_ENS_NPT) {
    // ExecutionNPT::Solve (ExecutionNPT.cpp:90-141) controls the pressure for BERENDSEN /
    // BERENDSEN (fix_press_berendsen) and NOSE_HOOVER / NOSE_HOOVER (MTK); its other pairings
    // integrate without any pressure control, or not at all (TEMP_RESCALE)
    const bool ber = p.temp_ctrl == RBMD_TC_BERENDSEN && p.press_ctrl == RBMD_PC_BERENDSEN;
    const bool mtk = p.temp_ctrl == RBMD_TC_NOSE_HOOVER && p.press_ctrl == RBMD_PC_NOSE_HOOVER;
    if (!ber && !mtk)
      return fail(RBMD_ERR_UNSUPPORTED,
                  "ensemble NPT needs temp_ctrl / press_ctrl BERENDSEN / BERENDSEN or NOSE_HOOVER / NOSE_HOOVER");
    if (!(p.pressure[2] > 0)) return fail(RBMD_ERR_ARG, "NPT needs a pressure damping time pressure[2] > 0");
    if (ber && !(p.bulk_modulus > 0)) return fail(RBMD_ERR_ARG, "NPT Berendsen needs bulk_modulus > 0");
  }
  if (p.near_table != RBMD_NEAR_ANALYTIC && p.near_table != RBMD_NEAR_TABLE)
    return fail(RBMD_ERR_ARG, "near_table must be RBMD_NEAR_ANALYTIC or RBMD_NEAR_TABLE");
  if (p.near_table == RBMD_NEAR_TABLE && p.cut_off > 12.0)
    return fail(RBMD_ERR_UNSUPPORTED, "near_table: the reference's table ends at r = 12, cut_off is " +
                                          std::to_string(p.cut_off));
  if (p.precision == RBMD_PREC_MIXED && d.n_types > kMaxF32Types)
    return fail(RBMD_ERR_UNSUPPORTED, "mixed precision supports at most " + std::to_string(kMaxF32Types) +
                                          " atom types");
  for (int k = 0; k < 3; ++k)
    if (!(d.box_hi[k] > d.box_lo[k])) return fail(RBMD_ERR_ARG, "box_hi must exceed box_lo");
  for (int i = 0; i < d.n_atoms; ++i) {
    if (d.type[i] < 0 || d.type[i] >= d.n_types) return fail(RBMD_ERR_ARG, "atom type out of range");
    if (!(d.mass[i] > 0)) return fail(RBMD_ERR_ARG, "atom masses must be > 0");
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(d.position[3 * i + k])) return fail(RBMD_ERR_NUMERIC, "non-finite position");
  }
  const bool coul_ff = (p.force_field == RBMD_FF_LJ_CUT_COUL_LONG || p.force_field == RBMD_FF_CVFF);
  if (coul_ff && p.coulomb == RBMD_COUL_NONE)
    return fail(RBMD_ERR_ARG, "a Coulomb force field needs coulomb RBE or EWALD");
  if (p.coulomb != RBMD_COUL_NONE && !(p.alpha > 0)) return fail(RBMD_ERR_ARG, "alpha must be > 0");
  if (p.coulomb == RBMD_COUL_RBE && (p.coulomb_sample_num < 1 || p.coulomb_sample_num > 8192))
    return fail(RBMD_ERR_ARG, "coulomb_sample_num must be in [1, 8192]");
  if (p.force_field == RBMD_FF_EAM &&
      (!d.eam_frho_spline || !d.eam_rhor_spline || !d.eam_z2r_spline || d.eam_nrho < 3 || d.eam_nr < 3))
    return fail(RBMD_ERR_ARG, "EAM needs the three spline tables");
  if (p.force_field == RBMD_FF_EAM && (d.eam_per_type < 0 || d.eam_per_type > 1))
    return fail(RBMD_ERR_ARG, "eam_per_type must be 0 or 1");
  if (d.n_bonds > 0 && (!d.bond_atoms || !d.bond_type || !d.bond_k || !d.bond_r0))
    return fail(RBMD_ERR_ARG, "bond arrays missing");
  if (d.n_angles > 0 && !d.angle_atoms) return fail(RBMD_ERR_ARG, "angle atoms missing");
  if (d.n_dihedrals < 0 || (d.n_dihedrals > 0 && (!d.dihedral_atoms || !d.dihedral_type || !d.dihedral_k ||
                                                   !d.dihedral_sign || !d.dihedral_multiplicity)))
    return fail(RBMD_ERR_ARG, "dihedral arrays missing");
  for (int q = 0; q < d.n_dihedrals; ++q) {
    if (d.dihedral_type[q] < 0 || d.dihedral_type[q] >= d.n_dihedral_types)
      return fail(RBMD_ERR_ARG, "dihedral type out of range");
    for (int t = 0; t < 4; ++t)
      if (d.dihedral_atoms[4 * q + t] < 0 || d.dihedral_atoms[4 * q + t] >= d.n_atoms)
        return fail(RBMD_ERR_ARG, "dihedral atom out of range");
  }
  for (int t = 0; t < d.n_dihedrals && t < 1; ++t)
    for (int y = 0; y < d.n_dihedral_types; ++y)
      if (d.dihedral_multiplicity[y] < 0) return fail(RBMD_ERR_ARG, "dihedral multiplicity must be >= 0");
  if (p.force_field == RBMD_FF_CVFF && d.n_angles > 0 && (!d.angle_type || !d.angle_k || !d.angle_theta0))
    return fail(RBMD_ERR_ARG, "angle coefficients missing");

  auto s = std::make_unique<System>();
  s->p = p;
  derive(d, p, s->dv);
  for (int k = 0; k < 3; ++k)
    if (s->dv.dims[k] < s->dv.num_cycles)
      return fail(RBMD_ERR_UNSUPPORTED, "box shorter than the cut-off: fewer cells than num_cycles");
  const int n = d.n_atoms;
  const Units u = make_units(p.units);
  SysDev& D = s->dev;
  std::memset(&D, 0, sizeof(D));
  D.n = n;
  D.ntypes = d.n_types;
  D.ff = p.force_field;
  D.neigh = p.neighbor;
  D.coul = coul_ff ? p.coulomb : RBMD_COUL_NONE;
  D.prec = p.precision;
  D.rbl_mode = p.rbl_mode;
  D.random_mode = p.random_mode;
  D.temp_ctrl = p.temp_ctrl;
  D.fix_shake = p.fix_shake;
  D.inbuild = p.init_inbuild;
  D.special = (d.special_offsets != nullptr && coul_ff) ? 1 : 0;
  D.pice = s->dv.pice_num;
  D.nc = s->dv.num_cycles;
  D.ncell = s->dv.n_cells;
  for (int k = 0; k < 3; ++k) {
    D.dims[k] = s->dv.dims[k];
    D.lo[k] = d.box_lo[k];
    D.hi[k] = d.box_hi[k];
    D.L[k] = d.box_hi[k] - d.box_lo[k];
    D.d[k] = s->dv.cell_width[k];
  }
  D.rc = p.cut_off;
  D.rs = (p.neighbor == RBMD_NEIGH_RBL) ? p.r_core : p.cut_off;
  D.rc2 = D.rc * D.rc;
  D.rs2 = D.rs * D.rs;
  D.cls_d[0] = thr_below<double>(D.rc2, 0.0001);
  D.cls_d[1] = thr_above<double>(D.rs2, 0.0001);
  D.cls_d[2] = thr_below<double>(D.rs2, 0.0001);
  D.cls_f[0] = thr_below<float>((float)D.rc2, 0.0001f);
  D.cls_f[1] = thr_above<float>((float)D.rs2, 0.0001f);
  D.cls_f[2] = thr_below<float>((float)D.rs2, 0.0001f);
  {
    // Error band of FP32 squared distances (mixed precision).  Each FP32 displacement component
    // inherits the rounding of the candidate position, the image shift, their difference, the home
    // position and the result: |e| <= u (3 Xmax + 6 Lmax + rc) with u = 2^-24, positions within
    // Xmax of the origin and shifts up to 3 Lmax; then |d2_32 - d2_64| <= 2 sqrt(3) r e + 3 e^2 +
    // 4 u r^2 near r^2 = t, doubled for safety.  NPT boxes are bounded by their largest box.
    const double u = std::ldexp(1.0, -24), grow = p.ensemble == RBMD_ENS_NPT ? kBoxGrow : 1.0;
    double xmax = 0.0, lmax = 0.0;
    for (int k = 0; k < 3; ++k) {
      xmax = std::max(xmax, std::fabs(0.5 * (D.lo[k] + D.hi[k])) + 1.25 * grow * D.L[k]);
      lmax = std::max(lmax, grow * D.L[k]);
    }
    const double e = u * (3 * xmax + 6 * lmax + D.rc);
    auto band = [&](double t) { return 2.0 * (2.0 * std::sqrt(3.0) * std::sqrt(t) * e + 3 * e * e + 4 * u * t); };
    auto ulpf = [](double t) { const float f = (float)t; return (double)(std::nextafter(f, 2 * f + 1) - f); };
    // band edges rounded outwards to float
    auto down = [](double v) { float f = (float)v; return (double)f > v ? std::nextafter(f, -INFINITY) : f; };
    auto up = [](double v) { float f = (float)v; return (double)f < v ? std::nextafter(f, INFINITY) : f; };
    const double w_rc = band(D.rc2) + 2 * ulpf(D.rc2) + std::fabs((double)D.cls_f[0] - D.cls_d[0]);
    D.band[2] = down(D.cls_d[0] - w_rc);
    D.band[3] = up(D.cls_d[0] + w_rc);
    if (p.neighbor == RBMD_NEIGH_RBL) {
      const double w_rs = band(D.rs2) + 2 * ulpf(D.rs2) +
                          std::max(std::fabs((double)D.cls_f[1] - D.cls_d[1]), std::fabs((double)D.cls_f[2] - D.cls_d[2]));
      D.band[0] = down(D.cls_d[2] - w_rs);
      D.band[1] = up(D.cls_d[1] + w_rs);
    } else {
      D.band[0] = D.band[1] = -1.0f;  // one threshold only: nothing is banded below rc
    }
  }
  D.alpha = p.alpha;
  D.volume = s->dv.volume;
  D.S = s->dv.S_rbe;
  D.qqr2e = u.qqr2e;
  D.fsa = (float)std::sqrt(p.alpha);
  D.falpha_l2 = (float)(p.alpha * 1.4426950408889634);
  D.fqq = (float)u.qqr2e;
  D.fmt2v = u.fmt2v;
  D.mvv2e = u.mvv2e;
  D.kB = u.kB;
  D.boltz = u.boltz;
  D.nktv2p = u.nktv2p;
  D.dt = p.timestep;
  D.t_start = p.temperature[0];
  D.t_stop = p.temperature[1];
  D.t_damp = p.temperature[2];
  D.num_steps = p.num_steps;
  D.seed_lo = (uint32_t)p.seed;
  D.seed_hi = (uint32_t)(p.seed >> 32);
  D.P = (D.coul == RBMD_COUL_RBE) ? p.coulomb_sample_num : 0;
  s->P = D.P;
  D.n_bonds = (p.force_field == RBMD_FF_CVFF) ? d.n_bonds : 0;
  D.n_angles = (p.force_field == RBMD_FF_CVFF) ? d.n_angles : 0;
  const bool shake = (p.fix_shake == RBMD_SHAKE_TRUE) && d.n_angles > 0 && d.angle_atoms;
  D.has_triples = shake ? 1 : 0;
  D.n_triples = shake ? d.n_angles : 0;
  // Pair traversal.  Both segment-table kernels need every dimension to hold the 2 nc + 1 cells of
  // a stencil without repeats; otherwise the general warp-per-atom kernel runs.  Of the two, the
  // tile kernel (warp per home cell, candidates shared by the cell's atoms) pays off in mixed
  // precision once cells hold a few atoms on average; the lean kernel (warp per atom) is faster
  // below that and in FP64, where the tile kernel's per-lane FP64 state no longer fits in
  // registers.  In mixed precision the column kernel (warp per column of home cells, lane per
  // atom) takes the tile kernel's systems for the RBL forces.  RBMD_PAIR_LAYOUT overrides the
  // choice for tuning and tests: "atom" (general), "lean", "cell" (tile), "column".
  const bool stencil_ok = D.dims[0] >= 2 * D.nc + 1 && D.dims[1] >= 2 * D.nc + 1 && D.dims[2] >= 2 * D.nc + 1;
  // The lean, tile and column kernels also walk stencils that repeat cells, as long as every
  // dimension holds more than nc cells (one periodic image per offset; the tile and column kernels
  // also need edges of 2 rc).  On the saline stream's 1000-1500-atom systems (4 cells per
  // dimension) the lean kernel took 0.85 ms per step, the general kernel 1.40 ms and the tile
  // kernel 1.76 ms; the column kernel takes them within the launch of the large systems for
  // about 0.24 ms more, so it is their default for mixed-precision RBL forces, the lean kernel
  // otherwise, and only the autotuner or RBMD_PAIR_LAYOUT=cell selects the tile kernel there.
  const bool tile_ok = tile_layout_ok(D);
  D.lean = lean_layout_ok(D) ? 1 : 0;
  const bool dense_ok = p.precision == RBMD_PREC_MIXED && n < (1 << 25) &&
                        (double)n >= kTileMinPerCell * (double)D.ncell;
  D.dense = (stencil_ok && dense_ok) ? 1 : 0;
  // dense mixed-precision RBL forces: the column kernel in place of the tile or lean kernel
  if (dense_ok && column_layout_ok(D)) D.dense = 2;
  const char* lay = std::getenv("RBMD_PAIR_LAYOUT");
  s->tuned = lay != nullptr && lay[0] != '\0' && std::strcmp(lay, "auto") != 0;  // a forced layout is not retuned
  if (lay) {
    if (std::strcmp(lay, "atom") == 0) {
      D.lean = 0;
      D.dense = 0;
    } else if (std::strcmp(lay, "lean") == 0) {
      D.dense = 0;
    } else if (std::strcmp(lay, "cell") == 0) {
      D.dense = (tile_ok && n < (1 << 25)) ? 1 : 0;
    } else if (std::strcmp(lay, "column") == 0) {
      D.dense = column_layout_ok(D) ? 2 : ((tile_ok && n < (1 << 25)) ? 1 : 0);
    }
  }
  if (p.ensemble == RBMD_ENS_NPT) {
    // The box changes every step: the general traversal (any dims), cell tables for the largest
    // box the barostat accepts.
    D.npt = p.press_ctrl == RBMD_PC_NOSE_HOOVER ? 2 : 1;
    s->tuned = true;  // one layout only
    D.lean = 0;
    D.dense = 0;
    D.ncell_cap = 1;
    for (int k = 0; k < 3; ++k) {
      D.L0[k] = D.L[k];
      D.kmax[k] = p.kmax[k];
      D.ncell_cap *= std::max(1, (int)((kBoxGrow * D.L0[k]) / (D.rc / D.nc)));
    }
    D.p_start = p.pressure[0];
    D.p_stop = p.pressure[1];
    D.p_damp = p.pressure[2];
    D.bulk = p.bulk_modulus;
  } else {
    D.ncell_cap = D.ncell;
  }
  D.blocks_pair = D.dense ? tile_blocks(D) : (n + kPairWarps - 1) / kPairWarps;
  D.blocks_atom = (n + kAtomBlock - 1) / kAtomBlock;
  D.blocks_rho = (n + kRhoChunk - 1) / kRhoChunk;
  D.blocks_tri = (D.n_triples + 127) / 128;

  // Ewald k lists
  std::vector<double4> ewk, enk;
  if (D.coul != RBMD_COUL_NONE) {
    const int* km = p.kmax;
    for (int a = -km[0]; a <= km[0]; ++a)
      for (int b = -km[1]; b <= km[1]; ++b)
        for (int c = -km[2]; c <= km[2]; ++c) {
          if (a == 0 && b == 0 && c == 0) continue;
          const double kx = 2 * kPi * a / D.L[0], ky = 2 * kPi * b / D.L[1], kz = 2 * kPi * c / D.L[2];
          const double k2 = kx * kx + ky * ky + kz * kz;
          const double rk = std::sqrt(k2);
          enk.push_back(make_double4(kx, ky, kz, std::exp(-rk * rk / (4 * p.alpha)) / (rk * rk)));
          if (D.coul == RBMD_COUL_EWALD)
            ewk.push_back(make_double4(kx, ky, kz, -4 * kPi / (D.volume * k2) * std::exp(-k2 / (4 * p.alpha))));
        }
    D.nk_e = (int)enk.size();
    D.nk_ewald = (int)ewk.size();
  }
  const int nk_force = std::max(D.P, D.nk_ewald);
  const int nk_rho = std::max(nk_force, D.nk_e);

  // RBE proposal tables P(m), q(m) (RBEPSample.h:85-113)
  std::vector<double> rbe_tab;
  if (D.coul == RBMD_COUL_RBE) {
    double smax = 0;
    for (int k = 0; k < 3; ++k) {
      D.rbe_sigma[k] = std::sqrt(p.alpha / 2.0) * D.L[k] / kPi;
      smax = std::max(smax, D.rbe_sigma[k] * (D.npt ? kBoxGrow : 1.0));  // NPT: table for the largest box
    }
    D.rbe_mmax = std::min(4096, (int)std::ceil(12.0 * smax) + 4);
    D.rbe_slots = std::min(1024, D.P + kRbeSlack);
    const int tw = 2 * D.rbe_mmax + 1;
    rbe_tab.assign((size_t)3 * tw * 2, 0.0);
    for (int k = 0; k < 3; ++k) {
      const double factor = -(p.alpha * D.L[k] * D.L[k]);
      double H = 0.0;
      for (int m = -10; m <= 10; ++m) H += std::exp(m * m * factor);
      H *= std::sqrt(-(factor) / kPi);
      const double sc = std::sqrt(p.alpha * std::pow(D.L[k], 2) / std::pow(kPi, 2));
      for (int m = -D.rbe_mmax; m <= D.rbe_mmax; ++m) {
        const double xm = (double)m;
        const double P_m = std::exp(-std::pow(2 * kPi * xm / D.L[k], 2) / (4 * p.alpha)) / H;
        double q_m;
        if (xm == 0) q_m = std::erf((1.0 / 2) / sc);
        else q_m = (std::erf(((1.0 / 2) + std::fabs(xm)) / sc) - std::erf((std::fabs(xm) - (1.0 / 2)) / sc)) / 2;
        rbe_tab[(size_t)k * tw * 2 + (m + D.rbe_mmax)] = P_m;
        rbe_tab[(size_t)k * tw * 2 + tw + (m + D.rbe_mmax)] = q_m;
      }
    }
  }

  // host-side packed atom data
  std::vector<double4> hx(n), hv(n);
  std::vector<int4> hmeta(n);
  std::vector<int> himg(3 * n, 0);
  s->charge.assign(n, 0.0);
  std::vector<uint8_t> in_triple(n, 0);
  if (shake)
    for (int a = 0; a < d.n_angles; ++a)
      for (int t = 0; t < 3; ++t) {
        const int ai = d.angle_atoms[3 * a + t];
        if (ai < 0 || ai >= n) return fail(RBMD_ERR_ARG, "angle atom out of range");
        in_triple[ai] = 1;
      }
  for (int i = 0; i < n; ++i) {
    const double q = (d.charge && p.force_field != RBMD_FF_EAM) ? d.charge[i] : 0.0;
    s->charge[i] = q;
    hx[i] = make_double4(d.position[3 * i], d.position[3 * i + 1], d.position[3 * i + 2], q);
    const double* vv = d.velocity ? d.velocity + 3 * i : nullptr;
    hv[i] = make_double4(vv ? vv[0] : 0.0, vv ? vv[1] : 0.0, vv ? vv[2] : 0.0, d.mass[i]);
    const int mol = d.molecule ? d.molecule[i] : i;
    hmeta[i] = make_int4(d.type[i], mol, in_triple[i] ? 1 : 0, 0);
    if (d.image)
      for (int k = 0; k < 3; ++k) himg[3 * i + k] = d.image[3 * i + k];
  }
  // molecule CSR
  int maxmol = 0;
  for (int i = 0; i < n; ++i) maxmol = std::max(maxmol, hmeta[i].y);
  std::vector<int> mol_off(maxmol + 2, 0), mol_atoms(n);
  for (int i = 0; i < n; ++i) mol_off[hmeta[i].y + 1]++;
  for (size_t k = 1; k < mol_off.size(); ++k) mol_off[k] += mol_off[k - 1];
  {
    std::vector<int> fill(mol_off.begin(), mol_off.end() - 1);
    for (int i = 0; i < n; ++i) mol_atoms[fill[hmeta[i].y]++] = i;
  }
  // bonded term slots per atom
  D.n_dihedrals = (p.force_field == RBMD_FF_CVFF) ? d.n_dihedrals : 0;
  const int nterms = D.n_bonds + D.n_angles + D.n_dihedrals;
  s->n_terms = nterms;
  std::vector<int> aterm_off(n + 1, 0), aterm;
  if (nterms > 0) {
    // slot s of the per-term forces belongs to atom owner(s); a counting sort over the slots in
    // increasing order gives every atom its slots in that order
    const int nslots = 2 * D.n_bonds + 3 * D.n_angles + 4 * D.n_dihedrals;
    auto owner = [&](int sl) {
      if (sl < 2 * D.n_bonds) return d.bond_atoms[sl];
      sl -= 2 * D.n_bonds;
      if (sl < 3 * D.n_angles) return d.angle_atoms[sl];
      return d.dihedral_atoms[sl - 3 * D.n_angles];
    };
    for (int sl = 0; sl < nslots; ++sl) aterm_off[owner(sl) + 1]++;
    for (int i = 0; i < n; ++i) aterm_off[i + 1] += aterm_off[i];
    aterm.assign(nslots, 0);
    std::vector<int> fill(aterm_off.begin(), aterm_off.end() - 1);
    for (int sl = 0; sl < nslots; ++sl) aterm[fill[owner(sl)]++] = sl;
  }
  // self energy per atom (ExecutionMD::ComputeSelfEnergy, ExecutionMD.cpp:544-558)
  if (D.coul != RBMD_COUL_NONE) {
    double sq = 0;
    for (int i = 0; i < n; ++i) sq += s->charge[i] * s->charge[i];
    s->self_energy = -std::sqrt(p.alpha / kPi) * sq / n * u.qqr2e;
  }

  // ---- device allocations
  int64_t total = 0;
  bool oom = false;
  auto dal = [&](size_t bytes) -> void* {
    if (bytes == 0) bytes = 16;
    void* ptr = dmalloc(bytes);
    if (!ptr) {
      oom = true;
      return nullptr;
    }
    s->allocs.push_back(ptr);
    total += (int64_t)bytes;
    return ptr;
  };
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (dst && src && bytes) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
  };
  D.x = (double4*)dal(sizeof(double4) * n);
  D.v = (double4*)dal(sizeof(double4) * n);
  D.f = (double4*)dal(sizeof(double4) * n);
  if (shake) {
    D.xold = (double4*)dal(sizeof(double4) * n);
    D.vold = (double4*)dal(sizeof(double4) * n);
    D.vold2 = (double4*)dal(sizeof(double4) * n);
  }
  D.meta = (int4*)dal(sizeof(int4) * n);
  D.image = (int*)dal(sizeof(int) * 3 * n);
  D.cell_of_atom = (int*)dal(sizeof(int) * n);
  D.cell_count = (int*)dal(sizeof(int) * D.ncell_cap);
  D.cell_start = (int*)dal(sizeof(int) * (D.ncell_cap + 1));
  D.cell_fill = (int*)dal(sizeof(int) * D.ncell_cap);
  D.sorted = (int*)dal(sizeof(int) * n);
  D.rank = (int*)dal(sizeof(int) * n);
  D.sx = (double4*)dal(sizeof(double4) * n);
  D.sxf = (float4*)dal(sizeof(float4) * n);
  D.smeta = (int4*)dal(sizeof(int4) * n);
  D.eps = (double*)dal(sizeof(double) * d.n_types);
  D.sig = (double*)dal(sizeof(double) * d.n_types);
  std::vector<float2> hlj;
  if (D.prec == RBMD_PREC_MIXED) {  // at most kMaxF32Types types (checked above)
    hlj.resize((size_t)d.n_types * d.n_types);
    for (int a = 0; a < d.n_types; ++a)
      for (int b = 0; b < d.n_types; ++b) {
        const double sg = (d.sigma[a] + d.sigma[b]) / 2;
        hlj[(size_t)a * d.n_types + b] =
            make_float2((float)(-24.0 * std::sqrt(d.epsilon[a] * d.epsilon[b])), (float)(sg * sg * sg * sg * sg * sg));
      }
    D.ljf = (float2*)dal(sizeof(float2) * hlj.size());
  }
  std::vector<float> hnear;
  if (p.near_table == RBMD_NEAR_TABLE && D.coul != RBMD_COUL_NONE && D.neigh == RBMD_NEIGH_RBL) {
    hnear.resize(kNearKeys);
    if (d.near_table_values) std::memcpy(hnear.data(), d.near_table_values, sizeof(float) * kNearKeys);
    else near_table_default(hnear.data());
    D.near_tab = (float*)dal(sizeof(float) * kNearKeys);
  }
  D.mol_off = (int*)dal(sizeof(int) * mol_off.size());
  D.mol_atoms = (int*)dal(sizeof(int) * n);
  std::vector<int> sp_off;
  if (D.special) {
    const int ns = d.special_offsets[n];
    D.sp_off = (int*)dal(sizeof(int) * (n + 1));
    D.sp_ids = (int*)dal(sizeof(int) * ns);
    D.sp_w = (double*)dal(sizeof(double) * ns);
    up(D.sp_off, d.special_offsets, sizeof(int) * (n + 1));
    up(D.sp_ids, d.special_ids, sizeof(int) * ns);
    up(D.sp_w, d.special_weights, sizeof(double) * ns);
  }
  if (nterms > 0) {
    if (D.n_bonds > 0) {
      D.bond_atoms = (int*)dal(sizeof(int) * 2 * D.n_bonds);
      D.bond_type = (int*)dal(sizeof(int) * D.n_bonds);
      D.bond_k = (double*)dal(sizeof(double) * d.n_bond_types);
      D.bond_r0 = (double*)dal(sizeof(double) * d.n_bond_types);
      up(D.bond_atoms, d.bond_atoms, sizeof(int) * 2 * D.n_bonds);
      up(D.bond_type, d.bond_type, sizeof(int) * D.n_bonds);
      up(D.bond_k, d.bond_k, sizeof(double) * d.n_bond_types);
      up(D.bond_r0, d.bond_r0, sizeof(double) * d.n_bond_types);
    }
    if (D.n_dihedrals > 0) {
      D.dih_atoms = (int*)dal(sizeof(int) * 4 * D.n_dihedrals);
      D.dih_type = (int*)dal(sizeof(int) * D.n_dihedrals);
      D.dih_k = (double*)dal(sizeof(double) * d.n_dihedral_types);
      D.dih_sign = (int*)dal(sizeof(int) * d.n_dihedral_types);
      D.dih_mult = (int*)dal(sizeof(int) * d.n_dihedral_types);
      up(D.dih_atoms, d.dihedral_atoms, sizeof(int) * 4 * D.n_dihedrals);
      up(D.dih_type, d.dihedral_type, sizeof(int) * D.n_dihedrals);
      up(D.dih_k, d.dihedral_k, sizeof(double) * d.n_dihedral_types);
      up(D.dih_sign, d.dihedral_sign, sizeof(int) * d.n_dihedral_types);
      up(D.dih_mult, d.dihedral_multiplicity, sizeof(int) * d.n_dihedral_types);
    }
    D.term_force = (double4*)dal(sizeof(double4) * (2 * D.n_bonds + 3 * D.n_angles + 4 * D.n_dihedrals));
    D.term_energy = (double*)dal(sizeof(double) * nterms);
    D.term_vir = (double*)dal(sizeof(double) * 6 * nterms);
    D.aterm_off = (int*)dal(sizeof(int) * (n + 1));
    D.aterm = (int*)dal(sizeof(int) * std::max<size_t>(1, aterm.size()));
    up(D.aterm_off, aterm_off.data(), sizeof(int) * (n + 1));
    up(D.aterm, aterm.data(), sizeof(int) * aterm.size());
  }
  if (d.n_angles > 0 && (D.n_angles > 0 || shake)) {
    D.angle_atoms = (int*)dal(sizeof(int) * 3 * d.n_angles);
    up(D.angle_atoms, d.angle_atoms, sizeof(int) * 3 * d.n_angles);
    if (D.n_angles > 0) {
      D.angle_type = (int*)dal(sizeof(int) * d.n_angles);
      D.angle_k = (double*)dal(sizeof(double) * d.n_angle_types);
      D.angle_t0 = (double*)dal(sizeof(double) * d.n_angle_types);
      up(D.angle_type, d.angle_type, sizeof(int) * d.n_angles);
      up(D.angle_k, d.angle_k, sizeof(double) * d.n_angle_types);
      up(D.angle_t0, d.angle_theta0, sizeof(double) * d.n_angle_types);
    }
  }
  if (D.coul != RBMD_COUL_NONE) {
    D.km = (int*)dal(sizeof(int) * 3 * std::max(1, D.P));
    D.kv = (double4*)dal(sizeof(double4) * std::max(1, nk_force));
    D.rhok = (double*)dal(sizeof(double) * 2 * std::max(1, nk_force));
    D.rho_part = (double*)dal(sizeof(double) * 2 * (size_t)D.blocks_rho * std::max(1, nk_rho));
    D.kv_e = (double4*)dal(sizeof(double4) * std::max(1, D.nk_e));
    D.rhok_e = (double*)dal(sizeof(double) * 2 * std::max(1, D.nk_e));
    up(D.kv_e, enk.data(), sizeof(double4) * enk.size());
    if (D.coul == RBMD_COUL_EWALD) up(D.kv, ewk.data(), sizeof(double4) * ewk.size());
    if (D.coul == RBMD_COUL_RBE) {
      D.rbe_tab = (double*)dal(sizeof(double) * rbe_tab.size());
      up(D.rbe_tab, rbe_tab.data(), sizeof(double) * rbe_tab.size());
    }
  }
  if (p.force_field == RBMD_FF_EAM) {
    D.eam_nrho = d.eam_nrho;
    D.eam_nr = d.eam_nr;
    D.eam_drho = d.eam_drho;
    D.eam_dr = d.eam_dr;
    D.eam_rhomax = d.eam_rhomax;
    D.eam_cut = d.eam_cut;
    D.eam_per_type = d.eam_per_type;
    size_t nf, nr, nz;
    eam_table_sizes(d, &nf, &nr, &nz);
    D.frho_s = (double*)dal(sizeof(double) * nf);
    D.rhor_s = (double*)dal(sizeof(double) * nr);
    D.z2r_s = (double*)dal(sizeof(double) * nz);
    D.eam_fp = (double*)dal(sizeof(double) * n);
    up(D.frho_s, d.eam_frho_spline, sizeof(double) * nf);
    up(D.rhor_s, d.eam_rhor_spline, sizeof(double) * nr);
    up(D.z2r_s, d.eam_z2r_spline, sizeof(double) * nz);
  }
  D.atom_part = (double*)dal(sizeof(double) * 8 * D.blocks_atom);
  // pair-kernel partials: enough blocks for any layout the autotuner may switch to
  D.vir_part = (double*)dal(sizeof(double) * 9 *
                            std::max((D.ncell_cap + kCellWarpsHost - 1) / kCellWarpsHost, (n + kPairWarps - 1) / kPairWarps));
  D.tri_part = (double*)dal(sizeof(double) * 6 * std::max(1, D.blocks_tri));
  D.st = (SysState*)dal(sizeof(SysState));
  if (oom) {
    for (void* ptr : s->allocs) dfree(ptr);
    return fail(RBMD_ERR_OOM, "device allocation failed for a system of " + std::to_string(n) + " atoms");
  }
  up(D.x, hx.data(), sizeof(double4) * n);
  up(D.v, hv.data(), sizeof(double4) * n);
  cudaMemsetAsync(D.f, 0, sizeof(double4) * n, stream);
  up(D.meta, hmeta.data(), sizeof(int4) * n);
  up(D.image, himg.data(), sizeof(int) * 3 * n);
  up(D.eps, d.epsilon, sizeof(double) * d.n_types);
  up(D.sig, d.sigma, sizeof(double) * d.n_types);
  up(D.ljf, hlj.data(), sizeof(float2) * hlj.size());
  up(D.near_tab, hnear.data(), sizeof(float) * hnear.size());
  up(D.mol_off, mol_off.data(), sizeof(int) * mol_off.size());
  up(D.mol_atoms, mol_atoms.data(), sizeof(int) * n);
  SysState st0;
  std::memset(&st0, 0, sizeof(st0));
  st0.t_freq = 1 / p.temperature[2];
  st0.tdrag = 1.0 - (p.timestep * st0.t_freq * 0.0 / 1);
  st0.tdof = 3.0 * n - 3;  // ExecutionMD::Computedof, ExecutionMD.cpp:1251-1261
  if (p.fix_shake == RBMD_SHAKE_TRUE) st0.tdof = st0.tdof - n;
  st0.vscale_pending = st0.vscale_pending_c = st0.vscale_a = 1.0;
  up(D.st, &st0, sizeof(SysState));
  s->bytes = total;

  // slot
  int slot;
  if (!free_slots_.empty()) {
    slot = free_slots_.back();
    free_slots_.pop_back();
  } else {
    slot = (int)systems_.size();
    systems_.push_back(nullptr);
  }
  int rc = ensure_slots(slot + 1);
  if (rc) return rc;
  s->slot = slot;
  s->id = next_id_++;
  upload_record(s.get());
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(RBMD_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(e));
  *out_id = s->id;
  systems_[slot] = s.release();
  return RBMD_OK;
}

void Context::drop_batches_with(int id) {
  for (auto it = batch_cache_.begin(); it != batch_cache_.end();) {
    BatchRec* br = it->second;
    if (std::find(br->ids.begin(), br->ids.end(), id) != br->ids.end()) {
      cudaStreamSynchronize(stream);
      if (br->graph) cudaGraphExecDestroy(br->graph);
      for (void* p : br->allocs) dfree(p);
      delete br;
      it = batch_cache_.erase(it);
    } else {
      ++it;
    }
  }
}

int Context::remove_system(int id) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id " + std::to_string(id));
  drop_batches_with(id);
  for (void* p : s->allocs) dfree(p);  // stream-ordered: after every launch that used them
  systems_[s->slot] = nullptr;
  free_slots_.push_back(s->slot);
  delete s;
  return RBMD_OK;
}

// ------------------------------------------------------------------------------ near-Coulomb table
int near_table_key(float r) {
  uint32_t b;
  std::memcpy(&b, &r, sizeof(b));
  return (int)((b & 0x03FF8000u) >> 15);
}

void near_table_default(float* out) {
  const double a = 0.1, sa = std::sqrt(a);
  auto g = [&](double r) {
    return std::erfc(sa * r) / (r * r) + 2.0 * sa * std::exp(-a * r * r) / (std::sqrt(kPi) * r);
  };
  // every key: G at its lower edge, 2^e (1 + m / 256) for mantissa top bits m and an exponent e whose
  // low three bits are the key's (e in [-4, 3] for the distances 1/16 .. 16 this covers)
  for (int k = 0; k < kNearKeys; ++k) {
    const int e3 = k >> 8, e = e3 <= 2 ? 1 + e3 : e3 - 7;
    out[k] = (float)g(std::ldexp(1.0 + (k & 255) / 256.0, e));
  }
  // the reference's tabulated points: the first r of each walk with a given key
  std::vector<char> seen(kNearKeys, 0);
  auto walk = [&](double r0, double dr, double r1) {
    for (long m = 0;; ++m) {
      const double r = r0 + (double)m * dr;
      if (r >= r1) break;
      const int k = near_table_key((float)r);
      if (!seen[k]) {
        seen[k] = 1;
        out[k] = (float)g(r);
      }
    }
  };
  walk(0.1, 1e-4, 2.0);
  walk(2.0, 1e-3, 12.0);
}

// ------------------------------------------------------------------------------ batches
bool same_group(const System* a, const System* b, bool layout) {
  const SysDev &x = a->dev, &y = b->dev;
  return x.ff == y.ff && x.neigh == y.neigh && x.coul == y.coul && x.prec == y.prec &&
         x.temp_ctrl == y.temp_ctrl && x.special == y.special && x.has_triples == y.has_triples &&
         ((x.n_bonds + x.n_angles + x.n_dihedrals) > 0) == ((y.n_bonds + y.n_angles + y.n_dihedrals) > 0) &&
         x.npt == y.npt && x.rc2 == y.rc2 && (x.near_tab != nullptr) == (y.near_tab != nullptr) &&
         x.rs2 == y.rs2 &&
         (!layout || (x.dense == y.dense && x.lean == y.lean));
}

Context::BatchRec* Context::build_batch(const std::vector<System*>& group, int& rc) {
  auto* br = new BatchRec();
  Batch& b = br->b;
  b.sys = d_sys_;
  b.nsys = (int)group.size();
  const SysDev& g = group[0]->dev;
  b.ff = g.ff;
  b.neigh = g.neigh;
  b.coul = g.coul;
  b.prec = g.prec;
  b.temp_ctrl = g.temp_ctrl;
  b.special = g.special;
  b.has_shake = g.has_triples;
  b.has_bonded = (g.n_bonds + g.n_angles + g.n_dihedrals) > 0;
  b.dense = g.dense;
  b.lean = g.lean;
  b.npt = g.npt;
  b.near = g.near_tab != nullptr;
  std::vector<int> slots;
  std::vector<int2> wa, wp, wc, wr, wt, wm, wpc;
  std::vector<std::pair<double, int2>> cols;  // column layout: (atoms per column, (slot, column))
  for (int k = 0; k < 4; ++k) b.band[k] = g.band[k];
  for (System* s : group) {
    const SysDev& D = s->dev;
    b.band[0] = std::min(b.band[0], D.band[0]);
    b.band[1] = std::max(b.band[1], D.band[1]);
    b.band[2] = std::min(b.band[2], D.band[2]);
    b.band[3] = std::max(b.band[3], D.band[3]);
    slots.push_back(s->slot);
    br->ids.push_back(s->id);
    b.max_P = std::max(b.max_P, std::max(D.P, D.nk_ewald));
    b.natoms += D.n;
    for (int k = 0; k < D.n; k += kAtomBlock) wa.push_back(make_int2(s->slot, k));
    if (D.dense == 2) {
      const int nxy = D.dims[0] * D.dims[1];
      for (int k = 0; k < nxy; ++k) cols.push_back({(double)D.n / nxy, make_int2(s->slot, k)});
      for (int k = 0; k < D.ncell; k += kCellWarpsHost) wpc.push_back(make_int2(s->slot, k));
    } else if (D.dense)
      for (int k = 0; k < D.ncell; k += kCellWarpsHost) wp.push_back(make_int2(s->slot, k));
    else
      for (int k = 0; k < D.n; k += kPairWarps) wp.push_back(make_int2(s->slot, k));
    for (int k = 0; k < D.ncell_cap; k += kCellBlock) wc.push_back(make_int2(s->slot, k));
    for (int k = 0; k < D.n; k += kRhoChunk) wr.push_back(make_int2(s->slot, k));
    for (int k = 0; k < D.n_triples; k += 128) wt.push_back(make_int2(s->slot, k));
    for (int k = 0; k < D.n_bonds + D.n_angles + D.n_dihedrals; k += 128) wm.push_back(make_int2(s->slot, k));
  }
  // the longest columns first, so that the persistent kernel's last columns are short ones
  std::stable_sort(cols.begin(), cols.end(), [](const std::pair<double, int2>& a, const std::pair<double, int2>& c) {
    return a.first > c.first;
  });
  for (const auto& c : cols) wp.push_back(c.second);
  auto mk = [&](const std::vector<int2>& h, Work& w) {
    w.n = (int)h.size();
    if (h.empty()) return;
    void* ptr = dmalloc(sizeof(int2) * h.size());
    if (!ptr) {
      rc = RBMD_ERR_OOM;
      return;
    }
    br->allocs.push_back(ptr);
    cudaMemcpyAsync(ptr, h.data(), sizeof(int2) * h.size(), cudaMemcpyHostToDevice, stream);
    w.d = (int2*)ptr;
  };
  mk(wa, b.atom);
  mk(wp, b.pair);
  mk(wpc, b.pair_cells);
  if (b.dense == 2 && b.pair.n > 0) {
    b.col_ctr = (unsigned*)dmalloc(4 * sizeof(unsigned));  // the column kernel's, then the stray pass's
    if (!b.col_ctr) rc = RBMD_ERR_OOM;
    else {
      br->allocs.push_back(b.col_ctr);
      cudaMemsetAsync(b.col_ctr, 0, 4 * sizeof(unsigned), stream);
    }
    b.col_grid = pair_col_grid(b.pair.n, b.ff, b.special, b.near, false);
    b.stray_grid = pair_col_grid(b.pair.n, b.ff, b.special, b.near, true);
  }
  mk(wc, b.cell);
  mk(wr, b.rho);
  mk(wt, b.tri);
  mk(wm, b.term);
  void* ps = dmalloc(sizeof(int) * slots.size());
  if (!ps) rc = RBMD_ERR_OOM;
  else {
    br->allocs.push_back(ps);
    cudaMemcpyAsync(ps, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice, stream);
    b.d_slots = (int*)ps;
  }
  cudaStreamSynchronize(stream);
  return br;
}

std::vector<Context::BatchRec*> Context::batches_for(const int32_t* ids, int n, int& rc) {
  rc = RBMD_OK;
  std::vector<System*> sys;
  for (int k = 0; k < n; ++k) {
    System* s = find(ids[k]);
    if (!s) {
      rc = fail(RBMD_ERR_STATE, "unknown system id " + std::to_string(ids[k]));
      return {};
    }
    sys.push_back(s);
  }
  // groups of identical kernel configuration; plain mode: one system per group
  std::vector<std::vector<System*>> groups;
  for (System* s : sys) {
    bool placed = false;
    if (cfg.batched)
      for (auto& g : groups)
        if (same_group(g[0], s, true)) {
          g.push_back(s);
          placed = true;
          break;
        }
    if (!placed) groups.push_back({s});
  }
  std::vector<BatchRec*> out;
  for (auto& g : groups) {
    std::vector<int> key;
    for (System* s : g) key.push_back(s->id);
    auto it = batch_cache_.find(key);
    if (it != batch_cache_.end()) {
      out.push_back(it->second);
      continue;
    }
    BatchRec* br = build_batch(g, rc);
    if (rc) {
      delete br;
      fail(rc, "work-table allocation failed");
      return {};
    }
    batch_cache_[key] = br;
    out.push_back(br);
  }
  return out;
}

template <class F>
void Context::timed(const char* name, double units, F&& fn) {
  if (!prof.on) {
    fn();
    return;
  }
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, stream);
  fn();
  cudaEventRecord(b, stream);
  auto& r = prof.recs[name];
  r.ev.push_back({a, b});
  r.units.push_back(units);
}

void Context::enqueue_forces(const Batch& b, FinalMode mode, int virial) {
  timed("cells", 0, [&] { launch_cells(b, stream); });
  if (b.coul == RBMD_COUL_RBE) timed("rbe_sample", 0, [&] { launch_rbe_sample(b, stream); });
  if (b.coul != RBMD_COUL_NONE) timed("rho", 0, [&] { launch_rho(b, stream, b.coul == RBMD_COUL_EWALD); });
  if (b.has_bonded) timed("bonded", 0, [&] { launch_bonded(b, stream, virial); });
  timed(pair_name(b), (double)b.natoms, [&] { launch_pair(b, stream, virial); });
  timed("final", (double)b.natoms, [&] { launch_final(b, stream, mode, virial); });
}

void Context::enqueue_step(const Batch& b) {
  if (b.npt == 2) timed("mtk", 0, [&] { launch_mtk_begin(b, stream); });
  else timed("nhc", 0, [&] { launch_nhc_a(b, stream); });
  timed("kick_drift", 0, [&] { launch_kick_drift(b, stream); });
  timed("cells", 0, [&] { launch_cells(b, stream); });
  if (b.has_shake) timed("shake", 0, [&] { launch_shake(b, stream); });
  if (b.coul == RBMD_COUL_RBE) timed("rbe_sample", 0, [&] { launch_rbe_sample(b, stream); });
  if (b.coul != RBMD_COUL_NONE) timed("rho", 0, [&] { launch_rho(b, stream, b.coul == RBMD_COUL_EWALD); });
  // NPT: the barostat needs the virial of this evaluation
  const int vir = b.npt;
  if (b.has_bonded) timed("bonded", 0, [&] { launch_bonded(b, stream, vir); });
  timed(pair_name(b), (double)b.natoms, [&] { launch_pair(b, stream, vir); });
  timed("final", (double)b.natoms, [&] { launch_final(b, stream, kFinalKick, vir); });
  if (b.has_shake) {
    timed("rattle", 0, [&] { launch_rattle(b, stream); });
    if (b.temp_ctrl != RBMD_TC_NOSE_HOOVER) timed("ke", 0, [&] { launch_ke_thermostat(b, stream); });
  }
  if (b.npt == 1) timed("barostat", 0, [&] { launch_barostat(b, stream); });
}

int Context::init(const int32_t* ids, int n) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  int rc;
  if (cfg.autotune) {  // before the first force evaluation: nothing to keep
    rc = autotune(ids, n, nullptr, 0, nullptr, false);
    if (rc) return rc;
  }
  auto bs = batches_for(ids, n, rc);
  if (rc) return rc;
  for (int k = 0; k < n; ++k) {
    System* s = find(ids[k]);
    SysState st0;
    cudaMemcpyAsync(&st0, s->dev.st, sizeof(SysState), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    st0.step = 0;
    for (int c = 0; c < 3; ++c) st0.eta[c] = st0.eta_dot[c] = st0.eta_dotdot[c] = 0.0;
    st0.eta_dot[3] = 0;
    st0.vscale_pending = st0.vscale_pending_c = st0.vscale_a = 1.0;
    // barostat state (ExecutionNPT::InitialCondition, ExecutionNPT.cpp:196-225); MTK reads the
    // virial of the init force evaluation at its first step
    for (int c = 0; c < 6; ++c) st0.virial[c] = 0.0;
    for (int c = 0; c < 3; ++c) {
      st0.omega_dot[c] = st0.omega_mass[c] = 0.0;
      st0.etap[c] = st0.etap_dot[c] = st0.etap_dotdot[c] = st0.etap_mass[c] = 0.0;
    }
    st0.etap_dot[3] = 0.0;
    cudaMemcpyAsync(s->dev.st, &st0, sizeof(SysState), cudaMemcpyHostToDevice, stream);
  }
  for (BatchRec* br : bs) enqueue_forces(br->b, kFinalInit, br->b.npt == 2 ? 1 : 0);
  return check_cuda("init");
}

int Context::step(const int32_t* ids, int n, int nsteps) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  if (nsteps <= 0) return RBMD_OK;
  int rc;
  if (cfg.autotune) {
    rc = autotune(ids, n, nullptr, 0, nullptr, true);
    if (rc) return rc;
  }
  auto bs = batches_for(ids, n, rc);
  if (rc) return rc;
  const bool graphs = cfg.use_graphs && !prof.on;
  if (graphs) {
    // one graph per batch set: the step of every group, replayed nsteps times
    std::vector<int> key;
    for (auto* br : bs)
      for (int id : br->ids) key.push_back(id);
    key.push_back(-1);  // distinguish from the per-group cache entries
    auto it = batch_cache_.find(key);
    BatchRec* gr = (it != batch_cache_.end()) ? it->second : nullptr;
    if (!gr) {
      gr = new BatchRec();
      gr->ids = key;
      batch_cache_[key] = gr;
    }
    if (!gr->graph) {
      long long before = launches_issued();
      cudaGraph_t g;
      cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
      for (auto* br : bs) enqueue_step(br->b);
      cudaStreamEndCapture(stream, &g);
      if (cudaGraphInstantiate(&gr->graph, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(RBMD_ERR_CUDA, "graph instantiate failed");
      }
      cudaGraphDestroy(g);
      gr->graph_steps = (int)(launches_issued() - before);
      note_launch(-(int)gr->graph_steps);
    }
    for (int k = 0; k < nsteps; ++k) cudaGraphLaunch(gr->graph, stream);
    note_launch(gr->graph_steps * nsteps);
  } else {
    for (int k = 0; k < nsteps; ++k)
      for (BatchRec* br : bs) enqueue_step(br->b);
  }
  for (BatchRec* br : bs) launch_flush_vscale(br->b, stream);
  return check_cuda("step");
}

int Context::compute_forces(const int32_t* ids, int n) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  int rc;
  auto bs = batches_for(ids, n, rc);
  if (rc) return rc;
  for (BatchRec* br : bs) enqueue_forces(br->b, kFinalForceOnly, 0);
  return check_cuda("compute_forces");
}

int Context::sync() {
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(RBMD_ERR_CUDA, std::string("sync: ") + cudaGetErrorString(e));
  return RBMD_OK;
}

// ------------------------------------------------------------------------------ getters
int Context::get_forces(int id, double* f) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (!f) return fail(RBMD_ERR_ARG, "null output");
  std::vector<double4> h(s->dev.n);
  cudaMemcpyAsync(h.data(), s->dev.f, sizeof(double4) * s->dev.n, cudaMemcpyDeviceToHost, stream);
  int rc = sync();
  if (rc) return rc;
  for (int i = 0; i < s->dev.n; ++i) {
    f[3 * i] = h[i].x;
    f[3 * i + 1] = h[i].y;
    f[3 * i + 2] = h[i].z;
  }
  return RBMD_OK;
}

int Context::get_state(int id, double* x, double* v, int32_t* image) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  const int n = s->dev.n;
  std::vector<double4> hx(x ? n : 0), hv(v ? n : 0);
  if (x) cudaMemcpyAsync(hx.data(), s->dev.x, sizeof(double4) * n, cudaMemcpyDeviceToHost, stream);
  if (v) cudaMemcpyAsync(hv.data(), s->dev.v, sizeof(double4) * n, cudaMemcpyDeviceToHost, stream);
  if (image) cudaMemcpyAsync(image, s->dev.image, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost, stream);
  int rc = sync();
  if (rc) return rc;
  for (int i = 0; i < n; ++i) {
    if (x) {
      x[3 * i] = hx[i].x;
      x[3 * i + 1] = hx[i].y;
      x[3 * i + 2] = hx[i].z;
    }
    if (v) {
      v[3 * i] = hv[i].x;
      v[3 * i + 1] = hv[i].y;
      v[3 * i + 2] = hv[i].z;
    }
  }
  return RBMD_OK;
}

int Context::set_state(int id, const double* x, const double* v, const int32_t* image) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  const int n = s->dev.n;
  int rc = sync();
  if (rc) return rc;
  if (x) {
    std::vector<double4> hx(n);
    cudaMemcpyAsync(hx.data(), s->dev.x, sizeof(double4) * n, cudaMemcpyDeviceToHost, stream);
    sync();
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(x[3 * i + k])) return fail(RBMD_ERR_NUMERIC, "non-finite position");
      hx[i].x = x[3 * i];
      hx[i].y = x[3 * i + 1];
      hx[i].z = x[3 * i + 2];
    }
    cudaMemcpyAsync(s->dev.x, hx.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, stream);
    sync();
  }
  if (v) {
    std::vector<double4> hv(n);
    cudaMemcpyAsync(hv.data(), s->dev.v, sizeof(double4) * n, cudaMemcpyDeviceToHost, stream);
    sync();
    for (int i = 0; i < n; ++i) {
      hv[i].x = v[3 * i];
      hv[i].y = v[3 * i + 1];
      hv[i].z = v[3 * i + 2];
    }
    cudaMemcpyAsync(s->dev.v, hv.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, stream);
    sync();
  }
  if (image) {
    cudaMemcpyAsync(s->dev.image, image, sizeof(int) * 3 * n, cudaMemcpyHostToDevice, stream);
    sync();
  }
  return check_cuda("set_state");
}

int Context::set_step(int id, int64_t step) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (step < 0) return fail(RBMD_ERR_ARG, "negative step");
  cudaMemcpyAsync(&s->dev.st->step, &step, sizeof(int64_t), cudaMemcpyHostToDevice, stream);
  const int rc = sync();
  return rc ? rc : check_cuda("set_step");
}

int Context::get_thermo(int id, rbmd_thermo* out) {
  int32_t one = id;
  return get_thermo_many(&one, 1, out);
}

// Thermo of several systems with one force / energy evaluation per batch of compatible systems and
// one synchronisation (the serving loop retires several systems per round).  Each system's
// arithmetic is independent of the others in its batch, so the values equal get_thermo's alone.
int Context::get_thermo_many(const int32_t* ids, int nsys, rbmd_thermo* outs) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  if (!outs || nsys <= 0) return fail(RBMD_ERR_ARG, "null output");
  struct Pending {
    System* s = nullptr;
    void* fsave = nullptr;
    std::vector<double> te_step, te;
    SysState st;
  };
  std::vector<Pending> ps(nsys);
  int rc = RBMD_OK;
  for (int q = 0; q < nsys; ++q) {
    System* s = find(ids[q]);
    if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
    rc = refresh(s);
    if (rc) return rc;
    ps[q].s = s;
  }
  auto bs = [&] {
    rbmd_device_cfg saved = cfg;
    cfg.batched = 1;
    auto r = batches_for(ids, nsys, rc);
    cfg = saved;
    return r;
  }();
  if (rc) return rc;
  for (auto& p : ps) {
    const SysDev& D = p.s->dev;
    // keep the step's forces: the pressure evaluation below recomputes them in FP64
    p.fsave = dmalloc(sizeof(double4) * D.n);
    if (!p.fsave) {
      for (auto& q : ps) dfree(q.fsave);
      return fail(RBMD_ERR_OOM, "thermo scratch");
    }
    cudaMemcpyAsync(p.fsave, D.f, sizeof(double4) * D.n, cudaMemcpyDeviceToDevice, stream);
    // NPT: bond and angle energies are those of the step's force evaluation, before the remap
    // (PARA_BOND_ENERGY / PARA_ANGLE_ENERGY are set there and read by ThermoOutput::Execute)
    p.te_step.resize(D.npt ? p.s->n_terms : 0);
    if (!p.te_step.empty())
      cudaMemcpyAsync(p.te_step.data(), D.term_energy, sizeof(double) * p.te_step.size(), cudaMemcpyDeviceToHost,
                      stream);
    cudaMemsetAsync(&D.st->virial[0], 0, sizeof(double) * 6, stream);
  }
  for (BatchRec* br : bs) {
    const Batch& b = br->b;
    launch_cells(b, stream);
    if (b.coul == RBMD_COUL_RBE) launch_rbe_sample(b, stream);
    if (b.coul != RBMD_COUL_NONE) launch_rho(b, stream, b.coul == RBMD_COUL_EWALD);
    if (b.has_bonded) launch_bonded(b, stream, 1);
    launch_pair(b, stream, 1);
    launch_final(b, stream, kFinalForceOnly, 1);
    launch_energy(b, stream);
    if (b.coul != RBMD_COUL_NONE) launch_ewald_energy(b, stream);
  }
  for (auto& p : ps) {
    const SysDev& D = p.s->dev;
    cudaMemcpyAsync(D.f, p.fsave, sizeof(double4) * D.n, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(&p.st, D.st, sizeof(SysState), cudaMemcpyDeviceToHost, stream);
    p.te.resize(p.s->n_terms);
    if (p.s->n_terms)
      cudaMemcpyAsync(p.te.data(), D.term_energy, sizeof(double) * p.s->n_terms, cudaMemcpyDeviceToHost, stream);
    dfree(p.fsave);
  }
  rc = sync();
  if (rc) return rc;
  for (int q = 0; q < nsys; ++q) {
    Pending& p = ps[q];
    System* s = p.s;
    const SysDev& D = s->dev;
    const SysState& st = p.st;
    std::vector<double>& te = p.te;
    rbmd_thermo* out = outs + q;
    if (!p.te_step.empty() && st.step > 0) te.swap(p.te_step);
    std::memset(out, 0, sizeof(*out));
    const int n = D.n;
    out->step = st.step;
    out->temperature = st.temperature;
    out->tempT_sum = st.tempT_sum;
    out->kinetic_energy = st.tempT_sum / n * 0.5;
    double eb = 0, ea = 0;
    for (int t = 0; t < D.n_bonds; ++t) eb += te[t];
    for (int t = 0; t < D.n_angles; ++t) ea += te[D.n_bonds + t];
    double ed = 0;
    for (int t = 0; t < D.n_dihedrals; ++t) ed += te[D.n_bonds + D.n_angles + t];
    out->e_dihedral = D.n_dihedrals ? ed / D.n_dihedrals : 0.0;
    out->e_bond = D.n_bonds ? eb / D.n_bonds : 0.0;
    out->e_angle = D.n_angles ? ea / D.n_angles : 0.0;
    if (D.ff == RBMD_FF_EAM) {
      out->e_eam = (st.energy[2] + st.energy[3]) / n;
    } else {
      out->e_lj = st.energy[0] / n;
      out->e_coul_near = st.energy[1] / n;
    }
    if (D.coul != RBMD_COUL_NONE)
      out->e_coul_far = D.qqr2e * st.energy[6] * ((2 * kPi / D.volume)) / n + s->self_energy;
    if (D.ff == RBMD_FF_LJ_CUT) out->potential_energy = out->e_lj;
    else if (D.ff == RBMD_FF_LJ_CUT_COUL_LONG) out->potential_energy = out->e_lj + out->e_coul_far + out->e_coul_near;
    else if (D.ff == RBMD_FF_CVFF)
      out->potential_energy =
          out->e_lj + out->e_coul_far + out->e_coul_near + out->e_bond + out->e_angle + out->e_dihedral;
    else out->potential_energy = out->e_eam;
    out->total_energy = out->potential_energy + out->kinetic_energy;
    double vir[6];
    for (int k = 0; k < 6; ++k) vir[k] = st.virial[k];
    if (s->p.fix_shake == RBMD_SHAKE_TRUE)
      for (int k = 0; k < 6; ++k) vir[k] += st.shake_virial[k];
    if (D.ff == RBMD_FF_EAM)
      for (int k = 0; k < 6; ++k) vir[k] = 0;
    out->pressure = (st.tdof * D.boltz * st.temperature + vir[0] + vir[1] + vir[2]) / 3.0 * (1.0 / D.volume) * D.nktv2p;
    if (D.npt && st.step > 0) {
      // NPT: the pressure of the step is the one the barostat used (PARA_PRESSURE,
      // ExecutionNPT.cpp:1446), taken before the remap
      out->pressure = st.baro_pressure;
      for (int k = 0; k < 6; ++k) vir[k] = st.baro_virial[k];
    }
    for (int k = 0; k < 6; ++k) out->virial[k] = vir[k];
    out->volume = D.volume;
    for (int k = 0; k < 3; ++k) {
      out->nhc_eta[k] = st.eta[k];
      out->box_lo[k] = D.lo[k];
      out->box_hi[k] = D.hi[k];
    }
    for (int k = 0; k < 4; ++k) out->nhc_eta_dot[k] = st.eta_dot[k];
    out->status = st.status;
  }
  return check_cuda("get_thermo");
}

int Context::get_cells(int id, int32_t* dims, int32_t* coa, int32_t* sorted, int32_t* lo, int32_t* up) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  int32_t one = id;
  int rc;
  rbmd_device_cfg saved = cfg;
  cfg.batched = 0;
  auto bs = batches_for(&one, 1, rc);
  cfg = saved;
  if (rc) return rc;
  launch_cells(bs[0]->b, stream);
  rc = refresh(s);
  if (rc) return rc;
  const SysDev& D = s->dev;
  if (dims)
    for (int k = 0; k < 3; ++k) dims[k] = D.dims[k];
  std::vector<int> start(D.ncell + 1), icell(D.n), isorted(D.n);
  cudaMemcpyAsync(icell.data(), D.cell_of_atom, sizeof(int) * D.n, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(isorted.data(), D.sorted, sizeof(int) * D.n, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(start.data(), D.cell_start, sizeof(int) * (D.ncell + 1), cudaMemcpyDeviceToHost, stream);
  rc = sync();
  if (rc) return rc;
  // internal id = z + dz (y + dy x); reference id = x + dx (y + dy z)
  const int dx = D.dims[0], dy = D.dims[1], dz = D.dims[2];
  auto to_ref = [&](int ic) {
    const int x = ic / (dz * dy), y = (ic / dz) % dy, z = ic % dz;
    return x + dx * (y + dy * z);
  };
  if (coa)
    for (int i = 0; i < D.n; ++i) coa[i] = to_ref(icell[i]);
  int run = 0;
  for (int z = 0; z < dz; ++z)
    for (int y = 0; y < dy; ++y)
      for (int x = 0; x < dx; ++x) {
        const int c = x + dx * (y + dy * z), ic = z + dz * (y + dy * x);
        if (lo) lo[c] = run;
        for (int k = start[ic]; k < start[ic + 1]; ++k) {
          if (sorted) sorted[run] = isorted[k];
          ++run;
        }
        if (up) up[c] = run;
      }
  return RBMD_OK;
}

int Context::get_rbl_lists(int id, int cap, int32_t* nc, int32_t* ns, int32_t* ids) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (cap <= 0 || !nc || !ns || !ids) return fail(RBMD_ERR_ARG, "bad list buffers");
  if (s->dev.neigh != RBMD_NEIGH_RBL) return fail(RBMD_ERR_STATE, "system does not use RBL");
  int32_t one = id;
  int rc;
  rbmd_device_cfg saved = cfg;
  cfg.batched = 0;
  auto bs = batches_for(&one, 1, rc);
  cfg = saved;
  if (rc) return rc;
  launch_cells(bs[0]->b, stream);
  rc = refresh(s);
  if (rc) return rc;
  const int n = s->dev.n;
  int *d_nc = nullptr, *d_ns = nullptr, *d_ids = nullptr;
  if (cudaMalloc(&d_nc, sizeof(int) * n) != cudaSuccess || cudaMalloc(&d_ns, sizeof(int) * n) != cudaSuccess ||
      cudaMalloc(&d_ids, sizeof(int) * 2 * (size_t)n * cap) != cudaSuccess) {
    cudaFree(d_nc);
    cudaFree(d_ns);
    return fail(RBMD_ERR_OOM, "list buffers");
  }
  launch_rbl_lists(d_sys_, s->slot, n, s->dev.ncell, s->dev.dense, cap, d_nc, d_ns, d_ids, stream);
  std::vector<int> core((size_t)n * cap), shell((size_t)n * cap);
  cudaMemcpyAsync(nc, d_nc, sizeof(int) * n, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(ns, d_ns, sizeof(int) * n, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(core.data(), d_ids, sizeof(int) * (size_t)n * cap, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(shell.data(), d_ids + (size_t)n * cap, sizeof(int) * (size_t)n * cap, cudaMemcpyDeviceToHost, stream);
  rc = sync();
  cudaFree(d_nc);
  cudaFree(d_ns);
  cudaFree(d_ids);
  if (rc) return rc;
  bool over = false;
  for (int i = 0; i < n; ++i) {
    const int a = nc[i], b2 = ns[i];
    if (a + b2 > cap) {
      over = true;
      continue;
    }
    for (int k = 0; k < a; ++k) ids[(size_t)i * cap + k] = core[(size_t)i * cap + k];
    for (int k = 0; k < b2; ++k) ids[(size_t)i * cap + a + k] = shell[(size_t)i * cap + k];
  }
  if (over) return fail(RBMD_ERR_ARG, "a list row exceeds cap");
  return RBMD_OK;
}

// Allocation-free lists: every temporary in the file-scope scratch of k_pair.cu.  The first call
// on a device looks the scratch address up (cudaGetSymbolAddress); later calls reuse it.
int Context::get_rbl_lists_static(int id, int cap, int32_t* nc, int32_t* ns, int32_t* ids) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (cap <= 0 || !nc || !ns || !ids) return fail(RBMD_ERR_ARG, "bad list buffers");
  if (s->dev.neigh != RBMD_NEIGH_RBL) return fail(RBMD_ERR_STATE, "system does not use RBL");
  const int rr = refresh(s);
  if (rr) return rr;
  const SysDev& D = s->dev;
  const long long need = static_list_ints(D.n, D.ncell, D.dense, cap);
  if (need > kStaticListInts)
    return fail(RBMD_ERR_ARG, "lists of " + std::to_string(D.n) + " atoms at cap " + std::to_string(cap) +
                                  " need " + std::to_string(need) + " ints of scratch; the static scratch holds " +
                                  std::to_string(kStaticListInts) + " (8 MiB)");
  int* scratch = nullptr;
  // The scratch lookup needs the context's device current; the caller's current device is put
  // back on every return, so an observer thread's own later CUDA work stays where it was.
  struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
      if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
      if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
      if (prev >= 0) cudaSetDevice(prev);
    }
  } guard(cfg.device);
  const int e = static_list_scratch(&scratch);
  if (e) return fail(RBMD_ERR_CUDA, std::string("static list scratch: ") + cudaGetErrorString((cudaError_t)e));
  StaticLists L;
  launch_rbl_lists_static(d_sys_, s->slot, D.n, D.ncell, D.dense, cap, scratch, stream, &L);
  int over = 0;
  cudaMemcpyAsync(nc, L.n_core, sizeof(int) * D.n, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(ns, L.n_shell, sizeof(int) * D.n, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(ids, L.rows, sizeof(int) * (size_t)D.n * cap, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(&over, L.flag, sizeof(int), cudaMemcpyDeviceToHost, stream);
  const int rc = sync();
  if (rc) return rc;
  if (over) return fail(RBMD_ERR_ARG, "a list row exceeds cap");
  return RBMD_OK;
}

int Context::get_kspace(int id, int32_t* m, double* rhok) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (s->dev.coul != RBMD_COUL_RBE) return fail(RBMD_ERR_STATE, "system does not use RBE");
  const int P = s->dev.P;
  if (m) cudaMemcpyAsync(m, s->dev.km, sizeof(int) * 3 * P, cudaMemcpyDeviceToHost, stream);
  if (rhok) cudaMemcpyAsync(rhok, s->dev.rhok, sizeof(double) * 2 * P, cudaMemcpyDeviceToHost, stream);
  return sync();
}

int Context::get_derived(int id, rbmd_derived* out) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  const int rc = refresh(s);
  if (rc) return rc;
  *out = s->dv;
  return RBMD_OK;
}

int Context::device_status(int id, int* status) {
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  int st = 0;
  cudaMemcpyAsync(&st, &s->dev.st->status, sizeof(int), cudaMemcpyDeviceToHost, stream);
  int rc = sync();
  *status = st;
  return rc;
}

}  // namespace rbmd
