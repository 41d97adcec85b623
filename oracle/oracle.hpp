// oracle.hpp -- FP64 CPU restatement of RBMD's per-step force-and-integrate path.
//
// TEST INFRASTRUCTURE ONLY.  This code is the checker for the CUDA library in rbmd_b200/; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may load it.
// The product never links, loads or calls it.
//
// PARITY UNPINNED: the reference (randbatch-md/rbmd 2.2.0) needs VTK-m 1.9, which is not in this
// environment, so it cannot be compiled or run here, and its own tests pin an older framework
// (tests/ is disabled in its CMakeLists.txt:37-45).  This restatement follows the reference source
// line by line (citations on every function, paths relative to the reference root) and is pinned
// instead by physics known-answer tests (Madelung constant, closed-form pair forces, Ewald alpha
// independence, RBE unbiasedness, SHAKE geometry, EAM spline vs analytic Johnson functions).
//
// Deliberate departures from the reference, each also implemented identically by the CUDA path:
//  * Coulomb real space uses analytic erfc, not the alpha=0.1 float-bit-indexed table of
//    framework/staticTable/ExecStaticTable.h:96-135 (which is only valid for alpha = 0.1).
//  * RBL lists are not sized from the mean density (framework/run/ExecutionMD.cpp:582-616), so a
//    core count above rs_num does not alias into the shell region (RunWorklet.cpp:955-970).
//  * Randomness comes from Philox4x32-10 keyed by (seed, step, index) instead of std::mt19937
//    reseeded from std::random_device on every draw (framework/math/Utiles.h:32-39).
//  * SHAKE/RATTLE update only the atoms of constrained triples; the reference copies the whole
//    pre-update position/velocity arrays back (ExecutionNVT.cpp:868-870,896), which freezes every
//    atom outside a water triple.  Triples themselves follow the reference exactly.
//  * Bonded forces are reduced per atom id; without special_bonds the reference's ReduceByKey
//    output is indexed by unique key, not atom id (ExecutionNVT.cpp:491-495).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "../include/rbmd_gpu.h"

namespace oracle {

// Parallel loop over [0, n) in contiguous chunks on std::threads (RBMD_ORACLE_THREADS, default all
// cores).  Every index writes only its own outputs, so results do not depend on the thread count.
template <class Fn>
inline void par_for(long n, Fn&& fn) {
  static int nt = [] {
    const char* e = std::getenv("RBMD_ORACLE_THREADS");
    int v = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
    return v > 0 ? v : 1;
  }();
  const long T = std::min<long>(nt, std::max<long>(1, n / 16));
  if (T <= 1) {
    for (long i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(T);
  for (long t = 0; t < T; ++t)
    th.emplace_back([&, t] {
      const long a = n * t / T, b = n * (t + 1) / T;
      for (long i = a; i < b; ++i) fn(i);
    });
  for (auto& x : th) x.join();
}

constexpr double kPi = 3.14159265358979323846;          // vtkm::Pi()
// NPT box limits of this implementation (the reference has none): a remap whose edge would leave
// [kBoxShrink, kBoxGrow] x the initial edge, or give fewer cells than num_cycles, is refused with
// RBMD_STATUS_BOX_RANGE and the box stays put.  The CUDA path sizes its cell tables by kBoxGrow.
constexpr double kBoxGrow = 1.25, kBoxShrink = 0.8;
constexpr double kPif = 3.1415927410125732421875;        // (double)vtkm::Pif(), the float pi

struct Units {  // ExecutionMD::InitParameters, framework/run/ExecutionMD.cpp:329-360
  double kB, fmt2v, mvv2e, qqr2e, boltz, nktv2p;
};
Units make_units(int units);

struct Derived {
  int rs_num = 0, rc_num = 0, pice_num = 1, num_cycles = 1;
  int dims[3] = {1, 1, 1};
  int ncell = 1;
  double rho = 0, S = 0, volume = 0;
  double d[3] = {0, 0, 0};
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), restated from the paper.
void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double u01(uint32_t hi, uint32_t lo);  // 53-bit uniform in [0, 1)

// Counter tags (third counter word) of the random streams.
enum : uint32_t {
  kTagRbeGauss = 0x52424531u,   // RBE proposal Box-Muller uniforms
  kTagRbeAccept = 0x52424532u,  // RBE Metropolis acceptance uniform
  kTagRblOffset = 0x52424c31u   // RBL stride start offset (philox RBL mode)
};

struct Cells {
  int dims[3] = {1, 1, 1};
  double d[3] = {0, 0, 0};
  std::vector<int> cell_of_atom, sorted, lower, upper;
};

struct Thermostat {  // ExecutionNVT::InitialCondition / SetUp, ExecutionNVT.cpp:139-187,1106-1122
  double eta[3] = {0, 0, 0};
  double eta_dot[4] = {0, 0, 0, 0};
  double eta_dotdot[3] = {0, 0, 0};
  double eta_mass[3] = {0, 0, 0};
  double t_target = 0, ke_target = 0, t_freq = 0, tdrag_factor = 1;
  double temperature = 0;  // PARA_TEMPT
  double tempT_sum = 0;    // PARA_TEMPT_SUM
  double tdof = 0;
};

struct Barostat {  // ExecutionNPT MTK state, ExecutionNPT.cpp:145-232, 1545-1603 (iso, pdim 3)
  double omega_dot[3] = {0, 0, 0}, omega_mass[3] = {0, 0, 0};
  double etap[3] = {0, 0, 0}, etap_dot[4] = {0, 0, 0, 0}, etap_dotdot[3] = {0, 0, 0}, etap_mass[3] = {0, 0, 0};
  double p_hydro = 0, p_current = 0, mtk_term1 = 0, mtk_term2 = 0;
};

// The reference's near-Coulomb table for alpha = 0.1 (model/ERFTable.h; the points its files
// res/json_files/Gnear_table_{leq,geq}2_2.txt list), [2048] by key; see oracle_core.cpp.
int near_key(float r);
void near_table(float* out);

class System {
 public:
  System(const rbmd_system_desc& desc, const rbmd_params& params);

  // ---- state (Para fields)
  int N = 0, ntypes = 0;
  std::vector<double> x, v, f;  // [3N]
  std::vector<int> image;       // [3N]
  std::vector<double> q, m;
  std::vector<int> type, mol;
  std::vector<double> eps, sig;
  std::vector<int> bond_atoms, bond_type, angle_atoms, angle_type;
  std::vector<double> bond_k, bond_r0, angle_k, angle_theta0;
  std::vector<int> dihedral_atoms, dihedral_type, dihedral_sign, dihedral_mult;
  std::vector<double> dihedral_k;
  std::vector<int> special_offsets, special_ids;
  std::vector<double> special_weights;
  std::vector<int> mol_offsets, mol_atoms;  // molecule member CSR (ContTopology source/offsets)
  int eam_nrho = 0, eam_nr = 0;
  double eam_drho = 0, eam_dr = 0, eam_rhomax = 0, eam_cut = 0;
  std::vector<double> frho_spline, rhor_spline, z2r_spline;
  // setfl (LAMMPS eam/alloy): tables per type, z2r per type pair i >= j at i (i+1)/2 + j
  int eam_per_type = 0;
  const double* frho_of(int t) const { return &frho_spline[eam_per_type ? (size_t)t * 7 * (eam_nrho + 1) : 0]; }
  const double* rhor_of(int t) const { return &rhor_spline[eam_per_type ? (size_t)t * 7 * (eam_nr + 1) : 0]; }
  const double* z2r_of(int a, int b) const {
    const int hi = a > b ? a : b, lo = a > b ? b : a;
    return &z2r_spline[eam_per_type ? (size_t)(hi * (hi + 1) / 2 + lo) * 7 * (eam_nr + 1) : 0];
  }

  // RBMD_NEAR_TABLE (RBL near Coulomb): G by the 11-bit key of the FP32 distance,
  // ExecStaticTable::Extract / TableGnearValue (staticTable/ExecStaticTable.h:96-135)
  std::vector<float> near_tab;
  double near_g(double dis) const;

  rbmd_params p;
  Units u;
  Derived dv;
  double lo[3], hi[3], L[3];
  double L0[3];                  // box edges at set-up (barostat range limits)
  int ncell_cap = 0;             // NPT: cells of the largest accepted box
  double baro_pressure = 0.0;    // NPT: pressure and virial the barostat last used (PARA_PRESSURE)
  double baro_virial[6] = {0, 0, 0, 0, 0, 0};
  int64_t step = 0;  // Executioner::_current_step
  Thermostat th;
  Barostat bs;
  Cells cells;

  // last force evaluation by-products
  std::vector<int> kspace_m;      // [3P]
  std::vector<double> rhok;       // [2P]
  std::vector<double> f_near, f_far, f_bonded;  // [3N]
  double virial[6] = {0, 0, 0, 0, 0, 0};
  double e_bond_avg = 0, e_angle_avg = 0, e_dihedral_avg = 0;
  std::vector<double> shake_virial_atom;  // [6 * n_angles]
  int status = 0;

  // ---- the path
  void build_cells();                                   // a1
  template <class Fn> void traverse(int i, Fn&& fn) const;  // a2
  void rbl_lists(std::vector<int>& ncore, std::vector<int>& nshell,
                 std::vector<std::vector<int>>& ids,
                 std::vector<std::vector<std::array<double, 3>>>* offs) const;  // a3
  void verlet_lists(std::vector<std::vector<int>>& ids,
                    std::vector<std::vector<std::array<double, 3>>>& offs) const;  // a4
  void sample_k();                                      // a10
  void structure_factor();                              // a11
  void rbe_force(std::vector<double>& F, double vir[6]) const;   // a12
  void ewald_force(std::vector<double>& F, double vir[6]) const; // a14
  void near_force(std::vector<double>& F);              // a5 / a7 / a8 / a15
  void bonded_force(std::vector<double>& F);            // a9 / a19
  void compute_force();                                 // a20 (ExecutionNVT::ComputeForce)
  void init();                                          // ExecutionNVT::Init tail
  void step_once();                                     // Executioner::TakeStep
  void thermo(rbmd_thermo* out);                        // a13 / a21 / a22

  // helpers
  void min_image(double r[3]) const;
  void set_box(const double nlo[3], const double nhi[3]);
  void pressure_scalar(double vir[6], double& press) const;
  void barostat_berendsen();
  bool mtk() const { return p.ensemble == RBMD_ENS_NPT && p.press_ctrl == RBMD_PC_NOSE_HOOVER; }
  void mtk_setup();
  void nhc_press_integrate();
  void compute_press_target();
  void nh_omega_dot();
  void nh_v_press();
  void mtk_remap();
  void step_mtk();
  void compute_tempe();
  void compute_temp_target();
  void nhc_integrate();
  void update_velocity(std::vector<double>* old_v);
  void update_position(std::vector<double>* old_x);
  void shake(const std::vector<double>& old_x, const std::vector<double>& old_v);
  void rattle(const std::vector<double>& old_v);
  double ewald_energy_total(const int kmax[3]) const;
  void energies(double& e_lj, double& e_coul, double& e_eam) const;
  int rbl_offset(int atom) const;
};

// EAM file handling (ExecutionNVT.cpp:899-1079).
struct EamFile {
  int nrho = 0, nr = 0;
  double drho = 0, dr = 0, cut = 0;
  std::vector<double> frho, zr, rhor;
};
bool read_funcfl(const std::string& path, EamFile& out);
// setfl (LAMMPS eam/alloy PairEAMAlloy::file2array + array2spline): tables splined on the file's
// grid, expanded to atom types (type t takes element type_element[t]); z2r per type pair i >= j at
// i (i+1)/2 + j.  frho [ne][nrho], rhor [ne][nr], z2r [ne(ne+1)/2][nr] row-major.
void build_setfl_splines(int ne, int nrho, double drho, int nr, double dr, const double* frho, const double* rhor,
                         const double* z2r, const int* type_element, int n_types, std::vector<double>& frho_s,
                         std::vector<double>& rhor_s, std::vector<double>& z2r_s, double& rhomax);
void build_splines(const EamFile& in, std::vector<double>& frho_s, std::vector<double>& rhor_s,
                   std::vector<double>& z2r_s, int& nrho, double& drho, int& nr, double& dr,
                   double& rhomax);

// ------------------------------------------------------------------ a2: traversal
// Calls fn(j, off[3], r[3], dis2) for every atom of the (2 nc + 1)^3 neighbour cells of atom i, in
// the reference order: x offset outermost, z innermost, ascending id within a cell.
// ComputeRBLNeighboursOnceWorklet, framework/run/worklet/RunWorklet.cpp:929-952, with
// ExecPointLocator::{InWhichCell,PeriodicIndexOffset,PeriodicCoordOffset}, ExecPointLocator.h:271-305.
template <class Fn>
inline void System::traverse(int i, Fn&& fn) const {
  const double pi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  const int* dims = cells.dims;
  int c[3];
  for (int k = 0; k < 3; ++k) c[k] = (int)((pi[k] - lo[k]) / cells.d[k]);
  const int nc = dv.num_cycles;
  for (int a = -nc; a <= nc; ++a)
    for (int b = -nc; b <= nc; ++b)
      for (int e = -nc; e <= nc; ++e) {
        int nb[3] = {c[0] + a, c[1] + b, c[2] + e};
        int w[3];
        double off[3];
        for (int k = 0; k < 3; ++k) {
          w[k] = ((nb[k] % dims[k]) + dims[k]) % dims[k];  // true modulo of (n + dims) % dims
          off[k] = cells.d[k] * (double)(w[k] - nb[k]);
        }
        int cell = w[0] + w[1] * dims[0] + w[2] * dims[0] * dims[1];
        for (int s = cells.lower[cell]; s < cells.upper[cell]; ++s) {
          int j = cells.sorted[s];
          double pj[3], r[3];
          for (int k = 0; k < 3; ++k) {
            pj[k] = x[3 * j + k] - off[k];
            r[k] = pj[k] - pi[k];
          }
          double dis2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
          fn(j, off, r, dis2);
        }
      }
}

}  // namespace oracle
