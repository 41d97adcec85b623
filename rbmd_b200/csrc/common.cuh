// common.cuh -- device-side system record, random streams and warp/block helpers shared by the
// sm_100a kernels of the RBMD force-and-integrate path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rbmd_gpu.h"

namespace rbmd {

constexpr double kPi = 3.14159265358979323846;
constexpr double kPif = 3.1415927410125732421875;  // float pi promoted, as the reference's Pif()

constexpr int kWarp = 32;
constexpr int kPairWarps = 8;          // atoms (warps) per block of the pair kernel
constexpr int kAtomBlock = 256;        // atoms per block of the streaming kernels
constexpr int kRhoChunk = 256;         // atoms per block of the structure-factor kernel
constexpr int kCellBlock = 256;        // cells per block of the cell kernels
constexpr int kRbeSlack = 64;          // extra Metropolis proposal slots beyond P
constexpr int kQueue = 64;             // per-warp pair queue of the pair kernel
constexpr int kMaxF32Types = 16;       // atom types of the FP32 (mixed) pair table

// device error word bits (rbmd_thermo.status)
enum : int {
  kErrShakeOverflow = 1, kErrShakeSingular = 2, kErrShakeNoConverge = 4, kErrRattleSingular = 8,
  kErrNonFinite = 16, kErrRbeSlots = 32, kErrBoxRange = 64
};

// NPT box limits (edges relative to the initial box); cell tables are sized for kBoxGrow.
constexpr double kBoxGrow = 1.25, kBoxShrink = 0.8;

// Random stream tags (third Philox counter word); must match the oracle's.
enum : uint32_t {
  kTagRbeGauss = 0x52424531u, kTagRbeAccept = 0x52424532u, kTagRblOffset = 0x52424c31u
};

// Binned cells of atoms that SHAKE wrapped across the box after the cell list was built, kept per
// step; beyond this many the culling pair kernels walk whole stencils for the step.
constexpr int kMaxMigrated = 16;

// Per-system scalar state that kernels read and update on the device (thermostat chain,
// reductions, step counter).  One record per system, in device memory.
struct SysState {
  double eta[3], eta_dot[4], eta_dotdot[3], eta_mass[3];
  double t_target, ke_target, t_freq, tdrag, tdof;
  double temperature;      // PARA_TEMPT
  double tempT_sum;        // PARA_TEMPT_SUM
  double vscale_pending;   // velocity factor not yet applied (end-of-step thermostat)
  double vscale_pending_c; // same for atoms of constrained triples
  double vscale_a;         // factor of the start-of-step half of the chain
  double fmean[3];         // RBL mean near force of the last evaluation
  double virial[6];        // last virial sum (when requested)
  double shake_virial[6];  // sum of the last SHAKE virials
  double energy[8];        // energy scratch: lj, coul, eam_embed, eam_pair, bond, angle, ewald, self
  double baro_pressure;    // NPT: pressure the barostat used this step (PARA_PRESSURE)
  double baro_virial[6];   // NPT: virial behind it
  double baro_lo_old[3];   // NPT: range minimum before this step's remap
  double baro_hinv_old[3]; // NPT: 1 / edge before this step's remap
  int baro_apply;          // NPT: this step's remap was accepted
  int mtk_ok[2];           // MTK: which of the two half-step remaps were accepted
  int baro_pad;
  // MTK barostat (isotropic): barostat velocity and mass, its chain, targets, NH_V_Press factors
  double omega_dot[3], omega_mass[3];
  double etap[3], etap_dot[4], etap_dotdot[3], etap_mass[3];
  double p_hydro, p_current, mtk_term1, mtk_term2;
  double f_press[3];
  // MTK half-step remaps: range minimum and 1 / edge of the box before each, and the box between
  double mtk_lo0[3], mtk_hinv0[3], mtk_lo1[3], mtk_hi1[3], mtk_L1[3], mtk_hinv1[3];
  int64_t step;            // Executioner current step
  int status;              // error word
  int pad;
  unsigned counter[8];     // last-block arrival counters
  // Positions SHAKE changed since this step's cell list was built (the reference's locator keeps
  // the cells of before the constraint, ExecutionNVT.cpp:843-870): the largest displacement (FP32
  // bits, non-negative) and the binned cells of atoms it wrapped across the box.  Reset with the
  // cell list.  The pair kernels that cull cells geometrically widen by the displacement and never
  // cull a recorded cell (an atom there sits on the far side of the box).
  unsigned shake_disp_bits;
  // The farthest any atom lay outside its binned cell when the cell list was built (FP32 bits,
  // rounded up): atoms given outside the box are binned into the clamped edge cell.  The culling
  // margins widen by it too.
  unsigned out_bits;
  int mig_n;
  int mig_cell[kMaxMigrated];
};

struct SysDev {
  // sizes and switches
  int n, ntypes, ff, neigh, coul, prec, rbl_mode, random_mode, temp_ctrl, fix_shake, inbuild;
  int special, pice, nc, ncell, P, n_bonds, n_angles, nk_ewald;
  int dims[3];
  int eam_nrho, eam_nr;
  int eam_per_type;  // EAM tables per type (setfl): frho / rhor by type, z2r by type pair
  int eam_pad;
  int lean;   // segment-table traversal usable (every dimension holds more than nc cells)
  int dense;  // pair kernel layout: 0 warp per atom, 1 tile (warp per home cell), 2 column (warp per
              // column of home cells, lane per atom; FP32 RBL forces only, the tile kernel otherwise)
  int blocks_pair, blocks_atom, blocks_rho, blocks_tri, rbe_mmax, rbe_slots, has_triples, n_triples;
  // NPT barostats (npt 1: Berendsen at the end of the step, 2: MTK around the integrator): the
  // box changes on the device every step.  Cell arrays and the cell work table hold ncell_cap cells
  // (the box at kBoxGrow x L0); kmax indexes the Ewald k lists.
  int npt, ncell_cap, kmax[3], npt_pad;
  double L0[3];
  double p_start, p_stop, p_damp, bulk;
  // geometry and physics
  double lo[3], hi[3], L[3], d[3];
  double rc, rs, rc2, rs2, alpha, volume, S;
  double qqr2e, fmt2v, mvv2e, kB, boltz, nktv2p;
  // FP32 constants of the mixed-precision pair evaluation: sqrt(alpha), alpha log2(e) (so that
  // exp(-alpha d2) = 2^(-falpha_l2 d2)) and qqr2e, each rounded once from FP64
  float fsa, falpha_l2, fqq, fpad;
  double dt, t_start, t_stop, t_damp;
  int64_t num_steps;
  double eam_dr, eam_drho, eam_rhomax, eam_cut;
  double rbe_sigma[3];
  // Pair classification thresholds, exact equivalents of the reference's tests on d2 in each
  // precision: d2 <= c[0]  <=>  rc2 - d2 > 1e-4;  d2 >= c[1]  <=>  d2 - rs2 > 1e-4;
  // d2 <= c[2]  <=>  rs2 - d2 > 1e-4 (each side of the test rounded as the reference rounds it).
  double cls_d[3];
  float cls_f[3];
  int cls_pad;
  // Mixed precision: bands [band[0], band[1]] around the rs thresholds and [band[2], band[3]]
  // around the rc threshold of FP32 squared distance (a bound on the FP32 rounding error) inside
  // which a pair is classified again in FP64; below band[0] a pair is surely core, between
  // band[1] and band[2] surely shell, above band[3] surely out
  float band[4];
  uint32_t seed_lo, seed_hi;
  // atom arrays (original order)
  double4* x;          // x, y, z, charge
  double4* v;          // vx, vy, vz, mass
  double4* f;          // force
  double4* xold;       // pre-drift positions (SHAKE)
  double4* vold;       // pre-kick velocities (SHAKE first half)
  double4* vold2;      // pre-kick velocities (RATTLE)
  int4* meta;          // type, molecule, flags (bit0: in a constrained triple), unused
  int* image;          // [3n]
  // cells
  int* cell_of_atom;   // reference flat cell id
  int* cell_count;     // [ncell]
  int* cell_start;     // [ncell + 1]
  int* cell_fill;      // [ncell] scatter cursors
  int* sorted;         // atom ids in cell order
  int* rank;           // [n] position of each atom in cell order (inverse of sorted)
  double4* sx;         // sorted positions + charge (FP64)
  float4* sxf;         // sorted positions + charge (FP32)
  int4* smeta;         // sorted: atom id, type, molecule, unused
  // per-type tables
  double* eps;
  double* sig;
  float2* ljf;  // mixed precision, [ntypes^2] by type pair a ntypes + b: -24 sqrt(eps_a eps_b) and
                // ((sig_a + sig_b) / 2)^6, each rounded once from FP64
  float* near_tab;  // RBMD_NEAR_TABLE with RBL Coulomb: G by key [kNearKeys]; nullptr: analytic G
  // special-bond CSR and molecules
  int* sp_off;
  int* sp_ids;
  double* sp_w;
  int* mol_off;
  int* mol_atoms;
  // bonded terms
  int* bond_atoms;
  int* bond_type;
  double* bond_k;
  double* bond_r0;
  int* angle_atoms;
  int* angle_type;
  double* angle_k;
  double* angle_t0;
  int n_dihedrals;      // harmonic dihedrals (CVFF with special bonds and a Dihedrals section)
  int dih_pad;
  int* dih_atoms;       // [4 n_dihedrals]
  int* dih_type;        // [n_dihedrals]
  double* dih_k;        // per type: K
  int* dih_sign;        // per type: d (1 or other: -1)
  int* dih_mult;        // per type: n
  double4* term_force; // [2 n_bonds + 3 n_angles + 4 n_dihedrals] per-term forces
  int* aterm_off;      // [n + 1] atom -> term-force slots (CSR)
  int* aterm;          // slots
  double* term_energy; // [n_bonds + n_angles + n_dihedrals]
  double* term_vir;    // [6 (n_bonds + n_angles + n_dihedrals)] per-term virials (pressure requests)
  // k space
  int* km;             // [3P] sampled m vectors
  double4* kv;         // [P or nk] k vector + coefficient -4 pi / (V k^2) (Ewald: x exp(-k^2/4a))
  double* rhok;        // [2P or 2nk]
  double* rho_part;    // [blocks_rho * 2P]
  double* rbe_tab;     // [3 * (2 mmax + 1) * 2]: P(m), q(m) per dimension
  double4* kv_e;       // [nk_e] Ewald-energy k vectors (kmax grid), w = exp(-k^2/4a)/k^2
  double* rhok_e;      // [2 nk_e]
  int nk_e;
  int pad_e;
  // EAM
  double* frho_s;
  double* rhor_s;
  double* z2r_s;
  double* eam_fp;      // [n]
  // reductions
  double* pair_part;   // [blocks_pair * 4]
  double* atom_part;   // [blocks_atom * 8]
  double* vir_part;    // [blocks_pair * 9] pair-kernel partials
  double* tri_part;    // [blocks_tri * 6] SHAKE virial partials
  SysState* st;
};

// ------------------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11.
__host__ __device__ inline void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
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

__host__ __device__ inline double u01(uint32_t hi, uint32_t lo) {
  uint64_t bits = ((uint64_t)(hi >> 5) << 26) | (uint64_t)(lo >> 6);
  return (double)bits * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------------------------ reductions
template <typename T>
__device__ inline T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ inline unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Last-block-done pattern: every block of a system calls this after writing its partials; the
// block that arrives last gets true and may reduce all partials of the system in a fixed order.
// The counter is reset by the last block, so the pattern needs no host-side clearing.
__device__ inline bool arrive_last(unsigned* counter, unsigned nblocks) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    s_last = (t == nblocks - 1);
    if (s_last) *counter = 0u;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// Orthorhombic minimum image (ExecPointLocator::MinDistanceVec).
template <typename R>
__device__ inline void min_image(R& x, R& y, R& z, R Lx, R Ly, R Lz) {
  if (fabs(x) > Lx * R(0.5)) x -= (x > R(0) ? Lx : -Lx);
  if (fabs(y) > Ly * R(0.5)) y -= (y > R(0) ? Ly : -Ly);
  if (fabs(z) > Lz * R(0.5)) z -= (z > R(0) ? Lz : -Lz);
}

}  // namespace rbmd
