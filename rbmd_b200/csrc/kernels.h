// kernels.h -- host-side launchers of the sm_100a kernels.  A launch covers every system listed
// in a Batch (segment-indexed work tables); the plain path builds one Batch per system.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace rbmd {

// Work item of a segment-indexed launch: (system slot, first element of the block).
struct Work {
  int2* d = nullptr;
  int n = 0;
};

struct Batch {
  SysDev* sys = nullptr;     // device array of all system records (indexed by slot)
  int* d_slots = nullptr;    // slots of this batch
  int nsys = 0;
  Work atom, pair, cell, rho, tri, term, kred, draw;
  Work pair_cells;           // column layout: the tile kernel's cell table (energies, other modes)
  // column layout: pair.d lists every column (slot, column index), most atoms per column first;
  // the persistent column kernel's warps take them in that order from col_ctr[0] (col_ctr[1] counts
  // the warps that are done; the last one resets both), col_grid blocks; the stray pass before it
  // uses col_ctr[2] and col_ctr[3] the same way, stray_grid blocks
  unsigned* col_ctr = nullptr;
  int col_grid = 0, stray_grid = 0;
  // uniform switches of the batch (a batch never mixes them)
  int ff = 0, neigh = 0, coul = 0, prec = 0, temp_ctrl = 0, special = 0;
  int has_shake = 0, has_bonded = 0;
  int dense = 0;             // pair kernel: 0 = warp per atom, 1 = warp per home cell, 2 = warp per column
  int lean = 0;              // warp per atom with segment tables (dims >= 2 nc + 1 everywhere)
  int npt = 0;               // NPT barostat: 0 none, 1 Berendsen (end of step), 2 MTK (around the integrator)
  int near = 0;              // RBL Coulomb with the reference's near-Coulomb table (RBMD_NEAR_TABLE)
  int max_P = 0;             // largest P (or Ewald nk) in the batch
  float band[4] = {0, 0, 0, 0};  // FP32 classification bands: union over the batch (same rc, rs)
  long long natoms = 0;      // atoms over all systems of the batch
};

enum FinalMode { kFinalForceOnly = 0, kFinalKick = 1, kFinalInit = 2 };

void launch_nhc_a(const Batch& b, cudaStream_t s);
void launch_kick_drift(const Batch& b, cudaStream_t s);
void launch_cells(const Batch& b, cudaStream_t s);
void launch_shake(const Batch& b, cudaStream_t s);
void launch_rattle(const Batch& b, cudaStream_t s);
void launch_rbe_sample(const Batch& b, cudaStream_t s);
void launch_rho(const Batch& b, cudaStream_t s, int ewald);
void launch_bonded(const Batch& b, cudaStream_t s, int virial);
void launch_pair(const Batch& b, cudaStream_t s, int virial);
// Blocks of the persistent column kernel for `ncols` columns: resident blocks per SM x SMs of the
// current device, fewer when the columns do not fill them (4 warps per block, a column per warp).
int pair_col_grid(int ncols, int ff, int special, int near, bool strays);
void launch_final(const Batch& b, cudaStream_t s, FinalMode mode, int virial);
void launch_ke_thermostat(const Batch& b, cudaStream_t s);
void launch_flush_vscale(const Batch& b, cudaStream_t s);
void launch_energy(const Batch& b, cudaStream_t s);
void launch_ewald_energy(const Batch& b, cudaStream_t s);
// NPT Berendsen barostat of every system of an NPT batch: new box and tables, then the remap.
void launch_barostat(const Batch& b, cudaStream_t s);
// MTK barostat systems: step start (both chains' first halves, barostat velocity, the two
// half-step boxes); replaces launch_nhc_a for such batches.
void launch_mtk_begin(const Batch& b, cudaStream_t s);

// RBL list materialisation for parity checks (not on the step path).
void launch_rbl_lists(const SysDev* sys, int slot, int n, int ncell, int dense, int cap, int* n_core,
                      int* n_shell, int* ids, cudaStream_t s);

// Allocation-free variant of the list materialisation: every temporary in one file-scope device
// array of kStaticListInts ints (8 MiB) per device.  static_list_scratch() looks its device address
// up once per device (the current one) and returns a cudaError_t; static_list_ints() is the number
// of ints a call needs; the launcher returns 1 (and launches nothing) when that exceeds
// kStaticListInts.  Calls that overlap on the GPU share the array and race.
constexpr long long kStaticListInts = 1LL << 21;
struct StaticLists {
  int* n_core = nullptr;   // [n]
  int* n_shell = nullptr;  // [n]
  int* rows = nullptr;     // [n * cap]: core ids, then shell ids, then -1
  int* flag = nullptr;     // nonzero: a row exceeded cap
};
int static_list_scratch(int** out);
long long static_list_ints(int n, int ncell, int dense, int cap);
int launch_rbl_lists_static(const SysDev* sys, int slot, int n, int ncell, int dense, int cap, int* scratch,
                            cudaStream_t s, StaticLists* out);

// Trajectory observables (between steps, not on the step path).
constexpr int kObsThreads = 256;
constexpr int kObsMaxBlocks = 4 * 148;        // partial sums of the MSD / VACF reduction
constexpr int kRdfTargetsPerBlock = 2048;     // targets one RDF block walks (grid.y splits the rest)
constexpr int kRdfSharedBins = 8192;          // bins counted in shared memory (32 KB); above, in global
int obs_blocks(int n);
// which: bit 0 positions and image counters, bit 1 velocities
void launch_obs_snapshot(const SysDev* sys, int slot, int n, int which, double4* x0, double4* v0, int4* img0,
                         cudaStream_t s);
// out[8] = (msd x, y, z, total, vacf x, y, z, total), averaged over atoms; part holds
// obs_blocks(n) x 8 doubles.
void launch_obs_msd_vacf(const SysDev* sys, int slot, int n, const double4* x0, const double4* v0, const int4* img0,
                         double* part, double* out, cudaStream_t s);
// Adds the RDF pair counts of one snapshot to counts[nb] (radii[b] = (b + 1) dr accumulated,
// upper[b] = radii[b] + 0.01 radii[b]).
void launch_rdf_count(const SysDev* sys, int slot, const int* centers, int nc, const int* targets, int nt,
                      const double* radii, const double* upper, int nb, double dr, int exclude_mol,
                      unsigned long long* counts, cudaStream_t s);

// Asynchronous snapshot: packed layout step (8 B), box lo / hi (6 doubles), x, v [3n] doubles,
// image [3n] ints; snapshot_bytes(n) in all.
size_t snapshot_bytes(int n);
void launch_snapshot_pack(const SysDev* sys, int slot, int n, void* out, cudaStream_t s);

constexpr int kCellWarpsHost = 4;  // home cells per block of the tile pair kernel
constexpr double kTileMinPerCell = 3.0;  // mean atoms per cell from which the tile kernel is used

double fma_peak_tflops(int fp64, cudaStream_t s);

// number of kernel launches issued by the launchers so far (all threads)
long long launches_issued();
void note_launch(int k = 1);

}  // namespace rbmd
