// engine.h -- host-side context, systems and step orchestration behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.h"

namespace rbmd {

struct Units {
  double kB, fmt2v, mvv2e, qqr2e, boltz, nktv2p;
};
Units make_units(int units);

// One system: its parameters, derived quantities and device allocations.
struct System {
  int id = -1;
  int slot = -1;
  rbmd_params p{};
  rbmd_derived dv{};
  SysDev dev{};                 // host mirror of the device record
  std::vector<void*> allocs;    // device allocations owned by the system
  int64_t bytes = 0;
  double self_energy = 0.0;     // per-atom Ewald self energy (qqr2e applied)
  int n_terms = 0;
  int P = 0;
  std::vector<double> charge;   // host copy (energies)
  bool tuned = false;           // pair layout chosen by the autotuner (or fixed: NPT, environment)
  // MSD / VACF reference configuration (allocated by the first observe_reset)
  double4* obs_x0 = nullptr;
  double4* obs_v0 = nullptr;
  int4* obs_img0 = nullptr;
  int obs_have = 0;             // RBMD_OBS_* bits taken
};

// The tile pair kernel's traversal: every dimension holds more than nc cells, so each stencil
// offset needs one periodic image at most (a stencil may still repeat cells), and every edge is at
// least 2 rc, so a pair within rc is at its nearest image (the reference evaluates forces at the
// minimum image; the tile kernel's FP32 evaluation uses the traversal image as it is).
inline bool tile_layout_ok(const SysDev& D) {
  for (int k = 0; k < 3; ++k)
    if (D.dims[k] < D.nc + 1 || D.L[k] < 2.0 * D.rc) return false;
  return true;
}
// The lean kernel's (warp per atom over per-row segment tables): more than nc cells per dimension,
// so a row's z cells take three ranges at most; it evaluates forces at the minimum image.
inline bool lean_layout_ok(const SysDev& D) {
  return D.dims[0] >= D.nc + 1 && D.dims[1] >= D.nc + 1 && D.dims[2] >= D.nc + 1;
}
// The column kernel's (warp per column of home cells, lane per atom): the tile kernel's boxes, FP32
// RBL forces of LJ/CUT, LJ/CUT/COUL/LONG and CVFF; every other pass of such a system runs the tile
// kernel over its cell table.
inline bool column_layout_ok(const SysDev& D) {
  return tile_layout_ok(D) && D.n < (1 << 25) && D.prec == RBMD_PREC_MIXED && D.neigh == RBMD_NEIGH_RBL &&
         D.ff != RBMD_FF_EAM;
}
// Blocks per system of the tile pair kernel (4 home cells per block; also the column layout's cell
// table for the passes the column kernel does not run).
inline int tile_blocks(const SysDev& D) { return (D.ncell + 3) / 4; }

// Doubles in each EAM spline array of a descriptor: frho, rhor and z2r (per type when
// eam_per_type, one table each otherwise).
inline void eam_table_sizes(const rbmd_system_desc& d, size_t* nf, size_t* nr, size_t* nz) {
  const size_t t = d.eam_per_type ? (size_t)d.n_types : 1, pairs = d.eam_per_type ? t * (t + 1) / 2 : 1;
  *nf = 7 * (size_t)(d.eam_nrho + 1) * t;
  *nr = 7 * (size_t)(d.eam_nr + 1) * t;
  *nz = 7 * (size_t)(d.eam_nr + 1) * pairs;
}

// The reference's near-Coulomb lookup table (ExecStaticTable.h:96-135, ERFTable.h): the key of a
// distance and the library's table of G for alpha = 0.1 by key (include/rbmd_gpu.h documents both).
constexpr int kNearKeys = RBMD_NEAR_TABLE_KEYS;
int near_table_key(float r);
void near_table_default(float* out);

// RDF bins of radius / dr (RDFOutput.cpp:42-53): (int)(radius / dr) radii, dr accumulated by
// repeated addition.  Returns the bin count, or -1 for a bad (radius, dr).
int rdf_bins(double radius, double dr, std::vector<double>* radii);

struct Profiler {
  bool on = false;
  struct Rec {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    std::vector<double> units;
    double ms = 0.0;
    long long n = 0;
    double units_sum = 0.0;
  };
  std::map<std::string, Rec> recs;
};

// Systems that one launch can cover: same kernel configuration (and, with layout, the same pair
// traversal layout).
bool same_group(const System* a, const System* b, bool layout);

class Context {
 public:
  explicit Context(const rbmd_device_cfg& cfg);
  ~Context();

  int add_system(const rbmd_system_desc& d, const rbmd_params& p, int32_t* id);
  int remove_system(int id);
  int init(const int32_t* ids, int n);
  int step(const int32_t* ids, int n, int nsteps);
  int compute_forces(const int32_t* ids, int n);
  int sync();
  int get_forces(int id, double* f);
  int get_state(int id, double* x, double* v, int32_t* image);
  int set_state(int id, const double* x, const double* v, const int32_t* image);
  int set_step(int id, int64_t step);
  int get_thermo(int id, rbmd_thermo* out);
  int get_thermo_many(const int32_t* ids, int n, rbmd_thermo* outs);
  int get_cells(int id, int32_t* dims, int32_t* coa, int32_t* sorted, int32_t* lo, int32_t* up);
  int get_rbl_lists(int id, int cap, int32_t* nc, int32_t* ns, int32_t* ids);
  int get_rbl_lists_static(int id, int cap, int32_t* nc, int32_t* ns, int32_t* ids);
  int get_kspace(int id, int32_t* m, double* rhok);
  int get_derived(int id, rbmd_derived* out);
  int device_status(int id, int* status);
  int autotune(const int32_t* ids, int n, rbmd_tune_result* out, int cap, int* n_groups, bool keep_forces = true);
  int observe_reset(int id, int which);
  int observe(int id, double* msd, double* vacf);
  int rdf_counts(int id, const int32_t* centers, int nc, const int32_t* targets, int nt, double radius, double dr,
                 int exclude_same_molecule, int64_t* counts, double* volume);
  int snapshot_begin(int id, double* x, double* v, int32_t* image, double* box, int64_t* step, int64_t* ticket);
  int snapshot_poll(int64_t ticket, int* done);
  int snapshot_wait(int64_t ticket, double timeout_s);

  int fail(int code, const std::string& msg);
  std::string last_error;
  rbmd_device_cfg cfg{};
  cudaStream_t stream = nullptr;
  Profiler prof;
  std::recursive_mutex mu;

  System* find(int id);
  static int64_t estimate_bytes(const rbmd_system_desc& d, const rbmd_params& p);
  // Stream-ordered device memory from the context's own pool (which keeps freed memory for reuse):
  // admitting and retiring systems then costs no device-wide synchronisation.  dmalloc returns
  // nullptr (and clears the error) when the pool cannot grow.
  void* dmalloc(size_t bytes);
  bool pooled() const { return pool_ != nullptr; }
  // bytes of device memory the pool holds (in use or free for reuse)
  int64_t pool_reserved() const {
    uint64_t v = 0;
    if (pool_) cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrReservedMemCurrent, &v);
    return (int64_t)v;
  }
  void dfree(void* p);

 private:
  struct BatchRec {
    Batch b;
    std::vector<void*> allocs;
    std::vector<int> ids;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
  };
  int ensure_slots(int need);
  int upload_record(System* s);
  int refresh(System* s);
  void set_layout(System* s, int layout);
  std::vector<int> usable_layouts(const System* s) const;
  std::vector<BatchRec*> batches_for(const int32_t* ids, int n, int& rc);
  BatchRec* build_batch(const std::vector<System*>& group, int& rc);
  void drop_batches_with(int id);
  void enqueue_step(const Batch& b);
  void enqueue_forces(const Batch& b, FinalMode mode, int virial);
  template <class F> void timed(const char* name, double units, F&& fn);
  int check_cuda(const char* where);

  std::vector<System*> systems_;
  std::vector<int> free_slots_;
  SysDev* d_sys_ = nullptr;
  cudaMemPool_t pool_ = nullptr;
  int slot_cap_ = 0;
  int next_id_ = 0;
  std::map<std::vector<int>, BatchRec*> batch_cache_;
  std::map<std::vector<int64_t>, int> tune_cache_;  // autotuner decisions by group signature
  // asynchronous snapshots: packed on `stream`, copied to pinned staging on copy_stream_
  struct Snap {
    int n = 0;
    double *x = nullptr, *v = nullptr, *box = nullptr;
    int32_t* image = nullptr;
    int64_t* step = nullptr;
    void* dbuf = nullptr;
    void* hbuf = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;
  };
  std::map<int64_t, Snap> snaps_;
  int64_t next_ticket_ = 1;
  cudaStream_t copy_stream_ = nullptr;
  std::vector<std::pair<size_t, void*>> pinned_free_;  // pinned staging kept for reuse
  void* pinned_get(size_t bytes, size_t* got);
  void pinned_put(void* p, size_t bytes);
  void snapshot_finish(int64_t ticket);
  void snapshots_release();
};

}  // namespace rbmd
