// tune.cpp -- autotuner of the pair traversal layout (rbmd_autotune).
//
// The three pair kernels compute the same forces with the work cut differently: the tile layout
// (warp per home cell, candidate batches shared by the cell's atoms) wins when cells hold several
// atoms and the arithmetic is FP32; the lean layout (warp per atom over per-row segment tables)
// when cells hold few atoms or in FP64, where the tile kernel's per-lane FP64 state spills; the
// general layout is the only one for small boxes and for boxes that change (NPT).  Instead of a
// fixed density threshold, the tuner times each usable layout on the systems themselves, grouped
// as rbmd_step batches them, and keeps the fastest for the group.  Decisions are cached by a
// signature of the group, so systems admitted later (the serving loop) take them without timing.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.h"

namespace rbmd {

std::vector<int> Context::usable_layouts(const System* s) const {
  const SysDev& D = s->dev;
  if (D.npt) return {RBMD_LAYOUT_GENERAL};
  std::vector<int> out;
  if (column_layout_ok(D)) out.push_back(RBMD_LAYOUT_COLUMN);
  if (tile_layout_ok(D) && D.n < (1 << 25)) out.push_back(RBMD_LAYOUT_TILE);
  if (lean_layout_ok(D)) out.push_back(RBMD_LAYOUT_LEAN);
  out.push_back(RBMD_LAYOUT_GENERAL);
  return out;
}

void Context::set_layout(System* s, int layout) {
  SysDev& D = s->dev;
  const int dense = layout == RBMD_LAYOUT_COLUMN ? 2 : (layout == RBMD_LAYOUT_TILE ? 1 : 0);
  const int lean = (layout != RBMD_LAYOUT_GENERAL && lean_layout_ok(D)) ? 1 : 0;
  if (D.dense == dense && D.lean == lean) return;
  drop_batches_with(s->id);  // cached work tables and graphs hold the old layout
  D.dense = dense;
  D.lean = lean;
  D.blocks_pair = dense ? tile_blocks(D) : (D.n + kPairWarps - 1) / kPairWarps;
  upload_record(s);
}

namespace {
int64_t log2_bin(double x) { return (int64_t)std::floor(std::log2(std::max(x, 1e-9))); }
}  // namespace

int Context::autotune(const int32_t* ids, int n, rbmd_tune_result* out, int cap, int* n_groups, bool keep_forces) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  if (!ids || n <= 0) return fail(RBMD_ERR_ARG, "autotune: no systems");
  // explicit calls cover every listed system; the implicit call of rbmd_init / rbmd_step only the
  // systems not tuned yet
  const bool only_untuned = out == nullptr;
  std::vector<System*> sys;
  for (int k = 0; k < n; ++k) {
    System* s = find(ids[k]);
    if (!s) return fail(RBMD_ERR_STATE, "unknown system id " + std::to_string(ids[k]));
    if (only_untuned && s->tuned) continue;
    if (std::find(sys.begin(), sys.end(), s) == sys.end()) sys.push_back(s);
  }
  std::vector<std::vector<System*>> groups;
  for (System* s : sys) {
    bool placed = false;
    if (cfg.batched)
      for (auto& g : groups)
        if (same_group(g[0], s, false)) {
          g.push_back(s);
          placed = true;
          break;
        }
    if (!placed) groups.push_back({s});
  }
  int ng = 0;
  for (auto& g : groups) {
    rbmd_tune_result r;
    std::memset(&r, 0, sizeof(r));
    for (double& m : r.ms) m = -1.0;
    r.n_systems = (int32_t)g.size();
    double cells = 0.0;
    for (System* s : g) {
      r.atoms += s->dev.n;
      cells += s->dev.ncell;
    }
    // layouts every system of the group can use
    std::vector<int> use = usable_layouts(g[0]);
    for (System* s : g) {
      const std::vector<int> u = usable_layouts(s);
      use.erase(std::remove_if(use.begin(), use.end(),
                               [&](int l) { return std::find(u.begin(), u.end(), l) == u.end(); }),
                use.end());
    }
    const SysDev& D0 = g[0]->dev;
    const std::vector<int64_t> sig = {D0.ff, D0.neigh, D0.coul, D0.prec, D0.special, (D0.n_bonds + D0.n_angles + D0.n_dihedrals) > 0,
                                      D0.has_triples, D0.npt, log2_bin((double)r.atoms / cells), log2_bin((double)r.atoms)};
    int best = use.size() == 1 ? use[0] : -1;
    auto hit = tune_cache_.find(sig);
    if (best < 0 && hit != tune_cache_.end() && std::find(use.begin(), use.end(), hit->second) != use.end()) {
      best = hit->second;
      r.from_cache = 1;
    }
    if (best < 0) {
      // keep the forces of the last evaluation: the timed launches overwrite them
      void* fsave = nullptr;
      std::vector<size_t> off;
      if (keep_forces) {
        size_t tot = 0;
        for (System* s : g) {
          off.push_back(tot);
          tot += sizeof(double4) * (size_t)s->dev.n;
        }
        fsave = dmalloc(tot);
        if (!fsave) return fail(RBMD_ERR_OOM, "autotune: force scratch");
        for (size_t k = 0; k < g.size(); ++k)
          cudaMemcpyAsync((char*)fsave + off[k], g[k]->dev.f, sizeof(double4) * g[k]->dev.n,
                          cudaMemcpyDeviceToDevice, stream);
      }
      cudaEvent_t ea, eb;
      cudaEventCreate(&ea);
      cudaEventCreate(&eb);
      double best_ms = 0.0;
      int rc = RBMD_OK;
      for (int l : use) {
        for (System* s : g) set_layout(s, l);
        BatchRec* br = build_batch(g, rc);
        if (rc) {
          for (void* p : br->allocs) dfree(p);
          delete br;
          break;
        }
        launch_cells(br->b, stream);
        launch_pair(br->b, stream, 0);  // warm-up
        float t_min = 0.f;
        for (int rep = 0; rep < 3; ++rep) {
          cudaEventRecord(ea, stream);
          launch_pair(br->b, stream, 0);
          cudaEventRecord(eb, stream);
          cudaEventSynchronize(eb);
          float t = 0.f;
          cudaEventElapsedTime(&t, ea, eb);
          if (rep == 0 || t < t_min) t_min = t;
        }
        cudaStreamSynchronize(stream);
        for (void* p : br->allocs) dfree(p);
        delete br;
        r.ms[l] = t_min;
        if (best < 0 || t_min < best_ms) {
          best = l;
          best_ms = t_min;
        }
      }
      cudaEventDestroy(ea);
      cudaEventDestroy(eb);
      if (fsave) {
        for (size_t k = 0; k < g.size(); ++k)
          cudaMemcpyAsync(g[k]->dev.f, (char*)fsave + off[k], sizeof(double4) * g[k]->dev.n,
                          cudaMemcpyDeviceToDevice, stream);
        dfree(fsave);
        cudaStreamSynchronize(stream);
      }
      if (rc) return fail(rc, "autotune: work-table allocation failed");
      rc = check_cuda("autotune");
      if (rc) return rc;
      tune_cache_[sig] = best;
    }
    for (System* s : g) {
      set_layout(s, best);
      s->tuned = true;
    }
    r.layout = best;
    if (out && ng < cap) out[ng] = r;
    ++ng;
  }
  if (n_groups) *n_groups = ng;
  return RBMD_OK;
}

}  // namespace rbmd
