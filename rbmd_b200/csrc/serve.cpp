// serve.cpp -- continuous batching of independent MD systems on one GPU.
//
// Requests arrive at any time.  Between rounds of batched steps the loop admits queued requests
// in arrival order while the HBM budget and the slot limit allow, runs `steps_per_round` steps
// of the round's systems in one segment-indexed launch sequence (replayed as a CUDA graph while
// the set is unchanged), and retires systems whose step count is reached.  A round takes every
// active system, or with `round_atoms` > 0 the systems with the least remaining work (remaining
// steps x atoms) up to that many atoms: small requests then finish in a few rounds instead of
// waiting for the largest ones, and the rounds stay large enough to fill the GPU.  Positions,
// velocities and thermostat state stay resident on the device for the whole request.  Each
// system's arithmetic is independent of the others in the batch (per-system work tables and
// per-system fixed-order reductions), so a result is the same alone and in the mix.
#include "serve.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace rbmd {

double monotonic_seconds() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

template <class T>
static void cp(std::vector<T>& dst, const T* src, size_t n) {
  if (src && n) dst.assign(src, src + n);
  else dst.clear();
}

void OwnedDesc::copy_from(const rbmd_system_desc& s) {
  d = s;
  const size_t n = (size_t)s.n_atoms;
  cp(pos, s.position, 3 * n);
  cp(vel, s.velocity, 3 * n);
  cp(chg, s.charge, n);
  cp(mass, s.mass, n);
  cp(type, s.type, n);
  cp(mol, s.molecule, n);
  cp(img, s.image, 3 * n);
  cp(eps, s.epsilon, (size_t)s.n_types);
  cp(sig, s.sigma, (size_t)s.n_types);
  cp(ba, s.bond_atoms, 2 * (size_t)s.n_bonds);
  cp(bt, s.bond_type, (size_t)s.n_bonds);
  cp(bk, s.bond_k, (size_t)s.n_bond_types);
  cp(br0, s.bond_r0, (size_t)s.n_bond_types);
  cp(aa, s.angle_atoms, 3 * (size_t)s.n_angles);
  cp(at, s.angle_type, (size_t)s.n_angles);
  cp(ak, s.angle_k, (size_t)s.n_angle_types);
  cp(at0, s.angle_theta0, (size_t)s.n_angle_types);
  cp(spo, s.special_offsets, s.special_offsets ? n + 1 : 0);
  const size_t ns = s.special_offsets ? (size_t)s.special_offsets[n] : 0;
  cp(spi, s.special_ids, ns);
  cp(spw, s.special_weights, ns);
  size_t nf, nr, nz;
  eam_table_sizes(s, &nf, &nr, &nz);
  cp(frho, s.eam_frho_spline, s.eam_frho_spline ? nf : 0);
  cp(rhor, s.eam_rhor_spline, s.eam_rhor_spline ? nr : 0);
  cp(z2r, s.eam_z2r_spline, s.eam_z2r_spline ? nz : 0);
  cp(da, s.dihedral_atoms, 4 * (size_t)std::max(0, s.n_dihedrals));
  cp(dt, s.dihedral_type, (size_t)std::max(0, s.n_dihedrals));
  cp(dk, s.dihedral_k, (size_t)std::max(0, s.n_dihedral_types));
  cp(dsg, s.dihedral_sign, (size_t)std::max(0, s.n_dihedral_types));
  cp(dm, s.dihedral_multiplicity, (size_t)std::max(0, s.n_dihedral_types));
  cp(near, s.near_table_values, s.near_table_values ? (size_t)kNearKeys : 0);
  auto P = [](auto& v) { return v.empty() ? nullptr : v.data(); };
  d.position = P(pos);
  d.velocity = P(vel);
  d.charge = P(chg);
  d.mass = P(mass);
  d.type = P(type);
  d.molecule = P(mol);
  d.image = P(img);
  d.epsilon = P(eps);
  d.sigma = P(sig);
  d.bond_atoms = P(ba);
  d.bond_type = P(bt);
  d.bond_k = P(bk);
  d.bond_r0 = P(br0);
  d.angle_atoms = P(aa);
  d.angle_type = P(at);
  d.angle_k = P(ak);
  d.angle_theta0 = P(at0);
  d.special_offsets = P(spo);
  d.special_ids = P(spi);
  d.special_weights = P(spw);
  d.eam_frho_spline = P(frho);
  d.eam_rhor_spline = P(rhor);
  d.eam_z2r_spline = P(z2r);
  d.dihedral_atoms = P(da);
  d.dihedral_type = P(dt);
  d.dihedral_k = P(dk);
  d.dihedral_sign = P(dsg);
  d.dihedral_multiplicity = P(dm);
  d.near_table_values = P(near);
}

Server::Server(Context* c, const rbmd_serve_cfg& cfg) : ctx_(c), cfg_(cfg) {
  if (cfg_.steps_per_round <= 0) cfg_.steps_per_round = 10;
  budget_ = cfg_.hbm_budget_bytes > 0 ? cfg_.hbm_budget_bytes : c->cfg.hbm_budget_bytes;
  if (budget_ <= 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    budget_ = (int64_t)(fr * 0.85);
  }
}

Server::~Server() { stop(); }

int Server::start() {
  std::lock_guard<std::mutex> lk(mu_);
  if (running_) return RBMD_OK;
  stop_ = false;
  running_ = true;
  th_ = std::thread([this] { loop(); });
  return RBMD_OK;
}

int Server::stop() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (!running_) return RBMD_OK;
    stop_ = true;
  }
  cv_.notify_all();
  if (th_.joinable()) th_.join();
  std::lock_guard<std::mutex> lk(mu_);
  running_ = false;
  if (const char* tr = std::getenv("RBMD_SERVE_TRACE"))
    if (tr[0] == '1')
      std::fprintf(stderr,
                   "serve phases (s): idle %.3f add %.3f init %.3f step %.3f state %.3f thermo %.3f remove %.3f; "
                   "rounds %lld steps %lld\n",
                   phase_[0], phase_[1], phase_[2], phase_[3], phase_[4], phase_[5], phase_[6], (long long)rounds_,
                   (long long)round_steps_);
  // fail whatever is still queued or active
  for (Request* r : queue_) {
    r->state = RBMD_REQ_FAILED;
    r->status = RBMD_ERR_STATE;
  }
  queue_.clear();
  for (Request* r : active_) {
    if (r->sys >= 0) ctx_->remove_system(r->sys);
    r->state = RBMD_REQ_FAILED;
    r->status = RBMD_ERR_STATE;
  }
  active_.clear();
  done_cv_.notify_all();
  return RBMD_OK;
}

int Server::submit(const rbmd_system_desc& d, const rbmd_params& p, int nsteps, int64_t* rid) {
  if (d.n_atoms <= 0 || !d.position || !d.mass || !d.type) return ctx_->fail(RBMD_ERR_ARG, "incomplete system");
  auto r = std::make_unique<Request>();
  r->desc.copy_from(d);
  r->params = p;
  r->nsteps = r->remaining = nsteps;
  r->bytes = Context::estimate_bytes(d, p);
  r->t_submit = monotonic_seconds();
  std::lock_guard<std::mutex> lk(mu_);
  if (!running_) return ctx_->fail(RBMD_ERR_STATE, "serving loop not running");
  if (r->bytes > budget_) return ctx_->fail(RBMD_ERR_BUDGET, "request larger than the HBM budget");
  r->id = next_id_++;
  *rid = r->id;
  queue_.push_back(r.get());
  all_[r->id] = std::move(r);
  cv_.notify_all();
  return RBMD_OK;
}

int Server::poll(int64_t rid, int32_t* state) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = all_.find(rid);
  if (it == all_.end()) return ctx_->fail(RBMD_ERR_STATE, "unknown request");
  if (state) *state = it->second->state;
  return RBMD_OK;
}

int Server::wait(int64_t rid, double timeout_s) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = all_.find(rid);
  if (it == all_.end()) return ctx_->fail(RBMD_ERR_STATE, "unknown request");
  Request* r = it->second.get();
  auto pred = [&] { return r->state == RBMD_REQ_DONE || r->state == RBMD_REQ_FAILED; };
  if (timeout_s < 0) {
    done_cv_.wait(lk, pred);
  } else if (!done_cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
    return RBMD_ERR_TIMEOUT;
  }
  return r->state == RBMD_REQ_DONE ? RBMD_OK : r->status;
}

int Server::result(int64_t rid, double* x, double* v, rbmd_thermo* th, rbmd_request_stats* stats) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = all_.find(rid);
  if (it == all_.end()) return ctx_->fail(RBMD_ERR_STATE, "unknown request");
  Request* r = it->second.get();
  if (r->state != RBMD_REQ_DONE && r->state != RBMD_REQ_FAILED) return RBMD_ERR_STATE;
  const size_t n = (size_t)r->desc.d.n_atoms;
  if (x && r->x.size() == 3 * n) std::memcpy(x, r->x.data(), sizeof(double) * 3 * n);
  if (v && r->v.size() == 3 * n) std::memcpy(v, r->v.data(), sizeof(double) * 3 * n);
  if (th) *th = r->thermo;
  if (stats) {
    stats->t_submit = r->t_submit;
    stats->t_admit = r->t_admit;
    stats->t_done = r->t_done;
    stats->atom_steps = (int64_t)n * r->nsteps;
    stats->n_atoms = (int32_t)n;
    stats->status = r->status;
  }
  const int status = r->status;
  all_.erase(it);
  return status;
}

void Server::finish(Request* r, int status) {
  r->status = status;
  r->state = status == RBMD_OK ? RBMD_REQ_DONE : RBMD_REQ_FAILED;
  r->t_done = monotonic_seconds();
}

void Server::admit_locked(std::vector<Request*>& admitted) {
  while (!queue_.empty()) {
    Request* r = queue_.front();
    if (cfg_.max_systems > 0 && (int)active_.size() + (int)admitted.size() >= cfg_.max_systems) break;
    if (used_ + r->bytes > budget_) break;  // admission strictly in arrival order
    queue_.pop_front();
    used_ += r->bytes;
    admitted.push_back(r);
  }
}

void Server::loop() {
  double t_mark = monotonic_seconds();
  auto lap = [&](int phase) {
    const double t = monotonic_seconds();
    phase_[phase] += t - t_mark;
    t_mark = t;
  };
  while (!stop_) {
    std::vector<Request*> admitted;
    {
      std::unique_lock<std::mutex> lk(mu_);
      admit_locked(admitted);
      if (admitted.empty() && active_.empty()) {
        cv_.wait_for(lk, std::chrono::milliseconds(2), [&] { return stop_ || !queue_.empty(); });
        lap(0);
        continue;
      }
    }
    lap(0);
    // Keep the context's memory pool at twice the admitted footprint (capped by the budget), grown
    // by one allocation freed at once (the pool keeps freed memory): the systems' own allocations,
    // a few dozen each, then come from memory the pool holds.  Growing the pool allocation by
    // allocation took up to 0.1 s per large system and 1.8 s of the saline stream's 37 s.
    if (!admitted.empty() && ctx_->pooled()) {
      const int64_t want = std::min<int64_t>(budget_, 2 * used_), have = ctx_->pool_reserved();
      if (want > have) ctx_->dfree(ctx_->dmalloc((size_t)(want - have)));
    }
    // upload + Init of the admitted systems (outside the queue lock)
    std::vector<int32_t> new_ids;
    for (Request* r : admitted) {
      int32_t sid = -1;
      int rc = ctx_->add_system(r->desc.d, r->params, &sid);
      std::lock_guard<std::mutex> lk(mu_);
      if (rc) {
        used_ -= r->bytes;
        finish(r, rc);
        done_cv_.notify_all();
        continue;
      }
      r->sys = sid;
      r->state = RBMD_REQ_RUNNING;
      r->t_admit = monotonic_seconds();
      new_ids.push_back(sid);
    }
    lap(1);
    if (!new_ids.empty()) {
      int rc = ctx_->init(new_ids.data(), (int)new_ids.size());
      if (!rc) rc = ctx_->sync();
      lap(2);
      if (rc) {
        std::lock_guard<std::mutex> lk(mu_);
        for (Request* r : admitted)
          if (r->sys >= 0) {
            ctx_->remove_system(r->sys);
            used_ -= r->bytes;
            finish(r, rc);
          }
        done_cv_.notify_all();
        continue;
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (Request* r : admitted)
        if (r->state == RBMD_REQ_RUNNING) active_.push_back(r);
    }
    if (active_.empty()) continue;
    // one round of batched steps: every active system, or the least remaining work first up
    // to round_atoms atoms (at least one system)
    std::vector<Request*> stepping;
    for (Request* r : active_)
      if (r->remaining > 0) stepping.push_back(r);
    if (cfg_.round_atoms > 0 && !stepping.empty()) {
      std::stable_sort(stepping.begin(), stepping.end(), [](const Request* a, const Request* b) {
        const double wa = (double)a->remaining * a->desc.d.n_atoms, wb = (double)b->remaining * b->desc.d.n_atoms;
        return wa != wb ? wa < wb : a->id < b->id;
      });
      int64_t atoms = 0;
      size_t take = 0;
      while (take < stepping.size() && (take == 0 || atoms + stepping[take]->desc.d.n_atoms <= cfg_.round_atoms)) {
        atoms += stepping[take]->desc.d.n_atoms;
        ++take;
      }
      stepping.resize(take);
      std::sort(stepping.begin(), stepping.end(), [](const Request* a, const Request* b) { return a->id < b->id; });
    }
    int k = cfg_.steps_per_round;
    for (Request* r : stepping) k = std::min(k, r->remaining);
    std::vector<int32_t> ids;
    for (Request* r : stepping) ids.push_back(r->sys);
    int rc = RBMD_OK;
    if (!ids.empty() && k > 0) {
      rc = ctx_->step(ids.data(), (int)ids.size(), k);
      if (!rc) rc = ctx_->sync();
      for (Request* r : stepping) r->remaining -= k;
      ++rounds_;
      round_steps_ += k;
    }
    lap(3);
    // retire finished systems: each one's state, then one thermo evaluation for all of them
    std::vector<Request*> keep, retiring;
    for (Request* r : active_) {
      if (r->remaining > 0 && !rc) keep.push_back(r);
      else retiring.push_back(r);
    }
    std::vector<int> status(retiring.size(), rc);
    for (size_t q = 0; q < retiring.size(); ++q) {
      Request* r = retiring[q];
      const int n = r->desc.d.n_atoms;
      r->x.assign(3 * (size_t)n, 0.0);
      r->v.assign(3 * (size_t)n, 0.0);
      if (!status[q]) status[q] = ctx_->get_state(r->sys, r->x.data(), r->v.data(), nullptr);
    }
    lap(4);
    std::vector<int32_t> tids;
    std::vector<size_t> tq;
    for (size_t q = 0; q < retiring.size(); ++q)
      if (!status[q]) {
        tids.push_back(retiring[q]->sys);
        tq.push_back(q);
      }
    if (!tids.empty()) {
      std::vector<rbmd_thermo> th(tids.size());
      const int trc = ctx_->get_thermo_many(tids.data(), (int)tids.size(), th.data());
      for (size_t u = 0; u < tq.size(); ++u) {
        Request* r = retiring[tq[u]];
        if (trc) {
          status[tq[u]] = trc;
          continue;
        }
        r->thermo = th[u];
        if (r->thermo.status != 0) status[tq[u]] = RBMD_ERR_NUMERIC;
      }
    }
    lap(5);
    for (size_t q = 0; q < retiring.size(); ++q) {
      Request* r = retiring[q];
      ctx_->remove_system(r->sys);
      std::lock_guard<std::mutex> lk(mu_);
      used_ -= r->bytes;
      finish(r, status[q]);
    }
    lap(6);
    {
      std::lock_guard<std::mutex> lk(mu_);
      active_ = keep;
    }
    done_cv_.notify_all();
  }
}

}  // namespace rbmd
