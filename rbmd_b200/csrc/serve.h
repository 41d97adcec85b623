// serve.h -- continuous-batching serving loop over independent MD systems.
#pragma once

#include <atomic>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace rbmd {

// Deep copy of an rbmd_system_desc (the caller's arrays may be freed after submit).
struct OwnedDesc {
  rbmd_system_desc d{};
  std::vector<double> pos, vel, chg, mass, eps, sig, bk, br0, ak, at0, spw, frho, rhor, z2r, dk;
  std::vector<int32_t> type, mol, img, ba, bt, aa, at, spo, spi, da, dt, dsg, dm;
  std::vector<float> near;
  void copy_from(const rbmd_system_desc& src);
};

class Server {
 public:
  Server(Context* c, const rbmd_serve_cfg& cfg);
  ~Server();
  int start();
  int stop();
  int submit(const rbmd_system_desc& d, const rbmd_params& p, int nsteps, int64_t* rid);
  int poll(int64_t rid, int32_t* state);
  int wait(int64_t rid, double timeout_s);
  int result(int64_t rid, double* x, double* v, rbmd_thermo* th, rbmd_request_stats* stats);

 private:
  struct Request {
    int64_t id = 0;
    OwnedDesc desc;
    rbmd_params params{};
    int nsteps = 0;
    int remaining = 0;
    int64_t bytes = 0;
    int sys = -1;
    int state = RBMD_REQ_QUEUED;
    int status = RBMD_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::vector<double> x, v;
    rbmd_thermo thermo{};
  };
  void loop();
  void admit_locked(std::vector<Request*>& admitted);
  void finish(Request* r, int status);

  Context* ctx_;
  rbmd_serve_cfg cfg_;
  int64_t budget_ = 0;
  int64_t used_ = 0;
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::atomic<bool> stop_{false};
  bool running_ = false;
  std::deque<Request*> queue_;
  std::vector<Request*> active_;
  std::map<int64_t, std::unique_ptr<Request>> all_;
  int64_t next_id_ = 1;
  // seconds spent by the loop per phase (RBMD_SERVE_TRACE=1 prints them at stop): idle, add,
  // init, step, retire-state, retire-thermo, retire-remove; rounds, steps
  double phase_[7] = {0, 0, 0, 0, 0, 0, 0};
  int64_t rounds_ = 0, round_steps_ = 0;
};

double monotonic_seconds();

}  // namespace rbmd
