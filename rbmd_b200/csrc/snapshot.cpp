// snapshot.cpp -- asynchronous state snapshots (rbmd_snapshot_begin / _poll / _wait).
//
// An output that reads the state with rbmd_get_state drains the context stream: every step queued
// so far must finish before the copy, and no step can be queued meanwhile.  A snapshot instead
// packs the state on the context stream (one small kernel, ordered after the queued steps), and a
// second stream copies the packed buffer to pinned host staging once the pack is done, so later
// steps run on the GPU while the copy crosses PCIe and the host writes the previous file.  The
// caller's destinations are filled when it waits for the ticket.  The reference's outputs read
// the fields synchronously (output/TrajectoryOutput.cpp:45-85).
#include <chrono>
#include <cstring>
#include <thread>

#include "engine.h"

namespace rbmd {

void* Context::pinned_get(size_t bytes, size_t* got) {
  size_t best = (size_t)-1;
  int at = -1;
  for (size_t k = 0; k < pinned_free_.size(); ++k)
    if (pinned_free_[k].first >= bytes && pinned_free_[k].first < best) {
      best = pinned_free_[k].first;
      at = (int)k;
    }
  if (at >= 0) {
    void* p = pinned_free_[at].second;
    *got = pinned_free_[at].first;
    pinned_free_.erase(pinned_free_.begin() + at);
    return p;
  }
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  *got = bytes;
  return p;
}

void Context::pinned_put(void* p, size_t bytes) {
  constexpr size_t kKeep = 8;  // staging blocks kept for reuse; larger ones replace smaller
  pinned_free_.emplace_back(bytes, p);
  if (pinned_free_.size() > kKeep) {
    size_t small = 0;
    for (size_t k = 1; k < pinned_free_.size(); ++k)
      if (pinned_free_[k].first < pinned_free_[small].first) small = k;
    cudaFreeHost(pinned_free_[small].second);
    pinned_free_.erase(pinned_free_.begin() + small);
  }
}

int Context::snapshot_begin(int id, double* x, double* v, int32_t* image, double* box, int64_t* step,
                            int64_t* ticket) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (!ticket) return fail(RBMD_ERR_ARG, "snapshot: null ticket");
  if (!copy_stream_ && cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking) != cudaSuccess) {
    copy_stream_ = nullptr;
    return check_cuda("snapshot stream");
  }
  Snap sn;
  sn.n = s->dev.n;
  sn.x = x;
  sn.v = v;
  sn.image = image;
  sn.box = box;
  sn.step = step;
  const size_t bytes = snapshot_bytes(sn.n);
  sn.dbuf = dmalloc(bytes);
  if (!sn.dbuf) return fail(RBMD_ERR_OOM, "snapshot device staging");
  sn.hbuf = pinned_get(bytes, &sn.bytes);
  if (!sn.hbuf) {
    dfree(sn.dbuf);
    return fail(RBMD_ERR_OOM, "snapshot pinned staging");
  }
  cudaEvent_t packed = nullptr;
  cudaEventCreateWithFlags(&packed, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&sn.done, cudaEventDisableTiming);
  launch_snapshot_pack(d_sys_, s->slot, sn.n, sn.dbuf, stream);
  cudaEventRecord(packed, stream);
  cudaStreamWaitEvent(copy_stream_, packed, 0);
  cudaMemcpyAsync(sn.hbuf, sn.dbuf, bytes, cudaMemcpyDeviceToHost, copy_stream_);
  cudaEventRecord(sn.done, copy_stream_);
  cudaEventDestroy(packed);  // released once the wait above has been satisfied
  const int rc = check_cuda("snapshot_begin");
  if (rc) {
    cudaStreamSynchronize(copy_stream_);
    cudaEventDestroy(sn.done);
    pinned_put(sn.hbuf, sn.bytes);
    dfree(sn.dbuf);
    return rc;
  }
  *ticket = next_ticket_++;
  snaps_[*ticket] = sn;
  return RBMD_OK;
}

// Copies a completed snapshot into its destinations and releases its staging.
void Context::snapshot_finish(int64_t ticket) {
  Snap& sn = snaps_[ticket];
  const char* h = (const char*)sn.hbuf;
  const size_t n3 = 3 * (size_t)sn.n;
  if (sn.step) {
    long long st;
    std::memcpy(&st, h, 8);
    *sn.step = st;
  }
  if (sn.box) std::memcpy(sn.box, h + 8, 6 * sizeof(double));
  if (sn.x) std::memcpy(sn.x, h + 56, n3 * sizeof(double));
  if (sn.v) std::memcpy(sn.v, h + 56 + n3 * sizeof(double), n3 * sizeof(double));
  if (sn.image) std::memcpy(sn.image, h + 56 + 2 * n3 * sizeof(double), n3 * sizeof(int32_t));
  pinned_put(sn.hbuf, sn.bytes);
  dfree(sn.dbuf);  // the copy has landed: stream-ordered release is safe
  cudaEventDestroy(sn.done);
  snaps_.erase(ticket);
}

int Context::snapshot_poll(int64_t ticket, int* done) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  auto it = snaps_.find(ticket);
  if (it == snaps_.end()) return fail(RBMD_ERR_STATE, "unknown snapshot ticket");
  const cudaError_t q = cudaEventQuery(it->second.done);
  if (q == cudaErrorNotReady) {
    *done = 0;
    return RBMD_OK;
  }
  if (q != cudaSuccess) return fail(RBMD_ERR_CUDA, std::string("snapshot: ") + cudaGetErrorString(q));
  *done = 1;
  return RBMD_OK;
}

int Context::snapshot_wait(int64_t ticket, double timeout_s) {
  cudaEvent_t ev = nullptr;
  {
    std::lock_guard<std::recursive_mutex> lk(mu);
    auto it = snaps_.find(ticket);
    if (it == snaps_.end()) return fail(RBMD_ERR_STATE, "unknown snapshot ticket");
    ev = it->second.done;
  }
  // poll without holding the context lock, so other threads keep queueing steps
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t q = cudaEventQuery(ev);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) {
      std::lock_guard<std::recursive_mutex> lk(mu);
      return fail(RBMD_ERR_CUDA, std::string("snapshot: ") + cudaGetErrorString(q));
    }
    if (timeout_s >= 0.0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s) {
      std::lock_guard<std::recursive_mutex> lk(mu);
      return fail(RBMD_ERR_TIMEOUT, "snapshot not complete within the timeout");
    }
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  std::lock_guard<std::recursive_mutex> lk(mu);
  if (snaps_.find(ticket) == snaps_.end()) return fail(RBMD_ERR_STATE, "snapshot ticket finished by another thread");
  snapshot_finish(ticket);
  return RBMD_OK;
}

// Context teardown: every pending snapshot is completed into nothing and its staging freed.
void Context::snapshots_release() {
  if (copy_stream_) cudaStreamSynchronize(copy_stream_);
  for (auto& kv : snaps_) {
    cudaEventDestroy(kv.second.done);
    dfree(kv.second.dbuf);
    cudaFreeHost(kv.second.hbuf);
  }
  snaps_.clear();
  for (auto& b : pinned_free_) cudaFreeHost(b.second);
  pinned_free_.clear();
  if (copy_stream_) cudaStreamDestroy(copy_stream_);
  copy_stream_ = nullptr;
}

}  // namespace rbmd
