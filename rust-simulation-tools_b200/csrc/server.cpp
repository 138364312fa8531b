// Serving loop: requests of different systems and frame counts arrive while
// others run; a dispatcher admits them into free slots when the device-memory
// budget allows (footprint of the request's batch buffers), each slot runs its
// request on its own CUDA stream so work of several requests overlaps on the
// device, and per-request latency (submit -> results ready) is recorded.
#include <algorithm>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "internal.hpp"
#include "system.hpp"

namespace rstg {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  System* sys = nullptr;
  std::vector<float> frames;
  int64_t n_frames = 0;
  std::vector<rstg_frame_energy> out;
  int64_t bytes = 0;
  Clock::time_point submitted, finished;
  enum State { QUEUED, RUNNING, DONE, FAILED, CANCELLED } state = QUEUED;
  rstg_status err = RSTG_OK;
  std::string msg;
};

struct Server {
  Ctx* ctx;
  rstg_server_opts opts;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<int64_t, std::shared_ptr<Request>> all;
  std::vector<std::thread> slots;
  std::vector<cudaStream_t> streams;
  std::map<System*, int> busy;  // systems with a running request
  // Device bytes each system holds between requests (its batch buffers stay
  // resident so that its next request reuses them and its captured graph);
  // idle systems are evicted, least recently used first, when an admission
  // needs the room.
  std::map<System*, int64_t> resident;
  std::map<System*, int64_t> last_use;
  int64_t use_clock = 0;
  int64_t resident_total = 0, peak_bytes = 0, next_id = 1, frames_done = 0;
  int running = 0;
  bool stop = false;
  int64_t device_bytes = 0;  // a request whose buffers exceed the device is refused at submit
  std::vector<double> latencies_ms;
  Clock::time_point first_submit, last_done;
  bool any = false;

  Server(Ctx* c, const rstg_server_opts& o) : ctx(c), opts(o) {
    int n = std::max(1, opts.max_inflight);
    c->bind();
    size_t fr = 0, tot = 0;
    RSTG_CUDA(cudaMemGetInfo(&fr, &tot));
    device_bytes = (int64_t)tot;
    streams = take_streams(c->device, n);
    for (int k = 0; k < n; k++) slots.emplace_back([this, k] { slot_loop(k); });
  }

  // Slot streams come from a per-device pool and are never destroyed: a
  // system that grew device buffers during a request frees them later with
  // cudaFreeAsync on the stream they were allocated on, which must still
  // exist then, whenever the system is destroyed.
  static std::mutex& pool_mu() {
    static std::mutex m;
    return m;
  }
  static std::map<int, std::vector<cudaStream_t>>& pool() {
    static auto* p = new std::map<int, std::vector<cudaStream_t>>();
    return *p;
  }
  static std::vector<cudaStream_t> take_streams(int device, int n) {
    std::lock_guard<std::mutex> lk(pool_mu());
    std::vector<cudaStream_t>& free = pool()[device];
    std::vector<cudaStream_t> out;
    while ((int)out.size() < n && !free.empty()) {
      out.push_back(free.back());
      free.pop_back();
    }
    while ((int)out.size() < n) {
      cudaStream_t s;
      RSTG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      out.push_back(s);
    }
    return out;
  }
  static void give_streams(int device, const std::vector<cudaStream_t>& s) {
    std::lock_guard<std::mutex> lk(pool_mu());
    auto& free = pool()[device];
    free.insert(free.end(), s.begin(), s.end());
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    for (auto& t : slots) t.join();
    ctx->bind();
    for (auto s : streams) cudaStreamSynchronize(s);
    give_streams(ctx->device, streams);
  }

  int64_t growth(const Request& r) {
    auto it = resident.find(r.sys);
    return std::max<int64_t>(0, r.bytes - (it == resident.end() ? 0 : it->second));
  }

  // Releases idle systems' buffers (least recently used first) until `need`
  // more bytes fit the budget.  A system whose lock is taken elsewhere, or a
  // plain-mode system (its evaluator's buffers are not released here), keeps
  // its bytes in the count and is passed over for the next candidate.
  void evict_for(int64_t need, System* keep) {
    std::vector<std::pair<int64_t, System*>> order;
    for (auto& kv : resident)
      if (kv.first != keep && !busy.count(kv.first)) order.push_back({last_use[kv.first], kv.first});
    std::sort(order.begin(), order.end());
    for (auto& o : order) {
      if (resident_total + need <= opts.memory_budget_bytes) return;
      System* victim = o.second;
      if (victim->opts.mode != RSTG_MODE_FUSED) continue;
      std::unique_lock<std::recursive_mutex> vl(victim->mu, std::try_to_lock);
      if (!vl.owns_lock()) continue;
      victim->release_buffers();
      resident_total -= resident[victim];
      resident.erase(victim);
    }
  }

  // Next admissible request: first in arrival order whose system is idle and
  // whose buffers fit the budget after evicting idle systems (a request
  // larger than the whole budget is admitted alone when nothing else runs,
  // so it cannot starve).
  std::shared_ptr<Request> pick() {
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      auto& r = *it;
      if (busy.count(r->sys)) continue;
      int64_t need = growth(*r);
      evict_for(need, r->sys);
      bool fits = resident_total + need <= opts.memory_budget_bytes || running == 0;
      if (!fits) continue;
      auto q = r;
      queue.erase(it);
      return q;
    }
    return nullptr;
  }

  void slot_loop(int k) {
    cudaSetDevice(ctx->device);
    for (;;) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || (r = pick()) != nullptr; });
        if (!r) return;
        r->state = Request::RUNNING;
        busy[r->sys] = 1;
        int64_t g = growth(*r);
        resident[r->sys] += g;
        resident_total += g;
        last_use[r->sys] = ++use_clock;
        peak_bytes = std::max(peak_bytes, resident_total);
        running++;
      }
      rstg_status st = RSTG_OK;
      std::string msg;
      try {
        std::lock_guard<std::recursive_mutex> sl(r->sys->mu);
        cudaStream_t prev = r->sys->stream_;
        if (r->sys->opts.mode == RSTG_MODE_FUSED) r->sys->stream_ = streams[k];
        try {
          r->sys->run(r->frames.data(), false, true, r->n_frames, r->out.data(), true, nullptr);
        } catch (...) {
          r->sys->stream_ = prev;
          throw;
        }
        r->sys->stream_ = prev;
      } catch (const Error& e) {
        st = e.code;
        msg = e.what();
      } catch (const std::exception& e) {
        st = RSTG_ERR_INVALID;
        msg = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        r->finished = Clock::now();
        busy.erase(r->sys);
        running--;
        if (r->state == Request::CANCELLED) {
          r->out.clear();
        } else if (st != RSTG_OK) {
          r->state = Request::FAILED;
          r->err = st;
          r->msg = msg;
        } else {
          r->state = Request::DONE;
          latencies_ms.push_back(std::chrono::duration<double, std::milli>(r->finished - r->submitted).count());
          frames_done += r->n_frames;
          last_done = r->finished;
        }
        r->frames.clear();
        r->frames.shrink_to_fit();
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  int64_t submit(System* sys, const float* frames, int64_t F) {
    auto r = std::make_shared<Request>();
    r->sys = sys;
    r->n_frames = F;
    r->frames.assign(frames, frames + (size_t)F * sys->n_top * 3);
    r->out.resize(F);
    r->bytes = sys->footprint(std::min<int64_t>(F, sys->batch > 0 ? sys->batch : F));
    if (r->bytes > device_bytes)
      throw Error(RSTG_ERR_NOMEM, "request needs " + std::to_string(r->bytes) + " bytes of device memory; the device has " +
                                      std::to_string(device_bytes));
    std::lock_guard<std::mutex> lk(mu);
    r->id = next_id++;
    r->submitted = Clock::now();
    if (!any) {
      first_submit = r->submitted;
      any = true;
    }
    queue.push_back(r);
    all[r->id] = r;
    cv_work.notify_all();
    return r->id;
  }

  std::shared_ptr<Request> find(int64_t id) {
    auto it = all.find(id);
    if (it == all.end()) throw Error(RSTG_ERR_INVALID, "unknown request id " + std::to_string(id));
    return it->second;
  }

  rstg_status collect(const std::shared_ptr<Request>& r, rstg_frame_energy* out) {
    if (r->state == Request::CANCELLED) {
      set_last_error("request " + std::to_string(r->id) + " was cancelled");
      return RSTG_ERR_CANCELLED;
    }
    if (r->state == Request::FAILED) {
      set_last_error(r->msg);
      return r->err;
    }
    if (r->state != Request::DONE) return RSTG_ERR_NOT_READY;
    if (out) memcpy(out, r->out.data(), r->out.size() * sizeof(rstg_frame_energy));
    return RSTG_OK;
  }
};

}  // namespace rstg

using namespace rstg;

struct rstg_server : Server {
  using Server::Server;
};

extern "C" {

void rstg_server_opts_default(rstg_server_opts* o) {
  o->memory_budget_bytes = (int64_t)16 << 30;
  o->max_inflight = 4;
  o->chunk_frames = 0;
}

rstg_status rstg_server_create(rstg_ctx* c, const rstg_server_opts* opts, rstg_server** out) {
  try {
    if (!c || !out) throw Error(RSTG_ERR_INVALID, "ctx and out must not be NULL");
    rstg_server_opts o;
    if (opts)
      o = *opts;
    else
      rstg_server_opts_default(&o);
    *out = new rstg_server(c, o);
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

void rstg_server_destroy(rstg_server* s) { delete s; }

rstg_status rstg_server_submit(rstg_server* s, rstg_system* sys, const float* frames, int64_t F, int64_t* id) {
  try {
    if (!s || !sys || !id || F < 0 || (F > 0 && !frames)) throw Error(RSTG_ERR_INVALID, "invalid submit arguments");
    *id = s->submit(sys, frames, F);
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return RSTG_ERR_NOMEM;
  }
}

rstg_status rstg_server_poll(rstg_server* s, int64_t id, rstg_frame_energy* out) {
  try {
    std::lock_guard<std::mutex> lk(s->mu);
    return s->collect(s->find(id), out);
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

rstg_status rstg_server_wait(rstg_server* s, int64_t id, int64_t timeout_ms, rstg_frame_energy* out) {
  try {
    std::unique_lock<std::mutex> lk(s->mu);
    auto r = s->find(id);
    auto done = [&] {
      return r->state == Request::DONE || r->state == Request::FAILED ||
             (r->state == Request::CANCELLED && r->finished != Clock::time_point());
    };
    if (timeout_ms < 0)
      s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
      set_last_error("request " + std::to_string(id) + " not finished within " + std::to_string(timeout_ms) + " ms");
      return RSTG_ERR_TIMEOUT;
    }
    return s->collect(r, out);
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

rstg_status rstg_server_cancel(rstg_server* s, int64_t id) {
  try {
    std::lock_guard<std::mutex> lk(s->mu);
    auto r = s->find(id);
    if (r->state == Request::QUEUED) {
      s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
      r->frames.clear();
      r->state = Request::CANCELLED;
      r->finished = Clock::now();
      s->cv_done.notify_all();
    } else if (r->state == Request::RUNNING) {
      r->state = Request::CANCELLED;  // results are discarded when the run ends
    }
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}

rstg_status rstg_server_stats(const rstg_server* cs, double* st) {
  rstg_server* s = const_cast<rstg_server*>(cs);
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> l = s->latencies_ms;
  std::sort(l.begin(), l.end());
  auto pct = [&](double p) {
    if (l.empty()) return 0.0;
    double k = p * (double)(l.size() - 1);
    size_t a = (size_t)k, b = std::min(a + 1, l.size() - 1);
    return l[a] + (k - (double)a) * (l[b] - l[a]);
  };
  double mean = 0.0;
  for (double v : l) mean += v;
  if (!l.empty()) mean /= (double)l.size();
  double wall = s->any && !l.empty() ? std::chrono::duration<double>(s->last_done - s->first_submit).count() : 0.0;
  double v[8] = {(double)l.size(), (double)s->frames_done, pct(0.5), pct(0.99), mean, (double)s->peak_bytes, wall,
                 wall > 0 ? (double)s->frames_done / wall : 0.0};
  memcpy(st, v, sizeof(v));
  return RSTG_OK;
}

}  // extern "C"
