// Serving loop: requests of different systems and frame counts arrive while
// others run.  Each request is cut into chunks of frames; worker threads
// (max_inflight of them) take chunks oldest request first, so at most one
// chunk of a request -- and of a system -- runs at a time, the device-memory
// budget admits a request's first chunk (footprint of its batch buffers), and
// work of several requests overlaps on the device.  A chunk runs on a stream
// whose priority is its request's age rank among the requests in flight (the
// oldest on the highest priority): the device hands freed SMs to the oldest
// request's blocks first, so a large request is not stretched by the small
// ones that fill the gaps, and at every chunk boundary the ranks are taken
// again.  Stream priorities cannot displace the blocks of a persistent kernel
// that is already resident, so the device work in flight is capped as well:
// a GB chunk of about a full chunk's pair evaluations fills the device, and
// chunks run beside it only while the work in flight stays under 1.5 full
// chunks; a request whose chunk does not fit holds back every younger one
// except tiny chunks (a tenth of a full one at most), so large requests run
// in arrival order at full speed while small ones overlap.  Per-request
// latency (submit -> results ready) is recorded.
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

// complex pair evaluations of a full GB chunk, the cap on those in flight,
// and the largest chunk that may pass an older request waiting for room
constexpr double kChunkWork = 2.5e9, kWorkCap = 1.5 * kChunkWork, kTinyWork = 0.1 * kChunkWork;

struct Request {
  int64_t id = 0;
  System* sys = nullptr;
  std::vector<float> frames;
  int64_t n_frames = 0;
  std::vector<rstg_frame_energy> out;
  int64_t bytes = 0;
  int64_t chunk = 1;     // frames per chunk
  double work_per_frame = 0.0;  // complex pair evaluations per frame (GB engine; 0: not capped)
  int64_t next = 0;      // first frame not yet dispatched
  int64_t done = 0;      // frames finished
  bool in_flight = false;
  bool admitted = false;  // its buffers are counted in the resident bytes
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
  std::deque<std::shared_ptr<Request>> queue;  // unfinished requests in submission order
  std::map<int64_t, std::shared_ptr<Request>> all;
  std::vector<std::thread> slots;
  std::vector<std::vector<cudaStream_t>> streams;  // [worker][priority level], level 0 the highest
  int prio_hi = 0, prio_lo = 0;
  std::map<System*, int> busy;  // systems with a chunk in flight
  // Device bytes each system holds between requests (its batch buffers stay
  // resident so that its next request reuses them and its captured graph);
  // idle systems are evicted, least recently used first, when an admission
  // needs the room.
  std::map<System*, int64_t> resident;
  std::map<System*, int64_t> last_use;
  int64_t use_clock = 0;
  int64_t resident_total = 0, peak_bytes = 0, next_id = 1, frames_done = 0;
  int running = 0;
  double inflight_work = 0.0;  // pair evaluations of the GB chunks in flight
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
    RSTG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));  // (least, greatest)
    int levels = std::min(n, prio_lo - prio_hi + 1);
    for (int k = 0; k < n; k++) {
      std::vector<cudaStream_t> per;
      for (int l = 0; l < levels; l++) per.push_back(take_stream(c->device, prio_hi + l));
      streams.push_back(per);
    }
    for (int k = 0; k < n; k++) slots.emplace_back([this, k] { slot_loop(k); });
  }

  // Streams come from a per-device, per-priority pool and are never
  // destroyed: a system that grew device buffers during a request frees them
  // later with cudaFreeAsync on the stream they were allocated on, which must
  // still exist then, whenever the system is destroyed.
  static std::mutex& pool_mu() {
    static std::mutex m;
    return m;
  }
  static std::map<std::pair<int, int>, std::vector<cudaStream_t>>& pool() {
    static auto* p = new std::map<std::pair<int, int>, std::vector<cudaStream_t>>();
    return *p;
  }
  static cudaStream_t take_stream(int device, int prio) {
    std::lock_guard<std::mutex> lk(pool_mu());
    std::vector<cudaStream_t>& free = pool()[{device, prio}];
    if (!free.empty()) {
      cudaStream_t s = free.back();
      free.pop_back();
      return s;
    }
    cudaStream_t s;
    RSTG_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio));
    return s;
  }
  void give_streams() {
    std::lock_guard<std::mutex> lk(pool_mu());
    for (auto& per : streams)
      for (size_t l = 0; l < per.size(); l++) pool()[{ctx->device, prio_hi + (int)l}].push_back(per[l]);
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    for (auto& t : slots) t.join();
    ctx->bind();
    for (auto& per : streams)
      for (auto st : per) cudaStreamSynchronize(st);
    give_streams();
  }

  // Frames per chunk: about 2.5e9 complex pair evaluations (some 20 ms of
  // device time whatever the system size) for the GB engine, 16 frames for
  // the batched PB engine (its lock-step cycles have a fixed cost per batch),
  // 8 frames in plain mode; opts.chunk_frames > 0 overrides.
  int64_t chunk_for(const System* sys, int64_t F) const {
    int64_t c;
    if (opts.chunk_frames > 0)
      c = opts.chunk_frames;
    else if (sys->opts.mode != RSTG_MODE_FUSED)
      c = 8;
    else if (sys->solv.method == 1)
      c = 16;
    else
      c = (int64_t)(kChunkWork / std::max(1.0, (double)sys->nC * (double)sys->nC));
    return std::max<int64_t>(1, std::min(c, std::max<int64_t>(F, 1)));
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
      if (kv.first != keep && !busy.count(kv.first)) {
        bool pending = false;  // a system with an admitted, unfinished request keeps its buffers
        for (auto& q : queue)
          if (q->sys == kv.first && q->admitted) pending = true;
        if (!pending) order.push_back({last_use[kv.first], kv.first});
      }
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

  double chunk_work(const Request& r) const {
    return r.work_per_frame * (double)std::min(r.chunk, r.n_frames - r.next);
  }

  // Next chunk to run: of the oldest request that has frames left, no chunk
  // in flight and an idle system, whose chunk keeps the work in flight under
  // kWorkCap (anything runs on an idle device); once an older request waits
  // for room, only tiny chunks may pass it.  A request's first chunk also
  // needs its buffers to fit the budget after evicting idle systems (a
  // request larger than the whole budget is admitted alone when nothing else
  // runs, so it cannot starve).
  std::shared_ptr<Request> pick() {
    bool held = false;  // an older request waits for the work in flight to drain
    for (auto& r : queue) {
      if (r->in_flight || r->next >= r->n_frames || r->state == Request::CANCELLED) continue;
      if (busy.count(r->sys)) continue;
      const double w = chunk_work(*r);
      if (running > 0 && inflight_work + w > kWorkCap) {
        held = true;
        continue;
      }
      if (held && w > kTinyWork) continue;
      if (!r->admitted) {
        int64_t need = growth(*r);
        evict_for(need, r->sys);
        if (!(resident_total + need <= opts.memory_budget_bytes || running == 0)) continue;
        resident[r->sys] += need;
        resident_total += need;
        peak_bytes = std::max(peak_bytes, resident_total);
        r->admitted = true;
      }
      return r;
    }
    return nullptr;
  }

  void finish(const std::shared_ptr<Request>& r) {  // with mu held
    r->finished = Clock::now();
    queue.erase(std::remove(queue.begin(), queue.end(), r), queue.end());
    r->frames.clear();
    r->frames.shrink_to_fit();
  }

  void slot_loop(int k) {
    cudaSetDevice(ctx->device);
    for (;;) {
      std::shared_ptr<Request> r;
      int64_t f0 = 0, B = 0;
      double work = 0.0;
      cudaStream_t st = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || (r = pick()) != nullptr; });
        if (!r) return;
        if (r->state == Request::QUEUED) r->state = Request::RUNNING;
        r->in_flight = true;
        busy[r->sys] = 1;
        last_use[r->sys] = ++use_clock;
        running++;
        work = chunk_work(*r);
        inflight_work += work;
        f0 = r->next;
        B = std::min(r->chunk, r->n_frames - f0);
        r->next += B;
        int rank = 0;  // requests older than r with a chunk in flight
        for (auto& q : queue) {
          if (q == r) break;
          if (q->in_flight) rank++;
        }
        st = streams[k][std::min<int>(rank, (int)streams[k].size() - 1)];
      }
      rstg_status code = RSTG_OK;
      std::string msg;
      try {
        std::lock_guard<std::recursive_mutex> sl(r->sys->mu);
        cudaStream_t prev = r->sys->stream_;
        if (r->sys->opts.mode == RSTG_MODE_FUSED) r->sys->stream_ = st;
        try {
          r->sys->run(r->frames.data() + (size_t)f0 * r->sys->n_top * 3, false, true, B, r->out.data() + f0, true,
                      nullptr);
        } catch (...) {
          r->sys->stream_ = prev;
          throw;
        }
        r->sys->stream_ = prev;
      } catch (const Error& e) {
        code = e.code;
        msg = e.what();
      } catch (const std::exception& e) {
        code = RSTG_ERR_INVALID;
        msg = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        busy.erase(r->sys);
        running--;
        inflight_work -= work;
        r->in_flight = false;
        r->done += B;
        if (r->state == Request::CANCELLED) {
          r->out.clear();
          finish(r);
        } else if (code != RSTG_OK) {
          r->state = Request::FAILED;
          r->err = code;
          r->msg = msg;
          finish(r);
        } else if (r->done == r->n_frames) {
          r->state = Request::DONE;
          finish(r);
          latencies_ms.push_back(std::chrono::duration<double, std::milli>(r->finished - r->submitted).count());
          frames_done += r->n_frames;
          last_done = r->finished;
        }
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
    r->chunk = chunk_for(sys, F);
    if (sys->opts.mode == RSTG_MODE_FUSED && sys->solv.method != 1)
      r->work_per_frame = (double)sys->nC * (double)sys->nC;
    r->bytes = sys->footprint(std::min<int64_t>(r->chunk, sys->batch > 0 ? sys->batch : r->chunk));
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
    all[r->id] = r;
    if (F == 0) {  // nothing to evaluate
      r->state = Request::DONE;
      r->finished = r->submitted;
      latencies_ms.push_back(0.0);
      cv_done.notify_all();
      return r->id;
    }
    queue.push_back(r);
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
    if (r->state == Request::QUEUED || r->state == Request::RUNNING) {
      r->state = Request::CANCELLED;  // no further chunk is dispatched
      if (!r->in_flight) {            // else the chunk's worker finishes it when the chunk ends
        r->out.clear();
        s->finish(r);
        s->cv_done.notify_all();
      }
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
