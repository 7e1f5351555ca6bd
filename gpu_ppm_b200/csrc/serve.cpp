// Serving: continuous batching of profile requests (ppm_submit / ppm_poll /
// ppm_wait).  The reference has no serving path; its conceptual caller is a
// sampler's likelihood loop (README.md:6) calling calc_one_star once per
// proposal (gpu/devarshi24st_gpu.cu:432).
//
// A scheduler thread keeps up to cfg.n_streams batches in flight, one per
// stream.  Whenever a stream is free it admits the oldest waiting requests
// whose device working set fits in what remains of the memory budget, builds
// them into one batch with stream-ordered allocations and enqueues plan ->
// integrand -> fold -> device-to-pinned copies; batches on different streams
// overlap on the device.  A host callback after the copies marks the batch
// finished; the scheduler then copies each request's results into its
// caller-owned buffers and completes the ticket with its submit-to-finish
// latency.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <list>
#include <memory>
#include <thread>
#include <unordered_map>

#include "engine.h"

namespace ppm {

using Clock = std::chrono::steady_clock;

namespace {
constexpr int kMaxRequestsPerBatch = 256;
}

struct Server {
  struct Request {
    uint64_t ticket;
    ppm_params p;
    double* flux;
    double* counts;
    long long n_flux, n_counts;
    size_t bytes;
    Clock::time_point t_submit;
  };
  struct Done {
    int status = PPM_OK;
    ppm_result_info info{};
    double latency_us = 0;
  };
  struct Slot {
    cudaStream_t stream = nullptr;
    HostBuffer pinned;  // device-to-host staging of the slot's current batch
    bool busy = false;
  };
  struct InFlight {
    std::vector<Request> reqs;
    std::unique_ptr<BatchImpl> B;
    int slot = 0;
    size_t bytes = 0;
    std::atomic<bool> finished{false};
    Clock::time_point t_done;
    Server* server = nullptr;
    int* ctrl = nullptr;                 // pinned copy of the queue control words
    unsigned long long* stats = nullptr; // pinned copy of the counters
    double* counts = nullptr;            // pinned copy of the counts pool
    double* flux = nullptr;              // pinned copy of the flux pool
  };

  Engine* eng = nullptr;
  std::mutex mu;
  std::condition_variable cv;       // wakes the scheduler
  std::condition_variable cv_done;  // wakes waiters
  std::deque<Request> pending;
  std::vector<Slot> slots;
  std::list<std::unique_ptr<InFlight>> inflight;
  std::unordered_map<uint64_t, Done> done;
  std::unordered_map<uint64_t, bool> known;
  size_t budget = 0, in_use = 0;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread thread;

  explicit Server(Engine* e) : eng(e) {
    budget = (size_t)e->cfg.memory_budget;
    slots.resize(e->cfg.n_streams);
    for (auto& s : slots) {
      cudaError_t err = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
      if (err != cudaSuccess) throw Error(PPM_E_CUDA, std::string("serving stream: ") + cudaGetErrorString(err));
    }
    // keep freed stream-ordered memory in the pool instead of returning it each time
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, e->cfg.device) == cudaSuccess) {
      uint64_t thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    thread = std::thread([this] { loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    if (thread.joinable()) thread.join();
    for (auto& s : slots) {
      if (s.stream) {
        cudaStreamSynchronize(s.stream);
        cudaStreamDestroy(s.stream);
      }
      s.pinned.release();
    }
  }

  static void CUDART_CB on_finished(void* arg) {
    InFlight* f = (InFlight*)arg;
    f->t_done = Clock::now();
    f->finished.store(true);
    {
      std::lock_guard<std::mutex> lk(f->server->mu);
    }
    f->server->cv.notify_all();
  }

  // Copies finished batches' results to their callers and completes the tickets.  Called with mu held.
  void retire() {
    for (auto it = inflight.begin(); it != inflight.end();) {
      InFlight& f = **it;
      if (!f.finished.load()) {
        ++it;
        continue;
      }
      const bool overflow = f.ctrl[2] || f.ctrl[5] || f.ctrl[8];
      const BatchImpl& B = *f.B;
      for (size_t i = 0; i < f.reqs.size(); ++i) {
        const Request& r = f.reqs[i];
        Done d;
        d.latency_us = std::chrono::duration<double, std::micro>(f.t_done - r.t_submit).count();
        if (overflow) {
          d.status = PPM_E_RANGE;
        } else {
          if (r.flux) std::memcpy(r.flux, f.flux + B.flux_off[i], sizeof(double) * (size_t)r.n_flux);
          if (r.counts && r.n_counts) std::memcpy(r.counts, f.counts + B.counts_off[i], sizeof(double) * (size_t)r.n_counts);
          const unsigned long long* s = f.stats + (size_t)kStats * i;
          d.info.n_active = (int64_t)(s[0] + s[5]);
          d.info.n_rings = (int64_t)s[1];
          d.info.n_dropped_rings = (int64_t)s[2];
          d.info.n_points = (int64_t)s[3];
          d.info.n_clamped = (int64_t)s[4];
          d.info.n_active_integrated = (int64_t)s[0];
        }
        d.info.status = d.status;
        done[r.ticket] = d;
      }
      slots[f.slot].busy = false;
      in_use -= f.bytes;
      // stream-ordered frees of the batch's device memory on its own stream
      cudaSetDevice(eng->cfg.device);
      it = inflight.erase(it);
      cv_done.notify_all();
    }
  }

  void fail(std::vector<Request>& reqs, int code) {
    for (auto& r : reqs) {
      Done d;
      d.status = code;
      d.info.status = code;
      d.latency_us = std::chrono::duration<double, std::micro>(Clock::now() - r.t_submit).count();
      done[r.ticket] = d;
    }
    cv_done.notify_all();
  }

  void loop() {
    cudaSetDevice(eng->cfg.device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      retire();
      if (stop && pending.empty() && inflight.empty()) break;
      int free_slot = -1;
      for (size_t k = 0; k < slots.size(); ++k)
        if (!slots[k].busy) {
          free_slot = (int)k;
          break;
        }
      if (pending.empty() || free_slot < 0) {
        cv.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      // admit the oldest requests that fit the remaining budget
      std::vector<Request> take;
      size_t bytes = 0;
      while (!pending.empty() && (int)take.size() < kMaxRequestsPerBatch &&
             in_use + bytes + pending.front().bytes <= budget) {
        bytes += pending.front().bytes;
        take.push_back(pending.front());
        pending.pop_front();
      }
      if (take.empty()) {  // waiting for memory to free up
        cv.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      Slot& slot = slots[free_slot];
      slot.busy = true;
      in_use += bytes;
      lk.unlock();
      std::unique_ptr<InFlight> f(new InFlight());
      f->server = this;
      f->slot = free_slot;
      f->bytes = bytes;
      f->reqs = std::move(take);
      int err = PPM_OK;
      try {
        launch(*f, slot);
      } catch (const Error& e) {
        err = e.code;
      }
      lk.lock();
      if (err != PPM_OK) {
        slot.busy = false;
        in_use -= bytes;
        fail(f->reqs, err);
        continue;
      }
      inflight.push_back(std::move(f));
    }
  }

  void launch(InFlight& f, Slot& slot) {
    const int n = (int)f.reqs.size();
    std::vector<ppm_params> ps(n);
    for (int i = 0; i < n; ++i) ps[i] = f.reqs[i].p;
    f.B.reset(new BatchImpl());
    BatchImpl& B = *f.B;
    B.mem.stream = slot.stream;
    {
      std::lock_guard<std::mutex> elk(eng->mu);
      eng->batch_build(B, n, ps.data(), slot.stream);
      eng->batch_enqueue(B, slot.stream, nullptr);
    }
    // device -> pinned staging
    const size_t n_counts = (size_t)B.counts_off[n], n_flux = (size_t)B.flux_off[n];
    bool want_flux = false;
    for (auto& r : f.reqs) want_flux |= r.flux != nullptr;
    const size_t bytes = 64 + sizeof(unsigned long long) * kStats * n + sizeof(double) * n_counts +
                         (want_flux ? sizeof(double) * n_flux : 0) + 256;
    slot.pinned.reserve(bytes);
    unsigned char* h = (unsigned char*)slot.pinned.ptr;
    f.ctrl = (int*)h;
    f.stats = (unsigned long long*)(h + 64);
    f.counts = (double*)(h + 64 + sizeof(unsigned long long) * kStats * n);
    f.flux = f.counts + n_counts;
    auto ck = [](cudaError_t e, const char* what) {
      if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    ck(cudaMemcpyAsync(f.ctrl, B.d_ctrl, sizeof(int) * 16, cudaMemcpyDeviceToHost, slot.stream), "serve copy");
    ck(cudaMemcpyAsync(f.stats, B.d_stats, sizeof(unsigned long long) * kStats * n, cudaMemcpyDeviceToHost, slot.stream),
       "serve copy");
    if (n_counts)
      ck(cudaMemcpyAsync(f.counts, B.d_counts, sizeof(double) * n_counts, cudaMemcpyDeviceToHost, slot.stream),
         "serve copy");
    if (want_flux)
      ck(cudaMemcpyAsync(f.flux, B.d_flux, sizeof(double) * n_flux, cudaMemcpyDeviceToHost, slot.stream), "serve copy");
    ck(cudaLaunchHostFunc(slot.stream, on_finished, &f), "serve callback");
  }
};

size_t Engine::request_bytes(const ppm_params& p) const {
  const size_t n_e = grids[p.energy_grid].E.size();
  size_t b = sizeof(double) * (size_t)p.n_bins * n_e;
  if (p.response >= 0) b += sizeof(double) * (size_t)resps[p.response].n_ch * p.n_bins;
  for (int s = 0; s < p.n_spots; ++s) {
    const long long rings = p.spots[s].kind == PPM_SPOT_POINT ? 1 : 4ll * p.n_side - 1;
    const size_t chunk = (size_t)std::min(tune.chunk, tune.small_chunk);  // the finest tiles a batch may use
    b += sizeof(Tile) * (size_t)rings * (2 + (4 * (size_t)p.n_side + chunk - 1) / chunk);
  }
  return b + sizeof(DevProfile) + sizeof(unsigned long long) * kStats + 4096;
}

// First-use tables are built here, in the submitting thread, so that the
// scheduler never allocates them mid-flight.
void Engine::warm_tables(const ppm_params& p) {
  ring_table(p.n_side);
  fine_table(p.n_fine);
  prepare_grid(p.energy_grid);
}

uint64_t Engine::submit(const ppm_params& p, double* flux, double* counts) {
  {
    std::lock_guard<std::mutex> lk(mu);
    validate(p);
    if (counts && p.response < 0) throw Error(PPM_E_INVALID, "counts requested without a response");
    cudaError_t e = cudaSetDevice(cfg.device);
    if (e != cudaSuccess) throw Error(PPM_E_CUDA, cudaGetErrorString(e));
    warm_tables(p);
    if (!server) server = new Server(this);
  }
  Server::Request r;
  r.p = p;
  r.flux = flux;
  r.counts = counts;
  r.n_flux = (long long)p.n_bins * (long long)grids[p.energy_grid].E.size();
  r.n_counts = p.response >= 0 ? (long long)resps[p.response].n_ch * p.n_bins : 0;
  r.bytes = request_bytes(p);
  if (r.bytes > server->budget) throw Error(PPM_E_OOM, "request larger than the serving memory budget");
  r.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(server->mu);
    r.ticket = server->next_ticket++;
    server->known[r.ticket] = true;
    server->pending.push_back(r);
  }
  server->cv.notify_all();
  return r.ticket;
}

int Engine::poll(uint64_t t) {
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::lock_guard<std::mutex> lk(server->mu);
  if (!server->known.count(t)) throw Error(PPM_E_INVALID, "unknown ticket");
  return server->done.count(t) ? 1 : 0;
}

int Engine::wait(uint64_t t, int timeout_ms, ppm_result_info* info) {
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::unique_lock<std::mutex> lk(server->mu);
  if (!server->known.count(t)) throw Error(PPM_E_INVALID, "unknown ticket");
  auto ready = [&] { return server->done.count(t) > 0; };
  if (timeout_ms < 0) {
    server->cv_done.wait(lk, ready);
  } else if (!server->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    throw Error(PPM_E_TIMEOUT, "ticket not finished within the timeout");
  }
  const Server::Done& d = server->done[t];
  if (info) *info = d.info;
  return d.status;
}

double Engine::latency_us(uint64_t t) {
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::lock_guard<std::mutex> lk(server->mu);
  auto it = server->done.find(t);
  if (it == server->done.end()) throw Error(PPM_E_STATE, "ticket not finished");
  return it->second.latency_us;
}

void Engine::serve_shutdown() {
  delete server;
  server = nullptr;
}

}  // namespace ppm
