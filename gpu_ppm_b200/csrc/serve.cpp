// Serving: continuous batching of profile requests (ppm_submit / ppm_poll /
// ppm_wait).  The reference has no serving path; its conceptual caller is a
// sampler's likelihood loop (README.md:6) calling calc_one_star once per
// proposal (gpu/devarshi24st_gpu.cu:432).
//
// A scheduler thread keeps up to cfg.n_streams batches in flight, one per
// stream.  Whenever a stream is free it admits the oldest waiting requests
// whose device working set fits in what remains of the memory budget, builds
// them into one batch with stream-ordered allocations and enqueues plan ->
// integrand -> fold -> device-to-pinned copies into a staging buffer of its
// own (from a pool allocated when the server starts; a batch holds at most
// one buffer's worth of results); batches on different streams overlap on
// the device.  A host callback
// after the copies marks the batch finished; the scheduler then frees its
// stream and device memory at once and hands the staging buffer to a
// completion thread, which copies each request's results into its
// caller-owned buffers outside the lock and completes the tickets.  The
// scheduler thus never waits on those host copies (page faults of fresh
// caller buffers included) before it fills the freed stream again.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <thread>
#include <unordered_map>

#include "engine.h"

namespace ppm {

using Clock = std::chrono::steady_clock;

namespace {
constexpr int kMaxRequestsPerBatch = 256;
constexpr size_t kMaxCompleting = 4;  // finished batches whose results are still being copied out
constexpr size_t kTraceRecords = 4096;  // served batches kept for ppm_serve_trace

HostBuffer take(HostBuffer& b) {
  HostBuffer r = b;
  b.ptr = nullptr;
  b.cap = 0;
  return r;
}

// Pinned staging: a fixed pool of kStageBytes buffers allocated when the
// server starts, so that no pinned allocation (hundreds of ms for a few
// hundred MB) ever runs while requests wait; admission caps a batch by the
// bytes it stages, and only a single request larger than a buffer gets its own.
constexpr size_t kStageBytes = size_t(32) << 20;
constexpr size_t kStageFixed = 64 + 256;  // control words and slack around the per-request arrays
// a full batch's uploads (profiles, fold jobs, control words), each rounded up to 256 bytes
constexpr size_t kUploadBytes = kMaxRequestsPerBatch * (sizeof(DevProfile) + sizeof(FoldJob)) + 4 * 256;

size_t staged_bytes(size_t n, size_t counts, size_t flux, bool want_flux) {
  return kStageFixed + sizeof(unsigned long long) * kStats * n + sizeof(double) * (counts + (want_flux ? flux : 0));
}
}  // namespace

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
    bool busy = false;
    HostBuffer upload;  // pinned source of the batch build's uploads; reused once the slot's batch has finished
  };
  struct InFlight {
    std::vector<Request> reqs;
    std::unique_ptr<BatchImpl> B;      // device side; freed as soon as the batch finished
    std::vector<long long> flux_off, counts_off;
    HostBuffer stage;                  // device-to-host staging of this batch, from the pool
    int slot = 0;
    size_t bytes = 0;
    std::atomic<bool> finished{false};
    Server* server = nullptr;
    int* ctrl = nullptr;                 // pinned copy of the queue control words
    unsigned long long* stats = nullptr; // pinned copy of the counters
    double* counts = nullptr;            // pinned copy of the counts pool
    double* flux = nullptr;              // pinned copy of the flux pool
    bool want_flux = false;
    ppm_serve_batch_trace trace{};
  };

  Engine* eng = nullptr;
  std::mutex mu;
  std::condition_variable cv;          // wakes the scheduler
  std::condition_variable cv_complete; // wakes the completion thread
  std::condition_variable cv_done;     // wakes waiters
  std::deque<Request> pending;
  std::vector<Slot> slots;
  std::list<std::unique_ptr<InFlight>> inflight;
  std::deque<std::unique_ptr<InFlight>> completing;
  std::vector<HostBuffer> stage_pool;
  std::unordered_map<uint64_t, Done> done;
  std::unordered_map<uint64_t, bool> known;
  size_t budget = 0, in_use = 0;
  uint64_t next_ticket = 1;
  bool stop = false, scheduler_done = false;
  std::thread thread, completer;
  const Clock::time_point t_start = Clock::now();
  std::deque<ppm_serve_batch_trace> traces;  // the last kTraceRecords batches

  double since_start_us(Clock::time_point t) const {
    return std::chrono::duration<double, std::micro>(t - t_start).count();
  }

  explicit Server(Engine* e) : eng(e) {
    budget = (size_t)e->cfg.memory_budget;
    slots.resize(e->cfg.n_streams);
    try {
      for (auto& s : slots) {
        cudaError_t err = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
        if (err != cudaSuccess) throw Error(PPM_E_CUDA, std::string("serving stream: ") + cudaGetErrorString(err));
      }
      // enough buffers that one is always free at admission: at most n_streams - 1
      // in flight, kMaxCompleting - 1 queued and one being copied out
      stage_pool.resize(slots.size() + kMaxCompleting);
      for (auto& b : stage_pool) b.reserve(kStageBytes);
      for (auto& s : slots) s.upload.reserve(kUploadBytes);
    } catch (...) {  // the destructor does not run for a constructor that throws
      for (auto& b : stage_pool) b.release();
      for (auto& s : slots) {
        if (s.stream) cudaStreamDestroy(s.stream);
        s.upload.release();
      }
      throw;
    }
    // keep freed stream-ordered memory in the pool instead of returning it each time
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, e->cfg.device) == cudaSuccess) {
      uint64_t thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    thread = std::thread([this] { loop(); });
    completer = std::thread([this] { complete_loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    if (thread.joinable()) thread.join();
    {
      std::lock_guard<std::mutex> lk(mu);
      scheduler_done = true;
    }
    cv_complete.notify_all();
    if (completer.joinable()) completer.join();
    for (auto& s : slots) {
      if (s.stream) {
        cudaStreamSynchronize(s.stream);
        cudaStreamDestroy(s.stream);
      }
      s.upload.release();
    }
    for (auto& b : stage_pool) b.release();
  }

  static void CUDART_CB on_finished(void* arg) {
    InFlight* f = (InFlight*)arg;
    Server* s = f->server;  // f may be retired and destroyed as soon as it is marked finished
    f->trace.t_finished = s->since_start_us(Clock::now());
    f->finished.store(true);
    {
      std::lock_guard<std::mutex> lk(s->mu);
    }
    s->cv.notify_all();
  }

  // Frees the streams and device memory of finished batches and queues their
  // results for the completion thread.  Called with mu held.
  void retire() {
    for (auto it = inflight.begin(); it != inflight.end();) {
      InFlight& f = **it;
      if (!f.finished.load()) {
        ++it;
        continue;
      }
      f.flux_off = std::move(f.B->flux_off);
      f.counts_off = std::move(f.B->counts_off);
      // stream-ordered frees of the batch's device memory on its own stream
      cudaSetDevice(eng->cfg.device);
      f.B.reset();
      slots[f.slot].busy = false;
      in_use -= f.bytes;
      completing.push_back(std::move(*it));
      it = inflight.erase(it);
      cv_complete.notify_all();
    }
  }

  // Copies one finished batch's results into the callers' buffers (no lock held).
  static std::vector<std::pair<uint64_t, Done>> copy_out(const InFlight& f) {
    std::vector<std::pair<uint64_t, Done>> out(f.reqs.size());
    const bool overflow = f.ctrl[2] || f.ctrl[5] || f.ctrl[8] || f.ctrl[11] || f.ctrl[14];
    for (size_t i = 0; i < f.reqs.size(); ++i) {
      const Request& r = f.reqs[i];
      Done& d = out[i].second;
      out[i].first = r.ticket;
      if (overflow) {
        d.status = PPM_E_RANGE;
      } else {
        if (r.flux) std::memcpy(r.flux, f.flux + f.flux_off[i], sizeof(double) * (size_t)r.n_flux);
        if (r.counts && r.n_counts) std::memcpy(r.counts, f.counts + f.counts_off[i], sizeof(double) * (size_t)r.n_counts);
        const unsigned long long* s = f.stats + (size_t)kStats * i;
        d.info.n_active = (int64_t)(s[0] + s[5]);
        d.info.n_rings = (int64_t)s[1];
        d.info.n_dropped_rings = (int64_t)s[2];
        d.info.n_points = (int64_t)s[3];
        d.info.n_clamped = (int64_t)s[4];
        d.info.n_active_integrated = (int64_t)s[0];
      }
      d.info.status = d.status;
    }
    const Clock::time_point t = Clock::now();
    for (size_t i = 0; i < f.reqs.size(); ++i)
      out[i].second.latency_us = std::chrono::duration<double, std::micro>(t - f.reqs[i].t_submit).count();
    return out;
  }

  void complete_loop() {
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      cv_complete.wait(lk, [&] { return !completing.empty() || scheduler_done; });
      if (completing.empty()) break;  // scheduler_done and nothing left
      std::unique_ptr<InFlight> f = std::move(completing.front());
      completing.pop_front();
      lk.unlock();
      std::vector<std::pair<uint64_t, Done>> out;
      {
        NvtxRange range("serve batch: publish");
        out = copy_out(*f);
      }
      lk.lock();
      for (auto& kv : out) done[kv.first] = kv.second;
      f->trace.t_published = since_start_us(Clock::now());
      f->trace.staging_bytes = (int64_t)f->stage.cap;
      traces.push_back(f->trace);
      if (traces.size() > kTraceRecords) traces.pop_front();
      stage_pool.push_back(take(f->stage));
      cv_done.notify_all();
      cv.notify_all();  // the scheduler may be waiting for room in the completion queue
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
      if (pending.empty() || free_slot < 0 || completing.size() >= kMaxCompleting) {
        cv.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      // admit the oldest requests that fit the remaining budget and one staging buffer
      std::vector<Request> take_reqs;
      size_t bytes = 0, counts = 0, flux = 0;
      bool want_flux = false;
      while (!pending.empty() && (int)take_reqs.size() < kMaxRequestsPerBatch &&
             in_use + bytes + pending.front().bytes <= budget) {
        const Request& r = pending.front();
        const bool wf = want_flux || r.flux != nullptr;
        if (!take_reqs.empty() &&
            staged_bytes(take_reqs.size() + 1, counts + (size_t)r.n_counts, flux + (size_t)r.n_flux, wf) > kStageBytes)
          break;
        bytes += r.bytes;
        counts += (size_t)r.n_counts;
        flux += (size_t)r.n_flux;
        want_flux = wf;
        take_reqs.push_back(r);
        pending.pop_front();
      }
      if (take_reqs.empty()) {  // waiting for memory to free up
        cv.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      Slot& slot = slots[free_slot];
      slot.busy = true;
      in_use += bytes;
      std::unique_ptr<InFlight> f(new InFlight());
      f->server = this;
      f->slot = free_slot;
      f->bytes = bytes;
      f->reqs = std::move(take_reqs);
      f->trace.t_admit = since_start_us(Clock::now());
      f->trace.n_requests = (int32_t)f->reqs.size();
      f->trace.stream_slot = free_slot;
      if (!stage_pool.empty()) {
        f->stage = take(stage_pool.back());
        stage_pool.pop_back();
      }
      lk.unlock();
      int err = PPM_OK;
      try {
        launch(*f, slot);
      } catch (const Error& e) {
        err = e.code;
      }
      f->trace.t_launched = since_start_us(Clock::now());
      lk.lock();
      if (err != PPM_OK) {
        slot.busy = false;
        in_use -= bytes;
        stage_pool.push_back(take(f->stage));
        fail(f->reqs, err);
        continue;
      }
      inflight.push_back(std::move(f));
    }
  }

  void launch(InFlight& f, Slot& slot) {
    NvtxRange range("serve batch: build + enqueue");
    const int n = (int)f.reqs.size();
    std::vector<ppm_params> ps(n);
    for (int i = 0; i < n; ++i) ps[i] = f.reqs[i].p;
    f.B.reset(new BatchImpl());
    BatchImpl& B = *f.B;
    B.mem.stream = slot.stream;
    B.h_upload = slot.upload.ptr;
    B.h_upload_cap = slot.upload.cap;
    {
      std::lock_guard<std::mutex> elk(eng->mu);
      eng->batch_build(B, n, ps.data(), slot.stream);
      eng->batch_enqueue(B, slot.stream, nullptr);
    }
    // device -> pinned staging
    const size_t n_counts = (size_t)B.counts_off[n], n_flux = (size_t)B.flux_off[n];
    f.want_flux = false;
    for (auto& r : f.reqs) f.want_flux |= r.flux != nullptr;
    const size_t bytes = staged_bytes((size_t)n, n_counts, n_flux, f.want_flux);
    f.stage.reserve(std::max(bytes, kStageBytes));  // a no-op unless one request alone exceeds a pooled buffer
    unsigned char* h = (unsigned char*)f.stage.ptr;
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
    if (f.want_flux)
      ck(cudaMemcpyAsync(f.flux, B.d_flux, sizeof(double) * n_flux, cudaMemcpyDeviceToHost, slot.stream), "serve copy");
    ck(cudaLaunchHostFunc(slot.stream, on_finished, &f), "serve callback");
  }
};

size_t Engine::request_bytes(const ppm_params& p) const {
  const size_t n_e = grids[p.energy_grid].E.size();
  size_t b = 2 * sizeof(double) * (size_t)p.n_bins * n_e;  // flux and its compensation pool
  if (p.response >= 0) b += sizeof(double) * (size_t)resps[p.response].n_ch * p.n_bins;
  // work tiles: the larger of the finest element chunks (pooled kernel) and the tuned chunks with the most
  // phase-node splits (home-cell and blackbody kernels)
  const size_t nodes = (size_t)p.n_bins * std::max(1, p.n_gl);
  const size_t splits = std::max<size_t>(1, nodes / kMinNodesPerTile);
  for (int s = 0; s < p.n_spots; ++s) {
    const long long rings = p.spots[s].kind == PPM_SPOT_POINT ? 1 : 4ll * p.n_side - 1;
    const size_t fine = (size_t)std::min(tune.chunk, tune.small_chunk);
    const size_t by_elements = (size_t)rings * (2 + (4 * (size_t)p.n_side + fine - 1) / fine);
    const size_t by_nodes = (size_t)rings * (2 + (4 * (size_t)p.n_side + tune.chunk - 1) / tune.chunk) * splits;
    b += sizeof(Tile) * std::max(by_elements, by_nodes);
  }
  b += sizeof(unsigned) * kMaxSpots * (4 * (size_t)p.n_side / 32 + 1);  // ring bits
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
  const Clock::time_point t_entry = Clock::now();  // latency counts any wait for the engine lock
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
  r.t_submit = t_entry;
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

void Engine::release_ticket(uint64_t t) {
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::lock_guard<std::mutex> lk(server->mu);
  if (!server->known.count(t)) throw Error(PPM_E_INVALID, "unknown ticket");
  if (!server->done.count(t)) throw Error(PPM_E_STATE, "ticket not finished");
  server->done.erase(t);
  server->known.erase(t);
}

int Engine::serve_trace(ppm_serve_batch_trace* out, int cap) {
  if (!server) return 0;
  std::lock_guard<std::mutex> lk(server->mu);
  const int avail = (int)server->traces.size();
  const int n = std::min(cap, avail);
  for (int i = 0; i < n; ++i) out[i] = server->traces[(size_t)(avail - n + i)];
  return n;
}

void Engine::serve_shutdown() {
  delete server;
  server = nullptr;
}

}  // namespace ppm
