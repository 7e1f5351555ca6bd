// Serving entry points (submit / poll / wait).  Placeholder: synchronous execution per request.
#include <chrono>
#include <unordered_map>

#include "engine.h"

namespace ppm {

struct Server {
  struct Done {
    int status;
    ppm_result_info info;
    double latency_us;
  };
  std::mutex mu;
  uint64_t next = 1;
  std::unordered_map<uint64_t, Done> done;
};

uint64_t Engine::submit(const ppm_params& p, double* flux, double* counts) {
  if (!server) server = new Server();
  auto t0 = std::chrono::steady_clock::now();
  Server::Done d{};
  try {
    profile(p, flux, counts, &d.info);
    d.status = PPM_OK;
  } catch (const Error& e) {
    d.status = e.code;
  }
  d.latency_us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
  std::lock_guard<std::mutex> lk(server->mu);
  uint64_t t = server->next++;
  server->done[t] = d;
  return t;
}

int Engine::poll(uint64_t t) {
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::lock_guard<std::mutex> lk(server->mu);
  return server->done.count(t) ? 1 : 0;
}

int Engine::wait(uint64_t t, int timeout_ms, ppm_result_info* info) {
  (void)timeout_ms;
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::lock_guard<std::mutex> lk(server->mu);
  auto it = server->done.find(t);
  if (it == server->done.end()) throw Error(PPM_E_INVALID, "unknown ticket");
  if (info) *info = it->second.info;
  return it->second.status;
}

double Engine::latency_us(uint64_t t) {
  if (!server) throw Error(PPM_E_INVALID, "unknown ticket");
  std::lock_guard<std::mutex> lk(server->mu);
  auto it = server->done.find(t);
  if (it == server->done.end()) throw Error(PPM_E_INVALID, "unknown ticket");
  return it->second.latency_us;
}

void Engine::serve_shutdown() {
  delete server;
  server = nullptr;
}

}  // namespace ppm
