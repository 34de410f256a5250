// serve.hpp — a request loop for independent LPs on one GPU (continuous batching).
//
// Requests are queued in arrival order. A request is admitted when a slot is free and the
// device memory it will need fits in what the requests already running leave of the budget (the
// first request in flight is always admitted, so an oversized request runs alone rather than
// blocking the queue forever). Each slot is a host thread that runs the full dispatcher
// (solve(): presolve, the GPU engine on the slot's own stream, postsolve, the gate), so requests
// that arrive while others run start as soon as a slot and memory free up, and their kernels
// overlap on the device. Every request records when it was submitted, started and finished
// (seconds on the server's steady clock) for latency percentiles.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "solver.hpp"

namespace b200 {

struct ServerOptions {
  int slots = 8;                  // requests solved at the same time (host threads, one stream each)
  double hbm_budget_bytes = 0.0;  // device memory the running requests may hold; 0 = 80% of free memory
  double dry_run_seconds = 0.0;   // > 0: requests are admitted and timed but not solved; each holds
                                  // its slot and memory estimate this long (load tests of the policy)
  bool grouped = true;            // the running requests' iteration kernels launched together (one
                                  // grouped launch per half-step, engine.cu GroupScheduler)
};

struct RequestTimes {
  double submitted = 0.0, started = 0.0, finished = 0.0;  // seconds since the server was created
};

// Device bytes a solve of this model holds at its peak: the uploaded model, the engine's CSR
// copies of Ã and Ãᵀ (fp64 and fp32), the iterate and term vectors, and a fixed reserve.
double request_device_bytes(const Model& m);

class Server {
 public:
  explicit Server(const ServerOptions& opt);
  ~Server();  // finishes every request already submitted, then joins the slots
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  // Queues a solve; returns its id (≥ 0).
  long long submit(Model model, Options options);
  // When request `id` has finished (waiting for it if `wait`), moves its solution and times out,
  // forgets the request and returns 1; returns 0 while it is pending, -1 for an unknown id.
  int take(long long id, bool wait, Solution& out, RequestTimes& times);

  double budget_bytes() const { return budget_; }
  double now() const;  // seconds since creation

 private:
  struct Request {
    Model model;
    Options options;
    double bytes = 0.0;
    RequestTimes times;
    Solution solution;
    bool done = false;
  };
  void slot_main(int device);

  ServerOptions opt_;
  double budget_ = 0.0;
  std::chrono::steady_clock::time_point t0_;
  std::mutex mu_;
  std::condition_variable work_cv_, done_cv_;
  std::deque<long long> queue_;
  std::map<long long, std::unique_ptr<Request>> requests_;
  long long next_id_ = 0;
  double in_flight_bytes_ = 0.0;
  int running_ = 0;
  bool stopping_ = false;
  std::vector<std::thread> slots_;
};

}  // namespace b200
