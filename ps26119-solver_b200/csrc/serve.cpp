// serve.cpp — the request loop (see serve.hpp).
#include "serve.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <utility>

namespace b200 {

double request_device_bytes(const Model& m) {
  const double nnz = static_cast<double>(m.nnz()), vec = static_cast<double>(m.num_rows) + m.num_cols;
  // per nonzero: the uploaded CSC (12 B), the engine's CSR of A and Aᵀ with original and scaled
  // values (40 B) and their fp32 copies (8 B); per row or column: about 35 fp64 vectors
  // (model, scaling, iterates, terms) and their fp32 copies; block-cache rounding and graphs
  return 1.25 * (60.0 * nnz + 280.0 * vec) + 32.0 * (1 << 20);
}

Server::Server(const ServerOptions& opt) : opt_(opt), t0_(std::chrono::steady_clock::now()) {
  if (opt_.slots <= 0) opt_.slots = 8;
  budget_ = opt_.hbm_budget_bytes;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) device = 0;
  if (budget_ <= 0.0) {
    std::size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget_ = 0.8 * static_cast<double>(free_b);
    (void)cudaGetLastError();
    if (budget_ <= 0.0) budget_ = 1e18;  // no device: the solves report it; admission by slots only
  }
  for (int k = 0; k < opt_.slots; ++k) slots_.emplace_back([this, device] { slot_main(device); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stopping_ = true;
  }
  work_cv_.notify_all();
  for (auto& t : slots_) t.join();
}

double Server::now() const {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

long long Server::submit(Model model, Options options) {
  auto r = std::make_unique<Request>();
  r->bytes = request_device_bytes(model);
  r->model = std::move(model);
  r->options = std::move(options);
  long long id;
  {
    std::lock_guard<std::mutex> lk(mu_);
    id = next_id_++;
    r->times.submitted = now();
    requests_.emplace(id, std::move(r));
    queue_.push_back(id);
  }
  work_cv_.notify_one();
  return id;
}

int Server::take(long long id, bool wait, Solution& out, RequestTimes& times) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) return -1;
  if (wait) done_cv_.wait(lk, [&] { return it->second->done; });
  if (!it->second->done) return 0;
  out = std::move(it->second->solution);
  times = it->second->times;
  requests_.erase(it);
  return 1;
}

void Server::slot_main(int device) {
  (void)cudaSetDevice(device);
  (void)cudaGetLastError();
  set_grouped_engine(opt_.grouped);  // this slot's solves run their epochs in the device's group
  std::unique_lock<std::mutex> lk(mu_);
  auto head_fits = [&] {
    if (queue_.empty()) return false;
    const Request& h = *requests_.at(queue_.front());
    return running_ == 0 || in_flight_bytes_ + h.bytes <= budget_;
  };
  for (;;) {
    work_cv_.wait(lk, [&] { return head_fits() || (stopping_ && queue_.empty()); });
    if (queue_.empty()) return;  // stopping, nothing left
    const long long id = queue_.front();
    queue_.pop_front();
    Request& r = *requests_.at(id);
    ++running_;
    in_flight_bytes_ += r.bytes;
    r.times.started = now();
    lk.unlock();
    work_cv_.notify_one();  // the next request may fit too
    Solution s;
    if (opt_.dry_run_seconds > 0.0) {
      std::this_thread::sleep_for(std::chrono::duration<double>(opt_.dry_run_seconds));
      s.status = Status::NotSolved;
      s.engine = "dry-run";
      s.message = "dry run: admitted and timed, not solved";
    } else {
      try {
        s = solve(r.model, r.options);
      } catch (const std::exception& e) {
        s = Solution{};
        s.status = Status::NumericalError;
        s.message = std::string("internal error: ") + e.what();
      }
    }
    lk.lock();
    r.solution = std::move(s);
    r.model = Model{};  // the host copy is no longer needed
    r.times.finished = now();
    r.done = true;
    --running_;
    in_flight_bytes_ -= r.bytes;
    done_cv_.notify_all();
    work_cv_.notify_all();
  }
}

}  // namespace b200
