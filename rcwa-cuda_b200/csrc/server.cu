// Serving loop with continuous batching (rcwa_server_*, include/rcwa_b200.h).
//
// The reference has no server: main.cpp:111-191 solves one problem per call.
// Here one worker thread per server owns a context on its device.  Callers
// queue requests (each with its own stack, source and port media) and poll
// for results; every iteration of the worker takes all requests queued at
// that moment (up to max_batch) and solves them as one rcwa_solve_batch
// call, so requests that arrive while a batch runs join the next one.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "solver.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  std::vector<rcwa_complex> er, ur;
  std::vector<double> t;
  rcwa_stack st{};
  rcwa_source src{};
  rcwa_params par{};
  std::vector<double> R, T;
  double R_tot = 0, T_tot = 0;
  uint32_t status = 0;
  int rc = 0;
  std::string err;   // the solver's message when rc is an error
  bool done = false;
  Clock::time_point t_submit, t_done;
};

}  // namespace

struct rcwa_server {
  int device = 0;
  int max_batch = 0, max_queue = 0, precision = 0;
  rcwa_context* ctx = nullptr;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  std::vector<double> lat_ms;
};

namespace {

void serve(rcwa_server* S) {
  cudaSetDevice(S->device);
  std::vector<Request*> batch;
  std::vector<rcwa_stack> st;
  std::vector<rcwa_source> src;
  std::vector<rcwa_params> par;
  std::vector<rcwa_result> out;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
      if (S->queue.empty() && S->stop) return;
      batch.clear();
      while (!S->queue.empty() && (int)batch.size() < S->max_batch) {
        batch.push_back(S->queue.front());
        S->queue.pop_front();
      }
    }
    const int n = (int)batch.size();
    st.resize(n);
    src.resize(n);
    par.resize(n);
    out.resize(n);
    for (int i = 0; i < n; ++i) {
      Request* r = batch[i];
      st[i] = r->st;
      src[i] = r->src;
      par[i] = r->par;
      const int N = (2 * r->par.nx_harmonics + 1) * (2 * r->par.ny_harmonics + 1);
      r->R.assign(N, 0.0);
      r->T.assign(N, 0.0);
      out[i] = rcwa_result{r->R.data(), r->T.data(), 0.0, 0.0, 0u};
    }
    const int rc = rcwa::solve_batch(S->ctx, n, st.data(), src.data(), par.data(), S->precision,
                                     S->max_batch, out.data());
    const std::string msg = (rc == RCWA_OK || rc == RCWA_ERR_NUMERIC) ? std::string() : rcwa_last_error();
    const auto now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (int i = 0; i < n; ++i) {
        Request* r = batch[i];
        r->R_tot = out[i].R_tot;
        r->T_tot = out[i].T_tot;
        r->status = out[i].status;
        if (rc == RCWA_OK || rc == RCWA_ERR_NUMERIC)
          r->rc = out[i].status ? RCWA_ERR_NUMERIC : RCWA_OK;
        else {
          r->rc = rc;
          r->err = msg;
        }
        r->done = true;
        r->t_done = now;
        S->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
      }
    }
    S->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int rcwa_server_create(int device, int max_batch, int max_queue, int precision, rcwa_server** out) {
  if (!out) {
    rcwa::set_last_error("out is NULL");
    return RCWA_ERR_INVALID;
  }
  *out = nullptr;
  if (max_batch <= 0 || max_queue <= 0) {
    rcwa::set_last_error("max_batch and max_queue must be positive");
    return RCWA_ERR_INVALID;
  }
  if (precision != RCWA_PREC_FP64 && precision != RCWA_PREC_MIXED) {
    rcwa::set_last_error("unknown precision mode %d", precision);
    return RCWA_ERR_INVALID;
  }
  rcwa_server* S = new (std::nothrow) rcwa_server();
  if (!S) return RCWA_ERR_NOMEM;
  S->device = device;
  S->max_batch = max_batch;
  S->max_queue = max_queue;
  S->precision = precision;
  int rc = rcwa_context_create(device, &S->ctx);
  if (rc) {
    delete S;
    return rc;
  }
  try {
    S->worker = std::thread(serve, S);
  } catch (...) {
    rcwa_context_destroy(S->ctx);
    delete S;
    rcwa::set_last_error("could not start the server thread");
    return RCWA_ERR_CUDA;
  }
  *out = S;
  return RCWA_OK;
}

int rcwa_server_submit(rcwa_server* S, const rcwa_stack* stack, const rcwa_source* source,
                       const rcwa_params* params, uint64_t* ticket) {
  if (!S || !stack || !source || !params || !ticket) {
    rcwa::set_last_error("NULL argument");
    return RCWA_ERR_INVALID;
  }
  if (stack->nx <= 0 || stack->ny <= 0 || stack->num_layers < 0 || stack->lx <= 0 || stack->ly <= 0 ||
      (stack->num_layers > 0 && (!stack->er || !stack->ur || !stack->t))) {
    rcwa::set_last_error("bad stack");
    return RCWA_ERR_INVALID;
  }
  if (params->nx_harmonics < 0 || params->ny_harmonics < 0 ||
      (2 * params->nx_harmonics + 1) * (2 * params->ny_harmonics + 1) > 4096) {
    rcwa::set_last_error("bad harmonic orders");
    return RCWA_ERR_INVALID;
  }
  auto r = std::make_unique<Request>();
  const size_t G = (size_t)stack->nx * stack->ny * stack->num_layers;
  r->er.assign(stack->er, stack->er + G);
  r->ur.assign(stack->ur, stack->ur + G);
  r->t.assign(stack->t, stack->t + stack->num_layers);
  r->st = *stack;
  r->st.er = r->er.data();
  r->st.ur = r->ur.data();
  r->st.t = r->t.data();
  r->src = *source;
  r->par = *params;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if ((int)S->queue.size() >= S->max_queue) {
      rcwa::set_last_error("server queue full");
      return RCWA_ERR_BUSY;
    }
    r->id = S->next_id++;
    *ticket = r->id;
    S->queue.push_back(r.get());
    S->reqs.emplace(r->id, std::move(r));
  }
  S->cv_work.notify_one();
  return RCWA_OK;
}

int rcwa_server_poll(rcwa_server* S, uint64_t ticket, int wait, rcwa_result* out, int* done) {
  if (!S || !done) {
    rcwa::set_last_error("NULL argument");
    return RCWA_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) {
    rcwa::set_last_error("unknown or already collected ticket");
    return RCWA_ERR_NOTFOUND;
  }
  Request* r = it->second.get();
  if (wait) S->cv_done.wait(lk, [&] { return r->done; });
  *done = r->done ? 1 : 0;
  if (!r->done) return RCWA_OK;
  if (out) {
    if (out->R) std::memcpy(out->R, r->R.data(), r->R.size() * sizeof(double));
    if (out->T) std::memcpy(out->T, r->T.data(), r->T.size() * sizeof(double));
    out->R_tot = r->R_tot;
    out->T_tot = r->T_tot;
    out->status = r->status;
  }
  const int rc = r->rc;
  if (rc && rc != RCWA_ERR_NUMERIC) rcwa::set_last_error("%s", r->err.c_str());
  S->reqs.erase(it);
  return rc;
}

int rcwa_server_stats(rcwa_server* S, uint64_t* completed, double* p50_ms, double* p99_ms) {
  if (!S) {
    rcwa::set_last_error("NULL argument");
    return RCWA_ERR_INVALID;
  }
  std::vector<double> v;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    v = S->lat_ms;
  }
  if (completed) *completed = v.size();
  double p50 = 0, p99 = 0;
  if (!v.empty()) {
    std::sort(v.begin(), v.end());
    auto q = [&](double f) {
      const double pos = f * (v.size() - 1);
      const size_t i = (size_t)pos;
      const double w = pos - i;
      return i + 1 < v.size() ? v[i] * (1 - w) + v[i + 1] * w : v[i];
    };
    p50 = q(0.50);
    p99 = q(0.99);
  }
  if (p50_ms) *p50_ms = p50;
  if (p99_ms) *p99_ms = p99;
  return RCWA_OK;
}

int rcwa_server_destroy(rcwa_server* S) {
  if (!S) return RCWA_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  rcwa_context_destroy(S->ctx);
  delete S;
  return RCWA_OK;
}

}  // extern "C"
