// Serving loop with continuous batching (rcwa_server_*, include/rcwa_b200.h).
//
// The reference has no server: main.cpp:111-191 solves one problem per call.
// Here a server owns `lanes` worker threads on one device, each with its own
// context (stream, workspace and the concurrent group workers of
// rcwa_solve_batch).  Callers queue requests (each with its own stack, source
// and port media) and poll for results.  Whenever a lane is free it admits
// queued requests and solves them as one batched solve on its stream, so
// requests that arrive while other batches run start as soon as a lane and
// device memory free up, and their work overlaps the batches already on the
// GPU.
//
// Admission is by device footprint: every request carries the bytes it
// occupies while solved (its share of the sweep plan and of the group's
// convolution matrices, problem_bytes), and a request is admitted only while
// the requests in flight on all lanes stay within the server's budget
// (default: 180 GB or 85 % of the free device memory, whichever is smaller).
// A lane fills its batch in arrival order up to its share of the budget
// (budget / lanes) and max_batch requests; a request that does not fit stays
// queued -- later, smaller requests may pass it -- and is admitted when
// memory frees.  A request larger than a lane's share is admitted alone once
// nothing else is in flight.  Each request's matrices and partial S-matrices
// live on the device for the duration of its batch; nothing is staged back
// to the host until its results.
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
  size_t bytes = 0;   // device footprint while solved
  int bypassed = 0;   // batches admitted past this request while it waited at the head
  std::vector<double> R, T;
  double R_tot = 0, T_tot = 0;
  uint32_t status = 0;
  int rc = 0;
  std::string err;   // the solver's message when rc is an error
  bool done = false;
  Clock::time_point t_submit, t_done;
};

// Latencies of the last kCap completed requests (a ring), for p50 / p99.
struct LatencyRing {
  static constexpr size_t kCap = 65536;
  std::vector<double> v;
  size_t next = 0;
  void add(double ms) {
    if (v.size() < kCap) {
      v.push_back(ms);
    } else {
      v[next] = ms;
      next = (next + 1) % kCap;
    }
  }
};

}  // namespace

struct rcwa_server {
  int device = 0;
  int max_batch = 0, max_queue = 0, precision = 0, nlanes = 0;
  unsigned mixed_stages = RCWA_MIXED_LAYER_GEMM | RCWA_MIXED_STAR_GEMM;
  int refine_sweeps = 1, gemm_digits = 5;
  size_t budget = 0;
  std::vector<rcwa_context*> ctx;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  size_t admitted = 0, peak_admitted = 0;
  uint64_t in_flight = 0, completed = 0, rejected = 0;
  LatencyRing lat;
};

namespace {

// Requests for one lane's next batch, taken from the queue (caller holds the
// lock).  Empty when nothing fits the budget right now.
std::vector<Request*> admit(rcwa_server* S) {
  constexpr int kMaxBypass = 8;   // then the head request waits for memory, nothing passes it
  std::vector<Request*> batch;
  const size_t share = std::max<size_t>(1, S->budget / (size_t)S->nlanes);
  size_t lane_bytes = 0;
  for (auto it = S->queue.begin(); it != S->queue.end() && (int)batch.size() < S->max_batch;) {
    Request* r = *it;
    const bool first = batch.empty();
    const bool global_ok = S->admitted + r->bytes <= S->budget;
    const bool lane_ok = lane_bytes + r->bytes <= share;
    const bool alone = first && S->admitted == 0;   // larger than the whole budget: runs alone
    if (((lane_ok || first) && global_ok) || alone) {
      batch.push_back(r);
      lane_bytes += r->bytes;
      S->admitted += r->bytes;
      it = S->queue.erase(it);
      if (!global_ok || !lane_ok) break;
    } else {
      if (it == S->queue.begin() && ++r->bypassed > kMaxBypass) break;
      ++it;
    }
  }
  S->in_flight += batch.size();
  S->peak_admitted = std::max(S->peak_admitted, S->admitted);
  return batch;
}

// Marks a request done and records its latency (caller holds the lock).
// Once done, a client may collect the request and free it at any time: the
// lane never touches it again (LaneBatch::fin).
void finish(rcwa_server* S, Request* r, const rcwa_result& o, int rc, const std::string& msg,
            Clock::time_point now) {
  r->R_tot = o.R_tot;
  r->T_tot = o.T_tot;
  r->status = o.status;
  if (rc == RCWA_OK || rc == RCWA_ERR_NUMERIC)
    r->rc = o.status ? RCWA_ERR_NUMERIC : RCWA_OK;
  else {
    r->rc = rc;
    r->err = msg;
  }
  r->done = true;
  r->t_done = now;
  S->lat.add(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
  S->admitted -= r->bytes;
  S->in_flight -= 1;
  S->completed += 1;
}

// A lane's batch while it is solved: the chunk callback of solve_batch
// completes its requests group by group.
struct LaneBatch {
  rcwa_server* S;
  const std::vector<Request*>* batch;
  const std::vector<rcwa_result>* out;
  std::vector<char>* fin;   // request i already finished (guarded by S->mu)
};

void chunk_done(void* user, const int* idx, int count) {
  LaneBatch* lb = static_cast<LaneBatch*>(user);
  const auto now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(lb->S->mu);
    for (int q = 0; q < count; ++q) {
      const int i = idx[q];
      if ((*lb->fin)[i]) continue;
      (*lb->fin)[i] = 1;
      finish(lb->S, (*lb->batch)[i], (*lb->out)[i], RCWA_OK, std::string(), now);
    }
  }
  lb->S->cv_done.notify_all();
  lb->S->cv_work.notify_all();   // freed memory may admit waiting requests on other lanes
}

void serve(rcwa_server* S, int lane) {
  cudaSetDevice(S->device);
  rcwa_context* ctx = S->ctx[lane];
  std::vector<Request*> batch;
  std::vector<rcwa_stack> st;
  std::vector<rcwa_source> src;
  std::vector<rcwa_params> par;
  std::vector<rcwa_result> out;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      for (;;) {
        if (S->queue.empty() && S->stop) return;
        if (!S->queue.empty()) {
          batch = admit(S);
          if (!batch.empty()) break;
        }
        S->cv_work.wait(lk);
      }
    }
    const int n = (int)batch.size();
    size_t bytes = 0;   // the batch's footprint: sizes its chunks
    st.resize(n);
    src.resize(n);
    par.resize(n);
    out.resize(n);
    for (int i = 0; i < n; ++i) {
      Request* r = batch[i];
      st[i] = r->st;
      src[i] = r->src;
      par[i] = r->par;
      bytes += r->bytes;
      const int N = (2 * r->par.nx_harmonics + 1) * (2 * r->par.ny_harmonics + 1);
      r->R.assign(N, 0.0);
      r->T.assign(N, 0.0);
      out[i] = rcwa_result{r->R.data(), r->T.data(), 0.0, 0.0, 0u};
    }
    // the batch's chunks are sized for what was admitted for it
    ctx->mem_budget = std::max<size_t>(bytes + (bytes >> 3), (size_t)1 << 28);
    std::vector<char> fin(n, 0);
    LaneBatch lb{S, &batch, &out, &fin};
    rcwa::ChunkSink sink;
    sink.fn = chunk_done;
    sink.user = &lb;
    const int rc = rcwa::solve_batch(ctx, n, st.data(), src.data(), par.data(), S->precision, S->max_batch,
                                     out.data(), &sink);
    const std::string msg = (rc == RCWA_OK || rc == RCWA_ERR_NUMERIC) ? std::string() : rcwa_last_error();
    const auto now = Clock::now();
    {
      // requests of chunks that did not complete carry the batch's error
      std::lock_guard<std::mutex> lk(S->mu);
      for (int i = 0; i < n; ++i)
        if (!fin[i]) {
          fin[i] = 1;
          finish(S, batch[i], out[i], rc == RCWA_OK ? RCWA_ERR_CUDA : rc, msg, now);
        }
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();
  }
}

double quantile(std::vector<double>& v, double f) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = f * (v.size() - 1);
  const size_t i = (size_t)pos;
  const double w = pos - i;
  return i + 1 < v.size() ? v[i] * (1 - w) + v[i + 1] * w : v[i];
}

}  // namespace

extern "C" {

int rcwa_server_create_ex(int device, const rcwa_server_config* cfg, rcwa_server** out) {
  if (!out || !cfg) {
    rcwa::set_last_error("NULL argument");
    return RCWA_ERR_INVALID;
  }
  *out = nullptr;
  if (cfg->max_batch <= 0 || cfg->max_queue <= 0 || cfg->lanes < 0 || cfg->lanes > 16) {
    rcwa::set_last_error("max_batch and max_queue must be positive, lanes 0..16");
    return RCWA_ERR_INVALID;
  }
  if (cfg->precision != RCWA_PREC_FP64 && cfg->precision != RCWA_PREC_MIXED) {
    rcwa::set_last_error("unknown precision mode %d", cfg->precision);
    return RCWA_ERR_INVALID;
  }
  rcwa_server* S = new (std::nothrow) rcwa_server();
  if (!S) return RCWA_ERR_NOMEM;
  S->device = device;
  S->max_batch = cfg->max_batch;
  S->max_queue = cfg->max_queue;
  S->precision = cfg->precision;
  S->nlanes = cfg->lanes ? cfg->lanes : 2;   // measured on the C3-type mix: 2 lanes of large batches serve most
  if (cfg->mixed_stages) S->mixed_stages = cfg->mixed_stages;
  if (cfg->refine_sweeps) S->refine_sweeps = cfg->refine_sweeps;
  if (cfg->gemm_digits) S->gemm_digits = cfg->gemm_digits;
  auto fail = [&](int rc) {
    for (rcwa_context* c : S->ctx) rcwa_context_destroy(c);
    delete S;
    return rc;
  };
  for (int l = 0; l < S->nlanes; ++l) {
    rcwa_context* c = nullptr;
    int rc = rcwa_context_create(device, &c);
    if (rc) return fail(rc);
    S->ctx.push_back(c);
    if ((rc = rcwa_context_set_mixed(c, S->mixed_stages, S->refine_sweeps, S->gemm_digits))) return fail(rc);
  }
  if (cfg->hbm_budget_bytes > 0) {
    S->budget = (size_t)cfg->hbm_budget_bytes;
  } else {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      rcwa::set_last_error("cudaMemGetInfo failed");
      return fail(RCWA_ERR_CUDA);
    }
    S->budget = std::min<size_t>((size_t)180 * 1000 * 1000 * 1000, (size_t)(0.85 * (double)fr));
  }
  try {
    for (int l = 0; l < S->nlanes; ++l) S->workers.emplace_back(serve, S, l);
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto& t : S->workers) t.join();
    rcwa::set_last_error("could not start the server threads");
    return fail(RCWA_ERR_CUDA);
  }
  *out = S;
  return RCWA_OK;
}

int rcwa_server_create(int device, int max_batch, int max_queue, int precision, rcwa_server** out) {
  rcwa_server_config cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.max_batch = max_batch;
  cfg.max_queue = max_queue;
  cfg.precision = precision;
  return rcwa_server_create_ex(device, &cfg, out);
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
  {
    std::lock_guard<std::mutex> lk(S->mu);   // fail fast before copying the grids
    if ((int)S->queue.size() >= S->max_queue) {
      ++S->rejected;
      rcwa::set_last_error("server queue full");
      return RCWA_ERR_BUSY;
    }
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
  r->bytes = rcwa::problem_bytes(r->st, r->par, S->precision, S->mixed_stages, S->refine_sweeps, S->gemm_digits);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if ((int)S->queue.size() >= S->max_queue) {
      ++S->rejected;
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

int rcwa_server_info_get(rcwa_server* S, rcwa_server_info* out) {
  if (!S || !out) {
    rcwa::set_last_error("NULL argument");
    return RCWA_ERR_INVALID;
  }
  std::vector<double> v;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    v = S->lat.v;
    out->completed = S->completed;
    out->queued = S->queue.size();
    out->in_flight = S->in_flight;
    out->rejected = S->rejected;
    out->admitted_bytes = S->admitted;
    out->peak_admitted_bytes = S->peak_admitted;
    out->budget_bytes = S->budget;
    out->lanes = S->nlanes;
  }
  out->p50_ms = quantile(v, 0.50);
  out->p99_ms = quantile(v, 0.99);
  return RCWA_OK;
}

int rcwa_server_stats(rcwa_server* S, uint64_t* completed, double* p50_ms, double* p99_ms) {
  rcwa_server_info info;
  const int rc = rcwa_server_info_get(S, &info);
  if (rc) return rc;
  if (completed) *completed = info.completed;
  if (p50_ms) *p50_ms = info.p50_ms;
  if (p99_ms) *p99_ms = info.p99_ms;
  return RCWA_OK;
}

int rcwa_server_destroy(rcwa_server* S) {
  if (!S) return RCWA_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers)
    if (t.joinable()) t.join();
  for (rcwa_context* c : S->ctx) rcwa_context_destroy(c);
  delete S;
  return RCWA_OK;
}

}  // extern "C"
