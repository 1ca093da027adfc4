// Batches of unrelated problems: every solve brings its own stack, source and
// port media (the C3 workload: stacks of 1-6 patterned layers, periods,
// thicknesses and harmonic orders that differ from solve to solve).
//
// The reference solves such a list one problem at a time (main.cpp:111-191
// per problem).  Here problems of equal shape -- harmonic orders, number of
// layers, grid size, port media and which layers are uniform -- form a group
// that runs as ONE batched solve: the convolution matrices of all its stacks
// are built by one batched ConvMat and one batched LU, and the layer loop of
// sweep_chunk runs over the whole group with per-item matrices (Layers with
// s_item != 0), per-item thicknesses and per-item lattice periods.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "solver.cuh"

namespace rcwa {

namespace {

// host check: a grid is uniform when every cell equals the first one
bool grid_uniform(const rcwa_complex* g, size_t G) {
  const rcwa_complex v = g[0];
  for (size_t i = 1; i < G; ++i)
    if (g[i].re != v.re || g[i].im != v.im) return false;
  return true;
}

// Stacks without uniform layers group regardless of depth (flex = 1, nl = -1):
// they are sorted deepest first and layer l runs for the leading solves that
// have it.  Stacks with uniform layers group by exact depth and uniform mask.
struct GroupKey {
  int flex, nxh, nyh, nl, nx, ny;
  double p[8];                  // er_ref, ur_ref, er_trn, ur_trn (re, im)
  std::vector<char> uniform;
  bool operator<(const GroupKey& o) const {
    return std::tie(flex, nxh, nyh, nl, nx, ny, p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], uniform) <
           std::tie(o.flex, o.nxh, o.nyh, o.nl, o.nx, o.ny, o.p[0], o.p[1], o.p[2], o.p[3], o.p[4], o.p[5],
                    o.p[6], o.p[7], o.uniform);
  }
};

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// Concurrent group chunks per batch: RCWA_BATCH_STREAMS (read once), default 4.
int batch_streams() {
  static int k = -1;
  if (k < 0) {
    const char* e = getenv("RCWA_BATCH_STREAMS");
    k = e ? std::max(1, std::min(16, atoi(e))) : 4;
  }
  return k;
}

// Worker contexts of ctx (created on first use, destroyed with ctx).
int ensure_workers(rcwa_context* ctx, int K) {
  while ((int)ctx->workers.size() < K) {
    rcwa_context* w = nullptr;
    int rc = rcwa_context_create(ctx->device, &w);
    if (rc) return rc;
    ctx->workers.push_back(w);
  }
  return RCWA_OK;
}

// device bytes per item of a group chunk besides the sweep plan
size_t geometry_bytes_per_item(const ModeDims& d, int nl, int nx, int ny) {
  const size_t NN = (size_t)d.N * d.N, G = (size_t)nx * ny;
  size_t b = 4 * al(nl * NN * sizeof(double2));                 // erc urc einv uinv
  b += 3 * al(nl * sizeof(double2));                            // t, ueps, umu
  b += 2 * nl * G * sizeof(double2);                            // staged grids
  b += convmat_scratch_bytes(nl, nx, ny, d);
  b += (size_t)2 * nl * 2 * NN * sizeof(double2);               // [erc | I], [urc | I]
  b += (size_t)2 * nl * d.N * sizeof(int) + 3 * sizeof(uint32_t) * nl;
  b += 2 * (size_t)d.N * sizeof(double) + 4 * sizeof(double);   // results
  return b + 1024;
}

}  // namespace

size_t problem_bytes(const rcwa_stack& st, const rcwa_params& p, int precision, unsigned mixed_stages,
                     int ir_sweeps, int gemm_digits) {
  ModeDims d;
  d.nxh = p.nx_harmonics;
  d.nyh = p.ny_harmonics;
  d.P = 2 * d.nxh + 1;
  d.Q = 2 * d.nyh + 1;
  d.N = d.P * d.Q;
  d.n = 2 * d.N;
  const size_t G = (size_t)st.nx * st.ny;
  int np = 0;
  for (int l = 0; l < st.num_layers; ++l)
    np += (grid_uniform(st.er + l * G, G) && grid_uniform(st.ur + l * G, G)) ? 0 : 1;
  rcwa_context probe;   // only the mixed-precision settings are read
  probe.tc = precision == RCWA_PREC_MIXED ? mixed_stages : 0u;
  probe.ir_sweeps = ir_sweeps;
  probe.oz_digits = gemm_digits;
  return sweep_bytes_per_source(&probe, d, np) + geometry_bytes_per_item(d, st.num_layers, st.nx, st.ny);
}

namespace {

// One group chunk: items idx0[0..B) share key k0.
int run_chunk(rcwa_context* ctx, const GroupKey& k0, const std::vector<int>& idx0,
              const rcwa_stack* stacks, const rcwa_source* sources, const rcwa_params* params,
              rcwa_result* out, bool& any_status, const ChunkSink* sink) {
  cudaStream_t s = ctx->stream;
  const int B = (int)idx0.size();
  // the chunk's budget comes from its own context (workers get a share)
  // deepest stacks first; layer l belongs to the first nb[l] items
  std::vector<int> idx(idx0);
  GroupKey k = k0;
  std::vector<int> nb;
  if (k.flex) {
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int a, int b) { return stacks[a].num_layers > stacks[b].num_layers; });
    k.nl = stacks[idx[0]].num_layers;
    k.uniform.assign(k.nl, 0);
    nb.assign(k.nl, 0);
    for (int i : idx)
      for (int l = 0; l < stacks[i].num_layers; ++l) ++nb[l];
  }
  const rcwa_params& p0 = params[idx[0]];
  ModeDims d;
  d.nxh = p0.nx_harmonics;
  d.nyh = p0.ny_harmonics;
  d.P = 2 * d.nxh + 1;
  d.Q = 2 * d.nyh + 1;
  d.N = d.P * d.Q;
  d.n = 2 * d.N;
  const int nl = k.nl;
  const size_t NN = (size_t)d.N * d.N, G = (size_t)k.nx * k.ny;
  const size_t L = (size_t)B * nl;   // layers of the chunk

  // per-chunk device memory (stream-ordered pool), released at the end
  std::vector<void*> owned;
  auto dalloc = [&](size_t bytes, void** p) -> int {
    cudaError_t e = cudaMallocAsync(p, std::max<size_t>(bytes, 256), s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_last_error("batch: allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
      return RCWA_ERR_NOMEM;
    }
    owned.push_back(*p);
    return RCWA_OK;
  };
  struct Release {
    std::vector<void*>& v;
    cudaStream_t s;
    ~Release() {
      for (void* p : v) cudaFreeAsync(p, s);
    }
  } release{owned, s};

  double2 *erc, *urc, *einv, *uinv, *grids, *scr, *aug, *ueps_d, *umu_d;
  double *t_d, *res;
  int* piv;
  uint32_t *gst, *dst;
  int rc;
  if ((rc = dalloc(L * NN * sizeof(double2), (void**)&erc)) ||
      (rc = dalloc(L * NN * sizeof(double2), (void**)&urc)) ||
      (rc = dalloc(L * NN * sizeof(double2), (void**)&einv)) ||
      (rc = dalloc(L * NN * sizeof(double2), (void**)&uinv)) ||
      (rc = dalloc(2 * L * G * sizeof(double2), (void**)&grids)) ||
      (rc = dalloc(convmat_scratch_bytes((int)L, k.nx, k.ny, d), (void**)&scr)) ||
      (rc = dalloc(L * sizeof(double), (void**)&t_d)) ||
      (rc = dalloc(L * sizeof(double2), (void**)&ueps_d)) ||
      (rc = dalloc(L * sizeof(double2), (void**)&umu_d)) ||
      (rc = dalloc((size_t)B * (2 * d.N + 2) * sizeof(double) + B * sizeof(uint32_t) + 256, (void**)&res)))
    return rc;

  // grids: er of every item's layers, then ur, in [item][layer][ny][nx] order
  // (slots past a shorter stack's depth stay zero and are never read)
  if (k.flex && L > 0) RCWA_CUDA_TRY(cudaMemsetAsync(grids, 0, 2 * L * G * sizeof(double2), s));
  for (int b = 0; b < B; ++b) {
    const rcwa_stack& st = stacks[idx[b]];
    const int lb = st.num_layers;
    if (lb == 0) continue;
    RCWA_CUDA_TRY(cudaMemcpyAsync(grids + (size_t)b * nl * G, st.er, lb * G * sizeof(double2),
                                  cudaMemcpyHostToDevice, s));
    RCWA_CUDA_TRY(cudaMemcpyAsync(grids + L * G + (size_t)b * nl * G, st.ur, lb * G * sizeof(double2),
                                  cudaMemcpyHostToDevice, s));
  }
  // per-item layer scalars
  std::vector<double> ht(L, 0.0);
  std::vector<double2> he(L, make_double2(1, 0)), hm(L, make_double2(1, 0));
  for (int b = 0; b < B; ++b) {
    const rcwa_stack& st = stacks[idx[b]];
    for (int l = 0; l < st.num_layers; ++l) {
      ht[(size_t)b * nl + l] = st.t[l];
      const rcwa_complex e = st.er[(size_t)l * G], m = st.ur[(size_t)l * G];
      he[(size_t)b * nl + l] = make_double2(e.re, e.im);
      hm[(size_t)b * nl + l] = make_double2(m.re, m.im);
    }
  }
  if (nl > 0) {
    RCWA_CUDA_TRY(cudaMemcpyAsync(t_d, ht.data(), L * sizeof(double), cudaMemcpyHostToDevice, s));
    RCWA_CUDA_TRY(cudaMemcpyAsync(ueps_d, he.data(), L * sizeof(double2), cudaMemcpyHostToDevice, s));
    RCWA_CUDA_TRY(cudaMemcpyAsync(umu_d, hm.data(), L * sizeof(double2), cudaMemcpyHostToDevice, s));
    // ConvMat of every layer of every item (main.cpp:126-138), one batched call per field
    if ((rc = convmat(s, grids, (int)L, k.nx, k.ny, d, erc, scr))) return rc;
    if ((rc = convmat(s, grids + L * G, (int)L, k.nx, k.ny, d, urc, scr))) return rc;
  }
  // inverses of the patterned layers: one LU batch over (item, layer, field)
  std::vector<size_t> slots;   // b * nl + l of every patterned layer present
  for (int b = 0; b < B; ++b)
    for (int l = 0; l < stacks[idx[b]].num_layers; ++l)
      if (!k.uniform[l]) slots.push_back((size_t)b * nl + l);
  const size_t ns = slots.size();
  if (ns > 0) {
    const size_t nsys = 2 * ns;
    const long long s2 = 2 * (long long)NN;
    if ((rc = dalloc(nsys * s2 * sizeof(double2), (void**)&aug)) ||
        (rc = dalloc(nsys * d.N * sizeof(int), (void**)&piv)) ||
        (rc = dalloc(nsys * sizeof(uint32_t), (void**)&gst)))
      return rc;
    for (size_t q = 0; q < ns; ++q) {
      RCWA_CUDA_TRY(cudaMemcpyAsync(aug + q * s2, erc + slots[q] * NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
      RCWA_CUDA_TRY(cudaMemcpyAsync(aug + (ns + q) * s2, urc + slots[q] * NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
    }
    if ((rc = set_identity(s, aug, d.N, d.N, s2, 2 * d.N, d.N, (int)nsys, make_double2(1, 0)))) return rc;
    RCWA_CUDA_TRY(cudaMemsetAsync(gst, 0, nsys * sizeof(uint32_t), s));
    if ((rc = zgesv(s, d.N, d.N, aug, d.N, s2, (int)nsys, piv, gst))) return rc;
    for (size_t q = 0; q < ns; ++q) {
      RCWA_CUDA_TRY(cudaMemcpyAsync(einv + slots[q] * NN, aug + q * s2 + NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
      RCWA_CUDA_TRY(cudaMemcpyAsync(uinv + slots[q] * NN, aug + (ns + q) * s2 + NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
    }
  }

  Layers Gl;
  Gl.d = d;
  Gl.nl = nl;
  Gl.er_ref = make_double2(k.p[0], k.p[1]);
  Gl.ur_ref = make_double2(k.p[2], k.p[3]);
  Gl.er_trn = make_double2(k.p[4], k.p[5]);
  Gl.ur_trn = make_double2(k.p[6], k.p[7]);
  Gl.uniform = k.uniform.data();
  Gl.erc = erc;
  Gl.urc = urc;
  Gl.einv = einv;
  Gl.uinv = uinv;
  Gl.s_layer = (long long)NN;
  Gl.s_item = (long long)nl * NN;
  Gl.t_item = t_d;
  Gl.ueps_item = ueps_d;
  Gl.umu_item = umu_d;
  Gl.nb = k.flex ? nb.data() : nullptr;

  std::vector<SourceDev> hs(B);
  for (int b = 0; b < B; ++b) {
    const rcwa_source& q = sources[idx[b]];
    const rcwa_stack& st = stacks[idx[b]];
    hs[b] = SourceDev{q.lambda0, q.theta, q.phi, q.pte, q.ptm, st.lx, st.ly};
  }
  double* dR = res;
  double* dT = dR + (size_t)B * d.N;
  double* dtot = dT + (size_t)B * d.N;
  dst = (uint32_t*)(dtot + 2 * (size_t)B);
  if ((rc = sweep_chunk_layers(ctx, Gl, hs.data(), B, dR, dT, dtot, dst))) return rc;

  std::vector<double> hR((size_t)B * d.N), hT((size_t)B * d.N), htot(2 * (size_t)B);
  std::vector<uint32_t> hst(B);
  RCWA_CUDA_TRY(cudaMemcpyAsync(hR.data(), dR, hR.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(hT.data(), dT, hT.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(htot.data(), dtot, htot.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(hst.data(), dst, B * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  for (int b = 0; b < B; ++b) {
    rcwa_result& o = out[idx[b]];
    if (o.R) std::memcpy(o.R, hR.data() + (size_t)b * d.N, d.N * sizeof(double));
    if (o.T) std::memcpy(o.T, hT.data() + (size_t)b * d.N, d.N * sizeof(double));
    o.R_tot = htot[2 * b];
    o.T_tot = htot[2 * b + 1];
    o.status = hst[b];
    any_status = any_status || hst[b] != 0;
  }
  if (ctx->tc) {   // a mixed-precision chunk is only handed out once its tensor-core waits all held
    int* terr = tc_error_flag();
    int h = 0;
    if (terr) RCWA_CUDA_TRY(cudaMemcpy(&h, terr, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
      set_last_error("tensor-core GEMM: a bounded mbarrier wait expired");
      return RCWA_ERR_CUDA;
    }
  }
  if (sink && sink->fn) sink->fn(sink->user, idx.data(), B);
  return RCWA_OK;
}

}  // namespace

int solve_batch(rcwa_context* ctx, int n, const rcwa_stack* stacks, const rcwa_source* sources,
                const rcwa_params* params, int precision, int max_group, rcwa_result* out,
                const ChunkSink* sink) {
  if (precision != RCWA_PREC_FP64 && precision != RCWA_PREC_MIXED) {
    set_last_error("unknown precision mode %d", precision);
    return RCWA_ERR_INVALID;
  }
  cudaGetLastError();   // no stale error from earlier unchecked calls on this thread
  // group by shape, keeping the order of first appearance
  std::map<GroupKey, int> gid;
  std::vector<GroupKey> keys;
  std::vector<std::vector<int>> members;
  for (int i = 0; i < n; ++i) {
    const rcwa_stack& st = stacks[i];
    const rcwa_params& p = params[i];
    GroupKey k;
    k.nxh = p.nx_harmonics;
    k.nyh = p.ny_harmonics;
    k.nl = st.num_layers;
    k.nx = st.nx;
    k.ny = st.ny;
    const double pv[8] = {p.er_ref.re, p.er_ref.im, p.ur_ref.re, p.ur_ref.im,
                          p.er_trn.re, p.er_trn.im, p.ur_trn.re, p.ur_trn.im};
    std::memcpy(k.p, pv, sizeof(pv));
    const size_t G = (size_t)st.nx * st.ny;
    k.uniform.resize(st.num_layers);
    bool any_uniform = false;
    for (int l = 0; l < st.num_layers; ++l) {
      k.uniform[l] = (grid_uniform(st.er + l * G, G) && grid_uniform(st.ur + l * G, G)) ? 1 : 0;
      any_uniform = any_uniform || k.uniform[l];
    }
    k.flex = (st.num_layers > 0 && !any_uniform) ? 1 : 0;
    if (k.flex) {
      k.nl = -1;
      k.uniform.clear();
    }
    auto it = gid.find(k);
    if (it == gid.end()) {
      it = gid.emplace(k, (int)keys.size()).first;
      keys.push_back(k);
      members.emplace_back();
    }
    members[it->second].push_back(i);
  }
  // memory budget per chunk
  size_t budget = ctx->mem_budget;
  if (budget == 0) {
    size_t fr = 0, totm = 0;
    RCWA_CUDA_TRY(cudaMemGetInfo(&fr, &totm));
    budget = (size_t)((fr + ctx->ws_bytes) * 0.5);
  }
  int* tc_err = nullptr;
  if (precision == RCWA_PREC_MIXED) {
    tc_err = tc_error_flag();
    if (!tc_err) {
      set_last_error("tensor-core GEMM error flag unavailable on this device");
      return RCWA_ERR_CUDA;
    }
    RCWA_CUDA_TRY(cudaMemsetAsync(tc_err, 0, sizeof(int), ctx->stream));
  }
  struct TcScope {
    rcwa_context* c;
    ~TcScope() { c->tc = 0; }
  } tc_scope{ctx};
  ctx->tc = precision == RCWA_PREC_MIXED ? ctx->mixed_stages : 0u;
  // chunks of every group, sized for a share of the budget each, so that
  // several can run at once
  const int kmax = batch_streams();
  struct Job {
    int g;
    std::vector<int> idx;
    double cost;
  };
  std::vector<Job> jobs;
  for (size_t g = 0; g < keys.size(); ++g) {
    const GroupKey& k = keys[g];
    ModeDims d;
    d.nxh = k.nxh;
    d.nyh = k.nyh;
    d.P = 2 * d.nxh + 1;
    d.Q = 2 * d.nyh + 1;
    d.N = d.P * d.Q;
    d.n = 2 * d.N;
    const std::vector<int>& m = members[g];
    int nl = k.nl, np = 0;
    if (k.flex) {
      nl = 0;
      for (int i : m) nl = std::max(nl, stacks[i].num_layers);
      np = nl;
    } else {
      for (int l = 0; l < k.nl; ++l) np += k.uniform[l] ? 0 : 1;
    }
    const size_t per = sweep_bytes_per_source(ctx, d, np) + geometry_bytes_per_item(d, nl, k.nx, k.ny);
    int chunk = (int)std::max<size_t>(1, budget / kmax / per);
    // launch grids index matrices in a 65535-wide grid dimension: at most
    // 2 * layers * items systems per batched LU
    chunk = std::min(chunk, std::max(1, 32000 / std::max(1, 2 * std::max(nl, 1))));
    if (max_group > 0) chunk = std::min(chunk, max_group);
    for (size_t b0 = 0; b0 < m.size(); b0 += chunk) {
      const size_t bc = std::min<size_t>(chunk, m.size() - b0);
      Job j{(int)g, std::vector<int>(m.begin() + b0, m.begin() + b0 + bc), 0.0};
      for (int i : j.idx) j.cost += (double)d.n * d.n * d.n * (stacks[i].num_layers + 2);
      jobs.push_back(std::move(j));
    }
  }
  const int K = std::min<int>(kmax, (int)jobs.size());
  std::atomic<bool> any_status{false};
  if (K <= 1) {
    for (const Job& j : jobs) {
      bool st = false;
      int rc = run_chunk(ctx, keys[j.g], j.idx, stacks, sources, params, out, st, sink);
      if (st) any_status = true;
      if (rc) return rc;
    }
  } else {
    // independent groups run concurrently, one worker context (own stream
    // and workspace) and host thread each; longest jobs are placed first
    std::vector<int> order(jobs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].cost > jobs[b].cost; });
    std::vector<std::vector<int>> bins(K);
    std::vector<double> load(K, 0.0);
    for (int j : order) {
      const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      bins[w].push_back(j);
      load[w] += jobs[j].cost;
    }
    int rc = ensure_workers(ctx, K);
    if (rc) return rc;
    // the workers' streams follow the caller's stream and the caller's
    // stream waits for them, so events on it bracket the whole batch
    cudaEvent_t start;
    RCWA_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    RCWA_CUDA_TRY(cudaEventRecord(start, ctx->stream));
    std::vector<int> rcs(K, RCWA_OK);
    std::vector<std::string> errs(K);
    std::vector<std::thread> th;
    for (int w = 0; w < K; ++w) {
      th.emplace_back([&, w] {
        rcwa_context* wc = ctx->workers[w];
        wc->tc = ctx->tc;
        wc->mixed_stages = ctx->mixed_stages;
        wc->ir_sweeps = ctx->ir_sweeps;
        wc->oz_digits = ctx->oz_digits;
        cudaError_t e = cudaSetDevice(wc->device);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(wc->stream, start, 0);
        cudaGetLastError();   // launch checks below must see only their own launches
        if (e != cudaSuccess) {
          rcs[w] = RCWA_ERR_CUDA;
          errs[w] = std::string("batch worker set-up: ") + cudaGetErrorString(e);
          return;
        }
        for (int j : bins[w]) {
          bool st = false;
          int r = run_chunk(wc, keys[jobs[j].g], jobs[j].idx, stacks, sources, params, out, st, sink);
          if (st) any_status = true;
          if (r) {
            rcs[w] = r;
            errs[w] = rcwa_last_error();
            break;
          }
        }
        wc->tc = 0;
      });
    }
    for (auto& t : th) t.join();
    for (int w = 0; w < K; ++w) {
      cudaEvent_t done;
      RCWA_CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
      RCWA_CUDA_TRY(cudaEventRecord(done, ctx->workers[w]->stream));
      RCWA_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, done, 0));
      RCWA_CUDA_TRY(cudaEventDestroy(done));
    }
    RCWA_CUDA_TRY(cudaEventDestroy(start));
    for (int w = 0; w < K; ++w)
      if (rcs[w]) {
        set_last_error("%s", errs[w].c_str());
        return rcs[w];
      }
  }
  if (tc_err) {
    int h = 0;
    RCWA_CUDA_TRY(cudaMemcpyAsync(&h, tc_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h) {
      set_last_error("tensor-core GEMM: a bounded mbarrier wait expired");
      return RCWA_ERR_CUDA;
    }
  }
  return any_status.load() ? RCWA_ERR_NUMERIC : RCWA_OK;
}

}  // namespace rcwa
