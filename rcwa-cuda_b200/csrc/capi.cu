// extern "C" boundary (include/rcwa_b200.h).  Host-pointer entry points stage
// through the context's device workspace; nothing here computes on the CPU.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <new>
#include <vector>

#include "solver.cuh"

namespace rcwa {

static thread_local char g_err[512] = "";
static std::atomic<uint64_t> g_launches{0};

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

int step_smatrix_layer(rcwa_context* ctx, int N, const double2* erc, const double2* urc,
                       const double2* Kx, const double2* Ky, const double2* V0d, double k0,
                       double t, double2* S11, double2* S12, uint32_t* status);
int step_port(rcwa_context* ctx, int side, int N, double2 er, double2 ur, const double2* Kx,
              const double2* Ky, const double2* Kz, const double2* V0d, double2* S[4]);
int step_redheffer(rcwa_context* ctx, int n, const double2* const A[4], const double2* const B[4],
                   double2* const S[4], uint32_t* status);
int step_efficiencies(rcwa_context* ctx, const rcwa_source* src, const rcwa_params* p,
                      const double2* kinc, const double2* Kx, const double2* Ky,
                      const double2* Kzr, const double2* Kzt, const double2* S11,
                      const double2* S21, rcwa_result* out);
int step_wave_vectors(rcwa_context* ctx, double lx, double ly, const rcwa_source* src,
                      const rcwa_params* p, double2* kinc, double2* Kx, double2* Ky, double2* Kzr,
                      double2* Kzt, double2* V0d);
int step_gap_v0(rcwa_context* ctx, int N, const double2* Kx, const double2* Ky, double2* V0d);

}  // namespace rcwa

using namespace rcwa;

#define CHECK_ARG(cond, msg)                 \
  do {                                       \
    if (!(cond)) {                           \
      rcwa::set_last_error("%s", msg);       \
      return RCWA_ERR_INVALID;               \
    }                                        \
  } while (0)

static int check_params(const rcwa_params* p) {
  CHECK_ARG(p, "params is NULL");
  CHECK_ARG(p->nx_harmonics >= 0 && p->ny_harmonics >= 0, "negative harmonic order");
  CHECK_ARG((2 * p->nx_harmonics + 1) * (2 * p->ny_harmonics + 1) <= 4096, "harmonic order too large");
  return RCWA_OK;
}
static int check_stack(const rcwa_stack* s) {
  CHECK_ARG(s, "stack is NULL");
  CHECK_ARG(s->nx > 0 && s->ny > 0 && s->num_layers >= 0, "bad grid size");
  CHECK_ARG(s->num_layers == 0 || (s->er && s->ur && s->t), "stack arrays are NULL");
  CHECK_ARG(s->lx > 0 && s->ly > 0, "bad period");
  return RCWA_OK;
}

extern "C" {

const char* rcwa_last_error(void) { return g_err; }
int rcwa_version(void) { return 10000; }

int rcwa_context_create(int device, rcwa_context** out) {
  CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  RCWA_CUDA_TRY(cudaGetDeviceCount(&ndev));
  CHECK_ARG(device >= 0 && device < ndev, "no such CUDA device");
  RCWA_CUDA_TRY(cudaSetDevice(device));
  rcwa_context* c = new (std::nothrow) rcwa_context();
  if (!c) return RCWA_ERR_NOMEM;
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_last_error("stream: %s", cudaGetErrorString(e));
    delete c;
    return RCWA_ERR_CUDA;
  }
  c->stream = c->own_stream;
  {
    // geometries and result buffers come from the device's default
    // stream-ordered pool; keep up to 1 GiB of it cached between calls so
    // that repeated solves do not return memory to the driver each time
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = 0;
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      if (keep < (1ull << 30)) {
        keep = 1ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
    }
    cudaGetLastError();
  }
  c->launches_at_create = launch_count();
  *out = c;
  return RCWA_OK;
}

int rcwa_context_destroy(rcwa_context* c) {
  if (!c) return RCWA_OK;
  cudaSetDevice(c->device);
  for (rcwa_context* w : c->workers) rcwa_context_destroy(w);
  c->workers.clear();
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->ws) cudaFree(c->ws);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return RCWA_OK;
}

int rcwa_context_set_stream(rcwa_context* c, void* stream) {
  CHECK_ARG(c, "ctx is NULL");
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return RCWA_OK;
}

int rcwa_context_synchronize(rcwa_context* c) {
  CHECK_ARG(c, "ctx is NULL");
  RCWA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return RCWA_OK;
}

int rcwa_context_kernel_launches(rcwa_context* c, uint64_t* count) {
  CHECK_ARG(c && count, "NULL argument");
  *count = launch_count() - c->launches_at_create;
  return RCWA_OK;
}

int rcwa_context_set_mixed(rcwa_context* c, unsigned stages, int refine_sweeps, int gemm_digits) {
  CHECK_ARG(c, "NULL context");
  CHECK_ARG(gemm_digits >= 4 && gemm_digits <= 6, "gemm_digits must be 4, 5 or 6");
  CHECK_ARG((stages & ~(unsigned)(RCWA_MIXED_ALL | RCWA_MIXED_GEMM_TF32 | RCWA_MIXED_REFINE_INT8)) == 0,
            "unknown mixed-precision stage bits");
  CHECK_ARG(refine_sweeps >= 1 && refine_sweeps <= 4, "refine_sweeps must be 1..4");
  c->mixed_stages = stages;
  c->ir_sweeps = refine_sweeps;
  c->oz_digits = gemm_digits;
  return RCWA_OK;
}

int rcwa_geometry_create(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_params* params,
                         int stack_on_device, rcwa_geometry** out) {
  return rcwa_geometry_create_ex(ctx, stack, params, stack_on_device, 0u, out);
}

int rcwa_geometry_create_ex(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_params* params,
                            int stack_on_device, unsigned flags, rcwa_geometry** out) {
  CHECK_ARG(ctx && out, "NULL argument");
  CHECK_ARG((flags & ~RCWA_GEOM_LI_RULE) == 0u, "unknown geometry flags");
  int rc = check_stack(stack);
  if (rc) return rc;
  if ((rc = check_params(params))) return rc;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  rcwa_geometry* g = new (std::nothrow) rcwa_geometry();
  if (!g) return RCWA_ERR_NOMEM;
  rc = geometry_build(ctx, g, stack, params, stack_on_device, flags);
  if (rc) {
    geometry_free(g);
    delete g;
    return rc;
  }
  *out = g;
  return RCWA_OK;
}

int rcwa_geometry_destroy(rcwa_geometry* g) {
  if (!g) return RCWA_OK;
  geometry_free(g);   // stream-ordered frees on the context stream
  delete g;
  return RCWA_OK;
}

int rcwa_solve_sweep_device(rcwa_context* ctx, const rcwa_geometry* geom, const rcwa_source* sources,
                            int n_sources, int precision, double* R_dev, double* T_dev,
                            double* tot_dev, uint32_t* status_dev) {
  CHECK_ARG(ctx && geom && sources && R_dev && T_dev && tot_dev && status_dev, "NULL argument");
  CHECK_ARG(n_sources >= 0, "negative source count");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  return sweep_device(ctx, geom, sources, n_sources, precision, R_dev, T_dev, tot_dev, status_dev);
}

int rcwa_solve_sweep(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_source* sources,
                     int n_sources, const rcwa_params* params, int precision, rcwa_result* out) {
  CHECK_ARG(ctx && sources && out, "NULL argument");
  CHECK_ARG(n_sources > 0, "no sources");
  rcwa_geometry* g = nullptr;
  int rc = rcwa_geometry_create(ctx, stack, params, 0, &g);
  if (rc) return rc;
  const int N = g->d.N;
  double *dR = nullptr, *dT = nullptr, *dtot = nullptr;
  uint32_t* dst = nullptr;
  const size_t nR = (size_t)n_sources * N;
  cudaError_t e = cudaMallocAsync((void**)&dR, 2 * nR * sizeof(double) + 2 * n_sources * sizeof(double) +
                                                    n_sources * sizeof(uint32_t) + 512, ctx->stream);
  if (e != cudaSuccess) {
    rcwa_geometry_destroy(g);
    set_last_error("result allocation failed: %s", cudaGetErrorString(e));
    return RCWA_ERR_NOMEM;
  }
  dT = dR + nR;
  dtot = dT + nR;
  dst = (uint32_t*)(dtot + 2 * n_sources);
  rc = sweep_device(ctx, g, sources, n_sources, precision, dR, dT, dtot, dst);
  std::vector<double> hR(nR), hT(nR), htot(2 * n_sources);
  std::vector<uint32_t> hst(n_sources);
  if (!rc) {
    cudaStream_t s = ctx->stream;
    e = cudaMemcpyAsync(hR.data(), dR, nR * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hT.data(), dT, nR * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(htot.data(), dtot, 2 * n_sources * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hst.data(), dst, n_sources * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_last_error("result copy: %s", cudaGetErrorString(e));
      rc = RCWA_ERR_CUDA;
    }
  }
  cudaFreeAsync(dR, ctx->stream);
  rcwa_geometry_destroy(g);
  if (rc) return rc;
  bool any = false;
  for (int i = 0; i < n_sources; ++i) {
    if (out[i].R) std::memcpy(out[i].R, hR.data() + (size_t)i * N, N * sizeof(double));
    if (out[i].T) std::memcpy(out[i].T, hT.data() + (size_t)i * N, N * sizeof(double));
    out[i].R_tot = htot[2 * i];
    out[i].T_tot = htot[2 * i + 1];
    out[i].status = hst[i];
    any = any || hst[i] != 0;
  }
  return any ? RCWA_ERR_NUMERIC : RCWA_OK;
}

int rcwa_solve(rcwa_context* ctx, const rcwa_stack* stack, const rcwa_source* source,
               const rcwa_params* params, int precision, rcwa_result* out) {
  return rcwa_solve_sweep(ctx, stack, source, 1, params, precision, out);
}

int rcwa_rasterize(rcwa_context* ctx, int nx, int ny, double lx, double ly, int nl,
                   const rcwa_layer_shapes* layers, rcwa_complex* er_dev, rcwa_complex* ur_dev,
                   double* t_dev) {
  CHECK_ARG(ctx && (nl == 0 || (layers && er_dev && ur_dev)), "NULL argument");
  CHECK_ARG(nx > 0 && ny > 0 && nl >= 0 && lx > 0 && ly > 0, "bad grid");
  for (int l = 0; l < nl; ++l) CHECK_ARG(layers[l].n_shapes >= 0 && (layers[l].n_shapes == 0 || layers[l].shapes), "bad layer");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  return rasterize(ctx, nx, ny, lx, ly, nl, layers, (double2*)er_dev, (double2*)ur_dev, t_dev);
}

int rcwa_geometry_create_shapes(rcwa_context* ctx, int nx, int ny, double lx, double ly, int nl,
                                const rcwa_layer_shapes* layers, const rcwa_params* params,
                                rcwa_geometry** out) {
  CHECK_ARG(ctx && out && (nl == 0 || layers), "NULL argument");
  CHECK_ARG(nx > 0 && ny > 0 && nl >= 0 && lx > 0 && ly > 0, "bad grid");
  int rc = check_params(params);
  if (rc) return rc;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t G = (size_t)nx * ny;
  char* buf = nullptr;
  const size_t bytes = 2 * (size_t)(nl > 0 ? nl : 1) * G * sizeof(double2) + (size_t)(nl + 1) * sizeof(double) + 512;
  RCWA_CUDA_TRY(cudaMallocAsync((void**)&buf, bytes, ctx->stream));
  double2* er = (double2*)buf;
  double2* ur = er + (size_t)nl * G;
  double* t = (double*)(ur + (size_t)nl * G);
  rc = rasterize(ctx, nx, ny, lx, ly, nl, layers, er, ur, t);
  if (!rc) {
    rcwa_stack st{nx, ny, nl, lx, ly, (const rcwa_complex*)er, (const rcwa_complex*)ur, t};
    rc = rcwa_geometry_create(ctx, &st, params, 1, out);   // reads the grids in place, synchronises
  }
  cudaFreeAsync(buf, ctx->stream);
  return rc;
}

int rcwa_solve_batch(rcwa_context* ctx, int n, const rcwa_stack* stacks, const rcwa_source* sources,
                     const rcwa_params* params, int precision, rcwa_result* out) {
  CHECK_ARG(ctx && stacks && sources && params && out, "NULL argument");
  CHECK_ARG(n >= 0, "negative problem count");
  for (int i = 0; i < n; ++i) {
    int rc = check_stack(stacks + i);
    if (!rc) rc = check_params(params + i);
    if (rc) return rc;
  }
  if (n == 0) return RCWA_OK;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  return solve_batch(ctx, n, stacks, sources, params, precision, 0, out);
}

// ---- step level -------------------------------------------------------------
int rcwa_convmat(rcwa_context* ctx, const rcwa_complex* field, int layer, int nx, int ny,
                 int nx_harmonics, int ny_harmonics, rcwa_complex* out) {
  CHECK_ARG(ctx && field && out, "NULL argument");
  CHECK_ARG(nx > 0 && ny > 0 && layer >= 0, "bad grid");
  rcwa_params p{};
  p.nx_harmonics = nx_harmonics;
  p.ny_harmonics = ny_harmonics;
  int rc = check_params(&p);
  if (rc) return rc;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  ModeDims d;
  d.nxh = nx_harmonics; d.nyh = ny_harmonics;
  d.P = 2 * d.nxh + 1; d.Q = 2 * d.nyh + 1; d.N = d.P * d.Q; d.n = 2 * d.N;
  const size_t G = (size_t)nx * ny, NN = (size_t)d.N * d.N;
  const size_t scr = convmat_scratch_bytes(1, nx, ny, d);
  if ((rc = ctx_reserve(ctx, G * 16 + NN * 16 + scr + 1024))) return rc;
  double2* dg = (double2*)ctx->ws;
  double2* dout = dg + G;
  double2* dscr = dout + NN;
  cudaStream_t s = ctx->stream;
  RCWA_CUDA_TRY(cudaMemcpyAsync(dg, field + (size_t)layer * G, G * 16, cudaMemcpyHostToDevice, s));
  if ((rc = convmat(s, dg, 1, nx, ny, d, dout, dscr))) return rc;
  RCWA_CUDA_TRY(cudaMemcpyAsync(out, dout, NN * 16, cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  return RCWA_OK;
}

int rcwa_wave_vectors(rcwa_context* ctx, double lx, double ly, const rcwa_source* source,
                      const rcwa_params* params, rcwa_complex* k_inc, rcwa_complex* Kx,
                      rcwa_complex* Ky, rcwa_complex* Kz_ref, rcwa_complex* Kz_trn) {
  CHECK_ARG(ctx && source && k_inc && Kx && Ky && Kz_ref && Kz_trn, "NULL argument");
  int rc = check_params(params);
  if (rc) return rc;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const int N = (2 * params->nx_harmonics + 1) * (2 * params->ny_harmonics + 1);
  std::vector<double2> kinc(4), v0(4 * N);
  rc = step_wave_vectors(ctx, lx, ly, source, params, kinc.data(), (double2*)Kx, (double2*)Ky,
                         (double2*)Kz_ref, (double2*)Kz_trn, v0.data());
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) k_inc[k] = rcwa_complex{kinc[k].x, kinc[k].y};
  return RCWA_OK;
}

static void v0_from_dense(int N, const rcwa_complex* V0, std::vector<double2>& d) {
  const int n = 2 * N;
  d.resize(4 * N);
  for (int i = 0; i < N; ++i) {
    const rcwa_complex a = V0[(size_t)i * n + i], b = V0[(size_t)(i + N) * n + i],
                       c = V0[(size_t)i * n + i + N], e = V0[(size_t)(i + N) * n + i + N];
    d[i] = make_double2(a.re, a.im);
    d[N + i] = make_double2(b.re, b.im);
    d[2 * N + i] = make_double2(c.re, c.im);
    d[3 * N + i] = make_double2(e.re, e.im);
  }
}

int rcwa_gap_medium(rcwa_context* ctx, int pq, const rcwa_complex* Kx, const rcwa_complex* Ky,
                    rcwa_complex* W0, rcwa_complex* V0) {
  CHECK_ARG(ctx && Kx && Ky && W0 && V0 && pq > 0, "bad argument");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  std::vector<double2> d(4 * pq);
  int rc = step_gap_v0(ctx, pq, (const double2*)Kx, (const double2*)Ky, d.data());
  if (rc) return rc;
  const int n = 2 * pq;
  std::memset(W0, 0, sizeof(rcwa_complex) * n * n);
  std::memset(V0, 0, sizeof(rcwa_complex) * n * n);
  for (int i = 0; i < n; ++i) W0[(size_t)i * n + i] = rcwa_complex{1.0, 0.0};
  for (int i = 0; i < pq; ++i) {
    V0[(size_t)i * n + i] = rcwa_complex{d[i].x, d[i].y};
    V0[(size_t)(i + pq) * n + i] = rcwa_complex{d[pq + i].x, d[pq + i].y};
    V0[(size_t)i * n + i + pq] = rcwa_complex{d[2 * pq + i].x, d[2 * pq + i].y};
    V0[(size_t)(i + pq) * n + i + pq] = rcwa_complex{d[3 * pq + i].x, d[3 * pq + i].y};
  }
  return RCWA_OK;
}

int rcwa_smatrix_layer(rcwa_context* ctx, int pq, const rcwa_complex* erc, const rcwa_complex* urc,
                       const rcwa_complex* Kx, const rcwa_complex* Ky, const rcwa_complex* V0,
                       double k0, double thickness, rcwa_complex* S11, rcwa_complex* S12,
                       uint32_t* status) {
  CHECK_ARG(ctx && erc && urc && Kx && Ky && V0 && S11 && S12 && pq > 0, "bad argument");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  std::vector<double2> v0;
  v0_from_dense(pq, V0, v0);
  uint32_t st = 0;
  int rc = step_smatrix_layer(ctx, pq, (const double2*)erc, (const double2*)urc, (const double2*)Kx,
                              (const double2*)Ky, v0.data(), k0, thickness, (double2*)S11,
                              (double2*)S12, &st);
  if (status) *status = st;
  return rc;
}

static int port_common(rcwa_context* ctx, int side, const rcwa_params* p, const rcwa_complex* Kx,
                       const rcwa_complex* Ky, const rcwa_complex* Kz, const rcwa_complex* V0,
                       rcwa_complex* S11, rcwa_complex* S12, rcwa_complex* S21, rcwa_complex* S22) {
  CHECK_ARG(ctx && Kx && Ky && Kz && V0 && S11 && S12 && S21 && S22, "NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const int N = (2 * p->nx_harmonics + 1) * (2 * p->ny_harmonics + 1);
  std::vector<double2> v0;
  v0_from_dense(N, V0, v0);
  double2* S[4] = {(double2*)S11, (double2*)S12, (double2*)S21, (double2*)S22};
  const rcwa_complex er = side == 0 ? p->er_ref : p->er_trn;
  const rcwa_complex ur = side == 0 ? p->ur_ref : p->ur_trn;
  return step_port(ctx, side, N, make_double2(er.re, er.im), make_double2(ur.re, ur.im),
                   (const double2*)Kx, (const double2*)Ky, (const double2*)Kz, v0.data(), S);
}

int rcwa_smatrix_reflection(rcwa_context* ctx, const rcwa_params* params, const rcwa_complex* Kx,
                            const rcwa_complex* Ky, const rcwa_complex* Kz_ref,
                            const rcwa_complex* V0, rcwa_complex* S11, rcwa_complex* S12,
                            rcwa_complex* S21, rcwa_complex* S22) {
  return port_common(ctx, 0, params, Kx, Ky, Kz_ref, V0, S11, S12, S21, S22);
}

int rcwa_smatrix_transmission(rcwa_context* ctx, const rcwa_params* params, const rcwa_complex* Kx,
                              const rcwa_complex* Ky, const rcwa_complex* Kz_trn,
                              const rcwa_complex* V0, rcwa_complex* S11, rcwa_complex* S12,
                              rcwa_complex* S21, rcwa_complex* S22) {
  return port_common(ctx, 1, params, Kx, Ky, Kz_trn, V0, S11, S12, S21, S22);
}

int rcwa_redheffer(rcwa_context* ctx, int n, const rcwa_complex* const A[4],
                   const rcwa_complex* const B[4], rcwa_complex* const S[4], uint32_t* status) {
  CHECK_ARG(ctx && A && B && S && n > 0, "bad argument");
  for (int k = 0; k < 4; ++k) CHECK_ARG(A[k] && B[k] && S[k], "NULL block");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  uint32_t st = 0;
  int rc = step_redheffer(ctx, n, (const double2* const*)A, (const double2* const*)B,
                          (double2* const*)S, &st);
  if (status) *status = st;
  return rc;
}

int rcwa_efficiencies(rcwa_context* ctx, const rcwa_source* source, const rcwa_params* params,
                      const rcwa_complex* k_inc, const rcwa_complex* Kx, const rcwa_complex* Ky,
                      const rcwa_complex* Kz_ref, const rcwa_complex* Kz_trn,
                      const rcwa_complex* S11, const rcwa_complex* S21, rcwa_result* out) {
  CHECK_ARG(ctx && source && k_inc && Kx && Ky && Kz_ref && Kz_trn && S11 && S21 && out, "NULL argument");
  int rc = check_params(params);
  if (rc) return rc;
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  return step_efficiencies(ctx, source, params, (const double2*)k_inc, (const double2*)Kx,
                           (const double2*)Ky, (const double2*)Kz_ref, (const double2*)Kz_trn,
                           (const double2*)S11, (const double2*)S21, out);
}

int rcwa_eig(rcwa_context* ctx, int n, int batch, const rcwa_complex* A, rcwa_complex* lam,
             rcwa_complex* W, uint32_t* status) {
  CHECK_ARG(ctx && A && lam && W && n > 0 && batch > 0, "bad argument");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t nn = (size_t)n * n;
  const size_t need = (2 * nn * batch + (size_t)n * batch) * 16 + zeig_workspace_bytes(n, batch) +
                      batch * sizeof(uint32_t) + 2048;
  int rc = ctx_reserve(ctx, need);
  if (rc) return rc;
  char* w = (char*)ctx->ws;
  double2* dA = (double2*)w;
  double2* dW = dA + nn * batch;
  double2* dl = dW + nn * batch;
  uint32_t* dst = (uint32_t*)(dl + (size_t)n * batch);
  void* eigws = (void*)(((uintptr_t)(dst + batch) + 255) & ~(uintptr_t)255);
  cudaStream_t s = ctx->stream;
  RCWA_CUDA_TRY(cudaMemcpyAsync(dA, A, nn * batch * 16, cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemsetAsync(dst, 0, batch * sizeof(uint32_t), s));
  if ((rc = zeig(s, n, batch, dA, n, nn, dW, nn, dl, n, dst, eigws))) return rc;
  RCWA_CUDA_TRY(cudaMemcpyAsync(W, dW, nn * batch * 16, cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(lam, dl, (size_t)n * batch * 16, cudaMemcpyDeviceToHost, s));
  std::vector<uint32_t> hst(batch);
  RCWA_CUDA_TRY(cudaMemcpyAsync(hst.data(), dst, batch * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  bool any = false;
  for (int b = 0; b < batch; ++b) {
    if (status) status[b] = hst[b];
    any = any || hst[b];
  }
  return any ? RCWA_ERR_NUMERIC : RCWA_OK;
}

int rcwa_lu_solve(rcwa_context* ctx, int n, int nrhs, int batch, const rcwa_complex* A,
                  const rcwa_complex* B, rcwa_complex* X, uint32_t* status) {
  return rcwa_lu_solve_ex(ctx, n, nrhs, batch, A, B, X, status, RCWA_PREC_FP64, 1);
}

int rcwa_lu_solve_ex(rcwa_context* ctx, int n, int nrhs, int batch, const rcwa_complex* A,
                     const rcwa_complex* B, rcwa_complex* X, uint32_t* status, int precision,
                     int refine_sweeps) {
  CHECK_ARG(ctx && A && B && X && n > 0 && nrhs > 0 && batch > 0, "bad argument");
  CHECK_ARG(precision == RCWA_PREC_FP64 || precision == RCWA_PREC_MIXED, "unknown precision mode");
  CHECK_ARG(refine_sweeps >= 1 && refine_sweeps <= 4, "refine_sweeps must be 1..4");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t nn = (size_t)n * n, nr = (size_t)n * nrhs, sa = nn + nr;
  const size_t base = ((sa * batch * 16 + (size_t)n * batch * sizeof(int) + batch * 4) + 511) & ~(size_t)255;
  const size_t irb = precision == RCWA_PREC_MIXED ? zgesv_ir_ws_bytes(n, nrhs, batch, refine_sweeps) : 0;
  int rc = ctx_reserve(ctx, base + irb + 1024);
  if (rc) return rc;
  double2* dM = (double2*)ctx->ws;
  int* piv = (int*)(dM + sa * batch);
  uint32_t* dst = (uint32_t*)(piv + (size_t)n * batch);
  void* irws = (char*)ctx->ws + base;
  cudaStream_t s = ctx->stream;
  RCWA_CUDA_TRY(cudaMemcpy2DAsync(dM, sa * 16, A, nn * 16, nn * 16, batch, cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemcpy2DAsync(dM + nn, sa * 16, B, nr * 16, nr * 16, batch, cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemsetAsync(dst, 0, batch * 4, s));
  if (precision == RCWA_PREC_MIXED)
    rc = zgesv_ir(s, n, nrhs, dM, n, (long long)sa, batch, piv, dst, irws, refine_sweeps);
  else
    rc = zgesv(s, n, nrhs, dM, n, (long long)sa, batch, piv, dst);
  if (rc) return rc;
  RCWA_CUDA_TRY(cudaMemcpy2DAsync(X, nr * 16, dM + nn, sa * 16, nr * 16, batch, cudaMemcpyDeviceToHost, s));
  std::vector<uint32_t> hst(batch);
  RCWA_CUDA_TRY(cudaMemcpyAsync(hst.data(), dst, batch * 4, cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  bool any = false;
  for (int b = 0; b < batch; ++b) {
    if (status) status[b] = hst[b];
    any = any || hst[b];
  }
  return any ? RCWA_ERR_NUMERIC : RCWA_OK;
}

int rcwa_gemm(rcwa_context* ctx, int m, int n, int k, int batch, const rcwa_complex* A,
              const rcwa_complex* B, rcwa_complex* C, int precision) {
  CHECK_ARG(ctx && A && B && C && m > 0 && n > 0 && k > 0 && batch > 0, "bad argument");
  CHECK_ARG(precision == RCWA_PREC_FP64 || precision == RCWA_PREC_MIXED, "unknown precision mode");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t na = (size_t)m * k, nb = (size_t)k * n, nc = (size_t)m * n;
  const int kind = precision != RCWA_PREC_MIXED ? 0 : (ctx->mixed_stages & RCWA_MIXED_GEMM_TF32) ? TC_TF32 : TC_INT8;
  const size_t base = ((na + nb + nc) * batch * 16 + 511) & ~(size_t)255;
  const size_t wsb = kind == TC_INT8 ? zgemm_oz_ws_bytes(m, n, k, batch, ctx->oz_digits) : 0;
  int rc = ctx_reserve(ctx, base + wsb + 1024);
  if (rc) return rc;
  double2* dA = (double2*)ctx->ws;
  double2* dB = dA + na * batch;
  double2* dC = dB + nb * batch;
  cudaStream_t s = ctx->stream;
  RCWA_CUDA_TRY(cudaMemcpyAsync(dA, A, na * batch * 16, cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(dB, B, nb * batch * 16, cudaMemcpyHostToDevice, s));
  ZGemm g;
  g.m = m; g.n = n; g.k = k; g.batch = batch;
  g.A = dA; g.lda = m; g.sA = (long long)na;
  g.B = dB; g.ldb = k; g.sB = (long long)nb;
  g.C = dC; g.ldc = m; g.sC = (long long)nc;
  g.tc = kind;
  g.digits = ctx->oz_digits;
  g.ws = (char*)ctx->ws + base;
  g.ws_bytes = wsb;
  // the tensor-core kernels of both precisions (the int8 / TF32 ones and the
  // TMA-fed FP64 one) set this flag when a bounded barrier wait runs out
  int* terr = tc_error_flag();
  if (g.tc && !terr) {
    set_last_error("tensor-core GEMM: device flag unavailable");
    return RCWA_ERR_CUDA;
  }
  if (terr) RCWA_CUDA_TRY(cudaMemsetAsync(terr, 0, sizeof(int), s));
  if ((rc = zgemm(s, g))) return rc;
  RCWA_CUDA_TRY(cudaMemcpyAsync(C, dC, nc * batch * 16, cudaMemcpyDeviceToHost, s));
  int herr = 0;
  if (terr) RCWA_CUDA_TRY(cudaMemcpyAsync(&herr, terr, sizeof(int), cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) {
    set_last_error("tensor-core GEMM: a bounded wait on a tile barrier expired");
    return RCWA_ERR_CUDA;
  }
  return RCWA_OK;
}

int rcwa_gemm_device(rcwa_context* ctx, int m, int n, int k, int batch, rcwa_complex alpha,
                     const rcwa_complex* A, const rcwa_complex* B, rcwa_complex beta, rcwa_complex* C,
                     int precision) {
  CHECK_ARG(ctx && A && B && C && m > 0 && n > 0 && k > 0 && batch > 0, "bad argument");
  CHECK_ARG(precision == RCWA_PREC_FP64 || precision == RCWA_PREC_MIXED, "unknown precision mode");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const int kind = precision != RCWA_PREC_MIXED ? 0 : (ctx->mixed_stages & RCWA_MIXED_GEMM_TF32) ? TC_TF32 : TC_INT8;
  const size_t wsb = kind == TC_INT8 ? zgemm_oz_ws_bytes(m, n, k, batch, ctx->oz_digits) : 0;
  int rc = ctx_reserve(ctx, wsb + 1024);
  if (rc) return rc;
  ZGemm g;
  g.m = m; g.n = n; g.k = k; g.batch = batch;
  g.A = (const double2*)A; g.lda = m; g.sA = (long long)m * k;
  g.B = (const double2*)B; g.ldb = k; g.sB = (long long)k * n;
  g.C = (double2*)C; g.ldc = m; g.sC = (long long)m * n;
  g.alpha = make_double2(alpha.re, alpha.im);
  g.beta = make_double2(beta.re, beta.im);
  g.tc = kind;
  g.digits = ctx->oz_digits;
  g.ws = ctx->ws;
  g.ws_bytes = wsb;
  return zgemm(ctx->stream, g);
}

int rcwa_gemm_ex(rcwa_context* ctx, int opa, int opb, int m, int n, int k, int batch,
                 rcwa_complex alpha, const rcwa_complex* A, const rcwa_complex* B, rcwa_complex beta,
                 rcwa_complex* C) {
  CHECK_ARG(ctx && A && B && C && m > 0 && n > 0 && k > 0 && batch > 0, "bad argument");
  CHECK_ARG((opa == 0 || opa == 1) && (opb == 0 || opb == 1), "op must be 0 or 1");
  RCWA_CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t na = (size_t)m * k, nb = (size_t)k * n, nc = (size_t)m * n;
  int rc = ctx_reserve(ctx, (na + nb + nc) * batch * 16 + 1024);
  if (rc) return rc;
  double2* dA = (double2*)ctx->ws;
  double2* dB = dA + na * batch;
  double2* dC = dB + nb * batch;
  cudaStream_t s = ctx->stream;
  RCWA_CUDA_TRY(cudaMemcpyAsync(dA, A, na * batch * 16, cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(dB, B, nb * batch * 16, cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(dC, C, nc * batch * 16, cudaMemcpyHostToDevice, s));
  ZGemm g;
  g.m = m; g.n = n; g.k = k; g.batch = batch;
  g.alpha = make_double2(alpha.re, alpha.im);
  g.beta = make_double2(beta.re, beta.im);
  g.A = dA; g.lda = opa ? k : m; g.sA = (long long)na; g.opA = opa;
  g.B = dB; g.ldb = opb ? n : k; g.sB = (long long)nb; g.opB = opb;
  g.C = dC; g.ldc = m; g.sC = (long long)nc;
  if ((rc = zgemm(s, g))) return rc;
  RCWA_CUDA_TRY(cudaMemcpyAsync(C, dC, nc * batch * 16, cudaMemcpyDeviceToHost, s));
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  return RCWA_OK;
}

}  // extern "C"
