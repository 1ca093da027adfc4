// Solve orchestration: the reference's main() sequence (main.cpp:111-191)
// re-planned for a batch of sources on one device.
//
//   geometry (once per stack):  ConvMat of every layer's er/ur grid
//                               (main.cpp:125-138) and, for patterned layers,
//                               erc^-1 / urc^-1 (the LU of rcwa.cpp:267-281
//                               is source independent, so it is hoisted).
//   per chunk of sources:       wave vectors + gap (rcwa.cpp:85-234), then for
//                               every layer its S-matrix and the star product
//                               into S_device (main.cpp:146-164), the port
//                               S-matrices and the two global star products
//                               (main.cpp:166-170), and the efficiencies
//                               (main.cpp:182-191).
// Every dense step is a batched kernel over the chunk (one GEMM / LU / eig
// launch covers all sources), so the launch count is independent of the
// number of sources.
#include <algorithm>
#include <cstring>

#include <map>
#include <tuple>

#include "solver.cuh"

namespace rcwa {

int ctx_reserve(rcwa_context* ctx, size_t bytes) {
  if (bytes <= ctx->ws_bytes) return RCWA_OK;
  if (ctx->ws) {
    RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RCWA_CUDA_TRY(cudaFree(ctx->ws));
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
  }
  cudaError_t e = cudaMalloc(&ctx->ws, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error("workspace allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    ctx->ws = nullptr;
    return RCWA_ERR_NOMEM;
  }
  ctx->ws_bytes = bytes;
  return RCWA_OK;
}

int ctx_pinned(rcwa_context* ctx, size_t bytes) {
  if (bytes <= ctx->pinned_bytes) return RCWA_OK;
  if (ctx->pinned) {
    RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RCWA_CUDA_TRY(cudaFreeHost(ctx->pinned));
    ctx->pinned = nullptr;
  }
  RCWA_CUDA_TRY(cudaMallocHost(&ctx->pinned, bytes));
  ctx->pinned_bytes = bytes;
  return RCWA_OK;
}

static ModeDims dims_of(const rcwa_params* p) {
  ModeDims d;
  d.nxh = p->nx_harmonics;
  d.nyh = p->ny_harmonics;
  d.P = 2 * d.nxh + 1;
  d.Q = 2 * d.nyh + 1;
  d.N = d.P * d.Q;
  d.n = 2 * d.N;
  return d;
}

static double2 c2(const rcwa_complex& c) { return make_double2(c.re, c.im); }

void geometry_free(rcwa_geometry* g) {
  if (!g) return;
  const cudaStream_t s = g->ctx ? g->ctx->stream : nullptr;
  if (g->erc) cudaFreeAsync(g->erc, s);
  if (g->urc) cudaFreeAsync(g->urc, s);
  if (g->einv) cudaFreeAsync(g->einv, s);
  if (g->uinv) cudaFreeAsync(g->uinv, s);
  if (g->li) cudaFreeAsync(g->li, s);
  g->erc = g->urc = g->einv = g->uinv = g->li = nullptr;
}

int geometry_build(rcwa_context* ctx, rcwa_geometry* g, const rcwa_stack* st,
                   const rcwa_params* p, int on_device, unsigned opts) {
  cudaStream_t s = ctx->stream;
  const ModeDims d = dims_of(p);
  g->ctx = ctx;
  g->d = d;
  g->nl = st->num_layers;
  g->nx = st->nx;
  g->ny = st->ny;
  g->lx = st->lx;
  g->ly = st->ly;
  g->er_ref = c2(p->er_ref);
  g->ur_ref = c2(p->ur_ref);
  g->er_trn = c2(p->er_trn);
  g->ur_trn = c2(p->ur_trn);
  const int nl = st->num_layers;
  const size_t G = (size_t)st->nx * st->ny;
  g->t.assign(nl, 0.0);
  g->uniform.assign(nl, 0);
  g->ueps.assign(nl, make_double2(0, 0));
  g->umu.assign(nl, make_double2(0, 0));
  const size_t NN = (size_t)d.N * d.N;

  // device copies of the grids (host input) or direct use (device input)
  const double2* der = nullptr;
  const double2* dur = nullptr;
  double2* staging = nullptr;
  if (on_device) {
    der = (const double2*)st->er;
    dur = (const double2*)st->ur;
    RCWA_CUDA_TRY(cudaMemcpyAsync(g->t.data(), st->t, nl * sizeof(double), cudaMemcpyDeviceToHost, s));
  } else {
    std::memcpy(g->t.data(), st->t, nl * sizeof(double));
  }

  // workspace: staging grids (host case) + convmat scratch + augmented [erc | I]
  const size_t conv_scr = convmat_scratch_bytes(nl, st->nx, st->ny, d);
  const size_t stage_b = on_device ? 0 : 2 * (size_t)nl * G * sizeof(double2);
  const size_t aug_b = (size_t)2 * nl * 2 * NN * sizeof(double2);
  const size_t piv_b = (size_t)2 * nl * d.N * sizeof(int);
  const size_t flags_b = 16 * (size_t)nl + 256;
  int rc = ctx_reserve(ctx, stage_b + conv_scr + aug_b + piv_b + flags_b + 4096);
  if (rc) return rc;
  char* w = (char*)ctx->ws;
  auto take = [&](size_t b) {
    char* q = w;
    w += (b + 255) & ~(size_t)255;
    return q;
  };
  if (!on_device) {
    staging = (double2*)take(stage_b);
    RCWA_CUDA_TRY(cudaMemcpyAsync(staging, st->er, nl * G * sizeof(double2), cudaMemcpyHostToDevice, s));
    RCWA_CUDA_TRY(cudaMemcpyAsync(staging + nl * G, st->ur, nl * G * sizeof(double2),
                                  cudaMemcpyHostToDevice, s));
    der = staging;
    dur = staging + nl * G;
  }
  double2* scr = (double2*)take(conv_scr);
  double2* aug = (double2*)take(aug_b);
  int* piv = (int*)take(piv_b);
  int* flags = (int*)take(flags_b);

  // uniform layers: both er and ur constant over the grid
  {
    RCWA_CUDA_TRY(cudaMemsetAsync(flags, 0, 2 * nl * sizeof(int), s));
    for (int l = 0; l < nl; ++l) {
      rc = any_nonuniform(s, der + l * G, G, flags + 2 * l);
      if (rc) return rc;
      rc = any_nonuniform(s, dur + l * G, G, flags + 2 * l + 1);
      if (rc) return rc;
    }
    std::vector<int> hf(2 * nl);
    std::vector<double2> v0(2 * nl);
    RCWA_CUDA_TRY(cudaMemcpyAsync(hf.data(), flags, 2 * nl * sizeof(int), cudaMemcpyDeviceToHost, s));
    for (int l = 0; l < nl; ++l) {
      RCWA_CUDA_TRY(cudaMemcpyAsync(&v0[2 * l], der + l * G, sizeof(double2), cudaMemcpyDeviceToHost, s));
      RCWA_CUDA_TRY(cudaMemcpyAsync(&v0[2 * l + 1], dur + l * G, sizeof(double2), cudaMemcpyDeviceToHost, s));
    }
    RCWA_CUDA_TRY(cudaStreamSynchronize(s));
    for (int l = 0; l < nl; ++l) {
      g->uniform[l] = (hf[2 * l] == 0 && hf[2 * l + 1] == 0) ? 1 : 0;
      g->ueps[l] = v0[2 * l];
      g->umu[l] = v0[2 * l + 1];
    }
  }

  geometry_free(g);
  RCWA_CUDA_TRY(cudaMallocAsync((void**)&g->erc, nl * NN * sizeof(double2), s));
  RCWA_CUDA_TRY(cudaMallocAsync((void**)&g->urc, nl * NN * sizeof(double2), s));
  RCWA_CUDA_TRY(cudaMallocAsync((void**)&g->einv, nl * NN * sizeof(double2), s));
  RCWA_CUDA_TRY(cudaMallocAsync((void**)&g->uinv, nl * NN * sizeof(double2), s));
  // ConvMat for er and ur of every layer (main.cpp:126-138)
  rc = convmat(s, der, nl, st->nx, st->ny, d, g->erc, scr);
  if (rc) return rc;
  rc = convmat(s, dur, nl, st->nx, st->ny, d, g->urc, scr);
  if (rc) return rc;
  // erc^-1 and urc^-1 of patterned layers: [erc | I] -> [U | erc^-1]
  std::vector<int> pat;
  for (int l = 0; l < nl; ++l)
    if (!g->uniform[l]) pat.push_back(l);
  const int np = (int)pat.size();
  if (np > 0) {
    const long long s2 = 2 * (long long)NN;
    for (int k = 0; k < np; ++k) {
      RCWA_CUDA_TRY(cudaMemcpyAsync(aug + k * s2, g->erc + pat[k] * NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
      RCWA_CUDA_TRY(cudaMemcpyAsync(aug + (np + k) * s2, g->urc + pat[k] * NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
    }
    rc = set_identity(s, aug, d.N, d.N, s2, 2 * d.N, d.N, 2 * np, make_double2(1.0, 0.0));
    if (rc) return rc;
    uint32_t* gst = (uint32_t*)(flags + 2 * nl);
    RCWA_CUDA_TRY(cudaMemsetAsync(gst, 0, 2 * np * sizeof(uint32_t), s));
    rc = zgesv(s, d.N, d.N, aug, d.N, s2, 2 * np, piv, gst);
    if (rc) return rc;
    for (int k = 0; k < np; ++k) {
      RCWA_CUDA_TRY(cudaMemcpyAsync(g->einv + pat[k] * NN, aug + k * s2 + NN, NN * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
      RCWA_CUDA_TRY(cudaMemcpyAsync(g->uinv + pat[k] * NN, aug + (np + k) * s2 + NN,
                                    NN * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    }
  }
  if ((opts & RCWA_GEOM_LI_RULE) && np > 0) {
    // eps_xx, eps_yy, mu_xx, mu_yy of every layer (uniform layers never read them)
    const size_t m = (size_t)nl * NN;
    RCWA_CUDA_TRY(cudaMallocAsync((void**)&g->li, 4 * m * sizeof(double2), s));
    char* lscr = nullptr;
    const size_t lb = li_convmat_scratch_bytes(nl, st->nx, st->ny, d);
    RCWA_CUDA_TRY(cudaMallocAsync((void**)&lscr, lb + 256, s));
    int* bad = (int*)(lscr + lb);
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), s);
    for (int k = 0; k < 4 && !rc && e == cudaSuccess; ++k)
      rc = li_convmat(s, k < 2 ? der : dur, nl, st->nx, st->ny, d, k & 1, g->li + k * m, lscr, bad);
    int hbad = 0;
    if (!rc && e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(lscr, s);
    if (rc) return rc;
    if (e != cudaSuccess) {
      set_last_error("Li rule: %s", cudaGetErrorString(e));
      return RCWA_ERR_CUDA;
    }
    if (hbad) {
      set_last_error(hbad & 1 ? "Li rule: a layer grid holds a zero or non-finite permittivity / permeability"
                              : "Li rule: singular Toeplitz matrix of 1/eps along a grid line");
      return RCWA_ERR_NUMERIC;
    }
  }
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  return RCWA_OK;
}

int active_ir_sweeps(const rcwa_context* ctx) {
  return (ctx->tc & (RCWA_MIXED_LAYER_LU | RCWA_MIXED_STAR_LU)) ? ctx->ir_sweeps : 0;
}

static bool int8_gemms(const rcwa_context* ctx) {
  return (ctx->tc & (RCWA_MIXED_LAYER_GEMM | RCWA_MIXED_STAR_GEMM)) && !(ctx->tc & RCWA_MIXED_GEMM_TF32);
}

void set_gemm_kind(const rcwa_context* ctx, unsigned stage, ZGemm& g) {
  g.tc = 0;
  g.ws = nullptr;
  g.ws_bytes = 0;
  if (!(ctx->tc & stage)) return;
  if (ctx->tc & RCWA_MIXED_GEMM_TF32) {
    g.tc = TC_TF32;
    return;
  }
  // the int8-slice kernel pays off on large products only: its 128-row
  // tiles and split passes are mostly waste below a few hundred rows, where
  // the FP64 kernel is both faster and exact
  constexpr int kInt8MinMN = 256;
  if (g.m < kInt8MinMN || g.n < kInt8MinMN || g.k < kInt8MinMN) return;
  g.tc = TC_INT8;
  g.digits = ctx->oz_digits;
  g.ws = ctx->ozws;
  g.ws_bytes = ctx->ozws_bytes;
}

// One batched solve of the S-matrix algebra: FP64 LU, or -- when `stage` runs
// mixed in this solve -- FP32 LU with FP64 refinement in the chunk's
// refinement workspace.
static int lu_stage(rcwa_context* ctx, unsigned stage, int n, int nrhs, double2* M, int ld,
                    long long stride, int batch, int* piv, uint32_t* status) {
  if (!(ctx->tc & stage)) return zgesv(ctx->stream, n, nrhs, M, ld, stride, batch, piv, status);
  const int r8 = (ctx->tc & RCWA_MIXED_REFINE_INT8) ? 1 : 0;
  const size_t need = zgesv_ir_ws_bytes(n, nrhs, batch, ctx->ir_sweeps, r8);
  if (!ctx->irws || need > ctx->irws_bytes) {
    set_last_error("internal: refinement workspace of %zu bytes, %zu needed", ctx->irws_bytes, need);
    return RCWA_ERR_INVALID;
  }
  return zgesv_ir(ctx->stream, n, nrhs, M, ld, stride, batch, piv, status, ctx->irws, ctx->ir_sweeps, r8);
}

// ---------------------------------------------------------------------------
// Redheffer star product A <- A (x) B (rcwa.cpp:588-615), batched.
//   augFG holds two stacked batches of n x 3n augmented systems:
//   [I - B11 A22 | B11 | B12] and [I - A22 B11 | A21 | A22].
// The new S12 is written into `tmp` and the pointers are swapped.
// ---------------------------------------------------------------------------
int star_product(rcwa_context* ctx, int B, int n, SMat& A, const SMat& Bm, double2*& tmp,
                 double2* augFG, int* piv, uint32_t* status) {
  cudaStream_t s = ctx->stream;
  const long long nn = (long long)n * n;
  const long long s3 = 3 * nn;
  double2* augF = augFG;
  double2* augG = augFG + (long long)B * s3;
  int rc;
  rc = set_identity(s, augF, n, n, s3, 3 * n, 0, B, make_double2(1, 0));
  if (rc) return rc;
  rc = set_identity(s, augG, n, n, s3, 3 * n, 0, B, make_double2(1, 0));
  if (rc) return rc;
  auto gemm = [&](double2* C, long long sC, const double2* X, long long sX, const double2* Y,
                  long long sY, double2 alpha, double2 beta) {
    ZGemm g;
    g.m = n; g.n = n; g.k = n;
    g.alpha = alpha; g.beta = beta;
    g.A = X; g.lda = n; g.sA = sX;
    g.B = Y; g.ldb = n; g.sB = sY;
    g.C = C; g.ldc = n; g.sC = sC;
    g.batch = B;
    set_gemm_kind(ctx, RCWA_MIXED_STAR_GEMM, g);
    return zgemm(s, g);
  };
  const double2 one = make_double2(1, 0), mone = make_double2(-1, 0), zero = make_double2(0, 0);
  // F = I - B11 A22 (:602), G = I - A22 B11 (:603)
  if ((rc = gemm(augF, s3, Bm.p[0], Bm.s[0], A.p[3], A.s[3], mone, one))) return rc;
  if ((rc = gemm(augG, s3, A.p[3], A.s[3], Bm.p[0], Bm.s[0], mone, one))) return rc;
  if ((rc = copy_blocks(s, augF + nn, s3, Bm.p[0], Bm.s[0], nn, B))) return rc;
  if ((rc = copy_blocks(s, augF + 2 * nn, s3, Bm.p[1], Bm.s[1], nn, B))) return rc;
  if ((rc = copy_blocks(s, augG + nn, s3, A.p[2], A.s[2], nn, B))) return rc;
  if ((rc = copy_blocks(s, augG + 2 * nn, s3, A.p[3], A.s[3], nn, B))) return rc;
  // F^-1 [B11 B12], G^-1 [A21 A22] (:605-611), both systems in one batch
  if ((rc = lu_stage(ctx, RCWA_MIXED_STAR_LU, n, 2 * n, augFG, n, s3, 2 * B, piv, status))) return rc;
  // note: status is indexed per system; the caller ORs the two halves.
  const double2* X1 = augF + nn;      // F^-1 B11
  const double2* X2 = augF + 2 * nn;  // F^-1 B12
  const double2* Y1 = augG + nn;      // G^-1 A21
  const double2* Y2 = augG + 2 * nn;  // G^-1 A22
  // S11 = A11 + A12 (F^-1 B11) A21 (:608)
  if ((rc = gemm(tmp, nn, X1, s3, A.p[2], A.s[2], one, zero))) return rc;
  if ((rc = gemm(A.p[0], A.s[0], A.p[1], A.s[1], tmp, nn, one, one))) return rc;
  // S21 = B21 (G^-1 A21) (:610) -- A21 is no longer needed
  if ((rc = gemm(A.p[2], A.s[2], Bm.p[2], Bm.s[2], Y1, s3, one, zero))) return rc;
  // S22 = B22 + B21 (G^-1 A22) B12 (:611) -- A22 was copied into augG
  if ((rc = gemm(tmp, nn, Y2, s3, Bm.p[1], Bm.s[1], one, zero))) return rc;
  if ((rc = copy_blocks(s, A.p[3], A.s[3], Bm.p[3], Bm.s[3], nn, B))) return rc;
  if ((rc = gemm(A.p[3], A.s[3], Bm.p[2], Bm.s[2], tmp, nn, one, one))) return rc;
  // S12 = A12 (F^-1 B12) (:609) into tmp, then swap
  if ((rc = gemm(tmp, nn, A.p[1], A.s[1], X2, s3, one, zero))) return rc;
  std::swap(A.p[1], tmp);
  A.s[1] = nn;
  return RCWA_OK;
}

// ---------------------------------------------------------------------------
// workspace plan of one sweep chunk (units: n x n complex blocks per source)
// ---------------------------------------------------------------------------
namespace {
struct Plan {
  int B;
  int n, N;
  // n^2-strided blocks
  double2* SD[4];
  double2* tmp;
  double2* s0;
  double2* s1;
  double2* s2;
  double2* s3;
  double2* pbd;     // [B] x 32N: BD reflection (16N) then transmission (16N) S-matrix
  double2* lbd;     // [B] x 8N: BD S11, S12 of a uniform layer
  // augmented
  double2* augWV;   // [2B] x 2n^2 : [W | I] then [V | I]
  double2* augA;    // [B] x 2n^2
  double2* augD;    // [B] x 3n^2
  double2* augFG;   // [2B] x 3n^2
  double2* eigws;   // zeig workspace for np * B matrices
  int np;           // patterned layers the plan holds eigen-decompositions for
  double2* OmA;     // [np][B] n x n: Omega^2 (destroyed by the eigensolver)
  double2* Wst;     // [np][B] n x n: eigenvectors W
  double2* L2st;    // [np][B][n]: eigenvalues lambda^2
  uint32_t* est;    // [np][B] eigensolver status
  double2* lam2;    // [B][n]
  double2* lam;     // [B][n]
  double2* ilam;    // [B][n]
  double2* X;       // [B][n]
  WaveVecs wv;
  SourceDev* src;   // [B]
  uint32_t* st;     // [3B] scratch status (per system)
  int* piv;         // [2B][n]
};

constexpr int kBlocksPerSource = 4 + 1 + 4 + 4 + 2 + 3 + 6;  // SD,tmp,s0-3,augWV,augA,augD,augFG

// ir > 0: room for the refinement workspace of the largest mixed-precision
// solve of a chunk (the star product's 2B systems with 2n right-hand sides)
size_t plan_bytes(const ModeDims& d, int B, int np, int ir = 0, bool oz = false) {
  const size_t nn = (size_t)d.n * d.n;
  const int ne = np > 0 ? np : 1;
  size_t b = (size_t)B * kBlocksPerSource * nn * sizeof(double2);
  b += (size_t)B * 40 * d.N * sizeof(double2);                // pbd, lbd
  b += zeig_workspace_bytes(d.n, ne * B);
  b += (size_t)ne * B * (2 * nn + d.n) * sizeof(double2) + (size_t)ne * B * sizeof(uint32_t) + 4 * 256;
  b += (size_t)B * 4 * d.n * sizeof(double2);                 // lam2, lam, ilam, X
  b += (size_t)B * (4 * d.N + 4 * d.N + 4) * sizeof(double2); // Kx Ky Kzr Kzt, V0, kinc
  b += (size_t)B * sizeof(SourceDev) + (size_t)3 * B * sizeof(uint32_t);
  b += (size_t)2 * B * d.n * sizeof(int);
  if (ir > 0) b += zgesv_ir_ws_bytes(d.n, 2 * d.n, 2 * B, ir, 1);
  if (oz) b += zgemm_oz_ws_bytes(d.n, d.n, d.n, B, 6);   // the largest product of a chunk, any digit count
  b += 64 * 256;  // alignment slack
  return (b + 255) & ~(size_t)255;  // callers place further buffers right after the plan
}

int plan_take(rcwa_context* ctx, const ModeDims& d, int B, int np, Plan& pl) {
  const int ir = active_ir_sweeps(ctx);
  const bool oz = int8_gemms(ctx);
  int rc = ctx_reserve(ctx, plan_bytes(d, B, np, ir, oz));
  if (rc) return rc;
  char* w = (char*)ctx->ws;
  auto take = [&](size_t bytes) {
    char* q = w;
    w += (bytes + 255) & ~(size_t)255;
    return q;
  };
  const size_t nn = (size_t)d.n * d.n;
  const size_t blk = (size_t)B * nn * sizeof(double2);
  pl.B = B;
  pl.n = d.n;
  pl.N = d.N;
  for (int k = 0; k < 4; ++k) pl.SD[k] = (double2*)take(blk);
  pl.tmp = (double2*)take(blk);
  pl.s0 = (double2*)take(blk);
  pl.s1 = (double2*)take(blk);
  pl.s2 = (double2*)take(blk);
  pl.s3 = (double2*)take(blk);
  pl.pbd = (double2*)take((size_t)B * 32 * d.N * sizeof(double2));
  pl.lbd = (double2*)take((size_t)B * 8 * d.N * sizeof(double2));
  pl.augWV = (double2*)take(4 * blk);
  pl.augA = (double2*)take(2 * blk);
  pl.augD = (double2*)take(3 * blk);
  pl.augFG = (double2*)take(6 * blk);
  const int ne = np > 0 ? np : 1;
  pl.np = ne;
  pl.eigws = (double2*)take(zeig_workspace_bytes(d.n, ne * B));
  pl.OmA = (double2*)take((size_t)ne * blk);
  pl.Wst = (double2*)take((size_t)ne * blk);
  pl.L2st = (double2*)take((size_t)ne * B * d.n * sizeof(double2));
  pl.est = (uint32_t*)take((size_t)ne * B * sizeof(uint32_t));
  pl.lam2 = (double2*)take((size_t)B * d.n * sizeof(double2));
  pl.lam = (double2*)take((size_t)B * d.n * sizeof(double2));
  pl.ilam = (double2*)take((size_t)B * d.n * sizeof(double2));
  pl.X = (double2*)take((size_t)B * d.n * sizeof(double2));
  pl.wv.Kx = (double2*)take((size_t)B * d.N * sizeof(double2));
  pl.wv.Ky = (double2*)take((size_t)B * d.N * sizeof(double2));
  pl.wv.Kzr = (double2*)take((size_t)B * d.N * sizeof(double2));
  pl.wv.Kzt = (double2*)take((size_t)B * d.N * sizeof(double2));
  pl.wv.V0 = (double2*)take((size_t)B * 4 * d.N * sizeof(double2));
  pl.wv.kinc = (double2*)take((size_t)B * 4 * sizeof(double2));
  pl.src = (SourceDev*)take((size_t)B * sizeof(SourceDev));
  pl.st = (uint32_t*)take((size_t)3 * B * sizeof(uint32_t));
  pl.piv = (int*)take((size_t)2 * B * d.n * sizeof(int));
  ctx->irws = nullptr;
  ctx->irws_bytes = 0;
  if (ir > 0) {
    ctx->irws_bytes = zgesv_ir_ws_bytes(d.n, 2 * d.n, 2 * B, ir, 1);
    ctx->irws = take(ctx->irws_bytes);
  }
  ctx->ozws = nullptr;
  ctx->ozws_bytes = 0;
  if (oz) {
    ctx->ozws_bytes = zgemm_oz_ws_bytes(d.n, d.n, d.n, B, 6);
    ctx->ozws = take(ctx->ozws_bytes);
  }
  return RCWA_OK;
}

__global__ void fold_status_kernel(uint32_t* dst, const uint32_t* a, int B, int k) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  uint32_t v = 0;
  for (int j = 0; j < k; ++j) v |= a[(long long)j * B + b];
  dst[b] |= v;
}

int fold_status(cudaStream_t s, uint32_t* dst, const uint32_t* scratch, int B, int k) {
  fold_status_kernel<<<cdiv_up(B, 128), 128, 0, s>>>(dst, scratch, B, k);
  count_launch();
  RCWA_LAUNCH_CHECK();
  return RCWA_OK;
}

// S-matrix of one patterned layer (rcwa.cpp:254-352) for the chunk.
// Output: S11 at augD[1] (stride 3n^2) and S12 in s2.
// P -> pl.s0, Q -> pl.s1 of patterned layer l (rcwa.cpp:262-286) for B items.
static int layer_pq(cudaStream_t s, const Layers& g, int l, int B, Plan& pl) {
  const long long lo = l * g.s_layer;
  const double2* exx = g.exx ? g.exx + lo : g.erc + lo;
  const double2* eyy = g.eyy ? g.eyy + lo : g.erc + lo;
  const double2* mxx = g.mxx ? g.mxx + lo : g.urc + lo;
  const double2* myy = g.myy ? g.myy + lo : g.urc + lo;
  return assemble_pq(s, B, g.d, exx, eyy, mxx, myy, g.einv + lo, g.uinv + lo, g.s_item, pl.wv,
                     pl.s0, pl.s1);
}

// Omega^2 = P Q of patterned layer l (rcwa.cpp:262-288) for the chunk -> out
// (packed n x n per source).
int layer_omega2(rcwa_context* ctx, const Layers& g, int l, Plan& pl, double2* out) {
  cudaStream_t s = ctx->stream;
  const ModeDims& d = g.d;
  const int B = pl.B, n = d.n;
  const long long nn = (long long)n * n;
  int rc;
  if ((rc = layer_pq(s, g, l, B, pl))) return rc;
  ZGemm gm;
  gm.m = n; gm.n = n; gm.k = n; gm.batch = B;
  gm.A = pl.s0; gm.lda = n; gm.sA = nn;
  gm.B = pl.s1; gm.ldb = n; gm.sB = nn;
  gm.C = out; gm.ldc = n; gm.sC = nn;
  return zgemm(s, gm);
}

// Eigen-decompositions (rcwa.cpp:298-306) of the patterned layers `pat` of the
// chunk, all in ONE batched eigensolver call (more independent matrices per
// launch fill the SMs better than one launch per layer).  Layer pat[k] holds
// the first nb(pat[k]) sources of the chunk; its matrices are packed after
// those of pat[0..k): W at pl.Wst + (off_k + b) n^2, lambda^2 at
// pl.L2st + (off_k + b) n, off_k = sum of the earlier layers' counts.
int eig_layers(rcwa_context* ctx, const Layers& g, const std::vector<int>& pat, Plan& pl,
               uint32_t* status) {
  cudaStream_t s = ctx->stream;
  const int n = g.d.n, np = (int)pat.size();
  long long total = 0;
  for (int k = 0; k < np; ++k) total += g.items(pat[k], pl.B);
  if (total == 0) return RCWA_OK;
  if (total > (long long)pl.np * pl.B) {
    set_last_error("internal: plan sized for %d x %d layer eigenproblems, %lld needed", pl.np, pl.B, total);
    return RCWA_ERR_INVALID;
  }
  const long long nn = (long long)n * n;
  int rc;
  long long off = 0;
  for (int k = 0; k < np; ++k) {
    Plan plk = pl;
    plk.B = g.items(pat[k], pl.B);
    if (plk.B == 0) continue;
    if ((rc = layer_omega2(ctx, g, pat[k], plk, pl.OmA + off * nn))) return rc;
    off += plk.B;
  }
  RCWA_CUDA_TRY(cudaMemsetAsync(pl.est, 0, (size_t)total * sizeof(uint32_t), s));
  if ((rc = zeig(s, n, (int)total, pl.OmA, n, nn, pl.Wst, nn, pl.L2st, n, pl.est, pl.eigws))) return rc;
  off = 0;
  for (int k = 0; k < np; ++k) {
    const int Bl = g.items(pat[k], pl.B);
    if (Bl == 0) continue;
    if ((rc = fold_status(s, status, pl.est + off, Bl, 1))) return rc;
    off += Bl;
  }
  return RCWA_OK;
}

// S-matrix of one patterned layer (rcwa.cpp:254-352) for the chunk, from its
// eigen-decomposition Wl (packed n x n per source) and lam2l (n per source).
// Output: S11 at augD[1] (stride 3n^2) and S12 at augD[2].
int patterned_layer(rcwa_context* ctx, const Layers& g, int l, Plan& pl, const double2* Wl,
                    const double2* lam2l, uint32_t* status) {
  cudaStream_t s = ctx->stream;
  const ModeDims& d = g.d;
  const int B = pl.B, n = d.n;
  const long long nn = (long long)n * n;
  const long long s2 = 2 * nn, s3 = 3 * nn;
  const double2 one = make_double2(1, 0), mone = make_double2(-1, 0), zero = make_double2(0, 0);
  int rc;
  // Q_i (:280-286) again (P is not needed past Omega^2)
  if ((rc = layer_pq(s, g, l, B, pl))) return rc;
  // W into the first half of [W | I]
  if ((rc = copy_blocks(s, pl.augWV, s2, Wl, nn, nn, B))) return rc;
  ZGemm gm;
  // lambda, 1/lambda, X (:317, :339)
  if ((rc = layer_modes(s, B, n, lam2l, pl.wv.kinc, g.t ? g.t[l] : 0.0, g.t_item ? g.t_item + l : nullptr,
                        g.nl, pl.lam, pl.ilam, pl.X)))
    return rc;
  // V = Q W lambda^-1 (:326-330) into the first half of [V | I]
  double2* augV = pl.augWV + (long long)B * s2;
  gm = ZGemm();
  gm.m = n; gm.n = n; gm.k = n; gm.batch = B;
  gm.A = pl.s1; gm.lda = n; gm.sA = nn;
  gm.B = pl.augWV; gm.ldb = n; gm.sB = s2;
  gm.C = augV; gm.ldc = n; gm.sC = s2;
  gm.dr = pl.ilam; gm.sdr = n;
  set_gemm_kind(ctx, RCWA_MIXED_LAYER_GEMM, gm);
  if ((rc = zgemm(s, gm))) return rc;
  // W^-1, V^-1 (:335-336), one batched solve for both
  if ((rc = set_identity(s, pl.augWV, n, n, s2, 2 * n, n, 2 * B, one))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(pl.st, 0, 3 * B * sizeof(uint32_t), s));
  if ((rc = lu_stage(ctx, RCWA_MIXED_LAYER_LU, n, n, pl.augWV, n, s2, 2 * B, pl.piv, pl.st))) return rc;
  if ((rc = fold_status(s, status, pl.st, B, 2))) return rc;
  // A = W^-1 W0 + V^-1 V0 -> s1, B -> s0 (:337-338)
  if ((rc = assemble_ab(s, B, d, pl.augWV + nn, s2, augV + nn, s2, pl.wv.V0, pl.s1, pl.s0))) return rc;
  // A^-1 via [A | I]
  if ((rc = copy_blocks(s, pl.augA, s2, pl.s1, nn, nn, B))) return rc;
  if ((rc = set_identity(s, pl.augA, n, n, s2, 2 * n, n, B, one))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(pl.st, 0, 3 * B * sizeof(uint32_t), s));
  if ((rc = lu_stage(ctx, RCWA_MIXED_LAYER_LU, n, n, pl.augA, n, s2, B, pl.piv, pl.st))) return rc;
  if ((rc = fold_status(s, status, pl.st, B, 1))) return rc;
  const double2* Ai = pl.augA + nn;
  // T1 = B A^-1 X -> s2   (X diag: column scaling)
  gm = ZGemm();
  gm.m = n; gm.n = n; gm.k = n; gm.batch = B;
  gm.A = pl.s0; gm.lda = n; gm.sA = nn;
  gm.B = Ai; gm.ldb = n; gm.sB = s2;
  gm.C = pl.s2; gm.ldc = n; gm.sC = nn;
  gm.dr = pl.X; gm.sdr = n;
  set_gemm_kind(ctx, RCWA_MIXED_LAYER_GEMM, gm);
  if ((rc = zgemm(s, gm))) return rc;
  // D = A - X T1 B -> augD[0] (:346)
  if ((rc = copy_blocks(s, pl.augD, s3, pl.s1, nn, nn, B))) return rc;
  gm = ZGemm();
  gm.m = n; gm.n = n; gm.k = n; gm.batch = B;
  gm.alpha = mone; gm.beta = one;
  gm.A = pl.s2; gm.lda = n; gm.sA = nn;
  gm.B = pl.s0; gm.ldb = n; gm.sB = nn;
  gm.C = pl.augD; gm.ldc = n; gm.sC = s3;
  gm.dl = pl.X; gm.sdl = n;
  set_gemm_kind(ctx, RCWA_MIXED_LAYER_GEMM, gm);
  if ((rc = zgemm(s, gm))) return rc;
  // R1 = X T1 A - B -> augD[1] (:347)
  if ((rc = copy_blocks(s, pl.augD + nn, s3, pl.s0, nn, nn, B))) return rc;
  gm.alpha = one; gm.beta = mone;
  gm.B = pl.s1;
  gm.C = pl.augD + nn;
  set_gemm_kind(ctx, RCWA_MIXED_LAYER_GEMM, gm);
  if ((rc = zgemm(s, gm))) return rc;
  // T3 = A^-1 B -> s3 ; R2 = A - B T3 -> s1 (in place) (:348)
  gm = ZGemm();
  gm.m = n; gm.n = n; gm.k = n; gm.batch = B;
  gm.A = Ai; gm.lda = n; gm.sA = s2;
  gm.B = pl.s0; gm.ldb = n; gm.sB = nn;
  gm.C = pl.s3; gm.ldc = n; gm.sC = nn;
  set_gemm_kind(ctx, RCWA_MIXED_LAYER_GEMM, gm);
  if ((rc = zgemm(s, gm))) return rc;
  gm.alpha = mone; gm.beta = one;
  gm.A = pl.s0; gm.sA = nn;
  gm.B = pl.s3; gm.sB = nn;
  gm.C = pl.s1;
  set_gemm_kind(ctx, RCWA_MIXED_LAYER_GEMM, gm);
  if ((rc = zgemm(s, gm))) return rc;
  // X R2 -> augD[2]; then [D | R1 | X R2] -> S11 = D^-1 R1 (:347), S12 = D^-1 X R2 (:348)
  if ((rc = scale_rows(s, pl.s1, n, n, n, nn, pl.X, n, B))) return rc;
  if ((rc = copy_blocks(s, pl.augD + 2 * nn, s3, pl.s1, nn, nn, B))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(pl.st, 0, 3 * B * sizeof(uint32_t), s));
  if ((rc = lu_stage(ctx, RCWA_MIXED_LAYER_LU, n, 2 * n, pl.augD, n, s3, B, pl.piv, pl.st))) return rc;
  (void)zero;
  return fold_status(s, status, pl.st, B, 1);
}

// Star product with a uniform layer whose S-matrix is BD (2x2-block
// diagonal): A <- A (x) L, L11 = L22 = Lbd[0], L12 = L21 = Lbd[1]
// (rcwa.cpp:588-615 with the sparse factors applied in O(n^2)).
//   [I - L11 A22 | L11 A21 | L12] -> X1 = F^-1 L11 A21, X2 = F^-1 L12
//   [I - A22 L11 | A21 | A22]     -> Y1 = G^-1 A21,     Y2 = G^-1 A22
//   S11 = A11 + A12 X1, S12 = A12 X2, S21 = L12 Y1, S22 = L11 + L12 Y2 L12
int star_product_bd(rcwa_context* ctx, int B, const ModeDims& d, SMat& A, const double2* Lbd,
                    long long sL, double2*& tmp, double2* augFG, int* piv, uint32_t* st) {
  cudaStream_t s = ctx->stream;
  const int n = d.n, N = d.N;
  const long long nn = (long long)n * n, s3 = 3 * nn;
  double2* augF = augFG;
  double2* augG = augFG + (long long)B * s3;
  const double2* L11 = Lbd;
  const double2* L12 = Lbd + 4 * N;
  const double2 one = make_double2(1, 0), mone = make_double2(-1, 0), zero = make_double2(0, 0);
  int rc;
  if ((rc = bd_apply(s, 0, N, n, n, L11, sL, A.p[3], n, A.s[3], augF, n, s3, mone, zero, 1, B))) return rc;
  if ((rc = bd_apply(s, 0, N, n, n, L11, sL, A.p[2], n, A.s[2], augF + nn, n, s3, one, zero, 0, B))) return rc;
  if ((rc = bd_dense(s, N, L12, sL, augF + 2 * nn, s3, 0, B))) return rc;
  if ((rc = bd_apply(s, 1, N, n, n, L11, sL, A.p[3], n, A.s[3], augG, n, s3, mone, zero, 1, B))) return rc;
  if ((rc = copy_blocks(s, augG + nn, s3, A.p[2], A.s[2], nn, B))) return rc;
  if ((rc = copy_blocks(s, augG + 2 * nn, s3, A.p[3], A.s[3], nn, B))) return rc;
  if ((rc = lu_stage(ctx, RCWA_MIXED_STAR_LU, n, 2 * n, augFG, n, s3, 2 * B, piv, st))) return rc;
  ZGemm g;
  g.m = n; g.n = n; g.k = n; g.batch = B;
  set_gemm_kind(ctx, RCWA_MIXED_STAR_GEMM, g);
  // S11 = A11 + A12 X1
  g.alpha = one; g.beta = one;
  g.A = A.p[1]; g.lda = n; g.sA = A.s[1];
  g.B = augF + nn; g.ldb = n; g.sB = s3;
  g.C = A.p[0]; g.ldc = n; g.sC = A.s[0];
  if ((rc = zgemm(s, g))) return rc;
  // S12 = A12 X2 -> tmp, swapped in below
  g.beta = zero;
  g.B = augF + 2 * nn;
  g.C = tmp; g.sC = nn;
  if ((rc = zgemm(s, g))) return rc;
  // S21 = L12 Y1 (A21 was copied into augG)
  if ((rc = bd_apply(s, 0, N, n, n, L12, sL, augG + nn, n, s3, A.p[2], n, A.s[2], one, zero, 0, B))) return rc;
  // S22 = L11 + (L12 Y2) L12: L12 Y2 -> augF[0] (F is consumed), then right-apply into A22
  if ((rc = bd_apply(s, 0, N, n, n, L12, sL, augG + 2 * nn, n, s3, augF, n, s3, one, zero, 0, B))) return rc;
  if ((rc = bd_apply(s, 1, N, n, n, L12, sL, augF, n, s3, A.p[3], n, A.s[3], one, zero, 0, B))) return rc;
  if ((rc = bd_dense(s, N, L11, sL, A.p[3], A.s[3], 1, B))) return rc;
  std::swap(A.p[1], tmp);
  A.s[1] = nn;
  return RCWA_OK;
}

// The two source columns of the global S11 and S21 (main.cpp:166-170; only
// columns PQ/2 and PQ/2+PQ reach the fields, rcwa.cpp:512-514, 535, 553):
//   S' = S_ref (x) S_dev, S'' = S' (x) S_trn with S_ref, S_trn in BD form.
//   G1 = I - R22 D11:  [G1 | R22 D12 | R21 E] -> Z2, y
//   S'22 = D22 + D21 Z2,  S'21 E = D21 y
//   F2 = I - T11 S'22: x = F2^-1 T11 S'21 E;  G2 = I - S'22 T11: z = G2^-1 S'21 E
//   S''21 E = T21 z
//   F1 = I - D11 R22:  q = F1^-1 (D11 R21 E + D12 x);  S''11 E = R11 E + R12 q
// Outputs S11E, S21E: n x 2 per source (stride 2n).
int global_columns(rcwa_context* ctx, int B, const ModeDims& d, const SMat& D, const double2* Rbd,
                   const double2* Tbd, long long sP, double2* S11E, double2* S21E,
                   double2* augFG, double2* augWV, double2* augA, double2* s0, double2* s1,
                   int* piv, uint32_t* st, uint32_t* status) {
  cudaStream_t s = ctx->stream;
  const int n = d.n, N = d.N, a = N / 2;
  const long long nn = (long long)n * n, s6 = 6 * nn, s2 = 2 * nn, c2 = 2LL * n;
  const double2 one = make_double2(1, 0), mone = make_double2(-1, 0), zero = make_double2(0, 0);
  const double2 *R11 = Rbd, *R12 = Rbd + 4 * N, *R21 = Rbd + 8 * N, *R22 = Rbd + 12 * N;
  const double2 *T11 = Tbd, *T21 = Tbd + 8 * N;
  int rc;
  auto gemm = [&](int m, int ncol, double2* C, long long sC, const double2* X, long long sX,
                  const double2* Y, long long sY, double2 beta) {
    ZGemm g;
    g.m = m; g.n = ncol; g.k = n; g.batch = B;
    g.beta = beta;
    g.A = X; g.lda = n; g.sA = sX;
    g.B = Y; g.ldb = n; g.sB = sY;
    g.C = C; g.ldc = n; g.sC = sC;
    set_gemm_kind(ctx, RCWA_MIXED_STAR_GEMM, g);
    return zgemm(s, g);
  };
  // [G1 | R22 D12 | R21 E] in augFG (stride 6n^2)
  double2* u = augFG + 2 * nn;
  if ((rc = bd_apply(s, 0, N, n, n, R22, sP, D.p[0], n, D.s[0], augFG, n, s6, mone, zero, 1, B))) return rc;
  if ((rc = bd_apply(s, 0, N, n, n, R22, sP, D.p[1], n, D.s[1], augFG + nn, n, s6, one, zero, 0, B))) return rc;
  if ((rc = bd_cols(s, N, a, R21, sP, u, n, s6, one, zero, B))) return rc;
  // [F1 | D11 R21 E (+ D12 x later)] in augA (stride 2n^2); F1 = I - D11 R22
  if ((rc = bd_apply(s, 1, N, n, n, R22, sP, D.p[0], n, D.s[0], augA, n, s2, mone, zero, 1, B))) return rc;
  if ((rc = gemm(n, 2, augA + nn, s2, D.p[0], D.s[0], u, s6, zero))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, 3 * B * sizeof(uint32_t), s));
  if ((rc = lu_stage(ctx, RCWA_MIXED_STAR_LU, n, n + 2, augFG, n, s6, B, piv, st))) return rc;
  if ((rc = fold_status(s, status, st, B, 1))) return rc;
  // S'22 -> s0, S'21 E -> s1
  if ((rc = copy_blocks(s, s0, nn, D.p[3], D.s[3], nn, B))) return rc;
  if ((rc = gemm(n, n, s0, nn, D.p[2], D.s[2], augFG + nn, s6, one))) return rc;
  if ((rc = gemm(n, 2, s1, nn, D.p[2], D.s[2], u, s6, zero))) return rc;
  // [F2 | T11 S'21E] (systems 0..B-1) and [G2 | S'21E] (systems B..2B-1) in augWV
  double2* augG2 = augWV + (long long)B * s2;
  if ((rc = bd_apply(s, 0, N, n, n, T11, sP, s0, n, nn, augWV, n, s2, mone, zero, 1, B))) return rc;
  if ((rc = bd_apply(s, 0, N, n, 2, T11, sP, s1, n, nn, augWV + nn, n, s2, one, zero, 0, B))) return rc;
  if ((rc = bd_apply(s, 1, N, n, n, T11, sP, s0, n, nn, augG2, n, s2, mone, zero, 1, B))) return rc;
  if ((rc = copy_blocks(s, augG2 + nn, s2, s1, nn, c2, B))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, 3 * B * sizeof(uint32_t), s));
  if ((rc = lu_stage(ctx, RCWA_MIXED_STAR_LU, n, 2, augWV, n, s2, 2 * B, piv, st))) return rc;
  if ((rc = fold_status(s, status, st, B, 2))) return rc;
  // S''21 E = T21 z
  if ((rc = bd_apply(s, 0, N, n, 2, T21, sP, augG2 + nn, n, s2, S21E, n, c2, one, zero, 0, B))) return rc;
  // v = D11 R21 E + D12 x, then q = F1^-1 v
  if ((rc = gemm(n, 2, augA + nn, s2, D.p[1], D.s[1], augWV + nn, s2, one))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, 3 * B * sizeof(uint32_t), s));
  if ((rc = lu_stage(ctx, RCWA_MIXED_STAR_LU, n, 2, augA, n, s2, B, piv, st))) return rc;
  if ((rc = fold_status(s, status, st, B, 1))) return rc;
  // S''11 E = R11 E + R12 q
  if ((rc = bd_cols(s, N, a, R11, sP, S11E, n, c2, one, zero, B))) return rc;
  return bd_apply(s, 0, N, n, 2, R12, sP, augA + nn, n, s2, S11E, n, c2, one, one, 0, B);
}

}  // namespace

size_t sweep_bytes_per_source(const ModeDims& d, int np, int ir_sweeps, bool oz) {
  return plan_bytes(d, 1, np, ir_sweeps, oz);
}

size_t sweep_bytes_per_source(const rcwa_context* ctx, const ModeDims& d, int np) {
  return plan_bytes(d, 1, np, active_ir_sweeps(ctx), int8_gemms(ctx));
}

// The layer set of one geometry, shared by every solve of a sweep.
Layers layers_of(const rcwa_geometry* g) {
  Layers G;
  G.d = g->d;
  G.nl = g->nl;
  G.er_ref = g->er_ref;
  G.ur_ref = g->ur_ref;
  G.er_trn = g->er_trn;
  G.ur_trn = g->ur_trn;
  G.uniform = g->uniform.data();
  G.t = g->t.data();
  G.ueps = g->ueps.data();
  G.umu = g->umu.data();
  G.erc = g->erc;
  G.urc = g->urc;
  G.einv = g->einv;
  G.uinv = g->uinv;
  G.s_layer = (long long)g->d.N * g->d.N;
  if (g->li) {
    const long long m = (long long)g->nl * G.s_layer;
    G.exx = g->li;
    G.eyy = g->li + m;
    G.mxx = g->li + 2 * m;
    G.myy = g->li + 3 * m;
  }
  G.s_item = 0;
  return G;
}

// One chunk of B solves on the layer set g; hsrc: host [B] sources with
// their lattice periods.
int sweep_chunk_layers(rcwa_context* ctx, const Layers& g, const SourceDev* hsrc, int B, double* R,
                       double* T, double* tot, uint32_t* status, const ShareMap* sh) {
  cudaStream_t s = ctx->stream;
  const ModeDims& d = g.d;
  const int n = d.n;
  const long long nn = (long long)n * n, s3 = 3 * nn;
  int np = 0;
  for (int l = 0; l < g.nl; ++l) np += g.uniform[l] ? 0 : 1;
  Plan pl;
  int rc = plan_take(ctx, d, B, np, pl);
  if (rc) return rc;
  // sources -> device (through the pinned staging buffer)
  if ((rc = ctx_pinned(ctx, (size_t)B * sizeof(SourceDev)))) return rc;
  SourceDev* hs = (SourceDev*)ctx->pinned;
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));  // staging buffer reuse
  std::memcpy(hs, hsrc, B * sizeof(SourceDev));
  RCWA_CUDA_TRY(cudaMemcpyAsync(pl.src, hs, B * sizeof(SourceDev), cudaMemcpyHostToDevice, s));
  RCWA_CUDA_TRY(cudaMemsetAsync(status, 0, B * sizeof(uint32_t), s));
  // wave vectors + gap (main.cpp:140-141)
  if ((rc = wave_vectors(s, pl.src, B, d, g.er_ref, g.ur_ref, g.er_trn, g.ur_trn, pl.wv, status)))
    return rc;
  // device S-matrix (main.cpp:143-164)
  SMat dev;
  for (int k = 0; k < 4; ++k) {
    dev.p[k] = pl.SD[k];
    dev.s[k] = nn;
  }
  double2* tmp = pl.tmp;
  const long long sL = 8LL * d.N;     // BD uniform layer: S11 (4N) + S12 (4N) per source
  std::vector<int> pat;
  std::vector<long long> off(g.nl, 0);
  {
    long long o = 0;
    for (int l = 0; l < g.nl; ++l)
      if (!g.uniform[l]) {
        off[l] = o;
        o += g.items(l, B);
        pat.push_back(l);
      }
  }
  if ((rc = eig_layers(ctx, g, pat, pl, status))) return rc;
  // sources without layer 0 (only in batches of stacks of different depth)
  // start from the empty-stack S-matrix (rcwa.cpp:237-250)
  if (g.nl > 0 && g.items(0, B) < B) {
    const int b0 = g.items(0, B), c = B - b0;
    for (int k = 0; k < 4; ++k)
      if ((rc = fill_zero(s, dev.p[k] + (size_t)b0 * nn, (size_t)c * nn))) return rc;
    if ((rc = set_identity(s, dev.p[1] + (size_t)b0 * nn, n, n, nn, n, 0, c, make_double2(1, 0)))) return rc;
    if ((rc = set_identity(s, dev.p[2] + (size_t)b0 * nn, n, n, nn, n, 0, c, make_double2(1, 0)))) return rc;
  }
  for (int l = 0; l < g.nl; ++l) {
    const int Bl = g.items(l, B);   // this layer belongs to sources 0 .. Bl-1
    if (Bl == 0) continue;
    double2* const S12_before = dev.p[1];
    if (g.uniform[l]) {
      if ((rc = uniform_layer(s, Bl, d, g.ueps ? g.ueps[l] : make_double2(1, 0),
                              g.umu ? g.umu[l] : make_double2(1, 0), g.t ? g.t[l] : 0.0,
                              g.ueps_item ? g.ueps_item + l : nullptr, g.umu_item ? g.umu_item + l : nullptr,
                              g.t_item ? g.t_item + l : nullptr, g.nl, pl.wv, pl.lbd, pl.lbd + 4 * d.N, sL, 1)))
        return rc;
      if (l == 0) {
        // S_init (x) S_layer == S_layer exactly (S11 = S22 = 0, S12 = S21 = I)
        if ((rc = bd_dense(s, d.N, pl.lbd, sL, dev.p[0], nn, 0, Bl))) return rc;
        if ((rc = bd_dense(s, d.N, pl.lbd + 4 * d.N, sL, dev.p[1], nn, 0, Bl))) return rc;
        if ((rc = bd_dense(s, d.N, pl.lbd + 4 * d.N, sL, dev.p[2], nn, 0, Bl))) return rc;
        if ((rc = bd_dense(s, d.N, pl.lbd, sL, dev.p[3], nn, 0, Bl))) return rc;
      } else {
        RCWA_CUDA_TRY(cudaMemsetAsync(pl.st, 0, 3 * (size_t)Bl * sizeof(uint32_t), s));
        if ((rc = star_product_bd(ctx, Bl, d, dev, pl.lbd, sL, tmp, pl.augFG, pl.piv, pl.st))) return rc;
        if ((rc = fold_status(s, status, pl.st, Bl, 2))) return rc;
      }
    } else {
      Plan plk = pl;
      plk.B = Bl;
      if ((rc = patterned_layer(ctx, g, l, plk, pl.Wst + off[l] * nn, pl.L2st + off[l] * n, status))) return rc;
      SMat lay;
      lay.p[0] = pl.augD + nn; lay.s[0] = s3;      // S11 = D^-1 R1
      lay.p[1] = pl.augD + 2 * nn; lay.s[1] = s3;  // S12 = D^-1 X R2
      lay.p[2] = lay.p[1]; lay.s[2] = lay.s[1];    // S21 = S12 (:351)
      lay.p[3] = lay.p[0]; lay.s[3] = lay.s[0];    // S22 = S11
      if (l == 0) {
        for (int k = 0; k < 4; ++k)
          if ((rc = copy_blocks(s, dev.p[k], dev.s[k], lay.p[k], lay.s[k], nn, Bl))) return rc;
      } else {
        RCWA_CUDA_TRY(cudaMemsetAsync(pl.st, 0, 3 * (size_t)Bl * sizeof(uint32_t), s));
        if ((rc = star_product(ctx, Bl, n, dev, lay, tmp, pl.augFG, pl.piv, pl.st))) return rc;
        if ((rc = fold_status(s, status, pl.st, Bl, 2))) return rc;
      }
    }
    // the star products leave the new S12 in the former scratch block: carry
    // the S12 of the sources past Bl (which skip this layer) across
    if (Bl < B && dev.p[1] != S12_before)
      if ((rc = copy_blocks(s, dev.p[1] + (size_t)Bl * nn, nn, S12_before + (size_t)Bl * nn, nn, nn, B - Bl)))
        return rc;
  }
  if (g.nl == 0) {
    for (int k = 0; k < 4; ++k) {
      if ((rc = fill_zero(s, dev.p[k], (size_t)B * nn))) return rc;
    }
    if ((rc = set_identity(s, dev.p[1], n, n, nn, n, 0, B, make_double2(1, 0)))) return rc;
    if ((rc = set_identity(s, dev.p[2], n, n, nn, n, 0, B, make_double2(1, 0)))) return rc;
  }
  // S_ref, S_trn in BD form (rcwa.cpp:354-466), then the two source columns of
  // S_ref (x) S_device (x) S_trn (main.cpp:166-170)
  const long long sP = 32LL * d.N;
  double2* Rbd = pl.pbd;
  double2* Tbd = pl.pbd + 16 * d.N;
  if ((rc = port_smatrix(s, B, d, 0, g.er_ref, g.ur_ref, pl.wv, Rbd, Rbd + 4 * d.N, Rbd + 8 * d.N,
                         Rbd + 12 * d.N, sP, 1)))
    return rc;
  if ((rc = port_smatrix(s, B, d, 1, g.er_trn, g.ur_trn, pl.wv, Tbd, Tbd + 4 * d.N, Tbd + 8 * d.N,
                         Tbd + 12 * d.N, sP, 1)))
    return rc;
  double2* S11E = pl.s2;
  double2* S21E = pl.s3;
  if ((rc = global_columns(ctx, B, d, dev, Rbd, Tbd, sP, S11E, S21E, pl.augFG, pl.augWV, pl.augA,
                           pl.s0, pl.s1, pl.piv, pl.st, status)))
    return rc;
  // efficiencies (main.cpp:182-191)
  if (sh)   // sources sharing these solves (polarisation variants)
    return efficiencies(s, sh->n, d, sh->src, g.ur_ref, g.ur_trn, pl.wv, S11E, S21E, 2LL * n, 1, sh->R,
                        sh->T, sh->tot, sh->status, sh->map, sh->oidx, status);
  return efficiencies(s, B, d, pl.src, g.ur_ref, g.ur_trn, pl.wv, S11E, S21E, 2LL * n, 1, R, T,
                      tot, status);
}

int sweep_device(rcwa_context* ctx, const rcwa_geometry* g, const rcwa_source* sources, int B,
                 int precision, double* R, double* T, double* tot, uint32_t* status) {
  if (precision != RCWA_PREC_FP64 && precision != RCWA_PREC_MIXED) {
    set_last_error("unknown precision mode %d", precision);
    return RCWA_ERR_INVALID;
  }
  if (B <= 0) return RCWA_OK;
  int* tc_err = nullptr;
  if (precision == RCWA_PREC_MIXED) {
    tc_err = tc_error_flag();
    if (!tc_err) {
      set_last_error("tensor-core GEMM error flag unavailable on this device");
      return RCWA_ERR_CUDA;
    }
    RCWA_CUDA_TRY(cudaMemsetAsync(tc_err, 0, sizeof(int), ctx->stream));
  }
  struct TcScope {  // the flag never outlives this sweep, also on early return
    rcwa_context* c;
    ~TcScope() { c->tc = 0; }
  } tc_scope{ctx};
  ctx->tc = precision == RCWA_PREC_MIXED ? ctx->mixed_stages : 0u;
  const ModeDims& d = g->d;
  // chunk size from the memory budget
  size_t budget = ctx->mem_budget;
  if (budget == 0) {
    size_t fr = 0, totm = 0;
    RCWA_CUDA_TRY(cudaMemGetInfo(&fr, &totm));
    budget = (size_t)((fr + ctx->ws_bytes) * 0.6);
  }
  int np = 0;
  for (int l = 0; l < g->nl; ++l) np += g->uniform[l] ? 0 : 1;
  const size_t per = sweep_bytes_per_source(ctx, d, np);
  int chunk = (int)std::max<size_t>(1, budget / per);
  chunk = std::min(chunk, B);
  const Layers G = layers_of(g);
  // sources that differ only in polarisation share one solve: the S-matrix
  // and wave vectors depend on (lambda0, theta, phi) alone; only the source
  // vector of the efficiencies (rcwa.cpp:469-523) sees pte/ptm
  std::map<std::tuple<double, double, double>, int> key;
  std::vector<int> uof(B);
  std::vector<int> firsts;
  for (int b = 0; b < B; ++b) {
    const auto k = std::make_tuple(sources[b].lambda0, sources[b].theta, sources[b].phi);
    auto it = key.find(k);
    if (it == key.end()) {
      it = key.emplace(k, (int)firsts.size()).first;
      firsts.push_back(b);
    }
    uof[b] = it->second;
  }
  const int U = (int)firsts.size();
  const long long N = d.N;
  if (U == B) {
    std::vector<SourceDev> hs(chunk);
    for (int b0 = 0; b0 < B; b0 += chunk) {
      const int bc = std::min(chunk, B - b0);
      for (int b = 0; b < bc; ++b) {
        const rcwa_source& q = sources[b0 + b];
        hs[b] = SourceDev{q.lambda0, q.theta, q.phi, q.pte, q.ptm, g->lx, g->ly};
      }
      int rc = sweep_chunk_layers(ctx, G, hs.data(), bc, R + b0 * N, T + b0 * N, tot + 2LL * b0, status + b0);
      if (rc) return rc;
    }
  } else {
    // solves for the U distinct (lambda0, theta, phi); efficiencies for all B
    std::vector<std::vector<int>> members(U);
    for (int b = 0; b < B; ++b) members[uof[b]].push_back(b);
    char* buf = nullptr;
    const size_t bytes = (size_t)B * (sizeof(SourceDev) + 2 * sizeof(int)) + (size_t)U * sizeof(uint32_t) + 1024;
    RCWA_CUDA_TRY(cudaMallocAsync((void**)&buf, bytes, ctx->stream));
    struct Free {
      char* p;
      cudaStream_t s;
      ~Free() { cudaFreeAsync(p, s); }
    } free_buf{buf, ctx->stream};
    SourceDev* esrc = (SourceDev*)buf;
    int* emap = (int*)(esrc + B);
    int* eoidx = emap + B;
    uint32_t* ust = (uint32_t*)(eoidx + B);
    std::vector<std::vector<SourceDev>> keep_src;   // host copies live until the end
    std::vector<std::vector<int>> keep_idx;
    for (int u0 = 0; u0 < U; u0 += chunk) {
      const int uc = std::min(chunk, U - u0);
      std::vector<SourceDev> hs(uc), es;
      std::vector<int> em, eo;
      for (int u = 0; u < uc; ++u) {
        const rcwa_source& q = sources[firsts[u0 + u]];
        hs[u] = SourceDev{q.lambda0, q.theta, q.phi, q.pte, q.ptm, g->lx, g->ly};
        for (int b : members[u0 + u]) {
          const rcwa_source& r = sources[b];
          es.push_back(SourceDev{r.lambda0, r.theta, r.phi, r.pte, r.ptm, g->lx, g->ly});
          em.push_back(u);
          eo.push_back(b);
        }
      }
      const int ne = (int)es.size();
      RCWA_CUDA_TRY(cudaMemcpyAsync(esrc, es.data(), ne * sizeof(SourceDev), cudaMemcpyHostToDevice, ctx->stream));
      RCWA_CUDA_TRY(cudaMemcpyAsync(emap, em.data(), ne * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
      RCWA_CUDA_TRY(cudaMemcpyAsync(eoidx, eo.data(), ne * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
      ShareMap sh;
      sh.n = ne;
      sh.src = esrc;
      sh.map = emap;
      sh.oidx = eoidx;
      sh.R = R;
      sh.T = T;
      sh.tot = tot;
      sh.status = status;
      int rc = sweep_chunk_layers(ctx, G, hs.data(), uc, nullptr, nullptr, nullptr, ust, &sh);
      if (rc) return rc;
      keep_src.push_back(std::move(es));
      keep_idx.push_back(std::move(em));
      keep_idx.push_back(std::move(eo));
      RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));   // the staging arrays are reused
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
  return RCWA_OK;
}

}  // namespace rcwa

// ===========================================================================
// Step-level entry points (one reference function each), single problem.
// ===========================================================================
namespace rcwa {

namespace {
struct Arena {
  char* p;
  char* take(size_t b) {
    char* q = p;
    p += (b + 255) & ~(size_t)255;
    return q;
  }
};
int h2d(rcwa_context* c, void* d, const void* h, size_t b) {
  RCWA_CUDA_TRY(cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, c->stream));
  return RCWA_OK;
}
int d2h(rcwa_context* c, void* h, const void* d, size_t b) {
  RCWA_CUDA_TRY(cudaMemcpyAsync(h, d, b, cudaMemcpyDeviceToHost, c->stream));
  return RCWA_OK;
}
ModeDims dims_n(int N) {
  ModeDims d{};
  d.N = N;
  d.n = 2 * N;
  d.P = N;  // only N / n are used by the per-mode kernels
  d.Q = 1;
  return d;
}
}  // namespace

int step_wave_vectors(rcwa_context* ctx, double lx, double ly, const rcwa_source* src,
                      const rcwa_params* p, double2* kinc, double2* Kx, double2* Ky, double2* Kzr,
                      double2* Kzt, double2* V0d) {
  const ModeDims d = dims_of(p);
  const size_t N = d.N;
  int rc = ctx_reserve(ctx, (8 * N + 4) * 16 + 64 + 8 * 256);
  if (rc) return rc;
  Arena a{(char*)ctx->ws};
  WaveVecs w;
  w.Kx = (double2*)a.take(N * 16);
  w.Ky = (double2*)a.take(N * 16);
  w.Kzr = (double2*)a.take(N * 16);
  w.Kzt = (double2*)a.take(N * 16);
  w.V0 = (double2*)a.take(4 * N * 16);
  w.kinc = (double2*)a.take(4 * 16);
  SourceDev* ds = (SourceDev*)a.take(sizeof(SourceDev));
  uint32_t* st = (uint32_t*)a.take(4);
  SourceDev hs{src->lambda0, src->theta, src->phi, src->pte, src->ptm, lx, ly};
  if ((rc = h2d(ctx, ds, &hs, sizeof(hs)))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, 4, ctx->stream));
  if ((rc = wave_vectors(ctx->stream, ds, 1, d, c2(p->er_ref), c2(p->ur_ref), c2(p->er_trn),
                         c2(p->ur_trn), w, st)))
    return rc;
  if ((rc = d2h(ctx, Kx, w.Kx, N * 16)) || (rc = d2h(ctx, Ky, w.Ky, N * 16)) ||
      (rc = d2h(ctx, Kzr, w.Kzr, N * 16)) || (rc = d2h(ctx, Kzt, w.Kzt, N * 16)) ||
      (rc = d2h(ctx, V0d, w.V0, 4 * N * 16)) || (rc = d2h(ctx, kinc, w.kinc, 4 * 16)))
    return rc;
  RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return RCWA_OK;
}

int step_gap_v0(rcwa_context* ctx, int N, const double2* Kx, const double2* Ky, double2* V0d) {
  int rc = ctx_reserve(ctx, (size_t)6 * N * 16 + 1024);
  if (rc) return rc;
  Arena a{(char*)ctx->ws};
  double2* dKx = (double2*)a.take((size_t)N * 16);
  double2* dKy = (double2*)a.take((size_t)N * 16);
  double2* dV = (double2*)a.take((size_t)4 * N * 16);
  if ((rc = h2d(ctx, dKx, Kx, (size_t)N * 16)) || (rc = h2d(ctx, dKy, Ky, (size_t)N * 16))) return rc;
  if ((rc = gap_v0(ctx->stream, N, dKx, dKy, dV))) return rc;
  if ((rc = d2h(ctx, V0d, dV, (size_t)4 * N * 16))) return rc;
  RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return RCWA_OK;
}

int step_smatrix_layer(rcwa_context* ctx, int N, const double2* erc, const double2* urc,
                       const double2* Kx, const double2* Ky, const double2* V0d, double k0,
                       double t, double2* S11, double2* S12, uint32_t* status) {
  const ModeDims d = dims_n(N);
  const size_t NN = (size_t)N * N, nn = (size_t)d.n * d.n;
  const size_t extra = 8 * NN * 16 + 2 * NN * 16 * 2 + 2 * (size_t)N * 4 + 1024 + 16 * 256;
  int rc = ctx_reserve(ctx, plan_bytes(d, 1, 1) + extra);
  if (rc) return rc;
  Plan pl;
  if ((rc = plan_take(ctx, d, 1, 1, pl))) return rc;
  Arena a{(char*)ctx->ws + ((plan_bytes(d, 1, 1) + 255) & ~(size_t)255)};
  rcwa_geometry g;
  g.ctx = ctx;
  g.d = d;
  g.nl = 1;
  g.t = {t};
  g.uniform = {0};
  g.erc = (double2*)a.take(NN * 16);
  g.urc = (double2*)a.take(NN * 16);
  g.einv = (double2*)a.take(NN * 16);
  g.uinv = (double2*)a.take(NN * 16);
  double2* aug = (double2*)a.take(4 * NN * 16);
  int* piv = (int*)a.take(2 * (size_t)N * 4);
  uint32_t* dst = (uint32_t*)a.take(16);
  cudaStream_t s = ctx->stream;
  if ((rc = h2d(ctx, g.erc, erc, NN * 16)) || (rc = h2d(ctx, g.urc, urc, NN * 16))) return rc;
  RCWA_CUDA_TRY(cudaMemcpyAsync(aug, g.erc, NN * 16, cudaMemcpyDeviceToDevice, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(aug + 2 * NN, g.urc, NN * 16, cudaMemcpyDeviceToDevice, s));
  if ((rc = set_identity(s, aug, N, N, 2 * NN, 2 * N, N, 2, make_double2(1, 0)))) return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(dst, 0, 16, s));
  if ((rc = zgesv(s, N, N, aug, N, 2 * NN, 2, piv, dst))) return rc;
  RCWA_CUDA_TRY(cudaMemcpyAsync(g.einv, aug + NN, NN * 16, cudaMemcpyDeviceToDevice, s));
  RCWA_CUDA_TRY(cudaMemcpyAsync(g.uinv, aug + 3 * NN, NN * 16, cudaMemcpyDeviceToDevice, s));
  double2 kinc[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(k0, 0)};
  if ((rc = h2d(ctx, pl.wv.Kx, Kx, (size_t)N * 16)) || (rc = h2d(ctx, pl.wv.Ky, Ky, (size_t)N * 16)) ||
      (rc = h2d(ctx, pl.wv.V0, V0d, (size_t)4 * N * 16)) || (rc = h2d(ctx, pl.wv.kinc, kinc, sizeof(kinc))))
    return rc;
  const Layers G = layers_of(&g);
  if ((rc = eig_layers(ctx, G, std::vector<int>{0}, pl, dst))) return rc;
  if ((rc = patterned_layer(ctx, G, 0, pl, pl.Wst, pl.L2st, dst))) return rc;
  if ((rc = d2h(ctx, S11, pl.augD + nn, nn * 16)) || (rc = d2h(ctx, S12, pl.augD + 2 * nn, nn * 16)))
    return rc;
  uint32_t hs[2] = {0, 0};
  if ((rc = d2h(ctx, hs, dst, 8))) return rc;
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  *status = hs[0] | hs[1];
  g.erc = g.urc = g.einv = g.uinv = nullptr;  // arena memory, not owned
  return RCWA_OK;
}

int step_port(rcwa_context* ctx, int side, int N, double2 er, double2 ur, const double2* Kx,
              const double2* Ky, const double2* Kz, const double2* V0d, double2* S[4]) {
  const ModeDims d = dims_n(N);
  const size_t nn = (size_t)d.n * d.n;
  int rc = ctx_reserve(ctx, 4 * nn * 16 + (size_t)8 * N * 16 + 64 + 16 * 256);
  if (rc) return rc;
  Arena a{(char*)ctx->ws};
  double2* dS[4];
  for (int k = 0; k < 4; ++k) dS[k] = (double2*)a.take(nn * 16);
  WaveVecs w;
  w.Kx = (double2*)a.take((size_t)N * 16);
  w.Ky = (double2*)a.take((size_t)N * 16);
  w.Kzr = (double2*)a.take((size_t)N * 16);
  w.Kzt = w.Kzr;
  w.V0 = (double2*)a.take((size_t)4 * N * 16);
  w.kinc = (double2*)a.take(64);
  cudaStream_t s = ctx->stream;
  if ((rc = h2d(ctx, w.Kx, Kx, (size_t)N * 16)) || (rc = h2d(ctx, w.Ky, Ky, (size_t)N * 16)) ||
      (rc = h2d(ctx, w.Kzr, Kz, (size_t)N * 16)) || (rc = h2d(ctx, w.V0, V0d, (size_t)4 * N * 16)))
    return rc;
  for (int k = 0; k < 4; ++k)
    if ((rc = fill_zero(s, dS[k], nn))) return rc;
  if ((rc = port_smatrix(s, 1, d, side, er, ur, w, dS[0], dS[1], dS[2], dS[3], (long long)nn, 0))) return rc;
  for (int k = 0; k < 4; ++k)
    if ((rc = d2h(ctx, S[k], dS[k], nn * 16))) return rc;
  RCWA_CUDA_TRY(cudaStreamSynchronize(s));
  return RCWA_OK;
}

int step_redheffer(rcwa_context* ctx, int n, const double2* const A[4], const double2* const B[4],
                   double2* const S[4], uint32_t* status) {
  const size_t nn = (size_t)n * n;
  int rc = ctx_reserve(ctx, (9 + 6) * nn * 16 + 2 * (size_t)n * 4 + 64 + 20 * 256);
  if (rc) return rc;
  Arena a{(char*)ctx->ws};
  SMat dA, dB;
  for (int k = 0; k < 4; ++k) {
    dA.p[k] = (double2*)a.take(nn * 16);
    dA.s[k] = (long long)nn;
    dB.p[k] = (double2*)a.take(nn * 16);
    dB.s[k] = (long long)nn;
    if ((rc = h2d(ctx, dA.p[k], A[k], nn * 16)) || (rc = h2d(ctx, dB.p[k], B[k], nn * 16))) return rc;
  }
  double2* tmp = (double2*)a.take(nn * 16);
  double2* augFG = (double2*)a.take(6 * nn * 16);
  int* piv = (int*)a.take(2 * (size_t)n * 4);
  uint32_t* st = (uint32_t*)a.take(16);
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, 16, ctx->stream));
  if ((rc = star_product(ctx, 1, n, dA, dB, tmp, augFG, piv, st))) return rc;
  for (int k = 0; k < 4; ++k)
    if ((rc = d2h(ctx, S[k], dA.p[k], nn * 16))) return rc;
  uint32_t hs[2] = {0, 0};
  if ((rc = d2h(ctx, hs, st, 8))) return rc;
  RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *status = hs[0] | hs[1];
  return RCWA_OK;
}

int step_efficiencies(rcwa_context* ctx, const rcwa_source* src, const rcwa_params* p,
                      const double2* kinc, const double2* Kx, const double2* Ky,
                      const double2* Kzr, const double2* Kzt, const double2* S11,
                      const double2* S21, rcwa_result* out) {
  const ModeDims d = dims_of(p);
  const size_t N = d.N, nn = (size_t)d.n * d.n;
  int rc = ctx_reserve(ctx, 2 * nn * 16 + 8 * N * 16 + 4 * N * 8 + 1024 + 16 * 256);
  if (rc) return rc;
  Arena a{(char*)ctx->ws};
  double2* dS11 = (double2*)a.take(nn * 16);
  double2* dS21 = (double2*)a.take(nn * 16);
  WaveVecs w;
  w.Kx = (double2*)a.take(N * 16);
  w.Ky = (double2*)a.take(N * 16);
  w.Kzr = (double2*)a.take(N * 16);
  w.Kzt = (double2*)a.take(N * 16);
  w.V0 = nullptr;
  w.kinc = (double2*)a.take(64);
  double* dR = (double*)a.take(N * 8);
  double* dT = (double*)a.take(N * 8);
  double* dtot = (double*)a.take(16);
  uint32_t* st = (uint32_t*)a.take(4);
  SourceDev* ds = (SourceDev*)a.take(sizeof(SourceDev));
  SourceDev hs{src->lambda0, src->theta, src->phi, src->pte, src->ptm};
  double2 ki[4] = {kinc[0], kinc[1], kinc[2], make_double2(2.0 * 3.14159265358979323846 / src->lambda0, 0)};
  if ((rc = h2d(ctx, dS11, S11, nn * 16)) || (rc = h2d(ctx, dS21, S21, nn * 16)) ||
      (rc = h2d(ctx, w.Kx, Kx, N * 16)) || (rc = h2d(ctx, w.Ky, Ky, N * 16)) ||
      (rc = h2d(ctx, w.Kzr, Kzr, N * 16)) || (rc = h2d(ctx, w.Kzt, Kzt, N * 16)) ||
      (rc = h2d(ctx, w.kinc, ki, sizeof(ki))) || (rc = h2d(ctx, ds, &hs, sizeof(hs))))
    return rc;
  RCWA_CUDA_TRY(cudaMemsetAsync(st, 0, 4, ctx->stream));
  if ((rc = efficiencies(ctx->stream, 1, d, ds, c2(p->ur_ref), c2(p->ur_trn), w, dS11, dS21,
                         (long long)nn, 0, dR, dT, dtot, st)))
    return rc;
  double htot[2];
  uint32_t hst = 0;
  if (out->R && (rc = d2h(ctx, out->R, dR, N * 8))) return rc;
  if (out->T && (rc = d2h(ctx, out->T, dT, N * 8))) return rc;
  if ((rc = d2h(ctx, htot, dtot, 16)) || (rc = d2h(ctx, &hst, st, 4))) return rc;
  RCWA_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  out->R_tot = htot[0];
  out->T_tot = htot[1];
  out->status = hst;
  return RCWA_OK;
}

}  // namespace rcwa
