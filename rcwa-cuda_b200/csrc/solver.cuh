// Host-side solver objects behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "kernels.cuh"

struct rcwa_context {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // grow-only device arena for per-call workspace
  void* ws = nullptr;
  size_t ws_bytes = 0;
  // small pinned host staging buffer
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  uint64_t launches_at_create = 0;
  size_t mem_budget = 0;  // bytes usable for one sweep chunk (0 = auto)
  // RCWA_MIXED_* stages active in the running solve: mixed_stages while a
  // mixed-precision sweep runs, 0 otherwise.  GEMM stages use split-TF32
  // tensor-core GEMMs, LU stages an FP32 LU with ir_sweeps FP64 refinement
  // sweeps; Omega^2 and the eigensolver stay FP64
  unsigned tc = 0;
  unsigned mixed_stages = RCWA_MIXED_LAYER_GEMM | RCWA_MIXED_STAR_GEMM;
  int ir_sweeps = 1;
  int oz_digits = 5;   // 7-bit digits per operand of the int8-slice GEMM
  // refinement workspace of the current sweep chunk (inside ws), see zgesv_ir
  void* irws = nullptr;
  size_t irws_bytes = 0;
  // int8-slice GEMM workspace of the current sweep chunk (inside ws), see zgemm_oz
  void* ozws = nullptr;
  size_t ozws_bytes = 0;
  // worker contexts (own stream + workspace) that run independent group
  // chunks of rcwa_solve_batch concurrently; owned by this context
  std::vector<rcwa_context*> workers;
};

struct rcwa_geometry {
  rcwa_context* ctx = nullptr;
  rcwa::ModeDims d{};
  int nl = 0, nx = 0, ny = 0;
  double lx = 0, ly = 0;
  std::vector<double> t;
  std::vector<char> uniform;
  std::vector<double2> ueps, umu;  // grid value of uniform layers
  double2 er_ref{}, ur_ref{}, er_trn{}, ur_trn{};
  double2* erc = nullptr;   // [nl][N*N]
  double2* urc = nullptr;
  double2* einv = nullptr;  // [nl][N*N], patterned layers only
  double2* uinv = nullptr;
  // Li's factorization rule (RCWA_GEOM_LI_RULE): [4][nl][N*N] eps_xx, eps_yy,
  // mu_xx, mu_yy; null under the reference's Laurent rule
  double2* li = nullptr;
};

namespace rcwa {

int ctx_reserve(rcwa_context* ctx, size_t bytes);
int ctx_pinned(rcwa_context* ctx, size_t bytes);

// The stack as one solve chunk sees it.  A sweep shares one geometry between
// all its solves (s_item = 0, per-layer scalars on the host); a batch of
// unrelated stacks of equal shape gives every solve its own matrices (item b,
// layer l at b * s_item + l * s_layer) and per-item scalars in device arrays
// [B][nl] (t_item, ueps_item, umu_item).
struct Layers {
  ModeDims d{};
  int nl = 0;
  double2 er_ref{}, ur_ref{}, er_trn{}, ur_trn{};
  const char* uniform = nullptr;   // host [nl]
  const double* t = nullptr;       // host [nl], shared
  const double2* ueps = nullptr;   // host [nl], shared
  const double2* umu = nullptr;
  const double2 *erc = nullptr, *urc = nullptr, *einv = nullptr, *uinv = nullptr;
  // in-plane matrices of Li's rule (same layout as erc); null: erc / urc
  const double2 *exx = nullptr, *eyy = nullptr, *mxx = nullptr, *myy = nullptr;
  long long s_layer = 0, s_item = 0;
  const double* t_item = nullptr;
  const double2* ueps_item = nullptr;
  const double2* umu_item = nullptr;
  // host [nl] (may be null): layer l belongs to the first nb[l] solves of the
  // chunk only (a batch of stacks of different depth, sorted deepest first);
  // the other solves pass through that layer unchanged
  const int* nb = nullptr;
  int items(int l, int B) const { return nb ? (nb[l] < B ? nb[l] : B) : B; }
};
Layers layers_of(const rcwa_geometry* g);
// Source records that share the chunk's solves (sources that differ only in
// polarisation): record e takes the S-matrix of solve map[e] and writes
// output row oidx[e].  All pointers are device pointers.
struct ShareMap {
  int n = 0;
  const SourceDev* src = nullptr;
  const int* map = nullptr;
  const int* oidx = nullptr;
  double *R = nullptr, *T = nullptr, *tot = nullptr;
  uint32_t* status = nullptr;
};
// One chunk of B solves (device outputs R/T [B][N], tot [B][2], status [B]);
// hsrc: host array of the B sources with their lattice periods.  With sh,
// the efficiencies are computed for sh's records instead (R, T, tot unused;
// status receives the B solves' flags).
int sweep_chunk_layers(rcwa_context* ctx, const Layers& g, const SourceDev* hsrc, int B, double* R,
                       double* T, double* tot, uint32_t* status, const ShareMap* sh = nullptr);
// Device-side rasterisers (raster.cu).
int rasterize(rcwa_context* ctx, int nx, int ny, double lx, double ly, int nl,
              const rcwa_layer_shapes* layers, double2* er, double2* ur, double* t_dev);
// Device bytes one problem occupies while it is solved in a batch (its share
// of the sweep plan and of the group's geometry), under the given precision
// settings (batch.cu).
size_t problem_bytes(const rcwa_stack& st, const rcwa_params& p, int precision, unsigned mixed_stages,
                     int ir_sweeps, int gemm_digits);
// Told about every group chunk of a batch as soon as its results are in
// out[] (called from the batch's worker threads): idx holds the count
// problem indices of the chunk.
struct ChunkSink {
  void (*fn)(void* user, const int* idx, int count) = nullptr;
  void* user = nullptr;
};
// n unrelated problems, grouped by shape into batched solves (batch.cu);
// max_group > 0 caps the solves per batched launch sequence.
int solve_batch(rcwa_context* ctx, int n, const rcwa_stack* stacks, const rcwa_source* sources,
                const rcwa_params* params, int precision, int max_group, rcwa_result* out,
                const ChunkSink* sink = nullptr);

// Build convolution matrices and their inverses.  grids_er/ur are device
// pointers ([nl][ny][nx]) when on_device, host pointers otherwise.
int geometry_build(rcwa_context* ctx, rcwa_geometry* g, const rcwa_stack* st,
                   const rcwa_params* p, int on_device, unsigned opts = 0);
void geometry_free(rcwa_geometry* g);

// Sweep over sources (host array) on a prepared geometry; outputs on device.
int sweep_device(rcwa_context* ctx, const rcwa_geometry* g, const rcwa_source* sources, int B,
                 int precision, double* R, double* T, double* tot, uint32_t* status);

// Bytes of device workspace per source for a sweep at this size with np
// patterned layers; ir_sweeps > 0 adds the refinement workspace of the
// mixed-precision LU stages.
size_t sweep_bytes_per_source(const ModeDims& d, int np, int ir_sweeps = 0, bool oz = false);
// the same for the mixed-precision stages active in ctx's running solve
size_t sweep_bytes_per_source(const rcwa_context* ctx, const ModeDims& d, int np);
// ir_sweeps of a context's running solve: its refinement sweeps when an LU
// stage runs mixed, else 0.
int active_ir_sweeps(const rcwa_context* ctx);
// The GEMM kernel of `stage` in the running solve (0 = FP64, TC_TF32,
// TC_INT8) with its workspace filled in.
void set_gemm_kind(const rcwa_context* ctx, unsigned stage, ZGemm& g);

// Dense building blocks on device pointers (used by the step-level ABI).
struct SMat {
  double2* p[4];
  long long s[4];
};
int star_product(rcwa_context* ctx, int B, int n, SMat& A, const SMat& Bm, double2*& tmp,
                 double2* augFG, int* piv, uint32_t* status);

}  // namespace rcwa
