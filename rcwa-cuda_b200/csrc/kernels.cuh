// Internal (C++) interface between the kernel files and the solver.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace rcwa {

void count_launch();
uint64_t launch_count();

// Optional event-pair timing of kernel families (prof.cu).
bool prof_on();
void* prof_begin(cudaStream_t s);
void prof_end(cudaStream_t s, void* tok, const char* name);
void prof_add_flops(const char* name, double flops);
void prof_suspend(bool on);

// ---- dense primitives ------------------------------------------------------
struct ZGemm {
  int m = 0, n = 0, k = 0;
  double2 alpha = {1.0, 0.0}, beta = {0.0, 0.0};
  const double2* A = nullptr;
  int lda = 0;
  long long sA = 0;
  const double2* B = nullptr;
  int ldb = 0;
  long long sB = 0;
  double2* C = nullptr;
  int ldc = 0;
  long long sC = 0;
  const double2* dl = nullptr;  // optional left (row) scaling, stride sdl per batch
  long long sdl = 0;
  const double2* dr = nullptr;  // optional right (column) scaling, stride sdr per batch
  long long sdr = 0;
  int batch = 1;
  int opA = 0, opB = 0;         // 1 = use the conjugate transpose of the stored operand
  // reduced-precision kernels of the mixed mode: 0 = FP64, TC_TF32 = split-TF32
  // on tcgen05 (ztc.cu), TC_INT8 = int8 digit slices on tcgen05 (zoz.cu,
  // needs ws of zgemm_oz_ws_bytes)
  int tc = 0;
  int digits = 5;               // TC_INT8: 7-bit digits per operand (4, 5 or 6)
  void* ws = nullptr;
  size_t ws_bytes = 0;
};
enum { TC_TF32 = 1, TC_INT8 = 2 };
int zgemm(cudaStream_t s, const ZGemm& g);
// split-TF32 tcgen05 GEMM (ztc.cu); *err is set when a bounded wait expires
int zgemm_tc(cudaStream_t s, const ZGemm& g, int* err);
// int8-sliced tcgen05 GEMM (zoz.cu); *err is set when a bounded wait expires
size_t zgemm_oz_ws_bytes(int m, int n, int k, int batch, int digits);
int zgemm_oz(cudaStream_t s, const ZGemm& g, int* err);
int* tc_error_flag();   // device flag of the current device (set-up once per device)
int gemm_inject_timeout();   // test hook state (rcwa_debug_gemm_inject_timeout)

// X = A^-1 B on the augmented [A | B] (n x (n+nrhs), column-major, ld >= n),
// all in FP64; the A part receives the LU factors.
int zgesv(cudaStream_t s, int n, int nrhs, double2* M, int ld, long long stride, int batch,
          int* piv, uint32_t* status);
// The same solve by an FP32 (complex64) LU with `sweeps` FP64 residual
// refinement sweeps (mixed-precision mode); the A part is left unchanged.
// ws: zgesv_ir_ws_bytes(n, nrhs, batch, sweeps) bytes of device memory.
// resid_int8 != 0 computes the residuals on the int8-slice GEMM instead.
size_t zgesv_ir_ws_bytes(int n, int nrhs, int batch, int sweeps, int resid_int8 = 0);
int zgesv_ir(cudaStream_t s, int n, int nrhs, double2* M, int ld, long long stride, int batch,
             int* piv, uint32_t* status, void* ws, int sweeps, int resid_int8 = 0);

// Blocked Hessenberg reduction of packed A (zero below the subdiagonal on
// return) and Z = Q; V is an n x n scratch per matrix, ws hess_ws_bytes().
size_t hess_ws_bytes(int n, int batch);
int hess_blocked(cudaStream_t s, int n, int batch, double2* A, double2* Z, double2* V, void* ws);
// Complex Schur form of upper Hessenberg H (in place) with Z <- Z * Schur vectors.
int schur_launch(cudaStream_t s, double2* H, int ld, long long sH, int n, double2* Z, double2* lam,
                 long long slam, uint32_t* status, int batch);
// Eigen-decomposition of packed n x n matrices (destroyed).
size_t zeig_workspace_bytes(int n, int batch);
int zeig(cudaStream_t s, int n, int batch, double2* A, int ld, long long sA, double2* W,
         long long sW, double2* lam, long long slam, uint32_t* status, void* ws);

// ---- RCWA building blocks (rcwa_kernels.cu) ---------------------------------
struct ModeDims {
  int nxh, nyh, P, Q, N, n;  // N = P*Q, n = 2N
};

// Convolution matrices of `nl` layer grids (rcwa.cpp:6-82): out[l] is N x N.
int convmat(cudaStream_t s, const double2* grids, int nl, int nx, int ny, const ModeDims& d,
            double2* out, double2* scratch);
size_t convmat_scratch_bytes(int nl, int nx, int ny, const ModeDims& d);
// Li's factorization rule: out[l] = eps_xx (axis_y = 0) or eps_yy (axis_y = 1)
// of `nl` layer grids, N x N.  *bad |= 1 for a zero / non-finite grid value,
// |= 2 for a singular line Toeplitz matrix.
int li_convmat(cudaStream_t s, const double2* grids, int nl, int nx, int ny, const ModeDims& d,
               int axis_y, double2* out, void* scratch, int* bad);
size_t li_convmat_scratch_bytes(int nl, int nx, int ny, const ModeDims& d);

// Per-source wave vectors (rcwa.cpp:85-160) and gap modes (rcwa.cpp:163-234).
// One solve's source plus its lattice periods: a sweep repeats the stack's
// Lx/Ly in every entry; a batch of unrelated stacks carries each its own.
struct SourceDev {
  double lambda0, theta, phi, pte, ptm;
  double lx, ly;
};
struct WaveVecs {
  double2* Kx;      // [B][N]
  double2* Ky;      // [B][N]
  double2* Kzr;     // [B][N]
  double2* Kzt;     // [B][N]
  double2* V0;      // [B][4][N]: diagonals (11, 12, 21, 22) of the gap V0
  double2* kinc;    // [B][4]: k_inc x, y, z, (k0, 0)
};
int wave_vectors(cudaStream_t s, const SourceDev* src_dev, int B, const ModeDims& d,
                 double2 er_ref, double2 ur_ref, double2 er_trn, double2 ur_trn,
                 const WaveVecs& w, uint32_t* status);

// P and Q of a patterned layer (rcwa.cpp:262-286) from erc^-1 / urc^-1.
// exx/eyy multiply E_x/E_y in Q, mxx/myy multiply H_x/H_y in P: erc, erc,
// urc, urc under the reference's Laurent rule, Li's matrices otherwise.
// Item b reads its matrices at offset b * s_item (0: one set for all items).
int assemble_pq(cudaStream_t s, int B, const ModeDims& d, const double2* exx, const double2* eyy,
                const double2* mxx, const double2* myy, const double2* einv, const double2* uinv,
                long long s_item, const WaveVecs& w, double2* P, double2* Qm);
// lam = usqrt(lam2), ilam = 1/lam, X = exp(-k0 t lam) (rcwa.cpp:317, 329, 339).
// t_item (device, may be null): item b's thickness at t_item[b * t_stride].
int layer_modes(cudaStream_t s, int B, int n, const double2* lam2, const double2* kinc,
                double t, const double* t_item, int t_stride, double2* lam, double2* ilam,
                double2* X);
// A = Wi + Vi V0, B = Wi - Vi V0 (rcwa.cpp:335-338); Wi, Vi dense inverses.
int assemble_ab(cudaStream_t s, int B, const ModeDims& d, const double2* Wi, long long sWi,
                const double2* Vi, long long sVi, const double2* V0, double2* A, double2* Bm);
// Uniform-layer S-matrix (analytic modes, W = I), rcwa.cpp:254-352 with
// erc = eps I, urc = mu I; writes dense S11 and S12.
// bd != 0 writes the 2x2-block-diagonal "BD" form: per block four diagonals
// [X(i,i), X(i,i+N), X(i+N,i), X(i+N,i+N)] of length N (4N values).
// eps_item / mu_item / t_item (device, may be null): per-item values at
// [b * stride], replacing eps / mu / t.
int uniform_layer(cudaStream_t s, int B, const ModeDims& d, double2 eps, double2 mu, double t,
                  const double2* eps_item, const double2* mu_item, const double* t_item,
                  int stride, const WaveVecs& w, double2* S11, double2* S12, long long sS, int bd);
// Reflection / transmission side S-matrices (rcwa.cpp:354-466), dense or BD.
int port_smatrix(cudaStream_t s, int B, const ModeDims& d, int side, double2 er, double2 ur,
                 const WaveVecs& w, double2* S11, double2* S12, double2* S21, double2* S22,
                 long long sS, int bd);
// Source, fields and efficiencies (rcwa.cpp:469-585) from S_global's S11/S21
// (full n x n blocks, or compact: only the two source columns, n x 2).
// map / oidx / ustatus (device, may be null): B source records that share
// solves -- record e uses the S columns and wave vectors of solve map[e],
// writes output row oidx[e] and takes the solve's status ustatus[map[e]].
int efficiencies(cudaStream_t s, int B, const ModeDims& d, const SourceDev* src_dev,
                 double2 ur_ref, double2 ur_trn, const WaveVecs& w, const double2* S11,
                 const double2* S21, long long sS, int compact, double* R, double* T, double* tot,
                 uint32_t* status, const int* map = nullptr, const int* oidx = nullptr,
                 const uint32_t* ustatus = nullptr);
// C = beta C + alpha (X M) (side 0) or (M X) (side 1) [+ I], X in BD form.
int bd_apply(cudaStream_t s, int side, int N, int rows, int cols, const double2* X, long long sX,
             const double2* M, int ldm, long long sM, double2* C, int ldc, long long sC,
             double2 alpha, double2 beta, int addI, int batch);
// C[:, 0:2] = beta C + alpha X[:, (a, a+N)], X in BD form.
int bd_cols(cudaStream_t s, int N, int a, const double2* X, long long sX, double2* C, int ldc,
            long long sC, double2 alpha, double2 beta, int batch);
// C = X (dense expansion) or C += X (accumulate), X in BD form.
int bd_dense(cudaStream_t s, int N, const double2* X, long long sX, double2* C, long long sC,
             int accumulate, int batch);

int gap_v0(cudaStream_t s, int N, const double2* Kx, const double2* Ky, double2* V0);

// small utilities
int set_identity(cudaStream_t s, double2* M, int n, int ld, long long stride, int ncols_total,
                 int col0, int batch, double2 diag);
int fill_zero(cudaStream_t s, double2* M, size_t count);
int scale_rows(cudaStream_t s, double2* M, int n, int ncols, int ld, long long stride,
               const double2* d, long long sd, int batch);
int copy_blocks(cudaStream_t s, double2* dst, long long sdst, const double2* src, long long ssrc,
                size_t count, int batch);
int any_nonuniform(cudaStream_t s, const double2* grid, size_t count, int* flag);

}  // namespace rcwa
