// rcwa_b200.hpp -- C++ host API with the reference's names and argument
// meanings (rcwa3d/include/rcwa.hpp), implemented on the C ABI of
// include/rcwa_b200.h.  Eigen-free: matrices are column-major
// std::vector<std::complex<double>> wrappers, like Eigen's default layout.
//
// Differences from the reference surface, all deliberate:
//  * errors throw rcwa_b200::Error (with the C ABI code) instead of abort()
//    (rcwa.cpp:300) -- numerical trouble inside a solve is reported in
//    Results::status and leaves the same Inf/NaN values the reference gives;
//  * W0/V0/W_ref/W_trn keep their reference meaning (W0 = W_ref = W_trn = I);
//  * the source/field/efficiency chain of rcwa.cpp:469-585 is one call,
//    ComputeResults(), because r and t are only consumed by the efficiencies;
//  * Solve()/SolveSweep() run the whole main.cpp:111-191 sequence on the GPU
//    in one call (batched over sources for a sweep).
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rcwa_b200.h"

namespace rcwa_b200 {

using Real = double;
using Complex = std::complex<Real>;
static_assert(sizeof(Complex) == sizeof(rcwa_complex), "layout");

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != RCWA_OK && rc != RCWA_ERR_NUMERIC)
    throw Error(rc, std::string("rcwa_b200: ") + rcwa_last_error());
}

// Column-major dense complex matrix (Eigen::MatrixXcd layout).
class Matrix {
 public:
  Matrix() = default;
  Matrix(int r, int c) : r_(r), c_(c), d_((size_t)r * c) {}
  static Matrix Zero(int r, int c) { return Matrix(r, c); }
  static Matrix Identity(int n) {
    Matrix m(n, n);
    for (int i = 0; i < n; ++i) m(i, i) = 1.0;
    return m;
  }
  int rows() const { return r_; }
  int cols() const { return c_; }
  Complex& operator()(int i, int j) { return d_[(size_t)j * r_ + i]; }
  const Complex& operator()(int i, int j) const { return d_[(size_t)j * r_ + i]; }
  Complex* data() { return d_.data(); }
  const Complex* data() const { return d_.data(); }
  rcwa_complex* c_data() { return reinterpret_cast<rcwa_complex*>(d_.data()); }
  const rcwa_complex* c_data() const { return reinterpret_cast<const rcwa_complex*>(d_.data()); }

 private:
  int r_ = 0, c_ = 0;
  std::vector<Complex> d_;
};
using Vector = std::vector<Complex>;

// Q x P real matrix, column-major (Eigen reshaped(Q, P), rcwa.cpp:576).
class RealMatrix {
 public:
  RealMatrix() = default;
  RealMatrix(int r, int c) : r_(r), c_(c), d_((size_t)r * c) {}
  int rows() const { return r_; }
  int cols() const { return c_; }
  Real& operator()(int i, int j) { return d_[(size_t)j * r_ + i]; }
  Real operator()(int i, int j) const { return d_[(size_t)j * r_ + i]; }
  Real* data() { return d_.data(); }
  Real sum() const {
    Real s = 0;
    for (Real v : d_) s += v;
    return s;
  }

 private:
  int r_ = 0, c_ = 0;
  std::vector<Real> d_;
};

// One library context per thread, on the device chosen by SetDevice (default 0).
namespace detail {
struct CtxDeleter {
  void operator()(rcwa_context* c) const { rcwa_context_destroy(c); }
};
inline int& device_index() {
  static thread_local int d = 0;
  return d;
}
inline std::unique_ptr<rcwa_context, CtxDeleter>& ctx_slot() {
  static thread_local std::unique_ptr<rcwa_context, CtxDeleter> c;
  return c;
}
inline const rcwa_complex* cc(const Vector& v) { return reinterpret_cast<const rcwa_complex*>(v.data()); }
inline rcwa_complex* cc(Vector& v) { return reinterpret_cast<rcwa_complex*>(v.data()); }
inline rcwa_complex cx(Complex z) { return rcwa_complex{z.real(), z.imag()}; }
}  // namespace detail

inline void SetDevice(int dev) {
  detail::device_index() = dev;
  detail::ctx_slot().reset();
}
inline rcwa_context* Context() {
  auto& s = detail::ctx_slot();
  if (!s) {
    rcwa_context* c = nullptr;
    check(rcwa_context_create(detail::device_index(), &c));
    s.reset(c);
  }
  return s.get();
}

// ---- data model (rcwa.hpp:48-162) -------------------------------------------
struct Device {
  int Nx{}, Ny{}, num_layers{};
  Real Lx{}, Ly{};
  std::vector<Complex> er{}, ur{};   // [layer][iy][ix]
  std::vector<Real> t{};
  std::vector<Matrix> erc{}, urc{};  // filled with ConvMat, main.cpp:126-138
  Device(int Nx_, int Ny_, int num_layers_, Real Lx_, Real Ly_, const std::vector<Complex>& er_,
         const std::vector<Complex>& ur_, const std::vector<Real>& t_, int Nx_harmonics_,
         int Ny_harmonics_)
      : Nx(Nx_), Ny(Ny_), num_layers(num_layers_), Lx(Lx_), Ly(Ly_), er(er_), ur(ur_), t(t_) {
    const int PQ = (2 * Nx_harmonics_ + 1) * (2 * Ny_harmonics_ + 1);
    erc.assign(num_layers_, Matrix::Zero(PQ, PQ));
    urc.assign(num_layers_, Matrix::Zero(PQ, PQ));
  }
  rcwa_stack c_stack() const {
    return rcwa_stack{Nx, Ny, num_layers, Lx, Ly, reinterpret_cast<const rcwa_complex*>(er.data()),
                      reinterpret_cast<const rcwa_complex*>(ur.data()), t.data()};
  }
};

struct Source {
  Real lambda0{}, k0{}, theta{}, phi{}, pte{}, ptm{};
  Source(Real lambda0_, Real theta_, Real phi_, Real pte_, Real ptm_)
      : lambda0(lambda0_), k0(2 * 3.14159265358979323846 / lambda0_), theta(theta_), phi(phi_),
        pte(pte_), ptm(ptm_) {}
  rcwa_source c_source() const { return rcwa_source{lambda0, theta, phi, pte, ptm}; }
};

struct RCWAParams {
  int Nx_harmonics{}, Ny_harmonics{};
  Complex er_ref{}, ur_ref{}, er_trn{}, ur_trn{};
  RCWAParams(int nxh, int nyh, Complex er_ref_, Complex ur_ref_, Complex er_trn_, Complex ur_trn_)
      : Nx_harmonics(nxh), Ny_harmonics(nyh), er_ref(er_ref_), ur_ref(ur_ref_), er_trn(er_trn_),
        ur_trn(ur_trn_) {}
  int P() const { return 2 * Nx_harmonics + 1; }
  int Q() const { return 2 * Ny_harmonics + 1; }
  rcwa_params c_params() const {
    return rcwa_params{Nx_harmonics, Ny_harmonics, detail::cx(er_ref), detail::cx(ur_ref),
                       detail::cx(er_trn), detail::cx(ur_trn)};
  }
};

struct Results {
  RealMatrix R{}, T{};
  Real R_tot{}, T_tot{};
  uint32_t status{};  // RCWA_STATUS_* bits; 0 = clean
};

struct ScatteringMatrix {
  Matrix S11{}, S12{}, S21{}, S22{};
  ScatteringMatrix() = default;
  ScatteringMatrix(Matrix a, Matrix b, Matrix c, Matrix d)
      : S11(std::move(a)), S12(std::move(b)), S21(std::move(c)), S22(std::move(d)) {}
};

// ---- step functions (rcwa.cpp) --------------------------------------------------
// rcwa.cpp:6-82
inline Matrix ConvMat(const std::vector<Complex>& field, int layer, int Nx, int Ny, int Nx_harmonics,
                      int Ny_harmonics) {
  const int PQ = (2 * Nx_harmonics + 1) * (2 * Ny_harmonics + 1);
  Matrix C(PQ, PQ);
  check(rcwa_convmat(Context(), reinterpret_cast<const rcwa_complex*>(field.data()), layer, Nx, Ny,
                     Nx_harmonics, Ny_harmonics, C.c_data()));
  return C;
}

// rcwa.cpp:85-160
inline void ComputeWaveVectors(const Device& device, const Source& source, const RCWAParams& params,
                               std::vector<Complex>& k_inc, Vector& Kx, Vector& Ky, Vector& Kz_ref,
                               Vector& Kz_trn) {
  const int PQ = params.P() * params.Q();
  k_inc.assign(3, 0.0);
  Kx.assign(PQ, 0.0);
  Ky.assign(PQ, 0.0);
  Kz_ref.assign(PQ, 0.0);
  Kz_trn.assign(PQ, 0.0);
  rcwa_source s = source.c_source();
  rcwa_params p = params.c_params();
  check(rcwa_wave_vectors(Context(), device.Lx, device.Ly, &s, &p, detail::cc(k_inc), detail::cc(Kx),
                          detail::cc(Ky), detail::cc(Kz_ref), detail::cc(Kz_trn)));
}

// rcwa.cpp:163-234
inline void GapMedium(const Vector& Kx, const Vector& Ky, Matrix& W0, Matrix& V0) {
  const int n = 2 * (int)Kx.size();
  W0 = Matrix(n, n);
  V0 = Matrix(n, n);
  check(rcwa_gap_medium(Context(), (int)Kx.size(), detail::cc(Kx), detail::cc(Ky), W0.c_data(),
                        V0.c_data()));
}

// rcwa.cpp:237-250
inline ScatteringMatrix SMatrixInit(int Nx_harmonics, int Ny_harmonics) {
  const int n = 2 * (2 * Nx_harmonics + 1) * (2 * Ny_harmonics + 1);
  return ScatteringMatrix(Matrix::Zero(n, n), Matrix::Identity(n), Matrix::Identity(n), Matrix::Zero(n, n));
}

// rcwa.cpp:254-352 (W0 = I is implied; V0 carries the gap modes)
inline ScatteringMatrix SMatrixLayer(int layer, const Device& device, const Source& source,
                                     const RCWAParams& params, const Vector& Kx, const Vector& Ky,
                                     const Matrix& /*W0*/, const Matrix& V0) {
  (void)params;
  const int PQ = (int)Kx.size(), n = 2 * PQ;
  Matrix S11(n, n), S12(n, n);
  uint32_t st = 0;
  check(rcwa_smatrix_layer(Context(), PQ, device.erc.at(layer).c_data(), device.urc.at(layer).c_data(),
                           detail::cc(Kx), detail::cc(Ky), V0.c_data(), source.k0, device.t.at(layer),
                           S11.c_data(), S12.c_data(), &st));
  if (st & RCWA_STATUS_EIG_NOCONV) throw Error(RCWA_ERR_NUMERIC, "rcwa_b200: eigensolver did not converge");
  Matrix S21 = S12, S22 = S11;
  return ScatteringMatrix(std::move(S11), std::move(S12), std::move(S21), std::move(S22));
}

inline ScatteringMatrix port(bool ref, const RCWAParams& params, const Vector& Kx, const Vector& Ky,
                             Vector& Kz, const Matrix& V0, Matrix& Wp) {
  const int n = 2 * (int)Kx.size();
  ScatteringMatrix S(Matrix(n, n), Matrix(n, n), Matrix(n, n), Matrix(n, n));
  rcwa_params p = params.c_params();
  auto f = ref ? rcwa_smatrix_reflection : rcwa_smatrix_transmission;
  check(f(Context(), &p, detail::cc(Kx), detail::cc(Ky), detail::cc(Kz), V0.c_data(), S.S11.c_data(),
          S.S12.c_data(), S.S21.c_data(), S.S22.c_data()));
  Wp = Matrix::Identity(n);
  return S;
}
// rcwa.cpp:354-411
inline ScatteringMatrix SMatrixReflection(const RCWAParams& params, const Vector& Kx, const Vector& Ky,
                                          Vector& Kz_ref, const Matrix& /*W0*/, const Matrix& V0,
                                          Matrix& W_ref) {
  return port(true, params, Kx, Ky, Kz_ref, V0, W_ref);
}
// rcwa.cpp:414-466
inline ScatteringMatrix SMatrixTransmission(const RCWAParams& params, const Vector& Kx, const Vector& Ky,
                                            Vector& Kz_trn, const Matrix& /*W0*/, const Matrix& V0,
                                            Matrix& W_trn) {
  return port(false, params, Kx, Ky, Kz_trn, V0, W_trn);
}

// rcwa.cpp:588-615
inline ScatteringMatrix RedhefferProduct(const ScatteringMatrix& A, const ScatteringMatrix& B) {
  const int n = A.S11.rows();
  ScatteringMatrix S(Matrix(n, n), Matrix(n, n), Matrix(n, n), Matrix(n, n));
  const rcwa_complex* a[4] = {A.S11.c_data(), A.S12.c_data(), A.S21.c_data(), A.S22.c_data()};
  const rcwa_complex* b[4] = {B.S11.c_data(), B.S12.c_data(), B.S21.c_data(), B.S22.c_data()};
  rcwa_complex* s[4] = {S.S11.c_data(), S.S12.c_data(), S.S21.c_data(), S.S22.c_data()};
  uint32_t st = 0;
  check(rcwa_redheffer(Context(), n, a, b, s, &st));
  return S;
}

// rcwa.cpp:469-585: source coefficients, reflected/transmitted fields and
// diffraction efficiencies from S_global, in one call.
inline Results ComputeResults(const Source& source, const RCWAParams& params,
                              const std::vector<Complex>& k_inc, const Vector& Kx, const Vector& Ky,
                              const Vector& Kz_ref, const Vector& Kz_trn, const ScatteringMatrix& S_global) {
  Results r;
  r.R = RealMatrix(params.Q(), params.P());
  r.T = RealMatrix(params.Q(), params.P());
  rcwa_result out{r.R.data(), r.T.data(), 0.0, 0.0, 0u};
  rcwa_source s = source.c_source();
  rcwa_params p = params.c_params();
  check(rcwa_efficiencies(Context(), &s, &p, detail::cc(k_inc), detail::cc(Kx), detail::cc(Ky),
                          detail::cc(Kz_ref), detail::cc(Kz_trn), S_global.S11.c_data(),
                          S_global.S21.c_data(), &out));
  r.R_tot = out.R_tot;
  r.T_tot = out.T_tot;
  r.status = out.status;
  return r;
}

// ---- one-call solves (main.cpp:111-191 on the GPU) -----------------------------
inline std::vector<Results> SolveSweep(const Device& device, const std::vector<Source>& sources,
                                       const RCWAParams& params, int precision = RCWA_PREC_FP64) {
  const int ns = (int)sources.size();
  std::vector<Results> res(ns);
  std::vector<rcwa_source> cs(ns);
  std::vector<rcwa_result> out(ns);
  for (int i = 0; i < ns; ++i) {
    cs[i] = sources[i].c_source();
    res[i].R = RealMatrix(params.Q(), params.P());
    res[i].T = RealMatrix(params.Q(), params.P());
    out[i] = rcwa_result{res[i].R.data(), res[i].T.data(), 0.0, 0.0, 0u};
  }
  rcwa_stack st = device.c_stack();
  rcwa_params p = params.c_params();
  check(rcwa_solve_sweep(Context(), &st, cs.data(), ns, &p, precision, out.data()));
  for (int i = 0; i < ns; ++i) {
    res[i].R_tot = out[i].R_tot;
    res[i].T_tot = out[i].T_tot;
    res[i].status = out[i].status;
  }
  return res;
}

inline Results Solve(const Device& device, const Source& source, const RCWAParams& params,
                     int precision = RCWA_PREC_FP64) {
  return SolveSweep(device, std::vector<Source>{source}, params, precision)[0];
}

// ---- batches of unrelated problems and the serving loop ------------------------
struct Problem {
  const Device* device;
  Source source;
  RCWAParams params;
};

// rcwa_solve_batch: every problem has its own stack, source and port media.
inline std::vector<Results> SolveBatch(const std::vector<Problem>& problems,
                                       int precision = RCWA_PREC_FP64) {
  const int n = (int)problems.size();
  std::vector<Results> res(n);
  std::vector<rcwa_stack> st(n);
  std::vector<rcwa_source> cs(n);
  std::vector<rcwa_params> cp(n);
  std::vector<rcwa_result> out(n);
  for (int i = 0; i < n; ++i) {
    const Problem& q = problems[i];
    st[i] = q.device->c_stack();
    cs[i] = q.source.c_source();
    cp[i] = q.params.c_params();
    res[i].R = RealMatrix(q.params.Q(), q.params.P());
    res[i].T = RealMatrix(q.params.Q(), q.params.P());
    out[i] = rcwa_result{res[i].R.data(), res[i].T.data(), 0.0, 0.0, 0u};
  }
  if (n > 0) check(rcwa_solve_batch(Context(), n, st.data(), cs.data(), cp.data(), precision, out.data()));
  for (int i = 0; i < n; ++i) {
    res[i].R_tot = out[i].R_tot;
    res[i].T_tot = out[i].T_tot;
    res[i].status = out[i].status;
  }
  return res;
}

// rcwa_server_*: requests are queued from any thread and solved in batches
// by the server's worker (continuous batching).
class Server {
 public:
  explicit Server(int device = 0, int max_batch = 256, int max_queue = 1 << 20,
                  int precision = RCWA_PREC_FP64) {
    check(rcwa_server_create(device, max_batch, max_queue, precision, &h_));
  }
  ~Server() { rcwa_server_destroy(h_); }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  uint64_t Submit(const Device& device, const Source& source, const RCWAParams& params) {
    rcwa_stack st = device.c_stack();
    rcwa_source cs = source.c_source();
    rcwa_params cp = params.c_params();
    uint64_t t = 0;
    check(rcwa_server_submit(h_, &st, &cs, &cp, &t));
    return t;
  }
  // Blocks until the request is done; the ticket is released.
  Results Wait(uint64_t ticket, const RCWAParams& params) {
    Results r;
    r.R = RealMatrix(params.Q(), params.P());
    r.T = RealMatrix(params.Q(), params.P());
    rcwa_result out{r.R.data(), r.T.data(), 0.0, 0.0, 0u};
    int done = 0;
    check(rcwa_server_poll(h_, ticket, 1, &out, &done));
    r.R_tot = out.R_tot;
    r.T_tot = out.T_tot;
    r.status = out.status;
    return r;
  }

 private:
  rcwa_server* h_ = nullptr;
};

}  // namespace rcwa_b200
