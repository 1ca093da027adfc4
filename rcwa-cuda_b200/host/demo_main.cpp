// The reference's built-in case (rcwa3d/src/main.cpp:35-198) written against
// the rcwa_b200 C++ host API: once step by step with the reference's function
// names, once as a single GPU solve.  Build from the repository root:
//   g++ -std=c++17 -O2 -Iinclude -Ircwa-cuda_b200/host rcwa-cuda_b200/host/demo_main.cpp \
//       -Lrcwa-cuda_b200/rcwa_b200 -lrcwa_b200 -Wl,-rpath,<dir of librcwa_b200.so> -o demo_main
#include <cmath>
#include <cstdio>
#include <vector>

#include "rcwa_b200.hpp"

using namespace rcwa_b200;

int main() {
  const int Nx = 1024, Ny = 1024;
  const int Nx_harmonics = 3, Ny_harmonics = 3;
  const Real Lx = 1.75, Ly = 1.50;
  std::vector<Complex> er_field(Ny * Nx), ur_field(Ny * Nx);
  for (int iy = 0; iy < Ny; ++iy) {          // triangle of eps=2 in eps=6, main.cpp:51-71
    const double y = (iy + 0.5) * Ly / Ny;
    for (int ix = 0; ix < Nx; ++ix) {
      const double x = (ix + 0.5) * Lx / Nx;
      const double w = 0.8 * Ly, xc = Lx / 2.0, yc = Ly / 2.0;
      const double y_rel = y - (yc - w / 2.0);
      const double half_base = (w / 2.0) * (y_rel / w);
      const bool inside = (y_rel >= 0) && (y_rel <= w) && (std::abs(x - xc) <= half_base);
      er_field[iy * Nx + ix] = inside ? Complex(2.0, 0.0) : Complex(6.0, 0.0);
      ur_field[iy * Nx + ix] = Complex(1.0, 0.0);
    }
  }
  std::vector<Complex> er = er_field, ur = ur_field;
  er.insert(er.end(), Ny * Nx, Complex(6.0, 0.0));
  ur.insert(ur.end(), Ny * Nx, Complex(1.0, 0.0));
  const std::vector<Real> thickness{0.5, 0.3};
  Device device(Nx, Ny, (int)thickness.size(), Lx, Ly, er, ur, thickness, Nx_harmonics, Ny_harmonics);
  Source source(2.0, 0.0, 0.0, 0.0, 1.0);
  RCWAParams params(Nx_harmonics, Ny_harmonics, Complex(2.0, 0.0), Complex(1.0, 0.0), Complex(9.0, 0.0),
                    Complex(1.0, 0.0));

  // step by step, mirroring main.cpp:125-191
  for (int layer = 0; layer < device.num_layers; ++layer) {
    device.erc.at(layer) = ConvMat(device.er, layer, device.Nx, device.Ny, Nx_harmonics, Ny_harmonics);
    device.urc.at(layer) = ConvMat(device.ur, layer, device.Nx, device.Ny, Nx_harmonics, Ny_harmonics);
  }
  std::vector<Complex> k_inc;
  Vector Kx, Ky, Kz_ref, Kz_trn;
  ComputeWaveVectors(device, source, params, k_inc, Kx, Ky, Kz_ref, Kz_trn);
  Matrix W0, V0, W_ref, W_trn;
  GapMedium(Kx, Ky, W0, V0);
  ScatteringMatrix S_device = SMatrixInit(Nx_harmonics, Ny_harmonics);
  for (int layer = 0; layer < device.num_layers; ++layer) {
    ScatteringMatrix S_layer = SMatrixLayer(layer, device, source, params, Kx, Ky, W0, V0);
    S_device = RedhefferProduct(S_device, S_layer);
  }
  ScatteringMatrix S_ref = SMatrixReflection(params, Kx, Ky, Kz_ref, W0, V0, W_ref);
  ScatteringMatrix S_trn = SMatrixTransmission(params, Kx, Ky, Kz_trn, W0, V0, W_trn);
  ScatteringMatrix S_global = RedhefferProduct(RedhefferProduct(S_ref, S_device), S_trn);
  Results stepwise = ComputeResults(source, params, k_inc, Kx, Ky, Kz_ref, Kz_trn, S_global);

  // the same as one call
  Results one = Solve(device, source, params);

  std::printf("step-by-step: R_tot=%.15f T_tot=%.15f sum=%.15f status=%u\n", stepwise.R_tot,
              stepwise.T_tot, stepwise.R_tot + stepwise.T_tot, stepwise.status);
  std::printf("one call    : R_tot=%.15f T_tot=%.15f sum=%.15f status=%u\n", one.R_tot, one.T_tot,
              one.R_tot + one.T_tot, one.status);
  double d = 0.0;
  for (int q = 0; q < params.Q(); ++q)
    for (int p = 0; p < params.P(); ++p) d = std::fmax(d, std::fabs(one.R(q, p) - stepwise.R(q, p)));
  std::printf("max |R_one - R_steps| = %.3e\n", d);
  return (d < 1e-10 && std::fabs(one.R_tot + one.T_tot - 1.0) < 1e-10) ? 0 : 1;
}
