// Device-side rasterisers: permittivity / permeability grids of pillar,
// hole, line-space, rectangle and the reference demo's triangle layers,
// written straight into device memory so a geometry can be built without
// host grids (the reference fills its host grids in main.cpp:48-91).
//
// Cells are sampled at their centres exactly as the host builders of
// rcwa_b200.configs do (same operation order, no fused multiply-add), so the
// device grids are bit-identical to the host ones.
#include <vector>

#include "solver.cuh"

namespace rcwa {

namespace {

struct ShapeDev {
  int kind;
  double cx, cy, a, b;
  double2 eps, mu;
};

__global__ void raster_kernel(int nx, int ny, double lx, double ly, const ShapeDev* __restrict__ shapes,
                              const int* __restrict__ first, const double2* __restrict__ bg,
                              double2* __restrict__ er, double2* __restrict__ ur) {
  const int l = blockIdx.y;
  const long long G = (long long)nx * ny;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= G) return;
  const int ix = (int)(e % nx), iy = (int)(e / nx);
  // centred coordinates: (i + 0.5) * (L / n) - L / 2
  const double x = __dadd_rn(__dmul_rn(ix + 0.5, __ddiv_rn(lx, (double)nx)), -__ddiv_rn(lx, 2.0));
  const double y = __dadd_rn(__dmul_rn(iy + 0.5, __ddiv_rn(ly, (double)ny)), -__ddiv_rn(ly, 2.0));
  double2 ev = bg[2 * l], mv = bg[2 * l + 1];
  for (int k = first[l]; k < first[l + 1]; ++k) {
    const ShapeDev sh = shapes[k];
    bool in = false;
    if (sh.kind == RCWA_SHAPE_CIRCLE) {
      const double dx = __dadd_rn(x, -sh.cx), dy = __dadd_rn(y, -sh.cy);
      in = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= __dmul_rn(sh.a, sh.a);
    } else if (sh.kind == RCWA_SHAPE_RECT) {
      in = fabs(__dadd_rn(x, -sh.cx)) <= __ddiv_rn(sh.a, 2.0) && fabs(__dadd_rn(y, -sh.cy)) <= __ddiv_rn(sh.b, 2.0);
    } else if (sh.kind == RCWA_SHAPE_LINES) {
      in = fabs(__dadd_rn(x, -sh.cx)) <= __ddiv_rn(sh.a, 2.0);
    } else if (sh.kind == RCWA_SHAPE_TRIANGLE) {
      // the reference demo (main.cpp:51-71): apex up, base = height = a,
      // uncentred coordinates (i + 0.5) * L / n
      const double xa = __ddiv_rn(__dmul_rn(ix + 0.5, lx), (double)nx);
      const double ya = __ddiv_rn(__dmul_rn(iy + 0.5, ly), (double)ny);
      const double xc = __dadd_rn(__ddiv_rn(lx, 2.0), sh.cx), yc = __dadd_rn(__ddiv_rn(ly, 2.0), sh.cy);
      const double yr = __dadd_rn(ya, -__dadd_rn(yc, -__ddiv_rn(sh.a, 2.0)));
      const double half = __dmul_rn(__ddiv_rn(sh.a, 2.0), __ddiv_rn(yr, sh.a));
      in = yr >= 0.0 && yr <= sh.a && fabs(__dadd_rn(xa, -xc)) <= half;
    }
    if (in) {
      ev = sh.eps;
      mv = sh.mu;
    }
  }
  er[(long long)l * G + e] = ev;
  ur[(long long)l * G + e] = mv;
}

}  // namespace

int rasterize(rcwa_context* ctx, int nx, int ny, double lx, double ly, int nl,
              const rcwa_layer_shapes* layers, double2* er, double2* ur, double* t_dev) {
  cudaStream_t s = ctx->stream;
  if (nl <= 0) return RCWA_OK;
  std::vector<ShapeDev> sh;
  std::vector<int> first(nl + 1, 0);
  std::vector<double2> bg(2 * nl);
  std::vector<double> t(nl);
  for (int l = 0; l < nl; ++l) {
    const rcwa_layer_shapes& L = layers[l];
    first[l] = (int)sh.size();
    bg[2 * l] = make_double2(L.eps_bg.re, L.eps_bg.im);
    bg[2 * l + 1] = make_double2(L.mu_bg.re, L.mu_bg.im);
    t[l] = L.t;
    for (int k = 0; k < L.n_shapes; ++k) {
      const rcwa_shape& q = L.shapes[k];
      if (q.kind < RCWA_SHAPE_CIRCLE || q.kind > RCWA_SHAPE_TRIANGLE) {
        set_last_error("rasterize: unknown shape kind %d (layer %d)", q.kind, l);
        return RCWA_ERR_INVALID;
      }
      if (q.kind == RCWA_SHAPE_TRIANGLE && !(q.a > 0.0)) {
        set_last_error("rasterize: triangle size must be positive (layer %d)", l);
        return RCWA_ERR_INVALID;
      }
      sh.push_back(ShapeDev{q.kind, q.cx, q.cy, q.a, q.b, make_double2(q.eps.re, q.eps.im),
                            make_double2(q.mu.re, q.mu.im)});
    }
  }
  first[nl] = (int)sh.size();
  const size_t b_sh = sh.size() * sizeof(ShapeDev), b_first = first.size() * sizeof(int);
  const size_t b_bg = bg.size() * sizeof(double2);
  char* buf = nullptr;
  RCWA_CUDA_TRY(cudaMallocAsync((void**)&buf, b_sh + b_first + b_bg + 512, s));
  ShapeDev* dsh = (ShapeDev*)buf;
  int* dfirst = (int*)(buf + ((b_sh + 15) & ~(size_t)15));
  double2* dbg = (double2*)(buf + ((b_sh + 15) & ~(size_t)15) + ((b_first + 15) & ~(size_t)15));
  cudaError_t e = cudaSuccess;
  if (b_sh) e = cudaMemcpyAsync(dsh, sh.data(), b_sh, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dfirst, first.data(), b_first, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dbg, bg.data(), b_bg, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && t_dev) e = cudaMemcpyAsync(t_dev, t.data(), nl * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    cudaFreeAsync(buf, s);
    set_last_error("rasterize: %s", cudaGetErrorString(e));
    return RCWA_ERR_CUDA;
  }
  const long long G = (long long)nx * ny;
  raster_kernel<<<dim3(cdiv_up(G, 256), nl), 256, 0, s>>>(nx, ny, lx, ly, dsh, dfirst, dbg, er, ur);
  count_launch();
  cudaFreeAsync(buf, s);
  RCWA_LAUNCH_CHECK();
  // the host vectors above were staged by the (pageable) copies before return
  return RCWA_OK;
}

}  // namespace rcwa
