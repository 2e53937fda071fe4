// Midplane rasteriser (reference: hybrid/gui/gpu_rasterizer.py:18-344) into a headless RGBA
// buffer.  The host locates every pixel's element on the cut plane and stores the element and
// its basis weights there; on the device
//   k_raster_sample  one thread per pixel: primitive variables (rho, u, v, w, p) interpolated
//                    from the element's nodal primitives with those weights;
//   k_raster_color   one thread per pixel: the displayed field (numerical schlieren from the
//                    density gradient by central differences, density, pressure, Mach or
//                    temperature), normalised to [vmin, vmax], looked up in a 256-entry RGBA
//                    table, and the body pixels painted with the background colour.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "dgb200.h"

namespace dgb {
int set_error(int code, const std::string& msg);
}

namespace {

constexpr int kRasterThreads = 256;

__global__ void __launch_bounds__(kRasterThreads) k_raster_sample(dgb_raster_desc d, dgb_state S, int nvars,
                                                                  double gamma, double* __restrict__ grid) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long npix = (long)d.nx * d.ny;
  if (p >= npix) return;
  double W[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int b = d.pixel_block[p];
  if (b >= 0) {
    const int np = d.block_nodes[b];
    const double* U = S.block[b] + (size_t)d.pixel_element[p] * np * nvars;
    const float* w = d.pixel_weights + p * d.max_nodes;
    for (int i = 0; i < np; ++i) {
      const double wi = (double)w[i];
      if (wi == 0.0) continue;
      const double* u = U + (size_t)i * nvars;
      const double rho = u[0];
      const double sr = fmax(rho, 1.0e-14);
      const double vx = u[1] / sr, vy = u[2] / sr, vz = u[3] / sr;
      const double ke = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / sr;
      const double pr = (gamma - 1.0) * (u[4] - ke);
      W[0] += wi * rho;
      W[1] += wi * vx;
      W[2] += wi * vy;
      W[3] += wi * vz;
      W[4] += wi * pr;
    }
  }
#pragma unroll
  for (int v = 0; v < 5; ++v) grid[p * 5 + v] = W[v];
}

// d rho / d(axis) like numpy.gradient: central differences inside, one-sided at the edges
__device__ __forceinline__ double grad_axis(const double* grid, int nx, int ny, int i, int j, bool along_x,
                                            double h) {
  const int n = along_x ? nx : ny, k = along_x ? i : j;
  if (n < 2) return 0.0;
  auto rho = [&](int kk) { return along_x ? grid[((long)j * nx + kk) * 5] : grid[((long)kk * nx + i) * 5]; };
  if (k == 0) return (rho(1) - rho(0)) / h;
  if (k == n - 1) return (rho(n - 1) - rho(n - 2)) / h;
  return (rho(k + 1) - rho(k - 1)) / (2.0 * h);
}

__global__ void __launch_bounds__(kRasterThreads) k_raster_color(dgb_raster_desc d, const double* __restrict__ grid,
                                                                 int mode, double vmin, double vmax, double gamma,
                                                                 uint8_t* __restrict__ rgba) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long npix = (long)d.nx * d.ny;
  if (p >= npix) return;
  const int i = (int)(p % d.nx), j = (int)(p / d.nx);
  const double* W = grid + p * 5;
  const double rho = W[0], pr = W[4];
  double s;
  if (mode == 0) {
    double gm = 0.0;
    if (!d.grad_mask[p]) {
      const double gx = grad_axis(grid, d.nx, d.ny, i, j, true, d.dx);
      const double gy = grad_axis(grid, d.nx, d.ny, i, j, false, d.dy);
      gm = sqrt(gx * gx + gy * gy);
    }
    s = 1.0 - exp(-0.08 * gm / fmax(rho, 0.1));
  } else if (mode == 1) {
    s = rho;
  } else if (mode == 2) {
    s = pr;
  } else if (mode == 3) {
    const double speed = sqrt(W[1] * W[1] + W[2] * W[2] + W[3] * W[3]);
    const double sound = sqrt(fmax(gamma * pr / fmax(rho, 1.0e-12), 0.0));
    s = speed / fmax(sound, 1.0e-12);
  } else {
    s = pr / fmax(rho, 1.0e-6) * 300.0;
  }
  const double span = fmax(vmax - vmin, 1.0e-6);
  const double t = fmin(fmax((s - vmin) / span * 255.0, 0.0), 255.0);
  const int level = isnan(t) ? 0 : (int)t;
  const uint8_t* lut = d.luts + (mode == 4 ? 256 * 4 : 0) + level * 4;
  uint8_t* out = rgba + p * 4;
  if (d.body_mask[p]) {
    out[0] = d.background[0];
    out[1] = d.background[1];
    out[2] = d.background[2];
    out[3] = d.background[3];
  } else {
    out[0] = lut[0];
    out[1] = lut[1];
    out[2] = lut[2];
    out[3] = lut[3];
  }
}

}  // namespace

extern "C" int dgb_raster_render(const dgb_raster_desc* d, const dgb_state* U, int nvars, double gamma, int mode,
                                 double vmin, double vmax, double* grid, uint8_t* rgba, void* stream) {
  if (!d || !U || !grid || !rgba || nvars < 5 || d->nx <= 0 || d->ny <= 0 || mode < 0 || mode > 4)
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad raster argument");
  const long npix = (long)d->nx * d->ny;
  const unsigned blocks = (unsigned)((npix + kRasterThreads - 1) / kRasterThreads);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_raster_sample<<<blocks, kRasterThreads, 0, st>>>(*d, *U, nvars, gamma, grid);
  k_raster_color<<<blocks, kRasterThreads, 0, st>>>(*d, grid, mode, vmin, vmax, gamma, rgba);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return dgb::set_error(DGB_ERR_CUDA, std::string("raster: ") + cudaGetErrorString(err));
  return DGB_OK;
}
