// Allocation-free time-step estimate (dgb_stable_dt_noalloc, declared in include/dgb200.h).
//
// Some callers cannot allocate device memory at the moment they need a time step: a
// coupling framework or host code that owns a fixed device-memory pool and forbids
// allocations from libraries it calls, or a time loop that must not call cudaMalloc
// (it synchronises the device and may fail once the pool is reserved).  This entry
// point needs no plan and no cudaMalloc: its only scratch is the file-scope device array
// below, which every GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/dgb200.h"

namespace {

// Per-element CFL rates of the last call (one element block).  8 MiB per device.
constexpr int kMaxElements = 1 << 20;
static __device__ __align__(256) double g_rate_scratch[kMaxElements];

thread_local std::string g_noalloc_error;
std::mutex g_setup_mutex;
double* g_scratch_ptr[64] = {nullptr};   // device address of g_rate_scratch per device ordinal

// Rate of one element (one warp per element): (2P+1) max(|u| + c) / h plus, when viscous,
// the BR2 diffusion rate 2 * br2 * (2P+1)^2 * max(4/3 mu/rho, kappa/(rho cp)) / max(h, 0.01)^2,
// with rho the element's mean nodal density floored at 0.1 (hybrid/time_integration.py:93-169).
__global__ void k_rates_noalloc(const double* U, const double* length, int E, int Np, int nv, int degree,
                                double gamma, double mu, double kappa, double cp, double br2, int viscous,
                                double* rate) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const double df = 2.0 * degree + 1.0;
  for (int e = warp; e < E; e += nwarps) {
    const double* Ue = U + (size_t)e * Np * nv;
    double smax = -INFINITY, rsum = 0.0;
    bool nan_seen = false;
    for (int i = lane; i < Np; i += 32) {
      const double* u = Ue + (size_t)i * nv;
      const double rho = u[0];
      const double srho = fmax(rho, 1.0e-14);
      const double vx = u[1] / srho, vy = u[2] / srho, vz = u[3] / srho;
      const double m2 = __dadd_rn(__dadd_rn(__dmul_rn(u[1], u[1]), __dmul_rn(u[2], u[2])), __dmul_rn(u[3], u[3]));
      const double p = __dmul_rn(gamma - 1.0, __dsub_rn(u[4], __dmul_rn(0.5, m2) / srho));
      // a NaN density or pressure makes the reference's rate NaN (jnp.maximum keeps NaN,
      // fmax would drop it), which it then maps to 1e7
      const double r = fmax(rho, 1.0e-14), pf = fmax(p, 1.0e-14);
      const double sp = sqrt(vx * vx + vy * vy + vz * vz) + sqrt(gamma * pf / r);
      nan_seen |= isnan(rho) || isnan(p) || isnan(sp);
      smax = fmax(smax, sp);
      rsum += r;
    }
    for (int o = 16; o > 0; o >>= 1) {
      smax = fmax(smax, __shfl_xor_sync(0xffffffff, smax, o));
      rsum += __shfl_xor_sync(0xffffffff, rsum, o);
    }
    nan_seen = __any_sync(0xffffffff, nan_seen);
    const double h = length[e];
    double rt = nan_seen ? NAN : df * smax / h;
    if (viscous) {
      const double rmin = fmax(rsum / Np, 0.1);
      const double diff = fmax((4.0 / 3.0) * mu / rmin, kappa / (rmin * cp));
      const double vl = fmax(h, 0.01);
      rt = rt + 2.0 * br2 * df * df * diff / (vl * vl);
    }
    if (isnan(rt) || (isinf(rt) && rt > 0.0)) rt = 1.0e7;
    else if (isinf(rt)) rt = -1.7976931348623157e308;
    if (lane == 0) rate[e] = rt;
  }
}

// dt = clip(cfl / max(max_e rate_e, 1e-12), 1e-7, 1e-3) by one CTA.
__global__ void k_dt_noalloc(const double* rate, int E, double cfl, double* dt_out) {
  __shared__ double red[256];
  double m = -INFINITY;
  for (int i = threadIdx.x; i < E; i += blockDim.x) m = fmax(m, rate[i]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *dt_out = fmin(fmax(cfl / fmax(red[0], 1.0e-12), 1.0e-7), 1.0e-3);
}

int noalloc_fail(const std::string& msg) {
  g_noalloc_error = msg;
  return DGB_ERR_ARGUMENT;
}

}  // namespace

extern "C" {

const char* dgb_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

int dgb_stable_dt_noalloc(const double* U, const double* length, int num_elements, int num_nodes, int nvars,
                          int degree, double gamma, double gas_constant, double dynamic_viscosity,
                          double thermal_conductivity, double br2_penalty, double cfl, double* dt_out,
                          void* stream) {
  if (!U || !length || !dt_out) return noalloc_fail("null pointer argument");
  if (num_elements < 1 || num_nodes < 1 || nvars < 5) return noalloc_fail("empty or malformed state");
  if (degree < 0) return noalloc_fail("polynomial degree must be non-negative");
  if (num_elements > kMaxElements)
    return noalloc_fail("dgb_stable_dt_noalloc handles at most 1048576 elements per call (" +
                        std::to_string(num_elements) + " given); use dgb_stable_dt or split the block");
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return noalloc_fail(std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  if (dev < 0 || dev >= 64) return noalloc_fail("device ordinal out of range");
  double* scratch = nullptr;
  {
    // once per device, with that device current: the host-side symbol is only a stand-in,
    // the kernels need the device address
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
      err = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_scratch_ptr[dev]), g_rate_scratch);
      if (err != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        return noalloc_fail(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
      }
    }
    scratch = g_scratch_ptr[dev];
  }
  const double cp = gamma * gas_constant / (gamma - 1.0);
  const int viscous = dynamic_viscosity > 0.0 ? 1 : 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int warps_per_cta = 4;
  int grid = (num_elements + warps_per_cta - 1) / warps_per_cta;
  if (grid > 2368) grid = 2368;
  k_rates_noalloc<<<grid, 32 * warps_per_cta, 0, st>>>(U, length, num_elements, num_nodes, nvars, degree, gamma,
                                                       dynamic_viscosity, thermal_conductivity, cp, br2_penalty,
                                                       viscous, scratch);
  k_dt_noalloc<<<1, 256, 0, st>>>(scratch, num_elements, cfl, dt_out);
  err = cudaGetLastError();
  if (err != cudaSuccess) {
    g_noalloc_error = std::string("launch: ") + cudaGetErrorString(err);
    return DGB_ERR_CUDA;
  }
  return DGB_OK;
}

}  // extern "C"
