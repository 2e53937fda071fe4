// Element-local limiter, detector and reduction kernels (float64).
//
//   k_positivity    Zhang-Shu scaling toward the cell mean: density theta in closed form,
//                   pressure theta by 30 bisection steps over node, volume-point and
//                   face-point samples (hybrid/limiter.py:69-147).
//   k_troubled      Persson-type high-mode sensor on (rho, p) plus the MOOD admissibility
//                   test at samples and the mean (hybrid/limiter.py:165-185, 285-300).
//   k_rate / k_dt   CFL rate per element, max by warp shuffles then one final CTA
//                   (hybrid/time_integration.py:93-169).
//   k_adm / k_adm_final   finite check and min rho / min p over all nodes
//                   (hybrid/time_integration.py:291-312), combined across stages.
#pragma once
#include "dg_kernels.cuh"

namespace dgb {

struct LimiterConst {
  double density_floor, pressure_floor, relative_floor;   // positivity limiter
  double adm_density_floor, adm_pressure_floor;           // integrator admissibility
  double sensor_threshold;
  double lebesgue;   // max over the limiter's sample points of sum_i |B_i(x)|; 0: no nodal certificate
};

template <int NV>
__device__ __forceinline__ double pressure_of(const Physics& ph, const double* U) {
  const double srho = fmax(U[0], kRhoFloor);
  const double ke = 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / srho;
  return (ph.gamma - 1.0) * (U[4] - ke);
}

// Certificate, from the nodal values alone, that density and pressure are admissible at every
// limiter sample of the element and at its cell mean.  A sample u(x) = sum_i B_i(x) U_i, with
// sum_i B_i = 1, obeys |u(x) - c| <= L h, for c and h the midpoint and half-range of the nodal
// values and L the largest sum_i |B_i| over the sample points (their Lebesgue constant).  Intervals of
// rho, m and E then bound rho and p = (gamma - 1)(E - |m|^2 / 2 rho) from below at every sample.
// The cell mean is a positive combination of samples, so its rho lies in the same interval and
// its p is at least the smallest sample p (p is concave in the conserved variables).  The margins
// tol_r and tol_p cover the rounding of the computed samples many times over.  True when
//   rho_lo - tol_r >= max(rho_floor, rel (rho_hi + tol_r)),
//   p_lo - tol_p >= max(p_floor, rel pmean_hi + tol_p),
// with rho_lo >= 1e-3 rho_hi, so that the relative rounding of |m|^2 / rho stays small.
// A non-finite nodal value gives false.  Every thread returns the same value.
// The bound check of the certificate, from the smallest and largest nodal value of rho, m and E.
__device__ __forceinline__ bool certificate_from_range(const double (&mn)[5], const double (&mx)[5],
                                                       const Physics& ph, double L, double rho_floor,
                                                       double p_floor, double rel) {
  if (!(L >= 1.0)) return false;
  double a[5], b[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const double c = 0.5 * (mn[v] + mx[v]), h = 0.5 * (mx[v] - mn[v]);
    a[v] = c - L * h;
    b[v] = c + L * h;
  }
  const double tol_r = 1.0e-12 * L * fmax(fabs(a[0]), fabs(b[0]));
  if (!(a[0] - tol_r > 0.0) || !(a[0] >= 1.0e-3 * b[0])) return false;
  double m2hi = 0.0, m2lo = 0.0;
#pragma unroll
  for (int d = 1; d <= 3; ++d) {
    m2hi += fmax(a[d] * a[d], b[d] * b[d]);
    m2lo += (a[d] <= 0.0 && b[d] >= 0.0) ? 0.0 : fmin(a[d] * a[d], b[d] * b[d]);
  }
  const double g1 = ph.gamma - 1.0;
  const double ke_hi = 0.5 * m2hi / a[0], ke_lo = 0.5 * m2lo / b[0];
  const double p_lo = g1 * (a[4] - ke_hi), pmean_hi = g1 * (b[4] - ke_lo);
  const double tol_p = 1.0e-6 * g1 * (L * fmax(fabs(a[4]), fabs(b[4])) + ke_hi);
  return (a[0] - tol_r >= fmax(rho_floor, rel * (b[0] + tol_r))) &&
         (p_lo - tol_p >= fmax(p_floor, rel * pmean_hi + tol_p));
}

// Warp-level range of the nodal rho, m, E of one element ([NP][NV] at Ug; lane l takes nodes l,
// l + 32, ..., so each variable goes straight to its own minimum and maximum) and whether every
// nodal value is finite.  Every lane returns the same range.
template <int NV, int NP>
__device__ __forceinline__ bool warp_nodal_range(const double* __restrict__ Ug, double (&mn)[5], double (&mx)[5]) {
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    mn[v] = INFINITY;
    mx[v] = -INFINITY;
  }
  bool fin = true;
#pragma unroll
  for (int l0 = 0; l0 < NP; l0 += 32) {
    const int l = l0 + (threadIdx.x & 31);
    if (l < NP) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double x = Ug[l * NV + v];
        fin &= isfinite(x);
        if (v < 5) {
          mn[v] = fmin(mn[v], x);
          mx[v] = fmax(mx[v], x);
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 5; ++v)
    for (int o = 16; o > 0; o >>= 1) {
      mn[v] = fmin(mn[v], __shfl_xor_sync(0xffffffff, mn[v], o));
      mx[v] = fmax(mx[v], __shfl_xor_sync(0xffffffff, mx[v], o));
    }
  return __all_sync(0xffffffff, fin);
}

// The certificate worked by a whole block for one element: each thread takes nodes in a stride,
// warps combine by shuffles and every thread combines the warps.  Every thread returns the same
// value.
template <int NV>
__device__ bool nodal_certificate(const double* __restrict__ Ug, int Np, const Physics& ph, double L,
                                  double rho_floor, double p_floor, double rel) {
  __shared__ double red[10][kThreads / 32];
  double mn[5], mx[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    mn[v] = INFINITY;
    mx[v] = -INFINITY;
  }
  bool fin = true;
  for (int l = threadIdx.x; l < Np; l += blockDim.x) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double x = Ug[l * NV + v];
      fin &= isfinite(x);
      if (v < 5) {
        mn[v] = fmin(mn[v], x);
        mx[v] = fmax(mx[v], x);
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 5; ++v)
    for (int o = 16; o > 0; o >>= 1) {
      mn[v] = fmin(mn[v], __shfl_xor_sync(0xffffffff, mn[v], o));
      mx[v] = fmax(mx[v], __shfl_xor_sync(0xffffffff, mx[v], o));
    }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      red[v][threadIdx.x >> 5] = mn[v];
      red[5 + v][threadIdx.x >> 5] = mx[v];
    }
  const bool all_finite = __syncthreads_and(fin);
  if (!all_finite) return false;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    mn[v] = red[v][0];
    mx[v] = red[5 + v][0];
    for (int k = 1; k < kThreads / 32; ++k) {
      mn[v] = fmin(mn[v], red[v][k]);
      mx[v] = fmax(mx[v], red[5 + v][k]);
    }
  }
  return certificate_from_range(mn, mx, ph, L, rho_floor, p_floor, rel);
}

// The SSP-RK stage blend out = alpha * base + beta * x of one element (as k_blend forms it), written
// to out, with the warp-level nodal range of the result (warp_nodal_range's layout and result).
template <int NV, int NP>
__device__ __forceinline__ bool warp_blend_range(const double* __restrict__ base, const double* __restrict__ x,
                                                 double alpha, double beta, double* __restrict__ out,
                                                 double (&mn)[5], double (&mx)[5]) {
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    mn[v] = INFINITY;
    mx[v] = -INFINITY;
  }
  bool fin = true;
#pragma unroll
  for (int l0 = 0; l0 < NP; l0 += 32) {
    const int l = l0 + (threadIdx.x & 31);
    if (l < NP) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double y = alpha * base[l * NV + v] + beta * x[l * NV + v];
        out[l * NV + v] = y;
        fin &= isfinite(y);
        if (v < 5) {
          mn[v] = fmin(mn[v], y);
          mx[v] = fmax(mx[v], y);
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 5; ++v)
    for (int o = 16; o > 0; o >>= 1) {
      mn[v] = fmin(mn[v], __shfl_xor_sync(0xffffffff, mn[v], o));
      mx[v] = fmax(mx[v], __shfl_xor_sync(0xffffffff, mx[v], o));
    }
  return __all_sync(0xffffffff, fin);
}

// k_certify on the stage blend: out = alpha * base + beta * x is written and certified in one pass.
template <int NV, int NP>
__global__ void __launch_bounds__(kThreads) k_blend_certify(const double* __restrict__ base,
                                                           const double* __restrict__ x, double alpha, double beta,
                                                           double* __restrict__ out, int E, const Physics ph,
                                                           double L, double rho_floor, double p_floor, double rel,
                                                           int* __restrict__ list, int* __restrict__ count) {
  const long long e = (long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (e >= E) return;
  double mn[5], mx[5];
  const size_t o = (size_t)e * NP * NV;
  const bool fin = warp_blend_range<NV, NP>(base + o, x + o, alpha, beta, out + o, mn, mx);
  if ((threadIdx.x & 31) == 0 && !(fin && certificate_from_range(mn, mx, ph, L, rho_floor, p_floor, rel)))
    list[atomicAdd(count, 1)] = (int)e;
}

// Certificate pre-pass, one warp per element of NP nodes: elements of block U that the
// certificate does not clear are appended to list (in no fixed order; each is then processed on
// its own, so results do not depend on it).  *count must be zero before the launch.
template <int NV, int NP>
__global__ void __launch_bounds__(kThreads) k_certify(const double* __restrict__ U, int E, const Physics ph, double L,
                                                     double rho_floor, double p_floor, double rel,
                                                     int* __restrict__ list, int* __restrict__ count) {
  const long long e = (long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (e >= E) return;
  double mn[5], mx[5];
  const bool fin = warp_nodal_range<NV, NP>(U + e * NP * NV, mn, mx);
  if ((threadIdx.x & 31) == 0 && !(fin && certificate_from_range(mn, mx, ph, L, rho_floor, p_floor, rel)))
    list[atomicAdd(count, 1)] = (int)e;
}

// samples = [U at nodes; B U at volume points; Bfs U at face points]  -> S[Ns_total][NV]
template <int NV>
__device__ void build_samples(const BlockDev& B, const double* U, double* S) {
  const int Np = B.Np, Nq = B.Nq, Ns = B.Ns;
  const int total = (Np + Nq + Ns) * NV;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int r = idx / NV, v = idx % NV;
    double val;
    if (r < Np) {
      val = U[r * NV + v];
    } else {
      const double* row = r < Np + Nq ? B.B + (size_t)(r - Np) * Np : B.fsB + (size_t)(r - Np - Nq) * Np;
      double s = 0.0;
      for (int i = 0; i < Np; ++i) s += row[i] * U[i * NV + v];
      val = s;
    }
    S[idx] = val;
  }
}

// Cell mean: sum_q wdet (B U) / sum_q wdet, from the volume samples [q][v], worked by all threads
// (a strided sum per thread, shuffles per warp, the warps added in order by thread 0); ends with
// the block synchronised and mean[] set.
template <int NV>
__device__ void cell_mean(const BlockDev& B, int e, const double* Svol, double* mean) {
  __shared__ double part[kThreads / 32][NV + 1];
  const double* wdet = B.wdet + (size_t)e * B.Nq;
  double s[NV + 1];
#pragma unroll
  for (int v = 0; v <= NV; ++v) s[v] = 0.0;
  for (int q = threadIdx.x; q < B.Nq; q += blockDim.x) {
    const double w = wdet[q];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] += Svol[q * NV + v] * w;
    s[NV] += w;
  }
#pragma unroll
  for (int v = 0; v <= NV; ++v)
    for (int o = 16; o > 0; o >>= 1) s[v] += __shfl_xor_sync(0xffffffff, s[v], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int v = 0; v <= NV; ++v) part[threadIdx.x >> 5][v] = s[v];
  __syncthreads();
  if (threadIdx.x < NV) {
    double a = 0.0, w = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += part[k][threadIdx.x];
      w += part[k][NV];
    }
    mean[threadIdx.x] = a / w;
  }
  __syncthreads();
}

template <int NV>
__global__ void __launch_bounds__(kThreads) k_positivity(const DevPlan P, const StatePtrs S, int b,
                                                        const LimiterConst L) {
  extern __shared__ double smem[];
  __shared__ double mean[NV];
  __shared__ double sh_theta_rho;
  const BlockDev& B = P.blk[b];
  const int e = blockIdx.x;
  const int Np = B.Np, Nq = B.Nq;
  const int Nt = Np + Nq + B.Ns;
  double* U = smem;
  double* Smp = U + Np * NV;
  double* Ug = S.b[b] + (size_t)e * Np * NV;
  // nodal certificate of theta = 1: the state stays as it is (mean + 1 * (U - mean) is U to rounding)
  if (nodal_certificate<NV>(Ug, Np, P.ph, B.lebesgue, L.density_floor, L.pressure_floor, L.relative_floor)) return;
  for (int i = threadIdx.x; i < Np * NV; i += blockDim.x) U[i] = Ug[i];
  __syncthreads();
  build_samples<NV>(B, U, Smp);
  __syncthreads();
  cell_mean<NV>(B, e, Smp + Np * NV, mean);
  __syncthreads();
  double Wm[NV];
  primitive<NV>(P.ph, mean, Wm);
  const double rfloor = fmax(L.density_floor, L.relative_floor * Wm[0]);
  const double pfloor = fmax(L.pressure_floor, L.relative_floor * Wm[4]);
  // minimum sampled density
  double rmin = INFINITY;
  bool nan_seen = false;
  for (int r = threadIdx.x; r < Nt; r += blockDim.x) {
    const double d = Smp[r * NV];
    nan_seen |= isnan(d);
    rmin = fmin(rmin, d);
  }
  // block min (NaN propagates like a jnp.min)
  __shared__ double red[kThreads / 32];
  __shared__ int red_nan;
  if (threadIdx.x == 0) red_nan = 0;
  for (int o = 16; o > 0; o >>= 1) rmin = fmin(rmin, __shfl_xor_sync(0xffffffff, rmin, o));
  __syncthreads();
  if (nan_seen) atomicOr(&red_nan, 1);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rmin;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int k = 1; k < kThreads / 32; ++k) m = fmin(m, red[k]);
    if (red_nan) m = NAN;
    const double denom = mean[0] - m;
    const double th = (m < rfloor) ? (mean[0] - rfloor) / fmax(denom, 1.0e-30) : 1.0;
    // jnp.clip(x, 0, 1) keeps NaN as NaN
    sh_theta_rho = isnan(th) ? th : fmin(fmax(th, 0.0), 1.0);
  }
  __syncthreads();
  const double upper = sh_theta_rho;
  // pressure admissibility of mean + theta*(sample - mean) at every sample
  auto pressure_ok = [&](double theta) -> bool {
    bool ok = true;
    for (int r = threadIdx.x; r < Nt; r += blockDim.x) {
      double s[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) s[v] = mean[v] + theta * (Smp[r * NV + v] - mean[v]);
      ok &= (pressure_of<NV>(P.ph, s) >= pfloor);
    }
    return __syncthreads_and(ok);
  };
  // theta = upper when the pressure is admissible there; only otherwise is the reference's
  // 30-step bisection result used, so it is computed only in that case (same theta)
  double theta = upper;
  if (!pressure_ok(upper)) {
    double lo = 0.0, hi = upper;
    for (int it = 0; it < 30; ++it) {
      const double mid = 0.5 * (lo + hi);
      const bool ok = pressure_ok(mid);
      lo = ok ? mid : lo;
      hi = ok ? hi : mid;
    }
    theta = lo;
  }
  for (int idx = threadIdx.x; idx < Np * NV; idx += blockDim.x) {
    const int v = idx % NV;
    Ug[idx] = mean[v] + theta * (U[idx] - mean[v]);
  }
}

// Learned-predictor hooks of the troubled-cell kernels.  mode 1 (learned): an element whose
// predicted flag is set goes to the subcell scheme without the a-posteriori test; mode 2
// (evaluate): every element is tested and the flag is the test's, the prediction is only
// counted.  counts: [1] predicted, [2] missed (tested troubled, not predicted),
// [3] false positive and [4] hit (mode 2 only).
struct PredictArgs {
  const uint8_t* pred;
  int mode;
  unsigned long long* counts;
};

__device__ __forceinline__ bool predicted_skip(const PredictArgs& pa, int e, uint8_t* flag_out) {
  if (pa.mode != 1 || !pa.pred || !pa.pred[e]) return false;
  if (threadIdx.x == 0) {
    if (flag_out) flag_out[e] = 1;
    if (pa.counts) atomicAdd(pa.counts + 1, 1ULL);
  }
  return true;
}

__device__ __forceinline__ void count_prediction(const PredictArgs& pa, int e, bool detected) {
  if (!pa.counts || !pa.pred || pa.mode == 0) return;
  const bool pr = pa.pred[e] != 0;
  if (pa.mode == 2 && pr) atomicAdd(pa.counts + 1, 1ULL);
  if (detected && !pr) atomicAdd(pa.counts + 2, 1ULL);
  if (pa.mode == 2 && pr && !detected) atomicAdd(pa.counts + 3, 1ULL);
  if (pa.mode == 2 && pr && detected) atomicAdd(pa.counts + 4, 1ULL);
}

template <int NV>
__global__ void __launch_bounds__(kThreads) k_troubled(const DevPlan P, const StatePtrs S, int b, const LimiterConst L,
                                                      double* sensor_out, uint8_t* flag_out, const PredictArgs pa) {
  extern __shared__ double smem[];
  __shared__ double mean[NV];
  __shared__ double red[4][kThreads / 32];
  const BlockDev& B = P.blk[b];
  const int e = blockIdx.x;
  if (predicted_skip(pa, e, flag_out)) return;
  const int Np = B.Np, Nq = B.Nq;
  const int Nt = Np + Nq + B.Ns;
  double* U = smem;
  double* Smp = U + Np * NV;
  double* Mon = Smp + Nt * NV;   // [Np][2] monitored (rho, p)
  const double* Ug = S.b[b] + (size_t)e * Np * NV;
  // nodal certificate of admissible samples and mean: then only the sensor needs computing
  const bool certified = nodal_certificate<NV>(Ug, Np, P.ph, B.lebesgue, L.density_floor, L.pressure_floor, 0.0);
  for (int i = threadIdx.x; i < Np * NV; i += blockDim.x) U[i] = Ug[i];
  __syncthreads();
  if (!certified) build_samples<NV>(B, U, Smp);
  for (int i = threadIdx.x; i < Np; i += blockDim.x) {
    double W[NV];
    primitive<NV>(P.ph, U + i * NV, W);
    Mon[i * 2 + 0] = W[0];
    Mon[i * 2 + 1] = W[4];
  }
  __syncthreads();
  if (!certified) cell_mean<NV>(B, e, Smp + Np * NV, mean);
  // sensor: sum_i (m - Pi m)^2 / max(sum_i m^2, 1e-12), max over (rho, p)
  double hi0 = 0.0, hi1 = 0.0, sc0 = 0.0, sc1 = 0.0;
  if (P.degree >= 2) {
    for (int i = threadIdx.x; i < Np; i += blockDim.x) {
      double l0 = 0.0, l1 = 0.0;
      for (int j = 0; j < Np; ++j) {
        l0 += B.p1proj[(size_t)i * Np + j] * Mon[j * 2 + 0];
        l1 += B.p1proj[(size_t)i * Np + j] * Mon[j * 2 + 1];
      }
      const double d0 = Mon[i * 2 + 0] - l0, d1 = Mon[i * 2 + 1] - l1;
      hi0 += d0 * d0;
      hi1 += d1 * d1;
      sc0 += Mon[i * 2 + 0] * Mon[i * 2 + 0];
      sc1 += Mon[i * 2 + 1] * Mon[i * 2 + 1];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    hi0 += __shfl_xor_sync(0xffffffff, hi0, o);
    hi1 += __shfl_xor_sync(0xffffffff, hi1, o);
    sc0 += __shfl_xor_sync(0xffffffff, sc0, o);
    sc1 += __shfl_xor_sync(0xffffffff, sc1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = hi0;
    red[1][threadIdx.x >> 5] = hi1;
    red[2][threadIdx.x >> 5] = sc0;
    red[3][threadIdx.x >> 5] = sc1;
  }
  __syncthreads();
  // invalid samples (including the cell mean)
  bool bad = false;
  for (int r = threadIdx.x; r <= (certified ? -1 : Nt); r += blockDim.x) {
    const double* s = r < Nt ? Smp + r * NV : mean;
    double W[NV];
    primitive<NV>(P.ph, s, W);
    bool finite = true;
#pragma unroll
    for (int v = 0; v < NV; ++v) finite &= isfinite(W[v]);
    bad |= !finite || (W[0] < L.density_floor) || (W[4] < L.pressure_floor);
  }
  const bool any_bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    double h0 = 0, h1 = 0, s0 = 0, s1 = 0;
    for (int k = 0; k < kThreads / 32; ++k) {
      h0 += red[0][k]; h1 += red[1][k]; s0 += red[2][k]; s1 += red[3][k];
    }
    double value = 0.0;
    if (P.degree >= 2) {
      const double r0 = h0 / fmax(s0, 1.0e-12), r1 = h1 / fmax(s1, 1.0e-12);
      value = (isnan(r0) || isnan(r1)) ? NAN : fmax(r0, r1);
    }
    const bool detected = (value > L.sensor_threshold) || any_bad;
    if (sensor_out) sensor_out[e] = value;
    if (flag_out) flag_out[e] = (uint8_t)detected;
    count_prediction(pa, e, detected);
  }
}

// ---------------------------------------------------------------- reductions
struct Partial {
  double a, b;   // (max rate) or (rho_min, p_min)
  int flag;      // finite / nan seen
  int pad;
};

template <int NV>
__global__ void __launch_bounds__(kThreads) k_rate(const DevPlan P, const StatePtrs S, int b, double cp,
                                                  Partial* partials, int offset) {
  // one warp per element; grid-stride over elements
  const BlockDev& B = P.blk[b];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const double df = 2.0 * P.degree + 1.0;
  double best = -INFINITY;
  for (int e = warp; e < B.E; e += nwarps) {
    const double* U = S.b[b] + (size_t)e * B.Np * NV;
    double smax = -INFINITY, rsum = 0.0;
    bool en = false;
    for (int i = lane; i < B.Np; i += 32) {
      double W[NV];
      primitive<NV>(P.ph, U + i * NV, W);
      // jnp.maximum propagates NaN where fmax drops it: a NaN density or pressure makes the
      // reference's rate NaN (then 1e7), so it is flagged before the floors
      const double rho = fmax(W[0], 1.0e-14), p = fmax(W[4], 1.0e-14);
      const double sp = sqrt(W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) + sqrt(P.ph.gamma * p / rho);
      en |= isnan(W[0]) || isnan(W[4]) || isnan(sp);
      smax = fmax(smax, sp);
      rsum += rho;
    }
    for (int o = 16; o > 0; o >>= 1) {
      smax = fmax(smax, __shfl_xor_sync(0xffffffff, smax, o));
      rsum += __shfl_xor_sync(0xffffffff, rsum, o);
    }
    en = __any_sync(0xffffffff, en);
    const double h = B.length[e];
    double rate = en ? NAN : df * smax / h;
    if (P.viscous) {
      const double rmin = fmax(rsum / B.Np, 0.1);
      const CaseView cv = case_view(P.ph, B.ecase, e);
      const double diff = fmax((4.0 / 3.0) * cv.mu / rmin, cv.kappa / (rmin * cp));
      const double vl = fmax(h, 0.01);
      rate = rate + 2.0 * P.ph.br2 * df * df * diff / (vl * vl);
    }
    // jnp.nan_to_num(rate, nan=1e7, posinf=1e7)
    if (isnan(rate) || (isinf(rate) && rate > 0.0)) rate = 1.0e7;
    else if (isinf(rate)) rate = -1.7976931348623157e308;
    best = fmax(best, rate);
  }
  __shared__ double red[kThreads / 32];
  if (lane == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int k = 1; k < kThreads / 32; ++k) m = fmax(m, red[k]);
    partials[offset + blockIdx.x].a = m;
  }
}

__global__ void k_dt(const Partial* partials, int n, double cfl, double* dt_out) {
  __shared__ double red[kThreads];
  double m = -INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, partials[i].a);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double dt = cfl / fmax(red[0], 1.0e-12);
    *dt_out = fmin(fmax(dt, 1.0e-7), 1.0e-3);
  }
}

template <int NV>
__global__ void __launch_bounds__(kThreads) k_adm(const DevPlan P, const StatePtrs S, int b, Partial* partials,
                                                 int offset) {
  const BlockDev& B = P.blk[b];
  const size_t nodes = (size_t)B.E * B.Np;
  double rmin = INFINITY, pmin = INFINITY;
  int finite = 1, rnan = 0, pnan = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nodes; k += (size_t)gridDim.x * blockDim.x) {
    const double* U = S.b[b] + k * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) finite &= isfinite(U[v]) ? 1 : 0;
    const double p = pressure_of<NV>(P.ph, U);
    rnan |= isnan(U[0]);
    pnan |= isnan(p);
    rmin = fmin(rmin, U[0]);
    pmin = fmin(pmin, p);
  }
  for (int o = 16; o > 0; o >>= 1) {
    rmin = fmin(rmin, __shfl_xor_sync(0xffffffff, rmin, o));
    pmin = fmin(pmin, __shfl_xor_sync(0xffffffff, pmin, o));
  }
  finite = __syncthreads_and(finite);
  rnan = __syncthreads_or(rnan);
  pnan = __syncthreads_or(pnan);
  __shared__ double r1[kThreads / 32], r2[kThreads / 32];
  if ((threadIdx.x & 31) == 0) {
    r1[threadIdx.x >> 5] = rmin;
    r2[threadIdx.x >> 5] = pmin;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = r1[0], c = r2[0];
    for (int k = 1; k < kThreads / 32; ++k) {
      a = fmin(a, r1[k]);
      c = fmin(c, r2[k]);
    }
    Partial out;
    out.a = rnan ? NAN : a;
    out.b = pnan ? NAN : c;
    out.flag = finite;
    out.pad = 0;
    partials[offset + blockIdx.x] = out;
  }
}

// combine: first stage overwrites the status, later stages AND / min into it.  One CTA of
// kAdmFinalThreads reduces the partials (a serial loop over thousands of them took 0.3 ms).
constexpr int kAdmFinalThreads = 256;

__global__ void __launch_bounds__(kAdmFinalThreads) k_adm_final(const Partial* partials, int n, double rho_floor,
                                                               double p_floor, int combine, dgb_status* status) {
  __shared__ double sr[kAdmFinalThreads], sp[kAdmFinalThreads];
  double rmin = INFINITY, pmin = INFINITY;
  int finite = 1, rnan = 0, pnan = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const Partial q = partials[i];
    rnan |= isnan(q.a);
    pnan |= isnan(q.b);
    rmin = fmin(rmin, q.a);
    pmin = fmin(pmin, q.b);
    finite &= q.flag;
  }
  finite = __syncthreads_and(finite);
  rnan = __syncthreads_or(rnan);
  pnan = __syncthreads_or(pnan);
  sr[threadIdx.x] = rmin;
  sp[threadIdx.x] = pmin;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sr[threadIdx.x] = fmin(sr[threadIdx.x], sr[threadIdx.x + s]);
      sp[threadIdx.x] = fmin(sp[threadIdx.x], sp[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  rmin = rnan ? NAN : sr[0];
  pmin = pnan ? NAN : sp[0];
  const int valid = finite && (rmin >= rho_floor) && (pmin >= p_floor);
  if (combine) {
    status->valid = status->valid && valid;
    status->rho_min = (isnan(status->rho_min) || isnan(rmin)) ? NAN : fmin(status->rho_min, rmin);
    status->p_min = (isnan(status->p_min) || isnan(pmin)) ? NAN : fmin(status->p_min, pmin);
  } else {
    status->valid = valid;
    status->rho_min = rmin;
    status->p_min = pmin;
  }
}

}  // namespace dgb
