// Learned troubled-cell predictor: element features, inference and training (no reference
// counterpart; the reference only has the a-posteriori MOOD detector, hybrid/limiter.py:150-185,
// 285-300, which stays the arbiter).
//
// Features (8 per element, from the stage's base state, before the high-order update):
//   0, 1  log10 of the Persson high-mode fraction of rho and of p (the detector's sensor:
//         ||m - P1 m||^2 / ||m||^2 over the element's nodes)
//   2, 3  largest relative jump of the nodal-mean rho and p across the element's faces
//   4, 5  min / max of rho and of p over the element's nodes
//   6, 7  the element's mean rho and p over the largest neighbouring mean
// Network: 8 -> 64 -> 64 -> 64 -> 1, ReLU hidden layers, sigmoid output.  Inference keeps the
// weights in float16 and accumulates in float32; training keeps float32 master weights (Adam).
#pragma once
#include <cuda_fp16.h>

#include "dg_kernels.cuh"

namespace dgb {

constexpr int kMlpIn = 8, kMlpH = 64, kMlpStats = 6;
// parameter offsets: W1 [8][64], b1, W2 [64][64], b2, W3 [64][64], b3, w4 [64], b4
constexpr int kW1 = 0, kB1 = kW1 + kMlpIn * kMlpH, kW2 = kB1 + kMlpH, kB2 = kW2 + kMlpH * kMlpH;
constexpr int kW3 = kB2 + kMlpH, kB3 = kW3 + kMlpH * kMlpH, kW4 = kB3 + kMlpH, kB4 = kW4 + kMlpH;
constexpr int kMlpParams = kB4 + 1;   // 8961

// ---------------------------------------------------------------- features
// One warp per element: nodal primitive rho and p, their means and extrema, and the Persson
// fractions with the block's P1 projector.  stats[e] = mean rho, mean p, min/max rho,
// min/max p, fraction rho, fraction p.
template <int NV>
__global__ void __launch_bounds__(kThreads) k_elem_stats(const DevPlan P, const StatePtrs S, int b,
                                                        float* __restrict__ stats) {
  extern __shared__ double smem[];
  const BlockDev& B = P.blk[b];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * (kThreads / 32) + warp;
  const int Np = B.Np;
  double* mon = smem + warp * 2 * Np;            // [Np][2]
  const bool live = e < B.E;
  double srho = 0, sp = 0, rmin = INFINITY, rmax = -INFINITY, pmin = INFINITY, pmax = -INFINITY;
  if (live) {
    const double* U = S.b[b] + (size_t)e * Np * NV;
    for (int i = lane; i < Np; i += 32) {
      double u[NV], W[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = U[i * NV + v];
      primitive<NV>(P.ph, u, W);
      mon[i * 2 + 0] = W[0];
      mon[i * 2 + 1] = W[4];
      srho += W[0];
      sp += W[4];
      rmin = fmin(rmin, W[0]);
      rmax = fmax(rmax, W[0]);
      pmin = fmin(pmin, W[4]);
      pmax = fmax(pmax, W[4]);
    }
  }
  __syncwarp();
  double h0 = 0, h1 = 0, s0 = 0, s1 = 0;
  if (live && P.degree >= 2) {
    for (int i = lane; i < Np; i += 32) {
      const double* row = B.p1proj + (size_t)i * Np;
      double l0 = 0, l1 = 0;
      for (int j = 0; j < Np; ++j) {
        const double pj = __ldg(row + j);
        l0 += pj * mon[j * 2 + 0];
        l1 += pj * mon[j * 2 + 1];
      }
      const double m0 = mon[i * 2 + 0], m1 = mon[i * 2 + 1];
      h0 += (m0 - l0) * (m0 - l0);
      h1 += (m1 - l1) * (m1 - l1);
      s0 += m0 * m0;
      s1 += m1 * m1;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    srho += __shfl_xor_sync(0xffffffff, srho, o);
    sp += __shfl_xor_sync(0xffffffff, sp, o);
    rmin = fmin(rmin, __shfl_xor_sync(0xffffffff, rmin, o));
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffff, rmax, o));
    pmin = fmin(pmin, __shfl_xor_sync(0xffffffff, pmin, o));
    pmax = fmax(pmax, __shfl_xor_sync(0xffffffff, pmax, o));
    h0 += __shfl_xor_sync(0xffffffff, h0, o);
    h1 += __shfl_xor_sync(0xffffffff, h1, o);
    s0 += __shfl_xor_sync(0xffffffff, s0, o);
    s1 += __shfl_xor_sync(0xffffffff, s1, o);
  }
  if (live && lane == 0) {
    float* st = stats + (size_t)e * kMlpStats;
    st[0] = (float)(srho / Np);
    st[1] = (float)(sp / Np);
    st[2] = (float)(rmin / fmax(fabs(rmax), 1e-30));
    st[3] = (float)(pmin / fmax(fabs(pmax), 1e-30));
    st[4] = (float)(h0 / fmax(s0, 1e-12));
    st[5] = (float)(h1 / fmax(s1, 1e-12));
  }
}

// One thread per element: neighbour means through the element's faces -> 8 features.
// stats_all[b] points at block b's stats; features are written for block b at feat.
__global__ void __launch_bounds__(kThreads) k_mlp_features(const DevPlan P, int b, const float* const* stats_all,
                                                          float* __restrict__ feat) {
  const BlockDev& B = P.blk[b];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B.E) return;
  const float* me = stats_all[b] + (size_t)e * kMlpStats;
  const float mr = me[0], mp = me[1];
  float jr = 0.f, jp = 0.f, nr = mr, np_ = mp;
  for (int lf = 0; lf < B.nlf; ++lf) {
    int ft, f, side;
    decode_face(B.elem_face[e * B.nlf + lf], ft, f, side);
    const FaceDev& fd = P.face[ft];
    const int ob = side == 0 ? fd.nb[f] : fd.ob[f];
    const int ol = side == 0 ? fd.nl[f] : fd.ol[f];
    if (ob < 0) continue;                            // boundary face: no neighbour
    const float* nbs = stats_all[ob] + (size_t)ol * kMlpStats;
    jr = fmaxf(jr, fabsf(nbs[0] - mr) / fmaxf(fabsf(mr), 1e-20f));
    jp = fmaxf(jp, fabsf(nbs[1] - mp) / fmaxf(fabsf(mp), 1e-20f));
    nr = fmaxf(nr, nbs[0]);
    np_ = fmaxf(np_, nbs[1]);
  }
  float* o = feat + (size_t)e * kMlpIn;
  o[0] = log10f(fmaxf(me[4], 1e-12f));
  o[1] = log10f(fmaxf(me[5], 1e-12f));
  o[2] = jr;
  o[3] = jp;
  o[4] = me[2];
  o[5] = me[3];
  o[6] = mr / fmaxf(nr, 1e-20f);
  o[7] = mp / fmaxf(np_, 1e-20f);
}

// ---------------------------------------------------------------- inference
// One thread per sample: normalised features -> probability; float16 weights staged in shared
// memory (every thread reads the same weight: broadcast), float32 accumulation.
// norm = [mean[8], inv_std[8]].  prob and/or flag (prob > threshold) may be null.
__global__ void __launch_bounds__(128) k_mlp_infer(const __half* __restrict__ w16, const float* __restrict__ norm,
                                                   const float* __restrict__ X, long long n, float threshold,
                                                   float* __restrict__ prob, uint8_t* __restrict__ flag) {
  __shared__ __half w[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) w[i] = w16[i];
  __syncthreads();
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) x[i] = (X[s * kMlpIn + i] - norm[i]) * norm[kMlpIn + i];
  float h[kMlpH], g[kMlpH];
#pragma unroll
  for (int j = 0; j < kMlpH; ++j) {
    float z = __half2float(w[kB1 + j]);
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) z = fmaf(x[i], __half2float(w[kW1 + i * kMlpH + j]), z);
    h[j] = fmaxf(z, 0.f);
  }
#pragma unroll
  for (int j = 0; j < kMlpH; ++j) {
    float z = __half2float(w[kB2 + j]);
#pragma unroll
    for (int i = 0; i < kMlpH; ++i) z = fmaf(h[i], __half2float(w[kW2 + i * kMlpH + j]), z);
    g[j] = fmaxf(z, 0.f);
  }
  float out = __half2float(w[kB4]);
#pragma unroll 4
  for (int j = 0; j < kMlpH; ++j) {
    float z = __half2float(w[kB3 + j]);
#pragma unroll
    for (int i = 0; i < kMlpH; ++i) z = fmaf(g[i], __half2float(w[kW3 + i * kMlpH + j]), z);
    out = fmaf(fmaxf(z, 0.f), __half2float(w[kW4 + j]), out);
  }
  const float p = 1.f / (1.f + __expf(-out));
  if (prob) prob[s] = p;
  if (flag) flag[s] = (uint8_t)(p > threshold);
}

// ---------------------------------------------------------------- training
// One CTA of 256 threads per chunk of 64 samples: forward, weighted binary cross-entropy,
// backward; the chunk's gradient is added to grad (float32, zeroed by the update kernel).
// Hidden activations H1..H3 [64 samples][64] and deltas live in shared memory; weight matrices
// are staged with a row stride of 65 floats so that column walks fall in distinct banks.
constexpr int kMlpChunk = 64, kMlpTrainThreads = 256, kWS = kMlpH + 1;
constexpr int kMlpTrainSmemFloats =
    kMlpIn * kWS + 2 * kMlpH * kWS + 4 * kMlpH + 1 + kMlpChunk * kMlpIn + 2 * kMlpChunk +
    3 * kMlpChunk * kMlpH + 2 * kMlpChunk * kMlpH + 2 * kMlpChunk;

__global__ void __launch_bounds__(kMlpTrainThreads) k_mlp_train(const float* __restrict__ wts,
                                                               const float* __restrict__ norm,
                                                               const float* __restrict__ X,
                                                               const uint8_t* __restrict__ y,
                                                               const int* __restrict__ idx, int batch,
                                                               float pos_weight, float* __restrict__ grad,
                                                               float* __restrict__ loss) {
  extern __shared__ float fs[];
  float* W1 = fs;                                  // [8][65]
  float* W2 = W1 + kMlpIn * kWS;                   // [64][65]
  float* W3 = W2 + kMlpH * kWS;                    // [64][65]
  float* bb = W3 + kMlpH * kWS;                    // b1, b2, b3, w4 (4 x 64), b4
  float* xs = bb + 4 * kMlpH + 1;                  // [64][8]
  float* ys = xs + kMlpChunk * kMlpIn;             // [64] label weight-signed targets
  float* ws = ys + kMlpChunk;                      // [64] sample weights (0 beyond the batch)
  float* H1 = ws + kMlpChunk;                      // [64][64]
  float* H2 = H1 + kMlpChunk * kMlpH;
  float* H3 = H2 + kMlpChunk * kMlpH;
  float* Da = H3 + kMlpChunk * kMlpH;              // deltas
  float* Db = Da + kMlpChunk * kMlpH;
  float* d4 = Db + kMlpChunk * kMlpH;              // [64] output delta
  float* pr = d4 + kMlpChunk;                      // [64] probabilities
  const int t = threadIdx.x;
  for (int i = t; i < kMlpIn * kMlpH; i += blockDim.x) W1[(i / kMlpH) * kWS + i % kMlpH] = wts[kW1 + i];
  for (int i = t; i < kMlpH * kMlpH; i += blockDim.x) {
    W2[(i / kMlpH) * kWS + i % kMlpH] = wts[kW2 + i];
    W3[(i / kMlpH) * kWS + i % kMlpH] = wts[kW3 + i];
  }
  for (int i = t; i < kMlpH; i += blockDim.x) {
    bb[i] = wts[kB1 + i];
    bb[kMlpH + i] = wts[kB2 + i];
    bb[2 * kMlpH + i] = wts[kB3 + i];
    bb[3 * kMlpH + i] = wts[kW4 + i];
  }
  if (t == 0) bb[4 * kMlpH] = wts[kB4];
  const int base = blockIdx.x * kMlpChunk;
  for (int i = t; i < kMlpChunk * kMlpIn; i += blockDim.x) {
    const int s = i / kMlpIn, k = i % kMlpIn;
    const int g = base + s;
    xs[i] = g < batch ? (X[(size_t)idx[g] * kMlpIn + k] - norm[k]) * norm[kMlpIn + k] : 0.f;
  }
  for (int s = t; s < kMlpChunk; s += blockDim.x) {
    const int g = base + s;
    const float lab = g < batch ? (float)y[idx[g]] : 0.f;
    ys[s] = lab;
    ws[s] = g < batch ? (lab > 0.5f ? pos_weight : 1.f) / (float)batch : 0.f;
  }
  __syncthreads();
  const int j = t % kMlpH, s0 = t / kMlpH;          // output unit, first sample of this thread
  // forward
  for (int s = s0; s < kMlpChunk; s += kMlpTrainThreads / kMlpH) {
    float z = bb[j];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) z = fmaf(xs[s * kMlpIn + i], W1[i * kWS + j], z);
    H1[s * kMlpH + j] = fmaxf(z, 0.f);
  }
  __syncthreads();
  for (int s = s0; s < kMlpChunk; s += kMlpTrainThreads / kMlpH) {
    float z = bb[kMlpH + j];
    for (int i = 0; i < kMlpH; ++i) z = fmaf(H1[s * kMlpH + i], W2[i * kWS + j], z);
    H2[s * kMlpH + j] = fmaxf(z, 0.f);
  }
  __syncthreads();
  for (int s = s0; s < kMlpChunk; s += kMlpTrainThreads / kMlpH) {
    float z = bb[2 * kMlpH + j];
    for (int i = 0; i < kMlpH; ++i) z = fmaf(H2[s * kMlpH + i], W3[i * kWS + j], z);
    H3[s * kMlpH + j] = fmaxf(z, 0.f);
  }
  __syncthreads();
  if (t < kMlpChunk) {
    float z = bb[4 * kMlpH];
    for (int i = 0; i < kMlpH; ++i) z = fmaf(H3[t * kMlpH + i], bb[3 * kMlpH + i], z);
    const float p = 1.f / (1.f + expf(-z));
    pr[t] = p;
    d4[t] = ws[t] * (p - ys[t]);                    // d(weighted BCE)/dz
    if (loss && ws[t] > 0.f) {
      const float l = ys[t] > 0.5f ? -logf(fmaxf(p, 1e-12f)) : -logf(fmaxf(1.f - p, 1e-12f));
      atomicAdd(loss, ws[t] * l);
    }
  }
  __syncthreads();
  // output layer gradients and delta of layer 3
  if (t < kMlpH) {
    float gw = 0.f, gb = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) gw = fmaf(H3[s * kMlpH + t], d4[s], gw);
    atomicAdd(grad + kW4 + t, gw);
    if (t == 0) {
      for (int s = 0; s < kMlpChunk; ++s) gb += d4[s];
      atomicAdd(grad + kB4, gb);
    }
  }
  for (int s = s0; s < kMlpChunk; s += kMlpTrainThreads / kMlpH)
    Da[s * kMlpH + j] = H3[s * kMlpH + j] > 0.f ? d4[s] * bb[3 * kMlpH + j] : 0.f;
  __syncthreads();
  // layer 3: dW3[i][j] = sum_s H2[s][i] Da[s][j]; delta2 = (Da W3^T) * (H2 > 0)
  for (int i = s0; i < kMlpH; i += kMlpTrainThreads / kMlpH) {
    float g = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) g = fmaf(H2[s * kMlpH + i], Da[s * kMlpH + j], g);
    atomicAdd(grad + kW3 + i * kMlpH + j, g);
  }
  if (t < kMlpH) {
    float g = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) g += Da[s * kMlpH + t];
    atomicAdd(grad + kB3 + t, g);
  }
  for (int s = s0; s < kMlpChunk; s += kMlpTrainThreads / kMlpH) {
    const int i = j;
    float d = 0.f;
    for (int k = 0; k < kMlpH; ++k) d = fmaf(Da[s * kMlpH + k], W3[i * kWS + k], d);
    Db[s * kMlpH + i] = H2[s * kMlpH + i] > 0.f ? d : 0.f;
  }
  __syncthreads();
  // layer 2
  for (int i = s0; i < kMlpH; i += kMlpTrainThreads / kMlpH) {
    float g = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) g = fmaf(H1[s * kMlpH + i], Db[s * kMlpH + j], g);
    atomicAdd(grad + kW2 + i * kMlpH + j, g);
  }
  if (t < kMlpH) {
    float g = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) g += Db[s * kMlpH + t];
    atomicAdd(grad + kB2 + t, g);
  }
  for (int s = s0; s < kMlpChunk; s += kMlpTrainThreads / kMlpH) {
    const int i = j;
    float d = 0.f;
    for (int k = 0; k < kMlpH; ++k) d = fmaf(Db[s * kMlpH + k], W2[i * kWS + k], d);
    Da[s * kMlpH + i] = H1[s * kMlpH + i] > 0.f ? d : 0.f;
  }
  __syncthreads();
  // layer 1
  for (int i = s0; i < kMlpIn; i += kMlpTrainThreads / kMlpH) {
    float g = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) g = fmaf(xs[s * kMlpIn + i], Da[s * kMlpH + j], g);
    atomicAdd(grad + kW1 + i * kMlpH + j, g);
  }
  if (t < kMlpH) {
    float g = 0.f;
    for (int s = 0; s < kMlpChunk; ++s) g += Da[s * kMlpH + t];
    atomicAdd(grad + kB1 + t, g);
  }
}

// Adam (Kingma & Ba 2015) on the float32 master weights; clears grad; refreshes the float16 copy.
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ grad, float* __restrict__ m,
                           float* __restrict__ v, __half* __restrict__ w16, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float g = grad[i];
  grad[i] = 0.f;
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  w[i] = wi;
  if (w16) w16[i] = __float2half_rn(wi);
}

}  // namespace dgb
