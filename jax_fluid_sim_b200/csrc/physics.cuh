// Pointwise compressible-flow physics shared by the DG kernels, templated on the real type T
// (float64 for the plain path; float32 inside the mixed-precision volume and lift kernels).
//
// Same arithmetic as the reference's hybrid/solver.py:
//   conserved_to_primitive  :83-98   (density floored at 1e-14 in divisions only)
//   normal_physical_flux    :100-122
//   rusanov_flux            :132-152
//   hllc_wave_speeds/_star  :163-243 (_safe_signed :154-161)
//   hllc_flux               :245-300 (Rusanov fallback, identical-state shortcut)
//   viscous_variables       :307-315
//   viscous_physical_flux   :357-406 (constant mu, kappa per case; WALE off)
// and hybrid/boundary.py:54-102 for the ghost states.
#pragma once
#include <math.h>
#include <stdint.h>

#include "../../include/dgb200.h"

namespace dgb {

constexpr double kRhoFloor = 1.0e-14;

struct Physics {
  double gamma, R, mu, kappa, br2;
  int has_boundary;
  double farfield_W[DGB_MAX_VARS];
  int inlet[DGB_MAX_TAGS], n_inlet;
  int wall[DGB_MAX_TAGS], n_wall;
  int no_slip[DGB_MAX_TAGS], n_no_slip;
  int slip[DGB_MAX_TAGS], n_slip;
  int has_wall_T;
  double wall_T;
  // ensembles of independent cases in one plan (optional): per case [mu, kappa, T_wall,
  // far-field primitive (nvars)], case_stride = 3 + nvars; elements carry their case id
  const double* cases;
  int case_stride;
};

// The transport coefficients, wall temperature and far-field state that apply to one element.
struct CaseView {
  double mu, kappa, wall_T;
  const double* far;
};

__device__ __forceinline__ CaseView case_view(const Physics& ph, const int32_t* element_case, size_t e) {
  if (ph.cases == nullptr || element_case == nullptr) return CaseView{ph.mu, ph.kappa, ph.wall_T, ph.farfield_W};
  const double* c = ph.cases + (size_t)element_case[e] * ph.case_stride;
  return CaseView{c[0], c[1], c[2], c + 3};
}

__device__ __forceinline__ bool tag_in(int tag, const int* set, int n) {
  bool hit = false;
  for (int i = 0; i < n; ++i) hit |= (set[i] == tag);
  return hit;
}

// The EOS and Euler-flux arithmetic below is written with explicit round-to-nearest
// intrinsics so the compiler cannot contract it into FMAs differently at different call
// sites: identical states then give bit-identical fluxes everywhere, which keeps the
// anchor-form residual exactly zero for a uniform state (hybrid/spatial.py:41-45).
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

template <int NV, typename T>
__device__ __forceinline__ void primitive(const Physics& ph, const T* U, T* W) {
  const T rho = U[0];
  const T srho = fmax(rho, T(kRhoFloor));
  W[0] = rho;
  W[1] = U[1] / srho;
  W[2] = U[2] / srho;
  W[3] = U[3] / srho;
  const T m2 = add(add(mul(U[1], U[1]), mul(U[2], U[2])), mul(U[3], U[3]));
  const T ke = mul(T(0.5), m2) / srho;
  W[4] = mul(T(ph.gamma - 1.0), sub(U[4], ke));
#pragma unroll
  for (int s = 5; s < NV; ++s) W[s] = U[s] / srho;
}

template <int NV, typename T>
__device__ __forceinline__ void conserved(const Physics& ph, const T* W, T* U) {
  const T rho = W[0];
  U[0] = rho;
  U[1] = mul(rho, W[1]);
  U[2] = mul(rho, W[2]);
  U[3] = mul(rho, W[3]);
  const T v2 = add(add(mul(W[1], W[1]), mul(W[2], W[2])), mul(W[3], W[3]));
  U[4] = add(W[4] / T(ph.gamma - 1.0), mul(mul(T(0.5), rho), v2));
#pragma unroll
  for (int s = 5; s < NV; ++s) U[s] = mul(rho, W[s]);
}

template <int NV, typename T>
__device__ __forceinline__ void normal_flux(const Physics& ph, const T* U, const T* n, T* F) {
  T W[NV];
  primitive<NV>(ph, U, W);
  const T un = add(add(mul(W[1], n[0]), mul(W[2], n[1])), mul(W[3], n[2]));
  const T ru = mul(W[0], un);
  F[0] = ru;
  F[1] = add(mul(mul(W[0], W[1]), un), mul(W[4], n[0]));
  F[2] = add(mul(mul(W[0], W[2]), un), mul(W[4], n[1]));
  F[3] = add(mul(mul(W[0], W[3]), un), mul(W[4], n[2]));
  F[4] = mul(un, add(U[4], W[4]));
#pragma unroll
  for (int s = 5; s < NV; ++s) F[s] = mul(U[s], un);
}

template <int NV>
__device__ __forceinline__ void rusanov(const Physics& ph, const double* UL, const double* UR, const double* n,
                                        double* F) {
  double WL[NV], WR[NV], FL[NV], FR[NV];
  primitive<NV>(ph, UL, WL);
  primitive<NV>(ph, UR, WR);
  const double unl = WL[1] * n[0] + WL[2] * n[1] + WL[3] * n[2];
  const double unr = WR[1] * n[0] + WR[2] * n[1] + WR[3] * n[2];
  const double cl = sqrt(ph.gamma * fmax(WL[4], 0.0) / fmax(WL[0], kRhoFloor));
  const double cr = sqrt(ph.gamma * fmax(WR[4], 0.0) / fmax(WR[0], kRhoFloor));
  const double smax = fmax(fabs(unl) + cl, fabs(unr) + cr);
  normal_flux<NV>(ph, UL, n, FL);
  normal_flux<NV>(ph, UR, n, FR);
#pragma unroll
  for (int v = 0; v < NV; ++v) F[v] = 0.5 * (FL[v] + FR[v]) - 0.5 * smax * (UR[v] - UL[v]);
}

__device__ __forceinline__ double safe_signed(double v) {
  const double tol = 1.0e-14;
  return fabs(v) > tol ? v : (v >= 0.0 ? tol : -tol);
}

// Star state between acoustic wave `s` and the contact `sm`.
template <int NV>
__device__ __forceinline__ void hllc_star(const Physics& ph, const double* U, const double* W, double s, double sm,
                                          const double* n, double* S) {
  const double un = W[1] * n[0] + W[2] * n[1] + W[3] * n[2];
  const double den = safe_signed(s - sm);
  const double comp = (s - un) / den;
  const double rs = W[0] * comp;
  S[0] = rs;
  S[1] = rs * (W[1] + (sm - un) * n[0]);
  S[2] = rs * (W[2] + (sm - un) * n[1]);
  S[3] = rs * (W[3] + (sm - un) * n[2]);
  const double ps = W[4] + W[0] * (s - un) * (sm - un);
  S[4] = ((s - un) * U[4] - W[4] * un + ps * sm) / den;
#pragma unroll
  for (int v = 5; v < NV; ++v) S[v] = U[v] * comp;
}

template <int NV>
__device__ void hllc(const Physics& ph, const double* UL, const double* UR, const double* n, double* F) {
  bool identical = true;
#pragma unroll
  for (int v = 0; v < NV; ++v) identical &= (UL[v] == UR[v]);
  double WL[NV], WR[NV], FL[NV], FR[NV];
  primitive<NV>(ph, UL, WL);
  primitive<NV>(ph, UR, WR);
  normal_flux<NV>(ph, UL, n, FL);
  if (identical) {
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = FL[v];
    return;
  }
  normal_flux<NV>(ph, UR, n, FR);
  const double rl = WL[0], rr = WR[0], pl = WL[4], pr = WR[4];
  const double unl = WL[1] * n[0] + WL[2] * n[1] + WL[3] * n[2];
  const double unr = WR[1] * n[0] + WR[2] * n[1] + WR[3] * n[2];
  const double cl = sqrt(fmax(ph.gamma * pl / fmax(rl, kRhoFloor), 0.0));
  const double cr = sqrt(fmax(ph.gamma * pr / fmax(rr, kRhoFloor), 0.0));
  const double sl = fmin(unl - cl, unr - cr);
  const double sr = fmax(unl + cl, unr + cr);
  const double den = rl * (sl - unl) - rr * (sr - unr);
  const double sm = (pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr)) / safe_signed(den);
  bool finite = true;
  if (sl >= 0.0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = FL[v];
  } else if (sm >= 0.0) {
    double S[NV];
    hllc_star<NV>(ph, UL, WL, sl, sm, n, S);
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = FL[v] + sl * (S[v] - UL[v]);
  } else if (sr > 0.0) {
    double S[NV];
    hllc_star<NV>(ph, UR, WR, sr, sm, n, S);
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = FR[v] + sr * (S[v] - UR[v]);
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = FR[v];
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) finite &= isfinite(F[v]);
  const bool valid = (rl > 0.0) && (rr > 0.0) && (pl > 0.0) && (pr > 0.0) && finite;
  if (!valid) rusanov<NV>(ph, UL, UR, n, F);
}

// Inviscid ghost state: slip reflection on walls, far-field on inlets, copy elsewhere.
template <int NV>
__device__ void ghost_state(const Physics& ph, const double* far, const double* U, const double* n, int tag,
                            double* G) {
  double W[NV];
  primitive<NV>(ph, U, W);
  if (tag_in(tag, ph.wall, ph.n_wall)) {
    const double un = W[1] * n[0] + W[2] * n[1] + W[3] * n[2];
    W[1] = W[1] - 2.0 * un * n[0];
    W[2] = W[2] - 2.0 * un * n[1];
    W[3] = W[3] - 2.0 * un * n[2];
  }
  if (tag_in(tag, ph.inlet, ph.n_inlet)) {
#pragma unroll
    for (int v = 0; v < NV; ++v) W[v] = far[v];
  }
  conserved<NV>(ph, W, G);
}

template <int NV, typename T>
__device__ __forceinline__ void viscous_vars(const Physics& ph, const T* U, T* out) {
  T W[NV];
  primitive<NV>(ph, U, W);
  out[0] = W[1];
  out[1] = W[2];
  out[2] = W[3];
  out[3] = W[4] / (fmax(W[0], T(kRhoFloor)) * T(ph.R));
}

// Ghost [u, v, w, T] for the viscous traces (boundary.py:74-102).
template <int NV>
__device__ void viscous_ghost(const Physics& ph, const double* far, double wall_T, const double* U, const double* n,
                              int tag, double* g) {
  double v[4];
  viscous_vars<NV>(ph, U, v);
  g[0] = v[0]; g[1] = v[1]; g[2] = v[2]; g[3] = v[3];
  if (tag_in(tag, ph.no_slip, ph.n_no_slip)) {
    g[0] = -v[0]; g[1] = -v[1]; g[2] = -v[2];
    g[3] = ph.has_wall_T ? 2.0 * wall_T - v[3] : v[3];
  }
  if (tag_in(tag, ph.slip, ph.n_slip)) {
    const double un = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
    g[0] = v[0] - 2.0 * un * n[0];
    g[1] = v[1] - 2.0 * un * n[1];
    g[2] = v[2] - 2.0 * un * n[2];
    g[3] = v[3];
  }
  if (tag_in(tag, ph.inlet, ph.n_inlet)) {
    double Uf[NV];
    conserved<NV>(ph, far, Uf);
    viscous_vars<NV>(ph, Uf, g);
  }
}

// Cartesian viscous flux F[d][v]; grad[m][d] = d(u,v,w,T)_m / dx_d.
template <int NV, typename T>
__device__ void viscous_flux(const Physics& ph, double mu_, double kappa, const T* U, const T* grad, T* F) {
  T W[NV];
  primitive<NV>(ph, U, W);
  const T div = grad[0 * 3 + 0] + grad[1 * 3 + 1] + grad[2 * 3 + 2];
  const T mu = T(mu_), two_thirds = T(2.0 / 3.0);
  T stress[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d)
      stress[i][d] = mu * (grad[i * 3 + d] + grad[d * 3 + i] - (i == d ? two_thirds * div : T(0)));
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    F[d * NV + 0] = T(0);
    F[d * NV + 1] = stress[0][d];
    F[d * NV + 2] = stress[1][d];
    F[d * NV + 3] = stress[2][d];
    F[d * NV + 4] = W[1] * stress[0][d] + W[2] * stress[1][d] + W[3] * stress[2][d] + T(kappa) * grad[3 * 3 + d];
#pragma unroll
    for (int v = 5; v < NV; ++v) F[d * NV + v] = T(0);
  }
}

}  // namespace dgb
