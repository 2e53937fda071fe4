// Finite-rate chemistry: operator-split point-implicit reaction advance, one thread per
// solution node, float64 throughout.
//
// Follows the reference's hybrid/chemistry package:
//   nasa.py:47-118          NASA-7 cp/R, h/RT, s/R with T clamped to each species' range
//   mechanism.py:125-220    forward rates, Gibbs equilibrium constants, mass-action net
//                           rates with third bodies, mass-conserving correction
//   mechanism.py:262-287    T(e) damped Newton inversion
//   integrator.py:31-104    Newton on R(rho) = rho - rho0 - dt w(rho, T) with the exact
//                           Jacobian, max(., 0) clipping, T re-derived from the initial
//                           internal energy after every update, final mass rescale
//   coupling.py:116-197     per-node coupling (species renormalisation, thermal energy,
//                           dimensionless scaling)
// The reference differentiates the residual with JAX; here d w/d rho is assembled
// analytically from the reaction structure, with JAX's convention at ties of max/clip
// (the derivative is split evenly between the two arguments).
//
// Layout: the mechanism travels as one __grid_constant__ kernel parameter (about 12 KB),
// so every warp-uniform table read is a constant-cache broadcast.  Per thread, the
// augmented Newton matrix [I - dt J | -R] (ns x ns+1) and the species vectors that the
// reaction loops index through the stoichiometry lists live in shared memory with a
// stride of one thread, so a warp's accesses fall in distinct banks.  The net rates
// accumulate in the matrix's last column.  At 176 doubles a node, a CTA of one warp takes
// 45 KB, and five CTAs share an SM.
//
// Work saved against a literal evaluation, each with the same result up to rounding:
//  - a reaction whose stoichiometric coefficients are all whole numbers up to 3 forms
//    prod C^nu by multiplication instead of exp(sum nu log C) (the clip at |.| = 700 is
//    applied to the product);
//  - the temperature inversion stops once an update moves T by at most 1e-13 T: Newton on
//    e(T) converges quadratically, so the remaining iterations of the fixed count change T
//    only in its last bits.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <string>

#include "dgb200.h"

namespace dgb {
int set_error(int code, const std::string& msg);
}

namespace {

constexpr int kThreads = 32;
constexpr int kMaxList = 6;
constexpr double kClipExp = 700.0, kMinKc = 1.0e-300, kMinC = 1.0e-100;
// exp(-700) and exp(700): the clip of the mass-action exponent applied to a product
constexpr double kExpLo = 9.8597628436862264e-305, kExpHi = 1.0142320547350045e304;
// the temperature inversion's convergence test (relative step)
constexpr double kTStop = 1.0e-13;
constexpr double kRUniv = 8.31446261815324, kPStd = 101325.0;

struct Reaction {
  double A, b, theta, dn;                 // Arrhenius; sum of net stoichiometry
  int fmode, rmode, third, nf, nr, nd;    // temperature modes, third-body flag, list sizes
  int whole;                              // every nu' and nu'' a whole number in 1..3
  int f_pw[3], r_pw[3];                   // those whole numbers
  int f_sp[3], r_sp[3], d_sp[kMaxList];   // species of nu', nu'', nu''-nu' (ascending)
  double f_nu[3], r_nu[3], d_nu[kMaxList];
};

struct Tables {
  int ns, nr;
  double W[DGB_CHEM_MAX_SPECIES];             // molar mass
  double RW[DGB_CHEM_MAX_SPECIES];            // R_univ / W
  double iW[DGB_CHEM_MAX_SPECIES];            // 1 / W
  double trange[DGB_CHEM_MAX_SPECIES][3];
  double clamp_log[DGB_CHEM_MAX_SPECIES][2];  // ln t_low, ln t_high
  double clamp_inv[DGB_CHEM_MAX_SPECIES][2];  // 1 / t_low, 1 / t_high
  double cp[DGB_CHEM_MAX_SPECIES][2][5];      // a0..a4
  double h[DGB_CHEM_MAX_SPECIES][2][6];       // a0, a1/2, a2/3, a3/4, a4/5, a5
  double s[DGB_CHEM_MAX_SPECIES][2][6];       // a0, a1, a2/2, a3/3, a4/4, a6
  double alpha[DGB_CHEM_MAX_REACTIONS][DGB_CHEM_MAX_SPECIES];
  Reaction rx[DGB_CHEM_MAX_REACTIONS];
  // coupler (coupling.py:26-71)
  int iters, dimensionless;
  double T_ref, rho_ref, e_ref, t_ref, gamma;
};

// max/min that propagate NaN like jnp.maximum/jnp.minimum
__device__ __forceinline__ double jmax(double a, double b) { return (a > b || a != a) ? a : b; }
__device__ __forceinline__ double jmin(double a, double b) { return (a < b || a != a) ? a : b; }
__device__ __forceinline__ double jclip(double x, double lo, double hi) { return jmin(jmax(x, lo), hi); }
// d max(x, c)/dx under JAX's tie rule
__device__ __forceinline__ double dmax_tie(double x, double c) { return x > c ? 1.0 : (x == c ? 0.5 : 0.0); }

template <int NS>
struct Slots {
  double* base;
  int stride;
  __device__ double& A(int i, int j) const { return base[(i * (NS + 1) + j) * stride]; }
  __device__ double& om(int q) const { return A(q, NS); }                              // net rates
  __device__ double& C(int q) const { return base[(NS * (NS + 1) + q) * stride]; }     // max(C, 1e-100)
  __device__ double& dlog(int q) const { return base[(NS * (NS + 2) + q) * stride]; }
  __device__ double& g(int q) const { return base[(NS * (NS + 3) + q) * stride]; }
  __device__ double& r0(int q) const { return base[(NS * (NS + 4) + q) * stride]; }    // Newton's rho0
  static constexpr int kDoubles = NS * (NS + 5);
};

// Temperature powers shared by every species at one temperature T: ln T and 1/T.  A species
// whose fit range clamps T uses the host-computed ln and reciprocal of its range end.
struct TPow {
  double T, lnT, invT;
};

__device__ __forceinline__ TPow tpow(double T) { return TPow{T, log(T), 1.0 / T}; }

// species q at T: T clamped to [t_low, t_high], coefficient set by T_c < t_mid
__device__ __forceinline__ int nasa_range(const Tables& M, int q, const TPow& t, double& Tc, double& lnTc,
                                          double& invTc) {
  Tc = jclip(t.T, M.trange[q][0], M.trange[q][2]);
  const bool lo = Tc == M.trange[q][0] && Tc != t.T;
  const bool hi = Tc == M.trange[q][2] && Tc != t.T;
  lnTc = lo ? M.clamp_log[q][0] : (hi ? M.clamp_log[q][1] : t.lnT);
  invTc = lo ? M.clamp_inv[q][0] : (hi ? M.clamp_inv[q][1] : t.invT);
  return Tc < M.trange[q][1] ? 0 : 1;
}

__device__ __forceinline__ double h_RT(const Tables& M, int q, const TPow& t) {
  double Tc, lnTc, invTc;
  const int r = nasa_range(M, q, t, Tc, lnTc, invTc);
  const double* a = M.h[q][r];
  const double T2 = Tc * Tc;
  return a[0] + a[1] * Tc + a[2] * T2 + a[3] * (T2 * Tc) + a[4] * (T2 * T2) + a[5] * invTc;
}

__device__ __forceinline__ double cp_R(const Tables& M, int q, const TPow& t) {
  double Tc, lnTc, invTc;
  const int r = nasa_range(M, q, t, Tc, lnTc, invTc);
  const double* a = M.cp[q][r];
  const double T2 = Tc * Tc;
  return a[0] + a[1] * Tc + a[2] * T2 + a[3] * (T2 * Tc) + a[4] * (T2 * T2);
}

__device__ __forceinline__ double g_RT(const Tables& M, int q, const TPow& t) {
  double Tc, lnTc, invTc;
  const int r = nasa_range(M, q, t, Tc, lnTc, invTc);
  const double* a = M.h[q][r];
  const double* c = M.s[q][r];
  const double T2 = Tc * Tc;
  const double h = a[0] + a[1] * Tc + a[2] * T2 + a[3] * (T2 * Tc) + a[4] * (T2 * T2) + a[5] * invTc;
  const double s = c[0] * lnTc + c[1] * Tc + c[2] * T2 + c[3] * (T2 * Tc) + c[4] * (T2 * T2) + c[5];
  return h - s;
}

// mechanism.py:125-128 with Tv = T (single temperature)
__device__ __forceinline__ double select_T(int mode, double T, double Tv) {
  if (mode == 1) return sqrt(jmax(T * Tv, 1.0));
  return mode == 2 ? Tv : T;
}

// mixture_properties()["internal_energy"], mechanism.py:222-260
template <int NS>
__device__ double internal_energy(const Tables& M, const double (&rho)[NS], double T) {
  double S = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) S += rho[q];
  S = jmax(S, 1.0e-14);
  const TPow t{T, 0.0, 1.0 / T};     // the energy fits need no logarithm
  double e = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) e += (jmax(rho[q], 0.0) / S) * ((h_RT(M, q, t) - 1.0) * (T * M.RW[q]));
  return e;
}

// recover_temperature_from_energy, mechanism.py:262-287
template <int NS>
__device__ double recover_T(const Tables& M, const double (&rho)[NS], double target, double T, int iters) {
  double S = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) S += rho[q];
  S = jmax(S, 1.0e-14);
  double Y[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) Y[q] = jmax(rho[q], 0.0) / S;
  for (int it = 0; it < iters; ++it) {
    const double Ts = jclip(T, 50.0, 50000.0);
    // 1/Ts is the only temperature power the energy fits need (no logarithm)
    const TPow t{Ts, 0.0, 1.0 / Ts};
    double e = 0.0, cv = 0.0;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      e += Y[q] * ((h_RT(M, q, t) - 1.0) * (Ts * M.RW[q]));
      cv += Y[q] * ((cp_R(M, q, t) - 1.0) * M.RW[q]);
    }
    const double dT = -(e - target) / jmax(cv, 1.0e-5);
    const double Tn = jclip(T + jclip(dT, -0.5 * T, 0.5 * T), 100.0, 50000.0);
    const bool done = fabs(Tn - T) <= kTStop * T;
    T = Tn;
    if (done) break;
  }
  return T;
}

// prod_k C[sp[k]]^pw[k] for whole exponents, clipped to [exp(-700), exp(700)] as the
// exponential of the summed logarithms is; ok receives d(clip)/d(arg) under JAX's tie rule.
template <int NS>
__device__ __forceinline__ double mass_action(const Slots<NS>& sl, int n, const int* sp, const int* pw, double& ok) {
  double v = 1.0;
  for (int k = 0; k < n; ++k) {
    const double c = sl.C(sp[k]);
    v *= pw[k] == 1 ? c : (pw[k] == 2 ? c * c : c * c * c);
  }
  ok = (v > kExpLo && v < kExpHi) ? 1.0 : ((v == kExpLo || v == kExpHi) ? 0.5 : 0.0);
  return jclip(v, kExpLo, kExpHi);
}

// Net rates at (rho, T): omega -> sl.om, and, when jac, sum_r dnu[r][s] dq_r/drho_j
// into sl.A(s, j) (d w/d rho before the molar-mass scaling and the mass correction).
template <int NS>
__device__ void rates(const Tables& M, const Slots<NS>& sl, const double (&rho)[NS], double T, bool jac) {
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const double craw = rho[q] * M.iW[q];
    const double c = jmax(craw, 0.0);
    const double dc = dmax_tie(craw, 0.0) * M.iW[q];
    const double cc = jmax(c, kMinC);
    sl.C(q) = cc;
    sl.dlog(q) = dmax_tie(c, kMinC) * dc / cc;
    sl.om(q) = 0.0;
  }
  const double Tg = jmax(T, 10.0);
  const TPow tg = tpow(Tg);
  const double base_g = kPStd / (kRUniv * Tg);
#pragma unroll
  for (int q = 0; q < NS; ++q) sl.g(q) = g_RT(M, q, tg);
  if (jac) {
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
      for (int j = 0; j < NS; ++j) sl.A(i, j) = 0.0;
  }
  for (int r = 0; r < M.nr; ++r) {
    const Reaction& R = M.rx[r];
    // kf = A T^b exp(-theta/T) as A exp(b ln T - theta/T); ln T and 1/T are shared
    const double Tf = jmax(select_T(R.fmode, T, T), 10.0);
    const TPow tf = Tf == Tg ? tg : tpow(Tf);
    const double kf = R.A * exp(R.b * tf.lnT - R.theta * tf.invT);
    const double Tr = jmax(select_T(R.rmode, T, T), 10.0);
    double dG = 0.0;
    if (Tr == Tg) {
      for (int k = 0; k < R.nd; ++k) dG += R.d_nu[k] * sl.g(R.d_sp[k]);
    } else {
      const TPow tr = tpow(Tr);
      for (int k = 0; k < R.nd; ++k) dG += R.d_nu[k] * g_RT(M, R.d_sp[k], tr);
    }
    const double base = Tr == Tg ? base_g : kPStd / (kRUniv * Tr);
    const double conv = R.dn == 0.0 ? 1.0 : (R.dn == 1.0 ? base : (R.dn == -1.0 ? 1.0 / base : pow(base, R.dn)));
    const double Kc = exp(-jclip(dG, -kClipExp, kClipExp)) * conv;
    const double kr = kf / jmax(Kc, kMinKc);
    double fwd, rev, okf, okr;
    if (R.whole) {
      fwd = mass_action(sl, R.nf, R.f_sp, R.f_pw, okf);
      rev = mass_action(sl, R.nr, R.r_sp, R.r_pw, okr);
    } else {
      double lf = 0.0, lr = 0.0;
      for (int k = 0; k < R.nf; ++k) lf += R.f_nu[k] * log(sl.C(R.f_sp[k]));
      for (int k = 0; k < R.nr; ++k) lr += R.r_nu[k] * log(sl.C(R.r_sp[k]));
      fwd = exp(jclip(lf, -kClipExp, kClipExp));
      rev = exp(jclip(lr, -kClipExp, kClipExp));
      // d q / d log C_j through the clipped exponentials; the tie rule at |l| == 700
      okf = fabs(lf) < kClipExp ? 1.0 : (fabs(lf) == kClipExp ? 0.5 : 0.0);
      okr = fabs(lr) < kClipExp ? 1.0 : (fabs(lr) == kClipExp ? 0.5 : 0.0);
    }
    double coll = 1.0;
    if (R.third) {
      coll = 0.0;
#pragma unroll
      for (int q = 0; q < NS; ++q) coll += M.alpha[r][q] * jmax(rho[q] * M.iW[q], 0.0);
    }
    const double qf = kf * fwd * coll, qr = kr * rev * coll;
    const double qn = qf - qr;
    for (int k = 0; k < R.nd; ++k) sl.om(R.d_sp[k]) += R.d_nu[k] * qn;
    if (!jac) continue;
    const double a = kf * fwd * okf * coll, b = kr * rev * okr * coll;
    const double qc = kf * fwd - kr * rev;
    for (int kd = 0; kd < R.nd; ++kd) {
      const int s = R.d_sp[kd];
      const double dn = R.d_nu[kd];
      for (int m = 0; m < R.nf; ++m) {
        const int j = R.f_sp[m];
        sl.A(s, j) += dn * (a * R.f_nu[m] * sl.dlog(j));
      }
      for (int m = 0; m < R.nr; ++m) {
        const int j = R.r_sp[m];
        sl.A(s, j) -= dn * (b * R.r_nu[m] * sl.dlog(j));
      }
      if (R.third) {
#pragma unroll
        for (int j = 0; j < NS; ++j) {
          const double dC = dmax_tie(rho[j] * M.iW[j], 0.0) * M.iW[j];
          sl.A(s, j) += dn * (qc * M.alpha[r][j] * dC);
        }
      }
    }
  }
}

// Mass-conserving correction (mechanism.py:214-218): w = W omega - Y sum(W omega) replaces
// omega in sl.om, and its Jacobian J = dwd - dY sum(wd) - Y colsum(dwd) replaces sl.A
// (newton: sl.A becomes [I - dt J | -res] with res = rho - rho0 - dt w).
template <int NS>
__device__ void finish(const Tables& M, const Slots<NS>& sl, const double (&rho)[NS], double dt, bool jac,
                       bool newton) {
  double Sraw = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) Sraw += rho[q];
  const double S = jmax(Sraw, 1.0e-14);
  const double dS = dmax_tie(Sraw, 1.0e-14);
  double sw = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const double wd = sl.om(q) * M.W[q];
    sl.om(q) = wd;
    sw += wd;
  }
#pragma unroll
  for (int q = 0; q < NS; ++q) sl.om(q) = sl.om(q) - (jmax(rho[q], 0.0) / S) * sw;
  if (!jac) return;
  // per row: Y_i, and dY_i/drho_j off the diagonal (the diagonal adds dmax(rho_i, 0)/S)
  double Yr[NS], dYo[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    Yr[i] = jmax(rho[i], 0.0) / S;
    dYo[i] = -(jmax(rho[i], 0.0) / (S * S)) * dS;
  }
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    double col = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      const double v = M.W[i] * sl.A(i, j);
      sl.A(i, j) = v;
      col += v;
    }
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      const double dY = i == j ? dmax_tie(rho[i], 0.0) / S + dYo[i] : dYo[i];
      const double J = sl.A(i, j) - dY * sw - Yr[i] * col;
      sl.A(i, j) = newton ? (i == j ? 1.0 : 0.0) - dt * J : J;
    }
  }
  if (newton) {
#pragma unroll
    for (int i = 0; i < NS; ++i) sl.A(i, NS) = -(rho[i] - sl.r0(i) - dt * sl.om(i));
  }
}

// Solve [A | b] in place by LU with partial pivoting (the first largest |pivot|, as
// LAPACK's getrf); x receives the solution.
template <int NS>
__device__ void lu_solve(const Slots<NS>& sl, double (&x)[NS]) {
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    int p = k;
    double amax = fabs(sl.A(k, k));
#pragma unroll
    for (int i = k + 1; i < NS; ++i) {
      const double v = fabs(sl.A(i, k));
      if (v > amax) {
        amax = v;
        p = i;
      }
    }
    if (p != k) {
#pragma unroll
      for (int j = k; j <= NS; ++j) {
        const double t = sl.A(k, j);
        sl.A(k, j) = sl.A(p, j);
        sl.A(p, j) = t;
      }
    }
    const double rp = 1.0 / sl.A(k, k);
#pragma unroll
    for (int i = k + 1; i < NS; ++i) {
      const double f = sl.A(i, k) * rp;
#pragma unroll
      for (int j = k + 1; j <= NS; ++j) sl.A(i, j) -= f * sl.A(k, j);
    }
  }
#pragma unroll
  for (int i = NS - 1; i >= 0; --i) {
    double acc = sl.A(i, NS);
#pragma unroll
    for (int j = i + 1; j < NS; ++j) acc -= sl.A(i, j) * x[j];
    x[i] = acc / sl.A(i, i);
  }
}

// ReactingFlowCoupler._react_single_cell for every node of a block.
template <int NS>
__global__ void __launch_bounds__(kThreads) k_react(const __grid_constant__ Tables M, const double* U, double* out,
                                                    long long nodes, int num_nodes, int nvars, double dt,
                                                    const double* __restrict__ dt_elem) {
  extern __shared__ double smem[];
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nodes) return;
  const Slots<NS> sl{smem + threadIdx.x, (int)blockDim.x};
  const double* u = U + n * nvars;
  const double step = dt_elem ? dt_elem[n / num_nodes] : dt;

  const double rho_t = jmax(u[0], 1.0e-14);
  double rs[NS], ssum = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    rs[q] = jmax(u[5 + q], 0.0);
    ssum += rs[q];
  }
  const double scale = rho_t / jmax(ssum, 1.0e-20);
#pragma unroll
  for (int q = 0; q < NS; ++q) rs[q] *= scale;
  const double ek = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / (rho_t * rho_t);

  double rp[NS], T0, dtp;
  if (M.dimensionless) {
    const double es = jmax(u[4] / rho_t - ek, 1.0e-4);
#pragma unroll
    for (int q = 0; q < NS; ++q) rp[q] = rs[q] * M.rho_ref;
    const double Tg = jmax((M.gamma - 1.0) * es * M.T_ref, 200.0);
    T0 = recover_T<NS>(M, rp, es * M.e_ref, Tg, 8);
    dtp = step * M.t_ref;
  } else {
    const double e = jmax(u[4] / rho_t - ek, 1.0e3);
#pragma unroll
    for (int q = 0; q < NS; ++q) rp[q] = rs[q];
    T0 = recover_T<NS>(M, rp, e, 1000.0, 8);
    dtp = step;
  }

  // PointImplicitIntegrator.step, constant_temperature=False
  double rho[NS], total = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    rho[q] = jmax(rp[q], 1.0e-20);
    sl.r0(q) = rho[q];
    total += rho[q];
  }
  const double e_init = internal_energy<NS>(M, rho, T0);
  double Tk = T0;
  for (int it = 0; it < M.iters; ++it) {
    double d[NS];
    rates<NS>(M, sl, rho, Tk, true);
    finish<NS>(M, sl, rho, dtp, true, true);
    lu_solve<NS>(sl, d);
#pragma unroll
    for (int q = 0; q < NS; ++q) rho[q] = jmax(rho[q] + d[q], 0.0);
    Tk = recover_T<NS>(M, rho, e_init, Tk, 10);
  }
  double fsum = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) fsum += rho[q];
  const double fs = total / fsum;
  double nsum = 0.0;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    double v = rho[q] * fs;
    if (M.dimensionless) v = v / M.rho_ref;
    rho[q] = jmax(v, 0.0);
    nsum += rho[q];
  }
  const double back = rho_t / jmax(nsum, 1.0e-20);
  double* o = out + n * nvars;
  if (o != u) {
    for (int v = 0; v < 5; ++v) o[v] = u[v];
    for (int v = 5 + NS; v < nvars; ++v) o[v] = u[v];
  }
#pragma unroll
  for (int q = 0; q < NS; ++q) o[5 + q] = rho[q] * back;
}

// ReactionMechanism.net_production_rates (and its Jacobian) for independent samples.
template <int NS>
__global__ void __launch_bounds__(kThreads) k_rates(const __grid_constant__ Tables M, const double* __restrict__ rho_in,
                                                    const double* __restrict__ T_in, long long count,
                                                    double* __restrict__ omega, double* __restrict__ wdot,
                                                    double* __restrict__ jac) {
  extern __shared__ double smem[];
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= count) return;
  const Slots<NS> sl{smem + threadIdx.x, (int)blockDim.x};
  double rho[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) rho[q] = rho_in[n * NS + q];
  const bool want = jac != nullptr;
  rates<NS>(M, sl, rho, T_in[n], want);
#pragma unroll
  for (int q = 0; q < NS; ++q)
    if (omega) omega[n * NS + q] = sl.om(q);
  finish<NS>(M, sl, rho, 0.0, want, false);
#pragma unroll
  for (int q = 0; q < NS; ++q)
    if (wdot) wdot[n * NS + q] = sl.om(q);
  if (want) {
#pragma unroll
    for (int i = 0; i < NS; ++i)
#pragma unroll
      for (int j = 0; j < NS; ++j) jac[(n * NS + i) * NS + j] = sl.A(i, j);
  }
}

int fail(int code, const std::string& msg) { return dgb::set_error(code, msg); }

template <int NS>
size_t smem_bytes() {
  return sizeof(double) * (size_t)Slots<NS>::kDoubles * kThreads;
}

template <int NS>
int launch_react(const Tables& M, const double* U, double* out, long long nodes, int num_nodes, int nvars, double dt,
                 const double* dt_elem, cudaStream_t st) {
  const size_t sm = smem_bytes<NS>();
  cudaError_t err = cudaFuncSetAttribute(k_react<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  // the largest shared-memory carve-out, so that five one-warp CTAs share an SM
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(k_react<NS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared);
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(err));
  const unsigned grid = (unsigned)((nodes + kThreads - 1) / kThreads);
  k_react<NS><<<grid, kThreads, sm, st>>>(M, U, out, nodes, num_nodes, nvars, dt, dt_elem);
  err = cudaGetLastError();
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, std::string("k_react: ") + cudaGetErrorString(err));
  return DGB_OK;
}

template <int NS>
int launch_rates(const Tables& M, const double* rho, const double* T, long long count, double* omega, double* wdot,
                 double* jac, cudaStream_t st) {
  const size_t sm = smem_bytes<NS>();
  cudaError_t err = cudaFuncSetAttribute(k_rates<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(err));
  const unsigned grid = (unsigned)((count + kThreads - 1) / kThreads);
  k_rates<NS><<<grid, kThreads, sm, st>>>(M, rho, T, count, omega, wdot, jac);
  err = cudaGetLastError();
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, std::string("k_rates: ") + cudaGetErrorString(err));
  return DGB_OK;
}

}  // namespace

struct dgb_chem {
  Tables tables;
};

extern "C" {

int dgb_chem_create(const dgb_chem_mechanism* m, const dgb_chem_params* prm, dgb_chem** out) {
  if (!m || !prm || !out) return fail(DGB_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  const int ns = m->num_species, nr = m->num_reactions;
  if (ns != 3 && ns != 11) return fail(DGB_ERR_UNSUPPORTED, "chemistry kernels are compiled for 3 or 11 species");
  if (nr < 1 || nr > DGB_CHEM_MAX_REACTIONS) return fail(DGB_ERR_UNSUPPORTED, "too many reactions");
  if (!m->molar_mass || !m->nu_forward || !m->nu_reverse || !m->efficiency || !m->arrhenius || !m->third_body ||
      !m->forward_mode || !m->reverse_mode || !m->nasa_range || !m->nasa_coeffs)
    return fail(DGB_ERR_ARGUMENT, "null mechanism table");
  if (prm->max_newton_iters < 0) return fail(DGB_ERR_ARGUMENT, "max_newton_iters must be >= 0");
  dgb_chem* c = new dgb_chem;
  Tables& M = c->tables;
  memset(&M, 0, sizeof(M));
  M.ns = ns;
  M.nr = nr;
  for (int q = 0; q < ns; ++q) {
    M.W[q] = m->molar_mass[q];
    M.RW[q] = kRUniv / m->molar_mass[q];
    M.iW[q] = 1.0 / m->molar_mass[q];
    for (int k = 0; k < 3; ++k) M.trange[q][k] = m->nasa_range[q * 3 + k];
    if (!(M.trange[q][0] > 0.0) || !(M.trange[q][2] > M.trange[q][0])) {
      delete c;
      return fail(DGB_ERR_ARGUMENT, "NASA-7 ranges must satisfy 0 < t_low < t_high");
    }
    M.clamp_log[q][0] = log(M.trange[q][0]);
    M.clamp_log[q][1] = log(M.trange[q][2]);
    M.clamp_inv[q][0] = 1.0 / M.trange[q][0];
    M.clamp_inv[q][1] = 1.0 / M.trange[q][2];
    for (int r = 0; r < 2; ++r) {
      const double* a = m->nasa_coeffs + (q * 2 + r) * 7;
      for (int k = 0; k < 5; ++k) M.cp[q][r][k] = a[k];
      M.h[q][r][0] = a[0];
      M.h[q][r][1] = a[1] / 2.0;
      M.h[q][r][2] = a[2] / 3.0;
      M.h[q][r][3] = a[3] / 4.0;
      M.h[q][r][4] = a[4] / 5.0;
      M.h[q][r][5] = a[5];
      M.s[q][r][0] = a[0];
      M.s[q][r][1] = a[1];
      M.s[q][r][2] = a[2] / 2.0;
      M.s[q][r][3] = a[3] / 3.0;
      M.s[q][r][4] = a[4] / 4.0;
      M.s[q][r][5] = a[6];
    }
  }
  for (int r = 0; r < nr; ++r) {
    Reaction& R = M.rx[r];
    R.A = m->arrhenius[r * 3 + 0];
    R.b = m->arrhenius[r * 3 + 1];
    R.theta = m->arrhenius[r * 3 + 2];
    R.third = m->third_body[r] ? 1 : 0;
    R.fmode = m->forward_mode[r];
    R.rmode = m->reverse_mode[r];
    if (R.fmode < 0 || R.fmode > 2 || R.rmode < 0 || R.rmode > 2) {
      delete c;
      return fail(DGB_ERR_ARGUMENT, "temperature mode must be 0, 1 or 2");
    }
    double dn = 0.0;
    for (int q = 0; q < ns; ++q) {
      const double f = m->nu_forward[r * ns + q], p = m->nu_reverse[r * ns + q], d = p - f;
      M.alpha[r][q] = m->efficiency[r * ns + q];
      dn += d;
      if (f != 0.0) {
        if (R.nf == 3) { delete c; return fail(DGB_ERR_UNSUPPORTED, "more than 3 reactant species"); }
        R.f_sp[R.nf] = q;
        R.f_nu[R.nf++] = f;
      }
      if (p != 0.0) {
        if (R.nr == 3) { delete c; return fail(DGB_ERR_UNSUPPORTED, "more than 3 product species"); }
        R.r_sp[R.nr] = q;
        R.r_nu[R.nr++] = p;
      }
      if (d != 0.0) {
        if (R.nd == kMaxList) { delete c; return fail(DGB_ERR_UNSUPPORTED, "more than 6 net species"); }
        R.d_sp[R.nd] = q;
        R.d_nu[R.nd++] = d;
      }
    }
    R.dn = dn;
    R.whole = 1;
    for (int k = 0; k < R.nf; ++k) {
      const double v = R.f_nu[k];
      R.whole &= (v == 1.0 || v == 2.0 || v == 3.0) ? 1 : 0;
      R.f_pw[k] = (int)v;
    }
    for (int k = 0; k < R.nr; ++k) {
      const double v = R.r_nu[k];
      R.whole &= (v == 1.0 || v == 2.0 || v == 3.0) ? 1 : 0;
      R.r_pw[k] = (int)v;
    }
  }
  // coupling.py:55-67
  M.iters = prm->max_newton_iters;
  M.dimensionless = prm->dimensionless ? 1 : 0;
  M.gamma = prm->gamma;
  M.T_ref = prm->reference_temperature;
  const double mw_n2 = 2.0 * 0.0140067, mw_o2 = 2.0 * 0.015999;
  const double mean_mw = 1.0 / (0.767 / mw_n2 + 0.233 / mw_o2);
  const double R_ref = kRUniv / mean_mw;
  M.rho_ref = prm->reference_pressure / (R_ref * prm->reference_temperature);
  const double u_ref = sqrt(R_ref * prm->reference_temperature);
  M.e_ref = u_ref * u_ref;
  M.t_ref = prm->reference_length / u_ref;
  *out = c;
  return DGB_OK;
}

int dgb_chem_destroy(dgb_chem* chem) {
  delete chem;
  return DGB_OK;
}

int dgb_react_block(dgb_chem* chem, const double* U, double* out, int64_t num_elements, int num_nodes, int nvars,
                    double dt, const double* dt_per_element, void* stream) {
  if (!chem) return fail(DGB_ERR_ARGUMENT, "null argument");
  const Tables& M = chem->tables;
  if (nvars < 5 + M.ns)
    return fail(DGB_ERR_ARGUMENT, "State has " + std::to_string(nvars) + " variables; expected at least " +
                                      std::to_string(5 + M.ns) + " for reacting mixture.");
  if (num_elements < 0 || num_nodes < 0) return fail(DGB_ERR_ARGUMENT, "negative block size");
  const long long nodes = (long long)num_elements * num_nodes;
  if (nodes == 0) return DGB_OK;                    // an empty block needs no buffers
  if (!U || !out) return fail(DGB_ERR_ARGUMENT, "null argument");
  if ((nodes + kThreads - 1) / kThreads > 0x7fffffffLL) return fail(DGB_ERR_ARGUMENT, "block too large");
  cudaStream_t st = (cudaStream_t)stream;
  return M.ns == 11 ? launch_react<11>(M, U, out, nodes, num_nodes, nvars, dt, dt_per_element, st)
                    : launch_react<3>(M, U, out, nodes, num_nodes, nvars, dt, dt_per_element, st);
}

int dgb_chem_rates(dgb_chem* chem, const double* rho, const double* T, int64_t count, double* omega, double* wdot,
                   double* jacobian, void* stream) {
  if (!chem || !rho || !T) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (count < 0) return fail(DGB_ERR_ARGUMENT, "negative count");
  if (count == 0) return DGB_OK;
  const Tables& M = chem->tables;
  cudaStream_t st = (cudaStream_t)stream;
  return M.ns == 11 ? launch_rates<11>(M, rho, T, count, omega, wdot, jacobian, st)
                    : launch_rates<3>(M, rho, T, count, omega, wdot, jacobian, st);
}

}  // extern "C"
