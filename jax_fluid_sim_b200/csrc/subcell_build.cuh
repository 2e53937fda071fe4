// Device construction of the MOOD subcell tables (HybridSubcellFV.__init__,
// hybrid/subcell.py:277-396 per element, :473-533 for the neighbour subface matching).
//
// Every element is split into the 64 reference subcells of its type.  Per element, one CTA forms
// in shared memory:
//   - the subcell vertices (the geometry map at the reference subcell vertices) and centres
//     (the mean of each subcell's vertices);
//   - |det J| of the geometry map at the P2 volume rule mapped onto each subcell, times the
//     rule weight; the subcell volumes are their sums;
//   - the metric-weighted projection P[s][i] = sum_q w|J| phi_i / V_s of the DG basis onto the
//     subcell means, and its volume-weighted least-squares left inverse
//     R = (P^T V P)^-1 P^T V, the Gram matrix inverted by Gauss-Jordan (gauss_jordan_spd);
//   - the subface area vectors (a triangle p0 p1 p2 gives (p1 - p0) x (p2 - p0) / 2, a
//     quadrilateral adds (p2 - p0) x (p3 - p0) / 2) turned to point from the owner subcell's
//     centre toward the neighbour's (toward the subface centre on the element boundary), their
//     lengths, unit vectors and, on the boundary, the subface centres.
// Shared memory per CTA: (3 ng + 3 V + 3 S + S Qs + S + S Np + Np^2 + 2 Np) doubles, 86 KB for
// P3 hexahedra.  The neighbour matching is one thread per parent face.
#pragma once

#include "dg_kernels.cuh"
#include "mood_kernels.cuh"

namespace dgb {

// In-place inverse of the symmetric positive definite n x n matrix A in shared memory by
// Gauss-Jordan elimination without pivoting (every pivot of an SPD matrix is positive), worked by
// the whole block; rk, ck: n doubles of shared scratch.  Returns false, uniformly across the
// block, at a pivot that is not positive and finite.  Ends with the block synchronised.
__device__ bool gauss_jordan_spd(double* A, int n, double* rk, double* ck) {
  for (int k = 0; k < n; ++k) {
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      rk[t] = A[k * n + t];
      ck[t] = A[t * n + k];
    }
    __syncthreads();
    const double piv = rk[k];
    if (!(piv > 0.0) || !isfinite(piv)) return false;   // every thread read the same pivot
    const double r = 1.0 / piv;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      const int i = idx / n, j = idx % n;
      if (i == k)
        A[idx] = j == k ? r : rk[j] * r;
      else if (j == k)
        A[idx] = -ck[i] * r;
      else
        A[idx] -= ck[i] * rk[j] * r;
    }
  }
  __syncthreads();
  return true;
}

struct SubcellRefDev {
  int S, Qs, ng, V, cs, NI, NB, Np;
  const double* rw;       // [S][Qs]
  const double* sb;       // [S][Qs][Np]
  const double* gq;       // [S][Qs][ng][3]
  const double* vg;       // [V][ng]
  const int32_t* cells;   // [S][cs]
  const int32_t* ifaces;  // [NI][4]
  const int32_t* bfaces;  // [NB][4]
  const int32_t* iown;    // [NI]
  const int32_t* inbr;    // [NI]
  const int32_t* bown;    // [NB]
};

struct SubcellBuildOut {
  double* P;     // [E][S][Np]
  double* R;     // [E][Np][S]
  double* vol;   // [E][S]
  double* cen;   // [E][S][3]
  double* in_n;  // [E][NI][3]
  double* in_a;  // [E][NI]
  double* bd_n;  // [E][NB][3]
  double* bd_a;  // [E][NB]
  double* bd_c;  // [E][NB][3]
};

inline size_t subcell_build_smem(const SubcellRefDev& r) {
  return sizeof(double) * (3 * (size_t)r.ng + 3 * (size_t)r.V + 3 * (size_t)r.S + (size_t)r.S * r.Qs + r.S +
                           (size_t)r.S * r.Np + (size_t)r.Np * r.Np + 2 * (size_t)r.Np);
}

// Area vector, length, unit normal and centre of one subface (3 or 4 vertices of pv), oriented
// along dir(fc); writes n[3], a, c[3] (c may be null).
template <typename Dir>
__device__ __forceinline__ void subface_metrics(const double* pv, const int32_t* f, Dir dir, double* n, double* a,
                                                double* c) {
  const int m = f[3] < 0 ? 3 : 4;
  const double* p[4];
  for (int k = 0; k < m; ++k) p[k] = pv + f[k] * 3;
  double u[3], w[3], v[3], fc[3];
  for (int d = 0; d < 3; ++d) {
    u[d] = p[1][d] - p[0][d];
    w[d] = p[2][d] - p[0][d];
  }
  v[0] = 0.5 * (u[1] * w[2] - u[2] * w[1]);
  v[1] = 0.5 * (u[2] * w[0] - u[0] * w[2]);
  v[2] = 0.5 * (u[0] * w[1] - u[1] * w[0]);
  if (m == 4) {
    double z[3];
    for (int d = 0; d < 3; ++d) z[d] = p[3][d] - p[0][d];
    v[0] = v[0] + 0.5 * (w[1] * z[2] - w[2] * z[1]);
    v[1] = v[1] + 0.5 * (w[2] * z[0] - w[0] * z[2]);
    v[2] = v[2] + 0.5 * (w[0] * z[1] - w[1] * z[0]);
  }
  for (int d = 0; d < 3; ++d) {
    double s = p[0][d] + p[1][d];
    for (int k = 2; k < m; ++k) s += p[k][d];
    fc[d] = s / m;
  }
  double dv[3];
  dir(fc, dv);
  const double sgn = (v[0] * dv[0] + v[1] * dv[1] + v[2] * dv[2]) >= 0.0 ? 1.0 : -1.0;
  for (int d = 0; d < 3; ++d) v[d] *= sgn;
  const double mag = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int d = 0; d < 3; ++d) n[d] = v[d] / mag;
  *a = mag;
  if (c)
    for (int d = 0; d < 3; ++d) c[d] = fc[d];
}

// One element per CTA; *bad receives 1 + the first element whose Gram matrix is not positive
// definite.
__global__ void __launch_bounds__(256) k_subcell_build(const SubcellRefDev r, const double* __restrict__ xyz_all,
                                                       SubcellBuildOut o, int* bad) {
  extern __shared__ double sm[];
  const int S = r.S, Qs = r.Qs, ng = r.ng, V = r.V, Np = r.Np, cs = r.cs;
  double* x = sm;                   // [ng][3] geometry nodes
  double* pv = x + 3 * ng;          // [V][3] subcell vertices
  double* cen = pv + 3 * V;         // [S][3] subcell centres
  double* pw = cen + 3 * S;         // [S][Qs] rule weight x |det J|
  double* vol = pw + S * Qs;        // [S]
  double* proj = vol + S;           // [S][Np]
  double* G = proj + S * Np;        // [Np][Np] Gram matrix, then its inverse
  double* rk = G + Np * Np;         // [Np] Gauss-Jordan scratch
  double* ck = rk + Np;             // [Np]
  const size_t e = blockIdx.x;
  const double* xe = xyz_all + e * ng * 3;
  for (int t = threadIdx.x; t < 3 * ng; t += blockDim.x) x[t] = xe[t];
  __syncthreads();
  for (int idx = threadIdx.x; idx < 3 * V; idx += blockDim.x) {
    const int v = idx / 3, d = idx % 3;
    double s = 0.0;
    for (int n = 0; n < ng; ++n) s += r.vg[v * ng + n] * x[n * 3 + d];
    pv[idx] = s;
  }
  // |det J| at the mapped rule points (the Jacobian summed over the geometry nodes in order)
  for (int idx = threadIdx.x; idx < S * Qs; idx += blockDim.x) {
    const double* g = r.gq + (size_t)idx * ng * 3;
    double J[3][3] = {};
    for (int k = 0; k < ng; ++k)
      for (int d = 0; d < 3; ++d)
        for (int c = 0; c < 3; ++c) J[d][c] += x[k * 3 + d] * g[k * 3 + c];
    const double A = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double B = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double C = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    pw[idx] = fabs(J[0][0] * A + J[0][1] * B + J[0][2] * C) * r.rw[idx];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 3 * S; idx += blockDim.x) {
    const int s = idx / 3, d = idx % 3;
    double a = 0.0;
    for (int k = 0; k < cs; ++k) a += pv[r.cells[s * cs + k] * 3 + d];
    cen[idx] = a / cs;
  }
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double a = 0.0;
    for (int q = 0; q < Qs; ++q) a += pw[s * Qs + q];
    vol[s] = a;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < S * Np; idx += blockDim.x) {
    const int s = idx / Np, i = idx % Np;
    double a = 0.0;
    for (int q = 0; q < Qs; ++q) a += pw[s * Qs + q] * r.sb[((size_t)s * Qs + q) * Np + i];
    proj[idx] = a / vol[s];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < Np * Np; idx += blockDim.x) {
    const int i = idx / Np, j = idx % Np;
    double a = 0.0;
    for (int s = 0; s < S; ++s) a += (proj[s * Np + i] * vol[s]) * proj[s * Np + j];
    G[idx] = a;
  }
  if (!gauss_jordan_spd(G, Np, rk, ck)) {      // uniform across the block
    if (threadIdx.x == 0) atomicCAS(bad, 0, (int)e + 1);
    return;
  }
  double* Re = o.R + e * Np * S;
  for (int idx = threadIdx.x; idx < Np * S; idx += blockDim.x) {
    const int i = idx / S, s = idx % S;
    double a = 0.0;
    for (int j = 0; j < Np; ++j) a += G[i * Np + j] * (proj[s * Np + j] * vol[s]);
    Re[idx] = a;
  }
  for (int idx = threadIdx.x; idx < S * Np; idx += blockDim.x) o.P[e * S * Np + idx] = proj[idx];
  for (int idx = threadIdx.x; idx < S; idx += blockDim.x) o.vol[e * S + idx] = vol[idx];
  for (int idx = threadIdx.x; idx < 3 * S; idx += blockDim.x) o.cen[e * S * 3 + idx] = cen[idx];
  for (int f = threadIdx.x; f < r.NI; f += blockDim.x) {
    const double* oc = cen + r.iown[f] * 3;
    const double* nc = cen + r.inbr[f] * 3;
    const size_t k = e * r.NI + f;
    subface_metrics(pv, r.ifaces + f * 4,
                    [&](const double*, double* dv) {
                      for (int d = 0; d < 3; ++d) dv[d] = nc[d] - oc[d];
                    },
                    o.in_n + k * 3, o.in_a + k, nullptr);
  }
  for (int f = threadIdx.x; f < r.NB; f += blockDim.x) {
    const double* oc = cen + r.bown[f] * 3;
    const size_t k = e * r.NB + f;
    subface_metrics(pv, r.bfaces + f * 4,
                    [&](const double* fc, double* dv) {
                      for (int d = 0; d < 3; ++d) dv[d] = fc[d] - oc[d];
                    },
                    o.bd_n + k * 3, o.bd_a + k, o.bd_c + k * 3);
  }
}

struct SubcellCentres {
  const double* c[DGB_MAX_BLOCKS];   // [E_b][NB_b][3] boundary subface centres per block
  int NB[DGB_MAX_BLOCKS];
};

// One parent face per thread: the neighbour's 16 boundary subfaces (ncand, in its reference order)
// matched to the owner's 16 (osub) by the nearest centre, both taken relative to their side's
// mean; *bad receives 1 + the first face whose match is not a permutation or is farther than
// 2e-6 of max(1, largest owner centre norm).
__global__ void __launch_bounds__(256) k_subcell_match(const FaceDev fd, const SubcellCentres C,
                                                       const int32_t* __restrict__ osub,
                                                       const int32_t* __restrict__ ncand, int32_t* __restrict__ nsub,
                                                       int* bad) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= fd.F) return;
  int32_t* out = nsub + f * kSub;
  const int nb = fd.nb[f];
  if (nb < 0) {
    for (int k = 0; k < kSub; ++k) out[k] = -1;
    return;
  }
  const int ob = fd.ob[f];
  const double* oc = C.c[ob] + (size_t)fd.ol[f] * C.NB[ob] * 3;
  const double* nc = C.c[nb] + (size_t)fd.nl[f] * C.NB[nb] * 3;
  double po[kSub][3], pn[kSub][3], mo[3] = {0.0, 0.0, 0.0}, mn[3] = {0.0, 0.0, 0.0}, scale = 1.0;
  for (int k = 0; k < kSub; ++k) {
    const int a = osub[f * kSub + k], b = ncand[f * kSub + k];
    double r2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      po[k][d] = oc[a * 3 + d];
      pn[k][d] = nc[b * 3 + d];
      mo[d] += po[k][d];
      mn[d] += pn[k][d];
      r2 += po[k][d] * po[k][d];
    }
    scale = fmax(scale, sqrt(r2));
  }
  for (int d = 0; d < 3; ++d) {
    mo[d] /= kSub;
    mn[d] /= kSub;
  }
  unsigned used = 0;
  bool ok = true;
  for (int k = 0; k < kSub; ++k) {
    int best = 0;
    double bd = 0.0;
    for (int m = 0; m < kSub; ++m) {
      double s = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double t = (po[k][d] - mo[d]) - (pn[m][d] - mn[d]);
        s += t * t;
      }
      const double dist = sqrt(s);
      if (m == 0 || dist < bd) {
        bd = dist;
        best = m;
      }
    }
    ok = ok && bd <= 2e-6 * scale && !(used & (1u << best));
    used |= 1u << best;
    out[k] = ncand[f * kSub + best];
  }
  if (!ok) atomicCAS(bad, 0, (int)f + 1);
}

}  // namespace dgb
