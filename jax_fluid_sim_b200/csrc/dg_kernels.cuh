// DG residual-and-update kernels (float64, any element type, P1-P3).
//
// Pipeline of one right-hand-side evaluation (reference: hybrid/spatial.py:137-249 and
// hybrid/navier_stokes.py:27-347):
//   k_traces      element-parallel: traces of U (anchor form and plain), of the viscous
//                 variables and of their raw physical gradients at every face point of the
//                 element's faces, written to face-side buffers.
//   k_face_flux   face-point-parallel: HLLC flux (or boundary ghost) minus each side's anchor
//                 flux, times w; BR2 jump 0.5*w*[v](x)n.
//   k_volume      element-parallel: BR2 lifts r_f = M^-1 (B_f^T jump) per face, their face
//                 values, volume gradients, inviscid and viscous volume residuals.
//   k_face_visc   face-point-parallel: averaged viscous normal flux times w.
//   k_finalize    element-parallel: gathers the element's face contributions in local-face
//                 order (no atomics: deterministic), applies M^-1, and either writes the
//                 right-hand sides or the fused SSP-RK stage (current + dt*rhs, blended).
// Every element kernel is one CTA per element; every face kernel one thread per face point.
#pragma once
#include <stdint.h>

#include "physics.cuh"

namespace dgb {

constexpr int kThreads = 128;

struct BlockDev {
  int type, E, Np, Nq, nlf, Ns;
  const double* B;        // [Nq][Np]
  const double* dB;       // [Nq][Np][3]
  const double* jinv;     // [E][Nq][9]
  const double* wdet;     // [E][Nq]
  const double* minv;     // [E][Np][Np]
  const double* length;   // [E]
  const double* fsB;      // [Ns][Np]
  const double* p1proj;   // [Np][Np]
  const int32_t* elem_face;  // [E][nlf]
  const double* trB[2];   // per face type: [codes][nq][Np]
  const double* trdB[2];  // per face type: [codes][nq][Np][3]
  double* Rinv;           // scratch [E][Np][NV]
  double* Rvis;
  // affine hexahedra (sum-factorised path, optional): constant metrics, M^-1 = coef * (m1i)^(x)3
  const uint8_t* affine;  // [E] 1 where the element map is affine
  const double* acoef;    // [E] sliver scale / det J
  const double* ajinv;    // [E][9] constant inverse Jacobian
  const double* adet;     // [E] det J
};

struct FaceDev {
  int F, nq;
  const int32_t *ob, *ol, *oc, *nb, *nl, *nc, *tag;
  const double* n;        // [F][nq][3]
  const double* w;        // [F][nq]
  const double* jinv;     // [F][2][nq][9]
  double* trA;            // [F][2][nq][NV] anchor-form U traces
  double* trP;            // [F][2][nq][NV] plain U traces
  double* trV;            // [F][2][nq][4]
  double* trG;            // [F][2][nq][12] raw gradients of the viscous variables
  double* fluxI;          // [F][2][nq][NV] (F_hat - F(anchor).n) w per side
  double* jumpW;          // [F][nq][12]    0.5 w [v] (x) n
  double* liftF;          // [F][2][nq][12] br2 * B_f r_f per side
  double* fluxV;          // [F][nq][NV]    viscous normal flux times w
};

struct DevPlan {
  int nv, nblocks, viscous, degree;
  BlockDev blk[DGB_MAX_BLOCKS];
  FaceDev face[2];
  Physics ph;
};

struct StatePtrs {
  double* b[DGB_MAX_BLOCKS];
};

__device__ __forceinline__ void decode_face(int32_t code, int& ft, int& f, int& side) {
  ft = (code >> 30) & 1;
  f = (code >> 1) & ((1 << 29) - 1);
  side = code & 1;
}

// ---------------------------------------------------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(kThreads) k_traces(const DevPlan P, const StatePtrs S, int b) {
  extern __shared__ double smem[];
  const BlockDev& B = P.blk[b];
  const int e = blockIdx.x;
  const int Np = B.Np;
  double* U = smem;                 // [Np][NV]
  double* V = U + Np * NV;          // [Np][4]
  const double* Ug = S.b[b] + (size_t)e * Np * NV;
  for (int i = threadIdx.x; i < Np * NV; i += blockDim.x) U[i] = Ug[i];
  __syncthreads();
  if (P.viscous) {
    for (int i = threadIdx.x; i < Np; i += blockDim.x) viscous_vars<NV>(P.ph, U + i * NV, V + i * 4);
    __syncthreads();
  }
  for (int lf = 0; lf < B.nlf; ++lf) {
    int ft, f, side;
    decode_face(B.elem_face[e * B.nlf + lf], ft, f, side);
    const FaceDev& fd = P.face[ft];
    const int nq = fd.nq;
    const int tc = side == 0 ? fd.oc[f] : fd.nc[f];
    const double* Bt = B.trB[ft] + (size_t)tc * nq * Np;
    const size_t slot = ((size_t)f * 2 + side) * nq;
    for (int idx = threadIdx.x; idx < nq * NV; idx += blockDim.x) {
      const int q = idx / NV, v = idx % NV;
      double s = 0.0;
      for (int i = 0; i < Np; ++i) s += Bt[q * Np + i] * (U[i * NV + v] - U[v]);
      fd.trA[(slot + q) * NV + v] = U[v] + s;
    }
    if (P.viscous) {
      const double* dBt = B.trdB[ft] + (size_t)tc * nq * Np * 3;
      for (int idx = threadIdx.x; idx < nq * NV; idx += blockDim.x) {
        const int q = idx / NV, v = idx % NV;
        double s = 0.0;
        for (int i = 0; i < Np; ++i) s += Bt[q * Np + i] * U[i * NV + v];
        fd.trP[(slot + q) * NV + v] = s;
      }
      for (int idx = threadIdx.x; idx < nq * 4; idx += blockDim.x) {
        const int q = idx / 4, m = idx % 4;
        double s = 0.0;
        for (int i = 0; i < Np; ++i) s += Bt[q * Np + i] * V[i * 4 + m];
        fd.trV[(slot + q) * 4 + m] = s;
      }
      for (int idx = threadIdx.x; idx < nq * 12; idx += blockDim.x) {
        const int q = idx / 12, m = (idx % 12) / 3, d = idx % 3;
        const double* J = fd.jinv + (slot + q) * 9;
        double s = 0.0;
        for (int i = 0; i < Np; ++i) {
          const double* g = dBt + ((size_t)q * Np + i) * 3;
          const double gp = g[0] * J[0 * 3 + d] + g[1] * J[1 * 3 + d] + g[2] * J[2 * 3 + d];
          s += V[i * 4 + m] * gp;
        }
        fd.trG[(slot + q) * 12 + m * 3 + d] = s;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(kThreads) k_face_flux(const DevPlan P, const StatePtrs S, int ft) {
  const FaceDev& fd = P.face[ft];
  const int nq = fd.nq;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= fd.F * nq) return;
  const int f = t / nq, q = t % nq;
  const int ob = fd.ob[f], nb = fd.nb[f];
  const double* n = fd.n + ((size_t)f * nq + q) * 3;
  const double w = fd.w[(size_t)f * nq + q];
  const size_t so = ((size_t)f * 2 + 0) * nq + q, sn = ((size_t)f * 2 + 1) * nq + q;
  double UL[NV], UR[NV], Fh[NV], Fa[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) UL[v] = fd.trA[so * NV + v];
  if (nb >= 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) UR[v] = fd.trA[sn * NV + v];
  } else if (P.ph.has_boundary) {
    ghost_state<NV>(P.ph, UL, n, fd.tag[f], UR);
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) UR[v] = UL[v];
  }
  hllc<NV>(P.ph, UL, UR, n, Fh);
  {
    const double* ao = S.b[ob] + (size_t)fd.ol[f] * P.blk[ob].Np * NV;
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = ao[v];
    normal_flux<NV>(P.ph, a, n, Fa);
#pragma unroll
    for (int v = 0; v < NV; ++v) fd.fluxI[so * NV + v] = (Fh[v] - Fa[v]) * w;
  }
  if (nb >= 0) {
    const double* an = S.b[nb] + (size_t)fd.nl[f] * P.blk[nb].Np * NV;
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = an[v];
    normal_flux<NV>(P.ph, a, n, Fa);
#pragma unroll
    for (int v = 0; v < NV; ++v) fd.fluxI[sn * NV + v] = (Fh[v] - Fa[v]) * w;
  }
  if (P.viscous) {
    double vo[4], vn[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) vo[m] = fd.trV[so * 4 + m];
    if (nb >= 0) {
#pragma unroll
      for (int m = 0; m < 4; ++m) vn[m] = fd.trV[sn * 4 + m];
    } else {
      double Up[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) Up[v] = fd.trP[so * NV + v];
      if (P.ph.has_boundary) viscous_ghost<NV>(P.ph, Up, n, fd.tag[f], vn);
      else viscous_vars<NV>(P.ph, Up, vn);
    }
    double* out = fd.jumpW + ((size_t)f * nq + q) * 12;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int d = 0; d < 3; ++d) out[m * 3 + d] = 0.5 * w * (vn[m] - vo[m]) * n[d];
  }
}

// ---------------------------------------------------------------------------------------------
// Shared-memory layout of k_volume, in doubles.
struct VolumeSmem {
  int U, V, lift, bf, rf, Gi, Gv, total;
  __host__ __device__ VolumeSmem(int Np, int Nq, int nlf, int nv, int viscous) {
    U = 0;
    V = U + Np * nv;
    lift = V + Np * 4;
    bf = lift + (viscous ? Np * 12 : 0);
    rf = bf + (viscous ? nlf * Np * 12 : 0);
    Gi = rf + (viscous ? nlf * Np * 12 : 0);
    Gv = Gi + Nq * 3 * nv;
    total = Gv + (viscous ? Nq * 3 * nv : 0);
  }
};

template <int NV>
__global__ void __launch_bounds__(kThreads) k_volume(const DevPlan P, const StatePtrs S, int b) {
  extern __shared__ double smem[];
  const BlockDev& B = P.blk[b];
  const int e = blockIdx.x;
  const int Np = B.Np, Nq = B.Nq, nlf = B.nlf;
  const VolumeSmem L(Np, Nq, nlf, NV, P.viscous);
  double* U = smem + L.U;
  double* V = smem + L.V;
  double* lift = smem + L.lift;
  double* bf = smem + L.bf;
  double* rf = smem + L.rf;
  double* Gi = smem + L.Gi;
  double* Gv = smem + L.Gv;
  const double* Ug = S.b[b] + (size_t)e * Np * NV;
  for (int i = threadIdx.x; i < Np * NV; i += blockDim.x) U[i] = Ug[i];
  __syncthreads();
  const double* jinv = B.jinv + (size_t)e * Nq * 9;
  const double* wdet = B.wdet + (size_t)e * Nq;
  if (P.viscous) {
    for (int i = threadIdx.x; i < Np; i += blockDim.x) viscous_vars<NV>(P.ph, U + i * NV, V + i * 4);
    // b_f[i][c] = sum_q B_f(q,i) jumpW_f(q,c)
    for (int idx = threadIdx.x; idx < nlf * Np * 12; idx += blockDim.x) {
      const int lf = idx / (Np * 12), i = (idx / 12) % Np, c = idx % 12;
      int ft, f, side;
      decode_face(B.elem_face[e * nlf + lf], ft, f, side);
      const FaceDev& fd = P.face[ft];
      const int nq = fd.nq;
      const int tc = side == 0 ? fd.oc[f] : fd.nc[f];
      const double* Bt = B.trB[ft] + (size_t)tc * nq * Np;
      const double* J = fd.jumpW + (size_t)f * nq * 12;
      double s = 0.0;
      for (int q = 0; q < nq; ++q) s += J[q * 12 + c] * Bt[q * Np + i];
      bf[idx] = s;
    }
    __syncthreads();
    // r_f = M^-1 b_f
    const double* Mi = B.minv + (size_t)e * Np * Np;
    for (int idx = threadIdx.x; idx < nlf * Np * 12; idx += blockDim.x) {
      const int lf = idx / (Np * 12), i = (idx / 12) % Np, c = idx % 12;
      const double* row = Mi + (size_t)i * Np;
      const double* col = bf + (size_t)lf * Np * 12 + c;
      double s = 0.0;
      for (int j = 0; j < Np; ++j) s += row[j] * col[j * 12];
      rf[idx] = s;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < Np * 12; idx += blockDim.x) {
      double s = 0.0;
      for (int lf = 0; lf < nlf; ++lf) s += rf[lf * Np * 12 + idx];
      lift[idx] = s;
    }
    // face values of each face's own lift, scaled by the BR2 penalty
    for (int lf = 0; lf < nlf; ++lf) {
      int ft, f, side;
      decode_face(B.elem_face[e * nlf + lf], ft, f, side);
      const FaceDev& fd = P.face[ft];
      const int nq = fd.nq;
      const int tc = side == 0 ? fd.oc[f] : fd.nc[f];
      const double* Bt = B.trB[ft] + (size_t)tc * nq * Np;
      for (int idx = threadIdx.x; idx < nq * 12; idx += blockDim.x) {
        const int q = idx / 12, c = idx % 12;
        double s = 0.0;
        for (int i = 0; i < Np; ++i) s += Bt[q * Np + i] * rf[(lf * Np + i) * 12 + c];
        fd.liftF[(((size_t)f * 2 + side) * nq + q) * 12 + c] = P.ph.br2 * s;
      }
    }
    __syncthreads();
  }
  // volume terms at each quadrature point
  double Fa[3][NV];
  {
    const double ex[3] = {1.0, 0.0, 0.0}, ey[3] = {0.0, 1.0, 0.0}, ez[3] = {0.0, 0.0, 1.0};
    normal_flux<NV>(P.ph, U, ex, Fa[0]);
    normal_flux<NV>(P.ph, U, ey, Fa[1]);
    normal_flux<NV>(P.ph, U, ez, Fa[2]);
  }
  for (int q = threadIdx.x; q < Nq; q += blockDim.x) {
    const double* Bq = B.B + (size_t)q * Np;
    const double* J = jinv + q * 9;
    const double wq = wdet[q];
    double Uq[NV], F[3][NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = 0.0;
      for (int i = 0; i < Np; ++i) s += Bq[i] * (U[i * NV + v] - U[v]);
      Uq[v] = U[v] + s;
    }
    {
      const double ex[3] = {1.0, 0.0, 0.0}, ey[3] = {0.0, 1.0, 0.0}, ez[3] = {0.0, 0.0, 1.0};
      normal_flux<NV>(P.ph, Uq, ex, F[0]);
      normal_flux<NV>(P.ph, Uq, ey, F[1]);
      normal_flux<NV>(P.ph, Uq, ez, F[2]);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int v = 0; v < NV; ++v)
        Gi[(q * 3 + r) * NV + v] = (J[r * 3 + 0] * (F[0][v] - Fa[0][v]) + J[r * 3 + 1] * (F[1][v] - Fa[1][v]) +
                                    J[r * 3 + 2] * (F[2][v] - Fa[2][v])) * wq;
    if (P.viscous) {
      double Up[NV], grad[12];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double s = 0.0;
        for (int i = 0; i < Np; ++i) s += Bq[i] * U[i * NV + v];
        Up[v] = s;
      }
#pragma unroll
      for (int c = 0; c < 12; ++c) grad[c] = 0.0;
      for (int i = 0; i < Np; ++i) {
        const double* g = B.dB + ((size_t)q * Np + i) * 3;
        double gp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) gp[d] = g[0] * J[0 * 3 + d] + g[1] * J[1 * 3 + d] + g[2] * J[2 * 3 + d];
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int d = 0; d < 3; ++d) grad[m * 3 + d] += V[i * 4 + m] * gp[d];
      }
#pragma unroll
      for (int c = 0; c < 12; ++c) {
        double s = 0.0;
        for (int i = 0; i < Np; ++i) s += Bq[i] * lift[i * 12 + c];
        grad[c] += s;
      }
      double Fv[3 * NV];
      viscous_flux<NV>(P.ph, Up, grad, Fv);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int v = 0; v < NV; ++v)
          Gv[(q * 3 + r) * NV + v] =
              -(J[r * 3 + 0] * Fv[0 * NV + v] + J[r * 3 + 1] * Fv[1 * NV + v] + J[r * 3 + 2] * Fv[2 * NV + v]) * wq;
    }
  }
  __syncthreads();
  double* Ri = B.Rinv + (size_t)e * Np * NV;
  double* Rv = B.Rvis + (size_t)e * Np * NV;
  for (int idx = threadIdx.x; idx < Np * NV; idx += blockDim.x) {
    const int i = idx / NV, v = idx % NV;
    double si = 0.0, sv = 0.0;
    for (int q = 0; q < Nq; ++q) {
      const double* g = B.dB + ((size_t)q * Np + i) * 3;
      si += g[0] * Gi[(q * 3 + 0) * NV + v] + g[1] * Gi[(q * 3 + 1) * NV + v] + g[2] * Gi[(q * 3 + 2) * NV + v];
      if (P.viscous)
        sv += g[0] * Gv[(q * 3 + 0) * NV + v] + g[1] * Gv[(q * 3 + 1) * NV + v] + g[2] * Gv[(q * 3 + 2) * NV + v];
    }
    Ri[idx] = si;
    if (P.viscous) Rv[idx] = sv;
  }
}

// ---------------------------------------------------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(kThreads) k_face_visc(const DevPlan P, int ft) {
  const FaceDev& fd = P.face[ft];
  const int nq = fd.nq;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= fd.F * nq) return;
  const int f = t / nq, q = t % nq;
  const int nb = fd.nb[f];
  const double* n = fd.n + ((size_t)f * nq + q) * 3;
  const double w = fd.w[(size_t)f * nq + q];
  const size_t so = ((size_t)f * 2 + 0) * nq + q, sn = ((size_t)f * 2 + 1) * nq + q;
  double U[NV], g[12], Fo[3 * NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) U[v] = fd.trP[so * NV + v];
#pragma unroll
  for (int c = 0; c < 12; ++c) g[c] = fd.trG[so * 12 + c] + fd.liftF[so * 12 + c];
  viscous_flux<NV>(P.ph, U, g, Fo);
  if (nb >= 0) {
    double Fn[3 * NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) U[v] = fd.trP[sn * NV + v];
#pragma unroll
    for (int c = 0; c < 12; ++c) g[c] = fd.trG[sn * 12 + c] + fd.liftF[sn * 12 + c];
    viscous_flux<NV>(P.ph, U, g, Fn);
#pragma unroll
    for (int k = 0; k < 3 * NV; ++k) Fo[k] = 0.5 * (Fo[k] + Fn[k]);
  }
  double out[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = Fo[0 * NV + v] * n[0] + Fo[1 * NV + v] * n[1] + Fo[2 * NV + v] * n[2];
  if (nb < 0 && P.ph.has_boundary && tag_in(fd.tag[f], P.ph.wall, P.ph.n_wall)) out[4] = 0.0;
#pragma unroll
  for (int v = 0; v < NV; ++v) fd.fluxV[((size_t)f * nq + q) * NV + v] = out[v] * w;
}

// ---------------------------------------------------------------------------------------------
struct FinalizeArgs {
  double* out_inv[DGB_MAX_BLOCKS];   // rhs outputs (may be null)
  double* out_vis[DGB_MAX_BLOCKS];
  // fused SSP-RK stage: dst = alpha*base + beta*(cur + dt*(rhs_inv + rhs_vis)); euler = cur + dt*rhs
  int stage;
  double alpha, beta, dt;
  const double* base[DGB_MAX_BLOCKS];
  double* dst[DGB_MAX_BLOCKS];
  double* euler[DGB_MAX_BLOCKS];     // may be null
};

template <int NV>
__global__ void __launch_bounds__(kThreads) k_finalize(const DevPlan P, const StatePtrs S, int b,
                                                      const FinalizeArgs A) {
  extern __shared__ double smem[];
  const BlockDev& B = P.blk[b];
  const int e = blockIdx.x;
  const int Np = B.Np, nlf = B.nlf;
  double* Ri = smem;
  double* Rv = smem + Np * NV;
  const size_t base = (size_t)e * Np * NV;
  for (int idx = threadIdx.x; idx < Np * NV; idx += blockDim.x) {
    const int i = idx / NV, v = idx % NV;
    double si = B.Rinv[base + idx];
    double sv = P.viscous ? B.Rvis[base + idx] : 0.0;
    for (int lf = 0; lf < nlf; ++lf) {
      int ft, f, side;
      decode_face(B.elem_face[e * nlf + lf], ft, f, side);
      const FaceDev& fd = P.face[ft];
      const int nq = fd.nq;
      const int tc = side == 0 ? fd.oc[f] : fd.nc[f];
      const double* Bt = B.trB[ft] + (size_t)tc * nq * Np;
      const double* fi = fd.fluxI + ((size_t)f * 2 + side) * nq * NV;
      double s = 0.0;
      for (int q = 0; q < nq; ++q) s += Bt[q * Np + i] * fi[q * NV + v];
      si += side == 0 ? -s : s;
      if (P.viscous) {
        const double* fv = fd.fluxV + (size_t)f * nq * NV;
        double t = 0.0;
        for (int q = 0; q < nq; ++q) t += Bt[q * Np + i] * fv[q * NV + v];
        sv += side == 0 ? t : -t;
      }
    }
    Ri[idx] = si;
    Rv[idx] = sv;
  }
  __syncthreads();
  const double* Mi = B.minv + (size_t)e * Np * Np;
  for (int idx = threadIdx.x; idx < Np * NV; idx += blockDim.x) {
    const int i = idx / NV, v = idx % NV;
    const double* row = Mi + (size_t)i * Np;
    double ri = 0.0, rv = 0.0;
    for (int j = 0; j < Np; ++j) {
      ri += row[j] * Ri[j * NV + v];
      rv += row[j] * Rv[j * NV + v];
    }
    if (!A.stage) {
      if (A.out_inv[b]) A.out_inv[b][base + idx] = ri;
      if (A.out_vis[b]) A.out_vis[b][base + idx] = rv;
    } else {
      const double total = P.viscous ? ri + rv : ri;
      const double eul = S.b[b][base + idx] + A.dt * total;
      if (A.out_vis[b]) A.out_vis[b][base + idx] = rv;
      if (A.euler[b]) A.euler[b][base + idx] = eul;
      A.dst[b][base + idx] = A.alpha * A.base[b][base + idx] + A.beta * eul;
    }
  }
}

}  // namespace dgb
