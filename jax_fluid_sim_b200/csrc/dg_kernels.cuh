// DG residual-and-update kernels for any element type (hexahedron, wedge, tetrahedron; P1-P3).
//
// Pipeline of one right-hand-side evaluation (reference: hybrid/spatial.py:137-249 and
// hybrid/navier_stokes.py:27-347):
//   k_traces      element-parallel: anchor-form traces of U, traces of the viscous variables
//                 and of their raw physical gradients at every face point of the element's
//                 faces, written to face-side buffers.
//   k_face_flux   face-point-parallel: HLLC flux (or boundary ghost) minus each side's anchor
//                 flux, times w; BR2 jump 0.5*w*[v](x)n.
//   k_volume      element-parallel: BR2 lifts r_f = M^-1 (B_f^T jump) per face, their face
//                 values, volume gradients, inviscid and viscous volume residuals.
//   k_face_visc   face-point-parallel: averaged viscous normal flux times w.
//   k_finalize    element-parallel: gathers the element's face contributions in local-face
//                 order (no atomics: deterministic), applies M^-1, and either writes the
//                 right-hand sides or the fused SSP-RK stage (current + dt*rhs, blended).
// The element kernels cover every block in one launch (ElemLaunch): a CTA of kThreads works on
// G = kThreads / W elements of one block, W threads each (W a power of two >= the element's
// nodes, volume points and face points, so P1 elements share a CTA and P2/P3 take one each).
// They are templated on the arithmetic type R: double, or float for precision mode 1 (state,
// anchors, face buffers and the stage update stay double).  Every face kernel is one thread per
// face point.
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
  double lebesgue;        // max over the limiter samples (nodes, volume, face) of sum_i |B_i|
  const double* length;   // [E]
  const double* fsB;      // [Ns][Np]
  const double* p1proj;   // [Np][Np]
  const int32_t* elem_face;  // [E][nlf]
  const double* trB[2];   // per face type: [codes][nq][Np]
  const double* trdB[2];  // per face type: [codes][nq][Np][3]
  // the same tables laid out so that the thread index runs along the fastest axis (coalesced):
  const double* Bt;       // [Np][Nq]            (thread per volume point)
  const double* dBq;      // [Np][3][Nq]         (thread per volume point)
  const double* dBi;      // [Nq][3][Np]         (thread per node)
  const double* trBt[2];  // [codes][Np][nq]     (thread per face point)
  const double* trdBt[2]; // [codes][Np][3][nq]  (thread per face point)
  double* Rinv;           // scratch [E][Np][NV]
  double* Rvis;
  // affine elements (optional): constant metrics; M^-1 = coef * (m1i)^(x)3 on the sum-factorised
  // hexahedron path, coef * mref_inv on the dense path
  const uint8_t* affine;  // [E] 1 where the element map is affine
  const double* acoef;    // [E] sliver scale / |det J|
  const double* ajinv;    // [E][9] constant inverse Jacobian
  const double* adet;     // [E] |det J|
  const double* wref;     // [Nq] reference quadrature weights (dense path)
  const double* mref_inv; // [Np][Np] inverse of the reference mass matrix B^T diag(wref) B (dense path)
  const int32_t* ecase;   // [E] case of each element (ensembles; null for one case)
  // float32 copies read by the mixed-precision hexahedron kernels (null in float64 plans)
  const float* minv32;    // [E][Np][Np], same layout as minv
  const float* jinv32;    // [E][Nq][9]
};

struct FaceDev {
  int F, nq;
  const int32_t *ob, *ol, *oc, *nb, *nl, *nc, *tag;
  const double* n;        // [F][nq][3]
  const double* w;        // [F][nq]
  const double* jinv;     // [F][2][nq][9]
  double* trA;            // [F][2][nq][NV] anchor-form U traces
  double* anc;            // [F][2][NV] anchor state (node 0) of each side's element
  double* trP;            // [F][2][nq][NV] plain U traces
  double* trV;            // [F][2][nq][4]
  double* trG;            // [F][2][nq][12] raw gradients of the viscous variables
  double* fluxI;          // [F][2][nq][NV] (F_hat - F(anchor).n) w per side
  double* jumpW;          // [F][nq][12]    0.5 w [v] (x) n
  double* liftF;          // [F][2][nq][12] br2 * B_f r_f per side
  double* fluxV;          // [F][nq][NV]    viscous normal flux times w
  const float* jinv32;    // float32 copy of jinv (mixed-precision plans; else null)
  // float32 traces of the viscous variables and their gradients, written and read by the fused
  // hexahedron kernels of mixed-precision plans (else null)
  float* trV32;           // [F][2][nq][4]
  float* trG32;           // [F][2][nq][12]
  // float32 face fluxes and BR2 jumps of the fused hexahedron kernels of mixed-precision plans (the
  // element kernel rounds them to float32 anyway)
  float* fluxI32;         // [F][2][nq][NV]
  float* fluxV32;         // [F][nq][NV]
  float* jumpW32;         // [F][nq][12]
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

// One launch over all blocks: CTAs [cta0[b], cta0[b+1]) work on block b, kThreads / W[b] elements
// per CTA, slot[b] bytes of dynamic shared memory per element.
struct ElemLaunch {
  int nblocks;
  int cta0[DGB_MAX_BLOCKS + 1];
  int W[DGB_MAX_BLOCKS];
  int slot[DGB_MAX_BLOCKS];
};

constexpr int kMaxGroups = kThreads / 16;   // W >= 16

__device__ __forceinline__ int launch_block(const ElemLaunch& L) {
  int b = 0;
  while (b + 1 < L.nblocks && (int)blockIdx.x >= L.cta0[b + 1]) ++b;
  return b;
}

__device__ __forceinline__ void decode_face(int32_t code, int& ft, int& f, int& side) {
  ft = (code >> 30) & 1;
  f = (code >> 1) & ((1 << 29) - 1);
  side = code & 1;
}

// ---------------------------------------------------------------------------------------------
// Per-element face table of the element kernels: for local face lf its face type, face index,
// side and trace code.
struct ElemFaces {
  int ft[6], f[6], side[6], code[6], nq[6];
};

__device__ __forceinline__ void load_faces(const DevPlan& P, const BlockDev& B, int e, int lane, ElemFaces& F) {
  if (lane < B.nlf) {
    int ft, f, side;
    decode_face(B.elem_face[(size_t)e * B.nlf + lane], ft, f, side);
    F.ft[lane] = ft;
    F.f[lane] = f;
    F.side[lane] = side;
    F.code[lane] = side == 0 ? P.face[ft].oc[f] : P.face[ft].nc[f];
    F.nq[lane] = P.face[ft].nq;
  }
}

// Shared memory per element (in R values) of k_traces: U - anchor [Np][NV], v [Np][4].
__host__ __device__ inline int traces_slot(int Np, int nv) { return Np * (nv + 4); }

template <int NV, typename R>
__global__ void __launch_bounds__(kThreads) k_traces(const DevPlan P, const StatePtrs S, const ElemLaunch L) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ ElemFaces faces[kMaxGroups];
  __shared__ double anchor[kMaxGroups][NV];
  const int b = launch_block(L);
  const BlockDev& B = P.blk[b];
  const int W = L.W[b], g = threadIdx.x / W, lane = threadIdx.x % W;
  const int e = (blockIdx.x - L.cta0[b]) * (kThreads / W) + g;
  const bool live = e < B.E;
  const int Np = B.Np, nlf = B.nlf;
  R* U = reinterpret_cast<R*>(dyn_smem + (size_t)g * L.slot[b]);
  R* V = U + Np * NV;
  const double* Ug = S.b[b] + (size_t)(live ? e : 0) * Np * NV;
  if (live) {
    load_faces(P, B, e, lane, faces[g]);
    if (lane < NV) anchor[g][lane] = Ug[lane];
  }
  __syncthreads();
  if (live) {
    for (int i = lane; i < Np * NV; i += W) U[i] = (R)(Ug[i] - anchor[g][i % NV]);
    if (P.viscous)
      for (int i = lane; i < Np; i += W) {
        double u[NV], vv[4];
#pragma unroll
        for (int v = 0; v < NV; ++v) u[v] = Ug[i * NV + v];
        viscous_vars<NV>(P.ph, u, vv);
#pragma unroll
        for (int m = 0; m < 4; ++m) V[i * 4 + m] = (R)vv[m];
      }
  }
  __syncthreads();
  if (!live) return;
  const ElemFaces& Fc = faces[g];
  int items = 0;
  for (int lf = 0; lf < nlf; ++lf) items += Fc.nq[lf];
  for (int t = lane; t < items; t += W) {
    int lf = 0, q = t;
    while (q >= Fc.nq[lf]) q -= Fc.nq[lf++];
    const int ft = Fc.ft[lf], nq = Fc.nq[lf];
    const FaceDev& fd = P.face[ft];
    const double* Bt = B.trBt[ft] + (size_t)Fc.code[lf] * Np * nq + q;    // [i][q]: stride nq
    const size_t pt = ((size_t)Fc.f[lf] * 2 + Fc.side[lf]) * nq + q;
    R acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = (R)0;
    for (int i = 0; i < Np; ++i) {
      const R bt = (R)Bt[(size_t)i * nq];
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] += bt * U[i * NV + v];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) fd.trA[pt * NV + v] = anchor[g][v] + (double)acc[v];
    if (q == 0)
#pragma unroll
      for (int v = 0; v < NV; ++v) fd.anc[((size_t)Fc.f[lf] * 2 + Fc.side[lf]) * NV + v] = anchor[g][v];
    if (P.viscous) {
      const double* dBt = B.trdBt[ft] + (size_t)Fc.code[lf] * Np * 3 * nq + q;   // [i][r][q]
      R J[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) J[k] = (R)fd.jinv[pt * 9 + k];
      R tv[4], tg[12];
#pragma unroll
      for (int k = 0; k < 4; ++k) tv[k] = (R)0;
#pragma unroll
      for (int k = 0; k < 12; ++k) tg[k] = (R)0;
      for (int i = 0; i < Np; ++i) {
        const R bt = (R)Bt[(size_t)i * nq];
        const double* gi = dBt + (size_t)i * 3 * nq;
        const R g0 = (R)gi[0], g1 = (R)gi[nq], g2 = (R)gi[2 * nq];
        R gp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) gp[d] = g0 * J[0 * 3 + d] + g1 * J[1 * 3 + d] + g2 * J[2 * 3 + d];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const R vm = V[i * 4 + m];
          tv[m] += bt * vm;
#pragma unroll
          for (int d = 0; d < 3; ++d) tg[m * 3 + d] += vm * gp[d];
        }
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) fd.trV[pt * 4 + m] = (double)tv[m];
#pragma unroll
      for (int k = 0; k < 12; ++k) fd.trG[pt * 12 + k] = (double)tg[k];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// k_face_flux: one thread per face point.  Every input is independent of the others (traces,
// normal, weight, and each side's anchor state, which the trace kernels write per face side), so
// a thread issues all its loads at once instead of chasing face -> element -> state.
template <int NV>
__global__ void __launch_bounds__(kThreads, NV <= 5 ? 6 : 1) k_face_flux(const DevPlan P, const StatePtrs S, int ft) {
  const FaceDev& fd = P.face[ft];
  const int nq = fd.nq;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= fd.F * nq) return;
  const int f = t / nq, q = t % nq;
  const int nb = fd.nb[f];
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
    ghost_state<NV>(P.ph, case_view(P.ph, P.blk[fd.ob[f]].ecase, fd.ol[f]).far, UL, n, fd.tag[f], UR);
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) UR[v] = UL[v];
  }
  hllc<NV>(P.ph, UL, UR, n, Fh);
  {
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = fd.anc[((size_t)f * 2 + 0) * NV + v];
    normal_flux<NV>(P.ph, a, n, Fa);
#pragma unroll
    for (int v = 0; v < NV; ++v) fd.fluxI[so * NV + v] = (Fh[v] - Fa[v]) * w;
  }
  if (nb >= 0) {
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = fd.anc[((size_t)f * 2 + 1) * NV + v];
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
    } else if (P.ph.has_boundary) {
      const CaseView cv = case_view(P.ph, P.blk[fd.ob[f]].ecase, fd.ol[f]);
      viscous_ghost<NV>(P.ph, cv.far, cv.wall_T, UL, n, fd.tag[f], vn);
    } else {
      viscous_vars<NV>(P.ph, UL, vn);
    }
    double* out = fd.jumpW + ((size_t)f * nq + q) * 12;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int d = 0; d < 3; ++d) out[m * 3 + d] = 0.5 * w * (vn[m] - vo[m]) * n[d];
  }
}

// ---------------------------------------------------------------------------------------------
// Shared-memory layout of k_volume per element, in R values.  The residual sum over volume points
// is split into C chunks of points (C = W / Np threads per node) and the chunks' partial sums
// are added in a second pass.
struct VolumeSmem {
  int U, V, lift, bf, rf, Gi, Gv, Rp, Rpv, total;
  __host__ __device__ VolumeSmem(int Np, int Nq, int nlf, int nv, int viscous, int C) {
    U = 0;
    V = U + Np * nv;
    lift = V + (viscous ? Np * 4 : 0);
    bf = lift + (viscous ? Np * 12 : 0);
    rf = bf + (viscous ? nlf * Np * 12 : 0);
    Gi = rf + (viscous ? nlf * Np * 12 : 0);
    Gv = Gi + Nq * 3 * nv;
    Rp = Gv + (viscous ? Nq * 3 * nv : 0);
    Rpv = Rp + C * Np * nv;
    total = Rpv + (viscous ? C * Np * nv : 0);
  }
};

__host__ __device__ inline int volume_chunks(int Np, int W) { return Np <= W ? W / Np : 1; }

template <int NV, typename R>
__global__ void __launch_bounds__(kThreads, NV <= 5 ? 4 : 1) k_volume(const DevPlan P, const StatePtrs S,
                                                                    const ElemLaunch L) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ ElemFaces faces[kMaxGroups];
  __shared__ double anchor[kMaxGroups][NV];
  const int b = launch_block(L);
  const BlockDev& B = P.blk[b];
  const int W = L.W[b], g = threadIdx.x / W, lane = threadIdx.x % W;
  const int e = (blockIdx.x - L.cta0[b]) * (kThreads / W) + g;
  const bool live = e < B.E;
  const int Np = B.Np, Nq = B.Nq, nlf = B.nlf;
  const int C = volume_chunks(Np, W);
  const VolumeSmem Ls(Np, Nq, nlf, NV, P.viscous, C);
  R* sm = reinterpret_cast<R*>(dyn_smem + (size_t)g * L.slot[b]);
  R* U = sm + Ls.U;
  R* V = sm + Ls.V;
  R* lift = sm + Ls.lift;
  R* bf = sm + Ls.bf;
  R* rf = sm + Ls.rf;
  R* Gi = sm + Ls.Gi;
  R* Gv = sm + Ls.Gv;
  R* Rp = sm + Ls.Rp;
  R* Rpv = sm + Ls.Rpv;
  const size_t ee = live ? e : 0;
  const double* Ug = S.b[b] + ee * Np * NV;
  if (live) {
    load_faces(P, B, (int)ee, lane, faces[g]);
    if (lane < NV) anchor[g][lane] = Ug[lane];
  }
  __syncthreads();
  // affine elements read one inverse Jacobian and |det J| instead of per-point tables
  const bool aff = B.affine != nullptr && B.affine[ee];
  const double* jinv = aff ? B.ajinv + ee * 9 : B.jinv + ee * Nq * 9;
  const int jstride = aff ? 0 : 9;
  const double* wdet = aff ? B.wref : B.wdet + ee * Nq;
  const double wscale = aff ? B.adet[ee] : 1.0;
  const double* Mi = aff ? B.mref_inv : B.minv + ee * Np * Np;
  const R mscale = (R)(aff ? B.acoef[ee] : 1.0);
  const CaseView cv = case_view(P.ph, B.ecase, ee);
  const ElemFaces& Fc = faces[g];
  if (live) {
    for (int i = lane; i < Np * NV; i += W) U[i] = (R)(Ug[i] - anchor[g][i % NV]);
    if (P.viscous) {
      for (int i = lane; i < Np; i += W) {
        double u[NV], vv[4];
#pragma unroll
        for (int v = 0; v < NV; ++v) u[v] = Ug[i * NV + v];
        viscous_vars<NV>(P.ph, u, vv);
#pragma unroll
        for (int m = 0; m < 4; ++m) V[i * 4 + m] = (R)vv[m];
      }
      // b_f[i][c] = sum_q B_f(q,i) jumpW_f(q,c)
      for (int idx = lane; idx < nlf * Np * 12; idx += W) {
        const int lf = idx / (Np * 12), i = (idx / 12) % Np, c = idx % 12;
        const int nq = Fc.nq[lf];
        const double* Bt = B.trB[Fc.ft[lf]] + (size_t)Fc.code[lf] * nq * Np;
        const double* Jw = P.face[Fc.ft[lf]].jumpW + (size_t)Fc.f[lf] * nq * 12;
        R acc = (R)0;
        for (int q = 0; q < nq; ++q) acc += (R)Jw[q * 12 + c] * (R)Bt[q * Np + i];
        bf[idx] = acc;
      }
    }
  }
  __syncthreads();
  if (live && P.viscous) {
    // r_f = M^-1 b_f
    for (int idx = lane; idx < nlf * Np * 12; idx += W) {
      const int lf = idx / (Np * 12), i = (idx / 12) % Np, c = idx % 12;
      const double* row = Mi + (size_t)i * Np;
      const R* col = bf + (size_t)lf * Np * 12 + c;
      R acc = (R)0;
      for (int j = 0; j < Np; ++j) acc += (R)row[j] * col[j * 12];
      rf[idx] = mscale * acc;
    }
  }
  __syncthreads();
  if (live && P.viscous) {
    for (int idx = lane; idx < Np * 12; idx += W) {
      R acc = (R)0;
      for (int lf = 0; lf < nlf; ++lf) acc += rf[lf * Np * 12 + idx];
      lift[idx] = acc;
    }
    // face values of each face's own lift, scaled by the BR2 penalty
    int items = 0;
    for (int lf = 0; lf < nlf; ++lf) items += Fc.nq[lf] * 12;
    for (int t = lane; t < items; t += W) {
      int lf = 0, r = t;
      while (r >= Fc.nq[lf] * 12) r -= Fc.nq[lf++] * 12;
      const int q = r / 12, c = r % 12, nq = Fc.nq[lf];
      const double* Bt = B.trB[Fc.ft[lf]] + ((size_t)Fc.code[lf] * nq + q) * Np;
      R acc = (R)0;
      for (int i = 0; i < Np; ++i) acc += (R)Bt[i] * rf[(lf * Np + i) * 12 + c];
      P.face[Fc.ft[lf]].liftF[(((size_t)Fc.f[lf] * 2 + Fc.side[lf]) * nq + q) * 12 + c] =
          P.ph.br2 * (double)acc;
    }
  }
  __syncthreads();
  // volume terms at each quadrature point
  if (live) {
    R a[NV], Fa[3][NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = (R)anchor[g][v];
    {
      const R ex[3] = {(R)1, (R)0, (R)0}, ey[3] = {(R)0, (R)1, (R)0}, ez[3] = {(R)0, (R)0, (R)1};
      normal_flux<NV>(P.ph, a, ex, Fa[0]);
      normal_flux<NV>(P.ph, a, ey, Fa[1]);
      normal_flux<NV>(P.ph, a, ez, Fa[2]);
    }
    for (int q = lane; q < Nq; q += W) {
      const double* Bq = B.Bt + q;                    // [i][q]: stride Nq
      const double* Jd = jinv + q * jstride;
      R J[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) J[k] = (R)Jd[k];
      const R wq = (R)(wdet[q] * wscale);
      R Uq[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) Uq[v] = (R)0;
      for (int i = 0; i < Np; ++i) {
        const R bq = (R)Bq[(size_t)i * Nq];
#pragma unroll
        for (int v = 0; v < NV; ++v) Uq[v] += bq * U[i * NV + v];
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) Uq[v] = (R)(anchor[g][v] + (double)Uq[v]);
      R F[3][NV];
      {
        const R ex[3] = {(R)1, (R)0, (R)0}, ey[3] = {(R)0, (R)1, (R)0}, ez[3] = {(R)0, (R)0, (R)1};
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
        R grad[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) grad[c] = (R)0;
        for (int i = 0; i < Np; ++i) {
          const double* gd = B.dBq + (size_t)i * 3 * Nq + q;   // [i][r][q]
          const R g0 = (R)gd[0], g1 = (R)gd[Nq], g2 = (R)gd[2 * Nq], bq = (R)Bq[(size_t)i * Nq];
          R gp[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) gp[d] = g0 * J[0 * 3 + d] + g1 * J[1 * 3 + d] + g2 * J[2 * 3 + d];
#pragma unroll
          for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int d = 0; d < 3; ++d) grad[m * 3 + d] += V[i * 4 + m] * gp[d] + bq * lift[i * 12 + m * 3 + d];
        }
        R Fv[3 * NV];
        viscous_flux<NV>(P.ph, cv.mu, cv.kappa, Uq, grad, Fv);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int v = 0; v < NV; ++v)
            Gv[(q * 3 + r) * NV + v] =
                -(J[r * 3 + 0] * Fv[0 * NV + v] + J[r * 3 + 1] * Fv[1 * NV + v] + J[r * 3 + 2] * Fv[2 * NV + v]) * wq;
      }
    }
  }
  __syncthreads();
  // residual: thread (node i, chunk c) sums its chunk of points, all variables at once
  if (live) {
    for (int t = lane; t < C * Np; t += W) {
      const int i = t % Np, c = t / Np;
      const int q0 = c * Nq / C, q1 = (c + 1) * Nq / C;
      R si[NV], sv[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) si[v] = sv[v] = (R)0;
      for (int q = q0; q < q1; ++q) {
        const double* gd = B.dBi + (size_t)q * 3 * Np + i;     // [q][r][i]
        const R g0 = (R)gd[0], g1 = (R)gd[Np], g2 = (R)gd[2 * Np];
        const R* G = Gi + q * 3 * NV;
#pragma unroll
        for (int v = 0; v < NV; ++v) si[v] += g0 * G[v] + g1 * G[NV + v] + g2 * G[2 * NV + v];
        if (P.viscous) {
          const R* H = Gv + q * 3 * NV;
#pragma unroll
          for (int v = 0; v < NV; ++v) sv[v] += g0 * H[v] + g1 * H[NV + v] + g2 * H[2 * NV + v];
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) Rp[(c * Np + i) * NV + v] = si[v];
      if (P.viscous)
#pragma unroll
        for (int v = 0; v < NV; ++v) Rpv[(c * Np + i) * NV + v] = sv[v];
    }
  }
  __syncthreads();
  if (live) {
    double* Ri = B.Rinv + ee * Np * NV;
    double* Rv = B.Rvis + ee * Np * NV;
    for (int idx = lane; idx < Np * NV; idx += W) {
      R si = (R)0, sv = (R)0;
      for (int c = 0; c < C; ++c) {
        si += Rp[c * Np * NV + idx];
        if (P.viscous) sv += Rpv[c * Np * NV + idx];
      }
      Ri[idx] = (double)si;
      if (P.viscous) Rv[idx] = (double)sv;
    }
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
  // the two sides of a face always belong to one case
  const CaseView cv = case_view(P.ph, P.blk[fd.ob[f]].ecase, fd.ol[f]);
  double U[NV], g[12], Fo[3 * NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) U[v] = fd.trP[so * NV + v];
#pragma unroll
  for (int c = 0; c < 12; ++c) g[c] = fd.trG[so * 12 + c] + fd.liftF[so * 12 + c];
  viscous_flux<NV>(P.ph, cv.mu, cv.kappa, U, g, Fo);
  if (nb >= 0) {
    double Fn[3 * NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) U[v] = fd.trP[sn * NV + v];
#pragma unroll
    for (int c = 0; c < 12; ++c) g[c] = fd.trG[sn * 12 + c] + fd.liftF[sn * 12 + c];
    viscous_flux<NV>(P.ph, cv.mu, cv.kappa, U, g, Fn);
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
// Surface forces on the wall faces (hybrid/aerodynamics.py:149-250), from the face buffers of a
// right-hand-side evaluation: pressure traction p n dA and viscous traction -(tau . n) dA of the
// owner side at every face point, and their moments about a centre.  One thread per face point;
// each CTA reduces its 12 sums in a fixed order into partials[blockIdx.x].
struct WallSet {
  int tags[DGB_MAX_TAGS];
  int n;
  double center[3];
};

constexpr int kForceValues = 12;   // F_pressure (3), M_pressure (3), F_viscous (3), M_viscous (3)

template <int NV>
__global__ void __launch_bounds__(kThreads) k_wall_forces(const DevPlan P, int ft, const double* __restrict__ points,
                                                         const WallSet walls, double* __restrict__ partials) {
  __shared__ double red[kForceValues][kThreads];
  const FaceDev& fd = P.face[ft];
  const int nq = fd.nq;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double c[kForceValues];
#pragma unroll
  for (int k = 0; k < kForceValues; ++k) c[k] = 0.0;
  if (t < (long)fd.F * nq) {
    const int f = (int)(t / nq), q = (int)(t % nq);
    if (fd.nb[f] < 0 && tag_in(fd.tag[f], walls.tags, walls.n)) {
      const size_t so = ((size_t)f * 2 + 0) * nq + q;
      const double* n = fd.n + ((size_t)f * nq + q) * 3;
      const double w = fd.w[(size_t)f * nq + q];
      const double* x = points + ((size_t)f * nq + q) * 3;
      const double r[3] = {x[0] - walls.center[0], x[1] - walls.center[1], x[2] - walls.center[2]};
      double U[NV], W[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) U[v] = fd.trA[so * NV + v];
      primitive<NV>(P.ph, U, W);
      double F[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) F[d] = W[4] * n[d] * w;
      c[0] = F[0];
      c[1] = F[1];
      c[2] = F[2];
      c[3] = r[1] * F[2] - r[2] * F[1];
      c[4] = r[2] * F[0] - r[0] * F[2];
      c[5] = r[0] * F[1] - r[1] * F[0];
      if (P.viscous) {
        double g[12], Fv[3 * NV];
#pragma unroll
        for (int k = 0; k < 12; ++k) g[k] = fd.trG[so * 12 + k] + fd.liftF[so * 12 + k];
        const CaseView cv = case_view(P.ph, P.blk[fd.ob[f]].ecase, fd.ol[f]);
        viscous_flux<NV>(P.ph, cv.mu, cv.kappa, U, g, Fv);
#pragma unroll
        for (int i = 0; i < 3; ++i)
          F[i] = -(Fv[0 * NV + 1 + i] * n[0] + Fv[1 * NV + 1 + i] * n[1] + Fv[2 * NV + 1 + i] * n[2]) * w;
        c[6] = F[0];
        c[7] = F[1];
        c[8] = F[2];
        c[9] = r[1] * F[2] - r[2] * F[1];
        c[10] = r[2] * F[0] - r[0] * F[2];
        c[11] = r[0] * F[1] - r[1] * F[0];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kForceValues; ++k) red[k][threadIdx.x] = c[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int k = 0; k < kForceValues; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < kForceValues) partials[(size_t)blockIdx.x * kForceValues + threadIdx.x] = red[threadIdx.x][0];
}

// Sums the CTAs' partials in order (one thread per component).
static __global__ void k_wall_forces_final(const double* __restrict__ partials, int n, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kForceValues) return;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += partials[(size_t)i * kForceValues + k];
  out[k] = s;
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
  // elements whose high-order inviscid update is not needed (the learned predictor sent them to
  // the subcell scheme, which uses only their viscous residual); null: none.  Read by the fused
  // hexahedron element kernel.
  const uint8_t* skip_inviscid;
  // element selection of the fused hexahedron element kernel (null: every element): only the
  // elements flagged in `only`, none of those flagged in `skip`
  const uint8_t* only;
  const uint8_t* skip;
};

// Shared memory per element (in R values) of k_finalize: face partials [nlf][Np][NV] and the
// totals [Np][NV], inviscid and (when viscous) viscous.
__host__ __device__ inline int finalize_slot(int Np, int nlf, int nv, int viscous) {
  return (viscous ? 2 : 1) * (nlf + 1) * Np * nv;
}

template <int NV, typename R>
__global__ void __launch_bounds__(kThreads) k_finalize(const DevPlan P, const StatePtrs S, const ElemLaunch L,
                                                      const FinalizeArgs A) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ ElemFaces faces[kMaxGroups];
  const int b = launch_block(L);
  const BlockDev& B = P.blk[b];
  const int W = L.W[b], g = threadIdx.x / W, lane = threadIdx.x % W;
  const int e = (blockIdx.x - L.cta0[b]) * (kThreads / W) + g;
  const bool live = e < B.E;
  const int Np = B.Np, nlf = B.nlf;
  const bool visc = P.viscous;
  R* Fp = reinterpret_cast<R*>(dyn_smem + (size_t)g * L.slot[b]);   // [nlf][Np][NV]
  R* Ft = Fp + nlf * Np * NV;                                         // [Np][NV]
  R* Vp = Ft + Np * NV;                                               // viscous copies
  R* Vt = Vp + nlf * Np * NV;
  const size_t ee = live ? e : 0;
  if (live) load_faces(P, B, (int)ee, lane, faces[g]);
  __syncthreads();
  const ElemFaces& Fc = faces[g];
  if (live) {
    // face contributions: thread (face, node) sums the face's points, all variables at once
    for (int t = lane; t < nlf * Np; t += W) {
      const int lf = t / Np, i = t % Np, nq = Fc.nq[lf];
      const FaceDev& fd = P.face[Fc.ft[lf]];
      const double* Bt = B.trB[Fc.ft[lf]] + (size_t)Fc.code[lf] * nq * Np + i;
      const double* fi = fd.fluxI + ((size_t)Fc.f[lf] * 2 + Fc.side[lf]) * nq * NV;
      const R sgn = Fc.side[lf] == 0 ? (R)-1 : (R)1;
      R si[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) si[v] = (R)0;
      for (int q = 0; q < nq; ++q) {
        const R bt = (R)Bt[(size_t)q * Np];
#pragma unroll
        for (int v = 0; v < NV; ++v) si[v] += bt * (R)fi[q * NV + v];
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) Fp[t * NV + v] = sgn * si[v];
      if (visc) {
        const double* fv = fd.fluxV + (size_t)Fc.f[lf] * nq * NV;
        R sv[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) sv[v] = (R)0;
        for (int q = 0; q < nq; ++q) {
          const R bt = (R)Bt[(size_t)q * Np];
#pragma unroll
          for (int v = 0; v < NV; ++v) sv[v] += bt * (R)fv[q * NV + v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) Vp[t * NV + v] = -sgn * sv[v];
      }
    }
  }
  __syncthreads();
  const size_t base = ee * Np * NV;
  if (live) {
    for (int idx = lane; idx < Np * NV; idx += W) {
      R si = (R)B.Rinv[base + idx];
      for (int lf = 0; lf < nlf; ++lf) si += Fp[lf * Np * NV + idx];
      Ft[idx] = si;
      if (visc) {
        R sv = (R)B.Rvis[base + idx];
        for (int lf = 0; lf < nlf; ++lf) sv += Vp[lf * Np * NV + idx];
        Vt[idx] = sv;
      }
    }
  }
  __syncthreads();
  if (!live) return;
  const bool aff = B.affine != nullptr && B.affine[ee];
  const double* Mi = aff ? B.mref_inv : B.minv + ee * Np * Np;
  const R mscale = (R)(aff ? B.acoef[ee] : 1.0);
  for (int idx = lane; idx < Np * NV; idx += W) {
    const int i = idx / NV, v = idx % NV;
    const double* row = Mi + (size_t)i * Np;
    R ri = (R)0, rv = (R)0;
    for (int j = 0; j < Np; ++j) {
      const R m = (R)row[j];
      ri += m * Ft[j * NV + v];
      if (visc) rv += m * Vt[j * NV + v];
    }
    const double rid = (double)(mscale * ri), rvd = visc ? (double)(mscale * rv) : 0.0;
    if (!A.stage) {
      if (A.out_inv[b]) A.out_inv[b][base + idx] = rid;
      if (A.out_vis[b]) A.out_vis[b][base + idx] = rvd;
    } else {
      const double total = visc ? rid + rvd : rid;
      const double eul = S.b[b][base + idx] + A.dt * total;
      if (A.out_vis[b]) A.out_vis[b][base + idx] = rvd;
      if (A.euler[b]) A.euler[b][base + idx] = eul;
      A.dst[b][base + idx] = A.alpha * A.base[b][base + idx] + A.beta * eul;
    }
  }
}

}  // namespace dgb
