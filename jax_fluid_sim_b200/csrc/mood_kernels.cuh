// MOOD subcell finite-volume recompute (float64, any element type).
//
// Reference: hybrid/subcell.py:442-950 and hybrid/limiter.py:267-343.  The reference runs
// the subcell scheme on every element and selects with `where`; here only troubled
// elements (flags from k_troubled on the unlimited candidate) and the parent faces they
// touch do work:
//   k_mood_fv      troubled element: subcell means (projection), Green-Gauss gradients,
//                  constant/TVD/CWENO-Z face states with admissibility clamps, HLLC on the
//                  internal subfaces, internal residual per subcell (gather, no atomics).
//   k_mood_faces   each warp screens 32 parent faces, then works those with a troubled side
//                  one at a time (mood_face): lanes 0-15 the 16
//                  DG-FV coupling subfaces (FV mean on a troubled side, DG value at the
//                  subface centre otherwise), lanes 16-31 the DG face flux integrated with
//                  the face rule; stores subface fluxes and (new - old) face flux.
//   k_mood_update  troubled element: subface fluxes added in local-face order, FV update
//                  (+ projected viscous rhs), bound-limited reconstruction to DG; other
//                  elements: the candidate plus the conservative correction from active
//                  faces on which they are not troubled.
#pragma once
#include "dg_kernels.cuh"

namespace dgb {

constexpr int kSub = 16;   // boundary subfaces per parent face at 4 divisions

struct SubcellBlockDev {
  int S, NI, NB;
  const double* P;        // [E][S][Np] projection
  const double* R;        // [E][Np][S] reconstruction
  const double* vol;      // [E][S]
  const double* cen;      // [E][S][3]
  const double* in_n;     // [E][NI][3]
  const double* in_a;     // [E][NI]
  const double* bd_n;     // [E][NB][3]
  const double* bd_a;     // [E][NB]
  const int32_t* iown;    // [NI]
  const int32_t* inbr;    // [NI]
  const int32_t* csr_ptr; // [S+1]
  const int32_t* csr_face;// [2 NI]
  const double* bbasis;   // [NB][Np] basis at the boundary subface centres
  const int32_t* gather;  // [NB] subcell read for a subface
  const int32_t* scatter; // [NB] subcell written for a subface (-1: none)
  double* ubar;           // [E][S][NV] scratch
  double* rsub;           // [E][S][NV] scratch
};

struct SubcellFaceDev {
  const int32_t* osub;    // [F][16] owner boundary subfaces
  const int32_t* nsub;    // [F][16] neighbour boundary subfaces matched to the owner's
  double* fsub;           // [F][16][NV] subface fluxes (times area)
  double* dflux;          // [F][NV]     new - old integrated face flux
  uint8_t* active;        // [F]
};

struct MoodDev {
  SubcellBlockDev blk[DGB_MAX_BLOCKS];
  SubcellFaceDev face[2];
  int recon;              // 0 constant, 1 tvd, 2 weno
};

struct FlagPtrs {
  const uint8_t* f[DGB_MAX_BLOCKS];
};

// Admissibility clamps of reconstructed subcell traces (hybrid/subcell.py:645-663)
template <int NV>
__device__ __forceinline__ void clamp_state(double* U) {
  U[0] = fmax(U[0], 1.0e-14);
  const double ek = 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
  U[4] = fmax(U[4], ek + 1.0e-12);
#pragma unroll
  for (int v = 5; v < NV; ++v) U[v] = fmax(U[v], 0.0);
}

// --------------------------------------------------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(kThreads) k_mood_fv(const DevPlan P, const MoodDev M, const StatePtrs S, int b,
                                                     const FlagPtrs F) {
  const int e = blockIdx.x;
  if (!F.f[b][e]) return;
  extern __shared__ double smem[];
  const BlockDev& B = P.blk[b];
  const SubcellBlockDev& C = M.blk[b];
  const int Np = B.Np, Sn = C.S, NI = C.NI;
  double* U = smem;                     // [Np][NV]
  double* ub = U + Np * NV;             // [S][NV]
  double* g = ub + Sn * NV;             // [S][3][NV]
  double* fi = g + Sn * 3 * NV;         // [NI][NV]
  const double* Ug = S.b[b] + (size_t)e * Np * NV;
  for (int i = threadIdx.x; i < Np * NV; i += kThreads) U[i] = Ug[i];
  __syncthreads();
  const double* Pe = C.P + (size_t)e * Sn * Np;
  for (int idx = threadIdx.x; idx < Sn * NV; idx += kThreads) {
    const int s = idx / NV, v = idx % NV;
    double acc = 0.0;
    for (int i = 0; i < Np; ++i) acc += Pe[s * Np + i] * U[i * NV + v];
    ub[idx] = acc;
    C.ubar[(size_t)e * Sn * NV + idx] = acc;
  }
  __syncthreads();
  const double* nrm = C.in_n + (size_t)e * NI * 3;
  const double* ar = C.in_a + (size_t)e * NI;
  const double* vol = C.vol + (size_t)e * Sn;
  const double* cen = C.cen + (size_t)e * Sn * 3;
  if (M.recon != 0) {
    // Green-Gauss gradient per subcell: sum over its internal subfaces of 0.5 n A (U_nbr - U_own) / V
    for (int idx = threadIdx.x; idx < Sn * 3 * NV; idx += kThreads) {
      const int s = idx / (3 * NV), d = (idx / NV) % 3, v = idx % NV;
      double acc = 0.0;
      for (int k = C.csr_ptr[s]; k < C.csr_ptr[s + 1]; ++k) {
        const int f = C.csr_face[k];
        acc += (0.5 * nrm[f * 3 + d] * ar[f]) * (ub[C.inbr[f] * NV + v] - ub[C.iown[f] * NV + v]);
      }
      g[idx] = acc / fmax(vol[s], 1.0e-14);
    }
    __syncthreads();
  }
  for (int f = threadIdx.x; f < NI; f += kThreads) {
    const int o = C.iown[f], n = C.inbr[f];
    double UL[NV], UR[NV], Fl[NV];
    if (M.recon == 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        UL[v] = ub[o * NV + v];
        UR[v] = ub[n * NV + v];
      }
    } else {
      double dc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) dc[d] = cen[n * 3 + d] - cen[o * 3 + d];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double dU = ub[n * NV + v] - ub[o * NV + v];
        double duo = 0.0, dun = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          duo += g[(o * 3 + d) * NV + v] * dc[d];
          dun -= g[(n * 3 + d) * NV + v] * dc[d];
        }
        if (M.recon == 1) {
          // smooth Venkatakrishnan-type TVD limiter (subcell.py:578-606)
          const double eps = 1.0e-12;
          const double ro = dU / (duo + (duo >= 0.0 ? eps : -eps));
          const double rn = (-dU) / (dun + (dun >= 0.0 ? eps : -eps));
          const double po = ro > 0.0 ? (ro * ro + 2.0 * ro) / (ro * ro + ro + 2.0) : 0.0;
          const double pn = rn > 0.0 ? (rn * rn + 2.0 * rn) / (rn * rn + rn + 2.0) : 0.0;
          UL[v] = ub[o * NV + v] + 0.5 * fmin(fmax(po, 0.0), 1.0) * duo;
          UR[v] = ub[n * NV + v] + 0.5 * fmin(fmax(pn, 0.0), 1.0) * dun;
        } else {
          // CWENO-Z (subcell.py:608-641)
          const double so = duo, sn = -dun;
          const double ph = 0.5 * (ub[o * NV + v] + ub[n * NV + v]) + 0.125 * (so - sn);
          const double po = ub[o * NV + v] + 0.5 * so, pn = ub[n * NV + v] - 0.5 * sn;
          const double es = 1.0e-12;
          const double bh = (sn - so) * (sn - so) + 0.1 * dU * dU;
          const double bo = (dU - so) * (dU - so) + 0.1 * dU * dU;
          const double bn = (dU - sn) * (dU - sn) + 0.1 * dU * dU;
          const double bc = dU * dU;
          const double tau = fabs(bc - bh);
          const double th = tau / (bh + es), to = tau / (bo + es), tn = tau / (bn + es), tc = tau / (bc + es);
          const double a0 = 0.70 * (1.0 + th * th), a1 = 0.28 * (1.0 + to * to), a2 = 0.02 * (1.0 + tc * tc);
          const double sl = a0 + a1 + a2;
          UL[v] = (a0 / sl) * ph + (a1 / sl) * po + (a2 / sl) * ub[o * NV + v];
          const double a1r = 0.28 * (1.0 + tn * tn);
          const double sr = a0 + a1r + a2;
          UR[v] = (a0 / sr) * ph + (a1r / sr) * pn + (a2 / sr) * ub[n * NV + v];
        }
      }
      clamp_state<NV>(UL);
      clamp_state<NV>(UR);
    }
    hllc<NV>(P.ph, UL, UR, nrm + f * 3, Fl);
#pragma unroll
    for (int v = 0; v < NV; ++v) fi[f * NV + v] = Fl[v] * ar[f];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < Sn * NV; idx += kThreads) {
    const int s = idx / NV, v = idx % NV;
    double acc = 0.0;
    for (int k = C.csr_ptr[s]; k < C.csr_ptr[s + 1]; ++k) {
      const int f = C.csr_face[k];
      acc += C.iown[f] == s ? -fi[f * NV + v] : fi[f * NV + v];
    }
    C.rsub[(size_t)e * Sn * NV + idx] = acc;
  }
}

// --------------------------------------------------------------------------------------------
template <int NV>
__device__ void dg_at_subface(const double* Ue, const double* basis_row, int Np, double* out) {
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = 0.0;
  for (int i = 0; i < Np; ++i) {
    const double bi = basis_row[i];
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] += bi * Ue[i * NV + v];
  }
}

// One parent face with a troubled side, worked by a whole warp (lane: see k_mood_faces).
template <int NV>
__device__ __forceinline__ void mood_face(const DevPlan& P, const MoodDev& M, const StatePtrs& S, int ft, int f,
                                          const FlagPtrs& Fl, int lane) {
  const FaceDev& fd = P.face[ft];
  const SubcellFaceDev& sf = M.face[ft];
  const int ob = fd.ob[f], ol = fd.ol[f], nb = fd.nb[f], nl = fd.nl[f];
  const bool tro = Fl.f[ob][ol] != 0;
  const bool trn = nb >= 0 && Fl.f[nb][nl] != 0;
  double Fv[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) Fv[v] = 0.0;
  if (lane < kSub) {
    const SubcellBlockDev& Co = M.blk[ob];
    const BlockDev& Bo = P.blk[ob];
    const int os = sf.osub[f * kSub + lane];
    double UL[NV], UR[NV];
    if (tro) {
      const double* ub = Co.ubar + ((size_t)ol * Co.S + Co.gather[os]) * NV;
#pragma unroll
      for (int v = 0; v < NV; ++v) UL[v] = ub[v];
    } else {
      dg_at_subface<NV>(S.b[ob] + (size_t)ol * Bo.Np * NV, Co.bbasis + (size_t)os * Bo.Np, Bo.Np, UL);
    }
    const double* n = Co.bd_n + ((size_t)ol * Co.NB + os) * 3;
    const double A = Co.bd_a[(size_t)ol * Co.NB + os];
    if (nb >= 0) {
      const SubcellBlockDev& Cn = M.blk[nb];
      const BlockDev& Bn = P.blk[nb];
      const int ns = sf.nsub[f * kSub + lane];
      if (trn) {
        const double* ub = Cn.ubar + ((size_t)nl * Cn.S + Cn.gather[ns]) * NV;
#pragma unroll
        for (int v = 0; v < NV; ++v) UR[v] = ub[v];
      } else {
        dg_at_subface<NV>(S.b[nb] + (size_t)nl * Bn.Np * NV, Cn.bbasis + (size_t)ns * Bn.Np, Bn.Np, UR);
      }
    } else if (P.ph.has_boundary) {
      ghost_state<NV>(P.ph, case_view(P.ph, P.blk[ob].ecase, ol).far, UL, n, fd.tag[f], UR);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) UR[v] = UL[v];
    }
    clamp_state<NV>(UL);
    clamp_state<NV>(UR);
    double H[NV];
    hllc<NV>(P.ph, UL, UR, n, H);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Fv[v] = H[v] * A;
      sf.fsub[((size_t)f * kSub + lane) * NV + v] = Fv[v];
    }
  } else {
    // DG face flux at the face rule points, integrated (hybrid/subcell.py:690-746); lanes
    // 16-31 stride over the face points.  It enters (new - old) with a minus sign.
    for (int q = lane - kSub; q < fd.nq; q += 32 - kSub) {
      const size_t so = ((size_t)f * 2 + 0) * fd.nq + q, sn = ((size_t)f * 2 + 1) * fd.nq + q;
      const double* n = fd.n + ((size_t)f * fd.nq + q) * 3;
      double UL[NV], UR[NV], H[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) UL[v] = fd.trA[so * NV + v];
      if (nb >= 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) UR[v] = fd.trA[sn * NV + v];
      } else if (P.ph.has_boundary) {
        ghost_state<NV>(P.ph, case_view(P.ph, P.blk[ob].ecase, ol).far, UL, n, fd.tag[f], UR);
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) UR[v] = UL[v];
      }
      clamp_state<NV>(UL);
      clamp_state<NV>(UR);
      hllc<NV>(P.ph, UL, UR, n, H);
      const double w = fd.w[(size_t)f * fd.nq + q];
#pragma unroll
      for (int v = 0; v < NV; ++v) Fv[v] -= H[v] * w;
    }
  }
  // warp sum: lanes 0-15 contribute new subface fluxes, lanes 16.. minus the old flux
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double x = Fv[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffff, x, o);
    if (lane == 0) sf.dflux[(size_t)f * NV + v] = x;
  }
}

// Each warp screens 32 parent faces (one per lane) for a troubled side, records which are active,
// then works its active faces one after another with the whole warp.
template <int NV>
__global__ void __launch_bounds__(kThreads) k_mood_faces(const DevPlan P, const MoodDev M, const StatePtrs S, int ft,
                                                        const FlagPtrs Fl) {
  const FaceDev& fd = P.face[ft];
  const SubcellFaceDev& sf = M.face[ft];
  const int lane = threadIdx.x & 31;
  const long f0 = ((long)blockIdx.x * kThreads + threadIdx.x) & ~31L;
  if (f0 >= fd.F) return;                       // whole warps leave together
  const long f = f0 + lane;
  bool active = false;
  if (f < fd.F) {
    const int ob = fd.ob[f], ol = fd.ol[f], nb = fd.nb[f], nl = fd.nl[f];
    active = Fl.f[ob][ol] != 0 || (nb >= 0 && Fl.f[nb][nl] != 0);
    sf.active[f] = active;
  }
  unsigned todo = __ballot_sync(0xffffffffu, active);
  while (todo) {
    const int k = __ffs(todo) - 1;
    todo &= todo - 1;
    mood_face<NV>(P, M, S, ft, (int)(f0 + k), Fl, lane);
  }
}

// --------------------------------------------------------------------------------------------
// out = troubled ? bound-limited reconstruction of the FV update : candidate + corrections.  out may
// be cand (in place): a troubled element's update does not read its candidate.
template <int NV>
__global__ void __launch_bounds__(kThreads) k_mood_update(const DevPlan P, const MoodDev M, int b, const FlagPtrs Fl,
                                                         const double* cand, const double* visc, double dt,
                                                         double* out) {
  extern __shared__ double smem[];
  const BlockDev& B = P.blk[b];
  const SubcellBlockDev& C = M.blk[b];
  const int e = blockIdx.x, Np = B.Np, Sn = C.S;
  const size_t base = (size_t)e * Np * NV;
  const double* vol = C.vol + (size_t)e * Sn;
  __shared__ double vtot;
  if (!Fl.f[b][e]) {
    // conservative correction from active faces where this element is not troubled; the element
    // volume is summed only when one is
    __shared__ double corr[DGB_MAX_VARS];
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (threadIdx.x < B.nlf) {
      int ft, f, side;
      decode_face(B.elem_face[e * B.nlf + threadIdx.x], ft, f, side);
      if (M.face[ft].active[f]) atomicOr(&any, 1);
    }
    __syncthreads();
    if (out == cand && !any) return;     // in place: an element without corrections keeps its candidate
    if (any && threadIdx.x == 0) {
      double s = 0.0;
      for (int k = 0; k < Sn; ++k) s += vol[k];
      vtot = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
      double c = 0.0;
      for (int lf = 0; lf < B.nlf; ++lf) {
        int ft, f, side;
        decode_face(B.elem_face[e * B.nlf + lf], ft, f, side);
        if (!M.face[ft].active[f]) continue;
        const double d = M.face[ft].dflux[(size_t)f * NV + threadIdx.x];
        c += side == 0 ? -dt * d / vtot : dt * d / vtot;
      }
      corr[threadIdx.x] = c;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < Np * NV; idx += kThreads)
      out[base + idx] = any ? cand[base + idx] + corr[idx % NV] : cand[base + idx];
    return;
  }
  double* res = smem;                    // [S][NV]
  double* fv = res + Sn * NV;            // [S][NV]
  double* raw = fv + Sn * NV;            // [Np][NV]
  for (int idx = threadIdx.x; idx < Sn * NV; idx += kThreads) res[idx] = C.rsub[(size_t)e * Sn * NV + idx];
  for (int lf = 0; lf < B.nlf; ++lf) {
    int ft, f, side;
    decode_face(B.elem_face[e * B.nlf + lf], ft, f, side);
    const SubcellFaceDev& sf = M.face[ft];
    const int32_t* sub = side == 0 ? sf.osub : sf.nsub;
    __syncthreads();
    for (int idx = threadIdx.x; idx < kSub * NV; idx += kThreads) {
      const int j = idx / NV, v = idx % NV;
      const int sc = C.scatter[sub[f * kSub + j]];
      if (sc < 0) continue;
      const double h = sf.fsub[((size_t)f * kSub + j) * NV + v];
      res[sc * NV + v] += side == 0 ? -h : h;
    }
  }
  __syncthreads();
  const double* Pe = C.P + (size_t)e * Sn * Np;
  for (int idx = threadIdx.x; idx < Sn * NV; idx += kThreads) {
    const int s = idx / NV, v = idx % NV;
    double x = C.ubar[(size_t)e * Sn * NV + idx] + dt * res[idx] / vol[s];
    if (visc) {
      double pv = 0.0;
      for (int i = 0; i < Np; ++i) pv += Pe[s * Np + i] * visc[base + i * NV + v];
      x += dt * pv;
    }
    fv[idx] = x;
  }
  __syncthreads();
  const double* Re = C.R + (size_t)e * Np * Sn;
  for (int idx = threadIdx.x; idx < Np * NV; idx += kThreads) {
    const int i = idx / NV, v = idx % NV;
    double acc = 0.0;
    for (int s = 0; s < Sn; ++s) acc += Re[i * Sn + s] * fv[s * NV + v];
    raw[idx] = acc;
  }
  __syncthreads();
  // Zhang-Shu bound limiting per variable (hybrid/subcell.py:406-439)
  if (threadIdx.x < NV) {
    const int v = threadIdx.x;
    double ms = 0.0, vs = 0.0, smin = INFINITY, smax = -INFINITY, dmin = INFINITY, dmax = -INFINITY;
    for (int s = 0; s < Sn; ++s) {
      ms += fv[s * NV + v] * vol[s];
      vs += vol[s];
      smin = fmin(smin, fv[s * NV + v]);
      smax = fmax(smax, fv[s * NV + v]);
    }
    const double mean = ms / fmax(vs, 1.0e-14);
    for (int i = 0; i < Np; ++i) {
      dmin = fmin(dmin, raw[i * NV + v]);
      dmax = fmax(dmax, raw[i * NV + v]);
    }
    const double eps = 1.0e-12;
    const double tmax = dmax > mean + eps ? (smax - mean) / (dmax - mean + eps) : 1.0;
    const double tmin = dmin < mean - eps ? (mean - smin) / (mean - dmin + eps) : 1.0;
    const double th = fmin(fmax(fmin(tmax, tmin), 0.0), 1.0);
    for (int i = 0; i < Np; ++i) out[base + i * NV + v] = mean + th * (raw[i * NV + v] - mean);
  }
}

__global__ void k_blend(const double* base, const double* x, double alpha, double beta, double* out, size_t n) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = alpha * base[i] + beta * x[i];
}

}  // namespace dgb
