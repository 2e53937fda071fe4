// Fused right-hand side of the sum-factorised hexahedron path: three launches per evaluation
// instead of six.
//
//   k_hex_traces   (hex_kernels.cuh, unchanged): face traces of U, of the viscous variables and of
//                  their raw gradients, per face side.
//   k_hex_face     one thread per face point, the points of a face in consecutive threads:
//                  HLLC (or the boundary ghost) minus each side's anchor flux, the BR2 jump,
//                  then each side's local lift at the face points, r_f = M^-1[slab_f] B_f^T jump
//                  seen through B_f (hybrid/navier_stokes.py:138-188), and the averaged viscous
//                  normal flux (hybrid/navier_stokes.py:210-324).  The local lift is a fixed linear
//                  map of the face's jumps: for an affine element br2 coef m1i[end][end] (K (x) K)
//                  with K = bf m1i bf^T, otherwise a QF^2 x QF^2 operator per element face built
//                  once from M^-1 (k_hex_lop).  This replaces k_face_flux, the per-face part of
//                  k_hex_lift and k_face_visc, and the traces are read once.
//   k_hex_element  one CTA per element: the nodal lift M^-1 sum_f B_f^T jump_f, the volume terms
//                  (U, grad v and lift at the volume points; inviscid and viscous fluxes), the face
//                  terms and M^-1 with the stage update.  The lift and the residuals stay in shared
//                  memory (no nodal-lift or residual buffers in HBM); M^-1 is read by the lift and
//                  by the final product.
// Arithmetic and summation order inside each phase are those of the unfused kernels; the local
// lift is summed as one operator instead of three factors, which moves results by round-off.
#pragma once
#include "hex_kernels.cuh"
#include "mlp_kernels.cuh"

namespace dgb {

// Local face of each face side of the hexahedron block: face_lf[f * 2 + side] (set-up).
__global__ void k_hex_face_lf(const DevPlan P_, int8_t* face_lf) {
  const BlockDev& B = P_.blk[0];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B.E * 6) return;
  int ft, f, side;
  decode_face(B.elem_face[t], ft, f, side);
  face_lf[(size_t)f * 2 + side] = (int8_t)(t % 6);
}

// Local-lift operator of every face of the non-affine elements (set-up), in the canonical face-point
// order of that face: L[c][c'] = sum_{i,j in slab} BF[c][i] M^-1[node i][node j] BF[c'][j], BF the
// face interpolation bf (x) bf.  One CTA per (listed element, local face).  Mt is M^-1 transposed
// in element node order (the hexahedron path's layout).
template <int P, typename T>
__global__ void k_hex_lop(const DevPlan P_, const HexTables tables, const int* __restrict__ elems, int count,
                          T* __restrict__ lop) {
  using D = HexDims<P>;
  constexpr int N = D::N, QF = D::QF, N2 = D::N2, N3 = D::N3, QF2 = D::QF2;
  __shared__ double ms[N2][N2];
  __shared__ double t1[N2][QF2];     // Mslab BF^T
  const int item = blockIdx.x;
  if (item >= count * 6) return;
  const int e = elems[item / 6], lf = item % 6;
  int a0, end, a1, a2;
  hex_face_axes(lf, a0, end, a1, a2);
  const int st0 = axis_stride<N>(a0), st1 = axis_stride<N>(a1), st2 = axis_stride<N>(a2);
  const double* Mt = P_.blk[0].minv + (size_t)e * N3 * N3;
  for (int idx = threadIdx.x; idx < N2 * N2; idx += blockDim.x) {
    const int si = idx / N2, sj = idx % N2;
    const int ni = tables.lex2node[end * st0 + (si % N) * st1 + (si / N) * st2];
    const int nj = tables.lex2node[end * st0 + (sj % N) * st1 + (sj / N) * st2];
    ms[si][sj] = Mt[(size_t)nj * N3 + ni];
  }
  __syncthreads();
  // BF[c][s] = bf[c % QF][s % N] bf[c / QF][s / N] (canonical face point c, slab node s)
  for (int idx = threadIdx.x; idx < N2 * QF2; idx += blockDim.x) {
    const int si = idx / QF2, c = idx % QF2;
    double acc = 0.0;
    for (int sj = 0; sj < N2; ++sj)
      acc += ms[si][sj] * tables.bf[(c % QF) * N + sj % N] * tables.bf[(c / QF) * N + sj / N];
    t1[si][c] = acc;
  }
  __syncthreads();
  T* out = lop + ((size_t)(item / 6) * 6 + lf) * QF2 * QF2;
  for (int idx = threadIdx.x; idx < QF2 * QF2; idx += blockDim.x) {
    const int c = idx / QF2, cp = idx % QF2;
    double acc = 0.0;
    for (int si = 0; si < N2; ++si)
      acc += tables.bf[(c % QF) * N + si % N] * tables.bf[(c / QF) * N + si / N] * t1[si][cp];
    out[idx] = (T)acc;
  }
}

// Inputs of the fused face kernel beyond the plan: the local face of each face side, the lift
// operators of the non-affine elements (lop_index[e] >= 0 selects one) and its precision.
struct HexFaceArgs {
  const int8_t* face_lf;      // [F][2]
  const int* lop_index;       // [E], -1 for affine elements
  const double* lop;          // [count][6][QF2][QF2], float64 plans
  const float* lop32;         // the same in float32, mixed-precision plans
};

// R: arithmetic of the local lifts and the viscous face flux (float in precision mode 1; HLLC and
// the jumps are float64 in both modes).  F32: the viscous traces come from trV32 / trG32.
template <int P, int NV, typename R = double, bool F32 = false>
__global__ void __launch_bounds__(kThreads, NV <= 5 ? 6 : 1) k_hex_face(const DevPlan P_, const HexTables tables,
                                                                       const HexCodes codes, const HexFaceArgs A) {
  using D = HexDims<P>;
  constexpr int N = D::N, QF = D::QF, QF2 = D::QF2;
  constexpr int FPC = kThreads / QF2;                // faces per CTA
  constexpr bool RF = sizeof(R) == sizeof(float);    // float32 face fluxes and jumps (mixed precision)
  // jumps of each face's points, [face][point][12]; the face stride is padded to a 16-byte
  // multiple (two doubles or four floats) so that a point's 12 jumps are read by 16-byte loads
  constexpr int JS = QF2 * 12 + (sizeof(R) == sizeof(float) ? 4 : 2);
  __shared__ __align__(16) R jmp[FPC * JS];
  __shared__ R K[QF][QF];                            // bf m1i bf^T
  const FaceDev& fd = P_.face[1];
  const int slot = threadIdx.x / QF2, q = threadIdx.x % QF2;
  const int f = blockIdx.x * FPC + slot;
  const bool live = slot < FPC && f < fd.F;
  if (threadIdx.x < QF * QF) {
    const int a = threadIdx.x / QF, c = threadIdx.x % QF;
    double acc = 0.0;
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) acc += tables.bf[a * N + j] * tables.m1i[j * N + k] * tables.bf[c * N + k];
    K[a][c] = (R)acc;
  }
  int nb = -1;
  double n[3] = {0.0, 0.0, 0.0}, w = 0.0;
  size_t so = 0, sn = 0;
  double UL[NV];
  if (live) {
    nb = fd.nb[f];
    const double* np_ = fd.n + ((size_t)f * QF2 + q) * 3;
    n[0] = np_[0], n[1] = np_[1], n[2] = np_[2];
    w = fd.w[(size_t)f * QF2 + q];
    so = ((size_t)f * 2 + 0) * QF2 + q;
    sn = ((size_t)f * 2 + 1) * QF2 + q;
    double UR[NV], Fh[NV], Fa[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) UL[v] = fd.trA[so * NV + v];
    if (nb >= 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) UR[v] = fd.trA[sn * NV + v];
    } else if (P_.ph.has_boundary) {
      ghost_state<NV>(P_.ph, case_view(P_.ph, P_.blk[0].ecase, fd.ol[f]).far, UL, n, fd.tag[f], UR);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) UR[v] = UL[v];
    }
    hllc<NV>(P_.ph, UL, UR, n, Fh);
    {
      double a[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) a[v] = fd.anc[((size_t)f * 2 + 0) * NV + v];
      normal_flux<NV>(P_.ph, a, n, Fa);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if (RF) fd.fluxI32[so * NV + v] = (float)((Fh[v] - Fa[v]) * w);
        else fd.fluxI[so * NV + v] = (Fh[v] - Fa[v]) * w;
      }
    }
    if (nb >= 0) {
      double a[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) a[v] = fd.anc[((size_t)f * 2 + 1) * NV + v];
      normal_flux<NV>(P_.ph, a, n, Fa);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if (RF) fd.fluxI32[sn * NV + v] = (float)((Fh[v] - Fa[v]) * w);
        else fd.fluxI[sn * NV + v] = (Fh[v] - Fa[v]) * w;
      }
    }
  }
  if (!P_.viscous) return;
  double vo[4], vn[4];
  // a face point's 4 viscous values: one 16-byte load (float32) or two (float64)
  auto load_v = [&](size_t pt, double* out) {
    if constexpr (F32) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(fd.trV32 + pt * 4));
      out[0] = t.x, out[1] = t.y, out[2] = t.z, out[3] = t.w;
    } else {
      const double2* t = reinterpret_cast<const double2*>(fd.trV + pt * 4);
      const double2 a = t[0], b2 = t[1];
      out[0] = a.x, out[1] = a.y, out[2] = b2.x, out[3] = b2.y;
    }
  };
  if (live) {
    load_v(so, vo);
    if (nb >= 0) {
      load_v(sn, vn);
    } else if (P_.ph.has_boundary) {
      const CaseView cv = case_view(P_.ph, P_.blk[0].ecase, fd.ol[f]);
      viscous_ghost<NV>(P_.ph, cv.far, cv.wall_T, UL, n, fd.tag[f], vn);
    } else {
      viscous_vars<NV>(P_.ph, UL, vn);
    }
    const size_t jo = ((size_t)f * QF2 + q) * 12;
    // a point's 12 jumps are contiguous in the face buffer and in jmp: 16-byte stores
    R jr[12];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int d = 0; d < 3; ++d) jr[m * 3 + d] = (R)(0.5 * w * (vn[m] - vo[m]) * n[d]);
    R* js = &jmp[slot * JS + q * 12];
    if constexpr (RF) {
      float4* g4 = reinterpret_cast<float4*>(fd.jumpW32 + jo);
      float4* s4 = reinterpret_cast<float4*>(js);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 v = make_float4(jr[4 * k], jr[4 * k + 1], jr[4 * k + 2], jr[4 * k + 3]);
        g4[k] = v;
        s4[k] = v;
      }
    } else {
      double2* g2 = reinterpret_cast<double2*>(fd.jumpW + jo);
      double2* s2 = reinterpret_cast<double2*>(js);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double2 v = make_double2(jr[2 * k], jr[2 * k + 1]);
        g2[k] = v;
        s2[k] = v;
      }
    }
  }
  __syncthreads();
  if (!live) return;
  const BlockDev& B = P_.blk[0];
  const CaseView cv = case_view(P_.ph, B.ecase, fd.ol[f]);
  const R* jf = &jmp[slot * JS];
  R Fo[3 * NV];
  const int nsides = nb >= 0 ? 2 : 1;
  for (int s = 0; s < nsides; ++s) {
    const int e = s == 0 ? fd.ol[f] : fd.nl[f];
    const int code = s == 0 ? fd.oc[f] : fd.nc[f];
    const uint8_t* perm = codes.perm + (size_t)code * QF2;
    const int lf = A.face_lf[(size_t)f * 2 + s];
    const int cq = perm[q];
    // the side's face-point permutation in registers (one 16-byte load for P3 faces), so that the
    // operator loads of the lift loop do not wait on the permutation loads one by one
    unsigned wd[4] = {0u, 0u, 0u, 0u};
    if constexpr (QF2 == 16) {
      const uint4 raw = __ldg(reinterpret_cast<const uint4*>(perm));
      wd[0] = raw.x, wd[1] = raw.y, wd[2] = raw.z, wd[3] = raw.w;
    }
    auto pm = [&](int k) -> int {
      if constexpr (QF2 == 16) return (int)((wd[k / 4] >> (8 * (k % 4))) & 0xFFu);
      else return perm[k];
    };
    // the 12 jumps of face point qp (16-byte loads from the padded rows)
    auto jrow = [&](int qp, R* r) {
      if constexpr (sizeof(R) == sizeof(float)) {
        const float4* p4 = reinterpret_cast<const float4*>(jf + qp * 12);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float4 v = p4[k];
          r[4 * k] = v.x, r[4 * k + 1] = v.y, r[4 * k + 2] = v.z, r[4 * k + 3] = v.w;
        }
      } else {
        const double2* p2 = reinterpret_cast<const double2*>(jf + qp * 12);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          const double2 v = p2[k];
          r[2 * k] = v.x, r[2 * k + 1] = v.y;
        }
      }
    };
    R lift[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) lift[c] = R(0);
    const int li = A.lop_index ? A.lop_index[e] : -1;
    if (li < 0) {
      // affine: br2 coef m1i[end][end] (K (x) K) in this side's canonical order
      int a0, end, a1, a2;
      hex_face_axes(lf, a0, end, a1, a2);
      const R scale = (R)(P_.ph.br2 * B.acoef[e] * tables.m1i[end * N + end]);
      const int c1 = cq % QF, c2 = cq / QF;
#pragma unroll
      for (int qp = 0; qp < QF2; ++qp) {
        const int cp = pm(qp);
        const R kk = K[c1][cp % QF] * K[c2][cp / QF];
        R jv[12];
        jrow(qp, jv);
#pragma unroll
        for (int c = 0; c < 12; ++c) lift[c] += kk * jv[c];
      }
#pragma unroll
      for (int c = 0; c < 12; ++c) lift[c] *= scale;
    } else {
      const size_t lo = ((size_t)li * 6 + lf) * QF2 * QF2 + (size_t)cq * QF2;
#pragma unroll
      for (int qp = 0; qp < QF2; ++qp) {
        R kk;
        if constexpr (sizeof(R) == sizeof(float)) kk = __ldg(A.lop32 + lo + pm(qp));
        else kk = (R)__ldg(A.lop + lo + pm(qp));
        R jv[12];
        jrow(qp, jv);
#pragma unroll
        for (int c = 0; c < 12; ++c) lift[c] += kk * jv[c];
      }
#pragma unroll
      for (int c = 0; c < 12; ++c) lift[c] *= (R)P_.ph.br2;
    }
    const size_t ss = s == 0 ? so : sn;
    // the owner's lift at boundary faces stays in the face buffers for the wall-force integral
    // (dgb_wall_forces reads the viscous traction there)
    if (nb < 0)
#pragma unroll
      for (int c = 0; c < 12; ++c) fd.liftF[ss * 12 + c] = (double)lift[c];
    R U[NV], g[12];
#pragma unroll
    for (int v = 0; v < NV; ++v) U[v] = (R)fd.trP[ss * NV + v];
    // the point's 12 gradients: 16-byte loads
    if constexpr (F32) {
      const float4* t = reinterpret_cast<const float4*>(fd.trG32 + ss * 12);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 a = __ldg(t + k);
        g[4 * k] = (R)a.x, g[4 * k + 1] = (R)a.y, g[4 * k + 2] = (R)a.z, g[4 * k + 3] = (R)a.w;
      }
    } else {
      const double2* t = reinterpret_cast<const double2*>(fd.trG + ss * 12);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double2 a = t[k];
        g[2 * k] = (R)a.x, g[2 * k + 1] = (R)a.y;
      }
    }
#pragma unroll
    for (int c = 0; c < 12; ++c) g[c] += lift[c];
    if (s == 0) {
      viscous_flux<NV>(P_.ph, cv.mu, cv.kappa, U, g, Fo);
    } else {
      R Fn[3 * NV];
      viscous_flux<NV>(P_.ph, cv.mu, cv.kappa, U, g, Fn);
#pragma unroll
      for (int k = 0; k < 3 * NV; ++k) Fo[k] = R(0.5) * (Fo[k] + Fn[k]);
    }
  }
  R out[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v)
    out[v] = Fo[0 * NV + v] * (R)n[0] + Fo[1 * NV + v] * (R)n[1] + Fo[2 * NV + v] * (R)n[2];
  if (nb < 0 && P_.ph.has_boundary && tag_in(fd.tag[f], P_.ph.wall, P_.ph.n_wall)) out[4] = R(0);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    if (RF) fd.fluxV32[((size_t)f * QF2 + q) * NV + v] = (float)(out[v] * (R)w);
    else fd.fluxV[((size_t)f * QF2 + q) * NV + v] = (double)(out[v] * (R)w);
  }
}

// Rotation of the thread <-> line assignment of a pencil pass, so that passes issued back to back
// without a barrier between them start on different threads.
__device__ __forceinline__ int rotated(int offset) {
  return (int)((threadIdx.x + kThreads - (unsigned)offset % kThreads) % kThreads);
}

// K consecutive shared-memory values at p (16-byte aligned) into r: 16-byte loads, then an 8-byte
// load of a float pair, then single values.
template <int K, typename T>
__device__ __forceinline__ void lds_vec(const T* p, T* r) {
  constexpr int VA = 16 / sizeof(T), K16 = K / VA * VA;
#pragma unroll
  for (int k = 0; k < K16; k += VA) load16(p + k, r + k);
  constexpr int K8 = (sizeof(T) == sizeof(float) && K - K16 >= 2) ? K16 + 2 : K16;
  if constexpr (K8 > K16) {
    const float2 v = *reinterpret_cast<const float2*>(p + K16);
    r[K16] = v.x;
    r[K16 + 1] = v.y;
  }
#pragma unroll
  for (int k = K8; k < K; ++k) r[k] = p[k];
}

// The three reference-gradient fields of C nodal channels at the Q^3 volume points,
// g[r][c][Q3] = (d/dxi_r of the interpolant), by the sum-factorised passes with the intermediates
// shared between directions: x (bq, dq), y (bq, dq on the bq branch; bq on the dq branch), z.  Each
// output goes through the same three 1-D products as a separate tensor3 per direction, so the values
// are the same; the barriers are three instead of nine.  s: 2 C N^2 Q + 3 C N Q^2 values of scratch.
template <int C, int N, int Q, typename T>
__device__ __forceinline__ void grad3(const T* V, T* g, T* s, const T* bq, const T* dq) {
  T* Bx = s;
  T* Dx = Bx + C * N * N * Q;
  T* BB = Dx + C * N * N * Q;
  T* BD = BB + C * N * Q * Q;
  T* DB = BD + C * N * Q * Q;
  constexpr int L1 = C * N * N, L2 = C * N * Q, L3 = C * Q * Q, Q3 = Q * Q * Q;
  const int st = kThreads;
  auto i1 = [](int l) { return l * N; };
  auto o1 = [](int l) { return l * Q; };
  pencil<N, Q, false>(V, Bx, bq, L1, 1, 1, i1, o1, rotated(0), st);
  pencil<N, Q, false>(V, Dx, dq, L1, 1, 1, i1, o1, rotated(L1), st);
  __syncthreads();
  auto i2 = [](int l) { return (l / Q) * N * Q + l % Q; };
  auto o2 = [](int l) { return (l / Q) * Q * Q + l % Q; };
  pencil<N, Q, false>(Bx, BB, bq, L2, Q, Q, i2, o2, rotated(0), st);
  pencil<N, Q, false>(Bx, BD, dq, L2, Q, Q, i2, o2, rotated(L2), st);
  pencil<N, Q, false>(Dx, DB, bq, L2, Q, Q, i2, o2, rotated(2 * L2), st);
  __syncthreads();
  auto i3 = [](int l) { return (l / (Q * Q)) * N * Q * Q + l % (Q * Q); };
  auto o3 = [](int l) { return (l / (Q * Q)) * Q * Q * Q + l % (Q * Q); };
  pencil<N, Q, false>(DB, g + 0 * C * Q3, bq, L3, Q * Q, Q * Q, i3, o3, rotated(0), st);
  pencil<N, Q, false>(BD, g + 1 * C * Q3, bq, L3, Q * Q, Q * Q, i3, o3, rotated(L3), st);
  pencil<N, Q, false>(BB, g + 2 * C * Q3, dq, L3, Q * Q, Q * Q, i3, o3, rotated(2 * L3), st);
  __syncthreads();
}

// The weak divergence R[c][N3] = sum_r (transposed gradient of direction r) G[r][c][Q3], by three
// passes (x, y with three inputs each, then z summing the three terms in the order of three
// accumulating tensor3 calls: (t0 + t1) + t2), so the values match that form with three barriers
// instead of nine.  A: 3 C Q^2 N values of scratch; the y-pass results overwrite G.
template <int C, int N, int Q, typename T>
__device__ __forceinline__ void div3(T* G, T* R, T* A, const T* bqT, const T* dqT) {
  constexpr int Q3 = Q * Q * Q, LX = C * Q * Q, LY = C * Q * N, LZ = C * N * N;
  constexpr int AS = C * Q * Q * N, BS = C * Q * N * N;
  const int st = kThreads;
  auto ix = [](int l) { return l * Q; };
  auto ox = [](int l) { return l * N; };
  pencil<Q, N, false>(G + 0 * C * Q3, A + 0 * AS, dqT, LX, 1, 1, ix, ox, rotated(0), st);
  pencil<Q, N, false>(G + 1 * C * Q3, A + 1 * AS, bqT, LX, 1, 1, ix, ox, rotated(LX), st);
  pencil<Q, N, false>(G + 2 * C * Q3, A + 2 * AS, bqT, LX, 1, 1, ix, ox, rotated(2 * LX), st);
  __syncthreads();
  T* B = G;                                    // [3][C][Q][N][N]
  auto iy = [](int l) { return (l / N) * Q * N + l % N; };
  auto oy = [](int l) { return (l / N) * N * N + l % N; };
  pencil<Q, N, false>(A + 0 * AS, B + 0 * BS, bqT, LY, N, N, iy, oy, rotated(0), st);
  pencil<Q, N, false>(A + 1 * AS, B + 1 * BS, dqT, LY, N, N, iy, oy, rotated(LY), st);
  pencil<Q, N, false>(A + 2 * AS, B + 2 * BS, bqT, LY, N, N, iy, oy, rotated(2 * LY), st);
  __syncthreads();
  const T* mb = bqT;                           // read from shared memory (broadcast)
  const T* md = dqT;
  for (int line = threadIdx.x; line < LZ; line += st) {
    const int ib = (line / (N * N)) * Q * N * N + line % (N * N);
    const int ob = (line / (N * N)) * N * N * N + line % (N * N);
    T x0[Q], x1[Q], x2[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      x0[i] = B[0 * BS + ib + i * N * N];
      x1[i] = B[1 * BS + ib + i * N * N];
      x2[i] = B[2 * BS + ib + i * N * N];
    }
#pragma unroll
    for (int o = 0; o < N; ++o) {
      T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
      for (int i = 0; i < Q; ++i) s0 += mb[o * Q + i] * x0[i];
#pragma unroll
      for (int i = 0; i < Q; ++i) s1 += mb[o * Q + i] * x1[i];
#pragma unroll
      for (int i = 0; i < Q; ++i) s2 += md[o * Q + i] * x2[i];
      T acc = s0;
      acc += s1;
      acc += s2;
      R[ob + o * N * N] = acc;
    }
  }
  __syncthreads();
}

// Shared-memory layout of k_hex_element, in units of R.
template <int P, int NV, bool SPLIT, typename R>
struct HexElemSmem {
  using D = HexDims<P>;
  static constexpr int N = D::N, Q = D::Q, QF = D::QF, N2 = D::N2, N3 = D::N3, Q3 = D::Q3, QF2 = D::QF2;
  // table size in R, rounded up to 16 bytes so that the arrays after the tables stay 16-byte aligned
  static constexpr int T = (int)((sizeof(HexTablesT<R>) + 15) / 16 * 16 / sizeof(R));
  static constexpr int C = SPLIT ? 2 * NV : NV;          // residual channels
  static constexpr int U = T, V = U + NV * N3, LF = V + 4 * N3, RR = LF + 12 * N3;
  // the phase scratch starts on a 16-byte boundary (N3 = 27 leaves RR + C N3 odd)
  static constexpr int W = (RR + C * N3 + 3) / 4 * 4;
  // phase scratch (aliased)
  // jc, tmp, bs, ball, then the affine elements' tensor3 scratch (two [12][N3] passes)
  static constexpr int LIFT = 72 * QF2 + 72 * QF * N + 72 * N2 + 12 * N3 + 2 * 12 * N3;
  // phase C: uq [NV][Q3], gq [12][Q3], then the lift at the points lq [12][Q3] (later Gi, Gv [3][NV][Q3]
  // each), then contraction scratch
  static constexpr int VOL_G = cmax(12 * Q3, (SPLIT ? 6 : 3) * NV * Q3);
  static constexpr int VOL_S = cmax(cmax(NV * N * N * Q + NV * N * Q * Q, 12 * N * N * Q + 12 * N * Q * Q),
                                    2 * 4 * N * N * Q + 3 * 4 * N * Q * Q);
  // the scratch lives beyond lq while Gi/Gv are not yet written; div3's x-pass results go to the
  // dead uq/gq region when they fit there, otherwise beyond Gi/Gv
  static constexpr int DIV_A = 3 * NV * Q * Q * N;
  static constexpr int DIV_AT = DIV_A <= NV * Q3 + 12 * Q3 ? 0 : NV * Q3 + 12 * Q3 + VOL_G;
  static constexpr int VOL2 = cmax(NV * Q3 + 12 * Q3 + cmax(VOL_G, 12 * Q3 + VOL_S), DIV_AT + DIV_A);
  static constexpr int FIN = 6 * C * (QF2 + QF * N) + cmax(6 * C * N2, 4 * NV * N3);
  static constexpr int TOTAL = W + cmax(LIFT, cmax(VOL2, FIN));
};

// Lift + volume + finalize of one hexahedron (see the file comment).  SPLIT keeps the inviscid
// and viscous residuals apart (right-hand-side outputs, the MOOD step's viscous residual).
template <int P, int NV, bool SPLIT, typename R = double>
__global__ void __launch_bounds__(kThreads, sizeof(R) == sizeof(float) ? 6 : 1) k_hex_element(const DevPlan P_, const StatePtrs S, const HexTables tables,
                                                         const HexCodes codes, const FinalizeArgs A) {
  using D = HexDims<P>;
  using L = HexElemSmem<P, NV, SPLIT, R>;
  constexpr int N = D::N, Q = D::Q, QF = D::QF, N2 = D::N2, N3 = D::N3, Q3 = D::Q3, QF2 = D::QF2;
  constexpr int C = L::C;
  constexpr int b = 0;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  R* smem = reinterpret_cast<R*>(dyn_smem);
  HexTablesT<R>* tb = reinterpret_cast<HexTablesT<R>*>(smem);
  R* U = smem + L::U;            // [NV][N3] minus anchor
  R* V = smem + L::V;            // [4][N3]
  R* Lf = smem + L::LF;          // [12][N3] nodal lift
  R* Rr = smem + L::RR;          // [C][N3] residuals (inviscid, then viscous)
  R* W = smem + L::W;
  __shared__ int node2lex[64], fslot[6], fperm[6], fface[6];
  __shared__ double anchor_d[NV];
  __shared__ R anchor[NV];
  const BlockDev& B = P_.blk[b];
  const FaceDev& fd = P_.face[1];
  const int e = blockIdx.x;
  if ((A.only && !A.only[e]) || (A.skip && A.skip[e])) return;     // uniform across the CTA
  const CaseView cv = case_view(P_.ph, B.ecase, e);
  load_tables<P>(tables, tb);
  const double* Ug = S.b[b] + (size_t)e * N3 * NV;
  if (threadIdx.x < NV) {
    anchor_d[threadIdx.x] = Ug[threadIdx.x];
    anchor[threadIdx.x] = (R)Ug[threadIdx.x];
  }
  if (threadIdx.x < 6) {
    int ft, f, side;
    decode_face(B.elem_face[e * 6 + threadIdx.x], ft, f, side);
    fslot[threadIdx.x] = (f * 2 + side) * QF2;
    fperm[threadIdx.x] = (side == 0 ? fd.oc[f] : fd.nc[f]) * QF2;
    fface[threadIdx.x] = (f << 1) | side;
  }
  __syncthreads();
  for (int l = threadIdx.x; l < N3; l += kThreads) node2lex[tb->lex2node[l]] = l;
  for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
    const int v = idx / N3, l = idx % N3;
    U[idx] = (R)(Ug[tb->lex2node[l] * NV + v] - anchor_d[v]);
  }
  const bool visc = P_.viscous;
  const bool aff = B.affine && B.affine[e];
  // a predicted troubled element: only its viscous residual is used (the subcell scheme replaces
  // its update), so the inviscid volume and face terms are not formed
  const bool skip_inv = SPLIT && A.skip_inviscid && A.skip_inviscid[e];
  const double* MT = B.minv + (size_t)e * N3 * N3;
  const float* MT32 = (sizeof(R) == sizeof(float) && B.minv32) ? B.minv32 + (size_t)e * N3 * N3 : nullptr;
  if (visc) {
    for (int l = threadIdx.x; l < N3; l += kThreads) {
      const int node = tb->lex2node[l];
      double u[NV], vv[4];
#pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = Ug[node * NV + v];
      viscous_vars<NV>(P_.ph, u, vv);
#pragma unroll
      for (int m = 0; m < 4; ++m) V[m * N3 + l] = (R)vv[m];
    }
    // ---- phase B: nodal lift M^-1 sum_f B_f^T jump_f
    constexpr int CH = 72;
    R* jc = W;                        // [6][12][QF2] jumps at the canonical face points
    R* tmp = jc + CH * QF2;           // [72][QF][N]
    R* bs = tmp + CH * QF * N;        // [6][12][N2]
    R* ball = bs + CH * N2;           // [12][N3]
    R* ax = ball + 12 * N3;           // affine scratch [2][12][N3]
    // dense-lift row groups of the non-affine elements: 6 channels padded to 16 bytes; the rows
    // (2 LR N3 values) reach into ax, which only affine elements use
    constexpr int LR = (6 * (int)sizeof(R) + 15) / 16 * 16 / (int)sizeof(R);
    static_assert(2 * LR <= 36, "the dense-lift rows must fit in ball and ax");
    // one face point per thread: its 12 jump components (contiguous) to the canonical point
    for (int it = threadIdx.x; it < 6 * QF2; it += kThreads) {
      const int lf = it / QF2, q = it % QF2;
      const int cp = codes.perm[fperm[lf] + q];
      const size_t jo = ((size_t)(fface[lf] >> 1) * QF2 + q) * 12;
      if constexpr (sizeof(R) == sizeof(float)) {
        const float4* src = reinterpret_cast<const float4*>(fd.jumpW32 + jo);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float4 v = src[k];
          jc[(lf * 12 + 4 * k) * QF2 + cp] = v.x;
          jc[(lf * 12 + 4 * k + 1) * QF2 + cp] = v.y;
          jc[(lf * 12 + 4 * k + 2) * QF2 + cp] = v.z;
          jc[(lf * 12 + 4 * k + 3) * QF2 + cp] = v.w;
        }
      } else {
        const double2* src = reinterpret_cast<const double2*>(fd.jumpW + jo);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          const double2 v = src[k];
          jc[(lf * 12 + 2 * k) * QF2 + cp] = (R)v.x;
          jc[(lf * 12 + 2 * k + 1) * QF2 + cp] = (R)v.y;
        }
      }
    }
    __syncthreads();
    tensor2<CH, QF, QF, N, N>(jc, bs, tmp, tb->bfT, tb->bfT);
    for (int idx = threadIdx.x; idx < 12 * N3; idx += kThreads) {
      const int c = idx / N3, l = idx % N3;
      const int xyz[3] = {l % N, (l / N) % N, l / N2};
      R acc = R(0);
#pragma unroll
      for (int lf = 0; lf < 6; ++lf) {
        int a0, end, a1, a2;
        hex_face_axes(lf, a0, end, a1, a2);
        if (xyz[a0] == end) acc += bs[(lf * 12 + c) * N2 + xyz[a2] * N + xyz[a1]];
      }
      // non-affine elements: rows of two 16-byte aligned groups of 6 channels (LR apart) in element
      // node order, for 16-byte loads in the dense M^-1 (summed in node order)
      ball[aff ? idx : tb->lex2node[l] * 2 * LR + (c / 6) * LR + c % 6] = acc;
    }
    __syncthreads();
    if (aff) {
      tensor3<12, N, N, N, N, N, N, false>(ball, Lf, ax, ax + 12 * N3, tb->m1i, tb->m1i, tb->m1i);
      const R cf = (R)B.acoef[e];
      for (int idx = threadIdx.x; idx < 12 * N3; idx += kThreads) Lf[idx] *= cf;
    } else {
      auto dense_lift = [&](const auto* M) {
        for (int idx = threadIdx.x; idx < 2 * N3; idx += kThreads) {
          const int i = idx % N3, g = idx / N3, c0 = g * 6;
          R sacc[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
#pragma unroll 4
          for (int j = 0; j < N3; ++j) {
            const R m = (R)__ldg(M + (size_t)j * N3 + i);
            R bj[6];
            lds_vec<6>(ball + j * 2 * LR + g * LR, bj);
#pragma unroll
            for (int k = 0; k < 6; ++k) sacc[k] += m * bj[k];
          }
          const int li = node2lex[i];
#pragma unroll
          for (int k = 0; k < 6; ++k) Lf[(c0 + k) * N3 + li] = sacc[k];
        }
      };
      if (MT32) dense_lift(MT32); else dense_lift(MT);
    }
  }
  __syncthreads();
  // ---- phase C: volume terms (k_hex_volume's arithmetic with the lift from shared memory; the
  // gradient and divergence contractions share their intermediate passes, grad3 / div3)
  {
    R* uq = W;                           // [NV][Q3]   U - anchor at volume points
    R* gq = uq + NV * Q3;                // [12][Q3]   gradients of v: reference (3 x 4), then physical + lift
    R* lq = gq + 12 * Q3;                // [12][Q3]   nodal lift at the points; Gi, Gv reuse this region
    R* sc = lq + 12 * Q3;                // contraction scratch (before Gi, Gv are written)
    tensor3<NV, N, N, N, Q, Q, Q, false>(U, uq, sc, sc + NV * N * N * Q, tb->bq, tb->bq, tb->bq);
    const double* jinv = B.jinv + (size_t)e * Q3 * 9;
    const float* jinv32 = (sizeof(R) == sizeof(float) && B.jinv32) ? B.jinv32 + (size_t)e * Q3 * 9 : nullptr;
    const double* wdet = B.wdet + (size_t)e * Q3;
    R Ja[9], deta = R(0);
    if (aff) {
#pragma unroll
      for (int k = 0; k < 9; ++k) Ja[k] = (R)B.ajinv[(size_t)e * 9 + k];
      deta = (R)B.adet[e];
    }
    if (visc) {
      tensor3<12, N, N, N, Q, Q, Q, false>(Lf, lq, sc, sc + 12 * N * N * Q, tb->bq, tb->bq, tb->bq);
      grad3<4, N, Q>(V, gq, sc, tb->bq, tb->dq);
      // reference -> physical gradient per point, plus the lift at the point
      for (int q = threadIdx.x; q < Q3; q += kThreads) {
        R J[9], gr[12];
#pragma unroll
        for (int k = 0; k < 9; ++k) J[k] = aff ? Ja[k] : (jinv32 ? (R)jinv32[q * 9 + k] : (R)jinv[q * 9 + k]);
#pragma unroll
        for (int k = 0; k < 12; ++k) gr[k] = gq[k * Q3 + q];
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            R x = gr[0 * 4 + m] * J[0 * 3 + d] + gr[1 * 4 + m] * J[1 * 3 + d] + gr[2 * 4 + m] * J[2 * 3 + d];
            x += lq[(m * 3 + d) * Q3 + q];
            gq[(m * 3 + d) * Q3 + q] = x;
          }
      }
      __syncthreads();
    }
    R* Gi = lq;                          // [3][NV][Q3]
    R* Gv = Gi + 3 * NV * Q3;            // [3][NV][Q3] (SPLIT only)
    R Fa[3][NV];
    {
      const R ex[3] = {R(1), R(0), R(0)}, ey[3] = {R(0), R(1), R(0)}, ez[3] = {R(0), R(0), R(1)};
      normal_flux<NV>(P_.ph, anchor, ex, Fa[0]);
      normal_flux<NV>(P_.ph, anchor, ey, Fa[1]);
      normal_flux<NV>(P_.ph, anchor, ez, Fa[2]);
    }
    for (int q = threadIdx.x; q < Q3; q += kThreads) {
      R J[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) J[k] = aff ? Ja[k] : (jinv32 ? (R)jinv32[q * 9 + k] : (R)jinv[q * 9 + k]);
      const R wq = aff ? tb->w1[q / (Q * Q)] * tb->w1[(q / Q) % Q] * tb->w1[q % Q] * deta : (R)wdet[q];
      R Uq[NV], F[3][NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) Uq[v] = anchor[v] + uq[v * Q3 + q];
      if (skip_inv) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int v = 0; v < NV; ++v) F[d][v] = Fa[d][v];
      } else {
        const R ex[3] = {R(1), R(0), R(0)}, ey[3] = {R(0), R(1), R(0)}, ez[3] = {R(0), R(0), R(1)};
        normal_flux<NV>(P_.ph, Uq, ex, F[0]);
        normal_flux<NV>(P_.ph, Uq, ey, F[1]);
        normal_flux<NV>(P_.ph, Uq, ez, F[2]);
      }
      R Fv[3 * NV];
#pragma unroll
      for (int k = 0; k < 3 * NV; ++k) Fv[k] = R(0);
      if (visc) {
        R grad[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) grad[k] = gq[k * Q3 + q];
        viscous_flux<NV>(P_.ph, cv.mu, cv.kappa, Uq, grad, Fv);
      }
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const R gi = (J[r * 3 + 0] * (F[0][v] - Fa[0][v]) + J[r * 3 + 1] * (F[1][v] - Fa[1][v]) +
                        J[r * 3 + 2] * (F[2][v] - Fa[2][v])) * wq;
          const R gv = -(J[r * 3 + 0] * Fv[0 * NV + v] + J[r * 3 + 1] * Fv[1 * NV + v] +
                         J[r * 3 + 2] * Fv[2 * NV + v]) * wq;
          if (SPLIT) {
            Gi[(r * NV + v) * Q3 + q] = gi;
            Gv[(r * NV + v) * Q3 + q] = gv;
          } else {
            Gi[(r * NV + v) * Q3 + q] = gi + gv;
          }
        }
    }
    __syncthreads();
    R* Ri = Rr;
    R* Rv = Rr + NV * N3;
    R* A = W + L::DIV_AT;                 // uq and gq are dead: the x-pass results go there if they fit
    if (skip_inv) {
      for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) Ri[idx] = R(0);
      __syncthreads();
    } else {
      div3<NV, N, Q>(Gi, Ri, A, tb->bqT, tb->dqT);
    }
    if (SPLIT) {
      if (visc) {
        div3<NV, N, Q>(Gv, Rv, A, tb->bqT, tb->dqT);
      } else {
        for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) Rv[idx] = R(0);
        __syncthreads();
      }
    }
  }
  // ---- phase D: face terms, M^-1, stage update (k_hex_finalize with the residuals in shared memory)
  R* hc = W;                                    // [6][C][QF2] face flux at canonical points
  R* tmp = hc + 6 * C * QF2;                    // [6][C][QF][N]
  R* hs = tmp + 6 * C * QF * N;                 // [6][C][N2]; reused for the M^-1 partial sums
  const size_t base = (size_t)e * N3 * NV;
  // one face point per thread: its NV inviscid and NV viscous flux values (contiguous)
  for (int it = threadIdx.x; it < 6 * QF2; it += kThreads) {
    const int lf = it / QF2, q = it % QF2;
    const int f = fface[lf] >> 1, side = fface[lf] & 1;
    const double si = side == 0 ? -1.0 : 1.0;
    const int c = codes.perm[fperm[lf] + q];
    const size_t ki = ((size_t)fslot[lf] + q) * NV, kv = ((size_t)f * QF2 + q) * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if constexpr (sizeof(R) == sizeof(float)) {
        // float32 fluxes of the mixed-precision face kernel
        const R hi = skip_inv ? R(0) : (R)si * fd.fluxI32[ki + v];
        const R hv = visc ? -(R)si * fd.fluxV32[kv + v] : R(0);
        if (SPLIT) {
          hc[(lf * C + v) * QF2 + c] = hi;
          hc[(lf * C + NV + v) * QF2 + c] = hv;
        } else {
          hc[(lf * C + v) * QF2 + c] = hi + hv;
        }
      } else {
        const double hi = skip_inv ? 0.0 : si * fd.fluxI[ki + v];
        const double hv = visc ? -si * fd.fluxV[kv + v] : 0.0;
        if (SPLIT) {
          hc[(lf * C + v) * QF2 + c] = (R)hi;
          hc[(lf * C + NV + v) * QF2 + c] = (R)hv;
        } else {
          hc[(lf * C + v) * QF2 + c] = (R)(hi + hv);
        }
      }
    }
  }
  __syncthreads();
  tensor2<6 * C, QF, QF, N, N>(hc, hs, tmp, tb->bfT, tb->bfT);
  // non-affine elements: the residuals go to rows RrT [N3][CS] in element node order (inviscid
  // channels, then from CSH the viscous ones) in the dead hc/tmp region, for pair loads in the
  // dense M^-1
  constexpr int CSH = (NV + 16 / (int)sizeof(R) - 1) / (16 / (int)sizeof(R)) * (16 / (int)sizeof(R));
  constexpr int CS = SPLIT ? 2 * CSH : CSH;
  static_assert(CS * N3 <= 6 * C * (QF2 + QF * N), "the residual rows must end before hs");
  R* RrT = W;
  for (int idx = threadIdx.x; idx < C * N3; idx += kThreads) {
    const int c = idx / N3, l = idx % N3;
    const int xyz[3] = {l % N, (l / N) % N, l / N2};
    R acc = Rr[idx];
#pragma unroll
    for (int lf = 0; lf < 6; ++lf) {
      int a0, end, a1, a2;
      hex_face_axes(lf, a0, end, a1, a2);
      if (xyz[a0] == end) acc += hs[(lf * C + c) * N2 + xyz[a2] * N + xyz[a1]];
    }
    if (aff)
      Rr[idx] = acc;
    else
      RrT[tb->lex2node[l] * CS + (c < NV ? c : CSH + c - NV)] = acc;
  }
  __syncthreads();
  auto emit = [&](size_t o, double ri, double rv) {
    if (!A.stage) {
      if (A.out_inv[b]) A.out_inv[b][o] = ri;
      if (SPLIT && A.out_vis[b]) A.out_vis[b][o] = rv;
    } else {
      const double total = SPLIT ? ri + rv : ri;
      const double eul = S.b[b][o] + A.dt * total;
      if (SPLIT && A.out_vis[b]) A.out_vis[b][o] = rv;
      if (A.euler[b]) A.euler[b][o] = eul;
      A.dst[b][o] = A.alpha * A.base[b][o] + A.beta * eul;
    }
  };
  if (aff) {
    tensor3<C, N, N, N, N, N, N, false>(Rr, hs, tmp, hc, tb->m1i, tb->m1i, tb->m1i);
    const R cf = (R)B.acoef[e];
    for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
      const int v = idx / N3, l = idx % N3;
      const double ri = (double)(cf * hs[v * N3 + l]);
      const double rv = SPLIT ? (double)(cf * hs[(NV + v) * N3 + l]) : 0.0;
      emit(base + (size_t)tb->lex2node[l] * NV + v, ri, rv);
    }
    return;
  }
  constexpr int VB = NV < 8 ? NV : 8;
  constexpr int NG = (NV + VB - 1) / VB;
  constexpr int HALVES = NG * N3 * 2 <= kThreads ? 2 : 1;
  constexpr int JH = (N3 + HALVES - 1) / HALVES;
  R* part = hs;                                       // [HALVES][2][NV][N3]
  auto apply = [&](const auto* M) {
    for (int idx = threadIdx.x; idx < HALVES * NG * N3; idx += kThreads) {
      const int i = idx % N3, g = (idx / N3) % NG, h = idx / (NG * N3);
      const int v0 = g * VB;
      R ri[VB], rv[VB];
#pragma unroll
      for (int k = 0; k < VB; ++k) ri[k] = rv[k] = R(0);
      const int j1 = (h + 1) * JH < N3 ? (h + 1) * JH : N3;
#pragma unroll 4
      for (int j = h * JH; j < j1; ++j) {
        const R m = (R)__ldg(M + (size_t)j * N3 + i);
        R xi[VB], xv[VB];
        lds_vec<VB>(RrT + j * CS + v0, xi);
        if (SPLIT) lds_vec<VB>(RrT + j * CS + CSH + v0, xv);
#pragma unroll
        for (int k = 0; k < VB; ++k) {
          if (v0 + k < NV) {
            ri[k] += m * xi[k];
            if (SPLIT) rv[k] += m * xv[k];
          }
        }
      }
#pragma unroll
      for (int k = 0; k < VB; ++k) {
        if (v0 + k >= NV) continue;
        part[((h * 2 + 0) * NV + v0 + k) * N3 + i] = ri[k];
        part[((h * 2 + 1) * NV + v0 + k) * N3 + i] = rv[k];
      }
    }
  };
  if (MT32) apply(MT32); else apply(MT);
  __syncthreads();
  for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
    const int v = idx / N3, i = idx % N3;
    R si = part[(0 * NV + v) * N3 + i], sv = part[(1 * NV + v) * N3 + i];
    if (HALVES == 2) {
      si += part[(2 * NV + v) * N3 + i];
      sv += part[(3 * NV + v) * N3 + i];
    }
    emit(base + (size_t)i * NV + v, (double)si, (double)sv);
  }
}

// Predictor statistics of the hexahedron block (the layout of k_elem_stats), one warp per element:
// the Persson fractions use the tensor-product P1 projector (three N x N pencil passes, as the
// troubled-cell sensor) instead of the dense Np x Np projector, whose rows every warp would
// stream from L2 for every element.
template <int P, int NV>
__global__ void __launch_bounds__(kThreads) k_hex_elem_stats(const DevPlan P_, const StatePtrs S,
                                                            const HexTables tables, float* __restrict__ stats) {
  using D = HexDims<P>;
  constexpr int N = D::N, N3 = D::N3;
  __shared__ double work[kThreads / 32][4 * 2 * N3];   // per warp: Mon, Low, t1, t2
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * (kThreads / 32) + warp;
  if (e >= P_.blk[0].E) return;
  const double* Ug = S.b[0] + (size_t)e * N3 * NV;
  double* Mon = work[warp];
  double* Low = Mon + 2 * N3;
  double* t1 = Low + 2 * N3;
  double* t2 = t1 + 2 * N3;
  double srho = 0, sp = 0, rmin = INFINITY, rmax = -INFINITY, pmin = INFINITY, pmax = -INFINITY;
  for (int l = lane; l < N3; l += 32) {
    double u[NV], W[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = Ug[tables.lex2node[l] * NV + v];
    primitive<NV>(P_.ph, u, W);
    Mon[l] = W[0];
    Mon[N3 + l] = W[4];
    srho += W[0];
    sp += W[4];
    rmin = fmin(rmin, W[0]);
    rmax = fmax(rmax, W[0]);
    pmin = fmin(pmin, W[4]);
    pmax = fmax(pmax, W[4]);
  }
  __syncwarp();
  double h0 = 0, h1 = 0, s0 = 0, s1 = 0;
  if (P >= 2) {
    warp_tensor3<2, N>(Mon, Low, t1, t2, tables.p1d);
    for (int i = lane; i < N3; i += 32) {
      const double m0 = Mon[i], m1 = Mon[N3 + i];
      const double d0 = m0 - Low[i], d1 = m1 - Low[N3 + i];
      h0 += d0 * d0;
      h1 += d1 * d1;
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
  if (lane == 0) {
    float* st = stats + (size_t)e * kMlpStats;
    st[0] = (float)(srho / N3);
    st[1] = (float)(sp / N3);
    st[2] = (float)(rmin / fmax(fabs(rmax), 1e-30));
    st[3] = (float)(pmin / fmax(fabs(pmax), 1e-30));
    st[4] = (float)(h0 / fmax(s0, 1e-12));
    st[5] = (float)(h1 / fmax(s1, 1e-12));
  }
}

}  // namespace dgb
