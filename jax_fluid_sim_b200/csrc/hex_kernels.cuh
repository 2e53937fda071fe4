// Sum-factorised hexahedron kernels (float64, P1-P3).
//
// The reference builds hexahedron bases as tensor products of 1-D Lagrange
// polynomials on the nodes (0, 1, interior...) and integrates with tensor Gauss
// rules (hybrid/elements.py:199-274, 325-456; volume rule :60-98; quad face rule
// hybrid/geometry.py:74-87), but contracts them as dense (Nq x Np) matrices.
// Here every contraction is applied one axis at a time:
//   nodes -> volume points   N^3 -> N^2 Q -> N Q^2 -> Q^3  (and the transpose),
//   face slab -> face points N^2 -> N Qf -> Qf^2           (and the transpose),
// so a P3 element costs ~1.2k multiply-adds per field per contraction instead of
// 8k, and a face trace touches only the (P+1)^2 nodes of its face plus, for the
// normal derivative, one line of nodes per face node.
//
// Face points are produced in the element's canonical face grid (free axes in
// increasing order, first axis fastest) and mapped to the owner's face-point order
// through a per-trace-code permutation, so the face-point kernels and buffers are
// shared with the generic path (dg_kernels.cuh).
#pragma once
#include "aux_kernels.cuh"
#include "dg_kernels.cuh"

namespace dgb {

template <typename R>
struct HexTablesT {
  // volume Gauss points (Q) and face Gauss points (QF); nodes in 1-D order (0, 1, interior)
  R bq[5 * 4], dq[5 * 4];          // [Q][N]
  R bqT[4 * 5], dqT[4 * 5];        // [N][Q]
  R bf[4 * 4], df[4 * 4];          // [QF][N]
  R bfT[4 * 4];                    // [N][QF]
  R d0[4], d1[4];                  // 1-D basis derivatives at xi = 0 and xi = 1
  R m1i[4 * 4];                    // [N][N] inverse of the 1-D mass matrix (affine elements)
  R w1[5];                         // 1-D volume Gauss weights on [0, 1]
  R p1d[4 * 4];                    // [N][N] nodal projector onto span{1, xi} (sensor: P1 = p1d^(x)3)
  int lex2node[64];                // lexicographic (x fastest) -> element node index
};
using HexTables = HexTablesT<double>;
constexpr int kHexTableValues = 4 * 20 + 3 * 16 + 2 * 4 + 16 + 5 + 16;   // reals before lex2node
static_assert(offsetof(HexTablesT<double>, lex2node) == kHexTableValues * sizeof(double), "table layout");
static_assert(offsetof(HexTablesT<float>, lex2node) == kHexTableValues * sizeof(float), "table layout");

struct HexCodes {
  const uint8_t* perm;   // [codes][QF*QF]: owner face-point order -> canonical face grid index
  const int8_t* face;    // [codes]: local face of the code
};

template <int P>
struct HexDims {
  static constexpr int N = P + 1;
  static constexpr int Q = P == 1 ? 2 : (P == 2 ? 3 : 5);
  static constexpr int QF = P == 1 ? 2 : (P == 2 ? 3 : 4);
  static constexpr int N3 = N * N * N, Q3 = Q * Q * Q, N2 = N * N, QF2 = QF * QF;
};

// local face -> (normal axis, end) for the reference's hexahedron face list (hybrid/mesh.py:51-58)
__device__ __forceinline__ void hex_face_axes(int lf, int& a0, int& end, int& a1, int& a2) {
  // faces 0,1: z = 0,1; 2,4: y = 0,1; 5,3: x = 0,1
  a0 = lf < 2 ? 2 : ((lf == 2 || lf == 4) ? 1 : 0);
  end = (lf == 1 || lf == 3 || lf == 4) ? 1 : 0;
  a1 = a0 == 0 ? 1 : 0;
  a2 = a0 == 2 ? 1 : 2;
}

// lexicographic index of (axis coordinates c[3]) with x fastest
template <int N>
__device__ __forceinline__ int lex3(int cx, int cy, int cz) { return (cz * N + cy) * N + cx; }

// stride of axis a in the lexicographic node numbering (x fastest)
template <int N>
__device__ __forceinline__ int axis_stride(int a) { return a == 0 ? 1 : (a == 1 ? N : N * N); }

// One 1-D contraction along an axis, in pencil form: every work item (a line of IN values
// at stride `stride` between consecutive entries) keeps its inputs and the (OUT x IN) matrix in
// registers and produces the whole output line.  lines = number of lines; a line's first input
// sits at in_base(line), its first output at out_base(line); outputs also at stride ostride.
// The lines are shared among the block's threads, or, with first/step = lane/32, among one warp's
// lanes; a line's arithmetic does not depend on which thread takes it.
// A contiguous run of 4 (float) or 2 (double) values at a 16-byte aligned address moves as one
// 16-byte shared-memory access: a warp's lines then fall on distinct banks, where element-wise
// accesses at a line stride of 4 floats meet 4-way bank conflicts.
template <typename T>
__device__ __forceinline__ bool vec16(const T* p, int stride) {
  return stride == 1 && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
}
__device__ __forceinline__ void load16(const float* p, float* x) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
}
__device__ __forceinline__ void load16(const double* p, double* x) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  x[0] = v.x, x[1] = v.y;
}
__device__ __forceinline__ void store16(float* p, const float* x) {
  *reinterpret_cast<float4*>(p) = make_float4(x[0], x[1], x[2], x[3]);
}
__device__ __forceinline__ void store16(double* p, const double* x) {
  *reinterpret_cast<double2*>(p) = make_double2(x[0], x[1]);
}

template <int IN, int OUT, bool ACC, typename T, typename InBase, typename OutBase>
__device__ __forceinline__ void pencil(const T* in, T* out, const T* M, int lines, int istride, int ostride,
                                       InBase in_base, OutBase out_base, int first = -1, int step = 0) {
  constexpr int VW = 16 / sizeof(T);               // values per 16-byte access
  T m[OUT * IN];
#pragma unroll
  for (int k = 0; k < OUT * IN; ++k) m[k] = M[k];
  if (first < 0) {
    // every kernel that works a pencil pass with the whole CTA is launched with kThreads threads;
    // the compile-time stride gives the compiler the trip count
    first = threadIdx.x;
    step = kThreads;
  }
  for (int line = first; line < lines; line += step) {
    const T* src = in + in_base(line);
    T x[IN];
    if (IN % VW == 0 && vec16(src, istride)) {
#pragma unroll
      for (int i = 0; i < IN; i += VW) load16(src + i, &x[i]);
    } else {
#pragma unroll
      for (int i = 0; i < IN; ++i) x[i] = src[i * istride];
    }
    T* dst = out + out_base(line);
    T y[OUT];
#pragma unroll
    for (int o = 0; o < OUT; ++o) {
      T s = T(0);
#pragma unroll
      for (int i = 0; i < IN; ++i) s += m[o * IN + i] * x[i];
      y[o] = s;
    }
    if (OUT % VW == 0 && vec16(dst, ostride)) {
#pragma unroll
      for (int o = 0; o < OUT; o += VW) {
        if (ACC) {
          T cur[VW];
          load16(dst + o, cur);
#pragma unroll
          for (int k = 0; k < VW; ++k) cur[k] += y[o + k];
          store16(dst + o, cur);
        } else {
          store16(dst + o, &y[o]);
        }
      }
    } else {
#pragma unroll
      for (int o = 0; o < OUT; ++o) {
        if (ACC) dst[o * ostride] += y[o]; else dst[o * ostride] = y[o];
      }
    }
  }
}

// out[c][oz][oy][ox] (+)= sum Mz[oz][iz] My[oy][iy] Mx[ox][ix] in[c][iz][iy][ix]
template <int C, int IX, int IY, int IZ, int OX, int OY, int OZ, bool ACC, typename T>
__device__ __forceinline__ void tensor3(const T* in, T* out, T* t1, T* t2, const T* Mx, const T* My, const T* Mz) {
  // x: lines (c, iz, iy), contiguous inputs; t1[c][iz][iy][ox]
  pencil<IX, OX, false>(in, t1, Mx, C * IZ * IY, 1, 1, [](int l) { return l * IX; }, [](int l) { return l * OX; });
  __syncthreads();
  // y: lines (c, iz, ox), inputs at stride OX; t2[c][iz][oy][ox]
  pencil<IY, OY, false>(t1, t2, My, C * IZ * OX, OX, OX,
                        [](int l) { return (l / OX) * IY * OX + l % OX; },
                        [](int l) { return (l / OX) * OY * OX + l % OX; });
  __syncthreads();
  // z: lines (c, oy, ox), inputs at stride OX*OY; out[c][oz][oy][ox]
  pencil<IZ, OZ, ACC>(t2, out, Mz, C * OY * OX, OX * OY, OX * OY,
                      [](int l) { return (l / (OX * OY)) * IZ * OX * OY + l % (OX * OY); },
                      [](int l) { return (l / (OX * OY)) * OZ * OX * OY + l % (OX * OY); });
  __syncthreads();
}

// tensor3 with one N x N matrix on all three axes, worked by one warp (same arithmetic per output).
template <int C, int N, typename T>
__device__ __forceinline__ void warp_tensor3(const T* in, T* out, T* t1, T* t2, const T* M) {
  const int lane = threadIdx.x & 31;
  pencil<N, N, false>(in, t1, M, C * N * N, 1, 1, [](int l) { return l * N; }, [](int l) { return l * N; }, lane, 32);
  __syncwarp();
  pencil<N, N, false>(t1, t2, M, C * N * N, N, N,
                      [](int l) { return (l / N) * N * N + l % N; },
                      [](int l) { return (l / N) * N * N + l % N; }, lane, 32);
  __syncwarp();
  pencil<N, N, false>(t2, out, M, C * N * N, N * N, N * N,
                      [](int l) { return (l / (N * N)) * N * N * N + l % (N * N); },
                      [](int l) { return (l / (N * N)) * N * N * N + l % (N * N); }, lane, 32);
  __syncwarp();
}

// 2-D: out[c][k2][k1] = sum M2[k2][j2] M1[k1][j1] in[c][j2][j1]
template <int C, int J1, int J2, int K1, int K2, typename T>
__device__ __forceinline__ void tensor2(const T* in, T* out, T* t, const T* M1, const T* M2) {
  pencil<J1, K1, false>(in, t, M1, C * J2, 1, 1, [](int l) { return l * J1; }, [](int l) { return l * K1; });
  __syncthreads();
  pencil<J2, K2, false>(t, out, M2, C * K1, K1, K1,
                        [](int l) { return (l / K1) * J2 * K1 + l % K1; },
                        [](int l) { return (l / K1) * K2 * K1 + l % K1; });
  __syncthreads();
}

// Gather the N^2 slab of face (a0, end) from lexicographic nodal data X[c][N^3] into slab[c][j2][j1].
template <int C, int N, typename T>
__device__ __forceinline__ void face_slab(const T* X, T* slab, int a0, int end, int a1, int a2) {
  for (int idx = threadIdx.x; idx < C * N * N; idx += kThreads) {
    const int j1 = idx % N, j2 = (idx / N) % N, c = idx / (N * N);
    // 1-D node 0 sits at xi=0, node 1 at xi=1
    const int l = end * axis_stride<N>(a0) + j1 * axis_stride<N>(a1) + j2 * axis_stride<N>(a2);
    slab[idx] = X[c * N * N * N + l];
  }
}

// --------------------------------------------------------------------------------------------
// Shared-memory layouts (doubles) of the hex element kernels; each kernel has its own.
constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Sizes are in units of the kernel's real type R (float64, or float32 in the mixed kernels).
template <int P, int NV, typename R = double>
struct HexSmem {
  using D = HexDims<P>;
  static constexpr int N = D::N, Q = D::Q, QF = D::QF, N2 = D::N2, N3 = D::N3, Q3 = D::Q3, QF2 = D::QF2;
  // table size in R, rounded up to 16 bytes so that the arrays after the tables stay 16-byte aligned
  static constexpr int T = (int)((sizeof(HexTablesT<R>) + 15) / 16 * 16 / sizeof(R));
  static constexpr int MS = N3 + 1;                 // padded row stride of the staged M^-1 (transposed)
  // traces: U, v, then the six faces' slabs, contraction scratch, face values and tangential derivatives
  static constexpr int TR_U = T, TR_V = TR_U + NV * N3, TR_W = TR_V + 4 * N3;
  // The face values alias the slabs when the three face contractions run as one merged pass (every read of
  // the slabs comes before the barrier after which the face values are written); N2 == QF2 at P1-P3.
  static constexpr bool TR_ALIAS = (NV + 4) * N3 >= 24 * N * QF && N2 == QF2;
  static constexpr int TRACES = TR_W + 6 * (NV + 8) * (N2 + N * QF + (TR_ALIAS ? 0 : QF2)) + 2 * 24 * QF2;
  // lift: staged M^-T, b per face on its slab, b on all nodes, scratch
  static constexpr int LI_BS = T, LI_B = LI_BS + 6 * 12 * N2, LI_W = LI_B + 12 * N3;
  static constexpr int LI_X = LI_W + 72 * QF2 + 72 * QF * N + 72 * N2 + 72 * QF2;   // affine scratch
  static constexpr int LIFT = LI_X + 3 * 12 * N3;
  // volume: U, v, lift nodes, then U and gradients at the points and contraction scratch
  static constexpr int C1 = NV > 12 ? NV : 12;
  static constexpr int VO_U = T, VO_V = VO_U + NV * N3, VO_L = VO_V + 4 * N3, VO_W = VO_L + 12 * N3;
  static constexpr int VOL1 = NV * Q3 + 12 * Q3 + C1 * N * N * Q + C1 * N * Q * Q;
  template <bool SPLIT>
  static constexpr int VOL2 =
      NV * Q3 + 12 * Q3 + (SPLIT ? 6 : 3) * NV * Q3 + NV * Q * Q * N + NV * Q * N * N + (SPLIT ? NV * N3 : 0);
  template <bool SPLIT>
  static constexpr int VOLUME = VO_W + cmax(VOL1, VOL2<SPLIT>);
  // finalize: staged M^-T, residuals, face scratch
  static constexpr int FI_R = T, FI_W = FI_R + 2 * NV * N3;
  static constexpr int FINAL = FI_W + 6 * 2 * NV * (QF2 + QF * N) + cmax(6 * 2 * NV * N2, 4 * NV * N3);
};

template <int P>
__device__ __forceinline__ void load_tables(const HexTables& src, HexTables* dst) {
  const double* s = reinterpret_cast<const double*>(&src);
  double* d = reinterpret_cast<double*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(HexTables) / sizeof(double)); i += kThreads) d[i] = s[i];
}

// float32 copy of the tables for the mixed-precision kernels
template <int P>
__device__ __forceinline__ void load_tables(const HexTables& src, HexTablesT<float>* dst) {
  const double* s = reinterpret_cast<const double*>(&src);
  float* d = reinterpret_cast<float*>(dst);
  for (int i = threadIdx.x; i < kHexTableValues; i += kThreads) d[i] = (float)s[i];
  for (int i = threadIdx.x; i < 64; i += kThreads) dst->lex2node[i] = src.lex2node[i];
}

// Stage M^-1 of one element transposed into shared memory, in lexicographic node order:
// Mt[lj * MS + li] = M^-1[node(li)][node(lj)].  Global reads are coalesced rows.
template <int N3, int MS>
__device__ __forceinline__ void stage_minv(const double* Mg, const int* lex2node, const int* node2lex, double* Mt) {
  for (int idx = threadIdx.x; idx < N3 * N3; idx += kThreads) {
    const int i = idx / N3, j = idx % N3;          // element node indices
    Mt[node2lex[j] * MS + node2lex[i]] = Mg[idx];
  }
}

// --------------------------------------------------------------------------------------------
// Face traces of one hexahedron: anchor-form U, viscous variables, their raw physical
// gradients, for each of the six faces, in the owner's face-point order.
// F32: the viscous traces go to the float32 buffers trV32 / trG32 (fused form, mixed precision).
template <int P, int NV, typename R = double, bool F32 = false>
__global__ void __launch_bounds__(kThreads) k_hex_traces(const DevPlan P_, const StatePtrs S, int b,
                                                        const HexTables tables, const HexCodes codes) {
  using D = HexDims<P>;
  using L = HexSmem<P, NV, R>;
  constexpr int N = D::N, QF = D::QF, N2 = D::N2, N3 = D::N3, QF2 = D::QF2;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  R* smem = reinterpret_cast<R*>(dyn_smem);
  HexTablesT<R>* tb = reinterpret_cast<HexTablesT<R>*>(smem);
  R* U = smem + L::TR_U;             // [NV][N3], minus anchor
  R* V = smem + L::TR_V;             // [4][N3]
  // all six faces at once, channel blocks [U: 6*NV][v: 6*4][dv/dn: 6*4], each of N2 (slabs)
  // or QF2 (face points) values
  constexpr int CH = 6 * (NV + 8);
  R* slabs = smem + L::TR_W;
  R* ftmp = slabs + CH * N2;         // tensor2 scratch [CH][N][QF]
  // [CH][QF2] values at the canonical face points (over the slabs when the layout aliases them)
  R* fo = L::TR_ALIAS ? slabs : ftmp + CH * N * QF;
  R* g1 = L::TR_ALIAS ? ftmp + CH * N * QF : fo + CH * QF2;   // [6*4][QF2] derivative of v along a1
  R* g2 = g1 + 24 * QF2;             // [6*4][QF2] derivative of v along a2
  __shared__ int fslot[6], fperm[6];
  const BlockDev& B = P_.blk[b];
  const FaceDev& fd = P_.face[1];
  const int e = blockIdx.x;
  load_tables<P>(tables, tb);
  const double* Ug = S.b[b] + (size_t)e * N3 * NV;
  __shared__ double anchor[NV];
  if (threadIdx.x < NV) anchor[threadIdx.x] = Ug[threadIdx.x];
  if (threadIdx.x < 6) {
    int ft, f, side;
    decode_face(B.elem_face[e * 6 + threadIdx.x], ft, f, side);
    fslot[threadIdx.x] = (f * 2 + side) * QF2;
    fperm[threadIdx.x] = (side == 0 ? fd.oc[f] : fd.nc[f]) * QF2;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
    const int v = idx / N3, l = idx % N3;
    U[idx] = (R)(Ug[tb->lex2node[l] * NV + v] - anchor[v]);
  }
  const bool visc = P_.viscous;
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
  }
  __syncthreads();
  // one face node (face, j1, j2) per thread: all its channels
  for (int it = threadIdx.x; it < 6 * N2; it += kThreads) {
    const int lf = it / N2, j = it % N2, j1 = j % N, j2 = j / N;
    int a0, end, a1, a2;
    hex_face_axes(lf, a0, end, a1, a2);
    const int st0 = axis_stride<N>(a0), off = j1 * axis_stride<N>(a1) + j2 * axis_stride<N>(a2);
    const int at = end * st0 + off;
#pragma unroll
    for (int m = 0; m < NV; ++m) slabs[(lf * NV + m) * N2 + j] = U[m * N3 + at];
    if (visc) {
      const R* dn = end ? tb->d1 : tb->d0;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        slabs[(6 * NV + lf * 4 + m) * N2 + j] = V[m * N3 + at];
        R val = R(0);
#pragma unroll
        for (int j0 = 0; j0 < N; ++j0) val += dn[j0] * V[m * N3 + j0 * st0 + off];
        slabs[(6 * NV + 24 + lf * 4 + m) * N2 + j] = val;
      }
    }
  }
  __syncthreads();
  if (visc) {
    if constexpr ((NV + 4) * N3 >= 24 * N * QF) {
      // The three face contractions with two barriers instead of six: the x-passes (bf on every
      // channel; df on the 24 v channels, into the U/V region, dead after the slab gather), then the
      // y-passes (bf -> fo; bf on the df pass -> g1; df on the bf pass of the v channels -> g2).  Each
      // output goes through the same two 1-D products as in three tensor2 calls.  Consecutive passes
      // start on rotated threads so that the lines spread evenly.
      R* xd = U;                                   // [24][N][QF]
      const R* vsl = slabs + 6 * NV * N2;
      const int st = kThreads;
      auto rot = [st](int off) { return (int)((threadIdx.x + st - off % st) % st); };
      auto i1 = [](int l) { return l * N; };
      auto o1 = [](int l) { return l * QF; };
      pencil<N, QF, false>(slabs, ftmp, tb->bf, CH * N, 1, 1, i1, o1, rot(0), st);
      pencil<N, QF, false>(vsl, xd, tb->df, 24 * N, 1, 1, i1, o1, rot(CH * N), st);
      __syncthreads();
      auto i2 = [](int l) { return (l / QF) * N * QF + l % QF; };
      auto o2 = [](int l) { return (l / QF) * QF * QF + l % QF; };
      pencil<N, QF, false>(ftmp, fo, tb->bf, CH * QF, QF, QF, i2, o2, rot(0), st);
      pencil<N, QF, false>(xd, g1, tb->bf, 24 * QF, QF, QF, i2, o2, rot(CH * QF), st);
      pencil<N, QF, false>(ftmp + 6 * NV * N * QF, g2, tb->df, 24 * QF, QF, QF, i2, o2, rot(CH * QF + 24 * QF), st);
      __syncthreads();
    } else {
      tensor2<CH, N, N, QF, QF>(slabs, fo, ftmp, tb->bf, tb->bf);
      tensor2<24, N, N, QF, QF>(slabs + 6 * NV * N2, g1, ftmp, tb->df, tb->bf);
      tensor2<24, N, N, QF, QF>(slabs + 6 * NV * N2, g2, ftmp, tb->bf, tb->df);
    }
  } else {
    tensor2<6 * NV, N, N, QF, QF>(slabs, fo, ftmp, tb->bf, tb->bf);
  }
  // one face point per thread from here on: its values are contiguous in the face buffers
  for (int it = threadIdx.x; it < 6 * QF2; it += kThreads) {
    const int lf = it / QF2, q = it % QF2;
    const int c = codes.perm[fperm[lf] + q];
    double* dst = fd.trA + ((size_t)fslot[lf] + q) * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) dst[v] = anchor[v] + (double)fo[(lf * NV + v) * QF2 + c];
  }
  // the anchor state per face side, for the face kernel's anchor flux
  for (int idx = threadIdx.x; idx < 6 * NV; idx += kThreads)
    fd.anc[(size_t)(fslot[idx / NV] / QF2) * NV + idx % NV] = anchor[idx % NV];
  if (visc) {
    const R* fv = fo + 6 * NV * QF2;          // [6][4][QF2]
    const R* gn = fv + 24 * QF2;              // [6][4][QF2]
    for (int it = threadIdx.x; it < 6 * QF2; it += kThreads) {
      const int lf = it / QF2, q = it % QF2;
      const int c = codes.perm[fperm[lf] + q];
      const size_t pt = (size_t)fslot[lf] + q;
      // a point's 4 values and 12 gradients are contiguous: 16-byte stores
      R tv[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) tv[m] = fv[(lf * 4 + m) * QF2 + c];
      if (F32) {
        *reinterpret_cast<float4*>(fd.trV32 + pt * 4) = make_float4((float)tv[0], (float)tv[1], (float)tv[2], (float)tv[3]);
      } else {
        double2* t2 = reinterpret_cast<double2*>(fd.trV + pt * 4);
        t2[0] = make_double2((double)tv[0], (double)tv[1]);
        t2[1] = make_double2((double)tv[2], (double)tv[3]);
      }
      int a0, end, a1, a2;
      hex_face_axes(lf, a0, end, a1, a2);
      R J[9];
      if (sizeof(R) == sizeof(float) && fd.jinv32) {
#pragma unroll
        for (int k = 0; k < 9; ++k) J[k] = (R)fd.jinv32[pt * 9 + k];
      } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) J[k] = (R)fd.jinv[pt * 9 + k];
      }
      R gout[12];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int k = (lf * 4 + m) * QF2 + c;
        const R gnv = gn[k], g1v = g1[k], g2v = g2[k];
        // reference gradient component along axis r: normal (a0) or tangential (a1 < a2)
        const R gx = a0 == 0 ? gnv : g1v;
        const R gy = a0 == 1 ? gnv : (a0 == 0 ? g1v : g2v);
        const R gz = a0 == 2 ? gnv : g2v;
#pragma unroll
        for (int d = 0; d < 3; ++d) gout[m * 3 + d] = gx * J[0 * 3 + d] + gy * J[1 * 3 + d] + gz * J[2 * 3 + d];
      }
      if (F32) {
        float4* g4 = reinterpret_cast<float4*>(fd.trG32 + pt * 12);
#pragma unroll
        for (int k = 0; k < 3; ++k)
          g4[k] = make_float4((float)gout[4 * k], (float)gout[4 * k + 1], (float)gout[4 * k + 2], (float)gout[4 * k + 3]);
      } else {
        double2* g2d = reinterpret_cast<double2*>(fd.trG + pt * 12);
#pragma unroll
        for (int k = 0; k < 6; ++k) g2d[k] = make_double2((double)gout[2 * k], (double)gout[2 * k + 1]);
      }
    }
  }
}

// --------------------------------------------------------------------------------------------
// BR2 lifts of one hexahedron (hybrid/navier_stokes.py:138-188), with M^-1 read once:
//   b_f  = B_f^T jumpW_f on the slab of face f (transposed face interpolation);
//   lift = M^-1 sum_f b_f                      (= sum_f r_f, r_f = M^-1 b_f);
//   B_f r_f = B_f M^-1[slab_f, slab_f] b_f     (b_f vanishes off its slab, B_f likewise).
// Writes the nodal lift [12][N3] (lexicographic) and br2 * B_f r_f at each face's points.
template <int P, int NV, typename R = double>
__global__ void __launch_bounds__(kThreads) k_hex_lift(const DevPlan P_, int b, const HexTables tables,
                                                      const HexCodes codes, double* lift_out) {
  using D = HexDims<P>;
  using L = HexSmem<P, NV, R>;
  constexpr int N = D::N, QF = D::QF, N2 = D::N2, N3 = D::N3, QF2 = D::QF2;
  constexpr int CH = 6 * 12;                    // the six faces' 12 lift components
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  R* smem = reinterpret_cast<R*>(dyn_smem);
  HexTablesT<R>* tb = reinterpret_cast<HexTablesT<R>*>(smem);
  R* bs = smem + L::LI_BS;              // [6][12][N2] b_f on each face's slab
  R* ball = smem + L::LI_B;             // [12][N3]    b on all nodes
  R* jc = smem + L::LI_W;               // [6][12][QF2] jumps at the canonical face points
  R* tmp = jc + CH * QF2;               // [6*12][QF][N] contraction scratch
  R* rs = tmp + CH * QF * N;            // [6][12][N2] r_f on each face's slab
  R* lq = rs + CH * N2;                 // [6][12][QF2] B_f r_f
  __shared__ int node2lex[64], fslot[6], fperm[6], fjump[6];
  const BlockDev& B = P_.blk[b];
  const FaceDev& fd = P_.face[1];
  const int e = blockIdx.x;
  load_tables<P>(tables, tb);
  if (threadIdx.x < 6) {
    int ft, f, side;
    decode_face(B.elem_face[e * 6 + threadIdx.x], ft, f, side);
    fslot[threadIdx.x] = (f * 2 + side) * QF2;
    fperm[threadIdx.x] = (side == 0 ? fd.oc[f] : fd.nc[f]) * QF2;
    fjump[threadIdx.x] = f;
  }
  __syncthreads();
  for (int l = threadIdx.x; l < N3; l += kThreads) node2lex[tb->lex2node[l]] = l;
  // M^-T of this element in element node order: MT[j][i] = M^-1[i][j] (float32 copy in
  // mixed-precision plans)
  const double* MT = B.minv + (size_t)e * N3 * N3;
  const float* MT32 = (sizeof(R) == sizeof(float) && B.minv32) ? B.minv32 + (size_t)e * N3 * N3 : nullptr;
  for (int idx = threadIdx.x; idx < 6 * QF2 * 12; idx += kThreads) {
    const int lf = idx / (QF2 * 12), q = (idx / 12) % QF2, c = idx % 12;
    jc[(lf * 12 + c) * QF2 + codes.perm[fperm[lf] + q]] = (R)fd.jumpW[((size_t)fjump[lf] * QF2 + q) * 12 + c];
  }
  __syncthreads();
  tensor2<CH, QF, QF, N, N>(jc, bs, tmp, tb->bfT, tb->bfT);
  // b on all nodes: each node gathers the faces holding it, in local-face order (deterministic)
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
    ball[idx] = acc;
  }
  __syncthreads();
  // nodal lift = M^-1 b
  double* lg = lift_out + (size_t)e * 12 * N3;
  const bool aff = B.affine && B.affine[e];
  if (aff) {
    // affine: M^-1 = coef (m1i (x) m1i (x) m1i), three 1-D passes over the lexicographic b
    R* ax = smem + L::LI_X;
    R* at1 = ax + 12 * N3;
    R* at2 = at1 + 12 * N3;
    tensor3<12, N, N, N, N, N, N, false>(ball, ax, at1, at2, tb->m1i, tb->m1i, tb->m1i);
    const R cf = (R)B.acoef[e];
    for (int idx = threadIdx.x; idx < 12 * N3; idx += kThreads) lg[idx] = (double)(cf * ax[idx]);
    // M^-1 restricted to each face's slab: coef m1i[end][end] (m1i (x) m1i) over the free axes
    tensor2<CH, N, N, N, N>(bs, rs, tmp, tb->m1i, tb->m1i);
    for (int idx = threadIdx.x; idx < CH * N2; idx += kThreads) {
      int a0, end, a1, a2;
      hex_face_axes(idx / (12 * N2), a0, end, a1, a2);
      rs[idx] *= cf * tb->m1i[end * N + end];
    }
  } else {
    auto dense_lift = [&](const auto* M) {
      // a thread owns one element node i and half of the 12 components; M rows are read
      // coalesced across consecutive nodes
      for (int idx = threadIdx.x; idx < 2 * N3; idx += kThreads) {
        const int i = idx % N3, c0 = (idx / N3) * 6;
        R sacc[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
#pragma unroll 4
        for (int j = 0; j < N3; ++j) {
          const R m = (R)__ldg(M + (size_t)j * N3 + i);
          const int lj = node2lex[j];
#pragma unroll
          for (int k = 0; k < 6; ++k) sacc[k] += m * ball[(c0 + k) * N3 + lj];
        }
        const int li = node2lex[i];
#pragma unroll
        for (int k = 0; k < 6; ++k) lg[(c0 + k) * N3 + li] = (double)sacc[k];
      }
      // r_f = M^-1[slab_f, slab_f] b_f for the six faces
      for (int idx = threadIdx.x; idx < 6 * 2 * N2; idx += kThreads) {
        const int lf = idx / (2 * N2), s_i = idx % N2, c0 = ((idx / N2) % 2) * 6;
        int a0, end, a1, a2;
        hex_face_axes(lf, a0, end, a1, a2);
        const int st0 = axis_stride<N>(a0), st1 = axis_stride<N>(a1), st2 = axis_stride<N>(a2);
        const int ni = tb->lex2node[end * st0 + (s_i % N) * st1 + (s_i / N) * st2];
        R acc[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
        for (int s_j = 0; s_j < N2; ++s_j) {
          const int nj = tb->lex2node[end * st0 + (s_j % N) * st1 + (s_j / N) * st2];
          const R m = (R)__ldg(M + (size_t)nj * N3 + ni);
#pragma unroll
          for (int k = 0; k < 6; ++k) acc[k] += m * bs[(lf * 12 + c0 + k) * N2 + s_j];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) rs[(lf * 12 + c0 + k) * N2 + s_i] = acc[k];
      }
    };
    if (MT32) dense_lift(MT32); else dense_lift(MT);
  }
  __syncthreads();
  // br2 * B_f r_f at every face's points
  tensor2<CH, N, N, QF, QF>(rs, lq, tmp, tb->bf, tb->bf);
  for (int idx = threadIdx.x; idx < 6 * QF2 * 12; idx += kThreads) {
    const int lf = idx / (QF2 * 12), q = (idx / 12) % QF2, c = idx % 12;
    fd.liftF[((size_t)fslot[lf] + q) * 12 + c] =
        P_.ph.br2 * (double)lq[(lf * 12 + c) * QF2 + codes.perm[fperm[lf] + q]];
  }
}

// --------------------------------------------------------------------------------------------
// Volume residuals of one hexahedron: U (anchor form), grad v and the lift at the volume
// points by sum factorisation; inviscid flux minus the anchor flux and the viscous flux,
// contracted with w J^-T and the reference gradients (transposed sum factorisation).
// SPLIT writes inviscid and viscous residuals separately, otherwise their sum into Rinv.
template <int P, int NV, bool SPLIT, typename R = double>
__global__ void __launch_bounds__(kThreads, sizeof(R) == sizeof(float) ? 6 : 1) k_hex_volume(const DevPlan P_, const StatePtrs S, int b,
                                                        const HexTables tables, const double* lift_in) {
  using D = HexDims<P>;
  using L = HexSmem<P, NV, R>;
  constexpr int N = D::N, Q = D::Q, N3 = D::N3, Q3 = D::Q3;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  R* smem = reinterpret_cast<R*>(dyn_smem);
  HexTablesT<R>* tb = reinterpret_cast<HexTablesT<R>*>(smem);
  R* U = smem + L::VO_U;             // [NV][N3] minus anchor
  R* V = smem + L::VO_V;             // [4][N3]
  R* Lf = smem + L::VO_L;            // [12][N3]
  R* W = smem + L::VO_W;
  const BlockDev& B = P_.blk[b];
  const int e = blockIdx.x;
  const CaseView cv = case_view(P_.ph, B.ecase, e);
  load_tables<P>(tables, tb);
  const double* Ug = S.b[b] + (size_t)e * N3 * NV;
  __shared__ double anchor_d[NV];
  __shared__ R anchor[NV];
  if (threadIdx.x < NV) {
    anchor_d[threadIdx.x] = Ug[threadIdx.x];
    anchor[threadIdx.x] = (R)Ug[threadIdx.x];
  }
  __syncthreads();
  // differences to the anchor are formed in float64, then rounded to R
  for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
    const int v = idx / N3, l = idx % N3;
    U[idx] = (R)(Ug[tb->lex2node[l] * NV + v] - anchor_d[v]);
  }
  const bool visc = P_.viscous;
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
    const double* lg = lift_in + (size_t)e * 12 * N3;
    for (int idx = threadIdx.x; idx < 12 * N3; idx += kThreads) Lf[idx] = (R)lg[idx];
  }
  __syncthreads();
  R* uq = W;                           // [NV][Q3]   U - anchor at volume points
  R* gq = uq + NV * Q3;                // [12][Q3]   gradients of v: reference (3 x 4), then physical + lift
  R* t1 = gq + 12 * Q3;                // contraction scratch
  R* t2 = t1 + L::C1 * N * N * Q;
  tensor3<NV, N, N, N, Q, Q, Q, false>(U, uq, t1, t2, tb->bq, tb->bq, tb->bq);
  const double* jinv = B.jinv + (size_t)e * Q3 * 9;
  const float* jinv32 = (sizeof(R) == sizeof(float) && B.jinv32) ? B.jinv32 + (size_t)e * Q3 * 9 : nullptr;
  const double* wdet = B.wdet + (size_t)e * Q3;
  // affine element: one inverse Jacobian, w |J| = w1 w1 w1 det J (no per-point metrics read)
  const bool aff = B.affine && B.affine[e];
  R Ja[9], deta = R(0);
  if (aff) {
#pragma unroll
    for (int k = 0; k < 9; ++k) Ja[k] = (R)B.ajinv[(size_t)e * 9 + k];
    deta = (R)B.adet[e];
  }
  if (visc) {
    tensor3<4, N, N, N, Q, Q, Q, false>(V, gq + 0 * 4 * Q3, t1, t2, tb->dq, tb->bq, tb->bq);
    tensor3<4, N, N, N, Q, Q, Q, false>(V, gq + 1 * 4 * Q3, t1, t2, tb->bq, tb->dq, tb->bq);
    tensor3<4, N, N, N, Q, Q, Q, false>(V, gq + 2 * 4 * Q3, t1, t2, tb->bq, tb->bq, tb->dq);
    // reference -> physical gradient, in place per point: g[m*3+d] = sum_r dv_m/dxi_r J^-1[r][d]
    for (int q = threadIdx.x; q < Q3; q += kThreads) {
      R J[9], gr[12];
#pragma unroll
      for (int k = 0; k < 9; ++k) J[k] = aff ? Ja[k] : (jinv32 ? (R)jinv32[q * 9 + k] : (R)jinv[q * 9 + k]);
#pragma unroll
      for (int k = 0; k < 12; ++k) gr[k] = gq[k * Q3 + q];      // [r][m]
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          gq[(m * 3 + d) * Q3 + q] = gr[0 * 4 + m] * J[0 * 3 + d] + gr[1 * 4 + m] * J[1 * 3 + d] +
                                     gr[2 * 4 + m] * J[2 * 3 + d];
    }
    __syncthreads();
    tensor3<12, N, N, N, Q, Q, Q, true>(Lf, gq, t1, t2, tb->bq, tb->bq, tb->bq);   // + lift
  }
  R* Gi = t1;                          // [3][NV][Q3]
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
    {
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
  R* Ri = uq;                          // reuse: [NV][N3] (NV*N3 <= NV*Q3)
  R* s1 = Gi + (SPLIT ? 6 : 3) * NV * Q3;
  R* s2 = s1 + NV * Q * Q * N;
  R* Rv = s2 + NV * Q * N * N;         // [NV][N3] (SPLIT only)
  tensor3<NV, Q, Q, Q, N, N, N, false>(Gi + 0 * NV * Q3, Ri, s1, s2, tb->dqT, tb->bqT, tb->bqT);
  tensor3<NV, Q, Q, Q, N, N, N, true>(Gi + 1 * NV * Q3, Ri, s1, s2, tb->bqT, tb->dqT, tb->bqT);
  tensor3<NV, Q, Q, Q, N, N, N, true>(Gi + 2 * NV * Q3, Ri, s1, s2, tb->bqT, tb->bqT, tb->dqT);
  if (SPLIT && visc) {
    tensor3<NV, Q, Q, Q, N, N, N, false>(Gv + 0 * NV * Q3, Rv, s1, s2, tb->dqT, tb->bqT, tb->bqT);
    tensor3<NV, Q, Q, Q, N, N, N, true>(Gv + 1 * NV * Q3, Rv, s1, s2, tb->bqT, tb->dqT, tb->bqT);
    tensor3<NV, Q, Q, Q, N, N, N, true>(Gv + 2 * NV * Q3, Rv, s1, s2, tb->bqT, tb->bqT, tb->dqT);
  }
  // residuals stay in lexicographic [NV][N3] order for k_hex_finalize
  double* Rig = B.Rinv + (size_t)e * N3 * NV;
  double* Rvg = B.Rvis + (size_t)e * N3 * NV;
  for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
    Rig[idx] = (double)Ri[idx];
    if (SPLIT && visc) Rvg[idx] = (double)Rv[idx];
  }
}

// --------------------------------------------------------------------------------------------
// Gather face contributions into the nodes (transposed face interpolation per face, in local
// face order: deterministic), apply M^-1 (staged in shared memory), and write either the
// right-hand sides or the fused SSP-RK stage.  Rinv holds the total volume residual when !SPLIT.
template <int P, int NV, bool SPLIT, typename R = double>
__global__ void __launch_bounds__(kThreads) k_hex_finalize(const DevPlan P_, const StatePtrs S, int b,
                                                          const HexTables tables, const HexCodes codes,
                                                          const FinalizeArgs A) {
  using D = HexDims<P>;
  using L = HexSmem<P, NV, R>;
  constexpr int N = D::N, QF = D::QF, N2 = D::N2, N3 = D::N3, QF2 = D::QF2;
  constexpr int C = SPLIT ? 2 * NV : NV;        // channels: inviscid (and viscous) residual
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  R* smem = reinterpret_cast<R*>(dyn_smem);
  HexTablesT<R>* tb = reinterpret_cast<HexTablesT<R>*>(smem);
  R* Rr = smem + L::FI_R;                       // [C][N3] lexicographic (Ri, then Rv)
  R* hc = smem + L::FI_W;                       // [6][C][QF2] face flux at canonical points
  R* tmp = hc + 6 * C * QF2;                    // [6][C][QF][N]
  R* hs = tmp + 6 * C * QF * N;                 // [6][C][N2]; reused for the M^-1 partial sums
  __shared__ int node2lex[64];
  __shared__ int fslot[6], fperm[6], fface[6];
  const BlockDev& B = P_.blk[b];
  const FaceDev& fd = P_.face[1];
  const int e = blockIdx.x;
  load_tables<P>(tables, tb);
  if (threadIdx.x < 6) {
    int ft, f, side;
    decode_face(B.elem_face[e * 6 + threadIdx.x], ft, f, side);
    fslot[threadIdx.x] = (f * 2 + side) * QF2;
    fperm[threadIdx.x] = (side == 0 ? fd.oc[f] : fd.nc[f]) * QF2;
    fface[threadIdx.x] = (f << 1) | side;
  }
  __syncthreads();
  for (int l = threadIdx.x; l < N3; l += kThreads) node2lex[tb->lex2node[l]] = l;
  const size_t base = (size_t)e * N3 * NV;
  const bool visc = P_.viscous;
  // the six faces' fluxes, signed for this side, at the canonical face points
  for (int idx = threadIdx.x; idx < 6 * QF2 * NV; idx += kThreads) {
    const int lf = idx / (QF2 * NV), q = (idx / NV) % QF2, v = idx % NV;
    const int f = fface[lf] >> 1, side = fface[lf] & 1;
    const double si = side == 0 ? -1.0 : 1.0;
    const double hi = si * fd.fluxI[((size_t)fslot[lf] + q) * NV + v];
    const double hv = visc ? -si * fd.fluxV[((size_t)f * QF2 + q) * NV + v] : 0.0;
    const int c = codes.perm[fperm[lf] + q];
    if (SPLIT) {
      hc[(lf * C + v) * QF2 + c] = (R)hi;
      hc[(lf * C + NV + v) * QF2 + c] = (R)hv;
    } else {
      hc[(lf * C + v) * QF2 + c] = (R)(hi + hv);
    }
  }
  __syncthreads();
  tensor2<6 * C, QF, QF, N, N>(hc, hs, tmp, tb->bfT, tb->bfT);
  // residual plus the face terms of every face holding the node, faces in local order
  for (int idx = threadIdx.x; idx < C * N3; idx += kThreads) {
    const int c = idx / N3, l = idx % N3;
    const int xyz[3] = {l % N, (l / N) % N, l / N2};
    R acc = (R)(c < NV ? B.Rinv[base + c * N3 + l] : ((SPLIT && visc) ? B.Rvis[base + (c - NV) * N3 + l] : 0.0));
#pragma unroll
    for (int lf = 0; lf < 6; ++lf) {
      int a0, end, a1, a2;
      hex_face_axes(lf, a0, end, a1, a2);
      if (xyz[a0] == end) acc += hs[(lf * C + c) * N2 + xyz[a2] * N + xyz[a1]];
    }
    Rr[idx] = acc;
  }
  __syncthreads();
  // the stage update (or right-hand-side output) of one value: node-order offset o
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
  if (B.affine && B.affine[e]) {
    // affine: M^-1 = coef (m1i (x) m1i (x) m1i), three 1-D passes over the lexicographic residual
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
  // M^-1: out[node(i)] = sum_j M^-T[j][i] R[lex(j)].  Work items (column half, variable group,
  // node i); consecutive threads take consecutive i, so the M^-T rows are read coalesced.  The
  // halves are added in a fixed order.
  constexpr int VB = NV < 8 ? NV : 8;
  constexpr int NG = (NV + VB - 1) / VB;
  constexpr int HALVES = NG * N3 * 2 <= kThreads ? 2 : 1;
  constexpr int JH = (N3 + HALVES - 1) / HALVES;      // N3 is odd at P2
  const double* MT = B.minv + (size_t)e * N3 * N3;   // M^-T in element node order
  const float* MT32 = (sizeof(R) == sizeof(float) && B.minv32) ? B.minv32 + (size_t)e * N3 * N3 : nullptr;
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
        const int lj = node2lex[j];
#pragma unroll
        for (int k = 0; k < VB; ++k) {
          if (v0 + k < NV) {
            ri[k] += m * Rr[(v0 + k) * N3 + lj];
            if (SPLIT) rv[k] += m * Rr[(NV + v0 + k) * N3 + lj];
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

// --------------------------------------------------------------------------------------------
// Limiter / detector samples of one element (hybrid/limiter.py:29-67): the state at the nodes,
// at the volume quadrature points and at the face quadrature points of the six faces, in that
// order -> Smp[v][NS]; U receives the element state in lexicographic order and vq the
// volume-point values [NV][Q3].  The six faces go through one 2-D contraction (their slabs
// stacked as 6*NV channels) in fs, which holds 6*NV*(N2 + N*QF + QF2) values.  Ends without a
// barrier: callers synchronise before reading.
// Cell mean sum_q u_q w_q |J_q| / sum_q w_q |J_q| of NV fields at the Q3 volume points, worked by
// all threads: each strides over the points, a warp combines its lanes by shuffles and thread 0
// adds the warps in order (deterministic).  Ends with the block synchronised and mean[] set.
template <int NV>
__device__ void hex_cell_mean(const double* vq, const double* __restrict__ wdet, int Q3, double* mean,
                              double (*part)[NV + 1]) {
  double s[NV + 1];
#pragma unroll
  for (int v = 0; v <= NV; ++v) s[v] = 0.0;
  for (int q = threadIdx.x; q < Q3; q += kThreads) {
    const double w = wdet[q];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] += vq[v * Q3 + q] * w;
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
    for (int k = 0; k < (int)(kThreads >> 5); ++k) {
      a += part[k][threadIdx.x];
      w += part[k][NV];
    }
    mean[threadIdx.x] = a / w;
  }
  __syncthreads();
}

template <int P, int NV>
__device__ void hex_samples(const HexTables* tb, const double* Ug, double* U, double* Smp, double* t1, double* t2,
                            double* vq, double* fs) {
  using D = HexDims<P>;
  constexpr int N = D::N, Q = D::Q, QF = D::QF, N2 = D::N2, N3 = D::N3, Q3 = D::Q3, QF2 = D::QF2;
  constexpr int NS = N3 + Q3 + 6 * QF2;
  for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
    const int v = idx / N3, l = idx % N3;
    const double x = Ug[tb->lex2node[l] * NV + v];
    U[idx] = x;
    Smp[v * NS + l] = x;
  }
  __syncthreads();
  tensor3<NV, N, N, N, Q, Q, Q, false>(U, vq, t1, t2, tb->bq, tb->bq, tb->bq);
  for (int idx = threadIdx.x; idx < NV * Q3; idx += kThreads) {
    const int v = idx / Q3, q = idx % Q3;
    Smp[v * NS + N3 + q] = vq[idx];
  }
  double* slabs = fs;                    // [6][NV][N2]
  double* ftmp = slabs + 6 * NV * N2;    // [6][NV][N][QF]
  double* fo = ftmp + 6 * NV * N * QF;   // [6][NV][QF2]
  for (int idx = threadIdx.x; idx < 6 * NV * N2; idx += kThreads) {
    const int j1 = idx % N, j2 = (idx / N) % N, c = idx / N2, lf = c / NV, v = c % NV;
    int a0, end, a1, a2;
    hex_face_axes(lf, a0, end, a1, a2);
    slabs[idx] = U[v * N3 + end * axis_stride<N>(a0) + j1 * axis_stride<N>(a1) + j2 * axis_stride<N>(a2)];
  }
  __syncthreads();
  tensor2<6 * NV, N, N, QF, QF>(slabs, fo, ftmp, tb->bf, tb->bf);
  for (int idx = threadIdx.x; idx < 6 * NV * QF2; idx += kThreads) {
    const int q = idx % QF2, c = idx / QF2, lf = c / NV, v = c % NV;
    Smp[v * NS + N3 + Q3 + lf * QF2 + q] = fo[idx];
  }
}

// Zhang-Shu positivity limiter for hexahedra (hybrid/limiter.py:69-147) with the samples built
// by sum factorisation: nodes, volume points (tensor Gauss grid) and the Gauss grids of the six
// faces -- for a hexahedron mesh these are exactly the distinct face points the reference
// collects from its face groups.
template <int P, int NV>
__global__ void __launch_bounds__(kThreads) k_hex_positivity(const DevPlan P_, const StatePtrs S, int b,
                                                            const HexTables tables, const LimiterConst Lc,
                                                            const int* __restrict__ list,
                                                            const int* __restrict__ count) {
  using D = HexDims<P>;
  constexpr int N = D::N, Q = D::Q, QF = D::QF, N3 = D::N3, Q3 = D::Q3, QF2 = D::QF2;
  constexpr int NS = N3 + Q3 + 6 * QF2;             // samples per element
  extern __shared__ double smem[];
  HexTables* tb = reinterpret_cast<HexTables*>(smem);
  double* U = smem + HexSmem<P, NV>::T;             // [NV][N3] lexicographic
  double* Smp = U + NV * N3;                        // [NV][NS]
  double* t1 = Smp + NV * NS;                       // contraction scratch
  double* t2 = t1 + NV * N * N * Q;
  double* vq = t2 + NV * N * Q * Q;                 // [NV][Q3]
  double* fs = vq + NV * Q3;                        // face contraction scratch
  __shared__ double mean[NV];
  __shared__ double red[kThreads / 32];
  __shared__ int red_nan;
  __shared__ double sh_upper;
  const BlockDev& B = P_.blk[b];
  // The elements are those of list[0, *count): the ones the certificate pre-pass (k_certify) did not
  // clear.  A cleared element keeps its state: its theta is 1, and the reference's
  // mean + 1 * (U - mean) equals U to rounding.  Each CTA loads the tables once and takes the
  // listed elements in a grid stride.
  load_tables<P>(tables, tb);
  __syncthreads();
  const int n = *count;
  for (int item = blockIdx.x; item < n; item += gridDim.x) {
    const int e = list[item];
    double* Ug = S.b[b] + (size_t)e * N3 * NV;
    hex_samples<P, NV>(tb, Ug, U, Smp, t1, t2, vq, fs);
    if (threadIdx.x == 0) red_nan = 0;
    __syncthreads();
    // cell mean from the volume samples
    __shared__ double part[kThreads / 32][NV + 1];
    hex_cell_mean<NV>(vq, B.wdet + (size_t)e * Q3, Q3, mean, part);
    double Wm[NV];
    primitive<NV>(P_.ph, mean, Wm);
    const double rfloor = fmax(Lc.density_floor, Lc.relative_floor * Wm[0]);
    const double pfloor = fmax(Lc.pressure_floor, Lc.relative_floor * Wm[4]);
    double rmin = INFINITY;
    bool nan_seen = false;
    for (int r = threadIdx.x; r < NS; r += kThreads) {
      const double d = Smp[r];
      nan_seen |= isnan(d);
      rmin = fmin(rmin, d);
    }
    for (int o = 16; o > 0; o >>= 1) rmin = fmin(rmin, __shfl_xor_sync(0xffffffff, rmin, o));
    if (nan_seen) atomicOr(&red_nan, 1);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rmin;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = red[0];
      for (int k = 1; k < kThreads / 32; ++k) m = fmin(m, red[k]);
      if (red_nan) m = NAN;
      const double th = (m < rfloor) ? (mean[0] - rfloor) / fmax(mean[0] - m, 1.0e-30) : 1.0;
      sh_upper = isnan(th) ? th : fmin(fmax(th, 0.0), 1.0);
    }
    __syncthreads();
    const double upper = sh_upper;
    auto pressure_ok = [&](double theta) -> bool {
      bool ok = true;
      for (int r = threadIdx.x; r < NS; r += kThreads) {
        double s[NV];
  #pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = mean[v] + theta * (Smp[v * NS + r] - mean[v]);
        ok &= (pressure_of<NV>(P_.ph, s) >= pfloor);
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
    for (int idx = threadIdx.x; idx < NV * N3; idx += kThreads) {
      const int v = idx / N3, l = idx % N3;
      Ug[tb->lex2node[l] * NV + v] = mean[v] + theta * (U[idx] - mean[v]);
    }
    __syncthreads();   // the next element reuses the shared buffers and scalars
  }
}

// Troubled-cell detector on the sum-factorised samples (hybrid/limiter.py:165-185 sensor on
// (rho, p) at the nodes with the P1 projector; MOOD admissibility of every sample and the
// cell mean, hybrid/limiter.py:285-300).  Same outputs as k_troubled.
template <int P, int NV>
__global__ void __launch_bounds__(kThreads) k_hex_troubled(const DevPlan P_, const StatePtrs S, int b,
                                                          const HexTables tables, const LimiterConst Lc,
                                                          double* sensor_out, uint8_t* flag_out, const PredictArgs pa,
                                                          const int* __restrict__ list,
                                                          const int* __restrict__ count) {
  using D = HexDims<P>;
  constexpr int N = D::N, Q = D::Q, N3 = D::N3, Q3 = D::Q3, QF2 = D::QF2;
  constexpr int NS = N3 + Q3 + 6 * QF2;
  extern __shared__ double smem[];
  HexTables* tb = reinterpret_cast<HexTables*>(smem);
  double* U = smem + HexSmem<P, NV>::T;
  double* Smp = U + NV * N3;
  double* t1 = Smp + NV * NS;
  double* t2 = t1 + NV * N * N * Q;
  double* vq = t2 + NV * N * Q * Q;
  double* fs = vq + NV * Q3;
  double* Mon = fs + 6 * NV * (D::N2 + N * D::QF + D::QF2);   // [2][N3] (rho, p), lexicographic
  double* Low = Mon + 2 * N3;                                   // [2][N3] their P1 projections
  __shared__ double mean[NV];
  __shared__ double red[4][kThreads / 32];
  const BlockDev& B = P_.blk[b];
  // The elements are those of list[0, *count): the ones k_hex_sensor neither skipped (predicted)
  // nor certified.  Each CTA loads the tables once and takes the listed elements in a grid stride.
  load_tables<P>(tables, tb);
  __syncthreads();
  const int n = *count;
  for (int item = blockIdx.x; item < n; item += gridDim.x) {
    const int e = list[item];
    const double* Ug = S.b[b] + (size_t)e * N3 * NV;
    hex_samples<P, NV>(tb, Ug, U, Smp, t1, t2, vq, fs);
    for (int l = threadIdx.x; l < N3; l += kThreads) {
      double u[NV], W[NV];
  #pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = U[v * N3 + l];
      primitive<NV>(P_.ph, u, W);
      Mon[l] = W[0];
      Mon[N3 + l] = W[4];
    }
    __syncthreads();
    // P1 projection of (rho, p): the nodal projector onto the trilinear space is the threefold
    // tensor product of the 1-D projector onto span{1, xi} (three passes of N x N)
    if (P >= 2) tensor3<2, N, N, N, N, N, N, false>(Mon, Low, t1, t2, tb->p1d, tb->p1d, tb->p1d);
    __shared__ double part[kThreads / 32][NV + 1];
    hex_cell_mean<NV>(vq, B.wdet + (size_t)e * Q3, Q3, mean, part);
    double hi0 = 0.0, hi1 = 0.0, sc0 = 0.0, sc1 = 0.0;
    if (P >= 2) {
      for (int i = threadIdx.x; i < N3; i += kThreads) {
        const double m0 = Mon[i], m1 = Mon[N3 + i];
        const double d0 = m0 - Low[i], d1 = m1 - Low[N3 + i];
        hi0 += d0 * d0;
        hi1 += d1 * d1;
        sc0 += m0 * m0;
        sc1 += m1 * m1;
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
    bool bad = false;
    for (int r = threadIdx.x; r <= NS; r += kThreads) {
      double s[NV], W[NV];
  #pragma unroll
      for (int v = 0; v < NV; ++v) s[v] = r < NS ? Smp[v * NS + r] : mean[v];
      primitive<NV>(P_.ph, s, W);
      bool finite = true;
  #pragma unroll
      for (int v = 0; v < NV; ++v) finite &= isfinite(W[v]);
      bad |= !finite || (W[0] < Lc.density_floor) || (W[4] < Lc.pressure_floor);
    }
    const bool any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
      double h0 = 0, h1 = 0, s0 = 0, s1 = 0;
      for (int k = 0; k < kThreads / 32; ++k) {
        h0 += red[0][k];
        h1 += red[1][k];
        s0 += red[2][k];
        s1 += red[3][k];
      }
      double value = 0.0;
      if (P >= 2) {
        const double r0 = h0 / fmax(s0, 1.0e-12), r1 = h1 / fmax(s1, 1.0e-12);
        value = (isnan(r0) || isnan(r1)) ? NAN : fmax(r0, r1);
      }
      const bool detected = (value > Lc.sensor_threshold) || any_bad;
      if (sensor_out) sensor_out[e] = value;
      if (flag_out) flag_out[e] = (uint8_t)detected;
      count_prediction(pa, e, detected);
    }
    __syncthreads();   // the next element reuses the shared buffers
  }
}

// Troubled-cell pre-pass, one warp per element: predicted elements are flagged and skipped (as in
// predicted_skip); an element whose nodal values certify admissible samples and mean
// (certificate_from_range with the absolute floors) gets its sensor here (the same arithmetic and
// summation order as k_hex_troubled: the P1 projection by the same pencils, the squares summed
// per 32 nodes by the same shuffle tree) and its flag; every other element is appended to list
// for k_hex_troubled.  *count must be zero before the launch.
template <int P, int NV>
__global__ void __launch_bounds__(kThreads) k_hex_sensor(const DevPlan P_, const StatePtrs S, int b,
                                                        const HexTables tables, const LimiterConst Lc,
                                                        double* sensor_out, uint8_t* flag_out, const PredictArgs pa,
                                                        int* __restrict__ list, int* __restrict__ count) {
  using D = HexDims<P>;
  constexpr int N = D::N, N3 = D::N3;
  __shared__ double work[kThreads / 32][4 * 2 * N3];   // per warp: Mon, Low, t1, t2
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int E = P_.blk[b].E;
  const int e = blockIdx.x * (kThreads / 32) + warp;
  if (e >= E) return;
  if (pa.mode == 1 && pa.pred && pa.pred[e]) {
    if (lane == 0) {
      if (flag_out) flag_out[e] = 1;
      if (pa.counts) atomicAdd(pa.counts + 1, 1ULL);
    }
    return;
  }
  const double* Ug = S.b[b] + (size_t)e * N3 * NV;
  double mn[5], mx[5];
  const bool fin = warp_nodal_range<NV, N3>(Ug, mn, mx);
  if (!(fin && certificate_from_range(mn, mx, P_.ph, Lc.lebesgue, Lc.density_floor, Lc.pressure_floor, 0.0))) {
    if (lane == 0) list[atomicAdd(count, 1)] = e;
    return;
  }
  double* Mon = work[warp];
  double* Low = Mon + 2 * N3;
  double* t1 = Low + 2 * N3;
  double* t2 = t1 + 2 * N3;
  for (int l = lane; l < N3; l += 32) {
    double u[NV], W[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = Ug[tables.lex2node[l] * NV + v];
    primitive<NV>(P_.ph, u, W);
    Mon[l] = W[0];
    Mon[N3 + l] = W[4];
  }
  __syncwarp();
  double value = 0.0;
  if (P >= 2) {
    warp_tensor3<2, N>(Mon, Low, t1, t2, tables.p1d);
    // squares of the nodes lane and lane + 32, each set reduced by the block kernel's tree
    double h[2][4] = {};
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int i = lane + 32 * half;
      if (i < N3) {
        const double m0 = Mon[i], m1 = Mon[N3 + i];
        const double d0 = m0 - Low[i], d1 = m1 - Low[N3 + i];
        h[half][0] += d0 * d0;
        h[half][1] += d1 * d1;
        h[half][2] += m0 * m0;
        h[half][3] += m1 * m1;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) h[half][k] += __shfl_xor_sync(0xffffffff, h[half][k], o);
    }
    double t[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) t[k] = ((0.0 + h[0][k]) + h[1][k]);
    const double r0 = t[0] / fmax(t[2], 1.0e-12), r1 = t[1] / fmax(t[3], 1.0e-12);
    value = (isnan(r0) || isnan(r1)) ? NAN : fmax(r0, r1);
  }
  if (lane == 0) {
    const bool detected = value > Lc.sensor_threshold;
    if (sensor_out) sensor_out[e] = value;
    if (flag_out) flag_out[e] = (uint8_t)detected;
    count_prediction(pa, e, detected);
  }
}

template <int P, int NV>
constexpr int hex_positivity_smem() {
  using D = HexDims<P>;
  constexpr int NS = D::N3 + D::Q3 + 6 * D::QF2;
  return HexSmem<P, NV>::T + NV * D::N3 + NV * NS + NV * D::N * D::N * D::Q + NV * D::N * D::Q * D::Q +
         NV * D::Q3 + 6 * NV * (D::N2 + D::N * D::QF + D::QF2);
}

template <int P, int NV>
constexpr int hex_troubled_smem() {
  return hex_positivity_smem<P, NV>() + 4 * HexDims<P>::N3;
}

}  // namespace dgb
