// C ABI of the dgb200 library: plan construction and the hot-path entry points.
// Declarations and the reference method each entry point replaces: include/dgb200.h.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <algorithm>
#include <vector>

#include "aux_kernels.cuh"
#include "hex_fused.cuh"
#include "hex_kernels.cuh"
#include "mlp_kernels.cuh"
#include "mood_kernels.cuh"
#include "subcell_build.cuh"
#include "tc_volume.h"

using namespace dgb;

namespace dgb {
int set_error(int code, const char* msg);
}

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t err__ = (call);                                                           \
    if (err__ != cudaSuccess)                                                             \
      return fail(DGB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err__));   \
  } while (0)

}  // namespace

namespace dgb {
// Error channel shared with the other translation units of the library (chemistry).
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace dgb

// What a captured step depends on besides the plan's device buffers: the caller's pointers, dt
// and the generation of the plan's parameters (bumped by every change that alters a kernel
// argument).  Compared bytewise, so it is zero-filled before it is set.
struct StepKey {
  double* block[DGB_MAX_BLOCKS];
  double dt;
  dgb_status* status;
  unsigned long long generation;
};

struct dgb_plan {
  dgb_params prm;
  DevPlan dev;
  LimiterConst lim;
  std::vector<void*> allocations;
  // CUDA graph of one checked step (dgb_ssprk3_step_graph)
  unsigned long long generation = 0;
  cudaStream_t capture_stream = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  StepKey step_key;
  bool block_set[DGB_MAX_BLOCKS] = {false, false, false};
  bool finalized = false;
  bool face_present[2] = {false, false};
  // stage buffers for SSP-RK3
  double* stage1[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  double* stage2[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  Partial* partials = nullptr;
  int rate_grid[DGB_MAX_BLOCKS] = {0, 0, 0};
  int adm_grid[DGB_MAX_BLOCKS] = {0, 0, 0};
  int npartials = 0;
  double* dt_scratch = nullptr;
  // batched launches of the dense element kernels (all blocks in one grid) and their shared memory
  int num_cases = 0;   // dgb_plan_set_cases
  const double* face_points[2] = {nullptr, nullptr};   // dgb_plan_set_face_points
  double* force_partials = nullptr;                    // dgb_wall_forces scratch
  size_t force_partials_n = 0;
  ElemLaunch launch_tr, launch_vol, launch_fin, launch_tr64;
  size_t smem_tr = 0, smem_vol = 0, smem_fin = 0, smem_tr64 = 0;
  size_t smem_pos[DGB_MAX_BLOCKS], smem_troubled[DGB_MAX_BLOCKS];
  // sum-factorised hexahedron path (single hexahedron block)
  bool hex = false;
  HexTables hex_tables;
  // hexahedron positivity: elements the certificate pre-pass did not clear, and the grid that
  // works through them (resident CTAs of k_hex_positivity)
  int* cert_list = nullptr;
  int* cert_count = nullptr;
  int pos_grid = 0;
  int trb_grid = 0;   // the same for k_hex_troubled, which shares the list
  HexCodes hex_codes = {nullptr, nullptr};
  double* hex_lift = nullptr;     // [E][12][N3] nodal BR2 lift scratch
  // fused right-hand side (hex_fused.cuh): on by default, dgb_plan_set_fused
  bool fused = true;
  // false while a caller needs the float64 viscous traces (the wall-force integral reads them)
  bool f32_traces = true;
  HexFaceArgs hex_face = {nullptr, nullptr, nullptr, nullptr};
  // MOOD subcell fallback
  MoodDev mood;
  bool sub_block_set[DGB_MAX_BLOCKS] = {false, false, false};
  // boundary subface centres of the device-built subcell tables, kept until the faces are matched
  double* sub_bdc[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  bool sub_face_set[2] = {false, false};
  bool mood_ready = false;
  uint8_t* flags[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  // learned troubled-cell predictor (dgb_plan_set_predictor)
  int pred_mode = 0;
  const __half* pred_w16 = nullptr;
  const float* pred_norm = nullptr;
  float pred_threshold = 0.5f;
  float* pred_stats[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  float** pred_stats_dev = nullptr;
  float* pred_feat = nullptr;
  uint8_t* pred_flags[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  unsigned long long* pred_counts = nullptr;
  double* unl[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  double* eul[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  double* vis[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  double* rec[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  // tensor-core (tcgen05) inviscid volume kernel of the dense blocks (dgb_plan_set_tensor_cores)
  TcShape tc[DGB_MAX_BLOCKS];
  float* tc_image[DGB_MAX_BLOCKS] = {nullptr, nullptr, nullptr};
  bool tc_on[DGB_MAX_BLOCKS] = {false, false, false};
  int sm_count = 0;
  int* dev_err = nullptr;   // DGB_DEVICE_* bits recorded by kernels with bounded waits
};

namespace {

template <typename T>
int upload(dgb_plan* p, const T* host, size_t count, const T** out) {
  if (count == 0) {
    *out = nullptr;
    return DGB_OK;
  }
  if (!host) return fail(DGB_ERR_ARGUMENT, "null host table");
  void* d = nullptr;
  CK(cudaMalloc(&d, count * sizeof(T)));
  p->allocations.push_back(d);
  CK(cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice));
  *out = static_cast<const T*>(d);
  return DGB_OK;
}

int alloc(dgb_plan* p, size_t count, double** out) {
  void* d = nullptr;
  if (count == 0) count = 1;
  CK(cudaMalloc(&d, count * sizeof(double)));
  p->allocations.push_back(d);
  CK(cudaMemset(d, 0, count * sizeof(double)));
  *out = static_cast<double*>(d);
  return DGB_OK;
}

__global__ void k_to_float32(const double* __restrict__ src, float* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

// A float32 copy of n device doubles, owned by the plan (null source: null copy).
int to_float32(dgb_plan* p, const double* src, size_t n, float** out) {
  *out = nullptr;
  if (!src || n == 0) return DGB_OK;
  void* d = nullptr;
  CK(cudaMalloc(&d, n * sizeof(float)));
  p->allocations.push_back(d);
  k_to_float32<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256>>>(src, static_cast<float*>(d), n);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  *out = static_cast<float*>(d);
  return DGB_OK;
}

StatePtrs to_ptrs(const dgb_state* s) {
  StatePtrs out;
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) out.b[b] = s ? s->block[b] : nullptr;
  return out;
}

template <typename K>
int prepare(K kernel, size_t smem) {
  if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return DGB_OK;
}

int blocks_for(long n, int per) { return (int)((n + per - 1) / per); }

template <int P, typename T>
void launch_hex_lop(dgb_plan* p, const int* elems, int count, T* lop) {
  k_hex_lop<P, T><<<count * 6, 128>>>(p->dev, p->hex_tables, elems, count, lop);
}

// Tables of the fused face kernel (set-up): the local face of every face side, and the local-lift
// operators of the elements whose map is not affine (all elements when the plan has no affine
// data), indexed through lop_index.
int build_hex_face_tables(dgb_plan* p) {
  const BlockDev& B = p->dev.blk[0];
  const FaceDev& F = p->dev.face[1];
  const int E = B.E, QF2 = F.nq;
  void* d = nullptr;
  CK(cudaMalloc(&d, sizeof(int8_t) * (size_t)F.F * 2));
  p->allocations.push_back(d);
  CK(cudaMemset(d, 0, sizeof(int8_t) * (size_t)F.F * 2));
  int8_t* face_lf = static_cast<int8_t*>(d);
  k_hex_face_lf<<<blocks_for((long)E * 6, 256), 256>>>(p->dev, face_lf);
  CK(cudaGetLastError());
  std::vector<uint8_t> aff(E, 0);
  if (B.affine) CK(cudaMemcpy(aff.data(), B.affine, E, cudaMemcpyDeviceToHost));
  std::vector<int> index(E, -1), elems;
  for (int e = 0; e < E; ++e)
    if (!aff[e]) {
      index[e] = (int)elems.size();
      elems.push_back(e);
    }
  const int* dindex = nullptr;
  int rc;
  if ((rc = upload(p, index.data(), index.size(), &dindex))) return rc;
  // float64 operators for float64 plans; mixed plans round them to float32 when they store them,
  // as the float32 face kernel does when it reads them, so they keep only that copy
  double* lop = nullptr;
  float* lop32 = nullptr;
  if (!elems.empty()) {
    const int* delems = nullptr;
    if ((rc = upload(p, elems.data(), elems.size(), &delems))) return rc;
    const size_t n = elems.size() * 6 * (size_t)QF2 * QF2;
    const int cnt = (int)elems.size();
    if (p->prm.precision == 1) {
      if ((rc = alloc(p, (n + 1) / 2, &lop))) return rc;
      lop32 = reinterpret_cast<float*>(lop);
      lop = nullptr;
      switch (p->dev.degree) {
        case 1: launch_hex_lop<1>(p, delems, cnt, lop32); break;
        case 2: launch_hex_lop<2>(p, delems, cnt, lop32); break;
        default: launch_hex_lop<3>(p, delems, cnt, lop32); break;
      }
    } else {
      if ((rc = alloc(p, n, &lop))) return rc;
      switch (p->dev.degree) {
        case 1: launch_hex_lop<1>(p, delems, cnt, lop); break;
        case 2: launch_hex_lop<2>(p, delems, cnt, lop); break;
        default: launch_hex_lop<3>(p, delems, cnt, lop); break;
      }
    }
    CK(cudaGetLastError());
  }
  CK(cudaDeviceSynchronize());
  p->hex_face = HexFaceArgs{face_lf, dindex, lop, lop32};
  return DGB_OK;
}

// ------------------------------------------------------------------ dense element launches
enum DenseKind { traces_kind, volume_kind, finalize_kind };

// Threads per element: a power of two covering the nodes, volume points and face points (the
// face-point count bounded by local faces x the largest face rule), 16 to kThreads.
int dense_width(const dgb_plan* p, const BlockDev& B) {
  int nq = 0;
  for (int ft = 0; ft < 2; ++ft)
    if (p->face_present[ft] && p->dev.face[ft].nq > nq) nq = p->dev.face[ft].nq;
  const int need = std::max(std::max(B.Np, B.Nq), B.nlf * nq);
  int w = 16;
  while (w < need && w < kThreads) w *= 2;
  return w;
}

// Per-element shared-memory slots (bytes, 16-aligned) for one kernel kind and real size.
void dense_slots(const dgb_plan* p, ElemLaunch& L, DenseKind kind, size_t rs) {
  const int NV = p->dev.nv;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    const BlockDev& B = p->dev.blk[b];
    size_t vals = 0;
    if (kind == traces_kind) vals = traces_slot(B.Np, NV);
    else if (kind == volume_kind)
      vals = VolumeSmem(B.Np, B.Nq, B.nlf, NV, p->dev.viscous, volume_chunks(B.Np, L.W[b])).total;
    else vals = finalize_slot(B.Np, B.nlf, NV, p->dev.viscous);
    L.slot[b] = (int)((vals * rs + 15) / 16 * 16);
  }
}

// Fills the launch (block offsets, widths, slots) and returns its dynamic shared memory.
// Lays the launch out for the widths in L.W (block offsets, slots) and returns its dynamic
// shared memory.
size_t dense_layout(const dgb_plan* p, ElemLaunch& L, DenseKind kind, size_t rs) {
  L.nblocks = p->dev.nblocks;
  L.cta0[0] = 0;
  for (int b = 0; b < p->dev.nblocks; ++b)
    L.cta0[b + 1] = L.cta0[b] + blocks_for(p->dev.blk[b].E, kThreads / L.W[b]);
  dense_slots(p, L, kind, rs);
  size_t most = 0;
  for (int b = 0; b < p->dev.nblocks; ++b)
    most = std::max(most, (size_t)(kThreads / L.W[b]) * (size_t)L.slot[b]);
  return most;
}

size_t dense_smem(const dgb_plan* p, ElemLaunch& L, DenseKind kind, size_t rs) {
  for (int b = 0; b < p->dev.nblocks; ++b) L.W[b] = dense_width(p, p->dev.blk[b]);
  return dense_layout(p, L, kind, rs);
}

// ------------------------------------------------------------------ RHS pipeline
template <int NV>
int launch_face_flux(dgb_plan* p, const StatePtrs& S, int ft, cudaStream_t st) {
  const FaceDev& F = p->dev.face[ft];
  if (F.F == 0) return DGB_OK;
  k_face_flux<NV><<<blocks_for((long)F.F * F.nq, kThreads), kThreads, 0, st>>>(p->dev, S, ft);
  return DGB_OK;
}

template <int P, int NV, bool SPLIT, typename R>
int run_rhs_hex(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st, cudaEvent_t* ev) {
  using LR = HexSmem<P, NV, R>;
  const DevPlan& D = p->dev;
  const int E = D.blk[0].E;
  const size_t sm_tr = sizeof(R) * (size_t)LR::TRACES, sm_li = sizeof(R) * (size_t)LR::LIFT;
  const size_t sm_vo = sizeof(R) * (size_t)LR::template VOLUME<SPLIT>, sm_fi = sizeof(R) * (size_t)LR::FINAL;
  int rc;
  if (ev) CK(cudaEventRecord(ev[0], st));
  if ((rc = prepare(k_hex_traces<P, NV, R>, sm_tr))) return rc;
  k_hex_traces<P, NV, R><<<E, kThreads, sm_tr, st>>>(D, S, 0, p->hex_tables, p->hex_codes);
  if (ev) CK(cudaEventRecord(ev[1], st));
  if ((rc = launch_face_flux<NV>(p, S, 1, st))) return rc;
  if (ev) CK(cudaEventRecord(ev[2], st));
  if (D.viscous) {
    if ((rc = prepare(k_hex_lift<P, NV, R>, sm_li))) return rc;
    k_hex_lift<P, NV, R><<<E, kThreads, sm_li, st>>>(D, 0, p->hex_tables, p->hex_codes, p->hex_lift);
  }
  if (ev) CK(cudaEventRecord(ev[3], st));
  if ((rc = prepare(k_hex_volume<P, NV, SPLIT, R>, sm_vo))) return rc;
  k_hex_volume<P, NV, SPLIT, R><<<E, kThreads, sm_vo, st>>>(D, S, 0, p->hex_tables, p->hex_lift);
  if (ev) CK(cudaEventRecord(ev[4], st));
  if (D.viscous)
    k_face_visc<NV><<<blocks_for((long)D.face[1].F * D.face[1].nq, kThreads), kThreads, 0, st>>>(D, 1);
  if (ev) CK(cudaEventRecord(ev[5], st));
  if ((rc = prepare(k_hex_finalize<P, NV, SPLIT, R>, sm_fi))) return rc;
  k_hex_finalize<P, NV, SPLIT, R><<<E, kThreads, sm_fi, st>>>(D, S, 0, p->hex_tables, p->hex_codes, A);
  if (ev) CK(cudaEventRecord(ev[6], st));
  CK(cudaGetLastError());
  return DGB_OK;
}

// The fused form: traces, one face kernel, one element kernel (hex_fused.cuh).  Stage events as
// in run_rhs_hex, the lift, viscous-face and finalize stages being part of the face and element
// kernels (zero-length).
template <int P, int NV, bool SPLIT, typename R>
int run_rhs_hex_fused(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st, cudaEvent_t* ev) {
  using LR = HexSmem<P, NV, R>;
  using LE = HexElemSmem<P, NV, SPLIT, R>;
  const DevPlan& D = p->dev;
  const int E = D.blk[0].E;
  const size_t sm_tr = sizeof(R) * (size_t)LR::TRACES, sm_el = sizeof(R) * (size_t)LE::TOTAL;
  int rc;
  if (ev) CK(cudaEventRecord(ev[0], st));
  // mixed precision: the viscous traces travel to the face kernel in float32
  constexpr bool MIXED = sizeof(R) == sizeof(float);
  const bool f32 = MIXED && D.face[1].trV32 != nullptr && p->f32_traces;
  constexpr int FPC = kThreads / HexDims<P>::QF2;
  const int fgrid = blocks_for(D.face[1].F, FPC);
  if (f32) {
    if ((rc = prepare(k_hex_traces<P, NV, R, MIXED>, sm_tr))) return rc;
    k_hex_traces<P, NV, R, MIXED><<<E, kThreads, sm_tr, st>>>(D, S, 0, p->hex_tables, p->hex_codes);
  } else {
    if ((rc = prepare(k_hex_traces<P, NV, R>, sm_tr))) return rc;
    k_hex_traces<P, NV, R><<<E, kThreads, sm_tr, st>>>(D, S, 0, p->hex_tables, p->hex_codes);
  }
  if (ev) CK(cudaEventRecord(ev[1], st));
  if (D.face[1].F > 0) {
    if (f32)
      k_hex_face<P, NV, R, MIXED><<<fgrid, kThreads, 0, st>>>(D, p->hex_tables, p->hex_codes, p->hex_face);
    else
      k_hex_face<P, NV, R><<<fgrid, kThreads, 0, st>>>(D, p->hex_tables, p->hex_codes, p->hex_face);
  }
  if (ev) {
    CK(cudaEventRecord(ev[2], st));
    CK(cudaEventRecord(ev[3], st));
  }
  if ((rc = prepare(k_hex_element<P, NV, SPLIT, R>, sm_el))) return rc;
  k_hex_element<P, NV, SPLIT, R><<<E, kThreads, sm_el, st>>>(D, S, p->hex_tables, p->hex_codes, A);
  if (ev) {
    CK(cudaEventRecord(ev[4], st));
    CK(cudaEventRecord(ev[5], st));
    CK(cudaEventRecord(ev[6], st));
  }
  CK(cudaGetLastError());
  return DGB_OK;
}

// The fused element kernel alone, split residuals, on the face buffers of the last right-hand side.
template <int P, int NV, typename R>
int run_hex_element_pass(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st) {
  using LE = HexElemSmem<P, NV, true, R>;
  const size_t sm_el = sizeof(R) * (size_t)LE::TOTAL;
  int rc;
  if ((rc = prepare(k_hex_element<P, NV, true, R>, sm_el))) return rc;
  k_hex_element<P, NV, true, R><<<p->dev.blk[0].E, kThreads, sm_el, st>>>(p->dev, S, p->hex_tables, p->hex_codes, A);
  CK(cudaGetLastError());
  return DGB_OK;
}

// The viscous residual of the flagged elements only (p->vis), for the subcell scheme: the fused
// element kernel with the inviscid terms skipped, on the face data of the stage's right-hand side.
template <int NV>
int run_viscous_flagged(dgb_plan* p, const StatePtrs& S, cudaStream_t st) {
  FinalizeArgs V;
  memset(&V, 0, sizeof(V));
  V.out_vis[0] = p->vis[0];
  V.skip_inviscid = p->flags[0];
  V.only = p->flags[0];
  const bool f32 = p->prm.precision == 1;
  switch (p->dev.degree) {
    case 1: return f32 ? run_hex_element_pass<1, NV, float>(p, S, V, st) : run_hex_element_pass<1, NV, double>(p, S, V, st);
    case 2: return f32 ? run_hex_element_pass<2, NV, float>(p, S, V, st) : run_hex_element_pass<2, NV, double>(p, S, V, st);
    default: return f32 ? run_hex_element_pass<3, NV, float>(p, S, V, st) : run_hex_element_pass<3, NV, double>(p, S, V, st);
  }
}

template <int NV, bool SPLIT, typename R>
int run_rhs_hex_deg(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st, cudaEvent_t* ev) {
  if (p->fused) {
    switch (p->dev.degree) {
      case 1: return run_rhs_hex_fused<1, NV, SPLIT, R>(p, S, A, st, ev);
      case 2: return run_rhs_hex_fused<2, NV, SPLIT, R>(p, S, A, st, ev);
      default: return run_rhs_hex_fused<3, NV, SPLIT, R>(p, S, A, st, ev);
    }
  }
  switch (p->dev.degree) {
    case 1: return run_rhs_hex<1, NV, SPLIT, R>(p, S, A, st, ev);
    case 2: return run_rhs_hex<2, NV, SPLIT, R>(p, S, A, st, ev);
    default: return run_rhs_hex<3, NV, SPLIT, R>(p, S, A, st, ev);
  }
}

template <int NV, bool SPLIT>
int run_rhs_hex_prec(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st, cudaEvent_t* ev) {
  return p->prm.precision == 1 ? run_rhs_hex_deg<NV, SPLIT, float>(p, S, A, st, ev)
                               : run_rhs_hex_deg<NV, SPLIT, double>(p, S, A, st, ev);
}

template <int NV, typename R>
int run_rhs_dense(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st, cudaEvent_t* ev) {
  const DevPlan& P = p->dev;
  int rc;
  if (ev) CK(cudaEventRecord(ev[0], st));
  if ((rc = prepare(k_traces<NV, R>, p->smem_tr))) return rc;
  k_traces<NV, R><<<p->launch_tr.cta0[P.nblocks], kThreads, p->smem_tr, st>>>(P, S, p->launch_tr);
  if (ev) CK(cudaEventRecord(ev[1], st));
  for (int ft = 0; ft < 2; ++ft)
    if (p->face_present[ft])
      if ((rc = launch_face_flux<NV>(p, S, ft, st))) return rc;
  if (ev) CK(cudaEventRecord(ev[2], st));
  if (ev) CK(cudaEventRecord(ev[3], st));     // the dense k_volume does the BR2 lift itself
  if ((rc = prepare(k_volume<NV, R>, p->smem_vol))) return rc;
  if (sizeof(R) == sizeof(float) && NV == 5 && !P.viscous && (p->tc_on[0] || p->tc_on[1] || p->tc_on[2])) {
    // tensor-core blocks first, then one launch of k_volume over the remaining blocks' CTA ranges
    ElemLaunch rest = p->launch_vol;
    rest.cta0[0] = 0;
    for (int b = 0; b < P.nblocks; ++b) {
      const int n = p->tc_on[b] ? 0 : p->launch_vol.cta0[b + 1] - p->launch_vol.cta0[b];
      rest.cta0[b + 1] = rest.cta0[b] + n;
      if (p->tc_on[b]) {
        const cudaError_t e = tc_volume(P, S, b, p->tc[b], p->tc_image[b], p->dev_err, p->sm_count, st);
        if (e != cudaSuccess)
          return fail(DGB_ERR_CUDA, std::string("tensor-core volume launch: ") + cudaGetErrorString(e));
      }
    }
    if (rest.cta0[P.nblocks] > 0)
      k_volume<NV, R><<<rest.cta0[P.nblocks], kThreads, p->smem_vol, st>>>(P, S, rest);
  } else {
    k_volume<NV, R><<<p->launch_vol.cta0[P.nblocks], kThreads, p->smem_vol, st>>>(P, S, p->launch_vol);
  }
  if (ev) CK(cudaEventRecord(ev[4], st));
  if (P.viscous)
    for (int ft = 0; ft < 2; ++ft)
      if (p->face_present[ft])
        k_face_visc<NV><<<blocks_for((long)P.face[ft].F * P.face[ft].nq, kThreads), kThreads, 0, st>>>(P, ft);
  if (ev) CK(cudaEventRecord(ev[5], st));
  if ((rc = prepare(k_finalize<NV, R>, p->smem_fin))) return rc;
  k_finalize<NV, R><<<p->launch_fin.cta0[P.nblocks], kThreads, p->smem_fin, st>>>(P, S, p->launch_fin, A);
  if (ev) CK(cudaEventRecord(ev[6], st));
  CK(cudaGetLastError());
  return DGB_OK;
}

// Autotuner of the dense element kernels: for each kernel and block, the threads per element W
// in {16, 32, 64, 128} that gives the shortest launch (best of `reps` CUDA-event timings with
// the other blocks' widths fixed, one coordinate sweep), on the plan's own buffers filled by one
// right-hand-side evaluation of U.  The choice is kept in the plan's launches.
template <int NV, typename R>
int autotune_dense(dgb_plan* p, const StatePtrs& S, int reps, cudaStream_t st, int* widths) {
  const DevPlan& P = p->dev;
  FinalizeArgs A;
  memset(&A, 0, sizeof(A));
  int rc;
  if ((rc = run_rhs_dense<NV, R>(p, S, A, st, nullptr))) return rc;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const size_t rs = sizeof(R);
  ElemLaunch* launches[3] = {&p->launch_tr, &p->launch_vol, &p->launch_fin};
  size_t* smems[3] = {&p->smem_tr, &p->smem_vol, &p->smem_fin};
  const DenseKind kinds[3] = {traces_kind, volume_kind, finalize_kind};
  auto launch = [&](int k, const ElemLaunch& L, size_t sm) -> int {
    int r;
    if (k == 0) {
      if ((r = prepare(k_traces<NV, R>, sm))) return r;
      k_traces<NV, R><<<L.cta0[P.nblocks], kThreads, sm, st>>>(P, S, L);
    } else if (k == 1) {
      if ((r = prepare(k_volume<NV, R>, sm))) return r;
      k_volume<NV, R><<<L.cta0[P.nblocks], kThreads, sm, st>>>(P, S, L);
    } else {
      if ((r = prepare(k_finalize<NV, R>, sm))) return r;
      k_finalize<NV, R><<<L.cta0[P.nblocks], kThreads, sm, st>>>(P, S, L, A);
    }
    CK(cudaGetLastError());
    return DGB_OK;
  };
  for (int k = 0; k < 3; ++k) {
    for (int b = 0; b < P.nblocks; ++b) {
      ElemLaunch best = *launches[k];
      size_t best_sm = *smems[k];
      float best_ms = 3.4e38f;
      for (int W = 16; W <= kThreads; W *= 2) {
        ElemLaunch L = best;
        L.W[b] = W;
        const size_t sm = dense_layout(p, L, kinds[k], rs);
        if (sm > 227 * 1024) continue;
        float t = 3.4e38f;
        for (int r = 0; r < reps; ++r) {
          CK(cudaEventRecord(e0, st));
          if ((rc = launch(k, L, sm))) return rc;
          CK(cudaEventRecord(e1, st));
          CK(cudaEventSynchronize(e1));
          float ms = 0.0f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          t = std::min(t, ms);
        }
        if (t < best_ms) {
          best_ms = t;
          best = L;
          best_sm = sm;
        }
      }
      *launches[k] = best;
      *smems[k] = best_sm;
    }
    if (widths)
      for (int b = 0; b < DGB_MAX_BLOCKS; ++b) widths[k * DGB_MAX_BLOCKS + b] = b < P.nblocks ? launches[k]->W[b] : 0;
  }
  CK(cudaEventDestroy(e0));
  CK(cudaEventDestroy(e1));
  ++p->generation;
  return DGB_OK;
}

// events: optional array of DGB_RHS_STAGES + 1 events recorded around the stages
template <int NV>
int run_rhs(dgb_plan* p, const StatePtrs& S, const FinalizeArgs& A, cudaStream_t st, cudaEvent_t* ev = nullptr) {
  const bool split = !A.stage || A.out_vis[0] != nullptr;
  if (p->hex) return split ? run_rhs_hex_prec<NV, true>(p, S, A, st, ev) : run_rhs_hex_prec<NV, false>(p, S, A, st, ev);
  return p->prm.precision == 1 ? run_rhs_dense<NV, float>(p, S, A, st, ev) : run_rhs_dense<NV, double>(p, S, A, st, ev);
}

// Resident CTAs of k_hex_positivity over the whole GPU (set-up; at most one per element).
template <int P, int NV>
int hex_positivity_grid(dgb_plan* p) {
  const size_t sm = sizeof(double) * (size_t)hex_positivity_smem<P, NV>();
  int rc;
  if ((rc = prepare(k_hex_positivity<P, NV>, sm))) return rc;
  int dev = 0, sms = 0, per_sm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hex_positivity<P, NV>, kThreads, sm));
  const long long grid = (long long)std::max(per_sm, 1) * std::max(sms, 1);
  p->pos_grid = (int)std::min<long long>(grid, std::max(p->dev.blk[0].E, 1));
  return DGB_OK;
}

// Positivity on the sum-factorised path: the certificate pre-pass (one warp per element) lists the
// elements it cannot clear, and k_hex_positivity limits only those.
template <int P, int NV>
int run_positivity_hex(dgb_plan* p, const StatePtrs& S, cudaStream_t st) {
  const size_t sm = sizeof(double) * (size_t)hex_positivity_smem<P, NV>();
  const BlockDev& B = p->dev.blk[0];
  if (B.E == 0) return DGB_OK;
  CK(cudaMemsetAsync(p->cert_count, 0, sizeof(int), st));
  k_certify<NV, HexDims<P>::N3><<<blocks_for(B.E, kThreads / 32), kThreads, 0, st>>>(
      S.b[0], B.E, p->dev.ph, p->lim.lebesgue, p->lim.density_floor, p->lim.pressure_floor,
      p->lim.relative_floor, p->cert_list, p->cert_count);
  k_hex_positivity<P, NV><<<p->pos_grid, kThreads, sm, st>>>(p->dev, S, 0, p->hex_tables, p->lim, p->cert_list,
                                                             p->cert_count);
  CK(cudaGetLastError());
  return DGB_OK;
}

// The stage blend dst = alpha * base + beta * x followed by positivity on the sum-factorised path,
// with the blend fused into the certificate pre-pass.
template <int P, int NV>
int run_blend_positivity_hex(dgb_plan* p, const double* base, const double* x, double alpha, double beta, double* dst,
                             cudaStream_t st) {
  const BlockDev& B = p->dev.blk[0];
  if (B.E == 0) return DGB_OK;
  CK(cudaMemsetAsync(p->cert_count, 0, sizeof(int), st));
  k_blend_certify<NV, HexDims<P>::N3><<<blocks_for(B.E, kThreads / 32), kThreads, 0, st>>>(
      base, x, alpha, beta, dst, B.E, p->dev.ph, p->lim.lebesgue, p->lim.density_floor, p->lim.pressure_floor,
      p->lim.relative_floor, p->cert_list, p->cert_count);
  StatePtrs S;
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) S.b[b] = nullptr;
  S.b[0] = dst;
  const size_t sm = sizeof(double) * (size_t)hex_positivity_smem<P, NV>();
  k_hex_positivity<P, NV><<<p->pos_grid, kThreads, sm, st>>>(p->dev, S, 0, p->hex_tables, p->lim, p->cert_list,
                                                             p->cert_count);
  CK(cudaGetLastError());
  return DGB_OK;
}

// Resident CTAs of k_hex_troubled over the whole GPU (set-up; at most one per element).
template <int P, int NV>
int hex_troubled_grid(dgb_plan* p) {
  const size_t sm = sizeof(double) * (size_t)hex_troubled_smem<P, NV>();
  int rc;
  if ((rc = prepare(k_hex_troubled<P, NV>, sm))) return rc;
  int dev = 0, sms = 0, per_sm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hex_troubled<P, NV>, kThreads, sm));
  const long long grid = (long long)std::max(per_sm, 1) * std::max(sms, 1);
  p->trb_grid = (int)std::min<long long>(grid, std::max(p->dev.blk[0].E, 1));
  return DGB_OK;
}

// Troubled-cell detection on the sum-factorised path: the warp pre-pass (k_hex_sensor) settles the
// predicted and the certified elements and lists the rest, which k_hex_troubled tests in full.
template <int P, int NV>
int run_troubled_hex(dgb_plan* p, const StatePtrs& S, double* sensor, uint8_t* flags, const PredictArgs& pa,
                     cudaStream_t st) {
  const size_t sm = sizeof(double) * (size_t)hex_troubled_smem<P, NV>();
  const BlockDev& B = p->dev.blk[0];
  if (B.E == 0) return DGB_OK;
  CK(cudaMemsetAsync(p->cert_count, 0, sizeof(int), st));
  k_hex_sensor<P, NV><<<blocks_for(B.E, kThreads / 32), kThreads, 0, st>>>(p->dev, S, 0, p->hex_tables, p->lim,
                                                                          sensor, flags, pa, p->cert_list,
                                                                          p->cert_count);
  k_hex_troubled<P, NV><<<p->trb_grid, kThreads, sm, st>>>(p->dev, S, 0, p->hex_tables, p->lim, sensor, flags, pa,
                                                           p->cert_list, p->cert_count);
  CK(cudaGetLastError());
  return DGB_OK;
}

template <int NV>
int run_positivity(dgb_plan* p, const StatePtrs& S, cudaStream_t st) {
  int rc;
  if (p->hex) {
    switch (p->dev.degree) {
      case 1: return run_positivity_hex<1, NV>(p, S, st);
      case 2: return run_positivity_hex<2, NV>(p, S, st);
      default: return run_positivity_hex<3, NV>(p, S, st);
    }
  }
  for (int b = 0; b < p->dev.nblocks; ++b) {
    if ((rc = prepare(k_positivity<NV>, p->smem_pos[b]))) return rc;
    k_positivity<NV><<<p->dev.blk[b].E, kThreads, p->smem_pos[b], st>>>(p->dev, S, b, p->lim);
  }
  CK(cudaGetLastError());
  return DGB_OK;
}

template <int NV>
int run_admissibility(dgb_plan* p, const StatePtrs& S, dgb_status* status, int combine, cudaStream_t st) {
  int off = 0;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    k_adm<NV><<<p->adm_grid[b], kThreads, 0, st>>>(p->dev, S, b, p->partials, off);
    off += p->adm_grid[b];
  }
  k_adm_final<<<1, kAdmFinalThreads, 0, st>>>(p->partials, off, p->lim.adm_density_floor, p->lim.adm_pressure_floor, combine,
                                status);
  CK(cudaGetLastError());
  return DGB_OK;
}

template <int NV>
int run_stable_dt(dgb_plan* p, const StatePtrs& S, double cfl, double* dt_out, cudaStream_t st) {
  int off = 0;
  const double cp = p->prm.gamma * p->prm.gas_constant / (p->prm.gamma - 1.0);
  for (int b = 0; b < p->dev.nblocks; ++b) {
    k_rate<NV><<<p->rate_grid[b], kThreads, 0, st>>>(p->dev, S, b, cp, p->partials, off);
    off += p->rate_grid[b];
  }
  k_dt<<<1, kThreads, 0, st>>>(p->partials, off, cfl, dt_out);
  CK(cudaGetLastError());
  return DGB_OK;
}

template <int NV>
int run_troubled(dgb_plan* p, const StatePtrs& S, double* const* sensor, uint8_t* const* flags, cudaStream_t st,
                 bool predicted = false) {
  int rc;
  auto pargs = [&](int b) {
    PredictArgs pa{nullptr, 0, nullptr};
    if (predicted && p->pred_mode) pa = PredictArgs{p->pred_flags[b], p->pred_mode, p->pred_counts};
    return pa;
  };
  if (p->hex) {
    double* so = sensor ? sensor[0] : nullptr;
    uint8_t* fo = flags ? flags[0] : nullptr;
    switch (p->dev.degree) {
      case 1: return run_troubled_hex<1, NV>(p, S, so, fo, pargs(0), st);
      case 2: return run_troubled_hex<2, NV>(p, S, so, fo, pargs(0), st);
      default: return run_troubled_hex<3, NV>(p, S, so, fo, pargs(0), st);
    }
  }
  for (int b = 0; b < p->dev.nblocks; ++b) {
    if ((rc = prepare(k_troubled<NV>, p->smem_troubled[b]))) return rc;
    k_troubled<NV><<<p->dev.blk[b].E, kThreads, p->smem_troubled[b], st>>>(
        p->dev, S, b, p->lim, sensor ? sensor[b] : nullptr, flags ? flags[b] : nullptr, pargs(b));
  }
  CK(cudaGetLastError());
  return DGB_OK;
}

FlagPtrs flag_ptrs(uint8_t* const* f) {
  FlagPtrs out;
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) out.f[b] = f ? f[b] : nullptr;
  return out;
}

// Subcell recompute of the candidate `cand` from the base `cur` (traces of `cur` must be in
// the face buffers): writes `out`.
template <int NV>
int run_subcell(dgb_plan* p, const StatePtrs& cur, double* const* cand, double* const* visc, double dt,
                const FlagPtrs& F, double* const* out, cudaStream_t st) {
  const DevPlan& P = p->dev;
  MoodDev M = p->mood;
  M.recon = p->prm.reconstruction;
  int rc;
  for (int b = 0; b < P.nblocks; ++b) {
    if (P.blk[b].E == 0) continue;
    const SubcellBlockDev& C = M.blk[b];
    const size_t sm = sizeof(double) * ((size_t)P.blk[b].Np * NV + (size_t)C.S * NV * 4 + (size_t)C.NI * NV);
    if ((rc = prepare(k_mood_fv<NV>, sm))) return rc;
    k_mood_fv<NV><<<P.blk[b].E, kThreads, sm, st>>>(P, M, cur, b, F);
  }
  for (int ft = 0; ft < 2; ++ft)
    if (p->face_present[ft])
      k_mood_faces<NV><<<blocks_for((long)P.face[ft].F, kThreads), kThreads, 0, st>>>(P, M, cur, ft, F);
  for (int b = 0; b < P.nblocks; ++b) {
    if (P.blk[b].E == 0) continue;
    const SubcellBlockDev& C = M.blk[b];
    const size_t sm = sizeof(double) * ((size_t)C.S * NV * 2 + (size_t)P.blk[b].Np * NV);
    if ((rc = prepare(k_mood_update<NV>, sm))) return rc;
    k_mood_update<NV><<<P.blk[b].E, kThreads, sm, st>>>(P, M, b, F, cand[b], visc ? visc[b] : nullptr, dt, out[b]);
  }
  CK(cudaGetLastError());
  return DGB_OK;
}

template <int NV>
int run_positivity(dgb_plan* p, const StatePtrs& S, cudaStream_t st);
template <int NV>
int run_troubled(dgb_plan* p, const StatePtrs& S, double* const* sensor, uint8_t* const* flags, cudaStream_t st,
                 bool predicted);
template <int NV>
int run_predict(dgb_plan* p, const StatePtrs& S, cudaStream_t st);
template <int NV>
int run_admissibility(dgb_plan* p, const StatePtrs& S, dgb_status* status, int combine, cudaStream_t st);

// Features of the stage's base state and the predictor's flags (learned MOOD).
template <int NV>
int run_predict(dgb_plan* p, const StatePtrs& S, cudaStream_t st) {
  const DevPlan& P = p->dev;
  constexpr int per = kThreads / 32;                // elements per CTA (one warp each)
  for (int b = 0; b < P.nblocks; ++b) {
    if (p->hex) {
      const int g = blocks_for(P.blk[0].E, per);
      switch (P.degree) {
        case 1: k_hex_elem_stats<1, NV><<<g, kThreads, 0, st>>>(P, S, p->hex_tables, p->pred_stats[0]); break;
        case 2: k_hex_elem_stats<2, NV><<<g, kThreads, 0, st>>>(P, S, p->hex_tables, p->pred_stats[0]); break;
        default: k_hex_elem_stats<3, NV><<<g, kThreads, 0, st>>>(P, S, p->hex_tables, p->pred_stats[0]); break;
      }
      continue;
    }
    const size_t sm = sizeof(double) * 2 * (size_t)P.blk[b].Np * per;
    k_elem_stats<NV><<<blocks_for(P.blk[b].E, per), kThreads, sm, st>>>(P, S, b, p->pred_stats[b]);
  }
  long off = 0;
  for (int b = 0; b < P.nblocks; ++b) {
    float* feat = p->pred_feat + (size_t)off * kMlpIn;
    k_mlp_features<<<blocks_for(P.blk[b].E, kThreads), kThreads, 0, st>>>(P, b, p->pred_stats_dev, feat);
    if (p->pred_w16)
      k_mlp_infer<<<blocks_for(P.blk[b].E, 128), 128, 0, st>>>(p->pred_w16, p->pred_norm, feat, P.blk[b].E,
                                                               p->pred_threshold, nullptr, p->pred_flags[b]);
    off += P.blk[b].E;
  }
  CK(cudaGetLastError());
  return DGB_OK;
}

// MOOD branch of checked_step (hybrid/time_integration.py:450-554)
template <int NV>
int run_step_mood(dgb_plan* p, const StatePtrs& U0, double dt, dgb_status* status, cudaStream_t st) {
  const DevPlan& P = p->dev;
  StatePtrs S1, S2, UNL, EUL;
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) {
    S1.b[b] = p->stage1[b];
    S2.b[b] = p->stage2[b];
    UNL.b[b] = p->unl[b];
    EUL.b[b] = p->eul[b];
  }
  const double alphas[3] = {0.0, 0.75, 1.0 / 3.0};
  const double betas[3] = {1.0, 0.25, 2.0 / 3.0};
  const StatePtrs* cur[3] = {&U0, &S1, &S2};
  const StatePtrs* dst[3] = {&S1, &S2, &U0};
  const FlagPtrs F = flag_ptrs(p->flags);
  // fused hexahedron path with viscous terms: the stage's right-hand side is formed as one
  // residual (one divergence pass per element), and the viscous residual that the subcell scheme
  // needs is formed afterwards for the flagged elements only
  const bool vis_after = p->hex && p->fused && P.viscous;
  int rc;
  for (int s = 0; s < 3; ++s) {
    FinalizeArgs A;
    memset(&A, 0, sizeof(A));
    A.stage = 1;
    A.alpha = alphas[s];
    A.beta = betas[s];
    A.dt = dt;
    for (int b = 0; b < P.nblocks; ++b) {
      A.base[b] = U0.b[b];
      A.dst[b] = p->unl[b];
      A.euler[b] = p->eul[b];
      A.out_vis[b] = vis_after ? nullptr : p->vis[b];
    }
    // the predictor reads the stage's base state: it decides before the high-order update, and
    // in learned mode its elements skip that update (fused hexahedron path): the subcell scheme
    // replaces it and needs only their viscous residual
    if (p->pred_mode && (rc = run_predict<NV>(p, *cur[s], st))) return rc;
    if (p->pred_mode == 1 && p->hex && p->fused) {
      if (vis_after) A.skip = p->pred_flags[0]; else A.skip_inviscid = p->pred_flags[0];
    }
    if ((rc = run_rhs<NV>(p, *cur[s], A, st))) return rc;
    if ((rc = run_troubled<NV>(p, UNL, nullptr, p->flags, st, true))) return rc;
    if (vis_after && (rc = run_viscous_flagged<NV>(p, *cur[s], st))) return rc;
    // the subcell update lands in place in the Euler candidate: elements that are neither
    // troubled nor corrected at a face keep theirs without a copy
    if ((rc = run_subcell<NV>(p, *cur[s], p->eul, p->vis, dt, F, p->eul, st))) return rc;
    if ((rc = run_positivity<NV>(p, EUL, st))) return rc;
    if (p->hex) {
      rc = p->dev.degree == 1 ? run_blend_positivity_hex<1, NV>(p, U0.b[0], p->eul[0], alphas[s], betas[s], dst[s]->b[0], st)
         : p->dev.degree == 2 ? run_blend_positivity_hex<2, NV>(p, U0.b[0], p->eul[0], alphas[s], betas[s], dst[s]->b[0], st)
                              : run_blend_positivity_hex<3, NV>(p, U0.b[0], p->eul[0], alphas[s], betas[s], dst[s]->b[0], st);
      if (rc) return rc;
    } else {
      for (int b = 0; b < P.nblocks; ++b) {
        const size_t n = (size_t)P.blk[b].E * P.blk[b].Np * NV;
        k_blend<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(U0.b[b], p->eul[b], alphas[s], betas[s], dst[s]->b[b], n);
      }
      if ((rc = run_positivity<NV>(p, *dst[s], st))) return rc;
    }
    if ((rc = run_admissibility<NV>(p, *dst[s], status, 0, st))) return rc;
  }
  return DGB_OK;
}

template <int NV>
int run_step(dgb_plan* p, const StatePtrs& U0, double dt, dgb_status* status, cudaStream_t st) {
  if (p->prm.limiter == 2) return run_step_mood<NV>(p, U0, dt, status, st);
  const DevPlan& P = p->dev;
  StatePtrs S1, S2;
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) {
    S1.b[b] = p->stage1[b];
    S2.b[b] = p->stage2[b];
  }
  const double alphas[3] = {0.0, 0.75, 1.0 / 3.0};
  const double betas[3] = {1.0, 0.25, 2.0 / 3.0};
  const StatePtrs* cur[3] = {&U0, &S1, &S2};
  const StatePtrs* dst[3] = {&S1, &S2, &U0};
  int rc;
  for (int s = 0; s < 3; ++s) {
    FinalizeArgs A;
    memset(&A, 0, sizeof(A));
    A.stage = 1;
    A.alpha = alphas[s];
    A.beta = betas[s];
    A.dt = dt;
    for (int b = 0; b < P.nblocks; ++b) {
      A.base[b] = U0.b[b];
      A.dst[b] = dst[s]->b[b];
    }
    if ((rc = run_rhs<NV>(p, *cur[s], A, st))) return rc;
    if (p->prm.limiter == 1 && (rc = run_positivity<NV>(p, *dst[s], st))) return rc;
    if ((rc = run_admissibility<NV>(p, *dst[s], status, s > 0, st))) return rc;
  }
  return DGB_OK;
}

int ensure_predictor_buffers(dgb_plan* p) {
  if (p->pred_feat) return DGB_OK;
  long total = 0;
  double* d;
  int rc;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    const int E = p->dev.blk[b].E;
    if ((rc = alloc(p, ((size_t)E * kMlpStats + 1) / 2, &d))) return rc;
    p->pred_stats[b] = reinterpret_cast<float*>(d);
    if ((rc = alloc(p, ((size_t)E + 7) / 8, &d))) return rc;
    p->pred_flags[b] = reinterpret_cast<uint8_t*>(d);
    total += E;
  }
  if ((rc = alloc(p, ((size_t)total * kMlpIn + 1) / 2, &d))) return rc;
  p->pred_feat = reinterpret_cast<float*>(d);
  if ((rc = alloc(p, DGB_MAX_BLOCKS, &d))) return rc;
  p->pred_stats_dev = reinterpret_cast<float**>(d);
  CK(cudaMemcpy(p->pred_stats_dev, p->pred_stats, sizeof(p->pred_stats), cudaMemcpyHostToDevice));
  if ((rc = alloc(p, 8, &d))) return rc;
  p->pred_counts = reinterpret_cast<unsigned long long*>(d);
  return DGB_OK;
}

int check_ready(dgb_plan* p) {
  if (!p) return fail(DGB_ERR_ARGUMENT, "null plan");
  if (!p->finalized) return fail(DGB_ERR_ARGUMENT, "plan not finalized");
  return DGB_OK;
}

int check_state(dgb_plan* p, const dgb_state* s, const char* what) {
  if (!s) return fail(DGB_ERR_ARGUMENT, std::string(what) + " is null");
  for (int b = 0; b < p->dev.nblocks; ++b)
    if (!s->block[b]) return fail(DGB_ERR_ARGUMENT, std::string(what) + ": null block pointer");
  return DGB_OK;
}

}  // namespace

namespace {
template <int NV>
int run_subcell_api(dgb_plan* p, const dgb_state* base, const dgb_state* cand, double dt, const dgb_state* arhs,
                    uint8_t* const* troubled, const dgb_state* out, cudaStream_t st) {
  // traces of the base state for the DG face flux (the RHS's first stage only)
  const DevPlan& P = p->dev;
  const StatePtrs S = to_ptrs(base);
  int rc;
  if (p->hex) {
    switch (P.degree) {
      case 1: {
        const size_t sm = sizeof(double) * (size_t)HexSmem<1, NV>::TRACES;
        if ((rc = prepare(k_hex_traces<1, NV>, sm))) return rc;
        k_hex_traces<1, NV><<<P.blk[0].E, kThreads, sm, st>>>(P, S, 0, p->hex_tables, p->hex_codes);
        break;
      }
      case 2: {
        const size_t sm = sizeof(double) * (size_t)HexSmem<2, NV>::TRACES;
        if ((rc = prepare(k_hex_traces<2, NV>, sm))) return rc;
        k_hex_traces<2, NV><<<P.blk[0].E, kThreads, sm, st>>>(P, S, 0, p->hex_tables, p->hex_codes);
        break;
      }
      default: {
        const size_t sm = sizeof(double) * (size_t)HexSmem<3, NV>::TRACES;
        if ((rc = prepare(k_hex_traces<3, NV>, sm))) return rc;
        k_hex_traces<3, NV><<<P.blk[0].E, kThreads, sm, st>>>(P, S, 0, p->hex_tables, p->hex_codes);
      }
    }
  } else {
    // the subcell scheme's DG face flux takes float64 traces in either precision mode
    if ((rc = prepare(k_traces<NV, double>, p->smem_tr64))) return rc;
    k_traces<NV, double><<<p->launch_tr64.cta0[P.nblocks], kThreads, p->smem_tr64, st>>>(P, S, p->launch_tr64);
  }
  double* candp[DGB_MAX_BLOCKS] = {cand->block[0], cand->block[1], cand->block[2]};
  double* visp[DGB_MAX_BLOCKS] = {arhs ? arhs->block[0] : nullptr, arhs ? arhs->block[1] : nullptr,
                                  arhs ? arhs->block[2] : nullptr};
  double* outp[DGB_MAX_BLOCKS] = {out->block[0], out->block[1], out->block[2]};
  return run_subcell<NV>(p, S, candp, arhs ? visp : nullptr, dt, flag_ptrs(troubled), outp, st);
}

}  // namespace

static void set_params(dgb_plan* p, const dgb_params* prm);

extern "C" {

const char* dgb_last_error(void) { return g_error.c_str(); }

int dgb_version(void) { return 1; }

int dgb_plan_create(const dgb_params* prm, dgb_plan** out) {
  if (!prm || !out) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (prm->degree < 1 || prm->degree > 3) return fail(DGB_ERR_ARGUMENT, "Only P1, P2, and P3 are currently implemented");
  if (prm->nvars != 5 && prm->nvars != 16) return fail(DGB_ERR_UNSUPPORTED, "nvars must be 5 or 16");
  if (prm->num_blocks < 1 || prm->num_blocks > DGB_MAX_BLOCKS) return fail(DGB_ERR_ARGUMENT, "num_blocks out of range");
  if (prm->precision != 0 && prm->precision != 1) return fail(DGB_ERR_ARGUMENT, "precision must be 0 or 1");
  if (prm->n_inlet > DGB_MAX_TAGS || prm->n_wall > DGB_MAX_TAGS || prm->n_no_slip > DGB_MAX_TAGS ||
      prm->n_slip > DGB_MAX_TAGS)
    return fail(DGB_ERR_ARGUMENT, "too many boundary tags");
  dgb_plan* p = new dgb_plan();
  memset(&p->dev, 0, sizeof(p->dev));
  p->dev.nv = prm->nvars;
  p->dev.nblocks = prm->num_blocks;
  p->dev.viscous = prm->viscous;
  p->dev.degree = prm->degree;
  set_params(p, prm);
  *out = p;
  return DGB_OK;
}

int dgb_plan_update_params(dgb_plan* p, const dgb_params* prm) {
  if (p) ++p->generation;    // invalidates a captured step
  if (!p || !prm) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (prm->degree != p->dev.degree || prm->nvars != p->dev.nv || prm->num_blocks != p->dev.nblocks ||
      prm->viscous != p->dev.viscous || prm->precision != p->prm.precision)
    return fail(DGB_ERR_ARGUMENT, "degree, nvars, blocks, viscous flag and precision are fixed for a plan");
  if (prm->n_inlet > DGB_MAX_TAGS || prm->n_wall > DGB_MAX_TAGS || prm->n_no_slip > DGB_MAX_TAGS ||
      prm->n_slip > DGB_MAX_TAGS)
    return fail(DGB_ERR_ARGUMENT, "too many boundary tags");
  set_params(p, prm);
  return DGB_OK;
}

}  // extern "C"

static void set_params(dgb_plan* p, const dgb_params* prm) {
  p->prm = *prm;
  Physics& ph = p->dev.ph;
  ph.gamma = prm->gamma;
  ph.R = prm->gas_constant;
  ph.mu = prm->dynamic_viscosity;
  ph.kappa = prm->thermal_conductivity;
  ph.br2 = prm->br2_penalty;
  ph.has_boundary = prm->has_boundary;
  for (int v = 0; v < DGB_MAX_VARS; ++v) ph.farfield_W[v] = prm->farfield_primitive[v];
  ph.n_inlet = prm->n_inlet;
  ph.n_wall = prm->n_wall;
  ph.n_no_slip = prm->n_no_slip;
  ph.n_slip = prm->n_slip;
  for (int k = 0; k < DGB_MAX_TAGS; ++k) {
    ph.inlet[k] = prm->inlet_tags[k];
    ph.wall[k] = prm->wall_tags[k];
    ph.no_slip[k] = prm->no_slip_tags[k];
    ph.slip[k] = prm->slip_tags[k];
  }
  ph.has_wall_T = prm->has_wall_temperature;
  ph.wall_T = prm->wall_temperature;
  p->lim.density_floor = prm->pos_density_floor;
  p->lim.pressure_floor = prm->pos_pressure_floor;
  p->lim.relative_floor = prm->pos_relative_floor;
  p->lim.adm_density_floor = prm->adm_density_floor;
  p->lim.adm_pressure_floor = prm->adm_pressure_floor;
  p->lim.sensor_threshold = prm->sensor_threshold;
}

extern "C" {

int dgb_plan_set_block(dgb_plan* p, int b, const dgb_block_desc* d) {
  if (!p || !d || b < 0 || b >= p->dev.nblocks) return fail(DGB_ERR_ARGUMENT, "bad block argument");
  if (p->finalized) return fail(DGB_ERR_ARGUMENT, "plan already finalized");
  BlockDev& B = p->dev.blk[b];
  B.type = d->element_type;
  B.E = d->num_elements;
  B.Np = d->num_nodes;
  B.Nq = d->num_qp;
  B.nlf = d->num_local_faces;
  B.Ns = d->num_face_samples;
  const size_t E = B.E, Np = B.Np, Nq = B.Nq;
  int rc;
  if ((rc = upload(p, d->basis, Nq * Np, &B.B))) return rc;
  if ((rc = upload(p, d->basis_grad, Nq * Np * 3, &B.dB))) return rc;
  if (d->basis && d->basis_grad) {
    std::vector<double> bt(Nq * Np), dq(Nq * Np * 3), di(Nq * Np * 3);
    for (size_t q = 0; q < Nq; ++q)
      for (size_t i = 0; i < Np; ++i) {
        bt[i * Nq + q] = d->basis[q * Np + i];
        for (size_t r = 0; r < 3; ++r) {
          const double g = d->basis_grad[(q * Np + i) * 3 + r];
          dq[(i * 3 + r) * Nq + q] = g;
          di[(q * 3 + r) * Np + i] = g;
        }
      }
    if ((rc = upload(p, bt.data(), bt.size(), &B.Bt))) return rc;
    if ((rc = upload(p, dq.data(), dq.size(), &B.dBq))) return rc;
    if ((rc = upload(p, di.data(), di.size(), &B.dBi))) return rc;
  }
  // Lebesgue constant of the limiter's sample set (nodes, volume points, face samples)
  B.lebesgue = 1.0;
  for (int tbl = 0; tbl < 2; ++tbl) {
    const double* rows = tbl == 0 ? d->basis : d->face_sample_basis;
    const size_t nrows = tbl == 0 ? Nq : (size_t)B.Ns;
    if (!rows) continue;
    for (size_t r = 0; r < nrows; ++r) {
      double a = 0.0;
      for (size_t i = 0; i < Np; ++i) a += fabs(rows[r * Np + i]);
      B.lebesgue = fmax(B.lebesgue, a);
    }
  }
  if ((rc = upload(p, d->inv_jacobian, E * Nq * 9, &B.jinv))) return rc;
  if ((rc = upload(p, d->wdet, E * Nq, &B.wdet))) return rc;
  // the inverse mass matrices may instead be built on the device (dgb_plan_build_inverse_mass)
  B.minv = nullptr;
  if (d->inv_mass && (rc = upload(p, d->inv_mass, E * Np * Np, &B.minv))) return rc;
  if ((rc = upload(p, d->length, E, &B.length))) return rc;
  if ((rc = upload(p, d->face_sample_basis, (size_t)B.Ns * Np, &B.fsB))) return rc;
  if ((rc = upload(p, d->p1_projector, Np * Np, &B.p1proj))) return rc;
  if ((rc = upload(p, d->elem_face, E * B.nlf, &B.elem_face))) return rc;
  p->block_set[b] = true;
  return DGB_OK;
}

int dgb_plan_set_faces(dgb_plan* p, const dgb_face_desc* d) {
  if (!p || !d || d->face_type < 0 || d->face_type > 1) return fail(DGB_ERR_ARGUMENT, "bad face argument");
  if (p->finalized) return fail(DGB_ERR_ARGUMENT, "plan already finalized");
  FaceDev& F = p->dev.face[d->face_type];
  F.F = d->num_faces;
  F.nq = d->num_qp;
  const size_t n = F.F, nq = F.nq;
  int rc;
  if ((rc = upload(p, d->owner_block, n, &F.ob))) return rc;
  if ((rc = upload(p, d->owner_local, n, &F.ol))) return rc;
  if ((rc = upload(p, d->owner_code, n, &F.oc))) return rc;
  if ((rc = upload(p, d->nbr_block, n, &F.nb))) return rc;
  if ((rc = upload(p, d->nbr_local, n, &F.nl))) return rc;
  if ((rc = upload(p, d->nbr_code, n, &F.nc))) return rc;
  if ((rc = upload(p, d->tags, n, &F.tag))) return rc;
  if ((rc = upload(p, d->normals, n * nq * 3, &F.n))) return rc;
  if ((rc = upload(p, d->weights, n * nq, &F.w))) return rc;
  if ((rc = upload(p, d->side_inv_jacobian, n * 2 * nq * 9, &F.jinv))) return rc;
  p->face_present[d->face_type] = n > 0;
  return DGB_OK;
}

int dgb_plan_set_trace(dgb_plan* p, int etype, int ftype, int ncodes, int nq, int np, const double* B,
                       const double* dB) {
  if (!p || ftype < 0 || ftype > 1) return fail(DGB_ERR_ARGUMENT, "bad trace argument");
  int found = 0;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    BlockDev& blk = p->dev.blk[b];
    if (!p->block_set[b] || blk.type != etype) continue;
    if (blk.Np != np) return fail(DGB_ERR_ARGUMENT, "trace table node count mismatch");
    int rc;
    if ((rc = upload(p, B, (size_t)ncodes * nq * np, &blk.trB[ftype]))) return rc;
    if ((rc = upload(p, dB, (size_t)ncodes * nq * np * 3, &blk.trdB[ftype]))) return rc;
    if (B && dB) {
      std::vector<double> bt((size_t)ncodes * nq * np), dt((size_t)ncodes * nq * np * 3);
      for (size_t c = 0; c < (size_t)ncodes; ++c)
        for (size_t q = 0; q < (size_t)nq; ++q)
          for (size_t i = 0; i < (size_t)np; ++i) {
            bt[(c * np + i) * nq + q] = B[(c * nq + q) * np + i];
            for (size_t r = 0; r < 3; ++r) dt[((c * np + i) * 3 + r) * nq + q] = dB[((c * nq + q) * np + i) * 3 + r];
          }
      if ((rc = upload(p, bt.data(), bt.size(), &blk.trBt[ftype]))) return rc;
      if ((rc = upload(p, dt.data(), dt.size(), &blk.trdBt[ftype]))) return rc;
    }
    found = 1;
  }
  if (!found) return fail(DGB_ERR_ARGUMENT, "trace table for an element type without a block");
  return DGB_OK;
}

int dgb_plan_set_hex(dgb_plan* p, const double* line_tables, const int32_t* lex2node, int num_codes, int face_points,
                     const uint8_t* perm) {
  if (!p || !line_tables || !lex2node || !perm) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (p->finalized) return fail(DGB_ERR_ARGUMENT, "plan already finalized");
  if (p->dev.nblocks != 1 || !p->block_set[0] || p->dev.blk[0].type != 0)
    return fail(DGB_ERR_UNSUPPORTED, "the sum-factorised path needs exactly one hexahedron block");
  const int qf = p->dev.degree == 1 ? 2 : (p->dev.degree == 2 ? 3 : 4);
  if (face_points != qf * qf) return fail(DGB_ERR_ARGUMENT, "face point count does not match the degree");
  HexTables& t = p->hex_tables;
  memset(&t, 0, sizeof(t));
  const double* src = line_tables;
  memcpy(t.bq, src, sizeof(t.bq)); src += 20;
  memcpy(t.dq, src, sizeof(t.dq)); src += 20;
  memcpy(t.bqT, src, sizeof(t.bqT)); src += 20;
  memcpy(t.dqT, src, sizeof(t.dqT)); src += 20;
  memcpy(t.bf, src, sizeof(t.bf)); src += 16;
  memcpy(t.df, src, sizeof(t.df)); src += 16;
  memcpy(t.bfT, src, sizeof(t.bfT)); src += 16;
  memcpy(t.d0, src, sizeof(t.d0)); src += 4;
  memcpy(t.d1, src, sizeof(t.d1)); src += 4;
  memcpy(t.m1i, src, sizeof(t.m1i)); src += 16;
  memcpy(t.w1, src, sizeof(t.w1)); src += 5;
  memcpy(t.p1d, src, sizeof(t.p1d)); src += 16;
  for (int i = 0; i < 64; ++i) t.lex2node[i] = lex2node[i];
  // Lebesgue constant of the limiter's samples: a volume point is a product of three 1-D rows of
  // bq, a face point of two rows of bf (its third coordinate is a node), a node gives 1
  {
    const int N = p->dev.degree + 1, Q = p->dev.degree == 1 ? 2 : (p->dev.degree == 2 ? 3 : 5);
    double lq = 0.0, lf = 0.0;
    for (int q = 0; q < Q; ++q) {
      double a = 0.0;
      for (int j = 0; j < N; ++j) a += fabs(t.bq[q * N + j]);   // [Q][N], packed
      lq = fmax(lq, a);
    }
    for (int q = 0; q < qf; ++q) {
      double a = 0.0;
      for (int j = 0; j < N; ++j) a += fabs(t.bf[q * N + j]);   // [QF][N], packed
      lf = fmax(lf, a);
    }
    p->lim.lebesgue = fmax(1.0, fmax(lq * lq * lq, lf * lf));
  }
  int rc;
  if ((rc = upload(p, perm, (size_t)num_codes * face_points, &p->hex_codes.perm))) return rc;
  p->hex = true;
  return DGB_OK;
}

int dgb_plan_set_hex_affine(dgb_plan* p, const uint8_t* affine, const double* coef, const double* jinv,
                            const double* det) {
  if (!p || !affine || !coef || !jinv || !det) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (p->finalized) return fail(DGB_ERR_ARGUMENT, "plan already finalized");
  if (!p->hex) return fail(DGB_ERR_ARGUMENT, "call dgb_plan_set_hex first");
  BlockDev& B = p->dev.blk[0];
  if (B.wref) return fail(DGB_ERR_ARGUMENT, "block 0 already has dense affine data");
  int rc;
  if ((rc = upload(p, affine, (size_t)B.E, &B.affine))) return rc;
  if ((rc = upload(p, coef, (size_t)B.E, &B.acoef))) return rc;
  if ((rc = upload(p, jinv, (size_t)B.E * 9, &B.ajinv))) return rc;
  if ((rc = upload(p, det, (size_t)B.E, &B.adet))) return rc;
  return DGB_OK;
}

// Inverse mass matrices, one element per CTA (plan set-up; hybrid/geometry.py:181-192):
// M_e = B^T diag(w|J|) B is formed in shared memory, each entry summed over the volume points in
// order and mirrored so that M_e is exactly symmetric, inverted in place (gauss_jordan_spd; a
// matrix that is not positive definite marks the element in *bad) and scaled by the sliver
// factor min(1, V/1e-4).  Shared memory: (Np^2 + Nq + 2 Np) doubles.
__global__ void __launch_bounds__(256) k_inverse_mass(const double* __restrict__ B, const double* __restrict__ wdet,
                                                      const double* __restrict__ volume, int Np, int Nq,
                                                      int transposed, double* __restrict__ minv, int* bad) {
  extern __shared__ double sm[];
  double* A = sm;
  double* w = A + Np * Np;
  double* rk = w + Nq;
  double* ck = rk + Np;
  const size_t e = blockIdx.x;
  for (int q = threadIdx.x; q < Nq; q += blockDim.x) w[q] = wdet[e * Nq + q];
  __syncthreads();
  for (int idx = threadIdx.x; idx < Np * Np; idx += blockDim.x) {
    const int i = idx / Np, j = idx % Np;
    if (i > j) continue;
    double s = 0.0;
    for (int q = 0; q < Nq; ++q) s += w[q] * B[q * Np + i] * B[q * Np + j];
    A[i * Np + j] = s;
    A[j * Np + i] = s;
  }
  if (!gauss_jordan_spd(A, Np, rk, ck)) {
    if (threadIdx.x == 0) *bad = (int)e + 1;
    return;
  }
  const double scale = fmin(1.0, volume[e] / 1.0e-4);
  double* out = minv + e * Np * Np;
  for (int idx = threadIdx.x; idx < Np * Np; idx += blockDim.x) {
    const int i = idx / Np, j = idx % Np;
    out[transposed ? j * Np + i : idx] = scale * A[idx];
  }
}

// In-place inverses of a batch of SPD matrices, one per CTA (set-up).
__global__ void __launch_bounds__(256) k_spd_inverse(double* __restrict__ mats, int n, int* bad) {
  extern __shared__ double sm[];
  double* A = sm;
  double* rk = A + n * n;
  double* ck = rk + n;
  double* m = mats + (size_t)blockIdx.x * n * n;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) A[idx] = m[idx];
  if (!gauss_jordan_spd(A, n, rk, ck)) {
    if (threadIdx.x == 0) *bad = (int)blockIdx.x + 1;
    return;
  }
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) m[idx] = A[idx];
}

int dgb_spd_inverse(double* matrices, int n, int count, int* status, void* stream) {
  if (!matrices || !status || n < 1 || count < 0) return fail(DGB_ERR_ARGUMENT, "bad SPD-inverse argument");
  const size_t smem = sizeof(double) * ((size_t)n * n + 2 * n);
  if (smem > 200 * 1024) return fail(DGB_ERR_ARGUMENT, "matrix too large for the SPD-inverse kernel");
  if (count == 0) return DGB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CK(cudaFuncSetAttribute(k_spd_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaMemsetAsync(status, 0, sizeof(int), st));
  k_spd_inverse<<<count, 256, smem, st>>>(matrices, n, status);
  CK(cudaGetLastError());
  return DGB_OK;
}

int dgb_plan_build_inverse_mass(dgb_plan* p, int b, const double* volume, int transposed) {
  if (!p || b < 0 || b >= p->dev.nblocks || !volume) return fail(DGB_ERR_ARGUMENT, "bad inverse-mass argument");
  if (p->finalized) return fail(DGB_ERR_ARGUMENT, "plan already finalized");
  if (!p->block_set[b]) return fail(DGB_ERR_ARGUMENT, "call dgb_plan_set_block first");
  BlockDev& B = p->dev.blk[b];
  if (B.minv) return fail(DGB_ERR_ARGUMENT, "block already has inverse mass matrices");
  if (B.E == 0) return DGB_OK;
  if (!B.B || !B.wdet) return fail(DGB_ERR_ARGUMENT, "block needs its basis and w|J| tables");
  const size_t smem = sizeof(double) * ((size_t)B.Np * B.Np + B.Nq + 2 * B.Np);
  if (smem > 200 * 1024) return fail(DGB_ERR_ARGUMENT, "element too large for the inverse-mass kernel");
  int rc;
  const double* vol = nullptr;
  if ((rc = upload(p, volume, (size_t)B.E, &vol))) return rc;
  double* out = nullptr;
  if ((rc = alloc(p, (size_t)B.E * B.Np * B.Np, &out))) return rc;
  int* bad = nullptr;
  CK(cudaMalloc(&bad, sizeof(int)));
  int h_bad = 0;
  cudaError_t err = cudaMemset(bad, 0, sizeof(int));
  if (err == cudaSuccess) err = cudaFuncSetAttribute(k_inverse_mass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err == cudaSuccess) {
    k_inverse_mass<<<B.E, 256, smem>>>(B.B, B.wdet, vol, B.Np, B.Nq, transposed, out, bad);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMemcpy(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, cudaGetErrorString(err));
  if (h_bad) return fail(DGB_ERR_ARGUMENT, "degenerate element: its mass matrix is not positive definite");
  B.minv = out;
  return DGB_OK;
}

int dgb_plan_set_block_affine(dgb_plan* p, int b, const uint8_t* affine, const double* coef, const double* jinv,
                              const double* det, const double* ref_weights, const double* ref_inv_mass) {
  if (!p || b < 0 || b >= p->dev.nblocks || !affine || !coef || !jinv || !det || !ref_weights || !ref_inv_mass)
    return fail(DGB_ERR_ARGUMENT, "bad block-affine argument");
  if (p->finalized) return fail(DGB_ERR_ARGUMENT, "plan already finalized");
  if (!p->block_set[b]) return fail(DGB_ERR_ARGUMENT, "call dgb_plan_set_block first");
  if (p->hex) return fail(DGB_ERR_ARGUMENT, "the sum-factorised path takes dgb_plan_set_hex_affine");
  BlockDev& B = p->dev.blk[b];
  int rc;
  if ((rc = upload(p, affine, (size_t)B.E, &B.affine))) return rc;
  if ((rc = upload(p, coef, (size_t)B.E, &B.acoef))) return rc;
  if ((rc = upload(p, jinv, (size_t)B.E * 9, &B.ajinv))) return rc;
  if ((rc = upload(p, det, (size_t)B.E, &B.adet))) return rc;
  if ((rc = upload(p, ref_weights, (size_t)B.Nq, &B.wref))) return rc;
  if ((rc = upload(p, ref_inv_mass, (size_t)B.Np * B.Np, &B.mref_inv))) return rc;
  return DGB_OK;
}

int dgb_plan_set_cases(dgb_plan* p, int num_cases, const double* cases, const int32_t* const* element_case) {
  if (!p || num_cases < 1 || !cases || !element_case) return fail(DGB_ERR_ARGUMENT, "bad case argument");
  const int stride = 3 + p->dev.nv;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    if (!p->block_set[b]) return fail(DGB_ERR_ARGUMENT, "call dgb_plan_set_block first");
    if (!element_case[b] && p->dev.blk[b].E > 0) return fail(DGB_ERR_ARGUMENT, "null element case array");
    for (int e = 0; e < p->dev.blk[b].E; ++e)
      if (element_case[b][e] < 0 || element_case[b][e] >= num_cases)
        return fail(DGB_ERR_ARGUMENT, "element case id out of range");
  }
  for (int c = 0; c < num_cases; ++c)
    if (!(cases[(size_t)c * stride] >= 0.0) || !(cases[(size_t)c * stride + 1] >= 0.0))
      return fail(DGB_ERR_ARGUMENT, "case viscosity and conductivity must be >= 0");
  int rc;
  const double* table = nullptr;
  if ((rc = upload(p, cases, (size_t)num_cases * stride, &table))) return rc;
  for (int b = 0; b < p->dev.nblocks; ++b)
    if ((rc = upload(p, element_case[b], (size_t)p->dev.blk[b].E, &p->dev.blk[b].ecase))) return rc;
  p->dev.ph.cases = table;
  p->dev.ph.case_stride = stride;
  p->num_cases = num_cases;
  ++p->generation;
  return DGB_OK;
}

int dgb_plan_finalize(dgb_plan* p) {
  if (!p) return fail(DGB_ERR_ARGUMENT, "null plan");
  const int NV = p->dev.nv;
  int rc;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    if (!p->block_set[b]) return fail(DGB_ERR_ARGUMENT, "block descriptor missing");
    if (!p->dev.blk[b].minv && p->dev.blk[b].E > 0)
      return fail(DGB_ERR_ARGUMENT, "block without inverse mass matrices: pass inv_mass or call "
                                    "dgb_plan_build_inverse_mass");
  }
  for (int ft = 0; ft < 2; ++ft) {
    FaceDev& F = p->dev.face[ft];
    if (!p->face_present[ft]) continue;
    const size_t n = F.F, nq = F.nq;
    if ((rc = alloc(p, n * 2 * nq * NV, &F.trA))) return rc;
    if ((rc = alloc(p, n * 2 * nq * NV, &F.fluxI))) return rc;
    if ((rc = alloc(p, n * 2 * NV, &F.anc))) return rc;
    if (p->dev.viscous) {
      F.trP = F.trA;   // the viscous terms take the anchor-form trace (equal to the plain one)
      if ((rc = alloc(p, n * 2 * nq * 4, &F.trV))) return rc;
      if ((rc = alloc(p, n * 2 * nq * 12, &F.trG))) return rc;
      if ((rc = alloc(p, n * nq * 12, &F.jumpW))) return rc;
      if ((rc = alloc(p, n * 2 * nq * 12, &F.liftF))) return rc;
      if ((rc = alloc(p, n * nq * NV, &F.fluxV))) return rc;
    }
  }
  if (p->hex && p->dev.blk[0].E > 0) {
    CK(cudaMalloc(&p->cert_list, sizeof(int) * (size_t)p->dev.blk[0].E));
    p->allocations.push_back(p->cert_list);
    CK(cudaMalloc(&p->cert_count, sizeof(int)));
    p->allocations.push_back(p->cert_count);
    const int deg = p->dev.degree;
    rc = NV == 5 ? (deg == 1 ? hex_positivity_grid<1, 5>(p) : deg == 2 ? hex_positivity_grid<2, 5>(p)
                                                              : hex_positivity_grid<3, 5>(p))
                 : (deg == 1 ? hex_positivity_grid<1, 16>(p) : deg == 2 ? hex_positivity_grid<2, 16>(p)
                                                               : hex_positivity_grid<3, 16>(p));
    if (rc) return rc;
    rc = NV == 5 ? (deg == 1 ? hex_troubled_grid<1, 5>(p) : deg == 2 ? hex_troubled_grid<2, 5>(p)
                                                             : hex_troubled_grid<3, 5>(p))
                 : (deg == 1 ? hex_troubled_grid<1, 16>(p) : deg == 2 ? hex_troubled_grid<2, 16>(p)
                                                              : hex_troubled_grid<3, 16>(p));
    if (rc) return rc;
  }
  p->npartials = 0;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    BlockDev& B = p->dev.blk[b];
    for (int ft = 0; ft < 2; ++ft) {
      // every face type this block touches needs its trace table
      (void)ft;
    }
    const size_t state = (size_t)B.E * B.Np * NV;
    if ((rc = alloc(p, state, &B.Rinv))) return rc;
    if ((rc = alloc(p, p->dev.viscous ? state : 1, &B.Rvis))) return rc;
    if ((rc = alloc(p, state, &p->stage1[b]))) return rc;
    if ((rc = alloc(p, state, &p->stage2[b]))) return rc;
    int max_nq = 0;
    for (int ft = 0; ft < 2; ++ft)
      if (p->face_present[ft] && p->dev.face[ft].nq > max_nq) max_nq = p->dev.face[ft].nq;
    (void)max_nq;
    p->smem_pos[b] = sizeof(double) * (size_t)(B.Np + B.Np + B.Nq + B.Ns) * NV;
    p->smem_troubled[b] = sizeof(double) * ((size_t)(B.Np + B.Np + B.Nq + B.Ns) * NV + 2 * B.Np);
    p->rate_grid[b] = blocks_for(B.E, kThreads / 32) < 2 * 148 * 8 ? blocks_for(B.E, kThreads / 32) : 2 * 148 * 8;
    const long nodes = (long)B.E * B.Np;
    p->adm_grid[b] = blocks_for(nodes, kThreads) < 148 * 8 ? blocks_for(nodes, kThreads) : 148 * 8;
    p->npartials += (p->rate_grid[b] > p->adm_grid[b] ? p->rate_grid[b] : p->adm_grid[b]);
    if (p->smem_pos[b] > 227 * 1024)
      return fail(DGB_ERR_UNSUPPORTED, "element too large for the shared-memory kernels");
  }
  if (!p->hex) {
    const size_t rs = p->prm.precision == 1 ? sizeof(float) : sizeof(double);
    p->smem_tr = dense_smem(p, p->launch_tr, traces_kind, rs);
    p->smem_vol = dense_smem(p, p->launch_vol, volume_kind, rs);
    p->smem_fin = dense_smem(p, p->launch_fin, finalize_kind, rs);
    p->smem_tr64 = dense_smem(p, p->launch_tr64, traces_kind, sizeof(double));
    if (p->smem_tr > 227 * 1024 || p->smem_vol > 227 * 1024 || p->smem_fin > 227 * 1024)
      return fail(DGB_ERR_UNSUPPORTED, "element too large for the shared-memory kernels");
  }
  {
    void* d = nullptr;
    CK(cudaMalloc(&d, sizeof(Partial) * (size_t)(p->npartials + 1)));
    p->allocations.push_back(d);
    p->partials = static_cast<Partial*>(d);
  }
  if ((rc = alloc(p, 1, &p->dt_scratch))) return rc;
  {
    double* d;
    if ((rc = alloc(p, 1, &d))) return rc;
    p->dev_err = reinterpret_cast<int*>(d);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, dev));
  }
  if (p->hex && p->dev.viscous)
    if ((rc = alloc(p, (size_t)p->dev.blk[0].E * 12 * p->dev.blk[0].Np, &p->hex_lift))) return rc;
  if (p->hex && p->dev.viscous && p->dev.blk[0].E > 0 && p->face_present[1]) {
    if ((rc = build_hex_face_tables(p))) return rc;
  }
  if (p->hex && p->prm.precision == 1) {
    // float32 copies of the inverse mass matrices and the per-point inverse Jacobians that the
    // mixed-precision hexahedron kernels read (half the bytes of the float64 tables)
    BlockDev& B = p->dev.blk[0];
    float* f;
    if ((rc = to_float32(p, B.minv, (size_t)B.E * B.Np * B.Np, &f))) return rc;
    B.minv32 = f;
    if ((rc = to_float32(p, B.jinv, (size_t)B.E * B.Nq * 9, &f))) return rc;
    B.jinv32 = f;
    FaceDev& F = p->dev.face[1];
    if (p->face_present[1]) {
      if ((rc = to_float32(p, F.jinv, (size_t)F.F * 2 * F.nq * 9, &f))) return rc;
      F.jinv32 = f;
      {
        double* d;
        if ((rc = alloc(p, ((size_t)F.F * 2 * F.nq * p->dev.nv + 1) / 2, &d))) return rc;
        F.fluxI32 = reinterpret_cast<float*>(d);
      }
      if (p->dev.viscous) {
        double* d;
        if ((rc = alloc(p, ((size_t)F.F * F.nq * p->dev.nv + 1) / 2, &d))) return rc;
        F.fluxV32 = reinterpret_cast<float*>(d);
        if ((rc = alloc(p, (size_t)F.F * F.nq * 6, &d))) return rc;
        F.jumpW32 = reinterpret_cast<float*>(d);
        if ((rc = alloc(p, ((size_t)F.F * 2 * F.nq * 4 + 1) / 2, &d))) return rc;
        F.trV32 = reinterpret_cast<float*>(d);
        if ((rc = alloc(p, (size_t)F.F * 2 * F.nq * 6, &d))) return rc;
        F.trG32 = reinterpret_cast<float*>(d);
      }
    }
  }
  p->finalized = true;
  return DGB_OK;
}

int dgb_plan_set_fused(dgb_plan* p, int enable) {
  if (!p) return fail(DGB_ERR_ARGUMENT, "null plan");
  if (enable && p->finalized && p->hex && p->dev.viscous && !p->hex_face.face_lf && p->face_present[1])
    return fail(DGB_ERR_ARGUMENT, "fused tables missing");
  p->fused = enable != 0;
  p->generation++;
  return DGB_OK;
}

int dgb_plan_set_tensor_cores(dgb_plan* p, int enable, int* blocks_out) {
  if (!p || !p->finalized) return fail(DGB_ERR_ARGUMENT, "plan not finalized");
  int n = 0;
  const bool allowed = enable && !p->hex && p->prm.precision == 1 && !p->dev.viscous && p->dev.nv == 5;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    const BlockDev& B = p->dev.blk[b];
    p->tc_on[b] = false;
    if (!allowed || B.E == 0) continue;
    const TcShape s = tc_shape(B.Np, B.Nq, p->dev.nv);
    if (!s.eligible) continue;
    if (!p->tc_image[b]) {
      double* d;
      int rc;
      if ((rc = alloc(p, ((size_t)s.image_floats + 1) / 2, &d))) return rc;
      p->tc_image[b] = reinterpret_cast<float*>(d);
      if (tc_pack(B, s, p->tc_image[b], nullptr)) return fail(DGB_ERR_CUDA, "tensor-core operand packing failed");
      CK(cudaDeviceSynchronize());
    }
    p->tc[b] = s;
    p->tc_on[b] = true;
    ++n;
  }
  p->generation++;
  if (blocks_out) *blocks_out = n;
  return DGB_OK;
}

int dgb_plan_device_errors(dgb_plan* p, int* out, int reset) {
  if (!p || !out || !p->dev_err) return fail(DGB_ERR_ARGUMENT, "plan not finalized or null output");
  CK(cudaMemcpy(out, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) CK(cudaMemset(p->dev_err, 0, sizeof(int)));
  return DGB_OK;
}

int dgb_plan_destroy(dgb_plan* p) {
  if (!p) return DGB_OK;
  if (p->step_exec) cudaGraphExecDestroy(p->step_exec);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  for (void* d : p->allocations) cudaFree(d);
  for (double* d : p->sub_bdc) cudaFree(d);
  delete p;
  return DGB_OK;
}

int dgb_rhs(dgb_plan* p, const dgb_state* U, const dgb_state* inv_out, const dgb_state* vis_out, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  FinalizeArgs A;
  memset(&A, 0, sizeof(A));
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) {
    A.out_inv[b] = inv_out ? inv_out->block[b] : nullptr;
    A.out_vis[b] = vis_out ? vis_out->block[b] : nullptr;
  }
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_rhs<5>(p, S, A, st) : run_rhs<16>(p, S, A, st);
}

int dgb_plan_autotune(dgb_plan* p, const dgb_state* U, int reps, int* widths, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (reps < 1) return fail(DGB_ERR_ARGUMENT, "reps must be >= 1");
  if (p->hex) {   // the sum-factorised kernels have fixed per-degree launches
    if (widths)
      for (int k = 0; k < 3 * DGB_MAX_BLOCKS; ++k) widths[k] = 0;
    return DGB_OK;
  }
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (p->prm.precision == 1)
    return p->dev.nv == 5 ? autotune_dense<5, float>(p, S, reps, st, widths)
                          : autotune_dense<16, float>(p, S, reps, st, widths);
  return p->dev.nv == 5 ? autotune_dense<5, double>(p, S, reps, st, widths)
                        : autotune_dense<16, double>(p, S, reps, st, widths);
}

int dgb_plan_set_face_points(dgb_plan* p, int face_type, const double* points) {
  if (!p || face_type < 0 || face_type > 1 || !points) return fail(DGB_ERR_ARGUMENT, "bad face point argument");
  if (!p->face_present[face_type]) return fail(DGB_ERR_ARGUMENT, "no faces of that type");
  const FaceDev& F = p->dev.face[face_type];
  return upload(p, points, (size_t)F.F * F.nq * 3, &p->face_points[face_type]);
}

int dgb_wall_forces(dgb_plan* p, const dgb_state* U, const int32_t* wall_tags, int n_wall_tags,
                    const double* moment_center, double* out, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!out || !moment_center || n_wall_tags < 0 || n_wall_tags > DGB_MAX_TAGS || (n_wall_tags && !wall_tags))
    return fail(DGB_ERR_ARGUMENT, "bad wall-force argument");
  WallSet walls;
  walls.n = n_wall_tags;
  for (int k = 0; k < DGB_MAX_TAGS; ++k) walls.tags[k] = k < n_wall_tags ? wall_tags[k] : -1;
  for (int d = 0; d < 3; ++d) walls.center[d] = moment_center[d];
  size_t blocks[2] = {0, 0}, total = 0;
  for (int ft = 0; ft < 2; ++ft)
    if (p->face_present[ft]) {
      if (!p->face_points[ft]) return fail(DGB_ERR_ARGUMENT, "call dgb_plan_set_face_points first");
      blocks[ft] = (size_t)blocks_for((long)p->dev.face[ft].F * p->dev.face[ft].nq, kThreads);
      total += blocks[ft];
    }
  if (total > p->force_partials_n) {
    if ((rc = alloc(p, total * kForceValues, &p->force_partials))) return rc;
    p->force_partials_n = total;
  }
  // the face buffers of one right-hand-side evaluation (traces, gradients, BR2 lifts)
  FinalizeArgs A;
  memset(&A, 0, sizeof(A));
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  p->f32_traces = false;
  rc = p->dev.nv == 5 ? run_rhs<5>(p, S, A, st) : run_rhs<16>(p, S, A, st);
  p->f32_traces = true;
  if (rc) return rc;
  size_t off = 0;
  for (int ft = 0; ft < 2; ++ft) {
    if (!blocks[ft]) continue;
    double* part = p->force_partials + off * kForceValues;
    if (p->dev.nv == 5)
      k_wall_forces<5><<<(unsigned)blocks[ft], kThreads, 0, st>>>(p->dev, ft, p->face_points[ft], walls, part);
    else
      k_wall_forces<16><<<(unsigned)blocks[ft], kThreads, 0, st>>>(p->dev, ft, p->face_points[ft], walls, part);
    off += blocks[ft];
  }
  k_wall_forces_final<<<1, 32, 0, st>>>(p->force_partials, (int)total, out);
  CK(cudaGetLastError());
  return DGB_OK;
}

int dgb_plan_set_subcells(dgb_plan* p, int b, const dgb_subcell_block_desc* d) {
  if (!p || !d || b < 0 || b >= p->dev.nblocks || !p->block_set[b]) return fail(DGB_ERR_ARGUMENT, "bad subcell block");
  SubcellBlockDev& C = p->mood.blk[b];
  const BlockDev& B = p->dev.blk[b];
  C.S = d->num_subcells;
  C.NI = d->num_internal;
  C.NB = d->num_boundary;
  if (C.S != 64) return fail(DGB_ERR_UNSUPPORTED, "subcell tables need 64 subcells (4 divisions)");
  const size_t E = B.E, S = C.S, Np = B.Np, NI = C.NI, NB = C.NB;
  int rc;
  if ((rc = upload(p, d->projection, E * S * Np, &C.P))) return rc;
  if ((rc = upload(p, d->reconstruction, E * Np * S, &C.R))) return rc;
  if ((rc = upload(p, d->volumes, E * S, &C.vol))) return rc;
  if ((rc = upload(p, d->centers, E * S * 3, &C.cen))) return rc;
  if ((rc = upload(p, d->internal_normals, E * NI * 3, &C.in_n))) return rc;
  if ((rc = upload(p, d->internal_areas, E * NI, &C.in_a))) return rc;
  if ((rc = upload(p, d->boundary_normals, E * NB * 3, &C.bd_n))) return rc;
  if ((rc = upload(p, d->boundary_areas, E * NB, &C.bd_a))) return rc;
  if ((rc = upload(p, d->internal_owner, NI, &C.iown))) return rc;
  if ((rc = upload(p, d->internal_neighbor, NI, &C.inbr))) return rc;
  if ((rc = upload(p, d->csr_ptr, S + 1, &C.csr_ptr))) return rc;
  if ((rc = upload(p, d->csr_face, 2 * NI, &C.csr_face))) return rc;
  if ((rc = upload(p, d->boundary_basis, NB * Np, &C.bbasis))) return rc;
  if ((rc = upload(p, d->gather, NB, &C.gather))) return rc;
  if ((rc = upload(p, d->scatter, NB, &C.scatter))) return rc;
  p->sub_block_set[b] = true;
  return DGB_OK;
}

int dgb_plan_build_subcells(dgb_plan* p, int b, const dgb_subcell_reference* r, const double* geometry_nodes) {
  if (!p || !r || b < 0 || b >= p->dev.nblocks || !p->block_set[b]) return fail(DGB_ERR_ARGUMENT, "bad subcell block");
  const BlockDev& B = p->dev.blk[b];
  if (r->num_subcells != 64) return fail(DGB_ERR_UNSUPPORTED, "subcell tables need 64 subcells (4 divisions)");
  if (r->num_points < 1 || r->num_geometry_nodes < 1 || r->num_vertices < 1 || r->num_internal < 1 ||
      r->num_boundary < 1 || (r->cell_size != 4 && r->cell_size != 6 && r->cell_size != 8))
    return fail(DGB_ERR_ARGUMENT, "bad subcell reference sizes");
  if (!r->rule_weights || !r->point_basis || !r->point_geometry_grad || !r->vertex_geometry || !r->cells ||
      !r->internal_faces || !r->boundary_faces || !r->internal_owner || !r->internal_neighbor || !r->boundary_owner ||
      !r->csr_ptr || !r->csr_face || !r->boundary_basis || !r->gather || !r->scatter)
    return fail(DGB_ERR_ARGUMENT, "null subcell reference table");
  const int S = r->num_subcells, NI = r->num_internal, NB = r->num_boundary, V = r->num_vertices;
  // every index the device follows stays inside its table
  for (int k = 0; k < S * r->cell_size; ++k)
    if (r->cells[k] < 0 || r->cells[k] >= V) return fail(DGB_ERR_ARGUMENT, "subcell vertex out of range");
  for (int f = 0; f < NI + NB; ++f) {
    const int32_t* fv = f < NI ? r->internal_faces + f * 4 : r->boundary_faces + (f - NI) * 4;
    for (int k = 0; k < 4; ++k)
      if ((k < 3 || fv[k] >= 0) && (fv[k] < 0 || fv[k] >= V)) return fail(DGB_ERR_ARGUMENT, "subface vertex out of range");
    const int own = f < NI ? r->internal_owner[f] : r->boundary_owner[f - NI];
    if (own < 0 || own >= S || (f < NI && (r->internal_neighbor[f] < 0 || r->internal_neighbor[f] >= S)))
      return fail(DGB_ERR_ARGUMENT, "subface subcell out of range");
  }
  SubcellBlockDev& C = p->mood.blk[b];
  if (p->sub_block_set[b]) return fail(DGB_ERR_ARGUMENT, "subcell tables already set for this block");
  C.S = S;
  C.NI = NI;
  C.NB = NB;
  const size_t E = B.E, Np = B.Np, Qs = r->num_points, ng = r->num_geometry_nodes;
  int rc;
  // the index tables the MOOD kernels read, as dgb_plan_set_subcells uploads them
  if ((rc = upload(p, r->internal_owner, (size_t)NI, &C.iown))) return rc;
  if ((rc = upload(p, r->internal_neighbor, (size_t)NI, &C.inbr))) return rc;
  if ((rc = upload(p, r->csr_ptr, (size_t)S + 1, &C.csr_ptr))) return rc;
  if ((rc = upload(p, r->csr_face, 2 * (size_t)NI, &C.csr_face))) return rc;
  if ((rc = upload(p, r->boundary_basis, (size_t)NB * Np, &C.bbasis))) return rc;
  if ((rc = upload(p, r->gather, (size_t)NB, &C.gather))) return rc;
  if ((rc = upload(p, r->scatter, (size_t)NB, &C.scatter))) return rc;
  if (E == 0) {
    p->sub_block_set[b] = true;
    return DGB_OK;
  }
  SubcellRefDev R{S, (int)Qs, (int)ng, V, r->cell_size, NI, NB, (int)Np, nullptr, nullptr, nullptr, nullptr,
                  nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  if ((rc = upload(p, r->rule_weights, (size_t)S * Qs, &R.rw))) return rc;
  if ((rc = upload(p, r->point_basis, (size_t)S * Qs * Np, &R.sb))) return rc;
  if ((rc = upload(p, r->point_geometry_grad, (size_t)S * Qs * ng * 3, &R.gq))) return rc;
  if ((rc = upload(p, r->vertex_geometry, (size_t)V * ng, &R.vg))) return rc;
  if ((rc = upload(p, r->cells, (size_t)S * r->cell_size, &R.cells))) return rc;
  if ((rc = upload(p, r->internal_faces, (size_t)NI * 4, &R.ifaces))) return rc;
  if ((rc = upload(p, r->boundary_faces, (size_t)NB * 4, &R.bfaces))) return rc;
  R.iown = C.iown;
  R.inbr = C.inbr;
  if ((rc = upload(p, r->boundary_owner, (size_t)NB, &R.bown))) return rc;
  const size_t smem = subcell_build_smem(R);
  if (smem > 220 * 1024) return fail(DGB_ERR_UNSUPPORTED, "element too large for the subcell-table kernel");
  SubcellBuildOut O;
  double* d;
  if ((rc = alloc(p, E * S * Np, &d))) return rc;
  O.P = d;
  if ((rc = alloc(p, E * Np * S, &d))) return rc;
  O.R = d;
  if ((rc = alloc(p, E * S, &d))) return rc;
  O.vol = d;
  if ((rc = alloc(p, E * S * 3, &d))) return rc;
  O.cen = d;
  if ((rc = alloc(p, E * NI * 3, &d))) return rc;
  O.in_n = d;
  if ((rc = alloc(p, E * NI, &d))) return rc;
  O.in_a = d;
  if ((rc = alloc(p, E * NB * 3, &d))) return rc;
  O.bd_n = d;
  if ((rc = alloc(p, E * NB, &d))) return rc;
  O.bd_a = d;
  CK(cudaMalloc(&O.bd_c, E * NB * 3 * sizeof(double)));
  p->sub_bdc[b] = O.bd_c;
  double* xyz = nullptr;
  int* bad = nullptr;
  int h_bad = 0;
  cudaError_t err = cudaMalloc(&xyz, E * ng * 3 * sizeof(double));
  if (err == cudaSuccess) err = cudaMalloc(&bad, sizeof(int));
  if (err == cudaSuccess) err = cudaMemcpy(xyz, geometry_nodes, E * ng * 3 * sizeof(double), cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemset(bad, 0, sizeof(int));
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(k_subcell_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err == cudaSuccess) {
    k_subcell_build<<<(unsigned)E, 256, smem>>>(R, xyz, O, bad);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMemcpy(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(xyz);
  cudaFree(bad);
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, std::string("subcell tables: ") + cudaGetErrorString(err));
  if (h_bad)
    return fail(DGB_ERR_ARGUMENT, "subcell Gram matrix of element " + std::to_string(h_bad - 1) +
                                      " is not positive definite");
  C.P = O.P;
  C.R = O.R;
  C.vol = O.vol;
  C.cen = O.cen;
  C.in_n = O.in_n;
  C.in_a = O.in_a;
  C.bd_n = O.bd_n;
  C.bd_a = O.bd_a;
  p->sub_block_set[b] = true;
  return DGB_OK;
}

int dgb_plan_match_subcell_faces(dgb_plan* p, int ft, const int32_t* osub, const int32_t* ncand) {
  if (!p || ft < 0 || ft > 1) return fail(DGB_ERR_ARGUMENT, "bad subcell face type");
  if (!p->face_present[ft]) return fail(DGB_ERR_ARGUMENT, "the plan has no faces of this type");
  const FaceDev& fd = p->dev.face[ft];
  const size_t F = fd.F;
  if (F && (!osub || !ncand)) return fail(DGB_ERR_ARGUMENT, "null subface table");
  SubcellCentres C;
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) {
    C.c[b] = b < p->dev.nblocks ? p->sub_bdc[b] : nullptr;
    C.NB[b] = b < p->dev.nblocks ? p->mood.blk[b].NB : 0;
  }
  // the host tables index the blocks' boundary subfaces: check them and the blocks they need
  std::vector<int32_t> ob(F), nb(F);
  if (F) {
    CK(cudaMemcpy(ob.data(), fd.ob, F * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(nb.data(), fd.nb, F * sizeof(int32_t), cudaMemcpyDeviceToHost));
  }
  for (size_t f = 0; f < F; ++f) {
    if (nb[f] < 0) continue;
    for (int side = 0; side < 2; ++side) {
      const int blk = side ? nb[f] : ob[f];
      if (blk < 0 || blk >= p->dev.nblocks || !p->sub_block_set[blk] || !p->sub_bdc[blk])
        return fail(DGB_ERR_ARGUMENT, "build the subcell tables of both sides' blocks first");
      const int32_t* ids = (side ? ncand : osub) + f * kSub;
      for (int k = 0; k < kSub; ++k)
        if (ids[k] < 0 || ids[k] >= C.NB[blk]) return fail(DGB_ERR_ARGUMENT, "boundary subface out of range");
    }
  }
  int rc;
  const int32_t* d_osub = nullptr;
  const int32_t* d_cand = nullptr;
  if ((rc = upload(p, osub, F * kSub, &d_osub))) return rc;
  if ((rc = upload(p, ncand, F * kSub, &d_cand))) return rc;
  int32_t* d_nsub = nullptr;
  if (F) {
    CK(cudaMalloc(&d_nsub, F * kSub * sizeof(int32_t)));
    p->allocations.push_back(d_nsub);
  }
  int* bad = nullptr;
  int h_bad = 0;
  CK(cudaMalloc(&bad, sizeof(int)));
  cudaError_t err = cudaMemset(bad, 0, sizeof(int));
  if (err == cudaSuccess && F) {
    k_subcell_match<<<blocks_for((long)F, 256), 256>>>(fd, C, d_osub, d_cand, d_nsub, bad);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMemcpy(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  if (err != cudaSuccess) return fail(DGB_ERR_CUDA, std::string("subface matching: ") + cudaGetErrorString(err));
  if (h_bad) return fail(DGB_ERR_ARGUMENT, "Nonconforming subfaces at face " + std::to_string(h_bad - 1));
  SubcellFaceDev& SF = p->mood.face[ft];
  SF.osub = d_osub;
  SF.nsub = d_nsub;
  p->sub_face_set[ft] = true;
  return DGB_OK;
}

int dgb_plan_set_subcell_faces(dgb_plan* p, int ft, const int32_t* osub, const int32_t* nsub) {
  if (!p || ft < 0 || ft > 1) return fail(DGB_ERR_ARGUMENT, "bad subcell face type");
  SubcellFaceDev& SF = p->mood.face[ft];
  const size_t F = p->dev.face[ft].F;
  int rc;
  if ((rc = upload(p, osub, F * kSub, &SF.osub))) return rc;
  if ((rc = upload(p, nsub, F * kSub, &SF.nsub))) return rc;
  p->sub_face_set[ft] = true;
  return DGB_OK;
}

int dgb_plan_enable_mood(dgb_plan* p) {
  if (p) ++p->generation;    // invalidates a captured step
  if (!p || !p->finalized) return fail(DGB_ERR_ARGUMENT, "finalize the plan first");
  if (p->mood_ready) return DGB_OK;
  for (int b = 0; b < p->dev.nblocks; ++b)
    if (!p->sub_block_set[b]) return fail(DGB_ERR_ARGUMENT, "subcell tables missing for a block");
  for (int ft = 0; ft < 2; ++ft)
    if (p->face_present[ft] && !p->sub_face_set[ft]) return fail(DGB_ERR_ARGUMENT, "subcell face tables missing");
  const int NV = p->dev.nv;
  int rc;
  for (int b = 0; b < p->dev.nblocks; ++b) {
    const size_t E = p->dev.blk[b].E, S = p->mood.blk[b].S, state = E * p->dev.blk[b].Np * NV;
    if ((rc = alloc(p, E * S * NV, &p->mood.blk[b].ubar))) return rc;
    if ((rc = alloc(p, E * S * NV, &p->mood.blk[b].rsub))) return rc;
    void* f = nullptr;
    CK(cudaMalloc(&f, E));
    p->allocations.push_back(f);
    CK(cudaMemset(f, 0, E));
    p->flags[b] = static_cast<uint8_t*>(f);
    if ((rc = alloc(p, state, &p->unl[b]))) return rc;
    if ((rc = alloc(p, state, &p->eul[b]))) return rc;
    if ((rc = alloc(p, state, &p->vis[b]))) return rc;
    if ((rc = alloc(p, state, &p->rec[b]))) return rc;
  }
  for (int ft = 0; ft < 2; ++ft) {
    if (!p->face_present[ft]) continue;
    const size_t F = p->dev.face[ft].F;
    if ((rc = alloc(p, F * kSub * NV, &p->mood.face[ft].fsub))) return rc;
    if ((rc = alloc(p, F * NV, &p->mood.face[ft].dflux))) return rc;
    void* a = nullptr;
    CK(cudaMalloc(&a, F));
    p->allocations.push_back(a);
    CK(cudaMemset(a, 0, F));
    p->mood.face[ft].active = static_cast<uint8_t*>(a);
  }
  for (double*& d : p->sub_bdc) {    // the boundary subface centres were only needed for matching
    cudaFree(d);
    d = nullptr;
  }
  p->mood_ready = true;
  return DGB_OK;
}

int dgb_subcell_recompute(dgb_plan* p, const dgb_state* base, const dgb_state* cand, double dt,
                          const dgb_state* arhs, uint8_t* const* troubled, const dgb_state* out, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, base, "base")) || (rc = check_state(p, cand, "candidate")) ||
      (rc = check_state(p, out, "out")))
    return rc;
  if (!p->mood_ready) return fail(DGB_ERR_ARGUMENT, "call dgb_plan_enable_mood first");
  if (!troubled) return fail(DGB_ERR_ARGUMENT, "troubled flags are null");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_subcell_api<5>(p, base, cand, dt, arhs, troubled, out, st)
                        : run_subcell_api<16>(p, base, cand, dt, arhs, troubled, out, st);
}

int dgb_mlp_features(dgb_plan* p, const dgb_state* U, float* features, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!features) return fail(DGB_ERR_ARGUMENT, "features is null");
  if ((rc = ensure_predictor_buffers(p))) return rc;
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const __half* keep = p->pred_w16;
  p->pred_w16 = nullptr;            // features only
  rc = p->dev.nv == 5 ? run_predict<5>(p, S, st) : run_predict<16>(p, S, st);
  p->pred_w16 = keep;
  if (rc) return rc;
  long total = 0;
  for (int b = 0; b < p->dev.nblocks; ++b) total += p->dev.blk[b].E;
  CK(cudaMemcpyAsync(features, p->pred_feat, sizeof(float) * (size_t)total * kMlpIn, cudaMemcpyDeviceToDevice, st));
  return DGB_OK;
}

int dgb_mlp_infer(const void* w16, const float* norm, const float* features, int64_t n, float threshold, float* prob,
                  uint8_t* flag, void* stream) {
  if (!w16 || !norm || !features) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (n < 0) return fail(DGB_ERR_ARGUMENT, "negative count");
  if (n == 0) return DGB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_mlp_infer<<<blocks_for(n, 128), 128, 0, st>>>(static_cast<const __half*>(w16), norm, features, n, threshold, prob,
                                                  flag);
  CK(cudaGetLastError());
  return DGB_OK;
}

int dgb_mlp_train_step(float* w, float* grad, float* m, float* v, void* w16, const float* norm, const float* features,
                       const uint8_t* labels, const int* index, int batch, float pos_weight, float lr, int step,
                       float* loss, void* stream) {
  if (!w || !grad || !m || !v || !norm || !features || !labels || !index) return fail(DGB_ERR_ARGUMENT, "null argument");
  if (batch < 1 || step < 1) return fail(DGB_ERR_ARGUMENT, "batch and step must be >= 1");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t sm = sizeof(float) * (size_t)kMlpTrainSmemFloats;
  int rc;
  if ((rc = prepare(k_mlp_train, sm))) return rc;
  k_mlp_train<<<blocks_for(batch, kMlpChunk), kMlpTrainThreads, sm, st>>>(w, norm, features, labels, index, batch,
                                                                         pos_weight, grad, loss);
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
  k_mlp_adam<<<blocks_for(kMlpParams, 256), 256, 0, st>>>(w, grad, m, v, static_cast<__half*>(w16), lr, b1, b2, 1e-8f,
                                                          c1, c2);
  CK(cudaGetLastError());
  return DGB_OK;
}

int dgb_plan_set_predictor(dgb_plan* p, const void* w16, const float* norm, float threshold, int mode) {
  if (p) ++p->generation;    // invalidates a captured step
  int rc;
  if ((rc = check_ready(p))) return rc;
  if (mode < 0 || mode > 2) return fail(DGB_ERR_ARGUMENT, "mode must be 0 (off), 1 (learned) or 2 (evaluate)");
  if (mode && (!w16 || !norm)) return fail(DGB_ERR_ARGUMENT, "weights and normalisation are needed");
  if (mode && !p->mood_ready) return fail(DGB_ERR_ARGUMENT, "the predictor feeds MOOD: call dgb_plan_enable_mood first");
  if (mode && (rc = ensure_predictor_buffers(p))) return rc;
  p->pred_mode = mode;
  p->pred_w16 = static_cast<const __half*>(w16);
  p->pred_norm = norm;
  p->pred_threshold = threshold;
  return DGB_OK;
}

int dgb_plan_predictor_counts(dgb_plan* p, int64_t* out, int reset) {
  int rc;
  if ((rc = check_ready(p))) return rc;
  if (!out) return fail(DGB_ERR_ARGUMENT, "out is null");
  if ((rc = ensure_predictor_buffers(p))) return rc;
  unsigned long long h[5];
  CK(cudaMemcpy(h, p->pred_counts, sizeof(h), cudaMemcpyDeviceToHost));
  for (int k = 0; k < 5; ++k) out[k] = (int64_t)h[k];
  if (reset) CK(cudaMemset(p->pred_counts, 0, sizeof(h)));
  return DGB_OK;
}

namespace {
int profile_rhs(dgb_plan* p, const dgb_state* U, const FinalizeArgs& A, float* ms_out, void* stream) {
  int rc;
  cudaEvent_t ev[DGB_RHS_STAGES + 1];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  rc = p->dev.nv == 5 ? run_rhs<5>(p, S, A, st, ev) : run_rhs<16>(p, S, A, st, ev);
  if (!rc) {
    CK(cudaEventSynchronize(ev[DGB_RHS_STAGES]));
    for (int k = 0; k < DGB_RHS_STAGES; ++k) CK(cudaEventElapsedTime(&ms_out[k], ev[k], ev[k + 1]));
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return rc;
}
}  // namespace

int dgb_rhs_profile(dgb_plan* p, const dgb_state* U, float* ms_out, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!ms_out) return fail(DGB_ERR_ARGUMENT, "ms_out is null");
  FinalizeArgs A;
  memset(&A, 0, sizeof(A));
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) {
    A.out_inv[b] = p->stage1[b];      // scratch outputs
    A.out_vis[b] = p->stage2[b];
  }
  return profile_rhs(p, U, A, ms_out, stream);
}

int dgb_rhs_profile_stage(dgb_plan* p, const dgb_state* U, int split, float* ms_out, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!ms_out) return fail(DGB_ERR_ARGUMENT, "ms_out is null");
  FinalizeArgs A;
  memset(&A, 0, sizeof(A));
  A.stage = 1;
  A.beta = 1.0;                       // dst = U + 0 * rhs: the stage update's arithmetic, dt = 0
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) {
    A.base[b] = U->block[b];
    A.dst[b] = p->stage1[b];
    A.out_vis[b] = split ? p->stage2[b] : nullptr;
  }
  return profile_rhs(p, U, A, ms_out, stream);
}

int dgb_stable_dt(dgb_plan* p, const dgb_state* U, double cfl, double* dt_out, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!dt_out) return fail(DGB_ERR_ARGUMENT, "dt_out is null");
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_stable_dt<5>(p, S, cfl, dt_out, st) : run_stable_dt<16>(p, S, cfl, dt_out, st);
}

int dgb_positivity(dgb_plan* p, const dgb_state* U, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_positivity<5>(p, S, st) : run_positivity<16>(p, S, st);
}

int dgb_troubled(dgb_plan* p, const dgb_state* U, double* const* sensor, uint8_t* const* flags, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_troubled<5>(p, S, sensor, flags, st) : run_troubled<16>(p, S, sensor, flags, st);
}

int dgb_admissibility(dgb_plan* p, const dgb_state* U, dgb_status* status, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!status) return fail(DGB_ERR_ARGUMENT, "status is null");
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_admissibility<5>(p, S, status, 0, st) : run_admissibility<16>(p, S, status, 0, st);
}

int dgb_ssprk3_step_graph(dgb_plan* p, const dgb_state* U, double dt, dgb_status* status, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!status) return fail(DGB_ERR_ARGUMENT, "status is null");
  if (p->prm.limiter == 2 && !p->mood_ready) return fail(DGB_ERR_ARGUMENT, "MOOD limiter needs dgb_plan_enable_mood");
  StepKey key;
  memset(&key, 0, sizeof(key));
  for (int b = 0; b < DGB_MAX_BLOCKS; ++b) key.block[b] = U->block[b];
  key.dt = dt;
  key.status = status;
  key.generation = p->generation;
  if (!p->step_exec || memcmp(&key, &p->step_key, sizeof(key)) != 0) {
    if (p->step_exec) {
      CK(cudaGraphExecDestroy(p->step_exec));
      p->step_exec = nullptr;
    }
    // the legacy default stream cannot be captured: capture on a private stream, replay on the caller's
    if (!p->capture_stream) CK(cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeRelaxed));
    const StatePtrs S = to_ptrs(U);
    rc = p->dev.nv == 5 ? run_step<5>(p, S, dt, status, p->capture_stream)
                        : run_step<16>(p, S, dt, status, p->capture_stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(p->capture_stream, &graph);
    if (rc || end != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc) return rc;
      return fail(DGB_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(end));
    }
    const cudaError_t inst = cudaGraphInstantiate(&p->step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (inst != cudaSuccess) {
      p->step_exec = nullptr;
      return fail(DGB_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(inst));
    }
    p->step_key = key;
  }
  CK(cudaGraphLaunch(p->step_exec, static_cast<cudaStream_t>(stream)));
  return DGB_OK;
}

int dgb_ssprk3_step(dgb_plan* p, const dgb_state* U, double dt, dgb_status* status, void* stream) {
  int rc;
  if ((rc = check_ready(p)) || (rc = check_state(p, U, "U"))) return rc;
  if (!status) return fail(DGB_ERR_ARGUMENT, "status is null");
  if (p->prm.limiter == 2 && !p->mood_ready) return fail(DGB_ERR_ARGUMENT, "MOOD limiter needs dgb_plan_enable_mood");
  const StatePtrs S = to_ptrs(U);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->dev.nv == 5 ? run_step<5>(p, S, dt, status, st) : run_step<16>(p, S, dt, status, st);
}

}  // extern "C"

namespace dgb {
// error reporting for the host-only set-up routines compiled in other translation units
int set_error(int code, const char* msg) { return fail(code, msg); }
}  // namespace dgb
