// Tensor-core (tcgen05) inviscid volume integrals of the dense element blocks: shapes and the host
// entry points that the plan calls (tc_volume.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace dgb {

struct BlockDev;
struct DevPlan;
struct StatePtrs;

// Device error bits recorded by kernels whose waits are bounded.
enum { DGB_DEVICE_TIMEOUT = 1 };

// Operand shapes and shared-memory layout of one block's tensor-core volume kernel.
struct TcShape {
  int Np, Nq;                // nodes, volume points
  int Te;                    // elements per tile
  int Kp1, Kq;               // GEMM 1 depth (Np rounded up to 8), GEMM 2 depth per direction (Nq rounded up to 8)
  int G8;                    // row groups of 8 holding the Np rows of A2
  int N1;                    // tile columns (Te * NV rounded up to 16)
  int a1_floats, a2_floats;  // one hi (or lo) copy of A1, of one A2_r
  int image_floats;          // A1 hi, lo, then A2_r hi, lo for r = 0, 1, 2
  size_t b_offset, stage_offset, smem;   // bytes of dynamic shared memory
  bool eligible;
};

TcShape tc_shape(int Np, int Nq, int nv);
// Packs the constant operands of block B into `image` (s.image_floats floats, device memory).
int tc_pack(const BlockDev& B, const TcShape& s, float* image, cudaStream_t st);
// Inviscid volume residuals of block b into B.Rinv; err: device word for DGB_DEVICE_TIMEOUT.
cudaError_t tc_volume(const DevPlan& P, const StatePtrs& S, int b, const TcShape& s, const float* image, int* err,
                      int sm_count, cudaStream_t st);

}  // namespace dgb
