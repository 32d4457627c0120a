// lw_net.h -- parameter and operand layouts of the learned gas optics
// (BF16 MLP 8 -> 128 -> 128 -> 288), shared by the network kernels of
// lw_mlp.cu and the fused column kernel of lw_fused.cu.
#pragma once

#include <cuda_bf16.h>

#include "lw_features.cuh"

namespace lw {

typedef __nv_bfloat16 bf16;

constexpr int HID = SG_HID, NOP = SG_NOUTP, NIN = SG_NFEAT, KIN = 16;
constexpr int P_W1 = 0;                      // [128][8]   (column 7: bias of layer 1)
constexpr int P_W2 = P_W1 + HID * NIN;       // [128][128]
constexpr int P_B2 = P_W2 + HID * HID;       // [128]
constexpr int P_W3 = P_B2 + HID;             // [288][128] (pad rows 140..143, 284..287 stay 0)
constexpr int P_B3 = P_W3 + NOP * HID;       // [288]
constexpr int P_N = P_B3 + NOP;              // 54,688 (53,656 trainable)

constexpr int O_W1 = 0;                      // bf16 [128][16]
constexpr int O_W2 = O_W1 + HID * KIN;       // bf16 [128][128]
constexpr int O_W2T = O_W2 + HID * HID;      // bf16 [128][128] = W2^T
constexpr int O_W3 = O_W2T + HID * HID;      // bf16 [288][128]: rows [0,140) log(taug/coldry), [144,284) fracs
constexpr int O_W3T = O_W3 + NOP * HID;      // bf16 [128][288] = W3^T
constexpr int O_N = O_W3T + HID * NOP;

// SiLU with the fast exp and division: the same function in training, in
// the network kernels and in the fused column kernel
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// Device state of the loaded network (lw_mlp.cu): operand copies, FP32
// master parameters (biases), normalisation, error flag, fallback counter.
struct SgNetView {
  const bf16* ops;
  const float* params;
  const float* norm;
  int* err;
  unsigned int* fallback;
  int ready;
};
SgNetView sg_net_view();

}  // namespace lw
