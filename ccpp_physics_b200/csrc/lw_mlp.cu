// lw_mlp.cu -- learned gas optics for the RRTMG-LW path: a BF16 MLP
// 8 -> 128 -> 128 -> 288 (7 layer features + 1; 140 log(taug/coldry) and
// 140 Planck fractions, padded to 288) on the 5th-generation tensor cores.
//
// Kernels (all hand-written, tcgen05 MMAs with FP32 accumulation in TMEM):
//   mlp_fwd_kernel<MODE>  persistent; the three weight matrices stay in
//                         shared memory; per 128-row tile: X -> MMA1 ->
//                         SiLU -> MMA2 -> SiLU -> MMA3 (2 x N=144) -> epilogue.
//                         MODE_FEATS: rows are feature vectors, writes the
//                         normalised outputs.  MODE_TRAIN: rows are gathered
//                         training samples; writes the activations the
//                         backward pass needs, dL/dy and the loss.  MODE_LW:
//                         rows are the layers of a chunk of columns; writes
//                         tau = exp(y) * coldry + aerosol and the band-
//                         normalised Planck fractions straight into the
//                         gas-optics -> transfer scratch of the column path.
//   mlp_h_kernel          the same network for the learned-gas-optics column
//                         path (lw_sg_path.cu): one column per tile, tau and
//                         the Planck fractions as FP16 8-layer blocks of its
//                         compact hand-off, and the list of the columns that
//                         have a layer outside the envelope.
//   gemm_tn_kernel<EPI>   C = A * B^T for the backward pass: dH = dZ W with
//                         the activation derivative fused (EPI_DACT), and
//                         split-K weight gradients dW = dZ^T H with FP32
//                         atomics (EPI_ATOMIC).  Bias gradients come out as
//                         the column of a constant-1 row appended to H.
//   adam_kernel           Adam on FP32 master weights; rewrites the BF16
//                         operand copies (W and W^T).
//   features_kernel       layer features + coldry of a block (training data).
//
// The network replaces setcoef+taumol (radlw_main.F90:2151-2406, 3836-6840)
// for layers inside the training envelope; the gas-optics kernel recomputes
// every other layer with plain taumol (lw_gas.cuh).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/rrtmg_lw_gpu.h"
#include "lw_common.cuh"
#include "lw_features.cuh"
#include "lw_launch.h"
#include "lw_net.h"
#include "lw_umma.cuh"

namespace lw {

// parameter / operand layouts (lw_net.h)

constexpr int GW2_LD = 144, GW3_ROWS = 384;  // gradients of [W | b] (column 128 = bias)
constexpr int G_W1 = 0;                      // f32 [128][16]
constexpr int G_W2 = G_W1 + HID * KIN;       // f32 [128][144]
constexpr int G_W3 = G_W2 + HID * GW2_LD;    // f32 [384][144]
constexpr int G_N = G_W3 + GW3_ROWS * GW2_LD;

__host__ __device__ inline bool pad_out_row(int j) { return (j >= 140 && j < 144) || j >= 284; }

// derivative of silu (lw_net.h) with the same fast exp and division
__device__ __forceinline__ float dsilu(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------------------
// forward kernel
enum { MODE_FEATS = 0, MODE_TRAIN = 1, MODE_LW = 2 };

struct FwdArgs {
  const bf16* ops;      // operand copies (O_*)
  const float* params;  // FP32 master (biases)
  const float* norm;    // SG_NORM_FLOATS
  long nrows;
  int* err;             // first error: 1 = MMA wait timed out
  // MODE_FEATS / MODE_TRAIN
  const float* feats;   // [*][8] raw features
  float* y;             // MODE_FEATS: [nrows][288] normalised outputs
  // MODE_TRAIN
  const float* targets; // [*][288] normalised targets
  long perm_a, perm_b, perm_n, perm_off;   // sample = (a * (perm_off + row) + b) mod n
  float loss_scale;     // 2 / (batch * 280)
  int tau_weight;       // 1: weight optical-depth errors by 1 / (1 + 1.66 tau), coldry in feats[., 7]
  float* loss;          // += sum of squared errors
  bf16 *xt, *z1, *h1t, *z2, *h2t, *dy, *dyt;   // activations, see the trainer
  long ldt;             // leading dimension (batch) of the transposed arrays
  // MODE_LW
  const Block* blocks;
  int nblocks;
  Block b0;
  Flags f;
  Scratch<float> sc;
  int nc;               // columns of this chunk
  // mlp_h_kernel (blocks, nblocks, b0, f, nc as MODE_LW)
  __half* hnd;          // [nc][nlay/8][tau 140 | frac 140][8 layers] (lw_sg_path.cu)
  const int* colmap;    // block of every global column (nblocks > 1)
  int c0;               // first global column of the chunk
  unsigned int* fb_flag;   // per global column: set once the column is listed
  int* fb_list;         // columns of the chunk with a layer outside the envelope
  int* fb_count;
  unsigned char* pk;    // [nc] packed column inputs, kSgPackBytes each (mlp_h_pack_kernel)
};

// Thread layout: 4 warpgroups.  Thread tid serves tile row (tid & 127) -- the
// TMEM lane its warp may read -- and column quarter q = tid >> 7 of every
// stage, so four threads share the epilogue work of a row and 16 warps per SM
// hide the load, TMEM and MMA latencies.
constexpr int FWD_THREADS = 512;
constexpr uint32_t SM_W1 = 0;                               // canon [128][16]
constexpr uint32_t SM_W2 = SM_W1 + HID * KIN * 2;           // canon [128][128]
constexpr uint32_t SM_W3 = SM_W2 + HID * HID * 2;           // canon [288][128]
constexpr uint32_t SM_X = SM_W3 + NOP * HID * 2;            // canon [128][16]
constexpr uint32_t SM_H = SM_X + 128 * KIN * 2;             // canon [128][128]
constexpr uint32_t SM_B2 = SM_H + 128 * HID * 2;            // f32 [128]
constexpr uint32_t SM_B3 = SM_B2 + HID * 4;                 // f32 [288]
constexpr uint32_t SM_NORM = SM_B3 + NOP * 4;               // f32 [608]
constexpr uint32_t SM_AER = SM_NORM + SG_NORM_FLOATS * 4;   // f32 [2][16][128] aerosol tau of the tile's layers
constexpr uint32_t SM_CD = SM_AER + 2 * NBANDS * 128 * 4;   // f32 [2][128] coldry of the tile's layers
constexpr uint32_t SM_OSC = SM_CD + 2 * 128 * 4;            // f32 [288] output scale  (std)
constexpr uint32_t SM_OSH = SM_OSC + NOP * 4;               // f32 [288] output shift (b3 * std + mean)
constexpr uint32_t SM_BLK = SM_OSH + NOP * 4;                // int [130] block of each column a tile spans
constexpr int TILE_MAX_COLS = 130;                           // 128 rows of >= 1 layer, +2 partial columns
constexpr uint32_t SM_BAR = (SM_BLK + TILE_MAX_COLS * 4 + 15) & ~15u;
constexpr uint32_t FWD_SMEM = SM_BAR + 32;
static_assert(FWD_SMEM > 116 * 1024, "forward kernel must hold its SM alone (512 TMEM columns)");
static_assert(FWD_SMEM <= 227 * 1024, "forward kernel shared memory");
constexpr uint32_t W3_HALF = 144 * HID * 2;                 // second 144-row B operand of MMA3

// band of each g-point (radlw_param.f:111-120 ngb)
__device__ __forceinline__ int band_of_g(int g) {
  return g < 10 ? 0 : g < 22 ? 1 : g < 38 ? 2 : g < 52 ? 3 : g < 68 ? 4 : g < 76 ? 5 : g < 88 ? 6 : g < 96 ? 7
       : g < 108 ? 8 : g < 114 ? 9 : g < 122 ? 10 : g < 130 ? 11 : g < 134 ? 12 : g < 136 ? 13 : g < 138 ? 14 : 15;
}

__device__ __forceinline__ void copy_rows_canon(unsigned char* dst, const bf16* src, int rows, int K, int tid) {
  const int chunks = rows * (K / 8);
  for (int c = tid; c < chunks; c += FWD_THREADS) {
    const int r = c / (K / 8), k = (c % (K / 8)) * 8;
    *reinterpret_cast<uint4*>(dst + umma::canon_off(r, k, K)) =
        __ldg(reinterpret_cast<const uint4*>(src + (size_t)r * K + k));
  }
}

// TMEM column of network output j: outputs [0,144) sit at columns 256.., [144,288) at 0..
__device__ __forceinline__ int out_col(int j) { return j < 144 ? 256 + j : j - 144; }

// Where a tile row of MODE_LW lives: chunk column, layer, block, block column,
// input row.  blk[] holds the block index of each column the tile spans
// (resolved once per tile), cfirst the tile's first chunk column.
struct LwRow {
  int cc, t, i, r;
  const Block* B;
};
__device__ __forceinline__ LwRow lw_row(const FwdArgs& a, long row, const int* blk, int cfirst) {
  LwRow w;
  const int nlay = a.f.nlay;
  w.cc = (int)(row / nlay);
  w.t = (int)(row - (long)w.cc * nlay);
  const int c = a.sc.c0 + w.cc;
  w.B = (a.nblocks == 1) ? &a.b0 : &a.blocks[blk[w.cc - cfirst]];
  w.i = c - w.B->col0;
  w.r = a.f.top_at_1 ? nlay - w.t - 1 : w.t;
  return w;
}

// MODE_LW output stage of one quarter: g-points [GA, GB) (whole bands), their
// optical depths and their band-normalised Planck fractions.  Ranges and bands
// are compile-time, so the loops carry no per-element tests.
template <int GA, int GB>
__device__ __forceinline__ void lw_out_quarter(uint32_t tb, int wl, bool live, float* tcol, float* fcol, size_t nlp,
                                               const float* osc, const float* osh, const float* aer_row, float cd) {
  constexpr int C0 = GA & ~15, NCH = (GB - C0 + 15) / 16;
  float v[NCH * 16];
#pragma unroll
  for (int c = 0; c < NCH; ++c) umma::tmem_ld16(umma::tmem_addr(tb, wl, 256 + C0 + 16 * c), v + 16 * c);
  if (live) {
#pragma unroll
    for (int g = GA; g < GB; ++g) {
      const float ly = fmaf(v[g - C0], osc[g], osh[g]);
      __stcs(tcol + (size_t)g * nlp, fmaf(__expf(ly), cd, aer_row[band_of_g(g) * 128]));
    }
  }
#pragma unroll
  for (int c = 0; c < NCH; ++c) umma::tmem_ld16(umma::tmem_addr(tb, wl, C0 + 16 * c), v + 16 * c);
  if (live) {
    float bsum[NBANDS];
#pragma unroll
    for (int b = 0; b < NBANDS; ++b) bsum[b] = 0.0f;
#pragma unroll
    for (int g = GA; g < GB; ++g) {
      const float fr = __saturatef(fmaf(v[g - C0], osc[144 + g], osh[144 + g]));
      v[g - C0] = fr;
      bsum[band_of_g(g)] += fr;
    }
#pragma unroll
    for (int b = 0; b < NBANDS; ++b) bsum[b] = bsum[b] > 0.0f ? 1.0f / bsum[b] : 1.0f;
#pragma unroll
    for (int g = GA; g < GB; ++g) __stcs(fcol + (size_t)g * nlp, v[g - C0] * bsum[band_of_g(g)]);
  }
}

// Polls of a tensor-core wait in the forward kernel before it gives up and
// records the error (default 1 << 22, seconds of waiting); lowered only by
// the failure-detection hook rrtmg_lw_gpu_surrogate_wait_limit.
constexpr uint32_t kFwdWaitPollsDefault = 1u << 22;
__constant__ uint32_t c_fwd_wait_polls = kFwdWaitPollsDefault;

template <int MODE>
__global__ void __launch_bounds__(FWD_THREADS, 1) mlp_fwd_kernel(FwdArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, wl = warp & 3, q = tid >> 7, tr = tid & 127;
  float* sb2 = reinterpret_cast<float*>(sm + SM_B2);
  float* sb3 = reinterpret_cast<float*>(sm + SM_B3);
  float* snorm = reinterpret_cast<float*>(sm + SM_NORM);
  float* saer0 = reinterpret_cast<float*>(sm + SM_AER);
  float* scd0 = reinterpret_cast<float*>(sm + SM_CD);
  float* osc = reinterpret_cast<float*>(sm + SM_OSC);
  float* osh = reinterpret_cast<float*>(sm + SM_OSH);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + SM_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SM_BAR + 8);
  int* sfail = reinterpret_cast<int*>(sm + SM_BAR + 12);
  int* sblk = reinterpret_cast<int*>(sm + SM_BLK);

  copy_rows_canon(sm + SM_W1, a.ops + O_W1, HID, KIN, tid);
  copy_rows_canon(sm + SM_W2, a.ops + O_W2, HID, HID, tid);
  copy_rows_canon(sm + SM_W3, a.ops + O_W3, NOP, HID, tid);
  for (int j = tid; j < HID; j += FWD_THREADS) sb2[j] = a.params[P_B2 + j];
  for (int j = tid; j < NOP; j += FWD_THREADS) sb3[j] = a.params[P_B3 + j];
  for (int j = tid; j < SG_NORM_FLOATS; j += FWD_THREADS) snorm[j] = a.norm[j];
  for (int j = tid; j < NOP; j += FWD_THREADS) {
    const float sd = a.norm[SG_OUT_STD + j];
    osc[j] = sd;
    osh[j] = fmaf(a.params[P_B3 + j], sd, a.norm[SG_OUT_MEAN + j]);
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(mbar, 1);
    *sfail = 0;
  }
  umma::fence_smem_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t sbase = umma::smem_u32(sm);
  constexpr uint32_t ID128 = umma::idesc_bf16(128, 128), ID144 = umma::idesc_bf16(128, 144);
  uint32_t phase = 0;
  const long ntiles = (a.nrows + 127) / 128;

  bool failed = false;   // uniform across the CTA
  auto wait_mma = [&]() -> bool {
    const bool ok = umma::mbar_wait(mbar, phase, c_fwd_wait_polls);
    phase ^= 1u;
    umma::fence_after_sync();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) *sfail = 1;
      failed = true;
      return false;
    }
    return true;
  };
  auto sync_for_mma = [&]() {
    umma::fence_smem_async();
    umma::fence_before_sync();
    __syncthreads();
  };

  int parity = 0;   // double buffer of the per-tile aerosol / coldry rows
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, parity ^= 1) {
    const long row = tile * 128 + tr;
    const bool live = row < a.nrows;
    float* saer = saer0 + parity * NBANDS * 128;
    float* scd = scd0 + parity * 128;
    int cfirst = 0;
    if (MODE == MODE_LW && a.nblocks > 1) {
      // block of every column this tile touches, one binary search per column
      const int nlay = a.f.nlay;
      cfirst = (int)((tile * 128) / nlay);
      const long rlast = min(tile * 128 + 127, a.nrows - 1);
      const int ncol = (int)(rlast / nlay) - cfirst + 1;
      __syncthreads();   // the previous tile's rows are done with sblk
      for (int j = tid; j < ncol; j += FWD_THREADS) sblk[j] = find_block(a.blocks, a.nblocks, a.sc.c0 + cfirst + j);
      __syncthreads();
    }
    long sample = row;
    if (MODE == MODE_TRAIN && live)
      sample = (long)(((unsigned long long)a.perm_a * (unsigned long long)(a.perm_off + row) +
                       (unsigned long long)a.perm_b) % (unsigned long long)a.perm_n);
    // ---------------- layer inputs (quarter 0: features; MODE_LW quarters 1-3: aerosol) ----
    if (q == 0) {
      float x[KIN];
#pragma unroll
      for (int j = 0; j < KIN; ++j) x[j] = 0.0f;
      if (live) {
        float raw[NIN];
        if (MODE == MODE_LW) {
          const LwRow w = lw_row(a, row, sblk, cfirst);
          const size_t o = (size_t)w.i + (size_t)w.B->ld * w.r;
          const double pavel = w.B->in[F_PLYR][o], tavel = w.B->in[F_TLYR][o], qv = w.B->in[F_QLYR][o];
          const double amdw = 28.9644 / 18.0154, amdo3 = 28.9644 / 47.9982;
          const double h2ovmr = fmax(0.0, qv * amdw / (1.0 - qv));
          const double o3vmr = fmax(0.0, w.B->in[F_OLYR][o] * amdo3);
          const double tem0 = (1.0 - h2ovmr) * 28.9644 + h2ovmr * 18.0154;
          scd[tr] = (float)((1.0e-20 * 1.0e3 * 6.0221415e23) * w.B->in[F_DELPIN][o] /
                            (100.0 * 9.80665 * tem0 * (1.0 + h2ovmr)));
          layer_features(pavel, tavel, h2ovmr, o3vmr, w.B->in[F_CO2][o], w.B->in[F_CH4][o], w.B->in[F_N2O][o], raw);
        } else {
          const float4* src = reinterpret_cast<const float4*>(a.feats + sample * NIN);
          const float4 u = __ldg(src), v = __ldg(src + 1);
          raw[0] = u.x; raw[1] = u.y; raw[2] = u.z; raw[3] = u.w; raw[4] = v.x; raw[5] = v.y; raw[6] = v.z;
        }
#pragma unroll
        for (int j = 0; j < 7; ++j) x[j] = (raw[j] - snorm[SG_IN_MEAN + j]) / snorm[SG_IN_STD + j];
        x[7] = 1.0f;
      }
      umma::st_canon8(sm + SM_X, tr, 0, KIN, x);
      umma::st_canon8(sm + SM_X, tr, 8, KIN, x + 8);
      if (MODE == MODE_TRAIN && live) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a.xt[(size_t)j * a.ldt + row] = __float2bfloat16_rn(x[j]);
      }
    } else if (MODE == MODE_LW && live) {
      const LwRow w = lw_row(a, row, sblk, cfirst);
      const size_t ldl = (size_t)w.B->ld;
      const int b0 = q == 1 ? 0 : q == 2 ? 6 : 11, b1 = q == 1 ? 6 : q == 2 ? 11 : 16;
      for (int b = b0; b < b1; ++b) {
        const size_t ab = (size_t)w.i + ldl * ((size_t)w.r + (size_t)a.f.nlay * b);
        saer[b * 128 + tr] = (float)(w.B->in[F_AERAOD][ab] * (1.0 - w.B->in[F_AERSSA][ab]));
      }
    }
    sync_for_mma();
    if (tid == 0) {
      umma::fence_after_sync();
      umma::mma(tb, umma::tile_desc(sbase + SM_X, KIN, 0), umma::tile_desc(sbase + SM_W1, KIN, 0), ID128, 0u);
      umma::commit(mbar);
    }
    if (!wait_mma()) break;

    // ---------------- hidden layers: quarter q owns hidden units [32q, 32q+32) ----------------
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
      const int dcol = layer == 0 ? 0 : 128;
      float v32[32];
      umma::tmem_ld32(umma::tmem_addr(tb, wl, dcol + 32 * q), v32);
#pragma unroll
      for (int h16 = 0; h16 < 2; ++h16) {
        const int c0 = 32 * q + 16 * h16;
        float* v = v32 + 16 * h16;
        float h[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float z = v[j] + (layer == 1 ? sb2[c0 + j] : 0.0f);
          v[j] = z;
          h[j] = silu(z);
        }
        umma::st_canon8(sm + SM_H, tr, c0, HID, h);
        umma::st_canon8(sm + SM_H, tr, c0 + 8, HID, h + 8);
        if (MODE == MODE_TRAIN && live) {
          bf16* z = (layer == 0 ? a.z1 : a.z2) + (size_t)row * HID + c0;
          __nv_bfloat162 zp[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) zp[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
          reinterpret_cast<uint4*>(z)[0] = reinterpret_cast<uint4*>(zp)[0];
          reinterpret_cast<uint4*>(z)[1] = reinterpret_cast<uint4*>(zp)[1];
          bf16* ht = (layer == 0 ? a.h1t : a.h2t);
#pragma unroll
          for (int j = 0; j < 16; ++j) ht[(size_t)(c0 + j) * a.ldt + row] = __float2bfloat16_rn(h[j]);
        }
      }
      sync_for_mma();
      if (tid == 0) {
        umma::fence_after_sync();
        if (layer == 0) {
#pragma unroll 1
          for (int s = 0; s < HID / 16; ++s)
            umma::mma(tb + 128, umma::tile_desc(sbase + SM_H, HID, s), umma::tile_desc(sbase + SM_W2, HID, s), ID128,
                      s > 0 ? 1u : 0u);
        } else {
#pragma unroll 1
          for (int s = 0; s < HID / 16; ++s)
            umma::mma(tb + 256, umma::tile_desc(sbase + SM_H, HID, s), umma::tile_desc(sbase + SM_W3, HID, s), ID144,
                      s > 0 ? 1u : 0u);
#pragma unroll 1
          for (int s = 0; s < HID / 16; ++s)
            umma::mma(tb, umma::tile_desc(sbase + SM_H, HID, s), umma::tile_desc(sbase + SM_W3 + W3_HALF, HID, s),
                      ID144, s > 0 ? 1u : 0u);
        }
        umma::commit(mbar);
      }
      if (!wait_mma()) break;
    }
    if (failed) break;

    // ---------------- output epilogue ----------------
    if (MODE == MODE_FEATS || MODE == MODE_TRAIN) {
      // quarter q owns outputs [72q, 72q+72) (8-aligned; 16-column TMEM chunks never straddle 144)
      const int ja = 72 * q, jb = ja + 72;
      float sse = 0.0f;
      const float coldry_s = (MODE == MODE_TRAIN && a.tau_weight && q < 2 && live) ? __ldg(a.feats + sample * NIN + 7) : 0.0f;
#pragma unroll 1
      for (int j0 = ja & ~15; j0 < jb; j0 += 16) {
        float v[16];
        umma::tmem_ld16(umma::tmem_addr(tb, wl, out_col(j0)), v);
        if (!live) continue;
#pragma unroll
        for (int g8 = 0; g8 < 2; ++g8) {
          const int jj = j0 + 8 * g8;
          if (jj < ja || jj >= jb) continue;
          float o[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) o[u] = v[8 * g8 + u] + sb3[jj + u];
          if (MODE == MODE_FEATS) {
            float4* dst = reinterpret_cast<float4*>(a.y + (size_t)row * NOP + jj);
            dst[0] = make_float4(o[0], o[1], o[2], o[3]);
            dst[1] = make_float4(o[4], o[5], o[6], o[7]);
          } else {
            const float4* tg = reinterpret_cast<const float4*>(a.targets + (size_t)sample * NOP + jj);
            const float4 t0 = __ldg(tg), t1 = __ldg(tg + 1);
            const float tt[8] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w};
            float d[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int j = jj + u;
              float wgt = 1.0f;
              if (a.tau_weight && j < 140) {
                // the layer's diffuse optical depth from the target: thin and moderate
                // layers set the fluxes, errors of opaque ones hardly matter
                const float tau = 1.66f * __expf(tt[u] * snorm[SG_OUT_STD + j] + snorm[SG_OUT_MEAN + j]) * coldry_s;
                wgt = 1.0f / (1.0f + tau);
              }
              const float e = pad_out_row(j) ? 0.0f : o[u] - tt[u];
              sse += wgt * e * e;
              d[u] = wgt * e * a.loss_scale;
            }
            __nv_bfloat162 dp[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) dp[u] = __floats2bfloat162_rn(d[2 * u], d[2 * u + 1]);
            *reinterpret_cast<uint4*>(a.dy + (size_t)row * NOP + jj) = *reinterpret_cast<uint4*>(dp);
#pragma unroll
            for (int u = 0; u < 8; ++u) a.dyt[(size_t)(jj + u) * a.ldt + row] = __float2bfloat16_rn(d[u]);
          }
        }
      }
      if (MODE == MODE_TRAIN) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sse += __shfl_xor_sync(0xffffffffu, sse, o);
        if ((tid & 31) == 0) atomicAdd(a.loss, sse);
      }
    } else {   // MODE_LW
      // quarters own whole bands: g-points [0,38), [38,68), [68,108), [108,140)
      const size_t nlp = (size_t)a.f.nlay <= 63 ? 64 : (size_t)a.f.nlay <= 127 ? 128 : 256;   // 32 V
      int cc = 0, t = 0;
      if (live) {
        cc = (int)(row / a.f.nlay);
        t = (int)(row - (long)cc * a.f.nlay);
      }
      float* tcol = a.sc.tau + (size_t)cc * NGPT * nlp + t;
      float* fcol = a.sc.frac + (size_t)cc * NGPT * nlp + t;
      const float cd = scd[tr];
      const float* ar = saer + tr;
      if (q == 0) lw_out_quarter<0, 38>(tb, wl, live, tcol, fcol, nlp, osc, osh, ar, cd);
      else if (q == 1) lw_out_quarter<38, 68>(tb, wl, live, tcol, fcol, nlp, osc, osh, ar, cd);
      else if (q == 2) lw_out_quarter<68, 108>(tb, wl, live, tcol, fcol, nlp, osc, osh, ar, cd);
      else lw_out_quarter<108, 140>(tb, wl, live, tcol, fcol, nlp, osc, osh, ar, cd);
    }
    // The next tile's first barrier orders these TMEM reads before MMA1 overwrites
    // the accumulators, and its per-tile rows use the other buffer.
    umma::fence_before_sync();
  }
  // leave: every MMA this CTA issued has completed (or the wait timed out and
  // the error is recorded); release tensor memory
  if (failed) umma::mbar_wait(mbar, phase ^ 1u, 1u << 20);   // one more bounded wait for the MMA in flight
  umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && *sfail && a.err) atomicCAS(a.err, 0, 1);
  if (warp == 0) umma::tmem_dealloc(tb, 512);
}

// ---------------------------------------------------------------------------
// Network stage of the learned-gas-optics column path (lw_sg_path.cu).  One
// column per 128-row tile: row t is layer t (surface first), rows nlay..127
// are padding.  Per tile: the layers' features and aerosol depths (their
// loads issued during the previous tile's output stage), MMA1 -> SiLU ->
// MMA2 -> SiLU -> MMA3, then the 140 optical depths and the 140 band-
// normalised Planck fractions (the values of lw_out_quarter), written
// straight into the column's hand-off [nlay/8][tau 140 | frac 140][8 layers]
// (a warp's 32 rows cover four 8-layer blocks, 16 contiguous bytes each per
// g-point).  The hidden layers' SiLU is 0.5 z (1 + tanh(0.5 z)) with the
// packed FP16 hardware tanh, one special-function operation per two values;
// H1, H2, W2 and W3 are FP16 operands (W2 the trained BF16 weights, exact in
// FP16), the features and W1 BF16.
//
// Two pipelines per CTA (below) each run that chain on their own columns.
// The output layer's normalisation is folded into MMA3: each CTA builds its
// W3 tile from the FP32 master weights with row j scaled by the output's
// standard deviation (times log2 e for the optical depths), and three extra
// K columns that carry the output's shift (b3 std + mean, the same scaling)
// as a BF16 hi + mid + lo split against constant-one columns of H2 (K = 144).
// The accumulator then holds log2(tau / coldry) and the fraction itself.
// The second layer's bias rides on MMA2 the same way (three extra K columns
// of W2 against the constant-one columns of H1), so the hidden epilogues
// read no bias.  The constant columns [128, 144) of the H tile are written
// once: the SiLU epilogues only write columns [0, 128).
constexpr int KH3 = HID + 16;                                  // K of MMA2 and MMA3: H + {1, 1, 1, 0 ...}
// Two independent tile pipelines per CTA (warps 0-7 and 8-15): while one
// waits for its MMAs or its barrier, the other runs its epilogues.  Each
// pipeline owns 144 TMEM columns, its X and H tiles and its per-tile rows;
// the weights are shared.
constexpr int HP = 2;                                          // pipelines per CTA
constexpr int HP_THREADS = FWD_THREADS / HP;                   // 256: two threads per tile row
constexpr uint32_t HSM_W1 = 0;                                 // canon [128][16]
constexpr uint32_t HSM_W2 = HSM_W1 + HID * KIN * 2;            // canon [128][144]
constexpr uint32_t HSM_W3 = HSM_W2 + HID * KH3 * 2;            // canon [288][144]
constexpr uint32_t HSM_P = HSM_W3 + NOP * KH3 * 2;             // per pipeline, HSM_PB bytes each:
constexpr uint32_t HPO_X = 0;                                  //   canon [128][16]
constexpr uint32_t HPO_H = HPO_X + 128 * KIN * 2;              //   canon [128][144]: H1 / H2 + {1, 1, 1, 0 ...}
constexpr uint32_t HPO_AER = HPO_H + 128 * KH3 * 2;            //   f16 [16][128] aerosol tau of the tile's layers
constexpr uint32_t HPO_CD = HPO_AER + NBANDS * 128 * 2;        //   f32 [128] coldry of the tile's layers
constexpr uint32_t HSM_PB = HPO_CD + 128 * 4;
constexpr uint32_t HSM_NORM = HSM_P + HP * HSM_PB;             // f32 [16] input mean, 1 / std
constexpr uint32_t HSM_BAR = HSM_NORM + 16 * 4;                // per pipeline: mbarrier (8 B); TMEM base; failure flag
constexpr uint32_t H_SMEM = HSM_BAR + 64;
static_assert(H_SMEM > 116 * 1024 && H_SMEM <= 227 * 1024, "one CTA per SM (512 TMEM columns), within shared memory");
static_assert(HSM_W3 % 128 == 0 && HSM_P % 128 == 0 && HSM_PB % 128 == 0 && HPO_H % 128 == 0, "canonical tiles");
constexpr uint32_t W3H_HALF = 144 * KH3 * 2;                   // second 144-row B operand of MMA3
constexpr float kLog2e = 1.4426950408889634f;

// SiLU of a pair, z sigmoid(z) = 0.5 z (1 + tanh(0.5 z)), in FP16 arithmetic:
// the pair rounded to FP16 (the operand type of MMA2 and MMA3 here), then
// h + h tanh(h) with h = z / 2 (exact), the packed hardware tanh (relative
// error ~2^-11, as the FP32 one) and one packed FMA.  FP16 keeps three more
// mantissa bits than the BF16 the network was trained with; BF16 pair
// arithmetic here raised the flux RMSE from 0.097 to 0.40 W/m2.
__device__ __forceinline__ uint32_t silu_f16x2(float z0, float z1) {
  const __half2 hz = __hmul2(__floats2half2_rn(z0, z1), __float2half2_rn(0.5f));
  const uint32_t hb = *reinterpret_cast<const uint32_t*>(&hz);
  uint32_t tb;
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(tb) : "r"(hb));
  const __half2 r = __hfma2(hz, *reinterpret_cast<const __half2*>(&tb), hz);
  return *reinterpret_cast<const uint32_t*>(&r);
}
__device__ __forceinline__ float ex2_fast(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// FP16 values of g-points g and g + 1 of this row and of the neighbouring
// row (lane ^ 1) as one 4-byte store each: the even row stores g-point g of
// rows (t, t + 1), the odd row g-point g + 1 of rows (t - 1, t).  dst_g is
// this row's slot of g-point g; a g-point's rows are adjacent in the hand-off.
// Every lane takes part in the exchange; rows past the column's last 8-layer
// block (store false, both rows of a pair alike) store nothing.
__device__ __forceinline__ void st_pair(__half* dst_g, int stride, bool odd, bool store, float v0, float v1) {
  const __half2 w = __floats2half2_rn(v0, v1);
  const uint32_t W = *reinterpret_cast<const uint32_t*>(&w);
  const uint32_t X = __shfl_xor_sync(0xffffffffu, W, 1);
  if (store) *reinterpret_cast<uint32_t*>(odd ? dst_g + stride - 1 : dst_g) = __byte_perm(W, X, odd ? 0x3276u : 0x5410u);
}

// FP16 values of g-points g..g+3 of this row and of the other rows of its
// 4-row group (lanes 4k..4k+3, layers of one 8-layer block) as one 8-byte
// store each: row q of the group stores g-point g + q of the group's four
// layers.  Two exchanges: rows q and q^2 swap one g-point pair, then rows q
// and q^1 swap halves.
__device__ __forceinline__ void st_quad(__half* dst_g, int stride, int q, bool store, float v0, float v1, float v2,
                                        float v3) {
  const __half2 a = __floats2half2_rn(v0, v1), b = __floats2half2_rn(v2, v3);
  const uint32_t w0 = *reinterpret_cast<const uint32_t*>(&a), w1 = *reinterpret_cast<const uint32_t*>(&b);
  const bool hi = q & 2, odd = q & 1;
  const uint32_t r1 = __shfl_xor_sync(0xffffffffu, hi ? w0 : w1, 2);
  // pair P (g, g+1 for rows 0-1; g+2, g+3 for rows 2-3) at layers (q & 1) and (q & 1) + 2
  const uint32_t x0 = hi ? r1 : w0, x1 = hi ? w1 : r1;
  const uint32_t r2 = __shfl_xor_sync(0xffffffffu, __byte_perm(x0, x1, odd ? 0x5410u : 0x7632u), 1);
  uint2 out;
  out.x = __byte_perm(x0, r2, odd ? 0x3254u : 0x5410u);
  out.y = __byte_perm(x1, r2, odd ? 0x3276u : 0x7610u);
  if (store) *reinterpret_cast<uint2*>(dst_g + q * stride - q) = out;
}

// optical depths of g-points [GA, GB) of this thread's row, FP16 at
// dst[g stride]: 2^acc * coldry + aerosol.  Every lane runs the TMEM loads
// (tcgen05.ld is a warp-wide instruction) and the store exchanges; padding
// rows inside the column's last 8-layer block store zeros.
template <int GA, int GB>
__device__ __forceinline__ void h_out_tau(uint32_t tb, int wl, int stride, bool live, int q, bool store, __half* dst,
                                          const __half* aer_row, float cd) {
  static_assert((GB - GA) % 2 == 0, "g-point pairs");
  constexpr int C0 = GA & ~15, NCH = (GB - C0 + 15) / 16;
  float v[NCH * 16];
#pragma unroll
  for (int c = 0; c < NCH; ++c) umma::tmem_ld16(umma::tmem_addr(tb, wl, C0 + 16 * c), v + 16 * c);
#pragma unroll
  for (int g = GA; g < GB; ++g) {
    const float e = ex2_fast(v[g - C0]);   // unconditional: a select, not a branch, drops padding rows
    v[g - C0] = live ? fminf(fmaf(e, cd, __half2float(aer_row[band_of_g(g) * 128])), 6.0e4f)
                     : 0.0f;   // below the FP16 maximum
  }
#pragma unroll
  for (int g = GA; g + 4 <= GB; g += 4)
    st_quad(dst + g * stride, stride, q, store, v[g - C0], v[g + 1 - C0], v[g + 2 - C0], v[g + 3 - C0]);
  if ((GB - GA) % 4) st_pair(dst + (GB - 2) * stride, stride, q & 1, store, v[GB - 2 - C0], v[GB - 1 - C0]);
}

// band-normalised Planck fractions of g-points [GA, GB) (whole bands), FP16 at dst[g stride]
template <int GA, int GB>
__device__ __forceinline__ void h_out_frac(uint32_t tb, int wl, int stride, bool live, int q, bool store,
                                           __half* dst) {
  static_assert((GB - GA) % 2 == 0, "g-point pairs");
  constexpr int C0 = GA & ~15, NCH = (GB - C0 + 15) / 16;
  float v[NCH * 16];
#pragma unroll
  for (int c = 0; c < NCH; ++c) umma::tmem_ld16(umma::tmem_addr(tb, wl, C0 + 16 * c), v + 16 * c);
  float bsum[NBANDS];
#pragma unroll
  for (int b = 0; b < NBANDS; ++b) bsum[b] = 0.0f;
#pragma unroll
  for (int g = GA; g < GB; ++g) {
    const float fr = __saturatef(v[g - C0]);
    v[g - C0] = fr;
    bsum[band_of_g(g)] += fr;
  }
#pragma unroll
  for (int b = 0; b < NBANDS; ++b) bsum[b] = bsum[b] > 0.0f ? __fdividef(1.0f, bsum[b]) : 1.0f;   // FP16 results
#pragma unroll
  for (int g = GA; g < GB; ++g) v[g - C0] = live ? v[g - C0] * bsum[band_of_g(g)] : 0.0f;
#pragma unroll
  for (int g = GA; g + 4 <= GB; g += 4)
    st_quad(dst + g * stride, stride, q, store, v[g - C0], v[g + 1 - C0], v[g + 2 - C0], v[g + 3 - C0]);
  if ((GB - GA) % 4) st_pair(dst + (GB - 2) * stride, stride, q & 1, store, v[GB - 2 - C0], v[GB - 1 - C0]);
}

// Per-column network inputs of the column path, packed by mlp_h_pack_kernel
// into the work area (kSgPackBytes per chunk column):
//   [128 rows][8] BF16  the normalised features x0..x6 and the constant 1
//                       (padding rows zero): the first 8 columns of the X tile
//   [128] FP32          coldry (RLM:835, 947)
//   [16 bands][128] FP16 aerosol optical depth aod (1 - ssa) (RLM:877-880, 986-989)
// The inputs lie column-fastest ((ldim, nlay) arrays), so the network's
// one-column tiles read them at a stride of a whole layer row; the pack
// kernel reads them 16 columns at a time (one whole 128-byte line per layer
// and field), stages 16 records in shared memory and writes them
// contiguously, and the network then reads a column's 6.5 KB record with
// coalesced 16-byte loads.  The same kernel runs the envelope test and lists
// the columns that need the fallback.
constexpr uint32_t PK_X = 0, PK_CD = 128 * 16, PK_AER = PK_CD + 128 * 4;
static_assert(PK_AER + NBANDS * 128 * 2 == kSgPackBytes, "packed column record");
constexpr int PK_COLS = 16, PK_THREADS = 256;   // 16 columns x 16 layers per step
// staged records 16 bytes apart in shared-memory banks (the record size is a multiple of 128 bytes)
constexpr uint32_t PK_STRIDE = kSgPackBytes + 16;
constexpr uint32_t PK_SMEM = PK_COLS * PK_STRIDE + 64;

__global__ void __launch_bounds__(PK_THREADS, 2) mlp_h_pack_kernel(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char st[];   // PK_COLS records of PK_STRIDE bytes, then snorm
  float* snorm = reinterpret_cast<float*>(st + PK_COLS * PK_STRIDE);   // input mean, 1 / std
  if (threadIdx.x < 16)
    snorm[threadIdx.x] = threadIdx.x < 8 ? a.norm[SG_IN_MEAN + threadIdx.x] : 1.0f / a.norm[SG_IN_STD + threadIdx.x - 8];
  __syncthreads();
  const int j = threadIdx.x & (PK_COLS - 1), tl = threadIdx.x / PK_COLS;
  const int nlay = a.f.nlay;
  const bool top = a.f.top_at_1 != 0;
  unsigned char* rec = st + j * PK_STRIDE;
  for (int cb = blockIdx.x * PK_COLS; cb < a.nc; cb += gridDim.x * PK_COLS) {
    const int cc = cb + j;
    const int c = a.c0 + cc;
    const bool colok = cc < a.nc;
    // the column's block: its field pointers straight from the kernel
    // arguments (one block) or from the block table
    const int bi = (a.nblocks == 1 || !colok) ? 0 : __ldg(a.colmap + c);
    auto fld = [&](int k) -> const double* { return a.nblocks == 1 ? a.b0.in[k] : a.blocks[bi].in[k]; };
    const size_t ld = (size_t)(a.nblocks == 1 ? a.b0.ld : a.blocks[bi].ld);
    const int col0 = a.nblocks == 1 ? a.b0.col0 : a.blocks[bi].col0;
#pragma unroll 1
    for (int t = tl; t < 128; t += PK_THREADS / PK_COLS) {
      float x[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
      float cd = 0.0f;
      __half2 aer[NBANDS / 2];
#pragma unroll
      for (int b = 0; b < NBANDS / 2; ++b) aer[b] = __floats2half2_rn(0.0f, 0.0f);
      if (colok && t < nlay) {
        const size_t o = (size_t)(c - col0) + ld * (size_t)(top ? nlay - 1 - t : t);
        const double pavel = fld(F_PLYR)[o], tavel = fld(F_TLYR)[o], qv = fld(F_QLYR)[o];
        const double o3 = fld(F_OLYR)[o], co2 = fld(F_CO2)[o], ch4 = fld(F_CH4)[o], n2o = fld(F_N2O)[o];
        const double delp = fld(F_DELPIN)[o];
        const double* paod = fld(F_AERAOD);
        const double* pssa = fld(F_AERSSA);
        double aod[NBANDS], ssa[NBANDS];
#pragma unroll
        for (int b = 0; b < NBANDS; ++b) {   // every load first, so their latencies overlap
          const size_t ab = o + ld * (size_t)nlay * (size_t)b;
          aod[b] = paod[ab];
          ssa[b] = pssa[ab];
        }
        const double amdw = 28.9644 / 18.0154, amdo3 = 28.9644 / 47.9982;
        const double h2ovmr = fmax(0.0, qv * amdw / (1.0 - qv));
        const double o3vmr = fmax(0.0, o3 * amdo3);
        const double tem0 = (1.0 - h2ovmr) * 28.9644 + h2ovmr * 18.0154;
        cd = (float)((1.0e-20 * 1.0e3 * 6.0221415e23) * delp / (100.0 * 9.80665 * tem0 * (1.0 + h2ovmr)));
        float raw[NIN];
        layer_features(pavel, tavel, h2ovmr, o3vmr, co2, ch4, n2o, raw);
        // a layer outside the training envelope: list its column once for the fallback
        if (!in_envelope(raw, a.norm) && atomicExch(a.fb_flag + c, 1u) == 0u) a.fb_list[atomicAdd(a.fb_count, 1)] = c;
#pragma unroll
        for (int k = 0; k < 7; ++k) x[k] = (raw[k] - snorm[k]) * snorm[8 + k];
        x[7] = 1.0f;
#pragma unroll
        for (int b = 0; b < NBANDS / 2; ++b)
          aer[b] = __floats2half2_rn((float)(aod[2 * b] * (1.0 - ssa[2 * b])), (float)(aod[2 * b + 1] * (1.0 - ssa[2 * b + 1])));
      }
      __nv_bfloat162 xb[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) xb[k] = __floats2bfloat162_rn(x[2 * k], x[2 * k + 1]);
      *reinterpret_cast<uint4*>(rec + PK_X + 16 * t) = *reinterpret_cast<const uint4*>(xb);
      *reinterpret_cast<float*>(rec + PK_CD + 4 * t) = cd;
      __half* ra = reinterpret_cast<__half*>(rec + PK_AER) + t;
#pragma unroll
      for (int b = 0; b < NBANDS / 2; ++b) {
        ra[(2 * b) * 128] = __low2half(aer[b]);
        ra[(2 * b + 1) * 128] = __high2half(aer[b]);
      }
    }
    __syncthreads();
    // the records of chunk columns [cb, cb + n) are contiguous in the work area
    const int n = min(PK_COLS, a.nc - cb);
    constexpr int Q = (int)(kSgPackBytes / 16);   // 16-byte pieces of a record
    uint4* dst = reinterpret_cast<uint4*>(a.pk + (size_t)cb * kSgPackBytes);
    for (int q = threadIdx.x; q < n * Q; q += PK_THREADS)
      dst[q] = *reinterpret_cast<const uint4*>(st + (q / Q) * PK_STRIDE + 16 * (q % Q));
    __syncthreads();
  }
}

__global__ void __launch_bounds__(FWD_THREADS, 1) mlp_h_kernel(FwdArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, wl = warp & 3;
  const int P = warp / (HP_THREADS / 32);            // this thread's pipeline
  const int ptid = tid - P * HP_THREADS;              // thread within the pipeline
  const int h = (warp % (HP_THREADS / 32)) / 4;       // half of the pipeline: two threads per row
  const int t = 32 * wl + (tid & 31);                 // tile row = layer
  float* snorm = reinterpret_cast<float*>(sm + HSM_NORM);
  unsigned char* pbase = sm + HSM_P + P * HSM_PB;
  __half* saer = reinterpret_cast<__half*>(pbase + HPO_AER);
  float* scd = reinterpret_cast<float*>(pbase + HPO_CD);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + HSM_BAR) + P;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + HSM_BAR + 16);
  int* sfail = reinterpret_cast<int*>(sm + HSM_BAR + 20);

  copy_rows_canon(sm + HSM_W1, a.ops + O_W1, HID, KIN, tid);
  // W2 in FP16: the trained BF16 weights (exact in FP16 down to 2^-14), the
  // bias as three FP16 terms in columns 128..130
  for (int ch = tid; ch < HID * (KH3 / 8); ch += FWD_THREADS) {
    const int j = ch / (KH3 / 8), k = (ch % (KH3 / 8)) * 8;
    float w[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (k < HID) {
#pragma unroll
      for (int u = 0; u < 8; ++u) w[u] = __bfloat162float(a.ops[O_W2 + (size_t)j * HID + k + u]);
    } else if (k == HID) {
      const float b = a.params[P_B2 + j];
      w[0] = __half2float(__float2half_rn(b));
      w[1] = __half2float(__float2half_rn(b - w[0]));
      w[2] = b - w[0] - w[1];
    }
    umma::st_canon8_h(sm + HSM_W2, j, k, KH3, w);
  }
  // the constant columns of both pipelines' H tiles, and the zero columns 8..15 of their X tiles
  for (int r = tid; r < HP * 128; r += FWD_THREADS) {
    const float one[8] = {1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const float zero[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    unsigned char* pt = sm + HSM_P + (r >> 7) * HSM_PB;
    umma::st_canon8_h(pt + HPO_H, r & 127, HID, KH3, one);
    umma::st_canon8_h(pt + HPO_H, r & 127, HID + 8, KH3, zero);
    umma::st_canon8(pt + HPO_X, r & 127, 8, KIN, zero);
  }
  // W3 with the output normalisation folded in (rows scaled, the shift as
  // three BF16 terms in columns 128..130), from the FP32 master weights
  for (int ch = tid; ch < NOP * (KH3 / 8); ch += FWD_THREADS) {
    const int j = ch / (KH3 / 8), k = (ch % (KH3 / 8)) * 8;
    const bool pad = pad_out_row(j);
    const float sd = a.norm[SG_OUT_STD + j];
    const float scale = j < 144 ? sd * kLog2e : sd;
    float w[8];
    if (k < HID) {
#pragma unroll
      for (int u = 0; u < 8; ++u) w[u] = pad ? 0.0f : a.params[P_W3 + j * HID + k + u] * scale;
    } else {
      const float sh = fmaf(a.params[P_B3 + j], sd, a.norm[SG_OUT_MEAN + j]) * (j < 144 ? kLog2e : 1.0f);
      const float hi = pad ? 0.0f : __half2float(__float2half_rn(sh));
      const float mid = pad ? 0.0f : __half2float(__float2half_rn(sh - hi));
      const float lo = pad ? 0.0f : sh - hi - mid;
#pragma unroll
      for (int u = 0; u < 8; ++u) w[u] = 0.0f;
      if (k == HID) { w[0] = hi; w[1] = mid; w[2] = lo; }
    }
    umma::st_canon8_h(sm + HSM_W3, j, k, KH3, w);
  }
  if (tid < 16) snorm[tid] = tid < 8 ? a.norm[SG_IN_MEAN + tid] : 1.0f / a.norm[SG_IN_STD + tid - 8];
  if (warp == 0) {
    umma::tmem_alloc(tslot, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(reinterpret_cast<uint64_t*>(sm + HSM_BAR), 1);
    umma::mbar_init(reinterpret_cast<uint64_t*>(sm + HSM_BAR) + 1, 1);
    *sfail = 0;
  }
  umma::fence_smem_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = *tslot + 256u * (uint32_t)P;     // this pipeline's TMEM columns [0, 144)
  const uint32_t sbase = umma::smem_u32(sm);
  const uint32_t sX = umma::smem_u32(pbase + HPO_X), sH = umma::smem_u32(pbase + HPO_H);
  // MMA1: BF16 features and W1; MMA2, MMA3: FP16 hidden activations and weights
  constexpr uint32_t ID1 = umma::idesc_bf16(128, 128), ID128 = umma::idesc_f16(128, 128),
                     ID144 = umma::idesc_f16(128, 144);
  const GroupSync psync{1 + P, HP_THREADS};           // this pipeline's barrier
  const bool issuer = ptid == 0;
  uint32_t phase = 0;
  bool failed = false;   // uniform across the pipeline
  auto wait_mma = [&]() -> bool {
    const bool ok = umma::mbar_wait(mbar, phase, c_fwd_wait_polls);
    phase ^= 1u;
    umma::fence_after_sync();
    if (psync.any(!ok)) {
      if (ptid == 0) atomicExch(sfail, 1);
      failed = true;
      return false;
    }
    return true;
  };
  auto sync_for_mma = [&]() {
    umma::fence_smem_async();
    umma::fence_before_sync();
    psync.sync();
  };
  auto mma3 = [&](uint32_t w3) {   // one half of the output layer into the pipeline's columns
    if (issuer) {
      umma::fence_after_sync();
#pragma unroll 1
      for (int s = 0; s < KH3 / 16; ++s)
        umma::mma(tb, umma::tile_desc(sH, KH3, s), umma::tile_desc(sbase + HSM_W3 + w3, KH3, s), ID144,
                  s > 0 ? 1u : 0u);
      umma::commit(mbar);
    }
  };

  const int nlay = a.f.nlay, nchk = (nlay + 7) >> 3;
  const bool live = t < nlay;
  const int q4 = t & 3;   // row within its 4-row group of the hand-off stores
  const bool inblk = t < 8 * nchk;   // the row lies in one of the column's 8-layer hand-off blocks

  // The column's packed inputs -> X (its feature columns), coldry and aerosol
  // rows, as 16-byte asynchronous copies issued a tile ahead: for the next
  // tile once this one's optical depths are out (X has been free since MMA1),
  // so they land during MMA3 and the fractions.
  auto prefetch = [&](int col) {
    const unsigned char* rec = a.pk + (size_t)col * kSgPackBytes;
    if (h == 0) umma::cp_async16(pbase + HPO_X + umma::canon_off(t, 0, KIN), rec + PK_X + 16 * t);
    umma::cp_async16(reinterpret_cast<unsigned char*>(saer) + 16 * ptid, rec + PK_AER + 16 * ptid);
    if (ptid < 32) umma::cp_async16(reinterpret_cast<unsigned char*>(scd) + 16 * ptid, rec + PK_CD + 16 * ptid);
    umma::cp_async_commit();
  };
  const int cstep = HP * gridDim.x;
  if (HP * (int)blockIdx.x + P < a.nc) prefetch(HP * blockIdx.x + P);

  for (int cc = HP * blockIdx.x + P; cc < a.nc; cc += cstep) {
    umma::cp_async_wait_all();   // this thread's copies of the tile's inputs
    sync_for_mma();
    if (issuer) {
      umma::fence_after_sync();
      umma::mma(tb, umma::tile_desc(sX, KIN, 0), umma::tile_desc(sbase + HSM_W1, KIN, 0), ID1, 0u);
      umma::commit(mbar);
    }
    if (!wait_mma()) break;

    // ---------------- hidden layers: half h owns hidden units [64h, 64h+64) ----------------
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
      // H1 feeds MMA2 and H2 feeds MMA3, both with the biases against the constant columns
#pragma unroll 1
      for (int part = 0; part < 2; ++part) {
        const int u0 = 64 * h + 32 * part;
        float v32[32];
        umma::tmem_ld32(umma::tmem_addr(tb, wl, u0), v32);
#pragma unroll
        for (int h8 = 0; h8 < 4; ++h8) {
          const int c0 = u0 + 8 * h8;
          uint32_t w[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) w[j] = silu_f16x2(v32[8 * h8 + 2 * j], v32[8 * h8 + 2 * j + 1]);
          *reinterpret_cast<uint4*>(pbase + HPO_H + umma::canon_off(t, c0, KH3)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
      }
      sync_for_mma();
      if (layer == 0) {
        if (issuer) {
          umma::fence_after_sync();
#pragma unroll 1
          for (int s = 0; s < KH3 / 16; ++s)
            umma::mma(tb, umma::tile_desc(sH, KH3, s), umma::tile_desc(sbase + HSM_W2, KH3, s), ID128, s > 0 ? 1u : 0u);
          umma::commit(mbar);
        }
      } else {
        mma3(0);   // optical depths: W3 rows [0, 144)
      }
      if (!wait_mma()) break;
    }
    if (failed) break;

    // ---------------- outputs into the hand-off ----------------
    // this row's slot of g-point 0 in its 8-layer block; g-point g at [8 g]
    __half* hrow = a.hnd + ((size_t)cc * nchk + (t >> 3)) * (2 * NGPT * 8) + (t & 7);
    const float cd = live ? scd[t] : 0.0f;
    const __half* ar = saer + t;
    // the two halves of a row own whole bands: g-points [0, 68) and [68, 140), in two passes each
    if (h == 0) {
      h_out_tau<0, 38>(tb, wl, 8, live, q4, inblk, hrow, ar, cd);
      h_out_tau<38, 68>(tb, wl, 8, live, q4, inblk, hrow, ar, cd);
    } else {
      h_out_tau<68, 108>(tb, wl, 8, live, q4, inblk, hrow, ar, cd);
      h_out_tau<108, 140>(tb, wl, 8, live, q4, inblk, hrow, ar, cd);
    }
    sync_for_mma();   // the optical depths are read out of TMEM; coldry and aerosol rows are free
    if (cc + cstep < a.nc) prefetch(cc + cstep);
    mma3(W3H_HALF);   // fractions: W3 rows [144, 288)
    if (!wait_mma()) break;
    hrow += 8 * NGPT;
    if (h == 0) {
      h_out_frac<0, 38>(tb, wl, 8, live, q4, inblk, hrow);
      h_out_frac<38, 68>(tb, wl, 8, live, q4, inblk, hrow);
    } else {
      h_out_frac<68, 108>(tb, wl, 8, live, q4, inblk, hrow);
      h_out_frac<108, 140>(tb, wl, 8, live, q4, inblk, hrow);
    }
    // the accumulators and this tile's rows are free for the next tile
    umma::fence_before_sync();
    psync.sync();
  }
  if (failed) umma::mbar_wait(mbar, phase ^ 1u, 1u << 20);   // one more bounded wait for the MMA in flight
  umma::cp_async_wait_all();   // no copy still in flight after a time-out
  umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && *sfail && a.err) atomicCAS(a.err, 0, 1);
  if (warp == 0) umma::tmem_dealloc(*tslot, 512);
}

// ---------------------------------------------------------------------------
// C[M x N] = A[M x K] * B[N x K]^T, BF16 in, FP32 accumulate (backward pass)
enum { EPI_ATOMIC = 0, EPI_DACT = 1 };

struct GemmArgs {
  const bf16* A; long lda;
  const bf16* B; long ldb;
  int M, N, K, kslice;
  float* C; long ldc;               // EPI_ATOMIC
  const bf16* Z; long ldz;          // EPI_DACT
  bf16* D; long ldd;                // EPI_DACT row-major out (nullable)
  bf16* Dt; long lddt;              // EPI_DACT transposed out (nullable)
  int* err;
};

constexpr int GK = 64;                                   // K per staged chunk
constexpr uint32_t GSM_A = 0;                            // canon [128][64]
constexpr uint32_t GSM_B = GSM_A + 128 * GK * 2;         // canon [288][64]
constexpr uint32_t GSM_BAR = GSM_B + 288 * GK * 2;
constexpr uint32_t GEMM_SMEM_MIN = GSM_BAR + 32;
constexpr uint32_t GEMM_SMEM = 120 * 1024;               // > half an SM: one CTA per SM (512 TMEM columns)
static_assert(GEMM_SMEM >= GEMM_SMEM_MIN, "gemm shared memory");

template <int EPI>
__global__ void __launch_bounds__(128, 1) gemm_tn_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + GSM_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + GSM_BAR + 8);
  if (warp == 0) {
    umma::tmem_alloc(tslot, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) umma::mbar_init(mbar, 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t sbase = umma::smem_u32(sm);
  const int m0 = blockIdx.x * 128;
  const int kb = blockIdx.y * g.kslice, ke = min(g.K, kb + g.kslice);
  const int nsplit = g.N > 256 ? 2 : 1, nh = g.N / nsplit;
  const uint32_t idesc = umma::idesc_bf16(128, nh);
  uint32_t phase = 0;
  bool ok = true, any = false;
  for (int k0 = kb; k0 < ke; k0 += GK) {
    const int kc = min(GK, ke - k0);   // multiple of 16
    // stage A [128 x kc] and B [N x kc] (zero-fill the unused K of a short chunk)
    for (int c = tid; c < 128 * (GK / 8); c += 128) {
      const int r = c / (GK / 8), k = (c % (GK / 8)) * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (k < kc && m0 + r < g.M) v = __ldg(reinterpret_cast<const uint4*>(g.A + (size_t)(m0 + r) * g.lda + k0 + k));
      *reinterpret_cast<uint4*>(sm + GSM_A + umma::canon_off(r, k, GK)) = v;
    }
    for (int c = tid; c < g.N * (GK / 8); c += 128) {
      const int r = c / (GK / 8), k = (c % (GK / 8)) * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (k < kc) v = __ldg(reinterpret_cast<const uint4*>(g.B + (size_t)r * g.ldb + k0 + k));
      *reinterpret_cast<uint4*>(sm + GSM_B + umma::canon_off(r, k, GK)) = v;
    }
    umma::fence_smem_async();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      for (int s = 0; s < kc / 16; ++s)
        for (int h = 0; h < nsplit; ++h)
          umma::mma(tb + (uint32_t)(h * nh), umma::tile_desc(sbase + GSM_A, GK, s),
                    umma::tile_desc(sbase + GSM_B + (uint32_t)(h * nh * GK * 2), GK, s), idesc,
                    (any || s > 0) ? 1u : 0u);
      umma::commit(mbar);
    }
    any = true;
    ok = umma::mbar_wait(mbar, phase);
    phase ^= 1u;
    umma::fence_after_sync();
    if (__syncthreads_or(!ok)) { ok = false; break; }
  }
  if (ok && any) {
    const int m = m0 + tid;
    for (int n0 = 0; n0 < g.N; n0 += 16) {
      float v[16];
      umma::tmem_ld16(umma::tmem_addr(tb, warp, n0), v);
      if (m >= g.M) continue;
      if (EPI == EPI_ATOMIC) {
#pragma unroll
        for (int j = 0; j < 16; ++j) atomicAdd(g.C + (size_t)m * g.ldc + n0 + j, v[j]);
      } else {
        float d[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) d[j] = v[j] * dsilu(__bfloat162float(g.Z[(size_t)m * g.ldz + n0 + j]));
        if (g.D) {
          __nv_bfloat162 dp[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) dp[j] = __floats2bfloat162_rn(d[2 * j], d[2 * j + 1]);
          uint4* dst = reinterpret_cast<uint4*>(g.D + (size_t)m * g.ldd + n0);
          dst[0] = reinterpret_cast<uint4*>(dp)[0];
          dst[1] = reinterpret_cast<uint4*>(dp)[1];
        }
        if (g.Dt) {
#pragma unroll
          for (int j = 0; j < 16; ++j) g.Dt[(size_t)(n0 + j) * g.lddt + m] = __float2bfloat16_rn(d[j]);
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && !ok && g.err) atomicCAS(g.err, 0, 1);
  if (warp == 0) umma::tmem_dealloc(tb, 512);
}

// ---------------------------------------------------------------------------
// Adam on the FP32 master weights, then the BF16 operand copies
__device__ inline void pack_param(int p, float w, bf16* ops) {
  const bf16 b = __float2bfloat16_rn(w);
  if (p < P_W2) {
    const int r = p / NIN, c = p % NIN;
    ops[O_W1 + r * KIN + c] = b;
  } else if (p < P_B2) {
    const int q = p - P_W2, r = q / HID, c = q % HID;
    ops[O_W2 + r * HID + c] = b;
    ops[O_W2T + c * HID + r] = b;
  } else if (p >= P_W3 && p < P_B3) {
    const int q = p - P_W3, r = q / HID, c = q % HID;
    ops[O_W3 + r * HID + c] = b;
    ops[O_W3T + c * NOP + r] = b;
  }
}

__device__ inline float grad_of(int p, const float* G) {
  if (p < P_W2) { const int r = p / NIN, c = p % NIN; return G[G_W1 + r * KIN + c]; }
  if (p < P_B2) { const int q = p - P_W2; return G[G_W2 + (q / HID) * GW2_LD + q % HID]; }
  if (p < P_W3) { return G[G_W2 + (p - P_B2) * GW2_LD + HID]; }
  if (p < P_B3) { const int q = p - P_W3; return G[G_W3 + (q / HID) * GW2_LD + q % HID]; }
  return G[G_W3 + (p - P_B3) * GW2_LD + HID];
}

__device__ inline bool frozen_param(int p) {   // padded output rows stay zero
  if (p >= P_W3 && p < P_B3) return pad_out_row((p - P_W3) / HID);
  if (p >= P_B3) return pad_out_row(p - P_B3);
  return false;
}

__global__ void adam_kernel(float* P, float* M, float* V, const float* G, bf16* ops, float lr, float b1, float b2,
                            float c1, float c2, float eps) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P_N; p += gridDim.x * blockDim.x) {
    float w = P[p];
    if (!frozen_param(p)) {
      const float gr = grad_of(p, G);
      const float m = b1 * M[p] + (1.0f - b1) * gr;
      const float v = b2 * V[p] + (1.0f - b2) * gr * gr;
      M[p] = m;
      V[p] = v;
      w -= lr * (m / c1) / (sqrtf(v / c2) + eps);
      P[p] = w;
    }
    pack_param(p, w, ops);
  }
}

__global__ void pack_kernel(const float* P, bf16* ops) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P_N; p += gridDim.x * blockDim.x) pack_param(p, P[p], ops);
}

// export the gradients in parameter order (gradient check)
__global__ void grads_kernel(const float* G, float* out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P_N; p += gridDim.x * blockDim.x)
    out[p] = frozen_param(p) ? 0.0f : grad_of(p, G);
}

// layer features and coldry of one block (internal layer order, surface first)
__global__ void features_kernel(Block B, int nlay, int top_at_1, float* feats, float* coldry_out) {
  const long n = (long)B.npts * nlay;
  for (long row = blockIdx.x * (long)blockDim.x + threadIdx.x; row < n; row += (long)gridDim.x * blockDim.x) {
    const int i = (int)(row / nlay), t = (int)(row - (long)i * nlay);
    const int r = top_at_1 ? nlay - t - 1 : t;
    const size_t o = (size_t)i + (size_t)B.ld * r;
    const double pavel = B.in[F_PLYR][o], tavel = B.in[F_TLYR][o], q = B.in[F_QLYR][o];
    const double amdw = 28.9644 / 18.0154, amdo3 = 28.9644 / 47.9982;
    const double h2ovmr = fmax(0.0, q * amdw / (1.0 - q));
    const double o3vmr = fmax(0.0, B.in[F_OLYR][o] * amdo3);
    const double tem0 = (1.0 - h2ovmr) * 28.9644 + h2ovmr * 18.0154;
    float x[SG_NFEAT];
    layer_features(pavel, tavel, h2ovmr, o3vmr, B.in[F_CO2][o], B.in[F_CH4][o], B.in[F_N2O][o], x);
    for (int j = 0; j < SG_NFEAT; ++j) feats[row * SG_NFEAT + j] = x[j];
    if (coldry_out)
      coldry_out[row] = (float)((1.0e-20 * 1.0e3 * 6.0221415e23) * B.in[F_DELPIN][o] /
                                (100.0 * 9.80665 * tem0 * (1.0 + h2ovmr)));
  }
}

// ---------------------------------------------------------------------------
// host side
namespace {

struct Net {
  bool ready = false;     // weights present (init or set)
  int device = -1;
  float* P = nullptr;     // master weights
  float* Madam = nullptr;
  float* Vadam = nullptr;
  float* G = nullptr;     // gradients
  bf16* ops = nullptr;    // operand copies
  float* norm = nullptr;  // SG_NORM_FLOATS
  int* err = nullptr;
  float* loss = nullptr;
  unsigned int* fallback = nullptr;   // layers the gas-optics kernel recomputed with taumol
  long adam_t = 0;
  int num_sms = 0;
  // training activations for batch `cap`
  long cap = 0;
  bf16 *xt = nullptr, *z1 = nullptr, *h1t = nullptr, *z2 = nullptr, *h2t = nullptr, *dy = nullptr, *dyt = nullptr,
       *dz2 = nullptr, *dz1t = nullptr;
  bool attrs = false;
};
Net net;
std::mutex net_mu;

void msg(char* e, int32_t n, const char* fmt, const char* what, cudaError_t c) {
  if (e && n > 0) std::snprintf(e, (size_t)n, fmt, what, cudaGetErrorString(c));
}
#define SG_CK(call, what)                                                                 \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      msg(errmsg, errmsg_len, "rrtmg_lw_gpu surrogate: %s failed: %s", what, e_);         \
      return 1;                                                                           \
    }                                                                                     \
  } while (0)
void smsg(char* e, int32_t n, const char* s) {
  if (e && n > 0) std::snprintf(e, (size_t)n, "%s", s);
}

cudaError_t set_attrs() {
  if (net.attrs) return cudaSuccess;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(mlp_fwd_kernel<MODE_FEATS>, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM)))
    return e;
  if ((e = cudaFuncSetAttribute(mlp_fwd_kernel<MODE_TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM)))
    return e;
  if ((e = cudaFuncSetAttribute(mlp_fwd_kernel<MODE_LW>, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM)))
    return e;
  if ((e = cudaFuncSetAttribute(mlp_h_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, H_SMEM))) return e;
  if ((e = cudaFuncSetAttribute(mlp_h_pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PK_SMEM))) return e;
  if ((e = cudaFuncSetAttribute(gemm_tn_kernel<EPI_ATOMIC>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM)))
    return e;
  if ((e = cudaFuncSetAttribute(gemm_tn_kernel<EPI_DACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM)))
    return e;
  // one CTA per SM is what makes the 512-column TMEM allocations safe
  int occ[6] = {0, 0, 0, 0, 0, 0};
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], mlp_fwd_kernel<MODE_FEATS>, FWD_THREADS, FWD_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], mlp_fwd_kernel<MODE_TRAIN>, FWD_THREADS, FWD_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], mlp_fwd_kernel<MODE_LW>, FWD_THREADS, FWD_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[3], gemm_tn_kernel<EPI_ATOMIC>, 128, GEMM_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[4], gemm_tn_kernel<EPI_DACT>, 128, GEMM_SMEM);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[5], mlp_h_kernel, FWD_THREADS, H_SMEM);
  for (int o : occ)
    if (o != 1) return cudaErrorLaunchOutOfResources;
  net.attrs = true;
  return cudaSuccess;
}

cudaError_t ensure_net(int device, int num_sms) {
  if (net.P && net.device == device) return cudaSuccess;
  cudaError_t e;
  net.device = device;
  net.num_sms = num_sms;
  if ((e = cudaMalloc(&net.P, sizeof(float) * P_N * 3))) return e;
  net.Madam = net.P + P_N;
  net.Vadam = net.P + 2 * P_N;
  if ((e = cudaMemset(net.P, 0, sizeof(float) * P_N * 3))) return e;
  if ((e = cudaMalloc(&net.G, sizeof(float) * G_N))) return e;
  if ((e = cudaMemset(net.G, 0, sizeof(float) * G_N))) return e;
  if ((e = cudaMalloc(&net.ops, sizeof(bf16) * O_N))) return e;
  if ((e = cudaMemset(net.ops, 0, sizeof(bf16) * O_N))) return e;
  if ((e = cudaMalloc(&net.norm, sizeof(float) * SG_NORM_FLOATS))) return e;
  if ((e = cudaMalloc(&net.err, 4 * sizeof(int)))) return e;
  net.loss = reinterpret_cast<float*>(net.err + 1);
  net.fallback = reinterpret_cast<unsigned int*>(net.err + 2);
  return cudaMemset(net.err, 0, 4 * sizeof(int));
}

cudaError_t ensure_batch(long batch) {
  if (net.cap >= batch) return cudaSuccess;
  bf16** bufs[] = {&net.xt, &net.z1, &net.h1t, &net.z2, &net.h2t, &net.dy, &net.dyt, &net.dz2, &net.dz1t};
  for (bf16** b : bufs)
    if (*b) { cudaFree(*b); *b = nullptr; }
  net.cap = 0;
  // rows: Xt 16, Z [B][128], H^T 144 (row 128 = 1), dY [B][288], dY^T 384, dZ2 [B][128], dZ1^T 128
  const size_t B = (size_t)batch;
  const size_t n[] = {16 * B, B * HID, 144 * B, B * HID, 144 * B, B * NOP, GW3_ROWS * B, B * HID, HID * B};
  cudaError_t e;
  for (int k = 0; k < 9; ++k) {
    if ((e = cudaMalloc(bufs[k], n[k] * sizeof(bf16)))) return e;
    if ((e = cudaMemset(*bufs[k], 0, n[k] * sizeof(bf16)))) return e;
  }
  // constant rows: the bias row of H1^T / H2^T and of X^T (feature 7 is written each step)
  std::vector<bf16> ones(B, __float2bfloat16_rn(1.0f));
  if ((e = cudaMemcpy(net.h1t + 128 * B, ones.data(), B * sizeof(bf16), cudaMemcpyHostToDevice))) return e;
  if ((e = cudaMemcpy(net.h2t + 128 * B, ones.data(), B * sizeof(bf16), cudaMemcpyHostToDevice))) return e;
  net.cap = batch;
  return cudaSuccess;
}

FwdArgs base_args() {
  FwdArgs a;
  std::memset(&a, 0, sizeof(a));
  a.ops = net.ops;
  a.params = net.P;
  a.norm = net.norm;
  a.err = net.err;
  return a;
}

cudaError_t launch_gemm(int epi, const GemmArgs& g, int ksplit, cudaStream_t st) {
  dim3 grid((g.M + 127) / 128, ksplit);
  if (epi == EPI_ATOMIC) gemm_tn_kernel<EPI_ATOMIC><<<grid, 128, GEMM_SMEM, st>>>(g);
  else gemm_tn_kernel<EPI_DACT><<<grid, 128, GEMM_SMEM, st>>>(g);
  return cudaGetLastError();
}

// forward (train mode) + backward of one batch: gradients accumulate in net.G
cudaError_t train_batch(const float* feats, const float* targets, long nsamp, long batch, long pa, long pb,
                        long off, int tau_weight, cudaStream_t st) {
  FwdArgs a = base_args();
  a.tau_weight = tau_weight;
  a.nrows = batch;
  a.feats = feats;
  a.targets = targets;
  a.perm_a = pa;
  a.perm_b = pb;
  a.perm_n = nsamp;
  a.perm_off = off;
  a.loss_scale = 2.0f / ((float)batch * (float)SG_NOUT);
  a.loss = net.loss;
  a.xt = net.xt; a.z1 = net.z1; a.h1t = net.h1t; a.z2 = net.z2; a.h2t = net.h2t; a.dy = net.dy; a.dyt = net.dyt;
  const long ldt = net.cap;   // pitch of the transposed activations (their constant rows sit at this pitch)
  a.ldt = ldt;
  const int tiles = (int)((batch + 127) / 128);
  mlp_fwd_kernel<MODE_TRAIN><<<std::min(tiles, net.num_sms), FWD_THREADS, FWD_SMEM, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  const int B = (int)batch;
  // dZ2 = (dY W3) * silu'(Z2): row-major for dH1, transposed for dW2
  GemmArgs g{};
  g.err = net.err;
  g.A = net.dy; g.lda = NOP; g.B = net.ops + O_W3T; g.ldb = NOP; g.M = B; g.N = HID; g.K = NOP; g.kslice = NOP;
  g.Z = net.z2; g.ldz = HID; g.D = net.dz2; g.ldd = HID; g.Dt = nullptr; g.lddt = 0;
  // dZ2^T (A operand of dW2) goes to the dZ1^T buffer: dW2 consumes it before dH1 overwrites it
  g.Dt = net.dz1t;
  g.lddt = ldt;
  if ((e = launch_gemm(EPI_DACT, g, 1, st))) return e;
  // dW3 += dY^T H2aug : [288 x B] x [144 x B]^T  (A rows 288..383 are zero)
  GemmArgs w3{};
  w3.err = net.err;
  w3.A = net.dyt; w3.lda = ldt; w3.B = net.h2t; w3.ldb = ldt; w3.M = NOP; w3.N = 144; w3.K = B;
  const int ks = std::max(1, std::min(32, B / 256));
  w3.kslice = ((B / ks + 63) / 64) * 64;
  w3.C = net.G + G_W3; w3.ldc = GW2_LD;
  if ((e = launch_gemm(EPI_ATOMIC, w3, (B + w3.kslice - 1) / w3.kslice, st))) return e;
  // dW2 += dZ2^T H1aug
  GemmArgs w2 = w3;
  w2.A = net.dz1t; w2.M = HID; w2.B = net.h1t; w2.C = net.G + G_W2;
  if ((e = launch_gemm(EPI_ATOMIC, w2, (B + w2.kslice - 1) / w2.kslice, st))) return e;
  // dZ1^T = ((dZ2 W2) * silu'(Z1))^T
  GemmArgs d1{};
  d1.err = net.err;
  d1.A = net.dz2; d1.lda = HID; d1.B = net.ops + O_W2T; d1.ldb = HID; d1.M = B; d1.N = HID; d1.K = HID;
  d1.kslice = HID;
  d1.Z = net.z1; d1.ldz = HID; d1.D = nullptr; d1.Dt = net.dz1t; d1.lddt = ldt;
  if ((e = launch_gemm(EPI_DACT, d1, 1, st))) return e;
  // dW1 += dZ1^T X : [128 x B] x [16 x B]^T
  GemmArgs w1 = w3;
  w1.A = net.dz1t; w1.M = HID; w1.B = net.xt; w1.N = 16; w1.C = net.G + G_W1; w1.ldc = KIN;
  return launch_gemm(EPI_ATOMIC, w1, (B + w1.kslice - 1) / w1.kslice, st);
}

int check_ready(char* errmsg, int32_t errmsg_len) {
  if (!net.ready) {
    smsg(errmsg, errmsg_len, "rrtmg_lw_gpu surrogate: no network (call rrtmg_lw_gpu_surrogate_init or _set)");
    return 1;
  }
  return 0;
}

}  // namespace

// MLP stage of the surrogate column path: writes tau/frac of every layer of
// the chunk into the scratch (the gas-optics kernel then redoes the layers
// outside the envelope).  Enqueue only.
cudaError_t mlp_lw_launch(const Block* blocks, int nblocks, const Block& b0, int nc, const Flags& f,
                          const Scratch<float>& sc, int num_sms, cudaStream_t st) {
  if (!net.ready || !net.attrs) return cudaErrorNotReady;
  FwdArgs a = base_args();
  a.nrows = (long)nc * f.nlay;
  a.blocks = blocks;
  a.nblocks = nblocks;
  a.b0 = b0;
  a.f = f;
  a.sc = sc;
  a.nc = nc;
  const long tiles = (a.nrows + 127) / 128;
  const int grid = (int)std::min<long>(tiles, num_sms);
  if (grid < 1) return cudaSuccess;
  mlp_fwd_kernel<MODE_LW><<<grid, FWD_THREADS, FWD_SMEM, st>>>(a);
  return cudaGetLastError();
}

// MLP stage of the learned-gas-optics path (lw_sg_path.cu): the compact FP16
// hand-off of chunk columns [c0, c0 + nc) and the list of columns with a
// layer outside the envelope.  Enqueue only.
cudaError_t mlp_h_launch(const Block* blocks, int nblocks, const Block& b0, const int* colmap, int c0, int nc,
                         const Flags& f, __half* hnd, unsigned int* fb_flag, int* fb_list, int* fb_count,
                         unsigned char* pack, int num_sms, cudaStream_t st) {
  if (!net.ready || !net.attrs) return cudaErrorNotReady;
  FwdArgs a = base_args();
  a.blocks = blocks;
  a.nblocks = nblocks;
  a.b0 = b0;
  a.f = f;
  a.nc = nc;
  a.hnd = hnd;
  a.colmap = colmap;
  a.c0 = c0;
  a.fb_flag = fb_flag;
  a.fb_list = fb_list;
  a.fb_count = fb_count;
  a.pk = pack;
  if (f.nlay > 127) return cudaErrorInvalidValue;   // one column per 128-row tile
  const int grid = std::min((nc + HP - 1) / HP, num_sms);
  if (grid < 1) return cudaSuccess;
  // two resident pack CTAs per SM (their registers: the 40 input loads of a layer are in flight at once)
  const int pgrid = std::min((nc + PK_COLS - 1) / PK_COLS, 2 * num_sms);
  mlp_h_pack_kernel<<<pgrid, PK_THREADS, PK_SMEM, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  mlp_h_kernel<<<grid, FWD_THREADS, H_SMEM, st>>>(a);
  return cudaGetLastError();
}

const float* surrogate_norm() { return net.ready ? net.norm : nullptr; }
SgNetView sg_net_view() { return SgNetView{net.ops, net.P, net.norm, net.err, net.fallback, net.ready ? 1 : 0}; }
unsigned int* surrogate_fallback_counter() { return net.fallback; }

}  // namespace lw

using namespace lw;

namespace {
int dev_of_init(int* dev, int* sms) {
  if (cudaGetDevice(dev) != cudaSuccess) return 1;
  if (cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, *dev) != cudaSuccess) return 1;
  return 0;
}
}  // namespace

extern "C" int rrtmg_lw_gpu_surrogate_features(const rrtmg_lw_run_args* a, float* feats, float* coldry, void* stream,
                                               char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  if (!a || !feats || a->npts < 0 || a->nlay < 1 || !a->plyr || !a->tlyr || !a->qlyr || !a->olyr || !a->delpin ||
      !a->gasvmr_co2 || !a->gasvmr_ch4 || !a->gasvmr_n2o) {
    smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_features: bad arguments");
    return 1;
  }
  if (a->npts == 0) return 0;
  Block B{};
  const double* in[N_IN] = {a->plyr, a->plvl, a->tlyr, a->tlvl, a->qlyr, a->olyr, a->gasvmr_co2, a->gasvmr_n2o,
                            a->gasvmr_ch4, a->gasvmr_o2, a->gasvmr_co, a->gasvmr_cfc11, a->gasvmr_cfc12,
                            a->gasvmr_cfc22, a->gasvmr_ccl4, a->aeraod, a->aerssa, a->sfemis, a->sfgtmp,
                            a->dzlyr, a->delpin, a->de_lgth, a->alpha, a->cld_cf, a->cld_lwp, a->cld_ref_liq,
                            a->cld_iwp, a->cld_ref_ice, a->cld_rwp, a->cld_ref_rain, a->cld_swp,
                            a->cld_ref_snow, a->cld_od};
  std::memcpy(B.in, in, sizeof(in));
  B.npts = a->npts;
  B.ld = a->ldim > 0 ? a->ldim : a->npts;
  cudaStream_t st = (cudaStream_t)stream;
  features_kernel<<<1024, 256, 0, st>>>(B, a->nlay, a->top_at_1, feats, coldry);
  SG_CK(cudaGetLastError(), "features kernel launch");
  SG_CK(cudaStreamSynchronize(st), "features kernel");
  return 0;
}

extern "C" int rrtmg_lw_gpu_surrogate_init(const float* norm, uint64_t seed, char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  if (!norm) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_init: NULL normalisation"); return 1; }
  std::lock_guard<std::mutex> lk(net_mu);
  int dev = 0, sms = 0;
  if (dev_of_init(&dev, &sms)) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_init: no CUDA device"); return 1; }
  SG_CK(set_attrs(), "kernel attributes (one CTA per SM)");
  SG_CK(ensure_net(dev, sms), "cudaMalloc(network)");
  // He-style uniform initialisation of the weights, zero biases
  std::vector<float> P(P_N * 3, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int rows, int cols, int fan_in) {
    const float lim = std::sqrt(6.0f / (float)fan_in);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) P[off + r * cols + c] = U(rng);
  };
  fill(P_W1, HID, NIN, NIN);
  for (int r = 0; r < HID; ++r) P[P_W1 + r * NIN + 7] = 0.0f;   // bias column
  fill(P_W2, HID, HID, HID);
  fill(P_W3, NOP, HID, HID);
  for (int r = 0; r < NOP; ++r)
    if (pad_out_row(r))
      for (int c = 0; c < HID; ++c) P[P_W3 + r * HID + c] = 0.0f;
  SG_CK(cudaMemcpy(net.P, P.data(), sizeof(float) * P.size(), cudaMemcpyHostToDevice), "cudaMemcpy(weights)");
  SG_CK(cudaMemcpy(net.norm, norm, sizeof(float) * SG_NORM_FLOATS, cudaMemcpyHostToDevice), "cudaMemcpy(norm)");
  SG_CK(cudaMemset(net.G, 0, sizeof(float) * G_N), "cudaMemset");
  pack_kernel<<<64, 256>>>(net.P, net.ops);
  SG_CK(cudaGetLastError(), "pack kernel");
  SG_CK(cudaDeviceSynchronize(), "pack kernel");
  SG_CK(cudaMemset(net.Madam, 0, sizeof(float) * P_N * 2), "cudaMemset(adam moments)");   // a fresh optimizer
  net.adam_t = 0;
  net.ready = true;
  return 0;
}

// weights in natural shapes: W1 [128][8] (column 7 = bias of layer 1), W2 [128][128], b2 [128],
// W3 [280][128], b3 [280]; norm float[SG_NORM_FLOATS]
extern "C" int rrtmg_lw_gpu_surrogate_set(const float* w, const float* norm, char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  if (!w || !norm) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_set: NULL argument"); return 1; }
  std::lock_guard<std::mutex> lk(net_mu);
  int dev = 0, sms = 0;
  if (dev_of_init(&dev, &sms)) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_set: no CUDA device"); return 1; }
  SG_CK(set_attrs(), "kernel attributes (one CTA per SM)");
  SG_CK(ensure_net(dev, sms), "cudaMalloc(network)");
  std::vector<float> P(P_N * 3, 0.0f);
  size_t k = 0;
  for (int j = 0; j < HID * NIN + HID * HID + HID; ++j) P[j] = w[k++];
  for (int r = 0; r < NOP; ++r) {
    if (pad_out_row(r)) continue;
    for (int c = 0; c < HID; ++c) P[P_W3 + r * HID + c] = w[k++];
  }
  for (int r = 0; r < NOP; ++r) {
    if (pad_out_row(r)) continue;
    P[P_B3 + r] = w[k++];
  }
  SG_CK(cudaMemcpy(net.P, P.data(), sizeof(float) * P.size(), cudaMemcpyHostToDevice), "cudaMemcpy(weights)");
  SG_CK(cudaMemcpy(net.norm, norm, sizeof(float) * SG_NORM_FLOATS, cudaMemcpyHostToDevice), "cudaMemcpy(norm)");
  pack_kernel<<<64, 256>>>(net.P, net.ops);
  SG_CK(cudaGetLastError(), "pack kernel");
  SG_CK(cudaDeviceSynchronize(), "pack kernel");
  SG_CK(cudaMemset(net.Madam, 0, sizeof(float) * P_N * 2), "cudaMemset(adam moments)");   // a fresh optimizer
  net.adam_t = 0;
  net.ready = true;
  return 0;
}

extern "C" int rrtmg_lw_gpu_surrogate_get(float* w, float* norm, char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  std::lock_guard<std::mutex> lk(net_mu);
  if (check_ready(errmsg, errmsg_len)) return 1;
  std::vector<float> P(P_N);
  SG_CK(cudaMemcpy(P.data(), net.P, sizeof(float) * P_N, cudaMemcpyDeviceToHost), "cudaMemcpy(weights)");
  if (w) {
    size_t k = 0;
    for (int j = 0; j < HID * NIN + HID * HID + HID; ++j) w[k++] = P[j];
    for (int r = 0; r < NOP; ++r)
      if (!pad_out_row(r))
        for (int c = 0; c < HID; ++c) w[k++] = P[P_W3 + r * HID + c];
    for (int r = 0; r < NOP; ++r)
      if (!pad_out_row(r)) w[k++] = P[P_B3 + r];
  }
  if (norm) SG_CK(cudaMemcpy(norm, net.norm, sizeof(float) * SG_NORM_FLOATS, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return 0;
}

static_assert(RRTMG_LW_SURROGATE_NSTATE == P_N, "training-state size in the C ABI");

// Training state for a checkpoint: the FP32 master parameters and Adam's
// first and second moment estimates, each float[P_N] in the padded layout,
// the step count and the normalisation.
extern "C" int rrtmg_lw_gpu_surrogate_get_state(float* params, float* m, float* v, int64_t* step, float* norm,
                                                char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  std::lock_guard<std::mutex> lk(net_mu);
  if (check_ready(errmsg, errmsg_len)) return 1;
  if (params) SG_CK(cudaMemcpy(params, net.P, sizeof(float) * P_N, cudaMemcpyDeviceToHost), "cudaMemcpy(params)");
  if (m) SG_CK(cudaMemcpy(m, net.Madam, sizeof(float) * P_N, cudaMemcpyDeviceToHost), "cudaMemcpy(adam m)");
  if (v) SG_CK(cudaMemcpy(v, net.Vadam, sizeof(float) * P_N, cudaMemcpyDeviceToHost), "cudaMemcpy(adam v)");
  if (step) *step = net.adam_t;
  if (norm) SG_CK(cudaMemcpy(norm, net.norm, sizeof(float) * SG_NORM_FLOATS, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return 0;
}

extern "C" int rrtmg_lw_gpu_surrogate_set_state(const float* params, const float* m, const float* v, int64_t step,
                                                const float* norm, char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  if (!params || !m || !v || !norm || step < 0) {
    smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_set_state: NULL argument or negative step");
    return 1;
  }
  std::lock_guard<std::mutex> lk(net_mu);
  int dev = 0, sms = 0;
  if (dev_of_init(&dev, &sms)) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_set_state: no CUDA device"); return 1; }
  SG_CK(set_attrs(), "kernel attributes (one CTA per SM)");
  SG_CK(ensure_net(dev, sms), "cudaMalloc(network)");
  SG_CK(cudaMemcpy(net.P, params, sizeof(float) * P_N, cudaMemcpyHostToDevice), "cudaMemcpy(params)");
  SG_CK(cudaMemcpy(net.Madam, m, sizeof(float) * P_N, cudaMemcpyHostToDevice), "cudaMemcpy(adam m)");
  SG_CK(cudaMemcpy(net.Vadam, v, sizeof(float) * P_N, cudaMemcpyHostToDevice), "cudaMemcpy(adam v)");
  SG_CK(cudaMemcpy(net.norm, norm, sizeof(float) * SG_NORM_FLOATS, cudaMemcpyHostToDevice), "cudaMemcpy(norm)");
  pack_kernel<<<64, 256>>>(net.P, net.ops);
  SG_CK(cudaGetLastError(), "pack kernel");
  SG_CK(cudaDeviceSynchronize(), "pack kernel");
  net.adam_t = (long)step;
  net.ready = true;
  return 0;
}

extern "C" int rrtmg_lw_gpu_surrogate_forward(const float* feats, int64_t n, float* y, void* stream, char* errmsg,
                                              int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  std::lock_guard<std::mutex> lk(net_mu);
  if (check_ready(errmsg, errmsg_len)) return 1;
  if (n < 0 || (n > 0 && (!feats || !y))) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_forward: bad arguments"); return 1; }
  if (n == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  FwdArgs a = base_args();
  a.nrows = n;
  a.feats = feats;
  a.y = y;
  const long tiles = (n + 127) / 128;
  SG_CK(cudaMemsetAsync(net.err, 0, sizeof(int), st), "cudaMemsetAsync");
  mlp_fwd_kernel<MODE_FEATS><<<(int)std::min<long>(tiles, net.num_sms), FWD_THREADS, FWD_SMEM, st>>>(a);
  SG_CK(cudaGetLastError(), "forward kernel launch");
  int herr = 0;
  SG_CK(cudaMemcpyAsync(&herr, net.err, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  SG_CK(cudaStreamSynchronize(st), "forward kernel");
  if (herr) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_forward: tensor-core wait timed out"); return 1; }
  return 0;
}

// One forward + backward pass over the first `batch` samples (no update):
// loss and the gradients in parameter order (float[54688], see the layout
// comments) for gradient checks.
extern "C" int rrtmg_lw_gpu_surrogate_grads(const float* feats, const float* targets, int32_t batch, float* grads,
                                            float* loss, void* stream, char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  std::lock_guard<std::mutex> lk(net_mu);
  if (check_ready(errmsg, errmsg_len)) return 1;
  if (batch < 128 || batch % 128 || !feats || !targets) {
    smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_grads: batch must be a positive multiple of 128");
    return 1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  SG_CK(ensure_batch(batch), "cudaMalloc(activations)");
  SG_CK(cudaMemsetAsync(net.G, 0, sizeof(float) * G_N, st), "cudaMemsetAsync");
  SG_CK(cudaMemsetAsync(net.err, 0, sizeof(int) + sizeof(float), st), "cudaMemsetAsync");
  SG_CK(train_batch(feats, targets, batch, batch, 1, 0, 0, 0, st), "training kernels launch");
  float* dgr = nullptr;
  SG_CK(cudaMallocAsync((void**)&dgr, sizeof(float) * P_N, st), "cudaMallocAsync");
  grads_kernel<<<64, 256, 0, st>>>(net.G, dgr);
  int herr[2] = {0, 0};
  SG_CK(cudaMemcpyAsync(herr, net.err, sizeof(int) + sizeof(float), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  if (grads) SG_CK(cudaMemcpyAsync(grads, dgr, sizeof(float) * P_N, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  SG_CK(cudaFreeAsync(dgr, st), "cudaFreeAsync");
  SG_CK(cudaStreamSynchronize(st), "training kernels");
  SG_CK(cudaMemsetAsync(net.G, 0, sizeof(float) * G_N, st), "cudaMemsetAsync");
  if (herr[0]) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_grads: tensor-core wait timed out"); return 1; }
  if (loss) { float l; std::memcpy(&l, &herr[1], sizeof(float)); *loss = l / (float)((long)batch * SG_NOUT); }
  return 0;
}

// Adam training on device-resident data: feats [n][8], targets [n][288]
// (normalised, padded layout).  flags bit 0: weight each optical-depth error
// by 1 / (1 + 1.66 tau) of its target, with the layer's coldry in feats[., 7].  Each epoch visits floor(n / batch) batches
// of an affine permutation of the samples.  loss_per_epoch (optional,
// float[epochs]) receives the mean squared error of each epoch.
extern "C" int rrtmg_lw_gpu_surrogate_train(const float* feats, const float* targets, int64_t n, int32_t epochs,
                                            int32_t batch, float lr, float lr_final, uint64_t seed, int32_t flags,
                                            float* loss_per_epoch, void* stream, char* errmsg, int32_t errmsg_len) {
  smsg(errmsg, errmsg_len, "");
  std::lock_guard<std::mutex> lk(net_mu);
  if (check_ready(errmsg, errmsg_len)) return 1;
  if (batch < 128 || batch % 128 || n < batch || epochs < 1 || !feats || !targets) {
    smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_train: need batch a multiple of 128, n >= batch, epochs >= 1");
    return 1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  SG_CK(ensure_batch(batch), "cudaMalloc(activations)");
  SG_CK(cudaMemsetAsync(net.err, 0, sizeof(int), st), "cudaMemsetAsync");
  std::mt19937_64 rng(seed);
  const long steps = n / batch;
  const long total = steps * (long)epochs;
  long done = 0;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    SG_CK(cudaMemsetAsync(net.loss, 0, sizeof(float), st), "cudaMemsetAsync");
    long pa;
    do { pa = (long)(rng() % (uint64_t)n); } while (pa == 0 || std::gcd(pa, (long)n) != 1);
    const long pb = (long)(rng() % (uint64_t)n);
    for (long s = 0; s < steps; ++s, ++done) {
      SG_CK(train_batch(feats, targets, n, batch, pa, pb, s * batch, flags & 1, st), "training kernels launch");
      ++net.adam_t;
      // cosine decay from lr to lr_final over the whole run
      const double fr = (double)done / (double)std::max(1L, total - 1);
      const float lr_t = (float)(lr_final + 0.5 * (lr - lr_final) * (1.0 + std::cos(3.14159265358979323846 * fr)));
      const float c1 = 1.0f - std::pow(b1, (float)net.adam_t), c2 = 1.0f - std::pow(b2, (float)net.adam_t);
      adam_kernel<<<64, 256, 0, st>>>(net.P, net.Madam, net.Vadam, net.G, net.ops, lr_t, b1, b2, c1, c2, eps);
      SG_CK(cudaGetLastError(), "adam kernel launch");
      SG_CK(cudaMemsetAsync(net.G, 0, sizeof(float) * G_N, st), "cudaMemsetAsync");
    }
    float l = 0.0f;
    int herr = 0;
    SG_CK(cudaMemcpyAsync(&l, net.loss, sizeof(float), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    SG_CK(cudaMemcpyAsync(&herr, net.err, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    SG_CK(cudaStreamSynchronize(st), "training kernels");
    if (herr) { smsg(errmsg, errmsg_len, "rrtmg_lw_gpu_surrogate_train: tensor-core wait timed out"); return 1; }
    if (loss_per_epoch) loss_per_epoch[ep] = l / (float)(steps * batch * (long)SG_NOUT);
  }
  return 0;
}

// Layers of surrogate runs that fell outside the training envelope and were
// recomputed with taumol, since the last reset; and the tensor-core error
// flag of the last surrogate launches.
extern "C" int rrtmg_lw_gpu_surrogate_wait_limit(int64_t polls) {
  std::lock_guard<std::mutex> lk(net_mu);
  const uint32_t v = polls < 0 ? kFwdWaitPollsDefault : (uint32_t)std::min<int64_t>(polls, 0xffffffffll);
  return cudaMemcpyToSymbol(c_fwd_wait_polls, &v, sizeof(v)) == cudaSuccess ? 0 : 1;
}

extern "C" int rrtmg_lw_gpu_surrogate_stats(uint64_t* fallback_layers, int32_t* mma_error, int32_t reset) {
  std::lock_guard<std::mutex> lk(net_mu);
  if (!net.err) return 1;
  int h[4] = {0, 0, 0, 0};
  if (cudaMemcpy(h, net.err, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  if (fallback_layers) *fallback_layers = (uint64_t)(unsigned int)h[2];
  if (mma_error) *mma_error = h[0];
  if (reset && cudaMemset(net.err, 0, sizeof(h)) != cudaSuccess) return 1;
  return 0;
}
