// lw_fused.cu -- the learned-gas-optics column path in one persistent kernel.
//
// Replaces, for RRTMG_LW_SURROGATE calls, the network stage + gas-optics
// kernel + transfer kernel chain (lw_mlp.cu, lw_gas.cuh, lw_rt.cuh) and its
// per-column hand-off through device memory.  Per column (one 128-row tile:
// layer t = row t, surface first) one CTA, alone on its SM, runs:
//
//   prologue   layer warps (thread <-> layer): the driver prologue of
//              rrtmg_lw_run (RLM:785-1050), the network's features, Planck
//              integrals (setcoef, RLM:2251-2283), band cloud optics
//              (cldprop, RLM:1589-1799) and aerosol optical depth; the
//              column's diffusivity angles (RLM:1041-1050).  It runs for
//              column i+1 while the transfer warps work on column i.
//   network    tcgen05 BF16 MMAs with FP32 accumulators in tensor memory:
//              H1 = SiLU(X W1), H2 = SiLU(H1 W2 + b2), then the output layer
//              twice: transposed for the 128 optical depths of g-points
//              0..127 (D = W3 H2^T, so TMEM lane = g-point and column =
//              layer: the transfer reads a g-point's whole column from its
//              own lane) and in the ordinary orientation for the 140 Planck
//              fractions and the optical depths of g-points 128..139, which
//              the epilogue normalises per band (RLM:3836-4013 taumol
//              outputs) into shared memory.
//   transfer   rtrnmc (RLM:3420-3785) with one lane per g-point: the down
//              sweep, surface emission/reflection and up sweep run in the
//              Fortran's order for each g-point; the layer terms the up sweep
//              needs (transmittance and sources) are kept in tensor memory.
//              Sums over g-points: a warp transpose-reduction per 16 levels,
//              then FP64 across warps; heating rates from the FP64 flux
//              divergence.
//
// Layers outside the network's training envelope fall back to plain FP32
// taumol: a column with any such layer runs the gas-optics kernel's column
// routine (gas_column, learned-gas-optics variant) into a per-CTA work area,
// and the epilogue and transfer take those layers' optical depths and Planck
// fractions from there.
#include <algorithm>
#include <cstdio>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lw_launch.h"
#include "lw_net.h"
#include "lw_rt.cuh"
#include "lw_umma.cuh"

namespace lw {
namespace {

constexpr int FZ_THREADS = 256;   // 8 warps: 0..3 layers (prologue, g 128..139), 4..7 g 0..127
constexpr int FZ_NL = 128;        // tile rows: padded layers (nlay <= 127)
constexpr int FZ_NT = NGPT - 128; // g-points 128..139, transferred by the layer warps
constexpr int FZ_NP = 8;          // flux partial sums: one per warp

// shared memory layout (bytes)
constexpr uint32_t SM_W1 = 0;                                   // canon [128][16]
constexpr uint32_t SM_W2 = SM_W1 + HID * KIN * 2;               // canon [128][128]
constexpr uint32_t SM_W3A = SM_W2 + HID * HID * 2;              // canon [128][128]: tau rows of g 0..127
constexpr uint32_t NF_ROWS = 160;                               // frac g 0..139, tau g 128..139, 8 zero rows
constexpr uint32_t SM_W3F = SM_W3A + 128 * HID * 2;             // canon [160][128]
constexpr uint32_t SM_X = SM_W3F + NF_ROWS * HID * 2;           // canon [128][16]
constexpr uint32_t SM_HF = SM_X + 128 * KIN * 2;                // canon [128][128] H | fp16 [128][140] fracs
constexpr uint32_t HF_BYTES = 128 * NGPT * 2;
constexpr uint32_t SM_TAIL = SM_HF + HF_BYTES;                  // f32 [128][12] raw outputs, tau of g 128..139
constexpr uint32_t SM_PKL = SM_TAIL + FZ_NL * FZ_NT * 4;        // f32 [128][16] pklay(b, t+1)
constexpr uint32_t SM_PKV = SM_PKL + FZ_NL * NBANDS * 4;        // f32 [129][16] pklev(b, l)
constexpr uint32_t SM_TCL = SM_PKV + (FZ_NL + 1) * NBANDS * 4;  // f32 [128][16] taucld
constexpr uint32_t SM_AER = SM_TCL + FZ_NL * NBANDS * 4;        // f32 [128][16] aerosol optical depth
constexpr uint32_t SM_CD = SM_AER + FZ_NL * NBANDS * 4;         // f32 [128] coldry
constexpr uint32_t NPART = 4 * (FZ_NL + 1);
constexpr uint32_t SM_PART = SM_CD + FZ_NL * 4;                 // f32 [8][4][129] per-warp flux sums
constexpr uint32_t SM_FN = SM_PART + FZ_NP * NPART * 4;         // f64 [2][129] net flux (total, clear)
constexpr uint32_t SM_RED = SM_FN + 2 * (FZ_NL + 1) * 8;        // f64 [2][128] coldry, colh2o
constexpr uint32_t SM_NRM = SM_RED + 2 * FZ_NL * 8;             // f32 [4][140] + [16]
constexpr int NRM_OSC_T = 0, NRM_OSH_T = 140, NRM_OSC_F = 280, NRM_OSH_F = 420, NRM_IN = 560, NRM_N = 576;
constexpr uint32_t SM_COL = SM_NRM + NRM_N * 4;                 // f32 [2][64] column scalars (double buffer)
constexpr int COL_SECD = 0, COL_PK0 = 16, COL_PKV0 = 32, COL_SEMIS = 48, COL_LCF1 = 49, COL_NFB = 50,
              COL_FB = 52, COL_SCR = 56, COL_N = 64;
constexpr uint32_t SM_BAR = SM_COL + 2 * COL_N * 4;             // mbarrier, TMEM slot, failure flag
constexpr uint32_t FZ_SMEM = SM_BAR + 64;
static_assert(FZ_SMEM <= 227 * 1024, "fused kernel shared memory");
static_assert(FZ_SMEM > 114 * 1024, "the fused kernel must hold its SM alone (512 TMEM columns)");
static_assert(SM_HF % 128 == 0 && SM_X % 128 == 0 && SM_W3F % 128 == 0, "canonical tiles");

// TMEM columns.  Network phase: D1/D2 [0,128), fractions [128,288), optical
// depths (transposed) [288,416).  Transfer phase: transmittance [0,128),
// clear-sky and total-sky up sources [128,256) and [256,288)+[416,512).
constexpr uint32_t TM_D12 = 0, TM_DF = 128, TM_TAU = 288, TM_TR = 0, TM_GSU = 128;
constexpr int CH = 16;   // layers per transfer chunk (one TMEM load/store of 16 columns)
__device__ __forceinline__ uint32_t tm_tsu(int j) { return j < 2 ? 256u + CH * j : 416u + CH * (j - 2); }

// Per-CTA device work area for columns with layers outside the envelope:
// gas_column's working arrays, then two column slots (tau, frac, band fields,
// column record) in the scratch layout of the gas-optics kernel (V = 4).
constexpr size_t FZ_NLP = 128;
constexpr size_t FZ_SLOT_BYTES = (2 * NGPT + 3 * NBANDS) * FZ_NLP * 4 + kColRec * 8;
__host__ __device__ constexpr size_t fz_gas_bytes() { return (gas_smem_bytes<float>(4) + 255) & ~size_t(255); }
__host__ __device__ constexpr size_t fz_cta_bytes() { return fz_gas_bytes() + 2 * ((FZ_SLOT_BYTES + 255) & ~size_t(255)); }

struct FusedArgs {
  const Block* blocks;
  int nblocks;
  Block b0;
  int ncols;              // columns of the call: global columns [0, ncols)
  Flags f;
  Consts cs;
  Tables<float> tab;      // FP32 coefficient tables and transfer records
  Tables<double> tab64;   // FP64 tables (setcoef, Planck, cloud optics)
  const uint32_t* bits;   // McICA sub-column flags [col][140][nw]
  SgNetView net;
  unsigned char* work;    // fz_cta_bytes() per CTA
};

constexpr uint32_t kFzWaitPolls = 1u << 22;

__device__ __forceinline__ int fz_band(int g) {
  return g < 10 ? 0 : g < 22 ? 1 : g < 38 ? 2 : g < 52 ? 3 : g < 68 ? 4 : g < 76 ? 5 : g < 88 ? 6 : g < 96 ? 7
       : g < 108 ? 8 : g < 114 ? 9 : g < 122 ? 10 : g < 130 ? 11 : g < 134 ? 12 : g < 136 ? 13 : g < 138 ? 14 : 15;
}

// Sum over the warp's lanes of a[i], i = 0..15: every lane returns the sum
// for index (lane >> 1) & 15 (recursive halving, 16 shuffles).
__device__ __forceinline__ float warp_sum16(const float (&a)[16], int lane) {
  float b[8], c[4], d[2];
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4, h2 = lane & 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float keep = h16 ? a[8 + j] : a[j], send = h16 ? a[j] : a[8 + j];
    b[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float keep = h8 ? b[4 + j] : b[j], send = h8 ? b[j] : b[4 + j];
    c[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float keep = h4 ? c[2 + j] : c[j], send = h4 ? c[j] : c[2 + j];
    d[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  float e = (h2 ? d[1] : d[0]) + __shfl_xor_sync(0xffffffffu, h2 ? d[0] : d[1], 2);
  return e + __shfl_xor_sync(0xffffffffu, e, 1);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The rlwinit lookup (RLM:1474-1501, 3598-3660) in FP32: for optical depth
// x above 0.06 (LE: x > 0.06 for the gas terms, RLM:3600; x >= 0.06 for the
// total-sky terms, RLM:3639) the index it = int(10000 x / (bpade + x) + 0.5)
// selects the record {exp_tbl, tfn_tbl, tau_tbl}; small depths take the
// Pade-free forms.  Returns the transmittance tr, atr = 1 - tr (each as the
// reference forms it), the Planck weight fac, and in tq the depth the record
// stands for (the reference replaces odepth by tau_tbl, RLM:3614).
template <bool LE>
__device__ __forceinline__ void fz_tbl(const float* trec, float x, float& tr, float& atr, float& fac, float& tq) {
  const float q = __fdividef(x, float(kBpade) + x);
  const int it = min(NTBL, max(0, (int)(float(kTblint) * q + 0.5f)));
  const float4 rec = __ldg(reinterpret_cast<const float4*>(trec + 4 * it));
  const bool small = LE ? x <= 0.06f : x < 0.06f;
  atr = small ? x - 0.5f * x * x : 1.0f - rec.x;
  tr = small ? 1.0f - atr : rec.x;
  fac = small ? float(kRec6) * x : rec.y;
  tq = small ? x : rec.z;
}

// cldprop band optics of one layer (RLM:1589-1799), FP64: the layer's band-
// independent terms once (set), then one band's table interpolation (band);
// the same arithmetic as band_taucld, hoisted out of the band loop.
struct CloudLayer {
  double cf, clwp, ciwp, cda1, tauran, tausnw, fliq, fice, refice;
  int iliq, iice;
  __device__ __forceinline__ void set(const Flags& f, double cf_, double clwp_, double relw, double ciwp_,
                                      double reiw, double cda1_, double cda3, double cda4) {
    cf = cf_; clwp = clwp_; ciwp = ciwp_; cda1 = cda1_;
    tauran = kAbsrain * cda1;
    tausnw = (cda3 > 0.0 && cda4 > 10.0) ? kAbssnow0 * 1.05756 * cda3 / cda4 : 0.0;
    const double lfac = relw - 1.5;
    iliq = max(1, min(57, (int)lfac));
    fliq = lfac - (double)iliq;
    refice = fmin(130.0, fmax(13.0, reiw));
    double ifac = 0.0;
    int ihi = 45;
    if (f.ilwcice == 2) { ifac = (reiw - 2.0) / 3.0; ihi = 42; }
    else if (f.ilwcice == 3) { const double dgeice = fmax(5.0, 1.0315 * reiw); ifac = (dgeice - 2.0) / 3.0; }
    iice = max(1, min(ihi, (int)ifac));
    fice = ifac - (double)iice;
  }
  __device__ __forceinline__ double band(int b, const Flags& f, const double* kt) const {
    if (!(cf > 2.2250738585072014e-308)) return 0.0;   // cfrac(k) > cldmin = tiny
    if (f.ilwcliq <= 0) return cda1;                    // diagnostic cloud optical depth
    double tauliq = 0.0, tauice = 0.0;
    if (clwp > 0.0 && f.ilwcliq == 1) {
      const double a = t64(kt, lwtab::absliq1 + (iliq - 1) + 58 * b);
      const double c = t64(kt, lwtab::absliq1 + iliq + 58 * b);
      tauliq = fmax(0.0, clwp * (a + fliq * (c - a)));
    }
    if (ciwp > 0.0) {
      if (f.ilwcice == 1) {
        const int ia = (int)t64(kt, lwtab::ipat + b);
        tauice = fmax(0.0, ciwp * (t64(kt, lwtab::absice1 + 2 * (ia - 1)) + t64(kt, lwtab::absice1 + 1 + 2 * (ia - 1)) / refice));
      } else if (f.ilwcice == 2) {
        const double a = t64(kt, lwtab::absice2 + (iice - 1) + 43 * b);
        const double c = t64(kt, lwtab::absice2 + iice + 43 * b);
        tauice = fmax(0.0, ciwp * (a + fice * (c - a)));
      } else if (f.ilwcice == 3) {
        const double a = t64(kt, lwtab::absice3 + (iice - 1) + 46 * b);
        const double c = t64(kt, lwtab::absice3 + iice + 46 * b);
        tauice = fmax(0.0, ciwp * (a + fice * (c - a)));
      }
    }
    return tauice + tauliq + tauran + tausnw;
  }
};

// band fields of one layer, produced by the prologue and held in registers
// until the transfer of the previous column has finished with shared memory
struct LayerFields {
  float pkl[NBANDS], pkv[NBANDS], tcl[NBANDS], aer[NBANDS];
  float cd;
};

template <int GA, int GB>
__device__ __forceinline__ void frac_epilogue(uint32_t tb, int wq, int t, bool live, bool fb, const float* nrm,
                                              const float* cd, const float* aer, __half* frs, float* tail,
                                              const float* slot_tau, const float* slot_frac) {
  constexpr int C0 = GA & ~15;
  constexpr int CE = (GB <= 140 ? GB : 140);     // fraction columns
  constexpr int NCH = ((GB > 140 ? 152 : GB) - C0 + 15) / 16;
  float v[NCH * 16];
#pragma unroll
  for (int c = 0; c < NCH; ++c) umma::tmem_ld16(umma::tmem_addr(tb, wq, TM_DF + C0 + 16 * c), v + 16 * c);
  if (!live) {
    // padding rows above the top layer: zero fractions and optical depths make
    // them neutral in the transfer (transmittance 1, no source)
#pragma unroll 1
    for (int g = GA; g < CE; ++g) frs[t * NGPT + g] = __float2half_rn(0.0f);
    if (GB > 140) {
#pragma unroll 1
      for (int g = 128; g < NGPT; ++g) tail[t * FZ_NT + (g - 128)] = 0.0f;
    }
    return;
  }
  if (!fb) {
    float bsum[NBANDS];
#pragma unroll
    for (int b = 0; b < NBANDS; ++b) bsum[b] = 0.0f;
#pragma unroll
    for (int g = GA; g < CE; ++g) {
      const float fr = __saturatef(fmaf(v[g - C0], nrm[NRM_OSC_F + g], nrm[NRM_OSH_F + g]));
      v[g - C0] = fr;
      bsum[fz_band(g)] += fr;
    }
#pragma unroll
    for (int b = 0; b < NBANDS; ++b) bsum[b] = bsum[b] > 0.0f ? 1.0f / bsum[b] : 1.0f;
#pragma unroll
    for (int g = GA; g < CE; ++g) frs[t * NGPT + g] = __float2half_rn(v[g - C0] * bsum[fz_band(g)]);
    if (GB > 140) {
      // raw outputs of g 128..139: the tail transfer warp evaluates them like TMEM lanes
#pragma unroll
      for (int g = 128; g < NGPT; ++g) tail[t * FZ_NT + (g - 128)] = v[140 + (g - 128) - C0];
    }
  } else {
    // out-of-envelope layer: plain taumol fractions of the work slot ([g][128]);
    // the transfer takes its optical depths from the slot too
#pragma unroll 1
    for (int g = GA; g < CE; ++g) frs[t * NGPT + g] = __float2half_rn(slot_frac[g * FZ_NLP + t]);
  }
}

// 8 warps, two per SM sub-partition, so up to 255 registers per thread (each
// sub-partition holds 16K); one CTA per SM (its shared memory and 512 TMEM
// columns require that anyway)
__global__ void __launch_bounds__(FZ_THREADS, 1) lw_sg_fused_kernel(FusedArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, wq = warp & 3;
  const Flags& f = a.f;
  const int nlay = f.nlay, nlp1 = nlay + 1;
  float* nrm = reinterpret_cast<float*>(sm + SM_NRM);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + SM_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SM_BAR + 8);
  int* sfail = reinterpret_cast<int*>(sm + SM_BAR + 12);
  __half* frs = reinterpret_cast<__half*>(sm + SM_HF);
  float* tail = reinterpret_cast<float*>(sm + SM_TAIL);
  float* pkl = reinterpret_cast<float*>(sm + SM_PKL);
  float* pkv = reinterpret_cast<float*>(sm + SM_PKV);
  float* tcl = reinterpret_cast<float*>(sm + SM_TCL);
  float* aer = reinterpret_cast<float*>(sm + SM_AER);
  float* cds = reinterpret_cast<float*>(sm + SM_CD);
  float* part = reinterpret_cast<float*>(sm + SM_PART);
  double* fn = reinterpret_cast<double*>(sm + SM_FN);
  double* red = reinterpret_cast<double*>(sm + SM_RED);
  float* colv0 = reinterpret_cast<float*>(sm + SM_COL);

  // ---- set-up: weights in canonical tiles, normalisation, TMEM, barrier ----
  {
    const bf16* ops = a.net.ops;
    for (int ch = tid; ch < HID * (KIN / 8); ch += FZ_THREADS) {
      const int r = ch / (KIN / 8), k = (ch % (KIN / 8)) * 8;
      *reinterpret_cast<uint4*>(sm + SM_W1 + umma::canon_off(r, k, KIN)) =
          __ldg(reinterpret_cast<const uint4*>(ops + O_W1 + r * KIN + k));
    }
    for (int ch = tid; ch < HID * (HID / 8); ch += FZ_THREADS) {
      const int r = ch / (HID / 8), k = (ch % (HID / 8)) * 8;
      *reinterpret_cast<uint4*>(sm + SM_W2 + umma::canon_off(r, k, HID)) =
          __ldg(reinterpret_cast<const uint4*>(ops + O_W2 + r * HID + k));
      *reinterpret_cast<uint4*>(sm + SM_W3A + umma::canon_off(r, k, HID)) =
          __ldg(reinterpret_cast<const uint4*>(ops + O_W3 + r * HID + k));   // tau rows 0..127
    }
    for (int ch = tid; ch < (int)NF_ROWS * (HID / 8); ch += FZ_THREADS) {
      const int r = ch / (HID / 8), k = (ch % (HID / 8)) * 8;
      uint4 w = make_uint4(0u, 0u, 0u, 0u);
      if (r < NGPT) w = __ldg(reinterpret_cast<const uint4*>(ops + O_W3 + (sg_frac_col(r)) * HID + k));
      else if (r < NGPT + FZ_NT) w = __ldg(reinterpret_cast<const uint4*>(ops + O_W3 + (128 + r - NGPT) * HID + k));
      *reinterpret_cast<uint4*>(sm + SM_W3F + umma::canon_off(r, k, HID)) = w;
    }
    const float* nm = a.net.norm;
    const float* pb3 = a.net.params + P_B3;
    for (int g = tid; g < NGPT; g += FZ_THREADS) {
      const float st = nm[SG_OUT_STD + sg_tau_col(g)], sf = nm[SG_OUT_STD + sg_frac_col(g)];
      nrm[NRM_OSC_T + g] = st;
      nrm[NRM_OSH_T + g] = fmaf(pb3[sg_tau_col(g)], st, nm[SG_OUT_MEAN + sg_tau_col(g)]);
      nrm[NRM_OSC_F + g] = sf;
      nrm[NRM_OSH_F + g] = fmaf(pb3[sg_frac_col(g)], sf, nm[SG_OUT_MEAN + sg_frac_col(g)]);
    }
    if (tid < 16) nrm[NRM_IN + tid] = nm[tid < 8 ? SG_IN_MEAN + tid : SG_IN_STD + tid - 8];
    if (warp == 0) {
      umma::tmem_alloc(tslot, 512);
      umma::tmem_relinquish();
    }
    if (tid == 0) {
      umma::mbar_init(mbar, 1);
      *sfail = 0;
    }
  }
  umma::fence_smem_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t sbase = umma::smem_u32(sm);
  constexpr uint32_t ID128 = umma::idesc_bf16(128, 128), IDF = umma::idesc_bf16(128, NF_ROWS);
  uint32_t phase = 0;
  bool failed = false;
  auto wait_mma = [&]() -> bool {
    const bool ok = umma::mbar_wait(mbar, phase, kFzWaitPolls);
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

  unsigned char* work = a.work + (size_t)blockIdx.x * fz_cta_bytes();
  const GasWork<float, 4> gw = GasWork<float, 4>::at(work);
  auto slot_base = [&](int s) -> float* {
    return reinterpret_cast<float*>(work + fz_gas_bytes() + (size_t)s * ((FZ_SLOT_BYTES + 255) & ~size_t(255)));
  };
  const bool is_layer = tid < FZ_NL;
  const int t = tid;   // layer of a layer thread
  LayerFields LF;

  // ---- prologue of column cc into column buffer `cb` and work slot `cb` (layer threads) ----
  auto prologue = [&](int cc, int cb) {
    const GroupSync S{1, FZ_NL};
    float* colv = colv0 + cb * COL_N;
    const int c = cc;
    const Block& B = (a.nblocks == 1) ? a.b0 : a.blocks[find_block(a.blocks, a.nblocks, c)];
    const int i = c - B.col0;
    const size_t ld = (size_t)B.ld;
    const bool top = f.top_at_1 != 0;
    const bool live = t < nlay;
    const int r = top ? nlp1 - (t + 1) - 1 : t;
    const int rl = top ? nlp1 - (t + 1) - 1 : t + 1;
    auto IN = [&](int fld, int row) -> double { return B.in[fld][i + ld * row]; };
    float x[KIN];
#pragma unroll
    for (int j = 0; j < KIN; ++j) x[j] = 0.0f;
    bool in_env = true, cldk = false;
    double tc7 = 0.0;   // band 7 cloud optical depth (cldtau output)
    double cf = 0.0, clwp = 0.0, relw = 0.0, ciwp = 0.0, reiw = 0.0, cda1 = 0.0, cda3 = 0.0, cda4 = 0.0;
    LF.cd = 0.0f;
#pragma unroll
    for (int b = 0; b < NBANDS; ++b) LF.pkl[b] = LF.pkv[b] = LF.tcl[b] = LF.aer[b] = 0.0f;
    if (live) {
      // every global load of the layer first, so their latencies overlap
      const double pavel = IN(F_PLYR, r), delp = IN(F_DELPIN, r), tavel = IN(F_TLYR, r), tz = IN(F_TLVL, rl);
      const double q = IN(F_QLYR, r), o3 = IN(F_OLYR, r);
      const double co2 = IN(F_CO2, r), ch4 = IN(F_CH4, r), n2o = IN(F_N2O, r);
      cf = IN(F_CLDCF, r);
      if (f.ilwcliq > 0) {
        clwp = IN(F_LWP, r); relw = IN(F_RELIQ, r); ciwp = IN(F_IWP, r); reiw = IN(F_REICE, r);
        cda1 = IN(F_RWP, r); cda3 = IN(F_SWP, r); cda4 = IN(F_RESNOW, r);
      } else {
        cda1 = IN(F_CLDOD, r);
      }
      double aod[NBANDS], ssa[NBANDS];
#pragma unroll
      for (int b = 0; b < NBANDS; ++b) {
        const size_t ab = i + ld * ((size_t)r + (size_t)nlay * b);
        aod[b] = B.in[F_AERAOD][ab];
        ssa[b] = B.in[F_AERSSA][ab];
      }
      const double amdw = kConAmd / kConAmw, amdo3 = kConAmd / kConAmo3;
      const double h2ovmr = fmax(0.0, q * amdw / (1.0 - q));
      const double o3vmr = fmax(0.0, o3 * amdo3);
      const double tem0 = (1.0 - h2ovmr) * kConAmd + h2ovmr * kConAmw;
      const double tem1c = 100.0 * kConG, tem2c = 1.0e-20 * 1.0e3 * kConAvgd;
      const double coldry = tem2c * delp / (tem1c * tem0 * (1.0 + h2ovmr));
      red[t] = coldry;
      red[FZ_NL + t] = fmax(0.0, coldry * h2ovmr);
      LF.cd = (float)coldry;
      float xf[SG_NFEAT];
      layer_features(pavel, tavel, h2ovmr, o3vmr, co2, ch4, n2o, xf);
      in_env = in_envelope(xf, a.net.norm);
#pragma unroll
      for (int j = 0; j < 7; ++j) x[j] = (xf[j] - nrm[NRM_IN + j]) / nrm[NRM_IN + 8 + j];
      x[7] = 1.0f;
      const int indlay = min(180, max(1, (int)(tavel - 159.0)));
      const double tlyrfr = tavel - (int)tavel;
      const int indlev = min(180, max(1, (int)(tz - 159.0)));
      const double tlvlfr = tz - (int)tz;
      cldk = cf > kEps;
      CloudLayer CL;
      CL.set(f, cf, clwp, relw, ciwp, reiw, cda1, cda3, cda4);
#pragma unroll
      for (int b = 0; b < NBANDS; ++b) {
        LF.pkl[b] = (float)planck_int(a.tab64.kt, b, indlay, tlyrfr);
        LF.pkv[b] = (float)planck_int(a.tab64.kt, b, indlev, tlvlfr);
        LF.aer[b] = (float)(aod[b] * (1.0 - ssa[b]));
        // zero in a clear column: kept only when the column has a cloud (lcf1, below)
        const double tc = CL.band(b, f, a.tab64.kt);
        LF.tcl[b] = (float)tc;
        if (b == 6) tc7 = tc;
      }
    }
    umma::st_canon8(sm + SM_X, t, 0, KIN, x);
    umma::st_canon8(sm + SM_X, t, 8, KIN, x + 8);
    const unsigned fbw = __ballot_sync(0xffffffffu, live && !in_env);
    if (lane == 0) reinterpret_cast<unsigned*>(colv)[COL_FB + warp] = fbw;
    const int nfb = S.count(live && !in_env);   // also: red[] complete
    const int lcf1 = S.any(live && cldk);
    if (t == 0) {
      // precipitable water and diffusivity angles (RLM:910-919, 1041-1050), surface terms
      double tem1 = 0.0, tem2 = 0.0;
      for (int k = 0; k < nlay; ++k) {
        tem1 = tem1 + red[k] + red[FZ_NL + k];
        tem2 = tem2 + red[FZ_NL + k];
      }
      const double amdw = kConAmd / kConAmw;
      const double tem0 = 10.0 * tem2 / (amdw * tem1 * kConG);
      const double pwvcm = tem0 * (top ? IN(F_PLVL, nlay) : IN(F_PLVL, 0));
      const double sfe = B.in[F_SFEMIS][i];
      colv[COL_SEMIS] = (float)((sfe > kEps && sfe <= 1.0) ? sfe : 1.0);
      colv[COL_LCF1] = lcf1 ? 1.0f : 0.0f;
      colv[COL_NFB] = (float)nfb;
      reinterpret_cast<double*>(colv + COL_SCR)[0] = pwvcm;
    }
    S.sync();
    if (t < NBANDS) {
      const double pwvcm = reinterpret_cast<const double*>(colv + COL_SCR)[0];
      const double secd = (t == 0 || t == 3 || t == 9) ? 1.66
                                                         : fmin(1.80, fmax(1.50, c_a0[t] + c_a1[t] * exp(c_a2[t] * pwvcm)));
      colv[COL_SECD + t] = (float)secd;
      const double stemp = B.in[F_SFGTMP][i];
      const double tz0 = top ? IN(F_TLVL, nlay) : IN(F_TLVL, 0);
      colv[COL_PK0 + t] = (float)planck_int(a.tab64.kt, t, min(180, max(1, (int)(stemp - 159.0))), stemp - (int)stemp);
      colv[COL_PKV0 + t] = (float)planck_int(a.tab64.kt, t, min(180, max(1, (int)(tz0 - 159.0))), tz0 - (int)tz0);
    }
    if (live) {
      if (!lcf1) {
#pragma unroll
        for (int b = 0; b < NBANDS; ++b) LF.tcl[b] = 0.0f;
      }
      // band 7 cloud optical depth output (RLM:1087-1097), in FP64
      B.out[O_CLDTAU][i + ld * r] = lcf1 ? tc7 : 0.0;
    }
    if (nfb > 0) {
      // plain taumol for the out-of-envelope layers (and the fallback count)
      float* sb = slot_base(cb);
      Scratch<float> sc;
      sc.tau = sb;
      sc.frac = sb + NGPT * FZ_NLP;
      sc.band = sb + 2 * NGPT * FZ_NLP;
      sc.col = reinterpret_cast<double*>(sb + (2 * NGPT + 3 * NBANDS) * FZ_NLP);
      sc.c0 = c;
      sc.cap = 1;
      sc.ntot = a.ncols;
      gas_column<float, 4, true>(0, t, S, gw, a.blocks, a.nblocks, a.b0, f, a.tab, a.tab64, sc, nullptr, nullptr);
    }
  };

  // ---- per-level sums of a column's flux partials -> outputs (all threads) ----
  auto output = [&](int cc) {
    const Block& B = (a.nblocks == 1) ? a.b0 : a.blocks[find_block(a.blocks, a.nblocks, cc)];
    const int i = cc - B.col0;
    const size_t ld = (size_t)B.ld;
    const bool top = f.top_at_1 != 0;
    const double flxfac = 0.5 * a.cs.fluxfac;   // wtdiff * fluxfac (RLM:3737)
    if (tid <= nlay) {
      const int l = tid;
      double s4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int ww = 0; ww < FZ_NP; ++ww) s4[q] += (double)part[ww * NPART + q * (FZ_NL + 1) + l];
      const double td = s4[0] * flxfac, cd = s4[1] * flxfac, tu = s4[2] * flxfac, cu = s4[3] * flxfac;
      fn[l] = tu - td;
      fn[(FZ_NL + 1) + l] = cu - cd;
      if (l == nlay) {
        B.out[O_TOPFLX][2 * i + 0] = tu;
        B.out[O_TOPFLX][2 * i + 1] = cu;
      }
      if (l == 0) {
        B.out[O_SFCFLX][4 * i + 0] = tu;
        B.out[O_SFCFLX][4 * i + 1] = cu;
        B.out[O_SFCFLX][4 * i + 2] = td;
        B.out[O_SFCFLX][4 * i + 3] = cd;
      }
      if (f.want_flxprf) {
        const int rl = top ? nlp1 - l - 1 : l;
        double* p = B.out[O_FLXPRF] + 4 * (i + ld * (size_t)rl);
        p[0] = tu; p[1] = td; p[2] = cu; p[3] = cd;
      }
    }
    __syncthreads();
    if (tid < nlay) {   // heating rates from the FP64 flux divergence (RLM:3754-3770)
      const int k = tid;
      const int r = top ? nlp1 - (k + 1) - 1 : k;
      const double rfdelp = a.cs.heatfac / B.in[F_DELPIN][i + ld * r];
      B.out[O_HLWC][i + ld * r] = (fn[k] - fn[k + 1]) * rfdelp;
      if (f.want_hlw0) B.out[O_HLW0][i + ld * r] = (fn[(FZ_NL + 1) + k] - fn[(FZ_NL + 1) + k + 1]) * rfdelp;
    }
  };

  // ---- transfer of g-points 128..139 by the layer warps: warp w takes three,
  // lane l layers 4 l .. 4 l + 3, the recurrences as affine-map warp scans ----
  auto tail_transfer = [&](int cc, const float* colv, const float* stau) {
    const int w = warp;   // 0..3
    const int k0 = 4 * lane;
    const bool anyfb = colv[COL_NFB] > 0.0f;
    const uint32_t fbw = anyfb ? (reinterpret_cast<const unsigned*>(colv)[COL_FB + (k0 >> 5)] >> (k0 & 31)) & 15u : 0u;
    const uint32_t lmask = nlay - k0 >= 4 ? 15u : nlay > k0 ? (1u << (nlay - k0)) - 1u : 0u;
    const float semis = colv[COL_SEMIS], reflct = 1.0f - semis;
    const bool mc = colv[COL_LCF1] != 0.0f && f.isubclw > 0;
    const int nw = (nlay + 31) >> 5;
    float a_td[4] = {0.f, 0.f, 0.f, 0.f}, a_cd[4] = {0.f, 0.f, 0.f, 0.f}, a_tu[4] = {0.f, 0.f, 0.f, 0.f},
          a_cu[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
    for (int gi = 0; gi < 3; ++gi) {
      const int g = 128 + 3 * w + gi;
      const int b = fz_band(g);
      const float secd = colv[COL_SECD + b];
      const float osc = nrm[NRM_OSC_T + g], osh = nrm[NRM_OSH_T + g];
      const uint32_t cw =
          (mc && k0 < nlay) ? (__ldg(a.bits + ((size_t)cc * NGPT + g) * nw + (k0 >> 5)) >> (k0 & 31)) & lmask : 0u;
      float tr[4], gsd[4], gsu[4], ef[4], tsd[4], tsu[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        float tau = fmaf(__expf(fmaf(tail[k * FZ_NT + (g - 128)], osc, osh)), cds[k], aer[k * NBANDS + b]);
        if ((fbw >> j) & 1u) tau = stau[g * FZ_NLP + k];
        const float frac = __half2float(frs[k * NGPT + g]);
        const float blay = pkl[k * NBANDS + b];
        const float dpu = pkv[(k + 1) * NBANDS + b] - blay, dpd = pkv[k * NBANDS + b] - blay;
        float atr, fac, tq;
        fz_tbl<true>(a.tab.trec, fmaxf(0.0f, secd * tau), tr[j], atr, fac, tq);
        gsd[j] = frac * (blay + dpd * fac) * atr;
        gsu[j] = frac * (blay + dpu * fac) * atr;
        ef[j] = 1.0f;
        tsd[j] = gsd[j];
        tsu[j] = gsu[j];
        if ((cw >> j) & 1u) {
          const float odcld = secd * tcl[k * NBANDS + b];
          ef[j] = 1.0f - (1.0f - exp_neg(odcld)) * 1.0f;
          float trt, atrt, fact, tqt;
          fz_tbl<false>(a.tab.trec, tq + odcld, trt, atrt, fact, tqt);
          tsd[j] = frac * (blay + dpd * fact) * atrt;
          tsu[j] = frac * (blay + dpu * fact) * atrt;
        }
      }
      // down maps x -> x A + B of the lane's layers, top first, then a suffix
      // scan from the top lane down (RLM:3663-3673)
      float Ac = 1.f, Bc = 0.f, At = 1.f, Bt = 0.f;
#pragma unroll
      for (int j = 3; j >= 0; --j) {
        Bc = tr[j] * Bc + gsd[j]; Ac = tr[j] * Ac;
        const float at = tr[j] * ef[j];
        Bt = at * Bt + (gsd[j] + (tsd[j] - gsd[j])); At = at * At;
      }
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const float ac = __shfl_down_sync(0xffffffffu, Ac, d), bc = __shfl_down_sync(0xffffffffu, Bc, d);
        const float at = __shfl_down_sync(0xffffffffu, At, d), bt = __shfl_down_sync(0xffffffffu, Bt, d);
        if (lane + d < 32) { Bc = Ac * bc + Bc; Ac = Ac * ac; Bt = At * bt + Bt; At = At * at; }
      }
      float xc = __shfl_down_sync(0xffffffffu, Bc, 1), xt = __shfl_down_sync(0xffffffffu, Bt, 1);
      if (lane == 31) { xc = 0.f; xt = 0.f; }
#pragma unroll
      for (int j = 3; j >= 0; --j) {
        xc = xc * tr[j] + gsd[j];
        if ((cw >> j) & 1u) xt = xt * tr[j] * ef[j] + gsd[j] + 1.0f * (tsd[j] - gsd[j]);
        else xt = xt * tr[j] + gsd[j];
        a_cd[j] += xc;
        a_td[j] += xt;
      }
      // surface emission and reflection (RLM:3682-3691)
      const float rad0 = semis * __half2float(frs[g]) * colv[COL_PK0 + b];
      const float r0c = rad0 + reflct * __shfl_sync(0xffffffffu, xc, 0);
      const float r0t = rad0 + reflct * __shfl_sync(0xffffffffu, xt, 0);
      // up maps, bottom first, prefix scan from lane 0 up (RLM:3700-3730)
      float Uc = 1.f, Wc = 0.f, Ut = 1.f, Wt = 0.f;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        Wc = tr[j] * Wc + gsu[j]; Uc = tr[j] * Uc;
        const float at = tr[j] * ef[j];
        Wt = at * Wt + (gsu[j] + (tsu[j] - gsu[j])); Ut = at * Ut;
      }
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const float uc = __shfl_up_sync(0xffffffffu, Uc, d), wc = __shfl_up_sync(0xffffffffu, Wc, d);
        const float ut = __shfl_up_sync(0xffffffffu, Ut, d), wt = __shfl_up_sync(0xffffffffu, Wt, d);
        if (lane >= d) { Wc = Uc * wc + Wc; Uc = Uc * uc; Wt = Ut * wt + Wt; Ut = Ut * ut; }
      }
      const float pu_c = __shfl_up_sync(0xffffffffu, Uc, 1), pw_c = __shfl_up_sync(0xffffffffu, Wc, 1);
      const float pu_t = __shfl_up_sync(0xffffffffu, Ut, 1), pw_t = __shfl_up_sync(0xffffffffu, Wt, 1);
      xc = lane == 0 ? r0c : pu_c * r0c + pw_c;
      xt = lane == 0 ? r0t : pu_t * r0t + pw_t;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        a_cu[j] += xc;
        a_tu[j] += xt;
        xc = xc * tr[j] + gsu[j];
        if ((cw >> j) & 1u) xt = xt * tr[j] * ef[j] + gsu[j] + 1.0f * (tsu[j] - gsu[j]);
        else xt = xt * tr[j] + gsu[j];
      }
    }
    float* mp = part + (4 + w) * NPART;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int lv = k0 + j;
      if (lv <= nlay) {
        mp[0 * (FZ_NL + 1) + lv] = lv == nlay ? 0.0f : a_td[j];
        mp[1 * (FZ_NL + 1) + lv] = lv == nlay ? 0.0f : a_cd[j];
        mp[2 * (FZ_NL + 1) + lv] = a_tu[j];
        mp[3 * (FZ_NL + 1) + lv] = a_cu[j];
      }
    }
  };

  int it = 0, prev = -1;
  if (is_layer && (int)blockIdx.x < a.ncols) prologue(blockIdx.x, 0);
  for (int cc = blockIdx.x; cc < a.ncols; cc += gridDim.x, ++it) {
    const int cb = it & 1;
    const float* colv = colv0 + cb * COL_N;
    __syncthreads();   // the previous column's transfer and this column's prologue are done
    if (prev >= 0) output(prev);
    if (is_layer) {
#pragma unroll
      for (int b = 0; b < NBANDS; ++b) {
        pkl[t * NBANDS + b] = LF.pkl[b];
        pkv[(t + 1) * NBANDS + b] = LF.pkv[b];
        tcl[t * NBANDS + b] = LF.tcl[b];
        aer[t * NBANDS + b] = LF.aer[b];
      }
      cds[t] = LF.cd;
      if (t < NBANDS) pkv[t] = colv[COL_PKV0 + t];
    }
    // ---------------- network: X -> H1 -> H2 -> outputs ----------------
    sync_for_mma();
    if (tid == 0) {
      umma::fence_after_sync();
      umma::mma(tb + TM_D12, umma::tile_desc(sbase + SM_X, KIN, 0), umma::tile_desc(sbase + SM_W1, KIN, 0), ID128, 0u);
      umma::commit(mbar);
    }
    if (!wait_mma()) break;
    const float* b2 = a.net.params + P_B2;
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
      // warpgroup q = warp / 4 owns hidden units [64 q, 64 q + 64)
      const int row = 32 * wq + lane;
      const int h0 = 64 * (warp >> 2);
#pragma unroll 1
      for (int c0 = h0; c0 < h0 + 64; c0 += 16) {
        float v[16], h[16];
        umma::tmem_ld16(umma::tmem_addr(tb, wq, TM_D12 + c0), v);
#pragma unroll
        for (int j = 0; j < 16; ++j) h[j] = silu(v[j] + (layer == 1 ? __ldg(b2 + c0 + j) : 0.0f));
        umma::st_canon8(sm + SM_HF, row, c0, HID, h);
        umma::st_canon8(sm + SM_HF, row, c0 + 8, HID, h + 8);
      }
      sync_for_mma();
      if (tid == 0) {
        umma::fence_after_sync();
        if (layer == 0) {
#pragma unroll 1
          for (int s = 0; s < HID / 16; ++s)
            umma::mma(tb + TM_D12, umma::tile_desc(sbase + SM_HF, HID, s), umma::tile_desc(sbase + SM_W2, HID, s),
                      ID128, s > 0 ? 1u : 0u);
        } else {
          // optical depths of g 0..127, transposed: D[g][layer] = W3[g] . H2[layer]
#pragma unroll 1
          for (int s = 0; s < HID / 16; ++s)
            umma::mma(tb + TM_TAU, umma::tile_desc(sbase + SM_W3A, HID, s), umma::tile_desc(sbase + SM_HF, HID, s),
                      ID128, s > 0 ? 1u : 0u);
          // fractions (and optical depths of g 128..139): D[layer][j] = H2[layer] . W3F[j]
#pragma unroll 1
          for (int s = 0; s < HID / 16; ++s)
            umma::mma(tb + TM_DF, umma::tile_desc(sbase + SM_HF, HID, s), umma::tile_desc(sbase + SM_W3F, HID, s),
                      IDF, s > 0 ? 1u : 0u);
        }
        umma::commit(mbar);
      }
      if (!wait_mma()) break;
    }
    if (failed) break;
    // ---------------- fraction epilogue (overwrites H2: its MMAs are complete) ----------------
    {
      const int row = 32 * wq + lane;
      const bool live = row < nlay;
      const bool fb = colv[COL_NFB] > 0.0f &&
                      ((reinterpret_cast<const unsigned*>(colv)[COL_FB + (row >> 5)] >> (row & 31)) & 1u);
      const float* sb = slot_base(cb);
      // warpgroup 0: bands 1-6 (g 0..75), warpgroup 1: bands 7-16 and the raw tail outputs
      if (warp < 4) frac_epilogue<0, 76>(tb, wq, row, live, fb, nrm, cds, aer, frs, tail, sb, sb + NGPT * FZ_NLP);
      else frac_epilogue<76, 152>(tb, wq, row, live, fb, nrm, cds, aer, frs, tail, sb, sb + NGPT * FZ_NLP);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();

    if (!is_layer) {
      // ---------------- transfer of g 0..127: lane <-> g-point ----------------
      const int w = warp - 4;
      const int g = 32 * w + lane;
      const int b = fz_band(g);
      const float secd = colv[COL_SECD + b];
      const float semis = colv[COL_SEMIS];
      const float reflct = 1.0f - semis;
      const bool mc = colv[COL_LCF1] != 0.0f && f.isubclw > 0;
      const int nw = (nlay + 31) >> 5;
      uint32_t cb0 = 0u, cb1 = 0u, cb2 = 0u, cb3 = 0u;   // sub-column flags, one word per 32 layers
      if (mc) {
        const uint32_t* bp = a.bits + ((size_t)cc * NGPT + g) * nw;
        cb0 = __ldg(bp);
        if (nw > 1) cb1 = __ldg(bp + 1);
        if (nw > 2) cb2 = __ldg(bp + 2);
        if (nw > 3) cb3 = __ldg(bp + 3);
      }
      // the flag bits of chunk j (layers CH j .. CH j + CH - 1 below nlay)
      auto chunk_bits = [&](int j) -> uint32_t {
        const int wd = (CH * j) >> 5;
        const uint32_t wv = wd == 0 ? cb0 : wd == 1 ? cb1 : wd == 2 ? cb2 : cb3;
        const int n = nlay - CH * j;
        const uint32_t m = n >= CH ? (1u << CH) - 1u : (1u << n) - 1u;
        return (wv >> ((CH * j) & 31)) & m;
      };
      const bool anyfb = colv[COL_NFB] > 0.0f;
      const unsigned* fbm = reinterpret_cast<const unsigned*>(colv) + COL_FB;
      const float* stau = slot_base(cb);
      const float osc = nrm[NRM_OSC_T + g], osh = nrm[NRM_OSH_T + g];
      float* mypart = part + w * NPART;
      const int nch = (nlay + CH - 1) / CH;
      float radtd = 0.0f, radcd = 0.0f;
      // ---- down sweep (RLM:3598-3673), layers top to bottom ----
#pragma unroll 1
      for (int j = nch - 1; j >= 0; --j) {
        float tauv[CH];
        umma::tmem_ld16(umma::tmem_addr(tb, wq, TM_TAU + CH * j), tauv);
#pragma unroll
        for (int ii = 0; ii < CH; ++ii) {
          const int k = CH * j + ii;
          tauv[ii] = fmaf(__expf(fmaf(tauv[ii], osc, osh)), cds[k], aer[k * NBANDS + b]);
        }
        const uint32_t cbj = chunk_bits(j);
        const uint32_t fbj = anyfb ? (fbm[(CH * j) >> 5] >> ((CH * j) & 31)) & ((1u << CH) - 1u) : 0u;
        if (fbj) {   // out-of-envelope layers (rare): optical depths of plain taumol
#pragma unroll 1
          for (int ii = 0; ii < CH; ++ii)
            if ((fbj >> ii) & 1u) tauv[ii] = stau[g * FZ_NLP + CH * j + ii];
        }
        // pass 1: clear-sky gas terms of the chunk's layers (RLM:3598-3624),
        // independent of one another; padding layers come out neutral
        float trs[CH], gss[CH], gsdv[CH], odqv[CH];
#pragma unroll
        for (int ii = 0; ii < CH; ++ii) {
          const int k = CH * j + ii;
          const float frac = __half2float(frs[k * NGPT + g]);
          const float blay = pkl[k * NBANDS + b];
          const float od = fmaxf(0.0f, secd * tauv[ii]);
          float atrgas, gasfac;
          fz_tbl<true>(a.tab.trec, od, trs[ii], atrgas, gasfac, odqv[ii]);
          gsdv[ii] = frac * (blay + (pkv[k * NBANDS + b] - blay) * gasfac) * atrgas;
          gss[ii] = frac * (blay + (pkv[(k + 1) * NBANDS + b] - blay) * gasfac) * atrgas;
        }
        // pass 2: the down recurrences layer by layer (RLM:3663-3673); cloudy
        // sub-columns add their total-sky terms (RLM:3627-3660, clfm = 1)
        float atd[CH], acd[CH], tss[CH];
#pragma unroll
        for (int ii = CH - 1; ii >= 0; --ii) {
          const int k = CH * j + ii;
          const bool cl = (cbj >> ii) & 1u;
          radcd = radcd * trs[ii] + gsdv[ii];
          float tsu = gss[ii];
          if (__any_sync(0xffffffffu, cl)) {
            float rtd = radtd * trs[ii] + gsdv[ii];
            if (cl) {
              const float frac = __half2float(frs[k * NGPT + g]);
              const float blay = pkl[k * NBANDS + b];
              const float odcld = secd * tcl[k * NBANDS + b];
              const float ef = 1.0f - (1.0f - exp_neg(odcld)) * 1.0f;
              float trtot, atrtot, totfac, tq2;
              fz_tbl<false>(a.tab.trec, odqv[ii] + odcld, trtot, atrtot, totfac, tq2);
              const float tsd = frac * (blay + (pkv[k * NBANDS + b] - blay) * totfac) * atrtot;
              tsu = frac * (blay + (pkv[(k + 1) * NBANDS + b] - blay) * totfac) * atrtot;
              rtd = radtd * trs[ii] * ef + gsdv[ii] + 1.0f * (tsd - gsdv[ii]);
            }
            radtd = rtd;
          } else {
            radtd = radtd * trs[ii] + gsdv[ii];
          }
          atd[ii] = radtd;
          acd[ii] = radcd;
          tss[ii] = tsu;
        }
        umma::tmem_st16(umma::tmem_addr(tb, wq, TM_TR + CH * j), trs);
        umma::tmem_st16(umma::tmem_addr(tb, wq, TM_GSU + CH * j), gss);
        umma::tmem_st16(umma::tmem_addr(tb, wq, tm_tsu(j)), tss);
        const float std_ = warp_sum16(atd, lane), scd_ = warp_sum16(acd, lane);
        const int lvl = CH * j + ((lane >> 1) & 15);
        if ((lane & 1) == 0 && lvl <= nlay) {
          mypart[0 * (FZ_NL + 1) + lvl] = lvl == nlay ? 0.0f : std_;
          mypart[1 * (FZ_NL + 1) + lvl] = lvl == nlay ? 0.0f : scd_;
        }
      }
      if (lane == 0 && (nlay % CH) == 0) {   // TOA level when it starts a chunk of its own
        mypart[0 * (FZ_NL + 1) + nlay] = 0.0f;
        mypart[1 * (FZ_NL + 1) + nlay] = 0.0f;
      }
      umma::tmem_wait_st();
      // ---- surface emission and reflection (RLM:3682-3691) ----
      const float rad0 = semis * __half2float(frs[g]) * colv[COL_PK0 + b];
      float radtu = rad0 + reflct * radtd, radcu = rad0 + reflct * radcd;
      {
        const float s0 = warp_sum(radtu), s1 = warp_sum(radcu);
        if (lane == 0) {
          mypart[2 * (FZ_NL + 1)] = s0;
          mypart[3 * (FZ_NL + 1)] = s1;
        }
      }
      // ---- up sweep (RLM:3700-3730), layers bottom to top ----
#pragma unroll 1
      for (int j = 0; j < nch; ++j) {
        float trs[CH], gss[CH], tss[CH];
        umma::tmem_ld16(umma::tmem_addr(tb, wq, TM_TR + CH * j), trs);
        umma::tmem_ld16(umma::tmem_addr(tb, wq, TM_GSU + CH * j), gss);
        umma::tmem_ld16(umma::tmem_addr(tb, wq, tm_tsu(j)), tss);
        const uint32_t cbj = chunk_bits(j);
        float atu[CH], acu[CH];
#pragma unroll
        for (int ii = 0; ii < CH; ++ii) {
          const int k = CH * j + ii;
          const bool cl = (cbj >> ii) & 1u;
          radcu = radcu * trs[ii] + gss[ii];
          // cloudy sub-column (clfm = 1): efclrfr = exp(-secdiff taucld), recomputed
          const float ef = 1.0f - (1.0f - exp_neg(secd * tcl[k * NBANDS + b])) * 1.0f;
          const float rcl = radtu * trs[ii] * ef + gss[ii] + 1.0f * (tss[ii] - gss[ii]);
          radtu = cl ? rcl : radtu * trs[ii] + gss[ii];
          atu[ii] = radtu;
          acu[ii] = radcu;
        }
        const float stu = warp_sum16(atu, lane), scu = warp_sum16(acu, lane);
        const int lvl = CH * j + 1 + ((lane >> 1) & 15);
        if ((lane & 1) == 0 && lvl <= nlay) {
          mypart[2 * (FZ_NL + 1) + lvl] = stu;
          mypart[3 * (FZ_NL + 1) + lvl] = scu;
        }
      }
    } else {
      if (cc + (int)gridDim.x < a.ncols) prologue(cc + gridDim.x, cb ^ 1);
      tail_transfer(cc, colv, slot_base(cb));
    }
    prev = cc;
  }
  if (!failed && prev >= 0) {
    __syncthreads();
    output(prev);
  }
  // leave: every MMA this CTA issued has completed (or the wait timed out and
  // the error is recorded); release tensor memory
  if (failed) umma::mbar_wait(mbar, phase ^ 1u, 1u << 20);
  umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && *sfail && a.net.err) atomicCAS(a.net.err, 0, 1);
  if (warp == 0) umma::tmem_dealloc(tb, 512);
}

bool s_prepared = false;

}  // namespace

size_t sg_fused_work_bytes(int num_sms) { return fz_cta_bytes() * (size_t)num_sms; }

bool sg_fused_applies(const Flags& f) {
  return f.surrogate && !f.gas_only && f.nlay >= 1 && f.nlay <= FZ_NL - 1 && f.isubclw > 0 && !f.want_hlwb;
}

cudaError_t sg_fused_prepare() {
  cudaError_t e = cudaFuncSetAttribute(lw_sg_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FZ_SMEM);
  if (e != cudaSuccess) return e;
  int occ = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, lw_sg_fused_kernel, FZ_THREADS, FZ_SMEM)) != cudaSuccess)
    return e;
  // one CTA per SM is what makes the 512-column TMEM allocation safe
  if (occ != 1) return cudaErrorLaunchOutOfResources;
  s_prepared = true;
  return cudaSuccess;
}

cudaError_t sg_fused_launch(const Block* blocks, int nblocks, const Block& b0, int ncols, const Flags& f,
                            const Consts& cs, const Tables<float>& tab, const Tables<double>& tab64,
                            const uint32_t* bits, void* work, size_t work_bytes, int num_sms, cudaStream_t st) {
  if (!s_prepared) return cudaErrorNotReady;
  const SgNetView net = sg_net_view();
  if (!net.ready) return cudaErrorNotReady;
  const int grid = std::min(ncols, num_sms);
  if (grid < 1) return cudaSuccess;
  if (work_bytes < fz_cta_bytes() * (size_t)grid) return cudaErrorMemoryAllocation;
  FusedArgs a;
  a.blocks = blocks;
  a.nblocks = nblocks;
  a.b0 = b0;
  a.ncols = ncols;
  a.f = f;
  a.cs = cs;
  a.tab = tab;
  a.tab64 = tab64;
  a.bits = bits;
  a.net = net;
  a.work = static_cast<unsigned char*>(work);
  lw_sg_fused_kernel<<<grid, FZ_THREADS, FZ_SMEM, st>>>(a);
  return cudaGetLastError();
}

}  // namespace lw
