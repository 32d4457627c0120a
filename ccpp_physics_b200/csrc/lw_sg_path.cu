// lw_sg_path.cu -- the column path behind the learned gas optics
// (RRTMG_LW_SURROGATE calls with McICA clouds, up to 127 layers, no hlwb).
//
// Per chunk of columns, after the McICA kernel (lw_mcica.cu):
//   mlp_h_pack_kernel (lw_mlp.cu)  the network inputs of every column
//       (normalised features, coldry, aerosol depths) as one contiguous
//       record, and the list of the columns that have a layer outside the
//       training envelope;
//   mlp_h_kernel (lw_mlp.cu)  the network: per layer the 140 gas + aerosol
//       optical depths and band-normalised Planck fractions (taumol
//       outputs, RLM:3836-4013) in a compact FP16 hand-off
//       hnd[column][8-layer block][{tau, frac} x 140 g-points][8 layers];
//   lw_sg_fallback_kernel  plain FP32 setcoef + taumol (lw_gas.cuh) for the
//       layers of the listed columns that lie outside the envelope, written
//       over the network's values in the hand-off;
//   lw_sg_rt_kernel  per column the rest of rrtmg_lw_run: the driver's
//       column terms (RLM:785-1050), Planck integrals (setcoef, RLM:2251-
//       2283), cloud optics (cldprop, RLM:1589-1799), rtrnmc (RLM:3420-3785)
//       and the output mapping (RLM:1228-1304).
//
// The transfer kernel gives each g-point a lane: 5 warps of 28 lanes cover
// a column's 140 g-points, and every lane runs the reference's down sweep,
// surface term and up sweep for its own g-point layer by layer, in the
// Fortran's operation order (FP32, as the FP32 path).  The down sweep keeps
// each layer's {1 - transmittance, upward source} as an FP16 pair in tensor
// memory (the lane's own TMEM lane, one column per layer), where the up
// sweep reads them back; only cloudy sub-column layers recompute their
// total-sky terms there.
// Per-level sums over g-points are warp reductions over 8 levels at a time,
// then an FP64 sum over the 5 warps; heating rates come from the FP64 flux
// divergence.  A lane reads its g-point's optical depths and fractions of 8
// layers with one 16-byte load each, one 8-layer block ahead of its work.
// A CTA holds 3 such column groups (15 warps) and one copy of the rlwinit
// records {1 - exp_tbl, tfn_tbl} in FP16 in shared memory, so each lookup is
// a shared-memory gather.  Each group first computes its column's band
// fields {pklay, pklev above - pklay, pklev below - pklay, secdiff * taucld}
// (FP64 arithmetic, stored FP32) into its shared memory.
#include <algorithm>
#include <cstdio>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lw_launch.h"
#include "lw_rt.cuh"
#include "lw_umma.cuh"

namespace lw {
namespace {

constexpr int SR_WARPS = 5;                   // warps of a column group
constexpr int SR_GPW = 28;                    // g-points per warp (5 x 28 = 140)
constexpr int SR_GT = SR_WARPS * 32;          // threads of a column group
#ifndef LW_SR_GROUPS
#define LW_SR_GROUPS 3
#endif
constexpr int SR_GROUPS = LW_SR_GROUPS;       // column groups per CTA
constexpr int SR_THREADS = SR_GROUPS * SR_GT;
constexpr int SR_NL = 128;                    // layers a group holds (nlay <= 127)
constexpr int SR_CH = 8;                      // layers per sweep chunk (one 16-byte hand-off load)
constexpr int SR_HCH = 2 * NGPT * SR_CH;      // halves per 8-layer hand-off block of a column
static_assert(SR_WARPS * SR_GPW == NGPT, "g-points per column");

// shared memory of one column group
struct SrGroup {
  float4 bf[SR_NL][NBANDS];             // {pklay, pklev above - pklay, pklev below - pklay, secdiff * taucld}
  float part[SR_WARPS][4][SR_NL + 1];   // per-warp level sums: total down, clear down, total up, clear up
  union {
    struct {
      float pkv[SR_NL + 1][NBANDS];     // pklev(b, l) (prologue)
    } p;
    double fn[2][SR_NL + 1];            // net flux (total, clear sky; output)
  } u;
  double pw[SR_WARPS][2];               // per-warp sums of coldry + colh2o and of colh2o (prologue)
  float secd[NBANDS];                   // diffusivity angle per band
  float pk0[NBANDS];                    // pklay(b, 0) (surface temperature)
  float semis;
  int lcf1;
  int pad_[2];
};
// rlwinit records {1 - exp_tbl, tfn_tbl} in FP16 (RLM:1474-1501)
constexpr size_t SR_TAB_BYTES = (((size_t)NTBL + 1) * sizeof(__half2) + 127) & ~(size_t)127;
constexpr size_t SR_GROUP_BYTES = (sizeof(SrGroup) + 127) & ~(size_t)127;
constexpr size_t SR_SMEM = SR_TAB_BYTES + SR_GROUPS * SR_GROUP_BYTES + 128;   // + the TMEM base
static_assert(SR_SMEM > 114 * 1024, "one CTA per SM: its 512 tensor-memory columns never wait");
static_assert(SR_GROUPS * SR_WARPS <= 16, "at most four warps per tensor-memory lane slice");
static_assert(SR_SMEM <= 227 * 1024, "transfer kernel shared memory");

struct SrArgs {
  const Block* blocks;
  int nblocks;
  Block b0;
  const int* colmap;      // block of every global column (nblocks > 1)
  int c0, nc;             // chunk: global columns [c0, c0 + nc)
  Flags f;
  Consts cs;
  const float* trec;      // FP32 rlwinit records {exp, tfn, tau, 0}
  const double* kt64;     // FP64 coefficient tables
  const uint32_t* bits;   // McICA sub-column flags [column][140][nw]
  const __half* hnd;      // [nc][nlay/8][tau 140 | frac 140][8 layers]
};

// Sum over the warp's lanes of a[i], i = 0..7: every lane returns the sum
// for index (lane >> 2) & 7 (recursive halving, 9 shuffles).
__device__ __forceinline__ float warp_sum8(const float (&a)[8], int lane) {
  float b[4], c[2];
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float keep = h16 ? a[4 + j] : a[j], send = h16 ? a[j] : a[4 + j];
    b[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float keep = h8 ? b[2 + j] : b[j], send = h8 ? b[j] : b[2 + j];
    c[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float d = (h4 ? c[1] : c[0]) + __shfl_xor_sync(0xffffffffu, h4 ? c[0] : c[1], 4);
  d += __shfl_xor_sync(0xffffffffu, d, 2);
  return d + __shfl_xor_sync(0xffffffffu, d, 1);
}

__device__ __forceinline__ float warp_sum_all(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// record index it = int(10000 x / (bpade + x) + 0.5) of an optical depth
// (RLM:3602-3603).  x is finite, >= 0 and at most ~1e10 here (the hand-off
// clamps optical depths below the FP16 maximum; a cloudy layer past the
// table's end adds 1e10), so x / (bpade + x) <= 1 and the index lies in
// [0, NTBL] without a clamp.
__device__ __forceinline__ int tbl_index(float x) {
  return (int)(float(kTblint) * __fdividef(x, float(kBpade) + x) + 0.5f);
}

// Total-sky terms of a cloudy sub-column layer (RLM:3627-3660, clfm = 1):
// efclrfr and {1 - exp_tbl, tfn_tbl} of odtot = odepth + odcld, where odepth
// is tau_tbl(it) = bpade it / (10000 - it) when the gas lookup used the table
// (RLM:3614, 1487-1488).
__device__ __forceinline__ void cloud_terms(float od, int it, float odcld, const __half2* tab, float& ef,
                                            float& atrtot, float& totfac) {
  ef = 1.0f - (1.0f - __expf(-odcld)) * 1.0f;
  const float odq = it < 0 ? od : it >= NTBL ? 1.0e10f : __fdividef(float(kBpade) * (float)it, (float)(NTBL - it));
  const float odtot = odq + odcld;
  if (odtot < 0.06f) {
    totfac = float(kRec6) * odtot;
    atrtot = odtot - 0.5f * odtot * odtot;
  } else {
    const float2 e = __half22float2(tab[tbl_index(odtot)]);
    atrtot = e.x;
    totfac = e.y;
  }
}

// cldprop band optics of one layer (RLM:1589-1799), FP64: the layer's
// band-independent terms once (set: indices and interpolation fractions,
// one division), then each band's table interpolation (band); the
// arithmetic of band_taucld (lw_gas.cuh) with the per-band work hoisted.
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
    else if (f.ilwcice == 3) { ifac = (fmax(5.0, 1.0315 * reiw) - 2.0) / 3.0; }
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

__device__ __forceinline__ int band_of(int g) {
  return g < 10 ? 0 : g < 22 ? 1 : g < 38 ? 2 : g < 52 ? 3 : g < 68 ? 4 : g < 76 ? 5 : g < 88 ? 6 : g < 96 ? 7
       : g < 108 ? 8 : g < 114 ? 9 : g < 122 ? 10 : g < 130 ? 11 : g < 134 ? 12 : g < 136 ? 13 : g < 138 ? 14 : 15;
}

// {a, b} rounded to an FP16 pair, as the bits of one 32-bit word
__device__ __forceinline__ uint32_t h2_bits(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// 8 FP16 values of a 16-byte hand-off load
__device__ __forceinline__ void unpack8(const uint4 q, float (&o)[8]) {
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
  const float2 c = __half22float2(*reinterpret_cast<const __half2*>(&q.z));
  const float2 d = __half22float2(*reinterpret_cast<const __half2*>(&q.w));
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y; o[6] = d.x; o[7] = d.y;
}

__global__ void __launch_bounds__(SR_THREADS, 1) lw_sg_rt_kernel(SrArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];
  __half2* tab = reinterpret_cast<__half2*>(sm);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SR_SMEM - 128);
  for (int i = threadIdx.x; i <= NTBL; i += SR_THREADS) {
    const float4 r = __ldg(reinterpret_cast<const float4*>(a.trec) + i);
    tab[i] = __floats2half2_rn(1.0f - r.x, r.y);
  }
  // tensor memory holds each lane's up-sweep terms between the two sweeps:
  // warp W uses lane slice W % 4 and columns [128 (W / 4), +128), one per layer
  if (threadIdx.x < 32) {
    umma::tmem_alloc(tslot, 512);
    umma::tmem_relinquish();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = *tslot;
  const int W = threadIdx.x >> 5;
  const uint32_t tw = umma::tmem_addr(tbase, W & 3, 128 * (W >> 2));
  const int G = threadIdx.x / SR_GT, gt = threadIdx.x - G * SR_GT;
  SrGroup& S = *reinterpret_cast<SrGroup*>(sm + SR_TAB_BYTES + G * SR_GROUP_BYTES);
  const GroupSync sync{1 + G, SR_GT};
  const int gw = gt >> 5, lane = gt & 31;
  const Flags& f = a.f;
  const int nlay = f.nlay, nlp1 = nlay + 1;
  const int nch = (nlay + SR_CH - 1) / SR_CH;
  const bool top = f.top_at_1 != 0;
  const double* kt64 = a.kt64;
  // band-field rows above the top layer stay zero: those padding layers are
  // neutral in the sweeps (no source; their optical depth is zero too)
  for (int t = nlay + gt / NBANDS; t < SR_NL; t += SR_GT / NBANDS) S.bf[t][gt % NBANDS] = make_float4(0.f, 0.f, 0.f, 0.f);

  for (int cc = blockIdx.x * SR_GROUPS + G; cc < a.nc; cc += gridDim.x * SR_GROUPS) {
    const int c = a.c0 + cc;
    const Block& B = (a.nblocks == 1) ? a.b0 : a.blocks[__ldg(a.colmap + c)];
    const int i = c - B.col0;
    const size_t ld = (size_t)B.ld;
    auto IN = [&](int fld, int row) -> double { return B.in[fld][i + ld * row]; };

    // ---------------- column terms and band fields (thread <-> layer) ----------------
    {
      const int t = gt;
      const bool live = t < nlay;
      const int r = top ? nlay - 1 - t : t;   // input row of layer t (and of its top level)
      const int rl = top ? nlay - 1 - t : t + 1;
      float pkl[NBANDS];
      bool cldk = false;
      double colw = 0.0, colh = 0.0;   // this layer's coldry and water column
      double cf = 0.0, clwp = 0.0, relw = 0.0, ciwp = 0.0, reiw = 0.0, cda1 = 0.0, cda3 = 0.0, cda4 = 0.0;
      if (live) {
        const double delp = IN(F_DELPIN, r), q = IN(F_QLYR, r), tavel = IN(F_TLYR, r), tz = IN(F_TLVL, rl);
        cf = IN(F_CLDCF, r);
        if (f.ilwcliq > 0) {
          clwp = IN(F_LWP, r); relw = IN(F_RELIQ, r); ciwp = IN(F_IWP, r); reiw = IN(F_REICE, r);
          cda1 = IN(F_RWP, r); cda3 = IN(F_SWP, r); cda4 = IN(F_RESNOW, r);
        } else {
          cda1 = IN(F_CLDOD, r);
        }
        // coldry and the water column (RLM:823-850)
        const double amdw = kConAmd / kConAmw;
        const double h2ovmr = fmax(0.0, q * amdw / (1.0 - q));
        const double tem0 = (1.0 - h2ovmr) * kConAmd + h2ovmr * kConAmw;
        const double tem1c = 100.0 * kConG, tem2c = 1.0e-20 * 1.0e3 * kConAvgd;
        const double coldry = tem2c * delp / (tem1c * tem0 * (1.0 + h2ovmr));
        colw = coldry;
        colh = fmax(0.0, coldry * h2ovmr);
        const int indlay = min(180, max(1, (int)(tavel - 159.0)));
        const double tlyrfr = tavel - (int)tavel;
        const int indlev = min(180, max(1, (int)(tz - 159.0)));
        const double tlvlfr = tz - (int)tz;
#pragma unroll
        for (int b = 0; b < NBANDS; ++b) {
          pkl[b] = (float)planck_int(kt64, b, indlay, tlyrfr);
          S.u.p.pkv[t + 1][b] = (float)planck_int(kt64, b, indlev, tlvlfr);
        }
        cldk = cf > kEps;
      }
      if (t < NBANDS) {
        // surface level and surface temperature (RLM:2251-2262)
        const double tz0 = top ? IN(F_TLVL, nlay) : IN(F_TLVL, 0);
        const double stemp = B.in[F_SFGTMP][i];
        S.u.p.pkv[0][t] = (float)planck_int(kt64, t, min(180, max(1, (int)(tz0 - 159.0))), tz0 - (int)tz0);
        S.pk0[t] = (float)planck_int(kt64, t, min(180, max(1, (int)(stemp - 159.0))), stemp - (int)stemp);
      }
      // the column sums of the precipitable water (RLM:910-919) as a warp
      // tree, then over the group's warps: the reference adds layer by layer,
      // which kept one warp in a serial FP64 chain while the group waited
      {
        double s1 = colw + colh, s2 = colh;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          s1 += __shfl_xor_sync(0xffffffffu, s1, o);
          s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        }
        if (lane == 0) {
          S.pw[gw][0] = s1;
          S.pw[gw][1] = s2;
        }
      }
      const int lcf1 = sync.any(live && cldk);   // also: pw[] and pkv[] complete
      if (t < NBANDS) {
        // precipitable water (every band's thread forms the same sum) and the
        // diffusivity angle (RLM:1041-1050)
        double tem1 = 0.0, tem2 = 0.0;
#pragma unroll
        for (int w = 0; w < SR_WARPS; ++w) {
          tem1 += S.pw[w][0];
          tem2 += S.pw[w][1];
        }
        const double amdw = kConAmd / kConAmw;
        const double tem0 = 10.0 * tem2 / (amdw * tem1 * kConG);
        const double pwvcm = tem0 * (top ? IN(F_PLVL, nlay) : IN(F_PLVL, 0));
        const double secd = (t == 0 || t == 3 || t == 9)
                                ? 1.66
                                : fmin(1.80, fmax(1.50, c_a0[t] + c_a1[t] * exp(c_a2[t] * pwvcm)));
        S.secd[t] = (float)secd;
        if (t == 0) {
          const double sfe = B.in[F_SFEMIS][i];
          S.semis = (float)((sfe > kEps && sfe <= 1.0) ? sfe : 1.0);
          S.lcf1 = lcf1;
        }
      }
      sync.sync();
      if (live) {
        CloudLayer CL;
        CL.set(f, cf, clwp, relw, ciwp, reiw, cda1, cda3, cda4);
#pragma unroll 1
        for (int b = 0; b < NBANDS; ++b) {
          const double tc = lcf1 ? CL.band(b, f, kt64) : 0.0;
          if (b == 6) B.out[O_CLDTAU][i + ld * r] = tc;   // band 7 cloud optical depth (RLM:1087-1097)
          S.bf[t][b] = make_float4(pkl[b], S.u.p.pkv[t + 1][b] - pkl[b], S.u.p.pkv[t][b] - pkl[b], S.secd[b] * (float)tc);
        }
      }
      sync.sync();   // band fields complete
    }

    // ---------------- transfer: lane <-> g-point ----------------
    {
      const bool act = lane < SR_GPW;
      const int g = act ? SR_GPW * gw + lane : NGPT - 1;
      const int b = band_of(g);
      const float secd = S.secd[b];
      const bool mc = S.lcf1 != 0 && f.isubclw > 0 && act;
      const int nw = (nlay + 31) >> 5;
      uint32_t cw0 = 0u, cw1 = 0u, cw2 = 0u, cw3 = 0u;   // sub-column flags, one word per 32 layers
      if (mc) {
        const uint32_t* bp = a.bits + ((size_t)c * NGPT + g) * nw;
        cw0 = __ldg(bp);
        if (nw > 1) cw1 = __ldg(bp + 1);
        if (nw > 2) cw2 = __ldg(bp + 2);
        if (nw > 3) cw3 = __ldg(bp + 3);
      }
      // The up-sweep sources are stored relative to the band's surface Planck
      // value, which keeps them O(1) and well inside the FP16 normal range (the
      // sources themselves are ~1e-5 in these radiance units).
      const float su_scale = S.pk0[b] > 0.0f ? S.pk0[b] : 1.0f, su_inv = 1.0f / su_scale;
      // this g-point's 8-layer blocks: tau at hq[j * 2 * NGPT], fractions at hq[j * 2 * NGPT + NGPT]
      const uint4* hq = reinterpret_cast<const uint4*>(a.hnd + (size_t)cc * nch * SR_HCH) + g;
      const uint4 zero4 = make_uint4(0u, 0u, 0u, 0u);
      float* P = &S.part[gw][0][0];
      auto chunk_bits = [&](int j) -> uint32_t {
        const int k0 = SR_CH * j;
        const int wd = k0 >> 5;
        const uint32_t wv = wd == 0 ? cw0 : wd == 1 ? cw1 : wd == 2 ? cw2 : cw3;
        const int n = nlay - k0;
        const uint32_t m = n >= SR_CH ? 0xffu : (1u << n) - 1u;
        return (wv >> (k0 & 31)) & m;
      };
      // the hand-off values of chunk j; layers above the top are padding
      auto chunk_vals = [&](int j, const uint4& qt, const uint4& qf, float (&tau)[SR_CH], float (&fr)[SR_CH]) {
        unpack8(qt, tau);
        unpack8(qf, fr);
        if (SR_CH * j + SR_CH > nlay) {
#pragma unroll
          for (int ii = 0; ii < SR_CH; ++ii)
            if (SR_CH * j + ii >= nlay) { tau[ii] = 0.0f; fr[ii] = 0.0f; }
        }
      };
      // ---- down sweep (RLM:3598-3673), layers top to bottom ----
      float radc = 0.0f, radt = 0.0f, fr0 = 0.0f;
      uint4 nt = act ? __ldg(hq + (size_t)(nch - 1) * 2 * NGPT) : zero4;
      uint4 nf = act ? __ldg(hq + (size_t)(nch - 1) * 2 * NGPT + NGPT) : zero4;
#pragma unroll 1
      for (int j = nch - 1; j >= 0; --j) {
        float tau[SR_CH], fr[SR_CH];
        chunk_vals(j, nt, nf, tau, fr);
        if (j > 0 && act) {   // the next chunk's loads overlap this chunk's work
          nt = __ldg(hq + (size_t)(j - 1) * 2 * NGPT);
          nf = __ldg(hq + (size_t)(j - 1) * 2 * NGPT + NGPT);
        }
        const uint32_t cb = chunk_bits(j);
        float aT[SR_CH], aC[SR_CH], stash[SR_CH];
        // the gas terms of the chunk's layers, independent of one another and
        // branch-free (both the Pade-free forms and the record, then a select)
        float trv[SR_CH], gsdv[SR_CH], odv[SR_CH];
        int itv[SR_CH];
#pragma unroll
        for (int ii = 0; ii < SR_CH; ++ii) {
          const float4 v = S.bf[SR_CH * j + ii][b];
          const float od = fmaxf(0.0f, secd * tau[ii]);
          const int it = tbl_index(od);
          const float2 e = __half22float2(tab[it]);
          const bool small = od <= 0.06f;
          const float atr = small ? od - 0.5f * od * od : e.x;
          const float fac = small ? float(kRec6) * od : e.y;
          trv[ii] = 1.0f - atr;
          gsdv[ii] = fr[ii] * (v.x + v.z * fac) * atr;
          stash[ii] = __uint_as_float(h2_bits(atr, fr[ii] * (v.x + v.y * fac) * atr * su_inv));
          odv[ii] = od;
          itv[ii] = small ? -1 : it;
        }
        // the recurrences, top layer of the chunk first; the total-sky terms
        // where the warp has a cloudy sub-column layer (a chunk without any
        // takes the clear-sky recurrence alone)
        if (!__any_sync(0xffffffffu, cb != 0u)) {
#pragma unroll
          for (int ii = SR_CH - 1; ii >= 0; --ii) {
            radc = radc * trv[ii] + gsdv[ii];
            radt = radt * trv[ii] + gsdv[ii];
            aT[ii] = radt;
            aC[ii] = radc;
          }
        } else {
#pragma unroll
        for (int ii = SR_CH - 1; ii >= 0; --ii) {
          const float tr = trv[ii], gsd = gsdv[ii];
          radc = radc * tr + gsd;
          const bool cl = (cb >> ii) & 1u;
          if (__any_sync(0xffffffffu, cl)) {
            float rt = radt * tr + gsd;
            if (cl) {
              const float4 v = S.bf[SR_CH * j + ii][b];
              float ef, atrtot, totfac;
              cloud_terms(odv[ii], itv[ii], v.w, tab, ef, atrtot, totfac);
              const float tsd = fr[ii] * (v.x + v.z * totfac) * atrtot;
              rt = radt * tr * ef + gsd + 1.0f * (tsd - gsd);
            }
            radt = rt;
          } else {
            radt = radt * tr + gsd;
          }
          aT[ii] = radt;
          aC[ii] = radc;
        }
        }
        umma::tmem_st8(tw + SR_CH * j, stash);
        if (j == 0) fr0 = fr[0];
        const float sT = warp_sum8(aT, lane), sC = warp_sum8(aC, lane);
        const int lvl = SR_CH * j + ((lane >> 2) & 7);
        if ((lane & 3) == 0 && lvl < nlay) {
          P[0 * (SR_NL + 1) + lvl] = sT;
          P[1 * (SR_NL + 1) + lvl] = sC;
        }
      }
      if (lane == 0) {   // no downward radiance at the top level
        P[0 * (SR_NL + 1) + nlay] = 0.0f;
        P[1 * (SR_NL + 1) + nlay] = 0.0f;
      }
      // ---- surface emission and reflection (RLM:3682-3691) ----
      const float rad0 = S.semis * fr0 * S.pk0[b];
      const float reflct = 1.0f - S.semis;
      float rutot = rad0 + reflct * radt, ruclr = rad0 + reflct * radc;
      {
        const float s0 = warp_sum_all(rutot), s1 = warp_sum_all(ruclr);
        if (lane == 0) {
          P[2 * (SR_NL + 1)] = s0;
          P[3 * (SR_NL + 1)] = s1;
        }
      }
      // ---- up sweep (RLM:3700-3730), layers bottom to top: the clear-sky terms
      // from tensor memory, the total-sky terms of cloudy sub-columns recomputed ----
      umma::tmem_wait_st();
      nt = act ? __ldg(hq) : zero4;
      nf = act ? __ldg(hq + NGPT) : zero4;
#pragma unroll 1
      for (int j = 0; j < nch; ++j) {
        float tau[SR_CH], fr[SR_CH], stash[SR_CH];
        chunk_vals(j, nt, nf, tau, fr);
        if (j + 1 < nch && act) {
          nt = __ldg(hq + (size_t)(j + 1) * 2 * NGPT);
          nf = __ldg(hq + (size_t)(j + 1) * 2 * NGPT + NGPT);
        }
        umma::tmem_ld8(tw + SR_CH * j, stash);
        const uint32_t cb = chunk_bits(j);
        float aT[SR_CH], aC[SR_CH];
        if (!__any_sync(0xffffffffu, cb != 0u)) {   // no cloudy sub-column layer in the chunk
#pragma unroll
          for (int ii = 0; ii < SR_CH; ++ii) {
            const float2 ag = __half22float2(*reinterpret_cast<const __half2*>(&stash[ii]));
            const float tr = 1.0f - ag.x, gsu = ag.y * su_scale;
            ruclr = ruclr * tr + gsu;
            rutot = rutot * tr + gsu;
            aT[ii] = rutot;
            aC[ii] = ruclr;
          }
        } else {
#pragma unroll
        for (int ii = 0; ii < SR_CH; ++ii) {
          const float2 ag = __half22float2(*reinterpret_cast<const __half2*>(&stash[ii]));
          const float tr = 1.0f - ag.x, gsu = ag.y * su_scale;
          ruclr = ruclr * tr + gsu;
          const bool cl = (cb >> ii) & 1u;   // clfm > eps (strict, RLM:3705): a cloudy sub-column
          if (__any_sync(0xffffffffu, cl)) {
            float rt = rutot * tr + gsu;
            if (cl) {
              const float4 v = S.bf[SR_CH * j + ii][b];
              const float od = fmaxf(0.0f, secd * tau[ii]);
              const int it = od <= 0.06f ? -1 : tbl_index(od);
              float ef, atrtot, totfac;
              cloud_terms(od, it, v.w, tab, ef, atrtot, totfac);
              const float tsu = fr[ii] * (v.x + v.y * totfac) * atrtot;
              rt = rutot * tr * ef + gsu + 1.0f * (tsu - gsu);
            }
            rutot = rt;
          } else {
            rutot = rutot * tr + gsu;
          }
          aT[ii] = rutot;
          aC[ii] = ruclr;
        }
        }
        const float sT = warp_sum8(aT, lane), sC = warp_sum8(aC, lane);
        const int lvl = SR_CH * j + 1 + ((lane >> 2) & 7);
        if ((lane & 3) == 0 && lvl <= nlay) {
          P[2 * (SR_NL + 1) + lvl] = sT;
          P[3 * (SR_NL + 1) + lvl] = sC;
        }
      }
    }
    sync.sync();

    // ---------------- fluxes and heating rates (RLM:3737-3770, 1228-1304) ----------------
    {
      const double flxfac = 0.5 * a.cs.fluxfac;   // wtdiff * fluxfac
      if (gt <= nlay) {
        const int l = gt;
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int w = 0; w < SR_WARPS; ++w) s4[q] += (double)S.part[w][q][l];
        const double td = s4[0] * flxfac, cd = s4[1] * flxfac, tu = s4[2] * flxfac, cu = s4[3] * flxfac;
        S.u.fn[0][l] = tu - td;
        S.u.fn[1][l] = cu - cd;
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
      sync.sync();
      if (gt < nlay) {
        const int k = gt;
        const int r = top ? nlay - 1 - k : k;
        const double rfdelp = a.cs.heatfac / IN(F_DELPIN, r);
        B.out[O_HLWC][i + ld * r] = (S.u.fn[0][k] - S.u.fn[0][k + 1]) * rfdelp;
        if (f.want_hlw0) B.out[O_HLW0][i + ld * r] = (S.u.fn[1][k] - S.u.fn[1][k + 1]) * rfdelp;
      }
      sync.sync();   // fn[] is read before the next column's prologue reuses its space
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) umma::tmem_dealloc(tbase, 512);
}

// ---------------------------------------------------------------------------
// Out-of-envelope layers: plain FP32 taumol (the FP32 path's gas optics) for
// the listed columns, written over the network's values in the hand-off.
constexpr int FB_V = 4;                        // 128 layer threads
constexpr size_t FB_NLP = 32 * FB_V;
constexpr size_t FB_SLOT_BYTES = (((2 * NGPT + 3 * NBANDS) * FB_NLP * sizeof(float) + kColRec * sizeof(double)) + 255) &
                                 ~(size_t)255;
constexpr int FB_GRID = 64;

struct FbArgs {
  const Block* blocks;
  int nblocks;
  Block b0;
  int c0;                   // first global column of the chunk
  Flags f;
  Tables<float> tab;
  Tables<double> tab64;
  const int* list;
  const int* count;
  unsigned int* flag;
  __half* hnd;
  unsigned char* slots;     // FB_SLOT_BYTES per CTA
};

__global__ void __launch_bounds__(32 * FB_V) lw_sg_fallback_kernel(FbArgs a) {
  extern __shared__ __align__(16) char fsm[];   // gas_smem_bytes<float>(FB_V)
  const GasWork<float, FB_V> W = GasWork<float, FB_V>::at(fsm);
  const int n = *a.count;
  const int t = threadIdx.x, nlay = a.f.nlay;
  float* slot = reinterpret_cast<float*>(a.slots + (size_t)blockIdx.x * FB_SLOT_BYTES);
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const int c = a.list[k];
    Scratch<float> sc;
    sc.tau = slot;
    sc.frac = slot + NGPT * FB_NLP;
    sc.band = slot + 2 * NGPT * FB_NLP;
    sc.col = reinterpret_cast<double*>(slot + (2 * NGPT + 3 * NBANDS) * FB_NLP);
    sc.c0 = c;
    sc.cap = 1;
    sc.ntot = c + 1;
    gas_column<float, FB_V, true>(0, t, CtaSync{}, W, a.blocks, a.nblocks, a.b0, a.f, a.tab, a.tab64, sc, nullptr,
                                  nullptr);
    __syncthreads();
    if (t < nlay) {
      // the network kernel's envelope test on the same features
      const Block& B = (a.nblocks == 1) ? a.b0 : a.blocks[find_block(a.blocks, a.nblocks, c)];
      const size_t o = (size_t)(c - B.col0) + (size_t)B.ld * (a.f.top_at_1 ? nlay - t - 1 : t);
      const double qv = B.in[F_QLYR][o];
      const double h2ovmr = fmax(0.0, qv * (kConAmd / kConAmw) / (1.0 - qv));
      const double o3vmr = fmax(0.0, B.in[F_OLYR][o] * (kConAmd / kConAmo3));
      float x[SG_NFEAT];
      layer_features(B.in[F_PLYR][o], B.in[F_TLYR][o], h2ovmr, o3vmr, B.in[F_CO2][o], B.in[F_CH4][o],
                     B.in[F_N2O][o], x);
      if (!in_envelope(x, a.f.sg_norm)) {
        const int nch = (nlay + SR_CH - 1) / SR_CH;
        __half* h = a.hnd + ((size_t)(c - a.c0) * nch + (t >> 3)) * SR_HCH + (t & 7);
        for (int g = 0; g < NGPT; ++g) {
          h[8 * g] = __float2half_rn(fminf(sc.tau[g * FB_NLP + t], 6.0e4f));
          h[8 * (NGPT + g)] = __float2half_rn(sc.frac[g * FB_NLP + t]);
        }
      }
    }
    if (t == 0) a.flag[c] = 0u;
    __syncthreads();
  }
}

// block of every global column
__global__ void lw_colmap_kernel(const Block* blocks, int nblocks, int* colmap) {
  const int lane = threadIdx.x & 31;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nblocks; b += (gridDim.x * blockDim.x) >> 5) {
    const int c0 = blocks[b].col0, n = blocks[b].npts;
    for (int j = lane; j < n; j += 32) colmap[c0 + j] = b;
  }
}

bool s_prepared = false;

// Work area layout (bytes, each part 256-aligned): colmap [ncols] int,
// flags [ncols] u32, count, list [chunk] int, fallback slots, packed network
// inputs [chunk] x kSgPackBytes, hand-off [chunk][nlay/8][280][8] half.
struct SgLayout {
  size_t colmap, flag, count, list, fb, pk, hnd, total;
  long chunk;
};
size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
SgLayout layout(int ncols, int nlay, int num_sms, size_t budget) {
  SgLayout L;
  L.colmap = 0;
  L.flag = L.colmap + al((size_t)ncols * sizeof(int));
  L.count = L.flag + al((size_t)ncols * sizeof(unsigned));
  L.list = L.count + 256;
  const size_t per_col = (size_t)((nlay + SR_CH - 1) / SR_CH) * SR_HCH * sizeof(__half) + kSgPackBytes;
  const size_t fb_bytes = al((size_t)FB_GRID * FB_SLOT_BYTES);
  const size_t fixed = L.list + al((size_t)ncols * sizeof(int)) + fb_bytes;
  long chunk = (long)ncols;
  if (budget > fixed + per_col) chunk = std::min<long>(chunk, (long)((budget - fixed) / per_col));
  else chunk = std::min<long>(chunk, 1);
  if (chunk < 1) chunk = 1;
  L.chunk = chunk;
  L.fb = L.list + al((size_t)chunk * sizeof(int));
  L.pk = L.fb + fb_bytes;
  L.hnd = L.pk + al((size_t)chunk * kSgPackBytes);
  L.total = L.hnd + al((size_t)chunk * (per_col - kSgPackBytes));
  return L;
}

}  // namespace

bool sg_path_applies(const Flags& f) {
  return f.surrogate && !f.gas_only && f.nlay >= 1 && f.nlay <= SR_NL - 1 && f.isubclw > 0 && !f.want_hlwb;
}

size_t sg_path_bytes(int ncols, int nlay, int num_sms, size_t budget) {
  return layout(ncols, nlay, num_sms, budget).total;
}

int sg_path_launches(int ncols, int nlay, int num_sms, size_t budget, int nblocks) {
  const SgLayout L = layout(ncols, nlay, num_sms, budget);
  const int nchunks = (int)((ncols + L.chunk - 1) / L.chunk);
  return (nblocks > 1 ? 1 : 0) + 4 * nchunks;
}

cudaError_t sg_path_prepare() {
  cudaError_t e = cudaFuncSetAttribute(lw_sg_rt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SR_SMEM);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(lw_sg_fallback_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gas_smem_bytes<float>(FB_V));
  if (e != cudaSuccess) return e;
  int occ = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, lw_sg_rt_kernel, SR_THREADS, SR_SMEM)) != cudaSuccess)
    return e;
  if (occ < 1) return cudaErrorLaunchOutOfResources;
  s_prepared = true;
  return cudaSuccess;
}

cudaError_t sg_path_launch(const Block* blocks, int nblocks, const Block& b0, int ncols, const Flags& f,
                           const Consts& cs, const Tables<float>& tab, const Tables<double>& tab64,
                           const uint32_t* bits, void* work, size_t work_bytes, size_t budget, int num_sms,
                           cudaStream_t st) {
  if (!s_prepared) return cudaErrorNotReady;
  const SgLayout L = layout(ncols, f.nlay, num_sms, budget);
  if (work_bytes < L.total || (reinterpret_cast<uintptr_t>(work) & 255) != 0) return cudaErrorMemoryAllocation;
  unsigned char* base = static_cast<unsigned char*>(work);
  int* colmap = reinterpret_cast<int*>(base + L.colmap);
  unsigned int* flag = reinterpret_cast<unsigned int*>(base + L.flag);
  int* count = reinterpret_cast<int*>(base + L.count);
  int* list = reinterpret_cast<int*>(base + L.list);
  unsigned char* fbs = base + L.fb;
  unsigned char* pk = base + L.pk;
  __half* hnd = reinterpret_cast<__half*>(base + L.hnd);
  cudaError_t e;
  if (nblocks > 1) {
    lw_colmap_kernel<<<std::max(1, std::min(num_sms * 4, (nblocks + 7) / 8)), 256, 0, st>>>(blocks, nblocks, colmap);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if ((e = cudaMemsetAsync(flag, 0, (size_t)ncols * sizeof(unsigned), st)) != cudaSuccess) return e;
  for (long c0 = 0; c0 < ncols; c0 += L.chunk) {
    const int nc = (int)std::min<long>(L.chunk, ncols - c0);
    if ((e = cudaMemsetAsync(count, 0, sizeof(int), st)) != cudaSuccess) return e;
    {
      NvtxRange r("learned gas optics (taumol network)");
      if ((e = mlp_h_launch(blocks, nblocks, b0, colmap, (int)c0, nc, f, hnd, flag, list, count, pk, num_sms,
                            st)) != cudaSuccess)
        return e;
    }
    FbArgs fa;
    fa.blocks = blocks;
    fa.nblocks = nblocks;
    fa.b0 = b0;
    fa.c0 = (int)c0;
    fa.f = f;
    fa.tab = tab;
    fa.tab64 = tab64;
    fa.list = list;
    fa.count = count;
    fa.flag = flag;
    fa.hnd = hnd;
    fa.slots = fbs;
    {
      NvtxRange r("taumol fallback (out of envelope)");
      lw_sg_fallback_kernel<<<FB_GRID, 32 * FB_V, gas_smem_bytes<float>(FB_V), st>>>(fa);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    SrArgs ra;
    ra.blocks = blocks;
    ra.nblocks = nblocks;
    ra.b0 = b0;
    ra.colmap = colmap;
    ra.c0 = (int)c0;
    ra.nc = nc;
    ra.f = f;
    ra.cs = cs;
    ra.trec = tab.trec;
    ra.kt64 = tab64.kt;
    ra.bits = bits;
    ra.hnd = hnd;
    const int grid = std::min(num_sms, (nc + SR_GROUPS - 1) / SR_GROUPS);
    {
      NvtxRange r("cldprop+rtrnmc");
      lw_sg_rt_kernel<<<grid, SR_THREADS, SR_SMEM, st>>>(ra);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

}  // namespace lw
