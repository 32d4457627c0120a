// lw_column.cuh -- fused RRTMG-LW column kernel (one CTA per column).
//
// Replaces the per-column body of rrtmg_lw_run (physics/Radiation/RRTMG/
// radlw_main.F90, RLM:782-1304): prologue (RLM:785-1050), cldprop band
// optics (RLM:1530-1799), setcoef (RLM:2151-2406), taumol (RLM:3836-6840)
// and rtrnmc (RLM:3420-3785).  McICA sub-columns come from lw_mcica.cu.
//
// Thread mapping (V = layers per lane, CTA = 32*V threads = V warps):
//   P0  thread t <-> layer t: prologue + setcoef in FP64 into shared memory.
//   per band b:
//     P1a thread t <-> layer t: band cloud/aerosol/Planck terms and the gas
//         optical depth + Planck fraction of every g-point of the band into
//         a shared [g][layer] tile (the per-layer set-up is done once).
//     P1b warp w <-> g-points w, w+V, ... of the band; lane l <-> layers
//         V*l .. V*l+V-1.  The two-stream down/up recurrences of rtrnmc are
//         affine maps per layer; each lane composes its V layers, a warp
//         shuffle scan composes across lanes, and each lane replays its
//         layers from the incoming radiance.  Flux sums stay in FP64
//         registers of the lane that owns the level.
//   epilogue: cross-warp flux sums, fluxes, heating rates (FP64), outputs.
#pragma once

#include "lw_bands.cuh"
#include "lw_common.cuh"

namespace lw {

// shared-memory SoA fields of the per-layer record
enum ScField {
  S_FAC00, S_FAC01, S_FAC10, S_FAC11, S_SELFFAC, S_SELFFRAC, S_FORFAC, S_FORFRAC, S_MINORFRAC,
  S_SCALEMINOR, S_SCALEMINORN2, S_COL1, S_COL2, S_COL3, S_COL4, S_COL5, S_COL6, S_COL7,
  S_COLDRY, S_COLBRD, S_WX1, S_WX2, S_WX3, S_WX4, S_PAVEL, S_TLYRFR, S_TLVLFR, S_CLDFRC,
  S_CLWP, S_RELW, S_CIWP, S_REIW, S_CDA1, S_CDA3, S_CDA4, S_DELP, N_SC
};

constexpr double kEps = 1.0e-6;                 // RLM:309
constexpr double kBpade = 1.0 / 0.278;          // RLM:312
constexpr double kStpfac = 296.0 / 1013.0;      // RLM:313
constexpr double kTblint = 10000.0;             // RLM:315 (ntbl)
constexpr double kRec6 = 0.166667;              // RLM:3548 (not 1/6)
constexpr double kConG = 9.80665, kConAvgd = 6.0221415e23;
constexpr double kConAmd = 28.9644, kConAmw = 18.0154, kConAmo3 = 47.9982;
constexpr double kAbsrain = 0.33e-3, kAbssnow0 = 1.5;   // radlw_datatb.f:941,944
static __device__ __constant__ double c_delwave[16] = {340., 150., 130., 70., 120., 160., 100., 100.,
                                                210., 90., 320., 280., 170., 130., 220., 650.};
static __device__ __constant__ double c_a0[16] = {1.66, 1.55, 1.58, 1.66, 1.54, 1.454, 1.89, 1.33,
                                           1.668, 1.66, 1.66, 1.66, 1.66, 1.66, 1.66, 1.66};
static __device__ __constant__ double c_a1[16] = {0.00, 0.25, 0.22, 0.00, 0.13, 0.446, -0.10, 0.40,
                                           -0.006, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00};
static __device__ __constant__ double c_a2[16] = {0.00, -12.0, -11.7, 0.00, -0.72, -0.243, 0.19, -0.062,
                                           0.414, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00};

template <typename R>
struct Smem {
  R* sc;            // [N_SC][NL]
  int* si;          // [2][NL]
  R* tf;            // [2][16][NL]: tau (gas + aerosol), Planck fraction
  R* pklay;         // [NL] pklay(b, 0..nlay) of the current band
  R* pklev;         // [NL]
  R* taucld;        // [NL] taucld(b, k)
  uint32_t* bits;   // [140][nw] McICA sub-column cloud flags
  double* red;      // [2*NL] scratch for sequential sums / net fluxes
  double* col;      // column scalars: [0..15] secdiff, [16] semiss, [17] pwvcm
  int* ci;          // column ints: [0] laytrop, [1] lcf1
};

// The [g][layer] tile is reused for the cross-warp flux sums of the
// epilogue (4 x V x NL doubles), so it is sized for the larger of the two.
template <typename R>
__host__ __device__ constexpr size_t tile_elems(int V) {
  size_t NL = 32 * (size_t)V;
  size_t tf = 2 * 16 * NL;
  size_t ep = (4 * (size_t)V * NL * sizeof(double) + sizeof(R) - 1) / sizeof(R);
  return tf > ep ? tf : ep;
}

template <typename R>
__host__ __device__ constexpr size_t smem_bytes(int V) {
  size_t NL = 32 * (size_t)V;
  return sizeof(R) * (N_SC * NL + tile_elems<R>(V) + 3 * NL) + sizeof(int) * 2 * NL +
         sizeof(uint32_t) * 140 * V + sizeof(double) * (2 * NL + 32) + sizeof(int) * 8 + 64;
}

template <typename R>
__device__ __forceinline__ Smem<R> carve(char* base, int V) {
  const int NL = 32 * V;
  Smem<R> s;
  double* d = reinterpret_cast<double*>(base);
  s.red = d;             d += 2 * NL;
  s.col = d;             d += 32;
  R* r = reinterpret_cast<R*>(d);
  s.sc = r;              r += N_SC * NL;
  s.tf = r;              r += tile_elems<R>(V);
  s.pklay = r;           r += NL;
  s.pklev = r;           r += NL;
  s.taucld = r;          r += NL;
  int* ip = reinterpret_cast<int*>(r);
  s.si = ip;             ip += 2 * NL;
  s.ci = ip;             ip += 8;
  s.bits = reinterpret_cast<uint32_t*>(ip);
  return s;
}

// ---- warp shuffles of doubles/floats --------------------------------------
template <typename R> __device__ __forceinline__ R shdn(R v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
template <typename R> __device__ __forceinline__ R shup(R v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <typename R> __device__ __forceinline__ R shidx(R v, int s) { return __shfl_sync(0xffffffffu, v, s); }

// Per-layer two-stream coefficients of one g-point (RLM:3598-3660).
template <typename R>
struct LayRT {
  R tr, gsd, gsu;       // clear-sky transmittance and layer sources
  R ef, tsd, tsu;       // cloudy: efclrfr and total-sky sources
};

template <typename R>
__device__ __forceinline__ void layer_rt(R tau, R frac, R secd, R blay, R plevu, R plevd, bool cloudy, R tcld,
                                         const Tables<R>& tab, LayRT<R>& o) {
  const R one = R(1);
  R odepth = fmax(R(0), secd * tau);
  R atrgas, trng, gasfac;
  if (odepth <= R(0.06)) {
    atrgas = odepth - R(0.5) * odepth * odepth;
    trng = one - atrgas;
    gasfac = R(kRec6) * odepth;
  } else {
    R tblind = odepth / (R(kBpade) + odepth);
    int itgas = min(NTBL, max(0, (int)(R(kTblint) * tblind + R(0.5))));
    trng = ldg(tab.exp_tbl + itgas);
    atrgas = one - trng;
    gasfac = ldg(tab.tfn_tbl + itgas);
    odepth = ldg(tab.tau_tbl + itgas);
  }
  R dplnku = plevu - blay;
  R dplnkd = plevd - blay;
  R bbdgas = frac * (blay + dplnkd * gasfac);
  R bbugas = frac * (blay + dplnku * gasfac);
  o.gsd = bbdgas * atrgas;
  o.gsu = bbugas * atrgas;
  o.tr = trng;
  if (cloudy) {
    R odcld = secd * tcld;
    o.ef = one - (one - exp(-odcld)) * one;   // clfm = 1 for a McICA cloudy sub-column
    R odtot = odepth + odcld;
    R totfac, atrtot;
    if (odtot < R(0.06)) {
      totfac = R(kRec6) * odtot;
      atrtot = odtot - R(0.5) * odtot * odtot;
    } else {
      R tblind = odtot / (R(kBpade) + odtot);
      int ittot = min(NTBL, max(0, (int)(R(kTblint) * tblind + R(0.5))));
      totfac = ldg(tab.tfn_tbl + ittot);
      atrtot = one - ldg(tab.exp_tbl + ittot);
    }
    R bbdtot = frac * (blay + dplnkd * totfac);
    R bbutot = frac * (blay + dplnku * totfac);
    o.tsd = bbdtot * atrtot;
    o.tsu = bbutot * atrtot;
  }
}

// cldprop band optics of one layer and band (RLM:1589-1799), FP64.
__device__ __forceinline__ double band_taucld(int b, const Flags& f, const double* kt, double cf, double clwp,
                                              double relw, double ciwp, double reiw, double cda1, double cda3,
                                              double cda4) {
  if (!(cf > 2.2250738585072014e-308)) return 0.0;   // cfrac(k) > cldmin = tiny
  if (f.ilwcliq <= 0) return cda1;                    // diagnostic cloud optical depth
  double tauran = kAbsrain * cda1;
  double tausnw = (cda3 > 0.0 && cda4 > 10.0) ? kAbssnow0 * 1.05756 * cda3 / cda4 : 0.0;
  double tauliq = 0.0, tauice = 0.0;
  if (clwp > 0.0 && f.ilwcliq == 1) {
    double factor = relw - 1.5;
    int index = max(1, min(57, (int)factor));
    double fint = factor - (double)index;
    double a = __ldg(kt + lwtab::absliq1 + (index - 1) + 58 * b);
    double c = __ldg(kt + lwtab::absliq1 + index + 58 * b);
    tauliq = fmax(0.0, clwp * (a + fint * (c - a)));
  }
  if (ciwp > 0.0) {
    if (f.ilwcice == 1) {
      double refice = fmin(130.0, fmax(13.0, reiw));
      int ia = (int)__ldg(kt + lwtab::ipat + b);
      tauice = fmax(0.0, ciwp * (__ldg(kt + lwtab::absice1 + 2 * (ia - 1)) +
                                 __ldg(kt + lwtab::absice1 + 1 + 2 * (ia - 1)) / refice));
    } else if (f.ilwcice == 2) {
      double factor = (reiw - 2.0) / 3.0;
      int index = max(1, min(42, (int)factor));
      double fint = factor - (double)index;
      double a = __ldg(kt + lwtab::absice2 + (index - 1) + 43 * b);
      double c = __ldg(kt + lwtab::absice2 + index + 43 * b);
      tauice = fmax(0.0, ciwp * (a + fint * (c - a)));
    } else if (f.ilwcice == 3) {
      double dgeice = fmax(5.0, 1.0315 * reiw);
      double factor = (dgeice - 2.0) / 3.0;
      int index = max(1, min(45, (int)factor));
      double fint = factor - (double)index;
      double a = __ldg(kt + lwtab::absice3 + (index - 1) + 46 * b);
      double c = __ldg(kt + lwtab::absice3 + index + 46 * b);
      tauice = fmax(0.0, ciwp * (a + fint * (c - a)));
    }
  }
  return tauice + tauliq + tauran + tausnw;
}

// Planck integral of band b at temperature index/fraction (RLM:2251-2283)
__device__ __forceinline__ double planck_int(const double* kt, int b, int ind, double frac) {
  double p0 = __ldg(kt + lwtab::totplnk + (ind - 1) + 181 * b);
  double p1 = __ldg(kt + lwtab::totplnk + ind + 181 * b);
  return c_delwave[b] * (p0 + frac * (p1 - p0));
}

template <typename R>
__device__ __forceinline__ Lay<R> load_lay(const Smem<R>& s, int NL, int t) {
  Lay<R> L;
  const R* sc = s.sc;
  L.fac00 = sc[S_FAC00 * NL + t]; L.fac01 = sc[S_FAC01 * NL + t];
  L.fac10 = sc[S_FAC10 * NL + t]; L.fac11 = sc[S_FAC11 * NL + t];
  L.selffac = sc[S_SELFFAC * NL + t]; L.selffrac = sc[S_SELFFRAC * NL + t];
  L.forfac = sc[S_FORFAC * NL + t]; L.forfrac = sc[S_FORFRAC * NL + t];
  L.minorfrac = sc[S_MINORFRAC * NL + t];
  L.scaleminor = sc[S_SCALEMINOR * NL + t]; L.scaleminorn2 = sc[S_SCALEMINORN2 * NL + t];
#pragma unroll
  for (int m = 0; m < 7; ++m) L.col[m] = sc[(S_COL1 + m) * NL + t];
  L.coldry = sc[S_COLDRY * NL + t]; L.colbrd = sc[S_COLBRD * NL + t];
#pragma unroll
  for (int m = 0; m < 4; ++m) L.wx[m] = sc[(S_WX1 + m) * NL + t];
  L.pavel = sc[S_PAVEL * NL + t];
  int i0 = s.si[t];
  L.jp = i0 & 0xff; L.jt = (i0 >> 8) & 0xf; L.jt1 = (i0 >> 12) & 0xf;
  L.indself = (i0 >> 16) & 0xf; L.indfor = (i0 >> 20) & 0xf; L.indminor = (i0 >> 24) & 0x1f;
  L.lower = (s.si[NL + t] >> 16) & 1;
  return L;
}

// ===========================================================================
template <typename R, int V, bool HLWB>
__global__ void __launch_bounds__(32 * V)
lw_column_kernel(const Block* __restrict__ blocks, int nblocks, const Block b0, int ncols, Flags f, Consts cs,
                 Tables<R> tab, Tables<double> tab64, const uint32_t* __restrict__ bits_g,
                 double* __restrict__ gas_taug, double* __restrict__ gas_fracs) {
  extern __shared__ __align__(16) char smem_raw[];
  constexpr int NL = 32 * V;
  const int nlay = f.nlay, nlp1 = nlay + 1;
  const int nw = (nlay + 31) >> 5;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  Smem<R> s = carve<R>(smem_raw, V);
  const KT<R> kt{tab.kt};
  const double* kt64 = tab64.kt;

  for (int c = blockIdx.x; c < ncols; c += gridDim.x) {
    __syncthreads();   // shared memory of the previous column is free
    const Block& B = (nblocks == 1) ? b0 : blocks[find_block(blocks, nblocks, c)];
    const int i = c - B.col0;            // column within its physics block
    const size_t ld = (size_t)B.ld;
    const bool top = f.top_at_1 != 0;
    auto IN = [&](int fld, int row) -> double { return B.in[fld][i + ld * row]; };

    // ------------------------------ P0 ----------------------------------
    // driver prologue (RLM:785-1050) and setcoef (RLM:2151-2406), FP64
    bool lowerk = false, cldk = false;
    double coldry = 0.0, col1 = 0.0;
    if (t < nlay) {
      const int kref = t + 1;                         // internal layer, surface first
      const int r = top ? nlp1 - kref - 1 : t;        // 0-based input row of layer
      const int rl = top ? nlp1 - kref - 1 : t + 1;   // 0-based input row of its top level
      double pavel = IN(F_PLYR, r), delp = IN(F_DELPIN, r), tavel = IN(F_TLYR, r), tz = IN(F_TLVL, rl);
      double q = IN(F_QLYR, r);
      const double amdw = kConAmd / kConAmw, amdo3 = kConAmd / kConAmo3;
      double h2ovmr = fmax(0.0, q * amdw / (1.0 - q));
      double o3vmr = fmax(0.0, IN(F_OLYR, r) * amdo3);
      double tem0 = (1.0 - h2ovmr) * kConAmd + h2ovmr * kConAmw;
      const double tem1c = 100.0 * kConG, tem2c = 1.0e-20 * 1.0e3 * kConAvgd;
      coldry = tem2c * delp / (tem1c * tem0 * (1.0 + h2ovmr));
      double temcol = 1.0e-12 * coldry;
      double colv[7], wxv[4];
      colv[0] = fmax(0.0, coldry * h2ovmr);
      colv[1] = fmax(temcol, coldry * IN(F_CO2, r));
      colv[2] = fmax(temcol, coldry * o3vmr);
      if (f.inc_minor_gas) {
        colv[3] = fmax(temcol, coldry * IN(F_N2O, r));
        colv[4] = fmax(temcol, coldry * IN(F_CH4, r));
        colv[5] = fmax(0.0, coldry * IN(F_O2, r));
        colv[6] = fmax(0.0, coldry * IN(F_CO, r));
        wxv[0] = fmax(0.0, coldry * IN(F_CCL4, r));
        wxv[1] = fmax(0.0, coldry * IN(F_CFC11, r));
        wxv[2] = fmax(0.0, coldry * IN(F_CFC12, r));
        wxv[3] = fmax(0.0, coldry * IN(F_CFC22, r));
      } else {
        colv[3] = colv[4] = colv[5] = colv[6] = 0.0;
        wxv[0] = wxv[1] = wxv[2] = wxv[3] = 0.0;
      }
      col1 = colv[0];
      double summol = 0.0;
      for (int m = 1; m < 7; ++m) summol = summol + colv[m];
      double colbrd = coldry - summol;

      // setcoef, layer part
      int indlay = min(180, max(1, (int)(tavel - 159.0)));
      double tlyrfr = tavel - (int)tavel;
      int indlev = min(180, max(1, (int)(tz - 159.0)));
      double tlvlfr = tz - (int)tz;
      double plog = log(pavel);
      int jp = max(1, min(58, (int)(36.0 - 5.0 * (plog + 0.04))));
      int jp1 = jp + 1;
      double fp = fmax(0.0, fmin(1.0, 5.0 * (__ldg(kt64 + lwtab::preflog + jp - 1) - plog)));
      double tem1 = (tavel - __ldg(kt64 + lwtab::tref + jp - 1)) / 15.0;
      double tem2 = (tavel - __ldg(kt64 + lwtab::tref + jp1 - 1)) / 15.0;
      int jt = max(1, min(4, (int)(3.0 + tem1)));
      int jt1 = max(1, min(4, (int)(3.0 + tem2)));
      double ft = fmax(-0.5, fmin(1.5, tem1 - (double)(jt - 3)));
      double ft1 = fmax(-0.5, fmin(1.5, tem2 - (double)(jt1 - 3)));
      tem1 = 1.0 - fp;
      double fac10 = tem1 * ft, fac00 = tem1 * (1.0 - ft), fac11 = fp * ft1, fac01 = fp * (1.0 - ft1);
      double forfac = pavel * kStpfac / (tavel * (1.0 + h2ovmr));
      double selffac = h2ovmr * forfac;
      double scaleminor = pavel / tavel;
      double scaleminorn2 = (pavel / tavel) * (colbrd / (coldry + colv[0]));
      tem1 = (tavel - 180.8) / 7.2;
      int indminor = min(18, max(1, (int)tem1));
      double minorfrac = tem1 - (double)indminor;
      int indfor, indself;
      double forfrac, selffrac;
      lowerk = plog > 4.56;
      if (lowerk) {
        tem1 = (332.0 - tavel) / 36.0;
        indfor = min(2, max(1, (int)tem1));
        forfrac = tem1 - (double)indfor;
        tem1 = (tavel - 188.0) / 7.2;
        indself = min(9, max(1, (int)tem1 - 7));
        selffrac = tem1 - (double)(indself + 7);
      } else {
        tem1 = (tavel - 188.0) / 36.0;
        indfor = 3;
        forfrac = tem1 - 1.0;
        indself = 0;
        selffrac = 0.0;
      }
      selffac = colv[0] * selffac;
      forfac = colv[0] * forfac;

      R* sc = s.sc;
      sc[S_FAC00 * NL + t] = R(fac00); sc[S_FAC01 * NL + t] = R(fac01);
      sc[S_FAC10 * NL + t] = R(fac10); sc[S_FAC11 * NL + t] = R(fac11);
      sc[S_SELFFAC * NL + t] = R(selffac); sc[S_SELFFRAC * NL + t] = R(selffrac);
      sc[S_FORFAC * NL + t] = R(forfac); sc[S_FORFRAC * NL + t] = R(forfrac);
      sc[S_MINORFRAC * NL + t] = R(minorfrac);
      sc[S_SCALEMINOR * NL + t] = R(scaleminor); sc[S_SCALEMINORN2 * NL + t] = R(scaleminorn2);
      for (int m = 0; m < 7; ++m) sc[(S_COL1 + m) * NL + t] = R(colv[m]);
      sc[S_COLDRY * NL + t] = R(coldry); sc[S_COLBRD * NL + t] = R(colbrd);
      for (int m = 0; m < 4; ++m) sc[(S_WX1 + m) * NL + t] = R(wxv[m]);
      sc[S_PAVEL * NL + t] = R(pavel);
      sc[S_TLYRFR * NL + t] = R(tlyrfr); sc[S_TLVLFR * NL + t] = R(tlvlfr);
      sc[S_DELP * NL + t] = R(delp);
      double cf = IN(F_CLDCF, r);
      cldk = cf > kEps;
      sc[S_CLDFRC * NL + t] = R(cf);
      if (f.ilwcliq > 0) {
        sc[S_CLWP * NL + t] = R(IN(F_LWP, r)); sc[S_RELW * NL + t] = R(IN(F_RELIQ, r));
        sc[S_CIWP * NL + t] = R(IN(F_IWP, r)); sc[S_REIW * NL + t] = R(IN(F_REICE, r));
        sc[S_CDA1 * NL + t] = R(IN(F_RWP, r)); sc[S_CDA3 * NL + t] = R(IN(F_SWP, r));
        sc[S_CDA4 * NL + t] = R(IN(F_RESNOW, r));
      } else {
        sc[S_CDA1 * NL + t] = R(IN(F_CLDOD, r));
      }
      s.si[t] = jp | (jt << 8) | (jt1 << 12) | (indself << 16) | (indfor << 20) | (indminor << 24);
      s.si[NL + t] = indlay | (indlev << 8) | ((lowerk ? 1 : 0) << 16);
      s.red[t] = coldry;
      s.red[NL + t] = col1;
    }
    const int laytrop = __syncthreads_count(lowerk);
    const int lcf1 = __syncthreads_or(cldk);
    if (t == 0) {
      // precipitable water (RLM:910-919 / 1012-1019): sequential, reference order
      double tem1 = 0.0, tem2 = 0.0;
      for (int k = 0; k < nlay; ++k) {
        tem1 = tem1 + s.red[k] + s.red[NL + k];
        tem2 = tem2 + s.red[NL + k];
      }
      const double amdw = kConAmd / kConAmw;
      double tem0 = 10.0 * tem2 / (amdw * tem1 * kConG);
      double psfc = top ? IN(F_PLVL, nlay) : IN(F_PLVL, 0);
      s.col[17] = tem0 * psfc;
      double sfe = B.in[F_SFEMIS][i];
      s.col[16] = (sfe > kEps && sfe <= 1.0) ? sfe : 1.0;
      // surface temperature indices (RLM:2251-2262): stemp and tz(0)
      double stemp = B.in[F_SFGTMP][i];
      double tz0 = top ? IN(F_TLVL, nlay) : IN(F_TLVL, 0);
      s.col[18] = stemp - (int)stemp;
      s.col[19] = tz0 - (int)tz0;
      s.ci[2] = min(180, max(1, (int)(stemp - 159.0)));
      s.ci[3] = min(180, max(1, (int)(tz0 - 159.0)));
    }
    // McICA sub-column flags of this column
    const bool mc = lcf1 && f.isubclw > 0 && !f.gas_only;   // gas-only launches have no McICA flags
    if (mc) {
      const uint32_t* src = bits_g + (size_t)c * NGPT * nw;
      for (int w = t; w < NGPT * nw; w += 32 * V) s.bits[w] = src[w];
    }
    __syncthreads();
    if (t < NBANDS) {   // diffusivity angle (RLM:1041-1050)
      double pwvcm = s.col[17];
      s.col[t] = (t == 0 || t == 3 || t == 9)
                     ? 1.66
                     : fmin(1.80, fmax(1.50, c_a0[t] + c_a1[t] * exp(c_a2[t] * pwvcm)));
    }
    // (visible to all after the first band barrier)

    double acc_tu[V], acc_td[V], acc_cu[V], acc_cd[V];
    double bnd_tu[HLWB ? V : 1], bnd_td[HLWB ? V : 1];
#pragma unroll
    for (int j = 0; j < V; ++j) acc_tu[j] = acc_td[j] = acc_cu[j] = acc_cd[j] = 0.0;

    // ------------------------------ bands --------------------------------
    for (int b = 0; b < NBANDS; ++b) {
      const int ng = ng_of(b), ns = ns_of(b);
      // P1a: thread <-> layer
      if (t < nlay) {
        const int r = top ? nlp1 - (t + 1) - 1 : t;
        int i1 = s.si[NL + t];
        int indlay = i1 & 0xff, indlev = (i1 >> 8) & 0xff;
        s.pklay[t + 1] = R(planck_int(kt64, b, indlay, (double)s.sc[S_TLYRFR * NL + t]));
        s.pklev[t + 1] = R(planck_int(kt64, b, indlev, (double)s.sc[S_TLVLFR * NL + t]));
        double tcld = 0.0;
        if (lcf1)
          tcld = band_taucld(b, f, kt64, (double)s.sc[S_CLDFRC * NL + t], (double)s.sc[S_CLWP * NL + t],
                             (double)s.sc[S_RELW * NL + t], (double)s.sc[S_CIWP * NL + t],
                             (double)s.sc[S_REIW * NL + t], (double)s.sc[S_CDA1 * NL + t],
                             (double)s.sc[S_CDA3 * NL + t], (double)s.sc[S_CDA4 * NL + t]);
        s.taucld[t] = R(tcld);
        if (b == 6 && !f.gas_only) B.out[O_CLDTAU][i + ld * r] = lcf1 ? tcld : 0.0;   // band 7 (RLM:1087-1097)
        const size_t ab = i + ld * ((size_t)r + (size_t)nlay * b);
        R tauaer = R(B.in[F_AERAOD][ab] * (1.0 - B.in[F_AERSSA][ab]));
        Lay<R> L = load_lay(s, NL, t);
        L.lower = t < laytrop;   // taumol splits at the count laytrop (RLM:2344-2346)
        // For a pressure profile that is not monotonic the count-based split
        // can send a layer to the branch of the other atmosphere, where the
        // reference indexes its tables out of bounds; keep indices in range.
        if (L.lower) { L.jp = min(L.jp, 12); L.indself = max(L.indself, 1); }
        else L.jp = max(L.jp, 13);
        R* tft = s.tf + t;
        R* tff = s.tf + 16 * NL + t;
        const size_t go = ((size_t)c * nlay + t) * NGPT + ns;
        band_gas_optics<R>(b, kt, L, [&](int g0, R tau, R frac) {
          tft[g0 * NL] = tau + tauaer;
          tff[g0 * NL] = frac;
          if (f.gas_only) {
            gas_taug[go + g0] = (double)tau;
            gas_fracs[go + g0] = (double)frac;
          }
        });
      }
      if (t == 0) {
        s.pklay[0] = R(planck_int(kt64, b, s.ci[2], s.col[18]));
        s.pklev[0] = R(planck_int(kt64, b, s.ci[3], s.col[19]));
      }
      __syncthreads();
      if (f.gas_only) { __syncthreads(); continue; }

      // P1b: warp <-> g-point, lane <-> V layers
      const R secd = R(s.col[b]);
      const R semis = R(s.col[16]);
#pragma unroll
      for (int j = 0; j < (HLWB ? V : 1); ++j) { bnd_tu[j] = 0.0; bnd_td[j] = 0.0; }
      for (int gi = warp; gi < ng; gi += V) {
        const int g = ns + gi;
        const int k0 = V * lane;
        uint32_t cbits = 0;
        if (mc && k0 < nlay) {
          // flags of layers k0..k0+V-1, none beyond nlay
          cbits = (s.bits[g * nw + (k0 >> 5)] >> (k0 & 31)) & ((1u << V) - 1u);
          if (nlay - k0 < V) cbits &= (1u << (nlay - k0)) - 1u;
        }
        LayRT<R> rt[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
          const int k = k0 + j;
          if (k < nlay) {
            layer_rt<R>(s.tf[gi * NL + k], s.tf[16 * NL + gi * NL + k], secd, s.pklay[k + 1], s.pklev[k + 1],
                        s.pklev[k], (cbits >> j) & 1u, s.taucld[k], tab, rt[j]);
          } else {
            rt[j].tr = R(1); rt[j].gsd = R(0); rt[j].gsu = R(0);
          }
        }
        const bool any_cloud = __any_sync(0xffffffffu, cbits != 0);
        // ---- down sweep: local composition, suffix scan, replay ----
        R Ac = R(1), Bc = R(0), At = R(1), Bt = R(0);
#pragma unroll
        for (int j = V - 1; j >= 0; --j) {
          Ac = rt[j].tr * Ac; Bc = rt[j].tr * Bc + rt[j].gsd;
          if ((cbits >> j) & 1u) {
            R a = rt[j].tr * rt[j].ef;
            At = a * At; Bt = a * Bt + (rt[j].gsd + (rt[j].tsd - rt[j].gsd));
          } else {
            At = rt[j].tr * At; Bt = rt[j].tr * Bt + rt[j].gsd;
          }
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          R ac = shdn(Ac, d), bc = shdn(Bc, d);
          R at = any_cloud ? shdn(At, d) : R(0), bt = any_cloud ? shdn(Bt, d) : R(0);
          if (lane + d < 32) {
            Bc = Ac * bc + Bc; Ac = Ac * ac;
            if (any_cloud) { Bt = At * bt + Bt; At = At * at; }
          }
        }
        R xc = shdn(Bc, 1), xt = any_cloud ? shdn(Bt, 1) : R(0);
        if (lane == 31) { xc = R(0); xt = R(0); }
        if (!any_cloud) xt = xc;
        R dn_c[V], dn_t[V];
#pragma unroll
        for (int j = V - 1; j >= 0; --j) {
          xc = xc * rt[j].tr + rt[j].gsd;
          if ((cbits >> j) & 1u) xt = xt * rt[j].tr * rt[j].ef + rt[j].gsd + R(1) * (rt[j].tsd - rt[j].gsd);
          else xt = xt * rt[j].tr + rt[j].gsd;
          dn_c[j] = xc; dn_t[j] = xt;
        }
        // surface emission and reflection (RLM:3682-3691)
        const R rd_c0 = shidx(dn_c[0], 0), rd_t0 = shidx(dn_t[0], 0);
        const R rad0 = semis * s.tf[16 * NL + gi * NL + 0] * s.pklay[0];
        const R reflct = R(1) - semis;
        const R r0c = rad0 + reflct * rd_c0, r0t = rad0 + reflct * rd_t0;
        // ---- up sweep: local composition, prefix scan, replay ----
        Ac = R(1); Bc = R(0); At = R(1); Bt = R(0);
#pragma unroll
        for (int j = 0; j < V; ++j) {
          Ac = rt[j].tr * Ac; Bc = rt[j].tr * Bc + rt[j].gsu;
          if ((cbits >> j) & 1u) {
            R a = rt[j].tr * rt[j].ef;
            At = a * At; Bt = a * Bt + (rt[j].gsu + (rt[j].tsu - rt[j].gsu));
          } else {
            At = rt[j].tr * At; Bt = rt[j].tr * Bt + rt[j].gsu;
          }
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          R ac = shup(Ac, d), bc = shup(Bc, d);
          R at = any_cloud ? shup(At, d) : R(0), bt = any_cloud ? shup(Bt, d) : R(0);
          if (lane >= d) {
            Bc = Ac * bc + Bc; Ac = Ac * ac;
            if (any_cloud) { Bt = At * bt + Bt; At = At * at; }
          }
        }
        R pac = shup(Ac, 1), pbc = shup(Bc, 1);
        R pat = any_cloud ? shup(At, 1) : R(0), pbt = any_cloud ? shup(Bt, 1) : R(0);
        if (lane == 0) { pac = R(1); pbc = R(0); pat = R(1); pbt = R(0); }
        xc = (lane == 0) ? r0c : pac * r0c + pbc;
        xt = any_cloud ? ((lane == 0) ? r0t : pat * r0t + pbt) : R(0);
        R up_c[V], up_t[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
          up_c[j] = xc;
          up_t[j] = any_cloud ? xt : xc;
          xc = xc * rt[j].tr + rt[j].gsu;
          if (any_cloud) {
            if ((cbits >> j) & 1u) xt = xt * rt[j].tr * rt[j].ef + rt[j].gsu + R(1) * (rt[j].tsu - rt[j].gsu);
            else xt = xt * rt[j].tr + rt[j].gsu;
          }
        }
#pragma unroll
        for (int j = 0; j < V; ++j) {
          acc_cd[j] += (double)dn_c[j];
          acc_td[j] += (double)dn_t[j];
          acc_cu[j] += (double)up_c[j];
          acc_tu[j] += (double)up_t[j];
          if constexpr (HLWB) { bnd_td[j] += (double)dn_t[j]; bnd_tu[j] += (double)up_t[j]; }
        }
      }
      __syncthreads();   // tile free for the next band
      if constexpr (HLWB) {
        // spectral band heating rate (RLM:3772-3780)
        double* e = reinterpret_cast<double*>(s.tf);
#pragma unroll
        for (int j = 0; j < V; ++j) {
          e[(warp * 2 + 0) * NL + V * lane + j] = bnd_tu[j];
          e[(warp * 2 + 1) * NL + V * lane + j] = bnd_td[j];
        }
        __syncthreads();
        const double flxfac = 0.5 * cs.fluxfac;
        if (t <= nlay) {
          double u = 0.0, d = 0.0;
          for (int w = 0; w < V; ++w) { u += e[(w * 2) * NL + t]; d += e[(w * 2 + 1) * NL + t]; }
          s.red[t] = (u - d) * flxfac;
        }
        __syncthreads();
        if (t < nlay) {
          const int r = top ? nlp1 - (t + 1) - 1 : t;
          double rfdelp = cs.heatfac / (double)s.sc[S_DELP * NL + t];
          B.out[O_HLWB][i + ld * ((size_t)r + (size_t)nlay * b)] = (s.red[t] - s.red[t + 1]) * rfdelp;
        }
        __syncthreads();
      }
    }
    if (f.gas_only) continue;

    // ------------------------------ epilogue -----------------------------
    double* e = reinterpret_cast<double*>(s.tf);   // [V warps][4][NL]
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int lv = V * lane + j;
      e[(warp * 4 + 0) * NL + lv] = acc_tu[j];
      e[(warp * 4 + 1) * NL + lv] = acc_td[j];
      e[(warp * 4 + 2) * NL + lv] = acc_cu[j];
      e[(warp * 4 + 3) * NL + lv] = acc_cd[j];
    }
    __syncthreads();
    const double flxfac = 0.5 * cs.fluxfac;   // wtdiff * fluxfac
    double tu = 0, td = 0, cu = 0, cd = 0;
    if (t <= nlay) {
      for (int w = 0; w < V; ++w) {
        tu += e[(w * 4 + 0) * NL + t]; td += e[(w * 4 + 1) * NL + t];
        cu += e[(w * 4 + 2) * NL + t]; cd += e[(w * 4 + 3) * NL + t];
      }
      tu = tu * flxfac; td = td * flxfac; cu = cu * flxfac; cd = cd * flxfac;
      s.red[t] = tu - td;            // fnet
      s.red[NL + t] = cu - cd;       // fnetc
      if (t == nlay) {
        B.out[O_TOPFLX][2 * i + 0] = tu;
        B.out[O_TOPFLX][2 * i + 1] = cu;
      }
      if (t == 0) {
        B.out[O_SFCFLX][4 * i + 0] = tu;
        B.out[O_SFCFLX][4 * i + 1] = cu;
        B.out[O_SFCFLX][4 * i + 2] = td;
        B.out[O_SFCFLX][4 * i + 3] = cd;
      }
      if (f.want_flxprf) {
        const int rl = top ? nlp1 - t - 1 : t;
        double* p = B.out[O_FLXPRF] + 4 * (i + ld * (size_t)rl);
        p[0] = tu; p[1] = td; p[2] = cu; p[3] = cd;
      }
    }
    __syncthreads();
    if (t < nlay) {   // heating rates (RLM:3754-3770)
      const int r = top ? nlp1 - (t + 1) - 1 : t;
      double rfdelp = cs.heatfac / (double)s.sc[S_DELP * NL + t];
      B.out[O_HLWC][i + ld * r] = (s.red[t] - s.red[t + 1]) * rfdelp;
      if (f.want_hlw0) B.out[O_HLW0][i + ld * r] = (s.red[NL + t] - s.red[NL + t + 1]) * rfdelp;
    }
  }
}

}  // namespace lw
