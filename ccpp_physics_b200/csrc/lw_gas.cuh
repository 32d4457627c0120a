// lw_gas.cuh -- kernel A of the RRTMG-LW path: per-layer column state,
// setcoef and the gas optics of all 140 g-points.
//
// Replaces, per column, the driver prologue of rrtmg_lw_run
// (physics/Radiation/RRTMG/radlw_main.F90, RLM:785-1050), the band cloud
// optics of cldprop (RLM:1589-1799), setcoef (RLM:2151-2406) and taumol
// (RLM:3836-6840).  One CTA owns one column at a time, one thread one layer;
// the setcoef state of the layer stays in that thread's registers and the 16
// bands are walked in order, so every table gather of a band happens while
// the band's coefficients are hot in L1/L2.
//
// Output (device scratch, read by kernel B in lw_rt.cuh), per column c of the
// chunk and layer k (0-based, surface first), NLP = 32*V >= nlay+1:
//   tau  [c][g][NLP]      gas + aerosol optical depth  (taumol tautot)
//   frac [c][g][NLP]      Planck fraction              (taumol fracs)
//   band [c][0][b][NLP]   pklay(b, k+1)
//        [c][1][b][NLP]   pklev(b, k)      k = 0..nlay
//        [c][2][b][NLP]   taucld(b, k+1)
//   col  [c][48]          secdiff(16), pklay(b,0)(16), semiss, lcf1
#pragma once

#include "lw_bands.cuh"
#include "lw_common.cuh"
#include "lw_features.cuh"

namespace lw {

constexpr double kEps = 1.0e-6;                 // RLM:309
constexpr double kBpade = 1.0 / 0.278;          // RLM:312
constexpr double kStpfac = 296.0 / 1013.0;      // RLM:313
constexpr double kTblint = 10000.0;             // RLM:315 (ntbl)
constexpr double kRec6 = 0.166667;              // RLM:3548 (not 1/6)
constexpr double kConG = 9.80665, kConAvgd = 6.0221415e23;
constexpr double kConAmd = 28.9644, kConAmw = 18.0154, kConAmo3 = 47.9982;
constexpr double kAbsrain = 0.33e-3, kAbssnow0 = 1.5;   // radlw_datatb.f:941,944
constexpr int kColRec = 48;                     // doubles per column record

// Minimum resident CTAs per SM requested from the register allocator
// (measured on B200, 16,384 columns x 127 layers: gas optics 3 in both
// precisions, transfer 4, gas optics behind the network 5).  The V = 8
// kernels (128..255 layers) are left uncapped: with the caps their
// transfer kernel spilled ~1 KB per thread and an illegal address was
// observed that reading the code did not explain.
#ifndef LW_GAS_MINB
#ifdef LW_GAS_MINB_SMALL   // build-time override for V <= 4 (tuning builds)
#define LW_GAS_MINB (V > 4 ? 1 : LW_GAS_MINB_SMALL)
#else
#define LW_GAS_MINB (V > 4 ? 1 : 3)
#endif
#endif
// gas optics behind the learned gas optics (setcoef/taumol only for
// out-of-envelope layers): light enough for more resident CTAs
#ifndef LW_GAS_MINB_SG
#define LW_GAS_MINB_SG (V > 4 ? 1 : 5)
#endif
#ifndef LW_RT_MINB
#ifdef LW_RT_MINB_SMALL
#define LW_RT_MINB (V > 4 ? 1 : LW_RT_MINB_SMALL)
#else
#define LW_RT_MINB (V > 4 ? 1 : 4)
#endif
#endif

static __device__ __constant__ double c_delwave[16] = {340., 150., 130., 70., 120., 160., 100., 100.,
                                                       210., 90., 320., 280., 170., 130., 220., 650.};
static __device__ __constant__ double c_a0[16] = {1.66, 1.55, 1.58, 1.66, 1.54, 1.454, 1.89, 1.33,
                                                  1.668, 1.66, 1.66, 1.66, 1.66, 1.66, 1.66, 1.66};
static __device__ __constant__ double c_a1[16] = {0.00, 0.25, 0.22, 0.00, 0.13, 0.446, -0.10, 0.40,
                                                  -0.006, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00};
static __device__ __constant__ double c_a2[16] = {0.00, -12.0, -11.7, 0.00, -0.72, -0.243, 0.19, -0.062,
                                                  0.414, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00};


// checked read of the FP64 coefficient tables
__device__ __forceinline__ double t64(const double* kt, long long o) {
  if (!LW_OK(o >= 0 && o < RRTMG_LW_TABLES_NDOUBLE, 11, o)) return 0.0;
  return __ldg(kt + o);
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
    double a = t64(kt, lwtab::absliq1 + (index - 1) + 58 * b);
    double c = t64(kt, lwtab::absliq1 + index + 58 * b);
    tauliq = fmax(0.0, clwp * (a + fint * (c - a)));
  }
  if (ciwp > 0.0) {
    if (f.ilwcice == 1) {
      double refice = fmin(130.0, fmax(13.0, reiw));
      int ia = (int)t64(kt, lwtab::ipat + b);
      tauice = fmax(0.0, ciwp * (t64(kt, lwtab::absice1 + 2 * (ia - 1)) +
                                 t64(kt, lwtab::absice1 + 1 + 2 * (ia - 1)) / refice));
    } else if (f.ilwcice == 2) {
      double factor = (reiw - 2.0) / 3.0;
      int index = max(1, min(42, (int)factor));
      double fint = factor - (double)index;
      double a = t64(kt, lwtab::absice2 + (index - 1) + 43 * b);
      double c = t64(kt, lwtab::absice2 + index + 43 * b);
      tauice = fmax(0.0, ciwp * (a + fint * (c - a)));
    } else if (f.ilwcice == 3) {
      double dgeice = fmax(5.0, 1.0315 * reiw);
      double factor = (dgeice - 2.0) / 3.0;
      int index = max(1, min(45, (int)factor));
      double fint = factor - (double)index;
      double a = t64(kt, lwtab::absice3 + (index - 1) + 46 * b);
      double c = t64(kt, lwtab::absice3 + index + 46 * b);
      tauice = fmax(0.0, ciwp * (a + fint * (c - a)));
    }
  }
  return tauice + tauliq + tauran + tausnw;
}

// Planck integral of band b at temperature index/fraction (RLM:2251-2283)
__device__ __forceinline__ double planck_int(const double* kt, int b, int ind, double frac) {
  double p0 = t64(kt, lwtab::totplnk + (ind - 1) + 181 * b);
  double p1 = t64(kt, lwtab::totplnk + ind + 181 * b);
  return c_delwave[b] * (p0 + frac * (p1 - p0));
}

template <typename R>
__host__ __device__ constexpr size_t gas_smem_bytes(int V) {
  const size_t NLP = 32 * (size_t)V;
  return sizeof(double) * (2 * NLP + 24 + 8 * NLP) + sizeof(R) * N_LF * NLP + sizeof(int) * (NLP + 4);
}

// Per-column working arrays of gas_column (shared memory in lw_gas_kernel,
// any memory the caller's threads can reach elsewhere); gas_smem_bytes<R>(V).
template <typename R, int V>
struct GasWork {
  double* red;   // [2 NLP]
  double* col;   // [24]
  double* cld;   // [8 NLP] cloud inputs of the layer
  R* lay;        // [N_LF NLP] setcoef record (LayRef)
  int* li;       // [NLP]
  int* ci;       // [4]
  __device__ __forceinline__ static GasWork at(void* base) {
    constexpr int NLP = 32 * V;
    GasWork w;
    w.red = reinterpret_cast<double*>(base);
    w.col = w.red + 2 * NLP;
    w.cld = w.col + 24;
    w.lay = reinterpret_cast<R*>(w.cld + 8 * NLP);
    w.li = reinterpret_cast<int*>(w.lay + N_LF * NLP);
    w.ci = w.li + NLP;
    return w;
  }
};

// Kernel A's work for one column cc of the chunk (global column sc.c0 + cc),
// run by the 32 V threads t = 0 .. 32 V - 1 that S synchronizes.
template <typename R, int V, bool SG, typename Sync>
__device__ __forceinline__ void gas_column(int cc, int t, const Sync& S, const GasWork<R, V>& W,
                                           const Block* __restrict__ blocks, int nblocks, const Block& b0,
                                           const Flags& f, const Tables<R>& tab, const Tables<double>& tab64,
                                           const Scratch<R>& sc, double* __restrict__ gas_taug,
                                           double* __restrict__ gas_fracs) {
  constexpr int NLP = 32 * V;
  double* s_red = W.red;
  double* s_col = W.col;
  double* s_cld = W.cld;
  R* s_lay = W.lay;
  int* s_li = W.li;
  int* s_ci = W.ci;
  const int nlay = f.nlay, nlp1 = nlay + 1;
  const KT<R> kt{tab.kt};
  const double* kt64 = tab64.kt;
  {
    const int c = sc.c0 + cc;                        // global column
    S.sync();
    const Block& B = (nblocks == 1) ? b0 : blocks[find_block(blocks, nblocks, c)];
    const int i = c - B.col0;
    const size_t ld = (size_t)B.ld;
    const bool top = f.top_at_1 != 0;
    auto IN = [&](int fld, int row) -> double {
      if (!LW_OK(row >= 0 && row <= nlay && i >= 0 && i < B.npts && B.in[fld], 12, row)) return 0.0;
      return B.in[fld][i + ld * row];
    };

    // ------------------------------ prologue + setcoef, FP64 -------------
    double tlyrfr = 0.0, tlvlfr = 0.0;
    int indlay = 1, indlev = 1, r = 0;
    bool lowerk = false, cldk = false;
    bool sg_skip = false;   // learned gas optics already wrote this layer's tau/frac
    if (t < nlay) {
      const int kref = t + 1;
      r = top ? nlp1 - kref - 1 : t;                  // 0-based input row of the layer
      const int rl = top ? nlp1 - kref - 1 : t + 1;   // 0-based input row of its top level
      double pavel = IN(F_PLYR, r), delp = IN(F_DELPIN, r), tavel = IN(F_TLYR, r), tz = IN(F_TLVL, rl);
      double q = IN(F_QLYR, r);
      const double amdw = kConAmd / kConAmw, amdo3 = kConAmd / kConAmo3;
      double h2ovmr = fmax(0.0, q * amdw / (1.0 - q));
      double o3vmr = fmax(0.0, IN(F_OLYR, r) * amdo3);
      double tem0 = (1.0 - h2ovmr) * kConAmd + h2ovmr * kConAmw;
      const double tem1c = 100.0 * kConG, tem2c = 1.0e-20 * 1.0e3 * kConAvgd;
      double coldry = tem2c * delp / (tem1c * tem0 * (1.0 + h2ovmr));
      double temcol = 1.0e-12 * coldry;
      const double colh2o = fmax(0.0, coldry * h2ovmr);
      // the learned gas optics already wrote tau/frac of layers inside its training
      // envelope: they need no setcoef record and no taumol here
      if (SG) {
        float xf[SG_NFEAT];
        layer_features(pavel, tavel, h2ovmr, o3vmr, IN(F_CO2, r), IN(F_CH4, r), IN(F_N2O, r), xf);
        sg_skip = in_envelope(xf, f.sg_norm);
        if (!sg_skip && f.sg_fallback) atomicAdd(f.sg_fallback, 1u);
      }
      indlay = min(180, max(1, (int)(tavel - 159.0)));
      tlyrfr = tavel - (int)tavel;
      indlev = min(180, max(1, (int)(tz - 159.0)));
      tlvlfr = tz - (int)tz;
      double plog = log(pavel);
      lowerk = plog > 4.56;
      if (!sg_skip) {
        double colv[7], wxv[4];
        colv[0] = colh2o;
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
        double summol = 0.0;
        for (int m = 1; m < 7; ++m) summol = summol + colv[m];
        double colbrd = coldry - summol;

        int jp = max(1, min(58, (int)(36.0 - 5.0 * (plog + 0.04))));
        int jp1 = jp + 1;
        double fp = fmax(0.0, fmin(1.0, 5.0 * (t64(kt64, lwtab::preflog + jp - 1) - plog)));
        double tem1 = (tavel - t64(kt64, lwtab::tref + jp - 1)) / 15.0;
        double tem2 = (tavel - t64(kt64, lwtab::tref + jp1 - 1)) / 15.0;
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

        R* ls = s_lay + t;
        ls[LF_FAC00 * NLP] = R(fac00); ls[LF_FAC01 * NLP] = R(fac01);
        ls[LF_FAC10 * NLP] = R(fac10); ls[LF_FAC11 * NLP] = R(fac11);
        ls[LF_SELFFAC * NLP] = R(selffac); ls[LF_SELFFRAC * NLP] = R(selffrac);
        ls[LF_FORFAC * NLP] = R(forfac); ls[LF_FORFRAC * NLP] = R(forfrac);
        ls[LF_MINORFRAC * NLP] = R(minorfrac);
        ls[LF_SCALEMINOR * NLP] = R(scaleminor); ls[LF_SCALEMINORN2 * NLP] = R(scaleminorn2);
        for (int m = 0; m < 7; ++m) ls[(LF_COL1 + m) * NLP] = R(colv[m]);
        ls[LF_COLDRY * NLP] = R(coldry); ls[LF_COLBRD * NLP] = R(colbrd);
        for (int m = 0; m < 4; ++m) ls[(LF_WX1 + m) * NLP] = R(wxv[m]);
        ls[LF_PAVEL * NLP] = R(pavel);
        s_li[t] = jp | (jt << 8) | (jt1 << 12) | (indself << 16) | (indfor << 20) | (indminor << 24);
      }
      double cf = IN(F_CLDCF, r);
      cldk = cf > kEps;
      double* cl = s_cld + t;
      cl[0 * NLP] = cf;
      if (f.ilwcliq > 0) {
        cl[1 * NLP] = IN(F_LWP, r); cl[2 * NLP] = IN(F_RELIQ, r); cl[3 * NLP] = IN(F_IWP, r);
        cl[4 * NLP] = IN(F_REICE, r); cl[5 * NLP] = IN(F_RWP, r); cl[6 * NLP] = IN(F_SWP, r);
        cl[7 * NLP] = IN(F_RESNOW, r);
      } else {
        cl[5 * NLP] = IN(F_CLDOD, r);
      }
      s_red[t] = coldry;
      s_red[NLP + t] = colh2o;
    }
    const int laytrop = S.count(lowerk);
    const int lcf1 = S.any(cldk);
    if (t == 0) {
      // precipitable water (RLM:910-919 / 1012-1019): sequential, reference order
      double tem1 = 0.0, tem2 = 0.0;
      for (int k = 0; k < nlay; ++k) {
        tem1 = tem1 + s_red[k] + s_red[NLP + k];
        tem2 = tem2 + s_red[NLP + k];
      }
      const double amdw = kConAmd / kConAmw;
      double tem0 = 10.0 * tem2 / (amdw * tem1 * kConG);
      s_col[17] = tem0 * (top ? IN(F_PLVL, nlay) : IN(F_PLVL, 0));
      double sfe = B.in[F_SFEMIS][i];
      s_col[16] = (sfe > kEps && sfe <= 1.0) ? sfe : 1.0;
      double stemp = B.in[F_SFGTMP][i];
      double tz0 = top ? IN(F_TLVL, nlay) : IN(F_TLVL, 0);
      s_col[18] = stemp - (int)stemp;
      s_col[19] = tz0 - (int)tz0;
      s_ci[0] = min(180, max(1, (int)(stemp - 159.0)));
      s_ci[1] = min(180, max(1, (int)(tz0 - 159.0)));
    }
    S.sync();
    const bool write_scratch = sc.tau != nullptr;
    double* crec = write_scratch ? sc.col + (size_t)cc * kColRec : nullptr;
    if (crec && !LW_OK(cc < sc.cap, 18, cc)) crec = nullptr;
    if (t < NBANDS) {
      // diffusivity angle (RLM:1041-1050) and surface Planck terms (RLM:2251-2262)
      double secd = (t == 0 || t == 3 || t == 9)
                        ? 1.66
                        : fmin(1.80, fmax(1.50, c_a0[t] + c_a1[t] * exp(c_a2[t] * s_col[17])));
      if (crec) {
        crec[t] = secd;
        crec[16 + t] = planck_int(kt64, t, s_ci[0], s_col[18]);   // pklay(b, 0): stemp
      }
    }
    if (t == 0 && crec) {
      crec[32] = s_col[16];
      crec[33] = lcf1 ? 1.0 : 0.0;
    }

    // ------------------------------ bands --------------------------------
    // taumol splits at the count laytrop (RLM:2344-2346)
    const LayRef<R> LR{s_lay, s_li, t, NLP, t < laytrop};
    R* tcol = write_scratch ? sc.tau + (size_t)cc * NGPT * NLP + t : nullptr;
    R* fcol = write_scratch ? sc.frac + (size_t)cc * NGPT * NLP + t : nullptr;
    R* bcol = write_scratch ? sc.band + (size_t)cc * 3 * NBANDS * NLP : nullptr;
#pragma unroll 1
    for (int b = 0; b < NBANDS; ++b) {
      if (t < nlay) {
        double tcld = 0.0;
        if (lcf1) {
          const double* cl = s_cld + t;
          tcld = band_taucld(b, f, kt64, cl[0], cl[NLP], cl[2 * NLP], cl[3 * NLP], cl[4 * NLP], cl[5 * NLP],
                             cl[6 * NLP], cl[7 * NLP]);
        }
        if (b == 6 && !f.gas_only && LW_OK(r < nlay && i < B.npts, 13, r)) B.out[O_CLDTAU][i + ld * r] = lcf1 ? tcld : 0.0;   // band 7 (RLM:1087-1097)
        if (bcol && LW_OK(cc < sc.cap && t + 1 < NLP, 14, cc)) {   // evict-first stores: the hand-off must not push the tables out of L2
          __stcs(bcol + (0 * NBANDS + b) * NLP + t, R(planck_int(kt64, b, indlay, tlyrfr)));
          __stcs(bcol + (1 * NBANDS + b) * NLP + t + 1, R(planck_int(kt64, b, indlev, tlvlfr)));
          __stcs(bcol + (2 * NBANDS + b) * NLP + t, R(tcld));
        }
        const size_t ab = i + ld * ((size_t)r + (size_t)nlay * b);
        R tauaer = R(0);
        if (!sg_skip && LW_OK(r < nlay && i < B.npts, 15, r)) tauaer = R(B.in[F_AERAOD][ab] * (1.0 - B.in[F_AERSSA][ab]));
        const int ns = ns_of(b);
        const size_t go = ((size_t)c * nlay + t) * NGPT + ns;
        if (!sg_skip) band_gas_optics<R>(b, kt, LR, [&](int g0, R tau, R frac) {
          if (tcol && LW_OK(cc < sc.cap && ns + g0 < NGPT, 16, ns + g0)) {
            __stcs(tcol + (size_t)(ns + g0) * NLP, tau + tauaer);
            __stcs(fcol + (size_t)(ns + g0) * NLP, frac);
          }
          if (f.gas_only && LW_OK(c < sc.ntot, 17, c)) {
            gas_taug[go + g0] = (double)tau;
            gas_fracs[go + g0] = (double)frac;
          }
        });
      }
      if (t == 0 && bcol) __stcs(bcol + (1 * NBANDS + b) * NLP, R(planck_int(kt64, b, s_ci[1], s_col[19])));
    }
  }
}

template <typename R, int V, bool SG>
__global__ void __launch_bounds__(32 * V, SG ? LW_GAS_MINB_SG : LW_GAS_MINB)
lw_gas_kernel(const Block* __restrict__ blocks, int nblocks, const Block b0, int ncols, Flags f,
              Tables<R> tab, Tables<double> tab64, Scratch<R> sc, double* __restrict__ gas_taug,
              double* __restrict__ gas_fracs) {
  extern __shared__ __align__(16) char smem_raw[];   // gas_smem_bytes<R>(V)
  const GasWork<R, V> W = GasWork<R, V>::at(smem_raw);
  for (int cc = blockIdx.x; cc < ncols; cc += gridDim.x)
    gas_column<R, V, SG>(cc, threadIdx.x, CtaSync{}, W, blocks, nblocks, b0, f, tab, tab64, sc, gas_taug, gas_fracs);
}

}  // namespace lw
