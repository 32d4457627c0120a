// sw_column.cu -- the RRTMG-SW column kernels for B200 (FP64).
//
// rrtmg_sw_run (physics/Radiation/RRTMG/radsw_main.F90:493-1379, RSM below)
// for the McICA configurations runs as three launches over a chunk of
// daytime columns:
//   sw_optics_kernel  one warp per column, lanes over layers: the driver's
//                     layer prologue (RSM:910-1094), setcoef (RSM:2242-2389),
//                     taumol16..29 (RSM:4094-5573; every lane runs the same
//                     band's code, so the band branches never diverge),
//                     the solar source sfluxzen, the clear/cloudy column test
//                     (RSM:1101-1125) and cldprop (RSM:1566-1938);
//   lw_mcica_kernel<112>  the sub-column generator (lw_mcica.cu);
//   sw_rt_kernel      one warp per column, lanes over g-points: spcvrtm
//                     (RSM:3228-3942) with vrtqdr (RSM:3959-4051) and the
//                     flux / heating-rate outputs (RSM:1225-1373).
// Per lane (g-point) the clear-sky and all-sky sweeps run side by side: the
// upward sweep evaluates each layer's clear two-stream optics once (the
// all-sky sweep re-evaluates only the layers whose McICA flag is set) and
// keeps them, with both adding recurrences (zrupb, zrupd), in global
// scratch; the downward sweep reads them back and produces both sweeps'
// fluxes level by level.  Fluxes are summed over g-points with warp
// butterflies in a fixed order.
//
// Built with -fmad=false: every statement keeps the reference's evaluation
// order and rounding.
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "sw_kernels.h"
#include "../data/rrtmg_sw_table_layout.h"

namespace sw {

__constant__ int c_ng[14] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};   // radsw_param.f NG16..29
__constant__ int c_ns[14] = {0, 6, 18, 26, 34, 44, 54, 56, 66, 74, 80, 86, 94, 100};
__constant__ int c_nspa[14] = {9, 9, 9, 9, 1, 9, 9, 1, 9, 1, 0, 1, 9, 1};      // RSM:359
__constant__ int c_nspb[14] = {1, 5, 1, 1, 1, 5, 1, 0, 1, 0, 0, 1, 5, 1};      // RSM:360
__constant__ int c_idxsfc[14] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 2, 2, 2, 2, 1};    // RSM:362
__constant__ int c_idxebc[14] = {5, 5, 4, 4, 3, 3, 2, 2, 1, 1, 1, 1, 1, 5};    // RSM:363

constexpr double kEps = 1.0e-6, kOneMinus = 1.0 - kEps, kBpade = 1.0 / 0.278, kStpfac = 296.0 / 1013.0;
constexpr double kFtiny = 1.0e-12, kFlimit = 1.0e-20;
constexpr double kConG = 9.80665, kConAvgd = 6.0221415e23, kConAmd = 28.9644, kConAmw = 18.0154,
                 kConAmo3 = 47.9982;
constexpr double kAmdw = kConAmd / kConAmw, kAmdo3 = kConAmd / kConAmo3;
constexpr int kNtbmx = 10000;

__device__ __forceinline__ int band_of(int g) {   // NGB (radsw_param.f), 0-based band
  int b = 0;
#pragma unroll
  for (int j = 1; j < 14; ++j) b += (g >= c_ns[j]) ? 1 : 0;
  return b;
}

// ---- one layer's prologue + setcoef record -------------------------------
struct Lay {
  double colamt[6], colmol, delp;
  double fac00, fac01, fac10, fac11, forfac, forfrac, selffac, selffrac;
  int jp, jt, jt1, indfor, indself;
  bool lower_plog;   // plog > 4.56
};

// rrtmg_sw_run's layer prologue (RSM:910-946 / 1001-1040) for internal
// layer k (0-based, surface first) of caller column i, then setcoef.
__device__ void layer_record(const SwArgs& a, int i, int k, const double* __restrict__ T, Lay& L) {
  const int r = a.top_at_1 ? a.nlay - 1 - k : k;
  const size_t x = (size_t)i + (size_t)a.ld * r;
  const double tem1 = 100.0 * kConG, tem2 = 1.0e-20 * 1.0e3 * kConAvgd;
  const double pavel = a.plyr[x], tavel = a.tlyr[x], q = a.qlyr[x];
  L.delp = a.delp[x];
  const double h2ovmr = fmax(0.0, q * kAmdw / (1.0 - q));
  const double o3vmr = fmax(0.0, a.olyr[x] * kAmdo3);
  const double tem0 = (1.0 - h2ovmr) * kConAmd + h2ovmr * kConAmw;
  const double coldry = tem2 * L.delp / (tem1 * tem0 * (1.0 + h2ovmr));
  const double temcol = 1.0e-12 * coldry;
  L.colamt[0] = fmax(0.0, coldry * h2ovmr);
  L.colamt[1] = fmax(temcol, coldry * a.co2[x]);
  L.colamt[2] = fmax(0.0, coldry * o3vmr);
  if (a.inc_minor) {
    L.colamt[3] = fmax(temcol, coldry * a.n2o[x]);
    L.colamt[4] = fmax(temcol, coldry * a.ch4[x]);
    L.colamt[5] = fmax(temcol, coldry * a.o2[x]);
  } else {
    L.colamt[3] = L.colamt[4] = L.colamt[5] = temcol;
  }
  L.colmol = coldry + L.colamt[0];
  // setcoef (RSM:2242-2389)
  L.forfac = pavel * kStpfac / (tavel * (1.0 + h2ovmr));
  const double plog = log(pavel);
  L.jp = max(1, min(58, (int)(36.0 - 5.0 * (plog + 0.04))));
  const int jp1 = L.jp + 1;
  const double fp = 5.0 * (__ldg(T + swtab::preflog + L.jp - 1) - plog);
  double t1 = (tavel - __ldg(T + swtab::tref + L.jp - 1)) / 15.0;
  double t2 = (tavel - __ldg(T + swtab::tref + jp1 - 1)) / 15.0;
  L.jt = max(1, min(4, (int)(3.0 + t1)));
  L.jt1 = max(1, min(4, (int)(3.0 + t2)));
  const double ft = t1 - (double)(L.jt - 3);
  const double ft1 = t2 - (double)(L.jt1 - 3);
  const double fp1 = 1.0 - fp;
  L.fac10 = fp1 * ft;
  L.fac00 = fp1 * (1.0 - ft);
  L.fac11 = fp * ft1;
  L.fac01 = fp * (1.0 - ft1);
  L.lower_plog = plog > 4.56;
  if (L.lower_plog) {
    t1 = (332.0 - tavel) / 36.0;
    L.indfor = min(2, max(1, (int)t1));
    L.forfrac = t1 - (double)L.indfor;
    t2 = (tavel - 188.0) / 7.2;
    L.indself = min(9, max(1, (int)t2 - 7));
    L.selffrac = t2 - (double)(L.indself + 7);
    L.selffac = h2ovmr * L.forfac;
  } else {
    t1 = (tavel - 188.0) / 36.0;
    L.indfor = 3;
    L.forfrac = t1 - 1.0;
    L.indself = 0;
    L.selffrac = 0.0;
    L.selffac = 0.0;
  }
}

// ---- taumol for one layer, every g-point (RSM:4094-5573) ------------------
// Table views with Fortran subscripts: ka(ind, j) of a (rows, ng) array.
struct Tab {
  const double* p;
  int rows;
  __device__ __forceinline__ double operator()(int ind, int j) const { return __ldg(p + (ind - 1) + rows * (j - 1)); }
};

// the eight-point binary-species interpolation (fac000*k(i01) + fac100*k(i01+1)
// + fac010*k(i01+d) + fac110*k(i01+d+1) + the same at i11), left to right
__device__ __forceinline__ double k8(const Tab& t, const double (&f)[8], int i01, int d, int i11, int j) {
  return f[0] * t(i01, j) + f[2] * t(i01 + 1, j) + f[1] * t(i01 + d, j) + f[3] * t(i01 + d + 1, j) +
         f[4] * t(i11, j) + f[6] * t(i11 + 1, j) + f[5] * t(i11 + d, j) + f[7] * t(i11 + d + 1, j);
}
__device__ __forceinline__ double k4(const Tab& t, const Lay& L, int i01, int i11, int j) {
  return L.fac00 * t(i01, j) + L.fac10 * t(i01 + 1, j) + L.fac01 * t(i11, j) + L.fac11 * t(i11 + 1, j);
}
// speccomb/specmult/js/fs and the eight weights (RSM:4386-4399)
__device__ __forceinline__ double spec8(const Lay& L, int g1, int g2, double strrat, double mult, int& js, double& fs,
                                        double (&f)[8]) {
  const double speccomb = L.colamt[g1] + strrat * L.colamt[g2];
  const double specmult = mult * fmin(kOneMinus, L.colamt[g1] / speccomb);
  js = 1 + (int)specmult;
  fs = fmod(specmult, 1.0);
  const double fs1 = 1.0 - fs;
  f[0] = fs1 * L.fac00;
  f[1] = fs1 * L.fac10;
  f[2] = fs * L.fac00;
  f[3] = fs * L.fac10;
  f[4] = fs1 * L.fac01;
  f[5] = fs1 * L.fac11;
  f[6] = fs * L.fac01;
  f[7] = fs * L.fac11;
  return speccomb;
}
__device__ __forceinline__ double selfc(const Tab& s, const Lay& L, int j) {
  const int a = L.indself, b = a + 1;
  return L.selffac * (s(a, j) + L.selffrac * (s(b, j) - s(a, j)));
}
__device__ __forceinline__ double forc(const Tab& f, const Lay& L, int j) {
  const int a = L.indfor, b = a + 1;
  return L.forfac * (f(a, j) + L.forfrac * (f(b, j) - f(a, j)));
}

__device__ void taumol_layer(const Lay& L, bool lower, const int id0[14], const int id1[14],
                             const double* __restrict__ T, double* __restrict__ tg, double* __restrict__ tr) {
  int js;
  double fs, f[8];
  const double* strr = T + swtab::strrat;
  // Rayleigh: one coefficient for bands 16-22, 28, 29
  const double rs[14] = {T[swtab::b16_rayl], T[swtab::b17_rayl], T[swtab::b18_rayl], T[swtab::b19_rayl],
                         T[swtab::b20_rayl], T[swtab::b21_rayl], T[swtab::b22_rayl], 0.0, 0.0, 0.0, 0.0, 0.0,
                         T[swtab::b28_rayl], T[swtab::b29_rayl]};
#pragma unroll 1
  for (int b = 0; b < 14; ++b) {
    if (b == 7 || b == 8 || b == 9 || b == 10 || b == 11) continue;
    const double tauray = L.colmol * rs[b];
    for (int j = 0; j < c_ng[b]; ++j) tr[c_ns[b] + j] = tauray;
  }
  {  // per-g Rayleigh of bands 23, 25, 26, 27
    const int bands[4] = {7, 9, 10, 11};
    const int offs[4] = {swtab::b23_rayl, swtab::b25_rayl, swtab::b26_rayl, swtab::b27_rayl};
#pragma unroll 1
    for (int q = 0; q < 4; ++q)
      for (int j = 0; j < c_ng[bands[q]]; ++j) tr[c_ns[bands[q]] + j] = L.colmol * __ldg(T + offs[q] + j);
  }
  const double o2tem = 4.35e-4 / (350.0 * 2.0), o2adj = 1.6;
  // bands 16, 17, 18, 19, 21, 22: binary species in the lower atmosphere
  {
    const int bands[6] = {0, 1, 2, 3, 5, 6};
    const int g2s[6] = {4, 1, 4, 1, 1, 5};
    const int oa[6] = {swtab::b16_absa, swtab::b17_absa, swtab::b18_absa, swtab::b19_absa, swtab::b21_absa,
                       swtab::b22_absa};
    const int ob[6] = {swtab::b16_absb, swtab::b17_absb, swtab::b18_absb, swtab::b19_absb, swtab::b21_absb,
                       swtab::b22_absb};
    const int os[6] = {swtab::b16_selfref, swtab::b17_selfref, swtab::b18_selfref, swtab::b19_selfref,
                       swtab::b21_selfref, swtab::b22_selfref};
    const int of[6] = {swtab::b16_forref, swtab::b17_forref, swtab::b18_forref, swtab::b19_forref,
                       swtab::b21_forref, swtab::b22_forref};
    const int mfr[6] = {3, 4, 3, 3, 4, 3};
#pragma unroll 1
    for (int q = 0; q < 6; ++q) {
      const int b = bands[q], ns = c_ns[b], ng = c_ng[b];
      const Tab absa{T + oa[q], 585}, selfref{T + os[q], 10}, forref{T + of[q], mfr[q]};
      const Tab absb{T + ob[q], (b == 1 || b == 5) ? 1175 : 235};
      if (lower) {
        const double speccomb = spec8(L, 0, g2s[q], strr[b], 8.0, js, fs, f);
        const int i01 = id0[b] + js, i11 = id1[b] + js;
        const double o2cont = o2tem * L.colamt[5];
        for (int j = 1; j <= ng; ++j) {
          double t = speccomb * k8(absa, f, i01, 9, i11, j) + L.colamt[0] * (selfc(selfref, L, j) + forc(forref, L, j));
          if (b == 6) t = t + o2cont;
          tg[ns + j - 1] = t;
        }
      } else if (b == 1 || b == 5) {   // 17, 21: binary species above too
        const double speccomb = spec8(L, 0, 1, strr[b], 4.0, js, fs, f);
        const int i01 = id0[b] + js, i11 = id1[b] + js;
        for (int j = 1; j <= ng; ++j) {
          const int a0 = L.indfor, a1 = a0 + 1;
          tg[ns + j - 1] = speccomb * k8(absb, f, i01, 5, i11, j) +
                           L.colamt[0] * L.forfac * (forref(a0, j) + L.forfrac * (forref(a1, j) - forref(a0, j)));
        }
      } else {
        const int i01 = id0[b] + 1, i11 = id1[b] + 1;
        const double o2cont = o2tem * L.colamt[5];
        for (int j = 1; j <= ng; ++j) {
          if (b == 6) tg[ns + j - 1] = L.colamt[5] * o2adj * k4(absb, L, i01, i11, j) + o2cont;
          else tg[ns + j - 1] = L.colamt[b == 3 ? 1 : 4] * k4(absb, L, i01, i11, j);
        }
      }
    }
  }
  {  // band 20: H2O, CH4
    const int b = 4, ns = c_ns[b];
    const Tab absa{T + swtab::b20_absa, 65}, absb{T + swtab::b20_absb, 235}, selfref{T + swtab::b20_selfref, 10},
        forref{T + swtab::b20_forref, 4};
    const double* absch4 = T + swtab::b20_absch4;
    const int i01 = id0[b] + 1, i11 = id1[b] + 1;
    for (int j = 1; j <= 10; ++j) {
      if (lower)
        tg[ns + j - 1] = L.colamt[0] * (k4(absa, L, i01, i11, j) + selfc(selfref, L, j) + forc(forref, L, j)) +
                         L.colamt[4] * __ldg(absch4 + j - 1);
      else
        tg[ns + j - 1] = L.colamt[0] * (k4(absb, L, i01, i11, j) + forc(forref, L, j)) + L.colamt[4] * __ldg(absch4 + j - 1);
    }
  }
  {  // band 23: H2O below, nothing above
    const int b = 7, ns = c_ns[b];
    const Tab absa{T + swtab::b23_absa, 65}, selfref{T + swtab::b23_selfref, 10}, forref{T + swtab::b23_forref, 3};
    const double givfac = T[swtab::b23_givfac];
    const int i01 = id0[b] + 1, i11 = id1[b] + 1;
    for (int j = 1; j <= 10; ++j)
      tg[ns + j - 1] = lower ? L.colamt[0] * (givfac * k4(absa, L, i01, i11, j) + selfc(selfref, L, j) + forc(forref, L, j))
                             : 0.0;
  }
  {  // band 24: H2O/O2 below, O2 above; O3 both; Rayleigh from the species bin
    const int b = 8, ns = c_ns[b];
    const Tab absa{T + swtab::b24_absa, 585}, absb{T + swtab::b24_absb, 235}, selfref{T + swtab::b24_selfref, 10},
        forref{T + swtab::b24_forref, 3};
    const double *abso3a = T + swtab::b24_abso3a, *abso3b = T + swtab::b24_abso3b, *rayla = T + swtab::b24_rayla,
                 *raylb = T + swtab::b24_raylb;
    if (lower) {
      const double speccomb = spec8(L, 0, 5, strr[b], 8.0, js, fs, f);
      const int i01 = id0[b] + js, i11 = id1[b] + js;
      for (int j = 1; j <= 8; ++j) {
        tg[ns + j - 1] = speccomb * k8(absa, f, i01, 9, i11, j) + L.colamt[2] * __ldg(abso3a + j - 1) +
                         L.colamt[0] * (selfc(selfref, L, j) + forc(forref, L, j));
        const double ra = __ldg(rayla + (j - 1) + 8 * (js - 1)), rb = __ldg(rayla + (j - 1) + 8 * js);
        tr[ns + j - 1] = L.colmol * (ra + fs * (rb - ra));
      }
    } else {
      const int i01 = id0[b] + 1, i11 = id1[b] + 1;
      for (int j = 1; j <= 8; ++j) {
        tg[ns + j - 1] = L.colamt[5] * k4(absb, L, i01, i11, j) + L.colamt[2] * __ldg(abso3b + j - 1);
        tr[ns + j - 1] = L.colmol * __ldg(raylb + j - 1);
      }
    }
  }
  {  // band 25: H2O below; O3 both
    const int b = 9, ns = c_ns[b];
    const Tab absa{T + swtab::b25_absa, 65};
    const double *abso3a = T + swtab::b25_abso3a, *abso3b = T + swtab::b25_abso3b;
    const int i01 = id0[b] + 1, i11 = id1[b] + 1;
    for (int j = 1; j <= 6; ++j)
      tg[ns + j - 1] = lower ? L.colamt[0] * k4(absa, L, i01, i11, j) + L.colamt[2] * __ldg(abso3a + j - 1)
                             : L.colamt[2] * __ldg(abso3b + j - 1);
  }
  for (int j = 0; j < 6; ++j) tg[c_ns[10] + j] = 0.0;   // band 26: Rayleigh only
  {  // band 27: O3
    const int b = 11, ns = c_ns[b];
    const Tab absa{T + swtab::b27_absa, 65}, absb{T + swtab::b27_absb, 235};
    const int i01 = id0[b] + 1, i11 = id1[b] + 1;
    for (int j = 1; j <= 8; ++j)
      tg[ns + j - 1] = L.colamt[2] * (lower ? k4(absa, L, i01, i11, j) : k4(absb, L, i01, i11, j));
  }
  {  // band 28: O3/O2 both
    const int b = 12, ns = c_ns[b];
    const Tab absa{T + swtab::b28_absa, 585}, absb{T + swtab::b28_absb, 1175};
    const double speccomb = spec8(L, 2, 5, strr[b], lower ? 8.0 : 4.0, js, fs, f);
    const int i01 = id0[b] + js, i11 = id1[b] + js;
    for (int j = 1; j <= 6; ++j)
      tg[ns + j - 1] = speccomb * (lower ? k8(absa, f, i01, 9, i11, j) : k8(absb, f, i01, 5, i11, j));
  }
  {  // band 29: H2O + CO2 below, CO2 + H2O above
    const int b = 13, ns = c_ns[b];
    const Tab absa{T + swtab::b29_absa, 65}, absb{T + swtab::b29_absb, 235}, selfref{T + swtab::b29_selfref, 10},
        forref{T + swtab::b29_forref, 4};
    const double *absco2 = T + swtab::b29_absco2, *absh2o = T + swtab::b29_absh2o;
    const int i01 = id0[b] + 1, i11 = id1[b] + 1;
    for (int j = 1; j <= 12; ++j) {
      if (lower)
        tg[ns + j - 1] = L.colamt[0] * (k4(absa, L, i01, i11, j) + selfc(selfref, L, j) + forc(forref, L, j)) +
                         L.colamt[1] * __ldg(absco2 + j - 1);
      else
        tg[ns + j - 1] = L.colamt[1] * k4(absb, L, i01, i11, j) + L.colamt[0] * __ldg(absh2o + j - 1);
    }
  }
}

// ---- cldprop for one layer (RSM:1687-1903) --------------------------------
__device__ void cloud_layer(const SwArgs& a, size_t x, const double* __restrict__ T, double* __restrict__ tw,
                            double* __restrict__ sw, double* __restrict__ gw) {
  double tauliq[14], ssaliq[14], asyliq[14], tauice[14], ssaice[14], asyice[14];
  const double cf = a.cf[x];
  if (!(cf > kFtiny)) {
    for (int b = 0; b < 14; ++b) { tw[b] = 0.0; sw[b] = 1.0; gw[b] = 0.0; }
    return;
  }
  if (a.iswcliq > 0) {
    const double cldran = a.rwp[x], cldsnw = a.swp[x], refsnw = a.res[x];
    const double dgesnw = 1.0315 * refsnw;
    const double tauran = cldran * T[swtab::a0r];
    const double tausnw = (cldsnw > 0.0 && refsnw > 10.0) ? cldsnw * 1.09087 * (T[swtab::a0s] + T[swtab::a1s] / dgesnw)
                                                         : 0.0;
    const double cldliq = a.lwp[x], cldice = a.iwp[x], refliq = a.rel[x];
    double refice = a.rei[x];
    for (int b = 0; b < 14; ++b) { tauliq[b] = ssaliq[b] = asyliq[b] = tauice[b] = ssaice[b] = asyice[b] = 0.0; }
    if (cldliq > 0.0 && (a.iswcliq == 1 || a.iswcliq == 2)) {
      const double factor = refliq - 1.5;
      const int index = max(1, min(57, (int)factor));
      const double fint = factor - (double)index;
      const Tab ext{T + (a.iswcliq == 1 ? swtab::extliq1 : swtab::extliq2), 58};
      const Tab ssa{T + (a.iswcliq == 1 ? swtab::ssaliq1 : swtab::ssaliq2), 58};
      const Tab asy{T + (a.iswcliq == 1 ? swtab::asyliq1 : swtab::asyliq2), 58};
      for (int b = 0; b < 14; ++b) {
        const int c = b + 1;
        const double e = fmax(0.0, ext(index, c) + fint * (ext(index + 1, c) - ext(index, c)));
        const double s = fmax(0.0, fmin(1.0, ssa(index, c) + fint * (ssa(index + 1, c) - ssa(index, c))));
        const double g = fmax(0.0, fmin(1.0, asy(index, c) + fint * (asy(index + 1, c) - asy(index, c))));
        tauliq[b] = cldliq * e;
        ssaliq[b] = tauliq[b] * s;
        asyliq[b] = ssaliq[b] * g;
      }
    }
    if (cldice > 0.0) {
      if (a.iswcice == 1) {
        refice = fmin(130.0, fmax(13.0, refice));
        for (int b = 0; b < 14; ++b) {
          const int ia = c_idxebc[b] - 1;
          const double e = fmax(0.0, T[swtab::abari + ia] + T[swtab::bbari + ia] / refice);
          const double s = fmax(0.0, fmin(1.0, 1.0 - T[swtab::cbari + ia] - T[swtab::dbari + ia] * refice));
          const double g = fmax(0.0, fmin(1.0, T[swtab::ebari + ia] + T[swtab::fbari + ia] * refice));
          tauice[b] = cldice * e;
          ssaice[b] = tauice[b] * s;
          asyice[b] = ssaice[b] * g;
        }
      } else if (a.iswcice == 2 || a.iswcice == 3) {
        int index, rows;
        double fint;
        if (a.iswcice == 2) {
          refice = fmin(131.0, fmax(5.0, refice));
          const double factor = (refice - 2.0) / 3.0;
          index = max(1, min(42, (int)factor));
          fint = factor - (double)index;
          rows = 43;
        } else {
          const double dgeice = fmax(5.0, fmin(140.0, 1.0315 * refice));
          const double factor = (dgeice - 2.0) / 3.0;
          index = max(1, min(45, (int)factor));
          fint = factor - (double)index;
          rows = 46;
        }
        const Tab ext{T + (a.iswcice == 2 ? swtab::extice2 : swtab::extice3), rows};
        const Tab ssa{T + (a.iswcice == 2 ? swtab::ssaice2 : swtab::ssaice3), rows};
        const Tab asy{T + (a.iswcice == 2 ? swtab::asyice2 : swtab::asyice3), rows};
        for (int b = 0; b < 14; ++b) {
          const int c = b + 1;
          const double e = fmax(0.0, ext(index, c) + fint * (ext(index + 1, c) - ext(index, c)));
          const double s = fmax(0.0, fmin(1.0, ssa(index, c) + fint * (ssa(index + 1, c) - ssa(index, c))));
          const double g = fmax(0.0, fmin(1.0, asy(index, c) + fint * (asy(index + 1, c) - asy(index, c))));
          tauice[b] = cldice * e;
          ssaice[b] = tauice[b] * s;
          asyice[b] = ssaice[b] * g;
        }
      }
    }
    for (int b = 0; b < 14; ++b) {
      const double ssaran = tauran * (1.0 - T[swtab::b0r + b]);
      const double ssasnw = tausnw * (1.0 - (T[swtab::b0s + b] + T[swtab::b1s + b] * dgesnw));
      const double asyran = ssaran * T[swtab::c0r + b];
      const double asysnw = ssasnw * T[swtab::c0s + b];
      tw[b] = tauliq[b] + tauice[b] + tauran + tausnw;
      sw[b] = ssaliq[b] + ssaice[b] + ssaran + ssasnw;
      gw[b] = asyliq[b] + asyice[b] + asyran + asysnw;
    }
  } else {
    const double od = a.cod[x], ss = a.cssa[x], as = a.casy[x];
    for (int b = 0; b < 14; ++b) {
      tw[b] = od;
      sw[b] = od * ss;
      gw[b] = sw[b] * as;
    }
  }
}

// ---- kernel 1: optics ------------------------------------------------------
constexpr int kOptWarps = 4;

// One column's optics: a = the argument record of the call (or of the
// physics block) the column belongs to, j1 its 1-based column there.
__device__ __forceinline__ void optics_body(const SwArgs& a, const SwScratch& s, int pl, int nc, int j1, int lane,
                                            int* s_jp_w, const double* __restrict__ T) {
  const int i = j1 - 1, nlay = a.nlay;
  // laytrop: the last layer with ln p > 4.56, nlay if none (RSM:2305, 2353)
  int laytrop = 0;
  for (int k0 = 0; k0 < nlay; k0 += 32) {
    const int k = k0 + lane;
    bool hi = false;
    if (k < nlay) {
      const int r = a.top_at_1 ? nlay - 1 - k : k;
      const double plog = log(a.plyr[(size_t)i + (size_t)a.ld * r]);
      s_jp_w[k] = max(1, min(58, (int)(36.0 - 5.0 * (plog + 0.04))));
      hi = plog > 4.56;
    }
    const unsigned m = __ballot_sync(0xffffffffu, hi);
    if (m) laytrop = k0 + 32 - __clz(m);
  }
  if (laytrop == 0) laytrop = nlay;
  __syncwarp();

  // gas optics, one layer per lane
  for (int k = lane; k < nlay; k += 32) {
    Lay L;
    layer_record(a, i, k, T, L);
    const bool lower = (k + 1) <= laytrop;
    int id0[14], id1[14];
#pragma unroll
    for (int b = 0; b < 14; ++b) {
      if (lower) {
        id0[b] = ((L.jp - 1) * 5 + (L.jt - 1)) * c_nspa[b];
        id1[b] = (L.jp * 5 + (L.jt1 - 1)) * c_nspa[b];
      } else {
        id0[b] = ((L.jp - 13) * 5 + (L.jt - 1)) * c_nspb[b];
        id1[b] = ((L.jp - 12) * 5 + (L.jt1 - 1)) * c_nspb[b];
      }
    }
    double* tg = s.taug + ((size_t)pl * nlay + k) * kSwNg;
    double* tr = s.taur + ((size_t)pl * nlay + k) * kSwNg;
    taumol_layer(L, lower, id0, id1, T, tg, tr);
  }

  // solar source per band (RSM:4225-4310), one band per lane
  if (lane < 14) {
    const int b = lane, jb = 16 + b, ng = c_ng[b], ns = c_ns[b];
    const int ibd = (int)T[swtab::ibx + b];
    double* sf = s.sflux + (size_t)pl * kSwNg + ns;
    if (jb == 16 || jb == 20 || jb == 23 || jb == 25 || jb == 26 || jb == 29) {
      for (int j = 0; j < ng; ++j) sf[j] = T[swtab::sfluxref01 + j + 16 * (ibd - 1)];
    } else if (jb == 27) {
      for (int j = 0; j < ng; ++j) sf[j] = T[swtab::scalekur] * T[swtab::sfluxref01 + j + 16 * (ibd - 1)];
    } else {
      const int lref = (int)T[swtab::layreffr + b];
      int ks;   // 1-based
      if (jb == 17 || jb == 28) {
        ks = nlay;
        for (int k = laytrop; k <= nlay - 1; ++k)
          if (s_jp_w[k - 1] < lref && s_jp_w[k] >= lref) { ks = k + 1; break; }
      } else {
        ks = laytrop;
        for (int k = 1; k <= laytrop - 1; ++k)
          if (s_jp_w[k - 1] < lref && s_jp_w[k] >= lref) { ks = k + 1; break; }
      }
      Lay L;
      layer_record(a, i, ks - 1, T, L);
      const double colm1 = L.colamt[(int)T[swtab::ix1 + b] - 1], colm2 = L.colamt[(int)T[swtab::ix2 + b] - 1];
      const double speccomb = colm1 + T[swtab::strrat + b] * colm2;
      const double specmult = T[swtab::specwt + b] * fmin(kOneMinus, colm1 / speccomb);
      const int js = 1 + (int)specmult;
      const double fs = fmod(specmult, 1.0);
      const bool two = (jb == 17 || jb == 28);
      const double* ref = T + (two ? swtab::sfluxref02 : swtab::sfluxref03);
      const int nbin = two ? 5 : 9;
      for (int j = 0; j < ng; ++j) {
        const double r0 = ref[j + 16 * ((js - 1) + nbin * (ibd - 1))], r1 = ref[j + 16 * (js + nbin * (ibd - 1))];
        sf[j] = r0 + fs * (r1 - r0);
      }
    }
  }

  if (a.gas_only) return;
  // clear / cloudy column (RSM:1101-1125), in layer order on lane 0
  double zcf1 = 0.0;
  if (lane == 0) {
    double zcf0 = 1.0, z1 = 1.0;
    for (int k = 0; k < nlay; ++k) {
      const int r = a.top_at_1 ? nlay - 1 - k : k;
      const double cf = a.cf[(size_t)i + (size_t)a.ld * r];
      if (a.iovr == a.iovr_rand) {
        zcf0 = zcf0 * (1.0 - cf);
      } else if (a.iovr == a.iovr_maxrand) {
        if (cf > kFtiny) z1 = fmin(z1, 1.0 - cf);
        else if (z1 < 1.0) { zcf0 = zcf0 * z1; z1 = 1.0; }
      } else if (a.iovr >= 2) {
        zcf0 = fmin(zcf0, 1.0 - cf);
      }
    }
    if (a.iovr == a.iovr_maxrand) zcf0 = zcf0 * z1;
    if (zcf0 <= kFtiny) zcf0 = 0.0;
    if (zcf0 > kOneMinus) zcf0 = 1.0;
    zcf1 = 1.0 - zcf0;
    s.zcf1[pl] = zcf1;
    s.zcf0[pl] = zcf0;
    // McICA seed: ipsdsw0 + i or icseed(i) (RSM:875-883); grid-mean clouds draw none
    s.seed[pl] = (a.isubcsw == 2) ? a.icseed[i] : 1 + a.seed0 + j1;
  }
  zcf1 = __shfl_sync(0xffffffffu, zcf1, 0);
  for (int k = lane; k < nlay; k += 32) {
    const int r = a.top_at_1 ? nlay - 1 - k : k;
    const size_t x = (size_t)i + (size_t)a.ld * r;
    const double cf = a.cf[x];
    s.cldf[(size_t)pl + (size_t)nc * k] = (cf < kFtiny) ? 0.0 : cf;   // mcica_subcol input (RSM:1904-1908)
    if (a.isubcsw <= 0) {   // grid-mean clouds: cldfrc = cfrac / cf1 (RSM:1930-1934)
      s.aux[(size_t)pl + (size_t)nc * k] = (zcf1 > 0.0) ? cf / zcf1 : 0.0;
    } else if (a.iovr == 3) {   // fac_lcf between layers k-1 and k (RSM:2106-2108), dz in internal order
      double f = 0.0;
      if (k > 0) {
        const int r1 = a.top_at_1 ? nlay - k : k - 1;
        f = exp(-0.5 * (a.dz[x] + a.dz[(size_t)i + (size_t)a.ld * r1]) / a.delg[i]);
      }
      s.aux[(size_t)pl + (size_t)nc * k] = f;
    } else if (a.iovr == 4 || a.iovr == 5) {   // alpha, in the caller's row order (RSM:921, 1012)
      s.aux[(size_t)pl + (size_t)nc * k] = a.alpha[(size_t)i + (size_t)a.ld * k];
    }
    if (zcf1 > 0.0) {
      double* tw = s.taucw + ((size_t)pl * nlay + k) * 14;
      double* sw = s.ssacw + ((size_t)pl * nlay + k) * 14;
      double* gw = s.asycw + ((size_t)pl * nlay + k) * 14;
      cloud_layer(a, x, T, tw, sw, gw);
      a.cldtau[x] = tw[9];   // band 25 (RSM:1144-1152)
    }
  }
}

__global__ void __launch_bounds__(32 * kOptWarps, 3)   // 168 registers: twelve warps per SM hide the table gathers better than eight
sw_optics_kernel(SwArgs a, SwScratch s, int p0, int nc, const double* __restrict__ T) {
  __shared__ int s_jp[kOptWarps][kSwMaxLay];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int pl = blockIdx.x * kOptWarps + w;
  if (pl >= nc) return;   // whole warps only: no block barrier below
  const int j1 = a.idxday[p0 + pl];
  if (j1 < 1 || j1 > a.npts) {   // idxday outside 1..npts: skip the column, report
    if (lane == 0) atomicOr(s.bad, 1);
    return;
  }
  optics_body(a, s, pl, nc, j1, lane, s_jp[w], T);
}

// many physics blocks in one launch: daytime point p is column pts[p].y of block pts[p].x
__global__ void __launch_bounds__(32 * kOptWarps, 3)
sw_optics_blocks_kernel(const SwArgs* __restrict__ tab, const int2* __restrict__ pts, SwScratch s, int p0, int nc,
                        const double* __restrict__ T) {
  __shared__ int s_jp[kOptWarps][kSwMaxLay];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int pl = blockIdx.x * kOptWarps + w;
  if (pl >= nc) return;
  const int2 q = pts[p0 + pl];
  optics_body(tab[q.x], s, pl, nc, q.y, lane, s_jp[w], T);
}

// ---- kernel 3: transfer ------------------------------------------------------
struct LayOpt {
  double rb, rd, tb, td, e3, e4;
};

__device__ __forceinline__ double exp_tab(const double* __restrict__ ET, double z) {
  // itind = ftind*NTBMX + 0.5 with truncation; ftind in [0, 1) so the
  // clamped form of RSM:3601-3602 selects the same entry
  const double ftind = z / (kBpade + z);
  return __ldg(ET + (int)(ftind * kNtbmx + 0.5));
}
__device__ __forceinline__ double exp_small(double z) { return 1.0 - z + 0.5 * z * z; }

// the two-stream layer reflectance / transmittance of spcvrtm (RSM:3447-3600)
__device__ __forceinline__ void two_stream(double ztau0, double zssa0, double zasy0, double cosz, double sntz,
                                           int iswmode, const double* __restrict__ ET, LayOpt& o) {
  const double zcrit = 0.9999995, od_lo = 0.06, eps1 = 1.0e-8;
  const double zssaw = fmin(kOneMinus, zssa0 / ztau0);
  const double zasyw = zasy0 / fmax(kFtiny, zssa0);
  double za1 = zasyw * zasyw;
  double za2 = zssaw * za1;
  const double ztau1 = (1.0 - za2) * ztau0;
  const double zssa1 = (zssaw - za2) / (1.0 - za2);
  const double zasy1 = zasyw / (1.0 + zasyw);
  const double zasy3 = 0.75 * zasy1;
  double zgam1, zgam2, zgam3;
  if (iswmode == 1) {
    zgam1 = 1.75 - zssa1 * (1.0 + zasy3);
    zgam2 = -0.25 + zssa1 * (1.0 - zasy3);
    zgam3 = 0.5 - zasy3 * cosz;
  } else if (iswmode == 2) {
    zgam1 = 2.0 - zssa1 * (1.25 + zasy3);
    zgam2 = 0.75 * zssa1 * (1.0 - zasy1);
    zgam3 = 0.5 - zasy3 * cosz;
  } else {
    const double zsr3 = sqrt(3.0);
    zgam1 = zsr3 * (2.0 - zssa1 * (1.0 + zasy1)) * 0.5;
    zgam2 = zsr3 * zssa1 * (1.0 - zasy1) * 0.5;
    zgam3 = (1.0 - zsr3 * zasy1 * cosz) * 0.5;
  }
  const double zgam4 = 1.0 - zgam3;
  if (zssaw >= zcrit) {
    za1 = zgam1 * cosz - zgam3;
    za2 = zgam1 * ztau1;
    const double zb1 = fmin(ztau1 * sntz, 500.0);
    const double zb2 = (zb1 <= od_lo) ? exp_small(zb1) : exp_tab(ET, zb1);
    o.rb = fmax(0.0, fmin(1.0, (za2 - za1 * (1.0 - zb2)) / (1.0 + za2)));
    o.tb = fmax(0.0, fmin(1.0, 1.0 - o.rb));
    o.rd = fmax(0.0, fmin(1.0, za2 / (1.0 + za2)));
    o.td = fmax(0.0, fmin(1.0, 1.0 - o.rd));
  } else {
    za1 = zgam1 * zgam4 + zgam2 * zgam3;
    za2 = zgam1 * zgam3 + zgam2 * zgam4;
    double zrk = (zgam1 - zgam2) * (zgam1 + zgam2);
    zrk = (zrk > eps1) ? sqrt(zrk) : 0.0;
    const double zrk2 = zrk + zrk;
    const double zrp = zrk * cosz;
    const double zrp1 = 1.0 + zrp, zrm1 = 1.0 - zrp;
    const double zrpp1 = 1.0 - zrp * zrp;
    const double zrpp = copysign(fmax(kFlimit, fabs(zrpp1)), zrpp1);
    const double zrkg1 = zrk + zgam1, zrkg3 = zrk * zgam3, zrkg4 = zrk * zgam4;
    const double zr1 = zrm1 * (za2 + zrkg3);
    const double zr2 = zrp1 * (za2 - zrkg3);
    const double zr3 = zrk2 * (zgam3 - za2 * cosz);
    const double zr4 = zrpp * zrkg1;
    const double zr5 = zrpp * (zrk - zgam1);
    const double zt1 = zrp1 * (za1 + zrkg4);
    const double zt2 = zrm1 * (za1 - zrkg4);
    const double zt3 = zrk2 * (zgam4 + za1 * cosz);
    const double zb1 = fmin(zrk * ztau1, 500.0);
    const double zexm1 = (zb1 <= od_lo) ? exp_small(zb1) : exp_tab(ET, zb1);
    const double zexp1 = 1.0 / zexm1;
    const double zb2 = fmin(sntz * ztau1, 500.0);
    const double zexm2 = (zb2 <= od_lo) ? exp_small(zb2) : exp_tab(ET, zb2);
    const double zexp2 = 1.0 / zexm2;
    const double ze1r45 = zr4 * zexp1 + zr5 * zexm1;
    if (fabs(ze1r45) <= eps1) {
      o.rb = eps1;
      o.tb = zexm2;
    } else {
      const double zden1 = zssa1 / ze1r45;
      o.rb = fmax(0.0, fmin(1.0, (zr1 * zexp1 - zr2 * zexm1 - zr3 * zexm2) * zden1));
      o.tb = fmax(0.0, fmin(1.0, zexm2 * (1.0 - (zt1 * zexp1 - zt2 * zexm1 - zt3 * zexp2) * zden1)));
    }
    const double zden1 = (ze1r45 >= 0.0) ? zr4 / fmax(eps1, ze1r45 * zrkg1) : zr4 / fmin(-eps1, ze1r45 * zrkg1);
    o.rd = fmax(0.0, fmin(1.0, zgam2 * (zexp1 - zexm1) * zden1));
    o.td = fmax(0.0, fmin(1.0, zrk2 * zden1));
  }
  const double od_lo2 = 0.06;
  double zr = ztau1 * sntz;
  o.e3 = (zr <= od_lo2) ? exp_small(zr) : exp_tab(ET, zr);
  zr = ztau0 * sntz;
  o.e4 = (zr <= od_lo2) ? exp_small(zr) : exp_tab(ET, zr);
}

struct ColIn {
  const double* taug;   // row k at taug + k*112
  const double* taur;
  const double *aod, *ssa, *asy;   // caller arrays, (i, r, b)
  const double *tcw, *scw, *gcw;   // [k][14]
  const uint32_t* bits;            // this g-point's nw words (McICA)
  const double* cfr;               // normalised cloud fraction, layer k at cfr[k * cfs] (grid-mean)
  size_t cfs;
  size_t i;
  int ld, nlay, top_at_1, nw;
  double cosz, sntz;
  int iswmode;
};

__device__ __forceinline__ bool cloud_bit(const ColIn& c, int k) { return (c.bits[k >> 5] >> (k & 31)) & 1u; }
// the all-sky sweep treats layer k as cloudy: its McICA flag, or cldfrc > ftiny (RSM:2885)
template <bool GRID>
__device__ __forceinline__ bool cloudy_layer(const ColIn& c, int k) {
  return GRID ? (c.cfr[(size_t)k * c.cfs] > kFtiny) : cloud_bit(c, k);
}
// spcvrtc's mixing of a cloudy layer's optics with its clear optics o
// (RSM:3039-3042, 3057, 3072): zc0 * clear + zc1 * cloudy
__device__ __forceinline__ void mix_grid(const ColIn& c, int k, const LayOpt& o, LayOpt& w) {
  const double zc1 = c.cfr[(size_t)k * c.cfs], zc0 = 1.0 - zc1;
  w.rb = zc0 * o.rb + zc1 * w.rb;
  w.rd = zc0 * o.rd + zc1 * w.rd;
  w.tb = zc0 * o.tb + zc1 * w.tb;
  w.td = zc0 * o.td + zc1 * w.td;
  w.e3 = zc0 * o.e3 + zc1 * w.e3;
  w.e4 = zc0 * o.e4 + zc1 * w.e4;
}

// the inputs of layer k of g-point g (band b): gas, Rayleigh and aerosol
// optics, plus the cloud optics when the cloudy pass flags the layer
struct LayIn {
  double tr, tg, tae, sae, gae, tcw, scw, gcw;
  bool cld;
};
template <bool GRID>
__device__ __forceinline__ void layer_in(const ColIn& c, int g, int b, int k, bool cloudy_pass, LayIn& v) {
  const int r = c.top_at_1 ? c.nlay - 1 - k : k;
  const size_t xa = c.i + (size_t)c.ld * ((size_t)r + (size_t)c.nlay * b);
  v.tr = c.taur[(size_t)k * kSwNg + g];
  v.tg = c.taug[(size_t)k * kSwNg + g];
  v.tae = __ldg(c.aod + xa);
  v.sae = __ldg(c.ssa + xa);
  v.gae = __ldg(c.asy + xa);
  v.cld = cloudy_pass && cloudy_layer<GRID>(c, k);
  if (v.cld) {
    v.tcw = c.tcw[(size_t)k * 14 + b];
    v.scw = c.scw[(size_t)k * 14 + b];
    v.gcw = c.gcw[(size_t)k * 14 + b];
  }
}
// the layer's two-stream optics (RSM:3447-3449 clear, 3678-3680 cloudy)
__device__ __forceinline__ void layer_opt(const ColIn& c, const LayIn& v, const double* __restrict__ ET, LayOpt& o) {
  double ztau0 = fmax(kFtiny, v.tr + v.tg + v.tae);
  double zssa0 = v.tr + v.tae * v.sae;
  double zasy0 = v.gae * v.sae * v.tae;
  if (v.cld) {
    ztau0 = ztau0 + v.tcw;
    zssa0 = zssa0 + v.scw;
    zasy0 = zasy0 + v.gcw;
  }
  two_stream(ztau0, zssa0, zasy0, c.cosz, c.sntz, c.iswmode, ET, o);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kRtWarps = 4;   // GRID: isubcsw <= 0, spcvrtc's cloud-fraction mixing; else McICA flags
constexpr int kLaneVals = 10;   // per-lane stored values per level

// One column's transfer and outputs: a = the argument record of the call
// (or of the physics block) the column belongs to, j1 its 1-based column
// there, acc0 this warp's shared-memory slice.
template <bool GRID>
__device__ __forceinline__ void rt_body(const SwArgs& a, const SwScratch& s, int pl, int nc, int j1, int lane,
                                        double* acc0, const double* __restrict__ ET) {
  const int nlay = a.nlay, nlp1 = nlay + 1;
  const bool want_b = a.hswb != nullptr;
  double* acc = acc0;
  double *up0 = acc, *dn0 = acc + nlp1, *upc = acc + 2 * nlp1, *dnc = acc + 3 * nlp1;
  double* accb = acc + 4 * nlp1;   // [14][2][nlp1] total-sky band fluxes (hswb)
  for (int q = lane; q < (want_b ? 32 : 4) * nlp1; q += 32) acc[q] = 0.0;
  __syncwarp();

  const size_t i = (size_t)(j1 - 1);
  ColIn c;
  c.taug = s.taug + (size_t)pl * nlay * kSwNg;
  c.taur = s.taur + (size_t)pl * nlay * kSwNg;
  c.aod = a.aod; c.ssa = a.ssa; c.asy = a.asy;
  c.tcw = s.taucw + (size_t)pl * nlay * 14;
  c.scw = s.ssacw + (size_t)pl * nlay * 14;
  c.gcw = s.asycw + (size_t)pl * nlay * 14;
  c.i = i; c.ld = a.ld; c.nlay = nlay; c.top_at_1 = a.top_at_1; c.nw = s.nw;
  c.cosz = a.cosz[i];
  c.sntz = 1.0 / a.cosz[i];
  c.iswmode = a.iswmode;
  const double ssolar = a.s0fac * a.cosz[i];
  const double albbm[2] = {a.alb_nir_dir[i], a.alb_uvis_dir[i]};
  const double albdf[2] = {a.alb_nir_dif[i], a.alb_uvis_dif[i]};
  const double cf1 = s.zcf1[pl], cf0 = s.zcf0[pl];
  const bool cloudy = cf1 > kEps;
  c.cfr = s.aux + pl;
  c.cfs = (size_t)nc;
  // surface partition and UV-B sums of lane 0: [pass][bm1, bm2, df1, df2, uvb]
  double sfc[2][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};

  // per-lane storage in global scratch, [level][value][lane] per column
  // (values: 6 clear-sky layer optics, clear zrupb/zrupd, cloudy
  // zrupb/zrupd): a warp touches 256 contiguous bytes per value, and the
  // L2-only (.cg) accesses keep L1 for exp_tbl and the streamed optical depths
  double* lst = s.lane_store + (size_t)pl * (size_t)(nlay + 1) * kLaneVals * 32 + lane;
  auto st8 = [&](int k, int q, double v) { __stcg(lst + ((size_t)k * kLaneVals + q) * 32, v); };
  auto ld8 = [&](int k, int q) { return __ldcg(lst + ((size_t)k * kLaneVals + q) * 32); };

  for (int r0 = 0; r0 < kSwNg; r0 += 32) {
    const int g = r0 + lane;
    const bool valid = g < kSwNg;
    const int gg = valid ? g : kSwNg - 1;
    const int b = band_of(gg), ibd = c_idxsfc[b];
    const double zsolar = ssolar * s.sflux[(size_t)pl * kSwNg + gg];
    const double wgt = valid ? zsolar : 0.0;
    const int blo = band_of(r0), bhi = band_of(min(r0 + 31, kSwNg - 1));
    c.bits = s.bits + ((size_t)pl * kSwNg + gg) * s.nw;
    const double refb1 = ibd ? albbm[ibd - 1] : 0.5 * (albbm[0] + albbm[1]);
    const double refd1 = ibd ? albdf[ibd - 1] : 0.5 * (albdf[0] + albdf[1]);
    // The clear-sky sweep and, in a cloudy column, the all-sky sweep of
    // spcvrtm (RSM:3444-3667, 3668-3893) run side by side: a layer's clear
    // optics are evaluated once and serve both, and the all-sky sweep
    // re-evaluates only the layers its sub-column flags cloudy, as spcvrtm
    // keeps the clear-pass arrays for clear layers (RSM:3849-3850).
    // upward adding (vrtqdr, RSM:4011-4020)
    double ub = refb1, ud = refd1, ubw = refb1, udw = refd1;
    st8(0, 6, ub);
    st8(0, 7, ud);
    if (cloudy) {
      st8(0, 8, ubw);
      st8(0, 9, udw);
    }
    LayIn vin;
    layer_in<GRID>(c, gg, b, 0, cloudy, vin);
    for (int k = 0; k < nlay; ++k) {
      const LayIn cur = vin;
      if (k + 1 < nlay) layer_in<GRID>(c, gg, b, k + 1, cloudy, vin);   // issued ahead of this layer's arithmetic
      LayIn clr = cur;
      clr.cld = false;
      LayOpt o;
      layer_opt(c, clr, ET, o);
      st8(k, 0, o.rb); st8(k, 1, o.rd); st8(k, 2, o.tb); st8(k, 3, o.td); st8(k, 4, o.e3); st8(k, 5, o.e4);
      {
        const double zden1 = 1.0 / (1.0 - ud * o.rd);
        const double nb = o.rb + (o.td * ((o.tb - o.e3) * ud + o.e3 * ub)) * zden1;
        const double nd = o.rd + o.td * o.td * ud * zden1;
        ub = nb;
        ud = nd;
        st8(k + 1, 6, ub);
        st8(k + 1, 7, ud);
      }
      if (cloudy) {
        LayOpt w = o;
        if (cur.cld) {
          layer_opt(c, cur, ET, w);
          if (GRID) mix_grid(c, k, o, w);
        }
        const double zden1 = 1.0 / (1.0 - udw * w.rd);
        const double nb = w.rb + (w.td * ((w.tb - w.e3) * udw + w.e3 * ubw)) * zden1;
        const double nd = w.rd + w.td * w.td * udw * zden1;
        ubw = nb;
        udw = nd;
        st8(k + 1, 8, ubw);
        st8(k + 1, 9, udw);
      }
    }
    // downward sweep (RSM:4026-4040) with the fluxes of each level (RSM:4041-4046)
    auto fetch = [&](int m, LayOpt& o, LayOpt& w) {
      o.rb = ld8(m, 0); o.rd = ld8(m, 1); o.tb = ld8(m, 2); o.td = ld8(m, 3); o.e3 = ld8(m, 4); o.e4 = ld8(m, 5);
      w = o;
      if (cloudy && cloudy_layer<GRID>(c, m)) {
        LayIn v;
        layer_in<GRID>(c, gg, b, m, true, v);
        layer_opt(c, v, ET, w);
        if (GRID) mix_grid(c, m, o, w);
      }
    };
    // one downward step of a sweep: layer optics o, state (tdbt, tdn, rdnd, tdbt0)
    auto down = [&](int m, const LayOpt& o, double& tdbt, double& tdn, double& rdnd, double& tdbt0) {
      double tdn_m, rdnd_m;
      if (m == nlay - 1) {
        tdn_m = o.tb;
        rdnd_m = o.rd;
      } else {
        const double zden1 = 1.0 / (1.0 - o.rd * rdnd);
        tdn_m = tdbt * o.tb + (o.td * ((tdn - tdbt) + tdbt * o.rb * rdnd)) * zden1;
        rdnd_m = o.rd + o.td * o.td * rdnd * zden1;
      }
      tdbt = o.e3 * tdbt;
      tdbt0 = o.e4 * tdbt0;
      tdn = tdn_m;
      rdnd = rdnd_m;
    };
    auto flux = [&](double tdbt, double tdn, double rdnd, double rub, double rud, double& fu, double& fd) {
      const double zden1 = 1.0 / (1.0 - rdnd * rud);
      fu = (tdbt * rub + (tdn - tdbt) * rud) * zden1;
      fd = tdbt + (tdn - tdbt + tdbt * rub * rdnd) * zden1;
    };
    double tdbt = 1.0, tdn = 1.0, rdnd = 0.0, tdbt0 = 1.0, fd0 = 0.0;
    double tdbtw = 1.0, tdnw = 1.0, rdndw = 0.0, tdbt0w = 1.0, fd0w = 0.0;
    LayOpt nx, nxw;
    fetch(nlay - 1, nx, nxw);
    for (int m = nlay; m >= 0; --m) {
      if (m < nlay) {
        const LayOpt o = nx, w = nxw;
        if (m > 0) fetch(m - 1, nx, nxw);   // the next layer's loads overlap this layer's recurrences
        down(m, o, tdbt, tdn, rdnd, tdbt0);
        if (cloudy) down(m, w, tdbtw, tdnw, rdndw, tdbt0w);
      }
      double fu, fd, fuw = 0.0, fdw = 0.0;
      flux(tdbt, tdn, rdnd, ld8(m, 6), ld8(m, 7), fu, fd);
      if (cloudy) flux(tdbtw, tdnw, rdndw, ld8(m, 8), ld8(m, 9), fuw, fdw);
      if (m == 0) {
        fd0 = fd;
        fd0w = fdw;
      }
      const double su = warp_sum(wgt * fu), sd = warp_sum(wgt * fd);
      if (lane == 0) {
        up0[m] += su;
        dn0[m] += sd;
      }
      if (cloudy) {
        const double suw = warp_sum(wgt * fuw), sdw = warp_sum(wgt * fdw);
        if (lane == 0) {
          upc[m] += suw;
          dnc[m] += sdw;
        }
      }
      if (want_b) {   // total-sky band fluxes (spcvrtc: cf1 * all-sky + cf0 * clear, RSM:3160-3161)
        const double tu = cloudy ? (GRID ? cf1 * fuw + cf0 * fu : fuw) : fu;
        const double td = cloudy ? (GRID ? cf1 * fdw + cf0 * fd : fdw) : fd;
        for (int bb = blo; bb <= bhi; ++bb) {
          const double mu = warp_sum(b == bb ? wgt * tu : 0.0), md = warp_sum(b == bb ? wgt * td : 0.0);
          if (lane == 0) {
            accb[(size_t)(2 * bb) * nlp1 + m] += mu;
            accb[(size_t)(2 * bb + 1) * nlp1 + m] += md;
          }
        }
      }
    }
    // surface direct / diffuse partition (RSM:3641-3655) and UV-B (RSM:3907)
    for (int pass = 0; pass < (cloudy ? 2 : 1); ++pass) {
      const double t0 = pass ? tdbt0w : tdbt0, f0 = pass ? fd0w : fd0;
      const double zb1 = wgt * t0, zb2 = wgt * (f0 - t0);
      const double bm1 = (ibd == 1) ? zb1 : (ibd == 0 ? 0.5 * zb1 : 0.0);
      const double bm2 = (ibd == 2) ? zb1 : (ibd == 0 ? 0.5 * zb1 : 0.0);
      const double df1 = (ibd == 1) ? zb2 : (ibd == 0 ? 0.5 * zb2 : 0.0);
      const double df2 = (ibd == 2) ? zb2 : (ibd == 0 ? 0.5 * zb2 : 0.0);
      const double uv = (b == 27 - 16) ? wgt * f0 : 0.0;
      const double v[5] = {warp_sum(bm1), warp_sum(bm2), warp_sum(df1), warp_sum(df2), warp_sum(uv)};
      if (lane == 0)
        for (int q = 0; q < 5; ++q) sfc[pass][q] += v[q];
    }
  }
  __syncwarp();
  if (cloudy && GRID) {   // spcvrtc's total-sky fluxes (RSM:3158-3178)
    for (int m = lane; m < nlp1; m += 32) {
      upc[m] = cf1 * upc[m] + cf0 * up0[m];
      dnc[m] = cf1 * dnc[m] + cf0 * dn0[m];
    }
    if (lane == 0)
      for (int q = 0; q < 5; ++q) sfc[1][q] = cf1 * sfc[1][q] + cf0 * sfc[0][q];
    __syncwarp();
  }

  // outputs (RSM:1225-1373)
  const int ld = a.ld;
  const double* fu_t = cloudy ? upc : up0;
  const double* fd_t = cloudy ? dnc : dn0;
  auto row = [&](int m) { return a.top_at_1 ? nlay - 1 - m : m; };     // internal layer -> caller row
  auto lev = [&](int k) { return a.top_at_1 ? nlay - k : k; };         // internal level -> caller level
  for (int m = lane; m < nlay; m += 32) {
    const int r = row(m);
    const size_t x = i + (size_t)ld * r;
    const double rfdelp = a.heatfac / a.delp[x];
    a.hswc[x] = ((fd_t[m + 1] - fu_t[m + 1]) - (fd_t[m] - fu_t[m])) * rfdelp;
    if (a.hsw0) a.hsw0[x] = ((dn0[m + 1] - up0[m + 1]) - (dn0[m] - up0[m])) * rfdelp;
    if (want_b)
      for (int bb = 0; bb < 14; ++bb) {
        const double* bu = accb + (size_t)(2 * bb) * nlp1;
        const double* bd = accb + (size_t)(2 * bb + 1) * nlp1;
        a.hswb[i + (size_t)ld * ((size_t)r + (size_t)nlay * bb)] = ((bd[m + 1] - bu[m + 1]) - (bd[m] - bu[m])) * rfdelp;
      }
  }
  if (a.flxprf)
    for (int k = lane; k < nlp1; k += 32) {
      double* rec = a.flxprf + 4 * (i + (size_t)ld * lev(k));
      rec[0] = fu_t[k];
      rec[1] = fd_t[k];
      rec[2] = up0[k];
      rec[3] = dn0[k];
    }
  if (lane == 0) {
    const int t = cloudy ? 1 : 0;
    double* tf = a.topflx + 3 * i;
    tf[0] = fu_t[nlay];
    tf[1] = dn0[nlay];
    tf[2] = up0[nlay];
    double* sf = a.sfcflx + 4 * i;
    sf[0] = fu_t[0];
    sf[1] = fd_t[0];
    sf[2] = up0[0];
    sf[3] = dn0[0];
    if (a.fdncmp) {
      double* r = a.fdncmp + 6 * i;
      r[0] = sfc[t][4];
      r[1] = sfc[0][4];
      r[2] = sfc[t][0];
      r[3] = sfc[t][2];
      r[4] = sfc[t][1];
      r[5] = sfc[t][3];
    }
  }
}

template <bool GRID>
__global__ void __launch_bounds__(32 * kRtWarps, 4)   // 128 registers: sixteen warps per SM
sw_rt_kernel(SwArgs a, SwScratch s, int p0, int nc, const double* __restrict__ ET) {
  extern __shared__ double sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int pl = blockIdx.x * kRtWarps + w;
  if (pl >= nc) return;
  const int j1 = a.idxday[p0 + pl];
  if (j1 < 1 || j1 > a.npts) return;   // reported by the optics kernel
  rt_body<GRID>(a, s, pl, nc, j1, lane, sm + (size_t)w * rt_warp_doubles(a.nlay, a.hswb != nullptr), ET);
}

template <bool GRID>
__global__ void __launch_bounds__(32 * kRtWarps, 4)
sw_rt_blocks_kernel(const SwArgs* __restrict__ tab, const int2* __restrict__ pts, bool want_b, SwScratch s, int p0,
                    int nc, int nlay, const double* __restrict__ ET) {
  extern __shared__ double sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int pl = blockIdx.x * kRtWarps + w;
  if (pl >= nc) return;
  const int2 q = pts[p0 + pl];
  rt_body<GRID>(tab[q.x], s, pl, nc, q.y, lane, sm + (size_t)w * rt_warp_doubles(nlay, want_b), ET);
}

// Zeroes every output of every column of the physics blocks (RSM:824-845):
// column c of the concatenation is column c - colpre[b] of block b.
__global__ void sw_zero_blocks_kernel(const SwArgs* __restrict__ tab, const int* __restrict__ colpre, int nb,
                                      int total) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x) {
    int lo = 0, hi = nb - 1;   // last block with colpre[b] <= c
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (colpre[mid] <= c) lo = mid;
      else hi = mid - 1;
    }
    const SwArgs& a = tab[lo];
    const size_t i = (size_t)(c - colpre[lo]), ld = (size_t)a.ld, nlay = (size_t)a.nlay;
    for (size_t k = 0; k < nlay; ++k) {
      a.hswc[i + ld * k] = 0.0;
      a.cldtau[i + ld * k] = 0.0;
      if (a.hsw0) a.hsw0[i + ld * k] = 0.0;
      if (a.hswb)
        for (size_t b = 0; b < 14; ++b) a.hswb[i + ld * (k + nlay * b)] = 0.0;
    }
    if (a.flxprf)
      for (size_t k = 0; k <= nlay; ++k)
        for (int q = 0; q < 4; ++q) a.flxprf[4 * (i + ld * k) + q] = 0.0;
    for (int q = 0; q < 3; ++q) a.topflx[3 * i + q] = 0.0;
    for (int q = 0; q < 4; ++q) a.sfcflx[4 * i + q] = 0.0;
    if (a.fdncmp)
      for (int q = 0; q < 6; ++q) a.fdncmp[6 * i + q] = 0.0;
  }
}

// The daytime-point table of the physics blocks: point dayp[b] + p is column
// idxday_b[p] of block b; an index outside 1..npts_b sets *bad.
__global__ void sw_points_kernel(const SwArgs* __restrict__ tab, const int* __restrict__ dayp, int nb,
                                 int2* __restrict__ pts, int* bad) {
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= nb) return;
  const SwArgs& a = tab[b];
  for (int p = lane; p < dayp[b + 1] - dayp[b]; p += 32) {
    int j1 = a.idxday[p];
    if (j1 < 1 || j1 > a.npts) {
      atomicOr(bad, 1);
      j1 = 1;   // a valid column; the call reports the error
    }
    pts[dayp[b] + p] = make_int2(b, j1);
  }
}

// The per-layer overlap parameter of the sub-column generator for the stage
// entry point: fac_lcf between layers k-1 and k (iovr 3, RSM:2106-2108) or
// alpha (iovr 4, 5), [c + ldo*k]; inputs [c + ld*k], internal layer order.
__global__ void sw_overlap_aux_kernel(int ncols, int nlay, int ld, int iovr, const double* __restrict__ dz,
                                      const double* __restrict__ delg, const double* __restrict__ alpha,
                                      double* __restrict__ aux, int ldo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ncols * nlay) return;
  const int c = (int)(t % ncols), k = (int)(t / ncols);
  double v;
  if (iovr == 3)
    v = (k > 0) ? exp(-0.5 * (dz[c + (size_t)ld * k] + dz[c + (size_t)ld * (k - 1)]) / delg[c]) : 0.0;
  else
    v = alpha[c + (size_t)ld * k];
  aux[c + (size_t)ldo * k] = v;
}

cudaError_t overlap_aux_launch(int ncols, int nlay, int ld, int iovr, const double* dz, const double* delg,
                               const double* alpha, double* aux, int ldo, cudaStream_t st) {
  const long long n = (long long)ncols * nlay;
  if (n <= 0) return cudaSuccess;
  sw_overlap_aux_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ncols, nlay, ld, iovr, dz, delg, alpha, aux, ldo);
  return cudaGetLastError();
}

cudaError_t optics_launch(const SwArgs& a, const SwScratch& s, int p0, int nc, const double* T, cudaStream_t st) {
  if (nc <= 0) return cudaSuccess;
  const int grid = (nc + kOptWarps - 1) / kOptWarps;
  sw_optics_kernel<<<grid, 32 * kOptWarps, 0, st>>>(a, s, p0, nc, T);
  return cudaGetLastError();
}

size_t rt_smem_bytes(int nlay, bool hswb) { return (size_t)kRtWarps * rt_warp_doubles(nlay, hswb) * sizeof(double); }

cudaError_t rt_prepare(int max_smem) {
  cudaError_t e = cudaFuncSetAttribute(sw_rt_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sw_rt_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sw_rt_blocks_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sw_rt_blocks_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  return e;
}

cudaError_t blocks_prepare(const SwArgs* tab, const int* colpre, const int* dayp, int nb, int total_cols,
                           int2* pts, int* bad, cudaStream_t st) {
  sw_points_kernel<<<(nb + 7) / 8, 256, 0, st>>>(tab, dayp, nb, pts, bad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || total_cols <= 0) return e;
  sw_zero_blocks_kernel<<<min((total_cols + 127) / 128, 4096), 128, 0, st>>>(tab, colpre, nb, total_cols);
  return cudaGetLastError();
}

cudaError_t optics_blocks_launch(const SwArgs* tab, const int2* pts, const SwScratch& s, int p0, int nc,
                                 const double* T, cudaStream_t st) {
  if (nc <= 0) return cudaSuccess;
  sw_optics_blocks_kernel<<<(nc + kOptWarps - 1) / kOptWarps, 32 * kOptWarps, 0, st>>>(tab, pts, s, p0, nc, T);
  return cudaGetLastError();
}

cudaError_t rt_blocks_launch(const SwArgs* tab, const int2* pts, bool grid, bool want_b, const SwScratch& s, int p0,
                             int nc, int nlay, const double* ET, cudaStream_t st) {
  if (nc <= 0) return cudaSuccess;
  const int g = (nc + kRtWarps - 1) / kRtWarps;
  const size_t smem = rt_smem_bytes(nlay, want_b);
  if (grid) sw_rt_blocks_kernel<true><<<g, 32 * kRtWarps, smem, st>>>(tab, pts, want_b, s, p0, nc, nlay, ET);
  else sw_rt_blocks_kernel<false><<<g, 32 * kRtWarps, smem, st>>>(tab, pts, want_b, s, p0, nc, nlay, ET);
  return cudaGetLastError();
}

cudaError_t rt_launch(const SwArgs& a, const SwScratch& s, int p0, int nc, const double* ET, cudaStream_t st) {
  if (nc <= 0) return cudaSuccess;
  const int grid = (nc + kRtWarps - 1) / kRtWarps;
  const size_t smem = rt_smem_bytes(a.nlay, a.hswb != nullptr);
  if (a.isubcsw <= 0) sw_rt_kernel<true><<<grid, 32 * kRtWarps, smem, st>>>(a, s, p0, nc, ET);
  else sw_rt_kernel<false><<<grid, 32 * kRtWarps, smem, st>>>(a, s, p0, nc, ET);
  return cudaGetLastError();
}

}  // namespace sw
