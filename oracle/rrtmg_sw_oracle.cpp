// rrtmg_sw_oracle.cpp -- CPU restatement of the RRTMG-SW column path.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only the tests, the smoke check and
// bench.py's CPU-baseline / reference arm may load this library.  It is the
// parity checker for the GPU shortwave path and its timed CPU baseline.
//
// It restates, statement by statement and in the same floating-point order,
// the Fortran of ccpp-physics physics/Radiation/RRTMG/radsw_main.F90 (RSM):
//     rrtmg_sw_run driver      RSM:493-1379
//     rswinit                  RSM:1388-1536
//     cldprop                  RSM:1566-1938
//     mcica_subcol             RSM:1952-2212
//     setcoef                  RSM:2242-2389
//     spcvrtm                  RSM:3228-3942
//     vrtqdr                   RSM:3959-4051
//     taumol, taumol16..29     RSM:4094-5573
// with the Mersenne twister of physics/Radiation/mersenne_twister.f
// (random_setseed_t :285-299, random_number_t :330-372) and the band layout
// of physics/Radiation/RRTMG/radsw_param.f.  Arithmetic is IEEE binary64 with
// FMA contraction disabled, Fortran int() = truncation toward zero,
// mod(x,1.) = fmod; literals are binary64 (promoted-real build).
//
//     spcvrtc (isubcsw <= 0)   RSM:2432-3183, as spcvrtm's grid-mean mode
//
// and the CCPP schemes either side of the run:
//     rad_sw_pre_run           physics/Radiation/RRTMG/rad_sw_pre.F90:14-51
//     rrtmg_sw_post_run        physics/Radiation/RRTMG/rrtmg_sw_post.F90:13-129
//
// Parity of this restatement is NOT pinned by the reference: the reference is
// Fortran, no Fortran compiler exists in this environment, and the reference
// tree holds no tests or golden vectors for this path.  The coefficient
// tables come from the blob written by
// ccpp_physics_b200/data/extract_sw_tables.py (radsw_datatb.f DATA).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../include/rrtmg_sw_gpu.h"
#include "../ccpp_physics_b200/data/rrtmg_sw_table_layout.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- constants (RSM:335-350; physcons.F90) --------------------------------
const double con_g = 9.80665, con_cp = 1.0046e+3, con_avgd = 6.0221415e23;
const double con_amd = 28.9644, con_amw = 18.0154, con_amo3 = 47.9982;
const double eps = 1.0e-6, oneminus = 1.0 - eps, bpade = 1.0 / 0.278;
const double stpfac = 296.0 / 1013.0, ftiny = 1.0e-12, flimit = 1.0e-20;
const double s0 = 1368.22, f_zero = 0.0, f_one = 1.0;
const double amdw = con_amd / con_amw, amdo3 = con_amd / con_amo3;

const int NBLOW = 16, NBHGH = 29, NBDSW = 14, NGPT = 112, NTBMX = 10000;
const int NG[14] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};     // radsw_param.f NG16..NG29
const int NSPA[14] = {9, 9, 9, 9, 1, 9, 9, 1, 9, 1, 0, 1, 9, 1};       // RSM:359
const int NSPB[14] = {1, 5, 1, 1, 1, 5, 1, 0, 1, 0, 0, 1, 5, 1};       // RSM:360
const int IDXSFC[14] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 2, 2, 2, 2, 1};     // RSM:362
const int IDXEBC[14] = {5, 5, 4, 4, 3, 3, 2, 2, 1, 1, 1, 1, 1, 5};     // RSM:363
const int MFR[14] = {3, 4, 3, 3, 4, 4, 3, 3, 3, 0, 0, 0, 0, 4};        // forref rows per band
const int NUVB = 27;

std::vector<double> T;
double heatfac = 0.0;
double exp_tbl[NTBMX + 1];
bool g_init = false;
int NS[14], NGB[NGPT];

void set_err(char* m, int n, const std::string& s) {
  if (!m || n <= 0) return;
  std::snprintf(m, (size_t)n, "%s", s.c_str());
}

// table accessors (Fortran subscripts)
inline double preflog(int jp) { return T[swtab::preflog + jp - 1]; }
inline double tref(int jp) { return T[swtab::tref + jp - 1]; }
inline double tab2(int off, int rows, int i, int ib) { return T[off + (i - 1) + rows * (ib - NBLOW)]; }
inline double tab1b(int off, int ib) { return T[off + ib - NBLOW]; }          // (nblow:nbhgh)
inline int itab1b(int off, int ib) { return (int)T[off + ib - NBLOW]; }
inline double sflux01(int j, int ibd) { return T[swtab::sfluxref01 + (j - 1) + 16 * (ibd - 1)]; }
inline double sflux02(int j, int js, int ibd) { return T[swtab::sfluxref02 + (j - 1) + 16 * ((js - 1) + 5 * (ibd - 1))]; }
inline double sflux03(int j, int js, int ibd) { return T[swtab::sfluxref03 + (j - 1) + 16 * ((js - 1) + 9 * (ibd - 1))]; }

// per-band k-distribution tables, absa(ind, j) etc. with Fortran subscripts
struct BandTab { int absa, absb, selfref, forref, msa, msb, mfr; };
BandTab band_tab(int jb) {
  BandTab b{-1, -1, -1, -1, 0, 0, 0};
  const int i = jb - NBLOW;
  b.msa = NSPA[i] == 9 ? 585 : 65;
  b.msb = NSPB[i] == 5 ? 1175 : 235;
  b.mfr = MFR[i];
  switch (jb) {
#define BT(N) case N: b.absa = swtab::b##N##_absa; b.selfref = swtab::b##N##_selfref; b.forref = swtab::b##N##_forref; break;
    BT(23)
#undef BT
#define BT(N) case N: b.absa = swtab::b##N##_absa; b.absb = swtab::b##N##_absb; b.selfref = swtab::b##N##_selfref; b.forref = swtab::b##N##_forref; break;
    BT(16) BT(17) BT(18) BT(19) BT(20) BT(21) BT(22) BT(24) BT(29)
#undef BT
    case 25: b.absa = swtab::b25_absa; break;
    case 27: b.absa = swtab::b27_absa; b.absb = swtab::b27_absb; break;
    case 28: b.absa = swtab::b28_absa; b.absb = swtab::b28_absb; break;
    default: break;
  }
  return b;
}

// ---- Mersenne twister (mersenne_twister.f:162-372) ------------------------
struct MTState { uint32_t mt[624]; int mti; };
const uint32_t MATA = 0x9908B0DFu, UMASK = 0x80000000u, LMASK = 0x7FFFFFFFu;
const uint32_t TMASKB = 0x9D2C5680u, TMASKC = 0xEFC60000u;
void mt_setseed(MTState& s, int32_t inseed) {            // random_setseed_t (MT:285-299)
  int32_t ii = inseed == 0 ? 4357 : inseed;
  s.mti = 624;
  s.mt[0] = (uint32_t)ii;
  for (int i = 1; i < 624; ++i) s.mt[i] = 69069u * s.mt[i - 1];
}
inline uint32_t mt_mag(uint32_t y) { return (y & 1u) ? MATA : 0u; }
double mt_next(MTState& s) {                              // random_number_t (MT:330-372)
  if (s.mti >= 624) {
    int kk;
    for (kk = 0; kk < 624 - 397; ++kk) {
      uint32_t y = (s.mt[kk] & UMASK) | (s.mt[kk + 1] & LMASK);
      s.mt[kk] = s.mt[kk + 397] ^ (y >> 1) ^ mt_mag(y);
    }
    for (; kk < 623; ++kk) {
      uint32_t y = (s.mt[kk] & UMASK) | (s.mt[kk + 1] & LMASK);
      s.mt[kk] = s.mt[kk + (397 - 624)] ^ (y >> 1) ^ mt_mag(y);
    }
    uint32_t y = (s.mt[623] & UMASK) | (s.mt[0] & LMASK);
    s.mt[623] = s.mt[396] ^ (y >> 1) ^ mt_mag(y);
    s.mti = 0;
  }
  uint32_t y = s.mt[s.mti++];
  y ^= y >> 11;
  y ^= (y << 7) & TMASKB;
  y ^= (y << 15) & TMASKC;
  y ^= y >> 18;
  return (double)y / 4294967295.0;
}

// ---- mcica_subcol (RSM:1952-2212); lcloudy(k, n) at lc[(n-1)*nlay + k-1] --
void mcica_subcol(int nlay, const double* cldf, int ipseed, const double* dz, double de_lgth,
                  const double* alpha, int iovr, std::vector<char>& lc) {
  MTState st;
  mt_setseed(st, ipseed);
  std::vector<double> cdf((size_t)nlay * NGPT), cd2;
  auto CDF = [&](int k, int n) -> double& { return cdf[(size_t)(n - 1) * nlay + (k - 1)]; };
  auto CD2 = [&](int k, int n) -> double& { return cd2[(size_t)(n - 1) * nlay + (k - 1)]; };
  if (iovr == 0 || iovr == 1) {
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 1; k <= nlay; ++k) CDF(k, n) = mt_next(st);
    if (iovr == 1) {
      for (int k = 2; k <= nlay; ++k) {
        const int k1 = k - 1;
        const double tem1 = f_one - cldf[k1 - 1];
        for (int n = 1; n <= NGPT; ++n) {
          if (CDF(k1, n) > tem1) CDF(k, n) = CDF(k1, n);
          else CDF(k, n) = CDF(k, n) * tem1;
        }
      }
    }
  } else if (iovr == 2) {
    double r1[NGPT];
    for (int n = 0; n < NGPT; ++n) r1[n] = mt_next(st);
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 1; k <= nlay; ++k) CDF(k, n) = r1[n - 1];
  } else if (iovr == 3) {
    std::vector<double> fac((size_t)nlay + 1, 0.0);
    for (int k = nlay; k >= 2; --k) fac[k] = std::exp(-0.5 * (dz[k - 1] + dz[k - 2]) / de_lgth);
    cd2.resize(cdf.size());
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 1; k <= nlay; ++k) CDF(k, n) = mt_next(st);
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 1; k <= nlay; ++k) CD2(k, n) = mt_next(st);
    for (int n = 1; n <= NGPT; ++n)
      for (int k = nlay - 1; k >= 1; --k)
        if (CD2(k, n) <= fac[k + 1]) CDF(k, n) = CDF(k + 1, n);
  } else {   // 4, 5
    cd2.resize(cdf.size());
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 1; k <= nlay; ++k) CDF(k, n) = mt_next(st);
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 1; k <= nlay; ++k) CD2(k, n) = mt_next(st);
    for (int n = 1; n <= NGPT; ++n)
      for (int k = 2; k <= nlay; ++k)
        if (CD2(k, n) < alpha[k - 1]) CDF(k, n) = CDF(k - 1, n);
  }
  lc.assign((size_t)nlay * NGPT, 0);
  for (int k = 1; k <= nlay; ++k) {
    const double tem1 = f_one - cldf[k - 1];
    for (int n = 1; n <= NGPT; ++n) lc[(size_t)(n - 1) * nlay + (k - 1)] = CDF(k, n) >= tem1;
  }
}

// ---- per-column work arrays (1-based access helpers) ----------------------
struct Col {
  int nlay;
  std::vector<double> pavel, tavel, delp, dz, alph, h2ovmr, o3vmr, coldry, temcol, colmol, colamt;
  std::vector<double> cfrac, cliqp, reliq, cicep, reice, cdat1, cdat2, cdat3, cdat4, cldfrc;
  std::vector<double> taucw, ssacw, asycw, tauae, ssaae, asyae, cldfmc;
  std::vector<double> fac00, fac01, fac10, fac11, forfac, forfrac, selffac, selffrac;
  std::vector<int> jp, jt, jt1, indfor, indself;
  std::vector<double> taug, taur, sfluxzen;
  std::vector<double> fxupc, fxdnc, fxup0, fxdn0;
  explicit Col(int n) : nlay(n) {
    for (auto* v : {&pavel, &tavel, &delp, &dz, &alph, &h2ovmr, &o3vmr, &coldry, &temcol, &colmol, &cfrac,
                    &cliqp, &reliq, &cicep, &reice, &cdat1, &cdat2, &cdat3, &cdat4, &cldfrc, &fac00, &fac01, &fac10,
                    &fac11, &forfac, &forfrac, &selffac, &selffrac})
      v->assign(n + 1, 0.0);
    colamt.assign((size_t)(n + 1) * 8, 0.0);
    for (auto* v : {&taucw, &ssacw, &asycw, &tauae, &ssaae, &asyae}) v->assign((size_t)(n + 1) * NBDSW, 0.0);
    cldfmc.assign((size_t)(n + 1) * NGPT, 0.0);
    for (auto* v : {&jp, &jt, &jt1, &indfor, &indself}) v->assign(n + 1, 0);
    taug.assign((size_t)(n + 1) * NGPT, 0.0);
    taur.assign((size_t)(n + 1) * NGPT, 0.0);
    sfluxzen.assign(NGPT, 0.0);
    for (auto* v : {&fxupc, &fxdnc, &fxup0, &fxdn0}) v->assign((size_t)(n + 2) * NBDSW, 0.0);
  }
  double& COLAMT(int k, int m) { return colamt[(size_t)(m - 1) * (nlay + 1) + k]; }
  double& TAUCW(int k, int ib) { return taucw[(size_t)(ib - 1) * (nlay + 1) + k]; }
  double& SSACW(int k, int ib) { return ssacw[(size_t)(ib - 1) * (nlay + 1) + k]; }
  double& ASYCW(int k, int ib) { return asycw[(size_t)(ib - 1) * (nlay + 1) + k]; }
  double& TAUAE(int k, int ib) { return tauae[(size_t)(ib - 1) * (nlay + 1) + k]; }
  double& SSAAE(int k, int ib) { return ssaae[(size_t)(ib - 1) * (nlay + 1) + k]; }
  double& ASYAE(int k, int ib) { return asyae[(size_t)(ib - 1) * (nlay + 1) + k]; }
  double& CLDFMC(int k, int g) { return cldfmc[(size_t)(g - 1) * (nlay + 1) + k]; }
  double& TAUG(int k, int g) { return taug[(size_t)(g - 1) * (nlay + 1) + k]; }
  double& TAUR(int k, int g) { return taur[(size_t)(g - 1) * (nlay + 1) + k]; }
  double& FXUPC(int k, int ib) { return fxupc[(size_t)(ib - 1) * (nlay + 2) + k]; }
  double& FXDNC(int k, int ib) { return fxdnc[(size_t)(ib - 1) * (nlay + 2) + k]; }
  double& FXUP0(int k, int ib) { return fxup0[(size_t)(ib - 1) * (nlay + 2) + k]; }
  double& FXDN0(int k, int ib) { return fxdn0[(size_t)(ib - 1) * (nlay + 2) + k]; }
};

// ---- cldprop (RSM:1566-1938) ----------------------------------------------
void cldprop(Col& c, int ipseed, double delgth, int iswcliq, int iswcice, int isubcsw, int iovr, double cf1) {
  const int nlay = c.nlay;
  for (int ib = 1; ib <= NBDSW; ++ib)
    for (int k = 1; k <= nlay; ++k) { c.TAUCW(k, ib) = f_zero; c.SSACW(k, ib) = f_one; c.ASYCW(k, ib) = f_zero; }
  double tauliq[14] = {}, tauice[14] = {}, ssaliq[14] = {}, ssaice[14] = {}, ssaran[14] = {}, ssasnw[14] = {},
         asyliq[14] = {}, asyice[14] = {}, asyran[14] = {}, asysnw[14] = {};
  if (iswcliq > 0) {
    for (int k = 1; k <= nlay; ++k) {
      if (!(c.cfrac[k] > ftiny)) continue;
      const double cldran = c.cdat1[k], cldsnw = c.cdat3[k], refsnw = c.cdat4[k];
      const double dgesnw = 1.0315 * refsnw;
      const double tauran = cldran * T[swtab::a0r];
      double tausnw;
      if (cldsnw > f_zero && refsnw > 10.0) tausnw = cldsnw * 1.09087 * (T[swtab::a0s] + T[swtab::a1s] / dgesnw);
      else tausnw = f_zero;
      for (int ib = NBLOW; ib <= NBHGH; ++ib) {
        const int j = ib - NBLOW;
        ssaran[j] = tauran * (f_one - tab1b(swtab::b0r, ib));
        ssasnw[j] = tausnw * (f_one - (tab1b(swtab::b0s, ib) + tab1b(swtab::b1s, ib) * dgesnw));
        asyran[j] = ssaran[j] * tab1b(swtab::c0r, ib);
        asysnw[j] = ssasnw[j] * tab1b(swtab::c0s, ib);
      }
      const double cldliq = c.cliqp[k], cldice = c.cicep[k], refliq = c.reliq[k];
      double refice = c.reice[k];
      if (cldliq <= f_zero) {
        for (int j = 0; j < 14; ++j) tauliq[j] = ssaliq[j] = asyliq[j] = f_zero;
      } else {
        const double factor = refliq - 1.5;
        const int index = std::max(1, std::min(57, (int)factor));
        const double fint = factor - (double)index;
        const int oe = iswcliq == 1 ? swtab::extliq1 : swtab::extliq2;
        const int os = iswcliq == 1 ? swtab::ssaliq1 : swtab::ssaliq2;
        const int oa = iswcliq == 1 ? swtab::asyliq1 : swtab::asyliq2;
        if (iswcliq == 1 || iswcliq == 2) {
          for (int ib = NBLOW; ib <= NBHGH; ++ib) {
            const int j = ib - NBLOW;
            const double extcoliq = std::max(f_zero, tab2(oe, 58, index, ib) +
                                                         fint * (tab2(oe, 58, index + 1, ib) - tab2(oe, 58, index, ib)));
            const double ssacoliq = std::max(f_zero, std::min(f_one, tab2(os, 58, index, ib) +
                                                         fint * (tab2(os, 58, index + 1, ib) - tab2(os, 58, index, ib))));
            const double asycoliq = std::max(f_zero, std::min(f_one, tab2(oa, 58, index, ib) +
                                                         fint * (tab2(oa, 58, index + 1, ib) - tab2(oa, 58, index, ib))));
            tauliq[j] = cldliq * extcoliq;
            ssaliq[j] = tauliq[j] * ssacoliq;
            asyliq[j] = ssaliq[j] * asycoliq;
          }
        }
      }
      if (cldice <= f_zero) {
        for (int j = 0; j < 14; ++j) tauice[j] = ssaice[j] = asyice[j] = f_zero;
      } else if (iswcice == 1) {
        refice = std::min(130.0, std::max(13.0, refice));
        for (int ib = NBLOW; ib <= NBHGH; ++ib) {
          const int j = ib - NBLOW, ia = IDXEBC[j];
          const double extcoice = std::max(f_zero, T[swtab::abari + ia - 1] + T[swtab::bbari + ia - 1] / refice);
          const double ssacoice = std::max(f_zero, std::min(f_one, f_one - T[swtab::cbari + ia - 1] -
                                                                       T[swtab::dbari + ia - 1] * refice));
          const double asycoice = std::max(f_zero, std::min(f_one, T[swtab::ebari + ia - 1] +
                                                                       T[swtab::fbari + ia - 1] * refice));
          tauice[j] = cldice * extcoice;
          ssaice[j] = tauice[j] * ssacoice;
          asyice[j] = ssaice[j] * asycoice;
        }
      } else if (iswcice == 2 || iswcice == 3) {
        int index, rows, oe, os, oa;
        double fint;
        if (iswcice == 2) {
          refice = std::min(131.0, std::max(5.0, refice));
          const double factor = (refice - 2.0) / 3.0;
          index = std::max(1, std::min(42, (int)factor));
          fint = factor - (double)index;
          rows = 43; oe = swtab::extice2; os = swtab::ssaice2; oa = swtab::asyice2;
        } else {
          const double dgeice = std::max(5.0, std::min(140.0, 1.0315 * refice));
          const double factor = (dgeice - 2.0) / 3.0;
          index = std::max(1, std::min(45, (int)factor));
          fint = factor - (double)index;
          rows = 46; oe = swtab::extice3; os = swtab::ssaice3; oa = swtab::asyice3;
        }
        for (int ib = NBLOW; ib <= NBHGH; ++ib) {
          const int j = ib - NBLOW;
          const double extcoice = std::max(f_zero, tab2(oe, rows, index, ib) +
                                                       fint * (tab2(oe, rows, index + 1, ib) - tab2(oe, rows, index, ib)));
          const double ssacoice = std::max(f_zero, std::min(f_one, tab2(os, rows, index, ib) +
                                                       fint * (tab2(os, rows, index + 1, ib) - tab2(os, rows, index, ib))));
          const double asycoice = std::max(f_zero, std::min(f_one, tab2(oa, rows, index, ib) +
                                                       fint * (tab2(oa, rows, index + 1, ib) - tab2(oa, rows, index, ib))));
          tauice[j] = cldice * extcoice;
          ssaice[j] = tauice[j] * ssacoice;
          asyice[j] = ssaice[j] * asycoice;
        }
      }
      for (int ib = 1; ib <= NBDSW; ++ib) {
        const int j = ib - 1;
        c.TAUCW(k, ib) = tauliq[j] + tauice[j] + tauran + tausnw;
        c.SSACW(k, ib) = ssaliq[j] + ssaice[j] + ssaran[j] + ssasnw[j];
        c.ASYCW(k, ib) = asyliq[j] + asyice[j] + asyran[j] + asysnw[j];
      }
    }
  } else {
    for (int k = 1; k <= nlay; ++k)
      if (c.cfrac[k] > ftiny)
        for (int ib = 1; ib <= NBDSW; ++ib) {
          c.TAUCW(k, ib) = c.cdat1[k];
          c.SSACW(k, ib) = c.cdat1[k] * c.cdat2[k];
          c.ASYCW(k, ib) = c.SSACW(k, ib) * c.cdat3[k];
        }
  }
  if (isubcsw > 0) {
    std::vector<double> cldf(nlay), dz(nlay), al(nlay);
    for (int k = 1; k <= nlay; ++k) {
      cldf[k - 1] = c.cfrac[k] < ftiny ? f_zero : c.cfrac[k];
      dz[k - 1] = c.dz[k];
      al[k - 1] = c.alph[k];
    }
    std::vector<char> lc;
    mcica_subcol(nlay, cldf.data(), ipseed, dz.data(), delgth, al.data(), iovr, lc);
    for (int ig = 1; ig <= NGPT; ++ig)
      for (int k = 1; k <= nlay; ++k) c.CLDFMC(k, ig) = lc[(size_t)(ig - 1) * nlay + (k - 1)] ? f_one : f_zero;
  } else {   // non-McICA: normalised cloud fraction (RSM:1930-1934)
    for (int k = 1; k <= nlay; ++k) c.cldfrc[k] = c.cfrac[k] / cf1;
  }
}

// ---- setcoef (RSM:2242-2389) ----------------------------------------------
int setcoef(Col& c) {
  const int nlay = c.nlay;
  int laytrop = nlay;
  for (int k = 1; k <= nlay; ++k) {
    c.forfac[k] = c.pavel[k] * stpfac / (c.tavel[k] * (f_one + c.h2ovmr[k]));
    const double plog = std::log(c.pavel[k]);
    c.jp[k] = std::max(1, std::min(58, (int)(36.0 - 5.0 * (plog + 0.04))));
    const int jp1 = c.jp[k] + 1;
    const double fp = 5.0 * (preflog(c.jp[k]) - plog);
    double tem1 = (c.tavel[k] - tref(c.jp[k])) / 15.0;
    double tem2 = (c.tavel[k] - tref(jp1)) / 15.0;
    c.jt[k] = std::max(1, std::min(4, (int)(3.0 + tem1)));
    c.jt1[k] = std::max(1, std::min(4, (int)(3.0 + tem2)));
    const double ft = tem1 - (double)(c.jt[k] - 3);
    const double ft1 = tem2 - (double)(c.jt1[k] - 3);
    const double fp1 = f_one - fp;
    c.fac10[k] = fp1 * ft;
    c.fac00[k] = fp1 * (f_one - ft);
    c.fac11[k] = fp * ft1;
    c.fac01[k] = fp * (f_one - ft1);
    if (plog > 4.56) {
      laytrop = k;
      tem1 = (332.0 - c.tavel[k]) / 36.0;
      c.indfor[k] = std::min(2, std::max(1, (int)tem1));
      c.forfrac[k] = tem1 - (double)c.indfor[k];
      tem2 = (c.tavel[k] - 188.0) / 7.2;
      c.indself[k] = std::min(9, std::max(1, (int)tem2 - 7));
      c.selffrac[k] = tem2 - (double)(c.indself[k] + 7);
      c.selffac[k] = c.h2ovmr[k] * c.forfac[k];
    } else {
      tem1 = (c.tavel[k] - 188.0) / 36.0;
      c.indfor[k] = 3;
      c.forfrac[k] = tem1 - f_one;
      c.indself[k] = 0;
      c.selffrac[k] = f_zero;
      c.selffac[k] = f_zero;
    }
  }
  return laytrop;
}

// ---- taumol (RSM:4094-5573) -----------------------------------------------
void taumol(Col& c, int laytrop) {
  const int nlay = c.nlay;
  std::vector<int> id0((size_t)(nlay + 1) * 14), id1((size_t)(nlay + 1) * 14);
  auto ID0 = [&](int k, int jb) -> int& { return id0[(size_t)(jb - NBLOW) * (nlay + 1) + k]; };
  auto ID1 = [&](int k, int jb) -> int& { return id1[(size_t)(jb - NBLOW) * (nlay + 1) + k]; };
  for (int jb = NBLOW; jb <= NBHGH; ++jb) {
    const int i = jb - NBLOW;
    for (int k = 1; k <= laytrop; ++k) {
      ID0(k, jb) = ((c.jp[k] - 1) * 5 + (c.jt[k] - 1)) * NSPA[i];
      ID1(k, jb) = (c.jp[k] * 5 + (c.jt1[k] - 1)) * NSPA[i];
    }
    for (int k = laytrop + 1; k <= nlay; ++k) {
      ID0(k, jb) = ((c.jp[k] - 13) * 5 + (c.jt[k] - 1)) * NSPB[i];
      ID1(k, jb) = ((c.jp[k] - 12) * 5 + (c.jt1[k] - 1)) * NSPB[i];
    }
    const int ibd = itab1b(swtab::ibx, jb), njb = NG[i], ns = NS[i];
    if (jb == 16 || jb == 20 || jb == 23 || jb == 25 || jb == 26 || jb == 29) {
      for (int j = 1; j <= njb; ++j) c.sfluxzen[ns + j - 1] = sflux01(j, ibd);
    } else if (jb == 27) {
      for (int j = 1; j <= njb; ++j) c.sfluxzen[ns + j - 1] = T[swtab::scalekur] * sflux01(j, ibd);
    } else {
      const int lref = itab1b(swtab::layreffr, jb);
      int ks;
      if (jb == 17 || jb == 28) {
        ks = nlay;
        for (int k = laytrop; k <= nlay - 1; ++k)
          if (c.jp[k] < lref && c.jp[k + 1] >= lref) { ks = k + 1; break; }
      } else {
        ks = laytrop;
        for (int k = 1; k <= laytrop - 1; ++k)
          if (c.jp[k] < lref && c.jp[k + 1] >= lref) { ks = k + 1; break; }
      }
      const double colm1 = c.COLAMT(ks, itab1b(swtab::ix1, jb));
      const double colm2 = c.COLAMT(ks, itab1b(swtab::ix2, jb));
      const double speccomb = colm1 + tab1b(swtab::strrat, jb) * colm2;
      const double specmult = tab1b(swtab::specwt, jb) * std::min(oneminus, colm1 / speccomb);
      const int js = 1 + (int)specmult;
      const double fs = std::fmod(specmult, f_one);
      for (int j = 1; j <= njb; ++j) {
        if (jb == 17 || jb == 28)
          c.sfluxzen[ns + j - 1] = sflux02(j, js, ibd) + fs * (sflux02(j, js + 1, ibd) - sflux02(j, js, ibd));
        else
          c.sfluxzen[ns + j - 1] = sflux03(j, js, ibd) + fs * (sflux03(j, js + 1, ibd) - sflux03(j, js, ibd));
      }
    }
  }

  for (int jb = NBLOW; jb <= NBHGH; ++jb) {
    const int i = jb - NBLOW, ngb = NG[i], ns = NS[i];
    const BandTab bt = band_tab(jb);
    auto absa = [&](int ind, int j) { return T[bt.absa + (ind - 1) + bt.msa * (j - 1)]; };
    auto absb = [&](int ind, int j) { return T[bt.absb + (ind - 1) + bt.msb * (j - 1)]; };
    auto selfref = [&](int ind, int j) { return T[bt.selfref + (ind - 1) + 10 * (j - 1)]; };
    auto forref = [&](int ind, int j) { return T[bt.forref + (ind - 1) + bt.mfr * (j - 1)]; };
    const double strrat = tab1b(swtab::strrat, jb);
    // Rayleigh: scalar rayl for 16-22, 28, 29; per-g for 23, 25, 26, 27; 24 below
    double rayl_s = 0.0;
    const double* rayl_v = nullptr;
    switch (jb) {
      case 16: rayl_s = T[swtab::b16_rayl]; break;
      case 17: rayl_s = T[swtab::b17_rayl]; break;
      case 18: rayl_s = T[swtab::b18_rayl]; break;
      case 19: rayl_s = T[swtab::b19_rayl]; break;
      case 20: rayl_s = T[swtab::b20_rayl]; break;
      case 21: rayl_s = T[swtab::b21_rayl]; break;
      case 22: rayl_s = T[swtab::b22_rayl]; break;
      case 28: rayl_s = T[swtab::b28_rayl]; break;
      case 29: rayl_s = T[swtab::b29_rayl]; break;
      case 23: rayl_v = &T[swtab::b23_rayl]; break;
      case 25: rayl_v = &T[swtab::b25_rayl]; break;
      case 26: rayl_v = &T[swtab::b26_rayl]; break;
      case 27: rayl_v = &T[swtab::b27_rayl]; break;
      default: break;
    }
    if (jb != 24) {
      for (int k = 1; k <= nlay; ++k) {
        if (rayl_v) {
          for (int j = 1; j <= ngb; ++j) c.TAUR(k, ns + j) = c.colmol[k] * rayl_v[j - 1];
        } else {
          const double tauray = c.colmol[k] * rayl_s;
          for (int j = 1; j <= ngb; ++j) c.TAUR(k, ns + j) = tauray;
        }
      }
    }
    // binary-species lower/upper atmosphere helper (bands 16-19, 21, 22, 24, 28)
    auto spec8 = [&](int k, int g1, int g2, double mult, int& js, double& fs, double f[8]) {
      const double speccomb = c.COLAMT(k, g1) + strrat * c.COLAMT(k, g2);
      const double specmult = mult * std::min(oneminus, c.COLAMT(k, g1) / speccomb);
      js = 1 + (int)specmult;
      fs = std::fmod(specmult, f_one);
      const double fs1 = f_one - fs;
      f[0] = fs1 * c.fac00[k];   // fac000
      f[1] = fs1 * c.fac10[k];   // fac010
      f[2] = fs * c.fac00[k];    // fac100
      f[3] = fs * c.fac10[k];    // fac110
      f[4] = fs1 * c.fac01[k];   // fac001
      f[5] = fs1 * c.fac11[k];   // fac011
      f[6] = fs * c.fac01[k];    // fac101
      f[7] = fs * c.fac11[k];    // fac111
      return speccomb;
    };
    auto selfc = [&](int k, int j) {
      const int inds = c.indself[k], indsp = inds + 1;
      return c.selffac[k] * (selfref(inds, j) + c.selffrac[k] * (selfref(indsp, j) - selfref(inds, j)));
    };
    auto forc = [&](int k, int j) {
      const int indf = c.indfor[k], indfp = indf + 1;
      return c.forfac[k] * (forref(indf, j) + c.forfrac[k] * (forref(indfp, j) - forref(indf, j)));
    };
    auto kab8 = [&](auto tab, const double f[8], int i01, int d3, int i11, int j) {
      // fac000*t(i01) + fac100*t(i01+1) + fac010*t(i01+d3) + fac110*t(i01+d3+1) + (same at i11)
      return f[0] * tab(i01, j) + f[2] * tab(i01 + 1, j) + f[1] * tab(i01 + d3, j) + f[3] * tab(i01 + d3 + 1, j) +
             f[4] * tab(i11, j) + f[6] * tab(i11 + 1, j) + f[5] * tab(i11 + d3, j) + f[7] * tab(i11 + d3 + 1, j);
    };
    auto kab4 = [&](auto tab, int k, int i01, int i11, int j) {
      return c.fac00[k] * tab(i01, j) + c.fac10[k] * tab(i01 + 1, j) + c.fac01[k] * tab(i11, j) +
             c.fac11[k] * tab(i11 + 1, j);
    };
    int js;
    double fs, f[8];
    switch (jb) {
      case 16: case 18: case 17: case 19: case 21: case 22: {
        const int g2 = (jb == 16 || jb == 18) ? 5 : (jb == 22 ? 6 : 2);
        const double o2tem = 4.35e-4 / (350.0 * 2.0), o2adj = 1.6;
        for (int k = 1; k <= laytrop; ++k) {
          const double speccomb = spec8(k, 1, g2, 8.0, js, fs, f);
          const int i01 = ID0(k, jb) + js, i11 = ID1(k, jb) + js;
          const double o2cont = o2tem * c.COLAMT(k, 6);
          for (int j = 1; j <= ngb; ++j) {
            double t = speccomb * kab8(absa, f, i01, 9, i11, j) + c.COLAMT(k, 1) * (selfc(k, j) + forc(k, j));
            if (jb == 22) t = t + o2cont;
            c.TAUG(k, ns + j) = t;
          }
        }
        for (int k = laytrop + 1; k <= nlay; ++k) {
          if (jb == 17 || jb == 21) {
            const double speccomb = spec8(k, 1, 2, 4.0, js, fs, f);
            const int i01 = ID0(k, jb) + js, i11 = ID1(k, jb) + js;
            for (int j = 1; j <= ngb; ++j) {
              const int indf = c.indfor[k], indfp = indf + 1;
              c.TAUG(k, ns + j) = speccomb * kab8(absb, f, i01, 5, i11, j) +
                                  c.COLAMT(k, 1) * c.forfac[k] *
                                      (forref(indf, j) + c.forfrac[k] * (forref(indfp, j) - forref(indf, j)));
            }
          } else {
            const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
            const double o2cont = o2tem * c.COLAMT(k, 6);
            for (int j = 1; j <= ngb; ++j) {
              if (jb == 22)
                c.TAUG(k, ns + j) = c.COLAMT(k, 6) * o2adj * kab4(absb, k, i01, i11, j) + o2cont;
              else
                c.TAUG(k, ns + j) = c.COLAMT(k, jb == 19 ? 2 : 5) * kab4(absb, k, i01, i11, j);
            }
          }
        }
        break;
      }
      case 20: {
        const double* absch4 = &T[swtab::b20_absch4];
        for (int k = 1; k <= laytrop; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j)
            c.TAUG(k, ns + j) = c.COLAMT(k, 1) * (kab4(absa, k, i01, i11, j) + selfc(k, j) + forc(k, j)) +
                                c.COLAMT(k, 5) * absch4[j - 1];
        }
        for (int k = laytrop + 1; k <= nlay; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j)
            c.TAUG(k, ns + j) = c.COLAMT(k, 1) * (kab4(absb, k, i01, i11, j) + forc(k, j)) +
                                c.COLAMT(k, 5) * absch4[j - 1];
        }
        break;
      }
      case 23: {
        const double givfac = T[swtab::b23_givfac];
        for (int k = 1; k <= laytrop; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j)
            c.TAUG(k, ns + j) = c.COLAMT(k, 1) * (givfac * kab4(absa, k, i01, i11, j) + selfc(k, j) + forc(k, j));
        }
        for (int k = laytrop + 1; k <= nlay; ++k)
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = f_zero;
        break;
      }
      case 24: {
        const double *abso3a = &T[swtab::b24_abso3a], *abso3b = &T[swtab::b24_abso3b];
        const double *rayla = &T[swtab::b24_rayla], *raylb = &T[swtab::b24_raylb];
        for (int k = 1; k <= laytrop; ++k) {
          const double speccomb = spec8(k, 1, 6, 8.0, js, fs, f);
          const int i01 = ID0(k, jb) + js, i11 = ID1(k, jb) + js;
          for (int j = 1; j <= ngb; ++j) {
            c.TAUG(k, ns + j) = speccomb * kab8(absa, f, i01, 9, i11, j) + c.COLAMT(k, 3) * abso3a[j - 1] +
                                c.COLAMT(k, 1) * (selfc(k, j) + forc(k, j));
            const double ra = rayla[(j - 1) + 8 * (js - 1)], rb = rayla[(j - 1) + 8 * js];
            c.TAUR(k, ns + j) = c.colmol[k] * (ra + fs * (rb - ra));
          }
        }
        for (int k = laytrop + 1; k <= nlay; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j) {
            c.TAUG(k, ns + j) = c.COLAMT(k, 6) * kab4(absb, k, i01, i11, j) + c.COLAMT(k, 3) * abso3b[j - 1];
            c.TAUR(k, ns + j) = c.colmol[k] * raylb[j - 1];
          }
        }
        break;
      }
      case 25: {
        const double *abso3a = &T[swtab::b25_abso3a], *abso3b = &T[swtab::b25_abso3b];
        for (int k = 1; k <= laytrop; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j)
            c.TAUG(k, ns + j) = c.COLAMT(k, 1) * kab4(absa, k, i01, i11, j) + c.COLAMT(k, 3) * abso3a[j - 1];
        }
        for (int k = laytrop + 1; k <= nlay; ++k)
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = c.COLAMT(k, 3) * abso3b[j - 1];
        break;
      }
      case 26: {
        for (int k = 1; k <= nlay; ++k)
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = f_zero;
        break;
      }
      case 27: {
        for (int k = 1; k <= laytrop; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = c.COLAMT(k, 3) * kab4(absa, k, i01, i11, j);
        }
        for (int k = laytrop + 1; k <= nlay; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = c.COLAMT(k, 3) * kab4(absb, k, i01, i11, j);
        }
        break;
      }
      case 28: {
        for (int k = 1; k <= laytrop; ++k) {
          const double speccomb = spec8(k, 3, 6, 8.0, js, fs, f);
          const int i01 = ID0(k, jb) + js, i11 = ID1(k, jb) + js;
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = speccomb * kab8(absa, f, i01, 9, i11, j);
        }
        for (int k = laytrop + 1; k <= nlay; ++k) {
          const double speccomb = spec8(k, 3, 6, 4.0, js, fs, f);
          const int i01 = ID0(k, jb) + js, i11 = ID1(k, jb) + js;
          for (int j = 1; j <= ngb; ++j) c.TAUG(k, ns + j) = speccomb * kab8(absb, f, i01, 5, i11, j);
        }
        break;
      }
      case 29: {
        const double *absco2 = &T[swtab::b29_absco2], *absh2o = &T[swtab::b29_absh2o];
        for (int k = 1; k <= laytrop; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j)
            c.TAUG(k, ns + j) = c.COLAMT(k, 1) * (kab4(absa, k, i01, i11, j) + selfc(k, j) + forc(k, j)) +
                                c.COLAMT(k, 2) * absco2[j - 1];
        }
        for (int k = laytrop + 1; k <= nlay; ++k) {
          const int i01 = ID0(k, jb) + 1, i11 = ID1(k, jb) + 1;
          for (int j = 1; j <= ngb; ++j)
            c.TAUG(k, ns + j) = c.COLAMT(k, 2) * kab4(absb, k, i01, i11, j) + c.COLAMT(k, 1) * absh2o[j - 1];
        }
        break;
      }
    }
  }
}

// ---- vrtqdr (RSM:3959-4051); arrays 1-based over 1..nlp1 ------------------
void vrtqdr(const double* zrefb, const double* zrefd, const double* ztrab, const double* ztrad,
            const double* zldbt, const double* ztdbt, int nlay, double* zfu, double* zfd) {
  const int nlp1 = nlay + 1;
  std::vector<double> zrupb(nlp1 + 1), zrupd(nlp1 + 1), zrdnd(nlp1 + 1), ztdn(nlp1 + 1);
  zrupb[1] = zrefb[1];
  zrupd[1] = zrefd[1];
  for (int k = 1; k <= nlay; ++k) {
    const int kp = k + 1;
    const double zden1 = f_one / (f_one - zrupd[k] * zrefd[kp]);
    zrupb[kp] = zrefb[kp] + (ztrad[kp] * ((ztrab[kp] - zldbt[kp]) * zrupd[k] + zldbt[kp] * zrupb[k])) * zden1;
    zrupd[kp] = zrefd[kp] + ztrad[kp] * ztrad[kp] * zrupd[k] * zden1;
  }
  ztdn[nlp1] = f_one;
  zrdnd[nlp1] = f_zero;
  ztdn[nlay] = ztrab[nlp1];
  zrdnd[nlay] = zrefd[nlp1];
  for (int k = nlay; k >= 2; --k) {
    const double zden1 = f_one / (f_one - zrefd[k] * zrdnd[k]);
    ztdn[k - 1] = ztdbt[k] * ztrab[k] + (ztrad[k] * ((ztdn[k] - ztdbt[k]) + ztdbt[k] * zrefb[k] * zrdnd[k])) * zden1;
    zrdnd[k - 1] = zrefd[k] + ztrad[k] * ztrad[k] * zrdnd[k] * zden1;
  }
  for (int k = 1; k <= nlp1; ++k) {
    const double zden1 = f_one / (f_one - zrdnd[k] * zrupd[k]);
    zfu[k] = (ztdbt[k] * zrupb[k] + (ztdn[k] - ztdbt[k]) * zrupd[k]) * zden1;
    zfd[k] = ztdbt[k] + (ztdn[k] - ztdbt[k] + ztdbt[k] * zrupb[k] * zrdnd[k]) * zden1;
  }
}

inline double exp_lookup_trunc(double zb) {     // itind = ftind*NTBMX + 0.5 (assignment truncates)
  const double ftind = zb / (bpade + zb);
  const int itind = (int)(ftind * NTBMX + 0.5);
  return exp_tbl[itind];
}
inline double exp_lookup_clamp(double zr) {     // itind = max(0, min(NTBMX, int(0.5+NTBMX*ftind)))
  const double ftind = zr / (bpade + zr);
  const int itind = std::max(0, std::min(NTBMX, (int)(0.5 + NTBMX * ftind)));
  return exp_tbl[itind];
}

// One layer's two-stream reflectance/transmittance (the body shared by the
// clear and cloudy sweeps of spcvrtm, RSM:3444-3624 and 3674-3853).
void two_stream(double ztau0, double zssa0, double zasy0, double cosz, double sntz, int iswmode, double& zrefb,
                double& ztrab, double& zrefd, double& ztrad, double& ztau1_out) {
  const double zcrit = 0.9999995, zsr3 = std::sqrt(3.0), od_lo = 0.06, eps1 = 1.0e-8;
  const double zssaw = std::min(oneminus, zssa0 / ztau0);
  const double zasyw = zasy0 / std::max(ftiny, zssa0);
  double za1 = zasyw * zasyw;
  double za2 = zssaw * za1;
  const double ztau1 = (f_one - za2) * ztau0;
  const double zssa1 = (zssaw - za2) / (f_one - za2);
  const double zasy1 = zasyw / (f_one + zasyw);
  const double zasy3 = 0.75 * zasy1;
  double zgam1 = 0, zgam2 = 0, zgam3 = 0;
  if (iswmode == 1) {
    zgam1 = 1.75 - zssa1 * (f_one + zasy3);
    zgam2 = -0.25 + zssa1 * (f_one - zasy3);
    zgam3 = 0.5 - zasy3 * cosz;
  } else if (iswmode == 2) {
    zgam1 = 2.0 - zssa1 * (1.25 + zasy3);
    zgam2 = 0.75 * zssa1 * (f_one - zasy1);
    zgam3 = 0.5 - zasy3 * cosz;
  } else if (iswmode == 3) {
    zgam1 = zsr3 * (2.0 - zssa1 * (1.0 + zasy1)) * 0.5;
    zgam2 = zsr3 * zssa1 * (1.0 - zasy1) * 0.5;
    zgam3 = (1.0 - zsr3 * zasy1 * cosz) * 0.5;
  }
  const double zgam4 = f_one - zgam3;
  if (zssaw >= zcrit) {
    za1 = zgam1 * cosz - zgam3;
    za2 = zgam1 * ztau1;
    const double zb1 = std::min(ztau1 * sntz, 500.0);
    double zb2;
    if (zb1 <= od_lo) zb2 = f_one - zb1 + 0.5 * zb1 * zb1;
    else zb2 = exp_lookup_trunc(zb1);
    zrefb = std::max(f_zero, std::min(f_one, (za2 - za1 * (f_one - zb2)) / (f_one + za2)));
    ztrab = std::max(f_zero, std::min(f_one, f_one - zrefb));
    zrefd = std::max(f_zero, std::min(f_one, za2 / (f_one + za2)));
    ztrad = std::max(f_zero, std::min(f_one, f_one - zrefd));
  } else {
    za1 = zgam1 * zgam4 + zgam2 * zgam3;
    za2 = zgam1 * zgam3 + zgam2 * zgam4;
    double zrk = (zgam1 - zgam2) * (zgam1 + zgam2);
    if (zrk > eps1) zrk = std::sqrt(zrk);
    else zrk = f_zero;
    const double zrk2 = zrk + zrk;
    const double zrp = zrk * cosz;
    const double zrp1 = f_one + zrp, zrm1 = f_one - zrp;
    const double zrpp1 = f_one - zrp * zrp;
    const double zrpp = std::copysign(std::max(flimit, std::fabs(zrpp1)), zrpp1);
    const double zrkg1 = zrk + zgam1, zrkg3 = zrk * zgam3, zrkg4 = zrk * zgam4;
    const double zr1 = zrm1 * (za2 + zrkg3);
    const double zr2 = zrp1 * (za2 - zrkg3);
    const double zr3 = zrk2 * (zgam3 - za2 * cosz);
    const double zr4 = zrpp * zrkg1;
    const double zr5 = zrpp * (zrk - zgam1);
    const double zt1 = zrp1 * (za1 + zrkg4);
    const double zt2 = zrm1 * (za1 - zrkg4);
    const double zt3 = zrk2 * (zgam4 + za1 * cosz);
    const double zb1 = std::min(zrk * ztau1, 500.0);
    double zexm1;
    if (zb1 <= od_lo) zexm1 = f_one - zb1 + 0.5 * zb1 * zb1;
    else zexm1 = exp_lookup_trunc(zb1);
    const double zexp1 = f_one / zexm1;
    const double zb2 = std::min(sntz * ztau1, 500.0);
    double zexm2;
    if (zb2 <= od_lo) zexm2 = f_one - zb2 + 0.5 * zb2 * zb2;
    else zexm2 = exp_lookup_trunc(zb2);
    const double zexp2 = f_one / zexm2;
    const double ze1r45 = zr4 * zexp1 + zr5 * zexm1;
    if (std::fabs(ze1r45) <= eps1) {
      zrefb = eps1;
      ztrab = zexm2;
    } else {
      const double zden1 = zssa1 / ze1r45;
      zrefb = std::max(f_zero, std::min(f_one, (zr1 * zexp1 - zr2 * zexm1 - zr3 * zexm2) * zden1));
      ztrab = std::max(f_zero, std::min(f_one, zexm2 * (f_one - (zt1 * zexp1 - zt2 * zexm1 - zt3 * zexp2) * zden1)));
    }
    double zden1;
    if (ze1r45 >= f_zero) zden1 = zr4 / std::max(eps1, ze1r45 * zrkg1);
    else zden1 = zr4 / std::min(-eps1, ze1r45 * zrkg1);
    zrefd = std::max(f_zero, std::min(f_one, zgam2 * (zexp1 - zexm1) * zden1));
    ztrad = std::max(f_zero, std::min(f_one, zrk2 * zden1));
  }
  ztau1_out = ztau1;
}

struct SwScalars {
  double ftoauc, ftoau0, ftoadc, fsfcuc, fsfcu0, fsfcdc, fsfcd0, suvbfc, suvbf0;
  double sfbmc[2], sfdfc[2], sfbm0[2], sfdf0[2];
};

// ---- spcvrtm (RSM:3228-3942) ----------------------------------------------
// spcvrtc (RSM:2432-3183) is the same sweep with the cloudy layers' optics
// mixed by the normalised cloud fraction instead of McICA flags
// (RSM:2925-2928, 3039-3042, 3057, 3072) and the column's fluxes mixed by
// cf1/cf0 (RSM:3158-3178); grid = true selects it.
void spcvrtm(Col& c, double ssolar, double cosz, double sntz, const double albbm[2], const double albdf[2],
             double cf1, double cf0, int iswmode, bool grid, SwScalars& o) {
  const int nlay = c.nlay, nlp1 = nlay + 1;
  const double od_lo = 0.06;
  for (auto* v : {&c.fxupc, &c.fxdnc, &c.fxup0, &c.fxdn0}) std::fill(v->begin(), v->end(), 0.0);
  o = SwScalars{};
  std::vector<double> ztaus(nlay + 1), zssas(nlay + 1), zasys(nlay + 1), zldbt0(nlay + 1);
  std::vector<double> zrefb(nlp1 + 1), zrefd(nlp1 + 1), ztrab(nlp1 + 1), ztrad(nlp1 + 1), ztdbt(nlp1 + 1),
      zldbt(nlp1 + 1), zfu(nlp1 + 1), zfd(nlp1 + 1);
  for (int jg = 1; jg <= NGPT; ++jg) {
    const int jb = NGB[jg - 1], ib = jb + 1 - NBLOW, ibd = IDXSFC[jb - NBLOW];
    const double zsolar = ssolar * c.sfluxzen[jg - 1];
    ztdbt[nlp1] = f_one;
    double ztdbt0 = f_one;
    zldbt[1] = f_zero;
    if (ibd != 0) {
      zrefb[1] = albbm[ibd - 1];
      zrefd[1] = albdf[ibd - 1];
    } else {
      zrefb[1] = 0.5 * (albbm[0] + albbm[1]);
      zrefd[1] = 0.5 * (albdf[0] + albdf[1]);
    }
    ztrab[1] = f_zero;
    ztrad[1] = f_zero;
    for (int k = nlay; k >= 1; --k) {
      const int kp = k + 1;
      const double ztau0 = std::max(ftiny, c.TAUR(k, jg) + c.TAUG(k, jg) + c.TAUAE(k, ib));
      const double zssa0 = c.TAUR(k, jg) + c.TAUAE(k, ib) * c.SSAAE(k, ib);
      const double zasy0 = c.ASYAE(k, ib) * c.SSAAE(k, ib) * c.TAUAE(k, ib);
      ztaus[k] = ztau0;
      zssas[k] = zssa0;
      zasys[k] = zasy0;
      double ztau1;
      two_stream(ztau0, zssa0, zasy0, cosz, sntz, iswmode, zrefb[kp], ztrab[kp], zrefd[kp], ztrad[kp], ztau1);
      double zr1 = ztau1 * sntz, zexp3, zexp4;
      if (zr1 <= od_lo) zexp3 = f_one - zr1 + 0.5 * zr1 * zr1;
      else zexp3 = exp_lookup_clamp(zr1);
      ztdbt[k] = zexp3 * ztdbt[kp];
      zldbt[kp] = zexp3;
      zr1 = ztau0 * sntz;
      if (zr1 <= od_lo) zexp4 = f_one - zr1 + 0.5 * zr1 * zr1;
      else zexp4 = exp_lookup_clamp(zr1);
      zldbt0[k] = zexp4;
      ztdbt0 = zexp4 * ztdbt0;
    }
    vrtqdr(zrefb.data(), zrefd.data(), ztrab.data(), ztrad.data(), zldbt.data(), ztdbt.data(), nlay, zfu.data(),
           zfd.data());
    for (int k = 1; k <= nlp1; ++k) {
      c.FXUP0(k, ib) = c.FXUP0(k, ib) + zsolar * zfu[k];
      c.FXDN0(k, ib) = c.FXDN0(k, ib) + zsolar * zfd[k];
    }
    double zb1 = zsolar * ztdbt0, zb2 = zsolar * (zfd[1] - ztdbt0);
    if (ibd != 0) {
      o.sfbm0[ibd - 1] = o.sfbm0[ibd - 1] + zb1;
      o.sfdf0[ibd - 1] = o.sfdf0[ibd - 1] + zb2;
    } else {
      const double zf1 = 0.5 * zb1, zf2 = 0.5 * zb2;
      o.sfbm0[0] = o.sfbm0[0] + zf1;
      o.sfdf0[0] = o.sfdf0[0] + zf2;
      o.sfbm0[1] = o.sfbm0[1] + zf1;
      o.sfdf0[1] = o.sfdf0[1] + zf2;
    }
    if (cf1 > eps) {
      ztdbt0 = f_one;
      zldbt[1] = f_zero;
      for (int k = nlay; k >= 1; --k) {
        const int kp = k + 1;
        const double zc0 = f_one - c.cldfrc[k], zc1 = c.cldfrc[k];
        if (grid ? (zc1 > ftiny) : (c.CLDFMC(k, jg) > ftiny)) {
          const double zrefb1 = zrefb[kp], zrefd1 = zrefd[kp], ztrab1 = ztrab[kp], ztrad1 = ztrad[kp];
          const double ztau0 = ztaus[k] + c.TAUCW(k, ib);
          const double zssa0 = zssas[k] + c.SSACW(k, ib);
          const double zasy0 = zasys[k] + c.ASYCW(k, ib);
          double ztau1;
          two_stream(ztau0, zssa0, zasy0, cosz, sntz, iswmode, zrefb[kp], ztrab[kp], zrefd[kp], ztrad[kp], ztau1);
          if (grid) {
            zrefb[kp] = zc0 * zrefb1 + zc1 * zrefb[kp];
            zrefd[kp] = zc0 * zrefd1 + zc1 * zrefd[kp];
            ztrab[kp] = zc0 * ztrab1 + zc1 * ztrab[kp];
            ztrad[kp] = zc0 * ztrad1 + zc1 * ztrad[kp];
          }
          double zr1 = ztau1 * sntz, zexp3, zexp4;
          if (zr1 <= od_lo) zexp3 = f_one - zr1 + 0.5 * zr1 * zr1;
          else zexp3 = exp_lookup_clamp(zr1);
          if (grid) {
            zldbt[kp] = zc0 * zldbt[kp] + zc1 * zexp3;
            ztdbt[k] = zldbt[kp] * ztdbt[kp];
          } else {
            zldbt[kp] = zexp3;
            ztdbt[k] = zexp3 * ztdbt[kp];
          }
          zr1 = ztau0 * sntz;
          if (zr1 <= od_lo) zexp4 = f_one - zr1 + 0.5 * zr1 * zr1;
          else zexp4 = exp_lookup_clamp(zr1);
          if (grid) ztdbt0 = (zc0 * zldbt0[k] + zc1 * zexp4) * ztdbt0;
          else ztdbt0 = zexp4 * ztdbt0;
        } else {
          ztdbt[k] = zldbt[kp] * ztdbt[kp];
          ztdbt0 = zldbt0[k] * ztdbt0;
        }
      }
      vrtqdr(zrefb.data(), zrefd.data(), ztrab.data(), ztrad.data(), zldbt.data(), ztdbt.data(), nlay, zfu.data(),
             zfd.data());
      for (int k = 1; k <= nlp1; ++k) {
        c.FXUPC(k, ib) = c.FXUPC(k, ib) + zsolar * zfu[k];
        c.FXDNC(k, ib) = c.FXDNC(k, ib) + zsolar * zfd[k];
      }
      zb1 = zsolar * ztdbt0;
      zb2 = zsolar * (zfd[1] - ztdbt0);
      if (ibd != 0) {
        o.sfbmc[ibd - 1] = o.sfbmc[ibd - 1] + zb1;
        o.sfdfc[ibd - 1] = o.sfdfc[ibd - 1] + zb2;
      } else {
        const double zf1 = 0.5 * zb1, zf2 = 0.5 * zb2;
        o.sfbmc[0] = o.sfbmc[0] + zf1;
        o.sfdfc[0] = o.sfdfc[0] + zf2;
        o.sfbmc[1] = o.sfbmc[1] + zf1;
        o.sfdfc[1] = o.sfdfc[1] + zf2;
      }
    }
  }
  for (int ib = 1; ib <= NBDSW; ++ib) {
    o.ftoadc = o.ftoadc + c.FXDN0(nlp1, ib);
    o.ftoau0 = o.ftoau0 + c.FXUP0(nlp1, ib);
    o.fsfcu0 = o.fsfcu0 + c.FXUP0(1, ib);
    o.fsfcd0 = o.fsfcd0 + c.FXDN0(1, ib);
  }
  const int ibd = NUVB - NBLOW + 1;
  o.suvbf0 = c.FXDN0(1, ibd);
  if (cf1 <= eps) {
    for (int ib = 1; ib <= NBDSW; ++ib)
      for (int k = 1; k <= nlp1; ++k) {
        c.FXUPC(k, ib) = c.FXUP0(k, ib);
        c.FXDNC(k, ib) = c.FXDN0(k, ib);
      }
    o.ftoauc = o.ftoau0;
    o.fsfcuc = o.fsfcu0;
    o.fsfcdc = o.fsfcd0;
    o.sfbmc[0] = o.sfbm0[0];
    o.sfdfc[0] = o.sfdf0[0];
    o.sfbmc[1] = o.sfbm0[1];
    o.sfdfc[1] = o.sfdf0[1];
    o.suvbfc = o.suvbf0;
  } else {
    if (grid)
      for (int ib = 1; ib <= NBDSW; ++ib)
        for (int k = 1; k <= nlp1; ++k) {
          c.FXUPC(k, ib) = cf1 * c.FXUPC(k, ib) + cf0 * c.FXUP0(k, ib);
          c.FXDNC(k, ib) = cf1 * c.FXDNC(k, ib) + cf0 * c.FXDN0(k, ib);
        }
    for (int ib = 1; ib <= NBDSW; ++ib) {
      o.ftoauc = o.ftoauc + c.FXUPC(nlp1, ib);
      o.fsfcuc = o.fsfcuc + c.FXUPC(1, ib);
      o.fsfcdc = o.fsfcdc + c.FXDNC(1, ib);
    }
    o.suvbfc = c.FXDNC(1, ibd);
    if (grid)
      for (int q = 0; q < 2; ++q) {
        o.sfbmc[q] = cf1 * o.sfbmc[q] + cf0 * o.sfbm0[q];
        o.sfdfc[q] = cf1 * o.sfdfc[q] + cf0 * o.sfdf0[q];
      }
  }
}

// Column prologue of rrtmg_sw_run (RSM:892-1094): internal surface-first arrays.
void load_column(const rrtmg_sw_run_args& a, int j1, Col& c) {
  const int nlay = a.nlay, nlp1 = a.nlp1;
  const long ld = a.ldim > 0 ? a.ldim : a.npts;
  auto A2 = [&](const double* p, int k) { return p[(j1 - 1) + ld * (k - 1)]; };
  auto A3 = [&](const double* p, int k, int b) { return p[(j1 - 1) + ld * ((k - 1) + (long)nlay * (b - 1))]; };
  const double tem1 = 100.0 * con_g, tem2 = 1.0e-20 * 1.0e3 * con_avgd;
  for (int k = 1; k <= nlay; ++k) {
    const int kk = a.top_at_1 ? nlp1 - k : k;
    c.pavel[k] = A2(a.plyr, kk);
    c.tavel[k] = A2(a.tlyr, kk);
    c.delp[k] = A2(a.delpin, kk);
    c.dz[k] = A2(a.dzlyr, kk);
    if (a.iovr == a.iovr_exp || a.iovr == a.iovr_exprand) c.alph[k] = A2(a.alpha, k);   // unflipped (RSM:921, 1012)
    c.h2ovmr[k] = std::max(f_zero, A2(a.qlyr, kk) * amdw / (f_one - A2(a.qlyr, kk)));
    c.o3vmr[k] = std::max(f_zero, A2(a.olyr, kk) * amdo3);
    const double tem0 = (f_one - c.h2ovmr[k]) * con_amd + c.h2ovmr[k] * con_amw;
    c.coldry[k] = tem2 * c.delp[k] / (tem1 * tem0 * (f_one + c.h2ovmr[k]));
    c.temcol[k] = 1.0e-12 * c.coldry[k];
    c.COLAMT(k, 1) = std::max(f_zero, c.coldry[k] * c.h2ovmr[k]);
    c.COLAMT(k, 2) = std::max(c.temcol[k], c.coldry[k] * A2(a.gasvmr_co2, kk));
    c.COLAMT(k, 3) = std::max(f_zero, c.coldry[k] * c.o3vmr[k]);
    c.colmol[k] = c.coldry[k] + c.COLAMT(k, 1);
  }
  for (int k = 1; k <= nlay; ++k) {
    const int kk = a.top_at_1 ? nlp1 - k : k;
    if (a.inc_minor_gas) {
      c.COLAMT(k, 4) = std::max(c.temcol[k], c.coldry[k] * A2(a.gasvmr_n2o, kk));
      c.COLAMT(k, 5) = std::max(c.temcol[k], c.coldry[k] * A2(a.gasvmr_ch4, kk));
      c.COLAMT(k, 6) = std::max(c.temcol[k], c.coldry[k] * A2(a.gasvmr_o2, kk));
    } else {
      c.COLAMT(k, 4) = c.temcol[k];
      c.COLAMT(k, 5) = c.temcol[k];
      c.COLAMT(k, 6) = c.temcol[k];
    }
    for (int ib = 1; ib <= NBDSW; ++ib) {
      c.TAUAE(k, ib) = A3(a.aeraod, kk, ib);
      c.SSAAE(k, ib) = A3(a.aerssa, kk, ib);
      c.ASYAE(k, ib) = A3(a.aerasy, kk, ib);
    }
    c.cfrac[k] = A2(a.cld_cf, kk);
    if (a.iswcliq > 0) {
      c.cliqp[k] = A2(a.cld_lwp, kk);
      c.reliq[k] = A2(a.cld_ref_liq, kk);
      c.cicep[k] = A2(a.cld_iwp, kk);
      c.reice[k] = A2(a.cld_ref_ice, kk);
      c.cdat1[k] = A2(a.cld_rwp, kk);
      c.cdat2[k] = A2(a.cld_ref_rain, kk);
      c.cdat3[k] = A2(a.cld_swp, kk);
      c.cdat4[k] = A2(a.cld_ref_snow, kk);
    } else {
      c.cdat1[k] = A2(a.cld_od, kk);
      c.cdat2[k] = A2(a.cld_ssa, kk);
      c.cdat3[k] = A2(a.cld_asy, kk);
    }
  }
}

void run_column(const rrtmg_sw_run_args& a, int ipt, Col& c) {
  const int nlay = a.nlay, nlp1 = a.nlp1;
  const long ld = a.ldim > 0 ? a.ldim : a.npts;
  const int j1 = a.idxday[ipt - 1];
  const int ipseed = (a.isubcsw == 2) ? a.icseed[j1 - 1] : 1 + j1;   // ipsdsw0 + i (RSM:875-883)
  const double cosz1 = a.cosz[j1 - 1];
  const double sntz1 = f_one / a.cosz[j1 - 1];
  const double ssolar = (a.solcon / s0) * a.cosz[j1 - 1];
  const double delgth = (a.iovr == a.iovr_dcorr) ? a.de_lgth[j1 - 1] : 0.0;
  const double albbm[2] = {a.sfcalb_nir_dir[j1 - 1], a.sfcalb_uvis_dir[j1 - 1]};
  const double albdf[2] = {a.sfcalb_nir_dif[j1 - 1], a.sfcalb_uvis_dif[j1 - 1]};
  load_column(a, j1, c);

  // clear/cloudy column indicator (RSM:1101-1125)
  double zcf0 = f_one, zcf1 = f_one;
  if (a.iovr == a.iovr_rand) {
    for (int k = 1; k <= nlay; ++k) zcf0 = zcf0 * (f_one - c.cfrac[k]);
  } else if (a.iovr == a.iovr_maxrand) {
    for (int k = 1; k <= nlay; ++k) {
      if (c.cfrac[k] > ftiny) zcf1 = std::min(zcf1, f_one - c.cfrac[k]);
      else if (zcf1 < f_one) { zcf0 = zcf0 * zcf1; zcf1 = f_one; }
    }
    zcf0 = zcf0 * zcf1;
  } else if (a.iovr >= 2) {
    for (int k = 1; k <= nlay; ++k) zcf0 = std::min(zcf0, f_one - c.cfrac[k]);
  }
  if (zcf0 <= ftiny) zcf0 = f_zero;
  if (zcf0 > oneminus) zcf0 = f_one;
  zcf1 = f_one - zcf0;
  if (zcf1 > f_zero) {
    cldprop(c, ipseed, delgth, a.iswcliq, a.iswcice, a.isubcsw, a.iovr, zcf1);
    for (int k = 1; k <= nlay; ++k) {
      const int kk = a.top_at_1 ? nlp1 - k : k;
      a.cldtau[(j1 - 1) + ld * (kk - 1)] = c.TAUCW(k, 10);
    }
  } else {
    std::fill(c.cldfrc.begin(), c.cldfrc.end(), 0.0);
    std::fill(c.cldfmc.begin(), c.cldfmc.end(), 0.0);
    std::fill(c.taucw.begin(), c.taucw.end(), 0.0);
    std::fill(c.ssacw.begin(), c.ssacw.end(), 0.0);
    std::fill(c.asycw.begin(), c.asycw.end(), 0.0);
  }
  const int laytrop = setcoef(c);
  taumol(c, laytrop);
  SwScalars o;
  spcvrtm(c, ssolar, cosz1, sntz1, albbm, albdf, zcf1, zcf0, a.iswmode, a.isubcsw <= 0, o);

  std::vector<double> flxuc(nlp1 + 1), flxdc(nlp1 + 1), flxu0(nlp1 + 1), flxd0(nlp1 + 1), fnet(nlp1 + 1),
      rfdelp(nlay + 1);
  for (int k = 1; k <= nlp1; ++k) {
    flxuc[k] = f_zero;
    flxdc[k] = f_zero;
    for (int ib = 1; ib <= NBDSW; ++ib) {
      flxuc[k] = flxuc[k] + c.FXUPC(k, ib);
      flxdc[k] = flxdc[k] + c.FXDNC(k, ib);
    }
  }
  if (a.hsw0 || a.flxprf) {
    for (int k = 1; k <= nlp1; ++k) {
      flxu0[k] = f_zero;
      flxd0[k] = f_zero;
      for (int ib = 1; ib <= NBDSW; ++ib) {
        flxu0[k] = flxu0[k] + c.FXUP0(k, ib);
        flxd0[k] = flxd0[k] + c.FXDN0(k, ib);
      }
    }
  }
  for (int k = 1; k <= nlay; ++k) rfdelp[k] = heatfac / c.delp[k];
  if (a.fdncmp) {
    double* r = a.fdncmp + 6 * (j1 - 1);
    r[0] = o.suvbfc; r[1] = o.suvbf0; r[2] = o.sfbmc[0]; r[3] = o.sfdfc[0]; r[4] = o.sfbmc[1]; r[5] = o.sfdfc[1];
  }
  double* tf = a.topflx + 3 * (j1 - 1);
  tf[0] = o.ftoauc; tf[1] = o.ftoadc; tf[2] = o.ftoau0;
  double* sf = a.sfcflx + 4 * (j1 - 1);
  sf[0] = o.fsfcuc; sf[1] = o.fsfcdc; sf[2] = o.fsfcu0; sf[3] = o.fsfcd0;
  // internal layer m (1 = surface) lands at caller row kk
  auto row = [&](int m) { return a.top_at_1 ? nlp1 - m : m; };
  auto lev = [&](int k) { return a.top_at_1 ? nlp1 - k + 1 : k; };
  fnet[1] = flxdc[1] - flxuc[1];
  for (int k = 2; k <= nlp1; ++k) {
    fnet[k] = flxdc[k] - flxuc[k];
    a.hswc[(j1 - 1) + ld * (row(k - 1) - 1)] = (fnet[k] - fnet[k - 1]) * rfdelp[k - 1];
  }
  if (a.flxprf)
    for (int k = 1; k <= nlp1; ++k) {
      double* r = a.flxprf + 4 * ((j1 - 1) + ld * (lev(k) - 1));
      r[0] = flxuc[k]; r[1] = flxdc[k]; r[2] = flxu0[k]; r[3] = flxd0[k];
    }
  if (a.hsw0) {
    fnet[1] = flxd0[1] - flxu0[1];
    for (int k = 2; k <= nlp1; ++k) {
      fnet[k] = flxd0[k] - flxu0[k];
      a.hsw0[(j1 - 1) + ld * (row(k - 1) - 1)] = (fnet[k] - fnet[k - 1]) * rfdelp[k - 1];
    }
  }
  if (a.hswb)
    for (int mb = 1; mb <= NBDSW; ++mb) {
      fnet[1] = c.FXDNC(1, mb) - c.FXUPC(1, mb);
      for (int k = 2; k <= nlp1; ++k) {
        fnet[k] = c.FXDNC(k, mb) - c.FXUPC(k, mb);
        a.hswb[(j1 - 1) + ld * ((row(k - 1) - 1) + (long)nlay * (mb - 1))] = (fnet[k] - fnet[k - 1]) * rfdelp[k - 1];
      }
    }
}

int check_args(const rrtmg_sw_run_args* a, char* errmsg, int errmsg_len) {
  if (a->iswcliq > 0) {
    if (!a->cld_lwp || !a->cld_ref_liq || !a->cld_iwp || !a->cld_ref_ice || !a->cld_rwp || !a->cld_ref_rain ||
        !a->cld_swp || !a->cld_ref_snow) {
      set_err(errmsg, errmsg_len,
              "Logic error: iswcliq>0 requires the following optional arguments to be present: "
              "cld_lwp, cld_ref_liq, cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow");
      return 1;
    }
  } else if (!a->cld_od || !a->cld_ssa || !a->cld_asy) {
    set_err(errmsg, errmsg_len,
            "Logic error: iswcliq<=0 requires the following optional arguments to be present: cld_od, cld_ssa, cld_asy");
    return 1;
  }
  if (a->isubcsw > 2) {
    set_err(errmsg, errmsg_len, "oracle: isubcsw must be 0 (spcvrtc), 1 or 2 (McICA, spcvrtm)");
    return 1;
  }
  if (a->isubcsw == 2 && !a->icseed) {
    set_err(errmsg, errmsg_len, "oracle: isubcsw=2 needs icseed");
    return 1;
  }
  return 0;
}

}  // namespace

extern "C" {

// rswinit (RSM:1388-1536) plus loading the coefficient blob.
int oracle_rswinit(const char* table_path, const rrtmg_sw_init_args* a, char* errmsg, int errmsg_len) {
  set_err(errmsg, errmsg_len, "");
  FILE* f = std::fopen(table_path, "rb");
  if (!f) { set_err(errmsg, errmsg_len, std::string("oracle: cannot open ") + table_path); return 1; }
  T.assign(RRTMG_SW_TABLES_NDOUBLE, 0.0);
  const size_t n = std::fread(T.data(), sizeof(double), T.size(), f);
  std::fclose(f);
  if (n != T.size()) { set_err(errmsg, errmsg_len, "oracle: short table blob"); return 1; }
  int errflg = 0;
  if (a->iovr != a->iovr_rand && a->iovr != a->iovr_maxrand && a->iovr != a->iovr_max &&
      a->iovr != a->iovr_dcorr && a->iovr != a->iovr_exp && a->iovr != a->iovr_exprand) {
    errflg = 1;
    set_err(errmsg, errmsg_len, "ERROR(rswinit): Error in specification of cloud overlap flag");
  }
  for (int b = 0, s = 0, g = 0; b < NBDSW; ++b) {
    NS[b] = s;
    s += NG[b];
    for (int j = 0; j < NG[b]; ++j) NGB[g++] = NBLOW + b;
  }
  heatfac = (a->rad_hr_units == 1) ? con_g * 864.0 / con_cp : con_g * 1.0e-2 / con_cp;
  exp_tbl[0] = 1.0;
  exp_tbl[NTBMX] = 1.e-20;
  for (int i = 1; i <= NTBMX - 1; ++i) {
    const double tfn = (double)i / (double)(NTBMX - i);
    const double tau = bpade * tfn;
    exp_tbl[i] = std::exp(-tau);
  }
  g_init = true;
  return errflg;
}

// rrtmg_sw_run (RSM:493-1379), OpenMP over daytime points with `nthreads`
// threads (0 = the OpenMP default).
int oracle_rrtmg_sw_run(const rrtmg_sw_run_args* a, int nthreads, char* errmsg, int errmsg_len) {
  set_err(errmsg, errmsg_len, "");
  if (!g_init) { set_err(errmsg, errmsg_len, "oracle: rswinit not called"); return 1; }
  if (!a->lsswr || a->nday <= 0) return 0;
  const long ld = a->ldim > 0 ? a->ldim : a->npts;
  const int nlay = a->nlay, nlp1 = a->nlp1, np = a->npts;
  for (int k = 0; k < nlay; ++k)
    for (int i = 0; i < np; ++i) {
      a->hswc[i + ld * k] = f_zero;
      a->cldtau[i + ld * k] = f_zero;
      if (a->hsw0) a->hsw0[i + ld * k] = f_zero;
      if (a->hswb)
        for (int b = 0; b < NBDSW; ++b) a->hswb[i + ld * (k + (long)nlay * b)] = f_zero;
    }
  for (int i = 0; i < np; ++i) {
    for (int q = 0; q < 3; ++q) a->topflx[3 * i + q] = f_zero;
    for (int q = 0; q < 4; ++q) a->sfcflx[4 * i + q] = f_zero;
    if (a->fdncmp)
      for (int q = 0; q < 6; ++q) a->fdncmp[6 * i + q] = f_zero;
    if (a->flxprf)
      for (int k = 0; k < nlp1; ++k)
        for (int q = 0; q < 4; ++q) a->flxprf[4 * (i + ld * k) + q] = f_zero;
  }
  if (check_args(a, errmsg, errmsg_len)) return 1;
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    Col c(nlay);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 8)
#endif
    for (int ipt = 1; ipt <= a->nday; ++ipt) run_column(*a, ipt, c);
  }
  return 0;
}

// Gas optics of daytime point ipt (1-based): taug/taur[(k-1)*112 + ig-1]
// in internal (surface-first) order, sfluxzen[112].  Returns laytrop.
int oracle_sw_gas_optics(const rrtmg_sw_run_args* a, int ipt, double* taug, double* taur, double* sfluxzen) {
  Col c(a->nlay);
  load_column(*a, a->idxday[ipt - 1], c);
  const int laytrop = setcoef(c);
  taumol(c, laytrop);
  for (int k = 1; k <= a->nlay; ++k)
    for (int g = 1; g <= NGPT; ++g) {
      taug[(size_t)(k - 1) * NGPT + g - 1] = c.TAUG(k, g);
      taur[(size_t)(k - 1) * NGPT + g - 1] = c.TAUR(k, g);
    }
  for (int g = 0; g < NGPT; ++g) sfluxzen[g] = c.sfluxzen[g];
  return laytrop;
}

// mcica_subcol (RSM:1952-2212) alone: lcloudy as bits
// bits[ig * nwords + (k >> 5)] bit (k & 31), nwords = (nlay + 31) / 32.
void oracle_sw_mcica(int nlay, int32_t seed, int iovr, const double* cldf, const double* dz, double de_lgth,
                     const double* alpha, uint32_t* bits) {
  std::vector<char> lc;
  std::vector<double> zero(nlay, 0.0);
  mcica_subcol(nlay, cldf, seed, dz ? dz : zero.data(), de_lgth, alpha ? alpha : zero.data(), iovr, lc);
  const int nw = (nlay + 31) / 32;
  std::memset(bits, 0, sizeof(uint32_t) * (size_t)NGPT * nw);
  for (int n = 0; n < NGPT; ++n)
    for (int k = 0; k < nlay; ++k)
      if (lc[(size_t)n * nlay + k]) bits[n * nw + (k >> 5)] |= 1u << (k & 31);
}

// rad_sw_pre_run (physics/Radiation/RRTMG/rad_sw_pre.F90:14-51): the daytime
// columns, in the reference's loop.
void oracle_sw_pre(int im, int lsswr, const double* coszen, int32_t* nday, int32_t* idxday) {
  *nday = 0;
  for (int i = 0; i < im; ++i) idxday[i] = 0;
  if (!lsswr) return;
  for (int i = 1; i <= im; ++i)
    if (coszen[i - 1] >= 0.0001) {
      *nday += 1;
      idxday[*nday - 1] = i;
    }
}

// rrtmg_sw_post_run (physics/Radiation/RRTMG/rrtmg_sw_post.F90:13-129), a
// scalar loop per statement in the reference's order; (im, ...) arrays
// column-major with leading dimension im, records as in the run's outputs.
void oracle_sw_post(const rrtmg_sw_post_args* a) {
  if (!a->lsswr) return;
  const int im = a->im, levs = a->levs, lm = a->lm, kd = a->kd;
  auto at = [im](int i, int k) { return (size_t)i + (size_t)im * (k - 1); };   // (i, k), k 1-based
  if (a->nday > 0) {
    for (int k = 1; k <= lm; ++k)
      for (int i = 0; i < im; ++i) a->htrsw[at(i, k)] = a->htswc[at(i, k + kd)];
    if (lm < levs)
      for (int k = lm + 1; k <= levs; ++k)
        for (int i = 0; i < im; ++i) a->htrsw[at(i, k)] = a->htrsw[at(i, lm)];
    if (a->swhtr) {
      for (int k = 1; k <= lm; ++k)
        for (int i = 0; i < im; ++i) a->swhc[at(i, k)] = a->htsw0[at(i, k + kd)];
      if (lm < levs)
        for (int k = lm + 1; k <= levs; ++k)
          for (int i = 0; i < im; ++i) a->swhc[at(i, k)] = a->swhc[at(i, lm)];
    }
    for (int i = 0; i < im; ++i) {
      const double* c = a->scmpsw + 6 * (size_t)i;   // {uvbfc, uvbf0, nirbm, nirdf, visbm, visdf}
      a->nirbmdi[i] = c[2];
      a->nirdfdi[i] = c[3];
      a->visbmdi[i] = c[4];
      a->visdfdi[i] = c[5];
      a->nirbmui[i] = c[2] * a->sfcalb1[i];
      a->nirdfui[i] = c[3] * a->sfcalb2[i];
      a->visbmui[i] = c[4] * a->sfcalb3[i];
      a->visdfui[i] = c[5] * a->sfcalb4[i];
    }
  } else {
    for (size_t e = 0; e < (size_t)im * levs; ++e) a->htrsw[e] = 0.0;
    for (int i = 0; i < im; ++i) {
      for (int j = 0; j < 4; ++j) a->sfcfsw[4 * (size_t)i + j] = 0.0;
      for (int j = 0; j < 3; ++j) a->topfsw[3 * (size_t)i + j] = 0.0;
      for (int j = 0; j < 6; ++j) a->scmpsw[6 * (size_t)i + j] = 0.0;
      a->nirbmdi[i] = a->nirdfdi[i] = a->visbmdi[i] = a->visdfdi[i] = 0.0;
      a->nirbmui[i] = a->nirdfui[i] = a->visbmui[i] = a->visdfui[i] = 0.0;
    }
    if (a->swhtr)
      for (size_t e = 0; e < (size_t)im * levs; ++e) a->swhc[e] = 0.0;
  }
  for (int i = 0; i < im; ++i) {
    const double* f = a->sfcfsw + 4 * (size_t)i;   // {upfxc, dnfxc, upfx0, dnfx0}
    a->sfcnsw[i] = f[1] - f[0];
    a->sfcdsw[i] = f[1];
  }
}

}  // extern "C"
