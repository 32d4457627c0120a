// rrtmg_lw_oracle.cpp -- CPU restatement of the RRTMG-LW column path.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only the tests, the smoke check and
// bench.py's CPU-baseline / reference arm may load this library.  It is the
// parity checker for the GPU library and the timed CPU baseline ("port").
//
// It restates, statement by statement and in the same floating-point order,
// the Fortran of ccpp-physics:
//   physics/Radiation/RRTMG/radlw_main.F90   (RLM below)
//     rrtmg_lw_run driver      RLM:419-1309
//     rlwinit tables           RLM:1322-1504
//     cldprop                  RLM:1530-1834
//     mcica_subcol             RLM:1847-2107
//     setcoef                  RLM:2151-2406
//     rtrnmc                   RLM:3420-3785
//     taumol, taugb01..16      RLM:3836-6840
//   physics/Radiation/mersenne_twister.f      random_setseed_t MT:285-299,
//                                             random_number_t  MT:330-372
//   physics/Radiation/RRTMG/radlw_param.f     band layout :103-142
// and the steps either side of rrtmg_lw_run:
//   physics/Radiation/mersenne_twister.f      random_index_t MT:489-503
//   physics/Interstitials/UFS_SCM_NEPTUNE/GFS_rad_time_vary.fv3.F90:59-84
//   physics/Radiation/radiation_cloud_overlap.F90:28-145, radiation_clouds.f:837-856
//   physics/Radiation/RRTMG/rrtmg_lw_post.F90:13-77
//   physics/hooks/physcons.F90                constants :52,66,107,110-112
// Arithmetic is IEEE binary64 with FMA contraction disabled
// (-ffp-contract=off), Fortran int() = truncation toward zero, mod(x,1.) =
// fmod.  Literals are binary64 (promoted-real build, kind_phys = 8).
//
// Parity of this restatement is NOT pinned by the reference itself: the
// reference is Fortran, no Fortran compiler exists in this environment and
// the reference tree holds no tests or golden vectors for this path.  The
// Mersenne-Twister core is pinned against numpy's independent MT19937 and
// the coefficient tables against literals read from radlw_datatb.f.
//
// The coefficient tables come from the blob written by
// ccpp_physics_b200/data/extract_tables.py (the DATA statements of
// radlw_datatb.f); the path is given to oracle_rlwinit.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../include/rrtmg_lw_gpu.h"
#include "../ccpp_physics_b200/data/rrtmg_lw_table_layout.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- constants (RLM:309-317, physcons.F90:52,66,107,110-112) -------------
const double con_g = 9.80665, con_cp = 1.0046e+3, con_avgd = 6.0221415e23;
const double con_amd = 28.9644, con_amw = 18.0154, con_amo3 = 47.9982;
const double eps = 1.0e-6;
const double oneminus = 1.0 - eps;
const double cldmin = DBL_MIN;          // tiny(cldmin)
const double bpade = 1.0 / 0.278;
const double stpfac = 296.0 / 1013.0;
const double wtdiff = 0.5;
const double tblint = 10000.0;          // ntbl
const double f_zero = 0.0, f_one = 1.0;
const double amdw = con_amd / con_amw;
const double amdo3 = con_amd / con_amo3;

const int NBANDS = 16, NGPT = 140, NTBL = 10000, MAXGAS = 7, MAXXSEC = 4;
// radlw_param.f:111-127
const int NGB_NG[16] = {10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2};
const int NS[16] = {0, 10, 22, 38, 52, 68, 76, 88, 96, 108, 114, 122, 130, 134, 136, 138};
// RLM:326-327
const int nspa[16] = {1, 1, 9, 9, 9, 1, 9, 1, 9, 1, 1, 9, 9, 1, 9, 9};
const int nspb[16] = {1, 1, 5, 5, 5, 0, 1, 1, 1, 1, 1, 0, 0, 1, 0, 0};
// radlw_param.f:141-142
const double delwave[16] = {340., 150., 130., 70., 120., 160., 100., 100.,
                            210., 90., 320., 280., 170., 130., 220., 650.};
// RLM:347-354
const double a0[16] = {1.66, 1.55, 1.58, 1.66, 1.54, 1.454, 1.89, 1.33,
                       1.668, 1.66, 1.66, 1.66, 1.66, 1.66, 1.66, 1.66};
const double a1[16] = {0.00, 0.25, 0.22, 0.00, 0.13, 0.446, -0.10, 0.40,
                       -0.006, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00};
const double a2[16] = {0.00, -12.0, -11.7, 0.00, -0.72, -0.243, 0.19, -0.062,
                       0.414, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00, 0.00};
const double absrain = 0.33e-3, abssnow0 = 1.5;  // radlw_datatb.f:941,944

// ---- module state set by rlwinit ------------------------------------------
std::vector<double> T;   // coefficient tables (Fortran order)
double fluxfac = 0, heatfac = 0;
double tau_tbl[NTBL + 1], exp_tbl[NTBL + 1], tfn_tbl[NTBL + 1];
int ngb[NGPT];            // 1-based band of each g-point
bool g_init = false;

inline double t1(int off, int i) { return T[off + (i - 1)]; }
inline double t2(int off, int n1, int i, int j) { return T[off + (i - 1) + n1 * (j - 1)]; }
inline double t3(int off, int n1, int n2, int i, int j, int k) {
  return T[off + (i - 1) + n1 * ((j - 1) + n2 * (k - 1))];
}
inline double ipow4(double p) { double p2 = p * p; return p2 * p2; }  // p**4
inline int fint(double x) { return (int)x; }                          // Fortran int()
inline double fmod1(double x) { return std::fmod(x, 1.0); }           // mod(x, 1.)

// ---- per-column work arrays (Fortran index helpers) ------------------------
struct Col {
  int nlay, nlp1;
  std::vector<double> pavel, tavel, delp, dz, tz, h2ovmr, o3vmr, coldry, temcol, colbrd;
  std::vector<double> colamt, wx, tauaer, cldfrc, clwp, relw, ciwp, reiw, cda1, cda2, cda3,
      cda4, alph;
  double semiss[16], secdiff[16], pwvcm, stemp, delgth;
  int laytrop;
  std::vector<int> jp, jt, jt1, indself, indfor, indminor;
  std::vector<double> fac00, fac01, fac10, fac11, selffac, selffrac, forfac, forfrac, minorfrac,
      scaleminor, scaleminorn2, rfrate, pklay, pklev;
  std::vector<double> taucld, cldfmc, taug, fracs, tautot;
  std::vector<uint8_t> lcloudy;
  std::vector<double> totuflux, totdflux, totuclfl, totdclfl, htr, htrcl, htrb;
  explicit Col(int n) : nlay(n), nlp1(n + 1) {
    auto r = [&](std::vector<double>& v, size_t s) { v.assign(s, 0.0); };
    for (auto* v : {&pavel, &tavel, &delp, &dz, &h2ovmr, &o3vmr, &coldry, &temcol, &colbrd,
                    &clwp, &relw, &ciwp, &reiw, &cda1, &cda2, &cda3, &cda4, &alph, &fac00,
                    &fac01, &fac10, &fac11, &selffac, &selffrac, &forfac, &forfrac, &minorfrac,
                    &scaleminor, &scaleminorn2, &htr, &htrcl})
      r(*v, n);
    r(tz, n + 1);
    r(colamt, (size_t)n * MAXGAS);
    r(wx, (size_t)n * MAXXSEC);
    r(tauaer, (size_t)NBANDS * n);
    r(cldfrc, n + 2);
    r(rfrate, (size_t)n * 6 * 2);
    r(pklay, (size_t)NBANDS * (n + 1));
    r(pklev, (size_t)NBANDS * (n + 1));
    r(taucld, (size_t)NBANDS * n);
    r(cldfmc, (size_t)NGPT * n);
    r(taug, (size_t)NGPT * n);
    r(fracs, (size_t)NGPT * n);
    r(tautot, (size_t)NGPT * n);
    r(htrb, (size_t)n * NBANDS);
    for (auto* v : {&totuflux, &totdflux, &totuclfl, &totdclfl}) r(*v, n + 1);
    lcloudy.assign((size_t)NGPT * n, 0);
    jp.assign(n, 0); jt.assign(n, 0); jt1.assign(n, 0);
    indself.assign(n, 0); indfor.assign(n, 0); indminor.assign(n, 0);
  }
  // Fortran-style 1-based accessors
  double& COL(int k, int m) { return colamt[(k - 1) + nlay * (m - 1)]; }
  double& WX(int k, int m) { return wx[(k - 1) + nlay * (m - 1)]; }
  double& TAUAER(int b, int k) { return tauaer[(b - 1) + NBANDS * (k - 1)]; }
  double& RF(int k, int m, int n) { return rfrate[(k - 1) + nlay * ((m - 1) + 6 * (n - 1))]; }
  double& PKLAY(int b, int k) { return pklay[(b - 1) + NBANDS * k]; }   // k = 0..nlay
  double& PKLEV(int b, int k) { return pklev[(b - 1) + NBANDS * k]; }
  double& TAUCLD(int b, int k) { return taucld[(b - 1) + NBANDS * (k - 1)]; }
  double& CLDFMC(int g, int k) { return cldfmc[(g - 1) + NGPT * (k - 1)]; }
  double& TAUG(int g, int k) { return taug[(g - 1) + NGPT * (k - 1)]; }
  double& FRACS(int g, int k) { return fracs[(g - 1) + NGPT * (k - 1)]; }
  double& TAUTOT(int g, int k) { return tautot[(g - 1) + NGPT * (k - 1)]; }
  double& HTRB(int k, int b) { return htrb[(k - 1) + nlay * (b - 1)]; }
  // 0-based index arrays used 1-based
  int& JP(int k) { return jp[k - 1]; }
  int& JT(int k) { return jt[k - 1]; }
  int& JT1(int k) { return jt1[k - 1]; }
};

// ---- Mersenne twister (mersenne_twister.f:162-372) ------------------------
struct MTState { uint32_t mt[624]; int mti; };
const uint32_t MATA = 0x9908B0DFu, UMASK = 0x80000000u, LMASK = 0x7FFFFFFFu;
const uint32_t TMASKB = 0x9D2C5680u, TMASKC = 0xEFC60000u;

// random_setseed_t (MT:285-299): mt(0) = seed (0 -> 4357), mt(i) = 69069*mt(i-1)
void mt_setseed(MTState& s, int32_t inseed) {
  int32_t ii = inseed;
  if (ii == 0) ii = 4357;
  s.mti = 624;
  s.mt[0] = (uint32_t)ii;
  for (int i = 1; i < 624; ++i) s.mt[i] = 69069u * s.mt[i - 1];
}
inline uint32_t mt_mag(uint32_t y) { return (y & 1u) ? MATA : 0u; }
// random_number_t (MT:330-372): twist every 624 draws, temper, u32/(2^32-1)
uint32_t mt_next_u32(MTState& s) {
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
  return y;
}
inline double mt_u32_to_real(uint32_t y) { return (double)y / 4294967295.0; }

// ---- mcica_subcol (RLM:1847-2107) -----------------------------------------
void mcica_subcol(Col& c, const std::vector<double>& cldf, int ipseed, int iovr) {
  const int nlay = c.nlay;
  std::vector<double> cdfunc((size_t)NGPT * nlay), cdfun2((size_t)NGPT * nlay), fac_lcf(nlay + 1);
  auto CDF = [&](int n, int k) -> double& { return cdfunc[(n - 1) + NGPT * (k - 1)]; };
  auto CD2 = [&](int n, int k) -> double& { return cdfun2[(n - 1) + NGPT * (k - 1)]; };
  MTState st;
  mt_setseed(st, ipseed);
  switch (iovr) {
    case 0:
    case 1: {
      // rand2d index k1 = (n-1)*nlay + k (RLM:1920-1926 / 1935-1941)
      for (int n = 1; n <= NGPT; ++n)
        for (int k = 1; k <= nlay; ++k) CDF(n, k) = mt_u32_to_real(mt_next_u32(st));
      if (iovr == 1) {
        for (int k = 2; k <= nlay; ++k) {  // bottom up (RLM:1949-1960)
          int k1 = k - 1;
          double tem1 = f_one - cldf[k1 - 1];
          for (int n = 1; n <= NGPT; ++n) {
            if (CDF(n, k1) > tem1) CDF(n, k) = CDF(n, k1);
            else CDF(n, k) = CDF(n, k) * tem1;
          }
        }
      }
      break;
    }
    case 2: {  // RLM:1981-1993
      double rand1d[NGPT];
      for (int n = 0; n < NGPT; ++n) rand1d[n] = mt_u32_to_real(mt_next_u32(st));
      for (int n = 1; n <= NGPT; ++n)
        for (int k = 1; k <= nlay; ++k) CDF(n, k) = rand1d[n - 1];
      break;
    }
    case 3: {  // RLM:1995-2035
      for (int k = nlay; k >= 2; --k)
        fac_lcf[k] = std::exp(-0.5 * (c.dz[k - 1] + c.dz[k - 2]) / c.delgth);
      for (int k = 1; k <= nlay; ++k)
        for (int n = 1; n <= NGPT; ++n) CDF(n, k) = mt_u32_to_real(mt_next_u32(st));
      for (int k = 1; k <= nlay; ++k)
        for (int n = 1; n <= NGPT; ++n) CD2(n, k) = mt_u32_to_real(mt_next_u32(st));
      for (int k = nlay - 1; k >= 1; --k) {
        int k1 = k + 1;
        for (int n = 1; n <= NGPT; ++n)
          if (CD2(n, k) <= fac_lcf[k1]) CDF(n, k) = CDF(n, k1);
      }
      break;
    }
    case 4:
    case 5: {  // RLM:2037-2091
      for (int k = 1; k <= nlay; ++k)
        for (int n = 1; n <= NGPT; ++n) CDF(n, k) = mt_u32_to_real(mt_next_u32(st));
      for (int k = 1; k <= nlay; ++k)
        for (int n = 1; n <= NGPT; ++n) CD2(n, k) = mt_u32_to_real(mt_next_u32(st));
      for (int k = 2; k <= nlay; ++k) {
        int k1 = k - 1;
        for (int n = 1; n <= NGPT; ++n)
          if (CD2(n, k) < c.alph[k - 1]) CDF(n, k) = CDF(n, k1);
      }
      break;
    }
    default:
      break;  // cdfunc undefined in the reference; left zero here
  }
  for (int k = 1; k <= nlay; ++k) {  // RLM:2097-2103
    double tem1 = f_one - cldf[k - 1];
    for (int n = 1; n <= NGPT; ++n) c.lcloudy[(n - 1) + NGPT * (k - 1)] = CDF(n, k) >= tem1;
  }
}

// ---- cldprop (RLM:1530-1834) ----------------------------------------------
void cldprop(Col& c, int ipseed, int iovr, int ilwcliq, int ilwcice, int isubclw) {
  const int nlay = c.nlay;
  double tauliq[16], tauice[16];
  std::fill(c.taucld.begin(), c.taucld.end(), 0.0);
  std::fill(c.cldfmc.begin(), c.cldfmc.end(), 0.0);
  if (ilwcliq > 0) {
    for (int k = 1; k <= nlay; ++k) {
      if (!(c.cldfrc[k] > cldmin)) continue;
      double tauran = absrain * c.cda1[k - 1];
      double tausnw;
      if (c.cda3[k - 1] > f_zero && c.cda4[k - 1] > 10.0)
        tausnw = abssnow0 * 1.05756 * c.cda3[k - 1] / c.cda4[k - 1];
      else
        tausnw = f_zero;
      double cldliq = c.clwp[k - 1], cldice = c.ciwp[k - 1];
      double refliq = c.relw[k - 1], refice = c.reiw[k - 1];
      if (cldliq <= f_zero) {
        for (int ib = 0; ib < 16; ++ib) tauliq[ib] = f_zero;
      } else {
        // only ilwcliq == 1 defines tauliq in the reference; others leave it unset
        for (int ib = 0; ib < 16; ++ib) tauliq[ib] = f_zero;
        if (ilwcliq == 1) {
          double factor = refliq - 1.5;
          int index = std::max(1, std::min(57, fint(factor)));
          double fint_ = factor - (double)index;
          for (int ib = 1; ib <= 16; ++ib) {
            double a = t2(lwtab::absliq1, 58, index, ib), b = t2(lwtab::absliq1, 58, index + 1, ib);
            tauliq[ib - 1] = std::max(f_zero, cldliq * (a + fint_ * (b - a)));
          }
        }
      }
      if (cldice <= f_zero) {
        for (int ib = 0; ib < 16; ++ib) tauice[ib] = f_zero;
      } else {
        for (int ib = 0; ib < 16; ++ib) tauice[ib] = f_zero;
        if (ilwcice == 1) {
          refice = std::min(130.0, std::max(13.0, refice));
          for (int ib = 1; ib <= 16; ++ib) {
            int ia = (int)t1(lwtab::ipat, ib);
            tauice[ib - 1] = std::max(f_zero, cldice * (t2(lwtab::absice1, 2, 1, ia) +
                                                         t2(lwtab::absice1, 2, 2, ia) / refice));
          }
        } else if (ilwcice == 2) {
          double factor = (refice - 2.0) / 3.0;
          int index = std::max(1, std::min(42, fint(factor)));
          double fint_ = factor - (double)index;
          for (int ib = 1; ib <= 16; ++ib) {
            double a = t2(lwtab::absice2, 43, index, ib), b = t2(lwtab::absice2, 43, index + 1, ib);
            tauice[ib - 1] = std::max(f_zero, cldice * (a + fint_ * (b - a)));
          }
        } else if (ilwcice == 3) {
          double dgeice = std::max(5.0, 1.0315 * refice);
          double factor = (dgeice - 2.0) / 3.0;
          int index = std::max(1, std::min(45, fint(factor)));
          double fint_ = factor - (double)index;
          for (int ib = 1; ib <= 16; ++ib) {
            double a = t2(lwtab::absice3, 46, index, ib), b = t2(lwtab::absice3, 46, index + 1, ib);
            tauice[ib - 1] = std::max(f_zero, cldice * (a + fint_ * (b - a)));
          }
        }
      }
      for (int ib = 1; ib <= 16; ++ib)
        c.TAUCLD(ib, k) = tauice[ib - 1] + tauliq[ib - 1] + tauran + tausnw;
    }
  } else {
    for (int k = 1; k <= nlay; ++k)
      if (c.cldfrc[k] > cldmin)
        for (int ib = 1; ib <= 16; ++ib) c.TAUCLD(ib, k) = c.cda1[k - 1];
  }
  if (isubclw > 0) {  // RLM:1803-1829
    std::vector<double> cldf(nlay);
    for (int k = 1; k <= nlay; ++k) cldf[k - 1] = (c.cldfrc[k] < cldmin) ? f_zero : c.cldfrc[k];
    mcica_subcol(c, cldf, ipseed, iovr);
    for (int k = 1; k <= nlay; ++k)
      for (int ig = 1; ig <= NGPT; ++ig)
        c.CLDFMC(ig, k) = c.lcloudy[(ig - 1) + NGPT * (k - 1)] ? f_one : f_zero;
  }
}

// ---- setcoef (RLM:2151-2406) ----------------------------------------------
void setcoef(Col& c) {
  const int nlay = c.nlay;
  const int TP = lwtab::totplnk;  // totplnk(181,16)
  auto totplnk = [&](int i, int b) { return t2(TP, 181, i, b); };
  auto preflog = [&](int j) { return t1(lwtab::preflog, j); };
  auto tref = [&](int j) { return t1(lwtab::tref, j); };
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };

  int indlay = std::min(180, std::max(1, fint(c.stemp - 159.0)));
  int indlev = std::min(180, std::max(1, fint(c.tz[0] - 159.0)));
  double tlyrfr = c.stemp - fint(c.stemp);
  double tlvlfr = c.tz[0] - fint(c.tz[0]);
  for (int i = 1; i <= NBANDS; ++i) {
    double tem1 = totplnk(indlay + 1, i) - totplnk(indlay, i);
    double tem2 = totplnk(indlev + 1, i) - totplnk(indlev, i);
    c.PKLAY(i, 0) = delwave[i - 1] * (totplnk(indlay, i) + tlyrfr * tem1);
    c.PKLEV(i, 0) = delwave[i - 1] * (totplnk(indlev, i) + tlvlfr * tem2);
  }
  c.laytrop = 0;
  for (int k = 1; k <= nlay; ++k) {
    double tav = c.tavel[k - 1], pav = c.pavel[k - 1];
    indlay = std::min(180, std::max(1, fint(tav - 159.0)));
    tlyrfr = tav - fint(tav);
    indlev = std::min(180, std::max(1, fint(c.tz[k] - 159.0)));
    tlvlfr = c.tz[k] - fint(c.tz[k]);
    for (int i = 1; i <= NBANDS; ++i) {
      c.PKLAY(i, k) = delwave[i - 1] * (totplnk(indlay, i) +
                                         tlyrfr * (totplnk(indlay + 1, i) - totplnk(indlay, i)));
      c.PKLEV(i, k) = delwave[i - 1] * (totplnk(indlev, i) +
                                         tlvlfr * (totplnk(indlev + 1, i) - totplnk(indlev, i)));
    }
    double plog = std::log(pav);
    c.JP(k) = std::max(1, std::min(58, fint(36.0 - 5.0 * (plog + 0.04))));
    int jp1 = c.JP(k) + 1;
    double fp = std::max(f_zero, std::min(f_one, 5.0 * (preflog(c.JP(k)) - plog)));
    double tem1 = (tav - tref(c.JP(k))) / 15.0;
    double tem2 = (tav - tref(jp1)) / 15.0;
    c.JT(k) = std::max(1, std::min(4, fint(3.0 + tem1)));
    c.JT1(k) = std::max(1, std::min(4, fint(3.0 + tem2)));
    double ft = std::max(-0.5, std::min(1.5, tem1 - (double)(c.JT(k) - 3)));
    double ft1 = std::max(-0.5, std::min(1.5, tem2 - (double)(c.JT1(k) - 3)));
    tem1 = f_one - fp;
    c.fac10[k - 1] = tem1 * ft;
    c.fac00[k - 1] = tem1 * (f_one - ft);
    c.fac11[k - 1] = fp * ft1;
    c.fac01[k - 1] = fp * (f_one - ft1);
    c.forfac[k - 1] = pav * stpfac / (tav * (1.0 + c.h2ovmr[k - 1]));
    c.selffac[k - 1] = c.h2ovmr[k - 1] * c.forfac[k - 1];
    c.scaleminor[k - 1] = pav / tav;
    c.scaleminorn2[k - 1] = (pav / tav) * (c.colbrd[k - 1] / (c.coldry[k - 1] + c.COL(k, 1)));
    tem1 = (tav - 180.8) / 7.2;
    c.indminor[k - 1] = std::min(18, std::max(1, fint(tem1)));
    c.minorfrac[k - 1] = tem1 - (double)c.indminor[k - 1];
    int j = c.JP(k);
    if (plog > 4.56) {
      c.laytrop = c.laytrop + 1;
      tem1 = (332.0 - tav) / 36.0;
      c.indfor[k - 1] = std::min(2, std::max(1, fint(tem1)));
      c.forfrac[k - 1] = tem1 - (double)c.indfor[k - 1];
      tem1 = (tav - 188.0) / 7.2;
      c.indself[k - 1] = std::min(9, std::max(1, fint(tem1) - 7));
      c.selffrac[k - 1] = tem1 - (double)(c.indself[k - 1] + 7);
      c.RF(k, 1, 1) = chi(1, j) / chi(2, j);
      c.RF(k, 1, 2) = chi(1, j + 1) / chi(2, j + 1);
      c.RF(k, 2, 1) = chi(1, j) / chi(3, j);
      c.RF(k, 2, 2) = chi(1, j + 1) / chi(3, j + 1);
      c.RF(k, 3, 1) = chi(1, j) / chi(4, j);
      c.RF(k, 3, 2) = chi(1, j + 1) / chi(4, j + 1);
      c.RF(k, 4, 1) = chi(1, j) / chi(6, j);
      c.RF(k, 4, 2) = chi(1, j + 1) / chi(6, j + 1);
      c.RF(k, 5, 1) = chi(4, j) / chi(2, j);
      c.RF(k, 5, 2) = chi(4, j + 1) / chi(2, j + 1);
    } else {
      tem1 = (tav - 188.0) / 36.0;
      c.indfor[k - 1] = 3;
      c.forfrac[k - 1] = tem1 - f_one;
      c.indself[k - 1] = 0;
      c.selffrac[k - 1] = f_zero;
      c.RF(k, 1, 1) = chi(1, j) / chi(2, j);
      c.RF(k, 1, 2) = chi(1, j + 1) / chi(2, j + 1);
      c.RF(k, 6, 1) = chi(3, j) / chi(2, j);
      c.RF(k, 6, 2) = chi(3, j + 1) / chi(2, j + 1);
    }
    c.selffac[k - 1] = c.COL(k, 1) * c.selffac[k - 1];
    c.forfac[k - 1] = c.COL(k, 1) * c.forfac[k - 1];
  }
}

// ---- taumol helpers ----------------------------------------------------------
// 3-point (near the species-range ends) or 2-point species interpolation of
// the lower-atmosphere binary-species bands (e.g. RLM:4299-4333).
struct Sp3 { double f0, f1, f2; int d0, d1, d2, e0, e1, e2; };  // fk and id offsets
inline Sp3 species3(double specparm, double fs, int ind) {
  Sp3 s;
  if (specparm < 0.125) {
    double p = fs - f_one, p4 = ipow4(p);
    s.f0 = p4; s.f1 = f_one - p - 2.0 * p4; s.f2 = p + p4;
    s.d0 = ind; s.e0 = ind + 9; s.d1 = ind + 1; s.e1 = ind + 10; s.d2 = ind + 2; s.e2 = ind + 11;
  } else if (specparm > 0.875) {
    double p = -fs, p4 = ipow4(p);
    s.f0 = p4; s.f1 = f_one - p - 2.0 * p4; s.f2 = p + p4;
    s.d0 = ind + 1; s.e0 = ind + 10; s.d1 = ind; s.e1 = ind + 9; s.d2 = ind - 1; s.e2 = ind + 8;
  } else {
    s.f0 = f_one - fs; s.f1 = fs; s.f2 = f_zero;
    s.d0 = ind; s.e0 = ind + 9; s.d1 = ind + 1; s.e1 = ind + 10; s.d2 = ind; s.e2 = ind;
  }
  return s;
}
// fac000..fac210 of one reference pressure: (fk0,fk1,fk2) x (fac_0, fac_1)
struct Fac6 { double f000, f100, f200, f010, f110, f210; };
inline Fac6 fac6(const Sp3& s, double facA, double facB) {
  return {s.f0 * facA, s.f1 * facA, s.f2 * facA, s.f0 * facB, s.f1 * facB, s.f2 * facB};
}
// sum  fac000*a(id000) + fac010*a(id010) + fac100*a(id100) + fac110*a(id110)
//    + fac200*a(id200) + fac210*a(id210)   (left to right as written)
inline double major6(int off, int ng, int ig, const Sp3& s, const Fac6& f) {
  return f.f000 * t2(off, ng, ig, s.d0) + f.f010 * t2(off, ng, ig, s.e0) +
         f.f100 * t2(off, ng, ig, s.d1) + f.f110 * t2(off, ng, ig, s.e1) +
         f.f200 * t2(off, ng, ig, s.d2) + f.f210 * t2(off, ng, ig, s.e2);
}
// 2-point interpolation of the upper-atmosphere binary-species bands
inline double major4(int off, int ng, int ig, int i0, double f000, double f010, double f100,
                     double f110, int dt) {
  return f000 * t2(off, ng, ig, i0) + f010 * t2(off, ng, ig, i0 + dt) +
         f100 * t2(off, ng, ig, i0 + 1) + f110 * t2(off, ng, ig, i0 + dt + 1);
}
inline double lerp(double a, double f, double b) { return a + f * (b - a); }

// Species parameter (speccomb / specparm / specmult / js / fs)
struct Spec { double comb, parm, mult, fs; int js; };
inline Spec spec(double a, double rat, double b, double nbin) {
  Spec s;
  s.comb = a + rat * b;
  s.parm = a / s.comb;
  s.mult = nbin * std::min(s.parm, oneminus);
  s.js = 1 + fint(s.mult);
  s.fs = fmod1(s.mult);
  return s;
}

// ---- taugb01 (RLM:4023-4125) ----
void taugb01(Col& c) {
  const int ng = 10, b = 1;
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = ((c.JP(k) - 1) * 5 + (c.JT(k) - 1)) * nspa[b - 1] + 1;
    int ind1 = (c.JP(k) * 5 + (c.JT1(k) - 1)) * nspa[b - 1] + 1;
    int inds = c.indself[k - 1], indf = c.indfor[k - 1], indm = c.indminor[k - 1];
    double pp = c.pavel[k - 1];
    double scalen2 = c.colbrd[k - 1] * c.scaleminorn2[k - 1];
    double corradj = (pp < 250.0) ? f_one - 0.15 * (250.0 - pp) / 154.4 : f_one;
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = c.selffac[k - 1] * lerp(t2(lwtab::b01_selfref, ng, ig, inds), c.selffrac[k - 1], t2(lwtab::b01_selfref, ng, ig, inds + 1));
      double taufor = c.forfac[k - 1] * lerp(t2(lwtab::b01_forref, ng, ig, indf), c.forfrac[k - 1], t2(lwtab::b01_forref, ng, ig, indf + 1));
      double taun2 = scalen2 * lerp(t2(lwtab::b01_ka_mn2, ng, ig, indm), c.minorfrac[k - 1], t2(lwtab::b01_ka_mn2, ng, ig, indm + 1));
      c.TAUG(ig, k) = corradj * (c.COL(k, 1) * (c.fac00[k - 1] * t2(lwtab::b01_absa, ng, ig, ind0) + c.fac10[k - 1] * t2(lwtab::b01_absa, ng, ig, ind0 + 1) +
                                                c.fac01[k - 1] * t2(lwtab::b01_absa, ng, ig, ind1) + c.fac11[k - 1] * t2(lwtab::b01_absa, ng, ig, ind1 + 1)) +
                                 tauself + taufor + taun2);
      c.FRACS(ig, k) = t1(lwtab::b01_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = ((c.JP(k) - 13) * 5 + (c.JT(k) - 1)) * nspb[b - 1] + 1;
    int ind1 = ((c.JP(k) - 12) * 5 + (c.JT1(k) - 1)) * nspb[b - 1] + 1;
    int indf = c.indfor[k - 1], indm = c.indminor[k - 1];
    double scalen2 = c.colbrd[k - 1] * c.scaleminorn2[k - 1];
    double corradj = f_one - 0.15 * (c.pavel[k - 1] / 95.6);
    for (int ig = 1; ig <= ng; ++ig) {
      double taufor = c.forfac[k - 1] * lerp(t2(lwtab::b01_forref, ng, ig, indf), c.forfrac[k - 1], t2(lwtab::b01_forref, ng, ig, indf + 1));
      double taun2 = scalen2 * lerp(t2(lwtab::b01_kb_mn2, ng, ig, indm), c.minorfrac[k - 1], t2(lwtab::b01_kb_mn2, ng, ig, indm + 1));
      c.TAUG(ig, k) = corradj * (c.COL(k, 1) * (c.fac00[k - 1] * t2(lwtab::b01_absb, ng, ig, ind0) + c.fac10[k - 1] * t2(lwtab::b01_absb, ng, ig, ind0 + 1) +
                                                c.fac01[k - 1] * t2(lwtab::b01_absb, ng, ig, ind1) + c.fac11[k - 1] * t2(lwtab::b01_absb, ng, ig, ind1 + 1)) +
                                 taufor + taun2);
      c.FRACS(ig, k) = t1(lwtab::b01_fracrefb, ig);
    }
  }
}

// Common body of the single-key-species bands' 4-point interpolation.
inline double absk(Col& c, int k, int off, int ng, int ig, int ind0, int ind1) {
  return c.fac00[k - 1] * t2(off, ng, ig, ind0) + c.fac10[k - 1] * t2(off, ng, ig, ind0 + 1) +
         c.fac01[k - 1] * t2(off, ng, ig, ind1) + c.fac11[k - 1] * t2(off, ng, ig, ind1 + 1);
}
inline int lowind(Col& c, int k, int jt, int ns) { return ((c.JP(k) - 1) * 5 + (jt - 1)) * ns; }
inline int lowind1(Col& c, int k, int jt, int ns) { return (c.JP(k) * 5 + (jt - 1)) * ns; }
inline int upind(Col& c, int k, int jt, int ns) { return ((c.JP(k) - 13) * 5 + (jt - 1)) * ns; }
inline int upind1(Col& c, int k, int jt, int ns) { return ((c.JP(k) - 12) * 5 + (jt - 1)) * ns; }
inline double selfcont(Col& c, int k, int off, int ng, int ig) {
  int inds = c.indself[k - 1];
  return c.selffac[k - 1] * lerp(t2(off, ng, ig, inds), c.selffrac[k - 1], t2(off, ng, ig, inds + 1));
}
inline double forcont(Col& c, int k, int off, int ng, int ig) {
  int indf = c.indfor[k - 1];
  return c.forfac[k - 1] * lerp(t2(off, ng, ig, indf), c.forfrac[k - 1], t2(off, ng, ig, indf + 1));
}
inline double minor2(Col& c, int k, int off, int ng, int ig) {
  int indm = c.indminor[k - 1];
  return lerp(t2(off, ng, ig, indm), c.minorfrac[k - 1], t2(off, ng, ig, indm + 1));
}
// 3-D minor table m(ig, js, indm) interpolated in js (fraction f) then in T
inline double minor3(Col& c, int k, int off, int ng, int nj, int ig, int j, double f) {
  int indm = c.indminor[k - 1];
  double m1 = t3(off, ng, nj, ig, j, indm) + f * (t3(off, ng, nj, ig, j + 1, indm) - t3(off, ng, nj, ig, j, indm));
  double m2 = t3(off, ng, nj, ig, j, indm + 1) + f * (t3(off, ng, nj, ig, j + 1, indm + 1) - t3(off, ng, nj, ig, j, indm + 1));
  return m1 + c.minorfrac[k - 1] * (m2 - m1);
}

// ---- taugb02 (RLM:4131-4203) ----
void taugb02(Col& c) {
  const int ng = 12, b = 2, ns = NS[b - 1];
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = lowind(c, k, c.JT(k), nspa[b - 1]) + 1, ind1 = lowind1(c, k, c.JT1(k), nspa[b - 1]) + 1;
    double corradj = f_one - 0.05 * (c.pavel[k - 1] - 100.0) / 900.0;
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b02_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b02_forref, ng, ig);
      c.TAUG(ns + ig, k) = corradj * (c.COL(k, 1) * absk(c, k, lwtab::b02_absa, ng, ig, ind0, ind1) + tauself + taufor);
      c.FRACS(ns + ig, k) = t1(lwtab::b02_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      double taufor = forcont(c, k, lwtab::b02_forref, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b02_absb, ng, ig, ind0, ind1) + taufor;
      c.FRACS(ns + ig, k) = t1(lwtab::b02_fracrefb, ig);
    }
  }
}

// Lower-atmosphere binary-species set-up shared by bands 3,4,5,7,9,12,13,15,16
struct Lower {
  Spec s0, s1; int ind0, ind1; Sp3 p0, p1; Fac6 f0, f1;
};
inline Lower lower_setup(Col& c, int k, int b, double a, double rat0, double rat1, double bb) {
  Lower L;
  L.s0 = spec(a, rat0, bb, 8.0);
  L.ind0 = ((c.JP(k) - 1) * 5 + (c.JT(k) - 1)) * nspa[b - 1] + L.s0.js;
  L.s1 = spec(a, rat1, bb, 8.0);
  L.ind1 = (c.JP(k) * 5 + (c.JT1(k) - 1)) * nspa[b - 1] + L.s1.js;
  L.p0 = species3(L.s0.parm, L.s0.fs, L.ind0);
  L.f0 = fac6(L.p0, c.fac00[k - 1], c.fac10[k - 1]);
  L.p1 = species3(L.s1.parm, L.s1.fs, L.ind1);
  L.f1 = fac6(L.p1, c.fac01[k - 1], c.fac11[k - 1]);
  return L;
}
// Upper-atmosphere binary-species set-up shared by bands 3,4,5
struct Upper { Spec s0, s1; int ind0, ind1; double f000, f010, f100, f110, f001, f011, f101, f111; };
inline Upper upper_setup(Col& c, int k, int b, double a, double rat0, double rat1, double bb) {
  Upper U;
  U.s0 = spec(a, rat0, bb, 4.0);
  U.ind0 = ((c.JP(k) - 13) * 5 + (c.JT(k) - 1)) * nspb[b - 1] + U.s0.js;
  U.s1 = spec(a, rat1, bb, 4.0);
  U.ind1 = ((c.JP(k) - 12) * 5 + (c.JT1(k) - 1)) * nspb[b - 1] + U.s1.js;
  double fk0 = f_one - U.s0.fs, fk1 = U.s0.fs;
  U.f000 = fk0 * c.fac00[k - 1]; U.f010 = fk0 * c.fac10[k - 1];
  U.f100 = fk1 * c.fac00[k - 1]; U.f110 = fk1 * c.fac10[k - 1];
  fk0 = f_one - U.s1.fs; fk1 = U.s1.fs;
  U.f001 = fk0 * c.fac01[k - 1]; U.f011 = fk0 * c.fac11[k - 1];
  U.f101 = fk1 * c.fac01[k - 1]; U.f111 = fk1 * c.fac11[k - 1];
  return U;
}
inline double lower_major(const Lower& L, int off, int ng, int ig) {
  return L.s0.comb * major6(off, ng, ig, L.p0, L.f0) + L.s1.comb * major6(off, ng, ig, L.p1, L.f1);
}
inline double upper_major(const Upper& U, int off, int ng, int ig) {
  return U.s0.comb * major4(off, ng, ig, U.ind0, U.f000, U.f010, U.f100, U.f110, 5) +
         U.s1.comb * major4(off, ng, ig, U.ind1, U.f001, U.f011, U.f101, U.f111, 5);
}
inline double planck_frac(int off, int ng, int ig, int jpl, double fpl) {
  return lerp(t2(off, ng, ig, jpl), fpl, t2(off, ng, ig, jpl + 1));
}
// adjusted minor column: ratio r of colamt to its reference amount `ref`
inline double adjcol(double col, double ref, double thresh, double base, double expo) {
  double rat = col / ref;
  if (rat > thresh) {
    double adjfac = base + std::pow(rat - base, expo);
    return adjfac * ref;
  }
  return col;
}

// ---- taugb03 (RLM:4210-4512) ----
void taugb03(Col& c) {
  const int ng = 16, b = 3, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 9) / chi(2, 9);
  double refrat_planck_b = chi(1, 13) / chi(2, 13);
  double refrat_m_a = chi(1, 3) / chi(2, 3);
  double refrat_m_b = chi(1, 13) / chi(2, 13);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 1, 1), c.RF(k, 1, 2), c.COL(k, 2));
    Spec sm = spec(c.COL(k, 1), refrat_m_a, c.COL(k, 2), 8.0);
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 2), 8.0);
    double adjcoln2o = adjcol(c.COL(k, 4), c.coldry[k - 1] * chi(4, c.JP(k) + 1), 1.5, 0.5, 0.65);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b03_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b03_forref, ng, ig);
      double absn2o = minor3(c, k, lwtab::b03_ka_mn2o, ng, 9, ig, sm.js, sm.fs);
      double tau_major = L.s0.comb * major6(lwtab::b03_absa, ng, ig, L.p0, L.f0);
      double tau_major1 = L.s1.comb * major6(lwtab::b03_absa, ng, ig, L.p1, L.f1);
      c.TAUG(ns + ig, k) = tau_major + tau_major1 + tauself + taufor + adjcoln2o * absn2o;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b03_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    Upper U = upper_setup(c, k, b, c.COL(k, 1), c.RF(k, 1, 1), c.RF(k, 1, 2), c.COL(k, 2));
    Spec sm = spec(c.COL(k, 1), refrat_m_b, c.COL(k, 2), 4.0);
    Spec sp = spec(c.COL(k, 1), refrat_planck_b, c.COL(k, 2), 4.0);
    double adjcoln2o = adjcol(c.COL(k, 4), c.coldry[k - 1] * chi(4, c.JP(k) + 1), 1.5, 0.5, 0.65);
    for (int ig = 1; ig <= ng; ++ig) {
      double taufor = forcont(c, k, lwtab::b03_forref, ng, ig);
      double absn2o = minor3(c, k, lwtab::b03_kb_mn2o, ng, 5, ig, sm.js, sm.fs);
      double tau_major = U.s0.comb * major4(lwtab::b03_absb, ng, ig, U.ind0, U.f000, U.f010, U.f100, U.f110, 5);
      double tau_major1 = U.s1.comb * major4(lwtab::b03_absb, ng, ig, U.ind1, U.f001, U.f011, U.f101, U.f111, 5);
      c.TAUG(ns + ig, k) = tau_major + tau_major1 + taufor + adjcoln2o * absn2o;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b03_fracrefb, ng, ig, sp.js, sp.fs);
    }
  }
}

// ---- taugb04 (RLM:4518-4757) ----
void taugb04(Col& c) {
  const int ng = 14, b = 4, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 11) / chi(2, 11);
  double refrat_planck_b = chi(3, 13) / chi(2, 13);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 1, 1), c.RF(k, 1, 2), c.COL(k, 2));
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 2), 8.0);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b04_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b04_forref, ng, ig);
      double tau_major = L.s0.comb * major6(lwtab::b04_absa, ng, ig, L.p0, L.f0);
      double tau_major1 = L.s1.comb * major6(lwtab::b04_absa, ng, ig, L.p1, L.f1);
      c.TAUG(ns + ig, k) = tau_major + tau_major1 + tauself + taufor;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b04_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    Upper U = upper_setup(c, k, b, c.COL(k, 3), c.RF(k, 6, 1), c.RF(k, 6, 2), c.COL(k, 2));
    Spec sp = spec(c.COL(k, 3), refrat_planck_b, c.COL(k, 2), 4.0);
    for (int ig = 1; ig <= ng; ++ig) {
      double tau_major = U.s0.comb * major4(lwtab::b04_absb, ng, ig, U.ind0, U.f000, U.f010, U.f100, U.f110, 5);
      double tau_major1 = U.s1.comb * major4(lwtab::b04_absb, ng, ig, U.ind1, U.f001, U.f011, U.f101, U.f111, 5);
      c.TAUG(ns + ig, k) = tau_major + tau_major1;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b04_fracrefb, ng, ig, sp.js, sp.fs);
    }
    // RLM:4746-4752 empirical scalings of g-points 8..14
    c.TAUG(ns + 8, k) = c.TAUG(ns + 8, k) * 0.92;
    c.TAUG(ns + 9, k) = c.TAUG(ns + 9, k) * 0.88;
    c.TAUG(ns + 10, k) = c.TAUG(ns + 10, k) * 1.07;
    c.TAUG(ns + 11, k) = c.TAUG(ns + 11, k) * 1.1;
    c.TAUG(ns + 12, k) = c.TAUG(ns + 12, k) * 0.99;
    c.TAUG(ns + 13, k) = c.TAUG(ns + 13, k) * 0.88;
    c.TAUG(ns + 14, k) = c.TAUG(ns + 14, k) * 0.943;
  }
}

// ---- taugb05 (RLM:4764-5023) ----
void taugb05(Col& c) {
  const int ng = 16, b = 5, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 5) / chi(2, 5);
  double refrat_planck_b = chi(3, 43) / chi(2, 43);
  double refrat_m_a = chi(1, 7) / chi(2, 7);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 1, 1), c.RF(k, 1, 2), c.COL(k, 2));
    Spec sm = spec(c.COL(k, 1), refrat_m_a, c.COL(k, 2), 8.0);
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 2), 8.0);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b05_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b05_forref, ng, ig);
      double abso3 = minor3(c, k, lwtab::b05_ka_mo3, ng, 9, ig, sm.js, sm.fs);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b05_absa, ng, ig) + tauself + taufor +
                           abso3 * c.COL(k, 3) + c.WX(k, 1) * t1(lwtab::b05_ccl4, ig);
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b05_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    Upper U = upper_setup(c, k, b, c.COL(k, 3), c.RF(k, 6, 1), c.RF(k, 6, 2), c.COL(k, 2));
    Spec sp = spec(c.COL(k, 3), refrat_planck_b, c.COL(k, 2), 4.0);
    for (int ig = 1; ig <= ng; ++ig) {
      c.TAUG(ns + ig, k) = upper_major(U, lwtab::b05_absb, ng, ig) + c.WX(k, 1) * t1(lwtab::b05_ccl4, ig);
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b05_fracrefb, ng, ig, sp.js, sp.fs);
    }
  }
}

// ---- taugb06 (RLM:5030-5111) ----
void taugb06(Col& c) {
  const int ng = 8, b = 6, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = lowind(c, k, c.JT(k), nspa[b - 1]) + 1, ind1 = lowind1(c, k, c.JT1(k), nspa[b - 1]) + 1;
    double adjcolco2 = adjcol(c.COL(k, 2), c.coldry[k - 1] * chi(2, c.JP(k) + 1), 3.0, 2.0, 0.77);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b06_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b06_forref, ng, ig);
      double absco2 = minor2(c, k, lwtab::b06_ka_mco2, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b06_absa, ng, ig, ind0, ind1) + tauself + taufor +
                           adjcolco2 * absco2 + c.WX(k, 2) * t1(lwtab::b06_cfc11adj, ig) +
                           c.WX(k, 3) * t1(lwtab::b06_cfc12, ig);
      c.FRACS(ns + ig, k) = t1(lwtab::b06_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k)
    for (int ig = 1; ig <= ng; ++ig) {
      c.TAUG(ns + ig, k) = c.WX(k, 2) * t1(lwtab::b06_cfc11adj, ig) + c.WX(k, 3) * t1(lwtab::b06_cfc12, ig);
      c.FRACS(ns + ig, k) = t1(lwtab::b06_fracrefa, ig);
    }
}

// ---- taugb07 (RLM:5118-5375) ----
void taugb07(Col& c) {
  const int ng = 12, b = 7, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 3) / chi(3, 3);
  double refrat_m_a = chi(1, 3) / chi(3, 3);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 2, 1), c.RF(k, 2, 2), c.COL(k, 3));
    Spec sm = spec(c.COL(k, 1), refrat_m_a, c.COL(k, 3), 8.0);
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 3), 8.0);
    double adjcolco2 = adjcol(c.COL(k, 2), c.coldry[k - 1] * chi(2, c.JP(k) + 1), 3.0, 3.0, 0.79);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b07_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b07_forref, ng, ig);
      double absco2 = minor3(c, k, lwtab::b07_ka_mco2, ng, 9, ig, sm.js, sm.fs);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b07_absa, ng, ig) + tauself + taufor + adjcolco2 * absco2;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b07_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    double adjcolco2 = adjcol(c.COL(k, 2), c.coldry[k - 1] * chi(2, c.JP(k) + 1), 3.0, 2.0, 0.79);
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      double absco2 = minor2(c, k, lwtab::b07_kb_mco2, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 3) * absk(c, k, lwtab::b07_absb, ng, ig, ind0, ind1) + adjcolco2 * absco2;
      c.FRACS(ns + ig, k) = t1(lwtab::b07_fracrefb, ig);
    }
    // RLM:5366-5371
    c.TAUG(ns + 6, k) = c.TAUG(ns + 6, k) * 0.92;
    c.TAUG(ns + 7, k) = c.TAUG(ns + 7, k) * 0.88;
    c.TAUG(ns + 8, k) = c.TAUG(ns + 8, k) * 1.07;
    c.TAUG(ns + 9, k) = c.TAUG(ns + 9, k) * 1.1;
    c.TAUG(ns + 10, k) = c.TAUG(ns + 10, k) * 0.99;
    c.TAUG(ns + 11, k) = c.TAUG(ns + 11, k) * 0.855;
  }
}

// ---- taugb08 (RLM:5382-5501) ----
void taugb08(Col& c) {
  const int ng = 8, b = 8, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = lowind(c, k, c.JT(k), nspa[b - 1]) + 1, ind1 = lowind1(c, k, c.JT1(k), nspa[b - 1]) + 1;
    double adjcolco2 = adjcol(c.COL(k, 2), c.coldry[k - 1] * chi(2, c.JP(k) + 1), 3.0, 2.0, 0.65);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b08_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b08_forref, ng, ig);
      double absco2 = minor2(c, k, lwtab::b08_ka_mco2, ng, ig);
      double abso3 = minor2(c, k, lwtab::b08_ka_mo3, ng, ig);
      double absn2o = minor2(c, k, lwtab::b08_ka_mn2o, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b08_absa, ng, ig, ind0, ind1) + tauself + taufor +
                           adjcolco2 * absco2 + c.COL(k, 3) * abso3 + c.COL(k, 4) * absn2o +
                           c.WX(k, 3) * t1(lwtab::b08_cfc12, ig) + c.WX(k, 4) * t1(lwtab::b08_cfc22adj, ig);
      c.FRACS(ns + ig, k) = t1(lwtab::b08_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    double adjcolco2 = adjcol(c.COL(k, 2), c.coldry[k - 1] * chi(2, c.JP(k) + 1), 3.0, 2.0, 0.65);
    for (int ig = 1; ig <= ng; ++ig) {
      double absco2 = minor2(c, k, lwtab::b08_kb_mco2, ng, ig);
      double absn2o = minor2(c, k, lwtab::b08_kb_mn2o, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 3) * absk(c, k, lwtab::b08_absb, ng, ig, ind0, ind1) + adjcolco2 * absco2 +
                           c.COL(k, 4) * absn2o + c.WX(k, 3) * t1(lwtab::b08_cfc12, ig) +
                           c.WX(k, 4) * t1(lwtab::b08_cfc22adj, ig);
      c.FRACS(ns + ig, k) = t1(lwtab::b08_fracrefb, ig);
    }
  }
}

// ---- taugb09 (RLM:5508-5753) ----
void taugb09(Col& c) {
  const int ng = 12, b = 9, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 9) / chi(6, 9);
  double refrat_m_a = chi(1, 3) / chi(6, 3);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 4, 1), c.RF(k, 4, 2), c.COL(k, 5));
    Spec sm = spec(c.COL(k, 1), refrat_m_a, c.COL(k, 5), 8.0);
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 5), 8.0);
    double adjcoln2o = adjcol(c.COL(k, 4), c.coldry[k - 1] * chi(4, c.JP(k) + 1), 1.5, 0.5, 0.65);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b09_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b09_forref, ng, ig);
      double absn2o = minor3(c, k, lwtab::b09_ka_mn2o, ng, 9, ig, sm.js, sm.fs);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b09_absa, ng, ig) + tauself + taufor + adjcoln2o * absn2o;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b09_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    double adjcoln2o = adjcol(c.COL(k, 4), c.coldry[k - 1] * chi(4, c.JP(k) + 1), 1.5, 0.5, 0.65);
    for (int ig = 1; ig <= ng; ++ig) {
      double absn2o = minor2(c, k, lwtab::b09_kb_mn2o, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 5) * absk(c, k, lwtab::b09_absb, ng, ig, ind0, ind1) + adjcoln2o * absn2o;
      c.FRACS(ns + ig, k) = t1(lwtab::b09_fracrefb, ig);
    }
  }
}

// ---- taugb10 (RLM:5759-5829) ----
void taugb10(Col& c) {
  const int ng = 6, b = 10, ns = NS[b - 1];
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = lowind(c, k, c.JT(k), nspa[b - 1]) + 1, ind1 = lowind1(c, k, c.JT1(k), nspa[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b10_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b10_forref, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b10_absa, ng, ig, ind0, ind1) + tauself + taufor;
      c.FRACS(ns + ig, k) = t1(lwtab::b10_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      double taufor = forcont(c, k, lwtab::b10_forref, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b10_absb, ng, ig, ind0, ind1) + taufor;
      c.FRACS(ns + ig, k) = t1(lwtab::b10_fracrefb, ig);
    }
  }
}

// ---- taugb11 (RLM:5836-5923) ----
void taugb11(Col& c) {
  const int ng = 8, b = 11, ns = NS[b - 1];
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = lowind(c, k, c.JT(k), nspa[b - 1]) + 1, ind1 = lowind1(c, k, c.JT1(k), nspa[b - 1]) + 1;
    double scaleo2 = c.COL(k, 6) * c.scaleminor[k - 1];
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b11_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b11_forref, ng, ig);
      double tauo2 = scaleo2 * minor2(c, k, lwtab::b11_ka_mo2, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b11_absa, ng, ig, ind0, ind1) + tauself + taufor + tauo2;
      c.FRACS(ns + ig, k) = t1(lwtab::b11_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    double scaleo2 = c.COL(k, 6) * c.scaleminor[k - 1];
    for (int ig = 1; ig <= ng; ++ig) {
      double taufor = forcont(c, k, lwtab::b11_forref, ng, ig);
      double tauo2 = scaleo2 * minor2(c, k, lwtab::b11_kb_mo2, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 1) * absk(c, k, lwtab::b11_absb, ng, ig, ind0, ind1) + taufor + tauo2;
      c.FRACS(ns + ig, k) = t1(lwtab::b11_fracrefb, ig);
    }
  }
}

// ---- taugb12 (RLM:5929-6111) ----
void taugb12(Col& c) {
  const int ng = 8, b = 12, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 10) / chi(2, 10);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 1, 1), c.RF(k, 1, 2), c.COL(k, 2));
    // RLM:5974-5977: clipped with '>= oneminus' instead of min()
    double speccomb_planck = c.COL(k, 1) + refrat_planck_a * c.COL(k, 2);
    double specparm_planck = c.COL(k, 1) / speccomb_planck;
    if (specparm_planck >= oneminus) specparm_planck = oneminus;
    double specmult_planck = 8.0 * specparm_planck;
    int jpl = 1 + fint(specmult_planck);
    double fpl = fmod1(specmult_planck);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b12_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b12_forref, ng, ig);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b12_absa, ng, ig) + tauself + taufor;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b12_fracrefa, ng, ig, jpl, fpl);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k)
    for (int ig = 1; ig <= ng; ++ig) {
      c.TAUG(ns + ig, k) = f_zero;
      c.FRACS(ns + ig, k) = f_zero;
    }
}

// ---- taugb13 (RLM:6117-6361) ----
void taugb13(Col& c) {
  const int ng = 4, b = 13, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 5) / chi(4, 5);
  double refrat_m_a = chi(1, 1) / chi(4, 1);
  double refrat_m_a3 = chi(1, 3) / chi(4, 3);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 3, 1), c.RF(k, 3, 2), c.COL(k, 4));
    Spec smco2 = spec(c.COL(k, 1), refrat_m_a, c.COL(k, 4), 8.0);
    Spec smco = spec(c.COL(k, 1), refrat_m_a3, c.COL(k, 4), 8.0);
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 4), 8.0);
    double adjcolco2 = adjcol(c.COL(k, 2), c.coldry[k - 1] * 3.55e-4, 3.0, 2.0, 0.68);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b13_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b13_forref, ng, ig);
      double absco2 = minor3(c, k, lwtab::b13_ka_mco2, ng, 9, ig, smco2.js, smco2.fs);
      double absco = minor3(c, k, lwtab::b13_ka_mco, ng, 9, ig, smco.js, smco.fs);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b13_absa, ng, ig) + tauself + taufor +
                           adjcolco2 * absco2 + c.COL(k, 7) * absco;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b13_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k)
    for (int ig = 1; ig <= ng; ++ig) {
      double abso3 = minor2(c, k, lwtab::b13_kb_mo3, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 3) * abso3;
      c.FRACS(ns + ig, k) = t1(lwtab::b13_fracrefb, ig);
    }
}

// ---- taugb14 (RLM:6367-6431) ----
void taugb14(Col& c) {
  const int ng = 2, b = 14, ns = NS[b - 1];
  for (int k = 1; k <= c.laytrop; ++k) {
    int ind0 = lowind(c, k, c.JT(k), nspa[b - 1]) + 1, ind1 = lowind1(c, k, c.JT1(k), nspa[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b14_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b14_forref, ng, ig);
      c.TAUG(ns + ig, k) = c.COL(k, 2) * absk(c, k, lwtab::b14_absa, ng, ig, ind0, ind1) + tauself + taufor;
      c.FRACS(ns + ig, k) = t1(lwtab::b14_fracrefa, ig);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      c.TAUG(ns + ig, k) = c.COL(k, 2) * absk(c, k, lwtab::b14_absb, ng, ig, ind0, ind1);
      c.FRACS(ns + ig, k) = t1(lwtab::b14_fracrefb, ig);
    }
  }
}

// ---- taugb15 (RLM:6438-6644) ----
void taugb15(Col& c) {
  const int ng = 2, b = 15, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(4, 1) / chi(2, 1);
  double refrat_m_a = chi(4, 1) / chi(2, 1);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 4), c.RF(k, 5, 1), c.RF(k, 5, 2), c.COL(k, 2));
    Spec sm = spec(c.COL(k, 4), refrat_m_a, c.COL(k, 2), 8.0);
    Spec sp = spec(c.COL(k, 4), refrat_planck_a, c.COL(k, 2), 8.0);
    double scalen2 = c.colbrd[k - 1] * c.scaleminor[k - 1];
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b15_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b15_forref, ng, ig);
      double taun2 = scalen2 * minor3(c, k, lwtab::b15_ka_mn2, ng, 9, ig, sm.js, sm.fs);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b15_absa, ng, ig) + tauself + taufor + taun2;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b15_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k)
    for (int ig = 1; ig <= ng; ++ig) {
      c.TAUG(ns + ig, k) = f_zero;
      c.FRACS(ns + ig, k) = f_zero;
    }
}

// ---- taugb16 (RLM:6650-6840) ----
void taugb16(Col& c) {
  const int ng = 2, b = 16, ns = NS[b - 1];
  auto chi = [&](int m, int j) { return t2(lwtab::chi_mls, 7, m, j); };
  double refrat_planck_a = chi(1, 6) / chi(6, 6);
  for (int k = 1; k <= c.laytrop; ++k) {
    Lower L = lower_setup(c, k, b, c.COL(k, 1), c.RF(k, 4, 1), c.RF(k, 4, 2), c.COL(k, 5));
    Spec sp = spec(c.COL(k, 1), refrat_planck_a, c.COL(k, 5), 8.0);
    for (int ig = 1; ig <= ng; ++ig) {
      double tauself = selfcont(c, k, lwtab::b16_selfref, ng, ig);
      double taufor = forcont(c, k, lwtab::b16_forref, ng, ig);
      c.TAUG(ns + ig, k) = lower_major(L, lwtab::b16_absa, ng, ig) + tauself + taufor;
      c.FRACS(ns + ig, k) = planck_frac(lwtab::b16_fracrefa, ng, ig, sp.js, sp.fs);
    }
  }
  for (int k = c.laytrop + 1; k <= c.nlay; ++k) {
    // nspb(16) = 0 (RLM:327), so both indices are 1 whatever jp/jt are
    int ind0 = upind(c, k, c.JT(k), nspb[b - 1]) + 1, ind1 = upind1(c, k, c.JT1(k), nspb[b - 1]) + 1;
    for (int ig = 1; ig <= ng; ++ig) {
      c.TAUG(ns + ig, k) = c.COL(k, 5) * absk(c, k, lwtab::b16_absb, ng, ig, ind0, ind1);
      c.FRACS(ns + ig, k) = t1(lwtab::b16_fracrefb, ig);
    }
  }
}

// ---- taumol (RLM:3836-4013) ----
void taumol(Col& c) {
  taugb01(c); taugb02(c); taugb03(c); taugb04(c); taugb05(c); taugb06(c); taugb07(c); taugb08(c);
  taugb09(c); taugb10(c); taugb11(c); taugb12(c); taugb13(c); taugb14(c); taugb15(c); taugb16(c);
  for (int ig = 1; ig <= NGPT; ++ig) {
    int ib = ngb[ig - 1];
    for (int k = 1; k <= c.nlay; ++k) c.TAUTOT(ig, k) = c.TAUG(ig, k) + c.TAUAER(ib, k);
  }
}

// ---- rtrnmc (RLM:3420-3785) ----------------------------------------------
// Band radiances of a transfer routine, (0:nlay, nbands) each.
struct BandRad {
  int nlay;
  std::vector<double> tu, td, cu, cd;   // total up/down, clear up/down
  explicit BandRad(int n) : nlay(n), tu((size_t)(n + 1) * 16, 0.0), td(tu), cu(tu), cd(tu) {}
  double& at(std::vector<double>& v, int k, int ib) { return v[k + (nlay + 1) * (ib - 1)]; }
};

// Gas part of one layer of one g-point, shared by rtrnmc/rtrn/rtrnmr
// (RLM:3598-3627, 2601-2627, 3174-3200): transmittance, down/up sources.
struct GasLayer {
  double trng, odepth, gassrcd, gassrcu, plfrac, blay, dplnku, dplnkd;
};
GasLayer gas_layer(Col& c, int ig, int ib, int k) {
  const double rec_6 = 0.166667;
  GasLayer g;
  double odepth = std::max(f_zero, c.secdiff[ib - 1] * c.TAUTOT(ig, k));
  double atrgas, gasfac;
  if (odepth <= 0.06) {
    atrgas = odepth - 0.5 * odepth * odepth;
    g.trng = f_one - atrgas;
    gasfac = rec_6 * odepth;
  } else {
    double tblind = odepth / (bpade + odepth);
    int itgas = (int)(tblint * tblind + 0.5);
    g.trng = exp_tbl[itgas];
    atrgas = f_one - g.trng;
    gasfac = tfn_tbl[itgas];
    odepth = tau_tbl[itgas];
  }
  g.odepth = odepth;
  g.plfrac = c.FRACS(ig, k);
  g.blay = c.PKLAY(ib, k);
  g.dplnku = c.PKLEV(ib, k) - g.blay;
  g.dplnkd = c.PKLEV(ib, k - 1) - g.blay;
  const double bbdgas = g.plfrac * (g.blay + g.dplnkd * gasfac);
  const double bbugas = g.plfrac * (g.blay + g.dplnku * gasfac);
  g.gassrcd = bbdgas * atrgas;
  g.gassrcu = bbugas * atrgas;
  return g;
}

// Cloudy part: total optical depth table terms (RLM:3636-3650).
void tot_layer(double odtot, double& totfac, double& atrtot, double& trnt) {
  const double rec_6 = 0.166667;
  if (odtot < 0.06) {
    totfac = rec_6 * odtot;
    atrtot = odtot - 0.5 * odtot * odtot;
    trnt = f_one - atrtot;
  } else {
    double tblind = odtot / (bpade + odtot);
    int ittot = (int)(tblint * tblind + 0.5);
    totfac = tfn_tbl[ittot];
    trnt = exp_tbl[ittot];
    atrtot = f_one - trnt;
  }
}

// Fluxes and heating rates from the band radiances (RLM:3737-3785).
void finish_fluxes(Col& c, BandRad& br, bool lhlw0, bool lhlwb) {
  const int nlay = c.nlay;
  std::vector<double> rfdelp(nlay + 1), fnet(nlay + 1), fnetc(nlay + 1);
  for (int k = 0; k <= nlay; ++k) c.totuflux[k] = c.totdflux[k] = c.totuclfl[k] = c.totdclfl[k] = f_zero;
  double flxfac = wtdiff * fluxfac;
  for (int k = 0; k <= nlay; ++k) {
    for (int ib = 1; ib <= NBANDS; ++ib) {
      c.totuflux[k] = c.totuflux[k] + br.at(br.tu, k, ib);
      c.totdflux[k] = c.totdflux[k] + br.at(br.td, k, ib);
      c.totuclfl[k] = c.totuclfl[k] + br.at(br.cu, k, ib);
      c.totdclfl[k] = c.totdclfl[k] + br.at(br.cd, k, ib);
    }
    c.totuflux[k] = c.totuflux[k] * flxfac;
    c.totdflux[k] = c.totdflux[k] * flxfac;
    c.totuclfl[k] = c.totuclfl[k] * flxfac;
    c.totdclfl[k] = c.totdclfl[k] * flxfac;
  }
  fnet[0] = c.totuflux[0] - c.totdflux[0];
  for (int k = 1; k <= nlay; ++k) {
    rfdelp[k] = heatfac / c.delp[k - 1];
    fnet[k] = c.totuflux[k] - c.totdflux[k];
    c.htr[k - 1] = (fnet[k - 1] - fnet[k]) * rfdelp[k];
  }
  if (lhlw0) {
    fnetc[0] = c.totuclfl[0] - c.totdclfl[0];
    for (int k = 1; k <= nlay; ++k) {
      fnetc[k] = c.totuclfl[k] - c.totdclfl[k];
      c.htrcl[k - 1] = (fnetc[k - 1] - fnetc[k]) * rfdelp[k];
    }
  }
  if (lhlwb) {
    for (int ib = 1; ib <= NBANDS; ++ib) {
      fnet[0] = (br.at(br.tu, 0, ib) - br.at(br.td, 0, ib)) * flxfac;
      for (int k = 1; k <= nlay; ++k) {
        fnet[k] = (br.at(br.tu, k, ib) - br.at(br.td, k, ib)) * flxfac;
        c.HTRB(k, ib) = (fnet[k - 1] - fnet[k]) * rfdelp[k];
      }
    }
  }
}

// rtrnmc (RLM:3420-3785) and rtrn (RLM:2445-2800).  They differ only in the
// cloud fraction of a layer -- McICA's 0/1 sub-column flag cldfmc(ig,k) or the
// layer fraction cldfrc(k) -- and in the up-sweep cloud test (strict > eps in
// rtrnmc, >= eps in rtrn).
void rtrn_random(Col& c, bool lhlw0, bool lhlwb, bool mcica) {
  const int nlay = c.nlay;
  BandRad br(nlay);
  std::vector<double> gassrcu(nlay + 1), totsrcu(nlay + 1), trngas(nlay + 1), efclrfr(nlay + 1);
  auto clfr_of = [&](int ig, int k) { return mcica ? c.CLDFMC(ig, k) : c.cldfrc[k]; };
  for (int ig = 1; ig <= NGPT; ++ig) {
    int ib = ngb[ig - 1];
    double radtotd = f_zero, radclrd = f_zero;
    for (int k = nlay; k >= 1; --k) {
      GasLayer g = gas_layer(c, ig, ib, k);
      gassrcu[k] = g.gassrcu;
      trngas[k] = g.trng;
      double clfm = clfr_of(ig, k);
      if (clfm >= eps) {
        double odcld = c.secdiff[ib - 1] * c.TAUCLD(ib, k);
        efclrfr[k] = f_one - (f_one - std::exp(-odcld)) * clfm;
        double totfac, atrtot, trnt;
        tot_layer(g.odepth + odcld, totfac, atrtot, trnt);
        double bbdtot = g.plfrac * (g.blay + g.dplnkd * totfac);
        double bbutot = g.plfrac * (g.blay + g.dplnku * totfac);
        double totsrcd = bbdtot * atrtot;
        totsrcu[k] = bbutot * atrtot;
        radtotd = radtotd * g.trng * efclrfr[k] + g.gassrcd + clfm * (totsrcd - g.gassrcd);
      } else {
        radtotd = radtotd * g.trng + g.gassrcd;
      }
      br.at(br.td, k - 1, ib) = br.at(br.td, k - 1, ib) + radtotd;
      radclrd = radclrd * g.trng + g.gassrcd;
      br.at(br.cd, k - 1, ib) = br.at(br.cd, k - 1, ib) + radclrd;
    }
    double reflct = f_one - c.semiss[ib - 1];
    double rad0 = c.semiss[ib - 1] * c.FRACS(ig, 1) * c.PKLAY(ib, 0);
    double radtotu = rad0 + reflct * radtotd;
    br.at(br.tu, 0, ib) = br.at(br.tu, 0, ib) + radtotu;
    double radclru = rad0 + reflct * radclrd;
    br.at(br.cu, 0, ib) = br.at(br.cu, 0, ib) + radclru;
    for (int k = 1; k <= nlay; ++k) {
      double clfm = clfr_of(ig, k);
      double trng = trngas[k];
      double gasu = gassrcu[k];
      if (mcica ? (clfm > eps) : (clfm >= eps)) {
        radtotu = radtotu * trng * efclrfr[k] + gasu + clfm * (totsrcu[k] - gasu);
      } else {
        radtotu = radtotu * trng + gasu;
      }
      br.at(br.tu, k, ib) = br.at(br.tu, k, ib) + radtotu;
      radclru = radclru * trng + gasu;
      br.at(br.cu, k, ib) = br.at(br.cu, k, ib) + radclru;
    }
  }
  finish_fluxes(c, br, lhlw0, lhlwb);
}

void rtrnmc(Col& c, bool lhlw0, bool lhlwb) { rtrn_random(c, lhlw0, lhlwb, true); }

// Maximum-random overlap coefficients of rtrnmr (RLM:2921-3092) in one
// direction.  With dir = +1 (upward sweep) layer k pairs with k+1 and looks
// back at k-1; with dir = -1 (downward) it pairs with k-1 and looks back at
// k+1.  The factors of the pair (k, k+dir) are stored at index k+dir.
struct MrFactors {
  std::vector<double> clr1, clr2, cld1, cld2, cmb1, cmb2;
  std::vector<char> lst;
  explicit MrFactors(int n) : clr1(n + 2, 0.0), clr2(clr1), cld1(clr1), cld2(clr1), cmb1(clr1), cmb2(clr1), lst(n + 2, 0) {}
};
void mr_factors(const Col& c, int dir, MrFactors& f) {
  const int nlay = c.nlay;
  const std::vector<double>& cf = c.cldfrc;   // 0:nlp1, padded with 1 and 0
  const int k0 = dir > 0 ? 1 : nlay, k1 = dir > 0 ? nlay - 1 : 2;
  f.lst[k0] = cf[k0] > eps;
  double rat1 = f_zero, rat2 = f_zero;
  for (int k = k0; dir > 0 ? k <= k1 : k >= k1; k += dir) {
    const int kn = k + dir, kb = k - dir;   // next layer in the sweep, the one behind
    f.lst[kn] = cf[kn] > eps && cf[k] <= eps;
    if (!(cf[k] > eps)) continue;
    if (cf[kn] >= cf[k]) {
      if (f.lst[k]) {
        if (cf[k] < f_one) f.clr2[kn] = (cf[kn] - cf[k]) / (f_one - cf[k]);
        f.clr2[k] = f_zero;
        f.cld2[k] = f_zero;
      } else {
        double fmax = std::max(cf[k], cf[kb]);
        if (cf[kn] > fmax) {
          f.clr1[kn] = rat2;
          f.clr2[kn] = (cf[kn] - fmax) / (f_one - fmax);
        } else if (cf[kn] < fmax) {
          f.clr1[kn] = (cf[kn] - cf[k]) / (cf[kb] - cf[k]);
        } else {
          f.clr1[kn] = rat2;
        }
      }
      if (f.clr1[kn] > f_zero || f.clr2[kn] > f_zero) { rat1 = f_one; rat2 = f_zero; }
      else { rat1 = f_zero; rat2 = f_zero; }
    } else {
      if (f.lst[k]) {
        f.cld2[kn] = (cf[k] - cf[kn]) / cf[k];
        f.clr2[k] = f_zero;
        f.cld2[k] = f_zero;
      } else {
        double fmin = std::min(cf[k], cf[kb]);
        if (cf[kn] <= fmin) {
          f.cld1[kn] = rat1;
          f.cld2[kn] = (fmin - cf[kn]) / fmin;
        } else {
          f.cld1[kn] = (cf[k] - cf[kn]) / (cf[k] - fmin);
        }
      }
      if (f.cld1[kn] > f_zero || f.cld2[kn] > f_zero) { rat1 = f_zero; rat2 = f_one; }
      else { rat1 = f_zero; rat2 = f_zero; }
    }
    f.cmb1[kn] = f.clr1[kn] * f.cld2[k] * cf[kb];
    f.cmb2[kn] = f.cld1[kn] * f.clr2[k] * (f_one - cf[kb]);
  }
}

// rtrnmr (RLM:2828-3392): maximum-random overlap of the layer cloud fractions.
// The split radiances (totradd, clrradd, rad and their upward twins) are
// reset at the first cloudy layer of every cloud block; a layer with a cloud
// fraction of exactly eps is "cloudy" without starting a block, where the
// Fortran reads the values left by the previous g-point -- here they start
// from zero for every g-point.
void rtrnmr(Col& c, bool lhlw0, bool lhlwb) {
  const int nlay = c.nlay;
  MrFactors up(nlay), dn(nlay);
  mr_factors(c, +1, up);
  mr_factors(c, -1, dn);
  BandRad br(nlay);
  std::vector<double> gassrcu(nlay + 1), totsrcu(nlay + 1), trngas(nlay + 1), trntot(nlay + 1);
  for (int ig = 1; ig <= NGPT; ++ig) {
    int ib = ngb[ig - 1];
    double radtotd = f_zero, radclrd = f_zero;
    double totradd = f_zero, clrradd = f_zero, rad = f_zero;
    for (int k = nlay; k >= 1; --k) {
      GasLayer g = gas_layer(c, ig, ib, k);
      gassrcu[k] = g.gassrcu;
      trngas[k] = g.trng;
      double clfr = c.cldfrc[k];
      if (dn.lst[k]) {
        totradd = clfr * radtotd;
        clrradd = radtotd - totradd;
        rad = f_zero;
      }
      if (clfr >= eps) {
        double odcld = c.secdiff[ib - 1] * c.TAUCLD(ib, k);
        double totfac, atrtot, trnt;
        tot_layer(g.odepth + odcld, totfac, atrtot, trnt);
        double bbdtot = g.plfrac * (g.blay + g.dplnkd * totfac);
        double bbutot = g.plfrac * (g.blay + g.dplnku * totfac);
        double totsrcd = bbdtot * atrtot;
        totsrcu[k] = bbutot * atrtot;
        trntot[k] = trnt;
        totradd = totradd * trnt + clfr * totsrcd;
        clrradd = clrradd * g.trng + (f_one - clfr) * g.gassrcd;
        radtotd = totradd + clrradd;
        br.at(br.td, k - 1, ib) = br.at(br.td, k - 1, ib) + radtotd;
        radclrd = radclrd * g.trng + g.gassrcd;
        br.at(br.cd, k - 1, ib) = br.at(br.cd, k - 1, ib) + radclrd;
        double radmod = rad * (dn.clr1[k - 1] * g.trng + dn.cld1[k - 1] * trnt) - dn.cmb1[k - 1] * g.gassrcd +
                        dn.cmb2[k - 1] * totsrcd;
        rad = -radmod + dn.clr2[k - 1] * (clrradd + radmod) - dn.cld2[k - 1] * (totradd - radmod);
        totradd = totradd + rad;
        clrradd = clrradd - rad;
      } else {
        radtotd = radtotd * g.trng + g.gassrcd;
        br.at(br.td, k - 1, ib) = br.at(br.td, k - 1, ib) + radtotd;
        radclrd = radclrd * g.trng + g.gassrcd;
        br.at(br.cd, k - 1, ib) = br.at(br.cd, k - 1, ib) + radclrd;
      }
    }
    double reflct = f_one - c.semiss[ib - 1];
    double rad0 = c.semiss[ib - 1] * c.FRACS(ig, 1) * c.PKLAY(ib, 0);
    double radtotu = rad0 + reflct * radtotd;
    br.at(br.tu, 0, ib) = br.at(br.tu, 0, ib) + radtotu;
    double radclru = rad0 + reflct * radclrd;
    br.at(br.cu, 0, ib) = br.at(br.cu, 0, ib) + radclru;
    double totradu = f_zero, clrradu = f_zero;
    for (int k = 1; k <= nlay; ++k) {
      double clfr = c.cldfrc[k];
      double trng = trngas[k];
      double gasu = gassrcu[k];
      if (up.lst[k]) {
        totradu = clfr * radtotu;
        clrradu = radtotu - totradu;
        rad = f_zero;
      }
      if (clfr >= eps) {
        double trnt = trntot[k];
        double totu = totsrcu[k];
        totradu = totradu * trnt + clfr * totu;
        clrradu = clrradu * trng + (f_one - clfr) * gasu;
        radtotu = totradu + clrradu;
        br.at(br.tu, k, ib) = br.at(br.tu, k, ib) + radtotu;
        radclru = radclru * trng + gasu;
        br.at(br.cu, k, ib) = br.at(br.cu, k, ib) + radclru;
        double radmod = rad * (up.clr1[k + 1] * trng + up.cld1[k + 1] * trnt) - up.cmb1[k + 1] * gasu +
                        up.cmb2[k + 1] * totu;
        rad = -radmod + up.clr2[k + 1] * (clrradu + radmod) - up.cld2[k + 1] * (totradu - radmod);
        totradu = totradu + rad;
        clrradu = clrradu - rad;
      } else {
        radtotu = radtotu * trng + gasu;
        br.at(br.tu, k, ib) = br.at(br.tu, k, ib) + radtotu;
        radclru = radclru * trng + gasu;
        br.at(br.cu, k, ib) = br.at(br.cu, k, ib) + radclru;
      }
    }
  }
  finish_fluxes(c, br, lhlw0, lhlwb);
}

inline void set_err(char* errmsg, int len, const std::string& s) {
  if (errmsg && len > 0) {
    std::snprintf(errmsg, (size_t)len, "%s", s.c_str());
  }
}

// Prologue of the column loop (RLM:785-1050) for column iplon (1-based).
void column_prologue(Col& c, const rrtmg_lw_run_args& a, int iplon) {
  const int nlay = a.nlay, nlp1 = a.nlp1;
  const long ld = a.ldim > 0 ? a.ldim : a.npts;
  auto A2 = [&](const double* p, int i, int k) { return p[(i - 1) + ld * (long)(k - 1)]; };
  auto A3 = [&](const double* p, int i, int k, int j) {
    return p[(i - 1) + ld * ((long)(k - 1) + (long)nlay * (j - 1))];
  };
  double sfe = a.sfemis[iplon - 1];
  for (int j = 0; j < NBANDS; ++j) c.semiss[j] = (sfe > eps && sfe <= 1.0) ? sfe : 1.0;
  c.stemp = a.sfgtmp[iplon - 1];
  c.delgth = 0.0;
  if (a.iovr == a.iovr_dcorr) c.delgth = a.de_lgth[iplon - 1];
  const double tem1c = 100.0 * con_g;
  const double tem2c = 1.0e-20 * 1.0e3 * con_avgd;
  const bool top = a.top_at_1 != 0;
  c.tz[0] = top ? A2(a.tlvl, iplon, nlp1) : A2(a.tlvl, iplon, 1);
  for (int k = 1; k <= nlay; ++k) {
    int k1 = top ? nlp1 - k : k;
    c.pavel[k - 1] = A2(a.plyr, iplon, k1);
    c.delp[k - 1] = A2(a.delpin, iplon, k1);
    c.tavel[k - 1] = A2(a.tlyr, iplon, k1);
    c.tz[k] = top ? A2(a.tlvl, iplon, k1) : A2(a.tlvl, iplon, k + 1);
    c.dz[k - 1] = A2(a.dzlyr, iplon, k1);
    if (a.iovr == a.iovr_exp || a.iovr == a.iovr_exprand) c.alph[k - 1] = A2(a.alpha, iplon, k);  // not flipped
    double q = A2(a.qlyr, iplon, k1);
    c.h2ovmr[k - 1] = std::max(f_zero, q * amdw / (f_one - q));
    c.o3vmr[k - 1] = std::max(f_zero, A2(a.olyr, iplon, k1) * amdo3);
    double tem0 = (f_one - c.h2ovmr[k - 1]) * con_amd + c.h2ovmr[k - 1] * con_amw;
    c.coldry[k - 1] = tem2c * c.delp[k - 1] / (tem1c * tem0 * (f_one + c.h2ovmr[k - 1]));
    c.temcol[k - 1] = 1.0e-12 * c.coldry[k - 1];
    c.COL(k, 1) = std::max(f_zero, c.coldry[k - 1] * c.h2ovmr[k - 1]);
    c.COL(k, 2) = std::max(c.temcol[k - 1], c.coldry[k - 1] * A2(a.gasvmr_co2, iplon, k1));
    c.COL(k, 3) = std::max(c.temcol[k - 1], c.coldry[k - 1] * c.o3vmr[k - 1]);
  }
  for (int k = 1; k <= nlay; ++k) {
    int k1 = top ? nlp1 - k : k;
    if (a.inc_minor_gas) {
      c.COL(k, 4) = std::max(c.temcol[k - 1], c.coldry[k - 1] * A2(a.gasvmr_n2o, iplon, k1));
      c.COL(k, 5) = std::max(c.temcol[k - 1], c.coldry[k - 1] * A2(a.gasvmr_ch4, iplon, k1));
      c.COL(k, 6) = std::max(f_zero, c.coldry[k - 1] * A2(a.gasvmr_o2, iplon, k1));
      c.COL(k, 7) = std::max(f_zero, c.coldry[k - 1] * A2(a.gasvmr_co, iplon, k1));
      c.WX(k, 1) = std::max(f_zero, c.coldry[k - 1] * A2(a.gasvmr_ccl4, iplon, k1));
      c.WX(k, 2) = std::max(f_zero, c.coldry[k - 1] * A2(a.gasvmr_cfc11, iplon, k1));
      c.WX(k, 3) = std::max(f_zero, c.coldry[k - 1] * A2(a.gasvmr_cfc12, iplon, k1));
      c.WX(k, 4) = std::max(f_zero, c.coldry[k - 1] * A2(a.gasvmr_cfc22, iplon, k1));
    } else {
      for (int m = 4; m <= 7; ++m) c.COL(k, m) = f_zero;
      for (int m = 1; m <= 4; ++m) c.WX(k, m) = f_zero;
    }
    for (int j = 1; j <= NBANDS; ++j)
      c.TAUAER(j, k) = A3(a.aeraod, iplon, k1, j) * (f_one - A3(a.aerssa, iplon, k1, j));
    c.cldfrc[k] = A2(a.cld_cf, iplon, k1);
    if (a.ilwcliq > 0) {
      c.clwp[k - 1] = A2(a.cld_lwp, iplon, k1);
      c.relw[k - 1] = A2(a.cld_ref_liq, iplon, k1);
      c.ciwp[k - 1] = A2(a.cld_iwp, iplon, k1);
      c.reiw[k - 1] = A2(a.cld_ref_ice, iplon, k1);
      c.cda1[k - 1] = A2(a.cld_rwp, iplon, k1);
      c.cda2[k - 1] = A2(a.cld_ref_rain, iplon, k1);
      c.cda3[k - 1] = A2(a.cld_swp, iplon, k1);
      c.cda4[k - 1] = A2(a.cld_ref_snow, iplon, k1);
    } else {
      c.cda1[k - 1] = A2(a.cld_od, iplon, k1);
    }
  }
  c.cldfrc[0] = f_one;
  c.cldfrc[nlp1] = f_zero;
  double tem1 = f_zero, tem2 = f_zero;
  for (int k = 1; k <= nlay; ++k) {
    tem1 = tem1 + c.coldry[k - 1] + c.COL(k, 1);
    tem2 = tem2 + c.COL(k, 1);
  }
  double tem0 = 10.0 * tem2 / (amdw * tem1 * con_g);
  c.pwvcm = tem0 * (top ? A2(a.plvl, iplon, nlp1) : A2(a.plvl, iplon, 1));
  for (int k = 1; k <= nlay; ++k) {  // RLM:1031-1037
    double summol = f_zero;
    for (int i = 2; i <= MAXGAS; ++i) summol = summol + c.COL(k, i);
    c.colbrd[k - 1] = c.coldry[k - 1] - summol;
  }
  for (int j = 1; j <= NBANDS; ++j) {  // RLM:1041-1050
    if (j == 1 || j == 4 || j == 10) c.secdiff[j - 1] = 1.66;
    else c.secdiff[j - 1] = std::min(1.80, std::max(1.50, a0[j - 1] + a1[j - 1] * std::exp(a2[j - 1] * c.pwvcm)));
  }
}

// One column of rrtmg_lw_run (RLM:782-1304); writes outputs unless c_only.
void run_column(const rrtmg_lw_run_args& a, int iplon, int ipseed, Col& c) {
  const int nlay = a.nlay, nlp1 = a.nlp1;
  const long ld = a.ldim > 0 ? a.ldim : a.npts;
  const bool top = a.top_at_1 != 0;
  column_prologue(c, a, iplon);
  bool lcf1 = false;
  for (int k = 1; k <= nlay; ++k)
    if (c.cldfrc[k] > eps) { lcf1 = true; break; }
  if (lcf1) {
    cldprop(c, ipseed, a.iovr, a.ilwcliq, a.ilwcice, a.isubclw);
    for (int k = 1; k <= nlay; ++k) {
      int k1 = top ? nlp1 - k : k;
      a.cldtau[(iplon - 1) + ld * (long)(k1 - 1)] = c.TAUCLD(7, k);
    }
  } else {
    std::fill(c.cldfmc.begin(), c.cldfmc.end(), 0.0);
    std::fill(c.taucld.begin(), c.taucld.end(), 0.0);
  }
  setcoef(c);
  taumol(c);
  if (a.isubclw <= 0) {   // RLM:1190-1224
    if (a.iovr <= 0) rtrn_random(c, a.hlw0 != nullptr, a.hlwb != nullptr, false);
    else rtrnmr(c, a.hlw0 != nullptr, a.hlwb != nullptr);
  } else {
    rtrnmc(c, a.hlw0 != nullptr, a.hlwb != nullptr);
  }
  a.topflx[2 * (iplon - 1) + 0] = c.totuflux[nlay];
  a.topflx[2 * (iplon - 1) + 1] = c.totuclfl[nlay];
  a.sfcflx[4 * (iplon - 1) + 0] = c.totuflux[0];
  a.sfcflx[4 * (iplon - 1) + 1] = c.totuclfl[0];
  a.sfcflx[4 * (iplon - 1) + 2] = c.totdflux[0];
  a.sfcflx[4 * (iplon - 1) + 3] = c.totdclfl[0];
  for (int k = 0; k <= nlay; ++k) {
    if (!a.flxprf) break;
    int k1 = top ? nlp1 - k : k + 1;
    double* r = a.flxprf + 4 * ((iplon - 1) + ld * (long)(k1 - 1));
    r[0] = c.totuflux[k]; r[1] = c.totdflux[k]; r[2] = c.totuclfl[k]; r[3] = c.totdclfl[k];
  }
  for (int k = 1; k <= nlay; ++k) {
    int k1 = top ? nlp1 - k : k;
    a.hlwc[(iplon - 1) + ld * (long)(k1 - 1)] = c.htr[k - 1];
    if (a.hlw0) a.hlw0[(iplon - 1) + ld * (long)(k1 - 1)] = c.htrcl[k - 1];
    if (a.hlwb)
      for (int j = 1; j <= NBANDS; ++j)
        a.hlwb[(iplon - 1) + ld * ((long)(k1 - 1) + (long)nlay * (j - 1))] = c.HTRB(k, j);
  }
}

int check_args(const rrtmg_lw_run_args* a, char* errmsg, int len) {
  if (!a) { set_err(errmsg, len, "rrtmg_lw_run: null argument struct"); return 1; }
  if (a->nlay < 1 || a->nlp1 != a->nlay + 1 || a->npts < 0 || (a->ldim != 0 && a->ldim < a->npts)) {
    set_err(errmsg, len, "rrtmg_lw_run: inconsistent dimensions (need nlay>=1, nlp1=nlay+1, npts>=0, ldim>=npts)");
    return 1;
  }
  return 0;
}

}  // namespace

extern "C" {

// rlwinit (RLM:1322-1504) plus loading the coefficient blob.
int oracle_rlwinit(const char* table_path, const rrtmg_lw_init_args* a, char* errmsg, int errmsg_len) {
  set_err(errmsg, errmsg_len, "");
  FILE* f = std::fopen(table_path, "rb");
  if (!f) { set_err(errmsg, errmsg_len, std::string("oracle: cannot open ") + table_path); return 1; }
  T.assign(RRTMG_LW_TABLES_NDOUBLE, 0.0);
  size_t n = std::fread(T.data(), sizeof(double), T.size(), f);
  std::fclose(f);
  if (n != T.size()) { set_err(errmsg, errmsg_len, "oracle: short table blob"); return 1; }
  int errflg = 0;
  if (a->iovr != a->iovr_rand && a->iovr != a->iovr_maxrand && a->iovr != a->iovr_max &&
      a->iovr != a->iovr_dcorr && a->iovr != a->iovr_exp && a->iovr != a->iovr_exprand) {
    errflg = 1;
    set_err(errmsg, errmsg_len, "ERROR(rlwinit): Error in specification of cloud overlap flag");
  }
  for (int b = 0, g = 0; b < NBANDS; ++b)
    for (int i = 0; i < NGB_NG[b]; ++i) ngb[g++] = b + 1;
  double pival = 2.0 * std::asin(f_one);
  fluxfac = pival * 2.0e4;
  heatfac = (a->rad_hr_units == 1) ? con_g * 864.0 / con_cp : con_g * 1.0e-2 / con_cp;
  const double expeps = 1.e-20;
  tau_tbl[0] = f_zero; exp_tbl[0] = f_one; tfn_tbl[0] = f_zero;
  tau_tbl[NTBL] = 1.e10; exp_tbl[NTBL] = expeps; tfn_tbl[NTBL] = f_one;
  double explimit = std::trunc(-std::log(DBL_MIN));
  for (int i = 1; i <= NTBL - 1; ++i) {
    double tfn = (double)i / (double)(NTBL - i);
    tau_tbl[i] = bpade * tfn;
    if (tau_tbl[i] >= explimit) exp_tbl[i] = expeps;
    else exp_tbl[i] = std::exp(-tau_tbl[i]);
    if (tau_tbl[i] < 0.06) tfn_tbl[i] = tau_tbl[i] / 6.0;
    else tfn_tbl[i] = f_one - 2.0 * ((f_one / tau_tbl[i]) - (exp_tbl[i] / (f_one - exp_tbl[i])));
  }
  g_init = true;
  return errflg;
}

// rrtmg_lw_run (RLM:419-1309), OpenMP over columns with `nthreads` threads
// (0 = the OpenMP default).
int oracle_rrtmg_lw_run(const rrtmg_lw_run_args* a, int nthreads, char* errmsg, int errmsg_len) {
  set_err(errmsg, errmsg_len, "");
  if (check_args(a, errmsg, errmsg_len)) return 1;
  if (!g_init) { set_err(errmsg, errmsg_len, "oracle: rlwinit not called"); return 1; }
  if (!a->lslwr) return 0;
  const long ld = a->ldim > 0 ? a->ldim : a->npts;
  for (int k = 0; k < a->nlay; ++k)
    for (int i = 0; i < a->npts; ++i) a->cldtau[i + ld * k] = f_zero;
  if (a->ilwcliq > 0) {
    if (!a->cld_lwp || !a->cld_ref_liq || !a->cld_iwp || !a->cld_ref_ice || !a->cld_rwp ||
        !a->cld_ref_rain || !a->cld_swp || !a->cld_ref_snow) {
      set_err(errmsg, errmsg_len,
              "Logic error: ilwcliq>0 requires the following optional arguments to be present: "
              "cld_lwp, cld_ref_liq, cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow");
      return 1;
    }
  } else if (!a->cld_od) {
    set_err(errmsg, errmsg_len, "Logic error: ilwcliq<=0 requires the following optional argument to be present: cld_od");
    return 1;
  }
  if (a->isubclw < 0 || a->isubclw > 2) {
    set_err(errmsg, errmsg_len, "oracle: isubclw must be 0 (rtrn/rtrnmr), 1 or 2 (McICA, rtrnmc)");
    return 1;
  }
#ifdef _OPENMP
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    Col c(a->nlay);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 8)
#endif
    for (int i = 1; i <= a->npts; ++i) {
      int ipseed = (a->isubclw == 1) ? 140 + i : a->icseed[i - 1];  // RLM:765-773
      run_column(*a, i, ipseed, c);
    }
  }
  return 0;
}

// Per-stage dump of one column (icol 1-based) for stage-level tests.  Any
// output pointer may be NULL.  Layer-resolved arrays are in internal order
// (surface first) and Fortran layout: taug/fracs/tautot/cldfmc (140, nlay),
// taucld (16, nlay), pklay/pklev (16, 0:nlay).  ints[0] = laytrop, ints[1..]
// = jp(nlay), jt(nlay), jt1(nlay).  col_scalars = {pwvcm, secdiff(16)}.
int oracle_column_stages(const rrtmg_lw_run_args* a, int icol, int* ints, double* taug, double* fracs,
                         double* tautot, double* cldfmc, double* taucld, double* pklay, double* pklev,
                         double* col_scalars, double* fac, char* errmsg, int errmsg_len) {
  if (check_args(a, errmsg, errmsg_len)) return 1;
  const int nlay = a->nlay;
  Col c(nlay);
  int ipseed = (a->isubclw == 1) ? 140 + icol : a->icseed[icol - 1];
  column_prologue(c, *a, icol);
  bool lcf1 = false;
  for (int k = 1; k <= nlay; ++k)
    if (c.cldfrc[k] > eps) { lcf1 = true; break; }
  if (lcf1) cldprop(c, ipseed, a->iovr, a->ilwcliq, a->ilwcice, a->isubclw);
  setcoef(c);
  taumol(c);
  auto cp = [](double* d, const std::vector<double>& s) { if (d) std::memcpy(d, s.data(), s.size() * sizeof(double)); };
  cp(taug, c.taug); cp(fracs, c.fracs); cp(tautot, c.tautot); cp(cldfmc, c.cldfmc); cp(taucld, c.taucld);
  cp(pklay, c.pklay); cp(pklev, c.pklev);
  if (ints) {
    ints[0] = c.laytrop;
    for (int k = 0; k < nlay; ++k) { ints[1 + k] = c.jp[k]; ints[1 + nlay + k] = c.jt[k]; ints[1 + 2 * nlay + k] = c.jt1[k]; }
  }
  if (col_scalars) {
    col_scalars[0] = c.pwvcm;
    for (int j = 0; j < 16; ++j) col_scalars[1 + j] = c.secdiff[j];
  }
  if (fac) {  // fac00, fac01, fac10, fac11, colamt(:,1..7), coldry, colbrd  (each nlay)
    int o = 0;
    for (auto* v : {&c.fac00, &c.fac01, &c.fac10, &c.fac11}) { std::memcpy(fac + o, v->data(), nlay * sizeof(double)); o += nlay; }
    std::memcpy(fac + o, c.colamt.data(), (size_t)nlay * 7 * sizeof(double)); o += 7 * nlay;
    std::memcpy(fac + o, c.coldry.data(), nlay * sizeof(double)); o += nlay;
    std::memcpy(fac + o, c.colbrd.data(), nlay * sizeof(double)); o += nlay;
  }
  return 0;
}

// Mersenne-twister stream: n raw tempered words and their real conversion
// after random_setseed_t(seed) (MT:285-372).  Also the seeded state words.
void oracle_mt_stream(int32_t seed, int n, uint32_t* u32, double* real, uint32_t* state624) {
  MTState s;
  mt_setseed(s, seed);
  if (state624) std::memcpy(state624, s.mt, sizeof(s.mt));
  for (int i = 0; i < n; ++i) {
    uint32_t y = mt_next_u32(s);
    if (u32) u32[i] = y;
    if (real) real[i] = mt_u32_to_real(y);
  }
}

// mcica_subcol for one column: lcloudy (140, nlay) as bytes, Fortran layout.
void oracle_mcica(int nlay, int32_t seed, int iovr, const double* cldf, const double* dz, double de_lgth,
                  const double* alpha, uint8_t* lcloudy) {
  Col c(nlay);
  for (int k = 0; k < nlay; ++k) { c.dz[k] = dz ? dz[k] : 0.0; c.alph[k] = alpha ? alpha[k] : 0.0; }
  c.delgth = de_lgth;
  std::vector<double> cf(cldf, cldf + nlay);
  mcica_subcol(c, cf, seed, iovr);
  std::memcpy(lcloudy, c.lcloudy.data(), c.lcloudy.size());
}

// rlwinit lookup tables (for table tests)
void oracle_tables(double* tau, double* ex, double* tfn, double* fluxfac_heatfac) {
  std::memcpy(tau, tau_tbl, sizeof(tau_tbl));
  std::memcpy(ex, exp_tbl, sizeof(exp_tbl));
  std::memcpy(tfn, tfn_tbl, sizeof(tfn_tbl));
  fluxfac_heatfac[0] = fluxfac;
  fluxfac_heatfac[1] = heatfac;
}

// Exhaustive check of the division-free McICA draw conversion used by the GPU
// kernel (csrc/lw_mcica.cu u32_unit): for every u in [start, start+count),
// u / (2^32-1) as the reference computes it (mersenne_twister.f:362-369,
// promoted reals) against fma(a, 2^-32, a) with a = u 2^-32 plus the
// round-half-up fix of exact ties.  Returns the number of mismatches.
unsigned long long oracle_check_u32_unit(unsigned long long start, unsigned long long count) {
  unsigned long long bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (long long j = 0; j < (long long)count; ++j) {
    const uint32_t u = (uint32_t)(start + (unsigned long long)j);
    const double ref = (double)u / 4294967295.0;
    const double a = (double)u * 0x1p-32;
    double r = std::fma(a, 0x1p-32, a);
    const int d = (u ? 32 - __builtin_clz(u) : 0) - 21;
    if (d >= 1) {
      const uint32_t half = 1u << (d - 1);
      if ((u & ((half << 1) - 1u)) == half && ((u >> d) & 1u) == 0u) {
        uint64_t b;
        std::memcpy(&b, &r, 8);
        ++b;
        std::memcpy(&r, &b, 8);
      }
    }
    if (std::memcmp(&r, &ref, 8) != 0) ++bad;
  }
  return bad;
}

// ---- Steps either side of rrtmg_lw_run -------------------------------------

// random_index_t (MT:489-503) after random_setseed_t(seed): m draws h of one
// stream (random_number_t in chunks of 624 continues the same stream), each
// max(ceiling(h * imax), 1).
void oracle_random_index(int32_t seed, int32_t imax, long long m, int32_t* out) {
  MTState st;
  mt_setseed(st, seed);
  for (long long j = 0; j < m; ++j) {
    const double h = mt_u32_to_real(mt_next_u32(st));
    const double c = std::ceil(h * (double)imax);
    out[j] = c < 1.0 ? 1 : (int32_t)c;
  }
}

// Seed part of GFS_rad_time_vary_timestep_init
// (physics/Interstitials/UFS_SCM_NEPTUNE/GFS_rad_time_vary.fv3.F90:59-84).
// rseeds is (ld_rseeds, 2) column-major when lrseeds.  Returns 1 for a grid
// index outside the face (the Fortran would read out of bounds), else 0.
int oracle_seeds(double sec, int32_t lslwr, int32_t lsswr, int32_t isubc_lw, int32_t isubc_sw, int32_t lrseeds,
                 int32_t ipsd0, int32_t ipsdlim, int32_t cnx, int32_t cny, int32_t isc, int32_t jsc, int32_t n,
                 int32_t ld_rseeds, const int32_t* imap, const int32_t* jmap, const int32_t* rseeds,
                 int32_t* icsdsw, int32_t* icsdlw) {
  if (!((lsswr || lslwr) && (isubc_lw == 2 || isubc_sw == 2))) return 0;
  if (lrseeds) {
    const int ld = ld_rseeds ? ld_rseeds : n;
    for (int ix = 0; ix < n; ++ix) {
      icsdsw[ix] = rseeds[ix];
      icsdlw[ix] = rseeds[ix + ld];
    }
    return 0;
  }
  const long long nr = std::llround(100.0 * std::sqrt(sec));       // nint(con_100*sqrt(sec))
  const int32_t ipseed = (int32_t)(uint32_t)((uint64_t)(nr % ipsdlim) + 1u + (uint64_t)(int64_t)ipsd0);
  const long long face = (long long)cnx * cny;
  std::vector<int32_t> numrdm((size_t)(2 * face));
  oracle_random_index(ipseed, ipsdlim, 2 * face, numrdm.data());
  for (int ix = 0; ix < n; ++ix) {
    const long long p = (long long)imap[ix] + isc - 1 + ((long long)jmap[ix] + jsc - 2) * cnx;
    if (p < 1 || p > face) return 1;
    icsdsw[ix] = numrdm[(size_t)(p - 1)];
    icsdlw[ix] = numrdm[(size_t)(p - 1 + face)];
  }
  return 0;
}

// cmp_dcorr_lgth_hogan (physics/Radiation/radiation_cloud_overlap.F90:28-50)
void oracle_dcorr_hogan(int ncol, const double* lat, double con_pi, double* dcorr) {
  const double min_dcorr = 0.6;
  for (int i = 0; i < ncol; ++i) dcorr[i] = std::max(min_dcorr, 2.78 - 4.6 * std::fabs(lat[i] / con_pi));
}

// cmp_dcorr_lgth_oreopoulos (radiation_cloud_overlap.F90:58-93)
void oracle_dcorr_oreopoulos(int ncol, const double* lat, double juldat, int yearlength, double* dcorr) {
  const double am1 = 1.4315, am2 = 2.1219, am4 = -25.584, amr = 7.0;
  for (int i = 0; i < ncol; ++i) {
    double am3;
    if (juldat > 181.0) am3 = -(4.0 * amr * (juldat - 272.0) / (double)yearlength);
    else am3 = 4.0 * amr * (juldat - 91.0) / (double)yearlength;
    const double d = lat[i] - am3;
    dcorr[i] = am1 + am2 * std::exp(-(d * d) / (am4 * am4));
  }
}

// get_alpha_exper (radiation_cloud_overlap.F90:99-145); (ncol, nlay) arrays
// column-major with leading dimension ld.
void oracle_alpha_exper(int ncol, int nlay, int ld, int iovr, int iovr_exprand, const double* dzlay,
                        const double* dcorr, const double* cld_frac, double* alpha) {
  for (int i = 0; i < ncol; ++i) {
    alpha[i] = 0.0;
    for (int k = 1; k < nlay; ++k) alpha[i + (size_t)ld * k] = std::exp(-dzlay[i + (size_t)ld * k] / dcorr[i]);
  }
  if (iovr == iovr_exprand) {
    for (int k = 1; k < nlay; ++k)
      for (int i = 0; i < ncol; ++i)
        if (cld_frac[i + (size_t)ld * k] == 0.0 && cld_frac[i + (size_t)ld * (k - 1)] > 0.0)
          alpha[i + (size_t)ld * k] = 0.0;
  }
}

// The overlap block of radiation_clouds.f:837-856.
void oracle_overlap_params(int ncol, int nlay, int ld, int idcor, int idcor_con, int idcor_hogan,
                           int idcor_oreopoulos, double dcorr_con, const double* xlat, const double* latdeg,
                           double julian, int yearlen, double con_pi, int iovr, int iovr_dcorr, int iovr_exp,
                           int iovr_exprand, const double* dzlay, const double* cld_frac, double* de_lgth,
                           double* alpha) {
  if (idcor == idcor_hogan) oracle_dcorr_hogan(ncol, xlat, con_pi, de_lgth);
  if (idcor == idcor_oreopoulos) oracle_dcorr_oreopoulos(ncol, latdeg, julian, yearlen, de_lgth);
  if (idcor == idcor_con)
    for (int i = 0; i < ncol; ++i) de_lgth[i] = dcorr_con;
  if (iovr == iovr_dcorr || iovr == iovr_exp || iovr == iovr_exprand) {
    oracle_alpha_exper(ncol, nlay, ld, iovr, iovr_exprand, dzlay, de_lgth, cld_frac, alpha);
  } else {
    for (int i = 0; i < ncol; ++i) de_lgth[i] = 0.0;
    for (int k = 0; k < nlay; ++k)
      for (int i = 0; i < ncol; ++i) alpha[i + (size_t)ld * k] = 0.0;
  }
}

// rrtmg_lw_post_run (physics/Radiation/RRTMG/rrtmg_lw_post.F90:13-77);
// (im, ...) arrays column-major with leading dimension im.
void oracle_post(int im, int levs, int ltp, int lm, int kd, int lslwr, int lwhtr, const double* tsfa,
                 const double* htlwc, const double* htlw0, const double* sfcflw, double* tsflw, double* sfcdlw,
                 double* htrlw, double* lwhc) {
  (void)ltp;
  if (!lslwr) return;
  for (int i = 0; i < im; ++i) tsflw[i] = tsfa[i];
  for (int k = 1; k <= lm; ++k) {
    const int k1 = k + kd;
    for (int i = 0; i < im; ++i) htrlw[i + (size_t)im * (k - 1)] = htlwc[i + (size_t)im * (k1 - 1)];
  }
  if (lm < levs)
    for (int k = lm + 1; k <= levs; ++k)
      for (int i = 0; i < im; ++i) htrlw[i + (size_t)im * (k - 1)] = htrlw[i + (size_t)im * (lm - 1)];
  if (lwhtr) {
    for (int k = 1; k <= lm; ++k) {
      const int k1 = k + kd;
      for (int i = 0; i < im; ++i) lwhc[i + (size_t)im * (k - 1)] = htlw0[i + (size_t)im * (k1 - 1)];
    }
    if (lm < levs)
      for (int k = lm + 1; k <= levs; ++k)
        for (int i = 0; i < im; ++i) lwhc[i + (size_t)im * (k - 1)] = lwhc[i + (size_t)im * (lm - 1)];
  }
  for (int i = 0; i < im; ++i) sfcdlw[i] = sfcflw[4 * (size_t)i + 2];   // sfcflw%dnfxc
}

}  // extern "C"
