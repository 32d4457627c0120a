// lw_bands.cuh -- gas optics of the 16 RRTMG-LW bands for one layer.
//
// One thread owns one layer and produces, for every g-point of a band, the
// gas optical depth and the Planck fraction (taugb01..taugb16 of
// physics/Radiation/RRTMG/radlw_main.F90, RLM:4023-6840).  The per-layer
// work that does not depend on the g-point (binary-species parameters,
// table indices, interpolation weights, minor-gas column adjustments) is
// done once per band and layer; the g loop only gathers table entries.
// The floating-point order of every expression follows the Fortran.
#pragma once

#include "lw_common.cuh"

// Unrolling of the per-band g-point loops.  Full unrolling makes every table
// gather a constant offset from a per-layer row pointer, but the sixteen
// unrolled bands overflow the instruction cache: measured on B200 (16,384
// columns x 127 layers) the rolled loops run the FP32 gas-optics kernel 25%
// faster (6.4 -> 4.8 ms) and the FP64 one 3% faster, with identical results.
#ifndef LW_GLOOP_FULL
#define LW_GLOOP_FULL 0
#endif
#ifndef LW_GLOOP_N
#define LW_GLOOP_N 1
#endif
#define LW_PRAGMA_(x) _Pragma(#x)
#define LW_PRAGMA(x) LW_PRAGMA_(x)
#if LW_GLOOP_FULL
#define LW_GLOOP _Pragma("unroll")
#else
#define LW_GLOOP LW_PRAGMA(unroll LW_GLOOP_N)
#endif

namespace lw {

// Per-layer state produced by setcoef (RLM:2151-2406) and the driver
// prologue (RLM:807-1050), in the arithmetic precision R.
template <typename R>
struct Lay {
  R fac00, fac01, fac10, fac11;
  R selffac, selffrac, forfac, forfrac, minorfrac, scaleminor, scaleminorn2;
  R col[7];            // colamt(k,1..7): h2o co2 o3 n2o ch4 o2 co
  R coldry, colbrd;
  R wx[4];             // ccl4 cfc11 cfc12 cfc22
  R pavel;
  int jp, jt, jt1, indself, indfor, indminor;   // 1-based, as in the reference
  bool lower;          // k <= laytrop
};

// Shared-memory SoA record of the per-layer state (fields below), read by
// each band routine for the fields it needs, so the record does not occupy
// registers across the band loop.
enum LayField {
  LF_FAC00, LF_FAC01, LF_FAC10, LF_FAC11, LF_SELFFAC, LF_SELFFRAC, LF_FORFAC, LF_FORFRAC, LF_MINORFRAC,
  LF_SCALEMINOR, LF_SCALEMINORN2, LF_COL1, LF_COL2, LF_COL3, LF_COL4, LF_COL5, LF_COL6, LF_COL7,
  LF_COLDRY, LF_COLBRD, LF_WX1, LF_WX2, LF_WX3, LF_WX4, LF_PAVEL, N_LF
};

template <typename R>
struct LayRef {
  const R* sc;      // [N_LF][nlp]
  const int* si;    // [nlp] packed indices
  int t, nlp;
  bool lower;
  __device__ __forceinline__ Lay<R> load() const {
    Lay<R> L;
    L.fac00 = sc[LF_FAC00 * nlp + t]; L.fac01 = sc[LF_FAC01 * nlp + t];
    L.fac10 = sc[LF_FAC10 * nlp + t]; L.fac11 = sc[LF_FAC11 * nlp + t];
    L.selffac = sc[LF_SELFFAC * nlp + t]; L.selffrac = sc[LF_SELFFRAC * nlp + t];
    L.forfac = sc[LF_FORFAC * nlp + t]; L.forfrac = sc[LF_FORFRAC * nlp + t];
    L.minorfrac = sc[LF_MINORFRAC * nlp + t];
    L.scaleminor = sc[LF_SCALEMINOR * nlp + t]; L.scaleminorn2 = sc[LF_SCALEMINORN2 * nlp + t];
#pragma unroll
    for (int m = 0; m < 7; ++m) L.col[m] = sc[(LF_COL1 + m) * nlp + t];
    L.coldry = sc[LF_COLDRY * nlp + t]; L.colbrd = sc[LF_COLBRD * nlp + t];
#pragma unroll
    for (int m = 0; m < 4; ++m) L.wx[m] = sc[(LF_WX1 + m) * nlp + t];
    L.pavel = sc[LF_PAVEL * nlp + t];
    const int i0 = si[t];
    L.jp = i0 & 0xff; L.jt = (i0 >> 8) & 0xf; L.jt1 = (i0 >> 12) & 0xf;
    L.indself = (i0 >> 16) & 0xf; L.indfor = (i0 >> 20) & 0xf; L.indminor = (i0 >> 24) & 0x1f;
    L.lower = lower;
    // For a pressure profile that is not monotonic the count-based split
    // (laytrop) can send a layer to the branch of the other atmosphere, where
    // the reference indexes its tables out of bounds; keep indices in range.
    if (L.lower) { L.jp = min(L.jp, 12); L.indself = max(L.indself, 1); }
    else L.jp = max(L.jp, 13);
    return L;
  }
};

template <typename R>
struct KT {
  const R* __restrict__ p;
  // Fortran-order accessors, 1-based indices
  __device__ __forceinline__ R at(long long o) const {
    if (!LW_OK(o >= 0 && o < RRTMG_LW_TABLES_NDOUBLE, 1, o)) return R(0);
    return ldg(p + o);
  }
  __device__ __forceinline__ R a1(int off, int i) const { return at(off + (i - 1)); }
  __device__ __forceinline__ R a2(int off, int n1, int i, int j) const {
    return at(off + (i - 1) + n1 * (j - 1));
  }
  __device__ __forceinline__ R a3(int off, int n1, int n2, int i, int j, int k) const {
    return at(off + (i - 1) + n1 * ((j - 1) + n2 * (k - 1)));
  }
  __device__ __forceinline__ R chi(int m, int j) const { return a2(lwtab::chi_mls, 7, m, j); }
};

template <typename R> __device__ __forceinline__ R one() { return R(1); }
template <typename R> __device__ __forceinline__ R oneminus() { return R(1) - R(1.0e-6); }
template <typename R> __device__ __forceinline__ R lerp(R a, R f, R b) { return a + f * (b - a); }
template <typename R> __device__ __forceinline__ R fracpart(R x) { return x - trunc(x); }  // mod(x,1), x>=0

// binary-species parameter of a pair of key gases
template <typename R>
struct Spec { R comb, parm, fs; int js; };
template <typename R>
__device__ __forceinline__ Spec<R> spec(R a, R rat, R b, R nbin) {
  Spec<R> s;
  s.comb = a + rat * b;
  s.parm = a / s.comb;
  R mult = nbin * fmin(s.parm, oneminus<R>());
  // 1 + int(mult) lies in [1, nbin] for any physical column; the clamp only
  // keeps degenerate inputs (negative or NaN amounts) inside the tables
  s.js = min((int)nbin, max(1, 1 + (int)mult));
  s.fs = fracpart(mult);
  return s;
}

// 3-point species interpolation near the range ends, 2-point inside
// (e.g. RLM:4299-4333): weights w[6] = fk*{fac_lo, fac_hi} and 6 indices.
template <typename R>
struct Maj6 { R w0, w1, w2, w3, w4, w5; int i0, i1, i2, i3, i4, i5; };
template <typename R>
__device__ __forceinline__ Maj6<R> major_setup(R specparm, R fs, int ind, R facA, R facB) {
  R fk0, fk1, fk2;
  Maj6<R> m;
  if (specparm < R(0.125)) {
    R p = fs - one<R>(), p2 = p * p, p4 = p2 * p2;
    fk0 = p4; fk1 = one<R>() - p - R(2) * p4; fk2 = p + p4;
    m.i0 = ind; m.i1 = ind + 9; m.i2 = ind + 1; m.i3 = ind + 10; m.i4 = ind + 2; m.i5 = ind + 11;
  } else if (specparm > R(0.875)) {
    R p = -fs, p2 = p * p, p4 = p2 * p2;
    fk0 = p4; fk1 = one<R>() - p - R(2) * p4; fk2 = p + p4;
    m.i0 = ind + 1; m.i1 = ind + 10; m.i2 = ind; m.i3 = ind + 9; m.i4 = ind - 1; m.i5 = ind + 8;
  } else {
    fk0 = one<R>() - fs; fk1 = fs; fk2 = R(0);
    m.i0 = ind; m.i1 = ind + 9; m.i2 = ind + 1; m.i3 = ind + 10; m.i4 = ind; m.i5 = ind;
  }
  // order of the sum: fac000 a(id000) + fac010 a(id010) + fac100 a(id100)
  //                 + fac110 a(id110) + fac200 a(id200) + fac210 a(id210)
  m.w0 = fk0 * facA; m.w1 = fk0 * facB; m.w2 = fk1 * facA; m.w3 = fk1 * facB;
  m.w4 = fk2 * facA; m.w5 = fk2 * facB;
  return m;
}
template <typename R>
__device__ __forceinline__ R major6(const KT<R>& t, int off, int ng, int ig, const Maj6<R>& m) {
  return m.w0 * t.a2(off, ng, ig, m.i0) + m.w1 * t.a2(off, ng, ig, m.i1) +
         m.w2 * t.a2(off, ng, ig, m.i2) + m.w3 * t.a2(off, ng, ig, m.i3) +
         m.w4 * t.a2(off, ng, ig, m.i4) + m.w5 * t.a2(off, ng, ig, m.i5);
}

// lower-atmosphere set-up of a binary-species band (two reference pressures)
template <typename R>
struct Low { Spec<R> s0, s1; Maj6<R> m0, m1; };
template <typename R, int B>
__device__ __forceinline__ Low<R> low_setup(const Lay<R>& L, R a, R r0, R r1, R b) {
  Low<R> o;
  o.s0 = spec<R>(a, r0, b, R(8));
  int ind0 = ((L.jp - 1) * 5 + (L.jt - 1)) * nspa_of(B) + o.s0.js;
  o.s1 = spec<R>(a, r1, b, R(8));
  int ind1 = (L.jp * 5 + (L.jt1 - 1)) * nspa_of(B) + o.s1.js;
  o.m0 = major_setup<R>(o.s0.parm, o.s0.fs, ind0, L.fac00, L.fac10);
  o.m1 = major_setup<R>(o.s1.parm, o.s1.fs, ind1, L.fac01, L.fac11);
  return o;
}
template <typename R>
__device__ __forceinline__ R low_major(const KT<R>& t, int off, int ng, int ig, const Low<R>& o) {
  return o.s0.comb * major6(t, off, ng, ig, o.m0) + o.s1.comb * major6(t, off, ng, ig, o.m1);
}

// upper-atmosphere set-up of a binary-species band (bands 3, 4, 5)
template <typename R>
struct Up { R comb0, comb1, f000, f010, f100, f110, f001, f011, f101, f111; int ind0, ind1; };
template <typename R, int B>
__device__ __forceinline__ Up<R> up_setup(const Lay<R>& L, R a, R r0, R r1, R b) {
  Up<R> u;
  Spec<R> s0 = spec<R>(a, r0, b, R(4));
  Spec<R> s1 = spec<R>(a, r1, b, R(4));
  u.comb0 = s0.comb; u.comb1 = s1.comb;
  u.ind0 = ((L.jp - 13) * 5 + (L.jt - 1)) * nspb_of(B) + s0.js;
  u.ind1 = ((L.jp - 12) * 5 + (L.jt1 - 1)) * nspb_of(B) + s1.js;
  R fk0 = one<R>() - s0.fs, fk1 = s0.fs;
  u.f000 = fk0 * L.fac00; u.f010 = fk0 * L.fac10; u.f100 = fk1 * L.fac00; u.f110 = fk1 * L.fac10;
  fk0 = one<R>() - s1.fs; fk1 = s1.fs;
  u.f001 = fk0 * L.fac01; u.f011 = fk0 * L.fac11; u.f101 = fk1 * L.fac01; u.f111 = fk1 * L.fac11;
  return u;
}
template <typename R>
__device__ __forceinline__ R up_major(const KT<R>& t, int off, int ng, int ig, const Up<R>& u) {
  R a = u.f000 * t.a2(off, ng, ig, u.ind0) + u.f010 * t.a2(off, ng, ig, u.ind0 + 5) +
        u.f100 * t.a2(off, ng, ig, u.ind0 + 1) + u.f110 * t.a2(off, ng, ig, u.ind0 + 6);
  R b = u.f001 * t.a2(off, ng, ig, u.ind1) + u.f011 * t.a2(off, ng, ig, u.ind1 + 5) +
        u.f101 * t.a2(off, ng, ig, u.ind1 + 1) + u.f111 * t.a2(off, ng, ig, u.ind1 + 6);
  return u.comb0 * a + u.comb1 * b;
}

// single-key-species 4-point interpolation
template <typename R>
__device__ __forceinline__ R absk(const KT<R>& t, int off, int ng, int ig, const Lay<R>& L, int ind0, int ind1) {
  return L.fac00 * t.a2(off, ng, ig, ind0) + L.fac10 * t.a2(off, ng, ig, ind0 + 1) +
         L.fac01 * t.a2(off, ng, ig, ind1) + L.fac11 * t.a2(off, ng, ig, ind1 + 1);
}
template <typename R, int B> __device__ __forceinline__ int lo0(const Lay<R>& L) { return ((L.jp - 1) * 5 + (L.jt - 1)) * nspa_of(B) + 1; }
template <typename R, int B> __device__ __forceinline__ int lo1(const Lay<R>& L) { return (L.jp * 5 + (L.jt1 - 1)) * nspa_of(B) + 1; }
template <typename R, int B> __device__ __forceinline__ int up0(const Lay<R>& L) { return ((L.jp - 13) * 5 + (L.jt - 1)) * nspb_of(B) + 1; }
template <typename R, int B> __device__ __forceinline__ int up1(const Lay<R>& L) { return ((L.jp - 12) * 5 + (L.jt1 - 1)) * nspb_of(B) + 1; }

template <typename R>
__device__ __forceinline__ R selfc(const KT<R>& t, int off, int ng, int ig, const Lay<R>& L) {
  return L.selffac * lerp(t.a2(off, ng, ig, L.indself), L.selffrac, t.a2(off, ng, ig, L.indself + 1));
}
template <typename R>
__device__ __forceinline__ R forc(const KT<R>& t, int off, int ng, int ig, const Lay<R>& L) {
  return L.forfac * lerp(t.a2(off, ng, ig, L.indfor), L.forfrac, t.a2(off, ng, ig, L.indfor + 1));
}
template <typename R>
__device__ __forceinline__ R minor2(const KT<R>& t, int off, int ng, int ig, const Lay<R>& L) {
  return lerp(t.a2(off, ng, ig, L.indminor), L.minorfrac, t.a2(off, ng, ig, L.indminor + 1));
}
template <typename R>
__device__ __forceinline__ R minor3(const KT<R>& t, int off, int ng, int nj, int ig, int j, R f, const Lay<R>& L) {
  int m = L.indminor;
  R m1 = t.a3(off, ng, nj, ig, j, m) + f * (t.a3(off, ng, nj, ig, j + 1, m) - t.a3(off, ng, nj, ig, j, m));
  R m2 = t.a3(off, ng, nj, ig, j, m + 1) + f * (t.a3(off, ng, nj, ig, j + 1, m + 1) - t.a3(off, ng, nj, ig, j, m + 1));
  return m1 + L.minorfrac * (m2 - m1);
}
template <typename R>
__device__ __forceinline__ R planck(const KT<R>& t, int off, int ng, int ig, int jpl, R fpl) {
  return lerp(t.a2(off, ng, ig, jpl), fpl, t.a2(off, ng, ig, jpl + 1));
}
// minor-gas column adjusted above `thresh` times its reference amount
template <typename R>
__device__ __forceinline__ R adjcol(R col, R ref, R thresh, R base, R expo) {
  R rat = col / ref;
  if (rat > thresh) return (base + pow(rat - base, expo)) * ref;
  return col;
}

// ---------------------------------------------------------------------------
// Each band: for g-points ig = 1..ng call emit(ig-1, taug, fracs).
// ---------------------------------------------------------------------------

template <typename R, typename E>  // taugb01, RLM:4023-4125
__device__ void taugb01(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 10;
  R scalen2 = L.colbrd * L.scaleminorn2;
  if (L.lower) {
    int i0 = lo0<R, 0>(L), i1 = lo1<R, 0>(L);
    R pp = L.pavel;
    R corradj = (pp < R(250)) ? one<R>() - R(0.15) * (R(250) - pp) / R(154.4) : one<R>();
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b01_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b01_forref, ng, ig, L);
      R taun2 = scalen2 * minor2(t, lwtab::b01_ka_mn2, ng, ig, L);
      emit(ig - 1, corradj * (L.col[0] * absk(t, lwtab::b01_absa, ng, ig, L, i0, i1) + tauself + taufor + taun2),
           t.a1(lwtab::b01_fracrefa, ig));
    }
  } else {
    int i0 = up0<R, 0>(L), i1 = up1<R, 0>(L);
    R corradj = one<R>() - R(0.15) * (L.pavel / R(95.6));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R taufor = forc(t, lwtab::b01_forref, ng, ig, L);
      R taun2 = scalen2 * minor2(t, lwtab::b01_kb_mn2, ng, ig, L);
      emit(ig - 1, corradj * (L.col[0] * absk(t, lwtab::b01_absb, ng, ig, L, i0, i1) + taufor + taun2),
           t.a1(lwtab::b01_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb02, RLM:4131-4203
__device__ void taugb02(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 12;
  if (L.lower) {
    int i0 = lo0<R, 1>(L), i1 = lo1<R, 1>(L);
    R corradj = one<R>() - R(0.05) * (L.pavel - R(100)) / R(900);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b02_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b02_forref, ng, ig, L);
      emit(ig - 1, corradj * (L.col[0] * absk(t, lwtab::b02_absa, ng, ig, L, i0, i1) + tauself + taufor),
           t.a1(lwtab::b02_fracrefa, ig));
    }
  } else {
    int i0 = up0<R, 1>(L), i1 = up1<R, 1>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R taufor = forc(t, lwtab::b02_forref, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b02_absb, ng, ig, L, i0, i1) + taufor, t.a1(lwtab::b02_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb03, RLM:4210-4512
__device__ void taugb03(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 16;
  R adjcoln2o = adjcol<R>(L.col[3], L.coldry * t.chi(4, L.jp + 1), R(1.5), R(0.5), R(0.65));
  if (L.lower) {
    R rpa = t.chi(1, 9) / t.chi(2, 9), rma = t.chi(1, 3) / t.chi(2, 3);
    Low<R> o = low_setup<R, 2>(L, L.col[0], t.chi(1, L.jp) / t.chi(2, L.jp), t.chi(1, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sm = spec<R>(L.col[0], rma, L.col[1], R(8));
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[1], R(8));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b03_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b03_forref, ng, ig, L);
      R absn2o = minor3(t, lwtab::b03_ka_mn2o, ng, 9, ig, sm.js, sm.fs, L);
      R tau_major = o.s0.comb * major6(t, lwtab::b03_absa, ng, ig, o.m0);
      R tau_major1 = o.s1.comb * major6(t, lwtab::b03_absa, ng, ig, o.m1);
      emit(ig - 1, tau_major + tau_major1 + tauself + taufor + adjcoln2o * absn2o,
           planck(t, lwtab::b03_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    R rpb = t.chi(1, 13) / t.chi(2, 13), rmb = t.chi(1, 13) / t.chi(2, 13);
    Up<R> u = up_setup<R, 2>(L, L.col[0], t.chi(1, L.jp) / t.chi(2, L.jp), t.chi(1, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sm = spec<R>(L.col[0], rmb, L.col[1], R(4));
    Spec<R> sp = spec<R>(L.col[0], rpb, L.col[1], R(4));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R taufor = forc(t, lwtab::b03_forref, ng, ig, L);
      R absn2o = minor3(t, lwtab::b03_kb_mn2o, ng, 5, ig, sm.js, sm.fs, L);
      emit(ig - 1, up_major(t, lwtab::b03_absb, ng, ig, u) + taufor + adjcoln2o * absn2o,
           planck(t, lwtab::b03_fracrefb, ng, ig, sp.js, sp.fs));
    }
  }
}

template <typename R, typename E>  // taugb04, RLM:4518-4757
__device__ void taugb04(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 14;
  if (L.lower) {
    R rpa = t.chi(1, 11) / t.chi(2, 11);
    Low<R> o = low_setup<R, 3>(L, L.col[0], t.chi(1, L.jp) / t.chi(2, L.jp), t.chi(1, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[1], R(8));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b04_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b04_forref, ng, ig, L);
      R tau_major = o.s0.comb * major6(t, lwtab::b04_absa, ng, ig, o.m0);
      R tau_major1 = o.s1.comb * major6(t, lwtab::b04_absa, ng, ig, o.m1);
      emit(ig - 1, tau_major + tau_major1 + tauself + taufor, planck(t, lwtab::b04_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    R rpb = t.chi(3, 13) / t.chi(2, 13);
    Up<R> u = up_setup<R, 3>(L, L.col[2], t.chi(3, L.jp) / t.chi(2, L.jp), t.chi(3, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sp = spec<R>(L.col[2], rpb, L.col[1], R(4));
    // empirical scalings of g-points 8..14 (RLM:4746-4752)
    const R sc[14] = {R(1), R(1), R(1), R(1), R(1), R(1), R(1), R(0.92), R(0.88), R(1.07), R(1.1), R(0.99), R(0.88), R(0.943)};
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tau = up_major(t, lwtab::b04_absb, ng, ig, u);
      if (ig >= 8) tau = tau * sc[ig - 1];
      emit(ig - 1, tau, planck(t, lwtab::b04_fracrefb, ng, ig, sp.js, sp.fs));
    }
  }
}

template <typename R, typename E>  // taugb05, RLM:4764-5023
__device__ void taugb05(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 16;
  if (L.lower) {
    R rpa = t.chi(1, 5) / t.chi(2, 5), rma = t.chi(1, 7) / t.chi(2, 7);
    Low<R> o = low_setup<R, 4>(L, L.col[0], t.chi(1, L.jp) / t.chi(2, L.jp), t.chi(1, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sm = spec<R>(L.col[0], rma, L.col[1], R(8));
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[1], R(8));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b05_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b05_forref, ng, ig, L);
      R abso3 = minor3(t, lwtab::b05_ka_mo3, ng, 9, ig, sm.js, sm.fs, L);
      emit(ig - 1, low_major(t, lwtab::b05_absa, ng, ig, o) + tauself + taufor + abso3 * L.col[2] +
                       L.wx[0] * t.a1(lwtab::b05_ccl4, ig),
           planck(t, lwtab::b05_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    R rpb = t.chi(3, 43) / t.chi(2, 43);
    Up<R> u = up_setup<R, 4>(L, L.col[2], t.chi(3, L.jp) / t.chi(2, L.jp), t.chi(3, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sp = spec<R>(L.col[2], rpb, L.col[1], R(4));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig)
      emit(ig - 1, up_major(t, lwtab::b05_absb, ng, ig, u) + L.wx[0] * t.a1(lwtab::b05_ccl4, ig),
           planck(t, lwtab::b05_fracrefb, ng, ig, sp.js, sp.fs));
  }
}

template <typename R, typename E>  // taugb06, RLM:5030-5111
__device__ void taugb06(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 8;
  if (L.lower) {
    int i0 = lo0<R, 5>(L), i1 = lo1<R, 5>(L);
    R adjcolco2 = adjcol<R>(L.col[1], L.coldry * t.chi(2, L.jp + 1), R(3), R(2), R(0.77));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b06_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b06_forref, ng, ig, L);
      R absco2 = minor2(t, lwtab::b06_ka_mco2, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b06_absa, ng, ig, L, i0, i1) + tauself + taufor + adjcolco2 * absco2 +
                       L.wx[1] * t.a1(lwtab::b06_cfc11adj, ig) + L.wx[2] * t.a1(lwtab::b06_cfc12, ig),
           t.a1(lwtab::b06_fracrefa, ig));
    }
  } else {
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig)
      emit(ig - 1, L.wx[1] * t.a1(lwtab::b06_cfc11adj, ig) + L.wx[2] * t.a1(lwtab::b06_cfc12, ig),
           t.a1(lwtab::b06_fracrefa, ig));
  }
}

template <typename R, typename E>  // taugb07, RLM:5118-5375
__device__ void taugb07(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 12;
  if (L.lower) {
    R rpa = t.chi(1, 3) / t.chi(3, 3), rma = t.chi(1, 3) / t.chi(3, 3);
    Low<R> o = low_setup<R, 6>(L, L.col[0], t.chi(1, L.jp) / t.chi(3, L.jp), t.chi(1, L.jp + 1) / t.chi(3, L.jp + 1), L.col[2]);
    Spec<R> sm = spec<R>(L.col[0], rma, L.col[2], R(8));
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[2], R(8));
    R adjcolco2 = adjcol<R>(L.col[1], L.coldry * t.chi(2, L.jp + 1), R(3), R(3), R(0.79));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b07_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b07_forref, ng, ig, L);
      R absco2 = minor3(t, lwtab::b07_ka_mco2, ng, 9, ig, sm.js, sm.fs, L);
      emit(ig - 1, low_major(t, lwtab::b07_absa, ng, ig, o) + tauself + taufor + adjcolco2 * absco2,
           planck(t, lwtab::b07_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    R adjcolco2 = adjcol<R>(L.col[1], L.coldry * t.chi(2, L.jp + 1), R(3), R(2), R(0.79));
    int i0 = up0<R, 6>(L), i1 = up1<R, 6>(L);
    // RLM:5366-5371
    const R sc[12] = {R(1), R(1), R(1), R(1), R(1), R(0.92), R(0.88), R(1.07), R(1.1), R(0.99), R(0.855), R(1)};
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R absco2 = minor2(t, lwtab::b07_kb_mco2, ng, ig, L);
      R tau = L.col[2] * absk(t, lwtab::b07_absb, ng, ig, L, i0, i1) + adjcolco2 * absco2;
      if (ig >= 6 && ig <= 11) tau = tau * sc[ig - 1];
      emit(ig - 1, tau, t.a1(lwtab::b07_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb08, RLM:5382-5501
__device__ void taugb08(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 8;
  R adjcolco2 = adjcol<R>(L.col[1], L.coldry * t.chi(2, L.jp + 1), R(3), R(2), R(0.65));
  if (L.lower) {
    int i0 = lo0<R, 7>(L), i1 = lo1<R, 7>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b08_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b08_forref, ng, ig, L);
      R absco2 = minor2(t, lwtab::b08_ka_mco2, ng, ig, L);
      R abso3 = minor2(t, lwtab::b08_ka_mo3, ng, ig, L);
      R absn2o = minor2(t, lwtab::b08_ka_mn2o, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b08_absa, ng, ig, L, i0, i1) + tauself + taufor + adjcolco2 * absco2 +
                       L.col[2] * abso3 + L.col[3] * absn2o + L.wx[2] * t.a1(lwtab::b08_cfc12, ig) +
                       L.wx[3] * t.a1(lwtab::b08_cfc22adj, ig),
           t.a1(lwtab::b08_fracrefa, ig));
    }
  } else {
    int i0 = up0<R, 7>(L), i1 = up1<R, 7>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R absco2 = minor2(t, lwtab::b08_kb_mco2, ng, ig, L);
      R absn2o = minor2(t, lwtab::b08_kb_mn2o, ng, ig, L);
      emit(ig - 1, L.col[2] * absk(t, lwtab::b08_absb, ng, ig, L, i0, i1) + adjcolco2 * absco2 + L.col[3] * absn2o +
                       L.wx[2] * t.a1(lwtab::b08_cfc12, ig) + L.wx[3] * t.a1(lwtab::b08_cfc22adj, ig),
           t.a1(lwtab::b08_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb09, RLM:5508-5753
__device__ void taugb09(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 12;
  R adjcoln2o = adjcol<R>(L.col[3], L.coldry * t.chi(4, L.jp + 1), R(1.5), R(0.5), R(0.65));
  if (L.lower) {
    R rpa = t.chi(1, 9) / t.chi(6, 9), rma = t.chi(1, 3) / t.chi(6, 3);
    Low<R> o = low_setup<R, 8>(L, L.col[0], t.chi(1, L.jp) / t.chi(6, L.jp), t.chi(1, L.jp + 1) / t.chi(6, L.jp + 1), L.col[4]);
    Spec<R> sm = spec<R>(L.col[0], rma, L.col[4], R(8));
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[4], R(8));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b09_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b09_forref, ng, ig, L);
      R absn2o = minor3(t, lwtab::b09_ka_mn2o, ng, 9, ig, sm.js, sm.fs, L);
      emit(ig - 1, low_major(t, lwtab::b09_absa, ng, ig, o) + tauself + taufor + adjcoln2o * absn2o,
           planck(t, lwtab::b09_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    int i0 = up0<R, 8>(L), i1 = up1<R, 8>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R absn2o = minor2(t, lwtab::b09_kb_mn2o, ng, ig, L);
      emit(ig - 1, L.col[4] * absk(t, lwtab::b09_absb, ng, ig, L, i0, i1) + adjcoln2o * absn2o,
           t.a1(lwtab::b09_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb10, RLM:5759-5829
__device__ void taugb10(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 6;
  if (L.lower) {
    int i0 = lo0<R, 9>(L), i1 = lo1<R, 9>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b10_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b10_forref, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b10_absa, ng, ig, L, i0, i1) + tauself + taufor, t.a1(lwtab::b10_fracrefa, ig));
    }
  } else {
    int i0 = up0<R, 9>(L), i1 = up1<R, 9>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R taufor = forc(t, lwtab::b10_forref, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b10_absb, ng, ig, L, i0, i1) + taufor, t.a1(lwtab::b10_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb11, RLM:5836-5923
__device__ void taugb11(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 8;
  R scaleo2 = L.col[5] * L.scaleminor;
  if (L.lower) {
    int i0 = lo0<R, 10>(L), i1 = lo1<R, 10>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b11_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b11_forref, ng, ig, L);
      R tauo2 = scaleo2 * minor2(t, lwtab::b11_ka_mo2, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b11_absa, ng, ig, L, i0, i1) + tauself + taufor + tauo2,
           t.a1(lwtab::b11_fracrefa, ig));
    }
  } else {
    int i0 = up0<R, 10>(L), i1 = up1<R, 10>(L);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R taufor = forc(t, lwtab::b11_forref, ng, ig, L);
      R tauo2 = scaleo2 * minor2(t, lwtab::b11_kb_mo2, ng, ig, L);
      emit(ig - 1, L.col[0] * absk(t, lwtab::b11_absb, ng, ig, L, i0, i1) + taufor + tauo2, t.a1(lwtab::b11_fracrefb, ig));
    }
  }
}

template <typename R, typename E>  // taugb12, RLM:5929-6111
__device__ void taugb12(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 8;
  if (L.lower) {
    R rpa = t.chi(1, 10) / t.chi(2, 10);
    Low<R> o = low_setup<R, 11>(L, L.col[0], t.chi(1, L.jp) / t.chi(2, L.jp), t.chi(1, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    // RLM:5974-5977: Planck parameter clipped with '>= oneminus'
    R comb = L.col[0] + rpa * L.col[1];
    R parm = L.col[0] / comb;
    if (parm >= oneminus<R>()) parm = oneminus<R>();
    R mult = R(8) * parm;
    int jpl = min(8, max(1, 1 + (int)mult));
    R fpl = fracpart(mult);
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b12_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b12_forref, ng, ig, L);
      emit(ig - 1, low_major(t, lwtab::b12_absa, ng, ig, o) + tauself + taufor, planck(t, lwtab::b12_fracrefa, ng, ig, jpl, fpl));
    }
  } else {
    for (int ig = 1; ig <= ng; ++ig) emit(ig - 1, R(0), R(0));
  }
}

template <typename R, typename E>  // taugb13, RLM:6117-6361
__device__ void taugb13(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 4;
  if (L.lower) {
    R rpa = t.chi(1, 5) / t.chi(4, 5), rma = t.chi(1, 1) / t.chi(4, 1), rma3 = t.chi(1, 3) / t.chi(4, 3);
    Low<R> o = low_setup<R, 12>(L, L.col[0], t.chi(1, L.jp) / t.chi(4, L.jp), t.chi(1, L.jp + 1) / t.chi(4, L.jp + 1), L.col[3]);
    Spec<R> smco2 = spec<R>(L.col[0], rma, L.col[3], R(8));
    Spec<R> smco = spec<R>(L.col[0], rma3, L.col[3], R(8));
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[3], R(8));
    R adjcolco2 = adjcol<R>(L.col[1], L.coldry * R(3.55e-4), R(3), R(2), R(0.68));
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b13_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b13_forref, ng, ig, L);
      R absco2 = minor3(t, lwtab::b13_ka_mco2, ng, 9, ig, smco2.js, smco2.fs, L);
      R absco = minor3(t, lwtab::b13_ka_mco, ng, 9, ig, smco.js, smco.fs, L);
      emit(ig - 1, low_major(t, lwtab::b13_absa, ng, ig, o) + tauself + taufor + adjcolco2 * absco2 + L.col[6] * absco,
           planck(t, lwtab::b13_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
LW_GLOOP
    for (int ig = 1; ig <= ng; ++ig)
      emit(ig - 1, L.col[2] * minor2(t, lwtab::b13_kb_mo3, ng, ig, L), t.a1(lwtab::b13_fracrefb, ig));
  }
}

template <typename R, typename E>  // taugb14, RLM:6367-6431
__device__ void taugb14(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 2;
  if (L.lower) {
    int i0 = lo0<R, 13>(L), i1 = lo1<R, 13>(L);
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b14_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b14_forref, ng, ig, L);
      emit(ig - 1, L.col[1] * absk(t, lwtab::b14_absa, ng, ig, L, i0, i1) + tauself + taufor, t.a1(lwtab::b14_fracrefa, ig));
    }
  } else {
    int i0 = up0<R, 13>(L), i1 = up1<R, 13>(L);
    for (int ig = 1; ig <= ng; ++ig)
      emit(ig - 1, L.col[1] * absk(t, lwtab::b14_absb, ng, ig, L, i0, i1), t.a1(lwtab::b14_fracrefb, ig));
  }
}

template <typename R, typename E>  // taugb15, RLM:6438-6644
__device__ void taugb15(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 2;
  if (L.lower) {
    R rpa = t.chi(4, 1) / t.chi(2, 1), rma = t.chi(4, 1) / t.chi(2, 1);
    Low<R> o = low_setup<R, 14>(L, L.col[3], t.chi(4, L.jp) / t.chi(2, L.jp), t.chi(4, L.jp + 1) / t.chi(2, L.jp + 1), L.col[1]);
    Spec<R> sm = spec<R>(L.col[3], rma, L.col[1], R(8));
    Spec<R> sp = spec<R>(L.col[3], rpa, L.col[1], R(8));
    R scalen2 = L.colbrd * L.scaleminor;
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b15_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b15_forref, ng, ig, L);
      R taun2 = scalen2 * minor3(t, lwtab::b15_ka_mn2, ng, 9, ig, sm.js, sm.fs, L);
      emit(ig - 1, low_major(t, lwtab::b15_absa, ng, ig, o) + tauself + taufor + taun2,
           planck(t, lwtab::b15_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    for (int ig = 1; ig <= ng; ++ig) emit(ig - 1, R(0), R(0));
  }
}

template <typename R, typename E>  // taugb16, RLM:6650-6840
__device__ void taugb16(const KT<R>& t, const LayRef<R>& LR, E emit) {
  const Lay<R> L = LR.load();
  constexpr int ng = 2;
  if (L.lower) {
    R rpa = t.chi(1, 6) / t.chi(6, 6);
    Low<R> o = low_setup<R, 15>(L, L.col[0], t.chi(1, L.jp) / t.chi(6, L.jp), t.chi(1, L.jp + 1) / t.chi(6, L.jp + 1), L.col[4]);
    Spec<R> sp = spec<R>(L.col[0], rpa, L.col[4], R(8));
    for (int ig = 1; ig <= ng; ++ig) {
      R tauself = selfc(t, lwtab::b16_selfref, ng, ig, L);
      R taufor = forc(t, lwtab::b16_forref, ng, ig, L);
      emit(ig - 1, low_major(t, lwtab::b16_absa, ng, ig, o) + tauself + taufor, planck(t, lwtab::b16_fracrefa, ng, ig, sp.js, sp.fs));
    }
  } else {
    // nspb(16) = 0 (RLM:327): both indices are 1 for every upper layer
    int i0 = up0<R, 15>(L), i1 = up1<R, 15>(L);
    for (int ig = 1; ig <= ng; ++ig)
      emit(ig - 1, L.col[4] * absk(t, lwtab::b16_absb, ng, ig, L, i0, i1), t.a1(lwtab::b16_fracrefb, ig));
  }
}

template <typename R, typename E>
__device__ __forceinline__ void band_gas_optics(int b, const KT<R>& t, const LayRef<R>& L, E emit) {
  switch (b) {
    case 0: taugb01(t, L, emit); break;
    case 1: taugb02(t, L, emit); break;
    case 2: taugb03(t, L, emit); break;
    case 3: taugb04(t, L, emit); break;
    case 4: taugb05(t, L, emit); break;
    case 5: taugb06(t, L, emit); break;
    case 6: taugb07(t, L, emit); break;
    case 7: taugb08(t, L, emit); break;
    case 8: taugb09(t, L, emit); break;
    case 9: taugb10(t, L, emit); break;
    case 10: taugb11(t, L, emit); break;
    case 11: taugb12(t, L, emit); break;
    case 12: taugb13(t, L, emit); break;
    case 13: taugb14(t, L, emit); break;
    case 14: taugb15(t, L, emit); break;
    default: taugb16(t, L, emit); break;
  }
}

}  // namespace lw
