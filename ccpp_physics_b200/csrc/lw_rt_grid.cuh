// lw_rt_grid.cuh -- kernel B for grid-mean clouds (isubclw = 0): the random
// overlap transfer rtrn (RLM:2445-2800, iovr <= 0) and the maximum-random
// overlap transfer rtrnmr (RLM:2828-3392, iovr > 0).
//
// Unlike McICA's 0/1 sub-columns, a layer here carries its cloud fraction,
// and rtrnmr splits the radiance into clear and cloudy parts whose exchange
// at cloud-block edges depends on the neighbouring layers' fractions.  The
// recurrences are run the way the reference runs them, layer by layer, with
// one lane per g-point: a warp owns a column and handles two bands per pass
// (one per 16-lane half; no band has more than 16 g-points), so the sums over
// a band's g-points are 4-step half-warp reductions.  The overlap factors of
// rtrnmr depend only on the cloud-fraction profile; lane 0 computes them once
// per column into shared memory.
//
// Scratch (written by the gas-optics kernel, layout of lw_gas.cuh): tau/frac
// per g-point and layer, pklay/pklev/taucld per band, the column record
// (secdiff, pklay at the surface, emissivity).  Layers are surface first,
// 1-based below as in the reference (internal layer k <-> scratch row k-1).
#pragma once

#include "lw_common.cuh"
#include "lw_gas.cuh"

namespace lw {

// doubles of shared memory per warp (one warp per CTA) for nlay layers
__host__ __device__ inline size_t rt_grid_smem_doubles(int nlay) {
  return (size_t)(nlay + 2) * 15 + (size_t)(nlay + 1) * 8;
}

// Maximum-random overlap factors (RLM:2921-3092) of one sweep direction, as in
// the oracle: dir = +1 pairs layer k with k+1 and looks back at k-1, dir = -1
// pairs k with k-1 and looks back at k+1; factors of a pair are stored at the
// index of the layer the sweep moves to.  cf is cldfrc(0:nlay+1).
__device__ inline void rt_grid_mr_factors(const double* cf, int nlay, int dir, double* clr1, double* clr2,
                                          double* cld1, double* cld2, double* cmb1, double* cmb2, double* lst) {
  const double eps = kEps;
  for (int k = 0; k <= nlay + 1; ++k) clr1[k] = clr2[k] = cld1[k] = cld2[k] = cmb1[k] = cmb2[k] = lst[k] = 0.0;
  const int k0 = dir > 0 ? 1 : nlay, k1 = dir > 0 ? nlay - 1 : 2;
  lst[k0] = cf[k0] > eps ? 1.0 : 0.0;
  double rat1 = 0.0, rat2 = 0.0;
  for (int k = k0; dir > 0 ? k <= k1 : k >= k1; k += dir) {
    const int kn = k + dir, kb = k - dir;
    lst[kn] = (cf[kn] > eps && cf[k] <= eps) ? 1.0 : 0.0;
    if (!(cf[k] > eps)) continue;
    if (cf[kn] >= cf[k]) {
      if (lst[k] != 0.0) {
        if (cf[k] < 1.0) clr2[kn] = (cf[kn] - cf[k]) / (1.0 - cf[k]);
        clr2[k] = 0.0;
        cld2[k] = 0.0;
      } else {
        const double fmx = fmax(cf[k], cf[kb]);
        if (cf[kn] > fmx) {
          clr1[kn] = rat2;
          clr2[kn] = (cf[kn] - fmx) / (1.0 - fmx);
        } else if (cf[kn] < fmx) {
          clr1[kn] = (cf[kn] - cf[k]) / (cf[kb] - cf[k]);
        } else {
          clr1[kn] = rat2;
        }
      }
      if (clr1[kn] > 0.0 || clr2[kn] > 0.0) { rat1 = 1.0; rat2 = 0.0; }
      else { rat1 = 0.0; rat2 = 0.0; }
    } else {
      if (lst[k] != 0.0) {
        cld2[kn] = (cf[k] - cf[kn]) / cf[k];
        clr2[k] = 0.0;
        cld2[k] = 0.0;
      } else {
        const double fmn = fmin(cf[k], cf[kb]);
        if (cf[kn] <= fmn) {
          cld1[kn] = rat1;
          cld2[kn] = (fmn - cf[kn]) / fmn;
        } else {
          cld1[kn] = (cf[k] - cf[kn]) / (cf[k] - fmn);
        }
      }
      if (cld1[kn] > 0.0 || cld2[kn] > 0.0) { rat1 = 0.0; rat2 = 1.0; }
      else { rat1 = 0.0; rat2 = 0.0; }
    }
    cmb1[kn] = clr1[kn] * cld2[k] * cf[kb];
    cmb2[kn] = cld1[kn] * clr2[k] * (1.0 - cf[kb]);
  }
}

// gas part of one layer (RLM:2601-2627): transmittance, optical depth after
// the table, and the down/up Planck sources
template <typename R>
struct GasL {
  R trng, odepth, gsd, gsu, frac, blay, dplnku, dplnkd;
};
template <typename R>
__device__ __forceinline__ GasL<R> grid_gas_layer(R tau, R frac, R secd, R blay, R plevu, R plevd,
                                                  const Tables<R>& tab) {
  GasL<R> o;
  R odepth = fmax(R(0), secd * tau);
  R atrgas, gasfac;
  if (odepth <= R(0.06)) {
    atrgas = odepth - R(0.5) * odepth * odepth;
    o.trng = R(1) - atrgas;
    gasfac = R(kRec6) * odepth;
  } else {
    const R tblind = tbl_quot(odepth);
    const int itgas = min(NTBL, max(0, (int)(R(kTblint) * tblind + R(0.5))));
    tbl_rec(tab.trec, itgas, o.trng, gasfac, odepth);
    atrgas = R(1) - o.trng;
  }
  o.odepth = odepth;
  o.frac = frac;
  o.blay = blay;
  o.dplnku = plevu - blay;
  o.dplnkd = plevd - blay;
  o.gsd = frac * (blay + o.dplnkd * gasfac) * atrgas;
  o.gsu = frac * (blay + o.dplnku * gasfac) * atrgas;
  return o;
}

// cloudy part: total-sky table terms (RLM:2636-2650, 3193-3202)
template <typename R>
__device__ __forceinline__ void grid_tot_layer(R odtot, const Tables<R>& tab, R& totfac, R& atrtot, R& trnt) {
  if (odtot < R(0.06)) {
    totfac = R(kRec6) * odtot;
    atrtot = odtot - R(0.5) * odtot * odtot;
    trnt = R(1) - atrtot;
  } else {
    const R tblind = tbl_quot(odtot);
    const int ittot = min(NTBL, max(0, (int)(R(kTblint) * tblind + R(0.5))));
    R ta;
    tbl_rec(tab.trec, ittot, trnt, totfac, ta);
    atrtot = R(1) - trnt;
  }
}

// sum over the 16 lanes of this half-warp (every lane gets the half's sum)
__device__ __forceinline__ double half_sum(double v) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename R, int V, bool HLWB>
__global__ void __launch_bounds__(32)
lw_rt_grid_kernel(const Block* __restrict__ blocks, int nblocks, const Block b0, int ncols, Flags f, Consts cs,
                  Tables<R> tab, Scratch<R> sc) {
  constexpr int NLP = 32 * V;
  extern __shared__ __align__(16) double sg[];
  const int lane = threadIdx.x & 31;
  const int nlay = f.nlay, nlp1 = nlay + 1, L2 = nlay + 2;
  const double eps = kEps;
  const bool mr = f.iovr > 0;
  double* cf = sg;                        // cldfrc(0:nlay+1)
  double* ufac = cf + L2;                 // up: clr1, clr2, cld1, cld2, cmb1, cmb2, lst (7 x L2)
  double* dfac = ufac + 7 * L2;           // down: same
  double* ftu = dfac + 7 * L2;            // level sums (0:nlay): total up/down, clear up/down
  double* ftd = ftu + nlp1;
  double* fcu = ftd + nlp1;
  double* fcd = fcu + nlp1;
  double* bnd = fcd + nlp1;               // band level sums of the pass: [half][up, down][0:nlay]
  const double flxfac = 0.5 * cs.fluxfac;

  for (int cc = blockIdx.x; cc < ncols; cc += gridDim.x) {
    const int c = sc.c0 + cc;
    const Block& B = (nblocks == 1) ? b0 : blocks[find_block(blocks, nblocks, c)];
    const int i = c - B.col0;
    const size_t ld = (size_t)B.ld;
    const bool top = f.top_at_1 != 0;
    if (!LW_OK(cc < sc.cap && c < sc.ntot && i >= 0 && i < B.npts, 41, cc)) continue;
    __syncwarp();
    // cloud-fraction profile in the internal order, padded (RLM:888-907)
    for (int k = lane; k <= nlay + 1; k += 32) {
      double v;
      if (k == 0) v = 1.0;
      else if (k == nlay + 1) v = 0.0;
      else v = B.in[F_CLDCF][i + ld * (size_t)(top ? nlp1 - k - 1 : k - 1)];
      cf[k] = v;
    }
    for (int k = lane; k <= nlay; k += 32) ftu[k] = ftd[k] = fcu[k] = fcd[k] = 0.0;
    __syncwarp();
    if (mr && lane == 0) {
      rt_grid_mr_factors(cf, nlay, +1, ufac, ufac + L2, ufac + 2 * L2, ufac + 3 * L2, ufac + 4 * L2, ufac + 5 * L2,
                         ufac + 6 * L2);
      rt_grid_mr_factors(cf, nlay, -1, dfac, dfac + L2, dfac + 2 * L2, dfac + 3 * L2, dfac + 4 * L2, dfac + 5 * L2,
                         dfac + 6 * L2);
    }
    __syncwarp();
    const double* crec = sc.col + (size_t)cc * kColRec;
    const R semis = R(crec[32]);
    const R reflct = R(1) - semis;

#pragma unroll 1
    for (int pass = 0; pass < NBANDS / 2; ++pass) {
      const int h = lane >> 4, il = lane & 15;
      const int b = 2 * pass + h;
      const int ng = ng_of(b), g = ns_of(b) + il;
      const bool act = il < ng;
      const R secd = R(crec[b]);
      const R* tcol = sc.tau + (size_t)cc * NGPT * NLP + (size_t)(act ? g : 0) * NLP;
      const R* fcol = sc.frac + (size_t)cc * NGPT * NLP + (size_t)(act ? g : 0) * NLP;
      const R* bl = sc.band + (size_t)cc * 3 * NBANDS * NLP + (size_t)(0 * NBANDS + b) * NLP;
      const R* pl = sc.band + (size_t)cc * 3 * NBANDS * NLP + (size_t)(1 * NBANDS + b) * NLP;
      const R* tc = sc.band + (size_t)cc * 3 * NBANDS * NLP + (size_t)(2 * NBANDS + b) * NLP;
      double* bu = bnd + (size_t)h * 2 * nlp1;
      double* bdn = bu + nlp1;
      if (HLWB && il == 0) bdn[nlay] = 0.0;   // no downward radiation enters at the top

      // ---- down sweep, k = nlay .. 1 ----
      R radtotd = R(0), radclrd = R(0);
      R totradd = R(0), clrradd = R(0), rad = R(0);
#pragma unroll 1
      for (int k = nlay; k >= 1; --k) {
        R rtot = R(0), rclr = R(0);
        if (act) {
          const GasL<R> gl = grid_gas_layer<R>(tcol[k - 1], fcol[k - 1], secd, bl[k - 1], pl[k], pl[k - 1], tab);
          const R clfr = R(cf[k]);
          if (!mr) {   // rtrn (RLM:2629-2665)
            if (cf[k] >= eps) {
              const R odcld = secd * tc[k - 1];
              const R efclrfr = R(1) - (R(1) - exp_neg(odcld)) * clfr;
              R totfac, atrtot, trnt;
              grid_tot_layer<R>(gl.odepth + odcld, tab, totfac, atrtot, trnt);
              const R totsrcd = gl.frac * (gl.blay + gl.dplnkd * totfac) * atrtot;
              radtotd = radtotd * gl.trng * efclrfr + gl.gsd + clfr * (totsrcd - gl.gsd);
            } else {
              radtotd = radtotd * gl.trng + gl.gsd;
            }
          } else {     // rtrnmr (RLM:3205-3254)
            if (dfac[6 * L2 + k] != 0.0) {
              totradd = clfr * radtotd;
              clrradd = radtotd - totradd;
              rad = R(0);
            }
            if (cf[k] >= eps) {
              const R odcld = secd * tc[k - 1];
              R totfac, atrtot, trnt;
              grid_tot_layer<R>(gl.odepth + odcld, tab, totfac, atrtot, trnt);
              const R totsrcd = gl.frac * (gl.blay + gl.dplnkd * totfac) * atrtot;
              totradd = totradd * trnt + clfr * totsrcd;
              clrradd = clrradd * gl.trng + (R(1) - clfr) * gl.gsd;
              radtotd = totradd + clrradd;
              const R radmod = rad * (R(dfac[k - 1]) * gl.trng + R(dfac[2 * L2 + k - 1]) * trnt) -
                               R(dfac[4 * L2 + k - 1]) * gl.gsd + R(dfac[5 * L2 + k - 1]) * totsrcd;
              rad = -radmod + R(dfac[L2 + k - 1]) * (clrradd + radmod) - R(dfac[3 * L2 + k - 1]) * (totradd - radmod);
              totradd = totradd + rad;
              clrradd = clrradd - rad;
            } else {
              radtotd = radtotd * gl.trng + gl.gsd;
            }
          }
          radclrd = radclrd * gl.trng + gl.gsd;
          rtot = radtotd;
          rclr = radclrd;
        }
        const double st = half_sum((double)rtot), sclr = half_sum((double)rclr);
        const double st_hi = __shfl_sync(0xffffffffu, st, 16), sc_hi = __shfl_sync(0xffffffffu, sclr, 16);
        if (lane == 0) {
          ftd[k - 1] += st + st_hi;
          fcd[k - 1] += sclr + sc_hi;
        }
        if (HLWB && il == 0) bdn[k - 1] = st;
      }

      // ---- surface (RLM:2668-2674) and up sweep, k = 1 .. nlay ----
      R radtotu = R(0), radclru = R(0);
      if (act) {
        const R rad0 = semis * fcol[0] * R(crec[16 + b]);
        radtotu = rad0 + reflct * radtotd;
        radclru = rad0 + reflct * radclrd;
      }
      {
        const double st = half_sum((double)radtotu), sclr = half_sum((double)radclru);
        const double st_hi = __shfl_sync(0xffffffffu, st, 16), sc_hi = __shfl_sync(0xffffffffu, sclr, 16);
        if (lane == 0) {
          ftu[0] += st + st_hi;
          fcu[0] += sclr + sc_hi;
        }
        if (HLWB && il == 0) bu[0] = st;
      }
      R totradu = R(0), clrradu = R(0);
#pragma unroll 1
      for (int k = 1; k <= nlay; ++k) {
        R rtot = R(0), rclr = R(0);
        if (act) {
          const GasL<R> gl = grid_gas_layer<R>(tcol[k - 1], fcol[k - 1], secd, bl[k - 1], pl[k], pl[k - 1], tab);
          const R clfr = R(cf[k]);
          if (!mr) {   // rtrn (RLM:2680-2698)
            if (cf[k] >= eps) {
              const R odcld = secd * tc[k - 1];
              const R efclrfr = R(1) - (R(1) - exp_neg(odcld)) * clfr;
              R totfac, atrtot, trnt;
              grid_tot_layer<R>(gl.odepth + odcld, tab, totfac, atrtot, trnt);
              const R totsrcu = gl.frac * (gl.blay + gl.dplnku * totfac) * atrtot;
              radtotu = radtotu * gl.trng * efclrfr + gl.gsu + clfr * (totsrcu - gl.gsu);
            } else {
              radtotu = radtotu * gl.trng + gl.gsu;
            }
          } else {     // rtrnmr (RLM:3270-3305)
            if (ufac[6 * L2 + k] != 0.0) {
              totradu = clfr * radtotu;
              clrradu = radtotu - totradu;
              rad = R(0);
            }
            if (cf[k] >= eps) {
              const R odcld = secd * tc[k - 1];
              R totfac, atrtot, trnt;
              grid_tot_layer<R>(gl.odepth + odcld, tab, totfac, atrtot, trnt);
              const R totu = gl.frac * (gl.blay + gl.dplnku * totfac) * atrtot;
              totradu = totradu * trnt + clfr * totu;
              clrradu = clrradu * gl.trng + (R(1) - clfr) * gl.gsu;
              radtotu = totradu + clrradu;
              const R radmod = rad * (R(ufac[k + 1]) * gl.trng + R(ufac[2 * L2 + k + 1]) * trnt) -
                               R(ufac[4 * L2 + k + 1]) * gl.gsu + R(ufac[5 * L2 + k + 1]) * totu;
              rad = -radmod + R(ufac[L2 + k + 1]) * (clrradu + radmod) - R(ufac[3 * L2 + k + 1]) * (totradu - radmod);
              totradu = totradu + rad;
              clrradu = clrradu - rad;
            } else {
              radtotu = radtotu * gl.trng + gl.gsu;
            }
          }
          radclru = radclru * gl.trng + gl.gsu;
          rtot = radtotu;
          rclr = radclru;
        }
        const double st = half_sum((double)rtot), sclr = half_sum((double)rclr);
        const double st_hi = __shfl_sync(0xffffffffu, st, 16), sc_hi = __shfl_sync(0xffffffffu, sclr, 16);
        if (lane == 0) {
          ftu[k] += st + st_hi;
          fcu[k] += sclr + sc_hi;
        }
        if (HLWB && il == 0) bu[k] = st;
      }
      if constexpr (HLWB) {
        // spectral band heating rates of the pass's two bands (RLM:2772-2780)
        __syncwarp();
        for (int hh = 0; hh < 2; ++hh) {
          const int bb = 2 * pass + hh;
          const double* u = bnd + (size_t)hh * 2 * nlp1;
          const double* dn = u + nlp1;
          for (int k = lane + 1; k <= nlay; k += 32) {
            const int r = top ? nlp1 - k - 1 : k - 1;
            const double rfdelp = cs.heatfac / B.in[F_DELPIN][i + ld * r];
            const double fnb = (u[k - 1] - dn[k - 1]) * flxfac, fna = (u[k] - dn[k]) * flxfac;
            B.out[O_HLWB][i + ld * ((size_t)r + (size_t)nlay * bb)] = (fnb - fna) * rfdelp;
          }
        }
        __syncwarp();
      }
    }
    __syncwarp();

    // ---- fluxes and heating rates (RLM:2735-2770) ----
    for (int lv = lane; lv <= nlay; lv += 32) {
      const double tu = ftu[lv] * flxfac, td = ftd[lv] * flxfac, cu = fcu[lv] * flxfac, cd = fcd[lv] * flxfac;
      if (lv == nlay) {
        B.out[O_TOPFLX][2 * i + 0] = tu;
        B.out[O_TOPFLX][2 * i + 1] = cu;
      }
      if (lv == 0) {
        B.out[O_SFCFLX][4 * i + 0] = tu;
        B.out[O_SFCFLX][4 * i + 1] = cu;
        B.out[O_SFCFLX][4 * i + 2] = td;
        B.out[O_SFCFLX][4 * i + 3] = cd;
      }
      if (f.want_flxprf) {
        const int rl = top ? nlp1 - lv - 1 : lv;
        double* p = B.out[O_FLXPRF] + 4 * (i + ld * (size_t)rl);
        p[0] = tu; p[1] = td; p[2] = cu; p[3] = cd;
      }
    }
    for (int k = lane + 1; k <= nlay; k += 32) {
      const int r = top ? nlp1 - k - 1 : k - 1;
      const double rfdelp = cs.heatfac / B.in[F_DELPIN][i + ld * r];
      // fluxes scaled first, then differenced, as the reference does
      const double fnb = ftu[k - 1] * flxfac - ftd[k - 1] * flxfac, fna = ftu[k] * flxfac - ftd[k] * flxfac;
      B.out[O_HLWC][i + ld * r] = (fnb - fna) * rfdelp;
      if (f.want_hlw0) {
        const double cb = fcu[k - 1] * flxfac - fcd[k - 1] * flxfac, ca = fcu[k] * flxfac - fcd[k] * flxfac;
        B.out[O_HLW0][i + ld * r] = (cb - ca) * rfdelp;
      }
    }
  }
}

}  // namespace lw
