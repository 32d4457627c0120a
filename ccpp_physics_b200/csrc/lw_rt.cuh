// lw_rt.cuh -- kernel B of the RRTMG-LW path: McICA radiative transfer.
//
// Replaces rtrnmc (physics/Radiation/RRTMG/radlw_main.F90, RLM:3420-3785)
// and the output mapping of rrtmg_lw_run (RLM:1228-1304).  One warp owns
// one column; lane l owns layers/levels V*l .. V*l+V-1 (surface first).  For
// each g-point the down- and up-sweep recurrences of the two-stream solution
// are affine maps per layer (radiance -> radiance*t + s): each lane composes
// its V layers, a 5-step shuffle scan composes across lanes, and each lane
// replays its layers from the radiance entering its segment, in the
// Fortran's operation order.  Per-level flux sums stay in FP64 registers of
// the lane that owns the level, so no cross-lane reduction over g-points is
// needed.  Inputs come from kernel A (lw_gas.cuh) and the McICA kernel.
#pragma once

#include "lw_gas.cuh"

namespace lw {

template <typename R> __device__ __forceinline__ R shdn(R v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
template <typename R> __device__ __forceinline__ R shup(R v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <typename R> __device__ __forceinline__ R shidx(R v, int s) { return __shfl_sync(0xffffffffu, v, s); }

// V consecutive values starting at a 16-byte aligned address; the scratch
// written by kernel A is read once, so it is loaded evict-first (.cs), and the
// FP32 4-wide form without an L1 allocation.
template <typename R, int V>
__device__ __forceinline__ void load_vec(const R* __restrict__ p, R (&o)[V]) {
  if constexpr (sizeof(R) == 8) {
#pragma unroll
    for (int j = 0; j < V; j += 2) {
      double2 v = __ldcs(reinterpret_cast<const double2*>(p + j));
      o[j] = v.x; o[j + 1] = v.y;
    }
  } else if constexpr (V % 4 == 0) {
    // read once: not allocated in L1, which stays with the table records
#pragma unroll
    for (int j = 0; j < V; j += 4) {
      float4 v;
      asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                   : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p + j));
      o[j] = v.x; o[j + 1] = v.y; o[j + 2] = v.z; o[j + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < V; j += 2) {
      float2 v = __ldcs(reinterpret_cast<const float2*>(p + j));
      o[j] = v.x; o[j + 1] = v.y;
    }
  }
}

// Shared-memory staging of the transfer kernel's inputs.  Each lane copies
// only its own V values of a field (cp.async, 16- or 8-byte pieces) and reads
// only them back, so no lane waits for another.  Per warp, in elements of R:
// kRtDepth stages of {tau, frac} for the g-point pipeline, then one buffer of
// the three band fields {pklay, pklev, taucld}, refilled at each band's last
// g-point; within a field, lane l's values sit at [l V, l V + V).
// Less staging leaves the SM a larger L1 for the table-record gathers: two
// stages (one g-point ahead) instead of three, 48 -> 40 KB per 4-warp CTA,
// took the FP64 transfer kernel from 5.31 to 5.19 ms at 16,384 x 127.
constexpr int kRtDepth = 2;
constexpr int kRtAhead = kRtDepth - 1;   // g-points copied ahead of the one in use
template <typename R>
__host__ __device__ constexpr bool rt_staged() { return sizeof(R) == 8; }
template <int V>
__host__ __device__ constexpr int rt_warp_elems() { return (2 * kRtDepth + 3) * 32 * V; }

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// V consecutive values (16-byte aligned for 16-byte pieces, 8-byte otherwise)
template <typename R, int V>
__device__ __forceinline__ void stage_vec(R* dst, const R* src) {
  constexpr int B = V * (int)sizeof(R);
  if constexpr (B % 16 == 0) {
#pragma unroll
    for (int o = 0; o < B; o += 16)
      cp_async16(reinterpret_cast<char*>(dst) + o, reinterpret_cast<const char*>(src) + o);
  } else {
    static_assert(B == 8, "8- or 16k-byte lane vectors");
    cp_async8(dst, src);
  }
}

template <typename R, int V>
__device__ __forceinline__ void lds_vec(const R* p, R (&o)[V]) {
  if constexpr (sizeof(R) == 8) {
#pragma unroll
    for (int j = 0; j < V; j += 2) {
      const double2 v = *reinterpret_cast<const double2*>(p + j);
      o[j] = v.x; o[j + 1] = v.y;
    }
  } else if constexpr (V % 4 == 0) {
#pragma unroll
    for (int j = 0; j < V; j += 4) {
      const float4 v = *reinterpret_cast<const float4*>(p + j);
      o[j] = v.x; o[j + 1] = v.y; o[j + 2] = v.z; o[j + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < V; j += 2) {
      const float2 v = *reinterpret_cast<const float2*>(p + j);
      o[j] = v.x; o[j + 1] = v.y;
    }
  }
}

// Table-index quotient x / (bpade + x) and cloud transmittance exp(-x).  The
// FP64 path keeps the exact operations (its table indices must match the
// reference's); the FP32 path, already within its error bound of the FP64
// result, uses the fast hardware approximations.
__device__ __forceinline__ double tbl_quot(double x) { return x / (kBpade + x); }
__device__ __forceinline__ float tbl_quot(float x) { return __fdividef(x, float(kBpade) + x); }
__device__ __forceinline__ double exp_neg(double x) { return exp(-x); }
__device__ __forceinline__ float exp_neg(float x) { return __expf(-x); }

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
    R tblind = tbl_quot(odepth);
    int itgas = min(NTBL, max(0, (int)(R(kTblint) * tblind + R(0.5))));
    if (!LW_OK(itgas >= 0 && itgas <= NTBL, 22, itgas)) itgas = 0;
    tbl_rec(tab.trec, itgas, trng, gasfac, odepth);
    atrgas = one - trng;
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
    o.ef = one - (one - exp_neg(odcld)) * one;   // clfm = 1 for a McICA cloudy sub-column
    R odtot = odepth + odcld;
    R totfac, atrtot;
    if (odtot < R(0.06)) {
      totfac = R(kRec6) * odtot;
      atrtot = odtot - R(0.5) * odtot * odtot;
    } else {
      R tblind = tbl_quot(odtot);
      int ittot = min(NTBL, max(0, (int)(R(kTblint) * tblind + R(0.5))));
      R ex, ta;
      tbl_rec(tab.trec, ittot, ex, totfac, ta);
      atrtot = one - ex;
    }
    R bbdtot = frac * (blay + dplnkd * totfac);
    R bbutot = frac * (blay + dplnku * totfac);
    o.tsd = bbdtot * atrtot;
    o.tsu = bbutot * atrtot;
  }
}

extern __shared__ __align__(16) unsigned char lw_rt_smem[];

template <typename R, int V, bool HLWB>
__global__ void __launch_bounds__(128, LW_RT_MINB)
lw_rt_kernel(const Block* __restrict__ blocks, int nblocks, const Block b0, int ncols, Flags f, Consts cs,
             Tables<R> tab, Scratch<R> sc, const uint32_t* __restrict__ bits_g) {
  constexpr int NLP = 32 * V;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int nlay = f.nlay, nlp1 = nlay + 1;
  const int nw = (nlay + 31) >> 5;
  const int k0 = V * lane;
  const double flxfac = 0.5 * cs.fluxfac;   // wtdiff * fluxfac

  for (int cc = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; cc < ncols; cc += nwarps) {
    const int c = sc.c0 + cc;
    const Block& B = (nblocks == 1) ? b0 : blocks[find_block(blocks, nblocks, c)];
    const int i = c - B.col0;
    const size_t ld = (size_t)B.ld;
    const bool top = f.top_at_1 != 0;
    if (!LW_OK(cc < sc.cap && c < sc.ntot && i >= 0 && i < B.npts, 21, cc)) continue;
    const double* crec = sc.col + (size_t)cc * kColRec;
    const bool mc = crec[33] != 0.0 && f.isubclw > 0;
    const R semis = R(crec[32]);
    const R reflct = R(1) - semis;
    const R* tcol = sc.tau + (size_t)cc * NGPT * NLP + k0;
    const R* fcol = sc.frac + (size_t)cc * NGPT * NLP + k0;
    const R* bcol = sc.band + (size_t)cc * 3 * NBANDS * NLP + k0;
    const uint32_t* cbw = bits_g + (size_t)c * NGPT * nw + (k0 >> 5);
    const uint32_t lmask = (k0 >= nlay) ? 0u : (nlay - k0 >= V ? (1u << V) - 1u : (1u << (nlay - k0)) - 1u);
    // FP64: inputs staged through shared memory (the register budget at 4
    // CTAs/SM cannot hold them); FP32: straight to registers.  This lane's
    // slots: g-point stage s field q at sl + (2 s + q) 32 V, band buffer p
    // field q at sl + (2 kRtDepth + 3 p + q) 32 V.
    constexpr bool kStage = rt_staged<R>();
    R* const sl = reinterpret_cast<R*>(lw_rt_smem) + (threadIdx.x >> 5) * rt_warp_elems<V>() + k0;

    double acc_tu[V], acc_td[V], acc_cu[V], acc_cd[V];
    double bnd_tu[HLWB ? V : 1], bnd_td[HLWB ? V : 1];
#pragma unroll
    for (int j = 0; j < V; ++j) {
      acc_tu[j] = acc_td[j] = acc_cu[j] = acc_cd[j] = 0.0;
      if constexpr (HLWB) bnd_tu[j] = bnd_td[j] = 0.0;
    }

    // copy groups (staged), kRtAhead = kRtDepth - 1 g-points ahead: group i
    // (i < kRtAhead) = g-point i, group 0 also band 0's fields; the iteration
    // of g-point g commits group g + kRtAhead (that g-point), then waits for
    // group g; a band's last g-point adds a group with the next band's fields
    if constexpr (kStage) {
#pragma unroll
      for (int q = 0; q < 3; ++q) stage_vec<R, V>(sl + (2 * kRtDepth + q) * 32 * V, bcol + (size_t)q * NBANDS * NLP);
#pragma unroll
      for (int g0 = 0; g0 < kRtAhead; ++g0) {
        stage_vec<R, V>(sl + (2 * g0) * 32 * V, tcol + (size_t)g0 * NLP);
        stage_vec<R, V>(sl + (2 * g0 + 1) * 32 * V, fcol + (size_t)g0 * NLP);
        cp_async_commit();
      }
    }
    uint32_t nbits = (mc && lmask && LW_OK((k0 >> 5) < nw, 27, k0)) ? __ldg(cbw) : 0u;

#pragma unroll 1
    for (int b = 0; b < NBANDS; ++b) {
      const R secd = R(crec[b]);
      const R pk0 = R(crec[16 + b]);          // pklay(b, 0): surface (RLM:2251-2262)
      const int ns = ns_of(b), ng = ng_of(b);
      R* const bsl = sl + (2 * kRtDepth) * 32 * V;
      // register path: the band's fields, and the band's first g-point (each
      // iteration prefetches the next)
      R rblay[kStage ? 1 : V], rplev[kStage ? 1 : V], rtcld[kStage ? 1 : V], ntau[kStage ? 1 : V],
          nfrac[kStage ? 1 : V];
      if constexpr (!kStage) {
        load_vec<R, V>(bcol + (0 * NBANDS + b) * NLP, rblay);
        load_vec<R, V>(bcol + (1 * NBANDS + b) * NLP, rplev);
        load_vec<R, V>(bcol + (2 * NBANDS + b) * NLP, rtcld);
        load_vec<R, V>(tcol + (size_t)ns * NLP, ntau);
        load_vec<R, V>(fcol + (size_t)ns * NLP, nfrac);
      }
#pragma unroll 1
      for (int g = ns; g < ns + ng; ++g) {
        // band terms of the lane's layers: pklay(b,k+1), pklev(b,k..k+1), taucld(b,k+1)
        R tau[V], frac[V], blay[V], plev[V], tcld[V];
        if constexpr (kStage) {
          if (g + kRtAhead < NGPT) {
            const int s2 = (g + kRtAhead) % kRtDepth;
            stage_vec<R, V>(sl + (2 * s2) * 32 * V, tcol + (size_t)(g + kRtAhead) * NLP);
            stage_vec<R, V>(sl + (2 * s2 + 1) * 32 * V, fcol + (size_t)(g + kRtAhead) * NLP);
          }
          cp_async_commit();
          cp_async_wait<kRtAhead>();
          const int s0 = g % kRtDepth;
          lds_vec<R, V>(sl + (2 * s0) * 32 * V, tau);
          lds_vec<R, V>(sl + (2 * s0 + 1) * 32 * V, frac);
          lds_vec<R, V>(bsl, blay);
          lds_vec<R, V>(bsl + 32 * V, plev);
          lds_vec<R, V>(bsl + 2 * 32 * V, tcld);
        } else {
#pragma unroll
          for (int j = 0; j < V; ++j) {
            tau[j] = ntau[j]; frac[j] = nfrac[j];
            blay[j] = rblay[j]; plev[j] = rplev[j]; tcld[j] = rtcld[j];
          }
          if (g + 1 < ns + ng) {
            load_vec<R, V>(tcol + (size_t)(g + 1) * NLP, ntau);
            load_vec<R, V>(fcol + (size_t)(g + 1) * NLP, nfrac);
          }
        }
        const R plev_top = shdn(plev[0], 1);    // pklev of the level above the segment
        const uint32_t cbits = (nbits >> (k0 & 31)) & lmask;
        if (g + 1 < NGPT && mc && lmask) nbits = __ldg(cbw + (size_t)(g + 1) * nw);
        LayRT<R> rt[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
          if (k0 + j < nlay) {
            const R pu = (j + 1 < V) ? plev[j + 1] : plev_top;
            layer_rt<R>(tau[j], frac[j], secd, blay[j], pu, plev[j], (cbits >> j) & 1u, tcld[j], tab, rt[j]);
          } else {
            rt[j].tr = R(1); rt[j].gsd = R(0); rt[j].gsu = R(0);
          }
        }
        // single band buffer: at a band's last g-point, once this lane's band
        // fields have been used, its slots take the next band's fields (a group
        // of its own, complete by the next iteration's wait)
        if constexpr (kStage) {
          static_assert(kRtAhead == 1, "the band buffer's group must complete one iteration later");
          if (g == ns + ng - 1 && b + 1 < NBANDS) {
#pragma unroll
            for (int q = 0; q < 3; ++q) stage_vec<R, V>(bsl + q * 32 * V, bcol + (size_t)(q * NBANDS + b + 1) * NLP);
            cp_async_commit();
          }
        }
        const bool any_cloud = __any_sync(0xffffffffu, cbits != 0);

        // ---- both sweeps' layer maps (down RLM:3598-3673, up RLM:3700-3730):
        // each lane composes its V layers' affine maps.  The up maps do not
        // depend on the down sweep (only the up replay needs the surface
        // radiance), so the down suffix scan and the up prefix scan run
        // interleaved, each in its own operation order. ----
        R Ac = R(1), Bc = R(0), At = R(1), Bt = R(0);      // down
        R Uc = R(1), Wc = R(0), Ut = R(1), Wt = R(0);      // up
#pragma unroll
        for (int j = V - 1; j >= 0; --j) {
          Bc = rt[j].tr * Bc + rt[j].gsd; Ac = rt[j].tr * Ac;
          if (any_cloud) {
            if ((cbits >> j) & 1u) {
              const R a = rt[j].tr * rt[j].ef;
              Bt = a * Bt + (rt[j].gsd + (rt[j].tsd - rt[j].gsd)); At = a * At;
            } else {
              Bt = rt[j].tr * Bt + rt[j].gsd; At = rt[j].tr * At;
            }
          }
        }
#pragma unroll
        for (int j = 0; j < V; ++j) {
          Wc = rt[j].tr * Wc + rt[j].gsu; Uc = rt[j].tr * Uc;
          if (any_cloud) {
            if ((cbits >> j) & 1u) {
              const R a = rt[j].tr * rt[j].ef;
              Wt = a * Wt + (rt[j].gsu + (rt[j].tsu - rt[j].gsu)); Ut = a * Ut;
            } else {
              Wt = rt[j].tr * Wt + rt[j].gsu; Ut = rt[j].tr * Ut;
            }
          }
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const R ac = shdn(Ac, d), bc = shdn(Bc, d), uc = shup(Uc, d), wc = shup(Wc, d);
          R at = R(0), bt = R(0), ut = R(0), wt = R(0);
          if (any_cloud) { at = shdn(At, d); bt = shdn(Bt, d); ut = shup(Ut, d); wt = shup(Wt, d); }
          if (lane + d < 32) {
            Bc = Ac * bc + Bc; Ac = Ac * ac;
            if (any_cloud) { Bt = At * bt + Bt; At = At * at; }
          }
          if (lane >= d) {
            Wc = Uc * wc + Wc; Uc = Uc * uc;
            if (any_cloud) { Wt = Ut * wt + Wt; Ut = Ut * ut; }
          }
        }
        // the up maps of the layers below each lane's segment (used once the
        // surface radiance is known)
        const R pac = shup(Uc, 1), pbc = shup(Wc, 1);
        R pat = R(0), pbt = R(0);
        if (any_cloud) { pat = shup(Ut, 1); pbt = shup(Wt, 1); }
        // ---- down replay ----
        R xc = shdn(Bc, 1), xt = any_cloud ? shdn(Bt, 1) : R(0);
        if (lane == 31) { xc = R(0); xt = R(0); }
#pragma unroll
        for (int j = V - 1; j >= 0; --j) {
          xc = xc * rt[j].tr + rt[j].gsd;
          if (any_cloud) {
            if ((cbits >> j) & 1u) xt = xt * rt[j].tr * rt[j].ef + rt[j].gsd + R(1) * (rt[j].tsd - rt[j].gsd);
            else xt = xt * rt[j].tr + rt[j].gsd;
          } else {
            xt = xc;
          }
          acc_cd[j] += (double)xc;
          acc_td[j] += (double)xt;
          if constexpr (HLWB) bnd_td[j] += (double)xt;
        }
        // ---- surface emission and reflection (RLM:3682-3691) ----
        const R rad0 = semis * shidx(frac[0], 0) * pk0;
        const R r0c = rad0 + reflct * shidx(xc, 0);
        const R r0t = rad0 + reflct * shidx(xt, 0);
        // ---- up replay from the surface ----
        xc = (lane == 0) ? r0c : pac * r0c + pbc;
        if (any_cloud) xt = (lane == 0) ? r0t : pat * r0t + pbt;
#pragma unroll
        for (int j = 0; j < V; ++j) {
          acc_cu[j] += (double)xc;
          const double ut = any_cloud ? (double)xt : (double)xc;
          acc_tu[j] += ut;
          if constexpr (HLWB) bnd_tu[j] += ut;
          xc = xc * rt[j].tr + rt[j].gsu;
          if (any_cloud) {
            if ((cbits >> j) & 1u) xt = xt * rt[j].tr * rt[j].ef + rt[j].gsu + R(1) * (rt[j].tsu - rt[j].gsu);
            else xt = xt * rt[j].tr + rt[j].gsu;
          }
        }
      }
      if constexpr (HLWB) {
        // spectral band heating rate (RLM:3772-3780)
        double fn[V];
#pragma unroll
        for (int j = 0; j < V; ++j) { fn[j] = (bnd_tu[j] - bnd_td[j]) * flxfac; bnd_tu[j] = bnd_td[j] = 0.0; }
        const double fn_top = __shfl_down_sync(0xffffffffu, fn[0], 1);
#pragma unroll
        for (int j = 0; j < V; ++j) {
          const int k = k0 + j;
          if (k < nlay && LW_OK(k >= 0, 23, k)) {
            const int r = top ? nlp1 - (k + 1) - 1 : k;
            const double above = (j + 1 < V) ? fn[j + 1] : fn_top;
            const double rfdelp = cs.heatfac / B.in[F_DELPIN][i + ld * r];
            B.out[O_HLWB][i + ld * ((size_t)r + (size_t)nlay * b)] = (fn[j] - above) * rfdelp;
          }
        }
      }
    }

    // ------------------------------ fluxes and heating rates --------------
    double fnet[V], fnetc[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int lv = k0 + j;
      const double tu = acc_tu[j] * flxfac, td = acc_td[j] * flxfac;
      const double cu = acc_cu[j] * flxfac, cd = acc_cd[j] * flxfac;
      fnet[j] = tu - td;
      fnetc[j] = cu - cd;
      if (lv <= nlay && LW_OK(lv >= 0, 25, lv)) {
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
    }
    const double fn_top = __shfl_down_sync(0xffffffffu, fnet[0], 1);
    const double fc_top = __shfl_down_sync(0xffffffffu, fnetc[0], 1);
#pragma unroll
    for (int j = 0; j < V; ++j) {   // RLM:3754-3770
      const int k = k0 + j;
      if (k < nlay && LW_OK(k >= 0 && (top ? nlp1 - (k + 1) - 1 : k) >= 0, 24, k)) {
        const int r = top ? nlp1 - (k + 1) - 1 : k;
        const double rfdelp = cs.heatfac / B.in[F_DELPIN][i + ld * r];
        const double up = (j + 1 < V) ? fnet[j + 1] : fn_top;
        const double upc = (j + 1 < V) ? fnetc[j + 1] : fc_top;
        B.out[O_HLWC][i + ld * r] = (fnet[j] - up) * rfdelp;
        if (f.want_hlw0) B.out[O_HLW0][i + ld * r] = (fnetc[j] - upc) * rfdelp;
      }
    }
  }
}

}  // namespace lw
