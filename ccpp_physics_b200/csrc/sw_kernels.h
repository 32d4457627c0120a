// sw_kernels.h -- device-side argument records and launchers of the RRTMG-SW
// column kernels (sw_column.cu), shared with the C ABI layer (sw_api.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sw {

constexpr int kSwNg = 112;       // g-points (radsw_param.f NGPTSW)
constexpr int kSwMaxLay = 200;   // layers a column may have on this path

// rrtmg_sw_run arguments, device pointers, caller layout: (i, k) at
// [i + ld*k], (i, k, b) at [i + ld*(k + nlay*b)]
struct SwArgs {
  const double *plyr, *tlyr, *qlyr, *olyr, *co2, *n2o, *ch4, *o2, *delp, *cf;
  const double *aod, *ssa, *asy, *cosz, *alb_nir_dir, *alb_nir_dif, *alb_uvis_dir, *alb_uvis_dif;
  const double *lwp, *rel, *iwp, *rei, *rwp, *rer, *swp, *res, *cod, *cssa, *casy;
  const double *dz, *alpha, *delg;   // layer thickness, alpha, de_lgth: sub-column overlaps 3..5
  const int32_t *icseed, *idxday;
  double *hswc, *topflx, *sfcflx, *cldtau, *hsw0, *hswb, *flxprf, *fdncmp;
  int npts, nlay, ld, top_at_1, inc_minor, iovr, iovr_rand, iovr_maxrand, iswcliq, iswcice, isubcsw, iswmode;
  int gas_only;   // 1: taug/taur/sfluxzen only (stage entry point)
  int seed0;      // global index of column 1 of these arrays (isubcsw = 1 seeds ipsdsw0 + i)
  double s0fac, heatfac;
};

// per-chunk scratch (pl = column within the chunk, k = internal layer)
struct SwScratch {
  double *taug, *taur;               // [pl][k][112]
  double* sflux;                     // [pl][112]
  double *taucw, *ssacw, *asycw;     // [pl][k][14]
  double* cldf;                      // [pl + nc*k], floored cloud fraction (McICA input)
  double* aux;                       // [pl + nc*k], fac_lcf (iovr 3) or alpha (iovr 4, 5); cldfrc (isubcsw 0)
  int32_t* seed;                     // [pl]
  double *zcf1, *zcf0;               // [pl] cloudy / clear column fractions (RSM:1101-1125)
  uint32_t* bits;                    // [pl][112][nw] McICA cloudy flags
  double* lane_store;                // [pl][k][10][32] the transfer's per-lane layer optics and recurrences
  int nw;
  int* bad;                          // set when idxday names a column outside 1..npts
};

__host__ __device__ inline size_t rt_warp_doubles(int nlay, bool hswb) { return (size_t)(hswb ? 32 : 4) * (nlay + 1); }

cudaError_t overlap_aux_launch(int ncols, int nlay, int ld, int iovr, const double* dz, const double* delg,
                               const double* alpha, double* aux, int ldo, cudaStream_t st);
cudaError_t optics_launch(const SwArgs& a, const SwScratch& s, int p0, int nc, const double* T, cudaStream_t st);
cudaError_t rt_prepare(int max_smem);
size_t rt_smem_bytes(int nlay, bool hswb);
cudaError_t rt_launch(const SwArgs& a, const SwScratch& s, int p0, int nc, const double* ET, cudaStream_t st);
// physics blocks in one call: tab[b] = block b's record (device), colpre[b] / dayp[b]
// = columns / daytime points before block b (dayp has nb + 1 entries)
cudaError_t blocks_prepare(const SwArgs* tab, const int* colpre, const int* dayp, int nb, int total_cols,
                           int2* pts, int* bad, cudaStream_t st);
cudaError_t optics_blocks_launch(const SwArgs* tab, const int2* pts, const SwScratch& s, int p0, int nc,
                                 const double* T, cudaStream_t st);
cudaError_t rt_blocks_launch(const SwArgs* tab, const int2* pts, bool grid, bool want_b, const SwScratch& s, int p0,
                             int nc, int nlay, const double* ET, cudaStream_t st);

}  // namespace sw
