// lw_common.cuh -- shared definitions of the B200 RRTMG-LW kernels.
//
// Band layout and constants follow physics/Radiation/RRTMG/radlw_param.f
// (:103-142) and radlw_main.F90 (RLM:309-354); the coefficient tables are
// the DATA of radlw_datatb.f, extracted into rrtmg_lw_tables.bin whose
// offsets are in rrtmg_lw_table_layout.h (namespace lwtab).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../data/rrtmg_lw_table_layout.h"

namespace lw {

constexpr int NBANDS = 16;
constexpr int NGPT = 140;
constexpr int kSwNgpt = 112;   // shortwave g-points (radsw_param.f NGPTSW)
constexpr int NTBL = 10000;

// g-points per band and first g-point of each band (radlw_param.f:111-120)
__host__ __device__ constexpr int ng_of(int b) {
  return b == 0 ? 10 : b == 1 ? 12 : b == 2 ? 16 : b == 3 ? 14 : b == 4 ? 16 : b == 5 ? 8
       : b == 6 ? 12 : b == 7 ? 8 : b == 8 ? 12 : b == 9 ? 6 : b == 10 ? 8 : b == 11 ? 8
       : b == 12 ? 4 : 2;
}
__host__ __device__ constexpr int ns_of(int b) {   // first g-point of band b (flat, no recursion)
  return b == 0 ? 0 : b == 1 ? 10 : b == 2 ? 22 : b == 3 ? 38 : b == 4 ? 52 : b == 5 ? 68 : b == 6 ? 76
       : b == 7 ? 88 : b == 8 ? 96 : b == 9 ? 108 : b == 10 ? 114 : b == 11 ? 122 : b == 12 ? 130
       : b == 13 ? 134 : b == 14 ? 136 : 138;
}
static_assert(ns_of(15) + ng_of(15) == NGPT, "band layout");
// reference-atmosphere counts per band (RLM:326-327); nspb(16) = 0 is kept
__host__ __device__ constexpr int nspa_of(int b) {
  return (b == 2 || b == 3 || b == 4 || b == 6 || b == 8 || b == 11 || b == 12 || b == 14 || b == 15) ? 9 : 1;
}
__host__ __device__ constexpr int nspb_of(int b) {
  return (b == 2 || b == 3 || b == 4) ? 5 : (b == 5 || b == 11 || b == 12 || b == 14 || b == 15) ? 0 : 1;
}

// Run-time constants shared by every column of a call.
struct Consts {
  double fluxfac, heatfac;
};

// Coefficient tables in device memory, in the arithmetic precision R.
// The rlwinit tables (RLM:1474-1501) are interleaved: record i is
// {exp_tbl(i), tfn_tbl(i), tau_tbl(i), 0} at trec[4 i], so one lookup of the
// transfer touches one 32-byte (FP64) or 16-byte (FP32) record.
template <typename R>
struct Tables {
  const R* kt;       // every radlw_datatb.f array (offsets lwtab::*)
  const R* trec;     // (NTBL+1) records of 4
};

// exp_tbl(it), tfn_tbl(it), tau_tbl(it) of one record.
__device__ __forceinline__ void tbl_rec(const double* trec, int it, double& ex, double& tf, double& ta) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(trec + 4 * it));
  ex = v.x;
  tf = v.y;
  ta = __ldg(trec + 4 * it + 2);
}
__device__ __forceinline__ void tbl_rec(const float* trec, int it, float& ex, float& tf, float& ta) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(trec + 4 * it));
  ex = v.x;
  tf = v.y;
  ta = v.z;
}

// Device-side view of one physics block (the arrays of one rrtmg_lw_run call).
enum InField {
  F_PLYR, F_PLVL, F_TLYR, F_TLVL, F_QLYR, F_OLYR, F_CO2, F_N2O, F_CH4, F_O2, F_CO, F_CFC11,
  F_CFC12, F_CFC22, F_CCL4, F_AERAOD, F_AERSSA, F_SFEMIS, F_SFGTMP, F_DZLYR, F_DELPIN,
  F_DELGTH, F_ALPHA, F_CLDCF, F_LWP, F_RELIQ, F_IWP, F_REICE, F_RWP, F_RERAIN, F_SWP,
  F_RESNOW, F_CLDOD, N_IN
};
enum OutField { O_HLWC, O_TOPFLX, O_SFCFLX, O_CLDTAU, O_HLW0, O_HLWB, O_FLXPRF, N_OUT };

struct Block {
  const double* in[N_IN];
  const int32_t* icseed;
  double* out[N_OUT];
  int npts;   // columns in this block
  int ld;     // leading dimension of its (npts, ...) arrays
  int col0;   // global index of its first column (prefix sum)
  int seed0;  // index of its first column within the caller's block (isubclw=1 seeds 140+i, RLM:765-768)
};

// Flags common to every block of a launch.
struct Flags {
  int nlay, top_at_1, inc_minor_gas, iovr, iovr_dcorr, iovr_exp, iovr_exprand;
  int ilwcliq, ilwcice, isubclw;
  int want_hlw0, want_hlwb, want_flxprf;
  int gas_only;        // 1: write taug/fracs only (training data / stage tests)
  int surrogate = 0;   // 1: the learned gas optics wrote tau/frac; recompute only out-of-envelope layers
  int pad_ = 0;
  const float* sg_norm = nullptr;        // normalisation + envelope of the network (lw_features.cuh)
  unsigned int* sg_fallback = nullptr;   // count of layers that fell back to taumol
};

// Device scratch of the gas-optics -> transfer hand-off (NLP = 32 V layers).
template <typename R>
struct Scratch {
  R* tau;        // [nc][NGPT][NLP]
  R* frac;       // [nc][NGPT][NLP]
  R* band;       // [nc][3][NBANDS][NLP]
  double* col;   // [nc][kColRec]
  int c0;        // first global column of the chunk
  int cap;       // columns the scratch holds
  int ntot;      // columns of the whole call
};

// Launch shape of the column kernels (host side; chosen by the autotuner
// or defaulted).  rt_warps: columns (one warp each) per CTA of the transfer
// kernel; chunk: columns per gas-optics -> transfer hand-off (0 = as many as
// the scratch budget holds); gas_per_sm: resident gas CTAs per SM to launch
// (0 = the occupancy limit).
struct Shape {
  int rt_warps = 4;
  int gas_per_sm = 0;
  long chunk = 0;
};

// Locate the block of a global column (blocks sorted by col0).
__device__ __forceinline__ int find_block(const Block* blocks, int nblocks, int col) {
  int lo = 0, hi = nblocks - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (blocks[mid].col0 <= col) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Barrier of a group of threads: the whole CTA (gas_column in lw_gas_kernel
// and the fallback kernel of the learned-gas-optics path), or a named
// barrier over `n` threads of a CTA that holds several groups (that path's
// network and transfer kernels).
struct CtaSync {
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  __device__ __forceinline__ int count(bool p) const { return __syncthreads_count(p); }
  __device__ __forceinline__ int any(bool p) const { return __syncthreads_or(p); }
};
struct GroupSync {
  int id, n;   // named barrier id (1..15) and thread count (a multiple of 32)
  __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
  __device__ __forceinline__ int count(bool p) const {
    int r;
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.popc.u32 %0, %2, %3, q;\n\t}"
                 : "=r"(r) : "r"((unsigned)p), "r"(id), "r"(n) : "memory");
    return r;
  }
  __device__ __forceinline__ int any(bool p) const { return count(p) != 0; }
};


// Debug builds (-DLW_DEBUG_CHECKS=1) bounds-check every table, scratch,
// input and output access of the column kernels: the first violation is
// recorded in lw_dbg_err {site, index, block, thread} and the access is
// skipped.  Release builds compile the checks out.
#ifndef LW_DEBUG_CHECKS
#define LW_DEBUG_CHECKS 0
#endif
#if LW_DEBUG_CHECKS
static __device__ unsigned int lw_dbg_err[8];
__device__ __forceinline__ bool lw_ok(bool cond, unsigned site, long long idx) {
  if (cond) return true;
  if (atomicCAS(&lw_dbg_err[0], 0u, site) == 0u) {
    lw_dbg_err[1] = (unsigned)(idx & 0xffffffffll);
    lw_dbg_err[2] = (unsigned)((unsigned long long)idx >> 32);
    lw_dbg_err[3] = blockIdx.x;
    lw_dbg_err[4] = threadIdx.x;
    __threadfence();
  }
  return false;
}
#define LW_OK(cond, site, idx) lw_ok((cond), (site), (long long)(idx))
#else
#define LW_OK(cond, site, idx) true
#endif

}  // namespace lw
