// lw_prep.cu -- the steps either side of rrtmg_lw_run, on the GPU
// (include/rrtmg_lw_gpu.h, "Steps either side of rrtmg_lw_run"):
//
// rrtmg_lw_gpu_seeds          <- GFS_rad_time_vary_timestep_init, seed part
//                                (physics/Interstitials/UFS_SCM_NEPTUNE/
//                                GFS_rad_time_vary.fv3.F90:59-84)
// rrtmg_lw_gpu_overlap_params <- radiation_clouds.f:837-856 with
//                                cmp_dcorr_lgth_hogan / _oreopoulos and
//                                get_alpha_exper (physics/Radiation/
//                                radiation_cloud_overlap.F90:28-145)
// rrtmg_lw_gpu_post           <- rrtmg_lw_post_run (physics/Radiation/RRTMG/
//                                rrtmg_lw_post.F90:13-77)
// rrtmg_sw_gpu_pre            <- rad_sw_pre_run (physics/Radiation/RRTMG/
//                                rad_sw_pre.F90:14-51)
// rrtmg_sw_gpu_post           <- rrtmg_sw_post_run (physics/Radiation/RRTMG/
//                                rrtmg_sw_post.F90:13-129)
//
// The seed stream is one Mersenne-twister stream walked by one CTA
// (lw_mcica.cu) into a device buffer of raw words; one thread per column then
// tempers and converts the two words it uses.  The overlap parameters run one thread per
// column over its layers (coalesced across columns); the post steps one
// thread per (column, level) element.  This file is compiled without FMA
// contraction, so every product and sum rounds as the Fortran's does.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rrtmg_lw_gpu.h"
#include "../../include/rrtmg_sw_gpu.h"
#include "lw_launch.h"

namespace {

// ---------------------------------------------------------------- kernels --

// lrseeds: seeds supplied by the host model (GFS_rad_time_vary.fv3.F90:66-70)
__global__ void seed_copy_kernel(const int32_t* __restrict__ rseeds, int n, int ld, int32_t* icsdsw,
                                 int32_t* icsdlw) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= n) return;
  icsdsw[ix] = rseeds[ix];
  icsdlw[ix] = rseeds[ix + ld];
}

enum DcorrKind { kDcorrNone = 0, kDcorrHogan, kDcorrOreopoulos, kDcorrCon };

struct OverlapK {
  int npts, nlay, ld;
  int dcorr;        // DcorrKind to evaluate (kDcorrNone: de_lgth untouched)
  int alpha;        // 1: get_alpha_exper
  int exprand;      // 1: the exponential-random revision of alpha
  int zero;         // 1: de_lgth = 0, alpha = 0 (radiation_clouds.f:853-855)
  int yearlen;
  double julian, dcorr_con, con_pi;
  const double *xlat, *latdeg, *dzlay, *cld_frac;
  double *de_lgth, *alpha_out;
};

// Decorrelation length of column i by the selected routine, or the stored one.
__device__ __forceinline__ double dcorr_of(const OverlapK& a, int i) {
  if (a.dcorr == kDcorrHogan) {
    // max(min_dcorr, 2.78 - 4.6 |lat / pi|), eq. 13 (radiation_cloud_overlap.F90:44-47)
    return fmax(0.6, 2.78 - 4.6 * fabs(a.xlat[i] / a.con_pi));
  }
  if (a.dcorr == kDcorrOreopoulos) {
    // eqs. 10-11 with am1, am2, am4, amr of Table 1 (radiation_cloud_overlap.F90:74-90)
    const double am1 = 1.4315, am2 = 2.1219, am4 = -25.584, amr = 7.0;
    const double am3 = (a.julian > 181.0) ? -(4.0 * amr * (a.julian - 272.0) / (double)a.yearlen)
                                          : 4.0 * amr * (a.julian - 91.0) / (double)a.yearlen;
    const double d = a.latdeg[i] - am3;
    return am1 + am2 * exp(-(d * d) / (am4 * am4));
  }
  if (a.dcorr == kDcorrCon) return a.dcorr_con;
  return a.de_lgth[i];
}

// One thread per column (coalesced across the warp for every layer): the
// column's decorrelation length, then alpha of its layers
// (get_alpha_exper, radiation_cloud_overlap.F90:122-141) kOverlapChunk at a
// time, the chunk's loads issued together ahead of its stores; the
// exponential-random rule keeps the layer below's cloud fraction in a
// register.
constexpr int kOverlapChunk = 8;

__global__ void overlap_kernel(OverlapK a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npts) return;
  const size_t ld = (size_t)a.ld;
  if (a.zero) {   // radiation_clouds.f:853-855
    a.de_lgth[i] = 0.0;
    for (int k = 0; k < a.nlay; ++k) a.alpha_out[i + ld * k] = 0.0;
    return;
  }
  const double dl = dcorr_of(a, i);
  if (a.dcorr != kDcorrNone) a.de_lgth[i] = dl;
  if (!a.alpha || a.nlay == 0) return;
  const double* __restrict__ dzp = a.dzlay + i;
  const double* __restrict__ cfp = a.cld_frac + i;
  double* __restrict__ out = a.alpha_out + i;
  out[0] = 0.0;
  double cf_prev = a.exprand ? cfp[0] : 0.0;
  for (int k0 = 1; k0 < a.nlay; k0 += kOverlapChunk) {
    double dz[kOverlapChunk], cf[kOverlapChunk];
#pragma unroll
    for (int u = 0; u < kOverlapChunk; ++u) {
      const int k = k0 + u;
      dz[u] = 1.0;
      cf[u] = 1.0;
      if (k < a.nlay) {
        dz[u] = __ldcs(dzp + ld * k);
        if (a.exprand) cf[u] = __ldcs(cfp + ld * k);
      }
    }
#pragma unroll
    for (int u = 0; u < kOverlapChunk; ++u) {
      const int k = k0 + u;
      if (k >= a.nlay) break;
      double al = exp(-dz[u] / dl);
      if (a.exprand) {
        if (cf[u] == 0.0 && cf_prev > 0.0) al = 0.0;
        cf_prev = cf[u];
      }
      __stcs(out + ld * k, al);
    }
  }
}

struct PostK {
  int im, levs, lm, kd, lwhtr;
  const double *tsfa, *htlwc, *htlw0, *sfcflw;
  double *tsflw, *sfcdlw, *htrlw, *lwhc;
};

// Level mapping of the post steps (rrtmg_lw_post.F90:48-70,
// rrtmg_sw_post.F90:54-77): dst(:,k) = src(:,k+kd) for k = 1..lm, and
// dst(:,lm) for k = lm+1..levs; dst0 from src0 likewise when `both`.  Levels
// 1..lm are one contiguous block of the source, copied with four loads in
// flight per thread.
__device__ void map_levels(const double* src, const double* src0, double* dst, double* dst0, bool both,
                           size_t im, int lm, int levs, int kd, size_t t0, size_t stride) {
  const size_t nb = im * lm;
  const double* s1 = src + im * kd;
  const double* s2 = src0 + im * kd;
  for (size_t e = t0; e < nb; e += 4 * stride) {
    double v[4], w[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const size_t q = e + u * stride;
      if (q < nb) {
        v[u] = __ldcs(s1 + q);
        if (both) w[u] = __ldcs(s2 + q);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const size_t q = e + u * stride;
      if (q < nb) {
        __stcs(dst + q, v[u]);
        if (both) __stcs(dst0 + q, w[u]);
      }
    }
  }
  if (lm >= 1) {
    for (int k = lm; k < levs; ++k) {
      for (size_t i = t0; i < im; i += stride) {
        dst[im * k + i] = s1[im * (lm - 1) + i];
        if (both) dst0[im * k + i] = s2[im * (lm - 1) + i];
      }
    }
  }
}

// rrtmg_lw_post_run (rrtmg_lw_post.F90:42-75): the heating-rate levels, then
// the per-column fields.
__global__ void post_kernel(PostK a) {
  const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t im = (size_t)a.im;
  map_levels(a.htlwc, a.htlw0, a.htrlw, a.lwhc, a.lwhtr != 0, im, a.lm, a.levs, a.kd, t0, stride);
  for (size_t i = t0; i < im; i += stride) {
    a.tsflw[i] = a.tsfa[i];
    a.sfcdlw[i] = a.sfcflw[4 * i + 2];
  }
}

// rad_sw_pre_run (rad_sw_pre.F90:36-49): the daytime columns in increasing
// order, as an ordered compaction in two passes over tiles of kPreTile
// columns.  Pass 1 counts each tile's daytime columns; pass 2 gives each tile
// its offset (the sum of the counts before it: a block-wide sum over at most
// a few thousand tiles) and writes its columns at their ballot ranks.
constexpr int kPreTile = 1024;
constexpr double kCoszenMin = 0.0001;   // rad_sw_pre.F90:41

__global__ void __launch_bounds__(kPreTile) sw_pre_count_kernel(const double* __restrict__ coszen, int im,
                                                                int* __restrict__ counts) {
  const long long i = (long long)blockIdx.x * kPreTile + threadIdx.x;
  const int c = __syncthreads_count(i < im && coszen[i] >= kCoszenMin);
  if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// idxday(1:nday) = daytime columns; idxday(nday+1:im) = 0 (rad_sw_pre.F90:39);
// nday into *nday_out by tile 0.
__global__ void __launch_bounds__(kPreTile) sw_pre_scatter_kernel(const double* __restrict__ coszen, int im,
                                                                  const int* __restrict__ counts, int ntiles,
                                                                  int32_t* __restrict__ idxday,
                                                                  int32_t* __restrict__ nday_out) {
  __shared__ int red[2][32];
  __shared__ int wbase[32];
  __shared__ int s_nday;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int before = 0, all = 0;
  for (int j = t; j < ntiles; j += kPreTile) {
    const int c = counts[j];
    all += c;
    if (j < (int)blockIdx.x) before += c;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    before += __shfl_xor_sync(0xffffffffu, before, o);
    all += __shfl_xor_sync(0xffffffffu, all, o);
  }
  if (lane == 0) {
    red[0][w] = before;
    red[1][w] = all;
  }
  const long long i = (long long)blockIdx.x * kPreTile + t;
  const bool day = i < im && coszen[i] >= kCoszenMin;
  const unsigned m = __ballot_sync(0xffffffffu, day);
  if (lane == 0) wbase[w] = __popc(m);
  __syncthreads();
  if (w == 0) {
    int b = red[0][lane], a = red[1][lane];
    const int n = wbase[lane];
    int incl = n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      b += __shfl_xor_sync(0xffffffffu, b, o);
      a += __shfl_xor_sync(0xffffffffu, a, o);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    wbase[lane] = b + incl - n;   // tile offset + daytime columns of the warps before
    if (lane == 0) s_nday = a;
  }
  __syncthreads();
  const int nday = s_nday;
  // a daytime column's rank is below nday and at most its own index, so the
  // two stores never meet
  if (day) idxday[wbase[w] + __popc(m & ((1u << lane) - 1u))] = (int32_t)(i + 1);
  if (i < im && i >= nday) idxday[i] = 0;
  if (blockIdx.x == 0 && t == 0) *nday_out = nday;
}

struct SwPostK {
  int im, levs, lm, kd, swhtr, day;
  const double* alb[4];              // sfcalb1..4
  const double *htswc, *htsw0;
  double* dn[4];                     // nirbmdi, nirdfdi, visbmdi, visdfdi
  double* up[4];                     // nirbmui, nirdfui, visbmui, visdfui
  double *sfcdsw, *sfcnsw, *htrsw, *swhc, *scmpsw, *sfcfsw, *topfsw;
};

// rrtmg_sw_post_run (rrtmg_sw_post.F90:52-127).  Daytime (nday > 0): the
// heating-rate levels as in the longwave step, then per column the four
// surface components of the cmpfsw record {uvbfc, uvbf0, nirbm, nirdf, visbm,
// visdf} and their products with the albedos.  No daytime point: the level
// arrays, the component fields and the three flux records set to zero.  Last,
// per column, the net and downward surface fluxes from the sfcfsw record
// {upfxc, dnfxc, upfx0, dnfx0}.
__global__ void sw_post_kernel(SwPostK a) {
  const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t im = (size_t)a.im;
  if (a.day) {
    map_levels(a.htswc, a.htsw0, a.htrsw, a.swhc, a.swhtr != 0, im, a.lm, a.levs, a.kd, t0, stride);
  } else {
    const size_t n = im * a.levs;
    for (size_t e = t0; e < n; e += stride) {
      __stcs(a.htrsw + e, 0.0);
      if (a.swhtr) __stcs(a.swhc + e, 0.0);
    }
  }
  for (size_t i = t0; i < im; i += stride) {
    double* c = a.scmpsw + 6 * i;
    double* f = a.sfcfsw + 4 * i;
    if (a.day) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double v = c[2 + j];
        a.dn[j][i] = v;
        a.up[j][i] = v * a.alb[j][i];
      }
    } else {
#pragma unroll
      for (int j = 0; j < 6; ++j) c[j] = 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        f[j] = 0.0;
        a.dn[j][i] = 0.0;
        a.up[j][i] = 0.0;
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) a.topfsw[3 * i + j] = 0.0;
    }
    a.sfcnsw[i] = f[1] - f[0];
    a.sfcdsw[i] = f[1];
  }
}

// ------------------------------------------------------------------- host --

// Entry point of the calling thread's current call, named in error messages.
thread_local const char* tl_who = "rrtmg_lw_gpu";

void set_msg(char* errmsg, int32_t len, const char* fmt, ...) {
  if (!errmsg || len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(errmsg, (size_t)len, fmt, ap);
  va_end(ap);
}

int fail(char* errmsg, int32_t len, const char* what, cudaError_t e) {
  set_msg(errmsg, len, "%s: %s failed: %s", tl_who, what, cudaGetErrorString(e));
  return 1;
}

#define CK(call, what)                                       \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return fail(errmsg, errmsg_len, what, e_); \
  } while (0)

// Device scratch of the calling thread (seed stream, host-memory staging),
// kept between calls.  Every call that uses it synchronises its stream before
// returning, so a later call of the same thread may reuse or replace it.
struct PrepScratch {
  int device = -1;
  char* p = nullptr;
  size_t bytes = 0;
};
std::mutex g_scratch_mu;
std::vector<PrepScratch*> g_scratch;   // every thread's scratch, released by prep_release
thread_local PrepScratch* tl_scratch = nullptr;

cudaError_t scratch(size_t need, char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!tl_scratch) {
    tl_scratch = new PrepScratch();
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    g_scratch.push_back(tl_scratch);
  }
  PrepScratch& s = *tl_scratch;
  if (s.p && (s.bytes < need || s.device != dev)) {
    cudaFree(s.p);   // no queued work uses it (see above)
    s.p = nullptr;
    s.bytes = 0;
  }
  if (!s.p) {
    const size_t n = std::max<size_t>(need, 1 << 20) * 5 / 4;
    e = cudaMalloc((void**)&s.p, n);
    if (e != cudaSuccess) return e;
    s.bytes = n;
    s.device = dev;
  }
  *out = s.p;
  return cudaSuccess;
}

// Host-memory calls: the arrays of a call are staged through the thread's
// scratch.  Outputs are copied in as well, so elements a step leaves alone
// keep the caller's values.  upload() also reserves `extra` device bytes for
// the call (returned in *extra_p), host memory or not.
class Stager {
 public:
  Stager(bool host, cudaStream_t st) : host_(host), st_(st) {}
  template <typename T>
  void add(T*& field, size_t count, bool out) {
    if (!host_ || !field || count == 0) return;
    items_.push_back(Item{reinterpret_cast<void**>(const_cast<typename std::remove_const<T>::type**>(&field)),
                          (void*)field, count * sizeof(T), out, total_});
    total_ += (count * sizeof(T) + 255) / 256 * 256;
  }
  cudaError_t upload(size_t extra = 0, char** extra_p = nullptr) {
    if (total_ + extra == 0) return cudaSuccess;
    cudaError_t e = scratch(total_ + extra, &buf_);
    if (e != cudaSuccess) return e;
    if (extra_p) *extra_p = buf_ + total_;
    for (Item& it : items_) {
      e = cudaMemcpyAsync(buf_ + it.off, it.host, it.bytes, cudaMemcpyHostToDevice, st_);
      if (e != cudaSuccess) return e;
      *it.field = buf_ + it.off;
    }
    return cudaSuccess;
  }
  cudaError_t download() {
    if (!host_) return cudaSuccess;
    for (Item& it : items_) {
      if (!it.out) continue;
      cudaError_t e = cudaMemcpyAsync(it.host, buf_ + it.off, it.bytes, cudaMemcpyDeviceToHost, st_);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

 private:
  struct Item {
    void** field;
    void* host;
    size_t bytes;
    bool out;
    size_t off;
  };
  bool host_;
  cudaStream_t st_;
  char* buf_ = nullptr;
  size_t total_ = 0;
  std::vector<Item> items_;
};

// Common prologue: memory space, device and stream.
int begin_on(int32_t memory, void* stream, int dev, bool* host, cudaStream_t* st, char* errmsg,
             int32_t errmsg_len) {
  if (memory != RRTMG_LW_HOST && memory != RRTMG_LW_DEVICE) {
    set_msg(errmsg, errmsg_len, "%s: memory must be 0 (host) or 1 (device)", tl_who);
    return 1;
  }
  *host = memory == RRTMG_LW_HOST;
  if (dev >= 0) CK(cudaSetDevice(dev), "cudaSetDevice");
  *st = stream ? (cudaStream_t)stream : cudaStreamPerThread;
  return 0;
}

int begin(const rrtmg_lw_exec* x, bool* host, cudaStream_t* st, char* errmsg, int32_t errmsg_len) {
  if (!x) { set_msg(errmsg, errmsg_len, "%s: null exec struct", tl_who); return 1; }
  return begin_on(x->memory, x->stream, lw::selected_device(), host, st, errmsg, errmsg_len);
}

int finish(Stager& S, bool host, bool sync, cudaStream_t st, char* errmsg, int32_t errmsg_len) {
  CK(cudaGetLastError(), "kernel launch");
  CK(S.download(), "cudaMemcpyAsync");
  if (host || sync) CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return 0;
}

int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace

extern "C" int rrtmg_lw_gpu_seeds(const rrtmg_lw_seed_args* a, const rrtmg_lw_exec* x, char* errmsg,
                                  int32_t errmsg_len) {
  tl_who = "rrtmg_lw_gpu_seeds";
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: null argument struct"); return 1; }
  // GFS_rad_time_vary.fv3.F90:59, :64
  if (!((a->lsswr || a->lslwr) && (a->isubc_lw == 2 || a->isubc_sw == 2))) return 0;
  const int n = a->n;
  if (n < 0) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: n must be >= 0"); return 1; }
  if (n == 0) return 0;
  if (!a->icsdsw || !a->icsdlw) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: icsdsw and icsdlw are required");
    return 1;
  }
  bool host;
  cudaStream_t st;
  if (begin(x, &host, &st, errmsg, errmsg_len)) return 1;
  rrtmg_lw_seed_args b = *a;
  Stager S(host, st);
  if (a->lrseeds) {
    const int ld = a->ld_rseeds ? a->ld_rseeds : n;
    if (!a->rseeds || ld < n) {
      set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: lrseeds needs rseeds with ld_rseeds >= n");
      return 1;
    }
    S.add(b.rseeds, (size_t)ld + n, false);
    S.add(b.icsdsw, n, true);
    S.add(b.icsdlw, n, true);
    CK(S.upload(), "staging");
    seed_copy_kernel<<<blocks_for(n, 256), 256, 0, st>>>(b.rseeds, n, ld, b.icsdsw, b.icsdlw);
    return finish(S, host, x->sync != 0, st, errmsg, errmsg_len);
  }
  if (!a->imap || !a->jmap) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: imap and jmap are required"); return 1; }
  if (a->ipsdlim <= 0 || a->cnx <= 0 || a->cny <= 0) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: ipsdlim, cnx and cny must be positive");
    return 1;
  }
  const long long face = (long long)a->cnx * a->cny;
  if (2 * face > INT_MAX) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: 2 cnx cny exceeds a default integer"); return 1; }
  // ipseed = mod(nint(con_100 sqrt(sec)), ipsdlim) + 1 + ipsd0 (:72)
  const double r = 100.0 * std::sqrt(a->sec);
  if (!(r < 2147483647.5)) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: nint(100 sqrt(sec)) is not a default integer"); return 1; }
  const long long nr = std::llround(r);   // NINT: nearest, halves away from zero
  const int32_t ipseed = (int32_t)(uint32_t)((uint64_t)(nr % a->ipsdlim) + 1u + (uint64_t)(int64_t)a->ipsd0);

  S.add(b.imap, n, false);
  S.add(b.jmap, n, false);
  S.add(b.icsdsw, n, true);
  S.add(b.icsdlw, n, true);
  char* extra = nullptr;
  const size_t raw_bytes = ((size_t)(2 * face) * sizeof(uint32_t) + 255) / 256 * 256;
  CK(S.upload(raw_bytes + 256, &extra), "staging");
  uint32_t* raw = (uint32_t*)extra;
  int* bad = (int*)(extra + raw_bytes);
  const int none = INT_MAX;
  int first_bad = INT_MAX;
  CK(cudaMemcpyAsync(bad, &none, sizeof(int), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
  CK(lw::seed_stream_launch(ipseed, 2 * face, raw, st), "seed stream launch");
  CK(lw::seed_gather_launch(raw, b.imap, b.jmap, n, a->isc, a->jsc, a->cnx, face, a->ipsdlim, b.icsdsw, b.icsdlw,
                            bad, st), "seed gather launch");
  CK(cudaMemcpyAsync(&first_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  if (finish(S, true, true, st, errmsg, errmsg_len)) return 1;
  if (first_bad != INT_MAX) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_seeds: column %d: imap/jmap/isc/jsc give a grid index outside the "
            "cnx x cny face", first_bad + 1);
    return 1;
  }
  return 0;
}

extern "C" int rrtmg_lw_gpu_overlap_params(const rrtmg_lw_overlap_args* a, const rrtmg_lw_exec* x, char* errmsg,
                                           int32_t errmsg_len) {
  tl_who = "rrtmg_lw_gpu_overlap_params";
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_overlap_params: null argument struct"); return 1; }
  if (a->mode < RRTMG_LW_OVERLAP_CLOUDS || a->mode > RRTMG_LW_OVERLAP_ALPHA) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_overlap_params: unknown mode %d", a->mode);
    return 1;
  }
  const int npts = a->npts, nlay = a->nlay, ld = a->ldim ? a->ldim : a->npts;
  if (npts < 0 || nlay < 0 || ld < npts) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_overlap_params: need npts >= 0, nlay >= 0, ldim >= npts");
    return 1;
  }
  OverlapK k{};
  k.npts = npts; k.nlay = nlay; k.ld = ld;
  k.yearlen = a->yearlen; k.julian = a->julian; k.dcorr_con = a->dcorr_con; k.con_pi = a->con_pi;
  // radiation_clouds.f:838-846: three independent tests, the last one that holds wins
  int kind = kDcorrNone;
  if (a->idcor == a->idcor_hogan) kind = kDcorrHogan;
  if (a->idcor == a->idcor_oreopoulos) kind = kDcorrOreopoulos;
  if (a->idcor == a->idcor_con) kind = kDcorrCon;
  const bool expo = a->iovr == a->iovr_dcorr || a->iovr == a->iovr_exp || a->iovr == a->iovr_exprand;
  if (a->mode != RRTMG_LW_OVERLAP_ALPHA) k.dcorr = kind;
  if (a->mode == RRTMG_LW_OVERLAP_ALPHA || (a->mode == RRTMG_LW_OVERLAP_CLOUDS && expo)) k.alpha = 1;
  if (a->mode == RRTMG_LW_OVERLAP_CLOUDS && !expo) { k.zero = 1; k.dcorr = kDcorrNone; }
  k.exprand = k.alpha && a->iovr == a->iovr_exprand;
  if (kind == kDcorrOreopoulos && k.dcorr && a->yearlen == 0) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_overlap_params: yearlen must be nonzero");
    return 1;
  }
  const char* missing = nullptr;
  if (!a->de_lgth) missing = "de_lgth";
  else if ((k.alpha || k.zero) && nlay > 0 && !a->alpha) missing = "alpha";
  else if (k.dcorr == kDcorrHogan && !a->xlat) missing = "xlat";
  else if (k.dcorr == kDcorrOreopoulos && !a->latdeg) missing = "latdeg";
  else if (k.alpha && nlay > 1 && !a->dzlay) missing = "dzlay";
  else if (k.exprand && nlay > 0 && !a->cld_frac) missing = "cld_frac";
  if (missing) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_overlap_params: %s is required", missing); return 1; }
  if (npts == 0) return 0;
  bool host;
  cudaStream_t st;
  if (begin(x, &host, &st, errmsg, errmsg_len)) return 1;
  rrtmg_lw_overlap_args b = *a;
  const size_t nf = (size_t)ld * (nlay > 0 ? nlay - 1 : 0) + npts;   // elements of one (ld, nlay) field
  Stager S(host, st);
  if (k.dcorr == kDcorrHogan) S.add(b.xlat, npts, false);
  if (k.dcorr == kDcorrOreopoulos) S.add(b.latdeg, npts, false);
  if (k.alpha && nlay > 1) S.add(b.dzlay, nf, false);
  if (k.exprand && nlay > 0) S.add(b.cld_frac, nf, false);
  S.add(b.de_lgth, npts, true);
  if ((k.alpha || k.zero) && nlay > 0) S.add(b.alpha, nf, true);
  CK(S.upload(), "staging");
  k.xlat = b.xlat; k.latdeg = b.latdeg; k.dzlay = b.dzlay; k.cld_frac = b.cld_frac;
  k.de_lgth = b.de_lgth; k.alpha_out = b.alpha;
  if (k.dcorr || k.alpha || k.zero) {
    overlap_kernel<<<blocks_for(npts, 128), 128, 0, st>>>(k);
  }
  return finish(S, host, x->sync != 0, st, errmsg, errmsg_len);
}

extern "C" int rrtmg_lw_gpu_post(const rrtmg_lw_post_args* a, const rrtmg_lw_exec* x, char* errmsg,
                                 int32_t errmsg_len) {
  tl_who = "rrtmg_lw_gpu_post";
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_post: null argument struct"); return 1; }
  if (!a->lslwr) return 0;   // rrtmg_lw_post.F90:42
  const int im = a->im, levs = a->levs, lm = a->lm, ltp = a->ltp, kd = a->kd;
  if (im < 0 || levs < 0 || lm < 0 || ltp < 0 || kd < 0 || kd > ltp || lm > levs || (levs > lm && lm < 1)) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_post: need im, levs, lm, ltp, kd >= 0, kd <= ltp, lm <= levs "
            "and lm >= 1 when levs > lm");
    return 1;
  }
  const char* missing = nullptr;
  if (!a->tsfa || !a->tsflw) missing = "tsfa and tsflw";
  else if (!a->sfcflw || !a->sfcdlw) missing = "sfcflw and sfcdlw";
  else if (levs > 0 && (!a->htlwc || !a->htrlw)) missing = "htlwc and htrlw";
  else if (levs > 0 && a->lwhtr && (!a->htlw0 || !a->lwhc)) missing = "htlw0 and lwhc (lwhtr)";
  if (missing) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_post: %s are required", missing); return 1; }
  if (im == 0) return 0;
  bool host;
  cudaStream_t st;
  if (begin(x, &host, &st, errmsg, errmsg_len)) return 1;
  rrtmg_lw_post_args b = *a;
  const size_t nin = (size_t)im * (lm + ltp), nout = (size_t)im * levs;
  Stager S(host, st);
  S.add(b.tsfa, im, false);
  S.add(b.sfcflw, 4 * (size_t)im, false);
  S.add(b.tsflw, im, true);
  S.add(b.sfcdlw, im, true);
  if (levs > 0) {
    S.add(b.htlwc, nin, false);
    S.add(b.htrlw, nout, true);
    if (a->lwhtr) {
      S.add(b.htlw0, nin, false);
      S.add(b.lwhc, nout, true);
    }
  }
  CK(S.upload(), "staging");
  PostK k{im, levs, lm, kd, a->lwhtr ? 1 : 0, b.tsfa, b.htlwc, b.htlw0, b.sfcflw, b.tsflw, b.sfcdlw, b.htrlw, b.lwhc};
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long work = std::max<long long>((long long)im * lm / 4, im);
  const int grid = (int)std::min<long long>(blocks_for(work, 256), 8LL * sms);
  post_kernel<<<grid, 256, 0, st>>>(k);
  return finish(S, host, x->sync != 0, st, errmsg, errmsg_len);
}

extern "C" int rrtmg_sw_gpu_pre(const rrtmg_sw_pre_args* a, const rrtmg_sw_exec* x, char* errmsg,
                                int32_t errmsg_len) {
  tl_who = "rrtmg_sw_gpu_pre";
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_pre: null argument struct"); return 1; }
  const int im = a->im;
  if (im < 0) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_pre: need im >= 0"); return 1; }
  if (!a->nday || (im > 0 && !a->idxday) || (im > 0 && a->lsswr && !a->coszen)) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_pre: nday, idxday and (lsswr) coszen are required");
    return 1;
  }
  *a->nday = 0;   // rad_sw_pre.F90:38, 47
  if (im == 0) return 0;
  const rrtmg_sw_exec dflt{0, RRTMG_LW_HOST, nullptr, 1, 0, nullptr};
  if (!x) x = &dflt;
  bool host;
  cudaStream_t st;
  if (begin_on(x->memory, x->stream, lw::sw_selected_device(), &host, &st, errmsg, errmsg_len)) return 1;
  const double* coszen = a->coszen;
  int32_t* idxday = a->idxday;
  const int ntiles = (int)(((long long)im + kPreTile - 1) / kPreTile);
  Stager S(host, st);
  if (a->lsswr) S.add(coszen, im, false);
  S.add(idxday, im, true);
  char* extra = nullptr;
  CK(S.upload(sizeof(int32_t) * ((size_t)ntiles + 1), &extra), "staging");
  int32_t nday = 0;
  if (!a->lsswr) {
    CK(cudaMemsetAsync(idxday, 0, sizeof(int32_t) * (size_t)im, st), "cudaMemsetAsync");   // rad_sw_pre.F90:48
  } else {
    int* counts = (int*)extra;
    int32_t* nday_dev = (int32_t*)(extra + sizeof(int32_t) * (size_t)ntiles);
    sw_pre_count_kernel<<<ntiles, kPreTile, 0, st>>>(coszen, im, counts);
    sw_pre_scatter_kernel<<<ntiles, kPreTile, 0, st>>>(coszen, im, counts, ntiles, idxday, nday_dev);
    CK(cudaGetLastError(), "kernel launch");
    CK(cudaMemcpyAsync(&nday, nday_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  }
  if (finish(S, host, true, st, errmsg, errmsg_len)) return 1;
  *a->nday = nday;
  return 0;
}

extern "C" int rrtmg_sw_gpu_post(const rrtmg_sw_post_args* a, const rrtmg_sw_exec* x, char* errmsg,
                                 int32_t errmsg_len) {
  tl_who = "rrtmg_sw_gpu_post";
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_post: null argument struct"); return 1; }
  if (!a->lsswr) return 0;   // rrtmg_sw_post.F90:52
  const int im = a->im, levs = a->levs, lm = a->lm, ltp = a->ltp, kd = a->kd;
  const bool day = a->nday > 0, hc = a->swhtr != 0;
  if (im < 0 || levs < 0) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_post: need im, levs >= 0");
    return 1;
  }
  if (day && (lm < 0 || ltp < 0 || kd < 0 || kd > ltp || lm > levs || (levs > lm && lm < 1))) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_post: with nday > 0 need lm, ltp, kd >= 0, kd <= ltp, "
            "lm <= levs and lm >= 1 when levs > lm");
    return 1;
  }
  double* const dn[4] = {a->nirbmdi, a->nirdfdi, a->visbmdi, a->visdfdi};
  double* const up[4] = {a->nirbmui, a->nirdfui, a->visbmui, a->visdfui};
  const double* const alb[4] = {a->sfcalb1, a->sfcalb2, a->sfcalb3, a->sfcalb4};
  bool comps = true, albs = true;
  for (int j = 0; j < 4; ++j) {
    comps = comps && dn[j] && up[j];
    albs = albs && alb[j];
  }
  const char* missing = nullptr;
  if (!a->sfcfsw || !a->sfcdsw || !a->sfcnsw) missing = "sfcfsw, sfcdsw and sfcnsw";
  else if (!a->scmpsw || !comps) missing = "scmpsw and the eight surface component fields";
  else if (levs > 0 && !a->htrsw) missing = "htrsw";
  else if (levs > 0 && hc && !a->swhc) missing = "swhc (swhtr)";
  else if (day && !albs) missing = "sfcalb1..sfcalb4 (nday > 0)";
  else if (day && lm > 0 && !a->htswc) missing = "htswc (nday > 0)";
  else if (day && lm > 0 && hc && !a->htsw0) missing = "htsw0 (nday > 0, swhtr)";
  else if (!day && !a->topfsw) missing = "topfsw (nday <= 0)";
  if (missing) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_post: %s are required", missing); return 1; }
  if (im == 0) return 0;
  const rrtmg_sw_exec dflt{0, RRTMG_LW_HOST, nullptr, 1, 0, nullptr};
  if (!x) x = &dflt;
  bool host;
  cudaStream_t st;
  if (begin_on(x->memory, x->stream, lw::sw_selected_device(), &host, &st, errmsg, errmsg_len)) return 1;
  SwPostK k{};
  k.im = im;
  k.levs = levs;
  k.lm = day ? lm : 0;
  k.kd = day ? kd : 0;
  k.swhtr = hc ? 1 : 0;
  k.day = day ? 1 : 0;
  for (int j = 0; j < 4; ++j) {
    k.alb[j] = day ? alb[j] : nullptr;
    k.dn[j] = dn[j];
    k.up[j] = up[j];
  }
  k.htswc = day ? a->htswc : nullptr;
  k.htsw0 = day && hc ? a->htsw0 : nullptr;
  k.sfcdsw = a->sfcdsw;
  k.sfcnsw = a->sfcnsw;
  k.htrsw = levs > 0 ? a->htrsw : nullptr;
  k.swhc = levs > 0 && hc ? a->swhc : nullptr;
  k.scmpsw = a->scmpsw;
  k.sfcfsw = a->sfcfsw;
  k.topfsw = day ? nullptr : a->topfsw;
  // host memory: inputs copied in; outputs copied in and back (records the
  // daytime branch only reads go one way)
  const size_t nin = (size_t)im * (lm + ltp), nout = (size_t)im * levs;
  Stager S(host, st);
  for (int j = 0; j < 4; ++j) {
    S.add(k.alb[j], im, false);
    S.add(k.dn[j], im, true);
    S.add(k.up[j], im, true);
  }
  S.add(k.sfcdsw, im, true);
  S.add(k.sfcnsw, im, true);
  S.add(k.scmpsw, 6 * (size_t)im, !day);
  S.add(k.sfcfsw, 4 * (size_t)im, !day);
  S.add(k.topfsw, 3 * (size_t)im, true);
  S.add(k.htrsw, nout, true);
  S.add(k.swhc, nout, true);
  if (day && lm > 0) {
    S.add(k.htswc, nin, false);
    S.add(k.htsw0, nin, false);
  }
  CK(S.upload(), "staging");
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long work = std::max<long long>((long long)im * std::max(k.lm, 1) / 4, (long long)im * (day ? 1 : levs));
  const int grid = (int)std::min<long long>(blocks_for(std::max<long long>(work, 1), 256), 8LL * sms);
  sw_post_kernel<<<grid, 256, 0, st>>>(k);
  return finish(S, host, x->sync != 0, st, errmsg, errmsg_len);
}

// Frees every thread's scratch (rrtmg_lw_gpu_finalize); the records stay, so a
// later call regrows its buffer.
void lw::prep_release() {
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  for (PrepScratch* sc : g_scratch) {
    if (sc->p) cudaFree(sc->p);
    sc->p = nullptr;
    sc->bytes = 0;
  }
}
