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
//
// The seed stream is one Mersenne-twister stream walked by one CTA
// (lw_mcica.cu); the face's indices land in a device buffer and one thread
// per column gathers its pair.  The overlap parameters run one thread per
// column over its layers (coalesced across columns); the post step one
// thread per (column, level) element.  This file is compiled without FMA
// contraction, so every product and sum rounds as the Fortran's does.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rrtmg_lw_gpu.h"
#include "lw_launch.h"

namespace {

// ---------------------------------------------------------------- kernels --

// icsdsw/icsdlw of column ix from the face's indices numrdm[0, 2 cnx cny)
// (GFS_rad_time_vary.fv3.F90:76-82); a grid index outside the face records
// the smallest such column in *bad and writes nothing for it.
__global__ void seed_gather_kernel(const int32_t* __restrict__ numrdm, const int32_t* __restrict__ imap,
                                   const int32_t* __restrict__ jmap, int n, int isc, int jsc, int cnx,
                                   long long face, int32_t* icsdsw, int32_t* icsdlw, int* bad) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= n) return;
  const long long p = (long long)imap[ix] + isc - 1 + ((long long)jmap[ix] + jsc - 2) * cnx;   // 1-based
  if (p < 1 || p > face) {
    atomicMin(bad, ix);
    return;
  }
  icsdsw[ix] = numrdm[p - 1];
  icsdlw[ix] = numrdm[p - 1 + face];
}

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

__global__ void overlap_kernel(OverlapK a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npts) return;
  if (a.zero) {
    a.de_lgth[i] = 0.0;
    for (int k = 0; k < a.nlay; ++k) a.alpha_out[i + (size_t)a.ld * k] = 0.0;
    return;
  }
  if (a.dcorr == kDcorrHogan) {
    // max(min_dcorr, 2.78 - 4.6 |lat / pi|), eq. 13 (radiation_cloud_overlap.F90:44-47)
    a.de_lgth[i] = fmax(0.6, 2.78 - 4.6 * fabs(a.xlat[i] / a.con_pi));
  } else if (a.dcorr == kDcorrOreopoulos) {
    // eqs. 10-11 with am1, am2, am4, amr of Table 1 (radiation_cloud_overlap.F90:74-90)
    const double am1 = 1.4315, am2 = 2.1219, am4 = -25.584, amr = 7.0;
    const double am3 = (a.julian > 181.0) ? -(4.0 * amr * (a.julian - 272.0) / (double)a.yearlen)
                                          : 4.0 * amr * (a.julian - 91.0) / (double)a.yearlen;
    const double d = a.latdeg[i] - am3;
    a.de_lgth[i] = am1 + am2 * exp(-(d * d) / (am4 * am4));
  } else if (a.dcorr == kDcorrCon) {
    a.de_lgth[i] = a.dcorr_con;
  }
  if (!a.alpha) return;
  // get_alpha_exper (radiation_cloud_overlap.F90:122-141); the exprand rule
  // reads only cld_frac, so it is applied in the same pass
  const double dl = a.de_lgth[i];
  a.alpha_out[i] = 0.0;
  double cf_prev = a.exprand ? a.cld_frac[i] : 0.0;
  for (int k = 1; k < a.nlay; ++k) {
    const size_t o = i + (size_t)a.ld * k;
    double al = exp(-a.dzlay[o] / dl);
    if (a.exprand) {
      const double cf = a.cld_frac[o];
      if (cf == 0.0 && cf_prev > 0.0) al = 0.0;
      cf_prev = cf;
    }
    a.alpha_out[o] = al;
  }
}

struct PostK {
  int im, levs, lm, kd, lwhtr;
  const double *tsfa, *htlwc, *htlw0, *sfcflw;
  double *tsflw, *sfcdlw, *htrlw, *lwhc;
};

// One thread per (column, level) element of htrlw/lwhc
// (rrtmg_lw_post.F90:48-70); the level-0 threads also copy the per-column
// fields (:46, :73).
__global__ void post_kernel(PostK a) {
  const long long total = (long long)a.im * a.levs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / a.im), i = (int)(e - (long long)k * a.im);
    const int src = (k < a.lm ? k : a.lm - 1) + a.kd;
    a.htrlw[e] = a.htlwc[i + (size_t)a.im * src];
    if (a.lwhtr) a.lwhc[e] = a.htlw0[i + (size_t)a.im * src];
    if (k == 0) {
      a.tsflw[i] = a.tsfa[i];
      a.sfcdlw[i] = a.sfcflw[4 * (size_t)i + 2];
    }
  }
  if (a.levs == 0) {   // no levels: the per-column fields only
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.im; i += gridDim.x * blockDim.x) {
      a.tsflw[i] = a.tsfa[i];
      a.sfcdlw[i] = a.sfcflw[4 * (size_t)i + 2];
    }
  }
}

// ------------------------------------------------------------------- host --

void set_msg(char* errmsg, int32_t len, const char* fmt, ...) {
  if (!errmsg || len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(errmsg, (size_t)len, fmt, ap);
  va_end(ap);
}

int fail(char* errmsg, int32_t len, const char* what, cudaError_t e) {
  set_msg(errmsg, len, "rrtmg_lw_gpu: %s failed: %s", what, cudaGetErrorString(e));
  return 1;
}

#define CK(call, what)                                       \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return fail(errmsg, errmsg_len, what, e_); \
  } while (0)

// Host-memory calls: the arrays of a call are staged through one device
// buffer (stream-ordered allocation).  Outputs are copied in as well, so
// elements a step leaves alone keep the caller's values.
class Stager {
 public:
  Stager(bool host, cudaStream_t st) : host_(host), st_(st) {}
  ~Stager() {
    if (buf_) cudaFreeAsync(buf_, st_);
  }
  template <typename T>
  void add(T*& field, size_t count, bool out) {
    if (!host_ || !field || count == 0) return;
    items_.push_back(Item{reinterpret_cast<void**>(const_cast<typename std::remove_const<T>::type**>(&field)),
                          (void*)field, count * sizeof(T), out, total_});
    total_ += (count * sizeof(T) + 255) / 256 * 256;
  }
  cudaError_t upload() {
    if (!host_ || total_ == 0) return cudaSuccess;
    cudaError_t e = cudaMallocAsync((void**)&buf_, total_, st_);
    if (e != cudaSuccess) return e;
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

// Common prologue: exec struct, device and stream.
int begin(const rrtmg_lw_exec* x, bool* host, cudaStream_t* st, char* errmsg, int32_t errmsg_len) {
  if (!x) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: null exec struct"); return 1; }
  if (x->memory != RRTMG_LW_HOST && x->memory != RRTMG_LW_DEVICE) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: memory must be RRTMG_LW_HOST or RRTMG_LW_DEVICE");
    return 1;
  }
  *host = x->memory == RRTMG_LW_HOST;
  const int dev = lw::selected_device();
  if (dev >= 0) CK(cudaSetDevice(dev), "cudaSetDevice");
  *st = x->stream ? (cudaStream_t)x->stream : cudaStreamPerThread;
  return 0;
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
  CK(S.upload(), "staging");
  char* tmp = nullptr;
  const size_t nbytes = ((size_t)(2 * face) * sizeof(int32_t) + 255) / 256 * 256;
  CK(cudaMallocAsync((void**)&tmp, nbytes + sizeof(int), st), "cudaMallocAsync(numrdm)");
  int32_t* numrdm = (int32_t*)tmp;
  int* bad = (int*)(tmp + nbytes);
  const int none = INT_MAX;
  cudaError_t e = cudaMemcpyAsync(bad, &none, sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = lw::seed_index_launch(ipseed, a->ipsdlim, 2 * face, numrdm, st);
  if (e == cudaSuccess) {
    seed_gather_kernel<<<blocks_for(n, 256), 256, 0, st>>>(numrdm, b.imap, b.jmap, n, a->isc, a->jsc, a->cnx, face,
                                                           b.icsdsw, b.icsdlw, bad);
    e = cudaGetLastError();
  }
  int first_bad = INT_MAX;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&first_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) return fail(errmsg, errmsg_len, "seed stream", e);
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
  if (k.dcorr || k.alpha || k.zero) overlap_kernel<<<blocks_for(npts, 128), 128, 0, st>>>(k);
  return finish(S, host, x->sync != 0, st, errmsg, errmsg_len);
}

extern "C" int rrtmg_lw_gpu_post(const rrtmg_lw_post_args* a, const rrtmg_lw_exec* x, char* errmsg,
                                 int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_post: null argument struct"); return 1; }
  if (!a->lslwr) return 0;   // rrtmg_lw_post.F90:41
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
  const long long total = levs > 0 ? (long long)im * levs : im;
  const int grid = (int)std::min<long long>(blocks_for(total, 256), 148LL * 16);
  post_kernel<<<grid, 256, 0, st>>>(k);
  return finish(S, host, x->sync != 0, st, errmsg, errmsg_len);
}
