// sw_api.cu -- C ABI of the B200 RRTMG-SW path (include/rrtmg_sw_gpu.h).
//
// rrtmg_sw_gpu_init   <- rswinit      (physics/Radiation/RRTMG/radsw_main.F90:1388-1536)
// rrtmg_sw_gpu_run*   <- rrtmg_sw_run (radsw_main.F90:493-1379)
//
// The module state of the reference (heatfac, exp_tbl and the coefficient
// DATA) becomes immutable device memory written once by init.  Each host
// thread that calls run gets its own stream and device workspace.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rrtmg_sw_gpu.h"
#include "../data/rrtmg_sw_table_layout.h"
#include "lw_common.cuh"
#include "lw_launch.h"
#include "sw_kernels.h"

extern "C" const unsigned char rrtmg_sw_tables_blob[];
extern "C" const unsigned char rrtmg_sw_tables_blob_end[];

namespace {

constexpr int kNtbmx = 10000;
constexpr double kS0 = 1368.22;                  // RSM:343
constexpr size_t kScratchBudget = (size_t)12 << 30;   // 16,384 columns of 127 layers in one chunk

struct SwState {
  bool ready = false;
  int device = 0, num_sms = 0;
  double* tab = nullptr;     // coefficient blob
  double* etab = nullptr;    // exp_tbl(0:NTBMX)
  double heatfac = 0.0;
};
SwState g;
std::mutex g_mu;

struct SwWorkspace {
  int device = -1;
  cudaStream_t stream = nullptr;
  char* scratch = nullptr;
  size_t scratch_bytes = 0;
  char* stage = nullptr;     // device copies of host arguments
  size_t stage_bytes = 0;
  int* bad = nullptr;
  // pipelined host path: copy streams, double-buffered staging and its events
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in[2] = {}, ev_done[2] = {}, ev_out[2] = {};
  char* pbuf = nullptr;
  size_t pbuf_bytes = 0;
  // physics blocks: the block table, its prefixes and the point table on the
  // device, and the host copies they are uploaded from
  char* btab = nullptr;
  size_t btab_bytes = 0;
  std::vector<sw::SwArgs> h_tab;
  std::vector<int> h_pre;
};
std::vector<SwWorkspace*> g_ws;
thread_local SwWorkspace* tl_ws = nullptr;

void set_msg(char* m, int32_t n, const char* fmt, ...) {
  if (!m || n <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(m, (size_t)n, fmt, ap);
  va_end(ap);
}
int cuda_fail(char* m, int32_t n, const char* what, cudaError_t e) {
  set_msg(m, n, "rrtmg_sw_gpu: %s failed: %s", what, cudaGetErrorString(e));
  return 1;
}
#define CK(call, what)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) return cuda_fail(errmsg, errmsg_len, what, e_);  \
  } while (0)

cudaError_t grow(char** p, size_t* have, size_t need) {
  if (*have >= need && *p) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  const size_t n = std::max<size_t>(need, 256) * 5 / 4;
  cudaError_t e = cudaMalloc((void**)p, n);
  if (e == cudaSuccess) *have = n;
  return e;
}

SwWorkspace* workspace(char* errmsg, int32_t errmsg_len, int* rc) {
  *rc = 0;
  if (tl_ws && tl_ws->device == g.device) return tl_ws;
  SwWorkspace* w = new SwWorkspace();
  w->device = g.device;
  cudaError_t e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&w->bad, sizeof(int));
  if (e != cudaSuccess) {
    *rc = cuda_fail(errmsg, errmsg_len, "workspace setup", e);
    delete w;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_ws.push_back(w);
  tl_ws = w;
  return w;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// per-column scratch bytes of the three kernels
size_t scratch_per_col(int nlay) {
  const int nw = (nlay + 31) / 32;
  return (size_t)(2 * nlay * sw::kSwNg + sw::kSwNg + 3 * nlay * 14 + 2 * nlay + 2 + (nlay + 1) * 10 * 32) * 8 + 4 +
         (size_t)sw::kSwNg * nw * 4 + 64;
}

// carve one chunk's scratch out of the workspace
sw::SwScratch carve(char* base, int nc, int nlay) {
  sw::SwScratch s{};
  const int nw = (nlay + 31) / 32;
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base + off; off += align256(bytes); return p; };
  s.taug = (double*)take((size_t)nc * nlay * sw::kSwNg * 8);
  s.taur = (double*)take((size_t)nc * nlay * sw::kSwNg * 8);
  s.sflux = (double*)take((size_t)nc * sw::kSwNg * 8);
  s.taucw = (double*)take((size_t)nc * nlay * 14 * 8);
  s.ssacw = (double*)take((size_t)nc * nlay * 14 * 8);
  s.asycw = (double*)take((size_t)nc * nlay * 14 * 8);
  s.cldf = (double*)take((size_t)nc * nlay * 8);
  s.aux = (double*)take((size_t)nc * nlay * 8);
  s.zcf1 = (double*)take((size_t)nc * 8);
  s.zcf0 = (double*)take((size_t)nc * 8);
  s.seed = (int32_t*)take((size_t)nc * 4);
  s.bits = (uint32_t*)take((size_t)nc * sw::kSwNg * nw * 4);
  s.lane_store = (double*)take((size_t)nc * (nlay + 1) * 10 * 32 * 8);
  s.nw = nw;
  return s;
}
size_t carve_bytes(int nc, int nlay) {
  const int nw = (nlay + 31) / 32;
  const size_t parts[13] = {(size_t)nc * 8, (size_t)nc * nlay * 8, (size_t)nc * (nlay + 1) * 10 * 32 * 8, (size_t)nc * nlay * sw::kSwNg * 8, (size_t)nc * nlay * sw::kSwNg * 8,
                            (size_t)nc * sw::kSwNg * 8,        (size_t)nc * nlay * 14 * 8,
                            (size_t)nc * nlay * 14 * 8,        (size_t)nc * nlay * 14 * 8,
                            (size_t)nc * nlay * 8,             (size_t)nc * 8,
                            (size_t)nc * 4,                    (size_t)nc * sw::kSwNg * nw * 4};
  size_t t = 0;
  for (size_t p : parts) t += align256(p);
  return t;
}

// Sizes (in elements) of the caller's arrays.
struct Sizes { size_t n2, n3, nlev, np, nd; };
Sizes sizes_of(const rrtmg_sw_run_args* a) {
  const size_t ld = a->ldim > 0 ? (size_t)a->ldim : (size_t)a->npts;
  return Sizes{ld * a->nlay, ld * a->nlay * RRTMG_SW_NBANDS, ld * (size_t)a->nlp1, (size_t)a->npts,
               (size_t)std::max(a->nday, 0)};
}

// 0 = run, -1 = nothing to do, 1 = error
int validate(const rrtmg_sw_run_args* a, const rrtmg_sw_exec* x, char* errmsg, int32_t errmsg_len) {
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_run: null argument struct"); return 1; }
  if (!a->lsswr || a->nday <= 0) return -1;                 // RSM:808-809
  if (a->iswcliq > 0) {                                      // RSM:847-870
    if (!a->cld_lwp || !a->cld_ref_liq || !a->cld_iwp || !a->cld_ref_ice || !a->cld_rwp || !a->cld_ref_rain ||
        !a->cld_swp || !a->cld_ref_snow) {
      set_msg(errmsg, errmsg_len,
              "Logic error: iswcliq>0 requires the following optional arguments to be present: "
              "cld_lwp, cld_ref_liq, cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow");
      return 1;
    }
  } else if (!a->cld_od || !a->cld_ssa || !a->cld_asy) {     // RSM:847-870
    set_msg(errmsg, errmsg_len,
            "Logic error: iswcliq<=0 requires the following optional arguments to be present: cld_od, cld_ssa, cld_asy");
    return 1;
  }
  if (x->precision != 0) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: only FP64 (precision 0) is built"); return 1; }
  if (x->memory != 0 && x->memory != 1) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: memory must be 0 or 1"); return 1; }
  if (a->isubcsw > 2) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: isubcsw=%d: 0 (spcvrtc), 1 or 2 (McICA, spcvrtm)", a->isubcsw);
    return 1;
  }
  if (a->iovr < 0 || a->iovr > 5) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: iovr=%d: mcica_subcol takes iovr 0..5", a->iovr);
    return 1;
  }
  if (a->isubcsw > 0 && a->iovr == 3 && (!a->dzlyr || !a->de_lgth)) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: iovr=3 needs dzlyr and de_lgth");
    return 1;
  }
  if (a->isubcsw > 0 && (a->iovr == 4 || a->iovr == 5) && !a->alpha) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: iovr=%d needs alpha", a->iovr);
    return 1;
  }
  if (a->iswmode < 1 || a->iswmode > 3) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: iswmode must be 1, 2 or 3"); return 1; }
  if (a->npts < 1 || a->nlay < 1 || a->nlp1 != a->nlay + 1 || a->nlay > sw::kSwMaxLay ||
      (a->ldim != 0 && a->ldim < a->npts)) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: bad sizes npts=%d nlay=%d nlp1=%d ldim=%d (nlay <= %d)", a->npts,
            a->nlay, a->nlp1, a->ldim, sw::kSwMaxLay);
    return 1;
  }
  const void* req[] = {a->plyr, a->tlyr, a->qlyr, a->olyr, a->gasvmr_co2, a->gasvmr_n2o, a->gasvmr_ch4,
                       a->gasvmr_o2, a->idxday, a->aeraod, a->aerssa, a->aerasy, a->sfcalb_nir_dir,
                       a->sfcalb_nir_dif, a->sfcalb_uvis_dir, a->sfcalb_uvis_dif, a->delpin, a->cosz, a->cld_cf,
                       a->hswc, a->topflx, a->sfcflx, a->cldtau};
  for (const void* p : req)
    if (!p) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: a required array is NULL"); return 1; }
  if (a->isubcsw == 2 && !a->icseed) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: isubcsw=2 needs icseed"); return 1; }
  if (x->memory == 0)
    for (int p = 0; p < a->nday; ++p)
      if (a->idxday[p] < 1 || a->idxday[p] > a->npts) {
        set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: idxday(%d)=%d outside 1..npts", p + 1, a->idxday[p]);
        return 1;
      }
  return 0;
}

sw::SwArgs device_args(const rrtmg_sw_run_args* a) {
  sw::SwArgs d{};
  d.plyr = a->plyr; d.tlyr = a->tlyr; d.qlyr = a->qlyr; d.olyr = a->olyr;
  d.co2 = a->gasvmr_co2; d.n2o = a->gasvmr_n2o; d.ch4 = a->gasvmr_ch4; d.o2 = a->gasvmr_o2;
  d.delp = a->delpin; d.cf = a->cld_cf;
  d.aod = a->aeraod; d.ssa = a->aerssa; d.asy = a->aerasy; d.cosz = a->cosz;
  d.alb_nir_dir = a->sfcalb_nir_dir; d.alb_nir_dif = a->sfcalb_nir_dif;
  d.alb_uvis_dir = a->sfcalb_uvis_dir; d.alb_uvis_dif = a->sfcalb_uvis_dif;
  d.lwp = a->cld_lwp; d.rel = a->cld_ref_liq; d.iwp = a->cld_iwp; d.rei = a->cld_ref_ice;
  d.rwp = a->cld_rwp; d.rer = a->cld_ref_rain; d.swp = a->cld_swp; d.res = a->cld_ref_snow;
  d.cod = a->cld_od; d.cssa = a->cld_ssa; d.casy = a->cld_asy;
  d.dz = a->dzlyr; d.alpha = a->alpha; d.delg = a->de_lgth;
  d.icseed = a->icseed; d.idxday = a->idxday;
  d.hswc = a->hswc; d.topflx = a->topflx; d.sfcflx = a->sfcflx; d.cldtau = a->cldtau;
  d.hsw0 = a->hsw0; d.hswb = a->hswb; d.flxprf = a->flxprf; d.fdncmp = a->fdncmp;
  d.npts = a->npts; d.nlay = a->nlay; d.ld = a->ldim > 0 ? a->ldim : a->npts;
  d.top_at_1 = a->top_at_1; d.inc_minor = a->inc_minor_gas; d.iovr = a->iovr;
  d.iovr_rand = a->iovr_rand; d.iovr_maxrand = a->iovr_maxrand;
  d.iswcliq = a->iswcliq; d.iswcice = a->iswcice; d.isubcsw = a->isubcsw; d.iswmode = a->iswmode;
  d.s0fac = a->solcon / kS0;   // RSM:820
  d.heatfac = g.heatfac;
  return d;
}

// zero every output of every column (RSM:824-845); device pointers
cudaError_t zero_outputs(const sw::SwArgs& d, const Sizes& z, int nlay, cudaStream_t st) {
  const size_t pitch = (size_t)d.ld * 8, width = (size_t)d.npts * 8;
  cudaError_t e = cudaMemset2DAsync(d.hswc, pitch, 0, width, nlay, st);
  if (e == cudaSuccess) e = cudaMemset2DAsync(d.cldtau, pitch, 0, width, nlay, st);
  if (e == cudaSuccess && d.hsw0) e = cudaMemset2DAsync(d.hsw0, pitch, 0, width, nlay, st);
  if (e == cudaSuccess && d.hswb) e = cudaMemset2DAsync(d.hswb, pitch, 0, width, (size_t)nlay * 14, st);
  if (e == cudaSuccess && d.flxprf) e = cudaMemset2DAsync(d.flxprf, pitch * 4, 0, width * 4, nlay + 1, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d.topflx, 0, z.np * 3 * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d.sfcflx, 0, z.np * 4 * 8, st);
  if (e == cudaSuccess && d.fdncmp) e = cudaMemsetAsync(d.fdncmp, 0, z.np * 6 * 8, st);
  return e;
}

// all kernels of one call on device arguments
int run_device(SwWorkspace* w, const sw::SwArgs& d, int nday, cudaStream_t st, float* kernel_ms, char* errmsg,
               int32_t errmsg_len, const Sizes& z) {
  CK(zero_outputs(d, z, d.nlay, st), "zeroing the outputs");
  const size_t per = scratch_per_col(d.nlay);
  int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nday, kScratchBudget / per));
  CK(grow(&w->scratch, &w->scratch_bytes, carve_bytes(chunk, d.nlay)), "scratch allocation");
  cudaEvent_t ev[4] = {};
  if (kernel_ms) {
    for (auto& e : ev) CK(cudaEventCreate(&e), "cudaEventCreate");
  }
  for (int p0 = 0; p0 < nday; p0 += chunk) {
    const int nc = std::min(chunk, nday - p0);
    sw::SwScratch s = carve(w->scratch, nc, d.nlay);
    s.bad = w->bad;
    const bool first = kernel_ms && p0 == 0;
    if (first) CK(cudaEventRecord(ev[0], st), "cudaEventRecord");
    CK(sw::optics_launch(d, s, p0, nc, g.tab, st), "optics kernel launch");
    if (first) CK(cudaEventRecord(ev[1], st), "cudaEventRecord");
    lw::McicaStage ms;
    ms.cldf = s.cldf;
    ms.seed = s.seed;
    ms.alpha = s.aux;
    ms.ld = nc;
    if (d.isubcsw <= 0) {
      // grid-mean clouds (spcvrtc): no sub-columns
    } else if (d.iovr <= 2) {
      CK(lw::mcica_sw_launch(nc, d.nlay, d.iovr, ms, s.bits, g.num_sms, st), "McICA kernel launch");
    } else {
      CK(lw::mcica_sw_two_set_launch(nc, d.nlay, d.iovr, ms, s.bits, g.num_sms, st), "McICA kernel launch");
    }
    if (first) CK(cudaEventRecord(ev[2], st), "cudaEventRecord");
    CK(sw::rt_launch(d, s, p0, nc, g.etab, st), "transfer kernel launch");
    if (first) CK(cudaEventRecord(ev[3], st), "cudaEventRecord");
  }
  if (kernel_ms) {
    CK(cudaEventSynchronize(ev[3]), "kernel execution");
    // [McICA, optics, transfer], the order of the longwave timings
    cudaEventElapsedTime(&kernel_ms[0], ev[1], ev[2]);
    cudaEventElapsedTime(&kernel_ms[1], ev[0], ev[1]);
    cudaEventElapsedTime(&kernel_ms[2], ev[2], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return 0;
}

int check_bad(SwWorkspace* w, cudaStream_t st, char* errmsg, int32_t errmsg_len) {
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, w->bad, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  CK(cudaStreamSynchronize(st), "kernel execution");
  if (bad) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: idxday names a column outside 1..npts (those points were skipped)");
    return 1;
  }
  return 0;
}

// Host arrays of many columns: chunks of kSwHostChunk columns, double-
// buffered, each chunk's inputs copied (strided, 2-D) on one copy stream,
// its kernels on the compute stream and its outputs copied back on a second
// copy stream, so copies of chunk j+1 and j-1 overlap the kernels of chunk j.
// The daytime points are split by chunk on the host (chunk-relative indices);
// seed0 keeps the isubcsw = 1 seeds global.
constexpr int kSwHostChunk = 4096;

struct HostField {
  const void* h;   // caller's array
  void** slot;     // the pointer in the chunk's argument record
  size_t rows;     // rows of ldim (0: a per-column vector of `width` values)
  size_t width;    // values per column in a row
  size_t elem;
  bool out;
};

int run_host_pipelined(SwWorkspace* w, const rrtmg_sw_run_args* a, cudaStream_t st, float* kernel_ms, char* errmsg,
                       int32_t errmsg_len) {
  const int npts = a->npts, nlay = a->nlay, nlp1 = nlay + 1;
  const size_t ld = a->ldim > 0 ? (size_t)a->ldim : (size_t)npts;
  const int nch = (npts + kSwHostChunk - 1) / kSwHostChunk;
  std::vector<std::vector<int32_t>> days(nch);
  for (int p = 0; p < a->nday; ++p) {
    const int j1 = a->idxday[p], ch = (j1 - 1) / kSwHostChunk;
    days[ch].push_back(j1 - ch * kSwHostChunk);
  }
  rrtmg_sw_run_args d = *a;
  std::vector<HostField> fl;
  auto in = [&](const double* const* p, size_t rows) {
    if (*p) fl.push_back({*p, (void**)const_cast<const double**>(p), rows, 1, 8, false});
  };
  const size_t L = nlay, LB = (size_t)nlay * RRTMG_SW_NBANDS;
  in(&d.plyr, L); in(&d.tlyr, L); in(&d.qlyr, L); in(&d.olyr, L); in(&d.gasvmr_co2, L); in(&d.gasvmr_n2o, L);
  in(&d.gasvmr_ch4, L); in(&d.gasvmr_o2, L); in(&d.aeraod, LB); in(&d.aerssa, LB); in(&d.aerasy, LB);
  in(&d.sfcalb_nir_dir, 0); in(&d.sfcalb_nir_dif, 0); in(&d.sfcalb_uvis_dir, 0); in(&d.sfcalb_uvis_dif, 0);
  in(&d.dzlyr, L); in(&d.delpin, L); in(&d.de_lgth, 0); in(&d.alpha, L); in(&d.cosz, 0); in(&d.cld_cf, L);
  in(&d.cld_lwp, L); in(&d.cld_ref_liq, L); in(&d.cld_iwp, L); in(&d.cld_ref_ice, L); in(&d.cld_rwp, L);
  in(&d.cld_ref_rain, L); in(&d.cld_swp, L); in(&d.cld_ref_snow, L); in(&d.cld_od, L); in(&d.cld_ssa, L);
  in(&d.cld_asy, L);
  if (d.icseed) fl.push_back({d.icseed, (void**)const_cast<const int32_t**>(&d.icseed), 0, 1, 4, false});
  d.plvl = d.tlvl = nullptr;   // not read by the shortwave scheme
  d.gasvmr_co = d.gasvmr_cfc11 = d.gasvmr_cfc12 = d.gasvmr_cfc22 = d.gasvmr_ccl4 = nullptr;
  auto out = [&](double** p, size_t rows, size_t width) {
    if (*p) fl.push_back({*p, (void**)p, rows, width, 8, true});
  };
  out(&d.hswc, L, 1); out(&d.topflx, 0, 3); out(&d.sfcflx, 0, 4); out(&d.cldtau, L, 1); out(&d.hsw0, L, 1);
  out(&d.hswb, LB, 1); out(&d.flxprf, nlp1, 4); out(&d.fdncmp, 0, 6);
  std::vector<size_t> off(fl.size() + 1);
  size_t per = 0;
  for (size_t k = 0; k < fl.size(); ++k) {
    off[k] = per;
    per += align256(std::max<size_t>(fl[k].rows, 1) * fl[k].width * kSwHostChunk * fl[k].elem);
  }
  off[fl.size()] = per;   // the chunk's daytime list
  per += align256((size_t)kSwHostChunk * 4);
  CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (!w->h2d) {
    CK(cudaStreamCreateWithFlags(&w->h2d, cudaStreamNonBlocking), "cudaStreamCreate");
    CK(cudaStreamCreateWithFlags(&w->d2h, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int k = 0; k < 2; ++k) {
      CK(cudaEventCreateWithFlags(&w->ev_in[k], cudaEventDisableTiming), "cudaEventCreate");
      CK(cudaEventCreateWithFlags(&w->ev_done[k], cudaEventDisableTiming), "cudaEventCreate");
      CK(cudaEventCreateWithFlags(&w->ev_out[k], cudaEventDisableTiming), "cudaEventCreate");
    }
  }
  CK(grow(&w->pbuf, &w->pbuf_bytes, 2 * per), "staging allocation");
  // the kernels' scratch for a whole chunk, allocated before any launch
  const size_t chunk_cols = std::min<size_t>(kSwHostChunk, kScratchBudget / scratch_per_col(nlay));
  CK(grow(&w->scratch, &w->scratch_bytes, carve_bytes((int)chunk_cols, nlay)), "scratch allocation");
  CK(cudaMemsetAsync(w->bad, 0, sizeof(int), st), "cudaMemsetAsync");
  for (int j = 0; j < nch; ++j) {
    const int b = j & 1, c0 = j * kSwHostChunk, n = std::min(kSwHostChunk, npts - c0);
    char* base = w->pbuf + (size_t)b * per;
    if (j >= 2) CK(cudaStreamWaitEvent(w->h2d, w->ev_done[b], 0), "cudaStreamWaitEvent");
    for (size_t k = 0; k < fl.size(); ++k) {
      char* dp = base + off[k];
      *fl[k].slot = dp;
      if (fl[k].out) continue;
      const size_t es = fl[k].elem, wd = fl[k].width;
      const char* hp = static_cast<const char*>(fl[k].h) + (size_t)c0 * wd * es;
      if (fl[k].rows == 0)
        CK(cudaMemcpyAsync(dp, hp, (size_t)n * wd * es, cudaMemcpyHostToDevice, w->h2d), "cudaMemcpyAsync(H2D)");
      else
        CK(cudaMemcpy2DAsync(dp, (size_t)n * wd * es, hp, ld * wd * es, (size_t)n * wd * es, fl[k].rows,
                             cudaMemcpyHostToDevice, w->h2d), "cudaMemcpy2DAsync(H2D)");
    }
    int32_t* didx = (int32_t*)(base + off[fl.size()]);
    if (!days[j].empty())
      CK(cudaMemcpyAsync(didx, days[j].data(), days[j].size() * 4, cudaMemcpyHostToDevice, w->h2d),
         "cudaMemcpyAsync(H2D)");
    CK(cudaEventRecord(w->ev_in[b], w->h2d), "cudaEventRecord");
    CK(cudaStreamWaitEvent(st, w->ev_in[b], 0), "cudaStreamWaitEvent");
    if (j >= 2) CK(cudaStreamWaitEvent(st, w->ev_out[b], 0), "cudaStreamWaitEvent");
    rrtmg_sw_run_args dc = d;
    dc.npts = n;
    dc.ldim = n;
    dc.idxday = didx;
    dc.nday = (int)days[j].size();
    sw::SwArgs da = device_args(&dc);
    da.seed0 = c0;
    const Sizes z = sizes_of(&dc);
    int r = run_device(w, da, dc.nday, st, (j == 0) ? kernel_ms : nullptr, errmsg, errmsg_len, z);
    if (r) return r;
    CK(cudaEventRecord(w->ev_done[b], st), "cudaEventRecord");
    CK(cudaStreamWaitEvent(w->d2h, w->ev_done[b], 0), "cudaStreamWaitEvent");
    for (size_t k = 0; k < fl.size(); ++k) {
      if (!fl[k].out) continue;
      const size_t es = fl[k].elem, wd = fl[k].width;
      char* hp = static_cast<char*>(const_cast<void*>(fl[k].h)) + (size_t)c0 * wd * es;
      const char* dp = base + off[k];
      if (fl[k].rows == 0)
        CK(cudaMemcpyAsync(hp, dp, (size_t)n * wd * es, cudaMemcpyDeviceToHost, w->d2h), "cudaMemcpyAsync(D2H)");
      else
        CK(cudaMemcpy2DAsync(hp, ld * wd * es, dp, (size_t)n * wd * es, (size_t)n * wd * es, fl[k].rows,
                             cudaMemcpyDeviceToHost, w->d2h), "cudaMemcpy2DAsync(D2H)");
    }
    CK(cudaEventRecord(w->ev_out[b], w->d2h), "cudaEventRecord");
  }
  CK(cudaStreamSynchronize(w->d2h), "kernel execution");
  return check_bad(w, st, errmsg, errmsg_len);
}

}  // namespace

extern "C" int rrtmg_sw_gpu_init(const rrtmg_sw_init_args* a, char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_init: null argument struct"); return 1; }
  int errflg = 0;
  if (a->iovr != a->iovr_rand && a->iovr != a->iovr_maxrand && a->iovr != a->iovr_max &&
      a->iovr != a->iovr_dcorr && a->iovr != a->iovr_exp && a->iovr != a->iovr_exprand) {   // RSM:1466-1471
    errflg = 1;
    set_msg(errmsg, errmsg_len, "ERROR(rswinit): Error in specification of cloud overlap flag");
  }
  if (a->me == 0) {   // RSM:1473-1503
    std::printf(" - Using AER Shortwave Radiation, Version: NCEP SW v5.1  Nov 2012 -RRTMG-SW v3.8   \n");
    if (a->iswmode == 1) std::printf("   --- Delta-eddington 2-stream transfer scheme\n");
    else if (a->iswmode == 2) std::printf("   --- PIFM 2-stream transfer scheme\n");
    else if (a->iswmode == 3) std::printf("   --- Discrete ordinates 2-stream transfer scheme\n");
    if (!a->inc_minor_gas) std::printf("   --- Rare gases absorption is NOT included in SW\n");
    else std::printf("   --- Include rare gases N2O, CH4, O2, absorptions in SW\n");
    if (a->isubcsw == 0) std::printf("   --- Using standard grid average clouds, no sub-column clouds approximation applied\n");
    else if (a->isubcsw == 1) std::printf("   --- Using MCICA sub-colum clouds approximation with a prescribed sequence of permutation seeds\n");
    else if (a->isubcsw == 2) std::printf("   --- Using MCICA sub-colum clouds approximation with provided input array of permutation seeds\n");
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g.heatfac = (a->rad_hr_units == 1) ? 9.80665 * 864.0 / 1.0046e+3 : 9.80665 * 1.0e-2 / 1.0046e+3;   // RSM:1507-1511
  // exp_tbl (RSM:1521-1531), on the host with the C library's exp
  std::vector<double> et(kNtbmx + 1);
  const double bpade = 1.0 / 0.278;
  et[0] = 1.0;
  et[kNtbmx] = 1.e-20;
  for (int i = 1; i <= kNtbmx - 1; ++i) {
    const double tfn = (double)i / (double)(kNtbmx - i);
    et[i] = std::exp(-(bpade * tfn));
  }
  CK(cudaSetDevice(a->device), "cudaSetDevice");
  if (!g.ready || g.device != a->device) {
    g.device = a->device;
    CK(cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, g.device), "cudaDeviceGetAttribute");
    const size_t nb = (size_t)(rrtmg_sw_tables_blob_end - rrtmg_sw_tables_blob);
    if (nb != (size_t)RRTMG_SW_TABLES_NDOUBLE * 8) {
      set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_init: embedded table blob has %zu bytes, expected %zu", nb,
              (size_t)RRTMG_SW_TABLES_NDOUBLE * 8);
      return 1;
    }
    CK(cudaMalloc((void**)&g.tab, nb), "cudaMalloc tables");
    CK(cudaMemcpy(g.tab, rrtmg_sw_tables_blob, nb, cudaMemcpyHostToDevice), "table upload");
    CK(cudaMalloc((void**)&g.etab, (kNtbmx + 1) * 8), "cudaMalloc exp_tbl");
    int max_smem = 0;
    CK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, g.device), "cudaDeviceGetAttribute");
    CK(lw::mcica_upload_powers(), "mcica powers upload");
    CK(lw::mcica_prepare(max_smem), "mcica kernel attributes");
    CK(sw::rt_prepare(max_smem), "transfer kernel attributes");
    CK(lw::mcica_sw_two_set_prepare(max_smem), "two-set McICA kernel attributes");
  }
  CK(cudaMemcpy(g.etab, et.data(), (kNtbmx + 1) * 8, cudaMemcpyHostToDevice), "exp_tbl upload");
  g.ready = true;
  return errflg;
}

extern "C" int rrtmg_sw_gpu_run_ex(const rrtmg_sw_run_args* a, const rrtmg_sw_exec* x, char* errmsg,
                                   int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: rrtmg_sw_gpu_init has not been called"); return 1; }
  rrtmg_sw_exec dflt{0, 0, nullptr, 1, 0, nullptr};
  if (!x) x = &dflt;
  const int v = validate(a, x, errmsg, errmsg_len);
  if (v == -1) return 0;
  if (v) return 1;
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  SwWorkspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = x->stream ? (cudaStream_t)x->stream : w->stream;
  const Sizes z = sizes_of(a);
  CK(cudaMemsetAsync(w->bad, 0, sizeof(int), st), "cudaMemsetAsync");
  if (x->memory == 1) {
    sw::SwArgs d = device_args(a);
    int r = run_device(w, d, a->nday, st, x->kernel_ms, errmsg, errmsg_len, z);
    if (r) return r;
    if (x->sync || x->kernel_ms) return check_bad(w, st, errmsg, errmsg_len);
    return 0;
  }
  if (a->npts >= 2 * kSwHostChunk) return run_host_pipelined(w, a, st, x->kernel_ms, errmsg, errmsg_len);
  // host arrays of few columns: stage every argument in one device buffer
  rrtmg_sw_run_args da = *a;
  std::vector<std::pair<const double**, size_t>> ins = {
      {&da.plyr, z.n2}, {&da.tlyr, z.n2}, {&da.qlyr, z.n2}, {&da.olyr, z.n2},
      {&da.gasvmr_co2, z.n2}, {&da.gasvmr_n2o, z.n2}, {&da.gasvmr_ch4, z.n2}, {&da.gasvmr_o2, z.n2},
      {&da.aeraod, z.n3}, {&da.aerssa, z.n3}, {&da.aerasy, z.n3},
      {&da.sfcalb_nir_dir, z.np}, {&da.sfcalb_nir_dif, z.np}, {&da.sfcalb_uvis_dir, z.np},
      {&da.sfcalb_uvis_dif, z.np}, {&da.delpin, z.n2}, {&da.cosz, z.np}, {&da.cld_cf, z.n2},
      {&da.dzlyr, z.n2}, {&da.de_lgth, z.np}, {&da.alpha, z.n2},
      {&da.cld_lwp, z.n2}, {&da.cld_ref_liq, z.n2}, {&da.cld_iwp, z.n2}, {&da.cld_ref_ice, z.n2},
      {&da.cld_rwp, z.n2}, {&da.cld_ref_rain, z.n2}, {&da.cld_swp, z.n2}, {&da.cld_ref_snow, z.n2},
      {&da.cld_od, z.n2}, {&da.cld_ssa, z.n2}, {&da.cld_asy, z.n2}};
  // outputs: (elements, record width, rows); only the first npts of every
  // row of ldim are the caller's to overwrite
  struct Out { double** p; size_t n, w, rows; };
  const size_t ldz = a->ldim > 0 ? (size_t)a->ldim : (size_t)a->npts;
  std::vector<Out> outs = {
      {&da.hswc, z.n2, 1, (size_t)a->nlay}, {&da.topflx, z.np * 3, 0, 0}, {&da.sfcflx, z.np * 4, 0, 0},
      {&da.cldtau, z.n2, 1, (size_t)a->nlay}, {&da.hsw0, z.n2, 1, (size_t)a->nlay},
      {&da.hswb, z.n3, 1, (size_t)a->nlay * RRTMG_SW_NBANDS}, {&da.flxprf, z.nlev * 4, 4, (size_t)a->nlp1},
      {&da.fdncmp, z.np * 6, 0, 0}};
  size_t total = align256(z.np * 4) + align256(z.nd * 4);
  for (auto& p : ins) if (*p.first) total += align256(p.second * 8);
  for (auto& p : outs) if (*p.p) total += align256(p.n * 8);
  CK(grow(&w->stage, &w->stage_bytes, total), "staging allocation");
  size_t off = 0;
  auto place = [&](size_t bytes) { char* p = w->stage + off; off += align256(bytes); return p; };
  if (a->icseed) {
    int32_t* p = (int32_t*)place(z.np * 4);
    CK(cudaMemcpyAsync(p, a->icseed, z.np * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
    da.icseed = p;
  }
  {
    int32_t* p = (int32_t*)place(z.nd * 4);
    CK(cudaMemcpyAsync(p, a->idxday, z.nd * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
    da.idxday = p;
  }
  for (auto& p : ins) {
    if (!*p.first) continue;
    double* d = (double*)place(p.second * 8);
    CK(cudaMemcpyAsync(d, *p.first, p.second * 8, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
    *p.first = d;
  }
  struct Back { double* host; double* dev; Out o; };
  std::vector<Back> back;
  for (auto& p : outs) {
    if (!*p.p) continue;
    double* d = (double*)place(p.n * 8);
    back.push_back({*p.p, d, p});
    *p.p = d;
  }
  sw::SwArgs d = device_args(&da);
  int r = run_device(w, d, a->nday, st, x->kernel_ms, errmsg, errmsg_len, z);
  if (r) return r;
  for (const Back& b : back) {
    if (b.o.w == 0) {   // per-column records: exactly npts of them
      CK(cudaMemcpyAsync(b.host, b.dev, b.o.n * 8, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    } else {            // (ldim, rows) arrays of w-double records: the npts-wide part of each row
      const size_t pitch = ldz * b.o.w * 8;
      CK(cudaMemcpy2DAsync(b.host, pitch, b.dev, pitch, (size_t)a->npts * b.o.w * 8, b.o.rows,
                           cudaMemcpyDeviceToHost, st), "cudaMemcpy2DAsync");
    }
  }
  return check_bad(w, st, errmsg, errmsg_len);
}

extern "C" int rrtmg_sw_gpu_run(const rrtmg_sw_run_args* a, char* errmsg, int32_t errmsg_len) {
  return rrtmg_sw_gpu_run_ex(a, nullptr, errmsg, errmsg_len);
}

extern "C" int rrtmg_sw_gpu_gas_optics(const rrtmg_sw_run_args* a, double* taug, double* taur, double* sfluxzen,
                                       void* stream, char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: rrtmg_sw_gpu_init has not been called"); return 1; }
  if (!a || a->nday <= 0 || a->nlay < 1 || a->nlay > sw::kSwMaxLay || !taug || !taur || !sfluxzen) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_gas_optics: bad arguments");
    return 1;
  }
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  SwWorkspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : w->stream;
  sw::SwArgs d = device_args(a);
  d.cldtau = nullptr;
  const int nday = a->nday, nlay = a->nlay;
  CK(grow(&w->scratch, &w->scratch_bytes, carve_bytes(nday, nlay)), "scratch allocation");
  sw::SwScratch s = carve(w->scratch, nday, nlay);
  s.bad = w->bad;
  d.gas_only = 1;
  CK(cudaMemsetAsync(w->bad, 0, sizeof(int), st), "cudaMemsetAsync");
  CK(sw::optics_launch(d, s, 0, nday, g.tab, st), "optics kernel launch");
  const size_t n = (size_t)nday * nlay * sw::kSwNg;
  CK(cudaMemcpyAsync(taug, s.taug, n * 8, cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
  CK(cudaMemcpyAsync(taur, s.taur, n * 8, cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
  CK(cudaMemcpyAsync(sfluxzen, s.sflux, (size_t)nday * sw::kSwNg * 8, cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
  return check_bad(w, st, errmsg, errmsg_len);
}

extern "C" int rrtmg_sw_gpu_run_blocks(const rrtmg_sw_run_args* blocks, int32_t nblocks, const rrtmg_sw_exec* x,
                                       char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: rrtmg_sw_gpu_init has not been called"); return 1; }
  if (!blocks || nblocks < 0 || !x || x->memory != 1) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_run_blocks: blocks, nblocks >= 0 and device memory (exec->memory = 1) needed");
    return 1;
  }
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  SwWorkspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = x->stream ? (cudaStream_t)x->stream : w->stream;
  // validate; blocks with nothing to do (lsswr off, nday <= 0) drop out
  w->h_tab.clear();
  std::vector<int> colpre, dayp(1, 0);
  const rrtmg_sw_run_args* first = nullptr;
  int total_cols = 0;
  for (int b = 0; b < nblocks; ++b) {
    const rrtmg_sw_run_args* a = &blocks[b];
    const int v = validate(a, x, errmsg, errmsg_len);
    if (v == -1) continue;
    if (v) {
      char tmp[256];
      std::snprintf(tmp, sizeof tmp, "%s", errmsg ? errmsg : "");
      set_msg(errmsg, errmsg_len, "block %d: %s", b, tmp);
      return 1;
    }
    if (!first) {
      first = a;
    } else if (a->nlay != first->nlay || a->top_at_1 != first->top_at_1 || a->inc_minor_gas != first->inc_minor_gas ||
               a->iovr != first->iovr || a->iovr_rand != first->iovr_rand || a->iovr_maxrand != first->iovr_maxrand ||
               a->iswcliq != first->iswcliq || a->iswcice != first->iswcice || a->isubcsw != first->isubcsw ||
               a->iswmode != first->iswmode || (a->hswb != nullptr) != (first->hswb != nullptr)) {
      set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_run_blocks: block %d differs from the first in nlay, flags or hswb", b);
      return 1;
    }
    w->h_tab.push_back(device_args(a));
    colpre.push_back(total_cols);
    total_cols += a->npts;
    dayp.push_back(dayp.back() + a->nday);
  }
  const int nb = (int)w->h_tab.size(), ndays = dayp.back();
  if (nb == 0) return 0;
  const int nlay = first->nlay;
  // device copies: table, column prefixes, day prefixes, point table
  w->h_pre.assign(colpre.begin(), colpre.end());
  w->h_pre.insert(w->h_pre.end(), dayp.begin(), dayp.end());
  const size_t tab_b = align256((size_t)nb * sizeof(sw::SwArgs)), pre_b = align256(w->h_pre.size() * 4);
  const size_t pts_b = align256((size_t)std::max(ndays, 1) * sizeof(int2));
  CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");   // an earlier call may still read the tables
  CK(grow(&w->btab, &w->btab_bytes, tab_b + pre_b + pts_b), "block table allocation");
  sw::SwArgs* d_tab = (sw::SwArgs*)w->btab;
  int* d_pre = (int*)(w->btab + tab_b);
  int2* d_pts = (int2*)(w->btab + tab_b + pre_b);
  CK(cudaMemcpyAsync(d_tab, w->h_tab.data(), (size_t)nb * sizeof(sw::SwArgs), cudaMemcpyHostToDevice, st),
     "cudaMemcpyAsync");
  CK(cudaMemcpyAsync(d_pre, w->h_pre.data(), w->h_pre.size() * 4, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
  CK(cudaMemsetAsync(w->bad, 0, sizeof(int), st), "cudaMemsetAsync");
  CK(sw::blocks_prepare(d_tab, d_pre, d_pre + nb, nb, total_cols, d_pts, w->bad, st), "block table kernels");
  // the kernels over all daytime points, in scratch-sized chunks
  const sw::SwArgs& f = w->h_tab[0];
  const size_t per = scratch_per_col(nlay);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(ndays, 1), kScratchBudget / per));
  CK(grow(&w->scratch, &w->scratch_bytes, carve_bytes(chunk, nlay)), "scratch allocation");
  cudaEvent_t ev[4] = {};
  float* kms = x->kernel_ms;
  if (kms)
    for (auto& e : ev) CK(cudaEventCreate(&e), "cudaEventCreate");
  for (int p0 = 0; p0 < ndays; p0 += chunk) {
    const int nc = std::min(chunk, ndays - p0);
    sw::SwScratch sc = carve(w->scratch, nc, nlay);
    sc.bad = w->bad;
    const bool first_chunk = kms && p0 == 0;
    if (first_chunk) CK(cudaEventRecord(ev[0], st), "cudaEventRecord");
    CK(sw::optics_blocks_launch(d_tab, d_pts, sc, p0, nc, g.tab, st), "optics kernel launch");
    if (first_chunk) CK(cudaEventRecord(ev[1], st), "cudaEventRecord");
    lw::McicaStage ms;
    ms.cldf = sc.cldf;
    ms.seed = sc.seed;
    ms.alpha = sc.aux;
    ms.ld = nc;
    if (f.isubcsw > 0 && f.iovr <= 2)
      CK(lw::mcica_sw_launch(nc, nlay, f.iovr, ms, sc.bits, g.num_sms, st), "McICA kernel launch");
    else if (f.isubcsw > 0)
      CK(lw::mcica_sw_two_set_launch(nc, nlay, f.iovr, ms, sc.bits, g.num_sms, st), "McICA kernel launch");
    if (first_chunk) CK(cudaEventRecord(ev[2], st), "cudaEventRecord");
    CK(sw::rt_blocks_launch(d_tab, d_pts, f.isubcsw <= 0, f.hswb != nullptr, sc, p0, nc, nlay, g.etab, st),
       "transfer kernel launch");
    if (first_chunk) CK(cudaEventRecord(ev[3], st), "cudaEventRecord");
  }
  if (kms) {
    CK(cudaEventSynchronize(ev[3]), "kernel execution");
    cudaEventElapsedTime(&kms[0], ev[1], ev[2]);
    cudaEventElapsedTime(&kms[1], ev[0], ev[1]);
    cudaEventElapsedTime(&kms[2], ev[2], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  if (x->sync || kms) return check_bad(w, st, errmsg, errmsg_len);
  return 0;
}

extern "C" int rrtmg_sw_gpu_mcica(int32_t npts, int32_t nlay, int32_t ldim, int32_t iovr, const int32_t* seed,
                                  const double* cldf, const double* dz, const double* de_lgth, const double* alpha,
                                  uint32_t* bits, void* stream, char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu: rrtmg_sw_gpu_init has not been called"); return 1; }
  const int ld = ldim > 0 ? ldim : npts;
  if (npts < 1 || nlay < 1 || nlay > sw::kSwMaxLay || ld < npts || iovr < 0 || iovr > 5 || !seed || !cldf || !bits ||
      (iovr == 3 && (!dz || !de_lgth)) || ((iovr == 4 || iovr == 5) && !alpha)) {
    set_msg(errmsg, errmsg_len, "rrtmg_sw_gpu_mcica: bad arguments");
    return 1;
  }
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  SwWorkspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : w->stream;
  lw::McicaStage ms;
  ms.cldf = cldf;
  ms.seed = seed;
  ms.ld = ld;
  if (iovr >= 3) {
    CK(grow(&w->scratch, &w->scratch_bytes, (size_t)ld * nlay * 8), "scratch allocation");
    double* aux = (double*)w->scratch;
    CK(sw::overlap_aux_launch(npts, nlay, ld, iovr, dz, de_lgth, alpha, aux, ld, st), "overlap kernel launch");
    ms.alpha = aux;
    CK(lw::mcica_sw_two_set_launch(npts, nlay, iovr, ms, bits, g.num_sms, st), "McICA kernel launch");
  } else {
    CK(lw::mcica_sw_launch(npts, nlay, iovr, ms, bits, g.num_sms, st), "McICA kernel launch");
  }
  CK(cudaStreamSynchronize(st), "McICA kernel execution");
  return 0;
}

// Device of the shortwave post step (lw_prep.cu): the init device, or -1
// before init.
int lw::sw_selected_device() {
  std::lock_guard<std::mutex> lk(g_mu);
  return g.ready ? g.device : -1;
}

extern "C" void rrtmg_sw_gpu_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (SwWorkspace* w : g_ws) {
    if (w->stream) cudaStreamSynchronize(w->stream);
    cudaFree(w->scratch);
    cudaFree(w->stage);
    cudaFree(w->bad);
    cudaFree(w->pbuf);
    cudaFree(w->btab);
    for (int k = 0; k < 2; ++k) {
      if (w->ev_in[k]) cudaEventDestroy(w->ev_in[k]);
      if (w->ev_done[k]) cudaEventDestroy(w->ev_done[k]);
      if (w->ev_out[k]) cudaEventDestroy(w->ev_out[k]);
    }
    if (w->h2d) cudaStreamDestroy(w->h2d);
    if (w->d2h) cudaStreamDestroy(w->d2h);
    if (w->stream) cudaStreamDestroy(w->stream);
    delete w;
  }
  g_ws.clear();
  tl_ws = nullptr;
  if (g.tab) cudaFree(g.tab);
  if (g.etab) cudaFree(g.etab);
  g = SwState{};
}
