// lw_api.cu -- C ABI of the B200 RRTMG-LW library (include/rrtmg_lw_gpu.h).
//
// rrtmg_lw_gpu_init   <- rlwinit      (physics/Radiation/RRTMG/radlw_main.F90:1322-1504)
// rrtmg_lw_gpu_run*   <- rrtmg_lw_run (radlw_main.F90:419-1309)
//
// Module state of the reference (fluxfac, heatfac, the lookup tables and the
// coefficient DATA) becomes immutable device memory written once by init.
// Each host thread that calls run gets its own stream and device workspace,
// so concurrent calls from OpenMP threads (one physics block each, as the
// CCPP host does) do not share mutable state.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rrtmg_lw_gpu.h"
#include "lw_common.cuh"

extern "C" const unsigned char rrtmg_lw_tables_blob[];
extern "C" const unsigned char rrtmg_lw_tables_blob_end[];

namespace lw {
struct NoAllocView {
  int ready, device, num_sms;
  const double* kt64;
  const float* kt32;
  const double* tbl64;
  const float* tbl32;
  Consts cs;
};
NoAllocView noalloc_view();
size_t scratch_per_column_fp64(int V);
size_t scratch_per_column_fp32(int V);
cudaError_t launch_column_fp64(int V, bool hlwb, const Block*, int, const Block&, int, const Flags&, const Consts&,
                               const Tables<double>&, const Tables<double>&, const uint32_t*, void*, size_t,
                               double*, double*, int, cudaStream_t, cudaEvent_t);
cudaError_t launch_column_fp32(int V, bool hlwb, const Block*, int, const Block&, int, const Flags&, const Consts&,
                               const Tables<float>&, const Tables<double>&, const uint32_t*, void*, size_t,
                               double*, double*, int, cudaStream_t, cudaEvent_t);
cudaError_t mcica_upload_powers();
cudaError_t mcica_launch(const Block*, int, const Block&, int, int, int, int, int, const double*,
                         const int32_t*, int, uint32_t*, int, cudaStream_t);
cudaError_t mcica_prepare(int max_smem);
}  // namespace lw

using namespace lw;

namespace {

struct DeviceState {
  bool ready = false;
  int device = 0;
  int num_sms = 0;
  double* kt64 = nullptr;
  float* kt32 = nullptr;
  double* tbl64 = nullptr;   // exp, tfn, tau (3 x (NTBL+1))
  float* tbl32 = nullptr;
  Consts cs{};
};
DeviceState g;
std::mutex g_mu;

struct Workspace {
  int device = -1;
  cudaStream_t stream = nullptr;
  char* dbuf = nullptr;       // device staging for host-memory calls
  size_t dbuf_bytes = 0;
  uint32_t* bits = nullptr;   // McICA sub-column flags
  size_t bits_bytes = 0;
  char* scratch = nullptr;    // gas optics -> transfer hand-off (kernel A -> B)
  size_t scratch_bytes = 0;
  Block* dblocks = nullptr;   // block descriptors on the device
  size_t dblocks_n = 0;
  Block* hblocks = nullptr;   // pinned host copy of the descriptors
  size_t hblocks_n = 0;
};
std::vector<Workspace*> g_workspaces;
thread_local Workspace* tl_ws = nullptr;

void set_msg(char* errmsg, int32_t len, const char* fmt, ...) {
  if (!errmsg || len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(errmsg, (size_t)len, fmt, ap);
  va_end(ap);
}

int cuda_fail(char* errmsg, int32_t len, const char* what, cudaError_t e) {
  set_msg(errmsg, len, "rrtmg_lw_gpu: %s failed: %s", what, cudaGetErrorString(e));
  return 1;
}

#define CK(call, what)                                              \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) return cuda_fail(errmsg, errmsg_len, what, e_); \
  } while (0)

Workspace* workspace(char* errmsg, int32_t errmsg_len, int* rc) {
  *rc = 0;
  if (tl_ws && tl_ws->device == g.device) return tl_ws;
  Workspace* w = new Workspace();
  w->device = g.device;
  cudaError_t e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    *rc = cuda_fail(errmsg, errmsg_len, "cudaStreamCreate", e);
    delete w;
    return nullptr;
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_workspaces.push_back(w);
  }
  tl_ws = w;
  return w;
}

template <typename T>
cudaError_t grow(T** p, size_t* have, size_t need_bytes) {
  if (*have >= need_bytes && *p) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  size_t n = std::max<size_t>(need_bytes, 1) * 5 / 4;
  cudaError_t e = cudaMalloc((void**)p, n);
  if (e == cudaSuccess) *have = n;
  return e;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" int rrtmg_lw_gpu_init(const rrtmg_lw_init_args* a, char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_init: null argument struct"); return 1; }
  int errflg = 0;
  // RLM:1415-1420
  if (a->iovr != a->iovr_rand && a->iovr != a->iovr_maxrand && a->iovr != a->iovr_max &&
      a->iovr != a->iovr_dcorr && a->iovr != a->iovr_exp && a->iovr != a->iovr_exprand) {
    errflg = 1;
    set_msg(errmsg, errmsg_len, "ERROR(rlwinit): Error in specification of cloud overlap flag");
  }
  std::lock_guard<std::mutex> lk(g_mu);
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_init: no CUDA device (%s)", cudaGetErrorString(e));
    return 1;
  }
  if (a->device < 0 || a->device >= ndev) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_init: device %d out of range", a->device);
    return 1;
  }
  CK(cudaSetDevice(a->device), "cudaSetDevice");
  g.device = a->device;
  CK(cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, g.device), "cudaDeviceGetAttribute");

  if (a->me == 0) {
    std::printf(" - Using AER Longwave Radiation (B200 rrtmg_lw_gpu), RRTMG-LW v4.82 tables\n");
    if (a->inc_minor_gas) std::printf("   --- Include rare gases N2O, CH4, O2, CFCs absorptions in LW\n");
    else std::printf("   --- Rare gases effect is NOT included in LW\n");
    if (a->isubclw == 1) std::printf("   --- Using MCICA sub-colum clouds approximation with a prescribed sequence of permutaion seeds\n");
    else if (a->isubclw == 2) std::printf("   --- Using MCICA sub-colum clouds approximation with provided input array of permutation seeds\n");
    else std::printf("   --- Using standard grid average clouds, no sub-column clouds approximation applied\n");
  }

  // fluxfac / heatfac (RLM:1449-1461)
  const double con_g = 9.80665, con_cp = 1.0046e+3;
  double pival = 2.0 * std::asin(1.0);
  g.cs.fluxfac = pival * 2.0e4;
  g.cs.heatfac = (a->rad_hr_units == 1) ? con_g * 864.0 / con_cp : con_g * 1.0e-2 / con_cp;

  // lookup tables (RLM:1474-1501), built on the host with the C library exp
  std::vector<double> tb(3 * (NTBL + 1));
  double* ex = tb.data();
  double* tf = ex + (NTBL + 1);
  double* ta = tf + (NTBL + 1);
  const double bpade = 1.0 / 0.278, expeps = 1.e-20;
  ta[0] = 0.0; ex[0] = 1.0; tf[0] = 0.0;
  ta[NTBL] = 1.e10; ex[NTBL] = expeps; tf[NTBL] = 1.0;
  double explimit = std::trunc(-std::log(DBL_MIN));
  for (int i = 1; i <= NTBL - 1; ++i) {
    double tfn = (double)i / (double)(NTBL - i);
    ta[i] = bpade * tfn;
    ex[i] = (ta[i] >= explimit) ? expeps : std::exp(-ta[i]);
    tf[i] = (ta[i] < 0.06) ? ta[i] / 6.0 : 1.0 - 2.0 * ((1.0 / ta[i]) - (ex[i] / (1.0 - ex[i])));
  }
  std::vector<float> tb32(tb.begin(), tb.end());

  size_t nblob = (size_t)(rrtmg_lw_tables_blob_end - rrtmg_lw_tables_blob);
  if (nblob != sizeof(double) * RRTMG_LW_TABLES_NDOUBLE) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_init: embedded table blob has %zu bytes, expected %zu", nblob,
            sizeof(double) * (size_t)RRTMG_LW_TABLES_NDOUBLE);
    return 1;
  }
  std::vector<double> kt(RRTMG_LW_TABLES_NDOUBLE);
  std::memcpy(kt.data(), rrtmg_lw_tables_blob, nblob);
  std::vector<float> kt32(kt.begin(), kt.end());

  if (!g.kt64) {
    CK(cudaMalloc(&g.kt64, kt.size() * sizeof(double)), "cudaMalloc(tables)");
    CK(cudaMalloc(&g.kt32, kt.size() * sizeof(float)), "cudaMalloc(tables)");
    CK(cudaMalloc(&g.tbl64, tb.size() * sizeof(double)), "cudaMalloc(tables)");
    CK(cudaMalloc(&g.tbl32, tb.size() * sizeof(float)), "cudaMalloc(tables)");
  }
  CK(cudaMemcpy(g.kt64, kt.data(), kt.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(cudaMemcpy(g.kt32, kt32.data(), kt32.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(cudaMemcpy(g.tbl64, tb.data(), tb.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(cudaMemcpy(g.tbl32, tb32.data(), tb32.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(mcica_upload_powers(), "mcica powers upload");
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, g.device), "cudaDeviceGetAttribute");
  CK(mcica_prepare(optin), "kernel attributes (mcica)");
  // per-thread stack for the spilled kernels (a context setting, gone with the process)
  size_t stack = 0;
  CK(cudaDeviceGetLimit(&stack, cudaLimitStackSize), "cudaDeviceGetLimit");
  if (stack < 4096) CK(cudaDeviceSetLimit(cudaLimitStackSize, 4096), "cudaDeviceSetLimit(stack)");
  g.ready = true;
  return errflg;
}

// ---------------------------------------------------------------------------
namespace {

// Validate arguments the way rrtmg_lw_run reports errors (RLM:713-760);
// returns -1 when the call is a no-op (lslwr false or npts == 0).
int validate(const rrtmg_lw_run_args* a, const rrtmg_lw_exec* x, char* errmsg, int32_t errmsg_len,
             bool need_outputs = true) {
  if (!a) { set_msg(errmsg, errmsg_len, "rrtmg_lw_run: null argument struct"); return 1; }
  if (!a->lslwr) return -1;                                  // RLM:727
  if (a->nlay < 1 || a->nlp1 != a->nlay + 1 || a->npts < 0 || (a->ldim != 0 && a->ldim < a->npts)) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_run: inconsistent dimensions (nlay=%d nlp1=%d npts=%d ldim=%d)",
            a->nlay, a->nlp1, a->npts, a->ldim);
    return 1;
  }
  if (a->ilwcliq > 0) {                                      // RLM:739-760
    if (!a->cld_lwp || !a->cld_ref_liq || !a->cld_iwp || !a->cld_ref_ice || !a->cld_rwp ||
        !a->cld_ref_rain || !a->cld_swp || !a->cld_ref_snow) {
      set_msg(errmsg, errmsg_len,
              "Logic error: ilwcliq>0 requires the following optional arguments to be present: "
              "cld_lwp, cld_ref_liq, cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow");
      return 2;
    }
  } else if (!a->cld_od) {
    set_msg(errmsg, errmsg_len, "Logic error: ilwcliq<=0 requires the following optional argument to be present: cld_od");
    return 2;
  }
  if (a->npts == 0) return -1;
  if (a->nlay > 255) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: nlay=%d exceeds the supported maximum of 255 layers", a->nlay);
    return 1;
  }
  if (a->isubclw != 1 && a->isubclw != 2) {
    set_msg(errmsg, errmsg_len,
            "rrtmg_lw_gpu: isubclw=%d not supported (the McICA paths isubclw=1,2 with rtrnmc are)", a->isubclw);
    return 1;
  }
  if (a->iovr < 0 || a->iovr > 2) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: McICA overlap iovr=%d not supported (0, 1, 2 are)", a->iovr);
    return 1;
  }
  const double* req[] = {a->plyr, a->plvl, a->tlyr, a->tlvl, a->qlyr, a->olyr, a->gasvmr_co2, a->gasvmr_n2o,
                         a->gasvmr_ch4, a->gasvmr_o2, a->gasvmr_co, a->gasvmr_cfc11, a->gasvmr_cfc12,
                         a->gasvmr_cfc22, a->gasvmr_ccl4, a->aeraod, a->aerssa, a->sfemis, a->sfgtmp,
                         a->dzlyr, a->delpin, a->cld_cf};
  for (const double* p : req)
    if (!p) { set_msg(errmsg, errmsg_len, "rrtmg_lw_run: a required input array pointer is NULL"); return 1; }
  const double* outs[] = {a->hlwc, a->topflx, a->sfcflx, a->cldtau};
  if (need_outputs)
    for (const double* p : outs)
      if (!p) { set_msg(errmsg, errmsg_len, "rrtmg_lw_run: a required output array pointer is NULL"); return 1; }
  if (a->isubclw == 2 && !a->icseed) { set_msg(errmsg, errmsg_len, "rrtmg_lw_run: icseed is NULL"); return 1; }
  if (x && x->precision != RRTMG_LW_FP64 && x->precision != RRTMG_LW_FP32) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: precision %d not available in this build", x->precision);
    return 1;
  }
  return 0;
}

int pick_v(int nlay) { return nlay <= 63 ? 2 : nlay <= 127 ? 4 : 8; }

// Device scratch budget of one call (columns are processed in chunks that fit).
constexpr size_t kScratchBudget = (size_t)6 << 30;

// Sizes (in doubles) of each input/output field for one block.
struct FieldSizes { size_t n2, n2l, n3, n1; };
FieldSizes sizes_of(const rrtmg_lw_run_args* a) {
  size_t ld = a->ldim > 0 ? (size_t)a->ldim : (size_t)a->npts;
  return {ld * a->nlay, ld * (a->nlay + 1), ld * a->nlay * NBANDS, (size_t)a->npts};
}

void fill_flags(const rrtmg_lw_run_args* a, Flags* f) {
  f->nlay = a->nlay;
  f->top_at_1 = a->top_at_1 != 0;
  f->inc_minor_gas = a->inc_minor_gas != 0;
  f->iovr = a->iovr;
  f->iovr_dcorr = a->iovr_dcorr;
  f->iovr_exp = a->iovr_exp;
  f->iovr_exprand = a->iovr_exprand;
  f->ilwcliq = a->ilwcliq;
  f->ilwcice = a->ilwcice;
  f->isubclw = a->isubclw;
  f->want_hlw0 = a->hlw0 != nullptr;
  f->want_hlwb = a->hlwb != nullptr;
  f->want_flxprf = a->flxprf != nullptr;
  f->gas_only = 0;
}

// Fill a block descriptor from (device) pointers of the argument struct.
void block_from_args(const rrtmg_lw_run_args* a, Block* B) {
  const double* in[N_IN] = {a->plyr, a->plvl, a->tlyr, a->tlvl, a->qlyr, a->olyr, a->gasvmr_co2,
                            a->gasvmr_n2o, a->gasvmr_ch4, a->gasvmr_o2, a->gasvmr_co, a->gasvmr_cfc11,
                            a->gasvmr_cfc12, a->gasvmr_cfc22, a->gasvmr_ccl4, a->aeraod, a->aerssa,
                            a->sfemis, a->sfgtmp, a->dzlyr, a->delpin, a->de_lgth, a->alpha, a->cld_cf,
                            a->cld_lwp, a->cld_ref_liq, a->cld_iwp, a->cld_ref_ice, a->cld_rwp,
                            a->cld_ref_rain, a->cld_swp, a->cld_ref_snow, a->cld_od};
  std::memcpy(B->in, in, sizeof(in));
  B->icseed = a->icseed;
  double* out[N_OUT] = {a->hlwc, a->topflx, a->sfcflx, a->cldtau, a->hlw0, a->hlwb, a->flxprf};
  std::memcpy(B->out, out, sizeof(out));
  B->npts = a->npts;
  B->ld = a->ldim > 0 ? a->ldim : a->npts;
  B->col0 = 0;
  B->pad = 0;
}

int launch(Workspace* w, const Block* hblocks, int nblocks, int ncols, const Flags& f, int precision,
           float* kernel_ms, char* errmsg, int32_t errmsg_len) {
  cudaStream_t st = w->stream;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (kernel_ms)
    for (auto& e : ev) CK(cudaEventCreate(&e), "cudaEventCreate");
  const Block* dblk = nullptr;
  if (nblocks > 1) {
  // descriptors: pinned host staging -> device
  if (w->hblocks_n < (size_t)nblocks) {
    if (w->hblocks) cudaFreeHost(w->hblocks);
    w->hblocks = nullptr;
    w->hblocks_n = 0;
    CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    CK(cudaMallocHost((void**)&w->hblocks, sizeof(Block) * nblocks), "cudaMallocHost");
    w->hblocks_n = nblocks;
  } else {
    CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");   // previous call done with the staging copy
  }
  if (hblocks != w->hblocks) std::memcpy(w->hblocks, hblocks, sizeof(Block) * nblocks);
  size_t have = w->dblocks_n * sizeof(Block);
  CK(grow(&w->dblocks, &have, sizeof(Block) * nblocks), "cudaMalloc(blocks)");
  w->dblocks_n = have / sizeof(Block);
  CK(cudaMemcpyAsync(w->dblocks, w->hblocks, sizeof(Block) * nblocks, cudaMemcpyHostToDevice, st),
     "cudaMemcpyAsync(blocks)");
  dblk = w->dblocks;
  }
  const Block& b0 = hblocks[0];
  const int nw = (f.nlay + 31) / 32;
  if (kernel_ms) CK(cudaEventRecord(ev[0], st), "cudaEventRecord");
  if (f.isubclw > 0 && !f.gas_only) {
    CK(grow(&w->bits, &w->bits_bytes, (size_t)ncols * NGPT * nw * sizeof(uint32_t)), "cudaMalloc(mcica bits)");
    CK(mcica_launch(dblk, nblocks, b0, ncols, f.nlay, f.iovr, f.isubclw, f.top_at_1, nullptr, nullptr, 0,
                    w->bits, g.num_sms, st),
       "McICA kernel launch");
  }
  const int V = pick_v(f.nlay);
  const bool hlwb = f.want_hlwb != 0;
  if (kernel_ms) CK(cudaEventRecord(ev[1], st), "cudaEventRecord");
  // scratch between the gas-optics and transfer kernels, in chunks of columns
  const size_t per = (precision == RRTMG_LW_FP64) ? scratch_per_column_fp64(V) : scratch_per_column_fp32(V);
  size_t budget = kScratchBudget;
  if (const char* env = std::getenv("RRTMG_LW_GPU_SCRATCH_MB")) budget = (size_t)std::atol(env) << 20;
  const size_t want = std::min<size_t>((size_t)ncols * per, std::max<size_t>(budget, per));
  CK(grow(&w->scratch, &w->scratch_bytes, want), "cudaMalloc(scratch)");
  if (precision == RRTMG_LW_FP64) {
    Tables<double> t{g.kt64, g.tbl64, g.tbl64 + (NTBL + 1), g.tbl64 + 2 * (NTBL + 1)};
    CK(launch_column_fp64(V, hlwb, dblk, nblocks, b0, ncols, f, g.cs, t, t, w->bits, w->scratch, w->scratch_bytes,
                          nullptr, nullptr, g.num_sms, st, ev[3]),
       "column kernels launch (fp64)");
  } else {
    Tables<float> t{g.kt32, g.tbl32, g.tbl32 + (NTBL + 1), g.tbl32 + 2 * (NTBL + 1)};
    Tables<double> t64{g.kt64, g.tbl64, g.tbl64 + (NTBL + 1), g.tbl64 + 2 * (NTBL + 1)};
    CK(launch_column_fp32(V, hlwb, dblk, nblocks, b0, ncols, f, g.cs, t, t64, w->bits, w->scratch,
                          w->scratch_bytes, nullptr, nullptr, g.num_sms, st, ev[3]),
       "column kernels launch (fp32)");
  }
  if (kernel_ms) {
    CK(cudaEventRecord(ev[2], st), "cudaEventRecord");
    CK(cudaEventSynchronize(ev[2]), "kernel execution");
    CK(cudaEventElapsedTime(&kernel_ms[0], ev[0], ev[1]), "cudaEventElapsedTime");
    CK(cudaEventElapsedTime(&kernel_ms[1], ev[1], ev[3]), "cudaEventElapsedTime");
    CK(cudaEventElapsedTime(&kernel_ms[2], ev[3], ev[2]), "cudaEventElapsedTime");
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return 0;
}

}  // namespace

extern "C" int rrtmg_lw_gpu_run_ex(const rrtmg_lw_run_args* a, const rrtmg_lw_exec* x, char* errmsg,
                                   int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: rrtmg_lw_gpu_init has not been called"); return 1; }
  rrtmg_lw_exec dflt{RRTMG_LW_FP64, RRTMG_LW_HOST, nullptr, 1, 0, nullptr};
  if (!x) x = &dflt;
  int v = validate(a, x, errmsg, errmsg_len);
  if (v == -1) return 0;
  if (v == 2) {
    // the reference zeroes cldtau before the optional-argument check (RLM:736)
    if (a->cldtau) {
      FieldSizes fs = sizes_of(a);
      if (x->memory == RRTMG_LW_DEVICE) cudaMemset(a->cldtau, 0, fs.n2 * sizeof(double));
      else std::memset(a->cldtau, 0, fs.n2 * sizeof(double));
    }
    return 1;
  }
  if (v) return 1;
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  Workspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  Flags f;
  fill_flags(a, &f);
  cudaStream_t st = x->stream ? (cudaStream_t)x->stream : w->stream;
  Workspace wl = *w;            // launch on the caller's stream if given
  wl.stream = st;

  if (x->memory == RRTMG_LW_DEVICE) {
    Block B;
    block_from_args(a, &B);
    int r = launch(&wl, &B, 1, a->npts, f, x->precision, x->kernel_ms, errmsg, errmsg_len);
    // launch() may have grown buffers
    w->bits = wl.bits; w->bits_bytes = wl.bits_bytes; w->dblocks = wl.dblocks; w->dblocks_n = wl.dblocks_n;
    w->scratch = wl.scratch; w->scratch_bytes = wl.scratch_bytes;
    w->hblocks = wl.hblocks; w->hblocks_n = wl.hblocks_n;
    if (r) return r;
    if (x->sync) CK(cudaStreamSynchronize(st), "kernel execution");
    return 0;
  }

  // host memory: stage every array through the workspace
  FieldSizes fs = sizes_of(a);
  struct Fld { const void* h; size_t n; bool out; bool in; size_t elem; };
  rrtmg_lw_run_args d = *a;   // same struct with device pointers
  const double** ins[] = {&d.plyr, &d.plvl, &d.tlyr, &d.tlvl, &d.qlyr, &d.olyr, &d.gasvmr_co2, &d.gasvmr_n2o,
                          &d.gasvmr_ch4, &d.gasvmr_o2, &d.gasvmr_co, &d.gasvmr_cfc11, &d.gasvmr_cfc12,
                          &d.gasvmr_cfc22, &d.gasvmr_ccl4, &d.aeraod, &d.aerssa, &d.sfemis, &d.sfgtmp,
                          &d.dzlyr, &d.delpin, &d.de_lgth, &d.alpha, &d.cld_cf, &d.cld_lwp, &d.cld_ref_liq,
                          &d.cld_iwp, &d.cld_ref_ice, &d.cld_rwp, &d.cld_ref_rain, &d.cld_swp,
                          &d.cld_ref_snow, &d.cld_od};
  size_t in_n[] = {fs.n2, fs.n2l, fs.n2, fs.n2l, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2,
                   fs.n2, fs.n2, fs.n3, fs.n3, fs.n1, fs.n1, fs.n2, fs.n2, fs.n1, fs.n2, fs.n2, fs.n2, fs.n2,
                   fs.n2, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2, fs.n2};
  double** outs[] = {&d.hlwc, &d.topflx, &d.sfcflx, &d.cldtau, &d.hlw0, &d.hlwb, &d.flxprf};
  size_t out_n[] = {fs.n2, 2 * fs.n1, 4 * fs.n1, fs.n2, fs.n2, fs.n3, 4 * fs.n2l};
  const int nin = sizeof(ins) / sizeof(ins[0]), nout = sizeof(outs) / sizeof(outs[0]);
  // layout the staging buffer
  size_t total = 0;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  for (int k = 0; k < nin; ++k) if (*ins[k]) total += al(in_n[k] * sizeof(double));
  for (int k = 0; k < nout; ++k) if (*outs[k]) total += al(out_n[k] * sizeof(double));
  if (d.icseed) total += al(fs.n1 * sizeof(int32_t));
  CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  CK(grow(&w->dbuf, &w->dbuf_bytes, total), "cudaMalloc(workspace)");
  char* p = w->dbuf;
  for (int k = 0; k < nin; ++k) {
    if (!*ins[k]) continue;
    size_t bytes = in_n[k] * sizeof(double);
    CK(cudaMemcpyAsync(p, *ins[k], bytes, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(H2D)");
    *ins[k] = reinterpret_cast<const double*>(p);
    p += al(bytes);
  }
  if (d.icseed) {
    size_t bytes = fs.n1 * sizeof(int32_t);
    CK(cudaMemcpyAsync(p, d.icseed, bytes, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(H2D)");
    d.icseed = reinterpret_cast<const int32_t*>(p);
    p += al(bytes);
  }
  double* host_out[N_OUT];
  for (int k = 0; k < nout; ++k) {
    host_out[k] = *outs[k];
    if (!*outs[k]) continue;
    *outs[k] = reinterpret_cast<double*>(p);
    p += al(out_n[k] * sizeof(double));
  }
  Block B;
  block_from_args(&d, &B);
  wl = *w;
  wl.stream = st;
  int r = launch(&wl, &B, 1, a->npts, f, x->precision, x->kernel_ms, errmsg, errmsg_len);
  w->bits = wl.bits; w->bits_bytes = wl.bits_bytes; w->dblocks = wl.dblocks; w->dblocks_n = wl.dblocks_n;
    w->scratch = wl.scratch; w->scratch_bytes = wl.scratch_bytes;
  w->hblocks = wl.hblocks; w->hblocks_n = wl.hblocks_n;
  if (r) return r;
  for (int k = 0; k < nout; ++k) {
    if (!host_out[k]) continue;
    CK(cudaMemcpyAsync(host_out[k], *outs[k], out_n[k] * sizeof(double), cudaMemcpyDeviceToHost, st),
       "cudaMemcpyAsync(D2H)");
  }
  CK(cudaStreamSynchronize(st), "kernel execution");
  return 0;
}

extern "C" int rrtmg_lw_gpu_run(const rrtmg_lw_run_args* a, char* errmsg, int32_t errmsg_len) {
  return rrtmg_lw_gpu_run_ex(a, nullptr, errmsg, errmsg_len);
}

extern "C" int rrtmg_lw_gpu_mcica(int32_t npts, int32_t nlay, int32_t ldim, int32_t iovr, const int32_t* seed,
                                  const double* cldf, const double* dz, const double* de_lgth,
                                  const double* alpha, uint32_t* bits, void* stream, char* errmsg,
                                  int32_t errmsg_len) {
  (void)dz; (void)de_lgth; (void)alpha;
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: rrtmg_lw_gpu_init has not been called"); return 1; }
  if (npts < 0 || nlay < 1 || nlay > 255 || (ldim != 0 && ldim < npts)) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_mcica: bad dimensions");
    return 1;
  }
  if (iovr < 0 || iovr > 2) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_mcica: overlap iovr=%d not supported (0, 1, 2 are)", iovr);
    return 1;
  }
  if (npts == 0) return 0;
  if (!seed || !cldf || !bits) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_mcica: NULL pointer"); return 1; }
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  Workspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : w->stream;
  Block none{};
  CK(mcica_launch(nullptr, 0, none, npts, nlay, iovr, 2, 0, cldf, seed, ldim > 0 ? ldim : npts, bits, g.num_sms, st),
     "McICA kernel launch");
  CK(cudaStreamSynchronize(st), "McICA kernel execution");
  return 0;
}

extern "C" int rrtmg_lw_gpu_gas_optics(const rrtmg_lw_run_args* a, int32_t precision, double* taug,
                                       double* fracs, void* stream, char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: rrtmg_lw_gpu_init has not been called"); return 1; }
  rrtmg_lw_exec x{precision, RRTMG_LW_DEVICE, stream, 1, 0, nullptr};
  rrtmg_lw_run_args a2 = *a;
  a2.lslwr = 1;
  int v = validate(&a2, &x, errmsg, errmsg_len, false);
  if (v == -1) return 0;
  if (v) return 1;
  if (!taug || !fracs) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_gas_optics: NULL output"); return 1; }
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  Workspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : w->stream;
  Flags f;
  fill_flags(&a2, &f);
  f.gas_only = 1;
  f.want_hlwb = 0;
  Block B;
  block_from_args(&a2, &B);
  const int V = pick_v(a2.nlay);
  Tables<double> t64{g.kt64, g.tbl64, g.tbl64 + (NTBL + 1), g.tbl64 + 2 * (NTBL + 1)};
  if (precision == RRTMG_LW_FP64) {
    CK(launch_column_fp64(V, false, nullptr, 1, B, a2.npts, f, g.cs, t64, t64, nullptr, nullptr, 0, taug, fracs,
                          g.num_sms, st, nullptr),
       "gas optics launch");
  } else {
    Tables<float> t{g.kt32, g.tbl32, g.tbl32 + (NTBL + 1), g.tbl32 + 2 * (NTBL + 1)};
    CK(launch_column_fp32(V, false, nullptr, 1, B, a2.npts, f, g.cs, t, t64, nullptr, nullptr, 0, taug, fracs,
                          g.num_sms, st, nullptr),
       "gas optics launch");
  }
  CK(cudaStreamSynchronize(st), "gas optics execution");
  return 0;
}

extern "C" void rrtmg_lw_gpu_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g.ready) return;
  cudaSetDevice(g.device);
  for (Workspace* w : g_workspaces) {
    if (w->stream) cudaStreamSynchronize(w->stream);
    if (w->dbuf) cudaFree(w->dbuf);
    if (w->bits) cudaFree(w->bits);
    if (w->scratch) cudaFree(w->scratch);
    if (w->dblocks) cudaFree(w->dblocks);
    if (w->hblocks) cudaFreeHost(w->hblocks);
    if (w->stream) cudaStreamDestroy(w->stream);
    delete w;
  }
  g_workspaces.clear();
  tl_ws = nullptr;
  cudaFree(g.kt64); cudaFree(g.kt32); cudaFree(g.tbl64); cudaFree(g.tbl32);
  g = DeviceState();
}

// Read-only view of the device tables for the allocation-free entry point
// (lw_noalloc.cu).
lw::NoAllocView lw::noalloc_view() {
  std::lock_guard<std::mutex> lk(g_mu);
  return NoAllocView{g.ready ? 1 : 0, g.device, g.num_sms, g.kt64, g.kt32, g.tbl64, g.tbl32, g.cs};
}
