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
#include "lw_launch.h"

extern "C" const unsigned char rrtmg_lw_tables_blob[];
extern "C" const unsigned char rrtmg_lw_tables_blob_end[];

using namespace lw;

namespace {

struct DeviceState {
  bool ready = false;
  int device = 0;
  int num_sms = 0;
  double* kt64 = nullptr;
  float* kt32 = nullptr;
  double* tbl64 = nullptr;   // records {exp, tfn, tau, 0} (4 x (NTBL+1))
  float* tbl32 = nullptr;
  Consts cs{};
  bool sgpath = false;       // the learned-gas-optics column path (lw_sg_path.cu) is usable on this device
  Shape tuned[2][9];         // autotuned launch shape per [fp32?][V]
  bool has_tuned[2][9] = {};
};
DeviceState g;
std::mutex g_mu;

struct GraphEntry;

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
  uint64_t gen = 0;           // bumped whenever bits/scratch move (graphs hold their addresses)
  int last_launches = 0;      // kernels enqueued by the thread's last run call
  // pipelined host-memory calls: copy streams, double-buffered staging, events
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
  char* pbuf = nullptr;
  size_t pbuf_bytes = 0;
  std::vector<GraphEntry*> graphs;
};

// A captured call of rrtmg_lw_gpu_run_blocks: the kernels of one block set
// with its own device copy of the block descriptors.
struct GraphEntry {
  std::vector<Block> blocks;
  Flags f;
  int precision = 0;
  Shape sh;
  int ncols = 0;
  uint64_t gen = 0;
  uint64_t last_use = 0;
  int launches = 0;           // kernels the graph holds
  Block* dblocks = nullptr;
  cudaGraphExec_t exec = nullptr;
};
constexpr size_t kMaxGraphs = 8;   // per workspace; least recently used is dropped

void drop_graph(GraphEntry* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->dblocks) cudaFree(e->dblocks);
  delete e;
}
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
  // interleave: record i = {exp_tbl(i), tfn_tbl(i), tau_tbl(i), 0}
  std::vector<double> rec(4 * (NTBL + 1), 0.0);
  for (int i = 0; i <= NTBL; ++i) {
    rec[4 * i + 0] = ex[i];
    rec[4 * i + 1] = tf[i];
    rec[4 * i + 2] = ta[i];
  }
  std::vector<float> rec32(rec.begin(), rec.end());

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
    CK(cudaMalloc(&g.tbl64, rec.size() * sizeof(double)), "cudaMalloc(tables)");
    CK(cudaMalloc(&g.tbl32, rec32.size() * sizeof(float)), "cudaMalloc(tables)");
  }
  CK(cudaMemcpy(g.kt64, kt.data(), kt.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(cudaMemcpy(g.kt32, kt32.data(), kt32.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(cudaMemcpy(g.tbl64, rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(cudaMemcpy(g.tbl32, rec32.data(), rec32.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy(tables)");
  CK(mcica_upload_powers(), "mcica powers upload");
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, g.device), "cudaDeviceGetAttribute");
  CK(mcica_prepare(optin), "kernel attributes (mcica)");
  CK(prepare_column_fp64(), "kernel attributes (column, fp64)");
  CK(prepare_column_fp32(), "kernel attributes (column, fp32)");
  g.sgpath = sg_path_prepare() == cudaSuccess;
  if (!g.sgpath) (void)cudaGetLastError();
  // No context limit is changed: every kernel's stack frame (at most 864
  // bytes per thread, -Xptxas -v) fits the default per-thread stack.
  // make the allocation-free entry point's fixed scratch resident now, before
  // a host hands the rest of the GPU's memory to its own pool; a failure here
  // is reported by that entry point's first call instead
  if (noalloc_prepare(g.device) != cudaSuccess) (void)cudaGetLastError();
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
  if (a->isubclw < 0 || a->isubclw > 2) {
    set_msg(errmsg, errmsg_len,
            "rrtmg_lw_gpu: isubclw=%d not supported (0: grid-mean clouds with rtrn/rtrnmr; 1, 2: McICA with rtrnmc)",
            a->isubclw);
    return 1;
  }
  if (a->iovr < 0 || a->iovr > 5) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: McICA overlap iovr=%d not supported (0..5 are)", a->iovr);
    return 1;
  }
  // the decorrelation-length and exponential overlaps read these (RLM:796, 820, 933)
  if (a->iovr == 3 && !a->de_lgth) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_run: iovr=3 (decorrelation length) needs de_lgth");
    return 1;
  }
  if ((a->iovr == 4 || a->iovr == 5) && !a->alpha) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_run: iovr=%d (exponential overlap) needs alpha", a->iovr);
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
  if (x && x->precision != RRTMG_LW_FP64 && x->precision != RRTMG_LW_FP32 && x->precision != RRTMG_LW_SURROGATE) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: unknown precision %d", x->precision);
    return 1;
  }
  if (x && x->precision == RRTMG_LW_SURROGATE && !surrogate_norm()) {
    set_msg(errmsg, errmsg_len,
            "rrtmg_lw_gpu: RRTMG_LW_SURROGATE needs a network (rrtmg_lw_gpu_surrogate_init/_set and _train)");
    return 1;
  }
  return 0;
}


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

// The learned gas optics runs the FP32 column kernels with the network
// stage in front: turn the surrogate precision into FP32 + flags.
int kernel_precision(int precision, Flags* f) {
  if (precision != RRTMG_LW_SURROGATE) return precision;
  f->surrogate = 1;
  f->sg_norm = surrogate_norm();
  f->sg_fallback = surrogate_fallback_counter();
  return RRTMG_LW_FP32;
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
  B->seed0 = 0;
}

// grow() for the buffers captured graphs refer to
template <typename T>
cudaError_t grow_ws(Workspace* w, T** p, size_t* have, size_t need_bytes) {
  if (*have >= need_bytes && *p) return cudaSuccess;
  ++w->gen;
  return grow(p, have, need_bytes);
}

Shape default_shape(int precision, int V) {
  const int pi = precision == RRTMG_LW_FP64 ? 0 : 1;
  return g.has_tuned[pi][V] ? g.tuned[pi][V] : Shape();
}

size_t scratch_budget() {
  size_t budget = kScratchBudget;
  if (const char* env = std::getenv("RRTMG_LW_GPU_SCRATCH_MB")) budget = (size_t)std::atol(env) << 20;
  return budget;
}

// Size the McICA flags and the kernel A -> B scratch for a call.
int reserve(Workspace* w, int ncols, const Flags& f, int precision, const Shape& sh, char* errmsg,
            int32_t errmsg_len) {
  const int nw = (f.nlay + 31) / 32;
  if (f.isubclw > 0 && !f.gas_only)
    CK(grow_ws(w, &w->bits, &w->bits_bytes, (size_t)ncols * NGPT * nw * sizeof(uint32_t)), "cudaMalloc(mcica bits)");
  if (precision != RRTMG_LW_FP64 && g.sgpath && sg_path_applies(f)) {
    // the learned-gas-optics path's work area: column map, fallback list,
    // band-field slots and the FP16 network -> transfer hand-off
    CK(grow_ws(w, &w->scratch, &w->scratch_bytes, sg_path_bytes(ncols, f.nlay, g.num_sms, scratch_budget())),
       "cudaMalloc(scratch)");
    return 0;
  }
  const int V = pick_v(f.nlay);
  const size_t per = (precision == RRTMG_LW_FP64) ? scratch_per_column_fp64(V) : scratch_per_column_fp32(V);
  size_t cols = std::min<size_t>((size_t)ncols, std::max<size_t>(scratch_budget() / per, 1));
  if (sh.chunk > 0) cols = std::min<size_t>(cols, (size_t)sh.chunk);
  CK(grow_ws(w, &w->scratch, &w->scratch_bytes, cols * per), "cudaMalloc(scratch)");
  return 0;
}

// Copy the block descriptors (nblocks > 1) to the workspace's device array.
int upload_blocks(Workspace* w, cudaStream_t st, const Block* hblocks, int nblocks, const Block** dblk,
                  char* errmsg, int32_t errmsg_len) {
  *dblk = nullptr;
  if (nblocks <= 1) return 0;
  CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");   // a previous call may still read the staging copy
  if (w->hblocks_n < (size_t)nblocks) {
    if (w->hblocks) cudaFreeHost(w->hblocks);
    w->hblocks = nullptr;
    w->hblocks_n = 0;
    CK(cudaMallocHost((void**)&w->hblocks, sizeof(Block) * nblocks), "cudaMallocHost");
    w->hblocks_n = nblocks;
  }
  std::memcpy(w->hblocks, hblocks, sizeof(Block) * nblocks);
  size_t have = w->dblocks_n * sizeof(Block);
  CK(grow(&w->dblocks, &have, sizeof(Block) * nblocks), "cudaMalloc(blocks)");
  w->dblocks_n = have / sizeof(Block);
  CK(cudaMemcpyAsync(w->dblocks, w->hblocks, sizeof(Block) * nblocks, cudaMemcpyHostToDevice, st),
     "cudaMemcpyAsync(blocks)");
  *dblk = w->dblocks;
  return 0;
}

// Enqueue the McICA and column kernels of a call (buffers already reserved).
// ev (optional, 4 events): before McICA, before gas optics, end, and after
// the first gas-optics launch.
cudaError_t enqueue(Workspace* w, cudaStream_t st, const Block* dblk, const Block& b0, int nblocks, int ncols,
                    const Flags& f, int precision, const Shape& sh, cudaEvent_t* ev) {
  cudaError_t e;
  const bool sgpath = precision != RRTMG_LW_FP64 && g.sgpath && sg_path_applies(f);
  if (sgpath) {
    // McICA, then the column map and per hand-off chunk network, fallback and transfer
    w->last_launches = 1 + sg_path_launches(ncols, f.nlay, g.num_sms, scratch_budget(), nblocks);
  } else {
    // kernels of this call: McICA, then per scratch chunk the network stage
    // (learned gas optics), gas optics and transfer
    const int V = pick_v(f.nlay);
    const int col = precision == RRTMG_LW_FP64 ? launches_column_fp64(V, ncols, w->scratch_bytes, sh)
                                                : launches_column_fp32(V, ncols, w->scratch_bytes, sh);
    w->last_launches = (f.isubclw > 0 && !f.gas_only ? 1 : 0) + col + (f.surrogate ? col / 2 : 0);
  }
  NvtxRange run_range("rrtmg_lw_run");
  if (ev && (e = cudaEventRecord(ev[0], st)) != cudaSuccess) return e;
  if (f.isubclw > 0 && !f.gas_only) {
    NvtxRange r("mcica_subcol");
    e = mcica_launch(dblk, nblocks, b0, ncols, f.nlay, f.iovr, f.isubclw, f.top_at_1, McicaStage(), w->bits,
                     g.num_sms, st);
    if (e != cudaSuccess) return e;
  }
  if (ev && (e = cudaEventRecord(ev[1], st)) != cudaSuccess) return e;
  const int V = pick_v(f.nlay);
  const bool hlwb = f.want_hlwb != 0;
  Tables<double> t64{g.kt64, g.tbl64};
  if (sgpath) {
    Tables<float> t{g.kt32, g.tbl32};
    e = sg_path_launch(dblk, nblocks, b0, ncols, f, g.cs, t, t64, w->bits, w->scratch, w->scratch_bytes,
                       scratch_budget(), g.num_sms, st);
    if (e == cudaSuccess && ev) e = cudaEventRecord(ev[3], st);
  } else if (precision == RRTMG_LW_FP64) {
    NvtxRange r("setcoef+taumol+rtrnmc (FP64)");
    e = launch_column_fp64(V, hlwb, dblk, nblocks, b0, ncols, f, g.cs, t64, t64, w->bits, w->scratch,
                           w->scratch_bytes, nullptr, nullptr, g.num_sms, sh, st, ev ? ev[3] : nullptr);
  } else {
    NvtxRange r(f.surrogate ? "learned gas optics+rtrnmc (FP32)" : "setcoef+taumol+rtrnmc (FP32)");
    Tables<float> t{g.kt32, g.tbl32};
    e = launch_column_fp32(V, hlwb, dblk, nblocks, b0, ncols, f, g.cs, t, t64, w->bits, w->scratch,
                           w->scratch_bytes, nullptr, nullptr, g.num_sms, sh, st, ev ? ev[3] : nullptr);
  }
  if (e != cudaSuccess) return e;
  if (ev && (e = cudaEventRecord(ev[2], st)) != cudaSuccess) return e;
  return cudaSuccess;
}

struct Events {
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  ~Events() { for (auto& e : ev) if (e) cudaEventDestroy(e); }
  cudaError_t create() {
    for (auto& e : ev) {
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
  }
};

int launch(Workspace* w, cudaStream_t st, const Block* hblocks, int nblocks, int ncols, const Flags& f,
           int precision, const Shape& sh, float* kernel_ms, char* errmsg, int32_t errmsg_len) {
  Events E;
  if (kernel_ms) CK(E.create(), "cudaEventCreate");
  int r = reserve(w, ncols, f, precision, sh, errmsg, errmsg_len);
  if (r) return r;
  const Block* dblk = nullptr;
  if ((r = upload_blocks(w, st, hblocks, nblocks, &dblk, errmsg, errmsg_len))) return r;
  CK(enqueue(w, st, dblk, hblocks[0], nblocks, ncols, f, precision, sh, kernel_ms ? E.ev : nullptr),
     "kernel launch");
  if (kernel_ms) {
    CK(cudaEventSynchronize(E.ev[2]), "kernel execution");
    CK(cudaEventElapsedTime(&kernel_ms[0], E.ev[0], E.ev[1]), "cudaEventElapsedTime");
    CK(cudaEventElapsedTime(&kernel_ms[1], E.ev[1], E.ev[3]), "cudaEventElapsedTime");
    CK(cudaEventElapsedTime(&kernel_ms[2], E.ev[3], E.ev[2]), "cudaEventElapsedTime");
  }
  return 0;
}

// Launch a block set through a cached CUDA graph (captured on first use).
int launch_graph(Workspace* w, cudaStream_t st, const std::vector<Block>& hb, int ncols, const Flags& f,
                 int precision, const Shape& sh, char* errmsg, int32_t errmsg_len) {
  static uint64_t tick = 0;
  int r = reserve(w, ncols, f, precision, sh, errmsg, errmsg_len);   // may move buffers: bump gen first
  if (r) return r;
  GraphEntry* hit = nullptr;
  for (size_t k = 0; k < w->graphs.size(); ++k) {
    GraphEntry* e = w->graphs[k];
    if (e->gen != w->gen) {            // refers to buffers that moved
      drop_graph(e);
      w->graphs.erase(w->graphs.begin() + k);
      --k;
      continue;
    }
    if (e->ncols == ncols && e->precision == precision && e->blocks.size() == hb.size() &&
        std::memcmp(&e->f, &f, sizeof(Flags)) == 0 && std::memcmp(&e->sh, &sh, sizeof(Shape)) == 0 &&
        std::memcmp(e->blocks.data(), hb.data(), sizeof(Block) * hb.size()) == 0) {
      hit = e;
      break;
    }
  }
  if (!hit) {
    if (w->graphs.size() >= kMaxGraphs) {
      auto lru = std::min_element(w->graphs.begin(), w->graphs.end(),
                                  [](GraphEntry* a, GraphEntry* b) { return a->last_use < b->last_use; });
      CK(cudaStreamSynchronize(st), "cudaStreamSynchronize");
      drop_graph(*lru);
      w->graphs.erase(lru);
    }
    GraphEntry* e = new GraphEntry();
    e->blocks = hb;
    e->f = f;
    e->precision = precision;
    e->sh = sh;
    e->ncols = ncols;
    e->gen = w->gen;
    const Block* dblk = nullptr;
    cudaError_t ce = cudaSuccess;
    if (hb.size() > 1) {
      ce = cudaMalloc((void**)&e->dblocks, sizeof(Block) * hb.size());
      if (ce == cudaSuccess)
        ce = cudaMemcpy(e->dblocks, hb.data(), sizeof(Block) * hb.size(), cudaMemcpyHostToDevice);
      dblk = e->dblocks;
    }
    // capture on the workspace's private stream, then launch on the caller's
    cudaGraph_t graph = nullptr;
    if (ce == cudaSuccess) ce = cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      cudaError_t ke = enqueue(w, w->stream, dblk, hb[0], (int)hb.size(), ncols, f, precision, sh, nullptr);
      ce = cudaStreamEndCapture(w->stream, &graph);
      if (ke != cudaSuccess) ce = ke;
    }
    e->launches = w->last_launches;
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      drop_graph(e);
      return cuda_fail(errmsg, errmsg_len, "CUDA graph capture", ce);
    }
    w->graphs.push_back(e);
    hit = e;
  }
  hit->last_use = ++tick;
  w->last_launches = hit->launches;
  CK(cudaGraphLaunch(hit->exec, st), "cudaGraphLaunch");
  return 0;
}

}  // namespace

namespace {

// Columns per chunk of a pipelined host-memory call (calls with fewer than two
// chunks' worth of columns run unpipelined).
constexpr int kHostChunk = 4096;

// One field of the caller's Fortran arrays: `rows` rows of `width` elements
// per column (1 = plain (ldim, rows) layout; 2 or 4 = the derived-type records
// topflx/sfcflx/flxprf) at pitch `width * ldim`; rows == 0 means a 1-D
// (npts) field.
struct HostField {
  const void* h;      // caller's array
  void** dslot;       // where the staged device pointer goes (in the run_args copy)
  int rows, width, elem;
  bool out;
};

// rrtmg_lw_run on host memory with the copies overlapped with the kernels:
// chunk j+1's inputs travel host -> device on one copy stream and chunk j-1's
// outputs device -> host on another while chunk j computes.  Staging is
// double-buffered; events order the reuse of each buffer.
int run_host_pipelined(Workspace* w, const rrtmg_lw_run_args* a, Flags f0, int precision, cudaStream_t st,
                       char* errmsg, int32_t errmsg_len) {
  const int npts = a->npts, nlay = a->nlay, nlp1 = nlay + 1;
  const size_t ld = a->ldim > 0 ? (size_t)a->ldim : (size_t)npts;
  rrtmg_lw_run_args d = *a;
  std::vector<HostField> fl;
  auto in2 = [&](const double* const* p, int rows) {
    if (*p) fl.push_back({*p, (void**)const_cast<const double**>(p), rows, 1, 8, false});
  };
  in2(&d.plyr, nlay); in2(&d.plvl, nlp1); in2(&d.tlyr, nlay); in2(&d.tlvl, nlp1); in2(&d.qlyr, nlay);
  in2(&d.olyr, nlay); in2(&d.gasvmr_co2, nlay); in2(&d.gasvmr_n2o, nlay); in2(&d.gasvmr_ch4, nlay);
  in2(&d.gasvmr_o2, nlay); in2(&d.gasvmr_co, nlay); in2(&d.gasvmr_cfc11, nlay); in2(&d.gasvmr_cfc12, nlay);
  in2(&d.gasvmr_cfc22, nlay); in2(&d.gasvmr_ccl4, nlay); in2(&d.aeraod, nlay * NBANDS);
  in2(&d.aerssa, nlay * NBANDS); in2(&d.sfemis, 0); in2(&d.sfgtmp, 0); in2(&d.dzlyr, nlay); in2(&d.delpin, nlay);
  in2(&d.de_lgth, 0); in2(&d.alpha, nlay); in2(&d.cld_cf, nlay); in2(&d.cld_lwp, nlay); in2(&d.cld_ref_liq, nlay);
  in2(&d.cld_iwp, nlay); in2(&d.cld_ref_ice, nlay); in2(&d.cld_rwp, nlay); in2(&d.cld_ref_rain, nlay);
  in2(&d.cld_swp, nlay); in2(&d.cld_ref_snow, nlay); in2(&d.cld_od, nlay);
  if (d.icseed) fl.push_back({d.icseed, (void**)const_cast<const int32_t**>(&d.icseed), 0, 1, 4, false});
  auto out = [&](double** p, int rows, int width) {
    if (*p) fl.push_back({*p, (void**)p, rows, width, 8, true});
  };
  out(&d.hlwc, nlay, 1); out(&d.topflx, 0, 2); out(&d.sfcflx, 0, 4); out(&d.cldtau, nlay, 1);
  out(&d.hlw0, nlay, 1); out(&d.hlwb, nlay * NBANDS, 1); out(&d.flxprf, nlp1, 4);
  // staging of one chunk (kHostChunk columns) and its layout
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  std::vector<size_t> off(fl.size());
  size_t per = 0;
  for (size_t k = 0; k < fl.size(); ++k) {
    off[k] = per;
    per += al((size_t)std::max(fl[k].rows, 1) * fl[k].width * kHostChunk * fl[k].elem);
  }
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
  CK(grow(&w->pbuf, &w->pbuf_bytes, 2 * per), "cudaMalloc(staging)");
  const int kp = kernel_precision(precision, &f0);
  const Shape sh = default_shape(kp, pick_v(nlay));
  const int nch = (npts + kHostChunk - 1) / kHostChunk;
  for (int j = 0; j < nch; ++j) {
    const int b = j & 1, c0 = j * kHostChunk, n = std::min(kHostChunk, npts - c0);
    char* base = w->pbuf + (size_t)b * per;
    // inputs: wait until chunk j-2 is done with this buffer
    if (j >= 2) CK(cudaStreamWaitEvent(w->h2d, w->ev_done[b], 0), "cudaStreamWaitEvent");
    for (size_t k = 0; k < fl.size(); ++k) {
      char* dptr = base + off[k];
      *fl[k].dslot = dptr;
      if (fl[k].out) continue;
      const size_t es = fl[k].elem, wdt = (size_t)fl[k].width;
      const char* hp = static_cast<const char*>(fl[k].h) + (size_t)c0 * wdt * es;
      if (fl[k].rows == 0)
        CK(cudaMemcpyAsync(dptr, hp, (size_t)n * wdt * es, cudaMemcpyHostToDevice, w->h2d), "cudaMemcpyAsync(H2D)");
      else
        CK(cudaMemcpy2DAsync(dptr, (size_t)n * wdt * es, hp, ld * wdt * es, (size_t)n * wdt * es, fl[k].rows,
                             cudaMemcpyHostToDevice, w->h2d),
           "cudaMemcpy2DAsync(H2D)");
    }
    CK(cudaEventRecord(w->ev_in[b], w->h2d), "cudaEventRecord");
    // kernels: after the inputs arrived and chunk j-2's outputs left this buffer
    CK(cudaStreamWaitEvent(st, w->ev_in[b], 0), "cudaStreamWaitEvent");
    if (j >= 2) CK(cudaStreamWaitEvent(st, w->ev_out[b], 0), "cudaStreamWaitEvent");
    rrtmg_lw_run_args dc = d;
    dc.npts = n;
    dc.ldim = n;
    Block B;
    block_from_args(&dc, &B);
    B.seed0 = c0;
    Flags f = f0;
    int r = launch(w, st, &B, 1, n, f, kp, sh, nullptr, errmsg, errmsg_len);
    if (r) return r;
    CK(cudaEventRecord(w->ev_done[b], st), "cudaEventRecord");
    // outputs back to the caller's arrays
    CK(cudaStreamWaitEvent(w->d2h, w->ev_done[b], 0), "cudaStreamWaitEvent");
    for (size_t k = 0; k < fl.size(); ++k) {
      if (!fl[k].out) continue;
      const size_t es = fl[k].elem, wdt = (size_t)fl[k].width;
      char* hp = static_cast<char*>(const_cast<void*>(fl[k].h)) + (size_t)c0 * wdt * es;
      const char* dptr = base + off[k];
      if (fl[k].rows == 0)
        CK(cudaMemcpyAsync(hp, dptr, (size_t)n * wdt * es, cudaMemcpyDeviceToHost, w->d2h), "cudaMemcpyAsync(D2H)");
      else
        CK(cudaMemcpy2DAsync(hp, ld * wdt * es, dptr, (size_t)n * wdt * es, (size_t)n * wdt * es, fl[k].rows,
                             cudaMemcpyDeviceToHost, w->d2h),
           "cudaMemcpy2DAsync(D2H)");
    }
    CK(cudaEventRecord(w->ev_out[b], w->d2h), "cudaEventRecord");
  }
  CK(cudaStreamSynchronize(w->d2h), "kernel execution");
  CK(cudaStreamSynchronize(st), "kernel execution");
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

  if (x->memory == RRTMG_LW_DEVICE) {
    Block B;
    block_from_args(a, &B);
    const int kp = kernel_precision(x->precision, &f);
    int r = launch(w, st, &B, 1, a->npts, f, kp, default_shape(kp, pick_v(f.nlay)), x->kernel_ms, errmsg,
                   errmsg_len);
    if (r) return r;
    if (x->sync) CK(cudaStreamSynchronize(st), "kernel execution");
    return 0;
  }

  // host memory, large calls: copies overlapped with the kernels, chunk by chunk
  if (a->npts >= 2 * kHostChunk && !x->kernel_ms) return run_host_pipelined(w, a, f, x->precision, st, errmsg, errmsg_len);

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
  const int kp = kernel_precision(x->precision, &f);
  int r = launch(w, st, &B, 1, a->npts, f, kp, default_shape(kp, pick_v(f.nlay)), x->kernel_ms, errmsg,
                 errmsg_len);
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
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: rrtmg_lw_gpu_init has not been called"); return 1; }
  if (npts < 0 || nlay < 1 || nlay > 255 || (ldim != 0 && ldim < npts)) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_mcica: bad dimensions");
    return 1;
  }
  if (iovr < 0 || iovr > 5) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_mcica: overlap iovr=%d not supported (0..5 are)", iovr);
    return 1;
  }
  if ((iovr == 3 && (!dz || !de_lgth)) || (iovr >= 4 && !alpha)) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_mcica: iovr=%d needs %s", iovr, iovr == 3 ? "dz and de_lgth" : "alpha");
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
  McicaStage stg;
  stg.cldf = cldf;
  stg.seed = seed;
  stg.dz = dz;
  stg.delg = de_lgth;
  stg.alpha = alpha;
  stg.ld = ldim > 0 ? ldim : npts;
  CK(mcica_launch(nullptr, 0, none, npts, nlay, iovr, 2, 0, stg, bits, g.num_sms, st),
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
  Tables<double> t64{g.kt64, g.tbl64};
  if (precision == RRTMG_LW_FP64) {
    CK(launch_column_fp64(V, false, nullptr, 1, B, a2.npts, f, g.cs, t64, t64, nullptr, nullptr, 0, taug, fracs,
                          g.num_sms, Shape(), st, nullptr),
       "gas optics launch");
  } else {
    Tables<float> t{g.kt32, g.tbl32};
    CK(launch_column_fp32(V, false, nullptr, 1, B, a2.npts, f, g.cs, t, t64, nullptr, nullptr, 0, taug, fracs,
                          g.num_sms, Shape(), st, nullptr),
       "gas optics launch");
  }
  CK(cudaStreamSynchronize(st), "gas optics execution");
  return 0;
}

// ---------------------------------------------------------------------------
namespace {

// Validate a block set for run_blocks / autotune and build its descriptors
// (empty blocks dropped, col0 = prefix sums).  Returns -1 if nothing to do.
int build_block_set(const rrtmg_lw_run_args* blocks, int32_t nblocks, const rrtmg_lw_exec* x, int64_t max_cols,
                    std::vector<Block>* hb, Flags* f, int* ncols, char* errmsg, int32_t errmsg_len) {
  if (nblocks < 0 || (nblocks > 0 && !blocks)) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_blocks: bad block array");
    return 1;
  }
  if (x->memory != RRTMG_LW_DEVICE) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_blocks: every block must be in device memory (RRTMG_LW_DEVICE)");
    return 1;
  }
  hb->clear();
  long total = 0;
  bool have_flags = false;
  for (int b = 0; b < nblocks; ++b) {
    int v = validate(&blocks[b], x, errmsg, errmsg_len);
    if (v == -1) continue;
    if (v) {
      char tmp[400];
      std::snprintf(tmp, sizeof(tmp), "%s", errmsg ? errmsg : "");
      set_msg(errmsg, errmsg_len, "block %d: %s", b, tmp);
      return 1;
    }
    Flags fb;
    fill_flags(&blocks[b], &fb);
    if (!have_flags) {
      *f = fb;
      have_flags = true;
    } else if (std::memcmp(&fb, f, sizeof(Flags)) != 0) {
      set_msg(errmsg, errmsg_len,
              "rrtmg_lw_gpu_run_blocks: block %d differs from block 0 in nlay, flags or optional outputs", b);
      return 1;
    }
    if (total + blocks[b].npts > (long)INT32_MAX) {
      set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_blocks: more than 2^31-1 columns");
      return 1;
    }
    Block B;
    block_from_args(&blocks[b], &B);
    B.col0 = (int)total;
    total += blocks[b].npts;
    hb->push_back(B);
    if (max_cols > 0 && total >= max_cols) break;
  }
  *ncols = (int)total;
  return hb->empty() ? -1 : 0;
}

}  // namespace

extern "C" int rrtmg_lw_gpu_run_blocks(const rrtmg_lw_run_args* blocks, int32_t nblocks, const rrtmg_lw_exec* x,
                                       const rrtmg_lw_tuning* tune, char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: rrtmg_lw_gpu_init has not been called"); return 1; }
  rrtmg_lw_exec dflt{RRTMG_LW_FP64, RRTMG_LW_DEVICE, nullptr, 1, 0, nullptr};
  if (!x) x = &dflt;
  std::vector<Block> hb;
  Flags f;
  int ncols = 0;
  int v = build_block_set(blocks, nblocks, x, 0, &hb, &f, &ncols, errmsg, errmsg_len);
  if (v == -1) return 0;
  if (v) return 1;
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  Workspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = x->stream ? (cudaStream_t)x->stream : w->stream;
  const int kp = kernel_precision(x->precision, &f);
  Shape sh = default_shape(kp, pick_v(f.nlay));
  bool graph = false;
  if (tune) {
    if (tune->rt_warps) sh.rt_warps = tune->rt_warps;
    if (tune->gas_per_sm) sh.gas_per_sm = tune->gas_per_sm;
    if (tune->chunk_cols) sh.chunk = tune->chunk_cols;
    graph = tune->use_graph != 0;
  }
  if (sh.rt_warps != 1 && sh.rt_warps != 2 && sh.rt_warps != 4) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_blocks: rt_warps must be 1, 2 or 4 (got %d)", sh.rt_warps);
    return 1;
  }
  if (sh.gas_per_sm < 0 || sh.chunk < 0) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_blocks: negative tuning value");
    return 1;
  }
  int r = graph ? launch_graph(w, st, hb, ncols, f, kp, sh, errmsg, errmsg_len)
                : launch(w, st, hb.data(), (int)hb.size(), ncols, f, kp, sh, x->kernel_ms, errmsg, errmsg_len);
  if (r) return r;
  if (x->sync) CK(cudaStreamSynchronize(st), "kernel execution");
  return 0;
}

extern "C" int rrtmg_lw_gpu_autotune(const rrtmg_lw_run_args* blocks, int32_t nblocks, int32_t precision,
                                     void* stream, int64_t sample_cols, rrtmg_lw_tuning* best, float* best_ms,
                                     char* errmsg, int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (!g.ready) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu: rrtmg_lw_gpu_init has not been called"); return 1; }
  rrtmg_lw_exec x{precision, RRTMG_LW_DEVICE, stream, 1, 0, nullptr};
  std::vector<Block> hb;
  Flags f;
  int ncols = 0;
  int v = build_block_set(blocks, nblocks, &x, sample_cols, &hb, &f, &ncols, errmsg, errmsg_len);
  if (v == -1) { set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_autotune: no columns to tune on"); return 1; }
  if (v) return 1;
  CK(cudaSetDevice(g.device), "cudaSetDevice");
  int rc = 0;
  Workspace* w = workspace(errmsg, errmsg_len, &rc);
  if (!w) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : w->stream;
  const int V = pick_v(f.nlay);
  precision = kernel_precision(precision, &f);
  // candidates: transfer CTA of 1, 2, 4 columns x hand-off chunk (all, 1/2, 1/4 of the columns)
  std::vector<Shape> cands;
  for (int wv : {4, 2, 1})
    for (long ch : {0L, (long)(ncols + 1) / 2, (long)(ncols + 3) / 4}) {
      if (ch > 0 && ch < 1024) continue;
      Shape s;
      s.rt_warps = wv;
      s.chunk = ch;
      cands.push_back(s);
    }
  Events E;
  CK(E.create(), "cudaEventCreate");
  float best_t = -1.f;
  Shape best_s;
  for (const Shape& s : cands) {
    int r = launch(w, st, hb.data(), (int)hb.size(), ncols, f, precision, s, nullptr, errmsg, errmsg_len);   // warm
    if (r) return r;
    CK(cudaEventRecord(E.ev[0], st), "cudaEventRecord");
    for (int rep = 0; rep < 2; ++rep)
      if ((r = launch(w, st, hb.data(), (int)hb.size(), ncols, f, precision, s, nullptr, errmsg, errmsg_len)))
        return r;
    CK(cudaEventRecord(E.ev[1], st), "cudaEventRecord");
    CK(cudaEventSynchronize(E.ev[1]), "kernel execution");
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, E.ev[0], E.ev[1]), "cudaEventElapsedTime");
    ms *= 0.5f;
    if (best_t < 0.f || ms < best_t) {
      best_t = ms;
      best_s = s;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const int pi = precision == RRTMG_LW_FP64 ? 0 : 1;
    g.tuned[pi][V] = best_s;
    g.has_tuned[pi][V] = true;
  }
  if (best) {
    best->rt_warps = best_s.rt_warps;
    best->gas_per_sm = best_s.gas_per_sm;
    best->chunk_cols = (int32_t)best_s.chunk;
    best->use_graph = 0;
  }
  if (best_ms) *best_ms = best_t;
  return 0;
}

// Sets (or with t == NULL clears) the default launch shape of later calls
// with this layer count and precision, as rrtmg_lw_gpu_autotune does after
// timing: a host that keeps the autotuner's choice (per layer count,
// precision and GPU) restores it without re-timing.
extern "C" int rrtmg_lw_gpu_set_tuning(int32_t nlay, int32_t precision, const rrtmg_lw_tuning* t, char* errmsg,
                                       int32_t errmsg_len) {
  set_msg(errmsg, errmsg_len, "");
  if (nlay < 1 || nlay > 255) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_set_tuning: nlay must be 1..255 (got %d)", nlay);
    return 1;
  }
  if (precision != RRTMG_LW_FP64 && precision != RRTMG_LW_FP32 && precision != RRTMG_LW_SURROGATE) {
    set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_set_tuning: unknown precision %d", precision);
    return 1;
  }
  Shape s;
  if (t) {
    if (t->rt_warps) s.rt_warps = t->rt_warps;
    if (t->gas_per_sm) s.gas_per_sm = t->gas_per_sm;
    if (t->chunk_cols) s.chunk = t->chunk_cols;
    if (s.rt_warps != 1 && s.rt_warps != 2 && s.rt_warps != 4) {
      set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_set_tuning: rt_warps must be 1, 2 or 4 (got %d)", s.rt_warps);
      return 1;
    }
    if (s.gas_per_sm < 0 || s.chunk < 0) {
      set_msg(errmsg, errmsg_len, "rrtmg_lw_gpu_set_tuning: negative tuning value");
      return 1;
    }
  }
  std::lock_guard<std::mutex> lk(g_mu);
  const int pi = precision == RRTMG_LW_FP64 ? 0 : 1, V = pick_v(nlay);
  g.tuned[pi][V] = s;
  g.has_tuned[pi][V] = t != nullptr;
  return 0;
}

extern "C" int32_t rrtmg_lw_gpu_last_launch_count(void) { return tl_ws ? tl_ws->last_launches : 0; }

extern "C" void rrtmg_lw_gpu_finalize(void) {
  lw::prep_release();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g.ready) return;
  cudaSetDevice(g.device);
  for (Workspace* w : g_workspaces) {
    if (w->stream) cudaStreamSynchronize(w->stream);
    for (GraphEntry* e : w->graphs) drop_graph(e);
    w->graphs.clear();
    if (w->dbuf) cudaFree(w->dbuf);
    if (w->pbuf) cudaFree(w->pbuf);
    if (w->h2d) cudaStreamDestroy(w->h2d);
    if (w->d2h) cudaStreamDestroy(w->d2h);
    for (int k = 0; k < 2; ++k) {
      if (w->ev_in[k]) cudaEventDestroy(w->ev_in[k]);
      if (w->ev_done[k]) cudaEventDestroy(w->ev_done[k]);
      if (w->ev_out[k]) cudaEventDestroy(w->ev_out[k]);
    }
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

int lw::run_args_check(const rrtmg_lw_run_args* a, const rrtmg_lw_exec* x, char* errmsg, int32_t errmsg_len,
                       bool need_outputs) {
  return validate(a, x, errmsg, errmsg_len, need_outputs);
}
void lw::flags_from_args(const rrtmg_lw_run_args* a, Flags* f) { fill_flags(a, f); }
void lw::block_from_run_args(const rrtmg_lw_run_args* a, Block* B) { block_from_args(a, B); }
Shape lw::launch_shape(int precision, int V) {
  std::lock_guard<std::mutex> lk(g_mu);
  return default_shape(precision, V);
}

// Device of the steps either side of the run (lw_prep.cu): the init device,
// or -1 before init.
int lw::selected_device() {
  std::lock_guard<std::mutex> lk(g_mu);
  return g.ready ? g.device : -1;
}
