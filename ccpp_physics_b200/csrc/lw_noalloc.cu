// lw_noalloc.cu -- rrtmg_lw_run on device memory without any allocation.
//
// Some hosts cannot let a library allocate device memory during a run:
// models that hand (nearly) all of the GPU's memory to their own pool
// allocator at start-up, so a cudaMalloc from a physics scheme fails or
// fragments their arena, and time-step loops that must not call cudaMalloc
// or cudaFree because those calls synchronize the whole device.  For them,
// rrtmg_lw_gpu_run_noalloc runs the same McICA, gas-optics and transfer
// kernels as rrtmg_lw_gpu_run_ex, with the same argument checks, flags and
// launch shape, but the kernels' scratch (the McICA sub-column flags and the
// gas-optics -> transfer hand-off) lives in one fixed array compiled into the
// library instead of in memory allocated at run time.  The caller still owns
// and passes every input and output array.
//
// Limits and rules of use:
//   * the scratch array is kNoAllocScratchBytes (64 MiB) per GPU, held by
//     every GPU that loads the library until the process exits; a call whose
//     columns do not fit is rejected with an error that states the maximum
//     (about 190 columns of 127 layers in FP64, about 380 in FP32);
//   * McICA sub-columns (isubclw 1 or 2) with the overlaps iovr 0, 1 and 2
//     only: the decorrelation-length and exponential overlaps (iovr 3..5)
//     and grid-mean clouds (isubclw 0) are refused with an error;
//   * all calls share the one array, so two calls that overlap on the GPU
//     (different streams or host threads without ordering) race on it and
//     corrupt each other's results: order them on one stream or serialize;
//   * nothing in the array has to start at zero: every scratch element a
//     kernel reads was written earlier in the same call (the transfer
//     kernel reads only the layers, g-points and columns that the
//     gas-optics kernel wrote, and the sub-column flags only of the columns
//     the McICA kernel flagged cloudy), so no clearing is done;
//   * rrtmg_lw_gpu_init looks up the device address of the array on its
//     device (cudaGetSymbolAddress, with that device current), which loads the
//     array there: call init before the host hands the GPU's free memory to
//     its own pool.  If that look-up failed at init, the first call on the
//     device repeats it; make that first call before any stream capture.
//   * the caller's current device is restored before return.
// This entry point has no counterpart in the reference.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/rrtmg_lw_gpu.h"
#include "lw_common.cuh"

#include "lw_launch.h"

using namespace lw;

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;   // 64 MiB per GPU

// The scratch itself: a fixed device array, resident on a device once its
// module is loaded there (rrtmg_lw_gpu_init forces that load).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

void msg(char* errmsg, int32_t len, const char* fmt, ...) {
  if (!errmsg || len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(errmsg, (size_t)len, fmt, ap);
  va_end(ap);
}

// Device address of g_noalloc_scratch on `device` (current), looked up once.
cudaError_t scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

// Restores the caller's current device when the call returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; }
  ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

}  // namespace

cudaError_t lw::noalloc_prepare(int device) {
  void* p = nullptr;
  return scratch_address(device, &p);
}

extern "C" int rrtmg_lw_gpu_run_noalloc(const rrtmg_lw_run_args* a, int32_t precision, void* stream,
                                        char* errmsg, int32_t errmsg_len) {
  msg(errmsg, errmsg_len, "");
  const NoAllocView v = noalloc_view();
  if (!v.ready) { msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: rrtmg_lw_gpu_init has not been called"); return 1; }
  if (precision != RRTMG_LW_FP64 && precision != RRTMG_LW_FP32) {
    msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: precision %d not available (FP64 and FP32 are)", precision);
    return 1;
  }
  DeviceGuard guard;
  // the checks of the regular entry point (rrtmg_lw_gpu_run_ex), device memory
  const rrtmg_lw_exec x{precision, RRTMG_LW_DEVICE, stream, 1, 0, nullptr};
  const int chk = run_args_check(a, &x, errmsg, errmsg_len, true);
  if (chk == -1) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (chk == 2) {
    // the reference zeroes cldtau before the optional-argument check (RLM:736)
    if (a->cldtau && cudaSetDevice(v.device) == cudaSuccess) {
      const size_t ld = a->ldim > 0 ? (size_t)a->ldim : (size_t)a->npts;
      if (cudaMemsetAsync(a->cldtau, 0, ld * a->nlay * sizeof(double), st) == cudaSuccess)
        cudaStreamSynchronize(st);
    }
    return 1;
  }
  if (chk) return 1;
  if (a->isubclw != 1 && a->isubclw != 2) {
    msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: isubclw=%d not supported (1, 2 are)", a->isubclw);
    return 1;
  }
  if (a->iovr < 0 || a->iovr > 2) {
    msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: overlap iovr=%d not supported (0, 1, 2 are)", a->iovr);
    return 1;
  }

  // scratch needed: McICA flags, then the per-column hand-off of the kernels
  const int V = pick_v(a->nlay);
  const size_t nw = (size_t)(a->nlay + 31) / 32;
  const size_t bits_bytes = (((size_t)a->npts * NGPT * nw * sizeof(uint32_t)) + 255) & ~(size_t)255;
  const size_t per = (precision == RRTMG_LW_FP64) ? scratch_per_column_fp64(V) : scratch_per_column_fp32(V);
  if (bits_bytes + (size_t)a->npts * per > kNoAllocScratchBytes) {
    const size_t per_all = per + NGPT * nw * sizeof(uint32_t);
    msg(errmsg, errmsg_len,
        "rrtmg_lw_gpu_run_noalloc: %d columns of %d layers need %zu bytes of scratch; the fixed scratch holds "
        "%zu bytes, i.e. at most %zu columns at this layer count and precision",
        a->npts, a->nlay, bits_bytes + (size_t)a->npts * per, kNoAllocScratchBytes,
        (kNoAllocScratchBytes - 256) / per_all);
    return 1;
  }

  cudaError_t e = cudaSetDevice(v.device);
  if (e != cudaSuccess) { msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: cudaSetDevice: %s", cudaGetErrorString(e)); return 1; }
  void* base = nullptr;
  if ((e = scratch_address(v.device, &base)) != cudaSuccess) {
    msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    return 1;
  }
  uint32_t* bits = static_cast<uint32_t*>(base);
  void* scratch = static_cast<unsigned char*>(base) + bits_bytes;
  const size_t scratch_bytes = kNoAllocScratchBytes - bits_bytes;

  Block B;
  block_from_run_args(a, &B);
  Flags f;
  flags_from_args(a, &f);
  const Shape sh = launch_shape(precision, V);

  e = mcica_launch(nullptr, 1, B, a->npts, a->nlay, a->iovr, a->isubclw, f.top_at_1, McicaStage(), bits,
                   v.num_sms, st);
  if (e == cudaSuccess) {
    if (precision == RRTMG_LW_FP64) {
      Tables<double> t{v.kt64, v.tbl64};
      e = launch_column_fp64(V, f.want_hlwb != 0, nullptr, 1, B, a->npts, f, v.cs, t, t, bits, scratch,
                             scratch_bytes, nullptr, nullptr, v.num_sms, sh, st, nullptr);
    } else {
      Tables<float> t{v.kt32, v.tbl32};
      Tables<double> t64{v.kt64, v.tbl64};
      e = launch_column_fp32(V, f.want_hlwb != 0, nullptr, 1, B, a->npts, f, v.cs, t, t64, bits, scratch,
                             scratch_bytes, nullptr, nullptr, v.num_sms, sh, st, nullptr);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    msg(errmsg, errmsg_len, "rrtmg_lw_gpu_run_noalloc: kernels failed: %s", cudaGetErrorString(e));
    return 1;
  }
  return 0;
}
