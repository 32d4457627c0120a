// lw_launch.h -- host-side launchers of the column kernels, shared by the
// entry points (lw_api.cu, lw_noalloc.cu).  Every launcher only enqueues
// work on the given stream.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include "../../include/rrtmg_lw_gpu.h"
#include "lw_common.cuh"

namespace lw {

// NVTX range around the enqueue of one stage of the path (named after the
// reference routine it replaces), so a profiler's timeline groups the
// kernels by stage; without a profiler attached it costs one check.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

size_t scratch_per_column_fp64(int V);
size_t scratch_per_column_fp32(int V);
cudaError_t prepare_column_fp64();
cudaError_t prepare_column_fp32();
int launches_column_fp64(int V, int ncols, size_t scratch_bytes, const Shape& sh);
int launches_column_fp32(int V, int ncols, size_t scratch_bytes, const Shape& sh);
cudaError_t launch_column_fp64(int V, bool hlwb, const Block* blocks, int nblocks, const Block& b0, int ncols,
                               const Flags& f, const Consts& cs, const Tables<double>& tab,
                               const Tables<double>& tab64, const uint32_t* bits, void* scratch,
                               size_t scratch_bytes, double* gas_taug, double* gas_fracs, int num_sms,
                               const Shape& sh, cudaStream_t st, cudaEvent_t ev_mid);
cudaError_t launch_column_fp32(int V, bool hlwb, const Block* blocks, int nblocks, const Block& b0, int ncols,
                               const Flags& f, const Consts& cs, const Tables<float>& tab,
                               const Tables<double>& tab64, const uint32_t* bits, void* scratch,
                               size_t scratch_bytes, double* gas_taug, double* gas_fracs, int num_sms,
                               const Shape& sh, cudaStream_t st, cudaEvent_t ev_mid);
cudaError_t mcica_upload_powers();
cudaError_t mcica_prepare(int max_smem);
// inputs of the McICA stage entry point (layer arrays [column + ld * layer], internal order)
struct McicaStage {
  const double* cldf = nullptr;
  const int32_t* seed = nullptr;
  const double* dz = nullptr;      // iovr 3
  const double* delg = nullptr;    // iovr 3, per column
  const double* alpha = nullptr;   // iovr 4, 5
  int ld = 0;
};
cudaError_t mcica_launch(const Block* blocks, int nblocks, const Block& b0, int ncols, int nlay, int iovr,
                         int isubclw, int top_at_1, const McicaStage& stage, uint32_t* bits, int num_sms,
                         cudaStream_t st);
// shortwave McICA sub-columns (lw_mcica.cu), stage inputs, iovr 0..2:
// bits[(c*112 + ig)*nw + (k >> 5)] bit (k & 31)
cudaError_t mcica_sw_launch(int ncols, int nlay, int iovr, const McicaStage& stage, uint32_t* bits, int num_sms,
                            cudaStream_t st);
// the same for iovr 3..5 (two g-major sets); stage.alpha = fac_lcf (iovr 3) or alpha (4, 5) per layer
cudaError_t mcica_sw_two_set_prepare(int max_smem);
cudaError_t mcica_sw_two_set_launch(int ncols, int nlay, int iovr, const McicaStage& stage, uint32_t* bits,
                                    int num_sms, cudaStream_t st);
// raw state words of one twister stream (lw_mcica.cu): raw[j] is what draw j tempers
cudaError_t seed_stream_launch(int32_t seed, long long m, uint32_t* raw, cudaStream_t st);
// icsdsw/icsdlw of n columns from the raw words of a face's stream
// (lw_mcica.cu); *bad receives the smallest column whose grid index is outside
// the face
cudaError_t seed_gather_launch(const uint32_t* raw, const int32_t* imap, const int32_t* jmap, int n, int isc,
                               int jsc, int cnx, long long face, int32_t imax, int32_t* icsdsw, int32_t* icsdlw,
                               int* bad, cudaStream_t st);

// learned gas optics (lw_mlp.cu): network stage of a chunk, its
// normalisation/envelope (nullptr until a network is loaded) and the
// fallback counter
cudaError_t mlp_lw_launch(const Block* blocks, int nblocks, const Block& b0, int nc, const Flags& f,
                          const Scratch<float>& sc, int num_sms, cudaStream_t st);
const float* surrogate_norm();
// network stage of the learned-gas-optics column path: the FP16 hand-off
// [nc][nlay/8][{tau, frac} x 140][8 layers] of chunk columns [c0, c0 + nc)
// and the list of its columns with a layer outside the training envelope
// (lw_mlp.cu); `pack` holds kSgPackBytes per chunk column for the packed
// network inputs (two launches: input packing, network)
constexpr size_t kSgPackBytes = 6656;
cudaError_t mlp_h_launch(const Block* blocks, int nblocks, const Block& b0, const int* colmap, int c0, int nc,
                         const Flags& f, __half* hnd, unsigned int* fb_flag, int* fb_list, int* fb_count,
                         unsigned char* pack, int num_sms, cudaStream_t st);
// the learned-gas-optics column path (lw_sg_path.cu): network, fallback for
// out-of-envelope layers and the g-point-per-lane transfer, per chunk of
// columns; used for McICA calls of up to 127 layers without hlwb.  Work-area
// size, launch count and launcher take the same (ncols, nlay, SMs, budget).
bool sg_path_applies(const Flags& f);
size_t sg_path_bytes(int ncols, int nlay, int num_sms, size_t budget);
int sg_path_launches(int ncols, int nlay, int num_sms, size_t budget, int nblocks);
cudaError_t sg_path_prepare();
cudaError_t sg_path_launch(const Block* blocks, int nblocks, const Block& b0, int ncols, const Flags& f,
                           const Consts& cs, const Tables<float>& tab, const Tables<double>& tab64,
                           const uint32_t* bits, void* work, size_t work_bytes, size_t budget, int num_sms,
                           cudaStream_t st);
unsigned int* surrogate_fallback_counter();

// device chosen by rrtmg_lw_gpu_init, -1 before init (lw_api.cu)
int selected_device();
// device chosen by rrtmg_sw_gpu_init, -1 before init (sw_api.cu)
int sw_selected_device();
// frees the device scratch of the steps either side of the run (lw_prep.cu)
void prep_release();

// layers per lane of the column kernels (NLP = 32 V padded layers)
inline int pick_v(int nlay) { return nlay <= 63 ? 2 : nlay <= 127 ? 4 : 8; }

// Argument handling shared by the entry points of lw_api.cu and lw_noalloc.cu.
// run_args_check: the error checks of rrtmg_lw_run (RLM:713-760); returns 0,
// 1 (error), 2 (a required optional cloud input is missing: the caller zeroes
// cldtau first, RLM:736) or -1 (nothing to do: lslwr false or npts == 0).
int run_args_check(const rrtmg_lw_run_args* a, const rrtmg_lw_exec* x, char* errmsg, int32_t errmsg_len,
                   bool need_outputs);
void flags_from_args(const rrtmg_lw_run_args* a, Flags* f);
void block_from_run_args(const rrtmg_lw_run_args* a, Block* B);
// launch shape of the column kernels: the autotuned one for (precision, V) if
// rrtmg_lw_gpu_autotune ran, else the defaults
Shape launch_shape(int precision, int V);
// device tables and constants written by rrtmg_lw_gpu_init (lw_api.cu)
struct NoAllocView {
  int ready, device, num_sms;
  const double* kt64;
  const float* kt32;
  const double* tbl64;
  const float* tbl32;
  Consts cs;
};
NoAllocView noalloc_view();
// looks up the device address of the allocation-free entry point's fixed
// scratch array on `device` (current), which loads the module that holds it
// (lw_noalloc.cu); rrtmg_lw_gpu_init calls it so the array is resident from
// init on
cudaError_t noalloc_prepare(int device);

}  // namespace lw
