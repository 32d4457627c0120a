// FP32 instantiation of the column kernel: gas optics and two-stream
// transfer in FP32 (FMA contraction allowed); setcoef interpolation weights,
// Planck integrals, cloud optics and the flux sums / flux divergence stay
// FP64 inside the kernel.
#include <algorithm>
#include <cstdio>

#include <type_traits>

#include "lw_launch.h"
#include "lw_rt.cuh"
#include "lw_rt_grid.cuh"

#define REAL float
#define LW_SCRATCH_FN scratch_per_column_fp32
#define LW_LAUNCH_FN launch_column_fp32
#define LW_PREPARE_FN prepare_column_fp32
#define LW_NLAUNCH_FN launches_column_fp32
#define LW_DBG_FN rrtmg_lw_gpu_debug_read_fp32
#include "lw_column_launch.inc"
