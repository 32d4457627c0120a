// FP64 instantiation of the column kernel.  Built with -fmad=false so that
// every multiply and add rounds separately, in the order of the Fortran.
#include <algorithm>
#include <cstdio>

#include <type_traits>

// FP64 gas optics runs fastest with its g-point loops unrolled by two (B200,
// 16,384 columns x 127 layers: 5.5 ms against 6.1 rolled and 6.3 fully unrolled).
#define LW_GLOOP_N 2

#include "lw_launch.h"
#include "lw_rt.cuh"
#include "lw_rt_grid.cuh"

#define REAL double
#define LW_SCRATCH_FN scratch_per_column_fp64
#define LW_LAUNCH_FN launch_column_fp64
#define LW_PREPARE_FN prepare_column_fp64
#define LW_NLAUNCH_FN launches_column_fp64
#define LW_DBG_FN rrtmg_lw_gpu_debug_read_fp64
#include "lw_column_launch.inc"
