// FP32 instantiation of the column kernel: gas optics and two-stream
// transfer in FP32 (FMA contraction allowed); setcoef interpolation weights,
// Planck integrals, cloud optics and the flux sums / flux divergence stay
// FP64 inside the kernel.
#include <algorithm>

#include "lw_column.cuh"

#define REAL float
#define LW_PREPARE_FN prepare_column_fp32
#define LW_LAUNCH_FN launch_column_fp32
#include "lw_column_launch.inc"
