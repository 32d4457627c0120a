// FP64 instantiation of the column kernel.  Built with -fmad=false so that
// every multiply and add rounds separately, in the order of the Fortran.
#include <algorithm>

#include "lw_column.cuh"

#define REAL double
#define LW_PREPARE_FN prepare_column_fp64
#define LW_LAUNCH_FN launch_column_fp64
#include "lw_column_launch.inc"
