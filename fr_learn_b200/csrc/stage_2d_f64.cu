// Stage, trace and wave-speed kernels for 2D, f64 arithmetic and storage.
#define FRG_UNIT_DIM 2
#define FRG_UNIT_R double
#define FRG_UNIT_S double
#define FRG_UNIT_NAME 2d_f64
#include "stage_impl.cuh"
