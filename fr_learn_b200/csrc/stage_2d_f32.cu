// Stage, trace and wave-speed kernels for 2D, f32 arithmetic and storage.
#define FRG_UNIT_DIM 2
#define FRG_UNIT_R float
#define FRG_UNIT_S float
#define FRG_UNIT_NAME 2d_f32
#include "stage_impl.cuh"
