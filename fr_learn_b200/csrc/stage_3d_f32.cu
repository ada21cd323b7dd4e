// Stage, trace and wave-speed kernels for 3D, f32 arithmetic and storage.
#define FRG_UNIT_DIM 3
#define FRG_UNIT_R float
#define FRG_UNIT_S float
#define FRG_UNIT_NAME 3d_f32
#include "stage_impl.cuh"
