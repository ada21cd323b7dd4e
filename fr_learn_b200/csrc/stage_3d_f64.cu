// Stage, trace and wave-speed kernels for 3D, f64 arithmetic and storage.
#define FRG_UNIT_DIM 3
#define FRG_UNIT_R double
#define FRG_UNIT_S double
#define FRG_UNIT_NAME 3d_f64
#include "stage_impl.cuh"
