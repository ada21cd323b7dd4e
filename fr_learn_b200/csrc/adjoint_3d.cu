// Adjoint kernels, 3D.
#define FRG_ADJ_DIM 3
#define FRG_ADJ_NAME 3d
#include <algorithm>
#include "adjoint_impl.cuh"
