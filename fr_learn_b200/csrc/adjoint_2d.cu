// Adjoint kernels, 2D.
#define FRG_ADJ_DIM 2
#define FRG_ADJ_NAME 2d
#include <algorithm>
#include "adjoint_impl.cuh"
