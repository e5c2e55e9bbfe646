// Solve kernels for 8 layer(s).
#define UNB_SOLVER_LAYERS 8
#include "solver_layers.cuh"
