// Solve kernels for 1 layer(s).
#define UNB_SOLVER_LAYERS 1
#include "solver_layers.cuh"
