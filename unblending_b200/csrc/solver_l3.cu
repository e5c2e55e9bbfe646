// Solve kernels for 3 layer(s).
#define UNB_SOLVER_LAYERS 3
#include "solver_layers.cuh"
