// Solve kernels for 2 layer(s).
#define UNB_SOLVER_LAYERS 2
#include "solver_layers.cuh"
