// Solve kernels for 4 layer(s).
#define UNB_SOLVER_LAYERS 4
#include "solver_layers.cuh"
