// Solve kernels for 5 layer(s).
#define UNB_SOLVER_LAYERS 5
#include "solver_layers.cuh"
