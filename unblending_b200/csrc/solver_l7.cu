// Solve kernels for 7 layer(s).
#define UNB_SOLVER_LAYERS 7
#include "solver_layers.cuh"
