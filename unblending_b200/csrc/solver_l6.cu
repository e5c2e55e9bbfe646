// Solve kernels for 6 layer(s).
#define UNB_SOLVER_LAYERS 6
#include "solver_layers.cuh"
