// Shared definitions of the B200 unblending kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace unb {

constexpr int kMaxLayers = 8;       // compiled layer counts 1..8
constexpr int kHistory = 6;         // L-BFGS memory (augmented_lagrangian.cuh:164)

// Layer descriptors in the solver's arithmetic type, passed by value as a
// kernel parameter (lives in the constant bank, no global state).
template <class T> struct Models {
    T mean[kMaxLayers][3];
    T prec[kMaxLayers][9];
    int mode[kMaxLayers];
    int X[kMaxLayers], Y[kMaxLayers], Z[kMaxLayers];
};

// Solver controls of augmented_lagrangian.cuh:163-167 (history fixed at 6).
struct SolverControls {
    int inner = 256, outer = 22, starts = 1;
    double inner_tolerance = 5e-3, outer_tolerance = 5e-3;
    int gradient_on_first_trial = 1;   // fuse the first line-search trial's gradient
};

// Everything one solve launch reads and writes. Device pointers only.
//   image    : f64 interleaved RGB, pixel i at image[3*i .. 3*i+2]
//   first    : refinement only, first pass packed f64 [l][i][RGBA]
//   targets  : refinement only, planar f64 [(L+3)][n]: filtered alphas then
//              the background RGB used when smoothing
//   out      : packed f64 [l][i][RGBA]
//   list     : optional pixel list (count in *list_count); null = all n
struct SolveArgs {
    int n = 0;
    const double* image = nullptr;
    const double* first = nullptr;
    const double* targets = nullptr;
    double* out = nullptr;
    int32_t* status = nullptr;         // per pixel: 0 ok, 3 misses the feasibility tolerance
    uint32_t* counters = nullptr;      // per pixel: values, gradients, iterations, backtracks, outer
    const int32_t* list = nullptr;
    const int32_t* list_count = nullptr;
    int32_t* miss_list = nullptr;      // pixels whose FP64-checked constraint norm misses tolerance
    int32_t* miss_count = nullptr;
    uint32_t* queue = nullptr;         // work-queue head (zeroed before launch)
    const int32_t* input_status = nullptr;  // refinement: nonzero = targets not normalizable (status 8, not solved)
    int32_t* input_failed = nullptr;        // count of such pixels
    int opaque = 1, smooth = 0;
};

}  // namespace unb
