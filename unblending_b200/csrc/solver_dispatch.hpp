// Host-side entry points of the compiled solve and filter kernels.
#pragma once
#include "common.cuh"

namespace unb {

// Persistent solve over SolveArgs::n pixels (or SolveArgs::list); the grid
// is `threads`-wide blocks times the occupancy limit times `sms`.
// variant 0: L-BFGS history in registers; 1: in shared memory.
cudaError_t launch_solve_fp32(int L, bool refine, int variant, const Models<float>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s);
cudaError_t launch_solve_fp64(int L, bool refine, const Models<double>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s);

// Guided-filter refinement targets, FP64 throughout.
struct FilterArgs {
    int width = 0, height = 0, layers = 0, radius = 0;
    double eps = 1e-4;
    int opaque = 1, smooth = 0, plus = 0;
    const double* image = nullptr;   // f64 interleaved RGB (n*3)
    const double* first = nullptr;   // packed f64 [l][i][RGBA]
    double* targets = nullptr;       // planar f64 [(L+3)][n]
    int32_t* status = nullptr;       // per pixel: 0, 1 zero Plus sum, 2 non-opaque SourceOver background
    double* scratch = nullptr;       // filter_scratch_doubles() doubles
};
size_t filter_scratch_doubles(int width, int height, int layers, int smooth);
cudaError_t launch_filter(const FilterArgs& a, cudaStream_t s);

// Fixed scratch of the allocation-free first pass (noalloc.cu): device
// address on the current device (resolved on the first call per device),
// its size, and the largest image it serves.
cudaError_t noalloc_scratch(void** ptr, size_t* bytes, size_t* max_pixels);
size_t noalloc_max_pixels();   // no CUDA call

}  // namespace unb
