// Host-side entry points of the compiled solve and filter kernels.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace unb {

// Persistent solve over SolveArgs::n pixels (or SolveArgs::list); the grid
// is `threads`-wide blocks times the occupancy limit times `sms`.
// FP32 variants: 0 L-BFGS history in registers; 1, 2 history in shared
// memory with registers capped for 4, 5 blocks of 128 threads per SM; 3 as 1
// with the evaluation rolled over the layers; 4 history in global memory
// (SolveArgs::history), evaluation rolled, capped for 5 blocks.
// FP64 variants: 0, 1 history in shared memory with uncapped registers or
// registers capped for 2 blocks per SM; 2 history in global memory, the
// iterate, gradient and direction in shared memory, evaluation rolled, capped
// for 3 blocks; 3 as 2 with the cold values (best point, outer-step start,
// start seed) in the global array too, capped for 4 blocks; 4 as 3 with three
// lanes per pixel in the refinement.
// Variant 5 (FP32 and FP64): the refinement with three lanes per pixel (its
// alphas are pinned, so no alpha lane: 10 pixels per warp), FP32 as 3 and
// FP64 as 2 otherwise; first passes run variant 3 / 2 for it.
// FP64 variant 6: 3 (first pass) and 5 (refinement) with the bookkeeping's
// per-layer loops rolled, the trial point and gradient in the slice. FP64
// variant 7: the refinement of 6 with its cold values in the global array,
// capped for 4 blocks per SM (first passes run 3).
constexpr int kFp32Variants = 6, kFp64Variants = 8;
inline bool variant_global_history(bool fp64, int variant) { return fp64 ? variant >= 2 : variant == 4; }
// FP64 variants whose kernels can defer and resume pixels (SolveArgs::
// defer_outer / resume): the refinement's variant 7. (Deferral was measured
// on the first pass too, where it cost more than it saved: 130 -> 133 ms
// on the 1024x1024 five-layer image, against 91.5 -> 88.1 ms for the
// refinement.)
inline bool variant_defers(int variant, bool refine) { return refine && variant == 7; }
// Blocks per SM that a global-history array is sized for (the launch clamps
// its grid to the array).
constexpr int kGlobalHistoryBlocksPerSm = 6;
cudaError_t launch_solve_fp32(int L, bool refine, int variant, const Models<float>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s);
cudaError_t launch_solve_fp64(int L, bool refine, int variant, const Models<double>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s);
// Batched first pass over the images of one layer-count group
// (SolveArgs::jobs / models); variants as above.
cudaError_t launch_solve_batch_fp32(int L, int variant, const SolverControls& c, const SolveArgs& a, int threads,
                                    int sms, cudaStream_t s);
cudaError_t launch_solve_batch_fp64(int L, int variant, const SolverControls& c, const SolveArgs& a, int threads,
                                    int sms, cudaStream_t s);

// The same per layer count: one translation unit per layer count
// (solver_l<L>.cu) defines these specializations, so the counts compile in
// parallel.
template <int L> cudaError_t solve_fp32_layers(bool refine, int variant, const Models<float>& m,
                                               const SolverControls& c, const SolveArgs& a, int threads, int sms,
                                               cudaStream_t s);
template <int L> cudaError_t solve_fp64_layers(bool refine, int variant, const Models<double>& m,
                                               const SolverControls& c, const SolveArgs& a, int threads, int sms,
                                               cudaStream_t s);
template <int L> cudaError_t solve_batch_fp32_layers(int variant, const SolverControls& c, const SolveArgs& a,
                                                     int threads, int sms, cudaStream_t s);
template <int L> cudaError_t solve_batch_fp64_layers(int variant, const SolverControls& c, const SolveArgs& a,
                                                     int threads, int sms, cudaStream_t s);
#define UNB_DECLARE_LAYER_SOLVES(L)                                                                              \
    template <> cudaError_t solve_fp32_layers<L>(bool, int, const Models<float>&, const SolverControls&,         \
                                                 const SolveArgs&, int, int, cudaStream_t);                      \
    template <> cudaError_t solve_fp64_layers<L>(bool, int, const Models<double>&, const SolverControls&,        \
                                                 const SolveArgs&, int, int, cudaStream_t);                      \
    template <> cudaError_t solve_batch_fp32_layers<L>(int, const SolverControls&, const SolveArgs&, int, int,   \
                                                       cudaStream_t);                                            \
    template <> cudaError_t solve_batch_fp64_layers<L>(int, const SolverControls&, const SolveArgs&, int, int,   \
                                                       cudaStream_t);
UNB_DECLARE_LAYER_SOLVES(1)
UNB_DECLARE_LAYER_SOLVES(2)
UNB_DECLARE_LAYER_SOLVES(3)
UNB_DECLARE_LAYER_SOLVES(4)
UNB_DECLARE_LAYER_SOLVES(5)
UNB_DECLARE_LAYER_SOLVES(6)
UNB_DECLARE_LAYER_SOLVES(7)
UNB_DECLARE_LAYER_SOLVES(8)
#undef UNB_DECLARE_LAYER_SOLVES

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
int filter_launches(int width, int radius);   // kernels one launch_filter call issues
cudaError_t launch_filter(const FilterArgs& a, cudaStream_t s);

// Work-queue order of a solve launch (order.cu): the pixels [first, first +
// count) of an image, grouped by colour, into order[0, count); `cells` is
// scratch of order_cells(count) words.
size_t order_cells(int count);
cudaError_t launch_pixel_order(const double* image, int first, int count, uint32_t* cells, int32_t* order, int sms,
                               cudaStream_t s);
// The same over the `total` queue indices of a batched group (order[k] is a
// queue index of the group; the pixels' colours are read through `jobs`).
cudaError_t launch_group_order(const BatchJob* jobs, int job_count, int total, uint32_t* cells, int32_t* order,
                               int sms, cudaStream_t s);

// Fixed scratch of the allocation-free first pass (noalloc.cu): device
// address on the current device (resolved on the first call per device),
// its size, and the largest image it serves.
cudaError_t noalloc_scratch(void** ptr, size_t* bytes, size_t* max_pixels);
size_t noalloc_max_pixels();   // no CUDA call

// Warm-start MLP (mlp.cu): 32 -> 64 -> 64 -> 64 -> 32, BF16 weights
// (out x in, row-major) and FP32 biases on the device.
struct MlpDevice {
    const __nv_bfloat16* w[4];
    const float* b[4];
};
struct MlpGrad {
    float* w[4];
    float* b[4];
    float* loss;
};
struct MlpMaster {
    float* w[4];
    float* b[4];
    float* mw[4];
    float* vw[4];
    float* mb[4];
    float* vb[4];
};
constexpr int kMlpIn = 32, kMlpHidden = 64, kMlpOut = 32;
cudaError_t launch_mlp_infer(const MlpDevice& p, const double* image, int w, int h, int L, float* out,
                             int32_t* error, int sms, cudaStream_t s);
cudaError_t launch_mlp_features(const double* image, int w, int h, float* feats, cudaStream_t s);
cudaError_t launch_mlp_train(const MlpDevice& p, const float* feats, const float* targets, int count, int outs,
                             const MlpGrad& g, int32_t* error, int sms, cudaStream_t s);
cudaError_t launch_mlp_adam(const MlpMaster& m, const MlpGrad& g, const MlpDevice& p, float lr, int step,
                            cudaStream_t s);
// Training batch assembly and targets (mlp_data.cu).
cudaError_t launch_gather_targets(const double* packed, int64_t n, int L, float* targets, cudaStream_t s);
cudaError_t launch_sample_batch(const float* feats, const float* targets, int64_t pool, int outs, int batch,
                                uint64_t seed, float* bfeats, float* btargets, cudaStream_t s);

}  // namespace unb
