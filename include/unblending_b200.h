/* Extensions of the unblending C ABI in the B200 implementation.
 *
 * New symbols only; the v1 entry points of unblending.h are unchanged. They
 * expose what the v1 signatures cannot carry: the arithmetic precision of
 * the per-pixel solve, the guided-filter radius (v1 derives it from the
 * image size, unblending.cpp:351), per-pixel status and work counters,
 * device-side timings, and device-resident inputs/outputs. None of them has
 * a counterpart in the reference's C ABI; their semantics follow the
 * reference functions named beside each. */
#ifndef UNBLENDING_B200_H
#define UNBLENDING_B200_H

#include "unblending.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    /* FP32 solve; every pixel's result is re-checked in FP64 and pixels that
     * miss the feasibility tolerance are re-solved in FP64. Faster, but the
     * method stops at its own loose tolerance (5e-3), so where it stops
     * depends on the arithmetic: about 1 % of pixels land more than 1e-3 from
     * the reference's FP64 result. */
    UNBLENDING_PRECISION_FP32 = 0,
    /* The reference's FP64 method and arithmetic (the default): results equal
     * the reference's FP64 solver's to rounding. */
    UNBLENDING_PRECISION_FP64 = 1
};

/* Controls of the per-pixel augmented-Lagrangian solve
 * (augmented_lagrangian.cuh:163-167) and of the refinement filter
 * (unblending.cpp:351-353). */
typedef struct unblending_solver_options {
    uint32_t struct_size;
    int32_t precision;          /* UNBLENDING_PRECISION_*, default FP64 */
    int32_t starts;             /* 1..3 solver starts, default 1 */
    int32_t radius;             /* refinement radius; < 0 selects 60 * min(w, h) / 1000 */
    double epsilon;             /* guided-filter regularizer, default 1e-4 */
    int32_t resolve_misses;     /* FP32 precision: FP64 re-solve of misses, default 1 */
    int32_t inner, outer;       /* iteration caps, default 256 and 22 */
    double inner_tolerance;     /* default 5e-3 */
    double outer_tolerance;     /* feasibility tolerance on |C|, default 5e-3 */
    int32_t threads_per_block;  /* 0 selects the tuned default */
    int32_t kernel_variant;     /* FP32 solve: -1 tuned default; 0 history in registers; 1/2 history in shared
                                   memory with registers capped for 4/5 blocks per SM; 3 as 1 with the evaluation
                                   rolled over the layers; 4 history in global memory, rolled, 5 blocks per SM;
                                   5 as 3, with three lanes per pixel where the alphas are pinned (refinement) */
    const struct unblending_mlp* warm_start;  /* first pass: learned start point, NULL = the reference's start.
                                   Pixels the learned start leaves unsolved get the plain solve from the
                                   reference's start (FP64 precision: the FP64 solve; FP32 precision with
                                   resolve_misses: the FP32 solve, and what that misses the FP64 re-solve). */
    int32_t fp64_variant;       /* FP64 solve and re-solve: -1 default; history in shared memory with 0
                                   uncapped registers, 1 capped for 2 blocks per SM; 2 history in global memory,
                                   x/g/d in shared memory, evaluation rolled, 3 blocks per SM; 3 as 2 with the
                                   start and bounds in global memory, 4 blocks per SM; 4/5 as 3/2 with three
                                   lanes per pixel where the alphas are pinned (refinement); 6 as 3 (first pass)
                                   and 5 (refinement) with the bookkeeping rolled over the layers; 7 the
                                   refinement of 6 with its start and bounds in global memory, 4 blocks per SM
                                   (first passes run 3). Default: 3 for the first pass, 7 for the refinement.
                                   Every variant gives the same results. */
    int32_t fp32_outer;         /* FP32 precision with resolve_misses: outer steps of the FP32 solve before a
                                   pixel is left to the FP64 re-solve (default 9; 0 = outer);
                                   a pixel stopped there unconverged is always re-solved */
    int32_t gradient_quorum;    /* scheduling of the pixels of one warp: an evaluation with a gradient runs when
                                   at least gradient_quorum/8 of the warp's pixels need one (or none needs a
                                   value alone); the others wait one evaluation. 0 = never wait. Results do not
                                   depend on it. Default 4 (FP64 solves of the 1024x1024 five-layer image:
                                   228 ms at 3, 225.5 at 4, 226.5 at 5, 240 at 2), range 0..8 */
    int32_t frozen_stop;        /* FP64 solves (the FP64 precision solve, and the re-solve behind the FP32 solve)
                                   stop a pixel after this many consecutive outer steps that moved neither its
                                   point nor its best point (default 4; 0 = run to the outer cap, the
                                   reference's schedule; results equal on every tested image) */
    int32_t pixel_order;        /* order in which a solve hands out the pixels it solves: 1 (default) grouped by
                                   colour (a Morton order of the quantized RGB), so the pixels that one warp solves
                                   together take similar paths through the method; 0 image order. Results do not
                                   depend on it. A caller built against the previous layout, whose struct_size
                                   ends before this field, gets the default. */
    int32_t defer_outer;        /* FP64 refinement solve (kernel variant 7, the default): a pixel still unsolved
                                   when it reaches this outer step leaves the solve launch with its state and is
                                   resumed, with the other such pixels, by a second launch right behind it; the
                                   pixels the method struggles with then share warps. 0 = no deferral. Results do
                                   not depend on it. Default 8 */
} unblending_solver_options;

#define UNBLENDING_SOLVER_OPTIONS_INIT \
    { (uint32_t)sizeof(unblending_solver_options), UNBLENDING_PRECISION_FP64, 1, -1, 1e-4, 1, 256, 22, 5e-3, 5e-3, 0, -1, \
      NULL, -1, 9, 4, 4, 1, 8 }

/* Learned warm start (no counterpart in the reference). A per-pixel MLP,
 * 30 inputs (RGB of the clamped 3x3 neighbourhood, and log(1/256 + c) of the
 * pixel's own colour) -> 64 -> 64 -> 64 (GELU) -> 4L outputs (sigmoid): the
 * solver's start point [alpha_0..alpha_{L-1}, rgb_0..rgb_{L-1}]. BF16 weights,
 * FP32 accumulation, tensor-core (tcgen05) training and inference kernels.
 * Weights are out x in, row-major; unused rows of w4/b4 are zero. */
typedef struct unblending_mlp {
    uint32_t struct_size;
    int32_t layer_count;        /* L the network predicts for (1..8) */
    float w1[64 * 32], w2[64 * 64], w3[64 * 64], w4[32 * 64];
    float b1[64], b2[64], b3[64], b4[32];
    float loss;                 /* mean squared error of the last training batch */
    int32_t steps;              /* Adam steps taken */
} unblending_mlp;

typedef struct unblending_mlp_options {
    uint32_t struct_size;
    int32_t batch;              /* samples per Adam step, default 8192 */
    int32_t steps;              /* Adam steps, default 512 */
    float learning_rate;        /* default 1e-3 */
    uint64_t seed;              /* initialization and batch sampling */
} unblending_mlp_options;

#define UNBLENDING_MLP_OPTIONS_INIT { (uint32_t)sizeof(unblending_mlp_options), 8192, 512, 1e-3f, 1 }

/* Trains `model` on the decompositions that this library's first pass
 * (cold start, `solver` controls, warm_start ignored) computes for `count`
 * device-resident images (packed RGB doubles, image k of widths[k] x
 * heights[k]) sharing the given layers. Synchronous. */
UNBLENDING_API int32_t unblending_mlp_train_device(
    int32_t count, const int32_t* widths, const int32_t* heights, const double* const* images,
    const unblending_layer* layers, size_t layer_count, const unblending_options* options,
    const unblending_solver_options* solver, const unblending_mlp_options* mlp_options, unblending_mlp* model);

/* Gradient of the training loss (mean over samples and outputs of the
 * squared error between the sigmoid outputs and targets) of `model` on
 * `count` samples: features (device, count x 32 floats, the last two zero)
 * and targets (device, count x 4L floats). dL/dW and dL/db are written to the
 * weight and bias fields of `gradient` (host), the loss to gradient->loss. */
UNBLENDING_API int32_t unblending_mlp_loss_grad_device(
    const unblending_mlp* model, int32_t count, const float* features, const float* targets, unblending_mlp* gradient);

/* The network's start point for every pixel of a device-resident image:
 * out is device memory of width*height*4L floats (pixel-major). */
UNBLENDING_API int32_t unblending_mlp_predict_device(
    const unblending_mlp* model, int32_t width, int32_t height, const double* image, float* out, void* stream);

/* Per-call report. Times are device time measured with CUDA events. */
typedef struct unblending_stats {
    uint32_t struct_size;
    int32_t radius;             /* refinement radius used */
    int64_t pixels;
    int64_t misses;             /* pixels whose first solve missed the tolerance */
    int64_t failed;             /* pixels still missing it at the end */
    int64_t normalization_failed; /* refinement: pixels whose targets could not be normalized */
    double ms_upload, ms_filter, ms_solve, ms_resolve, ms_download, ms_total;
    /* Evaluations of the call's solves over all pixels, with a value and with
     * a gradient: of the FP64 solves, and of the FP32 solve. */
    int64_t fp64_values, fp64_gradients, fp32_values, fp32_gradients;
} unblending_stats;

/* unblending_unmix / unblending_refine with solver options, an optional
 * per-pixel status (n int32: 0 ok, 3 misses the tolerance, 8 refinement
 * targets not normalizable), optional work counters (n x 5 uint32: values,
 * gradients, inner iterations, line-search trials, outer steps) and stats.
 * Any of solver, status, counters, stats may be NULL. */
UNBLENDING_API int32_t unblending_unmix_ex(
    const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
    const unblending_options* options, const unblending_solver_options* solver,
    double* output, size_t output_capacity, int32_t* status, uint32_t* counters, unblending_stats* stats);

UNBLENDING_API int32_t unblending_refine_ex(
    const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
    const double* first_pass, size_t first_pass_size, const unblending_options* options,
    const unblending_solver_options* solver, double* output, size_t output_capacity,
    int32_t* status, uint32_t* counters, unblending_stats* stats);

/* Device-resident variants. All pointers are device memory of the current
 * CUDA device: image is w*h packed RGB doubles, first_pass/output are packed
 * [layer][row][column][RGBA] doubles (output may alias first_pass), status
 * and counters as above (may be NULL). Work is enqueued on `stream` (a
 * cudaStream_t, NULL selects the library's stream); the call returns without
 * synchronizing unless `stats` is non-NULL. */
UNBLENDING_API int32_t unblending_unmix_device(
    int32_t width, int32_t height, const double* image, const unblending_layer* layers, size_t layer_count,
    const unblending_options* options, const unblending_solver_options* solver,
    double* output, int32_t* status, uint32_t* counters, void* stream, unblending_stats* stats);

UNBLENDING_API int32_t unblending_refine_device(
    int32_t width, int32_t height, const double* image, const unblending_layer* layers, size_t layer_count,
    const double* first_pass, const unblending_options* options, const unblending_solver_options* solver,
    double* output, int32_t* status, uint32_t* counters, void* stream, unblending_stats* stats);

/* The same two passes restricted to the pixels of rows [row_begin, row_end)
 * of the image (0 <= row_begin <= row_end <= height, else
 * UNBLENDING_INVALID_ARGUMENT): only their outputs,
 * status and counters are written. The refinement's guided filter still
 * covers the whole image and reads the whole first pass, so a band's results
 * equal the whole-image call's for its rows bit for bit: an image split into
 * row bands (one per GPU) and the first pass gathered between the passes
 * decomposes exactly as on one GPU. */
UNBLENDING_API int32_t unblending_unmix_device_rows(
    int32_t width, int32_t height, const double* image, const unblending_layer* layers, size_t layer_count,
    const unblending_options* options, const unblending_solver_options* solver, double* output, int32_t* status,
    uint32_t* counters, int32_t row_begin, int32_t row_end, void* stream, unblending_stats* stats);

UNBLENDING_API int32_t unblending_refine_device_rows(
    int32_t width, int32_t height, const double* image, const unblending_layer* layers, size_t layer_count,
    const double* first_pass, const unblending_options* options, const unblending_solver_options* solver,
    double* output, int32_t* status, uint32_t* counters, int32_t row_begin, int32_t row_end, void* stream,
    unblending_stats* stats);

/* First pass that allocates nothing. No counterpart in the reference: it
 * exists for callers that must not allocate device memory inside their
 * processing call, such as a host application that owns all device memory
 * through its own allocator, or a per-frame effect whose time budget cannot
 * absorb cudaMalloc/cudaFree (both can synchronize the device).
 *
 * Same arguments and results as unblending_unmix_device without counters and
 * stats; the caller still passes the input image, output and optional status
 * buffers (device memory). The solve's scratch (queue heads, miss counters,
 * miss lists) lives in a fixed 32 MiB + 256 B device array that every GPU
 * loading the library holds until the process exits; images larger than
 * 2048 * 2048 = 4,194,304 pixels return UNBLENDING_INVALID_ARGUMENT, and so
 * does a solver->warm_start (the learned start needs buffers of its own).
 * Kernel variants that keep their L-BFGS history in global memory are
 * replaced by their shared-memory counterparts: the same results, but the
 * FP64 solves run slower than unblending_unmix_device's (about 1.7x on the
 * FP64 re-solve of a 1024x1024 five-layer image). The call
 * uses no cudaMalloc, cudaFree, library stream or event; work is enqueued on
 * `stream` (NULL: the legacy default stream) and the call returns without
 * synchronizing. The first call on a device resolves the array's device
 * address (cudaGetSymbolAddress) and should come before any stream capture;
 * the address is kept for the process, so calls after a cudaDeviceReset of
 * that device are not supported. Every call shares the one array, so calls
 * whose GPU work overlaps (several streams, or several host threads) race and
 * must be serialized by the caller. */
UNBLENDING_API int32_t unblending_unmix_device_noalloc(
    int32_t width, int32_t height, const double* image, const unblending_layer* layers, size_t layer_count,
    const unblending_options* options, const unblending_solver_options* solver,
    double* output, int32_t* status, void* stream);

/* One image of a batched first pass. Device pointers: image (packed RGB
 * doubles), output (packed [layer][row][column][RGBA] doubles), status (or
 * NULL). Host pointers: layers (layer_count entries), warm_start (or NULL). */
typedef struct unblending_image_job {
    int32_t width, height;
    const double* image;
    const unblending_layer* layers;
    int32_t layer_count;
    double* output;
    int32_t* status;
    const unblending_mlp* warm_start;
} unblending_image_job;

/* First pass of many images of uneven size and layer count. No counterpart
 * in the reference (which solves one image per call). Images are grouped by
 * layer count; each group runs as one persistent launch whose work queue
 * spans all its images' pixels, and all groups (with their warm-start
 * inference and FP64 re-solves) are captured into one CUDA graph, replayed
 * while the same job list is submitted again. The kernel variant and block
 * size of each group come from a timing sweep on a pixel sample, cached per
 * layer count. Results equal those of unblending_unmix_device per image.
 * Synchronous when stats is non-NULL. */
UNBLENDING_API int32_t unblending_unmix_batch_device(
    const unblending_image_job* jobs, int32_t count, const unblending_options* options,
    const unblending_solver_options* solver, void* stream, unblending_stats* stats);

/* Number of GPU kernel launches the most recent call on this thread issued. */
UNBLENDING_API int64_t unblending_last_launch_count(void);

/* LayerInfos JSON, the reference's layer-info file (LayerInfos.md;
 * unblending/src/unblending_io.cpp:141-170 import_layer_infos). Host only.
 * Parses NUL-terminated `json` into at most `capacity` layers, bottom first,
 * with the precision = inverse of the file's covariance; *count receives the
 * file's layer count (UNBLENDING_BUFFER_TOO_SMALL when it exceeds capacity).
 * Malformed text, an unknown mode name or a singular covariance:
 * UNBLENDING_INVALID_ARGUMENT. */
UNBLENDING_API int32_t unblending_parse_layer_infos(const char* json, unblending_layer* layers, size_t capacity,
                                                    size_t* count);

/* JSON text of `layer_count` layers in the same format
 * (unblending_io.cpp:125-139 export_layer_infos): writes it NUL-terminated to
 * `text` when `capacity` bytes suffice; *length receives its length without
 * the NUL (UNBLENDING_BUFFER_TOO_SMALL when it does not fit). */
UNBLENDING_API int32_t unblending_format_layer_infos(const unblending_layer* layers, size_t layer_count, char* text,
                                                     size_t capacity, size_t* length);

#ifdef __cplusplus
}
#endif
#endif
