// Shared definitions of the B200 unblending kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace unb {

constexpr int kMaxLayers = 8;       // compiled layer counts 1..8
constexpr int kHistory = 6;         // L-BFGS memory (augmented_lagrangian.cuh:164)
// Lane stride of the solver's per-lane storage: the largest block (128
// threads), so that slice offsets are compile-time constants for any block size.
constexpr int kSliceStride = 128;

// Layer descriptors in the solver's arithmetic type, passed by value as a
// kernel parameter (lives in the constant bank, no global state).
template <class T> struct Models {
    T mean[kMaxLayers][3];
    T prec[kMaxLayers][9];
    int mode[kMaxLayers];
    int X[kMaxLayers], Y[kMaxLayers], Z[kMaxLayers];
    // Branch-free form of the ten piecewise-bilinear modes:
    //   B = c0 + cs s + cd d + csd s d, coefficient set [0] where
    //   t = ka s + kb d + kc satisfies t < 0 (strict) or t <= 0, else set [1];
    // special = 6, 7, 9 marks Dodge, Burn, SoftLight (evaluated directly).
    T c0[kMaxLayers][2], cs[kMaxLayers][2], cd[kMaxLayers][2], csd[kMaxLayers][2];
    T ka[kMaxLayers], kb[kMaxLayers], kc[kMaxLayers];
    int strict[kMaxLayers], special[kMaxLayers];
};

// Fills the bilinear table of layer l from its mode (blend_mode.hpp:90-196).
template <class T> inline void set_blend_table(Models<T>& m, int l, int mode) {
    auto set = [&](int k, double c0, double cs, double cd, double csd) {
        m.c0[l][k] = T(c0); m.cs[l][k] = T(cs); m.cd[l][k] = T(cd); m.csd[l][k] = T(csd);
    };
    auto both = [&](double c0, double cs, double cd, double csd) { set(0, c0, cs, cd, csd); set(1, c0, cs, cd, csd); };
    m.ka[l] = T(0); m.kb[l] = T(0); m.kc[l] = T(-1); m.strict[l] = 1; m.special[l] = 0;
    both(0, 0, 0, 0);
    switch (mode) {
    case 0: both(0, 1, 0, 0); break;                                   // normal: s
    case 1: both(0, 0, 0, 1); break;                                   // multiply: s d
    case 2: both(0, 1, 1, -1); break;                                  // screen: s + d - s d
    case 3: m.kb[l] = T(1); m.kc[l] = T(-0.5); m.strict[l] = 0;        // overlay: d <= 1/2
        set(0, 0, 0, 0, 2); set(1, -1, 2, 2, -2); break;
    case 4: m.ka[l] = T(1); m.kb[l] = T(-1); m.kc[l] = T(0);           // darken: s < d ? s : d
        set(0, 0, 1, 0, 0); set(1, 0, 0, 1, 0); break;
    case 5: m.ka[l] = T(1); m.kb[l] = T(-1); m.kc[l] = T(0);           // lighten: s < d ? d : s
        set(0, 0, 0, 1, 0); set(1, 0, 1, 0, 0); break;
    case 8: m.ka[l] = T(1); m.kc[l] = T(-0.5); m.strict[l] = 0;        // hard light: s <= 1/2
        set(0, 0, 0, 0, 2); set(1, -1, 2, 2, -2); break;
    case 10: m.ka[l] = T(1); m.kb[l] = T(-1); m.kc[l] = T(0);          // difference: |s - d|
        set(0, 0, -1, 1, 0); set(1, 0, 1, -1, 0); break;
    case 11: both(0, 1, 1, -2); break;                                 // exclusion: s + d - 2 s d
    case 12: both(0, 1, 1, 0); break;                                  // linear dodge: s + d
    default: m.special[l] = mode; break;                               // 6, 7, 9
    }
}

// Solver controls of augmented_lagrangian.cuh:163-167 (history fixed at 6).
struct SolverControls {
    int inner = 256, outer = 22, starts = 1;
    double inner_tolerance = 5e-3, outer_tolerance = 5e-3;
    int gradient_on_first_trial = 1;   // fuse the first line-search trial's gradient
    int gradient_quorum = 4;           // eighths of a warp's live pixels that start a gradient evaluation
    int direction_quorum = 0;          // eighths of a warp's live pixels that start a new direction (0 = no wait)
    int cap_is_miss = 0;               // a pixel that reaches the outer cap unconverged is a miss
    int frozen_stop = 0;               // stop after this many outer steps that move neither x nor the best point
};

// Words a lane of a deferred pixel keeps (SolveArgs::defer_state): x, the
// best point and the start seed (L each), up to L multipliers, and seven
// scalars.
__host__ __device__ constexpr int defer_words(int L) { return 4 * L + 7; }

// One image of a batched first pass: its pixels occupy global queue indices
// [offset, offset + n) of its layer-count group.
struct BatchJob {
    const double* image;
    double* out;
    int32_t* status;
    const float* warm;
    int64_t offset, n;
    int32_t model;      // index into the group's model table
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
    const float* warm = nullptr;            // optional start-0 seed: n x 4L floats, pixel-major x
    // Batched first pass: n is the group's total pixel count, pixels are
    // global queue indices decoded through `jobs` (sorted by offset), and
    // each job's layer models come from `models` (Models<T> entries).
    const BatchJob* jobs = nullptr;
    int job_count = 0;
    const void* models = nullptr;
    // Optional totals over the launch: evaluations with a value, with a gradient.
    unsigned long long* tally = nullptr;
    int opaque = 1, smooth = 0;
    // Global-memory L-BFGS history (kernels that keep it there): room for
    // history_lanes lanes; the launch uses at most history_lanes / 128 blocks.
    void* history = nullptr;
    int history_lanes = 0;
    // Without a list: the launch solves pixels [first_pixel, first_pixel +
    // pixel_count) of the image (pixel_count < 0: all n).
    int first_pixel = 0, pixel_count = -1;
    // Without a list: optional queue order, the pixel index of each queue
    // index (a permutation of the pixels the launch solves); null = in order.
    const int32_t* order = nullptr;
    // With a list: at most list_limit of its entries are solved.
    int list_limit = 0x7fffffff;
    // Deferral (defer_outer > 0): a pixel about to begin outer step
    // defer_outer (counted from 0) leaves the launch with its state at that
    // point in slot k of defer_state (k from *defer_count, up to
    // defer_capacity slots; past that it carries on) and its queue index in
    // defer_list[k]. A launch with resume set and list = defer_list resumes
    // entry k of its list from slot k at that outer step. defer_state holds
    // values of the solve's type: word w of lane q of slot k at
    // [w * defer_capacity * 4 + k * 4 + q], defer_words(L) words a lane.
    int defer_outer = 0, defer_capacity = 0;
    int32_t* defer_list = nullptr;
    int32_t* defer_count = nullptr;
    void* defer_state = nullptr;
    int resume = 0;
};

}  // namespace unb
