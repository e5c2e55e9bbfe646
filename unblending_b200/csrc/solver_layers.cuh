// Solve kernels of one layer count, UNB_SOLVER_LAYERS: FP32 and FP64, every
// variant, single-image and batched. Included by solver_l<L>.cu, which are
// compiled with --fmad=false: the FP64 arithmetic then rounds like the
// reference's FP64 solver (built with --fmad=false,
// unblending/CMakeLists.txt:28), and every FP32 variant gives bit-identical
// results (the variant changes speed only).
#include "solver_dispatch.hpp"
#include "solver_kernels.cuh"

#ifndef UNB_SOLVER_LAYERS
#error "define UNB_SOLVER_LAYERS before including solver_layers.cuh"
#endif

namespace unb {

namespace {
constexpr int kL = UNB_SOLVER_LAYERS;

template <class T, bool R, int S, int B, bool BATCH, int MODE = kPlain>
cudaError_t go(const Models<T>& m, const SolverControls& c, const SolveArgs& a, int threads, int sms, cudaStream_t s) {
    using Launch = SolveLauncher<T, kL, R, S, B, BATCH, MODE>;
    int per_sm = 0;
    cudaError_t e = Launch::occupancy(threads, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    return Launch::launch(m, c, a, per_sm * sms, threads, s);
}

// A kernel that can defer or resume pixels (SolveArgs::defer_outer / resume):
// the default FP64 refinement variant, compiled once per mode.
template <bool R, int S, int B>
cudaError_t go_modes(const Models<double>& m, const SolverControls& c, const SolveArgs& a, int threads, int sms,
                     cudaStream_t s) {
    if (a.resume) return go<double, R, S, B, false, kResumes>(m, c, a, threads, sms, s);
    if (a.defer_outer > 0) return go<double, R, S, B, false, kDefers>(m, c, a, threads, sms, s);
    return go<double, R, S, B, false>(m, c, a, threads, sms, s);
}

template <bool R, bool BATCH>
cudaError_t fp32(int variant, const Models<float>& m, const SolverControls& c, const SolveArgs& a, int threads,
                 int sms, cudaStream_t s) {
    switch (variant) {
    case 0: return go<float, R, kHistRegisters, 1, BATCH>(m, c, a, threads, sms, s);
    case 1: return go<float, R, kHistShared, 4, BATCH>(m, c, a, threads, sms, s);
    case 2: return go<float, R, kHistShared, 5, BATCH>(m, c, a, threads, sms, s);
    case 3: return go<float, R, kHistShared | kRolled, 4, BATCH>(m, c, a, threads, sms, s);
    case 4: return go<float, R, kHistGlobal | kRolled, 5, BATCH>(m, c, a, threads, sms, s);
    case 5:   // three lanes per pixel where the alphas are pinned (refinement), else variant 3
        if constexpr (R && !BATCH) return go<float, R, kHistShared | kRolled | kTriple, 4, BATCH>(m, c, a, threads, sms, s);
        else return go<float, R, kHistShared | kRolled, 4, BATCH>(m, c, a, threads, sms, s);
    default: return cudaErrorInvalidValue;
    }
}

template <bool R, bool BATCH>
cudaError_t fp64(int variant, const Models<double>& m, const SolverControls& c, const SolveArgs& a, int threads,
                 int sms, cudaStream_t s) {
    switch (variant) {
    case 0: return go<double, R, kHistShared, 1, BATCH>(m, c, a, threads, sms, s);
    case 1: return go<double, R, kHistShared, 2, BATCH>(m, c, a, threads, sms, s);
    case 2: return go<double, R, kHistGlobal | kVectorsShared | kRolled, 3, BATCH>(m, c, a, threads, sms, s);
    case 3: return go<double, R, kHistGlobal | kVectorsShared | kRolled | kColdGlobal, 4, BATCH>(m, c, a, threads, sms, s);
    case 4:   // as 3, three lanes per pixel where the alphas are pinned
        if constexpr (R && !BATCH)
            return go<double, R, kHistGlobal | kVectorsShared | kRolled | kColdGlobal | kTriple, 4, BATCH>(m, c, a, threads, sms, s);
        else return go<double, R, kHistGlobal | kVectorsShared | kRolled | kColdGlobal, 4, BATCH>(m, c, a, threads, sms, s);
    case 5:   // three lanes per pixel where the alphas are pinned (refinement), else variant 2
        if constexpr (R && !BATCH)
            return go<double, R, kHistGlobal | kVectorsShared | kRolled | kTriple, 3, BATCH>(m, c, a, threads, sms, s);
        else return go<double, R, kHistGlobal | kVectorsShared | kRolled, 3, BATCH>(m, c, a, threads, sms, s);
    case 6:   // 3 (first pass) and 5 (refinement) with the bookkeeping rolled over the layers
        if constexpr (R && !BATCH)
            return go<double, R, kHistGlobal | kVectorsShared | kRolled | kTriple | kBookRolled, 3, BATCH>(m, c, a, threads,
                                                                                                       sms, s);
        else if constexpr (!R)
            return go<double, R, kHistGlobal | kVectorsShared | kRolled | kColdGlobal | kBookRolled, 4, BATCH>(
                m, c, a, threads, sms, s);
        else return cudaErrorInvalidValue;
    case 7:   // 6 with the refinement's cold values in the global array, 4 blocks per SM; first passes run 3
        if constexpr (R && !BATCH)
            return go_modes<R, kHistGlobal | kVectorsShared | kRolled | kTriple | kBookRolled | kColdGlobal, 4>(
                m, c, a, threads, sms, s);
        else return go<double, R, kHistGlobal | kVectorsShared | kRolled | kColdGlobal, 4, BATCH>(m, c, a, threads, sms, s);
    default: return cudaErrorInvalidValue;
    }
}
}  // namespace

template <> cudaError_t solve_fp32_layers<kL>(bool refine, int variant, const Models<float>& m, const SolverControls& c,
                                              const SolveArgs& a, int threads, int sms, cudaStream_t s) {
    return refine ? fp32<true, false>(variant, m, c, a, threads, sms, s)
                  : fp32<false, false>(variant, m, c, a, threads, sms, s);
}

template <> cudaError_t solve_fp64_layers<kL>(bool refine, int variant, const Models<double>& m,
                                              const SolverControls& c, const SolveArgs& a, int threads, int sms,
                                              cudaStream_t s) {
    return refine ? fp64<true, false>(variant, m, c, a, threads, sms, s)
                  : fp64<false, false>(variant, m, c, a, threads, sms, s);
}

template <> cudaError_t solve_batch_fp32_layers<kL>(int variant, const SolverControls& c, const SolveArgs& a,
                                                    int threads, int sms, cudaStream_t s) {
    return fp32<false, true>(variant, Models<float>{}, c, a, threads, sms, s);
}

template <> cudaError_t solve_batch_fp64_layers<kL>(int variant, const SolverControls& c, const SolveArgs& a,
                                                    int threads, int sms, cudaStream_t s) {
    return fp64<false, true>(variant, Models<double>{}, c, a, threads, sms, s);
}

}  // namespace unb
