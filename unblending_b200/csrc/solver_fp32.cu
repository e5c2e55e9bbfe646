// FP32 instantiations of the per-pixel solve. Variant 0 keeps the L-BFGS
// history in registers (fewer, fatter warps); variants 1 and 2 keep it in
// shared memory and cap registers for four (1) or three (2) 128-thread
// blocks per SM.
#include "solver_dispatch.hpp"
#include "solver_kernels.cuh"

namespace unb {

namespace {
template <int L, bool R, bool H, int B> cudaError_t go(const Models<float>& m, const SolverControls& c, const SolveArgs& a,
                                                int threads, int sms, cudaStream_t s) {
    using Launch = SolveLauncher<float, L, R, H, B>;
    int per_sm = 0;
    cudaError_t e = Launch::occupancy(threads, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    return Launch::launch(m, c, a, per_sm * sms, threads, s);
}
template <bool R, bool H, int B> cudaError_t pick(int L, const Models<float>& m, const SolverControls& c, const SolveArgs& a,
                                           int threads, int sms, cudaStream_t s) {
    switch (L) {
    case 1: return go<1, R, H, B>(m, c, a, threads, sms, s);
    case 2: return go<2, R, H, B>(m, c, a, threads, sms, s);
    case 3: return go<3, R, H, B>(m, c, a, threads, sms, s);
    case 4: return go<4, R, H, B>(m, c, a, threads, sms, s);
    case 5: return go<5, R, H, B>(m, c, a, threads, sms, s);
    case 6: return go<6, R, H, B>(m, c, a, threads, sms, s);
    case 7: return go<7, R, H, B>(m, c, a, threads, sms, s);
    case 8: return go<8, R, H, B>(m, c, a, threads, sms, s);
    default: return cudaErrorInvalidValue;
    }
}
template <int L, bool H, int B> cudaError_t go_batch(const SolverControls& c, const SolveArgs& a, int threads,
                                                     int sms, cudaStream_t s) {
    using Launch = SolveLauncher<float, L, false, H, B, true>;
    int per_sm = 0;
    cudaError_t e = Launch::occupancy(threads, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    return Launch::launch(Models<float>{}, c, a, per_sm * sms, threads, s);
}
template <bool H, int B> cudaError_t pick_batch(int L, const SolverControls& c, const SolveArgs& a, int threads,
                                                int sms, cudaStream_t s) {
    switch (L) {
    case 1: return go_batch<1, H, B>(c, a, threads, sms, s);
    case 2: return go_batch<2, H, B>(c, a, threads, sms, s);
    case 3: return go_batch<3, H, B>(c, a, threads, sms, s);
    case 4: return go_batch<4, H, B>(c, a, threads, sms, s);
    case 5: return go_batch<5, H, B>(c, a, threads, sms, s);
    case 6: return go_batch<6, H, B>(c, a, threads, sms, s);
    case 7: return go_batch<7, H, B>(c, a, threads, sms, s);
    case 8: return go_batch<8, H, B>(c, a, threads, sms, s);
    default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t launch_solve_batch_fp32(int L, int variant, const SolverControls& c, const SolveArgs& a, int threads,
                                    int sms, cudaStream_t s) {
    return variant == 2 ? pick_batch<true, 3>(L, c, a, threads, sms, s) : pick_batch<false, 1>(L, c, a, threads, sms, s);
}

cudaError_t launch_solve_fp32(int L, bool refine, int variant, const Models<float>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s) {
    if (variant == 1)
        return refine ? pick<true, true, 4>(L, m, c, a, threads, sms, s) : pick<false, true, 4>(L, m, c, a, threads, sms, s);
    if (variant == 2)
        return refine ? pick<true, true, 3>(L, m, c, a, threads, sms, s) : pick<false, true, 3>(L, m, c, a, threads, sms, s);
    return refine ? pick<true, false, 1>(L, m, c, a, threads, sms, s) : pick<false, false, 1>(L, m, c, a, threads, sms, s);
}

}  // namespace unb
