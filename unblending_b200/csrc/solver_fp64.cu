// FP64 instantiations of the per-pixel solve (history in shared memory).
// This translation unit is compiled with --fmad=false so that its arithmetic
// rounds like the reference's FP64 solver (built with --fmad=false,
// unblending/CMakeLists.txt:28).
#include "solver_dispatch.hpp"
#include "solver_kernels.cuh"

namespace unb {

namespace {
template <int L, bool R> cudaError_t go(const Models<double>& m, const SolverControls& c, const SolveArgs& a,
                                         int threads, int sms, cudaStream_t s) {
    using Launch = SolveLauncher<double, L, R, true>;
    int per_sm = 0;
    cudaError_t e = Launch::occupancy(threads, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    return Launch::launch(m, c, a, per_sm * sms, threads, s);
}
template <bool R> cudaError_t pick(int L, const Models<double>& m, const SolverControls& c, const SolveArgs& a,
                                   int threads, int sms, cudaStream_t s) {
    switch (L) {
    case 1: return go<1, R>(m, c, a, threads, sms, s);
    case 2: return go<2, R>(m, c, a, threads, sms, s);
    case 3: return go<3, R>(m, c, a, threads, sms, s);
    case 4: return go<4, R>(m, c, a, threads, sms, s);
    case 5: return go<5, R>(m, c, a, threads, sms, s);
    case 6: return go<6, R>(m, c, a, threads, sms, s);
    case 7: return go<7, R>(m, c, a, threads, sms, s);
    case 8: return go<8, R>(m, c, a, threads, sms, s);
    default: return cudaErrorInvalidValue;
    }
}
template <int L> cudaError_t go_batch(const SolverControls& c, const SolveArgs& a, int threads, int sms,
                                      cudaStream_t s) {
    using Launch = SolveLauncher<double, L, false, true, 1, true>;
    int per_sm = 0;
    cudaError_t e = Launch::occupancy(threads, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    return Launch::launch(Models<double>{}, c, a, per_sm * sms, threads, s);
}
}  // namespace

cudaError_t launch_solve_batch_fp64(int L, const SolverControls& c, const SolveArgs& a, int threads, int sms,
                                    cudaStream_t s) {
    switch (L) {
    case 1: return go_batch<1>(c, a, threads, sms, s);
    case 2: return go_batch<2>(c, a, threads, sms, s);
    case 3: return go_batch<3>(c, a, threads, sms, s);
    case 4: return go_batch<4>(c, a, threads, sms, s);
    case 5: return go_batch<5>(c, a, threads, sms, s);
    case 6: return go_batch<6>(c, a, threads, sms, s);
    case 7: return go_batch<7>(c, a, threads, sms, s);
    case 8: return go_batch<8>(c, a, threads, sms, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_solve_fp64(int L, bool refine, const Models<double>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s) {
    return refine ? pick<true>(L, m, c, a, threads, sms, s) : pick<false>(L, m, c, a, threads, sms, s);
}

}  // namespace unb
