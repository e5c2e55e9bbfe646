// Layer-count dispatch of the solve kernels (the kernels themselves are
// compiled per layer count in solver_l<L>.cu).
#include "solver_dispatch.hpp"

namespace unb {

namespace {
template <class F> cudaError_t by_layers(int L, F&& f) {
    switch (L) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    case 8: return f(std::integral_constant<int, 8>{});
    default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t launch_solve_fp32(int L, bool refine, int variant, const Models<float>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s) {
    return by_layers(L, [&](auto k) { return solve_fp32_layers<decltype(k)::value>(refine, variant, m, c, a, threads, sms, s); });
}

cudaError_t launch_solve_fp64(int L, bool refine, int variant, const Models<double>& m, const SolverControls& c,
                              const SolveArgs& a, int threads, int sms, cudaStream_t s) {
    return by_layers(L, [&](auto k) { return solve_fp64_layers<decltype(k)::value>(refine, variant, m, c, a, threads, sms, s); });
}

cudaError_t launch_solve_batch_fp32(int L, int variant, const SolverControls& c, const SolveArgs& a, int threads,
                                    int sms, cudaStream_t s) {
    return by_layers(L, [&](auto k) { return solve_batch_fp32_layers<decltype(k)::value>(variant, c, a, threads, sms, s); });
}

cudaError_t launch_solve_batch_fp64(int L, int variant, const SolverControls& c, const SolveArgs& a, int threads,
                                    int sms, cudaStream_t s) {
    return by_layers(L, [&](auto k) { return solve_batch_fp64_layers<decltype(k)::value>(variant, c, a, threads, sms, s); });
}

}  // namespace unb
