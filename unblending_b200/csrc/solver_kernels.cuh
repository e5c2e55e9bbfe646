// Persistent per-pixel solve kernel and its host launcher.
#pragma once
#include <cstdio>

#include "solver.cuh"

namespace unb {

// Dynamic shared memory: every lane's slice (cold values, the L-BFGS
// history when it is kept there, the rolled evaluation's intermediates).
template <class T, int L, int S, bool BATCH> struct SolveSmem {
    using Slice = LaneSlice<T, L, S>;
    static size_t bytes(int threads) { (void)threads; return Slice::bytes(); }
};

// S: storage policy (history place | kVectorsShared); MINB: blocks per SM
// the register allocation must allow (launch bounds).
template <class T, int L, bool REFINE, int S, int MINB, bool BATCH, int MODE = kPlain>
__global__ void __launch_bounds__(128, MINB)
solve_pixels(const __grid_constant__ Models<T> m, const __grid_constant__ SolverControls ctl,
             const __grid_constant__ SolveArgs a) {
    QuadSolver<T, L, REFINE, S, BATCH, MODE> solver(&m, ctl, a);
    solver.run();
}

template <class T, int L, bool REFINE, int S, int MINB = 1, bool BATCH = false, int MODE = kPlain> struct SolveLauncher {
    using Smem = SolveSmem<T, L, S, BATCH>;

    static cudaError_t occupancy(int threads, int* blocks_per_sm) {
        auto k = solve_pixels<T, L, REFINE, S, MINB, BATCH, MODE>;
        const size_t sm = Smem::bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, sm);
    }

    static cudaError_t launch(const Models<T>& m, const SolverControls& ctl, const SolveArgs& a, int blocks,
                              int threads, cudaStream_t stream) {
        auto k = solve_pixels<T, L, REFINE, S, MINB, BATCH, MODE>;
        const size_t sm = Smem::bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        if constexpr (history_of(S) == kHistGlobal) {
            // Each resident lane owns a slice of the caller's history array.
            if (!a.history) return cudaErrorInvalidValue;
            blocks = blocks < a.history_lanes / kSliceStride ? blocks : a.history_lanes / kSliceStride;
            if (blocks < 1) return cudaErrorInvalidValue;
        }
        k<<<blocks, threads, sm, stream>>>(m, ctl, a);
        return cudaGetLastError();
    }
};

}  // namespace unb
