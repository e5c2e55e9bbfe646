// Persistent per-pixel solve kernel and its host launcher.
#pragma once
#include <cstdio>

#include "solver.cuh"

namespace unb {

// MINB: blocks per SM the register allocation must allow (launch bounds).
template <class T, int L, bool REFINE, bool HSMEM, int MINB>
__global__ void __launch_bounds__(128, MINB)
solve_pixels(const __grid_constant__ Models<T> m, const __grid_constant__ SolverControls ctl,
             const __grid_constant__ SolveArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    QuadSolver<T, L, REFINE, HSMEM> S(m, ctl, a);
    S.hist.init(reinterpret_cast<T*>(smem_raw));
    S.run();
}

template <class T, int L, bool REFINE, bool HSMEM, int MINB = 1> struct SolveLauncher {
    static size_t smem_bytes(int threads) { return HSMEM ? size_t(threads) * kHistory * L * 2 * sizeof(T) : 0; }

    static cudaError_t occupancy(int threads, int* blocks_per_sm) {
        auto k = solve_pixels<T, L, REFINE, HSMEM, MINB>;
        const size_t sm = smem_bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, sm);
    }

    static cudaError_t launch(const Models<T>& m, const SolverControls& ctl, const SolveArgs& a, int blocks,
                              int threads, cudaStream_t stream) {
        auto k = solve_pixels<T, L, REFINE, HSMEM, MINB>;
        const size_t sm = smem_bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        k<<<blocks, threads, sm, stream>>>(m, ctl, a);
        return cudaGetLastError();
    }
};

}  // namespace unb
