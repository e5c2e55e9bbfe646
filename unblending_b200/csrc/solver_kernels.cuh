// Persistent per-pixel solve kernel and its host launcher.
#pragma once
#include <cstdio>

#include "solver.cuh"

namespace unb {

// Dynamic shared memory: the L-BFGS history (HSMEM), then one layer-model
// slot per quad (BATCH).
template <class T, int L, bool HSMEM, bool BATCH> struct SolveSmem {
    __host__ __device__ static size_t history(int threads) {
        return HSMEM ? size_t(threads) * kHistory * L * 2 * sizeof(T) : 0;
    }
    static size_t bytes(int threads) {
        const size_t h = (history(threads) + 15) / 16 * 16;
        return h + (BATCH ? size_t(threads / 4) * sizeof(Models<T>) : 0);
    }
};

// MINB: blocks per SM the register allocation must allow (launch bounds).
template <class T, int L, bool REFINE, bool HSMEM, int MINB, bool BATCH>
__global__ void __launch_bounds__(128, MINB)
solve_pixels(const __grid_constant__ Models<T> m, const __grid_constant__ SolverControls ctl,
             const __grid_constant__ SolveArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if constexpr (BATCH) {
        const size_t h = (SolveSmem<T, L, HSMEM, BATCH>::history(blockDim.x) + 15) / 16 * 16;
        Models<T>* slots = reinterpret_cast<Models<T>*>(smem_raw + h);
        QuadSolver<T, L, REFINE, HSMEM, true> S(slots[threadIdx.x >> 2], ctl, a);
        S.hist.init(reinterpret_cast<T*>(smem_raw));
        S.run();
    } else {
        QuadSolver<T, L, REFINE, HSMEM, false> S(m, ctl, a);
        S.hist.init(reinterpret_cast<T*>(smem_raw));
        S.run();
    }
}

template <class T, int L, bool REFINE, bool HSMEM, int MINB = 1, bool BATCH = false> struct SolveLauncher {
    using Smem = SolveSmem<T, L, HSMEM, BATCH>;

    static cudaError_t occupancy(int threads, int* blocks_per_sm) {
        auto k = solve_pixels<T, L, REFINE, HSMEM, MINB, BATCH>;
        const size_t sm = Smem::bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, sm);
    }

    static cudaError_t launch(const Models<T>& m, const SolverControls& ctl, const SolveArgs& a, int blocks,
                              int threads, cudaStream_t stream) {
        auto k = solve_pixels<T, L, REFINE, HSMEM, MINB, BATCH>;
        const size_t sm = Smem::bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        k<<<blocks, threads, sm, stream>>>(m, ctl, a);
        return cudaGetLastError();
    }
};

}  // namespace unb
