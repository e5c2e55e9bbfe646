// Persistent per-pixel solve kernel and its host launcher.
#pragma once
#include <cstdio>

#include "solver.cuh"

namespace unb {

// FP64 feasibility check of a final point (the reference's guard,
// solver_workspace.cuh:18-38, restricted to the constraint rows): every lane
// holds its slice of the point as double; returns |C|^2, uniform.
template <int L, bool REFINE>
__device__ __forceinline__ double constraint_norm2_fp64(const Quad& Q, const int* mode, const int* X, const int* Y,
                                                        const int* Z, const double* v, double target,
                                                        const double* ahat) {
    const bool colour = Q.q < 3;
    double a[L];
#pragma unroll
    for (int l = 0; l < L; ++l) a[l] = Q.from(v[l], 3);
    double A = a[0], c = v[0];
#pragma unroll
    for (int l = 1; l < L; ++l) {
        const double al = a[l], dd = A;
        const double Al = double(X[l]) * al * dd + double(Y[l]) * al * (1.0 - dd) + double(Z[l]) * dd * (1.0 - al);
        const double s = v[l];
        const double pre = blend_value<double>(mode[l], s, c) * al * dd + double(Y[l]) * al * (1.0 - dd) * s +
                           double(Z[l]) * dd * (1.0 - al) * c;
        c = Al > 1e-12 ? pre / Al : pre;
        A = Al;
    }
    double norm = 0.0;
    if (colour) { const double r = c - target; norm = r * r; }
    else if (REFINE) {
#pragma unroll
        for (int l = 0; l < L; ++l) { const double r = v[l] - ahat[l]; norm += r * r; }
    } else { const double r = A - 1.0; norm = r * r; }
    return Q.sum(norm);
}

template <class T, int L, bool REFINE, bool HSMEM>
__global__ void __launch_bounds__(128)
solve_pixels(const __grid_constant__ Models<T> m, const __grid_constant__ SolverControls ctl,
             const __grid_constant__ SolveArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    QuadSolver<T, L, REFINE, HSMEM> S(m, ctl);
    S.hist.init(reinterpret_cast<T*>(smem_raw));
    S.opaque = a.opaque != 0;
    S.smooth = a.smooth != 0;
    S.tol2 = T(ctl.outer_tolerance * ctl.outer_tolerance);
    const Quad& Q = S.Q;
    const bool colour = Q.q < 3;
    const size_t n = size_t(a.n);
    const int total = a.list ? *a.list_count : a.n;
    const double tol2 = ctl.outer_tolerance * ctl.outer_tolerance;

    for (;;) {
        int job = 0;
        if (Q.q == 0) job = int(atomicAdd(a.queue, 1u));
        job = Q.from(job, 0);
        if (job >= total) break;
        const size_t i = size_t(a.list ? a.list[job] : job);

        // ---- inputs and bounds of this lane's slice
        double target64 = colour ? a.image[3 * i + Q.q] : 0.0;
        double ahat64[L], bg64 = 0.0;
        S.target = T(target64);
        if (REFINE && a.smooth && colour) bg64 = a.targets[(size_t(L) + Q.q) * n + i];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            ahat64[l] = REFINE ? a.targets[size_t(l) * n + i] : 0.0;
            if (REFINE && a.opaque && l == 0) ahat64[l] = 1.0;
            S.ahat[l] = T(ahat64[l]);
            T lo = T(0), hi = T(1), init;
            if (colour) {
                if (REFINE && a.smooth && l == 0) lo = hi = T(bg64);
                if (REFINE) init = (a.smooth && l == 0) ? T(bg64) : T(a.first[(size_t(l) * n + i) * 4 + Q.q]);
                else init = fmin(T(1), fmax(T(0), sel3(Q.q, m.mean[l][0], m.mean[l][1], m.mean[l][2])));
            } else {
                if (a.opaque && l == 0) lo = hi = T(1);
                else if (REFINE) lo = hi = S.ahat[l];
                init = (a.opaque && l == 0) ? T(1) : (REFINE ? S.ahat[l] : T(0.5));
            }
            S.lo[l] = lo; S.hi[l] = hi; S.init[l] = init;
        }

        const bool skip = REFINE && a.input_status && a.input_status[i] != 0;
        if (skip) {
            // Targets that cannot be normalized: keep the initial layers and
            // report status 8, as the reference's guard does (solver_workspace.cuh:144).
            S.have_best = false;
            S.n_values = S.n_gradients = S.n_iterations = S.n_backtracks = S.n_outer = 0;
        } else {
            S.run();
        }

        // ---- output: packed f64 [l][i][RGBA]; pinned values written exactly
        double v[L];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            v[l] = double(S.have_best ? S.best[l] : S.init[l]);
            if (REFINE && !colour) v[l] = ahat64[l];
            if (REFINE && a.smooth && colour && l == 0) v[l] = bg64;
            if (!REFINE && a.opaque && !colour && l == 0) v[l] = 1.0;
            a.out[(size_t(l) * n + i) * 4 + Q.q] = v[l];
        }
        const double norm = constraint_norm2_fp64<L, REFINE>(Q, m.mode, m.X, m.Y, m.Z, v, target64, ahat64);
        const bool miss = !(norm < tol2);
        if (Q.q == 0) {
            if (skip) {
                if (a.status) a.status[i] = 8;
                if (a.input_failed) atomicAdd(a.input_failed, 1);
            } else {
                if (a.status) a.status[i] = miss ? 3 : 0;
                if (miss && a.miss_list) a.miss_list[atomicAdd(a.miss_count, 1)] = int32_t(i);
            }
            if (a.counters) {
                uint32_t* c = a.counters + 5 * i;
                c[0] = S.n_values; c[1] = S.n_gradients; c[2] = S.n_iterations; c[3] = S.n_backtracks; c[4] = S.n_outer;
            }
        }
    }
}

template <class T, int L, bool REFINE, bool HSMEM> struct SolveLauncher {
    static size_t smem_bytes(int threads) { return HSMEM ? size_t(threads) * kHistory * L * 2 * sizeof(T) : 0; }

    static cudaError_t occupancy(int threads, int* blocks_per_sm) {
        auto k = solve_pixels<T, L, REFINE, HSMEM>;
        const size_t sm = smem_bytes(threads);
        if (sm > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
            if (e != cudaSuccess) return e;
        }
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, sm);
    }

    static cudaError_t launch(const Models<T>& m, const SolverControls& ctl, const SolveArgs& a, int blocks,
                              int threads, cudaStream_t stream) {
        auto k = solve_pixels<T, L, REFINE, HSMEM>;
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
