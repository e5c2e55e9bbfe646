// Per-pixel augmented-Lagrangian / projected L-BFGS solve on a 4-lane quad.
//
// Method (the reference's own, augmented_lagrangian.cuh:20-149 and
// pixel_problem.cuh:60-117): minimise
//     E(x) = sum_l alpha_l (c_l - mu_l)^T P_l (c_l - mu_l)  [+ 0.01 sum_l alpha_l when unmixing]
// subject to  composite(x) = target  (3 rows)  and  A_final = 1 (unmixing) or
// alpha_l = alpha_hat_l (refinement), with x in its bounds, by an AL outer
// loop (rho0 = 100, lambda -= rho C, rho *= 10 when |C|^2 > 0.0625 |C_prev|^2,
// at most 22 outer steps) around a projected L-BFGS inner solve (memory 6,
// Armijo c = 1e-4, up to 32 halvings and one steepest-descent retry, at most
// 256 iterations, relative tolerance 5e-3), several optional starts and
// best-feasible tracking over every evaluated point.
//
// B200 mapping: one pixel per quad of lanes. Lanes 0..2 own colour channel
// q of every layer (x = c_{l,q}, l = 0..L-1); lane 3 owns the alphas
// (x = alpha_l). Every vector of the method (x, gradient, direction, trial
// point, best point, the L-BFGS history) is split the same way, so dot
// products are a local sum plus two xor-shuffles and each lane keeps only L
// values of every vector. The five vectors the inner loop touches on every
// step (x, gradient, direction, trial point, trial gradient) live in
// registers; the cold ones (best point, the outer step's start point, the
// start-0 seed) live in a per-lane shared-memory slice,
// and so does the L-BFGS history in the shared-history variants (the
// register variant keeps it as a shift register). The composite is separable
// per channel given the alphas, which lane 3 broadcasts; the 3x3 colour prior
// needs the three deltas of a layer (two shuffles); the adjoint sweep reduces
// the alpha sensitivities of the three channels once per layer. Every branch
// is taken on quad-uniform values, so a quad never splits.
//
// Lockstep: every trip of the warp's loop performs exactly one objective
// evaluation per quad (the gradient half predicated on the quads that need
// it), followed by the evaluation-free bookkeeping of that quad. The
// bookkeeping is a small action machine (begin iteration, next line-search
// trial, accept, end of an outer step, begin start, begin outer step, store,
// fetch) run until the quad needs its next evaluation; each action's code
// exists once in the kernel, which keeps the loop's instruction footprint
// small enough for the instruction cache. A quad whose pixel is finished
// pulls the next pixel from an atomic queue; the warp leaves the loop when
// every quad is idle. The evaluated points and every decision are those of
// the reference method, step for step; the one evaluation left out is the
// re-evaluation at the end of an outer step, at a point already evaluated,
// whose residual the state keeps instead.
#pragma once
#include "blend.cuh"
#include "common.cuh"

namespace unb {

template <class T> __device__ __forceinline__ T sel3(int q, T a, T b, T c) { return q == 0 ? a : (q == 1 ? b : c); }

template <class T> __device__ __forceinline__ bool finite_(T v);
template <> __device__ __forceinline__ bool finite_<float>(float v) { return isfinite(v); }
template <> __device__ __forceinline__ bool finite_<double>(double v) { return isfinite(v); }

// a*b + c: one fused operation in the FP32 solver (shorter dependency chains,
// fewer instructions; the same in every kernel variant); a rounded multiply
// then a rounded add in FP64, as the reference computes it. Every FP64
// expression written with madd below keeps the reference's operation order
// (addition commutes exactly in IEEE arithmetic).
template <class T> __device__ __forceinline__ T madd(T a, T b, T c);
template <> __device__ __forceinline__ float madd<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <> __device__ __forceinline__ double madd<double>(double a, double b, double c) {
    return __dadd_rn(__dmul_rn(a, b), c);
}

// The FP64 blend functions (a switch over the thirteen modes) out of line:
// one copy of each serves every unrolled layer, which keeps the solver's loop
// small for the instruction cache. The FP32 solver uses blend_table.
template <class T> __device__ __noinline__ T blend_value_call(int mode, T s, T d) { return blend_value<T>(mode, s, d); }
template <class T> __device__ __noinline__ void blend_all_call(int mode, T s, T d, T& f, T& fs, T& fd) { blend_all<T>(mode, s, d, f, fs, fd); }

// Dynamic shared memory of the solve kernels (one declaration for all of
// them; addressed by thread index, so no pointer stays live in registers).
extern __shared__ __align__(16) unsigned char solver_smem[];

// Where the L-BFGS history lives: registers (a shift register), the lane's
// shared-memory slice, or a per-lane global-memory array (coalesced across
// lanes, served by L1/L2), which frees shared memory for more resident
// blocks when the values are wide (FP64).
enum : int { kHistRegisters = 0, kHistShared = 1, kHistGlobal = 2 };
// Storage policy of a solve kernel: a history place, optionally with
// kVectorsShared, which keeps the iterate x, its gradient g and the search
// direction d (vectors the evaluation does not touch) in the lane's
// shared-memory slice instead of registers.
enum : int { kVectorsShared = 4 };
// kRolled: the evaluation runs rolled over the layers, its per-layer
// intermediates in the lane's slice (one copy of each layer's code: a smaller
// instruction footprint for more shared memory).
enum : int { kRolled = 8 };
// kTriple (refinement only): three lanes per pixel, the colour channels; the
// pinned alphas need no lane (see Group).
enum : int { kTriple = 16 };
// kColdGlobal (with global history): the cold values (best point, outer-step
// start, start-0 seed) follow the history in the lane's global array, which
// shrinks the shared-memory slice; with kBookRolled and three lanes, so does
// the pinned alphas' gradient at x.
enum : int { kColdGlobal = 32 };
// kBookRolled (with kVectorsShared, kRolled and the global history): the
// trial point and the trial gradient live only in the lane's slice (the
// rolled evaluation's slots), so every per-layer loop of the bookkeeping
// runs rolled: one copy of each loop body instead of L, a smaller
// instruction footprint and fewer registers, the same operations in the same
// order.
enum : int { kBookRolled = 64 };
constexpr int history_of(int storage) { return storage & 3; }

// The lanes of one pixel. G = 4 (a quad, lanes 0..2 colour channels, lane 3
// the alphas): sums are xor-trees, identical on every lane. G = 3 (the
// refinement of pinned alphas: colour channels only, 10 pixels per warp,
// lanes 30-31 idle): sums gather the three values and add them in one fixed
// order, so every lane holds the identical result.
template <int G> struct Group {
    unsigned mask;
    int base, q;
    bool extra;   // a lane of no group (G = 3: lanes 30 and 31)
    __device__ __forceinline__ Group() {
        const int lane = threadIdx.x & 31;
        base = lane / G * G;
        q = lane - base;
        extra = G != 4 && base + G > 32;
        mask = extra ? 0u : ((1u << G) - 1u) << base;
    }
    template <class T> __device__ __forceinline__ T sum(T v) const {
        if constexpr (G == 4) {
            v += __shfl_xor_sync(mask, v, 1);
            v += __shfl_xor_sync(mask, v, 2);
            return v;
        } else {
            const T a0 = __shfl_sync(mask, v, base), a1 = __shfl_sync(mask, v, base + 1),
                    a2 = __shfl_sync(mask, v, base + 2);
            return (a0 + a1) + a2;
        }
    }
    template <class T> __device__ __forceinline__ void sum2(T& a, T& b) const {
        if constexpr (G == 4) {
            a += __shfl_xor_sync(mask, a, 1); b += __shfl_xor_sync(mask, b, 1);
            a += __shfl_xor_sync(mask, a, 2); b += __shfl_xor_sync(mask, b, 2);
        } else { a = sum(a); b = sum(b); }
    }
    template <class T> __device__ __forceinline__ void sum3(T& a, T& b, T& c) const {
        if constexpr (G == 4) {
            a += __shfl_xor_sync(mask, a, 1); b += __shfl_xor_sync(mask, b, 1); c += __shfl_xor_sync(mask, c, 1);
            a += __shfl_xor_sync(mask, a, 2); b += __shfl_xor_sync(mask, b, 2); c += __shfl_xor_sync(mask, c, 2);
        } else { a = sum(a); b = sum(b); c = sum(c); }
    }
    template <class T> __device__ __forceinline__ void sum4(T& a, T& b, T& c, T& d) const {
        if constexpr (G == 4) {
            a += __shfl_xor_sync(mask, a, 1); b += __shfl_xor_sync(mask, b, 1);
            c += __shfl_xor_sync(mask, c, 1); d += __shfl_xor_sync(mask, d, 1);
            a += __shfl_xor_sync(mask, a, 2); b += __shfl_xor_sync(mask, b, 2);
            c += __shfl_xor_sync(mask, c, 2); d += __shfl_xor_sync(mask, d, 2);
        } else { a = sum(a); b = sum(b); c = sum(c); d = sum(d); }
    }
    template <class T> __device__ __forceinline__ T max(T v) const {
        if constexpr (G == 4) {
            v = fmax(v, __shfl_xor_sync(mask, v, 1));
            v = fmax(v, __shfl_xor_sync(mask, v, 2));
            return v;
        } else {
            const T a0 = __shfl_sync(mask, v, base), a1 = __shfl_sync(mask, v, base + 1),
                    a2 = __shfl_sync(mask, v, base + 2);
            return fmax(fmax(a0, a1), a2);
        }
    }
    template <class T> __device__ __forceinline__ T from(T v, int src) const {
        return __shfl_sync(mask, v, base + src);
    }
};

// L-BFGS pairs, indexed by age j (0 = newest). Register form: a shift
// register with compile-time indices. Shared-memory form: a ring buffer in
// the lane's slice after its cold values, element (slot, l, s|y) at
// slice index 3L + (slot*L + l)*2 + w. Global form: the same ring buffer in
// SolveArgs::history, element k of lane g at [k * lanes + g] with
// g = blockIdx.x * kSliceStride + threadIdx.x and lanes = gridDim.x * kSliceStride.
template <class T, int L, int HS, int BASE> struct History;

template <class T, int L, int BASE> struct History<T, L, kHistRegisters, BASE> {
    T s_[kHistory][L], y_[kHistory][L];
    __device__ __forceinline__ void init(void*) {}
    __device__ __forceinline__ T s(int j, int l) const { return s_[j][l]; }
    __device__ __forceinline__ T y(int j, int l) const { return y_[j][l]; }
    __device__ __forceinline__ void push(const T* sv, const T* yv) {
#pragma unroll
        for (int j = kHistory - 1; j > 0; --j)
#pragma unroll
            for (int l = 0; l < L; ++l) { s_[j][l] = s_[j - 1][l]; y_[j][l] = y_[j - 1][l]; }
#pragma unroll
        for (int l = 0; l < L; ++l) { s_[0][l] = sv[l]; y_[0][l] = yv[l]; }
    }
    __device__ __forceinline__ void reset() {}
};

template <class T, int L, int BASE> struct History<T, L, kHistShared, BASE> {
    static constexpr int kBase = BASE;    // slice index of the ring buffer
    int next;
    // This lane's pair of age j: element l of s at row(j)[2*l*kSliceStride],
    // of y at row(j)[(2*l + 1)*kSliceStride].
    __device__ __forceinline__ T* row(int j) const {
        int k = next - 1 - j;
        k = k < 0 ? k + kHistory : k;
        return reinterpret_cast<T*>(solver_smem) + (kBase + k * 2 * L) * kSliceStride + threadIdx.x;
    }
    __device__ __forceinline__ void init(void*) { next = 0; }
    __device__ static constexpr int stride() { return kSliceStride; }
    __device__ __forceinline__ T s(int j, int l) const { return row(j)[2 * l * kSliceStride]; }
    __device__ __forceinline__ T y(int j, int l) const { return row(j)[(2 * l + 1) * kSliceStride]; }
    __device__ __forceinline__ void push(const T* sv, const T* yv) {
        T* p = reinterpret_cast<T*>(solver_smem) + (kBase + next * 2 * L) * kSliceStride + threadIdx.x;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            p[2 * l * kSliceStride] = sv[l];
            p[(2 * l + 1) * kSliceStride] = yv[l];
        }
        next = next + 1 == kHistory ? 0 : next + 1;
    }
    __device__ __forceinline__ void reset() { next = 0; }
};

template <class T, int L, int BASE> struct History<T, L, kHistGlobal, BASE> {
    T* base;       // this lane's element 0
    int lanes;     // element stride
    int next;
    __device__ __forceinline__ void init(void* h) {
        lanes = int(gridDim.x) * kSliceStride;
        base = static_cast<T*>(h) + blockIdx.x * kSliceStride + threadIdx.x;
        next = 0;
    }
    __device__ __forceinline__ int stride() const { return lanes; }
    __device__ __forceinline__ T* row(int j) const {
        int k = next - 1 - j;
        k = k < 0 ? k + kHistory : k;
        return base + size_t(k * 2 * L) * lanes;
    }
    __device__ __forceinline__ T s(int j, int l) const { return row(j)[size_t(2 * l) * lanes]; }
    __device__ __forceinline__ T y(int j, int l) const { return row(j)[size_t(2 * l + 1) * lanes]; }
    __device__ __forceinline__ void push(const T* sv, const T* yv) {
        T* p = base + size_t(next * 2 * L) * lanes;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            p[size_t(2 * l) * lanes] = sv[l];
            p[size_t(2 * l + 1) * lanes] = yv[l];
        }
        next = next + 1 == kHistory ? 0 : next + 1;
    }
    // The same one element at a time (rolled loops), then advance().
    __device__ __forceinline__ void push_elem(int l, T sv, T yv) {
        T* p = base + size_t(next * 2 * L) * lanes;
        p[size_t(2 * l) * lanes] = sv;
        p[size_t(2 * l + 1) * lanes] = yv;
    }
    __device__ __forceinline__ void advance() { next = next + 1 == kHistory ? 0 : next + 1; }
    __device__ __forceinline__ void reset() { next = 0; }
};

// Per-lane shared-memory slice of the solver: kValues values of T (cold
// values; the L-BFGS history when it is kept in shared memory; the two-loop
// coefficients when the history is not in registers); element k of a lane
// at [k * kSliceStride + threadIdx.x] (consecutive lanes, consecutive words).
// A batched launch places one layer-model slot per quad after the slices.
template <class T, int L, int S> struct LaneSlice {
    static constexpr int kCold = (S & kColdGlobal) ? 0 : 3 * L;          // best, outer-start point, start-0 seed
    static constexpr int kVec = kCold;                                   // x, g, d (kVectorsShared)
    static constexpr int kHist = kVec + ((S & kVectorsShared) ? 3 * L : 0);   // history ring (shared history)
    static constexpr int kCoeff = kHist + (history_of(S) == kHistShared ? 2 * kHistory * L : 0);   // two-loop coefficients
    // Rolled evaluation (kRolled): per-layer intermediates (trial point,
    // alphas, composite alpha and colour, trial gradient) in the slice.
    static constexpr bool kRolledEval = (S & kRolled) != 0;
    static constexpr int kScratch = history_of(S) == kHistRegisters ? kHist : kCoeff + 2 * kHistory;
    // kBookRolled with three lanes: the pinned alphas' gradient at x.
    static constexpr int kGa3 = kScratch + (kRolledEval ? 5 * L : 0);
    // (with kColdGlobal that slot follows the cold values in the global array)
    static constexpr int kValues = kGa3 + (((S & kBookRolled) && (S & kTriple) && !(S & kColdGlobal)) ? L : 0);
    __device__ __forceinline__ static T& value(int k) {
        return reinterpret_cast<T*>(solver_smem)[k * kSliceStride + threadIdx.x];
    }
    __host__ __device__ static constexpr size_t value_bytes() {
        return (size_t(kSliceStride) * kValues * sizeof(T) + 15) / 16 * 16;
    }
    __host__ __device__ static constexpr size_t bytes() { return value_bytes(); }
};

enum : int { kIdle = 0, kOuterEval = 1, kTrial = 2, kAcceptGrad = 3 };
// Bookkeeping actions; aEval hands the quad to the next evaluation.
enum : int { aEval = 0, aBeginIter, aNextTrial, aAccept, aEndOuter, aBeginStart, aBeginOuter, aFinish, aFetch };

// BATCH: pixels of many images (one layer-count group); the quad's layer
// models are those of its current image in the device model table.
// MODE: kPlain; kDefers, a launch that defers pixels (SolveArgs::defer_*);
// kResumes, the launch that resumes them. Only the code a mode runs is
// compiled into its kernel.
enum : int { kPlain = 0, kDefers = 1, kResumes = 2 };

template <class T, int L, bool REFINE, int S, bool BATCH = false, int MODE = kPlain> struct QuadSolver {
    // Residual rows of a lane: the alpha lane of a refinement owns the L rows
    // of the pinned alphas; a colour lane owns one (three-lane groups have
    // colour lanes only). RA: the pinned alphas a lane keeps.
    static constexpr int R = (REFINE && (S & kTriple) == 0) ? L : 1;
    static constexpr int RA = REFINE ? L : 1;
    static constexpr int kLanes = (S & kTriple) ? 3 : 4;   // lanes per pixel
    static_assert(kLanes == 4 || (REFINE && !BATCH), "three-lane groups serve the refinement only");
    using Slice = LaneSlice<T, L, S>;
    static constexpr int HS = history_of(S);
    static constexpr bool VS = (S & kVectorsShared) != 0;
    static constexpr bool BR = (S & kBookRolled) != 0;
    static_assert(!BR || (VS && (S & kRolled) && HS == kHistGlobal && (!REFINE || kLanes == 3)),
                  "rolled bookkeeping: x, g, d and the evaluation in the slice, global history, no alpha lane with "
                  "pinned alphas");
    // Unroll factors of the per-layer bookkeeping loops: kU for loops over
    // registers and shared memory (rolled with BR); kUC for loops over the cold
    // values, which stay unrolled when they live in global memory so that
    // their loads issue together.
    static constexpr int kU = BR ? 1 : L;
    static constexpr int kUC = (BR && (S & kColdGlobal) == 0) ? 1 : L;
    // The two-loop recursion's per-layer loops over the global history: rolled
    // in the three-lane refinement (measured faster: 102.5 against 106.5 ms on
    // the 1024x1024 five-layer image), unrolled in the first pass (145 against
    // 166 ms: its history loads then issue together).
    static constexpr int kUT = (BR && kLanes == 3) ? 1 : L;
    const Models<T>* models_;
    const Models<T>* batch_models_ = nullptr;   // batched launch: the current image's models
    const SolverControls& ctl;
    const SolveArgs& a;
    Group<kLanes> Q;
    bool colour, opaque, smooth;
    T tol2, itol;
    // Evaluations of this lane's pixels (lane q = 0 counts), with a value and
    // with a gradient, for SolveArgs::tally.
    uint32_t n_value = 0, n_grad = 0;

    // Current pixel (this lane's slice of it).
    int pixel = 0, gidx = 0;   // pixel index within its image, queue index
    int job_id = -1;
    T target, bgq;
    T ahat[RA];          // refinement: filtered alpha targets (pinned alphas)

    // Method state (this lane's slice).
    mutable T xr_[VS ? 1 : L], gr_[VS ? 1 : L], dr_[VS ? 1 : L];   // x, g, d in registers (!VS)
    mutable T tr_[BR ? 1 : L], ng_[BR ? 1 : L];   // trial point and gradient in registers (!BR)
    T lam[R], res[R], resx[R];   // multipliers, residual of the last evaluation, residual at x
    // G = 3: every lane's copy of the (pinned) alphas' gradient at x and at the
    // trial point; they enter only y.y of the curvature pairs.
    mutable T ga3_[(kLanes == 3 && !BR) ? L : 1], na3_[(kLanes == 3 && !BR) ? L : 1];
    History<T, L, HS, Slice::kHist> hist;

    // Per-quad scalars (uniform within the quad).
    int phase, start, outer, it, attempt, bt, valid;
    int frozen;      // consecutive outer steps that moved neither x nor the best point
    bool best_moved; // the best point changed during this outer step
    T rho, f, oldnorm, step, slope, cand;
    T best_norm, best_energy;
    bool have_best;
    bool capped;     // stopped unconverged at a shortened outer cap (counts as a miss)

    __device__ QuadSolver(const Models<T>* models, const SolverControls& c, const SolveArgs& args)
        : models_(models), ctl(c), a(args) {
        colour = kLanes == 3 || Q.q < 3;
        opaque = a.opaque != 0;
        smooth = a.smooth != 0;
        tol2 = T(ctl.outer_tolerance * ctl.outer_tolerance);
        itol = T(ctl.inner_tolerance);
        phase = kIdle;
        hist.init(a.history);
        // Batched: every lane evaluates on every trip, including the lanes of
        // a quad that has not fetched a pixel yet (or never will, in a batch
        // smaller than the grid), so the models point at a valid entry from
        // the start.
        if constexpr (BATCH) batch_models_ = static_cast<const Models<T>*>(a.models);
    }

    // The layer models: the kernel parameter, or (batched launch) the
    // current image's entry of the device model table (read through L1; the
    // quads of a warp mostly share it).
    __device__ __forceinline__ const Models<T>& models() const {
        if constexpr (BATCH) return *batch_models_;
        else return *models_;
    }

    // ------------------------------------------------------ cold values --
    __device__ __forceinline__ T& X(int l) const { if constexpr (VS) return Slice::value(Slice::kVec + l); else return xr_[l]; }
    __device__ __forceinline__ T& G(int l) const { if constexpr (VS) return Slice::value(Slice::kVec + L + l); else return gr_[l]; }
    __device__ __forceinline__ T& D(int l) const { if constexpr (VS) return Slice::value(Slice::kVec + 2 * L + l); else return dr_[l]; }
    __device__ __forceinline__ T& cold(int k) const {
        if constexpr ((S & kColdGlobal) != 0) {
            static_assert(HS == kHistGlobal, "global cold values follow a global history");
            return hist.base[size_t(2 * kHistory * L + k) * hist.lanes];
        } else {
            return Slice::value(k);
        }
    }
    // The trial point, the trial gradient and (G = 3) the pinned alphas'
    // gradient at the trial point and at x: registers, or the slice (BR).
    __device__ __forceinline__ T& TRv(int l) const {
        if constexpr (BR) return Slice::value(Slice::kScratch + l); else return tr_[l];
    }
    __device__ __forceinline__ T& NGv(int l) const {
        if constexpr (BR) return Slice::value(Slice::kScratch + 4 * L + l); else return ng_[l];
    }
    __device__ __forceinline__ T& NA3(int l) const {
        if constexpr (BR) return Slice::value(Slice::kScratch + L + l); else return na3_[l];
    }
    __device__ __forceinline__ T& GA3(int l) const {
        if constexpr (BR && (S & kColdGlobal) != 0) return hist.base[size_t(2 * kHistory * L + 3 * L + l) * hist.lanes];
        else if constexpr (BR) return Slice::value(Slice::kGa3 + l);
        else return ga3_[l];
    }
    __device__ __forceinline__ T& best(int l) const { return cold(l); }
    __device__ __forceinline__ T& ox(int l) const { return cold(L + l); }
    __device__ __forceinline__ T& init(int l) const { return cold(2 * L + l); }
    // Work counters go straight to SolveArgs::counters (only when requested).
    __device__ __forceinline__ uint32_t& counter(int k) const { return a.counters[5 * size_t(gidx) + k]; }
    __device__ __forceinline__ void count(int k) const { if (a.counters && Q.q == 0) ++counter(k); }

    // ------------------------------------------------- image accessors --
    __device__ __forceinline__ const double* image() const {
        if constexpr (BATCH) return a.jobs[job_id].image; else return a.image;
    }
    __device__ __forceinline__ double* output() const {
        if constexpr (BATCH) return a.jobs[job_id].out; else return a.out;
    }
    __device__ __forceinline__ int32_t* status() const {
        if constexpr (BATCH) return a.jobs[job_id].status; else return a.status;
    }
    __device__ __forceinline__ const float* warm() const {
        if constexpr (BATCH) return a.jobs[job_id].warm; else return a.warm;
    }
    __device__ __forceinline__ size_t pixels() const {
        if constexpr (BATCH) return job_id < 0 ? size_t(0) : size_t(a.jobs[job_id].n);
        else return size_t(a.n);
    }

    // ------------------------------------------------------------ bounds --
    __device__ __forceinline__ T lo(int l) const {
        if (kLanes == 3 || colour) return (REFINE && smooth && l == 0) ? bgq : T(0);
        if (opaque && l == 0) return T(1);
        return REFINE ? ahat[REFINE ? l : 0] : T(0);
    }
    __device__ __forceinline__ T hi(int l) const {
        if (kLanes == 3 || colour) return (REFINE && smooth && l == 0) ? bgq : T(1);
        if (opaque && l == 0) return T(1);
        return REFINE ? ahat[REFINE ? l : 0] : T(1);
    }
    __device__ __forceinline__ T clampb(int l, T v) const {
        const T lv = lo(l), hv = hi(l);
        return v < lv ? lv : (v > hv ? hv : v);
    }
    __device__ __forceinline__ bool fixed_at(int l, T gl) const {
        const T lv = lo(l), hv = hi(l);
        return lv == hv || (X(l) <= lv && gl > T(0)) || (X(l) >= hv && gl < T(0));
    }
    // Alpha of layer l at the point whose lane-3 slice is v (G = 4), or the
    // pinned alpha (G = 3).
    __device__ __forceinline__ T alpha_at(T v, int l) const {
        if constexpr (kLanes == 3) return ahat[REFINE ? l : 0];
        else return Q.from(v, 3);
    }
    __device__ __forceinline__ T mean_of(const Models<T>& m, int l) const {
        return colour ? sel3(Q.q, m.mean[l][0], m.mean[l][1], m.mean[l][2]) : T(0);
    }

    // FP32: table-driven blend and reciprocal-based division; FP64: the
    // reference's formulas with IEEE division.
    static constexpr bool kFast = sizeof(T) == 4;
    __device__ __forceinline__ T blend(const Models<T>& m, int l, T s, T d) const {
        if constexpr (kFast) { T f, fs, fd; blend_table<T>(m, l, s, d, f, fs, fd, false); return f; }
        else return blend_value_call<T>(m.mode[l], s, d);
    }
    __device__ __forceinline__ void blend3(const Models<T>& m, int l, T s, T d, T& f, T& fs, T& fd) const {
        if constexpr (kFast) blend_table<T>(m, l, s, d, f, fs, fd, true);
        else blend_all_call<T>(m.mode[l], s, d, f, fs, fd);
    }

    // The same, with the FP64 switch inline (the rolled evaluation has one
    // copy of each layer's code).
    __device__ __forceinline__ T blend_inline(const Models<T>& m, int l, T s, T d) const {
        if constexpr (kFast) return blend(m, l, s, d);
        else return blend_value<T>(m.mode[l], s, d);
    }
    __device__ __forceinline__ void blend3_inline(const Models<T>& m, int l, T s, T d, T& f, T& fs, T& fd) const {
        if constexpr (kFast) blend3(m, l, s, d, f, fs, fd);
        else blend_all<T>(m.mode[l], s, d, f, fs, fd);
    }

    // sy > 1e-9 sqrt(ss yy) and sy > 0 (augmented_lagrangian.cuh:193,290); the
    // FP32 solver compares squares instead of taking the root.
    __device__ __forceinline__ static bool curvature_ok(T sy, T ss, T yy) {
        if constexpr (kFast) return sy > T(0) && sy * sy > T(1e-18) * (ss * yy);
        else return sy > T(1e-9) * dsqrt(ss * yy) && sy > T(0);
    }

    // G = 3, reverse sweep, layer l: the alpha chain's sensitivities from the
    // three channels' terms (ga, gp of this lane), summed in the reference's
    // order (alpha term, then channels 0, 1, 2; pixel_problem.cuh:96-106), on
    // every lane.
    __device__ __forceinline__ void alpha_chain(int l, T da, T db, T ga, T gp, T& adj3, T& nal) const {
        const T a0 = Q.from(ga, 0), a1 = Q.from(ga, 1), a2 = Q.from(ga, 2);
        const T p0 = Q.from(gp, 0), p1 = Q.from(gp, 1), p2 = Q.from(gp, 2);
        T ta = adj3 * da, tp = adj3 * db;
        ta += a0; ta += a1; ta += a2;
        tp += p0; tp += p1; tp += p2;
        nal += ta;
        adj3 = tp;
        (void)l;
    }

    // ---------------------------------------------------------- evaluate --
    // Constraint rows, the AL value and best-point tracking of an evaluation
    // whose composite ended at alpha Afin and (this lane's channel) colour cfin.
    __device__ __forceinline__ T residual_value(T energy, T Afin, T cfin, bool need_grad, bool active) {
        T terms = T(0), norm = T(0);
        if (colour) {
            res[0] = cfin - target;
            terms = madd(T(0.5) * rho * res[0], res[0], -(lam[0] * res[0]));
            norm = res[0] * res[0];
        } else if (REFINE) {
#pragma unroll
            for (int l = 0; l < R; ++l) {
                res[l] = TRv(l) - ahat[l];
                terms += madd(T(0.5) * rho * res[l], res[l], -(lam[l] * res[l]));
                norm = madd(res[l], res[l], norm);
            }
        } else {
            res[0] = Afin - T(1);
            terms = madd(T(0.5) * rho * res[0], res[0], -(lam[0] * res[0]));
            norm = res[0] * res[0];
        }
        Q.sum2(terms, norm);
        const T value = energy + terms;
        if (active) {
            count(0);
            if (need_grad) count(1);
            if (Q.q == 0) { ++n_value; if (need_grad) ++n_grad; }
            const bool feasible = norm < tol2;
            if (finite_(energy) && finite_(norm) &&
                (!have_best || (feasible && (best_norm >= tol2 || energy < best_energy)) ||
                 (!feasible && best_norm >= tol2 && norm < best_norm))) {
                have_best = true; best_norm = norm; best_energy = energy;
                best_moved = true;
#pragma unroll kUC
                for (int l = 0; l < L; ++l) best(l) = TRv(l);
            }
        }
        return value;
    }

    // Evaluates the AL value at tr (uniform across the quad), sets res[] and,
    // when need_grad, the gradient slice ng[]. Tracks the best feasible point.
    __device__ __forceinline__ T evaluate(bool need_grad, bool active) {
        if constexpr (Slice::kRolledEval) return evaluate_rolled(need_grad, active);
        const Models<T>& m = models();
        T al[L], A[L], pc[L];
#pragma unroll
        for (int l = 0; l < L; ++l) al[l] = alpha_at(TRv(l), l);
        A[0] = al[0];
        pc[0] = TRv(0);
#pragma unroll
        for (int l = 1; l < L; ++l) {
            const T av = al[l], dd = A[l - 1];
            // X a d + Y a (1 - d) + Z d (1 - a), and the colour the same way.
            const T Al = madd(T(m.Z[l]) * dd, T(1) - av, madd(T(m.X[l]) * av, dd, T(m.Y[l]) * av * (T(1) - dd)));
            A[l] = Al;
            const T s = TRv(l), c = pc[l - 1];
            const T pre = madd(T(m.Z[l]) * dd * (T(1) - av), c,
                               madd(blend(m, l, s, c) * av, dd, T(m.Y[l]) * av * (T(1) - dd) * s));
            pc[l] = Al > T(1e-12) ? qdiv(pre, Al) : pre;
        }
        T energy = T(0), asum = T(0);
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const T mine = colour ? TRv(l) - mean_of(m, l) : T(0);
            const T d0 = Q.from(mine, 0), d1 = Q.from(mine, 1), d2 = Q.from(mine, 2);
            const T* P = m.prec[l];
            const T v0 = madd(P[2], d2, madd(P[0], d0, P[1] * d1));
            const T v1 = madd(P[5], d2, madd(P[3], d0, P[4] * d1));
            const T v2 = madd(P[8], d2, madd(P[6], d0, P[7] * d1));
            const T D = madd(d2, v2, madd(d0, v0, d1 * v1));
            energy = madd(al[l], D, energy);
            asum += al[l];
            if (need_grad) {
                if (colour) {
                    const T vq = sel3(Q.q, v0, v1, v2);
                    const T tq = madd(sel3(Q.q, P[6], P[7], P[8]), d2,
                                      madd(sel3(Q.q, P[0], P[1], P[2]), d0, sel3(Q.q, P[3], P[4], P[5]) * d1));
                    NGv(l) = al[l] * (vq + tq);
                } else {
                    NGv(l) = D + (REFINE ? T(0) : T(0.01));
                }
                if constexpr (kLanes == 3) NA3(l) = D;
            }
        }
        if (!REFINE) energy += T(0.01) * asum;
        const T value = residual_value(energy, A[L - 1], pc[L - 1], need_grad, active);
        if (need_grad) {
            T adj = colour ? rho * res[0] - lam[0] : T(0);
            T adj3 = (!colour && !REFINE) ? rho * res[0] - lam[0] : T(0);
            if (REFINE && !colour)
#pragma unroll
                for (int l = 0; l < R; ++l) NGv(l) += rho * res[l] - lam[l];
#pragma unroll
            for (int l = L - 1; l > 0; --l) {
                const T av = al[l], dd = A[l - 1], Al = A[l];
                const T X = T(m.X[l]), Y = T(m.Y[l]), Z = T(m.Z[l]);
                const T da = madd(X, dd, Y * (T(1) - dd)) - Z * dd;
                const T db = madd(Z, T(1) - av, X * av - Y * av);
                const bool big = Al > T(1e-12);
                T ga, gp;
                if constexpr (kFast) {
                    // FP32: the colour channel terms on all four lanes without
                    // a branch (lane 3 would idle through them anyway; its
                    // values are replaced by the alpha chain's terms below).
                    const T s = TRv(l), c = pc[l - 1], out = pc[l], v = adj;
                    T fv, fs, fd;
                    blend3(m, l, s, c, fv, fs, fd);
                    const T ds = madd(av * dd, fs, Y * av * (T(1) - dd));
                    const T dc = madd(av * dd, fd, Z * dd * (T(1) - av));
                    const T pa = madd(fv, dd, Y * (T(1) - dd) * s) - Z * dd * c;
                    const T pd = madd(Z * (T(1) - av), c, fv * av - Y * av * s);
                    const T r = big ? qdiv(T(1), Al) : T(1);
                    T gs, ad;
                    if (big) {
                        ga = v * (madd(-out, da, pa) * r);
                        gp = v * (madd(-out, db, pd) * r);
                        gs = v * (ds * r);
                        ad = v * (dc * r);
                    } else {
                        ga = v * pa; gp = v * pd; gs = v * ds; ad = v * dc;
                    }
                    if (colour) { NGv(l) += gs; adj = ad; }
                    else { ga = adj3 * da; gp = adj3 * db; }
                } else if (colour) {
                    const T s = TRv(l), c = pc[l - 1], out = pc[l], v = adj;
                    T fv, fs, fd;
                    blend3(m, l, s, c, fv, fs, fd);
                    const T ds = madd(av * dd, fs, Y * av * (T(1) - dd));
                    const T dc = madd(av * dd, fd, Z * dd * (T(1) - av));
                    const T pa = madd(fv, dd, Y * (T(1) - dd) * s) - Z * dd * c;
                    const T pd = madd(Z * (T(1) - av), c, fv * av - Y * av * s);
                    if (big) {
                        ga = v * ((pa - out * da) / Al);
                        gp = v * ((pd - out * db) / Al);
                        NGv(l) += v * (ds / Al);
                        adj = v * (dc / Al);
                    } else {
                        ga = v * pa; gp = v * pd;
                        NGv(l) += v * ds;
                        adj = v * dc;
                    }
                } else {
                    ga = adj3 * da;
                    gp = adj3 * db;
                }
                if constexpr (kLanes == 4) {
                    Q.sum2(ga, gp);
                    if (!colour) { NGv(l) += ga; adj3 = gp; }
                } else {
                    alpha_chain(l, da, db, ga, gp, adj3, NA3(l));
                }
            }
            NGv(0) += colour ? adj : adj3;
            if constexpr (kLanes == 3) NA3(0) += adj3;
        }
        return value;
    }

    // The same evaluation, rolled over the layers (one copy of each layer's
    // code, which keeps the FP64 kernels' instruction footprint small), with
    // the per-layer intermediates in the lane's slice. Same operations in the
    // same order as evaluate().
    __device__ __forceinline__ T evaluate_rolled(bool need_grad, bool active) {
        const Models<T>& m = models();
        T* sc = &Slice::value(Slice::kScratch);
        auto TRc = [sc](int l) -> T& { return sc[l * kSliceStride]; };
        // G = 4: the alphas of the trial point; G = 3: the slot holds the alpha
        // gradient (NA) and the pinned alphas are read from the filter targets.
        auto ALs = [sc](int l) -> T& { return sc[(L + l) * kSliceStride]; };
        const size_t npx = pixels(), pix = size_t(pixel);
        auto AL = [&](int l) -> T {
            if constexpr (kLanes == 3) return (opaque && l == 0) ? T(1) : T(a.targets[size_t(l) * npx + pix]);
            else return ALs(l);
        };
        auto AA = [sc](int l) -> T& { return sc[(2 * L + l) * kSliceStride]; };
        auto PC = [sc](int l) -> T& { return sc[(3 * L + l) * kSliceStride]; };
        auto NG = [sc](int l) -> T& { return sc[(4 * L + l) * kSliceStride]; };
        auto NA = [sc](int l) -> T& { return sc[(L + l) * kSliceStride]; };   // G = 3: alpha gradient
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            if constexpr (!BR) TRc(l) = TRv(l);   // (BR: the slot is the trial point)
            if constexpr (kLanes == 4) ALs(l) = alpha_at(TRc(l), l);
        }
        T dprev = AL(0), cprev = TRc(0);
        AA(0) = dprev;
        PC(0) = cprev;
#pragma unroll 1
        for (int l = 1; l < L; ++l) {
            const T av = AL(l), dd = dprev;
            const T Al = madd(T(m.Z[l]) * dd, T(1) - av, madd(T(m.X[l]) * av, dd, T(m.Y[l]) * av * (T(1) - dd)));
            const T s = TRc(l), c = cprev;
            const T pre = madd(T(m.Z[l]) * dd * (T(1) - av), c,
                               madd(blend_inline(m, l, s, c) * av, dd, T(m.Y[l]) * av * (T(1) - dd) * s));
            const T pcl = Al > T(1e-12) ? qdiv(pre, Al) : pre;
            AA(l) = Al;
            PC(l) = pcl;
            dprev = Al;
            cprev = pcl;
        }
        T energy = T(0), asum = T(0);
#pragma unroll 1
        for (int l = 0; l < L; ++l) {
            const T all = AL(l);
            const T mine = colour ? TRc(l) - mean_of(m, l) : T(0);
            const T d0 = Q.from(mine, 0), d1 = Q.from(mine, 1), d2 = Q.from(mine, 2);
            const T* P = m.prec[l];
            const T v0 = madd(P[2], d2, madd(P[0], d0, P[1] * d1));
            const T v1 = madd(P[5], d2, madd(P[3], d0, P[4] * d1));
            const T v2 = madd(P[8], d2, madd(P[6], d0, P[7] * d1));
            const T D = madd(d2, v2, madd(d0, v0, d1 * v1));
            energy = madd(all, D, energy);
            asum += all;
            if (need_grad) {
                if (colour) {
                    const T vq = sel3(Q.q, v0, v1, v2);
                    const T tq = madd(sel3(Q.q, P[6], P[7], P[8]), d2,
                                      madd(sel3(Q.q, P[0], P[1], P[2]), d0, sel3(Q.q, P[3], P[4], P[5]) * d1));
                    NG(l) = all * (vq + tq);
                } else {
                    NG(l) = D + (REFINE ? T(0) : T(0.01));
                }
                if constexpr (kLanes == 3) NA(l) = D;
            }
        }
        if (!REFINE) energy += T(0.01) * asum;
        const T value = residual_value(energy, dprev, cprev, need_grad, active);
        if (need_grad) {
            T adj = colour ? rho * res[0] - lam[0] : T(0);
            T adj3 = (!colour && !REFINE) ? rho * res[0] - lam[0] : T(0);
            if (REFINE && !colour)
#pragma unroll
                for (int l = 0; l < R; ++l) NG(l) += rho * res[l] - lam[l];
#pragma unroll 1
            for (int l = L - 1; l > 0; --l) {
                const T av = AL(l), dd = AA(l - 1), Al = AA(l);
                const T X = T(m.X[l]), Y = T(m.Y[l]), Z = T(m.Z[l]);
                const T da = madd(X, dd, Y * (T(1) - dd)) - Z * dd;
                const T db = madd(Z, T(1) - av, X * av - Y * av);
                const bool big = Al > T(1e-12);
                T ga, gp;
                if constexpr (kFast) {
                    const T s = TRc(l), c = PC(l - 1), out = PC(l), v = adj;
                    T fv, fs, fd;
                    blend3_inline(m, l, s, c, fv, fs, fd);
                    const T ds = madd(av * dd, fs, Y * av * (T(1) - dd));
                    const T dc = madd(av * dd, fd, Z * dd * (T(1) - av));
                    const T pa = madd(fv, dd, Y * (T(1) - dd) * s) - Z * dd * c;
                    const T pd = madd(Z * (T(1) - av), c, fv * av - Y * av * s);
                    const T r = big ? qdiv(T(1), Al) : T(1);
                    T gs, ad;
                    if (big) {
                        ga = v * (madd(-out, da, pa) * r);
                        gp = v * (madd(-out, db, pd) * r);
                        gs = v * (ds * r);
                        ad = v * (dc * r);
                    } else {
                        ga = v * pa; gp = v * pd; gs = v * ds; ad = v * dc;
                    }
                    if (colour) { NG(l) += gs; adj = ad; }
                    else { ga = adj3 * da; gp = adj3 * db; }
                } else if (colour) {
                    const T s = TRc(l), c = PC(l - 1), out = PC(l), v = adj;
                    T fv, fs, fd;
                    blend3_inline(m, l, s, c, fv, fs, fd);
                    const T ds = madd(av * dd, fs, Y * av * (T(1) - dd));
                    const T dc = madd(av * dd, fd, Z * dd * (T(1) - av));
                    const T pa = madd(fv, dd, Y * (T(1) - dd) * s) - Z * dd * c;
                    const T pd = madd(Z * (T(1) - av), c, fv * av - Y * av * s);
                    if (big) {
                        ga = v * ((pa - out * da) / Al);
                        gp = v * ((pd - out * db) / Al);
                        NG(l) += v * (ds / Al);
                        adj = v * (dc / Al);
                    } else {
                        ga = v * pa; gp = v * pd;
                        NG(l) += v * ds;
                        adj = v * dc;
                    }
                } else {
                    ga = adj3 * da;
                    gp = adj3 * db;
                }
                if constexpr (kLanes == 4) {
                    Q.sum2(ga, gp);
                    if (!colour) { NG(l) += ga; adj3 = gp; }
                } else {
                    alpha_chain(l, da, db, ga, gp, adj3, NA(l));
                }
            }
            NG(0) += colour ? adj : adj3;
            if constexpr (kLanes == 3) NA(0) += adj3;
            if constexpr (!BR) {
#pragma unroll
                for (int l = 0; l < L; ++l) NGv(l) = NG(l);
                if constexpr (kLanes == 3)
#pragma unroll
                    for (int l = 0; l < L; ++l) NA3(l) = NA(l);
            }
        }
        return value;
    }

    // ------------------------------------------------------ bookkeeping --
    __device__ __forceinline__ void steepest() {
#pragma unroll kU
        for (int l = 0; l < L; ++l) D(l) = fixed_at(l, G(l)) ? T(0) : -G(l);
    }

    // Layer l is free in this iteration's direction (BR: recomputed from x and
    // g, which do not change while the direction is formed).
    __device__ __forceinline__ bool is_free(const bool* freev, int l) const {
        if constexpr (BR) return !fixed_at(l, G(l)); else return freev[l];
    }

    // Two-loop recursion on the current free set; d holds q on entry/exit.
    // Register history: unrolled over the pairs. Shared history: one trip
    // per pair, the coefficients kept in the lane's slice (same arithmetic
    // in the same order).
    __device__ __forceinline__ void two_loop(const bool* freev) {
        if constexpr (HS != kHistRegisters) two_loop_rolled(freev);
        else two_loop_unrolled(freev);
    }

    __device__ __forceinline__ void two_loop_unrolled(const bool* freev) {
        T coeff[kHistory], inv[kHistory];
        T scaling = T(1);
        bool have_scaling = false;
#pragma unroll
        for (int j = 0; j < kHistory; ++j) {
            if (j < valid) {
                T dot = T(0), sy = T(0), ss = T(0), yy = T(0);
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) {
                        const T sa = hist.s(j, l), yb = hist.y(j, l);
                        dot = madd(sa, D(l), dot); sy = madd(sa, yb, sy); ss = madd(sa, sa, ss); yy = madd(yb, yb, yy);
                    }
                Q.sum4(dot, sy, ss, yy);
                const T r = qdiv(T(1), sy);
                inv[j] = (curvature_ok(sy, ss, yy) && finite_(r)) ? r : T(0);
                coeff[j] = dot * inv[j];
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) D(l) = madd(-coeff[j], hist.y(j, l), D(l));
                if (!have_scaling && inv[j] > T(0) && yy > T(0)) { scaling = qdiv(sy, yy); have_scaling = true; }
            }
        }
        scaling = fmax(T(1e-12), fmin(T(1e3), scaling));
#pragma unroll
        for (int l = 0; l < L; ++l) D(l) *= scaling;
#pragma unroll
        for (int j = kHistory - 1; j >= 0; --j) {
            if (j < valid) {
                T dot = T(0);
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) dot = madd(hist.y(j, l), D(l), dot);
                dot = Q.sum(dot);
                const T c = madd(-dot, inv[j], coeff[j]);
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) D(l) = madd(c, hist.s(j, l), D(l));
            }
        }
    }

    __device__ __forceinline__ void two_loop_rolled(const bool* freev) {
        T scaling = T(1);
        bool have_scaling = false;
        T* coeffs = &Slice::value(Slice::kCoeff);   // coefficient j at [2j], inverse at [2j+1] (times the stride)
        const int hs = hist.stride();               // element stride of the history
#pragma unroll 1
        for (int j = 0; j < valid; ++j) {
            const T* h = hist.row(j);
            T dot = T(0), sy = T(0), ss = T(0), yy = T(0);
#pragma unroll kUT
            for (int l = 0; l < L; ++l)
                if (is_free(freev, l)) {
                    const T sa = h[size_t(2 * l) * hs], yb = h[size_t(2 * l + 1) * hs];
                    dot = madd(sa, D(l), dot); sy = madd(sa, yb, sy); ss = madd(sa, sa, ss); yy = madd(yb, yb, yy);
                }
            Q.sum4(dot, sy, ss, yy);
            const T r = qdiv(T(1), sy);
            const T inv = (curvature_ok(sy, ss, yy) && finite_(r)) ? r : T(0);
            const T coeff = dot * inv;
#pragma unroll kUT
            for (int l = 0; l < L; ++l)
                if (is_free(freev, l)) D(l) = madd(-coeff, h[size_t(2 * l + 1) * hs], D(l));
            if (!have_scaling && inv > T(0) && yy > T(0)) { scaling = qdiv(sy, yy); have_scaling = true; }
            coeffs[2 * j * kSliceStride] = coeff;
            coeffs[(2 * j + 1) * kSliceStride] = inv;
        }
        scaling = fmax(T(1e-12), fmin(T(1e3), scaling));
#pragma unroll kUT
        for (int l = 0; l < L; ++l) D(l) *= scaling;
#pragma unroll 1
        for (int j = valid - 1; j >= 0; --j) {
            const T* h = hist.row(j);
            T dot = T(0);
#pragma unroll kUT
            for (int l = 0; l < L; ++l)
                if (is_free(freev, l)) dot = madd(h[size_t(2 * l + 1) * hs], D(l), dot);
            dot = Q.sum(dot);
            const T c = madd(-dot, coeffs[(2 * j + 1) * kSliceStride], coeffs[2 * j * kSliceStride]);
#pragma unroll kUT
            for (int l = 0; l < L; ++l)
                if (is_free(freev, l)) D(l) = madd(c, h[size_t(2 * l) * hs], D(l));
        }
    }

    // Starting point `start` (augmented_lagrangian.cuh:243-263).
    __device__ __forceinline__ int begin_start() {
        const Models<T>& m = models();
        const int s = start;
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            T v = init(l);
            if (!REFINE && s == 1) {
                if (!colour) v = l == 0 ? T(1) : T(0);
                else v = l == 0 ? fmin(T(1), fmax(T(0), target)) : mean_of(m, l);
            }
            if (REFINE && s && colour) v = mean_of(m, l);
            if (s == 2) {
                if (!colour) v = REFINE ? init(l) : T(0.5);
                else v = fmax(T(0.05), fmin(T(0.95), mean_of(m, l)));
            }
            X(l) = clampb(l, v);
        }
        if (s == 2) {
            // Move Dodge/Burn sources into the unsaturated branch.
            T av[L];
#pragma unroll
            for (int l = 0; l < L; ++l) av[l] = alpha_at(X(l), l);
            T dest = X(0), da = av[0];
#pragma unroll
            for (int l = 1; l < L; ++l) {
                const T al = av[l];
                const T Al = T(m.X[l]) * al * da + T(m.Y[l]) * al * (T(1) - da) + T(m.Z[l]) * da * (T(1) - al);
                if (colour) {
                    T sv = X(l);
                    if (dest >= T(0) && dest <= T(1) && m.mode[l] == 6) sv = fmin(sv, fmax(T(0), T(1) - dest - T(0.05)));
                    if (dest >= T(0) && dest <= T(1) && m.mode[l] == 7) sv = fmax(sv, fmin(T(1), T(1) - dest + T(0.05)));
                    sv = clampb(l, sv);
                    X(l) = sv;
                    const T pre = blend_value_call<T>(m.mode[l], sv, dest) * al * da + T(m.Y[l]) * al * (T(1) - da) * sv +
                                  T(m.Z[l]) * da * (T(1) - al) * dest;
                    dest = Al > T(1e-12) ? pre / Al : pre;
                }
                da = Al;
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) lam[r] = T(0);
        rho = T(100);
        outer = 0;
        frozen = 0;
        return aBeginOuter;
    }

    __device__ __forceinline__ int begin_outer() {
        count(4);
#pragma unroll kUC
        for (int l = 0; l < L; ++l) { ox(l) = X(l); TRv(l) = X(l); }
        phase = kOuterEval;
        best_moved = false;
        return aEval;
    }

    __device__ __forceinline__ T own_norm(const T* r) const {
        if (colour || !REFINE) return r[0] * r[0];
        T s = T(0);
#pragma unroll
        for (int l = 0; l < R; ++l) s += r[l] * r[l];
        return s;
    }

    // End of an outer step: multiplier and penalty update from the residual
    // at x, then the next outer step, the next start, or the pixel's result.
    __device__ __forceinline__ int end_outer() {
        const T norm = Q.sum(own_norm(resx));
        const bool feasible = norm < tol2;
#pragma unroll
        for (int r = 0; r < R; ++r) lam[r] = madd(-rho, resx[r], lam[r]);
        if (norm > T(0.0625) * oldnorm) rho *= T(10);
        T motion = T(0);
#pragma unroll kUC
        for (int l = 0; l < L; ++l) { const T dl = X(l) - ox(l); motion = madd(dl, dl, motion); }
        motion = Q.sum(motion);
        // A pixel whose last frozen_stop outer steps moved neither x nor the
        // best point stops here: past that point the method has not been
        // seen to change its result (its outputs equal the full run's on
        // every tested image); with frozen_stop = 0 it runs to the cap.
        frozen = (motion == T(0) && !best_moved) ? frozen + 1 : 0;
        if (ctl.frozen_stop > 0 && frozen >= ctl.frozen_stop) {
            if (start + 1 < ctl.starts) { ++start; return aBeginStart; }
            return aFinish;
        }
        if (!(motion < tol2 && feasible)) {
            if (outer + 1 < ctl.outer) {
                ++outer;
                if constexpr (MODE == kDefers)
                    if (outer == a.defer_outer && defer()) return aFetch;
                return aBeginOuter;
            }
            // A shortened FP32 solve (the FP64 re-solve behind it) hands an
            // unconverged pixel over whatever its best point: the re-solve
            // gives it the method's own result.
            if (ctl.cap_is_miss) { capped = true; return aFinish; }
        }
        if (start + 1 < ctl.starts) {
            ++start;
            return aBeginStart;
        }
        return aFinish;
    }

    // Next line-search trial point with non-zero motion (phase kTrial), the
    // steepest-descent retry, or the end of the inner solve when both
    // attempts are exhausted.
    __device__ __forceinline__ int next_trial() {
        if (bt < 32) {
            T sl = T(0), mo = T(0);
#pragma unroll kU
            for (int l = 0; l < L; ++l) {
                TRv(l) = clampb(l, madd(step, D(l), X(l)));
                const T delta = TRv(l) - X(l);
                sl = madd(G(l), delta, sl);
                mo = madd(delta, delta, mo);
            }
            Q.sum2(sl, mo);
            if (mo != T(0)) { slope = sl; phase = kTrial; return aEval; }
        }
        // This attempt failed: restart from steepest descent once.
        valid = 0; hist.reset(); steepest();
        if (attempt == 0) { attempt = 1; bt = 0; step = T(1); return aNextTrial; }
        return aEndOuter;
    }

    // Top of an inner iteration: projected gradient test, two-loop
    // direction, first trial.
    __device__ __forceinline__ int begin_iteration() {
        count(2);
        bool freev[BR ? 1 : L];
        T pg2 = T(0);
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            const bool fr = !fixed_at(l, G(l));
            if constexpr (!BR) freev[l] = fr;
            D(l) = fr ? G(l) : T(0);
            pg2 = madd(D(l), D(l), pg2);
        }
        pg2 = Q.sum(pg2);
        if (pg2 < T(1e-16) || !finite_(f)) return aEndOuter;
        two_loop(freev);
        T descent = T(0);
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            T v = -D(l);
            const T lv = lo(l), hv = hi(l);
            if (lv == hv || (X(l) <= lv && v < T(0)) || (X(l) >= hv && v > T(0))) v = T(0);
            D(l) = v;
            descent = madd(v, G(l), descent);
        }
        descent = Q.sum(descent);
        if (!(descent < T(0))) { valid = 0; hist.reset(); steepest(); }
        attempt = 0; bt = 0; step = T(1);
        return aNextTrial;
    }

    // Accepted step (value `cand`, gradient ng): curvature pair, move, inner
    // termination test.
    __device__ __forceinline__ int accept() {
        T sy = T(0), ss = T(0), yy = T(0), mm = T(0);
        T sv[BR ? 1 : L], yv[BR ? 1 : L];
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            const T svl = TRv(l) - X(l), yvl = NGv(l) - G(l);
            if constexpr (!BR) { sv[l] = svl; yv[l] = yvl; }
            sy = madd(svl, yvl, sy); ss = madd(svl, svl, ss); yy = madd(yvl, yvl, yy);
            if constexpr (kFast || !Slice::kRolledEval) mm = fmax(mm, qdiv(fabs(svl), T(1) + fabs(X(l))));
        }
        if constexpr (!kFast && Slice::kRolledEval) {
            // One copy of the FP64 division: the step from the accepted point
            // (the last point evaluated, kept in the scratch slice) per layer.
#pragma unroll 1
            for (int l = 0; l < L; ++l) {
                const T x = X(l), s = Slice::value(Slice::kScratch + l) - x;
                mm = fmax(mm, qdiv(fabs(s), T(1) + fabs(x)));
            }
        }
        Q.sum3(sy, ss, yy);
        if constexpr (kLanes == 3) {
            // The pinned alphas do not move, but their gradient change counts
            // in y.y (the same on every lane).
            T ya = T(0);
#pragma unroll kU
            for (int l = 0; l < L; ++l) { const T dy = NA3(l) - GA3(l); ya = madd(dy, dy, ya); }
            yy += ya;
        }
        mm = Q.max(mm);
        const T r = qdiv(T(1), sy);
        if (curvature_ok(sy, ss, yy) && finite_(r)) {
            if constexpr (BR) {
                // The pair again, element by element (the same differences).
#pragma unroll 1
                for (int l = 0; l < L; ++l) hist.push_elem(l, TRv(l) - X(l), NGv(l) - G(l));
                hist.advance();
            } else {
                hist.push(sv, yv);
            }
            valid = valid + 1 < kHistory ? valid + 1 : kHistory;
        }
        const T delta = fabs(f - cand), size = T(0.5) * (fabs(f) + fabs(cand));
#pragma unroll kU
        for (int l = 0; l < L; ++l) { X(l) = TRv(l); G(l) = NGv(l); }
        if constexpr (kLanes == 3)
#pragma unroll kU
            for (int l = 0; l < L; ++l) GA3(l) = NA3(l);
#pragma unroll
        for (int q = 0; q < R; ++q) resx[q] = res[q];
        f = cand;
        if (delta < itol * size || mm < itol) return aEndOuter;
        if (++it >= ctl.inner) return aEndOuter;
        return aBeginIter;
    }

    // Decision after an evaluation, by phase.
    __device__ __forceinline__ int after_evaluation(T value, bool need_grad) {
        if (phase == kOuterEval) {
            f = value;
#pragma unroll kU
            for (int l = 0; l < L; ++l) G(l) = NGv(l);
            if constexpr (kLanes == 3)
#pragma unroll kU
                for (int l = 0; l < L; ++l) GA3(l) = NA3(l);
#pragma unroll
            for (int q = 0; q < R; ++q) resx[q] = res[q];
            oldnorm = Q.sum(own_norm(res));
            valid = 0; hist.reset(); it = 0;
            return aBeginIter;
        }
        if (phase == kTrial) {
            count(3);
            if (slope < T(0) && finite_(value) && value <= f + T(1e-4) * slope) {
                if (need_grad) { cand = value; return aAccept; }
                phase = kAcceptGrad;
                return aEval;
            }
            step *= T(0.5);
            ++bt;
            return aNextTrial;
        }
        cand = value;   // kAcceptGrad
        return aAccept;
    }

    // ------------------------------------------------------- deferral --
    // The state a pixel needs to begin an outer step (SolveArgs::defer_*):
    // x, the best point, the start-0 seed, the multipliers, rho, the best
    // point's norm and energy, and the outer-step, frozen-step and start
    // counters. Everything else is set again by the outer step's first
    // evaluation. Word w of this lane in slot k: [w * capacity * 4 + k * 4 + q].
    __device__ bool defer() {
        static_assert(3 * L + R + 7 <= defer_words(L), "the deferred state fits its slot");
        int slot = 0;
        if (Q.q == 0) slot = int(atomicAdd(a.defer_count, 1));
        slot = Q.from(slot, 0);
        if (slot >= a.defer_capacity) return false;
        if (Q.q == 0) a.defer_list[slot] = int32_t(gidx);
        T* st = static_cast<T*>(a.defer_state) + size_t(slot) * 4 + Q.q;
        const size_t w = size_t(a.defer_capacity) * 4;
        int k = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) st[size_t(k++) * w] = X(l);
#pragma unroll
        for (int l = 0; l < L; ++l) st[size_t(k++) * w] = best(l);
#pragma unroll
        for (int l = 0; l < L; ++l) st[size_t(k++) * w] = init(l);
#pragma unroll
        for (int r = 0; r < R; ++r) st[size_t(k++) * w] = lam[r];
        st[size_t(k++) * w] = rho;
        st[size_t(k++) * w] = best_norm;
        st[size_t(k++) * w] = best_energy;
        st[size_t(k++) * w] = T(outer);
        st[size_t(k++) * w] = T(frozen);
        st[size_t(k++) * w] = T(start);
        st[size_t(k++) * w] = have_best ? T(1) : T(0);
        return true;
    }

    __device__ void restore(int slot) {
        const T* st = static_cast<const T*>(a.defer_state) + size_t(slot) * 4 + Q.q;
        const size_t w = size_t(a.defer_capacity) * 4;
        int k = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) X(l) = st[size_t(k++) * w];
#pragma unroll
        for (int l = 0; l < L; ++l) best(l) = st[size_t(k++) * w];
#pragma unroll
        for (int l = 0; l < L; ++l) init(l) = st[size_t(k++) * w];
#pragma unroll
        for (int r = 0; r < R; ++r) lam[r] = st[size_t(k++) * w];
        rho = st[size_t(k++) * w];
        best_norm = st[size_t(k++) * w];
        best_energy = st[size_t(k++) * w];
        outer = int(st[size_t(k++) * w]);
        frozen = int(st[size_t(k++) * w]);
        start = int(st[size_t(k++) * w]);
        have_best = st[size_t(k++) * w] != T(0);
        capped = false;
    }

    // ------------------------------------------------------------ pixels --
    // Loads pixel `i`: targets, bounds and the start-0 seed.
    __device__ __forceinline__ void load(int i) {
        const Models<T>& m = models();
        const size_t n = pixels();
        pixel = i;
        target = T(colour ? image()[3 * size_t(i) + Q.q] : 0.0);
        bgq = T((REFINE && smooth && colour) ? a.targets[(size_t(L) + Q.q) * n + i] : 0.0);
#pragma unroll
        for (int l = 0; l < RA; ++l) {
            double t = REFINE ? a.targets[size_t(l) * n + i] : 0.0;
            if (REFINE && opaque && l == 0) t = 1.0;
            ahat[l] = T(t);
        }
        const float* wp = REFINE ? nullptr : warm();
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            T v;
            if (kLanes == 3 || colour) {
                if (REFINE) v = (smooth && l == 0) ? bgq : T(a.first[(size_t(l) * n + i) * 4 + Q.q]);
                else v = fmin(T(1), fmax(T(0), mean_of(m, l)));
            } else {
                v = (opaque && l == 0) ? T(1) : (REFINE ? ahat[REFINE ? l : 0] : T(0.5));
            }
            if (!REFINE && wp) {
                // Learned warm start: the network's prediction replaces the
                // start-0 seed (bounds still apply when the start is seeded).
                const float* wv = wp + size_t(i) * size_t(4 * L);
                v = T(colour ? wv[L + 3 * l + Q.q] : wv[l]);
            }
            init(l) = v;
        }
        have_best = false;
        capped = false;
        best_norm = T(INFINITY); best_energy = T(INFINITY);
        if (a.counters && Q.q == 0 && MODE != kResumes)
#pragma unroll
            for (int k = 0; k < 5; ++k) counter(k) = 0;
    }

    // Writes the finished pixel: output (pinned values exactly), FP64
    // feasibility check, status, miss list, counters.
    __device__ void store(bool skipped) {
        const Models<T>& m = models();
        const size_t n = pixels(), i = size_t(pixel);
        double* outp = output();
        double v0 = 0.0;
#pragma unroll kU
        for (int l = 0; l < L; ++l) {
            double v = double(have_best ? best(l) : init(l));
            if (REFINE && !colour) v = (opaque && l == 0) ? 1.0 : a.targets[size_t(l) * n + i];
            if (REFINE && smooth && colour && l == 0) v = a.targets[(size_t(L) + Q.q) * n + i];
            if (!REFINE && opaque && !colour && l == 0) v = 1.0;
            outp[(size_t(l) * n + i) * 4 + Q.q] = v;
            if (kLanes == 3 && Q.q == 0)   // the pinned alpha (no alpha lane)
                outp[(size_t(l) * n + i) * 4 + 3] = (opaque && l == 0) ? 1.0 : a.targets[size_t(l) * n + i];
            if (l == 0) v0 = v;
        }
        // FP64 constraint check of the written point (solver_workspace.cuh:18-38),
        // one layer per trip, reading back the values just written.
        double A = kLanes == 3 ? (opaque ? 1.0 : a.targets[i]) : Q.from(v0, 3), c = v0;
#pragma unroll 1
        for (int l = 1; l < L; ++l) {
            const double s = outp[(size_t(l) * n + i) * 4 + Q.q];
            const double al = kLanes == 3 ? a.targets[size_t(l) * n + i] : Q.from(s, 3), dd = A;
            const double Al = double(m.X[l]) * al * dd + double(m.Y[l]) * al * (1.0 - dd) +
                              double(m.Z[l]) * dd * (1.0 - al);
            const double pre = blend_value_call<double>(m.mode[l], s, c) * al * dd + double(m.Y[l]) * al * (1.0 - dd) * s +
                               double(m.Z[l]) * dd * (1.0 - al) * c;
            c = Al > 1e-12 ? pre / Al : pre;
            A = Al;
        }
        double norm = 0.0;
        if (colour) {
            const double r = c - image()[3 * i + Q.q];
            norm = r * r;
        } else if (REFINE) {
#pragma unroll 1
            for (int l = 0; l < R; ++l) {
                const double t = (opaque && l == 0) ? 1.0 : a.targets[size_t(l) * n + i];
                const double r = outp[(size_t(l) * n + i) * 4 + 3] - t;
                norm += r * r;
            }
        } else {
            const double r = A - 1.0;
            norm = r * r;
        }
        norm = Q.sum(norm);
        const bool miss = capped || !(norm < ctl.outer_tolerance * ctl.outer_tolerance);
        if (Q.q == 0) {
            int32_t* stp = status();
            if (skipped) {
                if (stp) stp[i] = 8;
                if (a.input_failed) atomicAdd(a.input_failed, 1);
            } else {
                if (stp) stp[i] = miss ? 3 : 0;
                if (miss && a.miss_list) a.miss_list[atomicAdd(a.miss_count, 1)] = int32_t(gidx);
            }
        }
    }

    // Pulls the next pixel: aBeginStart when it needs solving, aFetch again
    // after a pixel that is written without solving, aEval with `live`
    // cleared when the queue is empty.
    __device__ int fetch(int total, bool& live) {
        int job = 0;
        if (Q.q == 0) job = int(atomicAdd(a.queue, 1u));
        job = Q.from(job, 0);
        if (job >= total) { phase = kIdle; live = false; return aEval; }
        gidx = a.list ? a.list[job] : (a.order ? a.order[job] : a.first_pixel + job);
        int i = gidx;
        if constexpr (BATCH) {
            // The image owning queue index gidx: last job with offset <= gidx.
            int lo = 0, hi = a.job_count - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (a.jobs[mid].offset <= int64_t(gidx)) lo = mid; else hi = mid - 1;
            }
            if (lo != job_id) {
                batch_models_ = static_cast<const Models<T>*>(a.models) + a.jobs[lo].model;
                job_id = lo;
            }
            i = gidx - int(a.jobs[lo].offset);
        }
        load(i);
        if (REFINE && a.input_status && a.input_status[i] != 0) {
            // Targets that cannot be normalized: keep the initial layers and
            // report status 8 (solver_workspace.cuh:144).
            store(true);
            return aFetch;
        }
        if constexpr (MODE == kResumes) {
            // A pixel deferred by an earlier launch: its state at the start of
            // the outer step it left at, from slot `job` of the list.
            restore(job);
            return aBeginOuter;
        }
        start = 0;
        return aBeginStart;
    }

    // ------------------------------------------------------------- loop --
    __device__ void run() {
        const int total = a.list ? min(*a.list_count, a.list_limit) : (a.pixel_count >= 0 ? a.pixel_count : a.n);
        bool live = !Q.extra;            // lanes of no group stay idle throughout
        int act = live ? aFetch : aEval;
        const int gq = ctl.gradient_quorum, bq = ctl.direction_quorum;
        for (;;) {
            // Pixels of the warp that reach a new quasi-Newton direction
            // (begin_iteration, the two-loop recursion) run it together: while
            // fewer than direction_quorum/8 of the live pixels are there (and
            // some are ready to evaluate), they wait one evaluation. A waiting
            // pixel's evaluate() is inactive at its accepted point, which
            // recomputes the residuals of that point unchanged.
            bool allow_bi = bq == 0;
            for (;;) {
                // The actions in the order the method chains them, each at
                // most once per pass: pixels that reach an action from
                // different points of their chains (a line-search step, or an
                // accept followed by a new direction) run it together. A
                // pixel's own sequence of actions is unchanged.
                while (act != aEval && (allow_bi || act != aBeginIter)) {
                    if (act == aAccept) act = accept();
                    if (act == aBeginIter && allow_bi) act = begin_iteration();
                    if (act == aNextTrial) act = next_trial();
                    if (act == aEndOuter) act = end_outer();
                    if (act == aFinish) { store(false); act = aFetch; }
                    if (act == aFetch) act = fetch(total, live);
                    if (act == aBeginStart) act = begin_start();
                    if (act == aBeginOuter) act = begin_outer();
                }
                if (allow_bi) break;
                const int nb = __popc(__ballot_sync(0xffffffffu, act == aBeginIter));
                if (nb == 0) break;
                const int nl = __popc(__ballot_sync(0xffffffffu, live));
                if (nb < nl && 8 * nb < bq * nl) break;
                allow_bi = true;
            }
            if (__all_sync(0xffffffffu, !live)) break;
            const bool ready = live && act == aEval;
            const bool need_grad = ready && (phase == kOuterEval || phase == kAcceptGrad ||
                                             (phase == kTrial && bt == 0 && ctl.gradient_on_first_trial));
            // The warp runs the gradient part of an evaluation if any of its
            // pixels needs it, with the others masked off. While fewer than
            // gradient_quorum/8 of the pixels ready to evaluate need a
            // gradient (and some need a value alone), those pixels wait: this
            // evaluation is value-only, and they evaluate with the next
            // quorum. A waiting pixel's evaluate() is inactive and recomputes
            // the residuals of its unchanged trial point, which its own
            // evaluation then recomputes identically, so its results do not
            // change.
            bool go = ready;
            if (gq > 0) {
                const int ng = __popc(__ballot_sync(0xffffffffu, need_grad));
                const int nr = __popc(__ballot_sync(0xffffffffu, ready));
                if (ng < nr && 8 * ng < gq * nr) go = ready && !need_grad;
            }
            const T value = Q.extra ? T(0) : evaluate(need_grad && go, go);
            if (go) act = after_evaluation(value, need_grad);
        }
        if (a.tally) {
            // One atomic per warp and count.
            const uint32_t v = __reduce_add_sync(0xffffffffu, n_value), g = __reduce_add_sync(0xffffffffu, n_grad);
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(a.tally + 0, (unsigned long long)v);
                atomicAdd(a.tally + 1, (unsigned long long)g);
            }
        }
    }
};

}  // namespace unb
