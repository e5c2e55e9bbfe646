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
// values of every vector: with L a template parameter all of it stays in
// registers (the FP64 build keeps its history in shared memory instead). The
// composite is separable per channel given the alphas, which lane 3
// broadcasts; the 3x3 colour prior needs the three deltas of a layer (two
// shuffles); the adjoint sweep reduces the alpha sensitivities of the three
// channels once per layer. Every branch is taken on quad-uniform values, so a
// quad never splits. A persistent grid pulls pixels from an atomic queue,
// one quad at a time, so slow pixels do not hold up a warp's other quads.
#pragma once
#include "blend.cuh"
#include "common.cuh"

namespace unb {

template <class T> __device__ __forceinline__ T sel3(int q, T a, T b, T c) { return q == 0 ? a : (q == 1 ? b : c); }

template <class T> __device__ __forceinline__ bool finite_(T v);
template <> __device__ __forceinline__ bool finite_<float>(float v) { return isfinite(v); }
template <> __device__ __forceinline__ bool finite_<double>(double v) { return isfinite(v); }

struct Quad {
    unsigned mask;
    int base, q;
    __device__ __forceinline__ Quad() {
        const int lane = threadIdx.x & 31;
        base = lane & ~3;
        q = lane & 3;
        mask = 0xFu << base;
    }
    template <class T> __device__ __forceinline__ T sum(T v) const {
        v += __shfl_xor_sync(mask, v, 1);
        v += __shfl_xor_sync(mask, v, 2);
        return v;
    }
    template <class T> __device__ __forceinline__ void sum2(T& a, T& b) const {
        a += __shfl_xor_sync(mask, a, 1); b += __shfl_xor_sync(mask, b, 1);
        a += __shfl_xor_sync(mask, a, 2); b += __shfl_xor_sync(mask, b, 2);
    }
    template <class T> __device__ __forceinline__ void sum3(T& a, T& b, T& c) const {
        a += __shfl_xor_sync(mask, a, 1); b += __shfl_xor_sync(mask, b, 1); c += __shfl_xor_sync(mask, c, 1);
        a += __shfl_xor_sync(mask, a, 2); b += __shfl_xor_sync(mask, b, 2); c += __shfl_xor_sync(mask, c, 2);
    }
    template <class T> __device__ __forceinline__ void sum4(T& a, T& b, T& c, T& d) const {
        a += __shfl_xor_sync(mask, a, 1); b += __shfl_xor_sync(mask, b, 1);
        c += __shfl_xor_sync(mask, c, 1); d += __shfl_xor_sync(mask, d, 1);
        a += __shfl_xor_sync(mask, a, 2); b += __shfl_xor_sync(mask, b, 2);
        c += __shfl_xor_sync(mask, c, 2); d += __shfl_xor_sync(mask, d, 2);
    }
    template <class T> __device__ __forceinline__ T max(T v) const {
        v = fmax(v, __shfl_xor_sync(mask, v, 1));
        v = fmax(v, __shfl_xor_sync(mask, v, 2));
        return v;
    }
    template <class T> __device__ __forceinline__ T from(T v, int src) const {
        return __shfl_sync(mask, v, base | src);
    }
};

// L-BFGS pairs, indexed by age j (0 = newest). Register form: a shift
// register with compile-time indices. Shared-memory form: a ring buffer.
template <class T, int L, bool SMEM> struct History;

template <class T, int L> struct History<T, L, false> {
    T s_[kHistory][L], y_[kHistory][L];
    __device__ __forceinline__ void init(T*) {}
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

template <class T, int L> struct History<T, L, true> {
    T* base;   // this lane's slice: element (slot, l, s|y) at base[((slot*L + l)*2 + w) * blockDim.x]
    int next;
    __device__ __forceinline__ void init(T* smem) { base = smem + threadIdx.x; next = 0; }
    __device__ __forceinline__ int slot(int j) const { int k = next - 1 - j; return k < 0 ? k + kHistory : k; }
    __device__ __forceinline__ T s(int j, int l) const { return base[size_t((slot(j) * L + l) * 2) * blockDim.x]; }
    __device__ __forceinline__ T y(int j, int l) const { return base[size_t((slot(j) * L + l) * 2 + 1) * blockDim.x]; }
    __device__ __forceinline__ void push(const T* sv, const T* yv) {
#pragma unroll
        for (int l = 0; l < L; ++l) {
            base[size_t((next * L + l) * 2) * blockDim.x] = sv[l];
            base[size_t((next * L + l) * 2 + 1) * blockDim.x] = yv[l];
        }
        next = next + 1 == kHistory ? 0 : next + 1;
    }
    __device__ __forceinline__ void reset() { next = 0; }
};

template <class T, int L, bool REFINE, bool HSMEM> struct QuadSolver {
    const Models<T>& m;
    const SolverControls& ctl;
    Quad Q;
    bool opaque, smooth;
    T tol2;

    // Per-pixel inputs (per lane).
    T target;            // colour lanes: target channel q
    T ahat[L];           // lane 3, refinement: filtered alpha targets
    T lo[L], hi[L];      // variable bounds of this lane's slice
    T init[L];           // start-0 seed before clamping

    // Method state (per lane slice).
    T x[L], g[L], d[L], tr[L], ng[L], ox[L], best[L];
    T lam[REFINE ? L : 1];   // colour lanes use lam[0]; lane 3 one (unmixing) or L (refinement) rows
    T res[REFINE ? L : 1];   // residual rows owned by this lane, from the last evaluation
    History<T, L, HSMEM> hist;
    T best_norm, best_energy;
    bool have_best;
    uint32_t n_values, n_gradients, n_iterations, n_backtracks, n_outer;

    __device__ QuadSolver(const Models<T>& models, const SolverControls& c) : m(models), ctl(c) {}

    // ---------------------------------------------------------- evaluate --
    // AL value E + sum(rho/2 C^2 - lambda C), uniform across the quad. Sets
    // res[], returns energy E and |C|^2 (uniform) and, if DERIV, the gradient
    // slice `gr`. Tracks the best feasible point.
    template <bool DERIV> __device__ __forceinline__ T evaluate(const T* pt, T rho, T* gr) {
        ++n_values;
        if (DERIV) ++n_gradients;
        const bool colour = Q.q < 3;
        T a[L], A[L], pc[L];
#pragma unroll
        for (int l = 0; l < L; ++l) a[l] = Q.from(pt[l], 3);
        // Forward composite, bottom to top. pc[l] = this channel after layer l.
        A[0] = a[0];
        pc[0] = pt[0];
#pragma unroll
        for (int l = 1; l < L; ++l) {
            const T al = a[l], dd = A[l - 1];
            const T Al = T(m.X[l]) * al * dd + T(m.Y[l]) * al * (T(1) - dd) + T(m.Z[l]) * dd * (T(1) - al);
            A[l] = Al;
            const T s = pt[l], c = pc[l - 1];
            const T pre = blend_value<T>(m.mode[l], s, c) * al * dd + T(m.Y[l]) * al * (T(1) - dd) * s +
                          T(m.Z[l]) * dd * (T(1) - al) * c;
            pc[l] = Al > T(1e-12) ? pre / Al : pre;
        }
        // Colour prior: every lane gathers the three deltas of each layer.
        T energy = T(0), asum = T(0), D[L];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const T mine = colour ? pt[l] - sel3(Q.q, m.mean[l][0], m.mean[l][1], m.mean[l][2]) : T(0);
            const T d0 = Q.from(mine, 0), d1 = Q.from(mine, 1), d2 = Q.from(mine, 2);
            const T* P = m.prec[l];
            const T v0 = P[0] * d0 + P[1] * d1 + P[2] * d2;
            const T v1 = P[3] * d0 + P[4] * d1 + P[5] * d2;
            const T v2 = P[6] * d0 + P[7] * d1 + P[8] * d2;
            D[l] = d0 * v0 + d1 * v1 + d2 * v2;
            energy += a[l] * D[l];
            asum += a[l];
            if (DERIV) {
                if (colour) {
                    // (P + P^T) delta, row q.
                    const T vq = Q.q == 0 ? v0 : (Q.q == 1 ? v1 : v2);
                    const T tq = sel3(Q.q, P[0], P[1], P[2]) * d0 + sel3(Q.q, P[3], P[4], P[5]) * d1 +
                                 sel3(Q.q, P[6], P[7], P[8]) * d2;
                    gr[l] = a[l] * (vq + tq);
                } else {
                    gr[l] = D[l];
                }
            }
        }
        if (!REFINE) {
            energy += T(0.01) * asum;
            if (DERIV && !colour)
#pragma unroll
                for (int l = 0; l < L; ++l) gr[l] += T(0.01);
        }
        // Residual rows and AL terms owned by this lane.
        T terms = T(0), norm = T(0);
        if (colour) {
            res[0] = pc[L - 1] - target;
            terms = T(0.5) * rho * res[0] * res[0] - lam[0] * res[0];
            norm = res[0] * res[0];
        } else if (REFINE) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                res[l] = pt[l] - ahat[l];
                terms += T(0.5) * rho * res[l] * res[l] - lam[l] * res[l];
                norm += res[l] * res[l];
            }
        } else {
            res[0] = A[L - 1] - T(1);
            terms = T(0.5) * rho * res[0] * res[0] - lam[0] * res[0];
            norm = res[0] * res[0];
        }
        Q.sum2(terms, norm);
        const T value = energy + terms;
        // Best-feasible tracking (augmented_lagrangian.cuh:237-240).
        const bool feasible = norm < tol2;
        if (finite_(energy) && finite_(norm) &&
            (!have_best || (feasible && (best_norm >= tol2 || energy < best_energy)) ||
             (!feasible && best_norm >= tol2 && norm < best_norm))) {
            have_best = true; best_norm = norm; best_energy = energy;
#pragma unroll
            for (int l = 0; l < L; ++l) best[l] = pt[l];
        }
        if (!DERIV) return value;

        // Reverse sweep. adj: this channel's cotangent; adj3: the alpha chain's.
        T adj = colour ? rho * res[0] - lam[0] : T(0);
        T adj3 = (!colour && !REFINE) ? rho * res[0] - lam[0] : T(0);
        if (REFINE && !colour)
#pragma unroll
            for (int l = 0; l < L; ++l) gr[l] += rho * res[l] - lam[l];
#pragma unroll
        for (int l = L - 1; l > 0; --l) {
            const T al = a[l], dd = A[l - 1], Al = A[l];
            const T X = T(m.X[l]), Y = T(m.Y[l]), Z = T(m.Z[l]);
            const T da = X * dd + Y * (T(1) - dd) - Z * dd;
            const T db = X * al - Y * al + Z * (T(1) - al);
            const bool big = Al > T(1e-12);
            T ga, gp;
            if (colour) {
                const T s = pt[l], c = pc[l - 1], out = pc[l], v = adj;
                T f, fs, fd;
                blend_all<T>(m.mode[l], s, c, f, fs, fd);
                const T ds = al * dd * fs + Y * al * (T(1) - dd);
                const T dc = al * dd * fd + Z * dd * (T(1) - al);
                const T pa = f * dd + Y * (T(1) - dd) * s - Z * dd * c;
                const T pd = f * al - Y * al * s + Z * (T(1) - al) * c;
                if (big) {
                    const T inv = T(1) / Al;
                    ga = v * ((pa - out * da) * inv);
                    gp = v * ((pd - out * db) * inv);
                    if (DERIV) gr[l] += v * (ds * inv);
                    adj = v * (dc * inv);
                } else {
                    ga = v * pa; gp = v * pd;
                    gr[l] += v * ds;
                    adj = v * dc;
                }
            } else {
                ga = adj3 * da;
                gp = adj3 * db;
            }
            Q.sum2(ga, gp);
            if (!colour) { gr[l] += ga; adj3 = gp; }
        }
        gr[0] += colour ? adj : adj3;
        return value;
    }

    // ------------------------------------------------------------ helpers --
    __device__ __forceinline__ bool fixed_at(int l, T gl) const {
        return lo[l] == hi[l] || (x[l] <= lo[l] && gl > T(0)) || (x[l] >= hi[l] && gl < T(0));
    }
    __device__ __forceinline__ void steepest() {
#pragma unroll
        for (int l = 0; l < L; ++l) d[l] = fixed_at(l, g[l]) ? T(0) : -g[l];
    }

    // Two-loop recursion on the current free set; d holds q on entry/exit.
    __device__ __forceinline__ void two_loop(int valid, const bool* freev) {
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
                        const T a = hist.s(j, l), b = hist.y(j, l);
                        dot += a * d[l]; sy += a * b; ss += a * a; yy += b * b;
                    }
                Q.sum4(dot, sy, ss, yy);
                const T r = T(1) / sy;
                inv[j] = (sy > T(1e-9) * dsqrt(ss * yy) && sy > T(0) && finite_(r)) ? r : T(0);
                coeff[j] = dot * inv[j];
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) d[l] -= coeff[j] * hist.y(j, l);
                if (!have_scaling && inv[j] > T(0) && yy > T(0)) { scaling = sy / yy; have_scaling = true; }
            }
        }
        scaling = fmax(T(1e-12), fmin(T(1e3), scaling));
#pragma unroll
        for (int l = 0; l < L; ++l) d[l] *= scaling;
#pragma unroll
        for (int j = kHistory - 1; j >= 0; --j) {
            if (j < valid) {
                T dot = T(0);
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) dot += hist.y(j, l) * d[l];
                dot = Q.sum(dot);
                const T a = coeff[j] - dot * inv[j];
#pragma unroll
                for (int l = 0; l < L; ++l)
                    if (freev[l]) d[l] += a * hist.s(j, l);
            }
        }
    }

    __device__ __forceinline__ T mean_of(int l) const {
        return Q.q < 3 ? sel3(Q.q, m.mean[l][0], m.mean[l][1], m.mean[l][2]) : T(0);
    }
    __device__ __forceinline__ T clampb(int l, T v) const { return v < lo[l] ? lo[l] : (v > hi[l] ? hi[l] : v); }

    // Starting point `start` (augmented_lagrangian.cuh:243-263).
    __device__ __forceinline__ void seed(int start) {
        const bool colour = Q.q < 3;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            T v = init[l];
            if (!REFINE && start == 1) {
                if (!colour) v = l == 0 ? T(1) : T(0);
                else v = l == 0 ? fmin(T(1), fmax(T(0), target)) : mean_of(l);
            }
            if (REFINE && start && colour) v = mean_of(l);
            if (start == 2) {
                if (!colour) v = REFINE ? init[l] : T(0.5);
                else v = fmax(T(0.05), fmin(T(0.95), mean_of(l)));
            }
            x[l] = v < lo[l] ? lo[l] : (v > hi[l] ? hi[l] : v);
        }
        if (start == 2) {
            // Move Dodge/Burn sources into the unsaturated branch.
            T a[L];
#pragma unroll
            for (int l = 0; l < L; ++l) a[l] = Q.from(x[l], 3);
            T dest = x[0], da = a[0];
#pragma unroll
            for (int l = 1; l < L; ++l) {
                const T al = a[l];
                const T Al = T(m.X[l]) * al * da + T(m.Y[l]) * al * (T(1) - da) + T(m.Z[l]) * da * (T(1) - al);
                if (colour) {
                    T s = x[l];
                    if (dest >= T(0) && dest <= T(1) && m.mode[l] == 6) s = fmin(s, fmax(T(0), T(1) - dest - T(0.05)));
                    if (dest >= T(0) && dest <= T(1) && m.mode[l] == 7) s = fmax(s, fmin(T(1), T(1) - dest + T(0.05)));
                    s = clampb(l, s);
                    x[l] = s;
                    const T pre = blend_value<T>(m.mode[l], s, dest) * al * da + T(m.Y[l]) * al * (T(1) - da) * s +
                                  T(m.Z[l]) * da * (T(1) - al) * dest;
                    dest = Al > T(1e-12) ? pre / Al : pre;
                }
                da = Al;
            }
        }
    }

    // --------------------------------------------------------------- solve --
    __device__ void run() {
        have_best = false;
        best_norm = T(INFINITY); best_energy = T(INFINITY);
        n_values = n_gradients = n_iterations = n_backtracks = n_outer = 0;
        const T itol = T(ctl.inner_tolerance);
        for (int start = 0; start < ctl.starts; ++start) {
            seed(start);
#pragma unroll
            for (int r = 0; r < (REFINE ? L : 1); ++r) lam[r] = T(0);
            T rho = T(100);
            for (int outer = 0; outer < ctl.outer; ++outer) {
                ++n_outer;
#pragma unroll
                for (int l = 0; l < L; ++l) ox[l] = x[l];
                T f = evaluate<true>(x, rho, g);
                T oldnorm = Q.sum(own_norm());
                int valid = 0;
                hist.reset();
                for (int it = 0; it < ctl.inner; ++it) {
                    ++n_iterations;
                    bool freev[L];
                    T pg2 = T(0);
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        freev[l] = !fixed_at(l, g[l]);
                        d[l] = freev[l] ? g[l] : T(0);
                        pg2 += d[l] * d[l];
                    }
                    pg2 = Q.sum(pg2);
                    if (pg2 < T(1e-16) || !finite_(f)) break;
                    two_loop(valid, freev);
                    T descent = T(0);
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        T v = -d[l];
                        if (lo[l] == hi[l] || (x[l] <= lo[l] && v < T(0)) || (x[l] >= hi[l] && v > T(0))) v = T(0);
                        d[l] = v;
                        descent += v * g[l];
                    }
                    descent = Q.sum(descent);
                    if (!(descent < T(0))) { valid = 0; hist.reset(); steepest(); }
                    bool accepted = false, have_grad = false;
                    T cand = f;
                    for (int attempt = 0; attempt < 2 && !accepted; ++attempt) {
                        T step = T(1);
                        for (int bt = 0; bt < 32; ++bt) {
                            T slope = T(0), motion = T(0);
#pragma unroll
                            for (int l = 0; l < L; ++l) {
                                tr[l] = clampb(l, x[l] + step * d[l]);
                                const T delta = tr[l] - x[l];
                                slope += g[l] * delta;
                                motion += delta * delta;
                            }
                            Q.sum2(slope, motion);
                            if (motion == T(0)) break;
                            ++n_backtracks;
                            if (bt == 0 && ctl.gradient_on_first_trial) { cand = evaluate<true>(tr, rho, ng); have_grad = true; }
                            else { cand = evaluate<false>(tr, rho, ng); have_grad = false; }
                            if (slope < T(0) && finite_(cand) && cand <= f + T(1e-4) * slope) { accepted = true; break; }
                            step *= T(0.5);
                        }
                        if (!accepted) { valid = 0; hist.reset(); steepest(); }
                    }
                    if (!accepted) break;
                    if (!have_grad) cand = evaluate<true>(tr, rho, ng);
                    T sy = T(0), ss = T(0), yy = T(0), mm = T(0);
                    T sv[L], yv[L];
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        sv[l] = tr[l] - x[l];
                        yv[l] = ng[l] - g[l];
                        sy += sv[l] * yv[l]; ss += sv[l] * sv[l]; yy += yv[l] * yv[l];
                        mm = fmax(mm, fabs(sv[l]) / (T(1) + fabs(x[l])));
                    }
                    Q.sum3(sy, ss, yy);
                    mm = Q.max(mm);
                    const T r = T(1) / sy;
                    if (sy > T(1e-9) * dsqrt(ss * yy) && sy > T(0) && finite_(r)) {
                        hist.push(sv, yv);
                        valid = valid + 1 < kHistory ? valid + 1 : kHistory;
                    }
                    const T delta = fabs(f - cand), size = T(0.5) * (fabs(f) + fabs(cand));
#pragma unroll
                    for (int l = 0; l < L; ++l) { x[l] = tr[l]; g[l] = ng[l]; }
                    f = cand;
                    if (delta < itol * size || mm < itol) break;
                }
                f = evaluate<true>(x, rho, g);
                const T norm = Q.sum(own_norm());
                const bool feasible = norm < tol2;
#pragma unroll
                for (int r = 0; r < (REFINE ? L : 1); ++r) lam[r] -= rho * res[r];
                if (norm > T(0.0625) * oldnorm) rho *= T(10);
                T motion = T(0);
#pragma unroll
                for (int l = 0; l < L; ++l) { const T dl = x[l] - ox[l]; motion += dl * dl; }
                motion = Q.sum(motion);
                if (motion < tol2 && feasible) break;
            }
        }
    }

    // |C|^2 contribution of the residual rows owned by this lane (res[] of
    // the last evaluation).
    __device__ __forceinline__ T own_norm() const {
        if (Q.q < 3 || !REFINE) return res[0] * res[0];
        T s = T(0);
#pragma unroll
        for (int l = 0; l < L; ++l) s += res[l] * res[l];
        return s;
    }
};

}  // namespace unb
