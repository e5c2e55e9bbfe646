// CPU oracle for the color-unmixing / matte-refinement hot path.
//
// TEST INFRASTRUCTURE ONLY. This header is the checker that the CUDA path is
// compared against; it is never linked into the product library. Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm load it.
//
// It restates, in plain double-precision C++, the algorithm of the reference
// (TheDucker1/unblending) for this path:
//   * scalar blend functions and partials ........ unblending/include/unblending/blend_mode.hpp:88-196
//                                                    (FP64 twin: unblending/src/cuda/compositing/blend_fp64.hpp)
//   * bottom-to-top composite ..................... unblending/src/equations.cpp:10-74,
//                                                    unblending/src/cuda/model/pixel_problem.cuh:68-74
//   * energy, constraint vector, AL value and the
//     reverse-mode gradient ....................... unblending/src/cuda/model/pixel_problem.cuh:40-49,75-110
//   * variable bounds ............................. unblending/src/cuda/model/pixel_problem.cuh:111-116,
//                                                    unblending/src/cuda/solver/augmented_lagrangian.cuh:49-52
//   * augmented-Lagrangian outer loop around a
//     projected L-BFGS inner solve, starts and
//     best-feasible tracking ...................... unblending/src/cuda/solver/augmented_lagrangian.cuh:20-149
//   * initial points .............................. unblending/src/cuda/solver/fallback_solver_kernels.cuh:68-76
//   * guided filter (O(r^2) box convolution) ..... unblending/src/image_processing.cpp:120-151,214-273,
//                                                    unblending/include/unblending/image_processing.hpp:215-222
//   * guided filter (O(n) sliding box) ........... unblending/src/cuda/refinement/guided_filter.cuh:14-45,
//                                                    unblending/src/cuda/refinement/streaming_guided_filter.cuh:34-111
//   * refinement targets, normalization .......... unblending/src/unblending.cpp:311-439,
//                                                    unblending/src/cuda/refinement/filtered_matte_targets.cuh:119-144
//
// Parity pin: oracle/Makefile (target ref) compiles the reference's own host-capable
// headers into oracle/_ref/libunbref.so; tests/golden/make_golden.py records
// its outputs as fixtures, and tests/test_oracle_golden.py checks this oracle
// against them (bit-exact for blend/evaluate/solve, 1e-12 for the filter).
//
// The inner arithmetic follows the reference's operation order so that an
// FP64 solve reproduces the reference's FP64 solve bit for bit when both are
// compiled with -ffp-contract=off.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <algorithm>
#include <limits>

namespace oracle {

enum Mode : int {
    Normal = 0, Multiply, Screen, Overlay, Darken, Lighten, ColorDodge, ColorBurn,
    HardLight, SoftLight, Difference, Exclusion, LinearDodge
};
constexpr int kModeCount = 13;

// One layer: Porter-Duff coefficients (X,Y,Z), separable blend mode, and a
// Gaussian color model (mean and precision = inverse covariance, row-major).
struct Layer {
    double mean[3];
    double precision[9];
    int mode;
    int X, Y, Z;
};

// Per-pass flags. Unmixing: refinement=false, minimum=true. Refinement:
// refinement=true, fixed_alpha=true (alphas pinned to the filtered targets by
// their bounds), smooth pins the background RGB to the filtered background.
struct Problem {
    int layers = 0;
    bool refinement = false, opaque = true, smooth = false, fixed_alpha = false, minimum = true;
    int constraints() const { return 3 + (refinement ? layers : 1); }
};

struct Options {
    int history = 6, inner = 256, outer = 22, starts = 1;
    bool canonical = false;
    double inner_tolerance = 5e-3, outer_tolerance = 5e-3;
    // Not in the reference: stop a start after this many consecutive outer
    // steps that moved neither x nor the best point (0 = never), the rule the
    // CUDA path's FP64 re-solve applies; lets the tests check on the CPU that
    // it leaves the results unchanged.
    int frozen_stop = 0;
};

struct Counters {
    unsigned values = 0, gradients = 0, iterations = 0, backtracks = 0, outer = 0;
};

// ---------------------------------------------------------------- blend -----
constexpr double kBlendEps = 1e-5;   // blend_mode.hpp:88

template <class T> inline T blend(T s, T d, int mode) {
    const T one = T(1), two = T(2), eps = T(kBlendEps);
    switch (mode) {
    case Normal: return s;
    case Multiply: return s * d;
    case Screen: return one - (one - s) * (one - d);
    case Overlay: return d <= T(0.5) ? two * s * d : one - two * (one - s) * (one - d);
    case Darken: return s < d ? s : d;
    case Lighten: return s < d ? d : s;
    case ColorDodge:
        if (d < eps) return T(0);
        if (one - s < eps) return one;
        return std::min(one, d / (one - s));
    case ColorBurn:
        if (one - d < eps) return one;
        if (s < eps) return T(0);
        return one - std::min(one, (one - d) / s);
    case HardLight: return s <= T(0.5) ? two * s * d : one - two * (one - s) * (one - d);
    case SoftLight: {
        if (s <= T(0.5)) return d - (one - two * s) * d * (one - d);
        const T g = d <= T(0.25) ? ((T(16) * d - T(12)) * d + T(4)) * d : std::sqrt(d);
        return d + (two * s - one) * (g - d);
    }
    case Difference: return s < d ? d - s : s - d;
    case Exclusion: return s + d - two * s * d;
    case LinearDodge: return s + d;
    default: return T(0);
    }
}

template <class T> inline T blend_ds(T s, T d, int mode) {
    const T one = T(1), two = T(2), eps = T(kBlendEps);
    switch (mode) {
    case Normal: return one;
    case Multiply: return d;
    case Screen: return one - d;
    case Overlay: return d <= T(0.5) ? two * d : two * (one - d);
    case Darken: return s < d ? one : T(0);
    case Lighten: return s < d ? T(0) : one;
    case ColorDodge:
        if (d < eps || one - s < eps || one < d / (one - s)) return T(0);
        return d / ((one - s) * (one - s));
    case ColorBurn:
        if (one - d < eps || s < eps) return T(0);
        return -(one < (one - d) / s ? T(0) : -(one - d) / (s * s));
    case HardLight: return s <= T(0.5) ? two * d : two * (one - d);
    case SoftLight: {
        if (s <= T(0.5)) return two * d * (one - d);
        const T g = d <= T(0.25) ? ((T(16) * d - T(12)) * d + T(4)) * d : std::sqrt(d);
        return two * (g - d);
    }
    case Difference: return s < d ? -one : one;
    case Exclusion: return one - two * d;
    case LinearDodge: return one;
    default: return T(0);
    }
}

template <class T> inline T blend_dd(T s, T d, int mode) {
    const T one = T(1), two = T(2), eps = T(kBlendEps);
    switch (mode) {
    case Normal: return T(0);
    case Multiply: return s;
    case Screen: return one - s;
    case Overlay: return d <= T(0.5) ? two * s : two * (one - s);
    case Darken: return s < d ? T(0) : one;
    case Lighten: return s < d ? one : T(0);
    case ColorDodge:
        if (d < eps || one - s < eps || one < d / (one - s)) return T(0);
        return one / (one - s);
    case ColorBurn:
        if (one - d < eps || s < eps) return T(0);
        return -(one < (one - d) / s ? T(0) : -one / s);
    case HardLight: return s <= T(0.5) ? two * s : two * (one - s);
    case SoftLight: {
        if (s <= T(0.5)) return two * s + two * d - T(4) * s * d;
        const T h = d <= T(0.25) ? (T(48) * d * d - T(24) * d + T(4)) : (one / (two * std::sqrt(d)));
        return one + (two * s - one) * h - (two * s - one);
    }
    case Difference: return s < d ? one : -one;
    case Exclusion: return one - two * s;
    case LinearDodge: return one;
    default: return T(0);
    }
}

template <class T> inline T clip01(T v) { return v < T(0) ? T(0) : (v > T(1) ? T(1) : v); }

// ------------------------------------------------------------ evaluation ----
// Quadratic color cost (c-mu)^T P (c-mu) and its gradient (P + P^T)(c-mu).
template <class T> inline T gaussian_cost(const Layer& m, const T* c, T* grad) {
    T delta[3], v[3] = {T(0), T(0), T(0)}, cost = T(0);
    for (int r = 0; r < 3; ++r) delta[r] = c[r] - T(m.mean[r]);
    for (int r = 0; r < 3; ++r) {
        for (int s = 0; s < 3; ++s) v[r] += T(m.precision[3 * r + s]) * delta[s];
        cost += delta[r] * v[r];
    }
    if (grad)
        for (int r = 0; r < 3; ++r) {
            grad[r] = v[r];
            for (int s = 0; s < 3; ++s) grad[r] += T(m.precision[3 * s + r]) * delta[s];
        }
    return cost;
}

// Bottom-to-top composite. x = [alpha_0..alpha_{L-1}, rgb_0..rgb_{L-1}];
// prefix holds (r,g,b,A) after each layer: prefix[4*l + {0,1,2,3}].
template <class T> inline void composite(const Layer* models, int L, const T* x, T* prefix) {
    for (int r = 0; r < 3; ++r) prefix[r] = x[L + r];
    prefix[3] = x[0];
    for (int l = 1; l < L; ++l) {
        const Layer& m = models[l];
        const T a = x[l], d = prefix[4 * (l - 1) + 3];
        const T A = T(m.X) * a * d + T(m.Y) * a * (T(1) - d) + T(m.Z) * d * (T(1) - a);
        prefix[4 * l + 3] = A;
        for (int r = 0; r < 3; ++r) {
            const T s = x[L + 3 * l + r], c = prefix[4 * (l - 1) + r];
            const T pre = blend(s, c, m.mode) * a * d + T(m.Y) * a * (T(1) - d) * s + T(m.Z) * d * (T(1) - a) * c;
            prefix[4 * l + r] = A > T(1e-12) ? pre / A : pre;
        }
    }
}

// Augmented-Lagrangian value E + sum(rho/2 C^2 - lambda C) and, optionally,
// its gradient. `energy` receives E alone (including the 0.01*sum(alpha)
// minimum-alpha term of the unmixing pass); `residual` receives C.
template <class T>
T evaluate(const Layer* models, const Problem& p, const T* x, const T* target, const T* alpha,
           const T* lambda, T rho, T* prefix, T* residual, T* gradient, bool derivatives, T* energy_out) {
    const int L = p.layers;
    composite(models, L, x, prefix);
    T energy = T(0), asum = T(0);
    for (int l = 0; l < L; ++l) {
        T g[3];
        const T D = gaussian_cost(models[l], x + L + 3 * l, derivatives ? g : nullptr);
        energy += x[l] * D;
        if (derivatives) {
            gradient[l] = D;
            for (int r = 0; r < 3; ++r) gradient[L + 3 * l + r] = x[l] * g[r];
        }
        asum += x[l];
    }
    if (p.minimum) {
        energy += T(0.01) * asum;
        if (derivatives)
            for (int l = 0; l < L; ++l) gradient[l] += T(0.01);
    }
    if (energy_out) *energy_out = energy;
    for (int r = 0; r < 3; ++r) residual[r] = prefix[4 * (L - 1) + r] - target[r];
    if (p.refinement)
        for (int l = 0; l < L; ++l) residual[3 + l] = x[l] - alpha[l];
    else
        residual[3] = prefix[4 * (L - 1) + 3] - T(1);
    const int C = p.constraints();
    for (int r = 0; r < C; ++r) energy += T(0.5) * rho * residual[r] * residual[r] - lambda[r] * residual[r];
    if (!derivatives) return energy;

    T adj[4];
    for (int r = 0; r < 3; ++r) adj[r] = rho * residual[r] - lambda[r];
    adj[3] = p.refinement ? T(0) : rho * residual[3] - lambda[3];
    if (p.refinement)
        for (int l = 0; l < L; ++l) gradient[l] += rho * residual[3 + l] - lambda[3 + l];
    for (int l = L - 1; l > 0; --l) {
        const Layer& m = models[l];
        const T a = x[l], d = prefix[4 * (l - 1) + 3], A = prefix[4 * l + 3];
        const T da = T(m.X) * d + T(m.Y) * (T(1) - d) - T(m.Z) * d;
        const T dd = T(m.X) * a - T(m.Y) * a + T(m.Z) * (T(1) - a);
        T ga = adj[3] * da, prev = adj[3] * dd;
        const bool big = A > T(1e-12);
        for (int r = 0; r < 3; ++r) {
            const T s = x[L + 3 * l + r], c = prefix[4 * (l - 1) + r];
            const T f = blend(s, c, m.mode), v = adj[r], out = prefix[4 * l + r];
            const T ds = a * d * blend_ds(s, c, m.mode) + T(m.Y) * a * (T(1) - d);
            const T dc = a * d * blend_dd(s, c, m.mode) + T(m.Z) * d * (T(1) - a);
            const T pa = f * d + T(m.Y) * (T(1) - d) * s - T(m.Z) * d * c;
            const T pd = f * a - T(m.Y) * a * s + T(m.Z) * (T(1) - a) * c;
            ga += v * (big ? (pa - out * da) / A : pa);
            prev += v * (big ? (pd - out * dd) / A : pd);
            gradient[L + 3 * l + r] += v * (big ? ds / A : ds);
            adj[r] = v * (big ? dc / A : dc);
        }
        gradient[l] += ga;
        adj[3] = prev;
    }
    gradient[0] += adj[3];
    for (int r = 0; r < 3; ++r) gradient[L + r] += adj[r];
    return energy;
}

// Bounds of variable k: alphas and colors live in [0,1]; an opaque
// background pins alpha_0 = 1; fixed refinement alphas pin alpha_l to the
// filtered target; background smoothing pins the background RGB.
template <class T> inline T bound(const Problem& p, const T* alpha, const T* bg, int k, bool high) {
    const int L = p.layers;
    if (k < L) {
        if (p.opaque && k == 0) return T(1);
        if (p.refinement && p.fixed_alpha) return alpha[k];
    }
    if (p.refinement && p.smooth && k >= L && k < L + 3) return bg[k - L];
    return high ? T(1) : T(0);
}

// ---------------------------------------------------------------- solver ----
constexpr int kMaxLayers = 16;
constexpr int kMaxN = 4 * kMaxLayers;
constexpr int kMaxHistory = 16;
constexpr int kMaxC = 3 + kMaxLayers;

template <class T> struct Solver {
    const Layer* models;
    Problem p;
    Options opt;
    const T* target;
    const T* alpha;
    const T* bg;
    Counters* counters;

    int L, N, H, C;
    T x[kMaxN], g[kMaxN], dir[kMaxN], trial[kMaxN], newg[kMaxN], outer_x[kMaxN], best[kMaxN];
    T prefix[4 * kMaxLayers], residual[kMaxC], lambda[kMaxC];
    T hs[kMaxHistory][kMaxN], hy[kMaxHistory][kMaxN], coeff[kMaxHistory], inv[kMaxHistory];
    T best_norm, best_energy;
    bool have_best;
    long best_updates = 0;

    T lo(int k) const { return bound(p, alpha, bg, k, false); }
    T hi(int k) const { return bound(p, alpha, bg, k, true); }

    // Objective evaluation with best-feasible tracking over every point that
    // the solver evaluates (augmented_lagrangian.cuh:233-241).
    T eval(T* point, T* gradient, T rho, bool derivative) {
        if (counters) { ++counters->values; if (derivative) ++counters->gradients; }
        T energy;
        const T value = evaluate(models, p, point, target, alpha, lambda, rho, prefix, residual, gradient, derivative, &energy);
        T norm = T(0);
        const T tol = T(opt.outer_tolerance * opt.outer_tolerance);
        for (int r = 0; r < C; ++r) norm += residual[r] * residual[r];
        const bool feasible = norm < tol;
        if (std::isfinite(energy) && std::isfinite(norm) &&
            (!have_best || (feasible && (best_norm >= tol || energy < best_energy)) ||
             (!feasible && best_norm >= tol && norm < best_norm))) {
            have_best = true; best_norm = norm; best_energy = energy;
            for (int k = 0; k < N; ++k) best[k] = point[k];
            ++best_updates;
        }
        return value;
    }

    // Two-loop recursion restricted to the current free set
    // (augmented_lagrangian.cuh:184-203). `free_mask`, `q` are length N.
    void inverse_step(int valid, int next, const T* free_mask, T* q) {
        for (int k = 0; k < N; ++k) q[k] = free_mask[k] != T(0) ? g[k] : T(0);
        T scaling = T(1);
        bool have_scaling = false;
        for (int j = 0; j < valid; ++j) {
            const int slot = (next - 1 - j + H) % H;
            T dot = T(0), sy = T(0), ss = T(0), yy = T(0);
            for (int k = 0; k < N; ++k)
                if (free_mask[k] != T(0)) {
                    const T a = hs[slot][k], b = hy[slot][k];
                    dot += a * q[k]; sy += a * b; ss += a * a; yy += b * b;
                }
            inv[slot] = (sy > T(1e-9) * std::sqrt(ss * yy) && sy > T(0) && std::isfinite(T(1) / sy)) ? T(1) / sy : T(0);
            coeff[slot] = dot * inv[slot];
            for (int k = 0; k < N; ++k)
                if (free_mask[k] != T(0)) q[k] -= coeff[slot] * hy[slot][k];
            if (!have_scaling && inv[slot] > T(0) && yy > T(0)) { scaling = sy / yy; have_scaling = true; }
        }
        scaling = std::max(T(1e-12), std::min(T(1e3), scaling));
        for (int k = 0; k < N; ++k) q[k] *= scaling;
        for (int j = valid - 1; j >= 0; --j) {
            const int slot = (next - 1 - j + H) % H;
            T dot = T(0);
            for (int k = 0; k < N; ++k)
                if (free_mask[k] != T(0)) dot += hy[slot][k] * q[k];
            const T a = coeff[slot] - dot * inv[slot];
            for (int k = 0; k < N; ++k)
                if (free_mask[k] != T(0)) q[k] += a * hs[slot][k];
        }
    }

    bool canonicalize(T* point) {
        bool changed = false;
        for (int l = 1; l < L; ++l)
            if (point[l] == T(0))
                for (int r = 0; r < 3; ++r) {
                    const int k = L + 3 * l + r;
                    T v = T(models[l].mean[r]);
                    v = std::max(lo(k), std::min(hi(k), v));
                    changed |= point[k] != v;
                    point[k] = v;
                }
        return changed;
    }

    bool is_fixed(int k, T gk) const {
        const T l = lo(k), h = hi(k);
        return l == h || (x[k] <= l && gk > T(0)) || (x[k] >= h && gk < T(0));
    }

    void steepest() {
        for (int k = 0; k < N; ++k) dir[k] = is_fixed(k, g[k]) ? T(0) : -g[k];
    }

    // Starting point `start` (augmented_lagrangian.cuh:243-263).
    void seed(int start, const T* initial) {
        for (int k = 0; k < N; ++k) {
            T value = initial[k];
            const int layer = (k - L) / 3, channel = (k - L) % 3;
            if (!p.refinement && start == 1)
                value = k < L ? (k == 0 ? T(1) : T(0)) : (k < L + 3 ? clip01(target[k - L]) : T(models[layer].mean[channel]));
            if (p.refinement && start && k >= L) value = T(models[layer].mean[channel]);
            if (start == 2) {
                if (k < L) value = p.refinement ? initial[k] : T(0.5);
                else value = std::max(T(0.05), std::min(T(0.95), T(models[layer].mean[channel])));
            }
            const T l = lo(k), h = hi(k);
            x[k] = value < l ? l : (value > h ? h : value);
        }
        if (start == 2) {
            // Move Dodge/Burn sources into the unsaturated branch of the
            // current destination (augmented_lagrangian.cuh:249-263).
            T dest[3];
            for (int r = 0; r < 3; ++r) dest[r] = x[L + r];
            T da = x[0];
            for (int l = 1; l < L; ++l) {
                const Layer& m = models[l];
                const T a = x[l];
                const T A = T(m.X) * a * da + T(m.Y) * a * (T(1) - da) + T(m.Z) * da * (T(1) - a);
                for (int r = 0; r < 3; ++r) {
                    const int k = L + 3 * l + r;
                    T s = x[k];
                    const T d = dest[r];
                    if (d >= T(0) && d <= T(1) && m.mode == ColorDodge) s = std::min(s, std::max(T(0), T(1) - d - T(0.05)));
                    if (d >= T(0) && d <= T(1) && m.mode == ColorBurn) s = std::max(s, std::min(T(1), T(1) - d + T(0.05)));
                    s = std::max(lo(k), std::min(hi(k), s));
                    x[k] = s;
                    const T pre = blend(s, d, m.mode) * a * da + T(m.Y) * a * (T(1) - da) * s + T(m.Z) * da * (T(1) - a) * d;
                    dest[r] = A > T(1e-12) ? pre / A : pre;
                }
                da = A;
            }
        }
    }

    void run(const T* initial, T* output) {
        L = p.layers; N = 4 * L; H = opt.history; C = p.constraints();
        have_best = false;
        best_norm = T(INFINITY); best_energy = T(INFINITY);
        for (int start = 0; start < opt.starts; ++start) {
            seed(start, initial);
            for (int r = 0; r < C; ++r) lambda[r] = T(0);
            augmented_lagrangian(T(100));
        }
        for (int k = 0; k < N; ++k) output[k] = have_best ? best[k] : initial[k];
    }

    // Least-squares multiplier estimate at x: min |grad E_F - J_F^T lambda|
    // over the variables F strictly inside their bounds.
    void estimate_multipliers() {
        T gE[kMaxN], J[kMaxC][kMaxN], zero[kMaxC] = {}, tmp[kMaxN];
        for (int r = 0; r < C; ++r) zero[r] = T(0);
        T e;
        evaluate(models, p, x, target, alpha, zero, T(0), prefix, residual, gE, true, &e);
        for (int r = 0; r < C; ++r) {
            T unit[kMaxC];
            for (int q = 0; q < C; ++q) unit[q] = q == r ? T(-1) : T(0);
            evaluate(models, p, x, target, alpha, unit, T(0), prefix, residual, tmp, true, &e);
            for (int k = 0; k < N; ++k) J[r][k] = tmp[k] - gE[k];
        }
        T A[kMaxC][kMaxC + 1];
        for (int r = 0; r < C; ++r) {
            for (int q = 0; q < C; ++q) {
                T s = T(0);
                for (int k = 0; k < N; ++k) if (lo(k) < x[k] && x[k] < hi(k)) s += J[r][k] * J[q][k];
                A[r][q] = s + (r == q ? T(1e-12) : T(0));
            }
            T s = T(0);
            for (int k = 0; k < N; ++k) if (lo(k) < x[k] && x[k] < hi(k)) s += J[r][k] * gE[k];
            A[r][C] = s;
        }
        for (int c = 0; c < C; ++c) {   // Gaussian elimination with partial pivoting
            int piv = c;
            for (int r = c + 1; r < C; ++r) if (std::abs(A[r][c]) > std::abs(A[piv][c])) piv = r;
            if (piv != c) for (int q = 0; q <= C; ++q) std::swap(A[c][q], A[piv][q]);
            for (int r = c + 1; r < C; ++r) {
                const T f = A[r][c] / A[c][c];
                for (int q = c; q <= C; ++q) A[r][q] -= f * A[c][q];
            }
        }
        for (int r = C - 1; r >= 0; --r) {
            T s = A[r][C];
            for (int q = r + 1; q < C; ++q) s -= A[r][q] * lambda[q];
            lambda[r] = s / A[r][r];
        }
    }

    // Tight continuation from a converged point: multipliers from the
    // least-squares estimate, then the same AL loop with this solver's
    // (tight) tolerances; best-feasible tracking at the tight tolerance.
    void polish(const T* start_point, T rho0, T* output) {
        L = p.layers; N = 4 * L; H = opt.history; C = p.constraints();
        have_best = false;
        best_norm = T(INFINITY); best_energy = T(INFINITY);
        for (int k = 0; k < N; ++k) x[k] = std::max(lo(k), std::min(hi(k), start_point[k]));
        estimate_multipliers();
        augmented_lagrangian(rho0);
        for (int k = 0; k < N; ++k) output[k] = have_best ? best[k] : start_point[k];
    }

    void augmented_lagrangian(T rho) {
        const T tol2 = T(opt.outer_tolerance * opt.outer_tolerance);
        {
            int frozen = 0;
            for (int outer = 0; outer < opt.outer; ++outer) {
                if (counters) ++counters->outer;
                const long updates_before = best_updates;
                if (opt.canonical) canonicalize(x);
                for (int k = 0; k < N; ++k) outer_x[k] = x[k];
                T f = eval(x, g, rho, true);
                T oldnorm = T(0);
                for (int r = 0; r < C; ++r) oldnorm += residual[r] * residual[r];
                int valid = 0, next = 0;
                for (int iteration = 0; iteration < opt.inner; ++iteration) {
                    if (counters) ++counters->iterations;
                    // trial[] doubles as the free-variable mask here.
                    T pg2 = T(0);
                    for (int k = 0; k < N; ++k) {
                        const bool fixed = is_fixed(k, g[k]);
                        trial[k] = fixed ? T(0) : T(1);
                        dir[k] = fixed ? T(0) : g[k];
                        pg2 += dir[k] * dir[k];
                    }
                    if (pg2 < T(1e-16) || !std::isfinite(f)) break;
                    inverse_step(valid, next, trial, dir);
                    T descent = T(0);
                    for (int k = 0; k < N; ++k) {
                        T d = -dir[k];
                        const T l = lo(k), h = hi(k);
                        if (l == h || (x[k] <= l && d < T(0)) || (x[k] >= h && d > T(0))) d = T(0);
                        dir[k] = d;
                        descent += d * g[k];
                    }
                    if (!(descent < T(0))) { valid = 0; next = 0; steepest(); }
                    bool accepted = false;
                    T candidate = f;
                    for (int attempt = 0; attempt < 2 && !accepted; ++attempt) {
                        T step = T(1);
                        for (int backtrack = 0; backtrack < 32; ++backtrack) {
                            T slope = T(0), motion = T(0);
                            for (int k = 0; k < N; ++k) {
                                trial[k] = std::max(lo(k), std::min(hi(k), x[k] + step * dir[k]));
                                const T delta = trial[k] - x[k];
                                slope += g[k] * delta;
                                motion += delta * delta;
                            }
                            if (motion == T(0)) break;
                            candidate = eval(trial, newg, rho, false);
                            if (counters) ++counters->backtracks;
                            if (slope < T(0) && std::isfinite(candidate) && candidate <= f + T(1e-4) * slope) { accepted = true; break; }
                            step *= T(0.5);
                        }
                        if (!accepted) { valid = 0; next = 0; steepest(); }
                    }
                    if (!accepted) break;
                    const bool canonical = opt.canonical && canonicalize(trial);
                    candidate = eval(trial, newg, rho, true);
                    T sy = T(0), ss = T(0), yy = T(0), maxmotion = T(0);
                    for (int k = 0; k < N; ++k) {
                        const T s = trial[k] - x[k], y = newg[k] - g[k];
                        sy += s * y; ss += s * s; yy += y * y;
                        maxmotion = std::max(maxmotion, std::abs(s) / (T(1) + std::abs(x[k])));
                    }
                    if (canonical) { valid = 0; next = 0; }
                    else if (sy > T(1e-9) * std::sqrt(ss * yy) && sy > T(0) && std::isfinite(T(1) / sy)) {
                        for (int k = 0; k < N; ++k) { hs[next][k] = trial[k] - x[k]; hy[next][k] = newg[k] - g[k]; }
                        inv[next] = T(1) / sy;
                        next = (next + 1) % H;
                        valid = std::min(valid + 1, H);
                    }
                    const T delta = std::abs(f - candidate), size = T(0.5) * (std::abs(f) + std::abs(candidate));
                    for (int k = 0; k < N; ++k) { x[k] = trial[k]; g[k] = newg[k]; }
                    f = candidate;
                    if (!canonical && (delta < T(opt.inner_tolerance) * size || maxmotion < T(opt.inner_tolerance))) break;
                }
                f = eval(x, g, rho, true);
                T norm = T(0), motion = T(0);
                for (int r = 0; r < C; ++r) norm += residual[r] * residual[r];
                const bool feasible = norm < tol2;
                for (int r = 0; r < C; ++r) lambda[r] -= rho * residual[r];
                if (norm > T(0.0625) * oldnorm) rho *= T(10);
                for (int k = 0; k < N; ++k) { const T d = x[k] - outer_x[k]; motion += d * d; }
                frozen = (motion == T(0) && best_updates == updates_before) ? frozen + 1 : 0;
                if (opt.frozen_stop > 0 && frozen >= opt.frozen_stop) break;
                if (motion < tol2 && feasible) break;
            }
        }
    }
};

// Initial point of the first pass (fallback_solver_kernels.cuh:68-71):
// alpha 0.5 (1 for an opaque background), colors at the clipped means.
template <class T> inline void initial_first(const Layer* models, const Problem& p, T* x) {
    const int L = p.layers;
    for (int l = 0; l < L; ++l) {
        x[l] = (p.opaque && l == 0) ? T(1) : T(0.5);
        for (int r = 0; r < 3; ++r) x[L + 3 * l + r] = clip01(T(models[l].mean[r]));
    }
}

// Squared constraint norm of a final point, used as the per-pixel
// feasibility check (tolerance 5e-3 on the norm, as the reference's guard).
template <class T> inline T constraint_norm2(const Layer* models, const Problem& p, const T* x, const T* target, const T* alpha) {
    T prefix[4 * kMaxLayers];
    const int L = p.layers;
    composite(models, L, x, prefix);
    T norm = T(0);
    for (int r = 0; r < 3; ++r) { const T d = prefix[4 * (L - 1) + r] - target[r]; norm += d * d; }
    if (p.refinement) for (int l = 0; l < L; ++l) { const T d = x[l] - alpha[l]; norm += d * d; }
    else { const T d = prefix[4 * (L - 1) + 3] - T(1); norm += d * d; }
    return norm;
}

}  // namespace oracle
