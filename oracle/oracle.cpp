// C entry points of the CPU oracle (test infrastructure; see oracle.hpp).
//
// Loaded by tests/ and bench.py through ctypes (oracle/__init__.py). Never
// linked into the product library.
#include "oracle.hpp"

#include <atomic>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

using namespace oracle;

extern "C" {

// Same field layout as unblending_layer of the C ABI (unblending.h:67-72).
typedef struct orc_layer {
    int32_t comp_x, comp_y, comp_z;
    int32_t blend_mode;
    double mean[3];
    double precision[9];
} orc_layer;

typedef struct orc_options {
    int32_t history, inner, outer, starts, canonical;
    double inner_tolerance, outer_tolerance;
    int32_t frozen_stop;
} orc_options;

typedef struct orc_problem {
    int32_t layers, refinement, opaque, smooth, fixed_alpha, minimum;
} orc_problem;

}  // extern "C"

namespace {

std::vector<Layer> to_layers(const orc_layer* in, int L) {
    std::vector<Layer> out(L);
    for (int l = 0; l < L; ++l) {
        for (int r = 0; r < 3; ++r) out[l].mean[r] = in[l].mean[r];
        for (int k = 0; k < 9; ++k) out[l].precision[k] = in[l].precision[k];
        out[l].mode = in[l].blend_mode;
        out[l].X = in[l].comp_x; out[l].Y = in[l].comp_y; out[l].Z = in[l].comp_z;
    }
    return out;
}

Problem to_problem(const orc_problem* q) {
    Problem p;
    p.layers = q->layers; p.refinement = q->refinement; p.opaque = q->opaque;
    p.smooth = q->smooth; p.fixed_alpha = q->fixed_alpha; p.minimum = q->minimum;
    return p;
}

Options to_options(const orc_options* o) {
    Options opt;
    if (o) {
        opt.history = o->history; opt.inner = o->inner; opt.outer = o->outer; opt.starts = o->starts;
        opt.canonical = o->canonical != 0;
        opt.inner_tolerance = o->inner_tolerance; opt.outer_tolerance = o->outer_tolerance;
        opt.frozen_stop = o->frozen_stop;
    }
    return opt;
}

// Runs f(begin, end) over [0, count) in chunks on `threads` workers.
void parallel_for(size_t count, int threads, const std::function<void(size_t, size_t)>& f) {
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    if (threads == 1 || count < 256) { f(0, count); return; }
    std::atomic<size_t> next{0};
    const size_t chunk = 64;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            for (;;) {
                const size_t b = next.fetch_add(chunk);
                if (b >= count) break;
                f(b, std::min(count, b + chunk));
            }
        });
    for (auto& t : pool) t.join();
}

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Clamp-to-edge (2r+1)^2 mean filter as a dense convolution, O(r^2) per
// pixel (image_processing.cpp:120-151 with the constant kernel of
// image_processing.hpp:215-222). Planes are row-major, index y*w + x.
void box_brute(const double* in, int w, int h, int r, double* out) {
    if (r == 0) { std::memcpy(out, in, sizeof(double) * size_t(w) * h); return; }
    const int size = 2 * r + 1;
    const double weight = 1.0 / double(size * size);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            double value = 0.0;
            for (int kx = 0; kx < size; ++kx)
                for (int ky = 0; ky < size; ++ky) {
                    const int sx = clampi(x + kx - r, 0, w - 1), sy = clampi(y + ky - r, 0, h - 1);
                    value += weight * in[size_t(sy) * w + sx];
                }
            out[size_t(y) * w + x] = value;
        }
}

// Same mean filter as two clamp-to-edge sliding sums, O(1) per pixel
// (guided_filter.cuh FilterCPU::box, lines 312-333).
void box_sliding(const double* in, int w, int h, int r, double* out) {
    if (r == 0) { std::memcpy(out, in, sizeof(double) * size_t(w) * h); return; }
    std::vector<double> horizontal(size_t(w) * h);
    const double norm = double(2 * r + 1);
    for (int y = 0; y < h; ++y) {
        const double* row = in + size_t(y) * w;
        double sum = double(r + 1) * row[0];
        const int hi = std::min(r, w - 1);
        for (int x = 1; x <= hi; ++x) sum += row[x];
        if (r >= w) sum += double(r - w + 1) * row[w - 1];
        for (int x = 0; x < w; ++x) {
            horizontal[size_t(y) * w + x] = sum / norm;
            sum += row[clampi(x + r + 1, 0, w - 1)] - row[clampi(x - r, 0, w - 1)];
        }
    }
    for (int x = 0; x < w; ++x) {
        double sum = double(r + 1) * horizontal[x];
        const int hi = std::min(r, h - 1);
        for (int y = 1; y <= hi; ++y) sum += horizontal[size_t(y) * w + x];
        if (r >= h) sum += double(r - h + 1) * horizontal[size_t(h - 1) * w + x];
        for (int y = 0; y < h; ++y) {
            out[size_t(y) * w + x] = sum / norm;
            sum += horizontal[size_t(clampi(y + r + 1, 0, h - 1)) * w + x] - horizontal[size_t(clampi(y - r, 0, h - 1)) * w + x];
        }
    }
}

using BoxFn = void (*)(const double*, int, int, int, double*);

// Guidance statistics shared by every filtered channel: box means of I and
// the inverse of (cov(I) + eps*Id) per pixel (image_processing.cpp:228-256).
struct Guidance {
    int w, h;
    size_t n;
    std::vector<double> mean[3], inv[9];
};

Guidance make_guidance(const double* I, int w, int h, int r, double eps, BoxFn box) {
    Guidance G;
    G.w = w; G.h = h; G.n = size_t(w) * h;
    const size_t n = G.n;
    for (int c = 0; c < 3; ++c) { G.mean[c].resize(n); box(I + c * n, w, h, r, G.mean[c].data()); }
    std::vector<double> prod(n), var[6];
    const int pr[6] = {0, 0, 0, 1, 1, 2}, ps[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) {
        for (size_t i = 0; i < n; ++i) prod[i] = I[pr[k] * n + i] * I[ps[k] * n + i];
        var[k].resize(n);
        box(prod.data(), w, h, r, var[k].data());
        for (size_t i = 0; i < n; ++i) var[k][i] -= G.mean[pr[k]][i] * G.mean[ps[k]][i];
    }
    for (int k = 0; k < 9; ++k) G.inv[k].resize(n);
    for (size_t i = 0; i < n; ++i) {
        // Symmetric 3x3 (rr rg rb / rg gg gb / rb gb bb) + eps*Id, inverted by cofactors.
        const double a = var[0][i] + eps, d = var[1][i], e = var[2][i];
        const double f = var[3][i] + eps, hh = var[4][i], ii = var[5][i] + eps;
        const double A = f * ii - hh * hh, B = e * hh - d * ii, Cc = d * hh - e * f;
        const double D = a * ii - e * e, E = d * e - a * hh, F = a * f - d * d;
        const double det = a * A + d * B + e * Cc;
        const double m[9] = {A, B, Cc, B, D, E, Cc, E, F};
        for (int k = 0; k < 9; ++k) G.inv[k][i] = m[k] / det;
    }
    return G;
}

// q = box(a)^T I + box(b) with a = (cov(I)+eps)^-1 cov(I,p), b = mean(p) - a^T mean(I)
// (image_processing.cpp:214-273). Not clipped.
void guided(const Guidance& G, const double* p, const double* I, int r, BoxFn box, double* q) {
    const size_t n = G.n;
    const int w = G.w, h = G.h;
    std::vector<double> mp(n), prod(n), mip[3], a[3], b(n), tmp(n);
    box(p, w, h, r, mp.data());
    for (int c = 0; c < 3; ++c) {
        for (size_t i = 0; i < n; ++i) prod[i] = I[c * n + i] * p[i];
        mip[c].resize(n);
        box(prod.data(), w, h, r, mip[c].data());
        a[c].resize(n);
    }
    for (size_t i = 0; i < n; ++i) {
        const double cov[3] = {mip[0][i] - G.mean[0][i] * mp[i], mip[1][i] - G.mean[1][i] * mp[i], mip[2][i] - G.mean[2][i] * mp[i]};
        for (int c = 0; c < 3; ++c)
            a[c][i] = G.inv[3 * c + 0][i] * cov[0] + G.inv[3 * c + 1][i] * cov[1] + G.inv[3 * c + 2][i] * cov[2];
        b[i] = mp[i] - a[0][i] * G.mean[0][i] - a[1][i] * G.mean[1][i] - a[2][i] * G.mean[2][i];
    }
    box(b.data(), w, h, r, q);
    for (int c = 0; c < 3; ++c) {
        box(a[c].data(), w, h, r, tmp.data());
        for (size_t i = 0; i < n; ++i) q[i] += tmp[i] * I[c * n + i];
    }
}

}  // namespace

extern "C" {

uint32_t orc_version(void) { return 1; }

// Blend value and partials for n (s, d) pairs.
int orc_blend(int mode, size_t n, const double* s, const double* d, double* value, double* ds, double* dd) {
    if (mode < 0 || mode >= kModeCount) return 1;
    for (size_t i = 0; i < n; ++i) {
        if (value) value[i] = blend(s[i], d[i], mode);
        if (ds) ds[i] = blend_ds(s[i], d[i], mode);
        if (dd) dd[i] = blend_dd(s[i], d[i], mode);
    }
    return 0;
}

// One objective evaluation (AL value returned; energy/residual/gradient out).
double orc_evaluate(const orc_layer* layers, const orc_problem* problem, const double* x, const double* target,
                    const double* alpha, const double* lambda, double rho, double* energy, double* residual,
                    double* gradient, int derivatives) {
    const auto models = to_layers(layers, problem->layers);
    const Problem p = to_problem(problem);
    double prefix[4 * kMaxLayers], res[kMaxC], grad[kMaxN];
    const double v = evaluate(models.data(), p, x, target, alpha, lambda, rho, prefix, res, grad, derivatives != 0, energy);
    if (residual) for (int r = 0; r < p.constraints(); ++r) residual[r] = res[r];
    if (gradient && derivatives) for (int k = 0; k < 4 * p.layers; ++k) gradient[k] = grad[k];
    return v;
}

// Per-pixel solve over n pixels. Pixel-major arrays: target n*3, alpha n*L
// (may be null for unmixing), bg n*3 (may be null), initial/out n*4L.
// counters: n*5 (values, gradients, iterations, backtracks, outer) or null.
int orc_solve(const orc_layer* layers, const orc_problem* problem, const orc_options* options, size_t n,
              const double* target, const double* alpha, const double* bg, const double* initial, double* out,
              uint32_t* counters, int threads) {
    if (!problem || problem->layers <= 0 || problem->layers > kMaxLayers) return 1;
    const auto models = to_layers(layers, problem->layers);
    const Problem p = to_problem(problem);
    const Options opt = to_options(options);
    if (opt.history <= 0 || opt.history > kMaxHistory) return 1;
    const int L = p.layers, N = 4 * L;
    parallel_for(n, threads, [&](size_t b, size_t e) {
        Solver<double> s;
        s.models = models.data(); s.p = p; s.opt = opt;
        double zero3[3] = {0, 0, 0}, zeroL[kMaxLayers] = {0};
        for (size_t i = b; i < e; ++i) {
            Counters c;
            s.target = target + 3 * i;
            s.alpha = alpha ? alpha + size_t(L) * i : zeroL;
            s.bg = bg ? bg + 3 * i : zero3;
            s.counters = &c;
            s.run(initial + size_t(N) * i, out + size_t(N) * i);
            if (counters) {
                uint32_t* o = counters + 5 * i;
                o[0] = c.values; o[1] = c.gradients; o[2] = c.iterations; o[3] = c.backtracks; o[4] = c.outer;
            }
        }
    });
    return 0;
}

// The same method in FP32 arithmetic (the oracle templated on float; inputs
// rounded to float, results widened back): how far a change of precision
// alone moves the method's results. counters (n*5, or null) as orc_solve's.
int orc_solve_f32(const orc_layer* layers, const orc_problem* problem, const orc_options* options, size_t n,
                  const double* target, const double* alpha, const double* bg, const double* initial, double* out,
                  uint32_t* counters, int threads) {
    if (!problem || problem->layers <= 0 || problem->layers > kMaxLayers) return 1;
    const auto models = to_layers(layers, problem->layers);
    const Problem p = to_problem(problem);
    const Options opt = to_options(options);
    if (opt.history <= 0 || opt.history > kMaxHistory) return 1;
    const int L = p.layers, N = 4 * L;
    parallel_for(n, threads, [&](size_t b, size_t e) {
        Solver<float> s;
        s.models = models.data(); s.p = p; s.opt = opt;
        float t3[3], a[kMaxLayers], g3[3], x0[kMaxN], x1[kMaxN];
        for (size_t i = b; i < e; ++i) {
            for (int r = 0; r < 3; ++r) {
                t3[r] = float(target[3 * i + r]);
                g3[r] = bg ? float(bg[3 * i + r]) : 0.0f;
            }
            for (int l = 0; l < L; ++l) a[l] = alpha ? float(alpha[size_t(L) * i + l]) : 0.0f;
            for (int k = 0; k < N; ++k) x0[k] = float(initial[size_t(N) * i + k]);
            Counters c;
            s.target = t3; s.alpha = a; s.bg = g3; s.counters = &c;
            s.run(x0, x1);
            for (int k = 0; k < N; ++k) out[size_t(N) * i + k] = double(x1[k]);
            if (counters) {
                uint32_t* o = counters + 5 * i;
                o[0] = c.values; o[1] = c.gradients; o[2] = c.iterations; o[3] = c.backtracks; o[4] = c.outer;
            }
        }
    });
    return 0;
}

// Tight continuation ("polish") of n converged points `start` (n*4L), with
// multipliers re-estimated by least squares and initial penalty rho0.
int orc_polish(const orc_layer* layers, const orc_problem* problem, const orc_options* options, size_t n,
               const double* target, const double* alpha, const double* bg, const double* start, double rho0,
               double* out, uint32_t* counters, int threads) {
    if (!problem || problem->layers <= 0 || problem->layers > kMaxLayers) return 1;
    const auto models = to_layers(layers, problem->layers);
    const Problem p = to_problem(problem);
    const Options opt = to_options(options);
    const int L = p.layers, N = 4 * L;
    parallel_for(n, threads, [&](size_t b, size_t e) {
        Solver<double> s;
        s.models = models.data(); s.p = p; s.opt = opt;
        double zero3[3] = {0, 0, 0}, zeroL[kMaxLayers] = {0};
        for (size_t i = b; i < e; ++i) {
            Counters c;
            s.target = target + 3 * i;
            s.alpha = alpha ? alpha + size_t(L) * i : zeroL;
            s.bg = bg ? bg + 3 * i : zero3;
            s.counters = &c;
            s.polish(start + size_t(N) * i, rho0, out + size_t(N) * i);
            if (counters) {
                uint32_t* o = counters + 5 * i;
                o[0] = c.values; o[1] = c.gradients; o[2] = c.iterations; o[3] = c.backtracks; o[4] = c.outer;
            }
        }
    });
    return 0;
}

// Squared constraint norm per pixel (pixel-major like orc_solve).
int orc_constraint_norm2(const orc_layer* layers, const orc_problem* problem, size_t n, const double* x,
                         const double* target, const double* alpha, double* out) {
    const auto models = to_layers(layers, problem->layers);
    const Problem p = to_problem(problem);
    const int L = p.layers;
    double zeroL[kMaxLayers] = {0};
    for (size_t i = 0; i < n; ++i)
        out[i] = constraint_norm2(models.data(), p, x + size_t(4 * L) * i, target + 3 * i, alpha ? alpha + size_t(L) * i : zeroL);
    return 0;
}

// Mean filter of one row-major plane; brute=1 uses the O(r^2) convolution.
int orc_box(const double* in, int w, int h, int r, int brute, double* out) {
    if (w <= 0 || h <= 0 || r < 0) return 1;
    (brute ? box_brute : box_sliding)(in, w, h, r, out);
    return 0;
}

// Guided filter of `channels` planes p (planar, channels*n) with the RGB
// guidance I (planar 3*n). Output q is not clipped.
int orc_guided(const double* p, int channels, const double* I, int w, int h, int r, double eps, int brute, double* q) {
    if (w <= 0 || h <= 0 || r < 0) return 1;
    const size_t n = size_t(w) * h;
    if (r == 0) { std::memcpy(q, p, sizeof(double) * n * channels); return 0; }
    BoxFn box = brute ? box_brute : box_sliding;
    const Guidance G = make_guidance(I, w, h, r, eps, box);
    for (int c = 0; c < channels; ++c) guided(G, p + c * n, I, r, box, q + c * n);
    return 0;
}

// Refinement targets from the first pass (planar [alpha_0..alpha_{L-1},
// rgb_0..rgb_{L-1}] x n): filter every alpha (and the background RGB when
// smooth), clip to [0,1], normalize (all-Plus divides by the alpha sum; an
// all-SourceOver stack needs alpha_0 == 1 within 1e-5), and carry the first-pass
// background when not smoothing. targets: planar (L+3) x n. status per pixel:
// 0 valid, 1 zero Plus sum, 2 non-opaque SourceOver background.
// (unblending.cpp:311-399; streaming_guided_filter.cuh:34-60)
int orc_refine_targets(const double* rgb, const double* first, const orc_layer* layers, int L, int w, int h,
                       int opaque, int smooth, int radius, double eps, int brute, double* targets, int32_t* status) {
    if (w <= 0 || h <= 0 || L <= 0 || radius < 0) return 1;
    bool plus = true, source_over = true;
    for (int l = 0; l < L; ++l) {
        plus &= layers[l].comp_x == 2 && layers[l].comp_y == 1 && layers[l].comp_z == 1;
        source_over &= layers[l].comp_x == 1 && layers[l].comp_y == 1 && layers[l].comp_z == 1;
    }
    if ((!plus && !source_over) || (smooth && !opaque)) return 1;
    const size_t n = size_t(w) * h;
    const int channels = L + (smooth ? 3 : 0);
    std::vector<double> q(size_t(channels) * n);
    orc_guided(first, channels, rgb, w, h, radius, eps, brute, q.data());
    for (size_t i = 0; i < n; ++i) {
        double sum = 0;
        for (int c = 0; c < channels; ++c) {
            const double v = clip01(q[c * n + i]);
            targets[c * n + i] = v;
            if (c < L) sum += v;
        }
        int32_t code = 0;
        if (plus) {
            if (sum > 0) for (int l = 0; l < L; ++l) targets[l * n + i] = targets[l * n + i] / sum;
            else code = 1;
        } else if (std::abs(targets[i] - 1.0) >= 1e-5) {
            code = 2;
        }
        if (!smooth) for (int r = 0; r < 3; ++r) targets[(L + r) * n + i] = first[(L + r) * n + i];
        if (status) status[i] = code;
    }
    return 0;
}

}  // extern "C"
