// Thin C shim over the reference's own host-capable solver headers.
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile (target ref) compiles this file against
// the reference sources where they lie (unblending/src/cuda, included by
// path) into oracle/_ref/libunbref.so. It is the pin for the oracle
// restatement in oracle.hpp: tests/golden/make_golden.py records its outputs.
//
// Wrapped reference symbols:
//   firstpass::blend / blend_grad_s / blend_grad_d    compositing/blend_fp64.hpp
//   general::Program<double,GaussianPrior>::evaluate  model/pixel_problem.cuh:75-110
//   general::Optimizer<double,GaussianPrior>::solve   solver/augmented_lagrangian.cuh:220-304
#include "solver/augmented_lagrangian.cuh"

#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

extern "C" {
typedef struct ref_layer {
    int32_t comp_x, comp_y, comp_z;
    int32_t blend_mode;
    double mean[3];
    double precision[9];
} ref_layer;
typedef struct ref_options {
    int32_t history, inner, outer, starts, canonical;
    double inner_tolerance, outer_tolerance;
} ref_options;
typedef struct ref_problem {
    int32_t layers, refinement, opaque, smooth, fixed_alpha, minimum;
} ref_problem;
}

namespace {
std::vector<general::Layer> convert(const ref_layer* in, int L) {
    std::vector<general::Layer> out(L);
    for (int l = 0; l < L; ++l) {
        for (int r = 0; r < 3; ++r) out[l].mean[r] = in[l].mean[r];
        for (int k = 0; k < 9; ++k) out[l].inverse[k] = in[l].precision[k];
        out[l].mode = in[l].blend_mode;
        out[l].X = in[l].comp_x; out[l].Y = in[l].comp_y; out[l].Z = in[l].comp_z;
        out[l].gray = 0;
    }
    return out;
}
general::Problem convert(const ref_problem* q) {
    general::Problem p{q->layers};
    p.refinement = q->refinement; p.opaque = q->opaque; p.smooth = q->smooth;
    p.fixed_alpha = q->fixed_alpha; p.minimum = q->minimum; p.sparsity = false;
    return p;
}
using Program = general::Program<double, general::GaussianPrior, general::Layer>;
using Optimizer = general::Optimizer<double, general::GaussianPrior, general::Layer>;
}  // namespace

extern "C" {

uint32_t ref_version(void) { return 1; }

int ref_blend(int mode, size_t n, const double* s, const double* d, double* value, double* ds, double* dd) {
    const auto m = static_cast<firstpass::BlendMode>(mode);
    for (size_t i = 0; i < n; ++i) {
        if (value) value[i] = firstpass::blend(s[i], d[i], m);
        if (ds) ds[i] = firstpass::blend_grad_s(s[i], d[i], m);
        if (dd) dd[i] = firstpass::blend_grad_d(s[i], d[i], m);
    }
    return 0;
}

double ref_evaluate(const ref_layer* layers, const ref_problem* problem, const double* x, const double* target,
                    const double* alpha, const double* lambda, double rho, double* energy, double* residual,
                    double* gradient, int derivatives) {
    const auto models = convert(layers, problem->layers);
    const auto p = convert(problem);
    std::vector<double> prefix(4 * p.layers), res(p.constraints(models.data())), grad(4 * p.layers);
    std::vector<double> alpha_buf(p.layers, 0.0);
    if (alpha) for (int l = 0; l < p.layers; ++l) alpha_buf[l] = alpha[l];
    const double v = Program::evaluate(models.data(), p, {x}, target, {alpha_buf.data()}, {lambda}, rho, {prefix.data()},
                                       {res.data()}, {grad.data()}, derivatives != 0, energy);
    if (residual) for (size_t r = 0; r < res.size(); ++r) residual[r] = res[r];
    if (gradient && derivatives) for (size_t k = 0; k < grad.size(); ++k) gradient[k] = grad[k];
    return v;
}

int ref_solve(const ref_layer* layers, const ref_problem* problem, const ref_options* options, size_t n,
              const double* target, const double* alpha, const double* bg, const double* initial, double* out,
              uint32_t* counters, int threads) {
    const auto models = convert(layers, problem->layers);
    const auto p = convert(problem);
    general::Options opt;
    opt.history = options->history; opt.inner = options->inner; opt.outer = options->outer;
    opt.starts = options->starts; opt.canonical = options->canonical != 0;
    opt.inner_tolerance = options->inner_tolerance; opt.outer_tolerance = options->outer_tolerance;
    opt.correction = false; opt.project_gray = false;
    const int L = p.layers, N = 4 * L, C = p.constraints(models.data());
    const int words = Optimizer::workspace(p, C, opt);
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    std::atomic<size_t> next{0};
    auto work = [&] {
        std::vector<double> memory(words), zeroL(L, 0.0), zero3(3, 0.0);
        for (;;) {
            const size_t b = next.fetch_add(64);
            if (b >= n) break;
            for (size_t i = b; i < std::min(n, b + 64); ++i) {
                general::Work w;
                const double* a = alpha ? alpha + size_t(L) * i : zeroL.data();
                const double* g = bg ? bg + 3 * i : zero3.data();
                Optimizer::solve(models.data(), p, target + 3 * i, {a}, g, {initial + size_t(N) * i},
                                 {out + size_t(N) * i}, {memory.data()}, opt, w);
                if (counters) {
                    uint32_t* o = counters + 5 * i;
                    o[0] = w.values; o[1] = w.gradients; o[2] = w.iterations; o[3] = w.backtracks; o[4] = w.outer;
                }
            }
        }
    };
    if (threads == 1) work();
    else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(work);
        for (auto& t : pool) t.join();
    }
    return 0;
}

}  // extern "C"
