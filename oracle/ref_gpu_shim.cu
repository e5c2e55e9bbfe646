// Thin C shim over the reference's own CUDA backend, for timing it on the
// same GPU as the B200 path (the "existing GPU kernel" bar).
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile (target refgpu)
// together with the reference's unblending/src/cuda/pixel_pipeline.cu, where
// those sources lie, into oracle/_ref/libunbrefgpu.so; never part of the
// product. Wraps
//   unblending::gpu::solve_cuda   pixel_pipeline.cu:33-107 (gpu_dispatch.hpp:43-45)
// with the planar layouts of gpu_dispatch.cpp:88-108: rgb [3][n]; first pass
// and output [alpha planes L][colour planes 3L].
#include "../gpu_dispatch.hpp"

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

extern "C" {
typedef struct ref_gpu_layer {
    int32_t comp_x, comp_y, comp_z;
    int32_t blend_mode;
    double mean[3];
    double precision[9];
} ref_gpu_layer;

// Returns 0 with `out` written; 2 when the backend rejected its own result
// (a pixel it could not solve: the work ran, nothing is returned); 1 on any
// other error. The message goes to `err` (errlen bytes).
int ref_gpu_solve(int w, int h, const ref_gpu_layer* layers, int L, const double* rgb, const double* first,
                  int opaque, int smooth, double* out, char* err, int errlen) {
    try {
        std::vector<unblending::gpu::Layer> model(L);
        for (int l = 0; l < L; ++l) {
            std::memcpy(model[l].mean, layers[l].mean, sizeof(model[l].mean));
            std::memcpy(model[l].precision, layers[l].precision, sizeof(model[l].precision));
            model[l].x = layers[l].comp_x; model[l].y = layers[l].comp_y; model[l].z = layers[l].comp_z;
            model[l].mode = layers[l].blend_mode;
        }
        const size_t n = size_t(w) * h;
        std::vector<double> planes(rgb, rgb + 3 * n);
        std::vector<double> initial;
        if (first) initial.assign(first, first + 4 * size_t(L) * n);
        unblending::gpu::Options options;
        options.opaque = opaque != 0;
        options.smooth = smooth != 0;
        const auto solved = unblending::gpu::solve_cuda(w, h, model, planes, first ? &initial : nullptr, options);
        std::memcpy(out, solved.data(), solved.size() * sizeof(double));
        return 0;
    } catch (const std::runtime_error& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return 2;
    } catch (const std::exception& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return 1;
    }
}
}
