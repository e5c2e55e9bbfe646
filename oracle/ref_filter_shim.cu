// Thin C shim over the reference's CPU twin of its streaming guided filter.
//
// TEST INFRASTRUCTURE ONLY. Compiled as host code by nvcc (the header pulls
// in CUB) by oracle/Makefile (target ref) against the reference sources where they lie;
// linked into oracle/_ref/libunbref.so. Wraps
//   general::StreamingFilterCPU<double>   refinement/streaming_guided_filter.cuh:92-112
// which produces the clipped, normalized refinement targets.
#include "refinement/streaming_guided_filter.cuh"

#include <cstdint>

extern "C" {
typedef struct ref_layer_f {
    int32_t comp_x, comp_y, comp_z;
    int32_t blend_mode;
    double mean[3];
    double precision[9];
} ref_layer_f;

// rgb: planar 3*n; first: planar 4L*n; targets: planar (L+3)*n; status: n.
int ref_refine_targets(const double* rgb, const double* first, const ref_layer_f* layers, int L, int w, int h,
                       int opaque, int smooth, int radius, int threads, double* targets, int32_t* status) {
    try {
        std::vector<general::Layer> models(L);
        for (int l = 0; l < L; ++l) {
            models[l].X = layers[l].comp_x; models[l].Y = layers[l].comp_y; models[l].Z = layers[l].comp_z;
            models[l].mode = layers[l].blend_mode;
        }
        twostage::Pool pool(threads > 0 ? threads : 1);
        general::StreamingFilterCPU<double> filter(w, h, L, opaque != 0, smooth != 0, models.data(), pool);
        filter.run(rgb, first, targets, radius);
        const auto& s = filter.statuses();
        for (size_t i = 0; i < s.size(); ++i) status[i] = s[i];
        return 0;
    } catch (...) {
        return 1;
    }
}
}
