// C++ buffer API over the C ABI (reference: unblending.cpp:505-636).
#include <unblending/pixels.hpp>

#include <limits>
#include <new>

#include "../../include/unblending.h"

namespace unblending {
namespace {

std::vector<unblending_layer> describe(const std::vector<LayerInfo>& infos) {
    std::vector<unblending_layer> out;
    out.reserve(infos.size());
    for (const auto& info : infos) {
        if (!info.color_model) throw std::invalid_argument("Each layer requires a color model");
        unblending_layer l{};
        l.comp_x = info.comp_op.X; l.comp_y = info.comp_op.Y; l.comp_z = info.comp_op.Z;
        l.blend_mode = static_cast<int32_t>(info.blend_mode);
        for (int r = 0; r < 3; ++r) l.mean[r] = info.color_model->get_mu()[r];
        for (int k = 0; k < 9; ++k) l.precision[k] = info.color_model->get_sigma_inv()[k];
        out.push_back(l);
    }
    return out;
}

// The reference's validate_pixels (unblending.cpp:508-534): argument errors
// are reported with the same exception types before any device work.
std::size_t packed_size(const RgbImageView& image, const std::vector<LayerInfo>& layers) {
    constexpr auto max_int = std::numeric_limits<int>::max();
    if (!image.data || image.width <= 0 || image.height <= 0 || image.width > max_int / image.height)
        throw std::invalid_argument("Invalid RGB image dimensions or data");
    const std::size_t max_doubles = std::vector<double>().max_size();
    if (std::size_t(image.width) > max_doubles / 3) throw std::length_error("RGB row is too large");
    const std::size_t row = 3 * std::size_t(image.width);
    const std::size_t stride = image.row_stride ? image.row_stride : row;
    if (stride < row || image.size < row || std::size_t(image.height - 1) > (image.size - row) / stride)
        throw std::invalid_argument("RGB buffer is too small or has an invalid row stride");
    if (layers.empty()) throw std::invalid_argument("Each layer requires a color model");
    for (const auto& l : layers)
        if (!l.color_model) throw std::invalid_argument("Each layer requires a color model");
    const std::size_t pixels = std::size_t(image.width) * image.height;
    if (layers.size() > std::size_t(max_int) / 4 || pixels > max_doubles / 4 / layers.size())
        throw std::length_error("RGBA layer stack is too large");
    return 4 * pixels * layers.size();
}

void raise(int32_t code) {
    switch (code) {
    case UNBLENDING_OK: return;
    case UNBLENDING_INVALID_ARGUMENT: throw std::invalid_argument("Invalid unblending arguments");
    case UNBLENDING_BUFFER_TOO_SMALL: throw std::length_error("Output buffer too small");
    case UNBLENDING_OUT_OF_MEMORY: throw std::bad_alloc();
    default: throw ExecutionError("CUDA unblending failed");
    }
}

}  // namespace

std::vector<double> compute_color_unmixing(RgbImageView image, const std::vector<LayerInfo>& layer_infos,
                                           bool has_opaque_background, int target_concurrency) {
    const std::size_t size = packed_size(image, layer_infos);
    const auto layers = describe(layer_infos);
    unblending_rgb_view view{image.data, image.size, image.width, image.height, image.row_stride};
    unblending_options options = UNBLENDING_OPTIONS_INIT;
    options.opaque_background = has_opaque_background ? 1 : 0;
    options.target_concurrency = target_concurrency < 0 ? 0 : target_concurrency;
    std::vector<double> out(size);
    raise(unblending_unmix(&view, layers.data(), layers.size(), &options, out.data(), out.size()));
    return out;
}

std::vector<double> perform_matte_refinement(RgbImageView image, RgbaLayersView first,
                                             const std::vector<LayerInfo>& layer_infos, bool has_opaque_background,
                                             bool force_smooth_background, int target_concurrency) {
    const std::size_t size = packed_size(image, layer_infos);
    if (!first.data || first.size != size)
        throw std::invalid_argument("Refinement requires one packed RGBA image per layer");
    if (force_smooth_background && !has_opaque_background)
        throw std::invalid_argument("Smoothing requires an opaque background");
    bool all_plus = true, all_over = true;
    for (const auto& l : layer_infos) { all_plus &= l.comp_op.is_plus(); all_over &= l.comp_op.is_source_over(); }
    if (!all_plus && !all_over) throw std::invalid_argument("Refinement requires an all-Plus or all-SourceOver stack");
    const auto layers = describe(layer_infos);
    unblending_rgb_view view{image.data, image.size, image.width, image.height, image.row_stride};
    unblending_options options = UNBLENDING_OPTIONS_INIT;
    options.opaque_background = has_opaque_background ? 1 : 0;
    options.smooth_background = force_smooth_background ? 1 : 0;
    options.target_concurrency = target_concurrency < 0 ? 0 : target_concurrency;
    std::vector<double> out(size);
    raise(unblending_refine(&view, layers.data(), layers.size(), first.data, first.size, &options, out.data(),
                            out.size()));
    return out;
}

}  // namespace unblending
