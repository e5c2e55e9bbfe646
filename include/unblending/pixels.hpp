// C++ buffer API of the B200 unblending path.
//
// Same function names, parameters and exception behaviour as the reference's
// buffer API (unblending/include/unblending/pixels.hpp:13-44 of
// TheDucker1/unblending): RgbImageView / RgbaLayersView, and
// compute_color_unmixing / perform_matte_refinement returning packed
// [layer][row][column][RGBA] doubles. The layer description types are
// self-contained (the reference builds them on Eigen); their fields carry the
// same meaning as LayerInfo / CompOp / BlendMode / GaussianColorModel
// (layer_info.hpp:10-15, comp_op.hpp:14-35, blend_mode.hpp:9-24,
// color_model.hpp:19-59). Invalid arguments throw std::invalid_argument or
// std::length_error; device failures throw unblending::ExecutionError.
#ifndef UNBLENDING_B200_PIXELS_HPP
#define UNBLENDING_B200_PIXELS_HPP

#include <array>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <vector>

namespace unblending {

enum class BlendMode {
    Normal, Multiply, Screen, Overlay, Darken, Lighten, ColorDodge, ColorBurn,
    HardLight, SoftLight, Difference, Exclusion, LinearDodge,
};

// Porter-Duff coefficients: source-over (1,1,1), plus (2,1,1).
struct CompOp {
    int X = 1, Y = 1, Z = 1;
    CompOp(int x = 0, int y = 0, int z = 0) : X(x), Y(y), Z(z) {}
    bool is_source_over() const { return X == 1 && Y == 1 && Z == 1; }
    bool is_plus() const { return X == 2 && Y == 1 && Z == 1; }
    static CompOp SourceOver() { return CompOp(1, 1, 1); }
    static CompOp Plus() { return CompOp(2, 1, 1); }
};

// Gaussian colour model: mean and precision (inverse covariance, row-major).
class GaussianColorModel {
public:
    GaussianColorModel(const std::array<double, 3>& mu, const std::array<double, 9>& sigma_inv)
        : mu_(mu), sigma_inv_(sigma_inv) {}
    const std::array<double, 3>& get_mu() const { return mu_; }
    const std::array<double, 9>& get_sigma_inv() const { return sigma_inv_; }
    double calculate_distance(const std::array<double, 3>& c) const {
        double d[3], cost = 0;
        for (int r = 0; r < 3; ++r) d[r] = c[r] - mu_[r];
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) cost += d[r] * sigma_inv_[3 * r + s] * d[s];
        return cost;
    }

private:
    std::array<double, 3> mu_;
    std::array<double, 9> sigma_inv_;
};
using ColorModelPtr = std::shared_ptr<const GaussianColorModel>;

struct LayerInfo {
    CompOp comp_op;
    BlendMode blend_mode;
    ColorModelPtr color_model;
};

struct ExecutionError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

/// Row-major RGB triples in [0,1]. Size and stride are measured in doubles.
/// A zero row stride uses tightly packed rows (3 * width).
struct RgbImageView {
    const double* data;
    std::size_t size;
    int width, height;
    std::size_t row_stride;
    RgbImageView(const double* data, std::size_t size, int width, int height, std::size_t row_stride = 0)
        : data(data), size(size), width(width), height(height), row_stride(row_stride) {}
};

/// Packed RGBA layer values in [0,1], with size measured in doubles.
/// Layout is [layer][row][column][channel]. Layers are ordered bottom to top.
struct RgbaLayersView {
    const double* data;
    std::size_t size;
};

/// Split RGB pixels into a packed RGBA layer buffer of size 4 * width * height * layer count.
std::vector<double> compute_color_unmixing(RgbImageView image, const std::vector<LayerInfo>& layer_infos,
                                           bool has_opaque_background, int target_concurrency = 0);

/// Refine a packed RGBA buffer from the first pass, using the original RGB pixels.
std::vector<double> perform_matte_refinement(RgbImageView image, RgbaLayersView layers,
                                             const std::vector<LayerInfo>& layer_infos, bool has_opaque_background,
                                             bool force_smooth_background, int target_concurrency = 0);

}  // namespace unblending

#endif
