// LayerInfos JSON front end of the B200 unblending path.
//
// Same file format and functions as the reference's layer-info I/O
// (LayerInfos.md; unblending/src/unblending_io.cpp:141-170,
// unblending/include/unblending/unblending.hpp:50-54): a JSON array of
// objects, bottom layer first, each with
//   "mode":        one of the thirteen blend-mode names ("Normal" ... "LinearDodge"),
//   "comp_op":     "source-over" (anything else reads as "plus"),
//   "color_model": {"primary_color": [r, g, b],
//                   "color_variance": v (covariance v * I) or nine numbers
//                                     (the 3x3 covariance, column by column)}.
// The colour model keeps the precision, the inverse of the covariance.
// Malformed input throws std::invalid_argument (the reference prints
// "LayerInfo parse error" and exits the process).
#ifndef UNBLENDING_B200_LAYER_INFOS_HPP
#define UNBLENDING_B200_LAYER_INFOS_HPP

#include <string>
#include <vector>

#include <unblending/pixels.hpp>

namespace unblending {

/// Name of a blend mode as the file spells it ("ColorDodge", ...).
std::string retrieve_name(BlendMode mode);
/// Blend mode of a name; throws std::invalid_argument for an unknown name.
BlendMode retrieve_by_name(const std::string& name);

/// Layer infos from JSON text.
std::vector<LayerInfo> parse_layer_infos(const std::string& json_text);
/// Layer infos from a JSON file.
std::vector<LayerInfo> import_layer_infos(const std::string& input_file_path);

/// JSON text of layer infos (keys in sorted order, numbers with 17
/// significant digits; a covariance that is a multiple of the identity is
/// written as one number).
std::string format_layer_infos(const std::vector<LayerInfo>& layer_infos);
/// Writes <output_directory_path>/layer_infos.json.
void export_layer_infos(const std::vector<LayerInfo>& layer_infos, const std::string& output_directory_path);

/// Inverse of a 3x3 matrix (row-major) by its adjugate; throws
/// std::invalid_argument when the matrix is singular.
std::array<double, 9> invert3(const std::array<double, 9>& m);

}  // namespace unblending

#endif
