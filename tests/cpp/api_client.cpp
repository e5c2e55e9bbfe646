// A C++ host of the library's C++ API, the way the reference's own callers
// use theirs (unblending-cli/main.cpp:52-67): layer infos from a JSON file,
// compute_color_unmixing, perform_matte_refinement, export_layer_infos.
//
//   api_client host <layer_infos.json> <out_dir>
//       argument rules and the layer-info file, no device work; prints
//       "ok <layer count>" on success
//   api_client solve <layer_infos.json> <image.f64> <width> <height> <first.f64> <final.f64>
//       both passes on a raw (height, width, 3) float64 image
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <unblending/layer_infos.hpp>
#include <unblending/pixels.hpp>

using namespace unblending;

namespace {

int failures = 0;

template <class E, class F> void expect_throw(const char* what, F&& f) {
    try {
        f();
    } catch (const E&) {
        return;
    } catch (const std::exception& e) {
        std::printf("FAIL %s: wrong exception %s\n", what, e.what());
        ++failures;
        return;
    }
    std::printf("FAIL %s: no exception\n", what);
    ++failures;
}

std::vector<double> read_doubles(const char* path, std::size_t n) {
    std::vector<double> v(n);
    std::ifstream in(path, std::ios::binary);
    in.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(double)));
    if (!in) throw std::runtime_error(std::string("cannot read ") + path);
    return v;
}

void write_doubles(const char* path, const std::vector<double>& v) {
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
}

int host(const char* json_path, const char* out_dir) {
    const std::vector<LayerInfo> infos = import_layer_infos(json_path);
    export_layer_infos(infos, out_dir);
    const std::vector<LayerInfo> back = import_layer_infos(std::string(out_dir) + "/layer_infos.json");
    if (back.size() != infos.size()) { std::printf("FAIL round trip size\n"); ++failures; }
    for (std::size_t i = 0; i < infos.size() && i < back.size(); ++i)
        if (back[i].blend_mode != infos[i].blend_mode || back[i].color_model->get_mu() != infos[i].color_model->get_mu()) {
            std::printf("FAIL round trip layer %zu\n", i);
            ++failures;
        }
    if (retrieve_name(BlendMode::ColorDodge) != "ColorDodge" || retrieve_by_name("SoftLight") != BlendMode::SoftLight) {
        std::printf("FAIL mode names\n");
        ++failures;
    }
    expect_throw<std::invalid_argument>("unknown mode", [] { retrieve_by_name("Vivid"); });
    expect_throw<std::invalid_argument>("malformed file", [] { parse_layer_infos("[{\"mode\": 1}]"); });
    expect_throw<std::invalid_argument>("missing file", [] { import_layer_infos("/nonexistent/layer_infos.json"); });

    // Argument rules of the buffer API (the reference's validate_pixels,
    // unblending.cpp:508-534,597-604): thrown before any device work.
    std::vector<double> rgb(3 * 6 * 5, 0.5);
    expect_throw<std::invalid_argument>("zero width", [&] {
        compute_color_unmixing(RgbImageView(rgb.data(), rgb.size(), 0, 5), infos, true);
    });
    expect_throw<std::invalid_argument>("short buffer", [&] {
        compute_color_unmixing(RgbImageView(rgb.data(), rgb.size() - 1, 6, 5), infos, true);
    });
    expect_throw<std::invalid_argument>("stride below the row", [&] {
        compute_color_unmixing(RgbImageView(rgb.data(), rgb.size(), 6, 5, 17), infos, true);
    });
    expect_throw<std::invalid_argument>("no layers", [&] {
        compute_color_unmixing(RgbImageView(rgb.data(), rgb.size(), 6, 5), {}, true);
    });
    std::vector<double> first(4 * 6 * 5 * infos.size(), 0.0);
    expect_throw<std::invalid_argument>("smooth without opaque", [&] {
        perform_matte_refinement(RgbImageView(rgb.data(), rgb.size(), 6, 5), RgbaLayersView{first.data(), first.size()},
                                 infos, false, true);
    });
    expect_throw<std::invalid_argument>("first pass size", [&] {
        perform_matte_refinement(RgbImageView(rgb.data(), rgb.size(), 6, 5),
                                 RgbaLayersView{first.data(), first.size() - 4}, infos, true, false);
    });
    std::vector<LayerInfo> mixed = infos;
    mixed.back().comp_op = CompOp::Plus();
    expect_throw<std::invalid_argument>("mixed comp ops", [&] {
        perform_matte_refinement(RgbImageView(rgb.data(), rgb.size(), 6, 5), RgbaLayersView{first.data(), first.size()},
                                 mixed, true, false);
    });
    if (failures) return 1;
    std::printf("ok %zu\n", infos.size());
    return 0;
}

int solve(const char* json_path, const char* image_path, int width, int height, const char* first_path,
          const char* final_path) {
    const std::vector<LayerInfo> infos = import_layer_infos(json_path);
    const std::vector<double> rgb = read_doubles(image_path, std::size_t(3) * width * height);
    const RgbImageView view(rgb.data(), rgb.size(), width, height);
    const std::vector<double> first = compute_color_unmixing(view, infos, true);
    const std::vector<double> final_layers =
        perform_matte_refinement(view, RgbaLayersView{first.data(), first.size()}, infos, true, true);
    write_doubles(first_path, first);
    write_doubles(final_path, final_layers);
    std::printf("ok %zu\n", final_layers.size());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc == 4 && std::strcmp(argv[1], "host") == 0) return host(argv[2], argv[3]);
        if (argc == 8 && std::strcmp(argv[1], "solve") == 0)
            return solve(argv[2], argv[3], std::atoi(argv[4]), std::atoi(argv[5]), argv[6], argv[7]);
    } catch (const std::exception& e) {
        std::printf("FAIL %s\n", e.what());
        return 1;
    }
    std::printf("usage: api_client host <json> <dir> | solve <json> <image> <w> <h> <first> <final>\n");
    return 2;
}
