// LayerInfos JSON front end (reference: unblending/src/unblending_io.cpp:12-170,
// LayerInfos.md): a small JSON reader and writer of the layer-info file and
// its C ABI entry points. Host code only.
#include <unblending/layer_infos.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <memory>
#include <sstream>

#include "../../include/unblending_b200.h"

namespace unblending {
namespace {

// ------------------------------------------------------------- JSON value --
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> items;
    std::map<std::string, Json> fields;

    const Json* get(const std::string& key) const {
        if (kind != Object) return nullptr;
        auto it = fields.find(key);
        return it == fields.end() ? nullptr : &it->second;
    }
};

[[noreturn]] void parse_error(const char* what) {
    throw std::invalid_argument(std::string("LayerInfo parse error: ") + what);
}

// Recursive-descent reader of RFC 8259 JSON (depth-limited).
class Reader {
public:
    explicit Reader(const std::string& text) : s_(text) {}

    Json document() {
        Json v = value(0);
        skip();
        if (p_ != s_.size()) parse_error("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    std::size_t p_ = 0;

    void skip() {
        while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) ++p_;
    }
    bool eat(char c) {
        skip();
        if (p_ < s_.size() && s_[p_] == c) { ++p_; return true; }
        return false;
    }
    void expect(char c) { if (!eat(c)) parse_error("unexpected character"); }
    bool literal(const char* word) {
        const std::size_t n = std::strlen(word);
        if (s_.compare(p_, n, word) == 0) { p_ += n; return true; }
        return false;
    }

    Json value(int depth) {
        if (depth > 64) parse_error("nesting too deep");
        skip();
        if (p_ >= s_.size()) parse_error("unexpected end");
        Json v;
        const char c = s_[p_];
        if (c == '{') {
            ++p_;
            v.kind = Json::Object;
            if (eat('}')) return v;
            do {
                skip();
                if (p_ >= s_.size() || s_[p_] != '"') parse_error("expected a key");
                std::string key = string();
                expect(':');
                v.fields[key] = value(depth + 1);
            } while (eat(','));
            expect('}');
        } else if (c == '[') {
            ++p_;
            v.kind = Json::Array;
            if (eat(']')) return v;
            do v.items.push_back(value(depth + 1));
            while (eat(','));
            expect(']');
        } else if (c == '"') {
            v.kind = Json::String;
            v.str = string();
        } else if (literal("true")) {
            v.kind = Json::Bool; v.b = true;
        } else if (literal("false")) {
            v.kind = Json::Bool; v.b = false;
        } else if (literal("null")) {
            v.kind = Json::Null;
        } else {
            v.kind = Json::Number;
            v.num = number();
        }
        return v;
    }

    // A number token by the JSON grammar, converted by strtod (correctly
    // rounded).
    double number() {
        const std::size_t start = p_;
        auto digits = [&]() {
            const std::size_t d = p_;
            while (p_ < s_.size() && s_[p_] >= '0' && s_[p_] <= '9') ++p_;
            return p_ > d;
        };
        if (p_ < s_.size() && s_[p_] == '-') ++p_;
        if (p_ < s_.size() && s_[p_] == '0') ++p_;
        else if (!digits()) parse_error("invalid number");
        if (p_ < s_.size() && s_[p_] == '.') { ++p_; if (!digits()) parse_error("invalid number"); }
        if (p_ < s_.size() && (s_[p_] == 'e' || s_[p_] == 'E')) {
            ++p_;
            if (p_ < s_.size() && (s_[p_] == '+' || s_[p_] == '-')) ++p_;
            if (!digits()) parse_error("invalid number");
        }
        const std::string token = s_.substr(start, p_ - start);
        return std::strtod(token.c_str(), nullptr);
    }

    static void utf8(std::string& out, unsigned cp) {
        if (cp < 0x80) out += char(cp);
        else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18)); out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F));
        }
    }
    unsigned hex4() {
        if (p_ + 4 > s_.size()) parse_error("invalid escape");
        unsigned v = 0;
        for (int k = 0; k < 4; ++k) {
            const char h = s_[p_++];
            v <<= 4;
            if (h >= '0' && h <= '9') v |= unsigned(h - '0');
            else if (h >= 'a' && h <= 'f') v |= unsigned(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F') v |= unsigned(h - 'A' + 10);
            else parse_error("invalid escape");
        }
        return v;
    }
    std::string string() {
        ++p_;   // opening quote
        std::string out;
        for (;;) {
            if (p_ >= s_.size()) parse_error("unterminated string");
            const char c = s_[p_++];
            if (c == '"') return out;
            if (static_cast<unsigned char>(c) < 0x20) parse_error("control character in string");
            if (c != '\\') { out += c; continue; }
            if (p_ >= s_.size()) parse_error("invalid escape");
            const char e = s_[p_++];
            switch (e) {
            case '"': out += '"'; break;
            case '\\': out += '\\'; break;
            case '/': out += '/'; break;
            case 'b': out += '\b'; break;
            case 'f': out += '\f'; break;
            case 'n': out += '\n'; break;
            case 'r': out += '\r'; break;
            case 't': out += '\t'; break;
            case 'u': {
                unsigned cp = hex4();
                if (cp >= 0xD800 && cp < 0xDC00 && p_ + 6 <= s_.size() && s_[p_] == '\\' && s_[p_ + 1] == 'u') {
                    p_ += 2;
                    const unsigned lo = hex4();
                    if (lo < 0xDC00 || lo >= 0xE000) parse_error("invalid surrogate pair");
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                utf8(out, cp);
                break;
            }
            default: parse_error("invalid escape");
            }
        }
    }
};

const char* const kModeNames[] = {"Normal",    "Multiply",   "Screen",     "Overlay", "Darken",
                                  "Lighten",   "ColorDodge", "ColorBurn",  "HardLight", "SoftLight",
                                  "Difference", "Exclusion", "LinearDodge"};

double number_of(const Json& v) {
    if (v.kind != Json::Number) parse_error("expected a number");
    return v.num;
}

// Covariance from "color_variance": v -> v I; nine numbers -> the matrix,
// element (row, col) at index col * 3 + row (unblending_io.cpp:42-53,70-85).
std::array<double, 9> covariance_of(const Json* v) {
    if (!v) parse_error("missing color_variance");
    std::array<double, 9> c{};
    if (v->kind == Json::Number) {
        c[0] = c[4] = c[8] = v->num;
    } else if (v->kind == Json::Array && v->items.size() == 9) {
        for (int col = 0; col < 3; ++col)
            for (int row = 0; row < 3; ++row) c[3 * row + col] = number_of(v->items[col * 3 + row]);
    } else {
        parse_error("color_variance must be a number or nine numbers");
    }
    return c;
}

LayerInfo layer_of(const Json& j) {
    if (j.kind != Json::Object) parse_error("a layer info must be an object");
    const Json* mode = j.get("mode");
    if (!mode || mode->kind != Json::String) parse_error("missing mode");
    const Json* op = j.get("comp_op");
    // Anything but "source-over" reads as plus (unblending_io.cpp:159).
    const bool source_over = op && op->kind == Json::String && op->str == "source-over";
    const Json* model = j.get("color_model");
    if (!model || model->kind != Json::Object) parse_error("missing color_model");
    const Json* mu = model->get("primary_color");
    if (!mu || mu->kind != Json::Array || mu->items.size() < 3) parse_error("primary_color must be three numbers");
    std::array<double, 3> mean{number_of(mu->items[0]), number_of(mu->items[1]), number_of(mu->items[2])};
    const std::array<double, 9> precision = invert3(covariance_of(model->get("color_variance")));
    LayerInfo info{source_over ? CompOp::SourceOver() : CompOp::Plus(), retrieve_by_name(mode->str),
                   std::make_shared<GaussianColorModel>(mean, precision)};
    return info;
}

void put_number(std::string& out, double v) {
    if (!std::isfinite(v)) { out += "null"; return; }
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    out += buf;
}

// Whether c / c00 is the identity to 1e-12 (the reference writes such a
// covariance as the single number c00, unblending_io.cpp:27-40).
bool scaled_identity(const std::array<double, 9>& c) {
    if (c[0] == 0.0) return false;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            const double v = c[3 * r + k] / c[0];
            if (r == k ? std::fabs(v - 1.0) > 1e-12 : std::fabs(v) > 1e-12) return false;
        }
    return true;
}

std::vector<LayerInfo> from_layers(const unblending_layer* layers, size_t count) {
    std::vector<LayerInfo> out;
    for (size_t i = 0; i < count; ++i) {
        const unblending_layer& l = layers[i];
        if (l.blend_mode < 0 || l.blend_mode > 12) throw std::invalid_argument("blend mode out of range");
        std::array<double, 3> mean{l.mean[0], l.mean[1], l.mean[2]};
        std::array<double, 9> prec{};
        for (int k = 0; k < 9; ++k) prec[k] = l.precision[k];
        out.push_back(LayerInfo{CompOp(l.comp_x, l.comp_y, l.comp_z), static_cast<BlendMode>(l.blend_mode),
                                std::make_shared<GaussianColorModel>(mean, prec)});
    }
    return out;
}

template <class F> int32_t guarded_call(F&& f) {
    try {
        return f();
    } catch (const std::invalid_argument&) {
        return UNBLENDING_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        return UNBLENDING_OUT_OF_MEMORY;
    } catch (...) {
        return UNBLENDING_INVALID_ARGUMENT;
    }
}

}  // namespace

std::string retrieve_name(BlendMode mode) {
    const int m = static_cast<int>(mode);
    if (m < 0 || m > 12) throw std::invalid_argument("blend mode out of range");
    return kModeNames[m];
}

BlendMode retrieve_by_name(const std::string& name) {
    for (int m = 0; m < 13; ++m)
        if (name == kModeNames[m]) return static_cast<BlendMode>(m);
    throw std::invalid_argument("LayerInfo parse error: unknown blend mode \"" + name + "\"");
}

// Adjugate inverse: cofactors C(i, j) = m(i1, j1) m(i2, j2) - m(i1, j2) m(i2, j1)
// with i1 = i+1, i2 = i+2, j1 = j+1, j2 = j+2 (mod 3); the determinant from
// the first column, det = C(0,0) m(0,0) + C(1,0) m(1,0) + C(2,0) m(2,0);
// inverse(i, j) = C(j, i) / det, formed as C(j, i) * (1 / det).
std::array<double, 9> invert3(const std::array<double, 9>& m) {
    auto at = [&](int r, int c) { return m[3 * r + c]; };
    auto cof = [&](int i, int j) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        return at(i1, j1) * at(i2, j2) - at(i1, j2) * at(i2, j1);
    };
    const double det = cof(0, 0) * at(0, 0) + cof(1, 0) * at(1, 0) + cof(2, 0) * at(2, 0);
    if (!(det != 0.0) || !std::isfinite(det)) throw std::invalid_argument("LayerInfo parse error: singular covariance");
    const double inv = 1.0 / det;
    std::array<double, 9> out{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[3 * i + j] = cof(j, i) * inv;
    return out;
}

std::vector<LayerInfo> parse_layer_infos(const std::string& json_text) {
    const Json doc = Reader(json_text).document();
    if (doc.kind != Json::Array) parse_error("the file must hold an array of layer infos");
    std::vector<LayerInfo> out;
    out.reserve(doc.items.size());
    for (const Json& j : doc.items) out.push_back(layer_of(j));
    return out;
}

std::vector<LayerInfo> import_layer_infos(const std::string& input_file_path) {
    std::ifstream in(input_file_path, std::ios::binary);
    if (!in) throw std::invalid_argument("cannot open " + input_file_path);
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    return parse_layer_infos(text);
}

std::string format_layer_infos(const std::vector<LayerInfo>& layer_infos) {
    std::string out = "[";
    for (std::size_t i = 0; i < layer_infos.size(); ++i) {
        const LayerInfo& info = layer_infos[i];
        if (!info.color_model) throw std::invalid_argument("Each layer requires a color model");
        if (i) out += ", ";
        const std::array<double, 9> cov = invert3(info.color_model->get_sigma_inv());
        out += "{\"color_model\": {\"color_variance\": ";
        if (scaled_identity(cov)) {
            put_number(out, cov[0]);
        } else {
            out += "[";
            for (int k = 0; k < 9; ++k) {   // row by row (unblending_io.cpp:14-25)
                if (k) out += ", ";
                put_number(out, cov[k]);
            }
            out += "]";
        }
        out += ", \"primary_color\": [";
        for (int r = 0; r < 3; ++r) {
            if (r) out += ", ";
            put_number(out, info.color_model->get_mu()[r]);
        }
        out += "]}, \"comp_op\": \"";
        out += info.comp_op.is_plus() ? "plus" : (info.comp_op.is_source_over() ? "source-over" : "unknown");
        out += "\", \"mode\": \"" + retrieve_name(info.blend_mode) + "\"}";
    }
    out += "]";
    return out;
}

void export_layer_infos(const std::vector<LayerInfo>& layer_infos, const std::string& output_directory_path) {
    const std::string text = format_layer_infos(layer_infos);
    const std::string path = output_directory_path + "/layer_infos.json";
    std::ofstream out(path, std::ios::binary);
    if (!out) throw std::invalid_argument("cannot write " + path);
    out << text;
    if (!out) throw std::invalid_argument("cannot write " + path);
}

}  // namespace unblending

extern "C" {

int32_t unblending_parse_layer_infos(const char* json, unblending_layer* layers, size_t capacity, size_t* count) {
    if (!json || !count || (capacity && !layers)) return UNBLENDING_INVALID_ARGUMENT;
    return unblending::guarded_call([&]() -> int32_t {
        const auto infos = unblending::parse_layer_infos(json);
        *count = infos.size();
        if (infos.size() > capacity) return UNBLENDING_BUFFER_TOO_SMALL;
        for (size_t i = 0; i < infos.size(); ++i) {
            unblending_layer l{};
            l.comp_x = infos[i].comp_op.X; l.comp_y = infos[i].comp_op.Y; l.comp_z = infos[i].comp_op.Z;
            l.blend_mode = static_cast<int32_t>(infos[i].blend_mode);
            for (int r = 0; r < 3; ++r) l.mean[r] = infos[i].color_model->get_mu()[r];
            for (int k = 0; k < 9; ++k) l.precision[k] = infos[i].color_model->get_sigma_inv()[k];
            layers[i] = l;
        }
        return UNBLENDING_OK;
    });
}

int32_t unblending_format_layer_infos(const unblending_layer* layers, size_t layer_count, char* text,
                                      size_t capacity, size_t* length) {
    if ((layer_count && !layers) || !length || (capacity && !text)) return UNBLENDING_INVALID_ARGUMENT;
    return unblending::guarded_call([&]() -> int32_t {
        const std::string s = unblending::format_layer_infos(unblending::from_layers(layers, layer_count));
        *length = s.size();
        if (s.size() + 1 > capacity) return UNBLENDING_BUFFER_TOO_SMALL;
        std::memcpy(text, s.c_str(), s.size() + 1);
        return UNBLENDING_OK;
    });
}

}  // extern "C"
