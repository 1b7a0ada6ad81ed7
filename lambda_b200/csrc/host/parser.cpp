// .lrd scene-language and .obj mesh reader.
//
// Behaviour follows the reference parser (src/core/parser.h) command for
// command, including its error texts ("file:line: message") and quirks, because
// this is a drop-in for it: the same file must give the same scene or the same
// error. Token extraction uses std::istringstream just as the reference does, so
// numbers, names and stream positions behave the same way (for example "0.5abc"
// reads as 0.5 where the reference calls std::stof, and `Texture <n> spectrum
// scalar <tex>` reads the texture name twice, parser.h:141).
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <iterator>
#include <limits>
#include <string_view>
#include <charconv>
#include <map>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "hmath.h"
#include "scene.h"

namespace lambda_host {

namespace {

using Complex = std::complex<double>;

std::string strerror_lower() {
    std::string e = std::strerror(errno);
    if (!e.empty()) e[0] = char(std::tolower(e[0]));
    return e;
}

// parser.h:384-401: drop the comment, pad brackets, commas become spaces.
std::string preprocess(const std::string &line) {
    const size_t hash = line.find('#');
    const std::string body = hash == std::string::npos ? line : line.substr(0, hash);
    std::string out;
    out.reserve(body.size() + 16);
    for (char ch : body) {
        if (ch == '(' || ch == ')' || ch == '[' || ch == ']') {
            out += ' ';
            out += ch;
            out += ' ';
        } else if (ch == ',') {
            out += ' ';
        } else {
            out += ch;
        }
    }
    return out;
}

float to_float(const std::string &s, size_t *idx = nullptr) { return std::stof(s, idx); }

// Scalar and spectrum texture statistics (texture.h:30-60, :112-141).
float scalar_texture_min(const HostScene &s, int t) {
    const lambda_scalar_texture &x = s.scalar_textures[t];
    return x.p[0];
}
float scalar_texture_max(const HostScene &s, int t) {
    const lambda_scalar_texture &x = s.scalar_textures[t];
    return x.type == LAMBDA_SCALAR_CONSTANT ? x.p[0] : x.p[1];
}
float scalar_texture_average(const HostScene &s, int t) {
    const lambda_scalar_texture &x = s.scalar_textures[t];
    return x.type == LAMBDA_SCALAR_CONSTANT ? x.p[0] : (x.p[0] + x.p[1]) / 2;
}

class LrdReader {
  public:
    LrdReader(const std::string &file, HostScene &scene) : file_(file), s_(scene) {}

    void run();

    const BuildAccel *accel_ = nullptr;  // build steps that run on a GPU (parse_lrd)

  private:
    const std::string &file_;
    HostScene &s_;
    int line_ = 0;
    std::vector<int> group_offsets_;
    std::map<std::string, int> groups_, materials_, scalar_textures_, spectrum_textures_;

    SceneError error(const std::string &msg) const {
        return SceneError(LAMBDA_ERR_PARSE, file_ + ":" + std::to_string(line_) + ": " + msg);
    }

    template <typename T>
    T value(std::istringstream &ss, const std::string &what) {
        T v;
        if (!(ss >> v)) throw error("'" + what + "' is missing or invalid");
        return v;
    }

    V3 vector(std::istringstream &ss, const std::string &what) {
        const std::string msg = "'" + what + "' is missing or invalid";
        std::string tok;
        if (!(ss >> tok) || tok != "(") throw error(msg);
        V3 v = v3(0, 0, 0);
        for (int k = 0; k < 3; k++)
            if (!(ss >> v[k])) throw error(msg);
        if (!(ss >> tok) || tok != ")") throw error(msg);
        return v;
    }

    // parser.h:414-453
    Complex complex_token(std::string tok, const std::string &msg) {
        if (tok == "i") return Complex(0, 1);
        if (tok == "-i") return Complex(0, -1);
        double re = 0, im = 0;
        try {
            size_t idx = 0;
            re = to_float(tok, &idx);
            if (idx < tok.size()) {
                tok = tok.substr(idx);
                if (tok.back() == 'i') tok.pop_back();
                else throw error(msg);
                if (tok == "+") im = 1;
                else if (tok == "-") im = -1;
                else if (tok.empty()) {
                    im = re;
                    re = 0;
                } else {
                    im = to_float(tok);
                }
            }
        } catch (const std::exception &) {
            throw error(msg);
        }
        return Complex(re, im);
    }

    void push_float_spectrum(const std::vector<float> &bins) { s_.spectra.insert(s_.spectra.end(), bins.begin(), bins.end()); }
    void push_complex_spectrum(const std::vector<Complex> &bins) {
        for (const Complex &c : bins) {
            s_.complex_spectra.push_back(c.real());
            s_.complex_spectra.push_back(c.imag());
        }
    }

    // parser.h:473-561: a bare value, or "( lambda value ... )" linearly
    // interpolated onto the 1 nm grid and held flat outside the samples.
    template <typename T>
    int spectrum(std::istringstream &ss, const std::string &what) {
        const std::string msg = "'" + what + "' is missing or invalid";
        std::string tok;
        if (!(ss >> tok)) throw error(msg);
        if (tok != "(") {
            if constexpr (std::is_same_v<T, float>) {
                float v;
                try {
                    v = to_float(tok);
                } catch (const std::exception &) {
                    throw error(msg);
                }
                push_float_spectrum(std::vector<float>(kBins, v));
                return s_.num_spectra() - 1;
            } else {
                Complex c = complex_token(tok, msg);
                push_complex_spectrum(std::vector<Complex>(kBins, c));
                return s_.num_complex_spectra() - 1;
            }
        }
        std::map<double, T> samples;
        while (ss >> tok) {
            if (tok == ")") break;
            double lambda;
            try {
                lambda = std::stod(tok);
            } catch (const std::exception &) {
                throw error(msg);
            }
            if (lambda < LAMBDA_CIE_LAMBDA_MIN || lambda > LAMBDA_CIE_LAMBDA_MAX) throw error(msg);
            if (!(ss >> tok)) throw error(msg);
            if constexpr (std::is_same_v<T, float>) {
                try {
                    samples[lambda] = to_float(tok);
                } catch (const std::exception &) {
                    throw error(msg);
                }
            } else {
                samples[lambda] = complex_token(tok, msg);
            }
        }
        if (tok != ")" || samples.empty()) throw error(msg);

        std::vector<T> bins(kBins);
        auto it = samples.begin();
        const double lo = samples.begin()->first;
        const double hi = samples.rbegin()->first;
        for (int i = 0; i < kBins; i++) {
            if (i <= lo - LAMBDA_CIE_LAMBDA_MIN || samples.size() == 1) {
                bins[i] = samples[lo];
            } else if (i >= hi - LAMBDA_CIE_LAMBDA_MIN) {
                bins[i] = samples[hi];
            } else {
                const double lambda = i + LAMBDA_CIE_LAMBDA_MIN;
                while (std::next(it) != samples.end() && std::next(it)->first < lambda) ++it;
                const double a = it->first;
                const double b = std::next(it)->first;
                bins[i] = T((b - lambda) / (b - a) * samples[a] + (lambda - a) / (b - a) * samples[b]);
            }
        }
        if constexpr (std::is_same_v<T, float>) {
            push_float_spectrum(bins);
            return s_.num_spectra() - 1;
        } else {
            push_complex_spectrum(bins);
            return s_.num_complex_spectra() - 1;
        }
    }

    // parser.h:594-612
    std::vector<int> complex_spectrum_array(std::istringstream &ss, const std::string &what) {
        const std::string msg = "'" + what + "' is missing or invalid";
        std::string tok;
        if (!(ss >> tok) || tok != "[") throw error(msg);
        std::streampos pos = ss.tellg();
        std::vector<int> out;
        while (ss >> tok) {
            if (tok == "]") return out;
            ss.seekg(pos);
            out.push_back(spectrum<Complex>(ss, what));
            pos = ss.tellg();
        }
        throw error(msg);
    }

    // parser.h:563-592
    std::vector<std::string> name_array(std::istringstream &ss, const std::string &what) {
        const std::string msg = "'" + what + "' is missing or invalid";
        std::string tok;
        if (!(ss >> tok) || tok != "[") throw error(msg);
        std::vector<std::string> out;
        while (ss >> tok) {
            if (tok == "]") return out;
            out.push_back(tok);
        }
        throw error(msg);
    }

    int push_spectrum_texture(int32_t type, int32_t v1, int32_t v2 = 0, float scale = 0) {
        lambda_spectrum_texture t{};
        t.type = type;
        t.value1 = v1;
        t.value2 = v2;
        t.scale = scale;
        s_.spectrum_textures.push_back(t);
        return int(s_.spectrum_textures.size()) - 1;
    }

    int push_scalar_texture(int32_t type, float a, float b = 0, float c = 0) {
        lambda_scalar_texture t{};
        t.type = type;
        t.p[0] = a;
        t.p[1] = b;
        t.p[2] = c;
        s_.scalar_textures.push_back(t);
        return int(s_.scalar_textures.size()) - 1;
    }

    // parser.h:614-637: an inline spectrum, else a spectrum texture name, else a
    // scalar texture name wrapped in a new spectrum texture.
    int spectrum_texture(std::istringstream &ss, const std::string &what) {
        std::streampos pos = ss.tellg();
        try {
            return push_spectrum_texture(LAMBDA_SPECTRUM_CONSTANT, spectrum<float>(ss, what));
        } catch (const std::exception &) {
            ss.seekg(pos);
            const std::string name = value<std::string>(ss, what);
            auto a = spectrum_textures_.find(name);
            if (a != spectrum_textures_.end()) return a->second;
            auto b = scalar_textures_.find(name);
            if (b != scalar_textures_.end()) return push_spectrum_texture(LAMBDA_SPECTRUM_SCALAR, b->second);
            throw error("'" + what + "' is not defined");
        }
    }

    void cmd_render(std::istringstream &ss);
    void cmd_texture(std::istringstream &ss);
    void cmd_material(std::istringstream &ss);
    void cmd_object(std::istringstream &ss);
    void cmd_instance(std::istringstream &ss);
    void cmd_background(std::istringstream &ss);
    void cmd_camera(std::istringstream &ss);
};

void read_obj(const std::string &path, std::vector<lambda_object> &objects, int material);

lambda_object make_tri(int material, const V3 &c, const V3 &h, const V3 &v, const V3 &n0, const V3 &n1, const V3 &n2,
                       float u0, float u1, float u2, float v0, float v1, float v2) {
    lambda_object o{};
    o.type = LAMBDA_OBJECT_TRI;
    o.material = material;
    const V3 n = cross(h, v);
    V3 a = n0, b = n1, d = n2;
    if (length(n0) < kEpsilon) {  // object.h:53-57
        a = normalize(n);
        b = a;
        d = a;
    }
    const V3 parts[7] = {c, h, v, n, a, b, d};
    for (int k = 0; k < 7; k++)
        for (int j = 0; j < 3; j++) o.g[3 * k + j] = parts[k][j];
    o.g[21] = u0;
    o.g[22] = u1;
    o.g[23] = u2;
    o.g[24] = v0;
    o.g[25] = v1;
    o.g[26] = v2;
    return o;
}

void LrdReader::cmd_render(std::istringstream &ss) {
    const int width = value<int>(ss, "width");
    if (width <= 0) throw error("'width' must be positive, got " + std::to_string(width));
    const int height = value<int>(ss, "height");
    if (height <= 0) throw error("'height' must be positive, got " + std::to_string(height));
    const int depth = value<int>(ss, "depth");
    if (depth < 0) throw error("'depth' must be non-negative, got " + std::to_string(depth));
    const int samples = value<int>(ss, "samples");
    if (samples < 1) throw error("'samples' must be at least 1, got " + std::to_string(samples));
    const int root = int(std::sqrt(samples));
    if (root * root != samples) throw error("'samples' must be a perfect square, got " + std::to_string(samples));
    const float lmin = value<float>(ss, "lambdaMin");
    if (lmin < 0) throw error("'lambdaMin' must be non-negative, got " + std::to_string(lmin));
    if (lmin < LAMBDA_CIE_LAMBDA_MIN)
        throw error("'lambdaMin' must be at least " + std::to_string(LAMBDA_CIE_LAMBDA_MIN) + ", got " + std::to_string(lmin));
    const float lmax = value<float>(ss, "lambdaMax");
    if (lmax < 0) throw error("'lambdaMax' must be non-negative, got " + std::to_string(lmax));
    if (lmax > LAMBDA_CIE_LAMBDA_MAX)
        throw error("'lambdaMax' must be at most " + std::to_string(LAMBDA_CIE_LAMBDA_MAX) + ", got " + std::to_string(lmax));
    if (lmin >= lmax)
        throw error("'lambdaMin' must be at most 'lambdaMax', got " + std::to_string(lmin) + " and " + std::to_string(lmax));
    // `renderer = Renderer(...)` (parser.h:101) also resets the camera.
    lambda_render_settings &r = s_.settings;
    r = lambda_render_settings{};
    r.width = width;
    r.height = height;
    r.depth = depth;
    r.samples = samples;
    r.sqrt_samples = root;
    r.lambda_min = lmin;
    r.lambda_max = lmax;
}

void LrdReader::cmd_texture(std::istringstream &ss) {
    const std::string name = value<std::string>(ss, "name");
    const std::string type = value<std::string>(ss, "type");
    const std::string subtype = value<std::string>(ss, "subtype");
    if (scalar_textures_.count(name) || spectrum_textures_.count(name)) throw error("'name' is already defined");
    if (type == "scalar") {
        if (subtype == "constant") {
            push_scalar_texture(LAMBDA_SCALAR_CONSTANT, value<float>(ss, "value"));
        } else if (subtype == "perlin" || subtype == "worley") {
            const float lo = value<float>(ss, "min");
            const float hi = value<float>(ss, "max");
            const float freq = value<float>(ss, "frequency");
            if (lo > hi) throw error("'min' must be at most 'max', got " + std::to_string(lo) + " and " + std::to_string(hi));
            push_scalar_texture(subtype == "perlin" ? LAMBDA_SCALAR_PERLIN : LAMBDA_SCALAR_WORLEY, lo, hi, freq);
        } else {
            throw error("'subtype' must be \"constant\", \"perlin\", or \"worley\"");
        }
        scalar_textures_[name] = int(s_.scalar_textures.size()) - 1;
    } else if (type == "spectrum") {
        if (subtype == "constant") {
            push_spectrum_texture(LAMBDA_SPECTRUM_CONSTANT, spectrum<float>(ss, "spectrum"));
        } else if (subtype == "checker") {
            const int a = spectrum<float>(ss, "value1");
            const int b = spectrum<float>(ss, "value2");
            const float scale = value<float>(ss, "scale");
            push_spectrum_texture(LAMBDA_SPECTRUM_CHECKER, a, b, scale);
        } else if (subtype == "scalar") {
            // The reference reads the texture name twice (parser.h:141).
            int index;
            if (scalar_textures_.count(value<std::string>(ss, "texture")))
                index = scalar_textures_.at(value<std::string>(ss, "texture"));
            else
                throw error("'texture' is not defined");
            push_spectrum_texture(LAMBDA_SPECTRUM_SCALAR, index);
        } else {
            throw error("'subtype' must be \"constant\", \"checker\", or \"scalar\"");
        }
        spectrum_textures_[name] = int(s_.spectrum_textures.size()) - 1;
    } else {
        throw error("'type' must be \"scalar\" or \"spectrum\"");
    }
}

void LrdReader::cmd_material(std::istringstream &ss) {
    const std::string name = value<std::string>(ss, "name");
    const std::string type = value<std::string>(ss, "type");
    if (materials_.count(name)) throw error("'name' is already defined");
    lambda_material m{};
    if (type == "lambertian" || type == "mirror") {
        const int albedo = spectrum_texture(ss, "albedo");
        const float lo = spectrum_texture_min(s_, albedo);
        const float hi = spectrum_texture_max(s_, albedo);
        if (lo < 0) throw error("'albedo' must be positive, got " + std::to_string(lo));
        else if (hi > 1) throw error("'albedo' must be at most 1, got " + std::to_string(hi));
        m.type = type == "lambertian" ? LAMBDA_MATERIAL_LAMBERTIAN : LAMBDA_MATERIAL_MIRROR;
        m.p[0] = albedo;
    } else if (type == "dielectric") {
        const int n0 = spectrum<float>(ss, "n0");
        const int n1 = spectrum<float>(ss, "n1");
        for (int i = 0; i < kBins; i++) {
            const float a = s_.spectra[size_t(n0) * kBins + i];
            const float b = s_.spectra[size_t(n1) * kBins + i];
            if (a <= 0) throw error("'n0' must be positive, got " + std::to_string(a));
            if (b <= 0) throw error("'n1' must be positive, got " + std::to_string(b));
        }
        m.type = LAMBDA_MATERIAL_DIELECTRIC;
        m.p[0] = n0;
        m.p[1] = n1;
    } else if (type == "emissive") {
        m.type = LAMBDA_MATERIAL_EMISSIVE;
        m.p[0] = spectrum_texture(ss, "emission");
    } else if (type == "thinfilm") {
        const std::vector<int> n = complex_spectrum_array(ss, "n");
        if (n.size() < 2) throw error("'n' must have at least 2 entries, got " + std::to_string(n.size()));
        const int n_offset = int(s_.material_properties.size());
        s_.material_properties.insert(s_.material_properties.end(), n.begin(), n.end());
        const int layers = int(n.size()) - 2;
        const std::vector<std::string> d = name_array(ss, "d");
        if (int(d.size()) != layers)
            throw error("'d' must have " + std::to_string(layers) + " entries, got " + std::to_string(d.size()));
        const int d_offset = int(s_.material_properties.size());
        for (int i = 0; i < layers; i++) {
            try {
                const int t = push_scalar_texture(LAMBDA_SCALAR_CONSTANT, to_float(d[i]));
                s_.material_properties.push_back(t);
            } catch (const std::exception &) {
                auto it = scalar_textures_.find(d[i]);
                if (it == scalar_textures_.end()) throw error("'d' is not defined");
                s_.material_properties.push_back(it->second);
            }
        }
        m.type = LAMBDA_MATERIAL_THINFILM;
        m.p[0] = layers;
        m.p[1] = n_offset;
        m.p[2] = d_offset;
    } else {
        throw error("'type' must be \"dielectric\", \"emissive\", \"lambertian\", \"mirror\", or \"thinfilm\"");
    }
    s_.materials.push_back(m);
    materials_[name] = int(s_.materials.size()) - 1;
}

void LrdReader::cmd_object(std::istringstream &ss) {
    const std::string name = value<std::string>(ss, "name");
    const std::string type = value<std::string>(ss, "type");
    const std::string material_name = value<std::string>(ss, "material");
    if (name == "default") throw error("'name' is already defined");
    auto g = groups_.find(name);
    if (g != groups_.end()) {
        if (g->second != int(group_offsets_.size()) - 1) throw error("'name' is already defined");
    } else {
        groups_[name] = int(group_offsets_.size());
        group_offsets_.push_back(int(s_.objects.size()));
    }
    auto mi = materials_.find(material_name);
    if (mi == materials_.end()) throw error("'material' is not defined");
    const int material = mi->second;

    if (type == "sphere") {
        const V3 c = vector(ss, "center");
        const float r = value<float>(ss, "radius");
        if (r <= 0) throw error("'radius' must be positive, got " + std::to_string(r));
        lambda_object o{};
        o.type = LAMBDA_OBJECT_SPHERE;
        o.material = material;
        o.g[0] = c[0];
        o.g[1] = c[1];
        o.g[2] = c[2];
        o.g[3] = r;
        s_.objects.push_back(o);
    } else if (type == "quad" || type == "tri") {
        const V3 c = vector(ss, "corner");
        const V3 h = vector(ss, "horizontal");
        const V3 v = vector(ss, "vertical");
        if (length(h) < kEpsilon) throw error("'horizontal' must be non-zero");
        if (length(v) < kEpsilon) throw error("'vertical' must be non-zero");
        if (length(cross(h, v)) < kEpsilon) throw error("'horizontal' and 'vertical' must be non-parallel");
        if (type == "quad") {
            lambda_object o{};
            o.type = LAMBDA_OBJECT_QUAD;
            o.material = material;
            const V3 n = cross(h, v);
            const V3 parts[4] = {c, h, v, n};
            for (int k = 0; k < 4; k++)
                for (int j = 0; j < 3; j++) o.g[3 * k + j] = parts[k][j];
            s_.objects.push_back(o);
        } else {
            const V3 z = v3(0, 0, 0);
            s_.objects.push_back(make_tri(material, c, h, v, z, z, z, 0, 0, 0, 0, 0, 0));
        }
    } else if (type == "mesh") {
        const std::string obj = value<std::string>(ss, "file");
        read_obj(obj, s_.objects, material);
    } else {
        throw error("'type' must be \"quad\", \"sphere\", or \"tri\"");
    }
}

void LrdReader::cmd_instance(std::istringstream &ss) {
    const std::string object_name = value<std::string>(ss, "object");
    const std::string material_name = value<std::string>(ss, "material");
    auto g = groups_.find(object_name);
    if (g == groups_.end()) throw error("'object' is not defined");
    const int group = g->second;
    const int first = group_offsets_[group];
    const int count = group < int(group_offsets_.size()) - 1 ? group_offsets_[group + 1] - first
                                                              : int(s_.objects.size()) - first;
    int material = -1;
    if (material_name != "default") {
        auto mi = materials_.find(material_name);
        if (mi == materials_.end()) throw error("'material' is not defined");
        material = mi->second;
    }
    const V3 t = vector(ss, "translation");
    const V3 r = vector(ss, "rotation");
    const V3 sc = vector(ss, "scale");
    if (std::fabs(sc[0]) < kEpsilon || std::fabs(sc[1]) < kEpsilon || std::fabs(sc[2]) < kEpsilon)
        throw error("'scale' must be non-zero");

    // instance.h:13-28: T * Rz * Ry * Rx * S and its inverse
    const float sx = std::sin(r[0]), cx = std::cos(r[0]);
    const float sy = std::sin(r[1]), cy = std::cos(r[1]);
    const float sz = std::sin(r[2]), cz = std::cos(r[2]);
    const M4 T{{1, 0, 0, t[0], 0, 1, 0, t[1], 0, 0, 1, t[2], 0, 0, 0, 1}};
    const M4 Rx{{1, 0, 0, 0, 0, cx, -sx, 0, 0, sx, cx, 0, 0, 0, 0, 1}};
    const M4 Ry{{cy, 0, sy, 0, 0, 1, 0, 0, -sy, 0, cy, 0, 0, 0, 0, 1}};
    const M4 Rz{{cz, -sz, 0, 0, sz, cz, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}};
    const M4 S{{sc[0], 0, 0, 0, 0, sc[1], 0, 0, 0, 0, sc[2], 0, 0, 0, 0, 1}};
    const M4 M = mat_mul(mat_mul(mat_mul(mat_mul(T, Rz), Ry), Rx), S);
    const M4 Mi = mat_inverse(M);

    lambda_instance in{};
    in.object = first;
    in.count = count;
    in.node = 0;
    in.material = material;
    std::memcpy(in.transform, M.m, sizeof(M.m));
    std::memcpy(in.inverse_transform, Mi.m, sizeof(Mi.m));

    if (std::fabs(sc[0] - sc[1]) > kEpsilon || std::fabs(sc[1] - sc[2]) > kEpsilon)
        for (int i = 0; i < count; i++) {
            const int m = material >= 0 ? material : s_.objects[first + i].material;
            if (s_.materials[m].type == LAMBDA_MATERIAL_EMISSIVE) throw error("'scale' must be uniform for emissive objects");
        }
    s_.instances.push_back(in);
}

void LrdReader::cmd_background(std::istringstream &ss) {
    const std::string type = value<std::string>(ss, "type");
    if (type != "equirectangular") throw error("'type' must be \"equirectangular\"");
    s_.background_texture = spectrum_texture(ss, "background");
}

void LrdReader::cmd_camera(std::istringstream &ss) {
    const V3 p = vector(ss, "position");
    const V3 c = vector(ss, "corner");
    const V3 h = vector(ss, "horizontal");
    const V3 v = vector(ss, "vertical");
    if (length(h) < kEpsilon) throw error("'horizontal' must be non-zero");
    if (length(v) < kEpsilon) throw error("'vertical' must be non-zero");
    if (length(cross(h, v)) < kEpsilon) throw error("'horizontal' and 'vertical' must be non-parallel");
    lambda_camera &cam = s_.settings.camera;
    for (int k = 0; k < 3; k++) {
        cam.position[k] = p[k];
        cam.corner[k] = c[k];
        cam.horizontal[k] = h[k];
        cam.vertical[k] = v[k];
    }
}

void LrdReader::run() {
    std::ifstream in(file_);
    if (!in.is_open()) throw SceneError(LAMBDA_ERR_IO, file_ + ": failed to open file (" + strerror_lower() + ")");

    // Defaults every scene starts with (parser.h:50-60).
    push_float_spectrum(std::vector<float>(kBins, 0.5f));
    push_spectrum_texture(LAMBDA_SPECTRUM_CONSTANT, 0);
    spectrum_textures_["default"] = 0;
    push_scalar_texture(LAMBDA_SCALAR_CONSTANT, 0.5f);
    scalar_textures_["default"] = 0;
    lambda_material lambertian{};
    lambertian.type = LAMBDA_MATERIAL_LAMBERTIAN;
    s_.materials.push_back(lambertian);
    materials_["default"] = 0;

    bool have_render = false, have_background = false, have_camera = false, have_instance = false;
    std::string raw;
    while (std::getline(in, raw)) {
        line_++;
        const std::string line = preprocess(raw);
        if (line.empty()) continue;
        std::istringstream ss(line);
        std::string cmd;
        if (!(ss >> cmd)) continue;
        if (!have_render && cmd != "Render") throw error("expected \"Render\", got \"" + cmd + "\"");
        if (cmd == "Render") {
            have_render = true;
            cmd_render(ss);
        } else if (cmd == "Texture") {
            cmd_texture(ss);
        } else if (cmd == "Material") {
            cmd_material(ss);
        } else if (cmd == "Object") {
            cmd_object(ss);
        } else if (cmd == "Instance") {
            have_instance = true;
            cmd_instance(ss);
        } else if (cmd == "Background") {
            have_background = true;
            cmd_background(ss);
        } else if (cmd == "Camera") {
            have_camera = true;
            cmd_camera(ss);
        } else {
            throw error("expected \"Background\", \"Camera\", \"Instance\", \"Material\", \"Render\", \"Object\", or \"Texture\", got \"" + cmd + "\"");
        }
        if (ss >> cmd) throw error("unexpected token \"" + cmd + "\"");
    }
    if (!have_render) throw SceneError(LAMBDA_ERR_PARSE, file_ + ": expected \"Render\"");
    if (!have_background) throw SceneError(LAMBDA_ERR_PARSE, file_ + ": expected \"Background\"");
    if (!have_camera) throw SceneError(LAMBDA_ERR_PARSE, file_ + ": expected \"Camera\"");
    if (!have_instance) throw SceneError(LAMBDA_ERR_PARSE, file_ + ": expected \"Instance\"");

    group_offsets_.push_back(int(s_.objects.size()));
    std::vector<float> boxes;
    build_bvh(s_, group_offsets_, accel_, &boxes);
    build_lights(s_, &boxes);
}

// parser.h:639-786. Faces are fan-triangulated; missing vt gives per-triangle
// uvs (0,0), (1,0), (0,1); missing vn gives the flat normal.
// Fast reading of the common OBJ lines ("v x y z", "vt u v", "vn x y z" with plain
// decimal numbers, "f a b c ..." with plain positive indices). A token is taken only
// when std::from_chars consumes it whole, its characters are [0-9.eE+-] (so no
// inf/nan, which the stream extraction rejects), and the value is zero or normal
// (no overflow or subnormal range, where stream extraction may fail): for those
// both give the same correctly rounded float. Any other line returns false and is
// read by the stream-based code, which keeps the reference's semantics and errors.
namespace obj_fast {

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

bool next_token(const char *&p, const char *end, const char *&tb, const char *&te) {
    while (p < end && is_space(*p)) p++;
    if (p >= end) return false;
    tb = p;
    while (p < end && !is_space(*p)) p++;
    te = p;
    return true;
}

bool number(const char *tb, const char *te, float &out) {
    bool digit_nonzero = false;
    for (const char *c = tb; c < te; c++) {
        if (!((*c >= '0' && *c <= '9') || *c == '.' || *c == 'e' || *c == 'E' || *c == '+' || *c == '-')) return false;
        if (*c >= '1' && *c <= '9') digit_nonzero = true;
    }
    if (*tb == '+') return false;
    float v = 0;
    const auto r = std::from_chars(tb, te, v, std::chars_format::general);
    if (r.ec != std::errc() || r.ptr != te) return false;
    if (v == 0.0f ? digit_nonzero : !(std::fabs(v) >= std::numeric_limits<float>::min())) return false;
    if (!std::isfinite(v)) return false;
    out = v;
    return true;
}

bool index(const char *tb, const char *te, int size, int &out) {
    if (te - tb > 9) return false;
    int v = 0;
    for (const char *c = tb; c < te; c++) {
        if (*c < '0' || *c > '9') return false;
        v = v * 10 + (*c - '0');
    }
    if (v < 1 || v > size) return false;
    out = v - 1;
    return true;
}

}  // namespace obj_fast

void read_obj(const std::string &path, std::vector<lambda_object> &objects, int material) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) throw SceneError(LAMBDA_ERR_IO, path + ": failed to open file (" + strerror_lower() + ")");
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    int line_no = 0;
    auto error = [&](const std::string &msg) {
        return SceneError(LAMBDA_ERR_PARSE, path + ":" + std::to_string(line_no) + ": " + msg);
    };
    bool have_face = false;
    std::vector<V3> vertices, normals;
    std::vector<float> us, vs;
    std::vector<int> vi, ti, ni;
    auto emit_face = [&]() {
        if (vi.size() < 3) throw error("'f' must have at least 3 vertices");
        const V3 zero = v3(0, 0, 0);
        const V3 p0 = vertices[vi[0]];
        const V3 n0 = ni[0] >= 0 ? normals[ni[0]] : zero;
        const float u0 = ti[0] >= 0 ? us[ti[0]] : 0, v0 = ti[0] >= 0 ? vs[ti[0]] : 0;
        for (size_t k = 1; k + 1 < vi.size(); k++) {
            const V3 p1 = vertices[vi[k]], p2 = vertices[vi[k + 1]];
            const V3 n1 = ni[k] >= 0 ? normals[ni[k]] : zero;
            const V3 n2 = ni[k + 1] >= 0 ? normals[ni[k + 1]] : zero;
            const float u1 = ti[k] >= 0 ? us[ti[k]] : 1, v1 = ti[k] >= 0 ? vs[ti[k]] : 0;
            const float u2 = ti[k + 1] >= 0 ? us[ti[k + 1]] : 0, v2 = ti[k + 1] >= 0 ? vs[ti[k + 1]] : 1;
            objects.push_back(make_tri(material, p0, p1 - p0, p2 - p0, n0, n1, n2, u0, u1, u2, v0, v1, v2));
        }
    };
    // One line by the fast rules; false leaves every container as it was.
    auto fast_line = [&](const char *p, const char *end) -> bool {
        const char *tb, *te;
        if (!obj_fast::next_token(p, end, tb, te)) return true;  // blank line
        const std::string_view tag(tb, size_t(te - tb));
        if (tag == "v" || tag == "vn") {
            float x[3];
            for (float &c : x)
                if (!obj_fast::next_token(p, end, tb, te) || !obj_fast::number(tb, te, c)) return false;
            if (obj_fast::next_token(p, end, tb, te)) return false;
            (tag == "v" ? vertices : normals).push_back(v3(x[0], x[1], x[2]));
            return true;
        }
        if (tag == "vt") {
            float u, v;
            if (!obj_fast::next_token(p, end, tb, te) || !obj_fast::number(tb, te, u)) return false;
            if (!obj_fast::next_token(p, end, tb, te) || !obj_fast::number(tb, te, v)) return false;
            if (obj_fast::next_token(p, end, tb, te)) return false;
            us.push_back(u);
            vs.push_back(v);
            return true;
        }
        if (tag == "f") {
            vi.clear();
            while (obj_fast::next_token(p, end, tb, te)) {
                int idx;
                if (!obj_fast::index(tb, te, int(vertices.size()), idx)) return false;
                vi.push_back(idx);
            }
            if (vi.size() < 3) return false;
            ti.assign(vi.size(), -1);
            ni.assign(vi.size(), -1);
            have_face = true;
            emit_face();
            return true;
        }
        return false;
    };
    std::string line;
    size_t pos = 0;
    while (pos < text.size()) {
        size_t eol = text.find('\n', pos);
        if (eol == std::string::npos) eol = text.size();
        const char *lb = text.data() + pos, *le = text.data() + eol;
        pos = eol + 1;
        line_no++;
        if (lb == le) continue;
        if (fast_line(lb, le)) continue;
        line.assign(lb, le);
        std::istringstream ss(line);
        std::string tag;
        if (!(ss >> tag)) continue;
        if (tag == "v") {
            V3 p = v3(0, 0, 0);
            if (!(ss >> p[0])) throw error("'x' is missing or invalid");
            if (!(ss >> p[1])) throw error("'y' is missing or invalid");
            if (!(ss >> p[2])) throw error("'z' is missing or invalid");
            vertices.push_back(p);
        } else if (tag == "vt") {
            float u, v;
            if (!(ss >> u)) throw error("'u' is missing or invalid");
            if (!(ss >> v)) throw error("'v' is missing or invalid");
            us.push_back(u);
            vs.push_back(v);
        } else if (tag == "vn") {
            V3 n = v3(0, 0, 0);
            if (!(ss >> n[0])) throw error("'x' is missing or invalid");
            if (!(ss >> n[1])) throw error("'y' is missing or invalid");
            if (!(ss >> n[2])) throw error("'z' is missing or invalid");
            normals.push_back(n);
        } else if (tag == "f") {
            have_face = true;
            vi.clear();
            ti.clear();
            ni.clear();
            std::string tok;
            while (ss >> tok) {
                std::istringstream ts(tok);
                std::string a, b, c;
                if (!std::getline(ts, a, '/')) throw error("'v' is missing or invalid");
                std::getline(ts, b, '/');
                std::getline(ts, c, '/');
                auto resolve = [&](const std::string &text, int size, const char *what) {
                    int idx;
                    try {
                        idx = std::stoi(text);
                    } catch (const std::exception &) {
                        throw error(std::string("'") + what + "' is missing or invalid");
                    }
                    if (idx < 0 && size + idx >= 0) return size + idx;
                    // index 0 would read before the first element in the reference
                    if (idx == 0 && what[1] == 0) throw error("'v' must be positive, got 0");
                    if (idx < 0) throw error(std::string("'") + what + "' must be positive, got " + std::to_string(idx));
                    if (idx > size)
                        throw error(std::string("'") + what + "' must be at most " + std::to_string(size - 1) + ", got " + std::to_string(idx));
                    return idx - 1;
                };
                vi.push_back(resolve(a, int(vertices.size()), "v"));
                ti.push_back(b.empty() ? -1 : resolve(b, int(us.size()), "vt"));
                ni.push_back(c.empty() ? -1 : resolve(c, int(normals.size()), "vn"));
            }
            emit_face();
        } else {
            continue;
        }
        if (ss >> tag) throw error("unexpected token \"" + tag + "\"");
    }
    if (!have_face) throw error("expected \"f\"");
}

}  // namespace

float spectrum_average(const HostScene &s, int i) {
    const float *d = &s.spectra[size_t(i) * kBins];
    float sum = 0;
    for (int k = 0; k < kBins; k++) sum += d[k];
    return sum / kBins;
}

float spectrum_min(const HostScene &s, int i) {
    const float *d = &s.spectra[size_t(i) * kBins];
    float m = d[0];
    for (int k = 1; k < kBins; k++)
        if (d[k] < m) m = d[k];
    return m;
}

float spectrum_max(const HostScene &s, int i) {
    const float *d = &s.spectra[size_t(i) * kBins];
    float m = d[0];
    for (int k = 1; k < kBins; k++)
        if (d[k] > m) m = d[k];
    return m;
}

float spectrum_texture_min(const HostScene &s, int t) {
    const lambda_spectrum_texture &x = s.spectrum_textures[t];
    switch (x.type) {
        case LAMBDA_SPECTRUM_CONSTANT: return spectrum_min(s, x.value1);
        case LAMBDA_SPECTRUM_CHECKER: return std::fmin(spectrum_min(s, x.value1), spectrum_min(s, x.value2));
        default: return scalar_texture_min(s, x.value1);
    }
}

float spectrum_texture_max(const HostScene &s, int t) {
    const lambda_spectrum_texture &x = s.spectrum_textures[t];
    switch (x.type) {
        case LAMBDA_SPECTRUM_CONSTANT: return spectrum_max(s, x.value1);
        case LAMBDA_SPECTRUM_CHECKER: return std::fmax(spectrum_max(s, x.value1), spectrum_max(s, x.value2));
        default: return scalar_texture_max(s, x.value1);
    }
}

float spectrum_texture_average(const HostScene &s, int t) {
    const lambda_spectrum_texture &x = s.spectrum_textures[t];
    switch (x.type) {
        case LAMBDA_SPECTRUM_CONSTANT: return spectrum_average(s, x.value1);
        case LAMBDA_SPECTRUM_CHECKER: return 0.5f * (spectrum_average(s, x.value1) + spectrum_average(s, x.value2));
        default: return scalar_texture_average(s, x.value1);
    }
}

void parse_lrd(const std::string &path, HostScene &scene, const BuildAccel *accel) {
    scene = HostScene{};
    LrdReader reader(path, scene);
    reader.accel_ = accel;
    reader.run();
}

lambda_scene_desc HostScene::desc() const {
    lambda_scene_desc d{};
    d.spectra = spectra.data();
    d.num_spectra = num_spectra();
    d.complex_spectra = complex_spectra.data();
    d.num_complex_spectra = num_complex_spectra();
    d.background_texture = background_texture;
    d.objects = objects.data();
    d.num_objects = int32_t(objects.size());
    d.instances = instances.data();
    d.num_instances = int32_t(instances.size());
    d.nodes = nodes.data();
    d.num_nodes = int32_t(nodes.size());
    d.light_instances = light_instances.data();
    d.light_objects = light_objects.data();
    d.light_powers = light_powers.data();
    d.num_lights = int32_t(light_instances.size());
    d.total_light_power = total_light_power;
    d.materials = materials.data();
    d.num_materials = int32_t(materials.size());
    d.material_properties = material_properties.data();
    d.num_material_properties = int32_t(material_properties.size());
    d.scalar_textures = scalar_textures.data();
    d.num_scalar_textures = int32_t(scalar_textures.size());
    d.spectrum_textures = spectrum_textures.data();
    d.num_spectrum_textures = int32_t(spectrum_textures.size());
    return d;
}

}  // namespace lambda_host
