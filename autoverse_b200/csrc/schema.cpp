// Host-side schema: JSON reader, config validation, seed generation and
// kernel construction.  Arithmetic is f32 in the reference's statement order
// (the translation unit is built with -ffp-contract=off) so that the initial
// state and the kernel taps are bit-identical to the reference's.
#include <algorithm>
#include "schema.h"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace flp {

// ------------------------------------------------------------------ JSON ----
namespace {

struct Parser {
    const char* p;
    const char* end;

    [[noreturn]] void fail(const char* what) {
        throw ConfigError(std::string("JSON parse error: ") + what);
    }
    void ws() {
        while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    }
    bool lit(const char* s) {
        size_t n = std::strlen(s);
        if (size_t(end - p) >= n && std::strncmp(p, s, n) == 0) {
            p += n;
            return true;
        }
        return false;
    }
    std::string string_body() {
        std::string out;
        ++p;  // opening quote
        while (p < end && *p != '"') {
            if (*p == '\\') {
                ++p;
                if (p >= end) fail("bad escape");
                char c = *p++;
                switch (c) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        if (end - p < 4) fail("bad \\u escape");
                        unsigned cp = std::strtoul(std::string(p, 4).c_str(), nullptr, 16);
                        p += 4;
                        if (cp < 0x80) out += char(cp);
                        else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
                        else { out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F)); }
                        break;
                    }
                    default: fail("bad escape");
                }
            } else {
                out += *p++;
            }
        }
        if (p >= end) fail("unterminated string");
        ++p;
        return out;
    }
    Json value(int depth) {
        if (depth > 64) fail("nesting too deep");
        ws();
        if (p >= end) fail("unexpected end");
        Json j;
        if (*p == '{') {
            j.kind = Json::Object;
            ++p;
            ws();
            if (p < end && *p == '}') { ++p; return j; }
            for (;;) {
                ws();
                if (p >= end || *p != '"') fail("expected key");
                std::string k = string_body();
                ws();
                if (p >= end || *p != ':') fail("expected ':'");
                ++p;
                j.obj[k] = value(depth + 1);
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == '}') { ++p; break; }
                fail("expected ',' or '}'");
            }
        } else if (*p == '[') {
            j.kind = Json::Array;
            ++p;
            ws();
            if (p < end && *p == ']') { ++p; return j; }
            for (;;) {
                j.arr.push_back(value(depth + 1));
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == ']') { ++p; break; }
                fail("expected ',' or ']'");
            }
        } else if (*p == '"') {
            j.kind = Json::String;
            j.str = string_body();
        } else if (lit("true")) {
            j.kind = Json::Bool; j.b = true;
        } else if (lit("false")) {
            j.kind = Json::Bool; j.b = false;
        } else if (lit("null")) {
            j.kind = Json::Null;
        } else {
            char* e = nullptr;
            std::string tok;
            const char* q = p;
            while (q < end && (std::strchr("+-0123456789.eE", *q) != nullptr)) ++q;
            tok.assign(p, q);
            if (tok.empty()) fail("unexpected character");
            j.kind = Json::Number;
            j.num = std::strtod(tok.c_str(), &e);
            if (e != tok.c_str() + tok.size()) fail("bad number");
            p = q;
        }
        return j;
    }
};

}  // namespace

Json parse_json(const std::string& text) {
    Parser ps{text.data(), text.data() + text.size()};
    Json j = ps.value(0);
    ps.ws();
    if (ps.p != ps.end) ps.fail("trailing characters");
    return j;
}

const Json& Json::at(const std::string& k) const {
    if (kind != Object) throw ConfigError("expected an object while looking up '" + k + "'");
    auto it = obj.find(k);
    if (it == obj.end()) throw ConfigError("missing field '" + k + "'");
    return it->second;
}

const Json& Json::at(size_t i) const {
    if (kind != Array || i >= arr.size()) throw ConfigError("array index out of range");
    return arr[i];
}

double Json::number() const {
    if (kind != Number) throw ConfigError("expected a number");
    return num;
}

int64_t Json::integer() const {
    double v = number();
    if (v < 0 || v != std::floor(v)) throw ConfigError("expected a non-negative integer");
    return static_cast<int64_t>(v);
}

// ---------------------------------------------------------------- config ----
void validate(const SimulationConfig& c) {
    if (c.width <= 0 || c.height <= 0 || c.depth <= 0)
        throw ConfigError("Grid dimensions (width, height, depth) must be non-zero");
    if (c.channels <= 0) throw ConfigError("Channel count must be non-zero");
    if (!(c.dt > 0.f)) throw ConfigError("Time step must be positive");
    if (c.kernel_radius <= 0) throw ConfigError("Kernel radius must be non-zero");
    for (size_t i = 0; i < c.kernels.size(); ++i) {
        const auto& k = c.kernels[i];
        if (k.source_channel >= c.channels)
            throw ConfigError("Kernel " + std::to_string(i) + " references invalid channel " +
                              std::to_string(k.source_channel));
        if (k.target_channel >= c.channels)
            throw ConfigError("Kernel " + std::to_string(i) + " references invalid channel " +
                              std::to_string(k.target_channel));
    }
}

SimulationConfig parse_config(const std::string& text) {
    Json j = parse_json(text);
    SimulationConfig c;
    c.width = int(j.at("width").integer());
    c.height = int(j.at("height").integer());
    c.depth = j.has("depth") ? int(j.at("depth").integer()) : 1;
    c.channels = int(j.at("channels").integer());
    c.dt = j.at("dt").f32();
    c.kernel_radius = int(j.at("kernel_radius").integer());
    for (const Json& kj : j.at("kernels").arr) {
        KernelConfig k;
        k.radius = kj.at("radius").f32();
        for (const Json& rj : kj.at("rings").arr)
            k.rings.push_back({rj.at("amplitude").f32(), rj.at("distance").f32(), rj.at("width").f32()});
        k.weight = kj.at("weight").f32();
        k.mu = kj.at("mu").f32();
        k.sigma = kj.at("sigma").f32();
        k.source_channel = int(kj.at("source_channel").integer());
        k.target_channel = int(kj.at("target_channel").integer());
        c.kernels.push_back(k);
    }
    const Json& f = j.at("flow");
    c.flow = {f.at("beta_a").f32(), f.at("n").f32(), f.at("distribution_size").f32()};
    if (j.has("embedding") && j.at("embedding").kind != Json::Null) {
        // a present EmbeddingConfig needs all three fields (no per-field serde defaults)
        const Json& e = j.at("embedding");
        if (e.kind != Json::Object || !e.has("enabled") || !e.has("mixing_temperature") || !e.has("linear_mixing") ||
            e.at("enabled").kind != Json::Bool || e.at("linear_mixing").kind != Json::Bool)
            throw ConfigError("embedding: expected {enabled, mixing_temperature, linear_mixing}");
        c.embedding_enabled = e.at("enabled").b;
        c.embedding_temperature = e.at("mixing_temperature").f32();
        c.embedding_linear = e.at("linear_mixing").b;
    }
    validate(c);
    return c;
}

// ----------------------------------------------------------------- kernel ----
// R = float is the engine's stencil (the reference's f32 arithmetic); the FP64
// twin instantiates the same statements in double.
template <class R>
KernelStencilT<R> build_kernel_t(const KernelConfig& kc, int max_radius, int dims) {
    KernelStencilT<R> k;
    R rr = std::round(R(kc.radius) * R(max_radius));
    int actual_radius = rr > R(0) ? int(rr) : 0;
    k.radius = actual_radius;
    k.size = actual_radius * 2 + 1;
    k.dims = dims;
    const int size = k.size;
    const R center = R(actual_radius);
    const int zs = dims == 3 ? size : 1;
    k.data.assign(size_t(size) * size * zs, R(0));
    R sum = R(0);
    for (int z = 0; z < zs; ++z)
        for (int y = 0; y < size; ++y)
            for (int x = 0; x < size; ++x) {
                R dx = R(x) - center, dy = R(y) - center;
                R dist;
                if (dims == 3) {
                    R dz = R(z) - center;
                    dist = std::sqrt(dx * dx + dy * dy + dz * dz);
                } else {
                    dist = std::sqrt(dx * dx + dy * dy);
                }
                R norm_dist = dist / R(actual_radius);
                if (norm_dist > R(1)) continue;
                R value = R(0);
                for (const auto& ring : kc.rings) {
                    R ring_dist = std::fabs(norm_dist - R(ring.distance));
                    R bump = R(ring.amplitude) *
                             std::exp(-ring_dist * ring_dist / (R(2) * R(ring.width) * R(ring.width)));
                    value += bump;
                }
                k.data[(size_t(z) * size + y) * size + x] = value;
                sum += value;
            }
    if (sum > R(0)) {
        R inv_sum = R(1) / sum;
        for (auto& v : k.data) v *= inv_sum;
    }
    return k;
}
template KernelStencilT<float> build_kernel_t<float>(const KernelConfig&, int, int);
template KernelStencilT<double> build_kernel_t<double>(const KernelConfig&, int, int);

KernelStencil build_kernel(const KernelConfig& kc, int max_radius, int dims) {
    return build_kernel_t<float>(kc, max_radius, dims);
}

template <class R>
std::vector<R> pad_kernel_t(const KernelStencilT<R>& k, int W, int H, int D) {
    // The reference indexes with ((dx + W) % W) as usize, which panics (an
    // out-of-range index) once r exceeds a side; report it instead.
    if (k.radius > W || k.radius > H || (k.dims == 3 && k.radius > D))
        throw ConfigError("kernel radius " + std::to_string(k.radius) + " exceeds a grid side");
    std::vector<R> out(size_t(W) * H * D, R(0));
    const int c = k.size / 2;
    const int zs = k.dims == 3 ? k.size : 1;
    for (int kz = 0; kz < zs; ++kz)
        for (int ky = 0; ky < k.size; ++ky)
            for (int kx = 0; kx < k.size; ++kx) {
                int tx = ((kx - c) + W) % W, ty = ((ky - c) + H) % H, tz = 0;
                if (k.dims == 3) tz = ((kz - c) + D) % D;
                out[(size_t(tz) * H + ty) * W + tx] = k.data[(size_t(kz) * k.size + ky) * k.size + kx];
            }
    return out;
}
template std::vector<float> pad_kernel_t<float>(const KernelStencilT<float>&, int, int, int);
template std::vector<double> pad_kernel_t<double>(const KernelStencilT<double>&, int, int, int);

std::vector<float> pad_kernel(const KernelStencil& k, int W, int H, int D) { return pad_kernel_t<float>(k, W, H, D); }

// ------------------------------------------------------------------- seed ----
namespace {

struct Grid {
    int W, H, D, C;
    float* g;
    float* plane(int c) { return g + size_t(c) * W * H * D; }
};

void gaussian_2d(Grid& G, int channel, float cx, float cy, float radius, float amplitude) {
    if (channel < 0 || channel >= G.C) return;
    float* g = G.plane(channel);
    float sigma_sq = (radius / 2.0f) * (radius / 2.0f);
    for (int y = 0; y < G.H; ++y)
        for (int x = 0; x < G.W; ++x) {
            float dx = float(x) - cx, dy = float(y) - cy;
            float dist_sq = dx * dx + dy * dy;
            g[size_t(y) * G.W + x] += amplitude * std::exp(-dist_sq / (2.0f * sigma_sq));
        }
}

void gaussian_3d(Grid& G, int channel, float cx, float cy, float cz, float radius, float amplitude) {
    if (channel < 0 || channel >= G.C) return;
    float* g = G.plane(channel);
    float sigma_sq = (radius / 2.0f) * (radius / 2.0f);
    for (int z = 0; z < G.D; ++z)
        for (int y = 0; y < G.H; ++y)
            for (int x = 0; x < G.W; ++x) {
                float dx = float(x) - cx, dy = float(y) - cy, dz = float(z) - cz;
                float dist_sq = dx * dx + dy * dy + dz * dz;
                g[(size_t(z) * G.H + y) * G.W + x] += amplitude * std::exp(-dist_sq / (2.0f * sigma_sq));
            }
}

void shell_like(Grid& G, int channel, float cx, float cy, float cz, float r_in, float r_out, float amplitude,
                bool flat) {
    if (channel < 0 || channel >= G.C) return;
    float* g = G.plane(channel);
    int zs = flat ? 1 : G.D;
    for (int z = 0; z < zs; ++z)
        for (int y = 0; y < G.H; ++y)
            for (int x = 0; x < G.W; ++x) {
                float dx = float(x) - cx, dy = float(y) - cy;
                float dist;
                if (flat) {
                    dist = std::sqrt(dx * dx + dy * dy);
                } else {
                    float dz = float(z) - cz;
                    dist = std::sqrt(dx * dx + dy * dy + dz * dz);
                }
                if (dist >= r_in && dist <= r_out) {
                    float edge = (r_out - r_in) * 0.2f;
                    float inner = std::fmin((dist - r_in) / edge, 1.0f);
                    float outer = std::fmin((r_out - dist) / edge, 1.0f);
                    g[(size_t(z) * G.H + y) * G.W + x] += amplitude * std::fmin(inner, outer);
                }
            }
}

void torus_3d(Grid& G, int channel, float cx, float cy, float cz, float rmaj, float rmin, float amplitude) {
    if (channel < 0 || channel >= G.C) return;
    float* g = G.plane(channel);
    float sigma_sq = (rmin / 2.0f) * (rmin / 2.0f);
    for (int z = 0; z < G.D; ++z)
        for (int y = 0; y < G.H; ++y)
            for (int x = 0; x < G.W; ++x) {
                float dx = float(x) - cx, dy = float(y) - cy, dz = float(z) - cz;
                float dist_xy = std::sqrt(dx * dx + dy * dy);
                float ring_dx = dist_xy - rmaj;
                float d = std::sqrt(ring_dx * ring_dx + dz * dz);
                float value = amplitude * std::exp(-d * d / (2.0f * sigma_sq));
                if (value > 1e-6f) g[(size_t(z) * G.H + y) * G.W + x] += value;
            }
}

float fpair(const Json& a, size_t i) { return a.at(i).f32(); }

}  // namespace

void generate_seed_into(const std::string& seed_json, const SimulationConfig& cfg, float* grid) {
    Json j = parse_json(seed_json);
    const Json& pat = j.at("pattern");
    if (!pat.has("type")) throw ConfigError("seed pattern needs a \"type\" tag");
    const std::string t = pat.at("type").str;
    const int W = cfg.width, H = cfg.height, D = cfg.depth, Cn = cfg.channels;
    std::fill(grid, grid + size_t(Cn) * W * H * D, 0.f);
    Grid G{W, H, D, Cn, grid};
    const float min_xy = float(std::min(W, H));
    const float min_dim = float(std::min(std::min(W, H), D));
    const int mid_z = D / 2;

    auto blob = [&](const Json& b) {
        const Json& c = b.at("center");
        float cx = fpair(c, 0) * float(W), cy = fpair(c, 1) * float(H);
        float r = b.at("radius").f32() * min_xy;
        int ch = int(b.at("channel").integer());
        if (D == 1) gaussian_2d(G, ch, cx, cy, r, b.at("amplitude").f32());
        else gaussian_3d(G, ch, cx, cy, 0.5f * float(D), r, b.at("amplitude").f32());
    };
    auto sphere = [&](const Json& s) {
        const Json& c = s.at("center");
        float cx = fpair(c, 0) * float(W), cy = fpair(c, 1) * float(H), cz = fpair(c, 2) * float(D);
        gaussian_3d(G, int(s.at("channel").integer()), cx, cy, cz, s.at("radius").f32() * min_dim,
                    s.at("amplitude").f32());
    };

    if (t == "GaussianBlob") {
        blob(pat);
    } else if (t == "MultiBlob") {
        for (const Json& b : pat.at("blobs").arr) blob(b);
    } else if (t == "Ring") {
        const Json& c = pat.at("center");
        float cx = fpair(c, 0) * float(W), cy = fpair(c, 1) * float(H);
        float r_in = pat.at("inner_radius").f32() * min_xy, r_out = pat.at("outer_radius").f32() * min_xy;
        int ch = int(pat.at("channel").integer());
        float amp = pat.at("amplitude").f32();
        if (D == 1) shell_like(G, ch, cx, cy, 0.f, r_in, r_out, amp, true);
        else shell_like(G, ch, cx, cy, 0.5f * float(D), r_in, r_out, amp, false);
    } else if (t == "GaussianSphere") {
        sphere(pat);
    } else if (t == "MultiSphere") {
        for (const Json& s : pat.at("spheres").arr) sphere(s);
    } else if (t == "Shell" || t == "Torus3D") {
        const Json& c = pat.at("center");
        float cx = fpair(c, 0) * float(W), cy = fpair(c, 1) * float(H), cz = fpair(c, 2) * float(D);
        int ch = int(pat.at("channel").integer());
        float amp = pat.at("amplitude").f32();
        if (t == "Shell")
            shell_like(G, ch, cx, cy, cz, pat.at("inner_radius").f32() * min_dim,
                       pat.at("outer_radius").f32() * min_dim, amp, false);
        else
            torus_3d(G, ch, cx, cy, cz, pat.at("major_radius").f32() * min_dim,
                     pat.at("minor_radius").f32() * min_dim, amp);
    } else if (t == "Noise") {
        float amp = pat.at("amplitude").f32();
        uint64_t st = 0;
        const Json& sj = pat.at("seed");
        if (sj.kind != Json::Number || sj.num < 0) throw ConfigError("noise seed must be a u64");
        st = uint64_t(sj.num);
        int c0 = 0, c1 = Cn;
        if (pat.has("channel") && pat.at("channel").kind != Json::Null) {
            c0 = int(pat.at("channel").integer());
            c1 = c0 + 1;
        }
        const size_t N = size_t(W) * H * D;
        for (int c = c0; c < c1; ++c) {
            if (c >= Cn) continue;
            float* g = G.plane(c);
            for (size_t i = 0; i < N; ++i) {
                st = st * 6364136223846793005ULL + 1ULL;
                float v = float(st >> 33) / float(1ULL << 31);
                g[i] += amp * v;
            }
        }
    } else if (t == "Custom") {
        for (const Json& e : pat.at("values").arr) {
            int64_t x = e.at(0).integer(), y = e.at(1).integer(), c = e.at(2).integer();
            float v = e.at(3).f32();
            if (c < Cn && y < H && x < W) grid[size_t(c) * W * H * D + (size_t(mid_z) * H + y) * W + x] = v;
        }
    } else if (t == "Custom3D") {
        for (const Json& e : pat.at("values").arr) {
            int64_t x = e.at(0).integer(), y = e.at(1).integer(), z = e.at(2).integer(), c = e.at(3).integer();
            float v = e.at(4).f32();
            if (c < Cn && z < D && y < H && x < W) grid[size_t(c) * W * H * D + (size_t(z) * H + y) * W + x] = v;
        }
    } else {
        throw ConfigError("unknown seed pattern type '" + t + "'");
    }
}

std::vector<float> generate_seed(const std::string& seed_json, const SimulationConfig& cfg) {
    std::vector<float> grid(size_t(cfg.channels) * cfg.width * cfg.height * cfg.depth);
    generate_seed_into(seed_json, cfg, grid.data());
    return grid;
}

}  // namespace flp
