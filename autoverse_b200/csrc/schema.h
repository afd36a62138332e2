// Host-side schema of the engine: the reference's JSON config and seed types
// (src/schema/config.rs:14-181, src/schema/seed.rs:13-304) parsed by a small
// JSON reader, validated, and turned into an initial state.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace flp {

// ---------------------------------------------------------------- JSON ----
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    bool has(const std::string& k) const { return kind == Object && obj.count(k) > 0; }
    const Json& at(const std::string& k) const;
    const Json& at(size_t i) const;
    double number() const;
    int64_t integer() const;
    // serde's f32: parse as f64, round to nearest f32.
    float f32() const { return static_cast<float>(number()); }
};

Json parse_json(const std::string& text);

struct ConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// --------------------------------------------------------------- config ----
struct RingConfig {
    float amplitude, distance, width;
};

struct KernelConfig {
    float radius;
    std::vector<RingConfig> rings;
    float weight, mu, sigma;
    int source_channel, target_channel;
};

struct FlowConfig {
    float beta_a, n, distribution_size;
};

struct SimulationConfig {
    int width = 0, height = 0, depth = 1, channels = 0;
    float dt = 0.f;
    int kernel_radius = 0;
    std::vector<KernelConfig> kernels;
    FlowConfig flow{};
    // EmbeddingConfig (schema/embedding.rs:331-352); serde fills it with its
    // Default when the field is absent (config.rs:33-34)
    bool embedding_enabled = false;
    float embedding_temperature = 1.0f;
    bool embedding_linear = false;

    bool is_3d() const { return depth > 1; }
    size_t grid_size() const { return size_t(width) * height * depth; }
};

// Parses and validates (config.rs:136-164); throws ConfigError.
SimulationConfig parse_config(const std::string& json);
void validate(const SimulationConfig& c);

// ----------------------------------------------------------------- seed ----
// Seed::generate (seed.rs:160-304): returns C planes of depth*height*width.
std::vector<float> generate_seed(const std::string& seed_json, const SimulationConfig& cfg);
// The same into out (channels * width * height * depth floats, zero-filled first).
void generate_seed_into(const std::string& seed_json, const SimulationConfig& cfg, float* out);

// --------------------------------------------------------------- kernel ----
// Kernel::from_config / Kernel3D::from_config (kernel.rs:32-92,
// kernel3d.rs:32-90): the normalised ring-sum stencil, side 2r+1.
template <class R>
struct KernelStencilT {
    int radius = 0;  // r = round(radius * kernel_radius)
    int size = 1;    // 2r+1
    int dims = 2;
    std::vector<R> data;  // size^dims values, row-major
};
using KernelStencil = KernelStencilT<float>;
// R = float (the engine) or double (the FP64 twin); instantiated in schema.cpp.
template <class R>
KernelStencilT<R> build_kernel_t(const KernelConfig& kc, int max_radius, int dims);
KernelStencil build_kernel(const KernelConfig& kc, int max_radius, int dims);

// Kernel::pad_to_size (kernel.rs:98-117, kernel3d.rs:103-133): wrap-padded
// onto the torus; later taps overwrite earlier ones when 2r+1 exceeds a side.
template <class R>
std::vector<R> pad_kernel_t(const KernelStencilT<R>& k, int W, int H, int D);
std::vector<float> pad_kernel(const KernelStencil& k, int W, int H, int D);

}  // namespace flp
