// bsnn_config.hpp -- the reference's JSON run configuration: the same flat schema, defaults,
// per-connection prefix overrides, output-directory path prefixing and checks as
// cpp_src/core/config.{h,cpp} (struct Config, config.h:10-154; load_config_json, config.cpp:68-318),
// with a small JSON reader of this project's own instead of the reference's third-party one.
//
// Semantics kept from the reference loader:
//  * a missing key keeps its default; a present key must have the field's JSON type (numbers
//    convert between integer and floating types as a C++ cast does; a wrong type throws);
//  * the global weight-generation keys (e_max_weight_value, max_connection_distance, ...) are
//    copied into all four per-connection parameter sets, then "<prefix>_<field>" keys override
//    them per connection (prefixes e_to_e, e_to_i, i_to_e, i_to_i; config.cpp:13-44, 132-166);
//  * weights_*_filename falls back to the legacy key weights_* (config.cpp:169-172);
//  * relative output paths are joined to output_directory unless their first component already
//    equals output_directory's first component (config.cpp:46-66, 291-301);
//  * array keys must be arrays; id / step arrays must hold non-negative integers; the checks of
//    config.cpp:202-316 raise std::runtime_error with the same messages.
#pragma once

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace bsnn {

// ---- a minimal JSON document model ---------------------------------------------------------------
class Json {
public:
    enum class Type { Null, Bool, Int, Uint, Float, String, Array, Object };

    Type type = Type::Null;
    bool b = false;
    int64_t i = 0;
    uint64_t u = 0;
    double d = 0.0;
    std::string s;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;  // in document order; later duplicates win

    bool is_object() const { return type == Type::Object; }
    bool is_array() const { return type == Type::Array; }
    bool is_number() const { return type == Type::Int || type == Type::Uint || type == Type::Float; }
    bool is_number_integer() const { return type == Type::Int || type == Type::Uint; }
    bool is_number_unsigned() const { return type == Type::Uint; }

    const Json* find(const std::string& key) const {
        const Json* hit = nullptr;
        for (const auto& kv : obj)
            if (kv.first == key) hit = &kv.second;
        return hit;
    }
    bool contains(const std::string& key) const { return is_object() && find(key) != nullptr; }

    template <class T>
    T get() const;

    // obj.value(key, default): the default when the key is missing, else the converted value.
    template <class T>
    T value(const std::string& key, const T& fallback) const {
        const Json* v = is_object() ? find(key) : nullptr;
        return v ? v->get<T>() : fallback;
    }

    static Json parse(const std::string& text);
};

namespace json_detail {

inline const char* type_name(Json::Type t) {
    switch (t) {
        case Json::Type::Null: return "null";
        case Json::Type::Bool: return "boolean";
        case Json::Type::Int:
        case Json::Type::Uint:
        case Json::Type::Float: return "number";
        case Json::Type::String: return "string";
        case Json::Type::Array: return "array";
        default: return "object";
    }
}

class Reader {
public:
    explicit Reader(const std::string& t) : t_(t) {}

    Json document() {
        Json v = value();
        ws();
        if (p_ != t_.size()) fail("unexpected trailing characters");
        return v;
    }

private:
    [[noreturn]] void fail(const std::string& what) const {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < p_ && k < t_.size(); ++k) {
            if (t_[k] == '\n') {
                ++line;
                col = 1;
            } else {
                ++col;
            }
        }
        throw std::runtime_error("JSON parse error: " + what + " at line " + std::to_string(line) + ", column " +
                                 std::to_string(col));
    }
    void ws() {
        while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\t' || t_[p_] == '\n' || t_[p_] == '\r')) ++p_;
    }
    bool eat(char c) {
        ws();
        if (p_ < t_.size() && t_[p_] == c) {
            ++p_;
            return true;
        }
        return false;
    }
    void expect(char c) {
        if (!eat(c)) fail(std::string("expected '") + c + "'");
    }
    bool word(const char* w) {
        const size_t n = std::char_traits<char>::length(w);
        if (t_.compare(p_, n, w) == 0) {
            p_ += n;
            return true;
        }
        return false;
    }
    static void put_utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += static_cast<char>(cp);
        } else if (cp < 0x800) {
            out += static_cast<char>(0xC0 | (cp >> 6));
            out += static_cast<char>(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += static_cast<char>(0xE0 | (cp >> 12));
            out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
            out += static_cast<char>(0x80 | (cp & 0x3F));
        } else {
            out += static_cast<char>(0xF0 | (cp >> 18));
            out += static_cast<char>(0x80 | ((cp >> 12) & 0x3F));
            out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
            out += static_cast<char>(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (p_ + 4 > t_.size()) fail("truncated \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = t_[p_++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= static_cast<uint32_t>(c - '0');
            else if (c >= 'a' && c <= 'f') v |= static_cast<uint32_t>(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= static_cast<uint32_t>(c - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string string_body() {
        std::string out;
        for (;;) {
            if (p_ >= t_.size()) fail("unterminated string");
            const char c = t_[p_++];
            if (c == '"') return out;
            if (static_cast<unsigned char>(c) < 0x20) fail("control character in string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (p_ >= t_.size()) fail("unterminated escape");
            const char e = t_[p_++];
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
                    uint32_t cp = hex4();
                    if (cp >= 0xD800 && cp <= 0xDBFF) {  // a surrogate pair
                        if (!(word("\\u"))) fail("lone high surrogate");
                        const uint32_t lo = hex4();
                        if (lo < 0xDC00 || lo > 0xDFFF) fail("bad low surrogate");
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    }
                    put_utf8(out, cp);
                    break;
                }
                default: fail("bad escape");
            }
        }
    }
    Json number() {
        const size_t b = p_;
        bool integral = true;
        if (t_[p_] == '-') ++p_;
        if (p_ >= t_.size() || !std::isdigit(static_cast<unsigned char>(t_[p_]))) fail("bad number");
        if (t_[p_] == '0') {
            ++p_;
        } else {
            while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) ++p_;
        }
        if (p_ < t_.size() && t_[p_] == '.') {
            integral = false;
            ++p_;
            if (p_ >= t_.size() || !std::isdigit(static_cast<unsigned char>(t_[p_]))) fail("bad number");
            while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) ++p_;
        }
        if (p_ < t_.size() && (t_[p_] == 'e' || t_[p_] == 'E')) {
            integral = false;
            ++p_;
            if (p_ < t_.size() && (t_[p_] == '+' || t_[p_] == '-')) ++p_;
            if (p_ >= t_.size() || !std::isdigit(static_cast<unsigned char>(t_[p_]))) fail("bad number");
            while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) ++p_;
        }
        const std::string lit = t_.substr(b, p_ - b);
        Json v;
        if (integral) {
            errno = 0;
            if (lit[0] == '-') {
                const long long x = std::strtoll(lit.c_str(), nullptr, 10);
                if (errno == 0) {
                    v.type = Json::Type::Int;
                    v.i = x;
                    v.d = static_cast<double>(x);
                    return v;
                }
            } else {
                const unsigned long long x = std::strtoull(lit.c_str(), nullptr, 10);
                if (errno == 0) {
                    v.type = Json::Type::Uint;
                    v.u = x;
                    v.i = static_cast<int64_t>(x);
                    v.d = static_cast<double>(x);
                    return v;
                }
            }
        }
        v.type = Json::Type::Float;
        v.d = std::strtod(lit.c_str(), nullptr);
        return v;
    }
    Json value() {
        ws();
        if (p_ >= t_.size()) fail("unexpected end of input");
        const char c = t_[p_];
        Json v;
        if (c == '{') {
            ++p_;
            v.type = Json::Type::Object;
            if (eat('}')) return v;
            do {
                ws();
                if (p_ >= t_.size() || t_[p_] != '"') fail("expected a key string");
                ++p_;
                std::string key = string_body();
                expect(':');
                v.obj.emplace_back(std::move(key), value());
            } while (eat(','));
            expect('}');
            return v;
        }
        if (c == '[') {
            ++p_;
            v.type = Json::Type::Array;
            if (eat(']')) return v;
            do {
                v.arr.push_back(value());
            } while (eat(','));
            expect(']');
            return v;
        }
        if (c == '"') {
            ++p_;
            v.type = Json::Type::String;
            v.s = string_body();
            return v;
        }
        if (word("true")) {
            v.type = Json::Type::Bool;
            v.b = true;
            return v;
        }
        if (word("false")) {
            v.type = Json::Type::Bool;
            return v;
        }
        if (word("null")) return v;
        if (c == '-' || std::isdigit(static_cast<unsigned char>(c))) return number();
        fail("unexpected character");
    }

    const std::string& t_;
    size_t p_ = 0;
};

// A number (or a boolean, as 0 / 1) converted as a C++ cast converts it.
template <class T>
T number_as(const Json& j) {
    if (j.type == Json::Type::Bool) return static_cast<T>(j.b);
    if (!j.is_number()) throw std::runtime_error(std::string("type must be number, but is ") + type_name(j.type));
    if (j.type == Json::Type::Uint) return static_cast<T>(j.u);
    if (j.type == Json::Type::Int) return static_cast<T>(j.i);
    return static_cast<T>(j.d);
}

}  // namespace json_detail

inline Json Json::parse(const std::string& text) { return json_detail::Reader(text).document(); }

template <>
inline float Json::get<float>() const { return json_detail::number_as<float>(*this); }
template <>
inline double Json::get<double>() const { return json_detail::number_as<double>(*this); }
template <>
inline int Json::get<int>() const { return json_detail::number_as<int>(*this); }
template <>
inline uint32_t Json::get<uint32_t>() const { return json_detail::number_as<uint32_t>(*this); }
template <>
inline bool Json::get<bool>() const {
    if (type != Type::Bool) throw std::runtime_error(std::string("type must be boolean, but is ") + json_detail::type_name(type));
    return b;
}
template <>
inline std::string Json::get<std::string>() const {
    if (type != Type::String) throw std::runtime_error(std::string("type must be string, but is ") + json_detail::type_name(type));
    return s;
}
template <>
inline std::vector<float> Json::get<std::vector<float>>() const {
    if (type != Type::Array) throw std::runtime_error(std::string("type must be array, but is ") + json_detail::type_name(type));
    std::vector<float> out;
    for (const auto& e : arr) out.push_back(e.get<float>());
    return out;
}
template <>
inline std::vector<uint32_t> Json::get<std::vector<uint32_t>>() const {
    if (type != Type::Array) throw std::runtime_error(std::string("type must be array, but is ") + json_detail::type_name(type));
    std::vector<uint32_t> out;
    for (const auto& e : arr) out.push_back(e.get<uint32_t>());
    return out;
}

// ---- the run configuration -----------------------------------------------------------------------

// generate_weights::WeightGenerationParams (cpp_src/generation/generate_weights.h:8-18).
struct WeightGenerationParams {
    float x_location_length;
    float y_location_length;
    float max_distance;
    float spread_scale;
    float max_weight_value;
    bool weight_value_normal_dropoff;
    bool probabilistic_normal_not_uniform;
    float probability_multiplier;
    bool no_diagonal_connections;
};

// struct Config (cpp_src/core/config.h:10-154): same field names, types and defaults.
struct Config {
    uint32_t simulation_steps = 10000;
    std::string output_directory = "../data/buryn_data/buryn_outputs_";
    std::string description;
    int rng_seed = 314;
    float timestep = 1e-4f;

    uint32_t num_excitatory_neurons = 100;
    uint32_t num_inhibitory_neurons = 100;
    float g_leak = 0.05e-6f;
    float membrane_capacitance = 1.0e-9f;
    float depolarization_slope_factor = 0.0065625f;
    float v_effective_spike_threshold = -0.0606250f;
    float v_excitatory_reversal = 0.0f;
    float v_inhibitory_reversal = -0.08f;
    float v_threshold = -0.04f;
    float v_reset = -0.06f;
    float v_rest = -0.07f;
    uint32_t refractory_steps = 50;

    float group_e_mean_background_excitatory_spikes = 0.0f;
    float group_e_mean_background_inhibitory_spikes = 0.0f;
    float group_e_background_excitatory_postsynaptic_r_trace_decay = 0.0f;
    float group_e_background_excitatory_postsynaptic_d_trace_decay = 0.0f;
    float group_e_background_inhibitory_postsynaptic_r_trace_decay = 0.0f;
    float group_e_background_inhibitory_postsynaptic_d_trace_decay = 0.0f;
    float group_e_background_excitatory_scaling_factor = 0.0f;
    float group_e_background_inhibitory_scaling_factor = 0.0f;
    float group_i_mean_background_excitatory_spikes = 0.0f;
    float group_i_mean_background_inhibitory_spikes = 0.0f;
    float group_i_background_excitatory_postsynaptic_r_trace_decay = 0.0f;
    float group_i_background_excitatory_postsynaptic_d_trace_decay = 0.0f;
    float group_i_background_inhibitory_postsynaptic_r_trace_decay = 0.0f;
    float group_i_background_inhibitory_postsynaptic_d_trace_decay = 0.0f;
    float group_i_background_excitatory_scaling_factor = 0.0f;
    float group_i_background_inhibitory_scaling_factor = 0.0f;

    std::string excitatory_locations_file = "../data/buryn_data/buryn_outputs_/locations/group_e_locations.txt";
    std::string inhibitory_locations_file = "../data/buryn_data/buryn_outputs_/locations/group_i_locations.txt";
    float excitatory_location_spacing = 1.0f;
    float inhibitory_location_spacing = 2.0f;
    uint32_t excitatory_side_points = 10;
    uint32_t inhibitory_side_points = 10;
    float side_length = 10.0f;

    float e_max_weight_value = 0.2235e-9f;
    float i_max_weight_value = 0.0578e-9f;
    float max_connection_distance = 3.0f;
    float connection_spread_scale = 1.0f;
    float connection_probability_multiplier = 1.0f;
    WeightGenerationParams weight_generation_params_e_to_e = {10.0f, 10.0f, 3.0f, 1.0f, 0.2235e-9f, false, true, 1.0f, true};
    WeightGenerationParams weight_generation_params_e_to_i = {10.0f, 10.0f, 3.0f, 1.0f, 0.2235e-9f, false, true, 1.0f, false};
    WeightGenerationParams weight_generation_params_i_to_e = {10.0f, 10.0f, 3.0f, 1.0f, 0.0578e-9f, false, false, 1.0f, false};
    WeightGenerationParams weight_generation_params_i_to_i = {10.0f, 10.0f, 3.0f, 1.0f, 0.0578e-9f, false, false, 1.0f, false};

    std::string weights_e_to_i_filename = "../data/buryn_data/buryn_outputs_/weights/weights_e_to_i.txt";
    std::string weights_i_to_e_filename = "../data/buryn_data/buryn_outputs_/weights/weights_i_to_e.txt";
    std::string weights_e_to_e_filename = "../data/buryn_data/buryn_outputs_/weights/weights_e_to_e.txt";
    std::string weights_i_to_i_filename = "../data/buryn_data/buryn_outputs_/weights/weights_i_to_i.txt";
    float tau_decay_e = 2e-3f;
    float tau_rise_e = 0.3e-3f;
    float tau_decay_i = 3e-3f;
    float tau_rise_i = 0.3e-3f;
    float postsynaptic_kernel_normalization_value = 1.0f;

    bool e_e_plasticity_enabled = true;
    float e_e_plasticity_ltp_A = 1.0e-12f;
    float e_e_plasticity_ltd_A = 1.0e-12f;
    float e_e_plasticity_ltp_B = 1.0e-12f;
    float e_e_plasticity_ltd_B = 1.0e-12f;
    float e_e_plasticity_tau_ltp = 0.02f;
    float e_e_plasticity_tau_ltd = 0.02f;
    float e_e_plasticity_triplet_tau_ltp = 0.02f;
    float e_e_plasticity_triplet_tau_ltd = 0.02f;
    float e_e_plasticity_weight_min = 0.0f;
    float e_e_plasticity_weight_max = 0.2235e-9f;
    bool i_e_plasticity_enabled = true;
    float i_e_plasticity_ltp_A = 1.0e-12f;
    float i_e_plasticity_ltd_A = 1.0e-12f;
    float i_e_plasticity_ltd_B = 1.0e-12f;
    float i_e_plasticity_tau_ltp = 0.02f;
    float i_e_plasticity_tau_ltd = 0.02f;
    float i_e_plasticity_weight_min = 0.0f;
    float i_e_plasticity_weight_max = 0.2235e-9f;

    std::vector<float> stimulus_input_values = {0.25e-9f};
    std::string stimulus_schedules_folder = "../data/buryn_data/buryn_outputs_/stimulus_schedules";
    std::vector<uint32_t> stimulus_selected_input_ids = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9};
    std::vector<uint32_t> stimulus_selected_input_post_group_offsets = std::vector<uint32_t>(10, 0);
    std::vector<uint32_t> stimulus_start_clock_steps = {5000};
    std::vector<uint32_t> stimulus_end_clock_steps = {6000};

    std::string e_spike_recording_file = "../data/buryn_data/buryn_outputs_/recordings/spikes_e.txt";
    std::string i_spike_recording_file = "../data/buryn_data/buryn_outputs_/recordings/spikes_i.txt";
    std::string voltage_recording_file = "../data/buryn_data/buryn_outputs_/recordings/voltages_step0.txt";
    std::vector<uint32_t> voltage_recording_neuron_ids = {10, 426};
    std::string e_e_weight_recording_file = "../data/buryn_data/buryn_outputs_/weights/weights_e_to_e_recordings.txt";
};

namespace config_detail {

inline void weight_overrides(WeightGenerationParams& p, const Json& j, const std::string& prefix) {
    p.max_weight_value = j.value(prefix + "_max_weight_value", p.max_weight_value);
    p.max_distance = j.value(prefix + "_max_distance", p.max_distance);
    p.spread_scale = j.value(prefix + "_spread_scale", p.spread_scale);
    p.weight_value_normal_dropoff = j.value(prefix + "_weight_value_normal_dropoff", p.weight_value_normal_dropoff);
    p.probabilistic_normal_not_uniform =
        j.value(prefix + "_probabilistic_normal_not_uniform", p.probabilistic_normal_not_uniform);
    p.probability_multiplier = j.value(prefix + "_probability_multiplier", p.probability_multiplier);
    p.no_diagonal_connections = j.value(prefix + "_no_diagonal_connections", p.no_diagonal_connections);
    p.x_location_length = j.value(prefix + "_x_location_length", p.x_location_length);
    p.y_location_length = j.value(prefix + "_y_location_length", p.y_location_length);
}

// A relative path under output_directory, unless it already starts at the directory's first
// component (so configs may name paths either way).
inline std::string prefix_output_path(const std::string& output_directory, const std::string& value) {
    if (value.empty()) return value;
    const std::filesystem::path path(value);
    if (path.is_absolute()) return value;
    const std::filesystem::path dir(output_directory);
    if (!output_directory.empty()) {
        auto pi = path.begin();
        auto di = dir.begin();
        if (pi != path.end() && di != dir.end() && *pi == *di) return value;
    }
    return (dir / path).lexically_normal().string();
}

// An array key whose elements must be non-negative integers.
inline void read_ids(const Json& j, const std::string& key, std::vector<uint32_t>& out) {
    if (!j.contains(key)) return;
    const Json& a = *j.find(key);
    if (!a.is_array()) throw std::runtime_error(key + " must be an array");
    for (const auto& e : a.arr) {
        if (!e.is_number_unsigned() && !e.is_number_integer()) throw std::runtime_error(key + " must contain only integers");
        if (e.is_number_integer() && e.i < 0) throw std::runtime_error(key + " must not contain negative values");
    }
    out = a.get<std::vector<uint32_t>>();
}

}  // namespace config_detail

// load_config_json (cpp_src/core/config.cpp:68-318).
inline Config load_config_json(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Failed to open config file: " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    const Json j = Json::parse(ss.str());
    if (!j.is_object()) throw std::runtime_error("Config JSON must be an object at the top level");

    Config c;
#define BSNN_CFG(field) c.field = j.value(#field, c.field)
    BSNN_CFG(simulation_steps);
    BSNN_CFG(output_directory);
    BSNN_CFG(description);
    BSNN_CFG(rng_seed);
    BSNN_CFG(timestep);
    BSNN_CFG(num_excitatory_neurons);
    BSNN_CFG(num_inhibitory_neurons);
    BSNN_CFG(g_leak);
    BSNN_CFG(membrane_capacitance);
    BSNN_CFG(depolarization_slope_factor);
    BSNN_CFG(v_effective_spike_threshold);
    BSNN_CFG(v_excitatory_reversal);
    BSNN_CFG(v_inhibitory_reversal);
    BSNN_CFG(v_threshold);
    BSNN_CFG(v_reset);
    BSNN_CFG(v_rest);
    BSNN_CFG(refractory_steps);
    BSNN_CFG(group_e_mean_background_excitatory_spikes);
    BSNN_CFG(group_e_mean_background_inhibitory_spikes);
    BSNN_CFG(group_e_background_excitatory_postsynaptic_r_trace_decay);
    BSNN_CFG(group_e_background_excitatory_postsynaptic_d_trace_decay);
    BSNN_CFG(group_e_background_inhibitory_postsynaptic_r_trace_decay);
    BSNN_CFG(group_e_background_inhibitory_postsynaptic_d_trace_decay);
    BSNN_CFG(group_e_background_excitatory_scaling_factor);
    BSNN_CFG(group_e_background_inhibitory_scaling_factor);
    BSNN_CFG(group_i_mean_background_excitatory_spikes);
    BSNN_CFG(group_i_mean_background_inhibitory_spikes);
    BSNN_CFG(group_i_background_excitatory_postsynaptic_r_trace_decay);
    BSNN_CFG(group_i_background_excitatory_postsynaptic_d_trace_decay);
    BSNN_CFG(group_i_background_inhibitory_postsynaptic_r_trace_decay);
    BSNN_CFG(group_i_background_inhibitory_postsynaptic_d_trace_decay);
    BSNN_CFG(group_i_background_excitatory_scaling_factor);
    BSNN_CFG(group_i_background_inhibitory_scaling_factor);
    BSNN_CFG(excitatory_locations_file);
    BSNN_CFG(inhibitory_locations_file);
    BSNN_CFG(excitatory_location_spacing);
    BSNN_CFG(inhibitory_location_spacing);
    BSNN_CFG(excitatory_side_points);
    BSNN_CFG(inhibitory_side_points);
    BSNN_CFG(side_length);
    BSNN_CFG(e_max_weight_value);
    BSNN_CFG(i_max_weight_value);
    BSNN_CFG(max_connection_distance);
    BSNN_CFG(connection_spread_scale);
    BSNN_CFG(connection_probability_multiplier);
    // the global generation keys go to all four connections, then the prefixed keys override them
    WeightGenerationParams* per_conn[4] = {&c.weight_generation_params_e_to_e, &c.weight_generation_params_e_to_i,
                                           &c.weight_generation_params_i_to_e, &c.weight_generation_params_i_to_i};
    for (int k = 0; k < 4; ++k) {
        WeightGenerationParams& p = *per_conn[k];
        p.max_weight_value = k < 2 ? c.e_max_weight_value : c.i_max_weight_value;
        p.max_distance = c.max_connection_distance;
        p.spread_scale = c.connection_spread_scale;
        p.probability_multiplier = c.connection_probability_multiplier;
        p.x_location_length = c.side_length;
        p.y_location_length = c.side_length;
    }
    config_detail::weight_overrides(c.weight_generation_params_e_to_e, j, "e_to_e");
    config_detail::weight_overrides(c.weight_generation_params_e_to_i, j, "e_to_i");
    config_detail::weight_overrides(c.weight_generation_params_i_to_e, j, "i_to_e");
    config_detail::weight_overrides(c.weight_generation_params_i_to_i, j, "i_to_i");
    c.weights_e_to_i_filename = j.value("weights_e_to_i_filename", j.value("weights_e_to_i", c.weights_e_to_i_filename));
    c.weights_i_to_e_filename = j.value("weights_i_to_e_filename", j.value("weights_i_to_e", c.weights_i_to_e_filename));
    c.weights_e_to_e_filename = j.value("weights_e_to_e_filename", j.value("weights_e_to_e", c.weights_e_to_e_filename));
    c.weights_i_to_i_filename = j.value("weights_i_to_i_filename", j.value("weights_i_to_i", c.weights_i_to_i_filename));
    BSNN_CFG(tau_decay_e);
    BSNN_CFG(tau_rise_e);
    BSNN_CFG(tau_decay_i);
    BSNN_CFG(tau_rise_i);
    BSNN_CFG(postsynaptic_kernel_normalization_value);
    BSNN_CFG(e_e_plasticity_enabled);
    BSNN_CFG(e_e_plasticity_ltp_A);
    BSNN_CFG(e_e_plasticity_ltd_A);
    BSNN_CFG(e_e_plasticity_ltp_B);
    BSNN_CFG(e_e_plasticity_ltd_B);
    BSNN_CFG(e_e_plasticity_tau_ltp);
    BSNN_CFG(e_e_plasticity_tau_ltd);
    BSNN_CFG(e_e_plasticity_triplet_tau_ltp);
    BSNN_CFG(e_e_plasticity_triplet_tau_ltd);
    BSNN_CFG(e_e_plasticity_weight_min);
    BSNN_CFG(e_e_plasticity_weight_max);
    BSNN_CFG(i_e_plasticity_enabled);
    BSNN_CFG(i_e_plasticity_ltp_A);
    BSNN_CFG(i_e_plasticity_ltd_A);
    BSNN_CFG(i_e_plasticity_ltd_B);
    BSNN_CFG(i_e_plasticity_tau_ltp);
    BSNN_CFG(i_e_plasticity_tau_ltd);
    BSNN_CFG(i_e_plasticity_weight_min);
    BSNN_CFG(i_e_plasticity_weight_max);
    if (j.contains("stimulus_input_values")) {
        const Json& a = *j.find("stimulus_input_values");
        if (!a.is_array()) throw std::runtime_error("stimulus_input_values must be an array");
        c.stimulus_input_values = a.get<std::vector<float>>();
    }
    BSNN_CFG(stimulus_schedules_folder);
    config_detail::read_ids(j, "stimulus_selected_input_ids", c.stimulus_selected_input_ids);
    config_detail::read_ids(j, "stimulus_selected_input_post_group_offsets", c.stimulus_selected_input_post_group_offsets);
    config_detail::read_ids(j, "stimulus_start_clock_steps", c.stimulus_start_clock_steps);
    config_detail::read_ids(j, "stimulus_end_clock_steps", c.stimulus_end_clock_steps);
    BSNN_CFG(e_spike_recording_file);
    BSNN_CFG(i_spike_recording_file);
    BSNN_CFG(voltage_recording_file);
    config_detail::read_ids(j, "voltage_recording_neuron_ids", c.voltage_recording_neuron_ids);
    BSNN_CFG(e_e_weight_recording_file);
#undef BSNN_CFG

    const std::string& od = c.output_directory;
    for (std::string* p : {&c.excitatory_locations_file, &c.inhibitory_locations_file, &c.weights_e_to_i_filename,
                           &c.weights_i_to_e_filename, &c.weights_e_to_e_filename, &c.weights_i_to_i_filename,
                           &c.stimulus_schedules_folder, &c.e_spike_recording_file, &c.i_spike_recording_file,
                           &c.voltage_recording_file, &c.e_e_weight_recording_file})
        *p = config_detail::prefix_output_path(od, *p);

    if (c.stimulus_selected_input_post_group_offsets.empty())
        c.stimulus_selected_input_post_group_offsets.assign(c.stimulus_selected_input_ids.size(), 0);
    if (c.stimulus_selected_input_post_group_offsets.size() != c.stimulus_selected_input_ids.size())
        throw std::runtime_error(
            "stimulus_selected_input_post_group_offsets size must match stimulus_selected_input_ids size");
    if (c.num_excitatory_neurons == 0 || c.num_inhibitory_neurons == 0)
        throw std::runtime_error("Neuron counts must be > 0");
    if (c.membrane_capacitance <= 0.0f) throw std::runtime_error("membrane_capacitance must be > 0");
    return c;
}

}  // namespace bsnn
