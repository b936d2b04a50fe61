// config.txt parsing and validation with the reference's rules
// (src/config_parser.cpp:1-212): key=value lines, '#' comments, whitespace trimmed, one pair
// of matching quotes stripped, the last duplicate key wins, unknown keys ignored.
#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "host.hpp"

namespace psmhost {
namespace {

std::string trim(const std::string& s) {  // config_parser.cpp:25-33
    const char* ws = " \t\n\r";
    size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

std::string unquote(const std::string& s) {  // config_parser.cpp:35-43
    std::string r = trim(s);
    if (r.size() >= 2 && ((r.front() == '"' && r.back() == '"') ||
                          (r.front() == '\'' && r.back() == '\'')))
        return r.substr(1, r.size() - 2);
    return r;
}

bool to_bool(const std::string& v) {  // config_parser.cpp:45-57
    std::string l = v;
    std::transform(l.begin(), l.end(), l.begin(), [](unsigned char c) { return std::tolower(c); });
    l = trim(l);
    if (l == "true" || l == "1" || l == "yes" || l == "on") return true;
    if (l == "false" || l == "0" || l == "no" || l == "off") return false;
    throw Error("Cannot parse boolean value: " + v);
}

// std::stod / std::stoi semantics: a leading number is taken, trailing text ignored.
double to_double(const std::string& v) {  // config_parser.cpp:59-65
    try {
        return std::stod(v);
    } catch (const std::exception&) {
        throw Error("Cannot parse double value: " + v);
    }
}

int to_int(const std::string& v) {  // config_parser.cpp:67-73
    try {
        return std::stoi(v);
    } catch (const std::exception&) {
        throw Error("Cannot parse int value: " + v);
    }
}

}  // namespace

Config parse_config(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) throw Error("Config file not found: " + path);
    std::map<std::string, std::string> kv;
    std::string line;
    int n = 0;
    while (std::getline(f, line)) {
        ++n;
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        size_t eq = line.find('=');
        if (eq == std::string::npos)
            throw Error("Invalid format at line " + std::to_string(n) +
                        ": expected key=value, got: " + line);
        kv[trim(line.substr(0, eq))] = unquote(trim(line.substr(eq + 1)));
    }
    std::vector<std::string> missing;
    for (const char* k : {"input_data", "output_data", "inline_step", "crossline_step",
                          "velocity"})
        if (!kv.count(k)) missing.push_back(k);
    if (!missing.empty()) {
        std::string msg = "Missing required parameters: ";
        for (size_t i = 0; i < missing.size(); ++i) msg += (i ? ", " : "") + missing[i];
        throw Error(msg);
    }
    Config c;
    try {
        c.input_data = kv["input_data"];
        c.output_data = kv["output_data"];
        c.inline_step = to_double(kv["inline_step"]);
        c.crossline_step = to_double(kv["crossline_step"]);
        c.velocity = kv["velocity"];
        if (kv.count("inline_padding")) c.inline_padding = to_int(kv["inline_padding"]);
        if (kv.count("crossline_padding")) c.crossline_padding = to_int(kv["crossline_padding"]);
        if (kv.count("angle_aperture")) c.angle_aperture = to_double(kv["angle_aperture"]);
        if (kv.count("amp_correction")) c.amp_correction = to_bool(kv["amp_correction"]);
        if (kv.count("n_threads")) c.n_threads = to_int(kv["n_threads"]);
        // keys beyond the reference's
        if (kv.count("precision")) {
            std::string p = kv["precision"];
            std::transform(p.begin(), p.end(), p.begin(),
                           [](unsigned char ch) { return std::tolower(ch); });
            if (p == "f32" || p == "fp32" || p == "float32") c.precision = 0;
            else if (p == "bf16" || p == "bfloat16") c.precision = 1;
            else if (p == "f16" || p == "fp16" || p == "float16") c.precision = 2;
            else throw Error("Cannot parse precision value: " + kv["precision"]);
        }
        if (kv.count("compensated")) c.compensated = to_bool(kv["compensated"]);
        if (kv.count("compat_omp_pad")) c.compat_omp_pad = to_bool(kv["compat_omp_pad"]);
        if (kv.count("device")) c.device = to_int(kv["device"]);
    } catch (const Error& e) {
        throw Error(std::string("Error parsing config values: ") + e.what());
    }
    return c;
}

void validate_config(const Config& c) {
    if (c.inline_step <= 0)
        throw Error("inline_step must be positive, got: " + std::to_string(c.inline_step));
    if (c.crossline_step <= 0)
        throw Error("crossline_step must be positive, got: " + std::to_string(c.crossline_step));
    if (c.inline_padding < 0)
        throw Error("inline_padding must be non-negative, got: " +
                    std::to_string(c.inline_padding));
    if (c.crossline_padding < 0)
        throw Error("crossline_padding must be non-negative, got: " +
                    std::to_string(c.crossline_padding));
    if (c.angle_aperture <= 0 || c.angle_aperture >= 90)
        throw Error("angle_aperture must be in range (0, 90), got: " +
                    std::to_string(c.angle_aperture));
    if (c.n_threads < 0)
        throw Error("n_threads must be non-negative (0 = use all available), got: " +
                    std::to_string(c.n_threads));
    // config_parser.cpp:201-211 checks a numeric velocity inside a try whose catch also
    // swallows its own "must be positive" error, so nothing is rejected here; a non-positive
    // constant fails when the provider is built (velocity_reader.cpp:12-18).
}

}  // namespace psmhost
