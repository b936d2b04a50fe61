// Internal C++ API of the host surface (libpsm_host.so).  Each piece restates one part of
// sergeevsn/poststackmig3d's host code; the file:line cited next to a function is the
// reference behaviour it keeps.  Errors are thrown as psmhost::Error and turned into
// status codes at the C ABI (host_abi.cpp).
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "psm.h"

namespace psmhost {

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ----------------------------------------------------------------------------- config

struct Config {  // include/config_parser.h:7-20 plus our extra keys
    std::string input_data, output_data;
    double inline_step = 0.0, crossline_step = 0.0;
    int inline_padding = 0, crossline_padding = 0;
    std::string velocity;
    double angle_aperture = 30.0;
    bool amp_correction = true;
    int n_threads = 0;
    int precision = 0;  // 0 f32, 1 bf16, 2 f16
    bool compensated = false;
    bool compat_omp_pad = false;  // trailing padded crosslines as the OpenMP build
    int device = 0;
};

Config parse_config(const std::string& path);  // config_parser.cpp:74-166
void validate_config(const Config& c);         // config_parser.cpp:168-212

// ----------------------------------------------------------------------------- SEG-Y

constexpr size_t kTextHeader = 3200, kBinaryHeader = 400, kTraceHeader = 240;

float ibm_to_ieee(uint32_t ibm);   // segy_utils.cpp:243-254
uint32_t ieee_to_ibm(float v);     // segy_utils.cpp:257-270

inline uint32_t be32(const unsigned char* p) {
    return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3];
}
inline uint16_t be16(const unsigned char* p) { return uint16_t((p[0] << 8) | p[1]); }
inline void put_be32(unsigned char* p, uint32_t v) {
    p[0] = v >> 24; p[1] = v >> 16; p[2] = v >> 8; p[3] = v;
}
inline void put_be16(unsigned char* p, uint16_t v) { p[0] = v >> 8; p[1] = v & 0xff; }

struct PairHash {
    size_t operator()(const std::pair<int32_t, int32_t>& p) const {
        return std::hash<int64_t>()((int64_t(p.first) << 32) ^ uint32_t(p.second));
    }
};
using Lookup = std::unordered_map<std::pair<int32_t, int32_t>, int64_t, PairHash>;

// A SEG-Y file held in memory (the whole file is read once).
class Segy {
public:
    explicit Segy(const std::string& path, bool quiet = false);  // segy_utils.cpp:22-111
    const std::string& path() const { return path_; }
    int64_t num_traces() const { return n_traces_; }
    int num_samples() const { return ns_; }
    int dt_us() const { return dt_us_; }
    double dt_seconds() const { return dt_s_; }
    int format() const { return format_; }
    const unsigned char* text_header() const { return raw_.data(); }
    const unsigned char* binary_header() const { return raw_.data() + kTextHeader; }
    const unsigned char* trace_header(int64_t i) const;
    // Lookup table and sorted unique labels (segy_utils.cpp:152-214).
    const Lookup& lookup() const { return lookup_; }
    const std::vector<int32_t>& il_labels() const { return il_; }
    const std::vector<int32_t>& xl_labels() const { return xl_; }
    // Decode one trace (segy_utils.cpp:272-318); out has num_samples() floats.
    void read_trace(int64_t i, float* out) const;
    // Trace by labels, zeros when absent (segy_utils.cpp:216-240).
    void read_trace_at(int32_t il, int32_t xl, float* out) const;
    // Dense cube [n_il][n_xl][ns] on the sorted labels, missing traces zero.
    void read_cube(float* cube) const;
    // The trace records as they follow the 3600 header bytes (num_traces() records of
    // 240 + 4 num_samples() bytes), and for each the cube trace il_index * n_xl + xl_index it
    // fills, or -1 (zero labels, or a duplicate that a later record overrides).
    const unsigned char* trace_records() const { return trace_header(0); }
    std::vector<int32_t> record_positions() const;

private:
    std::string path_;
    std::vector<unsigned char> raw_;
    int64_t n_traces_ = 0;
    int ns_ = 0, dt_us_ = 0, format_ = 5;
    double dt_s_ = 0.0;
    Lookup lookup_;
    std::vector<int32_t> il_, xl_;
};

// Output file rules of createOutputFile / SegyOutputFile::writeTrace and main.cpp:387-415:
// text header copied; binary header copied with ns@20 and format@24 rewritten; a trace
// keeps the input header when its output inline is a real inline and (IL, XL) exists in
// the input, else gets 240 zero bytes with IL@188, XL@192; samples in the input's format.
void write_output(const std::string& path, const Segy& in,
                  const std::vector<int32_t>& out_il, const std::vector<int32_t>& out_xl,
                  const std::vector<char>& il_is_padding, const float* image);
// The same file from output records already encoded (psm_get_image_segy): the header
// sources of those rules, and the file written around the records.
std::vector<int32_t> output_sources(const Segy& in, const std::vector<int32_t>& out_il,
                                    const std::vector<int32_t>& out_xl,
                                    const std::vector<char>& il_is_padding);
void write_output_records(const std::string& path, const Segy& in, const unsigned char* records,
                          size_t n_records);

// ----------------------------------------------------------------------------- velocity

class VelocityProvider {  // include/velocity_reader.h:11-26
public:
    virtual ~VelocityProvider() = default;
    virtual float velocity(int32_t il, int32_t xl, size_t t_idx, double dt, size_t n_t) = 0;
    // default: per-sample velocity() (velocity_reader.cpp:424-441)
    virtual void velocity_iline(int32_t il, const std::vector<int32_t>& xl, size_t n_t,
                                double dt, float* out /*[n_xl][n_t]*/);
    // Assemble the Vrms cube of ctx's geometry on the GPU (psm_set_vrms_table /
    // psm_set_vrms_grid) with the same arithmetic; false when the provider has no GPU path
    // (the caller then uploads velocity_iline's cube).
    virtual bool assemble_on_gpu(psm_ctx*, const std::vector<int32_t>& /*il*/,
                                 const std::vector<int32_t>& /*xl*/) {
        return false;
    }
};

std::unique_ptr<VelocityProvider> make_velocity_provider(const std::string& param);

// ----------------------------------------------------------------------------- driver

std::vector<int32_t> padded_labels(const std::vector<int32_t>& labels, int pad);
std::vector<int32_t> output_centers(const std::vector<int32_t>& in_labels,
                                    const std::vector<int32_t>& out_labels,
                                    std::vector<char>* is_padding);
float estimate_max_velocity(VelocityProvider& p, const std::vector<int32_t>& il,
                            const std::vector<int32_t>& xl, size_t n_t, double dt);
int max_aperture_il(float max_v, size_t n_t, double dt, float tan2, double inline_step);
float tan2_theta(double angle_deg);

struct Plan {
    int n_il = 0, n_xl = 0, n_t = 0, n_oi = 0, n_ox = 0, m_il = 0;
    float max_v = 0.0f, tan2 = 0.0f;
    double dt = 0.0;
};

void run(const Config& cfg, bool verbose, Plan* plan_only);

}  // namespace psmhost
