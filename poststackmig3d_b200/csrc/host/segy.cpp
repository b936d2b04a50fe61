// SEG-Y input/output with the reference's layout and rules (src/segy_utils.cpp):
// 3200 B text header, 400 B binary header (dt@16, ns@20, format@24, big-endian), 240 B trace
// headers (INLINE_3D@188, CROSSLINE_3D@192), samples as big-endian IBM (1) or IEEE (5) floats.
// The file is read into memory once; decoding and encoding run in parallel over traces.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <set>

#include "host.hpp"

namespace psmhost {

float ibm_to_ieee(uint32_t ibm) {
    if (ibm == 0) return 0.0f;
    const int sign = (ibm >> 31) & 1;
    const int expo = static_cast<int>((ibm >> 24) & 0x7F) - 64;  // base 16, bias 64
    const uint32_t frac = ibm & 0x00FFFFFFu;
    const double value = std::ldexp(static_cast<double>(frac) / 16777216.0, 4 * expo);
    const float f = static_cast<float>(value);
    return sign ? -f : f;
}

uint32_t ieee_to_ibm(float v) {
    if (v == 0.0f) return 0;  // +0 and -0 both encode as 0
    if (std::isnan(v)) return 0x40000000u;
    const uint32_t sign = v < 0 ? 0x80000000u : 0u;
    if (std::isinf(v)) return sign | 0x7FFFFFFFu;
    if (v < 0) v = -v;
    // normalise to [1/16, 1) by exact multiplications by 16 (segy_utils.cpp:263-265)
    int expo = 64;
    while (v < 1.0f) {
        v *= 16.0f;
        --expo;
    }
    while (v >= 1.0f) {
        v /= 16.0f;
        ++expo;
    }
    const uint32_t frac = static_cast<uint32_t>(v * 16777216.0f) & 0x00FFFFFFu;  // truncate
    return sign | (static_cast<uint32_t>(expo) << 24) | frac;
}

Segy::Segy(const std::string& path, bool quiet) : path_(path) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) throw Error("Cannot open SEGY file: " + path);
    f.seekg(0, std::ios::end);
    const std::streamoff size = f.tellg();
    f.seekg(0);
    raw_.resize(size > 0 ? static_cast<size_t>(size) : 0);
    if (size > 0) f.read(reinterpret_cast<char*>(raw_.data()), size);
    if (raw_.size() < kTextHeader) throw Error("Failed to read text header");
    if (raw_.size() < kTextHeader + kBinaryHeader) throw Error("Failed to read binary header");
    const unsigned char* bh = binary_header();
    dt_us_ = be16(bh + 16);
    if (dt_us_ == 0) throw Error("Sample interval (dt) is zero in binary header");
    dt_s_ = dt_us_ * 1e-6;
    ns_ = be16(bh + 20);
    if (ns_ == 0) throw Error("Number of samples per trace is zero in binary header");
    format_ = be16(bh + 24);
    if (format_ != 1 && format_ != 5) {
        std::cerr << "Warning: Unknown data format code: " << format_
                  << ", assuming IEEE Float (5)" << std::endl;
        format_ = 5;
    }
    const size_t tr = kTraceHeader + 4 * static_cast<size_t>(ns_);
    n_traces_ = static_cast<int64_t>((raw_.size() - kTextHeader - kBinaryHeader) / tr);
    if (n_traces_ == 0) throw Error("No traces found in SEGY file");
    // lookup table (segy_utils.cpp:164-204): zero labels skipped, later duplicates win
    std::set<int32_t> ils, xls;
    lookup_.reserve(static_cast<size_t>(n_traces_));
    for (int64_t i = 0; i < n_traces_; ++i) {
        const unsigned char* h = trace_header(i);
        const int32_t il = static_cast<int32_t>(be32(h + 188));
        const int32_t xl = static_cast<int32_t>(be32(h + 192));
        if (il == 0 || xl == 0) continue;
        lookup_[{il, xl}] = i;
        ils.insert(il);
        xls.insert(xl);
    }
    il_.assign(ils.begin(), ils.end());
    xl_.assign(xls.begin(), xls.end());
    if (!quiet)
        std::cout << "Lookup table created: " << lookup_.size() << " traces, " << il_.size()
                  << " inlines, " << xl_.size() << " crosslines\nData format: " << format_
                  << (format_ == 1 ? " (IBM Float)" : " (IEEE Float)") << std::endl;
}

const unsigned char* Segy::trace_header(int64_t i) const {
    return raw_.data() + kTextHeader + kBinaryHeader +
           static_cast<size_t>(i) * (kTraceHeader + 4 * static_cast<size_t>(ns_));
}

void Segy::read_trace(int64_t i, float* out) const {
    const unsigned char* p = trace_header(i) + kTraceHeader;
    if (format_ == 1) {
        for (int s = 0; s < ns_; ++s) out[s] = ibm_to_ieee(be32(p + 4 * s));
    } else {
        for (int s = 0; s < ns_; ++s) {
            const uint32_t w = be32(p + 4 * s);
            std::memcpy(out + s, &w, 4);
        }
    }
}

void Segy::read_trace_at(int32_t il, int32_t xl, float* out) const {
    auto it = lookup_.find({il, xl});
    if (it == lookup_.end()) {
        std::fill(out, out + ns_, 0.0f);
        return;
    }
    read_trace(it->second, out);
}

void Segy::read_cube(float* cube) const {
    const int64_t n_il = il_.size(), n_xl = xl_.size();
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < n_il * n_xl; ++t)
        read_trace_at(il_[t / n_xl], xl_[t % n_xl], cube + t * ns_);
}

std::vector<int32_t> Segy::record_positions() const {
    std::vector<int32_t> pos(static_cast<size_t>(n_traces_), -1);
    const int64_t n_xl = static_cast<int64_t>(xl_.size());
    for (const auto& kv : lookup_) {
        const int64_t a = std::lower_bound(il_.begin(), il_.end(), kv.first.first) - il_.begin();
        const int64_t b = std::lower_bound(xl_.begin(), xl_.end(), kv.first.second) - xl_.begin();
        pos[static_cast<size_t>(kv.second)] = static_cast<int32_t>(a * n_xl + b);
    }
    return pos;
}

std::vector<int32_t> output_sources(const Segy& in, const std::vector<int32_t>& out_il,
                                    const std::vector<int32_t>& out_xl,
                                    const std::vector<char>& il_is_padding) {
    std::vector<int32_t> src(out_il.size() * out_xl.size(), -1);
    for (size_t o = 0; o < out_il.size(); ++o) {
        if (il_is_padding[o]) continue;
        for (size_t x = 0; x < out_xl.size(); ++x) {
            auto it = in.lookup().find({out_il[o], out_xl[x]});
            if (it != in.lookup().end())
                src[o * out_xl.size() + x] = static_cast<int32_t>(it->second);
        }
    }
    return src;
}

static std::vector<unsigned char> output_file_header(const Segy& in) {
    std::vector<unsigned char> head(kTextHeader + kBinaryHeader);
    std::memcpy(head.data(), in.text_header(), kTextHeader);
    std::memcpy(head.data() + kTextHeader, in.binary_header(), kBinaryHeader);
    put_be16(head.data() + kTextHeader + 20, static_cast<uint16_t>(in.num_samples()));
    put_be16(head.data() + kTextHeader + 24, static_cast<uint16_t>(in.format()));
    return head;
}

void write_output_records(const std::string& path, const Segy& in, const unsigned char* records,
                          size_t n_records) {
    const std::vector<unsigned char> head = output_file_header(in);
    const size_t bytes = n_records * (kTraceHeader + 4 * static_cast<size_t>(in.num_samples()));
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw Error("Cannot create output SEGY file: " + path);
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    ok = ok && std::fwrite(records, 1, bytes, f) == bytes;
    if (std::fclose(f) != 0) ok = false;
    if (!ok) throw Error("Failed to write output SEGY file: " + path);
}

void write_output(const std::string& path, const Segy& in, const std::vector<int32_t>& out_il,
                  const std::vector<int32_t>& out_xl, const std::vector<char>& il_is_padding,
                  const float* image) {
    const size_t ns = static_cast<size_t>(in.num_samples());
    const size_t tr = kTraceHeader + 4 * ns;
    const size_t n_oi = out_il.size(), n_ox = out_xl.size();
    const std::vector<unsigned char> head = output_file_header(in);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw Error("Cannot create output SEGY file: " + path);
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    // one output inline at a time, encoded in parallel
    std::vector<unsigned char> buf(n_ox * tr);
    for (size_t o = 0; o < n_oi && ok; ++o) {
#pragma omp parallel for schedule(static)
        for (int64_t x = 0; x < static_cast<int64_t>(n_ox); ++x) {
            unsigned char* h = buf.data() + x * tr;
            auto it = in.lookup().end();
            if (!il_is_padding[o]) it = in.lookup().find({out_il[o], out_xl[x]});
            if (it != in.lookup().end()) {
                std::memcpy(h, in.trace_header(it->second), kTraceHeader);
            } else {
                std::memset(h, 0, kTraceHeader);
                put_be32(h + 188, static_cast<uint32_t>(out_il[o]));
                put_be32(h + 192, static_cast<uint32_t>(out_xl[x]));
            }
            const float* src = image + (o * n_ox + x) * ns;
            unsigned char* d = h + kTraceHeader;
            for (size_t s = 0; s < ns; ++s) {
                uint32_t w;
                if (in.format() == 1)
                    w = ieee_to_ibm(src[s]);
                else
                    std::memcpy(&w, src + s, 4);
                put_be32(d + 4 * s, w);
            }
        }
        ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) throw Error("Failed to write output SEGY file: " + path);
}

}  // namespace psmhost
