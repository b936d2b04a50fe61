// Vrms providers with the reference's rules (src/velocity_reader.cpp): a positive constant; a
// SEG-Y cube (traces copied when the grid and sampling match, otherwise linear in time and a
// 2x2 inverse-distance blend of the grid neighbours); a text table (inverse-distance blend of
// every point).  They produce the dense Vrms cube that is uploaded once to the GPU.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <iostream>
#include <sstream>

#include "host.hpp"

namespace psmhost {

void VelocityProvider::velocity_iline(int32_t il, const std::vector<int32_t>& xl, size_t n_t,
                                      double dt, float* out) {
    for (size_t x = 0; x < xl.size(); ++x)
        for (size_t t = 0; t < n_t; ++t) out[x * n_t + t] = velocity(il, xl[x], t, dt, n_t);
}

namespace {

class ConstantVelocity final : public VelocityProvider {  // velocity_reader.cpp:12-30
public:
    explicit ConstantVelocity(float v) : v_(v) {
        if (v_ <= 0) throw Error("Velocity must be positive, got: " + std::to_string(v_));
    }
    float velocity(int32_t, int32_t, size_t, double, size_t) override { return v_; }
    void velocity_iline(int32_t, const std::vector<int32_t>& xl, size_t n_t, double,
                        float* out) override {
        std::fill(out, out + xl.size() * n_t, v_);
    }

private:
    float v_;
};

class SegyVelocity final : public VelocityProvider {  // velocity_reader.cpp:33-261
public:
    explicit SegyVelocity(const std::string& path) : f_(path, false) {
        std::cout << "Velocity grid: IL=" << f_.il_labels().size()
                  << ", XL=" << f_.xl_labels().size() << ", T=" << f_.num_samples()
                  << ", dt=" << f_.dt_seconds() << "s" << std::endl;
        n_t_ = f_.num_samples();
        dt_ = f_.dt_seconds();
        times_.resize(n_t_);
        for (size_t i = 0; i < n_t_; ++i) times_[i] = i * dt_;
    }

    float velocity(int32_t il, int32_t xl, size_t t_idx, double dt, size_t) override {
        const double time = t_idx * dt;
        if (has(f_.il_labels(), il) && has(f_.xl_labels(), xl)) {  // :172-197
            std::vector<float> tr(n_t_);
            f_.read_trace_at(il, xl, tr.data());
            return in_time(tr.data(), time);
        }
        return blend(il, xl, time);
    }

    bool assemble_on_gpu(psm_ctx* ctx, const std::vector<int32_t>& il,
                         const std::vector<int32_t>& xl) override {
        const auto& gi = f_.il_labels();
        const auto& gx = f_.xl_labels();
        std::vector<float> grid(gi.size() * gx.size() * n_t_);
        f_.read_cube(grid.data());
        const int rc = psm_set_vrms_grid(ctx, grid.data(), gi.data(), static_cast<int32_t>(gi.size()),
                                         gx.data(), static_cast<int32_t>(gx.size()),
                                         static_cast<int32_t>(n_t_), dt_, il.data(), xl.data());
        if (rc != PSM_OK)
            throw Error(std::string("psm_set_vrms_grid failed: ") + psm_last_error(ctx));
        return true;
    }

    void velocity_iline(int32_t il, const std::vector<int32_t>& xl, size_t n_t, double dt,
                        float* out) override {  // :203-261
        std::fill(out, out + xl.size() * n_t, 0.0f);
        const bool exact_il = has(f_.il_labels(), il);
        std::vector<float> tr(n_t_);
        for (size_t x = 0; x < xl.size(); ++x) {
            float* o = out + x * n_t;
            if (exact_il && has(f_.xl_labels(), xl[x])) {
                if (std::abs(dt - dt_) < 1e-6 && n_t == n_t_) {
                    f_.read_trace_at(il, xl[x], tr.data());
                    std::copy(tr.begin(), tr.begin() + n_t, o);
                } else {
                    for (size_t t = 0; t < n_t; ++t) o[t] = velocity(il, xl[x], t, dt, n_t);
                }
            } else {
                for (size_t t = 0; t < n_t; ++t) o[t] = blend(il, xl[x], t * dt);
            }
        }
    }

private:
    static bool has(const std::vector<int32_t>& v, int32_t x) {
        return std::find(v.begin(), v.end(), x) != v.end();
    }

    // Linear interpolation in time with clamping at both ends (:184-196, :124-138).
    float in_time(const float* tr, double time) const {
        if (time <= times_[0]) return tr[0];
        if (time >= times_[n_t_ - 1]) return tr[n_t_ - 1];
        const double s = time / dt_;
        const size_t lo = static_cast<size_t>(s);
        if (lo >= n_t_ - 1) return tr[n_t_ - 1];
        const double fr = s - lo;
        return static_cast<float>(tr[lo] * (1.0 - fr) + tr[lo + 1] * fr);
    }

    // Nearest label, ties to the lower one (:70-91).
    static size_t nearest(const std::vector<int32_t>& v, int32_t x) {
        if (v.empty()) return 0;
        auto it = std::lower_bound(v.begin(), v.end(), x);
        if (it == v.begin()) return 0;
        if (it == v.end()) return v.size() - 1;
        const size_t i = it - v.begin();
        return std::abs(v[i] - x) < std::abs(v[i - 1] - x) ? i : i - 1;
    }

    // The neighbours one label below and above the nearest one (clamped), weighted by
    // 1 / (1 + |dIL| + |dXL|) in label units (:93-163).
    float blend(int32_t il, int32_t xl, double time) const {
        const auto& L = f_.il_labels();
        const auto& X = f_.xl_labels();
        const size_t ii = nearest(L, il), xi = nearest(X, xl);
        const size_t is[2] = {ii > 0 ? ii - 1 : 0, ii < L.size() - 1 ? ii + 1 : L.size() - 1};
        const size_t xs[2] = {xi > 0 ? xi - 1 : 0, xi < X.size() - 1 ? xi + 1 : X.size() - 1};
        float val[4], w[4];
        std::vector<float> tr(n_t_);
        int n = 0;
        for (size_t a : is)
            for (size_t b : xs) {
                f_.read_trace_at(L[a], X[b], tr.data());
                val[n] = in_time(tr.data(), time);
                const double d_il = std::abs(static_cast<double>(L[a] - il));
                const double d_xl = std::abs(static_cast<double>(X[b] - xl));
                w[n] = 1.0f / (1.0f + static_cast<float>(d_il + d_xl));
                ++n;
            }
        // source order; the reference's -ffast-math build reorders this sum, so results can
        // differ from it in the last bit or two
        float sv = 0.0f, sw = 0.0f;
        for (int i = 0; i < n; ++i) {
            sv += val[i] * w[i];
            sw += w[i];
        }
        return sw > 0 ? sv / sw : val[0];
    }

    Segy f_;
    size_t n_t_ = 0;
    double dt_ = 0.0;
    std::vector<double> times_;
};

class TableVelocity final : public VelocityProvider {  // velocity_reader.cpp:264-370
public:
    explicit TableVelocity(const std::string& path) {
        std::cout << "Reading velocity from table: " << path << std::endl;
        std::ifstream f(path);
        if (!f.is_open()) throw Error("Cannot open velocity table file: " + path);
        std::string line;
        int n = 0;
        while (std::getline(f, line)) {
            ++n;
            if (line.empty() || line[0] == '#') continue;
            std::istringstream is(line);
            Point p;
            if (!(is >> p.il >> p.xl >> p.time >> p.v))
                throw Error("Invalid format at line " + std::to_string(n) +
                            ": expected 4 columns (INLINE CROSSLINE TIME VEL)");
            pts_.push_back(p);
        }
        if (pts_.empty()) throw Error("No valid data found in velocity table");
        vmin_ = vmax_ = pts_[0].v;
        for (const auto& p : pts_) {
            vmin_ = std::min(vmin_, p.v);
            vmax_ = std::max(vmax_, p.v);
        }
        std::cout << "Loaded " << pts_.size() << " velocity points\nVelocity range: " << vmin_
                  << " - " << vmax_ << " m/s" << std::endl;
    }

    // Every point weighted by 1 / (1 + dist), dist mixing label units and seconds; an exact
    // hit returns that point (:320-361).
    float velocity(int32_t il, int32_t xl, size_t t_idx, double dt, size_t) override {
        const double time = t_idx * dt;
        float sv = 0.0f, sw = 0.0f;
        for (const auto& p : pts_) {
            const double a = std::abs(static_cast<double>(p.il - il));
            const double b = std::abs(static_cast<double>(p.xl - xl));
            const double c = std::abs(p.time - time);
            const double d = std::sqrt(a * a + b * b + c * c);
            if (d < 1e-10) return p.v;
            const float w = 1.0f / (1.0f + static_cast<float>(d));
            sv += p.v * w;  // reordered (vectorised) in the reference's -ffast-math build
            sw += w;
        }
        float r = sw > 0 ? sv / sw : vmin_;
        if (r <= 0) r = vmin_;
        return r;
    }

    bool assemble_on_gpu(psm_ctx* ctx, const std::vector<int32_t>& il,
                         const std::vector<int32_t>& xl) override {
        std::vector<int32_t> p_il, p_xl;
        std::vector<double> p_t;
        std::vector<float> p_v;
        for (const auto& p : pts_) {
            p_il.push_back(p.il);
            p_xl.push_back(p.xl);
            p_t.push_back(p.time);
            p_v.push_back(p.v);
        }
        const int rc = psm_set_vrms_table(ctx, p_il.data(), p_xl.data(), p_t.data(), p_v.data(),
                                          static_cast<int32_t>(pts_.size()), il.data(), xl.data());
        if (rc != PSM_OK)
            throw Error(std::string("psm_set_vrms_table failed: ") + psm_last_error(ctx));
        return true;
    }

private:
    struct Point {
        int32_t il = 0, xl = 0;
        double time = 0.0;
        float v = 0.0f;
    };
    std::vector<Point> pts_;
    float vmin_ = 0.0f, vmax_ = 0.0f;
};

// An optional sign, digits and at most one '.' (velocity_reader.cpp:373-396).
bool is_number(const std::string& s) {
    if (s.empty()) return false;
    size_t i = (s[0] == '-' || s[0] == '+') ? 1 : 0;
    bool dot = false;
    for (; i < s.size(); ++i) {
        if (s[i] == '.') {
            if (dot) return false;
            dot = true;
        } else if (!std::isdigit(static_cast<unsigned char>(s[i]))) {
            return false;
        }
    }
    return true;
}

bool is_segy_path(const std::string& p) {  // velocity_reader.cpp:398-403
    std::string l = p;
    std::transform(l.begin(), l.end(), l.begin(), [](unsigned char c) { return std::tolower(c); });
    return l.find(".sgy") != std::string::npos || l.find(".segy") != std::string::npos;
}

}  // namespace

std::unique_ptr<VelocityProvider> make_velocity_provider(const std::string& param) {
    if (is_number(param)) {
        float v;
        try {
            v = std::stof(param);
        } catch (const std::exception& e) {
            throw Error(e.what());
        }
        return std::unique_ptr<VelocityProvider>(new ConstantVelocity(v));
    }
    if (is_segy_path(param)) {
        std::cout << "Reading velocity from SEG-Y: " << param << std::endl;
        return std::unique_ptr<VelocityProvider>(new SegyVelocity(param));
    }
    return std::unique_ptr<VelocityProvider>(new TableVelocity(param));
}

}  // namespace psmhost
