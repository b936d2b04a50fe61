// extern "C" face of the host surface (include/psm_host.h).  Exceptions stop here and become
// status codes plus the message the reference prints after "Error: " (main.cpp:438-441).
#include <cstring>
#include <exception>
#include <string>

#include "host.hpp"
#include "psm.h"
#include "psm_host.h"

using namespace psmhost;

namespace {

void set_err(char* err, size_t len, const std::string& m) {
    if (!err || !len) return;
    std::strncpy(err, m.c_str(), len - 1);
    err[len - 1] = '\0';
}

void copy_str(char* dst, size_t n, const std::string& s) {
    std::strncpy(dst, s.c_str(), n - 1);
    dst[n - 1] = '\0';
}

template <class F>
int guarded(char* err, size_t len, F&& f) {
    set_err(err, len, "");
    try {
        f();
        return PSM_OK;
    } catch (const Error& e) {
        set_err(err, len, e.what());
        return PSM_ERR_ARG;
    } catch (const std::bad_alloc&) {
        set_err(err, len, "host allocation failed");
        return PSM_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_err(err, len, e.what());
        return PSM_ERR_ARG;
    }
}

}  // namespace

extern "C" {

int psm_config_load(const char* path, psm_config* out, char* err, size_t err_len) {
    if (!path || !out) return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        Config c = parse_config(path);
        validate_config(c);
        std::memset(out, 0, sizeof(*out));
        copy_str(out->input_data, sizeof(out->input_data), c.input_data);
        copy_str(out->output_data, sizeof(out->output_data), c.output_data);
        copy_str(out->velocity, sizeof(out->velocity), c.velocity);
        out->inline_step = c.inline_step;
        out->crossline_step = c.crossline_step;
        out->inline_padding = c.inline_padding;
        out->crossline_padding = c.crossline_padding;
        out->angle_aperture = c.angle_aperture;
        out->amp_correction = c.amp_correction;
        out->n_threads = c.n_threads;
        out->precision = c.precision;
        out->compensated = c.compensated;
        out->device = c.device;
        out->compat_omp_pad = c.compat_omp_pad;
    });
}

int psm_segy_scan(const char* path, psm_segy_info* info, char* err, size_t err_len) {
    if (!path || !info) return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        Segy s(path, true);
        info->num_traces = s.num_traces();
        info->num_samples = s.num_samples();
        info->dt_us = s.dt_us();
        info->dt_seconds = s.dt_seconds();
        info->format = s.format();
        info->n_il = static_cast<int32_t>(s.il_labels().size());
        info->n_xl = static_cast<int32_t>(s.xl_labels().size());
        info->n_mapped = static_cast<int64_t>(s.lookup().size());
    });
}

int psm_segy_read_cube(const char* path, int32_t* il_labels, int32_t* xl_labels, float* cube,
                       char* err, size_t err_len) {
    if (!path) return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        Segy s(path, true);
        if (il_labels) std::copy(s.il_labels().begin(), s.il_labels().end(), il_labels);
        if (xl_labels) std::copy(s.xl_labels().begin(), s.xl_labels().end(), xl_labels);
        if (cube) s.read_cube(cube);
    });
}

float psm_ibm_to_ieee(uint32_t ibm) { return ibm_to_ieee(ibm); }
uint32_t psm_ieee_to_ibm(float v) { return ieee_to_ibm(v); }

int psm_velocity_cube(const char* param, const int32_t* il_labels, int32_t n_il,
                      const int32_t* xl_labels, int32_t n_xl, int32_t n_t, double dt,
                      float* out, char* err, size_t err_len) {
    if (!param || !il_labels || !xl_labels || !out || n_il < 0 || n_xl < 0 || n_t <= 0)
        return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        auto p = make_velocity_provider(param);
        std::vector<int32_t> xl(xl_labels, xl_labels + n_xl);
        for (int32_t i = 0; i < n_il; ++i)
            p->velocity_iline(il_labels[i], xl, n_t, dt,
                              out + static_cast<size_t>(i) * n_xl * n_t);
    });
}

int psm_velocity_point(const char* param, int32_t il, int32_t xl, int32_t t_idx, double dt,
                       int32_t n_t, float* out, char* err, size_t err_len) {
    if (!param || !out || t_idx < 0 || n_t <= 0) return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        auto p = make_velocity_provider(param);
        *out = p->velocity(il, xl, t_idx, dt, n_t);
    });
}

int psm_plan_config(const char* config_path, psm_plan* plan, char* err, size_t err_len) {
    if (!config_path || !plan) return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        Config c = parse_config(config_path);
        validate_config(c);
        Plan p;
        run(c, false, &p);
        plan->n_il = p.n_il;
        plan->n_xl = p.n_xl;
        plan->n_t = p.n_t;
        plan->n_oi = p.n_oi;
        plan->n_ox = p.n_ox;
        plan->m_il = p.m_il;
        plan->max_v = p.max_v;
        plan->tan2_theta = p.tan2;
        plan->dt_seconds = p.dt;
    });
}

int psm_run_config(const char* config_path, int verbose, char* err, size_t err_len) {
    if (!config_path) return PSM_ERR_ARG;
    return guarded(err, err_len, [&] {
        Config c = parse_config(config_path);
        validate_config(c);
        run(c, verbose != 0, nullptr);
    });
}

}  // extern "C"
