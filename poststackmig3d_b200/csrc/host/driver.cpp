// The migration driver (src/main.cpp:66-442): read the input SEG-Y and its lookup table,
// build the Vrms cube, derive the output geometry and aperture, migrate every output inline
// on the GPU in one resident pass (libpsm_cuda.so), and write the output SEG-Y.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <iomanip>
#include <iostream>

#include "host.hpp"
#include "psm.h"

namespace psmhost {

std::vector<int32_t> padded_labels(const std::vector<int32_t>& labels, int pad) {
    // main.cpp:144-172
    if (pad > 0 && labels.size() > 1) {
        const int32_t step = labels[1] - labels[0];
        const int32_t first = labels.front() - pad * step;
        const int32_t last = labels.back() + pad * step;
        std::vector<int32_t> out;
        for (int32_t l = first; l <= last; l += step) out.push_back(l);
        return out;
    }
    return labels;
}

std::vector<int32_t> output_centers(const std::vector<int32_t>& in,
                                    const std::vector<int32_t>& out,
                                    std::vector<char>* is_padding) {
    // main.cpp:258-288: a label not among the input inlines is padding and migrates the
    // nearest real inline (the first one at the smallest distance)
    std::vector<int32_t> c(out.size());
    if (is_padding) is_padding->assign(out.size(), 0);
    const size_t n = in.size();
    for (size_t o = 0; o < out.size(); ++o) {
        auto it = std::find(in.begin(), in.end(), out[o]);
        if (it != in.end()) {
            c[o] = static_cast<int32_t>(it - in.begin());
            continue;
        }
        if (is_padding) (*is_padding)[o] = 1;
        if (out[o] < in.front()) {
            c[o] = 0;
        } else if (out[o] > in.back()) {
            c[o] = static_cast<int32_t>(n - 1);
        } else {
            size_t best = 0;
            int32_t bd = std::abs(out[o] - in[0]);
            for (size_t i = 1; i < n; ++i) {
                const int32_t d = std::abs(out[o] - in[i]);
                if (d < bd) {
                    bd = d;
                    best = i;
                }
            }
            c[o] = static_cast<int32_t>(best);
        }
    }
    return c;
}

float estimate_max_velocity(VelocityProvider& p, const std::vector<int32_t>& il,
                            const std::vector<int32_t>& xl, size_t n_t, double dt) {
    // main.cpp:22-64: first / middle / last inline x crossline at the last sample
    std::vector<size_t> ii = {0}, xx = {0};
    if (il.size() > 1) {
        ii.push_back(il.size() / 2);
        ii.push_back(il.size() - 1);
    }
    if (xl.size() > 1) {
        xx.push_back(xl.size() / 2);
        xx.push_back(xl.size() - 1);
    }
    float mv = 0.0f;
    for (size_t a : ii)
        for (size_t b : xx) mv = std::max(mv, p.velocity(il[a], xl[b], n_t - 1, dt, n_t));
    return mv < 100.0f ? 3000.0f : mv;
}

float tan2_theta(double angle_deg) {  // main.cpp:188-189
    const float t = static_cast<float>(std::tan(angle_deg * 3.14159265358979323846 / 180.0));
    return t * t;
}

int max_aperture_il(float max_v, size_t n_t, double dt, float tan2, double inline_step) {
    // main.cpp:197-201 (float radius, double division)
    const double max_t = (n_t - 1) * dt;
    const float rad = (max_v * static_cast<float>(max_t) / 2.0f) * std::sqrt(tan2);
    return static_cast<int>(rad / inline_step) + 1;
}

namespace {

struct Timer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double s() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

void cuda_check(int rc, psm_ctx* ctx, const char* what) {
    if (rc != PSM_OK)
        throw Error(std::string(what) + " failed: " + (ctx ? psm_last_error(ctx) : "") +
                    " (status " + std::to_string(rc) + ")");
}

}  // namespace

void run(const Config& cfg, bool verbose, Plan* plan_only) {
    Timer total;
    std::ostream& out = std::cout;
    const char* rule = "============================================================";
    if (verbose) {
        out << rule << "\nPost-stack 3D Kirchhoff Migration (B200)\n" << rule << "\n";
        out << "Input file: " << cfg.input_data << "\nOutput file: " << cfg.output_data
            << "\nInline step: " << cfg.inline_step << " m\nCrossline step: "
            << cfg.crossline_step << " m\nInline padding: " << cfg.inline_padding
            << "\nCrossline padding: " << cfg.crossline_padding
            << "\nAngle aperture: " << cfg.angle_aperture
            << " deg\nAmplitude correction: " << (cfg.amp_correction ? "true" : "false")
            << "\nCompute: CUDA device " << cfg.device << " (sm_100a)\n" << rule << std::endl;
        out << "\n[1/6] Opening input file and creating lookup table..." << std::endl;
    }
    Segy in(cfg.input_data, !verbose);
    const auto& il = in.il_labels();
    const auto& xl = in.xl_labels();
    const size_t n_il = il.size(), n_xl = xl.size(), n_t = in.num_samples();
    const double dt = in.dt_seconds();
    if (n_il == 0 || n_xl == 0) throw Error("No traces with non-zero INLINE_3D/CROSSLINE_3D");
    if (verbose)
        out << "Input geometry: IL=" << n_il << ", XL=" << n_xl << ", T=" << n_t
            << ", dt=" << dt << "s" << std::endl;

    if (verbose) out << "\n[2/6] Reading velocity..." << std::endl;
    auto prov = make_velocity_provider(cfg.velocity);

    if (verbose) out << "\n[3/6] Preparing output geometry..." << std::endl;
    const auto out_il = padded_labels(il, cfg.inline_padding);
    const auto out_xl = padded_labels(xl, cfg.crossline_padding);
    std::vector<char> il_pad;
    const auto centers = output_centers(il, out_il, &il_pad);

    if (verbose) out << "\n[4/6] Calculating migration parameters..." << std::endl;
    const float tan2 = tan2_theta(cfg.angle_aperture);
    const float max_v = estimate_max_velocity(*prov, il, xl, n_t, dt);
    const int m_il = max_aperture_il(max_v, n_t, dt, tan2, cfg.inline_step);
    if (verbose) {
        const double max_t = (n_t - 1) * dt;
        const float rad = (max_v * static_cast<float>(max_t) / 2.0f) * std::sqrt(tan2);
        out << std::fixed << std::setprecision(0) << "Maximum velocity: " << max_v
            << " m/s\nMaximum time: " << std::setprecision(2) << max_t
            << " s\nAperture radius: IL=" << std::setprecision(0) << rad << "m, XL=" << rad
            << "m\nBuffer size: IL=+-" << m_il << " lines, XL=+-"
            << static_cast<int>(rad / cfg.crossline_step) + 1 << " lines" << std::endl;
        out.unsetf(std::ios_base::fixed);
    }
    if (plan_only) {
        plan_only->n_il = static_cast<int>(n_il);
        plan_only->n_xl = static_cast<int>(n_xl);
        plan_only->n_t = static_cast<int>(n_t);
        plan_only->n_oi = static_cast<int>(out_il.size());
        plan_only->n_ox = static_cast<int>(out_xl.size());
        plan_only->m_il = m_il;
        plan_only->max_v = max_v;
        plan_only->tan2 = tan2;
        plan_only->dt = dt;
        return;
    }

    Timer t_io;
    const double s_io = t_io.s();

    if (verbose) out << "\n[5/6] Migrating on the GPU..." << std::endl;
    Timer t_gpu;
    psm_ctx* ctx = nullptr;
    cuda_check(psm_create(&ctx, cfg.device), nullptr, "psm_create");
    const size_t n_out = out_il.size() * out_xl.size();
    std::vector<unsigned char> records(n_out * (240 + 4 * n_t));
    try {
        psm_geom g{};
        g.n_il = static_cast<int32_t>(n_il);
        g.n_xl = static_cast<int32_t>(n_xl);
        g.n_t = static_cast<int32_t>(n_t);
        g.pad_il = cfg.inline_padding;
        g.pad_xl = cfg.crossline_padding;
        g.n_oi = static_cast<int32_t>(out_il.size());
        g.n_ox = static_cast<int32_t>(out_xl.size());
        g.m_il = m_il;
        g.amp_correction = cfg.amp_correction ? 1 : 0;
        g.precision = cfg.precision;
        g.compensated = cfg.compensated ? 1 : 0;
        g.compat_omp_pad = cfg.compat_omp_pad ? 1 : 0;
        g.dt = static_cast<float>(dt);
        g.d_il = static_cast<float>(cfg.inline_step);
        g.d_xl = static_cast<float>(cfg.crossline_step);
        g.tan2_theta = tan2;
        g.dt_seconds = dt;
        cuda_check(psm_set_geometry(ctx, &g, centers.data()), ctx, "psm_set_geometry");
        const std::vector<int32_t> pos = in.record_positions();
        cuda_check(psm_set_traces_segy(ctx, in.trace_records(), in.num_traces(), in.format(),
                                       pos.data()),
                   ctx, "psm_set_traces_segy");
        // the output points' Vrms on the real grid (main.cpp:296-321): assembled on the GPU
        // for the table and SEG-Y providers, filled on the host for a constant
        if (!prov->assemble_on_gpu(ctx, il, xl)) {
            std::vector<float> vrms(n_il * n_xl * n_t);
            for (size_t i = 0; i < n_il; ++i)
                prov->velocity_iline(il[i], xl, n_t, dt, vrms.data() + i * n_xl * n_t);
            cuda_check(psm_set_vrms(ctx, vrms.data()), ctx, "psm_set_vrms");
        }
        cuda_check(psm_forward_async(ctx), ctx, "psm_forward_async");
        // output records encoded on the GPU (segy_utils.cpp:398-487, :598-648)
        const std::vector<int32_t> src = output_sources(in, out_il, out_xl, il_pad);
        cuda_check(psm_get_image_segy(ctx, records.data(), in.format(), src.data(),
                                      out_il.data(), out_xl.data()),
                   ctx, "psm_get_image_segy");
    } catch (...) {
        psm_destroy(ctx);
        throw;
    }
    psm_destroy(ctx);
    const double s_gpu = t_gpu.s();

    if (verbose) out << "\n[6/6] Writing output file..." << std::endl;
    Timer t_w;
    write_output_records(cfg.output_data, in, records.data(), n_out);
    if (verbose) {
        out << "Output dimensions: IL=" << out_il.size() << ", XL=" << out_xl.size()
            << "\n\nMigration complete!\n\nTotal time: " << std::fixed << std::setprecision(2)
            << total.s() << " seconds (read " << s_io << " s, GPU " << s_gpu << " s, write "
            << t_w.s() << " s)\nProcessed: " << n_il << " inlines x " << n_xl
            << " crosslines x " << n_t << " samples" << std::endl;
        out.unsetf(std::ios_base::fixed);
    }
}

}  // namespace psmhost
