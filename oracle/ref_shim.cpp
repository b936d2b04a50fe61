// Test infrastructure only.  An extern "C" face over the REFERENCE's own compiled code
// (src/migration_kernel.cpp, src/velocity_reader.cpp, src/segy_utils.cpp), linked from the
// reference sources by oracle/Makefile into oracle/_ref/libref_{serial,omp}.so.  Nothing
// here computes anything itself: each function forwards to the reference implementation so
// the tests can run it on exactly the inputs the CUDA path gets.
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

// The IBM<->IEEE helpers are private members of SegyFile (include/segy_utils.h:127-128);
// open them up for this translation unit only.
#define private public
#include "segy_utils.h"
#include "velocity_reader.h"
#include "migration_kernel.h"
#undef private

extern "C" {

// MigrationKernel::kirchhoffKernel3DWithPadding (include/migration_kernel.h:16-31) with a
// flat [n_out_xl][n_t] output instead of vector<vector<float>>.
void ref_kirchhoff_inline(const float* input_buffer, size_t n_buf_il, size_t n_buf_xl,
                          size_t n_t, const float* velocity_slice, float* output,
                          size_t n_out_xl, const int32_t* il_pos, int32_t current_il_pos,
                          int32_t current_xl_start, float dt, const float* t0_times,
                          float tan_theta_sq, float d_il, float d_xl, int amp_correction) {
    std::vector<std::vector<float>> out(n_out_xl, std::vector<float>(n_t, 0.0f));
    std::vector<int32_t> ilp(il_pos, il_pos + n_buf_il);
    std::vector<int32_t> xlp(n_buf_xl);
    for (size_t i = 0; i < n_buf_xl; ++i) xlp[i] = static_cast<int32_t>(i);
    std::vector<float> t0(t0_times, t0_times + n_t);
    MigrationKernel::kirchhoffKernel3DWithPadding(
        input_buffer, n_buf_il, n_buf_xl, n_t, velocity_slice, out, ilp, xlp,
        current_il_pos, current_xl_start, dt, t0, tan_theta_sq, d_il, d_xl,
        amp_correction != 0);
    for (size_t x = 0; x < n_out_xl; ++x)
        std::memcpy(output + x * n_t, out[x].data(), n_t * sizeof(float));
}

// Dense Vrms cube [n_il][n_xl][n_t] exactly as main.cpp:312-321 assembles it per inline
// (VelocityProviderFactory::create + getVelocityIline on the real inline/crossline labels).
int ref_velocity_cube(const char* param, const int32_t* il_labels, int n_il,
                      const int32_t* xl_labels, int n_xl, int n_t, double dt, float* out) {
    try {
        auto prov = VelocityProviderFactory::create(param);
        std::vector<int32_t> xl(xl_labels, xl_labels + n_xl);
        for (int i = 0; i < n_il; ++i) {
            auto vl = prov->getVelocityIline(il_labels[i], xl, n_t, dt);
            for (int x = 0; x < n_xl; ++x)
                std::memcpy(out + (static_cast<size_t>(i) * n_xl + x) * n_t,
                            vl[x].data(), n_t * sizeof(float));
        }
        prov->close();
        return 0;
    } catch (...) {
        return -1;
    }
}

// VelocityProvider::getVelocity for one point (used by estimateMaxVelocity, main.cpp:47-50).
int ref_velocity_point(const char* param, int32_t il, int32_t xl, int t_idx, double dt,
                       int n_t, float* out) {
    try {
        auto prov = VelocityProviderFactory::create(param);
        *out = prov->getVelocity(il, xl, static_cast<size_t>(t_idx), dt,
                                 static_cast<size_t>(n_t));
        prov->close();
        return 0;
    } catch (...) {
        return -1;
    }
}

// SegyFile::ibmToIeee (src/segy_utils.cpp:243-254); it reads no member state.
float ref_ibm_to_ieee(uint32_t ibm) {
    alignas(SegyFile) static unsigned char storage[sizeof(SegyFile)];
    return reinterpret_cast<SegyFile*>(storage)->ibmToIeee(ibm);
}

// SegyFile::ieeeToIbm (src/segy_utils.cpp:257-270).  Never call it with +-inf: the
// reference loops forever there.
uint32_t ref_ieee_to_ibm(float v) { return SegyFile::ieeeToIbm(v); }

}  // extern "C"
