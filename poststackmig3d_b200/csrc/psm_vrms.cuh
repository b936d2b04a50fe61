// Vrms of the output points assembled on the GPU (sm_100a).
//
// The reference's providers are CPU loops (src/velocity_reader.cpp): the text table blends
// every table point into every sample (:320-361), O(points) per sample; an off-grid SEG-Y Vrms
// blends the 2x2 label neighbours (:93-163) and interpolates in time (:124-138, :184-196).
// Here one thread computes one sample (il, xl, t) of the dense Vrms cube with the same
// operations in the same order: double products and sums with explicit round-to-nearest
// intrinsics (the host build has no fused multiply-add), float weights 1 / (1 + float(d)),
// float accumulation in source order.  The result equals the host providers' bit for bit
// (their distance to the reference's -ffast-math build, which reorders those sums, is 1-2 ulp).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace psm {

// Text-table Vrms: every point (il, xl, time, v) weighted by 1 / (1 + dist) with dist mixing
// label units and seconds; an exact hit (dist < 1e-10) returns that point's v; a result <= 0
// (or no weight) gives vmin.  out [n_il][n_xl][n_t], t0 = t * dt.
__global__ void vrms_table_kernel(const int32_t* __restrict__ p_il,
                                  const int32_t* __restrict__ p_xl,
                                  const double* __restrict__ p_time,
                                  const float* __restrict__ p_v, int n_points, float vmin,
                                  const int32_t* __restrict__ il, const int32_t* __restrict__ xl,
                                  int n_il, int n_xl, int n_t, double dt,
                                  float* __restrict__ out) {
    const int64_t n = static_cast<int64_t>(n_il) * n_xl * n_t;
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(k % n_t);
        const int64_t tr = k / n_t;
        const int32_t a_il = il[tr / n_xl], a_xl = xl[tr % n_xl];
        const double time = __dmul_rn(static_cast<double>(t), dt);
        float sv = 0.0f, sw = 0.0f, hit_v = 0.0f;
        bool hit = false;
        for (int p = 0; p < n_points; ++p) {
            const double a = fabs(static_cast<double>(p_il[p] - a_il));
            const double b = fabs(static_cast<double>(p_xl[p] - a_xl));
            const double c = fabs(__dsub_rn(p_time[p], time));
            const double d =
                __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)));
            if (d < 1e-10) {
                hit = true;
                hit_v = p_v[p];
                break;
            }
            const float w = __fdiv_rn(1.0f, __fadd_rn(1.0f, __double2float_rn(d)));
            sv = __fadd_rn(sv, __fmul_rn(p_v[p], w));
            sw = __fadd_rn(sw, w);
        }
        float r = hit_v;
        if (!hit) {
            r = sw > 0.0f ? __fdiv_rn(sv, sw) : vmin;
            if (r <= 0.0f) r = vmin;
        }
        out[k] = r;
    }
}

// Linear interpolation in time of a grid trace, clamped at both ends.
__device__ __forceinline__ float grid_in_time(const float* tr, int g_nt, double gdt, double time) {
    if (time <= 0.0) return tr[0];
    if (time >= __dmul_rn(static_cast<double>(g_nt - 1), gdt)) return tr[g_nt - 1];
    const double s = __ddiv_rn(time, gdt);
    const int lo = static_cast<int>(s);
    if (lo >= g_nt - 1) return tr[g_nt - 1];
    const double fr = __dsub_rn(s, static_cast<double>(lo));
    return __double2float_rn(__dadd_rn(__dmul_rn(static_cast<double>(tr[lo]), __dsub_rn(1.0, fr)),
                                       __dmul_rn(static_cast<double>(tr[lo + 1]), fr)));
}

// Index of the label nearest to x in the sorted labels v (ties to the lower one).
__device__ __forceinline__ int nearest_label(const int32_t* v, int n, int32_t x) {
    int lo = 0, hi = n;  // first index with v[i] >= x
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (v[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo == 0) return 0;
    if (lo == n) return n - 1;
    return abs(v[lo] - x) < abs(v[lo - 1] - x) ? lo : lo - 1;
}

// SEG-Y-grid Vrms: grid [g_nil][g_nxl][g_nt] on sorted labels (missing traces zero), sample
// interval gdt.  A point on a grid inline and crossline copies its trace (same dt and n_t) or
// interpolates it in time; any other point blends the 4 neighbours one label below and above
// the nearest grid labels with weights 1 / (1 + |dIL| + |dXL|).
__global__ void vrms_grid_kernel(const float* __restrict__ grid, const int32_t* __restrict__ g_il,
                                 int g_nil, const int32_t* __restrict__ g_xl, int g_nxl, int g_nt,
                                 double gdt, const int32_t* __restrict__ il,
                                 const int32_t* __restrict__ xl, int n_il, int n_xl, int n_t,
                                 double dt, float* __restrict__ out) {
    const int64_t n = static_cast<int64_t>(n_il) * n_xl * n_t;
    const bool same_axis = fabs(dt - gdt) < 1e-6 && n_t == g_nt;
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(k % n_t);
        const int64_t tr = k / n_t;
        const int32_t a_il = il[tr / n_xl], a_xl = xl[tr % n_xl];
        const double time = __dmul_rn(static_cast<double>(t), dt);
        const int ii = nearest_label(g_il, g_nil, a_il), xi = nearest_label(g_xl, g_nxl, a_xl);
        float r;
        if (g_il[ii] == a_il && g_xl[xi] == a_xl) {
            const float* trc = grid + (static_cast<int64_t>(ii) * g_nxl + xi) * g_nt;
            r = same_axis ? trc[t] : grid_in_time(trc, g_nt, gdt, time);
        } else {
            const int is[2] = {ii > 0 ? ii - 1 : 0, ii < g_nil - 1 ? ii + 1 : g_nil - 1};
            const int xs[2] = {xi > 0 ? xi - 1 : 0, xi < g_nxl - 1 ? xi + 1 : g_nxl - 1};
            float sv = 0.0f, sw = 0.0f, v0 = 0.0f;
            for (int p = 0; p < 2; ++p)
                for (int q = 0; q < 2; ++q) {
                    const float* trc = grid + (static_cast<int64_t>(is[p]) * g_nxl + xs[q]) * g_nt;
                    const float val = grid_in_time(trc, g_nt, gdt, time);
                    if (p == 0 && q == 0) v0 = val;
                    const double d_il = fabs(static_cast<double>(g_il[is[p]] - a_il));
                    const double d_xl = fabs(static_cast<double>(g_xl[xs[q]] - a_xl));
                    const float w =
                        __fdiv_rn(1.0f, __fadd_rn(1.0f, __double2float_rn(__dadd_rn(d_il, d_xl))));
                    sv = __fadd_rn(sv, __fmul_rn(val, w));
                    sw = __fadd_rn(sw, w);
                }
            r = sw > 0.0f ? __fdiv_rn(sv, sw) : v0;
        }
        out[k] = r;
    }
}

}  // namespace psm
