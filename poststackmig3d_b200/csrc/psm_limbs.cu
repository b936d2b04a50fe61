// Throughput of the SM limbs the diffraction summation and its transpose draw on, measured on
// the device that runs them (psm_measure_limbs, include/psm.h).
//
// Each probe kernel runs a fixed number of independent operations per thread on every SM at
// once (148 SMs x kCtasPerSm CTAs of kThreads threads, all resident together) and records,
// for every CTA, its SM and its first and last clock64() reading.  An SM's busy span is the
// last end minus the first start over its CTAs (one SM clock counter), and a rate per clock
// per SM is
//     operations of the SM's CTAs / that span (cycles), median over the SMs,
// which does not depend on the clock the GPU ran at; the clock itself is the median span
// divided by the CUDA-event time of the launch.  Every shared-memory index stays inside the CTA's static
// array, and every loop has a fixed trip count.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "psm.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCtasPerSm = 4;  // 1024 threads per SM, 32 warps
constexpr int kSmemWords = 4096 + 64;  // 16.6 KB of floats per CTA

__device__ __forceinline__ void span_begin(unsigned long long* t) {
    __syncthreads();
    if (threadIdx.x == 0) *t = clock64();
}
// spans[3 b .. 3 b + 2] = SM id, start, end of CTA b
__device__ __forceinline__ void span_end(unsigned long long t0, unsigned long long* spans) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        spans[3 * blockIdx.x] = smid;
        spans[3 * blockIdx.x + 1] = t0;
        spans[3 * blockIdx.x + 2] = clock64();
    }
}

// 8 independent rsqrt chains per thread (MUFU.RSQ; the library builds with -ftz=true).
__global__ void __launch_bounds__(kThreads) rsq_probe(int iters, float* sink,
                                                      unsigned long long* spans) {
    float x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = 1.5f + 0.01f * static_cast<float>(threadIdx.x + i);
    __shared__ unsigned long long t0;
    span_begin(&t0);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = rsqrtf(x[i]);
    }
    span_end(t0, spans);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == 12345.0f) sink[threadIdx.x] = s;
}

// 8 independent scalar FMA chains per thread.
__global__ void __launch_bounds__(kThreads) ffma_probe(int iters, float* sink,
                                                       unsigned long long* spans) {
    float x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = 0.5f + 0.001f * static_cast<float>(threadIdx.x + i);
    const float a = 0.999f, b = 0.0005f;
    __shared__ unsigned long long t0;
    span_begin(&t0);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = __fmaf_rn(x[i], a, b);
    }
    span_end(t0, spans);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == 12345.0f) sink[threadIdx.x] = s;
}

// 8 independent packed-pair FMA chains per thread (fma.rn.f32x2: two FMAs per lane).
__global__ void __launch_bounds__(kThreads) ffma2_probe(int iters, float* sink,
                                                        unsigned long long* spans) {
    unsigned long long x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float v = 0.5f + 0.001f * static_cast<float>(threadIdx.x + i);
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[i]) : "f"(v), "f"(v + 0.25f));
    }
    unsigned long long a, b;
    asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(0.999f), "f"(0.998f));
    asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(0.0005f), "f"(0.0007f));
    __shared__ unsigned long long t0;
    span_begin(&t0);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[i]) : "l"(a), "l"(b));
    }
    span_end(t0, spans);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[i]));
        s += lo + hi;
    }
    if (s == 12345.0f) sink[threadIdx.x] = s;
}

// Lane l of a warp reads element base + idx(l) of an 8-byte array: idx(l) = l (consecutive),
// or floor(4 l / 5) (the forward's lanes at 32 consecutive output samples map to trace
// samples with ds/dt0 = t0 / t, about 0.8).  8 loads per iteration at distinct bases.
template <bool SLOPE>
__global__ void __launch_bounds__(kThreads) lds64_probe(int iters, float* sink,
                                                        unsigned long long* spans) {
    __shared__ float2 sm[kSmemWords / 2];
    for (int i = threadIdx.x; i < kSmemWords / 2; i += blockDim.x)
        sm[i] = make_float2(static_cast<float>(i), 1.0f);
    const int lane = threadIdx.x & 31;
    const int off = SLOPE ? (4 * lane) / 5 : lane;
    float2 acc = make_float2(0.0f, 0.0f);
    __shared__ unsigned long long t0;
    span_begin(&t0);
    for (int it = 0; it < iters; ++it) {
        const float2* p = sm + ((it & 15) << 6) + off;  // base <= 960, + 7 * 128 + 31 < 2080
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 v = p[i * 128];
            acc.x += v.x;
            acc.y += v.y;
        }
    }
    span_end(t0, spans);
    if (acc.x == 12345.0f) sink[threadIdx.x] = acc.x + acc.y;
}

// Shared-memory f32 reductions: lane l adds to element base + idx(l) (as lds64_probe, 4-byte
// elements), 8 per iteration at distinct bases; RED: red.shared.add.f32 (no return value),
// else atomicAdd.
template <bool SLOPE, bool RED>
__global__ void __launch_bounds__(kThreads) atom_probe(int iters, float* sink,
                                                       unsigned long long* spans) {
    __shared__ float sm[kSmemWords];
    for (int i = threadIdx.x; i < kSmemWords; i += blockDim.x) sm[i] = 0.0f;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int off = SLOPE ? (4 * lane) / 5 : lane;
    const float v = 1.0f + 0.001f * static_cast<float>(lane);
    __shared__ unsigned long long t0;
    span_begin(&t0);
    for (int it = 0; it < iters; ++it) {
        // base <= 15 * 64 + 7 * 32 = 1184; + 7 * 384 + 31 < 3904 < kSmemWords
        float* p = sm + ((it & 15) << 6) + warp * 32 + off;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (RED)
                asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(
                                 static_cast<unsigned>(__cvta_generic_to_shared(p + i * 384))),
                             "f"(v)
                             : "memory");
            else
                atomicAdd(p + i * 384, v);
        }
    }
    span_end(t0, spans);
    if (sm[threadIdx.x] == 12345.0f) sink[threadIdx.x] = sm[threadIdx.x];
}

// Shared-memory integer reductions (atomicAdd on 32- or 64-bit unsigned integers, return value
// unused), the same address patterns as atom_probe.
template <bool SLOPE, typename T>
__global__ void __launch_bounds__(kThreads) iatom_probe(int iters, float* sink,
                                                        unsigned long long* spans) {
    __shared__ T sm[kSmemWords];  // 16.6 KB (u32) or 33 KB (u64)
    for (int i = threadIdx.x; i < kSmemWords; i += blockDim.x) sm[i] = 0;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int off = SLOPE ? (4 * lane) / 5 : lane;
    const T v = static_cast<T>(1 + lane);
    __shared__ unsigned long long t0;
    span_begin(&t0);
    for (int it = 0; it < iters; ++it) {
        // as atom_probe: every index stays below 3904 < kSmemWords
        T* p = sm + ((it & 15) << 6) + warp * 32 + off;
#pragma unroll
        for (int i = 0; i < 8; ++i) atomicAdd(p + i * 384, v);
    }
    span_end(t0, spans);
    if (sm[threadIdx.x] == static_cast<T>(12345)) sink[threadIdx.x] = 1.0f;
}

// Median SM span (cycles), CTAs per SM that the spans cover, and event time (ms) of one
// launch of kernel k.
template <typename K>
int time_probe(K k, int iters, int n_sm, double* cycles, double* ms, double* ctas_per_sm) {
    const int n_cta = n_sm * kCtasPerSm;
    unsigned long long* spans = nullptr;
    float* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = PSM_OK;
    if (cudaMalloc(&spans, 3 * sizeof(unsigned long long) * n_cta) != cudaSuccess ||
        cudaMalloc(&sink, sizeof(float) * kThreads) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = PSM_ERR_NOMEM;
    } else {
        k<<<n_cta, kThreads>>>(iters / 8, sink, spans);  // warm-up
        cudaEventRecord(e0);
        k<<<n_cta, kThreads>>>(iters, sink, spans);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = PSM_ERR_CUDA;
        } else {
            std::vector<unsigned long long> h(3 * static_cast<size_t>(n_cta));
            cudaMemcpy(h.data(), spans, 3 * sizeof(unsigned long long) * n_cta,
                       cudaMemcpyDeviceToHost);
            // per SM: first start, last end, CTAs
            std::vector<unsigned long long> first(n_sm, ~0ull), last(n_sm, 0);
            std::vector<int> count(n_sm, 0);
            for (int b = 0; b < n_cta; ++b) {
                const unsigned long long sm = h[3 * b];
                if (sm >= static_cast<unsigned long long>(n_sm)) continue;
                first[sm] = std::min(first[sm], h[3 * b + 1]);
                last[sm] = std::max(last[sm], h[3 * b + 2]);
                ++count[sm];
            }
            std::vector<double> span, per;
            for (int sm = 0; sm < n_sm; ++sm)
                if (count[sm] > 0 && last[sm] > first[sm]) {
                    span.push_back(static_cast<double>(last[sm] - first[sm]) / count[sm]);
                    per.push_back(count[sm]);
                }
            if (span.empty()) {
                rc = PSM_ERR_CUDA;
            } else {
                // span per CTA of work, times the CTAs one SM ran: the cycles of kCtasPerSm
                // CTAs' work on one SM
                std::nth_element(span.begin(), span.begin() + span.size() / 2, span.end());
                *cycles = span[span.size() / 2] * kCtasPerSm;
                std::nth_element(per.begin(), per.begin() + per.size() / 2, per.end());
                *ctas_per_sm = per[per.size() / 2];
            }
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            *ms = t;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(spans);
    cudaFree(sink);
    return rc;
}

}  // namespace

extern "C" int psm_measure_limbs(int device, psm_limbs* out) {
    if (!out) return PSM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return PSM_ERR_ARG;
    int n_sm = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return PSM_ERR_CUDA;
    const double per_sm = static_cast<double>(kThreads) * kCtasPerSm;  // threads per SM
    constexpr int kIters = 1 << 14;
    double cyc = 0.0, ms = 0.0, clk_sum = 0.0, cps = kCtasPerSm;
    int n_clk = 0;
    int rc;
    // rate per clock per SM of `ops` operations per thread
    auto rate = [&](double ops) {
        clk_sum += cyc / kCtasPerSm * cps / (ms * 1e-3) / 1e6;
        ++n_clk;
        return ops * per_sm / cyc;
    };
    if ((rc = time_probe(rsq_probe, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->rsqrt_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(ffma_probe, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->ffma_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(ffma2_probe, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->ffma2_per_clk_sm = rate(16.0 * kIters);
    if ((rc = time_probe(lds64_probe<false>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->lds64_bytes_per_clk_sm = rate(64.0 * kIters);
    if ((rc = time_probe(lds64_probe<true>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->lds64_slope_bytes_per_clk_sm = rate(64.0 * kIters);
    if ((rc = time_probe(atom_probe<false, false>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->atom_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(atom_probe<true, false>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->atom_slope_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(atom_probe<false, true>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->red_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(atom_probe<true, true>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->red_slope_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(iatom_probe<false, unsigned>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->atom_u32_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(iatom_probe<true, unsigned>, kIters, n_sm, &cyc, &ms, &cps))) return rc;
    out->atom_u32_slope_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(iatom_probe<false, unsigned long long>, kIters, n_sm, &cyc, &ms, &cps)))
        return rc;
    out->atom_u64_per_clk_sm = rate(8.0 * kIters);
    if ((rc = time_probe(iatom_probe<true, unsigned long long>, kIters, n_sm, &cyc, &ms, &cps)))
        return rc;
    out->atom_u64_slope_per_clk_sm = rate(8.0 * kIters);
    out->sm_clock_mhz = clk_sum / n_clk;
    out->n_sm = n_sm;
    return PSM_OK;
}
