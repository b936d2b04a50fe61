// Device code of the B200 Kirchhoff post-stack 3D time migration (sm_100a).
//
// The operator is the reference's diffraction summation (sergeevsn/poststackmig3d,
// src/migration_kernel.cpp:17-383): for every output sample (inline c, crossline x, time t0)
//     out = sum over input traces (i, k) with r^2 = dx^2 + dy^2 <= (v t0 / 2)^2 tan^2(theta)
//           and floor(t / dt) < n_t - 1 of  interp(trace(i,k), t / dt) / (t v^2)
// with t = sqrt(t0^2 + 4 r^2 / v^2), v the output point's Vrms, interp the linear rule
// fma(frac, d[lo+1] - d[lo], d[lo]) (simdInterpolate, :544-550).
//
// HBM layout: the traces are held as a "pair cube" [inline][crossline][ns] of float2
// (d[t], d[t+1] - d[t]) built once after upload (pair_kernel), so one 8-byte shared-memory
// load gives both interpolation operands with the reference's own difference.
//
// Work decomposition (one CTA):
//   * one output row ("job": an output inline), kTX consecutive output crosslines and
//     kTT = 256 consecutive output samples (a "tile");
//   * warp 0 is the producer: it lists the input traces that can reach the tile, derives for
//     each a window [ws, we) of samples that covers every term of the tile that passes the
//     masks, and stages the windows into shared memory with TMA bulk copies (cp.async.bulk)
//     into a ring of kStages buffers guarded by mbarriers;
//   * warps 1..kTX are consumers: warp w owns output crossline x0 + w - 1; lane l holds the
//     8 samples t0 = T0 + l + 32 j (j = 0..7) as 4 register pairs, evaluated with packed
//     f32x2 arithmetic.  Per staged trace the quantities dy, r^2 and the window base are
//     warp-uniform.
// Masks: a term passes the reference's aperture and range masks exactly when r^2 <= B, B a
// per-sample bound found once with the reference's IEEE arithmetic (pass_bound).
// Every wait is bounded: on expiry the kernel records PSM_DEV_ERR_TIMEOUT in *err and leaves.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace psm {

constexpr int kTX = 8;          // output crosslines per CTA (one consumer warp each)
constexpr int kJ = 8;           // 32-sample blocks per consumer lane
constexpr int kTT = 32 * kJ;    // output samples per CTA
constexpr int kStages = 2;      // TMA ring depth
constexpr int kMaxG = 32;       // traces per ring stage
static_assert(kTX % 4 == 0, "per-slot r^2 rows are stored as float4");
constexpr int kStageCapMin = 6144;          // samples (8 B each) per ring stage, at least
// Bytes of one ring stage of a forward kernel built for minb CTAs per SM, and the offset of
// a mirrored pair's second window from its first: half a stage, a compile-time constant, so
// that the consumers read the second trace through the first trace's address plus an
// immediate offset.
__host__ __device__ constexpr int stage_bytes_for(int minb) {
    return minb == 4 ? 20480 : minb == 3 ? 32768 : 8 * kStageCapMin;
}
__host__ __device__ constexpr int pair_off_bytes(int minb) { return stage_bytes_for(minb) / 2; }
// mbarrier waits end after FwdParams::wait_us of %globaltimer time (kDefaultWaitUs when 0),
// or after kWaitPollCap polls, whichever comes first
constexpr unsigned kDefaultWaitUs = 4000000u;
constexpr unsigned kWaitPollCap = 1u << 30;
// FwdParams::fault: test-only failure injection, 0 in normal runs.  kFaultStallProducer: the
// producer never arrives on (and issues no copy into) the first stage of its tile, so the
// consumers' bounded wait on it runs out and the launch reports PSM_DEV_ERR_TIMEOUT.
constexpr int kFaultStallProducer = 1;

// Trace storage in HBM: fp32 pairs (d[t], d[t+1] - d[t]) (8 B a sample), or 16-bit words
// (q[t] | q[t+1] << 16) of bf16 / fp16 values d / scale with one fp32 scale per trace.
constexpr int kStoreF32 = 0;
constexpr int kStoreBF16 = 1;
constexpr int kStoreF16 = 2;
__host__ __device__ constexpr int store_bytes(int store) { return store == kStoreF32 ? 8 : 4; }

constexpr int PSM_DEV_ERR_TIMEOUT = 1;
constexpr int PSM_DEV_ERR_WINDOW = 2;  // debug-bounds build (PSM_DEBUG_BOUNDS) only

// Shared memory kept free after the staging ring: a read a few samples past the last staged
// window stays inside the CTA's allocation.
constexpr unsigned kSmemGuard = 128;

// One output inline of a launch.
struct Job {
    int row;   // output image row
    int vrow;  // Vrms plane (cube inline of the output point's velocity)
    int pos;   // inline position of the output point (dx = (il_pos[i] - pos) * d_il)
    int i0;    // cube inlines [i0, i1) form the buffer (migration_kernel.cpp:404-409)
    int i1;
};

struct FwdParams {
    const float2* pairs;  // [n_ci][n_cx][ns] (d[t], d[t+1]-d[t]); rows 16 B aligned
    const uint32_t* words;  // [n_ci][n_cx][ns] 16-bit storage: q[t] | q[t+1] << 16
    const float* scales;    // [n_ci][n_cx] 16-bit storage: d = q * scale
    const float* vrms;    // Vrms of the output points: (vrow, x, t) at vrow vs_row + x vs_x + t
    long long vs_row, vs_x;  // element strides ([n_vrow][n_vx][n_t]; 0 broadcasts one trace)
    float* image;         // [rows][n_ox][n_t]
    const Job* jobs;
    const int* il_pos;    // [n_ci] inline positions
    const float* t0;      // [n_t]
    int* err;
    unsigned wait_us;  // limit of every mbarrier wait in microseconds (0: kDefaultWaitUs)
    int fault;         // test-only failure injection (kFault*), 0 normally
    int compat_pad;    // trailing padded crosslines take the last real crossline's Vrms
    int n_ci, n_cx, n_t, ns;
    int n_vx;             // crosslines of a Vrms plane
    int n_ox;             // output crosslines per row
    int xoff;             // cube / Vrms crossline of output x is x + xoff
    int max_inl;          // largest i1 - i0 over the jobs (inline-table capacity)
    int stage_cap;        // samples per ring stage (of store_bytes each)
    int pairable;         // il_pos consecutive: mirrored inlines c - d, c + d can be paired
    float inv_dt, idt2, d_il, d_xl, inv_dxl, tan2, tanth;
    float ntm1f;          // n_t - 1
    float ntm1m;          // largest float below n_t - 1
};

struct StageMeta {
    int count;        // traces in this stage, -1 = end of stream
    int pad[3];
    int4 m[kMaxG];    // window base (smem bytes, see consumers), window start as float
                      // (bits), the mirrored trace's window base, 1 for a mirrored pair
    float sc[kMaxG];  // trace scale (16-bit storage)
    float wend[kMaxG];  // window end as float (read by the debug-bounds build)
    float scb[kMaxG];   // paired slots, 16-bit storage: the mirrored trace's scale
    float r2[kMaxG][kTX];  // r^2 of the slot's trace(s) to each consumer warp's crossline
};

struct TileStats {
    float vmin, vmax, bmax, t0min, t0max;
    int any;
};

// Dynamic shared memory layout, shared by the host (sizing) and the kernel.
struct SmemLayout {
    unsigned full, empty, meta, stats, inl_klo, inl_pre, inl_dx2, stage, total;
};

__host__ __device__ inline SmemLayout smem_layout(int max_inl, int cap, int elem_bytes = 8) {
    SmemLayout L;
    unsigned o = 0;
    L.full = o;
    o += 8 * kStages;
    L.empty = o;
    o += 8 * kStages;
    L.meta = o = (o + 15) & ~15u;
    o += sizeof(StageMeta) * kStages;
    L.stats = o;
    o += sizeof(TileStats) * kTX;
    L.inl_klo = o;
    o += 4 * max_inl;
    L.inl_pre = o;
    o += 4 * (max_inl + 1);
    L.inl_dx2 = o;
    o += 4 * max_inl;
    L.stage = o = (o + 127) & ~127u;
    o += static_cast<unsigned>(elem_bytes) * cap * kStages;
    L.total = o + kSmemGuard;
    return L;
}

// ----------------------------------------------------------------------------- PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
            smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: false (and *err set) once limit_us (0: kDefaultWaitUs) microseconds of
// globaltimer time have passed without the phase completing (the clock is read every 64
// polls; kWaitPollCap polls at most).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          unsigned limit_us) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long lim = 1000ull * (limit_us ? limit_us : kDefaultWaitUs);
    const unsigned long long start = global_ns();
    for (unsigned it = 1; it < kWaitPollCap; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0 && global_ns() - start > lim) break;
    }
    atomicOr(err, PSM_DEV_ERR_TIMEOUT);
    return false;
}

// TMA bulk copy global -> shared, completion counted on an mbarrier (bytes % 16 == 0,
// both addresses 16 B aligned).
__device__ __forceinline__ void tma_load_1d(uint32_t dst_smem, const void* src, uint32_t bytes,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(dst_smem),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// packed FP32 pairs (sm_100 f32x2 arithmetic)
__device__ __forceinline__ unsigned long long pk(float2 v) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
    return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
    return upk(r);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 add2_rm(float2 a, float2 b) {  // rounding toward -inf
    unsigned long long r;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ----------------------------------------------------------------------------- point setup

// Vrms trace of output point (vrow, xv).
__device__ __forceinline__ const float* vrms_trace(const FwdParams& P, int vrow, int xv) {
    return P.vrms + vrow * P.vs_row + xv * P.vs_x;
}

// Vrms crossline of output crossline x (cube crossline xv = x + xoff), or -1 when the point
// has none: padded crosslines have v = 0 and no terms (migration_kernel.cpp:486-510, the
// serial build).  With compat_pad, trailing padded crosslines take the last real crossline's
// Vrms, as the reference's OpenMP build computes them: there the kernel's crossline loop is a
// nested parallel region (src/main.cpp:255 already runs one output inline per thread), so
// one thread walks every crossline in order, and its per-sample caches
// (migration_kernel.cpp:60-72, :115-144), filled only where v >= 1e-5, still hold the last
// real crossline's values, while r^2 is taken from the padded crossline's own position.
__device__ __forceinline__ int vrms_col(const FwdParams& P, int x) {
    const int xv = x + P.xoff;
    if (x >= P.n_ox || xv < 0) return -1;
    if (xv < P.n_vx) return xv;
    return P.compat_pad ? P.n_vx - 1 : -1;
}

// Per output sample constants in the reference's FP32 order (migration_kernel.cpp:115-144).
// Division and products are pinned to round-to-nearest so the masks see the same numbers
// as the reference build; that build (GCC, -ffp-contract=fast) fuses v*v + 1e-10.
struct PointConst {
    bool valid;
    float t0sq, f4, md2, vsq;
};

__device__ __forceinline__ PointConst point_const(float v, float t0v, float tan2) {
    PointConst p;
    p.valid = (v >= 1e-5f) && (t0v >= 1e-5f);                 // :121
    p.t0sq = __fmul_rn(t0v, t0v);                              // :125
    p.vsq = __fmul_rn(v, v);                                   // :127
    float inv_vsq = __fdiv_rn(1.0f, __fmaf_rn(v, v, 1e-10f));  // :128
    p.f4 = __fmul_rn(4.0f, inv_vsq);                           // :129
    float vth = __fmul_rn(__fmul_rn(v, t0v), 0.5f);            // :133
    p.md2 = __fmul_rn(__fmul_rn(vth, vth), tan2);              // :134
    return p;
}

// The reference keeps a term when floor(s) < n_t - 1 with s = fl(sqrt(fma(f4, r2, t0^2)) *
// inv_dt) in IEEE FP32 (migration_kernel.cpp:209-226, :291-298).  s grows monotonically
// with r2, so the kept r2 form a prefix [0, R].  pass_bound returns B = min(md2, R): a term
// passes both of the reference's masks exactly when r2 <= B (B < 0: no term passes).  Found
// by a search on the bit patterns of the non-negative floats in [0, md2].
__device__ __forceinline__ bool range_ok(float r2, float f4, float t0sq, float inv_dt,
                                         float ntm1f) {
    return __fmul_rn(__fsqrt_rn(__fmaf_rn(f4, r2, t0sq)), inv_dt) < ntm1f;
}

// GALLOP: start from an estimate of the boundary (fewer evaluations; the adjoint keeps the
// plain bisection, whose smaller code spills less in its 4-CTA build).
template <bool GALLOP = true>
__device__ __forceinline__ float pass_bound(const PointConst& p, float inv_dt, float ntm1f) {
    if (!p.valid || !(p.md2 >= 0.0f)) return -1.0f;
    if (range_ok(p.md2, p.f4, p.t0sq, inv_dt, ntm1f)) return p.md2;
    if (!range_ok(0.0f, p.f4, p.t0sq, inv_dt, ntm1f)) return -1.0f;
    unsigned lo = 0u, hi = __float_as_uint(p.md2);  // ok(lo), !ok(hi)
    if (GALLOP && hi - lo > 1u) {
        // Gallop out from the boundary of the unrounded test, f4 r2 + t0^2 =
        // ((n_t - 1) / inv_dt)^2, to a bracket of doubling width; the bisection below then
        // closes it.  The test is monotone in r2, so any bracket gives the same bound as a
        // bisection of all of [0, md2]; about 7 evaluations instead of 32.
        const float a = __fdividef(ntm1f, inv_dt);
        const float e = __fdividef(__fmaf_rn(a, a, -p.t0sq), p.f4);
        unsigned m = e > 0.0f ? __float_as_uint(e) : 0u;
        m = min(max(m, lo + 1u), hi - 1u);
        unsigned step = 1u;
        if (range_ok(__uint_as_float(m), p.f4, p.t0sq, inv_dt, ntm1f)) {
            lo = m;
            while (hi - lo > step) {
                const unsigned c = lo + step;
                if (!range_ok(__uint_as_float(c), p.f4, p.t0sq, inv_dt, ntm1f)) {
                    hi = c;
                    break;
                }
                lo = c;
                step <<= 1;
            }
        } else {
            hi = m;
            while (hi - lo > step) {
                const unsigned c = hi - step;
                if (range_ok(__uint_as_float(c), p.f4, p.t0sq, inv_dt, ntm1f)) {
                    lo = c;
                    break;
                }
                hi = c;
                step <<= 1;
            }
        }
    }
    while (hi - lo > 1u) {
        const unsigned mid = lo + ((hi - lo) >> 1);
        if (range_ok(__uint_as_float(mid), p.f4, p.t0sq, inv_dt, ntm1f))
            lo = mid;
        else
            hi = mid;
    }
    return __uint_as_float(lo);
}

// dx^2 of a buffer inline (migration_kernel.cpp:51-56).
__device__ __forceinline__ float inline_dx2(int ipos, int pos, float d_il) {
    float dx = __fmul_rn(static_cast<float>(ipos - pos), d_il);
    return __fmul_rn(dx, dx);
}

// r^2 of a trace at crossline distance dk (migration_kernel.cpp:197-204 / :282-284, with the
// multiply-add fused as the reference's GCC build fuses it).
__device__ __forceinline__ float trace_r2(int dk, float d_xl, float dx2) {
    float dy = __fmul_rn(static_cast<float>(dk), d_xl);
    return __fmaf_rn(dy, dy, dx2);
}

// ----------------------------------------------------------------------------- pair cube

// pairs[t] = (d[t], d[t+1] - d[t]) over rows of ns samples (d beyond the row is 0).
__global__ void pair_kernel(const float* __restrict__ src, float2* __restrict__ dst,
                            size_t n_rows, int ns) {
    const size_t n = n_rows * static_cast<size_t>(ns);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(i % ns);
        const float a = src[i];
        const float b = (t + 1 < ns) ? src[i + 1] : 0.0f;
        dst[i] = make_float2(a, __fsub_rn(b, a));
    }
}

// 16-bit storage of rows of ns fp32 samples (zero beyond n_t): one warp per trace.
// scale = max |d| over the trace (1 for an all-zero trace), q[t] = RNE(d[t] / scale) as
// bf16 or fp16, words[t] = bits(q[t]) | bits(q[t+1]) << 16 with q[ns] = 0.
template <int STORE>
__device__ __forceinline__ uint32_t q16(float x) {
    if (STORE == kStoreBF16) return __bfloat16_as_ushort(__float2bfloat16_rn(x));
    return __half_as_ushort(__float2half_rn(x));
}

template <int STORE>
__global__ void quantize_kernel(const float* __restrict__ src, uint32_t* __restrict__ words,
                                float* __restrict__ scales, size_t n_rows, int ns) {
    const int lane = threadIdx.x & 31;
    const size_t warps = static_cast<size_t>(gridDim.x) * (blockDim.x >> 5);
    for (size_t r = blockIdx.x * static_cast<size_t>(blockDim.x >> 5) + (threadIdx.x >> 5);
         r < n_rows; r += warps) {
        const float* row = src + r * ns;
        float m = 0.0f;
        for (int t = lane; t < ns; t += 32) m = fmaxf(m, fabsf(row[t]));
        m = warp_max(m);
        const float scale = m > 0.0f ? m : 1.0f;
        if (lane == 0) scales[r] = scale;
        uint32_t* out = words + r * ns;
        for (int t = lane; t < ns; t += 32) {
            const uint32_t a = q16<STORE>(__fdiv_rn(row[t], scale));
            const uint32_t b = t + 1 < ns ? q16<STORE>(__fdiv_rn(row[t + 1], scale)) : 0u;
            out[t] = a | (b << 16);
        }
    }
}

// ----------------------------------------------------------------------------- forward

// Buffer inlines (local indices) of row r of the producer's trace list: with pc < 0 the row is
// inline r; else row r is the mirror distance from the centre inline pc, holding inlines
// pc - r and pc + r (*b = -1 when the row has one inline: r = 0, or one side outside the
// buffer).
__device__ __forceinline__ void row_inlines(int pc, int n_inl, int r, int* a, int* b) {
    if (pc < 0) {
        *a = r;
        *b = -1;
        return;
    }
    *a = pc - r;
    *b = r > 0 && pc + r < n_inl ? pc + r : -1;
    if (*a < 0) {
        *a = pc + r;
        *b = -1;
    }
}

// Producer: lo of every passing term of the tile on trace (dx2, kc) lies in [*lolo, *lohi]
// (with two samples of slack for rounding); false when the trace has no passing term.
// Bounds: t >= t0 and, inside the aperture r <= v t0 tan/2, t0 >= 2 r_min / (v_max tan);
// t^2 = t0^2 + f4 r^2 <= min(t0max^2 + 4 r_max^2 / v_min^2, t0max^2 (1 + tan^2)).
__device__ __forceinline__ bool trace_bounds(const FwdParams& P, const TileStats& S, int xa,
                                             int xb, float dx2, int kc, int* lolo_out,
                                             int* lohi_out) {
    const int dkmin = kc < xa ? xa - kc : (kc > xb ? kc - xb : 0);
    const int dkmax = max(abs(kc - xa), abs(kc - xb));
    const float dymin = static_cast<float>(dkmin) * P.d_xl;
    const float dymax = static_cast<float>(dkmax) * P.d_xl;
    const float rmin2 = fmaf(dymin, dymin, dx2);
    const float rmax2 = fmaf(dymax, dymax, dx2);
    if (rmin2 > S.bmax * 1.0001f + 1e-6f) return false;
    float t0lo = S.t0min;
    if (P.tanth > 0.0f) t0lo = fmaxf(t0lo, 2.0f * sqrtf(rmin2) / (S.vmax * P.tanth));
    const float tlo = sqrtf(fmaf(t0lo, t0lo, 4.0f * rmin2 / fmaf(S.vmax, S.vmax, 1e-10f)));
    const float thi2 =
        fminf(fmaf(S.t0max, S.t0max, 4.0f * rmax2 / fmaf(S.vmin, S.vmin, 1e-10f)),
              S.t0max * S.t0max * (1.0f + P.tan2) * 1.0001f);
    const float slo = tlo * P.inv_dt;
    const float shi = fminf(sqrtf(thi2) * P.inv_dt, 1.0e9f);
    *lolo_out = max(static_cast<int>(floorf(slo)) - 2, 0);
    *lohi_out = min(static_cast<int>(floorf(shi)) + 2, P.n_t - 2);
    return *lolo_out <= *lohi_out;
}

// Sample window of trace (dx2, kc) for the forward kernel: elements [ws, we) with ws and we
// multiples of 16 / store_bytes (the TMA granularity) cover lo in [lolo, lohi + 1] (element
// lo holds both interpolation operands; the extra element lets a passing term whose fast
// s rounds up across lohi + 1 read staged data without a clamp); size 0 when the trace has
// no passing term.  we <= ns: lohi + 2 <= n_t and ns is n_t rounded up to 8.
template <int STORE>
__device__ __forceinline__ void trace_window(const FwdParams& P, const TileStats& S, int xa,
                                             int xb, float dx2, int kc, int* ws_out,
                                             int* size_out) {
    constexpr int A = 16 / store_bytes(STORE);
    *ws_out = 0;
    *size_out = 0;
    int lolo, lohi;
    if (!trace_bounds(P, S, xa, xb, dx2, kc, &lolo, &lohi)) return;
    const int ws = lolo & ~(A - 1);
    const int we = (lohi + 1 + A) & ~(A - 1);  // elements [ws, we) cover [lolo, lohi + 1]
    *ws_out = ws;
    *size_out = we - ws;
}

// Staged window of one trace as the consumers see it.
struct Win {
    float wsf;  // first staged sample (float)
    float wef;  // end of the window (float): the debug-bounds build checks s < wef
    int* err;
};

// s of a term, kept inside the staged window.  A term that passes both masks needs no clamp:
// trace_window's bounds (two samples of slack, one extra element) put its floor(s) inside
// [ws, we).  A term that fails them (ok false, only in groups where some lane may fail) can
// have its s anywhere: it reads the window's first sample instead, and its value is dropped.
// The debug-bounds build checks the claim for passing terms and records PSM_DEV_ERR_WINDOW
// instead of reading outside the window.
__device__ __forceinline__ float window_s(float s, bool ok, const Win& w) {
    s = ok ? s : w.wsf;
#ifdef PSM_DEBUG_BOUNDS
    if (!(s >= w.wsf && s < w.wef)) {
        atomicOr(w.err, PSM_DEV_ERR_WINDOW);
        return w.wsf;
    }
#endif
    return s;
}

// One pair of blocks (j, j+1) = (2 pr, 2 pr + 1) for one staged trace.
// Sample n of the staged window sits at byte sbase + base2 + (bits(2^23 + n) << 3), with
// 32-bit wrap-around (see the producer).
// One term of block-pair component (scalar FP32 arithmetic).
template <bool AMP, bool MASK>
__device__ __forceinline__ void term_one(const unsigned char* sbase, float r2, uint32_t base2,
                                         const Win& w, float T2, float F4, float BB,
                                         float& ACC) {
    const bool ok = !MASK || r2 <= BB;                       // both reference masks
    const float t2 = __fmaf_rn(F4, r2, T2);                  // (t / dt)^2
    const float q = rsqrtf(t2);                              // dt / t
    const float s = window_s(t2 * q, ok, w);                 // t / dt inside the window
    const float mm = __fadd_rd(s, 8388608.0f);               // 2^23 + floor(s)
    const float fr = s - (mm - 8388608.0f);                  // frac
    const float2 p =
        *reinterpret_cast<const float2*>(sbase + (base2 + (__float_as_uint(mm) << 3)));
    float v = __fmaf_rn(fr, p.y, p.x);                       // simdInterpolate
    if (MASK) v = ok ? v : 0.0f;
    if (AMP)
        ACC = __fmaf_rn(v, q, ACC);
    else
        ACC += v;
}

template <bool AMP, bool MASK, bool PACKED>
__device__ __forceinline__ void term_pair(const unsigned char* sbase, float r2, uint32_t base2,
                                          const Win& w, const float2& T2,
                                          const float2& F4, const float2& BB, float2& ACC) {
    if (!PACKED) {
        term_one<AMP, MASK>(sbase, r2, base2, w, T2.x, F4.x, BB.x, ACC.x);
        term_one<AMP, MASK>(sbase, r2, base2, w, T2.y, F4.y, BB.y, ACC.y);
        return;
    }
    const bool ok0 = !MASK || r2 <= BB.x, ok1 = !MASK || r2 <= BB.y;  // reference masks
    const float2 t2 = fma2(F4, make_float2(r2, r2), T2);     // (t / dt)^2
    const float q0 = rsqrtf(t2.x), q1 = rsqrtf(t2.y);        // dt / t
    float2 s = mul2(t2, make_float2(q0, q1));                // t / dt
    s.x = window_s(s.x, ok0, w);                             // inside the staged window
    s.y = window_s(s.y, ok1, w);
    const float2 M = make_float2(8388608.0f, 8388608.0f);
    const float2 mm = add2_rm(s, M);                         // 2^23 + floor(s)
    const float2 fr = sub2(s, sub2(mm, M));                  // frac
    const float2 p0 =
        *reinterpret_cast<const float2*>(sbase + (base2 + (__float_as_uint(mm.x) << 3)));
    const float2 p1 =
        *reinterpret_cast<const float2*>(sbase + (base2 + (__float_as_uint(mm.y) << 3)));
    float v0 = fmaf(fr.x, p0.y, p0.x);                       // simdInterpolate
    float v1 = fmaf(fr.y, p1.y, p1.x);
    if (MASK) {
        v0 = ok0 ? v0 : 0.0f;
        v1 = ok1 ? v1 : 0.0f;
    }
    if (AMP)
        ACC = fma2(make_float2(v0, v1), make_float2(q0, q1), ACC);
    else
        ACC = add2(ACC, make_float2(v0, v1));
}

// Block pair of NT staged traces that share r^2 (the mirrored inlines c - d and c + d at one
// crossline): the same travel times, sample indices, fractions and weights.  Interpolation is
// linear in the samples, so the NT staged (d[lo], d[lo+1] - d[lo]) pairs are added first and
// interpolated once; each trace's window has its own base.
// POFF > 0: trace n's window lies n POFF bytes after the first's (base[n] unused).
template <bool AMP, bool MASK, int NT, int POFF>
__device__ __forceinline__ void term_multi(const unsigned char* sbase, float r2,
                                           const uint32_t (&base)[2], const Win& w,
                                           const float2& T2, const float2& F4, const float2& BB,
                                           float2& ACC) {
    const bool ok0 = !MASK || r2 <= BB.x, ok1 = !MASK || r2 <= BB.y;  // reference masks
    const float2 t2 = fma2(F4, make_float2(r2, r2), T2);     // (t / dt)^2
    const float q0 = rsqrtf(t2.x), q1 = rsqrtf(t2.y);        // dt / t
    float2 s = mul2(t2, make_float2(q0, q1));                // t / dt
    s.x = window_s(s.x, ok0, w);                             // inside the staged windows
    s.y = window_s(s.y, ok1, w);
    const float2 M = make_float2(8388608.0f, 8388608.0f);
    const float2 mm = add2_rm(s, M);                         // 2^23 + floor(s)
    const float2 fr = sub2(s, sub2(mm, M));                  // frac
    const uint32_t o0 = __float_as_uint(mm.x) << 3, o1 = __float_as_uint(mm.y) << 3;
    const unsigned char* p0 = sbase + (base[0] + o0);
    const unsigned char* p1 = sbase + (base[0] + o1);
    float2 a0 = *reinterpret_cast<const float2*>(p0);
    float2 a1 = *reinterpret_cast<const float2*>(p1);
#pragma unroll
    for (int n = 1; n < NT; ++n) {
        if (POFF > 0) {
            a0 = add2(a0, *reinterpret_cast<const float2*>(p0 + n * POFF));
            a1 = add2(a1, *reinterpret_cast<const float2*>(p1 + n * POFF));
        } else {
            a0 = add2(a0, *reinterpret_cast<const float2*>(sbase + (base[n] + o0)));
            a1 = add2(a1, *reinterpret_cast<const float2*>(sbase + (base[n] + o1)));
        }
    }
    float2 v = make_float2(fmaf(fr.x, a0.y, a0.x), fmaf(fr.y, a1.y, a1.x));
    if (MASK) {
        v.x = ok0 ? v.x : 0.0f;
        v.y = ok1 ? v.y : 0.0f;
    }
    if (AMP)
        ACC = fma2(v, make_float2(q0, q1), ACC);
    else
        ACC = add2(ACC, v);
}

// Both samples of a 16-bit storage word as fp32 (exact conversions).
template <int STORE>
__device__ __forceinline__ float2 unpack16(uint32_t w) {
    if (STORE == kStoreBF16)
        return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
    return make_float2(__half2float(__ushort_as_half(static_cast<unsigned short>(w & 0xffffu))),
                       __half2float(__ushort_as_half(static_cast<unsigned short>(w >> 16))));
}

// Block pair of one staged trace in 16-bit storage.  Sample n of the staged window sits at
// byte base2 + (bits(2^23 + n) << 2); the interpolation takes the difference of the two
// stored samples in fp32 (b - a, as the reference) and the trace scale joins the weight.
template <bool AMP, bool MASK, int STORE>
__device__ __forceinline__ void term_pair16(const unsigned char* sbase, float r2, uint32_t base2,
                                            const Win& w, float sc, const float2& T2,
                                            const float2& F4, const float2& BB, float2& ACC) {
    const bool ok0 = !MASK || r2 <= BB.x, ok1 = !MASK || r2 <= BB.y;  // reference masks
    const float2 t2 = fma2(F4, make_float2(r2, r2), T2);     // (t / dt)^2
    const float q0 = rsqrtf(t2.x), q1 = rsqrtf(t2.y);        // dt / t
    float2 s = mul2(t2, make_float2(q0, q1));                // t / dt
    s.x = window_s(s.x, ok0, w);                             // inside the staged window
    s.y = window_s(s.y, ok1, w);
    const float2 M = make_float2(8388608.0f, 8388608.0f);
    const float2 mm = add2_rm(s, M);                         // 2^23 + floor(s)
    const float2 fr = sub2(s, sub2(mm, M));                  // frac
    const uint32_t w0 =
        *reinterpret_cast<const uint32_t*>(sbase + (base2 + (__float_as_uint(mm.x) << 2)));
    const uint32_t w1 =
        *reinterpret_cast<const uint32_t*>(sbase + (base2 + (__float_as_uint(mm.y) << 2)));
    const float2 p0 = unpack16<STORE>(w0), p1 = unpack16<STORE>(w1);
    const float2 a = make_float2(p0.x, p1.x);
    float2 v = fma2(fr, sub2(make_float2(p0.y, p1.y), a), a);  // simdInterpolate
    if (MASK) {
        v.x = ok0 ? v.x : 0.0f;
        v.y = ok1 ? v.y : 0.0f;
    }
    if (AMP)
        ACC = fma2(v, mul2(make_float2(q0, q1), make_float2(sc, sc)), ACC);
    else
        ACC = fma2(v, make_float2(sc, sc), ACC);
}

// Block pair of a mirrored pair of staged traces in 16-bit storage: as term_pair2, each trace's
// interpolated value scaled by its own trace scale before the two are added.
template <bool AMP, bool MASK, int STORE, int POFF>
__device__ __forceinline__ void term_pair2_16(const unsigned char* sbase, float r2,
                                              uint32_t base2a, uint32_t base2b, const Win& w,
                                              float sca, float scb, const float2& T2,
                                              const float2& F4, const float2& BB, float2& ACC) {
    const bool ok0 = !MASK || r2 <= BB.x, ok1 = !MASK || r2 <= BB.y;  // reference masks
    const float2 t2 = fma2(F4, make_float2(r2, r2), T2);     // (t / dt)^2
    const float q0 = rsqrtf(t2.x), q1 = rsqrtf(t2.y);        // dt / t
    float2 s = mul2(t2, make_float2(q0, q1));                // t / dt
    s.x = window_s(s.x, ok0, w);                             // inside the staged windows
    s.y = window_s(s.y, ok1, w);
    const float2 M = make_float2(8388608.0f, 8388608.0f);
    const float2 mm = add2_rm(s, M);                         // 2^23 + floor(s)
    const float2 fr = sub2(s, sub2(mm, M));                  // frac
    const uint32_t o0 = __float_as_uint(mm.x) << 2, o1 = __float_as_uint(mm.y) << 2;
    const unsigned char* pa0 = sbase + (base2a + o0);
    const unsigned char* pa1 = sbase + (base2a + o1);
    const unsigned char* pb0 = POFF > 0 ? pa0 + POFF : sbase + (base2b + o0);
    const unsigned char* pb1 = POFF > 0 ? pa1 + POFF : sbase + (base2b + o1);
    const float2 a0 = unpack16<STORE>(*reinterpret_cast<const uint32_t*>(pa0));
    const float2 a1 = unpack16<STORE>(*reinterpret_cast<const uint32_t*>(pa1));
    const float2 b0 = unpack16<STORE>(*reinterpret_cast<const uint32_t*>(pb0));
    const float2 b1 = unpack16<STORE>(*reinterpret_cast<const uint32_t*>(pb1));
    const float2 la = make_float2(a0.x, a1.x), lb = make_float2(b0.x, b1.x);
    const float2 va = fma2(fr, sub2(make_float2(a0.y, a1.y), la), la);  // simdInterpolate
    const float2 vb = fma2(fr, sub2(make_float2(b0.y, b1.y), lb), lb);
    float2 v = fma2(va, make_float2(sca, sca), mul2(vb, make_float2(scb, scb)));
    if (MASK) {
        v.x = ok0 ? v.x : 0.0f;
        v.y = ok1 ? v.y : 0.0f;
    }
    if (AMP)
        ACC = fma2(v, make_float2(q0, q1), ACC);
    else
        ACC = add2(ACC, v);
}

// One block pair of a staged slot: a single trace (fp32 or 16-bit storage), or NT traces
// sharing r^2 (mirrored inlines; 16-bit storage: NT = 2 only).
template <bool AMP, bool MASK, bool PACKED, int STORE, int NT, int POFF>
__device__ __forceinline__ void eval_pair(const unsigned char* sbase, float r2,
                                          const uint32_t (&base)[2], const Win& w, float sc,
                                          float scb, const float2& T2, const float2& F4,
                                          const float2& BB, float2& ACC) {
    static_assert(NT == 1 || NT == 2, "traces per slot");
    if (NT > 1 && STORE == kStoreF32)
        term_multi<AMP, MASK, NT, POFF>(sbase, r2, base, w, T2, F4, BB, ACC);
    else if (NT > 1)
        term_pair2_16<AMP, MASK, STORE, POFF>(sbase, r2, base[0], base[1], w, sc, scb, T2, F4,
                                              BB, ACC);
    else if (STORE == kStoreF32)
        term_pair<AMP, MASK, PACKED>(sbase, r2, base[0], w, T2, F4, BB, ACC);
    else
        term_pair16<AMP, MASK, STORE>(sbase, r2, base[0], w, sc, T2, F4, BB, ACC);
}

// One staged slot for one consumer warp: every block pair of the lane where some lane of its
// group passes, without masks where every lane of the group (or of the tile) passes.
template <bool AMP, bool PACKED, int GB, int J, int STORE, int NT, int POFF>
__device__ __forceinline__ void visit_slot(const unsigned char* sbase, float r2,
                                           const uint32_t (&base)[2], const Win& w,
                                           float sc, float scb,
                                           float gminall, const float (&gmax)[J / GB],
                                           const float (&gmin)[J / GB], const float2 (&T2)[J / 2],
                                           const float2 (&F4)[J / 2], const float2 (&BB)[J / 2],
                                           float2 (&SUM)[J / 2]) {
    constexpr int NG = J / GB;
    constexpr int PG = GB / 2;
    if (r2 <= gminall) {  // interior trace: every term of the tile passes
#pragma unroll
        for (int p = 0; p < J / 2; ++p)
            eval_pair<AMP, false, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc, scb,
                                                            T2[p], F4[p], BB[p], SUM[p]);
        return;
    }
#pragma unroll
    for (int gr = 0; gr < NG; ++gr) {
        if (r2 <= gmax[gr]) {
            if (r2 <= gmin[gr]) {  // every lane of the group passes
#pragma unroll
                for (int p = PG * gr; p < PG * (gr + 1); ++p)
                    eval_pair<AMP, false, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc, scb,
                                                                   T2[p], F4[p], BB[p], SUM[p]);
            } else if constexpr (PG == 2) {
                // some lane may fail: a block pair where no lane passes (the aperture grows
                // with t0, so often the group's shallower pair) is skipped on a warp vote;
                // its terms would add exact zeros.  Both votes come first, so that when both
                // block pairs run they share one basic block and their dependency chains
                // (rsqrt, shared load, interpolation) interleave.
                const int p0 = PG * gr, p1 = p0 + 1;
                const bool a0 = __any_sync(0xffffffffu, r2 <= fmaxf(BB[p0].x, BB[p0].y));
                const bool a1 = __any_sync(0xffffffffu, r2 <= fmaxf(BB[p1].x, BB[p1].y));
                if (a0 && a1) {
                    eval_pair<AMP, true, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc, scb,
                                                                   T2[p0], F4[p0], BB[p0],
                                                                   SUM[p0]);
                    eval_pair<AMP, true, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc, scb,
                                                                   T2[p1], F4[p1], BB[p1],
                                                                   SUM[p1]);
                } else if (a1) {
                    eval_pair<AMP, true, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc, scb,
                                                                   T2[p1], F4[p1], BB[p1],
                                                                   SUM[p1]);
                } else if (a0) {
                    eval_pair<AMP, true, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc, scb,
                                                                   T2[p0], F4[p0], BB[p0],
                                                                   SUM[p0]);
                }
            } else {
#pragma unroll
                for (int p = PG * gr; p < PG * (gr + 1); ++p)
                    if (__any_sync(0xffffffffu, r2 <= fmaxf(BB[p].x, BB[p].y)))
                        eval_pair<AMP, true, PACKED, STORE, NT, POFF>(sbase, r2, base, w, sc,
                                                                       scb, T2[p], F4[p], BB[p],
                                                                       SUM[p]);
            }
        }
    }
}

// Kernel variants: PACKED selects f32x2 or scalar FP32 arithmetic for a block pair; GB is
// the number of 32-sample blocks behind one warp-uniform skip test (2, 4 or 8); J the number
// of 32-sample blocks per lane (the tile covers 32 J output samples).  STORE is the trace
// storage (kStoreF32 pairs, or 16-bit words with a per-trace scale; 16-bit storage always
// uses the packed arithmetic).  KAHAN adds compensated summation: each ring stage (at most
// kMaxG traces) is summed into a fresh partial, and the partials are added to the
// accumulator with Kahan's compensation, so the long sum over the aperture carries no
// growing rounding error.
//
// fwd_tile computes one tile (output row job, crosslines [x0, x0 + kTX), samples
// [T0, T0 + 32 J)) with all 9 warps of the CTA.  The ring's mbarriers are initialised once
// per CTA (ring_init); it counts the ring stages the CTA has used so far, so consecutive tiles
// of a persistent CTA continue the ring's phases (every stage, the end-of-stream marker
// included, is released by the consumers).  Returns false when a bounded wait expired.
// One tile of a batched launch: problem, job of that problem, first crossline and sample.
struct BatchItem {
    int prob, job, x0, T0;
};

// POFF (PAIRS): bytes from a mirrored pair's first window to its second (pair_off_bytes of
// the kernel's CTAs per SM).
template <bool AMP, bool PACKED, int GB, int J, int STORE, bool KAHAN, bool PAIRS = false,
          int POFF = 0>
__device__ __forceinline__ bool fwd_tile(const FwdParams& P, const Job job, int x0, int T0,
                                         unsigned char* smem_raw, const SmemLayout& L,
                                         uint32_t& it) {
    static_assert(GB == 2 || GB == 4 || GB == 8, "skip groups of 2, 4 or 8 blocks");
    static_assert(J % GB == 0, "whole skip groups per lane");
    static_assert(STORE == kStoreF32 || PACKED, "16-bit storage uses packed arithmetic");
    static_assert(!PAIRS || PACKED, "mirrored pairs use packed arithmetic");
    static_assert(!PAIRS || (POFF > 0 && POFF % 16 == 0), "pair windows 16-byte aligned");
    constexpr int NG = J / GB;   // skip groups per lane
    constexpr int EB = store_bytes(STORE);
    // bits(2^23) << log2(EB), modulo 2^32 (see the producer)
    constexpr uint32_t MAGIC = EB == 8 ? 0x58000000u : 0x2C000000u;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + L.full);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem_raw + L.empty);
    StageMeta* meta = reinterpret_cast<StageMeta*>(smem_raw + L.meta);
    TileStats* wstats = reinterpret_cast<TileStats*>(smem_raw + L.stats);
    const uint32_t stage0 = smem_u32(smem_raw + L.stage);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    // ---- consumers: per-sample constants (J / 2 register pairs) and tile statistics
    float2 T2[J / 2], F4[J / 2], BB[J / 2], ACC[J / 2];
    float2 PART[J / 2], CMP[J / 2];  // KAHAN: stage partials and compensation
    float2(&SUM)[J / 2] = KAHAN ? PART : ACC;
    float gmax[NG], gmin[NG];
    float warpmax = -1.0f;
    float gminall = 3.0e38f;  // every lane of every group passes when r2 <= gminall
    const int x = x0 + warp - 1;
    if (warp > 0) {
        const int vc = vrms_col(P, x);
        const bool xvalid = vc >= 0;
        const float* vp = vrms_trace(P, job.vrow, xvalid ? vc : 0);
        float vmin = 3.0e38f, vmax = 0.0f, bmax = -1.0f, t0min = 3.0e38f, t0max = 0.0f;
        float bj[J];
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int t = T0 + 32 * j + lane;
            float v = 0.0f, t0v = 0.0f;
            if (xvalid && t < P.n_t) {
                v = __ldg(vp + t);
                t0v = __ldg(P.t0 + t);
            }
            const PointConst pc = point_const(v, t0v, P.tan2);
            const float b = pass_bound(pc, P.inv_dt, P.ntm1f);
            float t2 = 1.0f, f4 = 0.0f;
            if (b >= 0.0f) {
                t2 = pc.t0sq * P.idt2;
                f4 = pc.f4 * P.idt2;
                vmin = fminf(vmin, v);
                vmax = fmaxf(vmax, v);
                bmax = fmaxf(bmax, b);
                t0min = fminf(t0min, t0v);
                t0max = fmaxf(t0max, t0v);
            }
            bj[j] = b;
            if (j & 1) {
                T2[j >> 1].y = t2;
                F4[j >> 1].y = f4;
                BB[j >> 1].y = b;
            } else {
                T2[j >> 1].x = t2;
                F4[j >> 1].x = f4;
                BB[j >> 1].x = b;
            }
        }
#pragma unroll
        for (int p = 0; p < J / 2; ++p) {
            ACC[p] = make_float2(0.0f, 0.0f);
            CMP[p] = make_float2(0.0f, 0.0f);
        }
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            float mx = bj[GB * g], mn = bj[GB * g];
#pragma unroll
            for (int b = 1; b < GB; ++b) {
                mx = fmaxf(mx, bj[GB * g + b]);
                mn = fminf(mn, bj[GB * g + b]);
            }
            gmax[g] = warp_max(mx);
            gmin[g] = warp_min(mn);
            warpmax = fmaxf(warpmax, gmax[g]);
            gminall = fminf(gminall, gmin[g]);
        }
        vmin = warp_min(vmin);
        vmax = warp_max(vmax);
        bmax = warp_max(bmax);
        t0min = warp_min(t0min);
        t0max = warp_max(t0max);
        if (lane == 0) {
            TileStats s;
            s.vmin = vmin;
            s.vmax = vmax;
            s.bmax = bmax;
            s.t0min = t0min;
            s.t0max = t0max;
            s.any = bmax >= 0.0f;
            wstats[warp - 1] = s;
        }
    }
    __syncthreads();

    if (warp == 0) {
        // ---------------------------------------------------------------- producer
        TileStats S;
        S.vmin = 3.0e38f;
        S.vmax = 0.0f;
        S.bmax = -1.0f;
        S.t0min = 3.0e38f;
        S.t0max = 0.0f;
        S.any = 0;
        for (int w = 0; w < kTX; ++w) {
            const TileStats s = wstats[w];
            if (!s.any) continue;
            S.any = 1;
            S.vmin = fminf(S.vmin, s.vmin);
            S.vmax = fmaxf(S.vmax, s.vmax);
            S.bmax = fmaxf(S.bmax, s.bmax);
            S.t0min = fminf(S.t0min, s.t0min);
            S.t0max = fmaxf(S.t0max, s.t0max);
        }
        // cube crossline range of the tile's output points
        const int xa = max(x0 + P.xoff, 0);
        const int xb = min(min(x0 + kTX, P.n_ox) - 1 + P.xoff,
                           P.compat_pad ? 0x3fffffff : P.n_vx - 1);
        int* inl_klo = reinterpret_cast<int*>(smem_raw + L.inl_klo);
        int* inl_pre = reinterpret_cast<int*>(smem_raw + L.inl_pre);
        float* inl_dx2 = reinterpret_cast<float*>(smem_raw + L.inl_dx2);
        const int n_inl = max(job.i1 - job.i0, 0);
        // rows of the trace list: the buffer inlines, or (PAIRS) the mirror distances d from the
        // centre inline pc, row d holding inlines pc - d and pc + d, whose traces at one
        // crossline have the same r^2 to every output point
        // pairs: a pair's second window lies POFF bytes after its first, so the first windows
        // of all slots fill the stage's first POFF bytes, where a whole window (at most ns
        // samples) must fit
        int pc = -1;
        if (PAIRS && P.pairable && P.ns * EB <= POFF && P.stage_cap * EB >= 2 * POFF &&
            n_inl > 0) {
            const int c = job.pos - __ldg(P.il_pos + job.i0);
            if (c >= 0 && c < n_inl) pc = c;
        }
        const int n_rows = pc >= 0 ? max(pc, n_inl - 1 - pc) + 1 : n_inl;
        const int cap = pc >= 0 ? POFF / EB : P.stage_cap;  // samples of first windows a stage
        int total = 0;
        if (S.any && xa <= xb) {
            // row table: crossline range and running slot count per row
            for (int base = 0; base < n_rows; base += 32) {
                const int n = base + lane;
                int cnt = 0, klo = 0;
                float dx2 = 0.0f;
                if (n < n_rows) {
                    int a, b;
                    row_inlines(pc, n_inl, n, &a, &b);
                    dx2 = inline_dx2(__ldg(P.il_pos + job.i0 + a), job.pos, P.d_il);
                    if (dx2 <= S.bmax) {
                        const int K =
                            static_cast<int>(sqrtf(fmaxf(S.bmax - dx2, 0.0f)) * P.inv_dxl) + 2;
                        klo = max(0, xa - K);
                        cnt = max(0, min(P.n_cx - 1, xb + K) - klo + 1);
                    }
                    inl_klo[n] = klo;
                    inl_dx2[n] = dx2;
                }
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                if (n < n_rows) inl_pre[n] = total + incl - cnt;
                total += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) inl_pre[n_rows] = total;
            __syncwarp();
        }
        bool alive = true;
        const uint32_t it_begin = it;       // the ring iteration of this tile's first stage
        uint32_t stalled = 0xffffffffu;     // test-only stall: the stage left unfilled
        int f = 0;
        while (f < total && alive) {
            const int idx = f + lane;
            int ws = 0, size = 0, kc = 0, row = 0, rowb = -1, slot_size = 0, tx_size = 0;
            float dx2 = 0.0f, sc = 1.0f, scb = 1.0f;
            if (idx < total) {
                // row of flat slot idx: the last n with inl_pre[n] <= idx
                int lo = 0, hi = n_rows - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (inl_pre[mid] <= idx)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                kc = inl_klo[lo] + (idx - inl_pre[lo]);
                dx2 = inl_dx2[lo];
                int a, b;
                row_inlines(pc, n_inl, lo, &a, &b);
                row = job.i0 + a;
                rowb = b >= 0 ? job.i0 + b : -1;
                trace_window<STORE>(P, S, xa, xb, dx2, kc, &ws, &size);
                if (STORE != kStoreF32 && size > 0) {
                    sc = __ldg(P.scales + static_cast<size_t>(row) * P.n_cx + kc);
                    if (rowb >= 0) scb = __ldg(P.scales + static_cast<size_t>(rowb) * P.n_cx + kc);
                }
                slot_size = size;                        // samples of the first region
                tx_size = rowb >= 0 ? 2 * size : size;   // samples copied (a pair: both)
            }
            // inclusive prefix sum of slot sizes; take the lanes that fit one stage
            int cum = slot_size;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, cum, o);
                if (lane >= o) cum += v;
            }
            const bool take = cum <= cap;
            const unsigned takemask = __ballot_sync(0xffffffffu, take);
            const int consumed = __popc(takemask);
            const unsigned nzmask = __ballot_sync(0xffffffffu, take && size > 0);
            const int n = __popc(nzmask);
            if (n > 0) {
                const int stage = it % kStages;
                const uint32_t par = ((it / kStages) & 1u) ^ 1u;
                const int ok = lane == 0 ? mbar_wait(&empty[stage], par, P.err, P.wait_us) : 0;
                if (!__shfl_sync(0xffffffffu, ok, 0)) {
                    alive = false;
                    break;
                }
                // test-only: the tile's first stage is never filled nor arrived on
                const bool stall = (P.fault & kFaultStallProducer) && it == it_begin;
                StageMeta& m = meta[stage];
                const int tot = __reduce_add_sync(0xffffffffu, take ? tx_size : 0);  // samples
                const uint32_t boff =  // a pair's second window from its first (bytes)
                    POFF > 0 ? static_cast<uint32_t>(POFF) : static_cast<uint32_t>(size) * EB;
                const uint32_t dst_rel =
                    L.stage +
                    (static_cast<uint32_t>(stage) * P.stage_cap + (cum - slot_size)) * EB;
                const uint32_t dst = stage0 + (dst_rel - L.stage);
                const int slot = __popc(nzmask & ((1u << lane) - 1u));
                if (take && size > 0) {
                    // consumers find sample n of the window at byte
                    // base2 + (bits(2^23 + n) << log2(EB)) from the shared-memory base (32-bit
                    // wrap-around): base2 = dst_rel - EB ws - (0x4B000000 << log2(EB)); a
                    // pair's second window lies boff bytes after its first
                    m.m[slot] = make_int4(static_cast<int>(dst_rel - EB * ws - MAGIC),
                                          __float_as_int(static_cast<float>(ws)),
                                          static_cast<int>(dst_rel + boff - EB * ws - MAGIC),
                                          rowb >= 0 ? 1 : 0);
                    m.sc[slot] = sc;
                    m.wend[slot] = static_cast<float>(ws + size);
                    m.scb[slot] = scb;
                    // r^2 to each consumer warp's output crossline, with the consumers'
                    // arithmetic (trace_r2), so that each warp reads it instead
                    float rr[kTX];
#pragma unroll
                    for (int w = 0; w < kTX; ++w)
                        rr[w] = trace_r2(kc - (x0 + w + P.xoff), P.d_xl, dx2);
                    float4* r2d = reinterpret_cast<float4*>(&m.r2[slot][0]);
#pragma unroll
                    for (int w = 0; w < kTX; w += 4)
                        r2d[w / 4] = make_float4(rr[w], rr[w + 1], rr[w + 2], rr[w + 3]);
                }
                if (lane == 0) m.count = n;
                __threadfence_block();
                __syncwarp();
                if (lane == 0 && !stall)
                    mbar_arrive_expect_tx(&full[stage], static_cast<uint32_t>(tot) * EB);
                __syncwarp();
                if (stall) {
                    stalled = it;
                } else if (take && size > 0) {
                    const size_t off = (static_cast<size_t>(row) * P.n_cx + kc) * P.ns + ws;
                    const void* src = STORE == kStoreF32
                                          ? static_cast<const void*>(P.pairs + off)
                                          : static_cast<const void*>(P.words + off);
                    tma_load_1d(dst, src, static_cast<uint32_t>(size) * EB, &full[stage]);
                    if (rowb >= 0) {  // the mirrored trace's window, boff bytes on
                        const size_t offb = (static_cast<size_t>(rowb) * P.n_cx + kc) * P.ns + ws;
                        const void* srcb = STORE == kStoreF32
                                               ? static_cast<const void*>(P.pairs + offb)
                                               : static_cast<const void*>(P.words + offb);
                        tma_load_1d(dst + boff, srcb, static_cast<uint32_t>(size) * EB,
                                    &full[stage]);
                    }
                }
                ++it;
            }
            f += consumed;
        }
        // end-of-stream marker
        if (alive) {
            int ok = 1;
            if (lane == 0) {
                const int stage = it % kStages;
                const uint32_t par = ((it / kStages) & 1u) ^ 1u;
                ok = mbar_wait(&empty[stage], par, P.err, P.wait_us);
                if (ok) {
                    meta[stage].count = -1;
                    __threadfence_block();
                    mbar_arrive(&full[stage]);
                }
            }
            alive = __shfl_sync(0xffffffffu, ok, 0) != 0;
            ++it;
        }
        if (!alive && lane == 0) {
            // a wait ran out: before the CTA can exit, let the bulk copies of this tile's
            // last fills land (earlier fills of a stage were consumed before it was refilled);
            // each of these waits is bounded too
            for (uint32_t i = it > it_begin + kStages ? it - kStages : it_begin; i < it; ++i)
                if (i != stalled) mbar_wait(&full[i % kStages], (i / kStages) & 1u, P.err, P.wait_us);
        }
        __syncwarp();
        return alive;
    }

    // -------------------------------------------------------------------- consumers
    bool alive = true;
    while (true) {
        const int stage = it % kStages;
        const uint32_t par = (it / kStages) & 1u;
        if (!mbar_wait(&full[stage], par, P.err, P.wait_us)) {
            alive = false;
            break;
        }
        const StageMeta& m = meta[stage];
        const int cnt = m.count;
        if (cnt < 0) {  // end of stream: release the marker's stage too
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            ++it;
            break;
        }
        if (KAHAN) {
#pragma unroll
            for (int p = 0; p < J / 2; ++p) PART[p] = make_float2(0.0f, 0.0f);
        }
        for (int g = 0; g < cnt; ++g) {
            const float r2 = m.r2[g][warp - 1];
            if (r2 > warpmax) continue;
            const int4 md = m.m[g];
            uint32_t base[2];
            base[0] = static_cast<uint32_t>(md.x);
            Win w;
            w.wsf = __int_as_float(md.y);
#ifdef PSM_DEBUG_BOUNDS
            w.wef = m.wend[g];
#else
            w.wef = 0.0f;
#endif
            w.err = P.err;
            const float sc = STORE == kStoreF32 ? 1.0f : m.sc[g];
            if (PAIRS && md.w) {
                base[1] = static_cast<uint32_t>(md.z);
                visit_slot<AMP, PACKED, GB, J, STORE, 2, POFF>(
                    smem_raw, r2, base, w, sc, STORE == kStoreF32 ? 1.0f : m.scb[g],
                    gminall, gmax, gmin, T2, F4, BB, SUM);
            } else {
                base[1] = 0u;
                visit_slot<AMP, PACKED, GB, J, STORE, 1, 0>(smem_raw, r2, base, w, sc, 1.0f,
                                                            gminall, gmax, gmin, T2, F4, BB,
                                                            SUM);
            }
        }
        if (KAHAN) {  // ACC += PART, compensated
#pragma unroll
            for (int p = 0; p < J / 2; ++p) {
                const float2 y = sub2(PART[p], CMP[p]);
                const float2 t = add2(ACC[p], y);
                CMP[p] = sub2(sub2(t, ACC[p]), y);
                ACC[p] = t;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
        ++it;
    }

    // ---- write the tile: weight 1/(t v^2) = (dt/t) * inv_dt / v^2 applied per output sample
    if (x < P.n_ox) {
        const int vc = vrms_col(P, x);
        const bool xvalid = vc >= 0;
        const float* vp = vrms_trace(P, job.vrow, xvalid ? vc : 0);
        float* op = P.image + (static_cast<size_t>(job.row) * P.n_ox + x) * P.n_t;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int t = T0 + 32 * j + lane;
            if (t < P.n_t) {
                const float b = (j & 1) ? BB[j >> 1].y : BB[j >> 1].x;
                const float a = (j & 1) ? ACC[j >> 1].y : ACC[j >> 1].x;
                float o = 0.0f;
                if (b >= 0.0f) {
                    if (AMP) {
                        const float v = __ldg(vp + t);
                        o = a * __fdiv_rn(P.inv_dt, __fmul_rn(v, v));
                    } else {
                        o = a;
                    }
                }
                op[t] = o;
            }
        }
    }
    return alive;
}

// The ring's mbarriers: full (one producer arrival + the TMA bytes), empty (kTX consumers).
__device__ __forceinline__ void ring_init(unsigned char* smem_raw, const SmemLayout& L) {
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + L.full);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem_raw + L.empty);
    for (int s = 0; s < kStages; ++s) {
        mbar_init(&full[s], 1);
        mbar_init(&empty[s], kTX);
    }
    fence_barrier_init();
}

// One tile per CTA: grid (crossline tiles, jobs, time tiles).  The time tile is the slowest
// dimension, deepest first: the block scheduler starts CTAs in grid order, and a deep tile
// holds several times the terms of a shallow one (the aperture grows with t0), so the light
// tiles come last and the launch's tail is short.
template <int J>
__device__ __forceinline__ int grid_T0() {
    return static_cast<int>(gridDim.z - 1 - blockIdx.z) * 32 * J;
}

template <bool AMP, bool PACKED, int GB, int J, int STORE = kStoreF32, bool KAHAN = false,
          bool PAIRS = false>
__global__ void __launch_bounds__(32 * (kTX + 1), 2) fwd_kernel(const FwdParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const SmemLayout L = smem_layout(P.max_inl, P.stage_cap, store_bytes(STORE));
    if (threadIdx.x == 0) ring_init(smem_raw, L);  // ordered by the tile's first barrier
    uint32_t it = 0;
    fwd_tile<AMP, PACKED, GB, J, STORE, KAHAN, PAIRS, PAIRS ? pair_off_bytes(2) : 0>(
        P, P.jobs[blockIdx.y], blockIdx.x * kTX, grid_T0<J>(), smem_raw, L, it);
}

// The same with 3 CTAs per SM (27 warps): registers are held to 72 per thread and the launcher
// gives it stages of 32 KB, so that three CTAs fit the SM's registers and shared memory.
template <bool AMP, bool PACKED, int GB, int J, int STORE = kStoreF32, bool KAHAN = false,
          bool PAIRS = false>
__global__ void __launch_bounds__(32 * (kTX + 1), 3) fwd_kernel_o3(const FwdParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const SmemLayout L = smem_layout(P.max_inl, P.stage_cap, store_bytes(STORE));
    if (threadIdx.x == 0) ring_init(smem_raw, L);
    uint32_t it = 0;
    fwd_tile<AMP, PACKED, GB, J, STORE, KAHAN, PAIRS, PAIRS ? pair_off_bytes(3) : 0>(
        P, P.jobs[blockIdx.y], blockIdx.x * kTX, grid_T0<J>(), smem_raw, L, it);
}

// The same with 4 CTAs per SM (36 warps): 56 registers per thread and 20 KB stages; for
// tiles of 128 samples (J = 4), whose per-lane state is half that of J = 8.
template <bool AMP, bool PACKED, int GB, int J, int STORE = kStoreF32, bool KAHAN = false,
          bool PAIRS = false>
__global__ void __launch_bounds__(32 * (kTX + 1), 4) fwd_kernel_o4(const FwdParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const SmemLayout L = smem_layout(P.max_inl, P.stage_cap, store_bytes(STORE));
    if (threadIdx.x == 0) ring_init(smem_raw, L);
    uint32_t it = 0;
    fwd_tile<AMP, PACKED, GB, J, STORE, KAHAN, PAIRS, PAIRS ? pair_off_bytes(4) : 0>(
        P, P.jobs[blockIdx.y], blockIdx.x * kTX, grid_T0<J>(), smem_raw, L, it);
}

// Parameters of every problem of a batched launch, passed by value: they live in the
// kernel-parameter constant bank, whose loads are cached and uniform across the CTA.
constexpr int kMaxBatchProblems = 184;
struct BatchParams {
    FwdParams p[kMaxBatchProblems];
};
static_assert(sizeof(BatchParams) + 64 <= 32764, "kernel parameters are limited to 32764 bytes");

// Persistent batched launch: each CTA takes tiles from the shared list in order (an atomic
// counter) until the list is exhausted, with the ring kept across tiles.  Problems (velocity
// panels, sub-volumes) each have their own FwdParams.  max_inl and stage_cap are the largest
// over the problems.  A device error (bounded wait expired) stops every CTA at its next tile.
// MINB: CTAs per SM the kernel is built for (3: the grid kernels' fwd_kernel_o3 budget of 72
// registers, with 32 KB stages from the host).
template <bool AMP, bool PACKED, int GB, int J, int STORE = kStoreF32, bool KAHAN = false,
          bool PAIRS = false, int MINB = 2>
__global__ void __launch_bounds__(32 * (kTX + 1), MINB)
    fwd_batch_kernel(const __grid_constant__ BatchParams B,
                     const BatchItem* __restrict__ items, int n_items, int* next,
                     const int* err, int max_inl, int stage_cap) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ BatchItem s_item;
    __shared__ Job s_job;
    const SmemLayout L = smem_layout(max_inl, stage_cap, store_bytes(STORE));
    if (threadIdx.x == 0) ring_init(smem_raw, L);
    uint32_t it = 0;
    while (true) {
        if (threadIdx.x == 0) {
            const int k = *reinterpret_cast<const volatile int*>(err) ? n_items
                                                                      : atomicAdd(next, 1);
            s_item = k < n_items ? items[k] : BatchItem{-1, 0, 0, 0};
            if (k < n_items) s_job = B.p[s_item.prob].jobs[s_item.job];
        }
        __syncthreads();
        const BatchItem w = s_item;
        if (w.prob < 0) break;
        const bool ok = fwd_tile<AMP, PACKED, GB, J, STORE, KAHAN, PAIRS,
                                 PAIRS ? pair_off_bytes(MINB) : 0>(
            B.p[w.prob], s_job, w.x0, w.T0, smem_raw, L, it);
        // barrier: the tile's tables, statistics, s_item and s_job are reused next
        if (__syncthreads_or(!ok)) break;
    }
}

// The same tile list in ONE grid launch: CTA b migrates tile items[b] (deepest tiles first in
// the depth-first order), and the hardware's block scheduler hands tiles to SMs as others
// finish, so the CTAs carry no state from tile to tile.
template <bool AMP, bool PACKED, int GB, int J, int STORE = kStoreF32, bool KAHAN = false,
          bool PAIRS = false, int MINB = 2>
__global__ void __launch_bounds__(32 * (kTX + 1), MINB)
    fwd_items_kernel(const __grid_constant__ BatchParams B, const BatchItem* __restrict__ items,
                     int max_inl, int stage_cap) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const SmemLayout L = smem_layout(max_inl, stage_cap, store_bytes(STORE));
    if (threadIdx.x == 0) ring_init(smem_raw, L);
    const BatchItem w = items[blockIdx.x];
    const FwdParams& P = B.p[w.prob];
    uint32_t it = 0;
    fwd_tile<AMP, PACKED, GB, J, STORE, KAHAN, PAIRS, PAIRS ? pair_off_bytes(MINB) : 0>(
        P, P.jobs[w.job], w.x0, w.T0, smem_raw, L, it);
}

// Padded output inlines repeat the migrated edge inline (main.cpp:268-285): row copies[k].x of
// the image gets row copies[k].y, every copy in one launch (a source row is never a
// destination).
__global__ void copy_rows_kernel(float* __restrict__ img, const int2* __restrict__ copies,
                                 int n_copies, size_t row) {
    const size_t total = static_cast<size_t>(n_copies) * row;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int k = static_cast<int>(i / row);
        const size_t e = i - static_cast<size_t>(k) * row;
        const int2 cp = copies[k];
        img[static_cast<size_t>(cp.x) * row + e] = img[static_cast<size_t>(cp.y) * row + e];
    }
}

// ----------------------------------------------------------------------------- term count

// One block per (job, output crossline); threads stride over t.  out[job] += terms.
// A term passes when r^2 <= B (pass_bound); r^2 grows with |k - x|, so for each buffer
// inline the passing crosslines are |k - x| <= d with d found from sqrt(B - dx^2) and exact
// fix-ups.
__global__ void count_kernel(const FwdParams P, unsigned long long* out) {
    __shared__ unsigned long long wsum[32];
    const int x = blockIdx.x;
    const Job job = P.jobs[blockIdx.y];
    const int xv = x + P.xoff;
    // the farthest trace of the cube from crossline xv (xv >= 0; beyond n_cx - 1 with
    // compat_pad), plus one
    const int dcap = max(xv, P.n_cx - 1 - xv) + 1;
    unsigned long long local = 0;
    for (int t = threadIdx.x; t < P.n_t; t += blockDim.x) {
        const int vc = vrms_col(P, x);
        if (vc < 0) break;
        const float v = vrms_trace(P, job.vrow, vc)[t];
        const PointConst pc = point_const(v, P.t0[t], P.tan2);
        const float B = pass_bound(pc, P.inv_dt, P.ntm1f);
        if (B < 0.0f) continue;
        for (int i = job.i0; i < job.i1; ++i) {
            const float dx2 = inline_dx2(P.il_pos[i], job.pos, P.d_il);
            if (dx2 > B) continue;  // d = 0 passes from here on
            int d = static_cast<int>(sqrtf(fmaxf(B - dx2, 0.0f)) * P.inv_dxl);
            d = min(d, dcap);
            while (d > 0 && trace_r2(d, P.d_xl, dx2) > B) --d;
            while (d < dcap && trace_r2(d + 1, P.d_xl, dx2) <= B) ++d;
            const int lo = max(0, xv - d), hi = min(P.n_cx - 1, xv + d);
            if (hi >= lo) local += static_cast<unsigned long long>(hi - lo + 1);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += wsum[w];
        if (s) atomicAdd(out + blockIdx.y, s);
    }
}

}  // namespace psm
