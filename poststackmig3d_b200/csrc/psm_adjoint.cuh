// Adjoint of the migration operator (demigration / spray), sm_100a.
//
// The forward kernel computes, for every passing term, val = fma(frac, d[lo+1]-d[lo], d[lo])
// = (1 - frac) d[lo] + frac d[lo+1], weighted by q K (q = dt/t, K = inv_dt / v^2, or 1 with
// amplitude correction off) and summed into the output sample.  Its transpose spreads each
// image sample m back along the same hyperbolae:
//     d[lo]   += (1 - frac) * q K m        d[lo+1] += frac * q K m
// for exactly the same terms (same masks B, same travel time, same frac and q), so the pair
// passes the dot-product test to FP32 summation noise.
//
// Same tile decomposition as fwd_kernel.  The producer stages no data: each ring stage is a
// zeroed shared-memory accumulator holding one fp32 window per listed trace; consumers add
// into it with shared-memory atomics; once a stage is released, the producer adds every
// window into the data cube in HBM with a TMA bulk reduction (cp.reduce.async.bulk .add.f32)
// and waits for the reduction to have read the stage before zeroing and reusing it.  As in
// the forward, the traces at inlines c - d and c + d of one crossline (mirrored about the
// output inline c) have the same r^2 to every output point, hence the same travel times,
// fractions and weights: every term adds the same two shares to both.  They share one slot
// and ONE window, which the flush adds into both traces (two bulk reductions of the same
// shared-memory window), so a pair costs the atomics of a single trace.
#pragma once

#include "psm_kernels.cuh"

namespace psm {

struct AdjParams {
    FwdParams F;          // geometry, tables, constants (F.pairs unused)
    const float* image;   // [n_jobs][n_ox][n_t]: image of each job (duplicate rows folded)
    float* data;          // [n_ci][n_cx][ns] accumulated in place (zero it first)
    double* data64;       // fixed-point form: [n_ci][n_cx][ns] accumulated in FP64 instead
};

struct AdjMeta {
    int count;         // slots in this stage, -1 = end of stream
    int tot;           // samples of the stage's windows, which lie from the stage's start
    int pad[2];
    int m[kMaxG];      // window base (smem bytes)
    int4 g[kMaxG];     // flush: cube row, crossline, window start, window length (samples)
    int rowb[kMaxG];   // paired slots: cube row of the mirrored trace (-1: none), which the
                       // flush adds the same window into
    float r2[kMaxG][kTX];  // r^2 of the slot's trace(s) to each consumer warp's crossline
};

struct AdjLayout {
    unsigned full, empty, meta, stats, mk, inl_klo, inl_pre, inl_dx2, stage, total;
};

// Windows of eb-byte samples (4: fp32 sums; 8: 64-bit fixed-point sums); cap counts samples
// per stage.
__host__ __device__ inline AdjLayout adj_layout(int max_inl, int cap, int eb = 4) {
    AdjLayout L;
    unsigned o = 0;
    L.full = o;
    o += 8 * kStages;
    L.empty = o;
    o += 8 * kStages;
    L.meta = o = (o + 15) & ~15u;
    o += sizeof(AdjMeta) * kStages;
    L.stats = o;
    o += sizeof(TileStats) * kTX;
    L.mk = o;  // per consumer warp: max |m K| of its samples (fixed-point scale)
    o += 4 * kTX;
    L.inl_klo = o;
    o += 4 * max_inl;
    L.inl_pre = o;
    o += 4 * (max_inl + 1);
    L.inl_dx2 = o;
    o += 4 * max_inl;
    L.stage = o = (o + 127) & ~127u;
    o += static_cast<unsigned>(eb) * cap * kStages;
    L.total = o;
    return L;
}

constexpr uint32_t kMagic4 = 0x2C000000u;  // (0x4B000000 << 2) mod 2^32
constexpr uint32_t kMagic8 = 0x58000000u;  // (0x4B000000 << 3) mod 2^32

// Fixed-point sums: a tile's shares are held as integers in units of 2^-s, s = 50 - e with
// max |m K| over the tile < 2^e, so that every share (|m K q (1 - frac)| <= |m K|, q <= 1) is
// below 2^50 and a window sample's sum of the stage's few dozen shares stays far inside
// 64 bits; integer adds are exact and independent of their order.
constexpr int kFixBits = 50;
__device__ __forceinline__ int fix_shift(float mkmax) {
    if (!(mkmax > 0.0f)) return 0;
    int e;
    frexpf(mkmax, &e);  // mkmax < 2^e
    return max(-100, min(100, kFixBits - e));
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_reduce_add_f32(float* dst_global, uint32_t src_smem,
                                                    uint32_t bytes) {
    asm volatile(
        "cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(
            dst_global),
        "r"(src_smem), "r"(bytes)
        : "memory");
}
__device__ __forceinline__ void bulk_reduce_add_f64(double* dst_global, uint32_t src_smem,
                                                    uint32_t bytes) {
    asm volatile(
        "cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(
            dst_global),
        "r"(src_smem), "r"(bytes)
        : "memory");
}
__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Producer: the window of trace (dx2, kc): samples [ws, we) cover lo and lo + 1 of every
// passing term of the tile; ws and we multiples of A = 16 bytes / sample size (the bulk-copy
// granularity).  trace_bounds puts lo of a passing term in [lolo, lohi + 1] (the extra sample
// for a fast s that rounds up across lohi + 1), and the consumers keep s below n_t - 1, so
// lo + 1 <= min(lohi + 2, n_t - 1): the window covers samples up to lohi + 2, or to the row's
// end.
template <int A>
__device__ __forceinline__ void adj_window(const FwdParams& P, const TileStats& S, int xa,
                                           int xb, float dx2, int kc, int* ws_out,
                                           int* size_out) {
    *ws_out = 0;
    *size_out = 0;
    int lolo, lohi;
    if (!trace_bounds(P, S, xa, xb, dx2, kc, &lolo, &lohi)) return;
    const int ws = lolo & ~(A - 1);
    const int we = min((lohi + 2 + A) & ~(A - 1), P.ns);  // ns >= n_t, a multiple of 8
    *ws_out = ws;
    *size_out = we - ws;
}

// One term of the transpose (scalar FP32) for a slot: the forward's s, frac and q, then two
// atomic adds into the slot's window.  A failing term (MASK) returns before touching memory;
// a passing term's lo lies in its window (adj_window), with s held below n_t - 1 (smax) so
// that lo + 1 stays on the trace.
// FIX: MK is m K in units of 2^-s (exact power-of-two scaling); the shares go into the
// window as 64-bit integers (rounded to nearest).
template <bool AMP, bool MASK, bool FIX>
__device__ __forceinline__ void adj_term(unsigned char* sbase, float r2, uint32_t base,
                                         float smax, float T2, float F4, float BB, float MK) {
    const float t2 = __fmaf_rn(F4, r2, T2);
    const float q = rsqrtf(t2);
    const float s = fminf(t2 * q, smax);
    const float mm = __fadd_rd(s, 8388608.0f);
    const float fr = s - (mm - 8388608.0f);
    if (MASK && !(r2 <= BB)) return;
    const float c = AMP ? MK * q : MK;
    const float c1 = c * fr;
    const float c0 = c - c1;
    if (FIX) {
        unsigned long long* p = reinterpret_cast<unsigned long long*>(
            sbase + (base + (__float_as_uint(mm) << 3)));
        atomicAdd(p, static_cast<unsigned long long>(__float2ll_rn(c0)));
        atomicAdd(p + 1, static_cast<unsigned long long>(__float2ll_rn(c1)));
    } else {
        float* p = reinterpret_cast<float*>(sbase + (base + (__float_as_uint(mm) << 2)));
        atomicAdd(p, c0);
        atomicAdd(p + 1, c1);
    }
}

// One slot for one consumer warp: the groups of blocks where some lane passes, without masks
// where every lane of the group passes.
// Two terms of one lane for a slot: samples t and t + 1 (blocks j and j + 1), fp32 sums.
// With ds/dt0 <= 1 their floor(s) are equal or adjacent, so their four shares fall on at
// most three window addresses: lo_a (c0_a), lo_a + 1 (c1_a, and c0_b when lo_b = lo_a + 1),
// lo_a + 2 (c1_b); the lane adds the shares that meet in registers first and issues three
// atomics where the two terms alone would issue four (two when lo_b = lo_a).  A term that
// fails the masks (MASK) contributes nothing and its address is never used; lo_b beyond
// lo_a + 1 (a steep Vrms) takes its own two atomics.
template <bool AMP, bool MASK>
__device__ __forceinline__ void adj_term2(unsigned char* sbase, float r2, uint32_t base,
                                          float smax, float T2a, float F4a, float BBa,
                                          float MKa, float T2b, float F4b, float BBb,
                                          float MKb) {
    const float2 t2 = fma2(make_float2(F4a, F4b), make_float2(r2, r2), make_float2(T2a, T2b));
    const float qa = rsqrtf(t2.x), qb = rsqrtf(t2.y);
    const float sa = fminf(t2.x * qa, smax), sb = fminf(t2.y * qb, smax);
    const float ma = __fadd_rd(sa, 8388608.0f), mb = __fadd_rd(sb, 8388608.0f);
    const float fa = sa - (ma - 8388608.0f), fb = sb - (mb - 8388608.0f);
    const bool oka = !MASK || r2 <= BBa, okb = !MASK || r2 <= BBb;
    if (MASK && !oka && !okb) return;
    const float ca = AMP ? MKa * qa : MKa, cb = AMP ? MKb * qb : MKb;
    const float c1a = oka ? ca * fa : 0.0f, c0a = oka ? ca - ca * fa : 0.0f;
    const float c1b = okb ? cb * fb : 0.0f, c0b = okb ? cb - cb * fb : 0.0f;
    const uint32_t la = __float_as_uint(ma), lb = __float_as_uint(mb);  // 2^23 + floor(s)
    const uint32_t l0 = oka ? la : lb;  // the first address the lane adds to
    const uint32_t d = lb - l0;         // 0, 1, or more (only when both pass)
    float* p = reinterpret_cast<float*>(sbase + (base + (l0 << 2)));
    const bool far = okb && d > 1u;
    atomicAdd(p, c0a + (okb && d == 0u ? c0b : 0.0f));
    atomicAdd(p + 1, c1a + (okb && d == 0u ? c1b : 0.0f) + (okb && d == 1u ? c0b : 0.0f));
    if (okb && d == 1u) atomicAdd(p + 2, c1b);
    if (far) {
        float* q = reinterpret_cast<float*>(sbase + (base + (lb << 2)));
        atomicAdd(q, c0b);
        atomicAdd(q + 1, c1b);
    }
}

template <bool AMP, bool FIX>
__device__ __forceinline__ void adj_visit(unsigned char* sbase, float r2, uint32_t base,
                                          float smax,
                                          const float (&gmax)[2], const float (&gmin)[2],
                                          const float (&T2)[kJ], const float (&F4)[kJ],
                                          const float (&BB)[kJ], const float (&MK)[kJ]) {
#pragma unroll
    for (int gr = 0; gr < 2; ++gr) {
        if (r2 <= gmax[gr]) {
            if (FIX) {  // exact integer shares: each term on its own
                if (r2 <= gmin[gr]) {
#pragma unroll
                    for (int j = 4 * gr; j < 4 * gr + 4; ++j)
                        adj_term<AMP, false, FIX>(sbase, r2, base, smax, T2[j], F4[j], BB[j],
                                                  MK[j]);
                } else {
#pragma unroll
                    for (int j = 4 * gr; j < 4 * gr + 4; ++j)
                        adj_term<AMP, true, FIX>(sbase, r2, base, smax, T2[j], F4[j], BB[j],
                                                 MK[j]);
                }
            } else if (r2 <= gmin[gr]) {  // blocks j, j + 1 hold samples t, t + 1
#pragma unroll
                for (int j = 4 * gr; j < 4 * gr + 4; j += 2)
                    adj_term2<AMP, false>(sbase, r2, base, smax, T2[j], F4[j], BB[j], MK[j],
                                          T2[j + 1], F4[j + 1], BB[j + 1], MK[j + 1]);
            } else {
#pragma unroll
                for (int j = 4 * gr; j < 4 * gr + 4; j += 2)
                    adj_term2<AMP, true>(sbase, r2, base, smax, T2[j], F4[j], BB[j], MK[j],
                                         T2[j + 1], F4[j + 1], BB[j + 1], MK[j + 1]);
            }
        }
    }
}

// Add the windows of one released stage into the data cube (one bulk reduction per window and
// trace, lanes in parallel; a pair's window goes to both of its traces) and wait until they
// have read shared memory.  FIX: the stage's 64-bit integer sums are first turned into FP64
// in place (times 2^-s, exact below 2^53), and the data cube accumulates in FP64.
template <bool FIX>
__device__ __forceinline__ void adj_flush(const AdjParams& A, const AdjMeta& m,
                                          unsigned char* stage, uint32_t smem_abs, int lane,
                                          double inv_scale) {
    if (FIX) {
        long long* w = reinterpret_cast<long long*>(stage);
        for (int i = lane; i < m.tot; i += 32)
            reinterpret_cast<double*>(w)[i] = static_cast<double>(w[i]) * inv_scale;
        __syncwarp();
    }
    fence_proxy_async_smem();  // the shared-memory sums -> the async proxy
    if constexpr (FIX) {
        for (int k = lane; k < m.count; k += 32) {
            const int4 gg = m.g[k];  // row, crossline, ws, size
            const uint32_t rel = static_cast<uint32_t>(m.m[k]) + 8u * gg.z + kMagic8;
            bulk_reduce_add_f64(
                A.data64 + (static_cast<size_t>(gg.x) * A.F.n_cx + gg.y) * A.F.ns + gg.z,
                smem_abs + rel, 8u * gg.w);
            const int rb = m.rowb[k];
            if (rb >= 0)
                bulk_reduce_add_f64(
                    A.data64 + (static_cast<size_t>(rb) * A.F.n_cx + gg.y) * A.F.ns + gg.z,
                    smem_abs + rel, 8u * gg.w);
        }
    } else {
        for (int k = lane; k < m.count; k += 32) {
            const int4 gg = m.g[k];  // row, crossline, ws, size
            const uint32_t rel = static_cast<uint32_t>(m.m[k]) + 4u * gg.z + kMagic4;
            bulk_reduce_add_f32(
                A.data + (static_cast<size_t>(gg.x) * A.F.n_cx + gg.y) * A.F.ns + gg.z,
                smem_abs + rel, 4u * gg.w);
            const int rb = m.rowb[k];
            if (rb >= 0)
                bulk_reduce_add_f32(
                    A.data + (static_cast<size_t>(rb) * A.F.n_cx + gg.y) * A.F.ns + gg.z,
                    smem_abs + rel, 4u * gg.w);
        }
    }
    bulk_commit();
    bulk_wait_read_all();
    __syncwarp();
}

// MINB: CTAs per SM the kernel is built for (the host gives 3-CTA launches 32 KB stages): the
// kernel is bound by the latency of its shared-memory atomics, which more warps hide.
// FIX: 64-bit fixed-point window sums and an FP64 data cube (A.data64); else fp32 atomics and
// an fp32 data cube (A.data).
template <bool AMP, int MINB = 2, bool FIX = false>
__global__ void __launch_bounds__(32 * (kTX + 1), MINB) adj_kernel(const AdjParams A) {
    constexpr int EB = FIX ? 8 : 4;           // bytes of a window sample
    constexpr uint32_t MAGIC = FIX ? kMagic8 : kMagic4;
    const FwdParams& P = A.F;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const AdjLayout L = adj_layout(P.max_inl, P.stage_cap, EB);
    float* mkw = reinterpret_cast<float*>(smem_raw + L.mk);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + L.full);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem_raw + L.empty);
    AdjMeta* meta = reinterpret_cast<AdjMeta*>(smem_raw + L.meta);
    TileStats* wstats = reinterpret_cast<TileStats*>(smem_raw + L.stats);
    const uint32_t smem_abs = smem_u32(smem_raw);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int jobi = blockIdx.y;  // grid (crossline tiles, jobs, time tiles), deepest first
    const Job job = P.jobs[jobi];
    const int x0 = blockIdx.x * kTX;
    const int T0 = static_cast<int>(gridDim.z - 1 - blockIdx.z) * kTT;

    float T2[kJ], F4[kJ], BB[kJ], MK[kJ];
    float gmax[2], gmin[2];
    float warpmax = -1.0f;
    const int x = x0 + warp - 1;
    if (warp > 0) {
        const int vc = vrms_col(P, x);
        const bool xvalid = vc >= 0;
        const float* vp = vrms_trace(P, job.vrow, xvalid ? vc : 0);
        const float* mp = A.image + (static_cast<size_t>(jobi) * P.n_ox +
                                     (x < P.n_ox ? x : 0)) * P.n_t;
        float vmin = 3.0e38f, vmax = 0.0f, bmax = -1.0f, t0min = 3.0e38f, t0max = 0.0f;
        // lane l holds samples T0 + 64 (j / 2) + 2 l + (j % 2): the 32 lanes of one block
        // are two samples apart, so their trace samples (ds/dt0 = t0 / t >= cos(aperture)
        // inside the aperture, 0.7 at 45 deg) fall on different window addresses, and the
        // shared-memory atomics of one instruction do not collide (the forward's mapping,
        // consecutive samples across lanes, puts about one lane in five on its neighbour's
        // address, which halves the atomics' rate); groups of 4 blocks still span 128
        // consecutive samples
#pragma unroll
        for (int j = 0; j < kJ; ++j) {
            const int t = T0 + 64 * (j >> 1) + 2 * lane + (j & 1);
            float v = 0.0f, t0v = 0.0f, mv = 0.0f;
            if (xvalid && t < P.n_t) {
                v = __ldg(vp + t);
                t0v = __ldg(P.t0 + t);
                mv = __ldg(mp + t);
            }
            const PointConst pc = point_const(v, t0v, P.tan2);
            const float b = pass_bound<false>(pc, P.inv_dt, P.ntm1f);
            T2[j] = 1.0f;
            F4[j] = 0.0f;
            MK[j] = 0.0f;
            if (b >= 0.0f) {
                T2[j] = pc.t0sq * P.idt2;
                F4[j] = pc.f4 * P.idt2;
                MK[j] = AMP ? mv * __fdiv_rn(P.inv_dt, __fmul_rn(v, v)) : mv;
                vmin = fminf(vmin, v);
                vmax = fmaxf(vmax, v);
                bmax = fmaxf(bmax, b);
                t0min = fminf(t0min, t0v);
                t0max = fmaxf(t0max, t0v);
            }
            BB[j] = b;
        }
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            float mx = BB[4 * g], mn = BB[4 * g];
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                mx = fmaxf(mx, BB[4 * g + k]);
                mn = fminf(mn, BB[4 * g + k]);
            }
            gmax[g] = warp_max(mx);
            gmin[g] = warp_min(mn);
            warpmax = fmaxf(warpmax, gmax[g]);
        }
        vmin = warp_min(vmin);
        vmax = warp_max(vmax);
        bmax = warp_max(bmax);
        t0min = warp_min(t0min);
        t0max = warp_max(t0max);
        float mkm = 0.0f;
#pragma unroll
        for (int j = 0; j < kJ; ++j) mkm = fmaxf(mkm, fabsf(MK[j]));
        mkm = warp_max(mkm);
        if (lane == 0) {
            TileStats s;
            s.vmin = vmin;
            s.vmax = vmax;
            s.bmax = bmax;
            s.t0min = t0min;
            s.t0max = t0max;
            s.any = bmax >= 0.0f;
            wstats[warp - 1] = s;
            mkw[warp - 1] = mkm;
        }
    } else if (lane == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTX);
        }
        fence_barrier_init();
    }
    __syncthreads();
    // fixed-point scale of the tile: shares in units of 2^-s (fix_shift)
    int shift = 0;
    if (FIX) {
        float mkmax = 0.0f;
        for (int w = 0; w < kTX; ++w) mkmax = fmaxf(mkmax, mkw[w]);
        shift = fix_shift(mkmax);
        if (warp > 0) {
            const float sc = ldexpf(1.0f, shift);
#pragma unroll
            for (int j = 0; j < kJ; ++j) MK[j] *= sc;
        }
    }

    if (warp == 0) {
        // ---------------------------------------------------------------- producer
        const double inv_scale = ldexp(1.0, -shift);
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
        const int xa = max(x0 + P.xoff, 0);
        const int xb = min(min(x0 + kTX, P.n_ox) - 1 + P.xoff,
                           P.compat_pad ? 0x3fffffff : P.n_vx - 1);
        int* inl_klo = reinterpret_cast<int*>(smem_raw + L.inl_klo);
        int* inl_pre = reinterpret_cast<int*>(smem_raw + L.inl_pre);
        float* inl_dx2 = reinterpret_cast<float*>(smem_raw + L.inl_dx2);
        const int n_inl = max(job.i1 - job.i0, 0);
        // rows of the trace list: the buffer inlines, or the mirror distances d from the centre
        // inline pc (row d holds inlines pc - d and pc + d; see row_inlines)
        int pc = -1;  // a pair needs one window (at most ns <= stage_cap samples)
        if (P.pairable && n_inl > 0) {
            const int c = job.pos - __ldg(P.il_pos + job.i0);
            if (c >= 0 && c < n_inl) pc = c;
        }
        const int n_rows = pc >= 0 ? max(pc, n_inl - 1 - pc) + 1 : n_inl;
        int total = 0;
        if (S.any && xa <= xb) {
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
        uint32_t it = 0;
        bool alive = true;
        int f = 0;
        while (f < total && alive) {
            const int idx = f + lane;
            int ws = 0, size = 0, kc = 0, row = 0, rowb = -1, slot_size = 0;
            float dx2 = 0.0f;
            if (idx < total) {
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
                adj_window<16 / EB>(P, S, xa, xb, dx2, kc, &ws, &size);
                slot_size = size;  // a pair shares one window
            }
            int cum = slot_size;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, cum, o);
                if (lane >= o) cum += v;
            }
            const bool take = cum <= P.stage_cap;
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
                AdjMeta& m = meta[stage];
                unsigned char* stage_ptr =
                    smem_raw + L.stage + static_cast<uint32_t>(EB) * stage * P.stage_cap;
                if (it >= static_cast<uint32_t>(kStages))
                    adj_flush<FIX>(A, m, stage_ptr, smem_abs, lane, inv_scale);
                const int tot = __shfl_sync(0xffffffffu, take ? cum : 0, consumed - 1);
                // zero the accumulator region of the new windows (16 B per lane per step;
                // windows are 16-byte multiples)
                float4* z = reinterpret_cast<float4*>(stage_ptr);
                for (int k = lane; k < tot * EB / 16; k += 32)
                    z[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                const uint32_t dst_rel =
                    L.stage + (static_cast<uint32_t>(stage) * P.stage_cap + (cum - slot_size)) *
                                  static_cast<uint32_t>(EB);
                const int slot = __popc(nzmask & ((1u << lane) - 1u));
                if (lane == 0) m.tot = tot;
                if (take && size > 0) {
                    m.m[slot] = static_cast<int>(dst_rel - static_cast<uint32_t>(EB) * ws - MAGIC);
                    m.g[slot] = make_int4(row, kc, ws, size);
                    m.rowb[slot] = rowb;
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
                if (lane == 0) mbar_arrive(&full[stage]);
                ++it;
            }
            f += consumed;
        }
        if (alive) {
            // end-of-stream marker in the next stage, after flushing that stage's last use
            const int stage = it % kStages;
            const uint32_t par = ((it / kStages) & 1u) ^ 1u;
            const int ok = lane == 0 ? mbar_wait(&empty[stage], par, P.err, P.wait_us) : 0;
            if (__shfl_sync(0xffffffffu, ok, 0)) {
                if (it >= static_cast<uint32_t>(kStages))
                    adj_flush<FIX>(A, meta[stage],
                                   smem_raw + L.stage + static_cast<uint32_t>(EB) * stage * P.stage_cap,
                                   smem_abs, lane, inv_scale);
                if (lane == 0) {
                    meta[stage].count = -1;
                    __threadfence_block();
                    mbar_arrive(&full[stage]);
                }
                // the other stage's last use (iteration it - 1), once the consumers release it
                if (it >= 1) {
                    const uint32_t last = it - 1;
                    const int s2 = last % kStages;
                    const uint32_t par2 = (last / kStages) & 1u;
                    const int ok2 = lane == 0 ? mbar_wait(&empty[s2], par2, P.err, P.wait_us) : 0;
                    if (__shfl_sync(0xffffffffu, ok2, 0))
                        adj_flush<FIX>(A, meta[s2],
                                       smem_raw + L.stage + static_cast<uint32_t>(EB) * s2 * P.stage_cap,
                                       smem_abs, lane, inv_scale);
                }
            }
        }
        bulk_wait_all();  // every reduction complete before the CTA retires
        return;
    }

    // -------------------------------------------------------------------- consumers
    uint32_t it = 0;
    while (true) {
        const int stage = it % kStages;
        const uint32_t par = (it / kStages) & 1u;
        if (!mbar_wait(&full[stage], par, P.err, P.wait_us)) break;
        const AdjMeta& m = meta[stage];
        const int cnt = m.count;
        if (cnt < 0) break;
        for (int g = 0; g < cnt; ++g) {
            const float r2 = m.r2[g][warp - 1];
            if (r2 > warpmax) continue;
            adj_visit<AMP, FIX>(smem_raw, r2, static_cast<uint32_t>(m.m[g]), P.ntm1m, gmax, gmin,
                                T2, F4, BB, MK);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
        ++it;
    }
}

// out[i] = float(in[i]) (the FP64 data cube of the fixed-point adjoint to the fp32 vector).
__global__ void f64_to_f32_kernel(const double* __restrict__ in, float* __restrict__ out,
                                  size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}

// Sum the image rows that repeat one migrated inline (the transpose of the forward's row
// copies): out[job] = sum of image rows mapped to that job.
__global__ void fold_rows_kernel(const float* __restrict__ image, const int* __restrict__ map,
                                 const int* __restrict__ map_off, int n_jobs, size_t row,
                                 float* __restrict__ out) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
         i < static_cast<size_t>(n_jobs) * row; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int j = static_cast<int>(i / row);
        const size_t e = i % row;
        float s = 0.0f;
        for (int k = map_off[j]; k < map_off[j + 1]; ++k) s += image[map[k] * row + e];
        out[i] = s;
    }
}

// ----------------------------------------------------------------------------- CG (LSM)

// out += <a, b> accumulated in FP64 (one atomic per block).
__global__ void dot_kernel(const float* __restrict__ a, const float* __restrict__ b, size_t n,
                           double* out) {
    __shared__ double ws[32];
    double s = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        s += static_cast<double>(a[i]) * static_cast<double>(b[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(out, s);
    }
}

// CG scalars, FP64, on the device.  sc: [0] gamma, [1] delta = <q,q>, [2] gamma_new,
// [3] alpha, [4] beta.
__global__ void cg_alpha_kernel(double* sc) {
    sc[3] = sc[1] > 0.0 ? sc[0] / sc[1] : 0.0;
}
__global__ void cg_beta_kernel(double* sc) {
    sc[4] = sc[0] > 0.0 ? sc[2] / sc[0] : 0.0;
    sc[0] = sc[2];
}

// m += alpha p (image space) and r -= alpha q (data space), alpha = sc[3].
__global__ void cg_update_kernel(float* __restrict__ m, const float* __restrict__ p, size_t nm,
                                 float* __restrict__ r, const float* __restrict__ q, size_t nr,
                                 const double* sc) {
    const float alpha = static_cast<float>(sc[3]);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < nm + nr;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        if (i < nm)
            m[i] = fmaf(alpha, p[i], m[i]);
        else
            r[i - nm] = fmaf(-alpha, q[i - nm], r[i - nm]);
    }
}

// p = s + beta p, beta = sc[4].
__global__ void cg_direction_kernel(float* __restrict__ p, const float* __restrict__ s,
                                    size_t n, const double* sc) {
    const float beta = static_cast<float>(sc[4]);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        p[i] = fmaf(beta, p[i], s[i]);
}

}  // namespace psm
